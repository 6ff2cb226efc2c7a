// drag_kernels.cuh — underwater drag and lift on surface faces
// (Environment::Step underwater branch, Dfobj::ComputeDragForces, Cd, Cl;
// sim/Environment.h:236-247, sim/Dfobj.h:803-838,904-998), and its adjoint.
//
// Per face (outward winding p1 p2 p3, vertex velocities v1 v2 v3, water at
// rest): v_rel = -(v1+v2+v3)/3 (face skipped below |v_rel| = 1e-6), u its
// direction, d = -n the inward unit normal, area = |(p2-p1) x (p3-p1)|/2,
// c = d.u; only faces with c > 0 act:
//   drag = 500 area Cd |v_rel|^2 u,  Cd(aoa) = (1 - cos 2 aoa)/2 = c^2
//          (aoa = pi/2 - acos c = asin c),
//   lift = 500 area Cl(aoa) |v_rel|^2 normalize(u x d) x u, Cl the table of
//          Dfobj::Cl in degrees (cutoff 85),
// each clipped to norm 1e3; every vertex of the face receives (drag+lift)/3
// as external force, so v_wc = v + h f / m (no gravity underwater).
//
// The adjoint evaluates the same face function on forward-mode dual numbers
// (a value and three derivatives), seeding one input vector at a time: six
// evaluations give the face's 18 input cotangents for a force cotangent.
#pragma once
#include "kernels.cuh"

namespace dfem {

struct Dual3 {
  double v, d[3];
  __device__ Dual3(double a = 0.0) : v(a) { d[0] = d[1] = d[2] = 0.0; }
};
__device__ inline double val(double a) { return a; }
__device__ inline double val(const Dual3& a) { return a.v; }
__device__ inline Dual3 operator+(const Dual3& a, const Dual3& b) {
  Dual3 r(a.v + b.v);
  for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
__device__ inline Dual3 operator-(const Dual3& a, const Dual3& b) {
  Dual3 r(a.v - b.v);
  for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
__device__ inline Dual3 operator*(const Dual3& a, const Dual3& b) {
  Dual3 r(a.v * b.v);
  for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
__device__ inline Dual3 operator/(const Dual3& a, const Dual3& b) {
  Dual3 r(a.v / b.v);
  for (int k = 0; k < 3; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
  return r;
}
__device__ inline Dual3 dsqrt(const Dual3& a) {
  Dual3 r(sqrt(a.v));
  for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] / (2.0 * r.v);
  return r;
}
__device__ inline double dsqrt(double a) { return sqrt(a); }
__device__ inline Dual3 dasin(const Dual3& a) {
  Dual3 r(asin(a.v));
  const double q = 1.0 / sqrt(1.0 - a.v * a.v);
  for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * q;
  return r;
}
__device__ inline double dasin(double a) { return asin(a); }

template <typename T>
struct DV3 {
  T x, y, z;
};
template <typename T> __device__ inline DV3<T> operator+(const DV3<T>& a, const DV3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> __device__ inline DV3<T> operator-(const DV3<T>& a, const DV3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> __device__ inline DV3<T> scale(const T& s, const DV3<T>& a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T> __device__ inline T dotp(const DV3<T>& a, const DV3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> __device__ inline DV3<T> crossp(const DV3<T>& a, const DV3<T>& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Dfobj::Cl with the table x = {-90, -10, -5, 15, 90} deg, y = {-0.5, -1.26,
// 0, 1.8, 0.5}, cutoff 85 deg: linear on the first matching segment.
template <typename T>
__device__ T lift_coefficient(const T& aoa) {
  const double xs[5] = {-90.0, -10.0, -5.0, 15.0, 90.0}, ys[5] = {-0.5, -1.26, 0.0, 1.8, 0.5};
  const T theta = T(180.0 / 3.14159265358979323846) * aoa;
  const double th = val(theta);
  if (fabs(th) > 85.0) return T(0.0);
  for (int k = 0; k < 4; ++k) {
    const bool in = k < 2 ? (xs[k] <= th && th < xs[k + 1]) : (xs[k] <= th && th <= xs[k + 1]);
    if (in) {
      const T t = T(1.0 / (xs[k + 1] - xs[k])) * (theta - T(xs[k]));
      return T(ys[k + 1] - ys[k]) * t + T(ys[k]);
    }
  }
  return T(0.0);
}

// The force a face adds to each of its three vertices.
template <typename T>
__device__ DV3<T> drag_face_force(const DV3<T>& p1, const DV3<T>& p2, const DV3<T>& p3, const DV3<T>& v1,
                                  const DV3<T>& v2, const DV3<T>& v3) {
  const DV3<T> zero{T(0.0), T(0.0), T(0.0)};
  const DV3<T> vrel = scale(T(-1.0 / 3.0), (v1 + v2) + v3);
  const T s2 = dotp(vrel, vrel);
  const T s = dsqrt(s2);
  if (val(s) < 1e-6) return zero;
  const DV3<T> u = scale(T(1.0) / s, vrel);
  const DV3<T> nv = crossp(p2 - p1, p3 - p1);
  const T an = dsqrt(dotp(nv, nv));
  const T area = T(0.5) * an;
  const DV3<T> dn = scale(T(-1.0) / an, nv);
  const T c = dotp(dn, u);
  if (!(val(c) > 0.0)) return zero;
  DV3<T> fd = scale(T(500.0) * area * (c * c) * s2, u);
  const T cl = val(c) < 1.0 ? lift_coefficient(dasin(c)) : T(0.0);  // c >= 1 (rounding) is past the cutoff
  const DV3<T> w = crossp(u, dn);
  const T wn2 = dotp(w, w);
  DV3<T> fl = zero;
  if (val(wn2) > 0.0) fl = scale(T(500.0) * area * cl * s2, crossp(scale(T(1.0) / dsqrt(wn2), w), u));
  const double fmax = 1.0e3;
  const T fdn = dsqrt(dotp(fd, fd)), fln = dsqrt(dotp(fl, fl));
  if (val(fdn) > fmax) fd = scale(T(fmax) / fdn, fd);
  if (val(fln) > fmax) fl = scale(T(fmax) / fln, fl);
  return scale(T(1.0 / 3.0), fd + fl);
}

__device__ inline DV3<double> ldv(const double* a, int i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }

// fface[3 f ..] = the force face f adds to each of its vertices.
__global__ void k_drag_faces(int F, const int* __restrict__ df, const double* __restrict__ x,
                             const double* __restrict__ v, double* __restrict__ fface) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const int a = df[3 * f], b = df[3 * f + 1], c = df[3 * f + 2];
  const DV3<double> g = drag_face_force(ldv(x, a), ldv(x, b), ldv(x, c), ldv(v, a), ldv(v, b), ldv(v, c));
  fface[3 * f] = g.x; fface[3 * f + 1] = g.y; fface[3 * f + 2] = g.z;
}

// Adjoint, per face: with vwcb the cotangent of v_wc, the face's force
// cotangent is sum over its vertices of h / m vwcb; writes the cotangents of
// its (p1 p2 p3 v1 v2 v3) to fbar[18 f ..].
__global__ void k_drag_adj_faces(int F, const int* __restrict__ df, const double* __restrict__ mass, double h,
                                 const double* __restrict__ x, const double* __restrict__ v,
                                 const double* __restrict__ vwcb, double* __restrict__ fbar) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const int vi[3] = {df[3 * f], df[3 * f + 1], df[3 * f + 2]};
  double gb[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < 3; ++k) {
    const double w = h / mass[vi[k]];
    for (int c = 0; c < 3; ++c) gb[c] += w * vwcb[3 * vi[k] + c];
  }
  for (int q = 0; q < 6; ++q) {
    DV3<Dual3> in[6];
    for (int j = 0; j < 6; ++j) {
      const double* src = j < 3 ? x : v;
      const int i = vi[j % 3];
      in[j] = {Dual3(src[3 * i]), Dual3(src[3 * i + 1]), Dual3(src[3 * i + 2])};
    }
    in[q].x.d[0] = 1.0; in[q].y.d[1] = 1.0; in[q].z.d[2] = 1.0;
    const DV3<Dual3> g = drag_face_force(in[0], in[1], in[2], in[3], in[4], in[5]);
    for (int k = 0; k < 3; ++k) fbar[18 * (size_t)f + 3 * q + k] = gb[0] * g.x.d[k] + gb[1] * g.y.d[k] + gb[2] * g.z.d[k];
  }
}

// Adjoint, per vertex: add its corners' cotangents (faces in ascending order)
// to the step input's cotangents gx (x) and gv (v).
__global__ void k_drag_adj_gather(int N, const int* __restrict__ vf_ptr, const int* __restrict__ vf_face,
                                  const double* __restrict__ fbar, double* gx, double* gv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  Vec3<double> ax = ld3(gx, i), av = ld3(gv, i);
  for (int k = vf_ptr[i]; k < vf_ptr[i + 1]; ++k) {
    const int e = vf_face[k], f = e / 3, corner = e % 3;
    const double* b = fbar + 18 * (size_t)f;
    ax = ax + mk3(b[3 * corner], b[3 * corner + 1], b[3 * corner + 2]);
    av = av + mk3(b[9 + 3 * corner], b[9 + 3 * corner + 1], b[9 + 3 * corner + 2]);
  }
  st3(gx, i, ax);
  st3(gv, i, av);
}

}  // namespace dfem
