// pd_math.cuh — per-element math of the PD local step and its adjoint, for
// one thread per element (templated on the arithmetic type: double for the
// plain form, float for the mixed form).
//
// Corotated projection (diff_fem sim/fem/Constraint/CorotateFEMConstraint.h:354-377):
//   F = Ds * invDm;  SVD F = U S V^T (S >= 0, like Eigen::JacobiSVD);
//   md = R = U V^T, with column 2 negated when det F < 0;
//   md_volume = U diag(S + D) V^T, D from 5 Newton steps projecting S onto prod = 1.
// R and U diag(g(S)) V^T do not depend on the SVD's sign/ordering choices, so
// the result equals the reference's for any exact SVD.  The SVD here is the
// one-sided (Hestenes) Jacobi method: rotate column pairs of F until they are
// orthogonal; singular values are the column norms.
#pragma once
#include <cuda_runtime.h>

namespace dfem {

template <typename T> struct Vec3 { T x, y, z; };
template <typename T> __device__ __forceinline__ Vec3<T> mk3(T a, T b, T c) { return {a, b, c}; }
template <typename T> __device__ __forceinline__ Vec3<T> operator+(Vec3<T> a, Vec3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> __device__ __forceinline__ Vec3<T> operator-(Vec3<T> a, Vec3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> __device__ __forceinline__ Vec3<T> operator*(T s, Vec3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T> __device__ __forceinline__ T dot3(Vec3<T> a, Vec3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> __device__ __forceinline__ Vec3<T> cross3(Vec3<T> a, Vec3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

template <typename T> __device__ __forceinline__ T dsqrt(T v);
template <> __device__ __forceinline__ double dsqrt<double>(double v) { return sqrt(v); }
template <> __device__ __forceinline__ float dsqrt<float>(float v) { return sqrtf(v); }
template <typename T> __device__ __forceinline__ T drsqrt(T v);
template <> __device__ __forceinline__ double drsqrt<double>(double v) { return rsqrt(v); }
template <> __device__ __forceinline__ float drsqrt<float>(float v) { return rsqrtf(v); }
template <typename T> __device__ __forceinline__ T dabs(T v) { return v < T(0) ? -v : v; }

template <typename T> struct Eps;
template <> struct Eps<double> { static constexpr double rot = 1e-15; static constexpr double rel = 1e-14; static constexpr int sweeps = 10; };
template <> struct Eps<float> { static constexpr float rot = 1e-7f; static constexpr float rel = 1e-6f; static constexpr int sweeps = 6; };

// 3x3 matrices as three column vectors c[0..2]
template <typename T> struct Mat3 { Vec3<T> c[3]; };

template <typename T> __device__ __forceinline__ T det3(const Mat3<T>& a) { return dot3(a.c[0], cross3(a.c[1], a.c[2])); }

template <typename T> struct Svd3 {
  Vec3<T> u[3], v[3];  // columns of U and V
  T s[3];              // singular values (>= 0), unsorted
};

template <typename T>
__device__ __forceinline__ void jacobi_rotate(Vec3<T>& bp, Vec3<T>& bq, Vec3<T>& vp, Vec3<T>& vq, bool& rotated) {
  T a = dot3(bp, bp), b = dot3(bq, bq), g = dot3(bp, bq);
  if (!(dabs(g) > Eps<T>::rot * dsqrt(a * b))) return;
  rotated = true;
  T zeta = (b - a) / (T(2) * g);
  T t = (zeta >= T(0) ? T(1) : T(-1)) / (dabs(zeta) + dsqrt(T(1) + zeta * zeta));
  T c = drsqrt(T(1) + t * t);
  T s = c * t;
  Vec3<T> nbp = c * bp - s * bq, nbq = s * bp + c * bq;
  Vec3<T> nvp = c * vp - s * vq, nvq = s * vp + c * vq;
  bp = nbp; bq = nbq; vp = nvp; vq = nvq;
}

template <typename T>
__device__ __forceinline__ Svd3<T> svd3(const Mat3<T>& F) {
  Svd3<T> o;
  Vec3<T> b0 = F.c[0], b1 = F.c[1], b2 = F.c[2];
  Vec3<T> v0 = mk3<T>(1, 0, 0), v1 = mk3<T>(0, 1, 0), v2 = mk3<T>(0, 0, 1);
#pragma unroll 1
  for (int sweep = 0; sweep < Eps<T>::sweeps; ++sweep) {
    bool rotated = false;
    jacobi_rotate(b0, b1, v0, v1, rotated);
    jacobi_rotate(b0, b2, v0, v2, rotated);
    jacobi_rotate(b1, b2, v1, v2, rotated);
    if (!rotated) break;
  }
  T s0 = dsqrt(dot3(b0, b0)), s1 = dsqrt(dot3(b1, b1)), s2 = dsqrt(dot3(b2, b2));
  // sort descending (keeps the degenerate-completion rule simple)
  if (s0 < s1) { T t = s0; s0 = s1; s1 = t; Vec3<T> tb = b0; b0 = b1; b1 = tb; Vec3<T> tv = v0; v0 = v1; v1 = tv; }
  if (s0 < s2) { T t = s0; s0 = s2; s2 = t; Vec3<T> tb = b0; b0 = b2; b2 = tb; Vec3<T> tv = v0; v0 = v2; v2 = tv; }
  if (s1 < s2) { T t = s1; s1 = s2; s2 = t; Vec3<T> tb = b1; b1 = b2; b2 = tb; Vec3<T> tv = v1; v1 = v2; v2 = tv; }
  o.s[0] = s0; o.s[1] = s1; o.s[2] = s2;
  o.v[0] = v0; o.v[1] = v1; o.v[2] = v2;
  const T tiny = Eps<T>::rel * s0;
  if (s0 > T(0)) o.u[0] = (T(1) / s0) * b0; else o.u[0] = mk3<T>(1, 0, 0);
  if (s1 > tiny) {
    o.u[1] = (T(1) / s1) * b1;
  } else {  // complete the basis: a direction orthogonal to u0
    Vec3<T> e = dabs(o.u[0].x) < T(0.9) ? mk3<T>(1, 0, 0) : mk3<T>(0, 1, 0);
    Vec3<T> w = cross3(o.u[0], e);
    o.u[1] = drsqrt(dot3(w, w)) * w;
  }
  if (s2 > tiny) o.u[2] = (T(1) / s2) * b2;
  else o.u[2] = cross3(o.u[0], o.u[1]);
  return o;
}

// Newton projection of S onto prod(S + D) = 1 (5 iterations, CorotateFEMConstraint.h:366-374).
template <typename T>
__device__ __forceinline__ void volume_projection(const T s[3], T g[3]) {
  T D0 = 0, D1 = 0, D2 = 0;
#pragma unroll
  for (int it = 0; it < 5; ++it) {
    T p0 = s[0] + D0, p1 = s[1] + D1, p2 = s[2] + D2;
    T C = p0 * p1 * p2 - T(1);
    T g0 = p1 * p2, g1 = p0 * p2, g2 = p0 * p1;
    T c = (g0 * D0 + g1 * D1 + g2 * D2 - C) / (g0 * g0 + g1 * g1 + g2 * g2);
    D0 = c * g0; D1 = c * g1; D2 = c * g2;
  }
  g[0] = s[0] + D0; g[1] = s[1] + D1; g[2] = s[2] + D2;
}

// Same projection with its derivatives for the adjoint:
//   J[i][k] = d g_i / d s_k (forward mode through the 5 iterations),
//   dd[q]   = (g_i - g_j) / (s_i - s_j) for the pairs (0,1), (0,2), (1,2), computed
//             by the exact recurrence r <- 1 - c * p_k * r (no cancellation, valid
//             for equal singular values too).
template <typename T>
__device__ __forceinline__ void volume_projection_d(const T s[3], T g[3], T J[3][3], T dd[3]) {
  T D[3] = {0, 0, 0};
  T dD[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  T r0 = 1, r1 = 1, r2 = 1;
#pragma unroll 1
  for (int it = 0; it < 5; ++it) {
    T p[3] = {s[0] + D[0], s[1] + D[1], s[2] + D[2]};
    T C = p[0] * p[1] * p[2] - T(1);
    T gr[3] = {p[1] * p[2], p[0] * p[2], p[0] * p[1]};
    T gg = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
    T num = gr[0] * D[0] + gr[1] * D[1] + gr[2] * D[2] - C;
    T c = num / gg;
    r0 = T(1) - c * p[2] * r0;
    r1 = T(1) - c * p[1] * r1;
    r2 = T(1) - c * p[0] * r2;
    T nD[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      T dp[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) dp[i] = (i == k ? T(1) : T(0)) + dD[i][k];
      T dC = gr[0] * dp[0] + gr[1] * dp[1] + gr[2] * dp[2];
      T dg0 = dp[1] * p[2] + p[1] * dp[2], dg1 = dp[0] * p[2] + p[0] * dp[2], dg2 = dp[0] * p[1] + p[0] * dp[1];
      T dnum = dg0 * D[0] + dg1 * D[1] + dg2 * D[2] + gr[0] * dD[0][k] + gr[1] * dD[1][k] + gr[2] * dD[2][k] - dC;
      T dgg = T(2) * (gr[0] * dg0 + gr[1] * dg1 + gr[2] * dg2);
      T dc = (dnum * gg - num * dgg) / (gg * gg);
      nD[0][k] = dc * gr[0] + c * dg0;
      nD[1][k] = dc * gr[1] + c * dg1;
      nD[2][k] = dc * gr[2] + c * dg2;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      D[i] = c * gr[i];
#pragma unroll
      for (int k = 0; k < 3; ++k) dD[i][k] = nD[i][k];
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    g[i] = s[i] + D[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) J[i][k] = (i == k ? T(1) : T(0)) + dD[i][k];
  }
  dd[0] = r0; dd[1] = r1; dd[2] = r2;
}

// md (reflected rotation) and md_volume of the corotated constraint, from the
// SVD of F (corot_project computes it; the adjoint shares one SVD between the
// projection and its VJP)
template <typename T>
__device__ __forceinline__ void corot_project_sv(const Svd3<T>& sv, const Mat3<T>& F, Mat3<T>& md, Mat3<T>& mdv,
                                                 T* s_ratio = nullptr) {
  if (s_ratio) {  // smallest / largest singular value (conditioning of the element)
    T smax = sv.s[0] > sv.s[1] ? (sv.s[0] > sv.s[2] ? sv.s[0] : sv.s[2]) : (sv.s[1] > sv.s[2] ? sv.s[1] : sv.s[2]);
    T smin = sv.s[0] < sv.s[1] ? (sv.s[0] < sv.s[2] ? sv.s[0] : sv.s[2]) : (sv.s[1] < sv.s[2] ? sv.s[1] : sv.s[2]);
    *s_ratio = smax > T(0) ? smin / smax : T(0);
  }
  T g[3];
  volume_projection(sv.s, g);
  // R = sum_i u_i v_i^T ; G = sum_i g_i u_i v_i^T   (column j of u v^T is v[j] * u)
  const T vj[3][3] = {{sv.v[0].x, sv.v[1].x, sv.v[2].x}, {sv.v[0].y, sv.v[1].y, sv.v[2].y}, {sv.v[0].z, sv.v[1].z, sv.v[2].z}};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    md.c[j] = vj[j][0] * sv.u[0] + vj[j][1] * sv.u[1] + vj[j][2] * sv.u[2];
    mdv.c[j] = (g[0] * vj[j][0]) * sv.u[0] + (g[1] * vj[j][1]) * sv.u[1] + (g[2] * vj[j][2]) * sv.u[2];
  }
  if (det3(F) < T(0)) md.c[2] = T(-1) * md.c[2];
}

template <typename T>
__device__ __forceinline__ void corot_project(const Mat3<T>& F, Mat3<T>& md, Mat3<T>& mdv, T* s_ratio = nullptr) {
  const Svd3<T> sv = svd3(F);
  corot_project_sv(sv, F, md, mdv, s_ratio);
}

// Near-degenerate test for the mixed form: an element whose smallest singular
// value is below kDegenerateRatio of its largest (nearly flat or inverted)
// has a badly conditioned U/V in FP32 and is recomputed in FP64.
constexpr float kDegenerateRatio = 0.05f;

// Unit quaternion (w, x, y, z) of a nearly orthogonal matrix with det > 0
// (Shepperd's method: the branch on the largest of trace and diagonal keeps
// the square root away from cancellation).
__device__ __forceinline__ void quat_from_rot(const Mat3<float>& R, float q[4]) {
  const float m00 = R.c[0].x, m11 = R.c[1].y, m22 = R.c[2].z;
  const float m01 = R.c[1].x, m10 = R.c[0].y, m02 = R.c[2].x, m20 = R.c[0].z, m12 = R.c[2].y, m21 = R.c[1].z;
  const float tr = m00 + m11 + m22;
  if (tr > 0.0f) {
    const float S = 2.0f * sqrtf(tr + 1.0f);
    q[0] = 0.25f * S; q[1] = (m21 - m12) / S; q[2] = (m02 - m20) / S; q[3] = (m10 - m01) / S;
  } else if (m00 > m11 && m00 > m22) {
    const float S = 2.0f * sqrtf(fmaxf(1.0f + m00 - m11 - m22, 1e-30f));
    q[0] = (m21 - m12) / S; q[1] = 0.25f * S; q[2] = (m01 + m10) / S; q[3] = (m02 + m20) / S;
  } else if (m11 > m22) {
    const float S = 2.0f * sqrtf(fmaxf(1.0f + m11 - m00 - m22, 1e-30f));
    q[0] = (m02 - m20) / S; q[1] = (m01 + m10) / S; q[2] = 0.25f * S; q[3] = (m12 + m21) / S;
  } else {
    const float S = 2.0f * sqrtf(fmaxf(1.0f + m22 - m00 - m11, 1e-30f));
    q[0] = (m10 - m01) / S; q[1] = (m02 + m20) / S; q[2] = (m12 + m21) / S; q[3] = 0.25f * S;
  }
}

// The rotation of quaternion q, normalised and evaluated in FP64: orthogonal
// to FP64 round-off whatever the FP32 rounding of q.
__device__ __forceinline__ Mat3<double> rot_from_quat(const float qf[4]) {
  double w = qf[0], x = qf[1], y = qf[2], z = qf[3];
  const double n = rsqrt(w * w + x * x + y * y + z * z);
  w *= n; x *= n; y *= n; z *= n;
  Mat3<double> R;
  R.c[0] = mk3(1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y + w * z), 2.0 * (x * z - w * y));
  R.c[1] = mk3(2.0 * (x * y - w * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z + w * x));
  R.c[2] = mk3(2.0 * (x * z + w * y), 2.0 * (y * z - w * x), 1.0 - 2.0 * (x * x + y * y));
  return R;
}

// Mixed-form corotated deviations DR = md - F and DV = md_volume - F (columns;
// the tet's J d - L x is G (wr DR + wv DV)).  Only the SVD runs in FP32; its
// error enters the deviations at second order:
//   1. FP32 SVD of F -> R0 = U V^T, its quaternion, and R = R(q) exactly
//      orthogonal in FP64;
//   2. A = R^T F, H = A - I in FP64 (strain-sized; its skew part is only
//      R0's rounding);
//   3. polar of A = (I + Omega) S_A to first order in the tiny skew part, in
//      the V basis: Omega_kl = 2 (V^T skew(H) V)_kl / (s_k + s_l);
//   4. md - F = R (Omega - H);  the volume projection's 5 Newton steps run on
//      e_k = v_k^T sym(H) v_k (= s_k - 1 to second order) with
//      prod(1 + a) - 1 expanded, and md_volume - F = R V diag(D) V^T.
// Steps 2-4 are FP64 arithmetic on the FP32 singular vectors (the one FP32
// rounding of the force is then the caller's store into its slots).
// Returns false (caller takes the full FP64 branch) for inverted or
// near-degenerate elements.
__device__ __forceinline__ bool corot_delta_mixed(const Mat3<double>& F, Vec3<double> DR[3], Vec3<double> DV[3]) {
  Mat3<float> Ff;
#pragma unroll
  for (int j = 0; j < 3; ++j) Ff.c[j] = mk3((float)F.c[j].x, (float)F.c[j].y, (float)F.c[j].z);
  const Svd3<float> sv = svd3(Ff);
  const float smax = fmaxf(sv.s[0], fmaxf(sv.s[1], sv.s[2]));
  const float smin = fminf(sv.s[0], fminf(sv.s[1], sv.s[2]));
  if (!(smax > 0.0f) || !(smin >= kDegenerateRatio * smax) || !(det3(F) > 0.0)) return false;
  const float vjf[3][3] = {{sv.v[0].x, sv.v[1].x, sv.v[2].x}, {sv.v[0].y, sv.v[1].y, sv.v[2].y},
                           {sv.v[0].z, sv.v[1].z, sv.v[2].z}};
  Mat3<float> R0;
#pragma unroll
  for (int j = 0; j < 3; ++j) R0.c[j] = vjf[j][0] * sv.u[0] + vjf[j][1] * sv.u[1] + vjf[j][2] * sv.u[2];
  float q[4];
  quat_from_rot(R0, q);
  const Mat3<double> R = rot_from_quat(q);
  Vec3<double> v[3];  // the FP32 right singular vectors, widened
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = mk3((double)sv.v[k].x, (double)sv.v[k].y, (double)sv.v[k].z);
  double H[3][3];  // H[i][j] = (R^T F - I)_ij
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) H[i][j] = dot3(R.c[i], F.c[j]) - (i == j ? 1.0 : 0.0);
  Vec3<double> Hvl[3], HTvl[3];  // H v_l and H^T v_l
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    const Vec3<double> w = v[l];
    Hvl[l] = mk3(H[0][0] * w.x + H[0][1] * w.y + H[0][2] * w.z, H[1][0] * w.x + H[1][1] * w.y + H[1][2] * w.z,
                 H[2][0] * w.x + H[2][1] * w.y + H[2][2] * w.z);
    HTvl[l] = mk3(H[0][0] * w.x + H[1][0] * w.y + H[2][0] * w.z, H[0][1] * w.x + H[1][1] * w.y + H[2][1] * w.z,
                  H[0][2] * w.x + H[1][2] * w.y + H[2][2] * w.z);
  }
  double e[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) e[k] = dot3(v[k], Hvl[k]);  // v^T H v = v^T sym(H) v
  // Omega in the V basis (pairs 01, 02, 12); Omega = sum_{k<l} om_kl (v_k v_l^T - v_l v_k^T)
  const int pk[3] = {0, 0, 1}, pl[3] = {1, 2, 2};
  double om[3];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const int k = pk[p], l = pl[p];
    const double kskew = 0.5 * (dot3(v[k], Hvl[l]) - dot3(v[k], HTvl[l]));  // v_k^T skew(H) v_l
    om[p] = 2.0 * kskew / ((double)sv.s[k] + (double)sv.s[l]);
  }
  // volume projection on the small quantities (same iterates as on s + D)
  double D[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int it = 0; it < 5; ++it) {
    const double a0 = e[0] + D[0], a1 = e[1] + D[1], a2 = e[2] + D[2];
    const double C = (a0 + a1 + a2) + (a0 * a1 + a0 * a2 + a1 * a2) + a0 * a1 * a2;
    const double g0 = 1.0 + a1 + a2 + a1 * a2, g1 = 1.0 + a0 + a2 + a0 * a2, g2 = 1.0 + a0 + a1 + a0 * a1;
    const double c = (g0 * D[0] + g1 * D[1] + g2 * D[2] - C) / (g0 * g0 + g1 * g1 + g2 * g2);
    D[0] = c * g0; D[1] = c * g1; D[2] = c * g2;
  }
  // md - F = R (Omega - H), md_volume - F = R V diag(D) V^T
  const double vj[3][3] = {{v[0].x, v[1].x, v[2].x}, {v[0].y, v[1].y, v[2].y}, {v[0].z, v[1].z, v[2].z}};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    Vec3<double> col = mk3(-H[0][j], -H[1][j], -H[2][j]);
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      const int k = pk[p], l = pl[p];
      col = col + (om[p] * vj[j][l]) * v[k] - (om[p] * vj[j][k]) * v[l];
    }
    const Vec3<double> vol = (D[0] * vj[j][0]) * v[0] + (D[1] * vj[j][1]) * v[1] + (D[2] * vj[j][2]) * v[2];
    DR[j] = col.x * R.c[0] + col.y * R.c[1] + col.z * R.c[2];
    DV[j] = vol.x * R.c[0] + vol.y * R.c[1] + vol.z * R.c[2];
  }
  return true;
}

// Mixed-form corotated force P = wr (md - F) + wv (md_volume - F) (columns).
__device__ __forceinline__ bool corot_force_mixed(const Mat3<double>& F, double wr, double wv, Vec3<double> P[3]) {
  Vec3<double> DR[3], DV[3];
  if (!corot_delta_mixed(F, DR, DV)) return false;
#pragma unroll
  for (int j = 0; j < 3; ++j) P[j] = wr * DR[j] + wv * DV[j];
  return true;
}

// VJP of (md, md_volume) with respect to F.  gmd, gmdv: cotangents (3x3).
//   P_bar_ij (i != j) = a_ij sym(M_G)_ij + b_ij asym(M_G)_ij + (M_R_ij - M_R_ji)/(s_i + s_j)
//   P_bar_ii = sum_k (M_G)_kk dg_k/ds_i
//   with M_X = U^T X V, a_ij = (g_i - g_j)/(s_i - s_j), b_ij = (g_i + g_j)/(s_i + s_j);
//   F_bar = U P_bar V^T.
template <typename T>
__device__ __forceinline__ Mat3<T> corot_vjp_sv(const Svd3<T>& sv, const Mat3<T>& F, Mat3<T> gmd,
                                                const Mat3<T>& gmdv) {
  T g[3], J[3][3], dd[3];
  volume_projection_d(sv.s, g, J, dd);
  if (det3(F) < T(0)) gmd.c[2] = T(-1) * gmd.c[2];
  // M = U^T X V : M_ij = u_i . (X v_j) ; X v_j = sum_k X.c[k] * v_j[k]
  T MR[3][3], MG[3][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    Vec3<T> xr = sv.v[j].x * gmd.c[0] + sv.v[j].y * gmd.c[1] + sv.v[j].z * gmd.c[2];
    Vec3<T> xg = sv.v[j].x * gmdv.c[0] + sv.v[j].y * gmdv.c[1] + sv.v[j].z * gmdv.c[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) { MR[i][j] = dot3(sv.u[i], xr); MG[i][j] = dot3(sv.u[i], xg); }
  }
  T P[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
    P[i][i] = MG[0][0] * J[0][i] + MG[1][1] * J[1][i] + MG[2][2] * J[2][i];
  const int pi[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    int i = pi[q], j = pj[q];
    T ssum = sv.s[i] + sv.s[j];
    T b = (g[i] + g[j]) / ssum;
    T a = dd[q];
    T symG = T(0.5) * (MG[i][j] + MG[j][i]);
    T asymG = T(0.5) * (MG[i][j] - MG[j][i]);
    T asymR = (MR[i][j] - MR[j][i]) / ssum;
    P[i][j] = a * symG + b * asymG + asymR;
    P[j][i] = a * symG - b * asymG - asymR;
  }
  // F_bar = U P V^T : column c = sum_{i,j} P_ij u_i v_j[c]
  Mat3<T> out;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T vc[3] = {c == 0 ? sv.v[0].x : (c == 1 ? sv.v[0].y : sv.v[0].z),
                     c == 0 ? sv.v[1].x : (c == 1 ? sv.v[1].y : sv.v[1].z),
                     c == 0 ? sv.v[2].x : (c == 1 ? sv.v[2].y : sv.v[2].z)};
    Vec3<T> acc = mk3<T>(0, 0, 0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      T w = P[i][0] * vc[0] + P[i][1] * vc[1] + P[i][2] * vc[2];
      acc = acc + w * sv.u[i];
    }
    out.c[c] = acc;
  }
  return out;
}

template <typename T>
__device__ __forceinline__ Mat3<T> corot_vjp(const Mat3<T>& F, Mat3<T> gmd, const Mat3<T>& gmdv) {
  const Svd3<T> sv = svd3(F);
  return corot_vjp_sv(sv, F, gmd, gmdv);
}

}  // namespace dfem
