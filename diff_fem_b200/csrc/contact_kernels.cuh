// contact_kernels.cuh — obstacle contact phase of a PD step on the GPU.
//
// After the local-global iterations, diff_fem (sim/fem/World.h:925-1023)
// alternates (1) continuous collision detection of the soft surface vertices
// against the static obstacle triangles (arcsim vertex-face test,
// sim/utils/arcsim/collision.cpp:127-326) and (2) up to K Jacobi iterations of
// the global step in velocity form, whose right-hand side at contact vertices
// is replaced by the Coulomb-cone reaction (CollisionHandling, World.h:1317-1430).
// The loop ends when a detection pass finds no impact.  Here the phase is one
// conditional WHILE graph node driven by a device-side state machine
//   state = [mode (0 detect, 1 Jacobi), pass, it, any, active]
// whose body runs at most max_passes * (K + 2) + 1 times.
#pragma once
#include <cooperative_groups.h>

#include "kernels.cuh"

namespace dfem {

// state words: [mode, pass, it, any, active, loop-body executions, computed
// Jacobi iterations, the computed iteration whose x_n1 the current ori_x is,
// obstacle impacts in the lists, self groups of this pass, of the last pass]
enum { CS_MODE = 0, CS_PASS = 1, CS_IT = 2, CS_ANY = 3, CS_ACTIVE = 4, CS_BODIES = 5, CS_COMP = 6, CS_SRC = 7,
       CS_NOBS = 8, CS_NGRP = 9, CS_NGRP_PREV = 10, CS_FANY0 = 11, CS_FANY1 = 12, CS_SIZE = 13 };

// per-step record of the phase: [passes, loop-body executions]; while the
// forward steps record their contact iterations, the step's place in the
// record (the next step's records follow it when it fit)
__global__ void k_contact_record(const int* step, const int* state, int* rec, ContactDev c) {
  const int s = *step;
  rec[2 * s] = state[CS_PASS];
  rec[2 * s + 1] = state[CS_BODIES];
  if (c.rec_on && *c.rec_on == 2) {
    const int base = *c.rec_base, comp = state[CS_COMP];
    const int ok = base + comp <= c.rec_fwd_cap ? 1 : 0;
    int* m = c.rec_meta + 4 * (size_t)s;
    m[0] = base; m[1] = comp; m[2] = state[CS_SRC]; m[3] = ok;
    if (ok) *c.rec_base = base + comp;
  }
}

// A cap was reached: status[0] = DFEM_ERR_CAP, status[2] = which (kCap*); the
// first error of the call is the one reported.
__device__ __forceinline__ void cap_reached(int* status, int which) {
  if (atomicCAS(status, 0, 6) == 0) atomicExch(status + 2, which);
}

// record index of the current computed iteration (-1: not recording or no room)
__device__ __forceinline__ int rec_index(const ContactDev& c) {
  if (!c.rec_on || *c.rec_on == 0) return -1;
  const int k = *c.rec_base + c.state[CS_COMP];
  return k < c.rec_cap ? k : -1;
}

// ---- vertex-face CCD (one vertex moving p0 -> p1, static face q0 q1 q2) ----

__device__ __forceinline__ double stp3(Vec3<double> u, Vec3<double> v, Vec3<double> w) { return dot3(u, cross3(v, w)); }
__device__ __forceinline__ Vec3<double> unit3(Vec3<double> a) { return (1.0 / sqrt(dot3(a, a))) * a; }
__device__ __forceinline__ double sgn1(double x) { return x < 0 ? -1.0 : 1.0; }

__device__ int ccd_quadratic(double a, double b, double c, double x[2]) {
  double d = b * b - 4 * a * c;
  if (d < 0) { x[0] = -b / (2 * a); return 0; }
  double q = -(b + sgn1(b) * sqrt(d)) / 2;
  int i = 0;
  if (fabs(a) > 1e-12 * fabs(q)) x[i++] = q / a;
  if (fabs(q) > 1e-12 * fabs(c)) x[i++] = c / q;
  if (i == 2 && x[0] > x[1]) { double t = x[0]; x[0] = x[1]; x[1] = t; }
  return i;
}

__device__ double ccd_newton(double a, double b, double c, double d, double x0, int init_dir) {
  if (init_dir != 0) {
    double y0 = d + x0 * (c + x0 * (b + x0 * a)), ddy0 = 2 * b + x0 * (6 * a);
    x0 += init_dir * sqrt(fabs(2 * y0 / ddy0));
  }
  for (int iter = 0; iter < 100; ++iter) {  // bounded like the reference's
    double y = d + x0 * (c + x0 * (b + x0 * a));
    double dy = c + x0 * (2 * b + x0 * 3 * a);
    if (dy == 0) return x0;
    double x1 = x0 - y / dy;
    if (fabs(x0 - x1) < 1e-6) return x0;
    x0 = x1;
  }
  return x0;
}

__device__ int ccd_cubic(double a, double b, double c, double d, double x[3]) {
  // start Newton's method at 0 when the quadratic helper finds no root (the
  // reference leaves that start uninitialised)
  double xc[2] = {0.0, 0.0};
  int ncrit = ccd_quadratic(3 * a, 2 * b, c, xc);
  if (ncrit == 0) { x[0] = ccd_newton(a, b, c, d, xc[0], 0); return 1; }
  if (ncrit == 1) return ccd_quadratic(b, c, d, x);
  double yc0 = d + xc[0] * (c + xc[0] * (b + xc[0] * a)), yc1 = d + xc[1] * (c + xc[1] * (b + xc[1] * a));
  int i = 0;
  if (yc0 * a >= 0) x[i++] = ccd_newton(a, b, c, d, xc[0], -1);
  if (yc0 * yc1 <= 0) {
    int closer = fabs(yc0) < fabs(yc1) ? 0 : 1;
    x[i++] = ccd_newton(a, b, c, d, xc[closer], closer == 0 ? 1 : -1);
  }
  if (yc1 * a <= 0) x[i++] = ccd_newton(a, b, c, d, xc[1], 1);
  return i;
}

__device__ bool vf_impact(Vec3<double> p0, Vec3<double> p1, Vec3<double> q0, Vec3<double> q1, Vec3<double> q2,
                          double mult, Vec3<double>* n_out) {
  const double thick = kContactThickness * mult;
  // swept vertex box against the face box dilated by the thickness
  if (fmax(p0.x, p1.x) < fmin(q0.x, fmin(q1.x, q2.x)) - thick || fmin(p0.x, p1.x) > fmax(q0.x, fmax(q1.x, q2.x)) + thick) return false;
  if (fmax(p0.y, p1.y) < fmin(q0.y, fmin(q1.y, q2.y)) - thick || fmin(p0.y, p1.y) > fmax(q0.y, fmax(q1.y, q2.y)) + thick) return false;
  if (fmax(p0.z, p1.z) < fmin(q0.z, fmin(q1.z, q2.z)) - thick || fmin(p0.z, p1.z) > fmax(q0.z, fmax(q1.z, q2.z)) + thick) return false;
  Vec3<double> v0 = p1 - p0;
  Vec3<double> x1 = q0 - p0, x2 = q1 - p0, x3 = q2 - p0;
  Vec3<double> v1 = (-1.0) * v0;  // static face: every face vertex moves by -v0 relative to the vertex
  double a0 = stp3(x1, x2, x3);
  double a1 = stp3(v1, x2, x3) + stp3(x1, v1, x3) + stp3(x1, x2, v1);
  double a2 = stp3(x1, v1, v1) + stp3(v1, x2, v1) + stp3(v1, v1, x3);
  double a3 = stp3(v1, v1, v1);
  double t[4];
  int nsol = ccd_cubic(a3, a2, a1, a0, t);
  t[nsol++] = 1;
  for (int i = 0; i < nsol; ++i) {
    if (t[i] < 0 || t[i] > 1) continue;
    Vec3<double> xt = p0 + t[i] * v0;
    // signed distance to the face plane and barycentric weights
    Vec3<double> n = cross3(unit3(q1 - q0), unit3(q2 - q0));
    double d, w1, w2, w3;
    if (dot3(n, n) < 1e-6) {
      d = INFINITY; w1 = w2 = w3 = 0.0;
    } else {
      n = unit3(n);
      d = dot3(xt - q0, n);
      double b0 = stp3(q1 - xt, q2 - xt, n), b1 = stp3(q2 - xt, q0 - xt, n), b2 = stp3(q0 - xt, q1 - xt, n);
      double sb = b0 + b1 + b2;
      w1 = -b0 / sb; w2 = -b1 / sb; w3 = -b2 / sb;
    }
    bool inside = fmin(fmin(-w1, -w2), -w3) >= -1e-6;
    if (t[i] == 1) {
      inside = inside || sqrt(dot3(xt - q0, xt - q0)) < thick || sqrt(dot3(xt - q1, xt - q1)) < thick ||
               sqrt(dot3(xt - q2, xt - q2)) < thick;
      Vec3<double> e;
      e = xt - q0 - (dot3(xt - q0, q1 - q0) / dot3(q1 - q0, q1 - q0)) * (q1 - q0);
      inside = inside || sqrt(dot3(e, e)) < thick;
      e = xt - q1 - (dot3(xt - q1, q2 - q1) / dot3(q2 - q1, q2 - q1)) * (q2 - q1);
      inside = inside || sqrt(dot3(e, e)) < thick;
      e = xt - q2 - (dot3(xt - q2, q0 - q2) / dot3(q0 - q2, q0 - q2)) * (q0 - q2);
      inside = inside || sqrt(dot3(e, e)) < thick;
    }
    Vec3<double> fn = cross3(unit3(q1 - q0), unit3(q2 - q0));
    if (dot3(n, w1 * v1 + w2 * v1 + w3 * v1) > 0) n = (-1.0) * fn; else n = fn;
    if (fabs(d) < thick && inside) { *n_out = n; return true; }
  }
  return false;
}

// contact basis [n, t, b] (CollisionBrutal::computeBasis)
// Vertex (p0 -> p1) against a moving face (qs -> qe): arcsim's vf_collision_test
// + collision_test (sim/utils/arcsim/collision.cpp:118-128, 211-274) with the
// swept boxes of the vertex and the face dilated by thickness * mult.  On an
// impact returns its time t, distance |d| and normal (the face's start normal,
// against the vertex's approach; not unit length).
__device__ bool vf_impact_moving(Vec3<double> p0, Vec3<double> p1, const Vec3<double> qs[3], const Vec3<double> qe[3],
                                 double mult, Vec3<double>* n_out, double* t_out, double* d_out) {
  const double thick = kContactThickness * mult;
  {
    const double plo[3] = {fmin(p0.x, p1.x), fmin(p0.y, p1.y), fmin(p0.z, p1.z)};
    const double phi[3] = {fmax(p0.x, p1.x), fmax(p0.y, p1.y), fmax(p0.z, p1.z)};
    double flo[3] = {1e300, 1e300, 1e300}, fhi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < 3; ++k) {
      flo[0] = fmin(flo[0], fmin(qs[k].x, qe[k].x)); fhi[0] = fmax(fhi[0], fmax(qs[k].x, qe[k].x));
      flo[1] = fmin(flo[1], fmin(qs[k].y, qe[k].y)); fhi[1] = fmax(fhi[1], fmax(qs[k].y, qe[k].y));
      flo[2] = fmin(flo[2], fmin(qs[k].z, qe[k].z)); fhi[2] = fmax(fhi[2], fmax(qs[k].z, qe[k].z));
    }
    for (int c = 0; c < 3; ++c)
      if (phi[c] < flo[c] - thick || plo[c] > fhi[c] + thick) return false;
  }
  const Vec3<double> v0 = p1 - p0;
  const Vec3<double> x1 = qs[0] - p0, x2 = qs[1] - p0, x3 = qs[2] - p0;
  const Vec3<double> v1 = (qe[0] - qs[0]) - v0, v2 = (qe[1] - qs[1]) - v0, v3 = (qe[2] - qs[2]) - v0;
  const double a0 = stp3(x1, x2, x3);
  const double a1 = stp3(v1, x2, x3) + stp3(x1, v2, x3) + stp3(x1, x2, v3);
  const double a2 = stp3(x1, v2, v3) + stp3(v1, x2, v3) + stp3(v1, v2, x3);
  const double a3 = stp3(v1, v2, v3);
  double t[4];
  int nsol = ccd_cubic(a3, a2, a1, a0, t);
  t[nsol++] = 1;
  for (int i = 0; i < nsol; ++i) {
    if (t[i] < 0 || t[i] > 1) continue;
    const Vec3<double> xt = p0 + t[i] * v0;
    const Vec3<double> y0 = qs[0] + t[i] * (qe[0] - qs[0]), y1 = qs[1] + t[i] * (qe[1] - qs[1]),
                       y2 = qs[2] + t[i] * (qe[2] - qs[2]);
    Vec3<double> n = cross3(unit3(y1 - y0), unit3(y2 - y0));
    double d, w1, w2, w3;
    if (dot3(n, n) < 1e-6) {
      d = INFINITY; w1 = w2 = w3 = 0.0;
    } else {
      n = unit3(n);
      d = dot3(xt - y0, n);
      const double b0 = stp3(y1 - xt, y2 - xt, n), b1 = stp3(y2 - xt, y0 - xt, n), b2 = stp3(y0 - xt, y1 - xt, n);
      const double sb = b0 + b1 + b2;
      w1 = -b0 / sb; w2 = -b1 / sb; w3 = -b2 / sb;
    }
    bool inside = fmin(fmin(-w1, -w2), -w3) >= -1e-6;
    if (t[i] == 1) {
      inside = inside || sqrt(dot3(xt - y0, xt - y0)) < thick || sqrt(dot3(xt - y1, xt - y1)) < thick ||
               sqrt(dot3(xt - y2, xt - y2)) < thick;
      Vec3<double> e;
      e = xt - y0 - (dot3(xt - y0, y1 - y0) / dot3(y1 - y0, y1 - y0)) * (y1 - y0);
      inside = inside || sqrt(dot3(e, e)) < thick;
      e = xt - y1 - (dot3(xt - y1, y2 - y1) / dot3(y2 - y1, y2 - y1)) * (y2 - y1);
      inside = inside || sqrt(dot3(e, e)) < thick;
      e = xt - y2 - (dot3(xt - y2, y0 - y2) / dot3(y0 - y2, y0 - y2)) * (y0 - y2);
      inside = inside || sqrt(dot3(e, e)) < thick;
    }
    const Vec3<double> fn = cross3(unit3(qs[1] - qs[0]), unit3(qs[2] - qs[0]));
    if (dot3(n, w1 * v1 + w2 * v2 + w3 * v3) > 0) n = (-1.0) * fn; else n = fn;
    if (fabs(d) < thick && inside) {
      *n_out = n; *t_out = t[i]; *d_out = fabs(d);
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ void contact_basis(Vec3<double> nrm, Vec3<double> B[3]) {
  Vec3<double> tg = cross3(nrm, mk3(1.0, 0.0, 0.0));
  if (sqrt(dot3(tg, tg)) < 1e-15) tg = cross3(nrm, mk3(0.0, 1.0, 0.0));
  tg = unit3(tg);
  B[0] = unit3(nrm); B[1] = tg; B[2] = unit3(cross3(nrm, tg));
}

// ---- phase kernels ---------------------------------------------------------------

// Before the loop: x_n1 = PD result, xold = 0, L x_t, empty impact lists.
// L x_t at vertex i (Hs x_t - M/h^2 x_t), the contact rhs's elastic term.
__device__ __forceinline__ Vec3<double> contact_lxt(const SceneDev& d, int i, const double* xt) {
  Vec3<double> acc = mk3(0.0, 0.0, 0.0);
  for (int k = d.hs_ptr[i]; k < d.hs_ptr[i + 1]; ++k) acc = acc + d.hs_val[k] * ld3(xt, d.hs_col[k]);
  return acc - (d.mass[i] / (d.h * d.h)) * ld3(xt, i);
}

// The step inputs the contact adjoint reads (v_wc and L x_t of the step with
// start state xt, vt), for a step whose contact iterations the forward
// recorded (no replay computes them); the same arithmetic as the forward.
__global__ void k_contact_step_inputs(SceneDev d, ContactDev c, const double* xt, const double* vt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  st3(c.vwc, i, step_vwc(d, i, ld3(vt, i)));
  st3(c.lxt, i, contact_lxt(d, i, xt));
}

__device__ __forceinline__ void contact_begin_item(const SceneDev& d, const ContactDev& c, int i, const double* xt,
                                                   const double* xk) {
  if (i < d.N) {
    st3(c.xn1, i, ld3(xk, i));
    st3(c.xold, i, mk3(0.0, 0.0, 0.0));
    st3(c.lxt, i, contact_lxt(d, i, xt));
  }
  if (i < c.nc) {
    c.imp_cnt[i] = 0;
    if (c.ncf > 0) c.simp_cnt[i] = 0;
  }
}

__global__ void k_contact_begin(SceneDev d, ContactDev c, const double* xt, const double* xk,
                                cudaGraphConditionalHandle h) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  contact_begin_item(d, c, i, xt, xk);
  if (i == 0) {
    for (int k = 0; k < CS_SIZE; ++k) c.state[k] = 0;
    cudaGraphSetConditional(h, (c.nc > 0 && (c.nof > 0 || c.ncf > 0)) ? 1u : 0u);
  }
}

__device__ __forceinline__ int bp_cell(const ContactDev& c, double v, int k) {
  const double u = floor((v - c.bp_org[k]) * c.bp_inv);
  return u < 0.0 ? 0 : (u >= (double)(c.bp_dim[k] - 1) ? c.bp_dim[k] - 1 : (int)u);
}

// Candidate obstacle faces of the swept box [lo, hi] from the grid, ascending
// and without repeats; false when the box covers too many cells or gathers
// too many faces (the caller then tests every face).
__device__ __forceinline__ bool bp_candidates(const ContactDev& c, Vec3<double> lo, Vec3<double> hi, int* cand, int* ncand) {
  if (c.bp_max_cells <= 0 || c.bp_dim[0] <= 0) return false;
  const double l[3] = {lo.x - kBroadPad, lo.y - kBroadPad, lo.z - kBroadPad};
  const double h[3] = {hi.x + kBroadPad, hi.y + kBroadPad, hi.z + kBroadPad};
  int i0[3], i1[3];
  long long cells = 1;
  for (int k = 0; k < 3; ++k) {
    i0[k] = bp_cell(c, l[k], k);
    i1[k] = bp_cell(c, h[k], k);
    cells *= (long long)(i1[k] - i0[k] + 1);
  }
  if (cells > c.bp_max_cells) return false;
  int n = 0;
  for (int z = i0[2]; z <= i1[2]; ++z)
    for (int y = i0[1]; y <= i1[1]; ++y)
      for (int x = i0[0]; x <= i1[0]; ++x) {
        const int cell = (z * c.bp_dim[1] + y) * c.bp_dim[0] + x;
        for (int k = c.bp_ptr[cell]; k < c.bp_ptr[cell + 1]; ++k) {
          const int f = c.bp_face[k];
          int j = n;  // insertion into the ascending list, repeats dropped
          while (j > 0 && cand[j - 1] > f) --j;
          if (j > 0 && cand[j - 1] == f) continue;
          if (n == kBroadMaxCandidates) return false;
          for (int q = n; q > j; --q) cand[q] = cand[q - 1];
          cand[j] = f;
          ++n;
        }
      }
  *ncand = n;
  return true;
}

// Detection of contact vertex a against the obstacle faces (the broad
// phase's candidates, or all of them — in a batch, all of its part's), in
// ascending face order; true when it hit a face.
__device__ __forceinline__ bool contact_detect_item(const ContactDev& c, int a, const double* xt, const double* xk,
                                                    int* status) {
  int gv = c.cverts[a];
  Vec3<double> p0 = ld3(xt, gv), p1 = ld3(xk, gv);
  bool any = false;
  int cand[kBroadMaxCandidates];
  int ncand = 0;
  const bool culled = bp_candidates(c, mk3(fmin(p0.x, p1.x), fmin(p0.y, p1.y), fmin(p0.z, p1.z)),
                                    mk3(fmax(p0.x, p1.x), fmax(p0.y, p1.y), fmax(p0.z, p1.z)), cand, &ncand);
  const int f0 = c.np > 1 ? c.pf0[c.cpart[a]] : 0;
  const int nf = culled ? ncand : (c.np > 1 ? c.pf0[c.cpart[a] + 1] - f0 : c.nof);
  for (int k = 0; k < nf; ++k) {
    const int f = culled ? cand[k] : f0 + k;
    Vec3<double> n;
    const int* fv = c.obs_f + 3 * f;
    if (!vf_impact(p0, p1, ld3(c.obs_x, fv[0]), ld3(c.obs_x, fv[1]), ld3(c.obs_x, fv[2]), 1.0, &n)) continue;
    any = true;
    int cnt = c.imp_cnt[a], slot = -1;
    for (int q = 0; q < cnt; ++q)
      if (c.imp_face[a * kMaxImpactsPerVertex + q] == f) slot = q;
    if (slot < 0) {
      if (cnt >= c.max_impacts) { cap_reached(status, kCapImpacts); continue; }
      slot = cnt;
      c.imp_face[a * kMaxImpactsPerVertex + slot] = f;
      c.imp_cnt[a] = cnt + 1;
      atomicAdd(&c.state[CS_NOBS], 1);
    }
    st3(c.imp_n, a * kMaxImpactsPerVertex + slot, n);
  }
  return any;
}

// Detection pass (mode 0): every contact vertex.
__global__ void k_contact_detect(ContactDev c, const double* xt, const double* xk, int* status) {
  if (c.state[CS_MODE] != 0) return;
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= c.nc) return;
  if (contact_detect_item(c, a, xt, xk, status)) atomicOr(&c.state[CS_ANY], 1);
}

// Soft impacts (thickness x 2) of contact vertex a (one warp per vertex) against
// every soft face not holding it: the lanes test 32 consecutive faces, then
// lane 0 applies the hits in ascending face order (a face met again refreshes
// its entry in place, a new one is appended), as one thread looping over the
// faces would.
__global__ void k_self_detect(ContactDev c, const double* xt, const double* xk, int* status) {
  if (c.state[CS_MODE] != 0) return;
  const int lane = threadIdx.x & 31;
  const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (a >= c.nc || !c.on_face[a]) return;  // uniform over the warp
  const int gv = c.cverts[a];
  const Vec3<double> p0 = ld3(xt, gv), p1 = ld3(xk, gv);
  const int base = a * kMaxSelfImpacts;
  for (int f0 = 0; f0 < c.ncf; f0 += 32) {
    const int f = f0 + lane;
    bool hit = false;
    Vec3<double> n = mk3(0.0, 0.0, 0.0);
    double t = 0.0, dd = 0.0;
    if (f < c.ncf) {
      const int* cf = c.cfaces + 3 * f;
      if (cf[0] != a && cf[1] != a && cf[2] != a) {
        Vec3<double> qs[3], qe[3];
        for (int k = 0; k < 3; ++k) {
          const int gq = c.cverts[cf[k]];
          qs[k] = ld3(xt, gq);
          qe[k] = ld3(xk, gq);
        }
        hit = vf_impact_moving(p0, p1, qs, qe, 2.0, &n, &t, &dd);
      }
    }
    unsigned mask = __ballot_sync(0xffffffffu, hit);
    while (mask) {
      const int src = __ffs(mask) - 1;
      mask &= mask - 1;
      const double nx = __shfl_sync(0xffffffffu, n.x, src), ny = __shfl_sync(0xffffffffu, n.y, src),
                   nz = __shfl_sync(0xffffffffu, n.z, src);
      const double ts = __shfl_sync(0xffffffffu, t, src), ds = __shfl_sync(0xffffffffu, dd, src);
      if (lane == 0) {
        const int fh = f0 + src;
        int cnt = c.simp_cnt[a], slot = -1;
        for (int q = 0; q < cnt; ++q)
          if (c.simp_face[base + q] == fh) { slot = q; break; }
        if (slot < 0) {
          if (cnt >= c.max_self_impacts) {
            cap_reached(status, kCapSoftImpacts);
          } else {
            slot = cnt;
            c.simp_face[base + slot] = fh;
            c.simp_cnt[a] = cnt + 1;
          }
        }
        if (slot >= 0) {
          c.simp_td[2 * (base + slot)] = ts;
          c.simp_td[2 * (base + slot) + 1] = ds;
          st3(c.simp_n, base + slot, mk3(nx, ny, nz));
        }
      }
      __syncwarp();
    }
  }
}

// After detection: finish when nothing was hit (or the pass cap is reached), else start Jacobi iterations.
__global__ void k_contact_ctl_detect(ContactDev c, cudaGraphConditionalHandle h) {
  if (c.state[CS_MODE] != 0) return;
  const bool same_groups = c.ncf == 0 || c.state[CS_NGRP] == c.state[CS_NGRP_PREV];
  if (c.state[CS_ANY] == 0 && same_groups) {
    cudaGraphSetConditional(h, 0u);
    return;
  }
  if (c.state[CS_PASS] >= c.max_passes) {  // new impacts, but no pass left: the phase ends with an error
    cap_reached(c.status, kCapContactPasses);
    cudaGraphSetConditional(h, 0u);
    return;
  }
  c.state[CS_ANY] = 0;
  c.state[CS_MODE] = 1;
  c.state[CS_IT] = 0;
  c.state[CS_PASS] += 1;
}

// Jacobi iteration, part 1 (mode 1): ori_x = x_n1 and the max-norm test against xold.
// ori_x = x_n1 at vertex i, its max-norm change; record of contact vertex i's
// impact lists for the iteration with record index rk (-1: none).
// ori_x = x_n1 at vertex i and its max-norm change
__device__ __forceinline__ double contact_prep_vertex(const ContactDev& c, int i, double* xk) {
  Vec3<double> x = ld3(c.xn1, i);
  st3(xk, i, x);
  Vec3<double> dl = x - ld3(c.xold, i);
  return fmax(fabs(dl.x), fmax(fabs(dl.y), fabs(dl.z)));
}

// recording for the adjoint: the impact lists of contact vertex a this
// iteration will use, at record index rk
__device__ __forceinline__ void contact_prep_record(const ContactDev& c, int a, int rk) {
  const int cnt = c.imp_cnt[a];
  c.rec_cnt[(size_t)rk * c.nc + a] = cnt;
  // 64-bit offset to the vertex's normals (the record spans billions of doubles)
  double* rn = c.rec_n + ((size_t)rk * c.nc + a) * kMaxImpactsPerVertex * 3;
  for (int q = 0; q < cnt; ++q) st3(rn, q, ld3(c.imp_n, a * kMaxImpactsPerVertex + q));
}

__device__ __forceinline__ double contact_prep_item(const ContactDev& c, int i, int N, double* xk, int rk) {
  double e = 0;
  if (i < N) e = contact_prep_vertex(c, i, xk);
  if (rk >= 0 && i < c.nc) contact_prep_record(c, i, rk);
  return e;
}

__global__ void k_contact_prep(int N, ContactDev c, double* xk, double* partial, unsigned* counter) {
  if (c.state[CS_MODE] != 1) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = contact_prep_item(c, i, N, xk, rec_index(c));
  // deterministic grid max
  __shared__ double ws[32];
  __shared__ bool last;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
  if (lane == 0) ws[warp] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) m = fmax(m, ws[w]);
    partial[blockIdx.x] = m;
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double m = 0;
    for (unsigned b = 0; b < gridDim.x; ++b) m = fmax(m, ((volatile double*)partial)[b]);
    *counter = 0u;
    bool conv = m < kConvergenceEps;
    c.state[CS_ACTIVE] = conv ? 0 : 1;
    c.state[CS_SRC] = c.state[CS_COMP];  // ori_x is the x_n1 of the last computed iteration
    if (conv) c.state[CS_MODE] = 0;  // back to detection
  }
}

// Jacobi iteration, part 2: right-hand side in velocity form, contact reaction, relaxation, update.
//   rhs = M v_wc + h (J d - L x_t) - h C (ori_x - x_t),  C = off-diagonal of Hs
//   contact vertex: rhs := B r, r = -B^T rhs with the tangential part clamped to mu r_n (last impact wins)
//   prev = alpha rhs + (1 - alpha) prev  (prev = rhs before the contact step on the first iteration)
//   x_n1 = x_t + prev / (h diag(Hs)),  xold = ori_x
// The Jacobi update of vertex i (obstacle contact only): rhs, the friction
// cone of its impacts, relaxation, x_n1; first: the pass's first iteration;
// rk: record index (-1: none).
__device__ __forceinline__ void contact_rhs_item(const SceneDev& d, const ContactDev& c, int i, const double* slot,
                                                 const double* xt, const double* xk, bool first, int rk) {
  Vec3<double> jd = ld3(d.attach_jd, i);
  for (int k = d.vslot_ptr[i]; k < d.vslot_ptr[i + 1]; ++k) jd = jd + ld3(slot, k);
  Vec3<double> cdx = mk3(0.0, 0.0, 0.0);
  for (int k = d.hs_ptr[i]; k < d.hs_ptr[i + 1]; ++k) {
    int j = d.hs_col[k];
    if (j != i) cdx = cdx + d.hs_val[k] * (ld3(xk, j) - ld3(xt, j));
  }
  Vec3<double> rhs = d.mass[i] * ld3(c.vwc, i) + d.h * (jd - ld3(c.lxt, i)) - d.h * cdx;
  Vec3<double> prev = first ? rhs : ld3(c.prev, i);
  int a = c.cidx[i];
  if (a >= 0) {
    Vec3<double> f = rhs;
    int cnt = c.imp_cnt[a];
    for (int q = 0; q < cnt; ++q) {
      Vec3<double> B[3];
      contact_basis(ld3(c.imp_n, a * kMaxImpactsPerVertex + q), B);
      double f0 = dot3(B[0], f), f1 = dot3(B[1], f), f2 = dot3(B[2], f);
      if (f0 > 0) continue;  // take-off
      double r0 = -f0, r1 = -f1, r2 = -f2;
      double rt = sqrt(r1 * r1 + r2 * r2);
      if (rt > c.mu * r0) { r1 *= c.mu * r0 / rt; r2 *= c.mu * r0 / rt; }
      rhs = r0 * B[0] + r1 * B[1] + r2 * B[2];
    }
  }
  prev = c.alpha * rhs + (1.0 - c.alpha) * prev;
  st3(c.prev, i, prev);
  st3(c.xn1, i, ld3(xt, i) + (1.0 / (d.h * c.hdiag[i])) * prev);
  st3(c.xold, i, ld3(xk, i));
  if (rk >= 0) {
    st3(c.rec_x + (size_t)rk * 3 * d.N, i, ld3(xk, i));
    st3(c.rec_prev + (size_t)rk * 3 * d.N, i, prev);
    if (i == 0 && c.np <= 1) c.rec_first[rk] = first ? 1 : 0;  // batches: per part, by their phase kernel
  }
}

__global__ void k_contact_rhs(SceneDev d, ContactDev c, const double* __restrict__ slot, const double* xt,
                              const double* xk) {
  if (c.state[CS_MODE] != 1 || c.state[CS_ACTIVE] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  contact_rhs_item(d, c, i, slot, xt, xk, c.state[CS_IT] == 0, rec_index(c));
}

// End of a Jacobi iteration: count it; after K iterations return to detection.
// (Also counts loop-body executions, for the launch statistics.)
__global__ void k_contact_ctl_iter(ContactDev c, int K) {
  c.state[CS_BODIES] += 1;
  if (c.state[CS_MODE] != 1 || c.state[CS_ACTIVE] == 0) return;
  int it = c.state[CS_IT] + 1;
  c.state[CS_IT] = it;
  c.state[CS_ACTIVE] = 0;
  if (c.rec_on && *c.rec_on == 1 && *c.rec_base + c.state[CS_COMP] >= c.rec_cap)
    atomicExch(c.status, 6);  // the replayed step's record is too small
  c.state[CS_COMP] += 1;
  if (it >= K) c.state[CS_MODE] = 0;
}

// ---- the obstacle contact phase in one cooperative launch --------------------
//
// The whole phase of a step without soft contact as one kernel whose CTAs are
// all resident (a cooperative launch): the state machine of the conditional
// loop of the kernels above — detection; Jacobi iterations until the
// max-norm change of ori_x drops below EPS or K iterations ran; detection
// again, until a detection finds no impact — with grid-wide barriers between
// its phases instead of kernel boundaries (3 barriers per Jacobi iteration, 1
// per detection, against 6 launches per loop body).  Every phase runs its
// kernel's per-item code (contact_detect_item, contact_prep_item, local_item,
// contact_rhs_item) in a grid-stride loop, so the arithmetic and the records
// for the adjoint are those of the loop of kernels, bit for bit.  Every
// thread keeps an identical copy of the state machine, updated from values
// read after a barrier; thread 0 writes the final state (passes, loop-body
// executions, computed iterations, source iteration) to c.state for the
// step's record.  The detections' hit flags alternate between two words, so
// clearing one never races with reading the other.
__device__ __forceinline__ int rec_index_at(const ContactDev& c, int comp) {
  if (!c.rec_on || *c.rec_on == 0) return -1;
  const int k = *c.rec_base + comp;
  return k < c.rec_cap ? k : -1;
}

__global__ void __launch_bounds__(128) k_contact_fused(SceneDev d, ContactDev c, const double* xt, double* xk,
                                                       const double* act_all, const int* step, double* slot,
                                                       double* partial, int* status) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ double ws[4];
  __shared__ double s_m;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
  const bool lead = tid == 0;
  const int ncons = d.T + d.M + d.S + d.B, nv = max(d.N, c.nc);
  for (int i = tid; i < nv; i += nthr) contact_begin_item(d, c, i, xt, xk);
  if (lead)
    for (int k = 0; k < CS_SIZE; ++k) c.state[k] = 0;
  if (!(c.nc > 0 && c.nof > 0)) return;  // uniform, before any barrier
  grid.sync();
  int mode = 0, pass = 0, it = 0, bodies = 0, comp = 0, src = 0, ndet = 0;
  const int cap = c.max_passes * (c.K + 2) + 2;
  for (;;) {
    bodies += 1;
    if (mode == 0) {  // detection pass (k_contact_detect, k_contact_ctl_detect)
      int* flag = c.state + ((ndet & 1) ? CS_FANY1 : CS_FANY0);
      for (int a = tid; a < c.nc; a += nthr)
        if (contact_detect_item(c, a, xt, xk, status)) atomicOr(flag, 1);
      grid.sync();
      const bool any = *(volatile int*)flag != 0;
      if (lead) c.state[(ndet & 1) ? CS_FANY0 : CS_FANY1] = 0;  // the other word: read a barrier ago
      ++ndet;
      if (!any) break;
      if (pass >= c.max_passes) {
        if (lead) cap_reached(status, kCapContactPasses);
        break;
      }
      mode = 1;
      it = 0;
      pass += 1;
    }
    // one Jacobi iteration (k_contact_prep, k_local, k_contact_rhs, k_contact_ctl_iter)
    const int rk = rec_index_at(c, comp);
    double e = 0.0;
    for (int i = tid; i < nv; i += nthr) e = fmax(e, contact_prep_item(c, i, d.N, xk, rk));
    for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) partial[blockIdx.x] = fmax(fmax(ws[0], ws[1]), fmax(ws[2], ws[3]));
    grid.sync();
    if (threadIdx.x < 32) {  // every CTA forms the same maximum (order-independent)
      double m = 0.0;
      for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) m = fmax(m, __ldcg(partial + b));
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (threadIdx.x == 0) s_m = m;
    }
    __syncthreads();
    const bool conv = s_m < kConvergenceEps;
    src = comp;
    if (conv) {
      mode = 0;  // back to detection
    } else {
      for (int t = tid; t < ncons; t += nthr) local_item(d, t, xk, act_all, step, slot);
      grid.sync();
      for (int i = tid; i < d.N; i += nthr) contact_rhs_item(d, c, i, slot, xt, xk, it == 0, rk);
      grid.sync();
      it += 1;
      if (lead && c.rec_on && *c.rec_on == 1 && *c.rec_base + comp >= c.rec_cap) atomicExch(status, 6);
      comp += 1;
      if (it >= c.K) mode = 0;
    }
    if (bodies > cap) {  // unreachable: passes and iterations are bounded above
      if (lead) cap_reached(status, kCapContactPasses);
      break;
    }
  }
  if (lead) {
    c.state[CS_MODE] = mode; c.state[CS_PASS] = pass; c.state[CS_IT] = it; c.state[CS_BODIES] = bodies;
    c.state[CS_COMP] = comp; c.state[CS_SRC] = src;
  }
}

// ---- the obstacle contact phase of a batch ---------------------------------
//
// Every part (scene) of a batch runs the state machine of k_contact_fused on
// its own: its own detections, Jacobi iterations, convergence test, passes
// and records.  One cooperative launch advances all of them in rounds — a
// detection phase for the parts in detection mode, then one Jacobi iteration
// for the parts in iteration mode — with grid-wide barriers shared by all
// parts.  A part's sequence of operations, and so its arithmetic, is the one
// it has alone (the items are those of k_contact_fused; a part's maximum is
// taken over its own vertices).  Each CTA keeps an identical copy of the
// per-part state in shared memory, updated from values read after a barrier.
// Records: the computed iteration j of part p is record base + j of its
// vertices (parts own disjoint rows of a record), its pass flag at
// rec_first[(base + j) np + p].
enum { PS_MODE = 0, PS_PASS = 1, PS_IT = 2, PS_COMP = 3, PS_SRC = 4, PS_DONE = 5, PS_RUN = 6, PS_SKIP = 7, PS_SIZE = 8 };
constexpr int kMaxContactParts = 1024;

__device__ __forceinline__ int rec_index_part(const ContactDev& c, int comp) { return rec_index_at(c, comp); }

__global__ void __launch_bounds__(128) k_contact_fused_parts(SceneDev d, ContactDev c, const double* xt, double* xk,
                                                             const double* act_all, const int* step, double* slot,
                                                             int* status) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ int sp[];  // PS_SIZE x np
  __shared__ int s_flag;
  const int np = c.np;
  int* s_mode = sp + PS_MODE * np;
  int* s_pass = sp + PS_PASS * np;
  int* s_it = sp + PS_IT * np;
  int* s_comp = sp + PS_COMP * np;
  int* s_src = sp + PS_SRC * np;
  int* s_done = sp + PS_DONE * np;
  int* s_run = sp + PS_RUN * np;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
  const bool lead = tid == 0;
  const int ncons = d.T + d.M + d.S + d.B, nv = max(d.N, c.nc);
  for (int i = tid; i < nv; i += nthr) contact_begin_item(d, c, i, xt, xk);
  for (int q = tid; q < 2 * np; q += nthr) { c.pany[q] = 0; c.pe[q] = 0ull; }
  if (lead)
    for (int k = 0; k < CS_SIZE; ++k) c.state[k] = 0;
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    s_mode[p] = 0; s_pass[p] = 0; s_it[p] = 0; s_comp[p] = 0; s_src[p] = 0; s_run[p] = 0;
    s_done[p] = (c.pf0[p + 1] == c.pf0[p]) ? 1 : 0;  // a part without obstacle faces has no phase
  }
  grid.sync();
  const int cap = c.max_passes * (c.K + 2) + 2;
  int rounds = 0;
  for (;;) {
    rounds += 1;
    // detection for the parts in detection mode (k_contact_detect)
    int* anyf = c.pany + (rounds & 1) * np;
    for (int a = tid; a < c.nc; a += nthr) {
      const int p = c.cpart[a];
      if (s_mode[p] == 0 && !s_done[p] && contact_detect_item(c, a, xt, xk, status)) atomicOr(anyf + p, 1);
    }
    grid.sync();
    // k_contact_ctl_detect per part
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
      if (s_done[p] || s_mode[p] != 0) continue;
      if (((volatile int*)anyf)[p] == 0) {
        s_done[p] = 1;
      } else if (s_pass[p] >= c.max_passes) {
        if (blockIdx.x == 0) cap_reached(status, kCapContactPasses);
        s_done[p] = 1;
      } else {
        s_mode[p] = 1; s_it[p] = 0; s_pass[p] += 1;
      }
    }
    if (lead)  // the other parity's flags: read a round ago
      for (int p = 0; p < np; ++p) c.pany[((rounds + 1) & 1) * np + p] = 0;
    if (threadIdx.x == 0) s_flag = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < np; p += blockDim.x)
      if (!s_done[p]) s_flag = 1;
    __syncthreads();
    if (!s_flag) break;  // every CTA reads the same state
    // one Jacobi iteration for the parts in iteration mode (k_contact_prep ..)
    unsigned long long* pe = c.pe + (rounds & 1) * np;
    const int lane = threadIdx.x & 31;
    for (int i0 = tid - lane; i0 < d.N; i0 += nthr) {  // warp-uniform trip count
      const int i = i0 + lane;
      const int p = i < d.N ? vpart_of(d, i) : -1;
      const bool on = p >= 0 && s_mode[p] == 1 && !s_done[p];
      double e = on ? contact_prep_vertex(c, i, xk) : 0.0;
      // a warp within one part reduces first (lane 0 is in range); the
      // per-part maximum (of doubles >= 0, as ordered bit patterns) does not
      // depend on the order of the atomics
      const int p0 = __shfl_sync(0xffffffffu, p, 0);
      if (__all_sync(0xffffffffu, p == p0 || p < 0)) {
        for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
        if (lane == 0 && on) atomicMax(pe + p, (unsigned long long)__double_as_longlong(e));
      } else if (on) {
        atomicMax(pe + p, (unsigned long long)__double_as_longlong(e));
      }
    }
    for (int a = tid; a < c.nc; a += nthr) {
      const int p = c.cpart[a];
      if (s_mode[p] != 1 || s_done[p]) continue;
      const int rk = rec_index_part(c, s_comp[p]);
      if (rk >= 0) contact_prep_record(c, a, rk);
    }
    grid.sync();
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
      s_run[p] = 0;
      if (s_done[p] || s_mode[p] != 1) continue;
      const double m = __longlong_as_double((long long)((volatile unsigned long long*)pe)[p]);
      s_src[p] = s_comp[p];
      if (m < kConvergenceEps) s_mode[p] = 0;  // back to detection
      else s_run[p] = 1;
    }
    if (lead)  // the other parity's maxima: read a round ago
      for (int p = 0; p < np; ++p) c.pe[((rounds + 1) & 1) * np + p] = 0ull;
    __syncthreads();
    for (int t = tid; t < ncons; t += nthr)
      if (s_run[cons_part(d, t)]) local_item(d, t, xk, act_all, step, slot);
    grid.sync();
    for (int i = tid; i < d.N; i += nthr) {
      const int p = vpart_of(d, i);
      if (s_run[p]) contact_rhs_item(d, c, i, slot, xt, xk, s_it[p] == 0, rec_index_part(c, s_comp[p]));
    }
    for (int p = tid; p < np; p += nthr)
      if (s_run[p]) {
        const int rk = rec_index_part(c, s_comp[p]);
        if (rk >= 0) c.rec_first[(size_t)rk * np + p] = s_it[p] == 0 ? 1 : 0;
      }
    grid.sync();
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
      if (!s_run[p]) continue;
      if (blockIdx.x == 0 && c.rec_on && *c.rec_on == 1 && *c.rec_base + s_comp[p] >= c.rec_cap) atomicExch(status, 6);
      s_it[p] += 1;
      s_comp[p] += 1;
      if (s_it[p] >= c.K) s_mode[p] = 0;
    }
    __syncthreads();
    if (rounds > cap) {  // unreachable: every part's passes and iterations are bounded
      if (lead) cap_reached(status, kCapContactPasses);
      break;
    }
  }
  if (blockIdx.x == 0) {
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
      c.pst[PS_MODE * np + p] = s_mode[p]; c.pst[PS_PASS * np + p] = s_pass[p]; c.pst[PS_IT * np + p] = s_it[p];
      c.pst[PS_COMP * np + p] = s_comp[p]; c.pst[PS_SRC * np + p] = s_src[p];
    }
    if (threadIdx.x == 0) {
      int mp = 0, mc = 0;
      for (int p = 0; p < np; ++p) { mp = max(mp, s_pass[p]); mc = max(mc, s_comp[p]); }
      c.state[CS_MODE] = 0; c.state[CS_PASS] = mp; c.state[CS_IT] = 0; c.state[CS_BODIES] = rounds;
      c.state[CS_COMP] = mc; c.state[CS_SRC] = 0;
    }
  }
}

// per-step record of a batch's phase: every part's source iteration (forward recording)
__global__ void k_contact_record_parts(const int* step, ContactDev c) {
  if (!(c.rec_on && *c.rec_on == 2)) return;
  const int s = *step;
  for (int p = threadIdx.x; p < c.np; p += blockDim.x) c.psrc[(size_t)s * c.np + p] = c.pst[PS_SRC * c.np + p];
}

// ---- the batched phase as a conditional loop of kernels ---------------------
//
// The same per-part state machine as k_contact_fused_parts, one kernel per
// phase, each with its own occupancy (the cooperative launch holds the
// largest per-item register set on every CTA): the state lives in c.pst
// (PS_* rows of np), the phase kernels read it, one-block control kernels
// advance it, and the last one decides whether the graph's loop runs again.
// Per part the operations and their order are those of the cooperative form.
__device__ __forceinline__ int& pst_at(const ContactDev& c, int row, int p) { return c.pst[row * c.np + p]; }

__global__ void k_cparts_begin(SceneDev d, ContactDev c, const double* xt, const double* xk,
                               cudaGraphConditionalHandle h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  contact_begin_item(d, c, i, xt, xk);
  if (blockIdx.x == 0) {
    for (int p = threadIdx.x; p < c.np; p += blockDim.x) {
      pst_at(c, PS_MODE, p) = 0; pst_at(c, PS_PASS, p) = 0; pst_at(c, PS_IT, p) = 0; pst_at(c, PS_COMP, p) = 0;
      pst_at(c, PS_SRC, p) = 0; pst_at(c, PS_RUN, p) = 0; pst_at(c, PS_SKIP, p) = 1;
      pst_at(c, PS_DONE, p) = (c.pf0[p + 1] == c.pf0[p]) ? 1 : 0;  // a part without obstacle faces has no phase
      c.pany[p] = 0;
      c.pe[p] = 0ull;
    }
    if (threadIdx.x == 0) {
      for (int k = 0; k < CS_SIZE; ++k) c.state[k] = 0;
      cudaGraphSetConditional(h, (c.nc > 0 && c.nof > 0) ? 1u : 0u);
    }
  }
}

// detection for the parts in detection mode
__global__ void k_cparts_detect(ContactDev c, const double* xt, const double* xk, int* status) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= c.nc) return;
  const int p = c.cpart[a];
  if (pst_at(c, PS_MODE, p) != 0 || pst_at(c, PS_DONE, p)) return;
  if (contact_detect_item(c, a, xt, xk, status)) atomicOr(c.pany + p, 1);
}

// after detection (k_contact_ctl_detect per part); clears the parts' maxima
__global__ void k_cparts_ctl_detect(ContactDev c, int* status) {
  for (int p = threadIdx.x; p < c.np; p += blockDim.x) {
    c.pe[p] = 0ull;
    if (pst_at(c, PS_DONE, p) || pst_at(c, PS_MODE, p) != 0) continue;
    const int any = c.pany[p];
    c.pany[p] = 0;
    if (!any) {
      pst_at(c, PS_DONE, p) = 1;
    } else if (pst_at(c, PS_PASS, p) >= c.max_passes) {
      cap_reached(status, kCapContactPasses);
      pst_at(c, PS_DONE, p) = 1;
    } else {
      pst_at(c, PS_MODE, p) = 1; pst_at(c, PS_IT, p) = 0; pst_at(c, PS_PASS, p) += 1;
    }
  }
}

// ori_x = x_n1 on the vertices of the parts in iteration mode, and each
// part's max-norm change (part-aligned blocks; the maximum of doubles >= 0
// as ordered bit patterns does not depend on the order of the atomics)
__global__ void k_cparts_prep(PartDev pd, ContactDev c, double* xk) {
  __shared__ double ws[32];
  const int b = blockIdx.x, p = pd.blk_part[b];
  if (pst_at(c, PS_MODE, p) != 1 || pst_at(c, PS_DONE, p)) return;  // uniform over the block
  const int i = pd.blk_v0[b] + threadIdx.x;
  double e = i < pd.part_v0[p + 1] ? contact_prep_vertex(c, i, xk) : 0.0;
  for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) m = fmax(m, ws[w]);
    atomicMax(c.pe + p, (unsigned long long)__double_as_longlong(m));
  }
}

// the impact lists each iterating part's contact vertices use, into its records
__global__ void k_cparts_record(ContactDev c) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= c.nc) return;
  const int p = c.cpart[a];
  if (pst_at(c, PS_MODE, p) != 1 || pst_at(c, PS_DONE, p)) return;
  const int rk = rec_index_at(c, pst_at(c, PS_COMP, p));
  if (rk >= 0) contact_prep_record(c, a, rk);
}

// per part: converged (back to detection) or one more Jacobi iteration
// (PS_RUN; PS_SKIP is its complement, the gate of the local step)
__global__ void k_cparts_ctl_conv(ContactDev c) {
  for (int p = threadIdx.x; p < c.np; p += blockDim.x) {
    pst_at(c, PS_RUN, p) = 0;
    pst_at(c, PS_SKIP, p) = 1;
    if (pst_at(c, PS_DONE, p) || pst_at(c, PS_MODE, p) != 1) continue;
    const double m = __longlong_as_double((long long)c.pe[p]);
    pst_at(c, PS_SRC, p) = pst_at(c, PS_COMP, p);
    if (m < kConvergenceEps) {
      pst_at(c, PS_MODE, p) = 0;
    } else {
      pst_at(c, PS_RUN, p) = 1;
      pst_at(c, PS_SKIP, p) = 0;
    }
  }
}

// the Jacobi update of the iterating parts' vertices (contact_rhs_item), and
// each part's pass flag for its record
__global__ void k_cparts_rhs(SceneDev d, PartDev pd, ContactDev c, const double* __restrict__ slot, const double* xt,
                             const double* xk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  const int p = vpart_of(d, i);
  if (!pst_at(c, PS_RUN, p)) return;
  const int first = pst_at(c, PS_IT, p) == 0 ? 1 : 0;
  const int rk = rec_index_at(c, pst_at(c, PS_COMP, p));
  contact_rhs_item(d, c, i, slot, xt, xk, first != 0, rk);
  if (i == pd.part_v0[p] && rk >= 0) c.rec_first[(size_t)rk * c.np + p] = first;
}

// end of a round: count the iterations, and loop while some part is not done
__global__ void k_cparts_ctl_iter(ContactDev c, int K, int* status, cudaGraphConditionalHandle h) {
  __shared__ int s_open, s_pass, s_comp;
  if (threadIdx.x == 0) { s_open = 0; s_pass = 0; s_comp = 0; }
  __syncthreads();
  for (int p = threadIdx.x; p < c.np; p += blockDim.x) {
    if (pst_at(c, PS_RUN, p)) {
      if (c.rec_on && *c.rec_on == 1 && *c.rec_base + pst_at(c, PS_COMP, p) >= c.rec_cap) atomicExch(status, 6);
      pst_at(c, PS_IT, p) += 1;
      pst_at(c, PS_COMP, p) += 1;
      if (pst_at(c, PS_IT, p) >= K) pst_at(c, PS_MODE, p) = 0;
    }
    if (!pst_at(c, PS_DONE, p)) s_open = 1;
    atomicMax(&s_pass, pst_at(c, PS_PASS, p));
    atomicMax(&s_comp, pst_at(c, PS_COMP, p));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int rounds = c.state[CS_BODIES] + 1;
    c.state[CS_BODIES] = rounds;
    c.state[CS_PASS] = s_pass;
    c.state[CS_COMP] = s_comp;
    bool open = s_open != 0;
    if (open && rounds > c.max_passes * (K + 2) + 2) {  // unreachable: every part's passes and iterations are bounded
      cap_reached(status, kCapContactPasses);
      open = false;
    }
    cudaGraphSetConditional(h, open ? 1u : 0u);
  }
}

// reverse sweep gate: part p takes part in computed iteration j when j <= top[p]
__global__ void k_cparts_gate(ContactDev c, const int* top, int j) {
  for (int p = threadIdx.x; p < c.np; p += blockDim.x) pst_at(c, PS_SKIP, p) = j > top[p] ? 1 : 0;
}

// ---- soft-soft (self) contact ------------------------------------------------
//
// CollisionBrutal::getSelfCollisionsInfo (collisionBrutal.h:645-700): each
// contact vertex's closest soft impact of the step (smallest t; at t = 1 the
// smallest distance; earlier list entries otherwise), its vertices grouped by
// face.  Groups are kept per face (g_ptr / g_mem, members ascending), the
// group normal is its first member's impact normal.  Run in detection mode
// after k_contact_detect; the pass ends when no new obstacle impact appeared
// and the number of groups did not change (BaseUpdateCollisions' return).

__global__ void k_self_reset(ContactDev c) {
  if (c.state[CS_MODE] != 0) return;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < c.ncf) { c.g_cnt[f] = 0; c.g_fill[f] = 0; }
  if (f == 0) { c.state[CS_NGRP_PREV] = c.state[CS_NGRP]; c.state[CS_NGRP] = 0; }
}

__global__ void k_self_closest(ContactDev c) {
  if (c.state[CS_MODE] != 0) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= c.nc) return;
  const int base = a * kMaxSelfImpacts, cnt = c.simp_cnt[a];
  int best = -1;
  for (int q = 0; q < cnt; ++q) {
    if (best < 0) { best = q; continue; }
    const double t = c.simp_td[2 * (base + q)], bt = c.simp_td[2 * (base + best)];
    if (t < bt) { best = q; continue; }
    if (bt == 1.0 && c.simp_td[2 * (base + best) + 1] > c.simp_td[2 * (base + q) + 1]) best = q;
  }
  c.cf_slot[a] = best;
  c.cf_face[a] = best >= 0 ? c.simp_face[base + best] : -1;
  if (best >= 0) atomicAdd(&c.g_cnt[c.simp_face[base + best]], 1);
}

// one block: g_ptr = exclusive scan of g_cnt, and the number of groups
__global__ void k_self_scan(ContactDev c) {
  if (c.state[CS_MODE] != 0) return;
  __shared__ int sh[1024];
  __shared__ int carry_s, groups_s;
  const int tid = threadIdx.x, bs = blockDim.x;
  if (tid == 0) { carry_s = 0; groups_s = 0; }
  __syncthreads();
  for (int base = 0; base < c.ncf; base += bs) {
    const int f = base + tid;
    const int v = f < c.ncf ? c.g_cnt[f] : 0;
    sh[tid] = v;
    const int nz = __syncthreads_count(v > 0);
    for (int off = 1; off < bs; off <<= 1) {  // inclusive Hillis-Steele scan
      const int add = tid >= off ? sh[tid - off] : 0;
      __syncthreads();
      sh[tid] += add;
      __syncthreads();
    }
    if (f < c.ncf) c.g_ptr[f] = carry_s + sh[tid] - v;
    __syncthreads();
    if (tid == 0) { carry_s += sh[bs - 1]; groups_s += nz; }
    __syncthreads();
  }
  if (tid == 0) {
    c.g_ptr[c.ncf] = carry_s;
    c.state[CS_NGRP] = groups_s;
  }
}

__global__ void k_self_fill(ContactDev c) {
  if (c.state[CS_MODE] != 0) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= c.nc) return;
  const int f = c.cf_face[a];
  if (f < 0) return;
  const int pos = atomicAdd(&c.g_fill[f], 1);
  c.g_mem[c.g_ptr[f] + pos] = a;
}

// members ascending (the fill order is arbitrary); group normal; member slots
__global__ void k_self_sort(ContactDev c, int* status) {
  if (c.state[CS_MODE] != 0) return;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= c.ncf) return;
  const int cnt = c.g_cnt[f];
  if (cnt == 0) return;
  if (cnt > c.max_members) cap_reached(status, kCapGroupMembers);
  int* m = c.g_mem + c.g_ptr[f];
  for (int k = 1; k < cnt; ++k) {
    const int v = m[k];
    int j = k - 1;
    while (j >= 0 && m[j] > v) { m[j + 1] = m[j]; --j; }
    m[j + 1] = v;
  }
  for (int k = 0; k < cnt; ++k) c.m_slot[m[k]] = c.g_ptr[f] + k;
  const int a0 = m[0];
  st3(c.g_n, f, ld3(c.simp_n, a0 * kMaxSelfImpacts + c.cf_slot[a0]));
}

__device__ __forceinline__ Vec3<double> to_local3(const Vec3<double> B[3], Vec3<double> p) {
  return mk3(p.x * B[0].x + p.y * B[0].y + p.z * B[0].z, p.x * B[1].x + p.y * B[1].y + p.z * B[1].z,
             p.x * B[2].x + p.y * B[2].y + p.z * B[2].z);
}
__device__ __forceinline__ Vec3<double> to_world3(const Vec3<double> B[3], Vec3<double> r) {
  return mk3(r.x * B[0].x + r.y * B[1].x + r.z * B[2].x, r.x * B[0].y + r.y * B[1].y + r.z * B[2].y,
             r.x * B[0].z + r.y * B[1].z + r.z * B[2].z);
}
__device__ __forceinline__ Vec3<double> div3(Vec3<double> a, double s) { return mk3(a.x / s, a.y / s, a.z / s); }

// World::do_solve_friction (World.h:1246-1315) on local-frame momenta: the
// sticking set (face + sticking members) moves tangentially together; sliding
// members receive mu times their normal force against their own slip, the
// sticking set mu f_n (sliding) along the mean slip.
__device__ void group_friction(Vec3<double> p0, double m0, Vec3<double>& r0, const Vec3<double>* ps, const double* ms,
                               Vec3<double>* rs, const unsigned char* stick, int n, double mu) {
  Vec3<double> pstick = p0;
  double mstick = m0;
  for (int k = 0; k < n; ++k)
    if (stick[k]) { pstick = pstick + ps[k]; mstick = mstick + ms[k]; }
  Vec3<double> pslide = mk3(0.0, 0.0, 0.0);
  double mslide = 0.0, fn = 0.0;
  for (int k = 0; k < n; ++k)
    if (!stick[k]) { pslide = pslide + ps[k]; mslide = mslide + ms[k]; fn = fn + rs[k].x; }
  const Vec3<double> v = div3(pstick, mstick);
  r0.y = v.y * m0 - p0.y;
  r0.z = v.z * m0 - p0.z;
  for (int k = 0; k < n; ++k)
    if (stick[k]) { rs[k].y = v.y * ms[k] - ps[k].y; rs[k].z = v.z * ms[k] - ps[k].z; }
  if (mslide > 0) {
    Vec3<double> rel = div3(pslide, mslide) - div3(pstick, mstick);
    rel = div3(rel, sqrt(rel.y * rel.y + rel.z * rel.z));
    const double mult = mu * fn / (mslide + mstick);
    r0.y = r0.y + rel.y * mult * m0;
    r0.z = r0.z + rel.z * mult * m0;
    for (int k = 0; k < n; ++k)
      if (stick[k]) { rs[k].y = rs[k].y + rel.y * mult * ms[k]; rs[k].z = rs[k].z + rel.z * mult * ms[k]; }
    const Vec3<double> abs_v0 = div3(p0 + r0, m0);
    for (int k = 0; k < n; ++k)
      if (!stick[k]) {
        Vec3<double> rk = div3(ps[k], ms[k]) - abs_v0;
        rk = div3(rk, sqrt(rk.y * rk.y + rk.z * rk.z));
        const double mk = -mu * rs[k].x * ms[k] / (ms[k] + mstick);
        rs[k].y = mk * rk.y;
        rs[k].z = mk * rk.z;
      }
  }
}

// One face group per thread (World.h:1462-1531): members approaching the face
// (normal relative velocity <= 0) and the face reach one normal velocity;
// tangential forces from the stick/slide iteration; the face's vertices end
// with the face's common velocity.  Inputs P = rhs + obstacle reactions,
// masses diag(Hs).
__global__ void k_self_exchange(ContactDev c) {
  if (c.state[CS_MODE] != 1 || c.state[CS_ACTIVE] == 0 || c.state[CS_NGRP] == 0) return;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= c.ncf) return;
  const int cnt = min(c.g_cnt[f], kMaxGroupMembers);
  if (cnt == 0) return;
  Vec3<double> B[3];
  contact_basis(ld3(c.g_n, f), B);
  Vec3<double> P[3];
  double mf[3];
  for (int i = 0; i < 3; ++i) {
    const int a = c.cfaces[3 * f + i];
    P[i] = ld3(c.rhs_pre, a) + ld3(c.cnext, a);
    mf[i] = c.hdiag[c.cverts[a]];
  }
  const int* mem = c.g_mem + c.g_ptr[f];
  const double m0 = mf[0] + mf[1] + mf[2];
  const Vec3<double> f0 = to_local3(B, (P[0] + P[1]) + P[2]);
  int inc[kMaxGroupMembers];
  double ms[kMaxGroupMembers];
  Vec3<double> fs[kMaxGroupMembers], rs[kMaxGroupMembers];
  unsigned char stick[kMaxGroupMembers];
  int n = 0;
  double sm = 0.0, smv = 0.0;
  for (int k = 0; k < cnt; ++k) {
    const int a = mem[k];
    const Vec3<double> pk = ld3(c.rhs_pre, a) + ld3(c.cnext, a);
    const double mk = c.hdiag[c.cverts[a]];
    const Vec3<double> fl = to_local3(B, pk);
    if (fl.x / mk - f0.x / m0 <= 0) {
      inc[n] = k; ms[n] = mk; fs[n] = fl;
      sm = sm + mk; smv = smv + fl.x;
      ++n;
    }
  }
  Vec3<double> r0 = mk3(0.0, 0.0, 0.0);
  for (int k = 0; k < n; ++k) {
    const double fn = (f0.x + smv) * ms[k] / (m0 + sm) - fs[k].x;
    rs[k] = mk3(0.0 + fn, 0.0, 0.0);
    r0.x = r0.x - fn;
    stick[k] = 1;
  }
  for (int round = 0; round <= n; ++round) {  // each round unsticks at least one member
    group_friction(f0, m0, r0, fs, ms, rs, stick, n, c.mu_self);
    bool changed = false;
    for (int k = 0; k < n; ++k)
      if (stick[k] && rs[k].y * rs[k].y + rs[k].z * rs[k].z > c.mu_self * rs[k].x * rs[k].x) {
        changed = true;
        stick[k] = 0;
      }
    if (!changed) break;
  }
  const Vec3<double> v0 = div3(to_world3(B, f0) + to_world3(B, r0), m0);
  for (int i = 0; i < 3; ++i) st3(c.g_outF, 3 * f + i, mf[i] * v0 - P[i]);
  const int gp = c.g_ptr[f];
  for (int k = 0; k < cnt; ++k) st3(c.g_outM, gp + k, mk3(0.0, 0.0, 0.0));
  for (int k = 0; k < n; ++k) st3(c.g_outM, gp + inc[k], to_world3(B, rs[k]));
}

// Jacobi iteration with self contact on, part A (per vertex): rhs before
// CollisionHandling; non-contact vertices finish here (relaxation, update);
// contact vertices keep it and their obstacle reaction, seen with the
// remembered self forces (forces + m_self_contact_forces[current]).
__global__ void k_contact_rhs_pre(SceneDev d, ContactDev c, const double* __restrict__ slot, const double* xt,
                                  const double* xk) {
  if (c.state[CS_MODE] != 1 || c.state[CS_ACTIVE] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  Vec3<double> jd = ld3(d.attach_jd, i);
  for (int k = d.vslot_ptr[i]; k < d.vslot_ptr[i + 1]; ++k) jd = jd + ld3(slot, k);
  Vec3<double> cdx = mk3(0.0, 0.0, 0.0);
  for (int k = d.hs_ptr[i]; k < d.hs_ptr[i + 1]; ++k) {
    int j = d.hs_col[k];
    if (j != i) cdx = cdx + d.hs_val[k] * (ld3(xk, j) - ld3(xt, j));
  }
  const Vec3<double> rhs = d.mass[i] * ld3(c.vwc, i) + d.h * (jd - ld3(c.lxt, i)) - d.h * cdx;
  const int a = c.cidx[i];
  const int rk = rec_index(c);
  if (rk >= 0) {
    st3(c.rec_x + (size_t)rk * 3 * d.N, i, ld3(xk, i));
    if (i == 0) c.rec_first[rk] = c.state[CS_IT] == 0 ? 1 : 0;
  }
  if (a < 0) {
    const bool first = c.state[CS_IT] == 0;
    Vec3<double> prev = first ? rhs : ld3(c.prev, i);
    prev = c.alpha * rhs + (1.0 - c.alpha) * prev;
    st3(c.prev, i, prev);
    st3(c.xn1, i, ld3(xt, i) + (1.0 / (d.h * c.hdiag[i])) * prev);
    st3(c.xold, i, ld3(xk, i));
    if (rk >= 0) st3(c.rec_prev + (size_t)rk * 3 * d.N, i, prev);
    return;
  }
  st3(c.rhs_pre, a, rhs);
  const Vec3<double> f = rhs + ld3(c.sc_cur, a);
  Vec3<double> out = mk3(0.0, 0.0, 0.0);
  int hit = 0;
  const int cnt = c.imp_cnt[a];
  for (int q = 0; q < cnt; ++q) {
    Vec3<double> B[3];
    contact_basis(ld3(c.imp_n, a * kMaxImpactsPerVertex + q), B);
    double f0 = dot3(B[0], f), f1 = dot3(B[1], f), f2 = dot3(B[2], f);
    if (f0 > 0) continue;  // take-off
    double r0 = -f0, r1 = -f1, r2 = -f2;
    double rt = sqrt(r1 * r1 + r2 * r2);
    if (rt > c.mu * r0) { r1 *= c.mu * r0 / rt; r2 *= c.mu * r0 / rt; }
    out = r0 * B[0] + r1 * B[1] + r2 * B[2];
    hit = 1;
  }
  c.chit[a] = hit;
  st3(c.cnext, a, out);
}

// Part C (per contact vertex): CollisionHandling's result and the update.
//   no contact at all: rhs unchanged, remembered self forces unchanged;
//   no self group: hit vertices rhs := B r, remembered self forces := 0;
//   self groups: rhs += B r + self forces (face vertices of the groups, faces
//   ascending, then the vertex's own member force), remembered := self forces.
__global__ void k_contact_rhs_post(SceneDev d, ContactDev c, const double* xt, const double* xk) {
  if (c.state[CS_MODE] != 1 || c.state[CS_ACTIVE] == 0) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= c.nc) return;
  const int i = c.cverts[a];
  const Vec3<double> rhs = ld3(c.rhs_pre, a);
  Vec3<double> post = rhs;
  const int nobs = c.state[CS_NOBS], ngrp = c.state[CS_NGRP];
  if (ngrp == 0) {
    if (nobs > 0) {
      if (c.chit[a]) post = ld3(c.cnext, a);
      st3(c.sc_cur, a, mk3(0.0, 0.0, 0.0));
    }
  } else {
    Vec3<double> sn = mk3(0.0, 0.0, 0.0);
    for (int k = c.cvf_ptr[a]; k < c.cvf_ptr[a + 1]; ++k) {
      const int f = c.cvf_face[k];
      if (c.g_cnt[f] == 0) continue;
      const int corner = c.cfaces[3 * f] == a ? 0 : (c.cfaces[3 * f + 1] == a ? 1 : 2);
      sn = sn + ld3(c.g_outF, 3 * f + corner);
    }
    if (c.cf_face[a] >= 0) sn = sn + ld3(c.g_outM, c.m_slot[a]);
    post = rhs + (ld3(c.cnext, a) + sn);
    st3(c.sc_cur, a, sn);
  }
  const bool first = c.state[CS_IT] == 0;
  Vec3<double> prev = first ? rhs : ld3(c.prev, i);
  prev = c.alpha * post + (1.0 - c.alpha) * prev;
  st3(c.prev, i, prev);
  st3(c.xn1, i, ld3(xt, i) + (1.0 / (d.h * c.hdiag[i])) * prev);
  st3(c.xold, i, ld3(xk, i));
  const int rk = rec_index(c);
  if (rk >= 0) st3(c.rec_prev + (size_t)rk * 3 * d.N, i, prev);
}

// Record of a computed iteration's soft-contact inputs for the adjoint (after
// k_contact_rhs_pre, before k_contact_rhs_post replaces the remembered forces).
__global__ void k_self_record(ContactDev c) {
  if (c.state[CS_MODE] != 1 || c.state[CS_ACTIVE] == 0) return;
  const int rk = rec_index(c);
  if (rk < 0) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.nc, ncf = c.ncf;
  int* si = c.rec_si + (size_t)rk * self_rec_si_stride(nc, ncf);
  double* sd = c.rec_sd + (size_t)rk * self_rec_sd_stride(nc, ncf);
  if (k < nc) {
    si[k] = c.cf_face[k];
    si[nc + k] = c.m_slot[k];
    si[2 * nc + k] = c.g_mem[k];
    st3(sd, k, ld3(c.sc_cur, k));
  }
  if (k < ncf) {
    si[3 * nc + k] = c.g_cnt[k];
    st3(sd + 3 * (size_t)nc, k, ld3(c.g_n, k));
  }
  if (k <= ncf) si[3 * nc + ncf + k] = c.g_ptr[k];
  if (k == 0) {
    si[3 * nc + 2 * ncf + 1] = c.state[CS_NOBS];
    si[3 * nc + 2 * ncf + 2] = c.state[CS_NGRP];
  }
}

// Every time step starts with no remembered self forces: World::TimeStepping
// calls updateCollisionScene before the PD solve (sim/fem/World.h:700), which
// zeroes the self-collision force buffers (World.h:742-753).
__global__ void k_self_clear(ContactDev c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < 3 * c.nc) c.sc_cur[k] = 0.0;
}

// ---- adjoint of the contact phase ------------------------------------------------
//
// Reverse of the recorded Jacobi iterations j = src .. 1 of one step (the
// detection is discrete: impacts and normals are constants, as on the
// reference's tape).  Per iteration, with rhs_pre = M v_wc + h (J d(ori) -
// L x_t) - h C (ori - x_t), rhs_post its contact projection, prev_j =
// alpha rhs_post + (1 - alpha) prev_{j-1} (prev_{j-1} := rhs_pre at the first
// iteration of a pass) and x_n1 = x_t + prev_j / (h diag(Hs)):
//   k_cadj_rhs    cotangents of prev, rhs_post, the projection, rhs_pre;
//                 accumulates those of x_t, v_wc and diag(Hs)
//   (k_local at ori, then k_cadj_local: VJP of J d, parameter terms)
//   k_cadj_hs     the C and L x_t terms; x_n1 bar of the previous iteration
// Buffers: xn1b (x_n1 bar), pb (prev bar), hdb (diag(Hs) bar), cxtb (x_t bar),
// vwcb (v_wc bar), yb = h rhs_pre bar.

struct ContactAdj {
  double* xn1b;
  double* pb;
  double* hdb;
  double* cxtb;
  double* vwcb;
  double* yb;
  double* orib;
  // soft-soft contact: cotangent of the remembered self forces (3 nc, carried
  // between iterations and steps), per contact vertex the relaxation total and
  // the rhs_post cotangent, the groups' input cotangents by slot (P of the
  // face's vertices 9 ncf, of the members 3 nc; masses 3 ncf, nc), and the
  // cotangent of the phase's output until its source iteration (3N)
  double* scb = nullptr;
  double* ptot = nullptr;
  double* sbp = nullptr;
  double* gPF = nullptr;
  double* gPM = nullptr;
  double* gmF = nullptr;
  double* gmM = nullptr;
  double* xout = nullptr;
};

// one recorded iteration's soft-contact inputs (views into rec_si / rec_sd)
struct SelfRec {
  const int* cf_face;
  const int* m_slot;
  const int* g_mem;
  const int* g_cnt;
  const int* g_ptr;
  const int* nobs;
  const int* ngrp;
  const double* sc_in;
  const double* g_n;
};
__host__ __device__ inline SelfRec self_rec_view(const ContactDev& c, size_t r) {
  const int nc = c.nc, ncf = c.ncf;
  const int* si = c.rec_si + r * self_rec_si_stride(nc, ncf);
  const double* sd = c.rec_sd + r * self_rec_sd_stride(nc, ncf);
  return SelfRec{si, si + nc, si + 2 * (size_t)nc, si + 3 * (size_t)nc, si + 3 * (size_t)nc + ncf,
                 si + 3 * (size_t)nc + 2 * (size_t)ncf + 1, si + 3 * (size_t)nc + 2 * (size_t)ncf + 2, sd,
                 sd + 3 * (size_t)nc};
}

__global__ void k_cadj_start(int N, double cv, double* io_a, double* io_b, ContactAdj a, int defer) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const Vec3<double> gv = ld3(io_b, i);
  const Vec3<double> xo = ld3(io_a, i) + cv * gv;  // v' = damping (x' - x_t)/h
  if (defer) {  // soft contact: the output's cotangent enters at its source iteration
    st3(a.xout, i, xo);
    st3(a.xn1b, i, mk3(0.0, 0.0, 0.0));
  } else {
    st3(a.xn1b, i, xo);
  }
  st3(a.cxtb, i, (-cv) * gv);
  st3(a.vwcb, i, mk3(0.0, 0.0, 0.0));
  st3(a.pb, i, mk3(0.0, 0.0, 0.0));
  a.hdb[i] = 0.0;
}

// slot: J d at ori (k_local); xt: the step's start positions; ori, prev: the
// recorded iteration j; first: whether it began its pass; rcnt / rn: its impacts.
__device__ __forceinline__ void cadj_rhs_item(const SceneDev& d, const ContactDev& c, const ContactAdj& a, int i,
                                              const double* slot, const double* xt, const double* ori,
                                              const double* prev, int first, const int* rcnt, const double* rn) {
  const double hd = c.hdiag[i];
  const Vec3<double> xb = ld3(a.xn1b, i), pv = ld3(prev, i);
  st3(a.cxtb, i, ld3(a.cxtb, i) + xb);
  a.hdb[i] -= dot3(xb, pv) / (d.h * hd * hd);
  const Vec3<double> ptot = ld3(a.pb, i) + (1.0 / (d.h * hd)) * xb;
  Vec3<double> rb = c.alpha * ptot;
  const int ac = c.cidx[i];
  if (ac >= 0 && rcnt[ac] > 0) {
    // rhs_pre of the contact vertex, as in k_contact_rhs
    Vec3<double> jd = ld3(d.attach_jd, i);
    for (int k = d.vslot_ptr[i]; k < d.vslot_ptr[i + 1]; ++k) jd = jd + ld3(slot, k);
    Vec3<double> cdx = mk3(0.0, 0.0, 0.0);
    for (int k = d.hs_ptr[i]; k < d.hs_ptr[i + 1]; ++k) {
      const int j = d.hs_col[k];
      if (j != i) cdx = cdx + d.hs_val[k] * (ld3(ori, j) - ld3(xt, j));
    }
    const Vec3<double> f = d.mass[i] * ld3(c.vwc, i) + d.h * (jd - ld3(c.lxt, i)) - d.h * cdx;
    Vec3<double> W[3];
    bool hit = false;
    double r0 = 0, r1 = 0, r2 = 0;
    for (int q = 0; q < rcnt[ac]; ++q) {
      Vec3<double> B[3];
      contact_basis(ld3(rn, ac * kMaxImpactsPerVertex + q), B);
      const double f0 = dot3(B[0], f);
      if (f0 > 0) continue;
      hit = true;
      W[0] = B[0]; W[1] = B[1]; W[2] = B[2];
      r0 = -f0; r1 = -dot3(B[1], f); r2 = -dot3(B[2], f);
    }
    if (hit) {  // rhs_post = r0 W0 + r1' W1 + r2' W2 (friction cone clamp)
      const double b0 = dot3(W[0], rb), b1 = dot3(W[1], rb), b2 = dot3(W[2], rb);
      const double rt = sqrt(r1 * r1 + r2 * r2);
      double g0 = b0, g1 = b1, g2 = b2;
      if (rt > c.mu * r0) {
        g0 = b0 + c.mu * (r1 * b1 + r2 * b2) / rt;
        g1 = c.mu * r0 * (r2 * r2 * b1 - r1 * r2 * b2) / (rt * rt * rt);
        g2 = c.mu * r0 * (r1 * r1 * b2 - r1 * r2 * b1) / (rt * rt * rt);
      }
      rb = (-1.0) * (g0 * W[0] + g1 * W[1] + g2 * W[2]);
    }
  }
  if (first) {
    rb = rb + (1.0 - c.alpha) * ptot;
    st3(a.pb, i, mk3(0.0, 0.0, 0.0));
  } else {
    st3(a.pb, i, (1.0 - c.alpha) * ptot);
  }
  st3(a.vwcb, i, ld3(a.vwcb, i) + d.mass[i] * rb);
  st3(a.yb, i, d.h * rb);
}

__global__ void k_cadj_rhs(SceneDev d, ContactDev c, ContactAdj a, const double* __restrict__ slot,
                           const double* __restrict__ xt, const double* __restrict__ ori,
                           const double* __restrict__ prev, int first, const int* __restrict__ rcnt,
                           const double* __restrict__ rn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  cadj_rhs_item(d, c, a, i, slot, xt, ori, prev, first, rcnt, rn);
}

// cadj_rhs_item for the vertices of the parts in the sweep, each with its own pass flag
__global__ void k_cadj_rhs_parts(SceneDev d, ContactDev c, ContactAdj a, const double* __restrict__ slot,
                                 const double* __restrict__ xt, const double* __restrict__ ori,
                                 const double* __restrict__ prev, const int* __restrict__ first,
                                 const int* __restrict__ rcnt, const double* __restrict__ rn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  const int p = vpart_of(d, i);
  if (pst_at(c, PS_SKIP, p)) return;
  cadj_rhs_item(d, c, a, i, slot, xt, ori, prev, first[p], rcnt, rn);
}

// VJP of J d at ori with cotangent yb, and the Hs terms of the tets' E gradient
__global__ void __launch_bounds__(128, DFEM_ADJ_MIN_BLOCKS) k_cadj_local(SceneDev d, ContactAdj a, const double* __restrict__ ori,
                                                    const double* __restrict__ xt, const double* __restrict__ act_all,
                                                    const int* step, double* __restrict__ slot, double* gE,
                                                    double* gnu, double* mg, Gate gate) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (gate.skip(cons_part(d, t))) return;
  adj_local_item(d, t, ori, a.yb, act_all + (size_t)(*step) * d.nseg, slot, gE, gnu, mg, nullptr, xt);
}

// orib = (sum of the slots) - C^T yb; x_t bar += (M/h^2 - Hs_ii) yb_i; the
// result is the x_n1 bar of the previous computed iteration
__global__ void k_cadj_add_xout(int N, ContactAdj a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) st3(a.xn1b, i, ld3(a.xn1b, i) + ld3(a.xout, i));
}

// winning obstacle reaction of contact vertex ac for force f (recorded normals)
__device__ __forceinline__ bool obstacle_winner(const ContactDev& c, int ac, Vec3<double> f, const int* rcnt,
                                                const double* rn, Vec3<double> W[3], double& r0, double& r1, double& r2) {
  bool hit = false;
  for (int q = 0; q < rcnt[ac]; ++q) {
    Vec3<double> B[3];
    contact_basis(ld3(rn, ac * kMaxImpactsPerVertex + q), B);
    const double f0 = dot3(B[0], f);
    if (f0 > 0) continue;
    hit = true;
    W[0] = B[0]; W[1] = B[1]; W[2] = B[2];
    r0 = -f0; r1 = -dot3(B[1], f); r2 = -dot3(B[2], f);
  }
  return hit;
}
// cotangent of f from the cotangent ob of the reaction B c(-B^T f) (c: cone clamp)
__device__ __forceinline__ Vec3<double> reaction_vjp(const Vec3<double> W[3], double r0, double r1, double r2,
                                                     Vec3<double> ob, double mu) {
  const double b0 = dot3(W[0], ob), b1 = dot3(W[1], ob), b2 = dot3(W[2], ob);
  const double rt = sqrt(r1 * r1 + r2 * r2);
  double g0 = b0, g1 = b1, g2 = b2;
  if (rt > mu * r0) {
    g0 = b0 + mu * (r1 * b1 + r2 * b2) / rt;
    g1 = mu * r0 * (r2 * r2 * b1 - r1 * r2 * b2) / (rt * rt * rt);
    g2 = mu * r0 * (r1 * r1 * b2 - r1 * r2 * b1) / (rt * rt * rt);
  }
  return (-1.0) * (g0 * W[0] + g1 * W[1] + g2 * W[2]);
}

// Soft-contact adjoint of one recorded iteration, part A (per vertex): the
// relaxation's cotangents; non-contact vertices finish; contact vertices keep
// rhs_pre, their obstacle reaction (with the recorded remembered forces), the
// relaxation total and the cotangent of rhs_post for parts G and B.
__global__ void k_cadj_self_a(SceneDev d, ContactDev c, ContactAdj a, SelfRec rv, const double* __restrict__ slot,
                              const double* __restrict__ xt, const double* __restrict__ ori,
                              const double* __restrict__ prev, int first, const int* __restrict__ rcnt,
                              const double* __restrict__ rn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  const double hd = c.hdiag[i];
  const Vec3<double> xb = ld3(a.xn1b, i), pv = ld3(prev, i);
  st3(a.cxtb, i, ld3(a.cxtb, i) + xb);
  a.hdb[i] -= dot3(xb, pv) / (d.h * hd * hd);
  const Vec3<double> ptot = ld3(a.pb, i) + (1.0 / (d.h * hd)) * xb;
  Vec3<double> rb = c.alpha * ptot;
  const int ac = c.cidx[i];
  if (ac < 0) {
    if (first) {
      rb = rb + (1.0 - c.alpha) * ptot;
      st3(a.pb, i, mk3(0.0, 0.0, 0.0));
    } else {
      st3(a.pb, i, (1.0 - c.alpha) * ptot);
    }
    st3(a.vwcb, i, ld3(a.vwcb, i) + d.mass[i] * rb);
    st3(a.yb, i, d.h * rb);
    return;
  }
  Vec3<double> jd = ld3(d.attach_jd, i);
  for (int k = d.vslot_ptr[i]; k < d.vslot_ptr[i + 1]; ++k) jd = jd + ld3(slot, k);
  Vec3<double> cdx = mk3(0.0, 0.0, 0.0);
  for (int k = d.hs_ptr[i]; k < d.hs_ptr[i + 1]; ++k) {
    const int j = d.hs_col[k];
    if (j != i) cdx = cdx + d.hs_val[k] * (ld3(ori, j) - ld3(xt, j));
  }
  const Vec3<double> f = d.mass[i] * ld3(c.vwc, i) + d.h * (jd - ld3(c.lxt, i)) - d.h * cdx;
  st3(c.rhs_pre, ac, f);
  Vec3<double> W[3];
  double r0 = 0, r1 = 0, r2 = 0;
  const bool hit = obstacle_winner(c, ac, f + ld3(rv.sc_in, ac), rcnt, rn, W, r0, r1, r2);
  c.chit[ac] = hit ? 1 : 0;
  if (hit) {
    const double rt = sqrt(r1 * r1 + r2 * r2);
    double q1 = r1, q2 = r2;
    if (rt > c.mu * r0) { q1 *= c.mu * r0 / rt; q2 *= c.mu * r0 / rt; }
    st3(c.cnext, ac, r0 * W[0] + q1 * W[1] + q2 * W[2]);
  } else {
    st3(c.cnext, ac, mk3(0.0, 0.0, 0.0));
  }
  st3(a.ptot, ac, ptot);
  st3(a.sbp, ac, rb);
}

// Part G (one thread per face group, iterations with groups): the reverse of
// k_self_exchange.  The tangential outputs depend only on the last
// stick/slide round (each round recomputes them from the normal parts and the
// stick set), so the forward is recomputed and that round reversed.  Writes
// the cotangents of the inputs P and masses by slot.
__global__ void k_cadj_self_group(ContactDev c, ContactAdj a, SelfRec rv) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= c.ncf || *rv.ngrp == 0) return;
  const int cnt = min(rv.g_cnt[f], kMaxGroupMembers);
  if (cnt == 0) return;
  const double mu = c.mu_self;
  Vec3<double> B[3];
  contact_basis(ld3(rv.g_n, f), B);
  int fa[3];
  Vec3<double> P[3];
  double mf[3];
  for (int i = 0; i < 3; ++i) {
    fa[i] = c.cfaces[3 * f + i];
    P[i] = ld3(c.rhs_pre, fa[i]) + ld3(c.cnext, fa[i]);
    mf[i] = c.hdiag[c.cverts[fa[i]]];
  }
  const int* mem = rv.g_mem + rv.g_ptr[f];
  const double m0 = mf[0] + mf[1] + mf[2];
  const Vec3<double> f0 = to_local3(B, (P[0] + P[1]) + P[2]);
  int inc[kMaxGroupMembers];
  double ms[kMaxGroupMembers];
  Vec3<double> fs[kMaxGroupMembers], rs[kMaxGroupMembers];
  unsigned char stick[kMaxGroupMembers];
  int n = 0;
  double sm = 0.0, smv = 0.0;
  for (int k = 0; k < cnt; ++k) {
    const int am = mem[k];
    const Vec3<double> pk = ld3(c.rhs_pre, am) + ld3(c.cnext, am);
    const double mk = c.hdiag[c.cverts[am]];
    const Vec3<double> fl = to_local3(B, pk);
    if (fl.x / mk - f0.x / m0 <= 0) {
      inc[n] = k; ms[n] = mk; fs[n] = fl;
      sm = sm + mk; smv = smv + fl.x;
      ++n;
    }
  }
  Vec3<double> r0 = mk3(0.0, 0.0, 0.0);
  for (int k = 0; k < n; ++k) {
    const double fn = (f0.x + smv) * ms[k] / (m0 + sm) - fs[k].x;
    rs[k] = mk3(0.0 + fn, 0.0, 0.0);
    r0.x = r0.x - fn;
    stick[k] = 1;
  }
  for (int round = 0; round <= n; ++round) {
    group_friction(f0, m0, r0, fs, ms, rs, stick, n, mu);
    bool changed = false;
    for (int k = 0; k < n; ++k)
      if (stick[k] && rs[k].y * rs[k].y + rs[k].z * rs[k].z > mu * rs[k].x * rs[k].x) { changed = true; stick[k] = 0; }
    if (!changed) break;
  }
  // the last round's intermediates (same operations as group_friction)
  Vec3<double> pstick = f0, pslide = mk3(0.0, 0.0, 0.0);
  double mstick = m0, mslide = 0.0;
  for (int k = 0; k < n; ++k)
    if (stick[k]) { pstick = pstick + fs[k]; mstick = mstick + ms[k]; }
  for (int k = 0; k < n; ++k)
    if (!stick[k]) { pslide = pslide + fs[k]; mslide = mslide + ms[k]; }
  const Vec3<double> v = div3(pstick, mstick);
  Vec3<double> rel = mk3(0.0, 0.0, 0.0), absv0 = mk3(0.0, 0.0, 0.0);
  double tl = 1.0, mult = 0.0;
  double tk[kMaxGroupMembers], mkk[kMaxGroupMembers];
  Vec3<double> rk[kMaxGroupMembers];
  if (mslide > 0) {
    rel = div3(pslide, mslide) - div3(pstick, mstick);
    tl = sqrt(rel.y * rel.y + rel.z * rel.z);
    rel = div3(rel, tl);
    double fnS = 0.0;
    for (int k = 0; k < n; ++k)
      if (!stick[k]) fnS = fnS + rs[k].x;
    mult = mu * fnS / (mslide + mstick);
    absv0 = div3(f0 + r0, m0);
    for (int k = 0; k < n; ++k)
      if (!stick[k]) {
        rk[k] = div3(fs[k], ms[k]) - absv0;
        tk[k] = sqrt(rk[k].y * rk[k].y + rk[k].z * rk[k].z);
        rk[k] = div3(rk[k], tk[k]);
        mkk[k] = -mu * rs[k].x * ms[k] / (ms[k] + mstick);
      }
  }
  const Vec3<double> v0 = div3(to_world3(B, f0) + to_world3(B, r0), m0);
  // reverse: outputs outF_i = mf_i v0 - P_i, outM_k = B rs_k
  Vec3<double> Pb[3], v0b = mk3(0.0, 0.0, 0.0);
  double mfb[3];
  for (int i = 0; i < 3; ++i) {
    const Vec3<double> G = ld3(a.sbp, fa[i]) + ld3(a.scb, fa[i]);
    v0b = v0b + mf[i] * G;
    mfb[i] = dot3(v0, G);
    Pb[i] = (-1.0) * G;
  }
  Vec3<double> rsb[kMaxGroupMembers], fsb[kMaxGroupMembers];
  double msb[kMaxGroupMembers];
  for (int k = 0; k < n; ++k) {
    const int am = mem[inc[k]];
    rsb[k] = to_local3(B, ld3(a.sbp, am) + ld3(a.scb, am));
    fsb[k] = mk3(0.0, 0.0, 0.0);
    msb[k] = 0.0;
  }
  // v0 = (B f0 + B r0) / m0
  const Vec3<double> ub = div3(v0b, m0);
  double m0b = -dot3(v0b, v0) / m0;
  Vec3<double> f0b = to_local3(B, ub), r0b = to_local3(B, ub);
  double mstickb = 0.0, mslideb = 0.0, fnSb = 0.0;
  Vec3<double> pstickb = mk3(0.0, 0.0, 0.0), pslideb = mk3(0.0, 0.0, 0.0);
  if (mslide > 0) {
    Vec3<double> absv0b = mk3(0.0, 0.0, 0.0);
    for (int k = 0; k < n; ++k) {
      if (stick[k]) continue;
      const double mkb = rsb[k].y * rk[k].y + rsb[k].z * rk[k].z;
      const double ry = mkk[k] * rsb[k].y, rz = mkk[k] * rsb[k].z;
      rsb[k].y = 0.0; rsb[k].z = 0.0;
      const double den = ms[k] + mstick;
      rsb[k].x += mkb * (-mu) * ms[k] / den;
      msb[k] += mkb * (-mu * rs[k].x) * mstick / (den * den);
      mstickb += mkb * (mu * rs[k].x * ms[k]) / (den * den);
      const double dp = rk[k].y * ry + rk[k].z * rz;
      const double wy = (ry - rk[k].y * dp) / tk[k], wz = (rz - rk[k].z * dp) / tk[k];
      fsb[k].y += wy / ms[k]; fsb[k].z += wz / ms[k];
      msb[k] -= (fs[k].y * wy + fs[k].z * wz) / (ms[k] * ms[k]);
      absv0b.y -= wy; absv0b.z -= wz;
    }
    f0b = f0b + (1.0 / m0) * absv0b;
    r0b = r0b + (1.0 / m0) * absv0b;
    m0b -= dot3(absv0b, absv0) / m0;
    Vec3<double> relb = mk3(0.0, 0.0, 0.0);
    double multb = 0.0;
    for (int k = 0; k < n; ++k) {
      if (!stick[k]) continue;
      relb.y += rsb[k].y * mult * ms[k]; relb.z += rsb[k].z * mult * ms[k];
      multb += (rsb[k].y * rel.y + rsb[k].z * rel.z) * ms[k];
      msb[k] += (rsb[k].y * rel.y + rsb[k].z * rel.z) * mult;
    }
    relb.y += r0b.y * mult * m0; relb.z += r0b.z * mult * m0;
    multb += (r0b.y * rel.y + r0b.z * rel.z) * m0;
    m0b += (r0b.y * rel.y + r0b.z * rel.z) * mult;
    const double dm = mslide + mstick;
    fnSb += multb * mu / dm;
    mslideb -= multb * mult / dm;
    mstickb -= multb * mult / dm;
    const double dr = rel.y * relb.y + rel.z * relb.z;
    const double qy = (relb.y - rel.y * dr) / tl, qz = (relb.z - rel.z * dr) / tl;
    pslideb.y += qy / mslide; pslideb.z += qz / mslide;
    mslideb -= (pslide.y * qy + pslide.z * qz) / (mslide * mslide);
    pstickb.y -= qy / mstick; pstickb.z -= qz / mstick;
    mstickb += (pstick.y * qy + pstick.z * qz) / (mstick * mstick);
  }
  Vec3<double> vb = mk3(0.0, 0.0, 0.0);
  for (int k = 0; k < n; ++k) {
    if (!stick[k]) continue;
    vb.y += rsb[k].y * ms[k]; vb.z += rsb[k].z * ms[k];
    msb[k] += rsb[k].y * v.y + rsb[k].z * v.z;
    fsb[k].y -= rsb[k].y; fsb[k].z -= rsb[k].z;
    rsb[k].y = 0.0; rsb[k].z = 0.0;
  }
  vb.y += r0b.y * m0; vb.z += r0b.z * m0;
  m0b += r0b.y * v.y + r0b.z * v.z;
  f0b.y -= r0b.y; f0b.z -= r0b.z;
  pstickb.y += vb.y / mstick; pstickb.z += vb.z / mstick;
  mstickb -= (v.y * vb.y + v.z * vb.z) / mstick;
  for (int k = 0; k < n; ++k) {
    if (stick[k]) { fsb[k] = fsb[k] + pstickb; msb[k] += mstickb; }
    else { fsb[k] = fsb[k] + pslideb; msb[k] += mslideb; rsb[k].x += fnSb; }
  }
  f0b = f0b + pstickb;
  m0b += mstickb;
  // normal parts: rs_k.x = fn_k, r0.x = -sum fn_k,
  // fn_k = (f0.x + smv) ms_k / (m0 + sm) - fs_k.x
  const double A = f0.x + smv, D = m0 + sm;
  double smb = 0.0, smvb = 0.0;
  for (int k = 0; k < n; ++k) {
    const double fnb = rsb[k].x - r0b.x;
    f0b.x += fnb * ms[k] / D;
    smvb += fnb * ms[k] / D;
    msb[k] += fnb * A / D;
    m0b -= fnb * A * ms[k] / (D * D);
    smb -= fnb * A * ms[k] / (D * D);
    fsb[k].x -= fnb;
  }
  for (int k = 0; k < n; ++k) { msb[k] += smb; fsb[k].x += smvb; }
  const Vec3<double> F0wb = to_world3(B, f0b);
  for (int i = 0; i < 3; ++i) {
    st3(a.gPF, 3 * f + i, Pb[i] + F0wb);
    a.gmF[3 * f + i] = mfb[i] + m0b;
  }
  const int gp = rv.g_ptr[f];
  for (int k = 0; k < cnt; ++k) { st3(a.gPM, gp + k, mk3(0.0, 0.0, 0.0)); a.gmM[gp + k] = 0.0; }
  for (int k = 0; k < n; ++k) {
    st3(a.gPM, gp + inc[k], to_world3(B, fsb[k]));
    a.gmM[gp + inc[k]] = msb[k];
  }
}

// Part B (per contact vertex): CollisionHandling's reverse by its outcome
// (as k_contact_rhs_post), the reaction's VJP, the relaxation's remainder;
// the remembered forces' cotangent before the call replaces the one after.
__global__ void k_cadj_self_b(SceneDev d, ContactDev c, ContactAdj a, SelfRec rv, int first,
                              const int* __restrict__ rcnt, const double* __restrict__ rn) {
  const int ac = blockIdx.x * blockDim.x + threadIdx.x;
  if (ac >= c.nc) return;
  const int i = c.cverts[ac];
  const Vec3<double> post_b = ld3(a.sbp, ac), ptot = ld3(a.ptot, ac);
  const int nobs = *rv.nobs, ngrp = *rv.ngrp;
  Vec3<double> rb = post_b;
  if (nobs > 0 || ngrp > 0) {
    Vec3<double> W[3];
    double r0 = 0, r1 = 0, r2 = 0;
    const bool hit = obstacle_winner(c, ac, ld3(c.rhs_pre, ac) + ld3(rv.sc_in, ac), rcnt, rn, W, r0, r1, r2);
    Vec3<double> scb_in = mk3(0.0, 0.0, 0.0);
    if (ngrp == 0) {
      if (hit) {
        rb = reaction_vjp(W, r0, r1, r2, post_b, c.mu);
        scb_in = rb;
      }
    } else {
      Vec3<double> gsum = mk3(0.0, 0.0, 0.0);
      double hsum = 0.0;
      for (int k = c.cvf_ptr[ac]; k < c.cvf_ptr[ac + 1]; ++k) {
        const int f = c.cvf_face[k];
        if (rv.g_cnt[f] == 0) continue;
        const int corner = c.cfaces[3 * f] == ac ? 0 : (c.cfaces[3 * f + 1] == ac ? 1 : 2);
        gsum = gsum + ld3(a.gPF, 3 * f + corner);
        hsum += a.gmF[3 * f + corner];
      }
      if (rv.cf_face[ac] >= 0) {
        gsum = gsum + ld3(a.gPM, rv.m_slot[ac]);
        hsum += a.gmM[rv.m_slot[ac]];
      }
      rb = post_b + gsum;
      if (hit) {
        const Vec3<double> fb = reaction_vjp(W, r0, r1, r2, post_b + gsum, c.mu);
        rb = rb + fb;
        scb_in = fb;
      }
      a.hdb[i] += hsum;
    }
    st3(a.scb, ac, scb_in);
  }
  if (first) {
    rb = rb + (1.0 - c.alpha) * ptot;
    st3(a.pb, i, mk3(0.0, 0.0, 0.0));
  } else {
    st3(a.pb, i, (1.0 - c.alpha) * ptot);
  }
  st3(a.vwcb, i, ld3(a.vwcb, i) + d.mass[i] * rb);
  st3(a.yb, i, d.h * rb);
}

__device__ __forceinline__ void cadj_hs_item(const SceneDev& d, const ContactAdj& a, int i) {
  Vec3<double> o = ld3(a.orib, i);
  double hii = 0.0;
  for (int k = d.hs_ptr[i]; k < d.hs_ptr[i + 1]; ++k) {
    const int j = d.hs_col[k];
    if (j != i) o = o - d.hs_val[k] * ld3(a.yb, j);
    else hii = d.hs_val[k];
  }
  st3(a.cxtb, i, ld3(a.cxtb, i) + (d.mass[i] / (d.h * d.h) - hii) * ld3(a.yb, i));
  st3(a.xn1b, i, o);
}

__global__ void k_cadj_hs(SceneDev d, ContactAdj a, Gate gate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N || gate.skip(vpart_of(d, i))) return;
  cadj_hs_item(d, a, i);
}

// after the reverse sweep: the diag(Hs) terms of the tets' E gradient
__device__ __forceinline__ void cadj_hd_item(const SceneDev& d, const ContactAdj& a, int t, double* gE) {
  int4 v = d.tv[t];
  const int vi[4] = {v.x, v.y, v.z, v.w};
  double G[4][3];
  load_g(d.tinv, d.T, t, G);
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) s += (G[q][0] * G[q][0] + G[q][1] * G[q][1] + G[q][2] * G[q][2]) * a.hdb[vi[q]];
  gE[t] += d.tvol[t] * s;
}

__global__ void k_cadj_hd(SceneDev d, ContactAdj a, double* gE) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.T || !gE) return;
  cadj_hd_item(d, a, t, gE);
}

// The reverse sweep of a step's obstacle contact phase (no soft contact) in
// one cooperative launch: k_cadj_start, then for the recorded computed
// iterations j = top .. 1 (records base + j - 1) the chain of
// contact_adjoint_step's kernels — local step at the iteration's input, the
// rhs VJP, the local VJP, the slot gather with the Hs terms and the
// segments' activation sums — with grid-wide barriers between them, then
// the diag(Hs) terms of dL/dE and the PD part's cotangent.  Same per-item
// code and order as the kernels: bit-identical results.  The records' pass
// flags are read on the device (the kernels' path copies them to the host).
__global__ void __launch_bounds__(128) k_cadj_fused(SceneDev d, ContactDev c, ContactAdj a, const double* xt,
                                                    const double* act_all, const int* step, double* slot, double* gE,
                                                    double* gnu, double* mg, double* gact, int base, int top, double cv,
                                                    double* io_a, double* io_b) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
  const int ncons = d.T + d.M + d.S + d.B;
  const size_t n3 = 3 * (size_t)d.N;
  const int st = *step;
  const double* act_row = act_all + (size_t)st * d.nseg;
  for (int i = tid; i < d.N; i += nthr) {  // k_cadj_start
    const Vec3<double> gv = ld3(io_b, i);
    st3(a.xn1b, i, ld3(io_a, i) + cv * gv);
    st3(a.cxtb, i, (-cv) * gv);
    st3(a.vwcb, i, mk3(0.0, 0.0, 0.0));
    st3(a.pb, i, mk3(0.0, 0.0, 0.0));
    a.hdb[i] = 0.0;
  }
  grid.sync();
  for (int j = top; j >= 1; --j) {
    const size_t r = (size_t)base + (j - 1);
    const double* ori = c.rec_x + r * n3;
    const double* prev = c.rec_prev + r * n3;
    const int* rcnt = c.rec_cnt + r * c.nc;
    const double* rn = c.rec_n + r * c.nc * kMaxImpactsPerVertex * 3;
    const int first = c.rec_first[r];
    for (int t = tid; t < ncons; t += nthr) local_item(d, t, ori, act_all, step, slot);
    grid.sync();
    for (int i = tid; i < d.N; i += nthr) cadj_rhs_item(d, c, a, i, slot, xt, ori, prev, first, rcnt, rn);
    grid.sync();
    for (int t = tid; t < ncons; t += nthr) adj_local_item(d, t, ori, a.yb, act_row, slot, gE, gnu, mg, nullptr, xt);
    grid.sync();
    for (int i = tid; i < d.N; i += nthr) {  // k_adj_gather_seq, then k_cadj_hs on the same vertex
      Vec3<double> acc = mk3(0.0, 0.0, 0.0);
      for (int k = d.vslot_ptr[i]; k < d.vslot_ptr[i + 1]; ++k) acc = acc + ld3(slot, k);
      st3(a.orib, i, acc);
      cadj_hs_item(d, a, i);
    }
    for (int q = tid; q < d.nseg; q += nthr) {  // k_seg_reduce
      double sum = 0;
      for (int k = d.seg_ptr[q]; k < d.seg_ptr[q + 1]; ++k) sum += mg[member_slot(d.M, d.seg_mus[k])];
      gact[(size_t)st * d.nseg + q] += sum;
    }
    grid.sync();
  }
  for (int t = tid; t < d.T; t += nthr) cadj_hd_item(d, a, t, gE);
  for (int i = tid; i < d.N; i += nthr) {  // k_cadj_to_pd
    st3(io_a, i, ld3(a.xn1b, i));
    st3(io_b, i, mk3(0.0, 0.0, 0.0));
  }
}

// The reverse sweep of a batch's obstacle contact phase in one cooperative
// launch: k_cadj_fused for every part, part p reversing its own computed
// iterations top[p] .. 1 (its records base + j - 1, pass flags
// rec_first[(base + j - 1) np + p]); the sweeps run side by side, iteration j
// of every part that has one in the same round.  Same per-item code as
// k_cadj_fused.
__global__ void __launch_bounds__(128) k_cadj_fused_parts(SceneDev d, ContactDev c, ContactAdj a, const double* xt,
                                                          const double* act_all, const int* step, double* slot,
                                                          double* gE, double* gnu, double* mg, double* gact, int base,
                                                          const int* top, double cv, double* io_a, double* io_b) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
  const int ncons = d.T + d.M + d.S + d.B, np = c.np;
  const size_t n3 = 3 * (size_t)d.N;
  const int st = *step;
  const double* act_row = act_all + (size_t)st * d.nseg;
  for (int i = tid; i < d.N; i += nthr) {  // k_cadj_start
    const Vec3<double> gv = ld3(io_b, i);
    st3(a.xn1b, i, ld3(io_a, i) + cv * gv);
    st3(a.cxtb, i, (-cv) * gv);
    st3(a.vwcb, i, mk3(0.0, 0.0, 0.0));
    st3(a.pb, i, mk3(0.0, 0.0, 0.0));
    a.hdb[i] = 0.0;
  }
  int jmax = 0;
  for (int p = 0; p < np; ++p) jmax = max(jmax, top[p]);
  grid.sync();
  for (int j = jmax; j >= 1; --j) {
    const size_t r = (size_t)base + (j - 1);
    const double* ori = c.rec_x + r * n3;
    const double* prev = c.rec_prev + r * n3;
    const int* rcnt = c.rec_cnt + r * c.nc;
    const double* rn = c.rec_n + r * c.nc * kMaxImpactsPerVertex * 3;
    for (int t = tid; t < ncons; t += nthr)
      if (j <= top[cons_part(d, t)]) local_item(d, t, ori, act_all, step, slot);
    grid.sync();
    for (int i = tid; i < d.N; i += nthr) {
      const int p = vpart_of(d, i);
      if (j <= top[p]) cadj_rhs_item(d, c, a, i, slot, xt, ori, prev, c.rec_first[r * np + p], rcnt, rn);
    }
    grid.sync();
    for (int t = tid; t < ncons; t += nthr)
      if (j <= top[cons_part(d, t)]) adj_local_item(d, t, ori, a.yb, act_row, slot, gE, gnu, mg, nullptr, xt);
    grid.sync();
    for (int i = tid; i < d.N; i += nthr) {  // k_adj_gather_seq, then k_cadj_hs on the same vertex
      if (j > top[vpart_of(d, i)]) continue;
      Vec3<double> acc = mk3(0.0, 0.0, 0.0);
      for (int k = d.vslot_ptr[i]; k < d.vslot_ptr[i + 1]; ++k) acc = acc + ld3(slot, k);
      st3(a.orib, i, acc);
      cadj_hs_item(d, a, i);
    }
    for (int q = tid; q < d.nseg; q += nthr) {  // k_seg_reduce
      if (j > top[d.seg_part ? d.seg_part[q] : 0]) continue;
      double sum = 0;
      for (int k = d.seg_ptr[q]; k < d.seg_ptr[q + 1]; ++k) sum += mg[member_slot(d.M, d.seg_mus[k])];
      gact[(size_t)st * d.nseg + q] += sum;
    }
    grid.sync();
  }
  for (int t = tid; t < d.T; t += nthr) cadj_hd_item(d, a, t, gE);
  for (int i = tid; i < d.N; i += nthr) {  // k_cadj_to_pd
    st3(io_a, i, ld3(a.xn1b, i));
    st3(io_b, i, mk3(0.0, 0.0, 0.0));
  }
}

// the PD part's input cotangent is the phase's input cotangent; the step's
// own v' term went to x_t bar
__global__ void k_cadj_to_pd(int N, ContactAdj a, double* io_a, double* io_b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  st3(io_a, i, ld3(a.xn1b, i));
  st3(io_b, i, mk3(0.0, 0.0, 0.0));
}

// after the PD adjoint: add the contact phase's x_t and v_wc (= v) cotangents
__global__ void k_cadj_finish(int N, ContactAdj a, double* io_a, double* io_b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  st3(io_a, i, ld3(io_a, i) + ld3(a.cxtb, i));
  st3(io_b, i, ld3(io_b, i) + ld3(a.vwcb, i));
}

}  // namespace dfem
