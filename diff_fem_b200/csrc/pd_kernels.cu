// pd_kernels.cu — the PD step kernels (FP64 plain form) and the adjoint kernels.
//
// One time step (diff_fem World::TimeStepping + ProjectiveDynamicsMethod,
// sim/fem/World.h:673-720, 835-917) is this kernel sequence, captured once as
// a CUDA graph and replayed for every step:
//   k_step_begin        v_wc = v + g h (+ h f_drag / m), q_n = x + h v_wc, c0 = M/h^2 q_n - Hs x + J_att d_att,
//                       x^0 = q_n, convergence test of the reference's first iteration
//   K x { k_local       per-constraint projection d and its J*d slot contributions
//         k_gather      rhs_i = c0_i + sum of vertex i's slots           (ori_c - Qf x)
//         k_fwd_level   L y = rhs, one launch per level of the supernodal tree
//         k_bwd_level   L^T z = y, levels in reverse (z = hvf)
//         k_update      x^{k+1} = x + z, ||x^{k+1}-x^k|| / 3N < 5e-7 -> converged flag }
//   k_step_end          v = damping (x^K - x)/h, x = x^K
#include "kernels.cuh"

namespace dfem {

// ------------------------------------------------------------- utilities ----

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic per-part reduction over part-aligned blocks: every block of
// the part writes its partial sum, the last block of the part to finish
// (counter) adds the partials b0 .. b0+nb-1 in block order.  Returns true in
// thread 0 of that block, with *total set.
__device__ bool part_reduce(double v, double* partial, unsigned* counter, int b0, int nb, double* total) {
  __shared__ double ws[32];
  __shared__ bool last;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) s += ws[w];
    partial[blockIdx.x] = s;
    __threadfence();
    unsigned ticket = atomicAdd(counter, 1u);
    last = (ticket == (unsigned)nb - 1);
  }
  __syncthreads();
  if (!last) return false;
  if (threadIdx.x == 0) {
    __threadfence();
    double s = 0;
    for (int b = b0; b < b0 + nb; ++b) s += ((volatile double*)partial)[b];
    *total = s;
    *counter = 0u;
    return true;
  }
  return false;
}

__device__ __forceinline__ Vec3<double> ld3(const double* p, int i) {
  return mk3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
__device__ __forceinline__ void st3(double* p, int i, Vec3<double> v) {
  p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z;
}

// G[v][j] coefficients from invDm planes: F(:,j) = sum_v G[v][j] x_v
__device__ __forceinline__ void load_g(const double* inv, int n, int e, double G[4][3]) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double a = inv[(0 * 3 + j) * n + e], b = inv[(1 * 3 + j) * n + e], c = inv[(2 * 3 + j) * n + e];
    G[1][j] = a; G[2][j] = b; G[3][j] = c;
    G[0][j] = -(a + b + c);
  }
}

__device__ __forceinline__ Mat3<double> deformation(const double G[4][3], const Vec3<double> xv[4]) {
  Mat3<double> F;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    F.c[j] = G[0][j] * xv[0] + G[1][j] * xv[1] + G[2][j] * xv[2] + G[3][j] * xv[3];
  return F;
}

// Minimum resident CTAs per SM asked of the register allocator for the
// heaviest per-constraint kernels (128 threads each): more resident warps hide
// the FP64 latency chains better than the registers they give up (the
// adjoint local step of the 256-scene batch: 1.12 ms at 174 registers, 0.85 ms
// at 128 with spills to L1; the mixed force step, then with an FP32 tail after
// its SVD, 0.315 -> 0.282 ms, the FP64 local step 0.411 -> 0.383 ms; the
// mixed force step with its FP64 tail takes 0.311 ms at 96 registers).  With
// the adjoint's projection and VJP sharing one SVD, three CTAs (168 registers,
// 40 bytes of spills) beat four (128, 360 bytes of spills) and two (255):
// 32-scene batch 104.6 / 107.1 / 135.3 us, inverse-stiffness beam 13.6 /
// 14.5 / 13.6 us per launch.
#ifndef DFEM_FORCE_MIN_BLOCKS
#define DFEM_FORCE_MIN_BLOCKS 5
#endif
#ifndef DFEM_ADJ_MIN_BLOCKS
#define DFEM_ADJ_MIN_BLOCKS 3
#endif
#ifndef DFEM_LOCAL_MIN_BLOCKS
#define DFEM_LOCAL_MIN_BLOCKS 5
#endif

// --------------------------------------------------------------- forward ----

// hist_step: doubles between the iterate records of consecutive steps (0: one
// record shared by all steps, the adjoint recomputes each step).
// v_wc of vertex i: v + g h (gravity-enabled vertices) + h f_drag / m (underwater: the
// drag and lift of the vertex's faces, ascending face order, from d.fdrag).
__device__ __forceinline__ Vec3<double> step_vwc(const SceneDev& d, int i, Vec3<double> v) {
  double gm = d.gmask[i] * d.h;
  Vec3<double> vwc = mk3(v.x + gm * d.g0, v.y + gm * d.g1, v.z + gm * d.g2);
  if (d.vf_ptr) {
    Vec3<double> f = mk3(0.0, 0.0, 0.0);
    for (int k = d.vf_ptr[i]; k < d.vf_ptr[i + 1]; ++k) f = f + ld3(d.fdrag, d.vf_face[k] / 3);
    const double m = d.mass[i];
    vwc = vwc + mk3(d.h * (f.x / m), d.h * (f.y / m), d.h * (f.z / m));
  }
  return vwc;
}

__global__ void k_step_begin(SceneDev d, PartDev pd, const int* step, double* xt, double* vt, double* qn,
                             double* c0, double* xk, double* hist, long long hist_step, int ckpt_every,
                             double* ckpt_x, double* ckpt_v,
                             int* flag, int* iters, double* partial, unsigned* counter, double* errv,
                             int* status, double* vwc_out) {
  const int b = blockIdx.x, p = pd.blk_part[b];
  const int pv0 = pd.part_v0[p], pv1 = pd.part_v0[p + 1];
  const int i = pd.blk_v0[b] + threadIdx.x;
  const int s = *step;
  if (hist) hist += (size_t)s * hist_step;
  double q2 = 0;
  if (i < pv1) {
    Vec3<double> x = ld3(xt, i), v = ld3(vt, i);
    if (ckpt_x && s % ckpt_every == 0) {  // the start state of every ckpt_every-th step
      const size_t slot = (size_t)(s / ckpt_every) * 3 * d.N;
      st3(ckpt_x + slot, i, x);
      st3(ckpt_v + slot, i, v);
    }
    // Environment::Step adds g h to v (gravity-enabled bodies); TimeStepping:
    // v_wc = v + h M^-1 f_ext (f_ext = 0), q_n = x + h v_wc
    const Vec3<double> vwc = step_vwc(d, i, v);
    if (vwc_out) st3(vwc_out, i, vwc);
    Vec3<double> q = x + d.h * vwc;
    st3(qn, i, q);
    st3(xk, i, q);
    if (hist) st3(hist, i, q);
    // c0 = M/h^2 q_n - Hs x + J_att d_att   (b - Qf*mNonrigidX plus the constant attachment term)
    double m = d.mass[i] / (d.h * d.h);
    Vec3<double> acc = m * q;
    for (int k = d.hs_ptr[i]; k < d.hs_ptr[i + 1]; ++k) {
      double a = d.hs_val[k];
      Vec3<double> xj = ld3(xt, d.hs_col[k]);
      acc = acc - a * xj;
    }
    acc = acc + ld3(d.attach_jd, i);
    st3(c0, i, acc);
    q2 = dot3(q, q);
  }
  if (threadIdx.x == 0 && b == pd.part_b0[p]) iters[(size_t)s * pd.nparts + p] = 0;
  double tot;
  if (part_reduce(q2, partial, counter + p, pd.part_b0[p], pd.part_b0[p + 1] - pd.part_b0[p], &tot)) {
    // iteration 0 of the reference compares q_n with a zero vector
    double e = sqrt(tot) / (3.0 * (pv1 - pv0));
    errv[p] = e;
    flag[p] = (e < kConvergenceEps) ? 1 : 0;
    if (!isfinite(tot)) *status = 4;
  }
}

// Projected length of spring t: its rest length, times its channel's
// activation for a pneumatic spring (md = m_rest_length * mActivationLevel * e,
// pneumaticEasy.h:133-147).
__device__ __forceinline__ double spring_length(const SceneDev& d, int t, const double* act_row) {
  const double r = d.srest[t];
  if (!d.sch) return r;
  const int c = d.sch[t];
  return c < 0 ? r : r * act_row[c];
}

// Local step of constraint t (tets, muscles, springs, bending stencils in
// that order): its projection and its J*d contribution to its slots.  The
// pointers are not restrict-qualified: a kernel that writes x in an earlier
// phase of the same launch (k_contact_fused) must not read it through the
// read-only data path.
__device__ __forceinline__ void local_item(const SceneDev& d, int t, const double* x, const double* act_all,
                                           const int* step, double* slot) {
  if (t < d.T) {
    // corotated FEM (CorotateFEMConstraint::EvaluateDVector + EvaluateJMatrix)
    int4 v = d.tv[t];
    Vec3<double> xv[4] = {ld3(x, v.x), ld3(x, v.y), ld3(x, v.z), ld3(x, v.w)};
    double G[4][3];
    load_g(d.tinv, d.T, t, G);
    Mat3<double> F = deformation(G, xv), md, mdv;
    corot_project(F, md, mdv);
    double wr = d.twr[t], wv = d.twv[t];
    Vec3<double> P[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) P[j] = wr * md.c[j] + wv * mdv.c[j];
    int4 sl = d.tslot[t];
    const int sv[4] = {sl.x, sl.y, sl.z, sl.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) st3(slot, sv[a], G[a][0] * P[0] + G[a][1] * P[1] + G[a][2] * P[2]);
    return;
  }
  t -= d.T;
  if (t < d.M) {
    // muscle (LinearMuscleConstraint::Computep0 + EvaluateJMatrix): d = (1-a) F f
    int4 v = d.mv[t];
    Vec3<double> xv[4] = {ld3(x, v.x), ld3(x, v.y), ld3(x, v.z), ld3(x, v.w)};
    double G[4][3];
    load_g(d.minv, d.M, t, G);
    Vec3<double> f = mk3(d.mfib[t], d.mfib[d.M + t], d.mfib[2 * d.M + t]);
    double c[4];
    Vec3<double> Ff = mk3(0.0, 0.0, 0.0);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      c[a] = G[a][0] * f.x + G[a][1] * f.y + G[a][2] * f.z;
      Ff = Ff + c[a] * xv[a];
    }
    double a_act = act_all[(size_t)(*step) * d.nseg + d.mseg[t]];
    Vec3<double> p0 = (1.0 - a_act) * Ff;
    double w = d.mw[t];
    int4 sl = d.mslot[t];
    const int sv[4] = {sl.x, sl.y, sl.z, sl.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) st3(slot, sv[a], (w * c[a]) * p0);
    return;
  }
  t -= d.M;
  if (t < d.S) {
    // spring (SpringConstraint::EvaluateDVector): d = rest * (x0-x1)/|x0-x1|, J = sqrt(w) [I; -I];
    // pneumatic spring (PneumaticConstraint::EvaluateDVector): rest * activation
    int2 v = d.sv[t];
    Vec3<double> e = ld3(x, v.x) - ld3(x, v.y);
    Vec3<double> dd = (spring_length(d, t, act_all + (size_t)(*step) * d.nseg) * rsqrt(dot3(e, e))) * e;
    double w = d.ssw[t];
    int2 sl = d.sslot[t];
    st3(slot, sl.x, w * dd);
    st3(slot, sl.y, (-w) * dd);
    return;
  }
  t -= d.S;
  if (t < d.B) {
    // bending (BendingConstraint::EvaluateDVector): d = w * lap * rest/|lap|, J = w beta
    int o0 = d.boff[t], o1 = d.boff[t + 1];
    Vec3<double> lap = mk3(0.0, 0.0, 0.0);
    for (int k = o0; k < o1; ++k) lap = lap + d.bbeta[k] * ld3(x, d.bv[k]);
    double ln = sqrt(dot3(lap, lap));
    double w = d.bw[t];
    Vec3<double> dd = mk3(0.0, 0.0, 0.0);
    if (ln > 1e-25) dd = (w * d.brest[t] / ln) * lap;
    for (int k = o0; k < o1; ++k) st3(slot, d.bslot[k], (w * d.bbeta[k]) * dd);
  }
}

// Local step: every constraint projects and writes its J*d contribution to its
// slots.  One thread per constraint; constraint types are consecutive ranges.
__global__ void __launch_bounds__(128, DFEM_LOCAL_MIN_BLOCKS) k_local(SceneDev d, Gate gate, const double* __restrict__ x,
                                               const double* __restrict__ act_all, const int* step,
                                               double* __restrict__ slot) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (gate.skip(cons_part(d, t))) return;
  local_item(d, t, x, act_all, step, slot);
}

// ---- mixed form: FP32 projections, FP32 slots and accumulation ----------------
// Positions stay FP64; each element forms Ds = x_k - x_0 in FP64 (no
// cancellation from absolute coordinates), then projects in FP32.  Elements
// that are nearly flat or inverted (smallest/largest singular value below
// kDegenerateRatio) are recomputed in FP64.

__device__ __forceinline__ Vec3<float> to_f(Vec3<double> a) { return mk3((float)a.x, (float)a.y, (float)a.z); }
__device__ __forceinline__ Vec3<double> to_d(Vec3<float> a) { return mk3((double)a.x, (double)a.y, (double)a.z); }
__device__ __forceinline__ void st3f(float* p, int i, Vec3<float> v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
__device__ __forceinline__ Vec3<float> ld3f(const float* p, int i) { return mk3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

// ------------------------------------------------------------ mixed form ----
//
// The mixed form writes, per constraint, its force f_c = J_c d_c - L_c x (the
// part of the rhs that varies with the iterate; strain-sized) as FP32 slots,
// and iterates x^{k+1} = x^k + Hs^-1 r with
//   r = M/h^2 (q_n - x^k) + sum_att k (p - x^k) + sum_c f_c,
// which is the reference's map b + J d(x^k) - Hs x rearranged (Hs = M/h^2 +
// sum_c L_c).  FP32 rounding is then relative to the forces, not to J d ~ L x.
// Inputs of cancelling differences (F, spring lengths, Laplacians) are formed
// in FP64 first; each slot is rounded to FP32 once, from an FP64 value, and a
// vertex's slots are summed in FP64.

__global__ void __launch_bounds__(128, DFEM_FORCE_MIN_BLOCKS) k_force_f32(SceneDev d, Gate gate, const double* __restrict__ x,
                                                   const double* __restrict__ act_all, const int* step,
                                                   float* __restrict__ slot) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (gate.skip(cons_part(d, t))) return;
  if (t < d.T) {
    int4 v = d.tv[t];
    Vec3<double> xv[4] = {ld3(x, v.x), ld3(x, v.y), ld3(x, v.z), ld3(x, v.w)};
    double G[4][3];
    load_g(d.tinv, d.T, t, G);
    const Mat3<double> F = deformation(G, xv);
    const double wr = d.twr[t], wv = d.twv[t];
    Vec3<double> P[3];
    if (!corot_force_mixed(F, wr, wv, P)) {  // inverted or near-degenerate: FP64
      Mat3<double> md, mdv;
      corot_project(F, md, mdv);
#pragma unroll
      for (int j = 0; j < 3; ++j) P[j] = wr * (md.c[j] - F.c[j]) + wv * (mdv.c[j] - F.c[j]);
    }
    // corner forces G_a P (their sum cancels to zero), each rounded once into its FP32 slot
    int4 sl = d.tslot[t];
    const int sv[4] = {sl.x, sl.y, sl.z, sl.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) st3f(slot, sv[a], to_f(G[a][0] * P[0] + G[a][1] * P[1] + G[a][2] * P[2]));
    return;
  }
  t -= d.T;
  if (t < d.M) {  // -a w c_a (F f): J d - L x of the muscle constraint
    int4 v = d.mv[t];
    const Vec3<double> x0 = ld3(x, v.x);
    const Vec3<double> ds[3] = {ld3(x, v.y) - x0, ld3(x, v.z) - x0, ld3(x, v.w) - x0};
    const Vec3<double> f = mk3(d.mfib[t], d.mfib[d.M + t], d.mfib[2 * d.M + t]);
    double c[4] = {0, 0, 0, 0};
    Vec3<double> Ff = mk3(0.0, 0.0, 0.0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double ck = d.minv[(k * 3 + 0) * d.M + t] * f.x + d.minv[(k * 3 + 1) * d.M + t] * f.y +
                  d.minv[(k * 3 + 2) * d.M + t] * f.z;
      c[k + 1] = ck;
      c[0] -= ck;
      Ff = Ff + ck * ds[k];
    }
    const double a_act = act_all[(size_t)(*step) * d.nseg + d.mseg[t]];
    const Vec3<double> p = (-a_act * d.mw[t]) * Ff;
    int4 sl = d.mslot[t];
    const int sv[4] = {sl.x, sl.y, sl.z, sl.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) st3f(slot, sv[a], to_f(c[a] * p));
    return;
  }
  t -= d.M;
  if (t < d.S) {  // sqrt(w) e (rest/|e| - 1)
    int2 v = d.sv[t];
    const Vec3<double> e = ld3(x, v.x) - ld3(x, v.y);
    const double len = sqrt(dot3(e, e));
    const Vec3<float> fs =
        to_f((d.ssw[t] * (spring_length(d, t, act_all + (size_t)(*step) * d.nseg) / len - 1.0)) * e);
    int2 sl = d.sslot[t];
    st3f(slot, sl.x, fs);
    st3f(slot, sl.y, (-1.0f) * fs);
    return;
  }
  t -= d.S;
  if (t < d.B) {  // w^2 beta_q (rest/|lap| - w) lap
    int o0 = d.boff[t], o1 = d.boff[t + 1];
    const Vec3<double> xc = ld3(x, d.bv[o0]);
    Vec3<double> lap = mk3(0.0, 0.0, 0.0);
    for (int k = o0 + 1; k < o1; ++k) lap = lap + d.bbeta[k] * (ld3(x, d.bv[k]) - xc);  // sum beta = 0
    const double ln = sqrt(dot3(lap, lap)), w = d.bw[t];
    const double sc = w * w * ((ln > 1e-25 ? d.brest[t] / ln : 0.0) - w);
    const Vec3<double> fl = sc * lap;
    for (int k = o0; k < o1; ++k) st3f(slot, d.bslot[k], to_f(d.bbeta[k] * fl));
  }
}

// r_i = m_i/h^2 (q_i - x_i) + attach_jd_i - attach_k_i x_i + the sum of vertex i's FP32 force
// slots, accumulated in FP64 (the slots' own rounding is then the only FP32 error of the rhs)
__global__ void k_gather_force(SceneDev d, Gate gate, const float* __restrict__ slot, const double* __restrict__ qn,
                               const double* __restrict__ x, double* __restrict__ rhs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N || gate.skip(vpart_of(d, i))) return;
  Vec3<double> acc = mk3(0.0, 0.0, 0.0);
  for (int k = d.vslot_ptr[i]; k < d.vslot_ptr[i + 1]; ++k) acc = acc + to_d(ld3f(slot, k));
  const Vec3<double> xi = ld3(x, i);
  const double m = d.mass[i] / (d.h * d.h);
  st3(rhs, i, m * (ld3(qn, i) - xi) + ld3(d.attach_jd, i) - d.attach_k[i] * xi + acc);
}

// rhs_i = c0_i + sum of the slots of vertex i
// Sum of a vertex's slots by one warp: lane l adds slots k0 + l, k0 + l + 32,
// ... in order, then the warp's fixed reduction tree (all lanes get the sum).
__device__ __forceinline__ Vec3<double> warp_sum_slots(const double* __restrict__ slot, int k0, int k1) {
  Vec3<double> acc = mk3(0.0, 0.0, 0.0);
  for (int k = k0 + (int)(threadIdx.x & 31); k < k1; k += 32) acc = acc + ld3(slot, k);
  return mk3(warp_sum(acc.x), warp_sum(acc.y), warp_sum(acc.z));
}

// The same sum by one thread, bit for bit: the lanes' partial sums (lane l:
// +0 + slot k0 + l + slot k0 + l + 32 + ...) combined by the warp's reduction
// tree, which is pairwise summation over the lanes in bit-reversed order
// (floating-point addition is commutative, so only the tree's shape matters).
__device__ __forceinline__ Vec3<double> thread_sum_slots(const double* __restrict__ slot, int k0, int k1) {
  Vec3<double> stk[5];
#pragma unroll
  for (int j = 0; j < 32; ++j) {  // unrolled: every index into stk is a constant
    const int l = (int)(__brev((unsigned)j) >> 27);
    Vec3<double> x = mk3(0.0, 0.0, 0.0);
    for (int k = k0 + l; k < k1; k += 32) x = x + ld3(slot, k);
    int b = 0;
#pragma unroll
    for (int q = 0; q < 5; ++q)
      if (b == q && ((j >> q) & 1)) {
        x = stk[q] + x;
        b = q + 1;
      }
    if (j == 31) return x;  // the whole tree
#pragma unroll
    for (int q = 0; q < 5; ++q)
      if (q == b) stk[q] = x;
  }
  return stk[0];  // not reached
}

// the slot sums' form: one warp per vertex below this many vertices (latency),
// one thread per vertex from it on (the same sums, bit for bit)
constexpr int kGatherThreadMin = 65536;

// rhs = c0 + J d, one thread per vertex
__global__ void k_gather_t(int N, Gate gate, const int* __restrict__ vpart, const int* __restrict__ vslot_ptr,
                           const double* __restrict__ slot, const double* __restrict__ c0, double* __restrict__ rhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || gate.skip(vpart ? vpart[i] : 0)) return;
  st3(rhs, i, ld3(c0, i) + thread_sum_slots(slot, vslot_ptr[i], vslot_ptr[i + 1]));
}

// rhs = c0 + J d: one warp per vertex (32 vertices' threads per 1024)
__global__ void k_gather(int N, Gate gate, const int* __restrict__ vpart, const int* __restrict__ vslot_ptr,
                             const double* __restrict__ slot,
                         const double* __restrict__ c0, double* __restrict__ rhs) {
  const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (i >= N || gate.skip(vpart ? vpart[i] : 0)) return;  // uniform over the warp
  const Vec3<double> s = warp_sum_slots(slot, vslot_ptr[i], vslot_ptr[i + 1]);
  if ((threadIdx.x & 31) == 0) st3(rhs, i, ld3(c0, i) + s);
}

// ----------------------------------------------------------- solves ----
//
// A supernode is solved by a group of threads: a whole CTA, or one warp of a
// CTA that solves several small supernodes side by side (one per warp).  The
// order of every sum is fixed by the supernode alone, not by the group, so the
// two forms, every CTA size and the persistent solve give bit-identical
// results.
struct CtaGroup {
  __device__ static int rank() { return threadIdx.x; }
  __device__ static int size() { return blockDim.x; }
  __device__ static int warp() { return threadIdx.x >> 5; }
  __device__ static int nwarps() { return blockDim.x >> 5; }
  __device__ static int index_in_block() { return 0; }
  __device__ static int per_block() { return 1; }
  __device__ static void sync() { __syncthreads(); }
  __device__ static bool all(bool p) { return __syncthreads_and(p ? 1 : 0) != 0; }
};
struct WarpGroup {
  __device__ static int rank() { return threadIdx.x & 31; }
  __device__ static int size() { return 32; }
  __device__ static int warp() { return 0; }
  __device__ static int nwarps() { return 1; }
  __device__ static int index_in_block() { return threadIdx.x >> 5; }
  __device__ static int per_block() { return blockDim.x >> 5; }
  __device__ static void sync() { __syncwarp(); }
  __device__ static bool all(bool p) {
    const bool r = __all_sync(0xffffffffu, p) != 0;
    __syncwarp();
    return r;
  }
};

__device__ __forceinline__ int even_count(int v) { return (v + 1) & ~1; }

// Shared memory of one supernode solve (doubles; the bulk-copy targets start
// at even offsets, i.e. 16-byte aligned):
//   D (even(w*w)) | L_{R,s} (even(r*w), if staged) | t (3w) | ...
//   forward:  ... | y_s (3w) | contributions (3 nseg) | row -> contribution range (w + 1 ints)
//   backward: ... | x_R (3r)
// (solve_shm_doubles in engine.cu sizes it.)

// Rows per thread of a streamed forward panel (its accumulators live in
// registers); a supernode with more rows than kStreamRows x the group size
// reads L_{R,s} from global memory instead.
constexpr int kStreamRows = 4;

template <class G>
__device__ __forceinline__ bool streamed(const SnInfo& in) {
  return !in.stage && in.cc > 0 && in.r <= kStreamRows * G::size();
}

// Doubles of the L_{R,s} region: the whole block (staged), two chunk buffers
// (streamed), or nothing.
__device__ __forceinline__ int lsh_doubles(const SnInfo& in) {
  return in.stage ? even_count(in.r * in.w) : in.cc > 0 ? 2 * in.cc * in.r : 0;
}

// Chunk k of a streamed L_{R,s} (columns k cc .. min(w, (k+1) cc), one
// contiguous range of the column-major block; cc is even, so every chunk but
// the last starts and ends on 16 bytes, and the last one's rounding stays
// inside the block's even-padded storage) into buffer k & 1.
__device__ __forceinline__ void issue_chunk(const FactorDev& f, const SnInfo& in, int k, double* Lsh, uint64_t* sbar) {
  const int c0 = k * in.cc, nc = min(in.cc, in.w - c0);
  const unsigned bytes = (unsigned)(even_count(nc * in.r) * sizeof(double));
  mbar_expect_tx(sbar + (k & 1), bytes);
  bulk_copy_g2s(Lsh + (size_t)(k & 1) * in.cc * in.r, f.Lcm + in.lofs + (size_t)c0 * in.r, bytes, sbar + (k & 1));
}

// Stage the diagonal-block inverse (column-major for the forward solve,
// row-major for the backward) and, if in.stage, L_{R,s}; for a streamed
// L_{R,s}, start its first two chunks.  Rank 0 of the group issues the bulk
// copies.  The proxy fence orders the group's earlier generic reads of the
// same shared memory (a previous supernode of the persistent solve) before
// the bulk writes.
template <class G>
__device__ __forceinline__ void stage_blocks_issue(const FactorDev& f, const SnInfo& in, bool fwd, double* Dsh,
                                                   double* Lsh, uint64_t* bar, uint64_t* sbar) {
  if (G::rank() == 0) {
    const unsigned bd = (unsigned)(even_count(in.w * in.w) * sizeof(double));
    const unsigned bl = in.stage ? (unsigned)(even_count(in.r * in.w) * sizeof(double)) : 0u;
    fence_proxy_async_smem();
    mbar_expect_tx(bar, bd + bl);
    bulk_copy_g2s(Dsh, (fwd ? f.DinvC : f.Dinv) + in.dofs, bd, bar);
    if (bl) bulk_copy_g2s(Lsh, f.Lcm + in.lofs, bl, bar);
    if (streamed<G>(in)) {
      issue_chunk(f, in, 0, Lsh, sbar);
      if (in.cc < in.w) issue_chunk(f, in, 1, Lsh, sbar);
    }
  }
}

// Let a streamed block's copies still in flight land (an aborted item).
template <class G>
__device__ __forceinline__ void drain_chunks(const SnInfo& in, uint64_t* sbar, const unsigned* sph) {
  if (G::rank() == 0 && streamed<G>(in)) {
    mbar_wait_bounded(sbar, sph[0]);
    if (in.cc < in.w) mbar_wait_bounded(sbar + 1, sph[1]);
  }
}

// A bounded wait gave up: status[0] = 6 (DFEM_ERR_CAP), status[1] = the
// supernode, status[2] = which wait (1 forward / 2 backward staging, 3 / 4
// persistent-solve dependency), status[3] counts the groups that gave up.
__device__ __forceinline__ void record_gave_up(const FactorDev& f, int s, int which) {
  f.status[0] = 6;
  f.status[1] = s;
  f.status[2] = which;
  atomicAdd(f.status + 3, 1);
}

// Wait for the staged blocks (phase parity `phase` of the barrier); false,
// uniformly across the group, when the bounded wait gave up.  Includes the
// group barrier.
template <class G>
__device__ __forceinline__ bool stage_blocks_wait(const FactorDev& f, uint64_t* bar, unsigned phase, int s, int which) {
  const bool ok = G::all(mbar_wait_bounded(bar, phase));
  if (!ok && G::rank() == 0) {
    record_gave_up(f, s, which);
    mbar_wait_bounded(bar, phase);  // give in-flight copies one more bounded chance to land
  }
  return ok;
}

// Wait for chunk k of a streamed block (buffer k & 1); false, uniformly across
// the group, when the bounded wait gave up (after letting the chunks still in
// flight land).
template <class G>
__device__ __forceinline__ bool wait_chunk(const FactorDev& f, const SnInfo& in, int k, int nch, uint64_t* sbar,
                                           unsigned* sph, int which) {
  const int b = k & 1;
  if (G::all(mbar_wait_bounded(sbar + b, sph[b]))) {
    sph[b] ^= 1u;
    return true;
  }
  if (G::rank() == 0) {
    record_gave_up(f, in.s, which);
    mbar_wait_bounded(sbar + b, sph[b]);
    if (k + 1 < nch) mbar_wait_bounded(sbar + (b ^ 1), sph[b ^ 1]);
  }
  return false;
}

// L_{R,s} y_s into the contribution slots with L_{R,s} streamed through two
// shared buffers: rows rk, rk + gs, .. of a thread accumulate in registers
// over the chunks, each row's sum in column order.
template <class G>
__device__ __forceinline__ bool fwd_panel_stream(const FactorDev& f, const SnInfo& in, double* Lsh, uint64_t* sbar,
                                                 unsigned* sph, const double* __restrict__ ysh) {
  const int r = in.r, w = in.w, cc = in.cc, rk = G::rank(), gs = G::size();
  const int nch = (w + cc - 1) / cc;
  double acc[kStreamRows][3];
#pragma unroll
  for (int j = 0; j < kStreamRows; ++j) acc[j][0] = acc[j][1] = acc[j][2] = 0.0;
  for (int k = 0; k < nch; ++k) {
    if (!wait_chunk<G>(f, in, k, nch, sbar, sph, 5)) return false;
    const double* Lb = Lsh + (size_t)(k & 1) * cc * r;
    const int c0 = k * cc, nc = min(cc, w - c0);
#pragma unroll
    for (int j = 0; j < kStreamRows; ++j) {
      const int a = rk + j * gs;
      if (a < r) {
        for (int c = 0; c < nc; ++c) {
          const double l = Lb[c * r + a];
          const double* yc = ysh + 3 * (c0 + c);
          acc[j][0] += l * yc[0]; acc[j][1] += l * yc[1]; acc[j][2] += l * yc[2];
        }
      }
    }
    G::sync();  // the buffer is free again
    if (rk == 0 && k + 2 < nch) {
      fence_proxy_async_smem();
      issue_chunk(f, in, k + 2, Lsh, sbar);
    }
  }
  const int* dst = f.cdst + in.rofs;
#pragma unroll
  for (int j = 0; j < kStreamRows; ++j) {
    const int a = rk + j * gs;
    if (a < r) {
      double* o = f.contrib + 3 * (size_t)dst[a];
      o[0] = acc[j][0]; o[1] = acc[j][1]; o[2] = acc[j][2];
    }
  }
  return true;
}

// u_c -= (L_{R,s}^T x_R)_c with L_{R,s} streamed: a warp per column of the
// chunk, lanes over rows, then the warp sum (per column the same order as
// bwd_panel).
template <class G>
__device__ __forceinline__ bool bwd_panel_stream(const FactorDev& f, const SnInfo& in, double* Lsh, uint64_t* sbar,
                                                 unsigned* sph, const double* __restrict__ xr, double* tsh) {
  const int r = in.r, w = in.w, cc = in.cc;
  const int lane = threadIdx.x & 31, warp = G::warp(), nw = G::nwarps();
  const int nch = (w + cc - 1) / cc;
  for (int k = 0; k < nch; ++k) {
    if (!wait_chunk<G>(f, in, k, nch, sbar, sph, 6)) return false;
    const double* Lb = Lsh + (size_t)(k & 1) * cc * r;
    const int c0 = k * cc, nc = min(cc, w - c0);
    for (int c = warp; c < nc; c += nw) {
      double a0 = 0, a1 = 0, a2 = 0;
      for (int a = lane; a < r; a += 32) {
        const double l = Lb[c * r + a];
        a0 += l * xr[3 * a]; a1 += l * xr[3 * a + 1]; a2 += l * xr[3 * a + 2];
      }
      a0 = warp_sum(a0); a1 = warp_sum(a1); a2 = warp_sum(a2);
      if (lane == 0) { tsh[3 * (c0 + c)] -= a0; tsh[3 * (c0 + c) + 1] -= a1; tsh[3 * (c0 + c) + 2] -= a2; }
    }
    G::sync();
    if (G::rank() == 0 && k + 2 < nch) {
      fence_proxy_async_smem();
      issue_chunk(f, in, k + 2, Lsh, sbar);
    }
  }
  return true;
}

// Forward solve of one supernode, push form:
//   t   = rhs_s - (contributions pushed to s's rows by its descendants)
//   y_s = Dinv_s t                       (one row per thread)
//   contributions of s = L_{R_s,s} y_s   (one below-diagonal row per thread)
// The contributions are stored grouped by destination row, so a supernode
// reads those to its rows as one contiguous range, with all threads at once,
// while its dense blocks are in flight; each row then sums its own in a fixed
// order.  Values written by other CTAs of the same launch (persistent solve)
// are read through L2 (ld.cg).
template <class G>
__device__ __forceinline__ bool fwd_supernode(const FactorDev& f, const SnInfo& in, const double* __restrict__ rhs,
                                              double* y, double* sh, uint64_t* bar, unsigned phase, uint64_t* sbar,
                                              unsigned* sph, bool issued) {
  const int c0 = in.c0, w = in.w, r = in.r, nseg = in.nseg;
  double* Dsh = sh;
  double* Lsh = sh + even_count(w * w);
  double* tsh = Lsh + lsh_doubles(in);
  double* ysh = tsh + 3 * w;
  double* qsh = ysh + 3 * w;
  int* psh = reinterpret_cast<int*>(qsh + 3 * nseg);
  if (!issued) stage_blocks_issue<G>(f, in, true, Dsh, Lsh, bar, sbar);
  const int rk = G::rank(), gs = G::size();
  const double* q = f.contrib + 3 * (size_t)in.seg0;
#pragma unroll 8
  for (int k = rk; k < 3 * nseg; k += gs) qsh[k] = __ldcg(q + k);
  for (int c = rk; c <= w; c += gs) psh[c] = f.rseg_ptr[c0 + c] - in.seg0;
  for (int k = rk; k < 3 * w; k += gs) tsh[k] = rhs[3 * (size_t)c0 + k];
  G::sync();
  for (int c = rk; c < w; c += gs) {
    double a0 = tsh[3 * c], a1 = tsh[3 * c + 1], a2 = tsh[3 * c + 2];
    for (int k = psh[c]; k < psh[c + 1]; ++k) { a0 -= qsh[3 * k]; a1 -= qsh[3 * k + 1]; a2 -= qsh[3 * k + 2]; }
    tsh[3 * c] = a0; tsh[3 * c + 1] = a1; tsh[3 * c + 2] = a2;
  }
  if (!stage_blocks_wait<G>(f, bar, phase, in.s, 1)) {
    drain_chunks<G>(in, sbar, sph);
    return false;
  }
  // column-major Dinv: the threads of a warp read consecutive words
  for (int c = rk; c < w; c += gs) {
    double a0 = 0, a1 = 0, a2 = 0;
#pragma unroll 4
    for (int k = 0; k <= c; ++k) {
      const double dv = Dsh[k * w + c];
      a0 += dv * tsh[3 * k]; a1 += dv * tsh[3 * k + 1]; a2 += dv * tsh[3 * k + 2];
    }
    ysh[3 * c] = a0; ysh[3 * c + 1] = a1; ysh[3 * c + 2] = a2;
    double* yo = y + 3 * (size_t)(c0 + c);
    yo[0] = a0; yo[1] = a1; yo[2] = a2;
  }
  G::sync();
  if (streamed<G>(in)) return fwd_panel_stream<G>(f, in, Lsh, sbar, sph, ysh);
  const double* Lc = in.stage ? Lsh : f.Lcm + in.lofs;
  const int* dst = f.cdst + in.rofs;
  for (int a = rk; a < r; a += gs) {
    const int d = dst[a];
    double a0 = 0, a1 = 0, a2 = 0;
    int c = 0;
    for (; c + 16 <= w; c += 16) {  // sixteen loads in flight, then the sums in column order
      double l[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) l[j] = Lc[(size_t)(c + j) * r + a];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const double* yc = ysh + 3 * (c + j);
        a0 += l[j] * yc[0]; a1 += l[j] * yc[1]; a2 += l[j] * yc[2];
      }
    }
    for (; c < w; ++c) {
      const double l = Lc[(size_t)c * r + a];
      a0 += l * ysh[3 * c]; a1 += l * ysh[3 * c + 1]; a2 += l * ysh[3 * c + 2];
    }
    double* o = f.contrib + 3 * (size_t)d;
    o[0] = a0; o[1] = a1; o[2] = a2;
  }
  return true;
}

// Backward solve of one supernode (in place in y):
//   u   = y_s - L_{R,s}^T y_R   (a warp per column, lanes over rows)
//   y_s = Dinv_s^T u            (one column per thread; row-major Dinv)
template <class G>
__device__ __forceinline__ bool bwd_supernode(const FactorDev& f, const SnInfo& in, double* y, double* sh,
                                              uint64_t* bar, unsigned phase, uint64_t* sbar, unsigned* sph,
                                              bool issued) {
  const int c0 = in.c0, w = in.w, r = in.r;
  const int* R = f.rowidx + in.rofs;
  double* Dsh = sh;
  double* Lsh = sh + even_count(w * w);
  double* tsh = Lsh + lsh_doubles(in);
  double* xr = tsh + 3 * w;
  if (!issued) stage_blocks_issue<G>(f, in, false, Dsh, Lsh, bar, sbar);
  const int rk = G::rank(), gs = G::size();
  for (int a = rk; a < r; a += gs) {
    const double* q = y + 3 * (size_t)R[a];
    xr[3 * a] = __ldcg(q); xr[3 * a + 1] = __ldcg(q + 1); xr[3 * a + 2] = __ldcg(q + 2);
  }
  for (int k = rk; k < 3 * w; k += gs) tsh[k] = __ldcg(y + 3 * (size_t)c0 + k);
  if (!stage_blocks_wait<G>(f, bar, phase, in.s, 2)) {
    drain_chunks<G>(in, sbar, sph);
    return false;
  }
  const double* Lc = in.stage ? Lsh : f.Lcm + in.lofs;
  const int lane = threadIdx.x & 31, warp = G::warp(), nw = G::nwarps();
  if (streamed<G>(in)) {
    if (!bwd_panel_stream<G>(f, in, Lsh, sbar, sph, xr, tsh)) return false;
  } else
  // four columns per warp pass: four independent load streams per lane
  for (int cb = warp; cb < w; cb += 4 * nw) {
    double acc[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q][0] = acc[q][1] = acc[q][2] = 0.0;
    const double* Lq[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) Lq[q] = Lc + (size_t)min(cb + q * nw, w - 1) * r;  // clamped: unused when c >= w
    int a = lane;
    for (; a + 96 < r; a += 128) {  // four rows x four columns: sixteen loads in flight, then the sums in row order
      double l[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) l[j][q] = Lq[q][a + 32 * j];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double* xa = xr + 3 * (a + 32 * j);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[q][0] += l[j][q] * xa[0]; acc[q][1] += l[j][q] * xa[1]; acc[q][2] += l[j][q] * xa[2];
        }
      }
    }
    for (; a < r; a += 32) {
      const double x0 = xr[3 * a], x1 = xr[3 * a + 1], x2 = xr[3 * a + 2];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double l = Lq[q][a];
        acc[q][0] += l * x0; acc[q][1] += l * x1; acc[q][2] += l * x2;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = cb + q * nw;
      const double a0 = warp_sum(acc[q][0]), a1 = warp_sum(acc[q][1]), a2 = warp_sum(acc[q][2]);
      if (lane == 0 && c < w) { tsh[3 * c] -= a0; tsh[3 * c + 1] -= a1; tsh[3 * c + 2] -= a2; }
    }
  }
  G::sync();
  for (int c = rk; c < w; c += gs) {
    double a0 = 0, a1 = 0, a2 = 0;
#pragma unroll 4
    for (int k = c; k < w; ++k) {
      const double dv = Dsh[k * w + c];
      a0 += dv * tsh[3 * k]; a1 += dv * tsh[3 * k + 1]; a2 += dv * tsh[3 * k + 2];
    }
    double* yo = y + 3 * (size_t)(c0 + c);
    yo[0] = a0; yo[1] = a1; yo[2] = a2;
  }
  return true;
}

// One level of the elimination tree per launch: supernodes lvl_begin ..
// lvl_begin + count of the level order, one per group (a CTA, or a warp with
// `shm_group` doubles of shared memory each); the launch boundary orders the
// levels.
template <class G>
__global__ void __launch_bounds__(256) k_fwd_level(FactorDev f, int lvl_begin, int count, int shm_group, Gate gate,
                                                   const double* __restrict__ rhs, double* y) {
  extern __shared__ __align__(16) double sh[];
  __shared__ __align__(8) uint64_t bars[8][3];  // per group: blocks, stream buffers 0 and 1
  const int gi = G::index_in_block(), item = blockIdx.x * G::per_block() + gi;
  if (item >= count) return;
  const SnInfo in = f.info[lvl_begin + item];
  if (gate.skip(in.part)) return;
  if (G::rank() == 0)
    for (int b = 0; b < 3; ++b) mbar_init(&bars[gi][b], 1);
  G::sync();
  unsigned sph[2] = {0u, 0u};
  fwd_supernode<G>(f, in, rhs, y, sh + (size_t)gi * shm_group, &bars[gi][0], 0, &bars[gi][1], sph, false);
}

template <class G>
__global__ void __launch_bounds__(256) k_bwd_level(FactorDev f, int lvl_begin, int count, int shm_group, Gate gate,
                                                   double* y) {
  extern __shared__ __align__(16) double sh[];
  __shared__ __align__(8) uint64_t bars[8][3];  // per group: blocks, stream buffers 0 and 1
  const int gi = G::index_in_block(), item = blockIdx.x * G::per_block() + gi;
  if (item >= count) return;
  const SnInfo in = f.info[lvl_begin + item];
  if (gate.skip(in.part)) return;
  if (G::rank() == 0)
    for (int b = 0; b < 3; ++b) mbar_init(&bars[gi][b], 1);
  G::sync();
  unsigned sph[2] = {0u, 0u};
  bwd_supernode<G>(f, in, y, sh + (size_t)gi * shm_group, &bars[gi][0], 0, &bars[gi][1], sph, false);
}

// The solve of the supernodes at level-order positions p0 .. ns-1 (L y = rhs,
// then L^T z = y, in place) in one launch; the positions below p0 are solved
// by level kernels before (forward) and after (backward) it — p0 = 0 is the
// whole solve.  The CTAs claim work items from a ticket counter: with
// n = ns - p0, tickets 0 .. n-1 are the forward solves of those supernodes in
// level order (leaves first), tickets n .. 2n-1 the backward solves in
// reverse level order (roots first).  A CTA claims its next ticket while it
// solves the current one (the claim's round trip overlaps the work).  It
// starts the claimed item's (read-only) block copies, then waits until the
// supernodes the item reads are done — forward: its children in the
// elimination tree at positions >= p0 (a child done implies its whole subtree
// done); backward: its parent's backward solve, or its own forward solve at a
// root.  Every awaited item has a lower ticket, and a CTA's claimed but
// unstarted ticket is higher than its current one, so the lowest unfinished
// ticket is always running with its dependencies done: the waits always end.
// They are bounded all the same (FactorDev::spin_tries polls, kSpinTries
// unless lowered by dfem_set_limit): a CTA that gives up
// records status 6 and raises the abort word, and every CTA then stops
// claiming.  Completion is an epoch stamp per supernode and direction
// (release store after the CTA's writes; acquire loads by the waiter).
// Control words ctl: [0] ticket, [1] CTAs finished, [2] epoch (>= 1),
// [3] abort; the last CTA to finish resets the ticket and advances the epoch
// for the next launch.  A part of a batch whose gate is closed is skipped
// whole (nothing outside the part depends on it).
constexpr int kSpinTries = 1 << 22;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait until *flag == epoch; false on abort or when the bound is reached.
__device__ __forceinline__ bool wait_epoch(const int* flag, int epoch, const int* abort_word, int tries) {
  for (int i = 0; i < tries; ++i) {
    if (ld_acquire(flag) == epoch) return true;
    if ((i & 63) == 63) {
      if (ld_acquire(abort_word) != 0) return false;
      __nanosleep(64);
    }
  }
  return false;
}

__global__ void __launch_bounds__(256) k_solve_persistent(FactorDev f, int p0, Gate gate,
                                                          const double* __restrict__ rhs, double* y) {
  extern __shared__ __align__(16) double sh[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ __align__(8) uint64_t sbar[2];  // stream buffers of a streamed L_{R,s}
  __shared__ int s_ticket, s_epoch, s_go;
  const int n = f.nsuper - p0;
  int* ctl = f.ctl;
  int next = 0;  // thread 0: the claimed next ticket
  unsigned sph[2] = {0u, 0u};  // phases of the stream buffers (every thread tracks them alike)
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init(sbar, 1);
    mbar_init(sbar + 1, 1);
    s_epoch = ld_acquire(ctl + 2);
    next = atomicAdd(ctl + 0, 1);
  }
  __syncthreads();
  const int epoch = s_epoch;
  unsigned phase = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      const int t = next;
      s_ticket = t;
      s_go = (t < 2 * n && ld_acquire(ctl + 3) == 0) ? 1 : 0;
      if (s_go) next = atomicAdd(ctl + 0, 1);
    }
    __syncthreads();
    if (!s_go) break;
    const int t = s_ticket;
    const bool fwd = t < n;
    const SnInfo in = f.info[fwd ? p0 + t : p0 + 2 * n - 1 - t];
    const int s = in.s;
    if (!gate.skip(in.part)) {
      // the factor blocks are read-only: start their copies before waiting on the dependencies
      stage_blocks_issue<CtaGroup>(f, in, fwd, sh, sh + even_count(in.w * in.w), &bar, sbar);
      if (threadIdx.x == 0) {
        bool ok = true;
        if (fwd) {
          for (int k = f.kid_ptr[s]; ok && k < f.kid_ptr[s + 1]; ++k) {
            const int kid = f.kid[k];
            if (f.sn_pos[kid] >= p0) ok = wait_epoch(f.done_f + kid, epoch, ctl + 3, f.spin_tries);
          }
        } else {
          const int p = f.sn_parent[s];
          ok = wait_epoch(p >= 0 ? f.done_b + p : f.done_f + s, epoch, ctl + 3, f.spin_tries);
        }
        if (!ok) {
          if (ld_acquire(ctl + 3) == 0) record_gave_up(f, s, fwd ? 3 : 4);
          atomicExch(ctl + 3, 1);
        }
        s_go = ok ? 1 : 0;
      }
      __syncthreads();
      if (!s_go) {  // aborted: let this CTA's copies land before it leaves
        if (threadIdx.x == 0) mbar_wait_bounded(&bar, phase);
        drain_chunks<CtaGroup>(in, sbar, sph);
        break;
      }
      const bool ok = fwd ? fwd_supernode<CtaGroup>(f, in, rhs, y, sh, &bar, phase, sbar, sph, true)
                          : bwd_supernode<CtaGroup>(f, in, y, sh, &bar, phase, sbar, sph, true);
      phase ^= 1u;
      if (!ok) {
        if (threadIdx.x == 0) atomicExch(ctl + 3, 1);
        break;
      }
      // every write of the item precedes the stamp: the CTA barrier orders the
      // other threads' writes before thread 0's release store, whose release
      // semantics (cumulative, gpu scope) make them visible to the acquirer
      __syncthreads();
      if (threadIdx.x == 0) st_release(fwd ? f.done_f + s : f.done_b + s, epoch);
    }
    __syncthreads();  // s_ticket / s_go are rewritten next round
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const int d = atomicAdd(ctl + 1, 1);
    if (d == (int)gridDim.x - 1) {  // every CTA has left the claim loop
      ctl[0] = 0;
      ctl[1] = 0;
      __threadfence();
      st_release(ctl + 2, epoch + 1);
    }
  }
}

// Whole solve in one thread-block cluster (kClusterCtas CTAs of 512 threads),
// for factors of few supernodes: the levels in order (leaves first, then
// back), each level's small supernodes (level-order positions lvl_ptr[l] ..
// lvl_warp[l]) one per warp of the cluster, then its other supernodes one per
// CTA; a cluster barrier (release / acquire) between levels orders the
// contributions and solution values the next level reads.  The per-level
// handoff is one hardware barrier instead of a completion stamp per
// supernode.  Every CTA takes every barrier: a supernode whose bounded copy
// wait gave up records the error status and the CTA carries on.
constexpr int kClusterCtas = 8;

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__global__ void __launch_bounds__(512) k_solve_cluster(FactorDev f, int nlev, const int* __restrict__ lvl_ptr,
                                                       const int* __restrict__ lvl_warp, int shm_warp, Gate gate,
                                                       const double* __restrict__ rhs, double* y) {
  extern __shared__ __align__(16) double sh[];
  __shared__ __align__(8) uint64_t wbar[16][3];  // per warp: blocks, stream buffers
  __shared__ __align__(8) uint64_t cbar[3];      // CTA items
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  const int rank = (int)cluster_rank();
  if (lane == 0)
    for (int b = 0; b < 3; ++b) mbar_init(&wbar[warp][b], 1);
  if (threadIdx.x == 0)
    for (int b = 0; b < 3; ++b) mbar_init(&cbar[b], 1);
  __syncthreads();
  unsigned wph = 0, wsph[2] = {0u, 0u};  // this warp's barrier phases
  unsigned cph = 0, csph[2] = {0u, 0u};  // the CTA barriers' phases (uniform over the CTA)
  double* wsh = sh + (size_t)warp * shm_warp;
  for (int pass = 0; pass < 2; ++pass) {
    const bool fwd = pass == 0;
    for (int k = 0; k < nlev; ++k) {
      const int l = fwd ? k : nlev - 1 - k;
      const int p0 = lvl_ptr[l], pw = lvl_warp[l], p1 = lvl_ptr[l + 1];
      for (int item = p0 + rank * nwarp + warp; item < pw; item += kClusterCtas * nwarp) {
        const SnInfo in = f.info[item];
        if (gate.skip(in.part)) continue;
        __syncwarp();  // the warp's reads of its region precede the next bulk writes into it
        if (fwd) fwd_supernode<WarpGroup>(f, in, rhs, y, wsh, &wbar[warp][0], wph, &wbar[warp][1], wsph, false);
        else bwd_supernode<WarpGroup>(f, in, y, wsh, &wbar[warp][0], wph, &wbar[warp][1], wsph, false);
        wph ^= 1u;
      }
      __syncthreads();  // the warps' regions overlap the CTA items' region
      for (int item = pw + rank; item < p1; item += kClusterCtas) {
        const SnInfo in = f.info[item];
        if (gate.skip(in.part)) continue;
        if (fwd) fwd_supernode<CtaGroup>(f, in, rhs, y, sh, &cbar[0], cph, &cbar[1], csph, false);
        else bwd_supernode<CtaGroup>(f, in, y, sh, &cbar[0], cph, &cbar[1], csph, false);
        cph ^= 1u;
        __syncthreads();  // the CTA's reads of the region precede the next item's bulk writes
      }
      cluster_sync_all();
    }
  }
}

// Reset of the persistent solve's completion stamps and control words.
__global__ void k_solve_reset(int ns, int* done_f, int* done_b, int* ctl) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
    done_f[i] = 0;
    done_b[i] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) { ctl[0] = 0; ctl[1] = 0; ctl[2] = 1; ctl[3] = 0; }
}

// x^{k+1}; per-part convergence test for the next iteration (k read from
// device memory).  Part-aligned blocks; a converged part's blocks do nothing.
__global__ void k_update(int N, PartDev pd, int from_iterate, const int* kptr, const double* __restrict__ xt,
                         const double* __restrict__ z, double* xk, double* hist, long long hist_step, const int* step,
                         int* flag, int* iters,
                         double* partial, unsigned* counter, double* errv, int* status) {
  const int b = blockIdx.x, p = pd.blk_part[b];
  if (flag[p]) return;
  const int k = *kptr;
  const int pv0 = pd.part_v0[p], pv1 = pd.part_v0[p + 1];
  const int i = pd.blk_v0[b] + threadIdx.x;
  double e2 = 0;
  if (i < pv1) {
    // plain form: x^{k+1} = x_t + hvf (reference delta form); mixed form: x^{k+1} = x^k + z
    Vec3<double> xn = (from_iterate ? ld3(xk, i) : ld3(xt, i)) + ld3(z, i);
    Vec3<double> dlt = xn - ld3(xk, i);
    e2 = dot3(dlt, dlt);
    st3(xk, i, xn);
    if (hist) st3(hist + (size_t)(*step) * hist_step + (size_t)(k + 1) * 3 * N, i, xn);
  }
  double tot;
  if (part_reduce(e2, partial, counter + p, pd.part_b0[p], pd.part_b0[p + 1] - pd.part_b0[p], &tot)) {
    double e = sqrt(tot) / (3.0 * (pv1 - pv0));
    errv[p] = e;
    iters[(size_t)(*step) * pd.nparts + p] += 1;
    if (e < kConvergenceEps) flag[p] = 1;
    if (!isfinite(tot)) { *status = 4; flag[p] = 1; }
  }
}

// v = damping (x^K - x)/h ; x = x^K ; optional trajectory row in user order
__global__ void k_step_end(SceneDev d, int* step, double* xt, double* vt, const double* xk,
                           double* traj, const int* to_user, const int* write_traj) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = *step;
  if (i < d.N) {
    Vec3<double> x1 = ld3(xk, i), x0 = ld3(xt, i);
    st3(vt, i, (d.damping / d.h) * (x1 - x0));
    st3(xt, i, x1);
    if (traj && *write_traj) st3(traj + (size_t)s * 3 * d.N, to_user[i], x1);
  }
  // the step counter is advanced by k_next_step (a separate launch, so every
  // block of this kernel has read it first)
}

__global__ void k_next_step(int* step) { *step += 1; }

// Loop control of the PD iterations (body of a conditional WHILE graph node),
// one block over the parts: advance the device-side iteration counter and
// continue while some part has not converged and k < K.  The counter advances
// on every body execution, so the loop runs at most K times whatever the
// convergence flags say.
__global__ void k_loop_ctl(int* kptr, const int* flag, int nparts, int K, cudaGraphConditionalHandle h) {
  int open = 0;
  for (int p = threadIdx.x; p < nparts; p += blockDim.x) open |= (flag[p] == 0);
  open = __syncthreads_or(open);
  if (threadIdx.x == 0) {
    int k = *kptr + 1;
    *kptr = k;
    cudaGraphSetConditional(h, (open && k < K) ? 1u : 0u);
  }
}

// Form of this iteration's solve in a batch: the summed weight (factor
// entries) of the parts still iterating against a threshold -- 1: the form
// tuned for the whole batch, 0: the persistent form, cheaper once few parts
// are left.  Both forms give identical results, so the choice only moves
// time.  sel_count counts the iterations that took the persistent form.
__global__ void k_solve_select(Gate gate, const double* __restrict__ part_w, int nparts, double threshold,
                               unsigned long long* sel_count, cudaGraphConditionalHandle h) {
  __shared__ double red[256];
  double a = 0.0;
  for (int p = threadIdx.x; p < nparts; p += blockDim.x)
    if (!gate.skip(p)) a += part_w[p];
  red[threadIdx.x] = a;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const bool full = red[0] >= threshold;
    if (!full) atomicAdd(sel_count, 1ull);
    cudaGraphSetConditional(h, full ? 1u : 0u);
  }
}

// Before the loop: run the body at all only if some part did not converge in the first test.
__global__ void k_loop_enter(int* kptr, const int* flag, int nparts, int K, cudaGraphConditionalHandle h) {
  int open = 0;
  for (int p = threadIdx.x; p < nparts; p += blockDim.x) open |= (flag[p] == 0);
  open = __syncthreads_or(open);
  if (threadIdx.x == 0) {
    *kptr = 0;
    cudaGraphSetConditional(h, (open && K > 0) ? 1u : 0u);
  }
}

// Reverse loop of the adjoint: k = n-1 .. 0, n the largest iteration count of
// the step over the parts (each part skips its k >= own count); the counter
// decreases every body execution.
__global__ void k_adj_loop_enter(int* kptr, const int* iters, const int* step, int nparts, int K,
                                 cudaGraphConditionalHandle h) {
  __shared__ int mx;
  if (threadIdx.x == 0) mx = 0;
  __syncthreads();
  const size_t row = (size_t)(*step) * nparts;
  int n = 0;
  for (int p = threadIdx.x; p < nparts; p += blockDim.x) n = max(n, min(max(iters[row + p], 0), K));
  atomicMax(&mx, n);
  __syncthreads();
  if (threadIdx.x == 0) {
    *kptr = mx - 1;
    cudaGraphSetConditional(h, mx > 0 ? 1u : 0u);
  }
}
__global__ void k_adj_loop_ctl(int* kptr, cudaGraphConditionalHandle h) {
  int k = *kptr - 1;
  *kptr = k;
  cudaGraphSetConditional(h, k >= 0 ? 1u : 0u);
}
__global__ void k_set_int(int* p, int v) { *p = v; }

// permutation between user and internal vertex order (3 doubles per vertex)
__global__ void k_to_internal(int N, const int* to_internal, const double* src, double* dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) st3(dst, to_internal[i], ld3(src, i));
}
__global__ void k_to_user(int N, const int* to_user, const double* src, double* dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) st3(dst, to_user[i], ld3(src, i));
}

// ---------------------------------------------------------------- adjoint ---
//
// Reverse of one step.  With x^{k+1} = Hs^-1 (b + J d(x^k)) (the reference's
// delta form x + Hs^-1(ori_c - Hs x) is the same map), for k = it-1 .. 0:
//   ybar = Hs^-1 xbar^{k+1}; bbar += ybar; xbar^k = (dd/dx)^T J^T ybar;
//   dE_t += ybar^T (dJ/dE_t d^k - dHs/dE_t x^{k+1}); dnu_t likewise; da_seg += -(J^T ybar).(F f)
// then qbar = xbar^0 + M/h^2 bbar, xbar = -damping/h vbar' + qbar, vbar = h qbar.

__global__ void k_adj_begin(int N, double c, const double* gx1, const double* gv1, double* xkb,
                            double* xtb, double* bb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  Vec3<double> gv = ld3(gv1, i);
  st3(xkb, i, ld3(gx1, i) + c * gv);
  st3(xtb, i, (-c) * gv);
  st3(bb, i, mk3(0.0, 0.0, 0.0));
}

// VJP of constraint t's J d at positions x with cotangent yb: writes the
// constraint's slot contributions to xbar and accumulates the parameter
// gradients of J d.  The tets' E-gradient also takes the Hs term of the map
// that consumed J d: PD iteration (x1 != null): -vol (G G^T) : (yb x1^T),
// x1 the next iterate; contact rhs (xt != null): -vol (G G^T) : (yb z^T) with
// z = x off the diagonal and x_t on it (rhs = ... - h C (x - x_t) - h L x_t).
// VJP of muscle constraint t (LinearMuscleConstraint): its slots and the
// activation term mg[t].  Not inlined: the kernels that call it (the PD
// adjoint, the contact adjoint as kernels or as one cooperative launch) then
// run one compiled copy of its arithmetic, so their activation gradients
// agree bit for bit.
__device__ __noinline__ void muscle_vjp(const SceneDev& d, int t, const double* x, const double* yb,
                                        const double* act_row, double* slot, double* mg) {
  int4 v = d.mv[t];
  const int vi[4] = {v.x, v.y, v.z, v.w};
  double G[4][3];
  load_g(d.minv, d.M, t, G);
  Vec3<double> f = mk3(d.mfib[t], d.mfib[d.M + t], d.mfib[2 * d.M + t]);
  double w = d.mw[t];
  double c[4];
  Vec3<double> db = mk3(0.0, 0.0, 0.0), Ff = mk3(0.0, 0.0, 0.0);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    c[a] = G[a][0] * f.x + G[a][1] * f.y + G[a][2] * f.z;
    db = db + (w * c[a]) * ld3(yb, vi[a]);
    Ff = Ff + c[a] * ld3(x, vi[a]);
  }
  double a_act = act_row[d.mseg[t]];
  mg[t] = -dot3(db, Ff);
  int4 sl = d.mslot[t];
  const int sv[4] = {sl.x, sl.y, sl.z, sl.w};
#pragma unroll
  for (int a = 0; a < 4; ++a) st3(slot, sv[a], ((1.0 - a_act) * c[a]) * db);
}

// (Plain pointers: k_cadj_fused writes yb earlier in the same launch; the
// kernels that call it keep their parameters restrict-qualified.)
__device__ __forceinline__ void adj_local_item(const SceneDev& d, int t, const double* x, const double* yb,
                                               const double* act_row, double* slot, double* gE, double* gnu,
                                               double* mg, const double* x1, const double* xt) {
  if (t < d.T) {
    int4 v = d.tv[t];
    const int vi[4] = {v.x, v.y, v.z, v.w};
    Vec3<double> xv[4], yv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) { xv[a] = ld3(x, vi[a]); yv[a] = ld3(yb, vi[a]); }
    double G[4][3];
    load_g(d.tinv, d.T, t, G);
    Mat3<double> F = deformation(G, xv), Y = deformation(G, yv), md, mdv;
    double E = d.tE[t], nu = d.tnu[t], vol = d.tvol[t];
    const Svd3<double> fsv = svd3(F);  // one SVD for the projection and its VJP
    corot_project_sv(fsv, F, md, mdv);
    double yr = 0, yvv = 0, yh = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) { yr += dot3(Y.c[j], md.c[j]); yvv += dot3(Y.c[j], mdv.c[j]); }
    if (x1) {
      Vec3<double> x1v[4] = {ld3(x1, vi[0]), ld3(x1, vi[1]), ld3(x1, vi[2]), ld3(x1, vi[3])};
      Mat3<double> F1 = deformation(G, x1v);
#pragma unroll
      for (int j = 0; j < 3; ++j) yh += dot3(Y.c[j], F1.c[j]);
    } else if (xt) {
#pragma unroll
      for (int j = 0; j < 3; ++j) yh += dot3(Y.c[j], F.c[j]);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const double gaa = G[a][0] * G[a][0] + G[a][1] * G[a][1] + G[a][2] * G[a][2];
        yh += gaa * dot3(yv[a], ld3(xt, vi[a]) - xv[a]);
      }
    }
    double opn = 1.0 + nu;
    if (gE) gE[t] += vol / opn * (yr + nu * yvv) - vol * yh;
    if (gnu) gnu[t] += E * vol / (opn * opn) * (yvv - yr);
    double wr = d.twr[t], wv = d.twv[t];
    Mat3<double> gmd, gmdv;
#pragma unroll
    for (int j = 0; j < 3; ++j) { gmd.c[j] = wr * Y.c[j]; gmdv.c[j] = wv * Y.c[j]; }
    Mat3<double> gF = corot_vjp_sv(fsv, F, gmd, gmdv);
    int4 sl = d.tslot[t];
    const int sv[4] = {sl.x, sl.y, sl.z, sl.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) st3(slot, sv[a], G[a][0] * gF.c[0] + G[a][1] * gF.c[1] + G[a][2] * gF.c[2]);
    return;
  }
  t -= d.T;
  if (t < d.M) {
    muscle_vjp(d, t, x, yb, act_row, slot, mg);
    return;
  }
  t -= d.M;
  if (t < d.S) {
    int2 v = d.sv[t];
    double w = d.ssw[t];
    Vec3<double> db = w * (ld3(yb, v.x) - ld3(yb, v.y));
    Vec3<double> e = ld3(x, v.x) - ld3(x, v.y);
    double inv = rsqrt(dot3(e, e));
    Vec3<double> eh = inv * e;
    // a pneumatic spring's activation term: d md / d a = rest * eh
    if (d.sch && d.sch[t] >= 0) mg[d.M + t] = d.srest[t] * dot3(db, eh);
    Vec3<double> ge = (spring_length(d, t, act_row) * inv) * (db - dot3(eh, db) * eh);
    int2 sl = d.sslot[t];
    st3(slot, sl.x, ge);
    st3(slot, sl.y, (-1.0) * ge);
    return;
  }
  t -= d.S;
  if (t < d.B) {
    int o0 = d.boff[t], o1 = d.boff[t + 1];
    double w = d.bw[t];
    Vec3<double> db = mk3(0.0, 0.0, 0.0), lap = mk3(0.0, 0.0, 0.0);
    for (int q = o0; q < o1; ++q) {
      db = db + (w * d.bbeta[q]) * ld3(yb, d.bv[q]);
      lap = lap + d.bbeta[q] * ld3(x, d.bv[q]);
    }
    double ln = sqrt(dot3(lap, lap));
    Vec3<double> gl = mk3(0.0, 0.0, 0.0);
    if (ln > 1e-25) {
      Vec3<double> lh = (1.0 / ln) * lap;
      gl = (w * d.brest[t] / ln) * (db - dot3(lh, db) * lh);
    }
    for (int q = o0; q < o1; ++q) st3(slot, d.bslot[q], d.bbeta[q] * gl);
  }
}

// Reverse PD iteration k (k read from device memory): local VJP at x^k with
// the Hs term of x^{k+1}, and bbar += ybar (b = M/h^2 q_n enters every iteration).
__global__ void __launch_bounds__(128, DFEM_ADJ_MIN_BLOCKS) k_adj_local(SceneDev d, Gate gate, const int* kptr, const int* step,
                                                   const double* __restrict__ hist, long long hist_step,
                                                   const double* __restrict__ yb,
                                                   double* bb, const double* __restrict__ act_all,
                                                   double* __restrict__ slot, double* gE, double* gnu, double* mg) {
  const int k = *kptr;
  hist += (size_t)(*step) * hist_step;
  const double* x = hist + (size_t)k * 3 * d.N;
  const double* x1 = hist + (size_t)(k + 1) * 3 * d.N;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < d.N && !gate.skip(vpart_of(d, t))) st3(bb, t, ld3(bb, t) + ld3(yb, t));
  if (gate.skip(cons_part(d, t))) return;
  adj_local_item(d, t, x, yb, act_all + (size_t)(*step) * d.nseg, slot, gE, gnu, mg, x1, nullptr);
}

// xbar^k = sum of the slots (constraints without x dependence contribute nothing)
// xbar = the slots' sum, one thread per vertex in slot order: the contact
// adjoint's kernel form (its cooperative form sums each vertex the same way)
__global__ void k_adj_gather_seq(int N, Gate gate, const int* __restrict__ vpart, const int* __restrict__ vslot_ptr,
                                 const double* __restrict__ slot, double* xkb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || gate.skip(vpart ? vpart[i] : 0)) return;
  Vec3<double> acc = mk3(0.0, 0.0, 0.0);
  for (int k = vslot_ptr[i]; k < vslot_ptr[i + 1]; ++k) acc = acc + ld3(slot, k);
  st3(xkb, i, acc);
}

// xbar = the slots' sum, one thread per vertex (k_adj_gather's sums)
__global__ void k_adj_gather_t(int N, Gate gate, const int* __restrict__ vpart, const int* __restrict__ vslot_ptr,
                               const double* __restrict__ slot, double* xkb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || gate.skip(vpart ? vpart[i] : 0)) return;
  st3(xkb, i, thread_sum_slots(slot, vslot_ptr[i], vslot_ptr[i + 1]));
}

__global__ void k_adj_gather(int N, Gate gate, const int* __restrict__ vpart, const int* __restrict__ vslot_ptr,
                                 const double* __restrict__ slot,
                             double* xkb) {
  const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);  // one warp per vertex
  if (i >= N || gate.skip(vpart ? vpart[i] : 0)) return;
  const Vec3<double> s = warp_sum_slots(slot, vslot_ptr[i], vslot_ptr[i + 1]);
  if ((threadIdx.x & 31) == 0) st3(xkb, i, s);
}

// activation gradient of the step: sum over the members of each channel
// (muscle constraints, then pneumatic springs)
__global__ void k_seg_reduce(int nseg, int M, Gate gate, const int* seg_part, const int* step, const int* seg_ptr,
                             const int* seg_mus, const double* mg, double* gact) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nseg || gate.skip(seg_part ? seg_part[q] : 0)) return;
  double s = 0;
  for (int k = seg_ptr[q]; k < seg_ptr[q + 1]; ++k) s += mg[member_slot(M, seg_mus[k])];
  gact[(size_t)(*step) * nseg + q] += s;
}

__global__ void k_adj_end(SceneDev d, const double* xkb, const double* xtb, const double* bb,
                          double* gx, double* gv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  double m = d.mass[i] / (d.h * d.h);
  Vec3<double> qb = ld3(xkb, i) + m * ld3(bb, i);
  st3(gx, i, ld3(xtb, i) + qb);
  st3(gv, i, d.h * qb);
}

}  // namespace dfem
