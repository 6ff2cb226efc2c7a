// Adjoint of the articulated-skeleton coupling (skeleton_kernels.cuh).
//
// The reference differentiates a step with links by taping it (CppAD in
// python/pydifem.cc backward_act: cotangents of q, qd, jq, jqd in, gradients of
// q, qd, jq, jqd and the actions out).  Here each PD iteration with links is
// read as the linear KKT system in (y, q, s) that its rigid stage solves,
//   Hs y - E_R q = c          (c = b + J d(x^k))
//   E_R^T y - tildaV s = V0   (the rigid rows follow the links, linearised)
//   tildaV^T q = tau          (the link system S s = tildaV^T C^-1 (u_R - V0) + tau)
// followed by x^{k+1} = [y_F ; V0(theta^{k+1})] and theta^{k+1} = UpdateT(theta^k, s).
// Its adjoint A^T mu = (ybar, 0, sbar) has the same shape as the forward:
//   yhat = Hs^-1 ybar (the step's solve), mu3 = S^-1 (sbar + tildaV^T C^-1 yhat_R),
//   mu2 = C^-1 (yhat_R - tildaV mu3), mu1 = yhat - Z mu2 (mu1_R = tildaV mu3),
// and gives cbar = mu1 (the usual local-step VJP and b cotangent), V0bar = mu2,
// taubar = mu3, tildaVbar = mu2 s^T - q mu3^T and, for the moduli, the Hs term
// -mu1^T dHs y with y_R = V0 + tildaV s (k_skel_adj_ecorr adds what that rigid
// part differs from the stored iterate).  The joint-state cotangent theta-bar
// collects V0bar and tildaVbar through the link kinematics in forward mode
// (one direction of theta per block, dual numbers), and UpdateT, guessNext and
// the polar factor of Transformation::linearize (R = polar(F): dR = R [w]x with
// (tr(P) I - P) w = ax(R^T dF), P = R^T F) in reverse.
#pragma once

#include "scene.h"
#include "skeleton_kernels.cuh"

namespace dfem {

// ---- dual numbers along one direction of theta -----------------------------
struct Dl { double v, t; };
__device__ __forceinline__ Dl dl(double v, double t = 0.0) { return Dl{v, t}; }
__device__ __forceinline__ Dl operator+(Dl a, Dl b) { return Dl{a.v + b.v, a.t + b.t}; }
__device__ __forceinline__ Dl operator-(Dl a, Dl b) { return Dl{a.v - b.v, a.t - b.t}; }
__device__ __forceinline__ Dl operator-(Dl a) { return Dl{-a.v, -a.t}; }
__device__ __forceinline__ Dl operator*(Dl a, Dl b) { return Dl{a.v * b.v, a.v * b.t + a.t * b.v}; }
__device__ __forceinline__ Dl operator*(double a, Dl b) { return Dl{a * b.v, a * b.t}; }
__device__ __forceinline__ Dl operator*(Dl a, double b) { return Dl{a.v * b, a.t * b}; }
__device__ __forceinline__ Dl dl_sin(Dl a) { return Dl{sin(a.v), cos(a.v) * a.t}; }
__device__ __forceinline__ Dl dl_cos(Dl a) { return Dl{cos(a.v), -sin(a.v) * a.t}; }

struct DXf { Dl R[9]; Dl d[3]; };

__device__ __forceinline__ void dx_identity(DXf& t) {
  for (int i = 0; i < 9; ++i) t.R[i] = dl((i % 4 == 0) ? 1.0 : 0.0);
  for (int i = 0; i < 3; ++i) t.d[i] = dl(0.0);
}
__device__ __forceinline__ void dx_mv(const Dl* a, const Dl* v, Dl* o) {
  for (int r = 0; r < 3; ++r) o[r] = a[3 * r] * v[0] + a[3 * r + 1] * v[1] + a[3 * r + 2] * v[2];
}
__device__ __forceinline__ DXf dx_mul(const DXf& a, const DXf& b) {
  DXf o;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o.R[3 * r + c] = a.R[3 * r] * b.R[c] + a.R[3 * r + 1] * b.R[3 + c] + a.R[3 * r + 2] * b.R[6 + c];
  Dl t[3];
  dx_mv(a.R, b.d, t);
  for (int i = 0; i < 3; ++i) o.d[i] = t[i] + a.d[i];
  return o;
}
__device__ __forceinline__ void dx_apply(const DXf& a, const Dl* v, Dl* o) {
  Dl t[3];
  dx_mv(a.R, v, t);
  for (int i = 0; i < 3; ++i) o[i] = t[i] + a.d[i];
}

// ---- the polar factor of linearize -----------------------------------------
// ax(B) = (B21 - B12, B02 - B20, B10 - B01): <B, [w]x> = w . ax(B)
__device__ __forceinline__ void sk_ax(const double* B, double* a) {
  a[0] = B[7] - B[5];
  a[1] = B[2] - B[6];
  a[2] = B[3] - B[1];
}
// x = (tr(P) I - P)^-1 b for P = R^T F (symmetric), by cofactors
__device__ __forceinline__ void sk_polar_sys(const double* R, const double* F, const double* b, double* x) {
  double P[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) P[3 * r + c] = R[r] * F[c] + R[3 + r] * F[3 + c] + R[6 + r] * F[6 + c];
  const double tr = P[0] + P[4] + P[8];
  double A[9];
  for (int i = 0; i < 9; ++i) A[i] = (i % 4 == 0 ? tr : 0.0) - 0.5 * (P[i] + P[3 * (i % 3) + i / 3]);
  const double c00 = A[4] * A[8] - A[5] * A[7], c01 = A[5] * A[6] - A[3] * A[8], c02 = A[3] * A[7] - A[4] * A[6];
  const double c10 = A[2] * A[7] - A[1] * A[8], c11 = A[0] * A[8] - A[2] * A[6], c12 = A[1] * A[6] - A[0] * A[7];
  const double c20 = A[1] * A[5] - A[2] * A[4], c21 = A[2] * A[3] - A[0] * A[5], c22 = A[0] * A[4] - A[1] * A[3];
  const double inv = 1.0 / (A[0] * c00 + A[1] * c01 + A[2] * c02);
  x[0] = inv * (c00 * b[0] + c10 * b[1] + c20 * b[2]);
  x[1] = inv * (c01 * b[0] + c11 * b[1] + c21 * b[2]);
  x[2] = inv * (c02 * b[0] + c12 * b[1] + c22 * b[2]);
}
// tangent of R = polar(F) along dF: R [w]x, (tr(P) I - P) w = ax(R^T dF)
__device__ __forceinline__ void sk_polar_tangent(const double* R, const double* F, const double* dF, double* dR) {
  double B[9], a[3], w[3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) B[3 * r + c] = R[r] * dF[c] + R[3 + r] * dF[3 + c] + R[6 + r] * dF[6 + c];
  sk_ax(B, a);
  sk_polar_sys(R, F, a, w);
  const double W[9] = {0.0, -w[2], w[1], w[2], 0.0, -w[0], -w[1], w[0], 0.0};
  sk_mm(R, W, dR);
}
// cotangent: Fbar = R [g]x, g = (tr(P) I - P)^-1 ax(R^T Rbar)
__device__ __forceinline__ void sk_polar_cotangent(const double* R, const double* F, const double* Rb, double* Fb) {
  double B[9], a[3], g[3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) B[3 * r + c] = R[r] * Rb[c] + R[3 + r] * Rb[3 + c] + R[6 + r] * Rb[6 + c];
  sk_ax(B, a);
  sk_polar_sys(R, F, a, g);
  const double G[9] = {0.0, -g[2], g[1], g[2], 0.0, -g[0], -g[1], g[0], 0.0};
  sk_mm(R, G, Fb);
}

// Link states of theta (jq layout) and their kinematics; one thread.
__device__ void sk_unpack_kinematics(const SkelDev& k, const double* th) {
  for (int l = 0; l < k.L; ++l) {
    const SkelLink& lk = k.link[l];
    SkelState& s = k.st[l];
    if (lk.type == DFEM_JOINT_ALL) {
      for (int i = 0; i < 9; ++i) s.T.R[i] = th[lk.sdof + i];
      for (int i = 0; i < 3; ++i) s.T.d[i] = th[lk.sdof + 9 + i];
    } else {
      s.mag = th[lk.sdof];
    }
    if (l == 0) sk_identity(s.prefix);
    if (lk.type == DFEM_JOINT_PRISMATIC)
      for (int i = 0; i < 9; ++i) s.Tr.R[i] = (i % 4 == 0) ? 1.0 : 0.0;
  }
  sk_kinematics(k);
}

// ---- kernels of one reverse PD iteration -----------------------------------

// theta-bar = the cotangent of the step's output jq (k_skel_adj_theta then adds
// the rigid rows of the last iterate's cotangent)
__global__ void k_skel_adj_init(SkelDev k) {
  for (int i = threadIdx.x; i < k.nq; i += blockDim.x) k.thb[i] = k.gjq[i];
}

// Reverse of UpdateT at iteration k: theta-bar^{k+1} -> sbar and theta-bar^k;
// the rigid rows of the cotangent of x^{k+1} (already in theta-bar) are cleared
// so that the solve sees ybar_R = 0.  One block.
__global__ void k_skel_adj_upd(SkelDev k, const int* kptr, const int* step, double* xkb) {
  const int it = *kptr;
  const double* h = sk_hrow(k, *step, it);
  const double* s = h + k.nq;
  for (int j = threadIdx.x; j < k.nr; j += blockDim.x) {
    const size_t g = 3 * (size_t)k.rv[j];
    xkb[g] = 0.0; xkb[g + 1] = 0.0; xkb[g + 2] = 0.0;
  }
  for (int l = threadIdx.x; l < k.L; l += blockDim.x) {
    const SkelLink& lk = k.link[l];
    const double* sv = s + lk.dof;
    double* sb = k.sb + lk.dof;
    if (lk.type == DFEM_JOINT_PRISMATIC) {
      sb[0] = k.thb[lk.sdof];  // mag' = mag + s
    } else if (lk.type == DFEM_JOINT_ROTATIONAL) {
      sb[0] = k.thb[lk.sdof] / (1.0 + sv[0] * sv[0]);  // mag' = mag + atan(s)
    } else {
      // T' = t(w) Tr, T'.d = t(w) Tr.d + s_v, Tr = linearize(T)
      SkelXf T;
      for (int i = 0; i < 9; ++i) T.R[i] = h[lk.sdof + i];
      for (int i = 0; i < 3; ++i) T.d[i] = h[lk.sdof + 9 + i];
      const SkelXf Tr = sk_linearize(T);
      const double t[9] = {1.0, -sv[2], sv[1], sv[2], 1.0, -sv[0], -sv[1], sv[0], 1.0};
      const double* Rb1 = k.thb + lk.sdof;
      const double* db1 = k.thb + lk.sdof + 9;
      double tb[9], Rrb[9], drb[3];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          tb[3 * r + c] = Rb1[3 * r] * Tr.R[3 * c] + Rb1[3 * r + 1] * Tr.R[3 * c + 1] + Rb1[3 * r + 2] * Tr.R[3 * c + 2] +
                          db1[r] * Tr.d[c];
          Rrb[3 * r + c] = t[r] * Rb1[c] + t[3 + r] * Rb1[3 + c] + t[6 + r] * Rb1[6 + c];
        }
      for (int c = 0; c < 3; ++c) drb[c] = t[c] * db1[0] + t[3 + c] * db1[1] + t[6 + c] * db1[2];
      sb[0] = tb[7] - tb[5];
      sb[1] = tb[2] - tb[6];
      sb[2] = tb[3] - tb[1];
      for (int i = 0; i < 3; ++i) sb[3 + i] = db1[i];
      double Fb[9];
      sk_polar_cotangent(Tr.R, T.R, Rrb, Fb);
      for (int i = 0; i < 9; ++i) k.thb[lk.sdof + i] = Fb[i];
      for (int i = 0; i < 3; ++i) k.thb[lk.sdof + 9 + i] = drb[i];
    }
  }
}

// The KKT adjoint of iteration k (one block): theta^k's links, tildaV, S;
// mu3 = S^-1 (sbar + tildaV^T C^-1 yhat_R), mu2 = C^-1 (yhat_R - tildaV mu3);
// y_R := tildaV mu3 (mu1 on the rigid rows), the torque channels' gradient,
// and dlt = V0^k + tildaV s^k - x^{k+1}_R for the moduli's Hs term.
__global__ void k_skel_adj_stage(SkelDev k, const int* kptr, const int* step, double* y, const double* hist_x,
                                 long long hist_step, double* gact, int nseg) {
  const int tid = threadIdx.x, nt = blockDim.x, nr = k.nr, nd = k.ndof;
  const int it = *kptr, st = *step;
  const double* h = sk_hrow(k, st, it);
  const double* s = h + k.nq;
  const double* x1 = hist_x + (size_t)st * hist_step + (size_t)(it + 1) * 3 * k.N;
  if (tid == 0) sk_unpack_kinematics(k, h);
  __syncthreads();
  for (int j = tid; j < nr; j += nt) {
    double p[3];
    sk_v0(k, j, p);
    const size_t g = 3 * (size_t)k.rv[j];
    for (int c = 0; c < 3; ++c) { k.v0[3 * j + c] = p[c]; k.w[3 * j + c] = y[g + c]; }
  }
  sk_dt(k, tid, nt);
  __syncthreads();
  sk_tildav(k, tid, nt);
  __syncthreads();
  sk_cinv_products(k, tid, nt);  // rr = C^-1 yhat_R, kt = C^-1 tildaV
  __syncthreads();
  for (int e = tid; e < nd * nd; e += nt) {
    const int a = e / nd, b = e % nd;
    double acc = 0.0;
    for (int r = 0; r < 3 * nr; ++r) acc += k.tv[(size_t)r * nd + a] * k.kt[(size_t)r * nd + b];
    k.sm[e] = acc;
  }
  for (int a = tid; a < nd; a += nt) {
    double acc = 0.0;
    for (int r = 0; r < 3 * nr; ++r) acc += k.tv[(size_t)r * nd + a] * k.rr[r];
    k.rhs[a] = k.sb[a] + acc;
  }
  __syncthreads();
  sk_fullpiv_block(nd, k.sm, k.rhs, k.mu3, k.perm);  // S is symmetric: S^-T = S^-1
  for (int r = tid; r < 3 * nr; r += nt) {
    double tm = 0.0, ts = 0.0;
    for (int a = 0; a < nd; ++a) {
      tm += k.tv[(size_t)r * nd + a] * k.mu3[a];
      ts += k.tv[(size_t)r * nd + a] * s[a];
    }
    const int j = r / 3, c = r % 3;
    const size_t g = 3 * (size_t)k.rv[j] + c;
    k.rr[r] = k.w[r] - tm;
    k.dlt[r] = (k.v0[r] + ts) - x1[g];
    y[g] = tm;
  }
  __syncthreads();
  for (int e = tid; e < 3 * nr; e += nt) {
    const int i = e / 3, c = e % 3;
    double acc = 0.0;
    for (int j = 0; j < nr; ++j) acc += k.cinv[(size_t)i * nr + j] * k.rr[3 * j + c];
    k.mu2[e] = acc;
  }
  for (int l = 1 + tid; l < k.L; l += nt)
    if (k.link[l].chan >= 0) gact[(size_t)st * nseg + k.link[l].chan] += k.mu3[k.link[l].dof];
}

// mu1_F = yhat_F - Z_F mu2
__global__ void k_skel_adj_apply(SkelDev k, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k.N || k.ridx[i] >= 0) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int j = 0; j < k.nr; ++j) {
    const double zz = k.zcm[(size_t)j * k.N + i];
    a0 += zz * k.mu2[3 * j]; a1 += zz * k.mu2[3 * j + 1]; a2 += zz * k.mu2[3 * j + 2];
  }
  y[3 * (size_t)i] -= a0; y[3 * (size_t)i + 1] -= a1; y[3 * (size_t)i + 2] -= a2;
}

// The moduli's Hs term takes x^{k+1} where the KKT system has y: on the rigid
// rows they differ by dlt.  -vol (G G^T) : (mu1 dlt^T) for the tets that touch
// a rigid vertex.
__global__ void k_skel_adj_ecorr(SceneDev d, SkelDev k, const double* y, double* gE) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.T) return;
  const int4 v = d.tv[t];
  const int vi[4] = {v.x, v.y, v.z, v.w};
  bool any = false;
  Vec3<double> yv[4], dv[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int j = k.ridx[vi[a]];
    any = any || j >= 0;
    yv[a] = ld3(y, vi[a]);
    dv[a] = j >= 0 ? mk3(k.dlt[3 * j], k.dlt[3 * j + 1], k.dlt[3 * j + 2]) : mk3(0.0, 0.0, 0.0);
  }
  if (!any) return;
  double G[4][3];
  load_g(d.tinv, d.T, t, G);
  const Mat3<double> Y = deformation(G, yv), Fd = deformation(G, dv);
  double yh = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) yh += dot3(Y.c[j], Fd.c[j]);
  gE[t] -= d.tvol[t] * yh;
}

// theta-bar[m] += d/dtheta_m of  sum_j (mu2_j + xbar_j) . V0_j
//                              + mu2_j . (tildaV_j s) - q_j . (tildaV_j mu3)
// at theta^{*kptr + koff} (the tildaV terms only with use_tv), block m one
// direction of theta: the links' kinematics in dual numbers by one thread,
// then one rigid vertex per thread.  xbar: the rigid rows of the cotangent of
// that iterate.
constexpr int kSkelAdjThreads = 128;
__global__ void __launch_bounds__(kSkelAdjThreads) k_skel_adj_theta(SkelDev k, const int* kptr, const int* step,
                                                                  int koff, int use_tv, const double* xkb) {
  __shared__ DXf s_tr[kMaxLinks], s_pre[kMaxLinks], s_dt[kMaxLinks];
  __shared__ double s_red[kSkelAdjThreads / 32];
  const int m = blockIdx.x, tid = threadIdx.x;
  const int it = *kptr, st = *step;
  const double* th = sk_hrow(k, st, it + koff);
  const double* hs = use_tv ? sk_hrow(k, st, it) : th;  // s^k and q^k (only read with use_tv)
  const double* sv = hs + k.nq;
  const double* qv = hs + k.nq + k.ndof;
  if (tid == 0) {
    for (int l = 0; l < k.L; ++l) {
      const SkelLink& lk = k.link[l];
      DXf tr, dt;
      for (int i = 0; i < 9; ++i) dt.R[i] = dl(0.0);
      for (int i = 0; i < 3; ++i) dt.d[i] = dl(0.0);
      if (lk.type == DFEM_JOINT_ALL) {
        SkelXf T;
        double dT[9];
        for (int i = 0; i < 9; ++i) { T.R[i] = th[lk.sdof + i]; dT[i] = (m == lk.sdof + i) ? 1.0 : 0.0; }
        for (int i = 0; i < 3; ++i) T.d[i] = th[lk.sdof + 9 + i];
        const SkelXf Tr = sk_linearize(T);
        double dR[9];
        sk_polar_tangent(Tr.R, T.R, dT, dR);
        for (int i = 0; i < 9; ++i) tr.R[i] = dl(Tr.R[i], dR[i]);
        for (int i = 0; i < 3; ++i) tr.d[i] = dl(T.d[i], (m == lk.sdof + 9 + i) ? 1.0 : 0.0);
      } else {
        const Dl mag = dl(th[lk.sdof], (m == lk.sdof) ? 1.0 : 0.0);
        if (lk.type == DFEM_JOINT_ROTATIONAL) {
          const Dl C = dl_cos(mag), S = dl_sin(mag);
          for (int i = 0; i < 9; ++i) {
            const double e = (i % 4 == 0) ? 1.0 : 0.0;
            tr.R[i] = (C * e + S * lk.nx[i]) + (dl(1.0) - C) * lk.nnt[i];
            dt.R[i] = ((-S) * e + C * lk.nx[i]) + S * lk.nnt[i];
          }
          for (int i = 0; i < 3; ++i) tr.d[i] = dl(lk.d0[i]);
        } else {
          for (int i = 0; i < 9; ++i) tr.R[i] = dl((i % 4 == 0) ? 1.0 : 0.0);
          for (int i = 0; i < 3; ++i) { tr.d[i] = mag * lk.axis[i] + dl(lk.d0[i]); dt.d[i] = dl(lk.axis[i]); }
        }
      }
      s_tr[l] = tr;
      s_dt[l] = dt;
      if (lk.parent < 0) dx_identity(s_pre[l]);
      else s_pre[l] = dx_mul(s_pre[lk.parent], s_tr[lk.parent]);
    }
  }
  __syncthreads();
  double acc = 0.0;
  for (int j = tid; j < k.nr; j += blockDim.x) {
    const int me = k.rlink[j];
    const SkelLink& ml = k.link[me];
    const Dl vinit[3] = {dl(k.rest[3 * j] - ml.joint[0]), dl(k.rest[3 * j + 1] - ml.joint[1]),
                         dl(k.rest[3 * j + 2] - ml.joint[2])};
    Dl a[3], v0[3];
    dx_apply(s_tr[me], vinit, a);
    dx_apply(s_pre[me], a, v0);
    const size_t g = 3 * (size_t)k.rv[j];
    for (int c = 0; c < 3; ++c) {
      const double vb = xkb[g + c] + (use_tv ? k.mu2[3 * j + c] : 0.0);
      acc += vb * v0[c].t;
    }
    if (!use_tv) continue;
    Dl fs[3] = {dl(0.0), dl(0.0), dl(0.0)}, fm[3] = {dl(0.0), dl(0.0), dl(0.0)};
    DXf suffix;
    dx_identity(suffix);
    int cur = me;
    while (k.link[cur].parent >= 0) {
      const SkelLink& cl = k.link[cur];
      Dl t[3];
      if (cl.type == DFEM_JOINT_ROTATIONAL) {
        Dl p[3], b[3];
        dx_apply(suffix, vinit, p);
        dx_mv(s_dt[cur].R, p, b);
        dx_mv(s_pre[cur].R, b, t);
      } else {
        dx_mv(s_pre[cur].R, s_dt[cur].d, t);
      }
      const double a1 = sv[cl.dof], a2 = k.mu3[cl.dof];
      for (int c = 0; c < 3; ++c) { fs[c] = fs[c] + t[c] * a1; fm[c] = fm[c] + t[c] * a2; }
      suffix = dx_mul(s_tr[cur], suffix);
      cur = cl.parent;
    }
    const int c0 = k.link[cur].dof;
    const double* w1 = sv + c0;
    const double* w2 = k.mu3 + c0;
    // root columns: w x V0 and the translation (constant)
    fs[0] = fs[0] + v0[2] * w1[1] - v0[1] * w1[2];
    fs[1] = fs[1] + v0[0] * w1[2] - v0[2] * w1[0];
    fs[2] = fs[2] + v0[1] * w1[0] - v0[0] * w1[1];
    fm[0] = fm[0] + v0[2] * w2[1] - v0[1] * w2[2];
    fm[1] = fm[1] + v0[0] * w2[2] - v0[2] * w2[0];
    fm[2] = fm[2] + v0[1] * w2[0] - v0[0] * w2[1];
    for (int c = 0; c < 3; ++c) acc += k.mu2[3 * j + c] * fs[c].t - qv[3 * j + c] * fm[c].t;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((tid & 31) == 0) s_red[tid >> 5] = acc;
  __syncthreads();
  if (tid == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) tot += s_red[w];
    k.thb[m] += tot;
  }
}

// Step start in reverse: theta-bar^0 (complete) through guessNext and ReadT to
// the cotangents of the step's input jq / jqd (the output jqd of guessNext,
// prevTr = linearize(T_in) and prevmag = jq_in, adds its own); the rigid rows
// of the cotangent of x^0 (V0, folded into theta-bar) are cleared.  One block.
__global__ void k_skel_adj_end(SkelDev k, const int* step, double* xkb) {
  const int st = *step;
  const double* jq = k.jin + 2 * (size_t)st * k.nq;
  const double* jqd = jq + k.nq;
  for (int j = threadIdx.x; j < k.nr; j += blockDim.x) {
    const size_t g = 3 * (size_t)k.rv[j];
    xkb[g] = 0.0; xkb[g + 1] = 0.0; xkb[g + 2] = 0.0;
  }
  for (int l = threadIdx.x; l < k.L; l += blockDim.x) {
    const SkelLink& lk = k.link[l];
    const int o = lk.sdof;
    if (lk.type != DFEM_JOINT_ALL) {  // mag^0 = 2 jq - jqd, prevmag = jq
      const double tb = k.thb[o];
      k.gjq[o] = 2.0 * tb + k.gjqd[o];
      k.gjqd[o] = -tb;
      continue;
    }
    SkelXf T;
    for (int i = 0; i < 9; ++i) T.R[i] = jq[o + i];
    for (int i = 0; i < 3; ++i) T.d[i] = jq[o + 9 + i];
    const SkelXf Tr = sk_linearize(T);
    // W = prevTr.R^-1 (T^0.R = Tr.R W Tr.R), by cofactors
    const double* P = jqd + o;
    double W[9];
    {
      const double c00 = P[4] * P[8] - P[5] * P[7], c01 = P[5] * P[6] - P[3] * P[8], c02 = P[3] * P[7] - P[4] * P[6];
      const double inv = 1.0 / (P[0] * c00 + P[1] * c01 + P[2] * c02);
      W[0] = inv * c00; W[3] = inv * c01; W[6] = inv * c02;
      W[1] = inv * (P[2] * P[7] - P[1] * P[8]); W[4] = inv * (P[0] * P[8] - P[2] * P[6]);
      W[7] = inv * (P[1] * P[6] - P[0] * P[7]);
      W[2] = inv * (P[1] * P[5] - P[2] * P[4]); W[5] = inv * (P[2] * P[3] - P[0] * P[5]);
      W[8] = inv * (P[0] * P[4] - P[1] * P[3]);
    }
    const double* Tb = k.thb + o;       // cotangent of T^0.R
    const double* tdb = k.thb + o + 9;  // of T^0.d
    const double* Gr = k.gjqd + o;      // of the output prevTr.R = Tr.R
    const double* Gd = k.gjqd + o + 9;
    double WR[9], RW[9], Rb[9], Wb[9], tmp[9], Pb[9];
    sk_mm(W, Tr.R, WR);
    sk_mm(Tr.R, W, RW);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < 3; ++q) {
          a += Tb[3 * r + q] * WR[3 * c + q];  // Tbar (W R)^T
          b += RW[3 * q + r] * Tb[3 * q + c];  // (R W)^T Tbar
        }
        Rb[3 * r + c] = a + b + Gr[3 * r + c];
      }
    for (int r = 0; r < 3; ++r)  // Wbar = R^T Tbar R^T
      for (int c = 0; c < 3; ++c) {
        double a = 0.0;
        for (int q = 0; q < 3; ++q) a += Tr.R[3 * q + r] * Tb[3 * q + c];
        tmp[3 * r + c] = a;
      }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double a = 0.0;
        for (int q = 0; q < 3; ++q) a += tmp[3 * r + q] * Tr.R[3 * c + q];
        Wb[3 * r + c] = a;
      }
    for (int r = 0; r < 3; ++r)  // Pbar = -W^T Wbar W^T
      for (int c = 0; c < 3; ++c) {
        double a = 0.0;
        for (int q = 0; q < 3; ++q) a += W[3 * q + r] * Wb[3 * q + c];
        tmp[3 * r + c] = a;
      }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double a = 0.0;
        for (int q = 0; q < 3; ++q) a += tmp[3 * r + q] * W[3 * c + q];
        Pb[3 * r + c] = -a;
      }
    double Fb[9];
    sk_polar_cotangent(Tr.R, T.R, Rb, Fb);
    double nd_[3], npd[3];
    for (int i = 0; i < 3; ++i) { nd_[i] = 2.0 * tdb[i] + Gd[i]; npd[i] = -tdb[i]; }
    for (int i = 0; i < 9; ++i) { k.gjq[o + i] = Fb[i]; k.gjqd[o + i] = Pb[i]; }
    for (int i = 0; i < 3; ++i) { k.gjq[o + 9 + i] = nd_[i]; k.gjqd[o + 9 + i] = npd[i]; }
  }
}

}  // namespace dfem
