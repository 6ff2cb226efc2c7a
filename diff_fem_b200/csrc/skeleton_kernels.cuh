// Articulated skeleton: links whose vertices move rigidly, coupled to the free
// vertices through the Schur complement of the PD system.
//
// Replaces Link (sim/constants.h:28-247: ReadT/WriteT, guessNext,
// ComputeV0NTr, ComputeTildaV, UpdateT) and the rigid branch of
// World::ComputeSolution (sim/fem/World.h:1600-1670) with its precomputed
// Schur complement Qb_M - Qc_L Qf^-1 Qc_L^T (World.h:1100-1135).
//
// Formulation.  The step's PD solve already computes u = H^-1 c (H the whole
// PD matrix, c = b + J d).  With the rigid positions prescribed as x_R, the
// free positions of the reference's Qf x_F = c_F - Qc_L^T x_R are
//   x_F = u_F + Z_F C^-1 (x_R - u_R),   Z = H^-1 E_R,  C = Z_R = (H^-1)_RR,
// and C^-1 is exactly the Schur complement Qb_M - Qc_L Qf^-1 Qc_L^T.  The
// reference's right-hand side of the link system, tildaV^T (c_R - Qb_M V0 -
// Qc_L y) with y = Qf^-1 (c_F - Qc_L^T V0), equals tildaV^T C^-1 (u_R - V0).
// So each PD iteration costs the step's usual solve plus, in one CTA, the
// dense link system S s = tildaV^T C^-1 (u_R - V0) + tau with
// S = tildaV^T C^-1 tildaV (LU with full pivoting like Eigen::FullPivLU),
// the multiplier q = C^-1 (V0 + tildaV s - u_R), the link update and the new
// V0, and then x_F = u_F + Z_F q over all vertices (k_skel_apply).  Z (N x nr,
// column-major) and C^-1 (nr x nr) are built once on the host from the factor.
//
// All scalars are 3x3 blocks of kron(., I3) in the reference; here the rigid
// vectors are (nr x 3) and the dense matrices scalar.
#pragma once

#include "kernels.cuh"
#include "pd_math.cuh"

namespace dfem {

struct SkelXf { double R[9]; double d[3]; };  // Transformation: x -> R x + d (R row-major)

struct SkelLink {         // constant per scene
  int parent, type, dof, sdof, chan, r0, r1;
  double joint[3], axis[3], d0[3], nx[9], nnt[9];
};

struct SkelState {        // per link, mutable
  double mag, prevmag;
  SkelXf T, Tr, prevTr, prefix, dT, M;  // M = prefix * Tr
};

struct SkelDev {
  int L, ndof, nr, N;
  const SkelLink* link;
  SkelState* st;
  const int* rv;          // rigid index j -> internal vertex
  const int* rlink;       // rigid index j -> link
  const int* ridx;        // internal vertex -> rigid index or -1
  const double* rest;     // 3 nr rest positions (Link::restpos)
  const double* cinv;     // nr x nr row-major
  const double* zcm;      // Z column-major: Z[j N + i]
  double* jq;             // joint state (World::mJointQ), 12 + L - 1
  double* jqd;            // (World::mJointQd)
  double* v0;             // 3 nr: V0 of the current links
  double* w;              // 3 nr: u_R - V0, then tildaV s - (u_R - V0)
  double* rr;             // 3 nr: C^-1 (u_R - V0)
  double* q;              // 3 nr: the multiplier C^-1 (V0 + tildaV s - u_R)
  double* tv;             // 3 nr x ndof: tildaV (row 3 j + c)
  double* kt;             // 3 nr x ndof: C^-1 tildaV per component
  double* sm;             // ndof x ndof: S, then its LU
  double* rhs;            // ndof
  double* sol;            // ndof
  int* perm;              // ndof column permutation of the LU
  // history for the adjoint: per step and PD iteration k, the joint state
  // theta^k (jq layout: the root's T, then one magnitude per link) | the link
  // system's solution s^k | the multiplier q^k; per step its input (jq, jqd)
  int nq, K;
  long long hstride;      // nq + ndof + 3 nr
  double* hist;           // steps x (K + 1) x hstride
  double* jin;            // steps x 2 nq
  // adjoint work
  double* thb;            // nq: cotangent of the current theta
  double* sb;             // ndof: cotangent of s
  double* gjq;            // nq: cotangent of the step's output jq (input jq after the step's adjoint)
  double* gjqd;           // nq: the same for jqd
  double* mu2;            // 3 nr: rigid block of the KKT adjoint
  double* mu3;            // ndof: link block of the KKT adjoint
  double* dlt;            // 3 nr: linear rigid positions minus the iterate's
};

__device__ __forceinline__ double* sk_hrow(const SkelDev& k, int step, int it) {
  return k.hist + ((long long)step * (k.K + 1) + it) * k.hstride;
}

// theta (jq layout) of the current link states, and back
__device__ __forceinline__ void sk_pack(const SkelDev& k, int l, double* th) {
  const SkelLink& lk = k.link[l];
  const SkelState& s = k.st[l];
  if (lk.type == DFEM_JOINT_ALL) {
    for (int i = 0; i < 9; ++i) th[lk.sdof + i] = s.T.R[i];
    for (int i = 0; i < 3; ++i) th[lk.sdof + 9 + i] = s.T.d[i];
  } else {
    th[lk.sdof] = s.mag;
  }
}

// ---- 3x3 and transformation helpers (row-major R) ---------------------------
__device__ __forceinline__ void sk_identity(SkelXf& t) {
  for (int i = 0; i < 9; ++i) t.R[i] = (i % 4 == 0) ? 1.0 : 0.0;
  t.d[0] = t.d[1] = t.d[2] = 0.0;
}
__device__ __forceinline__ void sk_mm(const double* a, const double* b, double* o) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
}
__device__ __forceinline__ void sk_mv(const double* a, const double* v, double* o) {
  for (int r = 0; r < 3; ++r) o[r] = a[3 * r] * v[0] + a[3 * r + 1] * v[1] + a[3 * r + 2] * v[2];
}
// a * b (Transformation::operator*)
__device__ __forceinline__ SkelXf sk_mul(const SkelXf& a, const SkelXf& b) {
  SkelXf o;
  sk_mm(a.R, b.R, o.R);
  double t[3];
  sk_mv(a.R, b.d, t);
  for (int i = 0; i < 3; ++i) o.d[i] = t[i] + a.d[i];
  return o;
}
__device__ __forceinline__ void sk_apply(const SkelXf& a, const double* v, double* o) {
  double t[3];
  sk_mv(a.R, v, t);
  for (int i = 0; i < 3; ++i) o[i] = t[i] + a.d[i];
}
// Transformation::linearize: the rotation U V^T of the SVD of R
__device__ __forceinline__ SkelXf sk_linearize(const SkelXf& t) {
  Mat3<double> F;
  for (int c = 0; c < 3; ++c) F.c[c] = mk3(t.R[c], t.R[3 + c], t.R[6 + c]);
  const Svd3<double> sv = svd3(F);
  SkelXf o;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const double u0 = r == 0 ? sv.u[0].x : r == 1 ? sv.u[0].y : sv.u[0].z;
      const double u1 = r == 0 ? sv.u[1].x : r == 1 ? sv.u[1].y : sv.u[1].z;
      const double u2 = r == 0 ? sv.u[2].x : r == 1 ? sv.u[2].y : sv.u[2].z;
      const double v0 = c == 0 ? sv.v[0].x : c == 1 ? sv.v[0].y : sv.v[0].z;
      const double v1 = c == 0 ? sv.v[1].x : c == 1 ? sv.v[1].y : sv.v[1].z;
      const double v2 = c == 0 ? sv.v[2].x : c == 1 ? sv.v[2].y : sv.v[2].z;
      o.R[3 * r + c] = u0 * v0 + u1 * v1 + u2 * v2;
    }
  o.d[0] = t.d[0]; o.d[1] = t.d[1]; o.d[2] = t.d[2];
  return o;
}

// Dense solve A x = B (n x n row-major, k right-hand sides row-major), LU with
// full pivoting: the pivot is the largest |a| of the remaining block, the
// first one in row-major order on ties.  One thread (3x3 systems).
__device__ void sk_fullpiv_small(int n, int k, double* A, double* B, double* X, int* cp) {
  for (int i = 0; i < n; ++i) cp[i] = i;
  for (int p = 0; p < n; ++p) {
    int pr = p, pc = p;
    double best = -1.0;
    for (int r = p; r < n; ++r)
      for (int c = p; c < n; ++c)
        if (fabs(A[r * n + c]) > best) { best = fabs(A[r * n + c]); pr = r; pc = c; }
    if (pr != p) {
      for (int c = 0; c < n; ++c) { double t = A[p * n + c]; A[p * n + c] = A[pr * n + c]; A[pr * n + c] = t; }
      for (int c = 0; c < k; ++c) { double t = B[p * k + c]; B[p * k + c] = B[pr * k + c]; B[pr * k + c] = t; }
    }
    if (pc != p) {
      for (int r = 0; r < n; ++r) { double t = A[r * n + p]; A[r * n + p] = A[r * n + pc]; A[r * n + pc] = t; }
      int t = cp[p]; cp[p] = cp[pc]; cp[pc] = t;
    }
    const double piv = A[p * n + p];
    for (int r = p + 1; r < n; ++r) {
      const double f = A[r * n + p] / piv;
      A[r * n + p] = f;
      for (int c = p + 1; c < n; ++c) A[r * n + c] -= f * A[p * n + c];
      for (int c = 0; c < k; ++c) B[r * k + c] -= f * B[p * k + c];
    }
  }
  for (int r = n - 1; r >= 0; --r)
    for (int c = 0; c < k; ++c) {
      double v = B[r * k + c];
      for (int q = r + 1; q < n; ++q) v -= A[r * n + q] * B[q * k + c];
      B[r * k + c] = v / A[r * n + r];
    }
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < k; ++c) X[cp[r] * k + c] = B[r * k + c];
}

// The same LU with full pivoting for the link system (n <= 6 + kMaxLinks - 1),
// one right-hand side, by a whole block: each pivot is found by a block
// argmax (largest |a|, ties to the first in row-major order, as the
// sequential scan) and the rows below it are eliminated in parallel.
__device__ void sk_fullpiv_block(int n, double* A, double* b, double* x, int* cp) {
  __shared__ double s_best[32];
  __shared__ int s_idx[32];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < n; i += nt) cp[i] = i;
  __syncthreads();
  for (int p = 0; p < n; ++p) {
    const int m = n - p;
    double best = -1.0;
    int bi = 0x7fffffff;
    for (int e = tid; e < m * m; e += nt) {  // e in row-major order of the block
      const int r = p + e / m, c = p + e % m;
      const double a = fabs(A[r * n + c]);
      if (a > best) { best = a; bi = e; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if ((tid & 31) == 0) { s_best[tid >> 5] = best; s_idx[tid >> 5] = bi; }
    __syncthreads();
    if (tid == 0) {
      for (int w = 1; w < (nt + 31) / 32; ++w)
        if (s_best[w] > s_best[0] || (s_best[w] == s_best[0] && s_idx[w] < s_idx[0])) {
          s_best[0] = s_best[w]; s_idx[0] = s_idx[w];
        }
    }
    __syncthreads();
    const int pr = p + s_idx[0] / m, pc = p + s_idx[0] % m;
    __syncthreads();
    if (pr != p) {
      for (int c = tid; c < n; c += nt) { double t = A[p * n + c]; A[p * n + c] = A[pr * n + c]; A[pr * n + c] = t; }
      if (tid == 0) { double t = b[p]; b[p] = b[pr]; b[pr] = t; }
    }
    __syncthreads();
    if (pc != p) {
      for (int r = tid; r < n; r += nt) { double t = A[r * n + p]; A[r * n + p] = A[r * n + pc]; A[r * n + pc] = t; }
      if (tid == 0) { int t = cp[p]; cp[p] = cp[pc]; cp[pc] = t; }
    }
    __syncthreads();
    const double piv = A[p * n + p];
    for (int r = p + 1 + tid; r < n; r += nt) {
      const double f = A[r * n + p] / piv;
      A[r * n + p] = f;
      for (int c = p + 1; c < n; ++c) A[r * n + c] -= f * A[p * n + c];
      b[r] -= f * b[p];
    }
    __syncthreads();
  }
  if (tid == 0) {
    for (int r = n - 1; r >= 0; --r) {
      double v = b[r];
      for (int q = r + 1; q < n; ++q) v -= A[r * n + q] * b[q];
      b[r] = v / A[r * n + r];
    }
    for (int r = 0; r < n; ++r) x[cp[r]] = b[r];
  }
  __syncthreads();
}

// Link::ComputeV0NTr for every link in index order (parents first): Tr,
// prefix and M = prefix * Tr.  One thread.
__device__ void sk_kinematics(const SkelDev& k) {
  for (int l = 0; l < k.L; ++l) {
    const SkelLink& lk = k.link[l];
    SkelState& s = k.st[l];
    if (lk.type == DFEM_JOINT_ALL) {
      s.Tr = sk_linearize(s.T);
    } else if (lk.type == DFEM_JOINT_ROTATIONAL) {
      const double C = cos(s.mag), S = sin(s.mag);
      for (int i = 0; i < 9; ++i) s.Tr.R[i] = (C * (i % 4 == 0 ? 1.0 : 0.0) + S * lk.nx[i]) + (1.0 - C) * lk.nnt[i];
      for (int i = 0; i < 3; ++i) s.Tr.d[i] = lk.d0[i];
    } else {
      for (int i = 0; i < 3; ++i) s.Tr.d[i] = s.mag * lk.axis[i] + lk.d0[i];
    }
    if (lk.parent >= 0) s.prefix = sk_mul(k.st[lk.parent].prefix, k.st[lk.parent].Tr);
    s.M = sk_mul(s.prefix, s.Tr);
  }
}

// V0 of rigid vertex j (the links' M current)
__device__ __forceinline__ void sk_v0(const SkelDev& k, int j, double* o) {
  const SkelLink& lk = k.link[k.rlink[j]];
  const double v[3] = {k.rest[3 * j] - lk.joint[0], k.rest[3 * j + 1] - lk.joint[1], k.rest[3 * j + 2] - lk.joint[2]};
  sk_apply(k.st[k.rlink[j]].M, v, o);
}

// dT of every rotational / prismatic link (ComputeTildaV), threads over links
__device__ void sk_dt(const SkelDev& k, int tid, int nt) {
  for (int l = tid; l < k.L; l += nt) {
    const SkelLink& lk = k.link[l];
    SkelState& s = k.st[l];
    if (lk.type == DFEM_JOINT_ROTATIONAL) {
      const double C = cos(s.mag), S = sin(s.mag);
      for (int i = 0; i < 9; ++i) s.dT.R[i] = (-S * (i % 4 == 0 ? 1.0 : 0.0) + C * lk.nx[i]) + S * lk.nnt[i];
    } else if (lk.type == DFEM_JOINT_PRISMATIC) {
      for (int i = 0; i < 9; ++i) s.dT.R[i] = 0.0;
      for (int i = 0; i < 3; ++i) s.dT.d[i] = lk.axis[i];
    }
  }
}

// tildaV (Link::ComputeTildaV): one rigid vertex per thread, walking its chain
// to the root (V0 of the current links in k.v0)
__device__ void sk_tildav(const SkelDev& k, int tid, int nt) {
  const int nr = k.nr, nd = k.ndof;
  for (int j = tid; j < nr; j += nt) {
    double* row0 = k.tv + (3 * (size_t)j) * nd;
    double* row1 = row0 + nd;
    double* row2 = row1 + nd;
    for (int a = 0; a < nd; ++a) { row0[a] = 0.0; row1[a] = 0.0; row2[a] = 0.0; }
    const int me = k.rlink[j];
    const SkelLink& ml = k.link[me];
    const double vinit[3] = {k.rest[3 * j] - ml.joint[0], k.rest[3 * j + 1] - ml.joint[1],
                             k.rest[3 * j + 2] - ml.joint[2]};
    SkelXf suffix;
    sk_identity(suffix);
    int cur = me;
    while (k.link[cur].parent >= 0) {
      const SkelLink& cl = k.link[cur];
      const SkelState& cs = k.st[cur];
      double t[3];
      if (cl.type == DFEM_JOINT_ROTATIONAL) {
        double a[3], b[3];
        sk_apply(suffix, vinit, a);
        sk_mv(cs.dT.R, a, b);
        sk_mv(cs.prefix.R, b, t);
      } else {
        sk_mv(cs.prefix.R, cs.dT.d, t);
      }
      row0[cl.dof] = t[0]; row1[cl.dof] = t[1]; row2[cl.dof] = t[2];
      suffix = sk_mul(cs.Tr, suffix);  // the parent's suffix: cur.Tr * cur.suffix
      cur = cl.parent;
    }
    const int c0 = k.link[cur].dof;
    const double vx = k.v0[3 * j], vy = k.v0[3 * j + 1], vz = k.v0[3 * j + 2];
    row0[c0 + 1] = vz;  row0[c0 + 2] = -vy;
    row1[c0 + 0] = -vz; row1[c0 + 2] = vx;
    row2[c0 + 0] = vy;  row2[c0 + 1] = -vx;
    row0[c0 + 3] = 1.0; row1[c0 + 4] = 1.0; row2[c0 + 5] = 1.0;
  }
}

// rr = C^-1 (u_R - V0) and kt = C^-1 tildaV, per component
__device__ void sk_cinv_products(const SkelDev& k, int tid, int nt) {
  const int nr = k.nr, nd = k.ndof;
  for (int e = tid; e < 3 * nr; e += nt) {
    const int i = e / 3, c = e % 3;
    double acc = 0.0;
    for (int j = 0; j < nr; ++j) acc += k.cinv[(size_t)i * nr + j] * k.w[3 * j + c];
    k.rr[e] = acc;
  }
  for (int e = tid; e < 3 * nr * nd; e += nt) {
    const int r = e / nd, a = e % nd, i = r / 3, c = r % 3;
    double acc = 0.0;
    for (int j = 0; j < nr; ++j) acc += k.cinv[(size_t)i * nr + j] * k.tv[(3 * (size_t)j + c) * nd + a];
    k.kt[e] = acc;
  }
}

// Step start: Link::ReadT (the root's Tr = linearize(T), its value after the
// previous step's last ComputeV0NTr), guessNext, ComputeV0NTr; the rigid
// vertices of the first iterate are V0 (also in the stored iterate 0).  The
// step's input joint state and theta^0 go to the adjoint's history.  One block.
__global__ void k_skel_begin(SkelDev k, double* xk, const int* step, double* hist_x, long long hist_step) {
  const int st = *step;
  if (k.jin)
    for (int i = threadIdx.x; i < k.nq; i += blockDim.x) {
      k.jin[2 * (size_t)st * k.nq + i] = k.jq[i];
      k.jin[(2 * (size_t)st + 1) * k.nq + i] = k.jqd[i];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int l = 0; l < k.L; ++l) {
      const SkelLink& lk = k.link[l];
      SkelState& s = k.st[l];
      if (lk.type == DFEM_JOINT_ALL) {
        for (int i = 0; i < 9; ++i) { s.T.R[i] = k.jq[lk.sdof + i]; s.prevTr.R[i] = k.jqd[lk.sdof + i]; }
        for (int i = 0; i < 3; ++i) { s.T.d[i] = k.jq[lk.sdof + 9 + i]; s.prevTr.d[i] = k.jqd[lk.sdof + 9 + i]; }
        s.Tr = sk_linearize(s.T);
        // guessNext: T.d = 2 Tr.d - prevTr.d, T.R = Tr.R prevTr.R^-1 Tr.R, prevTr = Tr
        for (int i = 0; i < 3; ++i) s.T.d[i] = 2.0 * s.Tr.d[i] - s.prevTr.d[i];
        double A[9], B[9], X[9];
        int cp[3];
        for (int i = 0; i < 9; ++i) { A[i] = s.prevTr.R[i]; B[i] = s.Tr.R[i]; }
        sk_fullpiv_small(3, 3, A, B, X, cp);
        sk_mm(s.Tr.R, X, s.T.R);
        s.prevTr = s.Tr;
      } else {
        s.mag = k.jq[lk.sdof];
        s.prevmag = k.jqd[lk.sdof];
        const double t = s.mag;
        s.mag = 2.0 * s.mag - s.prevmag;
        s.prevmag = t;
      }
      if (l == 0) sk_identity(s.prefix);
      if (lk.type == DFEM_JOINT_PRISMATIC) {  // Tr.R of a prismatic link stays the identity
        for (int i = 0; i < 9; ++i) s.Tr.R[i] = (i % 4 == 0) ? 1.0 : 0.0;
      }
    }
    sk_kinematics(k);
  }
  __syncthreads();
  if (k.hist)
    for (int l = threadIdx.x; l < k.L; l += blockDim.x) sk_pack(k, l, sk_hrow(k, st, 0));
  double* hx = hist_x ? hist_x + (size_t)st * hist_step : nullptr;
  for (int j = threadIdx.x; j < k.nr; j += blockDim.x) {
    double p[3];
    sk_v0(k, j, p);
    const int v = k.rv[j];
    for (int c = 0; c < 3; ++c) {
      k.v0[3 * j + c] = p[c];
      xk[3 * (size_t)v + c] = p[c];
      if (hx) hx[3 * (size_t)v + c] = p[c];
    }
  }
}

// One PD iteration's rigid stage (one block), after the solve wrote
// z = u - x_t: the link system, the multiplier q, UpdateT and the new V0
// (z of the rigid vertices becomes V0 - x_t).  s, q and the new theta of
// iteration k (*kptr) go to the adjoint's history.
__global__ void k_skel_stage(SkelDev k, const double* xt, double* z, const double* act_all, const int* step,
                             int nseg, const int* kptr) {
  const int tid = threadIdx.x, nt = blockDim.x, nr = k.nr, nd = k.ndof;
  const int it = *kptr;
  double* h0 = k.hist ? sk_hrow(k, *step, it) : nullptr;
  double* h1 = k.hist ? sk_hrow(k, *step, it + 1) : nullptr;
  // u_R - V0
  for (int e = tid; e < 3 * nr; e += nt) {
    const int j = e / 3, c = e % 3;
    const size_t g = 3 * (size_t)k.rv[j] + c;
    k.w[e] = (xt[g] + z[g]) - k.v0[e];
  }
  sk_dt(k, tid, nt);
  __syncthreads();
  sk_tildav(k, tid, nt);
  __syncthreads();
  sk_cinv_products(k, tid, nt);
  __syncthreads();
  // S = tildaV^T C^-1 tildaV and tmp = tildaV^T rr + tau (mcs[6+i] += mJointTorque[i])
  for (int e = tid; e < nd * nd; e += nt) {
    const int a = e / nd, b = e % nd;
    double acc = 0.0;
    for (int r = 0; r < 3 * nr; ++r) acc += k.tv[(size_t)r * nd + a] * k.kt[(size_t)r * nd + b];
    k.sm[e] = acc;
  }
  for (int a = tid; a < nd; a += nt) {
    double acc = 0.0;
    for (int r = 0; r < 3 * nr; ++r) acc += k.tv[(size_t)r * nd + a] * k.rr[r];
    k.rhs[a] = acc;
  }
  __syncthreads();
  for (int l = 1 + tid; l < k.L; l += nt)
    if (k.link[l].chan >= 0) k.rhs[k.link[l].dof] += act_all[(size_t)(*step) * nseg + k.link[l].chan];
  __syncthreads();
  sk_fullpiv_block(nd, k.sm, k.rhs, k.sol, k.perm);
  // q = C^-1 (tildaV s - (u_R - V0))
  for (int r = tid; r < 3 * nr; r += nt) {
    double acc = 0.0;
    for (int a = 0; a < nd; ++a) acc += k.tv[(size_t)r * nd + a] * k.sol[a];
    k.rr[r] = acc - k.w[r];
  }
  __syncthreads();
  for (int e = tid; e < 3 * nr; e += nt) {
    const int i = e / 3, c = e % 3;
    double acc = 0.0;
    for (int j = 0; j < nr; ++j) acc += k.cinv[(size_t)i * nr + j] * k.rr[3 * j + c];
    k.q[e] = acc;
    if (h0) h0[k.nq + nd + e] = acc;
  }
  if (h0)
    for (int a = tid; a < nd; a += nt) h0[k.nq + a] = k.sol[a];
  // Link::UpdateT
  for (int l = tid; l < k.L; l += nt) {
    const SkelLink& lk = k.link[l];
    SkelState& s = k.st[l];
    const double* sv = k.sol + lk.dof;
    if (lk.type == DFEM_JOINT_PRISMATIC) {
      s.mag += sv[0];
    } else if (lk.type == DFEM_JOINT_ROTATIONAL) {
      const double C = cos(s.mag), S = sin(s.mag);
      s.mag = atan2(S + C * sv[0], C - S * sv[0]);
    } else {
      const double t[9] = {1.0, -sv[2], sv[1], sv[2], 1.0, -sv[0], -sv[1], sv[0], 1.0};
      sk_mm(t, s.Tr.R, s.T.R);
      double td[3];
      sk_mv(t, s.Tr.d, td);
      for (int i = 0; i < 3; ++i) s.T.d[i] = td[i] + sv[3 + i];
    }
    if (h1) sk_pack(k, l, h1);
  }
  __syncthreads();
  if (tid == 0) sk_kinematics(k);
  __syncthreads();
  for (int j = tid; j < nr; j += nt) {
    double p[3];
    sk_v0(k, j, p);
    const size_t g = 3 * (size_t)k.rv[j];
    for (int c = 0; c < 3; ++c) { k.v0[3 * j + c] = p[c]; z[g + c] = p[c] - xt[g + c]; }
  }
}

// x_F = u_F + Z_F q: the free vertices' z gains Z q (rigid vertices were set
// by k_skel_stage)
__global__ void k_skel_apply(SkelDev k, double* z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k.N || k.ridx[i] >= 0) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int j = 0; j < k.nr; ++j) {
    const double zz = k.zcm[(size_t)j * k.N + i];
    a0 += zz * k.q[3 * j]; a1 += zz * k.q[3 * j + 1]; a2 += zz * k.q[3 * j + 2];
  }
  z[3 * (size_t)i] += a0; z[3 * (size_t)i + 1] += a1; z[3 * (size_t)i + 2] += a2;
}

// Step end: Link::WriteT
__global__ void k_skel_end(SkelDev k) {
  if (threadIdx.x != 0) return;
  for (int l = 0; l < k.L; ++l) {
    const SkelLink& lk = k.link[l];
    const SkelState& s = k.st[l];
    if (lk.type == DFEM_JOINT_ALL) {
      for (int i = 0; i < 9; ++i) { k.jq[lk.sdof + i] = s.T.R[i]; k.jqd[lk.sdof + i] = s.prevTr.R[i]; }
      for (int i = 0; i < 3; ++i) { k.jq[lk.sdof + 9 + i] = s.T.d[i]; k.jqd[lk.sdof + 9 + i] = s.prevTr.d[i]; }
    } else {
      k.jq[lk.sdof] = s.mag;
      k.jqd[lk.sdof] = s.prevmag;
    }
  }
}

}  // namespace dfem
