// factor_kernels.cuh — numeric refactorisation of Hs on the GPU after a
// material change (diff_fem: the COROTATE parameter update + PreComputation +
// FactorizeLDLT of forward_all, python/pydifem.cc:207-221,
// sim/fem/World.h:1089-1139,1212-1232).
//
// The symbolic structure (ordering, supernodes, row sets, levels) comes from
// the host and never changes; only values do:
//   k_materials   per tet: w_r = E/(1+nu) vol, w_v = nu w_r
//   k_hs_values   per entry of Hs: base (the E-independent terms: masses,
//                 attachments, muscles, springs, bending) + sum over the tets
//                 touching the entry of E_t * vol_t (G G^T)_ab, in a fixed order
//   k_factor_level one CTA per supernode of one level (leaves first), left
//                 looking: assemble the supernode's columns of Hs (+ the part's
//                 regularisation on the diagonal), subtract the updates of the
//                 descendants that reach these columns (fixed order), dense
//                 Cholesky of the diagonal block in shared memory, triangular
//                 solve of the rows below, inverse of the diagonal block.
// Every value is produced by one thread in a fixed order: the factor is
// deterministic.  The level structure is the one the solves use.  A
// non-positive or non-finite pivot raises the part's failure word; the host
// then retries that part with the reference's regularisation sequence
// (0, 1e-5, x10 ..., World::FactorizeLDLT).
//
// Diagonal of Hs for the contact phase's Jacobi sweeps:
//   k_hs_diag     hdiag_i = Hs_ii
#pragma once
#include "kernels.cuh"

namespace dfem {

struct RefactorDev {
  int T;
  const double* tvol;
  double* tE;
  double* tnu;
  double* twr;
  double* twv;
  int nnz;
  const double* hs_base;
  const int* hc_ptr;    // entry -> its tet contributions
  const int* hc_tet;
  const double* hc_coef;
  double* hs_val;
  const int* hs_ptr;
  const int* hs_col;
  // factor structure and values
  const int* sn_c0;
  const int* sn_w;
  const int* sn_r;
  const int* sn_rofs;
  const int* rowidx;
  const int* sn_lofs;
  double* Lcm;
  const int* sn_dofs;
  double* Dinv;         // row-major
  double* DinvC;        // column-major copy (forward solve)
  double* Ldw;          // diagonal-block workspace (column-major w x w per supernode)
  const int* lvl_sn;
  const int* up_ptr;    // supernode -> updates (descendant d, row range a0..a1 of R_d inside its columns)
  const int* up_d;
  const int* up_a0;
  const int* up_a1;
  const int* sn_part;   // null for a single scene
  const double* part_reg;
  int* part_fail;
};

// part_fail[nparts] (one word past the parts) flags an invalid material
// (non-finite E or nu, or nu <= -1); the tet then keeps its old values.
__global__ void k_materials(RefactorDev f, const double* __restrict__ E, const double* __restrict__ nu, int nparts) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= f.T) return;
  const double e = E[t], n = nu[t];
  if (!isfinite(e) || !isfinite(n) || !(n > -1.0)) {
    atomicExch(f.part_fail + nparts, 1);
    return;
  }
  f.tE[t] = e;
  f.tnu[t] = n;
  const double wr = e / (1.0 + n) * f.tvol[t];  // CorotateFEMConstraint: mMu = E/(1+nu)
  f.twr[t] = wr;
  f.twv[t] = wr * n;
}

__global__ void k_hs_values(RefactorDev f) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= f.nnz) return;
  double v = f.hs_base[k];
  for (int q = f.hc_ptr[k]; q < f.hc_ptr[k + 1]; ++q) v += f.tE[f.hc_tet[q]] * f.hc_coef[q];
  f.hs_val[k] = v;
}

__global__ void k_hs_diag(int N, const int* __restrict__ hs_ptr, const int* __restrict__ hs_col,
                          const double* __restrict__ hs_val, double* hdiag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double v = 0.0;
  for (int k = hs_ptr[i]; k < hs_ptr[i + 1]; ++k)
    if (hs_col[k] == i) v = hs_val[k];
  hdiag[i] = v;
}

// position of global row i among the rows of supernode s: its columns first, then R_s
__device__ __forceinline__ int sn_local_row(int i, int c0, int w, const int* R, int r) {
  if (i < c0 + w) return i - c0;
  int lo = 0, hi = r;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (R[mid] < i) lo = mid + 1; else hi = mid;
  }
  return (lo < r && R[lo] == i) ? w + lo : -1;
}

// FP64 tensor-core tile: D (8x8) += A (8x4, row-major) * B (4x8, column-major),
// one warp (mma.sync m8n8k4 f64).  Fragments: A[lane>>2][lane&3];
// B[lane&3][lane>>2]; C/D rows lane>>2, columns 2*(lane&3) + {0, 1}.
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// split form of a level: used where supernodes x kFactorSplitRatio <= SMs,
// with min(kFactorMaxShares, SMs / supernodes) CTAs per supernode
constexpr int kFactorSplitRatio = 8;
constexpr int kFactorMaxShares = 16;

constexpr int kRowChunk = 1024;  // rows of a descendant update mapped per pass (shared int buffer)
constexpr int kTrsmRows = 64;    // rows of the below-diagonal block staged per TRSM pass

// Shared memory (doubles): L (w x w, column-major) | X = L^-1 (w x w, column-major)
//   | S (kTrsmRows x w, row-major) ; then kRowChunk ints (update row map).
__host__ __device__ inline size_t factor_smem_bytes(int w) {
  return sizeof(double) * (2 * (size_t)w * w + (size_t)kTrsmRows * w) + sizeof(int) * kRowChunk;
}

// The phases of one supernode's factorisation, each run by a whole CTA.  The
// one-launch form (k_factor_level) runs them all in one CTA; the top levels of
// the tree, with few supernodes, split them over launches so that the
// descendant updates and the rows below the diagonal block spread over
// several CTAs per supernode (k_factor_scatter, k_factor_update,
// k_factor_diag, k_factor_trsm).  Each entry is computed by the same
// instructions in the same order either way.

struct FlSn {  // one supernode's layout
  int s, part, c0, w, r;
  const int* R;
  double* Lc;  // r x w, column-major (the panel's rows below)
  double* Ld;  // w x w, column-major (the panel's diagonal block)
};

__device__ __forceinline__ FlSn fl_sn(const RefactorDev& f, int s) {
  FlSn o;
  o.s = s;
  o.part = f.sn_part ? f.sn_part[s] : 0;
  o.c0 = f.sn_c0[s];
  o.w = f.sn_w[s];
  o.r = f.sn_r[s];
  o.R = f.rowidx + f.sn_rofs[s];
  o.Lc = f.Lcm + f.sn_lofs[s];
  o.Ld = f.Ldw + f.sn_dofs[s];
  return o;
}

// 1. this supernode's columns of Hs (lower part) into the panel
__device__ __forceinline__ void fl_scatter(const RefactorDev& f, const FlSn& n, int* s_bad) {
  const double reg = f.part_reg[n.part];
  const int c0 = n.c0, w = n.w, r = n.r;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) n.Ld[q] = 0.0;
  for (int q = threadIdx.x; q < r * w; q += blockDim.x) n.Lc[q] = 0.0;
  __syncthreads();
  for (int c = threadIdx.x; c < w; c += blockDim.x) {
    const int j = c0 + c;
    for (int k = f.hs_ptr[j]; k < f.hs_ptr[j + 1]; ++k) {
      const int i = f.hs_col[k];
      if (i < j) continue;
      const double v = f.hs_val[k] + (i == j ? reg : 0.0);
      const int a = sn_local_row(i, c0, w, n.R, r);
      if (a < 0) { *s_bad = 1; continue; }
      if (a < w) n.Ld[a + c * w] = v; else n.Lc[c * r + (a - w)] = v;
    }
  }
  __syncthreads();
}

// 2. left-looking updates, in list order: for descendant d with rows R_d[a0..a1)
//    in this supernode's columns, P[R_d[x], R_d[y]] -= sum_k L_d[x,k] L_d[y,k]
//    for a0 <= y < a1, y <= x < r_d: 8x8 output tiles on the FP64 tensor cores.
//    Only the panel rows (local index: columns first, then R_s) in [lo, hi)
//    are written; tiles none of whose rows map there are skipped.
__device__ __forceinline__ void fl_update(const RefactorDev& f, const FlSn& n, int* rowmap, int lo, int hi,
                                          int* s_bad) {
  const int c0 = n.c0, w = n.w, r = n.r;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int u = f.up_ptr[n.s]; u < f.up_ptr[n.s + 1]; ++u) {
    const int d = f.up_d[u], a0 = f.up_a0[u], a1 = f.up_a1[u];
    const int wd = f.sn_w[d], rd = f.sn_r[d];
    const int* Rd = f.rowidx + f.sn_rofs[d];
    const double* Lcd = f.Lcm + f.sn_lofs[d];
    const int m = a1 - a0;
    for (int xc = a0; xc < rd; xc += kRowChunk) {
      const int xe = min(rd, xc + kRowChunk);
      for (int x = xc + (int)threadIdx.x; x < xe; x += blockDim.x) {
        const int a = sn_local_row(Rd[x], c0, w, n.R, r);
        if (a < 0) *s_bad = 1;
        rowmap[x - xc] = a;
      }
      __syncthreads();
      const int nti = (xe - xc + 7) / 8, ntj = (m + 7) / 8;
      for (int t = warp; t < nti * ntj; t += nw) {
        const int x0 = xc + 8 * (t / ntj), y0 = a0 + 8 * (t % ntj);
        if (x0 + 7 < y0) continue;  // strictly upper tile
        if (lo > 0 || hi < w + r) {  // rows map monotonically: the tile's first and last row bound its range
          const int af = rowmap[x0 - xc], al = rowmap[min(x0 + 7, xe - 1) - xc];
          if ((al >= 0 && al < lo) || af >= hi) continue;
        }
        const int xa = x0 + (lane >> 2), yb = y0 + (lane >> 2);
        double d0 = 0.0, d1 = 0.0;
        const bool xin = xa < xe, yin = yb < a1;
        // loads of 8 k-steps are issued before their tensor-core steps (L2 latency)
        for (int kb = 0; kb < wd; kb += 32) {
          double av[8], bv[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int ka = kb + 4 * q + (lane & 3);
            av[q] = (xin && ka < wd) ? Lcd[(size_t)ka * rd + xa] : 0.0;
            bv[q] = (yin && ka < wd) ? Lcd[(size_t)ka * rd + yb] : 0.0;
          }
#pragma unroll
          for (int q = 0; q < 8; ++q) dmma_8x8x4(d0, d1, av[q], bv[q]);
        }
        const int xr = x0 + (lane >> 2);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int yc = y0 + 2 * (lane & 3) + i;
          if (xr < xe && yc < a1 && xr >= yc) {
            const int a = rowmap[xr - xc];
            if (a < lo || a >= hi) continue;  // (a < 0 too)
            const int c = Rd[yc] - c0;
            const double v = i == 0 ? d0 : d1;
            if (a < w) n.Ld[a + c * w] -= v; else n.Lc[c * r + (a - w)] -= v;
          }
        }
      }
      __syncthreads();
    }
  }
}

// 3. dense Cholesky of the diagonal block (right looking) in L (shared), kept
//    in the workspace Ld; 4. X = L_ss^-1 (one column per thread) into Dinv
//    (row-major) and DinvC (column-major)
__device__ __forceinline__ void fl_diag(const RefactorDev& f, const FlSn& n, double* L, double* X, int* s_bad) {
  const int w = n.w;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) L[q] = n.Ld[q];
  __syncthreads();
  // (column by column; the scaling and the trailing update of each column are
  // spread over the CTA: every element sees the same operations in the same
  // order as with one thread per row)
  for (int c = 0; c < w; ++c) {
    double dgl = L[c + c * w];
    const bool bad = !(dgl > 0.0) || !isfinite(dgl);
    if (bad) dgl = 1.0;
    const double piv = sqrt(dgl);
    __syncthreads();  // every thread has read the pivot before it is overwritten
    if (threadIdx.x == 0) {
      L[c + c * w] = piv;
      if (bad) *s_bad = 1;
    }
    for (int i = c + 1 + (int)threadIdx.x; i < w; i += blockDim.x) L[i + c * w] /= piv;
    __syncthreads();
    const int m = w - c - 1;  // trailing block: rows and columns c+1 .. w-1, lower part
    for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
      const int jj = q / m, ii = q % m;
      if (ii < jj) continue;
      const int i = c + 1 + ii, j = c + 1 + jj;
      const double ljc = L[j + c * w];
      L[i + j * w] -= L[i + c * w] * ljc;
    }
    __syncthreads();
  }
  // the factored diagonal block stays in the workspace (the dense-inverse form reads it)
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) n.Ld[q] = L[q];
  for (int c = threadIdx.x; c < w; c += blockDim.x) {
    for (int i = 0; i < c; ++i) X[i + c * w] = 0.0;
    for (int i = c; i < w; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) v -= L[i + k * w] * X[k + c * w];
      X[i + c * w] = v / L[i + i * w];
    }
  }
  __syncthreads();
  double* Di = f.Dinv + f.sn_dofs[n.s];  // row-major lower
  double* DiC = f.DinvC + f.sn_dofs[n.s];
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    Di[q] = X[(q / w) + (q % w) * w];
    DiC[q] = X[q];
  }
}

// 5. rows below: L_{R,s} = P_R X^T, kTrsmRows rows at a time (staged in S,
//    then overwritten), row chunks rb0, rb0 + rbs, ...
__device__ __forceinline__ void fl_trsm(const FlSn& n, const double* X, double* S, int rb0, int rbs) {
  const int w = n.w, r = n.r;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int rb = rb0; rb < r; rb += rbs) {
    const int nr = min(kTrsmRows, r - rb);
    for (int q = threadIdx.x; q < nr * w; q += blockDim.x) {
      const int x = q % nr, c = q / nr;  // coalesced along the column-major block
      S[x * w + c] = n.Lc[c * r + rb + x];
    }
    __syncthreads();
    const int nti = (nr + 7) / 8, ntj = (w + 7) / 8;
    for (int t = warp; t < nti * ntj; t += nw) {
      const int x0 = 8 * (t / ntj), y0 = 8 * (t % ntj);
      const int xa = x0 + (lane >> 2), yb = y0 + (lane >> 2);
      double d0 = 0.0, d1 = 0.0;
      for (int k0 = 0; k0 < w; k0 += 4) {
        const int ka = k0 + (lane & 3);
        const double av = (xa < nr && ka < w) ? S[xa * w + ka] : 0.0;
        const double bv = (yb < w && ka < w) ? X[yb + ka * w] : 0.0;  // (X^T)[k][y] = X[y][k]
        dmma_8x8x4(d0, d1, av, bv);
      }
      const int xr = x0 + (lane >> 2);
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int yc = y0 + 2 * (lane & 3) + i;
        if (xr < nr && yc < w) n.Lc[yc * r + rb + xr] = i == 0 ? d0 : d1;
      }
    }
    __syncthreads();
  }
}

// The one-launch form: one CTA per supernode of the level (shared memory as
// factor_smem_bytes).
__global__ void __launch_bounds__(256) k_factor_level(RefactorDev f, int lvl_begin) {
  extern __shared__ __align__(16) double fsh[];
  __shared__ int s_bad;
  const FlSn n = fl_sn(f, f.lvl_sn[lvl_begin + blockIdx.x]);
  double* L = fsh;
  double* X = fsh + n.w * n.w;
  double* S = X + n.w * n.w;
  int* rowmap = reinterpret_cast<int*>(S + kTrsmRows * n.w);
  if (threadIdx.x == 0) s_bad = 0;
  fl_scatter(f, n, &s_bad);
  fl_update(f, n, rowmap, 0, n.w + n.r, &s_bad);
  fl_diag(f, n, L, X, &s_bad);
  fl_trsm(n, X, S, 0, kTrsmRows);
  if (threadIdx.x == 0 && s_bad) atomicExch(f.part_fail + n.part, 1);
}

// The split form of one level (blockIdx.x: the supernode; blockIdx.y: its
// share of the work, gridDim.y shares).
__global__ void __launch_bounds__(256) k_factor_scatter(RefactorDev f, int lvl_begin) {
  __shared__ int s_bad;
  const FlSn n = fl_sn(f, f.lvl_sn[lvl_begin + blockIdx.x]);
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  fl_scatter(f, n, &s_bad);
  if (threadIdx.x == 0 && s_bad) atomicExch(f.part_fail + n.part, 1);
}

// the panel rows (local index) of share y: [y ceil((w + r) / shares), ...)
__global__ void __launch_bounds__(256) k_factor_update(RefactorDev f, int lvl_begin) {
  __shared__ int s_bad;
  __shared__ int rowmap[kRowChunk];
  const FlSn n = fl_sn(f, f.lvl_sn[lvl_begin + blockIdx.x]);
  const int rows = n.w + n.r, per = (rows + gridDim.y - 1) / gridDim.y;
  const int lo = blockIdx.y * per, hi = min(rows, lo + per);
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  if (lo < hi) fl_update(f, n, rowmap, lo, hi, &s_bad);
  if (threadIdx.x == 0 && s_bad) atomicExch(f.part_fail + n.part, 1);
}

__global__ void __launch_bounds__(256) k_factor_diag(RefactorDev f, int lvl_begin) {
  extern __shared__ __align__(16) double fsh[];
  __shared__ int s_bad;
  const FlSn n = fl_sn(f, f.lvl_sn[lvl_begin + blockIdx.x]);
  if (threadIdx.x == 0) s_bad = 0;
  fl_diag(f, n, fsh, fsh + n.w * n.w, &s_bad);
  if (threadIdx.x == 0 && s_bad) atomicExch(f.part_fail + n.part, 1);
}

// row chunks y, y + shares, ... of the rows below (X read back from DinvC)
__global__ void __launch_bounds__(256) k_factor_trsm(RefactorDev f, int lvl_begin) {
  extern __shared__ __align__(16) double fsh[];
  const FlSn n = fl_sn(f, f.lvl_sn[lvl_begin + blockIdx.x]);
  if (n.r <= (int)blockIdx.y * kTrsmRows) return;
  double* X = fsh;
  double* S = fsh + n.w * n.w;
  const double* DiC = f.DinvC + f.sn_dofs[n.s];
  for (int q = threadIdx.x; q < n.w * n.w; q += blockDim.x) X[q] = DiC[q];
  __syncthreads();
  fl_trsm(n, X, S, blockIdx.y * kTrsmRows, gridDim.y * kTrsmRows);
}

}  // namespace dfem
