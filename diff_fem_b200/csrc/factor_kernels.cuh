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
  double* Dinv;
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

// Shared memory: L (w x w, column-major) | X = L^-1 (w x w, column-major); 2 w^2 doubles.
__global__ void __launch_bounds__(256) k_factor_level(RefactorDev f, int lvl_begin) {
  extern __shared__ __align__(16) double fsh[];
  __shared__ int s_bad;
  const int s = f.lvl_sn[lvl_begin + blockIdx.x];
  const int part = f.sn_part ? f.sn_part[s] : 0;
  const int c0 = f.sn_c0[s], w = f.sn_w[s], r = f.sn_r[s];
  const int* R = f.rowidx + f.sn_rofs[s];
  double* Lc = f.Lcm + f.sn_lofs[s];   // r x w, column-major
  double* Ld = f.Ldw + f.sn_dofs[s];   // w x w, column-major
  const double reg = f.part_reg[part];
  if (threadIdx.x == 0) s_bad = 0;
  // 1. this supernode's columns of Hs (lower part)
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) Ld[q] = 0.0;
  for (int q = threadIdx.x; q < r * w; q += blockDim.x) Lc[q] = 0.0;
  __syncthreads();
  for (int c = threadIdx.x; c < w; c += blockDim.x) {
    const int j = c0 + c;
    for (int k = f.hs_ptr[j]; k < f.hs_ptr[j + 1]; ++k) {
      const int i = f.hs_col[k];
      if (i < j) continue;
      const double v = f.hs_val[k] + (i == j ? reg : 0.0);
      const int a = sn_local_row(i, c0, w, R, r);
      if (a < 0) { s_bad = 1; continue; }
      if (a < w) Ld[a + c * w] = v; else Lc[c * r + (a - w)] = v;
    }
  }
  __syncthreads();
  // 2. updates of the descendants, in list order: column block R_d[a0..a1) of s,
  //    rows R_d[a0..r_d) : P -= L_{rows, d} L_{cols, d}^T
  for (int u = f.up_ptr[s]; u < f.up_ptr[s + 1]; ++u) {
    const int d = f.up_d[u], a0 = f.up_a0[u], a1 = f.up_a1[u];
    const int wd = f.sn_w[d], rd = f.sn_r[d];
    const int* Rd = f.rowidx + f.sn_rofs[d];
    const double* Lcd = f.Lcm + f.sn_lofs[d];
    for (int x = a0 + (int)threadIdx.x; x < rd; x += blockDim.x) {
      const int a = sn_local_row(Rd[x], c0, w, R, r);
      if (a < 0) { s_bad = 1; continue; }
      const int yend = x < a1 ? x + 1 : a1;
      for (int y = a0; y < yend; ++y) {
        double acc = 0.0;
        for (int k = 0; k < wd; ++k) acc += Lcd[k * rd + x] * Lcd[k * rd + y];
        const int c = Rd[y] - c0;
        if (a < w) Ld[a + c * w] -= acc; else Lc[c * r + (a - w)] -= acc;
      }
    }
    __syncthreads();
  }
  // 3. dense Cholesky of the diagonal block in shared memory (right looking)
  double* L = fsh;
  double* X = fsh + w * w;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) L[q] = Ld[q];
  __syncthreads();
  for (int c = 0; c < w; ++c) {
    if (threadIdx.x == 0) {
      double dgl = L[c + c * w];
      if (!(dgl > 0.0) || !isfinite(dgl)) { s_bad = 1; dgl = 1.0; }
      L[c + c * w] = sqrt(dgl);
    }
    __syncthreads();
    const double piv = L[c + c * w];
    for (int i = c + 1 + (int)threadIdx.x; i < w; i += blockDim.x) L[i + c * w] /= piv;
    __syncthreads();
    const int m = w - c - 1;  // trailing (i >= j > c): pairs over the lower triangle
    for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
      const int i = c + 1 + q / m, j = c + 1 + q % m;
      if (j <= i) L[i + j * w] -= L[i + c * w] * L[j + c * w];
    }
    __syncthreads();
  }
  // 4. rows below: L_{R,s} = P_R L_ss^-T (one row per thread)
  for (int a = threadIdx.x; a < r; a += blockDim.x) {
    for (int c = 0; c < w; ++c) {
      double v = Lc[c * r + a];
      for (int k = 0; k < c; ++k) v -= Lc[k * r + a] * L[c + k * w];
      Lc[c * r + a] = v / L[c + c * w];
    }
  }
  // 5. X = L_ss^-1 (one column per thread), stored row-major lower in Dinv
  for (int c = threadIdx.x; c < w; c += blockDim.x) {
    for (int i = 0; i < c; ++i) X[i + c * w] = 0.0;
    for (int i = c; i < w; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) v -= L[i + k * w] * X[k + c * w];
      X[i + c * w] = v / L[i + i * w];
    }
  }
  __syncthreads();
  double* Di = f.Dinv + f.sn_dofs[s];
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q / w, c = q % w;
    Di[q] = X[i + c * w];
  }
  if (threadIdx.x == 0 && s_bad) atomicExch(f.part_fail + part, 1);
}

}  // namespace dfem
