// Dense-inverse form of the global solve, for single scenes small enough that
// X = Hs^-1 (N x N, FP64) fits comfortably in HBM (and mostly in L2).  Each
// solve is then one matrix-vector product over three right-hand sides, a
// stream of N^2 doubles with no dependency chain, instead of the 2 x levels
// dependent steps of the supernodal triangular solves.
//
// X is rebuilt from the GPU supernodal factor after every refactorisation:
//   1. the factor L (its diagonal blocks L_ss, kept by k_factor_level, and the
//      panels L_{R,s}) scattered into a dense lower-triangular N_p x N_p matrix
//      (N_p = N rounded up to 64; the padding is the identity),
//   2. the inverses of its 64 x 64 diagonal tiles (all tiles at once),
//   3. W = L^-1 by doubling diagonal ranges, bottom up: with the inverses of
//      ranges A = [a, m) and C = [m, b) known, the block below them is
//      W_CA = -(W_CC L_CA) W_AA (two tile-products per level, every range of
//      the level in one launch; log2(tiles) levels),
//   4. X = W^T W (lower tiles, mirrored: X is exactly symmetric).
// Products of 64 x 64 tiles run on the FP64 tensor cores (mma.sync m8n8k4)
// from shared memory in a fixed order, so X and every solve are
// deterministic.  The solve's result agrees with the triangular solves'
// to rounding (the same factor, applied as one inverse).
#pragma once

// (included by engine.cu after pd_kernels.cu: warp_sum, Gate, SnInfo, FactorDev)
#include "factor_kernels.cuh"

namespace dfem {

constexpr int kDenseTile = 64;
constexpr int kDenseLd = kDenseTile + 1;  // padded shared-memory row (doubles)
constexpr size_t kDenseSmem = 2 * (size_t)kDenseTile * kDenseLd * sizeof(double);

struct DenseDev {
  int N, Np, nb;        // vertices, padded size, tiles per side
  double* A;            // N_p x N_p row-major: L, then X
  double* W;            // N_p x N_p row-major: L^-1 (lower tiles)
  double* T;            // N_p x N_p row-major: W_CC L_CA of the current level
  double* Linv;         // nb x 64 x 64 row-major: inverses of L's diagonal tiles
};

constexpr int kDenseThreads = 128;  // CTA of the tile products: four warps, a 32 x 32 quadrant each

// P (64 x 64, [row][k]) times Q^T (Q [col][k]) added to the warp's 4 x 4 8x8
// output tiles: warp w holds the quadrant rows 32 (w >> 1) .., columns
// 32 (w & 1) ..; d[i][j][e] is row qr + 8 i + (lane >> 2), column
// qc + 8 j + 2 (lane & 3) + e.  Per k-step of four: four A and four B
// fragments from shared memory feed sixteen FP64 tensor-core products.
__device__ __forceinline__ void dense_quadrant(int& qr, int& qc) {
  const int w = threadIdx.x >> 5;
  qr = 32 * (w >> 1);
  qc = 32 * (w & 1);
}

__device__ __forceinline__ void dense_mma(const double* P, const double* Q, double d[4][4][2]) {
  const int lane = threadIdx.x & 31;
  int qr, qc;
  dense_quadrant(qr, qc);
  const double* pa = P + (qr + (lane >> 2)) * kDenseLd + (lane & 3);
  const double* qb = Q + (qc + (lane >> 2)) * kDenseLd + (lane & 3);
#pragma unroll 2
  for (int k0 = 0; k0 < kDenseTile; k0 += 4) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = pa[8 * i * kDenseLd + k0];
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = qb[8 * j * kDenseLd + k0];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma_8x8x4(d[i][j][0], d[i][j][1], a[i], b[j]);
  }
}

// tile (I, J) of a row-major N_p x N_p matrix into shared memory, as stored or
// transposed: 16-byte loads along the rows of M, all of a thread's loads
// issued before its shared-memory stores
__device__ __forceinline__ void dense_load(const double* M, int Np, int I, int J, bool trans, double* S) {
  const double* src = M + (size_t)I * kDenseTile * Np + (size_t)J * kDenseTile;
  constexpr int kPairs = kDenseTile * kDenseTile / 2, kPer = kPairs / kDenseThreads;
  double2 v[kPer];
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int q = threadIdx.x + kDenseThreads * u, r = q / (kDenseTile / 2), c = 2 * (q % (kDenseTile / 2));
    v[u] = __ldcg(reinterpret_cast<const double2*>(src + (size_t)r * Np + c));
  }
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int q = threadIdx.x + kDenseThreads * u, r = q / (kDenseTile / 2), c = 2 * (q % (kDenseTile / 2));
    if (trans) {
      S[c * kDenseLd + r] = v[u].x;
      S[(c + 1) * kDenseLd + r] = v[u].y;
    } else {
      S[r * kDenseLd + c] = v[u].x;
      S[r * kDenseLd + c + 1] = v[u].y;
    }
  }
}

__device__ __forceinline__ void dense_zero(double d[4][4][2]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) d[i][j][0] = d[i][j][1] = 0.0;
}

// the warp's output tiles, scaled by sc, to tile (I, J) of M (transp: to (J, I)
// transposed as well; skip_upper: only the lower triangle of a diagonal tile)
__device__ __forceinline__ void dense_store(const double d[4][4][2], double sc, double* M, int Np, int I, int J,
                                            bool transp, bool skip_upper) {
  const int lane = threadIdx.x & 31;
  int qr, qc;
  dense_quadrant(qr, qc);
  double* o = M + (size_t)I * kDenseTile * Np + (size_t)J * kDenseTile;
  double* ot = M + (size_t)J * kDenseTile * Np + (size_t)I * kDenseTile;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = qr + 8 * i + (lane >> 2), c = qc + 8 * j + 2 * (lane & 3) + e;
        if (skip_upper && r < c) continue;
        const double v = sc * d[i][j][e];
        o[(size_t)r * Np + c] = v;
        if (transp) ot[(size_t)c * Np + r] = v;
      }
}

// 1. the supernodal factor into the dense lower triangle (A zeroed before):
// one CTA per supernode; the padding rows get a unit diagonal
__global__ void k_dense_scatter(DenseDev dd, FactorDev f, const double* __restrict__ Ldw,
                                const int* __restrict__ sn_dofs) {
  const int s = blockIdx.x;
  if (s == 0)
    for (int i = dd.N + threadIdx.x; i < dd.Np; i += blockDim.x) dd.A[(size_t)i * dd.Np + i] = 1.0;
  const SnInfo in = f.info[s];
  const int c0 = in.c0, w = in.w, r = in.r;
  const double* Ld = Ldw + sn_dofs[in.s];
  const double* Lc = f.Lcm + in.lofs;
  const int* R = f.rowidx + in.rofs;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q / w, c = q % w;
    if (i >= c) dd.A[(size_t)(c0 + i) * dd.Np + c0 + c] = Ld[i + c * w];
  }
  for (int q = threadIdx.x; q < r * w; q += blockDim.x) {  // consecutive threads: consecutive columns of a row
    const int a = q / w, c = q % w;
    dd.A[(size_t)R[a] * dd.Np + c0 + c] = Lc[(size_t)c * r + a];
  }
}

// 2. inverse of diagonal tile J of L (lower triangular; one column per
// thread, forward substitution), to Linv and as W_JJ
__global__ void __launch_bounds__(kDenseThreads) k_dense_tile_inv(DenseDev dd) {
  extern __shared__ __align__(16) double dsh[];
  double* S = dsh;
  double* X = dsh + kDenseTile * kDenseLd;
  const int J = blockIdx.x;
  dense_load(dd.A, dd.Np, J, J, false, S);
  __syncthreads();
  const int c = threadIdx.x;
  if (c < kDenseTile) {
    for (int i = 0; i < c; ++i) X[i * kDenseLd + c] = 0.0;
    for (int i = c; i < kDenseTile; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) v -= S[i * kDenseLd + k] * X[k * kDenseLd + c];
      X[i * kDenseLd + c] = v / S[i * kDenseLd + i];
    }
  }
  __syncthreads();
  double* Li = dd.Linv + (size_t)J * kDenseTile * kDenseTile;
  double* Wd = dd.W + (size_t)J * kDenseTile * dd.Np + (size_t)J * kDenseTile;
  for (int q = threadIdx.x; q < kDenseTile * kDenseTile; q += blockDim.x) {
    const int r = q / kDenseTile, cc = q % kDenseTile;
    const double v = X[r * kDenseLd + cc];
    Li[q] = v;
    Wd[(size_t)r * dd.Np + cc] = v;
  }
}

// 3. one level of the triangular inverse (ranges of s tiles; blockIdx.y the
// pair of ranges A = [a, m), C = [m, b) with a = 2 s y, m = a + s,
// b = min(a + 2 s, nb); blockIdx.x the tile (I, J) of C x A):
//   t: T_IJ = sum_{K=m..I} W_IK L_KJ       w: W_IJ = -sum_{K=J..m-1} T_IK W_KJ
__device__ __forceinline__ bool dense_level_tile(const DenseDev& dd, int s, int& I, int& J, int& a, int& m) {
  a = 2 * s * blockIdx.y;
  m = a + s;
  const int b = min(a + 2 * s, dd.nb);
  I = m + (int)blockIdx.x / s;
  J = a + (int)blockIdx.x % s;
  return m < dd.nb && I < b;
}

__global__ void __launch_bounds__(kDenseThreads) k_dense_trtri_t(DenseDev dd, int s) {
  extern __shared__ __align__(16) double dsh[];
  double* P = dsh;
  double* Q = dsh + kDenseTile * kDenseLd;
  int I, J, a, m;
  if (!dense_level_tile(dd, s, I, J, a, m)) return;
  double d[4][4][2];
  dense_zero(d);
  for (int K = m; K <= I; ++K) {
    dense_load(dd.W, dd.Np, I, K, false, P);  // W_IK [row][k]
    dense_load(dd.A, dd.Np, K, J, true, Q);   // L_KJ as [col][k]
    __syncthreads();
    dense_mma(P, Q, d);
    __syncthreads();
  }
  dense_store(d, 1.0, dd.T, dd.Np, I, J, false, false);
}

__global__ void __launch_bounds__(kDenseThreads) k_dense_trtri_w(DenseDev dd, int s) {
  extern __shared__ __align__(16) double dsh[];
  double* P = dsh;
  double* Q = dsh + kDenseTile * kDenseLd;
  int I, J, a, m;
  if (!dense_level_tile(dd, s, I, J, a, m)) return;
  double d[4][4][2];
  dense_zero(d);
  for (int K = J; K < m; ++K) {
    dense_load(dd.T, dd.Np, I, K, false, P);  // T_IK [row][k]
    dense_load(dd.W, dd.Np, K, J, true, Q);   // W_KJ as [col][k]
    __syncthreads();
    dense_mma(P, Q, d);
    __syncthreads();
  }
  dense_store(d, -1.0, dd.W, dd.Np, I, J, false, false);
}

// 4. X = W^T W: tile (I, J), I >= J, sum over K = I .. nb-1 of W_KI^T W_KJ;
// written to (I, J) and transposed to (J, I)
__global__ void __launch_bounds__(kDenseThreads) k_dense_lauum(DenseDev dd) {
  extern __shared__ __align__(16) double dsh[];
  double* P = dsh;
  double* Q = dsh + kDenseTile * kDenseLd;
  const int b = blockIdx.x;
  int I = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= b) ++I;
  while (I * (I + 1) / 2 > b) --I;
  const int J = b - I * (I + 1) / 2;
  double d[4][4][2];
  dense_zero(d);
  for (int K = I; K < dd.nb; ++K) {
    dense_load(dd.W, dd.Np, K, I, true, P);  // W_KI as [row i][k]
    dense_load(dd.W, dd.Np, K, J, true, Q);  // W_KJ as [col j][k]
    __syncthreads();
    dense_mma(P, Q, d);
    __syncthreads();
  }
  dense_store(d, 1.0, dd.A, dd.Np, I, J, true, I == J);  // a diagonal tile is defined by its lower triangle
}

// The solve: y_i = sum_j X_ij rhs_j (three components).  One CTA of 1024
// threads per SM stages rhs in shared memory (x, y, z planes, zero past N),
// then one warp per row (rows dealt round-robin over the CTAs) streams the row in 16-byte pairs, eight per lane in
// flight, each lane summing its columns in a fixed order, then the warp's
// fixed reduction tree.  X's padding columns are zero.  Shared memory: 3 N_p
// doubles.
constexpr int kDenseSolveThreads = 1024;
__global__ void __launch_bounds__(kDenseSolveThreads, 1) k_dense_solve(DenseDev dd, Gate gate,
                                                                      const double* __restrict__ rhs, double* y) {
  extern __shared__ __align__(16) double bsh[];
  if (gate.skip(0)) return;
  const int Np = dd.Np, N = dd.N;
  for (int j = threadIdx.x; j < Np; j += blockDim.x) {
    const bool in = j < N;
    bsh[j] = in ? rhs[3 * (size_t)j] : 0.0;
    bsh[Np + j] = in ? rhs[3 * (size_t)j + 1] : 0.0;
    bsh[2 * Np + j] = in ? rhs[3 * (size_t)j + 2] : 0.0;
  }
  __syncthreads();
  const double2* bx = reinterpret_cast<const double2*>(bsh);
  const double2* by = reinterpret_cast<const double2*>(bsh + Np);
  const double2* bz = reinterpret_cast<const double2*>(bsh + 2 * Np);
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5, np2 = Np / 2;
  for (int i = (threadIdx.x >> 5) * gridDim.x + blockIdx.x; i < N; i += gridDim.x * nw) {  // rows spread over all CTAs
    const double2* row = reinterpret_cast<const double2*>(dd.A + (size_t)i * Np);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int q0 = lane; q0 < np2; q0 += 256) {
      double2 x[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = q0 + 32 * u;
        x[u] = k < np2 ? __ldcg(row + k) : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = q0 + 32 * u;
        if (k < np2) {
          const double2 b0 = bx[k], b1 = by[k], b2 = bz[k];
          a0 += x[u].x * b0.x + x[u].y * b0.y;
          a1 += x[u].x * b1.x + x[u].y * b1.y;
          a2 += x[u].x * b2.x + x[u].y * b2.y;
        }
      }
    }
    a0 = warp_sum(a0); a1 = warp_sum(a1); a2 = warp_sum(a2);
    if (lane == 0) { y[3 * (size_t)i] = a0; y[3 * (size_t)i + 1] = a1; y[3 * (size_t)i + 2] = a2; }
  }
}

}  // namespace dfem
