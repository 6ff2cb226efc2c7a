// resident_solve.cuh — the global solve with the whole factor resident in the
// distributed shared memory of one thread-block cluster.
//
// A small factor (a single scene of up to a few MB of blocks) is split over
// the C CTAs of one cluster (C = 16 where the device allows it): every
// supernode has an owner CTA that holds its diagonal-block inverse and its
// below-diagonal block in shared memory for the whole launch, loaded at the
// start by one bulk copy per CTA from a per-CTA image in global memory.  The
// sweeps walk the levels of the elimination tree with a cluster barrier
// between levels; the forward sweep pushes a supernode's contributions
// L_{R,s} y_s straight into the shared-memory inbox of the supernode owning
// each destination row (st.shared::cluster), the backward sweep pulls the
// ancestors' solution values x_R from their owners' shared memory
// (ld.shared::cluster).  A chain step is a hardware cluster barrier plus the
// supernode's dense work in shared memory, instead of a completion stamp
// polled through L2 and the re-staging of the blocks.
//
// Every sum runs in the order of fwd_supernode / bwd_supernode (pd_kernels.cu):
// contributions per row in their grouped order, diagonal-block products one
// thread per row in increasing k, panel products one thread per row in
// increasing column (forward) or per column lanes over rows and a warp sum
// (backward).  The results are bit-identical to the other solve forms.
#pragma once
// included after pd_kernels.cu (warp_sum, cluster_rank, cluster_sync_all)
#include "kernels.cuh"
#include "resident_plan.h"

namespace dfem {

// Every CTA's metadata lives in its image (resident_plan.h): a header (item
// count, the first item of each level, prefix sums for the flat loops), the
// item records (ResItem) and per item the address tables of its pushes and
// pulls (32-bit words rank << 24 | offset).  No step of the sweeps waits on
// a global-memory load; the header and items arrive by a small first bulk
// copy, so the right-hand side is fetched while the blocks are in flight.
struct ResDev {
  const double* img;        // every CTA's image, back to back
  const long long* img_ofs; // C + 1 offsets into img (doubles, even)
  const int* head_len;      // per CTA: doubles of the header + items part of its image
  int nlev;                 // levels (every CTA takes 2 nlev + 1 cluster barriers)
  int smem_doubles;         // dynamic shared memory of every CTA (doubles)
  int* status;              // error status word (as FactorDev::status)
};

__device__ __forceinline__ uint32_t cluster_map(const void* p, unsigned rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_addr(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster_f64(uint32_t addr, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
__device__ __forceinline__ double ld_cluster_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
  return v;
}

__device__ __forceinline__ void res_fail(const ResDev& d, int s, int which) {
  d.status[0] = 6;
  d.status[1] = s;
  d.status[2] = which;
  atomicAdd(d.status + 3, 1);
}

// A packed address (rank << 24 | offset) checked against the cluster and the
// shared memory; false (and the error recorded) when out of range.
__device__ __forceinline__ bool res_addr_ok(const ResDev& d, uint32_t v, int s, int which) {
  if ((v >> 24) < gridDim.x && (int)(v & 0xFFFFFFu) + 3 <= d.smem_doubles) return true;
  res_fail(d, s, which);
  return false;
}

// Forward solve of one supernode (order of fwd_supernode).
__device__ __forceinline__ void res_forward(const ResDev& d, const ResItem& in, double* sh, double* t) {
  const int w = in.w, r = in.r, tid = threadIdx.x, nt = blockDim.x;
  const double* D = sh + in.dofs;
  const double* L = sh + in.lofs;
  const int* prow = reinterpret_cast<const int*>(sh + in.pofs);
  const uint32_t* push = reinterpret_cast<const uint32_t*>(sh + in.tofs);
  const double* q = sh + in.qofs;
  double* ysh = sh + in.yofs;  // holds rhs_s on entry
  for (int c = tid; c < w; c += nt) {
    double a0 = ysh[3 * c], a1 = ysh[3 * c + 1], a2 = ysh[3 * c + 2];
    for (int k = prow[c]; k < prow[c + 1]; ++k) { a0 -= q[3 * k]; a1 -= q[3 * k + 1]; a2 -= q[3 * k + 2]; }
    t[3 * c] = a0; t[3 * c + 1] = a1; t[3 * c + 2] = a2;
  }
  __syncthreads();
  for (int c = tid; c < w; c += nt) {
    double a0 = 0, a1 = 0, a2 = 0;
    const double* Dc = D + (size_t)c * (c + 1) / 2;
#pragma unroll 4
    for (int k = 0; k <= c; ++k) {
      const double dv = Dc[k];
      a0 += dv * t[3 * k]; a1 += dv * t[3 * k + 1]; a2 += dv * t[3 * k + 2];
    }
    ysh[3 * c] = a0; ysh[3 * c + 1] = a1; ysh[3 * c + 2] = a2;
  }
  __syncthreads();
  for (int a = tid; a < r; a += nt) {
    double a0 = 0, a1 = 0, a2 = 0;
    int c = 0;
    for (; c + 16 <= w; c += 16) {  // sixteen loads in flight, then the sums in column order
      double l[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) l[j] = L[(size_t)(c + j) * r + a];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const double* yc = ysh + 3 * (c + j);
        a0 += l[j] * yc[0]; a1 += l[j] * yc[1]; a2 += l[j] * yc[2];
      }
    }
    for (; c < w; ++c) {
      const double l = L[(size_t)c * r + a];
      a0 += l * ysh[3 * c]; a1 += l * ysh[3 * c + 1]; a2 += l * ysh[3 * c + 2];
    }
    const uint32_t dst = push[a];
    if (!res_addr_ok(d, dst, in.s, 8)) continue;
    const uint32_t o = cluster_map(sh + (dst & 0xFFFFFFu), dst >> 24);
    st_cluster_f64(o, a0); st_cluster_f64(o + 8, a1); st_cluster_f64(o + 16, a2);
  }
  __syncthreads();  // t is reused by the next item
}

// Backward solve of one supernode (order of bwd_supernode).
__device__ __forceinline__ void res_backward(const ResDev& d, const ResItem& in, double* sh, double* t, double* xr) {
  const int w = in.w, r = in.r, tid = threadIdx.x, nt = blockDim.x;
  const double* D = sh + in.dofs;
  const double* L = sh + in.lofs;
  const uint32_t* pull = reinterpret_cast<const uint32_t*>(sh + in.tofs) + r;
  double* ysh = sh + in.yofs;  // holds y_s of the forward sweep on entry
  for (int a = tid; a < r; a += nt) {
    const uint32_t src = pull[a];
    if (!res_addr_ok(d, src, in.s, 9)) {
      xr[3 * a] = xr[3 * a + 1] = xr[3 * a + 2] = 0.0;
      continue;
    }
    const uint32_t o = cluster_map(sh + (src & 0xFFFFFFu), src >> 24);
    xr[3 * a] = ld_cluster_f64(o); xr[3 * a + 1] = ld_cluster_f64(o + 8); xr[3 * a + 2] = ld_cluster_f64(o + 16);
  }
  for (int k = tid; k < 3 * w; k += nt) t[k] = ysh[k];
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  for (int c = warp; c < w; c += nw) {
    double a0 = 0, a1 = 0, a2 = 0;
    const double* Lc = L + (size_t)c * r;
    for (int a = lane; a < r; a += 32) {
      const double l = Lc[a];
      a0 += l * xr[3 * a]; a1 += l * xr[3 * a + 1]; a2 += l * xr[3 * a + 2];
    }
    a0 = warp_sum(a0); a1 = warp_sum(a1); a2 = warp_sum(a2);
    if (lane == 0) { t[3 * c] -= a0; t[3 * c + 1] -= a1; t[3 * c + 2] -= a2; }
  }
  __syncthreads();
  for (int c = tid; c < w; c += nt) {
    double a0 = 0, a1 = 0, a2 = 0;
#pragma unroll 4
    for (int k = c; k < w; ++k) {
      const double dv = D[(size_t)k * (k + 1) / 2 + c];
      a0 += dv * t[3 * k]; a1 += dv * t[3 * k + 1]; a2 += dv * t[3 * k + 2];
    }
    ysh[3 * c] = a0; ysh[3 * c + 1] = a1; ysh[3 * c + 2] = a2;
  }
  __syncthreads();
}

// Small supernodes (w <= 32 columns, r <= 64 rows below) run one per warp,
// with the column values in registers (lane c holds column c, lanes hold rows
// lane and lane + 32) and shuffles instead of shared scratch and block
// barriers; every sum keeps the order of res_forward / res_backward (the
// products in increasing k or column, the backward's lane sums over rows a =
// lane, lane + 32 and the same butterfly), so the results are bit-identical.
__device__ __forceinline__ bool res_warp_item(const ResItem& in) { return in.w <= 32 && in.r <= 64; }
constexpr int kResWarpMin = 8;  // small items of a CTA at one level from which they run one per warp

__device__ __forceinline__ void res_forward_warp(const ResDev& d, const ResItem& in, double* sh) {
  const int w = in.w, r = in.r, lane = threadIdx.x & 31;
  const double* D = sh + in.dofs;
  const double* L = sh + in.lofs;
  const int* prow = reinterpret_cast<const int*>(sh + in.pofs);
  const uint32_t* push = reinterpret_cast<const uint32_t*>(sh + in.tofs);
  const double* q = sh + in.qofs;
  double* ysh = sh + in.yofs;
  double t0 = 0, t1 = 0, t2 = 0;
  if (lane < w) {
    t0 = ysh[3 * lane]; t1 = ysh[3 * lane + 1]; t2 = ysh[3 * lane + 2];
    for (int k = prow[lane]; k < prow[lane + 1]; ++k) { t0 -= q[3 * k]; t1 -= q[3 * k + 1]; t2 -= q[3 * k + 2]; }
  }
  double y0 = 0, y1 = 0, y2 = 0;
  const double* Dc = D + (size_t)lane * (lane + 1) / 2;
  for (int k = 0; k < w; ++k) {
    const double s0 = __shfl_sync(0xffffffffu, t0, k), s1 = __shfl_sync(0xffffffffu, t1, k),
                 s2 = __shfl_sync(0xffffffffu, t2, k);
    if (lane < w && k <= lane) {
      const double dv = Dc[k];
      y0 += dv * s0; y1 += dv * s1; y2 += dv * s2;
    }
  }
  if (lane < w) { ysh[3 * lane] = y0; ysh[3 * lane + 1] = y1; ysh[3 * lane + 2] = y2; }
  for (int a0r = 0; a0r < r; a0r += 32) {  // warp-uniform
    const int a = a0r + lane;
    double b0 = 0, b1 = 0, b2 = 0;
    for (int c = 0; c < w; ++c) {
      const double u0 = __shfl_sync(0xffffffffu, y0, c), u1 = __shfl_sync(0xffffffffu, y1, c),
                   u2 = __shfl_sync(0xffffffffu, y2, c);
      if (a < r) {
        const double l = L[(size_t)c * r + a];
        b0 += l * u0; b1 += l * u1; b2 += l * u2;
      }
    }
    if (a < r) {
      const uint32_t dst = push[a];
      if (res_addr_ok(d, dst, in.s, 8)) {
        const uint32_t o = cluster_map(sh + (dst & 0xFFFFFFu), dst >> 24);
        st_cluster_f64(o, b0); st_cluster_f64(o + 8, b1); st_cluster_f64(o + 16, b2);
      }
    }
  }
  __syncwarp();
}

__device__ __forceinline__ void res_backward_warp(const ResDev& d, const ResItem& in, double* sh) {
  const int w = in.w, r = in.r, lane = threadIdx.x & 31;
  const double* D = sh + in.dofs;
  const double* L = sh + in.lofs;
  const uint32_t* pull = reinterpret_cast<const uint32_t*>(sh + in.tofs) + r;
  double* ysh = sh + in.yofs;
  double xa[2][3] = {{0, 0, 0}, {0, 0, 0}};  // rows lane, lane + 32
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const int a = lane + 32 * m;
    if (a < r) {
      const uint32_t src = pull[a];
      if (res_addr_ok(d, src, in.s, 9)) {
        const uint32_t o = cluster_map(sh + (src & 0xFFFFFFu), src >> 24);
        xa[m][0] = ld_cluster_f64(o); xa[m][1] = ld_cluster_f64(o + 8); xa[m][2] = ld_cluster_f64(o + 16);
      }
    }
  }
  double t0 = 0, t1 = 0, t2 = 0;
  if (lane < w) { t0 = ysh[3 * lane]; t1 = ysh[3 * lane + 1]; t2 = ysh[3 * lane + 2]; }
  for (int c = 0; c < w; ++c) {
    const double* Lc = L + (size_t)c * r;
    double a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int a = lane + 32 * m;
      if (a < r) {
        const double l = Lc[a];
        a0 += l * xa[m][0]; a1 += l * xa[m][1]; a2 += l * xa[m][2];
      }
    }
    a0 = warp_sum(a0); a1 = warp_sum(a1); a2 = warp_sum(a2);
    if (lane == c) { t0 -= a0; t1 -= a1; t2 -= a2; }
  }
  double y0 = 0, y1 = 0, y2 = 0;
  for (int k = 0; k < w; ++k) {
    const double s0 = __shfl_sync(0xffffffffu, t0, k), s1 = __shfl_sync(0xffffffffu, t1, k),
                 s2 = __shfl_sync(0xffffffffu, t2, k);
    if (lane < w && k >= lane) {
      const double dv = D[(size_t)k * (k + 1) / 2 + lane];
      y0 += dv * s0; y1 += dv * s1; y2 += dv * s2;
    }
  }
  if (lane < w) { ysh[3 * lane] = y0; ysh[3 * lane + 1] = y1; ysh[3 * lane + 2] = y2; }
  __syncwarp();
}

// Element j of the CTA's solution regions (j < 3 sum(w)): its item and the
// offset in it, from the prefix sums cum[] (few items per CTA: linear scan).
__device__ __forceinline__ int res_item_of(const int* cum, int n, int j) {
  int i = 0;
  while (i + 1 < n && cum[i + 1] <= j) ++i;
  return i;
}

// Both sweeps in one launch of one cluster (grid = cluster = C CTAs).  Every
// CTA takes every cluster barrier (2 nlev + 1 of them), whatever happens to
// its own work, so the barriers always complete; a bounded wait that gives up
// records status 6 and the CTA skips its arithmetic (the solve's result is
// then invalid, and the caller reports DFEM_ERR_CAP).
__global__ void __launch_bounds__(512, 1) k_solve_resident(ResDev d, Gate gate, const double* __restrict__ rhs,
                                                           double* y) {
  extern __shared__ __align__(16) double sh[];
  __shared__ __align__(8) uint64_t bar[2];
  if (gate.skip(0)) return;  // uniform over the cluster: before any barrier
  const unsigned rank = cluster_rank();
  const long long i0 = d.img_ofs[rank], i1 = d.img_ofs[rank + 1];
  const int hl = d.head_len[rank];
  const unsigned bh = (unsigned)(hl * sizeof(double)), bb = (unsigned)((i1 - i0 - hl) * sizeof(double));
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_expect_tx(&bar[0], bh);
    bulk_copy_g2s(sh, d.img + i0, bh, &bar[0]);
    if (bb > 0) {
      mbar_expect_tx(&bar[1], bb);
      bulk_copy_g2s(sh + hl, d.img + i0 + hl, bb, &bar[1]);
    }
  }
  __syncthreads();  // the barriers are initialised before anyone waits on them
  const bool okh = __syncthreads_and(mbar_wait_bounded(&bar[0], 0)) != 0;
  const int* hdr = reinterpret_cast<const int*>(sh);
  const int n = okh ? hdr[0] : 0;
  const ResItem* items = reinterpret_cast<const ResItem*>(sh + (okh ? hdr[5] : 0));
  const int* sched = hdr + kResHeadInts;
  const int* cum = sched + d.nlev + 1;
  const int ncols3 = okh ? hdr[2] : 0;
  // the right-hand side of the owned columns into their solution regions
  for (int j = threadIdx.x; j < ncols3; j += blockDim.x) {
    const int i = res_item_of(cum, n, j);
    const int k = j - cum[i];
    sh[items[i].yofs + k] = rhs[3 * (size_t)items[i].c0 + k];
  }
  cluster_sync_all();  // every CTA of the cluster runs: its shared memory may be written
  const bool okb = __syncthreads_and(bb == 0 || mbar_wait_bounded(&bar[1], 0)) != 0;
  const bool ok = okh && okb;
  if (!ok && threadIdx.x == 0) res_fail(d, -1, 7);
  double* t = sh + (ok ? hdr[3] : 0);
  double* xr = sh + (ok ? hdr[4] : 0);
  // a level's supernodes are independent: when the CTA holds at least
  // kResWarpMin small ones at a level they run one per warp, side by side
  // (then the large ones by the whole CTA); with fewer, every item runs on
  // the whole CTA, whose shorter per-item latency then sets the level's pace
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int l = 0; l < d.nlev; ++l) {
    if (ok) {
      int ne = 0;
      for (int it = sched[l]; it < sched[l + 1]; ++it) ne += res_warp_item(items[it]) ? 1 : 0;
      const bool by_warp = ne >= kResWarpMin;
      if (by_warp) {
        for (int it = sched[l], e = 0; it < sched[l + 1]; ++it)
          if (res_warp_item(items[it]) && (e++ % nw) == warp) res_forward_warp(d, items[it], sh);
        __syncthreads();
      }
      for (int it = sched[l]; it < sched[l + 1]; ++it)
        if (!by_warp || !res_warp_item(items[it])) res_forward(d, items[it], sh, t);
    }
    cluster_sync_all();  // the level's contributions have landed in their owners' inboxes
  }
  for (int l = d.nlev - 1; l >= 0; --l) {
    if (ok) {
      int ne = 0;
      for (int it = sched[l]; it < sched[l + 1]; ++it) ne += res_warp_item(items[it]) ? 1 : 0;
      const bool by_warp = ne >= kResWarpMin;
      if (by_warp) {
        for (int it = sched[l], e = 0; it < sched[l + 1]; ++it)
          if (res_warp_item(items[it]) && (e++ % nw) == warp) res_backward_warp(d, items[it], sh);
        __syncthreads();
      }
      for (int it = sched[l]; it < sched[l + 1]; ++it)
        if (!by_warp || !res_warp_item(items[it])) res_backward(d, items[it], sh, t, xr);
    }
    cluster_sync_all();  // the level's solution values are final; no CTA reads another's after the last one
  }
  if (ok) {
    for (int j = threadIdx.x; j < ncols3; j += blockDim.x) {
      const int i = res_item_of(cum, n, j);
      const int k = j - cum[i];
      y[3 * (size_t)items[i].c0 + k] = sh[items[i].yofs + k];
    }
  } else if (threadIdx.x == 0) {  // give the copies one more bounded chance to land before the CTA exits
    mbar_wait_bounded(&bar[0], 0);
    if (bb > 0) mbar_wait_bounded(&bar[1], 0);
  }
}

// Copy of the factor's blocks (device arrays of the refactorisation) into the
// resident images: one CTA per supernode, after every refactorisation.
struct ResPack {
  int w, r;
  int src_d, src_l;      // Dinv (row-major w x w) and Lcm (column-major r x w) offsets in the factor arrays
  long long dst_d, dst_l; // offsets in the image array
};

__global__ void k_res_pack(const ResPack* __restrict__ pk, const double* __restrict__ Dinv, const double* __restrict__ Lcm,
                           double* img) {
  const ResPack p = pk[blockIdx.x];
  for (int k = threadIdx.x; k < p.w * p.w; k += blockDim.x) {  // the lower triangle, packed by rows
    const int i = k / p.w, j = k - i * p.w;
    if (j <= i) img[p.dst_d + (size_t)i * (i + 1) / 2 + j] = Dinv[p.src_d + k];
  }
  for (int k = threadIdx.x; k < p.r * p.w; k += blockDim.x) img[p.dst_l + k] = Lcm[p.src_l + k];
}

}  // namespace dfem
