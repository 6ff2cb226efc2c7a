// engine.cu — host driver of the PD engine and the C ABI of include/dfem.h.
//
// A scene owns one CUDA stream, its device arrays, and two CUDA graphs built
// on first use: the forward time step and the adjoint of one time step.  The
// step index lives in device memory, so one graph serves every step.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/dfem.h"
#include "pd_kernels.cu"
#include "contact_kernels.cuh"
#include "factor_kernels.cuh"
#include "drag_kernels.cuh"
#include "resident_solve.cuh"
#include "skeleton_kernels.cuh"
#include "skeleton_adjoint.cuh"
#include "dense_solve.cuh"
#include "resident_plan.h"
#include "scene.h"

namespace dfem {

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

// error reporting for entry points defined in other translation units
int report_error(int code, const std::string& msg) { return fail(code, msg); }

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? DFEM_ERR_NOMEM : DFEM_ERR_CUDA,         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

// Allocation-failure injection of dfem_debug_fail_allocations: the calling
// thread's device allocations fail once this many more have succeeded (-1: off).
static thread_local long long g_alloc_budget = -1;

#define RC(x) do { int rc_ = (x); if (rc_) return rc_; } while (0)

// A kernel's dynamic shared-memory limit (cudaFuncAttributeMaxDynamicSharedMemorySize)
// is a property of the kernel in the process, per device, not of a scene: it
// only ever grows here, so creating a scene that needs less never lowers the
// limit that an earlier, larger scene's launches rely on.
static cudaError_t raise_smem_limit(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> limit;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  bytes = std::max<size_t>(1, bytes);
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limit[{fn, dev}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

struct LoopGraph {
  cudaGraphExec_t exec = nullptr;
  size_t outside = 0;  // kernels outside the loops
  size_t body = 0;     // kernels per iteration of the first loop (its solve in the tuned form)
  size_t body2 = 0;    // kernels per iteration of the second loop (contact phase), if any
  size_t alt_less = 0; // kernels fewer in an iteration whose solve took the persistent form
};

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t count) {
    if (p) { cudaFree(p); p = nullptr; }
    n = count;
    if (count == 0) return cudaSuccess;
    if (g_alloc_budget == 0) { n = 0; return cudaErrorMemoryAllocation; }
    if (g_alloc_budget > 0) --g_alloc_budget;
    return cudaMalloc(&p, count * sizeof(T));
  }
  // copies into the existing allocation when the size is unchanged, so device
  // pointers captured in CUDA graphs stay valid across material updates
  cudaError_t upload(const std::vector<T>& h) {
    if (!(p && n == h.size())) {
      cudaError_t e = alloc(h.size());
      if (e != cudaSuccess || h.empty()) return e;
    }
    if (h.empty()) return cudaSuccess;
    return cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
  }
  void swap(DBuf& o) { std::swap(p, o.p); std::swap(n, o.n); }
};

}  // namespace dfem

using namespace dfem;

struct dfem_scene {
  HostScene hs;
  int device = 0;
  cudaStream_t stream = nullptr;
  // constraint tables
  DBuf<double> mass, gmask, tinv, twr, twv, tvol, tE, tnu, minv, mw, mfib, srest, ssw, bbeta, bw, brest, attach_jd;
  DBuf<int4> tv, tslot, mv, mslot;
  DBuf<int2> sv, sslot;
  DBuf<int> sch;
  DBuf<int> mseg, seg_ptr, seg_mus, boff, bv, bslot, vslot_ptr, hs_ptr, hs_col, to_user, to_internal;
  DBuf<double> hs_val;
  DBuf<double> attach_k;             // per-vertex attachment stiffness (mixed form's rhs)
  // underwater drag: faces, every vertex's face corners, per-face forces and their adjoint
  int nF = 0;
  DBuf<int> df, vf_ptr, vf_face;
  DBuf<double> fdrag, fdrag_b;
  // factor
  DBuf<int> rseg_ptr, cdst, sn_c0, sn_w, sn_r, sn_rofs, rowidx, sn_lofs, sn_dofs, lvl_sn;
  DBuf<double> contrib, Lcm, Dinv, DinvC;
  DBuf<SnInfo> sn_info;
  std::vector<int> lvl_ptr;
  // Launch segments of the level-kernel solve: every level of the elimination
  // tree, split into its small supernodes (one warp each, eight per CTA) and
  // the rest (one CTA each, autotuned CTA size); each launch gets the shared
  // memory of its largest member.
  struct LevelSeg {
    int begin, count, level;
    int warp;              // 1: one supernode per warp
    int grp_f, grp_b;      // doubles of shared memory per group (warp segments)
    size_t shm_f, shm_b;   // bytes per CTA
    int thr_f, thr_b;
  };
  std::vector<LevelSeg> segs;
  // persistent solve (one launch per solve) and the autotuned choice between it and the level kernels
  DBuf<int> sn_parent, sn_pos, kid_ptr, kid, done_f, done_b, solve_ctl;
  size_t shm_pers = 0;
  int pers_slots = 1;                    // CTAs of the persistent solve resident at once
  // The solve runs levels 0 .. solve_cut-1 as level kernels and the rest in
  // one persistent launch: solve_cut = number of levels is the level-kernel
  // form, 0 the persistent form, anything between the split form.
  // solve_cut = -1: the cluster form (one thread-block cluster walks the levels)
  int solve_cut = 0;
  int split_cut = 0;                     // the autotune's best split (0: none)
  double solve_ms[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // autotune timings (ms per solve): levels, persistent,
                                                          // best split, cluster, resident, dense
  // dense-inverse form (solve_cut = -3): X = Hs^-1 rebuilt after every refactorisation
  bool dense_ok = false;                 // the scene qualifies (single part, N <= kDenseMaxN)
  bool dense_built = false;
  double dense_build_ms = 0.0;
  DBuf<double> dn_A, dn_W, dn_T, dn_Linv;
  DenseDev dd{};
  int dense_grid = 1;                    // CTAs of the dense solve (one per SM at most)
  DBuf<int> lvl_ptr_d, lvl_warp_d;       // cluster form: level starts, end of each level's warp-sized supernodes
  size_t shm_cluster = 0;
  int shm_cluster_warp = 0;              // doubles of shared memory per warp item
  bool cluster_ok = false;
  cudaError_t cluster_launch_err = cudaSuccess;  // the last refused cluster launch (read and cleared by its checks)
  // resident form (solve_cut = -2): the factor in the distributed shared memory of one cluster
  bool res_ok = false;
  int res_ctas = 0;
  size_t shm_res = 0;
  DBuf<int> res_head;
  DBuf<double> res_img;
  DBuf<long long> res_img_ofs;
  DBuf<ResPack> res_pack;
  ResDev rdv{};
  double select_ms[2] = {0.0, 0.0};      // batches, only the largest part active: tuned form, persistent form
  // numeric refactorisation on the GPU (material changes)
  DBuf<double> hs_base, hc_coef, Ldw, part_reg, E_in, nu_in;
  DBuf<int> hc_ptr, hc_tet, up_ptr, up_d, up_a0, up_a1, part_fail;
  std::vector<double> part_reg_h;
  size_t shm_fact = 0;
  std::vector<size_t> shm_fact_lvl;      // dynamic shared memory of the refactorisation, per level
  std::vector<int> fact_shares;          // per level: CTAs per supernode of the split form (0: one launch)
  std::vector<int> fact_w;               // per level: widest supernode
  RefactorDev rd{};
  // batch layout (a single scene is one part)
  std::vector<HostScene> parts;          // the parts of a batch (empty for a single scene)
  DBuf<int> vpart, seg_part, sn_part, part_v0, part_b0, blk_part, blk_v0;
  int nblk_p = 1;                        // part-aligned blocks of the reducing vertex kernels
  PartDev pd{};
  // state
  DBuf<double> xt, vt, qn, c0, xk, rhs, y, slot, hist, io_a, io_b;
  DBuf<double> partial, errv;
  DBuf<unsigned> counter;
  DBuf<int> flag, iters, step, status, write_traj, zero;
  DBuf<double> act_all, act_cur;   // per-step activations; current activations
  DBuf<double> ckpt_x, ckpt_v, traj;
  DBuf<double> seg_x, seg_v;           // checkpoint_every > 1: the start states of one segment, regenerated by the adjoint
  int cap_steps = 0;
  // iterates of the last forward call: of every step when they fit the budget
  // (the adjoint then replays no step without contact), else of one step
  // (every step is recomputed from its checkpoint)
  long long hist_step = 0;
  size_t adj_budget = 0;  // set at creation: 45 % of the device memory, at most 60 % of the free memory
  // articulated skeleton (links whose vertices move rigidly)
  bool skel_on = false;
  int sk_nq = 0;                         // joint-state length 12 + L - 1
  DBuf<SkelLink> sk_link;
  DBuf<SkelState> sk_st;
  DBuf<int> sk_rv, sk_rlink, sk_ridx, sk_perm;
  DBuf<double> sk_rest, sk_cinv, sk_zcm, sk_jq, sk_jqd, sk_v0, sk_w, sk_rr, sk_q, sk_tv, sk_kt, sk_sm, sk_rhs, sk_sol;
  // the adjoint's history (per step and iteration) and work buffers
  DBuf<double> sk_hist, sk_jin, sk_thb, sk_sb, sk_gjq, sk_gjqd, sk_mu2, sk_mu3, sk_dlt, sk_jfin;
  std::vector<double> sk_gout;           // cotangents of the next backward's output (jq, jqd); empty: zero
  SkelDev skd{};
  // adjoint
  DBuf<double> xkb, xtb, bb, gE, gnu, mg, gact;
  // obstacle contact phase
  bool has_contact = false;
  DBuf<int> cverts, cidx, obs_f, imp_cnt, imp_face, cstate, cpasses;
  DBuf<int> bp_ptr, bp_face;             // broad phase of the obstacle detection
  // the obstacle contact phase as one cooperative launch (k_contact_fused) or
  // as the conditional loop of kernels
  bool fused_ok = false;                 // scene has obstacle contact only and the device runs the launch
  bool fused_on = true;                  // dfem_set_option(DFEM_OPTION_FUSED_CONTACT)
  bool split_factor = true;              // dfem_set_option(DFEM_OPTION_SPLIT_FACTOR)
  int gather_form = 0;                   // dfem_set_option(DFEM_OPTION_GATHER): 0 by size, 1 warp, 2 thread
  int fused_grid = 0;                    // CTAs of k_contact_fused (all resident)
  int cadj_grid = 0;                     // CTAs of k_cadj_fused (all resident)
  DBuf<double> fpartial;
  DBuf<double> obs_x, hdiag, imp_n, xn1, xold, cprev, lxt, vwc;
  // soft-soft contact (forward only: the adjoint refuses these scenes)
  bool self_contact = false;
  DBuf<int> s_cfaces, s_cvf_ptr, s_cvf_face, s_on_face, s_simp_cnt, s_simp_face, s_cf_face, s_cf_slot, s_m_slot,
      s_g_cnt, s_g_fill, s_g_ptr, s_g_mem, s_chit;
  DBuf<double> s_simp_td, s_simp_n, s_g_n, s_g_outF, s_g_outM, s_sc_cur, s_rhs_pre, s_cnext;
  DBuf<int> crec_si;                      // soft-contact records (per computed iteration)
  DBuf<double> crec_sd;
  DBuf<double> ca_scb, ca_ptot, ca_sbp, ca_gPF, ca_gPM, ca_gmF, ca_gmM, ca_xout;  // its adjoint
  // adjoint of the contact phase: the record of one step's Jacobi iterations and the reverse sweep's buffers
  DBuf<int> crec_on, crec_first, crec_cnt;
  // batched contact: contact vertices' parts, parts' obstacle faces, per-part phase state
  int cnp = 0;                           // parts of a batch with contact (0: single scene)
  DBuf<int> c_cpart, c_pf0, c_pst, c_pany, c_psrc;
  DBuf<unsigned long long> c_pe;
  DBuf<double> crec_x, crec_prev, crec_n, ca_xn1b, ca_pb, ca_hdb, ca_cxtb, ca_vwcb, ca_yb, ca_orib;
  int crec_cap = 0;
  // forward recording of every step's contact iterations (when the steps'
  // iterates are stored too, the adjoint then replays no contact step)
  DBuf<int> crec_base, crec_meta;
  std::vector<int> crec_meta_h;          // per step of the last forward: [first record, iterations, source, recorded]
  bool crec_fwd = false;                 // the last forward recorded
  int crec_used = 0;                     // records the last forward's steps occupy
  int crec_target = 0;                   // records the next forward asks for
  int crec_reserve = 0;                  // records kept free for the adjoint's replay of one step
  ContactDev cd{};
  std::vector<int> rec_passes;
  // graphs
  LoopGraph g_step, g_adj;
  cudaStream_t stream2 = nullptr;         // capture stream of the loop bodies
  cudaStream_t stream3 = nullptr;         // capture stream of the solve-form branches inside a body
  // Batches: per-iteration choice of the solve form (persistent once the
  // weight of the parts still iterating drops below select_w).
  bool solve_select = false;
  double select_w = 0.0;
  DBuf<double> part_w;                    // per part: its share of the factor's entries
  DBuf<unsigned long long> sel_count;     // [forward, adjoint]: iterations that took the persistent form
  size_t cur_alt_less = 0;                // capture bookkeeping of the body being built
  cudaError_t cur_capture_err = cudaSuccess;
  unsigned long long sel_seen[2] = {0, 0}; // sel_count as last read
  DBuf<int> kiter;                        // device-side iteration counter of the loops
  int64_t launches = 0;                   // kernels launched by this scene (graph nodes included)
  int rec_steps = 0;
  std::vector<int> rec_iters;  // per step: largest iteration count over the parts (recorded forward call)
  int nblk_v = 1;   // blocks of the vertex-parallel kernels
  SceneDev sd{};
  FactorDev fd{};
  int spin_tries = kSpinTries;            // polls of a persistent-solve dependency wait (dfem_set_limit)
  ~dfem_scene() {
    if (g_step.exec) cudaGraphExecDestroy(g_step.exec);
    if (g_adj.exec) cudaGraphExecDestroy(g_adj.exec);
    if (stream) cudaStreamDestroy(stream);
    if (stream2) cudaStreamDestroy(stream2);
    if (stream3) cudaStreamDestroy(stream3);
  }
};

namespace dfem {

// Run f(0) .. f(n-1) on up to hardware_concurrency host threads.
template <typename Fn>
static void parallel_for(int n, Fn f) {
  const int nt = std::max(1, std::min(n, (int)std::thread::hardware_concurrency()));
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&] {
      for (int i = next++; i < n; i = next++) f(i);
    });
  for (auto& th : pool) th.join();
}

// Captured graphs bake in device pointers; any change of them invalidates the graphs.
static void invalidate_graphs(dfem_scene* sc) {
  if (sc->g_step.exec) { cudaGraphExecDestroy(sc->g_step.exec); sc->g_step.exec = nullptr; }
  if (sc->g_adj.exec) { cudaGraphExecDestroy(sc->g_adj.exec); sc->g_adj.exec = nullptr; }
}

static void refresh_scene_view(dfem_scene* sc) {
  const HostScene& s = sc->hs;
  SceneDev sd{s.N, s.T, s.M, s.S, s.B, s.nseg, s.h, s.damping, s.g[0], s.g[1], s.g[2],
              sc->mass.p, sc->gmask.p, sc->tv.p, sc->tinv.p, sc->twr.p, sc->twv.p, sc->tvol.p, sc->tE.p, sc->tnu.p,
              sc->tslot.p, sc->mv.p, sc->minv.p, sc->mw.p, sc->mfib.p, sc->mseg.p, sc->mslot.p, sc->seg_ptr.p,
              sc->seg_mus.p, sc->sv.p, sc->srest.p, sc->ssw.p, sc->sslot.p,
              s.sch.empty() ? nullptr : sc->sch.p, sc->boff.p, sc->bv.p, sc->bbeta.p,
              sc->bw.p, sc->brest.p, sc->bslot.p, sc->vslot_ptr.p, sc->attach_jd.p, sc->hs_ptr.p, sc->hs_col.p,
              sc->hs_val.p, sc->attach_k.p, sc->vpart.p, sc->seg_part.p,
              sc->nF ? sc->vf_ptr.p : nullptr, sc->nF ? sc->vf_face.p : nullptr, sc->nF ? sc->fdrag.p : nullptr};
  if (std::memcmp(&sd, &sc->sd, sizeof(sd)) != 0) invalidate_graphs(sc);
  sc->sd = sd;
}

// Shared memory (doubles) of one supernode's forward / backward solve, with
// or without L_{R,s} staged; mirrors the layout in pd_kernels.cu.
static void solve_shm_doubles(int w, int r, int nseg, bool staged, int cc, size_t* nf, size_t* nb) {
  auto even = [](size_t v) { return (v + 1) & ~size_t(1); };
  const size_t W = w, R = r, l = staged ? even(R * W) : 2 * (size_t)cc * R;
  *nf = even(even(W * W) + l + 6 * W + 3 * (size_t)nseg + (W + 2) / 2);
  *nb = even(even(W * W) + l + 3 * W + 3 * R);
}

// Launch classes of the level-kernel solve by a supernode's shared-memory
// need (doubles): one warp per supernode up to kWarpGroupDoubles (eight per
// CTA); CTAs with at most kSmallCtaDoubles (several CTAs per SM); the rest.
// A class of a level with fewer than kMinClass members joins the next larger
// class of that level (one launch less; its members fit one wave anyway).
#ifndef DFEM_WARP_GROUP_DOUBLES
#define DFEM_WARP_GROUP_DOUBLES 512
#endif
#ifndef DFEM_SMALL_CTA_DOUBLES
#define DFEM_SMALL_CTA_DOUBLES 3072
#endif
constexpr size_t kWarpGroupDoubles = DFEM_WARP_GROUP_DOUBLES;
constexpr size_t kSmallCtaDoubles = DFEM_SMALL_CTA_DOUBLES;
constexpr int kMinClass = 64;
static int shm_class(size_t need) { return need <= kWarpGroupDoubles ? 0 : need <= kSmallCtaDoubles ? 1 : 2; }
// L_{R,s} is staged in shared memory whenever the solve then still fits 220 KB
// (on the 256-scene batch this ran 4 % faster than staging only where the
// supernode keeps its launch class: the long dependency chains at the top of
// the elimination trees gain more from the bulk copies than the launch
// classes lose in resident CTAs).

static int plan_resident(dfem_scene* sc, const std::vector<int>& nseg, const std::vector<int>& cdst);

static int upload_factor(dfem_scene* sc) {
  SupernodalFactor& F = sc->hs.F;
  if (F.sn_rofs.back() > INT32_MAX / 3 || F.sn_lofs.back() > INT32_MAX || F.sn_dofs.back() > INT32_MAX)
    return fail(DFEM_ERR_INVALID, "factor too large for 32-bit offsets");
  const int ns = F.nsuper;
  // contributions grouped by destination row: below-diagonal position p writes slot cdst[p]
  std::vector<int> cdst(std::max<size_t>(1, F.rowidx.size()));
  for (size_t k = 0; k < F.rseg_pos.size(); ++k) cdst[F.rseg_pos[k]] = (int)k;
  CK(sc->rseg_ptr.upload(F.rseg_ptr));
  CK(sc->cdst.upload(cdst));
  if (sc->contrib.n != 3 * F.rowidx.size() || !sc->contrib.p) CK(sc->contrib.alloc(3 * std::max<size_t>(1, F.rowidx.size())));
  auto to32 = [](const std::vector<int64_t>& v) { return std::vector<int>(v.begin(), v.end()); };
  CK(sc->sn_c0.upload(F.sn_c0));
  CK(sc->sn_w.upload(F.sn_w));
  CK(sc->sn_r.upload(F.sn_r));
  CK(sc->sn_rofs.upload(to32(F.sn_rofs)));
  CK(sc->rowidx.upload(F.rowidx));
  CK(sc->sn_lofs.upload(to32(F.sn_lofs)));
  CK(sc->Lcm.upload(F.Lcm));
  CK(sc->sn_dofs.upload(to32(F.sn_dofs)));
  CK(sc->Dinv.upload(F.Dinv));
  {  // column-major copy of every diagonal-block inverse (forward solve)
    std::vector<double> dc(F.Dinv.size(), 0.0);
    parallel_for(ns, [&](int q) {
      const int w = F.sn_w[q];
      const double* src = F.Dinv.data() + F.sn_dofs[q];
      double* dst = dc.data() + F.sn_dofs[q];
      for (int i = 0; i < w; ++i)
        for (int j = 0; j < w; ++j) dst[j * w + i] = src[i * w + j];
    });
    CK(sc->DinvC.upload(dc));
  }
  sc->lvl_ptr = F.lvl_ptr;
  // per supernode: staging or streaming of L_{R,s}, shared memory, launch class
  const size_t budget = 220 * 1024;
  std::vector<int> stage(ns), nseg(ns), cls(ns), chunk(ns, 0);
  std::vector<size_t> need(ns);
  size_t max_cta = 0;
  for (int q = 0; q < ns; ++q) {
    const int w = F.sn_w[q], r = F.sn_r[q];
    nseg[q] = F.rseg_ptr[F.sn_c0[q] + w] - F.rseg_ptr[F.sn_c0[q]];
    size_t uf, ub, tf, tb;
    solve_shm_doubles(w, r, nseg[q], false, 0, &uf, &ub);
    solve_shm_doubles(w, r, nseg[q], true, 0, &tf, &tb);
    const size_t u = std::max(uf, ub), t = std::max(tf, tb);
    if (8 * u > budget)
      return fail(DFEM_ERR_INVALID, "supernode too large for the shared-memory staging of the triangular solves");
    stage[q] = r > 0 && 8 * t <= budget;
    need[q] = stage[q] ? t : u;
    if (!stage[q] && r > 0) {  // stream it: the widest even chunk whose two buffers fit
      const size_t cc = std::min<size_t>(((budget / 8 - u) / (2 * (size_t)r)) & ~size_t(1), (size_t)w);
      if (cc >= 2) {
        chunk[q] = (int)cc;
        need[q] = u + 2 * cc * (size_t)r;
      }
    }
    cls[q] = shm_class(need[q]);
    max_cta = std::max(max_cta, 8 * need[q]);
  }
  // Within a level the supernodes are ordered by their shared-memory need (any
  // order within a level is valid for every solve form and the
  // refactorisation), then cut into launch classes.
  const int L = (int)F.lvl_ptr.size() - 1;
  sc->segs.clear();
  size_t max_warp_blk = 0, max_cta_blk = 0;
  for (int l = 0; l < L; ++l) {
    auto b = F.lvl_sn.begin() + F.lvl_ptr[l], e = F.lvl_sn.begin() + F.lvl_ptr[l + 1];
    std::stable_sort(b, e, [&](int x, int y) { return need[x] < need[y]; });
    int cut[4] = {F.lvl_ptr[l], F.lvl_ptr[l], F.lvl_ptr[l], F.lvl_ptr[l + 1]};
    for (int c = 1; c < 3; ++c) {
      cut[c] = cut[c - 1];
      while (cut[c] < F.lvl_ptr[l + 1] && cls[F.lvl_sn[cut[c]]] < c) ++cut[c];
    }
    for (int c = 0; c < 2; ++c)  // a small class joins the next one
      if (cut[c + 1] - cut[c] < kMinClass && cut[c + 1] < cut[3]) cut[c + 1] = cut[c];
    for (int c = 0; c < 3; ++c) {
      if (cut[c + 1] == cut[c]) continue;
      dfem_scene::LevelSeg sg{cut[c], cut[c + 1] - cut[c], l, c == 0 ? 1 : 0, 0, 0, 0, 0, 256, 256};
      size_t mf = 0, mb = 0;
      for (int k = cut[c]; k < cut[c + 1]; ++k) {
        const int q = F.lvl_sn[k];
        size_t nf, nb;
        solve_shm_doubles(F.sn_w[q], F.sn_r[q], nseg[q], stage[q] != 0, chunk[q], &nf, &nb);
        mf = std::max(mf, nf);
        mb = std::max(mb, nb);
      }
      if (sg.warp) {
        sg.grp_f = (int)mf;
        sg.grp_b = (int)mb;
        sg.shm_f = 8 * 8 * mf;
        sg.shm_b = 8 * 8 * mb;
        max_warp_blk = std::max({max_warp_blk, sg.shm_f, sg.shm_b});
      } else {
        sg.shm_f = 8 * mf;
        sg.shm_b = 8 * mb;
        max_cta_blk = std::max({max_cta_blk, sg.shm_f, sg.shm_b});
      }
      sc->segs.push_back(sg);
    }
  }
  CK(sc->lvl_sn.upload(F.lvl_sn));
  {  // cluster form: each level's warp-sized supernodes are a prefix of the level (sorted by need)
    std::vector<int> lw(L);
    size_t wneed = 0, cneed = 0;
    for (int l = 0; l < L; ++l) {
      int k = F.lvl_ptr[l];
      while (k < F.lvl_ptr[l + 1] && cls[F.lvl_sn[k]] == 0) wneed = std::max(wneed, need[F.lvl_sn[k++]]);
      lw[l] = k;
      for (; k < F.lvl_ptr[l + 1]; ++k) cneed = std::max(cneed, need[F.lvl_sn[k]]);
    }
    CK(sc->lvl_ptr_d.upload(F.lvl_ptr));
    CK(sc->lvl_warp_d.upload(lw));
    sc->shm_cluster_warp = (int)((wneed + 1) & ~size_t(1));
    sc->shm_cluster = std::max<size_t>(16 * 8 * (size_t)sc->shm_cluster_warp, 8 * cneed);
    sc->cluster_ok = sc->shm_cluster <= budget && raise_smem_limit((const void*)k_solve_cluster, sc->shm_cluster) == cudaSuccess;
    cudaGetLastError();
  }
  std::vector<int> snp(ns, 0);
  if (sc->hs.nparts > 1)
    for (int q = 0; q < ns; ++q)
      snp[q] = (int)(std::upper_bound(sc->hs.part_v0.begin(), sc->hs.part_v0.end(), F.sn_c0[q]) - sc->hs.part_v0.begin()) - 1;
  {
    std::vector<SnInfo> info(std::max(1, ns));
    for (int k = 0; k < ns; ++k) {
      const int q = F.lvl_sn[k];
      info[k] = SnInfo{F.sn_c0[q], F.sn_w[q], F.sn_r[q], (int)F.sn_rofs[q], (int)F.sn_lofs[q], (int)F.sn_dofs[q],
                       F.rseg_ptr[F.sn_c0[q]], nseg[q], q, snp[q], stage[q], chunk[q]};
    }
    CK(sc->sn_info.upload(info));
  }
  for (auto fn : {(const void*)k_fwd_level<CtaGroup>, (const void*)k_bwd_level<CtaGroup>})
    CK(raise_smem_limit(fn, max_cta_blk));
  for (auto fn : {(const void*)k_fwd_level<WarpGroup>, (const void*)k_bwd_level<WarpGroup>})
    CK(raise_smem_limit(fn, max_warp_blk));
  // persistent solve: elimination tree (children CSR), completion stamps, control words
  {
    std::vector<int> kp(ns + 1, 0), kd(std::max(1, ns));
    for (int q = 0; q < ns; ++q)
      if (F.sn_parent[q] >= 0) kp[F.sn_parent[q] + 1]++;
    for (int q = 0; q < ns; ++q) kp[q + 1] += kp[q];
    std::vector<int> fill(kp.begin(), kp.end() - 1);
    for (int q = 0; q < ns; ++q)
      if (F.sn_parent[q] >= 0) kd[fill[F.sn_parent[q]]++] = q;
    CK(sc->sn_parent.upload(F.sn_parent));
    CK(sc->kid_ptr.upload(kp));
    CK(sc->kid.upload(kd));
    if (sc->done_f.n != (size_t)ns || !sc->done_f.p) {
      CK(sc->done_f.alloc(std::max(1, ns)));
      CK(sc->done_b.alloc(std::max(1, ns)));
      CK(sc->solve_ctl.alloc(4));
    }
    sc->shm_pers = max_cta;
    CK(raise_smem_limit((const void*)k_solve_persistent, sc->shm_pers));
    int nsm = 1, per_sm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, sc->device));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_persistent, 256, sc->shm_pers));
    sc->pers_slots = std::max(1, nsm * std::max(1, per_sm));
  }
  if (sc->hs.nparts > 1) CK(sc->sn_part.upload(snp));
  {
    std::vector<int> pos(std::max(1, ns));
    for (int k = 0; k < ns; ++k) pos[F.lvl_sn[k]] = k;
    CK(sc->sn_pos.upload(pos));
  }
  RC(plan_resident(sc, nseg, cdst));
  FactorDev fd{sc->sn_info.p, sc->rseg_ptr.p, sc->cdst.p, sc->contrib.p, sc->rowidx.p, sc->Lcm.p, sc->Dinv.p,
               sc->DinvC.p, sc->status.p, ns, sc->sn_pos.p, sc->sn_parent.p, sc->kid_ptr.p, sc->kid.p, sc->done_f.p,
               sc->done_b.p, sc->solve_ctl.p, sc->spin_tries};
  if (std::memcmp(&fd, &sc->fd, sizeof(fd)) != 0) invalidate_graphs(sc);
  sc->fd = fd;
  return DFEM_OK;
}

// The resident solve form (k_solve_resident): a single scene whose factor
// fits the shared memory of one cluster.  The widest cluster the device
// schedules with the full shared memory per CTA (16, else 8), then the layout
// of plan_resident_layout (resident_plan.cpp): owners, shared-memory offsets,
// contribution and solution address tables, and the images with their row
// tables; the blocks are copied into the images after every refactorisation.
static int plan_resident(dfem_scene* sc, const std::vector<int>& nseg, const std::vector<int>& cdst) {
  sc->res_ok = false;
  const HostScene& s = sc->hs;
  const SupernodalFactor& F = s.F;
  if (s.nparts != 1 || F.nsuper == 0 || F.nlevels == 0) return DFEM_OK;
  int optin = 0;
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, sc->device));
  const size_t cap_bytes = optin > 2048 ? (size_t)optin - 1024 : 0;  // the static mbarrier and a margin
  CK(cudaFuncSetAttribute((const void*)k_solve_resident, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  CK(raise_smem_limit((const void*)k_solve_resident, cap_bytes));
  int C = 0;
  for (int c : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(512);
    cfg.dynamicSmemBytes = cap_bytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (const void*)k_solve_resident, &cfg) == cudaSuccess && n >= 1) {
      C = c;
      break;
    }
    cudaGetLastError();
  }
  ResidentPlan P;
  if (C == 0 || !plan_resident_layout(F, nseg, cdst, C, cap_bytes, P)) return DFEM_OK;
  std::vector<ResPack> pk;
  for (const auto& q : P.pack) pk.push_back(ResPack{q.w, q.r, q.src_d, q.src_l, q.dst_d, q.dst_l});
  CK(sc->res_head.upload(P.head_len));
  CK(sc->res_img.upload(P.img));
  CK(sc->res_img_ofs.upload(P.img_ofs));
  CK(sc->res_pack.upload(pk));
  CK(raise_smem_limit((const void*)k_solve_resident, 8 * P.smem_doubles));
  sc->res_ctas = C;
  sc->shm_res = 8 * P.smem_doubles;
  sc->rdv = ResDev{sc->res_img.p, sc->res_img_ofs.p, sc->res_head.p, P.L, (int)P.smem_doubles, sc->status.p};
  sc->res_ok = true;
  return DFEM_OK;
}

// The factor's blocks into the resident images (after a refactorisation).
static void pack_resident(dfem_scene* sc) {
  if (!sc->res_ok) return;
  k_res_pack<<<sc->hs.F.nsuper, 256, 0, sc->stream>>>(sc->res_pack.p, sc->Dinv.p, sc->Lcm.p, sc->res_img.p);
  sc->launches += 1;
}

static int upload_materials(dfem_scene* sc) {
  HostScene& s = sc->hs;
  std::vector<double> wr(s.T), wv(s.T);
  for (int e = 0; e < s.T; ++e) {
    double mu = s.tE[e] / (1.0 + s.tnu[e]);  // CorotateFEMConstraint: mMu = E/(1+nu)
    wr[e] = mu * s.tvol[e];
    wv[e] = wr[e] * s.tnu[e];                // second block scaled by nu (EvaluateJMatrix)
  }
  CK(sc->twr.upload(wr));
  CK(sc->twv.upload(wv));
  CK(sc->tE.upload(s.tE));
  CK(sc->tnu.upload(s.tnu));
  std::vector<int> hp(s.Hs.ptr.begin(), s.Hs.ptr.end());
  CK(sc->hs_ptr.upload(hp));
  CK(sc->hs_col.upload(s.Hs.col));
  CK(sc->hs_val.upload(s.Hs.val));
  return upload_factor(sc);
}

template <typename T>
static std::vector<T> planes(const std::vector<T>& aos, int n, int k) {  // AoS (k per item) -> k planes
  std::vector<T> out((size_t)n * k);
  for (int e = 0; e < n; ++e)
    for (int q = 0; q < k; ++q) out[(size_t)q * n + e] = aos[(size_t)e * k + q];
  return out;
}

// Structure of the GPU refactorisation: Hs split into its E-independent base
// and per-entry tet contributions (per part in parallel for a batch), and the
// left-looking update lists of every supernode (descendant d, rows R_d[a0..a1)
// inside the supernode's columns), in increasing d.
static int upload_refactor_plan(dfem_scene* sc) {
  HostScene& s = sc->hs;
  std::vector<double> base, coef;
  std::vector<int> cptr, ctet;
  if (sc->parts.empty()) {
    hs_split(s, base, cptr, ctet, coef);
  } else {
    const int np = (int)sc->parts.size();
    std::vector<std::vector<double>> pb(np), pc(np);
    std::vector<std::vector<int>> pp(np), pt(np);
    parallel_for(np, [&](int p) { hs_split(sc->parts[p], pb[p], pp[p], pt[p], pc[p]); });
    cptr = {0};
    for (int p = 0; p < np; ++p) {
      const int off = cptr.back(), t0 = s.part_t0[p];
      base.insert(base.end(), pb[p].begin(), pb[p].end());
      coef.insert(coef.end(), pc[p].begin(), pc[p].end());
      for (size_t k = 1; k < pp[p].size(); ++k) cptr.push_back(pp[p][k] + off);
      for (int t : pt[p]) ctet.push_back(t + t0);
    }
  }
  if (base.size() != s.Hs.val.size()) return fail(DFEM_ERR_INVALID, "refactorisation plan: Hs pattern mismatch");
  CK(sc->hs_base.upload(base));
  CK(sc->hc_ptr.upload(cptr));
  CK(sc->hc_tet.upload(ctet.empty() ? std::vector<int>{0} : ctet));
  CK(sc->hc_coef.upload(coef.empty() ? std::vector<double>{0.0} : coef));
  const SupernodalFactor& F = s.F;
  std::vector<std::vector<int>> ud(F.nsuper), ua0(F.nsuper), ua1(F.nsuper);
  for (int d = 0; d < F.nsuper; ++d) {
    const int r = F.sn_r[d];
    const int* R = &F.rowidx[F.sn_rofs[d]];
    int b0 = 0;
    while (b0 < r) {
      const int p = F.col_sn[R[b0]];
      int b1 = b0;
      while (b1 < r && F.col_sn[R[b1]] == p) ++b1;
      ud[p].push_back(d); ua0[p].push_back(b0); ua1[p].push_back(b1);
      b0 = b1;
    }
  }
  std::vector<int> uptr(F.nsuper + 1, 0), vd, va0, va1;
  for (int q = 0; q < F.nsuper; ++q) {
    vd.insert(vd.end(), ud[q].begin(), ud[q].end());
    va0.insert(va0.end(), ua0[q].begin(), ua0[q].end());
    va1.insert(va1.end(), ua1[q].begin(), ua1[q].end());
    uptr[q + 1] = (int)vd.size();
  }
  if (vd.empty()) { vd = {0}; va0 = {0}; va1 = {0}; }
  CK(sc->up_ptr.upload(uptr));
  CK(sc->up_d.upload(vd));
  CK(sc->up_a0.upload(va0));
  CK(sc->up_a1.upload(va1));
  CK(sc->Ldw.alloc(std::max<size_t>(1, F.Dinv.size())));
  const int np = s.nparts;
  sc->part_reg_h.assign(np, 0.0);
  CK(sc->part_reg.upload(sc->part_reg_h));
  CK(sc->part_fail.alloc(np + 1));
  CK(sc->E_in.alloc(std::max(1, s.T)));
  CK(sc->nu_in.alloc(std::max(1, s.T)));
  int maxw = 1;
  for (int w : F.sn_w) maxw = std::max(maxw, w);
  sc->shm_fact = factor_smem_bytes(maxw);
  if (sc->shm_fact > 227 * 1024) return fail(DFEM_ERR_INVALID, "supernode too wide for the GPU refactorisation");
  CK(raise_smem_limit((const void*)k_factor_level, sc->shm_fact));
  CK(raise_smem_limit((const void*)k_factor_diag, sc->shm_fact));
  CK(raise_smem_limit((const void*)k_factor_trsm, sc->shm_fact));
  int nsm = 1;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, sc->device));
  sc->shm_fact_lvl.assign(F.nlevels, 0);
  sc->fact_shares.assign(F.nlevels, 0);
  sc->fact_w.assign(F.nlevels, 1);
  for (int l = 0; l < F.nlevels; ++l) {
    int mw = 1;
    for (int k = F.lvl_ptr[l]; k < F.lvl_ptr[l + 1]; ++k) mw = std::max(mw, F.sn_w[F.lvl_sn[k]]);
    sc->shm_fact_lvl[l] = factor_smem_bytes(mw);
    sc->fact_w[l] = mw;
    // levels of few supernodes (the top of the tree) leave most SMs idle in
    // the one-launch form: their updates and rows below spread over CTAs
    const int cnt = F.lvl_ptr[l + 1] - F.lvl_ptr[l];
    if (cnt * kFactorSplitRatio <= nsm) sc->fact_shares[l] = std::min(kFactorMaxShares, nsm / cnt);
  }
  sc->rd = RefactorDev{s.T, sc->tvol.p, sc->tE.p, sc->tnu.p, sc->twr.p, sc->twv.p, (int)base.size(),
                       sc->hs_base.p, sc->hc_ptr.p, sc->hc_tet.p, sc->hc_coef.p, sc->hs_val.p, sc->hs_ptr.p,
                       sc->hs_col.p, sc->sn_c0.p, sc->sn_w.p, sc->sn_r.p, sc->sn_rofs.p, sc->rowidx.p,
                       sc->sn_lofs.p, sc->Lcm.p, sc->sn_dofs.p, sc->Dinv.p, sc->DinvC.p, sc->Ldw.p, sc->lvl_sn.p, sc->up_ptr.p,
                       sc->up_d.p, sc->up_a0.p, sc->up_a1.p, np > 1 ? sc->sn_part.p : nullptr, sc->part_reg.p,
                       sc->part_fail.p};
  return DFEM_OK;
}

// Largest single scene (vertices) served by the dense-inverse form: X and its
// workspace take 2 N_p^2 doubles (268 MB at 4,096 vertices).
constexpr int kDenseMaxN = 4096;
// The dense form is kept when its saving per solve, over this many solves,
// exceeds the time to rebuild X after a refactorisation.
constexpr double kDenseAmortSolves = 100.0;

static void dense_release(dfem_scene* sc) {
  sc->dn_A.alloc(0);
  sc->dn_W.alloc(0);
  sc->dn_T.alloc(0);
  sc->dn_Linv.alloc(0);
  sc->dense_built = false;
  sc->dd = DenseDev{};
}

// X = Hs^-1 from the current GPU factor (dense_solve.cuh), on the scene's stream.
static int dense_build(dfem_scene* sc) {
  const int N = sc->hs.N, nb = (N + kDenseTile - 1) / kDenseTile, Np = nb * kDenseTile;
  const size_t nn = (size_t)Np * Np;
  if (!sc->dn_A.p || !sc->dn_W.p || !sc->dn_T.p || !sc->dn_Linv.p || sc->dn_A.n != nn) {
    CK(raise_smem_limit((const void*)k_dense_tile_inv, kDenseSmem));
    CK(raise_smem_limit((const void*)k_dense_trtri_t, kDenseSmem));
    CK(raise_smem_limit((const void*)k_dense_trtri_w, kDenseSmem));
    CK(raise_smem_limit((const void*)k_dense_lauum, kDenseSmem));
    CK(raise_smem_limit((const void*)k_dense_solve, 3 * (size_t)Np * sizeof(double)));
    int nsm = 1;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, sc->device));
    sc->dense_grid = std::max(1, std::min(nsm, N));
    sc->dense_built = false;
    // all four or none: a failed allocation leaves no buffers behind
    cudaError_t e = sc->dn_A.alloc(nn);
    if (e == cudaSuccess) e = sc->dn_W.alloc(nn);
    if (e == cudaSuccess) e = sc->dn_T.alloc(nn);
    if (e == cudaSuccess) e = sc->dn_Linv.alloc((size_t)nb * kDenseTile * kDenseTile);
    if (e != cudaSuccess) {
      dense_release(sc);
      CK(e);
    }
  }
  sc->dd = DenseDev{N, Np, nb, sc->dn_A.p, sc->dn_W.p, sc->dn_T.p, sc->dn_Linv.p};
  CK(cudaMemsetAsync(sc->dn_A.p, 0, nn * sizeof(double), sc->stream));
  k_dense_scatter<<<sc->hs.F.nsuper, 256, 0, sc->stream>>>(sc->dd, sc->fd, sc->Ldw.p, sc->sn_dofs.p);
  k_dense_tile_inv<<<nb, kDenseThreads, kDenseSmem, sc->stream>>>(sc->dd);
  int levels = 0;
  for (int w = 1; w < nb; w *= 2, ++levels) {
    const dim3 grid(w * w, (nb + 2 * w - 1) / (2 * w));
    k_dense_trtri_t<<<grid, kDenseThreads, kDenseSmem, sc->stream>>>(sc->dd, w);
    k_dense_trtri_w<<<grid, kDenseThreads, kDenseSmem, sc->stream>>>(sc->dd, w);
  }
  k_dense_lauum<<<nb * (nb + 1) / 2, kDenseThreads, kDenseSmem, sc->stream>>>(sc->dd);
  sc->launches += 3 + 2 * levels;
  CK(cudaGetLastError());
  sc->dense_built = true;
  return DFEM_OK;
}

// Materials from E_in / nu_in (device), Hs values, and the factor on the GPU.
// A part whose factorisation meets a non-positive pivot is retried with the
// reference's regularisation sequence (0, 1e-5, x10 ..., 25 attempts); the
// other parts keep their regularisation, so their factors are unchanged.
static int gpu_refactor(dfem_scene* sc) {
  const HostScene& s = sc->hs;
  const int np = s.nparts;
  CK(cudaMemsetAsync(sc->part_fail.p, 0, sizeof(int) * (np + 1), sc->stream));
  if (s.T > 0) k_materials<<<(s.T + 127) / 128, 128, 0, sc->stream>>>(sc->rd, sc->E_in.p, sc->nu_in.p, np);
  k_hs_values<<<(sc->rd.nnz + 255) / 256, 256, 0, sc->stream>>>(sc->rd);
  sc->launches += (s.T > 0 ? 1 : 0) + 1;
  std::vector<int> failh(np + 1);
  CK(cudaMemcpyAsync(failh.data(), sc->part_fail.p, sizeof(int) * (np + 1), cudaMemcpyDeviceToHost, sc->stream));
  CK(cudaStreamSynchronize(sc->stream));
  if (failh[np]) return fail(DFEM_ERR_INVALID, "invalid material (non-finite E or nu, or nu <= -1)");
  std::fill(sc->part_reg_h.begin(), sc->part_reg_h.end(), 0.0);
  const int L = (int)sc->lvl_ptr.size() - 1;
  for (int attempt = 0; attempt < 25; ++attempt) {
    CK(cudaMemcpyAsync(sc->part_reg.p, sc->part_reg_h.data(), sizeof(double) * np, cudaMemcpyHostToDevice, sc->stream));
    CK(cudaMemsetAsync(sc->part_fail.p, 0, sizeof(int) * np, sc->stream));
    for (int l = 0; l < L; ++l) {
      const int cnt = sc->lvl_ptr[l + 1] - sc->lvl_ptr[l], p0 = sc->lvl_ptr[l];
      const int sh = sc->split_factor ? sc->fact_shares[l] : 0;
      if (sh == 0) {
        k_factor_level<<<cnt, 256, sc->shm_fact_lvl[l], sc->stream>>>(sc->rd, p0);
        sc->launches += 1;
        continue;
      }
      const size_t w = (size_t)sc->fact_w[l];
      k_factor_scatter<<<cnt, 256, 0, sc->stream>>>(sc->rd, p0);
      k_factor_update<<<dim3(cnt, sh), 256, 0, sc->stream>>>(sc->rd, p0);
      k_factor_diag<<<cnt, 256, 2 * w * w * sizeof(double), sc->stream>>>(sc->rd, p0);
      k_factor_trsm<<<dim3(cnt, sh), 256, (w * w + kTrsmRows * w) * sizeof(double), sc->stream>>>(sc->rd, p0);
      sc->launches += 4;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(failh.data(), sc->part_fail.p, sizeof(int) * np, cudaMemcpyDeviceToHost, sc->stream));
    CK(cudaStreamSynchronize(sc->stream));
    bool any = false;
    for (int p = 0; p < np; ++p)
      if (failh[p]) {
        any = true;
        sc->part_reg_h[p] = sc->part_reg_h[p] == 0.0 ? 1e-5 : sc->part_reg_h[p] * 10.0;
      }
    if (!any) {
      pack_resident(sc);
      sc->dense_built = false;  // X follows the factor (only while the dense form is in use)
      if (sc->solve_cut == -3) RC(dense_build(sc));
      return DFEM_OK;
    }
  }
  return fail(DFEM_ERR_FACTOR, "Cholesky factorisation failed after 25 regularisation retries");
}

// Uniform grid over the static obstacle faces for the detection's broad phase
// (the reference rebuilds an arcsim BVH over them at every detection,
// sim/utils/arcsim/collision.cpp:29-37): cell size twice the median extent of
// a face box, grown until the grid has at most 2^20 cells; every face listed,
// in ascending order, in every cell that its box dilated by kBroadPad touches.
// Cells are located with the same monotone formula as bp_cell on the device,
// so a vertex's query (its swept box, dilated alike) meets every face whose
// dilated box it overlaps: the culling drops no impact.  No grid (every face
// is tested) for fewer than 16 faces or more than 2^24 cell entries.
static int build_obstacle_grid(dfem_scene* sc) {
  const HostScene& s = sc->hs;
  ContactDev& c = sc->cd;
  const int nof = (int)s.obs_f.size() / 3;
  c.bp_max_cells = kBroadDefaultCells;
  c.bp_dim[0] = c.bp_dim[1] = c.bp_dim[2] = 0;
  c.bp_ptr = nullptr;
  c.bp_face = nullptr;
  if (nof < 16) return DFEM_OK;
  std::vector<double> lo(3 * (size_t)nof), hi(3 * (size_t)nof), ext(nof);
  double glo[3] = {1e300, 1e300, 1e300}, ghi[3] = {-1e300, -1e300, -1e300};
  for (int f = 0; f < nof; ++f) {
    double e = 0.0;
    for (int k = 0; k < 3; ++k) {
      double a = 1e300, b = -1e300;
      for (int q = 0; q < 3; ++q) {
        const double v = s.obs_x[3 * (size_t)s.obs_f[3 * f + q] + k];
        a = std::min(a, v);
        b = std::max(b, v);
      }
      e = std::max(e, b - a);
      lo[3 * f + k] = a - kBroadPad;
      hi[3 * f + k] = b + kBroadPad;
      glo[k] = std::min(glo[k], lo[3 * f + k]);
      ghi[k] = std::max(ghi[k], hi[3 * f + k]);
    }
    ext[f] = e;
  }
  std::vector<double> se(ext);
  std::nth_element(se.begin(), se.begin() + nof / 2, se.end());
  const double diag = std::sqrt((ghi[0] - glo[0]) * (ghi[0] - glo[0]) + (ghi[1] - glo[1]) * (ghi[1] - glo[1]) +
                                (ghi[2] - glo[2]) * (ghi[2] - glo[2]));
  double h = std::max({2.0 * se[nof / 2], 1e-6 * diag, 1e-9});
  int dim[3];
  for (;;) {
    long long cells = 1;
    for (int k = 0; k < 3; ++k) {
      dim[k] = std::max(1, (int)std::ceil((ghi[k] - glo[k]) / h));
      cells *= dim[k];
    }
    if (cells <= (1 << 20)) break;
    h *= 1.26;
  }
  const double inv = 1.0 / h;
  auto cell = [&](double v, int k) {  // bp_cell on the device
    const double u = std::floor((v - glo[k]) * inv);
    return u < 0.0 ? 0 : (u >= (double)(dim[k] - 1) ? dim[k] - 1 : (int)u);
  };
  const size_t ncell = (size_t)dim[0] * dim[1] * dim[2];
  std::vector<int> ptr(ncell + 1, 0);
  size_t total = 0;
  for (int pass = 0; pass < 2; ++pass) {
    std::vector<int> fill;
    std::vector<int> face;
    if (pass == 1) {
      for (size_t q = 0; q < ncell; ++q) ptr[q + 1] += ptr[q];
      fill.assign(ptr.begin(), ptr.end() - 1);
      face.resize(ptr[ncell]);
    }
    for (int f = 0; f < nof; ++f) {
      int i0[3], i1[3];
      for (int k = 0; k < 3; ++k) { i0[k] = cell(lo[3 * f + k], k); i1[k] = cell(hi[3 * f + k], k); }
      for (int z = i0[2]; z <= i1[2]; ++z)
        for (int y = i0[1]; y <= i1[1]; ++y)
          for (int x = i0[0]; x <= i1[0]; ++x) {
            const size_t q = ((size_t)z * dim[1] + y) * dim[0] + x;
            if (pass == 0) {
              ptr[q + 1]++;
              if (++total > (size_t)(1 << 24)) return DFEM_OK;  // too many entries: no grid
            } else {
              face[fill[q]++] = f;
            }
          }
    }
    if (pass == 1) {
      CK(sc->bp_ptr.upload(ptr));
      CK(sc->bp_face.upload(face.empty() ? std::vector<int>{0} : face));
    }
  }
  for (int k = 0; k < 3; ++k) { c.bp_dim[k] = dim[k]; c.bp_org[k] = glo[k]; }
  c.bp_inv = inv;
  c.bp_ptr = sc->bp_ptr.p;
  c.bp_face = sc->bp_face.p;
  return DFEM_OK;
}

static int upload_skeleton(dfem_scene* sc);

// the skeleton view's history and adjoint pointers (set by upload_skeleton and
// by ensure_steps, which sizes the history)
static void skel_bind(dfem_scene* sc) {
  SkelDev& k = sc->skd;
  k.nq = sc->sk_nq;
  k.K = sc->hs.K;
  k.hstride = (long long)k.nq + k.ndof + 3LL * k.nr;
  k.hist = sc->sk_hist.p;
  k.jin = sc->sk_jin.p;
  k.thb = sc->sk_thb.p; k.sb = sc->sk_sb.p; k.gjq = sc->sk_gjq.p; k.gjqd = sc->sk_gjqd.p;
  k.mu2 = sc->sk_mu2.p; k.mu3 = sc->sk_mu3.p; k.dlt = sc->sk_dlt.p;
}

// for the OBJ writer (obj_writer.cpp): the stream and device of a scene
cudaStream_t scene_stream(dfem_scene* sc) { return sc->stream; }
int scene_device(dfem_scene* sc) { return sc->device; }

static int upload_scene(dfem_scene* sc) {
  HostScene& s = sc->hs;
  CK(sc->mass.upload(s.mass));
  CK(sc->gmask.upload(s.gmask));
  CK(sc->tinv.upload(planes(s.tinv, s.T, 9)));
  CK(sc->tvol.upload(s.tvol));
  std::vector<int4> tv(s.T), tsl(s.T);
  for (int e = 0; e < s.T; ++e) {
    tv[e] = make_int4(s.tv[4 * e], s.tv[4 * e + 1], s.tv[4 * e + 2], s.tv[4 * e + 3]);
    tsl[e] = make_int4(s.tslot[4 * e], s.tslot[4 * e + 1], s.tslot[4 * e + 2], s.tslot[4 * e + 3]);
  }
  CK(sc->tv.upload(tv));
  CK(sc->tslot.upload(tsl));
  std::vector<int4> mv(s.M), msl(s.M);
  std::vector<double> mw(s.M);
  for (int m = 0; m < s.M; ++m) {
    mv[m] = make_int4(s.mv[4 * m], s.mv[4 * m + 1], s.mv[4 * m + 2], s.mv[4 * m + 3]);
    msl[m] = make_int4(s.mslot[4 * m], s.mslot[4 * m + 1], s.mslot[4 * m + 2], s.mslot[4 * m + 3]);
    mw[m] = s.mvol[m] * s.mk[m];
  }
  CK(sc->mv.upload(mv));
  CK(sc->mslot.upload(msl));
  CK(sc->mw.upload(mw));
  CK(sc->minv.upload(planes(s.minv, s.M, 9)));
  CK(sc->mfib.upload(planes(s.mfib, s.M, 3)));
  CK(sc->mseg.upload(s.mseg));
  CK(sc->seg_ptr.upload(s.seg_ptr));
  CK(sc->seg_mus.upload(s.seg_mus));
  std::vector<int2> sv(s.S), ssl(s.S);
  for (int k = 0; k < s.S; ++k) {
    sv[k] = make_int2(s.sv[2 * k], s.sv[2 * k + 1]);
    ssl[k] = make_int2(s.sslot[2 * k], s.sslot[2 * k + 1]);
  }
  CK(sc->sv.upload(sv));
  CK(sc->sslot.upload(ssl));
  CK(sc->srest.upload(s.srest));
  CK(sc->ssw.upload(s.ssw));
  if (!s.sch.empty()) CK(sc->sch.upload(s.sch));
  CK(sc->boff.upload(s.boff));
  CK(sc->bv.upload(s.bv));
  CK(sc->bslot.upload(s.bslot));
  CK(sc->bbeta.upload(s.bbeta));
  CK(sc->bw.upload(s.bw));
  CK(sc->brest.upload(s.brest));
  CK(sc->vslot_ptr.upload(s.vslot_ptr));
  std::vector<double> ajd(3 * (size_t)s.N, 0.0);  // AttachmentConstraint: J d = k p
  for (int a = 0; a < s.A; ++a)
    for (int c = 0; c < 3; ++c) ajd[3 * (size_t)s.av[a] + c] += s.ak[a] * s.ap[3 * a + c];
  CK(sc->attach_jd.upload(ajd));
  std::vector<double> ak(s.N, 0.0);
  for (int a = 0; a < s.A; ++a) ak[s.av[a]] += s.ak[a];
  CK(sc->attach_k.upload(ak));
  CK(sc->to_user.upload(s.to_user));
  CK(sc->to_internal.upload(s.to_internal));
  sc->nF = (int)s.df.size() / 3;
  if (sc->nF > 0) {
    CK(sc->df.upload(s.df));
    CK(sc->vf_ptr.upload(s.vf_ptr));
    CK(sc->vf_face.upload(s.vf_face));
    CK(sc->fdrag.alloc(3 * (size_t)sc->nF));
    CK(sc->fdrag_b.alloc(18 * (size_t)sc->nF));
  }
  int rc = upload_materials(sc);
  if (rc) return rc;
  const size_t n3 = 3 * (size_t)s.N;
  CK(sc->xt.alloc(n3)); CK(sc->vt.alloc(n3)); CK(sc->qn.alloc(n3)); CK(sc->c0.alloc(n3));
  CK(sc->xk.alloc(n3)); CK(sc->rhs.alloc(n3)); CK(sc->y.alloc(n3)); CK(sc->io_a.alloc(n3)); CK(sc->io_b.alloc(n3));
  CK(sc->slot.alloc(3 * (size_t)std::max(1, s.nslots)));
  CK(sc->xkb.alloc(n3)); CK(sc->xtb.alloc(n3)); CK(sc->bb.alloc(n3));
  CK(sc->gE.alloc(std::max(1, s.T))); CK(sc->gnu.alloc(std::max(1, s.T))); CK(sc->mg.alloc(std::max(1, s.M + (s.sch.empty() ? 0 : s.S))));
  sc->nblk_v = (s.N + 127) / 128;
  // part tables: part-aligned blocks of the reducing vertex kernels
  const int np = s.nparts;
  std::vector<int> pb0(np + 1, 0), bpart, bv0;
  for (int p = 0; p < np; ++p) {
    for (int v = s.part_v0[p]; v < s.part_v0[p + 1]; v += kPartBlock) { bpart.push_back(p); bv0.push_back(v); }
    pb0[p + 1] = (int)bpart.size();
  }
  sc->nblk_p = (int)bpart.size();
  CK(sc->part_v0.upload(s.part_v0));
  CK(sc->part_b0.upload(pb0));
  CK(sc->blk_part.upload(bpart));
  CK(sc->blk_v0.upload(bv0));
  sc->pd = PartDev{np, sc->part_v0.p, sc->part_b0.p, sc->blk_part.p, sc->blk_v0.p};
  if (np > 1) {
    std::vector<int> vp(s.N), sp(std::max(1, s.nseg), 0);
    for (int p = 0; p < np; ++p) {
      for (int v = s.part_v0[p]; v < s.part_v0[p + 1]; ++v) vp[v] = p;
      for (int q = s.part_seg0[p]; q < s.part_seg0[p + 1]; ++q) sp[q] = p;
    }
    CK(sc->vpart.upload(vp));
    CK(sc->seg_part.upload(sp));
  }
  CK(sc->partial.alloc(std::max(sc->nblk_p, 1)));
  CK(sc->errv.alloc(np));
  CK(sc->counter.alloc(np));
  CK(sc->flag.alloc(np)); CK(sc->step.alloc(1)); CK(sc->write_traj.alloc(1));
  CK(sc->zero.alloc(1));
  CK(cudaMemset(sc->counter.p, 0, sizeof(unsigned) * np));
  CK(cudaMemset(sc->status.p, 0, 4 * sizeof(int)));
  // activations until set: muscle segments 0, pneumatic channels 1
  // (PneumaticConstraint::mActivationLevel = 1, pneumaticEasy.h:31)
  {
    std::vector<double> a0(std::max(1, s.nseg), 0.0);
    for (int c : s.sch)
      if (c >= 0) a0[c] = 1.0;
    CK(sc->act_cur.upload(a0));
  }
  // obstacle contact phase
  const int nc = (int)s.cverts.size(), nof = (int)s.obs_f.size() / 3;
  sc->self_contact = s.self_collide;
  sc->has_contact = s.collide && nc > 0 && (nof > 0 || sc->self_contact);
  if (sc->has_contact) {
    std::vector<int> cidx(s.N, -1);
    for (int a = 0; a < nc; ++a) cidx[s.cverts[a]] = a;
    std::vector<double> hd(s.N, 0.0);
    for (int i = 0; i < s.N; ++i)
      for (int64_t k = s.Hs.ptr[i]; k < s.Hs.ptr[i + 1]; ++k)
        if (s.Hs.col[k] == i) hd[i] = s.Hs.val[k];
    CK(sc->cverts.upload(s.cverts));
    CK(sc->cidx.upload(cidx));
    CK(sc->obs_x.upload(s.obs_x));
    CK(sc->obs_f.upload(s.obs_f));
    CK(sc->hdiag.upload(hd));
    CK(sc->imp_cnt.alloc(nc));
    CK(sc->imp_face.alloc((size_t)nc * kMaxImpactsPerVertex));
    CK(sc->imp_n.alloc((size_t)nc * kMaxImpactsPerVertex * 3));
    CK(sc->xn1.alloc(n3)); CK(sc->xold.alloc(n3)); CK(sc->cprev.alloc(n3)); CK(sc->lxt.alloc(n3)); CK(sc->vwc.alloc(n3));
    CK(sc->cstate.alloc(CS_SIZE));
    CK(cudaMemset(sc->cstate.p, 0, sizeof(int) * CS_SIZE));
    CK(sc->crec_on.alloc(1));
    CK(cudaMemset(sc->crec_on.p, 0, sizeof(int)));
    CK(sc->crec_base.alloc(1));
    CK(cudaMemset(sc->crec_base.p, 0, sizeof(int)));
    sc->cd = ContactDev{nc, nof, s.K, kMaxContactPasses, kMaxImpactsPerVertex, kMaxSelfImpacts, kMaxGroupMembers,
                        kBroadDefaultCells, {0, 0, 0}, {0.0, 0.0, 0.0}, 0.0, nullptr, nullptr,
                        s.alpha, s.mu_obs, sc->cverts.p, sc->cidx.p, sc->obs_x.p,
                        sc->obs_f.p, sc->hdiag.p, sc->imp_cnt.p, sc->imp_face.p, sc->imp_n.p, sc->xn1.p, sc->xold.p,
                        sc->cprev.p, sc->lxt.p, sc->vwc.p, sc->cstate.p, sc->crec_on.p, 0, 0, nullptr, nullptr,
                        nullptr, nullptr, nullptr, sc->status.p, sc->crec_base.p, nullptr};
    if (s.nparts > 1) {  // a batch: per-part contact state, no broad phase
      const int np = s.nparts;
      if (np > kMaxContactParts)
        return fail(DFEM_ERR_UNSUPPORTED, "batch: obstacle contact needs at most " + std::to_string(kMaxContactParts) + " scenes");
      sc->cnp = np;
      CK(sc->c_cpart.upload(s.cpart));
      CK(sc->c_pf0.upload(s.pobs_f0));
      CK(sc->c_pst.alloc((size_t)PS_SIZE * np));
      CK(cudaMemset(sc->c_pst.p, 0, sizeof(int) * PS_SIZE * np));
      CK(sc->c_pany.alloc(2 * (size_t)np));
      CK(sc->c_pe.alloc(2 * (size_t)np));
      ContactDev& c = sc->cd;
      c.np = np; c.cpart = sc->c_cpart.p; c.pf0 = sc->c_pf0.p; c.pst = sc->c_pst.p;
      c.pany = sc->c_pany.p; c.pe = sc->c_pe.p;
    } else {
      RC(build_obstacle_grid(sc));
    }
    if (!sc->self_contact) {  // the fused phase: every CTA resident (cooperative launch)
      int nsm = 1, occ = 0, occ_a = 0, coop = 0;
      CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, sc->device));
      CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, sc->device));
      if (sc->cnp > 0) {
        const size_t shm = sizeof(int) * PS_SIZE * (size_t)sc->cnp;
        CK(raise_smem_limit((const void*)k_contact_fused_parts, shm));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_contact_fused_parts, 128, shm));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_cadj_fused_parts, 128, 0));
      } else {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_contact_fused, 128, 0));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_cadj_fused, 128, 0));
      }
      const int ncons = s.T + s.M + s.S + s.B;
      const int want = std::max(1, (std::max(ncons, s.N) + 127) / 128);
      sc->fused_grid = std::min(nsm * occ, want);
      sc->cadj_grid = std::min(nsm * occ_a, want);
      sc->fused_ok = coop != 0 && occ > 0 && occ_a > 0;
      if (sc->fused_ok) CK(sc->fpartial.alloc(std::max(1, sc->fused_grid)));
    }
    if (sc->cnp > 0) sc->fused_on = false;  // batches: the loop of kernels unless the cooperative form is asked for
    if (sc->self_contact) {
      const int ncf = (int)s.cfaces.size() / 3;
      CK(sc->s_cfaces.upload(s.cfaces));
      CK(sc->s_cvf_ptr.upload(s.cvf_ptr));
      CK(sc->s_cvf_face.upload(s.cvf_face));
      CK(sc->s_on_face.upload(s.on_face));
      CK(sc->s_simp_cnt.alloc(nc));
      CK(sc->s_simp_face.alloc((size_t)nc * kMaxSelfImpacts));
      CK(sc->s_simp_td.alloc((size_t)nc * kMaxSelfImpacts * 2));
      CK(sc->s_simp_n.alloc((size_t)nc * kMaxSelfImpacts * 3));
      CK(sc->s_cf_face.alloc(nc)); CK(sc->s_cf_slot.alloc(nc)); CK(sc->s_m_slot.alloc(nc));
      CK(sc->s_g_cnt.alloc(ncf)); CK(sc->s_g_fill.alloc(ncf)); CK(sc->s_g_ptr.alloc((size_t)ncf + 1));
      CK(sc->s_g_mem.alloc(nc)); CK(sc->s_chit.alloc(nc));
      CK(sc->s_g_n.alloc(3 * (size_t)ncf)); CK(sc->s_g_outF.alloc(9 * (size_t)ncf)); CK(sc->s_g_outM.alloc(3 * (size_t)nc));
      CK(sc->s_sc_cur.alloc(3 * (size_t)nc)); CK(sc->s_rhs_pre.alloc(3 * (size_t)nc)); CK(sc->s_cnext.alloc(3 * (size_t)nc));
      CK(cudaMemset(sc->s_g_cnt.p, 0, sizeof(int) * ncf));
      CK(cudaMemset(sc->s_sc_cur.p, 0, sizeof(double) * 3 * (size_t)nc));
      ContactDev& c = sc->cd;
      c.ncf = ncf; c.mu_self = s.mu_self;
      c.cfaces = sc->s_cfaces.p; c.cvf_ptr = sc->s_cvf_ptr.p; c.cvf_face = sc->s_cvf_face.p; c.on_face = sc->s_on_face.p;
      c.simp_cnt = sc->s_simp_cnt.p; c.simp_face = sc->s_simp_face.p; c.simp_td = sc->s_simp_td.p;
      c.simp_n = sc->s_simp_n.p; c.cf_face = sc->s_cf_face.p; c.cf_slot = sc->s_cf_slot.p; c.m_slot = sc->s_m_slot.p;
      c.g_cnt = sc->s_g_cnt.p; c.g_fill = sc->s_g_fill.p; c.g_ptr = sc->s_g_ptr.p; c.g_mem = sc->s_g_mem.p;
      c.g_n = sc->s_g_n.p; c.g_outF = sc->s_g_outF.p; c.g_outM = sc->s_g_outM.p; c.sc_cur = sc->s_sc_cur.p;
      c.rhs_pre = sc->s_rhs_pre.p; c.cnext = sc->s_cnext.p; c.chit = sc->s_chit.p;
    }
  }
  if (s.L > 0) RC(upload_skeleton(sc));
  refresh_scene_view(sc);
  return DFEM_OK;
}

// Skeleton tables and the dense blocks of the Schur formulation
// (skeleton_kernels.cuh): Z = Hs^-1 E_R (the columns of Hs^-1 at the rigid
// vertices, three per host solve) and C^-1 = ((Hs^-1)_RR)^-1 = Hs_RR - Hs_RF
// Hs_FF^-1 Hs_FR (World.h:1134-1135), by a dense Cholesky of C on the host.
static int upload_skeleton(dfem_scene* sc) {
  const HostScene& s = sc->hs;
  const int N = s.N, L = s.L, nr = s.loff[L], ndof = 6 + L - 1;
  std::vector<SkelLink> lk(L);
  std::vector<int> rlink(nr), ridx(N, -1);
  int sdof = 12;
  for (int l = 0; l < L; ++l) {
    SkelLink& k = lk[l];
    std::memset(&k, 0, sizeof(k));
    k.parent = s.lparent[l];
    k.type = s.ltype[l];
    k.chan = s.lchan[l];
    k.dof = l == 0 ? 0 : 6 + l - 1;
    k.sdof = l == 0 ? 0 : sdof++;
    k.r0 = s.loff[l];
    k.r1 = s.loff[l + 1];
    for (int c = 0; c < 3; ++c) {
      k.joint[c] = s.ljoint[3 * l + c];
      k.axis[c] = s.laxis[3 * l + c];
      k.d0[c] = l == 0 ? k.joint[c] : k.joint[c] - s.ljoint[3 * k.parent + c];  // Link: d0 = joint - parent->joint
    }
    const double* a = k.axis;
    if (k.type == DFEM_JOINT_ROTATIONAL) {
      const double nx[9] = {0, -a[2], a[1], a[2], 0, -a[0], -a[1], a[0], 0};
      for (int i = 0; i < 9; ++i) { k.nx[i] = nx[i]; k.nnt[i] = a[i / 3] * a[i % 3]; }
    }
    for (int j = k.r0; j < k.r1; ++j) { rlink[j] = l; ridx[s.lvert[j]] = j; }
  }
  // Z and C from the host factor (internal numbering, three columns per solve)
  std::vector<double> zcm((size_t)nr * N), C((size_t)nr * nr);
  {
    std::vector<double> b(3 * (size_t)N), x(3 * (size_t)N);
    for (int j0 = 0; j0 < nr; j0 += 3) {
      std::fill(b.begin(), b.end(), 0.0);
      for (int c = 0; c < 3 && j0 + c < nr; ++c) b[3 * (size_t)s.lvert[j0 + c] + c] = 1.0;
      host_solve(s.F, b.data(), x.data());
      for (int c = 0; c < 3 && j0 + c < nr; ++c)
        for (int i = 0; i < N; ++i) zcm[(size_t)(j0 + c) * N + i] = x[3 * (size_t)i + c];
    }
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < nr; ++j) C[(size_t)i * nr + j] = 0.5 * (zcm[(size_t)j * N + s.lvert[i]] + zcm[(size_t)i * N + s.lvert[j]]);
  }
  // C^-1 by Cholesky C = G G^T, then solving for the identity
  std::vector<double> G(C), cinv((size_t)nr * nr, 0.0);
  for (int i = 0; i < nr; ++i) {
    for (int j = 0; j <= i; ++j) {
      double v = G[(size_t)i * nr + j];
      for (int k = 0; k < j; ++k) v -= G[(size_t)i * nr + k] * G[(size_t)j * nr + k];
      if (i == j) {
        if (!(v > 0.0) || !std::isfinite(v)) return fail(DFEM_ERR_FACTOR, "skeleton: the rigid block of Hs^-1 is not positive definite");
        G[(size_t)i * nr + i] = std::sqrt(v);
      } else {
        G[(size_t)i * nr + j] = v / G[(size_t)j * nr + j];
      }
    }
  }
  for (int col = 0; col < nr; ++col) {
    std::vector<double> y(nr, 0.0);
    for (int i = 0; i < nr; ++i) {
      double v = i == col ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) v -= G[(size_t)i * nr + k] * y[k];
      y[i] = v / G[(size_t)i * nr + i];
    }
    for (int i = nr - 1; i >= 0; --i) {
      double v = y[i];
      for (int k = i + 1; k < nr; ++k) v -= G[(size_t)k * nr + i] * y[k];
      y[i] = v / G[(size_t)i * nr + i];
    }
    for (int i = 0; i < nr; ++i) cinv[(size_t)i * nr + col] = y[i];
  }
  CK(sc->sk_link.upload(lk));
  CK(sc->sk_st.alloc(L));
  CK(cudaMemset(sc->sk_st.p, 0, sizeof(SkelState) * L));
  CK(sc->sk_rv.upload(std::vector<int>(s.lvert.begin(), s.lvert.end())));
  CK(sc->sk_rlink.upload(rlink));
  CK(sc->sk_ridx.upload(ridx));
  CK(sc->sk_rest.upload(s.lrest));
  CK(sc->sk_cinv.upload(cinv));
  CK(sc->sk_zcm.upload(zcm));
  sc->sk_nq = 12 + L - 1;
  if (!sc->skel_on) {  // a new scene starts from the identity and zero magnitudes
    std::vector<double> q0(sc->sk_nq, 0.0);
    q0[0] = q0[4] = q0[8] = 1.0;
    CK(sc->sk_jq.upload(q0));
    CK(sc->sk_jqd.upload(q0));
  }
  CK(sc->sk_v0.alloc(3 * (size_t)nr)); CK(sc->sk_w.alloc(3 * (size_t)nr)); CK(sc->sk_rr.alloc(3 * (size_t)nr));
  CK(sc->sk_q.alloc(3 * (size_t)nr));
  CK(sc->sk_tv.alloc(3 * (size_t)nr * ndof)); CK(sc->sk_kt.alloc(3 * (size_t)nr * ndof));
  CK(sc->sk_sm.alloc((size_t)ndof * ndof)); CK(sc->sk_rhs.alloc(ndof)); CK(sc->sk_sol.alloc(ndof));
  CK(sc->sk_perm.alloc(ndof));
  const int nq = sc->sk_nq;
  if (!sc->sk_thb.p) {
    CK(sc->sk_thb.alloc(nq)); CK(sc->sk_sb.alloc(ndof)); CK(sc->sk_gjq.alloc(nq)); CK(sc->sk_gjqd.alloc(nq));
    CK(sc->sk_mu2.alloc(3 * (size_t)nr)); CK(sc->sk_mu3.alloc(ndof)); CK(sc->sk_dlt.alloc(3 * (size_t)nr));
    CK(sc->sk_jfin.alloc(2 * (size_t)nq));
  }
  sc->skd = SkelDev{L, ndof, nr, N, sc->sk_link.p, sc->sk_st.p, sc->sk_rv.p, sc->sk_rlink.p, sc->sk_ridx.p,
                    sc->sk_rest.p, sc->sk_cinv.p, sc->sk_zcm.p, sc->sk_jq.p, sc->sk_jqd.p, sc->sk_v0.p, sc->sk_w.p,
                    sc->sk_rr.p, sc->sk_q.p, sc->sk_tv.p, sc->sk_kt.p, sc->sk_sm.p, sc->sk_rhs.p, sc->sk_sol.p,
                    sc->sk_perm.p};
  skel_bind(sc);
  sc->skel_on = true;
  invalidate_graphs(sc);  // the graphs hold the view's pointers
  return DFEM_OK;
}

static int ensure_steps(dfem_scene* sc, int n_steps) {
  if (n_steps <= sc->cap_steps) return DFEM_OK;
  const HostScene& s = sc->hs;
  int cap = std::max(n_steps, 2 * sc->cap_steps);
  // the buffers below are reallocated in place: until all of them succeed the
  // scene has no per-step buffers (a failed allocation leaves cap_steps = 0,
  // so the next call allocates again) and no recorded forward
  sc->cap_steps = 0;
  sc->rec_steps = 0;
  invalidate_graphs(sc);
  const size_t n3 = 3 * (size_t)s.N;
  const int kc = std::max(1, s.checkpoint_every);
  const size_t nck = ((size_t)cap + kc - 1) / kc;  // one checkpoint per kc steps
  CK(sc->ckpt_x.alloc(n3 * nck));
  CK(sc->ckpt_v.alloc(n3 * nck));
  if (kc > 1 && !sc->seg_x.p) {
    CK(sc->seg_x.alloc(n3 * kc));
    CK(sc->seg_v.alloc(n3 * kc));
  }
  CK(sc->traj.alloc(n3 * cap));
  CK(sc->iters.alloc((size_t)cap * sc->hs.nparts));
  CK(sc->act_all.alloc((size_t)cap * std::max(1, s.nseg)));
  CK(sc->gact.alloc((size_t)cap * std::max(1, s.nseg)));
  CK(sc->cpasses.alloc(2 * (size_t)cap));
  const size_t rec = n3 * (size_t)(s.K + 1);
  const bool all = rec * (size_t)cap * sizeof(double) <= sc->adj_budget;
  CK(sc->hist.alloc(all ? rec * cap : rec));
  sc->hist_step = all ? (long long)rec : 0;
  CK(cudaMemset(sc->cpasses.p, 0, sizeof(int) * 2 * (size_t)cap));
  if (sc->has_contact && sc->cnp > 0) {
    CK(sc->c_psrc.alloc((size_t)cap * sc->cnp));
    sc->cd.psrc = sc->c_psrc.p;
  }
  if (sc->has_contact) {
    CK(sc->crec_meta.alloc(4 * (size_t)cap));
    sc->cd.rec_meta = sc->crec_meta.p;
  }
  if (sc->skel_on) {  // the links' history: every step's iterations (a few hundred doubles each)
    const size_t hs = (size_t)sc->sk_nq + sc->skd.ndof + 3 * (size_t)sc->skd.nr;
    CK(sc->sk_hist.alloc((size_t)cap * (s.K + 1) * hs));
    CK(sc->sk_jin.alloc((size_t)cap * 2 * sc->sk_nq));
    skel_bind(sc);
  }
  sc->cap_steps = cap;
  invalidate_graphs(sc);  // graphs hold the old pointers
  return DFEM_OK;
}

// The global solve Hs y = rhs: one persistent launch, or one launch per level
// and direction (the autotuned choice for the scene).
// One launch segment of the level-kernel solve in one direction (thr: CTA
// size of a CTA segment; warp segments run eight warps per CTA).
static void launch_segment(dfem_scene* sc, cudaStream_t st, const dfem_scene::LevelSeg& g, bool fwd, int thr,
                           Gate gate, const double* rhs, double* y) {
  if (g.warp) {
    const int nb = (g.count + 7) / 8;
    if (fwd) k_fwd_level<WarpGroup><<<nb, 256, g.shm_f, st>>>(sc->fd, g.begin, g.count, g.grp_f, gate, rhs, y);
    else k_bwd_level<WarpGroup><<<nb, 256, g.shm_b, st>>>(sc->fd, g.begin, g.count, g.grp_b, gate, y);
  } else {
    if (fwd) k_fwd_level<CtaGroup><<<g.count, thr, g.shm_f, st>>>(sc->fd, g.begin, g.count, 0, gate, rhs, y);
    else k_bwd_level<CtaGroup><<<g.count, thr, g.shm_b, st>>>(sc->fd, g.begin, g.count, 0, gate, y);
  }
}

static int n_levels(const dfem_scene* sc) { return (int)sc->lvl_ptr.size() - 1; }

static cudaError_t launch_cluster_solve(dfem_scene* sc, cudaStream_t st, Gate gate, const double* rhs, double* y) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kClusterCtas);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = sc->shm_cluster;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kClusterCtas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_solve_cluster, sc->fd, (int)sc->lvl_ptr.size() - 1, (const int*)sc->lvl_ptr_d.p,
                            (const int*)sc->lvl_warp_d.p, sc->shm_cluster_warp, gate, rhs, y);
}

static cudaError_t launch_resident_solve(dfem_scene* sc, cudaStream_t st, Gate gate, const double* rhs, double* y) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sc->res_ctas);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = sc->shm_res;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = sc->res_ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_solve_resident, sc->rdv, gate, rhs, y);
}

// Launch errors surface through cudaGetLastError, which every caller checks;
// the cluster launch's return value is also kept for the autotune, which drops
// the cluster form when the device refuses its launch.
static void enqueue_solve_cut(dfem_scene* sc, cudaStream_t st, Gate gate, const double* rhs, double* y, int c) {
  if (c == -3) {  // the dense-inverse form
    k_dense_solve<<<sc->dense_grid, kDenseSolveThreads, 3 * (size_t)sc->dd.Np * sizeof(double), st>>>(
        sc->dd, gate, rhs, y);
    return;
  }
  if (c < 0) {  // -1: cluster form, -2: resident form
    const cudaError_t e = c == -2 ? launch_resident_solve(sc, st, gate, rhs, y) : launch_cluster_solve(sc, st, gate, rhs, y);
    if (e != cudaSuccess) sc->cluster_launch_err = e;
    return;
  }
  for (const auto& g : sc->segs)
    if (g.level < c) launch_segment(sc, st, g, true, g.thr_f, gate, rhs, y);
  if (c < n_levels(sc)) {
    const int p0 = sc->lvl_ptr[c];
    const int grid = std::max(1, std::min(sc->pers_slots, 2 * (sc->hs.F.nsuper - p0)));
    k_solve_persistent<<<grid, 256, sc->shm_pers, st>>>(sc->fd, p0, gate, rhs, y);
  }
  for (auto it = sc->segs.rbegin(); it != sc->segs.rend(); ++it)
    if (it->level < c) launch_segment(sc, st, *it, false, it->thr_b, gate, rhs, y);
}

static void enqueue_solve(dfem_scene* sc, cudaStream_t st, Gate gate, const double* rhs, double* y) {
  enqueue_solve_cut(sc, st, gate, rhs, y, sc->solve_cut);
}

static int solve_launches_cut(const dfem_scene* sc, int c) {
  if (c < 0) return 1;
  int n = c < n_levels(sc) ? 1 : 0;
  for (const auto& g : sc->segs) n += g.level < c ? 2 : 0;
  return n;
}
static int solve_launches(const dfem_scene* sc) { return solve_launches_cut(sc, sc->solve_cut); }

// The solve inside a loop body being captured on st.  With the per-iteration
// choice on: a selection kernel, then a conditional IF/ELSE node whose
// branches hold the tuned form and the persistent form (captured on stream3).
// which: 0 forward, 1 adjoint (its counter of persistent iterations).
static cudaError_t capture_solve(dfem_scene* sc, cudaStream_t st, Gate gate, const double* rhs, double* y, int which) {
  if (!sc->solve_select || sc->solve_cut == 0) {
    enqueue_solve(sc, st, gate, rhs, y);
    return cudaGetLastError();
  }
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  cudaGraph_t cg = nullptr;
  cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd);
  cudaGraphConditionalHandle h{};
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return e;
  k_solve_select<<<1, 256, 0, st>>>(gate, sc->part_w.p, sc->hs.nparts, sc->select_w, sc->sel_count.p + which, h);
  e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeIf;
  p.conditional.size = 2;  // [0] condition true, [1] else
  cudaGraphNode_t cn = nullptr;
  e = cudaGraphAddNode(&cn, cg, deps, nd, &p);
  if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies);
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    e = cudaStreamBeginCaptureToGraph(sc->stream3, p.conditional.phGraph_out[b], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) break;
    enqueue_solve_cut(sc, sc->stream3, gate, rhs, y, b == 0 ? sc->solve_cut : 0);
    cudaGraph_t tmp;
    const cudaError_t e2 = cudaStreamEndCapture(sc->stream3, &tmp);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = e2;
  }
  // the body's node count sees the select kernel and the IF node: count the
  // tuned branch's kernels instead of the IF node, and what the other has fewer
  sc->cur_alt_less = (size_t)(solve_launches_cut(sc, sc->solve_cut) - solve_launches_cut(sc, 0));
  return e;
}

// 1: level kernels, 2: persistent, 3: split, 4: cluster, 5: resident, 6: dense inverse
static int solve_form(const dfem_scene* sc) {
  return sc->solve_cut == -3 ? 6 : sc->solve_cut == -2 ? 5 : sc->solve_cut < 0 ? 4
       : sc->solve_cut >= n_levels(sc) ? 1 : sc->solve_cut == 0 ? 2 : 3;
}

// Fresh completion stamps and control words of the persistent solve (each API
// call starts from them, whatever an earlier call left behind).
static void reset_solve_state(dfem_scene* sc) {
  k_solve_reset<<<std::max(1, std::min(256, (sc->hs.F.nsuper + 255) / 256)), 256, 0, sc->stream>>>(
      sc->hs.F.nsuper, sc->done_f.p, sc->done_b.p, sc->solve_ctl.p);
}

// A time step (and the adjoint of one) is a CUDA graph: pre-loop kernels, a
// conditional WHILE node whose body is one PD iteration, post-loop kernels.
// The body's last kernel advances a device-side iteration counter and sets
// the loop condition, so converged steps launch no further iterations and no
// host round trip is needed.
static const Gate kOpen{};

// Per-part gates of a batch (a single scene's loops never run a gated-off
// iteration, so it takes the open gate and saves the lookups).
static Gate fwd_gate(const dfem_scene* sc) {
  Gate g;
  if (sc->hs.nparts > 1) { g.flag = sc->flag.p; g.nparts = sc->hs.nparts; }
  return g;
}
static Gate adj_gate(const dfem_scene* sc) {
  Gate g;
  if (sc->hs.nparts > 1) {
    g.iters = sc->iters.p; g.step = sc->step.p; g.kptr = sc->kiter.p; g.nparts = sc->hs.nparts;
  }
  return g;
}

// The local step and its gather in the scene's precision form.  The plain
// form writes J d slots and forms c0 + sum (the reference's delta form); the
// mixed form writes FP32 force slots (J d - L x) and forms the iterate-relative
// rhs (k_gather_force).  Both use the same slot buffer (the mixed form half of
// it).  The contact phase and dfem_eval_local always use the plain kernels.
static bool mixed(const dfem_scene* sc) { return sc->hs.precision == DFEM_PREC_MIXED; }
static float* slot32(dfem_scene* sc) { return reinterpret_cast<float*>(sc->slot.p); }

static void launch_local(dfem_scene* sc, cudaStream_t st, Gate g, const double* x, const double* act, const int* step,
                         bool plain = false) {
  const HostScene& s = sc->hs;
  const int ncons = s.T + s.M + s.S + s.B;
  if (ncons == 0) return;
  if (mixed(sc) && !plain)
    k_force_f32<<<(ncons + 127) / 128, 128, 0, st>>>(sc->sd, g, x, act, step, slot32(sc));
  else
    k_local<<<(ncons + 127) / 128, 128, 0, st>>>(sc->sd, g, x, act, step, sc->slot.p);
}

// rhs of one PD iteration at the iterate x (mixed: also reads q_n and x)
// the slot sums one thread per vertex (large scenes) or one warp per vertex
// (small ones, latency-bound); the sums are the same bit for bit
static bool gather_threads(const dfem_scene* sc) {
  return sc->gather_form == 2 || (sc->gather_form == 0 && sc->hs.N >= kGatherThreadMin);
}

static void launch_gather(dfem_scene* sc, cudaStream_t st, Gate g, const double* c0, double* rhs, const double* x,
                          bool plain = false) {
  if (mixed(sc) && !plain)
    k_gather_force<<<sc->nblk_v, 128, 0, st>>>(sc->sd, g, slot32(sc), sc->qn.p, x, rhs);
  else if (gather_threads(sc))
    k_gather_t<<<sc->nblk_v, 128, 0, st>>>(sc->hs.N, g, sc->vpart.p, sc->vslot_ptr.p, sc->slot.p, c0, rhs);
  else
    k_gather<<<(sc->hs.N + 3) / 4, 128, 0, st>>>(sc->hs.N, g, sc->vpart.p, sc->vslot_ptr.p, sc->slot.p, c0, rhs);
}

// The adjoint of the local step runs in FP64 in both forms.  (An FP32 VJP with
// the parameter terms taken from the rotated-frame deviations md - F cut the
// adjoint local step from 1.14 to 0.73 ms on the 256-scene batch, 1.5 % of the
// batch step, but raised the activation-gradient error from 2e-7 to 1.5e-4.)
static void launch_adj_local(dfem_scene* sc, cudaStream_t st, Gate g, const int* kptr) {
  const HostScene& s = sc->hs;
  const int nthr = std::max(s.T + s.M + s.S + s.B, s.N);
  k_adj_local<<<(nthr + 127) / 128, 128, 0, st>>>(sc->sd, g, kptr, sc->step.p, sc->hist.p, sc->hist_step, sc->y.p, sc->bb.p,
                                            sc->act_all.p, sc->slot.p, sc->gE.p, sc->gnu.p, sc->mg.p);
}

static void launch_adj_gather(dfem_scene* sc, cudaStream_t st, Gate g) {
  if (gather_threads(sc))
    k_adj_gather_t<<<sc->nblk_v, 128, 0, st>>>(sc->hs.N, g, sc->vpart.p, sc->vslot_ptr.p, sc->slot.p, sc->xkb.p);
  else
    k_adj_gather<<<(sc->hs.N + 3) / 4, 128, 0, st>>>(sc->hs.N, g, sc->vpart.p, sc->vslot_ptr.p, sc->slot.p, sc->xkb.p);
}

static void step_pre(dfem_scene* sc, cudaStream_t st, cudaGraphConditionalHandle h) {
  if (sc->self_contact) k_self_clear<<<(3 * sc->cd.nc + 127) / 128, 128, 0, st>>>(sc->cd);
  if (sc->nF > 0) k_drag_faces<<<(sc->nF + 127) / 128, 128, 0, st>>>(sc->nF, sc->df.p, sc->xt.p, sc->vt.p, sc->fdrag.p);
  k_step_begin<<<sc->nblk_p, kPartBlock, 0, st>>>(sc->sd, sc->pd, sc->step.p, sc->xt.p, sc->vt.p, sc->qn.p, sc->c0.p, sc->xk.p,
                                   sc->hist.p, sc->hist_step, std::max(1, sc->hs.checkpoint_every), sc->ckpt_x.p,
                                   sc->ckpt_v.p, sc->flag.p, sc->iters.p,
                                   sc->partial.p, sc->counter.p, sc->errv.p, sc->status.p,
                                   sc->has_contact ? sc->vwc.p : nullptr);
  if (sc->skel_on) k_skel_begin<<<1, 128, 0, st>>>(sc->skd, sc->xk.p, sc->step.p, sc->hist.p, sc->hist_step);
  k_loop_enter<<<1, 256, 0, st>>>(sc->kiter.p, sc->flag.p, sc->hs.nparts, sc->hs.K, h);
}

// obstacle contact phase (second conditional loop of the step graph)
static void contact_pre(dfem_scene* sc, cudaStream_t st, cudaGraphConditionalHandle h) {
  const int n = std::max(sc->hs.N, sc->cd.nc);
  if (sc->cnp > 0) {  // a batch: per-part state machines
    k_cparts_begin<<<(n + 127) / 128, 128, 0, st>>>(sc->sd, sc->cd, sc->xt.p, sc->xk.p, h);
    return;
  }
  k_contact_begin<<<(n + 127) / 128, 128, 0, st>>>(sc->sd, sc->cd, sc->xt.p, sc->xk.p, h);
}

static void contact_body(dfem_scene* sc, cudaStream_t st, cudaGraphConditionalHandle h) {
  const HostScene& s = sc->hs;
  const int nb = sc->nblk_v;
  const int ncons = s.T + s.M + s.S + s.B;
  if (sc->cnp > 0) {  // a batch: one round of every part's state machine
    const int nca = (sc->cd.nc + 127) / 128;
    k_cparts_detect<<<nca, 128, 0, st>>>(sc->cd, sc->xt.p, sc->xk.p, sc->status.p);
    k_cparts_ctl_detect<<<1, 256, 0, st>>>(sc->cd, sc->status.p);
    k_cparts_prep<<<sc->nblk_p, kPartBlock, 0, st>>>(sc->pd, sc->cd, sc->xk.p);
    k_cparts_record<<<nca, 128, 0, st>>>(sc->cd);
    k_cparts_ctl_conv<<<1, 256, 0, st>>>(sc->cd);
    Gate run;
    run.flag = sc->c_pst.p + (size_t)PS_SKIP * sc->cnp;
    if (ncons > 0)
      k_local<<<(ncons + 127) / 128, 128, 0, st>>>(sc->sd, run, sc->xk.p, sc->act_all.p, sc->step.p, sc->slot.p);
    k_cparts_rhs<<<nb, 128, 0, st>>>(sc->sd, sc->pd, sc->cd, sc->slot.p, sc->xt.p, sc->xk.p);
    k_cparts_ctl_iter<<<1, 256, 0, st>>>(sc->cd, s.K, sc->status.p, h);
    return;
  }
  k_contact_detect<<<(sc->cd.nc + 127) / 128, 128, 0, st>>>(sc->cd, sc->xt.p, sc->xk.p, sc->status.p);
  const int ncf = sc->cd.ncf;
  if (sc->self_contact) {  // soft impacts, then the pass's self groups
    k_self_detect<<<(int)(((int64_t)sc->cd.nc * 32 + 127) / 128), 128, 0, st>>>(sc->cd, sc->xt.p, sc->xk.p, sc->status.p);
    k_self_reset<<<(ncf + 127) / 128, 128, 0, st>>>(sc->cd);
    k_self_closest<<<(sc->cd.nc + 127) / 128, 128, 0, st>>>(sc->cd);
    k_self_scan<<<1, 1024, 0, st>>>(sc->cd);
    k_self_fill<<<(sc->cd.nc + 127) / 128, 128, 0, st>>>(sc->cd);
    k_self_sort<<<(ncf + 127) / 128, 128, 0, st>>>(sc->cd, sc->status.p);
  }
  k_contact_ctl_detect<<<1, 1, 0, st>>>(sc->cd, h);
  k_contact_prep<<<nb, 128, 0, st>>>(s.N, sc->cd, sc->xk.p, sc->partial.p, sc->counter.p);
  Gate active;
  active.active = sc->cstate.p + CS_ACTIVE;
  if (ncons > 0)
    k_local<<<(ncons + 127) / 128, 128, 0, st>>>(sc->sd, active, sc->xk.p, sc->act_all.p, sc->step.p, sc->slot.p);
  if (sc->self_contact) {
    k_contact_rhs_pre<<<nb, 128, 0, st>>>(sc->sd, sc->cd, sc->slot.p, sc->xt.p, sc->xk.p);
    k_self_record<<<(std::max(sc->cd.nc, ncf + 1) + 127) / 128, 128, 0, st>>>(sc->cd);
    k_self_exchange<<<(ncf + 127) / 128, 128, 0, st>>>(sc->cd);
    k_contact_rhs_post<<<(sc->cd.nc + 127) / 128, 128, 0, st>>>(sc->sd, sc->cd, sc->xt.p, sc->xk.p);
  } else {
    k_contact_rhs<<<nb, 128, 0, st>>>(sc->sd, sc->cd, sc->slot.p, sc->xt.p, sc->xk.p);
  }
  k_contact_ctl_iter<<<1, 1, 0, st>>>(sc->cd, s.K);
}

static void step_body(dfem_scene* sc, cudaStream_t st, cudaGraphConditionalHandle h) {
  const HostScene& s = sc->hs;
  const Gate g = fwd_gate(sc);
  launch_local(sc, st, g, sc->xk.p, sc->act_all.p, sc->step.p);
  launch_gather(sc, st, g, sc->c0.p, sc->rhs.p, sc->xk.p);
  const cudaError_t ce = capture_solve(sc, st, g, sc->rhs.p, sc->y.p, 0);
  if (ce != cudaSuccess) sc->cur_capture_err = ce;
  if (sc->skel_on) {  // the links' system, then the free vertices' share of the rigid multiplier
    k_skel_stage<<<1, 256, 0, st>>>(sc->skd, sc->xt.p, sc->y.p, sc->act_all.p, sc->step.p, s.nseg, sc->kiter.p);
    k_skel_apply<<<sc->nblk_v, 128, 0, st>>>(sc->skd, sc->y.p);
  }
  k_update<<<sc->nblk_p, kPartBlock, 0, st>>>(s.N, sc->pd, mixed(sc) ? 1 : 0, sc->kiter.p, sc->xt.p, sc->y.p, sc->xk.p, sc->hist.p, sc->hist_step, sc->step.p,
                               sc->flag.p, sc->iters.p, sc->partial.p, sc->counter.p, sc->errv.p, sc->status.p);
  k_loop_ctl<<<1, 256, 0, st>>>(sc->kiter.p, sc->flag.p, s.nparts, s.K, h);
}

static bool fused_contact(const dfem_scene* sc) { return sc->has_contact && sc->fused_ok && sc->fused_on; }

// The obstacle contact phase of the step as one cooperative launch.
static cudaError_t launch_contact_fused(dfem_scene* sc, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sc->fused_grid);
  cfg.blockDim = dim3(128);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (sc->cnp > 0) {
    cfg.dynamicSmemBytes = sizeof(int) * PS_SIZE * (size_t)sc->cnp;
    return cudaLaunchKernelEx(&cfg, k_contact_fused_parts, sc->sd, sc->cd, (const double*)sc->xt.p, sc->xk.p,
                              (const double*)sc->act_all.p, (const int*)sc->step.p, sc->slot.p, sc->status.p);
  }
  return cudaLaunchKernelEx(&cfg, k_contact_fused, sc->sd, sc->cd, (const double*)sc->xt.p, sc->xk.p,
                            (const double*)sc->act_all.p, (const int*)sc->step.p, sc->slot.p, sc->fpartial.p,
                            sc->status.p);
}

static void step_post(dfem_scene* sc, cudaStream_t st) {
  const int nb = sc->nblk_v;
  if (fused_contact(sc)) launch_contact_fused(sc, st);  // a refused launch surfaces through cudaGetLastError
  if (sc->has_contact) k_contact_record<<<1, 1, 0, st>>>(sc->step.p, sc->cstate.p, sc->cpasses.p, sc->cd);
  if (sc->has_contact && sc->cnp > 0) k_contact_record_parts<<<1, 256, 0, st>>>(sc->step.p, sc->cd);
  if (sc->skel_on) k_skel_end<<<1, 32, 0, st>>>(sc->skd);
  k_step_end<<<nb, 128, 0, st>>>(sc->sd, sc->step.p, sc->xt.p, sc->vt.p, sc->xk.p, sc->traj.p, sc->to_user.p,
                                 sc->write_traj.p);
  k_next_step<<<1, 1, 0, st>>>(sc->step.p);
}

static void adj_pre(dfem_scene* sc, cudaStream_t st, cudaGraphConditionalHandle h) {
  const HostScene& s = sc->hs;
  // the cotangent of the step's output lives in io_a (x) / io_b (v); k_adj_end overwrites it with the input's
  k_adj_begin<<<sc->nblk_v, 128, 0, st>>>(s.N, s.damping / s.h, sc->io_a.p, sc->io_b.p, sc->xkb.p, sc->xtb.p, sc->bb.p);
  k_adj_loop_enter<<<1, 256, 0, st>>>(sc->kiter.p, sc->iters.p, sc->step.p, s.nparts, s.K, h);
  if (sc->skel_on) {  // theta-bar of the last iterate: the output jq's cotangent and its rigid rows' V0
    k_skel_adj_init<<<1, 32, 0, st>>>(sc->skd);
    k_skel_adj_theta<<<sc->sk_nq, kSkelAdjThreads, 0, st>>>(sc->skd, sc->kiter.p, sc->step.p, 1, 0, sc->xkb.p);
  }
}

static void adj_body(dfem_scene* sc, cudaStream_t st, cudaGraphConditionalHandle h) {
  const HostScene& s = sc->hs;
  const Gate g = adj_gate(sc);
  if (sc->skel_on) k_skel_adj_upd<<<1, 64, 0, st>>>(sc->skd, sc->kiter.p, sc->step.p, sc->xkb.p);
  const cudaError_t ce = capture_solve(sc, st, g, sc->xkb.p, sc->y.p, 1);
  if (ce != cudaSuccess) sc->cur_capture_err = ce;
  if (sc->skel_on) {  // the KKT adjoint of the rigid stage: y becomes mu1
    k_skel_adj_stage<<<1, 256, 0, st>>>(sc->skd, sc->kiter.p, sc->step.p, sc->y.p, sc->hist.p, sc->hist_step,
                                        sc->gact.p, s.nseg);
    k_skel_adj_apply<<<sc->nblk_v, 128, 0, st>>>(sc->skd, sc->y.p);
  }
  launch_adj_local(sc, st, g, sc->kiter.p);
  launch_adj_gather(sc, st, g);
  if (s.nseg > 0)
    k_seg_reduce<<<(s.nseg + 127) / 128, 128, 0, st>>>(s.nseg, s.M, g, sc->seg_part.p, sc->step.p, sc->seg_ptr.p,
                                                       sc->seg_mus.p, sc->mg.p, sc->gact.p);
  if (sc->skel_on) {  // the moduli's rigid-row term, then theta-bar^k
    if (s.T > 0) k_skel_adj_ecorr<<<(s.T + 127) / 128, 128, 0, st>>>(sc->sd, sc->skd, sc->y.p, sc->gE.p);
    k_skel_adj_theta<<<sc->sk_nq, kSkelAdjThreads, 0, st>>>(sc->skd, sc->kiter.p, sc->step.p, 0, 1, sc->xkb.p);
  }
  k_adj_loop_ctl<<<1, 1, 0, st>>>(sc->kiter.p, h);
}

static void adj_post(dfem_scene* sc, cudaStream_t st) {
  if (sc->skel_on) k_skel_adj_end<<<1, 64, 0, st>>>(sc->skd, sc->step.p, sc->xkb.p);
  k_adj_end<<<sc->nblk_v, 128, 0, st>>>(sc->sd, sc->xkb.p, sc->xtb.p, sc->bb.p, sc->io_a.p, sc->io_b.p);
}

using PreFn = void (*)(dfem_scene*, cudaStream_t, cudaGraphConditionalHandle);
using BodyFn = void (*)(dfem_scene*, cudaStream_t, cudaGraphConditionalHandle);
using PostFn = void (*)(dfem_scene*, cudaStream_t);

struct LoopStage {
  PreFn pre;
  BodyFn body;
};

// Graph = for each stage: pre kernels, then a conditional WHILE node with the
// stage's body; then the post kernels.  Each stage has its own condition handle.
static int build_loop_graph(dfem_scene* sc, const std::vector<LoopStage>& stages, PostFn post, LoopGraph* out) {
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  std::string where = "capture";
  std::vector<cudaGraph_t> bodies;
  std::vector<size_t> alt_less;
  cudaError_t e = cudaStreamBeginCaptureToGraph(sc->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (const LoopStage& stage : stages) {
      if (e != cudaSuccess) break;
      cudaStreamCaptureStatus st;
      const cudaGraphNode_t* deps = nullptr;
      size_t nd = 0;
      cudaGraph_t cg = nullptr;
      e = cudaStreamGetCaptureInfo(sc->stream, &st, nullptr, &cg, &deps, &nd);
      cudaGraphConditionalHandle h{};
      if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault);
      if (e != cudaSuccess) { where = "conditional handle"; break; }
      stage.pre(sc, sc->stream, h);
      e = cudaStreamGetCaptureInfo(sc->stream, &st, nullptr, &cg, &deps, &nd);
      cudaGraphNode_t cn = nullptr;
      cudaGraphNodeParams p{};
      if (e == cudaSuccess) {
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        e = cudaGraphAddNode(&cn, cg, deps, nd, &p);
        where = "add conditional node";
      }
      if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(sc->stream, &cn, 1, cudaStreamSetCaptureDependencies);
      if (e == cudaSuccess) {
        cudaGraph_t body_g = p.conditional.phGraph_out[0];
        bodies.push_back(body_g);
        e = cudaStreamBeginCaptureToGraph(sc->stream2, body_g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        where = "capture loop body";
        if (e == cudaSuccess) {
          sc->cur_alt_less = 0;
          sc->cur_capture_err = cudaSuccess;
          stage.body(sc, sc->stream2, h);
          cudaGraph_t tmp;
          const cudaError_t e2 = cudaStreamEndCapture(sc->stream2, &tmp);
          e = cudaGetLastError();
          if (e == cudaSuccess) e = sc->cur_capture_err;
          if (e == cudaSuccess) e = e2;
          alt_less.push_back(sc->cur_alt_less);
        }
      }
    }
    if (e == cudaSuccess) post(sc, sc->stream);
    cudaGraph_t done = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(sc->stream, &done);  // always leave capture mode
    if (e == cudaSuccess) e = e2;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) {
    size_t top = 0;
    cudaGraphGetNodes(g, nullptr, &top);
    out->outside = top - bodies.size();  // conditional nodes launch nothing themselves
    for (size_t k = 0; k < 2; ++k) {
      size_t inner = 0;
      if (k < bodies.size()) cudaGraphGetNodes(bodies[k], nullptr, &inner);
      // an IF node of the solve form: its tuned branch's kernels instead of the node
      if (k < alt_less.size() && alt_less[k] > 0)
        inner += (size_t)solve_launches(sc) - 1;
      (k == 0 ? out->body : out->body2) = inner;
    }
    out->alt_less = alt_less.empty() ? 0 : alt_less[0];
    e = cudaGraphInstantiate(&out->exec, g, 0);
    where = "instantiate";
  }
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(DFEM_ERR_CUDA, "loop graph (" + where + "): " + cudaGetErrorString(e));
  return DFEM_OK;
}

static int ensure_graphs(dfem_scene* sc) {
  if (!sc->g_step.exec) {
    std::vector<LoopStage> st{{step_pre, step_body}};
    if (sc->has_contact && !fused_contact(sc)) st.push_back({contact_pre, contact_body});
    RC(build_loop_graph(sc, st, step_post, &sc->g_step));
  }
  if (!sc->g_adj.exec) RC(build_loop_graph(sc, {{adj_pre, adj_body}}, adj_post, &sc->g_adj));
  return DFEM_OK;
}

static int copy_in(dfem_scene* sc, const double* src, size_t n, double* dst, int mem) {
  CK(cudaMemcpyAsync(dst, src, n * sizeof(double), mem == DFEM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     sc->stream));
  return DFEM_OK;
}
static int copy_out(dfem_scene* sc, const double* src, size_t n, double* dst, int mem) {
  CK(cudaMemcpyAsync(dst, src, n * sizeof(double), mem == DFEM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     sc->stream));
  return DFEM_OK;
}

// Record of the contact phase for its adjoint: room for `cap` computed Jacobi
// iterations; records 0 .. keep-1 survive a growth (the graphs hold the
// record's pointers: rebuilt when it grows).
static int ensure_contact_record(dfem_scene* sc, int cap, int keep = 0) {
  if (!sc->has_contact) return DFEM_OK;
  const HostScene& s = sc->hs;
  const size_t n3 = 3 * (size_t)s.N, nc = (size_t)sc->cd.nc, nn = nc * kMaxImpactsPerVertex * 3;
  // the reverse sweep's buffers (sizes fixed by the scene) first: a failed
  // allocation below then leaves the record as it was
  for (DBuf<double>* b : {&sc->ca_xn1b, &sc->ca_pb, &sc->ca_cxtb, &sc->ca_vwcb, &sc->ca_yb, &sc->ca_orib})
    if (!b->p) CK(b->alloc(n3));
  if (!sc->ca_hdb.p) CK(sc->ca_hdb.alloc(std::max(1, s.N)));
  if (sc->self_contact) {
    const int ncf = sc->cd.ncf;
    for (DBuf<double>* b : {&sc->ca_scb, &sc->ca_ptot, &sc->ca_sbp, &sc->ca_gPM})
      if (!b->p) CK(b->alloc(3 * nc));
    if (!sc->ca_gmM.p) CK(sc->ca_gmM.alloc(nc));
    if (!sc->ca_gPF.p) CK(sc->ca_gPF.alloc(9 * (size_t)ncf));
    if (!sc->ca_gmF.p) CK(sc->ca_gmF.alloc(3 * (size_t)ncf));
    if (!sc->ca_xout.p) CK(sc->ca_xout.alloc(n3));
  }
  if (cap <= sc->crec_cap) return DFEM_OK;
  keep = std::min(keep, sc->crec_cap);
  if (keep == 0 && sc->crec_cap > 0) {  // nothing to copy: release the old record before the new one is made
    sc->crec_x.alloc(0); sc->crec_prev.alloc(0); sc->crec_first.alloc(0); sc->crec_cnt.alloc(0); sc->crec_n.alloc(0);
    if (sc->self_contact) { sc->crec_si.alloc(0); sc->crec_sd.alloc(0); }
    sc->crec_cap = 0;
    sc->cd.rec_cap = 0;
    sc->cd.rec_x = sc->cd.rec_prev = sc->cd.rec_n = nullptr;
    sc->cd.rec_first = sc->cd.rec_cnt = nullptr;
    invalidate_graphs(sc);
  }
  DBuf<double> x, prev, nrm;
  DBuf<int> first, cnt;
  CK(x.alloc(n3 * cap));
  CK(prev.alloc(n3 * cap));
  const size_t fw = std::max(1, sc->cnp);  // pass flags per record: one per part in a batch
  CK(first.alloc(fw * cap));
  CK(cnt.alloc(nc * cap));
  CK(nrm.alloc(nn * cap));
  DBuf<int> rsi;
  DBuf<double> rsd;
  if (sc->self_contact) {
    const size_t si = self_rec_si_stride((int)nc, sc->cd.ncf), sd = self_rec_sd_stride((int)nc, sc->cd.ncf);
    CK(rsi.alloc(si * cap));
    CK(rsd.alloc(sd * cap));
    if (keep > 0) {
      CK(cudaMemcpyAsync(rsi.p, sc->crec_si.p, sizeof(int) * si * keep, cudaMemcpyDeviceToDevice, sc->stream));
      CK(cudaMemcpyAsync(rsd.p, sc->crec_sd.p, sizeof(double) * sd * keep, cudaMemcpyDeviceToDevice, sc->stream));
    }
  }
  if (keep > 0) {
    CK(cudaMemcpyAsync(x.p, sc->crec_x.p, sizeof(double) * n3 * keep, cudaMemcpyDeviceToDevice, sc->stream));
    CK(cudaMemcpyAsync(prev.p, sc->crec_prev.p, sizeof(double) * n3 * keep, cudaMemcpyDeviceToDevice, sc->stream));
    CK(cudaMemcpyAsync(first.p, sc->crec_first.p, sizeof(int) * fw * keep, cudaMemcpyDeviceToDevice, sc->stream));
    CK(cudaMemcpyAsync(cnt.p, sc->crec_cnt.p, sizeof(int) * nc * keep, cudaMemcpyDeviceToDevice, sc->stream));
    CK(cudaMemcpyAsync(nrm.p, sc->crec_n.p, sizeof(double) * nn * keep, cudaMemcpyDeviceToDevice, sc->stream));
    CK(cudaStreamSynchronize(sc->stream));
  }
  sc->crec_x.swap(x);
  sc->crec_prev.swap(prev);
  sc->crec_first.swap(first);
  sc->crec_cnt.swap(cnt);
  sc->crec_n.swap(nrm);
  if (sc->self_contact) {
    sc->crec_si.swap(rsi);
    sc->crec_sd.swap(rsd);
    sc->cd.rec_si = sc->crec_si.p;
    sc->cd.rec_sd = sc->crec_sd.p;
  }
  sc->crec_cap = cap;
  sc->cd.rec_cap = cap;
  sc->cd.rec_x = sc->crec_x.p;
  sc->cd.rec_prev = sc->crec_prev.p;
  sc->cd.rec_first = sc->crec_first.p;
  sc->cd.rec_cnt = sc->crec_cnt.p;
  sc->cd.rec_n = sc->crec_n.p;
  invalidate_graphs(sc);
  return DFEM_OK;
}

// Device bytes of one record (one computed Jacobi iteration of the contact phase).
static size_t contact_record_bytes(const dfem_scene* sc) {
  const size_t n3 = 3 * (size_t)sc->hs.N, nc = (size_t)sc->cd.nc;
  size_t b = sizeof(double) * 2 * n3 + sizeof(int) * (1 + nc) + sizeof(double) * nc * kMaxImpactsPerVertex * 3;
  if (sc->self_contact)
    b += sizeof(int) * self_rec_si_stride((int)nc, sc->cd.ncf) + sizeof(double) * self_rec_sd_stride((int)nc, sc->cd.ncf);
  return b;
}

static ContactAdj make_cadj(dfem_scene* sc) {
  ContactAdj a{sc->ca_xn1b.p, sc->ca_pb.p, sc->ca_hdb.p, sc->ca_cxtb.p, sc->ca_vwcb.p, sc->ca_yb.p, sc->ca_orib.p};
  if (sc->self_contact) {
    a.scb = sc->ca_scb.p; a.ptot = sc->ca_ptot.p; a.sbp = sc->ca_sbp.p; a.gPF = sc->ca_gPF.p;
    a.gPM = sc->ca_gPM.p; a.gmF = sc->ca_gmF.p; a.gmM = sc->ca_gmM.p; a.xout = sc->ca_xout.p;
  }
  return a;
}

// Reverse of step st's contact phase, from its record: the forward's (base,
// iterations, source from crec_meta_h) or, after the step graph re-ran the
// step with recording on, the replay's (base = rbase, the rest from the
// contact state).  In: io_a / io_b = cotangents of the step's x' and v'.
// Out: io_a = cotangent of the PD result (io_b = 0); the x_t and v_wc
// cotangents wait in ca_cxtb / ca_vwcb for k_cadj_finish after the PD adjoint.
static int contact_adjoint_step(dfem_scene* sc, int st, bool recorded, int rbase, const double* xt) {
  const HostScene& s = sc->hs;
  const size_t n3 = 3 * (size_t)s.N;
  const int nb = sc->nblk_v, ncons = s.T + s.M + s.S + s.B;
  int base = rbase, comp = 0, src = 0;
  if (recorded) {
    base = sc->crec_meta_h[4 * (size_t)st];
    comp = sc->crec_meta_h[4 * (size_t)st + 1];
    src = sc->crec_meta_h[4 * (size_t)st + 2];
  } else {
    int meta[CS_SIZE];
    CK(cudaMemcpyAsync(meta, sc->cstate.p, sizeof(meta), cudaMemcpyDeviceToHost, sc->stream));
    CK(cudaStreamSynchronize(sc->stream));
    comp = meta[CS_COMP];
    src = meta[CS_SRC];
  }
  if (base + comp > sc->crec_cap) return fail(DFEM_ERR_CAP, "contact record too small for the recomputed step");
  if (sc->cnp > 0 && !fused_contact(sc)) {  // a batch: every part's reverse sweep, a loop of gated kernels
    const int np = sc->cnp;
    const int* top = recorded ? sc->c_psrc.p + (size_t)st * np : sc->c_pst.p + (size_t)PS_SRC * np;
    std::vector<int> toph(np);
    CK(cudaMemcpyAsync(toph.data(), top, sizeof(int) * np, cudaMemcpyDeviceToHost, sc->stream));
    CK(cudaStreamSynchronize(sc->stream));
    const int jmax = *std::max_element(toph.begin(), toph.end());
    const ContactAdj a = make_cadj(sc);
    Gate g;
    g.flag = sc->c_pst.p + (size_t)PS_SKIP * np;
    k_cadj_start<<<nb, 128, 0, sc->stream>>>(s.N, s.damping / s.h, sc->io_a.p, sc->io_b.p, a, 0);
    int launches = 1;
    for (int j = jmax; j >= 1; --j) {
      const size_t r = (size_t)base + (j - 1);
      const double* ori = sc->crec_x.p + r * n3;
      const double* prev = sc->crec_prev.p + r * n3;
      const int* rcnt = sc->crec_cnt.p + r * sc->cd.nc;
      const double* rn = sc->crec_n.p + r * sc->cd.nc * kMaxImpactsPerVertex * 3;
      k_cparts_gate<<<1, 256, 0, sc->stream>>>(sc->cd, top, j);
      if (ncons > 0)
        k_local<<<(ncons + 127) / 128, 128, 0, sc->stream>>>(sc->sd, g, ori, sc->act_all.p, sc->step.p, sc->slot.p);
      k_cadj_rhs_parts<<<nb, 128, 0, sc->stream>>>(sc->sd, sc->cd, a, sc->slot.p, xt, ori, prev,
                                                   sc->crec_first.p + r * np, rcnt, rn);
      if (ncons > 0)
        k_cadj_local<<<(ncons + 127) / 128, 128, 0, sc->stream>>>(sc->sd, a, ori, xt, sc->act_all.p, sc->step.p,
                                                                  sc->slot.p, sc->gE.p, sc->gnu.p, sc->mg.p, g);
      k_adj_gather_seq<<<nb, 128, 0, sc->stream>>>(s.N, g, sc->vpart.p, sc->vslot_ptr.p, sc->slot.p, a.orib);
      if (s.nseg > 0)
        k_seg_reduce<<<(s.nseg + 127) / 128, 128, 0, sc->stream>>>(s.nseg, s.M, g, sc->seg_part.p, sc->step.p,
                                                                  sc->seg_ptr.p, sc->seg_mus.p, sc->mg.p, sc->gact.p);
      k_cadj_hs<<<nb, 128, 0, sc->stream>>>(sc->sd, a, g);
      launches += 5 + (ncons > 0 ? 2 : 0) + (s.nseg > 0 ? 1 : 0);
    }
    if (s.T > 0) k_cadj_hd<<<(s.T + 127) / 128, 128, 0, sc->stream>>>(sc->sd, a, sc->gE.p);
    k_cadj_to_pd<<<nb, 128, 0, sc->stream>>>(s.N, a, sc->io_a.p, sc->io_b.p);
    CK(cudaGetLastError());
    sc->launches += launches + 2;
    return DFEM_OK;
  }
  if (sc->cnp > 0) {  // a batch: every part's reverse sweep in one cooperative launch
    const ContactAdj a = make_cadj(sc);
    const int* top = recorded ? sc->c_psrc.p + (size_t)st * sc->cnp : sc->c_pst.p + (size_t)PS_SRC * sc->cnp;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(sc->cadj_grid);
    cfg.blockDim = dim3(128);
    cfg.stream = sc->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k_cadj_fused_parts, sc->sd, sc->cd, a, xt, (const double*)sc->act_all.p,
                          (const int*)sc->step.p, sc->slot.p, sc->gE.p, sc->gnu.p, sc->mg.p, sc->gact.p, base, top,
                          s.damping / s.h, sc->io_a.p, sc->io_b.p));
    sc->launches += 1;
    return DFEM_OK;
  }
  if (!sc->self_contact && fused_contact(sc)) {  // the whole reverse sweep in one cooperative launch
    const ContactAdj a = make_cadj(sc);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(sc->cadj_grid);
    cfg.blockDim = dim3(128);
    cfg.stream = sc->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k_cadj_fused, sc->sd, sc->cd, a, xt, (const double*)sc->act_all.p,
                          (const int*)sc->step.p, sc->slot.p, sc->gE.p, sc->gnu.p, sc->mg.p, sc->gact.p, base, src,
                          s.damping / s.h, sc->io_a.p, sc->io_b.p));
    sc->launches += 1;
    return DFEM_OK;
  }
  // soft contact: every computed iteration feeds the remembered self forces,
  // so the sweep starts at the last one and the output enters at its source;
  // the step's final remembered forces are zeroed before the next step reads
  // them (World.h:742-753), so their cotangent starts at zero
  const bool soft = sc->self_contact;
  if (soft) CK(cudaMemsetAsync(sc->ca_scb.p, 0, sizeof(double) * 3 * (size_t)sc->cd.nc, sc->stream));
  const int top = soft ? comp : src;
  std::vector<int> first(std::max(1, top));
  if (top > 0)
    CK(cudaMemcpy(first.data(), sc->crec_first.p + base, top * sizeof(int), cudaMemcpyDeviceToHost));
  const ContactAdj a = make_cadj(sc);
  k_cadj_start<<<nb, 128, 0, sc->stream>>>(s.N, s.damping / s.h, sc->io_a.p, sc->io_b.p, a, soft ? 1 : 0);
  int launches = 1;
  for (int j = top; j >= 1; --j) {
    if (soft) {
      if (j == src) {
        k_cadj_add_xout<<<nb, 128, 0, sc->stream>>>(s.N, a);
        ++launches;
      }
      const size_t r = (size_t)base + (j - 1);
      const double* ori = sc->crec_x.p + r * n3;
      const double* prev = sc->crec_prev.p + r * n3;
      const int* rcnt = sc->crec_cnt.p + r * sc->cd.nc;
      const double* rn = sc->crec_n.p + r * sc->cd.nc * kMaxImpactsPerVertex * 3;
      const SelfRec rv = self_rec_view(sc->cd, r);
      if (ncons > 0)
        k_local<<<(ncons + 127) / 128, 128, 0, sc->stream>>>(sc->sd, kOpen, ori, sc->act_all.p, sc->step.p, sc->slot.p);
      k_cadj_self_a<<<nb, 128, 0, sc->stream>>>(sc->sd, sc->cd, a, rv, sc->slot.p, xt, ori, prev, first[j - 1], rcnt, rn);
      k_cadj_self_group<<<(sc->cd.ncf + 127) / 128, 128, 0, sc->stream>>>(sc->cd, a, rv);
      k_cadj_self_b<<<(sc->cd.nc + 127) / 128, 128, 0, sc->stream>>>(sc->sd, sc->cd, a, rv, first[j - 1], rcnt, rn);
      if (ncons > 0)
        k_cadj_local<<<(ncons + 127) / 128, 128, 0, sc->stream>>>(sc->sd, a, ori, xt, sc->act_all.p, sc->step.p,
                                                                  sc->slot.p, sc->gE.p, sc->gnu.p, sc->mg.p, kOpen);
      k_adj_gather_seq<<<nb, 128, 0, sc->stream>>>(s.N, kOpen, sc->vpart.p, sc->vslot_ptr.p, sc->slot.p, a.orib);
      if (s.nseg > 0)
        k_seg_reduce<<<(s.nseg + 127) / 128, 128, 0, sc->stream>>>(s.nseg, s.M, kOpen, sc->seg_part.p, sc->step.p,
                                                                  sc->seg_ptr.p, sc->seg_mus.p, sc->mg.p, sc->gact.p);
      k_cadj_hs<<<nb, 128, 0, sc->stream>>>(sc->sd, a, kOpen);
      launches += 6 + (ncons > 0 ? 2 : 0) + (s.nseg > 0 ? 1 : 0);
      continue;
    }
    const size_t r = (size_t)base + (j - 1);
    const double* ori = sc->crec_x.p + r * n3;
    const double* prev = sc->crec_prev.p + r * n3;
    const int* rcnt = sc->crec_cnt.p + r * sc->cd.nc;
    const double* rn = sc->crec_n.p + r * sc->cd.nc * kMaxImpactsPerVertex * 3;
    if (ncons > 0)
      k_local<<<(ncons + 127) / 128, 128, 0, sc->stream>>>(sc->sd, kOpen, ori, sc->act_all.p, sc->step.p, sc->slot.p);
    k_cadj_rhs<<<nb, 128, 0, sc->stream>>>(sc->sd, sc->cd, a, sc->slot.p, xt, ori, prev, first[j - 1], rcnt, rn);
    if (ncons > 0)
      k_cadj_local<<<(ncons + 127) / 128, 128, 0, sc->stream>>>(sc->sd, a, ori, xt, sc->act_all.p, sc->step.p,
                                                                sc->slot.p, sc->gE.p, sc->gnu.p, sc->mg.p, kOpen);
    k_adj_gather_seq<<<nb, 128, 0, sc->stream>>>(s.N, kOpen, sc->vpart.p, sc->vslot_ptr.p, sc->slot.p, a.orib);
    if (s.nseg > 0)
      k_seg_reduce<<<(s.nseg + 127) / 128, 128, 0, sc->stream>>>(s.nseg, s.M, kOpen, sc->seg_part.p, sc->step.p,
                                                                sc->seg_ptr.p, sc->seg_mus.p, sc->mg.p, sc->gact.p);
    k_cadj_hs<<<nb, 128, 0, sc->stream>>>(sc->sd, a, kOpen);
    launches += 4 + (ncons > 0 ? 2 : 0) + (s.nseg > 0 ? 1 : 0);
  }
  if (soft && src == 0) {  // the output is the PD result itself
    k_cadj_add_xout<<<nb, 128, 0, sc->stream>>>(s.N, a);
    ++launches;
  }
  if (s.T > 0) k_cadj_hd<<<(s.T + 127) / 128, 128, 0, sc->stream>>>(sc->sd, a, sc->gE.p);
  k_cadj_to_pd<<<nb, 128, 0, sc->stream>>>(s.N, a, sc->io_a.p, sc->io_b.p);
  CK(cudaGetLastError());
  sc->launches += launches + 2;
  return DFEM_OK;
}

// The device status word: [code, supernode, which wait or check, blocks that gave up].
static int status_error(const int st4[4]) {
  static const char* const what[] = {"",
                                     "a staged-copy wait of the forward solve",
                                     "a staged-copy wait of the backward solve",
                                     "a dependency wait of the persistent forward solve",
                                     "a dependency wait of the persistent backward solve",
                                     "a streamed-block wait of the forward solve",
                                     "a streamed-block wait of the backward solve",
                                     "the resident solve's image copy",
                                     "a resident-solve contribution address check",
                                     "a resident-solve solution address check"};
  if (st4[0] == DFEM_ERR_CAP && st4[2] > 0 && st4[2] <= 9)
    return fail(DFEM_ERR_CAP, std::string(what[st4[2]]) + " gave up (supernode " + std::to_string(st4[1]) + ", " +
                                  std::to_string(st4[3]) + " blocks)");
  if (st4[0] == DFEM_ERR_CAP && st4[2] == kCapContactPasses)
    return fail(DFEM_ERR_CAP, "the contact phase still found new impacts after its last detection pass (pass cap)");
  if (st4[0] == DFEM_ERR_CAP && st4[2] == kCapImpacts)
    return fail(DFEM_ERR_CAP, "a contact vertex hit more obstacle faces than the impacts kept per vertex");
  if (st4[0] == DFEM_ERR_CAP && st4[2] == kCapSoftImpacts)
    return fail(DFEM_ERR_CAP, "a contact vertex hit more soft faces than the soft impacts kept per vertex");
  if (st4[0] == DFEM_ERR_CAP && st4[2] == kCapGroupMembers)
    return fail(DFEM_ERR_CAP, "a soft-contact face group has more members than the cap");
  if (st4[0] == DFEM_ERR_CAP) return fail(DFEM_ERR_CAP, "a bounded loop gave up (contact impacts per vertex)");
  if (st4[0]) return fail(DFEM_ERR_NONFINITE, "non-finite value in the PD iteration");
  return DFEM_OK;
}

// Batches: while the parts still iterating hold much of the work, the tuned
// form (level kernels below the cut) is fastest; with few left, the
// persistent form is (the level kernels launch every supernode's CTA to skip
// it).  Each form's time per solve is modelled as linear in the active
// weight w (the parts' shares of the factor's entries), between all parts
// active and only the largest one; the solve switches to the persistent form
// below the crossing.  Off for one scene or when the tuned form is the
// persistent one.
static int tune_solve_select(dfem_scene* sc) {
  const HostScene& s = sc->hs;
  sc->solve_select = false;
  invalidate_graphs(sc);
  if (s.nparts < 2 || sc->solve_cut == 0) return DFEM_OK;
  const SupernodalFactor& F = s.F;
  std::vector<double> w(s.nparts, 0.0);
  for (int q = 0; q < F.nsuper; ++q) {
    const int p = (int)(std::upper_bound(s.part_v0.begin(), s.part_v0.end(), F.sn_c0[q]) - s.part_v0.begin()) - 1;
    w[p] += (double)F.sn_w[q] * (F.sn_w[q] + F.sn_r[q]);
  }
  double tot = 0.0;
  for (double v : w) tot += v;
  for (double& v : w) v /= tot;
  const int big = (int)(std::max_element(w.begin(), w.end()) - w.begin());
  CK(sc->part_w.upload(w));
  if (!sc->sel_count.p) {
    CK(sc->sel_count.alloc(2));
    CK(cudaMemset(sc->sel_count.p, 0, 2 * sizeof(unsigned long long)));
    sc->sel_seen[0] = sc->sel_seen[1] = 0;
  }
  // a gate with only the largest part open
  std::vector<int> flags(s.nparts, 1);
  flags[big] = 0;
  DBuf<int> fl;
  CK(fl.upload(flags));
  Gate one;
  one.flag = fl.p;
  one.nparts = s.nparts;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto time_form = [&](int c, Gate g) -> double {
    for (int r = 0; r < 3; ++r) enqueue_solve_cut(sc, sc->stream, g, sc->rhs.p, sc->y.p, c);
    cudaEventRecord(e0, sc->stream);
    for (int r = 0; r < 10; ++r) enqueue_solve_cut(sc, sc->stream, g, sc->rhs.p, sc->y.p, c);
    cudaEventRecord(e1, sc->stream);
    float t = 0;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) return -1.0;
    sc->launches += 13 * (int64_t)solve_launches_cut(sc, c);
    return t / 10.0;
  };
  const double tc1 = time_form(sc->solve_cut, one), t01 = time_form(0, one);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaGetLastError());
  if (tc1 < 0 || t01 < 0) return fail(DFEM_ERR_CUDA, "solve-form selection timing failed");
  const double tcF = sc->solve_ms[sc->solve_cut == n_levels(sc) ? 0 : 2], t0F = sc->solve_ms[1];
  const double d1 = tc1 - t01, dF = tcF - t0F;  // tuned minus persistent: one part / all parts
  sc->select_ms[0] = tc1;
  sc->select_ms[1] = t01;
  if (d1 <= 0.0 || dF >= 0.0) return DFEM_OK;  // no crossing: the tuned form throughout
  const double f1 = w[big];
  sc->select_w = f1 + (1.0 - f1) * d1 / (d1 - dF);
  sc->solve_select = true;
  return DFEM_OK;
}

// Factors up to this many supernodes also try the cluster form.
constexpr int kClusterMaxSupernodes = 4096;

// Time the solve forms on this scene's factor (10 solves each after 3 warm-up
// solves): the CTA size of every level-kernel launch, then the level-kernel
// form, the persistent form and the split form at every cut level; keep the
// fastest, then tune the per-iteration selection of batches.
static int autotune_solve(dfem_scene* sc) {
  const size_t n3 = 3 * (size_t)sc->hs.N;
  CK(cudaMemsetAsync(sc->rhs.p, 0, n3 * sizeof(double), sc->stream));
  reset_solve_state(sc);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  // CTA size of every launch segment and direction: 64, 128 or 256 threads
  {
    const int cand[3] = {64, 128, 256};
    for (auto& g : sc->segs)
      for (int dir = 0; dir < 2; ++dir) {
        if (g.warp) continue;
        double best = 1e30;
        int pick = 256;
        for (int thr : cand) {
          auto launch = [&] { launch_segment(sc, sc->stream, g, dir == 0, thr, kOpen, sc->rhs.p, sc->y.p); };
          launch();
          cudaEventRecord(e0, sc->stream);
          for (int r = 0; r < 5; ++r) launch();
          cudaEventRecord(e1, sc->stream);
          CK(cudaEventSynchronize(e1));
          float t = 0;
          CK(cudaEventElapsedTime(&t, e0, e1));
          sc->launches += 6;
          if (t < best) { best = t; pick = thr; }
        }
        (dir == 0 ? g.thr_f : g.thr_b) = pick;
      }
  }
  const int reps = 10;
  auto time_cut = [&](int c, double* ms) -> int {
    sc->solve_cut = c;
    for (int r = 0; r < 3; ++r) enqueue_solve(sc, sc->stream, kOpen, sc->rhs.p, sc->y.p);
    cudaEventRecord(e0, sc->stream);
    for (int r = 0; r < reps; ++r) enqueue_solve(sc, sc->stream, kOpen, sc->rhs.p, sc->y.p);
    cudaEventRecord(e1, sc->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float t = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    if (e != cudaSuccess) return fail(DFEM_ERR_CUDA, std::string("solve autotune: ") + cudaGetErrorString(e));
    *ms = (double)t / reps;
    sc->launches += (int64_t)(reps + 3) * solve_launches(sc);
    return DFEM_OK;
  };
  const int L = n_levels(sc);
  int rc = time_cut(L, &sc->solve_ms[0]);
  if (rc == DFEM_OK) rc = time_cut(0, &sc->solve_ms[1]);
  sc->split_cut = 0;
  sc->solve_ms[2] = 0.0;
  for (int c = 1; c < L && rc == DFEM_OK; ++c) {
    double ms = 0.0;
    rc = time_cut(c, &ms);
    if (rc == DFEM_OK && (sc->split_cut == 0 || ms < sc->solve_ms[2])) {
      sc->split_cut = c;
      sc->solve_ms[2] = ms;
    }
  }
  // the cluster form: factors of few supernodes (one cluster walks them all)
  sc->solve_ms[3] = 0.0;
  if (rc == DFEM_OK && sc->cluster_ok && sc->hs.F.nsuper <= kClusterMaxSupernodes) {
    sc->cluster_launch_err = cudaSuccess;
    rc = time_cut(-1, &sc->solve_ms[3]);
    if (rc == DFEM_OK && sc->cluster_launch_err != cudaSuccess) rc = DFEM_ERR_CUDA;
    if (rc != DFEM_OK) {  // a launch the device refuses (cluster shape): not a candidate
      cudaGetLastError();
      sc->cluster_ok = false;
      sc->cluster_launch_err = cudaSuccess;
      sc->solve_ms[3] = 0.0;
      g_last_error.clear();  // the dropped candidate is not an error of the scene
      rc = DFEM_OK;
    }
  }
  // the resident form: single scenes whose factor fits one cluster's shared memory
  sc->solve_ms[4] = 0.0;
  if (rc == DFEM_OK && sc->res_ok) {
    sc->cluster_launch_err = cudaSuccess;
    rc = time_cut(-2, &sc->solve_ms[4]);
    if (rc == DFEM_OK && sc->cluster_launch_err != cudaSuccess) rc = DFEM_ERR_CUDA;
    if (rc != DFEM_OK) {  // a launch the device refuses: not a candidate
      cudaGetLastError();
      sc->res_ok = false;
      sc->cluster_launch_err = cudaSuccess;
      sc->solve_ms[4] = 0.0;
      g_last_error.clear();
      rc = DFEM_OK;
    }
  }
  // the dense-inverse form: single scenes up to kDenseMaxN vertices whose X
  // and workspace take at most an eighth of the free memory
  sc->solve_ms[5] = 0.0;
  sc->dense_build_ms = 0.0;
  {
    const size_t np = (size_t)((sc->hs.N + kDenseTile - 1) / kDenseTile) * kDenseTile;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    sc->dense_ok = sc->hs.nparts == 1 && sc->hs.N <= kDenseMaxN && 2 * np * np * sizeof(double) <= free_b / 8;
  }
  if (rc == DFEM_OK && sc->dense_ok) {
    int rb = dense_build(sc);  // allocates X and its workspace; the rebuild after a refactorisation is timed
    cudaEventRecord(e0, sc->stream);
    if (rb == DFEM_OK) rb = dense_build(sc);
    cudaEventRecord(e1, sc->stream);
    float tb = 0.0f;
    if (rb == DFEM_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&tb, e0, e1) != cudaSuccess))
      rb = DFEM_ERR_CUDA;
    sc->dense_build_ms = tb;
    if (rb == DFEM_OK) rb = time_cut(-3, &sc->solve_ms[5]);
    if (rb != DFEM_OK) {  // no room or a refused launch: not a candidate
      cudaGetLastError();
      g_last_error.clear();
      dense_release(sc);
      sc->solve_ms[5] = 0.0;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  RC(rc);
  int st4[4] = {0, 0, 0, 0};
  CK(cudaMemcpy(st4, sc->status.p, sizeof(st4), cudaMemcpyDeviceToHost));
  RC(status_error(st4));
  sc->solve_cut = sc->solve_ms[1] < sc->solve_ms[0] ? 0 : L;
  if (sc->split_cut > 0 && sc->solve_ms[2] < std::min(sc->solve_ms[0], sc->solve_ms[1])) sc->solve_cut = sc->split_cut;
  {
    double best = sc->solve_cut == 0 ? sc->solve_ms[1] : sc->solve_cut == L ? sc->solve_ms[0] : sc->solve_ms[2];
    if (sc->solve_ms[3] > 0.0 && sc->solve_ms[3] < best) { sc->solve_cut = -1; best = sc->solve_ms[3]; }
    if (sc->solve_ms[4] > 0.0 && sc->solve_ms[4] < best) { sc->solve_cut = -2; best = sc->solve_ms[4]; }
    if (sc->solve_ms[5] > 0.0 && (best - sc->solve_ms[5]) * kDenseAmortSolves > sc->dense_build_ms) sc->solve_cut = -3;
  }
  if (sc->solve_cut != -3 && sc->dn_A.p) dense_release(sc);
  RC(tune_solve_select(sc));
  invalidate_graphs(sc);
  return DFEM_OK;
}

// Device side of scene creation, once sc->hs (and sc->parts for a batch) is built.
static int create_on_device(std::unique_ptr<dfem_scene>& sc, int device, dfem_scene** out) {
  CK(cudaStreamCreate(&sc->stream));  // blocking: orders with the legacy default stream callers use
  CK(cudaStreamCreateWithFlags(&sc->stream2, cudaStreamNonBlocking));  // only used to capture loop bodies
  CK(cudaStreamCreateWithFlags(&sc->stream3, cudaStreamNonBlocking));
  CK(sc->kiter.alloc(1));
  CK(sc->status.alloc(4));  // before the factor upload, whose kernels report into it
  {
    // device memory the adjoint may fill with stored iterates and contact
    // records (each saves a replayed step): 45 % of the device, at most 60 %
    // of what is free when the scene is made.  The forward leaves room in the
    // record store for one replayed step, so the adjoint rarely grows it (a
    // growing store holds its old and new arrays at once; when that does not
    // fit, the adjoint drops the forward's records and replays every step).
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    sc->adj_budget = std::min(total_b / 100 * 45, free_b / 100 * 60);
  }
  RC(upload_scene(sc.get()));
  RC(ensure_steps(sc.get(), 1));
  // every factor the engine uses comes from the GPU refactorisation
  RC(upload_refactor_plan(sc.get()));
  if (sc->hs.T > 0) {
    CK(cudaMemcpyAsync(sc->E_in.p, sc->tE.p, sc->hs.T * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
    CK(cudaMemcpyAsync(sc->nu_in.p, sc->tnu.p, sc->hs.T * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
  }
  RC(gpu_refactor(sc.get()));
  CK(cudaMemsetAsync(sc->status.p, 0, 4 * sizeof(int), sc->stream));
  RC(autotune_solve(sc.get()));
  CK(cudaDeviceSynchronize());
  *out = sc.release();
  g_last_error.clear();
  return DFEM_OK;
}


}  // namespace dfem

extern "C" {

const char* dfem_last_error(void) { return g_last_error.c_str(); }
int dfem_abi_version(void) { return DFEM_ABI_VERSION; }

int dfem_scene_create(const dfem_scene_desc* desc, int device, dfem_scene** out) {
  if (!desc || !out) return fail(DFEM_ERR_INVALID, "null argument");
  *out = nullptr;
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(DFEM_ERR_INVALID, "device index out of range");
  CK(cudaSetDevice(device));
  std::unique_ptr<dfem_scene> sc(new dfem_scene());
  sc->device = device;
  std::string err;
  if (!build_host_scene(*desc, sc->hs, err))
    return fail(err.find("factor") != std::string::npos ? DFEM_ERR_FACTOR : DFEM_ERR_INVALID, err);
  if (!refactorize(sc->hs.Hs, sc->hs.F, err)) return fail(DFEM_ERR_FACTOR, err);
  return create_on_device(sc, device, out);
}

int dfem_scene_create_batch(const dfem_scene_desc* descs, int32_t n_scenes, int device, dfem_scene** out) {
  if (!descs || !out || n_scenes < 1) return fail(DFEM_ERR_INVALID, "null argument or n_scenes < 1");
  *out = nullptr;
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(DFEM_ERR_INVALID, "device index out of range");
  CK(cudaSetDevice(device));
  std::unique_ptr<dfem_scene> sc(new dfem_scene());
  sc->device = device;
  sc->parts.resize(n_scenes);
  std::vector<std::string> errs(n_scenes);
  std::vector<int> codes(n_scenes, DFEM_OK);
  parallel_for(n_scenes, [&](int i) {  // each part: preprocessing, ordering and factorisation
    if (!build_host_scene(descs[i], sc->parts[i], errs[i]))
      codes[i] = errs[i].find("factor") != std::string::npos ? DFEM_ERR_FACTOR : DFEM_ERR_INVALID;
    else if (!refactorize(sc->parts[i].Hs, sc->parts[i].F, errs[i]))
      codes[i] = DFEM_ERR_FACTOR;
  });
  for (int i = 0; i < n_scenes; ++i)
    if (codes[i]) return fail(codes[i], "scene " + std::to_string(i) + ": " + errs[i]);
  std::string err;
  if (!merge_parts(sc->parts, sc->hs, err)) return fail(DFEM_ERR_INVALID, err);
  return create_on_device(sc, device, out);
}

int dfem_batch_layout(const dfem_scene* sc, int32_t* n_parts, int32_t* vertex_offsets, int32_t* tet_offsets,
                      int32_t* segment_offsets) {
  if (!sc || !n_parts) return fail(DFEM_ERR_INVALID, "null argument");
  const HostScene& s = sc->hs;
  *n_parts = s.nparts;
  for (int p = 0; p <= s.nparts; ++p) {
    if (vertex_offsets) vertex_offsets[p] = s.part_v0[p];
    if (tet_offsets) tet_offsets[p] = s.part_t0[p];
    if (segment_offsets) segment_offsets[p] = s.part_seg0[p];
  }
  return DFEM_OK;
}

int dfem_scene_destroy(dfem_scene* scene) {
  if (!scene) return DFEM_OK;
  cudaSetDevice(scene->device);
  if (scene->stream) cudaStreamSynchronize(scene->stream);
  delete scene;
  return DFEM_OK;
}

int dfem_scene_get_info(const dfem_scene* sc, dfem_scene_info* info) {
  if (!sc || !info) return fail(DFEM_ERR_INVALID, "null argument");
  const HostScene& s = sc->hs;
  info->n_vertices = s.N; info->n_tets = s.T; info->n_attach = s.A; info->n_muscle = s.M;
  info->n_springs = s.S; info->n_bending = s.B;
  info->n_supernodes = s.F.nsuper; info->n_levels = s.F.nlevels; info->nnz_factor = s.F.nnz_factor;
  info->n_slots = s.nslots; info->device = sc->device;
  info->factor_regularisation = 0.0;
  for (double r : sc->part_reg_h) info->factor_regularisation = std::max(info->factor_regularisation, r);
  return DFEM_OK;
}

int dfem_set_materials(dfem_scene* sc, const double* youngs, const double* poisson, int mem) {
  if (!sc || !youngs || !poisson) return fail(DFEM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(sc->device));
  HostScene& s = sc->hs;
  const int T = s.T;
  CK(cudaStreamSynchronize(sc->stream));
  if (T > 0) {
    RC(copy_in(sc, youngs, T, sc->E_in.p, mem));
    RC(copy_in(sc, poisson, T, sc->nu_in.p, mem));
  }
  RC(gpu_refactor(sc));
  if (sc->has_contact)
    k_hs_diag<<<sc->nblk_v, 128, 0, sc->stream>>>(s.N, sc->hs_ptr.p, sc->hs_col.p, sc->hs_val.p, sc->hdiag.p);
  // the host factor is used after creation only by the skeleton's Schur
  // blocks: with links, the host copies of the moduli follow and it is
  // refactored for them (without, the call returns with the device work queued)
  if (sc->skel_on) {
    if (T > 0) {
      CK(cudaMemcpyAsync(s.tE.data(), sc->tE.p, T * sizeof(double), cudaMemcpyDeviceToHost, sc->stream));
      CK(cudaMemcpyAsync(s.tnu.data(), sc->tnu.p, T * sizeof(double), cudaMemcpyDeviceToHost, sc->stream));
    }
    CK(cudaStreamSynchronize(sc->stream));
    std::string err;
    const std::vector<double> E(s.tE), nu(s.tnu);
    if (!update_materials(s, E.data(), nu.data(), err)) return fail(DFEM_ERR_FACTOR, err);
    RC(upload_skeleton(sc));
  }
  sc->rec_steps = 0;  // the recorded forward used the old factor
  return DFEM_OK;
}

int dfem_set_joint_state(dfem_scene* sc, const double* jq, const double* jqd) {
  if (!sc || !jq || !jqd) return fail(DFEM_ERR_INVALID, "null argument");
  if (!sc->skel_on) return fail(DFEM_ERR_INVALID, "the scene has no skeleton");
  CK(cudaSetDevice(sc->device));
  CK(cudaStreamSynchronize(sc->stream));
  for (int i = 0; i < sc->sk_nq; ++i)
    if (!std::isfinite(jq[i]) || !std::isfinite(jqd[i])) return fail(DFEM_ERR_INVALID, "non-finite joint state");
  CK(cudaMemcpy(sc->sk_jq.p, jq, sizeof(double) * sc->sk_nq, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sc->sk_jqd.p, jqd, sizeof(double) * sc->sk_nq, cudaMemcpyHostToDevice));
  return DFEM_OK;
}

int dfem_get_joint_state(const dfem_scene* sc, double* jq, double* jqd) {
  if (!sc || !jq || !jqd) return fail(DFEM_ERR_INVALID, "null argument");
  if (!sc->skel_on) return fail(DFEM_ERR_INVALID, "the scene has no skeleton");
  CK(cudaSetDevice(sc->device));
  CK(cudaStreamSynchronize(sc->stream));
  CK(cudaMemcpy(jq, sc->sk_jq.p, sizeof(double) * sc->sk_nq, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(jqd, sc->sk_jqd.p, sizeof(double) * sc->sk_nq, cudaMemcpyDeviceToHost));
  return DFEM_OK;
}

int dfem_set_joint_state_grad(dfem_scene* sc, const double* gjq, const double* gjqd) {
  if (!sc || !gjq || !gjqd) return fail(DFEM_ERR_INVALID, "null argument");
  if (!sc->skel_on) return fail(DFEM_ERR_INVALID, "the scene has no skeleton");
  const int nq = sc->sk_nq;
  sc->sk_gout.assign(gjq, gjq + nq);
  sc->sk_gout.insert(sc->sk_gout.end(), gjqd, gjqd + nq);
  return DFEM_OK;
}

int dfem_get_joint_state_grad(const dfem_scene* sc, double* gjq, double* gjqd) {
  if (!sc || !gjq || !gjqd) return fail(DFEM_ERR_INVALID, "null argument");
  if (!sc->skel_on) return fail(DFEM_ERR_INVALID, "the scene has no skeleton");
  CK(cudaSetDevice(sc->device));
  CK(cudaStreamSynchronize(sc->stream));
  CK(cudaMemcpy(gjq, sc->sk_gjq.p, sizeof(double) * sc->sk_nq, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(gjqd, sc->sk_gjqd.p, sizeof(double) * sc->sk_nq, cudaMemcpyDeviceToHost));
  return DFEM_OK;
}

int dfem_set_activations(dfem_scene* sc, const double* act, int mem) {
  if (!sc || (!act && sc->hs.nseg > 0)) return fail(DFEM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(sc->device));
  if (sc->hs.nseg == 0) return DFEM_OK;
  RC(copy_in(sc, act, sc->hs.nseg, sc->act_cur.p, mem));
  CK(cudaStreamSynchronize(sc->stream));
  return DFEM_OK;
}

int dfem_step_forward(dfem_scene* sc, const double* x, const double* v, const double* act, int32_t n_steps,
                      double* x_out, double* v_out, double* traj_x, int mem) {
  if (!sc || !x || !v || !x_out || !v_out) return fail(DFEM_ERR_INVALID, "null argument");
  if (n_steps < 1) return fail(DFEM_ERR_INVALID, "n_steps must be >= 1");
  CK(cudaSetDevice(sc->device));
  RC(ensure_steps(sc, n_steps));
  const HostScene& s = sc->hs;
  const size_t n3 = 3 * (size_t)s.N;
  const int nseg = s.nseg;
  if (nseg > 0) {
    if (act) {
      RC(copy_in(sc, act, (size_t)n_steps * nseg, sc->act_all.p, mem));
    } else {
      for (int st = 0; st < n_steps; ++st)
        CK(cudaMemcpyAsync(sc->act_all.p + (size_t)st * nseg, sc->act_cur.p, nseg * sizeof(double), cudaMemcpyDeviceToDevice,
                           sc->stream));
    }
  }
  RC(copy_in(sc, x, n3, sc->io_a.p, mem));
  RC(copy_in(sc, v, n3, sc->io_b.p, mem));
  const int nb = sc->nblk_v;
  k_to_internal<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_internal.p, sc->io_a.p, sc->xt.p);
  k_to_internal<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_internal.p, sc->io_b.p, sc->vt.p);
  k_set_int<<<1, 1, 0, sc->stream>>>(sc->step.p, 0);
  k_set_int<<<1, 1, 0, sc->stream>>>(sc->write_traj.p, traj_x ? 1 : 0);
  CK(cudaMemsetAsync(sc->status.p, 0, 4 * sizeof(int), sc->stream));
  reset_solve_state(sc);
  // With every step's iterates stored, the contact steps also record their
  // contact iterations, in a row, within what the adjoint budget leaves: the
  // adjoint then replays none of them (a step that does not fit is replayed).
  bool fwd_rec = false;
  size_t rec_budget = 0;
  if (sc->has_contact) {
    const size_t hist_bytes = sizeof(double) * sc->hist.n;
    rec_budget = sc->hist_step != 0 && sc->adj_budget > hist_bytes
                     ? (sc->adj_budget - hist_bytes) / contact_record_bytes(sc) : 0;
    rec_budget = std::min<size_t>(rec_budget, INT32_MAX / 2);
    // the store: the forward's records plus room for the adjoint's replay of
    // one step (the most loop-body executions of a step in the last forward)
    const size_t tgt = sc->crec_target > 0 ? (size_t)sc->crec_target : 4 * (size_t)n_steps;
    const int total = (int)std::min<size_t>(rec_budget, tgt + (size_t)sc->crec_reserve);
    const int want = std::max(0, total - sc->crec_reserve);
    fwd_rec = want >= 1 && !sc->self_contact;  // soft-soft contact has no adjoint to record for
    if (fwd_rec) {
      const int rc = ensure_contact_record(sc, total);
      if (rc == DFEM_ERR_NOMEM) {  // no room to record: the adjoint replays the contact steps
        cudaGetLastError();
        g_last_error.clear();
        fwd_rec = false;
      } else {
        RC(rc);
      }
    }
    if (fwd_rec) {  // the forward's share of the store (the graphs hold it: rebuilt when it changes)
      const int fwd_cap = std::max(want, (int)std::min<size_t>((size_t)sc->crec_cap, rec_budget) - sc->crec_reserve);
      if (sc->cd.rec_fwd_cap != fwd_cap) {
        sc->cd.rec_fwd_cap = fwd_cap;
        invalidate_graphs(sc);
      }
    }
    const int on = fwd_rec ? 2 : 0;
    CK(cudaMemcpyAsync(sc->crec_on.p, &on, sizeof(int), cudaMemcpyHostToDevice, sc->stream));
    CK(cudaMemsetAsync(sc->crec_base.p, 0, sizeof(int), sc->stream));
    CK(cudaStreamSynchronize(sc->stream));  // `on` is a host local
  }
  CK(cudaGetLastError());
  RC(ensure_graphs(sc));
  for (int st = 0; st < n_steps; ++st) CK(cudaGraphLaunch(sc->g_step.exec, sc->stream));
  k_to_user<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_user.p, sc->xt.p, sc->io_a.p);
  k_to_user<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_user.p, sc->vt.p, sc->io_b.p);
  RC(copy_out(sc, sc->io_a.p, n3, x_out, mem));
  RC(copy_out(sc, sc->io_b.p, n3, v_out, mem));
  if (traj_x) RC(copy_out(sc, sc->traj.p, n3 * n_steps, traj_x, mem));
  int st4[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(st4, sc->status.p, sizeof(st4), cudaMemcpyDeviceToHost, sc->stream));
  const int np = s.nparts;
  std::vector<int> it_all((size_t)n_steps * np, 0);
  CK(cudaMemcpyAsync(it_all.data(), sc->iters.p, it_all.size() * sizeof(int), cudaMemcpyDeviceToHost, sc->stream));
  sc->rec_passes.assign(2 * (size_t)n_steps, 0);
  if (sc->has_contact)
    CK(cudaMemcpyAsync(sc->rec_passes.data(), sc->cpasses.p, 2 * n_steps * sizeof(int), cudaMemcpyDeviceToHost, sc->stream));
  int rec_used = 0;
  sc->crec_meta_h.assign(4 * (size_t)n_steps, 0);
  if (fwd_rec) {
    CK(cudaMemcpyAsync(sc->crec_meta_h.data(), sc->crec_meta.p, sizeof(int) * 4 * n_steps, cudaMemcpyDeviceToHost,
                       sc->stream));
    CK(cudaMemcpyAsync(&rec_used, sc->crec_base.p, sizeof(int), cudaMemcpyDeviceToHost, sc->stream));
  }
  unsigned long long sel[2] = {0, 0};
  if (sc->sel_count.p) CK(cudaMemcpyAsync(sel, sc->sel_count.p, sizeof(sel), cudaMemcpyDeviceToHost, sc->stream));
  CK(cudaStreamSynchronize(sc->stream));
  if (sc->sel_count.p) {  // iterations whose solve took the persistent form launched fewer kernels
    sc->launches -= (int64_t)((sel[0] - sc->sel_seen[0]) * sc->g_step.alt_less);
    sc->sel_seen[0] = sel[0];
  }
  sc->rec_iters.assign(n_steps, 0);
  for (int st = 0; st < n_steps; ++st)
    for (int p = 0; p < np; ++p) sc->rec_iters[st] = std::max(sc->rec_iters[st], it_all[(size_t)st * np + p]);
  sc->crec_fwd = fwd_rec;
  sc->crec_used = rec_used;
  if (fwd_rec) {  // the next forward asks for room for all of this one's records
    size_t need = 0;
    for (int st = 0; st < n_steps; ++st) need += (size_t)sc->crec_meta_h[4 * (size_t)st + 1];
    sc->crec_target = (int)std::min(rec_budget, std::max<size_t>(need + need / 8 + 16, (size_t)sc->crec_target));
  }
  if (sc->has_contact) {  // room the next forward leaves for one replayed step
    int most = 0;
    for (int st = 0; st < n_steps; ++st) most = std::max(most, sc->rec_passes[2 * (size_t)st + 1]);
    sc->crec_reserve = std::max(sc->crec_reserve, most + 1);
  }
  sc->launches += 7;
  for (int st = 0; st < n_steps; ++st)
    sc->launches += (int64_t)(sc->g_step.outside + (size_t)sc->rec_iters[st] * sc->g_step.body +
                              (size_t)sc->rec_passes[2 * st + 1] * sc->g_step.body2);
  sc->rec_steps = n_steps;
  RC(status_error(st4));
  return DFEM_OK;
}

int dfem_step_backward(dfem_scene* sc, const double* gx_out, const double* gv_out, double* gx, double* gv,
                       double* g_youngs, double* g_poisson, double* g_act, int mem) {
  if (!sc || !gx_out || !gv_out || !gx || !gv) return fail(DFEM_ERR_INVALID, "null argument");
  if (sc->rec_steps <= 0) return fail(DFEM_ERR_STATE, "dfem_step_backward needs a preceding dfem_step_forward");
  CK(cudaSetDevice(sc->device));
  const int nq = sc->sk_nq;
  // the joint state a replayed step starts from (restored to the forward's final one at the end)
  auto joint_state_at = [&](int st) -> int {
    CK(cudaMemcpyAsync(sc->sk_jq.p, sc->sk_jin.p + 2 * (size_t)st * nq, nq * sizeof(double), cudaMemcpyDeviceToDevice,
                       sc->stream));
    CK(cudaMemcpyAsync(sc->sk_jqd.p, sc->sk_jin.p + (2 * (size_t)st + 1) * nq, nq * sizeof(double),
                       cudaMemcpyDeviceToDevice, sc->stream));
    return DFEM_OK;
  };
  if (sc->skel_on) {
    CK(cudaMemcpyAsync(sc->sk_jfin.p, sc->sk_jq.p, nq * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
    CK(cudaMemcpyAsync(sc->sk_jfin.p + nq, sc->sk_jqd.p, nq * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
    if (sc->sk_gout.size() == 2 * (size_t)nq) {
      CK(cudaMemcpyAsync(sc->sk_gjq.p, sc->sk_gout.data(), nq * sizeof(double), cudaMemcpyHostToDevice, sc->stream));
      CK(cudaMemcpyAsync(sc->sk_gjqd.p, sc->sk_gout.data() + nq, nq * sizeof(double), cudaMemcpyHostToDevice,
                         sc->stream));
      CK(cudaStreamSynchronize(sc->stream));  // the host vector is released below
    } else {
      CK(cudaMemsetAsync(sc->sk_gjq.p, 0, nq * sizeof(double), sc->stream));
      CK(cudaMemsetAsync(sc->sk_gjqd.p, 0, nq * sizeof(double), sc->stream));
    }
    sc->sk_gout.clear();
  }
  // contact steps the forward recorded need no replay; the others are replayed
  // with recording on, into records after the forward's (room for the most
  // loop-body executions of any of them)
  int ccap = 0;
  bool any_contact = false;
  std::vector<char> recorded(std::max(1, sc->rec_steps), 0);
  for (int st = 0; st < sc->rec_steps && 2 * st + 1 < (int)sc->rec_passes.size(); ++st) {
    const bool c = sc->rec_passes[2 * st] > 0;
    any_contact = any_contact || c;
    recorded[st] = c && sc->crec_fwd && 4 * st + 3 < (int)sc->crec_meta_h.size() && sc->crec_meta_h[4 * st + 3] == 1;
    if (c && !recorded[st]) ccap = std::max(ccap, sc->rec_passes[2 * st + 1]);
  }
  int rbase = sc->crec_fwd ? sc->crec_used : 0;
  if (any_contact) {
    const int rc = ensure_contact_record(sc, rbase + std::max(1, ccap), rbase);
    if (rc == DFEM_ERR_NOMEM && rbase > 0) {
      // no room for the replays beside the forward's records: drop them, and
      // replay every contact step (same results, more time)
      cudaGetLastError();
      g_last_error.clear();
      rbase = 0;
      sc->crec_fwd = false;
      for (int st = 0; st < sc->rec_steps; ++st)
        if (recorded[st]) { recorded[st] = false; ccap = std::max(ccap, sc->rec_passes[2 * st + 1]); }
      RC(ensure_contact_record(sc, std::max(1, ccap), 0));
    } else {
      RC(rc);
    }
  }
  const HostScene& s = sc->hs;
  const size_t n3 = 3 * (size_t)s.N;
  const int nb = sc->nblk_v;
  // incoming cotangents -> internal order (staged through rhs / c0)
  RC(copy_in(sc, gx_out, n3, sc->rhs.p, mem));
  RC(copy_in(sc, gv_out, n3, sc->c0.p, mem));
  k_to_internal<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_internal.p, sc->rhs.p, sc->io_a.p);
  k_to_internal<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_internal.p, sc->c0.p, sc->io_b.p);
  CK(cudaMemsetAsync(sc->gE.p, 0, sizeof(double) * std::max(1, s.T), sc->stream));
  CK(cudaMemsetAsync(sc->gnu.p, 0, sizeof(double) * std::max(1, s.T), sc->stream));
  CK(cudaMemsetAsync(sc->gact.p, 0, sizeof(double) * (size_t)sc->rec_steps * std::max(1, s.nseg), sc->stream));
  k_set_int<<<1, 1, 0, sc->stream>>>(sc->write_traj.p, 0);
  CK(cudaMemsetAsync(sc->status.p, 0, 4 * sizeof(int), sc->stream));
  reset_solve_state(sc);
  RC(ensure_graphs(sc));
  if (any_contact) {
    k_set_int<<<1, 1, 0, sc->stream>>>(sc->crec_on.p, 1);
    k_set_int<<<1, 1, 0, sc->stream>>>(sc->crec_base.p, rbase);
  }
  // Checkpoints are kept every kc steps.  Working back one segment [s0, end)
  // at a time, the adjoint first regenerates the segment's start states from
  // its checkpoint (steps s0 .. end-2 forward again, no contact recording)
  // when anything below reads them: the replays (iterates not stored, or a
  // contact step not recorded), the contact adjoint and the drag adjoint.
  const int kc = std::max(1, s.checkpoint_every);
  const bool need_states = sc->hist_step == 0 || any_contact || sc->nF > 0;
  int seg0 = 0;
  auto sx = [&](int st) { return kc == 1 ? sc->ckpt_x.p + (size_t)st * n3 : sc->seg_x.p + (size_t)(st - seg0) * n3; };
  auto sv = [&](int st) { return kc == 1 ? sc->ckpt_v.p + (size_t)st * n3 : sc->seg_v.p + (size_t)(st - seg0) * n3; };
  std::vector<int> rerun(std::max(1, sc->rec_steps), 0);  // step graphs run again, per step (launch statistics)
  int recomputed = 0;
  for (int seg_end = sc->rec_steps; seg_end > 0; seg_end = seg0) {
    seg0 = ((seg_end - 1) / kc) * kc;
    if (kc > 1 && need_states) {
      CK(cudaMemcpyAsync(sc->xt.p, sc->ckpt_x.p + (size_t)(seg0 / kc) * n3, n3 * sizeof(double),
                         cudaMemcpyDeviceToDevice, sc->stream));
      CK(cudaMemcpyAsync(sc->vt.p, sc->ckpt_v.p + (size_t)(seg0 / kc) * n3, n3 * sizeof(double),
                         cudaMemcpyDeviceToDevice, sc->stream));
      if (any_contact) k_set_int<<<1, 1, 0, sc->stream>>>(sc->crec_on.p, 0);
      if (sc->skel_on) RC(joint_state_at(seg0));
      for (int q = seg0; q < seg_end; ++q) {
        CK(cudaMemcpyAsync(sc->seg_x.p + (size_t)(q - seg0) * n3, sc->xt.p, n3 * sizeof(double),
                           cudaMemcpyDeviceToDevice, sc->stream));
        CK(cudaMemcpyAsync(sc->seg_v.p + (size_t)(q - seg0) * n3, sc->vt.p, n3 * sizeof(double),
                           cudaMemcpyDeviceToDevice, sc->stream));
        if (q + 1 < seg_end) {
          k_set_int<<<1, 1, 0, sc->stream>>>(sc->step.p, q);
          CK(cudaGraphLaunch(sc->g_step.exec, sc->stream));
          rerun[q] += 1;
          ++recomputed;
        }
      }
      if (any_contact) k_set_int<<<1, 1, 0, sc->stream>>>(sc->crec_on.p, 1);
    }
    for (int st = seg_end - 1; st >= seg0; --st) {
      const bool contact_step = sc->has_contact && sc->rec_passes[2 * st] > 0;
      if (sc->hist_step == 0 || (contact_step && !recorded[st])) {
        // recompute the step's iterates from its start state (the step graph re-records the same values);
        // a contact step also records its contact iterations for the contact adjoint
        CK(cudaMemcpyAsync(sc->xt.p, sx(st), n3 * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
        CK(cudaMemcpyAsync(sc->vt.p, sv(st), n3 * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
        if (sc->skel_on) RC(joint_state_at(st));
        k_set_int<<<1, 1, 0, sc->stream>>>(sc->step.p, st);
        CK(cudaGraphLaunch(sc->g_step.exec, sc->stream));
        rerun[st] += 1;
        ++recomputed;
      }
      k_set_int<<<1, 1, 0, sc->stream>>>(sc->step.p, st);
      if (contact_step && recorded[st]) {  // the step's v_wc and L x_t, which a replay would have left behind
        if (sc->nF > 0)
          k_drag_faces<<<(sc->nF + 127) / 128, 128, 0, sc->stream>>>(sc->nF, sc->df.p, sx(st), sv(st), sc->fdrag.p);
        k_contact_step_inputs<<<nb, 128, 0, sc->stream>>>(sc->sd, sc->cd, sx(st), sv(st));
        sc->launches += 1 + (sc->nF > 0 ? 1 : 0);
      }
      if (contact_step) RC(contact_adjoint_step(sc, st, recorded[st] != 0, rbase, sx(st)));
      CK(cudaGraphLaunch(sc->g_adj.exec, sc->stream));
      if (contact_step) {
        const ContactAdj a = make_cadj(sc);
        k_cadj_finish<<<nb, 128, 0, sc->stream>>>(s.N, a, sc->io_a.p, sc->io_b.p);
        sc->launches += 1;
      }
      if (sc->nF > 0) {  // v_wc = v + h f_drag(x, v) / m: io_b holds the cotangent of v_wc here
        k_drag_adj_faces<<<(sc->nF + 127) / 128, 128, 0, sc->stream>>>(sc->nF, sc->df.p, sc->mass.p, s.h, sx(st), sv(st),
                                                                        sc->io_b.p, sc->fdrag_b.p);
        k_drag_adj_gather<<<nb, 128, 0, sc->stream>>>(s.N, sc->vf_ptr.p, sc->vf_face.p, sc->fdrag_b.p, sc->io_a.p,
                                                       sc->io_b.p);
        sc->launches += 2;
      }
    }
  }
  if (any_contact) k_set_int<<<1, 1, 0, sc->stream>>>(sc->crec_on.p, 0);
  if (sc->skel_on) {
    CK(cudaMemcpyAsync(sc->sk_jq.p, sc->sk_jfin.p, nq * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
    CK(cudaMemcpyAsync(sc->sk_jqd.p, sc->sk_jfin.p + nq, nq * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
  }
  sc->launches += 5;
  for (int st = 0; st < sc->rec_steps && st < (int)sc->rec_iters.size(); ++st)
    sc->launches += (int64_t)(1 + sc->g_adj.outside + (size_t)sc->rec_iters[st] * sc->g_adj.body);
  if (recomputed > 0)  // step graphs run again (iteration counts as recorded)
    for (int st = 0; st < sc->rec_steps && st < (int)sc->rec_iters.size(); ++st)
      if (rerun[st])
        sc->launches += (int64_t)rerun[st] * (int64_t)(1 + sc->g_step.outside + (size_t)sc->rec_iters[st] * sc->g_step.body +
                                  (size_t)sc->rec_passes[2 * st + 1] * sc->g_step.body2);
  k_to_user<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_user.p, sc->io_a.p, sc->rhs.p);
  k_to_user<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_user.p, sc->io_b.p, sc->c0.p);
  RC(copy_out(sc, sc->rhs.p, n3, gx, mem));
  RC(copy_out(sc, sc->c0.p, n3, gv, mem));
  if (g_youngs) RC(copy_out(sc, sc->gE.p, s.T, g_youngs, mem));
  if (g_poisson) RC(copy_out(sc, sc->gnu.p, s.T, g_poisson, mem));
  if (g_act && s.nseg > 0) RC(copy_out(sc, sc->gact.p, (size_t)sc->rec_steps * s.nseg, g_act, mem));
  int st4[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(st4, sc->status.p, sizeof(st4), cudaMemcpyDeviceToHost, sc->stream));
  unsigned long long sel[2] = {0, 0};
  if (sc->sel_count.p) CK(cudaMemcpyAsync(sel, sc->sel_count.p, sizeof(sel), cudaMemcpyDeviceToHost, sc->stream));
  CK(cudaStreamSynchronize(sc->stream));
  if (sc->sel_count.p) {  // replayed forward iterations and adjoint iterations that took the persistent form
    sc->launches -= (int64_t)((sel[0] - sc->sel_seen[0]) * sc->g_step.alt_less +
                              (sel[1] - sc->sel_seen[1]) * sc->g_adj.alt_less);
    sc->sel_seen[0] = sel[0];
    sc->sel_seen[1] = sel[1];
  }
  return status_error(st4);
}

int dfem_eval_local(dfem_scene* sc, const double* x, double* jd_out, int mem) {
  if (!sc || !x || !jd_out) return fail(DFEM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(sc->device));
  const HostScene& s = sc->hs;
  const size_t n3 = 3 * (size_t)s.N;
  const int nb = sc->nblk_v;
  const Gate open{nullptr, nullptr, nullptr, 0};
  RC(copy_in(sc, x, n3, sc->io_a.p, mem));
  k_to_internal<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_internal.p, sc->io_a.p, sc->rhs.p);
  k_set_int<<<1, 1, 0, sc->stream>>>(sc->zero.p, 0);
  launch_local(sc, sc->stream, open, sc->rhs.p, sc->act_cur.p, sc->zero.p, true);
  // J d = attachment term + the constraints' slots (c0 := J_att d_att)
  launch_gather(sc, sc->stream, open, sc->attach_jd.p, sc->io_b.p, nullptr, true);
  k_to_user<<<nb, 128, 0, sc->stream>>>(s.N, sc->to_user.p, sc->io_b.p, sc->io_a.p);
  CK(cudaGetLastError());
  sc->launches += 5;
  RC(copy_out(sc, sc->io_a.p, n3, jd_out, mem));
  CK(cudaStreamSynchronize(sc->stream));
  return DFEM_OK;
}

int dfem_get_contact_passes(const dfem_scene* sc, int32_t* passes, int32_t n) {
  if (!sc || !passes) return fail(DFEM_ERR_INVALID, "null argument");
  for (int st = 0; st < n; ++st) passes[st] = (2 * st < (int)sc->rec_passes.size()) ? sc->rec_passes[2 * st] : 0;
  return DFEM_OK;
}

int dfem_get_iterations(const dfem_scene* sc, int32_t* iters, int32_t n) {
  if (!sc || !iters) return fail(DFEM_ERR_INVALID, "null argument");
  if (n > sc->cap_steps) return fail(DFEM_ERR_INVALID, "n exceeds recorded steps");
  CK(cudaSetDevice(sc->device));
  CK(cudaMemcpy(iters, sc->iters.p, (size_t)n * sc->hs.nparts * sizeof(int), cudaMemcpyDeviceToHost));
  return DFEM_OK;
}

int dfem_host_factor_solve(const dfem_scene_desc* desc, const double* b, double* x, dfem_scene_info* info) {
  if (!desc || !b || !x) return fail(DFEM_ERR_INVALID, "null argument");
  HostScene hs;
  std::string err;
  if (!build_host_scene(*desc, hs, err)) return fail(DFEM_ERR_INVALID, err);
  if (!refactorize(hs.Hs, hs.F, err)) return fail(DFEM_ERR_FACTOR, err);
  const int N = hs.N;
  std::vector<double> bi(3 * (size_t)N), xi(3 * (size_t)N);
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) bi[3 * (size_t)hs.to_internal[i] + c] = b[3 * (size_t)i + c];
  host_solve(hs.F, bi.data(), xi.data());
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) x[3 * (size_t)i + c] = xi[3 * (size_t)hs.to_internal[i] + c];
  if (info) {
    info->n_vertices = hs.N; info->n_tets = hs.T; info->n_attach = hs.A; info->n_muscle = hs.M;
    info->n_springs = hs.S; info->n_bending = hs.B; info->n_supernodes = hs.F.nsuper;
    info->n_levels = hs.F.nlevels; info->nnz_factor = hs.F.nnz_factor; info->n_slots = hs.nslots;
    info->device = -1; info->factor_regularisation = hs.F.reg;
  }
  return DFEM_OK;
}

int dfem_profile_levels(dfem_scene* sc, int32_t reps, int32_t cap, int32_t* n_segments, double* ms_fwd, double* ms_bwd,
                        int32_t* n_supernodes, int32_t* level, int32_t* threads) {
  if (!sc || !n_segments || reps < 1) return fail(DFEM_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(sc->device));
  const int G = (int)sc->segs.size();
  *n_segments = G;
  if (!ms_fwd || !ms_bwd || cap < G) return DFEM_OK;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaMemsetAsync(sc->status.p, 0, 4 * sizeof(int), sc->stream));
  auto time_it = [&](auto&& launch) -> double {
    launch();
    cudaEventRecord(e0, sc->stream);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, sc->stream);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    sc->launches += reps + 1;
    return (double)t / reps;
  };
  for (int g = 0; g < G; ++g) {
    const auto& sg = sc->segs[g];
    if (n_supernodes) n_supernodes[g] = sg.count;
    if (level) level[g] = sg.level;
    if (threads) {  // 32: one supernode per warp
      threads[2 * g] = sg.warp ? 32 : sg.thr_f;
      threads[2 * g + 1] = sg.warp ? 32 : sg.thr_b;
    }
    ms_fwd[g] = time_it([&] { launch_segment(sc, sc->stream, sg, true, sg.thr_f, kOpen, sc->rhs.p, sc->y.p); });
    ms_bwd[g] = time_it([&] { launch_segment(sc, sc->stream, sg, false, sg.thr_b, kOpen, sc->rhs.p, sc->y.p); });
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaGetLastError());
  int st4[4] = {0, 0, 0, 0};
  CK(cudaMemcpy(st4, sc->status.p, sizeof(st4), cudaMemcpyDeviceToHost));
  RC(status_error(st4));
  sc->rec_steps = 0;
  return DFEM_OK;
}

int dfem_solve_mode(dfem_scene* sc, int32_t request, int32_t* chosen, double* ms) {
  if (!sc) return fail(DFEM_ERR_INVALID, "null argument");
  if (request < -1 || request > 6) return fail(DFEM_ERR_INVALID, "request must be -1, 0, 1, 2, 3, 4, 5 or 6");
  CK(cudaSetDevice(sc->device));
  if (request == 0) {
    CK(cudaStreamSynchronize(sc->stream));
    CK(cudaMemsetAsync(sc->status.p, 0, 4 * sizeof(int), sc->stream));
    RC(autotune_solve(sc));
    sc->rec_steps = 0;  // the tuning solves overwrote the recorded iterates
  } else if (request > 0) {
    if (request == 3 && sc->split_cut == 0) return fail(DFEM_ERR_INVALID, "no split form (fewer than two levels)");
    if (request == 4 && !sc->cluster_ok) return fail(DFEM_ERR_INVALID, "no cluster form for this factor");
    if (request == 5 && !sc->res_ok) return fail(DFEM_ERR_INVALID, "no resident form for this scene");
    if (request == 6) {
      if (!sc->dense_ok) return fail(DFEM_ERR_INVALID, "no dense form for this scene (a batch, or too many vertices)");
      if (!sc->dense_built) {
        CK(cudaStreamSynchronize(sc->stream));
        RC(dense_build(sc));
      }
    }
    const int c = request == 1 ? n_levels(sc) : request == 2 ? 0 : request == 3 ? sc->split_cut : request == 4 ? -1
                : request == 5 ? -2 : -3;
    if (c != sc->solve_cut || sc->solve_select) {  // a requested form is used in every iteration
      sc->solve_cut = c;
      sc->solve_select = false;
      invalidate_graphs(sc);
    }
  }
  if (chosen) *chosen = solve_form(sc);
  if (ms) { ms[0] = sc->solve_ms[0]; ms[1] = sc->solve_ms[1]; }
  return DFEM_OK;
}

int dfem_solve_select(const dfem_scene* sc, int32_t* on, double* weight_threshold, double* ms_one_part) {
  if (!sc) return fail(DFEM_ERR_INVALID, "null argument");
  if (on) *on = sc->solve_select ? 1 : 0;
  if (weight_threshold) *weight_threshold = sc->solve_select ? sc->select_w : 0.0;
  if (ms_one_part) { ms_one_part[0] = sc->select_ms[0]; ms_one_part[1] = sc->select_ms[1]; }
  return DFEM_OK;
}

int dfem_solve_times(const dfem_scene* sc, double* ms, int32_t n) {
  if (!sc || !ms || n < 0) return fail(DFEM_ERR_INVALID, "bad argument");
  for (int k = 0; k < std::min(n, 6); ++k) ms[k] = sc->solve_ms[k];
  if (n > 6) ms[6] = sc->dense_build_ms;
  return DFEM_OK;
}

int dfem_solve_split(const dfem_scene* sc, int32_t* cut_level, int32_t* n_levels_out, double* ms_split) {
  if (!sc) return fail(DFEM_ERR_INVALID, "null argument");
  if (cut_level) *cut_level = sc->split_cut;
  if (n_levels_out) *n_levels_out = n_levels(sc);
  if (ms_split) *ms_split = sc->solve_ms[2];
  return DFEM_OK;
}

int dfem_set_adjoint_budget(dfem_scene* sc, int64_t bytes) {
  if (!sc || bytes < 0) return fail(DFEM_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(sc->device));
  CK(cudaStreamSynchronize(sc->stream));
  sc->adj_budget = (size_t)bytes;
  const int cap = std::max(1, sc->cap_steps);
  sc->cap_steps = 0;  // reallocate the per-step buffers under the new budget
  RC(ensure_steps(sc, cap));
  sc->rec_steps = 0;  // the recorded forward's buffers are gone
  return DFEM_OK;
}

int dfem_get_launch_count(const dfem_scene* sc, int64_t* count) {
  if (!sc || !count) return fail(DFEM_ERR_INVALID, "null argument");
  *count = sc->launches;
  return DFEM_OK;
}

int dfem_profile_phases(dfem_scene* sc, int32_t reps, double* ms) {
  if (!sc || !ms || reps < 1) return fail(DFEM_ERR_INVALID, "bad argument");
  if (sc->rec_steps <= 0) return fail(DFEM_ERR_STATE, "dfem_profile_phases needs a preceding dfem_step_forward");
  CK(cudaSetDevice(sc->device));
  const HostScene& s = sc->hs;
  const int ncons = s.T + s.M + s.S + s.B;
  // every phase is launched ungated on the state of the last forward call (step 0, iteration 0)
  k_set_int<<<1, 1, 0, sc->stream>>>(sc->step.p, 0);
  k_set_int<<<1, 1, 0, sc->stream>>>(sc->zero.p, 0);
  CK(cudaMemsetAsync(sc->status.p, 0, 4 * sizeof(int), sc->stream));
  reset_solve_state(sc);
  const Gate gf = kOpen, ga = kOpen;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto timed = [&](int phase, auto&& launch) -> int {
    launch();  // warm-up
    CK(cudaEventRecord(e0, sc->stream));
    for (int r = 0; r < reps; ++r) launch();
    CK(cudaEventRecord(e1, sc->stream));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    ms[phase] = (double)t / reps;
    sc->launches += reps + 1;
    return DFEM_OK;
  };
  int rc = DFEM_OK;
  if (!rc && ncons > 0) rc = timed(0, [&] { launch_local(sc, sc->stream, gf, sc->xk.p, sc->act_all.p, sc->step.p); });
  if (!rc) rc = timed(1, [&] { launch_gather(sc, sc->stream, gf, sc->c0.p, sc->rhs.p, sc->xk.p); });
  if (!rc) rc = timed(2, [&] { enqueue_solve(sc, sc->stream, gf, sc->rhs.p, sc->y.p); });
  if (!rc && ncons > 0) rc = timed(3, [&] { launch_adj_local(sc, sc->stream, ga, sc->zero.p); });
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  CK(cudaGetLastError());
  int st4[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(st4, sc->status.p, sizeof(st4), cudaMemcpyDeviceToHost, sc->stream));
  CK(cudaStreamSynchronize(sc->stream));
  RC(status_error(st4));
  // the solve phase counted one launch per call above
  sc->launches += (int64_t)(reps + 1) * (solve_launches(sc) - 1);
  sc->rec_steps = 0;  // gates and iteration counts were overwritten: no backward of the old forward
  return DFEM_OK;
}

int dfem_set_limit(dfem_scene* sc, int32_t which, int64_t value) {
  if (!sc) return fail(DFEM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(sc->device));
  CK(cudaStreamSynchronize(sc->stream));
  const bool dflt = value < 0;
  switch (which) {
    case DFEM_LIMIT_CONTACT_PASSES:
    case DFEM_LIMIT_IMPACTS_PER_VERTEX:
    case DFEM_LIMIT_SOFT_IMPACTS_PER_VERTEX:
    case DFEM_LIMIT_GROUP_MEMBERS: {
      const int cap = which == DFEM_LIMIT_CONTACT_PASSES ? kMaxContactPasses
                      : which == DFEM_LIMIT_IMPACTS_PER_VERTEX ? kMaxImpactsPerVertex
                      : which == DFEM_LIMIT_SOFT_IMPACTS_PER_VERTEX ? kMaxSelfImpacts : kMaxGroupMembers;
      if (!dflt && value > cap) return fail(DFEM_ERR_INVALID, "limit above the built-in cap " + std::to_string(cap));
      const int v = dflt ? cap : (int)value;
      ContactDev& c = sc->cd;
      (which == DFEM_LIMIT_CONTACT_PASSES ? c.max_passes : which == DFEM_LIMIT_IMPACTS_PER_VERTEX ? c.max_impacts
       : which == DFEM_LIMIT_SOFT_IMPACTS_PER_VERTEX ? c.max_self_impacts : c.max_members) = v;
      break;
    }
    case DFEM_LIMIT_BROAD_PHASE_CELLS:
      if (!dflt && value > 4096) return fail(DFEM_ERR_INVALID, "broad-phase cell limit must be in [0, 4096]");
      sc->cd.bp_max_cells = dflt ? kBroadDefaultCells : (int)value;
      break;
    case DFEM_LIMIT_SOLVE_WAIT_POLLS:
      if (!dflt && (value < 1 || value > kSpinTries))
        return fail(DFEM_ERR_INVALID, "poll limit must be in [1, " + std::to_string(kSpinTries) + "]");
      sc->spin_tries = dflt ? kSpinTries : (int)value;
      sc->fd.spin_tries = sc->spin_tries;
      break;
    default:
      return fail(DFEM_ERR_INVALID, "unknown limit");
  }
  invalidate_graphs(sc);  // the kernels' parameters changed
  sc->rec_steps = 0;
  return DFEM_OK;
}

int dfem_set_option(dfem_scene* sc, int32_t which, int64_t value) {
  if (!sc) return fail(DFEM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(sc->device));
  CK(cudaStreamSynchronize(sc->stream));
  switch (which) {
    case DFEM_OPTION_FUSED_CONTACT:
      if (value != 0 && value != 1) return fail(DFEM_ERR_INVALID, "value must be 0 or 1");
      if (value == 1 && sc->cnp > 0 && !sc->fused_ok)
        return fail(DFEM_ERR_UNSUPPORTED, "the device cannot run the batch's cooperative contact phase");
      sc->fused_on = value != 0;
      break;
    case DFEM_OPTION_GATHER:
      if (value < 0 || value > 2) return fail(DFEM_ERR_INVALID, "value must be 0, 1 or 2");
      sc->gather_form = (int)value;
      break;
    case DFEM_OPTION_SPLIT_FACTOR:
      if (value != 0 && value != 1) return fail(DFEM_ERR_INVALID, "value must be 0 or 1");
      sc->split_factor = value != 0;
      break;
    default:
      return fail(DFEM_ERR_INVALID, "unknown option");
  }
  invalidate_graphs(sc);
  sc->rec_steps = 0;
  return DFEM_OK;
}

int dfem_debug_fail_allocations(int64_t after) {
  g_alloc_budget = after < 0 ? -1 : after;
  return DFEM_OK;
}

int dfem_synchronize(dfem_scene* sc) {
  if (!sc) return fail(DFEM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(sc->device));
  CK(cudaStreamSynchronize(sc->stream));
  return DFEM_OK;
}

}  // extern "C"
