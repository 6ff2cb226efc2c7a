// kernels.cuh — device-side data views and kernels of the PD step and its adjoint.
//
// Data layout in HBM (all arrays of one scene, internal vertex numbering):
//   positions / velocities / rhs : interleaved FP64 [x y z] per vertex (3N)
//   tets  : int4 vertex ids, invDm as 9 SoA planes (plane k holds invDm[k/3][k%3]),
//           weights w_r = mu*vol and w_v = nu*mu*vol, int4 slot positions
//   slots : one [x y z] FP64 contribution per (constraint, vertex) pair, sorted
//           by vertex, so the rhs gather reads one contiguous range per vertex
//   factor: supernodes (first column, width, rows below), row-wise CSR of the
//           below-diagonal entries (forward solve), column-major below-diagonal
//           blocks + row ids (backward solve), inverses of the diagonal blocks.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "pd_math.cuh"
#include "tma.cuh"

namespace dfem {

constexpr double kConvergenceEps = 5e-7;  // World.h:214 (EPS)

// Kernels of a PD iteration are gated on device state, per part of a batch (a
// single scene is a batch of one part): in the forward loop a part whose
// convergence flag is set does no further work; in the reverse loop a part
// skips the iterations k >= its recorded count; in the contact phase kernels
// run only while the phase is active.  The conditional graph loops stop once
// every part is done, so a single scene never executes a gated-off iteration.
struct Gate {
  const int* flag = nullptr;    // forward: per-part converged flags
  const int* iters = nullptr;   // adjoint: iteration counts [step][part]
  const int* step = nullptr;    // adjoint: current step index
  const int* kptr = nullptr;    // adjoint: current reverse iteration
  int nparts = 1;
  const int* active = nullptr;  // contact phase: run only while *active == 1
  __device__ __forceinline__ bool skip(int part) const {
    if (flag && flag[part]) return true;
    if (iters && *kptr >= iters[(size_t)(*step) * nparts + part]) return true;
    if (active && *active != 1) return true;
    return false;
  }
};

// Part-aligned blocks of the vertex kernels with per-part reductions: block b
// covers vertices [blk_v0[b], min(blk_v0[b] + 128, part_v0[p + 1])) of part
// p = blk_part[b]; the blocks of part p are part_b0[p] .. part_b0[p + 1] - 1.
constexpr int kPartBlock = 128;
struct PartDev {
  int nparts;
  const int* part_v0;   // nparts + 1
  const int* part_b0;   // nparts + 1
  const int* blk_part;
  const int* blk_v0;
};

struct SceneDev {
  int N, T, M, S, B, nseg;
  double h, damping, g0, g1, g2;
  const double* mass;
  const double* gmask;
  // tets
  const int4* tv;
  const double* tinv;   // 9 planes of T
  const double* twr;    // mu * vol
  const double* twv;    // nu * mu * vol
  const double* tvol;
  const double* tE;
  const double* tnu;
  const int4* tslot;
  // muscles
  const int4* mv;
  const double* minv;   // 9 planes of M
  const double* mw;     // vol * stiffness
  const double* mfib;   // 3 planes of M
  const int* mseg;
  const int4* mslot;
  const int* seg_ptr;   // channel -> members CSR
  const int* seg_mus;   // member: muscle m as m, pneumatic spring k as -(k+1)
  // springs
  const int2* sv;
  const double* srest;
  const double* ssw;
  const int2* sslot;
  const int* sch;       // activation channel per spring (-1 plain); null without pneumatic springs
  // bending
  const int* boff;
  const int* bv;
  const double* bbeta;
  const double* bw;
  const double* brest;
  const int* bslot;
  // slots
  const int* vslot_ptr;
  // attachment constant J*d (3N)
  const double* attach_jd;
  // Hs CSR
  const int* hs_ptr;
  const int* hs_col;
  const double* hs_val;
  // per-vertex sum of attachment stiffnesses (the attachments' diagonal of Hs)
  const double* attach_k;
  // batch: part of every vertex and muscle segment (null for a single scene)
  const int* vpart;
  const int* seg_part;
  // underwater drag: every vertex's face corners (3 f + corner, ascending) and
  // the per-face force of the step (null without drag faces)
  const int* vf_ptr;
  const int* vf_face;
  const double* fdrag;
};

__device__ __forceinline__ int vpart_of(const SceneDev& d, int i) { return d.vpart ? d.vpart[i] : 0; }

// Index into the activation-term array mg of channel member k (seg_mus):
// muscle m at m, pneumatic spring s at M + s.
__host__ __device__ __forceinline__ int member_slot(int M, int k) { return k >= 0 ? k : M - 1 - k; }

// part of constraint t (tets, muscles, springs, bending stencils in that order)
__device__ __forceinline__ int cons_part(const SceneDev& d, int t) {
  if (!d.vpart) return 0;
  if (t < d.T) return d.vpart[d.tv[t].x];
  t -= d.T;
  if (t < d.M) return d.vpart[d.mv[t].x];
  t -= d.M;
  if (t < d.S) return d.vpart[d.sv[t].x];
  t -= d.S;
  if (t < d.B) return d.vpart[d.bv[d.boff[t]]];
  return 0;
}

// Contact phase state (World::ProjectiveDynamicsMethod, sim/fem/World.h:925-1023).
constexpr int kMaxImpactsPerVertex = 8;  // a vertex at a corner of a tessellated obstacle touches up to 6 faces
constexpr int kMaxContactPasses = 64;       // the reference's detection loop has no cap
constexpr double kContactThickness = 1e-4;  // arcsim Impact::thickness
// Status word codes of the caps (status[2] when status[0] == DFEM_ERR_CAP); the
// solves use 1-9 (pd_kernels.cu, resident_solve.cuh).
enum { kCapContactPasses = 10, kCapImpacts = 11, kCapSoftImpacts = 12, kCapGroupMembers = 13 };

// Broad phase of the obstacle detection: a uniform grid over the static
// obstacle faces' boxes dilated by kBroadPad; a vertex tests the faces of the
// cells its swept box (dilated alike) covers, in ascending face order, and
// every face when that box covers more than bp_max_cells cells or gathers
// more than kBroadMaxCandidates faces.
constexpr double kBroadPad = 2.5e-4;          // > the obstacle contact thickness (1e-4)
constexpr int kBroadMaxCandidates = 128;
constexpr int kBroadDefaultCells = 64;

struct ContactDev {
  int nc, nof, K, max_passes;
  int max_impacts;        // obstacle impacts kept per vertex (<= kMaxImpactsPerVertex)
  int max_self_impacts;   // soft impacts kept per vertex (<= kMaxSelfImpacts)
  int max_members;        // members of one face group (<= kMaxGroupMembers)
  int bp_max_cells;       // broad phase: cells a query may cover (0: every face is tested)
  int bp_dim[3];          // grid cells per axis (0: no grid)
  double bp_org[3];       // grid origin
  double bp_inv;          // 1 / cell size
  const int* bp_ptr;      // cells + 1: each cell's faces bp_face[bp_ptr[c] .. bp_ptr[c + 1]) (ascending)
  const int* bp_face;
  double alpha, mu;
  const int* cverts;      // contact vertices (internal ids)
  const int* cidx;        // N: contact index or -1
  const double* obs_x;    // 3 per obstacle vertex
  const int* obs_f;       // 3 per obstacle face
  const double* hdiag;    // N: diagonal of Hs
  int* imp_cnt;           // nc
  int* imp_face;          // nc * kMax
  double* imp_n;          // nc * kMax * 3
  double* xn1;            // 3N: x_n1 of the reference's contact loop
  double* xold;           // 3N
  double* prev;           // 3N: relaxed rhs
  double* lxt;            // 3N: L x_t
  double* vwc;            // 3N: v + g h of the step
  int* state;             // see CS_* in contact_kernels.cuh
  // recording for the adjoint (written only while *rec_on != 0): 1 = a step
  // the adjoint replays (a record too small is an error), 2 = the forward
  // steps in a row (a step that does not fit is marked unrecorded and replayed)
  const int* rec_on;
  int rec_cap;            // computed iterations the record holds
  int rec_fwd_cap;        // of which the forward may fill (the rest: room for the adjoint's replays)
  double* rec_x;          // rec_cap x 3N: each computed iteration's input ori_x
  double* rec_prev;       // rec_cap x 3N: its relaxed rhs after the update
  int* rec_first;         // rec_cap: whether it began its pass
  int* rec_cnt;           // rec_cap x nc: impacts per contact vertex
  double* rec_n;          // rec_cap x nc x kMax x 3: their normals
  int* status;
  int* rec_base;          // the current step's first record (computed iteration j of it is record base + j)
  int* rec_meta;          // forward recording, per step: [first record, computed iterations, source, recorded]
  // soft-soft (self) contact; ncf == 0: off
  int ncf;                // soft contact faces
  double mu_self;         // "World Friction"
  const int* cfaces;      // 3 per soft face: contact indices
  const int* cvf_ptr;     // nc + 1: each contact vertex's soft faces (cvf_face, ascending)
  const int* cvf_face;
  const int* on_face;     // nc: 1 if the vertex lies on a soft face
  int* simp_cnt;          // nc: the step's soft impacts per vertex (list order)
  int* simp_face;         // nc * kMaxSelfImpacts
  double* simp_td;        // nc * kMaxSelfImpacts * 2: time t, distance |d|
  double* simp_n;         // nc * kMaxSelfImpacts * 3: normal
  int* cf_face;           // nc: face of the vertex's closest impact this pass (-1: none)
  int* cf_slot;           // nc: that impact's list slot
  int* m_slot;            // nc: the vertex's position in g_mem
  int* g_cnt;             // ncf: members of each face's group this pass
  int* g_fill;            // ncf: fill cursor
  int* g_ptr;             // ncf + 1: exclusive scan of g_cnt
  int* g_mem;             // nc: members grouped by face, ascending within a group
  double* g_n;            // 3 ncf: group normal (its first member's impact normal)
  double* g_outF;         // 9 ncf: a group's self forces on its face's three vertices
  double* g_outM;         // 3 nc: a member's self force (by its g_mem position)
  double* sc_cur;         // 3 nc: self forces of the step's last CollisionHandling call that swapped buffers
                          // (zero at every step's start)
  double* rhs_pre;        // 3 nc: contact vertices' rhs before this iteration's CollisionHandling
  double* cnext;          // 3 nc: obstacle reactions of this iteration (self contact on)
  int* chit;              // nc: the vertex has an obstacle reaction this iteration
  // records of soft contact for the adjoint (per computed iteration, at the
  // record index of rec_index): rec_si = [cf_face, m_slot, g_mem (nc each),
  // g_cnt (ncf), g_ptr (ncf + 1), obstacle impacts, groups], rec_sd =
  // [remembered self forces before the call (3 nc), g_n (3 ncf)]
  int* rec_si;
  double* rec_sd;
  // batches (np > 1, obstacle contact only): the part of each contact vertex,
  // each part's obstacle faces [pf0[p], pf0[p+1]), and the phase's per-part
  // state; the broad phase is off (a part's faces are tested in order)
  int np;
  const int* cpart;       // nc
  const int* pf0;         // np + 1
  int* pst;               // np x PS_SIZE (contact_kernels.cuh)
  unsigned long long* pe; // 2 x np: per-part max-norm change of ori_x (bits of a double >= 0), two parities
  int* pany;              // 2 x np: per-part detection hit flags, two parities
  int* psrc;              // per step x np: each part's source iteration (forward recording)
};
__host__ __device__ inline size_t self_rec_si_stride(int nc, int ncf) { return 3 * (size_t)nc + 2 * (size_t)ncf + 3; }
__host__ __device__ inline size_t self_rec_sd_stride(int nc, int ncf) { return 3 * (size_t)nc + 3 * (size_t)ncf; }
constexpr int kMaxSelfImpacts = 16;      // soft impacts per contact vertex in one step
constexpr int kMaxGroupMembers = 32;     // members of one face group

// One supernode of the triangular solves, stored in level order (position
// lvl_ptr[l] .. lvl_ptr[l+1] of level l) so that one load gives a solve
// everything it needs before its data loads.
struct SnInfo {
  int c0, w, r;   // first column, width, rows below the diagonal block
  int rofs;       // its below-diagonal rows: rowidx[rofs .. rofs + r)
  int lofs;       // L_{R,s} (column-major r x w) at Lcm + lofs
  int dofs;       // diagonal-block inverse at Dinv + dofs (row-major) and DinvC + dofs (column-major)
  int seg0, nseg; // the contributions to its rows: contrib[3 seg0 .. 3 (seg0 + nseg))
  int s;          // supernode id (elimination tree, completion stamps)
  int part;       // batch part
  int stage;      // 1: L_{R,s} is staged in shared memory too
  int cc;         // not staged: columns per chunk of L_{R,s} streamed through two shared buffers (0: read from global)
};

struct FactorDev {
  const SnInfo* info;    // level order
  const int* rseg_ptr;   // row -> its contributions: contrib[3 rseg_ptr[i] .. 3 rseg_ptr[i+1]) in a fixed order
  const int* cdst;       // below-diagonal row position (rowidx order) -> its contribution slot
  double* contrib;       // 3 doubles per below-diagonal row of every supernode, grouped by destination row
  const int* rowidx;
  const double* Lcm;
  const double* Dinv;    // row-major (backward solve)
  const double* DinvC;   // column-major (forward solve)
  int* status;   // error status word (6: a bounded wait gave up)
  // persistent solve: elimination tree, completion stamps, control words
  int nsuper;
  const int* sn_pos;     // supernode -> its level-order position
  const int* sn_parent;
  const int* kid_ptr;
  const int* kid;
  int* done_f;
  int* done_b;
  int* ctl;      // [ticket, CTAs finished, epoch, abort]
  int spin_tries;  // polls of a persistent-solve dependency wait before it gives up
};

}  // namespace dfem
