// scene.h — host-side preprocessing of a dfem_scene_desc into the constraint
// tables, the scalar system matrix Hs and the slot layout the kernels use.
//
// Internally every vertex is renumbered into the fill-reducing order of the
// Cholesky factor, so the local step, the rhs gather, the triangular solves
// and the position update all work in one numbering and the permutation is
// applied only at the API boundary.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dfem.h"
#include "cholesky.h"

namespace dfem {

// Skeleton limits: links (the root's 6 dofs plus one per other link form the
// dense system of World::ComputeSolution) and rigid vertices (the dense
// Schur complement of the free vertices, World.h:1134-1135).
constexpr int kMaxLinks = 64;
constexpr int kMaxRigidVertices = 2048;

struct HostScene {
  int N = 0;
  std::vector<double> x0, mass, gmask;  // internal order

  // corotated tets: re-oriented vertices, invDm (row-major 9), weights
  int T = 0;
  std::vector<int> tv;                  // 4T (internal ids)
  std::vector<double> tinv;             // 9T
  std::vector<double> tvol, tE, tnu;
  std::vector<int> tslot;               // 4T slot positions

  int M = 0, nseg = 0;                  // muscle constraints
  std::vector<int> mv;                  // 4M
  std::vector<double> minv, mvol, mk, mfib;  // 9M, M, M, 3M
  std::vector<int> mseg, mslot;
  std::vector<int> seg_ptr, seg_mus;    // CSR channel -> members: muscle m as m, pneumatic spring s as -(s+1)

  int S = 0;                            // springs
  std::vector<int> sv, sslot;           // 2S
  std::vector<double> srest, ssw;       // rest length, sqrt(weight)
  std::vector<int> sch;                 // activation channel of each spring (-1 = plain); empty if none

  int B = 0;                            // bending stencils
  std::vector<int> boff, bv, bslot;     // CSR (centre first), slots
  std::vector<double> bbeta, bw, brest;

  int A = 0;                            // attachments
  std::vector<int> av;
  std::vector<double> ap, ak;

  // obstacle contact (internal ids for the soft surface vertices)
  bool collide = false;
  double alpha = 1.0, mu_obs = 1.0;
  std::vector<int> cverts;
  std::vector<double> obs_x;
  std::vector<int> obs_f;
  // batches: the part of each contact vertex, and each part's obstacle faces
  // [pobs_f0[p], pobs_f0[p+1]) (empty for a single scene)
  std::vector<int> cpart, pobs_f0;
  // soft-soft (self) contact: soft faces as contact indices (3 each), each
  // contact vertex's soft faces ascending (CSR), and whether it lies on one
  bool self_collide = false;
  double mu_self = 1.0;
  std::vector<int> cfaces, cvf_ptr, cvf_face, on_face;

  // underwater drag and lift: faces (3 internal ids each, outward winding)
  // and every vertex's faces in ascending face order (CSR)
  bool underwater = false;
  std::vector<int> df, vf_ptr, vf_face;

  // articulated skeleton (Link tree; link 0 the root): per link parent,
  // joint type (enum dfem_joint), torque channel, joint position and unit
  // axis (3 each), and its vertices (CSR, internal ids) with their rest
  // positions (3 each); the links' dofs are 6 for the root, 1 for the others
  int L = 0;
  std::vector<int> lparent, ltype, lchan, loff, lvert;
  std::vector<double> ljoint, laxis, lrest;

  int nslots = 0;
  std::vector<int> vslot_ptr;           // N+1, slots sorted by vertex

  SparseSym Hs;                         // internal order
  SupernodalFactor F;                   // factor of Hs (perm = identity after renumbering)
  std::vector<int> to_internal;         // user vertex id -> internal id
  std::vector<int> to_user;             // internal id -> user vertex id

  double h = 0.01, damping = 1.0, g[3] = {0, 0, 0};
  int K = 10;
  int precision = DFEM_PREC_FP64;
  int checkpoint_every = 1;

  // A batch is the disjoint union of independent parts (scenes); a single
  // scene is a batch of one.  Part p owns vertices [part_v0[p], part_v0[p+1]),
  // tets [part_t0[p], ..), muscle segments [part_seg0[p], ..) — contiguous in
  // both the user and the internal numbering.
  int nparts = 1;
  std::vector<int> part_v0, part_t0, part_seg0;
};

// Build everything (including ordering + factorisation).  Returns false with err.
bool build_host_scene(const dfem_scene_desc& d, HostScene& hs, std::string& err);

// Re-assemble Hs values after material changes and refactor (same structure).
bool update_materials(HostScene& hs, const double* E_user_order, const double* nu_user_order, std::string& err);

// Hs split for refactorisation on the GPU: base values (every term but the
// tets' E vol G G^T) on Hs's pattern, and per entry of Hs the tets that touch
// it with coefficient vol (G G^T)_ab, in tet order (CSR by entry).
void hs_split(const HostScene& s, std::vector<double>& base, std::vector<int>& cptr, std::vector<int>& ctet,
              std::vector<double>& ccoef);

// Union of independent scenes: every table concatenated with its indices
// offset, Hs and the supernodal factor block-diagonal, the level schedules
// merged level by level (level l of the union = level l of every part).  The
// parts must share time_step, damping, gravity, max_iterations, precision and
// checkpoint_every; obstacle contact is not supported in a batch.
bool merge_parts(const std::vector<HostScene>& parts, HostScene& u, std::string& err);

// Copy the parts' material-dependent values (moduli, Hs values, factor blocks)
// into the union after the parts were refactored (same structure).
void merge_numeric(const std::vector<HostScene>& parts, HostScene& u);

}  // namespace dfem
