// resident_plan.h — host-side layout of the resident solve form: which CTA of
// a thread-block cluster owns each supernode of the factor, and where every
// block, row table, address table, contribution inbox, solution region and
// scratch vector sits in each CTA's shared memory.  Plain C++ (no CUDA
// calls), so the layout and a CPU emulation of the solve can be checked
// without a GPU.
//
// Shared memory of a CTA (offsets in doubles), the first part being its image
// (loaded from global memory by bulk copies at the start of every launch):
//   head   header ints [nitems, L, 3*sum(w), t offset, x_R offset, items
//          offset, sched[L + 1] (first item of each level), cum[nitems + 1]
//          (prefix sums of 3w)], then the item records (ResItem, 10 ints)
//   blocks per item: Dinv packed by rows, L_{R,s} column-major, row ->
//          inbox range (w + 1 ints), address tables (r push targets, r pull
//          sources: 32-bit words rank << 24 | offset)
//   then   inboxes (3 per contribution), solution regions (3 per column),
//          scratch t (3 w_max) and x_R (3 r_max)
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "cholesky.h"

namespace dfem {

// One supernode in its owner CTA's shared memory (offsets in doubles).
struct ResItem {
  int c0, w, r;   // first column, width, rows below
  int dofs;       // Dinv, packed lower triangle by rows (row i at dofs + i (i + 1) / 2)
  int lofs;       // L_{R,s}, column-major r x w
  int pofs;       // row -> inbox range (w + 1 ints)
  int qofs;       // inbox: 3 doubles per contribution to its rows, grouped by row
  int yofs;       // its solution values (3 per column)
  int tofs;       // address tables: r push targets, then r pull sources (uint32 each)
  int s;          // supernode id
};

constexpr int kResHeadInts = 6;  // ints before sched in the header

struct ResidentPlan {
  int C = 0, L = 0;                 // CTAs of the cluster, levels
  size_t smem_doubles = 0;          // dynamic shared memory of every CTA
  std::vector<int> owner;           // per supernode
  std::vector<std::vector<ResItem>> items;  // per CTA, level order
  std::vector<int> head_len;        // per CTA: doubles of the header + items part (first bulk copy)
  std::vector<long long> img_ofs;   // C + 1: the CTAs' images, back to back (doubles, even)
  std::vector<double> img;          // the images with headers and tables filled (blocks: pack_into_images)
  struct Pack { int w, r, src_d, src_l; long long dst_d, dst_l; };
  std::vector<Pack> pack;           // per supernode: where its blocks go in the images
};

// Owners and layout for a cluster of C CTAs with cap_bytes of shared memory
// each; nseg[q] = contributions to supernode q's rows, cdst[p] = the grouped
// contribution slot of below-diagonal row position p.  Returns false when the
// factor does not fit.
bool plan_resident_layout(const SupernodalFactor& F, const std::vector<int>& nseg, const std::vector<int>& cdst, int C,
                          size_t cap_bytes, ResidentPlan& P);

// The factor's blocks (Dinv row-major w x w at sn_dofs, Lcm column-major r x w
// at sn_lofs) into the images, as the device copy does after a refactorisation.
void pack_into_images(const ResidentPlan& P, const double* Dinv, const double* Lcm, double* img);

// Packed address of a value in a CTA's shared memory: rank << 24 | offset (doubles).
inline uint32_t res_addr(int rank, int ofs) { return ((uint32_t)rank << 24) | (uint32_t)ofs; }

}  // namespace dfem
