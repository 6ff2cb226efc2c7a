// resident_plan.h — host-side layout of the resident solve form: which CTA of
// a thread-block cluster owns each supernode of the factor, and where every
// block, row table, contribution inbox, solution region and scratch vector
// sits in each CTA's shared memory.  Plain C++ (no CUDA calls), so the layout
// and a CPU emulation of the solve can be checked without a GPU.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "cholesky.h"

namespace dfem {

struct ResidentPlan {
  int C = 0, L = 0;                 // CTAs of the cluster, levels
  size_t smem_doubles = 0;          // dynamic shared memory of every CTA
  struct Item {                     // one supernode, offsets in doubles into its owner's shared memory
    int c0, w, r, dofs, lofs, pofs, qofs, yofs, rofs, s;  // Dinv packed: row i of its lower triangle at dofs + i (i + 1) / 2
  };
  std::vector<Item> items;          // grouped by owner CTA, then by level
  std::vector<int> sched;           // C x (L + 1) item ranges
  std::vector<int> tsh;             // 2C: scratch t of CTA q at tsh[q], x_R at tsh[C + q]
  std::vector<int> cdst_rank, cdst_ofs;  // per below-diagonal row position: its contribution slot
  std::vector<int> xsrc_rank, xsrc_ofs;  // per below-diagonal row position: the row's solution values
  std::vector<long long> img_ofs;   // C + 1: the CTAs' images, back to back (doubles, even)
  std::vector<double> img;          // the images with the row tables filled (blocks: pack_into_images)
  struct Pack { int w, r, src_d, src_l; long long dst_d, dst_l; };
  std::vector<Pack> pack;           // per item: where its blocks go in the images
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

}  // namespace dfem
