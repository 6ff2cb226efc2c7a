// resident_plan.cpp — see resident_plan.h.
#include "resident_plan.h"

#include <algorithm>

namespace dfem {

bool plan_resident_layout(const SupernodalFactor& F, const std::vector<int>& nseg, const std::vector<int>& cdst, int C,
                          size_t cap_bytes, ResidentPlan& P) {
  const int ns = F.nsuper, L = F.nlevels;
  P = ResidentPlan();
  if (ns == 0 || L == 0 || C < 1) return false;
  auto even = [](size_t v) { return (v + 1) & ~size_t(1); };
  std::vector<int> owner(ns, -1), lvl_of(ns);
  std::vector<size_t> img(ns), buf(ns), work(ns);
  int wmax = 1, rmax = 1;
  for (int q = 0; q < ns; ++q) {
    const size_t w = F.sn_w[q], r = F.sn_r[q];
    img[q] = even(w * (w + 1) / 2) + even(r * w) + even((w + 2) / 2);  // packed lower-triangular inverse
    buf[q] = 3 * (size_t)nseg[q] + 3 * w;
    work[q] = w * (w + 1) / 2 + r * w;
    wmax = std::max(wmax, (int)w);
    rmax = std::max(rmax, (int)r);
  }
  const size_t scratch = 3 * (size_t)wmax + 3 * (size_t)rmax;
  if (cap_bytes / 8 <= scratch) return false;
  const size_t capd = cap_bytes / 8 - scratch;
  for (int l = 0; l < L; ++l)
    for (int k = F.lvl_ptr[l]; k < F.lvl_ptr[l + 1]; ++k) lvl_of[F.lvl_sn[k]] = l;
  // owners: levels from the top down, the largest supernodes of a level first,
  // each to the CTA with the least work at that level that still has room
  std::vector<size_t> total(C, 0), lvl_load(C, 0);
  for (int l = L - 1; l >= 0; --l) {
    std::vector<int> items(F.lvl_sn.begin() + F.lvl_ptr[l], F.lvl_sn.begin() + F.lvl_ptr[l + 1]);
    std::stable_sort(items.begin(), items.end(), [&](int a, int b) { return img[a] + buf[a] > img[b] + buf[b]; });
    std::fill(lvl_load.begin(), lvl_load.end(), 0);
    for (int q : items) {
      int best = -1;
      for (int c = 0; c < C; ++c) {
        if (total[c] + img[q] + buf[q] > capd) continue;
        if (best < 0 || lvl_load[c] < lvl_load[best] || (lvl_load[c] == lvl_load[best] && total[c] < total[best])) best = c;
      }
      if (best < 0) return false;
      owner[q] = best;
      total[best] += img[q] + buf[q];
      lvl_load[best] += work[q];
    }
  }
  std::vector<std::vector<int>> own(C);
  for (int k = 0; k < ns; ++k) own[owner[F.lvl_sn[k]]].push_back(F.lvl_sn[k]);  // level order
  P.C = C;
  P.L = L;
  P.sched.assign((size_t)C * (L + 1), 0);
  P.tsh.assign(2 * (size_t)C, 0);
  P.img_ofs.assign(C + 1, 0);
  std::vector<int> dofs(ns), lofs(ns), pofs(ns), qofs(ns), yofs(ns);
  size_t smax = 0;
  for (int c = 0; c < C; ++c) {
    size_t at = 0;
    for (int q : own[c]) {
      dofs[q] = (int)at; at += even((size_t)F.sn_w[q] * (F.sn_w[q] + 1) / 2);
      lofs[q] = (int)at; at += even((size_t)F.sn_r[q] * F.sn_w[q]);
      pofs[q] = (int)at; at += even(((size_t)F.sn_w[q] + 2) / 2);
    }
    P.img_ofs[c + 1] = P.img_ofs[c] + (long long)at;
    for (int q : own[c]) { qofs[q] = (int)at; at += 3 * (size_t)nseg[q]; }
    for (int q : own[c]) { yofs[q] = (int)at; at += 3 * (size_t)F.sn_w[q]; }
    P.tsh[c] = (int)at; at += 3 * (size_t)wmax;
    P.tsh[C + c] = (int)at; at += 3 * (size_t)rmax;
    smax = std::max(smax, at);
    int k = 0;
    const int base = (int)P.items.size();
    for (int l = 0; l <= L; ++l) {
      while (k < (int)own[c].size() && lvl_of[own[c][k]] < l) ++k;
      P.sched[(size_t)c * (L + 1) + l] = base + k;
    }
    for (int q : own[c]) {
      P.items.push_back({F.sn_c0[q], F.sn_w[q], F.sn_r[q], dofs[q], lofs[q], pofs[q], qofs[q], yofs[q],
                         (int)F.sn_rofs[q], q});
      P.pack.push_back({F.sn_w[q], F.sn_r[q], (int)F.sn_dofs[q], (int)F.sn_lofs[q], P.img_ofs[c] + dofs[q],
                        P.img_ofs[c] + lofs[q]});
    }
  }
  if (8 * smax > cap_bytes) return false;
  P.smem_doubles = smax;
  const size_t nrow = F.rowidx.size();
  P.cdst_rank.assign(nrow, 0); P.cdst_ofs.assign(nrow, 0);
  P.xsrc_rank.assign(nrow, 0); P.xsrc_ofs.assign(nrow, 0);
  for (int q = 0; q < ns; ++q)
    for (int a = 0; a < F.sn_r[q]; ++a) {
      const size_t p = (size_t)F.sn_rofs[q] + a;
      const int j = F.rowidx[p], d = F.col_sn[j];
      P.cdst_rank[p] = owner[d];
      P.cdst_ofs[p] = qofs[d] + 3 * (cdst[p] - F.rseg_ptr[F.sn_c0[d]]);
      P.xsrc_rank[p] = owner[d];
      P.xsrc_ofs[p] = yofs[d] + 3 * (j - F.sn_c0[d]);
    }
  P.img.assign(std::max<long long>(2, P.img_ofs[C]), 0.0);
  for (int c = 0; c < C; ++c)
    for (int q : own[c]) {
      int* pr = reinterpret_cast<int*>(P.img.data() + P.img_ofs[c] + pofs[q]);
      for (int k = 0; k <= F.sn_w[q]; ++k) pr[k] = F.rseg_ptr[F.sn_c0[q] + k] - F.rseg_ptr[F.sn_c0[q]];
    }
  return true;
}

void pack_into_images(const ResidentPlan& P, const double* Dinv, const double* Lcm, double* img) {
  for (const ResidentPlan::Pack& p : P.pack) {
    for (int i = 0; i < p.w; ++i)  // row i of the lower triangle at i (i + 1) / 2
      for (int j = 0; j <= i; ++j) img[p.dst_d + (size_t)i * (i + 1) / 2 + j] = Dinv[p.src_d + (size_t)i * p.w + j];
    for (int k = 0; k < p.r * p.w; ++k) img[p.dst_l + k] = Lcm[p.src_l + k];
  }
}

}  // namespace dfem
