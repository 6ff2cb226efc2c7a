// resident_plan.cpp — see resident_plan.h.
#include "resident_plan.h"

#include <algorithm>
#include <cstring>

namespace dfem {

bool plan_resident_layout(const SupernodalFactor& F, const std::vector<int>& nseg, const std::vector<int>& cdst, int C,
                          size_t cap_bytes, ResidentPlan& P) {
  const int ns = F.nsuper, L = F.nlevels;
  P = ResidentPlan();
  if (ns == 0 || L == 0 || C < 1 || C > 255) return false;
  auto even = [](size_t v) { return (v + 1) & ~size_t(1); };
  std::vector<int> owner(ns, -1), lvl_of(ns);
  std::vector<size_t> img(ns), buf(ns), work(ns);
  int wmax = 1, rmax = 1;
  for (int q = 0; q < ns; ++q) {
    const size_t w = F.sn_w[q], r = F.sn_r[q];
    img[q] = even(w * (w + 1) / 2) + even(r * w) + even((w + 2) / 2) + even(r);  // blocks, row table, address tables
    buf[q] = 3 * (size_t)nseg[q] + 3 * w + 5;  // inbox, solution values, item record
    work[q] = w * (w + 1) / 2 + r * w;
    wmax = std::max(wmax, (int)w);
    rmax = std::max(rmax, (int)r);
  }
  const size_t reserve = 3 * (size_t)wmax + 3 * (size_t)rmax + 8 + (size_t)L;  // scratch and header
  if (cap_bytes / 8 <= reserve) return false;
  const size_t capd = cap_bytes / 8 - reserve;
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
  P.owner = owner;
  P.items.assign(C, {});
  P.head_len.assign(C, 0);
  P.img_ofs.assign(C + 1, 0);
  std::vector<int> hints(C), dofs(ns), lofs(ns), pofs(ns), tofs(ns), qofs(ns), yofs(ns);
  std::vector<size_t> tsh(C), xrs(C);
  size_t smax = 0;
  for (int c = 0; c < C; ++c) {
    const int n = (int)own[c].size();
    hints[c] = kResHeadInts + (L + 1) + (n + 1);
    const size_t items_at = even((hints[c] + 1) / 2);
    size_t at = items_at + even(((size_t)n * 10 + 1) / 2);
    P.head_len[c] = (int)at;
    for (int q : own[c]) {
      dofs[q] = (int)at; at += even((size_t)F.sn_w[q] * (F.sn_w[q] + 1) / 2);
      lofs[q] = (int)at; at += even((size_t)F.sn_r[q] * F.sn_w[q]);
      pofs[q] = (int)at; at += even(((size_t)F.sn_w[q] + 2) / 2);
      tofs[q] = (int)at; at += even((size_t)F.sn_r[q]);
    }
    P.img_ofs[c + 1] = P.img_ofs[c] + (long long)at;
    for (int q : own[c]) { qofs[q] = (int)at; at += 3 * (size_t)nseg[q]; }
    for (int q : own[c]) { yofs[q] = (int)at; at += 3 * (size_t)F.sn_w[q]; }
    tsh[c] = at; at += 3 * (size_t)wmax;
    xrs[c] = at; at += 3 * (size_t)rmax;
    smax = std::max(smax, at);
    for (int q : own[c])
      P.items[c].push_back({F.sn_c0[q], F.sn_w[q], F.sn_r[q], dofs[q], lofs[q], pofs[q], qofs[q], yofs[q], tofs[q], q});
  }
  if (8 * smax > cap_bytes || smax >= (1u << 24)) return false;
  P.smem_doubles = smax;
  P.img.assign(std::max<long long>(2, P.img_ofs[C]), 0.0);
  for (int c = 0; c < C; ++c) {
    double* base = P.img.data() + P.img_ofs[c];
    int* hdr = reinterpret_cast<int*>(base);
    const int n = (int)own[c].size();
    const size_t items_at = even((hints[c] + 1) / 2);
    int ncols3 = 0;
    for (int q : own[c]) ncols3 += 3 * F.sn_w[q];
    hdr[0] = n; hdr[1] = L; hdr[2] = ncols3; hdr[3] = (int)tsh[c]; hdr[4] = (int)xrs[c]; hdr[5] = (int)items_at;
    int* sched = hdr + kResHeadInts;
    int* cum = sched + L + 1;
    for (int l = 0, k = 0; l <= L; ++l) {
      while (k < n && lvl_of[own[c][k]] < l) ++k;
      sched[l] = k;
    }
    cum[0] = 0;
    for (int k = 0; k < n; ++k) cum[k + 1] = cum[k] + 3 * F.sn_w[own[c][k]];
    std::memcpy(base + items_at, P.items[c].data(), sizeof(ResItem) * n);
    for (int q : own[c]) {
      int* pr = reinterpret_cast<int*>(base + pofs[q]);
      for (int k = 0; k <= F.sn_w[q]; ++k) pr[k] = F.rseg_ptr[F.sn_c0[q] + k] - F.rseg_ptr[F.sn_c0[q]];
      uint32_t* tab = reinterpret_cast<uint32_t*>(base + tofs[q]);
      for (int a = 0; a < F.sn_r[q]; ++a) {
        const size_t p = (size_t)F.sn_rofs[q] + a;
        const int j = F.rowidx[p], d = F.col_sn[j];
        tab[a] = res_addr(owner[d], qofs[d] + 3 * (cdst[p] - F.rseg_ptr[F.sn_c0[d]]));
        tab[F.sn_r[q] + a] = res_addr(owner[d], yofs[d] + 3 * (j - F.sn_c0[d]));
      }
    }
  }
  for (int q = 0; q < ns; ++q) {
    const int c = owner[q];
    P.pack.push_back({F.sn_w[q], F.sn_r[q], (int)F.sn_dofs[q], (int)F.sn_lofs[q], P.img_ofs[c] + dofs[q],
                      P.img_ofs[c] + lofs[q]});
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
