// cholesky.cpp — see cholesky.h.
#include "cholesky.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <numeric>
#include <queue>

namespace dfem {
namespace {

// ---------------------------------------------------------------- ordering --
struct NDContext {
  const SparseSym* A;
  const double* xyz;
  int leaf;
  std::vector<int> tag;   // per-vertex membership tag for the current split
  int next_tag = 1;
  std::vector<int> order;
};

void bfs_split(NDContext& C, const std::vector<int>& verts, std::vector<int>& left,
               std::vector<int>& sep, std::vector<int>& right) {
  // Level-set bisection from a pseudo-peripheral vertex (no coordinates).
  const SparseSym& A = *C.A;
  int t_in = C.next_tag++;
  for (int v : verts) C.tag[v] = t_in;
  std::vector<int> lvl_of;
  auto bfs = [&](int s, std::vector<int>& lv, int& last) {
    lv.clear();
    std::vector<int> q{s};
    int mark = C.next_tag++;
    C.tag[s] = mark;
    std::vector<int> level{0};
    size_t h = 0;
    std::vector<int> dist{0};
    last = s;
    while (h < q.size()) {
      int u = q[h];
      int du = dist[h];
      ++h;
      last = u;
      lv.push_back(du);
      for (int64_t k = A.ptr[u]; k < A.ptr[u + 1]; ++k) {
        int w = A.col[k];
        if (C.tag[w] == t_in) { C.tag[w] = mark; q.push_back(w); dist.push_back(du + 1); }
      }
    }
    // restore membership tag for visited vertices
    for (int u : q) C.tag[u] = t_in;
    return q;
  };
  int last = verts[0];
  std::vector<int> lv;
  std::vector<int> q;
  for (int sweep = 0; sweep < 2; ++sweep) q = bfs(last, lv, last);
  q = bfs(last, lv, last);
  int maxl = lv.empty() ? 0 : lv.back();
  // median level by count
  size_t half = q.size() / 2;
  int mlev = lv[std::min(half, lv.size() - 1)];
  if (mlev == 0 && maxl > 0) mlev = 1;
  std::vector<char> reached(0);
  int t_reach = C.next_tag++;
  for (size_t i = 0; i < q.size(); ++i) {
    C.tag[q[i]] = t_reach;
    if (lv[i] < mlev) left.push_back(q[i]);
    else if (lv[i] == mlev) sep.push_back(q[i]);
    else right.push_back(q[i]);
  }
  for (int v : verts)
    if (C.tag[v] != t_reach) right.push_back(v);  // other components
}

void nd_rec(NDContext& C, std::vector<int> verts) {
  if ((int)verts.size() <= C.leaf) {
    std::sort(verts.begin(), verts.end());
    C.order.insert(C.order.end(), verts.begin(), verts.end());
    return;
  }
  const SparseSym& A = *C.A;
  std::vector<int> left, sep, right;
  if (C.xyz) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int v : verts)
      for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], C.xyz[3 * v + d]); hi[d] = std::max(hi[d], C.xyz[3 * v + d]); }
    int ax = 0;
    for (int d = 1; d < 3; ++d) if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
    std::sort(verts.begin(), verts.end(), [&](int a, int b) {
      double pa = C.xyz[3 * a + ax], pb = C.xyz[3 * b + ax];
      return pa < pb || (pa == pb && a < b);
    });
    size_t mid = verts.size() / 2;
    int tl = C.next_tag++, tr = C.next_tag++;
    for (size_t i = 0; i < verts.size(); ++i) C.tag[verts[i]] = i < mid ? tl : tr;
    // candidate separators: left vertices touching the right, and vice versa
    std::vector<int> sepL, sepR;
    for (size_t i = 0; i < verts.size(); ++i) {
      int v = verts[i];
      int other = (i < mid) ? tr : tl;
      bool touch = false;
      for (int64_t k = A.ptr[v]; k < A.ptr[v + 1] && !touch; ++k) touch = C.tag[A.col[k]] == other;
      if (touch) (i < mid ? sepL : sepR).push_back(v);
    }
    bool useL = sepL.size() <= sepR.size();
    int ts = C.next_tag++;
    for (int v : (useL ? sepL : sepR)) C.tag[v] = ts;
    for (size_t i = 0; i < verts.size(); ++i) {
      int v = verts[i];
      if (C.tag[v] == ts) sep.push_back(v);
      else if (i < mid) left.push_back(v);
      else right.push_back(v);
    }
  } else {
    bfs_split(C, verts, left, sep, right);
  }
  if (left.empty() || right.empty()) {  // no progress: treat as a leaf
    std::sort(verts.begin(), verts.end());
    C.order.insert(C.order.end(), verts.begin(), verts.end());
    return;
  }
  nd_rec(C, std::move(left));
  nd_rec(C, std::move(right));
  std::sort(sep.begin(), sep.end());
  C.order.insert(C.order.end(), sep.begin(), sep.end());
}

// permuted lower pattern: for new column j, rows i > j
void permuted_lower(const SparseSym& A, const std::vector<int>& perm, const std::vector<int>& iperm,
                    std::vector<std::vector<int>>& lower, std::vector<std::vector<int>>& upper) {
  int n = A.n;
  lower.assign(n, {});
  upper.assign(n, {});
  for (int jn = 0; jn < n; ++jn) {
    int jo = perm[jn];
    for (int64_t k = A.ptr[jo]; k < A.ptr[jo + 1]; ++k) {
      int in = iperm[A.col[k]];
      if (in > jn) lower[jn].push_back(in);
      else if (in < jn) upper[jn].push_back(in);
    }
    std::sort(lower[jn].begin(), lower[jn].end());
    lower[jn].erase(std::unique(lower[jn].begin(), lower[jn].end()), lower[jn].end());
  }
}

void etree(int n, const std::vector<std::vector<int>>& upper, std::vector<int>& parent) {
  parent.assign(n, -1);
  std::vector<int> anc(n, -1);
  for (int j = 0; j < n; ++j)
    for (int i : upper[j]) {
      int r = i;
      while (anc[r] != -1 && anc[r] != j) { int nx = anc[r]; anc[r] = j; r = nx; }
      if (anc[r] == -1) { anc[r] = j; parent[r] = j; }
    }
}

std::vector<int> postorder(int n, const std::vector<int>& parent) {
  std::vector<std::vector<int>> kids(n);
  std::vector<int> roots;
  for (int j = 0; j < n; ++j) (parent[j] < 0 ? roots : kids[parent[j]]).push_back(j);
  std::vector<int> post;
  post.reserve(n);
  std::vector<std::pair<int, size_t>> st;
  for (int r : roots) {
    st.push_back({r, 0});
    while (!st.empty()) {
      auto& top = st.back();
      if (top.second < kids[top.first].size()) {
        int c = kids[top.first][top.second++];
        st.push_back({c, 0});
      } else {
        post.push_back(top.first);
        st.pop_back();
      }
    }
  }
  return post;  // post[k] = old node at position k
}

// ------------------------------------------------------------ numeric part --
bool numeric(const SparseSym& A, SupernodalFactor& F, double reg) {
  const int ns = F.nsuper;
  std::vector<std::vector<double>> blk(ns);
  std::vector<int> ld(ns);
  for (int s = 0; s < ns; ++s) {
    ld[s] = F.sn_w[s] + F.sn_r[s];
    blk[s].assign((size_t)ld[s] * F.sn_w[s], 0.0);
  }
  auto local_row = [&](int s, int i) -> int {
    int c0 = F.sn_c0[s], w = F.sn_w[s];
    if (i < c0 + w) return i - c0;
    const int* R = &F.rowidx[F.sn_rofs[s]];
    const int* p = std::lower_bound(R, R + F.sn_r[s], i);
    return w + (int)(p - R);
  };
  // assemble A (lower part, permuted)
  for (int jn = 0; jn < F.n; ++jn) {
    int jo = F.perm[jn];
    int s = F.col_sn[jn];
    int c0 = F.sn_c0[s];
    for (int64_t k = A.ptr[jo]; k < A.ptr[jo + 1]; ++k) {
      int in = F.iperm[A.col[k]];
      if (in < jn) continue;
      blk[s][(size_t)local_row(s, in) + (size_t)(jn - c0) * ld[s]] += A.val[k];
    }
    if (reg != 0.0) blk[s][(size_t)(jn - c0) + (size_t)(jn - c0) * ld[s]] += reg;
  }
  std::vector<double> U;
  std::vector<int> rel;
  for (int s = 0; s < ns; ++s) {
    const int w = F.sn_w[s], r = F.sn_r[s], L = ld[s];
    double* B = blk[s].data();
    // dense Cholesky of the top w x w (column-major, lower)
    for (int c = 0; c < w; ++c) {
      double d = B[c + (size_t)c * L];
      for (int k = 0; k < c; ++k) d -= B[c + (size_t)k * L] * B[c + (size_t)k * L];
      if (!(d > 0.0) || !std::isfinite(d)) return false;
      d = std::sqrt(d);
      B[c + (size_t)c * L] = d;
      for (int i = c + 1; i < L; ++i) {
        double v = B[i + (size_t)c * L];
        for (int k = 0; k < c; ++k) v -= B[i + (size_t)k * L] * B[c + (size_t)k * L];
        B[i + (size_t)c * L] = v / d;
      }
    }
    if (r == 0) continue;
    // U = Lbot Lbot^T (lower, r x r)
    U.assign((size_t)r * r, 0.0);
    for (int a = 0; a < r; ++a)
      for (int b = 0; b <= a; ++b) {
        double v = 0;
        for (int c = 0; c < w; ++c) v += B[(w + a) + (size_t)c * L] * B[(w + b) + (size_t)c * L];
        U[(size_t)a * r + b] = v;
      }
    // scatter into ancestors, grouped by target supernode
    const int* R = &F.rowidx[F.sn_rofs[s]];
    rel.assign(r, 0);
    int b0 = 0;
    while (b0 < r) {
      int p = F.col_sn[R[b0]];
      int b1 = b0;
      while (b1 < r && F.col_sn[R[b1]] == p) ++b1;
      // relative rows of R[b0..r) inside p (merge walk)
      int cp0 = F.sn_c0[p], wp = F.sn_w[p], rp = F.sn_r[p];
      const int* Rp = &F.rowidx[F.sn_rofs[p]];
      int q = 0;  // position in p's row list (cols then Rp)
      for (int a = b0; a < r; ++a) {
        int i = R[a];
        while (true) {
          int gi = q < wp ? cp0 + q : Rp[q - wp];
          if (gi == i) break;
          ++q;
          if (q >= wp + rp) return false;  // structure error (cannot happen for a valid etree)
        }
        rel[a] = q;
      }
      double* Bp = blk[p].data();
      int Lp = ld[p];
      for (int b = b0; b < b1; ++b) {
        int jc = R[b] - cp0;
        for (int a = b; a < r; ++a) Bp[(size_t)rel[a] + (size_t)jc * Lp] -= U[(size_t)a * r + b];
      }
      b0 = b1;
    }
  }
  // split into Ldiag (row-major lower), Dinv (row-major lower), Lcm (column-major r x w)
  F.Ldiag.assign(F.sn_dofs[ns], 0.0);
  F.Dinv.assign(F.sn_dofs[ns], 0.0);
  F.Lcm.assign(F.sn_lofs[ns], 0.0);
  for (int s = 0; s < ns; ++s) {
    const int w = F.sn_w[s], r = F.sn_r[s], L = ld[s];
    const double* B = blk[s].data();
    double* Ld = &F.Ldiag[F.sn_dofs[s]];
    double* Di = &F.Dinv[F.sn_dofs[s]];
    for (int i = 0; i < w; ++i)
      for (int c = 0; c <= i; ++c) Ld[(size_t)i * w + c] = B[i + (size_t)c * L];
    // inverse of the lower-triangular diagonal block, column by column
    for (int c = 0; c < w; ++c) {
      for (int i = c; i < w; ++i) {
        double v = (i == c) ? 1.0 : 0.0;
        for (int k = c; k < i; ++k) v -= Ld[(size_t)i * w + k] * Di[(size_t)k * w + c];
        Di[(size_t)i * w + c] = v / Ld[(size_t)i * w + i];
      }
    }
    double* Lc = &F.Lcm[F.sn_lofs[s]];
    for (int c = 0; c < w; ++c)
      for (int a = 0; a < r; ++a) Lc[(size_t)c * r + a] = B[(w + a) + (size_t)c * L];
  }
  F.reg = reg;
  return true;
}

bool numeric_with_retry(const SparseSym& A, SupernodalFactor& F, std::string& err) {
  // World::FactorizeLDLT: on failure retry with A + reg I, reg = 1e-5, x10 ... (bounded here)
  double reg = 0.0;
  for (int attempt = 0; attempt < 25; ++attempt) {
    if (numeric(A, F, reg)) return true;
    reg = (reg == 0.0) ? 1e-5 : reg * 10.0;
  }
  err = "Cholesky factorisation failed after 25 regularisation retries";
  return false;
}

}  // namespace

bool factorize(const SparseSym& A, const double* coords, const FactorOptions& opt,
               SupernodalFactor& F, std::string& err) {
  const int n = A.n;
  F = SupernodalFactor();
  F.n = n;
  if (n == 0) { err = "empty matrix"; return false; }
  // 1. nested dissection
  NDContext C;
  C.A = &A;
  C.xyz = coords;
  C.leaf = std::max(4, opt.leaf_size);
  C.tag.assign(n, 0);
  std::vector<int> all(n);
  std::iota(all.begin(), all.end(), 0);
  nd_rec(C, all);
  std::vector<int> perm = C.order;
  if ((int)perm.size() != n) { err = "ordering lost vertices"; return false; }
  std::vector<int> iperm(n);
  for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
  // 2. etree + postorder
  std::vector<std::vector<int>> lower, upper;
  permuted_lower(A, perm, iperm, lower, upper);
  std::vector<int> parent;
  etree(n, upper, parent);
  std::vector<int> post = postorder(n, parent);
  {
    std::vector<int> p2(n);
    for (int k = 0; k < n; ++k) p2[k] = perm[post[k]];
    perm.swap(p2);
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    permuted_lower(A, perm, iperm, lower, upper);
    etree(n, upper, parent);
  }
  // 3. column structures (rows > j)
  std::vector<std::vector<int>> colst(n);
  std::vector<std::vector<int>> kids(n);
  for (int j = 0; j < n; ++j)
    if (parent[j] >= 0) kids[parent[j]].push_back(j);
  std::vector<int> mark(n, -1);
  for (int j = 0; j < n; ++j) {
    std::vector<int>& st = colst[j];
    for (int i : lower[j]) if (mark[i] != j) { mark[i] = j; st.push_back(i); }
    for (int c : kids[j])
      for (int i : colst[c])
        if (i > j && mark[i] != j) { mark[i] = j; st.push_back(i); }
    std::sort(st.begin(), st.end());
  }
  // 4. fundamental supernodes
  std::vector<int> start;  // first columns
  for (int j = 0; j < n; ++j) {
    bool join = false;
    if (j > 0 && !start.empty()) {
      int s0 = start.back();
      join = parent[j - 1] == j && kids[j].size() == 1 &&
             colst[j - 1].size() == colst[j].size() + 1 && (j - s0) < opt.max_width;
    }
    if (!join) start.push_back(j);
  }
  // 5. relaxed amalgamation of a last child into its parent
  struct SN { int c0, c1; };
  std::vector<SN> sns;
  for (size_t k = 0; k < start.size(); ++k)
    sns.push_back({start[k], k + 1 < start.size() ? start[k + 1] : n});
  std::vector<SN> merged;
  auto rows_below = [&](const SN& s) { return (int)colst[s.c1 - 1].size(); };
  for (const SN& p : sns) {
    SN cur = p;
    while (!merged.empty()) {
      SN& c = merged.back();
      if (c.c1 != cur.c0 || parent[c.c1 - 1] != cur.c0) break;
      int wc = c.c1 - c.c0, wp = cur.c1 - cur.c0;
      if (wc + wp > opt.max_width) break;
      int rc = rows_below(c), rp = rows_below(cur);
      int64_t extra = (int64_t)wc * (wp + rp - rc);
      int64_t total = (int64_t)(wc + wp) * (wc + wp + 1) / 2 + (int64_t)rp * (wc + wp);
      bool ok = (wc + wp <= opt.relax_small) || (extra <= opt.relax_frac * total);
      if (!ok) break;
      cur.c0 = c.c0;
      merged.pop_back();
    }
    merged.push_back(cur);
  }
  // 6. supernode tables
  F.nsuper = (int)merged.size();
  F.col_sn.assign(n, 0);
  F.sn_rofs.assign(F.nsuper + 1, 0);
  F.sn_lofs.assign(F.nsuper + 1, 0);
  F.sn_dofs.assign(F.nsuper + 1, 0);
  for (int s = 0; s < F.nsuper; ++s) {
    int c0 = merged[s].c0, c1 = merged[s].c1, w = c1 - c0;
    F.sn_c0.push_back(c0);
    F.sn_w.push_back(w);
    for (int j = c0; j < c1; ++j) F.col_sn[j] = s;
    const std::vector<int>& st = colst[c1 - 1];
    F.sn_r.push_back((int)st.size());
    F.rowidx.insert(F.rowidx.end(), st.begin(), st.end());
    F.sn_rofs[s + 1] = F.sn_rofs[s] + (int64_t)st.size();
    // dense blocks start and end on 16 bytes (even count of doubles) so the GPU
    // can move each one with a single bulk asynchronous copy
    auto even = [](int64_t v) { return (v + 1) & ~int64_t(1); };
    F.sn_lofs[s + 1] = F.sn_lofs[s] + even((int64_t)st.size() * w);
    F.sn_dofs[s + 1] = F.sn_dofs[s] + even((int64_t)w * w);
  }
  // row -> contribution slots (positions in rowidx holding that row)
  F.rseg_ptr.assign(n + 1, 0);
  for (int i : F.rowidx) F.rseg_ptr[i + 1]++;
  for (int i = 0; i < n; ++i) F.rseg_ptr[i + 1] += F.rseg_ptr[i];
  F.rseg_pos.assign(F.rowidx.size(), 0);
  {
    std::vector<int> fill(F.rseg_ptr.begin(), F.rseg_ptr.end() - 1);
    for (size_t p = 0; p < F.rowidx.size(); ++p) F.rseg_pos[fill[F.rowidx[p]]++] = (int)p;
  }
  F.sn_parent.assign(F.nsuper, -1);
  for (int s = 0; s < F.nsuper; ++s) {
    int last = F.sn_c0[s] + F.sn_w[s] - 1;
    if (parent[last] >= 0) F.sn_parent[s] = F.col_sn[parent[last]];
  }
  // 7. levels (leaves = 0)
  std::vector<int> level(F.nsuper, 0);
  for (int s = 0; s < F.nsuper; ++s)  // children precede parents
    if (F.sn_parent[s] >= 0) level[F.sn_parent[s]] = std::max(level[F.sn_parent[s]], level[s] + 1);
  F.nlevels = 0;
  for (int s = 0; s < F.nsuper; ++s) F.nlevels = std::max(F.nlevels, level[s] + 1);
  F.lvl_ptr.assign(F.nlevels + 1, 0);
  for (int s = 0; s < F.nsuper; ++s) F.lvl_ptr[level[s] + 1]++;
  for (int l = 0; l < F.nlevels; ++l) F.lvl_ptr[l + 1] += F.lvl_ptr[l];
  F.lvl_sn.assign(F.nsuper, 0);
  {
    std::vector<int> fill(F.lvl_ptr.begin(), F.lvl_ptr.end() - 1);
    for (int s = 0; s < F.nsuper; ++s) F.lvl_sn[fill[level[s]]++] = s;
  }
  F.perm = perm;
  F.iperm = iperm;
  F.nnz_factor = 0;
  for (int s = 0; s < F.nsuper; ++s)
    F.nnz_factor += (int64_t)F.sn_w[s] * (F.sn_w[s] + 1) / 2 + (int64_t)F.sn_w[s] * F.sn_r[s];
  return numeric_with_retry(A, F, err);
}

bool refactorize(const SparseSym& A, SupernodalFactor& F, std::string& err) {
  return numeric_with_retry(A, F, err);
}

void host_solve(const SupernodalFactor& F, const double* b, double* x) {
  const int n = F.n;
  std::vector<double> y(3 * (size_t)n);
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) y[3 * i + c] = b[3 * F.perm[i] + c];
  // forward: L y = b, supernode by supernode, push form
  std::vector<double> contrib(3 * F.rowidx.size(), 0.0);
  for (int s = 0; s < F.nsuper; ++s) {
    int c0 = F.sn_c0[s], w = F.sn_w[s], r = F.sn_r[s];
    std::vector<double> t(3 * (size_t)w);
    for (int c = 0; c < w; ++c) {
      int i = c0 + c;
      double a0 = y[3 * i], a1 = y[3 * i + 1], a2 = y[3 * i + 2];
      for (int k = F.rseg_ptr[i]; k < F.rseg_ptr[i + 1]; ++k) {
        const double* q = &contrib[3 * (size_t)F.rseg_pos[k]];
        a0 -= q[0]; a1 -= q[1]; a2 -= q[2];
      }
      t[3 * c] = a0; t[3 * c + 1] = a1; t[3 * c + 2] = a2;
    }
    const double* Di = &F.Dinv[F.sn_dofs[s]];
    for (int c = 0; c < w; ++c) {
      double a0 = 0, a1 = 0, a2 = 0;
      for (int k = 0; k <= c; ++k) {
        double d = Di[(size_t)c * w + k];
        a0 += d * t[3 * k]; a1 += d * t[3 * k + 1]; a2 += d * t[3 * k + 2];
      }
      y[3 * (c0 + c)] = a0; y[3 * (c0 + c) + 1] = a1; y[3 * (c0 + c) + 2] = a2;
    }
    const double* Lc = &F.Lcm[F.sn_lofs[s]];
    for (int a = 0; a < r; ++a) {
      double a0 = 0, a1 = 0, a2 = 0;
      for (int c = 0; c < w; ++c) {
        double l = Lc[(size_t)c * r + a];
        a0 += l * y[3 * (c0 + c)]; a1 += l * y[3 * (c0 + c) + 1]; a2 += l * y[3 * (c0 + c) + 2];
      }
      double* q = &contrib[3 * (size_t)(F.sn_rofs[s] + a)];
      q[0] = a0; q[1] = a1; q[2] = a2;
    }
  }
  // backward: L^T x = y
  for (int s = F.nsuper - 1; s >= 0; --s) {
    int c0 = F.sn_c0[s], w = F.sn_w[s], r = F.sn_r[s];
    const int* R = &F.rowidx[F.sn_rofs[s]];
    const double* Lc = &F.Lcm[F.sn_lofs[s]];
    std::vector<double> u(3 * (size_t)w);
    for (int c = 0; c < w; ++c) {
      double a0 = y[3 * (c0 + c)], a1 = y[3 * (c0 + c) + 1], a2 = y[3 * (c0 + c) + 2];
      for (int a = 0; a < r; ++a) {
        double l = Lc[(size_t)c * r + a];
        int i = R[a];
        a0 -= l * y[3 * i]; a1 -= l * y[3 * i + 1]; a2 -= l * y[3 * i + 2];
      }
      u[3 * c] = a0; u[3 * c + 1] = a1; u[3 * c + 2] = a2;
    }
    const double* Di = &F.Dinv[F.sn_dofs[s]];
    for (int c = 0; c < w; ++c) {
      double a0 = 0, a1 = 0, a2 = 0;
      for (int k = c; k < w; ++k) {
        double d = Di[(size_t)k * w + c];
        a0 += d * u[3 * k]; a1 += d * u[3 * k + 1]; a2 += d * u[3 * k + 2];
      }
      y[3 * (c0 + c)] = a0; y[3 * (c0 + c) + 1] = a1; y[3 * (c0 + c) + 2] = a2;
    }
  }
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) x[3 * F.perm[i] + c] = y[3 * i + c];
}

}  // namespace dfem
