// scene.cpp — see scene.h.
#include "scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace dfem {
namespace {

struct P3 { double x, y, z; };
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double dotp(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline P3 crossp(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double normp(P3 a) { return std::sqrt(dotp(a, a)); }
inline P3 pt(const double* x, int i) { return {x[3 * i], x[3 * i + 1], x[3 * i + 2]}; }

// Element setup shared by corotated and muscle constraints (diff_fem
// sim/Dfobj.h:474-503, sim/Muscle.h:135-150): Dm = [p1-p0, p2-p0, p3-p0];
// when det(Dm) < 0 the vertices 1 and 2 swap; vol = det/6; invDm = Dm^-1
// (row-major here).
bool element(const double* x0, const int* idx, int out_idx[4], double inv[9], double& vol) {
  int i0 = idx[0], i1 = idx[1], i2 = idx[2], i3 = idx[3];
  P3 a = sub(pt(x0, i1), pt(x0, i0)), b = sub(pt(x0, i2), pt(x0, i0)), c = sub(pt(x0, i3), pt(x0, i0));
  double det = dotp(a, crossp(b, c));
  if (det < 0) {
    std::swap(i1, i2);
    std::swap(a, b);
    det = -det;
  }
  if (!(det > 0) || !std::isfinite(det)) return false;
  out_idx[0] = i0; out_idx[1] = i1; out_idx[2] = i2; out_idx[3] = i3;
  vol = det / 6.0;
  // Dm columns a, b, c; inverse rows are (b x c, c x a, a x b) / det
  P3 r0 = crossp(b, c), r1 = crossp(c, a), r2 = crossp(a, b);
  const P3 rows[3] = {r0, r1, r2};
  for (int r = 0; r < 3; ++r) {
    inv[3 * r + 0] = rows[r].x / det;
    inv[3 * r + 1] = rows[r].y / det;
    inv[3 * r + 2] = rows[r].z / det;
  }
  return true;
}

// G[v][j]: F(:,j) = sum_v G[v][j] x_v (rows of the reference's A_i,
// CorotateFEMConstraint.h:236-245)
void gcoef(const double* inv, double G[4][3]) {
  for (int j = 0; j < 3; ++j) {
    double s = 0;
    for (int k = 0; k < 3; ++k) { G[k + 1][j] = inv[3 * k + j]; s += inv[3 * k + j]; }
    G[0][j] = -s;
  }
}

double mv_cos(P3 a, P3 b, P3 c) { P3 e1 = sub(a, b), e2 = sub(c, b); return dotp(e1, e2) / (normp(e1) * normp(e2)); }
double mv_sin(P3 a, P3 b, P3 c) { P3 e1 = sub(a, b), e2 = sub(c, b); return normp(crossp(e1, e2)) / (normp(e1) * normp(e2)); }
double mv_weight(P3 a, P3 b, P3 c) {  // BendingConstraint::getMeanValue
  double num = 1.0 - mv_cos(a, b, c);
  return num == 0 ? 0.0 : num / mv_sin(a, b, c);
}

struct Triplets {
  std::vector<int> r, c;
  std::vector<double> v;
  void add(int i, int j, double x) { r.push_back(i); c.push_back(j); v.push_back(x); }
};

SparseSym to_csr(int n, const Triplets& t) {
  SparseSym A;
  A.n = n;
  std::vector<int64_t> cnt(n + 1, 0);
  for (int i : t.r) cnt[i + 1]++;
  for (int i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
  std::vector<int> col(t.r.size());
  std::vector<double> val(t.r.size());
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (size_t k = 0; k < t.r.size(); ++k) { int64_t p = fill[t.r[k]]++; col[p] = t.c[k]; val[p] = t.v[k]; }
  // sort + merge each row
  A.ptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    std::vector<std::pair<int, double>> row;
    for (int64_t k = cnt[i]; k < cnt[i + 1]; ++k) row.push_back({col[k], val[k]});
    std::sort(row.begin(), row.end(), [](auto& a, auto& b) { return a.first < b.first; });
    for (auto& e : row) {
      if (!A.col.empty() && (int64_t)A.col.size() > A.ptr[i] && A.col.back() == e.first) A.val.back() += e.second;
      else { A.col.push_back(e.first); A.val.push_back(e.second); }
    }
    A.ptr[i + 1] = (int64_t)A.col.size();
  }
  return A;
}

// Hs = M/h^2 + L_s in the numbering of the given tables (World.h:1093-1098).
SparseSym assemble_hs(const HostScene& s) {
  Triplets t;
  const double ih2 = 1.0 / (s.h * s.h);
  for (int i = 0; i < s.N; ++i) t.add(i, i, s.mass[i] * ih2);
  for (int e = 0; e < s.T; ++e) {
    double G[4][3];
    gcoef(&s.tinv[9 * e], G);
    // mu vol (1 + nu) G G^T = E vol G G^T (two blocks of CorotateFEMConstraint::EvaluateLMatrix)
    double mu = s.tE[e] / (1.0 + s.tnu[e]);
    double w = mu * s.tvol[e] * (1.0 + s.tnu[e]);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        double g = G[a][0] * G[b][0] + G[a][1] * G[b][1] + G[a][2] * G[b][2];
        t.add(s.tv[4 * e + a], s.tv[4 * e + b], w * g);
      }
  }
  for (int a = 0; a < s.A; ++a) t.add(s.av[a], s.av[a], s.ak[a]);
  for (int m = 0; m < s.M; ++m) {
    double G[4][3];
    gcoef(&s.minv[9 * m], G);
    double c[4];
    for (int v = 0; v < 4; ++v) c[v] = G[v][0] * s.mfib[3 * m] + G[v][1] * s.mfib[3 * m + 1] + G[v][2] * s.mfib[3 * m + 2];
    double w = s.mvol[m] * s.mk[m];  // LinearMuscleConstraint::EvaluateLMatrix
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) t.add(s.mv[4 * m + a], s.mv[4 * m + b], w * c[a] * c[b]);
  }
  for (int k = 0; k < s.S; ++k) {  // SpringConstraint::EvaluateLMatrix: sqrt(w) A^T A
    int i0 = s.sv[2 * k], i1 = s.sv[2 * k + 1];
    double w = s.ssw[k];
    t.add(i0, i0, w); t.add(i1, i1, w); t.add(i0, i1, -w); t.add(i1, i0, -w);
  }
  for (int b = 0; b < s.B; ++b) {  // BendingConstraint::EvaluateLMatrix: w * (w beta)^T (w beta)
    double w3 = s.bw[b] * s.bw[b] * s.bw[b];
    for (int p = s.boff[b]; p < s.boff[b + 1]; ++p)
      for (int q = s.boff[b]; q < s.boff[b + 1]; ++q) t.add(s.bv[p], s.bv[q], w3 * s.bbeta[p] * s.bbeta[q]);
  }
  return to_csr(s.N, t);
}

void build_slots(HostScene& s) {
  // constraint-local slots -> vertex
  std::vector<int> vert;
  vert.reserve(4 * s.T + 4 * s.M + 2 * s.S + s.bv.size());
  for (int e = 0; e < 4 * s.T; ++e) vert.push_back(s.tv[e]);
  for (int e = 0; e < 4 * s.M; ++e) vert.push_back(s.mv[e]);
  for (int e = 0; e < 2 * s.S; ++e) vert.push_back(s.sv[e]);
  for (size_t e = 0; e < s.bv.size(); ++e) vert.push_back(s.bv[e]);
  s.nslots = (int)vert.size();
  s.vslot_ptr.assign(s.N + 1, 0);
  for (int v : vert) s.vslot_ptr[v + 1]++;
  for (int i = 0; i < s.N; ++i) s.vslot_ptr[i + 1] += s.vslot_ptr[i];
  std::vector<int> fill(s.vslot_ptr.begin(), s.vslot_ptr.end() - 1);
  std::vector<int> pos(vert.size());
  for (size_t k = 0; k < vert.size(); ++k) pos[k] = fill[vert[k]]++;
  size_t o = 0;
  s.tslot.assign(pos.begin() + o, pos.begin() + o + 4 * s.T); o += 4 * s.T;
  s.mslot.assign(pos.begin() + o, pos.begin() + o + 4 * s.M); o += 4 * s.M;
  s.sslot.assign(pos.begin() + o, pos.begin() + o + 2 * s.S); o += 2 * s.S;
  s.bslot.assign(pos.begin() + o, pos.end());
}

void renumber(HostScene& s, const std::vector<int>& to_int) {
  auto remap = [&](std::vector<int>& v) { for (int& i : v) i = to_int[i]; };
  remap(s.tv); remap(s.mv); remap(s.sv); remap(s.bv); remap(s.av); remap(s.cverts);
  std::vector<double> x(3 * (size_t)s.N), m(s.N), g(s.N);
  for (int i = 0; i < s.N; ++i) {
    int j = to_int[i];
    for (int c = 0; c < 3; ++c) x[3 * j + c] = s.x0[3 * i + c];
    m[j] = s.mass[i];
    g[j] = s.gmask[i];
  }
  s.x0.swap(x); s.mass.swap(m); s.gmask.swap(g);
}

#define REQ(cond, msg) do { if (!(cond)) { err = msg; return false; } } while (0)

}  // namespace

bool build_host_scene(const dfem_scene_desc& d, HostScene& s, std::string& err) {
  REQ(d.n_vertices > 0 && d.x0 && d.mass, "descriptor: need n_vertices > 0, x0 and mass");
  REQ(d.time_step > 0 && std::isfinite(d.time_step), "descriptor: time_step must be positive");
  REQ(d.max_iterations >= 0 && d.max_iterations <= 100000, "descriptor: max_iterations out of range");
  REQ(d.n_tets >= 0 && d.n_attach >= 0 && d.n_muscle >= 0 && d.n_springs >= 0 && d.n_bending >= 0,
      "descriptor: negative count");
  REQ(d.n_tets == 0 || (d.tets && d.youngs && d.poisson), "descriptor: tets/youngs/poisson missing");
  REQ(d.n_attach == 0 || (d.attach_vertex && d.attach_target && d.attach_stiffness), "descriptor: attachment arrays missing");
  REQ(d.n_muscle == 0 || (d.muscle_tets && d.muscle_fiber && d.muscle_stiffness && d.muscle_segment && d.n_segments > 0),
      "descriptor: muscle arrays missing");
  REQ(d.n_springs == 0 || (d.spring_vertices && d.spring_weight), "descriptor: spring arrays missing");
  REQ(d.n_bending == 0 || (d.bend_offsets && d.bend_vertices && d.bend_weight), "descriptor: bending arrays missing");
  REQ(d.precision == DFEM_PREC_FP64 || d.precision == DFEM_PREC_MIXED, "descriptor: unknown precision");
  const int N = d.n_vertices;
  auto inrange = [&](const int32_t* p, int64_t n) {
    for (int64_t k = 0; k < n; ++k) if (p[k] < 0 || p[k] >= N) return false;
    return true;
  };
  REQ(inrange(d.tets, 4LL * d.n_tets), "descriptor: tet vertex index out of range");
  REQ(inrange(d.attach_vertex, d.n_attach), "descriptor: attachment vertex out of range");
  REQ(inrange(d.muscle_tets, 4LL * d.n_muscle), "descriptor: muscle vertex out of range");
  REQ(inrange(d.spring_vertices, 2LL * d.n_springs), "descriptor: spring vertex out of range");
  for (int i = 0; i < N; ++i) {
    REQ(d.mass[i] > 0 && std::isfinite(d.mass[i]), "descriptor: masses must be positive and finite");
    for (int c = 0; c < 3; ++c) REQ(std::isfinite(d.x0[3 * i + c]), "descriptor: non-finite rest position");
  }
  s = HostScene();
  s.N = N;
  s.x0.assign(d.x0, d.x0 + 3 * (size_t)N);
  s.mass.assign(d.mass, d.mass + N);
  s.gmask.assign(N, 1.0);
  if (d.gravity_mask) for (int i = 0; i < N; ++i) s.gmask[i] = d.gravity_mask[i] ? 1.0 : 0.0;
  s.h = d.time_step; s.K = d.max_iterations; s.damping = d.damping;
  for (int c = 0; c < 3; ++c) s.g[c] = d.gravity[c];
  s.precision = d.precision;
  s.checkpoint_every = std::max(1, d.checkpoint_every);

  s.T = d.n_tets;
  s.tv.resize(4 * (size_t)s.T); s.tinv.resize(9 * (size_t)s.T); s.tvol.resize(s.T);
  s.tE.assign(d.youngs, d.youngs + s.T); s.tnu.assign(d.poisson, d.poisson + s.T);
  for (int e = 0; e < s.T; ++e) {
    REQ(element(d.x0, d.tets + 4 * e, &s.tv[4 * e], &s.tinv[9 * e], s.tvol[e]), "descriptor: degenerate tet (zero volume)");
    REQ(std::isfinite(s.tE[e]) && std::isfinite(s.tnu[e]) && s.tnu[e] > -1.0, "descriptor: invalid material");
  }
  REQ(d.n_contact_vertices >= 0 && d.n_obstacle_vertices >= 0 && d.n_obstacle_faces >= 0, "descriptor: negative contact count");
  REQ(d.n_contact_vertices == 0 || d.contact_vertices, "descriptor: contact_vertices missing");
  REQ(inrange(d.contact_vertices, d.n_contact_vertices), "descriptor: contact vertex out of range");
  REQ(d.n_obstacle_faces == 0 || (d.obstacle_faces && d.obstacle_x), "descriptor: obstacle arrays missing");
  for (int64_t k = 0; k < 3LL * d.n_obstacle_faces; ++k)
    REQ(d.obstacle_faces[k] >= 0 && d.obstacle_faces[k] < d.n_obstacle_vertices, "descriptor: obstacle face index out of range");
  s.collide = d.handle_collision != 0;
  s.alpha = d.alpha;
  s.mu_obs = d.obstacle_friction;
  s.cverts.assign(d.contact_vertices, d.contact_vertices + d.n_contact_vertices);
  s.obs_x.assign(d.obstacle_x, d.obstacle_x + 3 * (size_t)d.n_obstacle_vertices);
  s.obs_f.assign(d.obstacle_faces, d.obstacle_faces + 3 * (size_t)d.n_obstacle_faces);

  s.A = d.n_attach;
  s.av.assign(d.attach_vertex, d.attach_vertex + s.A);
  s.ap.assign(d.attach_target, d.attach_target + 3 * (size_t)s.A);
  s.ak.assign(d.attach_stiffness, d.attach_stiffness + s.A);

  s.M = d.n_muscle; s.nseg = s.M > 0 ? d.n_segments : std::max(0, d.n_segments);
  s.mv.resize(4 * (size_t)s.M); s.minv.resize(9 * (size_t)s.M); s.mvol.resize(s.M);
  s.mk.assign(d.muscle_stiffness, d.muscle_stiffness + s.M);
  s.mfib.assign(d.muscle_fiber, d.muscle_fiber + 3 * (size_t)s.M);
  s.mseg.assign(d.muscle_segment, d.muscle_segment + s.M);
  for (int m = 0; m < s.M; ++m) {
    REQ(element(d.x0, d.muscle_tets + 4 * m, &s.mv[4 * m], &s.minv[9 * m], s.mvol[m]), "descriptor: degenerate muscle tet");
    REQ(s.mseg[m] >= 0 && s.mseg[m] < s.nseg, "descriptor: muscle segment id out of range");
  }
  s.seg_ptr.assign(s.nseg + 1, 0);
  for (int m = 0; m < s.M; ++m) s.seg_ptr[s.mseg[m] + 1]++;
  for (int q = 0; q < s.nseg; ++q) s.seg_ptr[q + 1] += s.seg_ptr[q];
  s.seg_mus.assign(s.M, 0);
  {
    std::vector<int> fill(s.seg_ptr.begin(), s.seg_ptr.end() - 1);
    for (int m = 0; m < s.M; ++m) s.seg_mus[fill[s.mseg[m]]++] = m;
  }

  s.S = d.n_springs;
  s.sv.assign(d.spring_vertices, d.spring_vertices + 2 * (size_t)s.S);
  s.srest.resize(s.S); s.ssw.resize(s.S);
  for (int k = 0; k < s.S; ++k) {
    int i0 = s.sv[2 * k], i1 = s.sv[2 * k + 1];
    REQ(i0 != i1, "descriptor: spring with identical vertices");
    s.srest[k] = d.spring_rest ? d.spring_rest[k] : normp(sub(pt(d.x0, i0), pt(d.x0, i1)));  // getEdgeLength
    REQ(d.spring_weight[k] >= 0, "descriptor: negative spring weight");
    s.ssw[k] = std::sqrt(d.spring_weight[k]);  // SpringConstraint: mStretch = sqrt(weight)
  }

  s.B = d.n_bending;
  s.boff.assign(d.bend_offsets, d.bend_offsets + s.B + 1);
  if (s.B > 0) {
    REQ(s.boff[0] == 0, "descriptor: bend_offsets must start at 0");
    for (int b = 0; b < s.B; ++b) REQ(s.boff[b + 1] - s.boff[b] >= 4, "descriptor: bending stencil needs a ring of >= 3");
    s.bv.assign(d.bend_vertices, d.bend_vertices + s.boff[s.B]);
    REQ(inrange(s.bv.data(), (int64_t)s.bv.size()), "descriptor: bending vertex out of range");
  }
  s.bw.assign(d.bend_weight, d.bend_weight + s.B);
  s.bbeta.assign(s.bv.size(), 0.0);
  s.brest.assign(s.B, 0.0);
  for (int b = 0; b < s.B; ++b) {
    // mean-value Laplace-Beltrami coefficients (BendingConstraint.h:220-276)
    int o = s.boff[b], nr = s.boff[b + 1] - o - 1;
    P3 mid = pt(d.x0, s.bv[o]);
    double sum = 0;
    for (int i = 0; i < nr; ++i) {
      P3 vi = pt(d.x0, s.bv[o + 1 + i]);
      P3 cw = pt(d.x0, s.bv[o + 1 + (i + 1) % nr]);
      P3 ccw = pt(d.x0, s.bv[o + 1 + (i + nr - 1) % nr]);
      double coeff = (mv_weight(vi, mid, cw) + mv_weight(vi, ccw, mid)) / normp(sub(vi, mid));
      s.bbeta[o + 1 + i] = -coeff;
      sum += coeff;
    }
    s.bbeta[o] = sum;
    // The reference evaluates the rest-state Laplacian before its coefficient
    // list is filled (BendingConstraint.h:83-95), so its rest norm is 0; kept.
    s.brest[b] = 0.0;
  }

  // Hs in user numbering, ordering + factorisation
  s.Hs = assemble_hs(s);
  FactorOptions opt;
  if (!factorize(s.Hs, s.x0.data(), opt, s.F, err)) return false;
  s.to_internal = s.F.iperm;
  s.to_user = s.F.perm;
  renumber(s, s.to_internal);
  // the factor's numbering is now the internal one
  for (int i = 0; i < N; ++i) { s.F.perm[i] = i; s.F.iperm[i] = i; }
  s.Hs = assemble_hs(s);
  build_slots(s);
  return true;
}

bool update_materials(HostScene& s, const double* E, const double* nu, std::string& err) {
  for (int e = 0; e < s.T; ++e) {
    if (!std::isfinite(E[e]) || !std::isfinite(nu[e]) || !(nu[e] > -1.0)) { err = "invalid material"; return false; }
    s.tE[e] = E[e];
    s.tnu[e] = nu[e];
  }
  s.Hs = assemble_hs(s);
  return refactorize(s.Hs, s.F, err);
}

}  // namespace dfem
