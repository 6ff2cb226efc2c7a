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
// E (per tet, may be null) overrides the tets' Young's moduli.
SparseSym assemble_hs(const HostScene& s, const double* E = nullptr) {
  Triplets t;
  const double ih2 = 1.0 / (s.h * s.h);
  for (int i = 0; i < s.N; ++i) t.add(i, i, s.mass[i] * ih2);
  for (int e = 0; e < s.T; ++e) {
    double G[4][3];
    gcoef(&s.tinv[9 * e], G);
    // mu vol (1 + nu) G G^T = E vol G G^T (two blocks of CorotateFEMConstraint::EvaluateLMatrix)
    const double Ee = E ? E[e] : s.tE[e];
    double mu = Ee / (1.0 + s.tnu[e]);
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
  remap(s.tv); remap(s.mv); remap(s.sv); remap(s.bv); remap(s.av); remap(s.cverts); remap(s.df); remap(s.lvert);
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
  // soft-soft contact (World::m_handle_self_collision, on only with collision
  // handling): the soft faces, by contact index (indices survive the
  // renumbering below, which maps the contact vertices in place)
  s.mu_self = d.friction;
  s.self_collide = s.collide && d.self_collision != 0 && d.n_contact_faces > 0 && !s.cverts.empty();
  if (s.self_collide) {
    REQ(d.contact_faces, "descriptor: contact_faces missing");
    REQ(d.n_contact_faces < INT32_MAX / 9, "descriptor: too many contact faces");
    const int nc = (int)s.cverts.size();
    std::vector<int> cid(N, -1);
    for (int a = 0; a < nc; ++a) {
      REQ(cid[s.cverts[a]] < 0, "descriptor: contact vertex listed twice");
      cid[s.cverts[a]] = a;
    }
    s.cfaces.resize(3 * (size_t)d.n_contact_faces);
    s.on_face.assign(nc, 0);
    s.cvf_ptr.assign(nc + 1, 0);
    for (int64_t k = 0; k < 3LL * d.n_contact_faces; ++k) {
      const int gv = d.contact_faces[k];
      REQ(gv >= 0 && gv < N && cid[gv] >= 0, "descriptor: contact face vertex is not a contact vertex");
      s.cfaces[k] = cid[gv];
      s.on_face[cid[gv]] = 1;
      s.cvf_ptr[cid[gv] + 1]++;
    }
    for (int a = 0; a < nc; ++a) s.cvf_ptr[a + 1] += s.cvf_ptr[a];
    s.cvf_face.assign(s.cvf_ptr[nc], 0);
    std::vector<int> fill(s.cvf_ptr.begin(), s.cvf_ptr.end() - 1);
    for (int f = 0; f < d.n_contact_faces; ++f)  // faces ascending per vertex
      for (int q = 0; q < 3; ++q) s.cvf_face[fill[s.cfaces[3 * f + q]]++] = f;
  }
  REQ(d.n_drag_faces >= 0 && d.n_drag_faces < INT32_MAX / 3 && (d.n_drag_faces == 0 || d.drag_faces),
      "descriptor: drag_faces missing or too many");
  REQ(inrange(d.drag_faces, 3LL * d.n_drag_faces), "descriptor: drag face vertex out of range");
  s.underwater = d.underwater != 0;
  if (s.underwater) std::fill(s.gmask.begin(), s.gmask.end(), 0.0);  // Environment::Step: no gravity underwater
  s.df.assign(d.drag_faces, d.drag_faces + 3 * (size_t)d.n_drag_faces);
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
  s.S = d.n_springs;
  s.sv.assign(d.spring_vertices, d.spring_vertices + 2 * (size_t)s.S);
  s.srest.resize(s.S); s.ssw.resize(s.S);
  for (int k = 0; k < s.S; ++k) {
    int i0 = s.sv[2 * k], i1 = s.sv[2 * k + 1];
    REQ(i0 != i1, "descriptor: spring with identical vertices");
    s.srest[k] = d.spring_rest ? d.spring_rest[k] : normp(sub(pt(d.x0, i0), pt(d.x0, i1)));  // getEdgeLength
    REQ(d.spring_weight[k] >= 0, "descriptor: negative spring weight");
    // SpringConstraint and PneumaticConstraint alike: mStretch = sqrt(weight)
    s.ssw[k] = std::sqrt(d.spring_weight[k]);
  }
  // pneumatic springs (Dfobj.h:232-251 builds one per consecutive pair of a
  // "Volume Verts" polyline; SetActions sets each one's activation directly)
  bool any_channel = false;
  if (d.spring_channel)
    for (int k = 0; k < s.S; ++k) {
      REQ(d.spring_channel[k] >= -1 && d.spring_channel[k] < s.nseg, "descriptor: spring channel out of range");
      any_channel = any_channel || d.spring_channel[k] >= 0;
    }
  if (any_channel) s.sch.assign(d.spring_channel, d.spring_channel + s.S);

  // channel -> members CSR (muscle m as m, pneumatic spring k as -(k+1)),
  // muscles first, each in ascending order
  s.seg_ptr.assign(s.nseg + 1, 0);
  for (int m = 0; m < s.M; ++m) s.seg_ptr[s.mseg[m] + 1]++;
  for (int k = 0; k < (int)s.sch.size(); ++k)
    if (s.sch[k] >= 0) s.seg_ptr[s.sch[k] + 1]++;
  for (int q = 0; q < s.nseg; ++q) s.seg_ptr[q + 1] += s.seg_ptr[q];
  s.seg_mus.assign(s.seg_ptr[s.nseg], 0);
  {
    std::vector<int> fill(s.seg_ptr.begin(), s.seg_ptr.end() - 1);
    for (int m = 0; m < s.M; ++m) s.seg_mus[fill[s.mseg[m]]++] = m;
    for (int k = 0; k < (int)s.sch.size(); ++k)
      if (s.sch[k] >= 0) s.seg_mus[fill[s.sch[k]]++] = -(k + 1);
  }

  // articulated skeleton (Dfobj.h:254-288, World::AddBody World.h:499-545)
  REQ(d.n_links >= 0 && d.n_links <= kMaxLinks, "descriptor: n_links out of range");
  if (d.n_links > 0) {
    REQ(d.link_parent && d.link_type && d.link_joint && d.link_axis && d.link_offsets && d.link_vertices,
        "descriptor: link arrays missing");
    REQ(d.precision == DFEM_PREC_FP64, "descriptor: skeleton links need the FP64 form");
    REQ(!d.handle_collision, "descriptor: skeleton links with collision handling are not supported (the "
        "reference's contact phase solves the rigid vertices with the free-vertex factor)");
    s.L = d.n_links;
    s.lparent.assign(d.link_parent, d.link_parent + s.L);
    s.ltype.assign(d.link_type, d.link_type + s.L);
    s.lchan.assign(s.L, -1);
    if (d.link_channel) s.lchan.assign(d.link_channel, d.link_channel + s.L);
    s.loff.assign(d.link_offsets, d.link_offsets + s.L + 1);
    s.ljoint.assign(d.link_joint, d.link_joint + 3 * (size_t)s.L);
    s.laxis.assign(3 * (size_t)s.L, 0.0);
    REQ(s.loff[0] == 0, "descriptor: link_offsets must start at 0");
    REQ(s.lparent[0] == -1 && s.ltype[0] == DFEM_JOINT_ALL, "descriptor: link 0 must be the root, of joint type ALL");
    for (int l = 0; l < s.L; ++l) {
      REQ(s.loff[l + 1] > s.loff[l], "descriptor: every link needs at least one vertex");
      REQ(s.lchan[l] >= -1 && s.lchan[l] < s.nseg, "descriptor: link torque channel out of range");
      for (int c = 0; c < 3; ++c) REQ(std::isfinite(s.ljoint[3 * l + c]), "descriptor: non-finite joint position");
      if (l == 0) continue;
      REQ(s.lparent[l] >= 0 && s.lparent[l] < l, "descriptor: a link's parent must precede it");
      REQ(s.ltype[l] == DFEM_JOINT_ROTATIONAL || s.ltype[l] == DFEM_JOINT_PRISMATIC,
          "descriptor: non-root links must be ROTATIONAL or PRISMATIC");
      const double* a = d.link_axis + 3 * l;
      const double n = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
      REQ(std::isfinite(n) && n > 0, "descriptor: zero or non-finite joint axis");
      for (int c = 0; c < 3; ++c) s.laxis[3 * l + c] = a[c] / n;  // jointAxis / jointAxis.norm()
    }
    const int nr = s.loff[s.L];
    REQ(nr <= kMaxRigidVertices, "descriptor: too many link vertices");
    s.lvert.assign(d.link_vertices, d.link_vertices + nr);
    REQ(inrange(s.lvert.data(), nr), "descriptor: link vertex out of range");
    std::vector<char> used(N, 0);
    s.lrest.resize(3 * (size_t)nr);
    for (int k = 0; k < nr; ++k) {
      REQ(!used[s.lvert[k]], "descriptor: a vertex belongs to two links");
      used[s.lvert[k]] = 1;
      for (int c = 0; c < 3; ++c) s.lrest[3 * k + c] = d.x0[3 * (size_t)s.lvert[k] + c];  // Link::restpos
    }
    REQ(nr < N, "descriptor: every vertex is rigid");
  }

  s.B = d.n_bending;
  if (d.bend_offsets) s.boff.assign(d.bend_offsets, d.bend_offsets + s.B + 1);
  else s.boff.assign(1, 0);
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
  {  // each vertex's drag faces, ascending
    const int F = (int)s.df.size() / 3;
    s.vf_ptr.assign(N + 1, 0);
    for (int e = 0; e < 3 * F; ++e) s.vf_ptr[s.df[e] + 1]++;
    for (int i = 0; i < N; ++i) s.vf_ptr[i + 1] += s.vf_ptr[i];
    s.vf_face.assign(3 * (size_t)F, 0);
    std::vector<int> fill(s.vf_ptr.begin(), s.vf_ptr.end() - 1);
    for (int e = 0; e < 3 * F; ++e) s.vf_face[fill[s.df[e]]++] = e;  // face slot e = 3 f + corner
  }
  s.nparts = 1;
  s.part_v0 = {0, s.N};
  s.part_t0 = {0, s.T};
  s.part_seg0 = {0, s.nseg};
  return true;
}

namespace {
template <typename T>
void cat(std::vector<T>& dst, const std::vector<T>& src) { dst.insert(dst.end(), src.begin(), src.end()); }
template <typename T, typename O>
void cat_off(std::vector<T>& dst, const std::vector<T>& src, O off) {
  for (const T& v : src) dst.push_back(static_cast<T>(v + off));
}
// CSR pointer arrays: append src[1..] shifted by off (dst already holds its leading 0)
template <typename T, typename O>
void cat_ptr(std::vector<T>& dst, const std::vector<T>& src, O off) {
  for (size_t k = 1; k < src.size(); ++k) dst.push_back(static_cast<T>(src[k] + off));
}
}  // namespace

bool merge_parts(const std::vector<HostScene>& P, HostScene& u, std::string& err) {
  REQ(!P.empty(), "batch: no scenes");
  const HostScene& a = P[0];
  int64_t totN = 0, totT = 0, totSlots = 0, totRows = 0, totL = 0, totD = 0, totF = 0;
  for (const HostScene& p : P) {
    REQ(p.h == a.h && p.damping == a.damping && p.g[0] == a.g[0] && p.g[1] == a.g[1] && p.g[2] == a.g[2] &&
            p.K == a.K && p.precision == a.precision && p.checkpoint_every == a.checkpoint_every,
        "batch: scenes must share time_step, damping, gravity, max_iterations, precision and checkpoint_every");
    REQ(!p.self_collide, "batch: soft-soft contact is supported for single scenes only");
    REQ(p.L == 0, "batch: skeleton links are supported for single scenes only");
    REQ(p.nparts == 1, "batch: parts must be single scenes");
    totN += p.N; totT += p.T; totSlots += p.nslots; totRows += (int64_t)p.F.rowidx.size();
    totL += (int64_t)p.F.Lcm.size(); totD += (int64_t)p.F.Dinv.size(); totF += (int64_t)p.df.size() / 3;
  }
  REQ(totN < INT32_MAX / 3 && totT < INT32_MAX / 4 && totSlots < INT32_MAX / 3 && totRows < INT32_MAX / 3 &&
          totL < INT32_MAX && totD < INT32_MAX && totF < INT32_MAX / 3,
      "batch: total size exceeds the 32-bit index range of the kernels");
  u = HostScene();
  u.h = a.h; u.damping = a.damping; u.g[0] = a.g[0]; u.g[1] = a.g[1]; u.g[2] = a.g[2];
  u.K = a.K; u.precision = a.precision; u.checkpoint_every = a.checkpoint_every;
  // obstacle contact: every part keeps its own contact vertices and obstacle
  // faces; the phase's parameters are shared
  auto contact_part = [](const HostScene& p) { return p.collide && !p.cverts.empty() && !p.obs_f.empty(); };
  const HostScene* c0 = nullptr;
  for (const HostScene& p : P)
    if (contact_part(p)) {
      if (!c0) c0 = &p;
      REQ(p.alpha == c0->alpha && p.mu_obs == c0->mu_obs, "batch: contact scenes must share alpha and the obstacle friction");
    }
  u.collide = c0 != nullptr;
  if (c0) { u.alpha = c0->alpha; u.mu_obs = c0->mu_obs; u.pobs_f0 = {0}; }
  u.underwater = false;
  u.nparts = (int)P.size();
  u.part_v0 = {0}; u.part_t0 = {0}; u.part_seg0 = {0};
  u.seg_ptr = {0}; u.boff = {0}; u.vslot_ptr = {0};
  u.Hs.ptr = {0};
  u.vf_ptr = {0};
  SupernodalFactor& F = u.F;
  F.sn_rofs = {0}; F.sn_lofs = {0}; F.sn_dofs = {0}; F.rseg_ptr = {0};
  int voff = 0, moff = 0, soff = 0, segoff = 0, slotoff = 0, bvoff = 0, snoff = 0, rsegoff = 0;
  bool any_channel = false;
  for (const HostScene& p : P) any_channel = any_channel || !p.sch.empty();
  int64_t hsoff = 0, rofs = 0, lofs = 0, dofs = 0;
  std::vector<int> sn_base(P.size());
  for (size_t q = 0; q < P.size(); ++q) {
    const HostScene& p = P[q];
    cat(u.x0, p.x0); cat(u.mass, p.mass); cat(u.gmask, p.gmask);
    cat_off(u.tv, p.tv, voff); cat(u.tinv, p.tinv); cat(u.tvol, p.tvol); cat(u.tE, p.tE); cat(u.tnu, p.tnu);
    cat_off(u.tslot, p.tslot, slotoff);
    cat_off(u.mv, p.mv, voff); cat(u.minv, p.minv); cat(u.mvol, p.mvol); cat(u.mk, p.mk); cat(u.mfib, p.mfib);
    cat_off(u.mseg, p.mseg, segoff); cat_off(u.mslot, p.mslot, slotoff);
    cat_ptr(u.seg_ptr, p.seg_ptr, (int)u.seg_mus.size());
    for (int k : p.seg_mus) u.seg_mus.push_back(k >= 0 ? k + moff : k - soff);
    cat_off(u.sv, p.sv, voff); cat_off(u.sslot, p.sslot, slotoff); cat(u.srest, p.srest); cat(u.ssw, p.ssw);
    cat_ptr(u.boff, p.boff, bvoff); cat_off(u.bv, p.bv, voff); cat_off(u.bslot, p.bslot, slotoff);
    cat(u.bbeta, p.bbeta); cat(u.bw, p.bw); cat(u.brest, p.brest);
    cat_off(u.av, p.av, voff); cat(u.ap, p.ap); cat(u.ak, p.ak);
    cat_ptr(u.vslot_ptr, p.vslot_ptr, slotoff);
    cat_ptr(u.Hs.ptr, p.Hs.ptr, hsoff); cat_off(u.Hs.col, p.Hs.col, voff); cat(u.Hs.val, p.Hs.val);
    cat_off(u.to_internal, p.to_internal, voff); cat_off(u.to_user, p.to_user, voff);
    // drag faces (gravity is already off per vertex in underwater parts); face
    // slots 3 f + corner shift by the face slots of the earlier parts
    const int fslot = (int)u.df.size();
    cat_off(u.df, p.df, voff);
    cat_ptr(u.vf_ptr, p.vf_ptr, fslot); cat_off(u.vf_face, p.vf_face, fslot);
    u.underwater = u.underwater || p.underwater;
    // factor (block diagonal)
    const SupernodalFactor& G = p.F;
    cat_off(F.perm, G.perm, voff); cat_off(F.iperm, G.iperm, voff);
    cat_off(F.sn_c0, G.sn_c0, voff); cat(F.sn_w, G.sn_w); cat(F.sn_r, G.sn_r);
    cat_ptr(F.sn_rofs, G.sn_rofs, rofs); cat_off(F.rowidx, G.rowidx, voff);
    cat_ptr(F.sn_lofs, G.sn_lofs, lofs); cat(F.Lcm, G.Lcm);
    cat_ptr(F.sn_dofs, G.sn_dofs, dofs); cat(F.Ldiag, G.Ldiag); cat(F.Dinv, G.Dinv);
    for (int par : G.sn_parent) F.sn_parent.push_back(par < 0 ? -1 : par + snoff);
    cat_off(F.col_sn, G.col_sn, snoff);
    cat_ptr(F.rseg_ptr, G.rseg_ptr, rsegoff); cat_off(F.rseg_pos, G.rseg_pos, (int)rofs);
    F.nnz_factor += G.nnz_factor;
    F.reg = std::max(F.reg, G.reg);
    F.nlevels = std::max(F.nlevels, G.nlevels);
    sn_base[q] = snoff;
    if (any_channel) {
      if (p.sch.empty()) u.sch.insert(u.sch.end(), p.S, -1);
      else for (int c : p.sch) u.sch.push_back(c < 0 ? -1 : c + segoff);
    }
    if (c0) {
      if (contact_part(p)) {
        const int ov = (int)u.obs_x.size() / 3;
        for (int v : p.cverts) { u.cverts.push_back(v + voff); u.cpart.push_back((int)q); }
        cat(u.obs_x, p.obs_x);
        cat_off(u.obs_f, p.obs_f, ov);
      }
      u.pobs_f0.push_back((int)u.obs_f.size() / 3);
    }
    voff += p.N; moff += p.M; soff += p.S; segoff += p.nseg; slotoff += p.nslots; bvoff += (int)p.bv.size();
    snoff += G.nsuper; rsegoff += (int)G.rseg_pos.size();
    hsoff += p.Hs.ptr[p.N]; rofs += (int64_t)G.rowidx.size(); lofs += (int64_t)G.Lcm.size(); dofs += (int64_t)G.Dinv.size();
    u.T += p.T; u.M += p.M; u.S += p.S; u.B += p.B; u.A += p.A;
    u.part_v0.push_back(voff); u.part_t0.push_back(u.T); u.part_seg0.push_back(segoff);
  }
  u.N = voff; u.nseg = segoff; u.nslots = slotoff;
  u.Hs.n = voff;
  F.n = voff; F.nsuper = snoff;
  F.lvl_ptr = {0};
  for (int l = 0; l < F.nlevels; ++l) {
    for (size_t q = 0; q < P.size(); ++q) {
      const SupernodalFactor& G = P[q].F;
      if (l >= G.nlevels) continue;
      for (int k = G.lvl_ptr[l]; k < G.lvl_ptr[l + 1]; ++k) F.lvl_sn.push_back(G.lvl_sn[k] + sn_base[q]);
    }
    F.lvl_ptr.push_back((int)F.lvl_sn.size());
  }
  return true;
}

void merge_numeric(const std::vector<HostScene>& P, HostScene& u) {
  size_t t = 0, h = 0, l = 0, d = 0;
  u.F.reg = 0.0;
  for (const HostScene& p : P) {
    std::copy(p.tE.begin(), p.tE.end(), u.tE.begin() + t);
    std::copy(p.tnu.begin(), p.tnu.end(), u.tnu.begin() + t);
    std::copy(p.Hs.val.begin(), p.Hs.val.end(), u.Hs.val.begin() + h);
    std::copy(p.F.Lcm.begin(), p.F.Lcm.end(), u.F.Lcm.begin() + l);
    std::copy(p.F.Ldiag.begin(), p.F.Ldiag.end(), u.F.Ldiag.begin() + d);
    std::copy(p.F.Dinv.begin(), p.F.Dinv.end(), u.F.Dinv.begin() + d);
    u.F.reg = std::max(u.F.reg, p.F.reg);
    t += p.tE.size(); h += p.Hs.val.size(); l += p.F.Lcm.size(); d += p.F.Dinv.size();
  }
}

void hs_split(const HostScene& s, std::vector<double>& base, std::vector<int>& cptr, std::vector<int>& ctet,
              std::vector<double>& ccoef) {
  const std::vector<double> zeroE(s.T, 0.0);
  base = assemble_hs(s, zeroE.data()).val;
  const int64_t nnz = (int64_t)s.Hs.col.size();
  auto entry = [&](int i, int j) -> int64_t {
    const int* c0 = s.Hs.col.data() + s.Hs.ptr[i];
    const int* c1 = s.Hs.col.data() + s.Hs.ptr[i + 1];
    return s.Hs.ptr[i] + (std::lower_bound(c0, c1, j) - c0);
  };
  // counting pass, then a fill pass in tet order (each entry's list is in tet order)
  std::vector<int64_t> cnt(nnz + 1, 0);
  for (int e = 0; e < s.T; ++e)
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) cnt[entry(s.tv[4 * e + a], s.tv[4 * e + b]) + 1]++;
  for (int64_t k = 0; k < nnz; ++k) cnt[k + 1] += cnt[k];
  cptr.assign(cnt.begin(), cnt.end());
  ctet.resize(cnt[nnz]);
  ccoef.resize(cnt[nnz]);
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (int e = 0; e < s.T; ++e) {
    double G[4][3];
    gcoef(&s.tinv[9 * e], G);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        const int64_t q = fill[entry(s.tv[4 * e + a], s.tv[4 * e + b])]++;
        ctet[q] = e;
        ccoef[q] = s.tvol[e] * (G[a][0] * G[b][0] + G[a][1] * G[b][1] + G[a][2] * G[b][2]);
      }
  }
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
