/*
 * pd_oracle.cpp — CPU FP64 restatement of diff_fem's projective-dynamics step
 * and a hand-written adjoint of it.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA engine is
 * compared against; the product (diff_fem_b200) never links, imports or calls
 * it.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference leg may load the oracle library.
 *
 * PARITY UNPINNED against the reference binary: diff_fem cannot be built or
 * imported here (Eigen, CppAD, CGAL and Boost are absent and there is no
 * network), and the reference ships no tests, golden vectors or fixtures with
 * outputs.  This restatement is pinned instead by known-answer invariants,
 * central finite differences of its adjoint, and the reference's own data
 * scenes (tests/test_oracle.py).
 *
 * What it restates (paths relative to the diff_fem repository):
 *   - World::TimeStepping / UpdatePositionsAndVelocities   sim/fem/World.h:673-720,757-766
 *   - World::ProjectiveDynamicsMethod main loop           sim/fem/World.h:835-917
 *   - World::ComputeSolution (both branches)              sim/fem/World.h:1601-1670
 *   - Link: kinematics, tildaV, UpdateT, guessNext        sim/constants.h:28-247
 *   - Schur complement of the free vertices (bones)       sim/fem/World.h:1100-1135
 *   - World::PreComputation / FactorizeLDLT (retry)       sim/fem/World.h:1089-1139,1212-1232
 *   - CorotateFEMConstraint (F, SVD, reflection, volume)   sim/fem/Constraint/CorotateFEMConstraint.h:64-392
 *   - LinearMuscleConstraint                              sim/fem/Constraint/LinearMuscleConstraint.h:91-270
 *   - AttachmentConstraint                                sim/fem/Constraint/AttachmentConstraint.h:70-99
 *   - SpringConstraint                                    sim/fem/Constraint/SpringConstraint.h:51-144
 *   - BendingConstraint                                   sim/fem/Constraint/BendingConstraint.h:66-187,220-300
 *   - Environment::Step gravity / underwater branch        sim/Environment.h:228-259
 *   - Dfobj::ComputeDragForces, Cd, Cl                    sim/Dfobj.h:803-838,904-998
 *   - Dfobj::Initialize tet re-orientation and masses     sim/Dfobj.h:442-525
 *
 * Choices that differ in mechanism but not in result:
 *   - The 3N x 3N H of the reference is kron(Hs, I3); the oracle factors the
 *     scalar N x N Hs (envelope Cholesky after reverse Cuthill–McKee) and
 *     solves 3 right-hand sides.  orc_full_L_triplets() rebuilds the
 *     reference's 3N x 3N triplets so a test can check the kron identity.
 *   - 3x3 SVD: one-sided Jacobi on F (Hestenes), singular values >= 0 like
 *     Eigen::JacobiSVD.  R = U V^T and U diag(g(S)) V^T do not depend on the
 *     SVD's sign/permutation choices, so any exact SVD gives the same d.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <queue>
#include <string>
#include <vector>
#include <map>
#include <array>
#include <limits>
#include <thread>

#include "../include/dfem.h"

namespace orc {

struct V3 { double x, y, z; };
static inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

/* column-major 3x3: m[c][r] is row r of column c */
struct M3 { double m[3][3]; };
static inline double& at(M3& a, int r, int c) { return a.m[c][r]; }
static inline double at(const M3& a, int r, int c) { return a.m[c][r]; }
static M3 mul(const M3& a, const M3& b) {
  M3 o{};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += at(a, r, k) * at(b, k, c);
      at(o, r, c) = s;
    }
  return o;
}
static M3 mulT(const M3& a, const M3& b) { /* a * b^T */
  M3 o{};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += at(a, r, k) * at(b, c, k);
      at(o, r, c) = s;
    }
  return o;
}
static M3 Tmul(const M3& a, const M3& b) { /* a^T * b */
  M3 o{};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += at(a, k, r) * at(b, k, c);
      at(o, r, c) = s;
    }
  return o;
}
static double det(const M3& a) {
  return at(a, 0, 0) * (at(a, 1, 1) * at(a, 2, 2) - at(a, 1, 2) * at(a, 2, 1)) -
         at(a, 0, 1) * (at(a, 1, 0) * at(a, 2, 2) - at(a, 1, 2) * at(a, 2, 0)) +
         at(a, 0, 2) * (at(a, 1, 0) * at(a, 2, 1) - at(a, 1, 1) * at(a, 2, 0));
}
static M3 inverse(const M3& a) {
  double d = det(a);
  M3 o{};
  at(o, 0, 0) = (at(a, 1, 1) * at(a, 2, 2) - at(a, 1, 2) * at(a, 2, 1)) / d;
  at(o, 0, 1) = (at(a, 0, 2) * at(a, 2, 1) - at(a, 0, 1) * at(a, 2, 2)) / d;
  at(o, 0, 2) = (at(a, 0, 1) * at(a, 1, 2) - at(a, 0, 2) * at(a, 1, 1)) / d;
  at(o, 1, 0) = (at(a, 1, 2) * at(a, 2, 0) - at(a, 1, 0) * at(a, 2, 2)) / d;
  at(o, 1, 1) = (at(a, 0, 0) * at(a, 2, 2) - at(a, 0, 2) * at(a, 2, 0)) / d;
  at(o, 1, 2) = (at(a, 0, 2) * at(a, 1, 0) - at(a, 0, 0) * at(a, 1, 2)) / d;
  at(o, 2, 0) = (at(a, 1, 0) * at(a, 2, 1) - at(a, 1, 1) * at(a, 2, 0)) / d;
  at(o, 2, 1) = (at(a, 0, 1) * at(a, 2, 0) - at(a, 0, 0) * at(a, 2, 1)) / d;
  at(o, 2, 2) = (at(a, 0, 0) * at(a, 1, 1) - at(a, 0, 1) * at(a, 1, 0)) / d;
  return o;
}
static inline V3 col(const M3& a, int c) { return {a.m[c][0], a.m[c][1], a.m[c][2]}; }
static inline void setcol(M3& a, int c, V3 v) { a.m[c][0] = v.x; a.m[c][1] = v.y; a.m[c][2] = v.z; }

/* ---- 3x3 SVD: one-sided (Hestenes) Jacobi on the columns of F ------------ */
struct SVD3 { M3 U, V; double s[3]; };

static SVD3 svd3(const M3& F) {
  M3 B = F;
  M3 V{};
  at(V, 0, 0) = at(V, 1, 1) = at(V, 2, 2) = 1.0;
  const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 30; ++sweep) {
    bool rotated = false;
    for (auto& pq : pairs) {
      int p = pq[0], q = pq[1];
      V3 bp = col(B, p), bq = col(B, q);
      double a = dot(bp, bp), b = dot(bq, bq), g = dot(bp, bq);
      if (std::fabs(g) <= 1e-15 * std::sqrt(a * b) || g == 0.0) continue;
      rotated = true;
      double zeta = (b - a) / (2.0 * g);
      double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
      double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
      setcol(B, p, c * bp - s * bq);
      setcol(B, q, s * bp + c * bq);
      V3 vp = col(V, p), vq = col(V, q);
      setcol(V, p, c * vp - s * vq);
      setcol(V, q, s * vp + c * vq);
    }
    if (!rotated) break;
  }
  SVD3 out;
  double sig[3];
  for (int i = 0; i < 3; ++i) sig[i] = norm(col(B, i));
  int order[3] = {0, 1, 2};
  std::sort(order, order + 3, [&](int i, int j) { return sig[i] > sig[j]; });
  M3 Bs{}, Vs{};
  for (int k = 0; k < 3; ++k) {
    setcol(Bs, k, col(B, order[k]));
    setcol(Vs, k, col(V, order[k]));
    out.s[k] = sig[order[k]];
  }
  out.V = Vs;
  const double tiny = 1e-300;
  /* U columns: normalised B columns; a (near) zero singular value takes the
     direction that completes an orthonormal basis. */
  for (int k = 0; k < 3; ++k) {
    if (out.s[k] > tiny && out.s[k] > 1e-14 * out.s[0]) {
      setcol(out.U, k, (1.0 / out.s[k]) * col(Bs, k));
    } else if (k == 2) {
      setcol(out.U, 2, cross(col(out.U, 0), col(out.U, 1)));
    } else {
      V3 u0 = col(out.U, 0);
      V3 e = std::fabs(u0.x) < 0.9 ? V3{1, 0, 0} : V3{0, 1, 0};
      V3 u1 = cross(u0, e);
      setcol(out.U, 1, (1.0 / norm(u1)) * u1);
      setcol(out.U, 2, cross(u0, col(out.U, 1)));
      break;
    }
  }
  return out;
}

/* ---- the 5-step Newton projection of S onto prod = 1 ---------------------
 * CorotateFEMConstraint.h:362-374.  Also returns, for the adjoint, the
 * Jacobian dg/ds (forward mode) and the exact divided differences
 * (g_i - g_j)/(s_i - s_j) via the recurrence r <- 1 - c * p_k * r. */
struct VolProj { double g[3]; double J[3][3]; double dd[3]; /* pairs 01,02,12 */ };

static VolProj volume_projection(const double s[3], bool want_derivs) {
  double D[3] = {0, 0, 0};
  double dD[3][3] = {{0}};      /* dD[i][dir] */
  double r[3] = {1, 1, 1};      /* divided-difference ratios for pairs 01,02,12 */
  const int pk[3] = {2, 1, 0};  /* third index of each pair */
  for (int it = 0; it < 5; ++it) {
    double p[3] = {s[0] + D[0], s[1] + D[1], s[2] + D[2]};
    double CD = p[0] * p[1] * p[2] - 1.0;
    double gr[3] = {p[1] * p[2], p[0] * p[2], p[0] * p[1]};
    double gg = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
    double num = gr[0] * D[0] + gr[1] * D[1] + gr[2] * D[2] - CD;
    double c = num / gg;
    if (want_derivs) {
      for (int q = 0; q < 3; ++q) r[q] = 1.0 - c * p[pk[q]] * r[q];
      double ndD[3][3];
      for (int dir = 0; dir < 3; ++dir) {
        double dp[3];
        for (int i = 0; i < 3; ++i) dp[i] = (i == dir ? 1.0 : 0.0) + dD[i][dir];
        double dC = gr[0] * dp[0] + gr[1] * dp[1] + gr[2] * dp[2];
        double dgr[3] = {dp[1] * p[2] + p[1] * dp[2], dp[0] * p[2] + p[0] * dp[2], dp[0] * p[1] + p[0] * dp[1]};
        double dnum = dgr[0] * D[0] + dgr[1] * D[1] + dgr[2] * D[2] +
                      gr[0] * dD[0][dir] + gr[1] * dD[1][dir] + gr[2] * dD[2][dir] - dC;
        double dgg = 2.0 * (gr[0] * dgr[0] + gr[1] * dgr[1] + gr[2] * dgr[2]);
        double dc = (dnum * gg - num * dgg) / (gg * gg);
        for (int i = 0; i < 3; ++i) ndD[i][dir] = dc * gr[i] + c * dgr[i];
      }
      std::memcpy(dD, ndD, sizeof(dD));
    }
    for (int i = 0; i < 3; ++i) D[i] = c * gr[i];
  }
  VolProj o;
  for (int i = 0; i < 3; ++i) {
    o.g[i] = s[i] + D[i];
    for (int j = 0; j < 3; ++j) o.J[i][j] = (i == j ? 1.0 : 0.0) + dD[i][j];
  }
  for (int q = 0; q < 3; ++q) o.dd[q] = r[q];
  return o;
}

/* ---- scene ----------------------------------------------------------------- */
struct Tet { int v[4]; M3 invDm; double vol; double G[4][3]; };

static Tet make_tet(const double* x0, const int* idx) {
  /* Dfobj.h:474-503: swap vertices 1 and 2 when det(Dm) < 0; vol = det/6. */
  Tet t;
  int i0 = idx[0], i1 = idx[1], i2 = idx[2], i3 = idx[3];
  auto P = [&](int i) { return V3{x0[3 * i], x0[3 * i + 1], x0[3 * i + 2]}; };
  M3 Dm{};
  setcol(Dm, 0, P(i1) - P(i0));
  setcol(Dm, 1, P(i2) - P(i0));
  setcol(Dm, 2, P(i3) - P(i0));
  if (det(Dm) < 0) {
    std::swap(i1, i2);
    setcol(Dm, 0, P(i1) - P(i0));
    setcol(Dm, 1, P(i2) - P(i0));
  }
  t.v[0] = i0; t.v[1] = i1; t.v[2] = i2; t.v[3] = i3;
  t.vol = det(Dm) / 6.0;
  t.invDm = inverse(Dm);
  /* Rows of the selection matrix A (CorotateFEMConstraint.h:236-245):
     F(:,j) = sum_v G[v][j] x_v with G[0][j] = -sum_k invDm(k,j), G[k+1][j] = invDm(k,j). */
  for (int j = 0; j < 3; ++j) {
    double s = 0;
    for (int k = 0; k < 3; ++k) { t.G[k + 1][j] = at(t.invDm, k, j); s += at(t.invDm, k, j); }
    t.G[0][j] = -s;
  }
  return t;
}

struct Bend { std::vector<int> v; std::vector<double> beta; double rest_norm; double w; };

static double bend_cos(V3 a, V3 b, V3 c) { V3 e1 = a - b, e2 = c - b; return dot(e1, e2) / (norm(e1) * norm(e2)); }
static double bend_sin(V3 a, V3 b, V3 c) { V3 e1 = a - b, e2 = c - b; return norm(cross(e1, e2)) / (norm(e1) * norm(e2)); }
static double mean_value(V3 a, V3 b, V3 c) {
  double num = 1.0 - bend_cos(a, b, c);
  if (num == 0) return 0;
  return num / bend_sin(a, b, c);
}

/* SelfCollisionInfo: a face, its normal (the first member's impact normal) and
 * the contact vertices whose closest impact is on it, ascending. */
struct SelfGroup { int f; V3 n; std::vector<int> verts; };

/* ---- articulated skeleton: Link (sim/constants.h:28-247) ------------------ */
struct Xf { M3 R; V3 d; };  /* Transformation: x -> R x + d */
static Xf xf_identity() {
  Xf t{};
  at(t.R, 0, 0) = at(t.R, 1, 1) = at(t.R, 2, 2) = 1.0;
  t.d = V3{0, 0, 0};
  return t;
}
static inline V3 mv(const M3& a, V3 v) {
  return V3{at(a, 0, 0) * v.x + at(a, 0, 1) * v.y + at(a, 0, 2) * v.z,
            at(a, 1, 0) * v.x + at(a, 1, 1) * v.y + at(a, 1, 2) * v.z,
            at(a, 2, 0) * v.x + at(a, 2, 1) * v.y + at(a, 2, 2) * v.z};
}
static inline Xf xf_mul(const Xf& a, const Xf& b) { return Xf{mul(a.R, b.R), mv(a.R, b.d) + a.d}; }
static inline V3 xf_apply(const Xf& a, V3 v) { return mv(a.R, v) + a.d; }

struct LinkO {
  int parent = -1, type = DFEM_JOINT_ALL, dof = 0, sdof = 0, chan = -1;
  V3 joint{0, 0, 0}, axis{0, 0, 0}, d0{0, 0, 0};
  M3 nx{}, nnt{};                 /* cross-product matrix of the axis, axis axis^T */
  int r0 = 0, r1 = 0;             /* its rigid vertices [r0, r1) */
  double mag = 0, prevmag = 0;
  Xf T = xf_identity(), Tr = xf_identity(), prevTr = xf_identity(), prefix = xf_identity(),
     dT = xf_identity(), suffix = xf_identity();
};

struct Skel {
  int L = 0, ndof = 0, nq = 0;    /* links, dofs (6 + L - 1), joint-state length (12 + L - 1) */
  std::vector<LinkO> links;
  std::vector<int> rv;            /* rigid vertex j -> vertex id, in link order */
  std::vector<V3> rest;           /* Link::restpos */
  std::vector<int> ridx;          /* vertex -> rigid index or -1 */
  std::vector<double> jq, jqd;    /* World::mJointQ / mJointQd */
  std::vector<double> Srr;        /* nr x nr: Hs_RR - Hs_RF Hs_FF^-1 Hs_FR (scalar) */
};

struct Scene {
  int N = 0;
  std::vector<double> x0, mass, gmask;
  std::vector<Tet> tets; std::vector<double> E, nu;
  std::vector<int> att_v; std::vector<V3> att_p; std::vector<double> att_k;
  std::vector<Tet> mtets; std::vector<V3> mfib; std::vector<double> mk; std::vector<int> mseg; int nseg = 0;
  std::vector<double> seg_act;
  std::vector<int> sp_v, sp_ch; std::vector<double> sp_rest, sp_w;  /* sp_ch: -1 or a pneumatic spring's channel */
  std::vector<Bend> bends;
  double h = 0.01, damping = 1.0; int K = 10; V3 g{0, 0, 0};
  /* contact: World::ProjectiveDynamicsMethod contact phase (World.h:925-1023),
     obstacle branch of CollisionHandling (World.h:1317-1430), vertex-face CCD */
  bool collide = false;
  double alpha = 1.0, mu_obs = 1.0;
  int max_passes = 64;
  std::vector<int> cverts;
  std::vector<V3> obs_x;
  std::vector<std::array<int, 3>> obs_f;
  int last_passes = 0;
  /* soft-soft (self) contact: the self branch of CollisionHandling
     (World.h:1446-1537), CollisionBrutal::getSelfCollisionsInfo
     (collisionBrutal.h:645-700), arcsim soft impacts (collision.cpp:29-120) */
  bool self_collide = false;
  double mu_self = 1.0;                     /* World Friction */
  std::vector<std::array<int, 3>> cfaces;   /* soft contact faces, contact-vertex ids */
  std::vector<char> on_face;                /* contact vertex lies on a soft face */
  std::vector<double> sc_cur;               /* self forces of the last swapping call, 3 per contact vertex */
  /* detection replay for derivative tests: 1 records each step's passes
     (impact normals per contact vertex, self groups), 2 replays them instead
     of detecting, so that perturbed runs keep the detection's outputs, which
     the adjoint treats as constants */
  struct PassRecord { std::vector<std::vector<V3>> normals; std::vector<SelfGroup> groups; };
  int freeze = 0, cur_step = 0;
  std::vector<std::vector<PassRecord>> frz;
  /* underwater drag and lift (Dfobj::ComputeDragForces) */
  bool underwater = false;
  std::vector<std::array<int, 3>> drag_f;
  /* envelope Cholesky of Hs in RCM order */
  std::vector<int> perm, iperm;  /* perm[new] = old */
  std::vector<int> first;        /* first column of row i in the envelope */
  std::vector<int64_t> rowptr;   /* start of row i in env */
  std::vector<double> env;
  std::vector<std::vector<std::pair<int, double>>> Hrows; /* Hs rows (old numbering) */
  double reg = 0.0;
  /* skeleton: the links and a second envelope factor of Hs with the rigid
     vertices' rows and columns replaced by the identity, i.e. of Qf (World.h:1100-1128) */
  Skel skel;
  Scene* qf = nullptr;
  ~Scene() { delete qf; }
  std::string err;
  /* recorded forward trajectory for the adjoint */
  int rec_steps = 0;
  std::vector<double> rec_x, rec_v;        /* step-start states */
  std::vector<double> rec_act;             /* per step activations */
  std::vector<int> rec_iters;
  std::vector<int> rec_passes;             /* contact passes per step */
};

static void add_H(std::vector<std::vector<std::pair<int, double>>>& rows, int i, int j, double v) {
  rows[i].push_back({j, v});
}

/* Hs = M/h^2 + L_s, with L = kron(L_s, I3) (World.h:1093-1098). */
static void assemble_H(Scene& S) {
  int N = S.N;
  std::vector<std::vector<std::pair<int, double>>> rows(N);
  double ih2 = 1.0 / (S.h * S.h);
  for (int i = 0; i < N; ++i) add_H(rows, i, i, S.mass[i] * ih2);
  for (size_t t = 0; t < S.tets.size(); ++t) {
    const Tet& T = S.tets[t];
    /* mu * vol * (1 + nu) * G G^T  (CorotateFEMConstraint.h:289-350: two blocks, the second scaled by nu) */
    double mu = S.E[t] / (1.0 + S.nu[t]);
    double w = mu * T.vol * (1.0 + S.nu[t]);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        double s = 0;
        for (int j = 0; j < 3; ++j) s += T.G[a][j] * T.G[b][j];
        add_H(rows, T.v[a], T.v[b], w * s);
      }
  }
  for (size_t a = 0; a < S.att_v.size(); ++a) add_H(rows, S.att_v[a], S.att_v[a], S.att_k[a]);
  for (size_t m = 0; m < S.mtets.size(); ++m) {
    const Tet& T = S.mtets[m];
    /* LinearMuscleConstraint.h:213-247: vol * k * A^T A with A = kron(c, I3), c = G f */
    double c[4];
    for (int v = 0; v < 4; ++v) c[v] = T.G[v][0] * S.mfib[m].x + T.G[v][1] * S.mfib[m].y + T.G[v][2] * S.mfib[m].z;
    double w = T.vol * S.mk[m];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) add_H(rows, T.v[a], T.v[b], w * c[a] * c[b]);
  }
  for (size_t s = 0; s < S.sp_w.size(); ++s) {
    /* SpringConstraint.h:109: sqrt(w) * A^T A, A = [I, -I] */
    double w = std::sqrt(S.sp_w[s]);
    int i0 = S.sp_v[2 * s], i1 = S.sp_v[2 * s + 1];
    add_H(rows, i0, i0, w); add_H(rows, i1, i1, w);
    add_H(rows, i0, i1, -w); add_H(rows, i1, i0, -w);
  }
  for (const Bend& B : S.bends) {
    /* BendingConstraint.h:139-160: mBend * A^T A with A = mBend * beta: w^3 beta beta^T */
    double w3 = B.w * B.w * B.w;
    for (size_t a = 0; a < B.v.size(); ++a)
      for (size_t b = 0; b < B.v.size(); ++b) add_H(rows, B.v[a], B.v[b], w3 * B.beta[a] * B.beta[b]);
  }
  /* merge duplicates */
  for (auto& r : rows) {
    std::sort(r.begin(), r.end(), [](auto& a, auto& b) { return a.first < b.first; });
    std::vector<std::pair<int, double>> m;
    for (auto& e : r) {
      if (!m.empty() && m.back().first == e.first) m.back().second += e.second;
      else m.push_back(e);
    }
    r.swap(m);
  }
  S.Hrows.swap(rows);
}

static void rcm_order(Scene& S) {
  int N = S.N;
  std::vector<int> deg(N);
  for (int i = 0; i < N; ++i) deg[i] = (int)S.Hrows[i].size();
  std::vector<char> seen(N, 0);
  std::vector<int> order;
  order.reserve(N);
  for (int start0 = 0; start0 < N; ++start0) {
    if (seen[start0]) continue;
    /* pseudo-peripheral start: a few BFS sweeps from the min-degree vertex of this component */
    int start = start0;
    for (int sweep = 0; sweep < 3; ++sweep) {
      std::vector<int> lvl(N, -1);
      std::queue<int> q; q.push(start); lvl[start] = 0; int last = start;
      while (!q.empty()) {
        int u = q.front(); q.pop(); last = u;
        for (auto& e : S.Hrows[u]) if (lvl[e.first] < 0 && !seen[e.first]) { lvl[e.first] = lvl[u] + 1; q.push(e.first); }
      }
      start = last;
    }
    std::queue<int> q; q.push(start); seen[start] = 1;
    while (!q.empty()) {
      int u = q.front(); q.pop(); order.push_back(u);
      std::vector<int> nb;
      for (auto& e : S.Hrows[u]) if (!seen[e.first]) { seen[e.first] = 1; nb.push_back(e.first); }
      std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b] || (deg[a] == deg[b] && a < b); });
      for (int v : nb) q.push(v);
    }
  }
  std::reverse(order.begin(), order.end());
  S.perm = order;
  S.iperm.assign(N, 0);
  for (int i = 0; i < N; ++i) S.iperm[order[i]] = i;
}

/* Envelope Cholesky with the regularise-and-retry loop of World::FactorizeLDLT
 * (World.h:1219-1229; reg starts at 1e-5, x10, bounded here). */
static bool factor(Scene& S) {
  int N = S.N;
  S.first.assign(N, 0);
  for (int i = 0; i < N; ++i) {
    int f = i;
    for (auto& e : S.Hrows[S.perm[i]]) f = std::min(f, S.iperm[e.first]);
    S.first[i] = f;
  }
  S.rowptr.assign(N + 1, 0);
  for (int i = 0; i < N; ++i) S.rowptr[i + 1] = S.rowptr[i] + (i - S.first[i] + 1);
  double reg = 0.0;
  for (int attempt = 0; attempt < 25; ++attempt) {
    S.env.assign(S.rowptr[N], 0.0);
    for (int i = 0; i < N; ++i)
      for (auto& e : S.Hrows[S.perm[i]]) {
        int j = S.iperm[e.first];
        if (j <= i) S.env[S.rowptr[i] + (j - S.first[i])] += e.second;
      }
    for (int i = 0; i < N; ++i) S.env[S.rowptr[i] + (i - S.first[i])] += reg;
    bool ok = true;
    for (int i = 0; i < N && ok; ++i) {
      double* Li = &S.env[S.rowptr[i]];
      int fi = S.first[i];
      for (int j = fi; j < i; ++j) {
        const double* Lj = &S.env[S.rowptr[j]];
        int fj = S.first[j];
        int k0 = std::max(fi, fj);
        double s = Li[j - fi];
        for (int k = k0; k < j; ++k) s -= Li[k - fi] * Lj[k - fj];
        Li[j - fi] = s / Lj[j - fj];
      }
      double d = Li[i - fi];
      for (int k = fi; k < i; ++k) d -= Li[k - fi] * Li[k - fi];
      if (!(d > 0) || !std::isfinite(d)) { ok = false; break; }
      Li[i - fi] = std::sqrt(d);
    }
    if (ok) { S.reg = reg; return true; }
    reg = (reg == 0.0) ? 1e-5 : reg * 10.0;
  }
  S.err = "factorisation failed after regularisation retries";
  return false;
}

/* solve Hs X = B for 3 right-hand sides; B and X interleaved (3N) */
static void solve(const Scene& S, const double* b, double* x) {
  int N = S.N;
  std::vector<double> y(3 * N);
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) y[3 * i + c] = b[3 * S.perm[i] + c];
  for (int i = 0; i < N; ++i) {
    const double* Li = &S.env[S.rowptr[i]];
    int fi = S.first[i];
    double s0 = y[3 * i], s1 = y[3 * i + 1], s2 = y[3 * i + 2];
    for (int k = fi; k < i; ++k) {
      double l = Li[k - fi];
      s0 -= l * y[3 * k]; s1 -= l * y[3 * k + 1]; s2 -= l * y[3 * k + 2];
    }
    double d = Li[i - fi];
    y[3 * i] = s0 / d; y[3 * i + 1] = s1 / d; y[3 * i + 2] = s2 / d;
  }
  for (int i = N - 1; i >= 0; --i) {
    const double* Li = &S.env[S.rowptr[i]];
    int fi = S.first[i];
    double d = Li[i - fi];
    double v0 = y[3 * i] / d, v1 = y[3 * i + 1] / d, v2 = y[3 * i + 2] / d;
    y[3 * i] = v0; y[3 * i + 1] = v1; y[3 * i + 2] = v2;
    for (int k = fi; k < i; ++k) {
      double l = Li[k - fi];
      y[3 * k] -= l * v0; y[3 * k + 1] -= l * v1; y[3 * k + 2] -= l * v2;
    }
  }
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) x[3 * S.perm[i] + c] = y[3 * i + c];
}

static void H_mul(const Scene& S, const double* x, double* y) {
  for (int i = 0; i < S.N; ++i) {
    double a = 0, b = 0, c = 0;
    for (auto& e : S.Hrows[i]) { a += e.second * x[3 * e.first]; b += e.second * x[3 * e.first + 1]; c += e.second * x[3 * e.first + 2]; }
    y[3 * i] = a; y[3 * i + 1] = b; y[3 * i + 2] = c;
  }
}

static inline V3 getx(const double* x, int i) { return {x[3 * i], x[3 * i + 1], x[3 * i + 2]}; }
static inline void addx(double* f, int i, V3 v) { f[3 * i] += v.x; f[3 * i + 1] += v.y; f[3 * i + 2] += v.z; }

static M3 deformation(const Tet& T, const double* x) {
  /* F = Ds * invDm (CorotateFEMConstraint.h:87-101), written as F(:,j) = sum_v G[v][j] x_v */
  M3 F{};
  for (int j = 0; j < 3; ++j) {
    V3 s{0, 0, 0};
    for (int v = 0; v < 4; ++v) s = s + T.G[v][j] * getx(x, T.v[v]);
    setcol(F, j, s);
  }
  return F;
}

/* corotated projection (CorotateFEMConstraint.h:354-377): md and md_volume */
static void corot_project(const M3& F, M3& md, M3& mdv) {
  SVD3 s = svd3(F);
  M3 R = mulT(s.U, s.V);
  md = R;
  if (det(F) < 0) setcol(md, 2, -1.0 * col(R, 2));
  VolProj vp = volume_projection(s.s, false);
  M3 Ug = s.U;
  for (int k = 0; k < 3; ++k) setcol(Ug, k, vp.g[k] * col(s.U, k));
  mdv = mulT(Ug, s.V);
}

/* J*d accumulated per vertex: f += J d(x).  Constraint order and weights follow
 * EvaluateJMatrix of each constraint type. */
static void local_Jd(const Scene& S, const double* x, const double* act, double* f, int nthreads) {
  int NT = (int)S.tets.size();
  std::vector<double> tf((size_t)NT * 12);
  auto tet_range = [&](int t0, int t1) {
  for (int t = t0; t < t1; ++t) {
    const Tet& T = S.tets[t];
    M3 F = deformation(T, x), md, mdv;
    corot_project(F, md, mdv);
    double mu = S.E[t] / (1.0 + S.nu[t]);
    double wr = mu * T.vol, wv = wr * S.nu[t];
    for (int v = 0; v < 4; ++v) {
      V3 s{0, 0, 0};
      for (int j = 0; j < 3; ++j) s = s + T.G[v][j] * (wr * col(md, j) + wv * col(mdv, j));
      tf[12 * t + 3 * v] = s.x; tf[12 * t + 3 * v + 1] = s.y; tf[12 * t + 3 * v + 2] = s.z;
    }
  }
  };
  /* element loop over nthreads host threads (the reference's loop is serial,
     World.h:1200 has its OpenMP pragma commented out) */
  if (nthreads <= 1 || NT < 256) {
    tet_range(0, NT);
  } else {
    std::vector<std::thread> pool;
    int chunk = (NT + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
      int t0 = k * chunk, t1 = std::min(NT, t0 + chunk);
      if (t0 < t1) pool.emplace_back(tet_range, t0, t1);
    }
    for (auto& th : pool) th.join();
  }
  for (int t = 0; t < NT; ++t)
    for (int v = 0; v < 4; ++v) addx(f, S.tets[t].v[v], V3{tf[12 * t + 3 * v], tf[12 * t + 3 * v + 1], tf[12 * t + 3 * v + 2]});
  for (size_t a = 0; a < S.att_v.size(); ++a) addx(f, S.att_v[a], S.att_k[a] * S.att_p[a]);
  for (size_t m = 0; m < S.mtets.size(); ++m) {
    const Tet& T = S.mtets[m];
    M3 F = deformation(T, x);
    V3 fib = S.mfib[m];
    V3 Ff = fib.x * col(F, 0) + fib.y * col(F, 1) + fib.z * col(F, 2);
    V3 p0 = (1.0 - act[S.mseg[m]]) * Ff;  /* Computep0, LinearMuscleConstraint.h:269 */
    double w = T.vol * S.mk[m];
    for (int v = 0; v < 4; ++v) {
      double c = T.G[v][0] * fib.x + T.G[v][1] * fib.y + T.G[v][2] * fib.z;
      addx(f, T.v[v], (w * c) * p0);
    }
  }
  for (size_t s = 0; s < S.sp_w.size(); ++s) {
    int i0 = S.sp_v[2 * s], i1 = S.sp_v[2 * s + 1];
    V3 e = getx(x, i0) - getx(x, i1);
    /* SpringConstraint.h:135-144; a pneumatic spring projects to rest * activation
       (PneumaticConstraint::EvaluateDVector, pneumaticEasy.h:133-147) */
    double len = S.sp_ch[s] >= 0 ? S.sp_rest[s] * act[S.sp_ch[s]] : S.sp_rest[s];
    V3 d = (len / norm(e)) * e;
    double w = std::sqrt(S.sp_w[s]);
    addx(f, i0, w * d);
    addx(f, i1, -w * d);
  }
  for (const Bend& B : S.bends) {
    V3 lap{0, 0, 0};
    for (size_t a = 0; a < B.v.size(); ++a) lap = lap + B.beta[a] * getx(x, B.v[a]);
    double ln = norm(lap);
    V3 d{0, 0, 0};
    if (ln > 1e-25) d = (B.w * B.rest_norm / ln) * lap;  /* BendingConstraint.h:164-187 */
    for (size_t a = 0; a < B.v.size(); ++a) addx(f, B.v[a], (B.w * B.beta[a]) * d);
  }
}

/* ---- articulated skeleton: kinematics and the rigid branch ----------------
 * Link::ComputeV0NTr, ComputeTildaV, UpdateT, guessNext, ReadT/WriteT
 * (sim/constants.h:83-228) and World::ComputeSolution's rigid branch
 * (World.h:1600-1670).  Links are visited in index order (parents first), which
 * gives the same values as the reference's depth-first recursion: a link reads
 * only its parent's prefix and Tr. */

/* Dense solve A X = B (n x n, k right-hand sides, row-major) by LU with full
 * pivoting (the largest |a| of the remaining block is the pivot), like
 * Eigen::FullPivLU::solve for an invertible A. */
static void fullpiv_solve(int n, int k, std::vector<double> A, const double* B, double* X) {
  std::vector<int> rp(n), cp(n);
  std::iota(rp.begin(), rp.end(), 0);
  std::iota(cp.begin(), cp.end(), 0);
  std::vector<double> Bw(B, B + (size_t)n * k);
  for (int p = 0; p < n; ++p) {
    int pr = p, pc = p;
    double best = -1.0;
    for (int r = p; r < n; ++r)
      for (int c = p; c < n; ++c)
        if (std::fabs(A[(size_t)r * n + c]) > best) { best = std::fabs(A[(size_t)r * n + c]); pr = r; pc = c; }
    if (pr != p) {
      for (int c = 0; c < n; ++c) std::swap(A[(size_t)p * n + c], A[(size_t)pr * n + c]);
      for (int c = 0; c < k; ++c) std::swap(Bw[(size_t)p * k + c], Bw[(size_t)pr * k + c]);
    }
    if (pc != p) {
      for (int r = 0; r < n; ++r) std::swap(A[(size_t)r * n + p], A[(size_t)r * n + pc]);
      std::swap(cp[p], cp[pc]);
    }
    const double piv = A[(size_t)p * n + p];
    for (int r = p + 1; r < n; ++r) {
      const double f = A[(size_t)r * n + p] / piv;
      A[(size_t)r * n + p] = f;
      for (int c = p + 1; c < n; ++c) A[(size_t)r * n + c] -= f * A[(size_t)p * n + c];
      for (int c = 0; c < k; ++c) Bw[(size_t)r * k + c] -= f * Bw[(size_t)p * k + c];
    }
  }
  std::vector<double> Y((size_t)n * k);
  for (int r = n - 1; r >= 0; --r)
    for (int c = 0; c < k; ++c) {
      double v = Bw[(size_t)r * k + c];
      for (int q = r + 1; q < n; ++q) v -= A[(size_t)r * n + q] * Y[(size_t)q * k + c];
      Y[(size_t)r * k + c] = v / A[(size_t)r * n + r];
    }
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < k; ++c) X[(size_t)cp[r] * k + c] = Y[(size_t)r * k + c];
}

/* Transformation::linearize: the rotation U V^T of the SVD of R */
static Xf xf_linearize(const Xf& t) {
  SVD3 sv = svd3(t.R);
  return Xf{mulT(sv.U, sv.V), t.d};
}

static M3 m3_from_rows(const double* r) {
  M3 a{};
  for (int i = 0; i < 9; ++i) at(a, i / 3, i % 3) = r[i];
  return a;
}

/* Link::ReadT for every link; the root's Tr (not part of the joint state) is
 * linearize(T), its value after the previous step's last ComputeV0NTr. */
static void skel_read(Skel& K) {
  for (LinkO& k : K.links) {
    if (k.type == DFEM_JOINT_ALL) {
      k.T = Xf{m3_from_rows(&K.jq[k.sdof]), V3{K.jq[k.sdof + 9], K.jq[k.sdof + 10], K.jq[k.sdof + 11]}};
      k.prevTr = Xf{m3_from_rows(&K.jqd[k.sdof]), V3{K.jqd[k.sdof + 9], K.jqd[k.sdof + 10], K.jqd[k.sdof + 11]}};
      k.Tr = xf_linearize(k.T);
    } else {
      k.mag = K.jq[k.sdof];
      k.prevmag = K.jqd[k.sdof];
    }
  }
}

static void skel_write(Skel& K) {
  for (const LinkO& k : K.links) {
    if (k.type == DFEM_JOINT_ALL) {
      for (int i = 0; i < 9; ++i) { K.jq[k.sdof + i] = at(k.T.R, i / 3, i % 3); K.jqd[k.sdof + i] = at(k.prevTr.R, i / 3, i % 3); }
      const double td[3] = {k.T.d.x, k.T.d.y, k.T.d.z}, pd[3] = {k.prevTr.d.x, k.prevTr.d.y, k.prevTr.d.z};
      for (int i = 0; i < 3; ++i) { K.jq[k.sdof + 9 + i] = td[i]; K.jqd[k.sdof + 9 + i] = pd[i]; }
    } else {
      K.jq[k.sdof] = k.mag;
      K.jqd[k.sdof] = k.prevmag;
    }
  }
}

/* Link::guessNext */
static void skel_guess(Skel& K) {
  for (LinkO& k : K.links) {
    if (k.type == DFEM_JOINT_ALL) {
      k.T.d = 2.0 * k.Tr.d - k.prevTr.d;
      double B[9], X[9];
      std::vector<double> A(9);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) { A[3 * r + c] = at(k.prevTr.R, r, c); B[3 * r + c] = at(k.Tr.R, r, c); }
      fullpiv_solve(3, 3, A, B, X);  /* prevTr.R^-1 Tr.R */
      k.T.R = mul(k.Tr.R, m3_from_rows(X));
      k.prevTr = k.Tr;
    } else {
      const double t = k.mag;
      k.mag = 2.0 * k.mag - k.prevmag;
      k.prevmag = t;
    }
  }
}

/* Link::ComputeV0NTr: every link's Tr and prefix, and V0 (3 per rigid vertex) */
static void skel_v0(Skel& K, std::vector<double>& V0) {
  V0.assign(3 * K.rv.size(), 0.0);
  for (LinkO& k : K.links) {
    if (k.type == DFEM_JOINT_ALL) {
      k.Tr = xf_linearize(k.T);
    } else if (k.type == DFEM_JOINT_ROTATIONAL) {
      const double C = std::cos(k.mag), S = std::sin(k.mag);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) at(k.Tr.R, r, c) = (C * (r == c ? 1.0 : 0.0) + S * at(k.nx, r, c)) + (1.0 - C) * at(k.nnt, r, c);
      k.Tr.d = k.d0;
    } else {
      k.Tr.d = k.mag * k.axis + k.d0;
    }
    if (k.parent >= 0) k.prefix = xf_mul(K.links[k.parent].prefix, K.links[k.parent].Tr);
    const Xf M = xf_mul(k.prefix, k.Tr);
    for (int j = k.r0; j < k.r1; ++j) {
      const V3 p = xf_apply(M, K.rest[j] - k.joint);
      V0[3 * j] = p.x; V0[3 * j + 1] = p.y; V0[3 * j + 2] = p.z;
    }
  }
}

/* Link::ComputeTildaV: dV0/ds (3 nr x ndof, row-major) at the state of the
 * last skel_v0 */
static void skel_tildav(Skel& K, const std::vector<double>& V0, std::vector<double>& TV) {
  const int nd = K.ndof;
  TV.assign(3 * K.rv.size() * (size_t)nd, 0.0);
  for (LinkO& k : K.links) {
    if (k.type == DFEM_JOINT_ROTATIONAL) {
      const double C = std::cos(k.mag), S = std::sin(k.mag);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) at(k.dT.R, r, c) = (-S * (r == c ? 1.0 : 0.0) + C * at(k.nx, r, c)) + S * at(k.nnt, r, c);
    } else if (k.type == DFEM_JOINT_PRISMATIC) {
      k.dT.R = M3{};
      k.dT.d = k.axis;
    }
  }
  for (int l = 0; l < K.L; ++l) {
    LinkO& me = K.links[l];
    me.suffix = xf_identity();
    for (int cur = l; K.links[cur].parent >= 0; cur = K.links[cur].parent)
      K.links[K.links[cur].parent].suffix = xf_mul(K.links[cur].Tr, K.links[cur].suffix);
    for (int j = me.r0; j < me.r1; ++j) {
      const V3 vinit = K.rest[j] - me.joint;
      double* row[3] = {&TV[(3 * (size_t)j) * nd], &TV[(3 * (size_t)j + 1) * nd], &TV[(3 * (size_t)j + 2) * nd]};
      int cur = l;
      for (; K.links[cur].parent >= 0; cur = K.links[cur].parent) {
        const LinkO& c = K.links[cur];
        V3 t = (c.type == DFEM_JOINT_ROTATIONAL) ? mv(c.prefix.R, mv(c.dT.R, xf_apply(c.suffix, vinit)))
                                                 : mv(c.prefix.R, c.dT.d);
        row[0][c.dof] = t.x; row[1][c.dof] = t.y; row[2][c.dof] = t.z;
      }
      const int c0 = K.links[cur].dof;
      const double vx = V0[3 * j], vy = V0[3 * j + 1], vz = V0[3 * j + 2];
      row[0][c0 + 1] = vz;  row[0][c0 + 2] = -vy;
      row[1][c0 + 0] = -vz; row[1][c0 + 2] = vx;
      row[2][c0 + 0] = vy;  row[2][c0 + 1] = -vx;
      row[0][c0 + 3] = 1.0; row[1][c0 + 4] = 1.0; row[2][c0 + 5] = 1.0;
    }
  }
}

/* Link::UpdateT */
static void skel_update(Skel& K, const std::vector<double>& s) {
  for (LinkO& k : K.links) {
    if (k.type == DFEM_JOINT_PRISMATIC) {
      k.mag += s[k.dof];
    } else if (k.type == DFEM_JOINT_ROTATIONAL) {
      const double C = std::cos(k.mag), S = std::sin(k.mag);
      k.mag = std::atan2(S + C * s[k.dof], C - S * s[k.dof]);
    } else {
      const V3 w{s[k.dof], s[k.dof + 1], s[k.dof + 2]}, l{s[k.dof + 3], s[k.dof + 4], s[k.dof + 5]};
      M3 t{};
      at(t, 0, 0) = 1; at(t, 0, 1) = -w.z; at(t, 0, 2) = w.y;
      at(t, 1, 0) = w.z; at(t, 1, 1) = 1; at(t, 1, 2) = -w.x;
      at(t, 2, 0) = -w.y; at(t, 2, 1) = w.x; at(t, 2, 2) = 1;
      k.T.R = mul(t, k.Tr.R);
      k.T.d = mv(t, k.Tr.d) + l;
    }
  }
}

/* Qf^-1 b on the free vertices (b's rigid entries are ignored) */
static void qf_solve(const Scene& S, const double* b, double* x) {
  std::vector<double> bb(b, b + 3 * (size_t)S.N);
  for (int v : S.skel.rv)
    for (int c = 0; c < 3; ++c) bb[3 * (size_t)v + c] = 0.0;
  solve(*S.qf, bb.data(), x);
}

/* y = H_{rows, cols} x restricted: rows/cols each "free" (-1) or "rigid" (1),
 * x and y full 3N vectors (entries outside `cols` / `rows` ignored / zero) */
static void H_block_mul(const Scene& S, int rows, int cols, const double* x, double* y) {
  const std::vector<int>& ri = S.skel.ridx;
  for (int i = 0; i < S.N; ++i) {
    double a = 0, b = 0, c = 0;
    if ((ri[i] >= 0 ? 1 : -1) == rows)
      for (auto& e : S.Hrows[i]) {
        if ((ri[e.first] >= 0 ? 1 : -1) != cols) continue;
        a += e.second * x[3 * e.first]; b += e.second * x[3 * e.first + 1]; c += e.second * x[3 * e.first + 2];
      }
    y[3 * i] = a; y[3 * i + 1] = b; y[3 * i + 2] = c;
  }
}

/* QbMmQcLQfm1QcLT = Qb_M - Qc_L Qf^-1 Qc_L^T (World.h:1134-1135), scalar
 * (kron(., I3) in the reference), one Qf solve per three rigid vertices */
static bool skel_precompute(Scene& S) {
  Skel& K = S.skel;
  const int N = S.N, nr = (int)K.rv.size();
  std::vector<std::vector<std::pair<int, double>>> rows(N);
  for (int i = 0; i < N; ++i) {
    if (K.ridx[i] >= 0) { rows[i].push_back({i, 1.0}); continue; }
    for (auto& e : S.Hrows[i])
      if (K.ridx[e.first] < 0) rows[i].push_back(e);
  }
  delete S.qf;
  S.qf = new Scene();
  S.qf->N = N;
  S.qf->Hrows.swap(rows);
  rcm_order(*S.qf);
  if (!factor(*S.qf)) { S.err = "Qf factorisation failed"; return false; }
  K.Srr.assign((size_t)nr * nr, 0.0);
  std::vector<double> b(3 * (size_t)N), w(3 * (size_t)N);
  for (int j0 = 0; j0 < nr; j0 += 3) {
    std::fill(b.begin(), b.end(), 0.0);
    for (int c = 0; c < 3 && j0 + c < nr; ++c)
      for (auto& e : S.Hrows[K.rv[j0 + c]])  /* column r_j of Hs (symmetric) on the free rows */
        if (K.ridx[e.first] < 0) b[3 * (size_t)e.first + c] = e.second;
    solve(*S.qf, b.data(), w.data());
    for (int c = 0; c < 3 && j0 + c < nr; ++c)
      for (int i = 0; i < nr; ++i) {
        double v = 0, acc = 0;
        for (auto& e : S.Hrows[K.rv[i]]) {
          if (e.first == K.rv[j0 + c]) v = e.second;
          if (K.ridx[e.first] < 0) acc += e.second * w[3 * (size_t)e.first + c];
        }
        K.Srr[(size_t)i * nr + j0 + c] = v - acc;
      }
  }
  return true;
}

/* ProjectiveDynamicsMethod with bones: the rigid vertices follow the links,
 * the free ones are solved through the Schur complement (ComputeSolution's
 * rigid branch, World.h:1611-1669) */
static int pd_solve_skel(Scene& S, const double* x, const double* qn, const double* act, double* out, int nthreads) {
  Skel& K = S.skel;
  const int N = S.N, n3 = 3 * N, nr = (int)K.rv.size(), nd = K.ndof;
  std::vector<double> b(n3), xk(qn, qn + n3), xold(n3, 0.0), c(n3), t1(n3), t2(n3), V0, TV;
  const double ih2 = 1.0 / (S.h * S.h);
  for (int i = 0; i < N; ++i)
    for (int q = 0; q < 3; ++q) b[3 * i + q] = S.mass[i] * ih2 * qn[3 * i + q];
  std::vector<double> Xfree(x, x + n3);           /* mNonrigidX */
  for (int v : K.rv) for (int q = 0; q < 3; ++q) Xfree[3 * (size_t)v + q] = 0.0;
  std::vector<double> HffX(n3), HrfX(n3);
  H_block_mul(S, -1, -1, Xfree.data(), HffX.data());   /* Qf mNonrigidX */
  H_block_mul(S, 1, -1, Xfree.data(), HrfX.data());    /* Qc_L mNonrigidX */
  /* S = tildaV^T kron(Srr, I3) tildaV, assembled per iteration */
  auto rigid_full = [&](const std::vector<double>& vr, std::vector<double>& full) {
    std::fill(full.begin(), full.end(), 0.0);
    for (int j = 0; j < nr; ++j)
      for (int q = 0; q < 3; ++q) full[3 * (size_t)K.rv[j] + q] = vr[3 * j + q];
  };
  skel_read(K);
  skel_guess(K);
  int it = 0;
  std::vector<double> full(n3), HfrV(n3), HrrV(n3), mcf(n3), sr(n3), Hrsr(n3), hvf(n3), vs(3 * (size_t)nr);
  for (int i = 0; i < S.K; ++i) {
    skel_v0(K, V0);
    for (int j = 0; j < nr; ++j)
      for (int q = 0; q < 3; ++q) xk[3 * (size_t)K.rv[j] + q] = V0[3 * j + q];
    double e2 = 0;
    for (int k = 0; k < n3; ++k) { double d = xk[k] - xold[k]; e2 += d * d; }
    if (std::sqrt(e2) / n3 < 5e-7) break;  /* EPS, World.h:891-895 */
    xold = xk;
    std::copy(b.begin(), b.end(), c.begin());
    local_Jd(S, xk.data(), act, c.data(), nthreads);       /* ori_c = b + J d */
    skel_tildav(K, V0, TV);
    rigid_full(V0, full);
    H_block_mul(S, -1, 1, full.data(), HfrV.data());        /* Qc_L^T V0 */
    H_block_mul(S, 1, 1, full.data(), HrrV.data());         /* Qb_M V0 */
    for (int k = 0; k < n3; ++k) mcf[k] = c[k] - HfrV[k] - HffX[k];
    std::vector<double> mcs(nd, 0.0), rr(3 * (size_t)nr);
    for (int j = 0; j < nr; ++j)
      for (int q = 0; q < 3; ++q) {
        const size_t g = 3 * (size_t)K.rv[j] + q;
        rr[3 * j + q] = c[g] - HrrV[g] - HrfX[g];
      }
    for (int a = 0; a < nd; ++a) {
      double v = 0;
      for (int r = 0; r < 3 * nr; ++r) v += TV[(size_t)r * nd + a] * rr[r];
      mcs[a] = v;
    }
    for (int l = 1; l < K.L; ++l)                          /* mcs[6+i] += mJointTorque[i] */
      if (K.links[l].chan >= 0) mcs[K.links[l].dof] += act[K.links[l].chan];
    std::vector<double> Sm((size_t)nd * nd, 0.0), KT(3 * (size_t)nr * nd);
    for (int i2 = 0; i2 < nr; ++i2)                         /* kron(Srr, I3) tildaV */
      for (int q = 0; q < 3; ++q)
        for (int a = 0; a < nd; ++a) {
          double v = 0;
          for (int j = 0; j < nr; ++j) v += K.Srr[(size_t)i2 * nr + j] * TV[(3 * (size_t)j + q) * nd + a];
          KT[(3 * (size_t)i2 + q) * nd + a] = v;
        }
    for (int a = 0; a < nd; ++a)
      for (int bq = 0; bq < nd; ++bq) {
        double v = 0;
        for (int r = 0; r < 3 * nr; ++r) v += TV[(size_t)r * nd + a] * KT[(size_t)r * nd + bq];
        Sm[(size_t)a * nd + bq] = v;
      }
    for (int k = 0; k < n3; ++k) t1[k] = -mcf[k];
    qf_solve(S, t1.data(), sr.data());                      /* solve_result = Qf^-1 (-mcf) */
    H_block_mul(S, 1, -1, sr.data(), Hrsr.data());          /* Qc_L solve_result */
    std::vector<double> tmp(nd), sv(nd);
    for (int a = 0; a < nd; ++a) {
      double v = 0;
      for (int j = 0; j < nr; ++j)
        for (int q = 0; q < 3; ++q) v += TV[(3 * (size_t)j + q) * nd + a] * Hrsr[3 * (size_t)K.rv[j] + q];
      tmp[a] = mcs[a] + v;
    }
    fullpiv_solve(nd, 1, Sm, tmp.data(), sv.data());        /* S.fullPivLu().solve(tmp) */
    for (int j = 0; j < nr; ++j)                            /* tildaV s */
      for (int q = 0; q < 3; ++q) {
        double v = 0;
        for (int a = 0; a < nd; ++a) v += TV[(3 * (size_t)j + q) * nd + a] * sv[a];
        vs[3 * j + q] = v;
      }
    rigid_full(vs, full);
    H_block_mul(S, -1, 1, full.data(), t2.data());          /* Qc^T s = Qc_L^T tildaV s */
    for (int k = 0; k < n3; ++k) t1[k] = mcf[k] - t2[k];
    qf_solve(S, t1.data(), hvf.data());
    skel_update(K, sv);
    for (int v = 0; v < N; ++v)
      if (K.ridx[v] < 0)
        for (int q = 0; q < 3; ++q) xk[3 * (size_t)v + q] = x[3 * (size_t)v + q] + hvf[3 * (size_t)v + q];
    ++it;
  }
  skel_v0(K, V0);
  for (int j = 0; j < nr; ++j)
    for (int q = 0; q < 3; ++q) xk[3 * (size_t)K.rv[j] + q] = V0[3 * j + q];
  skel_write(K);
  std::copy(xk.begin(), xk.end(), out);
  return it;
}

/* ProjectiveDynamicsMethod (World.h:835-917) with the iterate history */
static int pd_solve(const Scene& S, const double* x, const double* qn, const double* act,
                    std::vector<double>* hist, double* out, int nthreads) {
  int N = S.N, n3 = 3 * N;
  std::vector<double> b(n3), Hx(n3), xk(qn, qn + n3), xold(n3, 0.0), rhs(n3), hvf(n3);
  double ih2 = 1.0 / (S.h * S.h);
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) b[3 * i + c] = S.mass[i] * ih2 * qn[3 * i + c];
  H_mul(S, x, Hx.data());  /* Qf * mNonrigidX, constant over the step */
  if (hist) hist->assign(xk.begin(), xk.end());
  int it = 0;
  for (int i = 0; i < S.K; ++i) {
    double e2 = 0;
    for (int k = 0; k < n3; ++k) { double d = xk[k] - xold[k]; e2 += d * d; }
    if (std::sqrt(e2) / n3 < 5e-7) break;  /* EPS, World.h:214,891-895 */
    xold = xk;
    for (int k = 0; k < n3; ++k) rhs[k] = b[k] - Hx[k];
    local_Jd(S, xk.data(), act, rhs.data(), nthreads);  /* ori_c = b + J d; mcf = ori_c - Qf x */
    solve(S, rhs.data(), hvf.data());
    for (int k = 0; k < n3; ++k) xk[k] = x[k] + hvf[k];
    ++it;
    if (hist) hist->insert(hist->end(), xk.begin(), xk.end());
  }
  std::copy(xk.begin(), xk.end(), out);
  return it;
}

/* ---- underwater drag and lift ---------------------------------------------
 * Dfobj::ComputeDragForces (sim/Dfobj.h:904-998) per surface face p1 p2 p3
 * (outward winding) with vertex velocities v1 v2 v3, water at rest:
 *   v_rel = -(v1+v2+v3)/3 (face skipped when |v_rel| < 1e-6), u = v_rel/|v_rel|,
 *   d = -n (n the unit face normal), area = |(p2-p1) x (p3-p1)| / 2,
 *   c = d.u, aoa = pi/2 - acos(c) (= asin c); only faces with c > 0:
 *   drag = 500 area Cd(aoa) |v_rel|^2 u with Cd = (1-0)(1-cos 2 aoa)/2 + 0 = c^2,
 *   lift = 500 area Cl(aoa) |v_rel|^2 (normalize(u x d) x u), Cl the piecewise
 *   linear table of Dfobj::Cl in degrees with the 85 degree cutoff,
 *   each clipped to norm 1e3; each vertex of the face receives (drag + lift)/3.
 * Written once for double and once for a forward-mode dual number (value and
 * three derivatives) that the adjoint uses, seeding one input vector at a time. */
struct Dual3 {
  double v = 0, d[3] = {0, 0, 0};
  Dual3(double a = 0.0) : v(a) {}
};
static inline Dual3 dconst(double a) { return Dual3(a); }
static inline double val(double a) { return a; }
static inline double val(const Dual3& a) { return a.v; }
static inline Dual3 operator+(const Dual3& a, const Dual3& b) { Dual3 r; r.v = a.v + b.v; for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] + b.d[k]; return r; }
static inline Dual3 operator-(const Dual3& a, const Dual3& b) { Dual3 r; r.v = a.v - b.v; for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] - b.d[k]; return r; }
static inline Dual3 operator*(const Dual3& a, const Dual3& b) { Dual3 r; r.v = a.v * b.v; for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k]; return r; }
static inline Dual3 operator/(const Dual3& a, const Dual3& b) { Dual3 r; r.v = a.v / b.v; for (int k = 0; k < 3; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v; return r; }
static inline Dual3 dsqrt(const Dual3& a) { Dual3 r; r.v = std::sqrt(a.v); for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] / (2.0 * r.v); return r; }
static inline double dsqrt(double a) { return std::sqrt(a); }
static inline Dual3 dasin(const Dual3& a) { Dual3 r; r.v = std::asin(a.v); double q = 1.0 / std::sqrt(1.0 - a.v * a.v); for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * q; return r; }
static inline double dasin(double a) { return std::asin(a); }

template <typename T> struct TV3 { T x, y, z; };
template <typename T> static inline TV3<T> tadd(const TV3<T>& a, const TV3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> static inline TV3<T> tsub(const TV3<T>& a, const TV3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> static inline TV3<T> tscale(const T& s, const TV3<T>& a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T> static inline T tdot(const TV3<T>& a, const TV3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> static inline TV3<T> tcross(const TV3<T>& a, const TV3<T>& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

/* Dfobj::Cl (sim/Dfobj.h:813-838) with cutoff 85 and the table
   x = {-90, -10, -5, 15, 90}, y = {-0.5, -1.26, 0, 1.8, 0.5} (degrees):
   linear interpolation on the first matching segment. */
template <typename T> static T lift_coefficient(const T& aoa) {
  static const double xs[5] = {-90, -10, -5, 15, 90}, ys[5] = {-0.5, -1.26, 0.0, 1.8, 0.5};
  const T theta = T(180.0 / M_PI) * aoa;
  const double th = val(theta);
  const T zero(0.0);
  if (std::fabs(th) > 85.0) return zero;
  for (int k = 0; k < 4; ++k) {
    const bool in = (k < 2) ? (xs[k] <= th && th < xs[k + 1]) : (xs[k] <= th && th <= xs[k + 1]);
    if (in) {
      const T t = T(1.0 / (xs[k + 1] - xs[k])) * (theta - T(xs[k]));
      return T(ys[k + 1] - ys[k]) * t + T(ys[k]);   /* (1 - t) y_k + t y_{k+1} */
    }
  }
  return zero;
}

/* The force one face adds to each of its three vertices. */
template <typename T>
static TV3<T> drag_face_force(const TV3<T>& p1, const TV3<T>& p2, const TV3<T>& p3, const TV3<T>& v1,
                              const TV3<T>& v2, const TV3<T>& v3) {
  const TV3<T> zero{T(0.0), T(0.0), T(0.0)};
  const TV3<T> vrel = tscale(T(-1.0 / 3.0), tadd(tadd(v1, v2), v3));
  const T s2 = tdot(vrel, vrel);
  const T s = dsqrt(s2);
  if (val(s) < 1e-6) return zero;
  const TV3<T> u = tscale(T(1.0) / s, vrel);
  const TV3<T> nv = tcross(tsub(p2, p1), tsub(p3, p1));
  const T an = dsqrt(tdot(nv, nv));
  const T area = T(0.5) * an;
  const TV3<T> dd = tscale(T(-1.0) / an, nv);
  const T c = tdot(dd, u);
  if (!(val(c) > 0.0)) return zero;
  TV3<T> fd = tscale(T(500.0) * area * (c * c) * s2, u);
  /* Cl vanishes above 85 degrees; c >= 1 (rounding) lies there too */
  const T cl = val(c) < 1.0 ? lift_coefficient(dasin(c)) : T(0.0);
  const TV3<T> w = tcross(u, dd);
  const T wn2 = tdot(w, w);
  TV3<T> fl = zero;
  if (val(wn2) > 0.0) {
    const TV3<T> dl = tcross(tscale(T(1.0) / dsqrt(wn2), w), u);
    fl = tscale(T(500.0) * area * cl * s2, dl);
  }
  const double fmax = 1.0e3;
  const T fdn = dsqrt(tdot(fd, fd)), fln = dsqrt(tdot(fl, fl));
  if (val(fdn) > fmax) fd = tscale(T(fmax) / fdn, fd);
  if (val(fln) > fmax) fl = tscale(T(fmax) / fln, fl);
  return tscale(T(1.0 / 3.0), tadd(fd, fl));
}


static inline TV3<double> tv(const double* x, int i) { return {x[3 * i], x[3 * i + 1], x[3 * i + 2]}; }

/* Per-vertex external force f_ext of the step (zero unless underwater). */
static void drag_forces(const Scene& S, const double* x, const double* v, double* f) {
  std::fill(f, f + 3 * S.N, 0.0);
  for (const auto& fc : S.drag_f) {
    const TV3<double> g = drag_face_force(tv(x, fc[0]), tv(x, fc[1]), tv(x, fc[2]), tv(v, fc[0]), tv(v, fc[1]), tv(v, fc[2]));
    for (int k = 0; k < 3; ++k) {
      f[3 * fc[k]] += g.x; f[3 * fc[k] + 1] += g.y; f[3 * fc[k] + 2] += g.z;
    }
  }
}

/* Cotangents of x and v from the cotangent fb of the per-vertex drag force. */
static void drag_forces_vjp(const Scene& S, const double* x, const double* v, const double* fb, double* xb, double* vb) {
  for (const auto& fc : S.drag_f) {
    double gb[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c) gb[c] += fb[3 * fc[k] + c];
    for (int q = 0; q < 6; ++q) {  /* seed input vector q: p1 p2 p3 v1 v2 v3 */
      TV3<Dual3> in[6];
      for (int j = 0; j < 6; ++j) {
        const double* src = j < 3 ? x : v;
        const int vi = fc[j % 3];
        in[j] = {dconst(src[3 * vi]), dconst(src[3 * vi + 1]), dconst(src[3 * vi + 2])};
      }
      in[q].x.d[0] = 1.0; in[q].y.d[1] = 1.0; in[q].z.d[2] = 1.0;
      const TV3<Dual3> g = drag_face_force(in[0], in[1], in[2], in[3], in[4], in[5]);
      double* out = (q < 3 ? xb : vb) + 3 * fc[q % 3];
      for (int k = 0; k < 3; ++k) out[k] += gb[0] * g.x.d[k] + gb[1] * g.y.d[k] + gb[2] * g.z.d[k];
    }
  }
}

static void step_prep(const Scene& S, const double* x, const double* v, double* vwc, double* qn) {
  /* Environment::Step adds g*h to v of gravity-enabled bodies (none when
     underwater, which sets the drag force instead); TimeStepping:
     v_wc = v + h M^-1 f_ext, q_n = x + h v_wc. */
  std::vector<double> f(3 * (size_t)S.N, 0.0);
  if (!S.drag_f.empty()) drag_forces(S, x, v, f.data());
  for (int i = 0; i < S.N; ++i) {
    double gm = S.underwater ? 0.0 : S.gmask[i];
    double g3[3] = {S.g.x, S.g.y, S.g.z};
    for (int c = 0; c < 3; ++c) {
      vwc[3 * i + c] = v[3 * i + c] + gm * g3[c] * S.h + S.h * (f[3 * i + c] / S.mass[i]);
      qn[3 * i + c] = x[3 * i + c] + S.h * vwc[3 * i + c];
    }
  }
}

/* ---- contact ------------------------------------------------------------------
 * Vertex-face continuous collision test restated from the arcsim routines the
 * reference calls (sim/utils/arcsim/collision.cpp:127-326):  the vertex moves
 * from its step-start position p0 to p1, the obstacle face is static; the
 * times where the four points are coplanar are the roots in [0,1] of a cubic
 * (plus t = 1); at each, an impact is reported when the vertex is within
 * thickness * mult of the face plane and inside the face (at t = 1 also
 * within that distance of a face vertex or edge line).  The normal is the
 * (unnormalised) face normal oriented against the relative approach. */
static const double kThickness = 1e-4;  /* Impact::thickness */

static inline double stp(V3 u, V3 v, V3 w) { return dot(u, cross(v, w)); }
static inline V3 normalize(V3 a) { double n = norm(a); return (1.0 / n) * a; }
static inline double sgnd(double x) { return x < 0 ? -1.0 : 1.0; }

static int ccd_quadratic(double a, double b, double c, double x[2]) {
  double d = b * b - 4 * a * c;
  if (d < 0) { x[0] = -b / (2 * a); return 0; }
  double q = -(b + sgnd(b) * std::sqrt(d)) / 2;
  int i = 0;
  if (std::fabs(a) > 1e-12 * std::fabs(q)) x[i++] = q / a;
  if (std::fabs(q) > 1e-12 * std::fabs(c)) x[i++] = c / q;
  if (i == 2 && x[0] > x[1]) std::swap(x[0], x[1]);
  return i;
}

static double ccd_newton(double a, double b, double c, double d, double x0, int init_dir) {
  if (init_dir != 0) {
    double y0 = d + x0 * (c + x0 * (b + x0 * a)), ddy0 = 2 * b + x0 * (6 * a);
    x0 += init_dir * std::sqrt(std::fabs(2 * y0 / ddy0));
  }
  for (int iter = 0; iter < 100; ++iter) {
    double y = d + x0 * (c + x0 * (b + x0 * a));
    double dy = c + x0 * (2 * b + x0 * 3 * a);
    if (dy == 0) return x0;
    double x1 = x0 - y / dy;
    if (std::fabs(x0 - x1) < 1e-6) return x0;
    x0 = x1;
  }
  return x0;
}

static int ccd_cubic(double a, double b, double c, double d, double x[3]) {
  /* arcsim's solve_quadratic leaves xc[0] unset when it finds no root and the
     discriminant is >= 0 (the linear case of a static face); the reference
     then starts Newton's method from an uninitialised value.  0 here. */
  double xc[2] = {0.0, 0.0};
  int ncrit = ccd_quadratic(3 * a, 2 * b, c, xc);
  if (ncrit == 0) { x[0] = ccd_newton(a, b, c, d, xc[0], 0); return 1; }
  if (ncrit == 1) return ccd_quadratic(b, c, d, x);
  double yc[2] = {d + xc[0] * (c + xc[0] * (b + xc[0] * a)), d + xc[1] * (c + xc[1] * (b + xc[1] * a))};
  int i = 0;
  if (yc[0] * a >= 0) x[i++] = ccd_newton(a, b, c, d, xc[0], -1);
  if (yc[0] * yc[1] <= 0) {
    int closer = std::fabs(yc[0]) < std::fabs(yc[1]) ? 0 : 1;
    x[i++] = ccd_newton(a, b, c, d, xc[closer], closer == 0 ? 1 : -1);
  }
  if (yc[1] * a <= 0) x[i++] = ccd_newton(a, b, c, d, xc[1], 1);
  return i;
}

static double signed_vf(V3 x, V3 y0, V3 y1, V3 y2, V3* n, double w[4]) {
  *n = cross(normalize(y1 - y0), normalize(y2 - y0));
  if (dot(*n, *n) < 1e-6) return std::numeric_limits<double>::infinity();
  *n = normalize(*n);
  double h = dot(x - y0, *n);
  double b0 = stp(y1 - x, y2 - x, *n), b1 = stp(y2 - x, y0 - x, *n), b2 = stp(y0 - x, y1 - x, *n);
  w[0] = 1; w[1] = -b0 / (b0 + b1 + b2); w[2] = -b1 / (b0 + b1 + b2); w[3] = -b2 / (b0 + b1 + b2);
  return h;
}

/* vertex (p0 -> p1) against a static face (q0, q1, q2); mult = 1 for obstacles */
static bool vf_impact(V3 p0, V3 p1, V3 q0, V3 q1, V3 q2, double mult, V3* n_out) {
  const double thick = kThickness * mult;
  /* box overlap of the vertex's swept box and the face box dilated by thick (collision.cpp:132) */
  double lo[3], hi[3], flo[3], fhi[3];
  const double pv[2][3] = {{p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}};
  const double qv[3][3] = {{q0.x, q0.y, q0.z}, {q1.x, q1.y, q1.z}, {q2.x, q2.y, q2.z}};
  for (int c = 0; c < 3; ++c) {
    lo[c] = std::min(pv[0][c], pv[1][c]); hi[c] = std::max(pv[0][c], pv[1][c]);
    flo[c] = std::min(qv[0][c], std::min(qv[1][c], qv[2][c])) - thick;
    fhi[c] = std::max(qv[0][c], std::max(qv[1][c], qv[2][c])) + thick;
    if (hi[c] < flo[c] || lo[c] > fhi[c]) return false;
  }
  V3 x0 = p0, v0 = p1 - p0;
  V3 x1 = q0 - x0, x2 = q1 - x0, x3 = q2 - x0;
  V3 v1 = -1.0 * v0, v2 = -1.0 * v0, v3 = -1.0 * v0;  /* static face: relative velocities */
  double a0 = stp(x1, x2, x3);
  double a1 = stp(v1, x2, x3) + stp(x1, v2, x3) + stp(x1, x2, v3);
  double a2 = stp(x1, v2, v3) + stp(v1, x2, v3) + stp(v1, v2, x3);
  double a3 = stp(v1, v2, v3);
  double t[4];
  int nsol = ccd_cubic(a3, a2, a1, a0, t);
  t[nsol++] = 1;
  for (int i = 0; i < nsol; ++i) {
    if (t[i] < 0 || t[i] > 1) continue;
    V3 xt = p0 + t[i] * v0;
    V3 n{0, 0, 0};
    double w[4] = {0, 0, 0, 0};
    double d = signed_vf(xt, q0, q1, q2, &n, w);
    bool inside = std::min(std::min(-w[1], -w[2]), -w[3]) >= -1e-6;
    if (t[i] == 1) {
      inside = inside || norm(xt - q0) < thick || norm(xt - q1) < thick || norm(xt - q2) < thick;
      inside = inside || norm(xt - q0 - (dot(xt - q0, q1 - q0) / dot(q1 - q0, q1 - q0)) * (q1 - q0)) < thick;
      inside = inside || norm(xt - q1 - (dot(xt - q1, q2 - q1) / dot(q2 - q1, q2 - q1)) * (q2 - q1)) < thick;
      inside = inside || norm(xt - q2 - (dot(xt - q2, q0 - q2) / dot(q0 - q2, q0 - q2)) * (q0 - q2)) < thick;
    }
    V3 fn = cross(normalize(q1 - q0), normalize(q2 - q0));
    if (dot(n, w[1] * v1 + w[2] * v2 + w[3] * v3) > 0) n = -1.0 * fn; else n = fn;
    if (std::fabs(d) < thick && inside) { *n_out = n; return true; }
  }
  return false;
}

/* contact basis [n, t, b] (CollisionBrutal::computeBasis, collisionBrutal.h:408-426) */
static void contact_basis(V3 normal, V3 B[3]) {
  V3 tg = cross(normal, V3{1, 0, 0});
  if (norm(tg) < 1e-15) tg = cross(normal, V3{0, 1, 0});
  tg = normalize(tg);
  V3 bt = normalize(cross(normal, tg));
  B[0] = normalize(normal); B[1] = tg; B[2] = bt;
}

/* vertex (p0 -> p1) against a moving face (q*s -> q*e): arcsim's
 * vf_collision_test + collision_test (collision.cpp:118-128, 211-274) with the
 * swept boxes of the vertex and of the face dilated by thickness * mult.
 * Returns the impact's time t, distance |d| and normal (the face's start
 * normal, oriented against the vertex's approach, not unit length). */
static bool vf_impact_moving(V3 p0, V3 p1, const V3 qs[3], const V3 qe[3], double mult, V3* n_out, double* t_out,
                             double* d_out) {
  const double thick = kThickness * mult;
  const double pv[2][3] = {{p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}};
  for (int c = 0; c < 3; ++c) {
    double lo = std::min(pv[0][c], pv[1][c]), hi = std::max(pv[0][c], pv[1][c]);
    double flo = 1e300, fhi = -1e300;
    for (int k = 0; k < 3; ++k) {
      const double a = c == 0 ? qs[k].x : (c == 1 ? qs[k].y : qs[k].z);
      const double b = c == 0 ? qe[k].x : (c == 1 ? qe[k].y : qe[k].z);
      flo = std::min(flo, std::min(a, b));
      fhi = std::max(fhi, std::max(a, b));
    }
    if (hi < flo - thick || lo > fhi + thick) return false;
  }
  V3 x0 = p0, v0 = p1 - p0;
  V3 x1 = qs[0] - x0, x2 = qs[1] - x0, x3 = qs[2] - x0;
  V3 v1 = (qe[0] - qs[0]) - v0, v2 = (qe[1] - qs[1]) - v0, v3 = (qe[2] - qs[2]) - v0;
  double a0 = stp(x1, x2, x3);
  double a1 = stp(v1, x2, x3) + stp(x1, v2, x3) + stp(x1, x2, v3);
  double a2 = stp(x1, v2, v3) + stp(v1, x2, v3) + stp(v1, v2, x3);
  double a3 = stp(v1, v2, v3);
  double t[4];
  int nsol = ccd_cubic(a3, a2, a1, a0, t);
  t[nsol++] = 1;
  for (int i = 0; i < nsol; ++i) {
    if (t[i] < 0 || t[i] > 1) continue;
    V3 xt = p0 + t[i] * v0;
    V3 y0 = qs[0] + t[i] * (qe[0] - qs[0]), y1 = qs[1] + t[i] * (qe[1] - qs[1]), y2 = qs[2] + t[i] * (qe[2] - qs[2]);
    V3 n{0, 0, 0};
    double w[4] = {0, 0, 0, 0};
    double d = signed_vf(xt, y0, y1, y2, &n, w);
    bool inside = std::min(std::min(-w[1], -w[2]), -w[3]) >= -1e-6;
    if (t[i] == 1) {
      inside = inside || norm(xt - y0) < thick || norm(xt - y1) < thick || norm(xt - y2) < thick;
      inside = inside || norm(xt - y0 - (dot(xt - y0, y1 - y0) / dot(y1 - y0, y1 - y0)) * (y1 - y0)) < thick;
      inside = inside || norm(xt - y1 - (dot(xt - y1, y2 - y1) / dot(y2 - y1, y2 - y1)) * (y2 - y1)) < thick;
      inside = inside || norm(xt - y2 - (dot(xt - y2, y0 - y2) / dot(y0 - y2, y0 - y2)) * (y0 - y2)) < thick;
    }
    V3 fn = cross(normalize(qs[1] - qs[0]), normalize(qs[2] - qs[0]));
    if (dot(n, w[1] * v1 + w[2] * v2 + w[3] * v3) > 0) n = -1.0 * fn; else n = fn;
    if (std::fabs(d) < thick && inside) {
      *n_out = n; *t_out = t[i]; *d_out = std::fabs(d);
      return true;
    }
  }
  return false;
}

/* A soft impact of contact vertex a against soft face f (its node 4-tuple is
 * (a, face)); the step's list keeps one per tuple, refreshed in place. */
struct SelfImpact { int a, f; double t, d; V3 n; };

/* getSelfCollisionsInfo (collisionBrutal.h:645-700): per vertex the impact of
 * smallest t (ties at t = 1: smallest distance; earlier list entries win
 * otherwise), then the vertices grouped by face in ascending vertex order. */
static std::vector<SelfGroup> self_groups(const std::vector<SelfImpact>& simp) {
  std::map<int, int> closest;
  for (int i = 0; i < (int)simp.size(); ++i) {
    auto it = closest.find(simp[i].a);
    if (it == closest.end()) { closest[simp[i].a] = i; continue; }
    const SelfImpact& old = simp[it->second];
    if (simp[i].t < old.t) { it->second = i; continue; }
    if (old.t == 1 && old.d > simp[i].d) it->second = i;
  }
  std::vector<SelfGroup> out;
  for (auto& kv : closest) {
    const SelfImpact& im = simp[kv.second];
    int g = -1;
    for (int q = 0; q < (int)out.size(); ++q) if (out[q].f == im.f) { g = q; break; }
    if (g >= 0) out[g].verts.push_back(kv.first);
    else out.push_back(SelfGroup{im.f, im.n, {kv.first}});
  }
  return out;
}

/* forward-mode dual number with one derivative per input of a face group */
struct DN {
  double v = 0;
  std::vector<double> d;
  DN(double a = 0.0) : v(a) {}
};
static inline double val(const DN& a) { return a.v; }
static inline DN dn_combine(const DN& a, const DN& b, double v, double ca, double cb) {
  DN r(v);
  const size_t n = std::max(a.d.size(), b.d.size());
  r.d.assign(n, 0.0);
  for (size_t k = 0; k < a.d.size(); ++k) r.d[k] += ca * a.d[k];
  for (size_t k = 0; k < b.d.size(); ++k) r.d[k] += cb * b.d[k];
  return r;
}
static inline DN operator+(const DN& a, const DN& b) { return dn_combine(a, b, a.v + b.v, 1.0, 1.0); }
static inline DN operator-(const DN& a, const DN& b) { return dn_combine(a, b, a.v - b.v, 1.0, -1.0); }
static inline DN operator*(const DN& a, const DN& b) { return dn_combine(a, b, a.v * b.v, b.v, a.v); }
static inline DN operator/(const DN& a, const DN& b) {
  const double q = a.v / b.v;
  return dn_combine(a, b, q, 1.0 / b.v, -q / b.v);
}
static inline DN dsqrt(const DN& a) {
  DN r(std::sqrt(a.v));
  r.d.assign(a.d.size(), 0.0);
  for (size_t k = 0; k < a.d.size(); ++k) r.d[k] = a.d[k] / (2.0 * r.v);
  return r;
}

/* local frame [n, t, b] and back (local_basis^T f, local_basis r) */
template <typename T> static inline TV3<T> to_local(const V3 B[3], const TV3<T>& p) {
  return {p.x * B[0].x + p.y * B[0].y + p.z * B[0].z, p.x * B[1].x + p.y * B[1].y + p.z * B[1].z,
          p.x * B[2].x + p.y * B[2].y + p.z * B[2].z};
}
template <typename T> static inline TV3<T> to_world(const V3 B[3], const TV3<T>& r) {
  return {r.x * B[0].x + r.y * B[1].x + r.z * B[2].x, r.x * B[0].y + r.y * B[1].y + r.z * B[2].y,
          r.x * B[0].z + r.y * B[1].z + r.z * B[2].z};
}
template <typename T> static inline TV3<T> tdiv(const TV3<T>& a, const T& s) { return {a.x / s, a.y / s, a.z / s}; }

/* World::do_solve_friction (World.h:1246-1315): the sticking set (face +
 * sticking vertices) moves tangentially together; sliding vertices receive
 * mu times their normal force against their tangential slip, and the sticking
 * set the opposite sum. */
template <typename T>
static void solve_group_friction(const TV3<T>& p0, const T& m0, TV3<T>& r0, const std::vector<TV3<T>>& ps,
                                 const std::vector<T>& ms, std::vector<TV3<T>>& rs, const std::vector<char>& stick,
                                 double mu) {
  TV3<T> pstick = p0;
  T mstick = m0;
  const int n = (int)stick.size();
  for (int k = 0; k < n; ++k)
    if (stick[k]) { pstick = tadd(pstick, ps[k]); mstick = mstick + ms[k]; }
  TV3<T> pslide{T(0.0), T(0.0), T(0.0)};
  T mslide(0.0), fn(0.0);
  for (int k = 0; k < n; ++k)
    if (!stick[k]) { pslide = tadd(pslide, ps[k]); mslide = mslide + ms[k]; fn = fn + rs[k].x; }
  const TV3<T> v = tdiv(pstick, mstick);
  r0.y = v.y * m0 - p0.y;
  r0.z = v.z * m0 - p0.z;
  for (int k = 0; k < n; ++k)
    if (stick[k]) { rs[k].y = v.y * ms[k] - ps[k].y; rs[k].z = v.z * ms[k] - ps[k].z; }
  if (val(mslide) > 0) {
    TV3<T> rel = tsub(tdiv(pslide, mslide), tdiv(pstick, mstick));
    const T tl = dsqrt(rel.y * rel.y + rel.z * rel.z);
    rel = tdiv(rel, tl);
    const T mult = T(mu) * fn / (mslide + mstick);
    r0.y = r0.y + rel.y * mult * m0;
    r0.z = r0.z + rel.z * mult * m0;
    for (int k = 0; k < n; ++k)
      if (stick[k]) { rs[k].y = rs[k].y + rel.y * mult * ms[k]; rs[k].z = rs[k].z + rel.z * mult * ms[k]; }
    const TV3<T> abs_v0 = tdiv(tadd(p0, r0), m0);
    for (int k = 0; k < n; ++k)
      if (!stick[k]) {
        TV3<T> rk = tsub(tdiv(ps[k], ms[k]), abs_v0);
        const T tk = dsqrt(rk.y * rk.y + rk.z * rk.z);
        rk = tdiv(rk, tk);
        const T mk = T(-mu) * rs[k].x * ms[k] / (ms[k] + mstick);
        rs[k].y = mk * rk.y;
        rs[k].z = mk * rk.z;
      }
  }
}

/* One face group of the self branch of CollisionHandling (World.h:1462-1531).
 * P = forces + obstacle reactions of the face's vertices (P[0..2]) and of the
 * group's vertices (PL), masses = diag(Hs) (World::getVertexMass).  The group
 * vertices approaching the face (normal relative velocity <= 0) and the face
 * reach one normal velocity (the face's normal and tangential momenta are
 * pooled); their tangential forces come from the stick/slide iteration.  The
 * face's vertices end with the face's common velocity: outF[i] = v0 m_i - P_i;
 * a group vertex k receives outL[k] = B rs_k (zero if it left the group).
 * incl (when non-null) receives the membership decisions. */
template <typename T>
static void self_group_exchange(const V3 B[3], const TV3<T> P[3], const T mf[3], const std::vector<TV3<T>>& PL,
                                const std::vector<T>& mL, double mu, TV3<T> outF[3], std::vector<TV3<T>>& outL,
                                std::vector<char>* incl_out) {
  const T m0 = mf[0] + mf[1] + mf[2];
  const TV3<T> f0 = to_local(B, tadd(tadd(P[0], P[1]), P[2]));
  std::vector<int> inc;
  for (int k = 0; k < (int)PL.size(); ++k) {
    const TV3<T> f = to_local(B, PL[k]);
    if (val(f.x / mL[k] - f0.x / m0) <= 0) inc.push_back(k);
  }
  if (incl_out) {
    incl_out->assign(PL.size(), 0);
    for (int k : inc) (*incl_out)[k] = 1;
  }
  std::vector<T> ms;
  std::vector<TV3<T>> fs;
  T sm(0.0), smv(0.0);
  for (int k : inc) {
    ms.push_back(mL[k]);
    sm = sm + ms.back();
    fs.push_back(to_local(B, PL[k]));
    smv = smv + fs.back().x;
  }
  const int n = (int)inc.size();
  TV3<T> r0{T(0.0), T(0.0), T(0.0)};
  std::vector<TV3<T>> rs(n, TV3<T>{T(0.0), T(0.0), T(0.0)});
  for (int k = 0; k < n; ++k) {
    const T fn = (f0.x + smv) * ms[k] / (m0 + sm) - fs[k].x;
    rs[k].x = rs[k].x + fn;
    r0.x = r0.x - fn;
  }
  std::vector<char> stick(n, 1);
  for (;;) {
    solve_group_friction(f0, m0, r0, fs, ms, rs, stick, mu);
    bool changed = false;
    for (int k = 0; k < n; ++k)
      if (stick[k] && val(rs[k].y * rs[k].y + rs[k].z * rs[k].z) > val(T(mu) * rs[k].x * rs[k].x)) {
        changed = true;
        stick[k] = 0;
      }
    if (!changed) break;
  }
  const TV3<T> v0 = tdiv(tadd(to_world(B, f0), to_world(B, r0)), m0);
  for (int i = 0; i < 3; ++i) outF[i] = tsub(tscale(mf[i], v0), P[i]);
  outL.assign(PL.size(), TV3<T>{T(0.0), T(0.0), T(0.0)});
  for (int k = 0; k < n; ++k) outL[inc[k]] = to_world(B, rs[k]);
}

struct ObsImpact { int face; V3 n; };

/* What the adjoint of the contact phase needs from one run of it: every
 * computed Jacobi iteration's input ori_x, its relaxed rhs (prev) after the
 * update, whether it started its pass (prev restarts from its own rhs), the
 * impact normals of every contact vertex at that iteration (list order), the
 * mode of its CollisionHandling call, the pass's self-contact groups and the
 * self-force state before the call, and which computed iteration produced the
 * phase's output (0: the PD result).  The detection is discrete: impacts,
 * normals, groups and the stick/slide and membership decisions are constants
 * of the tape, as they are on the reference's CppAD tape (collision
 * detection runs in plain double). */
struct ContactTape {
  int out_src = 0;
  std::vector<std::vector<double>> ori, prev;
  std::vector<char> first;
  std::vector<std::vector<std::vector<V3>>> nrm;
  std::vector<double> hd;
  std::vector<char> mode;
  std::vector<int> gpass;
  std::vector<std::vector<SelfGroup>> groups;
  std::vector<std::vector<double>> sc_in;
};

/* The winning obstacle reaction of one contact vertex: the last impact whose
 * normal force is compressive (World.h:1364-1430: every later impact of the
 * vertex overwrites the earlier ones). */
struct ObsWin { bool hit = false; V3 B[3]; double r[3] = {0, 0, 0}; };
static ObsWin obstacle_reaction(V3 f, const std::vector<V3>& normals, double mu) {
  ObsWin w;
  for (const V3& nv : normals) {
    V3 B[3];
    contact_basis(nv, B);
    double fl[3] = {dot(B[0], f), dot(B[1], f), dot(B[2], f)};
    if (fl[0] > 0) continue;
    double rr[3] = {-fl[0], -fl[1], -fl[2]};
    double rt = std::sqrt(rr[1] * rr[1] + rr[2] * rr[2]);
    if (rt > mu * rr[0]) { rr[1] *= mu * rr[0] / rt; rr[2] *= mu * rr[0] / rt; }
    w.hit = true;
    w.B[0] = B[0]; w.B[1] = B[1]; w.B[2] = B[2];
    w.r[0] = rr[0]; w.r[1] = rr[1]; w.r[2] = rr[2];
  }
  return w;
}
static inline V3 reaction_world(const ObsWin& w) { return w.r[0] * w.B[0] + w.r[1] * w.B[1] + w.r[2] * w.B[2]; }

/* CollisionHandling (World.h:1317-1537) on the rhs of the contact vertices.
 * sc is the self-force state (m_self_contact_forces[m_current_index]), read
 * by the obstacle reactions and replaced by this call's self forces.  Returns
 * the mode: 0 = no contact (nothing changes, no buffer swap); 1 = no self
 * group (each obstacle-hit vertex's rhs := B r, the state becomes zero when
 * self contact is on); 2 = with self groups (rhs += obstacle reactions + self
 * forces of the groups, which see forces + obstacle reactions). */
static int collision_handling(const Scene& S, double* rhs, const std::vector<std::vector<V3>>& normals,
                              const std::vector<SelfGroup>& groups, const std::vector<double>& hd,
                              std::vector<double>& sc) {
  const int nc = (int)S.cverts.size();
  int nb_obs = 0;
  for (auto& l : normals) nb_obs += (int)l.size();
  const int nb_self = S.self_collide ? (int)groups.size() : 0;
  if (nb_obs == 0 && nb_self == 0) return 0;
  const V3 zero{0, 0, 0};
  std::vector<V3> forces(nc), cnext(nc, zero), snext(nc, zero);
  for (int a = 0; a < nc; ++a) forces[a] = getx(rhs, S.cverts[a]);
  for (int a = 0; a < nc; ++a) {
    const int gv = S.cverts[a];
    const V3 f = S.self_collide ? forces[a] + getx(sc.data(), a) : forces[a];
    const ObsWin w = obstacle_reaction(f, normals[a], S.mu_obs);
    if (!w.hit) continue;
    const V3 out = reaction_world(w);
    if (nb_self == 0) { rhs[3 * gv] = out.x; rhs[3 * gv + 1] = out.y; rhs[3 * gv + 2] = out.z; }
    if (S.self_collide) cnext[a] = out;
  }
  if (nb_self > 0) {
    for (const SelfGroup& g : groups) {
      V3 B[3];
      contact_basis(g.n, B);
      TV3<double> P[3], oF[3];
      double mf[3];
      for (int i = 0; i < 3; ++i) {
        const int a = S.cfaces[g.f][i];
        const V3 q = forces[a] + cnext[a];
        P[i] = {q.x, q.y, q.z};
        mf[i] = hd[S.cverts[a]];
      }
      std::vector<TV3<double>> PL, oL;
      std::vector<double> mL;
      for (int a : g.verts) {
        const V3 q = forces[a] + cnext[a];
        PL.push_back({q.x, q.y, q.z});
        mL.push_back(hd[S.cverts[a]]);
      }
      self_group_exchange(B, P, mf, PL, mL, S.mu_self, oF, oL, nullptr);
      for (int i = 0; i < 3; ++i) {
        V3& o = snext[S.cfaces[g.f][i]];
        o = o + V3{oF[i].x, oF[i].y, oF[i].z};
      }
      for (size_t k = 0; k < g.verts.size(); ++k) {
        V3& o = snext[g.verts[k]];
        o = o + V3{oL[k].x, oL[k].y, oL[k].z};
      }
    }
    for (int a = 0; a < nc; ++a) {
      const int gv = S.cverts[a];
      const V3 add = cnext[a] + snext[a];
      rhs[3 * gv] += add.x; rhs[3 * gv + 1] += add.y; rhs[3 * gv + 2] += add.z;
    }
  }
  if (S.self_collide)
    for (int a = 0; a < nc; ++a) { sc[3 * a] = snext[a].x; sc[3 * a + 1] = snext[a].y; sc[3 * a + 2] = snext[a].z; }
  return nb_self > 0 ? 2 : 1;
}

/* Contact phase of ProjectiveDynamicsMethod (World.h:925-1023) with obstacle
 * and (when on) soft-soft contacts.  ori_x enters as the PD result and leaves
 * as the returned positions; x_n1 follows the reference's (x_n1, ori_x)
 * bookkeeping exactly.  A pass ends the phase when it finds no new obstacle
 * impact and the number of self groups did not change
 * (CollisionBrutal::BaseUpdateCollisions' return value). */
static void contact_phase(Scene& S, const double* x_t, const double* vwc, const double* act, double* ori_x,
                          ContactTape* tape = nullptr) {
  const int N = S.N, n3 = 3 * N, nc = (int)S.cverts.size();
  S.last_passes = 0;
  if (tape) *tape = ContactTape();
  const bool soft = S.self_collide && !S.cfaces.empty();
  if (!S.collide || nc == 0 || (S.obs_f.empty() && !soft)) return;
  int computed = 0, src_ori = 0;
  std::vector<std::vector<ObsImpact>> imp(nc);
  std::vector<SelfImpact> simp;
  std::vector<SelfGroup> groups;
  std::vector<double> xold(n3, 0.0), x_n1(ori_x, ori_x + n3), rhs(n3), prev(n3, 0.0), jd(n3), Lxt(n3), Hx(n3);
  /* L x_t = Hs x_t - M/h^2 x_t ; C = Hs - diag(Hs) */
  H_mul(S, x_t, Hx.data());
  const double ih2 = 1.0 / (S.h * S.h);
  std::vector<double> hd(N, 0.0);
  for (int i = 0; i < N; ++i) {
    for (auto& e : S.Hrows[i]) if (e.first == i) hd[i] = e.second;
    for (int c = 0; c < 3; ++c) Lxt[3 * i + c] = Hx[3 * i + c] - S.mass[i] * ih2 * x_t[3 * i + c];
  }
  if (tape) tape->hd = hd;
  if (S.freeze == 1 && (int)S.frz.size() <= S.cur_step) S.frz.resize(S.cur_step + 1);
  for (int pass = 0; pass < S.max_passes; ++pass) {
    std::vector<std::vector<V3>> normals(nc);
    if (S.freeze == 2) {
      if (S.cur_step >= (int)S.frz.size() || pass >= (int)S.frz[S.cur_step].size()) break;
      normals = S.frz[S.cur_step][pass].normals;
      groups = S.frz[S.cur_step][pass].groups;
    } else {
    /* detection at ori_x (vertex start positions: x_t) */
    bool any = false;
    for (int a = 0; a < nc; ++a) {
      int gv = S.cverts[a];
      V3 p0 = getx(x_t, gv), p1 = getx(ori_x, gv);
      for (int f = 0; f < (int)S.obs_f.size(); ++f) {
        V3 n;
        if (!vf_impact(p0, p1, S.obs_x[S.obs_f[f][0]], S.obs_x[S.obs_f[f][1]], S.obs_x[S.obs_f[f][2]], 1.0, &n)) continue;
        any = true;
        bool found = false;
        for (auto& r : imp[a]) if (r.face == f) { r.n = n; found = true; }
        if (!found) imp[a].push_back({f, n});
      }
    }
    const int ngroups_prev = (int)groups.size();
    if (soft) {
      /* soft impacts (thickness x 2), vertex ascending then face ascending;
         a tuple found again is refreshed in place, a new one appended */
      for (int a = 0; a < nc; ++a) {
        if (!S.on_face[a]) continue;
        const int gv = S.cverts[a];
        const V3 p0 = getx(x_t, gv), p1 = getx(ori_x, gv);
        for (int f = 0; f < (int)S.cfaces.size(); ++f) {
          const std::array<int, 3>& cf = S.cfaces[f];
          if (cf[0] == a || cf[1] == a || cf[2] == a) continue;
          V3 qs[3], qe[3];
          for (int k = 0; k < 3; ++k) { qs[k] = getx(x_t, S.cverts[cf[k]]); qe[k] = getx(ori_x, S.cverts[cf[k]]); }
          V3 n;
          double t, d;
          if (!vf_impact_moving(p0, p1, qs, qe, 2.0, &n, &t, &d)) continue;
          bool found = false;
          for (auto& r : simp)
            if (r.a == a && r.f == f) { r.t = t; r.d = d; r.n = n; found = true; break; }
          if (!found) simp.push_back(SelfImpact{a, f, t, d, n});
        }
      }
      groups = self_groups(simp);
    }
    if (!any && ngroups_prev == (int)groups.size()) break;
    for (int a = 0; a < nc; ++a)
      for (auto& r : imp[a]) normals[a].push_back(r.n);
    if (S.freeze == 1) S.frz[S.cur_step].push_back(Scene::PassRecord{normals, groups});
    }
    S.last_passes = pass + 1;
    if (tape) tape->groups.push_back(groups);
    for (int it = 0; it < S.K; ++it) {
      for (int k = 0; k < n3; ++k) ori_x[k] = x_n1[k];
      src_ori = computed;
      double err = 0;
      for (int k = 0; k < n3; ++k) err = std::max(err, std::fabs(ori_x[k] - xold[k]));
      if (err < 5e-7) break;
      std::fill(jd.begin(), jd.end(), 0.0);
      local_Jd(S, ori_x, act, jd.data(), 1);
      /* m_rhs_speed = M v_wc + h (J d - L x_t) - h^2 C (ori_x - x_t)/h */
      for (int i = 0; i < N; ++i) {
        double cdx[3] = {0, 0, 0};
        for (auto& e : S.Hrows[i])
          if (e.first != i)
            for (int c = 0; c < 3; ++c) cdx[c] += e.second * (ori_x[3 * e.first + c] - x_t[3 * e.first + c]);
        for (int c = 0; c < 3; ++c)
          rhs[3 * i + c] = S.mass[i] * vwc[3 * i + c] + S.h * (jd[3 * i + c] - Lxt[3 * i + c]) - S.h * cdx[c];
      }
      if (it == 0) prev = rhs;
      if (tape) tape->sc_in.push_back(S.sc_cur);
      const int mode = collision_handling(S, rhs.data(), normals, groups, hd, S.sc_cur);
      for (int k = 0; k < n3; ++k) prev[k] = S.alpha * rhs[k] + (1.0 - S.alpha) * prev[k];
      for (int i = 0; i < N; ++i)
        for (int c = 0; c < 3; ++c) x_n1[3 * i + c] = x_t[3 * i + c] + prev[3 * i + c] / S.h / hd[i];
      for (int k = 0; k < n3; ++k) xold[k] = ori_x[k];
      ++computed;
      if (tape) {
        tape->ori.emplace_back(ori_x, ori_x + n3);
        tape->prev.push_back(prev);
        tape->first.push_back(it == 0 ? 1 : 0);
        tape->nrm.push_back(normals);
        tape->mode.push_back((char)mode);
        tape->gpass.push_back((int)tape->groups.size() - 1);
      }
    }
  }
  if (tape) tape->out_src = src_ori;
}

/* ---- adjoint ---------------------------------------------------------------- */

/* VJP of the corotated projection: given dmd, dmdv (3x3) return dF */
static M3 corot_vjp(const M3& F, const M3& gmd, const M3& gmdv) {
  SVD3 s = svd3(F);
  VolProj vp = volume_projection(s.s, true);
  M3 gR = gmd;
  if (det(F) < 0) setcol(gR, 2, -1.0 * col(gmd, 2));
  M3 MR = mul(Tmul(s.U, gR), s.V);     /* U^T gR V */
  M3 MG = mul(Tmul(s.U, gmdv), s.V);   /* U^T gG V */
  M3 P{};
  const int pair_of[3][3] = {{-1, 0, 1}, {0, -1, 2}, {1, 2, -1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      if (i == j) {
        double d = 0;
        for (int k = 0; k < 3; ++k) d += at(MG, k, k) * vp.J[k][i];
        at(P, i, i) = d;
      } else {
        double ssum = s.s[i] + s.s[j];
        double b = (vp.g[i] + vp.g[j]) / ssum;
        double a = vp.dd[pair_of[i][j]];
        double symG = 0.5 * (at(MG, i, j) + at(MG, j, i));
        double asymG = 0.5 * (at(MG, i, j) - at(MG, j, i));
        double asymR = (at(MR, i, j) - at(MR, j, i)) / ssum;
        at(P, i, j) = a * symG + b * asymG + asymR;
      }
    }
  return mulT(mul(s.U, P), s.V);  /* U P V^T */
}

struct Grad {
  std::vector<double> gE, gnu, gact;  /* gact per segment for one step */
};

/* adjoint of local_Jd: given ybar (3N), accumulate xbar += (dJd/dx)^T ybar and
 * parameter gradients of  ybar . J(theta) d(x, theta). */
static void local_Jd_vjp(const Scene& S, const double* x, const double* act, const double* yb,
                         double* xb, double* gE, double* gnu, double* gact) {
  int NT = (int)S.tets.size();
  for (int t = 0; t < NT; ++t) {
    const Tet& T = S.tets[t];
    M3 F = deformation(T, x), md, mdv;
    corot_project(F, md, mdv);
    double E = S.E[t], nu = S.nu[t];
    double mu = E / (1.0 + nu);
    double wr = mu * T.vol, wv = wr * nu;
    /* dbar for the two 3x3 blocks: column j of md gets wr * sum_v G[v][j] yb_v */
    M3 Y{};
    for (int j = 0; j < 3; ++j) {
      V3 s{0, 0, 0};
      for (int v = 0; v < 4; ++v) s = s + T.G[v][j] * getx(yb, T.v[v]);
      setcol(Y, j, s);
    }
    /* parameter gradients: ybar . (dJ/dtheta) d */
    double yr = 0, yv = 0;
    for (int j = 0; j < 3; ++j) { yr += dot(col(Y, j), col(md, j)); yv += dot(col(Y, j), col(mdv, j)); }
    if (gE) gE[t] += (T.vol / (1.0 + nu)) * (yr + nu * yv);
    if (gnu) gnu[t] += (-E * T.vol / ((1.0 + nu) * (1.0 + nu))) * yr + (E * T.vol / ((1.0 + nu) * (1.0 + nu))) * yv;
    M3 gmd{}, gmdv{};
    for (int j = 0; j < 3; ++j) { setcol(gmd, j, wr * col(Y, j)); setcol(gmdv, j, wv * col(Y, j)); }
    M3 gF = corot_vjp(F, gmd, gmdv);
    for (int v = 0; v < 4; ++v) {
      V3 s{0, 0, 0};
      for (int j = 0; j < 3; ++j) s = s + T.G[v][j] * col(gF, j);
      addx(xb, T.v[v], s);
    }
  }
  for (size_t m = 0; m < S.mtets.size(); ++m) {
    const Tet& T = S.mtets[m];
    V3 fib = S.mfib[m];
    double w = T.vol * S.mk[m];
    double c[4];
    V3 db{0, 0, 0};
    for (int v = 0; v < 4; ++v) {
      c[v] = T.G[v][0] * fib.x + T.G[v][1] * fib.y + T.G[v][2] * fib.z;
      db = db + (w * c[v]) * getx(yb, T.v[v]);
    }
    M3 F = deformation(T, x);
    V3 Ff = fib.x * col(F, 0) + fib.y * col(F, 1) + fib.z * col(F, 2);
    double a = act[S.mseg[m]];
    if (gact) gact[S.mseg[m]] += -dot(db, Ff);
    /* d = (1-a) F f, F f = sum_v c_v x_v */
    for (int v = 0; v < 4; ++v) addx(xb, T.v[v], ((1.0 - a) * c[v]) * db);
  }
  for (size_t s = 0; s < S.sp_w.size(); ++s) {
    int i0 = S.sp_v[2 * s], i1 = S.sp_v[2 * s + 1];
    double w = std::sqrt(S.sp_w[s]);
    V3 db = w * (getx(yb, i0) - getx(yb, i1));
    V3 e = getx(x, i0) - getx(x, i1);
    double n = norm(e);
    V3 eh = (1.0 / n) * e;
    double len = S.sp_rest[s];
    if (S.sp_ch[s] >= 0) {
      len *= act[S.sp_ch[s]];
      if (gact) gact[S.sp_ch[s]] += S.sp_rest[s] * dot(db, eh);
    }
    V3 ge = (len / n) * (db - dot(eh, db) * eh);
    addx(xb, i0, ge);
    addx(xb, i1, -1.0 * ge);
  }
  for (const Bend& B : S.bends) {
    V3 db{0, 0, 0};
    for (size_t a = 0; a < B.v.size(); ++a) db = db + (B.w * B.beta[a]) * getx(yb, B.v[a]);
    V3 lap{0, 0, 0};
    for (size_t a = 0; a < B.v.size(); ++a) lap = lap + B.beta[a] * getx(x, B.v[a]);
    double ln = norm(lap);
    if (!(ln > 1e-25)) continue;
    V3 lh = (1.0 / ln) * lap;
    V3 gl = (B.w * B.rest_norm / ln) * (db - dot(lh, db) * lh);
    for (size_t a = 0; a < B.v.size(); ++a) addx(xb, B.v[a], B.beta[a] * gl);
  }
}

/* ybar . (dH/dE_t) x per tet, subtracted from gE (and dH/dnu = 0: the L block
 * of a tet is E * vol * G G^T). */
static void H_param_vjp(const Scene& S, const double* yb, const double* x, double* gE) {
  if (!gE) return;
  for (size_t t = 0; t < S.tets.size(); ++t) {
    const Tet& T = S.tets[t];
    double s = 0;
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        double gg = 0;
        for (int j = 0; j < 3; ++j) gg += T.G[a][j] * T.G[b][j];
        s += gg * dot(getx(yb, T.v[a]), getx(x, T.v[b]));
      }
    gE[t] -= T.vol * s;
  }
}

/* Reverse of the contact phase (test restatement).  xb: in, the cotangent of
 * the phase's output; out, the cotangent of its input (the PD result).  xtb,
 * vwcb accumulate the cotangents of x_t and v_wc; gE, gnu, gact those of the
 * parameters (J d at each iteration's input; Hs through C, L x_t and diag(Hs)).
 * Per computed iteration j (in reverse), with rhs_pre = M v_wc + h (J d(ori) -
 * L x_t) - h C (ori - x_t), rhs_post its contact projection, prev_j =
 * alpha rhs_post + (1 - alpha) prev_{j-1} (prev_{j-1} := rhs_pre at the first
 * iteration of a pass) and x_n1 = x_t + prev_j / (h diag(Hs)). */
/* Cotangent of f from the cotangent ob of the winning reaction
 * out = B c(r), r = -B^T f, c the friction-cone clamp (r1, r2) -> mu r0 (r1, r2) / |(r1, r2)|. */
static V3 reaction_vjp(const ObsWin& w, V3 f, V3 ob, double mu) {
  const double r0 = -dot(w.B[0], f), r1 = -dot(w.B[1], f), r2 = -dot(w.B[2], f);
  const double b0 = dot(w.B[0], ob), b1 = dot(w.B[1], ob), b2 = dot(w.B[2], ob);
  const double rt = std::sqrt(r1 * r1 + r2 * r2);
  double g0 = b0, g1 = b1, g2 = b2;
  if (rt > mu * r0) {
    g0 = b0 + mu * (r1 * b1 + r2 * b2) / rt;
    g1 = mu * r0 * (r2 * r2 * b1 - r1 * r2 * b2) / (rt * rt * rt);
    g2 = mu * r0 * (r1 * r1 * b2 - r1 * r2 * b1) / (rt * rt * rt);
  }
  return -1.0 * (g0 * w.B[0] + g1 * w.B[1] + g2 * w.B[2]);
}

/* VJP of collision_handling at one computed iteration (same inputs as the
 * forward call): rb holds the cotangent of the rhs after the call and leaves
 * with the cotangent before it (contact vertices; other entries pass through);
 * scb likewise for the self-force state; hdb receives the cotangents of the
 * masses diag(Hs). */
static void collision_handling_vjp(const Scene& S, int mode, const double* rhs_pre,
                                   const std::vector<std::vector<V3>>& normals, const std::vector<SelfGroup>& groups,
                                   const std::vector<double>& sc_in, const std::vector<double>& hd, double* rb,
                                   std::vector<double>& scb, double* hdb) {
  if (mode == 0) return;
  const int nc = (int)S.cverts.size();
  const double mu = S.mu_obs;
  const V3 zero{0, 0, 0};
  std::vector<V3> forces(nc), cnext(nc, zero), Fb(nc, zero), Cb(nc, zero);
  std::vector<ObsWin> win(nc);
  std::vector<V3> fobs(nc);
  std::vector<double> scb_in(3 * (size_t)nc, 0.0);
  for (int a = 0; a < nc; ++a) {
    forces[a] = getx(rhs_pre, S.cverts[a]);
    fobs[a] = S.self_collide ? forces[a] + getx(sc_in.data(), a) : forces[a];
    win[a] = obstacle_reaction(fobs[a], normals[a], mu);
    if (win[a].hit && S.self_collide) cnext[a] = reaction_world(win[a]);
  }
  if (mode == 1) {
    for (int a = 0; a < nc; ++a) {
      if (!win[a].hit) continue;
      const int gv = S.cverts[a];
      const V3 fb = reaction_vjp(win[a], fobs[a], getx(rb, gv), mu);
      rb[3 * gv] = fb.x; rb[3 * gv + 1] = fb.y; rb[3 * gv + 2] = fb.z;
      if (S.self_collide) { scb_in[3 * a] = fb.x; scb_in[3 * a + 1] = fb.y; scb_in[3 * a + 2] = fb.z; }
    }
    if (S.self_collide) scb = scb_in;
    return;
  }
  std::vector<V3> Sb(nc);
  for (int a = 0; a < nc; ++a) {
    const V3 r = getx(rb, S.cverts[a]);
    Sb[a] = r + getx(scb.data(), a);
    Cb[a] = r;
    Fb[a] = r;
  }
  for (const SelfGroup& g : groups) {
    V3 B[3];
    contact_basis(g.n, B);
    const int nv = (int)g.verts.size(), nin = 12 + 4 * nv;
    auto seed = [&](double v, int idx) { DN d(v); d.d.assign(nin, 0.0); d.d[idx] = 1.0; return d; };
    TV3<DN> P[3], oF[3];
    DN mf[3];
    for (int i = 0; i < 3; ++i) {
      const int a = S.cfaces[g.f][i];
      const V3 q = forces[a] + cnext[a];
      P[i] = {seed(q.x, 3 * i), seed(q.y, 3 * i + 1), seed(q.z, 3 * i + 2)};
      mf[i] = seed(hd[S.cverts[a]], 9 + i);
    }
    std::vector<TV3<DN>> PL, oL;
    std::vector<DN> mL;
    for (int k = 0; k < nv; ++k) {
      const int a = g.verts[k];
      const V3 q = forces[a] + cnext[a];
      PL.push_back({seed(q.x, 12 + 3 * k), seed(q.y, 12 + 3 * k + 1), seed(q.z, 12 + 3 * k + 2)});
      mL.push_back(seed(hd[S.cverts[a]], 12 + 3 * nv + k));
    }
    self_group_exchange(B, P, mf, PL, mL, S.mu_self, oF, oL, nullptr);
    std::vector<double> gin(nin, 0.0);
    auto acc = [&](const TV3<DN>& o, V3 cot) {
      const DN* c[3] = {&o.x, &o.y, &o.z};
      const double w[3] = {cot.x, cot.y, cot.z};
      for (int q = 0; q < 3; ++q)
        for (size_t k = 0; k < c[q]->d.size(); ++k) gin[k] += w[q] * c[q]->d[k];
    };
    for (int i = 0; i < 3; ++i) acc(oF[i], Sb[S.cfaces[g.f][i]]);
    for (int k = 0; k < nv; ++k) acc(oL[k], Sb[g.verts[k]]);
    for (int i = 0; i < 3; ++i) {
      const int a = S.cfaces[g.f][i];
      const V3 pb{gin[3 * i], gin[3 * i + 1], gin[3 * i + 2]};
      Fb[a] = Fb[a] + pb;
      Cb[a] = Cb[a] + pb;
      hdb[S.cverts[a]] += gin[9 + i];
    }
    for (int k = 0; k < nv; ++k) {
      const int a = g.verts[k];
      const V3 pb{gin[12 + 3 * k], gin[12 + 3 * k + 1], gin[12 + 3 * k + 2]};
      Fb[a] = Fb[a] + pb;
      Cb[a] = Cb[a] + pb;
      hdb[S.cverts[a]] += gin[12 + 3 * nv + k];
    }
  }
  for (int a = 0; a < nc; ++a) {
    if (win[a].hit) {
      const V3 fb = reaction_vjp(win[a], fobs[a], Cb[a], mu);
      Fb[a] = Fb[a] + fb;
      scb_in[3 * a] = fb.x; scb_in[3 * a + 1] = fb.y; scb_in[3 * a + 2] = fb.z;
    }
    const int gv = S.cverts[a];
    rb[3 * gv] = Fb[a].x; rb[3 * gv + 1] = Fb[a].y; rb[3 * gv + 2] = Fb[a].z;
  }
  scb = scb_in;
}

/* Adjoint of contact_phase.  xb: cotangent of the phase's output (in) and of
 * its input, the PD result (out); scb: cotangent of the self-force state at
 * the phase's end (in) and at its start (out).  Runs over every computed
 * iteration: one after the output's source still feeds the state. */
static void contact_adjoint(const Scene& S, const double* x_t, const double* vwc, const double* act,
                            const ContactTape& tp, double* xb, double* xtb, double* vwcb, double* gE, double* gnu,
                            double* gact, std::vector<double>& scb) {
  const int N = S.N, n3 = 3 * N;
  const int total = (int)tp.ori.size();
  if (total == 0) return;
  const double h = S.h, ih2 = 1.0 / (h * h), al = S.alpha;
  std::vector<double> xout(xb, xb + n3), xn1b(n3, 0.0), pb(n3, 0.0), hdb(N, 0.0), rpb(n3), yb(n3), orib(n3),
      rhs(n3), jd(n3), Lxt(n3), Hx(n3);
  H_mul(S, x_t, Hx.data());
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) Lxt[3 * i + c] = Hx[3 * i + c] - S.mass[i] * ih2 * x_t[3 * i + c];
  for (int j = total; j >= 1; --j) {
    if (j == tp.out_src)
      for (int k = 0; k < n3; ++k) xn1b[k] += xout[k];
    const std::vector<double>& ori = tp.ori[j - 1];
    const std::vector<double>& prev = tp.prev[j - 1];
    /* x_n1 = x_t + prev / (h hd) */
    for (int i = 0; i < N; ++i)
      for (int c = 0; c < 3; ++c) {
        const int k = 3 * i + c;
        xtb[k] += xn1b[k];
        hdb[i] -= xn1b[k] * prev[k] / (h * tp.hd[i] * tp.hd[i]);
        pb[k] += xn1b[k] / (h * tp.hd[i]);
      }
    /* rhs_pre at ori (recomputed) */
    std::fill(jd.begin(), jd.end(), 0.0);
    local_Jd(S, ori.data(), act, jd.data(), 1);
    for (int i = 0; i < N; ++i) {
      double cdx[3] = {0, 0, 0};
      for (auto& e : S.Hrows[i])
        if (e.first != i)
          for (int c = 0; c < 3; ++c) cdx[c] += e.second * (ori[3 * e.first + c] - x_t[3 * e.first + c]);
      for (int c = 0; c < 3; ++c)
        rhs[3 * i + c] = S.mass[i] * vwc[3 * i + c] + h * (jd[3 * i + c] - Lxt[3 * i + c]) - h * cdx[c];
    }
    /* prev_j = al rhs_post + (1 - al) prev_{j-1} */
    for (int k = 0; k < n3; ++k) rpb[k] = al * pb[k];
    static const std::vector<SelfGroup> kNoGroups;
    const int gp = tp.gpass[j - 1];
    collision_handling_vjp(S, tp.mode[j - 1], rhs.data(), tp.nrm[j - 1], gp >= 0 ? tp.groups[gp] : kNoGroups,
                           tp.sc_in[j - 1], tp.hd, rpb.data(), scb, hdb.data());
    if (tp.first[j - 1]) {
      for (int k = 0; k < n3; ++k) { rpb[k] += (1.0 - al) * pb[k]; pb[k] = 0.0; }
    } else {
      for (int k = 0; k < n3; ++k) pb[k] = (1.0 - al) * pb[k];
    }
    /* rhs_pre = M v_wc + h (J d(ori) - L x_t) - h C (ori - x_t) */
    for (int i = 0; i < N; ++i)
      for (int c = 0; c < 3; ++c) vwcb[3 * i + c] += S.mass[i] * rpb[3 * i + c];
    for (int k = 0; k < n3; ++k) yb[k] = h * rpb[k];
    std::fill(orib.begin(), orib.end(), 0.0);
    local_Jd_vjp(S, ori.data(), act, yb.data(), orib.data(), gE, gnu, gact);
    for (int i = 0; i < N; ++i)
      for (auto& e : S.Hrows[i]) {
        const int jj = e.first;
        for (int c = 0; c < 3; ++c) {
          if (jj != i) {
            orib[3 * jj + c] -= e.second * yb[3 * i + c];   /* -h C (ori - x_t) */
            xtb[3 * jj + c] += e.second * yb[3 * i + c];
          }
          xtb[3 * jj + c] -= e.second * yb[3 * i + c];     /* -h L x_t, L x_t = Hs x_t - M/h^2 x_t */
        }
      }
    for (int i = 0; i < N; ++i)
      for (int c = 0; c < 3; ++c) xtb[3 * i + c] += S.mass[i] * ih2 * yb[3 * i + c];
    /* Hs entries: d rhs_pre_i / d Hs_ij = -h ori_j (i != j), -h x_t_i (i == j) */
    if (gE)
      for (size_t t = 0; t < S.tets.size(); ++t) {
        const Tet& T = S.tets[t];
        double sacc = 0;
        for (int a2 = 0; a2 < 4; ++a2)
          for (int b2 = 0; b2 < 4; ++b2) {
            double gg = 0;
            for (int q = 0; q < 3; ++q) gg += T.G[a2][q] * T.G[b2][q];
            const double* xs = a2 == b2 ? x_t : ori.data();
            sacc += gg * dot(getx(yb.data(), T.v[a2]), getx(xs, T.v[b2]));
          }
        gE[t] -= T.vol * sacc;
      }
    xn1b = orib;  /* ori_x of iteration j is x_n1 of iteration j - 1 */
  }
  if (tp.out_src == 0)
    for (int k = 0; k < n3; ++k) xn1b[k] += xout[k];
  /* diag(Hs) entries */
  if (gE)
    for (size_t t = 0; t < S.tets.size(); ++t) {
      const Tet& T = S.tets[t];
      double sacc = 0;
      for (int a2 = 0; a2 < 4; ++a2) {
        double gg = 0;
        for (int q = 0; q < 3; ++q) gg += T.G[a2][q] * T.G[a2][q];
        sacc += gg * hdb[T.v[a2]];
      }
      gE[t] += T.vol * sacc;
    }
  std::copy(xn1b.begin(), xn1b.end(), xb);
}

}  // namespace orc

using namespace orc;

extern "C" {

void* orc_create(const dfem_scene_desc* d) {
  Scene* S = new Scene();
  int N = d->n_vertices;
  S->N = N;
  S->x0.assign(d->x0, d->x0 + 3 * N);
  S->mass.assign(d->mass, d->mass + N);
  S->gmask.assign(N, 1.0);
  if (d->gravity_mask)
    for (int i = 0; i < N; ++i) S->gmask[i] = d->gravity_mask[i] ? 1.0 : 0.0;
  for (int t = 0; t < d->n_tets; ++t) {
    S->tets.push_back(make_tet(d->x0, d->tets + 4 * t));
    S->E.push_back(d->youngs[t]);
    S->nu.push_back(d->poisson[t]);
  }
  for (int a = 0; a < d->n_attach; ++a) {
    S->att_v.push_back(d->attach_vertex[a]);
    S->att_p.push_back(V3{d->attach_target[3 * a], d->attach_target[3 * a + 1], d->attach_target[3 * a + 2]});
    S->att_k.push_back(d->attach_stiffness[a]);
  }
  S->nseg = d->n_segments;
  S->seg_act.assign(std::max(0, d->n_segments), 0.0);
  for (int m = 0; m < d->n_muscle; ++m) {
    S->mtets.push_back(make_tet(d->x0, d->muscle_tets + 4 * m));
    S->mfib.push_back(V3{d->muscle_fiber[3 * m], d->muscle_fiber[3 * m + 1], d->muscle_fiber[3 * m + 2]});
    S->mk.push_back(d->muscle_stiffness[m]);
    S->mseg.push_back(d->muscle_segment[m]);
  }
  for (int s = 0; s < d->n_springs; ++s) {
    int i0 = d->spring_vertices[2 * s], i1 = d->spring_vertices[2 * s + 1];
    S->sp_v.push_back(i0); S->sp_v.push_back(i1);
    double rest = d->spring_rest ? d->spring_rest[s] : norm(getx(d->x0, i0) - getx(d->x0, i1));
    S->sp_rest.push_back(rest);
    S->sp_w.push_back(d->spring_weight[s]);
    S->sp_ch.push_back(d->spring_channel ? d->spring_channel[s] : -1);
  }
  for (int b = 0; b < d->n_bending; ++b) {
    Bend B;
    int o0 = d->bend_offsets[b], o1 = d->bend_offsets[b + 1];
    for (int k = o0; k < o1; ++k) B.v.push_back(d->bend_vertices[k]);
    B.w = d->bend_weight[b];
    /* mean-value Laplace-Beltrami coefficients (BendingConstraint.h:220-260) */
    V3 mid = getx(d->x0, B.v[0]);
    int nr = (int)B.v.size() - 1;
    std::vector<double> coeff(nr);
    for (int i = 0; i < nr; ++i) {
      V3 vi = getx(d->x0, B.v[1 + i]);
      V3 cw = getx(d->x0, B.v[1 + (i + 1) % nr]);
      V3 ccw = getx(d->x0, B.v[1 + (i + nr - 1) % nr]);
      double dist = norm(vi - mid);
      coeff[i] = (mean_value(vi, mid, cw) + mean_value(vi, ccw, mid)) / dist;
    }
    B.beta.assign(nr + 1, 0.0);
    for (int i = 0; i < nr; ++i) { B.beta[0] += coeff[i]; B.beta[1 + i] = -coeff[i]; }
    /* BendingConstraint.h:83-95 evaluates applyA() on the rest state before
       m_beltrami_coefficients is filled, so the stored rest norm is always 0
       (the projection target d vanishes; only the w^3 beta beta^T term of L
       acts).  The oracle follows that. */
    B.rest_norm = 0.0;
    S->bends.push_back(B);
  }
  S->collide = d->handle_collision != 0;
  S->alpha = d->alpha;
  S->mu_obs = d->obstacle_friction;
  for (int k = 0; k < d->n_contact_vertices; ++k) S->cverts.push_back(d->contact_vertices[k]);
  for (int k = 0; k < d->n_obstacle_vertices; ++k)
    S->obs_x.push_back(V3{d->obstacle_x[3 * k], d->obstacle_x[3 * k + 1], d->obstacle_x[3 * k + 2]});
  for (int k = 0; k < d->n_obstacle_faces; ++k)
    S->obs_f.push_back({d->obstacle_faces[3 * k], d->obstacle_faces[3 * k + 1], d->obstacle_faces[3 * k + 2]});
  /* soft contact faces (global vertex ids) as contact-vertex ids */
  S->self_collide = S->collide && d->self_collision != 0;
  S->mu_self = d->friction;
  {
    std::vector<int> cid(N, -1);
    for (int a = 0; a < (int)S->cverts.size(); ++a) cid[S->cverts[a]] = a;
    S->on_face.assign(S->cverts.size(), 0);
    for (int k = 0; S->self_collide && k < d->n_contact_faces; ++k) {
      std::array<int, 3> f;
      for (int q = 0; q < 3; ++q) {
        const int gv = d->contact_faces[3 * k + q];
        f[q] = (gv >= 0 && gv < N) ? cid[gv] : -1;
        if (f[q] < 0) { S->err = "contact face vertex is not a contact vertex"; delete S; return nullptr; }
      }
      S->cfaces.push_back(f);
      for (int q = 0; q < 3; ++q) S->on_face[f[q]] = 1;
    }
    S->sc_cur.assign(3 * S->cverts.size(), 0.0);
  }
  S->underwater = d->underwater != 0;
  for (int k = 0; k < d->n_drag_faces; ++k)
    S->drag_f.push_back({d->drag_faces[3 * k], d->drag_faces[3 * k + 1], d->drag_faces[3 * k + 2]});
  S->h = d->time_step;
  S->K = d->max_iterations;
  S->damping = d->damping;
  S->g = V3{d->gravity[0], d->gravity[1], d->gravity[2]};
  if (d->n_links > 0) {  /* Dfobj.h:254-288, World::AddBody (World.h:499-545) */
    Skel& K = S->skel;
    K.L = d->n_links;
    K.ridx.assign(N, -1);
    int dof = 0, sdof = 0;
    for (int l = 0; l < K.L; ++l) {
      LinkO k;
      k.parent = d->link_parent[l];
      k.type = d->link_type[l];
      k.chan = d->link_channel ? d->link_channel[l] : -1;
      k.joint = V3{d->link_joint[3 * l], d->link_joint[3 * l + 1], d->link_joint[3 * l + 2]};
      k.dof = dof; k.sdof = sdof;
      dof += (k.parent < 0) ? 6 : 1;
      sdof += (k.parent < 0) ? 12 : 1;
      if (k.parent >= 0) {
        V3 a{d->link_axis[3 * l], d->link_axis[3 * l + 1], d->link_axis[3 * l + 2]};
        k.axis = (1.0 / norm(a)) * a;
        k.d0 = k.joint - K.links[k.parent].joint;
        if (k.type == DFEM_JOINT_ROTATIONAL) {
          at(k.nx, 0, 1) = -k.axis.z; at(k.nx, 0, 2) = k.axis.y;
          at(k.nx, 1, 0) = k.axis.z;  at(k.nx, 1, 2) = -k.axis.x;
          at(k.nx, 2, 0) = -k.axis.y; at(k.nx, 2, 1) = k.axis.x;
          const double ax[3] = {k.axis.x, k.axis.y, k.axis.z};
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) at(k.nnt, r, c) = ax[r] * ax[c];
        }
      } else {
        k.d0 = k.joint;
      }
      k.r0 = (int)K.rv.size();
      for (int q = d->link_offsets[l]; q < d->link_offsets[l + 1]; ++q) {
        const int v = d->link_vertices[q];
        K.ridx[v] = (int)K.rv.size();
        K.rv.push_back(v);
        K.rest.push_back(getx(d->x0, v));
      }
      k.r1 = (int)K.rv.size();
      K.links.push_back(k);
    }
    K.ndof = dof;
    K.nq = sdof;
    K.jq.assign(sdof, 0.0);
    K.jqd.assign(sdof, 0.0);
    skel_write(K);  /* World::Initialize writes the fresh links (World.h:369-370) */
  }
  assemble_H(*S);
  rcm_order(*S);
  if (!factor(*S)) { delete S; return nullptr; }
  if (S->skel.L > 0 && !skel_precompute(*S)) { delete S; return nullptr; }
  return S;
}

int orc_joint_state_size(void* s) { return static_cast<Scene*>(s)->skel.nq; }

int orc_set_joint_state(void* s, const double* jq, const double* jqd) {
  Skel& K = static_cast<Scene*>(s)->skel;
  std::copy(jq, jq + K.nq, K.jq.begin());
  std::copy(jqd, jqd + K.nq, K.jqd.begin());
  return 0;
}

int orc_get_joint_state(void* s, double* jq, double* jqd) {
  const Skel& K = static_cast<Scene*>(s)->skel;
  std::copy(K.jq.begin(), K.jq.end(), jq);
  std::copy(K.jqd.begin(), K.jqd.end(), jqd);
  return 0;
}

void orc_destroy(void* s) { delete static_cast<Scene*>(s); }

double orc_regularisation(void* s) { return static_cast<Scene*>(s)->reg; }

int orc_set_materials(void* s, const double* E, const double* nu) {
  Scene* S = static_cast<Scene*>(s);
  for (size_t t = 0; t < S->tets.size(); ++t) { S->E[t] = E[t]; S->nu[t] = nu[t]; }
  assemble_H(*S);
  rcm_order(*S);
  if (!factor(*S)) return 3;
  return (S->skel.L > 0 && !skel_precompute(*S)) ? 3 : 0;
}

/* Forward: n_steps steps from (x, v); act = n_steps * n_segments (may be NULL);
 * traj = n_steps * 3N positions (may be NULL); iters = n_steps (may be NULL). */
int orc_forward(void* s, const double* x, const double* v, const double* act, int n_steps,
                double* x_out, double* v_out, double* traj, int* iters, int nthreads) {
  Scene* S = static_cast<Scene*>(s);
  int n3 = 3 * S->N;
  std::vector<double> xc(x, x + n3), vc(v, v + n3), vwc(n3), qn(n3), xn(n3);
  S->rec_steps = n_steps;
  S->rec_x.assign((size_t)n_steps * n3, 0.0);
  S->rec_v.assign((size_t)n_steps * n3, 0.0);
  S->rec_act.assign((size_t)n_steps * std::max(1, S->nseg), 0.0);
  S->rec_iters.assign(n_steps, 0);
  S->rec_passes.assign(n_steps, 0);
  if (S->freeze == 1) S->frz.assign(n_steps, {});
  /* without activations: muscle segments 0, pneumatic channels 1 (pneumaticEasy.h:31) */
  std::vector<double> zero_act(std::max(1, S->nseg), 0.0);
  for (int c : S->sp_ch)
    if (c >= 0) zero_act[c] = 1.0;
  for (int st = 0; st < n_steps; ++st) {
    const double* a = act ? act + (size_t)st * S->nseg : zero_act.data();
    /* every step starts with no remembered contact forces: World::TimeStepping
     * calls updateCollisionScene before the PD solve (World.h:700), which zeroes
     * the self-collision force buffers (World.h:742-753) */
    std::fill(S->sc_cur.begin(), S->sc_cur.end(), 0.0);
    S->cur_step = st;
    std::copy(xc.begin(), xc.end(), S->rec_x.begin() + (size_t)st * n3);
    std::copy(vc.begin(), vc.end(), S->rec_v.begin() + (size_t)st * n3);
    if (S->nseg > 0) std::copy(a, a + S->nseg, S->rec_act.begin() + (size_t)st * S->nseg);
    step_prep(*S, xc.data(), vc.data(), vwc.data(), qn.data());
    int it = S->skel.L > 0 ? pd_solve_skel(*S, xc.data(), qn.data(), a, xn.data(), nthreads)
                           : pd_solve(*S, xc.data(), qn.data(), a, nullptr, xn.data(), nthreads);
    contact_phase(*S, xc.data(), vwc.data(), a, xn.data());
    S->rec_passes[st] = S->last_passes;
    S->rec_iters[st] = it;
    if (iters) iters[st] = it;
    for (int k = 0; k < n3; ++k) {
      vc[k] = (xn[k] - xc[k]) * (1.0 / S->h) * S->damping;  /* World.h:708,757-766 */
      xc[k] = xn[k];
    }
    if (traj) std::copy(xc.begin(), xc.end(), traj + (size_t)st * n3);
    for (int k = 0; k < n3; ++k)
      if (!std::isfinite(xc[k])) { S->err = "non-finite state"; return 4; }
  }
  std::copy(xc.begin(), xc.end(), x_out);
  std::copy(vc.begin(), vc.end(), v_out);
  return 0;
}

/* Adjoint of the last orc_forward (recomputes each step's iterates). */
int orc_backward(void* s, const double* gx_out, const double* gv_out, double* gx, double* gv,
                 double* gE, double* gnu, double* gact) {
  Scene* S = static_cast<Scene*>(s);
  if (S->rec_steps <= 0) return 5;
  if (S->skel.L > 0) { S->err = "no adjoint for skeleton scenes"; return 8; }
  int N = S->N, n3 = 3 * N;
  int NT = (int)S->tets.size();
  std::vector<double> xb(gx_out, gx_out + n3), vb(gv_out, gv_out + n3);
  if (gE) std::fill(gE, gE + NT, 0.0);
  if (gnu) std::fill(gnu, gnu + NT, 0.0);
  if (gact) std::fill(gact, gact + (size_t)S->rec_steps * S->nseg, 0.0);
  std::vector<double> vwc(n3), qn(n3), xn(n3), hist, ybar(n3), xkb(n3), bb(n3), tmp(n3);
  double ih2 = 1.0 / (S->h * S->h);
  const size_t nsc = S->sc_cur.size();
  std::vector<double> scb(nsc, 0.0);  /* cotangent of the self-force state within a step */
  for (int st = S->rec_steps - 1; st >= 0; --st) {
    const double* x = &S->rec_x[(size_t)st * n3];
    const double* v = &S->rec_v[(size_t)st * n3];
    const double* a = &S->rec_act[(size_t)st * std::max(1, S->nseg)];
    step_prep(*S, x, v, vwc.data(), qn.data());
    int it = pd_solve(*S, x, qn.data(), a, &hist, xn.data(), 1);
    ContactTape tape;
    /* the step's contact phase starts from zero remembered forces (World.h:742-753)
     * and its final ones are zeroed before anything reads them: no cotangent
     * crosses the step boundary */
    std::fill(S->sc_cur.begin(), S->sc_cur.end(), 0.0);
    std::fill(scb.begin(), scb.end(), 0.0);
    S->cur_step = st;
    const int freeze0 = S->freeze;
    if (freeze0 == 1) S->freeze = 2;  /* re-runs replay what the forward recorded */
    contact_phase(*S, x, vwc.data(), a, xn.data(), &tape);
    S->freeze = freeze0;
    /* v' = damping (x' - x)/h; x' = contact phase output (x^it without contacts) */
    double c = S->damping / S->h;
    std::vector<double> xtb(n3), vwcb(n3, 0.0);
    for (int k = 0; k < n3; ++k) { xkb[k] = xb[k] + c * vb[k]; xtb[k] = -c * vb[k]; }
    contact_adjoint(*S, x, vwc.data(), a, tape, xkb.data(), xtb.data(), vwcb.data(), gE, gnu,
                    gact ? gact + (size_t)st * S->nseg : nullptr, scb);
    std::fill(bb.begin(), bb.end(), 0.0);
    for (int k = it - 1; k >= 0; --k) {
      const double* xk = &hist[(size_t)k * n3];
      const double* xk1 = &hist[(size_t)(k + 1) * n3];
      solve(*S, xkb.data(), ybar.data());          /* H symmetric */
      for (int q = 0; q < n3; ++q) bb[q] += ybar[q];
      std::fill(tmp.begin(), tmp.end(), 0.0);
      local_Jd_vjp(*S, xk, a, ybar.data(), tmp.data(), gE, gnu, gact ? gact + (size_t)st * S->nseg : nullptr);
      H_param_vjp(*S, ybar.data(), xk1, gE);
      xkb = tmp;
    }
    /* x^0 = q_n and b = M/h^2 q_n */
    std::vector<double> qnb(n3);
    for (int i = 0; i < N; ++i)
      for (int cc = 0; cc < 3; ++cc) qnb[3 * i + cc] = xkb[3 * i + cc] + S->mass[i] * ih2 * bb[3 * i + cc];
    /* q_n = x + h v_wc, v_wc = v + g h mask + h M^-1 f_ext(x, v) */
    for (int k = 0; k < n3; ++k) {
      xb[k] = xtb[k] + qnb[k];
      vb[k] = S->h * qnb[k] + vwcb[k];
    }
    if (!S->drag_f.empty()) {
      std::vector<double> fb(n3), vwct(vb);  /* vb holds the cotangent of v_wc here */
      for (int i = 0; i < N; ++i)
        for (int cc = 0; cc < 3; ++cc) fb[3 * i + cc] = S->h / S->mass[i] * vwct[3 * i + cc];
      drag_forces_vjp(*S, x, v, fb.data(), xb.data(), vb.data());
    }
  }
  std::copy(xb.begin(), xb.end(), gx);
  std::copy(vb.begin(), vb.end(), gv);
  return 0;
}

/* J d(x) of all constraints (World::EvaluateDVector + mJ * d, World.h:898-901);
 * act = per-segment activations (may be NULL = all zero). */
/* contact passes of each step of the last forward call */
/* One face group's exchange (self_group_exchange) for tests: normal n (3),
 * P = forces + reactions of the face's 3 vertices then of the n_list group
 * vertices (3 each), masses m (3 + n_list); out receives the self forces of
 * the same vertices (3 each), incl the membership of the group vertices. */
int orc_self_group(const double* n, const double* P, const double* m, int n_list, double mu, double* out, int* incl) {
  V3 B[3];
  contact_basis(V3{n[0], n[1], n[2]}, B);
  TV3<double> Pf[3], oF[3];
  double mf[3];
  for (int i = 0; i < 3; ++i) { Pf[i] = {P[3 * i], P[3 * i + 1], P[3 * i + 2]}; mf[i] = m[i]; }
  std::vector<TV3<double>> PL, oL;
  std::vector<double> mL;
  for (int k = 0; k < n_list; ++k) {
    PL.push_back({P[9 + 3 * k], P[9 + 3 * k + 1], P[9 + 3 * k + 2]});
    mL.push_back(m[3 + k]);
  }
  std::vector<char> inc;
  self_group_exchange(B, Pf, mf, PL, mL, mu, oF, oL, &inc);
  for (int i = 0; i < 3; ++i) { out[3 * i] = oF[i].x; out[3 * i + 1] = oF[i].y; out[3 * i + 2] = oF[i].z; }
  for (int k = 0; k < n_list; ++k) {
    out[9 + 3 * k] = oL[k].x; out[9 + 3 * k + 1] = oL[k].y; out[9 + 3 * k + 2] = oL[k].z;
    incl[k] = inc[k];
  }
  return 0;
}

/* detection replay mode for derivative tests (0 off, 1 record, 2 replay) */
void orc_set_detection_replay(void* s, int mode) { static_cast<Scene*>(s)->freeze = mode; }

int orc_contact_passes(void* s, int* out, int n) {
  Scene* S = static_cast<Scene*>(s);
  for (int k = 0; k < n && k < (int)S->rec_passes.size(); ++k) out[k] = S->rec_passes[k];
  return 0;
}

/* one vertex-face CCD test (vertex p0 -> p1 against the static face q0 q1 q2) */
int orc_vf_impact(const double* p0, const double* p1, const double* q0, const double* q1, const double* q2,
                  double mult, double* n_out) {
  V3 n{0, 0, 0};
  bool hit = vf_impact(getx(p0, 0), getx(p1, 0), getx(q0, 0), getx(q1, 0), getx(q2, 0), mult, &n);
  n_out[0] = n.x; n_out[1] = n.y; n_out[2] = n.z;
  return hit ? 1 : 0;
}

int orc_eval_local(void* s, const double* x, const double* act, double* out) {
  Scene* S = static_cast<Scene*>(s);
  std::vector<double> zero_act(std::max(1, S->nseg), 0.0);
  std::fill(out, out + 3 * (size_t)S->N, 0.0);
  local_Jd(*S, x, act ? act : zero_act.data(), out, 1);
  return 0;
}

/* Lumped masses of a tet mesh: Dfobj.h:506-525 (Is Mass Same = true: mass per
 * vertex = total / totvol * sum 0.25 vol; false: total / N). */
int orc_lumped_masses(int N, const double* x0, int T, const int* tets, double total_mass,
                      int is_mass_same, double* mass) {
  std::fill(mass, mass + N, 0.0);
  double totvol = 0;
  for (int t = 0; t < T; ++t) {
    Tet tt = make_tet(x0, tets + 4 * t);
    totvol += tt.vol;
    for (int k = 0; k < 4; ++k) mass[tets[4 * t + k]] += 0.25 * tt.vol;
  }
  for (int i = 0; i < N; ++i) mass[i] = is_mass_same ? total_mass / totvol * mass[i] : total_mass / N;
  return 0;
}

/* Corotated projection of one F (column-major 9): md, md_volume (column-major). */
void orc_corot_project(const double* F9, double* md9, double* mdv9) {
  M3 F; std::memcpy(F.m, F9, sizeof(F.m));
  M3 md, mdv;
  corot_project(F, md, mdv);
  std::memcpy(md9, md.m, sizeof(md.m));
  std::memcpy(mdv9, mdv.m, sizeof(mdv.m));
}

void orc_corot_vjp(const double* F9, const double* gmd9, const double* gmdv9, double* gF9) {
  M3 F, a, b; std::memcpy(F.m, F9, 72); std::memcpy(a.m, gmd9, 72); std::memcpy(b.m, gmdv9, 72);
  M3 g = corot_vjp(F, a, b);
  std::memcpy(gF9, g.m, 72);
}

/* SVD of one F: U, V column-major, s descending */
void orc_svd3(const double* F9, double* U9, double* s3, double* V9) {
  M3 F; std::memcpy(F.m, F9, 72);
  SVD3 s = svd3(F);
  std::memcpy(U9, s.U.m, 72); std::memcpy(V9, s.V.m, 72);
  for (int i = 0; i < 3; ++i) s3[i] = s.s[i];
}

/* Hs as COO (row, col, value), merged; returns nnz, fills up to cap. */
int64_t orc_hs_coo(void* s, int* rows, int* cols, double* vals, int64_t cap) {
  Scene* S = static_cast<Scene*>(s);
  int64_t k = 0;
  for (int i = 0; i < S->N; ++i)
    for (auto& e : S->Hrows[i]) {
      if (k < cap) { rows[k] = i; cols[k] = e.first; vals[k] = e.second; }
      ++k;
    }
  return k;
}

/* The reference's 3N x 3N L triplets from per-constraint A_i (EvaluateLMatrix of
 * the corotated, attachment, muscle and spring constraints), unmerged. */
int64_t orc_full_L_triplets(void* s, int* rows, int* cols, double* vals, int64_t cap) {
  Scene* S = static_cast<Scene*>(s);
  int64_t k = 0;
  auto push = [&](int r, int c, double v) { if (k < cap) { rows[k] = r; cols[k] = c; vals[k] = v; } ++k; };
  for (size_t t = 0; t < S->tets.size(); ++t) {
    const Tet& T = S->tets[t];
    /* A_i rows 3j+c, columns 3v+c': delta_{cc'} G[v][j] (CorotateFEMConstraint.h:236-245) */
    double A[9][12] = {{0}};
    for (int j = 0; j < 3; ++j)
      for (int c = 0; c < 3; ++c)
        for (int v = 0; v < 4; ++v) A[3 * j + c][3 * v + c] = T.G[v][j];
    double mu = S->E[t] / (1.0 + S->nu[t]);
    for (int blk = 0; blk < 2; ++blk) {
      double w = mu * T.vol * (blk ? S->nu[t] : 1.0);
      for (int a = 0; a < 12; ++a)
        for (int b = 0; b < 12; ++b) {
          double sum = 0;
          for (int r = 0; r < 9; ++r) sum += A[r][a] * A[r][b];
          push(3 * T.v[a / 3] + a % 3, 3 * T.v[b / 3] + b % 3, w * sum);
        }
    }
  }
  for (size_t a = 0; a < S->att_v.size(); ++a)
    for (int c = 0; c < 3; ++c) push(3 * S->att_v[a] + c, 3 * S->att_v[a] + c, S->att_k[a]);
  for (size_t m = 0; m < S->mtets.size(); ++m) {
    const Tet& T = S->mtets[m];
    V3 fib = S->mfib[m];
    double A[3][12] = {{0}};
    for (int v = 0; v < 4; ++v) {
      double c = T.G[v][0] * fib.x + T.G[v][1] * fib.y + T.G[v][2] * fib.z;
      for (int cc = 0; cc < 3; ++cc) A[cc][3 * v + cc] = c;
    }
    double w = T.vol * S->mk[m];
    for (int a = 0; a < 12; ++a)
      for (int b = 0; b < 12; ++b) {
        double sum = 0;
        for (int r = 0; r < 3; ++r) sum += A[r][a] * A[r][b];
        push(3 * T.v[a / 3] + a % 3, 3 * T.v[b / 3] + b % 3, w * sum);
      }
  }
  for (size_t sp = 0; sp < S->sp_w.size(); ++sp) {
    double w = std::sqrt(S->sp_w[sp]);
    int iv[2] = {S->sp_v[2 * sp], S->sp_v[2 * sp + 1]};
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 3; ++c) push(3 * iv[a] + c, 3 * iv[b] + c, w * (a == b ? 1.0 : -1.0));
  }
  return k;
}

const char* orc_last_error(void* s) { return static_cast<Scene*>(s)->err.c_str(); }

}  // extern "C"
