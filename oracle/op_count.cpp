// op_count.cpp — floating-point operation counts of one corotated tet in the
// local step (F_tet) and in the adjoint local step (F_tet_adj).
//
// Measurement infrastructure (not linked by the engine, not a checker): the
// engine's element math (diff_fem_b200/csrc/pd_math.cuh: svd3 by one-sided
// Jacobi, corot_project with the reference's reflection rule and 5 Newton
// steps of the volume projection, corot_vjp) is templated on its scalar type;
// here it is instantiated on a counting scalar, host-compiled, together with
// restatements of the tet branches of k_local and adj_local_item
// (pd_kernels.cu) around it.  The algorithm is the reference's corotated
// projection (CorotateFEMConstraint.h:187-205,354-377); the SVD method is the
// build's (one-sided Jacobi on the columns of F, which the oracle restates too).
// Counted: add/sub, mul, div, sqrt/rsqrt, comparisons; a fused multiply-add
// counts as one mul and one add.  The count depends on F through the number
// of Jacobi sweeps; its caller (op_count.py) averages it over a scene's tets.
#include <cmath>
#include <cstdint>

#define __device__
#define __host__
#define __forceinline__ inline
static inline double rsqrt(double v) { return 1.0 / std::sqrt(v); }  // device intrinsics, host stand-ins
static inline float rsqrtf(float v) { return 1.0f / std::sqrt(v); }
#include "../diff_fem_b200/csrc/pd_math.cuh"

namespace {

struct Ops { long long add = 0, mul = 0, div = 0, sqrt = 0, cmp = 0; };
Ops g;

struct Cnt {
  double v;
  Cnt() : v(0.0) {}
  Cnt(double x) : v(x) {}  // NOLINT: literals and doubles convert implicitly, as the math expects
};
inline Cnt operator+(Cnt a, Cnt b) { ++g.add; return a.v + b.v; }
inline Cnt operator-(Cnt a, Cnt b) { ++g.add; return a.v - b.v; }
inline Cnt operator-(Cnt a) { return -a.v; }  // a sign flip, not an operation
inline Cnt operator*(Cnt a, Cnt b) { ++g.mul; return a.v * b.v; }
inline Cnt operator/(Cnt a, Cnt b) { ++g.div; return a.v / b.v; }
inline Cnt& operator+=(Cnt& a, Cnt b) { a = a + b; return a; }
inline bool operator<(Cnt a, Cnt b) { ++g.cmp; return a.v < b.v; }
inline bool operator>(Cnt a, Cnt b) { ++g.cmp; return a.v > b.v; }
inline bool operator<=(Cnt a, Cnt b) { ++g.cmp; return a.v <= b.v; }
inline bool operator>=(Cnt a, Cnt b) { ++g.cmp; return a.v >= b.v; }

}  // namespace

namespace dfem {
template <> inline Cnt dsqrt<Cnt>(Cnt v) { ++g.sqrt; return std::sqrt(v.v); }
template <> inline Cnt drsqrt<Cnt>(Cnt v) { ++g.sqrt; return 1.0 / std::sqrt(v.v); }
template <> struct Eps<Cnt> { static constexpr double rot = Eps<double>::rot, rel = Eps<double>::rel;
                              static constexpr int sweeps = Eps<double>::sweeps; };
}  // namespace dfem

using dfem::Mat3;
using dfem::Vec3;

namespace {

// F(:,j) = sum_v G[v][j] x_v  (pd_kernels.cu: load_g, deformation)
Mat3<Cnt> deformation(const Cnt G[4][3], const Vec3<Cnt> xv[4]) {
  Mat3<Cnt> F;
  for (int j = 0; j < 3; ++j) F.c[j] = G[0][j] * xv[0] + G[1][j] * xv[1] + G[2][j] * xv[2] + G[3][j] * xv[3];
  return F;
}

// The tet branch of k_local: F, the projection, P = w_r md + w_v md_volume,
// the four vertex slots G[a] . P.
void tet_forward(const Cnt G[4][3], const Vec3<Cnt> xv[4], Cnt wr, Cnt wv) {
  Mat3<Cnt> F = deformation(G, xv), md, mdv;
  dfem::corot_project(F, md, mdv);
  Vec3<Cnt> P[3];
  for (int j = 0; j < 3; ++j) P[j] = wr * md.c[j] + wv * mdv.c[j];
  for (int a = 0; a < 4; ++a) {
    volatile double sink = (G[a][0] * P[0] + G[a][1] * P[1] + G[a][2] * P[2]).x.v;
    (void)sink;
  }
}

// The tet branch of adj_local_item with the next iterate x1 given: F, Y (the
// cotangent's deformation), the projection, the parameter terms of dL/dE and
// dL/dnu, the projection's VJP and the four vertex slots.
void tet_adjoint(const Cnt G[4][3], const Vec3<Cnt> xv[4], const Vec3<Cnt> yv[4], const Vec3<Cnt> x1v[4], Cnt E, Cnt nu,
                 Cnt vol, Cnt wr, Cnt wv) {
  Mat3<Cnt> F = deformation(G, xv), Y = deformation(G, yv), md, mdv;
  const dfem::Svd3<Cnt> sv = dfem::svd3(F);  // one SVD for the projection and its VJP
  dfem::corot_project_sv(sv, F, md, mdv);
  Cnt yr = 0.0, yvv = 0.0, yh = 0.0;
  for (int j = 0; j < 3; ++j) { yr += dfem::dot3(Y.c[j], md.c[j]); yvv += dfem::dot3(Y.c[j], mdv.c[j]); }
  Mat3<Cnt> F1 = deformation(G, x1v);
  for (int j = 0; j < 3; ++j) yh += dfem::dot3(Y.c[j], F1.c[j]);
  Cnt opn = Cnt(1.0) + nu;
  volatile double s0 = (vol / opn * (yr + nu * yvv) - vol * yh).v;
  volatile double s1 = (E * vol / (opn * opn) * (yvv - yr)).v;
  (void)s0; (void)s1;
  Mat3<Cnt> gmd, gmdv;
  for (int j = 0; j < 3; ++j) { gmd.c[j] = wr * Y.c[j]; gmdv.c[j] = wv * Y.c[j]; }
  Mat3<Cnt> gF = dfem::corot_vjp_sv(sv, F, gmd, gmdv);
  for (int a = 0; a < 4; ++a) {
    volatile double sink = (G[a][0] * gF.c[0] + G[a][1] * gF.c[1] + G[a][2] * gF.c[2]).x.v;
    (void)sink;
  }
}

void load(const double* p, Cnt G[4][3]) {  // invDm row-major (9) -> G (pd_kernels.cu: load_g)
  for (int j = 0; j < 3; ++j) {
    Cnt a = p[0 * 3 + j], b = p[1 * 3 + j], c = p[2 * 3 + j];
    G[1][j] = a; G[2][j] = b; G[3][j] = c;
    G[0][j] = -(a + b + c);
  }
}

}  // namespace

extern "C" {

/* Sums over n tets of the operation counts of the forward element (out[0..4])
 * and of the adjoint element (out[5..9]): add, mul, div, sqrt, cmp.  inv_dm:
 * 9 per tet (row-major); x, y, x1: 12 per tet (the four vertices' positions,
 * cotangents and next iterate); w: 5 per tet (E, nu, vol, w_r, w_v). */
int orc_count_tet_ops(int n, const double* inv_dm, const double* x, const double* y, const double* x1, const double* w,
                      long long* out) {
  for (int k = 0; k < 10; ++k) out[k] = 0;
  for (int t = 0; t < n; ++t) {
    Cnt G[4][3];
    Vec3<Cnt> xv[4], yv[4], x1v[4];
    for (int a = 0; a < 4; ++a) {
      const double* p = x + 12 * (size_t)t + 3 * a;
      const double* q = y + 12 * (size_t)t + 3 * a;
      const double* r = x1 + 12 * (size_t)t + 3 * a;
      xv[a] = {p[0], p[1], p[2]};
      yv[a] = {q[0], q[1], q[2]};
      x1v[a] = {r[0], r[1], r[2]};
    }
    const double* c = w + 5 * (size_t)t;
    g = Ops();
    load(inv_dm + 9 * (size_t)t, G);  // each kernel forms G from the invDm planes per element
    tet_forward(G, xv, c[3], c[4]);
    out[0] += g.add; out[1] += g.mul; out[2] += g.div; out[3] += g.sqrt; out[4] += g.cmp;
    g = Ops();
    load(inv_dm + 9 * (size_t)t, G);
    tet_adjoint(G, xv, yv, x1v, c[0], c[1], c[2], c[3], c[4]);
    out[5] += g.add; out[6] += g.mul; out[7] += g.div; out[8] += g.sqrt; out[9] += g.cmp;
  }
  return 0;
}

}  // extern "C"
