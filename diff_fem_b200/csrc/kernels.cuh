// kernels.cuh — device-side data views and kernels of the PD step and its adjoint.
//
// Data layout in HBM (all arrays of one scene, internal vertex numbering):
//   positions / velocities / rhs : interleaved FP64 [x y z] per vertex (3N)
//   tets  : int4 vertex ids, invDm as 9 SoA planes (plane k holds invDm[k/3][k%3]),
//           weights w_r = mu*vol and w_v = nu*mu*vol, int4 slot positions
//   slots : one [x y z] FP64 contribution per (constraint, vertex) pair, sorted
//           by vertex, so the rhs gather reads one contiguous range per vertex
//   factor: supernodes (first column, width, rows below), row-wise CSR of the
//           below-diagonal entries (forward solve), column-major below-diagonal
//           blocks + row ids (backward solve), inverses of the diagonal blocks.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "pd_math.cuh"
#include "tma.cuh"

namespace dfem {

constexpr double kConvergenceEps = 5e-7;  // World.h:214 (EPS)

// Kernels of a PD iteration are gated on device state so a whole step runs as
// one CUDA graph with no host round trip: forward kernels return early once
// the convergence flag is set; adjoint kernels of reverse iteration k return
// when k >= the iteration count recorded for the step.
struct Gate {
  const int* flag;   // forward: nonzero -> converged, skip
  const int* iters;  // adjoint: per-step iteration counts
  const int* step;   // adjoint: current step index
  int k;
  const int* active = nullptr;  // contact phase: run only while *active == 1
  __device__ __forceinline__ bool skip() const {
    if (flag && *flag) return true;
    if (iters && k >= iters[*step]) return true;
    if (active && *active != 1) return true;
    return false;
  }
};

struct SceneDev {
  int N, T, M, S, B, nseg;
  double h, damping, g0, g1, g2;
  const double* mass;
  const double* gmask;
  // tets
  const int4* tv;
  const double* tinv;   // 9 planes of T
  const double* twr;    // mu * vol
  const double* twv;    // nu * mu * vol
  const double* tvol;
  const double* tE;
  const double* tnu;
  const int4* tslot;
  // muscles
  const int4* mv;
  const double* minv;   // 9 planes of M
  const double* mw;     // vol * stiffness
  const double* mfib;   // 3 planes of M
  const int* mseg;
  const int4* mslot;
  const int* seg_ptr;
  const int* seg_mus;
  // springs
  const int2* sv;
  const double* srest;
  const double* ssw;
  const int2* sslot;
  // bending
  const int* boff;
  const int* bv;
  const double* bbeta;
  const double* bw;
  const double* brest;
  const int* bslot;
  // slots
  const int* vslot_ptr;
  // attachment constant J*d (3N)
  const double* attach_jd;
  // Hs CSR
  const int* hs_ptr;
  const int* hs_col;
  const double* hs_val;
  // mixed form: FP32 copies of the tet tables (null in the plain form)
  const float* tinv32;
  const float* twr32;
  const float* twv32;
};

// Contact phase state (World::ProjectiveDynamicsMethod, sim/fem/World.h:925-1023).
constexpr int kMaxImpactsPerVertex = 4;
constexpr int kMaxContactPasses = 64;       // the reference's detection loop has no cap
constexpr double kContactThickness = 1e-4;  // arcsim Impact::thickness
struct ContactDev {
  int nc, nof, K, max_passes;
  double alpha, mu;
  const int* cverts;      // contact vertices (internal ids)
  const int* cidx;        // N: contact index or -1
  const double* obs_x;    // 3 per obstacle vertex
  const int* obs_f;       // 3 per obstacle face
  const double* hdiag;    // N: diagonal of Hs
  int* imp_cnt;           // nc
  int* imp_face;          // nc * kMax
  double* imp_n;          // nc * kMax * 3
  double* xn1;            // 3N: x_n1 of the reference's contact loop
  double* xold;           // 3N
  double* prev;           // 3N: relaxed rhs
  double* lxt;            // 3N: L x_t
  double* vwc;            // 3N: v + g h of the step
  int* state;             // [mode, pass, it, any, active]
};

struct FactorDev {
  const int* rseg_ptr;   // row -> its contribution slots (push-form forward solve)
  const int* rseg_pos;
  double* contrib;       // 3 doubles per below-diagonal row of every supernode
  const int* sn_c0;
  const int* sn_w;
  const int* sn_r;
  const int* sn_rofs;
  const int* rowidx;
  const int* sn_lofs;
  const double* Lcm;
  const int* sn_dofs;
  const double* Dinv;
  const int* lvl_sn;
  int stage_l;   // 1: the below-diagonal blocks are staged in shared memory too
  int* status;   // error status word (6: a bounded wait gave up)
};

}  // namespace dfem
