// cholesky.h — host-side analysis and numeric factorisation of the scalar PD
// system matrix Hs (N x N, SPD), laid out for the GPU supernodal solves.
//
// diff_fem factors the 3N x 3N H = M/h^2 + L with Eigen::SimplicialLDLT
// (sim/fem/World.h:1097-1125, 1212-1232).  Every constraint's selection matrix
// is kron(coeffs, I3), so H = kron(Hs, I3): factoring Hs once and solving the
// x, y and z columns together gives the same solution with a 3x smaller factor.
//
// Pipeline: geometric nested dissection -> elimination tree -> postorder ->
// column structures -> fundamental supernodes (+ relaxed amalgamation, width
// capped) -> right-looking supernodal Cholesky (LL^T) with the
// regularise-and-retry rule of World::FactorizeLDLT -> inverses of the
// diagonal blocks -> level schedule of the supernodal elimination tree.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dfem {

struct SparseSym {           // symmetric matrix, full pattern, CSR by rows
  int n = 0;
  std::vector<int64_t> ptr;
  std::vector<int> col;
  std::vector<double> val;
};

struct SupernodalFactor {
  int n = 0;
  std::vector<int> perm;     // perm[new] = old
  std::vector<int> iperm;    // iperm[old] = new
  int nsuper = 0;
  std::vector<int> sn_c0, sn_w, sn_r;        // first column, width, rows below the diagonal block
  std::vector<int64_t> sn_rofs;               // offset into rowidx
  std::vector<int> rowidx;                    // below-diagonal row ids (permuted numbering)
  std::vector<int64_t> sn_lofs;               // offset into Lcm (column-major r x w block)
  std::vector<double> Lcm;
  std::vector<int64_t> sn_dofs;               // offset into Ldiag / Dinv (w x w, row-major)
  std::vector<double> Ldiag, Dinv;            // diagonal block and its inverse (both lower)
  std::vector<int> sn_parent;                 // -1 for roots
  std::vector<int> col_sn;                    // supernode of each column
  // forward solve in push form: supernode s writes L_{R_s,s} y_s to the
  // contribution slots sn_rofs[s] .. sn_rofs[s]+r_s (one per below-diagonal row);
  // row i then subtracts the contributions listed in rseg_pos[rseg_ptr[i] ..]
  std::vector<int> rseg_ptr;   // n+1
  std::vector<int> rseg_pos;   // positions into rowidx (== contribution slots)
  // level schedule: level 0 = leaves
  int nlevels = 0;
  std::vector<int> lvl_ptr, lvl_sn;
  double reg = 0.0;                           // regularisation that made the factor succeed
  int64_t nnz_factor = 0;
};

struct FactorOptions {
  int leaf_size = 48;        // nested-dissection leaf size
  int max_width = 96;        // supernode width cap
  int relax_small = 16;      // always merge child+parent while the merged width <= this
  double relax_frac = 0.15;  // otherwise merge when added zeros <= frac of the merged block
};

// Symbolic + numeric factorisation.  coords (3 per vertex, may be null) drive
// the geometric nested dissection; without coords a BFS level-set bisection is
// used.  Returns false with err set when the factorisation failed after the
// regularisation retries.
bool factorize(const SparseSym& A, const double* coords, const FactorOptions& opt,
               SupernodalFactor& F, std::string& err);

// Numeric re-factorisation with the same symbolic structure and new values
// (same pattern as the A passed to factorize).
bool refactorize(const SparseSym& A, SupernodalFactor& F, std::string& err);

// Host reference solve with the factor (3 right-hand sides interleaved).
void host_solve(const SupernodalFactor& F, const double* b, double* x);

}  // namespace dfem
