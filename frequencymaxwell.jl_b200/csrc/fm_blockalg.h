// Host algebra of s-step (block) GMRES for one right-hand side: the state of the basis X = V Rf, the
// Hessenberg matrix in V coordinates, the Givens rotations, and the small dense steps between the kernels.
// Used by the batched block solve (all right-hand sides at the same column m) and by the slot engine (each
// slot at its own m).  Every function works on one right-hand side; the device sums come in as FP64.
#pragma once
#include <complex>
#include <vector>
#include <vector_types.h>

namespace fm {

using cdb = std::complex<double>;

struct BlkState {
  bool active = true, solved = false;
  double beta = 0, eps = 0, rnorm = 0;
  int iters = 0;            // Krylov iterations (Hessenberg columns) taken
  int nvec = 0;             // stored basis vectors
  int ld = 0;               // leading dimension of H and Rf
  std::vector<cdb> H;       // V-coordinate Hessenberg, H[i + j*ld]
  std::vector<cdb> Rf;      // X = V Rf, Rf[i + k*ld]
  std::vector<int> b0;      // first index of the diagonal block of Rf that holds column k
  std::vector<double> c;    // Givens
  std::vector<cdb> s, z;
  std::vector<std::vector<cdb>> Rg;
  std::vector<cdb> theta;   // Newton shifts
};

// eigenvalues of an n x n complex upper Hessenberg matrix (column-major), shifted QR with deflation
bool hess_eigs(int n, std::vector<cdb> A, std::vector<cdb>& ev);
// Leja ordering: start from the largest modulus, then maximise the product of distances
void leja_order(std::vector<cdb>& z);
// G = R^H R for an n x n Hermitian positive definite G (column-major); false when not positive definite
bool chol_upper(int n, const std::vector<cdb>& G, std::vector<cdb>& R);
// d = Rf^{-1} c and d = Rf^{-H} c over the first K indices (K ends on a block boundary)
void rf_solve(const BlkState& st, int K, const cdb* c, cdb* d);
void rf_solve_h(const BlkState& st, int K, const cdb* c, cdb* d);

// Start of a solve from ||r0|| = beta: X_0 = r0, Rf = [beta].  Returns true when the right-hand side is solved
// already (beta = 0 or beta <= abstol + reltol beta); it is then marked inactive.
bool blk_init(BlkState& r, int ld, double beta, double abstol, double reltol);
// A new cycle of restarted block GMRES from the updated residual ||r|| = beta, keeping the first cycle's
// tolerance eps; as a restarted GMRES cycle begins, there is no stopping test here.
void blk_restart(BlkState& r, int ld, double beta, double eps);
// Givens update with Hessenberg column j (Krylov.jl gmres); true when the right-hand side stops at this column
// (solved, Krylov breakdown, or itmax columns).
bool blk_givens_col(BlkState& r, int j, int itmax);
// Classical Gram-Schmidt step m (the first s steps): from hr[k] = <X_k, w> (k <= m) the Hessenberg column
// H[k, m] = hr[k] / Rf[k,k] and the update coefficients cf[k] = H[k, m] / Rf[k,k] of w -= sum cf[k] X_k.
void blk_cgs_coefs(BlkState& r, int m, const double2* hr, double2* cf);
// ... and, with hb = ||w|| after the update, the new stored vector X_{m+1} = w; true when the RHS stops.
bool blk_cgs_close(BlkState& r, int m, double hb, int itmax);
// Newton shifts of the next block: Ritz values of the S x S diagonal Hessenberg block at column j0, Leja
// ordered (the previous shifts are kept when the eigenvalue iteration fails; zeros at first).
void blk_shifts(BlkState& r, int j0, int S);
// Start vector of the block at column m: Y_0 = V_m = sum_{a < nc} cc[a] X_{k0+a}.  Returns k0; nc = m - k0 + 1.
int blk_start(const BlkState& r, int m, double2* cc);
// From the block dot D[k*S + t] = <X_k, Y_t> (k <= m, t < S): the V coordinates Cv[k + t*K] (K = m + 1) and the
// X-coordinate update coefficients cf[k*S + t] of Y' = Y - X E.
void blk_project(const BlkState& r, int m, int S, const double2* D, std::vector<cdb>& Cv, double2* cf);
// From the Gram matrix of Y' (upper triangle tri(t,u) for S <= 8, the full S x S at t*S + u above): the new
// stored vectors, the Hessenberg columns m..m+S-1 from the block relations, refreshed shifts and the Givens
// rotations.  For the orthonormalised storage rbi[u*S + t] receives Rb^{-1} (V = Y' Rb^{-1}; zeros when the
// block lost rank).  Returns true when the right-hand side stops (block rank loss or a Givens stop).
bool blk_absorb(BlkState& r, int m, int S, bool ortho_store, const double2* G, const std::vector<cdb>& Cv,
                double2* rbi, int itmax);
// Krylov correction in X coordinates: x += sum_{k < n} d[k] X_k.  Returns n (0: nothing to add).
int blk_solution(const BlkState& r, double2* d);

}  // namespace fm
