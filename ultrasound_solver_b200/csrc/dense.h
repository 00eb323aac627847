// Small dense complex linear algebra on the host (FP64), for the harmonic
// Ritz step of the recycled (GCRO-DR) GMRES cycles: n <= 2 * USV_MAX_RESTART.
// Column-major std::complex<double> storage throughout.
#pragma once

#include <complex>
#include <vector>

namespace usv {
namespace dense {

using cd = std::complex<double>;

// Eigenvalues (and, for the indices in `want`, unit-norm eigenvectors) of a
// general complex n x n matrix: Householder reduction to Hessenberg form, then
// the single-shift implicit QR algorithm with Wilkinson shifts to the complex
// Schur form T = Z^H A Z, then back substitution in T. `a` is overwritten.
// Returns false if the QR iteration did not converge.
bool eig(int n, std::vector<cd>& a, std::vector<cd>& w);
bool eigvecs(int n, const std::vector<cd>& T, const std::vector<cd>& Z, const std::vector<int>& want,
             std::vector<cd>& vecs);
bool schur(int n, std::vector<cd>& a, std::vector<cd>& z, std::vector<cd>& w);

// The k eigenvalues of largest modulus of a general complex n x n matrix and
// unit eigenvectors: Hessenberg reduction, eigenvalue-only QR sweeps on the
// active window, then inverse iteration on the Hessenberg matrix.
bool eig_selected(int n, const std::vector<cd>& a, int k, std::vector<cd>& lam,
                  std::vector<cd>& vecs);
bool hessenberg_eigenvalues(int n, std::vector<cd>& h, std::vector<cd>& w);

// Cholesky A = L L^H of a Hermitian positive definite matrix (lower L in `a`).
bool cholesky(int n, std::vector<cd>& a);

// Harmonic Ritz vectors for the recycled GMRES cycle. G and W are the
// (m+1) x m matrices of A W_m = Vhat_{m+1} G and Vhat_{m+1}^H W_m; the k
// solutions z of G^H G z = theta G^H W z with the smallest |theta| are
// returned in P (m x k, unit columns), their theta in `theta`.
bool harmonic_ritz(int m, int k, const std::vector<cd>& G, const std::vector<cd>& W,
                   std::vector<cd>& P, std::vector<cd>& theta);

// Thin QR (modified Gram-Schmidt, applied twice) of the rows x cols matrix X:
// X = Q R, Q rows x cols with orthonormal columns, R cols x cols upper.
bool qr(int rows, int cols, const std::vector<cd>& X, std::vector<cd>& Q, std::vector<cd>& R);

}  // namespace dense
}  // namespace usv
