// Host dense complex linear algebra for the harmonic Ritz step (see dense.h).
//
// The eigen-solver is the textbook route (Golub & Van Loan, "Matrix
// Computations", 4th ed., sections 7.4-7.5): Householder reduction to upper
// Hessenberg form, single-shift implicit QR sweeps (Givens bulge chase) with
// the Wilkinson shift and deflation on negligible subdiagonals, exceptional
// shifts every 10 stalled sweeps, eigenvectors from the triangular Schur
// factor by back substitution.
#include "dense.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace usv {
namespace dense {

namespace {

inline cd& at(std::vector<cd>& a, int n, int i, int j) { return a[i + size_t(j) * n]; }
inline const cd& at(const std::vector<cd>& a, int n, int i, int j) { return a[i + size_t(j) * n]; }

// Givens rotation [[c, s], [-conj(s), c]] (c real) with G [x; y] = [r; 0].
inline void givens(cd x, cd y, double& c, cd& s) {
    const double ax = std::abs(x), ay = std::abs(y);
    if (ay == 0.0) {
        c = 1.0;
        s = 0.0;
    } else if (ax == 0.0) {
        c = 0.0;
        s = std::conj(y) / ay;
    } else {
        const double r = std::hypot(ax, ay);
        c = ax / r;
        s = (x / ax) * std::conj(y) / r;
    }
}

void hessenberg(int n, std::vector<cd>& a, std::vector<cd>& z) {
    std::vector<cd> v(n);
    for (int k = 0; k + 2 < n; ++k) {
        double xn2 = 0.0;
        for (int i = k + 1; i < n; ++i) xn2 += std::norm(at(a, n, i, k));
        const double xn = std::sqrt(xn2);
        if (xn == 0.0) continue;
        const cd x0 = at(a, n, k + 1, k);
        const cd phase = std::abs(x0) == 0.0 ? cd(1.0) : x0 / std::abs(x0);
        const cd alpha = -phase * xn;
        const int len = n - k - 1;
        v[0] = x0 - alpha;
        for (int i = 1; i < len; ++i) v[i] = at(a, n, k + 1 + i, k);
        double vn2 = 0.0;
        for (int i = 0; i < len; ++i) vn2 += std::norm(v[i]);
        if (vn2 == 0.0) continue;
        const double f = 2.0 / vn2;
        for (int j = k; j < n; ++j) {  // A <- H A
            cd s = 0.0;
            for (int i = 0; i < len; ++i) s += std::conj(v[i]) * at(a, n, k + 1 + i, j);
            s *= f;
            for (int i = 0; i < len; ++i) at(a, n, k + 1 + i, j) -= s * v[i];
        }
        for (int i = 0; i < n; ++i) {  // A <- A H, Z <- Z H
            cd s = 0.0, t = 0.0;
            for (int l = 0; l < len; ++l) {
                s += at(a, n, i, k + 1 + l) * v[l];
                t += at(z, n, i, k + 1 + l) * v[l];
            }
            s *= f;
            t *= f;
            for (int l = 0; l < len; ++l) {
                at(a, n, i, k + 1 + l) -= s * std::conj(v[l]);
                at(z, n, i, k + 1 + l) -= t * std::conj(v[l]);
            }
        }
        at(a, n, k + 1, k) = alpha;
        for (int i = k + 2; i < n; ++i) at(a, n, i, k) = 0.0;
    }
}

}  // namespace

bool schur(int n, std::vector<cd>& a, std::vector<cd>& z, std::vector<cd>& w) {
    z.assign(size_t(n) * n, cd(0.0));
    for (int i = 0; i < n; ++i) at(z, n, i, i) = 1.0;
    w.assign(n, cd(0.0));
    if (n == 0) return true;
    hessenberg(n, a, z);
    double anorm = 0.0;
    for (const cd& v : a) anorm = std::max(anorm, std::abs(v));
    if (anorm == 0.0) return true;
    const double eps = std::numeric_limits<double>::epsilon();
    int hi = n - 1, iter = 0, total = 0;
    while (hi > 0) {
        int l = hi;
        for (; l > 0; --l) {
            double s = std::abs(at(a, n, l - 1, l - 1)) + std::abs(at(a, n, l, l));
            if (s == 0.0) s = anorm;
            if (std::abs(at(a, n, l, l - 1)) <= eps * s) {
                at(a, n, l, l - 1) = 0.0;
                break;
            }
        }
        if (l == hi) {
            --hi;
            iter = 0;
            continue;
        }
        if (++total > 60 * n) return false;
        ++iter;
        cd mu;
        if (iter % 10 == 0) {
            mu = at(a, n, hi, hi) + 0.75 * std::abs(at(a, n, hi, hi - 1));
        } else {
            const cd a11 = at(a, n, hi - 1, hi - 1), a12 = at(a, n, hi - 1, hi);
            const cd a21 = at(a, n, hi, hi - 1), a22 = at(a, n, hi, hi);
            const cd half_tr = 0.5 * (a11 + a22);
            const cd disc = std::sqrt(half_tr * half_tr - (a11 * a22 - a12 * a21));
            const cd m1 = half_tr + disc, m2 = half_tr - disc;
            mu = std::abs(m1 - a22) < std::abs(m2 - a22) ? m1 : m2;
        }
        for (int k = l; k < hi; ++k) {
            cd x, y;
            if (k == l) {
                x = at(a, n, l, l) - mu;
                y = at(a, n, l + 1, l);
            } else {
                x = at(a, n, k, k - 1);
                y = at(a, n, k + 1, k - 1);
            }
            double c;
            cd s;
            givens(x, y, c, s);
            for (int j = (k > l ? k - 1 : l); j < n; ++j) {  // rows k, k+1
                const cd t1 = at(a, n, k, j), t2 = at(a, n, k + 1, j);
                at(a, n, k, j) = c * t1 + s * t2;
                at(a, n, k + 1, j) = -std::conj(s) * t1 + c * t2;
            }
            if (k > l) at(a, n, k + 1, k - 1) = 0.0;
            const int rmax = std::min(k + 2, hi);
            for (int i = 0; i <= rmax; ++i) {  // columns k, k+1 (times G^H)
                const cd t1 = at(a, n, i, k), t2 = at(a, n, i, k + 1);
                at(a, n, i, k) = c * t1 + std::conj(s) * t2;
                at(a, n, i, k + 1) = -s * t1 + c * t2;
            }
            for (int i = 0; i < n; ++i) {
                const cd t1 = at(z, n, i, k), t2 = at(z, n, i, k + 1);
                at(z, n, i, k) = c * t1 + std::conj(s) * t2;
                at(z, n, i, k + 1) = -s * t1 + c * t2;
            }
        }
    }
    for (int i = 0; i < n; ++i) w[i] = at(a, n, i, i);
    return true;
}

bool eig(int n, std::vector<cd>& a, std::vector<cd>& w) {
    std::vector<cd> z;
    return schur(n, a, z, w);
}

bool eigvecs(int n, const std::vector<cd>& T, const std::vector<cd>& Z, const std::vector<int>& want,
             std::vector<cd>& vecs) {
    double tnorm = 0.0;
    for (const cd& v : T) tnorm = std::max(tnorm, std::abs(v));
    const double small = std::max(tnorm, 1e-300) * std::numeric_limits<double>::epsilon();
    vecs.assign(size_t(n) * want.size(), cd(0.0));
    std::vector<cd> x(n);
    for (size_t q = 0; q < want.size(); ++q) {
        const int i = want[q];
        if (i < 0 || i >= n) return false;
        const cd lam = at(T, n, i, i);
        std::fill(x.begin(), x.end(), cd(0.0));
        x[i] = 1.0;
        for (int r = i - 1; r >= 0; --r) {
            cd s = 0.0;
            for (int c = r + 1; c <= i; ++c) s += at(T, n, r, c) * x[c];
            cd d = at(T, n, r, r) - lam;
            if (std::abs(d) < small) d = small;
            x[r] = -s / d;
        }
        double nrm = 0.0;
        cd* out = &vecs[q * size_t(n)];
        for (int r = 0; r < n; ++r) {
            cd s = 0.0;
            for (int c = 0; c <= i; ++c) s += at(Z, n, r, c) * x[c];
            out[r] = s;
            nrm += std::norm(s);
        }
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) return false;
        for (int r = 0; r < n; ++r) out[r] /= nrm;
    }
    return true;
}

bool hessenberg_eigenvalues(int n, std::vector<cd>& h, std::vector<cd>& w) {
    w.assign(n, cd(0.0));
    if (n == 0) return true;
    double anorm = 0.0;
    for (const cd& v : h) anorm = std::max(anorm, std::abs(v));
    if (anorm == 0.0) return true;
    const double eps = std::numeric_limits<double>::epsilon();
    int hi = n - 1, iter = 0, total = 0;
    while (hi > 0) {
        int l = hi;
        for (; l > 0; --l) {
            double s = std::abs(at(h, n, l - 1, l - 1)) + std::abs(at(h, n, l, l));
            if (s == 0.0) s = anorm;
            if (std::abs(at(h, n, l, l - 1)) <= eps * s) {
                at(h, n, l, l - 1) = 0.0;
                break;
            }
        }
        if (l == hi) {
            w[hi] = at(h, n, hi, hi);
            --hi;
            iter = 0;
            continue;
        }
        if (++total > 60 * n) return false;
        ++iter;
        cd mu;
        if (iter % 10 == 0) {
            mu = at(h, n, hi, hi) + 0.75 * std::abs(at(h, n, hi, hi - 1));
        } else {
            const cd a11 = at(h, n, hi - 1, hi - 1), a12 = at(h, n, hi - 1, hi);
            const cd a21 = at(h, n, hi, hi - 1), a22 = at(h, n, hi, hi);
            const cd half_tr = 0.5 * (a11 + a22);
            const cd disc = std::sqrt(half_tr * half_tr - (a11 * a22 - a12 * a21));
            const cd m1 = half_tr + disc, m2 = half_tr - disc;
            mu = std::abs(m1 - a22) < std::abs(m2 - a22) ? m1 : m2;
        }
        // bulge chase restricted to the active window [l, hi]
        for (int k = l; k < hi; ++k) {
            cd x, y;
            if (k == l) {
                x = at(h, n, l, l) - mu;
                y = at(h, n, l + 1, l);
            } else {
                x = at(h, n, k, k - 1);
                y = at(h, n, k + 1, k - 1);
            }
            double c;
            cd s;
            givens(x, y, c, s);
            for (int j = (k > l ? k - 1 : l); j <= hi; ++j) {
                const cd t1 = at(h, n, k, j), t2 = at(h, n, k + 1, j);
                at(h, n, k, j) = c * t1 + s * t2;
                at(h, n, k + 1, j) = -std::conj(s) * t1 + c * t2;
            }
            if (k > l) at(h, n, k + 1, k - 1) = 0.0;
            const int rmax = std::min(k + 2, hi);
            for (int i = l; i <= rmax; ++i) {
                const cd t1 = at(h, n, i, k), t2 = at(h, n, i, k + 1);
                at(h, n, i, k) = c * t1 + std::conj(s) * t2;
                at(h, n, i, k + 1) = -s * t1 + c * t2;
            }
        }
    }
    w[0] = at(h, n, 0, 0);
    return true;
}

// Solve (H - lam I) x = b for upper Hessenberg H by Gaussian elimination with
// partial pivoting between adjacent rows (O(n^2)); tiny pivots are nudged.
static void hessenberg_shifted_solve(int n, const std::vector<cd>& H, cd lam, std::vector<cd>& x,
                                     double small) {
    std::vector<cd> A(H);
    for (int i = 0; i < n; ++i) at(A, n, i, i) -= lam;
    for (int k = 0; k + 1 < n; ++k) {
        if (std::abs(at(A, n, k + 1, k)) > std::abs(at(A, n, k, k))) {
            for (int j = k; j < n; ++j) std::swap(at(A, n, k, j), at(A, n, k + 1, j));
            std::swap(x[k], x[k + 1]);
        }
        cd piv = at(A, n, k, k);
        if (std::abs(piv) < small) piv = at(A, n, k, k) = small;
        const cd f = at(A, n, k + 1, k) / piv;
        if (f != cd(0.0)) {
            for (int j = k + 1; j < n; ++j) at(A, n, k + 1, j) -= f * at(A, n, k, j);
            x[k + 1] -= f * x[k];
        }
        at(A, n, k + 1, k) = 0.0;
    }
    if (std::abs(at(A, n, n - 1, n - 1)) < small) at(A, n, n - 1, n - 1) = small;
    for (int i = n - 1; i >= 0; --i) {
        cd s = x[i];
        for (int j = i + 1; j < n; ++j) s -= at(A, n, i, j) * x[j];
        x[i] = s / at(A, n, i, i);
    }
}

bool eig_selected(int n, const std::vector<cd>& a, int k, std::vector<cd>& lam,
                  std::vector<cd>& vecs) {
    if (k < 1 || k > n) return false;
    std::vector<cd> h(a), q(size_t(n) * n, cd(0.0));
    for (int i = 0; i < n; ++i) at(q, n, i, i) = 1.0;
    hessenberg(n, h, q);
    std::vector<cd> hv(h), w;
    if (!hessenberg_eigenvalues(n, hv, w)) return false;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return std::abs(w[x]) > std::abs(w[y]); });
    double hnorm = 0.0;
    for (const cd& v : h) hnorm = std::max(hnorm, std::abs(v));
    const double small = std::max(hnorm, 1e-300) * 1e-14;
    lam.assign(k, cd(0.0));
    vecs.assign(size_t(n) * k, cd(0.0));
    std::vector<cd> x(n);
    for (int p = 0; p < k; ++p) {
        const cd l0 = w[order[p]];
        lam[p] = l0;
        // inverse iteration, two solves from a fixed start
        for (int i = 0; i < n; ++i) x[i] = cd(1.0, 0.1 * (i % 7));
        for (int it = 0; it < 2; ++it) {
            hessenberg_shifted_solve(n, h, l0, x, small);
            double nrm = 0.0;
            for (const cd& v : x) nrm += std::norm(v);
            nrm = std::sqrt(nrm);
            if (!(nrm > 0.0) || !std::isfinite(nrm)) return false;
            for (cd& v : x) v /= nrm;
        }
        cd* out = &vecs[size_t(p) * n];
        for (int r = 0; r < n; ++r) {
            cd s = 0.0;
            for (int c = 0; c < n; ++c) s += at(q, n, r, c) * x[c];
            out[r] = s;
        }
    }
    return true;
}

bool cholesky(int n, std::vector<cd>& a) {
    for (int j = 0; j < n; ++j) {
        double d = at(a, n, j, j).real();
        for (int k = 0; k < j; ++k) d -= std::norm(at(a, n, j, k));
        if (!(d > 0.0) || !std::isfinite(d)) return false;
        const double ljj = std::sqrt(d);
        at(a, n, j, j) = ljj;
        for (int i = j + 1; i < n; ++i) {
            cd s = at(a, n, i, j);
            for (int k = 0; k < j; ++k) s -= at(a, n, i, k) * std::conj(at(a, n, j, k));
            at(a, n, i, j) = s / ljj;
        }
        for (int i = 0; i < j; ++i) at(a, n, i, j) = 0.0;
    }
    return true;
}

bool harmonic_ritz(int m, int k, const std::vector<cd>& G, const std::vector<cd>& W,
                   std::vector<cd>& P, std::vector<cd>& theta) {
    if (k < 1 || k > m) return false;
    const int r = m + 1;
    // M1 = G^H G, M2 = G^H W
    std::vector<cd> M1(size_t(m) * m), M2(size_t(m) * m);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) {
            cd s1 = 0.0, s2 = 0.0;
            for (int q = 0; q < r; ++q) {
                const cd gq = std::conj(at(G, r, q, i));
                s1 += gq * at(G, r, q, j);
                s2 += gq * at(W, r, q, j);
            }
            at(M1, m, i, j) = s1;
            at(M2, m, i, j) = s2;
        }
    // Hermitian part only (round-off), then Cholesky M1 = L L^H
    for (int j = 0; j < m; ++j) {
        at(M1, m, j, j) = at(M1, m, j, j).real();
        for (int i = j + 1; i < m; ++i) at(M1, m, j, i) = std::conj(at(M1, m, i, j));
    }
    if (!cholesky(m, M1)) return false;
    // S = L^{-1} M2 L^{-H}: forward substitution on the columns of M2, then on the rows
    auto lsolve = [&](std::vector<cd>& X) {  // X <- L^{-1} X (column-wise)
        for (int c = 0; c < m; ++c)
            for (int i = 0; i < m; ++i) {
                cd s = at(X, m, i, c);
                for (int q = 0; q < i; ++q) s -= at(M1, m, i, q) * at(X, m, q, c);
                at(X, m, i, c) = s / at(M1, m, i, i);
            }
    };
    lsolve(M2);
    // (L^{-1} M2) L^{-H} = (L^{-1} (L^{-1} M2)^H)^H
    std::vector<cd> Tt(size_t(m) * m);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) at(Tt, m, i, j) = std::conj(at(M2, m, j, i));
    lsolve(Tt);
    std::vector<cd> S(size_t(m) * m);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) at(S, m, i, j) = std::conj(at(Tt, m, j, i));
    // eigenpairs of S with the largest |mu| (mu = 1/theta)
    std::vector<cd> mu, wv;
    if (!eig_selected(m, S, k, mu, wv)) return false;
    // z = L^{-H} w (back substitution with L^H)
    P.assign(size_t(m) * k, cd(0.0));
    theta.assign(k, cd(0.0));
    for (int q = 0; q < k; ++q) {
        cd* z = &P[size_t(q) * m];
        const cd* wq = &wv[size_t(q) * m];
        for (int i = m - 1; i >= 0; --i) {
            cd s = wq[i];
            for (int c = i + 1; c < m; ++c) s -= std::conj(at(M1, m, c, i)) * z[c];
            z[i] = s / at(M1, m, i, i);
        }
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += std::norm(z[i]);
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) return false;
        for (int i = 0; i < m; ++i) z[i] /= nrm;
        theta[q] = std::abs(mu[q]) > 0.0 ? 1.0 / mu[q] : cd(std::numeric_limits<double>::infinity());
    }
    return true;
}

bool qr(int rows, int cols, const std::vector<cd>& X, std::vector<cd>& Q, std::vector<cd>& R) {
    Q = X;
    R.assign(size_t(cols) * cols, cd(0.0));
    double scale = 0.0;
    for (const cd& v : X) scale = std::max(scale, std::abs(v));
    if (!(scale > 0.0)) return false;
    for (int j = 0; j < cols; ++j) {
        cd* qj = &Q[size_t(j) * rows];
        for (int pass = 0; pass < 2; ++pass)
            for (int i = 0; i < j; ++i) {
                const cd* qi = &Q[size_t(i) * rows];
                cd s = 0.0;
                for (int q = 0; q < rows; ++q) s += std::conj(qi[q]) * qj[q];
                for (int q = 0; q < rows; ++q) qj[q] -= s * qi[q];
                at(R, cols, i, j) += s;
            }
        double nrm = 0.0;
        for (int q = 0; q < rows; ++q) nrm += std::norm(qj[q]);
        nrm = std::sqrt(nrm);
        if (!(nrm > 1e-13 * scale) || !std::isfinite(nrm)) return false;
        at(R, cols, j, j) = nrm;
        for (int q = 0; q < rows; ++q) qj[q] /= nrm;
    }
    return true;
}

}  // namespace dense
}  // namespace usv
