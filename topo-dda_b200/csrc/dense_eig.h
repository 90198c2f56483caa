// Small dense complex eigenproblems on the host (the Krylov solvers' projected
// matrices, order <= a few hundred): Householder reduction to upper Hessenberg
// form, the shifted QR algorithm (Wilkinson shifts, deflation of negligible
// subdiagonal entries) with or without the Schur vectors, and eigenvectors of
// the triangular Schur factor by back substitution.  Matrices are
// column-major with a leading dimension.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace tdda {

using cplx = std::complex<double>;

struct DenseMat {
    int n = 0;
    std::vector<cplx> a;
    explicit DenseMat(int n_ = 0) : n(n_), a((size_t)n_ * n_, cplx(0.0)) {}
    cplx &operator()(int i, int j) { return a[i + (size_t)j * n]; }
    cplx operator()(int i, int j) const { return a[i + (size_t)j * n]; }
};

// A <- Q^H A Q upper Hessenberg; Q (if given) accumulates the reflections
// (starts as the identity).
inline void hessenberg_reduce(DenseMat &A, DenseMat *Q) {
    const int n = A.n;
    if (Q) {
        *Q = DenseMat(n);
        for (int i = 0; i < n; ++i) (*Q)(i, i) = 1.0;
    }
    std::vector<cplx> v(n);
    for (int k = 0; k + 2 < n; ++k) {
        // a column already zero below its subdiagonal needs no reflector
        bool zero_below = true;
        for (int i = k + 2; i < n && zero_below; ++i) zero_below = A(i, k) == cplx(0.0);
        if (zero_below) continue;
        double alpha2 = 0.0;
        for (int i = k + 1; i < n; ++i) alpha2 += std::norm(A(i, k));
        const double xnorm = std::sqrt(alpha2);
        if (xnorm == 0.0) continue;
        const cplx x0 = A(k + 1, k);
        const cplx ph = std::abs(x0) > 0 ? x0 / std::abs(x0) : cplx(1.0);
        // v = x + ph |x| e1, H = I - 2 v v^H / (v^H v)
        for (int i = 0; i < n; ++i) v[i] = 0.0;
        for (int i = k + 1; i < n; ++i) v[i] = A(i, k);
        v[k + 1] += ph * xnorm;
        double vv = 0.0;
        for (int i = k + 1; i < n; ++i) vv += std::norm(v[i]);
        if (vv == 0.0) continue;
        const double tau = 2.0 / vv;
        // A <- H A (columns k.. only: the earlier ones are zero below row k)
        for (int j = k; j < n; ++j) {
            cplx *col = &A.a[(size_t)j * n];
            cplx s = 0.0;
            for (int i = k + 1; i < n; ++i) s += std::conj(v[i]) * col[i];
            s *= tau;
            for (int i = k + 1; i < n; ++i) col[i] -= s * v[i];
        }
        // A <- A H, column by column (contiguous inner loops)
        auto right = [&](DenseMat &M) {
            std::vector<cplx> sv(n, cplx(0.0));
            for (int j = k + 1; j < n; ++j) {
                const cplx vj = v[j];
                const cplx *col = &M.a[(size_t)j * n];
                for (int i = 0; i < n; ++i) sv[i] += col[i] * vj;
            }
            for (int i = 0; i < n; ++i) sv[i] *= tau;
            for (int j = k + 1; j < n; ++j) {
                const cplx cj = std::conj(v[j]);
                cplx *col = &M.a[(size_t)j * n];
                for (int i = 0; i < n; ++i) col[i] -= sv[i] * cj;
            }
        };
        right(A);
        for (int i = k + 2; i < n; ++i) A(i, k) = 0.0;
        if (Q) right(*Q);
    }
}

// Shifted QR on the upper-Hessenberg H: with Z, H becomes the upper
// triangular Schur factor T (H_in = Z T Z^H, Z accumulated onto its input);
// without Z only the active blocks are updated and just the eigenvalues
// (the diagonal) are meaningful.  false if an eigenvalue did not converge.
inline bool hessenberg_qr(DenseMat &H, DenseMat *Z) {
    const int n = H.n;
    const bool full = Z != nullptr;
    int hi = n - 1, iter = 0;
    std::vector<cplx> cs, sn;
    while (hi > 0) {
        int lo = hi;
        while (lo > 0) {
            double s = std::abs(H(lo - 1, lo - 1)) + std::abs(H(lo, lo));
            if (s == 0.0) s = 1.0;
            if (std::abs(H(lo, lo - 1)) <= 1e-15 * s) { H(lo, lo - 1) = 0.0; break; }
            --lo;
        }
        if (lo == hi) { --hi; iter = 0; continue; }
        if (++iter > 60 * (hi - lo + 1)) return false;
        const cplx a = H(hi - 1, hi - 1), b = H(hi - 1, hi), c = H(hi, hi - 1), d = H(hi, hi);
        const cplx tr = a + d, det = a * d - b * c;
        const cplx disc = std::sqrt(tr * tr / 4.0 - det);
        const cplx l1 = tr / 2.0 + disc, l2 = tr / 2.0 - disc;
        cplx mu = (std::abs(l1 - d) < std::abs(l2 - d)) ? l1 : l2;
        if (iter % 11 == 10) mu = d + cplx(std::abs(c), 0.0);  // exceptional shift
        const int c0 = full ? 0 : lo, c1 = full ? n - 1 : hi;  // extent of the row / column updates
        for (int k = lo; k <= hi; ++k) H(k, k) -= mu;
        cs.assign(hi - lo, 0.0);
        sn.assign(hi - lo, 0.0);
        for (int k = lo; k < hi; ++k) {
            const cplx x = H(k, k), y = H(k + 1, k);
            const double r = std::sqrt(std::norm(x) + std::norm(y));
            const cplx cc = r == 0.0 ? cplx(1.0) : x / r, ss = r == 0.0 ? cplx(0.0) : y / r;
            cs[k - lo] = cc;
            sn[k - lo] = ss;
            for (int j = k; j <= c1; ++j) {
                const cplx u = H(k, j), v = H(k + 1, j);
                H(k, j) = std::conj(cc) * u + std::conj(ss) * v;
                H(k + 1, j) = -ss * u + cc * v;
            }
        }
        for (int k = lo; k < hi; ++k) {
            const cplx cc = cs[k - lo], ss = sn[k - lo];
            for (int i = c0; i <= std::min(k + 2, hi); ++i) {
                const cplx u = H(i, k), v = H(i, k + 1);
                H(i, k) = u * cc + v * ss;
                H(i, k + 1) = -u * std::conj(ss) + v * std::conj(cc);
            }
            if (full) {
                DenseMat &z = *Z;
                for (int i = 0; i < n; ++i) {
                    const cplx u = z(i, k), v = z(i, k + 1);
                    z(i, k) = u * cc + v * ss;
                    z(i, k + 1) = -u * std::conj(ss) + v * std::conj(cc);
                }
            }
        }
        for (int k = lo; k <= hi; ++k) H(k, k) += mu;
    }
    return true;
}

// Eigenvector of the upper triangular T for its eigenvalue T(p, p): x with
// x_p = 1, x_i = 0 for i > p, by back substitution (a tiny shift keeps
// repeated eigenvalues from dividing by zero).
inline std::vector<cplx> triangular_eigvec(const DenseMat &T, int p) {
    const int n = T.n;
    std::vector<cplx> x(n, cplx(0.0));
    x[p] = 1.0;
    const cplx lam = T(p, p);
    double scale = 0.0;
    for (int i = 0; i < n; ++i) scale = std::max(scale, std::abs(T(i, i)));
    const double tiny = 1e-14 * (scale > 0 ? scale : 1.0);
    for (int i = p - 1; i >= 0; --i) {
        cplx s = 0.0;
        for (int j = i + 1; j <= p; ++j) s += T(i, j) * x[j];
        cplx den = T(i, i) - lam;
        if (std::abs(den) < tiny) den = tiny;
        x[i] = -s / den;
    }
    return x;
}

// Eigenvalues of the general n x n A (copied).
inline bool eigenvalues(DenseMat A, std::vector<cplx> &ev) {
    hessenberg_reduce(A, nullptr);
    if (!hessenberg_qr(A, nullptr)) return false;
    ev.resize(A.n);
    for (int i = 0; i < A.n; ++i) ev[i] = A(i, i);
    return true;
}

// Eigenvalues of A (copied) and the eigenvectors (unit 2-norm) of those
// selected by pick(ev) -> indices.
template <class Pick>
bool eigenpairs(DenseMat A, std::vector<cplx> &ev, std::vector<std::vector<cplx>> &vecs, Pick pick) {
    const int n = A.n;
    DenseMat Z;
    hessenberg_reduce(A, &Z);
    if (!hessenberg_qr(A, &Z)) return false;
    ev.resize(n);
    for (int i = 0; i < n; ++i) ev[i] = A(i, i);
    const std::vector<int> idx = pick(ev);
    vecs.clear();
    for (int p : idx) {
        const std::vector<cplx> y = triangular_eigvec(A, p);
        std::vector<cplx> v(n, cplx(0.0));
        for (int j = 0; j <= p; ++j)
            if (y[j] != cplx(0.0))
                for (int i = 0; i < n; ++i) v[i] += Z(i, j) * y[j];
        double nr = 0.0;
        for (auto &e : v) nr += std::norm(e);
        nr = std::sqrt(nr);
        if (nr > 0)
            for (auto &e : v) e /= nr;
        vecs.push_back(v);
    }
    return true;
}

// Solves (H - theta I) x = b for the upper-Hessenberg H (column-major;
// Gaussian elimination with pivoting between neighbouring rows, O(n^2)); a
// zero pivot is replaced by a tiny one (theta may be an eigenvalue).
inline std::vector<cplx> hessenberg_shifted_solve(const DenseMat &H, cplx theta, std::vector<cplx> b) {
    const int n = H.n;
    DenseMat A = H;
    for (int i = 0; i < n; ++i) A(i, i) -= theta;
    double scale = 0.0;
    for (int i = 0; i < n; ++i) scale = std::max(scale, std::abs(H(i, i)));
    const double tiny = 1e-14 * (scale > 0 ? scale : 1.0);
    for (int k = 0; k + 1 < n; ++k) {
        if (std::abs(A(k + 1, k)) > std::abs(A(k, k))) {
            for (int j = k; j < n; ++j) std::swap(A(k, j), A(k + 1, j));
            std::swap(b[k], b[k + 1]);
        }
        if (std::abs(A(k, k)) < tiny) A(k, k) = tiny;
        const cplx f = A(k + 1, k) / A(k, k);
        if (f != cplx(0.0)) {
            for (int j = k; j < n; ++j) A(k + 1, j) -= f * A(k, j);
            b[k + 1] -= f * b[k];
        }
    }
    if (std::abs(A(n - 1, n - 1)) < tiny) A(n - 1, n - 1) = tiny;
    std::vector<cplx> x(n);
    for (int i = n - 1; i >= 0; --i) {
        cplx t = b[i];
        for (int j = i + 1; j < n; ++j) t -= A(i, j) * x[j];
        x[i] = t / A(i, i);
    }
    return x;
}

// As eigenpairs, for a few eigenvectors: the eigenvalues from the QR
// iteration without Schur vectors, the selected eigenvectors by two steps of
// inverse iteration on the Hessenberg form, mapped back through the
// reduction's reflections.  Much cheaper when few vectors are wanted.
template <class Pick>
bool eigenpairs_few(DenseMat A, std::vector<cplx> &ev, std::vector<std::vector<cplx>> &vecs, Pick pick) {
    const int n = A.n;
    DenseMat Q;
    hessenberg_reduce(A, &Q);
    DenseMat H = A;
    if (!hessenberg_qr(H, nullptr)) return false;
    ev.resize(n);
    for (int i = 0; i < n; ++i) ev[i] = H(i, i);
    const std::vector<int> idx = pick(ev);
    vecs.clear();
    for (int p : idx) {
        std::vector<cplx> x(n, cplx(1.0 / std::sqrt((double)n)));
        for (int it = 0; it < 2; ++it) {
            x = hessenberg_shifted_solve(A, ev[p], x);
            double nr = 0.0;
            for (auto &e : x) nr += std::norm(e);
            nr = std::sqrt(nr);
            if (!(nr > 0.0) || !std::isfinite(nr)) return false;
            for (auto &e : x) e /= nr;
        }
        std::vector<cplx> v(n, cplx(0.0));
        for (int j = 0; j < n; ++j) {
            const cplx xj = x[j];
            const cplx *col = &Q.a[(size_t)j * n];
            for (int i = 0; i < n; ++i) v[i] += col[i] * xj;
        }
        vecs.push_back(v);
    }
    return true;
}

}  // namespace tdda
