// Dense symmetric / Hermitian eigensolver for the small Rayleigh-Ritz problems of the Davidson
// iteration (k <= 128), on the host in FP64.
//
// Real symmetric: Householder reduction to tridiagonal form followed by the implicit QL algorithm with
// Wilkinson-type shifts (Golub & Van Loan, "Matrix Computations", sections 8.3 and 8.5), eigenvectors
// accumulated.  The code follows the published EISPACK routines TRED2 (Householder tridiagonalisation
// with accumulated transforms) and TQL2 (implicit QL on the tridiagonal matrix): Martin, Reinsch and
// Wilkinson, Numer. Math. 11 (1968) 181-195 and Bowdler, Martin, Reinsch and Wilkinson, Numer. Math. 11
// (1968) 293-306, as collected in the Handbook for Automatic Computation, vol. II (1971), and the EISPACK
// Guide (Smith et al., Lecture Notes in Computer Science 6, 1976): the same row scaling, the h / f / g
// Householder quantities and the off-diagonal vector e[] of those routines.  Complex Hermitian H = A + iB is solved through its real symmetric 2k x 2k form
// [[A, -B], [B, A]], whose eigenvectors [x; y] give eigenvectors x + iy of H; each eigenvalue appears
// twice there, and the duplicate (i times the same complex vector) is removed by Gram-Schmidt.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <numeric>
#include <vector>

namespace heff {

// a: n x n symmetric, column-major (overwritten by eigenvectors, column j <-> w[j]); w ascending.
inline int sym_eig(int n, std::vector<double> &a, std::vector<double> &w) {
    w.assign(n, 0.0);
    if(n == 0) return 0;
    std::vector<double> e(n, 0.0);
    auto A = [&](int i, int j) -> double & { return a[i + (size_t)n * j]; };
    // --- Householder tridiagonalisation (rows/cols n-1 .. 1), accumulating the transform in A
    for(int i = n - 1; i > 0; i--) {
        const int l     = i - 1;
        double    h     = 0.0;
        double    scale = 0.0;
        if(l > 0) {
            for(int k = 0; k <= l; k++) scale += std::fabs(A(i, k));
            if(scale == 0.0) {
                e[i] = A(i, l);
            } else {
                for(int k = 0; k <= l; k++) {
                    A(i, k) /= scale;
                    h += A(i, k) * A(i, k);
                }
                double f = A(i, l);
                double g = (f >= 0.0) ? -std::sqrt(h) : std::sqrt(h);
                e[i]     = scale * g;
                h -= f * g;
                A(i, l) = f - g;
                f       = 0.0;
                for(int j = 0; j <= l; j++) {
                    A(j, i) = A(i, j) / h;
                    g       = 0.0;
                    for(int k = 0; k <= j; k++) g += A(j, k) * A(i, k);
                    for(int k = j + 1; k <= l; k++) g += A(k, j) * A(i, k);
                    e[j] = g / h;
                    f += e[j] * A(i, j);
                }
                const double hh = f / (h + h);
                for(int j = 0; j <= l; j++) {
                    f       = A(i, j);
                    e[j]    = e[j] - hh * f;
                    g       = e[j];
                    for(int k = 0; k <= j; k++) A(j, k) -= (f * e[k] + g * A(i, k));
                }
            }
        } else {
            e[i] = A(i, l);
        }
        w[i] = h;
    }
    w[0] = 0.0;
    e[0] = 0.0;
    for(int i = 0; i < n; i++) {
        const int l = i - 1;
        if(w[i] != 0.0) {
            for(int j = 0; j <= l; j++) {
                double g = 0.0;
                for(int k = 0; k <= l; k++) g += A(i, k) * A(k, j);
                for(int k = 0; k <= l; k++) A(k, j) -= g * A(k, i);
            }
        }
        w[i]    = A(i, i);
        A(i, i) = 1.0;
        for(int j = 0; j <= l; j++) A(j, i) = A(i, j) = 0.0;
    }
    // --- implicit QL on the tridiagonal (diag w, offdiag e[1..n-1])
    for(int i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    for(int l = 0; l < n; l++) {
        int iter = 0;
        int m;
        do {
            for(m = l; m < n - 1; m++) {
                const double dd = std::fabs(w[m]) + std::fabs(w[m + 1]);
                if(std::fabs(e[m]) <= 1e-300 || std::fabs(e[m]) <= 2.2e-16 * dd) break;
            }
            if(m != l) {
                if(iter++ == 60) return 1;  // no convergence
                double g = (w[l + 1] - w[l]) / (2.0 * e[l]);
                double r = std::hypot(g, 1.0);
                g        = w[m] - w[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
                double s = 1.0, c = 1.0, p = 0.0;
                int    i;
                for(i = m - 1; i >= l; i--) {
                    double f = s * e[i];
                    double b = c * e[i];
                    r        = std::hypot(f, g);
                    e[i + 1] = r;
                    if(r == 0.0) {
                        w[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    s        = f / r;
                    c        = g / r;
                    g        = w[i + 1] - p;
                    r        = (w[i] - g) * s + 2.0 * c * b;
                    p        = s * r;
                    w[i + 1] = g + p;
                    g        = c * r - b;
                    for(int k = 0; k < n; k++) {
                        f           = A(k, i + 1);
                        A(k, i + 1) = s * A(k, i) + c * f;
                        A(k, i)     = c * A(k, i) - s * f;
                    }
                }
                if(r == 0.0 && i >= l) continue;
                w[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while(m != l);
    }
    // --- sort ascending
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](int x, int y) { return w[x] < w[y]; });
    std::vector<double> w2(n), a2((size_t)n * n);
    for(int j = 0; j < n; j++) {
        w2[j] = w[idx[j]];
        for(int i = 0; i < n; i++) a2[i + (size_t)n * j] = a[i + (size_t)n * idx[j]];
    }
    w.swap(w2);
    a.swap(a2);
    return 0;
}

// Hermitian k x k (column-major complex) -> ascending eigenvalues w[k], eigenvectors v (k x k complex).
inline int herm_eig(int k, const std::vector<std::complex<double>> &h, std::vector<double> &w, std::vector<std::complex<double>> &v) {
    const int           n2 = 2 * k;
    std::vector<double> a((size_t)n2 * n2);
    for(int j = 0; j < k; j++)
        for(int i = 0; i < k; i++) {
            const double re = h[i + (size_t)k * j].real(), im = h[i + (size_t)k * j].imag();
            a[i + (size_t)n2 * j]             = re;
            a[(i + k) + (size_t)n2 * (j + k)] = re;
            a[(i + k) + (size_t)n2 * j]       = im;
            a[i + (size_t)n2 * (j + k)]       = -im;
        }
    std::vector<double> ww;
    if(sym_eig(n2, a, ww)) return 1;
    w.clear();
    v.clear();
    for(int c = 0; c < n2 && (int)w.size() < k; c++) {
        std::vector<std::complex<double>> z(k);
        double                            nn = 0;
        for(int i = 0; i < k; i++) {
            z[i] = {a[i + (size_t)n2 * c], a[(i + k) + (size_t)n2 * c]};
            nn += std::norm(z[i]);
        }
        // remove components along accepted vectors (two passes)
        for(int pass = 0; pass < 2; pass++)
            for(size_t q = 0; q < w.size(); q++) {
                std::complex<double> dot = 0;
                for(int i = 0; i < k; i++) dot += std::conj(v[i + (size_t)k * q]) * z[i];
                for(int i = 0; i < k; i++) z[i] -= dot * v[i + (size_t)k * q];
            }
        double rn = 0;
        for(int i = 0; i < k; i++) rn += std::norm(z[i]);
        if(rn < 0.25 * nn) continue;  // duplicate (i * an accepted vector)
        rn = std::sqrt(rn);
        for(int i = 0; i < k; i++) v.push_back(z[i] / rn);
        w.push_back(ww[c]);
    }
    return (int)w.size() == k ? 0 : 1;
}

}  // namespace heff
