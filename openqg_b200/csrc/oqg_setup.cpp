// oqg_setup.cpp -- init-time host computations of init_qg (qg/qg.F90:60-103).
#include "oqg_setup.h"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace oqg {

// Symmetric eigenproblem by cyclic Jacobi rotations; S, V column-major n x n.
static void sym_eig(int n, std::vector<double> S, std::vector<double> &w, std::vector<double> &V) {
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[i + n * i] = 1.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0;
        for (int c = 0; c < n; ++c)
            for (int r = 0; r < n; ++r)
                if (r != c) off += S[r + n * c] * S[r + n * c];
        if (off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = S[p + n * q];
                if (apq == 0.0) continue;
                const double theta = (S[q + n * q] - S[p + n * p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double a = S[k + n * p], b = S[k + n * q];
                    S[k + n * p] = c * a - s * b;
                    S[k + n * q] = s * a + c * b;
                }
                for (int k = 0; k < n; ++k) {
                    const double a = S[p + n * k], b = S[q + n * k];
                    S[p + n * k] = c * a - s * b;
                    S[q + n * k] = s * a + c * b;
                }
                for (int k = 0; k < n; ++k) {
                    const double a = V[k + n * p], b = V[k + n * q];
                    V[k + n * p] = c * a - s * b;
                    V[k + n * q] = s * a + c * b;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = S[i + n * i];
}

bool setup_modes(int nl, const double *h, const double *gp, double fnot, Modes &md,
                 std::string &err) {
    md.nl = nl;
    std::vector<double> &A = md.amat;
    A.assign((size_t)nl * nl, 0.0);
    auto a = [&](int r, int c) -> double & { return A[r + nl * c]; };
    // compute_A (modes.F90:221-246)
    a(0, 1) = -1.0 / (gp[0] * h[0]);
    a(0, 0) = -a(0, 1);
    for (int k = 1; k < nl - 1; ++k) {
        a(k, k - 1) = -1.0 / (gp[k - 1] * h[k]);
        a(k, k + 1) = -1.0 / (gp[k] * h[k]);
        a(k, k) = -a(k, k - 1) - a(k, k + 1);
    }
    a(nl - 1, nl - 2) = -1.0 / (gp[nl - 2] * h[nl - 1]);
    a(nl - 1, nl - 1) = -a(nl - 1, nl - 2);
    // A = H^-1 T, T symmetric: eigenvectors from H^{1/2} A H^{-1/2}.
    // Right vectors H^{-1/2} v, left vectors H^{1/2} v (both unit length).
    std::vector<double> S((size_t)nl * nl), w, V;
    for (int c = 0; c < nl; ++c)
        for (int r = 0; r < nl; ++r) S[r + nl * c] = std::sqrt(h[r]) * A[r + nl * c] / std::sqrt(h[c]);
    for (int c = 0; c < nl; ++c)
        for (int r = c + 1; r < nl; ++r) {
            const double v = 0.5 * (S[r + nl * c] + S[c + nl * r]);
            S[r + nl * c] = S[c + nl * r] = v;
        }
    sym_eig(nl, S, w, V);
    std::vector<double> R((size_t)nl * nl), L((size_t)nl * nl);
    for (int m = 0; m < nl; ++m) {
        double nr = 0.0, nlv = 0.0;
        int kb = 0;
        for (int k = 0; k < nl; ++k) {
            R[k + nl * m] = V[k + nl * m] / std::sqrt(h[k]);
            L[k + nl * m] = V[k + nl * m] * std::sqrt(h[k]);
            nr += R[k + nl * m] * R[k + nl * m];
            nlv += L[k + nl * m] * L[k + nl * m];
            if (std::fabs(R[k + nl * m]) > std::fabs(R[kb + nl * m])) kb = k;
        }
        const double sg = R[kb + nl * m] < 0 ? -1.0 : 1.0;
        nr = std::sqrt(nr);
        nlv = std::sqrt(nlv);
        for (int k = 0; k < nl; ++k) {
            R[k + nl * m] *= sg / nr;
            L[k + nl * m] *= sg / nlv;
        }
    }
    // modes in increasing |eigenvalue| (barotropic first), modes.F90:99-131
    std::vector<int> idx(nl);
    for (int m = 0; m < nl; ++m) idx[m] = m;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int x, int y) { return std::fabs(w[x]) < std::fabs(w[y]); });
    md.rdm2.assign(nl, 0.0);
    for (int m = 1; m < nl; ++m) md.rdm2[m] = fnot * fnot * std::fabs(w[idx[m]]);
    md.ctl2m.assign((size_t)nl * nl, 0.0);
    md.ctm2l.assign((size_t)nl * nl, 0.0);
    for (int m = 0; m < nl; ++m) {
        const int im = idx[m];
        double eld = 0.0;
        for (int k = 0; k < nl; ++k) eld += L[k + nl * im] * R[k + nl * im];
        for (int k = 0; k < nl; ++k) {
            md.ctl2m[k + nl * m] = L[k + nl * im] / eld;   // ctl2m(k, m)
            md.ctm2l[m + nl * k] = R[k + nl * im];         // ctm2l(m, k)
        }
    }
    // identity check of the conversion matrices (modes.F90:148-161)
    for (int l = 0; l < nl; ++l)
        for (int k = 0; k < nl; ++k) {
            double s = 0.0;
            for (int m = 0; m < nl; ++m) s += md.ctm2l[m + nl * k] * md.ctl2m[l + nl * m];
            const double want = (k == l) ? 1.0 : 0.0;
            if (std::fabs(s - want) > 5.0e-15) {
                char buf[128];
                snprintf(buf, sizeof buf, "mode matrices: ccprod(%d,%d) = %.17g is not the identity", k + 1,
                         l + 1, s);
                err = buf;
                return false;
            }
        }
    return true;
}

void setup_pivots(bool cyclic, int nxp, int nyp, double dx, double dy,
                  const std::vector<double> &rdm2, PivotTable &pt, double &a_tri) {
    const double PI = 3.14159265358979324, TWOPI = 2.0 * PI;
    int nk, N;
    if (cyclic) { N = nxp - 1; nk = N / 2 + 1; }
    else { nk = nxp - 2; N = 2 * (nk + 1); }
    const int nl = (int)rdm2.size(), ny = nyp - 2;
    const double a = 1.0 / (dy * dy);
    const double dxm2 = 1.0 / (dx * dx);
    a_tri = a;
    pt.tab.clear();
    pt.off.assign((size_t)nl * nk, 0);
    pt.len.assign((size_t)nl * nk, 0);
    for (int m = 0; m < nl; ++m)
        for (int i = 1; i <= nk; ++i) {
            double bd2 = cyclic ? -2.0 * a + 2.0 * dxm2 * (std::cos((i - 1) * TWOPI / N) - 1.0)
                                : -2.0 * a + 2.0 * dxm2 * (std::cos(i * TWOPI / N) - 1.0);
            const double bb = bd2 - rdm2[m];
            const int p = m * nk + (i - 1);
            pt.off[p] = (int)pt.tab.size();
            double betinv = 1.0 / bb;
            pt.tab.push_back(betinv);
            for (int j = 1; j < ny; ++j) {
                const double gam = a * betinv;
                const double nb = 1.0 / (bb - a * gam);
                if (nb == betinv) break;   // fixed point: the rest repeat it
                betinv = nb;
                pt.tab.push_back(betinv);
            }
            pt.len[p] = (int)pt.tab.size() - pt.off[p];
        }
}

bool fft_radices(int M, std::vector<int> &rad) {
    rad.clear();
    int m = M;
    while (m % 16 == 0) { rad.push_back(16); m /= 16; }
    while (m % 8 == 0) { rad.push_back(8); m /= 8; }
    while (m % 4 == 0) { rad.push_back(4); m /= 4; }
    while (m % 2 == 0) { rad.push_back(2); m /= 2; }
    while (m % 3 == 0) { rad.push_back(3); m /= 3; }
    while (m % 5 == 0) { rad.push_back(5); m /= 5; }
    return m == 1;
}

void fft_stage_twiddles(int M, const std::vector<int> &rad, std::vector<double> &tw) {
    tw.assign(2 * (size_t)std::max(M, 1), 0.0);
    const long double pi = 3.14159265358979323846264338327950288L;
    long long Ns = 1;
    for (int R : rad) {
        // stage of radix R after Ns: entries (jm, r) at Ns-1 + (r-1) Ns + jm, so
        // the butterflies of a warp (consecutive jm) read consecutive entries
        for (long long jm = 0; jm < Ns; ++jm)
            for (int r = 1; r < R; ++r) {
                const long long k = (long long)r * jm;       // exponent k / (Ns R)
                const long double ang = -2.0L * pi * (long double)(k % (Ns * R)) / (long double)(Ns * R);
                const size_t e = (size_t)(Ns - 1 + (r - 1) * Ns + jm);
                tw[2 * e] = (double)cosl(ang);
                tw[2 * e + 1] = (double)sinl(ang);
            }
        Ns *= R;
    }
}

void dst_row_sums(int n, std::vector<double> &w) {
    const long double pi = 3.14159265358979323846264338327950288L;
    w.resize(n);
    for (int k = 1; k <= n; ++k) {
        long double s = 0.0L;
        for (int i = 1; i <= n; ++i) {
            long long r = ((long long)i * k) % (2 * (n + 1));
            s += sinl(pi * (long double)r / (long double)(n + 1));
        }
        w[k - 1] = (double)(2.0L * s);
    }
}

bool lu_factor(int n, const double *A, double *LU, int *piv) {
    std::copy(A, A + (size_t)n * n, LU);
    for (int c = 0; c < n; ++c) {
        int p = c;
        double mx = std::fabs(LU[c + n * c]);
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(LU[r + n * c]) > mx) { mx = std::fabs(LU[r + n * c]); p = r; }
        piv[c] = p;
        if (LU[p + n * c] == 0.0) return false;
        if (p != c)
            for (int k = 0; k < n; ++k) std::swap(LU[c + n * k], LU[p + n * k]);
        const double inv = 1.0 / LU[c + n * c];
        for (int r = c + 1; r < n; ++r) LU[r + n * c] *= inv;
        for (int k = c + 1; k < n; ++k)
            for (int r = c + 1; r < n; ++r) LU[r + n * k] -= LU[r + n * c] * LU[c + n * k];
    }
    return true;
}

}  // namespace oqg
