// oqg_oracle.cpp -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
//
// CPU FP64 restatement of OpenQG's per-timestep QG core (BreakawayLabs/openqg,
// Fortran 90), used as the parity oracle by tests/, by __graft_entry__.smoke()
// and as the timed CPU baseline of bench.py.  Nothing in openqg_b200/ links or
// calls this file.
//
// It follows the reference loop by loop, with full-array temporaries like the
// Fortran (function results), FP64 throughout, and the reference's evaluation
// order for each expression.  Each routine cites the Fortran it restates.
// The reference's two external libraries are replaced by own code:
//   * FFTW3 (fftw_plan_many_r2r RODFT00, fftw_plan_many_dft_r2c / c2r;
//     qg/inhomog.F90:103-122, system libfftw3, version unpinned) -> a
//     mixed-radix Stockham FFT; DST-I by the odd extension of length 2(n+1),
//     two rows per complex transform; r2c/c2r by packing two rows.
//   * LAPACK (DGEEVX, DGETRF, DGETRS, DGERFS; util/linalg.F90:24-122, system
//     liblapack, version unpinned) -> Jacobi on the symmetrised mode matrix
//     and a partially pivoted LU with DGERFS-style iterative refinement.
// Parity pins (tests/test_oracle_*.py): the reference's own Helmholtz residual
// tests (src/tests/test_inhomog.F90:123-154, 208-240), the mode-matrix identity
// check (qg/modes.F90:148-161), an O(n^2) long-double DST, Arakawa-Jacobian
// conservation, and mass-constraint closure.  There are no golden vectors in
// the reference for the step itself, so bitwise FFTW/LAPACK parity is unpinned.
//
// Only the region the reference parallelises is parallel here: the leapfrog
// update (qg/vorticity.F90:67-82, !$OMP PARALLEL WORKSHARE).

#include "../include/oqg.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace orc {

typedef std::complex<double> cd;
static const double PI = 3.14159265358979324;   // constants.F90:14
static const double TWOPI = 2.0 * PI;

// ---------------------------------------------------------------- box
// glam/box.F90:11-41, compute_derived_values :126-163
struct Box {
    int nxp, nyp, nl;
    bool cyclic;
    double dx, dy, fnot, beta;
    int dz_sign;
    std::vector<double> h, yp, yprel;
    double xl, yl, dxm2;
};

static Box make_box(const oqg_params &p) {
    Box b;
    b.nxp = p.nxp; b.nyp = p.nyp; b.nl = p.nl;
    b.cyclic = p.cyclic != 0;
    b.dx = p.dx; b.dy = p.dy; b.fnot = p.fnot; b.beta = p.beta;
    b.dz_sign = p.dz_sign;
    b.h.assign(p.h, p.h + p.nl);
    int nxt = b.nxp - 1, nyt = b.nyp - 1;
    b.xl = nxt * b.dx;
    b.yl = nyt * b.dy;
    b.dxm2 = 1.0 / (b.dx * b.dx);
    b.yp.resize(b.nyp);
    b.yprel.resize(b.nyp);
    for (int j = 0; j < b.nyp; ++j) {
        b.yp[j] = 0.0 + j * b.dy;
        b.yprel[j] = -0.5 * b.yl + j * b.dy;
    }
    return b;
}

// ---------------------------------------------------------------- numerics
// glam/numerics.F90.  2-D arrays are (nxp, nyp) column-major.
#define IX(i, j) ((i) + nxp * (j))

// int_P_dA_2d, numerics.F90:188-204 (Fortran sum order: i fastest)
static double int_P_dA(const Box &b, const double *f) {
    const int nxp = b.nxp, nyp = b.nyp;
    double s = 0.0;
    for (int j = 0; j < nyp; ++j)
        for (int i = 0; i < nxp; ++i) s += f[IX(i, j)];
    double s1 = 0.0, s2 = 0.0;
    for (int i = 0; i < nxp; ++i) s1 += f[IX(i, 0)];
    for (int i = 0; i < nxp; ++i) s2 += f[IX(i, nyp - 1)];
    s = s - 0.5 * (s1 + s2);
    double s3 = 0.0, s4 = 0.0;
    for (int j = 0; j < nyp; ++j) s3 += f[IX(0, j)];
    for (int j = 0; j < nyp; ++j) s4 += f[IX(nxp - 1, j)];
    s = s - 0.5 * (s3 + s4);
    s = s + 0.25 * (f[IX(0, 0)] + f[IX(0, nyp - 1)] + f[IX(nxp - 1, 0)] +
                    f[IX(nxp - 1, nyp - 1)]);
    return s * b.dx * b.dy;
}

// int_P_dx, numerics.F90:206-212; row with unit stride
static double int_P_dx(const Box &b, const double *row) {
    double s = 0.0;
    for (int i = 1; i < b.nxp - 1; ++i) s += row[i];
    return (0.5 * row[0] + s + 0.5 * row[b.nxp - 1]) * b.dx;
}

// dPdx_2, numerics.F90:311-325
static void dPdx_2(const Box &b, const double *p, double *o) {
    const int nxp = b.nxp, nyp = b.nyp;
    for (int j = 0; j < nyp; ++j) {
        for (int i = 1; i < nxp - 1; ++i) o[IX(i, j)] = p[IX(i + 1, j)] - p[IX(i - 1, j)];
        o[IX(0, j)] = b.cyclic ? p[IX(1, j)] - p[IX(nxp - 2, j)] : 0.0;
        o[IX(nxp - 1, j)] = o[IX(0, j)];
    }
}

// dPdy_2, numerics.F90:327-338
static void dPdy_2(const Box &b, const double *p, double *o) {
    const int nxp = b.nxp, nyp = b.nyp;
    for (int i = 0; i < nxp; ++i) o[IX(i, 0)] = 0.0;
    for (int j = 1; j < nyp - 1; ++j)
        for (int i = 0; i < nxp; ++i) o[IX(i, j)] = p[IX(i, j + 1)] - p[IX(i, j - 1)];
    for (int i = 0; i < nxp; ++i) o[IX(i, nyp - 1)] = 0.0;
}

// jacobian, numerics.F90:340-388 (one layer); ajis/ajin for the channel
static void jacobian2d(const Box &b, const double *p, const double *q, double *jac,
                       double *ajis, double *ajin) {
    const int nxp = b.nxp, nyp = b.nyp, n = nxp * nyp;
    double fac = 1.0 / (3.0 * (2.0 * b.dx) * (2.0 * b.dy) * b.fnot);
    std::vector<double> dpx(n), dpy(n), dqx(n), dqy(n), t(n), A(n), B(n), C(n), D(n);
    dPdx_2(b, p, dpx.data());
    dPdy_2(b, p, dpy.data());
    dPdx_2(b, q, dqx.data());
    dPdy_2(b, q, dqy.data());
    for (int x = 0; x < n; ++x) t[x] = q[x] * dpy[x];
    dPdx_2(b, t.data(), A.data());
    for (int x = 0; x < n; ++x) t[x] = q[x] * dpx[x];
    dPdy_2(b, t.data(), B.data());
    for (int x = 0; x < n; ++x) t[x] = p[x] * dqx[x];
    dPdy_2(b, t.data(), C.data());
    for (int x = 0; x < n; ++x) t[x] = p[x] * dqy[x];
    dPdx_2(b, t.data(), D.data());
    for (int x = 0; x < n; ++x)
        jac[x] = fac * (dqx[x] * dpy[x] - dqy[x] * dpx[x] + A[x] - B[x] + C[x] - D[x]);
    if (b.cyclic && ajis && ajin) {
        std::vector<double> r(nxp);
        for (int i = 0; i < nxp; ++i) r[i] = q[IX(i, 0)] * dpx[IX(i, 1)];
        double aj5sms = int_P_dx(b, r.data()) / (2.0 * b.dx);
        for (int i = 0; i < nxp; ++i) r[i] = q[IX(i, 1)] * dpx[IX(i, 1)];
        double aj9sms = int_P_dx(b, r.data()) / (2.0 * b.dx);
        *ajis = (aj5sms + 2.0 * aj9sms) / 6.0;
        for (int i = 0; i < nxp; ++i) r[i] = q[IX(i, nyp - 1)] * dpx[IX(i, nyp - 2)];
        double aj5smn = int_P_dx(b, r.data()) / (2.0 * b.dx);
        for (int i = 0; i < nxp; ++i) r[i] = q[IX(i, nyp - 2)] * dpx[IX(i, nyp - 2)];
        double aj9smn = int_P_dx(b, r.data()) / (2.0 * b.dx);
        *ajin = -(aj5smn + 2.0 * aj9smn) / 6.0;
    }
}

// dP2dx2_bc, numerics.F90:427-448
static void dP2dx2_bc(const Box &b, const double *p, double alpha, double *o) {
    const int nxp = b.nxp, nyp = b.nyp;
    double fac = 1.0 / (b.dx * b.dx);
    for (int j = 0; j < nyp; ++j) {
        for (int i = 1; i < nxp - 1; ++i)
            o[IX(i, j)] = fac * (p[IX(i - 1, j)] + p[IX(i + 1, j)] - 2.0 * p[IX(i, j)]);
        if (!b.cyclic) {
            o[IX(0, j)] = fac * alpha / (0.5 * alpha + 1.0) * (p[IX(1, j)] - p[IX(0, j)]);
            o[IX(nxp - 1, j)] =
                -fac * alpha / (0.5 * alpha + 1.0) * (p[IX(nxp - 1, j)] - p[IX(nxp - 2, j)]);
        } else {
            o[IX(0, j)] = fac * (p[IX(nxp - 2, j)] + p[IX(1, j)] - 2.0 * p[IX(0, j)]);
            o[IX(nxp - 1, j)] = o[IX(0, j)];
        }
    }
    for (int i = 0; i < nxp; ++i) { o[IX(i, 0)] = 0.0; o[IX(i, nyp - 1)] = 0.0; }
}

// dP2dy2_bc, numerics.F90:450-468
static void dP2dy2_bc(const Box &b, const double *p, double alpha, double *o) {
    const int nxp = b.nxp, nyp = b.nyp;
    double fac = 1.0 / (b.dy * b.dy);
    for (int j = 1; j < nyp - 1; ++j)
        for (int i = 0; i < nxp; ++i)
            o[IX(i, j)] = fac * (p[IX(i, j - 1)] + p[IX(i, j + 1)] - 2.0 * p[IX(i, j)]);
    for (int i = 0; i < nxp; ++i) {
        o[IX(i, 0)] = fac * alpha / (0.5 * alpha + 1.0) * (p[IX(i, 1)] - p[IX(i, 0)]);
        o[IX(i, nyp - 1)] =
            -fac * alpha / (0.5 * alpha + 1.0) * (p[IX(i, nyp - 1)] - p[IX(i, nyp - 2)]);
    }
    if (!b.cyclic)
        for (int j = 0; j < nyp; ++j) { o[IX(0, j)] = 0.0; o[IX(nxp - 1, j)] = 0.0; }
}

// del2_P_bc, numerics.F90:410-425 (one layer)
static void del2_bc(const Box &b, const double *p, double alpha, double *o) {
    int n = b.nxp * b.nyp;
    std::vector<double> X(n), Y(n);
    dP2dx2_bc(b, p, alpha, X.data());
    dP2dy2_bc(b, p, alpha, Y.data());
    for (int x = 0; x < n; ++x) o[x] = X[x] + Y[x];
}

// dPdx_2bc / dPdy_2bc, numerics.F90:470-513
static void dPdx_2bc(const Box &b, const double *p, double alpha, double *o) {
    const int nxp = b.nxp, nyp = b.nyp;
    for (int j = 0; j < nyp; ++j) {
        for (int i = 1; i < nxp - 1; ++i)
            o[IX(i, j)] = (p[IX(i + 1, j)] - p[IX(i - 1, j)]) / (2.0 * b.dx);
        if (!b.cyclic) {
            o[IX(0, j)] = (p[IX(1, j)] - p[IX(0, j)]) / (b.dx * (0.5 * alpha + 1.0));
            o[IX(nxp - 1, j)] =
                (p[IX(nxp - 1, j)] - p[IX(nxp - 2, j)]) / (b.dx * (0.5 * alpha + 1.0));
        } else {
            o[IX(0, j)] = (p[IX(1, j)] - p[IX(nxp - 2, j)]) / (2.0 * b.dx);
            o[IX(nxp - 1, j)] = o[IX(0, j)];
        }
    }
    for (int i = 0; i < nxp; ++i) { o[IX(i, 0)] = 0.0; o[IX(i, nyp - 1)] = 0.0; }
}
static void dPdy_2bc(const Box &b, const double *p, double alpha, double *o) {
    const int nxp = b.nxp, nyp = b.nyp;
    for (int j = 1; j < nyp - 1; ++j)
        for (int i = 0; i < nxp; ++i)
            o[IX(i, j)] = (p[IX(i, j + 1)] - p[IX(i, j - 1)]) / (2.0 * b.dy);
    for (int i = 0; i < nxp; ++i) {
        o[IX(i, 0)] = (p[IX(i, 1)] - p[IX(i, 0)]) / (b.dy * (0.5 * alpha + 1.0));
        o[IX(i, nyp - 1)] = (p[IX(i, nyp - 1)] - p[IX(i, nyp - 2)]) / (b.dy * (0.5 * alpha + 1.0));
    }
    if (!b.cyclic)
        for (int j = 0; j < nyp; ++j) { o[IX(0, j)] = 0.0; o[IX(nxp - 1, j)] = 0.0; }
}

// map_T_to_P, numerics.F90:64-107; t is (nxp-1, nyp-1)
static void map_T_to_P(const Box &b, const double *t, double *o) {
    const int nxp = b.nxp, nyp = b.nyp, nxt = nxp - 1;
#define TX(i, j) t[(i) + nxt * (j)]
    for (int j = 1; j < nyp - 1; ++j)
        for (int i = 1; i < nxp - 1; ++i)
            o[IX(i, j)] = 0.25 * (TX(i, j) + TX(i - 1, j) + TX(i, j - 1) + TX(i - 1, j - 1));
    for (int i = 1; i < nxp - 1; ++i) {
        o[IX(i, 0)] = 0.5 * (TX(i - 1, 0) + TX(i, 0));
        o[IX(i, nyp - 1)] = 0.5 * (TX(i - 1, nyp - 2) + TX(i, nyp - 2));
    }
    if (b.cyclic) {
        for (int j = 1; j < nyp - 1; ++j) {
            o[IX(0, j)] = 0.25 * (TX(0, j) + TX(nxp - 2, j) + TX(0, j - 1) + TX(nxp - 2, j - 1));
            o[IX(nxp - 1, j)] = o[IX(0, j)];
        }
        o[IX(0, 0)] = 0.5 * (TX(0, 0) + TX(nxp - 2, 0));
        o[IX(0, nyp - 1)] = 0.5 * (TX(0, nyp - 2) + TX(nxp - 2, nyp - 2));
        o[IX(nxp - 1, 0)] = o[IX(0, 0)];
        o[IX(nxp - 1, nyp - 1)] = o[IX(0, nyp - 1)];
    } else {
        for (int j = 1; j < nyp - 1; ++j) {
            o[IX(0, j)] = 0.5 * (TX(0, j - 1) + TX(0, j));
            o[IX(nxp - 1, j)] = 0.5 * (TX(nxp - 2, j - 1) + TX(nxp - 2, j));
        }
        o[IX(0, 0)] = TX(0, 0);
        o[IX(nxp - 1, 0)] = TX(nxp - 2, 0);
        o[IX(0, nyp - 1)] = TX(0, nyp - 2);
        o[IX(nxp - 1, nyp - 1)] = TX(nxp - 2, nyp - 2);
    }
#undef TX
}

// ---------------------------------------------------------------- FFT
// Mixed-radix Stockham autosort FFT (forward, e^{-2 pi i jk/n}), in place of
// FFTW.  Radices 4, 2, 3, 5 and a direct DFT for any other prime factor.
struct FFT {
    int n;
    std::vector<int> rad;
    std::vector<cd> tw;  // tw[t] = exp(-2 pi i t / n)
    explicit FFT(int n_) : n(n_) {
        int m = n;
        while (m % 4 == 0) { rad.push_back(4); m /= 4; }
        while (m % 2 == 0) { rad.push_back(2); m /= 2; }
        for (int p = 3; m > 1; p += 2)
            while (m % p == 0) { rad.push_back(p); m /= p; }
        tw.resize(n);
        for (int t = 0; t < n; ++t) {
            long double a = -2.0L * 3.14159265358979323846264338327950288L * t / n;
            tw[t] = cd((double)cosl(a), (double)sinl(a));
        }
    }
    // x: n complex in/out; y: n complex scratch
    void exec(cd *x, cd *y) const {
        cd *a = x, *b = y;
        int Ns = 1;
        std::vector<cd> v;
        for (int R : rad) {
            v.resize(R);
            int stride = n / R;
            int tstep = n / (Ns * R);
            for (int j = 0; j < n / R; ++j) {
                int jm = j % Ns;
                v[0] = a[j];
                for (int r = 1; r < R; ++r) v[r] = a[j + r * stride] * tw[(r * jm * tstep) % n];
                dft(R, v.data());
                int idxD = (j / Ns) * Ns * R + jm;
                for (int r = 0; r < R; ++r) b[idxD + r * Ns] = v[r];
            }
            std::swap(a, b);
            Ns *= R;
        }
        if (a != x) std::copy(a, a + n, x);
    }
    void dft(int R, cd *v) const {
        if (R == 2) {
            cd t = v[0];
            v[0] = t + v[1];
            v[1] = t - v[1];
        } else if (R == 4) {
            cd t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3];
            cd d = v[1] - v[3];
            cd t3(d.imag(), -d.real());  // (v1 - v3) * (-i)
            v[0] = t0 + t2; v[1] = t1 + t3; v[2] = t0 - t2; v[3] = t1 - t3;
        } else if (R == 3) {
            const double s3 = 0.86602540378443864676;
            cd s = v[1] + v[2], d = v[1] - v[2];
            cd m = v[0] - 0.5 * s;
            cd jd(d.imag() * s3, -d.real() * s3);  // -i * s3 * d
            v[0] = v[0] + s;
            v[1] = m + jd;
            v[2] = m - jd;
        } else {
            std::vector<cd> o(R);
            int base = n / R;
            for (int k = 0; k < R; ++k) {
                cd acc = v[0];
                for (int r = 1; r < R; ++r) acc += v[r] * tw[((r * k) % R) * base];
                o[k] = acc;
            }
            for (int k = 0; k < R; ++k) v[k] = o[k];
        }
    }
};

struct FFTCache {
    std::map<int, std::unique_ptr<FFT>> plans;
    const FFT &get(int n) {
        auto it = plans.find(n);
        if (it == plans.end()) it = plans.emplace(n, std::unique_ptr<FFT>(new FFT(n))).first;
        return *it->second;
    }
};
static FFTCache g_fft;

// DST-I with FFTW RODFT00 semantics: Y_k = 2 sum_j X_j sin(pi (j+1)(k+1)/(n+1)),
// for `howmany` rows of length n (row stride n).
static void dst1(int n, int howmany, const double *in, double *out) {
    int M = 2 * (n + 1);
    const FFT &f = g_fft.get(M);
    std::vector<cd> z(M), w(M);
    for (int r = 0; r < howmany; r += 2) {
        const double *x = in + (size_t)r * n;
        const double *y = (r + 1 < howmany) ? in + (size_t)(r + 1) * n : nullptr;
        z[0] = 0.0;
        z[n + 1] = 0.0;
        for (int j = 1; j <= n; ++j) {
            cd v(x[j - 1], y ? y[j - 1] : 0.0);
            z[j] = v;
            z[M - j] = -v;
        }
        f.exec(z.data(), w.data());
        double *ox = out + (size_t)r * n;
        double *oy = y ? out + (size_t)(r + 1) * n : nullptr;
        for (int k = 1; k <= n; ++k) {
            ox[k - 1] = -z[k].imag();
            if (oy) oy[k - 1] = z[k].real();
        }
    }
}

// r2c with FFTW semantics: X_k = sum_j x_j e^{-2 pi i jk/N}, k = 0..N/2
static void rfft(int N, int howmany, const double *in, cd *out) {
    const FFT &f = g_fft.get(N);
    int no = N / 2 + 1;
    std::vector<cd> z(N), w(N);
    for (int r = 0; r < howmany; r += 2) {
        const double *x = in + (size_t)r * N;
        const double *y = (r + 1 < howmany) ? in + (size_t)(r + 1) * N : nullptr;
        for (int j = 0; j < N; ++j) z[j] = cd(x[j], y ? y[j] : 0.0);
        f.exec(z.data(), w.data());
        cd *ox = out + (size_t)r * no;
        cd *oy = y ? out + (size_t)(r + 1) * no : nullptr;
        for (int k = 0; k < no; ++k) {
            cd a = z[k], c = std::conj(z[(N - k) % N]);
            ox[k] = 0.5 * (a + c);
            if (oy) {
                cd d = 0.5 * (a - c);
                oy[k] = cd(d.imag(), -d.real());  // d / i
            }
        }
    }
}

// c2r with FFTW semantics: x_j = sum_{k=0}^{N-1} X_k e^{+2 pi i jk/N} with the
// Hermitian extension; imaginary parts of X_0 and X_{N/2} are ignored.
static void irfft(int N, int howmany, const cd *in, double *out) {
    const FFT &f = g_fft.get(N);
    int no = N / 2 + 1;
    std::vector<cd> z(N), w(N), X(N), Y(N);
    for (int r = 0; r < howmany; r += 2) {
        const cd *x = in + (size_t)r * no;
        const cd *y = (r + 1 < howmany) ? in + (size_t)(r + 1) * no : nullptr;
        for (int k = 0; k < no; ++k) { X[k] = x[k]; Y[k] = y ? y[k] : cd(0.0); }
        X[0] = X[0].real(); Y[0] = Y[0].real();
        if (N % 2 == 0) { X[N / 2] = X[N / 2].real(); Y[N / 2] = Y[N / 2].real(); }
        for (int k = no; k < N; ++k) { X[k] = std::conj(X[N - k]); Y[k] = std::conj(Y[N - k]); }
        // inverse transform of Z = X + iY via conj(FFT(conj(Z)))
        for (int k = 0; k < N; ++k) z[k] = std::conj(X[k] + cd(-Y[k].imag(), Y[k].real()));
        f.exec(z.data(), w.data());
        double *ox = out + (size_t)r * N;
        double *oy = y ? out + (size_t)(r + 1) * N : nullptr;
        for (int j = 0; j < N; ++j) {
            cd v = std::conj(z[j]);
            ox[j] = v.real();
            if (oy) oy[j] = v.imag();
        }
    }
}

// ---------------------------------------------------------------- linalg
// LU_factor (linalg.F90:24-55, DGETRF) and solve_Ax_b (:57-93, DGETRS+DGERFS)
struct LU {
    int n = 0;
    std::vector<double> A, F;  // column-major original and factors
    std::vector<int> piv;
};

static bool lu_factor(LU &lu) {
    int n = lu.n;
    lu.F = lu.A;
    lu.piv.assign(n, 0);
    double *a = lu.F.data();
    for (int c = 0; c < n; ++c) {
        int p = c;
        double mx = std::fabs(a[c + n * c]);
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[r + n * c]) > mx) { mx = std::fabs(a[r + n * c]); p = r; }
        lu.piv[c] = p;
        if (a[p + n * c] == 0.0) return false;
        if (p != c)
            for (int k = 0; k < n; ++k) std::swap(a[c + n * k], a[p + n * k]);
        double inv = 1.0 / a[c + n * c];
        for (int r = c + 1; r < n; ++r) a[r + n * c] *= inv;
        for (int k = c + 1; k < n; ++k)
            for (int r = c + 1; r < n; ++r) a[r + n * k] -= a[r + n * c] * a[c + n * k];
    }
    return true;
}

static void lu_solve(const LU &lu, double *x) {
    int n = lu.n;
    const double *a = lu.F.data();
    for (int i = 0; i < n; ++i)
        if (lu.piv[i] != i) std::swap(x[i], x[lu.piv[i]]);
    for (int c = 0; c < n; ++c)
        for (int r = c + 1; r < n; ++r) x[r] -= x[c] * a[r + n * c];
    for (int c = n - 1; c >= 0; --c) {
        x[c] /= a[c + n * c];
        for (int r = 0; r < c; ++r) x[r] -= x[c] * a[r + n * c];
    }
}

// DGETRS followed by the DGERFS refinement loop (ITMAX = 5)
static void solve_Ax_b(const LU &lu, const double *b, double *x) {
    int n = lu.n;
    const double *A = lu.A.data();
    for (int i = 0; i < n; ++i) x[i] = b[i];
    lu_solve(lu, x);
    const double eps = std::ldexp(1.0, -53);
    const double safmin = 2.2250738585072014e-308;
    const double safe1 = (n + 1) * safmin, safe2 = safe1 / eps;
    double lstres = 3.0;
    int count = 1;
    std::vector<double> r(n), w(n);
    for (;;) {
        for (int i = 0; i < n; ++i) r[i] = b[i];
        for (int j = 0; j < n; ++j) {
            double t = -x[j];
            for (int i = 0; i < n; ++i) r[i] += t * A[i + n * j];
        }
        for (int i = 0; i < n; ++i) w[i] = std::fabs(b[i]);
        for (int j = 0; j < n; ++j) {
            double xk = std::fabs(x[j]);
            for (int i = 0; i < n; ++i) w[i] += std::fabs(A[i + n * j]) * xk;
        }
        double s = 0.0;
        for (int i = 0; i < n; ++i) {
            if (w[i] > safe2) s = std::max(s, std::fabs(r[i]) / w[i]);
            else s = std::max(s, (std::fabs(r[i]) + safe1) / (w[i] + safe1));
        }
        if (s > eps && 2.0 * s <= lstres && count <= 5) {
            lu_solve(lu, r.data());
            for (int i = 0; i < n; ++i) x[i] += r[i];
            lstres = s;
            ++count;
        } else {
            break;
        }
    }
}

// Symmetric eigenproblem by cyclic Jacobi; S column-major n x n, V columns.
static void jacobi_eig(int n, std::vector<double> S, std::vector<double> &w, std::vector<double> &V) {
    V.assign(n * n, 0.0);
    for (int i = 0; i < n; ++i) V[i + n * i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int c = 0; c < n; ++c)
            for (int r = 0; r < n; ++r)
                if (r != c) off += S[r + n * c] * S[r + n * c];
        if (off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = S[p + n * q];
                if (apq == 0.0) continue;
                double app = S[p + n * p], aqq = S[q + n * q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    double skp = S[k + n * p], skq = S[k + n * q];
                    S[k + n * p] = c * skp - s * skq;
                    S[k + n * q] = s * skp + c * skq;
                }
                for (int k = 0; k < n; ++k) {
                    double spk = S[p + n * k], sqk = S[q + n * k];
                    S[p + n * k] = c * spk - s * sqk;
                    S[q + n * k] = s * spk + c * sqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[k + n * p], vkq = V[k + n * q];
                    V[k + n * p] = c * vkp - s * vkq;
                    V[k + n * q] = s * vkp + c * vkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = S[i + n * i];
}

// ---------------------------------------------------------------- the model
struct Model {
    Box b;
    oqg_params prm;
    double bcco, delek, rho;
    int tau_sign, k_topo;  // k_topo 0-based
    std::vector<double> ah2, ah4, gp, ddyn;
    // modes (modes.F90:11-23), column-major nl x nl
    std::vector<double> amat, ctl2m, ctm2l, rdm2;
    // inhomog (inhomog.F90:41-62)
    int nx_tab = 0, Nlog = 0;
    double ftnorm = 0, a_tri = 0;
    std::vector<double> bb;  // (nx_tab, nl)
    // homog box (homog.F90:272-286)
    std::vector<double> hom_sol_bc;  // (nxp,nyp) per mode m=1..nl-1 (index m-1)
    LU cd_lu;
    // homog cyclic (homog.F90:288-311)
    std::vector<double> hom_sol_bt, hbc1, hbc2;  // (nyp), (nyp, nl)
    std::vector<double> hc1s, hc2s, hc1n, hc2n;
    double hbsi = 0;
    // state
    std::vector<double> p, pm, q, qm;
    std::vector<double> dpi, dpip;
    std::vector<double> cs, cn, csp, cnp, ajis, ajin, ap3s, ap3n, ap5s, ap5n, int_Be_s, int_Be_n;
    double bdrins = 0, bdrinn = 0, txis = 0, txin = 0;
    // forcing
    std::vector<double> wekp, ent;  // ent (nxp, nyp, nl-1)
    long long nt = 0;
    int suppress_period = 0;
    std::string err;

    size_t n2() const { return (size_t)b.nxp * b.nyp; }
    size_t n3() const { return n2() * b.nl; }
};

// compute_A, modes.F90:221-246
static void compute_A(Model &M) {
    int nl = M.b.nl;
    M.amat.assign(nl * nl, 0.0);
#define AM(r, c) M.amat[(r) + nl * (c)]
    const std::vector<double> &h = M.b.h, &g = M.gp;
    AM(0, 1) = -1.0 / (g[0] * h[0]);
    AM(0, 0) = -AM(0, 1);
    for (int k = 1; k < nl - 1; ++k) {
        AM(k, k - 1) = -1.0 / (g[k - 1] * h[k]);
        AM(k, k + 1) = -1.0 / (g[k] * h[k]);
        AM(k, k) = -AM(k, k - 1) - AM(k, k + 1);
    }
    AM(nl - 1, nl - 2) = -1.0 / (g[nl - 2] * h[nl - 1]);
    AM(nl - 1, nl - 1) = -AM(nl - 1, nl - 2);
#undef AM
}

// eigmod + derive_qg_modes, modes.F90:46-219
static bool eigmod(Model &M) {
    int nl = M.b.nl;
    compute_A(M);
    // A = H^-1 T with T symmetric: S = H^1/2 A H^-1/2 is symmetric.
    std::vector<double> S(nl * nl), w, V;
    for (int c = 0; c < nl; ++c)
        for (int r = 0; r < nl; ++r)
            S[r + nl * c] = std::sqrt(M.b.h[r]) * M.amat[r + nl * c] / std::sqrt(M.b.h[c]);
    for (int c = 0; c < nl; ++c)  // exact symmetry
        for (int r = c + 1; r < nl; ++r) {
            double v = 0.5 * (S[r + nl * c] + S[c + nl * r]);
            S[r + nl * c] = S[c + nl * r] = v;
        }
    jacobi_eig(nl, S, w, V);
    std::vector<double> evr(nl * nl), evl(nl * nl);
    for (int m = 0; m < nl; ++m) {
        double nr = 0, nlf = 0;
        for (int k = 0; k < nl; ++k) {
            evr[k + nl * m] = V[k + nl * m] / std::sqrt(M.b.h[k]);
            evl[k + nl * m] = V[k + nl * m] * std::sqrt(M.b.h[k]);
            nr += evr[k + nl * m] * evr[k + nl * m];
            nlf += evl[k + nl * m] * evl[k + nl * m];
        }
        nr = std::sqrt(nr);
        nlf = std::sqrt(nlf);
        // unit 2-norm (as DGEEVX); sign: largest component positive
        int kb = 0;
        for (int k = 1; k < nl; ++k)
            if (std::fabs(evr[k + nl * m]) > std::fabs(evr[kb + nl * m])) kb = k;
        double sg = evr[kb + nl * m] < 0 ? -1.0 : 1.0;
        for (int k = 0; k < nl; ++k) {
            evr[k + nl * m] *= sg / nr;
            evl[k + nl * m] *= sg / nlf;
        }
    }
    // ordering by |eigenvalue| (insertion sort, modes.F90:99-115)
    std::vector<double> c2rabs(nl);
    std::vector<int> index(nl);
    for (int m = 0; m < nl; ++m) { c2rabs[m] = std::fabs(w[m]); index[m] = m; }
    for (int m = 1; m < nl; ++m) {
        int indtmp = index[m];
        double c2temp = c2rabs[indtmp];
        int i = m - 1;
        for (; i >= 0; --i) {
            if (c2rabs[index[i]] <= c2temp) break;
            index[i + 1] = index[i];
        }
        index[i + 1] = indtmp;
    }
    M.rdm2.assign(nl, 0.0);
    for (int m = 1; m < nl; ++m) M.rdm2[m] = M.b.fnot * M.b.fnot * c2rabs[index[m]];
    std::vector<double> elder(nl * nl);
    for (int n = 0; n < nl; ++n)
        for (int m = 0; m < nl; ++m) {
            double s = 0;
            for (int k = 0; k < nl; ++k) s += evl[k + nl * m] * evr[k + nl * n];
            elder[m + nl * n] = s;
        }
    M.ctl2m.assign(nl * nl, 0.0);
    M.ctm2l.assign(nl * nl, 0.0);
    std::vector<double> cl2m(nl * nl), cm2l(nl * nl);
    for (int m = 0; m < nl; ++m) {
        int inm = index[m];
        for (int k = 0; k < nl; ++k) {
            cl2m[m + nl * k] = evl[k + nl * inm] / elder[inm + nl * inm];
            M.ctl2m[k + nl * m] = cl2m[m + nl * k];
            cm2l[k + nl * m] = evr[k + nl * inm];
            M.ctm2l[m + nl * k] = cm2l[k + nl * m];
        }
    }
    for (int l = 0; l < nl; ++l)
        for (int k = 0; k < nl; ++k) {
            double s = 0;
            for (int m = 0; m < nl; ++m) s += cm2l[k + nl * m] * cl2m[m + nl * l];
            double target = (k == l) ? 1.0 : 0.0;
            if (std::fabs(s - target) > 5.0e-15) {
                char buf[160];
                snprintf(buf, sizeof buf, "ccprod - Not identity %d %d %.17g", k + 1, l + 1, s);
                M.err = buf;
                return false;
            }
        }
    return true;
}

// init_inhomog, inhomog.F90:71-144
static void init_inhomog(Model &M) {
    const Box &b = M.b;
    int n_in, n_out, N;
    if (b.cyclic) { n_in = b.nxp - 1; n_out = n_in / 2 + 1; N = n_in; }
    else { n_in = b.nxp - 2; n_out = n_in; N = 2 * (n_in + 1); }
    M.nx_tab = n_out;
    M.Nlog = N;
    M.ftnorm = 1.0 / N;
    M.a_tri = 1.0 / (b.dy * b.dy);
    std::vector<double> bd2(n_out);
    for (int i = 1; i <= n_out; ++i) {
        if (b.cyclic) bd2[i - 1] = -2.0 * M.a_tri + 2.0 * b.dxm2 * (std::cos((i - 1) * TWOPI / N) - 1.0);
        else bd2[i - 1] = -2.0 * M.a_tri + 2.0 * b.dxm2 * (std::cos(i * TWOPI / N) - 1.0);
    }
    M.bb.resize((size_t)n_out * b.nl);
    for (int m = 0; m < b.nl; ++m)
        for (int i = 0; i < n_out; ++i) M.bb[i + (size_t)n_out * m] = bd2[i] - M.rdm2[m];
}

// solve_inhomog_box, inhomog.F90:170-212 (m 0-based)
static void solve_inhomog_box(Model &M, int m, const double *rhs, double *out) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nx = M.nx_tab, ny = nyp - 2;
    std::vector<double> in((size_t)nx * ny), tr((size_t)nx * ny);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) in[i + (size_t)nx * j] = rhs[IX(i + 1, j + 1)];
    dst1(nx, ny, in.data(), tr.data());
    std::vector<double> gam((size_t)nx * ny), betinv(nx), uvec((size_t)nx * ny);
    const double a = M.a_tri;
    const double *bb = &M.bb[(size_t)nx * m];
    for (int i = 0; i < nx; ++i) betinv[i] = 1.0 / bb[i];
    for (int i = 0; i < nx; ++i) uvec[i] = tr[i] * betinv[i];
    for (int j = 1; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            gam[i + (size_t)nx * j] = a * betinv[i];
            betinv[i] = 1.0 / (bb[i] - a * gam[i + (size_t)nx * j]);
            uvec[i + (size_t)nx * j] =
                (tr[i + (size_t)nx * j] - a * uvec[i + (size_t)nx * (j - 1)]) * betinv[i];
        }
    for (int j = ny - 2; j >= 0; --j)
        for (int i = 0; i < nx; ++i)
            uvec[i + (size_t)nx * j] =
                uvec[i + (size_t)nx * j] - gam[i + (size_t)nx * (j + 1)] * uvec[i + (size_t)nx * (j + 1)];
    for (size_t x = 0; x < in.size(); ++x) in[x] = M.ftnorm * uvec[x];
    dst1(nx, ny, in.data(), tr.data());
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) out[IX(i + 1, j + 1)] = tr[i + (size_t)nx * j];
    for (int j = 0; j < nyp; ++j) { out[IX(0, j)] = 0.0; out[IX(nxp - 1, j)] = 0.0; }
    for (int i = 0; i < nxp; ++i) { out[IX(i, 0)] = 0.0; out[IX(i, nyp - 1)] = 0.0; }
}

// solve_inhomog_cyclic, inhomog.F90:214-255
static void solve_inhomog_cyclic(Model &M, int m, const double *rhs, double *out) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, N = nxp - 1, nx = M.nx_tab, ny = nyp - 2;
    std::vector<double> in((size_t)N * ny);
    std::vector<cd> tr((size_t)nx * ny), uvec((size_t)nx * ny);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < N; ++i) in[i + (size_t)N * j] = rhs[IX(i, j + 1)];
    rfft(N, ny, in.data(), tr.data());
    std::vector<double> gam((size_t)nx * ny), betinv(nx);
    const double a = M.a_tri;
    const double *bb = &M.bb[(size_t)nx * m];
    for (int i = 0; i < nx; ++i) betinv[i] = 1.0 / bb[i];
    for (int i = 0; i < nx; ++i) uvec[i] = tr[i] * betinv[i];
    for (int j = 1; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            gam[i + (size_t)nx * j] = a * betinv[i];
            betinv[i] = 1.0 / (bb[i] - a * gam[i + (size_t)nx * j]);
            uvec[i + (size_t)nx * j] =
                (tr[i + (size_t)nx * j] - a * uvec[i + (size_t)nx * (j - 1)]) * betinv[i];
        }
    for (int j = ny - 2; j >= 0; --j)
        for (int i = 0; i < nx; ++i)
            uvec[i + (size_t)nx * j] =
                uvec[i + (size_t)nx * j] - gam[i + (size_t)nx * (j + 1)] * uvec[i + (size_t)nx * (j + 1)];
    for (size_t x = 0; x < uvec.size(); ++x) uvec[x] = M.ftnorm * uvec[x];
    irfft(N, ny, uvec.data(), in.data());
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < N; ++i) out[IX(i, j + 1)] = in[i + (size_t)N * j];
    for (int i = 0; i < nxp; ++i) { out[IX(i, 0)] = 0.0; out[IX(i, nyp - 1)] = 0.0; }
    for (int j = 0; j < nyp; ++j) out[IX(nxp - 1, j)] = out[IX(0, j)];
}

static void solve_inhomog_eqn(Model &M, int m, const double *rhs, double *out) {
    if (M.b.cyclic) solve_inhomog_cyclic(M, m, rhs, out);
    else solve_inhomog_box(M, m, rhs, out);
}

// generate_homog_soln, inhomog.F90:146-154
static void generate_homog_soln(Model &M, int m, const double *L, double *out) {
    std::vector<double> s(M.n2());
    solve_inhomog_eqn(M, m, L, s.data());
    for (size_t x = 0; x < M.n2(); ++x) out[x] = L[x] + M.rdm2[m] * s[x];
}

// homsol_box, homog.F90:214-278 (file lines of homsol_box)
static bool homsol_box(Model &M) {
    const Box &b = M.b;
    int nl = b.nl;
    std::vector<double> L(M.n2(), 1.0);
    M.hom_sol_bc.assign(M.n2() * (nl - 1), 0.0);
    std::vector<double> aipohs(nl, 0.0);
    for (int m = 1; m < nl; ++m) generate_homog_soln(M, m, L.data(), &M.hom_sol_bc[M.n2() * (m - 1)]);
    for (int m = 1; m < nl; ++m) aipohs[m] = int_P_dA(b, &M.hom_sol_bc[M.n2() * (m - 1)]);
    M.cd_lu.n = nl - 1;
    M.cd_lu.A.assign((nl - 1) * (nl - 1), 0.0);
    for (int k = 0; k < nl - 1; ++k)
        for (int m = 1; m < nl; ++m)
            M.cd_lu.A[k + (nl - 1) * (m - 1)] =
                (M.ctm2l[m + nl * (k + 1)] - M.ctm2l[m + nl * k]) * aipohs[m];
    if (!lu_factor(M.cd_lu)) { M.err = "Problem in DGETRF (singular cdhoc)"; return false; }
    return true;
}

// homsol_cyclic, homog.F90:128-212 (file lines of homsol_cyclic)
static void homsol_cyclic(Model &M) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    M.hom_sol_bt.resize(nyp);
    for (int j = 1; j <= nyp; ++j) M.hom_sol_bt[j - 1] = double(nyp - j) / double(nyp - 1);
    M.hbsi = b.yl / b.xl;
    std::vector<double> r1(M.n2()), r2(M.n2()), s1(M.n2()), s2(M.n2());
    for (int j = 0; j < nyp; ++j)
        for (int i = 0; i < nxp; ++i) {
            r1[IX(i, j)] = (b.yp[nyp - 1] - b.yp[j]) / b.yl;
            r2[IX(i, j)] = (b.yp[j] - b.yp[0]) / b.yl;
        }
    M.hbc1.assign((size_t)nyp * nl, 0.0);
    M.hbc2.assign((size_t)nyp * nl, 0.0);
    M.hc1s.assign(nl, 0.0); M.hc2s.assign(nl, 0.0); M.hc1n.assign(nl, 0.0); M.hc2n.assign(nl, 0.0);
    for (int m = 1; m < nl; ++m) {
        generate_homog_soln(M, m, r1.data(), s1.data());
        generate_homog_soln(M, m, r2.data(), s2.data());
        for (int j = 0; j < nyp; ++j) {
            M.hbc1[j + (size_t)nyp * m] = s1[IX(0, j)];
            M.hbc2[j + (size_t)nyp * m] = s2[IX(0, j)];
        }
    }
    for (int m = 1; m < nl; ++m) {
        const double *h1 = &M.hbc1[(size_t)nyp * m], *h2 = &M.hbc2[(size_t)nyp * m];
        double pch1ys = -b.xl * (h1[1] - h1[0]) / b.dy;
        double pch2ys = -b.xl * (h2[1] - h2[0]) / b.dy;
        double pch1yn = b.xl * (h1[nyp - 1] - h1[nyp - 2]) / b.dy;
        double pch2yn = b.xl * (h2[nyp - 1] - h2[nyp - 2]) / b.dy;
        pch1ys = pch1ys + 0.5 * b.dy * M.rdm2[m] * h1[0] * b.xl;
        pch2ys = pch2ys + 0.5 * b.dy * M.rdm2[m] * h2[0] * b.xl;
        pch1yn = pch1yn + 0.5 * b.dy * M.rdm2[m] * h1[nyp - 1] * b.xl;
        pch2yn = pch2yn + 0.5 * b.dy * M.rdm2[m] * h2[nyp - 1] * b.xl;
        double pchdet = pch1ys * pch2yn - pch2ys * pch1yn;
        M.hc1s[m] = pch1ys / pchdet;
        M.hc2s[m] = pch2ys / pchdet;
        M.hc1n[m] = pch1yn / pchdet;
        M.hc2n[m] = pch2yn / pchdet;
    }
}

// qcomp, vorsubs.F90:27-56
static void qcomp(Model &M, const double *p, double *q) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    const size_t n2 = M.n2();
    for (int k = 0; k < nl; ++k) {
        del2_bc(b, p + n2 * k, M.bcco, q + n2 * k);
        for (size_t x = 0; x < n2; ++x) q[n2 * k + x] = q[n2 * k + x] / b.fnot;
    }
    for (size_t x = 0; x < n2; ++x) q[n2 * M.k_topo + x] += M.ddyn[x];
    std::vector<double> mv(nl);
    for (int j = 0; j < nyp; ++j) {
        for (int k = 0; k < nl; ++k)
            for (int i = 0; i < nxp; ++i) q[IX(i, j) + n2 * k] += b.beta * b.yprel[j];
        for (int i = 0; i < nxp; ++i) {
            for (int k = 0; k < nl; ++k) {
                double s = 0;
                for (int l = 0; l < nl; ++l) s += M.amat[k + nl * l] * p[IX(i, j) + n2 * l];
                mv[k] = s;
            }
            for (int k = 0; k < nl; ++k) q[IX(i, j) + n2 * k] -= b.fnot * mv[k];
        }
    }
}

// ocqbdy, vorsubs.F90:58-114 (corners of a box take the matmul, beta and
// topography terms twice, as the reference's loops do)
static void ocqbdy(Model &M) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    const size_t n2 = M.n2();
    const double *p = M.p.data();
    double *q = M.q.data();
    double fac = M.bcco * b.dxm2 / (0.5 * M.bcco + 1.0) / b.fnot;
    for (int k = 0; k < nl; ++k) {
        const double *pk = p + n2 * k;
        double *qk = q + n2 * k;
        for (int i = 0; i < nxp; ++i) {
            qk[IX(i, 0)] = fac * (pk[IX(i, 1)] - pk[IX(i, 0)]);
            qk[IX(i, nyp - 1)] = fac * (pk[IX(i, nyp - 2)] - pk[IX(i, nyp - 1)]);
        }
        if (!b.cyclic)
            for (int j = 0; j < nyp; ++j) {
                qk[IX(0, j)] = fac * (pk[IX(1, j)] - pk[IX(0, j)]);
                qk[IX(nxp - 1, j)] = fac * (pk[IX(nxp - 2, j)] - pk[IX(nxp - 1, j)]);
            }
    }
    auto sub_amat = [&](int i, int j) {
        double mv[OQG_MAX_NL];
        for (int k = 0; k < nl; ++k) {
            double s = 0;
            for (int l = 0; l < nl; ++l) s += M.amat[k + nl * l] * p[IX(i, j) + n2 * l];
            mv[k] = s;
        }
        for (int k = 0; k < nl; ++k) q[IX(i, j) + n2 * k] -= b.fnot * mv[k];
    };
    for (int i = 0; i < nxp; ++i) { sub_amat(i, 0); sub_amat(i, nyp - 1); }
    if (!b.cyclic)
        for (int j = 0; j < nyp; ++j) { sub_amat(0, j); sub_amat(nxp - 1, j); }
    for (int k = 0; k < nl; ++k) {
        double *qk = q + n2 * k;
        for (int i = 0; i < nxp; ++i) {
            qk[IX(i, 0)] += b.beta * b.yprel[0];
            qk[IX(i, nyp - 1)] += b.beta * b.yprel[nyp - 1];
        }
        if (!b.cyclic)
            for (int j = 0; j < nyp; ++j) {
                qk[IX(0, j)] += b.beta * b.yprel[j];
                qk[IX(nxp - 1, j)] += b.beta * b.yprel[j];
            }
    }
    double *qt = q + n2 * M.k_topo;
    const double *dd = M.ddyn.data();
    for (int i = 0; i < nxp; ++i) {
        qt[IX(i, 0)] += dd[IX(i, 0)];
        qt[IX(i, nyp - 1)] += dd[IX(i, nyp - 1)];
    }
    if (!b.cyclic)
        for (int j = 0; j < nyp; ++j) {
            qt[IX(0, j)] += dd[IX(0, j)];
            qt[IX(nxp - 1, j)] += dd[IX(nxp - 1, j)];
        }
}

// init_constraint, constraint.F90:80-143
static void init_constraint(Model &M) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    const size_t n2 = M.n2();
    std::vector<double> pins(nl), pinn(nl), pinsp(nl), pinnp(nl), r(nxp);
    M.cs.assign(nl, 0); M.cn.assign(nl, 0); M.csp.assign(nl, 0); M.cnp.assign(nl, 0);
    for (int k = 0; k < nl; ++k) {
        const double *p = &M.p[n2 * k], *pm = &M.pm[n2 * k];
        pinsp[k] = int_P_dx(b, pm + IX(0, 0));
        pins[k] = int_P_dx(b, p + IX(0, 0));
        pinnp[k] = int_P_dx(b, pm + IX(0, nyp - 1));
        pinn[k] = int_P_dx(b, p + IX(0, nyp - 1));
        for (int i = 0; i < nxp; ++i) r[i] = pm[IX(i, 1)] - pm[IX(i, 0)];
        M.csp[k] = int_P_dx(b, r.data()) / b.dy;
        for (int i = 0; i < nxp; ++i) r[i] = pm[IX(i, nyp - 1)] - pm[IX(i, nyp - 2)];
        M.cnp[k] = int_P_dx(b, r.data()) / b.dy;
        for (int i = 0; i < nxp; ++i) r[i] = p[IX(i, 1)] - p[IX(i, 0)];
        M.cs[k] = int_P_dx(b, r.data()) / b.dy;
        for (int i = 0; i < nxp; ++i) r[i] = p[IX(i, nyp - 1)] - p[IX(i, nyp - 2)];
        M.cn[k] = int_P_dx(b, r.data()) / b.dy;
    }
    for (int k = 0; k < nl; ++k) {
        double apsp = 0, apnp = 0, aps = 0, apn = 0;
        for (int l = 0; l < nl; ++l) {
            double a = M.amat[k + nl * l];
            apsp += a * pinsp[l]; apnp += a * pinnp[l]; aps += a * pins[l]; apn += a * pinn[l];
        }
        M.csp[k] = -M.csp[k] + 0.5 * b.dy * b.fnot * b.fnot * apsp;
        M.cnp[k] = M.cnp[k] + 0.5 * b.dy * b.fnot * b.fnot * apnp;
        M.cs[k] = -M.cs[k] + 0.5 * b.dy * b.fnot * b.fnot * aps;
        M.cn[k] = M.cn[k] + 0.5 * b.dy * b.fnot * b.fnot * apn;
    }
}

// init_mass_constr, constraint.F90:145-165
static void init_mass_constr(Model &M) {
    const Box &b = M.b;
    int nl = b.nl;
    const size_t n2 = M.n2();
    M.dpi.assign(nl - 1, 0); M.dpip.assign(nl - 1, 0);
    std::vector<double> ip(nl), ipm(nl);
    for (int k = 0; k < nl; ++k) { ipm[k] = int_P_dA(b, &M.pm[n2 * k]); ip[k] = int_P_dA(b, &M.p[n2 * k]); }
    for (int k = 0; k < nl - 1; ++k) {
        M.dpip[k] = b.dz_sign * (ipm[k] - ipm[k + 1]);
        M.dpi[k] = b.dz_sign * (ip[k] - ip[k + 1]);
    }
}

// step_constraints, constraint.F90:182-215
static void step_constraints(Model &M, double tdt) {
    const Box &b = M.b;
    int nl = b.nl;
    std::vector<double> rhss(nl), rhsn(nl);
    for (int k = 0; k < nl; ++k) {
        rhss[k] = -0.5 * b.dy * b.fnot * M.int_Be_s[k];
        rhsn[k] = -0.5 * b.dy * b.fnot * M.int_Be_n[k];
    }
    rhss[0] = rhss[0] + M.tau_sign * (b.fnot / b.h[0]) * M.txis;
    rhsn[0] = rhsn[0] - M.tau_sign * (b.fnot / b.h[0]) * M.txin;
    rhss[nl - 1] = rhss[nl - 1] + (b.fnot / b.h[nl - 1]) * M.bdrins;
    rhsn[nl - 1] = rhsn[nl - 1] - (b.fnot / b.h[nl - 1]) * M.bdrinn;
    for (int k = 0; k < nl; ++k) {
        rhss[k] = rhss[k] + M.ajis[k] - M.ap3s[k] + M.ap5s[k];
        rhsn[k] = rhsn[k] + M.ajin[k] + M.ap3n[k] - M.ap5n[k];
    }
    for (int k = 0; k < nl; ++k) {
        double csnew = M.csp[k] + tdt * rhss[k];
        double cnnew = M.cnp[k] + tdt * rhsn[k];
        M.csp[k] = M.cs[k];
        M.cnp[k] = M.cn[k];
        M.cs[k] = csnew;
        M.cn[k] = cnnew;
    }
}

// vort_step, vorticity.F90:14-103
static void vort_step(Model &M, double tdt) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    const size_t n2 = M.n2(), n3 = M.n3();
    std::vector<double> dqdt(n3), del2p(n3), d4p(n3), d6p(n3), r(nxp);
    for (int k = 0; k < nl; ++k) {
        double ajs = 0, ajn = 0;
        jacobian2d(b, &M.p[n2 * k], &M.q[n2 * k], &dqdt[n2 * k], &ajs, &ajn);
        if (b.cyclic) { M.ajis[k] = ajs; M.ajin[k] = ajn; }
    }
    for (int k = 0; k < nl; ++k) del2_bc(b, &M.pm[n2 * k], M.bcco, &del2p[n2 * k]);
    for (int k = 0; k < nl; ++k) del2_bc(b, &del2p[n2 * k], M.bcco, &d4p[n2 * k]);
    for (int k = 0; k < nl; ++k) del2_bc(b, &d4p[n2 * k], M.bcco, &d6p[n2 * k]);
    for (int k = 0; k < nl; ++k) {
        double c2 = M.ah2[k] / b.fnot, c4 = M.ah4[k] / b.fnot;
        for (size_t x = 0; x < n2; ++x)
            dqdt[n2 * k + x] = dqdt[n2 * k + x] + c2 * d4p[n2 * k + x] - c4 * d6p[n2 * k + x];
        if (b.cyclic) {
            const double *d2 = &del2p[n2 * k], *d4 = &d4p[n2 * k];
            for (int i = 0; i < nxp; ++i) r[i] = d2[IX(i, 1)] - d2[IX(i, 0)];
            M.ap3s[k] = M.ah2[k] * int_P_dx(b, r.data()) / b.dy;
            for (int i = 0; i < nxp; ++i) r[i] = d2[IX(i, nyp - 1)] - d2[IX(i, nyp - 2)];
            M.ap3n[k] = M.ah2[k] * int_P_dx(b, r.data()) / b.dy;
            for (int i = 0; i < nxp; ++i) r[i] = d4[IX(i, 1)] - d4[IX(i, 0)];
            M.ap5s[k] = M.ah4[k] * int_P_dx(b, r.data()) / b.dy;
            for (int i = 0; i < nxp; ++i) r[i] = d4[IX(i, nyp - 1)] - d4[IX(i, nyp - 2)];
            M.ap5n[k] = M.ah4[k] * int_P_dx(b, r.data()) / b.dy;
        }
    }
    std::vector<double> fohfac(nl);
    for (int k = 0; k < nl; ++k) fohfac[k] = b.fnot / b.h[k];
    const double *ent1 = &M.ent[0];
    const double *wekp = M.wekp.data();
    const double c_ent1 = b.dz_sign * fohfac[0], c_wind = M.tau_sign * fohfac[0];
    const double c_ent2 = b.dz_sign * fohfac[1];
    const int kt = M.k_topo;
    const double c_drag = fohfac[kt] * M.delek / (2.0 * std::fabs(b.fnot));
    double *dq1 = &dqdt[0], *dq2 = &dqdt[n2], *dqt = &dqdt[n2 * kt];
    const double *d2t = &del2p[n2 * kt];
    double *q = M.q.data(), *qm = M.qm.data();
    const double *dq = dqdt.data();
    // The reference's only OpenMP region on this path (vorticity.F90:67-82).
    // Each statement of the WORKSHARE completes before the next starts.
    const long long N2 = (long long)n2, N3 = (long long)n3;
#pragma omp parallel
    {
#pragma omp for schedule(static)
        for (long long x = 0; x < N2; ++x) dq1[x] = dq1[x] + c_ent1 * ent1[x] + c_wind * wekp[x];
#pragma omp for schedule(static)
        for (long long x = 0; x < N2; ++x) dq2[x] = dq2[x] - c_ent2 * ent1[x];
#pragma omp for schedule(static)
        for (long long x = 0; x < N2; ++x) dqt[x] = dqt[x] - c_drag * d2t[x];
#pragma omp for schedule(static)
        for (long long x = 0; x < N3; ++x) {
            double qold = q[x];
            q[x] = qm[x] + tdt * dq[x];
            qm[x] = qold;
        }
    }
    if (b.cyclic) {
        const double *ent2 = (nl - 1 >= 2) ? &M.ent[n2] : nullptr;
        std::fill(M.int_Be_s.begin(), M.int_Be_s.end(), 0.0);
        std::fill(M.int_Be_n.begin(), M.int_Be_n.end(), 0.0);
        M.int_Be_s[0] = b.dz_sign * fohfac[0] * int_P_dx(b, ent1 + IX(0, 0));
        M.int_Be_s[1] = ent2 ? b.dz_sign * fohfac[0] * int_P_dx(b, ent2 + IX(0, 0)) : 0.0;
        M.int_Be_n[0] = -b.dz_sign * fohfac[1] * int_P_dx(b, ent1 + IX(0, nyp - 1));
        M.int_Be_n[1] = ent2 ? -b.dz_sign * fohfac[1] * int_P_dx(b, ent2 + IX(0, nyp - 1)) : 0.0;
        const double *pmt = &M.pm[n2 * kt];
        for (int i = 0; i < nxp; ++i) r[i] = pmt[IX(i, 1)] - pmt[IX(i, 0)];
        double bdsums = int_P_dx(b, r.data()) / b.dy;
        for (int i = 0; i < nxp; ++i) r[i] = pmt[IX(i, nyp - 1)] - pmt[IX(i, nyp - 2)];
        double bdsumn = int_P_dx(b, r.data()) / b.dy;
        M.bdrins = b.fnot * M.delek / (2.0 * std::fabs(b.fnot)) * bdsums;
        M.bdrinn = b.fnot * M.delek / (2.0 * std::fabs(b.fnot)) * bdsumn;
    }
}

// p_modes_rhs, modes.F90:248-266
static void p_modes_rhs(Model &M, double *rhs) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    const size_t n2 = M.n2();
    std::vector<double> ql(nl);
    for (int j = 0; j < nyp; ++j)
        for (int i = 0; i < nxp; ++i) {
            for (int k = 0; k < nl; ++k) ql[k] = M.q[IX(i, j) + n2 * k] - b.beta * b.yprel[j];
            ql[M.k_topo] = ql[M.k_topo] - M.ddyn[IX(i, j)];
            for (int m = 0; m < nl; ++m) {
                double s = 0;
                for (int k = 0; k < nl; ++k) s += ql[k] * M.ctl2m[k + nl * m];
                rhs[IX(i, j) + n2 * m] = b.fnot * s;
            }
        }
}

// box_homog, homog.F90:331-366 (file lines of box_homog)
static void box_homog(Model &M, const double *inhomog, double *homcor) {
    const Box &b = M.b;
    int nl = b.nl;
    const size_t n2 = M.n2();
    std::vector<double> im(nl), ik(nl), rhs(nl - 1), alpha(nl - 1);
    for (int m = 0; m < nl; ++m) im[m] = int_P_dA(b, inhomog + n2 * m);
    for (int k = 0; k < nl; ++k) {
        double s = 0;
        for (int m = 0; m < nl; ++m) s += M.ctm2l[m + nl * k] * im[m];
        ik[k] = s;
    }
    for (int l = 0; l < nl - 1; ++l) rhs[l] = M.dpi[l] - (ik[l + 1] - ik[l]);
    solve_Ax_b(M.cd_lu, rhs.data(), alpha.data());
    std::fill(homcor, homcor + n2, 0.0);
    for (int m = 1; m < nl; ++m) {
        const double *hs = &M.hom_sol_bc[n2 * (m - 1)];
        for (size_t x = 0; x < n2; ++x) homcor[n2 * m + x] = alpha[m - 1] * hs[x];
    }
}

// cyclic_homog, homog.F90:280-329 (file lines of cyclic_homog)
static void cyclic_homog(Model &M, double tdt, const double *inhomog, double *homcor) {
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    const size_t n2 = M.n2();
    step_constraints(M, tdt);
    std::vector<double> clhss(nl), clhsn(nl), c_bc1(nl), c_bc2(nl);
    for (int m = 0; m < nl; ++m) {
        double ss = 0, sn = 0;
        for (int k = 0; k < nl; ++k) { ss += M.ctl2m[k + nl * m] * M.cs[k]; sn += M.ctl2m[k + nl * m] * M.cn[k]; }
        clhss[m] = ss + int_P_dx(b, inhomog + n2 * m + IX(0, 1)) / b.dy;
        clhsn[m] = sn + int_P_dx(b, inhomog + n2 * m + IX(0, nyp - 2)) / b.dy;
    }
    double c_bt = clhss[0] * M.hbsi;
    for (int m = 1; m < nl; ++m) {
        c_bc1[m] = M.hc2n[m] * clhss[m] - M.hc2s[m] * clhsn[m];
        c_bc2[m] = M.hc1s[m] * clhsn[m] - M.hc1n[m] * clhss[m];
    }
    for (int j = 0; j < nyp; ++j) {
        double v0 = c_bt * M.hom_sol_bt[j];
        for (int i = 0; i < nxp; ++i) homcor[IX(i, j)] = v0;
        for (int m = 1; m < nl; ++m) {
            double v = c_bc1[m] * M.hbc1[j + (size_t)nyp * m] + c_bc2[m] * M.hbc2[j + (size_t)nyp * m];
            for (int i = 0; i < nxp; ++i) homcor[IX(i, j) + n2 * m] = v;
        }
    }
}

// solve_pressure, pressure.F90:21-69
static void solve_pressure(Model &M, double tdt) {
    const Box &b = M.b;
    int nl = b.nl;
    const size_t n2 = M.n2(), n3 = M.n3();
    M.pm = M.p;
    std::vector<double> rhs(n3), inhomog(n3), homcor(n3);
    p_modes_rhs(M, rhs.data());
    for (int m = 0; m < nl; ++m) solve_inhomog_eqn(M, m, &rhs[n2 * m], &inhomog[n2 * m]);
    std::vector<double> ent_xn(nl - 1, 0.0);
    ent_xn[0] = int_P_dA(b, &M.ent[0]);
    // update_mass_constr, constraint.F90:167-179
    for (int l = 0; l < nl - 1; ++l) {
        double aitmp = M.dpi[l];
        M.dpi[l] = M.dpip[l] - tdt * M.gp[l] * ent_xn[l];
        M.dpip[l] = aitmp;
    }
    if (b.cyclic) cyclic_homog(M, tdt, inhomog.data(), homcor.data());
    else box_homog(M, inhomog.data(), homcor.data());
    // modes_to_layers, modes.F90:268-284
    const int nxy = b.nxp * b.nyp;
    for (int x = 0; x < nxy; ++x)
        for (int k = 0; k < nl; ++k) {
            double s = 0;
            for (int m = 0; m < nl; ++m) s += (inhomog[x + n2 * m] + homcor[x + n2 * m]) * M.ctm2l[m + nl * k];
            M.p[x + n2 * k] = s;
        }
}

// step_qg, core.F90:16-33
static void step_qg(Model &M, double tdt) {
    vort_step(M, tdt);
    solve_pressure(M, tdt);
    ocqbdy(M);
}

// suppress_comp_mode, driver.F90:174-189
static void suppress_comp_mode(Model &M) {
    for (size_t x = 0; x < M.n3(); ++x) {
        M.q[x] = 0.5 * (M.q[x] + M.qm[x]);
        M.p[x] = 0.5 * (M.p[x] + M.pm[x]);
    }
    for (size_t l = 0; l < M.dpi.size(); ++l) M.dpi[l] = 0.5 * (M.dpi[l] + M.dpip[l]);
    if (M.b.cyclic)
        for (int k = 0; k < M.b.nl; ++k) {
            M.cs[k] = 0.5 * (M.cs[k] + M.csp[k]);
            M.cn[k] = 0.5 * (M.cn[k] + M.cnp[k]);
        }
}

static bool params_ok(const oqg_params *p, std::string &err) {
    if (!p) { err = "null params"; return false; }
    if (p->nl < 2 || p->nl > OQG_MAX_NL) { err = "nl must be in [2, OQG_MAX_NL]"; return false; }
    if (p->nxp < 4 || p->nyp < 4) { err = "grid too small"; return false; }
    if (!(p->dx > 0) || !(p->dy > 0) || p->fnot == 0.0) { err = "bad dx, dy or fnot"; return false; }
    if (p->k_topo < 1 || p->k_topo > p->nl) { err = "k_topo out of range"; return false; }
    for (int k = 0; k < p->nl; ++k) if (!(p->h[k] > 0)) { err = "layer thickness must be > 0"; return false; }
    for (int k = 0; k < p->nl - 1; ++k) if (!(p->gp[k] > 0)) { err = "reduced gravity must be > 0"; return false; }
    return true;
}

}  // namespace orc

using namespace orc;

extern "C" {

static std::string g_err;

const char *orc_last_error(void) { return g_err.c_str(); }

// init_qg, qg.F90:60-103 (+ zero state as init_dynamic_state with 'zero')
void *orc_create(const oqg_params *prm) {
    std::string err;
    if (!params_ok(prm, err)) { g_err = err; return nullptr; }
    Model *M = new Model();
    M->prm = *prm;
    M->prm.ddyn = nullptr;
    M->b = make_box(*prm);
    M->bcco = prm->bcco; M->delek = prm->delek; M->rho = prm->rho;
    M->tau_sign = prm->tau_sign; M->k_topo = prm->k_topo - 1;
    M->ah2.assign(prm->ah2, prm->ah2 + prm->nl);
    M->ah4.assign(prm->ah4, prm->ah4 + prm->nl);
    M->gp.assign(prm->gp, prm->gp + prm->nl - 1);
    M->ddyn.assign(M->n2(), 0.0);
    if (prm->ddyn) std::copy(prm->ddyn, prm->ddyn + M->n2(), M->ddyn.begin());
    M->suppress_period = prm->suppress_period;
    int nl = prm->nl;
    M->p.assign(M->n3(), 0.0); M->pm = M->p; M->q = M->p; M->qm = M->p;
    M->wekp.assign(M->n2(), 0.0);
    M->ent.assign(M->n2() * (nl - 1), 0.0);
    M->dpi.assign(nl - 1, 0.0); M->dpip.assign(nl - 1, 0.0);
    for (auto *v : {&M->cs, &M->cn, &M->csp, &M->cnp, &M->ajis, &M->ajin, &M->ap3s, &M->ap3n,
                    &M->ap5s, &M->ap5n, &M->int_Be_s, &M->int_Be_n})
        v->assign(nl, 0.0);
    if (!eigmod(*M)) { g_err = M->err; delete M; return nullptr; }
    init_inhomog(*M);
    if (M->b.cyclic) homsol_cyclic(*M);
    else if (!homsol_box(*M)) { g_err = M->err; delete M; return nullptr; }
    return M;
}

void orc_destroy(void *h) { delete static_cast<Model *>(h); }

// init_pv + init_constraint + init_mass_constr (openqg.F90:237-243)
int orc_set_state(void *h, const double *p, const double *pm) {
    Model &M = *static_cast<Model *>(h);
    std::copy(p, p + M.n3(), M.p.begin());
    std::copy(pm, pm + M.n3(), M.pm.begin());
    qcomp(M, M.p.data(), M.q.data());
    qcomp(M, M.pm.data(), M.qm.data());
    if (M.b.cyclic) init_constraint(M);
    init_mass_constr(M);
    return 0;
}

int orc_set_state_full(void *h, const double *p, const double *pm, const double *q,
                       const double *qm, const double *dpi, const double *dpip,
                       const double *cs, const double *cn, const double *csp, const double *cnp) {
    Model &M = *static_cast<Model *>(h);
    int nl = M.b.nl;
    std::copy(p, p + M.n3(), M.p.begin());
    std::copy(pm, pm + M.n3(), M.pm.begin());
    std::copy(q, q + M.n3(), M.q.begin());
    std::copy(qm, qm + M.n3(), M.qm.begin());
    std::copy(dpi, dpi + nl - 1, M.dpi.begin());
    std::copy(dpip, dpip + nl - 1, M.dpip.begin());
    if (cs) std::copy(cs, cs + nl, M.cs.begin());
    if (cn) std::copy(cn, cn + nl, M.cn.begin());
    if (csp) std::copy(csp, csp + nl, M.csp.begin());
    if (cnp) std::copy(cnp, cnp + nl, M.cnp.begin());
    return 0;
}

int orc_get_state(void *h, double *p, double *pm, double *q, double *qm) {
    Model &M = *static_cast<Model *>(h);
    if (p) std::copy(M.p.begin(), M.p.end(), p);
    if (pm) std::copy(M.pm.begin(), M.pm.end(), pm);
    if (q) std::copy(M.q.begin(), M.q.end(), q);
    if (qm) std::copy(M.qm.begin(), M.qm.end(), qm);
    return 0;
}

int orc_get_constraints(void *h, double *dpi, double *dpip, double *cs, double *cn,
                        double *csp, double *cnp) {
    Model &M = *static_cast<Model *>(h);
    if (dpi) std::copy(M.dpi.begin(), M.dpi.end(), dpi);
    if (dpip) std::copy(M.dpip.begin(), M.dpip.end(), dpip);
    if (cs) std::copy(M.cs.begin(), M.cs.end(), cs);
    if (cn) std::copy(M.cn.begin(), M.cn.end(), cn);
    if (csp) std::copy(M.csp.begin(), M.csp.end(), csp);
    if (cnp) std::copy(M.cnp.begin(), M.cnp.end(), cnp);
    return 0;
}

int orc_set_forcing(void *h, const double *wekp, const double *ent, double txis, double txin) {
    Model &M = *static_cast<Model *>(h);
    if (wekp) std::copy(wekp, wekp + M.n2(), M.wekp.begin());
    else std::fill(M.wekp.begin(), M.wekp.end(), 0.0);
    if (ent) std::copy(ent, ent + M.ent.size(), M.ent.begin());
    else std::fill(M.ent.begin(), M.ent.end(), 0.0);
    M.txis = txis;
    M.txin = txin;
    return 0;
}

int orc_step(void *h, double tdt, int nsteps) {
    Model &M = *static_cast<Model *>(h);
    for (int s = 0; s < nsteps; ++s) {
        step_qg(M, tdt);
        bool supp = M.suppress_period > 0 && (M.nt % M.suppress_period) == 0;
        if (supp) suppress_comp_mode(M);
        ++M.nt;
    }
    return 0;
}

int orc_set_step_index(void *h, long long nt) { static_cast<Model *>(h)->nt = nt; return 0; }

int orc_suppress(void *h) { suppress_comp_mode(*static_cast<Model *>(h)); return 0; }

// qg_diagno energetics and extrema, qg_monitor.F90:289-376
int orc_diag(void *h, double *ekei, double *sfmin, double *sfmax, double *circ) {
    Model &M = *static_cast<Model *>(h);
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    const size_t n2 = M.n2();
    std::vector<double> dx(n2), dy(n2), u2(n2), v2(n2);
    for (int k = 0; k < nl; ++k) {
        const double *p = &M.p[n2 * k];
        dPdy_2bc(b, p, M.bcco, dy.data());
        dPdx_2bc(b, p, M.bcco, dx.data());
        for (size_t x = 0; x < n2; ++x) {
            double u = -dy[x] / b.fnot, v = dx[x] / b.fnot;
            u2[x] = u * u;
            v2[x] = v * v;
        }
        double uke = int_P_dA(b, u2.data()), vke = int_P_dA(b, v2.data());
        if (ekei) ekei[k] = 0.5 * M.rho * b.h[k] * (uke + vke);
        if (circ) circ[k] = 1.0e-6 * ((p[IX(0, 0)] - p[IX(0, nyp - 1)]) / b.fnot);
        double poref = b.fnot > 0 ? p[IX(0, 0)] : p[IX(0, nyp - 1)];
        double pomin = p[0], pomax = p[0];
        for (size_t x = 1; x < n2; ++x) { pomin = std::min(pomin, p[x]); pomax = std::max(pomax, p[x]); }
        double e1 = std::min(pomin / b.fnot, pomax / b.fnot);
        double e2 = std::max(pomin / b.fnot, pomax / b.fnot);
        if (sfmin) sfmin[k] = 1.0e-6 * (b.h[k] * (e1 - poref / b.fnot));
        if (sfmax) sfmax[k] = 1.0e-6 * (b.h[k] * (e2 - poref / b.fnot));
    }
    return 0;
}

// qg_diagno, qg_monitor.F90:219-383 (with check_continuity :571-606 for a
// channel).  The jet search runs over the first nyp-1 rows, the extent of the
// reference's ujeto array.
int orc_diagno(void *h, const double *taux, const double *tauy, double tsec, double tdt,
               oqg_qg_monitor *mon) {
    Model &M = *static_cast<Model *>(h);
    const Box &b = M.b;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl;
    const size_t n2 = M.n2();
    const double area = b.xl * b.yl;
    auto avg = [&](const std::vector<double> &f) { return int_P_dA(b, f.data()) / area; };
    std::vector<double> t1(n2), t2(n2);
    // Ekman velocity and entrainment means (:254-263)
    for (size_t x = 0; x < n2; ++x) { t1[x] = M.wekp[x]; t2[x] = std::fabs(M.wekp[x]); }
    mon->wepm = avg(t1);
    mon->wapm = avg(t2);
    const bool have_ent = !M.ent.empty();
    for (size_t x = 0; x < n2; ++x) { t1[x] = have_ent ? M.ent[x] : 0.0; t2[x] = std::fabs(t1[x]); }
    mon->entm = avg(t1);
    mon->enam = avg(t2);
    // interface displacement (:265-287)
    std::vector<double> eta(n2);
    const double tprev = mon->tsec;
    for (int k = 0; k < nl - 1; ++k) {
        for (size_t x = 0; x < n2; ++x) eta[x] = b.dz_sign * (M.p[n2 * k + x] - M.p[n2 * (k + 1) + x]) / M.gp[k];
        mon->etam[k] = avg(eta);
        for (size_t x = 0; x < n2; ++x) t1[x] = eta[x] * eta[x];
        const double et2now = avg(t1);
        mon->pket[k] = tsec > tprev ? 0.5 * M.rho * M.gp[k] * (et2now - mon->et2m[k]) / (tsec - tprev) : 0.0;
        mon->et2m[k] = et2now;
        if (k == 0) {
            for (size_t x = 0; x < n2; ++x) t1[x] = eta[x] * (have_ent ? M.ent[x] : 0.0);
            mon->pken = M.rho * M.gp[0] * avg(t1);
        }
    }
    mon->tsec = tsec;
    // lagged and current geostrophic velocities (:291-304)
    std::vector<double> ug(n2 * nl), vg(n2 * nl), uc(n2 * nl), vc(n2 * nl), dx(n2), dy(n2);
    for (int k = 0; k < nl; ++k) {
        dPdx_2bc(b, &M.pm[n2 * k], M.bcco, dx.data());
        dPdy_2bc(b, &M.pm[n2 * k], M.bcco, dy.data());
        for (size_t x = 0; x < n2; ++x) { ug[n2 * k + x] = -dy[x] / b.fnot; vg[n2 * k + x] = dx[x] / b.fnot; }
        dPdy_2bc(b, &M.p[n2 * k], M.bcco, dy.data());
        dPdx_2bc(b, &M.p[n2 * k], M.bcco, dx.data());
        for (size_t x = 0; x < n2; ++x) { uc[n2 * k + x] = -dy[x] / b.fnot; vc[n2 * k + x] = dx[x] / b.fnot; }
    }
    // wind work (:306-309)
    if (taux && tauy) {
        for (size_t x = 0; x < n2; ++x) { t1[x] = taux[x] * uc[x]; t2[x] = tauy[x] * vc[x]; }
        mon->utau = M.rho * (int_P_dA(b, t2.data()) + int_P_dA(b, t1.data()));
    } else {
        mon->utau = 0.0;
    }
    for (int k = 0; k < nl; ++k) {
        mon->pavg[k] = int_P_dA(b, &M.p[n2 * k]) / area;
        mon->qavg[k] = int_P_dA(b, &M.q[n2 * k]) / area;
    }
    // lagged del^2 and del^4 of u, v (:316-320)
    std::vector<double> d2u(n2), d4u(n2), d2v(n2), d4v(n2);
    std::vector<double> ujeto(nyp);
    for (int k = 0; k < nl; ++k) {
        const double *U = &ug[n2 * k], *V = &vg[n2 * k], *Uc = &uc[n2 * k], *Vc = &vc[n2 * k];
        del2_bc(b, U, M.bcco, d2u.data());
        del2_bc(b, d2u.data(), M.bcco, d4u.data());
        del2_bc(b, V, M.bcco, d2v.data());
        del2_bc(b, d2v.data(), M.bcco, d4v.data());
        for (size_t x = 0; x < n2; ++x) { t1[x] = Uc[x] * d2u[x]; t2[x] = Vc[x] * d2v[x]; }
        mon->ah2d[k] = -M.rho * M.ah2[k] * b.h[k] * (int_P_dA(b, t1.data()) + int_P_dA(b, t2.data()));
        for (size_t x = 0; x < n2; ++x) { t1[x] = Uc[x] * d4u[x]; t2[x] = Vc[x] * d4v[x]; }
        mon->ah4d[k] = M.rho * M.ah4[k] * b.h[k] * (int_P_dA(b, t1.data()) + int_P_dA(b, t2.data()));
        for (size_t x = 0; x < n2; ++x) { t1[x] = Uc[x] * Uc[x]; t2[x] = Vc[x] * Vc[x]; }
        mon->ekei[k] = 0.5 * M.rho * b.h[k] * (int_P_dA(b, t1.data()) + int_P_dA(b, t2.data()));
        std::vector<double> row(nxp);
        for (int j = 0; j < nyp; ++j) {
            for (int i = 0; i < nxp; ++i) row[i] = Uc[IX(i, j)];
            ujeto[j] = std::fabs(int_P_dx(b, row.data())) / b.xl;
        }
        int jm = 0;
        for (int j = 1; j < nyp - 1; ++j)
            if (ujeto[j] > ujeto[jm]) jm = j;
        mon->pos[k] = jm + 1;
        mon->val[k] = ujeto[jm];
        const double *p = &M.p[n2 * k];
        mon->circ[k] = 1.0e-6 * ((p[IX(0, 0)] - p[IX(0, nyp - 1)]) / b.fnot);
    }
    mon->ctot = 0.0;
    for (int k = 0; k < nl; ++k) mon->ctot += mon->circ[k];
    // bottom drag, lagged velocities (:357-360)
    {
        const int kt = M.k_topo;
        for (size_t x = 0; x < n2; ++x) { t1[x] = ug[n2 * kt + x] * ug[n2 * kt + x]; t2[x] = vg[n2 * kt + x] * vg[n2 * kt + x]; }
        mon->btdg = 0.5 * M.rho * M.delek * std::fabs(b.fnot) * (int_P_dA(b, t1.data()) + int_P_dA(b, t2.data()));
    }
    // stream-function extrema (:362-382)
    for (int k = 0; k < nl; ++k) {
        const double *p = &M.p[n2 * k];
        const double poref = b.fnot > 0 ? p[IX(0, 0)] : p[IX(0, nyp - 1)];
        double pomin = p[0], pomax = p[0];
        for (size_t x = 1; x < n2; ++x) { pomin = std::min(pomin, p[x]); pomax = std::max(pomax, p[x]); }
        const double e1 = std::min(pomin / b.fnot, pomax / b.fnot), e2 = std::max(pomin / b.fnot, pomax / b.fnot);
        mon->sfmin[k] = 1.0e-6 * (b.h[k] * (e1 - poref / b.fnot));
        mon->sfmax[k] = 1.0e-6 * (b.h[k] * (e2 - poref / b.fnot));
    }
    // check_continuity (:571-606), channel only
    for (int k = 0; k < OQG_MAX_NL; ++k) { mon->ermas[k] = 0.0; mon->emfr[k] = 0.0; }
    if (b.cyclic) {
        std::vector<double> ip(nl);
        for (int k = 0; k < nl; ++k) ip[k] = int_P_dA(b, &M.p[n2 * k]);
        for (int k = 0; k < nl - 1; ++k) {
            const double est1 = b.dz_sign * (ip[k] - ip[k + 1]), est2 = M.dpi[k];
            const double edif = est1 - est2, esum = std::fabs(est1) + std::fabs(est2);
            mon->ermas[k] = edif;
            mon->emfr[k] = esum > 1.0e-13 * b.xl * b.yl * tdt * M.gp[k] ? 2.0 * edif / esum : 0.0;
        }
    }
    return 0;
}

int orc_solve_inhomog(void *h, int m, const double *rhs, double *out) {
    Model &M = *static_cast<Model *>(h);
    if (m < 1 || m > M.b.nl) return OQG_EINVAL;
    solve_inhomog_eqn(M, m - 1, rhs, out);
    return 0;
}

int orc_generate_homog_soln(void *h, int m, const double *L, double *out) {
    Model &M = *static_cast<Model *>(h);
    if (m < 1 || m > M.b.nl) return OQG_EINVAL;
    generate_homog_soln(M, m - 1, L, out);
    return 0;
}

// Replaces rdm2 and rebuilds the Helmholtz tables: init_inhomog(b, rdm2) with
// an explicit rdm2, as src/tests/test_inhomog.F90:34-37 does.
int orc_set_rdm2(void *h, const double *rdm2) {
    Model &M = *static_cast<Model *>(h);
    std::copy(rdm2, rdm2 + M.b.nl, M.rdm2.begin());
    init_inhomog(M);
    return 0;
}

int orc_get_modes(void *h, double *amat, double *rdm2, double *ctl2m, double *ctm2l) {
    Model &M = *static_cast<Model *>(h);
    if (amat) std::copy(M.amat.begin(), M.amat.end(), amat);
    if (rdm2) std::copy(M.rdm2.begin(), M.rdm2.end(), rdm2);
    if (ctl2m) std::copy(M.ctl2m.begin(), M.ctl2m.end(), ctl2m);
    if (ctm2l) std::copy(M.ctm2l.begin(), M.ctm2l.end(), ctm2l);
    return 0;
}

// hom_sol_bc (box: (nxp,nyp,nl-1)) or hom_sol_bc1/2 (channel: (nyp,nl) each)
int orc_get_homog(void *h, double *a, double *b2) {
    Model &M = *static_cast<Model *>(h);
    if (M.b.cyclic) {
        if (a) std::copy(M.hbc1.begin(), M.hbc1.end(), a);
        if (b2) std::copy(M.hbc2.begin(), M.hbc2.end(), b2);
    } else if (a) {
        std::copy(M.hom_sol_bc.begin(), M.hom_sol_bc.end(), a);
    }
    return 0;
}

int orc_jacobian(void *h, const double *p, const double *q, double *jac) {
    Model &M = *static_cast<Model *>(h);
    jacobian2d(M.b, p, q, jac, nullptr, nullptr);
    return 0;
}

int orc_del2(void *h, const double *f, double alpha, double *out) {
    Model &M = *static_cast<Model *>(h);
    del2_bc(M.b, f, alpha, out);
    return 0;
}

double orc_int_P_dA(void *h, const double *f) { return int_P_dA(static_cast<Model *>(h)->b, f); }

void orc_dst1(int n, int howmany, const double *in, double *out) { dst1(n, howmany, in, out); }

// O(n^2) long-double DST-I, the pin for orc_dst1
void orc_dst1_direct_ld(int n, const double *in, double *out) {
    const long double pi = 3.14159265358979323846264338327950288L;
    for (int k = 0; k < n; ++k) {
        long double s = 0;
        for (int j = 0; j < n; ++j) s += (long double)in[j] * sinl(pi * (long double)((j + 1) * (long long)(k + 1) % (2 * (n + 1))) / (n + 1));
        out[k] = (double)(2.0L * s);
    }
}

// r2c / c2r with interleaved complex (re, im) output/input
void orc_rfft(int N, int howmany, const double *in, double *out_c) {
    rfft(N, howmany, in, reinterpret_cast<cd *>(out_c));
}
void orc_irfft(int N, int howmany, const double *in_c, double *out) {
    irfft(N, howmany, reinterpret_cast<const cd *>(in_c), out);
}

// ekman_from_tau, ekman.F90:53-83 (wekp, txis, txin)
int orc_ekman_from_tau(const oqg_params *prm, const double *taux, const double *tauy,
                       double *wekp, double *txis, double *txin) {
    Box b = make_box(*prm);
    const int nxp = b.nxp, nyp = b.nyp, nxt = nxp - 1, nyt = nyp - 1;
    if (b.cyclic) {
        std::vector<double> r(nxp);
        for (int i = 0; i < nxp; ++i) r[i] = taux[IX(i, 0)] + taux[IX(i, 1)];
        if (txis) *txis = 0.5 * int_P_dx(b, r.data());
        for (int i = 0; i < nxp; ++i) r[i] = taux[IX(i, nyp - 2)] + taux[IX(i, nyp - 1)];
        if (txin) *txin = 0.5 * int_P_dx(b, r.data());
    } else {
        if (txis) *txis = 0.0;
        if (txin) *txin = 0.0;
    }
    std::vector<double> txt((size_t)nxt * nyp), tyt((size_t)nxp * nyt), wekt((size_t)nxt * nyt);
    for (int j = 0; j < nyp; ++j)
        for (int i = 0; i < nxt; ++i) txt[i + (size_t)nxt * j] = 0.5 * (taux[IX(i + 1, j)] + taux[IX(i, j)]);
    for (int j = 0; j < nyt; ++j)
        for (int i = 0; i < nxp; ++i) tyt[i + (size_t)nxp * j] = 0.5 * (tauy[IX(i, j + 1)] + tauy[IX(i, j)]);
    for (int j = 0; j < nyt; ++j)
        for (int i = 0; i < nxt; ++i)
            wekt[i + (size_t)nxt * j] =
                ((1.0 / (b.dx * b.fnot)) * (tyt[(i + 1) + (size_t)nxp * j] - tyt[i + (size_t)nxp * j]) -
                 (1.0 / (b.dy * b.fnot)) * (txt[i + (size_t)nxt * (j + 1)] - txt[i + (size_t)nxt * j]));
    map_T_to_P(b, wekt.data(), wekp);
    return 0;
}

}  // extern "C"
