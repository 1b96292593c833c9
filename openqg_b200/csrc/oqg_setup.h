// oqg_setup.h -- init-time host computations of init_qg (qg/qg.F90:60-103):
// vertical modes, Helmholtz tables, FFT plans.  Compiled without FMA
// contraction so the tables round like the reference's FP64 arithmetic.
#pragma once

#include <string>
#include <vector>

namespace oqg {

struct Modes {
    int nl = 0;
    std::vector<double> amat, ctl2m, ctm2l, rdm2;   // column-major nl x nl; rdm2[nl]
};

// compute_A + eigmod + derive_qg_modes (qg/modes.F90:46-246).  Returns false
// (with a message) when the mode matrices fail the identity check.
bool setup_modes(int nl, const double *h, const double *gp, double fnot, Modes &out,
                 std::string &err);

// Tridiagonal coefficients of init_inhomog (qg/inhomog.F90:126-141) and the
// pivots 1/(bb - a*gam) of the Thomas forward sweep (inhomog.F90:188-195),
// per (mode, wavenumber), stored up to their floating-point fixed point.
struct PivotTable {
    std::vector<double> tab;
    std::vector<int> off, len;   // [nl * nk]
};
void setup_pivots(bool cyclic, int nxp, int nyp, double dx, double dy,
                  const std::vector<double> &rdm2, PivotTable &out, double &a_tri);

// Radices (16, 8, 4, 2, 3, 5) of a transform length, in the order the
// device's compile-time plans take them; false if another prime remains.
bool fft_radices(int M, std::vector<int> &rad);

// Twiddles of every Stockham stage of a length-M transform with radices rad,
// interleaved (re, im) and correctly rounded: the stage of radix R that
// follows Ns = product of the earlier radices holds exp(-2 pi i r jm/(Ns R))
// for jm < Ns, 1 <= r < R at entry Ns - 1 + jm (R-1) + r - 1; M - 1 entries
// in all (the table has M).
void fft_stage_twiddles(int M, const std::vector<int> &rad, std::vector<double> &tw);

// w_k = sum_{i=1..n} 2 sin(pi i k/(n+1)), k = 1..n: the x-sum of the k-th
// inverse DST-I basis row.
void dst_row_sums(int n, std::vector<double> &w);

// DGETRF-style LU with partial pivoting (column-major); false if singular.
bool lu_factor(int n, const double *A, double *LU, int *piv);

}  // namespace oqg
