// The radiation scheme's start-up on the host: the coupled atmosphere's mean
// radiative balance, the linearised radiation coefficients, the
// radiative-balance coefficients, and the derived entrainment coefficients
// and zonal temperature profiles.  Follows src/mixed/radsubs.F90:63-674,
// src/mixed/mixed.F90:102-151, src/mixed/amlsubs.F90:100-182 and
// src/glam/numerics.F90:516-525.  Pure host arithmetic, run once per model.
#include <cmath>
#include <cstring>
#include <utility>

#include "../../include/oqg.h"

namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kStefan = 5.67040e-8;   // constants.F90 STEFAN
constexpr double kSigOv2 = 0.5 * kStefan;
constexpr int kNz = 10001;               // quadrature points of every integral
constexpr int kMaxIter = 200;
constexpr double kTol = 1.0e-13;

double trans(double thickness, double opt) { return std::exp(-thickness / opt); }   // A.1

double pow4(double t) { return t * t * t * t; }
double pow3(double t) { return t * t * t; }

// B(T0, z, gamma): half the black-body flux at height z of a column with
// lapse rate gamma.
double bflux(double t0, double z, double gamma) { return kSigOv2 * pow4(t0 - z * gamma); }

// The extended trapezoidal rule of f sampled on kNz points at spacing delz
// (trapin).  f is evaluated point by point to keep no table.
template <class F>
double trapin(F f, double delz) {
    double s = 0.0;
    for (int i = 1; i < kNz - 1; ++i) s += f(i);
    return delz * (0.5 * f(0) + s + 0.5 * f(kNz - 1));
}

}  // namespace

namespace oqg {
int host_fail(int code, const char *msg);   // oqg_capi.cu: sets the message oqg_last_error returns
}  // namespace oqg
using oqg::host_fail;

extern "C" {

int oqg_radiat(int nl, const double *h, double hm, double fnot, const oqg_rad_params *p, oqg_rad_state *out) {
    if (!h || !p || !out) return host_fail(OQG_EINVAL, "null argument");
    if (nl < 1 || nl > OQG_MAX_NL) return host_fail(OQG_EINVAL, "nl out of range");
    if (!(p->fspamp >= 0.0)) return host_fail(OQG_EINVAL, "fspamp must be >= 0 (load_rad)");
    if (!(hm > 0.0) || !(hm < h[0])) return host_fail(OQG_EINVAL, "need 0 < hm < h(1)");
    for (int k = 0; k <= nl; ++k)
        if (!(p->zopt[k] > 0.0)) return host_fail(OQG_EINVAL, "optical depths must be > 0");
    std::memset(out, 0, sizeof(*out));
    const double *zopt = p->zopt, *tabsat = p->tabsat, gamma = p->gamma;
    // compute_layer_trans (:159-176); index k is layer k, 0 the mixed layer
    double tauk[OQG_MAX_NL + 1];
    tauk[0] = trans(hm, zopt[0]);
    tauk[1] = trans(h[0] - hm, zopt[1]);
    for (int k = 2; k <= nl; ++k) tauk[k] = trans(h[k - 1], zopt[k]);
    // compute_mean_radiation (:186-242): sigma I_k / 2 up and down, A.26, A.41
    double uprad[OQG_MAX_NL + 1], dnrad[OQG_MAX_NL + 1];
    double hbot = hm, htop = h[0];
    for (int k = 1; k <= nl; ++k) {
        if (k > 1) {
            hbot = htop;
            htop = hbot + h[k - 1];
        }
        const double delz = k == 1 ? (htop - hbot) / double(kNz - 1) : h[k - 1] / double(kNz - 1);
        const double tk = tabsat[k - 1], zo = zopt[k], hb = hbot, ht = htop;
        auto up = [&](int i) {
            const double zz = hb + double(i) * delz;
            return kSigOv2 * pow4(tk - gamma * zz) * trans(ht - zz, zo);
        };
        auto dn = [&](int i) {
            const double zz = hb + double(i) * delz;
            return kSigOv2 * pow4(tk - gamma * zz) * trans(zz - hb, zo);
        };
        uprad[k] = trapin(up, delz) / zo;
        dnrad[k] = trapin(dn, delz) / zo;
    }
    // compute_ml_mean_temp (:244-300): the atmospheric mixed layer's mean
    // temperature that carries the required upgoing flux
    double rhstat = 0.0, prod = 1.0;
    for (int k = 1; k <= nl; ++k) rhstat = rhstat * tauk[k] + uprad[k];
    for (int k = 1; k <= nl; ++k) prod *= tauk[k];
    rhstat = (-rhstat - p->fsbar) / prod;
    double atm = 300.0, uprad_m = 0.0;
    {
        const double delz = hm / double(kNz - 1);
        for (int iter = 1;; ++iter) {
            const double ta = atm;
            auto f = [&](int i) {
                const double zz = double(i) * delz;
                return pow4(ta - gamma * zz) * trans(hm - zz, zopt[0]);
            };
            uprad_m = trapin(f, delz);
            uprad_m = uprad_m * kSigOv2 / zopt[0];
            const double deltm = 0.25 * (rhstat - uprad_m) * atm / uprad_m;
            atm = atm + 0.75 * deltm;
            if (iter > kMaxIter) return host_fail(OQG_ESETUP, "iteration for tmbara not converged (radiat)");
            if (std::fabs(deltm) <= kTol) break;
        }
    }
    // compute_oml_mean_temp (:302-336)
    const double rhstoc = p->xlamda * atm + bflux(atm, 0.0, 0.0) - p->fsbar;
    double ocn = atm;
    for (int iter = 1;; ++iter) {
        const double told = ocn;
        ocn = rhstoc / (p->xlamda + kStefan * pow3(told));
        if (iter > kMaxIter) return host_fail(OQG_ESETUP, "iteration for tmbaro not converged (radiat)");
        if (std::fabs(ocn - told) <= kTol) break;
    }
    // compute_mean_flux (:346-382): A.16, A.28, A.43
    double fupbar[OQG_MAX_NL + 1], fdnbar[OQG_MAX_NL + 2];
    fupbar[0] = uprad_m;
    for (int k = 1; k <= nl; ++k) fupbar[k] = fupbar[k - 1] * tauk[k] + uprad[k];
    fdnbar[nl] = -dnrad[nl];
    for (int k = nl - 1; k >= 1; --k) fdnbar[k] = fdnbar[k + 1] * tauk[k] - dnrad[k];
    // compute_perturb_rad_params (:443-538)
    double Z[OQG_MAX_NL + 1], btop[OQG_MAX_NL + 1], bbot[OQG_MAX_NL + 1];
    Z[1] = h[0];
    for (int k = 2; k <= nl; ++k) Z[k] = Z[k - 1] + h[k - 1];
    btop[0] = bflux(atm, hm, gamma);
    for (int k = 1; k <= nl; ++k) btop[k] = bflux(tabsat[k - 1], Z[k], gamma);
    bbot[0] = bflux(atm, 0.0, gamma);
    bbot[1] = bflux(tabsat[0], hm, gamma);
    for (int k = 2; k <= nl; ++k) bbot[k] = bflux(tabsat[k - 1], Z[k - 1], gamma);
    auto &Aup = out->aup;          // Aup(k, l) at [k][l]
    auto &Adn = out->adown;        // Adown(k, l) at [k-1][l]
    Aup[0][0] = (btop[0] - fupbar[0]) / zopt[0];
    for (int k = 1; k <= nl - 1; ++k) Aup[k][k] = (-tauk[k] * fupbar[k - 1] - uprad[k] + btop[k]) / zopt[k];
    for (int k = 1; k <= nl; ++k)
        Aup[k][k - 1] = tauk[k] * (Aup[k - 1][k - 1] + fupbar[k - 1] / zopt[k] - bbot[k] / zopt[k]);
    for (int k = 2; k <= nl; ++k)
        for (int l = 0; l <= k - 2; ++l) Aup[k][l] = Aup[k - 1][l] * tauk[k];
    const double d0up = 4.0 * kStefan * pow3(ocn);
    {
        const double delz = hm / double(kNz - 1);
        auto f = [&](int i) {
            const double zz = double(i) * delz;
            return pow3(atm - gamma * zz) * std::exp(-(hm - zz) / zopt[0]);
        };
        out->dup[0] = 2.0 * kStefan * trapin(f, delz) / zopt[0];
    }
    for (int k = 1; k <= nl; ++k) out->dup[k] = out->dup[k - 1] * tauk[k];
    for (int k = 1; k <= nl - 1; ++k) Adn[k - 1][k - 1] = (fdnbar[k + 1] * tauk[k] - dnrad[k] + bbot[k]) / zopt[k];
    Adn[nl - 1][nl - 1] = (bbot[nl] - dnrad[nl]) / zopt[nl];
    for (int k = nl - 1; k >= 1; --k) {
        for (int l = k + 1; l <= nl - 1; ++l) Adn[k - 1][l] = Adn[k][l] * tauk[k];
        Adn[k - 1][k] = tauk[k] * (Adn[k][k] - fdnbar[k + 1] / zopt[k] - btop[k] / zopt[k]);
    }
    const double dmdown = -2.0 * kStefan * pow3(atm);
    // compute_rad_bal_coeffs (:577-659): rbalar x = -1 by LU with partial
    // pivoting; row k, column i at a[k-1][i-1]
    double a[OQG_MAX_NL][OQG_MAX_NL] = {}, x[OQG_MAX_NL];
    for (int i = 1; i <= nl - 1; ++i) a[0][i - 1] = Adn[0][i];
    a[0][nl - 1] = out->dup[0];
    for (int k = 2; k <= nl - 1; ++k) {
        for (int i = 1; i <= nl - 1; ++i) a[k - 1][i - 1] = Adn[k][i] + Aup[k][i];
        a[k - 1][nl - 1] = out->dup[k];
    }
    for (int i = 1; i <= nl - 1; ++i) a[nl - 1][i - 1] = Aup[nl][i];
    a[nl - 1][nl - 1] = out->dup[nl];
    for (int k = 0; k < nl; ++k) x[k] = -1.0;
    for (int c = 0; c < nl; ++c) {
        int piv = c;
        for (int r = c + 1; r < nl; ++r)
            if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
        if (a[piv][c] == 0.0) return host_fail(OQG_ESETUP, "radiative balance matrix is singular (radiat)");
        if (piv != c) {
            for (int j = 0; j < nl; ++j) std::swap(a[c][j], a[piv][j]);
            std::swap(x[c], x[piv]);
        }
        for (int r = c + 1; r < nl; ++r) {
            const double m = a[r][c] / a[c][c];
            for (int j = c; j < nl; ++j) a[r][j] -= m * a[c][j];
            x[r] -= m * x[c];
        }
    }
    for (int r = nl - 1; r >= 0; --r) {
        double s = x[r];
        for (int j = r + 1; j < nl; ++j) s -= a[r][j] * x[j];
        x[r] = s / a[r][r];
    }
    for (int k = 1; k <= nl - 1; ++k) out->rbetat[k - 1] = x[k - 1];
    out->rbtmat = x[nl - 1];
    out->rbtmoc = ((p->xlamda - dmdown) * out->rbtmat - 1.0) / (p->xlamda + d0up);
    out->atm_tmbar = atm;
    out->ocn_tmbar = ocn;
    oqg_rad_coeffs &c = out->c;
    c.fspco = std::copysign(std::fabs(p->fspamp), fnot);   // load_rad: sign(fspamp, fnot)
    c.xlamda = p->xlamda;
    c.d0up = d0up;
    c.dmdown = dmdown;
    c.dup0 = out->dup[0];
    c.aup00 = Aup[0][0];
    c.adown10 = Adn[0][0];
    c.adown11 = nl >= 2 ? Adn[0][1] : 0.0;
    return OQG_OK;
}

int oqg_entrain_coeff(int nl, double rho_cp, double dt_12, const oqg_rad_state *rad, double *aface, double *bface,
                      double *dface) {
    if (!rad || !aface || !bface || !dface) return host_fail(OQG_EINVAL, "null argument");
    if (nl < 1 || nl > OQG_MAX_NL) return host_fail(OQG_EINVAL, "nl out of range");
    if (rho_cp * dt_12 == 0.0) return host_fail(OQG_EINVAL, "rho_cp * dt_12 must be nonzero");
    const double rrcpdt = -1.0 / (rho_cp * dt_12);
    for (int l = 1; l <= nl - 1; ++l) aface[l - 1] = rrcpdt * (0.0 + rad->adown[0][l] - rad->aup[nl][l]);
    *bface = rrcpdt * (rad->aup[0][0] + rad->adown[0][0] - rad->aup[nl][0]);
    *dface = rrcpdt * (rad->dup[0] + 0.0 - rad->dup[nl]);
    return OQG_OK;
}

int oqg_zonal_temp(int nyt, double y0, double dy, double fnot, double ya0, double yla, double dt_ns, double *out) {
    if (!out || nyt < 1) return host_fail(OQG_EINVAL, "null argument or nyt < 1");
    if (!(yla > 0.0)) return host_fail(OQG_EINVAL, "yla must be > 0");
    const double yc = ya0 + 0.5 * yla, yn = ya0 + yla;
    const double amp = -0.50 * std::copysign(std::fabs(dt_ns), fnot);
    for (int j = 0; j < nyt; ++j) {
        const double y = (y0 + double(j) * dy) + 0.5 * dy;
        out[j] = amp * std::sin((kPi / 2.0) * (y - yc) / (yn - yc));
    }
    return OQG_OK;
}

}  // extern "C"
