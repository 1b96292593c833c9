// oqg_mixed.cuh -- the ocean mixed layer's step and the Ekman fields that
// feed it, on the device (closed box, FP64 arithmetic).
//
//   ekman_from_tau   src/coupler/ekman.F90:53-83
//   step_oml         src/mixed/omlsubs.F90:69-119
//   adv_diff         src/mixed/mixed_layer.F90:16-95
//   del2_T, avg_T, map_T_to_x_face / y_face, c_grid_advection, dPdx, dPdy,
//   map_T_to_P       src/glam/numerics.F90:64-163, 223-309, 392-408
//
// T-grid fields are [nyt][nxt] (nxt = nxp-1, nyt = nyp-1), the wind stress
// [nyp][nxp], all FP64 and contiguous.  The QG layer-1 pressure is read from
// the handle's state and the results land in the handle's forcing fields.
#pragma once

#include "oqg_kernels.cuh"

#define OQG_OML_CTAS 296

namespace oqg {

struct OmlDev {
    int nxp, nyp, nxt, nyt, tau_sign, fluxn, fluxs;
    double dx, dy, fnot, hm, rho_cp, t1_rel, dt_12, st2d, st4d, ycexp, nval, sval;
    const double *taux, *tauy;   // [nyp][nxp]
    const double *fnet;          // [nyt][nxt] net heat flux into the ocean
    double *data, *datam;        // sst and its lagged value [nyt][nxt]
    double *snew, *wekt, *xfo;   // the next sst, T-grid Ekman pumping, entrainment [nyt][nxt]
    double *part;                // [OQG_OML_CTAS] partial sums of xfo
};

// del2_T (numerics.F90:109-145) of t at T point (i, j), closed box.
__device__ __forceinline__ double oml_del2(const OmlDev &o, const double *t, int i, int j, bool nflux, double nval,
                                           bool sflux, double sval) {
    const int nxt = o.nxt, nyt = o.nyt;
    const double c = t[(size_t)j * nxt + i];
    const double left = i == 0 ? 0.0 : c - t[(size_t)j * nxt + i - 1];
    const double right = i == nxt - 1 ? 0.0 : t[(size_t)j * nxt + i + 1] - c;
    const double bot = j == 0 ? (sflux ? c - sval : 0.0) : c - t[(size_t)(j - 1) * nxt + i];
    const double top = j == nyt - 1 ? (nflux ? nval - c : 0.0) : t[(size_t)(j + 1) * nxt + i] - c;
    return (1.0 / (o.dx * o.dx)) * (right - left + top - bot);
}

// Ekman pumping at T point (i, j) (ekman.F90:78-80) from map_P_to_y_face /
// map_P_to_x_face of the stress.
__device__ __forceinline__ double oml_wekt(const OmlDev &o, int i, int j) {
    const double *tx = o.taux, *ty = o.tauy;
    const int nxp = o.nxp;
    const double tyw = 0.5 * (ty[(size_t)(j + 1) * nxp + i] + ty[(size_t)j * nxp + i]);
    const double tye = 0.5 * (ty[(size_t)(j + 1) * nxp + i + 1] + ty[(size_t)j * nxp + i + 1]);
    const double txs = 0.5 * (tx[(size_t)j * nxp + i + 1] + tx[(size_t)j * nxp + i]);
    const double txn = 0.5 * (tx[(size_t)(j + 1) * nxp + i + 1] + tx[(size_t)(j + 1) * nxp + i]);
    return (1.0 / (o.dx * o.fnot)) * (tye - tyw) - (1.0 / (o.dy * o.fnot)) * (txn - txs);
}

// step_oml at T points: the Ekman pumping, advection (C grid, geostrophic
// from the layer-1 pressure P1 plus Ekman), Laplacian and biharmonic
// diffusion (del2_T of the lagged sst taken at the five points of the outer
// del2_T), heat and Ekman forcing, the convective adjustment and, when ent is
// computed, the layer 1/2 entrainment xfo with per-CTA partial sums for its
// mean.  The new sst goes to snew (the host then rotates snew, data, datam).
template <class T>
__global__ void __launch_bounds__(256) k_oml_step(OmlDev o, const T *__restrict__ P1, int px, double tdto,
                                                   int compute_ent) {
    __shared__ double red[32];
    const int nxt = o.nxt, nyt = o.nyt, nxp = o.nxp, nyp = o.nyp;
    const double ce = o.tau_sign / (o.fnot * o.hm), cg = o.ycexp / o.fnot;
    const double *tx = o.taux, *ty = o.tauy, *t = o.data;
    auto p = [&](int i, int j) { return (double)P1[(size_t)j * px + i]; };
    auto d2 = [&](int i, int j) { return oml_del2(o, o.datam, i, j, o.fluxn, o.nval, o.fluxs, o.sval); };
    // vel_u * mixed_x on the x-face of column f (0..nxt), row j
    auto uflux = [&](int f, int j) {
        if (f == 0 || f == nxp - 1) return 0.0;   // no normal flow through the walls
        const double dpdy = (1.0 / o.dy) * (p(f, j + 1) - p(f, j));
        const double uek = ce * (0.5 * (ty[(size_t)(j + 1) * nxp + f] + ty[(size_t)j * nxp + f]));
        const double vel = -cg * dpdy + uek;
        const double mx = 0.5 * (t[(size_t)j * nxt + f - 1] + t[(size_t)j * nxt + f]);
        return vel * mx;
    };
    // vel_v * mixed_y on the y-face of row g (0..nyt), column i
    auto vflux = [&](int i, int g) {
        const double vek = -ce * (0.5 * (tx[(size_t)g * nxp + i + 1] + tx[(size_t)g * nxp + i]));
        double vel, my;
        if (g == 0) {
            vel = o.fluxs ? vek : 0.0;
            my = o.fluxs ? t[i] : 0.5 * (t[i] + o.sval);
        } else if (g == nyp - 1) {
            vel = o.fluxn ? vek : 0.0;
            my = o.fluxn ? t[(size_t)(nyt - 1) * nxt + i] : 0.5 * (t[(size_t)(nyt - 1) * nxt + i] + o.nval);
        } else {
            const double dpdx = (1.0 / o.dx) * (p(i + 1, g) - p(i, g));
            vel = cg * dpdx + vek;
            my = 0.5 * (t[(size_t)(g - 1) * nxt + i] + t[(size_t)g * nxt + i]);
        }
        return vel * my;
    };
    double xs = 0.0;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nxt * nyt; idx += gridDim.x * blockDim.x) {
        const int j = idx / nxt, i = idx - j * nxt;
        const double wk = oml_wekt(o, i, j);
        o.wekt[idx] = wk;
        const double adv = (-1.0 / o.dx) * (uflux(i + 1, j) - uflux(i, j)) + (-1.0 / o.dy) * (vflux(i, j + 1) - vflux(i, j));
        // del2_T (no flux) of del2_T(datam): the inner one at the five points
        const double d2c = d2(i, j);
        const double left = i == 0 ? 0.0 : d2c - d2(i - 1, j);
        const double right = i == nxt - 1 ? 0.0 : d2(i + 1, j) - d2c;
        const double bot = j == 0 ? 0.0 : d2c - d2(i, j - 1);
        const double top = j == nyt - 1 ? 0.0 : d2(i, j + 1) - d2c;
        const double d4 = (1.0 / (o.dx * o.dx)) * (right - left + top - bot);
        const double ad = adv + o.st2d * d2c - o.st4d * d4;
        const double dm = o.datam[idx];
        const double half = 0.5 * wk * (dm - o.t1_rel);
        const double sstnew = dm + tdto * (ad + (1.0 / (o.rho_cp * o.hm)) * o.fnet[idx] + (1.0 / o.hm) * (wk * dm - half));
        const double conv = fmax(0.0, o.t1_rel - sstnew);
        o.snew[idx] = sstnew + conv;
        if (compute_ent) {
            const double x = (-1.0 / o.dt_12) * half - (o.hm / (tdto * o.dt_12)) * conv;
            o.xfo[idx] = x;
            xs += x;
        }
    }
    if (compute_ent) {
        const double v = block_sum(xs, red);
        if (threadIdx.x == 0) o.part[blockIdx.x] = v;
    }
}

// map_T_to_P (numerics.F90:64-107) of a T-grid field at p point (i, j), the
// constant c subtracted from every T value first.
__device__ __forceinline__ double oml_t2p(const OmlDev &o, const double *t, double c, int i, int j) {
    const int nxt = o.nxt, nyt = o.nyt, nxp = o.nxp, nyp = o.nyp;
    auto T_ = [&](int a, int bb) { return t[(size_t)bb * nxt + a] - c; };
    const bool w = i == 0, e = i == nxp - 1, s = j == 0, n = j == nyp - 1;
    if ((w || e) && (s || n)) return T_(w ? 0 : nxt - 1, s ? 0 : nyt - 1);
    if (s || n) {
        const int r = s ? 0 : nyt - 1;
        return 0.5 * (T_(i - 1, r) + T_(i, r));
    }
    if (w || e) {
        const int cc = w ? 0 : nxt - 1;
        return 0.5 * (T_(cc, j - 1) + T_(cc, j));
    }
    return 0.25 * (T_(i, j) + T_(i - 1, j) + T_(i, j - 1) + T_(i - 1, j - 1));
}

// The QG forcing from the mixed layer, one CTA of 128 threads per p row j:
// wekp = map_T_to_P(wekt) and, when computed, ent(:,:,1) =
// map_T_to_P(xfo - avg_T(xfo)), ent(:,:,2:) = 0, into the handle's pitched
// fields, with the trapezoid row sum of ent(:,:,1) into ent_rows[j] (as
// k_ent_rows forms it, for the forcing integrals).  Every CTA adds the
// partial sums of xfo in the same order (deterministic mean).
template <class T>
__global__ void __launch_bounds__(128) k_oml_post(OmlDev o, T *wekp, T *ent, double *ent_rows, int px, int nl,
                                                   int compute_ent, int nparts, const BasinDev *__restrict__ bas,
                                                   const T *ent_after, unsigned *ticket) {
    __shared__ double red[64];
    __shared__ double avg;
    if (threadIdx.x < 32) {
        double s = 0.0;
        if (compute_ent)
            for (int c = threadIdx.x; c < nparts; c += 32) s += o.part[c];
        s = warp_sum(s);
        if (threadIdx.x == 0) avg = s / ((double)o.nxt * o.nyt);
    }
    __syncthreads();
    const size_t n2 = (size_t)o.nyp * px;
    const int j = blockIdx.x;
    CSum rs;
    for (int i = threadIdx.x; i < o.nxp; i += blockDim.x) {
        const size_t op = (size_t)j * px + i;
        wekp[op] = (T)oml_t2p(o, o.wekt, 0.0, i, j);
        if (compute_ent) {
            const T v = (T)oml_t2p(o, o.xfo, avg, i, j);
            ent[op] = v;
            rs.add(((i == 0 || i == o.nxp - 1) ? 0.5 : 1.0) * (double)v);
            for (int k = 1; k < nl - 1; ++k) ent[k * n2 + op] = (T)0;
        }
    }
    if (compute_ent) {
        const CSum t = csum_block_pair(rs, red);
        if (threadIdx.x == 0) { ent_rows[2 * j] = t.s; ent_rows[2 * j + 1] = t.c; }
    }
    // the last CTA: the forcing integrals (ent_xn) and a closed box's zero
    // boundary stress integrals (ekman.F90:60-70)
    if (!last_cta(ticket)) return;
    __syncthreads();
    forcing_integrals_cta<T>(bas[0], ent_after, red);
    if (threadIdx.x == 0) {
        bas[0].frc->txis = 0.0;
        bas[0].frc->txin = 0.0;
    }
}


// ------------------------------------------------- stress on the ocean
// The ocean's wind stress from the atmosphere's lagged layer-1 pressure
// (compute_windstress, atmos_geos_vel, atmos_windstress; windstress.F90:
// 150-314, without the ocean-velocity dependence).
struct TauCpl {
    int ndxr, nxtoar, nytoar, c0, r0;   // load_grid (grid.F90:36-59), 0-based origin
    int nxp_a, nyp_a, px_a;
    double dxa, dya, f0a, ah, fxa, fya, fyb;   // the atmosphere's spacing and BC factors
    double cdat, hma, raoro;
    double *d;                          // [8][nytoar+1][nxtoar+1]: u, ux, uy, uxy, v, vx, vy, vxy
    int udiff;                          // tau_udiff: the stress of the velocity difference
    double hmo, f0o;                    // the ocean's mixed-layer depth and f0
    double *taux_a, *tauy_a;            // the atmosphere's stress [nyp_a][nxp_a] (tau_udiff writes it)
};

// The atmospheric geostrophic velocity and its scaled derivatives at the
// atmospheric p points over the ocean (atmos_geos_vel, :199-259), from the
// channel's dPdx_2bc, dPdy_2bc, dP2dx2_bc, dP2dy2_bc (numerics.F90:410-513)
// applied as there (dp2_dxy = Dx Dy p, dp3_dxxy = Dx Dx Dy p, dp3_dxyy =
// Dx Dyy p), each nested value taken at the points the outer one reads.
template <class T>
__global__ void k_cpl_derivs(TauCpl c, const T *__restrict__ PM1) {
    const int nx = c.nxtoar + 1, ny = c.nytoar + 1, nxp = c.nxp_a, nyp = c.nyp_a;
    auto P = [&](int i, int j) { return (double)PM1[(size_t)j * c.px_a + i]; };
    auto Dy = [&](int i, int j) {
        if (j == 0) return (P(i, 1) - P(i, 0)) / (c.dya * c.ah);
        if (j == nyp - 1) return (P(i, nyp - 1) - P(i, nyp - 2)) / (c.dya * c.ah);
        return (P(i, j + 1) - P(i, j - 1)) / (2.0 * c.dya);
    };
    auto Dyy = [&](int i, int j) {
        if (j == 0) return c.fyb * (P(i, 1) - P(i, 0));
        if (j == nyp - 1) return -c.fyb * (P(i, nyp - 1) - P(i, nyp - 2));
        return c.fya * (P(i, j - 1) + P(i, j + 1) - 2.0 * P(i, j));
    };
    // dPdx_2bc of a field given by F at (i, j), cyclic
    auto Dx = [&](auto F, int i, int j) {
        if (j == 0 || j == nyp - 1) return 0.0;
        if (i == 0 || i == nxp - 1) return (F(1, j) - F(nxp - 2, j)) / (2.0 * c.dxa);
        return (F(i + 1, j) - F(i - 1, j)) / (2.0 * c.dxa);
    };
    auto Dxx = [&](int i, int j) {
        if (j == 0 || j == nyp - 1) return 0.0;
        if (i == 0 || i == nxp - 1) return c.fxa * (P(nxp - 2, j) + P(1, j) - 2.0 * P(0, j));
        return c.fxa * (P(i - 1, j) + P(i + 1, j) - 2.0 * P(i, j));
    };
    auto DxDy = [&](int i, int j) { return Dx(Dy, i, j); };
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nx * ny; idx += gridDim.x * blockDim.x) {
        const int r = idx / nx, col = idx - r * nx;
        const int i = c.c0 + col, j = c.r0 + r;
        const double f0 = c.f0a, dx = c.dxa, dy = c.dya;
        const size_t n = (size_t)nx * ny;
        double *d = c.d + idx;
        d[0] = -Dy(i, j) / f0;
        d[n] = -(dx / f0) * DxDy(i, j);
        d[2 * n] = -(dy / f0) * Dyy(i, j);
        d[3 * n] = -(dx * dy / f0) * Dx(Dyy, i, j);
        d[4 * n] = Dx(P, i, j) / f0;
        d[5 * n] = (dx / f0) * Dxx(i, j);
        d[6 * n] = (dy / f0) * DxDy(i, j);
        d[7 * n] = (dx * dy / f0) * Dx(DxDy, i, j);
    }
}

// The bicubic interpolation of the atmospheric velocity to the ocean's p
// points (the unique bicubic matching each cell's nodal values and scaled
// derivatives, as new_bicubic, bicubic.F90:24-85; a shared cell edge takes
// the later cell) and the drag law there (atmos_windstress, :278-314), times
// the density ratio: the ocean's taux, tauy (compute_windstress, :187-195).
// With tau_udiff (compute_udiff, windstress.F90:255-276) the ocean's lagged
// geostrophic surface velocity (dPdx_2bc / dPdy_2bc of its layer-1 pm) is
// taken from the atmosphere's, the drag coefficient includes both mixed
// layers, and the atmosphere's stress at the p points the two grids share is
// the ocean-resolution one (compute_windstress, :179-187).
template <class T>
__global__ void k_cpl_tau(TauCpl c, OmlDev o, const BasinDev *__restrict__ bo, const T *__restrict__ PMo) {
    const int nx = c.nxtoar + 1, nd = c.ndxr;
    const size_t n = (size_t)nx * (c.nytoar + 1);
    const double cdhfaa = c.udiff ? (c.cdat / c.f0a) * (1.0 / c.hma + c.raoro / c.hmo) : (c.cdat / c.f0a) / c.hma;
    const double qpreaa = 1.0 / (fabs(cdhfaa) * sqrt(2.0));
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < o.nxp * o.nyp; idx += gridDim.x * blockDim.x) {
        const int jo = idx / o.nxp, io = idx - jo * o.nxp;
        const int ci = min(io / nd, c.nxtoar - 1), cj = min(jo / nd, c.nytoar - 1);
        const double s = (double)(io - ci * nd) / nd, t = (double)(jo - cj * nd) / nd;
        const double hs[2] = {1.0 - 3.0 * s * s + 2.0 * s * s * s, 3.0 * s * s - 2.0 * s * s * s};
        const double ks[2] = {s - 2.0 * s * s + s * s * s, -s * s + s * s * s};
        const double ht[2] = {1.0 - 3.0 * t * t + 2.0 * t * t * t, 3.0 * t * t - 2.0 * t * t * t};
        const double kt[2] = {t - 2.0 * t * t + t * t * t, -t * t + t * t * t};
        double uv[2] = {0.0, 0.0};
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const double *f = c.d + 4 * q * n;
            double acc = 0.0;
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b2 = 0; b2 < 2; ++b2) {
                    const size_t k = (size_t)(cj + b2) * nx + ci + a;
                    acc = acc + (f[k] * hs[a] * ht[b2] + f[n + k] * ks[a] * ht[b2] + f[2 * n + k] * hs[a] * kt[b2] +
                                 f[3 * n + k] * ks[a] * kt[b2]);
                }
            uv[q] = acc;
        }
        double u = uv[0], v = uv[1];
        if (c.udiff) {
            double dpx, dpy;
            dpdxy_bc(PMo, bo[0], io, jo, dpx, dpy);
            u = u + dpy / c.f0o;
            v = v - dpx / c.f0o;
        }
        const double shrmag = sqrt(-1.0 + sqrt(1.0 + 4.0 * cdhfaa * cdhfaa * (u * u + v * v)));
        const double cuohf = (qpreaa * cdhfaa) * shrmag;
        const double cdchi = (qpreaa * c.cdat) * shrmag / (1.0 + cuohf * cuohf);
        const double tx = cdchi * (u - cuohf * v), ty = cdchi * (v + cuohf * u);
        const_cast<double *>(o.taux)[idx] = c.raoro * tx;
        const_cast<double *>(o.tauy)[idx] = c.raoro * ty;
        if (c.udiff && io % nd == 0 && jo % nd == 0) {
            const size_t q = (size_t)(c.r0 + jo / nd) * c.nxp_a + c.c0 + io / nd;
            c.taux_a[q] = tx;
            c.tauy_a[q] = ty;
        }
    }
}

// ---------------------------------------------------------------- atmosphere
// The atmospheric mixed layer of a zonally periodic channel (step_aml,
// amlsubs.F90:184-326): temperature ast and height hmixa, advected and
// diffused like the ocean's sst with the cyclic branches of the numerics.
struct AmlDev {
    int nxp, nyp, nxt, nyt, nl, tau_sign;
    double dx, dy, fnot, hm, rho_cp, t1_rel, dt_12, hmamin, hmadmp, xcexp, at2d, at4d, ahmd, bface, dface, cdat;
    double aface[OQG_NLMAX], gp[OQG_NLMAX];
    const double *taux, *tauy;       // [nyp][nxp]
    const double *fnet;              // [nyt][nxt] net heat flux into the mixed layer (fnetat)
    double *ast, *astm, *asn;        // temperature, lagged, next [nyt][nxt]
    double *hmx, *hmxm, *hmn;        // height, lagged, next
    double *wekt, *xfa;              // Ekman pumping, entrainment at T points
    const double *xc1ast;            // set_xc1ast (amlsubs.F90:137-182) [nyt][nxt]
    const double *dtop;              // topography at p points [nyp][nxp] or null
};

// del2_T (numerics.F90:109-145) in a channel (cyclic in x).
__device__ __forceinline__ double aml_del2(const AmlDev &o, const double *t, int i, int j, bool nflux, double nval,
                                           bool sflux, double sval) {
    const int nxt = o.nxt, nyt = o.nyt;
    const double *row = t + (size_t)j * nxt;
    const double c = row[i];
    const double left = c - row[i == 0 ? nxt - 1 : i - 1];
    const double right = row[i == nxt - 1 ? 0 : i + 1] - c;
    const double bot = j == 0 ? (sflux ? c - sval : 0.0) : c - t[(size_t)(j - 1) * nxt + i];
    const double top = j == nyt - 1 ? (nflux ? nval - c : 0.0) : t[(size_t)(j + 1) * nxt + i] - c;
    return (1.0 / (o.dx * o.dx)) * (right - left + top - bot);
}

// adv_diff (mixed_layer.F90:16-58) of one mixed field at T point (i, j) in a
// channel: t the current field (advected), tm the lagged one (diffused).
template <class T>
__device__ __forceinline__ double aml_adv_diff(const AmlDev &o, const T *__restrict__ P1, int px, const double *t,
                                               const double *tm, double d2c, double d4c, bool nflux, double nval,
                                               bool sflux, double sval, int i, int j) {
    const int nxt = o.nxt, nyt = o.nyt, nxp = o.nxp, nyp = o.nyp;
    const double ce = o.tau_sign / (o.fnot * o.hm), cg = 1.0 / o.fnot;   // ycexp = 1 (init_atmos_ml)
    const double *tx = o.taux, *ty = o.tauy;
    auto p = [&](int a, int bb) { return (double)P1[(size_t)bb * px + a]; };
    auto uflux = [&](int f) {          // x-face f of row j, 0..nxt (no wall)
        const double dpdy = (1.0 / o.dy) * (p(f, j + 1) - p(f, j));
        const double uek = ce * (0.5 * (ty[(size_t)(j + 1) * nxp + f] + ty[(size_t)j * nxp + f]));
        const double vel = -cg * dpdy + uek;
        const double mx = (f == 0 || f == nxt) ? 0.5 * (t[(size_t)j * nxt] + t[(size_t)j * nxt + nxt - 1])
                                               : 0.5 * (t[(size_t)j * nxt + f - 1] + t[(size_t)j * nxt + f]);
        return vel * mx;
    };
    auto vflux = [&](int g) {          // y-face g of column i, 0..nyt
        const double vek = -ce * (0.5 * (tx[(size_t)g * nxp + i + 1] + tx[(size_t)g * nxp + i]));
        double vel, my;
        if (g == 0) {
            vel = sflux ? vek : 0.0;
            my = sflux ? t[i] : 0.5 * (t[i] + sval);
        } else if (g == nyp - 1) {
            vel = nflux ? vek : 0.0;
            my = nflux ? t[(size_t)(nyt - 1) * nxt + i] : 0.5 * (t[(size_t)(nyt - 1) * nxt + i] + nval);
        } else {
            const double dpdx = (1.0 / o.dx) * (p(i + 1, g) - p(i, g));
            vel = cg * dpdx + vek;
            my = 0.5 * (t[(size_t)(g - 1) * nxt + i] + t[(size_t)g * nxt + i]);
        }
        return vel * my;
    };
    const double adv = (-1.0 / o.dx) * (uflux(i + 1) - uflux(i)) + (-1.0 / o.dy) * (vflux(j + 1) - vflux(j));
    // del2_T (no flux) of del2_T(tm): the inner one at the five points
    auto d2 = [&](int a, int bb) { return aml_del2(o, tm, a, bb, nflux, nval, sflux, sval); };
    const double e2 = d2(i, j);
    double e4 = 0.0;
    if (d4c != 0.0) {
        const double left = e2 - d2(i == 0 ? nxt - 1 : i - 1, j);
        const double right = d2(i == nxt - 1 ? 0 : i + 1, j) - e2;
        const double bot = j == 0 ? 0.0 : e2 - d2(i, j - 1);
        const double top = j == nyt - 1 ? 0.0 : d2(i, j + 1) - e2;
        e4 = (1.0 / (o.dx * o.dx)) * (right - left + top - bot);
    }
    return adv + d2c * e2 - d4c * e4;
}

// step_aml at T points: the Ekman pumping, both fields' advection and
// diffusion, compute_new_aml (:231-285: height with its diabatic term and
// floor, temperature with the heat and Ekman terms, the convective
// correction) and the T-grid part of the entrainment (:302-306).  The new
// fields go to asn, hmn (the host then rotates the buffers).
template <class T>
__global__ void __launch_bounds__(256) k_aml_step(AmlDev o, const T *__restrict__ P1, int px, double tdta,
                                                   int compute_ent) {
    const int nxt = o.nxt, nyt = o.nyt;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nxt * nyt; idx += gridDim.x * blockDim.x) {
        const int j = idx / nxt, i = idx - j * nxt;
        const double *tx = o.taux, *ty = o.tauy;
        const int nxp = o.nxp;
        const double tyw = 0.5 * (ty[(size_t)(j + 1) * nxp + i] + ty[(size_t)j * nxp + i]);
        const double tye = 0.5 * (ty[(size_t)(j + 1) * nxp + i + 1] + ty[(size_t)j * nxp + i + 1]);
        const double txs = 0.5 * (tx[(size_t)j * nxp + i + 1] + tx[(size_t)j * nxp + i]);
        const double txn = 0.5 * (tx[(size_t)(j + 1) * nxp + i + 1] + tx[(size_t)(j + 1) * nxp + i]);
        const double wk = (1.0 / (o.dx * o.fnot)) * (tye - tyw) - (1.0 / (o.dy * o.fnot)) * (txn - txs);
        o.wekt[idx] = wk;
        const double tmrhs0 = aml_adv_diff(o, P1, px, o.ast, o.astm, o.at2d, o.at4d, false, 0.0, false, 0.0, i, j);
        const double dhdt = aml_adv_diff(o, P1, px, o.hmx, o.hmxm, o.ahmd, 0.0, true, o.hm, true, o.hm, i, j);
        const double am = o.astm[idx], hm_ = o.hmxm[idx];
        const double dT = o.t1_rel - am;
        const double hdrcdt = o.hmadmp / o.rho_cp;
        double hnew = o.hm, dT_fix = 0.0;
        if (dT >= 2.0 * hdrcdt * tdta) {
            const double diab = hdrcdt * (hm_ - o.hm) / dT;
            hnew = hm_ + tdta * (dhdt - diab);
            const double fix = fmax(o.hmamin - hnew, 0.0);
            hnew = hnew + fix;
            dT_fix = fix * dT / hm_;
        }
        const double tmrhs = tmrhs0 + (1.0 / o.rho_cp) * o.fnet[idx] / hm_ - (1.0 / o.hm) * wk * am;
        double astnew = am + tdta * tmrhs + dT_fix;
        const double conv = fmin(0.0, o.t1_rel - astnew);
        astnew = astnew + conv;
        if (compute_ent)
            o.xfa[idx] = o.xcexp * o.bface * (hm_ - o.hm) + o.dface * (o.xcexp * am + (1.0 - o.xcexp) * o.xc1ast[idx]) +
                         (o.xcexp / (tdta * o.dt_12)) * o.hmx[idx] * conv;
        o.asn[idx] = astnew;
        o.hmn[idx] = hnew;
    }
}

// map_T_to_P (numerics.F90:64-107, cyclic branches) at p point (i, j).
__device__ __forceinline__ double aml_t2p(const AmlDev &o, const double *t, int i, int j) {
    const int nxt = o.nxt, nyt = o.nyt, nxp = o.nxp, nyp = o.nyp;
    auto T_ = [&](int a, int bb) { return t[(size_t)bb * nxt + a]; };
    const bool s = j == 0, n = j == nyp - 1;
    if (i == 0 || i == nxp - 1) {
        if (s) return 0.5 * (T_(0, 0) + T_(nxt - 1, 0));
        if (n) return 0.5 * (T_(0, nyt - 1) + T_(nxt - 1, nyt - 1));
        return 0.25 * (T_(0, j) + T_(nxt - 1, j) + T_(0, j - 1) + T_(nxt - 1, j - 1));
    }
    if (s || n) {
        const int r = s ? 0 : nyt - 1;
        return 0.5 * (T_(i - 1, r) + T_(i, r));
    }
    return 0.25 * (T_(i, j) + T_(i - 1, j) + T_(i, j - 1) + T_(i - 1, j - 1));
}

// The boundary stress integrals of a channel (ekman.F90:60-70):
// txis = int_P_dx(taux(:,1) + taux(:,2)) / 2, txin likewise at the north.
__device__ void aml_strips_cta(const AmlDev &o, DevForcing *frc, double *red) {
    const int nxp = o.nxp;
    double s = 0.0, n = 0.0;
    for (int i = threadIdx.x; i < nxp; i += blockDim.x) {
        const double w = (i == 0 || i == nxp - 1) ? 0.5 : 1.0;
        s += w * (o.taux[i] + o.taux[(size_t)nxp + i]);
        n += w * (o.taux[(size_t)(o.nyp - 2) * nxp + i] + o.taux[(size_t)(o.nyp - 1) * nxp + i]);
    }
    double v[2] = {s, n};
    block_sum_n<2>(v);
    (void)red;
    if (threadIdx.x == 0) {
        frc->txis = 0.5 * (v[0] * o.dx);
        frc->txin = 0.5 * (v[1] * o.dx);
    }
}

// The QG forcing from the atmospheric mixed layer, one CTA of 128 threads
// per p row: wekp = map_T_to_P(wekt) and, when computed, ent(:,:,1) =
// map_T_to_P(xfa) + sum_k aface(k) eta(k) + bface dtop with eta(k) =
// (pm_k - pm_{k+1}) / gp_k from the handle's lagged pressure (driver.F90:
// 128-131; amlsubs.F90:308-323), ent(:,:,2:) = 0, and its row sums.
template <class T>
__global__ void __launch_bounds__(128) k_aml_post(AmlDev o, const T *__restrict__ PM, T *wekp, T *ent,
                                                   double *ent_rows, int px, int compute_ent,
                                                   const BasinDev *__restrict__ bas, const T *ent_after,
                                                   unsigned *ticket) {
    __shared__ double red[64];
    const size_t n2 = (size_t)o.nyp * px;
    const int j = blockIdx.x;
    CSum rs;
    for (int i = threadIdx.x; i < o.nxp; i += blockDim.x) {
        const size_t op = (size_t)j * px + i;
        wekp[op] = (T)aml_t2p(o, o.wekt, i, j);
        if (compute_ent) {
            double e1 = aml_t2p(o, o.xfa, i, j);
            for (int k = 0; k < o.nl - 1; ++k)
                e1 = e1 + o.aface[k] * (((double)PM[k * n2 + op] - (double)PM[(k + 1) * n2 + op]) / o.gp[k]);
            e1 = e1 + o.bface * (o.dtop ? o.dtop[(size_t)j * o.nxp + i] : 0.0);
            const T v = (T)e1;
            ent[op] = v;
            rs.add(((i == 0 || i == o.nxp - 1) ? 0.5 : 1.0) * (double)v);
            for (int k = 1; k < o.nl - 1; ++k) ent[k * n2 + op] = (T)0;
        }
    }
    if (compute_ent) {
        const CSum t = csum_block_pair(rs, red);
        if (threadIdx.x == 0) { ent_rows[2 * j] = t.s; ent_rows[2 * j + 1] = t.c; }
    }
    // the last CTA: the boundary stress integrals and the forcing integrals
    if (!last_cta(ticket)) return;
    __syncthreads();
    aml_strips_cta(o, bas[0].frc, red);
    __syncthreads();
    forcing_integrals_cta<T>(bas[0], ent_after, red);
}

// The atmosphere's wind stress from its lagged layer-1 pressure (xforc,
// windstress.F90:102-148, without the ocean-velocity dependence): the
// geostrophic velocity by dPdx_2bc / dPdy_2bc and the quadratic drag law
// with the Ekman-layer turning, at every p point of the channel.
template <class T>
__global__ void __launch_bounds__(256) k_aml_tau(const BasinDev *__restrict__ bas, AmlDev o, const T *__restrict__ PM1,
                                                  double *taux, double *tauy) {
    const BasinDev &b = bas[0];
    const double cdhfaa = (o.cdat / o.fnot) / o.hm;
    const double qpreaa = 1.0 / (fabs(cdhfaa) * sqrt(2.0));
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < o.nxp * o.nyp; idx += gridDim.x * blockDim.x) {
        const int j = idx / o.nxp, i = idx - j * o.nxp;
        double dpdx, dpdy;
        dpdxy_bc(PM1, b, i, j, dpdx, dpdy);
        const double u = -dpdy / o.fnot, v = dpdx / o.fnot;
        const double u2 = 4.0 * cdhfaa * cdhfaa * (u * u + v * v);
        const double shrmag = qpreaa * sqrt(-1.0 + sqrt(1.0 + u2));
        const double cuohf = cdhfaa * shrmag;
        const double cdochi = o.cdat * shrmag / (1.0 + cuohf * cuohf);
        taux[idx] = cdochi * (u - cuohf * v);
        tauy[idx] = cdochi * (v + cuohf * u);
    }
}


// ------------------------------------------------------ the coupled fluxes
// compute_forcing's radiation coefficients (radiate_type, radsubs.F90:15-54).
struct RadFlux {
    double fspco, xlamda, d0up, dmdown, dup0, aup00, adown10, adown11;
};

// bilint (numerics.F90:528-589) of the atmospheric T field at at ocean T
// point (io, jo), 0-based: the ocean's T points from its origin (c0 dxa,
// r0 dya), the atmosphere's at ((i - 1/2) dxa, (j - 1/2) dya) for 1-based
// (i, j); cyclic in x, the first and last T rows held beyond the channel's
// ends.  Indexes stay 1-based and truncate like Fortran's int, as there.
__device__ __forceinline__ double cpl_bilint(const TauCpl &c, const OmlDev &o, const AmlDev &a, const double *at,
                                             int io, int jo) {
    const double dxainv = 1.0 / a.dx, dyainv = 1.0 / a.dy;
    const double xta1 = 0.5 * a.dx, yta1 = 0.5 * a.dy;
    const double xto = (c.c0 * a.dx + io * o.dx) + 0.5 * o.dx;
    int iam = (int)(1.0 + dxainv * (xto - xta1));
    int iap = iam + 1;
    const double xam = iam >= 1 ? (iam - 1) * a.dx + xta1 : xta1 - a.dx;
    const double wpx = dxainv * (xto - xam), wmx = 1.0 - wpx;
    iam = 1 + (iam + a.nxt - 1) % a.nxt;
    iap = 1 + (iap + a.nxt - 1) % a.nxt;
    const double yto = (c.r0 * a.dy + jo * o.dy) + 0.5 * o.dy;
    int jam = (int)(1.0 + dyainv * (yto - yta1));
    int jap = jam + 1;
    jam = min(max(jam, 1), a.nyt);
    jap = min(jap, a.nyt);
    const double wpy = dyainv * (yto - ((jam - 1) * a.dy + yta1)), wmy = 1.0 - wpy;
    const double *rm = at + (size_t)(jam - 1) * a.nxt, *rp = at + (size_t)(jap - 1) * a.nxt;
    return wmx * wmy * rm[iam - 1] + wpx * wmy * rm[iap - 1] + wmx * wpy * rp[iam - 1] + wpx * wpy * rp[iap - 1];
}

// compute_forcing (forcing.F90:18-99): the ocean's net flux at its T points
// and the atmosphere's at its own, one thread per cell of either grid.  An
// atmospheric cell over the ocean sums its ndxr x ndxr ocean cells' upward
// fluxes in the reference's order (rows, then columns), recomputing their
// interpolated temperature.  PM is the atmosphere's lagged pressure (eta_1 =
// (pm_1 - pm_2) / gp_1 at its p points).
template <class T>
__global__ void __launch_bounds__(256) k_cpl_fluxes(TauCpl c, RadFlux r, OmlDev o, AmlDev a,
                                                    const T *__restrict__ PM, int px_a) {
    const double pi = 3.141592653589793;
    const int nto = o.nxt * o.nyt, nta = a.nxt * a.nyt, nd = c.ndxr;
    const double yla = a.nyt * a.dy, ylo = o.nyt * o.dy;
    const double ocfrac = o.dx * o.dy / (a.dx * a.dy);
    double *fnetoc = const_cast<double *>(o.fnet), *fnetat = const_cast<double *>(a.fnet);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nto + nta; idx += gridDim.x * blockDim.x) {
        if (idx < nto) {
            const int jo = idx / o.nxt, io = idx - jo * o.nxt;
            const double asto = cpl_bilint(c, o, a, a.astm, io, jo);
            const double sst = o.datam[idx];
            const double fsp = r.fspco * 0.5 * sin(pi * ((-0.5 * ylo + jo * o.dy) + 0.5 * o.dy) / yla);
            fnetoc[idx] = -fsp - r.dmdown * asto - r.d0up * sst - r.xlamda * (sst - asto);
            continue;
        }
        const int k = idx - nto, ja = k / a.nxt, ia = k - ja * a.nxt;
        const double ast = a.astm[k];
        double f = -r.dup0 * ast - r.fspco * 0.5 * sin(pi * ((-0.5 * yla + ja * a.dy) + 0.5 * a.dy) / yla);
        const int ci = ia - c.c0, cj = ja - c.r0;
        if (ci >= 0 && ci < c.nxtoar && cj >= 0 && cj < c.nytoar) {
            f = f + (r.dmdown - r.dup0) * ast;
            for (int jo = cj * nd; jo < (cj + 1) * nd; ++jo)
                for (int io = ci * nd; io < (ci + 1) * nd; ++io) {
                    const double sst = o.datam[(size_t)jo * o.nxt + io];
                    const double asto = cpl_bilint(c, o, a, a.astm, io, jo);
                    f = f + ocfrac * (r.d0up * sst + r.xlamda * (sst - asto));
                }
        }
        const size_t lay = (size_t)a.nyp * px_a;
        auto eta = [&](int i, int j) {
            const size_t q = (size_t)j * px_a + i;
            return ((double)PM[q] - (double)PM[lay + q]) / a.gp[0];
        };
        const double me = (r.adown11 * 0.25) * (eta(ia, ja) + eta(ia + 1, ja) + eta(ia, ja + 1) + eta(ia + 1, ja + 1));
        double mt = 0.0;
        if (a.dtop) {
            const double *d0 = a.dtop + (size_t)ja * a.nxp, *d1 = d0 + a.nxp;
            mt = ((r.aup00 + r.adown10) * 0.25) * (d0[ia] + d0[ia + 1] + d1[ia] + d1[ia + 1]);
        }
        const double hmafac = -a.hmadmp - r.aup00 - r.adown10;
        fnetat[k] = f - me - mt + hmafac * (a.hmxm[k] - a.hm);
    }
}

}  // namespace oqg
