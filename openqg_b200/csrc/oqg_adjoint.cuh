// oqg_adjoint.cuh -- the adjoint of the closed-box QG step, FP64.
//
// The step (step_qg, core.F90:16-33, then suppress_comp_mode when it is due)
// maps the state (p, pm, q, qm, dpi, dpip) and the Ekman pumping wekp to the
// next state.  It is affine in everything but the Arakawa Jacobian, which is
// bilinear in (p, q); so its transpose, for the input state of the step, is a
// chain of transposed linear operators:
//
//   suppress_comp_mode^T   lam_p' <- lam_p/2, lam_pm' <- lam_pm + lam_p/2, ...
//   ocqbdy^T               the wall q's dependence on the new p
//   modes_to_layers^T      nu_m = sum_k ctm2l(m,k) lam_p_k
//   box_homog^T            alpha's adjoint <hsb_m, nu_m>, the transposed
//                          (nl-1) constraint solve, the area integrals' weights
//   Helmholtz^T            the modal solve itself: the five-point operator with
//                          zero walls, less rdm2_m, is symmetric, so its
//                          inverse is applied again (the forward solver)
//   p_modes_rhs^T          lam_qnew_k = lam_q_k + f0 sum_m ctl2m(k,m) s_m
//   leapfrog^T             lam_qm = lam_qnew; dq's adjoint g = tdt lam_qnew
//   vort_step^T            the Jacobian's two transposes, the friction chain
//                          L^T L^T (L^T) and the drag's L^T, the wind's weight
//
// Every kernel writes each output point once, gathering the terms of the
// forward stencils that read it, so results do not depend on thread order.
// Fields are FP64 [nl][nyp][px] (the handle's layout).  The forward operators:
//   L   del2_P_bc (numerics.F90:410-468): 5-point Laplacian, mixed-BC
//       one-sided terms on the walls, zero in the corners;
//   t   the Arakawa sum of jacobian (numerics.F90:340-388): the step's
//       Jacobian is jac_fac t(p, q), nonzero at interior points only;
//   O   ocqbdy (vorsubs.F90:58-114): wall q from the new p; a corner takes
//       the meridional-wall difference and the A p term twice.
#pragma once

#include "oqg_kernels.cuh"

#define OQG_ADJ_CTAS 592     // CTAs of the grid-stride adjoint kernels (4 per SM)
#define OQG_ADJ_THREADS 256

namespace oqg {

// Weight of f at (iy + dxo, jy + dyo) in (L f)(iy, jy).
__device__ __forceinline__ double lap_weight(const BasinDev &b, int iy, int jy, int dxo, int dyo) {
    const int nxp = b.nxp, nyp = b.nyp;
    const bool zrow = (jy == 0 || jy == nyp - 1);
    const bool wl = iy == 0, wr = iy == nxp - 1;
    double w = 0.0;
    if (!zrow && dyo == 0) {   // dP2dx2_bc
        if (wl) w += dxo == 1 ? b.fx_bc : (dxo == 0 ? -b.fx_bc : 0.0);
        else if (wr) w += dxo == -1 ? b.fx_bc : (dxo == 0 ? -b.fx_bc : 0.0);
        else w += dxo == 0 ? -2.0 * b.fx : b.fx;
    }
    if (!(wl || wr) && dxo == 0) {   // dP2dy2_bc
        if (jy == 0) w += dyo == 1 ? b.fy_bc : (dyo == 0 ? -b.fy_bc : 0.0);
        else if (jy == nyp - 1) w += dyo == -1 ? b.fy_bc : (dyo == 0 ? -b.fy_bc : 0.0);
        else w += dyo == 0 ? -2.0 * b.fy : b.fy;
    }
    return w;
}

// (L^T g)(i, j) of one layer field g.
__device__ __forceinline__ double lapT_at(const BasinDev &b, const double *g, int i, int j) {
    const int di[5] = {0, 1, -1, 0, 0}, dj[5] = {0, 0, 0, 1, -1};
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        const int iy = i + di[t], jy = j + dj[t];
        if (iy < 0 || iy >= b.nxp || jy < 0 || jy >= b.nyp) continue;
        const double w = lap_weight(b, iy, jy, -di[t], -dj[t]);
        if (w != 0.0) s += w * g[(size_t)jy * b.px + iy];
    }
    return s;
}

struct AdjFields {
    double *lp, *lpm, *lq, *lqm;   // adjoint of the state after the step
    double *nu, *s;                // next lam_qm (scratch between steps), modal solution
    double *phi;                   // modal solutions of a unit interior rhs [nl][nyp][px]
    double *lw;                    // accumulated adjoint of wekp [nyp][px]
    double *part;                  // [OQG_ADJ_CTAS][nl-1] partial dots
    double *scal;                  // lam_dpi [0, 8), lam_dpip [8, 16), c_m [16, 24)
    unsigned int *ticket;          // CTAs of k_adj_wall done (0 between launches)
};

// suppress_comp_mode^T (driver.F90:174-189): x' = (x + xm)/2 for x = p, q, dpi.
__global__ void k_adj_suppress(const BasinDev *__restrict__ bas, AdjFields a) {
    pdl_trigger();
    pdl_wait();
    const BasinDev &b = bas[0];
    const size_t n = (size_t)b.nl * b.nyp * b.px;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double hp = 0.5 * a.lp[i], hq = 0.5 * a.lq[i];
        a.lp[i] = hp;
        a.lpm[i] += hp;
        a.lq[i] = hq;
        a.lqm[i] += hq;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int l = 0; l < b.nl - 1; ++l) {
            const double h = 0.5 * a.scal[l];
            a.scal[l] = h;
            a.scal[8 + l] += h;
        }
}

// Unit right-hand side on the interior of every mode (for phi).
__global__ void k_adj_unit_rhs(const BasinDev *__restrict__ bas) {
    const BasinDev &b = bas[0];
    double *rhs = (double *)b.rhs;
    const int n = b.nxin, ny = b.ny;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)b.nl * ny * n;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(idx / ((size_t)ny * n));
        const int rem = (int)(idx - (size_t)m * ny * n);
        const int jj = rem / n, xi = rem - jj * n;
        rhs[((size_t)m * ny + jj) * b.pr + xi] = 1.0;
    }
}

// ocqbdy^T, modes_to_layers^T and box_homog^T.  Per point
//   nu_m = sum_k ctm2l(m,k) (lam_p + O^T lam_q)_k,
// written as the modal solve's right-hand side on the interior; per CTA the
// partial dots <hsb_{m-1}, nu_m>, m >= 1.  The last CTA to finish adds the
// partial dots of all CTAs (fixed order), takes the transposed constraint
// solve (cdhoc^T with the LU of DGETRF: U^T, then L^T, then the row
// interchanges in reverse) and the adjoint of the modal area integrals,
// c_m = dx dy sum_k ctm2l(m,k) lam_ik_k: the modal solution's adjoint is
// then S_m(nu_m) + c_m phi_m, S_m linear and phi_m = S_m(1).  It also
// carries the constraint adjoints through update_mass_constr.
template <int NL>
__global__ void __launch_bounds__(OQG_ADJ_THREADS) k_adj_wall(const BasinDev *__restrict__ bas, AdjFields a) {
    pdl_trigger();
    pdl_wait();
    const BasinDev &b = bas[0];
    constexpr int N = NL - 1;
    const int nxp = b.nxp, nyp = b.nyp, px = b.px, ny = b.ny;
    const size_t n2 = (size_t)nyp * px;
    const double fac = b.qb_fac;
    const double *hsb = (const double *)b.hsb;
    double *rhs = (double *)b.rhs;
    __shared__ double red[32];
    __shared__ int last;
    double dot[N];
#pragma unroll
    for (int m = 0; m < N; ++m) dot[m] = 0.0;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)nyp * nxp;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / nxp), i = (int)(idx - (size_t)j * nxp);
        const size_t o = (size_t)j * px + i;
        const bool zon = (j == 0 || j == nyp - 1), mer = (i == 0 || i == nxp - 1);
        const int cnt = (zon ? 1 : 0) + (mer ? 1 : 0);
        double lq[NL], lpt[NL];
#pragma unroll
        for (int k = 0; k < NL; ++k) lq[k] = cnt ? a.lq[k * n2 + o] : 0.0;
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            double s = a.lp[k * n2 + o];
            if (cnt) {
                s -= fac * lq[k];
                double av = 0.0;
#pragma unroll
                for (int kk = 0; kk < NL; ++kk) av += b.amat[kk + NL * k] * lq[kk];
                s -= cnt * b.fnot * av;
            }
            // x as the inner neighbour of a wall point
            const double *L = a.lq + k * n2;
            if (i == 1) s += fac * L[(size_t)j * px];
            if (i == nxp - 2) s += fac * L[(size_t)j * px + nxp - 1];
            if (i >= 1 && i <= nxp - 2) {
                if (j == 1) s += fac * L[i];
                if (j == nyp - 2) s += fac * L[(size_t)(nyp - 1) * px + i];
            }
            lpt[k] = s;
        }
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < NL; ++k) v += b.ctm2l[m + NL * k] * lpt[k];
            if (m >= 1) dot[m - 1] += hsb[(m - 1) * n2 + o] * v;
            if (!cnt) rhs[((size_t)m * ny + j - 1) * b.pr + i - 1] = v;
        }
    }
#pragma unroll
    for (int m = 0; m < N; ++m) {
        const double v = block_sum(dot[m], red);
        if (threadIdx.x == 0) a.part[blockIdx.x * N + m] = v;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x >= 32) return;
    __threadfence();
    double la[N], z[N];
#pragma unroll
    for (int m = 0; m < N; ++m) la[m] = 0.0;
    for (int c = threadIdx.x; c < (int)gridDim.x; c += 32)
#pragma unroll
        for (int m = 0; m < N; ++m) la[m] += __ldcg(a.part + c * N + m);
#pragma unroll
    for (int m = 0; m < N; ++m) la[m] = warp_sum(la[m]);
    if (threadIdx.x != 0) return;
#pragma unroll
    for (int c = 0; c < N; ++c) {
        double v = la[c];
#pragma unroll
        for (int r = 0; r < c; ++r) v -= b.lu[r + N * c] * z[r];
        z[c] = v / b.lu[c + N * c];
    }
#pragma unroll
    for (int c = N - 1; c >= 0; --c) {
#pragma unroll
        for (int r = c + 1; r < N; ++r) z[c] -= b.lu[r + N * c] * z[r];
    }
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        const int r = b.piv[i];
        if (r != i) { const double t = z[i]; z[i] = z[r]; z[r] = t; }
    }
    // z = lam_r; r_l = dpi_l - (ik_{l+1} - ik_l)
    double lik[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) lik[k] = 0.0;
#pragma unroll
    for (int l = 0; l < N; ++l) { lik[l + 1] -= z[l]; lik[l] += z[l]; }
#pragma unroll
    for (int m = 0; m < NL; ++m) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < NL; ++k) v += b.ctm2l[m + NL * k] * lik[k];
        a.scal[16 + m] = v * b.dx * b.dy;
    }
#pragma unroll
    for (int l = 0; l < N; ++l) {   // dpi' = dpip, dpip' = dpi
        const double ldpi = a.scal[l];
        a.scal[l] = a.scal[8 + l];
        a.scal[8 + l] = ldpi + z[l];
    }
    *a.ticket = 0u;
}

// p_modes_rhs^T and the leapfrog: lam_qnew_k = lam_q_k + f0 sum_m ctl2m(k,m)
// (s_m + c_m phi_m) at interior points, zero on the walls (the step's own
// wall q is replaced by ocqbdy).  wk[m] = f0 ctl2m(k,m), wc[m] = wk[m] c_m.
template <int NL>
__device__ __forceinline__ double lam_qnew(const BasinDev &b, const AdjFields &a, const double (&wk)[NL],
                                           const double (&wc)[NL], int k, int i, int j) {
    if (i <= 0 || i >= b.nxp - 1 || j <= 0 || j >= b.nyp - 1) return 0.0;
    const size_t n2 = (size_t)b.nyp * b.px, o = (size_t)j * b.px + i;
    double v = a.lq[k * n2 + o];
#pragma unroll
    for (int m = 0; m < NL; ++m) v += wk[m] * a.s[m * n2 + o] + wc[m] * a.phi[m * n2 + o];
    return v;
}

// The Arakawa sum t(p, q) at the centre of 3x3 blocks P, Q ([dy+1][dx+1]).
__device__ __forceinline__ double arakawa9(const double (&P)[3][3], const double (&Q)[3][3]) {
    return (Q[1][2] - Q[1][0]) * (P[2][1] - P[0][1]) - (Q[2][1] - Q[0][1]) * (P[1][2] - P[1][0]) +
           Q[1][2] * (P[2][2] - P[0][2]) - Q[1][0] * (P[2][0] - P[0][0]) - Q[2][1] * (P[2][2] - P[2][0]) +
           Q[0][1] * (P[0][2] - P[0][0]) + P[2][1] * (Q[2][2] - Q[2][0]) - P[0][1] * (Q[0][2] - Q[0][0]) -
           P[1][2] * (Q[2][2] - Q[0][2]) + P[1][0] * (Q[2][0] - Q[0][0]);
}

// vort_step^T, on 2-D tiles of ADJ_TX x ADJ_TY points of one layer.  With
// g = lam_qnew (staged with a halo of 3),
//   lam_qm_in = g                                          (into nu)
//   lam_q_in  = lam_qm_out + tdt jac_fac t_q^T(g; p)        (into lqm, in place)
//   lam_p_in  = lam_pm_out + tdt jac_fac t_p^T(g; q)        (into lpm, in place)
//   lam_pm_in = tdt (c2 t2 - c4 t3 - [k = kt] c_drag t1)    (into lp)
//   lw += tdt c_wind g (layer 1)
// with t1 = L^T g, t2 = L^T t1, t3 = L^T t2 built in shared memory (halos
// 2, 1, 0).  g is zero off the interior, so t1 is the plain five-point sum
// of g; the wall rows of L enter t2 and t3.  P, Q: p and q of the step's
// input state (halo 1: every term of the Arakawa sum's transpose reads the
// 3x3 block around its point).  Where that block is interior, the sum's skew
// symmetry (it conserves energy and enstrophy, numerics.F90:340-388) gives
// t_q^T(g; p) = -t(p, g) and t_p^T(g; q) = -t(g, q).
#define ADJ_TX 32
#define ADJ_TY 16

template <int NL, bool ALL>
__global__ void __launch_bounds__(256, 3) k_adj_vort(const BasinDev *__restrict__ bas, AdjFields a,
                                                  const double *__restrict__ P, const double *__restrict__ Q,
                                                  double tdt, int tiles_x, int tiles_y) {
    pdl_trigger();
    pdl_wait();
    const BasinDev &b = bas[0];
    const int nxp = b.nxp, nyp = b.nyp, px = b.px;
    const size_t n2 = (size_t)nyp * px;
    constexpr int GW = ADJ_TX + 6, GH = ADJ_TY + 6;   // g, halo 3
    constexpr int AW = ADJ_TX + 4, AH = ADJ_TY + 4;   // t1, halo 2
    constexpr int BW = ADJ_TX + 2, BH = ADJ_TY + 2;   // t2, p, q, halo 1
    constexpr int NG = ALL ? NL : 1;                  // layers of g held at once
    __shared__ double G[NG][GH][GW], T1[AH][AW], T2[BH][BW], Ps[BH][BW], Qs[BH][BW];
    const int tile = blockIdx.x % (tiles_x * tiles_y);
    const int x0 = (tile % tiles_x) * ADJ_TX, y0 = (tile / tiles_x) * ADJ_TY;
    const double fx = b.fx, fy = b.fy;
    if (ALL) {
        // every layer's g from one pass over the modal solutions (each s_m
        // and phi_m value is read once for all layers)
        __shared__ double sW[2][NL][NL];   // f0 ctl2m(k,m) and its product with c_m
        if (threadIdx.x < NL * NL) {
            const int k = threadIdx.x / NL, m = threadIdx.x - k * NL;
            sW[0][k][m] = b.fnot * b.ctl2m[k + NL * m];
            sW[1][k][m] = sW[0][k][m] * a.scal[16 + m];
        }
        __syncthreads();
        for (int e = threadIdx.x; e < GH * GW; e += 256) {
            const int r = e / GW, c = e - r * GW;
            const int i = x0 - 3 + c, j = y0 - 3 + r;
            if (i <= 0 || i >= nxp - 1 || j <= 0 || j >= nyp - 1) {
#pragma unroll
                for (int k = 0; k < NL; ++k) G[k % NG][r][c] = 0.0;
                continue;
            }
            const size_t o = (size_t)j * px + i;
            double sv[NL], pv[NL];
#pragma unroll
            for (int m = 0; m < NL; ++m) {
                sv[m] = a.s[m * n2 + o];
                pv[m] = a.phi[m * n2 + o];
            }
#pragma unroll
            for (int k = 0; k < NL; ++k) {
                double v = a.lq[k * n2 + o];
#pragma unroll
                for (int m = 0; m < NL; ++m) v += sW[0][k][m] * sv[m] + sW[1][k][m] * pv[m];
                G[k % NG][r][c] = v;
            }
        }
    }
#pragma unroll 1
    for (int kk = 0; kk < (ALL ? NL : 1); ++kk) {
    const int k = ALL ? kk : blockIdx.x / (tiles_x * tiles_y);
    double (*Gk)[GW] = G[ALL ? kk : 0];
    if (!ALL) {
        double wk[NL], wc[NL];
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            wk[m] = b.fnot * b.ctl2m[k + NL * m];
            wc[m] = wk[m] * a.scal[16 + m];
        }
        // constant strides (256 threads) let the staging loop unroll and keep
        // its loads in flight together
#pragma unroll
        for (int e = threadIdx.x; e < GH * GW; e += 256) {
            const int r = e / GW, c = e - r * GW;
            Gk[r][c] = lam_qnew<NL>(b, a, wk, wc, k, x0 - 3 + c, y0 - 3 + r);
        }
    } else if (kk > 0) {
        __syncthreads();   // the previous layer's tiles are no longer read
    }
    const double *p = P + k * n2, *q = Q + k * n2;
#pragma unroll
    for (int e = threadIdx.x; e < BH * BW; e += 256) {
        const int r = e / BW, c = e - r * BW;
        const int i = x0 - 1 + c, j = y0 - 1 + r;
        const bool in = i >= 0 && i < nxp && j >= 0 && j < nyp;
        Ps[r][c] = in ? p[(size_t)j * px + i] : 0.0;
        Qs[r][c] = in ? q[(size_t)j * px + i] : 0.0;
    }
    __syncthreads();
    // t1 = L^T g: g vanishes off the interior, where L's rows are the plain ones
#pragma unroll
    for (int e = threadIdx.x; e < AH * AW; e += 256) {
        const int r = e / AW, c = e - r * AW;
        const int i = x0 - 2 + c, j = y0 - 2 + r;
        double v = 0.0;
        if (i >= 0 && i < nxp && j >= 0 && j < nyp)
            v = fx * (Gk[r + 1][c] + Gk[r + 1][c + 2] - 2.0 * Gk[r + 1][c + 1]) +
                fy * (Gk[r][c + 1] + Gk[r + 2][c + 1] - 2.0 * Gk[r + 1][c + 1]);
        T1[r][c] = v;
    }
    __syncthreads();
    // t2 = L^T t1 (the wall rows of L enter here)
    const int di[5] = {0, 1, -1, 0, 0}, dj[5] = {0, 0, 0, 1, -1};
    for (int e = threadIdx.x; e < BH * BW; e += 256) {
        const int r = e / BW, c = e - r * BW;
        const int i = x0 - 1 + c, j = y0 - 1 + r;
        double v = 0.0;
        if (i >= 2 && i <= nxp - 3 && j >= 2 && j <= nyp - 3) {
            v = fx * (T1[r + 1][c] + T1[r + 1][c + 2] - 2.0 * T1[r + 1][c + 1]) +
                fy * (T1[r][c + 1] + T1[r + 2][c + 1] - 2.0 * T1[r + 1][c + 1]);
        } else if (i >= 0 && i < nxp && j >= 0 && j < nyp) {
#pragma unroll
            for (int t = 0; t < 5; ++t) {
                const int iy = i + di[t], jy = j + dj[t];
                if (iy < 0 || iy >= nxp || jy < 0 || jy >= nyp) continue;
                v += lap_weight(b, iy, jy, -di[t], -dj[t]) * T1[r + 1 + dj[t]][c + 1 + di[t]];
            }
        }
        T2[r][c] = v;
    }
    __syncthreads();
    const double s = tdt * b.jac_fac;
    const int cx = threadIdx.x & 31;
    for (int ry = threadIdx.x >> 5; ry < ADJ_TY; ry += 8) {
        const int i = x0 + cx, j = y0 + ry;
        if (i >= nxp || j >= nyp) continue;
        const int rg = ry + 3, cg = cx + 3;   // in G
        const int rb = ry + 1, cb = cx + 1;   // in T2, Ps, Qs
        double g3[3][3], p3[3][3], q3[3][3];
#pragma unroll
        for (int c = -1; c <= 1; ++c)
#pragma unroll
            for (int e = -1; e <= 1; ++e) {
                g3[c + 1][e + 1] = Gk[rg + c][cg + e];
                p3[c + 1][e + 1] = Ps[rb + c][cb + e];
                q3[c + 1][e + 1] = Qs[rb + c][cb + e];
            }
        double sq = 0.0, sp = 0.0, t3 = 0.0;
        if (i >= 2 && i <= nxp - 3 && j >= 2 && j <= nyp - 3) {
            sq = -arakawa9(p3, g3);
            sp = -arakawa9(g3, q3);
            t3 = fx * (T2[rb][cb - 1] + T2[rb][cb + 1] - 2.0 * T2[rb][cb]) +
                 fy * (T2[rb - 1][cb] + T2[rb + 1][cb] - 2.0 * T2[rb][cb]);
        } else {
            // every interior y = x - (e, c) whose Arakawa stencil holds x;
            // P3, Q3 index the 3x3 block around x
#define P3(ii, jj) p3[(jj) + 1][(ii) + 1]
#define Q3(ii, jj) q3[(jj) + 1][(ii) + 1]
#pragma unroll
            for (int c = -1; c <= 1; ++c)
#pragma unroll
                for (int e = -1; e <= 1; ++e) {
                    if (e == 0 && c == 0) continue;   // t(y) does not read q(y) or p(y)
                    const double gy = g3[1 - c][1 - e];
                    if (gy == 0.0) continue;          // walls and outside
                    double cq, cp;
                    if (c == 0) {          // x = y + (e, 0), y = x - (e, 0)
                        const double dpy = (P3(-e, 1) - P3(-e, -1)) + (P3(0, 1) - P3(0, -1));
                        const double dqy = (Q3(-e, 1) - Q3(-e, -1)) + (Q3(0, 1) - Q3(0, -1));
                        cq = e * dpy;
                        cp = -e * dqy;
                    } else if (e == 0) {   // x = y + (0, c)
                        const double dpx = (P3(1, -c) - P3(-1, -c)) + (P3(1, 0) - P3(-1, 0));
                        const double dqx = (Q3(1, -c) - Q3(-1, -c)) + (Q3(1, 0) - Q3(-1, 0));
                        cq = -c * dpx;
                        cp = c * dqx;
                    } else {               // diagonal x = y + (e, c)
                        cq = (double)(e * c) * (P3(-e, 0) - P3(0, -c));
                        cp = (double)(e * c) * (Q3(0, -c) - Q3(-e, 0));
                    }
                    sq += cq * gy;
                    sp += cp * gy;
                }
#undef P3
#undef Q3
#pragma unroll
            for (int t = 0; t < 5; ++t) {
                const int iy = i + di[t], jy = j + dj[t];
                if (iy < 0 || iy >= nxp || jy < 0 || jy >= nyp) continue;
                t3 += lap_weight(b, iy, jy, -di[t], -dj[t]) * T2[rb + dj[t]][cb + di[t]];
            }
        }
        const size_t o = k * n2 + (size_t)j * px + i;
        const double g = g3[1][1];
        a.nu[o] = g;
        a.lqm[o] += s * sq;
        a.lpm[o] += s * sp;
        double v = b.c2[k] * T2[rb][cb] - b.c4[k] * t3;
        if (k == b.kt) v -= b.c_drag * T1[ry + 2][cx + 2];
        a.lp[o] = tdt * v;
        if (k == 0) a.lw[(size_t)j * px + i] += tdt * b.c_wind * g;
    }
    }   // layers
}

// The transpose of set_state (qcomp, vorsubs.F90:27-56; init_mass_constr,
// constraint.F90:145-165) applied to the adjoint state:
//   g_p  = lam_p  + L^T lam_q / f0  - f0 A^T lam_q  + M^T lam_dpi
//   g_pm = lam_pm + L^T lam_qm / f0 - f0 A^T lam_qm + M^T lam_dpip
// with M^T d at layer k = dz_sign w (d_k - d_{k-1}) (trapezoid weights w dx dy).
template <int NL>
__global__ void __launch_bounds__(OQG_ADJ_THREADS) k_adj_init(const BasinDev *__restrict__ bas, AdjFields a,
                                                              double *gp, double *gpm) {
    const BasinDev &b = bas[0];
    const int nxp = b.nxp, nyp = b.nyp, px = b.px;
    const size_t n2 = (size_t)nyp * px;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)nyp * nxp;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / nxp), i = (int)(idx - (size_t)j * nxp);
        const size_t o = (size_t)j * px + i;
        const double w = ((i == 0 || i == nxp - 1) ? 0.5 : 1.0) * ((j == 0 || j == nyp - 1) ? 0.5 : 1.0) * b.dx * b.dy;
        for (int f = 0; f < 2; ++f) {
            const double *LP = f ? a.lpm : a.lp, *LQ = f ? a.lqm : a.lq, *LD = a.scal + (f ? 8 : 0);
            double *G = f ? gpm : gp;
            double lq[NL];
#pragma unroll
            for (int k = 0; k < NL; ++k) lq[k] = LQ[k * n2 + o];
#pragma unroll
            for (int l = 0; l < NL; ++l) {
                double v = LP[l * n2 + o] + lapT_at(b, LQ + l * n2, i, j) / b.fnot;
                double av = 0.0;
#pragma unroll
                for (int k = 0; k < NL; ++k) av += b.amat[k + NL * l] * lq[k];
                v -= b.fnot * av;
                const double dl = (l < NL - 1 ? LD[l] : 0.0) - (l > 0 ? LD[l - 1] : 0.0);
                v += b.dz_sign * w * dl;
                G[l * n2 + o] = v;
            }
        }
    }
}

}  // namespace oqg
