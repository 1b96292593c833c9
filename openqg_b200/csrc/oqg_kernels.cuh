// oqg_kernels.cuh -- the per-step kernels of the QG core (sm_100a).
//
// One step_qg (qg/core.F90:16-33) is four launches, one per dependent phase:
//   k_vort   vort_step (qg/vorticity.F90:14-103) + p_modes_rhs (qg/modes.F90:248-266)
//            2-D tiles staged in shared memory; the layer loop runs inside the
//            CTA so the modal right-hand side is formed in registers.
//   k_xfwd   forward x-transform of solve_inhomog_box / _cyclic
//            (qg/inhomog.F90:170-255): DST-I (box) or r2c FFT (channel).
//   k_ysolve Thomas solve in y per (mode, wavenumber) (inhomog.F90:187-199),
//            one warp per column as a warp-parallel affine scan; its last CTA
//            runs the scalar phase: update_mass_constr (constraint.F90:167-179),
//            box_homog's 2x2 solve (homog.F90:331-366) or step_constraints +
//            cyclic_homog (constraint.F90:182-215, homog.F90:280-329), and the
//            suppress_comp_mode schedule (openqg.F90:485-487).
//   k_xinv   inverse x-transform + homogeneous correction + modes_to_layers
//            (modes.F90:268-284) + ocqbdy (vorsubs.F90:58-114) +
//            suppress_comp_mode (driver.F90:174-189).
// Every launch takes a work list, so one launch serves one basin or an
// ensemble of basins of uneven size.
#pragma once

#include "oqg_dev.cuh"
#include "oqg_fft.cuh"

namespace oqg {

// ------------------------------------------------------------------ helpers
template <class T> __device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

__device__ __forceinline__ double shfl_up_d(double v, int o) { return __shfl_up_sync(0xffffffffu, v, o); }
__device__ __forceinline__ double shfl_dn_d(double v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic CTA sum (result valid in every thread). red: >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        s = lane < nw ? red[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0) red[0] = s;
    }
    __syncthreads();
    s = red[0];
    __syncthreads();
    return s;
}

// ------------------------------------------------------------------ k_vort
#define VTX 64
#define VTY 16
#define VTHREADS 256

// Laplacian with the mixed wall condition (del2_P_bc, numerics.F90:410-468) at
// tile point (r, c) of s (leading dimension ld); gi, gj are global indices
// (canonical columns for a channel).
template <class T>
__device__ __forceinline__ T lap_bc(const T *s, int ld, int r, int c, int gi, int gj,
                                    const BasinDev &b) {
    const T fx = (T)b.fx, fy = (T)b.fy, fxb = (T)b.fx_bc, fyb = (T)b.fy_bc;
    const T v = s[r * ld + c];
    T xp, yp;
    const bool wall_x = !b.cyclic && (gi == 0 || gi == b.nxp - 1);
    if (gj == 0 || gj == b.nyp - 1) xp = (T)0;
    else if (!b.cyclic && gi == 0) xp = fxb * (s[r * ld + c + 1] - v);
    else if (!b.cyclic && gi == b.nxp - 1) xp = -(fxb * (v - s[r * ld + c - 1]));
    else xp = fx * (s[r * ld + c - 1] + s[r * ld + c + 1] - (T)2 * v);
    if (wall_x) yp = (T)0;
    else if (gj == 0) yp = fyb * (s[(r + 1) * ld + c] - v);
    else if (gj == b.nyp - 1) yp = -(fyb * (v - s[(r - 1) * ld + c]));
    else yp = fy * (s[(r - 1) * ld + c] + s[(r + 1) * ld + c] - (T)2 * v);
    return xp + yp;
}

// Arakawa Jacobian J(q, p) (numerics.F90:340-373) at tile point (r, c) of
// the halo-1 tiles sp, sq.
template <class T>
__device__ __forceinline__ T arakawa(const T *sp, const T *sq, int ld, int r, int c, int gi,
                                     int gj, const BasinDev &b) {
    const bool zx = !b.cyclic && (gi == 0 || gi == b.nxp - 1);   // dPdx_2 = 0 here
    const bool zy = (gj == 0 || gj == b.nyp - 1);                 // dPdy_2 = 0 here
#define SP(rr, cc) sp[(rr) * ld + (cc)]
#define SQ(rr, cc) sq[(rr) * ld + (cc)]
    T pxc = zx ? (T)0 : SP(r, c + 1) - SP(r, c - 1);
    T pyc = zy ? (T)0 : SP(r + 1, c) - SP(r - 1, c);
    T qxc = zx ? (T)0 : SQ(r, c + 1) - SQ(r, c - 1);
    T qyc = zy ? (T)0 : SQ(r + 1, c) - SQ(r - 1, c);
    T A = (T)0, Bv = (T)0, C = (T)0, D = (T)0;
    if (!zx) {
        // dPdx_2(q * dPdy_2(p)) and dPdx_2(p * dPdy_2(q)) at column gi: values
        // at gi +- 1 of row gj; dPdy_2 is zero on the zonal walls.
        T pyR = zy ? (T)0 : SP(r + 1, c + 1) - SP(r - 1, c + 1);
        T pyL = zy ? (T)0 : SP(r + 1, c - 1) - SP(r - 1, c - 1);
        T qyR = zy ? (T)0 : SQ(r + 1, c + 1) - SQ(r - 1, c + 1);
        T qyL = zy ? (T)0 : SQ(r + 1, c - 1) - SQ(r - 1, c - 1);
        A = SQ(r, c + 1) * pyR - SQ(r, c - 1) * pyL;
        D = SP(r, c + 1) * qyR - SP(r, c - 1) * qyL;
    }
    if (!zy) {
        // dPdy_2(q * dPdx_2(p)) and dPdy_2(p * dPdx_2(q)) at row gj: dPdx_2 at
        // column gi is zero on box walls.
        T pxU = zx ? (T)0 : SP(r + 1, c + 1) - SP(r + 1, c - 1);
        T pxD = zx ? (T)0 : SP(r - 1, c + 1) - SP(r - 1, c - 1);
        T qxU = zx ? (T)0 : SQ(r + 1, c + 1) - SQ(r + 1, c - 1);
        T qxD = zx ? (T)0 : SQ(r - 1, c + 1) - SQ(r - 1, c - 1);
        Bv = SQ(r + 1, c) * pxU - SQ(r - 1, c) * pxD;
        C = SP(r + 1, c) * qxU - SP(r - 1, c) * qxD;
    }
#undef SP
#undef SQ
    T t = qxc * pyc - qyc * pxc + A - Bv + C - D;
    return (T)b.jac_fac * t;
}

// Loads rows [jlo, jlo+nr) x cols [ilo, ilo+nc) of layer k of field f into s
// (leading dimension nc); outside the basin -> 0; channel columns wrap.
template <class T>
__device__ __forceinline__ void load_tile(T *s, const T *__restrict__ f, const BasinDev &b, int k,
                                          int jlo, int nr, int ilo, int nc) {
    const int N = b.nxp - 1;
    for (int idx = threadIdx.x; idx < nr * nc; idx += blockDim.x) {
        int r = idx / nc, c = idx - r * nc;
        int j = jlo + r, i = ilo + c;
        T v = (T)0;
        if (j >= 0 && j < b.nyp) {
            if (b.cyclic) {
                i %= N;
                if (i < 0) i += N;
                v = ldg(f + ((size_t)k * b.nyp + j) * b.px + i);
            } else if (i >= 0 && i < b.nxp) {
                v = ldg(f + ((size_t)k * b.nyp + j) * b.px + i);
            }
        }
        s[idx] = v;
    }
}

template <class T, int NL>
__global__ void __launch_bounds__(VTHREADS)
k_vort(const BasinDev *__restrict__ bas, const Work *__restrict__ work, int par, double tdt) {
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    const int tile_x = w.block % b.tiles_x, tile_y = w.block / b.tiles_x;
    const int i0 = tile_x * VTX, j0 = tile_y * VTY;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sPM = reinterpret_cast<T *>(smem_raw);
    T *sD2 = sPM + (VTY + 6) * (VTX + 6);
    T *sD4 = sD2 + (VTY + 4) * (VTX + 4);
    T *sP = sD4 + (VTY + 2) * (VTX + 2);
    T *sQ = sP + (VTY + 2) * (VTX + 2);
    __shared__ double red[32];

    const T *P = (const T *)b.F[par];
    const T *PM = (const T *)b.F[1 - par];
    const T *Q = (const T *)b.F[2 + par];
    T *QM = (T *)b.F[3 - par];
    const T *WEK = (const T *)b.wekp;
    const T *ENT = (const T *)b.ent;
    const int N = b.nxp - 1;

    double acc[4][NL];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int m = 0; m < NL; ++m) acc[u][m] = 0.0;

    const int tx = threadIdx.x & (VTX - 1);
    const int ty0 = threadIdx.x >> 6;   // 0..3
    // channel strip integrals are formed by tiles holding rows 0, 1, nyp-2, nyp-1
    const bool strips = b.cyclic &&
        (j0 <= 1 || j0 + VTY > b.nyp - 2);

#pragma unroll 1
    for (int k = 0; k < NL; ++k) {
        load_tile(sPM, PM, b, k, j0 - 3, VTY + 6, i0 - 3, VTX + 6);
        load_tile(sP, P, b, k, j0 - 1, VTY + 2, i0 - 1, VTX + 2);
        load_tile(sQ, Q, b, k, j0 - 1, VTY + 2, i0 - 1, VTX + 2);
        __syncthreads();
        // del2p on the halo-2 region
        for (int idx = threadIdx.x; idx < (VTY + 4) * (VTX + 4); idx += blockDim.x) {
            int r = idx / (VTX + 4), c = idx - r * (VTX + 4);
            int gj = j0 - 2 + r, gi = i0 - 2 + c;
            T v = (T)0;
            if (gj >= 0 && gj < b.nyp) {
                if (b.cyclic) {
                    int ci = gi % N; if (ci < 0) ci += N;
                    v = lap_bc(sPM, VTX + 6, r + 1, c + 1, ci, gj, b);
                } else if (gi >= 0 && gi < b.nxp) {
                    v = lap_bc(sPM, VTX + 6, r + 1, c + 1, gi, gj, b);
                }
            }
            sD2[idx] = v;
        }
        __syncthreads();
        // d4p on the halo-1 region
        for (int idx = threadIdx.x; idx < (VTY + 2) * (VTX + 2); idx += blockDim.x) {
            int r = idx / (VTX + 2), c = idx - r * (VTX + 2);
            int gj = j0 - 1 + r, gi = i0 - 1 + c;
            T v = (T)0;
            if (gj >= 0 && gj < b.nyp) {
                if (b.cyclic) {
                    int ci = gi % N; if (ci < 0) ci += N;
                    v = lap_bc(sD2, VTX + 4, r + 1, c + 1, ci, gj, b);
                } else if (gi >= 0 && gi < b.nxp) {
                    v = lap_bc(sD2, VTX + 4, r + 1, c + 1, gi, gj, b);
                }
            }
            sD4[idx] = v;
        }
        __syncthreads();

        double sq[OQG_NQ];
#pragma unroll
        for (int q = 0; q < OQG_NQ; ++q) sq[q] = 0.0;

#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int ty = ty0 + 4 * u;
            const int gj = j0 + ty, gi = i0 + tx;
            if (gj >= b.nyp || gi >= b.nxp) continue;
            int ci = gi;
            if (b.cyclic && ci == N) ci = 0;
            T d4 = sD4[(ty + 1) * (VTX + 2) + tx + 1];
            T d6 = lap_bc(sD4, VTX + 2, ty + 1, tx + 1, ci, gj, b);
            T jac = arakawa(sP, sQ, VTX + 2, ty + 1, tx + 1, ci, gj, b);
            T dq = jac + (T)b.c2[k] * d4 - (T)b.c4[k] * d6;
            const size_t o2 = (size_t)gj * b.px + gi;
            if (k == 0) {
                T e1 = ENT ? ldg(ENT + o2) : (T)0;
                dq = dq + (T)b.c_ent1 * e1 + (T)b.c_wind * ldg(WEK + o2);
            }
            if (k == 1 && ENT) dq = dq - (T)b.c_ent2 * ldg(ENT + o2);
            T d2 = sD2[(ty + 2) * (VTX + 4) + tx + 2];
            if (k == b.kt) dq = dq - (T)b.c_drag * d2;
            const size_t o3 = ((size_t)k * b.nyp + gj) * b.px + gi;
            T qn = QM[o3] + (T)tdt * dq;
            QM[o3] = qn;
            // modal right-hand side, FP64 (p_modes_rhs)
            double ql = (double)qn - b.beta * b.yprel[gj];
            if (k == b.kt && b.topo_active) ql -= b.ddyn[(size_t)gj * b.px + gi];
#pragma unroll
            for (int m = 0; m < NL; ++m) acc[u][m] += ql * b.ctl2m[k + NL * m];
            if (strips && gi < N) {
                // channel strip integrands (vorticity.F90:84-101, numerics.F90:374-386)
                const int ld = VTX + 2, r = ty + 1, c = tx + 1;
                if (gj == 0) {
                    T px1 = sP[(r + 1) * ld + c + 1] - sP[(r + 1) * ld + c - 1];
                    sq[0] += (double)(sQ[r * ld + c] * px1);
                    sq[4] += (double)(sD2[(ty + 3) * (VTX + 4) + tx + 2] - d2);
                    sq[6] += (double)(sD4[(ty + 2) * (VTX + 2) + tx + 1] - d4);
                    if (k == b.kt)
                        sq[8] += (double)(sPM[(ty + 4) * (VTX + 6) + tx + 3] - sPM[(ty + 3) * (VTX + 6) + tx + 3]);
                }
                if (gj == 1) {
                    T px1 = sP[r * ld + c + 1] - sP[r * ld + c - 1];
                    sq[1] += (double)(sQ[r * ld + c] * px1);
                }
                if (gj == b.nyp - 1) {
                    T pxs = sP[(r - 1) * ld + c + 1] - sP[(r - 1) * ld + c - 1];
                    sq[2] += (double)(sQ[r * ld + c] * pxs);
                    sq[5] += (double)(d2 - sD2[(ty + 1) * (VTX + 4) + tx + 2]);
                    sq[7] += (double)(d4 - sD4[ty * (VTX + 2) + tx + 1]);
                    if (k == b.kt)
                        sq[9] += (double)(sPM[(ty + 3) * (VTX + 6) + tx + 3] - sPM[(ty + 2) * (VTX + 6) + tx + 3]);
                }
                if (gj == b.nyp - 2) {
                    T px1 = sP[r * ld + c + 1] - sP[r * ld + c - 1];
                    sq[3] += (double)(sQ[r * ld + c] * px1);
                }
            }
        }
        if (strips) {
            double *pt = b.part_tile + ((size_t)w.block * b.nl + k) * OQG_NQ;
#pragma unroll 1
            for (int q = 0; q < OQG_NQ; ++q) {
                double s = block_sum(sq[q], red);
                if (threadIdx.x == 0) pt[q] = s;
            }
        }
        __syncthreads();
    }

    // write the modal right-hand side of the interior points
    T *RHS = (T *)b.rhs;
    const int ioff = b.cyclic ? 0 : 1;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int gj = j0 + ty0 + 4 * u, gi = i0 + tx;
        if (gj < 1 || gj > b.nyp - 2) continue;
        const int xi = gi - ioff;
        if (xi < 0 || xi >= b.nxin) continue;
#pragma unroll
        for (int m = 0; m < NL; ++m)
            RHS[((size_t)m * b.ny + (gj - 1)) * b.pr + xi] = (T)(b.fnot * acc[u][m]);
    }
}

// ------------------------------------------------------------------ k_xfwd
// Threads per transform TT = ceil(M/E); G = blockDim/TT transforms per CTA.
template <class T, int E>
__global__ void k_xfwd(const BasinDev *__restrict__ bas, const Work *__restrict__ work,
                       const void *rhs_override) {
    typedef typename C2<T>::t T2;
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2 *zs = reinterpret_cast<T2 *>(smem_raw);
    const int M = b.M, TT = (M + E - 1) / E, G = blockDim.x / TT;
    const int g = threadIdx.x / TT, t = threadIdx.x - g * TT;
    const int npm = (b.ny + 1) >> 1;          // row pairs per mode
    const int pair = w.block * G + g;
    const bool live = g < G && pair < b.nl * npm;
    const int m = live ? pair / npm : 0;
    const int j = live ? 2 * (pair - m * npm) : 0;
    const bool two = live && (j + 1 < b.ny);
    T2 *z = zs + (size_t)(g < G ? g : 0) * M;
    const T *R = (const T *)(rhs_override ? rhs_override : b.rhs);
    const T *x = R + ((size_t)m * b.ny + j) * b.pr;
    const T *y = x + b.pr;
    const T2 *tw = (const T2 *)b.tw;
    const int n = b.nxin;
    if (!b.cyclic) {
        // odd extension of two rows: z_0 = z_{n+1} = 0, z_{M-jj} = -z_jj
        if (live) {
            for (int jj = t; jj < M; jj += TT) {
                T2 v;
                if (jj == 0 || jj == n + 1) { v.x = (T)0; v.y = (T)0; }
                else if (jj <= n) { v.x = x[jj - 1]; v.y = two ? y[jj - 1] : (T)0; }
                else { int s = M - jj; v.x = -x[s - 1]; v.y = two ? -y[s - 1] : (T)0; }
                z[jj] = v;
            }
        }
    } else {
        if (live) {
            for (int jj = t; jj < M; jj += TT) {
                T2 v;
                v.x = x[jj];
                v.y = two ? y[jj] : (T)0;
                z[jj] = v;
            }
        }
    }
    __syncthreads();
    fft_smem<T, E>(z, M, b.rad, b.nrad, tw, live ? t : TT, TT);
    if (!live) return;
    if (!b.cyclic) {
        T *S = (T *)b.spec;
        T *sx = S + ((size_t)m * b.ny + j) * b.pk;
        T *sy = sx + b.pk;
        for (int kk = t; kk < n; kk += TT) {
            T2 v = z[kk + 1];
            sx[kk] = -v.y;
            if (two) sy[kk] = v.x;
        }
    } else {
        T2 *S = (T2 *)b.spec;
        T2 *sx = S + ((size_t)m * b.ny + j) * b.pk;
        T2 *sy = sx + b.pk;
        for (int kk = t; kk < b.nk; kk += TT) {
            T2 a = z[kk], c = z[(M - kk) % M];
            T2 X, Y;
            X.x = (T)0.5 * (a.x + c.x);
            X.y = (T)0.5 * (a.y - c.y);
            // (a - conj(c)) / (2i)
            T dx_ = (T)0.5 * (a.x - c.x), dy_ = (T)0.5 * (a.y + c.y);
            Y.x = dy_;
            Y.y = -dx_;
            sx[kk] = X;
            if (two) sy[kk] = Y;
        }
    }
}

// ------------------------------------------------------------------ k_ysolve
// One warp per wavenumber column; blockDim = 32*KB.  Tile [ny][KB] (FP64) in
// shared memory; the forward and back substitutions of the Thomas algorithm
// are affine recurrences, solved by a per-lane chunk pass, a warp scan of the
// chunk maps and a second chunk pass.
template <class T, bool CPLX> struct YT;
template <class T> struct YT<T, false> { typedef double v; typedef T g; };
template <class T> struct YT<T, true> { typedef double2 v; typedef typename C2<T>::t g; };

__device__ __forceinline__ double yt_zero(double) { return 0.0; }
__device__ __forceinline__ double2 yt_zero(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double yt_axpy(double c, double d, double x) { return c + d * x; }
__device__ __forceinline__ double2 yt_axpy(double2 c, double d, double2 x) {
    return make_double2(c.x + d * x.x, c.y + d * x.y);
}
__device__ __forceinline__ double yt_scale(double f, double s) { return f * s; }
__device__ __forceinline__ double2 yt_scale(double2 f, double s) { return make_double2(f.x * s, f.y * s); }
__device__ __forceinline__ double yt_up(double v, int o) { return shfl_up_d(v, o); }
__device__ __forceinline__ double2 yt_up(double2 v, int o) { return make_double2(shfl_up_d(v.x, o), shfl_up_d(v.y, o)); }
__device__ __forceinline__ double yt_dn(double v, int o) { return shfl_dn_d(v, o); }
__device__ __forceinline__ double2 yt_dn(double2 v, int o) { return make_double2(shfl_dn_d(v.x, o), shfl_dn_d(v.y, o)); }
__device__ __forceinline__ double yt_load(float v) { return (double)v; }
__device__ __forceinline__ double yt_load(double v) { return v; }
__device__ __forceinline__ double2 yt_load(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 yt_load(double2 v) { return v; }
template <class G> __device__ __forceinline__ G yt_store(double v);
template <> __device__ __forceinline__ double yt_store<double>(double v) { return v; }
template <> __device__ __forceinline__ float yt_store<float>(double v) { return (float)v; }
template <class G> __device__ __forceinline__ G yt_store2(double2 v);
template <> __device__ __forceinline__ double2 yt_store2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 yt_store2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ double yt_re(double v) { return v; }
__device__ __forceinline__ double yt_re(double2 v) { return v.x; }

// forward declaration of the scalar phase
template <class T, int NL> __device__ void scalar_phase(const BasinDev &b, double tdt);

template <class T, bool CPLX, int NL>
__global__ void k_ysolve(const BasinDev *__restrict__ bas, const Work *__restrict__ work,
                         double tdt, int do_scalar) {
    typedef typename YT<T, CPLX>::v V;
    typedef typename YT<T, CPLX>::g Gm;
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    const int KB = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
    const int nkb = (b.nk + KB - 1) / KB;
    const int m = w.block / nkb, k0 = (w.block - m * nkb) * KB;
    const int ny = b.ny;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tile = reinterpret_cast<V *>(smem_raw);   // [ny][KB]
    __shared__ int s_last;

    Gm *S = (Gm *)b.spec + (size_t)m * ny * b.pk;
    // load (coalesced along k)
    for (int idx = threadIdx.x; idx < ny * KB; idx += blockDim.x) {
        int jj = idx / KB, cc = idx - jj * KB;
        int k = k0 + cc;
        tile[idx] = k < b.nk ? yt_load(S[(size_t)jj * b.pk + k]) : yt_zero(V());
    }
    __syncthreads();

    const int k = k0 + c;
    if (k < b.nk) {
        const double a = b.a_tri;
        const int pidx = m * b.nk + k;
        const double *piv = b.piv_tab + b.piv_off[pidx];
        const int plen = b.piv_len[pidx];
        const int S_ = (ny + 31) >> 5;
        const int s = lane * S_, e = min(s + S_, ny);
        // forward elimination: u_j = f_j beta_j - a beta_j u_{j-1}
        V C = yt_zero(V());
        double D = 1.0;
        for (int jj = s; jj < e; ++jj) {
            double bt = piv[min(jj, plen - 1)];
            V f = tile[jj * KB + c];
            C = yt_axpy(yt_scale(f, bt), -a * bt, C);
            D = -a * bt * D;
        }
        for (int o = 1; o < 32; o <<= 1) {
            V Co = yt_up(C, o);
            double Do = shfl_up_d(D, o);
            if (lane >= o) { C = yt_axpy(C, D, Co); D = D * Do; }
        }
        V u = yt_up(C, 1);
        if (lane == 0) u = yt_zero(V());
        for (int jj = s; jj < e; ++jj) {
            double bt = piv[min(jj, plen - 1)];
            V f = tile[jj * KB + c];
            u = yt_axpy(yt_scale(f, bt), -a * bt, u);
            tile[jj * KB + c] = u;
        }
        // back substitution: u_j = u'_j - a beta_j u_{j+1}
        C = yt_zero(V());
        D = 1.0;
        for (int jj = e - 1; jj >= s; --jj) {
            double ej = (jj == ny - 1) ? 0.0 : -a * piv[min(jj, plen - 1)];
            C = yt_axpy(tile[jj * KB + c], ej, C);
            D = ej * D;
        }
        for (int o = 1; o < 32; o <<= 1) {
            V Co = yt_dn(C, o);
            double Do = shfl_dn_d(D, o);
            if (lane + o < 32) { C = yt_axpy(C, D, Co); D = D * Do; }
        }
        u = yt_dn(C, 1);
        if (lane == 31) u = yt_zero(V());
        double colsum = 0.0;
        for (int jj = e - 1; jj >= s; --jj) {
            double ej = (jj == ny - 1) ? 0.0 : -a * piv[min(jj, plen - 1)];
            u = yt_axpy(tile[jj * KB + c], ej, u);
            tile[jj * KB + c] = u;
            colsum += yt_re(u);
        }
        if (!CPLX) {
            colsum = warp_sum(colsum);
            if (lane == 0) b.part_col[pidx] = colsum;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < ny * KB; idx += blockDim.x) {
        int jj = idx / KB, cc = idx - jj * KB;
        int kk = k0 + cc;
        if (kk < b.nk) {
            if constexpr (CPLX) S[(size_t)jj * b.pk + kk] = yt_store2<Gm>(tile[idx]);
            else S[(size_t)jj * b.pk + kk] = yt_store<Gm>(tile[idx]);
        }
    }
    if (!do_scalar) return;
    // last CTA of this basin runs the scalar phase
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int old = atomicAdd(&b.sc->counter, 1u);
        s_last = (old == (unsigned int)(b.k3_blocks - 1));
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x < 32) scalar_phase<T, NL>(b, tdt);
    if (threadIdx.x == 0) b.sc->counter = 0u;
}

// LU solve with the pivots of DGETRF (column-major n x n) -- DGETRS 'N'.
template <int NL>
__device__ void lu_solve_dev(const double *lu, const int *piv, int n, double *x) {
    for (int i = 0; i < n; ++i)
        if (piv[i] != i) { double t = x[i]; x[i] = x[piv[i]]; x[piv[i]] = t; }
    for (int c = 0; c < n; ++c)
        for (int r = c + 1; r < n; ++r) x[r] -= x[c] * lu[r + n * c];
    for (int c = n - 1; c >= 0; --c) {
        x[c] /= lu[c + n * c];
        for (int r = 0; r < c; ++r) x[r] -= x[c] * lu[r + n * c];
    }
}

// solve_Ax_b (util/linalg.F90:57-93): DGETRS then the DGERFS refinement loop.
template <int NL>
__device__ void solve_ax_b_dev(const BasinDev &b, const double *rhs, double *x) {
    const int n = NL - 1;
    const double *A = b.cdhoc;
    for (int i = 0; i < n; ++i) x[i] = rhs[i];
    lu_solve_dev<NL>(b.lu, b.piv, n, x);
    const double eps = 1.1102230246251565e-16;
    const double safe1 = (n + 1) * 2.2250738585072014e-308, safe2 = safe1 / eps;
    double lstres = 3.0;
    int count = 1;
    double r[OQG_NLMAX], wv[OQG_NLMAX];
    for (int it = 0; it < 8; ++it) {
        for (int i = 0; i < n; ++i) r[i] = rhs[i];
        for (int j = 0; j < n; ++j) {
            double t = -x[j];
            for (int i = 0; i < n; ++i) r[i] += t * A[i + n * j];
        }
        for (int i = 0; i < n; ++i) wv[i] = fabs(rhs[i]);
        for (int j = 0; j < n; ++j) {
            double xk = fabs(x[j]);
            for (int i = 0; i < n; ++i) wv[i] += fabs(A[i + n * j]) * xk;
        }
        double s = 0.0;
        for (int i = 0; i < n; ++i) {
            double q = (wv[i] > safe2) ? fabs(r[i]) / wv[i] : (fabs(r[i]) + safe1) / (wv[i] + safe1);
            s = fmax(s, q);
        }
        if (s > eps && 2.0 * s <= lstres && count <= 5) {
            lu_solve_dev<NL>(b.lu, b.piv, n, r);
            for (int i = 0; i < n; ++i) x[i] += r[i];
            lstres = s;
            ++count;
        } else {
            break;
        }
    }
}

// The scalar phase of one step (one warp; lane 0 writes).
template <class T, int NL>
__device__ void scalar_phase(const BasinDev &b, double tdt) {
    const int lane = threadIdx.x & 31;
    DevScalars *sc = b.sc;
    double imode[OQG_NLMAX];
    double S[OQG_NLMAX][OQG_NQ];
    if (!b.cyclic) {
        // area integrals of the modal inhomogeneous solutions, formed from the
        // column sums of the spectral solution (the inverse DST is linear)
        for (int m = 0; m < NL; ++m) {
            double s = 0.0;
            for (int k = lane; k < b.nk; k += 32) s += b.dst_w[k] * b.part_col[m * b.nk + k];
            s = warp_sum(s);
            s = __shfl_sync(0xffffffffu, s, 0);
            imode[m] = s * b.ftnorm * b.dx * b.dy;
        }
    } else {
        const int ntile = b.tiles_x * b.tiles_y;
        for (int k = 0; k < NL; ++k)
            for (int q = 0; q < OQG_NQ; ++q) {
                double s = 0.0;
                for (int t = lane; t < ntile; t += 32) {
                    const int ty0 = (t / b.tiles_x) * VTY;
                    if (ty0 <= 1 || ty0 + VTY > b.nyp - 2)
                        s += b.part_tile[((size_t)t * b.nl + k) * OQG_NQ + q];
                }
                s = warp_sum(s);
                S[k][q] = __shfl_sync(0xffffffffu, s, 0);
            }
    }
    if (lane != 0) return;
    // update_mass_constr (constraint.F90:167-179)
    for (int l = 0; l < NL - 1; ++l) {
        double ait = sc->dpi[l];
        double exn = (l == 0) ? sc->ent_xn : 0.0;
        sc->dpi[l] = sc->dpip[l] - tdt * b.gp[l] * exn;
        sc->dpip[l] = ait;
    }
    if (!b.cyclic) {
        // box_homog (homog.F90:331-366)
        double ik[OQG_NLMAX], rhs[OQG_NLMAX], al[OQG_NLMAX];
        for (int k = 0; k < NL; ++k) {
            double s = 0.0;
            for (int m = 0; m < NL; ++m) s += b.ctm2l[m + NL * k] * imode[m];
            ik[k] = s;
        }
        for (int l = 0; l < NL - 1; ++l) rhs[l] = sc->dpi[l] - (ik[l + 1] - ik[l]);
        solve_ax_b_dev<NL>(b, rhs, al);
        for (int l = 0; l < NL - 1; ++l) sc->alpha[l] = al[l];
    } else {
        // strip integrals (vorticity.F90:84-101, numerics.F90:374-386)
        double ajis[OQG_NLMAX], ajin[OQG_NLMAX], ap3s[OQG_NLMAX], ap3n[OQG_NLMAX];
        double ap5s[OQG_NLMAX], ap5n[OQG_NLMAX];
        const double dx = b.dx, dy = b.dy;
        for (int k = 0; k < NL; ++k) {
            double a5s = (S[k][0] * dx) / (2.0 * dx), a9s = (S[k][1] * dx) / (2.0 * dx);
            double a5n = (S[k][2] * dx) / (2.0 * dx), a9n = (S[k][3] * dx) / (2.0 * dx);
            ajis[k] = (a5s + 2.0 * a9s) / 6.0;
            ajin[k] = -(a5n + 2.0 * a9n) / 6.0;
            ap3s[k] = b.ah2[k] * (S[k][4] * dx) / dy;
            ap3n[k] = b.ah2[k] * (S[k][5] * dx) / dy;
            ap5s[k] = b.ah4[k] * (S[k][6] * dx) / dy;
            ap5n[k] = b.ah4[k] * (S[k][7] * dx) / dy;
        }
        double bdsums = (S[b.kt][8] * dx) / dy, bdsumn = (S[b.kt][9] * dx) / dy;
        double dfac = b.fnot * b.delek / (2.0 * fabs(b.fnot));
        double bdrins = dfac * bdsums, bdrinn = dfac * bdsumn;
        // step_constraints (constraint.F90:182-215)
        double rhss[OQG_NLMAX], rhsn[OQG_NLMAX];
        for (int k = 0; k < NL; ++k) {
            rhss[k] = -0.5 * dy * b.fnot * sc->int_Be_s[k];
            rhsn[k] = -0.5 * dy * b.fnot * sc->int_Be_n[k];
        }
        rhss[0] = rhss[0] + b.tau_sign * (b.fnot / b.h[0]) * sc->txis;
        rhsn[0] = rhsn[0] - b.tau_sign * (b.fnot / b.h[0]) * sc->txin;
        rhss[NL - 1] = rhss[NL - 1] + (b.fnot / b.h[NL - 1]) * bdrins;
        rhsn[NL - 1] = rhsn[NL - 1] - (b.fnot / b.h[NL - 1]) * bdrinn;
        for (int k = 0; k < NL; ++k) {
            rhss[k] = rhss[k] + ajis[k] - ap3s[k] + ap5s[k];
            rhsn[k] = rhsn[k] + ajin[k] + ap3n[k] - ap5n[k];
        }
        for (int k = 0; k < NL; ++k) {
            double csn = sc->csp[k] + tdt * rhss[k];
            double cnn = sc->cnp[k] + tdt * rhsn[k];
            sc->csp[k] = sc->cs[k];
            sc->cnp[k] = sc->cn[k];
            sc->cs[k] = csn;
            sc->cn[k] = cnn;
        }
        // cyclic_homog (homog.F90:280-329).  The x-integral of row j of the
        // modal solution is dx times its zero wavenumber (before the 1/N of the
        // inverse transform, which the N-term row sum cancels).
        typedef typename C2<T>::t T2;
        const T2 *Sp = (const T2 *)b.spec;
        double clhss[OQG_NLMAX], clhsn[OQG_NLMAX];
        for (int m = 0; m < NL; ++m) {
            double ss = 0.0, sn = 0.0;
            for (int k = 0; k < NL; ++k) {
                ss += b.ctl2m[k + NL * m] * sc->cs[k];
                sn += b.ctl2m[k + NL * m] * sc->cn[k];
            }
            double u0s = (double)Sp[((size_t)m * b.ny) * b.pk].x;
            double u0n = (double)Sp[((size_t)m * b.ny + (b.ny - 1)) * b.pk].x;
            clhss[m] = ss + (u0s * dx) / dy;
            clhsn[m] = sn + (u0n * dx) / dy;
        }
        sc->c_bt = clhss[0] * b.hbsi;
        for (int m = 1; m < NL; ++m) {
            sc->c_bc1[m] = b.hc2n[m] * clhss[m] - b.hc2s[m] * clhsn[m];
            sc->c_bc2[m] = b.hc1s[m] * clhsn[m] - b.hc1n[m] * clhss[m];
        }
    }
    // suppress_comp_mode schedule (openqg.F90:485-487) and its scalar part
    // (driver.F90:183-188)
    const int supp = (b.suppress_period > 0 && (sc->nt % b.suppress_period) == 0) ? 1 : 0;
    if (supp) {
        for (int l = 0; l < NL - 1; ++l) sc->dpi[l] = 0.5 * (sc->dpi[l] + sc->dpip[l]);
        if (b.cyclic)
            for (int k = 0; k < NL; ++k) {
                sc->cs[k] = 0.5 * (sc->cs[k] + sc->csp[k]);
                sc->cn[k] = 0.5 * (sc->cn[k] + sc->cnp[k]);
            }
    }
    sc->suppress_flag = supp;
    sc->nt += 1;
}

// ------------------------------------------------------------------ k_xinv
// Rows of one CTA: interior rows [jlo, jhi) plus wall row 0 (first CTA) and
// wall row nyp-1 (last CTA).
__device__ __forceinline__ void xinv_rows(const BasinDev &b, int rb, int &jlo, int &jhi,
                                          int &jfirst, int &nra) {
    jlo = 1 + rb * b.k4_rows;
    jhi = min(jlo + b.k4_rows, b.nyp - 1);
    jfirst = (rb == 0) ? 0 : jlo;
    int jlast = (jhi == b.nyp - 1) ? b.nyp - 1 : jhi - 1;
    nra = jlast - jfirst + 1;
}

// out != null: solve-only mode, writes the modal inhomogeneous solutions
// (FP64, [nl][nyp][px]) and nothing else.
template <class T, int E, int NL>
__global__ void k_xinv(const BasinDev *__restrict__ bas, const Work *__restrict__ work, int par,
                       double *out) {
    typedef typename C2<T>::t T2;
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    const int M = b.M, TT = (M + E - 1) / E, G = blockDim.x / TT;
    const int g = threadIdx.x / TT, t = threadIdx.x - g * TT;
    int jlo, jhi, jfirst, nra;
    xinv_rows(b, w.block, jlo, jhi, jfirst, nra);
    const int nr = jhi - jlo;                    // interior rows
    const int nxp = b.nxp, n = b.nxin;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2 *zs = reinterpret_cast<T2 *>(smem_raw);
    T *inh = reinterpret_cast<T *>(zs + (size_t)G * M);   // [NL][nra][nxp]
    const T2 *tw = (const T2 *)b.tw;
    const T ftn = (T)b.ftnorm;

    // zero the wall rows / columns of the modal fields
    for (int idx = threadIdx.x; idx < NL * nra * nxp; idx += blockDim.x) inh[idx] = (T)0;
    __syncthreads();

    const int npr = (nr + 1) >> 1;               // row pairs per mode
    const int npairs = NL * npr;
    for (int base = 0; base < npairs; base += G) {
        const int pair = base + g;
        const bool live = g < G && pair < npairs;
        const int m = live ? pair / npr : 0;
        const int r0 = live ? 2 * (pair - m * npr) : 0;     // interior row offset
        const bool two = live && r0 + 1 < nr;
        T2 *z = zs + (size_t)(g < G ? g : 0) * M;
        const int sj = jlo + r0 - 1;                        // spectral row
        if (!b.cyclic) {
            const T *S = (const T *)b.spec;
            const T *x = S + ((size_t)m * b.ny + sj) * b.pk;
            const T *y = x + b.pk;
            if (live)
                for (int jj = t; jj < M; jj += TT) {
                    T2 v;
                    if (jj == 0 || jj == n + 1) { v.x = (T)0; v.y = (T)0; }
                    else if (jj <= n) { v.x = ftn * x[jj - 1]; v.y = two ? ftn * y[jj - 1] : (T)0; }
                    else { int s2 = M - jj; v.x = -(ftn * x[s2 - 1]); v.y = two ? -(ftn * y[s2 - 1]) : (T)0; }
                    z[jj] = v;
                }
        } else {
            const T2 *S = (const T2 *)b.spec;
            const T2 *x = S + ((size_t)m * b.ny + sj) * b.pk;
            const T2 *y = x + b.pk;
            if (live)
                for (int kk = t; kk < M; kk += TT) {
                    T2 X, Y;
                    const bool lo = kk <= M / 2;
                    const int ks = lo ? kk : M - kk;
                    X = x[ks];
                    if (two) Y = y[ks]; else { Y.x = (T)0; Y.y = (T)0; }
                    if (!lo) { X.y = -X.y; Y.y = -Y.y; }
                    if (kk == 0 || 2 * kk == M) { X.y = (T)0; Y.y = (T)0; }
                    // conj(ftnorm (X + iY))
                    T2 v;
                    v.x = ftn * X.x - ftn * Y.y;
                    v.y = -(ftn * X.y + ftn * Y.x);
                    z[kk] = v;
                }
        }
        __syncthreads();
        fft_smem<T, E>(z, M, b.rad, b.nrad, tw, live ? t : TT, TT);
        if (live) {
            const int lr = (jlo + r0) - jfirst;
            T *ox = inh + ((size_t)m * nra + lr) * nxp;
            T *oy = ox + nxp;
            if (!b.cyclic) {
                for (int kk = t; kk < n; kk += TT) {
                    T2 v = z[kk + 1];
                    ox[kk + 1] = -v.y;
                    if (two) oy[kk + 1] = v.x;
                }
            } else {
                for (int i = t; i < M; i += TT) {
                    T2 v = z[i];
                    ox[i] = v.x;
                    if (two) oy[i] = -v.y;
                }
                if (t == 0) {
                    ox[M] = z[0].x;
                    if (two) oy[M] = -z[0].y;
                }
            }
        }
        __syncthreads();
    }

    if (out) {
        for (int idx = threadIdx.x; idx < NL * nra * nxp; idx += blockDim.x) {
            int m = idx / (nra * nxp), rem = idx - m * nra * nxp;
            int lr = rem / nxp, i = rem - lr * nxp;
            out[((size_t)m * b.nyp + jfirst + lr) * b.px + i] = (double)inh[idx];
        }
        return;
    }

    // homogeneous correction + modes_to_layers, in place (modes -> layers)
    const DevScalars *sc = b.sc;
    const int supp = sc->suppress_flag;
    const T *Pold = (const T *)b.F[par];
    T *Pnew = (T *)b.F[1 - par];
    for (int idx = threadIdx.x; idx < nra * nxp; idx += blockDim.x) {
        const int lr = idx / nxp, i = idx - lr * nxp;
        const int j = jfirst + lr;
        double pm_[NL];
#pragma unroll
        for (int m = 0; m < NL; ++m) pm_[m] = (double)inh[((size_t)m * nra + lr) * nxp + i];
        if (!b.cyclic) {
            const T *H = (const T *)b.hsb;
#pragma unroll
            for (int m = 1; m < NL; ++m)
                pm_[m] = pm_[m] + sc->alpha[m - 1] * (double)H[((size_t)(m - 1) * b.nyp + j) * b.px + i];
        } else {
            pm_[0] = pm_[0] + sc->c_bt * b.hbt[j];
#pragma unroll
            for (int m = 1; m < NL; ++m)
                pm_[m] = pm_[m] + (sc->c_bc1[m] * b.hbc1[m * b.nyp + j] + sc->c_bc2[m] * b.hbc2[m * b.nyp + j]);
        }
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            double s = 0.0;
#pragma unroll
            for (int m = 0; m < NL; ++m) s += pm_[m] * b.ctm2l[m + NL * k];
            T pn = (T)s;
            inh[((size_t)k * nra + lr) * nxp + i] = pn;
            const size_t o3 = ((size_t)k * b.nyp + j) * b.px + i;
            Pnew[o3] = supp ? (T)((T)0.5 * (pn + Pold[o3])) : pn;
        }
    }
    __syncthreads();

    // ocqbdy (vorsubs.F90:58-114) on the walls of these rows, then the
    // suppress_comp_mode average of q (driver.F90:180)
    T *Qc = (T *)b.F[3 - par];        // q after this step (qm buffer of K1)
    const T *Qm = (const T *)b.F[2 + par];
    const T fac = (T)b.qb_fac;
    for (int idx = threadIdx.x; idx < nra * nxp; idx += blockDim.x) {
        const int lr = idx / nxp, i = idx - lr * nxp;
        const int j = jfirst + lr;
        const bool zon = (j == 0 || j == b.nyp - 1);
        const bool mer = !b.cyclic && (i == 0 || i == nxp - 1);
        if (!zon && !mer) {
            if (supp)
                for (int k = 0; k < NL; ++k) {
                    const size_t o3 = ((size_t)k * b.nyp + j) * b.px + i;
                    Qc[o3] = (T)0.5 * (Qc[o3] + Qm[o3]);
                }
            continue;
        }
        const int cnt = (zon ? 1 : 0) + (mer ? 1 : 0);
#define PN(kk, rr, ii) inh[((size_t)(kk) * nra + (rr)) * nxp + (ii)]
        T pv[NL];
#pragma unroll
        for (int k = 0; k < NL; ++k) pv[k] = PN(k, lr, i);
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            T qv;
            if (mer) {
                qv = (i == 0) ? fac * (PN(k, lr, 1) - pv[k]) : fac * (PN(k, lr, nxp - 2) - pv[k]);
            } else {
                qv = (j == 0) ? fac * (PN(k, lr + 1, i) - pv[k]) : fac * (PN(k, lr - 1, i) - pv[k]);
            }
            double mv = 0.0;
#pragma unroll
            for (int l = 0; l < NL; ++l) mv += b.amat[k + NL * l] * (double)pv[l];
            const T fmv = (T)(b.fnot * mv);
            const T by = (T)(b.beta * b.yprel[j]);
            for (int c = 0; c < cnt; ++c) qv = qv - fmv;
            for (int c = 0; c < cnt; ++c) qv = qv + by;
            if (k == b.kt && b.topo_active) {
                const T dd = (T)b.ddyn[(size_t)j * b.px + i];
                for (int c = 0; c < cnt; ++c) qv = qv + dd;
            }
            const size_t o3 = ((size_t)k * b.nyp + j) * b.px + i;
            Qc[o3] = supp ? (T)((T)0.5 * (qv + Qm[o3])) : qv;
        }
#undef PN
    }
}

// ------------------------------------------------------------------ init / aux
// Laplacian with the wall condition on a global FP64 field (one layer),
// numerics.F90:410-468; the channel's column nxp-1 repeats column 0.
__device__ __forceinline__ double lap_bc_g(const double *f, const BasinDev &b, int i, int j, double alpha_fac) {
    const int px = b.px, nxp = b.nxp, nyp = b.nyp;
    if (b.cyclic && i == nxp - 1) i = 0;
    const double v = f[(size_t)j * px + i];
    double xp, yp;
    const bool wall_x = !b.cyclic && (i == 0 || i == nxp - 1);
    if (j == 0 || j == nyp - 1) xp = 0.0;
    else if (!b.cyclic && i == 0) xp = b.fx * alpha_fac * (f[(size_t)j * px + 1] - v);
    else if (!b.cyclic && i == nxp - 1) xp = -(b.fx * alpha_fac * (v - f[(size_t)j * px + i - 1]));
    else {
        int il = (i == 0) ? nxp - 2 : i - 1;
        xp = b.fx * (f[(size_t)j * px + il] + f[(size_t)j * px + i + 1] - 2.0 * v);
    }
    if (wall_x) yp = 0.0;
    else if (j == 0) yp = b.fy * alpha_fac * (f[(size_t)px + i] - v);
    else if (j == nyp - 1) yp = -(b.fy * alpha_fac * (v - f[(size_t)(j - 1) * px + i]));
    else yp = b.fy * (f[(size_t)(j - 1) * px + i] + f[(size_t)(j + 1) * px + i] - 2.0 * v);
    return xp + yp;
}

// qcomp (vorsubs.F90:27-56): q = del2(p)/f0 + ddyn[kt] + beta y - f0 A p.
// p: FP64 staging [nl][nyp][px]; q: field of type T.
template <class T, int NL>
__global__ void k_qcomp(const BasinDev *__restrict__ bas, int member, const double *p, T *q) {
    const BasinDev &b = bas[member];
    const size_t n2 = (size_t)b.nyp * b.px;
    const double afac = b.fx_bc / b.fx;   // alpha/(alpha/2+1)
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)b.nyp * b.nxp;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / b.nxp), i = (int)(idx - (size_t)j * b.nxp);
        const size_t o2 = (size_t)j * b.px + i;
        double pv[NL];
#pragma unroll
        for (int l = 0; l < NL; ++l) pv[l] = p[l * n2 + o2];
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            double v = lap_bc_g(p + k * n2, b, i, j, afac) / b.fnot;
            if (k == b.kt && b.topo_active) v += b.ddyn[o2];
            v += b.beta * b.yprel[j];
            double mv = 0.0;
#pragma unroll
            for (int l = 0; l < NL; ++l) mv += b.amat[k + NL * l] * pv[l];
            v -= b.fnot * mv;
            q[k * n2 + o2] = (T)v;
        }
    }
}

template <class T>
__global__ void k_cvt_in(const double *src, T *dst, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (T)src[i];
}
template <class T>
__global__ void k_cvt_out(const T *src, double *dst, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

// Trapezoid weight of int_P_dA (numerics.F90:188-204) at (i, j).
__device__ __forceinline__ double trap_w(const BasinDev &b, int i, int j) {
    double w = 1.0;
    if (i == 0 || i == b.nxp - 1) w *= 0.5;
    if (j == 0 || j == b.nyp - 1) w *= 0.5;
    return w;
}
// int_P_dx (numerics.F90:206-212) weight.
__device__ __forceinline__ double trap_x(const BasinDev &b, int i) {
    return (i == 0 || i == b.nxp - 1) ? 0.5 : 1.0;
}

template <class T>
__device__ double area_integral(const BasinDev &b, const T *f, double *red) {
    double s = 0.0;
    for (int idx = threadIdx.x; idx < b.nyp * b.nxp; idx += blockDim.x) {
        int j = idx / b.nxp, i = idx - j * b.nxp;
        s += trap_w(b, i, j) * (double)f[(size_t)j * b.px + i];
    }
    return block_sum(s, red) * b.dx * b.dy;
}
// int_P_dx of row ja of f minus row jb (jb < 0: no subtraction)
template <class T>
__device__ double row_integral(const BasinDev &b, const T *f, int ja, int jb, double *red) {
    double s = 0.0;
    for (int i = threadIdx.x; i < b.nxp; i += blockDim.x) {
        double v = (double)f[(size_t)ja * b.px + i];
        if (jb >= 0) v -= (double)f[(size_t)jb * b.px + i];
        s += trap_x(b, i) * v;
    }
    return block_sum(s, red) * b.dx;
}

// init_mass_constr (constraint.F90:145-165) and, for a channel,
// init_constraint (constraint.F90:80-143).  One CTA.
template <class T, int NL>
__global__ void k_init_constraints(const BasinDev *__restrict__ bas, int member, int par) {
    const BasinDev &b = bas[member];
    __shared__ double red[32];
    __shared__ double ip[OQG_NLMAX], ipm[OQG_NLMAX], pins[OQG_NLMAX], pinn[OQG_NLMAX],
        pinsp[OQG_NLMAX], pinnp[OQG_NLMAX], cs[OQG_NLMAX], cn[OQG_NLMAX], csp[OQG_NLMAX],
        cnp[OQG_NLMAX];
    const T *P = (const T *)b.F[par];
    const T *PM = (const T *)b.F[1 - par];
    const size_t n2 = (size_t)b.nyp * b.px;
    const int ny1 = b.nyp - 1;
    for (int k = 0; k < NL; ++k) {
        double a = area_integral(b, P + k * n2, red);
        double am = area_integral(b, PM + k * n2, red);
        if (threadIdx.x == 0) { ip[k] = a; ipm[k] = am; }
        if (b.cyclic) {
            double v0 = row_integral(b, PM + k * n2, 0, -1, red);
            double v1 = row_integral(b, P + k * n2, 0, -1, red);
            double v2 = row_integral(b, PM + k * n2, ny1, -1, red);
            double v3 = row_integral(b, P + k * n2, ny1, -1, red);
            double v4 = row_integral(b, PM + k * n2, 1, 0, red) / b.dy;
            double v5 = row_integral(b, PM + k * n2, ny1, ny1 - 1, red) / b.dy;
            double v6 = row_integral(b, P + k * n2, 1, 0, red) / b.dy;
            double v7 = row_integral(b, P + k * n2, ny1, ny1 - 1, red) / b.dy;
            if (threadIdx.x == 0) {
                pinsp[k] = v0; pins[k] = v1; pinnp[k] = v2; pinn[k] = v3;
                csp[k] = v4; cnp[k] = v5; cs[k] = v6; cn[k] = v7;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    DevScalars *sc = b.sc;
    for (int k = 0; k < NL - 1; ++k) {
        sc->dpip[k] = b.dz_sign * (ipm[k] - ipm[k + 1]);
        sc->dpi[k] = b.dz_sign * (ip[k] - ip[k + 1]);
    }
    if (b.cyclic) {
        const double f2 = 0.5 * b.dy * b.fnot * b.fnot;
        for (int k = 0; k < NL; ++k) {
            double apsp = 0, apnp = 0, aps = 0, apn = 0;
            for (int l = 0; l < NL; ++l) {
                double a = b.amat[k + NL * l];
                apsp += a * pinsp[l]; apnp += a * pinnp[l]; aps += a * pins[l]; apn += a * pinn[l];
            }
            sc->csp[k] = -csp[k] + f2 * apsp;
            sc->cnp[k] = cnp[k] + f2 * apnp;
            sc->cs[k] = -cs[k] + f2 * aps;
            sc->cn[k] = cn[k] + f2 * apn;
        }
    }
}

// Forcing integrals that depend only on ent: ent_xn = int_P_dA(ent(:,:,1))
// (pressure.F90:52-54) and the channel strip integrals int_Be_s/n
// (vorticity.F90:122-128).  One CTA.
template <class T>
__global__ void k_forcing_integrals(const BasinDev *__restrict__ bas, int member) {
    const BasinDev &b = bas[member];
    __shared__ double red[32];
    DevScalars *sc = b.sc;
    const T *E = (const T *)b.ent;
    const size_t n2 = (size_t)b.nyp * b.px;
    double exn = 0.0, s1 = 0.0, s2 = 0.0, n1 = 0.0, n2v = 0.0;
    if (E) {
        exn = area_integral(b, E, red);
        if (b.cyclic) {
            s1 = row_integral(b, E, 0, -1, red);
            n1 = row_integral(b, E, b.nyp - 1, -1, red);
            if (b.nl - 1 >= 2) {
                s2 = row_integral(b, E + n2, 0, -1, red);
                n2v = row_integral(b, E + n2, b.nyp - 1, -1, red);
            }
        }
    }
    if (threadIdx.x != 0) return;
    sc->ent_xn = exn;
    for (int k = 0; k < OQG_NLMAX; ++k) { sc->int_Be_s[k] = 0.0; sc->int_Be_n[k] = 0.0; }
    const double f1 = b.fnot / b.h[0], f2 = b.fnot / b.h[1];
    sc->int_Be_s[0] = b.dz_sign * f1 * s1;
    sc->int_Be_s[1] = b.dz_sign * f1 * s2;
    sc->int_Be_n[0] = -b.dz_sign * f2 * n1;
    sc->int_Be_n[1] = -b.dz_sign * f2 * n2v;
}

// Solve-only input: the same (nxp, nyp) right-hand side for every mode.
template <class T>
__global__ void k_rhs_from_field(const BasinDev *__restrict__ bas, int member, const double *f, T *rhs) {
    const BasinDev &b = bas[member];
    const int ioff = b.cyclic ? 0 : 1;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < b.nl * b.ny * b.nxin;
         idx += gridDim.x * blockDim.x) {
        int m = idx / (b.ny * b.nxin), rem = idx - m * b.ny * b.nxin;
        int jj = rem / b.nxin, xi = rem - jj * b.nxin;
        rhs[((size_t)m * b.ny + jj) * b.pr + xi] = (T)f[(size_t)(jj + 1) * b.px + xi + ioff];
    }
}

// suppress_comp_mode now (driver.F90:174-189).
template <class T>
__global__ void k_suppress(const BasinDev *__restrict__ bas, int member, int par) {
    const BasinDev &b = bas[member];
    T *P = (T *)b.F[par];
    const T *PM = (const T *)b.F[1 - par];
    T *Q = (T *)b.F[2 + par];
    const T *QM = (const T *)b.F[3 - par];
    const size_t n = (size_t)b.nl * b.nyp * b.px;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        Q[i] = (T)0.5 * (Q[i] + QM[i]);
        P[i] = (T)0.5 * (P[i] + PM[i]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        DevScalars *sc = b.sc;
        for (int l = 0; l < b.nl - 1; ++l) sc->dpi[l] = 0.5 * (sc->dpi[l] + sc->dpip[l]);
        if (b.cyclic)
            for (int k = 0; k < b.nl; ++k) {
                sc->cs[k] = 0.5 * (sc->cs[k] + sc->csp[k]);
                sc->cn[k] = 0.5 * (sc->cn[k] + sc->cnp[k]);
            }
    }
}

// Count of non-finite values of p and q (the role of valids).
template <class T>
__global__ void k_check_finite(const BasinDev *__restrict__ bas, int member, int par,
                               unsigned long long *bad) {
    const BasinDev &b = bas[member];
    const T *P = (const T *)b.F[par];
    const T *Q = (const T *)b.F[2 + par];
    unsigned long long c = 0;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)b.nl * b.nyp * b.nxp;
         idx += (size_t)gridDim.x * blockDim.x) {
        size_t k = idx / ((size_t)b.nyp * b.nxp), rem = idx - k * b.nyp * b.nxp;
        size_t j = rem / b.nxp, i = rem - j * b.nxp;
        size_t o = (k * b.nyp + j) * b.px + i;
        if (!isfinite((double)P[o])) ++c;
        if (!isfinite((double)Q[o])) ++c;
    }
    if (c) atomicAdd(bad, c);
}

// qg_diagno energetics and extrema (qg_monitor.F90:289-376): one CTA per layer.
// out[k*4 + 0..3] = ekei, sfmin, sfmax, circ.
template <class T>
__global__ void k_diag(const BasinDev *__restrict__ bas, int member, int par, double rho, double *out) {
    const BasinDev &b = bas[member];
    const int k = blockIdx.x;
    __shared__ double red[32];
    const T *P = (const T *)b.F[par] + (size_t)k * b.nyp * b.px;
    double uke = 0.0, vke = 0.0, pmin = 1e308, pmax = -1e308;
    const int nxp = b.nxp, nyp = b.nyp, px = b.px;
    // (alpha/2 + 1) of dPdx_2bc/dPdy_2bc, recovered from the mixed-BC factor
    const double ah = b.bc_half1;
    for (int idx = threadIdx.x; idx < nxp * nyp; idx += blockDim.x) {
        int j = idx / nxp, i = idx - j * nxp;
        double pv = (double)P[(size_t)j * px + i];
        pmin = fmin(pmin, pv);
        pmax = fmax(pmax, pv);
        // dPdx_2bc / dPdy_2bc (numerics.F90:470-513)
        double dpx, dpy;
        if (j == 0 || j == nyp - 1) dpx = 0.0;
        else if (b.cyclic && (i == 0 || i == nxp - 1))
            dpx = ((double)P[(size_t)j * px + 1] - (double)P[(size_t)j * px + nxp - 2]) / (2.0 * b.dx);
        else if (i == 0) dpx = ((double)P[(size_t)j * px + 1] - pv) / (b.dx * ah);
        else if (i == nxp - 1) dpx = (pv - (double)P[(size_t)j * px + i - 1]) / (b.dx * ah);
        else dpx = ((double)P[(size_t)j * px + i + 1] - (double)P[(size_t)j * px + i - 1]) / (2.0 * b.dx);
        if (!b.cyclic && (i == 0 || i == nxp - 1)) dpy = 0.0;
        else if (j == 0) dpy = ((double)P[(size_t)px + i] - pv) / (b.dy * ah);
        else if (j == nyp - 1) dpy = (pv - (double)P[(size_t)(j - 1) * px + i]) / (b.dy * ah);
        else dpy = ((double)P[(size_t)(j + 1) * px + i] - (double)P[(size_t)(j - 1) * px + i]) / (2.0 * b.dy);
        double u = -dpy / b.fnot, v = dpx / b.fnot;
        double w = trap_w(b, i, j);
        uke += w * (u * u);
        vke += w * (v * v);
    }
    uke = block_sum(uke, red) * b.dx * b.dy;
    vke = block_sum(vke, red) * b.dx * b.dy;
    // min / max
    __shared__ double mn[32], mx[32];
    for (int o = 16; o > 0; o >>= 1) {
        pmin = fmin(pmin, __shfl_down_sync(0xffffffffu, pmin, o));
        pmax = fmax(pmax, __shfl_down_sync(0xffffffffu, pmax, o));
    }
    if ((threadIdx.x & 31) == 0) { mn[threadIdx.x >> 5] = pmin; mx[threadIdx.x >> 5] = pmax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int wv = 1; wv < (int)(blockDim.x >> 5); ++wv) { pmin = fmin(pmin, mn[wv]); pmax = fmax(pmax, mx[wv]); }
        const double p00 = (double)P[0], p0n = (double)P[(size_t)(nyp - 1) * px];
        const double poref = b.fnot > 0 ? p00 : p0n;
        const double e1 = fmin(pmin / b.fnot, pmax / b.fnot), e2 = fmax(pmin / b.fnot, pmax / b.fnot);
        out[k * 4 + 0] = 0.5 * rho * b.h[k] * (uke + vke);
        out[k * 4 + 1] = 1.0e-6 * (b.h[k] * (e1 - poref / b.fnot));
        out[k * 4 + 2] = 1.0e-6 * (b.h[k] * (e2 - poref / b.fnot));
        out[k * 4 + 3] = 1.0e-6 * ((p00 - p0n) / b.fnot);
    }
}

}  // namespace oqg
