// oqg_noalloc.cuh -- qg_diagno diagnostics whose scratch is a fixed device
// array compiled into the library, for oqg_diag_noalloc.
//
// The handle's own diagnostics (k_diag) write into a buffer that oqg_create
// allocated.  This variant keeps its per-row partial sums, its completion
// ticket and its results in g_noalloc_scratch instead (defined in
// oqg_capi.cu), a file-scope device array of OQG_NOALLOC_DOUBLES doubles
// (256 KiB) that the CUDA runtime places when it loads the library's device
// code, so a call needs no allocation.
//
// Layout of the array (in doubles):
//   [0]                      completion ticket (64-bit counter; 0 at launch)
//   [8, 8 + 4 nl)            results: ekei, sfmin, sfmax, circ per layer
//   [OQG_NOALLOC_PART, ...)  partials: 4 per (layer, row), 4 nl nyp in all
// A basin fits when OQG_NOALLOC_PART + 4 nl nyp <= OQG_NOALLOC_DOUBLES.
#pragma once

#include "oqg_kernels.cuh"

namespace oqg {

#define OQG_NOALLOC_DOUBLES 32768                            // 256 KiB
#define OQG_NOALLOC_OUT 8                                    // first result slot
#define OQG_NOALLOC_PART (OQG_NOALLOC_OUT + 4 * OQG_NLMAX)   // first partial slot

__host__ __device__ __forceinline__ long long noalloc_doubles(int nl, int nyp) {
    return OQG_NOALLOC_PART + 4LL * nl * nyp;
}

// One CTA per (row j = blockIdx.x, layer k = blockIdx.y) forms the row's
// kinetic-energy sums (trapezoid weights) and stream-function extrema; the
// last CTA to finish (the ticket) reduces the rows of every layer in a fixed
// order and writes the results as k_diag does (qg_monitor.F90:289-376).
template <class T>
__global__ void __launch_bounds__(128)
k_diag_rows(const BasinDev *__restrict__ bas, int member, int par, double rho, double *scr) {
    const BasinDev &b = bas[member];
    const int j = blockIdx.x, k = blockIdx.y;
    const int nxp = b.nxp, nyp = b.nyp, px = b.px, nl = b.nl;
    __shared__ double red[32];
    __shared__ double mn[32], mx[32];
    __shared__ int last;
    const T *P = (const T *)b.F[par] + (size_t)k * nyp * px;
    const double ah = b.bc_half1;
    double uke = 0.0, vke = 0.0, pmin = 1e308, pmax = -1e308;
    for (int i = threadIdx.x; i < nxp; i += blockDim.x) {
        const double pv = (double)P[(size_t)j * px + i];
        pmin = fmin(pmin, pv);
        pmax = fmax(pmax, pv);
        // dPdx_2bc / dPdy_2bc (numerics.F90:470-513), as in k_diag
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
        const double u = -dpy / b.fnot, v = dpx / b.fnot;
        const double w = trap_w(b, i, j);
        uke += w * (u * u);
        vke += w * (v * v);
    }
    uke = block_sum(uke, red);
    vke = block_sum(vke, red);
    for (int o = 16; o > 0; o >>= 1) {
        pmin = fmin(pmin, __shfl_down_sync(0xffffffffu, pmin, o));
        pmax = fmax(pmax, __shfl_down_sync(0xffffffffu, pmax, o));
    }
    if ((threadIdx.x & 31) == 0) { mn[threadIdx.x >> 5] = pmin; mx[threadIdx.x >> 5] = pmax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int wv = 1; wv < (int)(blockDim.x >> 5); ++wv) { pmin = fmin(pmin, mn[wv]); pmax = fmax(pmax, mx[wv]); }
        double *part = scr + OQG_NOALLOC_PART + ((size_t)k * nyp + j) * 4;
        part[0] = uke;
        part[1] = vke;
        part[2] = pmin;
        part[3] = pmax;
        __threadfence();
        unsigned long long *ticket = reinterpret_cast<unsigned long long *>(scr);
        const unsigned long long n = (unsigned long long)gridDim.x * gridDim.y;
        last = (atomicAdd(ticket, 1ull) == n - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last CTA: per layer, rows summed in a fixed order (thread t takes
    // rows t, t + blockDim, ...; then a fixed tree), so results repeat exactly
    for (int kk = 0; kk < nl; ++kk) {
        const double *pk = scr + OQG_NOALLOC_PART + (size_t)kk * nyp * 4;
        double su = 0.0, sv = 0.0, lo = 1e308, hi = -1e308;
        for (int r = threadIdx.x; r < nyp; r += blockDim.x) {
            su += __ldcg(pk + 4 * r);
            sv += __ldcg(pk + 4 * r + 1);
            lo = fmin(lo, __ldcg(pk + 4 * r + 2));
            hi = fmax(hi, __ldcg(pk + 4 * r + 3));
        }
        su = block_sum(su, red) * b.dx * b.dy;
        sv = block_sum(sv, red) * b.dx * b.dy;
        for (int o = 16; o > 0; o >>= 1) {
            lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, o));
        }
        if ((threadIdx.x & 31) == 0) { mn[threadIdx.x >> 5] = lo; mx[threadIdx.x >> 5] = hi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int wv = 1; wv < (int)(blockDim.x >> 5); ++wv) { lo = fmin(lo, mn[wv]); hi = fmax(hi, mx[wv]); }
            const T *Pk = (const T *)b.F[par] + (size_t)kk * nyp * px;
            const double p00 = (double)Pk[0], p0n = (double)Pk[(size_t)(nyp - 1) * px];
            const double poref = b.fnot > 0 ? p00 : p0n;
            const double e1 = fmin(lo / b.fnot, hi / b.fnot), e2 = fmax(lo / b.fnot, hi / b.fnot);
            double *out = scr + OQG_NOALLOC_OUT + 4 * kk;
            out[0] = 0.5 * rho * b.h[kk] * (su + sv);
            out[1] = 1.0e-6 * (b.h[kk] * (e1 - poref / b.fnot));
            out[2] = 1.0e-6 * (b.h[kk] * (e2 - poref / b.fnot));
            out[3] = 1.0e-6 * ((p00 - p0n) / b.fnot);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *reinterpret_cast<unsigned long long *>(scr) = 0ull;
}

}  // namespace oqg
