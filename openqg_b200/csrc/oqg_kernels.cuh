// oqg_kernels.cuh -- the per-step kernels of the QG core (sm_100a).
//
// One step_qg (qg/core.F90:16-33) is a chain of launches, one per dependent
// phase:
//   k_vort   vort_step (qg/vorticity.F90:14-103) + p_modes_rhs (qg/modes.F90:248-266)
//            2-D tiles staged in shared memory; the layer loop runs inside the
//            CTA so the modal right-hand side is formed in registers.
//   k_xfwd   forward x-transform of solve_inhomog_box / _cyclic
//            (qg/inhomog.F90:170-255): DST-I (box) or r2c FFT (channel).
//   k_ysolve Thomas solve in y per (mode, wavenumber) (inhomog.F90:187-199),
//            one to four warps per column as a warp-parallel affine scan.
//   k_xinv   inverse x-transform + homogeneous correction + modes_to_layers
//            (modes.F90:268-284) + ocqbdy (vorsubs.F90:58-114) +
//            suppress_comp_mode (driver.F90:174-189).  One warp of each CTA
//            runs the scalar phase meanwhile: update_mass_constr
//            (constraint.F90:167-179), box_homog's 2x2 solve (homog.F90:331-366)
//            or step_constraints + cyclic_homog (constraint.F90:182-215,
//            homog.F90:280-329), and the suppress_comp_mode schedule
//            (openqg.F90:485-487).
//   or, as two launches (the default for boxes, measured for channels):
//   k_xinv_rows  the inverse x-transforms alone, shaped like k_xfwd, with one
//            extra CTA per basin for the scalar phase;
//   k_xinv_asm   the homogeneous correction, modes_to_layers, ocqbdy and the
//            suppression averages, one thread per point.
// Every launch takes a work list, so one launch serves one basin or an
// ensemble of basins of uneven size.
#pragma once

#include "oqg_dev.cuh"
#include "oqg_fft.cuh"
#include "oqg_tma.cuh"

#include <type_traits>

namespace oqg {

// ------------------------------------------------------------------ helpers
template <class T> __device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// Programmatic dependent launch: the next kernel of the step may be scheduled
// now; and wait until the previous kernel's results are visible.  Without the
// launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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

// ------------------------------------------------------------------ compensated sums
// The mass-constraint and area integrals (int_P_dA, numerics.F90:165-204;
// box_homog's modal integrals, homog.F90:331-366) are summed with a running
// compensation: every addition is Knuth's error-free TwoSum, s + e = a + b
// exactly, and the rounding errors are summed beside the sum (Neumaier's
// scheme), so the result is correct to about one rounding of the total
// whatever the cancellation among the terms.  Nothing here is contracted
// into FMAs (no products).
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    s = a + b;
    const double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
struct CSum {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        double t, e;
        two_sum(s, x, t, e);
        s = t;
        c += e;
    }
    // another compensated sum (its sum and its compensation)
    __device__ __forceinline__ void merge(double os, double oc) {
        add(os);
        c += oc;
    }
    // the exact product w * x of a weight and a term, added (the product's
    // rounding error comes from an FMA)
    __device__ __forceinline__ void add_prod(double w, double x) {
        const double p = w * x;
        add(p);
        c += fma(w, x, -p);
    }
    __device__ __forceinline__ double value() const { return s + c; }
};
// Warp reduction of compensated sums; the total is in lane 0 (all lanes
// with full=true).
__device__ __forceinline__ CSum csum_warp(CSum v, bool full = false) {
    for (int o = 16; o > 0; o >>= 1) {
        const double os = full ? __shfl_xor_sync(0xffffffffu, v.s, o) : __shfl_down_sync(0xffffffffu, v.s, o);
        const double oc = full ? __shfl_xor_sync(0xffffffffu, v.c, o) : __shfl_down_sync(0xffffffffu, v.c, o);
        v.merge(os, oc);
    }
    return v;
}
// CTA reduction of compensated sums: the total as a compensated pair, valid
// in every thread.  red: >= 64 doubles of shared memory.
__device__ __forceinline__ CSum csum_block_pair(CSum v, double *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = csum_warp(v);
    __syncthreads();
    if (lane == 0) { red[wid] = v.s; red[32 + wid] = v.c; }
    __syncthreads();
    if (wid == 0) {
        CSum t;
        if (lane < nw) { t.s = red[lane]; t.c = red[32 + lane]; }
        t = csum_warp(t);
        if (lane == 0) { red[0] = t.s; red[1] = t.c; }
    }
    __syncthreads();
    CSum r;
    r.s = red[0];
    r.c = red[1];
    __syncthreads();
    return r;
}
__device__ __forceinline__ double csum_block(CSum v, double *red) { return csum_block_pair(v, red).value(); }

// ------------------------------------------------------------------ k_vort
#define VTX 60          // output columns of a vorticity tile
#define VTYMAX 17       // output rows of a vorticity tile (at most)
#define VTHREADS 256    // 64 column lanes x 4 row strips
#define XINV_E 16           // complex values per transform thread in k_xinv
#define XINV_FFT_MAX 512    // at most this many transform threads per k_xinv CTA

// Storage of q: FP64 handles keep q itself; FP32 handles keep the anomaly
// q - beta yprel (the planetary vorticity is most of q, and in FP32 its
// rounding would swamp the relative and stretching vorticity that the
// Helmholtz inversion recovers from q - beta y).  Every kernel that reads or
// writes q applies this; the host converts at the boundary (oqg_get_state,
// oqg_set_state_full).
template <class T> __host__ __device__ constexpr bool q_anom_stored() { return sizeof(T) == 4; }

// Geometry of a basin for the stencils; the coefficients sit in a shared
// table (K = fx, fy, fxb, fyb, jac) that the kernel fills once.
template <class T> struct GeoS {
    int nxp, nyp, cyclic;
    const T *K;
};
template <class T> __device__ __forceinline__ T gfx(const GeoS<T> &g) { return g.K[0]; }
template <class T> __device__ __forceinline__ T gfy(const GeoS<T> &g) { return g.K[1]; }
template <class T> __device__ __forceinline__ T gfxb(const GeoS<T> &g) { return g.K[2]; }
template <class T> __device__ __forceinline__ T gfyb(const GeoS<T> &g) { return g.K[3]; }
template <class T> __device__ __forceinline__ T gjac(const GeoS<T> &g) { return g.K[4]; }

// Laplacian with the mixed wall condition (del2_P_bc, numerics.F90:410-468)
// from the five stencil values (W, E, S, N, C): the interior formula, or on
// a wall the one-sided mixed-BC terms, chosen by selects (no divergent
// branches).  fx, fy: 1/dx^2, 1/dy^2; fxb, fyb: their mixed-BC factors.
template <class T>
__device__ __forceinline__ T lap5_sel(T wv, T ev, T sv, T nv, T c, bool zrow, bool wl, bool wr, bool jlo,
                                      bool jhi, T fx, T fy, T fxb, T fyb) {
    T xp = fx * (wv + ev - (T)2 * c);
    if (wl) xp = fxb * (ev - c);
    if (wr) xp = -(fxb * (c - wv));
    if (zrow) xp = (T)0;
    T yp = fy * (sv + nv - (T)2 * c);
    if (jlo) yp = fyb * (nv - c);
    if (jhi) yp = -(fyb * (c - sv));
    if (wl || wr) yp = (T)0;
    return xp + yp;
}

// cp.async copy of one element into shared memory; zero-filled when !valid
// (the source is then not read).
template <class T>
__device__ __forceinline__ void cp_async_el(T *dst, const T *src, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? (int)sizeof(T) : 0;
    if (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Queues the copy of rows [jlo, jlo+nr) x cols [ilo, ilo+nc) of layer k of f
// into s (leading dimension nc); outside the basin -> 0.  Channel columns of
// a halo tile wrap with period nxp-1; an `own` tile (the CTA's output columns
// only) reads columns < nxp as stored, including the duplicate column nxp-1,
// and zeros beyond, so it never reads a column that another CTA writes.
// Thread layout: 64 columns x 4 rows.
template <class T, class G>
__device__ __forceinline__ void load_tile_async(T *s, const T *__restrict__ f, const G &g, int px,
                                                int k, int jlo, int nr, int ilo, int nc,
                                                bool own = false) {
    const int N = g.nxp - 1;
    const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;
    const T *fk = f + (size_t)k * g.nyp * px;
    for (int r = ty; r < nr; r += 4) {
        const int j = jlo + r;
        const bool jv = (j >= 0 && j < g.nyp);
        const T *row = fk + (size_t)(jv ? j : 0) * px;
        for (int c = tx; c < nc; c += 64) {
            int i = ilo + c;
            bool v = jv;
            if (g.cyclic && !own) {
                while (i < 0) i += N;
                while (i >= N) i -= N;
            } else {
                v = v && i >= 0 && i < g.nxp;
            }
            cp_async_el(s + r * nc + c, row + (v ? i : 0), v);
        }
    }
}

// Tiles are VTX columns by b.vty rows (b.vty <= VTYMAX, chosen per basin so
// that the tiles fill whole waves); a box's tile rows start at row 1.  Shared tiles per layer (origin, pitch):
//   pm     rows j0-3 .. j0+vty+2, cols from i0-4   (LPQ = VTX+8 = 68)
//   p, q   rows j0-1 .. j0+vty,   cols from i0-4   (LPQ)
//   qm     rows j0 .. j0+vty-1,   cols from i0     (LO = VTX)
//   d2     rows j0-2 .. j0+vty+1, cols from i0-2   (L2 = VTX+4 = 64), computed
//   d4     rows j0-1 .. j0+vty,   cols from i0-1   (L1 = VTX+2), computed
// The x-origins are multiples of 4 elements (16 bytes), as tensor loads need.
// Closed-box tiles arrive by TMA (one thread issues, an mbarrier counts the
// bytes); channel tiles wrap periodically and come by cp.async.  Thread
// (lane x, strip y) owns column x of each phase and marches down a strip of
// rows with a rolling window of the stencil in registers.
struct VortLayout {
    int HPM, H2, H1, VT;
    int pm, p, q, qm, nbuf;     // offsets within a layer buffer (elements)
    int d2, d4, wk, by, total;  // offsets after the two layer buffers
};
__host__ __device__ __forceinline__ int vort_round(int n, int esz) {
    const int a = 128 / esz;
    return (n + a - 1) / a * a;
}
__host__ __device__ __forceinline__ VortLayout vort_layout(int vt, int esz) {
    constexpr int LPQ = VTX + 8, L2 = VTX + 4, L1 = VTX + 2, LO = VTX;
    VortLayout L;
    L.VT = vt;
    L.HPM = vt + 6;
    L.H2 = vt + 4;
    L.H1 = vt + 2;
    L.pm = 0;
    L.p = L.pm + vort_round(L.HPM * LPQ, esz);
    L.q = L.p + vort_round(L.H1 * LPQ, esz);
    L.qm = L.q + vort_round(L.H1 * LPQ, esz);
    L.nbuf = L.qm + vort_round(vt * LO, esz);
    L.d2 = 2 * L.nbuf;
    L.d4 = L.d2 + vort_round(L.H2 * L2, esz);
    L.wk = L.d4 + vort_round(L.H1 * L1, esz);
    L.by = L.wk + vort_round(vt * LO, esz);
    L.total = L.by + vort_round(vt * 8 / esz + 1, esz);   // vt doubles
    return L;
}
// Rows of vorticity tiles: a box tiles its interior rows, a channel all.
__host__ __device__ __forceinline__ int vort_tile_rows(int nyp, int cyclic, int vt) {
    return cyclic ? (nyp + vt - 1) / vt : (nyp - 2 + vt - 1) / vt;
}
// Dynamic shared bytes of k_vort (plus slack to align the base to 128 bytes).
__host__ __device__ __forceinline__ size_t vort_smem_bytes(int vt, int esz) {
    return (size_t)vort_layout(vt, esz).total * esz + 128;
}

// Tensor maps of a box basin, in this order: p/q-shaped boxes of F[0..3],
// pm-shaped boxes of F[0], F[1], qm-shaped boxes of F[2], F[3], wekp.
#define OQG_TMAP_PQ 0
#define OQG_TMAP_PM 4
#define OQG_TMAP_QM 6
#define OQG_TMAP_WK 8
#define OQG_NTMAP 9
#define OQG_TMAP_BYTES 128

// tdt = 0: each member steps with its own b.tdt_m (ensemble launches).
// VT: the tile's rows (b.vty), a compile-time multiple of 4 (vort_tile_rows),
// so every strip's row loop has a fixed trip count: the loops unroll with no
// predicates and the rolling windows live in renamed registers.
template <class T, int NL, int VT>
__global__ void __launch_bounds__(VTHREADS, 2)
k_vort(const BasinDev *__restrict__ bas, const Work *__restrict__ work, int par, double tdt) {
    static_assert(VT % 4 == 0 && VT >= 8 && VT <= VTYMAX, "tile rows: a multiple of 4 in [8, VTYMAX]");
    constexpr int LPQ = VTX + 8, L2 = VTX + 4, L1 = VTX + 2, LO = VTX;
    constexpr int HPM = VT + 6, H2 = VT + 4, H1 = VT + 2;
    // rows per strip of each phase (4 strips); the last d4 strip starts
    // early and recomputes a row or two of its neighbour (the same values)
    constexpr int RMAX = VT / 4, R2MAX = H2 / 4, R1MAX = (H1 + 3) / 4;
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    // uniform constants in shared memory: fx fy fxb fyb jac | c_ent1 c_wind
    // c_ent2 c_drag tdt | c2[k] | c4[k]; FP64 ctl2m
    __shared__ T sK[11 + 2 * OQG_NLMAX];
    __shared__ double sCtl[NL * NL];
    // FP32 storage keeps q as its anomaly q - beta yprel (q_anom_stored): the
    // planetary term's Jacobian then comes from p alone (its coefficient,
    // jac_fac beta dy, is sK[10 + 2 NL])
    constexpr bool QA = q_anom_stored<T>();
    if (QA && threadIdx.x == 10 + 2 * NL) sK[10 + 2 * NL] = (T)(b.jac_fac * b.beta * b.dy);
    if (threadIdx.x < 10 + 2 * NL) {
        const int i = threadIdx.x;
        T v;
        if (i == 0) v = (T)b.fx; else if (i == 1) v = (T)b.fy; else if (i == 2) v = (T)b.fx_bc;
        else if (i == 3) v = (T)b.fy_bc; else if (i == 4) v = (T)b.jac_fac; else if (i == 5) v = (T)b.c_ent1;
        else if (i == 6) v = (T)b.c_wind; else if (i == 7) v = (T)b.c_ent2; else if (i == 8) v = (T)b.c_drag;
        else if (i == 9) v = (T)(tdt != 0.0 ? tdt : b.tdt_m); else if (i < 10 + NL) v = (T)b.c2[i - 10]; else v = (T)b.c4[i - 10 - NL];
        sK[i] = v;
    }
    if (threadIdx.x < NL * NL) sCtl[threadIdx.x] = b.ctl2m[threadIdx.x];
    GeoS<T> g;
    g.nxp = b.nxp; g.nyp = b.nyp; g.cyclic = b.cyclic; g.K = sK;
    const VortLayout LY = vort_layout(VT, (int)sizeof(T));
    const int tile_x = w.block % b.tiles_x, tile_y = w.block / b.tiles_x;
    // a box's tiles cover its interior rows 1 .. nyp-2 (the walls are not
    // stepped); a channel's start at row 0 (its strip integrals hold row 0)
    const int i0 = tile_x * VTX, j0 = tile_y * VT + (g.cyclic ? 0 : 1);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sm = reinterpret_cast<T *>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    T *sD2 = sm + LY.d2;
    T *sD4 = sm + LY.d4;
    T *sWK = sm + LY.wk;
    double *sBY = reinterpret_cast<double *>(sm + LY.by);
    __shared__ double red[32];
    __shared__ __align__(8) unsigned long long bars[2];

    T *QM = (T *)b.F[3 - par];
    const T *ENT = (const T *)b.ent;
    const double *__restrict__ DD = b.ddyn;
    const int N = g.nxp - 1;
    const int nyp = g.nyp, nxp = g.nxp, px = b.px, kt = b.kt;
    const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;
    const bool tma = !g.cyclic && b.tmaps != nullptr;
    const unsigned char *tm = (const unsigned char *)b.tmaps;

    if (tma && threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    // beta * yprel of the tile's rows (constant)
    for (int r = threadIdx.x; r < VT; r += blockDim.x) {
        const int gj = j0 + r;
        sBY[r] = gj < nyp ? b.beta * b.yprel[gj] : 0.0;
    }
    __syncthreads();
    pdl_trigger();
    pdl_wait();

    auto issue = [&](int k) {
        T *bf = sm + (k & 1) * LY.nbuf;
        if (tma) {
            if (threadIdx.x == 0) {
                fence_proxy_async();
                unsigned bytes = (unsigned)((HPM * LPQ + 2 * H1 * LPQ + VT * LO) * sizeof(T));
                if (k == 0) bytes += (unsigned)(VT * LO * sizeof(T));
                unsigned long long *bar = &bars[k & 1];
                mbar_expect_tx(bar, bytes);
                tma_load_3d(bf + LY.pm, tm + (OQG_TMAP_PM + 1 - par) * OQG_TMAP_BYTES, i0 - 4, j0 - 3, k, bar);
                tma_load_3d(bf + LY.p, tm + (OQG_TMAP_PQ + par) * OQG_TMAP_BYTES, i0 - 4, j0 - 1, k, bar);
                tma_load_3d(bf + LY.q, tm + (OQG_TMAP_PQ + 2 + par) * OQG_TMAP_BYTES, i0 - 4, j0 - 1, k, bar);
                tma_load_3d(bf + LY.qm, tm + (OQG_TMAP_QM + 1 - par) * OQG_TMAP_BYTES, i0, j0, k, bar);
                if (k == 0) tma_load_2d(sWK, tm + OQG_TMAP_WK * OQG_TMAP_BYTES, i0, j0, bar);
            }
        } else {
            load_tile_async(bf + LY.pm, (const T *)b.F[1 - par], g, px, k, j0 - 3, HPM, i0 - 4, LPQ);
            load_tile_async(bf + LY.p, (const T *)b.F[par], g, px, k, j0 - 1, H1, i0 - 4, LPQ);
            load_tile_async(bf + LY.q, (const T *)b.F[2 + par], g, px, k, j0 - 1, H1, i0 - 4, LPQ);
            load_tile_async(bf + LY.qm, (const T *)QM, g, px, k, j0, VT, i0, LO, true);
            if (k == 0) load_tile_async(sWK, (const T *)b.wekp, g, px, 0, j0, VT, i0, LO, true);
            cp_async_commit();
        }
    };
    issue(0);

    // strips of rows: [ty*R, ty*R + R) of each region
    constexpr int R2 = R2MAX, R1 = R1MAX, R0 = RMAX;
    const int r0 = ty * R0;
    double acc[RMAX][NL];
#pragma unroll
    for (int u = 0; u < RMAX; ++u)
#pragma unroll
        for (int m = 0; m < NL; ++m) acc[u][m] = 0.0;
    const bool topo = b.topo_active != 0;
    // channel strip integrals are formed by tiles holding rows 0, 1, nyp-2, nyp-1
    const bool strips = g.cyclic && (j0 <= 1 || j0 + VT > nyp - 2);
    // in-domain test of a column (a channel has none outside)
    auto colok = [&](int gi) { return g.cyclic || (gi >= 0 && gi < nxp); };
    // the del2 region (rows j0-2 .. j0+VT+1, columns i0-2 .. i0+VTX+1) lies
    // strictly inside the walls, and every output column exists
    const bool interior = (j0 - 2 >= 1 && j0 + VT + 1 <= nyp - 2) &&
                          (g.cyclic ? (i0 + VTX <= nxp) : (i0 - 2 >= 1 && i0 + VTX + 1 <= nxp - 2));

#pragma unroll 1
    for (int k = 0; k < NL; ++k) {
        if (k + 1 < NL) issue(k + 1);
        if (tma) {
            // one thread polls the barrier; the CTA barrier then publishes
            // the tile to the others without spinning warps taking issue slots
            bool ok = true;
            if (threadIdx.x == 0) ok = mbar_wait_bounded(&bars[k & 1], (k >> 1) & 1, b.wait_limit);
            if (__syncthreads_or(!ok)) {
                // a tile never arrived: report, drain what is in flight, stop
                if (threadIdx.x == 0) {
                    atomicOr(b.err, OQG_DERR_TIMEOUT);
                    mbar_wait_bounded(&bars[k & 1], (k >> 1) & 1, OQG_WAIT_LIMIT);
                    if (k + 1 < NL) mbar_wait_bounded(&bars[(k + 1) & 1], ((k + 1) >> 1) & 1, OQG_WAIT_LIMIT);
                }
                __syncthreads();
                return;
            }
        } else {
            if (k + 1 < NL) cp_async_wait<1>();
            else cp_async_wait<0>();
            __syncthreads();
        }
        const T *sPM = sm + (k & 1) * LY.nbuf + LY.pm;
        const T *sP = sm + (k & 1) * LY.nbuf + LY.p;
        const T *sQ = sm + (k & 1) * LY.nbuf + LY.q;
        const T *sQM = sm + (k & 1) * LY.nbuf + LY.qm;
        // The layer's stencils; I: every point of the tile and its halo is
        // off the walls, so the wall rules and range tests drop out.
        auto layer = [&](auto inner) {
            constexpr bool I = decltype(inner)::value;
            const T fx = gfx(g), fy = gfy(g), fxb = gfxb(g), fyb = gfyb(g);
            // ---- del2(pm) on rows j0-2.., cols i0-2.. (column tx of L2 = 64)
            {
                const int gi = i0 - 2 + tx, cs = tx + 2;          // column in the pm tile
                const bool cv = colok(gi);
                const bool wl = !g.cyclic && gi == 0, wr = !g.cyclic && gi == nxp - 1;
                const int rb = ty * R2;          // H2 = 4 R2: the strips tile exactly
                const T *col = sPM + rb * LPQ + cs;
                T sv = col[0], cv_ = col[LPQ];
    #pragma unroll
                for (int u = 0; u < R2MAX; ++u) {
                    const int r = rb + u;
                    {
                        const T nv = col[(u + 2) * LPQ];
                        const T wv = col[(u + 1) * LPQ - 1], ev = col[(u + 1) * LPQ + 1];
                        const int gj = j0 - 2 + r;
                        T v = (T)0;
                        if (I) v = fx * (wv + ev - (T)2 * cv_) + fy * (sv + nv - (T)2 * cv_);
                        else if (cv && gj >= 0 && gj < nyp)
                            v = lap5_sel(wv, ev, sv, nv, cv_, gj == 0 || gj == nyp - 1, wl, wr, gj == 0,
                                         gj == nyp - 1, fx, fy, fxb, fyb);
                        sD2[r * L2 + tx] = v;
                        sv = cv_;
                        cv_ = nv;
                    }
                }
            }
            __syncthreads();
            // ---- del4 on rows j0-1.., cols i0-1.. (column tx < L1 = 62)
            if (tx < L1) {
                const int gi = i0 - 1 + tx, cs = tx + 1;          // column in the d2 tile
                const bool cv = colok(gi);
                const bool wl = !g.cyclic && gi == 0, wr = !g.cyclic && gi == nxp - 1;
                const int rb = min(ty * R1, H1 - R1);
                const T *col = sD2 + rb * L2 + cs;
                T sv = col[0], cv_ = col[L2];
    #pragma unroll
                for (int u = 0; u < R1MAX; ++u) {
                    const int r = rb + u;
                    {
                        const T nv = col[(u + 2) * L2];
                        const T wv = col[(u + 1) * L2 - 1], ev = col[(u + 1) * L2 + 1];
                        const int gj = j0 - 1 + r;
                        T v = (T)0;
                        if (I) v = fx * (wv + ev - (T)2 * cv_) + fy * (sv + nv - (T)2 * cv_);
                        else if (cv && gj >= 0 && gj < nyp)
                            v = lap5_sel(wv, ev, sv, nv, cv_, gj == 0 || gj == nyp - 1, wl, wr, gj == 0,
                                         gj == nyp - 1, fx, fy, fxb, fyb);
                        sD4[r * L1 + tx] = v;
                        sv = cv_;
                        cv_ = nv;
                    }
                }
            }
            __syncthreads();

            // ---- outputs: column tx < VTX, rows r0 .. r0+R0-1 of the tile.
            // Only points off the solid walls are stepped: on a wall the Arakawa
            // Jacobian is zero and the stepped q is replaced by ocqbdy
            // (vorsubs.F90:58-114) in the assembly kernel, so the interior
            // stencils are the whole computation here.
            if (tx < VTX) {
                const int gi = i0 + tx;
                const bool xin = g.cyclic ? (gi < nxp) : (gi >= 1 && gi <= nxp - 2);
                const T *d4col = sD4 + r0 * L1 + tx + 1;       // column in the d4 tile
                const T *pcol = sP + r0 * LPQ + tx + 4;         // column in the p/q tiles
                const T *qcol = sQ + r0 * LPQ + tx + 4;
                // rolling windows: d4 (column), p and q (3 x 3)
                T d4s = d4col[0], d4c = d4col[L1];
                T pw[3][3], qw[3][3];
    #pragma unroll
                for (int a = 0; a < 2; ++a)
    #pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        pw[a + 1][cc] = pcol[a * LPQ - 1 + cc];
                        qw[a + 1][cc] = qcol[a * LPQ - 1 + cc];
                    }
    #pragma unroll
                for (int u = 0; u < RMAX; ++u) {
                    const int r = r0 + u;
                    const int gj = j0 + r;
                    {
                        // shift the windows down one row and load the new bottom row
                        const T d4n = d4col[(u + 2) * L1];
                        const T d4w = d4col[(u + 1) * L1 - 1], d4e = d4col[(u + 1) * L1 + 1];
    #pragma unroll
                        for (int cc = 0; cc < 3; ++cc) {
                            pw[0][cc] = pw[1][cc]; pw[1][cc] = pw[2][cc];
                            qw[0][cc] = qw[1][cc]; qw[1][cc] = qw[2][cc];
                            pw[2][cc] = pcol[(u + 2) * LPQ - 1 + cc];
                            qw[2][cc] = qcol[(u + 2) * LPQ - 1 + cc];
                        }
                        if (I || (xin && gj >= 1 && gj <= nyp - 2)) {
                            const T d6 = fx * (d4w + d4e - (T)2 * d4c) + fy * (d4s + d4n - (T)2 * d4c);
                            // Arakawa J(q, p), numerics.F90:370-372
                            const T pxc = pw[1][2] - pw[1][0], pyc = pw[2][1] - pw[0][1];
                            const T qxc = qw[1][2] - qw[1][0], qyc = qw[2][1] - qw[0][1];
                            const T A = qw[1][2] * (pw[2][2] - pw[0][2]) - qw[1][0] * (pw[2][0] - pw[0][0]);
                            const T Dd = pw[1][2] * (qw[2][2] - qw[0][2]) - pw[1][0] * (qw[2][0] - qw[0][0]);
                            const T Bv = qw[2][1] * (pw[2][2] - pw[2][0]) - qw[0][1] * (pw[0][2] - pw[0][0]);
                            const T Cc = pw[2][1] * (qw[2][2] - qw[2][0]) - pw[0][1] * (qw[0][2] - qw[0][0]);
                            T jac = gjac(g) * (qxc * pyc - qyc * pxc + A - Bv + Cc - Dd);
                            if (QA) {
                                // + J(beta y, p): the Arakawa sum of a field linear in y is
                                // -dy (4 (pE - pW) + (pNE - pNW) + (pSE - pSW)); explicit FMAs
                                // keep the rounding the same in every tile instance
                                const T py = fma((T)4, pxc, (pw[2][2] - pw[2][0]) + (pw[0][2] - pw[0][0]));
                                jac = fma(-sK[10 + 2 * NL], py, jac);
                            }
                            T dq = jac + sK[10 + k] * d4c - sK[10 + NL + k] * d6;
                            const size_t o2 = (size_t)gj * px + gi;
                            if (k == 0) {
                                const T e1 = ENT ? ldg(ENT + o2) : (T)0;
                                dq = dq + sK[5] * e1 + sK[6] * sWK[r * LO + tx];
                            }
                            if (k == 1 && ENT) dq = dq - sK[7] * ldg(ENT + o2);
                            if (k == kt) dq = dq - sK[8] * sD2[(r + 2) * L2 + tx + 2];
                            const T qn = sQM[r * LO + tx] + sK[9] * dq;
                            QM[((size_t)k * nyp + gj) * px + gi] = qn;
                            // modal right-hand side, FP64 (p_modes_rhs)
                            double ql = QA ? (double)qn : (double)qn - sBY[r];
                            if (k == kt && topo) ql -= DD[o2];
    #pragma unroll
                            for (int m = 0; m < NL; ++m) acc[u][m] += ql * sCtl[k + NL * m];
                        }
                        d4s = d4c;
                        d4c = d4n;
                    }
                }
            }
        };
        if (interior) layer(std::true_type{});
        else layer(std::false_type{});
        if (strips) {
            // channel strip integrands (vorticity.F90:84-101, numerics.F90:374-386)
            // of the rows 0, 1, nyp-2, nyp-1 held by this tile
            double sq[OQG_NQ];
#pragma unroll
            for (int q = 0; q < OQG_NQ; ++q) sq[q] = 0.0;
            const int gi = i0 + tx;
            if (ty == 0 && tx < VTX && gi < N) {
                for (int r = 0; r < VT; ++r) {
                    const int gj = j0 + r;
                    if (!(gj == 0 || gj == 1 || gj == nyp - 2 || gj == nyp - 1)) continue;
                    const int c = tx + 4;                   // p/q tile column
                    // q itself (FP32 storage holds q - beta y), in FP64
                    const double qc = QA ? (double)sQ[(r + 1) * LPQ + c] + sBY[r] : (double)sQ[(r + 1) * LPQ + c];
                    const T d2 = sD2[(r + 2) * L2 + tx + 2], d4 = sD4[(r + 1) * L1 + tx + 1];
                    if (gj == 0) {
                        sq[0] += qc * (double)(sP[(r + 2) * LPQ + c + 1] - sP[(r + 2) * LPQ + c - 1]);
                        sq[4] += (double)(sD2[(r + 3) * L2 + tx + 2] - d2);
                        sq[6] += (double)(sD4[(r + 2) * L1 + tx + 1] - d4);
                        if (k == kt)
                            sq[8] += (double)(sPM[(r + 4) * LPQ + tx + 4] - sPM[(r + 3) * LPQ + tx + 4]);
                    }
                    if (gj == 1) sq[1] += qc * (double)(sP[(r + 1) * LPQ + c + 1] - sP[(r + 1) * LPQ + c - 1]);
                    if (gj == nyp - 1) {
                        sq[2] += qc * (double)(sP[r * LPQ + c + 1] - sP[r * LPQ + c - 1]);
                        sq[5] += (double)(d2 - sD2[(r + 1) * L2 + tx + 2]);
                        sq[7] += (double)(d4 - sD4[r * L1 + tx + 1]);
                        if (k == kt)
                            sq[9] += (double)(sPM[(r + 3) * LPQ + tx + 4] - sPM[(r + 2) * LPQ + tx + 4]);
                    }
                    if (gj == nyp - 2) sq[3] += qc * (double)(sP[(r + 1) * LPQ + c + 1] - sP[(r + 1) * LPQ + c - 1]);
                }
            }
            // only the row ty = 0 (warps 0 and 1) holds terms: reduce the
            // OQG_NQ sums together in those two warps, then add warp 1's to
            // warp 0's (the value block_sum gives, without its barriers)
            double *pt = b.part_tile + ((size_t)w.block * b.nl + k) * OQG_NQ;
            if (ty == 0) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                    for (int q = 0; q < OQG_NQ; ++q) sq[q] += __shfl_down_sync(0xffffffffu, sq[q], o);
                if (threadIdx.x == 32)
#pragma unroll
                    for (int q = 0; q < OQG_NQ; ++q) red[q] = sq[q];
            }
            __syncthreads();
            if (threadIdx.x == 0)
#pragma unroll
                for (int q = 0; q < OQG_NQ; ++q) pt[q] = sq[q] + red[q];
        }
        __syncthreads();
    }

    // write the modal right-hand side of the interior points
    T *RHS = (T *)b.rhs;
    const int ioff = g.cyclic ? 0 : 1;
    const double f0 = b.fnot;
    if (tx < VTX) {
#pragma unroll
        for (int u = 0; u < RMAX; ++u) {
            const int r = r0 + u;
            const int gj = j0 + r, gi = i0 + tx;
            if (gj < 1 || gj > nyp - 2) continue;
            const int xi = gi - ioff;
            if (xi < 0 || xi >= b.nxin) continue;
#pragma unroll
            for (int m = 0; m < NL; ++m)
                RHS[((size_t)m * b.ny + (gj - 1)) * b.pr + xi] = (T)(f0 * acc[u][m]);
        }
    }
}

// ------------------------------------------------------------------ k_xfwd
// Threads per transform TT = ceil(M/E); G = blockDim/TT transforms per CTA.
// Shared memory: per group two padded buffers of fft_buf_len(M) complex
// values; the input rows are staged by cp.async into the second buffer and
// expanded into the first.  The stage twiddles are read from global memory.
__host__ __device__ __forceinline__ int round16(int bytes) { return (bytes + 15) & ~15; }

// MC > 0: an instance for transforms of length MC only (the host picks it
// for a basin of that length); MC = 0 serves any length (ensembles).
template <class T, int E, int MC = 0>
__global__ void __launch_bounds__(256, 2)
k_xfwd(const BasinDev *__restrict__ bas, const Work *__restrict__ work, const void *rhs_override) {
    typedef typename C2<T>::t T2;
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = MC > 0 ? MC : b.M, TT = (M + E - 1) / E, G = blockDim.x / TT;
    const int g = threadIdx.x / TT, t = threadIdx.x - g * TT;
    const int LB = fft_buf_len(M);
    T2 *zs = reinterpret_cast<T2 *>(smem_raw);
    const int npm = (b.ny + 1) >> 1;          // row pairs per mode
    const int pair = w.block * G + g;
    const bool live = g < G && pair < b.nl * npm;
    const int m = live ? pair / npm : 0;
    const int j = live ? 2 * (pair - m * npm) : 0;
    const bool two = live && (j + 1 < b.ny);
    const int n = b.nxin;
    const int RO = (n + 3) & ~3;              // offset of the second row (16-byte aligned)
    // the long lengths transform in place: one buffer per group, the input
    // rows staged after all the groups' buffers
    const bool ip = E == 16 && fft_inplace_len(M);
    T2 *za = zs + (size_t)(g < G ? g : 0) * (ip ? LB : 2 * LB);
    T2 *zb = za + LB;
    T *raw = ip ? reinterpret_cast<T *>(zs + (size_t)G * LB) + (size_t)(g < G ? g : 0) * 2 * RO
                : reinterpret_cast<T *>(zb);
    const T *R = (const T *)(rhs_override ? rhs_override : b.rhs);
    const T *x = R + ((size_t)m * b.ny + j) * b.pr;
    pdl_trigger();
    pdl_wait();
    if (live) {
        cp_async_16(raw, x, round16(n * (int)sizeof(T)), t, TT);
        if (two) cp_async_16(raw + RO, x + b.pr, round16(n * (int)sizeof(T)), t, TT);
    }
    cp_async_commit_wait_all();
    __syncthreads();
    if (live) {
        if (!b.cyclic) {
            // odd extension of two rows: z_0 = z_{n+1} = 0, z_{M-jj} = -z_jj
            if (t == 0) {
                T2 zero;
                zero.x = (T)0;
                zero.y = (T)0;
                za[fpad(0)] = zero;
                za[fpad(n + 1)] = zero;
            }
            for (int jj = 1 + t; jj <= n; jj += TT) {
                T2 v, vm;
                v.x = raw[jj - 1];
                v.y = two ? raw[RO + jj - 1] : (T)0;
                vm.x = -v.x;
                vm.y = -v.y;
                za[fpad(jj)] = v;
                za[fpad(M - jj)] = vm;
            }
        } else {
            for (int jj = t; jj < M; jj += TT) {
                T2 v;
                v.x = raw[jj];
                v.y = two ? raw[RO + jj] : (T)0;
                za[fpad(jj)] = v;
            }
        }
    }
    __syncthreads();
    T2 *z = za;
    if (ip) fft_inplace<T, MC>(za, M, (const T2 *)b.tw, live ? t : M, 0, 0);
    else z = fft_run<T, E, MC>(za, zb, M, b.rad, b.nrad, (const T2 *)b.tw, live ? t : TT, TT, 0, 0);
    if (!live) return;
    if (!b.cyclic) {
        T *S = (T *)b.spec;
        T *sx = S + ((size_t)m * b.ny + j) * b.pk;
        T *sy = sx + b.pk;
        for (int kk = t; kk < n; kk += TT) {
            const T2 v = z[fpad(kk + 1)];
            sx[kk] = -v.y;
            if (two) sy[kk] = v.x;
        }
    } else {
        T2 *S = (T2 *)b.spec;
        T2 *sx = S + ((size_t)m * b.ny + j) * b.pk;
        T2 *sy = sx + b.pk;
        for (int kk = t; kk < b.nk; kk += TT) {
            const T2 a = z[fpad(kk)], c = z[fpad((M - kk) % M)];
            T2 X, Y;
            X.x = (T)0.5 * (a.x + c.x);
            X.y = (T)0.5 * (a.y - c.y);
            // (a - conj(c)) / (2i)
            const T dx_ = (T)0.5 * (a.x - c.x), dy_ = (T)0.5 * (a.y + c.y);
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

// The maps of the two sweeps compose across the lanes of a column: lane l's
// rows give an affine map u_out = C + D u_in, and the lanes' maps are scanned
// in sweep order.  A column spread over W warps also composes across them:
// each warp publishes its aggregate map (lane 31 going down the rows, lane 0
// going up) and a warp's carry-in is the composition of the warps before it.
// Returns this lane's input value: its exclusive prefix applied to the carry.
// Every thread of the CTA calls it (a CTA barrier when W > 1).
template <class V, int W, bool DOWN>
__device__ __forceinline__ V ysolve_scan(V C, double D, int lane, int wc, V *sC, double *sD) {
    for (int q = 1; q < 32; q <<= 1) {
        const V Co = DOWN ? yt_up(C, q) : yt_dn(C, q);
        const double Do = DOWN ? shfl_up_d(D, q) : shfl_dn_d(D, q);
        if (DOWN ? lane >= q : lane + q < 32) { C = yt_axpy(C, D, Co); D = D * Do; }
    }
    V Ce = DOWN ? yt_up(C, 1) : yt_dn(C, 1);
    if constexpr (W == 1) {
        if (lane == (DOWN ? 0 : 31)) Ce = yt_zero(V());
        return Ce;
    } else {
        double De = DOWN ? shfl_up_d(D, 1) : shfl_dn_d(D, 1);
        if (lane == (DOWN ? 0 : 31)) { Ce = yt_zero(V()); De = 1.0; }
        if (lane == (DOWN ? 31 : 0)) { sC[wc] = C; sD[wc] = D; }
        __syncthreads();
        V u = yt_zero(V());
        if (DOWN) { for (int v = 0; v < wc; ++v) u = yt_axpy(sC[v], sD[v], u); }
        else { for (int v = W - 1; v > wc; --v) u = yt_axpy(sC[v], sD[v], u); }
        return yt_axpy(Ce, De, u);
    }
}

// The column solve with each lane's rows [s, s+SM) held in registers through
// all four passes: forward elimination as an affine scan (chunk pass, scan
// of the chunk maps, chunk pass), then back substitution the same way from
// the bottom.  Rows at or beyond ny are padding: their value and pivot are
// zero, so they map everything to zero in both sweeps and the last row's
// zero neighbour below needs no special case; the passes then run without
// per-row predicates.  col: the column in shared memory at padded offset o;
// piv: its pivots (global, plen stored); sC/sD: the column's W carry slots
// of each sweep.
#define YREG 16
template <class V, int W, int SM>
__device__ __forceinline__ void ysolve_chunk_regs(V *col, const double *__restrict__ piv, int plen, double a,
                                                  int lane, int wc, int s, int o, int ny, V *sC, double *sD,
                                                  CSum &colsum) {
    V x[SM];
    double bt[SM];
#pragma unroll
    for (int t = 0; t < SM; ++t) {
        const bool in = s + t < ny;
        x[t] = in ? col[o + t] : yt_zero(V());
        bt[t] = in ? __ldg(piv + min(s + t, plen - 1)) : 0.0;
    }
    // forward elimination: u_j = f_j beta_j - a beta_j u_{j-1}
    V C = yt_zero(V());
    double D = 1.0;
#pragma unroll
    for (int t = 0; t < SM; ++t) {
        C = yt_axpy(yt_scale(x[t], bt[t]), -a * bt[t], C);
        D = -a * bt[t] * D;
    }
    V uu = ysolve_scan<V, W, true>(C, D, lane, wc, sC, sD);
#pragma unroll
    for (int t = 0; t < SM; ++t) {
        uu = yt_axpy(yt_scale(x[t], bt[t]), -a * bt[t], uu);
        x[t] = uu;
    }
    // back substitution: u_j = u'_j - a beta_j u_{j+1}
    C = yt_zero(V());
    D = 1.0;
#pragma unroll
    for (int t = SM - 1; t >= 0; --t) {
        const double ej = -a * bt[t];
        C = yt_axpy(x[t], ej, C);
        D = ej * D;
    }
    uu = ysolve_scan<V, W, false>(C, D, lane, wc, sC + W, sD + W);
#pragma unroll
    for (int t = SM - 1; t >= 0; --t) {
        const double ej = -a * bt[t];
        uu = yt_axpy(x[t], ej, uu);
        x[t] = uu;
        // the box's dst_w-weighted column sum (a channel has none)
        if constexpr (std::is_same<V, double>::value) colsum.add(yt_re(uu));
    }
#pragma unroll
    for (int t = 0; t < SM; ++t)
        if (s + t < ny) col[o + t] = x[t];
}

// Rows per lane of a column spread over W warps and the padded column
// length of its tile: up to 32 W YREG rows the smallest of 4, 8 and 16 rows
// per lane that covers them (the register path, one instance each), beyond
// that ceil(ny / 32 W) rows per lane through shared memory.
__host__ __device__ __forceinline__ int ysolve_rows_per_lane(int ny, int W) {
    const int L = 32 * W;
    return ny <= 4 * L ? 4 : ny <= 8 * L ? 8 : ny <= YREG * L ? YREG : (ny + L - 1) / L;
}
__host__ __device__ __forceinline__ int ysolve_ld(int ny, int W) {
    const int s = ysolve_rows_per_lane(ny, W);
    const int need = 32 * W * (s + 1) + 1;             // 32 W lanes of s rows, one pad each
    const int ld = (ny + 32) | 1;
    return ld > need ? ld : (need | 1);
}

// One column per W warps, 4 columns per CTA (blockDim = 128 W).  More warps
// per column cut the rows each lane carries through the sweeps and put more
// warps on the SMs when the grid has few columns.
template <class T, bool CPLX, int W>
__global__ void __launch_bounds__(128 * W, W == 1 ? 1 : W == 2 ? 3 : 1)
k_ysolve(const BasinDev *__restrict__ bas, const Work *__restrict__ work) {
    typedef typename YT<T, CPLX>::v V;
    typedef typename YT<T, CPLX>::g Gm;
    constexpr int KB = 4;                       // columns per CTA
    constexpr int NT = 128 * W;                 // threads
    constexpr int CH = 16 / W;                  // loads in flight per thread and pass
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int c = wid / W, wc = wid - c * W;    // column of the CTA, warp within it
    const int nk = b.nk, ny = b.ny, pk = b.pk;
    const int nkb = (nk + KB - 1) / KB;
    const int m = w.block / nkb, k0 = (w.block - m * nkb) * KB;
    // Lane l of warp wc owns rows [(32 wc + l) S, +S).  Columns are stored
    // with one pad word per S rows (row j at j + j / S), so the 32 lanes of a
    // warp reading their chunks hit distinct banks.
    const int S_ = ysolve_rows_per_lane(ny, W);
    const int LD = ysolve_ld(ny, W);            // > 32 W (S + 1), odd
    const FastDiv fdS(S_);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tile = reinterpret_cast<V *>(smem_raw);                 // [KB][LD]
    __shared__ V sC[KB][2 * W];                 // carries of the two sweeps
    __shared__ double sD[KB][2 * W];
    const int k = k0 + c;
    const bool live = k < nk;
    const int pidx = m * nk + (live ? k : 0);
    // this column's pivots (constant data, read through L1); beyond the
    // stored length a pivot repeats its fixed point
    const double *__restrict__ piv = b.piv_tab + b.piv_off[pidx];
    const int plen = b.piv_len[pidx];
    Gm *S = (Gm *)b.spec + (size_t)m * ny * pk;
    pdl_trigger();
    pdl_wait();
    // load the spectral columns: thread -> (row, column), coalesced along k
    for (int i0 = threadIdx.x; i0 < ny * KB; i0 += NT * CH) {
        V v[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int idx = i0 + NT * u;
            const int jj = idx >> 2, cc = idx & 3, kk = k0 + cc;
            v[u] = (idx < ny * KB && kk < nk) ? yt_load(S[(size_t)jj * pk + kk]) : yt_zero(V());
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int idx = i0 + NT * u;
            const int jj = idx >> 2, cc = idx & 3;
            if (idx < ny * KB) tile[cc * LD + jj + fdS.div(jj)] = v[u];
        }
    }
    __syncthreads();

    // Every warp runs the sweeps (a column past nk solves zeros) so that the
    // carry barriers are uniform over the CTA.
    const double a = b.a_tri;
    V *col = tile + c * LD;
    const int gl = wc * 32 + lane;
    const int s = gl * S_, e = min(s + S_, ny);
    const int o = gl * (S_ + 1);                // padded offset of row s
    const int n = max(e - s, 0);
    CSum colsum;
    if (S_ == 4) ysolve_chunk_regs<V, W, 4>(col, piv, plen, a, lane, wc, s, o, ny, sC[c], sD[c], colsum);
    else if (S_ == 8) ysolve_chunk_regs<V, W, 8>(col, piv, plen, a, lane, wc, s, o, ny, sC[c], sD[c], colsum);
    // (16 rows per lane with one warp per column, and with four for the
    // box; the two-warp instances run at most 8 within their register budget)
    else if ((W == 1 || (W == 4 && !CPLX)) && S_ == YREG)
        ysolve_chunk_regs<V, W, YREG>(col, piv, plen, a, lane, wc, s, o, ny, sC[c], sD[c], colsum);
    else {
        // forward elimination: u_j = f_j beta_j - a beta_j u_{j-1}
        V C = yt_zero(V());
        double D = 1.0;
#pragma unroll 8
        for (int t = 0; t < n; ++t) {
            const double bt = __ldg(piv + min(s + t, plen - 1));
            C = yt_axpy(yt_scale(col[o + t], bt), -a * bt, C);
            D = -a * bt * D;
        }
        V uu = ysolve_scan<V, W, true>(C, D, lane, wc, sC[c], sD[c]);
#pragma unroll 8
        for (int t = 0; t < n; ++t) {
            const double bt = __ldg(piv + min(s + t, plen - 1));
            uu = yt_axpy(yt_scale(col[o + t], bt), -a * bt, uu);
            col[o + t] = uu;
        }
        // back substitution: u_j = u'_j - a beta_j u_{j+1}
        C = yt_zero(V());
        D = 1.0;
#pragma unroll 8
        for (int t = n - 1; t >= 0; --t) {
            const double ej = (s + t == ny - 1) ? 0.0 : -a * __ldg(piv + min(s + t, plen - 1));
            C = yt_axpy(col[o + t], ej, C);
            D = ej * D;
        }
        uu = ysolve_scan<V, W, false>(C, D, lane, wc, sC[c] + W, sD[c] + W);
#pragma unroll 8
        for (int t = n - 1; t >= 0; --t) {
            const double ej = (s + t == ny - 1) ? 0.0 : -a * __ldg(piv + min(s + t, plen - 1));
            uu = yt_axpy(col[o + t], ej, uu);
            col[o + t] = uu;
            if constexpr (std::is_same<V, double>::value) colsum.add(yt_re(uu));
        }
    }
    // dst_w-weighted column sum (box), one compensated partial per warp
    CSum wsum;
    if (!CPLX) {
        const CSum cw = csum_warp(colsum);
        if (live) {
            const double wk = b.dst_w[k];
            wsum.add_prod(wk, cw.s);
            wsum.add_prod(wk, cw.c);
        }
    }
    __syncthreads();
    for (int i0 = threadIdx.x; i0 < ny * KB; i0 += NT * CH) {
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int idx = i0 + NT * u;
            const int jj = idx >> 2, cc = idx & 3, kk = k0 + cc;
            if (idx < ny * KB && kk < nk) {
                if constexpr (CPLX) S[(size_t)jj * pk + kk] = yt_store2<Gm>(tile[cc * LD + jj + fdS.div(jj)]);
                else S[(size_t)jj * pk + kk] = yt_store<Gm>(tile[cc * LD + jj + fdS.div(jj)]);
            }
        }
    }
    if (!CPLX) {
        // the CTA's partial (sum, compensation), its warps merged in a fixed
        // order
        __shared__ double wpart[2 * KB * W];
        if (lane == 0) { wpart[wid] = wsum.s; wpart[KB * W + wid] = wsum.c; }
        __syncthreads();
        if (threadIdx.x == 0) {
            CSum t;
#pragma unroll
            for (int x = 0; x < KB * W; ++x) t.merge(wpart[x], wpart[KB * W + x]);
            b.part_col[2 * w.block] = t.s;
            b.part_col[2 * w.block + 1] = t.c;
        }
    }
}

// LU solve with the pivots of DGETRF (column-major n x n) -- DGETRS 'N'.
template <int N>
__device__ __forceinline__ void lu_solve_dev(const double (&lu)[N * N], const int (&piv)[N], double (&x)[N]) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
        // row interchange i <-> piv[i]
#pragma unroll
        for (int r = 0; r < N; ++r)
            if (r > i && piv[i] == r) { double t = x[i]; x[i] = x[r]; x[r] = t; }
    }
#pragma unroll
    for (int c = 0; c < N; ++c)
#pragma unroll
        for (int r = c + 1; r < N; ++r) x[r] -= x[c] * lu[r + N * c];
#pragma unroll
    for (int c = N - 1; c >= 0; --c) {
        x[c] /= lu[c + N * c];
#pragma unroll
        for (int r = 0; r < c; ++r) x[r] -= x[c] * lu[r + N * c];
    }
}

// solve_Ax_b (util/linalg.F90:57-93): DGETRS then the DGERFS refinement loop
// (at most 5 refinements), in registers.
template <int N>
__device__ __forceinline__ void solve_ax_b_dev(const double (&A)[N * N], const double (&lu)[N * N],
                                               const int (&piv)[N], const double (&rhs)[N], double (&x)[N]) {
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] = rhs[i];
    lu_solve_dev<N>(lu, piv, x);
    const double eps = 1.1102230246251565e-16;
    const double safe1 = (N + 1) * 2.2250738585072014e-308, safe2 = safe1 / eps;
    double lstres = 3.0;
#pragma unroll 1
    for (int count = 1; count <= 6; ++count) {
        double r[N], wv[N];
#pragma unroll
        for (int i = 0; i < N; ++i) { r[i] = rhs[i]; wv[i] = fabs(rhs[i]); }
#pragma unroll
        for (int j = 0; j < N; ++j) {
            const double t = -x[j], xk = fabs(x[j]);
#pragma unroll
            for (int i = 0; i < N; ++i) {
                r[i] += t * A[i + N * j];
                wv[i] += fabs(A[i + N * j]) * xk;
            }
        }
        double sm = 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const double q = (wv[i] > safe2) ? fabs(r[i]) / wv[i] : (fabs(r[i]) + safe1) / (wv[i] + safe1);
            sm = fmax(sm, q);
        }
        if (!(sm > eps && 2.0 * sm <= lstres && count <= 5)) break;
        lu_solve_dev<N>(lu, piv, r);
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] += r[i];
        lstres = sm;
    }
}

// Per-step scalars the assembly needs: the homogeneous-correction
// coefficients and the suppress_comp_mode flag of this step.
struct XinvScal {
    double alpha[OQG_NLMAX];                             // box
    double c_bt, c_bc1[OQG_NLMAX], c_bc2[OQG_NLMAX];     // channel
    double S[OQG_NLMAX][OQG_NQ];                         // channel strip sums (scratch)
    int supp;
};

// The scalar phase of one step, run by one warp of every assembly CTA from
// the current state st[par] (all CTAs compute the same values); CTA 0 also
// writes the next state st[1-par].
//   update_mass_constr (constraint.F90:167-179);
//   box_homog's area integrals and 2x2 solve (homog.F90:331-366), from the
//     dst_w-weighted spectral column sums of the y-solve (the inverse DST is
//     linear, so the area integral of the modal solution is known before it);
//   or, for a channel, the strip integrals of the vorticity kernel,
//     step_constraints (constraint.F90:182-215) and cyclic_homog
//     (homog.F90:280-329);
//   the suppress_comp_mode schedule and its scalar part (openqg.F90:485-487,
//     driver.F90:183-188).
template <class T, int NL>
__device__ __noinline__ void scalar_phase(const BasinDev &b, double tdt, int par, bool writer,
                                          XinvScal *out) {
    const int lane = threadIdx.x & 31;
    const DevState *st = b.st + par;
    const DevForcing *fr = b.frc;
    double imode[NL];
    double (*S)[OQG_NQ] = out->S;
    if (!b.cyclic) {
        const int nkb = (b.nk + 3) / 4;       // y-solve CTAs per mode (4 columns each)
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            CSum s;
#pragma unroll 4
            for (int x = lane; x < nkb; x += 32) s.merge(b.part_col[2 * (m * nkb + x)], b.part_col[2 * (m * nkb + x) + 1]);
            s = csum_warp(s, true);
            imode[m] = s.value() * b.ftnorm * b.dx * b.dy;
        }
    } else {
        // strip sums over the tiles touching rows 0, 1, nyp-2, nyp-1: per
        // layer the OQG_NQ sums together, so their loads and shuffles overlap
        // (the additions keep warp_sum's order)
        const int ntile = b.tiles_x * b.tiles_y;
#pragma unroll 1
        for (int k = 0; k < NL; ++k) {
            double acc[OQG_NQ];
#pragma unroll
            for (int q = 0; q < OQG_NQ; ++q) acc[q] = 0.0;
            for (int t = lane; t < ntile; t += 32) {
                const int ty0 = (t / b.tiles_x) * b.vty;
                if (ty0 <= 1 || ty0 + b.vty > b.nyp - 2) {
                    const double *pt = b.part_tile + ((size_t)t * NL + k) * OQG_NQ;
#pragma unroll
                    for (int q = 0; q < OQG_NQ; ++q) acc[q] += pt[q];
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int q = 0; q < OQG_NQ; ++q) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
            if (lane == 0)
#pragma unroll
                for (int q = 0; q < OQG_NQ; ++q) S[k][q] = acc[q];
        }
        __syncwarp();
    }
    if (lane != 0) return;
    DevState ns;                                          // the next state
    const long long nt = st->nt;
    const double ent_xn = fr->ent_xn;
    // update_mass_constr (constraint.F90:167-179)
#pragma unroll
    for (int l = 0; l < NL - 1; ++l) {
        ns.dpi[l] = st->dpip[l] - tdt * b.gp[l] * (l == 0 ? ent_xn : 0.0);
        ns.dpip[l] = st->dpi[l];
    }
    const int supp = (b.suppress_period > 0 && (nt % b.suppress_period) == 0) ? 1 : 0;
    if (!b.cyclic) {
        // box_homog (homog.F90:331-366)
        double ik[NL];
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            double s = 0.0;
#pragma unroll
            for (int m = 0; m < NL; ++m) s += b.ctm2l[m + NL * k] * imode[m];
            ik[k] = s;
        }
        constexpr int N = (NL > 1) ? NL - 1 : 1;
        double A[N * N], LU[N * N], rhs[N], al[N];
        int pv[N];
#pragma unroll
        for (int x = 0; x < N * N; ++x) { A[x] = b.cdhoc[x]; LU[x] = b.lu[x]; }
#pragma unroll
        for (int x = 0; x < N; ++x) { pv[x] = b.piv[x]; rhs[x] = ns.dpi[x] - (ik[x + 1] - ik[x]); }
        solve_ax_b_dev<N>(A, LU, pv, rhs, al);
#pragma unroll
        for (int l = 0; l < N; ++l) out->alpha[l] = al[l];
    } else {
        double cs[NL], cn[NL], csp[NL], cnp[NL];
#pragma unroll
        for (int k = 0; k < NL; ++k) { cs[k] = st->cs[k]; cn[k] = st->cn[k]; csp[k] = st->csp[k]; cnp[k] = st->cnp[k]; }
        const double dx = b.dx, dy = b.dy;
        double rhss[NL], rhsn[NL];
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            rhss[k] = -0.5 * dy * b.fnot * fr->int_Be_s[k];
            rhsn[k] = -0.5 * dy * b.fnot * fr->int_Be_n[k];
        }
        // step_constraints (constraint.F90:182-215)
        rhss[0] = rhss[0] + b.tau_sign * (b.fnot / b.h[0]) * fr->txis;
        rhsn[0] = rhsn[0] - b.tau_sign * (b.fnot / b.h[0]) * fr->txin;
        const double dfac = b.fnot * b.delek / (2.0 * fabs(b.fnot));
        double bs = 0.0, bn = 0.0;
#pragma unroll
        for (int k = 0; k < NL; ++k)
            if (k == b.kt) { bs = S[k][8]; bn = S[k][9]; }
        const double bdrins = dfac * ((bs * dx) / dy), bdrinn = dfac * ((bn * dx) / dy);
        rhss[NL - 1] = rhss[NL - 1] + (b.fnot / b.h[NL - 1]) * bdrins;
        rhsn[NL - 1] = rhsn[NL - 1] - (b.fnot / b.h[NL - 1]) * bdrinn;
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            const double a5s = (S[k][0] * dx) / (2.0 * dx), a9s = (S[k][1] * dx) / (2.0 * dx);
            const double a5n = (S[k][2] * dx) / (2.0 * dx), a9n = (S[k][3] * dx) / (2.0 * dx);
            const double ajis = (a5s + 2.0 * a9s) / 6.0, ajin = -(a5n + 2.0 * a9n) / 6.0;
            const double ap3s = b.ah2[k] * (S[k][4] * dx) / dy, ap3n = b.ah2[k] * (S[k][5] * dx) / dy;
            const double ap5s = b.ah4[k] * (S[k][6] * dx) / dy, ap5n = b.ah4[k] * (S[k][7] * dx) / dy;
            rhss[k] = rhss[k] + ajis - ap3s + ap5s;
            rhsn[k] = rhsn[k] + ajin + ap3n - ap5n;
        }
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            const double csn = csp[k] + tdt * rhss[k];
            const double cnn = cnp[k] + tdt * rhsn[k];
            csp[k] = cs[k];
            cnp[k] = cn[k];
            cs[k] = csn;
            cn[k] = cnn;
        }
        // cyclic_homog (homog.F90:280-329).  The x-integral of row j of the
        // modal solution is dx times its zero wavenumber (before the 1/N of the
        // inverse transform, which the N-term row sum cancels).
        typedef typename C2<T>::t T2;
        const T2 *Sp = (const T2 *)b.spec;
        double clhss[NL], clhsn[NL];
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            double ss = 0.0, sn = 0.0;
#pragma unroll
            for (int k = 0; k < NL; ++k) {
                ss += b.ctl2m[k + NL * m] * cs[k];
                sn += b.ctl2m[k + NL * m] * cn[k];
            }
            const double u0s = (double)Sp[((size_t)m * b.ny) * b.pk].x;
            const double u0n = (double)Sp[((size_t)m * b.ny + (b.ny - 1)) * b.pk].x;
            clhss[m] = ss + (u0s * dx) / dy;
            clhsn[m] = sn + (u0n * dx) / dy;
        }
        out->c_bt = clhss[0] * b.hbsi;
#pragma unroll
        for (int m = 1; m < NL; ++m) {
            out->c_bc1[m] = b.hc2n[m] * clhss[m] - b.hc2s[m] * clhsn[m];
            out->c_bc2[m] = b.hc1s[m] * clhsn[m] - b.hc1n[m] * clhss[m];
        }
        // suppress_comp_mode's channel scalars (driver.F90:185-188)
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            if (supp) { cs[k] = 0.5 * (cs[k] + csp[k]); cn[k] = 0.5 * (cn[k] + cnp[k]); }
            ns.cs[k] = cs[k]; ns.cn[k] = cn[k]; ns.csp[k] = csp[k]; ns.cnp[k] = cnp[k];
        }
    }
    out->supp = supp;
    if (!writer) return;
    DevState *nx = b.st + (1 - par);
#pragma unroll
    for (int l = 0; l < NL - 1; ++l) {
        nx->dpi[l] = supp ? 0.5 * (ns.dpi[l] + ns.dpip[l]) : ns.dpi[l];
        nx->dpip[l] = ns.dpip[l];
    }
    if (b.cyclic) {
#pragma unroll
        for (int k = 0; k < NL; ++k) { nx->cs[k] = ns.cs[k]; nx->cn[k] = ns.cn[k]; nx->csp[k] = ns.csp[k]; nx->cnp[k] = ns.cnp[k]; }
    }
    nx->nt = nt + 1;
}

// ------------------------------------------------------------------ k_xinv_rows
// The inverse x-transforms of the y-solved spectral rows as a launch of
// their own, shaped like k_xfwd (one row pair per group, the 2048- and
// 4096-point box lengths in place), into the modal rows b.inh_g, which
// k_xinv_asm assembles.  A box's inverse DST-I is the forward transform
// scaled by ftnorm (inhomog.F90:200-211): the modal row j + 1 of mode m gets
// the n interior values and zeros on both walls.  A channel's c2r
// (inhomog.F90:214-255) fills every column, the last repeating the first.
// The first and last row
// pairs of a mode clear the wall rows 0 and nyp - 1 (into out instead of
// inh_g when out != null: the solve-only mode).  A scalar CTA after the
// transforms' runs a basin's scalar phase once into b.scal_g (the assembly
// reads it there) and writes the basin's next scalar state.
// G: transforms per CTA (the forward launch's; <= 0: blockDim / TT, per
// member of an ensemble), blockDim >= G TT rounded up to whole warps so the
// scalar CTAs have a full warp.  scal: the last scal CTAs run the scalar
// phase of member 0, 1, ... (0: none).
template <class T, int NL, int E, int MC = 0>
__global__ void __launch_bounds__(256, 2)
k_xinv_rows(const BasinDev *__restrict__ bas, const Work *__restrict__ work, int G, int scal, int par,
            double tdt, T *out) {
    typedef typename C2<T>::t T2;
    if (scal > 0 && (int)blockIdx.x >= (int)gridDim.x - scal) {
        pdl_trigger();
        pdl_wait();
        if (threadIdx.x < 32) {
            const BasinDev &b = bas[blockIdx.x - (gridDim.x - scal)];
            scalar_phase<T, NL>(b, tdt != 0.0 ? tdt : b.tdt_m, par, true, (XinvScal *)b.scal_g);
        }
        return;
    }
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = MC > 0 ? MC : b.M, TT = (M + E - 1) / E;
    if (G <= 0) G = blockDim.x / TT;            // an ensemble: per member, as k_xfwd
    const int g = threadIdx.x / TT, t = threadIdx.x - g * TT;
    const int LB = fft_buf_len(M);
    T2 *zs = reinterpret_cast<T2 *>(smem_raw);
    const int npm = (b.ny + 1) >> 1;          // row pairs per mode
    const int pair = w.block * G + g;
    const bool live = g < G && pair < b.nl * npm;
    const int m = live ? pair / npm : 0;
    const int j = live ? 2 * (pair - m * npm) : 0;
    const bool two = live && (j + 1 < b.ny);
    const int n = b.nxin, nxp = b.nxp, px = b.px;
    // a spectral row: n reals (box) or nk complex values (channel); a channel
    // transforms through the ping-pong pair, whose second buffer holds both
    const bool cyc = b.cyclic != 0;
    const int rowbytes = cyc ? b.nk * (int)sizeof(T2) : n * (int)sizeof(T);
    const int RO = round16(rowbytes) / (int)sizeof(T);   // offset of the second row (16-byte aligned)
    const bool ip = E == 16 && !cyc && fft_inplace_len(M);
    T2 *za = zs + (size_t)(g < G ? g : 0) * (ip ? LB : 2 * LB);
    T2 *zb = za + LB;
    T *raw = ip ? reinterpret_cast<T *>(zs + (size_t)G * LB) + (size_t)(g < G ? g : 0) * 2 * RO
                : reinterpret_cast<T *>(zb);
    const size_t pitchb = (size_t)b.pk * (cyc ? sizeof(T2) : sizeof(T));
    const char *x = (const char *)b.spec + ((size_t)m * b.ny + j) * pitchb;
    // out != null: solve-only mode, the modal solutions go straight to out
    // ([nl][nyp][px], the same layout)
    T *inh = out ? out : (T *)b.inh_g;
    const T ftn = (T)b.ftnorm;
    pdl_trigger();
    pdl_wait();
    if (live) {
        cp_async_16(raw, x, round16(rowbytes), t, TT);
        if (two) cp_async_16(raw + RO, x + pitchb, round16(rowbytes), t, TT);
    }
    cp_async_commit_wait_all();
    __syncthreads();
    if (live && cyc) {
        // c2r by one complex transform of two rows: the Hermitian extension
        // of X + iY, conjugated (inhomog.F90:214-255)
        const T2 *xr = reinterpret_cast<const T2 *>(raw), *yr = reinterpret_cast<const T2 *>(raw + RO);
        for (int kk = t; kk < M; kk += TT) {
            T2 X, Y;
            const bool lo = kk <= M / 2;
            const int ks = lo ? kk : M - kk;
            X = xr[ks];
            if (two) Y = yr[ks]; else { Y.x = (T)0; Y.y = (T)0; }
            if (!lo) { X.y = -X.y; Y.y = -Y.y; }
            if (kk == 0 || 2 * kk == M) { X.y = (T)0; Y.y = (T)0; }
            T2 v;
            v.x = ftn * X.x - ftn * Y.y;
            v.y = -(ftn * X.y + ftn * Y.x);
            za[fpad(kk)] = v;
        }
    } else if (live) {
        if (t == 0) {
            T2 zero;
            zero.x = (T)0;
            zero.y = (T)0;
            za[fpad(0)] = zero;
            za[fpad(n + 1)] = zero;
        }
        for (int jj = 1 + t; jj <= n; jj += TT) {
            T2 v, vm;
            v.x = ftn * raw[jj - 1];
            v.y = two ? ftn * raw[RO + jj - 1] : (T)0;
            vm.x = -v.x;
            vm.y = -v.y;
            za[fpad(jj)] = v;
            za[fpad(M - jj)] = vm;
        }
    }
    __syncthreads();
    T2 *z = za;
    if (ip) fft_inplace<T, MC>(za, M, (const T2 *)b.tw, live ? t : M, 0, 0);
    else z = fft_run<T, E, MC>(za, zb, M, b.rad, b.nrad, (const T2 *)b.tw, live ? t : TT, TT, 0, 0);
    if (!live) return;
    T *ox = inh + ((size_t)m * b.nyp + j + 1) * px;
    T *oy = ox + px;
    if (cyc) {
        // every column; column nxp-1 = M repeats column 0 (inhomog.F90:250)
        for (int i = t; i < M; i += TT) {
            const T2 v = z[fpad(i)];
            ox[i] = v.x;
            if (two) oy[i] = -v.y;
        }
        if (t == 0) {
            const T2 v = z[fpad(0)];
            ox[M] = v.x;
            if (two) oy[M] = -v.y;
        }
    } else {
        for (int kk = t; kk < n; kk += TT) {
            const T2 v = z[fpad(kk + 1)];
            ox[kk + 1] = -v.y;
            if (two) oy[kk + 1] = v.x;
        }
    }
    if (t == 0 && !cyc) {
        ox[0] = (T)0;
        ox[nxp - 1] = (T)0;
        if (two) { oy[0] = (T)0; oy[nxp - 1] = (T)0; }
    }
    // the wall rows (zonal walls of either geometry)
    T *wrow = nullptr;
    if (j == 0) wrow = inh + (size_t)m * b.nyp * px;
    if (j + 2 >= b.ny) {
        T *last = inh + ((size_t)m * b.nyp + b.nyp - 1) * px;
        for (int i = t; i < nxp; i += TT) last[i] = (T)0;
    }
    if (wrow)
        for (int i = t; i < nxp; i += TT) wrow[i] = (T)0;
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

// The last warp of the CTA runs the scalar phase of the step while the
// other nfft = blockDim.x - 32 threads run the inverse transforms; those
// synchronise among themselves on named barrier 1.
// out != null: solve-only mode, writes the modal inhomogeneous solutions
// (FP64, [nl][nyp][px]) and nothing else (no scalar phase).
// tdt = 0: each member steps with its own b.tdt_m (ensemble launches).
template <class T, int NL>
__global__ void __maxnreg__(112)
k_xinv(const BasinDev *__restrict__ bas, const Work *__restrict__ work, int par, double tdt, double *out) {
    typedef typename C2<T>::t T2;
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    const int nfft = blockDim.x - 32;
    const bool fft_thread = (int)threadIdx.x < nfft;
    const int M = b.M, TT = (M + XINV_E - 1) / XINV_E, G = nfft / TT;
    const int g = threadIdx.x / TT, t = threadIdx.x - g * TT;
    int jlo, jhi, jfirst, nra;
    xinv_rows(b, w.block, jlo, jhi, jfirst, nra);
    const int nr = jhi - jlo;                    // interior rows
    const int nxp = b.nxp, n = b.nxin, nyp = b.nyp, px = b.px;
    const int LB = fft_buf_len(M);
    const int npr = (nr + 1) >> 1;               // row pairs per mode
    const int npairs = NL * npr;
    const bool one_round = G >= npairs;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ XinvScal sS;
    // Two sets of G transform buffers; each transform starts in the set that
    // makes its last stage end in set A, and its spectral rows are staged in
    // the other.  With every row pair in one round the modal rows inh alias
    // set B once the transforms are done; otherwise they follow both sets.
    // Grids too wide for the modal rows in shared memory keep them in the
    // global buffer b.inh_g ([nl][nyp][px], rows of this CTA only).
    T2 *setA = reinterpret_cast<T2 *>(smem_raw), *setB = setA + (size_t)G * LB;
    T2 *set_in = (b.nrad & 1) ? setB : setA, *set_st = (b.nrad & 1) ? setA : setB;
    const bool split = b.xinv_split != 0;
    const bool alias = one_round && !split;
    // a row of the spectral buffer: n reals (box) or nk complex (channel)
    const int rowbytes = b.cyclic ? b.nk * (int)sizeof(T2) : n * (int)sizeof(T);
    const int RO = round16(rowbytes) / (int)sizeof(T);   // second row offset (T units)
    T *inh;
    size_t ms, rs;                               // mode and row strides of inh
    if (split) { inh = (T *)b.inh_g + (size_t)jfirst * px; ms = (size_t)nyp * px; rs = px; }
    else {
        inh = alias ? reinterpret_cast<T *>(setB) : reinterpret_cast<T *>(setA + (size_t)2 * G * LB);
        ms = (size_t)nra * nxp;
        rs = nxp;
    }
    const T ftn = (T)b.ftnorm;

    pdl_trigger();
    if (!fft_thread) {
        pdl_wait();
        if (!out) scalar_phase<T, NL>(b, tdt != 0.0 ? tdt : b.tdt_m, par, w.block == 0, &sS);
    } else if (split && b.xinv_sep) {
        // (solve-only mode) the modal rows come from k_xinv_rows
        pdl_wait();
    } else {
    // zero the wall rows / columns of the modal fields
    if (!alias)
        for (int m = 0; m < NL; ++m)
            for (int lr = 0; lr < nra; ++lr)
                for (int i = threadIdx.x; i < nxp; i += nfft) inh[m * ms + lr * rs + i] = (T)0;
    pdl_wait();

    for (int base = 0; base < npairs; base += G) {
        const int pair = base + g;
        const bool live = g < G && pair < npairs;
        const int m = live ? pair / npr : 0;
        const int r0 = live ? 2 * (pair - m * npr) : 0;     // interior row offset
        const bool two = live && r0 + 1 < nr;
        T2 *za = set_in + (size_t)(g < G ? g : 0) * LB;
        T2 *zb = set_st + (size_t)(g < G ? g : 0) * LB;
        T *raw = reinterpret_cast<T *>(zb);
        const int sj = jlo + r0 - 1;                        // spectral row
        const char *srow = (const char *)b.spec + ((size_t)m * b.ny + sj) * b.pk * (b.cyclic ? sizeof(T2) : sizeof(T));
        const size_t pitchb = (size_t)b.pk * (b.cyclic ? sizeof(T2) : sizeof(T));
        if (live) {
            cp_async_16(raw, srow, round16(rowbytes), t, TT);
            if (two) cp_async_16(raw + RO, srow + pitchb, round16(rowbytes), t, TT);
        }
        cp_async_commit_wait_all();
        bar_sync(1, nfft);
        if (live) {
            if (!b.cyclic) {
                const T *x = raw, *y = raw + RO;
                // odd extension: z_0 = z_{n+1} = 0, z_{M-jj} = -z_jj
                if (t == 0) {
                    T2 zero;
                    zero.x = (T)0;
                    zero.y = (T)0;
                    za[fpad(0)] = zero;
                    za[fpad(n + 1)] = zero;
                }
                for (int jj = 1 + t; jj <= n; jj += TT) {
                    T2 v, vm;
                    v.x = ftn * x[jj - 1];
                    v.y = two ? ftn * y[jj - 1] : (T)0;
                    vm.x = -v.x;
                    vm.y = -v.y;
                    za[fpad(jj)] = v;
                    za[fpad(M - jj)] = vm;
                }
            } else {
                const T2 *x = reinterpret_cast<const T2 *>(raw), *y = reinterpret_cast<const T2 *>(raw + RO);
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
                    za[fpad(kk)] = v;
                }
            }
        }
        bar_sync(1, nfft);
        T2 *z = fft_run<T, XINV_E>(za, zb, M, b.rad, b.nrad, (const T2 *)b.tw, live ? t : TT, TT, 1, nfft);
        if (alias) {
            // set B is free now: clear it for the modal rows
            for (int idx = threadIdx.x; idx < NL * nra * nxp; idx += nfft) inh[idx] = (T)0;
            bar_sync(1, nfft);
        }
        if (live) {
            const int lr = (jlo + r0) - jfirst;
            T *ox = inh + m * ms + lr * rs;
            T *oy = ox + rs;
            if (!b.cyclic) {
                for (int kk = t; kk < n; kk += TT) {
                    const T2 v = z[fpad(kk + 1)];
                    ox[kk + 1] = -v.y;
                    if (two) oy[kk + 1] = v.x;
                }
            } else {
                for (int i = t; i < M; i += TT) {
                    const T2 v = z[fpad(i)];
                    ox[i] = v.x;
                    if (two) oy[i] = -v.y;
                }
                if (t == 0) {
                    const T2 v = z[fpad(0)];
                    ox[M] = v.x;
                    if (two) oy[M] = -v.y;
                }
            }
        }
        bar_sync(1, nfft);
    }
    }   // fft threads
    __syncthreads();

    if (out) {
        for (int idx = threadIdx.x; idx < NL * nra * nxp; idx += blockDim.x) {
            const int m = idx / (nra * nxp), rem = idx - m * nra * nxp;
            const int lr = rem / nxp, i = rem - lr * nxp;
            out[((size_t)m * nyp + jfirst + lr) * px + i] = (double)inh[m * ms + lr * rs + i];
        }
        return;
    }

    // homogeneous correction + modes_to_layers, in place (modes -> layers)
    const XinvScal *sc = &sS;
    const int supp = sc->supp;
    double ctm[NL * NL], hc[NL > 1 ? NL - 1 : 1];
#pragma unroll
    for (int x = 0; x < NL * NL; ++x) ctm[x] = b.ctm2l[x];
    const T *__restrict__ Pold = (const T *)b.F[par];
    T *__restrict__ Pnew = (T *)b.F[1 - par];
    const size_t n2 = (size_t)nyp * px;
    if (!b.cyclic) {
#pragma unroll
        for (int m = 1; m < NL; ++m) hc[m - 1] = sc->alpha[m - 1];
    }
    const T *__restrict__ H = (const T *)b.hsb;
    const FastDiv fdx(nxp);
    constexpr int U = 4;
    for (int base = threadIdx.x; base < nra * nxp; base += U * blockDim.x) {
        // gather the inputs of U points first (independent loads), then compute
        double hv[U][NL], po[U][NL];
        int lrs[U], is[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * blockDim.x;
            const bool ok = idx < nra * nxp;
            const int lr = ok ? fdx.div(idx) : 0, i = ok ? idx - lr * nxp : 0;
            const int j = jfirst + lr;
            lrs[u] = ok ? lr : -1;
            is[u] = i;
#pragma unroll
            for (int m = 0; m < NL; ++m) {
                po[u][m] = (ok && supp) ? (double)Pold[m * n2 + (size_t)j * px + i] : 0.0;
                if (!b.cyclic) hv[u][m] = (ok && m >= 1) ? (double)H[((size_t)(m - 1) * nyp + j) * px + i] : 0.0;
                else if (m == 0) hv[u][m] = ok ? b.hbt[j] : 0.0;
                else hv[u][m] = ok ? b.hbc1[m * nyp + j] : 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (lrs[u] < 0) continue;
            const int lr = lrs[u], i = is[u], j = jfirst + lr;
            double pm_[NL];
#pragma unroll
            for (int m = 0; m < NL; ++m) pm_[m] = (double)inh[m * ms + lr * rs + i];
            if (!b.cyclic) {
#pragma unroll
                for (int m = 1; m < NL; ++m) pm_[m] = pm_[m] + hc[m - 1] * hv[u][m];
            } else {
                pm_[0] = pm_[0] + sc->c_bt * hv[u][0];
#pragma unroll
                for (int m = 1; m < NL; ++m)
                    pm_[m] = pm_[m] + (sc->c_bc1[m] * hv[u][m] + sc->c_bc2[m] * b.hbc2[m * nyp + j]);
            }
#pragma unroll
            for (int k = 0; k < NL; ++k) {
                double s2 = 0.0;
#pragma unroll
                for (int m = 0; m < NL; ++m) s2 += pm_[m] * ctm[m + NL * k];
                const T pn = (T)s2;
                // ocqbdy reads the layer values on and next to the walls
                // (in shared memory they go back everywhere)
                if (!split || i <= 1 || i >= nxp - 2 || j <= 1 || j >= nyp - 2) inh[k * ms + lr * rs + i] = pn;
                Pnew[k * n2 + (size_t)j * px + i] = supp ? (T)((T)0.5 * (pn + (T)po[u][k])) : pn;
            }
        }
    }
    __syncthreads();

    // ocqbdy (vorsubs.F90:58-114) on the walls of these rows, then the
    // suppress_comp_mode average of q (driver.F90:180)
    T *Qc = (T *)b.F[3 - par];        // q after this step (qm buffer of K1)
    const T *Qm = (const T *)b.F[2 + par];
    const T fac = (T)b.qb_fac;
    // the point (lr, i) of these rows: q's average on a suppression step,
    // ocqbdy's value on a wall
    auto wall_point = [&](int lr, int i) {
        const int j = jfirst + lr;
        const bool zon = (j == 0 || j == nyp - 1);
        const bool mer = !b.cyclic && (i == 0 || i == nxp - 1);
        if (!zon && !mer) {
            if (supp)
                for (int k = 0; k < NL; ++k) {
                    const size_t o3 = ((size_t)k * nyp + j) * px + i;
                    Qc[o3] = (T)0.5 * (Qc[o3] + Qm[o3]);
                }
            return;
        }
        const int cnt = (zon ? 1 : 0) + (mer ? 1 : 0);
#define PN(kk, rr, ii) inh[(kk) * ms + (rr) * rs + (ii)]
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
            // (FP32 storage holds q - beta y: one beta y fewer)
            for (int c = q_anom_stored<T>() ? 1 : 0; c < cnt; ++c) qv = qv + by;
            if (k == b.kt && b.topo_active) {
                const T dd = (T)b.ddyn[(size_t)j * px + i];
                for (int c = 0; c < cnt; ++c) qv = qv + dd;
            }
            const size_t o3 = ((size_t)k * nyp + j) * px + i;
            Qc[o3] = supp ? (T)((T)0.5 * (qv + Qm[o3])) : qv;
        }
#undef PN
    };
    // every point on a suppression step and along the zonal walls; else the
    // two meridional wall points of each row
    for (int lr = 0; lr < nra; ++lr) {
        const int j = jfirst + lr;
        if (supp || j == 0 || j == nyp - 1) {
            for (int i = threadIdx.x; i < nxp; i += blockDim.x) wall_point(lr, i);
        } else if (!b.cyclic && threadIdx.x < 2) {
            wall_point(lr, threadIdx.x == 0 ? 0 : nxp - 1);
        }
    }
}

// ------------------------------------------------------------------ k_xinv_asm
#define XASM_ENS_POINTS 1024   // points per assembly work item of an ensemble's member
// The assembly of a basin whose inverse transforms ran as k_xinv_rows: the
// homogeneous correction and modes_to_layers (modes.F90:268-284) of every
// point from the modal rows in b.inh_g, ocqbdy (vorsubs.F90:58-114) on the
// walls and the suppress_comp_mode averages (driver.F90:174-189), with the
// step's scalars from b.scal_g.  The work items of a basin (the work list
// spans an ensemble's members) take interleaved runs of 256 points, one
// point per thread in each; a wall point also
// forms the layer values of its inner neighbour (the same arithmetic as the
// neighbour's own thread), so no point waits for another.
// hc: the box's alpha (nl-1), or the channel's c_bt, c_bc1[1..], c_bc2[1..]
// (homog.F90:280-366, by k_xinv_rows' scalar CTA).
template <class T, int NL>
__device__ __forceinline__ void xinv_layers(const BasinDev &b, const T *__restrict__ inh, const T *__restrict__ H,
                                            const double *ctm, const double *hc, size_t o2, int j, T *pn) {
    const size_t ms = (size_t)b.nyp * b.px;
    double pm_[NL];
#pragma unroll
    for (int m = 0; m < NL; ++m) pm_[m] = (double)inh[m * ms + o2];
    if (!b.cyclic) {
#pragma unroll
        for (int m = 1; m < NL; ++m) pm_[m] = pm_[m] + hc[m - 1] * (double)H[(m - 1) * ms + o2];
    } else {
        const int nyp = b.nyp;
        pm_[0] = pm_[0] + hc[0] * b.hbt[j];
#pragma unroll
        for (int m = 1; m < NL; ++m)
            pm_[m] = pm_[m] + (hc[m] * b.hbc1[m * nyp + j] + hc[NL + m] * b.hbc2[m * nyp + j]);
    }
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        double s2 = 0.0;
#pragma unroll
        for (int m = 0; m < NL; ++m) s2 += pm_[m] * ctm[m + NL * k];
        pn[k] = (T)s2;
    }
}

template <class T, int NL>
__global__ void __launch_bounds__(256)
k_xinv_asm(const BasinDev *__restrict__ bas, const Work *__restrict__ work, int par) {
    const Work w = work[blockIdx.x];
    const BasinDev &b = bas[w.member];
    __shared__ double sCtm[NL * NL], sAmat[NL * NL], sHc[2 * NL];
    __shared__ int sSupp;
    pdl_trigger();
    // the basin's constant tables before the wait for the previous launch
    if (threadIdx.x < NL * NL) {
        sCtm[threadIdx.x] = b.ctm2l[threadIdx.x];
        sAmat[threadIdx.x] = b.amat[threadIdx.x];
    }
    pdl_wait();
    const XinvScal *sc = (const XinvScal *)b.scal_g;
    if (!b.cyclic) {
        if (threadIdx.x < NL - 1) sHc[threadIdx.x] = sc->alpha[threadIdx.x];
    } else if (threadIdx.x < 2 * NL) {
        // c_bt, c_bc1[1..NL), then c_bc2 at NL + m
        const int x = threadIdx.x;
        sHc[x] = x == 0 ? sc->c_bt : (x < NL ? sc->c_bc1[x] : (x == NL ? 0.0 : sc->c_bc2[x - NL]));
    }
    if (threadIdx.x == 0) sSupp = sc->supp;
    __syncthreads();
    double ctm[NL * NL], hc[2 * NL];
#pragma unroll
    for (int x = 0; x < NL * NL; ++x) ctm[x] = sCtm[x];
#pragma unroll
    for (int m = 0; m < 2 * NL; ++m) hc[m] = sHc[m];
    const bool supp = sSupp != 0;
    const int nxp = b.nxp, nyp = b.nyp, px = b.px;
    const size_t ms = (size_t)nyp * px;
    const T *__restrict__ inh = (const T *)b.inh_g;
    const T *__restrict__ H = (const T *)b.hsb;
    const T *__restrict__ Pold = (const T *)b.F[par];
    T *__restrict__ Pnew = (T *)b.F[1 - par];
    T *__restrict__ Qc = (T *)b.F[3 - par];          // q after this step
    const T *__restrict__ Qm = (const T *)b.F[2 + par];
    const T fac = (T)b.qb_fac;
    const FastDiv fdx(nxp);
    const int npts = nxp * nyp;
    // the basin's b.asm_items work items interleave: item w.block takes the
    // points w.block * 256 + t, then every b.asm_items * 256 further
    const int stride = b.asm_items * 256;
    for (int idx = w.block * 256 + threadIdx.x; idx < npts; idx += stride) {
        const int j = fdx.div(idx), i = idx - j * nxp;
        const size_t o2 = (size_t)j * px + i;
        T pn[NL];
        xinv_layers<T, NL>(b, inh, H, ctm, hc, o2, j, pn);
#pragma unroll
        for (int k = 0; k < NL; ++k)
            Pnew[k * ms + o2] = supp ? (T)((T)0.5 * (pn[k] + Pold[k * ms + o2])) : pn[k];
        const bool zon = (j == 0 || j == nyp - 1);
        const bool mer = !b.cyclic && (i == 0 || i == nxp - 1);
        if (!zon && !mer) {
            if (supp)
#pragma unroll
                for (int k = 0; k < NL; ++k) Qc[k * ms + o2] = (T)0.5 * (Qc[k * ms + o2] + Qm[k * ms + o2]);
            continue;
        }
        // ocqbdy: the inner neighbour across the meridional wall (a corner
        // takes that one), else across the zonal wall
        const int jn = mer ? j : (j == 0 ? 1 : nyp - 2);
        const size_t on = mer ? (size_t)j * px + (i == 0 ? 1 : nxp - 2) : (size_t)jn * px + i;
        T pnb[NL];
        xinv_layers<T, NL>(b, inh, H, ctm, hc, on, jn, pnb);
        const int cnt = (zon ? 1 : 0) + (mer ? 1 : 0);
        const T by = (T)(b.beta * b.yprel[j]);
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            T qv = fac * (pnb[k] - pn[k]);
            double mv = 0.0;
#pragma unroll
            for (int l = 0; l < NL; ++l) mv += sAmat[k + NL * l] * (double)pn[l];
            const T fmv = (T)(b.fnot * mv);
            for (int c = 0; c < cnt; ++c) qv = qv - fmv;
            // (FP32 storage holds q - beta y: one beta y fewer)
            for (int c = q_anom_stored<T>() ? 1 : 0; c < cnt; ++c) qv = qv + by;
            if (k == b.kt && b.topo_active) {
                const T dd = (T)b.ddyn[o2];
                for (int c = 0; c < cnt; ++c) qv = qv + dd;
            }
            Qc[k * ms + o2] = supp ? (T)((T)0.5 * (qv + Qm[k * ms + o2])) : qv;
        }
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
            if (!q_anom_stored<T>()) v += b.beta * b.yprel[j];
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

// q fields [nl][nyp][px] <-> FP64 staging, with the storage's anomaly
// (q_anom_stored) removed on the way out and applied on the way in.
template <class T>
__global__ void k_q_out(const BasinDev *__restrict__ bas, int member, const T *src, double *dst, size_t n) {
    const BasinDev &b = bas[member];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)((i / b.px) % b.nyp);
        dst[i] = (double)src[i] + (q_anom_stored<T>() ? b.beta * b.yprel[j] : 0.0);
    }
}
template <class T>
__global__ void k_q_in(const BasinDev *__restrict__ bas, int member, const double *src, T *dst, size_t n) {
    const BasinDev &b = bas[member];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)((i / b.px) % b.nyp);
        dst[i] = (T)(q_anom_stored<T>() ? src[i] - b.beta * b.yprel[j] : src[i]);
    }
}

// Host-order rows (nxp contiguous FP64 values per row) <-> pitched field rows
// of type T: the unpacking and packing of contiguous host copies.
template <class T>
__global__ void k_rows_in(const double *src, T *dst, int nxp, int px, size_t nrows) {
    const size_t n = nrows * (size_t)nxp;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / (size_t)nxp, c = i - r * nxp;
        dst[r * px + c] = (T)src[i];
    }
}
template <class T>
__global__ void k_rows_out(const T *src, double *dst, int nxp, int px, size_t nrows) {
    const size_t n = nrows * (size_t)nxp;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / (size_t)nxp, c = i - r * nxp;
        dst[i] = (double)src[r * px + c];
    }
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

// int_P_dA (numerics.F90:165-204), compensated; red: >= 64 doubles.
template <class T>
__device__ double area_integral(const BasinDev &b, const T *f, double *red) {
    CSum s;
    for (int idx = threadIdx.x; idx < b.nyp * b.nxp; idx += blockDim.x) {
        int j = idx / b.nxp, i = idx - j * b.nxp;
        s.add(trap_w(b, i, j) * (double)f[(size_t)j * b.px + i]);
    }
    return csum_block(s, red) * b.dx * b.dy;
}
// int_P_dx of row ja of f minus row jb (jb < 0: no subtraction), compensated
template <class T>
__device__ double row_integral(const BasinDev &b, const T *f, int ja, int jb, double *red) {
    CSum s;
    for (int i = threadIdx.x; i < b.nxp; i += blockDim.x) {
        double v = (double)f[(size_t)ja * b.px + i];
        if (jb >= 0) v -= (double)f[(size_t)jb * b.px + i];
        s.add(trap_x(b, i) * v);
    }
    return csum_block(s, red) * b.dx;
}

// int_P_dA of one FP64 field [nyp][px] into out[0] (one CTA): the integral
// the mass constraint uses, exposed for tests of its compensation.
__global__ void k_area_integral(const BasinDev *__restrict__ bas, int member, const double *f, double *out) {
    __shared__ double red[64];
    const double v = area_integral(bas[member], f, red);
    if (threadIdx.x == 0) out[0] = v;
}

// init_mass_constr (constraint.F90:145-165) and, for a channel,
// init_constraint (constraint.F90:80-143).  One CTA.
template <class T, int NL>
__global__ void k_init_constraints(const BasinDev *__restrict__ bas, int member, int par) {
    const BasinDev &b = bas[member];
    __shared__ double red[64];
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
    DevState *sc = b.st + par;
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

// Row sums of the ent area integral (int_P_dA, numerics.F90:165-204): one
// CTA per row j writes sum_i trap_x(i) ent(i, j, 1) to ent_rows[2j] with its
// compensation in ent_rows[2j+1].
template <class T>
__global__ void __launch_bounds__(128) k_ent_rows(const BasinDev *__restrict__ bas, int member) {
    const BasinDev &b = bas[member];
    __shared__ double red[64];
    const T *E = (const T *)b.ent + (size_t)blockIdx.x * b.px;
    CSum s;
    for (int i = threadIdx.x; i < b.nxp; i += blockDim.x) s.add(trap_x(b, i) * (double)E[i]);
    const CSum t = csum_block_pair(s, red);
    if (threadIdx.x == 0) { b.ent_rows[2 * blockIdx.x] = t.s; b.ent_rows[2 * blockIdx.x + 1] = t.c; }
}

// Forcing integrals that depend only on ent: ent_xn = int_P_dA(ent(:,:,1))
// (pressure.F90:52-54) from the row sums of k_ent_rows, in a fixed order,
// and the channel strip integrals int_Be_s/n (vorticity.F90:122-128).  One CTA.
// K CTA sums in one pass: the warps' shuffles of the K values interleave and
// three barriers serve them all.  The result is valid in every thread.
template <int K>
__device__ __forceinline__ void block_sum_n(double (&v)[K]) {
    __shared__ double r[K][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < K; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) r[q][wid] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) v[q] = lane < nw ? r[q][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < K; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < K; ++q) r[q][0] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = r[q][0];
}

template <class T>
__device__ void forcing_integrals_cta(const BasinDev &b, const T *E, double *red) {
    DevForcing *sc = b.frc;
    const size_t n2 = (size_t)b.nyp * b.px;
    // ent_rows' trapezoidal sum, and for a channel the trapezoidal x-sums of
    // ent's rows 0 and nyp-1 in layers 1 and 2 (row_integral), together
    // (compensated: the mass constraint's area integral, numerics.F90:165-204)
    CSum cv[5];
    if (E) {
        for (int j = threadIdx.x; j < b.nyp; j += blockDim.x) {
            const double wj = (j == 0 || j == b.nyp - 1) ? 0.5 : 1.0;   // exact scaling
            cv[0].merge(wj * b.ent_rows[2 * j], wj * b.ent_rows[2 * j + 1]);
        }
        if (b.cyclic) {
            const size_t last = (size_t)(b.nyp - 1) * b.px;
            const bool two = b.nl - 1 >= 2;
            for (int i = threadIdx.x; i < b.nxp; i += blockDim.x) {
                const double t = trap_x(b, i);
                cv[1].add(t * (double)E[i]);
                cv[2].add(t * (double)E[last + i]);
                if (two) {
                    cv[3].add(t * (double)E[n2 + i]);
                    cv[4].add(t * (double)E[n2 + last + i]);
                }
            }
        }
    }
    double v[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) v[q] = csum_block(cv[q], red);
    const double exn = v[0] * b.dx * b.dy;
    const double s1 = v[1] * b.dx, n1 = v[2] * b.dx, s2 = v[3] * b.dx, n2v = v[4] * b.dx;
    if (threadIdx.x != 0) return;
    sc->ent_xn = exn;
    for (int k = 0; k < OQG_NLMAX; ++k) { sc->int_Be_s[k] = 0.0; sc->int_Be_n[k] = 0.0; }
    const double f1 = b.fnot / b.h[0], f2 = b.fnot / b.h[1];
    sc->int_Be_s[0] = b.dz_sign * f1 * s1;
    sc->int_Be_s[1] = b.dz_sign * f1 * s2;
    sc->int_Be_n[0] = -b.dz_sign * f2 * n1;
    sc->int_Be_n[1] = -b.dz_sign * f2 * n2v;
}

// The forcing's integrals (ent_xn; a channel's ent strip integrals) from the
// descriptor's entrainment, one CTA.
template <class T>
__global__ void k_forcing_integrals(const BasinDev *__restrict__ bas, int member) {
    __shared__ double red[64];
    const BasinDev &b = bas[member];
    forcing_integrals_cta<T>(b, (const T *)b.ent, red);
}

// Whether this CTA is the last of its grid to arrive (a ticket counter that
// the last one resets): every CTA's global writes before the call are then
// visible to it.  No CTA waits.
__device__ __forceinline__ bool last_cta(unsigned *ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
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
        DevState *sc = b.st + par;
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

// ------------------------------------------------------------------ valids
// Extremes of p, q (all layers) and wekp for the validity scan (valsubs.F90:
// 46-139), and the count of non-finite values among them: per CTA into
// out[blockIdx.x * 7 + (pmin, pmax, qmin, qmax, wmin, wmax, nonfinite)].
template <class T>
__global__ void __launch_bounds__(256) k_valids(const BasinDev *__restrict__ bas, int member, int par, double *out) {
    const BasinDev &b = bas[member];
    const T *P = (const T *)b.F[par], *Q = (const T *)b.F[2 + par], *W = (const T *)b.wekp;
    const size_t n2 = (size_t)b.nyp * b.px;
    double v[6] = {1e308, -1e308, 1e308, -1e308, 1e308, -1e308};
    double bad = 0.0;
    const size_t tot = (size_t)b.nl * b.nyp * b.nxp;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < tot; idx += (size_t)gridDim.x * blockDim.x) {
        const size_t k = idx / ((size_t)b.nyp * b.nxp), rem = idx - k * b.nyp * b.nxp;
        const size_t j = rem / b.nxp, i = rem - j * b.nxp;
        const size_t o = k * n2 + j * b.px + i;
        const double pv = (double)P[o], qv = (double)Q[o] + (q_anom_stored<T>() ? b.beta * b.yprel[j] : 0.0);
        if (!isfinite(pv)) bad += 1.0; else { v[0] = fmin(v[0], pv); v[1] = fmax(v[1], pv); }
        if (!isfinite(qv)) bad += 1.0; else { v[2] = fmin(v[2], qv); v[3] = fmax(v[3], qv); }
        if (k == 0) {
            const double wv = (double)W[j * b.px + i];
            if (!isfinite(wv)) bad += 1.0; else { v[4] = fmin(v[4], wv); v[5] = fmax(v[5], wv); }
        }
    }
    __shared__ double red[7][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < 6; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, o);
            x = (q & 1) ? fmax(x, y) : fmin(x, y);
        }
        if (lane == 0) red[q][wid] = x;
    }
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, o);
    if (lane == 0) red[6][wid] = bad;
    __syncthreads();
    if (threadIdx.x < 7) {
        const int q = threadIdx.x;
        double x = red[q][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
            x = q == 6 ? x + red[q][w] : ((q & 1) ? fmax(x, red[q][w]) : fmin(x, red[q][w]));
        out[blockIdx.x * 7 + q] = x;
    }
}

// ------------------------------------------------------------------ qg_diagno
// The monitor record of qg_diagno (qg_monitor.F90:219-383) on the device:
// velocity fields, their wall Laplacians, then per-row sums of every
// integrand; the host adds the rows in a fixed order.

// dPdx_2bc / dPdy_2bc (numerics.F90:470-513) of layer field P at (i, j).
template <class T>
__device__ __forceinline__ void dpdxy_bc(const T *P, const BasinDev &b, int i, int j, double &dpx, double &dpy) {
    const int nxp = b.nxp, nyp = b.nyp, px = b.px;
    const double ah = b.bc_half1;
    const double pv = (double)P[(size_t)j * px + i];
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
}

// Lagged (from pm) and current (from p) geostrophic velocities, FP64:
// V[0..3] = ug, vg, uc, vc, each [nl][nyp][px].
template <class T>
__global__ void k_dg_vel(const BasinDev *__restrict__ bas, int member, int par, double *V) {
    const BasinDev &b = bas[member];
    const size_t n2 = (size_t)b.nyp * b.px, n3 = n2 * b.nl;
    const T *P = (const T *)b.F[par], *PM = (const T *)b.F[1 - par];
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)b.nl * b.nyp * b.nxp;
         idx += (size_t)gridDim.x * blockDim.x) {
        const size_t k = idx / ((size_t)b.nyp * b.nxp), rem = idx - k * b.nyp * b.nxp;
        const int j = (int)(rem / b.nxp), i = (int)(rem - (size_t)j * b.nxp);
        const size_t o = k * n2 + (size_t)j * b.px + i;
        double dx, dy;
        dpdxy_bc(PM + k * n2, b, i, j, dx, dy);
        V[o] = -dy / b.fnot;
        V[n3 + o] = dx / b.fnot;
        dpdxy_bc(P + k * n2, b, i, j, dx, dy);
        V[2 * n3 + o] = -dy / b.fnot;
        V[3 * n3 + o] = dx / b.fnot;
    }
}

// del2_P_bc (numerics.F90:410-425) of nf FP64 fields [nl][nyp][px] each.
__global__ void k_dg_del2(const BasinDev *__restrict__ bas, int member, const double *in, double *out, int nf) {
    const BasinDev &b = bas[member];
    const size_t n2 = (size_t)b.nyp * b.px;
    const double afac = b.fx_bc / b.fx;   // alpha/(alpha/2+1)
    const size_t tot = (size_t)nf * b.nl * b.nyp * b.nxp;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < tot; idx += (size_t)gridDim.x * blockDim.x) {
        const size_t f = idx / ((size_t)b.nyp * b.nxp), rem = idx - f * b.nyp * b.nxp;
        const int j = (int)(rem / b.nxp), i = (int)(rem - (size_t)j * b.nxp);
        out[f * n2 + (size_t)j * b.px + i] = lap_bc_g(in + f * n2, b, i, j, afac);
    }
}

#define OQG_DGQ 22   // row sums per (layer, row) of k_dg_rows

// One CTA per (row j, layer k): trapezoid-in-x row sums (int_P_dx / dx) of
// the qg_diagno integrands, into R[(q nl + k) nyp + j]; q 20 and 21 are the
// row minimum and maximum of p.  V: ug, vg, uc, vc, del2 u, del4 u, del2 v,
// del4 v (FP64 [nl][nyp][px] each); tau: taux, tauy rows (or null).
template <class T>
__global__ void __launch_bounds__(128) k_dg_rows(const BasinDev *__restrict__ bas, int member, int par,
                                                 const double *V, const double *tau, double *R) {
    const BasinDev &b = bas[member];
    const int j = blockIdx.x, k = blockIdx.y, nl = b.nl, nxp = b.nxp, nyp = b.nyp;
    const size_t n2 = (size_t)nyp * b.px, n3 = n2 * nl, o0 = (size_t)k * n2 + (size_t)j * b.px;
    const T *P = (const T *)b.F[par], *Q = (const T *)b.F[2 + par];
    const T *WK = (const T *)b.wekp, *EN = (const T *)b.ent;
    __shared__ double red[32];
    double s[OQG_DGQ];
#pragma unroll
    for (int q = 0; q < OQG_DGQ; ++q) s[q] = 0.0;
    double pmin = 1e308, pmax = -1e308;
    const double gpk = k < nl - 1 ? b.gp[k] : 1.0;
    for (int i = threadIdx.x; i < nxp; i += blockDim.x) {
        const double w = trap_x(b, i);
        const size_t o = o0 + i, oj = (size_t)j * b.px + i;
        const double pv = (double)P[o];
        const double ug = V[o], vg = V[n3 + o], uc = V[2 * n3 + o], vc = V[3 * n3 + o];
        s[0] += w * pv;
        s[1] += w * ((double)Q[o] + (q_anom_stored<T>() ? b.beta * b.yprel[j] : 0.0));
        s[2] += w * (uc * V[4 * n3 + o]);
        s[3] += w * (vc * V[6 * n3 + o]);
        s[4] += w * (uc * V[5 * n3 + o]);
        s[5] += w * (vc * V[7 * n3 + o]);
        s[6] += w * (uc * uc);
        s[7] += w * (vc * vc);
        s[8] += w * uc;
        s[9] += w * (ug * ug);
        s[10] += w * (vg * vg);
        if (k < nl - 1) {
            const double eta = b.dz_sign * (pv - (double)P[o + n2]) / gpk;
            s[11] += w * eta;
            s[12] += w * (eta * eta);
            if (k == 0) s[13] += w * (eta * (EN ? (double)EN[oj] : 0.0));
        }
        if (k == 0) {
            const double wk = (double)WK[oj], e1 = EN ? (double)EN[oj] : 0.0;
            s[14] += w * wk;
            s[15] += w * fabs(wk);
            s[16] += w * e1;
            s[17] += w * fabs(e1);
            if (tau) {
                s[18] += w * (tau[oj] * uc);
                s[19] += w * (tau[n2 + oj] * vc);
            }
        }
        pmin = fmin(pmin, pv);
        pmax = fmax(pmax, pv);
    }
    for (int q = 0; q < 20; ++q) {
        const double v = block_sum(s[q], red);
        if (threadIdx.x == 0) R[((size_t)q * nl + k) * nyp + j] = v;
    }
    __shared__ double mn[32], mx[32];
    for (int o = 16; o > 0; o >>= 1) {
        pmin = fmin(pmin, __shfl_down_sync(0xffffffffu, pmin, o));
        pmax = fmax(pmax, __shfl_down_sync(0xffffffffu, pmax, o));
    }
    if ((threadIdx.x & 31) == 0) { mn[threadIdx.x >> 5] = pmin; mx[threadIdx.x >> 5] = pmax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int wv = 1; wv < (int)(blockDim.x >> 5); ++wv) { pmin = fmin(pmin, mn[wv]); pmax = fmax(pmax, mx[wv]); }
        R[((size_t)20 * nl + k) * nyp + j] = pmin;
        R[((size_t)21 * nl + k) * nyp + j] = pmax;
    }
}

}  // namespace oqg
