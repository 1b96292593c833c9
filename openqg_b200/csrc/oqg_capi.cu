// oqg_capi.cu -- the C ABI of include/oqg.h: handles, device memory, launches.
//
// A handle is one basin on one device with its own stream.  oqg_step queues
// step_qg (qg/core.F90:16-33) as five kernels per step (four when the inverse
// transforms and the assembly share one kernel); runs of steps are captured
// into CUDA graphs (the parity of the p/q buffers returns after two steps)
// and replayed.
#include "../../include/oqg.h"
#include "oqg_dev.cuh"
#include "oqg_kernels.cuh"
#include "oqg_adjoint.cuh"
#include "oqg_mixed.cuh"
#include "oqg_noalloc.cuh"
#include "oqg_setup.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace oqg;

static thread_local std::string g_err;

static int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

// The error reporter of the library's host-only files (oqg_radiat.cpp).
namespace oqg {
__attribute__((visibility("hidden"))) int host_fail(int code, const char *msg) { return fail(code, msg); }
}  // namespace oqg

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) return fail(OQG_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static inline int rup(int v, int m) { return (v + m - 1) / m * m; }

struct oqg_handle {
    int dev = 0;
    cudaStream_t st = nullptr;
    oqg_params prm{};
    bool mixed = false;
    size_t esz = 8;
    BasinDev hb{}, hb64{};
    BasinDev *d_bas = nullptr, *d_bas64 = nullptr;
    std::vector<void *> allocs;
    Work *d_wv = nullptr, *d_wx = nullptr, *d_wy = nullptr, *d_wi = nullptr;
    Work *d_wa = nullptr;                // k_xinv_asm work items
    int nv = 0, nx = 0, nys = 0, ni = 0;
    int E = 8, KB = 16, xthreads = 128, xi_threads = 64;
    int yW = 1;                          // warps per y-solve column
    bool xinv_split_needed = false;      // the modal rows do not fit in shared memory
    size_t smem_i_full = 0, smem_i64_full = 0;   // k_xinv's shared memory when it transforms
    int na = 0;                          // CTAs of k_xinv_asm
    int xg = 1;                          // transforms per CTA of k_xfwd and k_xinv_rows
    size_t smem_v = 0, smem_x = 0, smem_x64 = 0, smem_y = 0, smem_i = 0, smem_i64 = 0;
    double *stage[2] = {nullptr, nullptr};
    double *hrow = nullptr;     // contiguous host-order copy buffer [nl][nyp][nxp]
    double *dg = nullptr;       // qg_diagno scratch, made on its first call
    double *vs = nullptr;       // valids partials, made on its first call
    unsigned long long *d_bad = nullptr;
    double *d_diag = nullptr;
    void *ent_buf = nullptr;
    int par = 0;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    double g_tdt[2] = {0.0, 0.0};
    cudaGraphExec_t g1exec[2] = {nullptr, nullptr};   // one step, by parity
    double g1_tdt[2] = {0.0, 0.0};
    cudaGraphExec_t gbig[2] = {nullptr, nullptr};     // gbig_n (even) steps, by parity
    double gbig_tdt[2] = {0.0, 0.0};
    int gbig_n[2] = {0, 0};
    std::vector<double> modes_amat, modes_ctl2m, modes_ctm2l, modes_rdm2;
    double *adj = nullptr;      // adjoint buffers, made on the first oqg_adj_set
    AdjFields af{};             // their current roles
    cudaEvent_t up_ev = nullptr;   // oqg_set_forcing: the host arrays have been read
    double frc_host[2] = {0.0, 0.0};   // txis, txin as last queued for the device
};

template <class X>
static X *dalloc(oqg_handle *h, size_t count) {
    void *p = nullptr;
    if (cudaMalloc(&p, count * sizeof(X) + 16) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, count * sizeof(X) + 16);
    h->allocs.push_back(p);
    return (X *)p;
}

// ----------------------------------------------------------- launch helpers

// Launch with programmatic stream serialisation: the kernel may be scheduled
// while its predecessor drains and waits in griddepcontrol.wait for its data.
// Inverse-transform CTA: transform threads for all NL row pairs of a CTA in
// one round where they fit (XINV_E values per thread), plus the scalar warp.
static int xinv_fft_threads(int M, int nl) {
    const int tt = (M + XINV_E - 1) / XINV_E;
    int nfft = std::min(XINV_FFT_MAX, rup(nl * tt, 32));
    return std::max(nfft, rup(tt, 32));
}
// Dynamic shared bytes of k_xinv for nfft transform threads (element size
// esz); split: the modal rows live in global memory instead.
static size_t xinv_smem(int M, int nl, int nra, int nxp, int nfft, size_t esz, bool split = false) {
    const int tt = (M + XINV_E - 1) / XINV_E, G = nfft / tt;
    const size_t set = (size_t)G * fft_buf_len(M) * 2 * esz;
    if (split) return 2 * set;
    const size_t inh = (size_t)nl * nra * nxp * esz;
    return G >= nl ? std::max(2 * set, set + inh) : 2 * set + inh;
}

template <typename... KArgs, typename... Args>
static void launch_pdl(void (*kern)(KArgs...), int grid, int block, size_t smem, cudaStream_t st,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// The y-solve instance for a column spread over W warps (1, 2 or 4) in the
// box (real) or channel (complex) form.
template <class T, bool CPLX, int W>
static void ysolve_w(int grid, size_t smem, cudaStream_t st, const BasinDev *bas, const Work *wy, bool pdl) {
    if (pdl) launch_pdl(k_ysolve<T, CPLX, W>, grid, 128 * W, smem, st, bas, wy);
    else k_ysolve<T, CPLX, W><<<grid, 128 * W, smem, st>>>(bas, wy);
}
template <class T>
static void launch_ysolve(bool cplx, int W, int grid, size_t smem, cudaStream_t st, const BasinDev *bas,
                          const Work *wy, bool pdl) {
    if (cplx) {
        if (W == 4) ysolve_w<T, true, 4>(grid, smem, st, bas, wy, pdl);
        else if (W == 2) ysolve_w<T, true, 2>(grid, smem, st, bas, wy, pdl);
        else ysolve_w<T, true, 1>(grid, smem, st, bas, wy, pdl);
    } else {
        if (W == 4) ysolve_w<T, false, 4>(grid, smem, st, bas, wy, pdl);
        else if (W == 2) ysolve_w<T, false, 2>(grid, smem, st, bas, wy, pdl);
        else ysolve_w<T, false, 1>(grid, smem, st, bas, wy, pdl);
    }
}
// Warps per y-solve column for ncols columns of ny rows: enough that the
// columns put about 20 warps on each of the 148 SMs, as long as every warp
// keeps 4 or more rows per lane and no lane more than 8 (the register path
// within the instance's register budget).
static int ysolve_warps(int ny, long long ncols) {
    int W = 1;
    while (W < 4 && ncols * W < 148LL * 20) {
        const int W2 = 2 * W;
        if (ny <= 32 * W * 4 || ny > 32 * W2 * 8) break;
        W = W2;
    }
    return W;
}

// The transform kernels' instance for a basin's transform length: one built
// for each length of the configurations' grids (boxes of 65 to 2049 points,
// the 193-point channel; only that FFT plan in its code), the any-length one
// otherwise (and for ensembles).
#define OQG_XLENS(X) X(128) X(192) X(256) X(384) X(512) X(1024) X(2048) X(4096)
template <class T, int E>
static void (*xfwd_kernel(int M))(const BasinDev *, const Work *, const void *) {
    // FP32 storage keeps the any-length instances below the in-place lengths:
    // at 513^2 the step measured 44.5 us with them against 48.1 us with the
    // per-length ones (which take 80 registers instead of 128), while at
    // 2049^2 the per-length forward transform measured 72 against 79 us;
    // FP64 measured 51.0 against 53.8 us at 513^2 the other way round
    if (std::is_same<T, float>::value && !fft_inplace_len(M)) M = 0;
    switch (M) {
#define OQG_XF(MM) case MM: return k_xfwd<T, E, MM>;
        OQG_XLENS(OQG_XF)
#undef OQG_XF
        default: return k_xfwd<T, E>;
    }
}
template <class T, int NL, int E>
static void (*xinv_rows_kernel(int M))(const BasinDev *, const Work *, int, int, int, double, T *) {
    if (std::is_same<T, float>::value && !fft_inplace_len(M)) M = 0;      // as xfwd_kernel
    switch (M) {
#define OQG_XI(MM) case MM: return k_xinv_rows<T, NL, E, MM>;
        OQG_XLENS(OQG_XI)
#undef OQG_XI
        default: return k_xinv_rows<T, NL, E>;
    }
}

// The vorticity kernel instance of a tile height (vort_tile_ok).
typedef void (*VortFn)(const BasinDev *, const Work *, int, double);
template <class T, int NL>
static VortFn vort_kernel(int vt) {
    switch (vt) {
        case 8: return k_vort<T, NL, 8>;
        case 12: return k_vort<T, NL, 12>;
        default: return k_vort<T, NL, 16>;
    }
}

// The inverse transforms as k_xinv_rows and the one-pass k_xinv_asm (box),
// or inside k_xinv; k_xinv keeps its modal rows in global memory when they
// run separately or do not fit in shared memory.
static void apply_xinv_sep(oqg_handle *h, bool on) {
    BasinDev &b = h->hb;
    b.xinv_sep = on ? 1 : 0;
    b.xinv_split = (on || h->xinv_split_needed) ? 1 : 0;
    h->smem_i = on ? 0 : h->smem_i_full;
    h->smem_i64 = on ? 0 : h->smem_i64_full;
    h->hb64.xinv_sep = b.xinv_sep;
    h->hb64.xinv_split = b.xinv_split;
}

template <class T, int NL, int E>
static void launch_step_t(oqg_handle *h, int par, double tdt) {
    const BasinDev &b = h->hb;
    launch_pdl(vort_kernel<T, NL>(h->hb.vty), h->nv, VTHREADS, h->smem_v, h->st, h->d_bas, h->d_wv, par, tdt);
    launch_pdl(xfwd_kernel<T, E>(b.M), h->nx, h->xthreads, h->smem_x, h->st, h->d_bas, h->d_wx, (const void *)nullptr);
    launch_ysolve<T>(b.cyclic, h->yW, h->nys, h->smem_y, h->st, h->d_bas, h->d_wy, true);
    if (b.xinv_sep) {
        launch_pdl(xinv_rows_kernel<T, NL, E>(b.M), h->nx + 1, rup(h->xthreads, 32), h->smem_x, h->st, h->d_bas, h->d_wx,
                   h->xg, 1, par, tdt, (T *)nullptr);
        launch_pdl(k_xinv_asm<T, NL>, h->na, 256, 0, h->st, h->d_bas, (const Work *)h->d_wa, par);
    } else {
        launch_pdl(k_xinv<T, NL>, h->ni, h->xi_threads, h->smem_i, h->st, h->d_bas, h->d_wi, par, tdt,
                   (double *)nullptr);
    }
}

// FP64 solve of the modal Helmholtz problems with the rhs buffer as input;
// modal solutions into out ([nl][nyp][px] FP64).  pdl: launched with
// programmatic stream serialisation (each kernel waits for its predecessor
// in griddepcontrol.wait before its first dependent read).
template <int NL, int E>
static void launch_solve_t(oqg_handle *h, double *out, bool pdl) {
    if (pdl) {
        launch_pdl(xfwd_kernel<double, E>(h->hb.M), h->nx, h->xthreads, h->smem_x64, h->st, h->d_bas64, h->d_wx,
                   (const void *)nullptr);
        launch_ysolve<double>(h->hb.cyclic, h->yW, h->nys, h->smem_y, h->st, h->d_bas64, h->d_wy, true);
        if (h->hb.xinv_sep)
            launch_pdl(xinv_rows_kernel<double, NL, E>(h->hb.M), h->nx, rup(h->xthreads, 32), h->smem_x64, h->st, h->d_bas64,
                       h->d_wx, h->xg, 0, 0, 0.0, out);
        else
            launch_pdl(k_xinv<double, NL>, h->ni, h->xi_threads, h->smem_i64, h->st, h->d_bas64, h->d_wi, 0, 0.0,
                       out);
        return;
    }
    xfwd_kernel<double, E>(h->hb.M)<<<h->nx, h->xthreads, h->smem_x64, h->st>>>(h->d_bas64, h->d_wx, nullptr);
    launch_ysolve<double>(h->hb.cyclic, h->yW, h->nys, h->smem_y, h->st, h->d_bas64, h->d_wy, false);
    if (h->hb.xinv_sep)
        xinv_rows_kernel<double, NL, E>(h->hb.M)<<<h->nx, rup(h->xthreads, 32), h->smem_x64, h->st>>>(h->d_bas64, h->d_wx, h->xg,
                                                                                        0, 0, 0.0, out);
    else
        k_xinv<double, NL><<<h->ni, h->xi_threads, h->smem_i64, h->st>>>(h->d_bas64, h->d_wi, 0, 0.0, out);
}

// The dynamic shared-memory limit of a kernel is a property of the function
// on a device, shared by every handle: it only ever rises, to the largest
// size any handle or ensemble on that device launches with.
static std::mutex g_smem_mu;
static std::vector<std::pair<std::pair<int, const void *>, int>> g_smem_set;

static void raise_smem(const void *fn, size_t bytes) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_smem_mu);
    for (auto &e : g_smem_set)
        if (e.first.first == dev && e.first.second == fn) {
            if ((int)bytes > e.second && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                              (int)bytes) == cudaSuccess)
                e.second = (int)bytes;
            return;
        }
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess)
        g_smem_set.push_back({{dev, fn}, (int)bytes});
}

template <class T>
static void raise_ysolve_smem(size_t y) {
    raise_smem((const void *)k_ysolve<T, true, 1>, y);
    raise_smem((const void *)k_ysolve<T, true, 2>, y);
    raise_smem((const void *)k_ysolve<T, true, 4>, y);
    raise_smem((const void *)k_ysolve<T, false, 1>, y);
    raise_smem((const void *)k_ysolve<T, false, 2>, y);
    raise_smem((const void *)k_ysolve<T, false, 4>, y);
}

template <class T, int NL, int E>
static void raise_step_smem(size_t v, size_t x, size_t y, size_t i) {
    for (int vt : {8, 12, 16}) raise_smem((const void *)vort_kernel<T, NL>(vt), v);
    raise_smem((const void *)k_xfwd<T, E>, x);
    raise_smem((const void *)k_xinv_rows<T, NL, E>, x);
#define OQG_RX(MM) raise_smem((const void *)k_xfwd<T, E, MM>, x); raise_smem((const void *)k_xinv_rows<T, NL, E, MM>, x);
    OQG_XLENS(OQG_RX)
#undef OQG_RX
    raise_ysolve_smem<T>(y);
    raise_smem((const void *)k_xinv<T, NL>, i);
}

template <class T, int NL, int E>
static void set_attrs_t(oqg_handle *h) {
    raise_step_smem<T, NL, E>(h->smem_v, h->smem_x, h->smem_y, h->smem_i);
    raise_smem((const void *)xfwd_kernel<double, E>(h->hb.M), h->smem_x64);
    raise_smem((const void *)xinv_rows_kernel<double, NL, E>(h->hb.M), h->smem_x64);
    raise_ysolve_smem<double>(h->smem_y);
    raise_smem((const void *)k_xinv<double, NL>, h->smem_i64);
}

// dispatch over (T, NL); 16 values per transform thread
#define OQG_DISPATCH(FN, h, ...)                                                      \
    do {                                                                              \
        const int nl_ = (h)->hb.nl;                                                   \
        if ((h)->mixed) {                                                             \
            if (nl_ == 2) FN<float, 2, 16>(__VA_ARGS__);                              \
            else if (nl_ == 3) FN<float, 3, 16>(__VA_ARGS__);                         \
            else FN<float, 4, 16>(__VA_ARGS__);                                       \
        } else {                                                                      \
            if (nl_ == 2) FN<double, 2, 16>(__VA_ARGS__);                             \
            else if (nl_ == 3) FN<double, 3, 16>(__VA_ARGS__);                        \
            else FN<double, 4, 16>(__VA_ARGS__);                                      \
        }                                                                             \
    } while (0)

static void launch_step(oqg_handle *h, int par, double tdt) { OQG_DISPATCH(launch_step_t, h, h, par, tdt); }
static void set_attrs(oqg_handle *h) { OQG_DISPATCH(set_attrs_t, h, h); }

static void launch_solve(oqg_handle *h, double *out, bool pdl = false) {
    const int nl = h->hb.nl;
    if (nl == 2) launch_solve_t<2, 16>(h, out, pdl);
    else if (nl == 3) launch_solve_t<3, 16>(h, out, pdl);
    else launch_solve_t<4, 16>(h, out, pdl);
}

#define OQG_NL_T(FN, h, ...)                                                                   \
    do {                                                                                       \
        const int nl_ = (h)->hb.nl;                                                            \
        if ((h)->mixed) { if (nl_ == 2) FN<float, 2>(__VA_ARGS__); else if (nl_ == 3) FN<float, 3>(__VA_ARGS__); else FN<float, 4>(__VA_ARGS__); } \
        else { if (nl_ == 2) FN<double, 2>(__VA_ARGS__); else if (nl_ == 3) FN<double, 3>(__VA_ARGS__); else FN<double, 4>(__VA_ARGS__); } \
    } while (0)

template <class T, int NL>
static void launch_qcomp_t(oqg_handle *h, const double *p, void *q) {
    k_qcomp<T, NL><<<296, 256, 0, h->st>>>(h->d_bas, 0, p, (T *)q);
}
template <class T, int NL>
static void launch_initc_t(oqg_handle *h, int par) {
    k_init_constraints<T, NL><<<1, 512, 0, h->st>>>(h->d_bas, 0, par);
}

// ----------------------------------------------------------- host copies
// host (nxp, nyp, nl) Fortran order <-> device staging [nl][nyp][px] FP64
static int upload3(oqg_handle *h, const double *src, double *dst, int nlay) {
    const BasinDev &b = h->hb;
    CK(cudaMemcpy2DAsync(dst, b.px * sizeof(double), src, b.nxp * sizeof(double),
                         b.nxp * sizeof(double), (size_t)b.nyp * nlay, cudaMemcpyHostToDevice, h->st));
    return OQG_OK;
}
static int download3(oqg_handle *h, const double *src, double *dst, int nlay) {
    const BasinDev &b = h->hb;
    CK(cudaMemcpy2DAsync(dst, b.nxp * sizeof(double), src, b.px * sizeof(double),
                         b.nxp * sizeof(double), (size_t)b.nyp * nlay, cudaMemcpyDeviceToHost, h->st));
    return OQG_OK;
}
// Field -> host rows: packed on the device, then one contiguous copy.
static int download_rows(oqg_handle *h, const void *field, double *dst, int nlay) {
    const BasinDev &b = h->hb;
    const size_t nrows = (size_t)b.nyp * nlay;
    if (h->mixed) k_rows_out<float><<<296, 256, 0, h->st>>>((const float *)field, h->hrow, b.nxp, b.px, nrows);
    else k_rows_out<double><<<296, 256, 0, h->st>>>((const double *)field, h->hrow, b.nxp, b.px, nrows);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, h->hrow, nrows * b.nxp * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    return OQG_OK;
}
// staging FP64 -> field of the storage type
static void stage_to_field(oqg_handle *h, const double *s, void *f, size_t n) {
    if (h->mixed) k_cvt_in<float><<<296, 256, 0, h->st>>>(s, (float *)f, n);
    else cudaMemcpyAsync(f, s, n * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
}
static void field_to_stage(oqg_handle *h, const void *f, double *s, size_t n) {
    if (h->mixed) k_cvt_out<float><<<296, 256, 0, h->st>>>((const float *)f, s, n);
    else cudaMemcpyAsync(s, f, n * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
}
// The same for q fields, whose FP32 storage holds q - beta yprel.
static void stage_to_qfield(oqg_handle *h, const double *s, void *f, size_t n) {
    if (h->mixed) k_q_in<float><<<296, 256, 0, h->st>>>(h->d_bas64, 0, s, (float *)f, n);
    else cudaMemcpyAsync(f, s, n * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
}
static void qfield_to_stage(oqg_handle *h, const void *f, double *s, size_t n) {
    if (h->mixed) k_q_out<float><<<296, 256, 0, h->st>>>(h->d_bas64, 0, (const float *)f, s, n);
    else cudaMemcpyAsync(s, f, n * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
}

static int push_desc(oqg_handle *h) {
    CK(cudaMemcpyAsync(h->d_bas, &h->hb, sizeof(BasinDev), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_bas64, &h->hb64, sizeof(BasinDev), cudaMemcpyHostToDevice, h->st));
    return OQG_OK;
}

static void drop_graphs(oqg_handle *h) {
    for (int i = 0; i < 2; ++i) {
        if (h->gexec[i]) { cudaGraphExecDestroy(h->gexec[i]); h->gexec[i] = nullptr; }
        if (h->g1exec[i]) { cudaGraphExecDestroy(h->g1exec[i]); h->g1exec[i] = nullptr; }
        if (h->gbig[i]) { cudaGraphExecDestroy(h->gbig[i]); h->gbig[i] = nullptr; }
    }
}

// Captures `count` steps starting at parity par into an executable graph.
static int capture_steps(oqg_handle *h, int par, double tdt, int count, cudaGraphExec_t *out) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < count; ++i) launch_step(h, (par + i) & 1, tdt);
    cudaError_t e1 = cudaGetLastError();
    cudaError_t e2 = cudaStreamEndCapture(h->st, &g);
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(OQG_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    }
    cudaError_t e3 = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) return fail(OQG_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e3));
    return OQG_OK;
}

// Solve (Del^2 - rdm2_m) s_m = f for every mode m with f the (FP64, staging 0)
// field; modal solutions into staging 1.  Synchronous.
static int solve_all_modes(oqg_handle *h) {
    const BasinDev &b = h->hb;
    k_rhs_from_field<double><<<296, 256, 0, h->st>>>(h->d_bas64, 0, h->stage[0], (double *)b.rhs);
    launch_solve(h, h->stage[1]);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

// ----------------------------------------------------------- tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// Tensor maps of the closed-box tiles of k_vort (order in oqg_kernels.cuh).
// Returns false when the driver cannot encode them; the kernel then loads
// the tiles with cp.async.
static bool make_tmaps(oqg_handle *h) {
    BasinDev &b = h->hb;
    if (b.cyclic) return false;
    const char *env = std::getenv("OQG_NO_TMA");
    if (env && env[0] == '1') return false;
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const CUtensorMapDataType dt = h->mixed ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t esz = h->esz;
    std::vector<CUtensorMap> maps(OQG_NTMAP);
    auto enc3 = [&](CUtensorMap *m, void *base, cuuint32_t bx, cuuint32_t by) {
        cuuint64_t dims[3] = {(cuuint64_t)b.nxp, (cuuint64_t)b.nyp, (cuuint64_t)b.nl};
        cuuint64_t strides[2] = {(cuuint64_t)b.px * esz, (cuuint64_t)b.nyp * b.px * esz};
        cuuint32_t box[3] = {bx, by, 1}, es[3] = {1, 1, 1};
        return enc(m, dt, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    const cuuint32_t vt = (cuuint32_t)b.vty, wpq = VTX + 8, wo = VTX;
    bool ok = true;
    for (int f = 0; f < 4; ++f) ok = ok && enc3(&maps[OQG_TMAP_PQ + f], b.F[f], wpq, vt + 2);
    for (int f = 0; f < 2; ++f) ok = ok && enc3(&maps[OQG_TMAP_PM + f], b.F[f], wpq, vt + 6);
    for (int f = 0; f < 2; ++f) ok = ok && enc3(&maps[OQG_TMAP_QM + f], b.F[2 + f], wo, vt);
    {
        cuuint64_t dims[2] = {(cuuint64_t)b.nxp, (cuuint64_t)b.nyp};
        cuuint64_t strides[1] = {(cuuint64_t)b.px * esz};
        cuuint32_t box[2] = {wo, vt}, es[2] = {1, 1};
        ok = ok && enc(&maps[OQG_TMAP_WK], dt, 2, const_cast<void *>(b.wekp), dims, strides, box, es,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    if (!ok) return false;
    void *d = b.tmaps ? const_cast<void *>(b.tmaps) : dalloc<unsigned char>(h, (size_t)OQG_NTMAP * OQG_TMAP_BYTES);
    if (!d) return false;
    if (cudaMemcpy(d, maps.data(), (size_t)OQG_NTMAP * sizeof(CUtensorMap), cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    b.tmaps = d;
    return true;
}

// ----------------------------------------------------------- homogeneous solutions
// homsol_box (homog.F90:214-278) and homsol_cyclic (homog.F90:128-212); the
// Helmholtz solves run on the device.
static int homsol(oqg_handle *h) {
    BasinDev &b = h->hb;
    const int nxp = b.nxp, nyp = b.nyp, nl = b.nl, px = b.px;
    const size_t n2 = (size_t)nyp * px;
    std::vector<double> L(n2 * nl, 0.0), sol(n2 * nl);
    auto solve = [&](const std::vector<double> &f) -> int {
        CK(cudaMemcpyAsync(h->stage[0], f.data(), n2 * sizeof(double), cudaMemcpyHostToDevice, h->st));
        int rc = solve_all_modes(h);
        if (rc) return rc;
        CK(cudaMemcpy(sol.data(), h->stage[1], n2 * nl * sizeof(double), cudaMemcpyDeviceToHost));
        return OQG_OK;
    };
    const double xl = (nxp - 1) * b.dx, yl = (nyp - 1) * b.dy;
    if (!b.cyclic) {
        std::fill(L.begin(), L.begin() + n2, 1.0);
        int rc = solve(L);
        if (rc) return rc;
        std::vector<double> hsb((size_t)(nl - 1) * n2, 0.0), aipohs(nl, 0.0);
        for (int m = 1; m < nl; ++m) {
            double *H = &hsb[(m - 1) * n2];
            for (size_t x = 0; x < n2; ++x) H[x] = L[x] + b.rdm2[m] * sol[m * n2 + x];
            // int_P_dA (numerics.F90:188-204)
            double s = 0.0;
            for (int j = 0; j < nyp; ++j)
                for (int i = 0; i < nxp; ++i) {
                    double w = ((i == 0 || i == nxp - 1) ? 0.5 : 1.0) * ((j == 0 || j == nyp - 1) ? 0.5 : 1.0);
                    s += w * H[(size_t)j * px + i];
                }
            aipohs[m] = s * b.dx * b.dy;
        }
        const int n = nl - 1;
        for (int k = 0; k < n; ++k)
            for (int m = 1; m < nl; ++m)
                b.cdhoc[k + n * (m - 1)] = (b.ctm2l[m + nl * (k + 1)] - b.ctm2l[m + nl * k]) * aipohs[m];
        if (!lu_factor(n, b.cdhoc, b.lu, b.piv)) return fail(OQG_ESETUP, "Problem in DGETRF: singular cdhoc");
        void *dst = const_cast<void *>(b.hsb);
        if (h->mixed) {
            std::vector<float> f(hsb.size());
            for (size_t x = 0; x < f.size(); ++x) f[x] = (float)hsb[x];
            CK(cudaMemcpy(dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
        } else {
            CK(cudaMemcpy(dst, hsb.data(), hsb.size() * sizeof(double), cudaMemcpyHostToDevice));
        }
    } else {
        std::vector<double> hbt(nyp), hbc1((size_t)nl * nyp, 0.0), hbc2((size_t)nl * nyp, 0.0);
        for (int j = 1; j <= nyp; ++j) hbt[j - 1] = double(nyp - j) / double(nyp - 1);
        b.hbsi = yl / xl;
        for (int pass = 0; pass < 2; ++pass) {
            std::fill(L.begin(), L.end(), 0.0);
            for (int j = 0; j < nyp; ++j) {
                double ypj = j * b.dy, ypn = (nyp - 1) * b.dy;
                double v = pass == 0 ? (ypn - ypj) / yl : (ypj - 0.0) / yl;
                for (int i = 0; i < nxp; ++i) L[(size_t)j * px + i] = v;
            }
            int rc = solve(L);
            if (rc) return rc;
            std::vector<double> &dst = pass == 0 ? hbc1 : hbc2;
            for (int m = 1; m < nl; ++m)
                for (int j = 0; j < nyp; ++j)
                    dst[(size_t)m * nyp + j] = L[(size_t)j * px] + b.rdm2[m] * sol[m * n2 + (size_t)j * px];
        }
        for (int m = 1; m < nl; ++m) {
            const double *h1 = &hbc1[(size_t)m * nyp], *h2 = &hbc2[(size_t)m * nyp];
            double p1s = -xl * (h1[1] - h1[0]) / b.dy, p2s = -xl * (h2[1] - h2[0]) / b.dy;
            double p1n = xl * (h1[nyp - 1] - h1[nyp - 2]) / b.dy, p2n = xl * (h2[nyp - 1] - h2[nyp - 2]) / b.dy;
            p1s = p1s + 0.5 * b.dy * b.rdm2[m] * h1[0] * xl;
            p2s = p2s + 0.5 * b.dy * b.rdm2[m] * h2[0] * xl;
            p1n = p1n + 0.5 * b.dy * b.rdm2[m] * h1[nyp - 1] * xl;
            p2n = p2n + 0.5 * b.dy * b.rdm2[m] * h2[nyp - 1] * xl;
            double det = p1s * p2n - p2s * p1n;
            b.hc1s[m] = p1s / det;
            b.hc2s[m] = p2s / det;
            b.hc1n[m] = p1n / det;
            b.hc2n[m] = p2n / det;
        }
        CK(cudaMemcpy(const_cast<double *>(b.hbt), hbt.data(), nyp * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(const_cast<double *>(b.hbc1), hbc1.data(), hbc1.size() * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(const_cast<double *>(b.hbc2), hbc2.data(), hbc2.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    // the FP64 solve descriptor shares the constants
    std::memcpy(h->hb64.cdhoc, b.cdhoc, sizeof b.cdhoc);
    std::memcpy(h->hb64.lu, b.lu, sizeof b.lu);
    std::memcpy(h->hb64.piv, b.piv, sizeof b.piv);
    std::memcpy(h->hb64.hc1s, b.hc1s, sizeof b.hc1s);
    std::memcpy(h->hb64.hc2s, b.hc2s, sizeof b.hc2s);
    std::memcpy(h->hb64.hc1n, b.hc1n, sizeof b.hc1n);
    std::memcpy(h->hb64.hc2n, b.hc2n, sizeof b.hc2n);
    h->hb64.hbsi = b.hbsi;
    return OQG_OK;
}

static void destroy_all(oqg_handle *h) {
    if (!h) return;
    drop_graphs(h);
    if (h->st) cudaStreamSynchronize(h->st);
    if (h->up_ev) cudaEventDestroy(h->up_ev);
    for (void *p : h->allocs) cudaFree(p);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

template <class T, int NL, int E>
static void launch_phase_t(oqg_handle *h, int phase, int par, double tdt) {
    const BasinDev &b = h->hb;
    switch (phase) {
        case 0: vort_kernel<T, NL>(b.vty)<<<h->nv, VTHREADS, h->smem_v, h->st>>>(h->d_bas, h->d_wv, par, tdt); break;
        case 1: xfwd_kernel<T, E>(b.M)<<<h->nx, h->xthreads, h->smem_x, h->st>>>(h->d_bas, h->d_wx, nullptr); break;
        case 2: launch_ysolve<T>(b.cyclic, h->yW, h->nys, h->smem_y, h->st, h->d_bas, h->d_wy, false); break;
        case 3:
            if (b.xinv_sep)
                xinv_rows_kernel<T, NL, E>(b.M)<<<h->nx + 1, rup(h->xthreads, 32), h->smem_x, h->st>>>(h->d_bas, h->d_wx, h->xg,
                                                                                           1, par, tdt, nullptr);
            else
                k_xinv<T, NL><<<h->ni, h->xi_threads, h->smem_i, h->st>>>(h->d_bas, h->d_wi, par, tdt, nullptr);
            break;
        default: k_xinv_asm<T, NL><<<h->na, 256, 0, h->st>>>(h->d_bas, h->d_wa, par); break;
    }
}
static void launch_phase(oqg_handle *h, int phase, int par, double tdt) {
    OQG_DISPATCH(launch_phase_t, h, h, phase, par, tdt);
}

// ----------------------------------------------------------- ensembles
// An ensemble steps many basins of uneven size with one launch per phase:
// every member is a full handle (its fields, tables and homogeneous
// solutions, made by oqg_create), and the ensemble holds an array of their
// descriptors and one work list per kernel that concatenates the members'
// blocks, the largest members first so that small ones fill the tail.
struct oqg_ensemble {
    int dev = 0;
    cudaStream_t st = nullptr;
    std::vector<oqg_handle *> m;
    std::vector<BasinDev> hb;          // descriptors as uploaded (tdt_m per member)
    bool mixed = false;
    int nl = 3, E = 8, cyclic = 0;
    BasinDev *d_bas = nullptr;
    Work *d_wv = nullptr, *d_wx = nullptr, *d_wy = nullptr, *d_wi = nullptr;
    Work *d_wa = nullptr;              // k_xinv_asm work items (boxes)
    int na = 0;                        // k_xinv_asm work items
    bool sep = false;                  // boxes: k_xinv_rows + k_xinv_asm
    int Mu = 0;                        // the members' common transform length, else 0
    int nv = 0, nx = 0, nys = 0, ni = 0;
    size_t smem_v = 0, smem_x = 0, smem_y = 0, smem_i = 0;
    int xi_threads = 64, xthreads = 128;
    int yW = 1;                        // warps per y-solve column, one for every member
    int par = 0;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    std::vector<void *> allocs;
    size_t wv_cap = 0;                 // entries the vorticity work list can hold
};

#define OQG_DISPATCH_E(FN, e, ...)                                                    \
    do {                                                                              \
        const int nl_ = (e)->nl;                                                      \
        if ((e)->mixed) {                                                             \
            if (nl_ == 2) FN<float, 2, 16>(__VA_ARGS__);                              \
            else if (nl_ == 3) FN<float, 3, 16>(__VA_ARGS__);                         \
            else FN<float, 4, 16>(__VA_ARGS__);                                       \
        } else {                                                                      \
            if (nl_ == 2) FN<double, 2, 16>(__VA_ARGS__);                             \
            else if (nl_ == 3) FN<double, 3, 16>(__VA_ARGS__);                        \
            else FN<double, 4, 16>(__VA_ARGS__);                                      \
        }                                                                             \
    } while (0)

// One step of every member: the kernels read each member's step from its
// descriptor (tdt = 0).
template <class T, int NL, int E>
static void launch_ens_step_t(oqg_ensemble *e, int par) {
    launch_pdl(vort_kernel<T, NL>(e->hb[0].vty), e->nv, VTHREADS, e->smem_v, e->st, e->d_bas, e->d_wv, par, 0.0);
    // members of one transform length take that length's instance
    launch_pdl(xfwd_kernel<T, E>(e->Mu), e->nx, e->xthreads, e->smem_x, e->st, e->d_bas, e->d_wx,
               (const void *)nullptr);
    launch_ysolve<T>(e->cyclic, e->yW, e->nys, e->smem_y, e->st, e->d_bas, e->d_wy, true);
    if (e->sep) {
        // per-member transform groups (G = 0) and one scalar CTA per member
        const int nm = (int)e->m.size();
        launch_pdl(xinv_rows_kernel<T, NL, E>(e->Mu), e->nx + nm, e->xthreads, e->smem_x, e->st, e->d_bas, e->d_wx,
                   0, nm, par, 0.0, (T *)nullptr);
        launch_pdl(k_xinv_asm<T, NL>, e->na, 256, 0, e->st, e->d_bas, (const Work *)e->d_wa, par);
    } else {
        launch_pdl(k_xinv<T, NL>, e->ni, e->xi_threads, e->smem_i, e->st, e->d_bas, e->d_wi, par, 0.0,
                   (double *)nullptr);
    }
}
template <class T, int NL, int E>
static void raise_ens_smem_t(oqg_ensemble *e) {
    raise_step_smem<T, NL, E>(e->smem_v, e->smem_x, e->smem_y, e->smem_i);
}
static void launch_ens_step(oqg_ensemble *e, int par) { OQG_DISPATCH_E(launch_ens_step_t, e, e, par); }

static void ens_free(oqg_ensemble *e) {
    if (!e) return;
    if (e->st) cudaStreamSynchronize(e->st);
    for (int i = 0; i < 2; ++i)
        if (e->gexec[i]) cudaGraphExecDestroy(e->gexec[i]);
    for (void *p : e->allocs) cudaFree(p);
    for (oqg_handle *h : e->m) destroy_all(h);
    if (e->st) cudaStreamDestroy(e->st);
    delete e;
}

extern "C" {

const char *oqg_last_error(void) { return g_err.c_str(); }

int oqg_version(char *buf, int buflen) {
    int dev = 0, n = 0;
    cudaDeviceProp pr{};
    std::string s = "openqg_b200 (sm_100a)";
    if (cudaGetDeviceCount(&n) == cudaSuccess && n > 0 && cudaGetDevice(&dev) == cudaSuccess &&
        cudaGetDeviceProperties(&pr, dev) == cudaSuccess)
        s += std::string("; device ") + pr.name;
    else
        s += "; no device";
    if (buf && buflen > 0) {
        std::strncpy(buf, s.c_str(), buflen - 1);
        buf[buflen - 1] = 0;
    }
    return OQG_OK;
}

// batched: a member of an ensemble, whose tiles need not fill whole waves on
// their own (the ensemble's work list does), so the vorticity tiles take the
// tallest height and the least halo.
// Tile heights of the vorticity kernel measured by oqg_autotune, per basin
// shape and precision; a handle created later with the same shape starts
// from the measured height instead of the waves model.
struct TunedVty {
    int nxp, nyp, nl, cyclic, mixed, vty;
};
static std::mutex g_tuned_mu;
static std::vector<TunedVty> g_tuned;

static int tuned_vty(const oqg_params &P, bool mixed) {
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    for (const TunedVty &t : g_tuned)
        if (t.nxp == P.nxp && t.nyp == P.nyp && t.nl == P.nl && t.cyclic == (P.cyclic != 0) && t.mixed == (int)mixed)
            return t.vty;
    return 0;
}

static void record_vty(const oqg_params &P, bool mixed, int vty) {
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    for (TunedVty &t : g_tuned)
        if (t.nxp == P.nxp && t.nyp == P.nyp && t.nl == P.nl && t.cyclic == (P.cyclic != 0) && t.mixed == (int)mixed) {
            t.vty = vty;
            return;
        }
    g_tuned.push_back(TunedVty{P.nxp, P.nyp, P.nl, P.cyclic != 0, (int)mixed, vty});
}

static int create_impl(const oqg_params *prm, oqg_handle **out, bool batched) {
    if (!prm || !out) return fail(OQG_EINVAL, "null argument");
    *out = nullptr;
    const oqg_params &P = *prm;
    if (P.nl < 2 || P.nl > 4) return fail(OQG_EUNSUPPORTED, "this build handles nl in [2, 4]");
    if (P.nxp < 5 || P.nyp < 5) return fail(OQG_EINVAL, "grid too small (nxp, nyp >= 5)");
    if (!(P.dx > 0) || !(P.dy > 0) || P.fnot == 0.0) return fail(OQG_EINVAL, "bad dx, dy or fnot");
    if (P.k_topo < 1 || P.k_topo > P.nl) return fail(OQG_EINVAL, "k_topo out of range");
    for (int k = 0; k < P.nl; ++k)
        if (!(P.h[k] > 0)) return fail(OQG_EINVAL, "layer thickness must be > 0");
    for (int k = 0; k < P.nl - 1; ++k)
        if (!(P.gp[k] > 0)) return fail(OQG_EINVAL, "reduced gravity must be > 0");
    if (P.precision != OQG_FP64 && P.precision != OQG_MIXED) return fail(OQG_EINVAL, "bad precision");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(OQG_ENODEV, "no CUDA device");

    oqg_handle *h = new oqg_handle();
    h->prm = P;
    h->prm.ddyn = nullptr;
    h->mixed = P.precision == OQG_MIXED;
    h->esz = h->mixed ? 4 : 8;
    cudaGetDevice(&h->dev);
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return fail(OQG_ECUDA, "cudaStreamCreate failed");
    }
    auto bail = [&](int code, const std::string &msg) {
        destroy_all(h);
        return fail(code, msg);
    };

    // ---- init-time tables (qg.F90:60-103)
    Modes md;
    std::string err;
    if (!setup_modes(P.nl, P.h, P.gp, P.fnot, md, err)) return bail(OQG_ESETUP, err);
    h->modes_amat = md.amat; h->modes_ctl2m = md.ctl2m; h->modes_ctm2l = md.ctm2l; h->modes_rdm2 = md.rdm2;

    BasinDev &b = h->hb;
    b.nxp = P.nxp; b.nyp = P.nyp; b.nl = P.nl; b.cyclic = P.cyclic ? 1 : 0;
    b.px = rup(P.nxp, 32);
    b.ny = P.nyp - 2;
    if (b.cyclic) { b.nxin = P.nxp - 1; b.M = P.nxp - 1; b.nk = b.M / 2 + 1; }
    else { b.nxin = P.nxp - 2; b.M = 2 * (P.nxp - 1); b.nk = P.nxp - 2; }
    std::vector<int> rad;
    if (!fft_radices(b.M, rad) || (int)rad.size() > OQG_MAXRAD)
        return bail(OQG_EUNSUPPORTED, "x-transform length must factor into 2, 3 and 5");
    if (b.M > 4096) return bail(OQG_EUNSUPPORTED, "x-transform length above 4096");
    b.nrad = (int)rad.size();
    for (int i = 0; i < b.nrad; ++i) b.rad[i] = rad[i];
    b.pr = rup(b.nxin, 32);
    b.pk = rup(b.nk, 32);
    // vorticity tiles: VTX columns by vty rows, vty chosen so that the tiles
    // fill whole waves of 2 CTAs per SM (cost ~ waves x halo'd rows)
    {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
        const int slots = 2 * nsm;
        b.tiles_x = (P.nxp + VTX - 1) / VTX;
        int best = 16;
        long best_cost = -1;
        for (int vt = 16; vt >= 8 && !batched; vt -= 4) {          // the compiled heights
            const int ty = vort_tile_rows(P.nyp, P.cyclic, vt);
            const long waves = ((long)b.tiles_x * ty + slots - 1) / slots;
            const long cost = waves * (vt + 6);
            if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = vt; }
        }
        const int tuned = tuned_vty(P, h->mixed);
        if (tuned > 0 && !batched) best = tuned;
        b.vty = best;
        b.tiles_y = vort_tile_rows(P.nyp, P.cyclic, b.vty);
    }
    b.kt = P.k_topo - 1;
    b.wait_limit = OQG_WAIT_LIMIT;
    b.dz_sign = P.dz_sign; b.tau_sign = P.tau_sign;
    b.suppress_period = P.suppress_period;
    b.dx = P.dx; b.dy = P.dy; b.fnot = P.fnot; b.beta = P.beta;
    b.fx = 1.0 / (P.dx * P.dx);
    b.fy = 1.0 / (P.dy * P.dy);
    b.fx_bc = b.fx * P.bcco / (0.5 * P.bcco + 1.0);
    b.fy_bc = b.fy * P.bcco / (0.5 * P.bcco + 1.0);
    b.bc_half1 = 0.5 * P.bcco + 1.0;
    b.jac_fac = 1.0 / (3.0 * (2.0 * P.dx) * (2.0 * P.dy) * P.fnot);
    b.qb_fac = P.bcco * (1.0 / (P.dx * P.dx)) / (0.5 * P.bcco + 1.0) / P.fnot;
    for (int k = 0; k < P.nl; ++k) {
        b.c2[k] = P.ah2[k] / P.fnot;
        b.c4[k] = P.ah4[k] / P.fnot;
        b.h[k] = P.h[k]; b.ah2[k] = P.ah2[k]; b.ah4[k] = P.ah4[k];
    }
    for (int k = 0; k < P.nl - 1; ++k) b.gp[k] = P.gp[k];
    const double foh0 = P.fnot / P.h[0], foh1 = P.fnot / P.h[1], foht = P.fnot / P.h[b.kt];
    b.c_ent1 = P.dz_sign * foh0;
    b.c_wind = P.tau_sign * foh0;
    b.c_ent2 = P.dz_sign * foh1;
    b.c_drag = foht * P.delek / (2.0 * std::fabs(P.fnot));
    b.delek = P.delek;
    std::copy(md.amat.begin(), md.amat.end(), b.amat);
    std::copy(md.ctl2m.begin(), md.ctl2m.end(), b.ctl2m);
    std::copy(md.ctm2l.begin(), md.ctm2l.end(), b.ctm2l);
    std::copy(md.rdm2.begin(), md.rdm2.end(), b.rdm2);
    PivotTable pt;
    setup_pivots(b.cyclic, P.nxp, P.nyp, P.dx, P.dy, md.rdm2, pt, b.a_tri);
    b.ftnorm = 1.0 / (double)(b.cyclic ? b.M : 2 * (b.nxin + 1));

    // ---- device memory
    const size_t n2 = (size_t)b.nyp * b.px, n3 = n2 * b.nl;
    for (int i = 0; i < 4; ++i) {
        b.F[i] = dalloc<char>(h, n3 * h->esz);
        if (!b.F[i]) return bail(OQG_ECUDA, "out of device memory");
    }
    b.wekp = dalloc<char>(h, n2 * h->esz);
    std::vector<double> yp(b.nyp);
    const double yl = (b.nyp - 1) * b.dy;
    for (int j = 0; j < b.nyp; ++j) yp[j] = -0.5 * yl + j * b.dy;
    double *d_yp = dalloc<double>(h, b.nyp);
    b.yprel = d_yp;
    b.topo_active = 0;
    b.ddyn = nullptr;
    if (P.ddyn) {
        double *d_dd = dalloc<double>(h, n2);
        if (!d_dd) return bail(OQG_ECUDA, "out of device memory");
        CK(cudaMemcpy2D(d_dd, b.px * sizeof(double), P.ddyn, P.nxp * sizeof(double), P.nxp * sizeof(double),
                        P.nyp, cudaMemcpyHostToDevice));
        b.ddyn = d_dd;
        b.topo_active = 1;
    }
    b.rhs = dalloc<double>(h, (size_t)b.nl * b.ny * b.pr);
    b.spec = dalloc<double>(h, (size_t)b.nl * b.ny * b.pk * (b.cyclic ? 2 : 1));
    std::vector<double> tw;
    fft_stage_twiddles(b.M, rad, tw);
    double *d_tw64 = dalloc<double>(h, tw.size());
    void *d_tw = d_tw64;
    if (h->mixed) {
        float *d_tw32 = dalloc<float>(h, tw.size());
        std::vector<float> tf(tw.begin(), tw.end());
        CK(cudaMemcpy(d_tw32, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice));
        d_tw = d_tw32;
    }
    CK(cudaMemcpy(d_tw64, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice));
    b.tw = d_tw;
    double *d_pt = dalloc<double>(h, pt.tab.size());
    int *d_po = dalloc<int>(h, pt.off.size()), *d_pl = dalloc<int>(h, pt.len.size());
    CK(cudaMemcpy(d_pt, pt.tab.data(), pt.tab.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_po, pt.off.data(), pt.off.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_pl, pt.len.data(), pt.len.size() * sizeof(int), cudaMemcpyHostToDevice));
    b.piv_tab = d_pt; b.piv_off = d_po; b.piv_len = d_pl;
    if (!b.cyclic) {
        std::vector<double> dw;
        dst_row_sums(b.nk, dw);
        double *d_dw = dalloc<double>(h, dw.size());
        CK(cudaMemcpy(d_dw, dw.data(), dw.size() * sizeof(double), cudaMemcpyHostToDevice));
        b.dst_w = d_dw;
        b.hsb = dalloc<char>(h, (size_t)(b.nl - 1) * n2 * h->esz);
    } else {
        b.hbt = dalloc<double>(h, b.nyp);
        b.hbc1 = dalloc<double>(h, (size_t)b.nl * b.nyp);
        b.hbc2 = dalloc<double>(h, (size_t)b.nl * b.nyp);
    }
    // sized for the shortest tiles (8 rows), so oqg_autotune can retile in place
    b.part_tile = dalloc<double>(h, (size_t)b.tiles_x * ((P.nyp + 7) / 8) * b.nl * OQG_NQ);
    b.part_col = dalloc<double>(h, 2 * (size_t)b.nl * b.nk);
    b.st = dalloc<DevState>(h, 2);
    b.frc = dalloc<DevForcing>(h, 1);
    b.ent_rows = dalloc<double>(h, 2 * (size_t)b.nyp);
    b.err = dalloc<int>(h, 1);
    h->stage[0] = dalloc<double>(h, n3);
    h->stage[1] = dalloc<double>(h, n3);
    h->hrow = dalloc<double>(h, (size_t)b.nl * b.nyp * b.nxp);
    h->d_bad = dalloc<unsigned long long>(h, 1);
    h->d_diag = dalloc<double>(h, 4 * (size_t)b.nl);
    if (!b.st || !b.frc || !b.err || !h->stage[1] || !h->d_diag) return bail(OQG_ECUDA, "out of device memory");
    CK(cudaMemcpy(d_yp, yp.data(), yp.size() * sizeof(double), cudaMemcpyHostToDevice));

    // ---- launch geometry
    // 16 values per transform thread: one radix-16 butterfly per stage
    h->E = 16;
    const int TT = (b.M + h->E - 1) / h->E;
    const size_t t2 = 2 * h->esz;
    const int npm = (b.ny + 1) / 2;
    h->nv = b.tiles_x * b.tiles_y;
    // forward transform: one row pair per group, CTAs of >= 128 threads; a
    // grid whose row pairs would not fill the SMs that way spreads them over
    // more, smaller CTAs (each transform is a latency chain of FFT stages)
    int GX = std::max(1, 128 / TT);
    if ((b.nl * npm + GX - 1) / GX < 148) GX = std::max(1, std::min(GX, b.nl * npm / 148));
    h->xthreads = GX * TT;
    h->xg = GX;
    h->nx = (b.nl * npm + GX - 1) / GX;
    const size_t vsz = (size_t)(b.cyclic ? 16 : 8);
    // y-solve: 4 columns (warps) per CTA; the padded column tile (pivots come through L1)
    h->KB = 4;
    h->yW = ysolve_warps(b.ny, (long long)b.nl * b.nk);
    const int LDy = ysolve_ld(b.ny, h->yW);
    h->nys = b.nl * ((b.nk + h->KB - 1) / h->KB);
    b.k4_rows = 2;
    h->ni = (b.ny + b.k4_rows - 1) / b.k4_rows;
    h->smem_v = vort_smem_bytes(b.vty, (int)h->esz);
    const int LB = fft_buf_len(b.M);
    // the long lengths transform in place: one buffer plus two staged rows per group
    const size_t xrow = (size_t)((b.nxin + 3) & ~3);
    h->smem_x = fft_inplace_len(b.M) ? (size_t)GX * (LB * t2 + 2 * xrow * h->esz) : (size_t)GX * 2 * LB * t2;
    h->smem_x64 = fft_inplace_len(b.M) ? (size_t)GX * (LB * 16 + 2 * xrow * 8) : (size_t)GX * 2 * LB * 16;
    h->smem_y = (size_t)LDy * h->KB * vsz;
    // rows of an assembly CTA: k4_rows interior rows plus at most one wall row
    const int nra = (b.ny > b.k4_rows) ? b.k4_rows + 1 : b.ny + 2;
    int nfft_i = xinv_fft_threads(b.M, b.nl);
    bool split = false;
    b.inh_g = nullptr;
    if (xinv_smem(b.M, b.nl, nra, b.nxp, nfft_i, 8) > 227 * 1024) {
        // wide grid: the modal rows go to a global buffer, and a round holds
        // as many FP64 transforms as shared memory does
        split = true;
        const int tt = (b.M + XINV_E - 1) / XINV_E;
        const size_t per = 2 * (size_t)fft_buf_len(b.M) * 16;
        const int G = std::max(1, std::min(b.nl, (int)((227 * 1024) / per)));
        nfft_i = std::min(XINV_FFT_MAX, rup(G * tt, 32));
        if ((nfft_i / tt) * per > 227 * 1024) nfft_i = rup(tt, 32);
    }
    // the buffers of the separate inverse transforms (the modal rows in
    // global memory, the step's scalars), kept at any width
    b.inh_g = dalloc<char>(h, (size_t)b.nl * b.nyp * b.px * 8);
    b.scal_g = dalloc<char>(h, sizeof(XinvScal));
    if (!b.inh_g || !b.scal_g) return bail(OQG_ECUDA, "out of device memory");
    h->xi_threads = nfft_i + 32;
    h->smem_i_full = xinv_smem(b.M, b.nl, nra, b.nxp, nfft_i, h->esz, split);
    h->smem_i64_full = xinv_smem(b.M, b.nl, nra, b.nxp, nfft_i, 8, split);
    h->xinv_split_needed = split;
    // one point per thread, at most 8 work items of 256 threads per SM (the
    // items stride over larger grids)
    b.asm_items = std::min((b.nxp * b.nyp + 255) / 256, 148 * 8);
    h->na = b.asm_items;
    // boxes: the inverse transforms run as a launch of their own, shaped like
    // the forward one, then a one-pass assembly (oqg_set_xinv_sep; faster at
    // 513^2 and the only form once the modal rows leave shared memory);
    // channels start with the one-kernel form (oqg_autotune_xinv measures both)
    apply_xinv_sep(h, !b.cyclic || split);
    if (h->smem_i64_full > 227 * 1024 || h->smem_x64 > 227 * 1024 || h->smem_y > 227 * 1024)
        return bail(OQG_EUNSUPPORTED, "grid too large for this build's shared-memory tiling");
    std::vector<Work> wv(h->nv), wx(h->nx), wy(h->nys), wi(h->ni), wa(h->na);
    for (int i = 0; i < h->na; ++i) wa[i] = Work{0, i};
    for (int i = 0; i < h->nv; ++i) wv[i] = Work{0, i};
    for (int i = 0; i < h->nx; ++i) wx[i] = Work{0, i};
    for (int i = 0; i < h->nys; ++i) wy[i] = Work{0, i};
    for (int i = 0; i < h->ni; ++i) wi[i] = Work{0, i};
    h->d_wv = dalloc<Work>(h, (size_t)b.tiles_x * ((P.nyp + 7) / 8));
    h->d_wx = dalloc<Work>(h, wx.size());
    h->d_wy = dalloc<Work>(h, wy.size());
    h->d_wi = dalloc<Work>(h, wi.size());
    h->d_wa = dalloc<Work>(h, wa.size());
    CK(cudaMemcpy(h->d_wv, wv.data(), wv.size() * sizeof(Work), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_wx, wx.data(), wx.size() * sizeof(Work), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_wy, wy.data(), wy.size() * sizeof(Work), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_wi, wi.data(), wi.size() * sizeof(Work), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_wa, wa.data(), wa.size() * sizeof(Work), cudaMemcpyHostToDevice));

    b.tmaps = nullptr;
    make_tmaps(h);
    h->hb64 = b;
    h->hb64.tw = d_tw64;
    h->d_bas = dalloc<BasinDev>(h, 1);
    h->d_bas64 = dalloc<BasinDev>(h, 1);
    set_attrs(h);
    int rc = push_desc(h);
    if (rc) { destroy_all(h); return rc; }
    rc = homsol(h);
    if (rc) { std::string m = g_err; destroy_all(h); return fail(rc, m); }
    rc = push_desc(h);
    if (rc) { destroy_all(h); return rc; }
    if (cudaStreamSynchronize(h->st) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return bail(OQG_ECUDA, "device error during setup");
    *out = h;
    return OQG_OK;
}

int oqg_create(const oqg_params *prm, oqg_handle **out) { return create_impl(prm, out, false); }

int oqg_destroy(oqg_handle *h) {
    destroy_all(h);
    return OQG_OK;
}

int oqg_set_state(oqg_handle *h, const double *p, const double *pm) {
    if (!h || !p || !pm) return fail(OQG_EINVAL, "null argument");
    const BasinDev &b = h->hb;
    const size_t n3 = (size_t)b.nl * b.nyp * b.px;
    int rc;
    if ((rc = upload3(h, p, h->stage[0], b.nl))) return rc;
    if ((rc = upload3(h, pm, h->stage[1], b.nl))) return rc;
    const int par = h->par;
    stage_to_field(h, h->stage[0], b.F[par], n3);
    stage_to_field(h, h->stage[1], b.F[1 - par], n3);
    OQG_NL_T(launch_qcomp_t, h, h, h->stage[0], b.F[2 + par]);
    OQG_NL_T(launch_qcomp_t, h, h, h->stage[1], b.F[3 - par]);
    OQG_NL_T(launch_initc_t, h, h, par);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_set_state_full(oqg_handle *h, const double *p, const double *pm, const double *q,
                       const double *qm, const double *dpi, const double *dpip, const double *cs,
                       const double *cn, const double *csp, const double *cnp) {
    if (!h || !p || !pm || !q || !qm || !dpi || !dpip) return fail(OQG_EINVAL, "null argument");
    const BasinDev &b = h->hb;
    const size_t n3 = (size_t)b.nl * b.nyp * b.px;
    const int par = h->par;
    const double *src[4] = {p, pm, q, qm};
    const int dst[4] = {par, 1 - par, 2 + par, 3 - par};
    for (int f = 0; f < 4; ++f) {
        int rc = upload3(h, src[f], h->stage[0], b.nl);
        if (rc) return rc;
        if (f < 2) stage_to_field(h, h->stage[0], b.F[dst[f]], n3);
        else stage_to_qfield(h, h->stage[0], b.F[dst[f]], n3);
        CK(cudaStreamSynchronize(h->st));
    }
    DevState sc;
    CK(cudaMemcpy(&sc, b.st + par, sizeof sc, cudaMemcpyDeviceToHost));
    for (int l = 0; l < b.nl - 1; ++l) { sc.dpi[l] = dpi[l]; sc.dpip[l] = dpip[l]; }
    for (int k = 0; k < b.nl; ++k) {
        if (cs) sc.cs[k] = cs[k];
        if (cn) sc.cn[k] = cn[k];
        if (csp) sc.csp[k] = csp[k];
        if (cnp) sc.cnp[k] = cnp[k];
    }
    CK(cudaMemcpy(b.st + par, &sc, sizeof sc, cudaMemcpyHostToDevice));
    return OQG_OK;
}

int oqg_get_state(oqg_handle *h, double *p, double *pm, double *q, double *qm) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    const BasinDev &b = h->hb;
    const size_t n3 = (size_t)b.nl * b.nyp * b.px;
    const int par = h->par;
    double *dst[4] = {p, pm, q, qm};
    const int src[4] = {par, 1 - par, 2 + par, 3 - par};
    for (int f = 0; f < 4; ++f) {
        if (!dst[f]) continue;
        if (f < 2) field_to_stage(h, b.F[src[f]], h->stage[0], n3);
        else qfield_to_stage(h, b.F[src[f]], h->stage[0], n3);
        int rc = download3(h, h->stage[0], dst[f], b.nl);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->st));
    }
    return OQG_OK;
}

int oqg_get_p_layer(oqg_handle *h, int k, double *out) {
    if (!h || !out || k < 0 || k >= h->hb.nl) return fail(OQG_EINVAL, "bad argument");
    const BasinDev &b = h->hb;
    const size_t n2 = (size_t)b.nyp * b.px;
    const char *src = (const char *)b.F[h->par] + k * n2 * h->esz;
    int rc = download_rows(h, src, out, 1);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_get_constraints(oqg_handle *h, double *dpi, double *dpip, double *cs, double *cn,
                        double *csp, double *cnp) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    DevState sc;
    CK(cudaStreamSynchronize(h->st));
    CK(cudaMemcpy(&sc, h->hb.st + h->par, sizeof sc, cudaMemcpyDeviceToHost));
    const int nl = h->hb.nl;
    for (int l = 0; l < nl - 1; ++l) {
        if (dpi) dpi[l] = sc.dpi[l];
        if (dpip) dpip[l] = sc.dpip[l];
    }
    for (int k = 0; k < nl; ++k) {
        if (cs) cs[k] = sc.cs[k];
        if (cn) cn[k] = sc.cn[k];
        if (csp) csp[k] = sc.csp[k];
        if (cnp) cnp[k] = sc.cnp[k];
    }
    return OQG_OK;
}

int oqg_set_forcing(oqg_handle *h, const double *wekp, const double *ent, double txis, double txin) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    BasinDev &b = h->hb;
    const size_t n2 = (size_t)b.nyp * b.px, plane = (size_t)b.nyp * b.nxp;
    if (ent && !h->ent_buf) {
        h->ent_buf = dalloc<char>(h, (size_t)(b.nl - 1) * n2 * h->esz);
        if (!h->ent_buf) return fail(OQG_ECUDA, "out of device memory");
    }
    if (!h->up_ev && cudaEventCreateWithFlags(&h->up_ev, cudaEventDisableTiming) != cudaSuccess)
        return fail(OQG_ECUDA, "cudaEventCreate failed");
    // both host arrays cross in back-to-back copies into the contiguous
    // staging rows (wekp in layer 0, ent in layers 1..nl-1); the call waits
    // only until the copies have read the caller's buffers, and the unpack
    // and integral kernels run on the stream after it returns
    if (wekp)
        CK(cudaMemcpyAsync(h->hrow, wekp, plane * sizeof(double), cudaMemcpyHostToDevice, h->st));
    // a closed box's step reads ent(:,:,1) alone (vorticity.F90:71-72,
    // pressure.F90:52-53): only that layer crosses; a channel's momentum
    // constraints also read layer 2's wall rows (vorticity.F90:88-93)
    const int ent_layers = b.cyclic ? b.nl - 1 : 1;
    if (ent)
        CK(cudaMemcpyAsync(h->hrow + plane, ent, ent_layers * plane * sizeof(double), cudaMemcpyHostToDevice,
                           h->st));
    CK(cudaEventRecord(h->up_ev, h->st));
    if (wekp) {
        if (h->mixed) k_rows_in<float><<<296, 256, 0, h->st>>>(h->hrow, (float *)b.wekp, b.nxp, b.px, b.nyp);
        else k_rows_in<double><<<296, 256, 0, h->st>>>(h->hrow, (double *)b.wekp, b.nxp, b.px, b.nyp);
    } else {
        CK(cudaMemsetAsync(const_cast<void *>(b.wekp), 0, n2 * h->esz, h->st));
    }
    const void *old_ent = b.ent;
    if (ent) {
        const size_t nr = (size_t)ent_layers * b.nyp;
        if (h->mixed) k_rows_in<float><<<296, 256, 0, h->st>>>(h->hrow + plane, (float *)h->ent_buf, b.nxp, b.px, nr);
        else k_rows_in<double><<<296, 256, 0, h->st>>>(h->hrow + plane, (double *)h->ent_buf, b.nxp, b.px, nr);
        b.ent = h->ent_buf;
    } else {
        b.ent = nullptr;
    }
    h->hb64.ent = b.ent;
    if (b.ent != old_ent) {
        int rc = push_desc(h);
        if (rc) return rc;
    }
    if (b.ent) {
        if (h->mixed) k_ent_rows<float><<<b.nyp, 128, 0, h->st>>>(h->d_bas, 0);
        else k_ent_rows<double><<<b.nyp, 128, 0, h->st>>>(h->d_bas, 0);
    }
    if (h->mixed) k_forcing_integrals<float><<<1, 512, 0, h->st>>>(h->d_bas, 0);
    else k_forcing_integrals<double><<<1, 512, 0, h->st>>>(h->d_bas, 0);
    // the two scalars are copied from the handle, not from this stack frame
    h->frc_host[0] = txis;
    h->frc_host[1] = txin;
    CK(cudaMemcpyAsync(&b.frc->txis, h->frc_host, 2 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(h->up_ev));
    return OQG_OK;
}

int oqg_step(oqg_handle *h, double tdt, int nsteps) {
    if (!h || nsteps < 0) return fail(OQG_EINVAL, "bad argument");
    int done = 0;
    // runs of steps replay a graph of up to 16 steps (one host launch for
    // many steps), pairs a two-step graph and a last step a one-step graph,
    // each cached per step parity and step length
    if (nsteps >= 4) {
        const int par = h->par;
        const int want = std::min(nsteps & ~1, 16);
        if (!h->gbig[par] || h->gbig_tdt[par] != tdt) {
            if (h->gbig[par]) { cudaGraphExecDestroy(h->gbig[par]); h->gbig[par] = nullptr; }
            int rc = capture_steps(h, par, tdt, want, &h->gbig[par]);
            if (rc) return rc;
            h->gbig_tdt[par] = tdt;
            h->gbig_n[par] = want;
        }
        for (; done + h->gbig_n[par] <= nsteps; done += h->gbig_n[par]) CK(cudaGraphLaunch(h->gbig[par], h->st));
    }
    if (nsteps - done >= 2) {
        const int par = h->par;
        if (!h->gexec[par] || h->g_tdt[par] != tdt) {
            if (h->gexec[par]) { cudaGraphExecDestroy(h->gexec[par]); h->gexec[par] = nullptr; }
            int rc = capture_steps(h, par, tdt, 2, &h->gexec[par]);
            if (rc) return rc;
            h->g_tdt[par] = tdt;
        }
        for (; done + 2 <= nsteps; done += 2) CK(cudaGraphLaunch(h->gexec[par], h->st));
    }
    if (done < nsteps) {
        const int par = h->par;
        if (!h->g1exec[par] || h->g1_tdt[par] != tdt) {
            if (h->g1exec[par]) { cudaGraphExecDestroy(h->g1exec[par]); h->g1exec[par] = nullptr; }
            int rc = capture_steps(h, par, tdt, 1, &h->g1exec[par]);
            if (rc) return rc;
            h->g1_tdt[par] = tdt;
        }
        CK(cudaGraphLaunch(h->g1exec[par], h->st));
        h->par ^= 1;
    }
    CK(cudaGetLastError());
    return OQG_OK;
}

int oqg_set_step_index(oqg_handle *h, long long steps_done) {
    if (!h || steps_done < 0) return fail(OQG_EINVAL, "bad argument");
    CK(cudaMemcpyAsync(&h->hb.st[h->par].nt, &steps_done, sizeof(long long), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_get_step_index(oqg_handle *h, long long *steps_done) {
    if (!h || !steps_done) return fail(OQG_EINVAL, "bad argument");
    CK(cudaStreamSynchronize(h->st));
    CK(cudaMemcpy(steps_done, &h->hb.st[h->par].nt, sizeof(long long), cudaMemcpyDeviceToHost));
    return OQG_OK;
}

int oqg_suppress(oqg_handle *h) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    if (h->mixed) k_suppress<float><<<296, 256, 0, h->st>>>(h->d_bas, 0, h->par);
    else k_suppress<double><<<296, 256, 0, h->st>>>(h->d_bas, 0, h->par);
    CK(cudaGetLastError());
    return OQG_OK;
}

// Reads and clears the device error word of a basin after its stream has
// drained: a timeout of a bounded wait is OQG_ETIMEOUT, any other bit
// OQG_ECUDA.  `who` names the basin in the message.
static int take_device_error(const BasinDev &b, const std::string &who) {
    int err = 0;
    CK(cudaMemcpy(&err, b.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!err) return OQG_OK;
    CK(cudaMemset(b.err, 0, sizeof(int)));
    if (err & OQG_DERR_TIMEOUT)
        return fail(OQG_ETIMEOUT, "a bounded device wait ran out" + who + "; the step's results are invalid");
    return fail(OQG_ECUDA, "device error flag set" + who);
}

int oqg_sync(oqg_handle *h) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    CK(cudaStreamSynchronize(h->st));
    return take_device_error(h->hb, "");
}

int oqg_set_wait_limit(oqg_handle *h, long long polls) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    const unsigned v = polls < 0 ? OQG_WAIT_LIMIT : (unsigned)std::min<long long>(polls, OQG_WAIT_LIMIT);
    h->hb.wait_limit = v;
    h->hb64.wait_limit = v;
    int rc = push_desc(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_check_finite(oqg_handle *h, long long *bad) {
    if (!h || !bad) return fail(OQG_EINVAL, "bad argument");
    CK(cudaMemsetAsync(h->d_bad, 0, sizeof(unsigned long long), h->st));
    if (h->mixed) k_check_finite<float><<<296, 256, 0, h->st>>>(h->d_bas, 0, h->par, h->d_bad);
    else k_check_finite<double><<<296, 256, 0, h->st>>>(h->d_bas, 0, h->par, h->d_bad);
    unsigned long long v = 0;
    CK(cudaMemcpyAsync(&v, h->d_bad, sizeof v, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    *bad = (long long)v;
    return v ? fail(OQG_ENAN, "non-finite values in the state") : OQG_OK;
}

int oqg_diag(oqg_handle *h, double *ekei, double *sfmin, double *sfmax, double *circ) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    const int nl = h->hb.nl;
    if (h->mixed) k_diag<float><<<nl, 256, 0, h->st>>>(h->d_bas, 0, h->par, h->prm.rho, h->d_diag);
    else k_diag<double><<<nl, 256, 0, h->st>>>(h->d_bas, 0, h->par, h->prm.rho, h->d_diag);
    std::vector<double> o(4 * nl);
    CK(cudaMemcpyAsync(o.data(), h->d_diag, o.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int k = 0; k < nl; ++k) {
        if (ekei) ekei[k] = o[4 * k];
        if (sfmin) sfmin[k] = o[4 * k + 1];
        if (sfmax) sfmax[k] = o[4 * k + 2];
        if (circ) circ[k] = o[4 * k + 3];
    }
    return OQG_OK;
}

int oqg_diagno(oqg_handle *h, const double *taux, const double *tauy, double tsec, double tdt,
               oqg_qg_monitor *mon) {
    if (!h || !mon) return fail(OQG_EINVAL, "bad argument");
    const BasinDev &b = h->hb;
    const int nl = b.nl, nyp = b.nyp, nxp = b.nxp;
    const size_t n2 = (size_t)nyp * b.px, n3 = n2 * nl;
    const size_t nrow = (size_t)OQG_DGQ * nl * nyp;
    if (!h->dg) {
        h->dg = dalloc<double>(h, 8 * n3 + 2 * n2 + nrow);
        if (!h->dg) return fail(OQG_ECUDA, "out of device memory");
    }
    double *V = h->dg, *tau = h->dg + 8 * n3, *R = tau + 2 * n2;
    const bool have_tau = taux && tauy;
    if (have_tau) {
        int rc = upload3(h, taux, tau, 1);
        if (!rc) rc = upload3(h, tauy, tau + n2, 1);
        if (rc) return rc;
    }
    if (h->mixed) k_dg_vel<float><<<296, 256, 0, h->st>>>(h->d_bas, 0, h->par, V);
    else k_dg_vel<double><<<296, 256, 0, h->st>>>(h->d_bas, 0, h->par, V);
    // del2 of ug, vg into slots 4 and 6, then del4 into 5 and 7
    k_dg_del2<<<296, 256, 0, h->st>>>(h->d_bas, 0, V, V + 4 * n3, 1);
    k_dg_del2<<<296, 256, 0, h->st>>>(h->d_bas, 0, V + n3, V + 6 * n3, 1);
    k_dg_del2<<<296, 256, 0, h->st>>>(h->d_bas, 0, V + 4 * n3, V + 5 * n3, 1);
    k_dg_del2<<<296, 256, 0, h->st>>>(h->d_bas, 0, V + 6 * n3, V + 7 * n3, 1);
    const dim3 grid((unsigned)nyp, (unsigned)nl);
    if (h->mixed) k_dg_rows<float><<<grid, 128, 0, h->st>>>(h->d_bas, 0, h->par, V, have_tau ? tau : nullptr, R);
    else k_dg_rows<double><<<grid, 128, 0, h->st>>>(h->d_bas, 0, h->par, V, have_tau ? tau : nullptr, R);
    CK(cudaGetLastError());
    std::vector<double> r(nrow);
    CK(cudaMemcpyAsync(r.data(), R, nrow * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    DevState stt;
    CK(cudaMemcpyAsync(&stt, b.st + h->par, sizeof stt, cudaMemcpyDeviceToHost, h->st));
    // p at the two west corners, for circ and the reference pressure
    std::vector<double> corner(2 * nl);
    for (int k = 0; k < nl; ++k) {
        field_to_stage(h, (const char *)b.F[h->par] + k * n2 * h->esz, h->stage[0] + k * n2, n2);
    }
    for (int k = 0; k < nl; ++k) {
        CK(cudaMemcpyAsync(&corner[2 * k], h->stage[0] + k * n2, sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(cudaMemcpyAsync(&corner[2 * k + 1], h->stage[0] + k * n2 + (size_t)(nyp - 1) * b.px, sizeof(double),
                           cudaMemcpyDeviceToHost, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    const oqg_params &P = h->prm;
    const double dx = b.dx, dy = b.dy, xl = (nxp - 1) * dx, yl = (nyp - 1) * dy, area = xl * yl;
    // int_P_dA of integrand q, layer k: rows in order with the y trapezoid weights
    auto I = [&](int q, int k) {
        double s = 0.0;
        const double *row = &r[((size_t)q * nl + k) * nyp];
        for (int j = 0; j < nyp; ++j) s += ((j == 0 || j == nyp - 1) ? 0.5 : 1.0) * row[j];
        return s * dx * dy;
    };
    mon->wepm = I(14, 0) / area;
    mon->wapm = I(15, 0) / area;
    mon->entm = I(16, 0) / area;
    mon->enam = I(17, 0) / area;
    const double tprev = mon->tsec;
    for (int k = 0; k < nl - 1; ++k) {
        mon->etam[k] = I(11, k) / area;
        const double et2now = I(12, k) / area;
        mon->pket[k] = tsec > tprev ? 0.5 * P.rho * P.gp[k] * (et2now - mon->et2m[k]) / (tsec - tprev) : 0.0;
        mon->et2m[k] = et2now;
    }
    mon->pken = nl > 1 ? P.rho * P.gp[0] * I(13, 0) / area : 0.0;
    mon->tsec = tsec;
    mon->utau = have_tau ? P.rho * (I(19, 0) + I(18, 0)) : 0.0;
    mon->ctot = 0.0;
    for (int k = 0; k < nl; ++k) {
        mon->pavg[k] = I(0, k) / area;
        mon->qavg[k] = I(1, k) / area;
        mon->ah2d[k] = -P.rho * P.ah2[k] * P.h[k] * (I(2, k) + I(3, k));
        mon->ah4d[k] = P.rho * P.ah4[k] * P.h[k] * (I(4, k) + I(5, k));
        mon->ekei[k] = 0.5 * P.rho * P.h[k] * (I(6, k) + I(7, k));
        // jet: |int_P_dx u| / xl per row, over the first nyp-1 rows
        const double *ru = &r[((size_t)8 * nl + k) * nyp];
        int jm = 0;
        for (int j = 1; j < nyp - 1; ++j)
            if (std::fabs(ru[j] * dx) / xl > std::fabs(ru[jm] * dx) / xl) jm = j;
        mon->pos[k] = jm + 1;
        mon->val[k] = std::fabs(ru[jm] * dx) / xl;
        const double p00 = corner[2 * k], p0n = corner[2 * k + 1];
        mon->circ[k] = 1.0e-6 * ((p00 - p0n) / P.fnot);
        mon->ctot += mon->circ[k];
        double pomin = 1e308, pomax = -1e308;
        for (int j = 0; j < nyp; ++j) {
            pomin = std::min(pomin, r[((size_t)20 * nl + k) * nyp + j]);
            pomax = std::max(pomax, r[((size_t)21 * nl + k) * nyp + j]);
        }
        const double poref = P.fnot > 0 ? p00 : p0n;
        const double e1 = std::min(pomin / P.fnot, pomax / P.fnot), e2 = std::max(pomin / P.fnot, pomax / P.fnot);
        mon->sfmin[k] = 1.0e-6 * (P.h[k] * (e1 - poref / P.fnot));
        mon->sfmax[k] = 1.0e-6 * (P.h[k] * (e2 - poref / P.fnot));
    }
    const int kt = P.k_topo - 1;
    mon->btdg = 0.5 * P.rho * P.delek * std::fabs(P.fnot) * (I(9, kt) + I(10, kt));
    for (int k = 0; k < OQG_MAX_NL; ++k) { mon->ermas[k] = 0.0; mon->emfr[k] = 0.0; }
    if (b.cyclic) {
        for (int k = 0; k < nl - 1; ++k) {
            const double est1 = P.dz_sign * (I(0, k) - I(0, k + 1)), est2 = stt.dpi[k];
            const double edif = est1 - est2, esum = std::fabs(est1) + std::fabs(est2);
            mon->ermas[k] = edif;
            mon->emfr[k] = esum > 1.0e-13 * xl * yl * tdt * P.gp[k] ? 2.0 * edif / esum : 0.0;
        }
    }
    return OQG_OK;
}

int oqg_valids(oqg_handle *h, double pext, double qext, double wext, double *ext, long long *nonfinite, int *ok) {
    if (!h || !ok) return fail(OQG_EINVAL, "bad argument");
    const int nb = 296;
    if (!h->vs) {
        h->vs = dalloc<double>(h, (size_t)nb * 7);
        if (!h->vs) return fail(OQG_ECUDA, "out of device memory");
    }
    if (h->mixed) k_valids<float><<<nb, 256, 0, h->st>>>(h->d_bas, 0, h->par, h->vs);
    else k_valids<double><<<nb, 256, 0, h->st>>>(h->d_bas, 0, h->par, h->vs);
    CK(cudaGetLastError());
    std::vector<double> r((size_t)nb * 7);
    CK(cudaMemcpyAsync(r.data(), h->vs, r.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    double e[6] = {1e308, -1e308, 1e308, -1e308, 1e308, -1e308}, bad = 0.0;
    for (int c = 0; c < nb; ++c) {
        for (int q = 0; q < 6; ++q) e[q] = (q & 1) ? std::max(e[q], r[c * 7 + q]) : std::min(e[q], r[c * 7 + q]);
        bad += r[c * 7 + 6];
    }
    const bool valid = bad == 0.0 && std::fabs(e[0]) < pext && std::fabs(e[1]) < pext && std::fabs(e[2]) < qext &&
                       std::fabs(e[3]) < qext && std::fabs(e[4]) < wext && std::fabs(e[5]) < wext;
    if (ext)
        for (int q = 0; q < 6; ++q) ext[q] = e[q];
    if (nonfinite) *nonfinite = (long long)bad;
    *ok = valid ? 1 : 0;
    return OQG_OK;
}

int oqg_solve_inhomog(oqg_handle *h, int m, const double *rhs, double *out) {
    if (!h || !rhs || !out || m < 1 || m > h->hb.nl) return fail(OQG_EINVAL, "bad argument");
    const BasinDev &b = h->hb;
    const size_t n2 = (size_t)b.nyp * b.px;
    int rc = upload3(h, rhs, h->stage[0], 1);
    if (rc) return rc;
    if ((rc = solve_all_modes(h))) return rc;
    rc = download3(h, h->stage[1] + (m - 1) * n2, out, 1);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_int_P_dA(oqg_handle *h, const double *field, double *out) {
    if (!h || !field || !out) return fail(OQG_EINVAL, "bad argument");
    int rc = upload3(h, field, h->stage[0], 1);
    if (rc) return rc;
    k_area_integral<<<1, 512, 0, h->st>>>(h->d_bas64, 0, h->stage[0], h->d_diag);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, h->d_diag, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_generate_homog_soln(oqg_handle *h, int m, const double *L, double *out) {
    int rc = oqg_solve_inhomog(h, m, L, out);
    if (rc) return rc;
    const double r = h->hb.rdm2[m - 1];
    const size_t n = (size_t)h->hb.nxp * h->hb.nyp;
    for (size_t x = 0; x < n; ++x) out[x] = L[x] + r * out[x];
    return OQG_OK;
}

int oqg_get_modes(oqg_handle *h, double *amat, double *rdm2, double *ctl2m, double *ctm2l) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    if (amat) std::copy(h->modes_amat.begin(), h->modes_amat.end(), amat);
    if (rdm2) std::copy(h->modes_rdm2.begin(), h->modes_rdm2.end(), rdm2);
    if (ctl2m) std::copy(h->modes_ctl2m.begin(), h->modes_ctl2m.end(), ctl2m);
    if (ctm2l) std::copy(h->modes_ctm2l.begin(), h->modes_ctm2l.end(), ctm2l);
    return OQG_OK;
}

// ekman_from_tau (ekman.F90:53-83), init-time on the host.
int oqg_ekman_from_tau(const oqg_params *prm, const double *taux, const double *tauy, double *wekp,
                       double *txis, double *txin) {
    if (!prm || !taux || !tauy || !wekp) return fail(OQG_EINVAL, "null argument");
    const int nxp = prm->nxp, nyp = prm->nyp, nxt = nxp - 1, nyt = nyp - 1;
    const double dx = prm->dx, dy = prm->dy, f0 = prm->fnot;
    auto P = [&](const double *a, int i, int j) { return a[i + (size_t)nxp * j]; };
    auto rowint = [&](const std::vector<double> &r) {
        double s = 0.0;
        for (int i = 1; i < nxp - 1; ++i) s += r[i];
        return (0.5 * r[0] + s + 0.5 * r[nxp - 1]) * dx;
    };
    if (prm->cyclic) {
        std::vector<double> r(nxp);
        for (int i = 0; i < nxp; ++i) r[i] = P(taux, i, 0) + P(taux, i, 1);
        if (txis) *txis = 0.5 * rowint(r);
        for (int i = 0; i < nxp; ++i) r[i] = P(taux, i, nyp - 2) + P(taux, i, nyp - 1);
        if (txin) *txin = 0.5 * rowint(r);
    } else {
        if (txis) *txis = 0.0;
        if (txin) *txin = 0.0;
    }
    std::vector<double> txt((size_t)nxt * nyp), tyt((size_t)nxp * nyt), wt((size_t)nxt * nyt);
    for (int j = 0; j < nyp; ++j)
        for (int i = 0; i < nxt; ++i) txt[i + (size_t)nxt * j] = 0.5 * (P(taux, i + 1, j) + P(taux, i, j));
    for (int j = 0; j < nyt; ++j)
        for (int i = 0; i < nxp; ++i) tyt[i + (size_t)nxp * j] = 0.5 * (P(tauy, i, j + 1) + P(tauy, i, j));
    for (int j = 0; j < nyt; ++j)
        for (int i = 0; i < nxt; ++i)
            wt[i + (size_t)nxt * j] = ((1.0 / (dx * f0)) * (tyt[(i + 1) + (size_t)nxp * j] - tyt[i + (size_t)nxp * j]) -
                                       (1.0 / (dy * f0)) * (txt[i + (size_t)nxt * (j + 1)] - txt[i + (size_t)nxt * j]));
    // map_T_to_P (numerics.F90:64-107)
    auto T_ = [&](int i, int j) { return wt[i + (size_t)nxt * j]; };
    auto W = [&](int i, int j) -> double & { return wekp[i + (size_t)nxp * j]; };
    for (int j = 1; j < nyp - 1; ++j)
        for (int i = 1; i < nxp - 1; ++i)
            W(i, j) = 0.25 * (T_(i, j) + T_(i - 1, j) + T_(i, j - 1) + T_(i - 1, j - 1));
    for (int i = 1; i < nxp - 1; ++i) {
        W(i, 0) = 0.5 * (T_(i - 1, 0) + T_(i, 0));
        W(i, nyp - 1) = 0.5 * (T_(i - 1, nyp - 2) + T_(i, nyp - 2));
    }
    if (prm->cyclic) {
        for (int j = 1; j < nyp - 1; ++j) {
            W(0, j) = 0.25 * (T_(0, j) + T_(nxp - 2, j) + T_(0, j - 1) + T_(nxp - 2, j - 1));
            W(nxp - 1, j) = W(0, j);
        }
        W(0, 0) = 0.5 * (T_(0, 0) + T_(nxp - 2, 0));
        W(0, nyp - 1) = 0.5 * (T_(0, nyp - 2) + T_(nxp - 2, nyp - 2));
        W(nxp - 1, 0) = W(0, 0);
        W(nxp - 1, nyp - 1) = W(0, nyp - 1);
    } else {
        for (int j = 1; j < nyp - 1; ++j) {
            W(0, j) = 0.5 * (T_(0, j - 1) + T_(0, j));
            W(nxp - 1, j) = 0.5 * (T_(nxp - 2, j - 1) + T_(nxp - 2, j));
        }
        W(0, 0) = T_(0, 0);
        W(nxp - 1, 0) = T_(nxp - 2, 0);
        W(0, nyp - 1) = T_(0, nyp - 2);
        W(nxp - 1, nyp - 1) = T_(nxp - 2, nyp - 2);
    }
    return OQG_OK;
}

int oqg_device_state(oqg_handle *h, void **p, void **pm, void **q, void **qm, int *pitch, int *elem_bytes) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    const int par = h->par;
    if (p) *p = h->hb.F[par];
    if (pm) *pm = h->hb.F[1 - par];
    if (q) *q = h->hb.F[2 + par];
    if (qm) *qm = h->hb.F[3 - par];
    if (pitch) *pitch = h->hb.px;
    if (elem_bytes) *elem_bytes = (int)h->esz;
    return OQG_OK;
}

int oqg_profile_phases(oqg_handle *h, double tdt, int nsteps, double *ms) {
    if (!h || !ms || nsteps < 1) return fail(OQG_EINVAL, "bad argument");
    const int np = h->hb.xinv_sep ? 5 : 4;
    cudaEvent_t ev[6];
    for (int i = 0; i <= np; ++i) CK(cudaEventCreate(&ev[i]));
    double acc[5] = {0, 0, 0, 0, 0};
    for (int s = 0; s < nsteps; ++s) {
        CK(cudaEventRecord(ev[0], h->st));
        for (int ph = 0; ph < np; ++ph) {
            launch_phase(h, ph, h->par, tdt);
            CK(cudaEventRecord(ev[ph + 1], h->st));
        }
        h->par ^= 1;
        CK(cudaEventSynchronize(ev[np]));
        for (int ph = 0; ph < np; ++ph) {
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, ev[ph], ev[ph + 1]));
            acc[ph] += t;
        }
    }
    for (int i = 0; i <= np; ++i) cudaEventDestroy(ev[i]);
    for (int ph = 0; ph < 5; ++ph) ms[ph] = acc[ph] / nsteps;
    CK(cudaGetLastError());
    return OQG_OK;
}

int oqg_stream(oqg_handle *h, void **stream) {
    if (!h || !stream) return fail(OQG_EINVAL, "bad argument");
    *stream = (void *)h->st;
    return OQG_OK;
}

int oqg_step_launches(oqg_handle *h, int *launches) {
    if (!h || !launches) return fail(OQG_EINVAL, "bad argument");
    *launches = h->hb.xinv_sep ? 5 : 4;
    return OQG_OK;
}

// A launch of the step chain with no work: it triggers its dependent and
// waits for its predecessor like the step kernels, and nothing else.
__global__ void k_chain_empty() {
    pdl_trigger();
    pdl_wait();
}

int oqg_launch_floor(oqg_handle *h, int nsteps, double *us_per_step) {
    if (!h || !us_per_step || nsteps < 1) return fail(OQG_EINVAL, "bad argument");
    struct Shape { int grid, block; size_t smem; };
    std::vector<Shape> sh = {{h->nv, VTHREADS, h->smem_v}, {h->nx, h->xthreads, h->smem_x},
                             {h->nys, 128 * h->yW, h->smem_y}};
    if (h->hb.xinv_sep) {
        sh.push_back({h->nx + 1, rup(h->xthreads, 32), h->smem_x});
        sh.push_back({h->na, 256, 0});
    } else {
        sh.push_back({h->ni, h->xi_threads, h->smem_i});
    }
    size_t mx = 0;
    for (const Shape &x : sh) mx = std::max(mx, x.smem);
    raise_smem((const void *)k_chain_empty, mx);
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < nsteps; ++s)
        for (const Shape &x : sh) launch_pdl(k_chain_empty, x.grid, x.block, x.smem, h->st);
    CK(cudaStreamEndCapture(h->st, &g));
    if (cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(OQG_ECUDA, "graph instantiation failed");
    }
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    for (int i = 0; i < 3; ++i) CK(cudaGraphLaunch(ge, h->st));
    constexpr int REP = 10;
    CK(cudaEventRecord(a, h->st));
    for (int i = 0; i < REP; ++i) CK(cudaGraphLaunch(ge, h->st));
    CK(cudaEventRecord(b, h->st));
    CK(cudaEventSynchronize(b));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    *us_per_step = 1000.0 * ms / ((double)REP * nsteps);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    CK(cudaGetLastError());
    return OQG_OK;
}

// Scratch of oqg_diag_noalloc (layout in oqg_noalloc.cuh).  Every GPU that
// loads the library holds these 256 KiB until the process exits.  Host code
// must not pass the name itself to a kernel: on the host it is only a
// stand-in symbol; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_noalloc_scratch[OQG_NOALLOC_DOUBLES];

// Address of g_noalloc_scratch on each device, found once per device by
// oqg_diag_noalloc.  Finding it (and the first touch of the kernels that use
// it) lets the CUDA runtime load the library's device code on that device,
// which is the only step of that entry point that may allocate; later calls
// only read this table.
#define OQG_NOALLOC_MAXDEV 64
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[OQG_NOALLOC_MAXDEV] = {};

int oqg_diag_noalloc(oqg_handle *h, double *ekei, double *sfmin, double *sfmax, double *circ) {
    if (!h) return OQG_EINVAL;
    const BasinDev &b = h->hb;
    if (noalloc_doubles(b.nl, b.nyp) > OQG_NOALLOC_DOUBLES) return OQG_ESCRATCH;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return OQG_ECUDA;
    if (cur != h->dev) return OQG_EINVAL;          // the handle's device must be current
    if (cur < 0 || cur >= OQG_NOALLOC_MAXDEV) return OQG_EUNSUPPORTED;
    double *scr = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[cur]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return OQG_ECUDA;
            cudaFuncAttributes fa;
            if (cudaFuncGetAttributes(&fa, k_diag_rows<double>) != cudaSuccess ||
                cudaFuncGetAttributes(&fa, k_diag_rows<float>) != cudaSuccess)
                return OQG_ECUDA;
            g_noalloc_ptr[cur] = (double *)p;
        }
        scr = g_noalloc_ptr[cur];
    }
    // the completion ticket must read zero when the kernel starts; every
    // partial and result slot is written before it is read
    if (cudaMemsetAsync(scr, 0, sizeof(unsigned long long), h->st) != cudaSuccess) return OQG_ECUDA;
    const dim3 grid((unsigned)b.nyp, (unsigned)b.nl);
    if (h->mixed) k_diag_rows<float><<<grid, 128, 0, h->st>>>(h->d_bas, 0, h->par, h->prm.rho, scr);
    else k_diag_rows<double><<<grid, 128, 0, h->st>>>(h->d_bas, 0, h->par, h->prm.rho, scr);
    if (cudaGetLastError() != cudaSuccess) return OQG_ECUDA;
    double o[4 * OQG_NLMAX];
    if (cudaMemcpyAsync(o, scr + OQG_NOALLOC_OUT, 4 * (size_t)b.nl * sizeof(double), cudaMemcpyDeviceToHost,
                        h->st) != cudaSuccess)
        return OQG_ECUDA;
    if (cudaStreamSynchronize(h->st) != cudaSuccess) return OQG_ECUDA;
    for (int k = 0; k < b.nl; ++k) {
        if (ekei) ekei[k] = o[4 * k];
        if (sfmin) sfmin[k] = o[4 * k + 1];
        if (sfmax) sfmax[k] = o[4 * k + 2];
        if (circ) circ[k] = o[4 * k + 3];
    }
    return OQG_OK;
}

// ---- ensembles (oqg_ensemble_*)
int oqg_ensemble_create(const oqg_params *members, int nmembers, oqg_ensemble **out) {
    if (!members || nmembers < 1 || !out) return fail(OQG_EINVAL, "bad argument");
    *out = nullptr;
    for (int i = 1; i < nmembers; ++i) {
        if (members[i].nl != members[0].nl || members[i].precision != members[0].precision)
            return fail(OQG_EINVAL, "ensemble members must share nl and precision");
        if ((members[i].cyclic != 0) != (members[0].cyclic != 0))
            return fail(OQG_EUNSUPPORTED, "ensemble members must be all boxes or all channels");
    }
    oqg_ensemble *e = new oqg_ensemble();
    cudaGetDevice(&e->dev);
    if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete e;
        return fail(OQG_ECUDA, "cudaStreamCreate failed");
    }
    for (int i = 0; i < nmembers; ++i) {
        oqg_handle *h = nullptr;
        const int rc = create_impl(&members[i], &h, true);
        if (rc) {
            std::string msg = "member " + std::to_string(i) + ": " + g_err;
            ens_free(e);
            return fail(rc, msg);
        }
        e->m.push_back(h);
    }
    e->mixed = e->m[0]->mixed;
    e->nl = e->m[0]->hb.nl;
    e->cyclic = e->m[0]->hb.cyclic;
    // 16 values per transform thread, as single handles take them; the
    // forward-transform CTAs hold 128 threads, or one transform of the
    // longest member if that is longer
    e->E = 16;
    e->xthreads = 128;
    for (oqg_handle *h : e->m) e->xthreads = std::max(e->xthreads, rup((h->hb.M + e->E - 1) / e->E, 32));
    const size_t esz = e->m[0]->esz, t2 = 2 * esz, vsz = e->cyclic ? 16 : 8;
    // launch sizes per member, with the ensemble's E and fixed block sizes
    std::vector<int> order(nmembers);
    for (int i = 0; i < nmembers; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return (long)e->m[a]->hb.nxp * e->m[a]->hb.nyp > (long)e->m[c]->hb.nxp * e->m[c]->hb.nyp;
    });
    std::vector<Work> wv, wx, wy, wi, wa;
    // boxes invert as a transform launch and a one-pass assembly, as single
    // handles do
    e->sep = !e->cyclic;
    e->Mu = e->m[0]->hb.M;
    for (oqg_handle *h : e->m)
        if (h->hb.M != e->Mu) e->Mu = 0;
    int nfft_e = 32;
    for (oqg_handle *h : e->m) nfft_e = std::max(nfft_e, xinv_fft_threads(h->hb.M, h->hb.nl));
    e->xi_threads = nfft_e + 32;
    {
        long long cols = 0;
        int ny_max = 0;
        for (oqg_handle *h : e->m) { cols += (long long)h->hb.nl * h->hb.nk; ny_max = std::max(ny_max, h->hb.ny); }
        e->yW = ysolve_warps(ny_max, cols);
    }
    for (int i : order) {
        const BasinDev &b = e->m[i]->hb;
        const int TT = (b.M + e->E - 1) / e->E;
        const int G = std::max(1, e->xthreads / TT);
        const int LB = fft_buf_len(b.M);
        const int npm = (b.ny + 1) / 2;
        const int nvb = b.tiles_x * b.tiles_y;
        const int nxb = (b.nl * npm + G - 1) / G;
        const int nyb = b.nl * ((b.nk + 3) / 4);
        const int nib = (b.ny + b.k4_rows - 1) / b.k4_rows;
        for (int k = 0; k < nvb; ++k) wv.push_back(Work{i, k});
        for (int k = 0; k < nxb; ++k) wx.push_back(Work{i, k});
        for (int k = 0; k < nyb; ++k) wy.push_back(Work{i, k});
        for (int k = 0; k < nib; ++k) wi.push_back(Work{i, k});
        for (int k = 0; k < (b.nxp * b.nyp + XASM_ENS_POINTS - 1) / XASM_ENS_POINTS; ++k) wa.push_back(Work{i, k});
        const int nra = (b.ny > b.k4_rows) ? b.k4_rows + 1 : b.ny + 2;
        e->smem_v = std::max(e->smem_v, vort_smem_bytes(b.vty, (int)esz));
        const size_t xrow = (size_t)((b.nxin + 3) & ~3);
        e->smem_x = std::max(e->smem_x, fft_inplace_len(b.M) ? (size_t)G * (LB * t2 + 2 * xrow * esz)
                                                               : (size_t)G * 2 * LB * t2);
        e->smem_y = std::max(e->smem_y, (size_t)ysolve_ld(b.ny, e->yW) * 4 * vsz);
        e->smem_i = std::max(e->smem_i, xinv_smem(b.M, b.nl, nra, b.nxp, nfft_e, esz, e->m[i]->xinv_split_needed));
    }
    if (e->smem_x > 227 * 1024 || e->smem_i > 227 * 1024 || e->smem_v > 227 * 1024) {
        ens_free(e);
        return fail(OQG_EUNSUPPORTED, "ensemble member too large for the shared-memory tiling");
    }
    e->nv = (int)wv.size(); e->nx = (int)wx.size(); e->nys = (int)wy.size(); e->ni = (int)wi.size();
    e->na = (int)wa.size();
    e->wv_cap = wv.size();
    auto up = [&](const void *src, size_t bytes) -> void * {
        void *d = nullptr;
        if (cudaMalloc(&d, bytes) != cudaSuccess) return nullptr;
        e->allocs.push_back(d);
        if (cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
        return d;
    };
    e->hb.resize(nmembers);
    for (int i = 0; i < nmembers; ++i) {
        e->hb[i] = e->m[i]->hb;
        e->hb[i].xinv_sep = e->sep ? 1 : 0;
        e->hb[i].xinv_split = (e->sep || e->m[i]->xinv_split_needed) ? 1 : 0;
        e->hb[i].asm_items = (e->hb[i].nxp * e->hb[i].nyp + XASM_ENS_POINTS - 1) / XASM_ENS_POINTS;
    }
    e->d_bas = (BasinDev *)up(e->hb.data(), e->hb.size() * sizeof(BasinDev));
    e->d_wv = (Work *)up(wv.data(), wv.size() * sizeof(Work));
    e->d_wx = (Work *)up(wx.data(), wx.size() * sizeof(Work));
    e->d_wy = (Work *)up(wy.data(), wy.size() * sizeof(Work));
    e->d_wi = (Work *)up(wi.data(), wi.size() * sizeof(Work));
    e->d_wa = (Work *)up(wa.data(), wa.size() * sizeof(Work));
    if (!e->d_bas || !e->d_wv || !e->d_wx || !e->d_wy || !e->d_wi || !e->d_wa) {
        ens_free(e);
        return fail(OQG_ECUDA, "out of device memory");
    }
    OQG_DISPATCH_E(raise_ens_smem_t, e, e);
    *out = e;
    return OQG_OK;
}

int oqg_ensemble_destroy(oqg_ensemble *e) {
    ens_free(e);
    return OQG_OK;
}

// Member calls run on the member's own stream: the ensemble's stream is
// drained first, and the member sees the ensemble's step parity.
static int ens_member(oqg_ensemble *e, int member, oqg_handle **h) {
    if (!e || member < 0 || member >= (int)e->m.size()) return fail(OQG_EINVAL, "bad member");
    CK(cudaStreamSynchronize(e->st));
    *h = e->m[member];
    (*h)->par = e->par;
    return OQG_OK;
}

// The member's descriptor may have changed (forcing buffers): upload it again.
static int ens_refresh(oqg_ensemble *e, int member) {
    const double tdt = e->hb[member].tdt_m;
    e->hb[member] = e->m[member]->hb;
    e->hb[member].xinv_sep = e->sep ? 1 : 0;
    e->hb[member].xinv_split = (e->sep || e->m[member]->xinv_split_needed) ? 1 : 0;
    e->hb[member].asm_items = (e->hb[member].nxp * e->hb[member].nyp + XASM_ENS_POINTS - 1) / XASM_ENS_POINTS;
    e->hb[member].tdt_m = tdt;
    CK(cudaMemcpyAsync(e->d_bas + member, &e->hb[member], sizeof(BasinDev), cudaMemcpyHostToDevice, e->st));
    CK(cudaStreamSynchronize(e->st));
    return OQG_OK;
}

int oqg_ensemble_set_state(oqg_ensemble *e, int member, const double *p, const double *pm) {
    oqg_handle *h = nullptr;
    int rc = ens_member(e, member, &h);
    if (rc) return rc;
    return oqg_set_state(h, p, pm);
}

int oqg_ensemble_get_state(oqg_ensemble *e, int member, double *p, double *pm, double *q, double *qm) {
    oqg_handle *h = nullptr;
    int rc = ens_member(e, member, &h);
    if (rc) return rc;
    return oqg_get_state(h, p, pm, q, qm);
}

int oqg_ensemble_set_forcing(oqg_ensemble *e, int member, const double *wekp, const double *ent, double txis,
                             double txin) {
    oqg_handle *h = nullptr;
    int rc = ens_member(e, member, &h);
    if (rc) return rc;
    if ((rc = oqg_set_forcing(h, wekp, ent, txis, txin))) return rc;
    // the ensemble steps on its own stream: the member's forcing must be in place
    CK(cudaStreamSynchronize(h->st));
    return ens_refresh(e, member);
}

int oqg_ensemble_step(oqg_ensemble *e, const double *tdt, int nsteps) {
    if (!e || !tdt || nsteps < 0) return fail(OQG_EINVAL, "bad argument");
    const int n = (int)e->m.size();
    bool changed = false;
    for (int i = 0; i < n; ++i) {
        if (!(tdt[i] > 0.0)) return fail(OQG_EINVAL, "tdt must be > 0 for every member");
        if (e->hb[i].tdt_m != tdt[i]) { e->hb[i].tdt_m = tdt[i]; changed = true; }
    }
    if (changed) {
        CK(cudaMemcpyAsync(e->d_bas, e->hb.data(), n * sizeof(BasinDev), cudaMemcpyHostToDevice, e->st));
        CK(cudaStreamSynchronize(e->st));
    }
    int done = 0;
    if (nsteps >= 2) {
        const int par = e->par;
        if (!e->gexec[par]) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
            launch_ens_step(e, par);
            launch_ens_step(e, 1 - par);
            cudaError_t e1 = cudaGetLastError();
            cudaError_t e2 = cudaStreamEndCapture(e->st, &g);
            if (e1 != cudaSuccess || e2 != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return fail(OQG_ECUDA, std::string("graph capture: ") +
                                           cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
            }
            cudaError_t e3 = cudaGraphInstantiate(&e->gexec[par], g, 0);
            cudaGraphDestroy(g);
            if (e3 != cudaSuccess) return fail(OQG_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e3));
        }
        for (; done + 2 <= nsteps; done += 2) CK(cudaGraphLaunch(e->gexec[par], e->st));
    }
    for (; done < nsteps; ++done) {
        launch_ens_step(e, e->par);
        e->par ^= 1;
    }
    CK(cudaGetLastError());
    return OQG_OK;
}

int oqg_ensemble_stream(oqg_ensemble *e, void **stream) {
    if (!e || !stream) return fail(OQG_EINVAL, "bad argument");
    *stream = (void *)e->st;
    return OQG_OK;
}

int oqg_ensemble_sync(oqg_ensemble *e) {
    if (!e) return fail(OQG_EINVAL, "null ensemble");
    CK(cudaStreamSynchronize(e->st));
    for (size_t i = 0; i < e->m.size(); ++i) {
        int rc = take_device_error(e->m[i]->hb, " in member " + std::to_string(i));
        if (rc) return rc;
    }
    return OQG_OK;
}

}  // extern "C"

// ===================================================================== adjoint
// The adjoint of the closed-box FP64 step (kernels in oqg_adjoint.cuh): one
// reversed step is five launches on the handle's stream (six when a
// suppress_comp_mode is transposed), the modal solve among them being the
// forward solver's own three kernels.
template <int NL>
static void launch_adj_step_t(oqg_handle *h, const double *P, const double *Q, double tdt, bool supp) {
    AdjFields &a = h->af;
    const BasinDev *d = h->d_bas64;
    const BasinDev &b = h->hb;
    // one point of one layer per thread
    const int gl = std::min((NL * b.nyp * b.nxp + OQG_ADJ_THREADS - 1) / OQG_ADJ_THREADS, 148 * 64);
    // a chain with programmatic stream serialisation: every kernel waits in
    // griddepcontrol.wait before it touches memory, and every CTA of the
    // chain waits before it exits, so a wait covers all earlier kernels
    if (supp) launch_pdl(k_adj_suppress, gl, OQG_ADJ_THREADS, 0, h->st, d, a);
    launch_pdl(k_adj_wall<NL>, OQG_ADJ_CTAS, OQG_ADJ_THREADS, 0, h->st, d, a);
    launch_solve(h, a.s, true);
    const int tx = (b.nxp + ADJ_TX - 1) / ADJ_TX, ty = (b.nyp + ADJ_TY - 1) / ADJ_TY;
    // large grids: one CTA per tile for all layers (the modal solutions are
    // read once); small ones: one CTA per tile and layer, to fill the GPU
    bool all = false;
    if constexpr (NL <= 3) all = tx * ty >= 3 * 148 * 3;
    if constexpr (NL <= 3) {
        if (all) launch_pdl(k_adj_vort<NL, true>, tx * ty, 256, 0, h->st, d, a, P, Q, tdt, tx, ty);
    }
    if (!all) launch_pdl(k_adj_vort<NL, false>, tx * ty * NL, 256, 0, h->st, d, a, P, Q, tdt, tx, ty);
    // the state adjoints change roles: (p, pm, q, qm) of the step's input
    // (nu now holds lam_qm; the old lam_q buffer becomes the scratch)
    std::swap(a.lp, a.lpm);
    double *lq_old = a.lq;
    a.lq = a.lqm;
    a.lqm = a.nu;
    a.nu = lq_old;
}

static int adj_check(oqg_handle *h, bool need_bufs) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    if (h->hb.cyclic || h->mixed)
        return fail(OQG_EUNSUPPORTED, "the adjoint covers the closed box in FP64 only");
    if (need_bufs && !h->adj) return fail(OQG_EINVAL, "no adjoint state: call oqg_adj_set first");
    return OQG_OK;
}

// (nxp, nyp, nlay) Fortran-order array, host or device memory, <-> pitched field
static int put_field(oqg_handle *h, const double *src, double *dst, int nlay) {
    const BasinDev &b = h->hb;
    CK(cudaMemcpy2DAsync(dst, b.px * sizeof(double), src, b.nxp * sizeof(double), b.nxp * sizeof(double),
                         (size_t)b.nyp * nlay, cudaMemcpyDefault, h->st));
    return OQG_OK;
}
static int get_field(oqg_handle *h, const double *src, double *dst, int nlay) {
    const BasinDev &b = h->hb;
    CK(cudaMemcpy2DAsync(dst, b.nxp * sizeof(double), src, b.px * sizeof(double), b.nxp * sizeof(double),
                         (size_t)b.nyp * nlay, cudaMemcpyDefault, h->st));
    return OQG_OK;
}

static size_t state_field_bytes(const oqg_handle *h) {
    const BasinDev &b = h->hb;
    return (size_t)b.nl * b.nyp * b.px * h->esz;
}

extern "C" {

int oqg_state_bytes(oqg_handle *h, size_t *full, size_t *pq) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    const size_t f = state_field_bytes(h);
    if (full) *full = 4 * f + sizeof(DevState);
    if (pq) *pq = 2 * f;
    return OQG_OK;
}

int oqg_state_save(oqg_handle *h, void *dst) {
    if (!h || !dst) return fail(OQG_EINVAL, "bad argument");
    const BasinDev &b = h->hb;
    const size_t f = state_field_bytes(h);
    const int par = h->par, src[4] = {par, 1 - par, 2 + par, 3 - par};
    char *o = (char *)dst;
    for (int i = 0; i < 4; ++i) CK(cudaMemcpyAsync(o + i * f, b.F[src[i]], f, cudaMemcpyDefault, h->st));
    CK(cudaMemcpyAsync(o + 4 * f, b.st + par, sizeof(DevState), cudaMemcpyDefault, h->st));
    return OQG_OK;
}

int oqg_state_load(oqg_handle *h, const void *src) {
    if (!h || !src) return fail(OQG_EINVAL, "bad argument");
    const BasinDev &b = h->hb;
    const size_t f = state_field_bytes(h);
    const int par = h->par, dst[4] = {par, 1 - par, 2 + par, 3 - par};
    const char *s = (const char *)src;
    for (int i = 0; i < 4; ++i) CK(cudaMemcpyAsync(b.F[dst[i]], s + i * f, f, cudaMemcpyDefault, h->st));
    CK(cudaMemcpyAsync(b.st + par, s + 4 * f, sizeof(DevState), cudaMemcpyDefault, h->st));
    return OQG_OK;
}

int oqg_pq_save(oqg_handle *h, void *dst) {
    if (!h || !dst) return fail(OQG_EINVAL, "bad argument");
    const BasinDev &b = h->hb;
    const size_t f = state_field_bytes(h);
    CK(cudaMemcpyAsync(dst, b.F[h->par], f, cudaMemcpyDefault, h->st));
    CK(cudaMemcpyAsync((char *)dst + f, b.F[2 + h->par], f, cudaMemcpyDefault, h->st));
    return OQG_OK;
}

int oqg_adj_set(oqg_handle *h, const double *lp, const double *lpm, const double *lq, const double *lqm,
                const double *ldpi, const double *ldpip) {
    int rc = adj_check(h, false);
    if (rc) return rc;
    const BasinDev &b = h->hb;
    const size_t n2 = (size_t)b.nyp * b.px, n3 = n2 * b.nl;
    const size_t nparts = (size_t)OQG_ADJ_CTAS * (b.nl - 1);
    if (!h->adj) {
        h->adj = dalloc<double>(h, 7 * n3 + n2 + nparts + 32 + 1);
        if (!h->adj) return fail(OQG_ECUDA, "cudaMalloc of the adjoint buffers failed");
        double *x = h->adj;
        AdjFields &a = h->af;
        a.lp = x; a.lpm = x + n3; a.lq = x + 2 * n3; a.lqm = x + 3 * n3;
        a.nu = x + 4 * n3; a.s = x + 5 * n3; a.phi = x + 6 * n3;
        a.lw = x + 7 * n3; a.part = a.lw + n2; a.scal = a.part + nparts;
        a.ticket = (unsigned int *)(a.scal + 32);
        // phi_m = S_m(1): the modal solutions of a unit interior rhs
        k_adj_unit_rhs<<<OQG_ADJ_CTAS, OQG_ADJ_THREADS, 0, h->st>>>(h->d_bas64);
        launch_solve(h, a.phi);
        CK(cudaGetLastError());
    }
    const AdjFields &a = h->af;
    double *dst[4] = {a.lp, a.lpm, a.lq, a.lqm};
    const double *src[4] = {lp, lpm, lq, lqm};
    for (int f = 0; f < 4; ++f) {
        CK(cudaMemsetAsync(dst[f], 0, n3 * sizeof(double), h->st));
        if (src[f] && (rc = put_field(h, src[f], dst[f], b.nl))) return rc;
    }
    CK(cudaMemsetAsync(a.lw, 0, n2 * sizeof(double), h->st));
    CK(cudaMemsetAsync(a.ticket, 0, sizeof(unsigned int), h->st));
    double sc[16] = {0.0};
    for (int l = 0; l < b.nl - 1; ++l) {
        sc[l] = ldpi ? ldpi[l] : 0.0;
        sc[8 + l] = ldpip ? ldpip[l] : 0.0;
    }
    CK(cudaMemcpyAsync(a.scal, sc, sizeof sc, cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_adj_get(oqg_handle *h, double *lp, double *lpm, double *lq, double *lqm, double *ldpi, double *ldpip,
                double *lwekp) {
    int rc = adj_check(h, true);
    if (rc) return rc;
    const BasinDev &b = h->hb;
    const AdjFields &a = h->af;
    const double *src[4] = {a.lp, a.lpm, a.lq, a.lqm};
    double *dst[4] = {lp, lpm, lq, lqm};
    for (int f = 0; f < 4; ++f)
        if (dst[f] && (rc = get_field(h, src[f], dst[f], b.nl))) return rc;
    if (lwekp && (rc = get_field(h, a.lw, lwekp, 1))) return rc;
    double sc[16];
    CK(cudaMemcpyAsync(sc, a.scal, sizeof sc, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int l = 0; l < b.nl - 1; ++l) {
        if (ldpi) ldpi[l] = sc[l];
        if (ldpip) ldpip[l] = sc[8 + l];
    }
    return OQG_OK;
}

int oqg_adj_step(oqg_handle *h, const void *pq, double tdt, long long step_no) {
    int rc = adj_check(h, true);
    if (rc) return rc;
    if (!pq || step_no < 1) return fail(OQG_EINVAL, "bad argument");
    const BasinDev &b = h->hb;
    const size_t n3 = (size_t)b.nl * b.nyp * b.px;
    const double *P = (const double *)pq, *Q = P + n3;
    const int per = h->prm.suppress_period;
    const bool supp = per > 0 && (step_no - 1) % per == 0;
    if (b.nl == 2) launch_adj_step_t<2>(h, P, Q, tdt, supp);
    else if (b.nl == 3) launch_adj_step_t<3>(h, P, Q, tdt, supp);
    else launch_adj_step_t<4>(h, P, Q, tdt, supp);
    CK(cudaGetLastError());
    return OQG_OK;
}

int oqg_adj_segment(oqg_handle *h, const void *ckpt, void *slots, size_t slot_stride, int n, double tdt,
                    long long first_step_no) {
    int rc = adj_check(h, true);
    if (rc) return rc;
    if (!ckpt || !slots || n < 1 || first_step_no < 1) return fail(OQG_EINVAL, "bad argument");
    size_t pqb = 0;
    oqg_state_bytes(h, nullptr, &pqb);
    if (slot_stride < pqb) return fail(OQG_EINVAL, "slot stride smaller than a p-and-q slot");
    char *sl = (char *)slots;
    if ((rc = oqg_state_load(h, ckpt))) return rc;
    for (int i = 0; i < n; ++i) {
        if ((rc = oqg_pq_save(h, sl + i * slot_stride))) return rc;
        if (i < n - 1 && (rc = oqg_step(h, tdt, 1))) return rc;
    }
    for (int i = n - 1; i >= 0; --i)
        if ((rc = oqg_adj_step(h, sl + i * slot_stride, tdt, first_step_no + i))) return rc;
    return OQG_OK;
}

int oqg_adj_initial(oqg_handle *h, double *gp, double *gpm) {
    int rc = adj_check(h, true);
    if (rc) return rc;
    const BasinDev &b = h->hb;
    const AdjFields &a = h->af;
    if (b.nl == 2) k_adj_init<2><<<OQG_ADJ_CTAS, OQG_ADJ_THREADS, 0, h->st>>>(h->d_bas64, a, a.nu, a.s);
    else if (b.nl == 3) k_adj_init<3><<<OQG_ADJ_CTAS, OQG_ADJ_THREADS, 0, h->st>>>(h->d_bas64, a, a.nu, a.s);
    else k_adj_init<4><<<OQG_ADJ_CTAS, OQG_ADJ_THREADS, 0, h->st>>>(h->d_bas64, a, a.nu, a.s);
    CK(cudaGetLastError());
    if (gp && (rc = get_field(h, a.nu, gp, b.nl))) return rc;
    if (gpm && (rc = get_field(h, a.s, gpm, b.nl))) return rc;
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

}  // extern "C"

// ================================================================ mixed layer
// The ocean mixed layer (step_oml) and the Ekman fields from the wind stress,
// on the device, feeding the QG handle's forcing (kernels in oqg_mixed.cuh).
struct oqg_oml {
    oqg_handle *h = nullptr;
    oqg_oml_params prm{};
    std::vector<void *> allocs;
    OmlDev o{};
    oqg_handle *ha = nullptr;             // the coupled atmosphere's handle (oqg_oml_couple)
    oqg_aml *am = nullptr;                // and its mixed layer
    TauCpl cpl{};
    cudaEvent_t ev_a = nullptr, ev_o = nullptr;
    unsigned *ticket = nullptr;           // k_oml_post's last-CTA counter (zero between launches)
};

extern "C" {

int oqg_oml_create(oqg_handle *h, const oqg_oml_params *prm, oqg_oml **out) {
    if (!h || !prm || !out) return fail(OQG_EINVAL, "null argument");
    *out = nullptr;
    const BasinDev &b = h->hb;
    if (b.cyclic) return fail(OQG_EUNSUPPORTED, "the ocean mixed layer needs a closed box");
    if (!(prm->hm > 0.0) || !(prm->rho_cp > 0.0) || prm->dt_12 == 0.0)
        return fail(OQG_EINVAL, "hm and rho_cp must be > 0 and dt_12 nonzero");
    // heat-flux conditions against the hemisphere (omlsubs.F90:45-66)
    if (prm->fluxs && b.fnot < 0.0)
        return fail(OQG_EINVAL, "southern heat-flux condition with fnot < 0 (southern hemisphere)");
    if (prm->fluxn && b.fnot > 0.0)
        return fail(OQG_EINVAL, "northern heat-flux condition with fnot > 0 (northern hemisphere)");
    oqg_oml *m = new oqg_oml();
    m->h = h;
    m->prm = *prm;
    OmlDev &o = m->o;
    o.nxp = b.nxp; o.nyp = b.nyp; o.nxt = b.nxp - 1; o.nyt = b.nyp - 1;
    o.tau_sign = b.tau_sign; o.fluxn = prm->fluxn != 0; o.fluxs = prm->fluxs != 0;
    o.dx = b.dx; o.dy = b.dy; o.fnot = b.fnot; o.hm = prm->hm; o.rho_cp = prm->rho_cp;
    o.t1_rel = prm->t1_rel; o.dt_12 = prm->dt_12; o.st2d = prm->st2d; o.st4d = prm->st4d;
    o.ycexp = prm->ycexp; o.nval = prm->nval; o.sval = prm->sval;
    const size_t nt = (size_t)o.nxt * o.nyt, np = (size_t)o.nxp * o.nyp;
    const size_t total = 6 * nt + 2 * np + OQG_OML_CTAS + 1;   // + the post kernel's ticket
    void *x = nullptr;
    if (cudaMalloc(&x, total * sizeof(double)) != cudaSuccess) {
        delete m;
        return fail(OQG_ECUDA, "cudaMalloc of the mixed-layer buffers failed");
    }
    m->allocs.push_back(x);
    double *d = (double *)x;
    o.data = d; o.datam = d + nt; o.snew = d + 2 * nt; o.wekt = d + 3 * nt; o.xfo = d + 4 * nt;
    double *fn = d + 5 * nt;
    o.fnet = fn;
    o.taux = d + 6 * nt;
    o.tauy = d + 6 * nt + np;
    o.part = d + 6 * nt + 2 * np;
    m->ticket = reinterpret_cast<unsigned *>(d + 6 * nt + 2 * np + OQG_OML_CTAS);
    if (cudaMemsetAsync(x, 0, total * sizeof(double), h->st) != cudaSuccess ||
        cudaStreamSynchronize(h->st) != cudaSuccess) {
        cudaFree(x);
        delete m;
        return fail(OQG_ECUDA, "cudaMemset of the mixed-layer buffers failed");
    }
    *out = m;
    return OQG_OK;
}

int oqg_oml_destroy(oqg_oml *m) {
    if (!m) return OQG_OK;
    // the handle may be gone already: cudaFree waits for the device by itself
    for (void *p : m->allocs) cudaFree(p);
    if (m->ev_a) cudaEventDestroy(m->ev_a);
    if (m->ev_o) cudaEventDestroy(m->ev_o);
    delete m;
    return OQG_OK;
}

int oqg_oml_set_sst(oqg_oml *m, const double *sst, const double *sstm) {
    if (!m || !sst || !sstm) return fail(OQG_EINVAL, "null argument");
    const size_t bytes = (size_t)m->o.nxt * m->o.nyt * sizeof(double);
    CK(cudaMemcpyAsync(m->o.data, sst, bytes, cudaMemcpyDefault, m->h->st));
    CK(cudaMemcpyAsync(m->o.datam, sstm, bytes, cudaMemcpyDefault, m->h->st));
    CK(cudaStreamSynchronize(m->h->st));
    return OQG_OK;
}

int oqg_oml_get_sst(oqg_oml *m, double *sst, double *sstm) {
    if (!m) return fail(OQG_EINVAL, "null argument");
    const size_t bytes = (size_t)m->o.nxt * m->o.nyt * sizeof(double);
    if (sst) CK(cudaMemcpyAsync(sst, m->o.data, bytes, cudaMemcpyDefault, m->h->st));
    if (sstm) CK(cudaMemcpyAsync(sstm, m->o.datam, bytes, cudaMemcpyDefault, m->h->st));
    CK(cudaStreamSynchronize(m->h->st));
    return OQG_OK;
}

int oqg_ocean_forcing(oqg_oml *m, const double *taux, const double *tauy, const double *fnetoc, int compute_ent,
                      double tdto) {
    if (!m || (!taux) != (!tauy)) return fail(OQG_EINVAL, "null argument");
    if (!(tdto > 0.0)) return fail(OQG_EINVAL, "tdto must be > 0");
    oqg_handle *h = m->h;
    BasinDev &b = h->hb;
    OmlDev &o = m->o;
    const size_t nt = (size_t)o.nxt * o.nyt, np = (size_t)o.nxp * o.nyp, n2 = (size_t)b.nyp * b.px;
    if (compute_ent && !h->ent_buf) {
        h->ent_buf = dalloc<char>(h, (size_t)(b.nl - 1) * n2 * h->esz);
        if (!h->ent_buf) return fail(OQG_ECUDA, "out of device memory");
    }
    if (!h->up_ev && cudaEventCreateWithFlags(&h->up_ev, cudaEventDisableTiming) != cudaSuccess)
        return fail(OQG_ECUDA, "cudaEventCreate failed");
    if (taux) {
        CK(cudaMemcpyAsync(const_cast<double *>(o.taux), taux, np * sizeof(double), cudaMemcpyDefault, h->st));
        CK(cudaMemcpyAsync(const_cast<double *>(o.tauy), tauy, np * sizeof(double), cudaMemcpyDefault, h->st));
    }
    if (fnetoc)
        CK(cudaMemcpyAsync(const_cast<double *>(o.fnet), fnetoc, nt * sizeof(double), cudaMemcpyDefault, h->st));
    // the caller may reuse its arrays once their copies are done; with
    // nothing copied the call returns without waiting for the device
    const bool copies = taux || fnetoc;
    if (copies) CK(cudaEventRecord(h->up_ev, h->st));
    const void *p1 = b.F[h->par];   // layer 1 of the current p (driver.F90:96-103)
    if (h->mixed) k_oml_step<float><<<OQG_OML_CTAS, 256, 0, h->st>>>(o, (const float *)p1, b.px, tdto, compute_ent);
    else k_oml_step<double><<<OQG_OML_CTAS, 256, 0, h->st>>>(o, (const double *)p1, b.px, tdto, compute_ent);
    // the entrainment the handle holds after this call; the last CTA of
    // k_oml_post forms its integrals and zeroes txis, txin (a closed box)
    const void *ent_after = compute_ent ? h->ent_buf : b.ent;
    if (h->mixed)
        k_oml_post<float><<<b.nyp, 128, 0, h->st>>>(o, (float *)b.wekp, (float *)h->ent_buf, b.ent_rows, b.px, b.nl,
                                                    compute_ent, OQG_OML_CTAS, h->d_bas, (const float *)ent_after,
                                                    m->ticket);
    else
        k_oml_post<double><<<b.nyp, 128, 0, h->st>>>(o, (double *)b.wekp, (double *)h->ent_buf, b.ent_rows, b.px,
                                                     b.nl, compute_ent, OQG_OML_CTAS, h->d_bas,
                                                     (const double *)ent_after, m->ticket);
    CK(cudaGetLastError());
    // datam <- data, data <- the new sst; the old datam becomes the next scratch
    double *dm_old = o.datam;
    o.datam = o.data;
    o.data = o.snew;
    o.snew = dm_old;
    if (compute_ent && b.ent != h->ent_buf) {
        b.ent = h->ent_buf;
        h->hb64.ent = b.ent;
        int rc = push_desc(h);
        if (rc) return rc;
    }
    if (copies) CK(cudaEventSynchronize(h->up_ev));
    return OQG_OK;
}

int oqg_get_forcing(oqg_handle *h, double *wekp, double *ent) {
    if (!h) return fail(OQG_EINVAL, "null handle");
    const BasinDev &b = h->hb;
    int rc;
    if (wekp && (rc = download_rows(h, b.wekp, wekp, 1))) return rc;
    if (ent) {
        if (b.ent) {
            if ((rc = download_rows(h, b.ent, ent, b.nl - 1))) return rc;
        } else {
            std::fill(ent, ent + (size_t)(b.nl - 1) * b.nyp * b.nxp, 0.0);
        }
    }
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

}  // extern "C"

// ================================================================ autotuning
// Rebuilds the vorticity kernel's tiling for tile height vt: the work list,
// the tensor maps, the shared-memory size; drops the captured graphs.
static int set_vty(oqg_handle *h, int vt) {
    BasinDev &b = h->hb;
    b.vty = vt;
    b.tiles_y = vort_tile_rows(b.nyp, b.cyclic, vt);
    h->nv = b.tiles_x * b.tiles_y;
    std::vector<Work> wv(h->nv);
    for (int i = 0; i < h->nv; ++i) wv[i] = Work{0, i};
    CK(cudaMemcpy(h->d_wv, wv.data(), wv.size() * sizeof(Work), cudaMemcpyHostToDevice));
    if (b.tmaps && !make_tmaps(h)) return fail(OQG_ECUDA, "tensor maps could not be encoded");
    h->smem_v = vort_smem_bytes(vt, (int)h->esz);
    set_attrs(h);
    h->hb64.vty = b.vty;
    h->hb64.tiles_y = b.tiles_y;
    h->hb64.tmaps = b.tmaps;
    drop_graphs(h);
    return push_desc(h);
}

// The y-solve spread over W warps per column: launch shape, shared memory,
// the graphs.
static int set_ysolve_w(oqg_handle *h, int W) {
    const size_t smem = (size_t)ysolve_ld(h->hb.ny, W) * h->KB * (h->hb.cyclic ? 16 : 8);
    if (smem > 227 * 1024) return fail(OQG_EUNSUPPORTED, "y-solve tile too large");
    h->yW = W;
    h->smem_y = smem;
    set_attrs(h);
    drop_graphs(h);
    return OQG_OK;
}

// Times nsteps steps of tdt from the handle's state under each candidate
// setting (set(h, c)), restoring the state before each; keeps the fastest
// setting and the state as found.  ms[i]: ms per step of cand[i].
template <class Set>
static int tune_setting(oqg_handle *h, double tdt, int nsteps, const std::vector<int> &cand, Set set, int *best_out,
                        std::vector<float> &ms) {
    size_t full = 0;
    oqg_state_bytes(h, &full, nullptr);
    void *save = nullptr;
    if (cudaMalloc(&save, full) != cudaSuccess) return fail(OQG_ECUDA, "cudaMalloc of the state copy failed");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = oqg_state_save(h, save);
    int best = -1;
    ms.assign(cand.size(), -1.0f);
    // three rounds over the candidates, the fastest time of each kept: one
    // timing of a few steps varies by several percent from run to run
    for (int round = 0; round < 3 && rc == OQG_OK; ++round)
    for (size_t ci = 0; ci < cand.size() && rc == OQG_OK; ++ci) {
        if ((rc = set(h, cand[ci]))) break;
        // warm up (captures the graphs), then time nsteps from the saved state
        if ((rc = oqg_state_load(h, save)) || (rc = oqg_step(h, tdt, nsteps))) break;
        if ((rc = oqg_state_load(h, save))) break;
        if (cudaStreamSynchronize(h->st) != cudaSuccess) { rc = fail(OQG_ECUDA, "autotune warm-up failed"); break; }
        cudaEventRecord(e0, h->st);
        if ((rc = oqg_step(h, tdt, nsteps))) break;
        cudaEventRecord(e1, h->st);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = fail(OQG_ECUDA, "autotune timing failed"); break; }
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        if (ms[ci] < 0.0f || t / nsteps < ms[ci]) ms[ci] = t / nsteps;
    }
    for (size_t ci = 0; ci < cand.size(); ++ci)
        if (ms[ci] >= 0.0f && (best < 0 || ms[ci] < ms[best])) best = (int)ci;
    if (best >= 0) best = cand[best];
    if (rc == OQG_OK && best >= 0) rc = set(h, best);
    if (rc == OQG_OK) rc = oqg_state_load(h, save);
    if (rc == OQG_OK && cudaStreamSynchronize(h->st) != cudaSuccess) rc = fail(OQG_ECUDA, "autotune restore failed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(save);
    if (rc == OQG_OK && best_out) *best_out = best;
    return rc;
}

extern "C" {

int oqg_get_vty(oqg_handle *h, int *vty) {
    if (!h || !vty) return fail(OQG_EINVAL, "bad argument");
    *vty = h->hb.vty;
    return OQG_OK;
}

int oqg_autotune(oqg_handle *h, double tdt, int nsteps, int *best_vty, double *ms) {
    if (!h || nsteps < 2 || !(tdt > 0.0)) return fail(OQG_EINVAL, "bad argument");
    const std::vector<int> cand = {8, 12, 16};            // the compiled heights
    std::vector<float> t;
    int best = h->hb.vty;
    const int rc = tune_setting(h, tdt, nsteps, cand, set_vty, &best, t);
    if (rc) return rc;
    if (ms)
        for (size_t i = 0; i < cand.size(); ++i) ms[cand[i]] = t[i];
    record_vty(h->prm, h->mixed, best);
    if (best_vty) *best_vty = best;
    return OQG_OK;
}

int oqg_set_xinv_sep(oqg_handle *h, int on) {
    if (!h) return fail(OQG_EINVAL, "bad argument");
    if (!on && h->xinv_split_needed)
        return fail(OQG_EUNSUPPORTED, "this width keeps its modal rows in global memory: the transforms run separately");
    apply_xinv_sep(h, on != 0);
    set_attrs(h);
    drop_graphs(h);
    const int rc = push_desc(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_get_xinv_sep(oqg_handle *h, int *on) {
    if (!h || !on) return fail(OQG_EINVAL, "bad argument");
    *on = h->hb.xinv_sep;
    return OQG_OK;
}

int oqg_autotune_xinv(oqg_handle *h, double tdt, int nsteps, int *best_sep, double *ms) {
    if (!h || nsteps < 2 || !(tdt > 0.0)) return fail(OQG_EINVAL, "bad argument");
    if (ms) ms[0] = ms[1] = -1.0;
    // grids whose modal rows leave shared memory have the two-launch form only
    if (h->xinv_split_needed) {
        if (best_sep) *best_sep = h->hb.xinv_sep;
        return OQG_OK;
    }
    auto set = [](oqg_handle *hh, int on) {
        apply_xinv_sep(hh, on != 0);
        set_attrs(hh);
        drop_graphs(hh);
        return push_desc(hh);
    };
    const std::vector<int> cand = {1, 0};
    std::vector<float> t;
    int best = h->hb.xinv_sep;
    const int rc = tune_setting(h, tdt, nsteps, cand, set, &best, t);
    if (rc) return rc;
    if (ms) { ms[1] = t[0]; ms[0] = t[1]; }
    if (best_sep) *best_sep = best;
    return OQG_OK;
}

int oqg_set_vty(oqg_handle *h, int vty) {
    if (!h || (vty != 8 && vty != 12 && vty != 16)) return fail(OQG_EINVAL, "tile height must be 8, 12 or 16");
    const int rc = set_vty(h, vty);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_set_ysolve_warps(oqg_handle *h, int warps) {
    if (!h || (warps != 1 && warps != 2 && warps != 4)) return fail(OQG_EINVAL, "warps per column must be 1, 2 or 4");
    const int rc = set_ysolve_w(h, warps);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

int oqg_get_ysolve_warps(oqg_handle *h, int *warps) {
    if (!h || !warps) return fail(OQG_EINVAL, "bad argument");
    *warps = h->yW;
    return OQG_OK;
}

int oqg_autotune_ysolve(oqg_handle *h, double tdt, int nsteps, int *best_warps, double *ms) {
    if (!h || nsteps < 2 || !(tdt > 0.0)) return fail(OQG_EINVAL, "bad argument");
    const std::vector<int> cand = {1, 2, 4};
    std::vector<float> t;
    int best = h->yW;
    const int rc = tune_setting(h, tdt, nsteps, cand, set_ysolve_w, &best, t);
    if (rc) return rc;
    if (ms)
        for (size_t i = 0; i < cand.size(); ++i) ms[i] = t[i];
    if (best_warps) *best_warps = best;
    return OQG_OK;
}

}  // extern "C"

// ------------------------------------------------- ensemble autotuning
// All members retiled to tile height vt: member descriptors and tensor maps,
// the concatenated vorticity work list (largest members first), the shared
// memory, the graphs.
static int ens_set_vty(oqg_ensemble *e, int vt) {
    const int n = (int)e->m.size();
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return (long)e->m[a]->hb.nxp * e->m[a]->hb.nyp > (long)e->m[c]->hb.nxp * e->m[c]->hb.nyp;
    });
    std::vector<Work> wv;
    for (int i = 0; i < n; ++i) {
        oqg_handle *h = e->m[i];
        BasinDev &b = h->hb;
        b.vty = vt;
        b.tiles_y = vort_tile_rows(b.nyp, b.cyclic, vt);
        if (b.tmaps && !make_tmaps(h)) return fail(OQG_ECUDA, "tensor maps could not be encoded");
        h->hb64.vty = b.vty;
        h->hb64.tiles_y = b.tiles_y;
        h->hb64.tmaps = b.tmaps;
        int rc = push_desc(h);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->st));
        e->hb[i].vty = b.vty;
        e->hb[i].tiles_y = b.tiles_y;
        e->hb[i].tmaps = b.tmaps;
    }
    for (int i : order)
        for (int k = 0; k < e->hb[i].tiles_x * e->hb[i].tiles_y; ++k) wv.push_back(Work{i, k});
    if (wv.size() > e->wv_cap) {
        void *d = nullptr;
        if (cudaMalloc(&d, wv.size() * sizeof(Work)) != cudaSuccess) return fail(OQG_ECUDA, "out of device memory");
        e->allocs.push_back(d);
        e->d_wv = (Work *)d;
        e->wv_cap = wv.size();
    }
    CK(cudaMemcpy(e->d_wv, wv.data(), wv.size() * sizeof(Work), cudaMemcpyHostToDevice));
    e->nv = (int)wv.size();
    e->smem_v = vort_smem_bytes(vt, (int)e->m[0]->esz);
    OQG_DISPATCH_E(raise_ens_smem_t, e, e);
    CK(cudaMemcpy(e->d_bas, e->hb.data(), n * sizeof(BasinDev), cudaMemcpyHostToDevice));
    for (int i = 0; i < 2; ++i)
        if (e->gexec[i]) { cudaGraphExecDestroy(e->gexec[i]); e->gexec[i] = nullptr; }
    return OQG_OK;
}

extern "C" {

int oqg_ensemble_autotune(oqg_ensemble *e, const double *tdt, int nsteps, int *best_vty, double *ms) {
    if (!e || !tdt || nsteps < 2) return fail(OQG_EINVAL, "bad argument");
    const int n = (int)e->m.size();
    CK(cudaStreamSynchronize(e->st));
    // every member's state, saved in the ensemble's current parity
    std::vector<size_t> off(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        size_t full = 0;
        oqg_state_bytes(e->m[i], &full, nullptr);
        off[i + 1] = off[i] + (full + 255) / 256 * 256;
    }
    char *save = nullptr;
    if (cudaMalloc(&save, off[n]) != cudaSuccess) return fail(OQG_ECUDA, "cudaMalloc of the state copies failed");
    auto each = [&](bool load) -> int {
        for (int i = 0; i < n; ++i) {
            oqg_handle *h = e->m[i];
            h->par = e->par;
            const int rc = load ? oqg_state_load(h, save + off[i]) : oqg_state_save(h, save + off[i]);
            if (rc) return rc;
            CK(cudaStreamSynchronize(h->st));
        }
        return OQG_OK;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = each(false);
    int best = e->hb[0].vty;
    float best_ms = -1.0f;
    for (int vt = 8; vt <= 16 && rc == OQG_OK; vt += 4) {           // the compiled heights
        if ((rc = ens_set_vty(e, vt)) || (rc = each(true)) || (rc = oqg_ensemble_step(e, tdt, nsteps))) break;
        if ((rc = oqg_ensemble_sync(e)) || (rc = each(true))) break;
        cudaEventRecord(e0, e->st);
        if ((rc = oqg_ensemble_step(e, tdt, nsteps))) break;
        cudaEventRecord(e1, e->st);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = fail(OQG_ECUDA, "autotune timing failed"); break; }
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        if (ms) ms[vt] = t / nsteps;
        if (best_ms < 0.0f || t < best_ms) { best_ms = t; best = vt; }
    }
    if (rc == OQG_OK) rc = ens_set_vty(e, best);
    if (rc == OQG_OK) rc = each(true);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(save);
    if (rc) return rc;
    if (best_vty) *best_vty = best;
    return OQG_OK;
}

}  // extern "C"

// ======================================================= atmospheric mixed layer
struct oqg_aml {
    oqg_handle *h = nullptr;
    std::vector<void *> allocs;
    AmlDev o{};
    unsigned *ticket = nullptr;           // k_aml_post's last-CTA counter (zero between launches)
};

extern "C" {

int oqg_aml_create(oqg_handle *h, const oqg_aml_params *prm, const double *xc1ast, const double *dtop,
                   oqg_aml **out) {
    if (!h || !prm || !out) return fail(OQG_EINVAL, "null argument");
    *out = nullptr;
    const BasinDev &b = h->hb;
    if (!b.cyclic) return fail(OQG_EUNSUPPORTED, "the atmospheric mixed layer needs a zonally periodic channel");
    if (!(prm->hm > 0.0) || !(prm->rho_cp > 0.0) || prm->dt_12 == 0.0)
        return fail(OQG_EINVAL, "hm and rho_cp must be > 0 and dt_12 nonzero");
    oqg_aml *m = new oqg_aml();
    m->h = h;
    AmlDev &o = m->o;
    o.nxp = b.nxp; o.nyp = b.nyp; o.nxt = b.nxp - 1; o.nyt = b.nyp - 1; o.nl = b.nl; o.tau_sign = b.tau_sign;
    o.dx = b.dx; o.dy = b.dy; o.fnot = b.fnot; o.hm = prm->hm; o.rho_cp = prm->rho_cp; o.t1_rel = prm->t1_rel;
    o.dt_12 = prm->dt_12; o.hmamin = prm->hmamin; o.hmadmp = prm->hmadmp; o.xcexp = prm->xcexp;
    o.at2d = prm->at2d; o.at4d = prm->at4d; o.ahmd = prm->ahmd; o.bface = prm->bface; o.dface = prm->dface;
    o.cdat = prm->cdat;
    for (int k = 0; k < OQG_NLMAX; ++k) {
        o.aface[k] = k < b.nl - 1 ? prm->aface[k] : 0.0;
        o.gp[k] = k < b.nl - 1 ? b.gp[k] : 1.0;
    }
    const size_t nt = (size_t)o.nxt * o.nyt, np = (size_t)o.nxp * o.nyp;
    const size_t total = 10 * nt + 3 * np + 1;   // + the post kernel's ticket
    void *x = nullptr;
    if (cudaMalloc(&x, total * sizeof(double)) != cudaSuccess) {
        delete m;
        return fail(OQG_ECUDA, "cudaMalloc of the mixed-layer buffers failed");
    }
    m->allocs.push_back(x);
    double *d = (double *)x;
    o.ast = d; o.astm = d + nt; o.asn = d + 2 * nt; o.hmx = d + 3 * nt; o.hmxm = d + 4 * nt; o.hmn = d + 5 * nt;
    o.wekt = d + 6 * nt; o.xfa = d + 7 * nt;
    double *xc = d + 8 * nt, *fn = d + 9 * nt;
    o.xc1ast = xc;
    o.fnet = fn;
    o.taux = d + 10 * nt;
    o.tauy = d + 10 * nt + np;
    double *dt = d + 10 * nt + 2 * np;
    o.dtop = dtop ? dt : nullptr;
    m->ticket = reinterpret_cast<unsigned *>(d + 10 * nt + 3 * np);
    bool ok = cudaMemsetAsync(x, 0, total * sizeof(double), h->st) == cudaSuccess;
    // init_atmos_ml: ast starts at 0, hmixa at the box's hm (amlsubs.F90:88-91)
    std::vector<double> hm0(nt, prm->hm);
    ok = ok && cudaMemcpyAsync(o.hmx, hm0.data(), nt * sizeof(double), cudaMemcpyHostToDevice, h->st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(o.hmxm, hm0.data(), nt * sizeof(double), cudaMemcpyHostToDevice, h->st) == cudaSuccess;
    if (xc1ast) ok = ok && cudaMemcpyAsync(xc, xc1ast, nt * sizeof(double), cudaMemcpyDefault, h->st) == cudaSuccess;
    if (dtop) ok = ok && cudaMemcpyAsync(dt, dtop, np * sizeof(double), cudaMemcpyDefault, h->st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(h->st) == cudaSuccess;
    if (!ok) {
        cudaFree(x);
        delete m;
        return fail(OQG_ECUDA, "setting up the mixed-layer buffers failed");
    }
    *out = m;
    return OQG_OK;
}

int oqg_aml_destroy(oqg_aml *m) {
    if (!m) return OQG_OK;
    // the handle may be gone already: cudaFree waits for the device by itself
    for (void *p : m->allocs) cudaFree(p);
    delete m;
    return OQG_OK;
}

int oqg_aml_set_state(oqg_aml *m, const double *ast, const double *astm, const double *hmixa, const double *hmixam) {
    if (!m || !ast || !astm || !hmixa || !hmixam) return fail(OQG_EINVAL, "null argument");
    const size_t bytes = (size_t)m->o.nxt * m->o.nyt * sizeof(double);
    const double *src[4] = {ast, astm, hmixa, hmixam};
    double *dst[4] = {m->o.ast, m->o.astm, m->o.hmx, m->o.hmxm};
    for (int f = 0; f < 4; ++f) CK(cudaMemcpyAsync(dst[f], src[f], bytes, cudaMemcpyDefault, m->h->st));
    CK(cudaStreamSynchronize(m->h->st));
    return OQG_OK;
}

int oqg_aml_get_state(oqg_aml *m, double *ast, double *astm, double *hmixa, double *hmixam) {
    if (!m) return fail(OQG_EINVAL, "null argument");
    const size_t bytes = (size_t)m->o.nxt * m->o.nyt * sizeof(double);
    double *dst[4] = {ast, astm, hmixa, hmixam};
    const double *src[4] = {m->o.ast, m->o.astm, m->o.hmx, m->o.hmxm};
    for (int f = 0; f < 4; ++f)
        if (dst[f]) CK(cudaMemcpyAsync(dst[f], src[f], bytes, cudaMemcpyDefault, m->h->st));
    CK(cudaStreamSynchronize(m->h->st));
    return OQG_OK;
}

int oqg_atmos_forcing(oqg_aml *m, const double *taux, const double *tauy, const double *fnetat, int compute_ent,
                      double tdta) {
    if (!m || (!taux) != (!tauy)) return fail(OQG_EINVAL, "null argument");
    if (!(tdta > 0.0)) return fail(OQG_EINVAL, "tdta must be > 0");
    oqg_handle *h = m->h;
    BasinDev &b = h->hb;
    AmlDev &o = m->o;
    const size_t nt = (size_t)o.nxt * o.nyt, np = (size_t)o.nxp * o.nyp, n2 = (size_t)b.nyp * b.px;
    if (compute_ent && !h->ent_buf) {
        h->ent_buf = dalloc<char>(h, (size_t)(b.nl - 1) * n2 * h->esz);
        if (!h->ent_buf) return fail(OQG_ECUDA, "out of device memory");
    }
    if (!h->up_ev && cudaEventCreateWithFlags(&h->up_ev, cudaEventDisableTiming) != cudaSuccess)
        return fail(OQG_ECUDA, "cudaEventCreate failed");
    const void *p1 = b.F[h->par], *pm = b.F[1 - h->par];   // driver.F90:127-135
    if (taux) {
        CK(cudaMemcpyAsync(const_cast<double *>(o.taux), taux, np * sizeof(double), cudaMemcpyDefault, h->st));
        CK(cudaMemcpyAsync(const_cast<double *>(o.tauy), tauy, np * sizeof(double), cudaMemcpyDefault, h->st));
    }
    if (fnetat)
        CK(cudaMemcpyAsync(const_cast<double *>(o.fnet), fnetat, nt * sizeof(double), cudaMemcpyDefault, h->st));
    // the caller may reuse its arrays once their copies are done; with
    // nothing copied the call returns without waiting for the device
    const bool copies = taux || fnetat;
    if (copies) CK(cudaEventRecord(h->up_ev, h->st));
    // 128-thread CTAs: a channel's T cells then reach every SM
    const int grid = std::min((int)((nt + 127) / 128), 148 * 8);
    // the entrainment the handle holds after this call; the last CTA of
    // k_aml_post forms txis, txin and the forcing integrals
    const void *ent_after = compute_ent ? h->ent_buf : b.ent;
    if (h->mixed) {
        k_aml_step<float><<<grid, 128, 0, h->st>>>(o, (const float *)p1, b.px, tdta, compute_ent);
        k_aml_post<float><<<b.nyp, 128, 0, h->st>>>(o, (const float *)pm, (float *)b.wekp, (float *)h->ent_buf,
                                                    b.ent_rows, b.px, compute_ent, h->d_bas,
                                                    (const float *)ent_after, m->ticket);
    } else {
        k_aml_step<double><<<grid, 128, 0, h->st>>>(o, (const double *)p1, b.px, tdta, compute_ent);
        k_aml_post<double><<<b.nyp, 128, 0, h->st>>>(o, (const double *)pm, (double *)b.wekp,
                                                     (double *)h->ent_buf, b.ent_rows, b.px, compute_ent, h->d_bas,
                                                     (const double *)ent_after, m->ticket);
    }
    CK(cudaGetLastError());
    // lagged <- current, current <- new; the old lagged buffers become scratch
    double *a_old = o.astm, *h_old = o.hmxm;
    o.astm = o.ast; o.ast = o.asn; o.asn = a_old;
    o.hmxm = o.hmx; o.hmx = o.hmn; o.hmn = h_old;
    if (compute_ent && b.ent != h->ent_buf) {
        b.ent = h->ent_buf;
        h->hb64.ent = b.ent;
        int rc = push_desc(h);
        if (rc) return rc;
    }
    if (copies) CK(cudaEventSynchronize(h->up_ev));
    return OQG_OK;
}

}  // extern "C"

// ================================================== atmosphere -> ocean stress
extern "C" {

int oqg_oml_couple(oqg_oml *m, oqg_aml *a, double raoro) {
    if (!m) return fail(OQG_EINVAL, "null argument");
    if (!a) {
        m->ha = nullptr;
        m->am = nullptr;
        return OQG_OK;
    }
    const BasinDev &bo = m->h->hb, &ba = a->h->hb;
    const int ndxr = (int)std::lround(ba.dx / bo.dx);
    if (ndxr < 1 || (bo.nxp - 1) % ndxr || (bo.nyp - 1) % ndxr)
        return fail(OQG_EINVAL, "the ocean grid must hold whole atmospheric cells (nxt, nyt multiples of dxa/dxo)");
    TauCpl &c = m->cpl;
    const int nxtoar = (bo.nxp - 1) / ndxr, nytoar = (bo.nyp - 1) / ndxr;
    const int r0 = (ba.nyp - 1 - nytoar) / 2;   // load_grid (grid.F90:56-57), 0-based
    if (nxtoar + 1 > ba.nxp || r0 < 0 || r0 + nytoar + 1 > ba.nyp)
        return fail(OQG_EINVAL, "the ocean does not fit inside the atmosphere's channel");
    if (!c.d || c.nxtoar != nxtoar || c.nytoar != nytoar) {
        void *d = nullptr;
        if (cudaMalloc(&d, (size_t)8 * (nxtoar + 1) * (nytoar + 1) * sizeof(double)) != cudaSuccess)
            return fail(OQG_ECUDA, "cudaMalloc of the coupling buffer failed");
        m->allocs.push_back(d);
        c.d = (double *)d;
    }
    if (!m->ev_a && cudaEventCreateWithFlags(&m->ev_a, cudaEventDisableTiming) != cudaSuccess)
        return fail(OQG_ECUDA, "cudaEventCreate failed");
    if (!m->ev_o && cudaEventCreateWithFlags(&m->ev_o, cudaEventDisableTiming) != cudaSuccess)
        return fail(OQG_ECUDA, "cudaEventCreate failed");
    c.ndxr = ndxr; c.nxtoar = nxtoar; c.nytoar = nytoar; c.c0 = 0; c.r0 = r0;
    c.nxp_a = ba.nxp; c.nyp_a = ba.nyp; c.px_a = ba.px;
    c.dxa = ba.dx; c.dya = ba.dy; c.f0a = ba.fnot; c.ah = ba.bc_half1;
    c.fxa = ba.fx; c.fya = ba.fy; c.fyb = ba.fy_bc;
    c.cdat = a->o.cdat; c.hma = a->o.hm; c.raoro = raoro;
    c.hmo = m->o.hm; c.f0o = bo.fnot;
    m->ha = a->h;
    m->am = a;
    return OQG_OK;
}

int oqg_xforc(oqg_aml *a, oqg_oml *m) {
    if (!a) return fail(OQG_EINVAL, "null argument");
    if (m && m->am != a) return fail(OQG_EINVAL, "the ocean mixed layer is not coupled to this atmosphere");
    oqg_handle *ha = a->h;
    const AmlDev &ao = a->o;
    const void *pma = ha->hb.F[1 - ha->par];   // the lagged pressure (driver.F90:47-54, before step_atm)
    const int npa = ao.nxp * ao.nyp;
    const int gp = std::min((npa + 255) / 256, 148 * 8);
    if (ha->mixed)
        k_aml_tau<float><<<gp, 256, 0, ha->st>>>(ha->d_bas, ao, (const float *)pma, const_cast<double *>(ao.taux),
                                                 const_cast<double *>(ao.tauy));
    else
        k_aml_tau<double><<<gp, 256, 0, ha->st>>>(ha->d_bas, ao, (const double *)pma, const_cast<double *>(ao.taux),
                                                  const_cast<double *>(ao.tauy));
    CK(cudaGetLastError());
    if (!m) return OQG_OK;
    // the ocean's stress: its stream waits for the atmosphere's queued work,
    // and the atmosphere's stream waits until the pressure has been read
    oqg_handle *h = m->h;
    CK(cudaEventRecord(m->ev_a, ha->st));
    CK(cudaStreamWaitEvent(h->st, m->ev_a, 0));
    const int nsub = (m->cpl.nxtoar + 1) * (m->cpl.nytoar + 1);
    const int gs = std::min((nsub + 255) / 256, 148 * 4);
    if (ha->mixed) k_cpl_derivs<float><<<gs, 256, 0, h->st>>>(m->cpl, (const float *)pma);
    else k_cpl_derivs<double><<<gs, 256, 0, h->st>>>(m->cpl, (const double *)pma);
    const int npo = m->o.nxp * m->o.nyp;
    const int gt = std::min((npo + 255) / 256, 148 * 8);
    TauCpl c = m->cpl;
    c.taux_a = const_cast<double *>(ao.taux);
    c.tauy_a = const_cast<double *>(ao.tauy);
    const void *pmo = h->hb.F[1 - h->par];    // the ocean's lagged pressure (compute_udiff)
    if (h->mixed) k_cpl_tau<float><<<gt, 256, 0, h->st>>>(c, m->o, h->d_bas, (const float *)pmo);
    else k_cpl_tau<double><<<gt, 256, 0, h->st>>>(c, m->o, h->d_bas, (const double *)pmo);
    CK(cudaGetLastError());
    // the atmosphere's stream waits for the read of its pressure and, with
    // tau_udiff, for the stress written over the ocean
    CK(cudaEventRecord(m->ev_o, h->st));
    CK(cudaStreamWaitEvent(ha->st, m->ev_o, 0));
    return OQG_OK;
}

int oqg_oml_tau_udiff(oqg_oml *m, int on) {
    if (!m) return fail(OQG_EINVAL, "null argument");
    m->cpl.udiff = on != 0;
    return OQG_OK;
}

int oqg_compute_forcing(oqg_oml *m, const oqg_rad_coeffs *rad) {
    if (!m || !rad) return fail(OQG_EINVAL, "null argument");
    if (!m->am) return fail(OQG_EINVAL, "no atmosphere coupled (oqg_oml_couple)");
    oqg_handle *h = m->h, *ha = m->ha;
    const AmlDev &ao = m->am->o;
    if (ao.nl < 2) return fail(OQG_EUNSUPPORTED, "compute_forcing needs an atmosphere of two or more layers (eta_1)");
    const RadFlux r{rad->fspco, rad->xlamda, rad->d0up, rad->dmdown, rad->dup0, rad->aup00, rad->adown10,
                    rad->adown11};
    // on the ocean's stream, after the atmosphere's queued work; the
    // atmosphere's stream waits for the fluxes (its next step reads fnetat)
    CK(cudaEventRecord(m->ev_a, ha->st));
    CK(cudaStreamWaitEvent(h->st, m->ev_a, 0));
    const void *pma = ha->hb.F[1 - ha->par];
    const int n = m->o.nxt * m->o.nyt + ao.nxt * ao.nyt;
    const int gs = std::min((n + 255) / 256, 148 * 8);
    if (ha->mixed) k_cpl_fluxes<float><<<gs, 256, 0, h->st>>>(m->cpl, r, m->o, ao, (const float *)pma, ha->hb.px);
    else k_cpl_fluxes<double><<<gs, 256, 0, h->st>>>(m->cpl, r, m->o, ao, (const double *)pma, ha->hb.px);
    CK(cudaGetLastError());
    CK(cudaEventRecord(m->ev_o, h->st));
    CK(cudaStreamWaitEvent(ha->st, m->ev_o, 0));
    return OQG_OK;
}

int oqg_get_fluxes(oqg_oml *m, double *fnetoc, double *fnetat) {
    if (!m) return fail(OQG_EINVAL, "null argument");
    if (fnetat && !m->am) return fail(OQG_EINVAL, "no atmosphere coupled (oqg_oml_couple)");
    oqg_handle *h = m->h;
    if (m->am) {
        CK(cudaEventRecord(m->ev_a, m->ha->st));
        CK(cudaStreamWaitEvent(h->st, m->ev_a, 0));
    }
    if (fnetoc)
        CK(cudaMemcpyAsync(fnetoc, m->o.fnet, (size_t)m->o.nxt * m->o.nyt * sizeof(double), cudaMemcpyDefault,
                           h->st));
    if (fnetat) {
        const AmlDev &ao = m->am->o;
        CK(cudaMemcpyAsync(fnetat, ao.fnet, (size_t)ao.nxt * ao.nyt * sizeof(double), cudaMemcpyDefault, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    return OQG_OK;
}

}  // extern "C"
