// oqg_fft.cuh -- shared-memory mixed-radix FFT for the x-transforms.
//
// The x-direction transforms of the Helmholtz inverter (qg/inhomog.F90:170-255;
// FFTW RODFT00 for the closed box, r2c/c2r for the channel) run as complex
// FFTs of length M over rows staged in shared memory.  Two real rows share one
// complex transform (real and imaginary parts).  The algorithm is the Stockham
// autosort FFT (decimation in time, e^{-2 pi i jk/M}), radices 16, 8, 4, 2, 3
// and 5, ping-ponging between two shared buffers of M complex values per
// transform.  A CTA holds G transforms; TT threads serve one transform.  The
// lengths of the configurations' grids run compile-time plans (fft_run).
#pragma once

#include "oqg_dev.cuh"

namespace oqg {

template <class T2> __device__ __forceinline__ T2 c_mul(T2 a, T2 b) {
    T2 r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <class T2> __device__ __forceinline__ T2 c_add(T2 a, T2 b) {
    T2 r; r.x = a.x + b.x; r.y = a.y + b.y; return r;
}
template <class T2> __device__ __forceinline__ T2 c_sub(T2 a, T2 b) {
    T2 r; r.x = a.x - b.x; r.y = a.y - b.y; return r;
}
// -i z
template <class T2> __device__ __forceinline__ T2 c_mi(T2 z) { T2 r; r.x = z.y; r.y = -z.x; return r; }

template <class T> struct FftConst;
template <> struct FftConst<double> {
    static __device__ __forceinline__ double s3() { return 0.86602540378443864676; }
    static __device__ __forceinline__ double h2() { return 0.70710678118654752440; }
    static __device__ __forceinline__ double c51() { return 0.30901699437494742410; }
    static __device__ __forceinline__ double c52() { return -0.80901699437494742410; }
    static __device__ __forceinline__ double s51() { return 0.95105651629515357212; }
    static __device__ __forceinline__ double s52() { return 0.58778525229247312917; }
    static __device__ __forceinline__ double c16() { return 0.92387953251128675613; }
    static __device__ __forceinline__ double s16() { return 0.38268343236508977173; }
};
template <> struct FftConst<float> {
    static __device__ __forceinline__ float s3() { return 0.86602540378443864676f; }
    static __device__ __forceinline__ float h2() { return 0.70710678118654752440f; }
    static __device__ __forceinline__ float c51() { return 0.30901699437494742410f; }
    static __device__ __forceinline__ float c52() { return -0.80901699437494742410f; }
    static __device__ __forceinline__ float s51() { return 0.95105651629515357212f; }
    static __device__ __forceinline__ float s52() { return 0.58778525229247312917f; }
    static __device__ __forceinline__ float c16() { return 0.92387953251128675613f; }
    static __device__ __forceinline__ float s16() { return 0.38268343236508977173f; }
};

// In-register forward DFT of size R.
template <class T, int R> struct Dft;

template <class T> struct Dft<T, 2> {
    typedef typename C2<T>::t T2;
    static __device__ __forceinline__ void run(T2 *v) {
        T2 a = v[0];
        v[0] = c_add(a, v[1]);
        v[1] = c_sub(a, v[1]);
    }
};

template <class T> struct Dft<T, 4> {
    typedef typename C2<T>::t T2;
    static __device__ __forceinline__ void run(T2 *v) {
        T2 t0 = c_add(v[0], v[2]), t1 = c_sub(v[0], v[2]);
        T2 t2 = c_add(v[1], v[3]), t3 = c_mi(c_sub(v[1], v[3]));
        v[0] = c_add(t0, t2);
        v[1] = c_add(t1, t3);
        v[2] = c_sub(t0, t2);
        v[3] = c_sub(t1, t3);
    }
};

template <class T> struct Dft<T, 8> {
    typedef typename C2<T>::t T2;
    static __device__ __forceinline__ void run(T2 *v) {
        T2 e[4] = {v[0], v[2], v[4], v[6]};
        T2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<T, 4>::run(e);
        Dft<T, 4>::run(o);
        const T h = FftConst<T>::h2();
        T2 w1, w3;
        // o1 * (h - i h), o2 * (-i), o3 * (-h - i h)
        w1.x = h * (o[1].x + o[1].y);
        w1.y = h * (o[1].y - o[1].x);
        T2 w2 = c_mi(o[2]);
        w3.x = h * (o[3].y - o[3].x);
        w3.y = -h * (o[3].x + o[3].y);
        v[0] = c_add(e[0], o[0]);
        v[4] = c_sub(e[0], o[0]);
        v[1] = c_add(e[1], w1);
        v[5] = c_sub(e[1], w1);
        v[2] = c_add(e[2], w2);
        v[6] = c_sub(e[2], w2);
        v[3] = c_add(e[3], w3);
        v[7] = c_sub(e[3], w3);
    }
};

template <class T> struct Dft<T, 3> {
    typedef typename C2<T>::t T2;
    static __device__ __forceinline__ void run(T2 *v) {
        const T s3 = FftConst<T>::s3();
        T2 s = c_add(v[1], v[2]), d = c_sub(v[1], v[2]);
        T2 m;
        m.x = v[0].x - T(0.5) * s.x;
        m.y = v[0].y - T(0.5) * s.y;
        T2 jd;  // -i s3 d
        jd.x = s3 * d.y;
        jd.y = -s3 * d.x;
        v[0] = c_add(v[0], s);
        v[1] = c_add(m, jd);
        v[2] = c_sub(m, jd);
    }
};

template <class T> struct Dft<T, 5> {
    typedef typename C2<T>::t T2;
    static __device__ __forceinline__ void run(T2 *v) {
        const T c1 = FftConst<T>::c51(), c2 = FftConst<T>::c52();
        const T s1 = FftConst<T>::s51(), s2 = FftConst<T>::s52();
        T2 t1 = c_add(v[1], v[4]), t2 = c_add(v[2], v[3]);
        T2 t3 = c_sub(v[1], v[4]), t4 = c_sub(v[2], v[3]);
        T2 a, bq, u, w;
        a.x = v[0].x + c1 * t1.x + c2 * t2.x;
        a.y = v[0].y + c1 * t1.y + c2 * t2.y;
        bq.x = v[0].x + c2 * t1.x + c1 * t2.x;
        bq.y = v[0].y + c2 * t1.y + c1 * t2.y;
        u.x = s1 * t3.x + s2 * t4.x;      // (s1 t3 + s2 t4)
        u.y = s1 * t3.y + s2 * t4.y;
        w.x = s2 * t3.x - s1 * t4.x;      // (s2 t3 - s1 t4)
        w.y = s2 * t3.y - s1 * t4.y;
        v[0].x = v[0].x + t1.x + t2.x;
        v[0].y = v[0].y + t1.y + t2.y;
        v[1] = c_add(a, c_mi(u));
        v[4] = c_sub(a, c_mi(u));
        v[2] = c_add(bq, c_mi(w));
        v[3] = c_sub(bq, c_mi(w));
    }
};

// 16-point DFT as 4 x 4 (decimation in time, n = 4 n1 + n2, k = k1 + 4 k2):
// length-4 DFTs over n1, the twiddles W16^(n2 k1), length-4 DFTs over n2.
template <class T> struct Dft<T, 16> {
    typedef typename C2<T>::t T2;
    // z * W16^e for the e the 4 x 4 split needs: W16^e = exp(-2 pi i e / 16)
    template <int E> static __device__ __forceinline__ T2 w16(T2 z) {
        const T c = FftConst<T>::c16(), s = FftConst<T>::s16(), h = FftConst<T>::h2();
        T2 r;
        if (E == 1) { r.x = c * z.x + s * z.y; r.y = c * z.y - s * z.x; }          // (c - i s)
        else if (E == 2) { r.x = h * (z.x + z.y); r.y = h * (z.y - z.x); }          // (h - i h)
        else if (E == 3) { r.x = s * z.x + c * z.y; r.y = s * z.y - c * z.x; }      // (s - i c)
        else if (E == 6) { r.x = h * (z.y - z.x); r.y = -h * (z.x + z.y); }         // (-h - i h)
        else { r.x = -(c * z.x + s * z.y); r.y = s * z.x - c * z.y; }               // E == 9: (-c + i s)
        return r;
    }
    static __device__ __forceinline__ void run(T2 *v) {
        T2 a[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            T2 t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
            Dft<T, 4>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
        }
        a[1][1] = w16<1>(a[1][1]);
        a[1][2] = w16<2>(a[1][2]);
        a[1][3] = w16<3>(a[1][3]);
        a[2][1] = w16<2>(a[2][1]);
        a[2][2] = c_mi(a[2][2]);
        a[2][3] = w16<6>(a[2][3]);
        a[3][1] = w16<3>(a[3][1]);
        a[3][2] = w16<6>(a[3][2]);
        a[3][3] = w16<9>(a[3][3]);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            T2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
            Dft<T, 4>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
        }
    }
};

// Shared work buffers hold element i at fpad(i) = i + i/8: with one pad per 8
// complex values the stride-R stores of the early Stockham stages and the
// unit-stride loads both spread over all banks.
__device__ __forceinline__ int fpad(int i) { return i + (i >> 3); }
__host__ __device__ __forceinline__ int fft_buf_len(int M) { return M + (M >> 3) + 4; }
// fpad(i + r S) for a compile-time stride S: when S is a multiple of 8 the
// pad of i + r S is the pad of i plus r S / 8, so the index is affine in r
// (one address per butterfly, constant offsets for its R values).
template <int S> __device__ __forceinline__ int fpad_step(int i, int r) {
    if constexpr (S % 8 == 0) return fpad(i) + r * (S + S / 8);
    else return fpad(i + r * S);
}

// One Stockham stage of radix R: src -> dst (both shared, padded, length M).
// Threads t < TT of the transform's group each take butterflies t, t+TT, ...
// tws: this stage's twiddles in global memory (read through L1), entry
// (r - 1) Ns + jm = exp(-2 pi i r jm / (Ns R)).  lg = log2(Ns) when Ns is a
// power of two (a shift), else -1 (fd divides by Ns).
template <class T, int R>
__device__ __forceinline__ void fft_stage(const typename C2<T>::t *__restrict__ src,
                                          typename C2<T>::t *__restrict__ dst, int M, int Ns, int lg,
                                          FastDiv fd, const typename C2<T>::t *__restrict__ tws, int t,
                                          int TT) {
    typedef typename C2<T>::t T2;
    const int nb = M / R;
    for (int j = t; j < nb; j += TT) {
        const int q = lg >= 0 ? (j >> lg) : fd.div(j), jm = j - q * Ns;
        T2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[fpad(j + r * nb)];
        if (jm != 0) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = c_mul(v[r], __ldg(tws + (r - 1) * Ns + jm));
        }
        Dft<T, R>::run(v);
        const int d = q * Ns * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[fpad(d + r * Ns)] = v[r];
    }
}

// The radix-3 and radix-5 stages out of line: most transform lengths are
// powers of two, and keeping these stages out of the hot loop's code leaves
// more of the instruction cache to it.
template <class T, int R>
__device__ __noinline__ void fft_stage_cold(const typename C2<T>::t *__restrict__ src,
                                            typename C2<T>::t *__restrict__ dst, int M, int Ns, int lg,
                                            FastDiv fd, const typename C2<T>::t *__restrict__ tws, int t,
                                            int TT) {
    fft_stage<T, R>(src, dst, M, Ns, lg, fd, tws, t, TT);
}

// Barrier `id` over the first `n` threads of the CTA (n a multiple of 32);
// n = 0: all threads of the CTA (__syncthreads).
__device__ __forceinline__ void bar_sync(int id, int n) {
    if (n == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Forward FFT of length M (radices rad[0..nrad)) from padded buffer a, using
// padded buffer b as the second buffer of the ping-pong.  Returns the buffer
// holding the result.  tw: the per-stage twiddle tables (global memory; the
// stage after Ns starts at entry Ns - 1).  The nbar threads that synchronise
// on barrier bar_id must all call it; threads with t >= TT only take part in
// the barriers.
template <class T>
__device__ typename C2<T>::t *fft_smem(typename C2<T>::t *a, typename C2<T>::t *b, int M,
                                       const int *rad, int nrad,
                                       const typename C2<T>::t *__restrict__ tw, int t, int TT,
                                       int bar_id, int nbar) {
    typedef typename C2<T>::t T2;
    T2 *src = a, *dst = b;
    int Ns = 1;
    for (int s = 0; s < nrad; ++s) {
        const int R = rad[s];
        const int lg = (Ns & (Ns - 1)) == 0 ? __ffs(Ns) - 1 : -1;
        const T2 *tws = tw + (Ns - 1);
        FastDiv fd;
        if (lg < 0) fd = FastDiv(Ns);
        switch (R) {
            case 16: fft_stage<T, 16>(src, dst, M, Ns, lg, fd, tws, t, TT); break;
            case 8: fft_stage<T, 8>(src, dst, M, Ns, lg, fd, tws, t, TT); break;
            case 4: fft_stage<T, 4>(src, dst, M, Ns, lg, fd, tws, t, TT); break;
            case 2: fft_stage<T, 2>(src, dst, M, Ns, lg, fd, tws, t, TT); break;
            case 3: fft_stage_cold<T, 3>(src, dst, M, Ns, lg, fd, tws, t, TT); break;
            default: fft_stage_cold<T, 5>(src, dst, M, Ns, lg, fd, tws, t, TT); break;
        }
        bar_sync(bar_id, nbar);
        T2 *x = src; src = dst; dst = x;
        Ns *= R;
    }
    return src;
}

// ---- compile-time plans for the common transform lengths.  The radix after
// span Ns of a length-M transform follows the host's fft_radices rule
// (16 while it divides, then 8, 4, 2, then 3 and 5), so the per-stage
// twiddle tables are the same for both paths.
__host__ __device__ constexpr int fft_next_radix(int rem) {
    return rem % 16 == 0 ? 16 : rem % 8 == 0 ? 8 : rem % 4 == 0 ? 4 : rem % 2 == 0 ? 2
         : rem % 3 == 0 ? 3 : rem % 5 == 0 ? 5 : 0;
}

// One Stockham stage with every size known at compile time: the loop over
// a thread's butterflies unrolls and the index arithmetic folds to shifts
// and constants.
template <class T, int R, int Ns, int M, int TT>
__device__ __forceinline__ void fft_stage_ct(const typename C2<T>::t *__restrict__ src,
                                             typename C2<T>::t *__restrict__ dst,
                                             const typename C2<T>::t *__restrict__ tws, int t) {
    typedef typename C2<T>::t T2;
    constexpr int nb = M / R;
#pragma unroll
    for (int j0 = 0; j0 < nb; j0 += TT) {
        const int j = j0 + t;
        if (nb % TT == 0 || j < nb) {
            const int q = j / Ns, jm = j - q * Ns;
            T2 v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = src[fpad_step<nb>(j, r)];
            if (Ns > 1 && jm != 0) {
#pragma unroll
                for (int r = 1; r < R; ++r) v[r] = c_mul(v[r], __ldg(tws + (r - 1) * Ns + jm));
            }
            Dft<T, R>::run(v);
            const int d = q * Ns * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) dst[fpad_step<Ns>(d, r)] = v[r];
        }
    }
}

// The stages from span Ns on; returns the buffer holding the result.  Threads
// with live = false only take part in the barriers.
template <class T, int M, int TT, int Ns>
__device__ __forceinline__ typename C2<T>::t *fft_ct_from(typename C2<T>::t *src, typename C2<T>::t *dst,
                                                         const typename C2<T>::t *__restrict__ tw, int t,
                                                         bool live, int bar_id, int nbar) {
    if constexpr (Ns >= M) {
        return src;
    } else {
        constexpr int R = fft_next_radix(M / Ns);
        static_assert(R > 1, "transform length must factor into 2, 3 and 5");
        if (live) fft_stage_ct<T, R, Ns, M, TT>(src, dst, tw + (Ns - 1), t);
        bar_sync(bar_id, nbar);
        return fft_ct_from<T, M, TT, Ns * R>(dst, src, tw, t, live, bar_id, nbar);
    }
}

// ---- in-place stages for the long power-of-two lengths: one padded buffer
// per transform, so two transforms of 4096 FP64 values fit where the
// ping-pong pair fits one.  Each thread holds the inputs of all its
// butterflies in registers (E = M / TT values, E a multiple of every radix of
// the plan), the group synchronises, then the thread computes and stores.
template <class T, int R, int Ns, int M, int TT>
__device__ __forceinline__ void fft_stage_ip(typename C2<T>::t *buf, const typename C2<T>::t *__restrict__ tws,
                                             int t, bool live, int bar_id, int nbar) {
    typedef typename C2<T>::t T2;
    constexpr int nb = M / R, NB = nb / TT;
    static_assert(nb % TT == 0, "in-place stages need whole butterflies per thread");
    T2 v[NB][R];
    if (live) {
#pragma unroll
        for (int u = 0; u < NB; ++u)
#pragma unroll
            for (int r = 0; r < R; ++r) v[u][r] = buf[fpad_step<nb>(t + u * TT, r)];
    }
    bar_sync(bar_id, nbar);
    if (live) {
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            const int j = t + u * TT;
            const int q = j / Ns, jm = j - q * Ns;
            if (Ns > 1 && jm != 0) {
#pragma unroll
                for (int r = 1; r < R; ++r) v[u][r] = c_mul(v[u][r], __ldg(tws + (r - 1) * Ns + jm));
            }
            Dft<T, R>::run(v[u]);
            const int d = q * Ns * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[fpad_step<Ns>(d, r)] = v[u][r];
        }
    }
    bar_sync(bar_id, nbar);
}
template <class T, int M, int TT, int Ns>
__device__ __forceinline__ void fft_ip_from(typename C2<T>::t *buf, const typename C2<T>::t *__restrict__ tw, int t,
                                            bool live, int bar_id, int nbar) {
    if constexpr (Ns < M) {
        constexpr int R = fft_next_radix(M / Ns);
        fft_stage_ip<T, R, Ns, M, TT>(buf, tw + (Ns - 1), t, live, bar_id, nbar);
        fft_ip_from<T, M, TT, Ns * R>(buf, tw, t, live, bar_id, nbar);
    }
}
// The lengths that transform in place (16 values per thread).
__host__ __device__ constexpr bool fft_inplace_len(int M) { return M == 2048 || M == 4096; }
// In-place forward FFT of length M (fft_inplace_len) by groups of TT = M / 16
// threads (t >= TT: barriers only); the input is in buf, the barrier after
// its writes taken.
// MC > 0: the kernel is built for that one length, and only its plan is
// compiled.
template <class T, int MC = 0>
__device__ __forceinline__ void fft_inplace(typename C2<T>::t *buf, int M, const typename C2<T>::t *__restrict__ tw,
                                            int t, int bar_id, int nbar) {
    if constexpr (MC == 2048 || MC == 4096) {
        fft_ip_from<T, MC, MC / 16, 1>(buf, tw, t, t < MC / 16, bar_id, nbar);
    } else if constexpr (MC == 0) {
        if (M == 2048) fft_ip_from<T, 2048, 128, 1>(buf, tw, t, t < 128, bar_id, nbar);
        else if (M == 4096) fft_ip_from<T, 4096, 256, 1>(buf, tw, t, t < 256, bar_id, nbar);
    }
}

// Forward FFT of length M by groups of TT = M / E threads: the compile-time
// stages for the lengths of the configurations' grids, the general stages
// otherwise.  Same contract as fft_smem (t >= TT: barriers only).  MC > 0:
// the kernel is built for that one length (M == MC), and only its plan is
// compiled, which keeps the kernel's code within the instruction cache.
#define OQG_FFT_CT(MM)                                                                                      \
    case MM:                                                                                                \
        if constexpr ((MM) % E == 0) return fft_ct_from<T, MM, (MM) / E, 1>(a, b, tw, t, t < TT, bar_id, nbar); \
        break;
template <class T, int E, int MC = 0>
__device__ __forceinline__ typename C2<T>::t *fft_run(typename C2<T>::t *a, typename C2<T>::t *b, int M,
                                                      const int *rad, int nrad,
                                                      const typename C2<T>::t *__restrict__ tw, int t, int TT,
                                                      int bar_id, int nbar) {
    if constexpr (MC > 0 && MC % E == 0) {
        return fft_ct_from<T, MC, MC / E, 1>(a, b, tw, t, t < TT, bar_id, nbar);
    } else {
        switch (M) {
            OQG_FFT_CT(128)
            OQG_FFT_CT(192)
            OQG_FFT_CT(256)
            OQG_FFT_CT(384)
            OQG_FFT_CT(512)
            OQG_FFT_CT(1024)
            OQG_FFT_CT(2048)
            OQG_FFT_CT(4096)
            default: break;
        }
        return fft_smem<T>(a, b, M, rad, nrad, tw, t, TT, bar_id, nbar);
    }
}
#undef OQG_FFT_CT

// 16-byte cp.async of n bytes (n a multiple of 16, both addresses 16-byte
// aligned) by threads t < TT.
__device__ __forceinline__ void cp_async_16(void *dst, const void *src, int nbytes, int t, int TT) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    const char *g = (const char *)src;
    for (int o = t * 16; o < nbytes; o += TT * 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa + o), "l"(g + o) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

}  // namespace oqg
