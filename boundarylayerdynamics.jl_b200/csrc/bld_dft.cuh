// Register DFT codelets of size N in {2,3,4,5,6,7,8,9,10,12,14,15,16,18,24,32}.
//
// dft<R, N, DIR>(x) transforms x[0..N) in place (registers, compile-time
// indices after unrolling): X[k] = sum_n x[n] exp(DIR * 2 pi i n k / N).
// Composite sizes split N = Rr * M (Rr = 4, 2 or 3; decimation in time): M-point
// DFTs of the Rr interleaved subsequences, twiddles W_N^(r k'), then Rr-point
// DFTs.  The odd primes 5 and 7 pair x[k] with x[N - k]: with s_k = x[k] +
// x[N - k] and d_k = x[k] - x[N - k], X[m] = x[0] + sum_k cos(2 pi k m / N) s_k
// + i DIR sum_k sin(2 pi k m / N) d_k and X[N - m] the same with -i.  The twiddles W_N^m of every codelet size live in one small table
// (constant memory on the device, a host array in host builds) filled from
// long-double cos/sin on the host.
#pragma once

#include <cuda_runtime.h>

#include "bld_fft.cuh"

#define BLD_WTAB_SIZE 176

// largest codelets compiled for double and single precision (register budget)
#ifndef BLD_FP64_MAXR
#define BLD_FP64_MAXR 18
#endif
#ifndef BLD_FP32_MAXR
#define BLD_FP32_MAXR 18
#endif

// offsets of W_N (m = 0..N-1) in the twiddle table
__host__ __device__ constexpr int woff(int N) {
    return N == 6 ? 0 : N == 8 ? 6 : N == 9 ? 14 : N == 12 ? 23 : N == 16 ? 35 : N == 18 ? 51 : N == 24 ? 69
         : N == 32 ? 93 : N == 5 ? 125 : N == 7 ? 130 : N == 10 ? 137 : N == 14 ? 147 : N == 15 ? 161 : -1;
}
__host__ __device__ constexpr bool codelet_size(int N) {
    return N == 2 || N == 3 || N == 4 || N == 5 || N == 6 || N == 7 || N == 8 || N == 9 || N == 10 || N == 12 ||
           N == 14 || N == 15 || N == 16 || N == 18 || N == 24 || N == 32;
}

#ifdef __CUDACC__
__constant__ double2 c_wtab64[BLD_WTAB_SIZE];
__constant__ float2 c_wtab32[BLD_WTAB_SIZE];
#endif
extern double2 h_wtab64[BLD_WTAB_SIZE];
extern float2 h_wtab32[BLD_WTAB_SIZE];

template <typename R> __host__ __device__ __forceinline__ cplx<R> wtab(int i);
template <> __host__ __device__ __forceinline__ double2 wtab<double>(int i) {
#ifdef __CUDA_ARCH__
    return c_wtab64[i];
#else
    return h_wtab64[i];
#endif
}
template <> __host__ __device__ __forceinline__ float2 wtab<float>(int i) {
#ifdef __CUDA_ARCH__
    return c_wtab32[i];
#else
    return h_wtab32[i];
#endif
}

template <typename R> __host__ __device__ __forceinline__ R hsin60() { return R(0.86602540378443864676); }

template <typename C>
__host__ __device__ __forceinline__ C c_add(C a, C b) {
    C r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}
template <typename C>
__host__ __device__ __forceinline__ C c_sub(C a, C b) {
    C r;
    r.x = a.x - b.x;
    r.y = a.y - b.y;
    return r;
}
// x * w for DIR < 0, x * conj(w) for DIR > 0
template <int DIR, typename C>
__host__ __device__ __forceinline__ C c_tw(C x, C w) {
    C r;
    if (DIR < 0) {
        r.x = x.x * w.x - x.y * w.y;
        r.y = x.x * w.y + x.y * w.x;
    } else {
        r.x = x.x * w.x + x.y * w.y;
        r.y = x.y * w.x - x.x * w.y;
    }
    return r;
}

template <typename R, int N, int DIR>
__host__ __device__ __forceinline__ void dft(cplx<R> (&x)[N]) {
    using C = cplx<R>;
    if constexpr (N == 1) {
        return;
    } else if constexpr (N == 2) {
        const C a = x[0], b = x[1];
        x[0] = c_add(a, b);
        x[1] = c_sub(a, b);
    } else if constexpr (N == 3) {
        const C s = c_add(x[1], x[2]);
        const C d = c_sub(x[1], x[2]);
        C m = x[0];
        m.x -= R(0.5) * s.x;
        m.y -= R(0.5) * s.y;
        C t;
        t.x = -d.y * hsin60<R>();
        t.y = d.x * hsin60<R>();
        x[0] = c_add(x[0], s);
        if (DIR < 0) {
            x[1] = c_sub(m, t);
            x[2] = c_add(m, t);
        } else {
            x[1] = c_add(m, t);
            x[2] = c_sub(m, t);
        }
    } else if constexpr (N == 4) {
        const C a0 = c_add(x[0], x[2]), a1 = c_sub(x[0], x[2]);
        const C a2 = c_add(x[1], x[3]);
        const C d = c_sub(x[1], x[3]);
        C a3;
        a3.x = -d.y;
        a3.y = d.x;  // i (x1 - x3)
        x[0] = c_add(a0, a2);
        x[2] = c_sub(a0, a2);
        if (DIR < 0) {
            x[1] = c_sub(a1, a3);
            x[3] = c_add(a1, a3);
        } else {
            x[1] = c_add(a1, a3);
            x[3] = c_sub(a1, a3);
        }
    } else if constexpr (N == 5 || N == 7) {
        constexpr int H = (N - 1) / 2;
        C sp[H], dm[H];
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            sp[k - 1] = c_add(x[k], x[N - k]);
            dm[k - 1] = c_sub(x[k], x[N - k]);
        }
        const C x0 = x[0];
        C sum = x0;
#pragma unroll
        for (int k = 0; k < H; ++k) sum = c_add(sum, sp[k]);
#pragma unroll
        for (int m = 1; m <= H; ++m) {
            C a = x0, b;
            b.x = R(0);
            b.y = R(0);
#pragma unroll
            for (int k = 1; k <= H; ++k) {
                // W_N^(m k) = (cos, -sin) of 2 pi (m k mod N) / N
                const C w = wtab<R>(woff(N) + (m * k) % N);
                a.x += w.x * sp[k - 1].x;
                a.y += w.x * sp[k - 1].y;
                b.x -= w.y * dm[k - 1].x;
                b.y -= w.y * dm[k - 1].y;
            }
            C ib;   // i b
            ib.x = -b.y;
            ib.y = b.x;
            if (DIR > 0) {
                x[m] = c_add(a, ib);
                x[N - m] = c_sub(a, ib);
            } else {
                x[m] = c_sub(a, ib);
                x[N - m] = c_add(a, ib);
            }
        }
        x[0] = sum;
    } else {
        constexpr int Rr = (N % 4 == 0) ? 4 : (N % 2 == 0) ? 2 : 3;
        constexpr int M = N / Rr;
        C sub[Rr][M];
#pragma unroll
        for (int r = 0; r < Rr; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) sub[r][m] = x[m * Rr + r];
#pragma unroll
        for (int r = 0; r < Rr; ++r) dft<R, M, DIR>(sub[r]);
#pragma unroll
        for (int r = 1; r < Rr; ++r)
#pragma unroll
            for (int k = 1; k < M; ++k) sub[r][k] = c_tw<DIR>(sub[r][k], wtab<R>(woff(N) + r * k));
#pragma unroll
        for (int k = 0; k < M; ++k) {
            C t[Rr];
#pragma unroll
            for (int r = 0; r < Rr; ++r) t[r] = sub[r][k];
            dft<R, Rr, DIR>(t);
#pragma unroll
            for (int q = 0; q < Rr; ++q) x[k + M * q] = t[q];
        }
    }
}

// One Stockham stage of radix RAD over `nlines` lines of length n (element p of
// line l at base[l*ls + p*ps]); Ns = product of the radices of earlier stages.
template <typename R, int DIR, int RAD>
__device__ __forceinline__ void stockham_stage(const cplx<R>* src, cplx<R>* dst, int n, int Ns, int nlines, int ls,
                                               int ps, bool pos_fastest, const cplx<R>* __restrict__ tw) {
    using C = cplx<R>;
    const int nb = n / RAD;
    const int total = nb * nlines;
    const int tws = n / (Ns * RAD);
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        int j, l;
        if (pos_fastest) {
            l = w / nb;
            j = w - l * nb;
        } else {
            j = w / nlines;
            l = w - j * nlines;
        }
        const int k = j % Ns;
        const C* in = src + l * ls;
        C* out = dst + l * ls;
        C x[RAD];
#pragma unroll
        for (int t = 0; t < RAD; ++t) x[t] = in[(j + t * nb) * ps];
        if (k) {
#pragma unroll
            for (int t = 1; t < RAD; ++t) x[t] = c_tw<DIR>(x[t], tw[k * t * tws]);
        }
        dft<R, RAD, DIR>(x);
        const int od = (j - k) * RAD + k;
#pragma unroll
        for (int q = 0; q < RAD; ++q) out[(od + q * Ns) * ps] = x[q];
    }
}

// Mixed-radix Stockham FFT with register codelets; same contract as fft_run.
template <typename R, int DIR>
__device__ __forceinline__ cplx<R>* fft_big(cplx<R>* a, cplx<R>* b, int nlines, int ls, int ps, bool pos_fastest, const FftPlan& pl,
                            const cplx<R>* __restrict__ tw) {
    using C = cplx<R>;
    const int n = pl.n;
    int Ns = 1;
    C* src = a;
    C* dst = b;
    for (int s = 0; s < pl.nst; ++s) {
        const int r = pl.radix[s];
        constexpr int MAXR = sizeof(R) == 4 ? BLD_FP32_MAXR : BLD_FP64_MAXR;
        switch (r) {
            case 2: stockham_stage<R, DIR, 2>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 3: stockham_stage<R, DIR, 3>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 4: stockham_stage<R, DIR, 4>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 6: stockham_stage<R, DIR, 6>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 8: stockham_stage<R, DIR, 8>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 5: stockham_stage<R, DIR, 5>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 7: stockham_stage<R, DIR, 7>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 10: stockham_stage<R, DIR, 10>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 14: stockham_stage<R, DIR, 14>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 15: stockham_stage<R, DIR, 15>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 9:
                if constexpr (MAXR >= 9) stockham_stage<R, DIR, 9>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw);
                break;
            case 12:
                if constexpr (MAXR >= 12) stockham_stage<R, DIR, 12>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw);
                break;
            case 16:
                if constexpr (MAXR >= 16) stockham_stage<R, DIR, 16>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw);
                break;
            case 18:
                if constexpr (MAXR >= 18) stockham_stage<R, DIR, 18>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw);
                break;
            case 24:
                if constexpr (MAXR >= 24) stockham_stage<R, DIR, 24>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw);
                break;
            default:
                if constexpr (MAXR >= 32) stockham_stage<R, DIR, 32>(src, dst, n, Ns, nlines, ls, ps, pos_fastest, tw);
                break;
        }
        __syncthreads();
        C* t = src;
        src = dst;
        dst = t;
        Ns *= r;
    }
    return src;
}

// In-place Stockham stages: every task reads its RAD inputs into registers, the
// block synchronises, then every task writes its RAD outputs into the same
// buffer.  A thread holds up to inplace_tpt(RAD) tasks (4 for radix <= 4, 3 for
// radix 6, else 1), so nlines * n / RAD <= inplace_tpt(RAD) * blockDim.x.  The
// barriers sit outside the radix switch (one register array spans both halves).
__host__ __device__ constexpr int inplace_tpt(int rad) { return rad <= 4 ? 4 : (rad == 6 ? 3 : 1); }

template <typename R> struct InplaceMax;
template <> struct InplaceMax<double> { static constexpr int X = 18; };
template <> struct InplaceMax<float> { static constexpr int X = BLD_FP32_MAXR > 18 ? BLD_FP32_MAXR : 18; };

__device__ __forceinline__ void inplace_task(int w, int nb, int nlines, bool pos_fastest, int& j, int& l) {
    if (pos_fastest) {
        l = w / nb;
        j = w - l * nb;
    } else {
        j = w / nlines;
        l = w - j * nlines;
    }
}

template <typename R, int RAD>
__device__ __forceinline__ void inplace_load(cplx<R> (&x)[InplaceMax<R>::X], const cplx<R>* buf, int n, int nlines,
                                             int ls, int ps, bool pos_fastest) {
    constexpr int TPT = inplace_tpt(RAD);
    static_assert(TPT * RAD <= InplaceMax<R>::X, "register array too small");
    const int nb = n / RAD, total = nb * nlines;
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
        const int w = threadIdx.x + u * blockDim.x;
        if (w < total) {
            int j, l;
            inplace_task(w, nb, nlines, pos_fastest, j, l);
            const cplx<R>* in = buf + l * ls;
#pragma unroll
            for (int t = 0; t < RAD; ++t) x[u * RAD + t] = in[(j + t * nb) * ps];
        }
    }
}

template <typename R, int DIR, int RAD>
__device__ __forceinline__ void inplace_store(cplx<R> (&x)[InplaceMax<R>::X], cplx<R>* buf, int n, int Ns, int nlines,
                                              int ls, int ps, bool pos_fastest, const cplx<R>* __restrict__ tw) {
    using C = cplx<R>;
    constexpr int TPT = inplace_tpt(RAD);
    const int nb = n / RAD, total = nb * nlines;
    const int tws = n / (Ns * RAD);
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
        const int w = threadIdx.x + u * blockDim.x;
        if (w < total) {
            int j, l;
            inplace_task(w, nb, nlines, pos_fastest, j, l);
            const int k = j % Ns;
            C(&y)[RAD] = *reinterpret_cast<C(*)[RAD]>(&x[u * RAD]);  // task u's slice, no copy
            if (k) {
#pragma unroll
                for (int t = 1; t < RAD; ++t) y[t] = c_tw<DIR>(y[t], tw[k * t * tws]);
            }
            dft<R, RAD, DIR>(y);
            const int od = (j - k) * RAD + k;
            C* out = buf + l * ls;
#pragma unroll
            for (int q = 0; q < RAD; ++q) out[(od + q * Ns) * ps] = y[q];
        }
    }
}

// In-place mixed-radix FFT of `nlines` lines in `buf` (result in buf); all
// threads must call it after a __syncthreads() that publishes buf.
template <typename R, int DIR>
__device__ __forceinline__ void fft_inplace(cplx<R>* buf, int nlines, int ls, int ps, bool pos_fastest,
                                            const FftPlan& pl, const cplx<R>* __restrict__ tw) {
    using C = cplx<R>;
    const int n = pl.n;
    int Ns = 1;
    constexpr int MAXR = sizeof(R) == 4 ? BLD_FP32_MAXR : BLD_FP64_MAXR;
    C x[InplaceMax<R>::X];
    for (int s = 0; s < pl.nst; ++s) {
        const int r = pl.radix[s];
        switch (r) {
            case 2: inplace_load<R, 2>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 3: inplace_load<R, 3>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 4: inplace_load<R, 4>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 6: inplace_load<R, 6>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 8: inplace_load<R, 8>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 5: inplace_load<R, 5>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 7: inplace_load<R, 7>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 10: inplace_load<R, 10>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 14: inplace_load<R, 14>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 15: inplace_load<R, 15>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 9: if constexpr (MAXR >= 9) inplace_load<R, 9>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 12: if constexpr (MAXR >= 12) inplace_load<R, 12>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 16: if constexpr (MAXR >= 16) inplace_load<R, 16>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 18: if constexpr (MAXR >= 18) inplace_load<R, 18>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            case 24: if constexpr (MAXR >= 24) inplace_load<R, 24>(x, buf, n, nlines, ls, ps, pos_fastest); break;
            default: if constexpr (MAXR >= 32) inplace_load<R, 32>(x, buf, n, nlines, ls, ps, pos_fastest); break;
        }
        __syncthreads();
        switch (r) {
            case 2: inplace_store<R, DIR, 2>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 3: inplace_store<R, DIR, 3>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 4: inplace_store<R, DIR, 4>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 6: inplace_store<R, DIR, 6>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 8: inplace_store<R, DIR, 8>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 5: inplace_store<R, DIR, 5>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 7: inplace_store<R, DIR, 7>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 10: inplace_store<R, DIR, 10>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 14: inplace_store<R, DIR, 14>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 15: inplace_store<R, DIR, 15>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 9: if constexpr (MAXR >= 9) inplace_store<R, DIR, 9>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 12: if constexpr (MAXR >= 12) inplace_store<R, DIR, 12>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 16: if constexpr (MAXR >= 16) inplace_store<R, DIR, 16>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 18: if constexpr (MAXR >= 18) inplace_store<R, DIR, 18>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            case 24: if constexpr (MAXR >= 24) inplace_store<R, DIR, 24>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
            default: if constexpr (MAXR >= 32) inplace_store<R, DIR, 32>(x, buf, n, Ns, nlines, ls, ps, pos_fastest, tw); break;
        }
        __syncthreads();
        Ns *= r;
    }
}
