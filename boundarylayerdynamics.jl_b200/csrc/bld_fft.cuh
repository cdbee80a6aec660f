// Shared-memory mixed-radix (4, 2, 3) Stockham FFT for batches of lines.
//
// Replaces the FFTW plans of Transform2D (src/physical_space.jl:9-22), which
// the reference executes one z layer at a time (src/physical_space.jl:222,293).
// A thread block transforms `nlines` lines of length n held in shared memory;
// element p of line l sits at buf[l*ls + p*ps].  Each stage reads one buffer
// and writes the other (autosort, natural order out), so the caller provides
// a scratch buffer of the same extent and gets back the buffer holding the
// result.  Twiddles come from a table W[m] = exp(-2*pi*i*m/n) computed on the
// host in long double; the inverse direction uses conj(W).
#pragma once

#include <cuda_runtime.h>

#define BLD_MAX_STAGES 12

struct FftPlan {
    int n;
    int nst;
    int radix[BLD_MAX_STAGES];
};

template <typename R> struct CplxOf;
template <> struct CplxOf<double> { using T = double2; };
template <> struct CplxOf<float> { using T = float2; };
template <typename R> using cplx = typename CplxOf<R>::T;

template <typename R>
__device__ __forceinline__ cplx<R> mk(R a, R b) {
    cplx<R> c;
    c.x = a;
    c.y = b;
    return c;
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
    a.x += b.x;
    a.y += b.y;
    return a;
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
    a.x -= b.x;
    a.y -= b.y;
    return a;
}
// x * w (DIR = -1) or x * conj(w) (DIR = +1)
template <int DIR, typename C>
__device__ __forceinline__ C twmul(C x, C w) {
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
// i * x
template <typename C>
__device__ __forceinline__ C imul(C x) {
    C r;
    r.x = -x.y;
    r.y = x.x;
    return r;
}

// sin(2*pi/3) rounded to the nearest double / float
template <typename R> __device__ __forceinline__ R sin60();
template <> __device__ __forceinline__ double sin60<double>() { return 0.86602540378443864676; }
template <> __device__ __forceinline__ float sin60<float>() { return 0.866025403784438646f; }

// Runs the FFT; all threads of the block must call it after a __syncthreads()
// that makes `a` visible.  Returns the buffer that holds the result (a or b);
// ends with a __syncthreads().
template <typename R, int DIR>
__device__ cplx<R>* fft_run(cplx<R>* a, cplx<R>* b, int nlines, int ls, int ps, bool pos_fastest,
                            const FftPlan& pl, const cplx<R>* __restrict__ tw) {
    using C = cplx<R>;
    const int n = pl.n;
    int Ns = 1;
    C* src = a;
    C* dst = b;
    for (int s = 0; s < pl.nst; ++s) {
        const int r = pl.radix[s];
        const int nb = n / r;
        const int total = nb * nlines;
        const int tws = n / (Ns * r);
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
            const int od = (j - k) * r + k;
            if (r == 4) {
                C x0 = in[j * ps], x1 = in[(j + nb) * ps], x2 = in[(j + 2 * nb) * ps], x3 = in[(j + 3 * nb) * ps];
                if (k) {
                    x1 = twmul<DIR>(x1, tw[k * tws]);
                    x2 = twmul<DIR>(x2, tw[2 * k * tws]);
                    x3 = twmul<DIR>(x3, tw[3 * k * tws]);
                }
                const C a0 = cadd(x0, x2), a1 = csub(x0, x2), a2 = cadd(x1, x3), a3 = imul(csub(x1, x3));
                out[od * ps] = cadd(a0, a2);
                out[(od + 2 * Ns) * ps] = csub(a0, a2);
                if (DIR < 0) {
                    out[(od + Ns) * ps] = csub(a1, a3);
                    out[(od + 3 * Ns) * ps] = cadd(a1, a3);
                } else {
                    out[(od + Ns) * ps] = cadd(a1, a3);
                    out[(od + 3 * Ns) * ps] = csub(a1, a3);
                }
            } else if (r == 2) {
                C x0 = in[j * ps], x1 = in[(j + nb) * ps];
                if (k) x1 = twmul<DIR>(x1, tw[k * tws]);
                out[od * ps] = cadd(x0, x1);
                out[(od + Ns) * ps] = csub(x0, x1);
            } else {  // r == 3
                C x0 = in[j * ps], x1 = in[(j + nb) * ps], x2 = in[(j + 2 * nb) * ps];
                if (k) {
                    x1 = twmul<DIR>(x1, tw[k * tws]);
                    x2 = twmul<DIR>(x2, tw[2 * k * tws]);
                }
                const C s12 = cadd(x1, x2);
                const C d12 = csub(x1, x2);
                C m = x0;
                m.x -= R(0.5) * s12.x;
                m.y -= R(0.5) * s12.y;
                C t = imul(d12);
                t.x *= sin60<R>();
                t.y *= sin60<R>();
                out[od * ps] = cadd(x0, s12);
                if (DIR < 0) {
                    out[(od + Ns) * ps] = csub(m, t);
                    out[(od + 2 * Ns) * ps] = cadd(m, t);
                } else {
                    out[(od + Ns) * ps] = cadd(m, t);
                    out[(od + 2 * Ns) * ps] = csub(m, t);
                }
            }
        }
        __syncthreads();
        C* tmp = src;
        src = dst;
        dst = tmp;
        Ns *= r;
    }
    return src;
}
