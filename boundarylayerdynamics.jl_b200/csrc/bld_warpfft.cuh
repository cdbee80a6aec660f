// Warp-level complex transforms of P = 32 * RAD points held in registers.
//
// A line is split as n = l + 32 m (lane l, register m):
//   X[k + RAD q] = sum_l W_32^(l q) W_P^(l k) sum_m x[l + 32 m] W_RAD^(m k)
// so each lane first runs a RAD-point register codelet over m, multiplies by
// W_P^(l k), and the 32-point transforms over l run across the lanes as five
// radix-2 butterfly stages with shuffles (decimation in frequency: natural lane
// order in, bit-reversed out).  An inverse transform leaves point
// k + RAD * brev5(l) in lane l, register k; the forward transform starts from
// that layout (decimation in time over the lanes, twiddle, codelet) and leaves
// coefficient a + 32 b in lane a, register b.  Twiddles W_P^(-l k) are read as
// tw[k * tstride]: a [RAD][32] table at +lane with stride 32, or the [P] table
// W_P^(-m) with stride lane.
#pragma once

#include "bld_dft.cuh"

template <typename R>
__device__ __forceinline__ cplx<R> c_shfl_xor(cplx<R> v, int mask) {
    cplx<R> r;
    r.x = __shfl_xor_sync(0xffffffffu, v.x, mask);
    r.y = __shfl_xor_sync(0xffffffffu, v.y, mask);
    return r;
}
template <typename R>
__device__ __forceinline__ cplx<R> c_shfl(cplx<R> v, int src) {
    cplx<R> r;
    r.x = __shfl_sync(0xffffffffu, v.x, src);
    r.y = __shfl_sync(0xffffffffu, v.y, src);
    return r;
}
template <typename R>
__device__ __forceinline__ cplx<R> c_mul(cplx<R> a, cplx<R> b) {
    return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Lane twiddles of the cross-lane stages h = 16, 8, 4, 2: W_{2h}^{-(l mod h)}
// (forward sign; the inverse uses the conjugate) on lanes whose bit h is set, 1
// on the others, so that every lane multiplies unconditionally.
template <typename R>
struct LaneTw {
    cplx<R> w[4];  // h = 16, 8, 4, 2
};

template <typename R>
__device__ __forceinline__ void lane_twiddles(LaneTw<R>& t, int lane) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int h = 16 >> i;
        double s = 0.0, c = 1.0;
        if (lane & h) sincospi(-(double)(lane % h) / (double)h, &s, &c);
        t.w[i] = mk<R>((R)c, (R)s);
    }
}

// the same from the [P] table W_P^(-m): W_{2h}^(-j) = W_P^(-j P / (2h))
template <typename R>
__device__ __forceinline__ void lane_twiddles_tab(LaneTw<R>& t, int lane, const cplx<R>* __restrict__ tw, int P) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int h = 16 >> i;
        t.w[i] = (lane & h) ? tw[(lane % h) * (P / (2 * h))] : mk<R>(R(1), R(0));
    }
}

template <typename R, int DIR>
__device__ __forceinline__ cplx<R> lane_w(const LaneTw<R>& t, int i) {
    cplx<R> w = t.w[i];
    if (DIR > 0) w.y = -w.y;
    return w;
}

// 32-point transforms across the lanes of each register value, DIF: natural
// order in, lane l ends with the coefficient brev5(l).  At span h the lower lane
// of a pair keeps v + p and the upper lane (p - v) W_{2h}^(l mod h): both are
// (p + sgn v) w_self.  DIR = +1 inverse.
template <typename R, int N, int DIR>
__device__ __forceinline__ void lanes_dif(cplx<R> (&v)[N], int lane, const LaneTw<R>& t) {
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const int h = 16 >> i;
        const R sg = (lane & h) ? R(-1) : R(1);
        const cplx<R> w = lane_w<R, DIR>(t, i < 4 ? i : 0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const cplx<R> p = c_shfl_xor<R>(v[k], h);
            const cplx<R> s = mk<R>(p.x + sg * v[k].x, p.y + sg * v[k].y);
            v[k] = (i < 4) ? c_mul<R>(s, w) : s;
        }
    }
}

// 32-point transforms across the lanes, DIT: lane l holds the input coefficient
// brev5(l); natural order out.  The upper lane of a pair scales its own value by
// the twiddle before the exchange, so the lower lane receives w p and keeps
// v + w p while the upper lane keeps p - w v: both are p' + sgn t.  DIR = -1 forward.
template <typename R, int N, int DIR>
__device__ __forceinline__ void lanes_dit(cplx<R> (&v)[N], int lane, const LaneTw<R>& t) {
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const int h = 1 << i;           // spans 1, 2, 4, 8, 16
        const R sg = (lane & h) ? R(-1) : R(1);
        const cplx<R> w = lane_w<R, DIR>(t, h > 1 ? 4 - i : 0);   // index 3 for h = 2 ... 0 for h = 16
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const cplx<R> tv = (h > 1) ? c_mul<R>(v[k], w) : v[k];
            const cplx<R> p = c_shfl_xor<R>(tv, h);
            v[k] = mk<R>(p.x + sg * tv.x, p.y + sg * tv.y);
        }
    }
}

// asynchronous element copies global -> shared (per-thread, completion by groups)
template <typename C>
__device__ __forceinline__ void cp_async_elem(C* sdst, const C* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    if constexpr (sizeof(C) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// packed line Z = A + i B of two Hermitian half-spectra (FFTW c2r conventions: the
// DC imaginary parts are dropped) at n = lane + 32 m
template <typename R, int RAD>
__device__ __forceinline__ void load_packed(cplx<R> (&z)[RAD], const cplx<R>* __restrict__ rowA,
                                            const cplx<R>* __restrict__ rowB, int lane, int P1, int k1max) {
#pragma unroll
    for (int m = 0; m < RAD; ++m) {
        const int n = lane + 32 * m;
        const bool lo = n <= k1max, hi = n >= P1 - k1max;
        const int idx = lo ? n : P1 - n;
        cplx<R> A = mk<R>(R(0), R(0)), B = mk<R>(R(0), R(0));
        if (lo || hi) {
            if (rowA) A = rowA[idx];
            if (rowB) B = rowB[idx];
        }
        if (n == 0)
            z[m] = mk<R>(A.x, B.x);
        else if (lo)
            z[m] = mk<R>(A.x - B.y, A.y + B.x);
        else
            z[m] = mk<R>(A.x + B.y, -A.y + B.x);   // zero outside the bands (A = B = 0)
    }
}

// inverse transform of a packed line: natural order in, physical point
// k + RAD * brev5(lane) in register k out
template <typename R, int RAD>
__device__ __forceinline__ void inverse_line(cplx<R> (&z)[RAD], int lane, const cplx<R>* __restrict__ tw, int tstride,
                                             const LaneTw<R>& lt) {
    dft<R, RAD, +1>(z);
#pragma unroll
    for (int k = 1; k < RAD; ++k) {
        cplx<R> w = tw[k * tstride];      // W_P^{-lane k}
        w.y = -w.y;
        z[k] = c_mul<R>(z[k], w);
    }
    lanes_dif<R, RAD, +1>(z, lane, lt);
}

// forward transform from the physical layout of inverse_line; mode lane + 32 b in register b
template <typename R, int RAD>
__device__ __forceinline__ void forward_line(cplx<R> (&z)[RAD], int lane, const cplx<R>* __restrict__ tw, int tstride,
                                             const LaneTw<R>& lt) {
    lanes_dit<R, RAD, -1>(z, lane, lt);
#pragma unroll
    for (int k = 1; k < RAD; ++k) z[k] = c_mul<R>(z[k], tw[k * tstride]);
    dft<R, RAD, -1>(z);
}

// Z[P1 - f] for the modes f = lane + 32 b this lane holds (two-real unpack partner)
template <typename R, int RAD>
__device__ __forceinline__ cplx<R> mirror_mode(const cplx<R> (&z)[RAD], int lane, int b) {
    // lane a != 0: P1 - f = (32 - a) + 32 (RAD - 1 - b); lane 0: 32 (RAD - b) mod P1, same lane
    const cplx<R> other = c_shfl<R>(z[RAD - 1 - b], (32 - lane) & 31);
    return lane == 0 ? z[(RAD - b) % RAD] : other;
}


// Shared-memory buffers that hold lines in physical order after a warp
// transform (lane l holds points k + RAD brev5(l)) store point p at position
// swz(p) = p + (p / RAD) >> SH, on a padded extent P + 32.  Without it the lanes
// of one shared-memory wavefront (8 lanes for 16-byte complex values, 16 for
// 8-byte ones) land in the same banks, up to 8-way for even RAD; the pad adds the
// bits of brev5(l) that RAD brev5(l) does not spread over the banks, and
// consecutive points stay consecutive between pads.
__host__ __device__ constexpr int ctz_c(int v) { return (v & 1) ? 0 : 1 + ctz_c(v >> 1); }
template <typename C, int RAD>
__device__ __forceinline__ int swz(int p) {
    if constexpr (RAD == 0) {
        return p;
    } else {
        constexpr int a = ctz_c(RAD) < 3 ? ctz_c(RAD) : 3;
        constexpr int SH = sizeof(C) == 16 ? ((RAD & 1) ? 3 : 2) : 4 - a;
        return p + ((p / RAD) >> SH);
    }
}

__device__ __forceinline__ int brev5(int lane) { return (int)(__brev((unsigned)lane) >> 27); }

// In-place transforms of `nlines` lines of P = 32 RAD points in shared memory,
// natural order in and out, one line per warp at a time (the block-wide Stockham
// stages replaced by register work).  Line l starts at lines + l (P + 32) and
// holds point p at swz(p).  `tw` is the lane-major [RAD][32] table W_P^(-l k) in
// shared memory, `twg` the [P] table W_P^(-m) in global memory.  The caller
// synchronises the block before and after.
template <typename R, int RAD, int DIR>
__device__ __forceinline__ void warp_lines_inplace(cplx<R>* lines, int nlines, int P, const cplx<R>* __restrict__ tw,
                                                   const cplx<R>* __restrict__ twg) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int brl = brev5(lane);
    LaneTw<R> lt;
    lane_twiddles_tab<R>(lt, lane, twg, P);
    for (int l = threadIdx.x >> 5; l < nlines; l += nw) {
        using C = cplx<R>;
        C* L = lines + (size_t)l * (P + 32);
        C z[RAD];
        if constexpr (DIR > 0) {
#pragma unroll
            for (int m = 0; m < RAD; ++m) z[m] = L[swz<C, RAD>(lane + 32 * m)];
            inverse_line<R, RAD>(z, lane, tw + lane, 32, lt);
#pragma unroll
            for (int k = 0; k < RAD; ++k) L[swz<C, RAD>(k + RAD * brl)] = z[k];
        } else {
#pragma unroll
            for (int k = 0; k < RAD; ++k) z[k] = L[swz<C, RAD>(k + RAD * brl)];
            forward_line<R, RAD>(z, lane, tw + lane, 32, lt);
#pragma unroll
            for (int b = 0; b < RAD; ++b) L[swz<C, RAD>(lane + 32 * b)] = z[b];
        }
    }
}
