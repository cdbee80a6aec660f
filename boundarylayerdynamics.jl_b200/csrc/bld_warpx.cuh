// Warp-per-row x pass of the advection term: register-resident transforms.
//
// Each warp owns one y row of one z chunk and streams up in z like k_adv_x, but
// the x transforms never touch shared memory and need no block barrier.  A line
// of P1 = 32 * RAD points is split as n = l + 32 m (lane l, register m):
//   X[k + RAD q] = sum_l W_32^(l q) W_P^(l k) sum_m x[l + 32 m] W_RAD^(m k)
// so each lane first runs a RAD-point register codelet over m, multiplies by
// W_P^(l k), and the 32-point transforms over l run across the lanes as five
// radix-2 butterfly stages with shuffles (decimation in frequency: natural lane
// order in, bit-reversed out).  After the inverse transforms lane l holds the
// physical points x = k + RAD * brev5(l), k = 0..RAD-1, of every line, so the
// products and the z-neighbour values stay in registers with a fixed mapping.
// The forward transform runs the same steps backwards (decimation in time over
// the lanes: bit-reversed in, natural out; twiddle; codelet), leaving mode
// a + 32 b in lane a, register b.  Input rows are read straight from global
// memory into the packed Hermitian lines, output modes are written straight
// back; mode pairs (f, P1 - f) for the two-real unpack meet through one shuffle.
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
__device__ __forceinline__ void inverse_line(cplx<R> (&z)[RAD], int lane, const cplx<R>* __restrict__ twl,
                                             const LaneTw<R>& lt) {
    dft<R, RAD, +1>(z);
#pragma unroll
    for (int k = 1; k < RAD; ++k) {
        cplx<R> w = twl[k * 32];          // W_P^{-lane k}
        w.y = -w.y;
        z[k] = c_mul<R>(z[k], w);
    }
    lanes_dif<R, RAD, +1>(z, lane, lt);
}

// forward transform from the physical layout of inverse_line; mode lane + 32 b in register b
template <typename R, int RAD>
__device__ __forceinline__ void forward_line(cplx<R> (&z)[RAD], int lane, const cplx<R>* __restrict__ twl,
                                             const LaneTw<R>& lt) {
    lanes_dit<R, RAD, -1>(z, lane, lt);
#pragma unroll
    for (int k = 1; k < RAD; ++k) z[k] = c_mul<R>(z[k], twl[k * 32]);
    dft<R, RAD, -1>(z);
}

// Z[P1 - f] for the modes f = lane + 32 b this lane holds (two-real unpack partner)
template <typename R, int RAD>
__device__ __forceinline__ cplx<R> mirror_mode(const cplx<R> (&z)[RAD], int lane, int b) {
    // lane a != 0: P1 - f = (32 - a) + 32 (RAD - 1 - b); lane 0: 32 (RAD - b) mod P1, same lane
    const cplx<R> other = c_shfl<R>(z[RAD - 1 - b], (32 - lane) & 31);
    return lane == 0 ? z[(RAD - b) % RAD] : other;
}

// Rotation-form advection (src/processes/momentum_advection.jl:44-206), same
// arithmetic and term layout as k_adv_x.  The six input rows of layer j+1 are
// copied into the warp's shared buffer (cp.async) while layer j is transformed.
// grid (ceil(P2 / WPB), nchunks, members), block 32 * WPB; dynamic smem:
// W_P^{-l k} as [k][32] (RAD * 32 complex), then per warp 2 x 6 rows of K1.
template <typename R, int RAD>
__global__ void __launch_bounds__(128) k_adv_xw(XArgs a) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* twl_all = reinterpret_cast<C*>(smem_raw);
    const int P1 = a.P1, n3 = a.g.n3, k1max = a.g.k1max, K1 = a.g.K1;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    for (int i = threadIdx.x; i < RAD * 32; i += blockDim.x) {
        const int k = i >> 5, l = i & 31;
        double s, c;
        sincospi(-2.0 * (double)(l * k) / (double)P1, &s, &c);
        twl_all[i] = mk<R>((R)c, (R)s);
    }
    __syncthreads();
    const int y = blockIdx.x * (blockDim.x >> 5) + wib;
    if (y >= a.P2) return;
    C* wbuf = twl_all + RAD * 32 + (size_t)wib * 12 * K1;   // [2][6][K1]
    const C* twl = twl_all + lane;
    LaneTw<R> lt;
    lane_twiddles<R>(lt, lane);
    const int z0 = blockIdx.y * a.zchunk;
    const int z1 = min(n3, z0 + a.zchunk);
    const C* Min = reinterpret_cast<const C*>(a.min) + (long long)m * a.min_mstride;
    C* Mout = reinterpret_cast<C*>(a.mout) + (long long)m * a.mout_mstride;
    const int nb = (k1max + 32) / 32;   // registers b holding modes <= k1max
    // buffer rows: 0 u, 1 v, 2 vort3 (C); 3 w, 4 vort1, 5 vort2 (I, absent on the top C layer)
    const int terms[6] = {0, 1, 5, 2, 3, 4};
    auto issue = [&](int j, C* buf) {
        const int nrows = (j < n3 - 1) ? 6 : 3;
        for (int r = 0; r < nrows; ++r) {
            const C* src = mrow(Min, a, terms[r], j, y);
            for (int i = lane; i < K1; i += 32) cp_async_elem<C>(buf + r * K1 + i, src + i);
        }
    };

    R pu[RAD], pv[RAD], pw[RAD], po1[RAD], po2[RAD];
#pragma unroll
    for (int i = 0; i < RAD; ++i) pu[i] = pv[i] = pw[i] = po1[i] = po2[i] = R(0);

    const int jb = max(0, z0 - 1);
    issue(jb, wbuf);
    cp_async_commit();
    for (int j = jb; j < z1; ++j) {
        const bool hasI = (j < n3 - 1);
        C* cur = wbuf + ((j - jb) & 1) * 6 * K1;
        if (j + 1 < z1) issue(j + 1, wbuf + ((j + 1 - jb) & 1) * 6 * K1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncwarp();
        // inverse transforms, one line at a time through the same code (a small
        // loop body keeps the instruction working set in cache):
        // line 0 (u, v), line 1 (vort3, w), line 2 (vort1, vort2)
        R U[RAD], V[RAD], O3[RAD], W[RAD], Q1[RAD], Q2[RAD];
        const int nlin = hasI ? 3 : 2;
#pragma unroll 1
        for (int t = 0; t < nlin; ++t) {
            C zl[RAD];
            const C* ra = cur + (t == 0 ? 0 : (t == 1 ? 2 : 4)) * K1;
            const C* rb = (t == 1 && !hasI) ? nullptr : cur + (t == 0 ? 1 : (t == 1 ? 3 : 5)) * K1;
            load_packed<R, RAD>(zl, ra, rb, lane, P1, k1max);
            inverse_line<R, RAD>(zl, lane, twl, lt);
#pragma unroll
            for (int i = 0; i < RAD; ++i) {
                if (t == 0) {
                    U[i] = zl[i].x;
                    V[i] = zl[i].y;
                } else if (t == 1) {
                    O3[i] = zl[i].x;
                    W[i] = hasI ? zl[i].y : R(0);
                } else {
                    Q1[i] = zl[i].x;
                    Q2[i] = zl[i].y;
                }
            }
        }
        __syncwarp();   // every lane is done with `cur` before it is refilled
        if (!hasI) {
#pragma unroll
            for (int i = 0; i < RAD; ++i) Q1[i] = Q2[i] = R(0);
        }
        const bool emitC = (j >= z0);
        const bool emitI = (j >= z0) && (j >= 1);
        R A1[RAD], A2[RAD], A3[RAD];
#pragma unroll
        for (int i = 0; i < RAD; ++i) {
            const R u = U[i], v = V[i], o3 = O3[i], w = W[i], q1 = Q1[i], q2 = Q2[i];
            if (j == 0) {  // w below is the (zero) boundary value (:181-184,:194-197)
                A1[i] = o3 * v - R(0.5) * (q2 * w);
                A2[i] = R(0.5) * (q1 * w) - o3 * u;
            } else if (j == n3 - 1) {  // w above is the boundary value (:185-188,:198-201)
                A1[i] = o3 * v - R(0.5) * (po2[i] * pw[i]);
                A2[i] = R(0.5) * (po1[i] * pw[i]) - o3 * u;
            } else {  // (:180,:193)
                A1[i] = o3 * v - R(0.5) * (po2[i] * pw[i] + q2 * w);
                A2[i] = R(0.5) * (po1[i] * pw[i] + q1 * w) - o3 * u;
            }
            // adv3 on I layer j-1 (:206)
            A3[i] = po2[i] * R(0.5) * (pu[i] + u) - po1[i] * R(0.5) * (pv[i] + v);
            pu[i] = u;
            pv[i] = v;
            pw[i] = w;
            po1[i] = q1;
            po2[i] = q2;
        }
        // forward transforms: line 0 (adv1, adv2) on C layer j, line 1 (adv3, 0) on I layer j-1
#pragma unroll 1
        for (int t = 0; t < 2; ++t) {
            if (!(t == 0 ? emitC : emitI)) continue;
            C zl[RAD];
#pragma unroll
            for (int i = 0; i < RAD; ++i) zl[i] = t == 0 ? mk<R>(A1[i], A2[i]) : mk<R>(A3[i], R(0));
            forward_line<R, RAD>(zl, lane, twl, lt);
            C* rA = mrow_w(Mout, a, t == 0 ? 0 : 2, t == 0 ? j : j - 1, y);
            C* rB = mrow_w(Mout, a, 1, j, y);
#pragma unroll
            for (int b = 0; b < RAD; ++b) {
                if (b >= nb) break;
                const int f = lane + 32 * b;
                const C Zk = zl[b];
                const C Zr = mirror_mode<R, RAD>(zl, lane, b);
                if (f <= k1max) {
                    rA[f] = mk<R>((Zk.x + Zr.x) * R(0.5), (Zk.y - Zr.y) * R(0.5));
                    if (t == 0) rB[f] = mk<R>((Zk.y + Zr.y) * R(0.5), -(Zk.x - Zr.x) * R(0.5));
                }
            }
        }
    }
    cp_async_wait<0>();
}
