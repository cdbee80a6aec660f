// Advection x passes built on the warp transforms of bld_warpfft.cuh.
//
// k_adv_xw: each warp owns one y row of one z chunk and streams up in z like
// k_adv_x, but the x transforms never touch shared memory and need no block
// barrier: after the inverse transforms lane l holds the physical points
// x = k + RAD * brev5(l) of every line, so the products and the z-neighbour
// values stay in registers with a fixed mapping; mode pairs (f, P1 - f) for the
// two-real unpack meet through one shuffle.
// k_adv_xb: a block of three warps per row, one line per warp, products in
// shared memory (fits the FP64 form's register budget).
#pragma once

#include "bld_warpfft.cuh"

// Rotation-form advection (src/processes/momentum_advection.jl:44-206), same
// arithmetic and term layout as k_adv_x.  The six input rows of layer j+1 are
// copied into the warp's shared buffer (cp.async) while layer j is transformed.
// grid (ceil(P2 / WPB), nchunks, members), block 32 * WPB; dynamic smem:
// W_P^{-l k} as [k][32] (RAD * 32 complex), then per warp 2 x 6 rows of K1.
// k_adv_xwc<R, RAD, MINB> is the same kernel with the registers capped at
// 65536 / (128 MINB) per thread, so that more warps share an SM (the values of
// the previous layer may then spill a little).
template <typename R, int RAD>
__device__ __forceinline__ void adv_xw_body(const XArgs& a) {
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
            inverse_line<R, RAD>(zl, lane, twl, 32, lt);
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
            forward_line<R, RAD>(zl, lane, twl, 32, lt);
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

template <typename R, int RAD>
__global__ void __launch_bounds__(128) k_adv_xw(XArgs a) { adv_xw_body<R, RAD>(a); }

template <typename R, int RAD, int MINB>
__global__ void __launch_bounds__(128, MINB) k_adv_xwc(XArgs a) { adv_xw_body<R, RAD>(a); }

// Rotation-form advection with one block of three warps per y row: each warp
// transforms one packed line in registers (inverse: (u, v), (vort3, w),
// (vort1, vort2)) and leaves it in shared memory in physical order; the block
// forms the products point by point with the z-neighbour values in registers
// (PPT points per thread); two warps forward-transform (adv1, adv2) and
// (adv3, 0) and write the modes.  Three barriers per layer, no shared-memory FFT
// stages, and only one line in registers per thread, so the FP64 form fits.
// The six input rows of layer j+1 are staged with cp.async while layer j runs.
// grid (P2, nchunks, members), block 96; dynamic smem: W_P^{-l k} [RAD][32],
// lines [3][P1 + 32], staging [2][6][K1] (complex).
template <typename R, int RAD>
__global__ void __launch_bounds__(96) k_adv_xb(XArgs a) {
    using C = cplx<R>;
    constexpr int PPT = (RAD + 2) / 3;   // points per thread of the products (96 threads, P1 = 32 RAD)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* twl_all = reinterpret_cast<C*>(smem_raw);
    const int P1 = a.P1, n3 = a.g.n3, k1max = a.g.k1max, K1 = a.g.K1;
    C* L = twl_all + RAD * 32;            // [3][P1]
    const int LP = P1 + 32;               // padded line stride (see swz)
    C* stage = L + 3 * LP;                // [2][6][K1]
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    for (int i = threadIdx.x; i < RAD * 32; i += blockDim.x) {
        const int k = i >> 5, l = i & 31;
        double s, c;
        sincospi(-2.0 * (double)(l * k) / (double)P1, &s, &c);
        twl_all[i] = mk<R>((R)c, (R)s);
    }
    const int y = blockIdx.x;
    const C* twl = twl_all + lane;
    LaneTw<R> lt;
    lane_twiddles<R>(lt, lane);
    const int brl = (int)(__brev((unsigned)lane) >> 27);
    const int z0 = blockIdx.y * a.zchunk;
    const int z1 = min(n3, z0 + a.zchunk);
    const C* Min = reinterpret_cast<const C*>(a.min) + (long long)m * a.min_mstride;
    C* Mout = reinterpret_cast<C*>(a.mout) + (long long)m * a.mout_mstride;
    const int nb = (k1max + 32) / 32;
    // staged rows: u, v, vort3 (C); w, vort1, vort2 (I) = terms 0, 1, 5, 2, 3, 4
    auto issue = [&](int j, C* buf) {
        const int nrows = (j < n3 - 1) ? 6 : 3;
        for (int i = threadIdx.x; i < nrows * K1; i += blockDim.x) {
            const int r = fdiv(i, a.k1_magic), k = i - r * K1;
            const int t = r < 2 ? r : (r == 2 ? 5 : r - 1);
            cp_async_elem<C>(buf + i, mrow(Min, a, t, j, y) + k);
        }
    };

    R pu[PPT], pv[PPT], pw[PPT], po1[PPT], po2[PPT], pa3[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) pu[i] = pv[i] = pw[i] = po1[i] = po2[i] = pa3[i] = R(0);
    // adv3 lines of consecutive I layers are forward-transformed in pairs
    // (adv3(i - 1) + i adv3(i)): the chunk emits I layers first_e..last_e
    const int first_e = max(z0, 1) - 1, last_e = z1 - 2;

    const int jb = max(0, z0 - 1);
    issue(jb, stage);
    cp_async_commit();
    for (int j = jb; j < z1; ++j) {
        const bool hasI = (j < n3 - 1);
        C* cur = stage + ((j - jb) & 1) * 6 * K1;
        cp_async_wait<0>();
        __syncthreads();   // staged rows of j visible; previous layer's forward reads of L done
        if (j + 1 < z1) issue(j + 1, stage + ((j + 1 - jb) & 1) * 6 * K1);
        cp_async_commit();
        // ---- inverse: warp t transforms line t into L[t] (physical order)
        if (wib < (hasI ? 3 : 2)) {
            C zl[RAD];
            const C* ra = cur + (wib == 0 ? 0 : (wib == 1 ? 2 : 4)) * K1;
            const C* rb = (wib == 1 && !hasI) ? nullptr : cur + (wib == 0 ? 1 : (wib == 1 ? 3 : 5)) * K1;
            load_packed<R, RAD>(zl, ra, rb, lane, P1, k1max);
            inverse_line<R, RAD>(zl, lane, twl, 32, lt);
#pragma unroll
            for (int k = 0; k < RAD; ++k) L[wib * LP + swz<C, RAD>(k + RAD * brl)] = zl[k];
        }
        __syncthreads();
        // ---- products at the thread's points; outputs overwrite L[0] and L[1]
        const bool emitC = (j >= z0);
        const bool emitI = (j >= z0) && (j >= 1);
        const int i3 = j - 1;                                  // I layer of this layer's adv3
        const bool odd3 = ((i3 - first_e) & 1) != 0;           // second of a pair
        const bool single3 = !odd3 && i3 == last_e;            // unpaired last one
#pragma unroll
        for (int i = 0; i < PPT; ++i) {
            const int x = threadIdx.x + 96 * i;
            if (x < P1) {
                const int xs = swz<C, RAD>(x);
                const C c0 = L[xs], c1 = L[LP + xs];
                const C c2 = hasI ? L[2 * LP + xs] : mk<R>(R(0), R(0));
                const R u = c0.x, v = c0.y, o3 = c1.x;
                const R w = hasI ? c1.y : R(0);
                const R q1 = c2.x, q2 = c2.y;
                R adv1, adv2;
                if (j == 0) {  // w below is the (zero) boundary value (:181-184,:194-197)
                    adv1 = o3 * v - R(0.5) * (q2 * w);
                    adv2 = R(0.5) * (q1 * w) - o3 * u;
                } else if (j == n3 - 1) {  // w above is the boundary value (:185-188,:198-201)
                    adv1 = o3 * v - R(0.5) * (po2[i] * pw[i]);
                    adv2 = R(0.5) * (po1[i] * pw[i]) - o3 * u;
                } else {  // (:180,:193)
                    adv1 = o3 * v - R(0.5) * (po2[i] * pw[i] + q2 * w);
                    adv2 = R(0.5) * (po1[i] * pw[i] + q1 * w) - o3 * u;
                }
                // adv3 on I layer j-1 (:206)
                const R adv3 = po2[i] * R(0.5) * (pu[i] + u) - po1[i] * R(0.5) * (pv[i] + v);
                L[xs] = mk<R>(adv1, adv2);
                if (emitI) {
                    if (odd3) L[LP + xs] = mk<R>(pa3[i], adv3);
                    else if (single3) L[LP + xs] = mk<R>(adv3, R(0));
                    pa3[i] = adv3;
                }
                pu[i] = u;
                pv[i] = v;
                pw[i] = w;
                po1[i] = q1;
                po2[i] = q2;
            }
        }
        __syncthreads();
        // ---- forward: warp 0 (adv1, adv2) on C layer j; warp 1 (adv3(j - 2), adv3(j - 1))
        // of I layers j - 2, j - 1 once a pair is complete, or the unpaired last one
        if (wib < 2 && (wib == 0 ? emitC : (emitI && (odd3 || single3)))) {
            C zl[RAD];
#pragma unroll
            for (int k = 0; k < RAD; ++k) zl[k] = L[wib * LP + swz<C, RAD>(k + RAD * brl)];
            forward_line<R, RAD>(zl, lane, twl, 32, lt);
            const bool two = wib == 0 || odd3;
            C* rA = mrow_w(Mout, a, wib == 0 ? 0 : 2, wib == 0 ? j : (odd3 ? i3 - 1 : i3), y);
            C* rB = mrow_w(Mout, a, wib == 0 ? 1 : 2, wib == 0 ? j : i3, y);
#pragma unroll
            for (int b = 0; b < RAD; ++b) {
                if (b >= nb) break;
                const int f = lane + 32 * b;
                const C Zk = zl[b];
                const C Zr = mirror_mode<R, RAD>(zl, lane, b);
                if (f <= k1max) {
                    rA[f] = mk<R>((Zk.x + Zr.x) * R(0.5), (Zk.y - Zr.y) * R(0.5));
                    if (two) rB[f] = mk<R>((Zk.y + Zr.y) * R(0.5), -(Zk.x - Zr.x) * R(0.5));
                }
            }
        }
    }
    cp_async_wait<0>();
}

// k_adv_xb with its transforms pipelined over two warp groups: five warps per y
// row, where warps 0-2 run the inverse transforms of layer j while warps 3-4 run
// the forward transforms of layer j - 1, then all five form the products of
// layer j (shared memory L -> F).  Two barriers per layer instead of three, and
// no warp idles while the forward lines run.  The staged rows of layer j + 1
// are requested (cp.async) at the top of iteration j and waited for before the
// barrier that ends the products.
// grid (P2, nchunks, members), block 160; dynamic smem: W_P^{-l k} [RAD][32],
// inverse lines L [3][P1 + 32], product lines F [2][P1 + 32], staging [2][6][K1] (complex).
template <typename R, int RAD>
__global__ void __launch_bounds__(160) k_adv_xp(XArgs a) {
    using C = cplx<R>;
    constexpr int NT = 160;
    constexpr int PPT = (32 * RAD + NT - 1) / NT;   // product points per thread
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* twl_all = reinterpret_cast<C*>(smem_raw);
    const int P1 = a.P1, n3 = a.g.n3, k1max = a.g.k1max, K1 = a.g.K1;
    C* L = twl_all + RAD * 32;            // [3][P1]
    const int LP = P1 + 32;               // padded line stride (see swz)
    C* F = L + 3 * LP;                    // [2][LP]
    C* stage = F + 2 * LP;                // [2][6][K1]
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    for (int i = threadIdx.x; i < RAD * 32; i += blockDim.x) {
        const int k = i >> 5, l = i & 31;
        double s, c;
        sincospi(-2.0 * (double)(l * k) / (double)P1, &s, &c);
        twl_all[i] = mk<R>((R)c, (R)s);
    }
    const int y = blockIdx.x;
    const C* twl = twl_all + lane;
    LaneTw<R> lt;
    lane_twiddles<R>(lt, lane);
    const int brl = (int)(__brev((unsigned)lane) >> 27);
    const int z0 = blockIdx.y * a.zchunk;
    const int z1 = min(n3, z0 + a.zchunk);
    const C* Min = reinterpret_cast<const C*>(a.min) + (long long)m * a.min_mstride;
    C* Mout = reinterpret_cast<C*>(a.mout) + (long long)m * a.mout_mstride;
    const int nb = (k1max + 32) / 32;
    // staged rows: u, v, vort3 (C); w, vort1, vort2 (I) = terms 0, 1, 5, 2, 3, 4
    auto issue = [&](int j, C* buf) {
        const int nrows = (j < n3 - 1) ? 6 : 3;
        for (int i = threadIdx.x; i < nrows * K1; i += blockDim.x) {
            const int r = fdiv(i, a.k1_magic), k = i - r * K1;
            const int t = r < 2 ? r : (r == 2 ? 5 : r - 1);
            cp_async_elem<C>(buf + i, mrow(Min, a, t, j, y) + k);
        }
    };

    R pu[PPT], pv[PPT], pw[PPT], po1[PPT], po2[PPT], pa3[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) pu[i] = pv[i] = pw[i] = po1[i] = po2[i] = pa3[i] = R(0);
    // adv3 lines of consecutive I layers are forward-transformed in pairs (as in
    // k_adv_xb): the chunk emits I layers first_e..last_e
    const int first_e = max(z0, 1) - 1, last_e = z1 - 2;

    const int jb = max(0, z0 - 1);
    issue(jb, stage);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();   // staged rows of jb and the twiddle table visible
    for (int j = jb; j <= z1; ++j) {
        const bool inv = j < z1;
        const bool hasI = (j < n3 - 1);
        if (j + 1 < z1) issue(j + 1, stage + ((j + 1 - jb) & 1) * 6 * K1);
        cp_async_commit();
        if (wib < 3) {
            // ---- inverse: warp t transforms line t of layer j into L[t] (physical order)
            if (inv && wib < (hasI ? 3 : 2)) {
                const C* cur = stage + ((j - jb) & 1) * 6 * K1;
                C zl[RAD];
                const C* ra = cur + (wib == 0 ? 0 : (wib == 1 ? 2 : 4)) * K1;
                const C* rb = (wib == 1 && !hasI) ? nullptr : cur + (wib == 0 ? 1 : (wib == 1 ? 3 : 5)) * K1;
                load_packed<R, RAD>(zl, ra, rb, lane, P1, k1max);
                inverse_line<R, RAD>(zl, lane, twl, 32, lt);
#pragma unroll
                for (int k = 0; k < RAD; ++k) L[wib * LP + swz<C, RAD>(k + RAD * brl)] = zl[k];
            }
        } else {
            // ---- forward of layer lj = j - 1: warp 3 (adv1, adv2) on C layer lj,
            // warp 4 (adv3, 0) on I layer lj - 1
            const int lj = j - 1, fw = wib - 3;
            const int i3 = lj - 1;                                   // I layer of lj's adv3
            const bool odd3 = ((i3 - first_e) & 1) != 0, single3 = !odd3 && i3 == last_e;
            const bool emit = lj >= jb && lj >= z0 && (fw == 0 || (lj >= 1 && (odd3 || single3)));
            if (emit) {
                C zl[RAD];
#pragma unroll
                for (int k = 0; k < RAD; ++k) zl[k] = F[fw * LP + swz<C, RAD>(k + RAD * brl)];
                forward_line<R, RAD>(zl, lane, twl, 32, lt);
                const bool two = fw == 0 || odd3;
                C* rA = mrow_w(Mout, a, fw == 0 ? 0 : 2, fw == 0 ? lj : (odd3 ? i3 - 1 : i3), y);
                C* rB = mrow_w(Mout, a, fw == 0 ? 1 : 2, fw == 0 ? lj : i3, y);
#pragma unroll
                for (int b = 0; b < RAD; ++b) {
                    if (b >= nb) break;
                    const int f = lane + 32 * b;
                    const C Zk = zl[b];
                    const C Zr = mirror_mode<R, RAD>(zl, lane, b);
                    if (f <= k1max) {
                        rA[f] = mk<R>((Zk.x + Zr.x) * R(0.5), (Zk.y - Zr.y) * R(0.5));
                        if (two) rB[f] = mk<R>((Zk.y + Zr.y) * R(0.5), -(Zk.x - Zr.x) * R(0.5));
                    }
                }
            }
        }
        __syncthreads();   // L of layer j written; F of layer j - 1 read
        if (inv) {
            // ---- products at the thread's points: L -> F
#pragma unroll
            for (int i = 0; i < PPT; ++i) {
                const int x = threadIdx.x + NT * i;
                if (x < P1) {
                    const int xs = swz<C, RAD>(x);
                    const C c0 = L[xs], c1 = L[LP + xs];
                    const C c2 = hasI ? L[2 * LP + xs] : mk<R>(R(0), R(0));
                    const R u = c0.x, v = c0.y, o3 = c1.x;
                    const R w = hasI ? c1.y : R(0);
                    const R q1 = c2.x, q2 = c2.y;
                    R adv1, adv2;
                    if (j == 0) {  // w below is the (zero) boundary value (:181-184,:194-197)
                        adv1 = o3 * v - R(0.5) * (q2 * w);
                        adv2 = R(0.5) * (q1 * w) - o3 * u;
                    } else if (j == n3 - 1) {  // w above is the boundary value (:185-188,:198-201)
                        adv1 = o3 * v - R(0.5) * (po2[i] * pw[i]);
                        adv2 = R(0.5) * (po1[i] * pw[i]) - o3 * u;
                    } else {  // (:180,:193)
                        adv1 = o3 * v - R(0.5) * (po2[i] * pw[i] + q2 * w);
                        adv2 = R(0.5) * (po1[i] * pw[i] + q1 * w) - o3 * u;
                    }
                    // adv3 on I layer j-1 (:206)
                    const R adv3 = po2[i] * R(0.5) * (pu[i] + u) - po1[i] * R(0.5) * (pv[i] + v);
                    F[xs] = mk<R>(adv1, adv2);
                    if (j >= z0 && j >= 1) {   // adv3 of I layer j - 1 is emitted
                        const bool odd = ((j - 1 - first_e) & 1) != 0;
                        if (odd) F[LP + xs] = mk<R>(pa3[i], adv3);
                        else if (j - 1 == last_e) F[LP + xs] = mk<R>(adv3, R(0));
                        pa3[i] = adv3;
                    }
                    pu[i] = u;
                    pv[i] = v;
                    pw[i] = w;
                    po1[i] = q1;
                    po2[i] = q2;
                }
            }
        }
        cp_async_wait<0>();   // this thread's copies of layer j + 1
        __syncthreads();      // F of layer j written, L read; staged rows of j + 1 visible
    }
}
