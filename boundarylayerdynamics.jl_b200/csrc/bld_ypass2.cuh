// y passes with two-pass transforms of P2 = A * B points.
//
// A block owns NL neighbouring k1 lines of one term (or rate field) at one
// layer.  The transform of a line runs in two Stockham passes with register
// codelets, one barrier between them:
//   pass 1: B tasks per line; task j gathers points j + B t (t < A), runs a
//           radix-A DFT and stores X1[j A + q] in shared memory;
//   pass 2: A tasks per line; task j reads X1[j + A t] (t < B), multiplies by
//           W_P^(j t), runs a radix-B DFT and holds X[j + A q] (q < B).
// (X[j + A q] = sum_t W_P^(j t) W_B^(t q) X1[j + A t], X1[j A + q'] = sum_t'
// x[j + B t'] W_A^(t' q'): the DFT of n = j + B t' split by n mod B.)
// Thread tid works on line tid % NL and task tid / NL, so the lanes of a warp
// read and write NL consecutive k1 values: coalesced global rows and
// conflict-free shared rows [position][line].
//
// Inverse y pass (get_layer! along y, src/physical_space.jl:277-295): pass 1
// gathers the padded spectral line straight from the state (term prefactors
// and vorticity stencils applied on load), pass 2 writes physical rows of the
// mixed array M[term][z][y][k1] from registers.  Forward y pass (add_layer!
// along y, src/physical_space.jl:208-233): pass 1 gathers M, pass 2 writes the
// spectrum back to shared memory and the epilogue of k_fwd_y truncates, scales
// and adds the linear terms.
#pragma once

#define BLD_Y2_NL 16
// resident blocks per SM the register allocation is held to (launch bounds):
// up to ~110 registers per thread for blocks of up to 288 threads
template <typename R>
__host__ __device__ constexpr int y2_min_blocks(int threads) {
    return threads <= 256 ? (sizeof(R) == 8 ? 2 : 3) : 2;
}
// the inverse pass holds fewer values: single precision fits three blocks of 288
template <typename R>
__host__ __device__ constexpr int y2_min_blocks_inv(int threads) {
    return sizeof(R) == 4 && threads <= 288 ? 3 : y2_min_blocks<R>(threads);
}

// spectral term `OP` of the inverse pass at mode (jj, k1) of layer z; the
// pointers address layer z of u, v, w (Su1/Sv1: layer z + 1); same arithmetic as
// inv_term_value (src/derivatives.jl:67-80,198-230)
template <int OP>
__device__ __forceinline__ double2 y2_term(const double2* __restrict__ Sf, const double2* __restrict__ Su,
                                           const double2* __restrict__ Sv, const double2* __restrict__ Sw, int F,
                                           int mo, double e1, double e2, double al) {
    if constexpr (OP == T_DIRECT) {
        return __ldg(Sf + mo);
    } else if constexpr (OP == T_D1) {
        const double2 s = __ldg(Sf + mo);
        return make_double2(-e1 * s.y, e1 * s.x);
    } else if constexpr (OP == T_D2) {
        const double2 s = __ldg(Sf + mo);
        return make_double2(-e2 * s.y, e2 * s.x);
    } else if constexpr (OP == T_VORT1) {  // D2 w - (-a v(z) + a v(z+1))
        const double2 w = __ldg(Sw + mo), v0 = __ldg(Sv + mo), v1 = __ldg(Sv + F + mo);
        const double dzx = -al * v0.x + al * v1.x, dzy = -al * v0.y + al * v1.y;
        return make_double2(-e2 * w.y - dzx, e2 * w.x - dzy);
    } else if constexpr (OP == T_VORT2) {  // (-a u(z) + a u(z+1)) - D1 w
        const double2 w = __ldg(Sw + mo), u0 = __ldg(Su + mo), u1 = __ldg(Su + F + mo);
        const double dzx = -al * u0.x + al * u1.x, dzy = -al * u0.y + al * u1.y;
        return make_double2(dzx - (-e1 * w.y), dzy - e1 * w.x);
    } else {  // T_VORT3: D1 v - D2 u
        const double2 v = __ldg(Sv + mo), u = __ldg(Su + mo);
        return make_double2(-e1 * v.y - (-e2 * u.y), e1 * v.x - e2 * u.x);
    }
}

// pass 1 of the inverse transform for term kind OP: gather, radix-A DFT, store X1
template <typename R, int A, int B, int OP, int NL = BLD_Y2_NL>
__device__ __forceinline__ void inv_y2_pass1(const InvYArgs& a, const double2* __restrict__ S, int f, int z, int k1,
                                             bool ok, int j, int l, cplx<R>* buf) {
    using C = cplx<R>;
    constexpr int P = A * B;
    const Geo& g = a.g;
    const int F = g.F, n3 = g.n3, k2max = g.k2max, shift = P - g.K2;
    const double2* Su = S + (long long)z * F;
    const double2* Sv = Su + (long long)n3 * F;
    const double2* Sw = Sv + (long long)n3 * F;
    const double2* Sf = S + ((long long)f * n3 + z) * F;
    const double e1 = ok ? __ldg(a.d1 + k1) : 0.0;
    const double al = (OP == T_VORT1 || OP == T_VORT2) ? __ldg(a.alpha_i + z) : 0.0;
    C x[A];
#pragma unroll
    for (int t = 0; t < A; ++t) {
        const int p = j + B * t;
        const int jj = p <= k2max ? p : (p >= P - k2max ? p - shift : -1);
        double2 v = make_double2(0.0, 0.0);
        if (ok && jj >= 0) {
            const double e2 = (OP == T_D2 || OP == T_VORT1 || OP == T_VORT3) ? __ldg(a.d2 + jj) : 0.0;
            v = y2_term<OP>(Sf, Su, Sv, Sw, F, jj * g.K1 + k1, e1, e2, al);
        }
        x[t] = mk<R>((R)v.x, (R)v.y);
    }
    dft<R, A, +1>(x);
#pragma unroll
    for (int q = 0; q < A; ++q) buf[(j * A + q) * NL + l] = x[q];
}

// grid (nterms * members, ceil(K1 / NL), n3), block B * NL threads;
// smem tw[P] + P * NL complex; NL = 16 lines per block, or 8 with more blocks per SM
template <typename R, int A, int B, int MINB, int NL = BLD_Y2_NL>
__global__ void __launch_bounds__(B * NL, MINB) k_inv_y2(InvYArgs a) {
    using C = cplx<R>;
    constexpr int P = A * B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + P;
    const int t = blockIdx.x % a.nterms, m = a.m0 + blockIdx.x / a.nterms;
    BLD_SKIP_INACTIVE(a, m);
    const int z = blockIdx.z;
    const int nz = a.isI[t] ? a.g.n3 - 1 : a.g.n3;
    if (z >= nz) return;
    const int op = a.op[t], f = a.fld[t];
    const int K1 = a.g.K1;
    const int l = threadIdx.x % NL, j = threadIdx.x / NL;
    const int k1 = blockIdx.y * NL + l;
    const bool ok = k1 < K1;
    const C* twg = reinterpret_cast<const C*>(a.tw);
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const double2* S = a.state + (long long)m * a.g.mstride;
    switch (op) {
        case T_DIRECT: inv_y2_pass1<R, A, B, T_DIRECT, NL>(a, S, f, z, k1, ok, j, l, buf); break;
        case T_D1: inv_y2_pass1<R, A, B, T_D1, NL>(a, S, f, z, k1, ok, j, l, buf); break;
        case T_D2: inv_y2_pass1<R, A, B, T_D2, NL>(a, S, f, z, k1, ok, j, l, buf); break;
        case T_VORT1: inv_y2_pass1<R, A, B, T_VORT1, NL>(a, S, f, z, k1, ok, j, l, buf); break;
        case T_VORT2: inv_y2_pass1<R, A, B, T_VORT2, NL>(a, S, f, z, k1, ok, j, l, buf); break;
        default: inv_y2_pass1<R, A, B, T_VORT3, NL>(a, S, f, z, k1, ok, j, l, buf); break;
    }
    __syncthreads();
    if (j >= A) return;
    C x[B];
#pragma unroll
    for (int s = 0; s < B; ++s) x[s] = buf[(j + A * s) * NL + l];
#pragma unroll
    for (int s = 1; s < B; ++s) x[s] = c_tw<+1>(x[s], tw[j * s]);
    dft<R, B, +1>(x);
    if (!ok) return;
    C* out = reinterpret_cast<C*>(a.mixed) + (long long)m * a.mixed_mstride + (long long)(t * a.g.n3 + z) * P * K1 + k1;
#pragma unroll
    for (int q = 0; q < B; ++q) out[(long long)(j + A * q) * K1] = x[q];
}

// grid (fields * members, ceil(K1 / NL), n3), block B * NL threads;
// smem tw[P] + P * nlines complex (nlines = NL, or 2 NL with a D2 contribution).
// NL = 16 lines per block, or 8 with more blocks per SM and OB = 4 outputs of
// the epilogue in flight per thread
template <typename R, int A, int B, int MINB, int NL = BLD_Y2_NL, int OB = 1>
__global__ void __launch_bounds__(B * NL, MINB) k_fwd_y2(FwdYArgs a) {
    using C = cplx<R>;
    constexpr int P = A * B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int fi = blockIdx.x % a.fields, m = a.m0 + blockIdx.x / a.fields;
    BLD_SKIP_INACTIVE(a, m);
    const int f = a.field0 + fi;
    const int z = blockIdx.z;
    const Geo& g = a.g;
    const int nz = (f == 2) ? g.n3 - 1 : g.n3;
    if (z >= nz) return;
    const int K1 = g.K1;
    const int k10 = blockIdx.y * NL;
    const int nc = a.ncontrib[fi];
    bool hasB = false;
    for (int ci = 0; ci < nc; ++ci) hasB |= (a.c[fi][ci].pref == 2);
    const int nlines = hasB ? 2 * NL : NL;
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + P;
    const C* twg = reinterpret_cast<const C*>(a.tw);
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int l = threadIdx.x % NL, j = threadIdx.x / NL;
    const int k1 = k10 + l;
    const bool ok = k1 < K1;
    const C* base = reinterpret_cast<const C*>(a.mout) + (long long)m * a.mout_mstride + k1;
    const long long layer = (long long)P * K1;
    const R d1 = ok ? (R)__ldg(a.d1 + k1) : R(0);
    // pass 1: line set 0 holds the contributions with prefactor 1 or D1 (summed in
    // contribution order), set 1 the D2 contribution
    for (int set = 0; set < (hasB ? 2 : 1); ++set) {
        C x[A];
#pragma unroll
        for (int t = 0; t < A; ++t) x[t] = mk<R>(0, 0);
        if (ok && nc == 1 && a.c[fi][0].pref == 0) {
            // a single contribution without prefactor (the advection rates): loads only
            const C* src = base + (long long)(a.c[fi][0].term * g.n3 + z) * layer;
#pragma unroll
            for (int t = 0; t < A; ++t) x[t] = src[(long long)(j + B * t) * K1];
        } else if (ok) {
            for (int ci = 0; ci < nc; ++ci) {
                const FwdContrib cb = a.c[fi][ci];
                if ((cb.pref == 2) != (set == 1)) continue;
                const C* src = base + (long long)(cb.term * g.n3 + z) * layer;
                const R d = cb.pref == 1 ? d1 : R(0);
#pragma unroll
                for (int t = 0; t < A; ++t) {
                    C v = src[(long long)(j + B * t) * K1];
                    if (cb.pref == 1) v = mk<R>(-d * v.y, d * v.x);   // D1 = i d1[k1]
                    x[t] = mk<R>(x[t].x + v.x, x[t].y + v.y);
                }
            }
        }
        dft<R, A, -1>(x);
        const int L = set * NL + l;
#pragma unroll
        for (int q = 0; q < A; ++q) buf[(j * A + q) * nlines + L] = x[q];
    }
    __syncthreads();
    if (j < A) {
        for (int set = 0; set < (hasB ? 2 : 1); ++set) {
            const int L = set * NL + l;
            C x[B];
#pragma unroll
            for (int s = 0; s < B; ++s) x[s] = buf[(j + A * s) * nlines + L];
#pragma unroll
            for (int s = 1; s < B; ++s) x[s] = c_tw<-1>(x[s], tw[j * s]);
            dft<R, B, -1>(x);
#pragma unroll
            for (int q = 0; q < B; ++q) buf[(j + A * q) * nlines + L] = x[q];
        }
    }
    __syncthreads();
    constexpr int nls = NL == 16 ? 4 : 3;   // log2(NL)
    static_assert((1 << nls) == NL, "NL is 8 or 16");
    fwd_y_epilogue<R, 0, OB>(a, buf, nlines, m, f, z, nz, k10, NL, nls, hasB);
}

// ----------------------------------------------------------------------------
// Inverse y pass with TMA-staged input tiles (k_inv_y3).
//
// A block owns one term, a tile of BLD_Y3_NL k1 lines and a chunk of layers,
// and walks up the chunk.  The spectral rows a term needs at layer z -- one
// [K2 x NL] tile of its field, or for the vorticity terms the tiles of w(z) and
// of v or u at z and z + 1 (the staggered d/dx3 stencil, src/derivatives.jl:
// 104-110,198-230) -- are copied into shared memory by TMA, two layers ahead
// of the transform: while the block transforms layer z, the tiles of z + 1 are
// in flight and those of z + 2 are issued as soon as layer z's tiles are read.
// The transform is the two-pass one of k_inv_y2 (pass 1 reads the staged tile,
// pass 2 writes the physical rows of M from registers), so the loads never wait
// on registers or on the block's other warps.
// ----------------------------------------------------------------------------
#include "bld_tma.cuh"

#define BLD_Y3_NL 8
#define BLD_Y3_TILES 3   // tiles per layer at most (vorticity terms)

__host__ __device__ constexpr int y3_align(int b) { return (b + 127) / 128 * 128; }
// shared memory of k_inv_y3: barriers, twiddles, pass-1 buffer, 2 x 3 input tiles
__host__ __device__ constexpr int y3_smem(int P, int K2, int csz) {
    return 128 + y3_align(P * csz) + y3_align(P * BLD_Y3_NL * csz) + 2 * BLD_Y3_TILES * y3_align(K2 * BLD_Y3_NL * 16);
}

// term kind OP at mode row jj, line l of the staged tiles T0..T2 (see the tile
// order in k_inv_y3); same arithmetic as y2_term / inv_term_value
template <int OP>
__device__ __forceinline__ double2 y3_term(const double2* __restrict__ T0, const double2* __restrict__ T1,
                                           const double2* __restrict__ T2, int idx, double e1, double e2, double al) {
    if constexpr (OP == T_DIRECT) {
        return T0[idx];
    } else if constexpr (OP == T_D1) {
        const double2 s = T0[idx];
        return make_double2(-e1 * s.y, e1 * s.x);
    } else if constexpr (OP == T_D2) {
        const double2 s = T0[idx];
        return make_double2(-e2 * s.y, e2 * s.x);
    } else if constexpr (OP == T_VORT1) {  // T0 = w(z), T1 = v(z), T2 = v(z+1)
        const double2 w = T0[idx], v0 = T1[idx], v1 = T2[idx];
        const double dzx = -al * v0.x + al * v1.x, dzy = -al * v0.y + al * v1.y;
        return make_double2(-e2 * w.y - dzx, e2 * w.x - dzy);
    } else if constexpr (OP == T_VORT2) {  // T0 = w(z), T1 = u(z), T2 = u(z+1)
        const double2 w = T0[idx], u0 = T1[idx], u1 = T2[idx];
        const double dzx = -al * u0.x + al * u1.x, dzy = -al * u0.y + al * u1.y;
        return make_double2(dzx - (-e1 * w.y), dzy - e1 * w.x);
    } else {  // T_VORT3, T0 = v(z), T1 = u(z)
        const double2 v = T0[idx], u = T1[idx];
        return make_double2(-e1 * v.y - (-e2 * u.y), e1 * v.x - e2 * u.x);
    }
}

template <typename R, int A, int B, int OP>
__device__ __forceinline__ void inv_y3_pass1(const InvYArgs& a, const double2* __restrict__ tiles, int tile_elems,
                                             int z, bool ok, double e1, int j, int l, cplx<R>* X1) {
    using C = cplx<R>;
    constexpr int P = A * B, NL = BLD_Y3_NL;
    const int k2max = a.g.k2max, shift = P - a.g.K2;
    const double al = (OP == T_VORT1 || OP == T_VORT2) ? __ldg(a.alpha_i + z) : 0.0;
    const double2* T0 = tiles;
    const double2* T1 = tiles + tile_elems;
    const double2* T2 = tiles + 2 * tile_elems;
    C x[A];
#pragma unroll
    for (int t = 0; t < A; ++t) {
        const int p = j + B * t;
        const int jj = p <= k2max ? p : (p >= P - k2max ? p - shift : -1);
        double2 v = make_double2(0.0, 0.0);
        if (ok && jj >= 0) {
            const double e2 = (OP == T_D2 || OP == T_VORT1 || OP == T_VORT3) ? __ldg(a.d2 + jj) : 0.0;
            v = y3_term<OP>(T0, T1, T2, jj * NL + l, e1, e2, al);
        }
        x[t] = mk<R>((R)v.x, (R)v.y);
    }
    dft<R, A, +1>(x);
#pragma unroll
    for (int q = 0; q < A; ++q) X1[(j * A + q) * NL + l] = x[q];
}

// grid (nterms * members, ceil(K1 / NL), chunks of a.zchunk layers), block B * NL
// threads, dynamic smem y3_smem(P, K2, sizeof(C)).  `smap`: the state as a
// 4-d float64 tensor (2 K1, K2, 3 n3 - 1 layers of the three fields, members)
// with the box (2 NL, K2, 1, 1).
template <typename R, int A, int B>
__global__ void __launch_bounds__(B * BLD_Y3_NL) k_inv_y3(InvYArgs a, const __grid_constant__ CUtensorMap smap) {
    using C = cplx<R>;
    constexpr int P = A * B, NL = BLD_Y3_NL, NT = BLD_Y3_TILES;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const Geo& g = a.g;
    const int K1 = g.K1, K2 = g.K2, n3 = g.n3;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
    C* tw = reinterpret_cast<C*>(smem_raw + 128);
    C* X1 = reinterpret_cast<C*>(smem_raw + 128 + y3_align(P * (int)sizeof(C)));
    const int tile_bytes = y3_align(K2 * NL * 16);
    const int tile_elems = tile_bytes / 16;
    double2* tiles = reinterpret_cast<double2*>(smem_raw + 128 + y3_align(P * (int)sizeof(C)) +
                                                y3_align(P * NL * (int)sizeof(C)));
    const int t = blockIdx.x % a.nterms, m = a.m0 + blockIdx.x / a.nterms;
    BLD_SKIP_INACTIVE(a, m);
    const int op = a.op[t], f = a.fld[t];
    const int nz = a.isI[t] ? n3 - 1 : n3;
    const int z0 = blockIdx.z * a.zchunk, z1 = min(nz, z0 + a.zchunk);
    if (z0 >= z1) return;
    const int k10 = blockIdx.y * NL;
    const int nt = (op == T_VORT1 || op == T_VORT2) ? 3 : (op == T_VORT3 ? 2 : 1);
    // layer index (field * n3 + z) of tile i at layer z
    auto tile_layer = [&](int i, int z) -> int {
        switch (op) {
            case T_VORT1: return i == 0 ? 2 * n3 + z : n3 + z + (i == 2 ? 1 : 0);
            case T_VORT2: return i == 0 ? 2 * n3 + z : z + (i == 2 ? 1 : 0);
            case T_VORT3: return i == 0 ? n3 + z : z;
            default: return f * n3 + z;
        }
    };
    const unsigned stage_bytes = (unsigned)(nt * K2 * NL * 16);
    auto issue = [&](int z, int s) {
        mbar_arrive_expect_tx(&bar[s], stage_bytes);
        for (int i = 0; i < nt; ++i)
            tma_load_4d(tiles + (size_t)(s * NT + i) * tile_elems, &smap, 2 * k10, 0, tile_layer(i, z), m, &bar[s]);
    };
    if (threadIdx.x == 0) {
        prefetch_tmap(&smap);
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_async_shared();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        issue(z0, 0);
        if (z0 + 1 < z1) issue(z0 + 1, 1);
    }
    const C* twg = reinterpret_cast<const C*>(a.tw);
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const long long wait_limit = g_bld_wait_limit;
    const int l = threadIdx.x % NL, j = threadIdx.x / NL;
    const int k1 = k10 + l;
    const bool ok = k1 < K1;
    const double e1 = ok ? __ldg(a.d1 + k1) : 0.0;
    C* outm = reinterpret_cast<C*>(a.mixed) + (long long)m * a.mixed_mstride + (long long)t * n3 * P * K1 + k1;
    for (int z = z0; z < z1; ++z) {
        const int s = (z - z0) & 1;
        const unsigned parity = ((z - z0) >> 1) & 1;
        const bool arrived = mbar_wait_bounded(&bar[s], parity, wait_limit);
        const double2* ts = tiles + (size_t)s * NT * tile_elems;
        switch (op) {
            case T_DIRECT: inv_y3_pass1<R, A, B, T_DIRECT>(a, ts, tile_elems, z, ok, e1, j, l, X1); break;
            case T_D1: inv_y3_pass1<R, A, B, T_D1>(a, ts, tile_elems, z, ok, e1, j, l, X1); break;
            case T_D2: inv_y3_pass1<R, A, B, T_D2>(a, ts, tile_elems, z, ok, e1, j, l, X1); break;
            case T_VORT1: inv_y3_pass1<R, A, B, T_VORT1>(a, ts, tile_elems, z, ok, e1, j, l, X1); break;
            case T_VORT2: inv_y3_pass1<R, A, B, T_VORT2>(a, ts, tile_elems, z, ok, e1, j, l, X1); break;
            default: inv_y3_pass1<R, A, B, T_VORT3>(a, ts, tile_elems, z, ok, e1, j, l, X1); break;
        }
        // every thread is done with stage s and X1 is complete; a block whose wait
        // expired stops here (uniformly) after the copies it issued have landed
        if (__syncthreads_or(!arrived)) {
            if (threadIdx.x == 0) {
                atomicOr(a.flag + m, BLD_FLAG_TIMEOUT);
                for (int zz = z; zz < min(z1, z + 2); ++zz)
                    mbar_wait_bounded(&bar[(zz - z0) & 1], ((zz - z0) >> 1) & 1);
            }
            return;
        }
        if (threadIdx.x == 0 && z + 2 < z1) {
            fence_async_shared();
            issue(z + 2, s);
        }
        if (j < A) {
            C x[B];
#pragma unroll
            for (int q = 0; q < B; ++q) x[q] = X1[(j + A * q) * NL + l];
#pragma unroll
            for (int q = 1; q < B; ++q) x[q] = c_tw<+1>(x[q], tw[j * q]);
            dft<R, B, +1>(x);
            if (ok) {
                C* out = outm + (long long)z * P * K1;
#pragma unroll
                for (int q = 0; q < B; ++q) out[(long long)(j + A * q) * K1] = x[q];
            }
        }
        __syncthreads();   // X1 is free for the next layer
    }
}
