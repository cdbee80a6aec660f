// Device kernels of the right-hand side, the pressure projection and the
// SSP-RK stage update.  R is the arithmetic type of the physical-domain path
// (double for the plain form, float for the mixed form); the spectral state,
// the linear terms and the pressure solve are always double.
//
// Data flow of one nonlinear process (physical-domain size P1 x P2):
//   k_inv_y  : spectral terms (per z layer, per k1 line) -> complex IFFT along y
//              -> "mixed" array M[term][z][y][k1]                 (get_layer! part 1)
//   k_adv_x / k_sgs_x : per y row, streaming upward in z: c2r along x of two
//              terms packed in one complex FFT, the physical-domain products with
//              their z neighbours, r2c along x of the rates      (get_layer! part 2,
//              the process's add_rates!, add_layer! part 1)
//   k_fwd_y  : complex FFT along y of every rate term, truncation, 1/(P1 P2),
//              D1/D2 prefactors, summed with the linear terms into du
//                                                               (add_layer! part 2)
#pragma once

#include <type_traits>

#include "bld_fft.cuh"
#include "bld_dft.cuh"
#include "bld_warpfft.cuh"
#include "bld_tma.cuh"

#define BLD_MAXT 10
#define BLD_MAXC 4

// the two-pass factorisations compiled (P = A B with A <= B; the transforms of
// bld_ypass2.cuh, the advection x kernel of bld_advx2.cuh and k_sgs_x<.., TP>)
__host__ __device__ constexpr int y2_radix_a(int P) {
    return P == 64 ? 8 : P == 96 ? 8 : P == 128 ? 8 : P == 144 ? 12 : P == 192 ? 12 : P == 256 ? 16 : P == 288 ? 16
         : P == 384 ? 16 : P == 512 ? 16 : P == 768 ? 24 : 0;
}
__host__ __device__ constexpr int y2_radix_b(int P) { return y2_radix_a(P) ? P / y2_radix_a(P) : 0; }

struct Geo {
    int K1, K2, k1max, k2max, n3, F;  // F = K1*K2 modes per layer
    long long mstride;                // complex values per member state (3*n3-1)*F
};

__host__ __device__ __forceinline__ long long fld_off(const Geo& g, int f) { return (long long)f * g.n3 * g.F; }

// inactive ensemble slots (serving) skip their blocks; uniform per block
#define BLD_SKIP_INACTIVE(a, m) \
    if ((a).active && !(a).active[m]) return

// Copies n table entries from global to shared memory with up to 8 loads in
// flight per thread (a load-then-store loop would wait one DRAM latency per entry).
template <typename C>
__device__ __forceinline__ void copy_table(C* dst, const C* __restrict__ src, int n) {
    constexpr int B = 8;
    for (int i0 = 0; i0 < n; i0 += B * blockDim.x) {
        C v[B];
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            if (i < n) v[q] = __ldg(src + i);
        }
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            if (i < n) dst[i] = v[q];
        }
    }
}

// The twiddles of a block's transforms in shared memory: for the block-wide
// stages (RAD = 0) the [P] table W_P^(-m) as it is; for the warp transforms
// (P = 32 RAD) the lane-major [RAD][32] table W_P^(-l k), which lane l reads at
// stride 32 without bank conflicts (at stride l, lanes collide for even k)
template <int RAD, typename C>
__device__ __forceinline__ void lane_table(C* dst, const C* __restrict__ src, int P) {
    if constexpr (RAD > 0) {
        for (int i = threadIdx.x; i < P; i += blockDim.x) dst[i] = src[(i >> 5) * (i & 31)];
    } else {
        copy_table(dst, src, P);
    }
}

// ------------------------------------------------------------------ inverse y pass
enum TermOp { T_DIRECT = 0, T_D1 = 1, T_D2 = 2, T_VORT1 = 3, T_VORT2 = 4, T_VORT3 = 5 };

struct InvYArgs {
    Geo g;
    int P2;
    int nterms;
    int op[BLD_MAXT];
    int fld[BLD_MAXT];
    int isI[BLD_MAXT];
    int m0;                      // first member
    int NL;                      // k1 lines per block
    int zchunk;                  // layers per block (k_inv_y3)
    int* flag;                   // [members] error flags (k_inv_y3: a bounded wait expired)
    const int* active;           // [members] 0 = skip the member (NULL: all active)
    const double2* state;
    void* mixed;
    long long mixed_mstride;     // elements per member
    const double* d1;            // [K1] k1 * 2pi/L1
    const double* d2;            // [K2] k2 * 2pi/L2
    const double* alpha_i;       // [n3-1]
    FftPlan plan;
    const void* tw;
};

// value of spectral term `op` at (z, j, k1); D1 = i*d1, D2 = i*d2
// (src/derivatives.jl:67-80,228-230; src/Domains.jl:142-145)
__device__ __forceinline__ double2 inv_term_value(const InvYArgs& a, const double2* __restrict__ S, int op, int f,
                                                  int z, int j, int k1) {
    const Geo& g = a.g;
    const long long mo = (long long)j * g.K1 + k1;
    switch (op) {
        case T_DIRECT:
            return S[fld_off(g, f) + (long long)z * g.F + mo];
        case T_D1: {
            const double2 s = S[fld_off(g, f) + (long long)z * g.F + mo];
            const double d = a.d1[k1];
            return make_double2(-d * s.y, d * s.x);
        }
        case T_D2: {
            const double2 s = S[fld_off(g, f) + (long long)z * g.F + mo];
            const double d = a.d2[j];
            return make_double2(-d * s.y, d * s.x);
        }
        case T_VORT1: {  // D2*w - (-a*v(z) + a*v(z+1))
            const double2 w = S[fld_off(g, 2) + (long long)z * g.F + mo];
            const double2 v0 = S[fld_off(g, 1) + (long long)z * g.F + mo];
            const double2 v1 = S[fld_off(g, 1) + (long long)(z + 1) * g.F + mo];
            const double al = a.alpha_i[z], d = a.d2[j];
            const double dzx = -al * v0.x + al * v1.x, dzy = -al * v0.y + al * v1.y;
            return make_double2(-d * w.y - dzx, d * w.x - dzy);
        }
        case T_VORT2: {  // (-a*u(z) + a*u(z+1)) - D1*w
            const double2 w = S[fld_off(g, 2) + (long long)z * g.F + mo];
            const double2 u0 = S[fld_off(g, 0) + (long long)z * g.F + mo];
            const double2 u1 = S[fld_off(g, 0) + (long long)(z + 1) * g.F + mo];
            const double al = a.alpha_i[z], d = a.d1[k1];
            const double dzx = -al * u0.x + al * u1.x, dzy = -al * u0.y + al * u1.y;
            return make_double2(dzx - (-d * w.y), dzy - d * w.x);
        }
        default: {  // T_VORT3: D1*v - D2*u
            const double2 v = S[fld_off(g, 1) + (long long)z * g.F + mo];
            const double2 u = S[fld_off(g, 0) + (long long)z * g.F + mo];
            const double e1 = a.d1[k1], e2 = a.d2[j];
            return make_double2(-e1 * v.y - (-e2 * u.y), e1 * v.x - e2 * u.x);
        }
    }
}

// grid (ceil(K1/NL), n3, nterms*members); smem: tw[P2] + 2*P2*NL complex
// Gather of one term's K2 x NL modes into the line buffer with the term kind
// fixed at compile time (the loads of a batch are straight-line code).
template <typename R, int OP, int RAD>
__device__ __forceinline__ void gather_term(const InvYArgs& a, const double2* __restrict__ S, int f, int z, int k10,
                                            int nls, int LS, cplx<R>* b0) {
    const int NL = a.NL, K1 = a.g.K1, K2 = a.g.K2, k2max = a.g.k2max, P2 = a.P2;
    constexpr int BATCH = 8;
    const int nmodes = K2 * NL;
    for (int i0 = 0; i0 < nmodes; i0 += BATCH * blockDim.x) {
        double2 v[BATCH];
#pragma unroll
        for (int q = 0; q < BATCH; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            v[q] = make_double2(0.0, 0.0);
            if (i < nmodes) {
                const int j = i >> nls, l = i & (NL - 1), k1 = k10 + l;
                if (k1 < K1) v[q] = inv_term_value(a, S, OP, f, z, j, k1);
            }
        }
#pragma unroll
        for (int q = 0; q < BATCH; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            if (i < nmodes) {
                const int j = i >> nls, l = i & (NL - 1);
                const int p = (j <= k2max) ? j : P2 - (K2 - j);
                b0[swz<cplx<R>, RAD>(p) * LS + l] = mk<R>((R)v[q].x, (R)v[q].y);
            }
        }
    }
}

// grid (nterms*members, ceil(K1/NL), n3): the terms of one (layer, k1 tile) are
// neighbouring blocks, so their shared state reads (vorticity needs z and z+1)
// hit L2.  smem: tw[P2] + 2*P2*NL complex.
// RAD > 0: the transform runs one line per warp in registers (P2 = 32 RAD)
// on a line stride padded to NL + 1, instead of block-wide Stockham stages.
template <typename R, int RAD>
__global__ void __launch_bounds__(256) k_inv_y(InvYArgs a) {
    using C = cplx<R>;
    const int NL = a.NL;
    const int LS = RAD ? NL + 1 : NL;   // stride of a position in the line buffer
    const int nls = __ffs(NL) - 1;     // NL is a power of two
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* b0 = tw + a.P2;
    C* b1 = b0 + a.P2 * NL;
    const int t = blockIdx.x % a.nterms, m = a.m0 + blockIdx.x / a.nterms;
    BLD_SKIP_INACTIVE(a, m);
    const int z = blockIdx.z;
    const int nz = a.isI[t] ? a.g.n3 - 1 : a.g.n3;
    if (z >= nz) return;
    const int op = a.op[t], f = a.fld[t];
    const int K1 = a.g.K1, K2 = a.g.K2, k2max = a.g.k2max, P2 = a.P2;
    const int k10 = blockIdx.y * NL;
    const C* twg = reinterpret_cast<const C*>(a.tw);
    lane_table<RAD>(tw, twg, P2);
    const double2* S = a.state + (long long)m * a.g.mstride;
    // zero the padding band, then gather the K2*NL modes in batches of 8 per thread
    for (int i = threadIdx.x; i < (P2 - K2) * NL; i += blockDim.x) {
        const int p = k2max + 1 + (i >> nls), l = i & (NL - 1);
        b0[swz<C, RAD>(p) * LS + l] = mk<R>(0, 0);
    }
    switch (op) {
        case T_DIRECT: gather_term<R, T_DIRECT, RAD>(a, S, f, z, k10, nls, LS, b0); break;
        case T_D1: gather_term<R, T_D1, RAD>(a, S, f, z, k10, nls, LS, b0); break;
        case T_D2: gather_term<R, T_D2, RAD>(a, S, f, z, k10, nls, LS, b0); break;
        case T_VORT1: gather_term<R, T_VORT1, RAD>(a, S, f, z, k10, nls, LS, b0); break;
        case T_VORT2: gather_term<R, T_VORT2, RAD>(a, S, f, z, k10, nls, LS, b0); break;
        default: gather_term<R, T_VORT3, RAD>(a, S, f, z, k10, nls, LS, b0); break;
    }
    __syncthreads();
    C* res = b0;
    if constexpr (RAD > 0) {
        const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        const int brl = (int)(__brev((unsigned)lane) >> 27);
        LaneTw<R> lt;
        lane_twiddles_tab<R>(lt, lane, twg, P2);
        for (int l = threadIdx.x >> 5; l < NL; l += nw) {
            C zl[RAD];
#pragma unroll
            for (int q = 0; q < RAD; ++q) zl[q] = b0[swz<C, RAD>(lane + 32 * q) * LS + l];
            inverse_line<R, RAD>(zl, lane, tw + lane, 32, lt);
#pragma unroll
            for (int k = 0; k < RAD; ++k) b0[swz<C, RAD>(k + RAD * brl) * LS + l] = zl[k];
        }
        __syncthreads();
    } else {
        res = fft_big<R, +1>(b0, b1, NL, 1, NL, false, a.plan, tw);
    }
    C* out = reinterpret_cast<C*>(a.mixed) + (long long)m * a.mixed_mstride + (long long)(t * a.g.n3 + z) * P2 * K1;
    if constexpr (sizeof(C) == 8) {
        // single precision: two neighbouring modes per 16-byte store (rows and
        // tiles start at even k1 when K1 is even)
        if ((K1 & 1) == 0 && NL >= 2) {
            const int half = NL >> 1;
            for (int i = threadIdx.x; i < P2 * half; i += blockDim.x) {
                const int y = i >> (nls - 1), l = 2 * (i & (half - 1)), k1 = k10 + l;
                if (k1 < K1) {
                    const int ry = swz<C, RAD>(y) * LS;
                    const C v0 = res[ry + l], v1 = res[ry + l + 1];
                    *reinterpret_cast<float4*>(out + (long long)y * K1 + k1) = make_float4(v0.x, v0.y, v1.x, v1.y);
                }
            }
            return;
        }
    }
    for (int i = threadIdx.x; i < P2 * NL; i += blockDim.x) {
        const int y = i >> nls, l = i & (NL - 1), k1 = k10 + l;
        if (k1 < K1) out[(long long)y * K1 + k1] = res[swz<C, RAD>(y) * LS + l];
    }
}

// value of spectral term `op` from the preloaded mode values of layer z (u, v, w)
// and z+1 (u1, v1); same arithmetic as inv_term_value
__device__ __forceinline__ double2 term_from(int op, int f, double2 u, double2 v, double2 w, double2 u1, double2 v1,
                                             double e1, double e2, double al) {
    switch (op) {
        case T_DIRECT:
            return f == 0 ? u : (f == 1 ? v : w);
        case T_D1: {
            const double2 q = f == 0 ? u : (f == 1 ? v : w);
            return make_double2(-e1 * q.y, e1 * q.x);
        }
        case T_D2: {
            const double2 q = f == 0 ? u : (f == 1 ? v : w);
            return make_double2(-e2 * q.y, e2 * q.x);
        }
        case T_VORT1: {
            const double dzx = -al * v.x + al * v1.x, dzy = -al * v.y + al * v1.y;
            return make_double2(-e2 * w.y - dzx, e2 * w.x - dzy);
        }
        case T_VORT2: {
            const double dzx = -al * u.x + al * u1.x, dzy = -al * u.y + al * u1.y;
            return make_double2(dzx - (-e1 * w.y), dzy - e1 * w.x);
        }
        default:
            return make_double2(-e1 * v.y - (-e2 * u.y), e1 * v.x - e2 * u.x);
    }
}

// Inverse y pass of every term of a process at one layer: one block per
// (k1 tile of NL lines, layer z, member); u, v, w at z and u, v at z+1 are read
// once per mode and all nterms*NL lines are transformed together, in place.
// grid (ceil(K1/NL), n3, members); smem tw[P2] + P2*nterms*NL complex.
template <typename R>
__global__ void __launch_bounds__(384) k_inv_y_all(InvYArgs a) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NL = a.NL, nt = a.nterms, NLT = nt * NL;
    const Geo& g = a.g;
    const int K1 = g.K1, K2 = g.K2, k2max = g.k2max, P2 = a.P2, n3 = g.n3;
    const int k10 = blockIdx.x * NL;
    const int nls = __ffs(NL) - 1;   // NL is a power of two
    const int z = blockIdx.y;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    const bool hasI = z < n3 - 1;
    BLD_SKIP_INACTIVE(a, m);
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + P2;
    copy_table(tw, reinterpret_cast<const C*>(a.tw), P2);
    bool needW = false, needUp = false;
    for (int t = 0; t < nt; ++t) {
        needW |= (a.op[t] >= T_VORT1 && a.op[t] <= T_VORT2) || a.fld[t] == 2;
        needUp |= (a.op[t] == T_VORT1 || a.op[t] == T_VORT2);
    }
    needW &= hasI;
    needUp &= hasI;
    const int band = P2 - K2;
    for (int i = threadIdx.x; i < band * NLT; i += blockDim.x) {
        const int p = k2max + 1 + i / NLT, L = i - (i / NLT) * NLT;
        buf[p * NLT + L] = mk<R>(0, 0);
    }
    const double2* S = a.state + (long long)m * g.mstride;
    const long long Fz = (long long)g.F;
    const double2* Su = S + (long long)z * Fz;
    const double2* Sv = S + (long long)n3 * Fz + (long long)z * Fz;
    const double2* Sw = S + 2LL * n3 * Fz + (long long)z * Fz;
    const int nmodes = K2 * NL;
    constexpr int B = 4;
    for (int i0 = 0; i0 < nmodes; i0 += B * blockDim.x) {
        double2 u[B], v[B], w[B], u1[B], v1[B];
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            const int j = i >> nls, l = i & (NL - 1), k1 = k10 + l;
            u[q] = v[q] = w[q] = u1[q] = v1[q] = make_double2(0.0, 0.0);
            if (i < nmodes && k1 < K1) {
                const long long mo = (long long)j * K1 + k1;
                u[q] = Su[mo];
                v[q] = Sv[mo];
                if (needW) w[q] = Sw[mo];
                if (needUp) {
                    u1[q] = Su[Fz + mo];
                    v1[q] = Sv[Fz + mo];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            if (i >= nmodes) continue;
            const int j = i >> nls, l = i & (NL - 1), k1 = k10 + l;
            const int p = (j <= k2max) ? j : P2 - (K2 - j);
            const bool ok = k1 < K1;
            const double e1 = ok ? a.d1[k1] : 0.0, e2 = a.d2[j];
            const double al = hasI ? a.alpha_i[z] : 0.0;
            for (int t = 0; t < nt; ++t) {
                double2 val = make_double2(0.0, 0.0);
                if (ok && (!a.isI[t] || hasI)) val = term_from(a.op[t], a.fld[t], u[q], v[q], w[q], u1[q], v1[q], e1, e2, al);
                buf[p * NLT + t * NL + l] = mk<R>((R)val.x, (R)val.y);
            }
        }
    }
    __syncthreads();
    fft_inplace<R, +1>(buf, NLT, 1, NLT, false, a.plan, tw);
    C* outbase = reinterpret_cast<C*>(a.mixed) + (long long)m * a.mixed_mstride;
    for (int i = threadIdx.x; i < P2 * NLT; i += blockDim.x) {
        const int y = i / NLT, L = i - y * NLT;
        const int t = L / NL, l = L - t * NL, k1 = k10 + l;
        if (k1 < K1 && (!a.isI[t] || hasI))
            outbase[((long long)(t * n3 + z) * P2 + y) * K1 + k1] = buf[i];
    }
}

// ----------------------------------------------------------- physical x kernels
struct XArgs {
    Geo g;
    int P1, P2, YT, zchunk;
    int m0;
    const int* active;
    const void* min;
    void* mout;
    long long min_mstride, mout_mstride;  // elements per member
    FftPlan plan;
    const void* tw;
    // SGS only
    const double* alpha_c;   // [n3]
    const double* alpha_i;   // [n3-1]
    const double* lc;        // [members][n3]   Smagorinsky length^2 at C nodes
    const double* li;        // [members][n3-1] ... at I nodes
    const double* wall;      // [members][4]: strain factor lo, hi; stress factor lo, hi
    int dyn_lo, dyn_hi;      // rough wall (dynamic wall-model values) below / above
    double w_lo, w_hi;       // Dirichlet values of vel3
    // two-pass SGS kernel: the input rows of layer j + 1 are copied into shared
    // memory by 1-d TMA bulk copies while layer j is processed (needs YT K1
    // elements to fill whole 16-byte units); a timed-out wait sets flag[m]
    int staged;
    int* flag;
    // ceil(2^32 / K1) and ceil(2^32 / P1) (0 for a divisor of 1): fdiv
    unsigned k1_magic, p1_magic;
};

// n / d for 0 <= n < 2^16 and 1 <= d < 2^16 by one multiply-high with
// magic = ceil(2^32 / d) (0 for d = 1): with n = q d + r, n magic / 2^32 exceeds
// n / d by less than 2^-16 <= 1 / d, so its floor is q.  Replaces runtime integer
// divisions (tens of instructions each) in the index arithmetic of the x kernels.
__host__ __device__ __forceinline__ int fdiv(int n, unsigned magic) {
#ifdef __CUDA_ARCH__
    return magic ? (int)__umulhi((unsigned)n, magic) : n;
#else
    return magic ? (int)(((unsigned long long)(unsigned)n * magic) >> 32) : n;
#endif
}
inline unsigned fdiv_magic(unsigned d) { return d <= 1 ? 0u : (unsigned)(((1ull << 32) + d - 1) / d); }

template <typename C>
__device__ __forceinline__ const C* mrow(const C* M, const XArgs& a, int t, int z, int y) {
    return M + ((long long)(t * a.g.n3 + z) * a.P2 + y) * a.g.K1;
}
template <typename C>
__device__ __forceinline__ C* mrow_w(C* M, const XArgs& a, int t, int z, int y) {
    return M + ((long long)(t * a.g.n3 + z) * a.P2 + y) * a.g.K1;
}

// Build packed line Z[k] = A[k] + i B[k] (Hermitian-extended, DC imaginary parts
// dropped as in FFTW's c2r) from mixed rows A (term ta) and B (term tb).
template <typename R>
__device__ __forceinline__ void build_packed(cplx<R>* line, const cplx<R>* rowA, const cplx<R>* rowB, int k, int P1) {
    using C = cplx<R>;
    C A = rowA ? rowA[k] : mk<R>(0, 0);
    C B = rowB ? rowB[k] : mk<R>(0, 0);
    if (k == 0) {
        line[0] = mk<R>(A.x, B.x);
    } else {
        line[k] = mk<R>(A.x - B.y, A.y + B.x);          // A + iB
        line[P1 - k] = mk<R>(A.x + B.y, -A.y + B.x);    // conj(A) + i conj(B)
    }
}

// RAD > 0: the line is stored on swizzled positions (swz, bld_warpfft.cuh)
template <typename R, int RAD = 0>
__device__ __forceinline__ void put_packed(cplx<R>* line, cplx<R> A, cplx<R> B, int k, int P1) {
    using C = cplx<R>;
    if (k == 0) {
        line[0] = mk<R>(A.x, B.x);
    } else {
        line[swz<C, RAD>(k)] = mk<R>(A.x - B.y, A.y + B.x);
        line[swz<C, RAD>(P1 - k)] = mk<R>(A.x + B.y, -A.y + B.x);
    }
}

// Unpack forward FFT Z of a + ib: A[k] = (Z[k] + conj(Z[-k]))/2, B[k] = (Z[k] - conj(Z[-k]))/(2i)
template <typename R, int RAD = 0>
__device__ __forceinline__ void unpack_pair(const cplx<R>* line, int k, int P1, cplx<R>& A, cplx<R>& B) {
    using C = cplx<R>;
    const cplx<R> Zk = line[swz<C, RAD>(k)];
    const cplx<R> Zr = line[swz<C, RAD>(k == 0 ? 0 : P1 - k)];
    A = mk<R>((Zk.x + Zr.x) * R(0.5), (Zk.y - Zr.y) * R(0.5));
    const R dx = Zk.x - Zr.x, dy = Zk.y + Zr.y;
    B = mk<R>(dy * R(0.5), -dx * R(0.5));
}

// Rotation-form advection (src/processes/momentum_advection.jl:44-206).
// Inputs: terms 0 u, 1 v, 5 vort3 (C); 2 w, 3 vort1, 4 vort2 (I).
// Outputs: 0 adv1, 1 adv2 (C); 2 adv3 (I).
// grid (P2/YT, nchunks, members), block YT*P1/PPT <= 256 threads.
// RAD > 0: the x transforms run one line per warp in registers (P1 = 32 RAD).
template <typename R, int PPT, int RAD>
__global__ void __launch_bounds__(256) k_adv_x(XArgs a) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int P1 = a.P1, YT = a.YT, n3 = a.g.n3, k1max = a.g.k1max;
    const int NLin = 3 * YT, NLout = YT + (YT + 1) / 2;
    // two line buffers of NLin lines: inputs/physical values and outputs ping-pong
    // between them; RAD > 0: swizzled positions on a line stride P1 + 32
    const int LP = RAD ? P1 + 32 : P1;
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* bufA = tw + P1;
    C* bufB = bufA + NLin * LP;
    const int y0 = blockIdx.x * YT;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    const int z0 = blockIdx.y * a.zchunk;
    const int z1 = min(n3, z0 + a.zchunk);
    const int nthr = blockDim.x;
    const C* twg = reinterpret_cast<const C*>(a.tw);
    lane_table<RAD>(tw, twg, P1);
    const C* Min = reinterpret_cast<const C*>(a.min) + (long long)m * a.min_mstride;
    C* Mout = reinterpret_cast<C*>(a.mout) + (long long)m * a.mout_mstride;

    R pu[PPT], pv[PPT], pw[PPT], po1[PPT], po2[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) pu[i] = pv[i] = pw[i] = po1[i] = po2[i] = R(0);

    for (int j = max(0, z0 - 1); j < z1; ++j) {
        const bool hasI = (j < n3 - 1);
        C* cur = bufA;
        // ---- build packed input lines: (u, v), (vort3, w), (vort1, vort2) per y;
        // zero band first, then the resolved modes with 4 rows in flight per thread
        const int nk = k1max + 1;
        for (int i = threadIdx.x; i < NLin * (P1 - 2 * k1max - 1); i += nthr) {
            const int line = i / (P1 - 2 * k1max - 1), k = k1max + 1 + i % (P1 - 2 * k1max - 1);
            cur[line * LP + swz<C, RAD>(k)] = mk<R>(0, 0);
        }
        for (int i0 = 0; i0 < NLin * nk; i0 += 4 * nthr) {
            C va[4], vb[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = i0 + q * nthr + threadIdx.x;
                va[q] = vb[q] = mk<R>(0, 0);
                if (i < NLin * nk) {
                    const int line = fdiv(i, a.k1_magic), k = i - line * nk;
                    const int yl = line / 3, qq = line - yl * 3, y = y0 + yl;
                    // packed line qq: terms (0,1) (5,2) (3,4); w and the I-node
                    // vorticities only below the top layer (branch-free loads)
                    const int ta = (0x350 >> (4 * qq)) & 0xF, tb = (0x421 >> (4 * qq)) & 0xF;
                    const bool oka = qq < 2 || hasI, okb = qq == 0 || hasI;
                    if (oka) va[q] = mrow(Min, a, ta, j, y)[k];
                    if (okb) vb[q] = mrow(Min, a, tb, j, y)[k];
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = i0 + q * nthr + threadIdx.x;
                if (i < NLin * nk) {
                    const int line = fdiv(i, a.k1_magic), k = i - line * nk;
                    put_packed<R, RAD>(cur + line * LP, va[q], vb[q], k, P1);
                }
            }
        }
        __syncthreads();
        C* phys = bufA;
        if constexpr (RAD > 0) {
            warp_lines_inplace<R, RAD, +1>(bufA, NLin, P1, tw, twg);
            __syncthreads();
        } else {
            if constexpr (RAD > 0) {
                warp_lines_inplace<R, RAD, +1>(bufA, NLin, P1, tw, twg);
                __syncthreads();
            } else {
                phys = fft_big<R, +1>(bufA, bufB, NLin, P1, 1, true, a.plan, tw);
            }
        }
        C* outb = (phys == bufA) ? bufB : bufA;
        const bool emitC = (j >= z0);
        const bool emitI = (j >= z0) && (j >= 1);
#pragma unroll
        for (int i = 0; i < PPT; ++i) {
            const int p = threadIdx.x + i * nthr;
            const int yl = fdiv(p, a.p1_magic), x = p - yl * P1;
            const int xs = swz<C, RAD>(x);
            const C c0 = phys[(yl * 3 + 0) * LP + xs];
            const C c1 = phys[(yl * 3 + 1) * LP + xs];
            const C c2 = phys[(yl * 3 + 2) * LP + xs];
            const R u = c0.x, v = c0.y, o3 = c1.x;
            const R w = hasI ? c1.y : R(0);
            const R o1 = hasI ? c2.x : R(0);
            const R o2 = hasI ? c2.y : R(0);
            if (emitC) {
                R adv1, adv2;
                if (j == 0) {  // w below is the (zero) boundary value (:181-184,:194-197)
                    adv1 = o3 * v - R(0.5) * (o2 * w);
                    adv2 = R(0.5) * (o1 * w) - o3 * u;
                } else if (j == n3 - 1) {  // w above is the boundary value (:185-188,:198-201)
                    adv1 = o3 * v - R(0.5) * (po2[i] * pw[i]);
                    adv2 = R(0.5) * (po1[i] * pw[i]) - o3 * u;
                } else {  // (:180,:193)
                    adv1 = o3 * v - R(0.5) * (po2[i] * pw[i] + o2 * w);
                    adv2 = R(0.5) * (po1[i] * pw[i] + o1 * w) - o3 * u;
                }
                outb[yl * LP + xs] = mk<R>(adv1, adv2);
            }
            if (emitI) {  // adv3 on I layer j-1 (:206)
                const R adv3 = po2[i] * R(0.5) * (pu[i] + u) - po1[i] * R(0.5) * (pv[i] + v);
                C* o = outb + (YT + yl / 2) * LP + xs;
                if (yl & 1) {
                    o->y = adv3;
                } else {
                    o->x = adv3;
                    if (yl + 1 >= YT) o->y = R(0);
                }
            }
            pu[i] = u;
            pv[i] = v;
            pw[i] = w;
            po1[i] = o1;
            po2[i] = o2;
        }
        if (emitC) {
            __syncthreads();
            C* r2 = outb;
            if constexpr (RAD > 0) {
                warp_lines_inplace<R, RAD, -1>(outb, NLout, P1, tw, twg);
                __syncthreads();
            } else {
                r2 = fft_big<R, -1>(outb, phys, NLout, P1, 1, true, a.plan, tw);
            }
            const int nk = k1max + 1;
            for (int i = threadIdx.x; i < NLout * nk; i += nthr) {
                const int line = fdiv(i, a.k1_magic), k = i - line * nk;
                C A, B;
                unpack_pair<R, RAD>(r2 + line * LP, k, P1, A, B);
                if (line < YT) {
                    const int y = y0 + line;
                    mrow_w(Mout, a, 0, j, y)[k] = A;
                    mrow_w(Mout, a, 1, j, y)[k] = B;
                } else if (emitI) {
                    const int q = line - YT;
                    const int ya = y0 + 2 * q, yb = ya + 1;
                    mrow_w(Mout, a, 2, j - 1, ya)[k] = A;
                    if (2 * q + 1 < YT) mrow_w(Mout, a, 2, j - 1, yb)[k] = B;
                }
            }
        }
        __syncthreads();
    }
}

// Static Smagorinsky model with the rough-wall model
// (src/processes/static_smagorinsky.jl:129-249, src/derivatives.jl:104-138,235-241).
// Inputs: 0 u, 1 v, 3 u_1, 4 u_2, 5 v_1, 6 v_2 (C); 2 w, 7 w_1, 8 w_2 (I).
// Outputs (physical-domain rates, i.e. minus the SGS stress terms):
//   0 -tau11 (C, D1 -> vel1)   1 -tau12 (C, D2 -> vel1 and D1 -> vel2)
//   2 -tau22 (C, D2 -> vel2)   3 -d3 tau13 (C -> vel1)   4 -d3 tau23 (C -> vel2)
//   5 -d3 tau33 (I -> vel3)    6 -tau13 (I, D1 -> vel3)   7 -tau23 (I, D2 -> vel3)
// Streaming in z with a two-layer lag: step j loads C layer j and I layer j and
// completes C layer j-1, I layer j-1 and the d3 tau33 of I layer j-2.
// RAD > 0: the x transforms run one line per warp in registers (P1 = 32 RAD).
// In-place transforms of `nlines` lines of P = A B points in shared memory
// (point p of line L at buf[L LP + p], natural order in and out) by the two
// passes of the y kernels: pass 1 (B tasks per line, radix-A DFTs of points
// j + B t) into the scratch X1 at q (B + 1) + j of its line, pass 2 (A tasks
// per line, W_P^(DIR j t) then radix-B DFTs) back into buf at j + A q.  `tw2`
// holds W_P^(-j t) as [t][j] (P entries).  X1 needs nlines * twopass_line(A, B)
// values.  All threads of the block call it after a barrier that publishes buf;
// it ends with a barrier.
template <typename C>
__host__ __device__ constexpr int twopass_line(int A, int B) {
    return A * (B + 1) + ((B - A * (B + 1)) % (int)(128 / sizeof(C)) + (int)(128 / sizeof(C))) % (int)(128 / sizeof(C));
}
template <typename R, int A, int B, int DIR>
__device__ __forceinline__ void twopass_inplace(cplx<R>* buf, int nlines, int LP, cplx<R>* X1,
                                                const cplx<R>* __restrict__ tw2) {
    using C = cplx<R>;
    constexpr int X1S = B + 1, X1L = twopass_line<C>(A, B);
    for (int task = threadIdx.x; task < nlines * B; task += blockDim.x) {
        const int L = task / B, jt = task - L * B;
        C x[A];
#pragma unroll
        for (int t = 0; t < A; ++t) x[t] = buf[L * LP + jt + B * t];
        dft<R, A, DIR>(x);
#pragma unroll
        for (int q = 0; q < A; ++q) X1[L * X1L + q * X1S + jt] = x[q];
    }
    __syncthreads();
    for (int task = threadIdx.x; task < nlines * A; task += blockDim.x) {
        const int L = task / A, j2 = task - L * A;
        C x[B];
#pragma unroll
        for (int t = 0; t < B; ++t) x[t] = X1[L * X1L + j2 * X1S + t];
#pragma unroll
        for (int t = 1; t < B; ++t) x[t] = c_tw<DIR>(x[t], tw2[t * A + j2]);
        dft<R, B, DIR>(x);
#pragma unroll
        for (int q = 0; q < B; ++q) buf[L * LP + j2 + A * q] = x[q];
    }
    __syncthreads();
}

// Values the Smagorinsky x pass carries from one layer to the next at one
// (x, y) point: the previous C layer's velocities, strain and |S|^2 terms, and
// the previous I layer's S13, S23, tau13, tau23, tau33.
template <typename R>
struct SgsCarry {
    R u, v, w, w1, w2, s11, s22, s33, s12, sc, s13, s23, t13, t23, t33;
};

// The Smagorinsky model at one (x, y) point of the x pass when C layer j enters
// (src/processes/static_smagorinsky.jl:129-249): strain on C layer j, S13, S23,
// eddy viscosity and tau13, tau23 on I layer j - 1, |S| and the stresses of C
// layer c = j - 1 with the wall model at the boundary layers, d3 tau_i3 by
// stencil; o[0..7] are the packed outputs (tau11, tau12, tau22, d3 tau13,
// d3 tau23, d3 tau33 on I layer c - 1, tau13, tau23 on I layer c), all negated as
// the rates add them.  Updates the carried values.
template <typename R>
__device__ __forceinline__ void sgs_point(const XArgs& a, int j, int n3, bool hasC, const double* lcm,
                                          const double* lim, R fs_lo, R fs_hi, R ft_lo, R ft_hi, R wlo, R u, R v,
                                          R u1, R u2, R v1, R v2, R w, R w1, R w2, SgsCarry<R>& cy, R (&o)[8]) {
    const int c = j - 1;
    // (a) strain on C layer j (vel3_3 by dx3_i2c with Dirichlet w, :202-216)
    R s11 = 0, s22 = 0, s33 = 0, s12 = 0, sc = 0;
    if (hasC) {
        const R ac = (R)a.alpha_c[j];
        const R wb = (j == 0) ? wlo : cy.w;
        s33 = -ac * wb + ac * w;
        s11 = u1;
        s22 = v2;
        s12 = (u2 + v1) / R(2);
        sc = s11 * s11 + s22 * s22 + s33 * s33 + R(2) * (s12 * s12);
    }
    // (b) I layer j-1: S13, S23, eddy viscosity, tau13, tau23
    R s13 = 0, s23 = 0, sg13 = 0, sg23 = 0;
    if (j >= 1 && j <= n3 - 1) {
        const R ai = (R)a.alpha_i[j - 1];
        s13 = ((-ai * cy.u + ai * u) + cy.w1) / R(2);
        s23 = ((-ai * cy.v + ai * v) + cy.w2) / R(2);
        R si = R(2) * (s13 * s13) + R(2) * (s23 * s23);
        R t;
        t = cy.s11 + s11; si += t * t / R(4);
        t = cy.s22 + s22; si += t * t / R(4);
        t = cy.s33 + s33; si += t * t / R(4);
        t = cy.s12 + s12; si += R(2) * (t * t) / R(4);
        const R l2 = (R)lim[j - 1];
        const R evi = sqrt(R(2) * si) * l2;
        sg13 = R(-2) * evi * s13;
        sg23 = R(-2) * evi * s23;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) o[q] = 0;
    R sg33 = 0;
    if (j >= 1) {
        // (c) C layer c = j-1
        R scc = cy.sc;
        // S13 (:232-233); dynamic values are not interpolated (:245-249)
        if (c == 0) {
            if (a.dyn_lo) { const R d = cy.u * fs_lo; scc += R(2) * (d * d); }
            else { const R d = R(0) + s13; scc += R(2) * (d * d) / R(4); }
        } else if (c == n3 - 1) {
            if (a.dyn_hi) { const R d = cy.u * fs_hi; scc += R(2) * (d * d); }
            else { const R d = cy.s13 + R(0); scc += R(2) * (d * d) / R(4); }
        } else {
            const R d = cy.s13 + s13; scc += R(2) * (d * d) / R(4);
        }
        if (c == 0) {
            if (a.dyn_lo) { const R d = cy.v * fs_lo; scc += R(2) * (d * d); }
            else { const R d = R(0) + s23; scc += R(2) * (d * d) / R(4); }
        } else if (c == n3 - 1) {
            if (a.dyn_hi) { const R d = cy.v * fs_hi; scc += R(2) * (d * d); }
            else { const R d = cy.s23 + R(0); scc += R(2) * (d * d) / R(4); }
        } else {
            const R d = cy.s23 + s23; scc += R(2) * (d * d) / R(4);
        }
        const R evc = sqrt(R(2) * scc) * (R)lcm[c];
        o[0] = -(R(-2) * evc * cy.s11);
        o[2] = -(R(-2) * evc * cy.s22);
        sg33 = R(-2) * evc * cy.s33;
        o[1] = -(R(-2) * evc * cy.s12);
        // wall stress (stress_bc, :195-200) from the wall-adjacent C layer
        const R uh = sqrt(cy.u * cy.u + cy.v * cy.v);
        const R b13lo = a.dyn_lo ? ft_lo * cy.u * uh : R(0);
        const R b23lo = a.dyn_lo ? ft_lo * cy.v * uh : R(0);
        const R b13hi = a.dyn_hi ? ft_hi * cy.u * uh : R(0);
        const R b23hi = a.dyn_hi ? ft_hi * cy.v * uh : R(0);
        const R below13 = (c == 0) ? b13lo : cy.t13;
        const R below23 = (c == 0) ? b23lo : cy.t23;
        const R above13 = (c == n3 - 1) ? b13hi : sg13;
        const R above23 = (c == n3 - 1) ? b23hi : sg23;
        const R ac = (R)a.alpha_c[c];
        o[3] = -(-ac * below13 + ac * above13);
        o[4] = -(-ac * below23 + ac * above23);
        if (c >= 1) {  // d3 tau33 on I layer c-1 (dx3_c2i!, :363)
            const R ai = (R)a.alpha_i[c - 1];
            o[5] = -(-ai * cy.t33 + ai * sg33);
        }
        o[6] = -sg13;
        o[7] = -sg23;
    }
    // (d) carry
    if (j >= 1 && j <= n3 - 1) {
        cy.s13 = s13;
        cy.s23 = s23;
        cy.t13 = sg13;
        cy.t23 = sg23;
    }
    if (j >= 1) cy.t33 = sg33;
    if (hasC) {
        cy.s11 = s11; cy.s22 = s22; cy.s33 = s33; cy.s12 = s12; cy.sc = sc;
        cy.u = u; cy.v = v; cy.w = w; cy.w1 = w1; cy.w2 = w2;
    }
}

// byte offset of the staging area of the two-pass SGS x kernel: after the
// twiddles and the two line buffers, rounded up to 128 bytes; the area holds
// the two barriers (128 bytes) and 2 x 9 staged rows of YT K1 values
__host__ __device__ constexpr int sgs_stage_offset(int P1, int NLin, int LP, int csz) {
    return ((P1 + 2 * NLin * LP) * csz + 127) & ~127;
}

// TP > 0: the x transforms of a compile-time P1 = TP by twopass_inplace (the
// other buffer is the scratch; lines at stride twopass_line), RAD must be 0
template <typename R, int PPT, int RAD, int TP = 0, int MINB = 0>
__global__ void __launch_bounds__(256, MINB) k_sgs_x(XArgs a) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int P1 = a.P1, YT = a.YT, n3 = a.g.n3, k1max = a.g.k1max;
    const int NLin = 5 * YT, NLout = 4 * YT;
    constexpr int TA = TP ? y2_radix_a(TP) : 1, TB = TP ? y2_radix_b(TP) : 1;
    // RAD > 0: swizzled positions on a padded line stride; TP > 0: the two-pass scratch stride
    const int LP = TP ? twopass_line<C>(TA, TB) : (RAD ? P1 + 32 : P1);
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* bufA = tw + P1;
    C* bufB = bufA + NLin * LP;
    const int y0 = blockIdx.x * YT;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    const int z0 = blockIdx.y * a.zchunk;
    const int z1 = min(n3, z0 + a.zchunk);
    const int nthr = blockDim.x;
    // staging (two-pass form): barriers and 2 x 9 terms x YT rows after the line
    // buffers, on 128-byte boundaries (sgs_stage_offset)
    const bool staged = TP > 0 && a.staged;
    const int K1 = a.g.K1;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + sgs_stage_offset(P1, NLin, LP, (int)sizeof(C)));
    C* stage = reinterpret_cast<C*>(reinterpret_cast<unsigned char*>(bar) + 128);
    const unsigned row_bytes = (unsigned)(YT * K1 * (int)sizeof(C));
    const long long wait_limit = g_bld_wait_limit;
    const int jb = max(0, z0 - 2);
    // input terms of C layer j: u, v, u1, u2, v1, v2, and below the top layer w, w1, w2
    auto issue = [&](int j, int sl) {
        const bool hi = (j <= n3 - 2);
        mbar_arrive_expect_tx(&bar[sl], (hi ? 9u : 6u) * row_bytes);
        for (int t = 0; t < 9; ++t)
            if (hi || (t != 2 && t != 7 && t != 8))
                bulk_load(stage + (size_t)(sl * 9 + t) * YT * K1, mrow(reinterpret_cast<const C*>(a.min) +
                                                                          (long long)m * a.min_mstride, a, t, j, y0),
                          row_bytes, &bar[sl]);
    };
    if (staged) {
        if (threadIdx.x == 0) {
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
            fence_async_shared();
        }
        __syncthreads();
        if (threadIdx.x == 0 && jb <= n3 - 1) issue(jb, 0);
    }
    const C* twg = reinterpret_cast<const C*>(a.tw);
    if constexpr (TP > 0) {
        for (int i = threadIdx.x; i < TP; i += blockDim.x) tw[i] = twg[(i / TA) * (i % TA)];
    } else {
        lane_table<RAD>(tw, twg, P1);
    }
    const C* Min = reinterpret_cast<const C*>(a.min) + (long long)m * a.min_mstride;
    C* Mout = reinterpret_cast<C*>(a.mout) + (long long)m * a.mout_mstride;
    const double* lcm = a.lc + (long long)m * n3;
    const double* lim = a.li + (long long)m * (n3 - 1);
    const R fs_lo = (R)a.wall[4 * m + 0], fs_hi = (R)a.wall[4 * m + 1];
    const R ft_lo = (R)a.wall[4 * m + 2], ft_hi = (R)a.wall[4 * m + 3];
    const R wlo = (R)a.w_lo, whi = (R)a.w_hi;

    SgsCarry<R> cy[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) cy[i] = SgsCarry<R>{};

    const int jend = min(n3, z1 + 1);
    for (int j = jb; j <= jend; ++j) {
        const bool hasC = (j <= n3 - 1), hasI = (j <= n3 - 2);
        C* cur = bufA;
        C* phys = bufA;
        const int sl = (j - jb) & 1;
        bool arrived = true;
        if (staged && hasC) {
            // slot sl ^ 1 was last read by layer j - 1's packing, several barriers ago
            if (threadIdx.x == 0 && j + 1 <= min(jend, n3 - 1)) {
                fence_async_shared();
                issue(j + 1, sl ^ 1);
            }
            arrived = mbar_wait_bounded(&bar[sl], ((j - jb) >> 1) & 1, wait_limit);
        }
        const C* srow = stage + (size_t)sl * 9 * YT * K1;
        if (hasC) {
            const int nk = k1max + 1;
            for (int i = threadIdx.x; i < NLin * (P1 - 2 * k1max - 1); i += nthr) {
                const int line = i / (P1 - 2 * k1max - 1), k = k1max + 1 + i % (P1 - 2 * k1max - 1);
                cur[line * LP + swz<C, RAD>(k)] = mk<R>(0, 0);
            }
            for (int i0 = 0; i0 < NLin * nk; i0 += 4 * nthr) {
                C va[4], vb[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int i = i0 + q * nthr + threadIdx.x;
                    va[q] = vb[q] = mk<R>(0, 0);
                    if (i < NLin * nk) {
                        const int line = fdiv(i, a.k1_magic), k = i - line * nk;
                        const int yl = line / 5, qq = line - yl * 5, y = y0 + yl;
                        // packed line qq: terms (0,1) (3,4) (5,6) (2,7) (8,-), the last two
                        // only below the top layer; table lookups keep the loads branch-free
                        const int ta = (0x82530 >> (4 * qq)) & 0xF, tb = (0xF7641 >> (4 * qq)) & 0xF;
                        const bool oka = qq < 3 || hasI, okb = qq < 3 || (qq == 3 && hasI);
                        if (staged) {
                            if (oka) va[q] = srow[(ta * YT + yl) * K1 + k];
                            if (okb) vb[q] = srow[(tb * YT + yl) * K1 + k];
                        } else {
                            if (oka) va[q] = mrow(Min, a, ta, j, y)[k];
                            if (okb) vb[q] = mrow(Min, a, tb, j, y)[k];
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int i = i0 + q * nthr + threadIdx.x;
                    if (i < NLin * nk) {
                        const int line = fdiv(i, a.k1_magic), k = i - line * nk;
                        put_packed<R, RAD>(cur + line * LP, va[q], vb[q], k, P1);
                    }
                }
            }
            // a block whose staged wait expired stops here (uniformly), after the
            // copies it issued have landed
            if (__syncthreads_or(!arrived)) {
                if (threadIdx.x == 0) {
                    atomicOr(a.flag + m, BLD_FLAG_TIMEOUT);
                    mbar_wait_bounded(&bar[sl], ((j - jb) >> 1) & 1);
                    if (j + 1 <= min(jend, n3 - 1)) mbar_wait_bounded(&bar[sl ^ 1], ((j + 1 - jb) >> 1) & 1);
                }
                return;
            }
            if constexpr (TP > 0) {
                twopass_inplace<R, TA, TB, +1>(bufA, NLin, LP, bufB, tw);
            } else if constexpr (RAD > 0) {
                warp_lines_inplace<R, RAD, +1>(bufA, NLin, P1, tw, twg);
                __syncthreads();
            } else {
                phys = fft_big<R, +1>(bufA, bufB, NLin, P1, 1, true, a.plan, tw);
            }
        }
        C* outb = (phys == bufA) ? bufB : bufA;
        const int c = j - 1;                                   // C layer completed at this step
        const bool doC = (j >= 1) && (c >= z0) && (c < z1);
        const bool do67 = (j >= 1) && (j <= n3 - 1) && (c >= z0) && (c < z1);
        const bool do5 = (j >= 2) && (j - 2 >= z0) && (j - 2 < z1) && (j - 2 <= n3 - 2);
#pragma unroll
        for (int i = 0; i < PPT; ++i) {
            const int p = threadIdx.x + i * nthr;
            const int yl = fdiv(p, a.p1_magic), x = p - yl * P1;
            R u = 0, v = 0, u1 = 0, u2 = 0, v1 = 0, v2 = 0, w = whi, w1 = 0, w2 = 0;
            const int xs = swz<C, RAD>(x);
            if (hasC) {
                const C c0 = phys[(yl * 5 + 0) * LP + xs], c1 = phys[(yl * 5 + 1) * LP + xs];
                const C c2 = phys[(yl * 5 + 2) * LP + xs];
                u = c0.x; v = c0.y; u1 = c1.x; u2 = c1.y; v1 = c2.x; v2 = c2.y;
                if (hasI) {
                    const C c3 = phys[(yl * 5 + 3) * LP + xs], c4 = phys[(yl * 5 + 4) * LP + xs];
                    w = c3.x; w1 = c3.y; w2 = c4.x;
                }
            }
            R o[8];
            sgs_point<R>(a, j, n3, hasC, lcm, lim, fs_lo, fs_hi, ft_lo, ft_hi, wlo, u, v, u1, u2, v1, v2, w, w1, w2,
                         cy[i], o);
            if (doC || do5) {
#pragma unroll
                for (int q = 0; q < 4; ++q) outb[(yl * 4 + q) * LP + xs] = mk<R>(o[2 * q], o[2 * q + 1]);
            }
        }
        if (doC || do5) {
            __syncthreads();
            C* r2 = outb;
            if constexpr (TP > 0) {
                twopass_inplace<R, TA, TB, -1>(outb, NLout, LP, phys, tw);
            } else if constexpr (RAD > 0) {
                warp_lines_inplace<R, RAD, -1>(outb, NLout, P1, tw, twg);
                __syncthreads();
            } else {
                r2 = fft_big<R, -1>(outb, phys, NLout, P1, 1, true, a.plan, tw);
            }
            const int nk = k1max + 1;
            for (int i = threadIdx.x; i < NLout * nk; i += nthr) {
                const int line = fdiv(i, a.k1_magic), k = i - line * nk;
                const int yl = line / 4, q = line - yl * 4, y = y0 + yl;
                C A, B;
                unpack_pair<R, RAD>(r2 + line * LP, k, P1, A, B);
                // pairs (0,1) (2,3) (4,5) (6,7)
                const int ta = 2 * q, tb = 2 * q + 1;
                if (ta <= 4) {
                    if (doC) mrow_w(Mout, a, ta, c, y)[k] = A;
                } else if (do67) {
                    mrow_w(Mout, a, ta, c, y)[k] = A;
                }
                if (tb <= 4) {
                    if (doC) mrow_w(Mout, a, tb, c, y)[k] = B;
                } else if (tb == 5) {
                    if (do5) mrow_w(Mout, a, 5, j - 2, y)[k] = B;
                } else if (do67) {
                    mrow_w(Mout, a, tb, c, y)[k] = B;
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ forward y pass
struct FwdContrib {
    int term;  // mixed output term index
    int pref;  // 0 none, 1 D1, 2 D2
};

struct Linear {
    int diff_on[3];
    double nu[3];
    const double* DD1;        // [K1]
    const double* DD2;        // [K2]
    const double* alpha_c;    // [n3]
    const double* alpha_i;    // [n3-1]
    const double* alpha_ext;  // [n3+1] alpha at I positions incl. boundaries
    int bc_kind[3][2];
    double bc_val[3][2];      // Dirichlet value
    double bc_diff[3][2];     // Neumann gradient * dx3 (ConstantGradient.difference)
    int src_on[3];
    const double* src;        // [members][3]
};

struct FwdYArgs {
    Geo g;
    int P1, P2;
    const void* mout;
    long long mout_mstride;
    int ncontrib[3];
    FwdContrib c[3][BLD_MAXC];
    int mode;                  // 0: du += acc; 1: du = linear + acc; 2: du = acc (transform only)
    int check;                 // set *flag on a non-finite result
    double2* du;               // member stride g.mstride
    long long du_mstride;
    // fused stage update (k_fwd_y, modes 0 and 1): instead of the rate d, write
    // sout = (st_cu su + st_ct state + st_cd d) * st_inv, the explicit
    // SSP-RK stage value that the projection would otherwise form from d
    // (src/ODEMethods.jl:101,143,157,164; the reference divides by 2, 3 or 4,
    // here the host passes the reciprocal: exact for 2 and 4, within one
    // rounding of the quotient for 3); su (NULL: no su term, st_ct = st_inv = 1)
    // and sout have the member stride of du
    int fuse;
    const double2* su;
    double2* sout;
    double st_cu, st_ct, st_cd, st_inv;
    const double2* state;
    Linear lin;
    const double* d1;
    const double* d2;
    double inv_n;              // 1/(P1*P2)
    int* flag;                 // per member
    int fields;                // number of target fields (3 for rates, 1 for transforms)
    int field0;                // first target field
    int m0;                    // first member
    int NL;                    // k1 lines per block
    const int* active;
    FftPlan plan;
    const void* tw;
};

// Frequency-domain Laplacian with ghost layers (src/processes/molecular_diffusion.jl:57-72,
// src/boundary_conditions.jl:254-359) and the constant source (src/processes/sources.jl:32-35).
__device__ __forceinline__ double2 linear_terms(const Geo& g, const Linear& L, const double2* __restrict__ S, int f,
                                                int z, int j, int k1, int m) {
    double2 val = make_double2(0.0, 0.0);
    const long long mo = (long long)j * g.K1 + k1;
    const bool mean_mode = (j == 0 && k1 == 0);
    if (L.diff_on[f]) {
        const double2* Sf = S + fld_off(g, f);
        const int n = (f == 2) ? g.n3 - 1 : g.n3;
        const double2 q0 = Sf[(long long)z * g.F + mo];
        double2 qm, qp;
        double A, B, Cc;
        if (f != 2) {
            A = L.alpha_ext[z];
            B = L.alpha_c[z];
            Cc = L.alpha_ext[z + 1];
            if (z == 0) {
                const double2 l1 = Sf[mo], l2 = Sf[g.F + mo], l3 = Sf[2LL * g.F + mo];
                if (L.bc_kind[f][0] == 0) {
                    qm.x = (-15.0 * l1.x + 5.0 * l2.x - l3.x) / 5.0;
                    qm.y = (-15.0 * l1.y + 5.0 * l2.y - l3.y) / 5.0;
                    if (mean_mode) qm.x += 16.0 * L.bc_val[f][0] / 5.0;
                } else {
                    qm.x = (21.0 * l1.x + 3.0 * l2.x - l3.x) / 23.0;
                    qm.y = (21.0 * l1.y + 3.0 * l2.y - l3.y) / 23.0;
                    if (mean_mode) qm.x -= 24.0 * L.bc_diff[f][0] / 23.0;
                }
            } else {
                qm = Sf[(long long)(z - 1) * g.F + mo];
            }
            if (z == n - 1) {
                const double2 l1 = Sf[(long long)(n - 1) * g.F + mo], l2 = Sf[(long long)(n - 2) * g.F + mo],
                              l3 = Sf[(long long)(n - 3) * g.F + mo];
                if (L.bc_kind[f][1] == 0) {
                    qp.x = (-15.0 * l1.x + 5.0 * l2.x - l3.x) / 5.0;
                    qp.y = (-15.0 * l1.y + 5.0 * l2.y - l3.y) / 5.0;
                    if (mean_mode) qp.x += 16.0 * L.bc_val[f][1] / 5.0;
                } else {
                    qp.x = (21.0 * l1.x + 3.0 * l2.x - l3.x) / 23.0;
                    qp.y = (21.0 * l1.y + 3.0 * l2.y - l3.y) / 23.0;
                    if (mean_mode) qp.x -= 24.0 * (-L.bc_diff[f][1]) / 23.0;
                }
            } else {
                qp = Sf[(long long)(z + 1) * g.F + mo];
            }
        } else {
            A = L.alpha_c[z];
            B = L.alpha_i[z];
            Cc = L.alpha_c[z + 1];
            // Dirichlet values enter every mode (src/boundary_conditions.jl:263-273)
            qm = (z == 0) ? make_double2(L.bc_val[2][0], 0.0) : Sf[(long long)(z - 1) * g.F + mo];
            qp = (z == n - 1) ? make_double2(L.bc_val[2][1], 0.0) : Sf[(long long)(z + 1) * g.F + mo];
        }
        const double ab = A * B, bc = B * Cc;
        const double coef = ((L.DD1[k1] + L.DD2[j]) - ab) - bc;
        const double nu = L.nu[f];
        val.x = nu * ((ab * qm.x + coef * q0.x) + bc * qp.x);
        val.y = nu * ((ab * qm.y + coef * q0.y) + bc * qp.y);
    }
    if (L.src_on[f] && mean_mode) val.x += L.src[3 * m + f];
    return val;
}

// Forward y pass.  Contributions with prefactor 1 or D1 (which depends on k1
// only) are summed into NL "A" lines before the transform; the D2 contribution
// (at most one per field) goes to NL "B" lines transformed in the same batch, so
// the result is A + D2 * B without per-thread accumulators.
// Layers a rate at layer z needs for the Laplacian: a window of up to three
// consecutive layers starting at w0 (ghost extrapolation at the walls uses the
// three layers next to the wall).
__device__ __forceinline__ int lin_window_start(int z, int nz) { return max(0, min(z - 1, nz - 3)); }

// linear_terms computed from preloaded window values W[0..2] = S[w0..w0+2]
__device__ __forceinline__ double2 linear_terms_w(const Geo& g, const Linear& L, const double2 (&W)[3], int w0, int f,
                                                  int z, int j, int k1, int m) {
    double2 val = make_double2(0.0, 0.0);
    const bool mean_mode = (j == 0 && k1 == 0);
    if (L.diff_on[f]) {
        const int n = (f == 2) ? g.n3 - 1 : g.n3;
        auto at = [&](int zz) {  // selects keep the window in registers
            const int r = zz - w0;
            return r == 0 ? W[0] : (r == 1 ? W[1] : W[2]);
        };
        const double2 q0 = at(z);
        double2 qm, qp;
        double A, B, Cc;
        if (f != 2) {
            A = L.alpha_ext[z];
            B = L.alpha_c[z];
            Cc = L.alpha_ext[z + 1];
            if (z == 0) {
                const double2 l1 = at(0), l2 = at(1), l3 = at(2);
                if (L.bc_kind[f][0] == 0) {
                    qm.x = (-15.0 * l1.x + 5.0 * l2.x - l3.x) / 5.0;
                    qm.y = (-15.0 * l1.y + 5.0 * l2.y - l3.y) / 5.0;
                    if (mean_mode) qm.x += 16.0 * L.bc_val[f][0] / 5.0;
                } else {
                    qm.x = (21.0 * l1.x + 3.0 * l2.x - l3.x) / 23.0;
                    qm.y = (21.0 * l1.y + 3.0 * l2.y - l3.y) / 23.0;
                    if (mean_mode) qm.x -= 24.0 * L.bc_diff[f][0] / 23.0;
                }
            } else {
                qm = at(z - 1);
            }
            if (z == n - 1) {
                const double2 l1 = at(n - 1), l2 = at(n - 2), l3 = at(n - 3);
                if (L.bc_kind[f][1] == 0) {
                    qp.x = (-15.0 * l1.x + 5.0 * l2.x - l3.x) / 5.0;
                    qp.y = (-15.0 * l1.y + 5.0 * l2.y - l3.y) / 5.0;
                    if (mean_mode) qp.x += 16.0 * L.bc_val[f][1] / 5.0;
                } else {
                    qp.x = (21.0 * l1.x + 3.0 * l2.x - l3.x) / 23.0;
                    qp.y = (21.0 * l1.y + 3.0 * l2.y - l3.y) / 23.0;
                    if (mean_mode) qp.x -= 24.0 * (-L.bc_diff[f][1]) / 23.0;
                }
            } else {
                qp = at(z + 1);
            }
        } else {
            A = L.alpha_c[z];
            B = L.alpha_i[z];
            Cc = L.alpha_c[z + 1];
            qm = (z == 0) ? make_double2(L.bc_val[2][0], 0.0) : at(z - 1);
            qp = (z == n - 1) ? make_double2(L.bc_val[2][1], 0.0) : at(z + 1);
        }
        const double ab = A * B, bc = B * Cc;
        const double coef = ((L.DD1[k1] + L.DD2[j]) - ab) - bc;
        const double nu = L.nu[f];
        val.x = nu * ((ab * qm.x + coef * q0.x) + bc * qp.x);
        val.y = nu * ((ab * qm.y + coef * q0.y) + bc * qp.y);
    }
    if (L.src_on[f] && mean_mode) val.x += L.src[3 * m + f];
    return val;
}

// Epilogue of the forward y pass: the transformed lines `res` (position p of
// line l at res[swz(p) * LS + l]; B lines at l + NL) give the truncated, scaled
// rate of field f at layer z, summed with the linear terms, written as the rate
// or as the fused stage value (see FwdYArgs), with the non-finite check.
template <typename R, int RAD, int OB = 4>
__device__ __forceinline__ void fwd_y_epilogue(const FwdYArgs& a, const cplx<R>* __restrict__ res, int LS, int m,
                                               int f, int z, int nz, int k10, int NL, int nls, bool hasB) {
    using C = cplx<R>;
    const Geo& g = a.g;
    const int K1 = g.K1, K2 = g.K2, k2max = g.k2max, P2 = a.P2;
    double2* du = a.du + (long long)m * a.du_mstride + fld_off(g, f) + (long long)z * g.F;
    const double2* Sf = a.state ? a.state + (long long)m * g.mstride + fld_off(g, f) : nullptr;
    const bool need_win = (a.mode == 1) && a.lin.diff_on[f];
    const int w0 = lin_window_start(z, nz);
    const int wn = min(3, nz);
    bool bad = false;
    // OB: outputs per thread whose loads are issued together
    const int nout = K2 * NL;
    // the epilogue with the mode and the window loads fixed at compile time, so
    // that the loads of OB outputs are straight-line code
    double2* so = a.fuse ? a.sout + (long long)m * a.du_mstride + fld_off(g, f) + (long long)z * g.F : nullptr;
    const double2* su = (a.fuse && a.su) ? a.su + (long long)m * a.du_mstride + fld_off(g, f) + (long long)z * g.F : nullptr;
    auto epilogue = [&](auto mode_c, auto win_c, auto fuse_c) {
        constexpr int MODE = decltype(mode_c)::value;
        constexpr bool WIN = decltype(win_c)::value;
        // 0: the rate; 1: (cu su + ct state + cd rate) / div; 2: state + cd rate
        constexpr int FZ = decltype(fuse_c)::value;
        constexpr bool FUSE = FZ != 0;
        for (int o0 = 0; o0 < nout; o0 += OB * blockDim.x) {
            double2 W[OB][3];
            double2 old[OB], U[OB], T[OB];
#pragma unroll
            for (int q = 0; q < OB; ++q) {
                const int o = o0 + q * blockDim.x + threadIdx.x;
                const int j = o >> nls, l = o & (NL - 1), k1 = k10 + l;
                if (o < nout && k1 < K1) {
                    const long long idx = (long long)j * K1 + k1;
                    if constexpr (WIN) {
#pragma unroll
                        for (int r = 0; r < 3; ++r)
                            if (r < wn) W[q][r] = Sf[(long long)(w0 + r) * g.F + idx];
                    }
                    if constexpr (MODE == 0) old[q] = du[idx];
                    if constexpr (FZ == 1) U[q] = su[idx];
                    if constexpr (FUSE && !WIN) T[q] = Sf[(long long)z * g.F + idx];
                }
            }
#pragma unroll
            for (int q = 0; q < OB; ++q) {
                const int o = o0 + q * blockDim.x + threadIdx.x;
                const int j = o >> nls, l = o & (NL - 1), k1 = k10 + l;
                if (o >= nout || k1 >= K1) continue;
                const int pos = swz<C, RAD>((j <= k2max) ? j : P2 - (K2 - j));
                const C X = res[pos * LS + l];
                double vx = (double)X.x * a.inv_n, vy = (double)X.y * a.inv_n;
                if (hasB) {
                    const C Y = res[pos * LS + NL + l];
                    const double d = a.d2[j];
                    const double bx = (double)Y.x * a.inv_n, by = (double)Y.y * a.inv_n;
                    vx += -d * by;
                    vy += d * bx;
                }
                const long long idx = (long long)j * K1 + k1;
                double2 v;
                if constexpr (MODE == 1) {
                    double2 lin;
                    if constexpr (WIN)
                        lin = linear_terms_w(g, a.lin, W[q], w0, f, z, j, k1, m);
                    else
                        lin = linear_terms(g, a.lin, nullptr, f, z, j, k1, m);
                    v = make_double2(lin.x + vx, lin.y + vy);
                } else if constexpr (MODE == 2) {
                    v = make_double2(vx, vy);
                } else {
                    v = make_double2(old[q].x + vx, old[q].y + vy);
                }
                if constexpr (FUSE) {
                    double2 tz;
                    if constexpr (WIN) {
                        const int r = z - w0;   // the window holds layer z
                        tz = r == 0 ? W[q][0] : (r == 1 ? W[q][1] : W[q][2]);
                    } else {
                        tz = T[q];
                    }
                    if constexpr (FZ == 1) {
                        const double2 uz = U[q];
                        so[idx] = make_double2((a.st_cu * uz.x + a.st_ct * tz.x + a.st_cd * v.x) * a.st_inv,
                                               (a.st_cu * uz.y + a.st_ct * tz.y + a.st_cd * v.y) * a.st_inv);
                    } else {   // Euler stage: state + dt rate (src/ODEMethods.jl:101)
                        so[idx] = make_double2(tz.x + a.st_cd * v.x, tz.y + a.st_cd * v.y);
                    }
                } else {
                    du[idx] = v;
                }
                if (!(isfinite(v.x) && isfinite(v.y))) bad = true;
            }
        }
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    using BT = std::integral_constant<bool, true>;
    using BF = std::integral_constant<bool, false>;
    const int fz = a.fuse ? (a.su ? 1 : 2) : 0;
    if (fz == 1 && a.mode == 1 && need_win)
        epilogue(I1{}, BT{}, I1{});
    else if (fz == 1 && a.mode == 1)
        epilogue(I1{}, BF{}, I1{});
    else if (fz == 1 && a.mode == 0)
        epilogue(I0{}, BF{}, I1{});
    else if (fz == 2 && a.mode == 1 && need_win)
        epilogue(I1{}, BT{}, I2{});
    else if (fz == 2 && a.mode == 1)
        epilogue(I1{}, BF{}, I2{});
    else if (fz == 2 && a.mode == 0)
        epilogue(I0{}, BF{}, I2{});
    else if (a.mode == 1 && need_win)
        epilogue(I1{}, BT{}, I0{});
    else if (a.mode == 1)
        epilogue(I1{}, BF{}, I0{});
    else if (a.mode == 0)
        epilogue(I0{}, BF{}, I0{});
    else
        epilogue(I2{}, BF{}, I0{});
    if (a.check && bad) atomicOr(a.flag + m, 1);
}

// grid (fields*members, ceil(K1/NL), n3); smem tw[P2] + 2*P2*nlines complex (nlines = NL or 2NL)
// RAD > 0: one line per warp in registers on a padded line stride (see k_inv_y)
template <typename R, int RAD>
__global__ void __launch_bounds__(256) k_fwd_y(FwdYArgs a) {
    using C = cplx<R>;
    const int NL = a.NL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int fi = blockIdx.x % a.fields, m = a.m0 + blockIdx.x / a.fields;
    BLD_SKIP_INACTIVE(a, m);
    const int f = a.field0 + fi;
    const int z = blockIdx.z;
    const Geo& g = a.g;
    const int nz = (f == 2) ? g.n3 - 1 : g.n3;
    if (z >= nz) return;
    const int K1 = g.K1, K2 = g.K2, k2max = g.k2max, P2 = a.P2;
    const int k10 = blockIdx.y * NL;
    const int nc = a.ncontrib[fi];
    bool hasB = false;
    for (int ci = 0; ci < nc; ++ci) hasB |= (a.c[fi][ci].pref == 2);
    const int nlines = hasB ? 2 * NL : NL;
    const int LS = RAD ? nlines + 1 : nlines;                 // stride of a position in the line buffer
    const int nls = __ffs(NL) - 1, nlsl = __ffs(nlines) - 1;   // NL and nlines are powers of two
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* b0 = tw + P2;
    C* b1 = b0 + P2 * nlines;
    const C* twg = reinterpret_cast<const C*>(a.tw);
    lane_table<RAD>(tw, twg, P2);
    const C* base = reinterpret_cast<const C*>(a.mout) + (long long)m * a.mout_mstride;
    const long long layer = (long long)P2 * K1;
    // line l < NL: A set (k1 = k10 + l); NL <= l < 2NL: B set; loads batched 4 per thread
    constexpr int BATCH = 4;
    const int nval = P2 * nlines;
    if (nc == 1 && a.c[fi][0].pref == 0) {
        // a single contribution without prefactor (the advection rates): a plain
        // strided copy, whose loads issue together
        const C* src = base + (long long)(a.c[fi][0].term * g.n3 + z) * layer + k10;
        constexpr int B2 = 8;
        for (int i0 = 0; i0 < nval; i0 += B2 * blockDim.x) {
            C v[B2];
#pragma unroll
            for (int q = 0; q < B2; ++q) {
                const int i = i0 + q * blockDim.x + threadIdx.x;
                v[q] = mk<R>(0, 0);
                const int y = i >> nlsl, l = i & (nlines - 1);
                if (i < nval && k10 + l < K1) v[q] = src[(long long)y * K1 + l];
            }
#pragma unroll
            for (int q = 0; q < B2; ++q) {
                const int i = i0 + q * blockDim.x + threadIdx.x;
                if (i < nval) {
                    const int y = i >> nlsl, l = i & (nlines - 1);
                    b0[swz<C, RAD>(y) * LS + l] = v[q];
                }
            }
        }
    } else if (nc == 3 && hasB && a.c[fi][0].pref == 0 && a.c[fi][1].pref == 1 && a.c[fi][2].pref == 2) {
        // the SGS pattern: A lines = T0 + D1 T1, B lines = T2; loads predicated, not branched
        const C* s0 = base + (long long)(a.c[fi][0].term * g.n3 + z) * layer;
        const C* s1 = base + (long long)(a.c[fi][1].term * g.n3 + z) * layer;
        const C* s2 = base + (long long)(a.c[fi][2].term * g.n3 + z) * layer;
        for (int i0 = 0; i0 < nval; i0 += BATCH * blockDim.x) {
            C v[BATCH];
#pragma unroll
            for (int q = 0; q < BATCH; ++q) {
                const int i = i0 + q * blockDim.x + threadIdx.x;
                const int y = i >> nlsl, l = i & (nlines - 1);
                const bool isB = l >= NL;
                const int k1 = k10 + (isB ? l - NL : l);
                const bool ok = i < nval && k1 < K1;
                const long long off = (long long)y * K1 + k1;
                C x0 = mk<R>(0, 0), x1 = mk<R>(0, 0), x2 = mk<R>(0, 0);
                if (ok && !isB) {
                    x0 = s0[off];
                    x1 = s1[off];
                }
                if (ok && isB) x2 = s2[off];
                const R d = ok ? (R)a.d1[k1] : R(0);
                // D1 = i d1[k1] applied to T1, added after T0 (the order of the generic path)
                v[q] = isB ? x2 : mk<R>(x0.x + (-d * x1.y), x0.y + d * x1.x);
            }
#pragma unroll
            for (int q = 0; q < BATCH; ++q) {
                const int i = i0 + q * blockDim.x + threadIdx.x;
                if (i < nval) {
                    const int y = i >> nlsl, l = i & (nlines - 1);
                    b0[swz<C, RAD>(y) * LS + l] = v[q];
                }
            }
        }
    } else
    for (int i0 = 0; i0 < nval; i0 += BATCH * blockDim.x) {
        C v[BATCH];
#pragma unroll
        for (int q = 0; q < BATCH; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            v[q] = mk<R>(0, 0);
            if (i < nval) {
                const int y = i >> nlsl, l = i & (nlines - 1);
                const bool isB = l >= NL;
                const int k1 = k10 + (isB ? l - NL : l);
                if (k1 < K1) {
                    for (int ci = 0; ci < nc; ++ci) {
                        const FwdContrib cb = a.c[fi][ci];
                        if ((cb.pref == 2) != isB) continue;
                        C x = base[(long long)(cb.term * g.n3 + z) * layer + (long long)y * K1 + k1];
                        if (cb.pref == 1) {  // D1 = i d1[k1]
                            const R d = (R)a.d1[k1];
                            const R tx = -d * x.y;
                            x.y = d * x.x;
                            x.x = tx;
                        }
                        v[q].x += x.x;
                        v[q].y += x.y;
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < BATCH; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            if (i < nval) {
                const int y = i >> nlsl, l = i & (nlines - 1);
                b0[swz<C, RAD>(y) * LS + l] = v[q];
            }
        }
    }
    __syncthreads();
    const C* res = b0;
    if constexpr (RAD > 0) {
        const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        const int brl = (int)(__brev((unsigned)lane) >> 27);
        LaneTw<R> lt;
        lane_twiddles_tab<R>(lt, lane, twg, P2);
        for (int l = threadIdx.x >> 5; l < nlines; l += nw) {
            C zl[RAD];
#pragma unroll
            for (int k = 0; k < RAD; ++k) zl[k] = b0[swz<C, RAD>(k + RAD * brl) * LS + l];
            forward_line<R, RAD>(zl, lane, tw + lane, 32, lt);
#pragma unroll
            for (int b = 0; b < RAD; ++b) b0[swz<C, RAD>(lane + 32 * b) * LS + l] = zl[b];
        }
        __syncthreads();
    } else {
        res = fft_big<R, -1>(b0, b1, nlines, 1, nlines, false, a.plan, tw);
    }
    fwd_y_epilogue<R, RAD>(a, res, LS, m, f, z, nz, k10, NL, nls, hasB);
}

// Forward y pass of all three rate fields at one layer: one block per (k1 tile,
// layer, member).  Per field, contributions with prefactor 1 or D1 are summed
// into an A line set and the D2 contribution into a B line set before one
// in-place transform of all 3*sets*NL lines; the epilogue adds the linear terms.
// grid (ceil(K1/NL), n3, members); smem tw[P2] + P2*NLT complex.
template <typename R>
__global__ void __launch_bounds__(384) k_fwd_y_all(FwdYArgs a) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NL = a.NL;
    const Geo& g = a.g;
    const int K1 = g.K1, K2 = g.K2, k2max = g.k2max, P2 = a.P2, n3 = g.n3;
    const int k10 = blockIdx.x * NL;
    const int z = blockIdx.y;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    bool hasB = false;
    for (int f = 0; f < 3; ++f)
        for (int ci = 0; ci < a.ncontrib[f]; ++ci) hasB |= (a.c[f][ci].pref == 2);
    const int sets = hasB ? 2 : 1;
    const int NLF = sets * NL;       // lines per field
    const int NLT = 3 * NLF;         // line index L = f*NLF + set*NL + l
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + P2;
    copy_table(tw, reinterpret_cast<const C*>(a.tw), P2);
    const C* base = reinterpret_cast<const C*>(a.mout) + (long long)m * a.mout_mstride;
    const long long layer = (long long)P2 * K1;
    const int nval = P2 * NLT;
    constexpr int B = 4;
    for (int i0 = 0; i0 < nval; i0 += B * blockDim.x) {
        C v[B];
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            v[q] = mk<R>(0, 0);
            if (i < nval) {
                const int y = i / NLT, L = i - y * NLT;
                const int f = L / NLF, r = L - f * NLF;
                const bool isB = r >= NL;
                const int k1 = k10 + (isB ? r - NL : r);
                const int nz = (f == 2) ? n3 - 1 : n3;
                if (k1 < K1 && z < nz) {
                    for (int ci = 0; ci < a.ncontrib[f]; ++ci) {
                        const FwdContrib cb = a.c[f][ci];
                        if ((cb.pref == 2) != isB) continue;
                        C x = base[(long long)(cb.term * n3 + z) * layer + (long long)y * K1 + k1];
                        if (cb.pref == 1) {
                            const R d = (R)a.d1[k1];
                            const R tx = -d * x.y;
                            x.y = d * x.x;
                            x.x = tx;
                        }
                        v[q].x += x.x;
                        v[q].y += x.y;
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int i = i0 + q * blockDim.x + threadIdx.x;
            if (i < nval) buf[i] = v[q];
        }
    }
    __syncthreads();
    fft_inplace<R, -1>(buf, NLT, 1, NLT, false, a.plan, tw);
    // epilogue: outputs (f, j, l), state windows and old rates loaded OB at a time
    const double2* S = a.state ? a.state + (long long)m * g.mstride : nullptr;
    double2* dum = a.du + (long long)m * a.du_mstride;
    bool bad = false;
    const int nout = 3 * K2 * NL;
    constexpr int OB = 2;
    for (int o0 = 0; o0 < nout; o0 += OB * blockDim.x) {
        double2 W[OB][3];
        double2 old[OB];
#pragma unroll
        for (int q = 0; q < OB; ++q) {
            const int o = o0 + q * blockDim.x + threadIdx.x;
            const int f = o / (K2 * NL), r = o - f * (K2 * NL);
            const int j = r / NL, l = r - j * NL, k1 = k10 + l;
            const int nz = (f == 2) ? n3 - 1 : n3;
            if (o < nout && k1 < K1 && z < nz) {
                const long long idx = (long long)j * K1 + k1;
                if (a.mode == 1 && a.lin.diff_on[f]) {
                    const int w0 = lin_window_start(z, nz), wn = min(3, nz);
                    const double2* Sf = S + fld_off(g, f);
#pragma unroll
                    for (int rr = 0; rr < 3; ++rr)
                        if (rr < wn) W[q][rr] = Sf[(long long)(w0 + rr) * g.F + idx];
                }
                if (a.mode == 0) old[q] = dum[fld_off(g, f) + (long long)z * g.F + idx];
            }
        }
#pragma unroll
        for (int q = 0; q < OB; ++q) {
            const int o = o0 + q * blockDim.x + threadIdx.x;
            const int f = o / (K2 * NL), r = o - f * (K2 * NL);
            const int j = r / NL, l = r - j * NL, k1 = k10 + l;
            const int nz = (f == 2) ? n3 - 1 : n3;
            if (o >= nout || k1 >= K1 || z >= nz) continue;
            const int pos = (j <= k2max) ? j : P2 - (K2 - j);
            const C X = buf[pos * NLT + f * NLF + l];
            double vx = (double)X.x * a.inv_n, vy = (double)X.y * a.inv_n;
            if (hasB) {
                const C Y = buf[pos * NLT + f * NLF + NL + l];
                const double d = a.d2[j];
                const double bx = (double)Y.x * a.inv_n, by = (double)Y.y * a.inv_n;
                vx += -d * by;
                vy += d * bx;
            }
            const long long idx = (long long)j * K1 + k1;
            double2 v;
            if (a.mode == 1) {
                double2 lin;
                if (a.lin.diff_on[f])
                    lin = linear_terms_w(g, a.lin, W[q], lin_window_start(z, nz), f, z, j, k1, m);
                else
                    lin = linear_terms(g, a.lin, nullptr, f, z, j, k1, m);
                v = make_double2(lin.x + vx, lin.y + vy);
            } else if (a.mode == 2) {
                v = make_double2(vx, vy);
            } else {
                v = make_double2(old[q].x + vx, old[q].y + vy);
            }
            dum[fld_off(g, f) + (long long)z * g.F + idx] = v;
            if (!(isfinite(v.x) && isfinite(v.y))) bad = true;
        }
    }
    if (a.check && bad) atomicOr(a.flag + m, 1);
}

// Linear terms only (no physical-domain process): grid (ceil(F/256), n3, 3*members)
__global__ void __launch_bounds__(256) k_linear(FwdYArgs a) {
    const Geo& g = a.g;
    const int f = blockIdx.z % 3, m = a.m0 + blockIdx.z / 3;
    BLD_SKIP_INACTIVE(a, m);
    const int z = blockIdx.y;
    const int nz = (f == 2) ? g.n3 - 1 : g.n3;
    const int mo = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nz || mo >= g.F) return;
    const int j = mo / g.K1, k1 = mo - j * g.K1;
    const double2* S = a.state + (long long)m * g.mstride;
    const double2 v = linear_terms(g, a.lin, S, f, z, j, k1, m);
    a.du[(long long)m * a.du_mstride + fld_off(g, f) + (long long)z * g.F + mo] = v;
    if (a.check && !(isfinite(v.x) && isfinite(v.y))) atomicOr(a.flag + m, 1);
}

// --------------------------------------------------- stage update + projection
enum StageKind {
    S_NONE = 0,     // out = u (projection only)
    S_EULER = 1,    // u + dt du                       (src/ODEMethods.jl:101,137,150)
    S_RK22_2 = 2,   // (u + t + dt du) / 2             (:143)
    S_RK33_2 = 3,   // (3u + t + dt du) / 4            (:157)
    S_RK33_3 = 4,   // (u + 2t + 2 dt du) / 3          (:164)
    S_AB2_1 = 5,    // u + dt (du - dp) / 2            (:120)
    S_AB2 = 6       // u + dt/2 (3 du - dp)            (:127)
};

struct ProjArgs {
    Geo g;
    int m0;
    const int* active;
    const double2* u;
    const double2* t;
    const double2* du;
    const double2* dp;
    double2* out;
    int kind;
    double dt;
    int pressure;
    double2* pscr;           // [members][n3][F] forward-sweep scratch
    const double* gamma;     // [n3][F]
    const double* alpha_c;   // [n3]
    const double* alpha_i;   // [n3-1]  (off-diagonal beta)
    const double* inv_alpha_c;   // [n3] 1 / alpha_c, rounded as the division (segmented and tile kernels)
    const double* d1;
    const double* d2;
    double w_lo, w_hi;
    int mean_on[3];
    const double* mean_w;    // [n3] weights (dx3/dzeta)/(n3 L3)
    const double* mean_val;  // [members][3]
};

__device__ __forceinline__ double2 stage_value(const ProjArgs& a, long long idx) {
    const double2 u = a.u[idx];
    const double dt = a.dt;
    switch (a.kind) {
        case S_NONE:
            return u;
        case S_EULER: {
            const double2 d = a.du[idx];
            return make_double2(u.x + dt * d.x, u.y + dt * d.y);
        }
        case S_RK22_2: {
            const double2 t = a.t[idx], d = a.du[idx];
            return make_double2((u.x + t.x + dt * d.x) / 2.0, (u.y + t.y + dt * d.y) / 2.0);
        }
        case S_RK33_2: {
            const double2 t = a.t[idx], d = a.du[idx];
            return make_double2((3.0 * u.x + t.x + dt * d.x) / 4.0, (3.0 * u.y + t.y + dt * d.y) / 4.0);
        }
        case S_RK33_3: {
            const double2 t = a.t[idx], d = a.du[idx];
            const double dt2 = 2.0 * dt;
            return make_double2((u.x + 2.0 * t.x + dt2 * d.x) / 3.0, (u.y + 2.0 * t.y + dt2 * d.y) / 3.0);
        }
        case S_AB2_1: {
            const double2 d = a.du[idx], p = a.dp[idx];
            return make_double2(u.x + dt * (d.x - p.x) / 2.0, u.y + dt * (d.y - p.y) / 2.0);
        }
        default: {  // S_AB2
            const double2 d = a.du[idx], p = a.dp[idx];
            const double h = dt / 2.0;
            return make_double2(u.x + h * (3.0 * d.x - p.x), u.y + h * (3.0 * d.y - p.y));
        }
    }
}

// the same with the stage kind fixed at compile time: the loads of a layer batch
// are straight-line code that the compiler issues together
template <int KIND>
__device__ __forceinline__ double2 stage_value_k(const ProjArgs& a, long long idx) {
    const double2 u = a.u[idx];
    const double dt = a.dt;
    if constexpr (KIND == S_NONE) {
        return u;
    } else if constexpr (KIND == S_EULER) {
        const double2 d = a.du[idx];
        return make_double2(u.x + dt * d.x, u.y + dt * d.y);
    } else if constexpr (KIND == S_RK22_2) {
        const double2 t = a.t[idx], d = a.du[idx];
        return make_double2((u.x + t.x + dt * d.x) / 2.0, (u.y + t.y + dt * d.y) / 2.0);
    } else if constexpr (KIND == S_RK33_2) {
        const double2 t = a.t[idx], d = a.du[idx];
        return make_double2((3.0 * u.x + t.x + dt * d.x) / 4.0, (3.0 * u.y + t.y + dt * d.y) / 4.0);
    } else if constexpr (KIND == S_RK33_3) {
        const double2 t = a.t[idx], d = a.du[idx];
        const double dt2 = 2.0 * dt;
        return make_double2((u.x + 2.0 * t.x + dt2 * d.x) / 3.0, (u.y + 2.0 * t.y + dt2 * d.y) / 3.0);
    } else if constexpr (KIND == S_AB2_1) {
        const double2 d = a.du[idx], p = a.dp[idx];
        return make_double2(u.x + dt * (d.x - p.x) / 2.0, u.y + dt * (d.y - p.y) / 2.0);
    } else {  // S_AB2
        const double2 d = a.du[idx], p = a.dp[idx];
        const double h = dt / 2.0;
        return make_double2(u.x + h * (3.0 * d.x - p.x), u.y + h * (3.0 * d.y - p.y));
    }
}

// One thread per (k1, k2) column: stage update, divergence (div!, src/processes/pressure.jl:368-378),
// forward/backward Thomas (:106-165), gradient (add_gradient!, :405-426), then ConstantMean
// (src/processes/sources.jl:71-77) on the (0,0) column.  grid (ceil(F/128), members)
__global__ void __launch_bounds__(128) k_project(ProjArgs a) {
    const Geo& g = a.g;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = a.m0 + blockIdx.y;
    BLD_SKIP_INACTIVE(a, m);
    if (c >= g.F) return;
    const long long mb = (long long)m * g.mstride;
    const long long F = g.F;
    const int n = g.n3;
    const long long o1 = mb, o2 = mb + (long long)n * F, o3 = mb + 2LL * n * F;
    if (a.pressure) {
        const int j = c / g.K1, k1 = c - j * g.K1;
        const bool mean_mode = (c == 0);
        const double e1 = a.d1[k1], e2 = a.d2[j];
        double2* P = a.pscr + (long long)m * n * F + c;
        double2 wprev = make_double2(0.0, 0.0);
        double2 b = make_double2(0.0, 0.0);
        constexpr int NB = 4;  // layers whose loads are issued together
        for (int zb = 0; zb < n; zb += NB) {
            double2 U[NB], V[NB], W[NB];
            double G[NB];
#pragma unroll
            for (int q = 0; q < NB; ++q) {
                const int z = zb + q;
                if (z < n) {
                    U[q] = stage_value(a, o1 + z * F + c);
                    V[q] = stage_value(a, o2 + z * F + c);
                    W[q] = (z < n - 1) ? stage_value(a, o3 + z * F + c) : make_double2(0.0, 0.0);
                    G[q] = a.gamma[(long long)z * F + c];
                }
            }
#pragma unroll
            for (int q = 0; q < NB; ++q) {
                const int z = zb + q;
                if (z >= n) break;
                const double2 uz = U[q], vz = V[q], wz = W[q];
                a.out[o1 + z * F + c] = uz;
                a.out[o2 + z * F + c] = vz;
                if (z < n - 1) a.out[o3 + z * F + c] = wz;
                const double h = 1.0 / a.alpha_c[z];
                double2 val;
                val.x = (-e1 * uz.y) * h + (-e2 * vz.y) * h;
                val.y = (e1 * uz.x) * h + (e2 * vz.x) * h;
                if (z == 0) {
                    val.x += wz.x;
                    val.y += wz.y;
                    if (mean_mode) val.x -= a.w_lo;
                } else if (z == n - 1) {
                    val.x -= wprev.x;
                    val.y -= wprev.y;
                    if (mean_mode) val.x += a.w_hi;
                } else {
                    val.x = val.x - wprev.x + wz.x;
                    val.y = val.y - wprev.y + wz.y;
                }
                if (mean_mode && z == n - 1) val = make_double2(0.0, 0.0);  // adjust_pressure_rhs! (:396)
                const double gm = G[q];
                if (z == 0) {
                    b = make_double2(gm * val.x, gm * val.y);
                } else {
                    const double be = a.alpha_i[z - 1];
                    b = make_double2(gm * (val.x - be * b.x), gm * (val.y - be * b.y));
                }
                P[(long long)z * F] = b;
                wprev = wz;
            }
        }
        // backward sweep and gradient, top to bottom
        double2 pn = b;  // p at z = n-1
        {
            const int z = n - 1;
            double2 u = a.out[o1 + z * F + c], v = a.out[o2 + z * F + c];
            u.x += e1 * pn.y; u.y += -e1 * pn.x;
            v.x += e2 * pn.y; v.y += -e2 * pn.x;
            a.out[o1 + z * F + c] = u;
            a.out[o2 + z * F + c] = v;
        }
        for (int zt = n - 2; zt >= 0; zt -= NB) {
            double2 Bz[NB], U[NB], V[NB], W[NB];
            double G[NB];
#pragma unroll
            for (int q = 0; q < NB; ++q) {
                const int z = zt - q;
                if (z >= 0) {
                    Bz[q] = P[(long long)z * F];
                    G[q] = a.gamma[(long long)z * F + c];
                    U[q] = a.out[o1 + z * F + c];
                    V[q] = a.out[o2 + z * F + c];
                    W[q] = a.out[o3 + z * F + c];
                }
            }
#pragma unroll
            for (int q = 0; q < NB; ++q) {
                const int z = zt - q;
                if (z < 0) break;
                const double ai = a.alpha_i[z];
                const double gb = G[q] * ai;
                const double2 pz = make_double2(Bz[q].x - gb * pn.x, Bz[q].y - gb * pn.y);
                double2 u = U[q], v = V[q], w = W[q];
                u.x += e1 * pz.y; u.y += -e1 * pz.x;
                v.x += e2 * pz.y; v.y += -e2 * pz.x;
                w.x += -1.0 * (-ai * pz.x + ai * pn.x);
                w.y += -1.0 * (-ai * pz.y + ai * pn.y);
                a.out[o1 + z * F + c] = u;
                a.out[o2 + z * F + c] = v;
                a.out[o3 + z * F + c] = w;
                pn = pz;
            }
        }
    } else if (a.kind != S_NONE || a.out != a.u) {
        for (int z = 0; z < n; ++z) {
            a.out[o1 + z * F + c] = stage_value(a, o1 + z * F + c);
            a.out[o2 + z * F + c] = stage_value(a, o2 + z * F + c);
            if (z < n - 1) a.out[o3 + z * F + c] = stage_value(a, o3 + z * F + c);
        }
    }
    if (c == 0) {
        for (int f = 0; f < 2; ++f) {
            if (!a.mean_on[f]) continue;
            const long long of = (f == 0) ? o1 : o2;
            double s = 0.0;
            for (int z = 0; z < n; ++z) s += a.out[of + z * F].x * a.mean_w[z];
            const double add = a.mean_val[3 * m + f] - s;
            for (int z = 0; z < n; ++z) a.out[of + z * F].x += add;
        }
    }
}

// Segmented projection: block (32 columns, NS z segments of <= LMAX layers),
// grid (ceil(F/32), members).  The Thomas sweeps are first-order linear
// recurrences, so each segment solves its part as an affine function of the
// value entering from below (forward: b_z = P_z + Q_z b_in) or from above
// (backward: p_z = G_z + H_z p_out) and the segments are chained through shared
// memory.  Same arithmetic as k_project up to the order of operations.
// Body of k_project_seg for one stage kind.  TILE: the stage values of the
// block's columns stay in shared memory between the phases ([3][n3][lanes],
// dynamic) instead of a round trip through `out`.
template <int LMAX, bool TILE, int KIND>
__device__ __forceinline__ void project_seg_body(const ProjArgs& a, double2* tile, double2 (&sP)[32][32],
                                                 double (&sQ)[32][32]) {
    const Geo& g = a.g;
    const int n = g.n3;
    const long long F = g.F;
    const int NS = blockDim.y, s = threadIdx.y, lane = threadIdx.x;
    const int c = blockIdx.x * blockDim.x + lane;
    const int m = a.m0 + blockIdx.y;
    BLD_SKIP_INACTIVE(a, m);
    const bool valid = c < g.F;
    const int L = (n + NS - 1) / NS;
    const int z0 = min(n, s * L), z1 = min(n, z0 + L);
    const int len = z1 - z0;
    const long long mb = (long long)m * g.mstride;
    const long long o1 = mb, o2 = mb + (long long)n * F, o3 = mb + 2LL * n * F;
    const int cc = valid ? c : 0;
    const int j = cc / g.K1, k1 = cc - j * g.K1;
    const bool mean_mode = (c == 0);
    const double e1 = a.d1[k1], e2 = a.d2[j];
    // a plain projection in place: the stage values are the stored values, so
    // phase 1 need not write them out again (phase 3 reads them from u = out)
    const bool in_place = (KIND == S_NONE) && (a.out == a.u);
    // stage value of w just below the segment, read before any thread writes `out`
    double2 wprev = make_double2(0.0, 0.0);
    if (valid && z0 > 0 && len > 0) wprev = stage_value_k<KIND>(a, o3 + (long long)(z0 - 1) * F + c);
    __syncthreads();
    double2 X[LMAX];
    double Y[LMAX];
    // ---- phase 1: stage values, divergence, segment-local forward sweep
    // (loads of 4 layers issued together, then the dependent recurrence)
    constexpr int NBL = 4;
#pragma unroll
    for (int qb = 0; qb < LMAX; qb += NBL) {
        double2 Ub[NBL], Vb[NBL], Wb[NBL];
        double Gb[NBL];
#pragma unroll
        for (int r = 0; r < NBL; ++r) {
            const int q = qb + r, z = z0 + q;
            if (q < len && valid) {
                Ub[r] = stage_value_k<KIND>(a, o1 + z * F + c);
                Vb[r] = stage_value_k<KIND>(a, o2 + z * F + c);
                Wb[r] = (z < n - 1) ? stage_value_k<KIND>(a, o3 + z * F + c) : make_double2(0.0, 0.0);
                Gb[r] = a.gamma[z * F + c];
            }
        }
#pragma unroll
        for (int r = 0; r < NBL; ++r) {
            const int q = qb + r, z = z0 + q;
            if (q < len && valid) {
                const double2 uz = Ub[r], vz = Vb[r], wz = Wb[r];
                if constexpr (TILE) {
                    const int LN = blockDim.x;
                    tile[(0 * n + z) * LN + lane] = uz;
                    tile[(1 * n + z) * LN + lane] = vz;
                    if (z < n - 1) tile[(2 * n + z) * LN + lane] = wz;
                } else if (!in_place) {
                    a.out[o1 + z * F + c] = uz;
                    a.out[o2 + z * F + c] = vz;
                    if (z < n - 1) a.out[o3 + z * F + c] = wz;
                }
                const double h = a.inv_alpha_c[z];
                double2 val;
                val.x = (-e1 * uz.y) * h + (-e2 * vz.y) * h;
                val.y = (e1 * uz.x) * h + (e2 * vz.x) * h;
                if (z == 0) {
                    val.x += wz.x;
                    val.y += wz.y;
                    if (mean_mode) val.x -= a.w_lo;
                } else if (z == n - 1) {
                    val.x -= wprev.x;
                    val.y -= wprev.y;
                    if (mean_mode) val.x += a.w_hi;
                } else {
                    val.x = val.x - wprev.x + wz.x;
                    val.y = val.y - wprev.y + wz.y;
                }
                if (mean_mode && z == n - 1) val = make_double2(0.0, 0.0);
                const double gm = Gb[r];
                if (z == 0) {
                    X[q] = make_double2(gm * val.x, gm * val.y);
                    Y[q] = 0.0;
                } else if (q == 0) {
                    X[q] = make_double2(gm * val.x, gm * val.y);
                    Y[q] = -gm * a.alpha_i[z - 1];
                } else {
                    const double be = a.alpha_i[z - 1];
                    X[q] = make_double2(gm * (val.x - be * X[q - 1].x), gm * (val.y - be * X[q - 1].y));
                    Y[q] = -gm * be * Y[q - 1];
                }
                wprev = wz;
            }
        }
    }
    // segment summaries: an empty segment passes its input through unchanged
    {
        double2 pe = make_double2(0.0, 0.0);
        double qe = 1.0;
        if (len > 0 && valid) {
#pragma unroll
            for (int q = 0; q < LMAX; ++q)
                if (q < len) {   // the last valid layer wins; `q == len - 1` would become a dynamic index
                    pe = X[q];
                    qe = Y[q];
                }
        }
        sP[s][lane] = pe;
        sQ[s][lane] = qe;
    }
    __syncthreads();
    double2 bin = make_double2(0.0, 0.0);
    for (int t = 0; t < s; ++t) {
        const double2 pe = sP[t][lane];
        const double qe = sQ[t][lane];
        bin = make_double2(pe.x + qe * bin.x, pe.y + qe * bin.y);
    }
    __syncthreads();
    // ---- phase 2: b_z, then the segment-local backward sweep
#pragma unroll
    for (int q = 0; q < LMAX; ++q)
        if (q < len) X[q] = make_double2(X[q].x + Y[q] * bin.x, X[q].y + Y[q] * bin.y);
#pragma unroll
    for (int qq = 0; qq < LMAX; ++qq) {
        const int q = LMAX - 1 - qq;
        if (q >= len || !valid) continue;
        const int z = z0 + q;
        if (z == n - 1) {
            Y[q] = 0.0;  // p_{n-1} = b_{n-1}
        } else {
            const double cz = a.gamma[z * F + c] * a.alpha_i[z];
            // len <= LMAX, so q == LMAX-1 implies q == len-1; spelling it out keeps
            // X[q + 1] in range for the compiler and the arrays in registers
            if (q == len - 1 || q == LMAX - 1) {
                Y[q] = -cz;
            } else {
                X[q] = make_double2(X[q].x - cz * X[q + 1].x, X[q].y - cz * X[q + 1].y);
                Y[q] = -cz * Y[q + 1];
            }
        }
    }
    {
        double2 ps = make_double2(0.0, 0.0);
        double hs = 1.0;
        if (len > 0 && valid) {
            ps = X[0];
            hs = Y[0];
        }
        sP[s][lane] = ps;
        sQ[s][lane] = hs;
    }
    __syncthreads();
    double2 pout = make_double2(0.0, 0.0);
    for (int t = NS - 1; t > s; --t) {
        const double2 ps = sP[t][lane];
        const double hs = sQ[t][lane];
        pout = make_double2(ps.x + hs * pout.x, ps.y + hs * pout.y);
    }
    // ---- phase 3: pressure and gradient
#pragma unroll
    for (int q = 0; q < LMAX; ++q)
        if (q < len) X[q] = make_double2(X[q].x + Y[q] * pout.x, X[q].y + Y[q] * pout.y);
#pragma unroll
    for (int qb = 0; qb < LMAX; qb += NBL) {
        double2 Ub[NBL], Vb[NBL], Wb[NBL];
#pragma unroll
        for (int r = 0; r < NBL; ++r) {
            const int q = qb + r, z = z0 + q;
            if (q < len && valid) {
                if constexpr (TILE) {
                    const int LN = blockDim.x;
                    Ub[r] = tile[(0 * n + z) * LN + lane];
                    Vb[r] = tile[(1 * n + z) * LN + lane];
                    if (z < n - 1) Wb[r] = tile[(2 * n + z) * LN + lane];
                } else {
                    Ub[r] = a.out[o1 + z * F + c];
                    Vb[r] = a.out[o2 + z * F + c];
                    if (z < n - 1) Wb[r] = a.out[o3 + z * F + c];
                }
            }
        }
#pragma unroll
        for (int r = 0; r < NBL; ++r) {
            const int q = qb + r, z = z0 + q;
            if (q < len && valid) {
                const double2 pz = X[q];
                double2 pn = pout;
#pragma unroll
                for (int rr = 0; rr < LMAX; ++rr)
                    if (rr == q + 1 && rr < len) pn = X[rr];
                double2 u = Ub[r], v = Vb[r];
                u.x += e1 * pz.y;
                u.y += -e1 * pz.x;
                v.x += e2 * pz.y;
                v.y += -e2 * pz.x;
                a.out[o1 + z * F + c] = u;
                a.out[o2 + z * F + c] = v;
                if (z < n - 1) {
                    double2 w = Wb[r];
                    const double ai = a.alpha_i[z];
                    w.x += -1.0 * (-ai * pz.x + ai * pn.x);
                    w.y += -1.0 * (-ai * pz.y + ai * pn.y);
                    a.out[o3 + z * F + c] = w;
                }
            }
        }
    }
    // ConstantMean on the (0,0) column (src/processes/sources.jl:71-77)
    __syncthreads();
    if (c == 0 && s == 0) {
        for (int f = 0; f < 2; ++f) {
            if (!a.mean_on[f]) continue;
            const long long of = (f == 0) ? o1 : o2;
            double sum = 0.0;
            for (int z = 0; z < n; ++z) sum += a.out[of + z * F].x * a.mean_w[z];
            const double add = a.mean_val[3 * m + f] - sum;
            for (int z = 0; z < n; ++z) a.out[of + z * F].x += add;
        }
    }
}

template <int LMAX, int MINB, bool TILE>
__global__ void __launch_bounds__(256, MINB) k_project_seg(ProjArgs a) {
    extern __shared__ __align__(16) double2 tile[];
    __shared__ double2 sP[32][32];
    __shared__ double sQ[32][32];
    switch (a.kind) {
        case S_NONE: project_seg_body<LMAX, TILE, S_NONE>(a, tile, sP, sQ); break;
        case S_EULER: project_seg_body<LMAX, TILE, S_EULER>(a, tile, sP, sQ); break;
        case S_RK22_2: project_seg_body<LMAX, TILE, S_RK22_2>(a, tile, sP, sQ); break;
        case S_RK33_2: project_seg_body<LMAX, TILE, S_RK33_2>(a, tile, sP, sQ); break;
        case S_RK33_3: project_seg_body<LMAX, TILE, S_RK33_3>(a, tile, sP, sQ); break;
        case S_AB2_1: project_seg_body<LMAX, TILE, S_AB2_1>(a, tile, sP, sQ); break;
        default: project_seg_body<LMAX, TILE, S_AB2>(a, tile, sP, sQ); break;
    }
}

// ---------------------------------------- segmented batched tridiagonal solve
// L D L^T x = b per system (ldiv!(::DistributedBatchLDLt, b),
// src/processes/pressure.jl:106-201): forward b_z = g_z (b_z - beta_{z-1} b_{z-1}),
// backward x_z = b_z - g_z beta_z x_{z+1}.  Instead of one thread walking all n
// layers of a system twice (two reads of b and g), each thread holds LMAX
// consecutive layers of one system in registers and solves them as an affine
// function of the value entering its segment: forward b_z = X_z + Y_z b_in with
// Y_z = prod(-g beta); the segment ends (X, Y) are combined through shared
// memory, and the backward sweep is done the same way.  b and g are read once and
// x is written once: 40 bytes per complex unknown (24 real).
// block (LANES, NS): LANES systems side by side (coalesced rows), NS segments;
// grid ceil(nsys / LANES); dynamic smem (n-1) doubles + NS*LANES*(sizeof(T)+8).
__device__ __forceinline__ double v_scale(double a, double x) { return a * x; }
__device__ __forceinline__ double2 v_scale(double a, double2 x) { return make_double2(a * x.x, a * x.y); }
__device__ __forceinline__ double v_axpy(double a, double x, double y) { return y + a * x; }
__device__ __forceinline__ double2 v_axpy(double a, double2 x, double2 y) {
    return make_double2(y.x + a * x.x, y.y + a * x.y);
}
template <typename T>
__device__ __forceinline__ T v_zero();
template <>
__device__ __forceinline__ double v_zero<double>() { return 0.0; }
template <>
__device__ __forceinline__ double2 v_zero<double2>() { return make_double2(0.0, 0.0); }

template <typename T, int LMAX>
__global__ void __launch_bounds__(512) k_ldlt_seg(const double* __restrict__ gamma, const double* __restrict__ beta,
                                                  T* __restrict__ rhs, long long nsys, int n) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int LANES = blockDim.x, NS = blockDim.y, lane = threadIdx.x, s = threadIdx.y;
    double* sb = reinterpret_cast<double*>(smem_raw);                  // beta [n-1]
    T* sP = reinterpret_cast<T*>(sb + (n & ~1));                       // [NS][LANES] (n & ~1 >= n-1, even)
    double* sQ = reinterpret_cast<double*>(sP + NS * LANES);            // [NS][LANES]
    for (int i = s * LANES + lane; i < n - 1; i += NS * LANES) sb[i] = beta[i];
    const long long c = (long long)blockIdx.x * LANES + lane;
    const bool valid = c < nsys;
    const int L = (n + NS - 1) / NS;
    const int z0 = min(n, s * L), z1 = min(n, z0 + L);
    const int len = valid ? z1 - z0 : 0;
    T X[LMAX];
    double G[LMAX];
#pragma unroll
    for (int q = 0; q < LMAX; ++q)
        if (q < len) {
            X[q] = rhs[(long long)(z0 + q) * nsys + c];
            G[q] = gamma[(long long)(z0 + q) * nsys + c];
        }
    __syncthreads();
    // forward sweep, local input 0
    double y = 1.0;
#pragma unroll
    for (int q = 0; q < LMAX; ++q)
        if (q < len) {
            const int z = z0 + q;
            if (q == 0) {
                X[0] = v_scale(G[0], X[0]);
                y = (z == 0) ? 0.0 : -G[0] * sb[z - 1];
            } else {
                X[q] = v_scale(G[q], v_axpy(-sb[z - 1], X[q - 1], X[q]));
                y = -G[q] * sb[z - 1] * y;
            }
        }
    {
        T pe = v_zero<T>();
        double qe = 1.0;
#pragma unroll
        for (int q = 0; q < LMAX; ++q)
            if (q < len) {   // the last valid layer wins; `q == len - 1` would become a dynamic index
                pe = X[q];
                qe = y;
            }
        sP[s * LANES + lane] = pe;
        sQ[s * LANES + lane] = qe;
    }
    __syncthreads();
    T bin = v_zero<T>();
    for (int t = 0; t < s; ++t) bin = v_axpy(sQ[t * LANES + lane], bin, sP[t * LANES + lane]);
    __syncthreads();
    // b_z = X_z + Y_z b_in, with Y_z rebuilt from g and beta
#pragma unroll
    for (int q = 0; q < LMAX; ++q)
        if (q < len) {
            const int z = z0 + q;
            y = (q == 0) ? ((z == 0) ? 0.0 : -G[0] * sb[z - 1]) : -G[q] * sb[z - 1] * y;
            X[q] = v_axpy(y, bin, X[q]);
        }
    // backward sweep, local input x_{z1} = 0
    double h = 1.0;
#pragma unroll
    for (int qq = 0; qq < LMAX; ++qq) {
        const int q = LMAX - 1 - qq;
        if (q < len) {
            const int z = z0 + q;
            const double cz = (z == n - 1) ? 0.0 : G[q] * sb[z];
            if (q == len - 1 || q == LMAX - 1) {   // len <= LMAX: keeps X[q + 1] in range
                h = -cz;
            } else {
                X[q] = v_axpy(-cz, X[q + 1], X[q]);
                h = -cz * h;
            }
        }
    }
    sP[s * LANES + lane] = len > 0 ? X[0] : v_zero<T>();
    sQ[s * LANES + lane] = len > 0 ? h : 1.0;
    __syncthreads();
    T xin = v_zero<T>();
    for (int t = NS - 1; t > s; --t) xin = v_axpy(sQ[t * LANES + lane], xin, sP[t * LANES + lane]);
    // x_z = X_z + H_z x_in, H rebuilt from the end of the segment
#pragma unroll
    for (int qq = 0; qq < LMAX; ++qq) {
        const int q = LMAX - 1 - qq;
        if (q < len) {
            const int z = z0 + q;
            const double cz = (z == n - 1) ? 0.0 : G[q] * sb[z];
            h = (q == len - 1) ? -cz : -cz * h;
            rhs[(long long)z * nsys + c] = v_axpy(h, xin, X[q]);
        }
    }
}

// ------------------------------------------- plain x transforms (initialize!/getindex)
struct XPlainArgs {
    int P1, P2, K1, k1max, nz;
    const double* pd;     // [nz][P2][P1]
    double* pd_out;
    const double2* mixed_in;  // [nz][P2][K1]
    double2* mixed_out;
    FftPlan plan;
    const double2* tw;
};

// r2c along x of two physical rows per block -> mixed rows; grid ceil(nz*P2/2)
__global__ void __launch_bounds__(256) k_x_r2c(XPlainArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* b0 = tw + a.P1;
    double2* b1 = b0 + a.P1;
    const long long rows = (long long)a.nz * a.P2;
    const long long r0 = 2LL * blockIdx.x, r1 = r0 + 1;
    for (int i = threadIdx.x; i < a.P1; i += blockDim.x) tw[i] = a.tw[i];
    for (int x = threadIdx.x; x < a.P1; x += blockDim.x) {
        const double va = a.pd[r0 * a.P1 + x];
        const double vb = (r1 < rows) ? a.pd[r1 * a.P1 + x] : 0.0;
        b0[x] = make_double2(va, vb);
    }
    __syncthreads();
    double2* res = fft_big<double, -1>(b0, b1, 1, a.P1, 1, true, a.plan, tw);
    for (int k = threadIdx.x; k <= a.k1max; k += blockDim.x) {
        double2 A, B;
        unpack_pair<double>(res, k, a.P1, A, B);
        a.mixed_out[r0 * a.K1 + k] = A;
        if (r1 < rows) a.mixed_out[r1 * a.K1 + k] = B;
    }
}

// c2r along x of two mixed rows per block -> physical rows; grid ceil(nz*P2/2)
__global__ void __launch_bounds__(256) k_x_c2r(XPlainArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* b0 = tw + a.P1;
    double2* b1 = b0 + a.P1;
    const long long rows = (long long)a.nz * a.P2;
    const long long r0 = 2LL * blockIdx.x, r1 = r0 + 1;
    for (int i = threadIdx.x; i < a.P1; i += blockDim.x) tw[i] = a.tw[i];
    for (int k = threadIdx.x; k < a.P1; k += blockDim.x) {
        if (k > a.k1max && k < a.P1 - a.k1max) b0[k] = make_double2(0.0, 0.0);
        if (k <= a.k1max)
            build_packed<double>(b0, a.mixed_in + r0 * a.K1, (r1 < rows) ? a.mixed_in + r1 * a.K1 : nullptr, k, a.P1);
    }
    __syncthreads();
    double2* res = fft_big<double, +1>(b0, b1, 1, a.P1, 1, true, a.plan, tw);
    for (int x = threadIdx.x; x < a.P1; x += blockDim.x) {
        a.pd_out[r0 * a.P1 + x] = res[x].x;
        if (r1 < rows) a.pd_out[r1 * a.P1 + x] = res[x].y;
    }
}

// ------------------------------------------- output helpers (snapshots, profiles)
// Half-grid-point shift of one field in the frequency domain (shift!/unshift!,
// src/physical_space.jl:321-336): q(k1, k2) *= exp(sign i pi (k1/P1 + k2/P2)) for
// the default physical size (P1, P2).  grid (ceil(F/256), nz), dst may equal src.
__global__ void __launch_bounds__(256) k_half_shift(double2* dst, const double2* __restrict__ src, Geo g, int P1, int P2,
                                                     double sign) {
    const int mo = blockIdx.x * blockDim.x + threadIdx.x;
    if (mo >= g.F) return;
    const int z = blockIdx.y;
    const int j = mo / g.K1, k1 = mo - j * g.K1;
    const int k2 = j <= g.k2max ? j : j - g.K2;
    double s, c;
    sincospi(sign * ((double)k1 / (double)P1 + (double)k2 / (double)P2), &s, &c);
    const long long idx = (long long)z * g.F + mo;
    const double2 q = src[idx];
    dst[idx] = make_double2(q.x * c - q.y * s, q.x * s + q.y * c);
}

// Mean profiles on the device (MeanProfiles, src/logging.jl:333-491): the
// horizontal mean of a frequency-space field is the real part of its (0,0) mode.
// prof[m][f][0..n3] holds one sample per field (vel3 with its two boundary entries,
// which stay zero as in log_state!); acc += w (prev + sample) adds one trapezoid,
// and prev takes the new sample.  w = 0 only records the sample.
// grid (members), block 128.
__global__ void __launch_bounds__(128) k_profile_sample(Geo g, const double2* __restrict__ u, double* acc, double* prev,
                                                         double w, int m0, const int* active) {
    const int m = m0 + blockIdx.x;
    if (active && !active[m]) return;
    const int n = g.n3 + 1;
    const double2* S = u + (long long)m * g.mstride;
    double* A = acc + (long long)m * 3 * n;
    double* Pv = prev + (long long)m * 3 * n;
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
        const int f = i / n, z = i - f * n;
        double v = 0.0;
        if (f < 2) {
            if (z < g.n3) v = S[fld_off(g, f) + (long long)z * g.F].x;
        } else if (z >= 1 && z <= g.n3 - 1) {
            v = S[fld_off(g, 2) + (long long)(z - 1) * g.F].x;
        }
        A[i] += w * (Pv[i] + v);
        Pv[i] = v;
    }
}

#include "bld_ypass2.cuh"

// ------------------------------------------------------------ progress statistics
// Horizontal statistics of one member's spectral state per (field, layer): the
// mean Re q(0,0) and the mean square over the physical plane by Parseval,
// sum |q|^2 with the modes k1 > 0 counted twice (their conjugates are not
// stored); the physical grids that sample a field band-limited to |k| <= kmax
// hold at least 2 kmax + 1 points, so both are exact (ProgressMonitor,
// src/logging.jl:246-266).  grid (n3, 3), block 256; out[(f n3 + z) 2 + {0,1}].
__global__ void __launch_bounds__(256) k_progress_modes(Geo g, const double2* __restrict__ S, double* out) {
    const int z = blockIdx.x, f = blockIdx.y;
    if (f == 2 && z >= g.n3 - 1) return;
    const double2* L = S + fld_off(g, f) + (long long)z * g.F;
    double s = 0.0;
    for (int i = threadIdx.x; i < g.F; i += blockDim.x) {
        const double2 q = L[i];
        const int k1 = i % g.K1;
        s += (k1 == 0 ? 1.0 : 2.0) * (q.x * q.x + q.y * q.y);
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[(f * g.n3 + z) * 2 + 0] = L[0].x;
        out[(f * g.n3 + z) * 2 + 1] = red[0];
    }
}

// max |v| over each of `nz` physical layers of n points; grid nz, block 256
__global__ void __launch_bounds__(256) k_layer_absmax(const double* __restrict__ v, long long n, double* out) {
    const double* L = v + (long long)blockIdx.x * n;
    double mx = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, fabs(L[i]));
    __shared__ double red[256];
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// Horizontal means of the wall-model stresses factor u_i sqrt(u_1^2 + u_2^2)
// over one physical layer of n points of u_1 (pu) and u_2 (pv)
// (stress_bc, src/processes/static_smagorinsky.jl:195-200; hmean,
// src/logging.jl:411-413).  One block of 256; out[0] tau13, out[1] tau23.
__global__ void __launch_bounds__(256) k_wall_stress_mean(const double* __restrict__ pu, const double* __restrict__ pv,
                                                          long long n, double factor, double* out) {
    double s1 = 0.0, s2 = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        const double u = pu[i], v = pv[i];
        const double sp = sqrt(u * u + v * v);
        s1 += factor * u * sp;
        s2 += factor * v * sp;
    }
    __shared__ double r1[256], r2[256];
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            r1[threadIdx.x] += r1[threadIdx.x + w];
            r2[threadIdx.x] += r2[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = r1[0] / (double)n;
        out[1] = r2[0] / (double)n;
    }
}

// ----------------------------------------------------------- seeded initial fields
// Counter-based random numbers: the SplitMix64 output function (Steele, Lea and
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014) of a
// key plus a counter, so that any point's variate is computed independently
// and the host (numpy) produces the same bits.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// the stream key of one field: splitmix64(seed) xor splitmix64(field + 1)
__host__ __device__ __forceinline__ uint64_t init_key(uint64_t seed, int field) {
    return splitmix64(seed) ^ splitmix64((uint64_t)field + 1);
}

#define BLD_INIT_MAX_LAYERS 512
struct InitTables {
    double base[BLD_INIT_MAX_LAYERS];
    double scale[BLD_INIT_MAX_LAYERS];
};

// physical values base[z] + scale[z] r at the nz x plane points of the default
// grid (index i = z plane + y P1 + x); r uniform on [-1, 1) (distribution 0:
// 2 u - 1 with u = (splitmix64(key + 2 i) >> 11) 2^-53) or standard normal
// (distribution 1: Box-Muller, sqrt(-2 log(1 - u)) cos(2 pi u') with u' from
// key + 2 i + 1).  Grid-stride loop.
__global__ void __launch_bounds__(256) k_init_random(double* __restrict__ pd, int plane, int nz, InitTables t,
                                                     int distribution, uint64_t key) {
    const long long n = (long long)nz * plane;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(i / plane);
        const double u = (double)(splitmix64(key + 2ull * (uint64_t)i) >> 11) * 0x1.0p-53;
        double r;
        if (distribution == 0) {
            r = 2.0 * u - 1.0;
        } else {
            const double u2 = (double)(splitmix64(key + 2ull * (uint64_t)i + 1ull) >> 11) * 0x1.0p-53;
            r = sqrt(-2.0 * log(1.0 - u)) * cospi(2.0 * u2);
        }
        pd[i] = __dadd_rn(t.base[z], __dmul_rn(t.scale[z], r));   // rounded like the host's base + scale * r
    }
}
