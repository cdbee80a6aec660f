// Smagorinsky x pass with two-pass shared-memory transforms (k_sgs_x2).
//
// The same model and z-neighbour handling as k_sgs_x (sgs_point), organised as
// k_adv_x2 organises the advection x pass: NR y rows per block walk up a z chunk;
// per C layer j
//   * the nine mixed rows of each row (u, v, w and their x and y derivatives;
//     six at the top layer, where w does not exist) were copied into shared
//     memory by 1-d TMA bulk copies (one per term: the NR rows are contiguous)
//     while layer j - 1 ran;
//   * five packed lines per row, (u, v), (u1, u2), (v1, v2), (w, w1), (w2, 0), go
//     to the physical domain by a two-pass inverse transform of P1 = A * B
//     points: pass 1 (B tasks per line) builds the Hermitian-extended packed
//     spectrum from the staged rows and runs radix-A DFTs; pass 2 (A tasks per
//     line) applies W_P^(j t) and runs radix-B DFTs;
//   * one thread per (x, row) evaluates the model (sgs_point) with the previous
//     layers' values in registers;
//   * the eight outputs of each row, as four packed lines, are forward-
//     transformed the same way and unpacked to the k1 <= k1max modes.
// The block has one thread per pass-1 task of the inverse transform (5 NR B),
// so that pass, the widest, runs in one round.
#pragma once

#include "bld_tma.cuh"

// y rows per block: 2 in double precision and above P1 = 384 in single, else 4;
// variant 1 takes 2 in single precision too (smaller blocks, more of them per SM)
__host__ __device__ constexpr int sx2_rows(int csz, int P, int V = 0) { return V == 1 || csz == 16 || P > 384 ? 2 : 4; }
__host__ __device__ constexpr int sx2_threads(int B, int NR) { return (5 * NR * B + 31) / 32 * 32; }
// dynamic shared memory: barriers, twiddles, 2 stages x 9 terms x NR rows, the
// pass-1 buffer (5 NR lines of A (B + 1) plus padding), physical / spectral
// lines (5 NR x P), forward inputs (4 NR x P)
__host__ __device__ constexpr int sx2_smem(int A, int B, int K1, int csz, int V = 0) {
    return 128 + x2_al(A * B * csz) + x2_al(2 * 9 * sx2_rows(csz, A * B, V) * K1 * csz) +
           x2_al(5 * sx2_rows(csz, A * B, V) * (A * (B + 1) + 128 / csz) * csz) +
           x2_al(5 * sx2_rows(csz, A * B, V) * A * B * csz) + x2_al(4 * sx2_rows(csz, A * B, V) * A * B * csz);
}

// grid (P2 / NR, nchunks, members), block sx2_threads(B, NR); NR = sx2_rows(sizeof(C), P, V)
template <typename R, int A, int B, int V = 0>
__global__ void __launch_bounds__(sx2_threads(B, sx2_rows(sizeof(cplx<R>), A * B, V))) k_sgs_x2(XArgs a) {
    using C = cplx<R>;
    constexpr int P = A * B, NR = sx2_rows(sizeof(C), P, V), NLI = 5 * NR, NLF = 4 * NR;
    constexpr int T = sx2_threads(B, NR);
    constexpr int PPT = (NR * P + T - 1) / T;   // model points per thread
    constexpr int X1S = B + 1;                  // pass-1 stride of a task's outputs
    constexpr int E = 128 / (int)sizeof(C);     // elements per 128-byte bank row
    constexpr int X1L = A * X1S + ((B - A * X1S) % E + E) % E;
    constexpr int csz = (int)sizeof(C);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n3 = a.g.n3, k1max = a.g.k1max, K1 = a.g.K1;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    const int y0 = blockIdx.x * NR;
    const int z0 = blockIdx.y * a.zchunk, z1 = min(n3, z0 + a.zchunk);
    if (z0 >= z1) return;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
    unsigned char* p = smem_raw + 128;
    C* tw = reinterpret_cast<C*>(p);
    p += x2_al(P * csz);
    C* stage = reinterpret_cast<C*>(p);
    p += x2_al(2 * 9 * NR * K1 * csz);
    C* X1 = reinterpret_cast<C*>(p);
    p += x2_al(NLI * X1L * csz);
    C* Ph = reinterpret_cast<C*>(p);   // physical lines; later the forward spectra
    p += x2_al(NLI * P * csz);
    C* Fw = reinterpret_cast<C*>(p);   // forward inputs: four packed output lines per row
    const C* Min = reinterpret_cast<const C*>(a.min) + (long long)m * a.min_mstride;
    C* Mout = reinterpret_cast<C*>(a.mout) + (long long)m * a.mout_mstride;
    const double* lcm = a.lc + (long long)m * n3;
    const double* lim = a.li + (long long)m * (n3 - 1);
    const R fs_lo = (R)a.wall[4 * m + 0], fs_hi = (R)a.wall[4 * m + 1];
    const R ft_lo = (R)a.wall[4 * m + 2], ft_hi = (R)a.wall[4 * m + 3];
    const R wlo = (R)a.w_lo, whi = (R)a.w_hi;
    const unsigned row_bytes = (unsigned)(NR * K1 * csz);
    const long long wait_limit = g_bld_wait_limit;
    // input terms of C layer j: u, v, u1, u2, v1, v2, and below the top layer w, w1, w2
    auto issue = [&](int j, int s) {
        const bool hi = (j <= n3 - 2);
        mbar_arrive_expect_tx(&bar[s], (hi ? 9u : 6u) * row_bytes);
        for (int t = 0; t < 9; ++t)
            if (hi || (t != 2 && t != 7 && t != 8))
                bulk_load(stage + (size_t)(s * 9 + t) * NR * K1, mrow(Min, a, t, j, y0), row_bytes, &bar[s]);
    };
    const int jb = max(0, z0 - 2);
    const int jend = min(n3, z1 + 1);
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_async_shared();
    }
    __syncthreads();
    if (threadIdx.x == 0) issue(jb, 0);   // jb <= z0 <= n3 - 1
    // pass-2 twiddles W_P^(-j2 t) as [t][j2]
    const C* twg = reinterpret_cast<const C*>(a.tw);
    for (int i = threadIdx.x; i < P; i += T) tw[i] = twg[(i / A) * (i % A)];

    SgsCarry<R> cy[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) cy[i] = SgsCarry<R>{};

    // forward lines of the previous layer, and which of its outputs it writes
    bool pfw = false, pdoC = false, pdo67 = false, pdo5 = false;
    // the last pass (j = jend + 1) only unpacks layer jend
    for (int j = jb; j <= jend + 1; ++j) {
        const bool hasC = (j <= n3 - 1), hasI = (j <= n3 - 2);
        const int s = (j - jb) & 1;
        // stage s ^ 1 was last read by layer j - 1's pass 1, several barriers ago
        const bool more = hasC && j + 1 <= min(jend, n3 - 1);
        if (threadIdx.x == 0 && more) {
            fence_async_shared();
            issue(j + 1, s ^ 1);
        }
        // the unpack of layer j - 1 shares a barrier interval with the pass 1 of
        // layer j: they touch different buffers (Ph, X1)
        if (pfw) {
            // ---- unpack layer j - 1's spectra: pairs (0,1) (2,3) (4,5) (6,7)
            for (int task = threadIdx.x; task < NLF * K1; task += T) {
                const int line = fdiv(task, a.k1_magic), k = task - line * K1;
                const int r = line / 4, q = line - 4 * r, y = y0 + r;
                C Av, Bv;
                unpack_pair<R, 0>(Ph + line * P, k, P, Av, Bv);
                const int ta = 2 * q, tb = 2 * q + 1;
                if (ta <= 4) {
                    if (pdoC) mrow_w(Mout, a, ta, j - 2, y)[k] = Av;
                } else if (pdo67) {
                    mrow_w(Mout, a, ta, j - 2, y)[k] = Av;
                }
                if (tb <= 4) {
                    if (pdoC) mrow_w(Mout, a, tb, j - 2, y)[k] = Bv;
                } else if (tb == 5) {
                    if (pdo5) mrow_w(Mout, a, 5, j - 3, y)[k] = Bv;
                } else if (pdo67) {
                    mrow_w(Mout, a, tb, j - 2, y)[k] = Bv;
                }
            }
        }
        if (j == jend + 1) break;
        bool arrived = true;
        if (hasC) {
            arrived = mbar_wait_bounded(&bar[s], ((j - jb) >> 1) & 1, wait_limit);
            const C* cur = stage + (size_t)s * 9 * NR * K1;
            // ---- inverse pass 1: lines L = 5 r + qq, packed pairs of terms
            // (0,1) (3,4) (5,6) (2,7) (8,-), the last two only below the top layer
            for (int task = threadIdx.x; task < NLI * B; task += T) {
                const int L = task / B, jt = task - L * B;
                const int r = L / 5, qq = L - 5 * r;
                const int ta = (0x82530 >> (4 * qq)) & 0xF, tb = (0xF7641 >> (4 * qq)) & 0xF;
                const bool oka = qq < 3 || hasI, okb = qq < 3 || (qq == 3 && hasI);
                const C* ra = cur + (size_t)(ta * NR + r) * K1;
                const C* rb = cur + (size_t)(tb * NR + r) * K1;
                C x[A];
#pragma unroll
                for (int t = 0; t < A; ++t) {
                    const int n = jt + B * t;
                    const bool lo = n <= k1max, hi = n >= P - k1max;
                    const int idx = lo ? n : P - n;
                    C va = mk<R>(R(0), R(0)), vb = mk<R>(R(0), R(0));
                    if (lo || hi) {
                        if (oka) va = ra[idx];
                        if (okb) vb = rb[idx];
                    }
                    if (n == 0)
                        x[t] = mk<R>(va.x, vb.x);
                    else if (lo)
                        x[t] = mk<R>(va.x - vb.y, va.y + vb.x);
                    else
                        x[t] = mk<R>(va.x + vb.y, -va.y + vb.x);   // zero outside the bands
                }
                dft<R, A, +1>(x);
#pragma unroll
                for (int q = 0; q < A; ++q) X1[L * X1L + q * X1S + jt] = x[q];
            }
        }
        // a block whose wait expired stops here (uniformly), after the copies it
        // issued have landed
        if (__syncthreads_or(!arrived)) {
            if (threadIdx.x == 0) {
                atomicOr(a.flag + m, BLD_FLAG_TIMEOUT);
                mbar_wait_bounded(&bar[s], ((j - jb) >> 1) & 1);
                if (more) mbar_wait_bounded(&bar[s ^ 1], ((j + 1 - jb) >> 1) & 1);
            }
            return;
        }
        if (hasC) {
            // ---- inverse pass 2 -> physical lines Ph[L][x]
            for (int task = threadIdx.x; task < NLI * A; task += T) {
                const int L = task / A, j2 = task - L * A;
                C x[B];
#pragma unroll
                for (int t = 0; t < B; ++t) x[t] = X1[L * X1L + j2 * X1S + t];
#pragma unroll
                for (int t = 1; t < B; ++t) x[t] = c_tw<+1>(x[t], tw[t * A + j2]);
                dft<R, B, +1>(x);
#pragma unroll
                for (int q = 0; q < B; ++q) Ph[L * P + j2 + A * q] = x[q];
            }
            __syncthreads();
        }
        const int c = j - 1;   // C layer completed at this step
        const bool doC = (j >= 1) && (c >= z0) && (c < z1);
        const bool do67 = (j >= 1) && (j <= n3 - 1) && (c >= z0) && (c < z1);
        const bool do5 = (j >= 2) && (j - 2 >= z0) && (j - 2 < z1) && (j - 2 <= n3 - 2);
        // ---- the model at (x, row)
#pragma unroll
        for (int i = 0; i < PPT; ++i) {
            const int idx = threadIdx.x + T * i;
            if (idx < NR * P) {
                const int r = idx / P, x = idx - r * P;
                R u = 0, v = 0, u1 = 0, u2 = 0, v1 = 0, v2 = 0, w = whi, w1 = 0, w2 = 0;
                if (hasC) {
                    const C c0 = Ph[(5 * r + 0) * P + x], c1 = Ph[(5 * r + 1) * P + x];
                    const C c2 = Ph[(5 * r + 2) * P + x];
                    u = c0.x; v = c0.y; u1 = c1.x; u2 = c1.y; v1 = c2.x; v2 = c2.y;
                    if (hasI) {
                        const C c3 = Ph[(5 * r + 3) * P + x], c4 = Ph[(5 * r + 4) * P + x];
                        w = c3.x; w1 = c3.y; w2 = c4.x;
                    }
                }
                R o[8];
                sgs_point<R>(a, j, n3, hasC, lcm, lim, fs_lo, fs_hi, ft_lo, ft_hi, wlo, u, v, u1, u2, v1, v2, w, w1,
                             w2, cy[i], o);
                if (doC || do5) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) Fw[(4 * r + q) * P + x] = mk<R>(o[2 * q], o[2 * q + 1]);
                }
            }
        }
        if (doC || do5) {
            __syncthreads();
            // ---- forward pass 1
            for (int task = threadIdx.x; task < NLF * B; task += T) {
                const int L = task / B, jt = task - L * B;
                C x[A];
#pragma unroll
                for (int t = 0; t < A; ++t) x[t] = Fw[L * P + jt + B * t];
                dft<R, A, -1>(x);
#pragma unroll
                for (int q = 0; q < A; ++q) X1[L * X1L + q * X1S + jt] = x[q];
            }
            __syncthreads();
            // ---- forward pass 2 -> spectra in Ph
            for (int task = threadIdx.x; task < NLF * A; task += T) {
                const int L = task / A, j2 = task - L * A;
                C x[B];
#pragma unroll
                for (int t = 0; t < B; ++t) x[t] = X1[L * X1L + j2 * X1S + t];
#pragma unroll
                for (int t = 1; t < B; ++t) x[t] = c_tw<-1>(x[t], tw[t * A + j2]);
                dft<R, B, -1>(x);
#pragma unroll
                for (int q = 0; q < B; ++q) Ph[L * P + j2 + A * q] = x[q];
            }
            __syncthreads();
        }
        pfw = doC || do5;
        pdoC = doC;
        pdo67 = do67;
        pdo5 = do5;
    }
}
