// Advection x pass with two-pass shared-memory transforms (k_adv_x2).
//
// Rotation-form advection (src/processes/momentum_advection.jl:44-206), the same
// products and z-neighbour handling as k_adv_xb, for NR y rows per block
// streaming up a z chunk.  Per layer j:
//   * the six mixed rows of each of the NR rows (u, v, vort3 on C nodes; w,
//     vort1, vort2 on I nodes) were copied into shared memory by 1-d TMA bulk
//     copies (one per term: the NR rows are contiguous) while layer j - 1 ran;
//   * three packed lines per row, (u, v), (vort3, w), (vort1, vort2), go to the
//     physical domain by a two-pass inverse transform of P1 = A * B points:
//     pass 1 (B tasks per line) builds the Hermitian-extended packed spectrum
//     from the staged rows (FFTW's c2r convention: DC imaginary parts dropped)
//     and runs radix-A DFTs; pass 2 (A tasks per line) applies W_P^(j t) and
//     runs radix-B DFTs;
//   * one thread per (x, row) forms adv1, adv2 on C layer j and adv3 on I layer
//     j - 1 with the previous layer's values in registers;
//   * (adv1, adv2) of each row, and adv3 of two rows paired, are forward-
//     transformed the same way and unpacked to the k1 <= k1max modes.
// Pass-1 outputs sit at q (B + 1) + j in their line, so that both passes read
// and write consecutive addresses across a warp.
//
// The layers are software-pipelined by one phase: the unpack of layer j - 1
// (which reads the spectra) and pass 1 of layer j (which writes the pass-1
// buffer) touch different buffers, so they share one barrier interval, five
// barriers per layer in all, and the unpack's many small tasks fill the threads
// that pass 1 leaves idle.
//
// Variants (V): 0 as above; 2 (wide) runs it with 1.5x the threads (fewer
// product points, hence fewer registers, per thread: two blocks of six warps
// per SM in double precision instead of two of four); 3 (single precision up
// to P1 = 384) takes two rows per block instead of four: blocks of four warps,
// four per SM.
#pragma once

#include "bld_tma.cuh"

// y rows per block: 2 in double precision, 4 in single up to P1 = 384 (shared
// memory per block); variant 3 takes 2 in single precision too
__host__ __device__ constexpr int x2_rows(int csz, int P, int V = 0) {
    return V == 3 || csz == 16 || P > 384 ? 2 : 4;
}
__host__ __device__ constexpr int x2_threads(int B, int NR, int V = 0) {
    return (V == 2 ? (9 * NR * B / 2 + 31) : (3 * NR * B + 31)) / 32 * 32;
}
__host__ __device__ constexpr int x2_al(int b) { return (b + 127) / 128 * 128; }
// dynamic shared memory: barriers, twiddles, 2 stages x 6 terms x NR rows,
// pass-1 buffer (3 NR lines of A (B + 1)), physical / spectral lines (3 NR x P),
// forward inputs (NR + NR / 2 lines of P)
__host__ __device__ constexpr int x2_smem(int A, int B, int K1, int csz, int V = 0) {
    return 128 + x2_al(A * B * csz) + x2_al(2 * 6 * x2_rows(csz, A * B, V) * K1 * csz) +
           x2_al(3 * x2_rows(csz, A * B, V) * (A * (B + 1) + 128 / csz) * csz) +
           x2_al(3 * x2_rows(csz, A * B, V) * A * B * csz) +
           x2_al((x2_rows(csz, A * B, V) + x2_rows(csz, A * B, V) / 2) * A * B * csz);
}
// blocks per SM a variant is compiled for (its register cap; 0: the compiler's choice)
__host__ __device__ constexpr int x2_minb(int csz, int V) { return V == 2 ? 2 : (V == 3 ? 4 : 0); }

// grid (P2 / NR, nchunks, members), block x2_threads(B, NR, V); NR = x2_rows(sizeof(C), P, V)
template <typename R, int A, int B, int V = 0>
__global__ void __launch_bounds__(x2_threads(B, x2_rows(sizeof(cplx<R>), A * B, V), V), x2_minb(sizeof(cplx<R>), V))
    k_adv_x2(XArgs a, int* flag) {
    using C = cplx<R>;
    constexpr int P = A * B, NR = x2_rows(sizeof(C), P, V), NLI = 3 * NR, NLF = NR + NR / 2;
    constexpr int T = x2_threads(B, NR, V);
    constexpr int PPT = (NR * P + T - 1) / T;   // product points per thread
    constexpr int X1S = B + 1;                  // pass-1 stride of a task's outputs
    constexpr int E = 128 / (int)sizeof(C);     // elements per 128-byte bank row
    // line stride of the pass-1 buffer: line L + 1 starts where line L's task
    // B would, modulo a bank row, so warps spanning two lines stay conflict-free
    constexpr int X1L = A * X1S + ((B - A * X1S) % E + E) % E;
    static_assert(NR % 2 == 0, "adv3 lines pair two rows");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n3 = a.g.n3, k1max = a.g.k1max, K1 = a.g.K1;
    const int m = a.m0 + blockIdx.z;
    BLD_SKIP_INACTIVE(a, m);
    const int y0 = blockIdx.x * NR;
    const int z0 = blockIdx.y * a.zchunk, z1 = min(n3, z0 + a.zchunk);
    if (z0 >= z1) return;
    constexpr int csz = (int)sizeof(C);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
    unsigned char* p = smem_raw + 128;
    C* tw = reinterpret_cast<C*>(p);
    p += x2_al(P * csz);
    C* stage = reinterpret_cast<C*>(p);
    p += x2_al(2 * 6 * NR * K1 * csz);
    C* X1 = reinterpret_cast<C*>(p);
    p += x2_al(NLI * X1L * csz);
    C* Ph = reinterpret_cast<C*>(p);    // physical lines; later the forward spectra
    p += x2_al(NLI * P * csz);
    C* Fw = reinterpret_cast<C*>(p);    // forward inputs: NR (adv1, adv2) lines, NR / 2 adv3 pairs
    const C* Min = reinterpret_cast<const C*>(a.min) + (long long)m * a.min_mstride;
    C* Mout = reinterpret_cast<C*>(a.mout) + (long long)m * a.mout_mstride;
    const unsigned row_bytes = (unsigned)(NR * K1 * csz);
    // staged slots: u, v, vort3 (C); w, vort1, vort2 (I) = mixed terms 0, 1, 5, 2, 3, 4
    auto issue = [&](int j, int s) {
        const int nslots = (j < n3 - 1) ? 6 : 3;
        mbar_arrive_expect_tx(&bar[s], nslots * row_bytes);
        for (int r = 0; r < nslots; ++r) {
            const int t = r < 2 ? r : (r == 2 ? 5 : r - 1);
            bulk_load(stage + (size_t)(s * 6 + r) * NR * K1, mrow(Min, a, t, j, y0), row_bytes, &bar[s]);
        }
    };
    const int jb = max(0, z0 - 1);
    const long long wait_limit = g_bld_wait_limit;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_async_shared();
    }
    __syncthreads();
    if (threadIdx.x == 0) issue(jb, 0);
    // pass-2 twiddles W_P^(-j2 t) as [t][j2]: the lanes of a warp (consecutive j2)
    // read consecutive entries
    const C* twg = reinterpret_cast<const C*>(a.tw);
    for (int i = threadIdx.x; i < P; i += T) tw[i] = twg[(i / A) * (i % A)];

    R pu[PPT], pv[PPT], pw[PPT], po1[PPT], po2[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) pu[i] = pv[i] = pw[i] = po1[i] = po2[i] = R(0);

    int plf0 = 0, plf1 = 0;   // forward lines of the previous layer
    // layer j sits in stage slot (j - jb) & 1 and completes that slot's phase
    // ((j - jb) >> 1) & 1; the last pass (j = z1) only unpacks layer z1 - 1
    for (int j = jb; j <= z1; ++j) {
        const int s = (j - jb) & 1;
        // stage slot s ^ 1 was last read by layer j - 1's pass 1, several barriers ago
        if (threadIdx.x == 0 && j + 1 < z1) {
            fence_async_shared();
            issue(j + 1, s ^ 1);
        }
        // the unpack of layer j - 1 and the pass 1 of layer j share one barrier
        // interval: they touch different buffers (Ph, X1)
        if (j > jb) {
            for (int task = threadIdx.x; task < (plf1 - plf0) * K1; task += T) {
                const int Lr = fdiv(task, a.k1_magic), L = plf0 + Lr, f = task - Lr * K1;
                const C Zk = Ph[L * P + f], Zr = Ph[L * P + (P - f) % P];
                const C va = mk<R>((Zk.x + Zr.x) * R(0.5), (Zk.y - Zr.y) * R(0.5));
                const C vb = mk<R>((Zk.y + Zr.y) * R(0.5), -(Zk.x - Zr.x) * R(0.5));
                if (L < NR) {
                    mrow_w(Mout, a, 0, j - 1, y0 + L)[f] = va;
                    mrow_w(Mout, a, 1, j - 1, y0 + L)[f] = vb;
                } else {
                    const int r = 2 * (L - NR);
                    mrow_w(Mout, a, 2, j - 2, y0 + r)[f] = va;
                    mrow_w(Mout, a, 2, j - 2, y0 + r + 1)[f] = vb;
                }
            }
        }
        if (j == z1) break;
        const bool hasI = (j < n3 - 1);
        const bool arrived = mbar_wait_bounded(&bar[s], ((j - jb) >> 1) & 1, wait_limit);
        const C* cur = stage + (size_t)s * 6 * NR * K1;
        // ---- inverse pass 1: lines L = 3 r + p (pairs (u, v), (vort3, w), (vort1, vort2))
        for (int task = threadIdx.x; task < NLI * B; task += T) {
            const int L = task / B, jt = task - L * B;
            const int r = L / 3, pp = L - 3 * r;
            if (pp == 2 && !hasI) continue;
            const C* ra = cur + (size_t)((2 * pp) * NR + r) * K1;
            const C* rb = (pp == 1 && !hasI) ? nullptr : cur + (size_t)((2 * pp + 1) * NR + r) * K1;
            C x[A];
#pragma unroll
            for (int t = 0; t < A; ++t) {
                const int n = jt + B * t;
                const bool lo = n <= k1max, hi = n >= P - k1max;
                const int idx = lo ? n : P - n;
                C va = mk<R>(R(0), R(0)), vb = mk<R>(R(0), R(0));
                if (lo || hi) {
                    va = ra[idx];
                    if (rb) vb = rb[idx];
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
        // a block whose wait expired stops here (uniformly), after the copies it
        // issued have landed
        if (__syncthreads_or(!arrived)) {
            if (threadIdx.x == 0) {
                atomicOr(flag + m, BLD_FLAG_TIMEOUT);
                mbar_wait_bounded(&bar[s], ((j - jb) >> 1) & 1);
                if (j + 1 < z1) mbar_wait_bounded(&bar[s ^ 1], ((j + 1 - jb) >> 1) & 1);
            }
            return;
        }
        // ---- inverse pass 2 -> physical lines Ph[L][x]
        for (int task = threadIdx.x; task < NLI * A; task += T) {
            const int L = task / A, j2 = task - L * A;
            if (L % 3 == 2 && !hasI) continue;
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
        // ---- products at (x, row); outputs into Fw
        const bool emitC = (j >= z0);
        const bool emitI = (j >= z0) && (j >= 1);
#pragma unroll
        for (int i = 0; i < PPT; ++i) {
            const int idx = threadIdx.x + T * i;
            if (idx < NR * P) {
                const int r = idx / P, x = idx - r * P;
                const C c0 = Ph[(3 * r) * P + x], c1 = Ph[(3 * r + 1) * P + x];
                const C c2 = hasI ? Ph[(3 * r + 2) * P + x] : mk<R>(R(0), R(0));
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
                // adv3 on I layer j - 1 (:206)
                const R adv3 = po2[i] * R(0.5) * (pu[i] + u) - po1[i] * R(0.5) * (pv[i] + v);
                Fw[r * P + x] = mk<R>(adv1, adv2);
                R* a3 = reinterpret_cast<R*>(Fw + (NR + r / 2) * P + x);
                a3[r & 1] = adv3;
                pu[i] = u;
                pv[i] = v;
                pw[i] = w;
                po1[i] = q1;
                po2[i] = q2;
            }
        }
        __syncthreads();
        // ---- forward pass 1 (lines 0..NR-1: C layer j; NR..: I layer j - 1)
        const int lf0 = emitC ? 0 : NR, lf1 = emitI ? NLF : NR;
        for (int task = threadIdx.x; task < (lf1 - lf0) * B; task += T) {
            const int L = lf0 + task / B, jt = task % B;
            C x[A];
#pragma unroll
            for (int t = 0; t < A; ++t) x[t] = Fw[L * P + jt + B * t];
            dft<R, A, -1>(x);
#pragma unroll
            for (int q = 0; q < A; ++q) X1[L * X1L + q * X1S + jt] = x[q];
        }
        __syncthreads();
        // ---- forward pass 2 -> spectra in Ph
        for (int task = threadIdx.x; task < (lf1 - lf0) * A; task += T) {
            const int L = lf0 + task / A, j2 = task % A;
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
        plf0 = lf0;
        plf1 = lf1;
    }
}
