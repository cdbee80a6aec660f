// Pressure projection of a stage value that is already stored (k_project_tile).
//
// Same arithmetic as k_project_seg for the stage kind S_NONE (div!,
// src/processes/pressure.jl:368-378; the LDL^T sweeps of ldiv!, :106-165;
// add_gradient!, :405-426; ConstantMean, src/processes/sources.jl:71-77), but
// each block's LN columns are brought into shared memory whole before any
// arithmetic: one 3-d TMA tensor copy per velocity component (LN modes x n3
// layers) and one 2-d copy of the LDL^T factors gamma, all completing on one
// mbarrier.  The loads of a block are then all in flight at once, with no
// registers held for them, and the segment sweeps read their layers from
// shared memory; the block writes u + grad p once.
//
// block (LN, NS) with NS segments of <= LMAX layers; grid (ceil(F / LN), members);
// dynamic shared memory project_tile_smem(n3, LN).  A tensor copy's shared-memory
// destination starts on a 128-byte boundary: the component tiles are padded to
// project_tile_stride values.
//
// k_project_pipe runs the same solve as a persistent kernel: each block walks the
// (member, LN-column tile) items i = blockIdx.x + k gridDim.x with two stages of
// shared memory, and the copies of item k + 1 are in flight while item k is
// solved and written, so a block's loads never wait behind its own arithmetic.
#pragma once

#include "bld_tma.cuh"

// values per component tile: n3 LN rounded up to 8 (128 bytes), so that every
// TMA destination starts on a 128-byte boundary whatever n3 and LN are
__host__ __device__ constexpr int project_tile_stride(int n3, int LN) { return (n3 * LN + 7) / 8 * 8; }
// bytes: alignment slack, the barrier, the three components, gamma
__host__ __device__ constexpr int project_tile_smem(int n3, int LN) {
    return 128 + 128 + 3 * project_tile_stride(n3, LN) * 16 + n3 * LN * 8;
}

// bytes of one stage of k_project_pipe (the three component tiles and gamma),
// rounded to 128; dynamic shared memory of k_project_pipe: slack, the two
// barriers, two stages
__host__ __device__ constexpr int project_stage_bytes(int n3, int LN) {
    return (3 * project_tile_stride(n3, LN) * 16 + n3 * LN * 8 + 127) / 128 * 128;
}
__host__ __device__ constexpr int project_pipe_smem(int n3, int LN) {
    return 128 + 128 + 2 * project_stage_bytes(n3, LN);
}

// Issues the TMA copies of the LN columns from c0 of member m into one stage
// (`tile` [3][FS], then gamma [n3][LN]), completing on `bar`.  The components
// sit at rows 0, n3, 2 n3 of the member's (3 n3 - 1)-row state; the last row of
// the third box lies past the state and is filled with zeros, as are columns
// past F.
template <int LN>
__device__ __forceinline__ void project_tile_issue(const CUtensorMap* umap, const CUtensorMap* gmap, double2* tile,
                                                   int FS, int n, int c0, int m, uint64_t* bar) {
    mbar_arrive_expect_tx(bar, (unsigned)(3 * n * LN * 16 + n * LN * 8));
    for (int f = 0; f < 3; ++f) tma_load_3d(tile + (size_t)f * FS, umap, 2 * c0, f * n, m, bar);
    tma_load_2d(reinterpret_cast<double*>(tile + 3 * FS), gmap, c0, 0, bar);
}

// The solve of one staged tile (columns c0 .. c0 + LN - 1 of member m), writing
// u + grad p to a.out; every thread of the block calls it, and it ends after a
// barrier that follows the block's last read of the tile.
template <int LMAX, int LN>
__device__ __forceinline__ void project_tile_solve(const ProjArgs& a, const double2* tile, int FS, int c0, int m,
                                                   double2 (*sP)[LN], double (*sQ)[LN]) {
    const Geo& g = a.g;
    const int n = g.n3;
    const long long F = g.F;
    const double* gt = reinterpret_cast<const double*>(tile + 3 * FS);   // [n][LN]
    const int NS = blockDim.y, s = threadIdx.y, lane = threadIdx.x;
    const int c = c0 + lane;
    const bool valid = c < F;
    const int L = (n + NS - 1) / NS;
    const int z0 = min(n, s * L), z1 = min(n, z0 + L);
    const int len = z1 - z0;
    const long long mb = (long long)m * g.mstride;
    const long long o1 = mb, o2 = mb + (long long)n * F, o3 = mb + 2LL * n * F;
    const int cc = valid ? c : 0;
    const int j = cc / g.K1, k1 = cc - j * g.K1;
    const bool mean_mode = (c == 0);
    const double e1 = a.d1[k1], e2 = a.d2[j];
    auto U = [&](int f, int z) -> double2 { return tile[f * FS + z * LN + lane]; };
    double2 wprev = make_double2(0.0, 0.0);
    if (z0 > 0 && len > 0) wprev = U(2, z0 - 1);
    double2 X[LMAX];
    double Y[LMAX];
    // ---- divergence and the segment-local forward sweep
#pragma unroll
    for (int q = 0; q < LMAX; ++q) {
        const int z = z0 + q;
        if (q < len) {
            const double2 uz = U(0, z), vz = U(1, z);
            const double2 wz = (z < n - 1) ? U(2, z) : make_double2(0.0, 0.0);
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
            const double gm = gt[z * LN + lane];
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
    // segment summaries: an empty segment passes its input through unchanged
    {
        double2 pe = make_double2(0.0, 0.0);
        double qe = 1.0;
        if (len > 0) {
#pragma unroll
            for (int q = 0; q < LMAX; ++q)
                if (q < len) {
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
    // ---- b_z, then the segment-local backward sweep
#pragma unroll
    for (int q = 0; q < LMAX; ++q)
        if (q < len) X[q] = make_double2(X[q].x + Y[q] * bin.x, X[q].y + Y[q] * bin.y);
#pragma unroll
    for (int qq = 0; qq < LMAX; ++qq) {
        const int q = LMAX - 1 - qq;
        if (q >= len) continue;
        const int z = z0 + q;
        if (z == n - 1) {
            Y[q] = 0.0;   // p_{n-1} = b_{n-1}
        } else {
            const double cz = gt[z * LN + lane] * a.alpha_i[z];
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
        if (len > 0) {
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
    // ---- pressure and gradient
#pragma unroll
    for (int q = 0; q < LMAX; ++q)
        if (q < len) X[q] = make_double2(X[q].x + Y[q] * pout.x, X[q].y + Y[q] * pout.y);
#pragma unroll
    for (int q = 0; q < LMAX; ++q) {
        const int z = z0 + q;
        if (q < len && valid) {
            const double2 pz = X[q];
            double2 pn = pout;
#pragma unroll
            for (int rr = 0; rr < LMAX; ++rr)
                if (rr == q + 1 && rr < len) pn = X[rr];
            double2 u = U(0, z), v = U(1, z);
            u.x += e1 * pz.y;
            u.y += -e1 * pz.x;
            v.x += e2 * pz.y;
            v.y += -e2 * pz.x;
            a.out[o1 + z * F + c] = u;
            a.out[o2 + z * F + c] = v;
            if (z < n - 1) {
                double2 w = U(2, z);
                const double ai = a.alpha_i[z];
                w.x += -1.0 * (-ai * pz.x + ai * pn.x);
                w.y += -1.0 * (-ai * pz.y + ai * pn.y);
                a.out[o3 + z * F + c] = w;
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

template <int LMAX, int LN>
__global__ void __launch_bounds__(LN * 32) k_project_tile(ProjArgs a, const __grid_constant__ CUtensorMap umap,
                                                        const __grid_constant__ CUtensorMap gmap, int* flag) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double2 sP[32][LN];
    __shared__ double sQ[32][LN];
    // the TMA destinations start on 128-byte boundaries
    unsigned char* base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    uint64_t* bar = reinterpret_cast<uint64_t*>(base);
    const int n = a.g.n3;
    const int FS = project_tile_stride(n, LN);
    double2* tile = reinterpret_cast<double2*>(base + 128);   // [3][FS >= n LN], then gamma
    const int tid = threadIdx.y * LN + threadIdx.x;
    const int c0 = blockIdx.x * LN;
    const int m = a.m0 + blockIdx.y;
    BLD_SKIP_INACTIVE(a, m);
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_async_shared();
    }
    __syncthreads();
    if (tid == 0) {
        prefetch_tmap(&umap);
        prefetch_tmap(&gmap);
        project_tile_issue<LN>(&umap, &gmap, tile, FS, n, c0, m, bar);
    }
    const long long wait_limit = g_bld_wait_limit;
    const bool arrived = mbar_wait_bounded(bar, 0, wait_limit);
    if (__syncthreads_or(!arrived)) {
        if (tid == 0) {
            atomicOr(flag + m, BLD_FLAG_TIMEOUT);
            mbar_wait_bounded(bar, 0);
        }
        return;
    }
    project_tile_solve<LMAX, LN>(a, tile, FS, c0, m, sP, sQ);
}

// persistent form: grid (blocks, 1), block (LN, NS), dynamic shared memory
// project_pipe_smem(n3, LN); the items are the ceil(F / LN) tiles of each of the
// nm members from a.m0 (inactive members skipped)
template <int LMAX, int LN>
__global__ void __launch_bounds__(LN * 32) k_project_pipe(ProjArgs a, int nm, const __grid_constant__ CUtensorMap umap,
                                                        const __grid_constant__ CUtensorMap gmap, int* flag) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double2 sP[32][LN];
    __shared__ double sQ[32][LN];
    unsigned char* base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    uint64_t* bar = reinterpret_cast<uint64_t*>(base);   // [2]
    const int n = a.g.n3;
    const int FS = project_tile_stride(n, LN);
    const int SB = project_stage_bytes(n, LN);
    const int tid = threadIdx.y * LN + threadIdx.x;
    const int ntiles = (int)((a.g.F + LN - 1) / LN);
    const int total = ntiles * nm;
    const int step = (int)gridDim.x;
    // this block's first active item
    int it = blockIdx.x;
    while (it < total && a.active && !a.active[a.m0 + it / ntiles]) it += step;
    if (it >= total) return;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_async_shared();
    }
    __syncthreads();
    if (tid == 0) {
        prefetch_tmap(&umap);
        prefetch_tmap(&gmap);
        project_tile_issue<LN>(&umap, &gmap, reinterpret_cast<double2*>(base + 128), FS, n, (it % ntiles) * LN,
                               a.m0 + it / ntiles, &bar[0]);
    }
    const long long wait_limit = g_bld_wait_limit;
    for (int k = 0; it < total; ++k) {
        const int s = k & 1;
        int nx = it + step;
        while (nx < total && a.active && !a.active[a.m0 + nx / ntiles]) nx += step;
        // stage s ^ 1 was last read by item k - 1, whose solve ended in a barrier
        if (tid == 0 && nx < total) {
            fence_async_shared();
            project_tile_issue<LN>(&umap, &gmap, reinterpret_cast<double2*>(base + 128 + (s ^ 1) * SB), FS, n,
                                   (nx % ntiles) * LN, a.m0 + nx / ntiles, &bar[s ^ 1]);
        }
        const int m = a.m0 + it / ntiles, c0 = (it % ntiles) * LN;
        const bool arrived = mbar_wait_bounded(&bar[s], (k >> 1) & 1, wait_limit);
        // a block whose wait expired stops here (uniformly), after the copies it
        // issued have landed
        if (__syncthreads_or(!arrived)) {
            if (tid == 0) {
                atomicOr(flag + m, BLD_FLAG_TIMEOUT);
                mbar_wait_bounded(&bar[s], (k >> 1) & 1);
                if (nx < total) mbar_wait_bounded(&bar[s ^ 1], ((k + 1) >> 1) & 1);
            }
            return;
        }
        project_tile_solve<LMAX, LN>(a, reinterpret_cast<const double2*>(base + 128 + s * SB), FS, c0, m, sP, sQ);
        it = nx;
    }
}
