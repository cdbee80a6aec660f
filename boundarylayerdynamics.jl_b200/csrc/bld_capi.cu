// Host side of the engine: the C ABI declared in include/bld.h, set-up of the
// discretisation tables (the reference's init_process methods), device buffers,
// kernel launch schedules per RK stage and CUDA-graph replay of whole steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <functional>
#include <string>
#include <tuple>
#include <initializer_list>
#include <vector>

#include "bld.h"
#include "bld_kernels.cuh"
#include "bld_warpx.cuh"
#include "bld_advx2.cuh"
#include "bld_project_tile.cuh"
#include "bld_sgsx2.cuh"

double2 h_wtab64[BLD_WTAB_SIZE];
float2 h_wtab32[BLD_WTAB_SIZE];

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? BLD_ERR_OUT_OF_MEMORY : BLD_ERR_CUDA, \
                        "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__);  \
    } while (0)

#define BLD_TRY(expr)          \
    do {                       \
        int s_ = (expr);       \
        if (s_ != BLD_OK) return s_; \
    } while (0)

// ---------------------------------------------------------------- FFT sizes and plans
bool smooth_of(int n, std::initializer_list<int> primes) {
    if (n < 2) return false;
    for (int p : primes)
        while (n % p == 0) n /= p;
    return n == 1;
}
bool smooth23(int n) { return smooth_of(n, {2, 3}); }
// sizes the block Stockham kernels transform: products of 2, 3, 5 and 7
bool smooth2357(int n) { return smooth_of(n, {2, 3, 5, 7}); }

int next_even_smooth(int n) {
    int m = std::max(n, 2);
    while (!(m % 2 == 0 && smooth23(m))) ++m;
    return m;
}

// Fewest Stockham stages whose radices are register codelet sizes, then the
// smallest largest radix (register pressure), capped at BLD_FP32_MAXR / BLD_FP64_MAXR;
// nst = 0 if no such plan of at most four stages exists.
FftPlan make_plan(int n, bool fp32 = false) {
    static const int rads[] = {32, 24, 18, 16, 15, 14, 12, 10, 9, 8, 7, 6, 5, 4, 3, 2};
    const int cap = fp32 ? BLD_FP32_MAXR : BLD_FP64_MAXR;
    FftPlan best{};
    best.n = n;
    best.nst = 0;
    int best_st = 99, best_max = 99;
    int seq[6];
    // depth-first search over radix sequences (n <= 1024 of 2, 3, 5, 7 needs at most 4 stages of <= 18)
    auto dfs = [&](auto&& self, int rem, int depth, int mx) -> void {
        if (depth > 4 || depth > best_st) return;
        if (rem == 1) {
            if (depth < best_st || (depth == best_st && mx < best_max)) {
                best_st = depth;
                best_max = mx;
                best.nst = depth;
                for (int i = 0; i < depth; ++i) best.radix[i] = seq[i];
            }
            return;
        }
        for (int r : rads) {
            if (r > cap || rem % r) continue;
            seq[depth] = r;
            self(self, rem / r, depth + 1, std::max(mx, r));
        }
    };
    dfs(dfs, n, 0, 0);
    return best;
}

// quadratic-dealiasing size of the reference (src/physical_space.jl:49-56)
int pdsize_quadratic(int kmax) {
    const double l = std::log2(1.0 + kmax);
    if (l == std::floor(l)) return 3 * kmax + 3;
    return 3 * kmax + ((kmax % 2 == 1) ? 1 : 2);
}

struct DevTw {
    void* d64 = nullptr;
    void* d32 = nullptr;
};

// a y-pass variant: per-term (per-field) blocks with a two-buffer FFT, or one
// block for all terms (fields) of a layer with an in-place FFT
struct YCfg {
    int all = 0;
    int NL = 4;    // k1 lines per term (per field and line set)
    int thr = 256;
    int wfft = 0;  // per-term kernels: radix of the warp transform (P2 = 32 wfft), 0 = block stages
    int tp = 0;    // 1: two-pass kernels (k_inv_y2 / k_fwd_y2), BLD_Y2_NL lines, P2 = A * B;
                   // 2: inverse pass with TMA-staged tiles (k_inv_y3), BLD_Y3_NL lines;
                   // 3: two-pass kernels on 8 lines (forward: 3 blocks per SM, 4 outputs in flight;
                   //    inverse: 3 blocks per SM in double, 4 in single precision);
                   // 4: forward two-pass kernel, single precision, 2 outputs in flight
    int zc = 1;    // tp 2: layer chunks (blocks along z)
};

// radices of the warp y transforms compiled for the per-term y kernels
// (24 in single precision only)
bool wfft_radix_ok(int r, bool fp32) {
    return r == 2 || r == 3 || r == 4 || r == 6 || r == 8 || r == 9 || r == 12 || r == 16 || (fp32 && r == 24);
}

struct Space {
    bool on = false;
    int P1 = 0, P2 = 0, ref_P1 = 0, ref_P2 = 0;
    FftPlan plan1{}, plan2{};
    int ntin = 0, ntout = 0;
    void* min = nullptr;
    void* mout = nullptr;
    long long min_ms = 0, mout_ms = 0;  // elements per member
    int YT = 1, PPT = 1, zchunk = 1, nchunks = 1;  // x kernels: rows per block, points per thread, z chunks
    int xw = 0;                                     // > 0: warp-per-row x kernel with xw warps per block
    int xwmb = 1;                                   // warp-per-row kernel: register cap (min blocks of 128 threads)
    int zmult = 2;                                  // x kernels: z-chunk count multiplier in halves (autotuned)
    int xb = 0;                                     // block of warps per row (advection): 1 three warps, 2 five (pipelined)
    int x2 = 0;                                     // 1 + V: two-pass shared-memory x kernel k_adv_x2<.., V> (advection)
    int sx2 = 0;                                    // SGS block x kernel with two-pass line transforms: 1 plain,
                                                    // 2 registers capped for two blocks of 256 threads per SM,
                                                    // 3 / 4 as 1 / 2 with the input rows staged by bulk copies
    int sxk = 0;                                    // 1 + V: SGS x kernel k_sgs_x2<.., V> (rows staged by bulk copies, two-pass lines)
    int xr = 0;                                     // block x kernels: warp-transform radix (P1 = 32 xr), 0 = Stockham
    int fsets = 1;                                  // forward line sets (2 when a D2 contribution exists)
    YCfg inv, fwd;                                  // y-pass variants (chosen by the autotuner)
};

}  // namespace

struct bld_handle {
    bld_config cfg{};
    int device = 0;
    int B = 1;
    Geo g{};
    bool fp32 = false;
    cudaStream_t stream = nullptr;
    // state and integrator buffers [member][vel1|vel2|vel3]
    double2* u = nullptr;
    double2* t = nullptr;
    double2* du = nullptr;
    double2* dp = nullptr;
    double2* io = nullptr;     // staging for host-buffer calls
    double2* io2 = nullptr;
    double2* pscr = nullptr;
    double* gamma = nullptr;
    // tables
    double *d1 = nullptr, *d2 = nullptr, *DD1 = nullptr, *DD2 = nullptr;
    double *alpha_c = nullptr, *alpha_i = nullptr, *alpha_ext = nullptr, *mean_w = nullptr;
    double* inv_alpha_c = nullptr;   // 1 / alpha_c (the projections' divergence)
    double *lc2 = nullptr, *li2 = nullptr, *wall = nullptr, *src = nullptr, *mean_val = nullptr;
    int* flag = nullptr;
    int* flag_host = nullptr;
    std::vector<int> diverged;   // members whose rates turned non-finite since the last bld_get_diverged
    int* active = nullptr;        // [members] device mask of active ensemble slots
    std::vector<int> active_host;
    bool mask_on = false;        // the active mask applies to whole-ensemble steps only
    int proj_variant = 1;        // 0: column kernel, 1/2: z-segmented kernel, 3: with a shared tile (autotuned)
    int proj_tile = 0;           // LN > 0: projections of stored stage values by k_project_tile<.., LN> (autotuned)
    int proj_pipe = 0;           // 1: ... by its persistent two-stage form k_project_pipe<.., LN> (autotuned)
    double* prof_acc = nullptr;  // [members][3][n3+1] time integral of the mean profiles
    double* prof_prev = nullptr; // [members][3][n3+1] last sample
    bool prof_on = false;        // step graphs sample the profiles after every step
    std::vector<double> tab_dx3c, tab_dx3i, tab_x3c, tab_x3i;  // copies of the mapping tables
    std::vector<double> member_cs, member_z0;                  // current per-member SGS parameters
    std::map<int, DevTw> tw;
    Space adv, sgs;
    // physical-domain transforms at the default size
    int Pd1 = 0, Pd2 = 0;
    void* pd_buf = nullptr;     // double [nz][Pd2][Pd1]
    void* pd_mixed = nullptr;   // double2 [nz][Pd2][K1]
    // progress statistics (allocated by the first bld_progress_stats call)
    double* prog_small = nullptr;  // per-layer sums and maxima
    void* prog_buf = nullptr;      // double [n3][P2][P1] at the largest physical size
    void* prog_mixed = nullptr;    // double2 [n3][P2][K1]
    // host-side copies used by launches
    double w_lo = 0, w_hi = 0;
    int dyn_lo = 0, dyn_hi = 0;
    Linear lin{};
    bool slope_valid = false;
    bool ab2_started = false;
    double ab2_dt = 0;
    std::map<std::pair<int, double>, cudaGraphExec_t> graphs;
    std::map<std::pair<int, double>, cudaGraph_t> graph_src;   // kept for ensemble parent graphs
    std::map<std::vector<const void*>, cudaGraphExec_t> ens_graphs;  // parent graphs led by this handle
    size_t bytes = 0;
};

namespace {

int dalloc(bld_handle* h, void** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return fail(BLD_ERR_OUT_OF_MEMORY, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    h->bytes += bytes;
    return BLD_OK;
}

template <typename T>
int upload(bld_handle* h, T** dst, const std::vector<T>& v) {
    BLD_TRY(dalloc(h, (void**)dst, v.size() * sizeof(T)));
    if (!v.empty()) CUDA_TRY(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return BLD_OK;
}

int twiddles(bld_handle* h, int n) {
    if (h->tw.count(n)) return BLD_OK;
    std::vector<double2> w64(n);
    std::vector<float2> w32(n);
    for (int m = 0; m < n; ++m) {
        const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        const long double c = cosl(ang), s = sinl(ang);
        w64[m] = make_double2((double)c, (double)s);
        w32[m] = make_float2((float)c, (float)s);
    }
    DevTw t;
    BLD_TRY(dalloc(h, &t.d64, n * sizeof(double2)));
    BLD_TRY(dalloc(h, &t.d32, n * sizeof(float2)));
    CUDA_TRY(cudaMemcpy(t.d64, w64.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(t.d32, w32.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    h->tw[n] = t;
    return BLD_OK;
}

const void* twp(const bld_handle* h, int n, bool fp32) {
    const DevTw& t = h->tw.at(n);
    return fp32 ? t.d32 : t.d64;
}

size_t csize(bool fp32) { return fp32 ? sizeof(float2) : sizeof(double2); }

// y-pass lines per block: shared memory <= ~100 KB and outputs per thread <= 16
// y-pass lines per block: the largest of 16 (single) / 8, 4, 2 whose two
// shared line buffers (times `sets`) and twiddles stay within ~110 KB
int pick_y(int P2, bool fp32, int sets) {
    const size_t cs = csize(fp32);
    int NL = fp32 ? 16 : 8;
    while (NL > 2 && (size_t)(P2 + 2 * P2 * sets * NL) * cs > 110 * 1024) NL /= 2;
    return NL;
}

// choose tiles for a physical-domain space
// z chunks of the x kernels for the current rows per block: enough blocks to
// fill the GPU a few times over, at least 8 layers per chunk
void x_chunks(const bld_handle* h, Space& s) {
    const int n3 = h->g.n3;
    const int rows = s.x2 ? x2_rows((int)csize(h->fp32), s.P1, s.x2 - 1)
                           : (s.sxk ? sx2_rows((int)csize(h->fp32), s.P1, s.sxk - 1) : (s.xb ? 1 : (s.xw ? s.xw : s.YT)));
    const long long blocks_per_chunk = (long long)((s.P2 + rows - 1) / rows) * h->B;
    int want = (int)std::max<long long>(1, (900 + blocks_per_chunk - 1) / blocks_per_chunk);
    want = std::min(want, std::max(1, n3 / 8));
    // the autotuner may ask for more chunks (shorter streams, more blocks: a
    // smaller partial last wave), down to 4 layers per chunk
    want = std::min(std::max(1, want * s.zmult / 2), std::max(1, n3 / 4));
    s.zchunk = (n3 + want - 1) / want;
    s.nchunks = (n3 + s.zchunk - 1) / s.zchunk;
}

// (rows per block, points per thread) candidates of the x kernels: blocks of
// 32..256 threads whose two line buffers fit in 150 KB of shared memory
std::vector<std::pair<int, int>> x_candidates(const bld_handle* h, const Space& s, bool is_adv) {
    std::vector<std::pair<int, int>> out;
    const int lines = is_adv ? 3 : 5;
    for (int yt : {1, 2, 4}) {
        if (s.P2 % yt || yt * s.P1 > 1024) continue;
        if ((size_t)(s.P1 + 2 * lines * yt * s.P1) * csize(h->fp32) > 150 * 1024) continue;
        for (int ppt = 1; ppt <= 4; ++ppt) {
            const int pts = yt * s.P1;
            if (pts % ppt) continue;
            const int thr = pts / ppt;
            if (thr > 256 || thr < 32) continue;
            out.emplace_back(yt, ppt);
        }
    }
    return out;
}

void tile_space(const bld_handle* h, Space& s, bool is_adv) {
    // initial choice near 96 (advection, double) / 128 (SGS, double) / 192 (single)
    // threads; the autotuner replaces it with the measured best
    const int target = h->fp32 ? 192 : (is_adv ? 96 : 128);
    int best = 1 << 30;
    s.YT = 1;
    s.PPT = 0;
    for (auto c : x_candidates(h, s, is_adv)) {
        const int thr = c.first * s.P1 / c.second;
        const int score = std::abs(thr - target) + 24 * (c.second - 1) + 8 * (c.first - 1);
        if (score < best) {
            best = score;
            s.YT = c.first;
            s.PPT = c.second;
        }
    }
    x_chunks(h, s);
}

size_t smem_y(int P2, int NL, bool fp32) { return (size_t)(P2 + 2 * P2 * NL) * csize(fp32); }
// per-term y kernels with `lines` lines: twiddles and two line buffers for the
// block-wide stages, or twiddles and one buffer of P2 + 32 (swizzled) positions
// on a line stride of lines + 1 for the warp transforms
size_t smem_y_term(int P2, int lines, int wfft, bool fp32) {
    return (size_t)(wfft ? P2 + (P2 + 32) * (lines + 1) : P2 + 2 * P2 * lines) * csize(fp32);
}
// block x kernels: twiddles and two buffers of (3 or 5) YT lines, on a line stride
// P1 + 32 (swizzled positions) with warp line transforms (xr > 0)
size_t smem_adv(const Space& s, bool fp32) {
    return (size_t)(s.P1 + 2 * 3 * s.YT * (s.P1 + (s.xr ? 32 : 0))) * csize(fp32);
}
// the two-pass SGS kernel stages its input rows by bulk copies when a block's
// YT rows of K1 values fill whole 16-byte units
bool sgs_stage_fits(const Space& s, bool fp32, int K1) { return !fp32 || K1 % 2 == 0 || s.YT % 2 == 0; }
bool sgs_staged(const Space& s, bool fp32, int K1) { return s.sx2 >= 3 && sgs_stage_fits(s, fp32, K1); }

size_t smem_sgs(const Space& s, bool fp32, int K1) {
    if (s.sx2) {
        const int A = y2_radix_a(s.P1), B = y2_radix_b(s.P1);
        const int lp = fp32 ? twopass_line<float2>(A, B) : twopass_line<double2>(A, B);
        if (sgs_staged(s, fp32, K1))
            return (size_t)sgs_stage_offset(s.P1, 5 * s.YT, lp, (int)csize(fp32)) + 128 +
                   (size_t)2 * 9 * s.YT * K1 * csize(fp32);
        return (size_t)(s.P1 + 2 * 5 * s.YT * lp) * csize(fp32);
    }
    return (size_t)(s.P1 + 2 * 5 * s.YT * (s.P1 + (s.xr ? 32 : 0))) * csize(fp32);
}

// ------------------------------------------------------------------ kernel dispatch
// threads for an in-place transform of `lines` lines (one task per thread for
// radix >= 8, up to four for smaller radices); 0 if more than 384 are needed
int inplace_threads(const FftPlan& pl, int lines) {
    int thr = 32;
    for (int i = 0; i < pl.nst; ++i) {
        const int r = pl.radix[i];
        const int tpt = r <= 4 ? 4 : (r == 6 ? 3 : 1);  // inplace_tpt
        const int tasks = lines * pl.n / r;
        thr = std::max(thr, (tasks + tpt - 1) / tpt);
    }
    thr = (thr + 31) / 32 * 32;
    return thr <= 384 ? thr : 0;
}

// threads of a y-pass block: enough for the widest FFT stage of `lines` lines
int y_threads(const FftPlan& pl, int lines) {
    int rmin = 64;
    for (int i = 0; i < pl.nst; ++i) rmin = std::min(rmin, pl.radix[i]);
    const int tasks = lines * pl.n / rmin;
    return std::min(256, std::max(64, (tasks + 31) / 32 * 32));
}

// two-pass y kernels: compiled for P2 with a factorisation y2_radix_a/b (single
// precision up to 768, double up to 288) and their registers per block count
bool y2_ok(int P2, bool fp32) { return y2_radix_a(P2) > 0 && (fp32 || P2 <= 288); }
size_t smem_y2(int P2, int lines, bool fp32) { return (size_t)P2 * (1 + lines) * csize(fp32); }

template <typename R, int P>
int launch_y2_p(bld_handle* h, bool inverse, const void* args, dim3 grid, size_t sm, int tp) {
    constexpr int A = y2_radix_a(P), B = y2_radix_b(P);
    constexpr int MINB = y2_min_blocks<R>(B * BLD_Y2_NL);
    constexpr int MINBI = y2_min_blocks_inv<R>(B * BLD_Y2_NL);
    if (!inverse && tp == 3)
        k_fwd_y2<R, A, B, 3, 8, 4><<<grid, B * 8, sm, h->stream>>>(*static_cast<const FwdYArgs*>(args));
    else if (inverse && tp == 3)   // eight lines: three (double) or four (single precision) blocks per SM
        k_inv_y2<R, A, B, sizeof(R) == 8 ? 3 : 4, 8><<<grid, B * 8, sm, h->stream>>>(
            *static_cast<const InvYArgs*>(args));
    else if (!inverse && tp == 4 && sizeof(R) == 4)
        k_fwd_y2<R, A, B, MINB, BLD_Y2_NL, 2><<<grid, B * BLD_Y2_NL, sm, h->stream>>>(
            *static_cast<const FwdYArgs*>(args));
    else if (inverse)
        k_inv_y2<R, A, B, MINBI><<<grid, B * BLD_Y2_NL, sm, h->stream>>>(*static_cast<const InvYArgs*>(args));
    else
        k_fwd_y2<R, A, B, MINB><<<grid, B * BLD_Y2_NL, sm, h->stream>>>(*static_cast<const FwdYArgs*>(args));
    return BLD_OK;
}

template <typename R>
int launch_y2(bld_handle* h, int P2, bool inverse, const void* args, dim3 grid, size_t sm, int tp = 1) {
    switch (P2) {
        case 64: return launch_y2_p<R, 64>(h, inverse, args, grid, sm, tp);
        case 96: return launch_y2_p<R, 96>(h, inverse, args, grid, sm, tp);
        case 128: return launch_y2_p<R, 128>(h, inverse, args, grid, sm, tp);
        case 144: return launch_y2_p<R, 144>(h, inverse, args, grid, sm, tp);
        case 192: return launch_y2_p<R, 192>(h, inverse, args, grid, sm, tp);
        case 256: return launch_y2_p<R, 256>(h, inverse, args, grid, sm, tp);
        case 288: return launch_y2_p<R, 288>(h, inverse, args, grid, sm, tp);
        default: break;
    }
    if constexpr (sizeof(R) == 4) {
        switch (P2) {
            case 384: return launch_y2_p<R, 384>(h, inverse, args, grid, sm, tp);
            case 512: return launch_y2_p<R, 512>(h, inverse, args, grid, sm, tp);
            case 768: return launch_y2_p<R, 768>(h, inverse, args, grid, sm, tp);
            default: break;
        }
    }
    return fail(BLD_ERR_INVALID_CONFIG, "no two-pass y transform for P2=%d", P2);
}

// cuTensorMapEncodeTiled from the driver, found through the runtime (the
// library links only the static CUDA runtime)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// the members' states from `base` as a float64 tensor (2 K1, K2, 3 n3 - 1, members)
// with the box (2 NL, K2, 1, 1) of k_inv_y3
int state_tmap(const bld_handle* h, const void* base, int nl, CUtensorMap* out) {
    const Geo& g = h->g;
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return fail(BLD_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[4] = {(cuuint64_t)(2 * g.K1), (cuuint64_t)g.K2, (cuuint64_t)(3 * g.n3 - 1), (cuuint64_t)h->B};
    const cuuint64_t strides[3] = {(cuuint64_t)g.K1 * 16, (cuuint64_t)g.F * 16, (cuuint64_t)g.mstride * 16};
    const cuuint32_t box[4] = {(cuuint32_t)(2 * nl), (cuuint32_t)g.K2, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(BLD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return BLD_OK;
}

// k_project_tile applies: the pressure solve with <= 256 layers, an even number
// of modes per layer (gamma rows are 16-byte multiples for the TMA map) and
// LN columns x all layers within a block's shared memory
bool project_tile_ok(const bld_handle* h, int ln) {
    return h->cfg.pressure && h->g.n3 <= 256 && h->g.F % 2 == 0 && (ln == 4 || ln == 8 || ln == 16) &&
           project_tile_smem(h->g.n3, ln) <= 200 * 1024 && encode_tiled() != nullptr;
}

// k_project_pipe applies where k_project_tile does and two stages fit in 200 KB
bool project_pipe_ok(const bld_handle* h, int ln) {
    return project_tile_ok(h, ln) && project_pipe_smem(h->g.n3, ln) <= 200 * 1024;
}

// launches k_project_pipe<LMAX, LN>: as many blocks as are resident at once on
// the device (at most one per item)
template <int LMAX, int LN>
int launch_project_pipe(bld_handle* h, const ProjArgs& a, int nm, const CUtensorMap& umap, const CUtensorMap& gmap) {
    const int n3 = h->g.n3;
    dim3 block(LN, std::max(1, std::min(16, (n3 + LMAX - 1) / LMAX)));
    const size_t sm = project_pipe_smem(n3, LN);
    // resident blocks per SM at this block shape and shared memory, found once
    // per (kernel, n3) (the autotuner's first launch, outside any capture)
    static std::mutex mu;
    static std::map<int, int> per_sm_of_n3;
    int dev = 0, nsm = 0, per_sm = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = per_sm_of_n3.find(n3);
        if (it != per_sm_of_n3.end()) {
            per_sm = it->second;
        } else {
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_project_pipe<LMAX, LN>,
                                                                   (int)(block.x * block.y), sm));
            per_sm_of_n3[n3] = per_sm;
        }
    }
    const long long items = (h->g.F + LN - 1) / LN * (long long)nm;
    const int blocks = (int)std::min<long long>(items, (long long)std::max(1, per_sm) * nsm);
    k_project_pipe<LMAX, LN><<<blocks, block, sm, h->stream>>>(a, nm, umap, gmap, h->flag);
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// tensor maps of k_project_tile: the members' states from `u` as float64
// (2 F, 3 n3 - 1, members) with the box (2 LN, n3, 1), and gamma as (F, n3) with
// the box (LN, n3)
int project_tmaps(const bld_handle* h, const void* u, int ln, CUtensorMap* umap, CUtensorMap* gmap) {
    const Geo& g = h->g;
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return fail(BLD_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t udims[3] = {(cuuint64_t)(2 * g.F), (cuuint64_t)(3 * g.n3 - 1), (cuuint64_t)h->B};
    const cuuint64_t ustr[2] = {(cuuint64_t)g.F * 16, (cuuint64_t)g.mstride * 16};
    const cuuint32_t ubox[3] = {(cuuint32_t)(2 * ln), (cuuint32_t)g.n3, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(umap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(u), udims, ustr, ubox, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(BLD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    const cuuint64_t gdims[2] = {(cuuint64_t)g.F, (cuuint64_t)g.n3};
    const cuuint64_t gstr[1] = {(cuuint64_t)g.F * 8};
    const cuuint32_t gbox[2] = {(cuuint32_t)ln, (cuuint32_t)g.n3};
    r = fn(gmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, h->gamma, gdims, gstr, gbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(BLD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return BLD_OK;
}

// k_inv_y3 applies: a two-pass factorisation, whole K2 columns in one TMA box
// (K2 <= 256) and the staged tiles within the shared memory of a block
bool y3_ok(const bld_handle* h, int P2) {
    return y2_ok(P2, h->fp32) && h->g.K2 <= 256 &&
           y3_smem(P2, h->g.K2, (int)csize(h->fp32)) <= 227 * 1024 && encode_tiled() != nullptr;
}

template <typename R, int P>
int launch_y3_p(bld_handle* h, const InvYArgs& a, const CUtensorMap& map, dim3 grid) {
    constexpr int A = y2_radix_a(P), B = y2_radix_b(P);
    const size_t sm = y3_smem(P, h->g.K2, (int)sizeof(cplx<R>));
    k_inv_y3<R, A, B><<<grid, B * BLD_Y3_NL, sm, h->stream>>>(a, map);
    return BLD_OK;
}

template <typename R>
int launch_inv_y3(bld_handle* h, const Space& s, InvYArgs a, int nm) {
    CUtensorMap map;
    BLD_TRY(state_tmap(h, a.state, BLD_Y3_NL, &map));
    a.NL = BLD_Y3_NL;
    a.zchunk = (h->g.n3 + s.inv.zc - 1) / s.inv.zc;
    a.flag = h->flag;
    dim3 grid(a.nterms * nm, (h->g.K1 + BLD_Y3_NL - 1) / BLD_Y3_NL, (h->g.n3 + a.zchunk - 1) / a.zchunk);
    switch (s.P2) {
        case 64: return launch_y3_p<R, 64>(h, a, map, grid);
        case 96: return launch_y3_p<R, 96>(h, a, map, grid);
        case 128: return launch_y3_p<R, 128>(h, a, map, grid);
        case 144: return launch_y3_p<R, 144>(h, a, map, grid);
        case 192: return launch_y3_p<R, 192>(h, a, map, grid);
        case 256: return launch_y3_p<R, 256>(h, a, map, grid);
        case 288: return launch_y3_p<R, 288>(h, a, map, grid);
        default: break;
    }
    if constexpr (sizeof(R) == 4) {
        switch (s.P2) {
            case 384: return launch_y3_p<R, 384>(h, a, map, grid);
            case 512: return launch_y3_p<R, 512>(h, a, map, grid);
            case 768: return launch_y3_p<R, 768>(h, a, map, grid);
            default: break;
        }
    }
    return fail(BLD_ERR_INVALID_CONFIG, "no TMA y transform for P2=%d", s.P2);
}

template <typename R>
int launch_inv_y(bld_handle* h, const Space& s, InvYArgs a, int nm) {
    const YCfg& c = s.inv;
    a.NL = c.NL;
    const size_t cs = csize(sizeof(R) == 4);
    if (c.tp == 2) {
        BLD_TRY(launch_inv_y3<R>(h, s, a, nm));
        CUDA_TRY(cudaGetLastError());
        return BLD_OK;
    }
    if (c.tp) {
        const int nl = c.tp == 3 ? 8 : BLD_Y2_NL;
        a.NL = nl;
        dim3 grid(a.nterms * nm, (h->g.K1 + nl - 1) / nl, h->g.n3);
        BLD_TRY(launch_y2<R>(h, s.P2, true, &a, grid, smem_y2(s.P2, nl, sizeof(R) == 4), c.tp));
        CUDA_TRY(cudaGetLastError());
        return BLD_OK;
    }
    if (c.all) {
        dim3 grid((h->g.K1 + c.NL - 1) / c.NL, h->g.n3, nm);
        k_inv_y_all<R><<<grid, c.thr, (size_t)(s.P2 + s.P2 * a.nterms * c.NL) * cs, h->stream>>>(a);
    } else {
        dim3 grid(a.nterms * nm, (h->g.K1 + c.NL - 1) / c.NL, h->g.n3);
        const size_t sm = smem_y_term(s.P2, c.NL, c.wfft, sizeof(R) == 4);
        switch (c.wfft) {
            case 0: k_inv_y<R, 0><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 2: k_inv_y<R, 2><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 3: k_inv_y<R, 3><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 4: k_inv_y<R, 4><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 6: k_inv_y<R, 6><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 8: k_inv_y<R, 8><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 9: k_inv_y<R, 9><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 12: k_inv_y<R, 12><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 16: k_inv_y<R, 16><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 24:
                if constexpr (sizeof(R) == 4) {
                    k_inv_y<R, 24><<<grid, c.thr, sm, h->stream>>>(a);
                    break;
                }
                return fail(BLD_ERR_INVALID_CONFIG, "no warp y transform of radix %d", c.wfft);
            default: return fail(BLD_ERR_INVALID_CONFIG, "no warp y transform of radix %d", c.wfft);
        }
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

template <typename R>
int launch_fwd_y(bld_handle* h, const Space& s, FwdYArgs a, int nm) {
    const YCfg& c = s.fwd;
    a.NL = c.NL;
    const size_t cs = csize(sizeof(R) == 4);
    if (c.tp) {
        const int nl = c.tp == 3 ? 8 : BLD_Y2_NL;   // tp 1, 2, 4: BLD_Y2_NL lines
        a.NL = nl;
        dim3 grid(a.fields * nm, (h->g.K1 + nl - 1) / nl, h->g.n3);
        BLD_TRY(launch_y2<R>(h, s.P2, false, &a, grid, smem_y2(s.P2, s.fsets * nl, sizeof(R) == 4), c.tp));
        CUDA_TRY(cudaGetLastError());
        return BLD_OK;
    }
    if (c.all) {
        dim3 grid((h->g.K1 + c.NL - 1) / c.NL, h->g.n3, nm);
        k_fwd_y_all<R><<<grid, c.thr, (size_t)(s.P2 + s.P2 * 3 * s.fsets * c.NL) * cs, h->stream>>>(a);
    } else {
        dim3 grid(a.fields * nm, (h->g.K1 + c.NL - 1) / c.NL, h->g.n3);
        const size_t sm = smem_y_term(s.P2, s.fsets * c.NL, c.wfft, sizeof(R) == 4);
        switch (c.wfft) {
            case 0: k_fwd_y<R, 0><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 2: k_fwd_y<R, 2><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 3: k_fwd_y<R, 3><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 4: k_fwd_y<R, 4><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 6: k_fwd_y<R, 6><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 8: k_fwd_y<R, 8><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 9: k_fwd_y<R, 9><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 12: k_fwd_y<R, 12><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 16: k_fwd_y<R, 16><<<grid, c.thr, sm, h->stream>>>(a); break;
            case 24:
                if constexpr (sizeof(R) == 4) {
                    k_fwd_y<R, 24><<<grid, c.thr, sm, h->stream>>>(a);
                    break;
                }
                return fail(BLD_ERR_INVALID_CONFIG, "no warp y transform of radix %d", c.wfft);
            default: return fail(BLD_ERR_INVALID_CONFIG, "no warp y transform of radix %d", c.wfft);
        }
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// two-pass advection x kernel: compiled for P1 with a two-pass factorisation
// (single precision up to 768, double up to 288), whole row pairs per block;
// variants V = 2 (wide) in double precision, V = 3 (two rows) in single precision up to 384
bool x2_ok(const bld_handle* h, const Space& s, int V = 0) {
    const int cs = (int)csize(h->fp32);
    return y2_ok(s.P1, h->fp32) && s.P2 % x2_rows(cs, s.P1, V) == 0 &&
           (V == 0 || (V == 2 && !h->fp32) || (V == 3 && h->fp32 && s.P1 <= 384)) &&
           x2_smem(y2_radix_a(s.P1), y2_radix_b(s.P1), h->g.K1, cs, V) <= 227 * 1024;
}

template <typename R, int P, int V>
void launch_x2_pv(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    constexpr int A = y2_radix_a(P), B = y2_radix_b(P);
    constexpr int NR = x2_rows((int)sizeof(cplx<R>), P, V);
    dim3 grid(s.P2 / NR, s.nchunks, nm);
    const size_t sm = x2_smem(A, B, h->g.K1, (int)sizeof(cplx<R>), V);
    k_adv_x2<R, A, B, V><<<grid, x2_threads(B, NR, V), sm, h->stream>>>(a, h->flag);
}

template <typename R, int P>
int launch_x2_p(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    if constexpr (sizeof(R) == 8) {
        if (s.x2 == 3) return launch_x2_pv<R, P, 2>(h, s, a, nm), BLD_OK;
    }
    if constexpr (sizeof(R) == 4 && P <= 384) {
        if (s.x2 == 4) return launch_x2_pv<R, P, 3>(h, s, a, nm), BLD_OK;
    }
    launch_x2_pv<R, P, 0>(h, s, a, nm);
    return BLD_OK;
}

template <typename R>
int launch_adv_x2(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    switch (s.P1) {
        case 64: BLD_TRY((launch_x2_p<R, 64>(h, s, a, nm))); break;
        case 96: BLD_TRY((launch_x2_p<R, 96>(h, s, a, nm))); break;
        case 128: BLD_TRY((launch_x2_p<R, 128>(h, s, a, nm))); break;
        case 144: BLD_TRY((launch_x2_p<R, 144>(h, s, a, nm))); break;
        case 192: BLD_TRY((launch_x2_p<R, 192>(h, s, a, nm))); break;
        case 256: BLD_TRY((launch_x2_p<R, 256>(h, s, a, nm))); break;
        case 288: BLD_TRY((launch_x2_p<R, 288>(h, s, a, nm))); break;
        default:
            if constexpr (sizeof(R) == 4) {
                if (s.P1 == 384) { BLD_TRY((launch_x2_p<R, 384>(h, s, a, nm))); break; }
                if (s.P1 == 512) { BLD_TRY((launch_x2_p<R, 512>(h, s, a, nm))); break; }
                if (s.P1 == 768) { BLD_TRY((launch_x2_p<R, 768>(h, s, a, nm))); break; }
            }
            return fail(BLD_ERR_INVALID_CONFIG, "no two-pass x kernel for P1=%d", s.P1);
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// radices of the warp line transforms compiled into the block x kernels, and the
// points per thread that go with each (so that YT * 32 RAD / PPT threads are whole warps)
bool xr_radix_ok(int r) { return r == 2 || r == 3 || r == 4 || r == 6 || r == 8 || r == 9 || r == 12 || r == 16 || r == 24; }
constexpr int xr_ppt(int r) { return r <= 4 ? 1 : r <= 8 ? 2 : r <= 12 ? 3 : 4; }

#define BLD_XR_CASES(KERNEL)                                                                          \
    case 2: KERNEL<R, xr_ppt(2), 2><<<grid, thr, sm, h->stream>>>(a); break;                         \
    case 3: KERNEL<R, xr_ppt(3), 3><<<grid, thr, sm, h->stream>>>(a); break;                         \
    case 4: KERNEL<R, xr_ppt(4), 4><<<grid, thr, sm, h->stream>>>(a); break;                         \
    case 6: KERNEL<R, xr_ppt(6), 6><<<grid, thr, sm, h->stream>>>(a); break;                         \
    case 8: KERNEL<R, xr_ppt(8), 8><<<grid, thr, sm, h->stream>>>(a); break;                         \
    case 9: KERNEL<R, xr_ppt(9), 9><<<grid, thr, sm, h->stream>>>(a); break;                         \
    case 12: KERNEL<R, xr_ppt(12), 12><<<grid, thr, sm, h->stream>>>(a); break;                      \
    case 16: KERNEL<R, xr_ppt(16), 16><<<grid, thr, sm, h->stream>>>(a); break;                      \
    case 24: KERNEL<R, xr_ppt(24), 24><<<grid, thr, sm, h->stream>>>(a); break;

template <typename R>
int launch_adv_x(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    dim3 grid(s.P2 / s.YT, s.nchunks, nm);
    const int thr = s.YT * s.P1 / s.PPT;
    const size_t sm = smem_adv(s, sizeof(R) == 4);
    if (s.xr) {
        switch (s.xr) {
            BLD_XR_CASES(k_adv_x)
            default: return fail(BLD_ERR_INVALID_CONFIG, "no warp x transform of radix %d", s.xr);
        }
    } else {
        switch (s.PPT) {
            case 1: k_adv_x<R, 1, 0><<<grid, thr, sm, h->stream>>>(a); break;
            case 2: k_adv_x<R, 2, 0><<<grid, thr, sm, h->stream>>>(a); break;
            case 3: k_adv_x<R, 3, 0><<<grid, thr, sm, h->stream>>>(a); break;
            default: k_adv_x<R, 4, 0><<<grid, thr, sm, h->stream>>>(a); break;
        }
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// radix of the warp-per-row x kernel for P1 = 32 * radix, or 0 if no variant is compiled
template <typename R>
int warpx_radix(int P1) {
    if (P1 % 32) return 0;
    const int r = P1 / 32;
    if (sizeof(R) == 8) return (r == 2 || r == 3 || r == 4 || r == 6) ? r : 0;
    return (r == 2 || r == 3 || r == 4 || r == 6 || r == 8 || r == 9 || r == 12) ? r : 0;
}

// register caps compiled for the warp-per-row x kernel (single precision, radix >= 8)
template <typename R>
bool warpx_minb_ok(int r, int mb) {
    if (mb == 1) return true;
    return sizeof(R) == 4 && (r == 8 || r == 9 || r == 12) && (mb == 3 || mb == 4);
}

template <typename R>
int launch_adv_xw(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    const int r = warpx_radix<R>(s.P1);
    dim3 grid((s.P2 + s.xw - 1) / s.xw, s.nchunks, nm);
    const int thr = 32 * s.xw;
    const size_t sm = ((size_t)r * 32 + (size_t)s.xw * 12 * h->g.K1) * csize(sizeof(R) == 4);
    if constexpr (sizeof(R) == 4) {
        if (s.xwmb > 1) {
            if (!warpx_minb_ok<R>(r, s.xwmb)) return fail(BLD_ERR_INVALID_CONFIG, "no capped warp x kernel");
#define BLD_XW_MB(RR)                                                                   \
    case RR:                                                                            \
        if (s.xwmb == 3) k_adv_xwc<R, RR, 3><<<grid, thr, sm, h->stream>>>(a);          \
        else k_adv_xwc<R, RR, 4><<<grid, thr, sm, h->stream>>>(a);                      \
        break;
            switch (r) {
                BLD_XW_MB(8)
                BLD_XW_MB(9)
                BLD_XW_MB(12)
                default: return fail(BLD_ERR_INVALID_CONFIG, "no capped warp x kernel");
            }
#undef BLD_XW_MB
            CUDA_TRY(cudaGetLastError());
            return BLD_OK;
        }
    }
    switch (r) {
        case 2: k_adv_xw<R, 2><<<grid, thr, sm, h->stream>>>(a); break;
        case 3: k_adv_xw<R, 3><<<grid, thr, sm, h->stream>>>(a); break;
        case 4: k_adv_xw<R, 4><<<grid, thr, sm, h->stream>>>(a); break;
        case 6: k_adv_xw<R, 6><<<grid, thr, sm, h->stream>>>(a); break;
        default:
            if constexpr (sizeof(R) == 4) {
                switch (r) {
                    case 8: k_adv_xw<R, 8><<<grid, thr, sm, h->stream>>>(a); break;
                    case 9: k_adv_xw<R, 9><<<grid, thr, sm, h->stream>>>(a); break;
                    case 12: k_adv_xw<R, 12><<<grid, thr, sm, h->stream>>>(a); break;
                    default: return fail(BLD_ERR_INVALID_CONFIG, "no warp x kernel for P1=%d", s.P1);
                }
            } else {
                return fail(BLD_ERR_INVALID_CONFIG, "no warp x kernel for P1=%d", s.P1);
            }
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// radix of the block-of-warps x kernels for P1 = 32 * radix (16 and 24 in single
// precision only: one line of 24 FP64 complex values per lane would spill), or 0
int xb_radix(int P1, bool fp32) {
    if (P1 % 32) return 0;
    const int r = P1 / 32;
    if (fp32 && (r == 16 || r == 24)) return r;
    return (r == 2 || r == 3 || r == 4 || r == 6 || r == 8 || r == 9 || r == 12) ? r : 0;
}

template <typename R>
int launch_adv_xb(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    const int r = xb_radix(s.P1, sizeof(R) == 4);
    dim3 grid(s.P2, s.nchunks, nm);
    if (s.xb == 2) {
        const size_t smp = ((size_t)r * 32 + 5 * (size_t)(s.P1 + 32) + 12 * (size_t)h->g.K1) * csize(sizeof(R) == 4);
        switch (r) {
            case 2: k_adv_xp<R, 2><<<grid, 160, smp, h->stream>>>(a); break;
            case 3: k_adv_xp<R, 3><<<grid, 160, smp, h->stream>>>(a); break;
            case 4: k_adv_xp<R, 4><<<grid, 160, smp, h->stream>>>(a); break;
            case 6: k_adv_xp<R, 6><<<grid, 160, smp, h->stream>>>(a); break;
            case 8: k_adv_xp<R, 8><<<grid, 160, smp, h->stream>>>(a); break;
            case 9: k_adv_xp<R, 9><<<grid, 160, smp, h->stream>>>(a); break;
            case 12: k_adv_xp<R, 12><<<grid, 160, smp, h->stream>>>(a); break;
            default:
                if constexpr (sizeof(R) == 4) {
                    if (r == 16) { k_adv_xp<R, 16><<<grid, 160, smp, h->stream>>>(a); break; }
                    if (r == 24) { k_adv_xp<R, 24><<<grid, 160, smp, h->stream>>>(a); break; }
                }
                return fail(BLD_ERR_INVALID_CONFIG, "no pipelined block-of-warps x kernel for P1=%d", s.P1);
        }
        CUDA_TRY(cudaGetLastError());
        return BLD_OK;
    }
    const size_t sm = ((size_t)r * 32 + 3 * (size_t)(s.P1 + 32) + 12 * (size_t)h->g.K1) * csize(sizeof(R) == 4);
    switch (r) {
        case 2: k_adv_xb<R, 2><<<grid, 96, sm, h->stream>>>(a); break;
        case 3: k_adv_xb<R, 3><<<grid, 96, sm, h->stream>>>(a); break;
        case 4: k_adv_xb<R, 4><<<grid, 96, sm, h->stream>>>(a); break;
        case 6: k_adv_xb<R, 6><<<grid, 96, sm, h->stream>>>(a); break;
        case 8: k_adv_xb<R, 8><<<grid, 96, sm, h->stream>>>(a); break;
        case 9: k_adv_xb<R, 9><<<grid, 96, sm, h->stream>>>(a); break;
        case 12: k_adv_xb<R, 12><<<grid, 96, sm, h->stream>>>(a); break;
        default:
            if constexpr (sizeof(R) == 4) {
                if (r == 16) { k_adv_xb<R, 16><<<grid, 96, sm, h->stream>>>(a); break; }
                if (r == 24) { k_adv_xb<R, 24><<<grid, 96, sm, h->stream>>>(a); break; }
            }
            return fail(BLD_ERR_INVALID_CONFIG, "no block-of-warps x kernel for P1=%d", s.P1);
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// the register-capped two-pass SGS x kernels: single precision, P1 >= 256
// (where the uncapped kernel needs ~170 registers, one block per SM)
__host__ __device__ constexpr bool sx2_capped_size(int P) { return P >= 256; }

template <typename R, int P>
int launch_sgs_x2_p(bld_handle* h, const Space& s, const XArgs& a, dim3 grid, int thr, size_t sm) {
    if constexpr (sizeof(R) == 4 && sx2_capped_size(P)) {
        if (s.sx2 == 2 || s.sx2 == 4) {
            if (s.PPT == 1)
                k_sgs_x<R, 1, 0, P, 2><<<grid, thr, sm, h->stream>>>(a);
            else
                k_sgs_x<R, 2, 0, P, 2><<<grid, thr, sm, h->stream>>>(a);
            return BLD_OK;
        }
    }
    if (s.PPT == 1)
        k_sgs_x<R, 1, 0, P><<<grid, thr, sm, h->stream>>>(a);
    else
        k_sgs_x<R, 2, 0, P><<<grid, thr, sm, h->stream>>>(a);
    return BLD_OK;
}

// SGS x kernel with two-pass line transforms: compiled for the two-pass sizes and
// one or two points per thread of the products; v = 2: the register-capped form
bool sx2_ok(const bld_handle* h, const Space& s, int v = 1) {
    return y2_ok(s.P1, h->fp32) && (v % 2 == 1 || (h->fp32 && sx2_capped_size(s.P1)));
}

// k_sgs_x2: compiled for the two-pass sizes; whole row groups per block
// V = 1 (two rows per block) in single precision up to P1 = 384
bool sxk_ok(const bld_handle* h, const Space& s, int V = 0) {
    const int cs = (int)csize(h->fp32);
    return y2_ok(s.P1, h->fp32) && (V == 0 || (h->fp32 && s.P1 <= 384)) && s.P2 % sx2_rows(cs, s.P1, V) == 0 &&
           sx2_smem(y2_radix_a(s.P1), y2_radix_b(s.P1), h->g.K1, cs, V) <= 227 * 1024;
}

template <typename R, int P, int V>
void launch_sgs_xk_pv(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    constexpr int A = y2_radix_a(P), B = y2_radix_b(P);
    constexpr int NR = sx2_rows((int)sizeof(cplx<R>), P, V);
    dim3 grid(s.P2 / NR, s.nchunks, nm);
    const size_t sm = sx2_smem(A, B, h->g.K1, (int)sizeof(cplx<R>), V);
    k_sgs_x2<R, A, B, V><<<grid, sx2_threads(B, NR), sm, h->stream>>>(a);
}

template <typename R, int P>
int launch_sgs_xk_p(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    if constexpr (sizeof(R) == 4 && P <= 384) {
        if (s.sxk == 2) return launch_sgs_xk_pv<R, P, 1>(h, s, a, nm), BLD_OK;
    }
    launch_sgs_xk_pv<R, P, 0>(h, s, a, nm);
    return BLD_OK;
}

template <typename R>
int launch_sgs_xk(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    switch (s.P1) {
        case 64: BLD_TRY((launch_sgs_xk_p<R, 64>(h, s, a, nm))); break;
        case 96: BLD_TRY((launch_sgs_xk_p<R, 96>(h, s, a, nm))); break;
        case 128: BLD_TRY((launch_sgs_xk_p<R, 128>(h, s, a, nm))); break;
        case 144: BLD_TRY((launch_sgs_xk_p<R, 144>(h, s, a, nm))); break;
        case 192: BLD_TRY((launch_sgs_xk_p<R, 192>(h, s, a, nm))); break;
        case 256: BLD_TRY((launch_sgs_xk_p<R, 256>(h, s, a, nm))); break;
        case 288: BLD_TRY((launch_sgs_xk_p<R, 288>(h, s, a, nm))); break;
        default:
            if constexpr (sizeof(R) == 4) {
                if (s.P1 == 384) { BLD_TRY((launch_sgs_xk_p<R, 384>(h, s, a, nm))); break; }
                if (s.P1 == 512) { BLD_TRY((launch_sgs_xk_p<R, 512>(h, s, a, nm))); break; }
                if (s.P1 == 768) { BLD_TRY((launch_sgs_xk_p<R, 768>(h, s, a, nm))); break; }
            }
            return fail(BLD_ERR_INVALID_CONFIG, "no k_sgs_x2 kernel for P1=%d", s.P1);
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

template <typename R>
int launch_sgs_x(bld_handle* h, const Space& s, const XArgs& a, int nm) {
    if (s.sxk) return launch_sgs_xk<R>(h, s, a, nm);
    dim3 grid(s.P2 / s.YT, s.nchunks, nm);
    const int thr = s.YT * s.P1 / s.PPT;
    const size_t sm = smem_sgs(s, sizeof(R) == 4, h->g.K1);
    if (s.sx2) {
        switch (s.P1) {
            case 64: BLD_TRY((launch_sgs_x2_p<R, 64>(h, s, a, grid, thr, sm))); break;
            case 96: BLD_TRY((launch_sgs_x2_p<R, 96>(h, s, a, grid, thr, sm))); break;
            case 128: BLD_TRY((launch_sgs_x2_p<R, 128>(h, s, a, grid, thr, sm))); break;
            case 144: BLD_TRY((launch_sgs_x2_p<R, 144>(h, s, a, grid, thr, sm))); break;
            case 192: BLD_TRY((launch_sgs_x2_p<R, 192>(h, s, a, grid, thr, sm))); break;
            case 256: BLD_TRY((launch_sgs_x2_p<R, 256>(h, s, a, grid, thr, sm))); break;
            case 288: BLD_TRY((launch_sgs_x2_p<R, 288>(h, s, a, grid, thr, sm))); break;
            default:
                if constexpr (sizeof(R) == 4) {
                    if (s.P1 == 384) { BLD_TRY((launch_sgs_x2_p<R, 384>(h, s, a, grid, thr, sm))); break; }
                    if (s.P1 == 512) { BLD_TRY((launch_sgs_x2_p<R, 512>(h, s, a, grid, thr, sm))); break; }
                    if (s.P1 == 768) { BLD_TRY((launch_sgs_x2_p<R, 768>(h, s, a, grid, thr, sm))); break; }
                }
                return fail(BLD_ERR_INVALID_CONFIG, "no two-pass SGS x kernel for P1=%d", s.P1);
        }
        CUDA_TRY(cudaGetLastError());
        return BLD_OK;
    }
    if (s.xr) {
        switch (s.xr) {
            BLD_XR_CASES(k_sgs_x)
            default: return fail(BLD_ERR_INVALID_CONFIG, "no warp x transform of radix %d", s.xr);
        }
    } else {
        switch (s.PPT) {
            case 1: k_sgs_x<R, 1, 0><<<grid, thr, sm, h->stream>>>(a); break;
            case 2: k_sgs_x<R, 2, 0><<<grid, thr, sm, h->stream>>>(a); break;
            case 3: k_sgs_x<R, 3, 0><<<grid, thr, sm, h->stream>>>(a); break;
            default: k_sgs_x<R, 4, 0><<<grid, thr, sm, h->stream>>>(a); break;
        }
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

template <typename R>
int set_smem_limits_R() {
    const int lim = 227 * 1024;   // the largest dynamic shared memory a B200 block may opt into
    // large dynamic shared memory, and the largest shared-memory carveout so the
    // per-SM block count is set by the kernel's real footprint
#define BLD_SET(K)                                                                           \
    do {                                                                                     \
        CUDA_TRY(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)); \
        CUDA_TRY(cudaFuncSetAttribute(K, cudaFuncAttributePreferredSharedMemoryCarveout,     \
                                      cudaSharedmemCarveoutMaxShared));                      \
    } while (0)
    BLD_SET((k_inv_y<R, 0>));
    BLD_SET((k_fwd_y<R, 0>));
    BLD_SET((k_inv_y<R, 2>));
    BLD_SET((k_fwd_y<R, 2>));
    BLD_SET((k_inv_y<R, 3>));
    BLD_SET((k_fwd_y<R, 3>));
    BLD_SET((k_inv_y<R, 4>));
    BLD_SET((k_fwd_y<R, 4>));
    BLD_SET((k_inv_y<R, 6>));
    BLD_SET((k_fwd_y<R, 6>));
    BLD_SET((k_inv_y<R, 8>));
    BLD_SET((k_fwd_y<R, 8>));
    BLD_SET((k_inv_y<R, 9>));
    BLD_SET((k_fwd_y<R, 9>));
    BLD_SET((k_inv_y<R, 12>));
    BLD_SET((k_fwd_y<R, 12>));
    BLD_SET((k_inv_y<R, 16>));
    BLD_SET((k_fwd_y<R, 16>));
    if constexpr (sizeof(R) == 4) {
        BLD_SET((k_inv_y<R, 24>));
        BLD_SET((k_fwd_y<R, 24>));
    }
    BLD_SET((k_inv_y_all<R>));
    BLD_SET((k_fwd_y_all<R>));
#define BLD_SET_Y2(P)                                                                                  \
    BLD_SET((k_inv_y2<R, y2_radix_a(P), y2_radix_b(P), y2_min_blocks_inv<R>(y2_radix_b(P) * BLD_Y2_NL)>)); \
    BLD_SET((k_fwd_y2<R, y2_radix_a(P), y2_radix_b(P), y2_min_blocks<R>(y2_radix_b(P) * BLD_Y2_NL)>)); \
    BLD_SET((k_fwd_y2<R, y2_radix_a(P), y2_radix_b(P), 3, 8, 4>));                                                                   \
    BLD_SET((k_inv_y2<R, y2_radix_a(P), y2_radix_b(P), sizeof(R) == 8 ? 3 : 4, 8>));                                                \
    if constexpr (sizeof(R) == 4)                                                                    \
        BLD_SET((k_fwd_y2<R, y2_radix_a(P), y2_radix_b(P), y2_min_blocks<R>(y2_radix_b(P) * BLD_Y2_NL), BLD_Y2_NL, 2>));
    BLD_SET_Y2(64)
    BLD_SET_Y2(96)
    BLD_SET_Y2(128)
    BLD_SET_Y2(144)
    BLD_SET_Y2(192)
    BLD_SET_Y2(256)
    BLD_SET_Y2(288)
    if constexpr (sizeof(R) == 4) {
        BLD_SET_Y2(384)
        BLD_SET_Y2(512)
        BLD_SET_Y2(768)
    }
#undef BLD_SET_Y2
#define BLD_SET_Y3(P) BLD_SET((k_inv_y3<R, y2_radix_a(P), y2_radix_b(P)>));
    BLD_SET_Y3(64)
    BLD_SET_Y3(96)
    BLD_SET_Y3(128)
    BLD_SET_Y3(144)
    BLD_SET_Y3(192)
    BLD_SET_Y3(256)
    BLD_SET_Y3(288)
    if constexpr (sizeof(R) == 4) {
        BLD_SET_Y3(384)
        BLD_SET_Y3(512)
        BLD_SET_Y3(768)
    }
#undef BLD_SET_Y3
#define BLD_SET_X2(P)                                                   \
    BLD_SET((k_adv_x2<R, y2_radix_a(P), y2_radix_b(P), 0>));            \
    if constexpr (sizeof(R) == 8) {                                     \
        BLD_SET((k_adv_x2<R, y2_radix_a(P), y2_radix_b(P), 2>));        \
    }                                                                   \
    if constexpr (sizeof(R) == 4 && P <= 384) {                         \
        BLD_SET((k_adv_x2<R, y2_radix_a(P), y2_radix_b(P), 3>));        \
    }
    BLD_SET_X2(64)
    BLD_SET_X2(96)
    BLD_SET_X2(128)
    BLD_SET_X2(144)
    BLD_SET_X2(192)
    BLD_SET_X2(256)
    BLD_SET_X2(288)
    if constexpr (sizeof(R) == 4) {
        BLD_SET_X2(384)
        BLD_SET_X2(512)
        BLD_SET_X2(768)
    }
#undef BLD_SET_X2
#define BLD_SET_SX2(P) BLD_SET((k_sgs_x<R, 1, 0, P>)); BLD_SET((k_sgs_x<R, 2, 0, P>));   \
    if constexpr (P <= 288) BLD_SET((k_sgs_x2<R, y2_radix_a(P), y2_radix_b(P)>));          \
    if constexpr (sizeof(R) == 4 && P <= 384) BLD_SET((k_sgs_x2<R, y2_radix_a(P), y2_radix_b(P), 1>));
    BLD_SET_SX2(64)
    BLD_SET_SX2(96)
    BLD_SET_SX2(128)
    BLD_SET_SX2(144)
    BLD_SET_SX2(192)
    BLD_SET_SX2(256)
    BLD_SET_SX2(288)
    if constexpr (sizeof(R) == 4) {
        BLD_SET_SX2(384)
        BLD_SET_SX2(512)
        BLD_SET_SX2(768)
        BLD_SET((k_sgs_x2<R, y2_radix_a(384), y2_radix_b(384)>));
        BLD_SET((k_sgs_x2<R, y2_radix_a(512), y2_radix_b(512)>));
        BLD_SET((k_sgs_x2<R, y2_radix_a(768), y2_radix_b(768)>));
#define BLD_SET_SX2C(P) BLD_SET((k_sgs_x<R, 1, 0, P, 2>)); BLD_SET((k_sgs_x<R, 2, 0, P, 2>));
        BLD_SET_SX2C(256)
        BLD_SET_SX2C(288)
        BLD_SET_SX2C(384)
        BLD_SET_SX2C(512)
        BLD_SET_SX2C(768)
#undef BLD_SET_SX2C
    }
#undef BLD_SET_SX2
    BLD_SET((k_adv_x<R, 1, 0>));
    BLD_SET((k_adv_x<R, 2, 0>));
    BLD_SET((k_adv_x<R, 3, 0>));
    BLD_SET((k_adv_x<R, 4, 0>));
    BLD_SET((k_sgs_x<R, 1, 0>));
    BLD_SET((k_sgs_x<R, 2, 0>));
    BLD_SET((k_sgs_x<R, 3, 0>));
    BLD_SET((k_sgs_x<R, 4, 0>));
#define BLD_SET_XR(r)                              \
    BLD_SET((k_adv_x<R, xr_ppt(r), r>));           \
    BLD_SET((k_sgs_x<R, xr_ppt(r), r>));
    BLD_SET_XR(2)
    BLD_SET_XR(3)
    BLD_SET_XR(4)
    BLD_SET_XR(6)
    BLD_SET_XR(8)
    BLD_SET_XR(9)
    BLD_SET_XR(12)
    BLD_SET_XR(16)
    BLD_SET_XR(24)
#undef BLD_SET_XR
    BLD_SET((k_adv_xb<R, 2>));
    BLD_SET((k_adv_xb<R, 3>));
    BLD_SET((k_adv_xb<R, 4>));
    BLD_SET((k_adv_xb<R, 6>));
    BLD_SET((k_adv_xb<R, 8>));
    BLD_SET((k_adv_xb<R, 9>));
    BLD_SET((k_adv_xb<R, 12>));
    BLD_SET((k_adv_xp<R, 2>));
    BLD_SET((k_adv_xp<R, 3>));
    BLD_SET((k_adv_xp<R, 4>));
    BLD_SET((k_adv_xp<R, 6>));
    BLD_SET((k_adv_xp<R, 8>));
    BLD_SET((k_adv_xp<R, 9>));
    BLD_SET((k_adv_xp<R, 12>));
    if constexpr (sizeof(R) == 4) {
        BLD_SET((k_adv_xb<R, 16>));
        BLD_SET((k_adv_xb<R, 24>));
        BLD_SET((k_adv_xp<R, 16>));
        BLD_SET((k_adv_xp<R, 24>));
    }
    BLD_SET((k_adv_xw<R, 2>));
    BLD_SET((k_adv_xw<R, 3>));
    BLD_SET((k_adv_xw<R, 4>));
    BLD_SET((k_adv_xw<R, 6>));
    if constexpr (sizeof(R) == 4) {
        BLD_SET((k_adv_xw<R, 8>));
        BLD_SET((k_adv_xw<R, 9>));
        BLD_SET((k_adv_xw<R, 12>));
        BLD_SET((k_adv_xwc<R, 8, 3>));
        BLD_SET((k_adv_xwc<R, 9, 3>));
        BLD_SET((k_adv_xwc<R, 12, 3>));
        BLD_SET((k_adv_xwc<R, 8, 4>));
        BLD_SET((k_adv_xwc<R, 9, 4>));
        BLD_SET((k_adv_xwc<R, 12, 4>));
    }
#undef BLD_SET
    return BLD_OK;
}

// codelet twiddles W_N^m for N in {6,8,9,12,16,18,24,32}, once per device
int init_codelet_twiddles() {
    static std::mutex mu;
    static std::map<int, bool> done;
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return BLD_OK;
    const int sizes[] = {5, 6, 7, 8, 9, 10, 12, 14, 15, 16, 18, 24, 32};
    for (int N : sizes)
        for (int m = 0; m < N; ++m) {
            const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)N;
            h_wtab64[woff(N) + m] = make_double2((double)cosl(a), (double)sinl(a));
            h_wtab32[woff(N) + m] = make_float2((float)cosl(a), (float)sinl(a));
        }
    CUDA_TRY(cudaMemcpyToSymbol(c_wtab64, h_wtab64, sizeof(h_wtab64)));
    CUDA_TRY(cudaMemcpyToSymbol(c_wtab32, h_wtab32, sizeof(h_wtab32)));
    done[dev] = true;
    return BLD_OK;
}

int set_smem_limits() {
    BLD_TRY(init_codelet_twiddles());
    static int done = 0;
    if (done) return BLD_OK;
    BLD_TRY(set_smem_limits_R<double>());
    BLD_TRY(set_smem_limits_R<float>());
    CUDA_TRY(cudaFuncSetAttribute(k_x_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_seg<8, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    // dynamic shared memory of k_project_tile: at most 200 KB (project_tile_ok)
    CUDA_TRY(cudaFuncSetAttribute(k_project_tile<8, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_tile<8, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_tile<16, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_tile<16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_tile<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_tile<16, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    // k_project_pipe: at most 200 KB as well (project_pipe_ok)
    CUDA_TRY(cudaFuncSetAttribute(k_project_pipe<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_pipe<8, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_pipe<8, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_pipe<16, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_pipe<16, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_project_pipe<16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    done = 1;
    return BLD_OK;
}

// ------------------------------------------------------------------ schedules
template <typename R>
int enqueue_inv_y_R(bld_handle* h, int sp, const double2* state, int m0, int nm) {
    Space& s = sp == 0 ? h->adv : h->sgs;
    InvYArgs ia{};
    ia.g = h->g;
    ia.P2 = s.P2;
    ia.m0 = m0;
    ia.state = state;
    ia.mixed = s.min;
    ia.mixed_mstride = s.min_ms;
    ia.d1 = h->d1;
    ia.d2 = h->d2;
    ia.alpha_i = h->alpha_i;
    ia.active = h->mask_on ? h->active : nullptr;
    ia.plan = s.plan2;
    ia.tw = twp(h, s.P2, sizeof(R) == 4);
    if (sp == 0) {  // u, v, w, vort1, vort2, vort3 (src/processes/momentum_advection.jl:40-41)
        const int op[6] = {T_DIRECT, T_DIRECT, T_DIRECT, T_VORT1, T_VORT2, T_VORT3};
        const int fl[6] = {0, 1, 2, 0, 0, 0};
        const int isI[6] = {0, 0, 1, 1, 1, 0};
        ia.nterms = 6;
        for (int i = 0; i < 6; ++i) {
            ia.op[i] = op[i];
            ia.fld[i] = fl[i];
            ia.isI[i] = isI[i];
        }
    } else {  // u, v, w, u_1, u_2, v_1, v_2, w_1, w_2 (src/processes/static_smagorinsky.jl:39-42)
        const int op[9] = {T_DIRECT, T_DIRECT, T_DIRECT, T_D1, T_D2, T_D1, T_D2, T_D1, T_D2};
        const int fl[9] = {0, 1, 2, 0, 0, 1, 1, 2, 2};
        const int isI[9] = {0, 0, 1, 0, 0, 0, 0, 1, 1};
        ia.nterms = 9;
        for (int i = 0; i < 9; ++i) {
            ia.op[i] = op[i];
            ia.fld[i] = fl[i];
            ia.isI[i] = isI[i];
        }
    }
    return launch_inv_y<R>(h, s, ia, nm);
}

template <typename R>
int enqueue_x_R(bld_handle* h, int sp, int m0, int nm) {
    Space& s = sp == 0 ? h->adv : h->sgs;
    XArgs xa{};
    xa.g = h->g;
    xa.P1 = s.P1;
    xa.P2 = s.P2;
    xa.YT = s.YT;
    xa.zchunk = s.zchunk;
    xa.m0 = m0;
    xa.min = s.min;
    xa.mout = s.mout;
    xa.min_mstride = s.min_ms;
    xa.mout_mstride = s.mout_ms;
    xa.plan = s.plan1;
    xa.tw = twp(h, s.P1, sizeof(R) == 4);
    xa.alpha_c = h->alpha_c;
    xa.alpha_i = h->alpha_i;
    xa.lc = h->lc2;
    xa.li = h->li2;
    xa.wall = h->wall;
    xa.dyn_lo = h->dyn_lo;
    xa.dyn_hi = h->dyn_hi;
    xa.w_lo = h->w_lo;
    xa.w_hi = h->w_hi;
    xa.staged = sgs_staged(s, sizeof(R) == 4, h->g.K1) ? 1 : 0;
    xa.k1_magic = fdiv_magic((unsigned)h->g.K1);
    xa.p1_magic = fdiv_magic((unsigned)s.P1);
    xa.flag = h->flag;
    xa.active = h->mask_on ? h->active : nullptr;
    if (sp == 0) {
        if (s.x2) return launch_adv_x2<R>(h, s, xa, nm);
        if (s.xb) return launch_adv_xb<R>(h, s, xa, nm);
        return s.xw ? launch_adv_xw<R>(h, s, xa, nm) : launch_adv_x<R>(h, s, xa, nm);
    }
    return launch_sgs_x<R>(h, s, xa, nm);
}

// explicit stage update fused into the last forward y pass of a right-hand side:
// sout = (cu su + ct state + cd rate) / div
struct StageFuse {
    const double2* su;
    double2* sout;
    double cu, ct, cd, div;
};

template <typename R>
int enqueue_fwd_y_R(bld_handle* h, int sp, bool first, bool last, const double2* state, double2* du, int m0, int nm,
                    const StageFuse* sf = nullptr) {
    Space& s = sp == 0 ? h->adv : h->sgs;
    FwdYArgs fa{};
    fa.g = h->g;
    fa.P1 = s.P1;
    fa.P2 = s.P2;
    fa.mout = s.mout;
    fa.mout_mstride = s.mout_ms;
    if (sp == 0) {  // adv1 -> vel1, adv2 -> vel2, adv3 -> vel3
        for (int f = 0; f < 3; ++f) {
            fa.ncontrib[f] = 1;
            fa.c[f][0] = FwdContrib{f, 0};
        }
    } else {  // rate order of add_rates! (src/physical_space.jl:191-204)
        fa.ncontrib[0] = 3;
        fa.c[0][0] = FwdContrib{3, 0};
        fa.c[0][1] = FwdContrib{0, 1};
        fa.c[0][2] = FwdContrib{1, 2};
        fa.ncontrib[1] = 3;
        fa.c[1][0] = FwdContrib{4, 0};
        fa.c[1][1] = FwdContrib{1, 1};
        fa.c[1][2] = FwdContrib{2, 2};
        fa.ncontrib[2] = 3;
        fa.c[2][0] = FwdContrib{5, 0};
        fa.c[2][1] = FwdContrib{6, 1};
        fa.c[2][2] = FwdContrib{7, 2};
    }
    fa.mode = first ? 1 : 0;
    fa.check = last ? 1 : 0;
    fa.du = du;
    fa.du_mstride = h->g.mstride;
    fa.state = state;
    fa.lin = h->lin;
    fa.d1 = h->d1;
    fa.d2 = h->d2;
    fa.inv_n = 1.0 / ((double)s.P1 * (double)s.P2);
    fa.flag = h->flag;
    fa.fields = 3;
    fa.field0 = 0;
    fa.m0 = m0;
    fa.active = h->mask_on ? h->active : nullptr;
    fa.plan = s.plan2;
    fa.tw = twp(h, s.P2, sizeof(R) == 4);
    if (sf) {
        if (s.fwd.all) return fail(BLD_ERR_INVALID_CONFIG, "stage fusion needs the per-term forward y kernel");
        fa.fuse = 1;
        fa.su = sf->su;
        fa.sout = sf->sout;
        fa.st_cu = sf->cu;
        fa.st_ct = sf->ct;
        fa.st_cd = sf->cd;
        fa.st_inv = 1.0 / sf->div;
    }
    return launch_fwd_y<R>(h, s, fa, nm);
}

int enqueue_linear(bld_handle* h, const double2* state, double2* du, int m0, int nm) {
    FwdYArgs fa{};
    fa.g = h->g;
    fa.mode = 1;
    fa.check = 1;
    fa.du = du;
    fa.du_mstride = h->g.mstride;
    fa.state = state;
    fa.lin = h->lin;
    fa.flag = h->flag;
    fa.m0 = m0;
    fa.active = h->mask_on ? h->active : nullptr;
    dim3 grid((h->g.F + 255) / 256, h->g.n3, 3 * nm);
    k_linear<<<grid, 256, 0, h->stream>>>(fa);
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

int enqueue_inv_y(bld_handle* h, int sp, const double2* st, int m0, int nm) {
    return h->fp32 ? enqueue_inv_y_R<float>(h, sp, st, m0, nm) : enqueue_inv_y_R<double>(h, sp, st, m0, nm);
}
int enqueue_x(bld_handle* h, int sp, int m0, int nm) {
    return h->fp32 ? enqueue_x_R<float>(h, sp, m0, nm) : enqueue_x_R<double>(h, sp, m0, nm);
}
int enqueue_fwd_y(bld_handle* h, int sp, bool first, bool last, const double2* st, double2* du, int m0, int nm,
                  const StageFuse* sf = nullptr) {
    return h->fp32 ? enqueue_fwd_y_R<float>(h, sp, first, last, st, du, m0, nm, sf)
                   : enqueue_fwd_y_R<double>(h, sp, first, last, st, du, m0, nm, sf);
}

int enqueue_project(bld_handle* h, int kind, double dt, const double2* u, const double2* t, const double2* du,
                    const double2* dp, double2* out, int m0, int nm);

// ------------------------------------------------------------------ autotuner
// BLD_X_LINES=block keeps the block x kernels on block-wide Stockham stages
bool xdisable_wlines() {
    const char* e = getenv("BLD_X_LINES");
    return e && !strcmp(e, "block");
}

// BLD_Y_KERNEL=block keeps the y passes on block-wide Stockham stages
bool ydisable_warp() {
    const char* e = getenv("BLD_Y_KERNEL");
    return e && !strcmp(e, "block");
}
bool yforce_warp() {
    const char* e = getenv("BLD_Y_KERNEL");
    return e && !strcmp(e, "warp");
}
// BLD_Y_KERNEL=twopass keeps only the two-pass y kernels (where compiled);
// BLD_Y_KERNEL=tma the inverse pass with TMA-staged tiles (forward: two-pass)
bool yforce_twopass() {
    const char* e = getenv("BLD_Y_KERNEL");
    return e && !strcmp(e, "twopass");
}
bool yforce_tma() {
    const char* e = getenv("BLD_Y_KERNEL");
    return e && !strcmp(e, "tma");
}
// BLD_Y_KERNEL=twopass8: the two-pass kernels with the eight-line forward pass
bool yforce_twopass8() {
    const char* e = getenv("BLD_Y_KERNEL");
    return e && !strcmp(e, "twopass8");
}
// BLD_Y_KERNEL=twopass2: the two-pass kernels with two outputs of the forward
// epilogue in flight (single precision; double keeps one)
bool yforce_twopass2() {
    const char* e = getenv("BLD_Y_KERNEL");
    return e && !strcmp(e, "twopass2");
}

// y-pass candidates: per-term blocks (two-buffer FFT) with several line counts
// and block sizes, and all-terms blocks (in-place FFT); lines * element size of
// at least 32 bytes keeps global accesses sector-sized
std::vector<YCfg> y_candidates(const bld_handle* h, const Space& s, int lines_per_nl, int all_lines_per_nl,
                               bool inverse) {
    std::vector<YCfg> out;
    // inverse pass with TMA-staged tiles: one candidate per z-chunk count
    if (inverse && y3_ok(h, s.P2) && (getenv("BLD_Y_KERNEL") == nullptr || yforce_tma())) {
        const int n3 = h->g.n3;
        int last = -1;
        for (int zc : {1, 2, 3, 4, 6, 8, 12}) {
            const int zchunk = (n3 + zc - 1) / zc;
            if (zchunk == last || (zc > 1 && zchunk < 4)) continue;
            last = zchunk;
            YCfg c{};
            c.NL = BLD_Y3_NL;
            c.thr = y2_radix_b(s.P2) * BLD_Y3_NL;
            c.tp = 2;
            c.zc = zc;
            out.push_back(c);
        }
        if (yforce_tma()) return out;
    }
    const bool tp_ok = y2_ok(s.P2, h->fp32) && smem_y2(s.P2, lines_per_nl * BLD_Y2_NL, h->fp32) <= 200 * 1024;
    if (tp_ok && !yforce_warp() && getenv("BLD_Y_KERNEL") == nullptr) {
        YCfg c{};
        c.NL = BLD_Y2_NL;
        c.thr = y2_radix_b(s.P2) * BLD_Y2_NL;
        c.tp = 1;
        out.push_back(c);
        if (!inverse && h->fp32) {   // single precision: two outputs of the epilogue in flight
            c.tp = 4;
            out.push_back(c);
        }
        {   // eight lines, more blocks per SM
            c.NL = 8;
            c.thr = y2_radix_b(s.P2) * 8;
            c.tp = 3;
            out.push_back(c);
        }
    }
    if (tp_ok && (yforce_twopass() || yforce_twopass8() || yforce_twopass2() || (yforce_tma() && !inverse))) {
        YCfg c{};
        c.NL = BLD_Y2_NL;
        c.thr = y2_radix_b(s.P2) * BLD_Y2_NL;
        c.tp = (yforce_twopass2() && !inverse && h->fp32) ? 4 : 1;
        if (yforce_twopass8()) {
            c.NL = 8;
            c.thr = y2_radix_b(s.P2) * 8;
            c.tp = 3;
        }
        return {c};
    }
    const size_t cs = csize(h->fp32);
    const int nls_pt[4] = {h->fp32 ? 4 : 2, h->fp32 ? 8 : 4, h->fp32 ? 16 : 8, h->fp32 ? 32 : 16};
    for (int nl : nls_pt) {
        const int wr = s.P2 % 32 ? 0 : s.P2 / 32;
        if (wfft_radix_ok(wr, h->fp32) && !ydisable_warp() && smem_y_term(s.P2, lines_per_nl * nl, wr, h->fp32) <= 150 * 1024) {
            out.push_back(YCfg{0, nl, 128, wr});
            out.push_back(YCfg{0, nl, 256, wr});
        }
        if (nl == nls_pt[3] || (size_t)(s.P2 + 2 * s.P2 * lines_per_nl * nl) * cs > 150 * 1024) continue;
        int thrs[3] = {y_threads(s.plan2, lines_per_nl * nl), 128, 256};
        for (int i = 0; i < 3; ++i) {
            bool dup = false;
            for (int k = 0; k < i; ++k) dup |= thrs[k] == thrs[i];
            const bool warp_possible = wfft_radix_ok(s.P2 % 32 ? 0 : s.P2 / 32, h->fp32);
            if (!dup && !(yforce_warp() && warp_possible)) out.push_back(YCfg{0, nl, thrs[i], 0});
        }
    }
    const int nls_all[2] = {h->fp32 ? 2 : 1, h->fp32 ? 4 : 2};
    for (int nl : nls_all) {
        const int thr = inplace_threads(s.plan2, all_lines_per_nl * nl);
        if (thr && !yforce_warp() && (size_t)(s.P2 + s.P2 * all_lines_per_nl * nl) * cs <= 150 * 1024) out.push_back(YCfg{1, nl, thr, 0});
    }
    return out;
}

// average device time of `iters` launches of fn after one warm-up launch
template <typename F>
int time_launches(bld_handle* h, F&& fn, int iters, float* ms) {
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    int st = fn();
    if (st == BLD_OK && cudaEventRecord(e0, h->stream) != cudaSuccess) st = BLD_ERR_CUDA;
    for (int i = 0; i < iters && st == BLD_OK; ++i) st = fn();
    if (st == BLD_OK && cudaEventRecord(e1, h->stream) != cudaSuccess) st = BLD_ERR_CUDA;
    if (st == BLD_OK && cudaEventSynchronize(e1) != cudaSuccess) st = BLD_ERR_CUDA;
    float t = 0;
    if (st == BLD_OK) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / iters;
    return st == BLD_ERR_CUDA ? fail(BLD_ERR_CUDA, "autotune timing failed") : st;
}

bool stage_fusable(const bld_handle* h);

// Picks, per physical-domain space, the fastest y-pass variants and x-kernel
// tiling by timing every candidate on the handle's own buffers.  All candidates
// perform the same arithmetic, so the choice changes speed, not results.

// Autotuner choices of earlier handles of the same geometry, precision, process
// set and member count on the same device (process-wide), so that handles
// created again and again (the sub-pools of a server) are not re-timed.
struct TuneKey {
    int device, n1, n2, n3, members, fp32, adv_p1, adv_p2, sgs_p1, sgs_p2, pressure, env;
    bool operator<(const TuneKey& o) const {
        return std::tie(device, n1, n2, n3, members, fp32, adv_p1, adv_p2, sgs_p1, sgs_p2, pressure, env) <
               std::tie(o.device, o.n1, o.n2, o.n3, o.members, o.fp32, o.adv_p1, o.adv_p2, o.sgs_p1, o.sgs_p2,
                        o.pressure, o.env);
    }
};
struct TuneVal {
    Space adv, sgs;
    int proj_variant, proj_tile, proj_pipe;
};
std::mutex g_tune_mutex;
std::map<TuneKey, TuneVal> g_tune_cache;

TuneKey tune_key(const bld_handle* h) {
    // any kernel-family switch in the environment makes its own entry
    int env = 0;
    for (const char* v : {"BLD_X_KERNEL", "BLD_Y_KERNEL", "BLD_XW_MINB", "BLD_PROJ_VARIANT", "BLD_X_LINES",
                          "BLD_SGS_X_KERNEL", "BLD_X2_VARIANT", "BLD_PROJ_TILE", "BLD_PROJ_PIPE", "BLD_SGS_X2_VARIANT"}) {
        const char* e = getenv(v);
        env = env * 31 + (e ? (int)(std::hash<std::string>{}(e) % 1000003) + 1 : 0);
    }
    return TuneKey{h->device, h->cfg.n1, h->cfg.n2, h->g.n3, h->B, h->fp32 ? 1 : 0, h->adv.P1, h->adv.P2, h->sgs.P1,
                   h->sgs.P2, h->cfg.pressure, env};
}

// the tuned fields of a space (its buffers stay the handle's own)
void copy_tuning(Space& dst, const Space& src) {
    dst.YT = src.YT;
    dst.PPT = src.PPT;
    dst.xw = src.xw;
    dst.xwmb = src.xwmb;
    dst.zmult = src.zmult;
    dst.xb = src.xb;
    dst.xr = src.xr;
    dst.x2 = src.x2;
    dst.sx2 = src.sx2;
    dst.sxk = src.sxk;
    dst.inv = src.inv;
    dst.fwd = src.fwd;
}

int autotune_impl(bld_handle* h);

int autotune(bld_handle* h) {
    const char* env = getenv("BLD_NO_AUTOTUNE");
    const bool cached = !(env && env[0] && env[0] != '0');
    const TuneKey key = tune_key(h);
    if (cached) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            copy_tuning(h->adv, it->second.adv);
            copy_tuning(h->sgs, it->second.sgs);
            if (h->adv.on) x_chunks(h, h->adv);
            if (h->sgs.on) x_chunks(h, h->sgs);
            h->proj_variant = it->second.proj_variant;
            h->proj_tile = it->second.proj_tile;
            h->proj_pipe = it->second.proj_pipe;
            return BLD_OK;
        }
    }
    BLD_TRY(autotune_impl(h));
    if (cached) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        TuneVal v;
        copy_tuning(v.adv, h->adv);
        copy_tuning(v.sgs, h->sgs);
        v.proj_variant = h->proj_variant;
        v.proj_tile = h->proj_tile;
        v.proj_pipe = h->proj_pipe;
        g_tune_cache[key] = v;
    }
    return BLD_OK;
}

int autotune_impl(bld_handle* h) {
    // BLD_X_KERNEL=warp|block restricts the advection x kernel to one family
    const char* xk = getenv("BLD_X_KERNEL");
    const bool only_warp = xk && !strcmp(xk, "warp"), only_block = xk && !strcmp(xk, "block");
    const bool only_bw3 = xk && !strcmp(xk, "blockwarp"), only_pipe = xk && !strcmp(xk, "pipe");
    const bool only_bw = only_bw3 || only_pipe;   // a block-of-warps kernel (three warps, or five pipelined)
    const bool only_lines = xk && !strcmp(xk, "lines");   // block kernels with warp line transforms
    // the two-pass shared-memory x kernel (where it applies; elsewhere the other families)
    const bool only_x2 = xk && !strcmp(xk, "twopass") && h->adv.on && x2_ok(h, h->adv);
    const bool x2_asked = xk && !strcmp(xk, "twopass");
    // BLD_SGS_X_KERNEL=twopass keeps the SGS x pass on two-pass line transforms
    const char* sk = getenv("BLD_SGS_X_KERNEL");
    // (twopass_capped: only the register-capped two-pass kernels, where compiled)
    // (twopass_staged: only those with the input rows staged by bulk copies)
    const bool sx2_capped_only = sk && !strcmp(sk, "twopass_capped") && h->sgs.on && sx2_ok(h, h->sgs, 2);
    const bool sx2_staged_only = sk && !strcmp(sk, "twopass_staged") && h->sgs.on && sx2_ok(h, h->sgs);
    const bool only_sx2 = sk && (!strcmp(sk, "twopass") || sx2_capped_only || sx2_staged_only) && h->sgs.on &&
                          sx2_ok(h, h->sgs);
    const bool only_sxk = sk && !strcmp(sk, "rows") && h->sgs.on && sxk_ok(h, h->sgs);
    const bool adv_bw_ok = h->adv.on && xb_radix(h->adv.P1, h->fp32) > 0;
    if (only_bw && !adv_bw_ok && h->adv.on) return fail(BLD_ERR_INVALID_CONFIG, "no block-of-warps x kernel for P1=%d", h->adv.P1);
    const bool adv_warp_ok = h->adv.on && (h->fp32 ? warpx_radix<float>(h->adv.P1) : warpx_radix<double>(h->adv.P1)) > 0;
    if (only_warp && !adv_warp_ok && h->adv.on) return fail(BLD_ERR_INVALID_CONFIG, "no warp x kernel for P1=%d", h->adv.P1);
    const char* env = getenv("BLD_NO_AUTOTUNE");
    if (env && env[0] && env[0] != '0') {
        if (only_warp && adv_warp_ok) {
            h->adv.xw = 4;
            x_chunks(h, h->adv);
        }
        if (only_bw && adv_bw_ok) {
            h->adv.xb = only_pipe ? 2 : 1;
            x_chunks(h, h->adv);
        }
        return BLD_OK;
    }
    const int B = h->B;
    for (int sp = 0; sp < 2; ++sp) {
        Space& s = sp == 0 ? h->adv : h->sgs;
        if (!s.on) continue;
        float best = 1e30f, t = 0;
        YCfg bi = s.inv;
        for (const YCfg& c : y_candidates(h, s, 1, s.ntin, true)) {
            s.inv = c;
            BLD_TRY(time_launches(h, [&] { return enqueue_inv_y(h, sp, h->u, 0, B); }, 3, &t));
            if (t < best) {
                best = t;
                bi = c;
            }
        }
        s.inv = bi;
        BLD_TRY(enqueue_inv_y(h, sp, h->u, 0, B));
        best = 1e30f;
        int byt = s.YT, bppt = s.PPT;
        for (auto c : x_candidates(h, s, sp == 0)) {
            if ((sp == 0 && (only_warp || only_bw)) || only_lines) break;
            s.YT = c.first;
            s.PPT = c.second;
            x_chunks(h, s);
            BLD_TRY(time_launches(h, [&] { return enqueue_x(h, sp, 0, B); }, 3, &t));
            if (t < best) {
                best = t;
                byt = c.first;
                bppt = c.second;
            }
        }
        // block x kernels with warp line transforms (YT = 1, 2)
        int bxr = 0;
        const int xrr = s.P1 % 32 ? 0 : s.P1 / 32;
        if (xr_radix_ok(xrr) && !(sp == 0 && (only_warp || only_bw)) && !only_block && !xdisable_wlines()) {
            for (int yt = 1; yt <= 2; ++yt) {
                const size_t smx = (size_t)(s.P1 + 2 * (sp == 0 ? 3 : 5) * yt * (s.P1 + 32)) * csize(h->fp32);
                if (s.P2 % yt || smx > 150 * 1024 || yt * s.P1 / xr_ppt(xrr) > 256) continue;
                s.xr = xrr;
                s.YT = yt;
                s.PPT = xr_ppt(xrr);
                x_chunks(h, s);
                BLD_TRY(time_launches(h, [&] { return enqueue_x(h, sp, 0, B); }, 3, &t));
                if (t < best) {
                    best = t;
                    bxr = xrr;
                    byt = yt;
                    bppt = xr_ppt(xrr);
                }
            }
            s.xr = 0;
        }
        // SGS: the block kernel with two-pass line transforms
        int bsx2 = 0;
        if (sp == 1 && sx2_ok(h, s) && !only_block && !only_lines) {
            float best2 = 1e30f;
            int yt2 = 1, ppt2 = 1, v2 = 1;
            for (int v = 1; v <= 4; ++v)
                for (int yt = 1; yt <= 4; yt *= 2)
                    for (int ppt = 1; ppt <= 2; ++ppt) {
                        const int thr = yt * s.P1 / ppt;
                        if (!sx2_ok(h, s, v) || s.P2 % yt || thr > 256 || thr < 32 || thr % 32) continue;
                        if ((sx2_capped_only && v % 2 == 1) || (sx2_staged_only && v < 3)) continue;
                        s.YT = yt;
                        if (v >= 3 && !sgs_stage_fits(s, h->fp32, h->g.K1)) continue;
                        s.sx2 = v;
                        s.xr = 0;
                        s.YT = yt;
                        s.PPT = ppt;
                        if (smem_sgs(s, h->fp32, h->g.K1) > 200 * 1024) continue;
                        x_chunks(h, s);
                        BLD_TRY(time_launches(h, [&] { return enqueue_x(h, sp, 0, B); }, 3, &t));
                        if (t < best2) {
                            best2 = t;
                            yt2 = yt;
                            ppt2 = ppt;
                            v2 = v;
                        }
                    }
            s.sx2 = 0;
            if (best2 < 1e30f && (best2 < best || only_sx2)) {
                best = best2;
                bsx2 = v2;
                bxr = 0;
                byt = yt2;
                bppt = ppt2;
            }
        }
        // finalists: the best block kernel above, the warp-per-row kernel with
        // 1, 2, 4 warps per block and the block-of-warps kernels, each timed at
        // its best z-chunk count (and, for the warp-per-row kernel, register
        // cap: more resident warps want more chunks)
        struct XPick {
            int YT, PPT, xr, xw, xwmb, xb, zmult, x2, sx2, sxk;
        };
        auto get_pick = [&]() { return XPick{s.YT, s.PPT, s.xr, s.xw, s.xwmb, s.xb, s.zmult, s.x2, s.sx2, s.sxk}; };
        auto set_pick = [&](const XPick& p) {
            s.YT = p.YT;
            s.PPT = p.PPT;
            s.xr = p.xr;
            s.xw = p.xw;
            s.xwmb = p.xwmb;
            s.xb = p.xb;
            s.zmult = p.zmult;
            s.x2 = p.x2;
            s.sx2 = p.sx2;
            s.sxk = p.sxk;
            x_chunks(h, s);
        };
        const char* mbe = getenv("BLD_XW_MINB");   // force one register cap (1, 3, 4)
        const int mb_only = mbe && mbe[0] ? atoi(mbe) : 0;
        float bx = 1e30f;
        XPick bp{};
        auto tune_chunks = [&](XPick base) -> int {
            const int r = h->fp32 ? warpx_radix<float>(s.P1) : warpx_radix<double>(s.P1);
            for (int mb : {1, 3, 4}) {
                if (mb > 1 && !(base.xw && (h->fp32 ? warpx_minb_ok<float>(r, mb) : warpx_minb_ok<double>(r, mb))))
                    continue;
                if (mb_only && base.xw && mb != mb_only) continue;
                int last_chunks = -1;
                for (int mult : {2, 3, 4, 6, 8, 12, 16}) {
                    XPick p = base;
                    p.xwmb = mb;
                    p.zmult = mult;
                    set_pick(p);
                    if (s.nchunks == last_chunks) continue;
                    last_chunks = s.nchunks;
                    BLD_TRY(time_launches(h, [&] { return enqueue_x(h, sp, 0, B); }, 3, &t));
                    if (t < bx) {
                        bx = t;
                        bp = p;
                    }
                }
            }
            return BLD_OK;
        };
        const bool block_ok = best < 1e30f;   // a block kernel was timed above
        if (block_ok && (sp == 1 || !only_x2) && !(sp == 1 && only_sxk))
            BLD_TRY(tune_chunks(XPick{byt, bppt, bxr, 0, 1, 0, 2, 0, bsx2, 0}));
        // the SGS kernel with staged rows and two-pass lines (BLD_SGS_X_KERNEL=rows keeps it)
        // (BLD_SGS_X2_VARIANT = 0, 1 keeps one of its variants)
        const char* sxv = getenv("BLD_SGS_X2_VARIANT");
        const int sxv_only = sxv && sxv[0] ? atoi(sxv) : -1;
        for (int v = 0; v <= 1; ++v)
            if (sp == 1 && sxk_ok(h, s, v) && (!sk || only_sxk) && (sxv_only < 0 || sxv_only == v))
                BLD_TRY(tune_chunks(XPick{1, 1, 0, 0, 1, 0, 2, 0, 0, 1 + v}));
        const bool warp_ok = sp == 0 && adv_warp_ok && !only_block && !only_bw && !only_lines && !only_x2;
        for (int wpb = 1; warp_ok && wpb <= 4; wpb *= 2) BLD_TRY(tune_chunks(XPick{1, 1, 0, wpb, 1, 0, 2, 0, 0, 0}));
        for (int xbk = 1; xbk <= 2; ++xbk) {
            if (!(sp == 0 && adv_bw_ok && !only_block && !only_warp && !only_lines && !only_x2)) break;
            if ((xbk == 1 && only_pipe) || (xbk == 2 && only_bw3)) continue;
            BLD_TRY(tune_chunks(XPick{1, 1, 0, 0, 1, xbk, 2, 0, 0, 0}));
        }
        // the two-pass kernel's variants (BLD_X2_VARIANT = 0, 2, 3 forces one)
        const char* x2v = getenv("BLD_X2_VARIANT");
        const int x2_only = x2v && x2v[0] ? atoi(x2v) : -1;
        for (int v = 0; v <= 3; ++v)
            if (sp == 0 && x2_ok(h, s, v) && (only_x2 || !xk || x2_asked) && (x2_only < 0 || x2_only == v))
                BLD_TRY(tune_chunks(XPick{1, 1, 0, 0, 1, 0, 2, 1 + v, 0, 0}));
        if (bx >= 1e30f) return fail(BLD_ERR_INVALID_CONFIG, "no x kernel could be timed");
        set_pick(bp);
        x_chunks(h, s);
        best = 1e30f;
        YCfg bf = s.fwd;
        for (const YCfg& c : y_candidates(h, s, s.fsets, 3 * s.fsets, false)) {
            s.fwd = c;
            BLD_TRY(time_launches(h, [&] { return enqueue_fwd_y(h, sp, true, false, h->u, h->io2, 0, B); }, 3, &t));
            if (t < best) {
                best = t;
                bf = c;
            }
        }
        s.fwd = bf;
        const char* v = getenv("BLD_VERBOSE");
        if (v && v[0] && v[0] != '0')
            fprintf(stderr, "bld autotune %s P=%dx%d: inv all=%d NL=%d thr=%d wfft=%d tp=%d | x YT=%d PPT=%d xr=%d warps=%d bw=%d x2=%d sx2=%d sxk=%d chunks=%d | fwd all=%d NL=%d thr=%d wfft=%d tp=%d\n",
                    sp == 0 ? "advection" : "sgs", s.P1, s.P2, s.inv.all, s.inv.NL, s.inv.thr, s.inv.wfft, s.inv.tp, s.YT, s.PPT, s.xr, s.xw, (int)s.xb,
                    s.x2, s.sx2, s.sxk, s.nchunks, s.fwd.all, s.fwd.NL, s.fwd.thr, s.fwd.wfft, s.fwd.tp);
    }
    if (h->cfg.pressure && h->g.n3 <= 256) {
        float best = 1e30f, t = 0;
        int bv = h->proj_variant;
        // BLD_PROJ_VARIANT=0..3 keeps one variant (tests check each against the oracle)
        const char* pv = getenv("BLD_PROJ_VARIANT");
        const int only_v = (pv && pv[0] >= '0' && pv[0] <= '3') ? pv[0] - '0' : -1;
        for (int v = 0; v < 4; ++v) {
            if (v == 3 && h->g.n3 > 128) break;   // the tile variant holds n3 <= 128 layers
            if (only_v >= 0 && v != only_v) continue;
            h->proj_variant = v;
            // timed as the projections of one SSP-RK33 step: with the stage update
            // fused into the forward y pass, one Euler stage and two plain
            // projections in place; otherwise an Euler stage and two middle stages
            // (three inputs)
            const bool fz = stage_fusable(h);
            BLD_TRY(time_launches(h, [&] {
                BLD_TRY(enqueue_project(h, S_EULER, 1e-4, h->u, nullptr, h->du, nullptr, h->io, 0, B));
                for (int k = 0; k < 2; ++k) {
                    if (fz) BLD_TRY(enqueue_project(h, S_NONE, 1e-4, h->io, nullptr, nullptr, nullptr, h->io, 0, B));
                    else BLD_TRY(enqueue_project(h, S_RK33_2, 1e-4, h->u, h->t, h->du, nullptr, h->io, 0, B));
                }
                return (int)BLD_OK;
            }, 3, &t));
            if (t < best) {
                best = t;
                bv = v;
            }
        }
        h->proj_variant = bv;
        // projections of stored stage values (the step's in-place projections):
        // the chosen kernel against k_project_tile with 8 or 16 columns per block
        // (BLD_PROJ_TILE = 0, 4, 8, 16 keeps one), each also in its persistent
        // two-stage form (BLD_PROJ_PIPE = 0 or 1 keeps one form)
        const char* pt = getenv("BLD_PROJ_TILE");
        const int only_t = (pt && pt[0]) ? atoi(pt) : -1;
        const char* pp = getenv("BLD_PROJ_PIPE");
        const int only_p = (pp && pp[0]) ? atoi(pp) : -1;
        float bt = 1e30f;
        int btile = 0, bpipe = 0;
        for (int ln : {0, 4, 8, 16})
            for (int pipe = 0; pipe < 2; ++pipe) {
                if (ln && !project_tile_ok(h, ln)) continue;
                if (pipe && (!ln || !project_pipe_ok(h, ln))) continue;
                if (only_t >= 0 && ln != only_t) continue;
                // a forced persistent form that does not fit keeps the plain one
                if (ln && only_p >= 0 && pipe != only_p && !(only_p == 1 && !project_pipe_ok(h, ln))) continue;
                h->proj_tile = ln;
                h->proj_pipe = pipe;
                BLD_TRY(time_launches(h, [&] {
                    for (int k = 0; k < 3; ++k)
                        BLD_TRY(enqueue_project(h, S_NONE, 1e-4, h->io, nullptr, nullptr, nullptr, h->io, 0, B));
                    return (int)BLD_OK;
                }, 3, &t));
                if (t < bt) {
                    bt = t;
                    btile = ln;
                    bpipe = pipe;
                }
            }
        h->proj_tile = btile;
        h->proj_pipe = bpipe;
        const char* v = getenv("BLD_VERBOSE");
        if (v && v[0] && v[0] != '0') fprintf(stderr, "bld autotune projection: variant %d, tile %d, persistent %d\n", bv, btile, bpipe);
    }
    CUDA_TRY(cudaMemsetAsync(h->flag, 0, h->B * sizeof(int), h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

// compute_rates! (src/Processes.jl:39-62): nonlinear processes in the reference's
// process order (advection, then SGS), each rate written once with the linear terms
int enqueue_rates_impl(bld_handle* h, const double2* state, double2* du, int m0, int nm,
                       const StageFuse* sf = nullptr) {
    for (int sp = 0; sp < 2; ++sp) {
        if (!(sp == 0 ? h->adv.on : h->sgs.on)) continue;
        BLD_TRY(enqueue_inv_y(h, sp, state, m0, nm));
        BLD_TRY(enqueue_x(h, sp, m0, nm));
    }
    bool first = true;
    for (int sp = 0; sp < 2; ++sp) {
        if (!(sp == 0 ? h->adv.on : h->sgs.on)) continue;
        const bool last = (sp == 1) || !h->sgs.on;
        BLD_TRY(enqueue_fwd_y(h, sp, first, last, state, du, m0, nm, last ? sf : nullptr));
        first = false;
    }
    if (first) {
        if (sf) return fail(BLD_ERR_INVALID_CONFIG, "stage fusion needs a forward y pass");
        BLD_TRY(enqueue_linear(h, state, du, m0, nm));
    }
    return BLD_OK;
}

// The stage update can ride on the last forward y pass when that pass is the
// per-term kernel (BLD_NO_STAGE_FUSION=1 keeps the update in the projection).
bool stage_fusable(const bld_handle* h) {
    const char* e = getenv("BLD_NO_STAGE_FUSION");
    if (e && e[0] && e[0] != '0') return false;
    if (!h->adv.on && !h->sgs.on) return false;
    const Space& last = h->sgs.on ? h->sgs : h->adv;
    return !last.fwd.all;
}

// steps of one call may be chained (BLD_NO_STEP_CHAIN=1 keeps every step whole)
bool chain_ok(const bld_handle* h, int method) {
    if (method != BLD_SSPRK33 && method != BLD_SSPRK22) return false;
    const char* e = getenv("BLD_NO_STEP_CHAIN");
    if (e && e[0] && e[0] != '0') return false;
    return stage_fusable(h);
}

int enqueue_rates(bld_handle* h, const double2* state, double2* du, int m0, int nm) {
    return enqueue_rates_impl(h, state, du, m0, nm);
}

int enqueue_project(bld_handle* h, int kind, double dt, const double2* u, const double2* t, const double2* du,
                    const double2* dp, double2* out, int m0, int nm) {
    ProjArgs a{};
    a.g = h->g;
    a.m0 = m0;
    a.active = h->mask_on ? h->active : nullptr;
    a.u = u;
    a.t = t;
    a.du = du;
    a.dp = dp;
    a.out = out;
    a.kind = kind;
    a.dt = dt;
    a.pressure = h->cfg.pressure;
    a.pscr = h->pscr;
    a.gamma = h->gamma;
    a.alpha_c = h->alpha_c;
    a.inv_alpha_c = h->inv_alpha_c;
    a.alpha_i = h->alpha_i;
    a.d1 = h->d1;
    a.d2 = h->d2;
    a.w_lo = h->w_lo;
    a.w_hi = h->w_hi;
    for (int f = 0; f < 3; ++f) a.mean_on[f] = h->cfg.mean[f];
    a.mean_w = h->mean_w;
    a.mean_val = h->mean_val;
    const bool any_mean = h->cfg.mean[0] || h->cfg.mean[1];
    if (!a.pressure && !any_mean && kind == S_NONE && out == u) return BLD_OK;
    const int n3 = h->g.n3;
    if (kind == S_NONE && h->proj_tile && project_tile_ok(h, h->proj_tile)) {
        const int ln = h->proj_tile, lmax = n3 <= 128 ? 8 : 16;
        CUtensorMap umap, gmap;
        BLD_TRY(project_tmaps(h, u, ln, &umap, &gmap));
        dim3 grid((unsigned)((h->g.F + ln - 1) / ln), nm);
        dim3 block(ln, std::max(1, std::min(16, (n3 + lmax - 1) / lmax)));
        if (h->proj_pipe && project_pipe_ok(h, ln)) {
            if (lmax == 8 && ln == 4) return launch_project_pipe<8, 4>(h, a, nm, umap, gmap);
            if (lmax == 8 && ln == 8) return launch_project_pipe<8, 8>(h, a, nm, umap, gmap);
            if (lmax == 8) return launch_project_pipe<8, 16>(h, a, nm, umap, gmap);
            if (ln == 4) return launch_project_pipe<16, 4>(h, a, nm, umap, gmap);
            if (ln == 8) return launch_project_pipe<16, 8>(h, a, nm, umap, gmap);
            return launch_project_pipe<16, 16>(h, a, nm, umap, gmap);
        }
        const size_t sm = project_tile_smem(n3, ln);
        if (lmax == 8 && ln == 4) k_project_tile<8, 4><<<grid, block, sm, h->stream>>>(a, umap, gmap, h->flag);
        else if (lmax == 8 && ln == 8) k_project_tile<8, 8><<<grid, block, sm, h->stream>>>(a, umap, gmap, h->flag);
        else if (lmax == 8) k_project_tile<8, 16><<<grid, block, sm, h->stream>>>(a, umap, gmap, h->flag);
        else if (ln == 4) k_project_tile<16, 4><<<grid, block, sm, h->stream>>>(a, umap, gmap, h->flag);
        else if (ln == 8) k_project_tile<16, 8><<<grid, block, sm, h->stream>>>(a, umap, gmap, h->flag);
        else k_project_tile<16, 16><<<grid, block, sm, h->stream>>>(a, umap, gmap, h->flag);
        CUDA_TRY(cudaGetLastError());
        return BLD_OK;
    }
    if (a.pressure && n3 <= 256 && h->proj_variant > 0) {
        // z-segmented solve: <= 16 segments of <= 8 (n3 <= 128) or <= 16 layers;
        // 16 modes side by side (256-byte rows), <= 256 threads; variant 1 lets the
        // compiler use all registers it wants, variant 2 caps them for 2 blocks per SM
        const int lmax = n3 <= 128 ? 8 : 16;
        const int ns = std::max(1, std::min(16, (n3 + lmax - 1) / lmax));
        dim3 grid((h->g.F + 15) / 16, nm);
        dim3 block(16, ns);
        const size_t tsm = (size_t)3 * n3 * 16 * sizeof(double2);   // variant 3: stage values in shared memory
        if (lmax == 8 && h->proj_variant == 3)
            k_project_seg<8, 1, true><<<grid, block, tsm, h->stream>>>(a);
        else if (lmax == 8 && h->proj_variant == 1)
            k_project_seg<8, 1, false><<<grid, block, 0, h->stream>>>(a);
        else if (lmax == 8)
            k_project_seg<8, 2, false><<<grid, block, 0, h->stream>>>(a);
        else if (h->proj_variant == 1)
            k_project_seg<16, 1, false><<<grid, block, 0, h->stream>>>(a);
        else
            k_project_seg<16, 2, false><<<grid, block, 0, h->stream>>>(a);
    } else {
        dim3 grid((h->g.F + 127) / 128, nm);
        k_project<<<grid, 128, 0, h->stream>>>(a);
    }
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// one time step of `method` (perform_step! + the trailing rate!, src/ODEMethods.jl:217-234)
// chain (SSPRK22 / SSPRK33 with the stage update fused, steps inside one
// multi-step call): CHAIN_ENTER = the step starts from t = u + dt f(u) formed by
// the previous step's trailing forward pass, so its first stage is a plain
// projection of t in place; CHAIN_LEAVE = the trailing right-hand side writes
// t = u + dt f(u) for the next step instead of f(u).  The last step of a call
// never leaves, so du holds f(u) between calls.
enum { CHAIN_ENTER = 1, CHAIN_LEAVE = 2 };

// the right-hand side of the new state at the end of a step: f(u) into du, or
// (CHAIN_LEAVE) the next step's first stage value u + dt f(u) into t
int enqueue_trailing_rates(bld_handle* h, double dt, int chain) {
    if (chain & CHAIN_LEAVE) {
        const StageFuse sf{nullptr, h->t, 0.0, 1.0, dt, 1.0};
        return enqueue_rates_impl(h, h->u, h->du, 0, h->B, &sf);
    }
    return enqueue_rates(h, h->u, h->du, 0, h->B);
}

int enqueue_step(bld_handle* h, int method, double dt, bool ab2_first, int chain = 0) {
    const int B = h->B;
    struct MaskScope {
        bld_handle* h;
        ~MaskScope() { h->mask_on = false; }
    } scope{h};
    h->mask_on = true;
    switch (method) {
        case BLD_EULER:
            BLD_TRY(enqueue_project(h, S_EULER, dt, h->u, nullptr, h->du, nullptr, h->u, 0, B));
            BLD_TRY(enqueue_rates(h, h->u, h->du, 0, B));
            break;
        case BLD_SSPRK22:
            if (chain & CHAIN_ENTER)
                BLD_TRY(enqueue_project(h, S_NONE, dt, h->t, nullptr, nullptr, nullptr, h->t, 0, B));
            else
                BLD_TRY(enqueue_project(h, S_EULER, dt, h->u, nullptr, h->du, nullptr, h->t, 0, B));
            if (stage_fusable(h)) {
                // u <- (u + t + dt f(t)) / 2 in the forward y pass (u is read and
                // written element by element; the pass reads t), then project u
                const StageFuse sf{h->u, h->u, 1.0, 1.0, dt, 2.0};
                BLD_TRY(enqueue_rates_impl(h, h->t, h->du, 0, B, &sf));
                BLD_TRY(enqueue_project(h, S_NONE, dt, h->u, nullptr, nullptr, nullptr, h->u, 0, B));
            } else {
                BLD_TRY(enqueue_rates(h, h->t, h->du, 0, B));
                BLD_TRY(enqueue_project(h, S_RK22_2, dt, h->u, h->t, h->du, nullptr, h->u, 0, B));
            }
            BLD_TRY(enqueue_trailing_rates(h, dt, chain));
            break;
        case BLD_SSPRK33:
            if (chain & CHAIN_ENTER)
                BLD_TRY(enqueue_project(h, S_NONE, dt, h->t, nullptr, nullptr, nullptr, h->t, 0, B));
            else
                BLD_TRY(enqueue_project(h, S_EULER, dt, h->u, nullptr, h->du, nullptr, h->t, 0, B));
            if (stage_fusable(h)) {
                // second stage into du (free once the first stage consumed it; the
                // pass reads t, so the stage value cannot overwrite t in place)
                const StageFuse s2{h->u, h->du, 3.0, 1.0, dt, 4.0};
                BLD_TRY(enqueue_rates_impl(h, h->t, h->du, 0, B, &s2));
                BLD_TRY(enqueue_project(h, S_NONE, dt, h->du, nullptr, nullptr, nullptr, h->du, 0, B));
                // third stage into u from the second-stage state held in du; the
                // partial rates of a first forward pass (when two physical-domain
                // spaces contribute) go to t, which the first stage left free
                const StageFuse s3{h->u, h->u, 1.0, 2.0, 2.0 * dt, 3.0};
                BLD_TRY(enqueue_rates_impl(h, h->du, h->t, 0, B, &s3));
                BLD_TRY(enqueue_project(h, S_NONE, dt, h->u, nullptr, nullptr, nullptr, h->u, 0, B));
            } else {
                BLD_TRY(enqueue_rates(h, h->t, h->du, 0, B));
                BLD_TRY(enqueue_project(h, S_RK33_2, dt, h->u, h->t, h->du, nullptr, h->t, 0, B));
                BLD_TRY(enqueue_rates(h, h->t, h->du, 0, B));
                BLD_TRY(enqueue_project(h, S_RK33_3, dt, h->u, h->t, h->du, nullptr, h->u, 0, B));
            }
            BLD_TRY(enqueue_trailing_rates(h, dt, chain));
            break;
        case BLD_AB2: {
            const size_t bytes = (size_t)B * h->g.mstride * sizeof(double2);
            if (ab2_first) {
                BLD_TRY(enqueue_project(h, S_EULER, dt, h->u, nullptr, h->du, nullptr, h->u, 0, B));
                CUDA_TRY(cudaMemcpyAsync(h->dp, h->du, bytes, cudaMemcpyDeviceToDevice, h->stream));
                BLD_TRY(enqueue_rates(h, h->u, h->du, 0, B));
                BLD_TRY(enqueue_project(h, S_AB2_1, dt, h->u, nullptr, h->du, h->dp, h->u, 0, B));
            } else {
                BLD_TRY(enqueue_project(h, S_AB2, dt, h->u, nullptr, h->du, h->dp, h->u, 0, B));
                CUDA_TRY(cudaMemcpyAsync(h->dp, h->du, bytes, cudaMemcpyDeviceToDevice, h->stream));
            }
            BLD_TRY(enqueue_rates(h, h->u, h->du, 0, B));
            break;
        }
        default:
            return fail(BLD_ERR_ARGUMENT, "unknown method %d", method);
    }
    return BLD_OK;
}

// segmented batched LDL^T solve: LMAX layers per thread, NS = ceil(n / LMAX)
// segments, LANES systems per block with LANES * NS <= 512
template <typename T>
int ldlt_launch(const double* gamma, const double* beta, T* rhs, long long nsys, int n, cudaStream_t st) {
    if (n > 1024) return fail(BLD_ERR_ARGUMENT, "tridiagonal systems longer than 1024 are not supported");
    // layers per thread and systems per block (BLD_LDLT_LMAX = 4|8|16, BLD_LDLT_LANES override them).
    // 16 layers and 16 systems per thread row measured best at n = 256 (5.5 TB/s complex,
    // against 3.5 TB/s with 8 layers x 16 systems): more loads in flight per thread
    int lmax = 16;
    const char* el = getenv("BLD_LDLT_LMAX");
    if (el && (atoi(el) == 4 || atoi(el) == 8 || atoi(el) == 16) && (n + atoi(el) - 1) / atoi(el) <= 512)
        lmax = atoi(el);
    const int NS = (n + lmax - 1) / lmax;
    int lanes = 16;
    while (lanes > 1 && lanes * NS > 512) lanes /= 2;    // rows of >= 64 bytes for n <= 1024 at lmax 16
    const char* eln = getenv("BLD_LDLT_LANES");
    if (eln) {
        const int v = atoi(eln);
        if ((v == 4 || v == 8 || v == 16 || v == 32) && v * NS <= 512) lanes = v;
    }
    const dim3 block(lanes, NS);
    const long long nb = (nsys + lanes - 1) / lanes;
    if (nb > 2147483647LL) return fail(BLD_ERR_ARGUMENT, "too many systems");
    const size_t smem = (size_t)(n & ~1) * sizeof(double) + (size_t)NS * lanes * (sizeof(T) + sizeof(double));
    if (lmax == 4)
        k_ldlt_seg<T, 4><<<(unsigned)nb, block, smem, st>>>(gamma, beta, rhs, nsys, n);
    else if (lmax == 8)
        k_ldlt_seg<T, 8><<<(unsigned)nb, block, smem, st>>>(gamma, beta, rhs, nsys, n);
    else
        k_ldlt_seg<T, 16><<<(unsigned)nb, block, smem, st>>>(gamma, beta, rhs, nsys, n);
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// reads the per-member non-finite flags; members that diverged are remembered
// (bld_get_diverged) and the flags are cleared
int check_flag(bld_handle* h) {
    CUDA_TRY(cudaMemcpyAsync(h->flag_host, h->flag, h->B * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    bool any = false, timeout = false;
    for (int m = 0; m < h->B; ++m)
        if (h->flag_host[m]) {
            any = true;
            if (h->flag_host[m] & BLD_FLAG_TIMEOUT) timeout = true;
            if (h->flag_host[m] & BLD_FLAG_NONFINITE) h->diverged[m] = 1;
            h->flag_host[m] = 0;
        }
    if (any) {
        CUDA_TRY(cudaMemsetAsync(h->flag, 0, h->B * sizeof(int), h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        if (timeout) return fail(BLD_ERR_TIMEOUT, "a bounded device wait expired (a TMA copy did not complete)");
        return fail(BLD_ERR_DIVERGED, "The simulation has diverged.");
    }
    return BLD_OK;
}

int validate(const bld_config* c) {
    if (c->n3 < 3) return fail(BLD_ERR_INVALID_CONFIG, "Due to boundary stencils, the grid needs at least 3 vertical layers");
    if (c->n1 < 1 || c->n2 < 1) return fail(BLD_ERR_INVALID_CONFIG, "invalid horizontal resolution");
    if (c->members < 1) return fail(BLD_ERR_INVALID_CONFIG, "members must be >= 1");
    if (!c->dx3_c || !c->dx3_i || !c->x3_c || !c->x3_i) return fail(BLD_ERR_ARGUMENT, "vertical mapping tables missing");
    if (c->pressure) {
        if (c->bc_kind[2][0] != BLD_BC_DIRICHLET || c->bc_kind[2][1] != BLD_BC_DIRICHLET)
            return fail(BLD_ERR_UNSUPPORTED_BC, "The pressure solver only supports Dirichlet BCs");
        if (c->bc_value[2][0] != c->bc_value[2][1])
            return fail(BLD_ERR_UNSUPPORTED_BC, "The mean flow must be equal at both vertical boundaries.");
    }
    if (c->advection || c->sgs) {
        if (c->bc_kind[2][0] != BLD_BC_DIRICHLET || c->bc_kind[2][1] != BLD_BC_DIRICHLET)
            return fail(BLD_ERR_UNSUPPORTED_BC, "physical-domain processes need Dirichlet boundaries for vel3");
    }
    if (c->advection && (c->bc_value[2][0] != 0.0 || c->bc_value[2][1] != 0.0))
        return fail(BLD_ERR_UNSUPPORTED_BC, "Advection for non-zero w at boundary not implemented");
    if (c->sgs) {
        for (int s = 0; s < 2; ++s)
            if (c->wall_kind[s] != BLD_WALL_ROUGH && c->wall_kind[s] != BLD_WALL_FREESLIP)
                return fail(BLD_ERR_UNSUPPORTED_BC, "SGS model only supports rough-wall and free-slip boundaries");
    }
    if (c->diffusion[2] && (c->bc_kind[2][0] != BLD_BC_DIRICHLET || c->bc_kind[2][1] != BLD_BC_DIRICHLET))
        return fail(BLD_ERR_UNSUPPORTED_BC, "diffusion of vel3 needs Dirichlet boundaries");
    if (c->mean[2]) return fail(BLD_ERR_INVALID_CONFIG, "The constant-mean source currently does not handle I-nodes correctly");
    return BLD_OK;
}

int setup_space(bld_handle* h, Space& s, int dealias, int e1, int e2, bool is_adv) {
    const int k1 = h->g.k1max, k2 = h->g.k2max;
    int r1, r2;
    if (dealias == BLD_DEALIAS_QUADRATIC) {
        r1 = pdsize_quadratic(k1);
        r2 = pdsize_quadratic(k2);
        s.P1 = next_even_smooth(r1);
        s.P2 = next_even_smooth(r2);
    } else if (dealias == BLD_DEALIAS_NONE) {
        r1 = 2 * k1 + 2;
        r2 = 2 * k2 + 2;
        s.P1 = r1;
        s.P2 = r2;
    } else {
        r1 = e1;
        r2 = e2;
        s.P1 = e1;
        s.P2 = e2;
    }
    s.ref_P1 = r1;
    s.ref_P2 = r2;
    for (int P : {s.P1, s.P2})
        if (!(P % 2 == 0 && smooth2357(P)) || make_plan(P, h->fp32).nst == 0)
            return fail(BLD_ERR_INVALID_CONFIG,
                        "physical-domain size %d is not an even product of 2, 3, 5 and 7 with at most four "
                        "codelet stages", P);
    if (s.P1 < 2 * k1 + 2 || s.P2 < 2 * k2 + 2)
        return fail(BLD_ERR_INVALID_CONFIG, "physical-domain size (%d, %d) smaller than the resolved modes", s.P1, s.P2);
    if (s.P1 > 1024 || s.P2 > 1024) return fail(BLD_ERR_INVALID_CONFIG, "physical-domain size above 1024");
    s.plan1 = make_plan(s.P1, h->fp32);
    s.plan2 = make_plan(s.P2, h->fp32);
    BLD_TRY(twiddles(h, s.P1));
    BLD_TRY(twiddles(h, s.P2));
    s.ntin = is_adv ? 6 : 9;
    s.ntout = is_adv ? 3 : 8;
    s.fsets = is_adv ? 1 : 2;
    tile_space(h, s, is_adv);
    if (!s.PPT) return fail(BLD_ERR_INVALID_CONFIG, "no thread tiling for physical size %d", s.P1);
    // defaults until the autotuner runs: per-term y passes
    s.inv = YCfg{0, h->fp32 ? 8 : 4, 256};
    s.fwd = YCfg{0, h->fp32 ? 8 : 4, 256};
    while (s.inv.NL > 1 && (size_t)(s.P2 + 2 * s.P2 * s.inv.NL) * csize(h->fp32) > 110 * 1024) s.inv.NL /= 2;
    while (s.fwd.NL > 1 && (size_t)(s.P2 + 2 * s.P2 * s.fsets * s.fwd.NL) * csize(h->fp32) > 110 * 1024) s.fwd.NL /= 2;
    const size_t cs = csize(h->fp32);
    const long long layer = (long long)s.P2 * h->g.K1;
    s.min_ms = (long long)s.ntin * h->g.n3 * layer;
    s.mout_ms = (long long)s.ntout * h->g.n3 * layer;
    BLD_TRY(dalloc(h, &s.min, (size_t)s.min_ms * h->B * cs));
    BLD_TRY(dalloc(h, &s.mout, (size_t)s.mout_ms * h->B * cs));
    CUDA_TRY(cudaMemset(s.mout, 0, (size_t)s.mout_ms * h->B * cs));
    const size_t sm = is_adv ? smem_adv(s, h->fp32) : smem_sgs(s, h->fp32, h->g.K1);
    if (sm > 200 * 1024 || (size_t)(s.P2 + 2 * s.P2 * s.fsets * s.fwd.NL) * csize(h->fp32) > 200 * 1024)
        return fail(BLD_ERR_INVALID_CONFIG, "physical-domain size (%d, %d) needs too much shared memory", s.P1, s.P2);
    s.on = true;
    return BLD_OK;
}

// Smagorinsky length scales squared and wall-model factors of one member
// (src/processes/static_smagorinsky.jl:44-123): l = Cs cbrt(D1 D2 D3), wall
// damping (l^-N + (kappa z)^-N)^(-1/N), strain factor 1/(2 dz log(dz/z0)) and
// stress factor -kappa^2/log^2(dz/z0) (upper-wall factors negated).
void member_sgs_tables(const bld_handle* h, double cs, double z0lo, double* lc2, double* li2, double* wall4) {
    const bld_config* cfg = &h->cfg;
    const Geo& g = h->g;
    const int n3 = g.n3;
    const double D1 = cfg->l1 / (2.0 * g.k1max + 2.0), D2 = cfg->l2 / (2.0 * g.k2max + 2.0);
    auto ml = [&](double x3) {
        double lo = INFINITY, hi = INFINITY;
        if (cfg->wall_kind[0] == BLD_WALL_ROUGH) lo = (x3 - cfg->x3_min) * cfg->wall_kappa[0];
        if (cfg->wall_kind[1] == BLD_WALL_ROUGH) hi = (cfg->x3_max - x3) * cfg->wall_kappa[1];
        return std::min(lo, hi);
    };
    const double N = cfg->sgs_wall_damping_exponent;
    for (int i = 0; i < n3; ++i) {
        double l = cs * std::cbrt(D1 * D2 * (h->tab_dx3c[i] / n3));
        if (cfg->sgs_wall_damping) l = std::pow(std::pow(l, -N) + std::pow(ml(h->tab_x3c[i]), -N), -1.0 / N);
        lc2[i] = l * l;
    }
    for (int i = 0; i < n3 - 1; ++i) {
        double l = cs * std::cbrt(D1 * D2 * (h->tab_dx3i[i + 1] / n3));
        if (cfg->sgs_wall_damping) l = std::pow(std::pow(l, -N) + std::pow(ml(h->tab_x3i[i]), -N), -1.0 / N);
        li2[i] = l * l;
    }
    const double dxb = h->tab_x3c[0] - cfg->x3_min, dxa = cfg->x3_max - h->tab_x3c[n3 - 1];
    double fs[2] = {0, 0}, ft[2] = {0, 0};
    for (int sd = 0; sd < 2; ++sd) {
        if (cfg->wall_kind[sd] != BLD_WALL_ROUGH) continue;
        const double dx = sd == 0 ? dxb : dxa;
        const double z0 = sd == 0 ? z0lo : cfg->wall_z0[1];
        const double lg = std::log(dx / z0);
        fs[sd] = 1.0 / (2.0 * dx * lg);
        ft[sd] = -(cfg->wall_kappa[sd] * cfg->wall_kappa[sd]) / (lg * lg);
    }
    wall4[0] = fs[0];
    wall4[1] = -fs[1];
    wall4[2] = ft[0];
    wall4[3] = -ft[1];
}

void free_handle(bld_handle* h) {
    if (!h) return;
    for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
    for (auto& kv : h->graph_src) cudaGraphDestroy(kv.second);
    if (h->prof_acc) cudaFree(h->prof_acc);
    if (h->prof_prev) cudaFree(h->prof_prev);
    for (auto& kv : h->ens_graphs) cudaGraphExecDestroy(kv.second);
    void* ptrs[] = {h->u, h->t, h->du, h->dp, h->io, h->io2, h->pscr, h->gamma, h->d1, h->d2, h->DD1, h->DD2,
                    h->alpha_c, h->inv_alpha_c, h->alpha_i, h->alpha_ext, h->mean_w, h->lc2, h->li2, h->wall, h->src,
                    h->mean_val, h->flag, h->active, h->adv.min, h->adv.mout, h->sgs.min, h->sgs.mout, h->pd_buf, h->pd_mixed,
                    h->prog_small, h->prog_buf, h->prog_mixed};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (auto& kv : h->tw) {
        cudaFree(kv.second.d64);
        cudaFree(kv.second.d32);
    }
    if (h->flag_host) cudaFreeHost(h->flag_host);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // namespace

// ======================================================================== C ABI
extern "C" {

int32_t bld_abi_version(void) { return BLD_ABI_VERSION; }

const char* bld_status_string(int32_t s) {
    switch (s) {
        case BLD_OK: return "ok";
        case BLD_ERR_INVALID_CONFIG: return "invalid configuration";
        case BLD_ERR_OUT_OF_MEMORY: return "out of device memory";
        case BLD_ERR_DIVERGED: return "The simulation has diverged.";
        case BLD_ERR_UNSUPPORTED_BC: return "unsupported boundary condition";
        case BLD_ERR_CUDA: return "CUDA error";
        case BLD_ERR_TIMEOUT: return "device wait timed out";
        case BLD_ERR_ARGUMENT: return "invalid argument";
        case BLD_ERR_NO_DEVICE: return "no usable CUDA device";
        default: return "unknown status";
    }
}

int32_t bld_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return BLD_ERR_ARGUMENT;
    snprintf(buf, len, "%s", g_last_error.c_str());
    return BLD_OK;
}

int32_t bld_create(const bld_config* cfg, bld_handle** out) {
    if (!cfg || !out) return fail(BLD_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    BLD_TRY(validate(cfg));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || cfg->device >= ndev)
        return fail(BLD_ERR_NO_DEVICE, "no CUDA device %d available", cfg->device);
    CUDA_TRY(cudaSetDevice(cfg->device));
    BLD_TRY(set_smem_limits());
    bld_handle* h = new bld_handle();
    h->cfg = *cfg;
    h->cfg.dx3_c = h->cfg.dx3_i = h->cfg.x3_c = h->cfg.x3_i = nullptr;  // caller memory: copied below
    h->cfg.member_cs = h->cfg.member_z0_lower = h->cfg.member_source1 = nullptr;
    h->device = cfg->device;
    h->B = cfg->members;
    h->fp32 = (cfg->precision == BLD_MIXED);
    Geo& g = h->g;
    g.k1max = (cfg->n1 - 1) / 2;
    g.k2max = (cfg->n2 - 1) / 2;
    g.K1 = g.k1max + 1;
    g.K2 = 2 * g.k2max + 1;
    g.n3 = cfg->n3;
    g.F = g.K1 * g.K2;
    g.mstride = (long long)(3 * g.n3 - 1) * g.F;
    const int n3 = g.n3, K1 = g.K1, K2 = g.K2, B = h->B;
    auto bail = [&](int code) {
        free_handle(h);
        return code;
    };
#define H_TRY(expr)                   \
    do {                              \
        int s_ = (expr);              \
        if (s_ != BLD_OK) return bail(s_); \
    } while (0)
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(BLD_ERR_CUDA, "cudaStreamCreate failed"));
    const size_t sbytes = (size_t)B * g.mstride * sizeof(double2);
    H_TRY(dalloc(h, (void**)&h->u, sbytes));
    H_TRY(dalloc(h, (void**)&h->t, sbytes));
    H_TRY(dalloc(h, (void**)&h->du, sbytes));
    H_TRY(dalloc(h, (void**)&h->dp, sbytes));
    H_TRY(dalloc(h, (void**)&h->io, sbytes));
    H_TRY(dalloc(h, (void**)&h->io2, sbytes));
    for (void* p : {(void*)h->u, (void*)h->t, (void*)h->du, (void*)h->dp, (void*)h->io, (void*)h->io2})
        if (cudaMemset(p, 0, sbytes) != cudaSuccess) return bail(fail(BLD_ERR_CUDA, "cudaMemset failed"));
    if (cfg->pressure) H_TRY(dalloc(h, (void**)&h->pscr, (size_t)B * n3 * g.F * sizeof(double2)));
    H_TRY(dalloc(h, (void**)&h->flag, h->B * sizeof(int)));
    h->active_host.assign(B, 1);
    H_TRY(upload(h, &h->active, h->active_host));
    if (cudaMemset(h->flag, 0, h->B * sizeof(int)) != cudaSuccess) return bail(fail(BLD_ERR_CUDA, "cudaMemset failed"));
    if (cudaMallocHost(&h->flag_host, h->B * sizeof(int)) != cudaSuccess)
        return bail(fail(BLD_ERR_CUDA, "cudaMallocHost failed"));
    for (int m = 0; m < h->B; ++m) h->flag_host[m] = 0;
    h->diverged.assign(h->B, 0);

    // ---- wavenumber factors (src/Domains.jl:142-145, src/derivatives.jl:21-27)
    const double TWO_PI = 2.0 * M_PI;
    std::vector<double> d1(K1), d2(K2), DD1(K1), DD2(K2);
    const double c1 = TWO_PI / cfg->l1, c2 = TWO_PI / cfg->l2;
    for (int k = 0; k < K1; ++k) {
        d1[k] = (double)k * c1;
        DD1[k] = (double)(-(long long)k * k) * (c1 * c1);
    }
    for (int j = 0; j < K2; ++j) {
        const long long k2 = (j <= g.k2max) ? j : j - K2;
        d2[j] = (double)k2 * c2;
        DD2[j] = (double)(-k2 * k2) * (c2 * c2);
    }
    // ---- vertical factors alpha = N3 / (dx3/dzeta) (src/derivatives.jl:10-19)
    std::vector<double> ac(n3), ai(n3 - 1), aext(n3 + 1), mw(n3), iac(n3);
    for (int i = 0; i < n3; ++i) ac[i] = (double)n3 / cfg->dx3_c[i];
    for (int i = 0; i < n3; ++i) iac[i] = 1.0 / ac[i];
    for (int i = 0; i <= n3; ++i) aext[i] = (double)n3 / cfg->dx3_i[i];
    for (int i = 0; i < n3 - 1; ++i) ai[i] = aext[i + 1];
    const double L3 = cfg->x3_max - cfg->x3_min;
    for (int i = 0; i < n3; ++i) mw[i] = 1.0 / ac[i] / L3;  // ConstantMean weight (src/processes/sources.jl:64)
    H_TRY(upload(h, &h->d1, d1));
    H_TRY(upload(h, &h->d2, d2));
    H_TRY(upload(h, &h->DD1, DD1));
    H_TRY(upload(h, &h->DD2, DD2));
    H_TRY(upload(h, &h->alpha_c, ac));
    H_TRY(upload(h, &h->inv_alpha_c, iac));
    H_TRY(upload(h, &h->alpha_i, ai));
    H_TRY(upload(h, &h->alpha_ext, aext));
    H_TRY(upload(h, &h->mean_w, mw));

    // ---- pressure: d3g3 diagonal and LDL^T factor (src/processes/pressure.jl:231-296,85-95)
    if (cfg->pressure) {
        std::vector<double> d3g3(n3, 0.0);
        for (int i = 1; i < n3; ++i) d3g3[i] -= aext[i];
        for (int i = 0; i < n3 - 1; ++i) d3g3[i] -= aext[i + 1];
        const double s1 = 1.0 / cfg->l1, s2 = 1.0 / cfg->l2;
        const double fourpi2 = 4.0 * (M_PI * M_PI);
        std::vector<double> gam((size_t)n3 * g.F);
        std::vector<double> dv(n3);
        for (int j = 0; j < K2; ++j) {
            const long long k2 = (j <= g.k2max) ? j : j - K2;
            for (int k = 0; k < K1; ++k) {
                const int c = j * K1 + k;
                if (k == 0 && k2 == 0) {
                    for (int z = 0; z < n3; ++z) dv[z] = d3g3[z];
                    dv[n3 - 1] = -3.0 * aext[n3 - 1];
                } else {
                    const double kk = (double)((long long)k * k) * (s1 * s1) + (double)(k2 * k2) * (s2 * s2);
                    for (int z = 0; z < n3; ++z) dv[z] = d3g3[z] - fourpi2 * kk / ac[z];
                }
                double gp = 1.0 / dv[0];
                gam[c] = gp;
                for (int z = 1; z < n3; ++z) {
                    const double be = ai[z - 1];
                    gp = 1.0 / (dv[z] - gp * (be * be));
                    gam[(size_t)z * g.F + c] = gp;
                }
            }
        }
        H_TRY(upload(h, &h->gamma, gam));
    }

    // ---- boundary conditions and the linear processes
    h->w_lo = cfg->bc_value[2][0];
    h->w_hi = cfg->bc_value[2][1];
    Linear& L = h->lin;
    for (int f = 0; f < 3; ++f) {
        L.diff_on[f] = cfg->diffusion[f];
        L.nu[f] = cfg->diffusivity[f];
        L.src_on[f] = cfg->source[f];
        for (int s = 0; s < 2; ++s) {
            L.bc_kind[f][s] = cfg->bc_kind[f][s];
            L.bc_val[f][s] = cfg->bc_value[f][s];
            // ConstantGradient.difference = gradient * Dvmap(zeta_wall) / N3 (src/boundary_conditions.jl:56-57,69,76)
            L.bc_diff[f][s] = cfg->bc_value[f][s] * (cfg->dx3_i[s == 0 ? 0 : n3] / (double)n3);
        }
    }
    std::vector<double> src((size_t)3 * B), mval((size_t)3 * B);
    for (int m = 0; m < B; ++m)
        for (int f = 0; f < 3; ++f) {
            src[3 * m + f] = cfg->source_strength[f];
            if (f == 0 && cfg->member_source1) src[3 * m + f] = cfg->member_source1[m];
            mval[3 * m + f] = cfg->mean_value[f];
        }
    H_TRY(upload(h, &h->src, src));
    H_TRY(upload(h, &h->mean_val, mval));
    L.DD1 = h->DD1;
    L.DD2 = h->DD2;
    L.alpha_c = h->alpha_c;
    L.alpha_i = h->alpha_i;
    L.alpha_ext = h->alpha_ext;
    L.src = h->src;

    // ---- SGS length scales and wall model (src/processes/static_smagorinsky.jl:44-123)
    std::vector<double> lc2((size_t)B * n3, 0.0), li2((size_t)B * (n3 - 1), 0.0), wall((size_t)4 * B, 0.0);
    h->tab_dx3c.assign(cfg->dx3_c, cfg->dx3_c + n3);
    h->tab_dx3i.assign(cfg->dx3_i, cfg->dx3_i + n3 + 1);
    h->tab_x3c.assign(cfg->x3_c, cfg->x3_c + n3);
    h->tab_x3i.assign(cfg->x3_i, cfg->x3_i + n3 - 1);
    if (cfg->sgs) {
        h->dyn_lo = cfg->wall_kind[0] == BLD_WALL_ROUGH;
        h->dyn_hi = cfg->wall_kind[1] == BLD_WALL_ROUGH;
        for (int m = 0; m < B; ++m) {
            const double cs = cfg->member_cs ? cfg->member_cs[m] : cfg->sgs_cs;
            const double z0lo = (cfg->member_z0_lower) ? cfg->member_z0_lower[m] : cfg->wall_z0[0];
            member_sgs_tables(h, cs, z0lo, &lc2[(size_t)m * n3], &li2[(size_t)m * (n3 - 1)], &wall[4 * (size_t)m]);
            h->member_cs.push_back(cs);
            h->member_z0.push_back(z0lo);
        }
    }
    H_TRY(upload(h, &h->lc2, lc2));
    H_TRY(upload(h, &h->li2, li2));
    H_TRY(upload(h, &h->wall, wall));

    // ---- physical-domain spaces
    if (cfg->advection) H_TRY(setup_space(h, h->adv, cfg->adv_dealias, cfg->adv_p1, cfg->adv_p2, true));
    if (cfg->sgs) H_TRY(setup_space(h, h->sgs, cfg->sgs_dealias, cfg->sgs_p1, cfg->sgs_p2, false));
    // default-size transform for initialize!/getindex (src/physical_space.jl:44)
    h->Pd1 = 2 * g.k1max + 2;
    h->Pd2 = 2 * g.k2max + 2;
    if (smooth23(h->Pd1) && smooth23(h->Pd2)) {
        H_TRY(twiddles(h, h->Pd1));
        H_TRY(twiddles(h, h->Pd2));
        H_TRY(dalloc(h, &h->pd_buf, (size_t)n3 * h->Pd2 * h->Pd1 * sizeof(double)));
        H_TRY(dalloc(h, &h->pd_mixed, (size_t)n3 * h->Pd2 * K1 * sizeof(double2)));
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(BLD_ERR_CUDA, "set-up failed"));
    H_TRY(autotune(h));
#undef H_TRY
    *out = h;
    return BLD_OK;
}

void bld_destroy(bld_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_handle(h);
}

int32_t bld_get_info(const bld_handle* h, bld_info* info) {
    if (!h || !info) return fail(BLD_ERR_ARGUMENT, "null argument");
    memset(info, 0, sizeof *info);
    info->k1max = h->g.k1max;
    info->k2max = h->g.k2max;
    info->n3 = h->g.n3;
    info->members = h->B;
    info->modes_per_layer = h->g.F;
    info->state_doubles = 2 * h->g.mstride;
    if (h->adv.on) {
        info->adv_p1 = h->adv.P1;
        info->adv_p2 = h->adv.P2;
        info->adv_ref_p1 = h->adv.ref_P1;
        info->adv_ref_p2 = h->adv.ref_P2;
    }
    if (h->sgs.on) {
        info->sgs_p1 = h->sgs.P1;
        info->sgs_p2 = h->sgs.P2;
    }
    info->device_bytes = (int64_t)h->bytes;
    info->precision = h->cfg.precision;
    return BLD_OK;
}

static int member_ok(const bld_handle* h, int m) { return h && m >= 0 && m < h->B; }

static int copy_fields_h2d(bld_handle* h, double2* base, int m, const double* v1, const double* v2, const double* v3) {
    const Geo& g = h->g;
    double2* dst = base + (size_t)m * g.mstride;
    const size_t nc = (size_t)g.n3 * g.F, ni = (size_t)(g.n3 - 1) * g.F;
    CUDA_TRY(cudaMemcpyAsync(dst, v1, nc * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(dst + nc, v2, nc * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(dst + 2 * nc, v3, ni * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    return BLD_OK;
}

static int copy_fields_d2h(bld_handle* h, const double2* base, int m, double* v1, double* v2, double* v3) {
    const Geo& g = h->g;
    const double2* src = base + (size_t)m * g.mstride;
    const size_t nc = (size_t)g.n3 * g.F, ni = (size_t)(g.n3 - 1) * g.F;
    CUDA_TRY(cudaMemcpyAsync(v1, src, nc * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaMemcpyAsync(v2, src + nc, nc * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaMemcpyAsync(v3, src + 2 * nc, ni * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

int32_t bld_set_state(bld_handle* h, int32_t m, const double* v1, const double* v2, const double* v3) {
    if (!member_ok(h, m) || !v1 || !v2 || !v3) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    CUDA_TRY(cudaSetDevice(h->device));
    BLD_TRY(copy_fields_h2d(h, h->u, m, v1, v2, v3));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->slope_valid = false;
    h->ab2_started = false;
    return BLD_OK;
}

int32_t bld_get_state(bld_handle* h, int32_t m, double* v1, double* v2, double* v3) {
    if (!member_ok(h, m) || !v1 || !v2 || !v3) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    CUDA_TRY(cudaSetDevice(h->device));
    return copy_fields_d2h(h, h->u, m, v1, v2, v3);
}

int32_t bld_compute_rates(bld_handle* h, int32_t m, const double* v1, const double* v2, const double* v3,
                          double* r1, double* r2, double* r3) {
    if (!member_ok(h, m) || !v1 || !v2 || !v3 || !r1 || !r2 || !r3) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    CUDA_TRY(cudaSetDevice(h->device));
    BLD_TRY(copy_fields_h2d(h, h->io, m, v1, v2, v3));
    BLD_TRY(enqueue_rates(h, h->io, h->io2, m, 1));
    BLD_TRY(copy_fields_d2h(h, h->io2, m, r1, r2, r3));
    return check_flag(h);
}

int32_t bld_apply_projections(bld_handle* h, int32_t m, double* v1, double* v2, double* v3) {
    if (!member_ok(h, m) || !v1 || !v2 || !v3) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    CUDA_TRY(cudaSetDevice(h->device));
    BLD_TRY(copy_fields_h2d(h, h->io, m, v1, v2, v3));
    BLD_TRY(enqueue_project(h, S_NONE, 0.0, h->io, nullptr, nullptr, nullptr, h->io, m, 1));
    BLD_TRY(copy_fields_d2h(h, h->io, m, v1, v2, v3));
    // the tile projection's bounded wait reports through the flags
    return check_flag(h);
}

int32_t bld_prepare(bld_handle* h) {
    if (!h) return fail(BLD_ERR_ARGUMENT, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    BLD_TRY(enqueue_project(h, S_NONE, 0.0, h->u, nullptr, nullptr, nullptr, h->u, 0, h->B));
    BLD_TRY(enqueue_rates(h, h->u, h->du, 0, h->B));
    h->slope_valid = true;
    h->ab2_started = false;
    return check_flag(h);
}

static int step_impl(bld_handle* h, int64_t nsteps, double dt, int32_t method);

// step graphs with and without the mean-profile sample are kept apart
static int gkey(const bld_handle* h, int method) { return method + (h->prof_on ? 16 : 0); }

// one trapezoid of the device mean profiles for every member (w = dt/2), or a bare sample (w = 0)
static int enqueue_profile_sample(bld_handle* h, double w) {
    k_profile_sample<<<h->B, 128, 0, h->stream>>>(h->g, h->u, h->prof_acc, h->prof_prev, w, 0,
                                                  h->mask_on ? h->active : nullptr);
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

// captures one step of `method` (regular steps; AB2 after its start-up step) into
// a CUDA graph, kept as source graph and instantiated executable
static int step_graph(bld_handle* h, int method, double dt, int chain = 0) {
    const auto key = std::make_pair(gkey(h, method) + 32 * chain, dt);
    if (h->graphs.count(key)) return BLD_OK;
    cudaGraph_t graph;
    CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int st = enqueue_step(h, method, dt, false, chain);
    if (st == BLD_OK && h->prof_on) {
        h->mask_on = true;
        st = enqueue_profile_sample(h, 0.5 * dt);
        h->mask_on = false;
    }
    cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
    if (st != BLD_OK) {
        if (ce == cudaSuccess) cudaGraphDestroy(graph);
        return st;
    }
    CUDA_TRY(ce);
    cudaGraphExec_t exec;
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(graph);
        CUDA_TRY(ie);
    }
    h->graphs.emplace(key, exec);
    h->graph_src.emplace(key, graph);
    return BLD_OK;
}

int32_t bld_step(bld_handle* h, int64_t nsteps, double dt, int32_t method) {
    BLD_TRY(step_impl(h, nsteps, dt, method));
    return check_flag(h);
}

int32_t bld_step_async(bld_handle* h, int64_t nsteps, double dt, int32_t method) {
    return step_impl(h, nsteps, dt, method);
}

static int step_impl(bld_handle* h, int64_t nsteps, double dt, int32_t method) {
    if (!h) return fail(BLD_ERR_ARGUMENT, "null handle");
    if (method < BLD_EULER || method > BLD_SSPRK33) return fail(BLD_ERR_ARGUMENT, "unknown method %d", method);
    if (!h->slope_valid) return fail(BLD_ERR_ARGUMENT, "bld_prepare or bld_evolve must run before bld_step");
    if (nsteps <= 0) return BLD_OK;
    CUDA_TRY(cudaSetDevice(h->device));
    int64_t done = 0;
    if (method == BLD_AB2) {
        if (h->ab2_started && h->ab2_dt != dt) return fail(BLD_ERR_ARGUMENT, "Cannot change time step for multi-step methods");
        if (!h->ab2_started) {
            BLD_TRY(enqueue_step(h, method, dt, true));
            if (h->prof_on) {
                h->mask_on = true;
                const int st = enqueue_profile_sample(h, 0.5 * dt);
                h->mask_on = false;
                BLD_TRY(st);
            }
            h->ab2_started = true;
            h->ab2_dt = dt;
            done = 1;
        }
    }
    if (done < nsteps) {
        // chained steps: the first leaves the next step's first stage value in t,
        // the middle ones enter and leave, the last one enters and ends with f(u)
        const bool chain = nsteps - done >= 2 && chain_ok(h, method);
        auto graph_for = [&](int c, cudaGraphExec_t* g) -> int {
            const auto key = std::make_pair(gkey(h, method) + 32 * c, dt);
            auto it = h->graphs.find(key);
            if (it == h->graphs.end()) {
                BLD_TRY(step_graph(h, method, dt, c));
                it = h->graphs.find(key);
            }
            *g = it->second;
            return BLD_OK;
        };
        if (!chain) {
            cudaGraphExec_t g;
            BLD_TRY(graph_for(0, &g));
            for (; done < nsteps; ++done) CUDA_TRY(cudaGraphLaunch(g, h->stream));
        } else {
            cudaGraphExec_t gfirst, gmid, glast;
            BLD_TRY(graph_for(CHAIN_LEAVE, &gfirst));
            BLD_TRY(graph_for(CHAIN_ENTER | CHAIN_LEAVE, &gmid));
            BLD_TRY(graph_for(CHAIN_ENTER, &glast));
            const int64_t last = nsteps - 1;
            for (; done < nsteps; ++done)
                CUDA_TRY(cudaGraphLaunch(done == 0 ? gfirst : (done == last ? glast : gmid), h->stream));
        }
    }
    return BLD_OK;
}

int32_t bld_ensemble_step(bld_handle* const* hs, int32_t n, int64_t nsteps, double dt, int32_t method) {
    if (!hs || n < 1) return fail(BLD_ERR_ARGUMENT, "no handles");
    if (method == BLD_AB2) return fail(BLD_ERR_ARGUMENT, "ensemble stepping supports the one-step methods");
    if (method < BLD_EULER || method > BLD_SSPRK33) return fail(BLD_ERR_ARGUMENT, "unknown method %d", method);
    bld_handle* lead = hs[0];
    for (int i = 0; i < n; ++i) {
        if (!hs[i] || !hs[i]->slope_valid) return fail(BLD_ERR_ARGUMENT, "handle %d is not prepared", i);
        if (hs[i]->device != lead->device) return fail(BLD_ERR_ARGUMENT, "handles on different devices");
    }
    if (nsteps <= 0) return BLD_OK;
    CUDA_TRY(cudaSetDevice(lead->device));
    // chained steps as in bld_step (every class must allow it): the first leaves
    // the next step's first stage value, the middle ones enter and leave, the
    // last enters and ends with f(u)
    bool chain = nsteps >= 2;
    for (int i = 0; i < n; ++i) chain = chain && chain_ok(hs[i], method);
    // the parent graph of one step variant `c`: the classes' step graphs as
    // independent children
    auto parent_for = [&](int c, cudaGraphExec_t* out) -> int {
        std::vector<const void*> key;
        for (int i = 0; i < n; ++i) {
            key.push_back(hs[i]);
            key.push_back((const void*)(intptr_t)(gkey(hs[i], method) + 32 * c));
        }
        double dtk = dt;
        const void* dtp;
        memcpy(&dtp, &dtk, sizeof(dtp) < sizeof(dtk) ? sizeof(dtp) : sizeof(dtk));
        key.push_back(dtp);
        auto it = lead->ens_graphs.find(key);
        if (it == lead->ens_graphs.end()) {
            cudaGraph_t parent;
            CUDA_TRY(cudaGraphCreate(&parent, 0));
            for (int i = 0; i < n; ++i) {
                int st = step_graph(hs[i], method, dt, c);
                if (st != BLD_OK) {
                    cudaGraphDestroy(parent);
                    return st;
                }
                cudaGraphNode_t node;
                cudaError_t e = cudaGraphAddChildGraphNode(
                    &node, parent, nullptr, 0, hs[i]->graph_src.at(std::make_pair(gkey(hs[i], method) + 32 * c, dt)));
                if (e != cudaSuccess) {
                    cudaGraphDestroy(parent);
                    CUDA_TRY(e);
                }
            }
            cudaGraphExec_t exec;
            cudaError_t ie = cudaGraphInstantiate(&exec, parent, 0);
            cudaGraphDestroy(parent);
            CUDA_TRY(ie);
            it = lead->ens_graphs.emplace(key, exec).first;
        }
        *out = it->second;
        return BLD_OK;
    };
    if (!chain) {
        cudaGraphExec_t g;
        BLD_TRY(parent_for(0, &g));
        for (int64_t s = 0; s < nsteps; ++s) CUDA_TRY(cudaGraphLaunch(g, lead->stream));
    } else {
        cudaGraphExec_t gfirst, gmid, glast;
        BLD_TRY(parent_for(CHAIN_LEAVE, &gfirst));
        BLD_TRY(parent_for(CHAIN_ENTER | CHAIN_LEAVE, &gmid));
        BLD_TRY(parent_for(CHAIN_ENTER, &glast));
        for (int64_t s = 0; s < nsteps; ++s)
            CUDA_TRY(cudaGraphLaunch(s == 0 ? gfirst : (s == nsteps - 1 ? glast : gmid), lead->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(lead->stream));
    int status = BLD_OK;
    for (int i = 0; i < n; ++i) {
        const int st = check_flag(hs[i]);
        if (st != BLD_OK) status = st;
    }
    return status;
}

int32_t bld_get_stream(bld_handle* h, void** stream) {
    if (!h || !stream) return fail(BLD_ERR_ARGUMENT, "null argument");
    *stream = (void*)h->stream;
    return BLD_OK;
}

static int launches_per_rhs(const bld_handle* h) {
    int n = 0;
    if (h->adv.on) n += 3;
    if (h->sgs.on) n += 3;
    return n ? n : 1;
}

int32_t bld_time_phases(bld_handle* h, int32_t iters, int32_t method, bld_phase_times* out) {
    if (!h || !out || iters < 1) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    CUDA_TRY(cudaSetDevice(h->device));
    memset(out, 0, sizeof *out);
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    auto timeit = [&](auto&& fn, double* ms) -> int {
        BLD_TRY(fn());  // warm-up launch
        CUDA_TRY(cudaEventRecord(e0, h->stream));
        for (int i = 0; i < iters; ++i) BLD_TRY(fn());
        CUDA_TRY(cudaEventRecord(e1, h->stream));
        CUDA_TRY(cudaEventSynchronize(e1));
        float t = 0;
        CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
        *ms = (double)t / iters;
        return BLD_OK;
    };
    int st = BLD_OK;
    const int B = h->B;
    for (int sp = 0; sp < 2 && st == BLD_OK; ++sp) {
        if (!(sp == 0 ? h->adv.on : h->sgs.on)) continue;
        st = timeit([&] { return enqueue_inv_y(h, sp, h->u, 0, B); }, &out->inv_y_ms[sp]);
        if (st == BLD_OK) st = timeit([&] { return enqueue_x(h, sp, 0, B); }, &out->x_ms[sp]);
        if (st == BLD_OK)
            st = timeit([&] { return enqueue_fwd_y(h, sp, true, false, h->u, h->io2, 0, B); }, &out->fwd_y_ms[sp]);
    }
    if (st == BLD_OK && !h->adv.on && !h->sgs.on)
        st = timeit([&] { return enqueue_linear(h, h->u, h->io2, 0, B); }, &out->linear_ms);
    if (st == BLD_OK)
        st = timeit([&] { return enqueue_project(h, S_NONE, 0.0, h->u, nullptr, nullptr, nullptr, h->io, 0, B); },
                    &out->project_ms);
    const int stages = method == BLD_SSPRK33 ? 3 : method == BLD_SSPRK22 ? 2 : 1;
    const bool proj = h->cfg.pressure || h->cfg.mean[0] || h->cfg.mean[1];
    out->launches_per_step = stages * (launches_per_rhs(h) + (proj || stages > 1 ? 1 : 1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st == BLD_OK) CUDA_TRY(cudaMemsetAsync(h->flag, 0, h->B * sizeof(int), h->stream));
    return st;
}

int32_t bld_evolve(bld_handle* h, double t1, double t2, double dt, int32_t method) {
    if (!h) return fail(BLD_ERR_ARGUMENT, "null handle");
    if (t1 > t2) return fail(BLD_ERR_ARGUMENT, "Integration start time is larger than end time");
    BLD_TRY(bld_prepare(h));
    if (h->prof_on) {  // the first sample is the projected initial state (src/ODEMethods.jl:179-185)
        BLD_TRY(enqueue_profile_sample(h, 0.0));
    }
    if (t2 > t1) {
        const double r = (t2 - t1) / dt;
        const double ri = std::round(r);
        if (std::fabs(r - ri) > std::sqrt(2.220446049250313e-16) * std::max(std::fabs(r), std::fabs(ri)))
            return fail(BLD_ERR_ARGUMENT, "Division has a non-integer result");
        BLD_TRY(bld_step(h, (int64_t)ri, dt, method));
    }
    return BLD_OK;
}

int32_t bld_compute_rates_device(bld_handle* h, const void* state, void* rates, void* stream) {
    if (!h || !state || !rates) return fail(BLD_ERR_ARGUMENT, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t keep = h->stream;
    if (stream) h->stream = (cudaStream_t)stream;
    int s = enqueue_rates(h, (const double2*)state, (double2*)rates, 0, h->B);
    h->stream = keep;
    return s;
}

int32_t bld_apply_projections_device(bld_handle* h, void* state, void* stream) {
    if (!h || !state) return fail(BLD_ERR_ARGUMENT, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t keep = h->stream;
    if (stream) h->stream = (cudaStream_t)stream;
    int s = enqueue_project(h, S_NONE, 0.0, (const double2*)state, nullptr, nullptr, nullptr, (double2*)state, 0, h->B);
    h->stream = keep;
    return s;
}

int32_t bld_state_device_ptr(bld_handle* h, void** state) {
    if (!h || !state) return fail(BLD_ERR_ARGUMENT, "null argument");
    *state = h->u;
    return BLD_OK;
}

int32_t bld_sync(bld_handle* h) {
    if (!h) return fail(BLD_ERR_ARGUMENT, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    return check_flag(h);
}

int32_t bld_stream_idle(bld_handle* h, int32_t* idle) {
    if (!h || !idle) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    CUDA_TRY(cudaSetDevice(h->device));
    const cudaError_t e = cudaStreamQuery(h->stream);
    if (e == cudaErrorNotReady) {
        *idle = 0;
        return BLD_OK;
    }
    CUDA_TRY(e);
    *idle = 1;
    return BLD_OK;
}

int32_t bld_set_wait_limit(int32_t device, int64_t cycles) {
    int prev = 0;
    CUDA_TRY(cudaGetDevice(&prev));
    CUDA_TRY(cudaSetDevice(device));
    const long long v = cycles < 0 ? BLD_WAIT_CYCLES : (long long)cycles;
    const cudaError_t e = cudaMemcpyToSymbol(g_bld_wait_limit, &v, sizeof(v));
    cudaSetDevice(prev);
    CUDA_TRY(e);
    return BLD_OK;
}

int32_t bld_set_active(bld_handle* h, const int32_t* mask) {
    if (!h) return fail(BLD_ERR_ARGUMENT, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    for (int m = 0; m < h->B; ++m) h->active_host[m] = mask ? (mask[m] != 0) : 1;
    CUDA_TRY(cudaMemcpyAsync(h->active, h->active_host.data(), h->B * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

int32_t bld_set_member_params(bld_handle* h, int32_t m, double cs, double z0_lower, double source1) {
    if (!member_ok(h, m)) return fail(BLD_ERR_ARGUMENT, "invalid member");
    CUDA_TRY(cudaSetDevice(h->device));
    const int n3 = h->g.n3;
    if (h->cfg.sgs && (!std::isnan(cs) || !std::isnan(z0_lower))) {
        if (std::isnan(cs)) cs = h->member_cs[m];
        if (std::isnan(z0_lower)) z0_lower = h->member_z0[m];
        if (!(cs > 0) || (h->cfg.wall_kind[0] == BLD_WALL_ROUGH && !(z0_lower > 0)))
            return fail(BLD_ERR_ARGUMENT, "invalid Cs or roughness length");
        std::vector<double> lc2(n3), li2(n3 - 1), wall(4);
        member_sgs_tables(h, cs, z0_lower, lc2.data(), li2.data(), wall.data());
        CUDA_TRY(cudaMemcpyAsync(h->lc2 + (size_t)m * n3, lc2.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(cudaMemcpyAsync(h->li2 + (size_t)m * (n3 - 1), li2.data(), (n3 - 1) * sizeof(double),
                                 cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(cudaMemcpyAsync(h->wall + 4 * (size_t)m, wall.data(), 4 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        h->member_cs[m] = cs;
        h->member_z0[m] = z0_lower;
    }
    if (!std::isnan(source1)) {
        CUDA_TRY(cudaMemcpyAsync(h->src + 3 * (size_t)m, &source1, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

int32_t bld_describe(bld_handle* h, char* buf, size_t len) {
    if (!h || !buf || len == 0) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    const char* R = h->fp32 ? "float" : "double";
    std::string out = "{";
    for (int sp = 0; sp < 2; ++sp) {
        const Space& s = sp == 0 ? h->adv : h->sgs;
        if (!s.on) continue;
        char tmp[768];
        const char* xk = sp == 0 ? "k_adv_x" : "k_sgs_x";
        char xname[96];
        if (sp == 0 && s.x2)
            snprintf(xname, sizeof xname, "k_adv_x2<%s, %d, %d%s>", R, y2_radix_a(s.P1), y2_radix_b(s.P1),
                     s.x2 == 3 ? ", wide" : (s.x2 == 4 ? ", 2 rows" : ""));
        else if (sp == 0 && s.xb)
            snprintf(xname, sizeof xname, "%s<%s, %d>", s.xb == 2 ? "k_adv_xp" : "k_adv_xb", R, s.P1 / 32);
        else if (sp == 0 && s.xw && s.xwmb > 1)
            snprintf(xname, sizeof xname, "k_adv_xwc<%s, %d, %d>", R, s.P1 / 32, s.xwmb);
        else if (sp == 0 && s.xw)
            snprintf(xname, sizeof xname, "k_adv_xw<%s, %d>", R, s.P1 / 32);
        else if (sp == 1 && s.sxk)
            snprintf(xname, sizeof xname, "k_sgs_x2<%s, %d, %d%s>", R, y2_radix_a(s.P1), y2_radix_b(s.P1),
                     s.sxk == 2 ? ", 2 rows" : "");
        else if (sp == 1 && s.sx2)
            snprintf(xname, sizeof xname, "%s<%s, %d, 0, %d%s>", xk, R, s.PPT, s.P1, s.sx2 % 2 == 0 ? ", 2" : "");
        else
            snprintf(xname, sizeof xname, "%s<%s, %d, %d>", xk, R, s.PPT, s.xr);
        char iname[64], fname[64];
        if (s.inv.tp == 2) snprintf(iname, sizeof iname, "k_inv_y3<%s, %d, %d>", R, y2_radix_a(s.P2), y2_radix_b(s.P2));
        else if (s.inv.tp) snprintf(iname, sizeof iname, "k_inv_y2<%s, %d, %d%s>", R, y2_radix_a(s.P2), y2_radix_b(s.P2),
                                    s.inv.tp == 3 ? ", 8 lines" : "");
        else if (s.inv.all) snprintf(iname, sizeof iname, "k_inv_y_all<%s>", R);
        else snprintf(iname, sizeof iname, "k_inv_y<%s, %d>", R, s.inv.wfft);
        if (s.fwd.tp) snprintf(fname, sizeof fname, "k_fwd_y2<%s, %d, %d%s>", R, y2_radix_a(s.P2), y2_radix_b(s.P2),
                               s.fwd.tp == 3 ? ", 8 lines" : (s.fwd.tp == 4 ? ", 2 outputs" : ""));
        else if (s.fwd.all) snprintf(fname, sizeof fname, "k_fwd_y_all<%s>", R);
        else snprintf(fname, sizeof fname, "k_fwd_y<%s, %d>", R, s.fwd.wfft);
        snprintf(tmp, sizeof tmp,
                 "%s\"%s\": {\"P\": [%d, %d], \"inv_y\": \"%s\", \"x\": \"%s\", \"fwd_y\": \"%s\", "
                 "\"inv_NL\": %d, \"fwd_NL\": %d, \"x_rows\": %d, \"x_chunks\": %d}",
                 out.size() > 1 ? ", " : "", sp == 0 ? "advection" : "sgs", s.P1, s.P2, iname, xname, fname, s.inv.NL,
                 s.fwd.NL, s.xb ? 1 : (s.xw ? s.xw : s.YT), s.nchunks);
        out += tmp;
    }
    char tmp[160];
    const bool seg = h->cfg.pressure && h->g.n3 <= 256 && h->proj_variant > 0;
    if (seg)
        snprintf(tmp, sizeof tmp, "%s\"projection\": \"k_project_seg<%d, %d, %s>\"", out.size() > 1 ? ", " : "",
                 h->g.n3 <= 128 ? 8 : 16, h->proj_variant == 2 ? 2 : 1, h->proj_variant == 3 ? "true" : "false");
    else
        snprintf(tmp, sizeof tmp, "%s\"projection\": \"k_project\"", out.size() > 1 ? ", " : "");
    out += tmp;
    if (h->proj_tile)
        snprintf(tmp, sizeof tmp, ", \"projection_stored\": \"%s<%d, %d>\"}",
                 h->proj_pipe ? "k_project_pipe" : "k_project_tile", h->g.n3 <= 128 ? 8 : 16, h->proj_tile);
    else
        snprintf(tmp, sizeof tmp, "}");
    out += tmp;
    if (out.size() + 1 > len) return fail(BLD_ERR_ARGUMENT, "buffer too small (%zu bytes needed)", out.size() + 1);
    memcpy(buf, out.c_str(), out.size() + 1);
    return BLD_OK;
}

int32_t bld_get_diverged(bld_handle* h, int32_t* out) {
    if (!h || !out) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    for (int m = 0; m < h->B; ++m) {
        out[m] = h->diverged[m];
        h->diverged[m] = 0;
    }
    return BLD_OK;
}

int32_t bld_prepare_member(bld_handle* h, int32_t m) {
    if (!member_ok(h, m)) return fail(BLD_ERR_ARGUMENT, "invalid member");
    CUDA_TRY(cudaSetDevice(h->device));
    BLD_TRY(enqueue_project(h, S_NONE, 0.0, h->u, nullptr, nullptr, nullptr, h->u, m, 1));
    BLD_TRY(enqueue_rates(h, h->u, h->du, m, 1));
    h->slope_valid = true;
    return check_flag(h);
}

// set_field! of `field` of member m from the physical values already in
// h->pd_buf (default size): r2c rows, then the forward y pass assigning the
// truncated modes (src/physical_space.jl:253-256).  Stream-ordered.
static int set_field_from_pd(bld_handle* h, int m, int field) {
    const Geo& g = h->g;
    const int nz = field == 2 ? g.n3 - 1 : g.n3;
    const int P1 = h->Pd1, P2 = h->Pd2;
    XPlainArgs xa{};
    xa.P1 = P1;
    xa.P2 = P2;
    xa.K1 = g.K1;
    xa.k1max = g.k1max;
    xa.nz = nz;
    xa.pd = (const double*)h->pd_buf;
    xa.mixed_out = (double2*)h->pd_mixed;
    xa.plan = make_plan(P1);
    xa.tw = (const double2*)twp(h, P1, false);
    const long long rows = (long long)nz * P2;
    k_x_r2c<<<(unsigned)((rows + 1) / 2), 256, (size_t)3 * P1 * sizeof(double2), h->stream>>>(xa);
    CUDA_TRY(cudaGetLastError());
    Space s{};
    s.P1 = P1;
    s.P2 = P2;
    s.inv = s.fwd = YCfg{0, pick_y(P2, false, 1), 256};
    FwdYArgs fa{};
    fa.g = g;
    fa.P1 = P1;
    fa.P2 = P2;
    fa.mout = h->pd_mixed;
    fa.mout_mstride = 0;
    fa.ncontrib[0] = 1;
    fa.c[0][0] = FwdContrib{0, 0};
    fa.mode = 2;
    fa.check = 0;
    fa.du = h->u + (size_t)m * g.mstride;
    fa.du_mstride = 0;
    fa.inv_n = 1.0 / ((double)P1 * (double)P2);
    fa.flag = h->flag;
    fa.fields = 1;
    fa.field0 = field;
    fa.m0 = 0;
    fa.plan = make_plan(P2);
    fa.tw = twp(h, P2, false);
    BLD_TRY(launch_fwd_y<double>(h, s, fa, 1));
    h->slope_valid = false;
    return BLD_OK;
}

int32_t bld_set_field_physical(bld_handle* h, int32_t m, int32_t field, const double* values) {
    if (!member_ok(h, m) || field < 0 || field > 2 || !values) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    if (!h->pd_buf) return fail(BLD_ERR_INVALID_CONFIG, "default physical size is not an even 2^a*3^b");
    CUDA_TRY(cudaSetDevice(h->device));
    const int nz = field == 2 ? h->g.n3 - 1 : h->g.n3;
    CUDA_TRY(cudaMemcpyAsync(h->pd_buf, values, (size_t)nz * h->Pd2 * h->Pd1 * sizeof(double), cudaMemcpyHostToDevice,
                             h->stream));
    BLD_TRY(set_field_from_pd(h, m, field));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

int32_t bld_init_random_field(bld_handle* h, int32_t m, int32_t field, const double* base, const double* scale,
                              int32_t distribution, uint64_t seed) {
    if (!member_ok(h, m) || field < 0 || field > 2 || !base || !scale || distribution < 0 || distribution > 1)
        return fail(BLD_ERR_ARGUMENT, "invalid argument");
    if (!h->pd_buf) return fail(BLD_ERR_INVALID_CONFIG, "default physical size is not an even 2^a*3^b");
    CUDA_TRY(cudaSetDevice(h->device));
    const int nz = field == 2 ? h->g.n3 - 1 : h->g.n3;
    // the per-layer tables travel in the kernel's argument buffer (no allocation):
    // at most BLD_INIT_MAX_LAYERS layers
    if (nz > BLD_INIT_MAX_LAYERS) return fail(BLD_ERR_INVALID_CONFIG, "more than %d layers", BLD_INIT_MAX_LAYERS);
    InitTables t{};
    for (int z = 0; z < nz; ++z) {
        t.base[z] = base[z];
        t.scale[z] = scale[z];
    }
    const long long n = (long long)nz * h->Pd2 * h->Pd1;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_init_random<<<blocks, 256, 0, h->stream>>>((double*)h->pd_buf, h->Pd1 * h->Pd2, nz, t, distribution,
                                                  init_key(seed, field));
    CUDA_TRY(cudaGetLastError());
    BLD_TRY(set_field_from_pd(h, m, field));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

// The physical values of `field` of member m on the P1 x P2 grid (inverse y pass
// and c2r rows with the block-Stockham kernels of the default-size transforms)
// into out [nz][P2][P1]; `mixed` holds nz P2 K1 complex values.  Stream-ordered.
static int physical_field_dev(bld_handle* h, int m, int field, int P1, int P2, double2* mixed, double* out) {
    const Geo& g = h->g;
    const int nz = field == 2 ? g.n3 - 1 : g.n3;
    Space s{};
    s.P1 = P1;
    s.P2 = P2;
    s.inv = s.fwd = YCfg{0, pick_y(P2, false, 1), 256};
    InvYArgs ia{};
    ia.g = g;
    ia.P2 = P2;
    ia.nterms = 1;
    ia.op[0] = T_DIRECT;
    ia.fld[0] = field;
    ia.isI[0] = field == 2;
    ia.m0 = m;
    ia.state = h->u;
    ia.mixed = mixed;
    ia.mixed_mstride = 0;
    ia.d1 = h->d1;
    ia.d2 = h->d2;
    ia.alpha_i = h->alpha_i;
    ia.plan = make_plan(P2);
    ia.tw = twp(h, P2, false);
    BLD_TRY(launch_inv_y<double>(h, s, ia, 1));
    XPlainArgs xa{};
    xa.P1 = P1;
    xa.P2 = P2;
    xa.K1 = g.K1;
    xa.k1max = g.k1max;
    xa.nz = nz;
    xa.pd_out = out;
    xa.mixed_in = mixed;
    xa.plan = make_plan(P1);
    xa.tw = (const double2*)twp(h, P1, false);
    const long long rows = (long long)nz * P2;
    k_x_c2r<<<(unsigned)((rows + 1) / 2), 256, (size_t)3 * P1 * sizeof(double2), h->stream>>>(xa);
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

int32_t bld_get_field_physical(bld_handle* h, int32_t m, int32_t field, double* values) {
    if (!member_ok(h, m) || field < 0 || field > 2 || !values) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    if (!h->pd_buf) return fail(BLD_ERR_INVALID_CONFIG, "default physical size is not an even 2^a*3^b");
    CUDA_TRY(cudaSetDevice(h->device));
    const int nz = field == 2 ? h->g.n3 - 1 : h->g.n3;
    const int P1 = h->Pd1, P2 = h->Pd2;
    BLD_TRY(physical_field_dev(h, m, field, P1, P2, (double2*)h->pd_mixed, (double*)h->pd_buf));
    CUDA_TRY(cudaMemcpyAsync(values, h->pd_buf, (size_t)nz * P2 * P1 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

int32_t bld_progress_stats(bld_handle* h, int32_t m, bld_progress* out) {
    if (!member_ok(h, m) || !out) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    CUDA_TRY(cudaSetDevice(h->device));
    const Geo& g = h->g;
    const int n3 = g.n3;
    // the largest physical grid of the model: advection, else SGS, else the default size
    const Space* big = h->adv.on ? &h->adv : (h->sgs.on ? &h->sgs : nullptr);
    const int P1 = big ? big->P1 : h->Pd1, P2 = big ? big->P2 : h->Pd2;
    if (!big && !h->pd_buf) return fail(BLD_ERR_INVALID_CONFIG, "default physical size is not an even 2^a*3^b");
    const int nsmall = 6 * n3 + n3 + 4;
    // prog_buf holds w on the largest grid, later u and v on the SGS grid
    const size_t buf_doubles = (size_t)n3 * std::max((size_t)P2 * P1, h->sgs.on ? 2 * (size_t)h->sgs.P1 * h->sgs.P2 : 0);
    if (!h->prog_small) {
        BLD_TRY(dalloc(h, (void**)&h->prog_small, nsmall * sizeof(double)));
        BLD_TRY(dalloc(h, &h->prog_buf, buf_doubles * sizeof(double)));
        BLD_TRY(dalloc(h, &h->prog_mixed, (size_t)n3 * P2 * g.K1 * sizeof(double2)));
    }
    CUDA_TRY(cudaMemsetAsync(h->prog_small, 0, nsmall * sizeof(double), h->stream));
    k_progress_modes<<<dim3(n3, 3), 256, 0, h->stream>>>(g, h->u + (size_t)m * g.mstride, h->prog_small);
    CUDA_TRY(cudaGetLastError());
    BLD_TRY(physical_field_dev(h, m, 2, P1, P2, (double2*)h->prog_mixed, (double*)h->prog_buf));
    k_layer_absmax<<<n3 - 1, 256, 0, h->stream>>>((const double*)h->prog_buf, (long long)P1 * P2, h->prog_small + 6 * n3);
    CUDA_TRY(cudaGetLastError());
    // wall-model stresses at the rough walls, from u and v on the SGS grid
    double wall4[4] = {0, 0, 0, 0};
    const bool wall = h->sgs.on && (h->dyn_lo || h->dyn_hi);
    if (wall) {
        const int S1 = h->sgs.P1, S2 = h->sgs.P2;
        std::vector<double> lc(n3), li(n3);
        member_sgs_tables(h, h->member_cs[m], h->member_z0[m], lc.data(), li.data(), wall4);
        double* bu = (double*)h->prog_buf;   // u, then v behind it
        double2* mx = (double2*)h->prog_mixed;
        const long long lay = (long long)S1 * S2;
        BLD_TRY(physical_field_dev(h, m, 0, S1, S2, mx, bu));
        BLD_TRY(physical_field_dev(h, m, 1, S1, S2, mx, bu + (long long)n3 * lay));
        if (h->dyn_lo)
            k_wall_stress_mean<<<1, 256, 0, h->stream>>>(bu, bu + (long long)n3 * lay, lay, wall4[2], h->prog_small + 7 * n3);
        if (h->dyn_hi)
            k_wall_stress_mean<<<1, 256, 0, h->stream>>>(bu + (long long)(n3 - 1) * lay, bu + (long long)(2 * n3 - 1) * lay,
                                                        lay, wall4[3], h->prog_small + 7 * n3 + 2);
        CUDA_TRY(cudaGetLastError());
    }
    std::vector<double> r(nsmall);
    CUDA_TRY(cudaMemcpyAsync(r.data(), h->prog_small, nsmall * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    const double L3 = h->cfg.x3_max - h->cfg.x3_min;
    *out = bld_progress{};
    double mke = 0, ke = 0, dtmin = INFINITY;
    for (int z = 0; z < n3; ++z) {
        const double wc = h->tab_dx3c[z] / n3 / L3;   // cweight = dx3(zeta_C) / (n3 L3)
        const double mu = r[(0 * n3 + z) * 2], mv = r[(1 * n3 + z) * 2];
        out->mean_velocity[0] += mu * wc;
        out->mean_velocity[1] += mv * wc;
        mke += mu * mu + mv * mv;
        ke += r[(0 * n3 + z) * 2 + 1] + r[(1 * n3 + z) * 2 + 1];
    }
    for (int z = 0; z < n3 - 1; ++z) {
        const double dxi = h->tab_dx3i[z + 1] / n3;   // interior I node zeta = (z + 1) / n3
        out->mean_velocity[2] += r[(2 * n3 + z) * 2] * dxi / L3;
        const double mw = r[6 * n3 + z];
        dtmin = std::min(dtmin, mw > 0 ? dxi / mw : INFINITY);
    }
    out->mean_ke = mke;
    out->turbulent_ke = ke - mke;
    out->advective_timescale = dtmin;
    out->wall_stress[0][0] = r[7 * n3 + 0];
    out->wall_stress[1][0] = r[7 * n3 + 1];
    out->wall_stress[0][1] = r[7 * n3 + 2];
    out->wall_stress[1][1] = r[7 * n3 + 3];
    out->grid_p1 = P1;
    out->grid_p2 = P2;
    return BLD_OK;
}

static int half_shift(bld_handle* h, double2* dst, const double2* src, int field, double sign) {
    const Geo& g = h->g;
    const int nz = field == 2 ? g.n3 - 1 : g.n3;
    dim3 grid((unsigned)((g.F + 255) / 256), nz);
    k_half_shift<<<grid, 256, 0, h->stream>>>(dst, src, g, h->Pd1, h->Pd2, sign);
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}

int32_t bld_get_field_centered(bld_handle* h, int32_t m, int32_t field, double* values) {
    if (!member_ok(h, m) || field < 0 || field > 2 || !values) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    if (!h->pd_buf) return fail(BLD_ERR_INVALID_CONFIG, "default physical size is not an even 2^a*3^b");
    CUDA_TRY(cudaSetDevice(h->device));
    // shift a copy of the member's field (in the staging buffer) and transform it
    const size_t off = (size_t)m * h->g.mstride + fld_off(h->g, field);
    BLD_TRY(half_shift(h, h->io + off, h->u + off, field, 1.0));
    double2* keep = h->u;
    h->u = h->io;
    const int st = bld_get_field_physical(h, m, field, values);
    h->u = keep;
    return st;
}

int32_t bld_set_field_centered(bld_handle* h, int32_t m, int32_t field, const double* values) {
    BLD_TRY(bld_set_field_physical(h, m, field, values));
    CUDA_TRY(cudaSetDevice(h->device));
    const size_t off = (size_t)m * h->g.mstride + fld_off(h->g, field);
    BLD_TRY(half_shift(h, h->u + off, h->u + off, field, -1.0));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

int32_t bld_profiles_start(bld_handle* h, int32_t on) {
    if (!h) return fail(BLD_ERR_ARGUMENT, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    if (!on) {
        h->prof_on = false;
        return BLD_OK;
    }
    const size_t n = (size_t)h->B * 3 * (h->g.n3 + 1);
    if (!h->prof_acc) {
        BLD_TRY(dalloc(h, (void**)&h->prof_acc, n * sizeof(double)));
        BLD_TRY(dalloc(h, (void**)&h->prof_prev, n * sizeof(double)));
    }
    CUDA_TRY(cudaMemsetAsync(h->prof_acc, 0, n * sizeof(double), h->stream));
    BLD_TRY(enqueue_profile_sample(h, 0.0));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->prof_on = true;
    return BLD_OK;
}

static int profiles_copy(bld_handle* h, int m, const double* src, double* out) {
    if (!member_ok(h, m) || !out) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    if (!h->prof_acc) return fail(BLD_ERR_ARGUMENT, "bld_profiles_start was not called");
    CUDA_TRY(cudaSetDevice(h->device));
    const size_t n = 3 * (size_t)(h->g.n3 + 1);
    CUDA_TRY(cudaMemcpyAsync(out, src + (size_t)m * n, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BLD_OK;
}

int32_t bld_profiles_read(bld_handle* h, int32_t m, double* out) {
    return h ? profiles_copy(h, m, h->prof_acc, out) : fail(BLD_ERR_ARGUMENT, "null handle");
}

int32_t bld_profiles_sample(bld_handle* h, int32_t m, double* out) {
    if (!h) return fail(BLD_ERR_ARGUMENT, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    if (!h->prof_acc) {
        const size_t n = (size_t)h->B * 3 * (h->g.n3 + 1);
        BLD_TRY(dalloc(h, (void**)&h->prof_acc, n * sizeof(double)));
        BLD_TRY(dalloc(h, (void**)&h->prof_prev, n * sizeof(double)));
        CUDA_TRY(cudaMemsetAsync(h->prof_acc, 0, n * sizeof(double), h->stream));
    }
    // a bare sample only replaces the last sample, which is the current state's anyway
    BLD_TRY(enqueue_profile_sample(h, 0.0));
    return profiles_copy(h, m, h->prof_prev, out);
}

int32_t bld_ldlt_solve_device(const double* gamma, const double* beta, void* rhs, int64_t nsys, int32_t n, void* stream) {
    if (!gamma || !beta || !rhs || nsys <= 0 || n < 1) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    return ldlt_launch<double2>(gamma, beta, (double2*)rhs, nsys, n, (cudaStream_t)stream);
}

int32_t bld_ldlt_solve_real_device(const double* gamma, const double* beta, double* rhs, int64_t nsys, int32_t n,
                                   void* stream) {
    if (!gamma || !beta || !rhs || nsys <= 0 || n < 1) return fail(BLD_ERR_ARGUMENT, "invalid argument");
    return ldlt_launch<double>(gamma, beta, rhs, nsys, n, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------- no-alloc projection
// Scratch of bld_project_noalloc: one fixed array per device, whose device
// address host code gets from cudaGetSymbolAddress (the symbol itself is not an
// address in host code).
static __device__ __align__(256) double2 g_noalloc_scratch[BLD_NOALLOC_MAX_VALUES];

namespace {
std::mutex g_noalloc_mutex;
std::map<int, void*> g_noalloc_ptr;  // device ordinal -> device address of g_noalloc_scratch

// The device address of the scratch array on the current device.  Outside a
// stream capture it is looked up on every call, so an address recorded before a
// device reset or under an earlier primary context is never reused; during a
// capture (where the lookup could load the module) the address recorded by an
// earlier call on this device is used.
int noalloc_scratch(cudaStream_t stream, void** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void* ptr = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_noalloc_ptr[dev] = ptr;
    }
    auto it = g_noalloc_ptr.find(dev);
    if (it == g_noalloc_ptr.end())
        return fail(BLD_ERR_ARGUMENT, "bld_project_noalloc: the first call on a device must come before any stream capture");
    *out = it->second;
    return BLD_OK;
}
}  // namespace

extern "C" int32_t bld_project_noalloc(int32_t k1max, int32_t k2max, int32_t n3, const double* gamma,
                                       const double* alpha_c, const double* alpha_i, const double* d1,
                                       const double* d2, double w_lo, double w_hi, void* state, void* stream) {
    if (!gamma || !alpha_c || !alpha_i || !d1 || !d2 || !state) return fail(BLD_ERR_ARGUMENT, "null argument");
    if (k1max < 0 || k2max < 0 || n3 < 3) return fail(BLD_ERR_INVALID_CONFIG, "invalid grid size");
    // the regular projection's check (src/processes/pressure.jl:357)
    if (w_lo != w_hi) return fail(BLD_ERR_UNSUPPORTED_BC, "The mean flow must be equal at both vertical boundaries.");
    // sizes in 64 bits before any product, so that none wraps past the limit
    const long long F = ((long long)k1max + 1) * (2LL * k2max + 1);
    const long long values = F > (long long)BLD_NOALLOC_MAX_VALUES ? F : (long long)n3 * F;
    if (values > (long long)BLD_NOALLOC_MAX_VALUES)
        return fail(BLD_ERR_INVALID_CONFIG,
                    "bld_project_noalloc: n3*(k1max+1)*(2*k2max+1) = %lld exceeds the fixed scratch of %d values",
                    values, BLD_NOALLOC_MAX_VALUES);
    void* scratch = nullptr;
    BLD_TRY(noalloc_scratch((cudaStream_t)stream, &scratch));
    ProjArgs a{};
    a.g.k1max = k1max;
    a.g.k2max = k2max;
    a.g.K1 = k1max + 1;
    a.g.K2 = 2 * k2max + 1;
    a.g.n3 = n3;
    a.g.F = (int)F;
    a.g.mstride = (long long)(3 * n3 - 1) * F;
    a.m0 = 0;
    a.u = (const double2*)state;
    a.out = (double2*)state;
    a.kind = S_NONE;
    a.pressure = 1;
    a.pscr = (double2*)scratch;
    a.gamma = gamma;
    a.alpha_c = alpha_c;
    a.alpha_i = alpha_i;
    a.d1 = d1;
    a.d2 = d2;
    a.w_lo = w_lo;
    a.w_hi = w_hi;
    dim3 grid((unsigned)((F + 127) / 128), 1);
    k_project<<<grid, 128, 0, (cudaStream_t)stream>>>(a);
    CUDA_TRY(cudaGetLastError());
    return BLD_OK;
}
