// qg_batch.cu -- many independent lattices updated together (a beta scan,
// lattices of different sizes): one launch per phase over all ensembles,
// batched plaquette / Polyakov measurements with per-ensemble
// deterministic reductions, batched reunitarisation, and the whole
// sweep + measurement captured in one CUDA graph.
//
// No counterpart in the reference, which runs one lattice per process.
// Each block of a batched launch finds its ensemble in a prefix table of
// block counts; inside an ensemble the blocks, threads and the per-thread
// work are those of the single-lattice kernels (phase_site, plaq_site,
// poly_site, gs_site, reduce_partials), so ensemble e's chain is
// bit-identical to a single context with the same size, coupling and
// RANDSERIES.
#include <algorithm>
#include <string>
#include <vector>

#include "qg_internal.h"
#include "qg_observe.cuh"
#include "qg_update.cuh"

void qg_set_global_error(const std::string &m);

namespace qg {

struct EnsDesc {
    Geom G;
    void *links;
    const double *params;      // device {BETA/N, 0, 0}
    uint2 key;                 // Philox key (RANDSERIES, constant)
};

// largest e with pre[e] <= b (pre[0] = 0, n entries searched)
__device__ __forceinline__ int find_ensemble(const uint32_t *pre, int n, uint32_t b)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(pre + mid) <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int NC, typename Real, bool OR, int mu, int MINB, bool STAGED>
__global__ void __launch_bounds__(kPhaseBlock, MINB)
k_phase_batch(const EnsDesc *ens, const uint32_t *pre, int n, int parity, const uint64_t *phase_base,
              uint32_t phase_offset, int nhit, int nhitpar)
{
    const int e = find_ensemble(pre, n, blockIdx.x);
    const EnsDesc &d = ens[e];
    const uint32_t t = (blockIdx.x - __ldg(pre + e)) * kPhaseBlock + threadIdx.x;
    const Geom G = d.G;
    if (t >= G.half) return;
    PhaseArgs A;
    A.parity = parity;
    A.dir = mu;
    A.params = d.params;
    A.twist = 0;
    A.nhit = nhit;
    A.nhitpar = nhitpar;
    A.prn_mode = OR ? -1 : 1;
    A.prns = nullptr;
    A.prngstep = 0;
    A.key = d.key;
    A.phase_base = phase_base;
    A.phase_offset = phase_offset;
    A.variant = 0;
    A.t_begin = 0;
    A.t_end = G.half;
    A.t_prn = 0;
    Field<Real> U;
    U.p = reinterpret_cast<typename V4<Real>::T *>(d.links);
    U.pstride = G.pstride;
    if constexpr (STAGED) {
        __shared__ __align__(16) StageBuf sb;
        phase_site<NC, Real, 1, OR, mu, STAGED>(U, G, A, t, &sb);
    } else {
        phase_site<NC, Real, 1, OR, mu, STAGED>(U, G, A, t, nullptr);
    }
}

// ---------------------------------------------- persistent half-sweep
// One launch per parity runs the four directions of that parity over all
// ensembles: the blocks take the 128-link tiles of the batch (tile k of the
// phase's prefix table) from a counter of direction 0 until none is left,
// wait at a grid barrier, go on with direction 1, and so on -- the phases of one
// parity depend on each other (phase (p, nu) reads the links of parity p
// and direction mu that phase (p, mu) wrote), so the barrier stands where
// the per-phase launches had a kernel boundary.  All blocks are resident
// (cooperative launch sized from the occupancy), and every wait is bounded:
// a barrier that does not complete within kBarrierNs sets bar->err and the
// blocks return.  skip_block >= 0 makes that block leave out its arrival at
// the first barrier (a test of the bounded wait).
struct GridBarrier {
    unsigned count, gen, err, pad;
};
constexpr unsigned long long kBarrierNs = 1000000000ull;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// all blocks of the grid; false (block-uniform) when the wait ran out
__device__ bool grid_sync(GridBarrier *bar, bool arrive)
{
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0) {
        const unsigned g = ld_acquire_u32(&bar->gen);
        __threadfence();
        bool last = false;
        if (arrive && atomicAdd(&bar->count, 1u) + 1u == gridDim.x) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicAdd(&bar->gen, 1u);
            last = true;
        }
        if (!last) {
            const unsigned long long t0 = global_ns();
            while (ld_acquire_u32(&bar->gen) == g) {
                if (global_ns() - t0 > kBarrierNs) {
                    atomicOr(&bar->err, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(256);
            }
        }
        __threadfence();
    }
    return __syncthreads_and(ok) != 0;
}

// the tiles of direction mu: one loop per direction, so that each loop is
// compiled with its own register allocation (one loop around a switch over
// the four directions held 160 registers: 3 blocks per SM instead of 5)
template <int NC, typename Real, bool OR, int mu, bool STAGED>
__device__ __forceinline__ void tiles_of_phase(const EnsDesc *ens, const uint32_t *pre, int n, int parity,
                                               const uint64_t *phase_base, uint32_t phase_offset0, int nhit,
                                               int nhitpar, StageBuf *sb, uint32_t ntiles, unsigned *tile_ctr)
{
    // tiles handed out by a counter (zeroed before the launch), so that a
    // block that finishes early takes the next tile as a new block of a
    // per-phase launch would; thread 0 takes the block's next tile when it
    // starts a tile and publishes it after, so the atomic's round trip runs
    // under the tile's work
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    uint32_t tile = s_tile;
    uint32_t next = 0;
    auto advance = [&]() {                            // publish the next tile (every path of the body)
        if (threadIdx.x == 0) s_tile = next;
        __syncthreads();
        return s_tile;
    };
    for (; tile < ntiles; tile = advance()) {
        __syncthreads();                              // every thread has read s_tile
        if (threadIdx.x == 0) next = atomicAdd(tile_ctr, 1u);
        const int e = find_ensemble(pre, n, tile);
        const EnsDesc &d = ens[e];
        const uint32_t t = (tile - __ldg(pre + e)) * kPhaseBlock + threadIdx.x;
        const Geom G = d.G;
        if (t >= G.half) continue;
        PhaseArgs A;
        A.parity = parity;
        A.dir = mu;
        A.params = d.params;
        A.twist = 0;
        A.nhit = nhit;
        A.nhitpar = nhitpar;
        A.prn_mode = OR ? -1 : 1;
        A.prns = nullptr;
        A.prngstep = 0;
        A.key = d.key;
        A.phase_base = phase_base;
        A.phase_offset = phase_offset0 + (uint32_t)mu;
        A.variant = 0;
        A.t_begin = 0;
        A.t_end = G.half;
        A.t_prn = 0;
        Field<Real> U;
        U.p = reinterpret_cast<typename V4<Real>::T *>(d.links);
        U.pstride = G.pstride;
        phase_site<NC, Real, 1, OR, mu, STAGED>(U, G, A, t, sb);
    }
}

template <int NC, typename Real, bool OR, bool STAGED>
__device__ __forceinline__ void half_sweep_body(const EnsDesc *ens, const uint32_t *pre, int n, int parity,
                                                const uint64_t *phase_base, uint32_t phase_offset0, int nhit,
                                                int nhitpar, GridBarrier *bar, int skip_block, StageBuf *sb,
                                                unsigned *tiles)
{
    const uint32_t ntiles = __ldg(pre + n);
    tiles_of_phase<NC, Real, OR, 0, STAGED>(ens, pre, n, parity, phase_base, phase_offset0, nhit, nhitpar, sb, ntiles,
                                            tiles + 0);
    if (!grid_sync(bar, (int)blockIdx.x != skip_block)) return;
    tiles_of_phase<NC, Real, OR, 1, STAGED>(ens, pre, n, parity, phase_base, phase_offset0, nhit, nhitpar, sb, ntiles,
                                            tiles + 1);
    if (!grid_sync(bar, true)) return;
    tiles_of_phase<NC, Real, OR, 2, STAGED>(ens, pre, n, parity, phase_base, phase_offset0, nhit, nhitpar, sb, ntiles,
                                            tiles + 2);
    if (!grid_sync(bar, true)) return;
    tiles_of_phase<NC, Real, OR, 3, STAGED>(ens, pre, n, parity, phase_base, phase_offset0, nhit, nhitpar, sb, ntiles,
                                            tiles + 3);
}

template <int NC, typename Real, bool OR, int MINB, bool STAGED>
__global__ void __launch_bounds__(kPhaseBlock, MINB)
k_half_sweep_batch(const EnsDesc *ens, const uint32_t *pre, int n, int parity, const uint64_t *phase_base,
                   uint32_t phase_offset0, int nhit, int nhitpar, GridBarrier *bar, int skip_block, unsigned *tiles)
{
    if constexpr (STAGED) {
        __shared__ __align__(16) StageBuf sb;
        half_sweep_body<NC, Real, OR, STAGED>(ens, pre, n, parity, phase_base, phase_offset0, nhit, nhitpar, bar,
                                              skip_block, &sb, tiles);
    } else {
        half_sweep_body<NC, Real, OR, STAGED>(ens, pre, n, parity, phase_base, phase_offset0, nhit, nhitpar, bar,
                                              skip_block, nullptr, tiles);
    }
}

template <int NC, typename Real>
__global__ void __launch_bounds__(256) k_plaq_batch(const EnsDesc *ens, const uint32_t *pre, int n, double *partials)
{
    const int e = find_ensemble(pre, n, blockIdx.x);
    const EnsDesc &d = ens[e];
    const Geom G = d.G;
    const uint32_t s = (blockIdx.x - __ldg(pre + e)) * 256 + threadIdx.x;
    Field<Real> U;
    U.p = reinterpret_cast<typename V4<Real>::T *>(d.links);
    U.pstride = G.pstride;
    double v[4] = { 0, 0, 0, 0 };
    if (s < G.V) plaq_site<NC, Real>(U, G, d.params, 0, s, v);
    block_sum_store<4>(v, partials, blockIdx.x);
}

// k_plaq_batch with FP32 products (FP32 links): the sums of k_plaquette_f32
template <int NC>
__global__ void __launch_bounds__(256) k_plaq_batch_f32(const EnsDesc *ens, const uint32_t *pre, int n,
                                                         double *partials)
{
    const int e = find_ensemble(pre, n, blockIdx.x);
    const EnsDesc &d = ens[e];
    const Geom G = d.G;
    const uint32_t s = (blockIdx.x - __ldg(pre + e)) * 256 + threadIdx.x;
    Field<float> U;
    U.p = reinterpret_cast<float4 *>(d.links);
    U.pstride = G.pstride;
    double v[4] = { 0, 0, 0, 0 };
    if (s < G.V) plaq_site_f32<NC>(U, G, d.params, 0, lex2crd(G, s), v);
    block_sum_store<4>(v, partials, blockIdx.x);
}

template <int NC, typename Real>
__global__ void __launch_bounds__(256) k_poly_batch(const EnsDesc *ens, const uint32_t *pre, int n, double *partials)
{
    const int e = find_ensemble(pre, n, blockIdx.x);
    const EnsDesc &d = ens[e];
    const Geom G = d.G;
    const uint32_t i = (blockIdx.x - __ldg(pre + e)) * 256 + threadIdx.x;
    Field<Real> U;
    U.p = reinterpret_cast<typename V4<Real>::T *>(d.links);
    U.pstride = G.pstride;
    double v[4] = { 0, 0, 0, 0 };
    if (i < (uint32_t)G.n[0] * G.n[1] * G.n[2]) poly_site<NC, Real>(U, G, i, v);
    block_sum_store<4>(v, partials, blockIdx.x);
}

// block e: ensemble e's plaquette and Polyakov partials -> 8 sums in the
// series slot of measurement *counter; past the series' capacity the sums
// are dropped and block 0 counts the drop in *overflow
__global__ void __launch_bounds__(1024) k_reduce_batch(const double *pl_partials, const double *po_partials,
                                                       const uint32_t *pre_pl, const uint32_t *pre_po, int n,
                                                       const uint64_t *counter, uint64_t capacity, double *series,
                                                       uint32_t *overflow)
{
    const int e = blockIdx.x;
    const uint64_t m = *counter;
    double *out = (m < capacity) ? series + ((size_t)m * n + e) * 8 : nullptr;
    if (!out && threadIdx.x == 0 && e == 0) atomicAdd(overflow, 1u);
    reduce_partials(pl_partials + (size_t)pre_pl[e] * 4, pre_pl[e + 1] - pre_pl[e], 4, out);
    reduce_partials(po_partials + (size_t)pre_po[e] * 4, pre_po[e + 1] - pre_po[e], 4, out ? out + 4 : nullptr);
}

template <int NC, typename Real, typename Acc>
__global__ void k_gs_batch(const EnsDesc *ens, const uint32_t *pre, int n)
{
    const int e = find_ensemble(pre, n, blockIdx.x);
    const EnsDesc &d = ens[e];
    const Geom G = d.G;
    const uint32_t i = (blockIdx.x - __ldg(pre + e)) * 128 + threadIdx.x;
    if (i >= 2 * G.cb) return;
    const uint32_t h = (i < G.cb) ? i : i - G.cb;
    if (h >= G.half) return;
    Field<Real> U;
    U.p = reinterpret_cast<typename V4<Real>::T *>(d.links);
    U.pstride = G.pstride;
    gs_site<NC, Real, Acc>(U, i);
}

}  // namespace qg

using namespace qg;

struct qg_batch {
    qg_config cfg;
    int n = 0;
    std::vector<Geom> G;
    std::vector<size_t> offset;        // byte offset of each ensemble's field
    std::vector<qg_ensemble> ens;
    std::vector<uint32_t> pre_phase, pre_plaq, pre_poly, pre_gs;   // host copies of the prefix tables
    size_t field_bytes = 0;
    void *links = nullptr;
    double *d_params = nullptr;        // 4 doubles per ensemble
    EnsDesc *d_ens = nullptr;
    uint32_t *d_pre = nullptr;         // the 4 prefix tables, n + 1 entries each
    double *d_pl = nullptr, *d_po = nullptr;
    uint64_t *d_phase = nullptr, *d_meas = nullptr;
    uint32_t *d_overflow = nullptr;
    double *d_series = nullptr;
    uint64_t capacity = 0;
    uint64_t measurements = 0, sweeps_done = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph[4] = { nullptr, nullptr, nullptr, nullptr };   // [measure * 2 + reunit]
    int shape_hb = 4, shape_or = 4;    // phase-kernel launch shapes (qg_batch_tune)
    bool persistent = false;           // one launch per half-sweep (qg_batch_set_persistent)
    bool plaq_fp32 = false;            // FP32-product plaquette (qg_batch_set_measure_products)
    GridBarrier *d_bar = nullptr;
    unsigned *d_tiles = nullptr;       // the persistent half-sweep's tile counters, one per direction
};

namespace {

int bfail(const std::string &m, int code = QG_ERR_ARG)
{
    qg_set_global_error(m);
    return code;
}
int bcuda(cudaError_t e, const char *what)
{
    cudaGetLastError();   // reported here; not left pending for the next launch check
    return bfail(std::string(what) + ": " + cudaGetErrorString(e), QG_ERR_CUDA);
}
#define QB_CK(x, what)                                   \
    do {                                                 \
        cudaError_t e_ = (x);                            \
        if (e_ != cudaSuccess) return bcuda(e_, what);   \
    } while (0)

template <typename Real>
cudaError_t launch_phase_batch(qg_batch *b, int parity, int mu, bool OR, uint32_t offset)
{
    const unsigned nb = b->pre_phase[b->n];
    const uint32_t *pre = b->d_pre;
    const int g = b->cfg.group, nh = b->cfg.nhit, np = b->cfg.nhitpar;
    constexpr bool F32 = sizeof(Real) == 4;
    cudaStream_t s = b->stream;
    // the single-lattice launch shapes 0-4 (qg_tune): 0 registers, 1 / 2 the
    // same held to 5 / 6 blocks per SM, 3 / 4 staple staged through shared
    // memory (SU(3) FP32; elsewhere shapes 0 / 1)
    const int shape = OR ? b->shape_or : b->shape_hb;
#define QB_K(NC, OR_, MU, MB, ST) \
    k_phase_batch<NC, Real, OR_, MU, MB, ST><<<nb, kPhaseBlock, 0, s>>>(b->d_ens, pre, b->n, parity, b->d_phase, offset, nh, np)
#define QB_L(NC, OR_, MU)                                          \
    do {                                                           \
        constexpr bool kSt = NC == 3 && F32;                       \
        if (shape == 1) QB_K(NC, OR_, MU, 5, false);               \
        else if (shape == 2) QB_K(NC, OR_, MU, 6, false);          \
        else if (shape == 3) QB_K(NC, OR_, MU, 0, kSt);            \
        else if (shape == 4) QB_K(NC, OR_, MU, 5, kSt);            \
        else QB_K(NC, OR_, MU, 0, false);                          \
    } while (0)
#define QB_MU(NC, OR_)                               \
    do {                                             \
        switch (mu) {                                \
        case 0: QB_L(NC, OR_, 0); break;             \
        case 1: QB_L(NC, OR_, 1); break;             \
        case 2: QB_L(NC, OR_, 2); break;             \
        default: QB_L(NC, OR_, 3); break;            \
        }                                            \
    } while (0)
    if (g == 3) { if (OR) QB_MU(3, true); else QB_MU(3, false); }
    else { if (OR) QB_MU(2, true); else QB_MU(2, false); }
#undef QB_MU
#undef QB_L
#undef QB_K
    return cudaGetLastError();
}

cudaError_t phase_batch(qg_batch *b, int parity, int mu, bool OR, uint32_t offset)
{
    return b->cfg.precision ? launch_phase_batch<double>(b, parity, mu, OR, offset)
                            : launch_phase_batch<float>(b, parity, mu, OR, offset);
}

// one cooperative launch of the persistent half-sweep: as many blocks as
// are resident at once (at most one per tile)
template <typename KernelT>
cudaError_t launch_half(qg_batch *b, KernelT kern, int parity, uint32_t offset0, int skip_block)
{
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPhaseBlock, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const unsigned ntiles = b->pre_phase[b->n];
    const unsigned grid = std::min<unsigned>((unsigned)(sms * per_sm), ntiles);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kPhaseBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = b->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if ((e = cudaMemsetAsync(b->d_tiles, 0, 4 * sizeof(unsigned), b->stream)) != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, kern, (const EnsDesc *)b->d_ens, (const uint32_t *)b->d_pre, b->n, parity,
                              (const uint64_t *)b->d_phase, offset0, b->cfg.nhit, b->cfg.nhitpar, b->d_bar,
                              skip_block, b->d_tiles);
}

template <typename Real>
cudaError_t half_sweep_T(qg_batch *b, int parity, bool OR, uint32_t offset0, int skip_block)
{
    constexpr bool F32 = sizeof(Real) == 4;
    const int shape = OR ? b->shape_or : b->shape_hb;
    const bool g3 = b->cfg.group == 3;
    // shapes as in launch_phase_batch: 1 / 2 hold 5 / 6 blocks per SM, 3 / 4
    // stage the staple (SU(3) FP32)
#define QB_H(NC, OR_, MB, ST) return launch_half(b, k_half_sweep_batch<NC, Real, OR_, MB, ST>, parity, offset0, skip_block)
#define QB_HS(NC, OR_)                                                     \
    do {                                                                   \
        constexpr bool kSt = NC == 3 && F32;                               \
        if (shape == 1) QB_H(NC, OR_, 5, false);                           \
        else if (shape == 2) QB_H(NC, OR_, 6, false);                      \
        else if (shape == 3) QB_H(NC, OR_, 0, kSt);                        \
        else if (shape == 4) QB_H(NC, OR_, 5, kSt);                        \
        else QB_H(NC, OR_, 0, false);                                      \
    } while (0)
    if (g3) { if (OR) QB_HS(3, true); else QB_HS(3, false); }
    else { if (OR) QB_HS(2, true); else QB_HS(2, false); }
#undef QB_HS
#undef QB_H
}

cudaError_t half_sweep(qg_batch *b, int parity, bool OR, uint32_t offset0, int skip_block = -1)
{
    return b->cfg.precision ? half_sweep_T<double>(b, parity, OR, offset0, skip_block)
                            : half_sweep_T<float>(b, parity, OR, offset0, skip_block);
}

cudaError_t gs_batch(qg_batch *b)
{
    const unsigned nb = b->pre_gs[b->n];
    const uint32_t *pre = b->d_pre + 3 * (b->n + 1);
    cudaStream_t s = b->stream;
    const int g = b->cfg.group;
    if (b->cfg.precision) {
        if (g == 3) k_gs_batch<3, double, double><<<nb, 128, 0, s>>>(b->d_ens, pre, b->n);
        else k_gs_batch<2, double, double><<<nb, 128, 0, s>>>(b->d_ens, pre, b->n);
    } else if (b->cfg.reunit_fp64) {
        if (g == 3) k_gs_batch<3, float, double><<<nb, 128, 0, s>>>(b->d_ens, pre, b->n);
        else k_gs_batch<2, float, double><<<nb, 128, 0, s>>>(b->d_ens, pre, b->n);
    } else {
        if (g == 3) k_gs_batch<3, float, float><<<nb, 128, 0, s>>>(b->d_ens, pre, b->n);
        else k_gs_batch<2, float, float><<<nb, 128, 0, s>>>(b->d_ens, pre, b->n);
    }
    return cudaGetLastError();
}

cudaError_t measure_batch(qg_batch *b)
{
    const uint32_t *pre_pl = b->d_pre + 1 * (b->n + 1), *pre_po = b->d_pre + 2 * (b->n + 1);
    const unsigned npl = b->pre_plaq[b->n], npo = b->pre_poly[b->n];
    cudaStream_t s = b->stream;
    const int g = b->cfg.group;
    if (b->cfg.precision) {
        if (g == 3) {
            k_plaq_batch<3, double><<<npl, 256, 0, s>>>(b->d_ens, pre_pl, b->n, b->d_pl);
            k_poly_batch<3, double><<<npo, 256, 0, s>>>(b->d_ens, pre_po, b->n, b->d_po);
        } else {
            k_plaq_batch<2, double><<<npl, 256, 0, s>>>(b->d_ens, pre_pl, b->n, b->d_pl);
            k_poly_batch<2, double><<<npo, 256, 0, s>>>(b->d_ens, pre_po, b->n, b->d_po);
        }
    } else {
        if (g == 3) {
            if (b->plaq_fp32) k_plaq_batch_f32<3><<<npl, 256, 0, s>>>(b->d_ens, pre_pl, b->n, b->d_pl);
            else k_plaq_batch<3, float><<<npl, 256, 0, s>>>(b->d_ens, pre_pl, b->n, b->d_pl);
            k_poly_batch<3, float><<<npo, 256, 0, s>>>(b->d_ens, pre_po, b->n, b->d_po);
        } else {
            if (b->plaq_fp32) k_plaq_batch_f32<2><<<npl, 256, 0, s>>>(b->d_ens, pre_pl, b->n, b->d_pl);
            else k_plaq_batch<2, float><<<npl, 256, 0, s>>>(b->d_ens, pre_pl, b->n, b->d_pl);
            k_poly_batch<2, float><<<npo, 256, 0, s>>>(b->d_ens, pre_po, b->n, b->d_po);
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_reduce_batch<<<b->n, 1024, 0, s>>>(b->d_pl, b->d_po, pre_pl, pre_po, b->n, b->d_meas, b->capacity,
                                         b->d_series, b->d_overflow);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_add_u64(b->d_meas, 1, s);
}

// one sweep of every ensemble in the single-lattice order (odd X..T, even
// X..T heatbath, n_or overrelaxation sweeps, Gram-Schmidt when due), then
// optionally one measurement
cudaError_t enqueue_batch_sweep(qg_batch *b, bool reunit, bool measure)
{
    cudaError_t e;
    const int par_order[2] = { 1, 0 };
    uint32_t hb = 0;
    if (b->persistent) {
        for (int pi = 0; pi < 2; pi++) {
            if ((e = half_sweep(b, par_order[pi], false, hb)) != cudaSuccess) return e;
            hb += 4;
        }
        for (int k = 0; k < b->cfg.n_or; k++)
            for (int pi = 0; pi < 2; pi++)
                if ((e = half_sweep(b, par_order[pi], true, 0)) != cudaSuccess) return e;
    } else {
        for (int pi = 0; pi < 2; pi++)
            for (int mu = 0; mu < 4; mu++) {
                if ((e = phase_batch(b, par_order[pi], mu, false, hb)) != cudaSuccess) return e;
                hb++;
            }
        for (int k = 0; k < b->cfg.n_or; k++)
            for (int pi = 0; pi < 2; pi++)
                for (int mu = 0; mu < 4; mu++)
                    if ((e = phase_batch(b, par_order[pi], mu, true, 0)) != cudaSuccess) return e;
    }
    if ((e = launch_add_u64(b->d_phase, hb, b->stream)) != cudaSuccess) return e;
    if (reunit && (e = gs_batch(b)) != cudaSuccess) return e;
    if (measure && (e = measure_batch(b)) != cudaSuccess) return e;
    return cudaSuccess;
}

void destroy_batch_graphs(qg_batch *b)
{
    for (auto &g : b->graph)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

}  // namespace

extern "C" int qg_batch_destroy(qg_batch *b)
{
    if (!b) return QG_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    destroy_batch_graphs(b);
    cudaFree(b->links);
    cudaFree(b->d_params);
    cudaFree(b->d_ens);
    cudaFree(b->d_pre);
    cudaFree(b->d_pl);
    cudaFree(b->d_po);
    cudaFree(b->d_phase);
    cudaFree(b->d_overflow);
    cudaFree(b->d_series);
    cudaFree(b->d_bar);
    cudaFree(b->d_tiles);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return QG_OK;
}

extern "C" int qg_batch_create(const qg_config *common, const qg_ensemble *ens, int n, int max_measurements,
                               qg_batch **out)
{
    if (!common || !ens || !out || n < 1) return bfail("qg_batch_create: bad argument");
    *out = nullptr;
    const qg_config &c = *common;
    if (c.group != 2 && c.group != 3) return bfail("group must be 2 or 3");
    if (c.precision != 0 && c.precision != 1) return bfail("precision must be 0 or 1");
    if (c.prng != QG_PRNG_PHILOX) return bfail("batched ensembles use the Philox stream (QG_PRNG_PHILOX)");
    if (c.nhit < 1 || c.nhitpar < 1 || c.n_or < 0 || max_measurements < 0) return bfail("bad NHIT/NHITPar/n_or");
    const size_t real = c.precision ? 8 : 4, planes = (c.group == 3) ? 12 : 4;
    for (int e = 0; e < n; e++) {
        const int *L = ens[e].size;
        for (int i = 0; i < 4; i++)
            if (L[i] < 2 || L[i] > 1024) return bfail("ensemble " + std::to_string(e) + ": extents must be in [2, 1024]");
        if (L[1] % 2) return bfail("ensemble " + std::to_string(e) + ": N2 must be even");
        if ((uint64_t)L[0] * L[1] * L[2] * L[3] >= (1ull << 31)) return bfail("ensemble too large");
        if (ens[e].randseries == 0) return bfail("RANDSERIES 0 is not reproducible");
    }
    qg_batch *b = new qg_batch;
    b->cfg = c;
    b->n = n;
    b->capacity = (uint64_t)max_measurements;
    b->ens.assign(ens, ens + n);
    size_t off = 0;
    b->pre_phase.assign(1, 0); b->pre_plaq.assign(1, 0); b->pre_poly.assign(1, 0); b->pre_gs.assign(1, 0);
    for (int e = 0; e < n; e++) {
        Geom G = make_geom(ens[e].size);
        b->G.push_back(G);
        b->offset.push_back(off);
        off += ((planes * G.pstride * 4 * real) + 255) / 256 * 256;
        b->pre_phase.push_back(b->pre_phase.back() + (G.half + kPhaseBlock - 1) / kPhaseBlock);
        b->pre_plaq.push_back(b->pre_plaq.back() + plaq_blocks(G));
        b->pre_poly.push_back(b->pre_poly.back() + poly_blocks(G));
        b->pre_gs.push_back(b->pre_gs.back() + (2 * G.cb + 127) / 128);
    }
    b->field_bytes = off;
    auto fail_free = [&](cudaError_t e, const char *what) {
        qg_batch_destroy(b);
        return bcuda(e, what);
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail_free(e, "stream");
    if ((e = cudaMalloc(&b->links, off)) != cudaSuccess) return fail_free(e, "links");
    if ((e = cudaMemset(b->links, 0, off)) != cudaSuccess) return fail_free(e, "links clear");
    if ((e = cudaMalloc(&b->d_params, sizeof(double) * 4 * n)) != cudaSuccess) return fail_free(e, "params");
    if ((e = cudaMalloc(&b->d_ens, sizeof(EnsDesc) * n)) != cudaSuccess) return fail_free(e, "descriptors");
    if ((e = cudaMalloc(&b->d_pre, sizeof(uint32_t) * 4 * (n + 1))) != cudaSuccess) return fail_free(e, "prefix");
    if ((e = cudaMalloc(&b->d_pl, sizeof(double) * 4 * (b->pre_plaq[n] + 1))) != cudaSuccess)
        return fail_free(e, "partials");
    if ((e = cudaMalloc(&b->d_po, sizeof(double) * 4 * (b->pre_poly[n] + 1))) != cudaSuccess)
        return fail_free(e, "partials");
    if ((e = cudaMalloc(&b->d_phase, sizeof(uint64_t) * 2)) != cudaSuccess) return fail_free(e, "counters");
    b->d_meas = b->d_phase + 1;
    if ((e = cudaMalloc(&b->d_overflow, sizeof(uint32_t))) != cudaSuccess) return fail_free(e, "overflow");
    if ((e = cudaMalloc(&b->d_bar, sizeof(GridBarrier))) != cudaSuccess) return fail_free(e, "barrier");
    if ((e = cudaMemset(b->d_bar, 0, sizeof(GridBarrier))) != cudaSuccess) return fail_free(e, "barrier clear");
    if ((e = cudaMalloc(&b->d_tiles, 4 * sizeof(unsigned))) != cudaSuccess) return fail_free(e, "tile counters");
    if ((e = cudaMalloc(&b->d_series, sizeof(double) * 8 * n * (b->capacity ? b->capacity : 1))) != cudaSuccess)
        return fail_free(e, "series");
    std::vector<double> params(4 * (size_t)n, 0.0);
    std::vector<EnsDesc> desc(n);
    for (int k = 0; k < n; k++) {
        params[4 * k] = ens[k].beta / c.group;
        desc[k].G = b->G[k];
        desc[k].links = (char *)b->links + b->offset[k];
        desc[k].params = b->d_params + 4 * k;
        desc[k].key = make_uint2(ens[k].randseries, 0x5D3E1A27u);   // the single-context Philox key
    }
    std::vector<uint32_t> pre;
    for (auto *v : { &b->pre_phase, &b->pre_plaq, &b->pre_poly, &b->pre_gs }) pre.insert(pre.end(), v->begin(), v->end());
    if ((e = cudaMemcpy(b->d_params, params.data(), params.size() * sizeof(double), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(b->d_ens, desc.data(), desc.size() * sizeof(EnsDesc), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(b->d_pre, pre.data(), pre.size() * sizeof(uint32_t), cudaMemcpyHostToDevice)) ||
        (e = cudaMemset(b->d_phase, 0, 2 * sizeof(uint64_t))) || (e = cudaMemset(b->d_overflow, 0, sizeof(uint32_t))))
        return fail_free(e, "batch upload");
    *out = b;
    return QG_OK;
}

extern "C" int qg_batch_init(qg_batch *b, int start)
{
    if (!b) return QG_ERR_ARG;
    int kind;
    switch (start) {
    case QG_START_COLD: kind = INIT_COLD; break;
    case QG_START_HOT: kind = INIT_HOT_PHILOX; break;
    case QG_START_HAAR: kind = INIT_HAAR; break;
    default: return bfail("batched ensembles start cold, hot or Haar");
    }
    for (int e = 0; e < b->n; e++)
        QB_CK(launch_init(b->G[e], (char *)b->links + b->offset[e], b->cfg.group, b->cfg.precision, kind, 0, nullptr,
                          0, make_uint2(b->ens[e].randseries, 0x5D3E1A27u), b->stream), "init");
    QB_CK(cudaMemsetAsync(b->d_phase, 0, 2 * sizeof(uint64_t), b->stream), "counters");
    QB_CK(cudaMemsetAsync(b->d_overflow, 0, sizeof(uint32_t), b->stream), "overflow");
    QB_CK(cudaStreamSynchronize(b->stream), "init sync");
    b->measurements = 0;
    b->sweeps_done = 0;
    return QG_OK;
}

extern "C" int qg_batch_set_shapes(qg_batch *b, int heatbath_shape, int overrelax_shape)
{
    if (!b) return QG_ERR_ARG;
    if (heatbath_shape < 0 || heatbath_shape >= QG_BATCH_SHAPES || overrelax_shape < 0 ||
        overrelax_shape >= QG_BATCH_SHAPES)
        return bfail("batched launch shape out of range [0, QG_BATCH_SHAPES)");
    b->shape_hb = heatbath_shape;
    b->shape_or = overrelax_shape;
    destroy_batch_graphs(b);
    return QG_OK;
}

extern "C" int qg_batch_set_shape(qg_batch *b, int shape)
{
    return qg_batch_set_shapes(b, shape, shape);
}

extern "C" int qg_batch_get_shapes(qg_batch *b, int *heatbath_shape, int *overrelax_shape)
{
    if (!b || !heatbath_shape || !overrelax_shape) return QG_ERR_ARG;
    *heatbath_shape = b->shape_hb;
    *overrelax_shape = b->shape_or;
    return QG_OK;
}

// times every launch shape of the batched heatbath and overrelaxation
// phase launches on the live fields (restored afterwards; the Philox phase
// counter is only read by the phase kernels) and keeps the fastest per kind
extern "C" int qg_batch_tune(qg_batch *b, int reps, float *times_ms)
{
    if (!b) return QG_ERR_ARG;
    if (reps < 1) reps = 4;
    void *backup = nullptr;
    QB_CK(cudaMallocAsync(&backup, b->field_bytes, b->stream), "tune backup");
    {
        cudaError_t eb = cudaMemcpyAsync(backup, b->links, b->field_bytes, cudaMemcpyDeviceToDevice, b->stream);
        if (eb != cudaSuccess) {
            cudaFreeAsync(backup, b->stream);
            return bcuda(eb, "tune backup copy");
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int keep[2] = { b->shape_hb, b->shape_or };
    float best[2] = { 1e30f, 1e30f };
    int arg[2] = { keep[0], keep[1] };
    cudaError_t e = cudaSuccess;
    for (int v = 0; v < QG_BATCH_SHAPES && e == cudaSuccess; v++)
        for (int kind = 0; kind < 2 && e == cudaSuccess; kind++) {
            b->shape_hb = b->shape_or = v;
            // one untimed launch, then reps timed ones over the 8 phase classes
            for (int r = -1; r < reps && e == cudaSuccess; r++) {
                if (r == 0) cudaEventRecord(e0, b->stream);
                e = phase_batch(b, (r + 1) & 1, ((r + 1) >> 1) & 3, kind == 1, 0);
            }
            if (e != cudaSuccess) break;
            cudaEventRecord(e1, b->stream);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= reps;
            if (times_ms) times_ms[2 * v + kind] = ms;
            if (ms < best[kind]) { best[kind] = ms; arg[kind] = v; }
        }
    cudaError_t er = cudaMemcpyAsync(b->links, backup, b->field_bytes, cudaMemcpyDeviceToDevice, b->stream);
    cudaFreeAsync(backup, b->stream);
    cudaError_t es = cudaStreamSynchronize(b->stream);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        b->shape_hb = keep[0];
        b->shape_or = keep[1];
        return bcuda(e, "tune launch");
    }
    if (er != cudaSuccess) return bcuda(er, "tune restore");
    if (es != cudaSuccess) return bcuda(es, "tune sync");
    b->shape_hb = arg[0];
    b->shape_or = arg[1];
    destroy_batch_graphs(b);
    return QG_OK;
}

extern "C" int qg_batch_run(qg_batch *b, int nsweeps, int measure_every)
{
    if (!b || nsweeps < 0 || measure_every < 0) return QG_ERR_ARG;
    const int every = b->cfg.reunit_every;
    for (int k = 0; k < nsweeps; k++) {
        const bool reunit = every > 0 && ((b->sweeps_done + 1) % (uint64_t)every) == 0;
        const bool measure = measure_every > 0 && ((b->sweeps_done + 1) % (uint64_t)measure_every) == 0;
        const int which = (measure ? 2 : 0) + (reunit ? 1 : 0);
        if (!b->graph[which]) {
            cudaGraph_t g = nullptr;
            QB_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            cudaError_t e = enqueue_batch_sweep(b, reunit, measure);
            cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
            if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return bcuda(e, "batch sweep capture"); }
            if (e2 != cudaSuccess) return bcuda(e2, "end capture");
            e = cudaGraphInstantiate(&b->graph[which], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return bcuda(e, "graph instantiate");
        }
        QB_CK(cudaGraphLaunch(b->graph[which], b->stream), "graph launch");
        b->sweeps_done++;
        if (measure) b->measurements++;
    }
    return QG_OK;
}

// a grid barrier of the persistent half-sweep that ran out: reported once,
// the barrier state reset (the fields are not trustworthy afterwards)
static int barrier_check(qg_batch *b)
{
    GridBarrier h;
    QB_CK(cudaMemcpy(&h, b->d_bar, sizeof(h), cudaMemcpyDeviceToHost), "barrier read");
    if (h.err) {
        QB_CK(cudaMemset(b->d_bar, 0, sizeof(GridBarrier)), "barrier reset");
        return bfail("a grid barrier of the persistent half-sweep ran out (fields not updated consistently)",
                     QG_ERR_CUDA);
    }
    return QG_OK;
}

extern "C" int qg_batch_sync(qg_batch *b)
{
    if (!b) return QG_ERR_ARG;
    QB_CK(cudaStreamSynchronize(b->stream), "batch sync");
    return barrier_check(b);
}

extern "C" int qg_batch_set_persistent(qg_batch *b, int enable)
{
    if (!b) return QG_ERR_ARG;
    b->persistent = enable != 0;
    destroy_batch_graphs(b);
    return QG_OK;
}

extern "C" int qg_batch_set_measure_products(qg_batch *b, int fp32)
{
    if (!b) return QG_ERR_ARG;
    b->plaq_fp32 = fp32 != 0;
    destroy_batch_graphs(b);
    return QG_OK;
}

extern "C" int qg_batch_barrier_test(qg_batch *b, int skip_block)
{
    if (!b || skip_block < 0) return QG_ERR_ARG;
    QB_CK(cudaStreamSynchronize(b->stream), "batch sync");
    QB_CK(half_sweep(b, 1, false, 0, skip_block), "half sweep");
    QB_CK(cudaStreamSynchronize(b->stream), "batch sync");
    return barrier_check(b);
}

extern "C" int qg_batch_get_stream(qg_batch *b, void **stream)
{
    if (!b || !stream) return QG_ERR_ARG;
    *stream = (void *)b->stream;
    return QG_OK;
}

extern "C" int qg_batch_series(qg_batch *b, double *out, uint64_t max_measurements, uint64_t *n_measurements)
{
    if (!b || !n_measurements) return QG_ERR_ARG;
    QB_CK(cudaStreamSynchronize(b->stream), "batch sync");
    if (int r = barrier_check(b)) return r;
    uint32_t ovf = 0;
    QB_CK(cudaMemcpy(&ovf, b->d_overflow, sizeof(ovf), cudaMemcpyDeviceToHost), "overflow read");
    const uint64_t have = b->measurements < b->capacity ? b->measurements : b->capacity;
    *n_measurements = have;
    if (out) {
        const uint64_t m = have < max_measurements ? have : max_measurements;
        if (m) QB_CK(cudaMemcpy(out, b->d_series, sizeof(double) * 8 * b->n * m, cudaMemcpyDeviceToHost), "series read");
    }
    if (ovf) return bfail("batched series overflowed its capacity of " + std::to_string(b->capacity) +
                          " measurements (" + std::to_string(ovf) + " dropped)", QG_ERR_STATE);
    return QG_OK;
}

extern "C" int qg_batch_links_download(qg_batch *b, int e, void *host)
{
    if (!b || !host || e < 0 || e >= b->n) return QG_ERR_ARG;
    const Geom &G = b->G[e];
    const qg_config &c = b->cfg;
    const uint32_t a = c.row_align > 0 ? (uint32_t)c.row_align : 64;
    const uint32_t rowsize = (G.V + a - 1) / a * a;
    const size_t bytes = (size_t)(c.group == 3 ? 12 : 4) * rowsize * 4 * (c.precision ? 8 : 4);
    void *tmp = nullptr;
    QB_CK(cudaMallocAsync(&tmp, bytes, b->stream), "download staging");
    cudaError_t err = cudaMemsetAsync(tmp, 0, bytes, b->stream);
    if (err == cudaSuccess)
        err = launch_to_ref(G, (char *)b->links + b->offset[e], tmp, c.group, c.precision, rowsize, b->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, b->stream);
    cudaFreeAsync(tmp, b->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(b->stream);
    if (err != cudaSuccess) return bcuda(err, "batch download");
    return QG_OK;
}

extern "C" int qg_batch_info(qg_batch *b, uint64_t *total_sites, uint64_t *sweeps_done, uint64_t *field_bytes)
{
    if (!b) return QG_ERR_ARG;
    uint64_t v = 0;
    for (auto &G : b->G) v += G.V;
    if (total_sites) *total_sites = v;
    if (sweeps_done) *sweeps_done = b->sweeps_done;
    if (field_bytes) *field_bytes = b->field_bytes;
    return QG_OK;
}
