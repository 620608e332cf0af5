// qg_noalloc.cu -- plaquette/action sums of a caller-owned link table with
// no device allocation at all.
//
// Who needs it: a host program that is not allowed to call cudaMalloc at
// the point where it wants this observable -- for example a driver running
// inside another framework that owns the whole device-memory pool and
// forbids allocations behind its back, or a latency-critical loop in which
// a cudaMalloc/cudaFree pair would synchronise the device and stall work on
// other streams.  Such a caller hands in its own device buffers for the
// input (the link table) and the output (four doubles); the per-block
// partial sums this reduction needs live in a fixed scratch array that is
// part of the library image itself.
//
// The scratch array below is held by every GPU that loads the library,
// for the life of the process.  All calls share it: two calls whose kernels
// run at the same time on the GPU (different streams, no ordering between
// them) race on it and give wrong sums, so callers must order their calls
// (one stream, or events).  Each call writes every slot it later reads, so
// nothing has to start at zero and the contents a previous call left behind
// are never used.
//
// The first call on each device does a one-time set-up with that device
// current: it looks up the device address of the scratch array
// (cudaGetSymbolAddress).  Make that first call before any stream capture.
// Lattices are limited to kMaxBlocks * kTile = 2^24 sites (64^4); larger
// ones are rejected with QG_ERR_ARG before anything is queued.
#include <mutex>

#include "qg_internal.h"

namespace {

constexpr int kTile = 1024;                 // sites per block (256 threads x 4)
constexpr int kThreads = 256;
constexpr int kMaxBlocks = 16384;           // => at most 16384 * 1024 = 2^24 sites (64^4)
constexpr int kComp = 4;                    // spatial, temporal plaquette; spatial, temporal action

// 16384 blocks x 4 doubles = 512 KiB of partial sums
static __device__ __align__(256) double g_plaq_scratch[kMaxBlocks * kComp];

std::mutex g_setup_mutex;
double *g_scratch_ptr[64] = {};             // device address of the scratch, per device ordinal

}  // namespace

namespace qg {

// reference-layout link (SU(N)/suncl/su3_matrix_memory.cl:43-176), promoted
// to FP64 with the third row rebuilt
template <int NC, typename Real>
__device__ __forceinline__ M3<double> ref_link(const Real *tab, uint32_t rowsize, uint32_t site, int mu)
{
    auto at = [&](int plane, int c) { return (double)tab[((size_t)site + (size_t)plane * rowsize) * 4 + c]; };
    M3<double> d;
    if (NC == 3) {
        G3<double> g;
        g.uv1 = { at(mu, 0), at(mu, 1), at(mu, 2), at(mu, 3) };
        g.uv2 = { at(mu + 4, 0), at(mu + 4, 1), at(mu + 4, 2), at(mu + 4, 3) };
        g.uv3 = { at(mu + 8, 0), at(mu + 8, 1), at(mu + 8, 2), at(mu + 8, 3) };
        d = expand(g);
    } else {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) d.m[i][j] = { 0.0, 0.0 };
        double x = at(mu, 0), y = at(mu, 1), z = at(mu, 2), w = at(mu, 3);
        d.m[0][0] = { x, z }; d.m[0][1] = { y, w };
        d.m[1][0] = { -y, w }; d.m[1][1] = { x, -z };
    }
    return d;
}

__device__ __forceinline__ M3<double> mul_d(const M3<double> &u, const M3<double> &v)
{
    M3<double> t;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) t.m[i][j] = dot3(&u.m[i][0], 1, &v.m[0][j], 3);
    return t;
}

// Re Tr(a b c^+ d^+)
__device__ __forceinline__ double retr4_d(const M3<double> &a, const M3<double> &b, const M3<double> &c,
                                          const M3<double> &d)
{
    M3<double> ab = mul_d(a, b), abc;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) abc.m[i][j] = dotc3(&ab.m[i][0], 1, &c.m[j][0], 1);
    double tr = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) tr += dotc3(&abc.m[i][0], 1, &d.m[i][0], 1).re;
    return tr;
}

// the plaquette/action pass of k_plaquette for a reference-layout table;
// block b sums sites [b*kTile, (b+1)*kTile) into scratch[b*4 .. b*4+3]
template <int NC, typename Real>
__global__ void __launch_bounds__(kThreads) k_plaq_ref(const Real *tab, uint32_t rowsize, Geom G, double bet,
                                                       double *scratch)
{
    double v[kComp] = { 0, 0, 0, 0 };
    for (int k = 0; k < kTile / kThreads; k++) {
        uint32_t s = blockIdx.x * kTile + k * kThreads + threadIdx.x;
        if (s >= G.V) break;
        Crd c = lex2crd(G, s);
        Crd nb[4] = { step_plus(G, c, 0), step_plus(G, c, 1), step_plus(G, c, 2), step_plus(G, c, 3) };
        M3<double> own[4];
#pragma unroll
        for (int mu = 0; mu < 4; mu++) own[mu] = ref_link<NC, Real>(tab, rowsize, s, mu);
        double rs = 0, rt = 0;
#pragma unroll
        for (int mu = 0; mu < 3; mu++)
#pragma unroll
            for (int nu = mu + 1; nu < 4; nu++) {
                double r = retr4_d(own[mu], ref_link<NC, Real>(tab, rowsize, crd2lex(G, nb[mu]), nu),
                                   ref_link<NC, Real>(tab, rowsize, crd2lex(G, nb[nu]), mu), own[nu]);
                if (nu == 3) rt += r; else rs += r;
            }
        v[0] += rs; v[1] += rt;
        v[2] += bet * (3.0 * NC - rs);
        v[3] += bet * (3.0 * NC - rt);
    }
    __shared__ double sh[kComp][kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kComp; q++) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < kComp) {
        double x = 0;
        for (int w = 0; w < kThreads / 32; w++) x += sh[threadIdx.x][w];
        scratch[(size_t)blockIdx.x * kComp + threadIdx.x] = x;
    }
}

// fixed-order sum of the block partials into the caller's output
__global__ void __launch_bounds__(1024) k_plaq_ref_final(const double *scratch, uint32_t nblocks, double *out)
{
    __shared__ double sh[32];
    for (int q = 0; q < kComp; q++) {
        double x = 0;
        for (uint32_t b = threadIdx.x; b < nblocks; b += blockDim.x) x += scratch[(size_t)b * kComp + q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            x = sh[threadIdx.x];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (threadIdx.x == 0) out[q] = x;
        }
        __syncthreads();
    }
}

}  // namespace qg

void qg_set_global_error(const std::string &m);

extern "C" int qg_plaquette_noalloc(const void *links, int group, int precision, const int size[4], uint32_t rowsize,
                                    double beta, double *out, void *stream)
{
    using namespace qg;
    if (!links || !out || !size) { qg_set_global_error("null argument"); return QG_ERR_ARG; }
    if (group != 2 && group != 3) { qg_set_global_error("group must be 2 or 3"); return QG_ERR_ARG; }
    if (precision != 0 && precision != 1) { qg_set_global_error("precision must be 0 or 1"); return QG_ERR_ARG; }
    uint64_t V = 1;
    for (int i = 0; i < 4; i++) {
        if (size[i] < 2 || size[i] > 4096) { qg_set_global_error("lattice extents must be in [2, 4096]"); return QG_ERR_ARG; }
        V *= (uint64_t)size[i];
    }
    const uint64_t nblocks = (V + kTile - 1) / kTile;
    if (nblocks > (uint64_t)kMaxBlocks) {
        qg_set_global_error("qg_plaquette_noalloc: lattice of " + std::to_string(V) + " sites exceeds the fixed scratch "
                            "capacity of " + std::to_string((uint64_t)kMaxBlocks * kTile) + " sites (64^4)");
        return QG_ERR_ARG;
    }
    if ((uint64_t)rowsize < V) { qg_set_global_error("rowsize smaller than the number of sites"); return QG_ERR_ARG; }
    // an error left pending by the caller's earlier work is reported, not
    // consumed: the launch checks below read the error state
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        qg_set_global_error(std::string("qg_plaquette_noalloc: a CUDA error was pending before the call: ") +
                            cudaGetErrorString(e));
        return QG_ERR_CUDA;
    }
    // set-up, once per device, with that device current: the device
    // address of the scratch array (the host-side symbol is only a handle).
    // The address is kept for the process: it belongs to the device's
    // primary context and is not valid after cudaDeviceReset.
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { qg_set_global_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e)); return QG_ERR_CUDA; }
    if (dev < 0 || dev >= 64) { qg_set_global_error("device ordinal out of range"); return QG_ERR_ARG; }
    double *scratch;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            double *p = nullptr;
            e = cudaGetSymbolAddress((void **)&p, g_plaq_scratch);
            if (e != cudaSuccess || !p) {
                qg_set_global_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return QG_ERR_CUDA;
            }
            g_scratch_ptr[dev] = p;
        }
        scratch = g_scratch_ptr[dev];
    }
    Geom G = make_geom(size);
    cudaStream_t s = (cudaStream_t)stream;
    const double bet_d = beta / group;
    if (precision) {
        if (group == 3) k_plaq_ref<3, double><<<(unsigned)nblocks, kThreads, 0, s>>>((const double *)links, rowsize, G, bet_d, scratch);
        else k_plaq_ref<2, double><<<(unsigned)nblocks, kThreads, 0, s>>>((const double *)links, rowsize, G, bet_d, scratch);
    } else {
        const double bet_f = (double)(float)bet_d;     // FP32 runs keep BETA/N as a float
        if (group == 3) k_plaq_ref<3, float><<<(unsigned)nblocks, kThreads, 0, s>>>((const float *)links, rowsize, G, bet_f, scratch);
        else k_plaq_ref<2, float><<<(unsigned)nblocks, kThreads, 0, s>>>((const float *)links, rowsize, G, bet_f, scratch);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        k_plaq_ref_final<<<1, 1024, 0, s>>>(scratch, (uint32_t)nblocks, out);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) { qg_set_global_error(std::string("qg_plaquette_noalloc: ") + cudaGetErrorString(e)); return QG_ERR_CUDA; }
    return QG_OK;
}
