// qg_capi.cu -- the C-ABI of include/qcdgpu_b200.h: context, buffers,
// PRN cadence, sweep graphs and measurements on one CUDA stream.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <string>
#include <algorithm>
#include <vector>

#include "qg_internal.h"

using namespace qg;

struct qg_ctx {
    qg_config cfg;
    Geom G;
    uint32_t rowsize = 0, prngstep = 0, samples = 0;
    int instances = 0;
    size_t link_bytes = 0;
    void *links = nullptr;
    float4 *prns = nullptr;
    float4 *rl_table = nullptr;
    RanluxSplit rl_split = { 1, nullptr, nullptr };   // batches over several threads per generator
    uint32_t *d_seeds = nullptr;
    double *partials = nullptr;
    size_t partials_n = 0;
    double *d_results = nullptr;
    double *h_results = nullptr;    // pinned
    uint64_t *d_phase = nullptr;
    double *d_params = nullptr;     // {BETA/N, PHI, OMEGA, 0}: lattice_parameters
    double *h_params = nullptr;     // pinned staging, kParamSlots x 4 doubles
    cudaEvent_t param_ev[8] = {};   // slot's upload done
    uint32_t param_next = 0;
    // asynchronous measurements: pinned result slots, their copy events and tickets
    double *h_ring = nullptr;       // QG_MEASURE_SLOTS x 8 doubles
    cudaEvent_t ring_ev[QG_MEASURE_SLOTS] = {};
    uint64_t ring_ticket[QG_MEASURE_SLOTS] = {};
    int ring_what[QG_MEASURE_SLOTS] = {};
    uint64_t ticket_next = 1;
    int twist_built = 0;            // twist flag the cached graphs were built with
    int variant_hb = 0, variant_or = 0;   // phase-kernel launch shapes (qg_tune)
    uint64_t phase_counter = 0;     // host mirror of *d_phase
    uint32_t prng_counter = 0;      // RANLUX batches produced
    uint64_t sweeps_done = 0;
    uint2 key = { 0, 0 };
    bool seeded = false;
    cudaStream_t stream = nullptr;
    // sweep graphs: [0] / [1] without / with reunitarisation; with the
    // RANLUX lookahead [2 + 2 v + reunit] for buffer variant v
    cudaGraphExec_t graph[6] = {};
    // RANLUX lookahead: while a sweep runs, a second stream generates the
    // next sweep's 8 batches.  rl_buf[7] is the reference-layout PRN buffer;
    // rl_buf[0..6], rl_buf[8] are allocated on the first RANLUX sweep (if
    // memory allows).  Heatbath phase k of a sweep reads rl_buf[k] (k < 7)
    // or rl_buf[7 + v]; the next sweep's batch k overwrites rl_buf[k] once
    // phase k is done, its last batch goes to rl_buf[8 - v].  prns points at
    // the buffer holding the last batch consumed.
    float4 *rl_buf[9] = {};
    float4 *rl_snap = nullptr;      // generator state as of the last batch consumed
    bool rl_ahead = false;          // the generator has run 8 batches past the consumed ones
    int rl_var = 0;                 // variant v of the next lookahead sweep
    int rl_look = -1;               // lookahead: -1 not set up yet, 0 off / unavailable, 1 ready
    bool rl_look_enabled = true;    // qg_set_prng_lookahead
    // x-slab of a larger lattice (qg_set_slab): this context's x-slices 1..w
    // are the global slices x0 .. x0+w-1, slices 0 and w+1 are halos
    bool slab = false;
    int slab_x0 = 0, slab_n1 = 0;
    unsigned long long *d_bad = nullptr;   // qg_field_check counter
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_phase[8] = {};
    // learned-proposal Metropolis (qg_net_*, qg_mh_*)
    uint16_t *d_netw = nullptr;     // BF16 weights the kernels read
    float *d_master = nullptr, *d_adam_m = nullptr, *d_adam_v = nullptr;
    float *d_grad = nullptr, *d_gpart = nullptr;    // QG_NET_PARAMS + 4 stats; per-block partials
    double *d_wpart = nullptr, *d_wout = nullptr;   // all-loops Wilson measurement (lazy)
    int wpart_rmax = 0;
    double *d_fpart = nullptr, *d_ppart = nullptr, *d_pout = nullptr;   // F_munu / profiles (lazy)
    double *d_sites = nullptr;      // per-site values of the one-pass measurements (lazy)
    unsigned long long *d_mh_acc = nullptr;
    double *d_mh_jump = nullptr;
    unsigned *d_net_err = nullptr;  // set by the network kernels when a tensor-core wait runs out
    float *d_eps = nullptr;         // per-link steps of qg_net_eps (lazy)
    double eps_max = 0.0;
    int adam_t = 0;
    uint64_t train_phase = 0, mh_hits = 0;
    std::string err;
};

static thread_local std::string g_create_err;

// errors of calls without a context (qg_create, the host driver)
void qg_set_global_error(const std::string &m) { g_create_err = m; }

static int fail(qg_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg; else g_create_err = msg;
    return code;
}
static int cuda_fail(qg_ctx *c, cudaError_t e, const char *where)
{
    // the error is reported here: consume it, so that a non-sticky one (a
    // failed allocation) is not picked up by the next launch check as if
    // that kernel had failed
    cudaGetLastError();
    return fail(c, QG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define QG_CK(call, where) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return cuda_fail(c, e_, where); } while (0)

static uint32_t align_up(uint64_t n, uint32_t a) { return (uint32_t)(((n + a - 1) / a) * a); }

extern "C" int qg_default_config(qg_config *cfg)
{
    if (!cfg) return QG_ERR_ARG;
    memset(cfg, 0, sizeof(*cfg));
    cfg->group = 3;
    for (int i = 0; i < 4; i++) cfg->size[i] = 32;
    cfg->precision = 1;
    cfg->start = QG_START_COLD;
    cfg->beta = 6.5;
    cfg->nhit = 10;
    cfg->nhitpar = 1;
    cfg->prng = QG_PRNG_RANLUX;
    cfg->ranlux_nskip = 223;
    cfg->prng_instances = 16384;
    cfg->randseries = 54;
    cfg->row_align = 64;
    cfg->n_or = 0;
    cfg->reunit_every = 1;
    cfg->reunit_fp64 = 0;
    cfg->wilson_r = 7;
    cfg->wilson_t = 2;
    return QG_OK;
}

extern "C" const char *qg_last_error(const qg_ctx *c) { return c ? c->err.c_str() : g_create_err.c_str(); }

static int validate(const qg_config *cfg, std::string &why)
{
    if (cfg->group != 2 && cfg->group != 3) { why = "GROUP must be 2 or 3"; return 0; }
    for (int i = 0; i < 4; i++)
        if (cfg->size[i] < 2 || cfg->size[i] > 4096) { why = "lattice extents must be in [2, 4096]"; return 0; }
    if (cfg->size[1] % 2) { why = "L2 (y extent) must be even for the checkerboard"; return 0; }
    uint64_t V = (uint64_t)cfg->size[0] * cfg->size[1] * cfg->size[2] * cfg->size[3];
    if (V > (1ull << 31)) { why = "lattice volume exceeds 2^31 sites"; return 0; }
    if (cfg->precision != 0 && cfg->precision != 1) { why = "precision must be 0 or 1"; return 0; }
    if (cfg->start < 0 || cfg->start > 3) { why = "unknown start type"; return 0; }
    if (cfg->nhit < 1 || cfg->nhit > 1000) { why = "NHIT must be in [1, 1000]"; return 0; }
    if (cfg->nhitpar < 1 || cfg->nhitpar > 16) { why = "NHITPar must be in [1, 16]"; return 0; }
    if (cfg->prng != QG_PRNG_RANLUX && cfg->prng != QG_PRNG_PHILOX) { why = "unknown PRNG"; return 0; }
    int ns = cfg->ranlux_nskip;
    if (ns != 24 && ns != 48 && ns != 97 && ns != 223 && ns != 389) { why = "RANLUX skip must be 24/48/97/223/389"; return 0; }
    if (cfg->prng_instances < 1 || cfg->prng_instances > (1 << 24)) { why = "PRNG instances out of range"; return 0; }
    if (cfg->randseries == 0) { why = "RANDSERIES 0 (time seeding) is not reproducible; give a seed"; return 0; }
    if (cfg->row_align < 1 || cfg->row_align > 65536) { why = "row alignment out of range"; return 0; }
    if (cfg->n_or < 0 || cfg->n_or > 64) { why = "n_or must be in [0, 64]"; return 0; }
    if (cfg->reunit_every < 0) { why = "reunit_every must be >= 0"; return 0; }
    if (cfg->wilson_r < 1 || cfg->wilson_t < 1) { why = "Wilson loop extents must be >= 1"; return 0; }
    return 1;
}

static void destroy_graphs(qg_ctx *c)
{
    for (auto &g : c->graph)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

static size_t rl_table_bytes(const qg_ctx *c) { return (size_t)7 * c->instances * sizeof(float4); }
static size_t rl_batch_bytes(const qg_ctx *c) { return (size_t)c->instances * c->samples * sizeof(float4); }

// the generator back at the last batch consumed (drops the lookahead
// batches; they are generated again when needed)
static cudaError_t rl_settle(qg_ctx *c)
{
    if (!c->rl_ahead) return cudaSuccess;
    c->rl_ahead = false;
    return cudaMemcpyAsync(c->rl_table, c->rl_snap, rl_table_bytes(c), cudaMemcpyDeviceToDevice, c->stream);
}

static void rl_free_lookahead(qg_ctx *c)
{
    for (int k = 0; k < 9; k++)
        if (k != 7 && c->rl_buf[k]) { cudaFree(c->rl_buf[k]); c->rl_buf[k] = nullptr; }
    if (c->rl_snap) { cudaFree(c->rl_snap); c->rl_snap = nullptr; }
    for (cudaEvent_t &ev : c->ev_phase) if (ev) { cudaEventDestroy(ev); ev = nullptr; }
    if (c->ev_fork) { cudaEventDestroy(c->ev_fork); c->ev_fork = nullptr; }
    if (c->ev_join) { cudaEventDestroy(c->ev_join); c->ev_join = nullptr; }
    if (c->side) { cudaStreamDestroy(c->side); c->side = nullptr; }
}

// buffers, stream and events of the lookahead, once; false (and the plain
// sweep) when disabled or when they would not leave 1 GiB of device memory
static bool rl_lookahead_ready(qg_ctx *c)
{
    if (!c->rl_look_enabled) return false;
    if (c->rl_look >= 0) return c->rl_look == 1;
    c->rl_look = 0;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); return false; }
    const size_t need = 8 * rl_batch_bytes(c) + rl_table_bytes(c);
    if (free_b < need + ((size_t)1 << 30)) return false;
    bool ok = cudaMalloc(&c->rl_snap, rl_table_bytes(c)) == cudaSuccess &&
              cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; k < 8 && ok; k++)
        ok = cudaEventCreateWithFlags(&c->ev_phase[k], cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; k < 9 && ok; k++)
        if (k != 7) ok = cudaMalloc(&c->rl_buf[k], rl_batch_bytes(c)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        rl_free_lookahead(c);
        return false;
    }
    c->rl_look = 1;
    return true;
}

// the buffer heatbath phase k of a lookahead sweep of variant v reads, and
// the one the next sweep's batch k is written to
static float4 *rl_in(qg_ctx *c, int v, int k) { return c->rl_buf[k < 7 ? k : 7 + v]; }
static float4 *rl_out(qg_ctx *c, int v, int k) { return c->rl_buf[k < 7 ? k : 8 - v]; }

extern "C" int qg_destroy(qg_ctx *c)
{
    if (!c) return QG_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    destroy_graphs(c);
    if (c->side) cudaStreamSynchronize(c->side);
    rl_free_lookahead(c);
    cudaFree(c->links); cudaFree(c->rl_buf[7]); cudaFree(c->rl_table); cudaFree(c->d_seeds);
    cudaFree(const_cast<uint32_t *>(c->rl_split.mult)); cudaFree(c->rl_split.seg);
    cudaFree(c->partials); cudaFree(c->d_results); cudaFree(c->d_phase); cudaFree(c->d_params);
    cudaFree(c->d_netw); cudaFree(c->d_master); cudaFree(c->d_adam_m); cudaFree(c->d_adam_v);
    cudaFree(c->d_grad); cudaFree(c->d_gpart); cudaFree(c->d_mh_acc); cudaFree(c->d_mh_jump);
    cudaFree(c->d_net_err); cudaFree(c->d_eps);
    cudaFree(c->d_wpart); cudaFree(c->d_wout);
    cudaFree(c->d_fpart); cudaFree(c->d_ppart); cudaFree(c->d_pout); cudaFree(c->d_sites);
    cudaFree(c->d_bad);
    if (c->h_results) cudaFreeHost(c->h_results);
    if (c->h_params) cudaFreeHost(c->h_params);
    if (c->h_ring) cudaFreeHost(c->h_ring);
    for (cudaEvent_t ev : c->param_ev) if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : c->ring_ev) if (ev) cudaEventDestroy(ev);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return QG_OK;
}

extern "C" int qg_create(const qg_config *cfg, qg_ctx **out)
{
    qg_ctx *c = nullptr;
    if (!cfg || !out) return fail(nullptr, QG_ERR_ARG, "null argument");
    *out = nullptr;
    std::string why;
    if (!validate(cfg, why)) return fail(nullptr, QG_ERR_ARG, why);
    c = new (std::nothrow) qg_ctx;
    if (!c) return fail(nullptr, QG_ERR_NOMEM, "host allocation failed");
    c->cfg = *cfg;
    c->G = make_geom(cfg->size);
    const uint32_t V = c->G.V;
    const uint32_t A = (uint32_t)cfg->row_align;
    c->rowsize = align_up(V, A);
    c->prngstep = align_up(V / 2, A);
    c->instances = cfg->prng_instances;
    // PRNG_samples (suncl.cpp:2304-2307); the hot-start batch must also
    // cover the heatbath's NHITPar * 3 * (NHIT+1) quads per link
    uint64_t total = align_up((uint64_t)cfg->nhitpar * 3ull * c->prngstep * (cfg->nhit + 1), A);
    if (cfg->start == QG_START_HOT) {
        uint64_t hot = align_up((uint64_t)c->rowsize * 4 + 3ull * c->prngstep * (cfg->nhit + 1), A);
        if (hot > total) total = hot;
    }
    c->samples = (uint32_t)(1 + (total - 1) / (uint64_t)c->instances);
    const int planes = cfg->group == 3 ? 12 : 4;
    const size_t rsz = cfg->precision ? sizeof(double) : sizeof(float);
    c->link_bytes = (size_t)planes * c->G.pstride * 4 * rsz;
    c->partials_n = (size_t)((V + 127) / 128) * 4 + 64;
    cudaError_t e;
    auto bad = [&](const char *w) { int r = cuda_fail(nullptr, e, w); qg_destroy(c); return r; };
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bad("cudaStreamCreate");
    if ((e = cudaMalloc(&c->links, c->link_bytes)) != cudaSuccess) return bad("cudaMalloc(links)");
    if ((e = cudaMemsetAsync(c->links, 0, c->link_bytes, c->stream)) != cudaSuccess) return bad("cudaMemset(links)");
    if (cfg->prng == QG_PRNG_RANLUX) {
        size_t nq = (size_t)c->instances * c->samples;
        if ((e = cudaMalloc(&c->rl_buf[7], nq * sizeof(float4))) != cudaSuccess) return bad("cudaMalloc(prns)");
        c->prns = c->rl_buf[7];
        if ((e = cudaMemsetAsync(c->prns, 0, nq * sizeof(float4), c->stream)) != cudaSuccess) return bad("cudaMemset(prns)");
        if ((e = cudaMalloc(&c->rl_table, (size_t)7 * c->instances * sizeof(float4))) != cudaSuccess) return bad("cudaMalloc(table)");
        if ((e = cudaMalloc(&c->d_seeds, (size_t)c->instances * sizeof(uint32_t))) != cudaSuccess) return bad("cudaMalloc(seeds)");
        // batches of whole luxury blocks: each generator's batch over several
        // threads (the same outputs); without room for the scratch, one thread
        const int parts = ranlux_split_parts(c->instances, (int)c->samples);
        if (parts > 1) {
            std::vector<uint32_t> mult((size_t)parts * 18);
            ranlux_split_multipliers((int)c->samples, cfg->ranlux_nskip, parts, mult.data());
            uint32_t *dm = nullptr;
            float4 *seg = nullptr;
            if (cudaMalloc(&dm, mult.size() * sizeof(uint32_t)) == cudaSuccess &&
                cudaMalloc(&seg, (size_t)parts * 7 * c->instances * sizeof(float4)) == cudaSuccess &&
                cudaMemcpy(dm, mult.data(), mult.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess) {
                c->rl_split = { parts, dm, seg };
            } else {
                cudaGetLastError();
                cudaFree(dm);
                cudaFree(seg);
            }
        }
    }
    if ((e = cudaMalloc(&c->partials, c->partials_n * sizeof(double))) != cudaSuccess) return bad("cudaMalloc(partials)");
    if ((e = cudaMalloc(&c->d_results, 64 * sizeof(double))) != cudaSuccess) return bad("cudaMalloc(results)");
    if ((e = cudaMallocHost(&c->h_results, 64 * sizeof(double))) != cudaSuccess) return bad("cudaMallocHost");
    if ((e = cudaMalloc(&c->d_phase, sizeof(uint64_t))) != cudaSuccess) return bad("cudaMalloc(phase)");
    if ((e = cudaMemsetAsync(c->d_phase, 0, sizeof(uint64_t), c->stream)) != cudaSuccess) return bad("cudaMemset(phase)");
    if ((e = cudaMalloc(&c->d_params, 4 * sizeof(double))) != cudaSuccess) return bad("cudaMalloc(params)");
    if ((e = cudaMallocHost(&c->h_params, 8 * 4 * sizeof(double))) != cudaSuccess) return bad("cudaMallocHost(params)");
    if ((e = cudaMallocHost(&c->h_ring, (size_t)QG_MEASURE_SLOTS * 8 * sizeof(double))) != cudaSuccess)
        return bad("cudaMallocHost(results ring)");
    for (cudaEvent_t &ev : c->param_ev)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return bad("cudaEventCreate");
    for (cudaEvent_t &ev : c->ring_ev)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return bad("cudaEventCreate");
    if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return bad("create sync");
    if (qg_set_params(c, cfg->beta, cfg->phi, cfg->omega) != QG_OK) { g_create_err = c->err; qg_destroy(c); return QG_ERR_CUDA; }
    *out = c;
    return QG_OK;
}

static int twist_of(const qg_config &f) { return !(f.phi == 0.0 && f.omega == 0.0); }

extern "C" int qg_set_params(qg_ctx *c, double beta, double phi, double omega)
{
    if (!c) return QG_ERR_ARG;
    if (!(beta > 0.0)) return fail(c, QG_ERR_ARG, "BETA must be positive");
    c->cfg.beta = beta;
    c->cfg.phi = phi;
    c->cfg.omega = omega;
    // stream-ordered upload from one of 8 pinned staging slots; a slot is
    // rewritten only after its previous upload has completed, so the call
    // does not wait for the stream
    const uint32_t slot = c->param_next++ % 8;
    QG_CK(cudaEventSynchronize(c->param_ev[slot]), "params slot");
    double *h = c->h_params + 4 * slot;
    h[0] = beta / c->cfg.group;
    h[1] = phi;
    h[2] = omega;
    h[3] = 0.0;
    QG_CK(cudaMemcpyAsync(c->d_params, h, 4 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "params upload");
    QG_CK(cudaEventRecord(c->param_ev[slot], c->stream), "params event");
    if (twist_of(c->cfg) != c->twist_built) destroy_graphs(c);
    return QG_OK;
}

extern "C" int qg_get_stream(qg_ctx *c, void **stream)
{
    if (!c || !stream) return QG_ERR_ARG;
    *stream = (void *)c->stream;
    return QG_OK;
}

extern "C" int qg_get_info(qg_ctx *c, qg_info *info)
{
    if (!c || !info) return QG_ERR_ARG;
    info->sites = c->G.V;
    info->rowsize = c->rowsize;
    info->prngstep = c->prngstep;
    info->prng_samples = c->samples;
    info->link_bytes = c->link_bytes;
    info->ref_elems = (uint64_t)(c->cfg.group == 3 ? 12 : 4) * c->rowsize * 4;
    info->prn_quads = (uint64_t)c->instances * c->samples;
    info->phase_counter = c->phase_counter;
    info->prng_counter = c->prng_counter;
    info->sweeps_done = c->sweeps_done;
    return QG_OK;
}

extern "C" int qg_sync(qg_ctx *c)
{
    if (!c) return QG_ERR_ARG;
    QG_CK(cudaStreamSynchronize(c->stream), "qg_sync");
    return QG_OK;
}

// glibc rand() sequence after srand(seed): random_r on a private TYPE_3
// (128-byte) state, so the process-wide rand() state is left alone.
static void glibc_rand_seeds(uint32_t series, int n, std::vector<uint32_t> &out)
{
    struct random_data rd;
    int32_t statebuf[32];
    memset(&rd, 0, sizeof(rd));
    memset(statebuf, 0, sizeof(statebuf));
    initstate_r(series, (char *)statebuf, sizeof(statebuf), &rd);
    srandom_r(series, &rd);
    out.resize(n);
    int32_t r;
    random_r(&rd, &r);
    out[0] = (uint32_t)(r % 2147483647);
    for (int i = 1; i < n; i++) { random_r(&rd, &r); out[i] = (uint32_t)r; }
}

extern "C" int qg_glibc_seeds(uint32_t series, int n, uint32_t *seeds)
{
    if (n < 1 || !seeds) return QG_ERR_ARG;
    std::vector<uint32_t> v;
    glibc_rand_seeds(series, n, v);
    memcpy(seeds, v.data(), (size_t)n * sizeof(uint32_t));
    return QG_OK;
}

extern "C" int qg_prng_produce(qg_ctx *c)
{
    NvtxRange nvtx_range("qg_prng_produce");
    if (!c) return QG_ERR_ARG;
    if (c->cfg.prng != QG_PRNG_RANLUX) return fail(c, QG_ERR_STATE, "qg_prng_produce needs the RANLUX stream");
    if (!c->seeded) return fail(c, QG_ERR_STATE, "PRNG not seeded (qg_prng_seed)");
    QG_CK(rl_settle(c), "ranlux settle");
    QG_CK(launch_ranlux_produce(c->rl_table, c->prns, c->instances, (int)c->samples, c->cfg.ranlux_nskip, c->stream,
                                &c->rl_split),
          "ranlux");
    c->prng_counter++;
    return QG_OK;
}

extern "C" int qg_set_prng_lookahead(qg_ctx *c, int on)
{
    if (!c) return QG_ERR_ARG;
    QG_CK(rl_settle(c), "ranlux settle");
    c->rl_look_enabled = on != 0;
    destroy_graphs(c);
    return QG_OK;
}

extern "C" int qg_prng_seed(qg_ctx *c, uint32_t series)
{
    if (!c) return QG_ERR_ARG;
    if (series == 0) return fail(c, QG_ERR_ARG, "RANDSERIES 0 is not reproducible");
    c->cfg.randseries = series;
    destroy_graphs(c);
    if (c->cfg.prng == QG_PRNG_RANLUX) {
        std::vector<uint32_t> seeds;
        glibc_rand_seeds(series, c->instances, seeds);
        QG_CK(cudaMemcpyAsync(c->d_seeds, seeds.data(), seeds.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                              c->stream), "seed upload");
        QG_CK(launch_ranlux_init(c->d_seeds, c->rl_table, c->instances, c->stream), "ranlux_init");
        QG_CK(cudaStreamSynchronize(c->stream), "seed sync");
        c->rl_ahead = false;
        c->seeded = true;
        c->prng_counter = 0;
        return qg_prng_produce(c);   // PRNG::initialize ends with one produce()
    }
    c->key = make_uint2(series, 0x5D3E1A27u);
    c->phase_counter = 0;
    QG_CK(cudaMemsetAsync(c->d_phase, 0, sizeof(uint64_t), c->stream), "phase reset");
    c->seeded = true;
    return QG_OK;
}

extern "C" int qg_set_phase_counter(qg_ctx *c, uint64_t v)
{
    if (!c) return QG_ERR_ARG;
    c->phase_counter = v;
    QG_CK(cudaMemcpyAsync(c->d_phase, &c->phase_counter, sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream),
          "phase set");
    QG_CK(cudaStreamSynchronize(c->stream), "phase set sync");
    return QG_OK;
}

extern "C" int qg_get_config(qg_ctx *c, qg_config *cfg)
{
    if (!c || !cfg) return QG_ERR_ARG;
    *cfg = c->cfg;
    return QG_OK;
}

extern "C" int qg_set_sweeps_done(qg_ctx *c, uint64_t v)
{
    if (!c) return QG_ERR_ARG;
    c->sweeps_done = v;
    return QG_OK;
}

extern "C" int qg_prns_upload(qg_ctx *c, const float *h, uint64_t nq)
{
    if (!c || !h) return QG_ERR_ARG;
    if (!c->prns) return fail(c, QG_ERR_STATE, "no PRN buffer (Philox mode)");
    if (nq > (uint64_t)c->instances * c->samples) return fail(c, QG_ERR_ARG, "too many PRN quads");
    QG_CK(rl_settle(c), "ranlux settle");
    QG_CK(cudaMemcpyAsync(c->prns, h, nq * sizeof(float4), cudaMemcpyHostToDevice, c->stream), "prns upload");
    QG_CK(cudaStreamSynchronize(c->stream), "prns upload sync");
    return QG_OK;
}

extern "C" int qg_prns_download(qg_ctx *c, float *h, uint64_t nq)
{
    if (!c || !h) return QG_ERR_ARG;
    if (!c->prns) return fail(c, QG_ERR_STATE, "no PRN buffer (Philox mode)");
    if (nq > (uint64_t)c->instances * c->samples) return fail(c, QG_ERR_ARG, "too many PRN quads");
    QG_CK(cudaMemcpyAsync(h, c->prns, nq * sizeof(float4), cudaMemcpyDeviceToHost, c->stream), "prns download");
    QG_CK(cudaStreamSynchronize(c->stream), "prns download sync");
    return QG_OK;
}

extern "C" int qg_init_links(qg_ctx *c, int start)
{
    NvtxRange nvtx_range("qg_init_links");
    if (!c) return QG_ERR_ARG;
    const qg_config &f = c->cfg;
    if (c->slab && start != QG_START_COLD)
        return fail(c, QG_ERR_UNSUPPORTED, "a slab starts cold or from qg_links_upload of its part of a lattice");
    cudaError_t e;
    switch (start) {
    case QG_START_COLD:
        e = launch_init(c->G, c->links, f.group, f.precision, INIT_COLD, 0, nullptr, 0, c->key, c->stream);
        break;
    case QG_START_GID:
        e = launch_init(c->G, c->links, f.group, f.precision, INIT_GID, 0, nullptr, 0, c->key, c->stream);
        break;
    case QG_START_HOT:
        if (!c->seeded) return fail(c, QG_ERR_STATE, "hot start needs a seeded PRNG (qg_prng_seed)");
        if (f.prng == QG_PRNG_RANLUX) {
            // lattice_simulate: produce; init X; produce; init Y; produce; init Z; produce; init T
            e = cudaSuccess;
            for (int mu = 0; mu < 4 && e == cudaSuccess; mu++) {
                int r = qg_prng_produce(c);
                if (r) return r;
                e = launch_init(c->G, c->links, f.group, f.precision, INIT_HOT_REF, mu, c->prns, c->rowsize, c->key,
                                c->stream);
            }
        } else {
            e = launch_init(c->G, c->links, f.group, f.precision, INIT_HOT_PHILOX, 0, nullptr, 0, c->key, c->stream);
        }
        break;
    case QG_START_HAAR:
        if (!c->seeded) return fail(c, QG_ERR_STATE, "Haar start needs a seeded PRNG (qg_prng_seed)");
        e = launch_init(c->G, c->links, f.group, f.precision, INIT_HAAR, 0, nullptr, 0, c->key, c->stream);
        break;
    default:
        return fail(c, QG_ERR_ARG, "unknown start type");
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "init kernel");
    return QG_OK;
}

static PhaseArgs phase_args(qg_ctx *c, int parity, int dir, int kind, uint32_t offset)
{
    const qg_config &f = c->cfg;
    PhaseArgs a;
    a.parity = parity;
    a.dir = dir;
    a.params = c->d_params;
    a.twist = twist_of(f);
    a.nhit = f.nhit;
    a.nhitpar = f.nhitpar;
    if (kind == QG_UPDATE_OVERRELAX) a.prn_mode = -1;
    else if (f.start == QG_START_GID) a.prn_mode = 2;
    else a.prn_mode = f.prng;
    a.prns = c->prns;
    a.prngstep = c->prngstep;
    a.key = c->key;
    a.phase_base = c->d_phase;
    a.phase_offset = offset;
    a.variant = (kind == QG_UPDATE_OVERRELAX) ? c->variant_or : c->variant_hb;
    a.t_begin = 0;
    a.t_end = c->G.half;
    a.t_prn = 0;
    if (c->slab) {
        // interior slices 1..w only; the global lattice's thread indices
        // and parity (global x = local x + x0 - 1)
        const uint32_t h = c->G.n2n3n4 / 2;
        a.t_begin = h;
        a.t_end = (uint32_t)(c->G.n[0] - 1) * h;
        a.t_prn = (int32_t)(c->slab_x0 - 1) * (int32_t)h;
        a.parity = parity ^ ((c->slab_x0 - 1) & 1);
    }
    return a;
}

static cudaError_t launch_phase(qg_ctx *c, const PhaseArgs &a)
{
    return c->cfg.precision ? launch_phase_f64(c->G, c->links, c->cfg.group, a, c->stream)
                            : launch_phase_f32(c->G, c->links, c->cfg.group, a, c->stream);
}

static bool needs_seed(const qg_ctx *c, int kind)
{
    return kind == QG_UPDATE_HEATBATH && c->cfg.start != QG_START_GID && !c->seeded;
}

extern "C" int qg_phase(qg_ctx *c, int parity, int dir, int kind)
{
    NvtxRange nvtx_range("qg_phase");
    if (!c) return QG_ERR_ARG;
    if ((parity != 0 && parity != 1) || dir < 0 || dir > 3) return fail(c, QG_ERR_ARG, "bad parity/direction");
    if (kind != QG_UPDATE_HEATBATH && kind != QG_UPDATE_OVERRELAX) return fail(c, QG_ERR_ARG, "bad update kind");
    if (needs_seed(c, kind)) return fail(c, QG_ERR_STATE, "heatbath needs a seeded PRNG (qg_prng_seed)");
    PhaseArgs a = phase_args(c, parity, dir, kind, 0);
    QG_CK(launch_phase(c, a), "phase kernel");
    if (kind == QG_UPDATE_HEATBATH && a.prn_mode == QG_PRNG_PHILOX) {
        QG_CK(launch_add_u64(c->d_phase, 1, c->stream), "phase counter");
        c->phase_counter++;
    }
    return QG_OK;
}

// one phase of a slab in parts, so that its halo exchange can overlap the
// interior: part 0 updates the boundary slices x = 1 and x = w, part 1 the
// interior slices 2 .. w-1 and then advances the heatbath counter as
// qg_phase does.  The updates of one phase are independent of each other,
// so part 0 then part 1 is qg_phase bit for bit.
extern "C" int qg_slab_phase(qg_ctx *c, int parity, int dir, int kind, int part)
{
    NvtxRange nvtx_range("qg_slab_phase");
    if (!c) return QG_ERR_ARG;
    if (!c->slab) return fail(c, QG_ERR_STATE, "not a slab (qg_set_slab)");
    if ((parity != 0 && parity != 1) || dir < 0 || dir > 3) return fail(c, QG_ERR_ARG, "bad parity/direction");
    if (kind != QG_UPDATE_HEATBATH && kind != QG_UPDATE_OVERRELAX) return fail(c, QG_ERR_ARG, "bad update kind");
    if (part != 0 && part != 1) return fail(c, QG_ERR_ARG, "part: 0 boundary slices, 1 interior slices");
    if (needs_seed(c, kind)) return fail(c, QG_ERR_STATE, "heatbath needs a seeded PRNG (qg_prng_seed)");
    PhaseArgs a = phase_args(c, parity, dir, kind, 0);
    const uint32_t h = c->G.n2n3n4 / 2, w = (uint32_t)c->G.n[0] - 2;
    if (part == 0) {
        a.t_begin = h;                                   // slice 1
        a.t_end = 2 * h;
        QG_CK(launch_phase(c, a), "phase kernel");
        if (w > 1) {
            a.t_begin = w * h;                           // slice w
            a.t_end = (w + 1) * h;
            QG_CK(launch_phase(c, a), "phase kernel");
        }
        return QG_OK;
    }
    if (w > 2) {
        a.t_begin = 2 * h;                               // slices 2 .. w-1
        a.t_end = w * h;
        QG_CK(launch_phase(c, a), "phase kernel");
    }
    if (kind == QG_UPDATE_HEATBATH && a.prn_mode == QG_PRNG_PHILOX) {
        QG_CK(launch_add_u64(c->d_phase, 1, c->stream), "phase counter");
        c->phase_counter++;
    }
    return QG_OK;
}

// per-launch device time of each kernel class (the reference's per-kernel
// profiling table, clinterface.cpp:1254-1266,1626-1668): reps launches of
// each, every one between two CUDA events, on the live field (restored
// afterwards; no PRN counter moves)
extern "C" int qg_profile_kernels(qg_ctx *c, int reps, double *mean_ms, double *sigma_ms)
{
    NvtxRange nvtx_range("qg_profile_kernels");
    if (!c || !mean_ms || !sigma_ms) return QG_ERR_ARG;
    if (reps < 2) reps = 2;
    if (needs_seed(c, QG_UPDATE_HEATBATH)) return fail(c, QG_ERR_STATE, "profiling needs a seeded PRNG (qg_prng_seed)");
    const qg_config &f = c->cfg;
    const int tw = twist_of(f);
    void *backup = nullptr;
    QG_CK(cudaMallocAsync(&backup, c->link_bytes, c->stream), "profile backup");
    cudaError_t e = cudaMemcpyAsync(backup, c->links, c->link_bytes, cudaMemcpyDeviceToDevice, c->stream);
    std::vector<cudaEvent_t> ev(2 * (size_t)reps);
    for (auto &x : ev) cudaEventCreate(&x);
    for (int k = 0; k < QG_KERNEL_CLASSES && e == cudaSuccess; k++) {
        for (int r = -1; r < reps && e == cudaSuccess; r++) {     // one untimed launch first
            if (r >= 0) cudaEventRecord(ev[2 * r], c->stream);
            const int par = (r + 1) & 1, dir = ((r + 1) >> 1) & 3;
            switch (k) {
            case QG_KERNEL_HEATBATH: e = launch_phase(c, phase_args(c, par, dir, QG_UPDATE_HEATBATH, 0)); break;
            case QG_KERNEL_OVERRELAX: e = launch_phase(c, phase_args(c, par, dir, QG_UPDATE_OVERRELAX, 0)); break;
            case QG_KERNEL_REUNIT:
                e = launch_gramschmidt(c->G, c->links, f.group, f.precision, f.reunit_fp64, c->stream);
                break;
            case QG_KERNEL_PLAQUETTE:
                e = launch_plaquette(c->G, c->links, f.group, f.precision, c->d_params, tw, c->partials, c->d_results,
                                     c->stream);
                break;
            case QG_KERNEL_POLYAKOV:
                e = launch_polyakov(c->G, c->links, f.group, f.precision, c->partials, c->d_results, c->stream);
                break;
            default:
                e = launch_wilson(c->G, c->links, f.group, f.precision, f.wilson_r, f.wilson_t, c->d_params, tw,
                                  c->partials, c->d_results, c->stream);
                break;
            }
            if (r >= 0) cudaEventRecord(ev[2 * r + 1], c->stream);
        }
        if (e != cudaSuccess) break;
        cudaEventSynchronize(ev[2 * reps - 1]);
        double m = 0, m2 = 0;
        for (int r = 0; r < reps; r++) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]);
            m += ms;
            m2 += (double)ms * ms;
        }
        m /= reps;
        mean_ms[k] = m;
        sigma_ms[k] = sqrt(fmax(0.0, m2 / reps - m * m) * reps / (reps - 1));
    }
    cudaError_t e2 = cudaMemcpyAsync(c->links, backup, c->link_bytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaFreeAsync(backup, c->stream);
    cudaError_t e3 = cudaStreamSynchronize(c->stream);
    for (auto &x : ev) cudaEventDestroy(x);
    if (e != cudaSuccess) return cuda_fail(c, e, "profile launch");
    if (e2 != cudaSuccess) return cuda_fail(c, e2, "profile restore");
    if (e3 != cudaSuccess) return cuda_fail(c, e3, "profile sync");
    return QG_OK;
}

// times each launch shape of the heatbath and overrelaxation phase kernels
// on the live field (restored afterwards, PRN counters untouched) and keeps
// the fastest per kind
extern "C" int qg_tune(qg_ctx *c, int reps, float *times_ms)
{
    NvtxRange nvtx_range("qg_tune");
    if (!c) return QG_ERR_ARG;
    if (reps < 1) reps = 4;
    if (needs_seed(c, QG_UPDATE_HEATBATH)) return fail(c, QG_ERR_STATE, "tuning needs a seeded PRNG (qg_prng_seed)");
    void *backup = nullptr;
    QG_CK(cudaMallocAsync(&backup, c->link_bytes, c->stream), "tune backup");
    QG_CK(cudaMemcpyAsync(backup, c->links, c->link_bytes, cudaMemcpyDeviceToDevice, c->stream), "tune backup copy");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best[2] = { 1e30f, 1e30f };
    int arg[2] = { 0, 0 };
    cudaError_t e = cudaSuccess;
    for (int v = 0; v < kPhaseVariants && e == cudaSuccess; v++)
        for (int kind = 0; kind < 2 && e == cudaSuccess; kind++) {
            PhaseArgs a = phase_args(c, 0, 0, kind, 0);
            a.variant = v;
            // one untimed launch, then reps timed ones over the 8 phase classes
            for (int r = -1; r < reps && e == cudaSuccess; r++) {
                if (r == 0) cudaEventRecord(e0, c->stream);
                a.parity = (r + 1) & 1;
                a.dir = ((r + 1) >> 1) & 3;
                e = launch_phase(c, a);
            }
            cudaEventRecord(e1, c->stream);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= reps;
            if (times_ms) times_ms[2 * v + kind] = ms;
            if (ms < best[kind]) { best[kind] = ms; arg[kind] = v; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t e2 = cudaMemcpyAsync(c->links, backup, c->link_bytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaFreeAsync(backup, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "tune launch");
    if (e2 != cudaSuccess) return cuda_fail(c, e2, "tune restore");
    QG_CK(cudaStreamSynchronize(c->stream), "tune sync");
    c->variant_hb = arg[0];
    c->variant_or = arg[1];
    destroy_graphs(c);
    return QG_OK;
}

extern "C" int qg_set_shapes(qg_ctx *c, int heatbath_shape, int overrelax_shape)
{
    if (!c) return QG_ERR_ARG;
    if (heatbath_shape < 0 || heatbath_shape >= kPhaseVariants || overrelax_shape < 0 ||
        overrelax_shape >= kPhaseVariants)
        return fail(c, QG_ERR_ARG, "launch shape out of range [0, QG_TUNE_SHAPES)");
    c->variant_hb = heatbath_shape;
    c->variant_or = overrelax_shape;
    destroy_graphs(c);
    return QG_OK;
}

extern "C" int qg_get_shapes(qg_ctx *c, int *heatbath_shape, int *overrelax_shape)
{
    if (!c || !heatbath_shape || !overrelax_shape) return QG_ERR_ARG;
    *heatbath_shape = c->variant_hb;
    *overrelax_shape = c->variant_or;
    return QG_OK;
}

extern "C" int qg_reunitarize(qg_ctx *c, int fp64)
{
    NvtxRange nvtx_range("qg_reunitarize");
    if (!c) return QG_ERR_ARG;
    QG_CK(launch_gramschmidt(c->G, c->links, c->cfg.group, c->cfg.precision, fp64, c->stream), "gramschmidt");
    return QG_OK;
}

// one sweep's launches: lattice_simulate's working-cycle body
// (suncl.cpp:5393-5412) plus the overrelaxation sweeps.  ev (optional):
// an event recorded before and after every phase launch, ev[2k] and
// ev[2k + 1] around the sweep's k-th phase (heatbath phases first)
static cudaError_t enqueue_sweep(qg_ctx *c, bool reunit, cudaEvent_t *ev = nullptr)
{
    const qg_config &f = c->cfg;
    cudaError_t e;
    uint32_t hb = 0;
    int k_ph = 0;
    auto timed_phase = [&](const PhaseArgs &a) {
        cudaError_t r;
        if (ev && (r = cudaEventRecordWithFlags(ev[2 * k_ph], c->stream, cudaEventRecordExternal)) != cudaSuccess)
            return r;
        if ((r = launch_phase(c, a)) != cudaSuccess) return r;
        if (ev && (r = cudaEventRecordWithFlags(ev[2 * k_ph + 1], c->stream, cudaEventRecordExternal)) != cudaSuccess)
            return r;
        k_ph++;
        return cudaSuccess;
    };
    const int par_order[2] = { 1, 0 };   // odd first, then even
    for (int pi = 0; pi < 2; pi++)
        for (int mu = 0; mu < 4; mu++) {
            PhaseArgs a = phase_args(c, par_order[pi], mu, QG_UPDATE_HEATBATH, hb);
            if (a.prn_mode == QG_PRNG_RANLUX) {
                e = launch_ranlux_produce(c->rl_table, c->prns, c->instances, (int)c->samples, f.ranlux_nskip, c->stream,
                                          &c->rl_split);
                if (e != cudaSuccess) return e;
            }
            if ((e = timed_phase(a)) != cudaSuccess) return e;
            if (a.prn_mode == QG_PRNG_PHILOX) hb++;
        }
    for (int k = 0; k < f.n_or; k++)
        for (int pi = 0; pi < 2; pi++)
            for (int mu = 0; mu < 4; mu++) {
                PhaseArgs a = phase_args(c, par_order[pi], mu, QG_UPDATE_OVERRELAX, 0);
                if ((e = timed_phase(a)) != cudaSuccess) return e;
            }
    if (hb) {
        if ((e = launch_add_u64(c->d_phase, hb, c->stream)) != cudaSuccess) return e;
    }
    if (reunit) {
        if ((e = launch_gramschmidt(c->G, c->links, f.group, f.precision, f.reunit_fp64, c->stream)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

// A RANLUX-mode sweep with the next sweep's batches generated alongside:
// the heatbath phases read this sweep's batches (generated by the previous
// sweep or the prologue in qg_sweep) from rl_in(v, k); the second stream
// first saves the generator state (the state at this sweep's last batch,
// for rl_settle), then produces the next 8 batches into rl_out(v, k), batch
// k only after phase k has read its buffer.  The batches and the order in
// which each is consumed are those of enqueue_sweep.
static cudaError_t enqueue_sweep_lookahead(qg_ctx *c, bool reunit, int v)
{
    const qg_config &f = c->cfg;
    cudaError_t e;
    const int par_order[2] = { 1, 0 };
    if ((e = cudaEventRecord(c->ev_fork, c->stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(c->side, c->ev_fork, 0)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(c->rl_snap, c->rl_table, rl_table_bytes(c), cudaMemcpyDeviceToDevice, c->side)) !=
        cudaSuccess)
        return e;
    int k = 0;
    for (int pi = 0; pi < 2; pi++)
        for (int mu = 0; mu < 4; mu++, k++) {
            PhaseArgs a = phase_args(c, par_order[pi], mu, QG_UPDATE_HEATBATH, 0);
            a.prns = rl_in(c, v, k);
            if ((e = launch_phase(c, a)) != cudaSuccess) return e;
            if ((e = cudaEventRecord(c->ev_phase[k], c->stream)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(c->side, c->ev_phase[k], 0)) != cudaSuccess) return e;
            if ((e = launch_ranlux_produce(c->rl_table, rl_out(c, v, k), c->instances, (int)c->samples,
                                           f.ranlux_nskip, c->side, &c->rl_split)) != cudaSuccess)
                return e;
        }
    for (int n = 0; n < f.n_or; n++)
        for (int pi = 0; pi < 2; pi++)
            for (int mu = 0; mu < 4; mu++) {
                PhaseArgs a = phase_args(c, par_order[pi], mu, QG_UPDATE_OVERRELAX, 0);
                if ((e = launch_phase(c, a)) != cudaSuccess) return e;
            }
    if (reunit) {
        if ((e = launch_gramschmidt(c->G, c->links, f.group, f.precision, f.reunit_fp64, c->stream)) != cudaSuccess)
            return e;
    }
    if ((e = cudaEventRecord(c->ev_join, c->side)) != cudaSuccess) return e;
    return cudaStreamWaitEvent(c->stream, c->ev_join, 0);
}

static int build_graph(qg_ctx *c, int which)
{
    cudaGraph_t g = nullptr;
    QG_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t e = which >= 2 ? enqueue_sweep_lookahead(c, (which & 1) != 0, (which - 2) >> 1)
                               : enqueue_sweep(c, which == 1);
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(c, e, "sweep capture"); }
    if (e2 != cudaSuccess) return cuda_fail(c, e2, "end capture");
    c->twist_built = twist_of(c->cfg);
    e = cudaGraphInstantiate(&c->graph[which], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(c, e, "graph instantiate");
    return QG_OK;
}

// links that are not finite or not in SU(N) to within tol (rows of unit
// norm, orthogonal); synchronous
extern "C" int qg_field_check(qg_ctx *c, double tol, uint64_t *bad_links)
{
    NvtxRange nvtx_range("qg_field_check");
    if (!c || !bad_links || !(tol > 0)) return QG_ERR_ARG;
    if (!c->d_bad) QG_CK(cudaMalloc(&c->d_bad, sizeof(unsigned long long)), "field check counter");
    QG_CK(cudaMemsetAsync(c->d_bad, 0, sizeof(unsigned long long), c->stream), "field check reset");
    QG_CK(launch_field_check(c->G, c->links, c->cfg.group, c->cfg.precision, tol, c->d_bad, c->stream),
          "field check kernel");
    unsigned long long n = 0;
    QG_CK(cudaMemcpyAsync(&n, c->d_bad, sizeof(n), cudaMemcpyDeviceToHost, c->stream), "field check read");
    QG_CK(cudaStreamSynchronize(c->stream), "field check sync");
    *bad_links = n;
    return QG_OK;
}

// ------------------------------------------------------------ x-slabs
extern "C" int qg_set_slab(qg_ctx *c, int x0, int n1_global)
{
    if (!c) return QG_ERR_ARG;
    const qg_config &f = c->cfg;
    const int w = f.size[0] - 2;
    if (w < 1 || n1_global < 2 || x0 < 0 || x0 >= n1_global || w > n1_global)
        return fail(c, QG_ERR_ARG, "slab: size[0] - 2 interior slices starting at global x0 of n1_global");
    if (n1_global % 2 || c->G.n2n3n4 % 2)
        return fail(c, QG_ERR_ARG, "slab: the global N1 and N2*N3*N4 must be even (checkerboard across slabs)");
    if (f.prng != QG_PRNG_PHILOX || f.start == QG_START_GID)
        return fail(c, QG_ERR_UNSUPPORTED, "slabs run the Philox stream (its numbers depend on the site only)");
    if (twist_of(f)) return fail(c, QG_ERR_UNSUPPORTED, "slabs need periodic boundaries (PHI = OMEGA = 0)");
    c->slab = true;
    c->slab_x0 = x0;
    c->slab_n1 = n1_global;
    destroy_graphs(c);
    return QG_OK;
}

static uint32_t slab_planes(const qg_ctx *c) { return c->cfg.group == 3 ? 3u : 1u; }
static size_t slab_elem(const qg_ctx *c) { return c->cfg.precision ? 32 : 16; }

extern "C" int qg_slab_halo_bytes(qg_ctx *c, uint64_t *bytes)
{
    if (!c || !bytes) return QG_ERR_ARG;
    *bytes = (uint64_t)slab_planes(c) * (c->G.n2n3n4 / 2) * slab_elem(c);
    return QG_OK;
}

// the links of direction dir and global parity p of one x-slice, plane by
// plane: to_buf = 1 copies the boundary slice (x = 1 for side 0, x = w for
// side 1) into buf, to_buf = 0 copies buf into the halo (x = 0 / x = w+1).
// In a slice of parity q they are the elements q cb + x h .. + h of each
// plane, ordered by the site index within the slice -- the same order in
// every slab, so a boundary packed by one slab unpacks into the halo of its
// neighbour.
extern "C" int qg_slab_halo(qg_ctx *c, int dir, int parity, int side, void *buf, int to_buf)
{
    if (!c || !buf) return QG_ERR_ARG;
    if (!c->slab) return fail(c, QG_ERR_STATE, "not a slab (qg_set_slab)");
    if (dir < 0 || dir > 3 || (parity != 0 && parity != 1) || (side != 0 && side != 1))
        return fail(c, QG_ERR_ARG, "bad direction / parity / side");
    const uint32_t h = c->G.n2n3n4 / 2, w = (uint32_t)c->G.n[0] - 2;
    const uint32_t x = to_buf ? (side ? w : 1) : (side ? w + 1 : 0);
    const uint32_t q = (uint32_t)(parity ^ ((c->slab_x0 - 1) & 1));
    const size_t es = slab_elem(c), n = (size_t)h * es;
    char *base = static_cast<char *>(c->links);
    char *b = static_cast<char *>(buf);
    for (uint32_t k = 0; k < slab_planes(c); k++) {
        const size_t plane = (size_t)dir + 4 * k;
        char *lk = base + (plane * c->G.pstride + (size_t)q * c->G.cb + (size_t)x * h) * es;
        char *bk = b + k * n;
        QG_CK(cudaMemcpyAsync(to_buf ? bk : lk, to_buf ? lk : bk, n, cudaMemcpyDefault, c->stream), "slab halo copy");
    }
    return QG_OK;
}

// both sides in one launch: to_buf = 1 packs boundary slices x = 1 into
// buf_lo and x = w into buf_hi; to_buf = 0 unpacks buf_lo into halo x = 0
// and buf_hi into halo x = w+1 (buffers in device memory, 16-byte aligned)
extern "C" int qg_slab_halo2(qg_ctx *c, int dir, int parity, void *buf_lo, void *buf_hi, int to_buf)
{
    NvtxRange nvtx_range("qg_slab_halo2");
    if (!c || !buf_lo || !buf_hi) return QG_ERR_ARG;
    if (!c->slab) return fail(c, QG_ERR_STATE, "not a slab (qg_set_slab)");
    if (dir < 0 || dir > 3 || (parity != 0 && parity != 1)) return fail(c, QG_ERR_ARG, "bad direction / parity");
    if (((uintptr_t)buf_lo | (uintptr_t)buf_hi) & 15) return fail(c, QG_ERR_ARG, "halo buffers must be 16-byte aligned");
    for (void *b : { buf_lo, buf_hi }) {       // the kernel reads and writes them: device memory only
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, b) != cudaSuccess ||
            (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
            cudaGetLastError();
            return fail(c, QG_ERR_ARG, "qg_slab_halo2 needs device buffers (qg_slab_halo copies from host memory)");
        }
    }
    const uint32_t h = c->G.n2n3n4 / 2, w = (uint32_t)c->G.n[0] - 2;
    const uint32_t q = (uint32_t)(parity ^ ((c->slab_x0 - 1) & 1));
    const size_t unit = slab_elem(c) / 16;                       // 16-byte words per element
    uint4 *base = static_cast<uint4 *>(c->links);
    SlabCopy cp;
    cp.n = 0;
    cp.words = (uint32_t)(h * unit);
    for (int side = 0; side < 2; side++) {
        const uint32_t x = to_buf ? (side ? w : 1) : (side ? w + 1 : 0);
        uint4 *b = static_cast<uint4 *>(side ? buf_hi : buf_lo);
        for (uint32_t k = 0; k < slab_planes(c); k++) {
            uint4 *lk = base + ((size_t)(dir + 4 * k) * c->G.pstride + (size_t)q * c->G.cb + (size_t)x * h) * unit;
            uint4 *bk = b + (size_t)k * h * unit;
            cp.src[cp.n] = to_buf ? lk : bk;
            cp.dst[cp.n] = to_buf ? bk : lk;
            cp.n++;
        }
    }
    QG_CK(launch_slab_copy(cp, c->stream), "slab halo kernel");
    return QG_OK;
}

extern "C" int qg_sweep(qg_ctx *c, int nsweeps)
{
    NvtxRange nvtx_range("qg_sweep");
    if (!c) return QG_ERR_ARG;
    if (c->slab) return fail(c, QG_ERR_STATE, "a slab sweeps phase by phase with halo exchanges (qcdgpu_b200.slabs)");
    if (nsweeps < 0) return fail(c, QG_ERR_ARG, "negative sweep count");
    if (needs_seed(c, QG_UPDATE_HEATBATH)) return fail(c, QG_ERR_STATE, "heatbath needs a seeded PRNG (qg_prng_seed)");
    const qg_config &f = c->cfg;
    const bool philox = (f.prng == QG_PRNG_PHILOX && f.start != QG_START_GID);
    const bool ranlux = (f.prng == QG_PRNG_RANLUX && f.start != QG_START_GID);
    const bool look = ranlux && nsweeps > 0 && rl_lookahead_ready(c);
    if (look && !c->rl_ahead) {
        // prologue: this sweep's 8 batches, into the buffers of a variant
        // that leaves the last batch consumed (prns) in place
        c->rl_var = (c->prns == c->rl_buf[7]) ? 1 : 0;
        QG_CK(cudaMemcpyAsync(c->rl_snap, c->rl_table, rl_table_bytes(c), cudaMemcpyDeviceToDevice, c->stream),
              "ranlux snapshot");
        for (int k = 0; k < 8; k++)
            QG_CK(launch_ranlux_produce(c->rl_table, rl_in(c, c->rl_var, k), c->instances, (int)c->samples,
                                        f.ranlux_nskip, c->stream, &c->rl_split), "ranlux");
        c->rl_ahead = true;
    }
    for (int n = 0; n < nsweeps; n++) {
        const bool reunit = f.reunit_every > 0 && ((c->sweeps_done + 1) % (uint64_t)f.reunit_every) == 0;
        const int which = look ? 2 + 2 * c->rl_var + (reunit ? 1 : 0) : (reunit ? 1 : 0);
        if (!c->graph[which]) {
            int r = build_graph(c, which);
            if (r) return r;
        }
        QG_CK(cudaGraphLaunch(c->graph[which], c->stream), "graph launch");
        c->sweeps_done++;
        if (philox) c->phase_counter += 8;
        if (ranlux) c->prng_counter += 8;
        if (look) {
            c->prns = c->rl_buf[7 + c->rl_var];   // this sweep's last batch
            c->rl_var ^= 1;
        }
    }
    return QG_OK;
}

// nsweeps sweeps of the qg_sweep chain (Philox stream, same launches and
// reunitarisation cadence) captured as one graph with an event node before
// and after every phase launch and around the whole: the mean duration of a
// heatbath and of an overrelaxation phase as they run inside the sweep
// graph, and of a whole sweep in that graph
extern "C" int qg_sweep_phase_times(qg_ctx *c, int nsweeps, double *ms_heatbath, double *ms_overrelax,
                                    double *ms_sweep)
{
    NvtxRange nvtx_range("qg_sweep_phase_times");
    if (!c || !ms_heatbath || !ms_overrelax || !ms_sweep) return QG_ERR_ARG;
    if (c->slab) return fail(c, QG_ERR_STATE, "a slab sweeps phase by phase with halo exchanges (qcdgpu_b200.slabs)");
    if (nsweeps < 1 || nsweeps > 256) return fail(c, QG_ERR_ARG, "phase timing: nsweeps in [1, 256]");
    const qg_config &f = c->cfg;
    if (f.prng != QG_PRNG_PHILOX || f.start == QG_START_GID)
        return fail(c, QG_ERR_UNSUPPORTED, "phase timing inside the sweep graph runs the Philox stream");
    if (needs_seed(c, QG_UPDATE_HEATBATH)) return fail(c, QG_ERR_STATE, "heatbath needs a seeded PRNG (qg_prng_seed)");
    const int nph = 8 * (1 + f.n_or);
    // the phases' events, then the two around the whole graph
    std::vector<cudaEvent_t> ev((size_t)2 * nph * nsweeps + 2, nullptr);
    const size_t all0 = (size_t)2 * nph * nsweeps, all1 = all0 + 1;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t gx = nullptr;
    cudaError_t e = cudaSuccess;
    const char *where = "event create";
    for (auto &x : ev)
        if ((e = cudaEventCreate(&x)) != cudaSuccess) break;
    if (e == cudaSuccess) {
        where = "timed sweep capture";
        e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            e = cudaEventRecordWithFlags(ev[all0], c->stream, cudaEventRecordExternal);
            for (int n = 0; n < nsweeps && e == cudaSuccess; n++) {
                const bool reunit = f.reunit_every > 0 && ((c->sweeps_done + n + 1) % (uint64_t)f.reunit_every) == 0;
                e = enqueue_sweep(c, reunit, ev.data() + (size_t)2 * nph * n);
            }
            if (e == cudaSuccess) e = cudaEventRecordWithFlags(ev[all1], c->stream, cudaEventRecordExternal);
            cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
            if (e == cudaSuccess) e = e2;
        }
    }
    if (e == cudaSuccess) { where = "timed sweep instantiate"; e = cudaGraphInstantiate(&gx, g, 0); }
    if (e == cudaSuccess) { where = "timed sweep launch"; e = cudaGraphLaunch(gx, c->stream); }
    if (e == cudaSuccess) { where = "timed sweep sync"; e = cudaStreamSynchronize(c->stream); }
    double sum_hb = 0, sum_or = 0;
    float all_ms = 0;
    if (e == cudaSuccess) {
        c->sweeps_done += (uint64_t)nsweeps;
        c->phase_counter += 8 * (uint64_t)nsweeps;
        where = "phase event time";
        for (int n = 0; n < nsweeps && e == cudaSuccess; n++)
            for (int k = 0; k < nph && e == cudaSuccess; k++) {
                float ms = 0;
                const size_t i = (size_t)2 * nph * n + 2 * k;
                if ((e = cudaEventElapsedTime(&ms, ev[i], ev[i + 1])) == cudaSuccess) (k < 8 ? sum_hb : sum_or) += ms;
            }
        if (e == cudaSuccess) e = cudaEventElapsedTime(&all_ms, ev[all0], ev[all1]);
    }
    if (gx) cudaGraphExecDestroy(gx);
    if (g) cudaGraphDestroy(g);
    for (auto &x : ev)
        if (x) cudaEventDestroy(x);
    if (e != cudaSuccess) return cuda_fail(c, e, where);
    *ms_heatbath = sum_hb / (8.0 * nsweeps);
    *ms_overrelax = f.n_or > 0 ? sum_or / (8.0 * f.n_or * nsweeps) : 0.0;
    *ms_sweep = (double)all_ms / nsweeps;
    return QG_OK;
}

// ------------------------------------------------- learned-proposal Metropolis
static int net_check(qg_ctx *c)
{
    if (c->slab) return fail(c, QG_ERR_UNSUPPORTED, "the learned proposal runs on whole lattices");
    if (c->cfg.group != 3 || c->cfg.precision != 0 || c->cfg.prng != QG_PRNG_PHILOX)
        return fail(c, QG_ERR_UNSUPPORTED, "the learned proposal runs on SU(3) FP32 links with the Philox stream");
    if (c->cfg.phi != 0.0 || c->cfg.omega != 0.0)
        return fail(c, QG_ERR_UNSUPPORTED, "the learned proposal needs periodic boundaries (PHI = OMEGA = 0)");
    return QG_OK;
}

extern "C" int qg_net_set(qg_ctx *c, const float *params, double eps_max)
{
    if (!c || !params) return QG_ERR_ARG;
    int r = net_check(c);
    if (r) return r;
    if (!(eps_max > 0.0 && eps_max <= 3.2)) return fail(c, QG_ERR_ARG, "eps_max must be in (0, 3.2]");
    const size_t np = QG_NET_PARAMS;
    if (!c->d_master) {
        QG_CK(cudaMalloc(&c->d_netw, np * sizeof(uint16_t)), "net alloc");
        QG_CK(cudaMalloc(&c->d_master, np * sizeof(float)), "net alloc");
        QG_CK(cudaMalloc(&c->d_adam_m, np * sizeof(float)), "net alloc");
        QG_CK(cudaMalloc(&c->d_adam_v, np * sizeof(float)), "net alloc");
        QG_CK(cudaMalloc(&c->d_grad, (np + 4) * sizeof(float)), "net alloc");
        QG_CK(cudaMalloc(&c->d_gpart, (size_t)mh_grad_blocks(c->G) * (np + 4) * sizeof(float)), "net alloc");
        QG_CK(cudaMalloc(&c->d_mh_acc, sizeof(unsigned long long)), "net alloc");
        QG_CK(cudaMalloc(&c->d_mh_jump, sizeof(double)), "net alloc");
        QG_CK(cudaMalloc(&c->d_net_err, sizeof(unsigned)), "net alloc");
        QG_CK(cudaMemsetAsync(c->d_net_err, 0, sizeof(unsigned), c->stream), "net clear");
        QG_CK(cudaMemsetAsync(c->d_mh_acc, 0, sizeof(unsigned long long), c->stream), "net clear");
        QG_CK(cudaMemsetAsync(c->d_mh_jump, 0, sizeof(double), c->stream), "net clear");
    }
    QG_CK(cudaMemcpyAsync(c->d_master, params, np * sizeof(float), cudaMemcpyHostToDevice, c->stream), "net upload");
    QG_CK(cudaMemsetAsync(c->d_adam_m, 0, np * sizeof(float), c->stream), "net clear");
    QG_CK(cudaMemsetAsync(c->d_adam_v, 0, np * sizeof(float), c->stream), "net clear");
    QG_CK(launch_to_bf16(c->d_master, c->d_netw, c->stream), "net bf16");
    QG_CK(cudaStreamSynchronize(c->stream), "net sync");
    c->eps_max = eps_max;
    c->adam_t = 0;
    return QG_OK;
}

extern "C" int qg_net_get(qg_ctx *c, float *master, float *weights_bf16)
{
    if (!c) return QG_ERR_ARG;
    if (!c->d_master) return fail(c, QG_ERR_STATE, "no network set (qg_net_set)");
    const size_t np = QG_NET_PARAMS;
    if (master) QG_CK(cudaMemcpyAsync(master, c->d_master, np * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "net get");
    std::vector<uint16_t> b(np);
    QG_CK(cudaMemcpyAsync(b.data(), c->d_netw, np * sizeof(uint16_t), cudaMemcpyDeviceToHost, c->stream), "net get");
    QG_CK(cudaStreamSynchronize(c->stream), "net get sync");
    if (weights_bf16)
        for (size_t i = 0; i < np; i++) {
            uint32_t u = (uint32_t)b[i] << 16;
            memcpy(&weights_bf16[i], &u, 4);
        }
    return QG_OK;
}

static int mh_ready(qg_ctx *c)
{
    int r = net_check(c);
    if (r) return r;
    if (!c->d_master) return fail(c, QG_ERR_STATE, "no network set (qg_net_set)");
    if (!c->seeded) return fail(c, QG_ERR_STATE, "the learned proposal needs a seeded PRNG (qg_prng_seed)");
    return QG_OK;
}

static cudaError_t mh_launch(qg_ctx *c, int parity, int dir, int nhit, uint32_t offset, float *eps_out = nullptr)
{
    PhaseArgs a = phase_args(c, parity, dir, QG_UPDATE_HEATBATH, offset);
    return launch_mh_phase(c->G, c->links, a, c->d_netw, c->eps_max, nhit, c->d_mh_acc, c->d_mh_jump, eps_out,
                           c->d_net_err, c->stream);
}

// the tensor-core waits of the network kernels are bounded; a wait that
// ran out is reported here (the call that observes it fails, the flag is
// cleared)
static int net_err_check(qg_ctx *c)
{
    unsigned flag = 0;
    QG_CK(cudaMemcpyAsync(&flag, c->d_net_err, sizeof(flag), cudaMemcpyDeviceToHost, c->stream), "net flag");
    QG_CK(cudaStreamSynchronize(c->stream), "net flag sync");
    if (flag) {
        QG_CK(cudaMemsetAsync(c->d_net_err, 0, sizeof(unsigned), c->stream), "net flag clear");
        return fail(c, QG_ERR_CUDA, "a tensor-core wait of the network kernels ran out");
    }
    return QG_OK;
}

// the step eps of every link of phase (parity, dir) as the next qg_mh_phase
// on the same field and weights computes it (thread order, G.half values)
extern "C" int qg_net_eps(qg_ctx *c, int parity, int dir, float *eps)
{
    if (!c || !eps) return QG_ERR_ARG;
    if (parity < 0 || parity > 1 || dir < 0 || dir > 3) return fail(c, QG_ERR_ARG, "bad phase");
    int r = mh_ready(c);
    if (r) return r;
    if (!c->d_eps) QG_CK(cudaMalloc(&c->d_eps, (size_t)c->G.half * sizeof(float)), "eps alloc");
    QG_CK(mh_launch(c, parity, dir, 1, 0, c->d_eps), "net eps");
    QG_CK(cudaMemcpyAsync(eps, c->d_eps, (size_t)c->G.half * sizeof(float), cudaMemcpyDeviceToHost, c->stream),
          "eps copy");
    return net_err_check(c);
}

extern "C" int qg_mh_phase(qg_ctx *c, int parity, int dir, int nhit)
{
    if (!c) return QG_ERR_ARG;
    if (parity < 0 || parity > 1 || dir < 0 || dir > 3 || nhit < 1) return fail(c, QG_ERR_ARG, "bad phase");
    int r = mh_ready(c);
    if (r) return r;
    QG_CK(mh_launch(c, parity, dir, nhit, 0), "mh phase");
    QG_CK(launch_add_u64(c->d_phase, 1, c->stream), "phase counter");
    c->phase_counter++;
    c->mh_hits += (uint64_t)c->G.half * 3 * nhit;
    return QG_OK;
}

// learned-proposal sweeps: odd X..T, even X..T Metropolis phases (nhit
// hits per subgroup and link), the global Gram-Schmidt on the cadence of
// qg_sweep (the sweep counter is shared)
extern "C" int qg_mh_sweep(qg_ctx *c, int nsweeps, int nhit)
{
    NvtxRange nvtx_range("qg_mh_sweep");
    if (!c) return QG_ERR_ARG;
    if (nsweeps < 0 || nhit < 1) return fail(c, QG_ERR_ARG, "bad sweep arguments");
    int r = mh_ready(c);
    if (r) return r;
    const qg_config &f = c->cfg;
    const int par_order[2] = { 1, 0 };
    for (int n = 0; n < nsweeps; n++) {
        uint32_t k = 0;
        for (int pi = 0; pi < 2; pi++)
            for (int mu = 0; mu < 4; mu++) QG_CK(mh_launch(c, par_order[pi], mu, nhit, k++), "mh phase");
        QG_CK(launch_add_u64(c->d_phase, 8, c->stream), "phase counter");
        c->phase_counter += 8;
        c->mh_hits += (uint64_t)c->G.half * 2 * 4 * 3 * nhit;
        const bool reunit = f.reunit_every > 0 && ((c->sweeps_done + 1) % (uint64_t)f.reunit_every) == 0;
        if (reunit)
            QG_CK(launch_gramschmidt(c->G, c->links, f.group, f.precision, f.reunit_fp64, c->stream), "gramschmidt");
        c->sweeps_done++;
    }
    return QG_OK;
}

extern "C" int qg_mh_stats(qg_ctx *c, double *accept_rate, double *jump_per_hit, uint64_t *hits, int reset)
{
    if (!c) return QG_ERR_ARG;
    unsigned long long acc = 0;
    double jump = 0.0;
    if (c->d_mh_acc) {
        QG_CK(cudaMemcpyAsync(&acc, c->d_mh_acc, sizeof(acc), cudaMemcpyDeviceToHost, c->stream), "stats");
        QG_CK(cudaMemcpyAsync(&jump, c->d_mh_jump, sizeof(jump), cudaMemcpyDeviceToHost, c->stream), "stats");
        QG_CK(cudaStreamSynchronize(c->stream), "stats sync");
    }
    if (c->d_net_err) {
        int r = net_err_check(c);
        if (r) return r;
    }
    const double h = (double)c->mh_hits;
    if (accept_rate) *accept_rate = h > 0 ? (double)acc / h : 0.0;
    if (jump_per_hit) *jump_per_hit = h > 0 ? jump / h : 0.0;
    if (hits) *hits = c->mh_hits;
    if (reset && c->d_mh_acc) {
        QG_CK(cudaMemsetAsync(c->d_mh_acc, 0, sizeof(unsigned long long), c->stream), "stats reset");
        QG_CK(cudaMemsetAsync(c->d_mh_jump, 0, sizeof(double), c->stream), "stats reset");
        c->mh_hits = 0;
    }
    return QG_OK;
}

static const uint32_t kTrainKey = 0x2C1B3A49u;

extern "C" int qg_net_grad(qg_ctx *c, int parity, int dir, float *grad, double *stats)
{
    if (!c) return QG_ERR_ARG;
    if (parity < 0 || parity > 1 || dir < 0 || dir > 3) return fail(c, QG_ERR_ARG, "bad phase");
    int r = mh_ready(c);
    if (r) return r;
    QG_CK(launch_mh_grad(c->G, c->links, parity, dir, c->d_params, c->d_netw, c->eps_max,
                         make_uint2(c->cfg.randseries, kTrainKey), c->train_phase++, c->d_gpart, c->d_grad,
                         c->d_net_err, c->stream),
          "net grad");
    std::vector<float> h(QG_NET_PARAMS + 4);
    QG_CK(cudaMemcpyAsync(h.data(), c->d_grad, h.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "grad copy");
    QG_CK(cudaStreamSynchronize(c->stream), "grad sync");
    r = net_err_check(c);
    if (r) return r;
    if (grad) memcpy(grad, h.data(), QG_NET_PARAMS * sizeof(float));
    if (stats) {
        const double n = h[QG_NET_PARAMS + 3] > 0 ? h[QG_NET_PARAMS + 3] : 1.0;
        stats[0] = h[QG_NET_PARAMS] / n;          // loss per link
        stats[1] = h[QG_NET_PARAMS + 1] / n;      // ESJD per link (3 proposals)
        stats[2] = h[QG_NET_PARAMS + 2] / n;      // mean acceptance
        stats[3] = h[QG_NET_PARAMS + 3];          // links
    }
    return QG_OK;
}

// steps Adam steps; step s uses the links of phase (s % 8) in the sweep
// order; stats: the mean over the steps of (loss, ESJD, acceptance, links)
extern "C" int qg_net_train(qg_ctx *c, int steps, double lr, double *stats)
{
    NvtxRange nvtx_range("qg_net_train");
    if (!c) return QG_ERR_ARG;
    if (steps < 0 || !(lr > 0.0)) return fail(c, QG_ERR_ARG, "bad training arguments");
    int r = mh_ready(c);
    if (r) return r;
    const int par_order[2] = { 1, 0 };
    double acc[4] = { 0, 0, 0, 0 };
    std::vector<float> h(QG_NET_PARAMS + 4);
    for (int s = 0; s < steps; s++) {
        const int k = s % 8;
        QG_CK(launch_mh_grad(c->G, c->links, par_order[k / 4], k % 4, c->d_params, c->d_netw, c->eps_max,
                             make_uint2(c->cfg.randseries, kTrainKey), c->train_phase++, c->d_gpart, c->d_grad,
                             c->d_net_err, c->stream), "net grad");
        c->adam_t++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - powf(b1, (float)c->adam_t), c2 = 1.0f - powf(b2, (float)c->adam_t);
        QG_CK(launch_adam(c->d_master, c->d_adam_m, c->d_adam_v, c->d_grad, c->d_netw, (float)lr, b1, b2, c1, c2,
                          1e-8f, c->stream), "adam");
        if (stats) {
            QG_CK(cudaMemcpyAsync(h.data(), c->d_grad, h.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream),
                  "grad copy");
            QG_CK(cudaStreamSynchronize(c->stream), "train sync");
            const double n = h[QG_NET_PARAMS + 3] > 0 ? h[QG_NET_PARAMS + 3] : 1.0;
            acc[0] += h[QG_NET_PARAMS] / n;
            acc[1] += h[QG_NET_PARAMS + 1] / n;
            acc[2] += h[QG_NET_PARAMS + 2] / n;
            acc[3] += h[QG_NET_PARAMS + 3];
        }
    }
    if (stats)
        for (int k = 0; k < 4; k++) stats[k] = steps > 0 ? acc[k] / steps : 0.0;
    return net_err_check(c);
}

static int measure_to_host(qg_ctx *c, int ncomp, double *out)
{
    QG_CK(cudaMemcpyAsync(c->h_results, c->d_results, ncomp * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
          "result copy");
    QG_CK(cudaStreamSynchronize(c->stream), "measure sync");
    for (int i = 0; i < ncomp; i++) out[i] = c->h_results[i];
    return QG_OK;
}

extern "C" int qg_measure_wilson(qg_ctx *c, int R, int T, double *out)
{
    if (!c || !out) return QG_ERR_ARG;
    if (R < 1 || T < 1 || R > c->G.n[0] || T > c->G.n[3]) return fail(c, QG_ERR_ARG, "Wilson loop extent out of range");
    const qg_config &f = c->cfg;
    int tw = !(f.phi == 0.0 && f.omega == 0.0);
    QG_CK(launch_wilson(c->G, c->links, f.group, f.precision, R, T, c->d_params, tw, c->partials, c->d_results,
                        c->stream), "wilson");
    return measure_to_host(c, 1, out);
}

extern "C" int qg_measure_wilson_all(qg_ctx *c, int Rmax, int Tmax, int fp64_products, double *out)
{
    NvtxRange nvtx_range("qg_measure_wilson_all");
    if (!c || !out) return QG_ERR_ARG;
    const int ns = std::min(c->G.n[0], std::min(c->G.n[1], c->G.n[2]));
    if (Rmax < 1 || Tmax < 1 || Rmax > 16 || Tmax > 16 || Rmax > ns || Tmax > c->G.n[3])
        return fail(c, QG_ERR_ARG, "Wilson loop extents must be in [1, 16] and within the lattice");
    const qg_config &f = c->cfg;
    int tw = !(f.phi == 0.0 && f.omega == 0.0);
    if (c->wpart_rmax < Rmax) {
        cudaFree(c->d_wpart);
        c->d_wpart = nullptr;
        QG_CK(cudaMalloc(&c->d_wpart, wilson_all_partials(wilson_all_blocks(c->G), Rmax) * sizeof(double)),
              "wilson scratch");
        c->wpart_rmax = Rmax;
    }
    if (!c->d_wout) QG_CK(cudaMalloc(&c->d_wout, 256 * sizeof(double)), "wilson scratch");
    QG_CK(launch_wilson_all(c->G, c->links, f.group, f.precision, Rmax, Tmax, fp64_products, c->d_params, tw,
                            c->d_wpart, c->d_wout, c->stream), "wilson all");
    QG_CK(cudaMemcpyAsync(out, c->d_wout, (size_t)Rmax * Tmax * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
          "wilson copy");
    QG_CK(cudaStreamSynchronize(c->stream), "wilson sync");
    return QG_OK;
}

extern "C" int qg_measure_fmunu(qg_ctx *c, int field, int index1, int index2, double *out)
{
    NvtxRange nvtx_range("qg_measure_fmunu");
    if (!c || !out) return QG_ERR_ARG;
    const qg_config &f = c->cfg;
    const int na = f.group == 3 ? 8 : 3;
    if (field != QG_FMUNU_H && field != QG_FMUNU_E) return fail(c, QG_ERR_ARG, "field must be QG_FMUNU_H or QG_FMUNU_E");
    if (index1 < 1 || index1 > na || index2 < 1 || index2 > na)
        return fail(c, QG_ERR_ARG, "generator index out of range (1..8 for SU(3), 1..3 for SU(2))");
    int tw = !(f.phi == 0.0 && f.omega == 0.0);
    if (!c->d_fpart) QG_CK(cudaMalloc(&c->d_fpart, fmunu_partials(c->G) * sizeof(double)), "fmunu scratch");
    if (!c->d_pout) QG_CK(cudaMalloc(&c->d_pout, 2 * 4096 * sizeof(double)), "measurement scratch");
    QG_CK(launch_fmunu(c->G, c->links, f.group, f.precision, c->d_params, tw, field, index1, index2, c->d_fpart,
                       c->d_pout, c->stream), "fmunu");
    QG_CK(cudaMemcpyAsync(out, c->d_pout, 12 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "fmunu copy");
    QG_CK(cudaStreamSynchronize(c->stream), "fmunu sync");
    return QG_OK;
}

static int measure_profile(qg_ctx *c, int kind, int axis, double *out)
{
    if (!c || !out) return QG_ERR_ARG;
    if (axis < 0 || axis > 2) return fail(c, QG_ERR_ARG, "profile axis must be 0 (x), 1 (y) or 2 (z)");
    if (c->G.n[axis] > 4096) return fail(c, QG_ERR_ARG, "profile longer than 4096 slices");
    const qg_config &f = c->cfg;
    int tw = !(f.phi == 0.0 && f.omega == 0.0);
    if (!c->d_ppart) QG_CK(cudaMalloc(&c->d_ppart, profile_partials(c->G) * sizeof(double)), "profile scratch");
    if (!c->d_pout) QG_CK(cudaMalloc(&c->d_pout, 2 * 4096 * sizeof(double)), "measurement scratch");
    QG_CK(launch_profile(c->G, c->links, f.group, f.precision, c->d_params, tw, kind, axis, c->d_ppart, c->d_pout,
                         c->stream), "profile");
    QG_CK(cudaMemcpyAsync(out, c->d_pout, 2 * (size_t)c->G.n[axis] * sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream), "profile copy");
    QG_CK(cudaStreamSynchronize(c->stream), "profile sync");
    return QG_OK;
}
static int measure_all(qg_ctx *c, int kind, double *out)
{
    if (!c || !out) return QG_ERR_ARG;
    const int nout = 4 + 2 * (c->G.n[0] + c->G.n[1] + c->G.n[2]);
    if (nout > 2 * 4096) return fail(c, QG_ERR_ARG, "profiles longer than the measurement buffer");
    const qg_config &f = c->cfg;
    int tw = !(f.phi == 0.0 && f.omega == 0.0);
    if (!c->d_ppart) QG_CK(cudaMalloc(&c->d_ppart, profile_partials(c->G) * sizeof(double)), "profile scratch");
    if (!c->d_pout) QG_CK(cudaMalloc(&c->d_pout, 2 * 4096 * sizeof(double)), "measurement scratch");
    if (!c->d_sites) QG_CK(cudaMalloc(&c->d_sites, sites_buffer_doubles(c->G) * sizeof(double)), "site buffer");
    QG_CK(launch_measure_all(c->G, c->links, f.group, f.precision, c->d_params, tw, kind, c->partials, c->d_ppart,
                             c->d_sites, c->d_pout, c->stream), "one-pass measurement");
    QG_CK(cudaMemcpyAsync(out, c->d_pout, (size_t)nout * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
          "measurement copy");
    QG_CK(cudaStreamSynchronize(c->stream), "measurement sync");
    return QG_OK;
}
extern "C" int qg_measure_plaquette_all(qg_ctx *c, double *out) { return measure_all(c, 0, out); }
extern "C" int qg_measure_polyakov_all(qg_ctx *c, double *out) { return measure_all(c, 1, out); }
extern "C" int qg_measure_action_profile(qg_ctx *c, int axis, double *out) { return measure_profile(c, 0, axis, out); }
extern "C" int qg_measure_polyakov_profile(qg_ctx *c, int axis, double *out) { return measure_profile(c, 1, axis, out); }

extern "C" int qg_measure(qg_ctx *c, int what, double *out)
{
    if (!c || !out) return QG_ERR_ARG;
    const qg_config &f = c->cfg;
    int tw = !(f.phi == 0.0 && f.omega == 0.0);
    switch (what) {
    case QG_MEAS_PLAQUETTE:
    case QG_MEAS_ACTION: {
        QG_CK(launch_plaquette(c->G, c->links, f.group, f.precision, c->d_params, tw, c->partials, c->d_results,
                               c->stream), "plaquette");
        double r[4];
        int rc = measure_to_host(c, 4, r);
        if (rc) return rc;
        if (what == QG_MEAS_PLAQUETTE) { out[0] = r[0]; out[1] = r[1]; }
        else { out[0] = r[2]; out[1] = r[3]; }
        return QG_OK;
    }
    case QG_MEAS_PLAQUETTE_F32:
        QG_CK(launch_plaquette_f32(c->G, c->links, f.group, f.precision, c->d_params, tw, c->partials, c->d_results,
                                   c->stream), "plaquette (FP32 products)");
        return measure_to_host(c, 2, out);
    case QG_MEAS_POLYAKOV:
        QG_CK(launch_polyakov(c->G, c->links, f.group, f.precision, c->partials, c->d_results, c->stream), "polyakov");
        return measure_to_host(c, 4, out);
    case QG_MEAS_WILSON:
        return qg_measure_wilson(c, f.wilson_r, f.wilson_t, out);
    default:
        return fail(c, QG_ERR_ARG, "unknown measurement");
    }
}

// the measurement kernels of `what` into d_results; ncomp values there
static int measure_launch(qg_ctx *c, int what, int &ncomp, int &first)
{
    const qg_config &f = c->cfg;
    int tw = !(f.phi == 0.0 && f.omega == 0.0);
    switch (what) {
    case QG_MEAS_PLAQUETTE:
    case QG_MEAS_ACTION:
        QG_CK(launch_plaquette(c->G, c->links, f.group, f.precision, c->d_params, tw, c->partials, c->d_results,
                               c->stream), "plaquette");
        ncomp = 2;
        first = what == QG_MEAS_PLAQUETTE ? 0 : 2;
        return QG_OK;
    case QG_MEAS_PLAQUETTE_F32:
        QG_CK(launch_plaquette_f32(c->G, c->links, f.group, f.precision, c->d_params, tw, c->partials, c->d_results,
                                   c->stream), "plaquette (FP32 products)");
        ncomp = 2;
        first = 0;
        return QG_OK;
    case QG_MEAS_POLYAKOV:
        QG_CK(launch_polyakov(c->G, c->links, f.group, f.precision, c->partials, c->d_results, c->stream), "polyakov");
        ncomp = 4;
        first = 0;
        return QG_OK;
    case QG_MEAS_WILSON:
        if (f.wilson_r < 1 || f.wilson_t < 1 || f.wilson_r > c->G.n[0] || f.wilson_t > c->G.n[3])
            return fail(c, QG_ERR_ARG, "Wilson loop extent out of range");
        QG_CK(launch_wilson(c->G, c->links, f.group, f.precision, f.wilson_r, f.wilson_t, c->d_params, tw, c->partials,
                            c->d_results, c->stream), "wilson");
        ncomp = 1;
        first = 0;
        return QG_OK;
    default:
        return fail(c, QG_ERR_ARG, "unknown measurement");
    }
}

extern "C" int qg_measure_enqueue(qg_ctx *c, int what, uint64_t *ticket)
{
    NvtxRange nvtx_range("qg_measure_enqueue");
    if (!c || !ticket) return QG_ERR_ARG;
    const uint64_t t = c->ticket_next;
    const int slot = (int)(t % QG_MEASURE_SLOTS);
    // the slot's previous copy must have landed before it is reused
    QG_CK(cudaEventSynchronize(c->ring_ev[slot]), "measure slot");
    int ncomp = 0, first = 0;
    int r = measure_launch(c, what, ncomp, first);
    if (r) return r;
    QG_CK(cudaMemcpyAsync(c->h_ring + 8 * slot, c->d_results + first, ncomp * sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream), "measure copy");
    QG_CK(cudaEventRecord(c->ring_ev[slot], c->stream), "measure event");
    c->ring_ticket[slot] = t;
    c->ring_what[slot] = what;
    c->ticket_next++;
    *ticket = t;
    return QG_OK;
}

extern "C" int qg_measure_fetch(qg_ctx *c, uint64_t ticket, double *out)
{
    if (!c || !out) return QG_ERR_ARG;
    const int slot = (int)(ticket % QG_MEASURE_SLOTS);
    if (ticket == 0 || c->ring_ticket[slot] != ticket)
        return fail(c, QG_ERR_ARG, "unknown measurement ticket (never issued, or more than QG_MEASURE_SLOTS ago)");
    QG_CK(cudaEventSynchronize(c->ring_ev[slot]), "measure fetch");
    const int n = c->ring_what[slot] == QG_MEAS_POLYAKOV ? 4 : c->ring_what[slot] == QG_MEAS_WILSON ? 1 : 2;
    for (int i = 0; i < n; i++) out[i] = c->h_ring[8 * slot + i];
    return QG_OK;
}

extern "C" int qg_links_upload(qg_ctx *c, const void *host, int layout)
{
    if (!c || !host) return QG_ERR_ARG;
    if (layout != QG_LAYOUT_REFERENCE) return fail(c, QG_ERR_ARG, "unknown layout");
    const size_t rsz = c->cfg.precision ? sizeof(double) : sizeof(float);
    const size_t bytes = (size_t)(c->cfg.group == 3 ? 12 : 4) * c->rowsize * 4 * rsz;
    void *tmp = nullptr;
    QG_CK(cudaMallocAsync(&tmp, bytes, c->stream), "upload staging");
    cudaError_t e = cudaMemcpyAsync(tmp, host, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_to_native(c->G, tmp, c->links, c->cfg.group, c->cfg.precision, c->rowsize, c->stream);
    cudaFreeAsync(tmp, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "links upload");
    QG_CK(cudaStreamSynchronize(c->stream), "upload sync");
    return QG_OK;
}

extern "C" int qg_links_download(qg_ctx *c, void *host, int layout)
{
    if (!c || !host) return QG_ERR_ARG;
    if (layout != QG_LAYOUT_REFERENCE) return fail(c, QG_ERR_ARG, "unknown layout");
    const size_t rsz = c->cfg.precision ? sizeof(double) : sizeof(float);
    const size_t bytes = (size_t)(c->cfg.group == 3 ? 12 : 4) * c->rowsize * 4 * rsz;
    void *tmp = nullptr;
    QG_CK(cudaMallocAsync(&tmp, bytes, c->stream), "download staging");
    cudaError_t e = cudaMemsetAsync(tmp, 0, bytes, c->stream);
    if (e == cudaSuccess) e = launch_to_ref(c->G, c->links, tmp, c->cfg.group, c->cfg.precision, c->rowsize, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(tmp, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "links download");
    QG_CK(cudaStreamSynchronize(c->stream), "download sync");
    return QG_OK;
}

extern "C" int qg_device_info(char *platform, size_t platform_len, char *device, size_t device_len)
{
    int rt = 0, dev = 0;
    cudaDeviceProp prop;
    cudaError_t e = cudaRuntimeGetVersion(&rt);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) {
        qg_set_global_error(std::string("qg_device_info: ") + cudaGetErrorString(e));
        return QG_ERR_CUDA;
    }
    if (platform && platform_len) snprintf(platform, platform_len, "CUDA %d.%d", rt / 1000, (rt % 1000) / 10);
    if (device && device_len) snprintf(device, device_len, "%s", prop.name);
    return QG_OK;
}
