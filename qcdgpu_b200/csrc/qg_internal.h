// qg_internal.h -- state shared by the CUDA translation units behind the
// C-ABI in include/qcdgpu_b200.h.  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/qcdgpu_b200.h"
#include <nvtx3/nvToolsExt.h>
#include "qg_lattice.cuh"

namespace qg {

struct PhaseArgs {
    int parity, dir;
    const double *params;    // device block {BETA/N, PHI, OMEGA} (lattice_parameters)
    int twist;               // PHI or OMEGA non-zero
    int nhit, nhitpar;
    int prn_mode;            // QG_PRNG_RANLUX / QG_PRNG_PHILOX / gid (2)
    const float4 *prns;      // reference-layout batch
    uint32_t prngstep;
    uint2 key;               // Philox key
    const uint64_t *phase_base;  // device counter (graph-replayable)
    uint32_t phase_offset;       // added to *phase_base
    int variant;                 // launch shape, 0 .. kPhaseVariants-1 (launch_phase_T)
    uint32_t t_begin, t_end;     // threads updated: [t_begin, t_end) (a slab: its interior x-slices)
    int32_t t_prn;               // added to the thread index for the Philox stream (a slab: its
                                 // threads' indices in the whole lattice)
};
constexpr int kPhaseVariants = QG_TUNE_SHAPES;

// launchers (return cudaError_t of the launch)
cudaError_t launch_phase_f32(const Geom &G, void *links, int group, const PhaseArgs &a, cudaStream_t s);
cudaError_t launch_phase_f64(const Geom &G, void *links, int group, const PhaseArgs &a, cudaStream_t s);

enum InitKind { INIT_COLD = 0, INIT_GID = 1, INIT_HOT_REF = 2, INIT_HOT_PHILOX = 3, INIT_HAAR = 4 };
cudaError_t launch_init(const Geom &G, void *links, int group, int prec, int kind, int dir,
                        const float4 *prns, uint32_t rowsize, uint2 key, cudaStream_t s);
cudaError_t launch_gramschmidt(const Geom &G, void *links, int group, int prec, int fp64, cudaStream_t s);
cudaError_t launch_to_native(const Geom &G, const void *ref, void *links, int group, int prec, uint32_t rowsize,
                             cudaStream_t s);
cudaError_t launch_to_ref(const Geom &G, const void *links, void *ref, int group, int prec, uint32_t rowsize,
                          cudaStream_t s);

// measurements: per-block partials into scratch, then a fixed-order final
// reduction into out (device).  Partials sizes returned by *_blocks().
uint32_t plaq_blocks(const Geom &G);
cudaError_t launch_plaquette(const Geom &G, const void *links, int group, int prec, const double *params, int twist,
                             double *partials, double *out, cudaStream_t s);
// the plaquette with FP32 products on FP32 links (as launch_plaquette on FP64 links)
cudaError_t launch_plaquette_f32(const Geom &G, const void *links, int group, int prec, const double *params,
                                 int twist, double *partials, double *out, cudaStream_t s);
uint32_t poly_blocks(const Geom &G);
cudaError_t launch_polyakov(const Geom &G, const void *links, int group, int prec, double *partials, double *out,
                            cudaStream_t s);
cudaError_t launch_wilson(const Geom &G, const void *links, int group, int prec, int R, int T, const double *params,
                          int twist, double *partials, double *out, cudaStream_t s);
cudaError_t launch_reduce(const double *partials, uint32_t nblocks, int ncomp, double *out, cudaStream_t s);
// F_munu sums (12) of the plaquettes of field 0 (xy,xz,yz) / 1 (xt,yt,zt)
uint32_t fmunu_partials(const Geom &G);
cudaError_t launch_fmunu(const Geom &G, const void *links, int group, int prec, const double *params, int twist,
                         int field, int i1, int i2, double *partials, double *out, cudaStream_t s);
// per-slice sums along axis 0..2: kind 0 action (spatial, temporal), kind 1
// Polyakov trace (Re, Im); out holds 2 n[axis] doubles
uint32_t profile_partials(const Geom &G);
// kind 0: plaquette/action totals (out[0..3] as k_plaquette) and the action
// profiles along x, y, z; kind 1: Polyakov totals (as k_polyakov) and its
// profiles; out[4 ..] = 2 n1 + 2 n2 + 2 n3 per-slice sums; sites holds
// sites_buffer_doubles(G)
size_t sites_buffer_doubles(const Geom &G);
cudaError_t launch_measure_all(const Geom &G, const void *links, int group, int prec, const double *params, int twist,
                               int kind, double *partials, double *ppartials, double *sites, double *out,
                               cudaStream_t s);
cudaError_t launch_profile(const Geom &G, const void *links, int group, int prec, const double *params, int twist,
                           int kind, int axis, double *partials, double *out, cudaStream_t s);
int wilson_all_blocks(const Geom &G);
size_t wilson_all_partials(int nbx, int Rmax);
cudaError_t launch_wilson_all(const Geom &G, const void *links, int group, int prec, int Rmax, int Tmax,
                              int fp64_products, const double *params, int twist, double *partials, double *out,
                              cudaStream_t s);
cudaError_t launch_add_u64(uint64_t *p, uint64_t v, cudaStream_t s);
// slab halo exchange: both sides of one (direction, parity) slice in one
// launch; `unit` = 16-byte words per link-plane element, src / dst offsets
// in those words
struct SlabCopy {
    const uint4 *src[6];
    uint4 *dst[6];
    int n;                 // copies (sides x planes)
    uint32_t words;        // 16-byte words per copy
};
cudaError_t launch_slab_copy(const SlabCopy &c, cudaStream_t s);

// a named NVTX range for the scope (shows the C-ABI calls on a profiler's
// timeline; nothing happens without a tool attached)
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
cudaError_t launch_field_check(const Geom &G, const void *links, int group, int prec, double tol,
                               unsigned long long *bad, cudaStream_t s);

// RANLUX, reference layout: one generator per instance, seed table of 7
// float4 per instance (SoA), output prns[s*instances + i]
cudaError_t launch_ranlux_init(const uint32_t *seeds, float4 *table, int instances, cudaStream_t s);
// a RANLUX batch split over `parts` threads per generator (qg_ranlux.cu):
// mult = parts x 18 limbs of the jump multipliers, seg = parts x 7 x
// instances float4 of segment start states; parts = 1: one thread each
struct RanluxSplit {
    int parts;
    const uint32_t *mult;
    float4 *seg;
};
int ranlux_split_parts(int instances, int samples);
void ranlux_split_multipliers(int samples, int nskip, int parts, uint32_t *out);
cudaError_t launch_ranlux_produce(float4 *table, float4 *prns, int instances, int samples, int nskip, cudaStream_t s,
                                  const RanluxSplit *split = nullptr);

Geom make_geom(const int n[4]);

// learned-proposal Metropolis (qg_learned.cu)
// eps_out non-null: only the per-link step into eps_out (no update); err:
// set when a tensor-core wait ran out
cudaError_t launch_mh_phase(const Geom &G, void *links, const PhaseArgs &a, const uint16_t *wq, double eps_max,
                            int nhit, unsigned long long *acc_count, double *jump_sum, float *eps_out, unsigned *err,
                            cudaStream_t s);
uint32_t mh_grad_blocks(const Geom &G);
cudaError_t launch_mh_grad(const Geom &G, const void *links, int parity, int dir, const double *params,
                           const uint16_t *wq, double eps_max, uint2 key, uint64_t phase, float *partials,
                           float *grad, unsigned *err, cudaStream_t s);
cudaError_t launch_adam(float *master, float *m, float *v, const float *grad, uint16_t *wq, float lr, float b1,
                        float b2, float c1, float c2, float epsa, cudaStream_t s);
cudaError_t launch_to_bf16(const float *master, uint16_t *wq, cudaStream_t s);

}  // namespace qg
