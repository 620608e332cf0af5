/*
 * qcdgpu_b200.h -- C-ABI of the B200 lattice sweep library (libqg_sun.so).
 *
 * This interface replaces the OpenCL kernel-ID layer through which the
 * QCDGPU reference (vadimdi/QCDGPU) drives its SU(2)/SU(3) Monte Carlo
 * sweep: GPU_CL::GPU::program_create / kernel_init / kernel_init_buffer /
 * kernel_init_constant / kernel_run / buffer_init / buffer_map
 * (SU(N)/clinterface/clinterface.cpp:921-1539) as called by
 * model_CL::model::lattice_make_programs / lattice_simulate /
 * lattice_analysis (SU(N)/suncl/suncl.cpp:3265-3648, 5212-5505, 1328-1612)
 * and PRNG_CL::PRNG::initialize / produce (SU(N)/random/random.cpp:216-284).
 *
 * Conventions: plain pointers and sizes only; every call returns an int
 * status (QG_OK = 0, negative on error; the message is in qg_last_error);
 * nothing exits, aborts or traps.  A context owns all device memory and
 * one CUDA stream; calls are asynchronous on that stream except those that
 * return host data, which synchronise it.  Contexts are independent: one
 * host thread per GPU may drive its own context.
 */
#ifndef QCDGPU_B200_H
#define QCDGPU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QG_OK              0
#define QG_ERR_ARG        -1
#define QG_ERR_CUDA       -2
#define QG_ERR_STATE      -3
#define QG_ERR_NOMEM      -4
#define QG_ERR_IO         -5
#define QG_ERR_UNSUPPORTED -6
#define QG_ERR_NUMERIC    -7   /* the field left SU(N) or is not finite (qg_field_check) */

/* start types: the reference's INTS key (0=hot, 1=cold, 2=gid),
 * SU(N)/suncl/suncl.cpp:725-730; QG_START_HAAR is new (Haar-distributed). */
#define QG_START_HOT   0
#define QG_START_COLD  1
#define QG_START_GID   2
#define QG_START_HAAR  3

/* PRN streams */
#define QG_PRNG_RANLUX 0   /* reference layout: RANLUX batch before every heatbath phase */
#define QG_PRNG_PHILOX 1   /* counter-based stream generated in registers              */

/* link layouts for upload/download */
#define QG_LAYOUT_REFERENCE 0  /* reference SoA planes, site index = lexicographic gid   */

/* update kinds */
#define QG_UPDATE_HEATBATH 0
#define QG_UPDATE_OVERRELAX 1

/* measurements (qg_measure) */
#define QG_MEAS_PLAQUETTE 0   /* out[0..1] = sum ReTr spatial / temporal plaquettes     */
#define QG_MEAS_ACTION    1   /* out[0..1] = sum (beta/N)(3N - ReTr) spatial / temporal */
#define QG_MEAS_POLYAKOV  2   /* out[0..3] = sum Re P, Im P, |P|^2, |P|^4 (traces)      */
#define QG_MEAS_WILSON    3   /* out[0]    = sum ReTr W(R,T) over sites and x,y,z       */
/* out[0..1] as QG_MEAS_PLAQUETTE, with the products of each plaquette and its
 * trace in FP32 on an FP32-link lattice (the site and lattice sums in FP64);
 * on an FP64-link lattice the same values as QG_MEAS_PLAQUETTE */
#define QG_MEAS_PLAQUETTE_F32 4

typedef struct qg_ctx qg_ctx;

/* Run configuration.  Field meanings follow the reference's init.dat keys
 * and model defaults (SU(N)/QCDGPU.cpp:98-220, SU(N)/suncl/suncl.cpp:289-464). */
typedef struct qg_config {
    int group;            /* GROUP: 2 or 3                                   */
    int size[4];          /* L1..L4 (N1=x, N2=y, N3=z, N4=t); N2 even        */
    int precision;        /* 0 = FP32 links, 1 = FP64 links                  */
    int start;            /* INTS / QG_START_*                               */
    double beta;          /* BETA                                            */
    double phi, omega;    /* PHI, OMEGA: twisted boundary (0,0 = periodic)   */
    int nhit;             /* NHIT: Kennedy-Pendleton tries                   */
    int nhitpar;          /* NHITPar                                         */
    int prng;             /* QG_PRNG_*                                       */
    int ranlux_nskip;     /* 24, 48, 97, 223 (RANLUX3), 389                  */
    int prng_instances;   /* RANLUX generator instances                      */
    uint32_t randseries;  /* RANDSERIES (seed; 0 is rejected)                */
    int row_align;        /* alignment of ROWSIZE / PRNGSTEP                 */
    int n_or;             /* overrelaxation sweeps after each heatbath sweep */
    int reunit_every;     /* global reunitarisation every n sweeps (0=never) */
    int reunit_fp64;      /* 1: global reunitarisation in FP64               */
    int wilson_r, wilson_t; /* WILSONR, WILSONT                              */
} qg_config;

typedef struct qg_info {
    uint32_t sites;       /* V                                               */
    uint32_t rowsize;     /* ROWSIZE of the reference layout                 */
    uint32_t prngstep;    /* PRNGSTEP                                        */
    uint32_t prng_samples;/* float4 per RANLUX instance per batch            */
    uint64_t link_bytes;  /* device bytes of the link field                  */
    uint64_t ref_elems;   /* Real elements of a reference-layout table       */
    uint64_t prn_quads;   /* float4 in one RANLUX batch                      */
    uint64_t phase_counter;/* Philox phase counter (next phase)              */
    uint32_t prng_counter;/* RANLUX batches produced (PRNG_counter)          */
    uint64_t sweeps_done; /* sweeps since the start (reunitarisation cadence)*/
} qg_info;

/* defaults of the reference main() where it has one (QCDGPU.cpp:98-220) */
int qg_default_config(qg_config *cfg);

/* model::lattice_init + lattice_create_buffers (suncl.cpp:672-706,3877-3991):
 * validates cfg, allocates the field, PRN and measurement buffers. */
int qg_create(const qg_config *cfg, qg_ctx **out);
int qg_destroy(qg_ctx *ctx);
const char *qg_last_error(const qg_ctx *ctx);  /* ctx may be NULL (last create error) */
int qg_get_info(qg_ctx *ctx, qg_info *info);
/* the context's configuration: as created, with beta/phi/omega as last set
 * by qg_set_params                                                        */
int qg_get_config(qg_ctx *ctx, qg_config *cfg);
int qg_sync(qg_ctx *ctx);

/* PRNG::initialize (random.cpp:216-277): glibc srand(series) seeding of all
 * RANLUX instances, then one produce(); in Philox mode sets the key.      */
int qg_prng_seed(qg_ctx *ctx, uint32_t randseries);
/* Host only (no GPU needed): the RANLUX instance seeds PRNG::initialize
 * derives from RANDSERIES -- instance 0 = rand() % (2^31-1), instances
 * 1..n-1 = the next rand() values after srand(series) (random.cpp:228-235,
 * 462-465, 508) -- computed on a private glibc random_r state.           */
int qg_glibc_seeds(uint32_t randseries, int n, uint32_t *seeds);
/* PRNG::produce (random.cpp:278-284): one reference-layout RANLUX batch.  */
int qg_prng_produce(qg_ctx *ctx);
/* RANLUX lookahead (new; on by default): qg_sweep generates the next
 * sweep's 8 batches on a second stream while the current sweep's phases
 * run (8 more batch buffers, allocated on the first RANLUX sweep when they
 * leave 1 GiB free).  The batches, and which phase reads which, are
 * unchanged; qg_prng_produce / qg_prns_upload / qg_prns_download /
 * qg_prng_seed first return the generator to the last batch consumed, and
 * qg_prns_download after sweeps returns that batch, as without it.       */
int qg_set_prng_lookahead(qg_ctx *ctx, int on);
int qg_prns_upload(qg_ctx *ctx, const float *host_quads, uint64_t nquads);
int qg_prns_download(qg_ctx *ctx, float *host_quads, uint64_t nquads);

/* lattice_init_{cold,gid,hot_X..T} kernels and their PRN cadence
 * (suncl.cl:56-347, suncl.cpp:5236-5252).                                 */
int qg_init_links(qg_ctx *ctx, int start);

/* one update_{even,odd}_{X,Y,Z,T} kernel (suncl.cl:399-975) or its
 * overrelaxation counterpart; parity 0 = even, 1 = odd.  In RANLUX mode the
 * caller produces the batch first, as lattice_simulate does.              */
int qg_phase(qg_ctx *ctx, int parity, int dir, int kind);
/* the reference's working sweep (suncl.cpp:5393-5412): for each of odd
 * X,Y,Z,T, even X,Y,Z,T a RANLUX batch (RANLUX mode) and a heatbath phase,
 * then cfg.n_or overrelaxation sweeps in the same phase order, and a
 * global reunitarisation when the sweep count hits cfg.reunit_every.
 * Replayed from a captured CUDA graph.                                    */
int qg_sweep(qg_ctx *ctx, int nsweeps);
/* (new) nsweeps (1..256) sweeps of the qg_sweep chain -- the same launches,
 * Philox stream, reunitarisation cadence and counters, so the chain goes on
 * exactly as after qg_sweep(ctx, nsweeps) -- replayed from one graph with an
 * event before and after every phase launch and around the whole;
 * *ms_heatbath and *ms_overrelax are the mean durations of one heatbath and
 * one overrelaxation phase inside the sweep graph (0 without
 * overrelaxation), *ms_sweep that of a whole sweep in it.  Synchronous.
 * The RANLUX mode returns QG_ERR_UNSUPPORTED.                              */
int qg_sweep_phase_times(qg_ctx *ctx, int nsweeps, double *ms_heatbath, double *ms_overrelax, double *ms_sweep);
/* Autotuner (new): times each launch shape of the heatbath and the
 * overrelaxation phase kernels on this context's lattice (`reps` launches
 * each; the field is restored and no PRN counter moves) and keeps the
 * fastest for later phases and sweeps.  Shapes: 0 = links loaded straight
 * into registers, compiler's register count; 1, 2 = the same held to 5 / 6
 * resident blocks per SM; 3, 4 = staple links streamed through shared
 * memory two staple terms ahead (SU(3) FP32; other cases run shape 0 / 1);
 * 5 = overrelaxation two links per thread with packed FP32 (FFMA2)
 * arithmetic (SU(3) FP32, periodic boundaries; otherwise shape 4).
 * All shapes compute the same operation sequence.  times_ms (optional,
 * 2*QG_TUNE_SHAPES floats): per shape v, [2v] heatbath and [2v+1]
 * overrelaxation ms/launch.                                               */
#define QG_TUNE_SHAPES 6
int qg_tune(qg_ctx *ctx, int reps, float *times_ms);
/* pin / read the launch shapes (0 .. QG_TUNE_SHAPES-1) without tuning     */
int qg_set_shapes(qg_ctx *ctx, int heatbath_shape, int overrelax_shape);
int qg_get_shapes(qg_ctx *ctx, int *heatbath_shape, int *overrelax_shape);
/* lattice_GramSchmidt kernel (suncl.cl:350-396); fp64 != 0 computes in FP64 */
int qg_reunitarize(qg_ctx *ctx, int fp64);
/* new: count the links whose stored rows are not finite, not of unit norm
 * or not orthogonal to within tol (one pass over the field, synchronous);
 * qg_run checks its final configuration this way (tol 1e-3 for FP32 links,
 * 1e-9 for FP64) and returns QG_ERR_NUMERIC if any link fails.           */
int qg_field_check(qg_ctx *ctx, double tol, uint64_t *bad_links);
/* per-kernel device times (the reference's GPU_debug.profiling table,
 * clinterface.cpp:1254-1266,1626-1668): `reps` launches of each class, each
 * between two CUDA events, on the live field (restored; no PRN counter
 * moves); mean and standard deviation in ms per launch, indexed by class */
#define QG_KERNEL_HEATBATH   0   /* one heatbath phase                          */
#define QG_KERNEL_OVERRELAX  1   /* one overrelaxation phase                    */
#define QG_KERNEL_REUNIT     2   /* global Gram-Schmidt                         */
#define QG_KERNEL_PLAQUETTE  3   /* plaquette / action measurement + reduction  */
#define QG_KERNEL_POLYAKOV   4   /* Polyakov-loop measurement + reduction       */
#define QG_KERNEL_WILSON     5   /* one WILSONR x WILSONT loop + reduction      */
#define QG_KERNEL_CLASSES    6
int qg_profile_kernels(qg_ctx *ctx, int reps, double *mean_ms, double *sigma_ms);
/* x-slabs (the BIGLAT decomposition, suncl.cpp:4004-4062, as x-slices of
 * one lattice): a context created with size[0] = w + 2 becomes slab
 * [x0, x0 + w) of a lattice with n1_global x-slices; its slices 0 and w+1
 * are halos (global x0 - 1 and x0 + w).  qg_phase then updates the w
 * interior slices only, with the whole lattice's parity and Philox thread
 * indices, so every slab draws the numbers the undecomposed lattice draws.
 * Philox stream, periodic boundaries, even global N1; starts cold or from
 * qg_links_upload; qg_sweep is refused (phases need halo exchanges).      */
int qg_set_slab(qg_ctx *ctx, int x0, int n1_global);
/* halo exchange of the links of direction dir and global parity p: to_buf
 * = 1 packs boundary slice x = 1 (side 0) or x = w (side 1) into buf
 * (device or pinned host memory, qg_slab_halo_bytes bytes: the planes one
 * after another), to_buf = 0 unpacks buf into halo slice x = 0 (side 0) or
 * x = w + 1 (side 1).  Side 1 of a slab feeds side 0 of its right
 * neighbour and vice versa.  Asynchronous on the context's stream.       */
int qg_slab_halo(qg_ctx *ctx, int dir, int parity, int side, void *buf, int to_buf);
/* both sides in one kernel launch: buf_lo for side 0, buf_hi for side 1
 * (device memory, 16-byte aligned, qg_slab_halo_bytes bytes each)        */
int qg_slab_halo2(qg_ctx *ctx, int dir, int parity, void *buf_lo, void *buf_hi, int to_buf);
/* qg_phase of a slab in two parts, so that the exchange of the boundary
 * links overlaps the interior update: part 0 updates the boundary slices
 * x = 1 and x = w, part 1 the slices 2 .. w-1 (and advances the heatbath
 * PRN counter).  Part 0 then part 1 equals qg_phase bit for bit.          */
int qg_slab_phase(qg_ctx *ctx, int parity, int dir, int kind, int part);
int qg_slab_halo_bytes(qg_ctx *ctx, uint64_t *bytes);

/* lattice_measurement_plq / lattice_measurement / lattice_polyakov /
 * lattice_measurement_wilson + their reductions (sun_measurements_cl.cl:
 * 55-184,1178-1357; polyakov.cl:54-140,405-432; wilson_loop.cl:55-465).
 * Results are raw lattice sums (normalise as suncl.cpp:1328-1612 does).
 * Synchronous: out is host memory.                                        */
int qg_measure(qg_ctx *ctx, int what, double *out);
/* Asynchronous form (new): qg_measure_enqueue puts qg_measure(what)'s
 * kernels and the copy of its result into a pinned host slot on the
 * context's stream and returns at once with a ticket; qg_measure_fetch
 * waits for that ticket's copy and writes the same values qg_measure gives
 * (2, 2, 4 or 1 doubles).  A run loop can so read every step's result
 * without stalling the device between steps.  Up to QG_MEASURE_SLOTS
 * tickets are kept; an older ticket is an error.                          */
#define QG_MEASURE_SLOTS 64
int qg_measure_enqueue(qg_ctx *ctx, int what, uint64_t *ticket);
int qg_measure_fetch(qg_ctx *ctx, uint64_t ticket, double *out);
/* same, generalised Wilson loop of extent R x T (config keys WILSONR/T)   */
int qg_measure_wilson(qg_ctx *ctx, int R, int T, double *out);
/* all planar Wilson loops R x T for R <= Rmax, T <= Tmax (both <= 16): in
 * one launch, out[(R-1)*Tmax + (T-1)] = the raw sum qg_measure_wilson
 * gives (new; the reference measures one R x T per run).  fp64_products:
 * 1 = matrix products in FP64 as qg_measure_wilson; 0 = in FP32 on FP32
 * links (traces summed in FP64; about 4x faster, relative error ~1e-6)  */
int qg_measure_wilson_all(qg_ctx *ctx, int Rmax, int Tmax, int fp64_products, double *out);

/* F_munu: the projections -i Tr(P T_a) of every plaquette P of three planes
 * onto two group generators, summed over sites (the FMUNU / F0MU variants
 * of lattice_measurement_plq, sun_measurements_cl.cl:712-1175, with
 * trace_lambda1..8_double, su3_measurements_cl.cl:355-460, and
 * trace_sigma1..3_double, su2_measurements_cl.cl:89-124).  field:
 * QG_FMUNU_H = planes xy, xz, yz (chromomagnetic, key FMUNU), QG_FMUNU_E =
 * xt, yt, zt (chromoelectric, key F0MU).  T_a = lambda_a / 2 (SU(3),
 * a = 1..8; the reference offers index1 in {1,2,3,4}, default 3, and
 * index2 in {5,6,7,8}, default 8) or sigma_a / 2 (SU(2), a = 1..3, real
 * part only; reference: index1 3 or 1, index2 2).  out[12]: out[2p],
 * out[2p+1] = Re, Im sum for index1 and plane p; out[6+2p], out[7+2p] for
 * index2.  Normalise by the number of sites (suncl.cpp:1613-1670).
 * Allocates its scratch on first use.                                      */
#define QG_FMUNU_H 0
#define QG_FMUNU_E 1
int qg_measure_fmunu(qg_ctx *ctx, int field, int index1, int index2, double *out);
/* Profiles along coordinate axis (0 x, 1 y, 2 z), out[2 n[axis]]:
 * action: out[2i], out[2i+1] = sum over the sites with coordinate i of the
 * spatial and temporal action (beta/N)(3N - ReTr) (lattice_action_diff_
 * {x,y,z}, sun_measurements_cl.cl:187-615; normalise by 3 V / n[axis],
 * suncl.cpp:1376-1481); Polyakov: out[2i], out[2i+1] = sum of Re, Im Tr P
 * over the spatial sites with coordinate i (lattice_polyakov_diff_{x,y,z},
 * polyakov.cl:142-402; normalise by N n1 n2 n3 / n[axis],
 * suncl.cpp:1497-1586).  Allocate their scratch on first use.            */
int qg_measure_action_profile(qg_ctx *ctx, int axis, double *out);
int qg_measure_polyakov_profile(qg_ctx *ctx, int axis, double *out);
/* One-pass forms (new): the per-site work once for the totals and the
 * profiles along all three axes.  out[0..3] = qg_measure's four sums
 * (plaquette: ReTr spatial, temporal, action spatial, temporal; Polyakov:
 * Re P, Im P, |P|^2, |P|^4), then 2 n1 + 2 n2 + 2 n3 per-slice sums along
 * x, y, z (action spatial, temporal; Polyakov Re, Im).  Bit-identical to
 * qg_measure and qg_measure_*_profile; allocate a 2 V-double site buffer
 * on first use.                                                            */
int qg_measure_plaquette_all(qg_ctx *ctx, double *out);
int qg_measure_polyakov_all(qg_ctx *ctx, double *out);

/* buffer_init / buffer_map of the link table (clinterface.cpp:1296-1434):
 * host arrays in the reference layout, Real = float (precision 0) or
 * double (precision 1), qg_info.ref_elems elements.                       */
int qg_links_upload(qg_ctx *ctx, const void *host, int layout);
int qg_links_download(qg_ctx *ctx, void *host, int layout);

/* the per-run parameter block the kernels read from device memory, as
 * the reference's lattice_parameters buffer {BETA/N, PHI, OMEGA}
 * (suncl.cpp:3936-3949): stream-ordered host->device copy from one of 8
 * pinned staging slots (the call does not wait for the stream); later
 * sweeps and measurements use the new values.                            */
int qg_set_params(qg_ctx *ctx, double beta, double phi, double omega);
/* the context's CUDA stream (cudaStream_t), for event timing / interop   */
int qg_get_stream(qg_ctx *ctx, void **stream);

/* Philox phase counter (fast mode): read / set for checkpoint and resume */
int qg_set_phase_counter(qg_ctx *ctx, uint64_t counter);
/* sweeps counted for the reunitarisation cadence (qg_info.sweeps_done):
 * set on resume so that the global Gram-Schmidt falls on the same sweeps */
int qg_set_sweeps_done(qg_ctx *ctx, uint64_t sweeps);

/* Allocation-free plaquette/action sums.  No counterpart in the reference:
 * it exists for callers that may not allocate device memory at the call
 * site -- a program embedded in a framework that owns the device memory
 * pool, or a latency-critical loop where cudaMalloc/cudaFree would
 * synchronise the device.  The caller passes device pointers: `links`, a
 * reference-layout table (QG_LAYOUT_REFERENCE; float if precision == 0,
 * double if 1; `rowsize` >= sites) and `out`, four doubles receiving the
 * sums of qg_measure: spatial and temporal Re Tr plaquette, spatial and
 * temporal (beta/N)(3N - Re Tr).  Periodic boundaries.  Work is queued on
 * `stream` (NULL = legacy default stream); nothing is allocated or freed.
 * The per-block partial sums use a fixed 512 KiB array inside the library,
 * present on every GPU that loads it until the process exits, so lattices
 * are limited to 2^24 sites (64^4); larger ones are rejected with
 * QG_ERR_ARG.  The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress) and keeps it for the process; make that
 * first call before any stream capture.  The address belongs to the
 * device's primary context: after cudaDeviceReset the entry point must not
 * be called again in that process.  All calls share the array: calls whose
 * kernels may overlap on the GPU race and must be ordered by the caller.
 * A CUDA error already pending when the call starts is reported as
 * QG_ERR_CUDA and left pending.  Errors: qg_last_error(NULL). */
int qg_plaquette_noalloc(const void *links, int group, int precision, const int size[4], uint32_t rowsize,
                         double beta, double *out, void *stream);

/* ===================================================================== */
/* Learned local proposal with an exact Metropolis step (new; the          */
/* reference has only the heatbath).  SU(3), FP32 links, Philox stream,    */
/* periodic boundaries.  Each hit proposes, per SU(2) subgroup of the link */
/* U_mu(x), U' = X U with X = exp(i eps a.sigma), a ~ N(0,1)^3, accepted   */
/* with min(1, exp(-dS)) for the Wilson action.  eps = eps_max sigmoid(f)  */
/* with f a 3-layer network (QG_NET_FEATURES -> QG_NET_HIDDEN ->           */
/* QG_NET_HIDDEN -> 1, ReLU) of gauge-invariant features of the staple     */
/* alone (Tr AA^+, Tr (AA^+)^2, det A, 1x2 loop traces Tr F B^+ per plane),*/
/* which no link of the phase changes: the proposal is symmetric and the   */
/* chain exact for any weights.  Weights are BF16 in the kernels, FP32 for */
/* the optimiser; the network is trained on the GPU to maximise the        */
/* expected squared jump distance.  Its layers run on the tcgen05 tensor   */
/* cores (128 links per MMA, BF16 operands, FP32 accumulators in tensor    */
/* memory), forward and backward.  Layout of the QG_NET_PARAMS floats:      */
/* W1[32][8], b1[32], W2[32][32], b2[32], w3[32], b3.                       */
/* The tensor-core waits are bounded: a wait that runs out makes the next  */
/* qg_net_eps / qg_net_grad / qg_net_train / qg_mh_stats return QG_ERR_CUDA. */
/* ===================================================================== */
#define QG_NET_FEATURES 8
#define QG_NET_HIDDEN 32
#define QG_NET_PARAMS 1377
/* set the FP32 master weights (the kernels use their BF16 rounding) and
 * eps_max in (0, 3.2]; resets the optimiser state                          */
int qg_net_set(qg_ctx *ctx, const float *params, double eps_max);
/* master: FP32 master weights; weights_bf16: the BF16 weights as floats   */
int qg_net_get(qg_ctx *ctx, float *master, float *weights_bf16);
/* one Metropolis phase (parity, dir) with nhit hits per subgroup and link */
int qg_mh_phase(qg_ctx *ctx, int parity, int dir, int nhit);
/* the step eps of every link of phase (parity, dir) -- the values the next
 * qg_mh_phase on the same field and weights uses -- into eps[sites/2], in
 * the phase's link order (the t-th link of the (parity, dir) class); the
 * field is not changed                                                     */
int qg_net_eps(qg_ctx *ctx, int parity, int dir, float *eps);
/* nsweeps sweeps of Metropolis phases in the heatbath's phase order, with
 * the global reunitarisation on qg_sweep's cadence                         */
int qg_mh_sweep(qg_ctx *ctx, int nsweeps, int nhit);
/* acceptance rate and mean squared jump angle per proposal since the last
 * reset, and the number of proposals; reset != 0 clears them             */
int qg_mh_stats(qg_ctx *ctx, double *accept_rate, double *jump_per_hit, uint64_t *hits, int reset);
/* gradient (QG_NET_PARAMS floats) of the training loss -- minus the mean
 * over the phase's links of sum_subgroups min(1, exp(-dS)) (eps|a|)^2 for
 * proposals from the current links -- and stats = {loss, ESJD, mean
 * acceptance, links}; the field is not changed                             */
int qg_net_grad(qg_ctx *ctx, int parity, int dir, float *grad, double *stats);
/* steps Adam steps (learning rate lr) on the current field, step s on the
 * links of phase s % 8; stats (optional) = mean of qg_net_grad's stats     */
int qg_net_train(qg_ctx *ctx, int steps, double lr, double *stats);

/* ===================================================================== */
/* Batched ensembles (new; no counterpart in the reference, which runs one */
/* lattice per process): many independent lattices of one group and link   */
/* precision -- different extents, couplings and seeds, e.g. a beta scan --  */
/* updated together.  Each phase is ONE launch over all ensembles (a block  */
/* finds its ensemble in a prefix table of block counts), the sweep and the */
/* measurement are captured in one CUDA graph, and the measurements stay in */
/* device memory until read.  Philox stream only.  Ensemble e's chain is    */
/* bit-identical to a single context (qg_create) with its extents, coupling */
/* and RANDSERIES and the common settings (start, NHIT, n_or, cadences).    */
/* Errors: qg_last_error(NULL).                                             */
/* ===================================================================== */
typedef struct qg_ensemble {
    int size[4];          /* L1..L4, N2 even                                 */
    double beta;          /* BETA                                            */
    uint32_t randseries;  /* Philox key (non-zero)                           */
} qg_ensemble;
typedef struct qg_batch qg_batch;
/* common: group, precision, prng (must be QG_PRNG_PHILOX), nhit, nhitpar,
 * n_or, reunit_every, reunit_fp64, row_align (for downloads); its size,
 * beta and randseries are ignored.  max_measurements: capacity of the
 * device series (measurements beyond it are dropped and reported).        */
int qg_batch_create(const qg_config *common, const qg_ensemble *ens, int n, int max_measurements, qg_batch **out);
int qg_batch_destroy(qg_batch *b);
/* QG_START_COLD / HOT (Philox hot start) / HAAR for every ensemble; resets
 * the phase and measurement counters                                      */
int qg_batch_init(qg_batch *b, int start);
/* phase-kernel launch shapes of the batched launches, numbered as for
 * qg_tune (0-4; shape 5 is single-lattice only): set_shape sets both kinds,
 * set_shapes each; qg_batch_tune (new) times every shape of both kinds on
 * the live fields (restored; no counter moves), keeps the fastest per kind
 * and, if times_ms is given (2*QG_BATCH_SHAPES floats), stores per shape v
 * [2v] heatbath and [2v+1] overrelaxation ms per launch.  All shapes
 * compute the same operation sequence.                                    */
#define QG_BATCH_SHAPES 5
int qg_batch_set_shape(qg_batch *b, int shape);
int qg_batch_set_shapes(qg_batch *b, int heatbath_shape, int overrelax_shape);
int qg_batch_get_shapes(qg_batch *b, int *heatbath_shape, int *overrelax_shape);
int qg_batch_tune(qg_batch *b, int reps, float *times_ms);
/* enable != 0: each half-sweep (the four direction phases of one parity) is
 * ONE persistent launch over all ensembles -- every resident block walks
 * the batch's tiles direction by direction with a grid barrier between
 * directions (cooperative launch; the same chains bit for bit).  A barrier
 * that does not complete within a second sets a device flag and the blocks
 * return; qg_batch_sync / qg_batch_series then return QG_ERR_CUDA (the
 * fields are then not consistent) and clear the flag.  Default: off.       */
int qg_batch_set_persistent(qg_batch *b, int enable);
/* (new) the plaquette and action sums of the measurement series with each
 * plaquette's products and trace in FP32 (FP32 links; the sums of
 * QG_MEAS_PLAQUETTE_F32), fp32 = 1, or in FP64 as the reference (0, the
 * default).  The Polyakov sums and FP64-link batches are unchanged.        */
int qg_batch_set_measure_products(qg_batch *b, int fp32);
/* test of the bounded barrier: one persistent heatbath half-sweep in which
 * block skip_block leaves out its first arrival; every other block's wait
 * runs out.  Returns QG_ERR_CUDA (the flag) when the timeout path works; it
 * changes the fields.                                                      */
int qg_batch_barrier_test(qg_batch *b, int skip_block);
/* nsweeps sweeps of every ensemble (graph replays); after every
 * measure_every-th sweep (0 = never) plaquette, action and Polyakov sums of
 * every ensemble are appended to the device series                         */
int qg_batch_run(qg_batch *b, int nsweeps, int measure_every);
int qg_batch_sync(qg_batch *b);
int qg_batch_get_stream(qg_batch *b, void **stream);
/* the series: out[m][e][8] = sum ReTr spatial, temporal, sum (beta/N)(3N -
 * ReTr) spatial, temporal, sum Re P, Im P, |P|^2, |P|^4 (qg_measure's raw
 * sums); *n_measurements = measurements held.  QG_ERR_STATE if any were
 * dropped for capacity.                                                   */
int qg_batch_series(qg_batch *b, double *out, uint64_t max_measurements, uint64_t *n_measurements);
/* ensemble e's links in the reference layout (row_align of common)        */
int qg_batch_links_download(qg_batch *b, int e, void *host);
int qg_batch_info(qg_batch *b, uint64_t *total_sites, uint64_t *sweeps_done, uint64_t *field_bytes);

/* ===================================================================== */
/* Host driver: the reference's init.dat run setup, run loop and output   */
/* (SU(N)/QCDGPU.cpp:61-269, model::lattice_get_init_file / lattice_init / */
/* lattice_simulate / lattice_analysis / lattice_write_results,            */
/* SU(N)/suncl/suncl.cpp:289-464, 5212-5505, 1328-1854).                   */
/* ===================================================================== */

/* observables of a run, in the reference's results order */
#define QG_OBS_S_TOTAL      0
#define QG_OBS_PLQ_TOTAL    1
#define QG_OBS_POLYAKOV     2
#define QG_OBS_POLYAKOV_IM  3
#define QG_OBS_POLYAKOV_P2  4
#define QG_OBS_POLYAKOV_P4  5
#define QG_OBS_WILSON       6
#define QG_OBS_PLQ_SPAT     7
#define QG_OBS_PLQ_TEMP     8
#define QG_OBS_S_SPAT       9
#define QG_OBS_S_TEMP      10
#define QG_OBS_COUNT       11
#define QG_FMUNU_COLS      16

typedef struct qg_run_options {
    int iter;              /* ITER: measurements, the first on the start configuration */
    int niter;             /* NITER: sweeps between measurements                       */
    int nav;               /* NAV: thermalisation sweeps                               */
    int pl_level;          /* PL_LEVEL: 0 none, 1 P, >= 2 P, |P|^2, |P|^4              */
    int get_wilson;        /* GETWILSON                                                */
    int get_plaquettes;    /* GETRETRACE / plaquette averages                         */
    int get_actions;       /* action averages                                          */
    int verify;            /* CPU FP64 re-measurement of the last configuration       */
    int write_results;     /* write the results .txt                                   */
    int quiet;             /* no console output                                        */
    char output_path[512]; /* OUTPUTPATH (directory prefix of the results file)        */
    char prefix[32];       /* file prefix, "su3-" / "su2-"                              */
    int init;              /* INIT: 1 start from cfg.start, 0 continue from state_file  */
    char state_file[512];  /* STATEFILE: .qcg read when init == 0                       */
    int save_state;        /* SAVESTATE: 1 write a .qcg after the start measurement and */
                           /* at the end, as lattice_simulate does                      */
    int save_every_iter;   /* SAVEEVERY: also after every n-th measured iteration (0 off)*/
    char state_out[512];   /* STATEOUT: .qcg path written (empty: OUTPUTPATH + prefix + */
                           /* the reference's date-stamped name)                       */
    int fmunu;             /* F_munu every measurement: 0 off (TURNOFFFMUNU), 1 planes   */
                           /* xy,xz,yz (FMUNU), 2 planes xt,yt,zt (F0MU)               */
    int fmunu_index1;      /* generator of the first F series: 0 = the reference's     */
                           /* default 3 (FMUNU1/2/4 keys: 1, 2, 4)                     */
    int fmunu_index2;      /* second: 0 = default 8 (SU(3), FMUNU5/6/7: 5..7), 2 (SU(2))*/
    int get_actions_diff;  /* action profiles along x, y, z (ACTIONS_DIFF; the         */
                           /* reference's get_actions_diff, set in its main())         */
    int tune_shapes;       /* 1 (default): time the phase-kernel launch shapes on this */
                           /* lattice before the run (qg_tune; all shapes give the     */
                           /* same chain, so the results do not change)               */
    int profile;           /* PROFILE: per-kernel time table after the run            */
                           /* (qg_profile_kernels; printed unless quiet, and in        */
                           /* qg_run_result.kernel_ms)                                 */
} qg_run_options;

typedef struct qg_run_result {
    double mean[QG_OBS_COUNT];       /* over samples 1..ITER-1 (sample 0 dropped)  */
    double variance[QG_OBS_COUNT];
    double gpu_last[QG_OBS_COUNT];
    double cpu_last[QG_OBS_COUNT];   /* host FP64 re-measurement (verify)          */
    int verification_passed;         /* 1 passed, 0 failed, -1 not run             */
    int samples;
    double seconds;                  /* wall time of the update + measure loop     */
    double link_updates_per_second;
    char results_file[640];
    /* new: integrated autocorrelation time of each series over samples
     * 1..ITER-1 (Madras-Sokal window, c = 6) and the error of its mean,
     * sqrt(2 tau_int variance / n); the reference reports neither        */
    double tau_int[QG_OBS_COUNT];
    double error[QG_OBS_COUNT];
    char state_file[640];            /* last .qcg written ("" if none)             */
    /* F_munu series (when opts.fmunu): the reference's 16 columns in its
     * order (DM_Fmunu_3 .. DM_Fmunu_abs_8_im, suncl.h:235-252): planes
     * p0, p1, p2 of generator index1 (Re, Im each), the same for index2,
     * then |F| = sqrt of the sum of squares over the planes (Re, Im) for
     * index1 and index2; each normalised by the number of sites          */
    double fmunu_mean[QG_FMUNU_COLS];
    double fmunu_variance[QG_FMUNU_COLS];
    double fmunu_gpu_last[QG_FMUNU_COLS];
    double fmunu_cpu_last[QG_FMUNU_COLS];
    /* opts.profile: ms per launch of each QG_KERNEL_* class, mean and sigma */
    double kernel_ms[QG_KERNEL_CLASSES];
    double kernel_ms_sigma[QG_KERNEL_CLASSES];
} qg_run_result;

/* Writes a run's results file in the reference's layout (model::
 * lattice_write_results with lattice_make_header, model_make_header and
 * lattice_make_header2, SU(N)/suncl/suncl.cpp:534-615,779-865,1679-1854):
 * opts->output_path + opts->prefix + the reference's date-stamped name
 * (from t_end) + ".txt"; the same sections, labels, column widths and
 * order as the reference's GPU build, its device lines naming the CUDA
 * platform and device; the F_munu blocks are always present (zero when
 * F_munu is not measured), as the reference prints them.  What this
 * library adds -- tau_int and the error of every mean, the overrelaxation
 * and reunitarisation settings, the update rate -- goes to a companion file
 * of the same name ending in "-stats.txt".  qg_run calls it; host only.
 *   series:   [QG_OBS_COUNT][opts->iter] per-measurement values (zero for
 *             observables not measured)
 *   fmunu:    [QG_FMUNU_COLS][opts->iter] (opts->fmunu) or NULL
 *   profiles: for axis 0..2 and each slice 6 values -- PL, PL_im,
 *             PL_variance, PL_im_variance, S, S_variance (needed when
 *             opts->pl_level > 2 or opts->get_actions_diff) or NULL
 *   fmunu_cpu_lattice_variance: the 12 "CPU l.varnc" values or NULL (zero)
 *   t_start, t_end: wall-clock times of the run (seconds since the epoch)
 * path (path_len bytes) receives the results file's name.                 */
int qg_write_results(const qg_config *cfg, const qg_run_options *opts, const qg_run_result *res, int resumed,
                     const double *series, const double *fmunu, const double *profiles,
                     const double *fmunu_cpu_lattice_variance, int64_t t_start, int64_t t_end,
                     const char *platform, const char *device, char *path, size_t path_len);
/* the CUDA runtime ("CUDA 12.9") and the current device's name            */
int qg_device_info(char *platform, size_t platform_len, char *device, size_t device_len);

/* defaults of the reference main() (QCDGPU.cpp:183-205) */
int qg_default_run_options(qg_run_options *opts);
/* Host only: read KEY = value lines ('#' starts a comment) and apply the
 * keys onto cfg / opts as lattice_get_init_file does.  Keys: GROUP ND L1..L4
 * LS LT ITER NITER NAV NHIT BETA PHI OMEGA INTS RANDSERIES PRNG OUTPUTPATH
 * GETWILSON GETRETRACE PL_LEVEL WILSONR WILSONT FMUNU F0MU TURNOFFFMUNU
 * FMUNU1 FMUNU2 FMUNU4 FMUNU5 FMUNU6 FMUNU7 (reference) and PRECISION
 * NHITPAR NOR REUNIT_EVERY REUNIT_FP64 PRNG_INSTANCES ROW_ALIGN INIT
 * STATEFILE SAVESTATE SAVEEVERY STATEOUT ACTIONS_DIFF TUNE PROFILE (this library; the
 * reference sets INIT, the state file name and get_actions_diff in main());
 * PLATFORM DEVICE FINISHPATH TURNOFFWAITING REBUILDBINARY are accepted and
 * ignored.  Unknown generators are an error.                               */
int qg_parse_init_file(const char *path, qg_config *cfg, qg_run_options *opts);
/* lattice_init + lattice_simulate + LatticeCheckCPU + lattice_analysis +
 * lattice_write_results on the current CUDA device.  With opts->init == 0
 * the run continues from opts->state_file: the file's header replaces the
 * lattice, coupling, PRNG and cadence settings of cfg/opts (as
 * lattice_load_bin_header does), the link table and the measured series
 * are restored, the RANLUX stream is replayed to the saved PRNG_counter
 * (suncl.cpp:5349-5354) or the Philox phase counter is set, and the
 * thermalisation and measurement loops resume at NAV_counter and
 * ITER_counter.                                                           */
int qg_run(const qg_config *cfg, const qg_run_options *opts, qg_run_result *res);

/* ----------------------------------------------------------------------- */
/* Lattice state files (.qcg): model::lattice_save_state / lattice_load_state
 * / lattice_make_bin_header / lattice_load_bin_header (suncl.cpp:1857-2079).
 * Layout: a header of 64 uint32 (QCDGPU_STATE_HEADER_WORDS), then
 * lattice_measurement (double2 x header[32]), lattice_energies (double2 x
 * header[33]: S_spat, S_temp sums per iteration), lattice_energies_plq
 * (double2 x header[34]: ReTr spatial, temporal sums) if header[30],
 * lattice_wilson_loop (double x header[33]) if header[31],
 * lattice_polyakov_loop (double2 x header[35]: Re, Im sums) if header[25],
 * then the link table in the reference layout (float4 / double4).  Words
 * 48-59 of the header and a tagged block after the link table (|P|^2,
 * |P|^4 sums) are this library's additions; the reference's loader does not
 * read them.                                                              */
#define QCDGPU_STATE_HEADER_WORDS 64
typedef struct qg_run_state {
    int init;               /* INIT of the run that wrote the file           */
    int nav, nav_counter;   /* NAV, thermalisation sweeps done               */
    int niter, iter, iter_counter; /* NITER, ITER, measured iterations done  */
    int pl_level, get_actions, get_plaquettes, get_wilson;
    uint32_t prng_counter;  /* RANLUX batches produced (PRNG_counter)        */
    uint64_t phase_counter; /* Philox phase counter                          */
    uint64_t sweeps_done;   /* sweeps since the start                        */
    /* measured series as raw lattice sums, `iter` entries each (the first
     * iter_counter used); NULL when absent / not wanted                     */
    double *actions;        /* 2 per iteration: S_spat, S_temp               */
    double *plaquettes;     /* 2 per iteration: ReTr spatial, temporal       */
    double *wilson;         /* 1 per iteration                               */
    double *polyakov;       /* 4 per iteration: Re P, Im P, |P|^2, |P|^4     */
    int fmunu, fmunu_index1, fmunu_index2, get_actions_diff;   /* as qg_run_options */
    double *fmunu_series;   /* 12 per iteration: qg_measure_fmunu's out      */
    /* per iteration: the Polyakov profiles along x, y, z (2 n1 + 2 n2 + 2 n3
     * doubles, qg_measure_polyakov_profile's out) when pl_level > 2, then
     * the action profiles (same length) when get_actions_diff            */
    double *profiles;
} qg_run_state;
/* Host only: write a state file from a reference-layout link table
 * (links_bytes = qg_info.ref_elems * sizeof(Real)).                       */
int qg_write_state_file(const char *path, const qg_config *cfg, const qg_run_state *st, const void *links_ref,
                        uint64_t links_bytes);
/* Host only: read a state file's header into cfg and st (settings and
 * counters; the series pointers are left alone), and, where st's series
 * pointers and links_ref are non-NULL, the series and the link table.
 * Errors: wrong magic/version, truncated file, size mismatch.             */
int qg_read_state_file(const char *path, qg_config *cfg, qg_run_state *st, void *links_ref,
                       uint64_t links_bytes);
/* the context's link table and counters into a state file                 */
int qg_save_state(qg_ctx *ctx, const char *path, const qg_run_state *st);

/* Host only, new: integrated autocorrelation time of x[0..n-1],
 * tau = 1/2 + sum_{t=1..W} rho(t) with the smallest window W >= c tau(W)
 * (Madras & Sokal 1988, automatic windowing; c = 6 is customary).
 * Returns tau in *tau and W in *window; n < 2 or zero variance gives
 * tau = 0.5, W = 0.                                                       */
int qg_tau_int(const double *x, int n, double c, double *tau, int *window);

#ifdef __cplusplus
}
#endif
#endif
