"""qcdgpu_b200 -- B200-native SU(2)/SU(3) lattice Monte Carlo sweep.

Python binding (ctypes) of the C-ABI in include/qcdgpu_b200.h, implemented
by hand-written sm_100a CUDA kernels in qcdgpu_b200/lib/libqg_sun.so.  The
binding mirrors the reference's model interface (vadimdi/QCDGPU,
SU(N)/suncl/suncl.h: lattice_init / lattice_simulate / lattice_analysis);
there is no CPU fallback: if the CUDA library is missing, importing the
runtime raises.
"""
import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libqg_sun.so")

QG_OK = 0
QG_ERR_ARG, QG_ERR_CUDA, QG_ERR_STATE, QG_ERR_NOMEM, QG_ERR_IO, QG_ERR_UNSUPPORTED, QG_ERR_NUMERIC = \
    -1, -2, -3, -4, -5, -6, -7
START_HOT, START_COLD, START_GID, START_HAAR = 0, 1, 2, 3
PRNG_RANLUX, PRNG_PHILOX = 0, 1
LAYOUT_REFERENCE = 0
HEATBATH, OVERRELAX = 0, 1
MEAS_PLAQUETTE, MEAS_ACTION, MEAS_POLYAKOV, MEAS_WILSON = 0, 1, 2, 3
MEAS_PLAQUETTE_F32 = 4             # QG_MEAS_PLAQUETTE_F32
FMUNU_H, FMUNU_E = 0, 1
FMUNU_COLS = 16                     # QG_FMUNU_COLS
MEASURE_SLOTS = 64                  # QG_MEASURE_SLOTS
TUNE_SHAPES = 6                     # QG_TUNE_SHAPES
BATCH_SHAPES = 5                    # QG_BATCH_SHAPES
KERNEL_CLASSES = 6                  # QG_KERNEL_CLASSES
KERNEL_NAMES = ("heatbath phase", "overrelaxation phase", "Gram-Schmidt", "plaquette + action", "Polyakov loop",
                "Wilson loop")
NET_FEATURES, NET_HIDDEN, NET_PARAMS = 8, 32, 1377   # QG_NET_*

EXPORTED_SYMBOLS = (
    "qg_default_config", "qg_create", "qg_destroy", "qg_last_error", "qg_get_info", "qg_sync",
    "qg_prng_seed", "qg_prng_produce", "qg_prns_upload", "qg_prns_download", "qg_init_links",
    "qg_set_prng_lookahead", "qg_set_slab", "qg_slab_halo", "qg_slab_halo_bytes", "qg_slab_halo2",
    "qg_slab_phase", "qg_field_check", "qg_profile_kernels",
    "qg_phase", "qg_sweep", "qg_sweep_phase_times", "qg_reunitarize", "qg_measure", "qg_measure_wilson",
    "qg_links_upload", "qg_links_download", "qg_set_phase_counter", "qg_glibc_seeds", "qg_set_params", "qg_get_stream",
    "qg_default_run_options", "qg_parse_init_file", "qg_run", "qg_tune", "qg_plaquette_noalloc",
    "qg_set_shapes", "qg_get_shapes", "qg_get_config", "qg_set_sweeps_done",
    "qg_write_state_file", "qg_read_state_file", "qg_save_state", "qg_tau_int",
    "qg_batch_create", "qg_batch_destroy", "qg_batch_init", "qg_batch_set_shape", "qg_batch_run", "qg_batch_sync",
    "qg_batch_get_stream", "qg_batch_series", "qg_batch_links_download", "qg_batch_info",
    "qg_batch_set_shapes", "qg_batch_get_shapes", "qg_batch_tune", "qg_batch_set_persistent",
    "qg_batch_set_measure_products",
    "qg_batch_barrier_test",
    "qg_measure_wilson_all", "qg_measure_fmunu", "qg_measure_action_profile", "qg_measure_polyakov_profile",
    "qg_measure_enqueue", "qg_measure_fetch", "qg_measure_plaquette_all", "qg_measure_polyakov_all",
    "qg_net_set", "qg_net_get", "qg_mh_phase", "qg_net_eps", "qg_mh_sweep", "qg_mh_stats", "qg_net_grad",
    "qg_net_train", "qg_write_results", "qg_device_info",
)


class Config(ctypes.Structure):
    _fields_ = [
        ("group", ctypes.c_int),
        ("size", ctypes.c_int * 4),
        ("precision", ctypes.c_int),
        ("start", ctypes.c_int),
        ("beta", ctypes.c_double),
        ("phi", ctypes.c_double),
        ("omega", ctypes.c_double),
        ("nhit", ctypes.c_int),
        ("nhitpar", ctypes.c_int),
        ("prng", ctypes.c_int),
        ("ranlux_nskip", ctypes.c_int),
        ("prng_instances", ctypes.c_int),
        ("randseries", ctypes.c_uint32),
        ("row_align", ctypes.c_int),
        ("n_or", ctypes.c_int),
        ("reunit_every", ctypes.c_int),
        ("reunit_fp64", ctypes.c_int),
        ("wilson_r", ctypes.c_int),
        ("wilson_t", ctypes.c_int),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("sites", ctypes.c_uint32),
        ("rowsize", ctypes.c_uint32),
        ("prngstep", ctypes.c_uint32),
        ("prng_samples", ctypes.c_uint32),
        ("link_bytes", ctypes.c_uint64),
        ("ref_elems", ctypes.c_uint64),
        ("prn_quads", ctypes.c_uint64),
        ("phase_counter", ctypes.c_uint64),
        ("prng_counter", ctypes.c_uint32),
        ("sweeps_done", ctypes.c_uint64),
    ]


(OBS_S_TOTAL, OBS_PLQ_TOTAL, OBS_POLYAKOV, OBS_POLYAKOV_IM, OBS_POLYAKOV_P2, OBS_POLYAKOV_P4, OBS_WILSON,
 OBS_PLQ_SPAT, OBS_PLQ_TEMP, OBS_S_SPAT, OBS_S_TEMP) = range(11)          # QG_OBS_*
OBS_COUNT = 11
OBS_NAMES = ("S_total", "Plq_total", "Polyakov_loop", "Polyakov_loop_im", "Polyakov_loop_P2",
             "Polyakov_loop_P4", "Wilson_loop", "Plq_spat", "Plq_temp", "S_spat", "S_temp")


class RunOptions(ctypes.Structure):
    _fields_ = [
        ("iter", ctypes.c_int),
        ("niter", ctypes.c_int),
        ("nav", ctypes.c_int),
        ("pl_level", ctypes.c_int),
        ("get_wilson", ctypes.c_int),
        ("get_plaquettes", ctypes.c_int),
        ("get_actions", ctypes.c_int),
        ("verify", ctypes.c_int),
        ("write_results", ctypes.c_int),
        ("quiet", ctypes.c_int),
        ("output_path", ctypes.c_char * 512),
        ("prefix", ctypes.c_char * 32),
        ("init", ctypes.c_int),
        ("state_file", ctypes.c_char * 512),
        ("save_state", ctypes.c_int),
        ("save_every_iter", ctypes.c_int),
        ("state_out", ctypes.c_char * 512),
        ("fmunu", ctypes.c_int),
        ("fmunu_index1", ctypes.c_int),
        ("fmunu_index2", ctypes.c_int),
        ("get_actions_diff", ctypes.c_int),
        ("tune_shapes", ctypes.c_int),
        ("profile", ctypes.c_int),
    ]


class RunResult(ctypes.Structure):
    _fields_ = [
        ("mean", ctypes.c_double * 11),
        ("variance", ctypes.c_double * 11),
        ("gpu_last", ctypes.c_double * 11),
        ("cpu_last", ctypes.c_double * 11),
        ("verification_passed", ctypes.c_int),
        ("samples", ctypes.c_int),
        ("seconds", ctypes.c_double),
        ("link_updates_per_second", ctypes.c_double),
        ("results_file", ctypes.c_char * 640),
        ("tau_int", ctypes.c_double * 11),
        ("error", ctypes.c_double * 11),
        ("state_file", ctypes.c_char * 640),
        ("fmunu_mean", ctypes.c_double * FMUNU_COLS),
        ("fmunu_variance", ctypes.c_double * FMUNU_COLS),
        ("fmunu_gpu_last", ctypes.c_double * FMUNU_COLS),
        ("fmunu_cpu_last", ctypes.c_double * FMUNU_COLS),
        ("kernel_ms", ctypes.c_double * KERNEL_CLASSES),
        ("kernel_ms_sigma", ctypes.c_double * KERNEL_CLASSES),
    ]


class Ensemble(ctypes.Structure):
    """qg_ensemble: one lattice of a batch."""
    _fields_ = [("size", ctypes.c_int * 4), ("beta", ctypes.c_double), ("randseries", ctypes.c_uint32)]


class RunState(ctypes.Structure):
    """qg_run_state: counters of a run and its measured series (raw sums)."""
    _fields_ = [
        ("init", ctypes.c_int),
        ("nav", ctypes.c_int),
        ("nav_counter", ctypes.c_int),
        ("niter", ctypes.c_int),
        ("iter", ctypes.c_int),
        ("iter_counter", ctypes.c_int),
        ("pl_level", ctypes.c_int),
        ("get_actions", ctypes.c_int),
        ("get_plaquettes", ctypes.c_int),
        ("get_wilson", ctypes.c_int),
        ("prng_counter", ctypes.c_uint32),
        ("phase_counter", ctypes.c_uint64),
        ("sweeps_done", ctypes.c_uint64),
        ("actions", ctypes.POINTER(ctypes.c_double)),
        ("plaquettes", ctypes.POINTER(ctypes.c_double)),
        ("wilson", ctypes.POINTER(ctypes.c_double)),
        ("polyakov", ctypes.POINTER(ctypes.c_double)),
        ("fmunu", ctypes.c_int),
        ("fmunu_index1", ctypes.c_int),
        ("fmunu_index2", ctypes.c_int),
        ("get_actions_diff", ctypes.c_int),
        ("fmunu_series", ctypes.POINTER(ctypes.c_double)),
        ("profiles", ctypes.POINTER(ctypes.c_double)),
    ]


_lib = None


class QGError(RuntimeError):
    pass


def load_library(path=LIB_PATH):
    """Load libqg_sun.so and declare the C-ABI; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise QGError("CUDA library %s is not built (run __graft_entry__.build() or "
                      "python qcdgpu_b200/build.py)" % path)
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    lib.qg_default_config.argtypes = [P(Config)]
    lib.qg_create.argtypes = [P(Config), P(vp)]
    lib.qg_destroy.argtypes = [vp]
    lib.qg_last_error.argtypes = [vp]
    lib.qg_last_error.restype = ctypes.c_char_p
    lib.qg_get_info.argtypes = [vp, P(Info)]
    lib.qg_sync.argtypes = [vp]
    lib.qg_prng_seed.argtypes = [vp, ctypes.c_uint32]
    lib.qg_prng_produce.argtypes = [vp]
    lib.qg_set_prng_lookahead.argtypes = [vp, ctypes.c_int]
    lib.qg_set_slab.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.qg_slab_halo.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
    lib.qg_slab_halo_bytes.argtypes = [vp, P(ctypes.c_uint64)]
    lib.qg_slab_halo2.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int]
    lib.qg_slab_phase.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.qg_field_check.argtypes = [vp, ctypes.c_double, P(ctypes.c_uint64)]
    lib.qg_profile_kernels.argtypes = [vp, ctypes.c_int, P(ctypes.c_double), P(ctypes.c_double)]
    lib.qg_prns_upload.argtypes = [vp, vp, ctypes.c_uint64]
    lib.qg_prns_download.argtypes = [vp, vp, ctypes.c_uint64]
    lib.qg_init_links.argtypes = [vp, ctypes.c_int]
    lib.qg_phase.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.qg_sweep.argtypes = [vp, ctypes.c_int]
    lib.qg_sweep_phase_times.argtypes = [vp, ctypes.c_int, P(ctypes.c_double), P(ctypes.c_double),
                                         P(ctypes.c_double)]
    lib.qg_reunitarize.argtypes = [vp, ctypes.c_int]
    lib.qg_measure.argtypes = [vp, ctypes.c_int, P(ctypes.c_double)]
    lib.qg_measure_wilson.argtypes = [vp, ctypes.c_int, ctypes.c_int, P(ctypes.c_double)]
    lib.qg_measure_wilson_all.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, P(ctypes.c_double)]
    lib.qg_measure_fmunu.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, P(ctypes.c_double)]
    lib.qg_measure_enqueue.argtypes = [vp, ctypes.c_int, P(ctypes.c_uint64)]
    lib.qg_measure_plaquette_all.argtypes = [vp, P(ctypes.c_double)]
    lib.qg_measure_polyakov_all.argtypes = [vp, P(ctypes.c_double)]
    lib.qg_measure_fetch.argtypes = [vp, ctypes.c_uint64, P(ctypes.c_double)]
    lib.qg_measure_action_profile.argtypes = [vp, ctypes.c_int, P(ctypes.c_double)]
    lib.qg_measure_polyakov_profile.argtypes = [vp, ctypes.c_int, P(ctypes.c_double)]
    lib.qg_links_upload.argtypes = [vp, vp, ctypes.c_int]
    lib.qg_links_download.argtypes = [vp, vp, ctypes.c_int]
    lib.qg_set_phase_counter.argtypes = [vp, ctypes.c_uint64]
    lib.qg_glibc_seeds.argtypes = [ctypes.c_uint32, ctypes.c_int, P(ctypes.c_uint32)]
    lib.qg_set_params.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.qg_get_stream.argtypes = [vp, P(vp)]
    lib.qg_tune.argtypes = [vp, ctypes.c_int, P(ctypes.c_float)]
    lib.qg_set_shapes.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.qg_get_shapes.argtypes = [vp, P(ctypes.c_int), P(ctypes.c_int)]
    lib.qg_plaquette_noalloc.argtypes = [vp, ctypes.c_int, ctypes.c_int, P(ctypes.c_int), ctypes.c_uint32,
                                         ctypes.c_double, vp, vp]
    lib.qg_get_config.argtypes = [vp, P(Config)]
    lib.qg_set_sweeps_done.argtypes = [vp, ctypes.c_uint64]
    lib.qg_write_state_file.argtypes = [ctypes.c_char_p, P(Config), P(RunState), vp, ctypes.c_uint64]
    lib.qg_read_state_file.argtypes = [ctypes.c_char_p, P(Config), P(RunState), vp, ctypes.c_uint64]
    lib.qg_save_state.argtypes = [vp, ctypes.c_char_p, P(RunState)]
    lib.qg_tau_int.argtypes = [P(ctypes.c_double), ctypes.c_int, ctypes.c_double, P(ctypes.c_double),
                               P(ctypes.c_int)]
    fp = P(ctypes.c_float)
    lib.qg_net_set.argtypes = [vp, fp, ctypes.c_double]
    lib.qg_net_get.argtypes = [vp, fp, fp]
    lib.qg_mh_phase.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.qg_net_eps.argtypes = [vp, ctypes.c_int, ctypes.c_int, fp]
    lib.qg_mh_sweep.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.qg_mh_stats.argtypes = [vp, P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_uint64), ctypes.c_int]
    lib.qg_net_grad.argtypes = [vp, ctypes.c_int, ctypes.c_int, fp, P(ctypes.c_double)]
    lib.qg_net_train.argtypes = [vp, ctypes.c_int, ctypes.c_double, P(ctypes.c_double)]
    lib.qg_batch_create.argtypes = [P(Config), P(Ensemble), ctypes.c_int, ctypes.c_int, P(vp)]
    lib.qg_batch_destroy.argtypes = [vp]
    lib.qg_batch_init.argtypes = [vp, ctypes.c_int]
    lib.qg_batch_set_shape.argtypes = [vp, ctypes.c_int]
    lib.qg_batch_set_shapes.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.qg_batch_get_shapes.argtypes = [vp, P(ctypes.c_int), P(ctypes.c_int)]
    lib.qg_write_results.argtypes = [P(Config), P(RunOptions), P(RunResult), ctypes.c_int, P(ctypes.c_double),
                                     P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double), ctypes.c_int64,
                                     ctypes.c_int64, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                     ctypes.c_size_t]
    lib.qg_device_info.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t]
    lib.qg_batch_tune.argtypes = [vp, ctypes.c_int, P(ctypes.c_float)]
    lib.qg_batch_set_persistent.argtypes = [vp, ctypes.c_int]
    lib.qg_batch_set_measure_products.argtypes = [vp, ctypes.c_int]
    lib.qg_batch_barrier_test.argtypes = [vp, ctypes.c_int]
    lib.qg_batch_run.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.qg_batch_sync.argtypes = [vp]
    lib.qg_batch_get_stream.argtypes = [vp, P(vp)]
    lib.qg_batch_series.argtypes = [vp, P(ctypes.c_double), ctypes.c_uint64, P(ctypes.c_uint64)]
    lib.qg_batch_links_download.argtypes = [vp, ctypes.c_int, vp]
    lib.qg_batch_info.argtypes = [vp, P(ctypes.c_uint64), P(ctypes.c_uint64), P(ctypes.c_uint64)]
    lib.qg_default_run_options.argtypes = [P(RunOptions)]
    lib.qg_parse_init_file.argtypes = [ctypes.c_char_p, P(Config), P(RunOptions)]
    lib.qg_run.argtypes = [P(Config), P(RunOptions), P(RunResult)]
    _lib = lib
    return lib


def glibc_seeds(randseries, n):
    """RANLUX instance seeds for RANDSERIES (host only, no GPU needed)."""
    lib = load_library()
    out = np.zeros(n, dtype=np.uint32)
    rc = lib.qg_glibc_seeds(randseries, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    if rc != QG_OK:
        raise QGError("qg_glibc_seeds failed")
    return out


def bf16_round(a):
    """Round float32 values to the nearest BF16 (ties to even), as floats --
    the weights the learned-proposal kernels compute with."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32)


def net_init(seed=0, out_bias=0.0):
    """He-normal initial weights of the step-size network (QG_NET_PARAMS
    floats: W1[32][8], b1[32], W2[32][32], b2[32], w3[32], b3)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NET_PARAMS, dtype=np.float32)
    nf, nh = NET_FEATURES, NET_HIDDEN
    o = 0
    p[o:o + nh * nf] = rng.standard_normal(nh * nf) * np.sqrt(2.0 / nf); o += nh * nf
    o += nh
    p[o:o + nh * nh] = rng.standard_normal(nh * nh) * np.sqrt(2.0 / nh); o += nh * nh
    o += nh
    p[o:o + nh] = rng.standard_normal(nh) * np.sqrt(1.0 / nh) * 0.1; o += nh
    p[o] = out_bias
    return p


def net_constant(eps, eps_max):
    """Weights that give the constant step eps (the proposal without a
    network): everything zero except the output bias logit(eps/eps_max)."""
    p = np.zeros(NET_PARAMS, dtype=np.float32)
    r = eps / eps_max
    p[-1] = np.log(r / (1.0 - r))
    return p


def tau_int(x, c=6.0):
    """qg_tau_int: integrated autocorrelation time of a series (Madras-Sokal
    automatic window, W >= c tau); returns (tau, W).  Host only."""
    lib = load_library()
    a = np.ascontiguousarray(x, dtype=np.float64)
    t = ctypes.c_double()
    w = ctypes.c_int()
    rc = lib.qg_tau_int(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(a), c, ctypes.byref(t),
                        ctypes.byref(w))
    if rc != QG_OK:
        raise QGError("qg_tau_int: " + lib.qg_last_error(None).decode())
    return t.value, w.value


def profile_row(cfg, st):
    """doubles per iteration of a run state's profile series: Polyakov
    profiles along x, y, z when pl_level > 2, then the action profiles when
    get_actions_diff"""
    plen = 2 * (cfg.size[0] + cfg.size[1] + cfg.size[2])
    return (plen if st.pl_level > 2 else 0) + (plen if st.get_actions_diff else 0)


def read_state_file(path, cfg=None):
    """qg_read_state_file: (config, state, series dict, link table) of a .qcg
    file; the table is the reference layout (float32 / float64).  Host only."""
    lib = load_library()
    cfg = cfg if cfg is not None else default_config()
    st = RunState()
    rc = lib.qg_read_state_file(path.encode(), ctypes.byref(cfg), ctypes.byref(st), None, 0)
    if rc != QG_OK:
        raise QGError("qg_read_state_file: " + lib.qg_last_error(None).decode())
    n = max(st.iter, 1)
    ser = {"actions": np.zeros(2 * n), "plaquettes": np.zeros(2 * n), "wilson": np.zeros(n),
           "polyakov": np.zeros(4 * n), "fmunu_series": np.zeros(12 * n),
           "profiles": np.zeros(profile_row(cfg, st) * n + 1)}
    dp = ctypes.POINTER(ctypes.c_double)
    for k, v in ser.items():
        setattr(st, k, v.ctypes.data_as(dp))
    V = cfg.size[0] * cfg.size[1] * cfg.size[2] * cfg.size[3]
    a = cfg.row_align if cfg.row_align > 0 else 64
    rowsize = (V + a - 1) // a * a
    elems = (12 if cfg.group == 3 else 4) * rowsize * 4
    table = np.zeros(elems, dtype=np.float64 if cfg.precision else np.float32)
    rc = lib.qg_read_state_file(path.encode(), ctypes.byref(cfg), ctypes.byref(st),
                                table.ctypes.data_as(ctypes.c_void_p), table.nbytes)
    if rc != QG_OK:
        raise QGError("qg_read_state_file: " + lib.qg_last_error(None).decode())
    for k in ser:
        setattr(st, k, None)
    return cfg, st, ser, table


def write_state_file(path, cfg, st, table, series=None):
    """qg_write_state_file from host arrays (series: dict as read_state_file
    returns; missing entries are written as zeros).  Host only."""
    lib = load_library()
    n = max(st.iter, 1)
    series = dict(series or {})
    keep = {}
    dp = ctypes.POINTER(ctypes.c_double)
    for k, m in (("actions", 2), ("plaquettes", 2), ("wilson", 1), ("polyakov", 4), ("fmunu_series", 12),
                 ("profiles", profile_row(cfg, st))):
        v = np.ascontiguousarray(series.get(k, np.zeros(m * n + 1)), dtype=np.float64)
        keep[k] = v
        setattr(st, k, v.ctypes.data_as(dp))
    t = np.ascontiguousarray(table)
    rc = lib.qg_write_state_file(path.encode(), ctypes.byref(cfg), ctypes.byref(st),
                                 t.ctypes.data_as(ctypes.c_void_p), t.nbytes)
    for k in keep:
        setattr(st, k, None)
    if rc != QG_OK:
        raise QGError("qg_write_state_file: " + lib.qg_last_error(None).decode())


def default_config(**kw):
    """qg_default_config (the reference main()'s defaults) overridden by kw;
    `size` may be an int (L^4) or a 4-tuple (L1..L4)."""
    lib = load_library()
    c = Config()
    lib.qg_default_config(ctypes.byref(c))
    for k, v in kw.items():
        if k == "size":
            v = (v,) * 4 if isinstance(v, int) else tuple(v)
            for i in range(4):
                c.size[i] = int(v[i])
        else:
            if not hasattr(c, k):
                raise KeyError(k)
            setattr(c, k, v)
    return c


def default_run_options(**kw):
    """qg_default_run_options (the reference main()'s run cadence) + kw."""
    lib = load_library()
    o = RunOptions()
    lib.qg_default_run_options(ctypes.byref(o))
    for k, v in kw.items():
        if k in ("output_path", "prefix", "state_file", "state_out"):
            v = v.encode()
        setattr(o, k, v)
    return o


def parse_init_file(path, cfg=None, opts=None):
    """Apply an init.dat onto (cfg, opts) -- host only, no GPU needed."""
    lib = load_library()
    cfg = default_config() if cfg is None else cfg
    opts = default_run_options() if opts is None else opts
    rc = lib.qg_parse_init_file(path.encode(), ctypes.byref(cfg), ctypes.byref(opts))
    if rc != QG_OK:
        raise QGError("qg_parse_init_file: %s" % lib.qg_last_error(None).decode())
    return cfg, opts


def write_results(cfg, opts, res, series, fmunu=None, profiles=None, fmunu_cpu_lattice_variance=None,
                  t_start=0, t_end=0, resumed=False, platform="", device=""):
    """qg_write_results: the reference-layout results file of a finished run
    (series [QG_OBS_COUNT][iter]); returns the file's path"""
    lib = load_library()
    dp = ctypes.POINTER(ctypes.c_double)

    def arr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        return a, a.ctypes.data_as(dp)
    keep = [arr(series), arr(fmunu), arr(profiles), arr(fmunu_cpu_lattice_variance)]
    ptrs = [k[1] if k is not None else None for k in keep]
    out = ctypes.create_string_buffer(1024)
    rc = lib.qg_write_results(ctypes.byref(cfg), ctypes.byref(opts), ctypes.byref(res), int(resumed), ptrs[0],
                              ptrs[1], ptrs[2], ptrs[3], int(t_start), int(t_end), platform.encode(),
                              device.encode(), out, len(out))
    if rc != QG_OK:
        raise QGError("qg_write_results: %s" % lib.qg_last_error(None).decode())
    return out.value.decode()


def run(cfg, opts):
    """One run as the reference's main() does it: start, measurements every
    NITER sweeps, statistics, CPU re-check, results file.  Returns RunResult."""
    lib = load_library()
    res = RunResult()
    rc = lib.qg_run(ctypes.byref(cfg), ctypes.byref(opts), ctypes.byref(res))
    if rc != QG_OK:
        raise QGError("qg_run: %s" % lib.qg_last_error(None).decode())
    return res


class Lattice:
    """One lattice on one GPU (a qg_ctx).  Mirrors model_CL::model."""

    def __init__(self, cfg=None, **kw):
        self.lib = load_library()
        self.cfg = cfg if cfg is not None else default_config(**kw)
        self.ctx = ctypes.c_void_p()
        rc = self.lib.qg_create(ctypes.byref(self.cfg), ctypes.byref(self.ctx))
        if rc != QG_OK:
            raise QGError("qg_create: %s" % self.lib.qg_last_error(None).decode())

    def _ck(self, rc, what):
        if rc != QG_OK:
            raise QGError("%s: %s" % (what, self.lib.qg_last_error(self.ctx).decode()))

    def close(self):
        if self.ctx:
            self.lib.qg_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- setup
    def info(self):
        i = Info()
        self._ck(self.lib.qg_get_info(self.ctx, ctypes.byref(i)), "qg_get_info")
        return i

    def seed(self, randseries=None):
        self._ck(self.lib.qg_prng_seed(self.ctx, self.cfg.randseries if randseries is None else randseries),
                 "qg_prng_seed")

    def produce(self):
        self._ck(self.lib.qg_prng_produce(self.ctx), "qg_prng_produce")

    def set_slab(self, x0, n1_global):
        """Make this lattice (size[0] = w + 2) the x-slab [x0, x0 + w) of a
        lattice of n1_global x-slices, with halo slices 0 and w + 1."""
        self._ck(self.lib.qg_set_slab(self.ctx, int(x0), int(n1_global)), "qg_set_slab")

    def slab_halo_bytes(self):
        n = ctypes.c_uint64()
        self._ck(self.lib.qg_slab_halo_bytes(self.ctx, ctypes.byref(n)), "qg_slab_halo_bytes")
        return n.value

    def slab_halo(self, direction, parity, side, ptr, to_buf):
        """Pack the boundary slice (to_buf) or unpack into the halo slice;
        ptr is a device (or pinned host) address of slab_halo_bytes() bytes."""
        self._ck(self.lib.qg_slab_halo(self.ctx, int(direction), int(parity), int(side), ctypes.c_void_p(ptr),
                                       int(bool(to_buf))), "qg_slab_halo")

    def slab_halo2(self, direction, parity, ptr_lo, ptr_hi, to_buf):
        """Both sides of slab_halo in one kernel launch (device buffers)."""
        self._ck(self.lib.qg_slab_halo2(self.ctx, int(direction), int(parity), ctypes.c_void_p(ptr_lo),
                                        ctypes.c_void_p(ptr_hi), int(bool(to_buf))), "qg_slab_halo2")

    def profile_kernels(self, reps=20):
        """{kernel class: (mean ms, sigma ms) per launch} on the live field
        (restored afterwards)"""
        m, sd = (ctypes.c_double * KERNEL_CLASSES)(), (ctypes.c_double * KERNEL_CLASSES)()
        self._ck(self.lib.qg_profile_kernels(self.ctx, int(reps), m, sd), "qg_profile_kernels")
        return {KERNEL_NAMES[k]: (m[k], sd[k]) for k in range(KERNEL_CLASSES)}

    def field_check(self, tol=None):
        """number of links not finite or off SU(N) by more than tol (default
        1e-3 for FP32 links, 1e-9 for FP64)"""
        if tol is None:
            tol = 1e-9 if self.cfg.precision else 1e-3
        n = ctypes.c_uint64()
        self._ck(self.lib.qg_field_check(self.ctx, float(tol), ctypes.byref(n)), "qg_field_check")
        return n.value

    def slab_phase(self, parity, direction, kind, part):
        """qg_slab_phase: part 0 the boundary slices, part 1 the interior."""
        self._ck(self.lib.qg_slab_phase(self.ctx, int(parity), int(direction), int(kind), int(part)),
                 "qg_slab_phase")

    def set_prng_lookahead(self, on):
        """RANLUX mode: generate the next sweep's batches alongside the current
        sweep (default on); the stream and its use are the same either way."""
        self._ck(self.lib.qg_set_prng_lookahead(self.ctx, int(bool(on))), "qg_set_prng_lookahead")

    def init(self, start=None):
        self._ck(self.lib.qg_init_links(self.ctx, self.cfg.start if start is None else start), "qg_init_links")

    # ---- updates
    def phase(self, parity, direction, kind=HEATBATH):
        self._ck(self.lib.qg_phase(self.ctx, parity, direction, kind), "qg_phase")

    def sweep(self, n=1):
        self._ck(self.lib.qg_sweep(self.ctx, n), "qg_sweep")

    def sweep_phase_times(self, n=20):
        """qg_sweep_phase_times: n sweeps of the qg_sweep chain, returning the
        mean (heatbath phase, overrelaxation phase, whole sweep) durations
        in ms inside the sweep graph"""
        hb, orx, sw = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._ck(self.lib.qg_sweep_phase_times(self.ctx, n, ctypes.byref(hb), ctypes.byref(orx), ctypes.byref(sw)),
                 "qg_sweep_phase_times")
        return hb.value, orx.value, sw.value

    def reunitarize(self, fp64=False):
        self._ck(self.lib.qg_reunitarize(self.ctx, 1 if fp64 else 0), "qg_reunitarize")

    def tune(self, reps=4):
        """Pick the fastest phase-kernel launch shapes on this lattice; returns
        the measured ms per launch as [(heatbath, overrelaxation)] per shape."""
        t = (ctypes.c_float * (2 * TUNE_SHAPES))()
        self._ck(self.lib.qg_tune(self.ctx, reps, t), "qg_tune")
        return [(t[2 * v], t[2 * v + 1]) for v in range(TUNE_SHAPES)]

    def set_shapes(self, heatbath, overrelax):
        """Pin the phase-kernel launch shapes (0 .. TUNE_SHAPES-1)."""
        self._ck(self.lib.qg_set_shapes(self.ctx, heatbath, overrelax), "qg_set_shapes")

    def shapes(self):
        h, o = ctypes.c_int(), ctypes.c_int()
        self._ck(self.lib.qg_get_shapes(self.ctx, ctypes.byref(h), ctypes.byref(o)), "qg_get_shapes")
        return h.value, o.value

    # ---- learned proposal (SU(3), FP32 links, Philox)
    def net_set(self, params, eps_max):
        a = np.ascontiguousarray(params, dtype=np.float32)
        assert a.size == NET_PARAMS
        self._ck(self.lib.qg_net_set(self.ctx, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), eps_max),
                 "qg_net_set")
        self.eps_max = eps_max

    def net_get(self):
        """(FP32 master weights, the BF16 weights as floats)"""
        m = np.zeros(NET_PARAMS, dtype=np.float32)
        b = np.zeros(NET_PARAMS, dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self._ck(self.lib.qg_net_get(self.ctx, m.ctypes.data_as(fp), b.ctypes.data_as(fp)), "qg_net_get")
        return m, b

    def mh_phase(self, parity, direction, nhit=1):
        self._ck(self.lib.qg_mh_phase(self.ctx, parity, direction, nhit), "qg_mh_phase")

    def net_eps(self, parity, direction):
        """the step eps of every link of phase (parity, direction) that the
        next mh_phase uses (the field is not changed)"""
        e = np.zeros(self.info().sites // 2, dtype=np.float32)
        self._ck(self.lib.qg_net_eps(self.ctx, parity, direction, e.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                 "qg_net_eps")
        return e

    def mh_sweep(self, n=1, nhit=1):
        self._ck(self.lib.qg_mh_sweep(self.ctx, n, nhit), "qg_mh_sweep")

    def mh_stats(self, reset=False):
        """(acceptance rate, mean squared jump angle per proposal, proposals)"""
        a, j, h = ctypes.c_double(), ctypes.c_double(), ctypes.c_uint64()
        self._ck(self.lib.qg_mh_stats(self.ctx, ctypes.byref(a), ctypes.byref(j), ctypes.byref(h), int(reset)),
                 "qg_mh_stats")
        return a.value, j.value, h.value

    def net_grad(self, parity, direction):
        """(gradient, stats = [loss, ESJD, acceptance, links])"""
        g = np.zeros(NET_PARAMS, dtype=np.float32)
        st = (ctypes.c_double * 4)()
        self._ck(self.lib.qg_net_grad(self.ctx, parity, direction, g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                      st), "qg_net_grad")
        return g, list(st)

    def net_train(self, steps, lr):
        st = (ctypes.c_double * 4)()
        self._ck(self.lib.qg_net_train(self.ctx, steps, lr, st), "qg_net_train")
        return list(st)

    def sync(self):
        self._ck(self.lib.qg_sync(self.ctx), "qg_sync")

    def set_params(self, beta, phi=0.0, omega=0.0):
        self._ck(self.lib.qg_set_params(self.ctx, beta, phi, omega), "qg_set_params")
        self.cfg.beta, self.cfg.phi, self.cfg.omega = beta, phi, omega

    def stream(self):
        s = ctypes.c_void_p()
        self._ck(self.lib.qg_get_stream(self.ctx, ctypes.byref(s)), "qg_get_stream")
        return s.value

    def set_phase_counter(self, v):
        self._ck(self.lib.qg_set_phase_counter(self.ctx, v), "qg_set_phase_counter")

    # ---- measurements (raw lattice sums, see include/qcdgpu_b200.h)
    def _measure(self, what, n):
        out = (ctypes.c_double * 4)()
        self._ck(self.lib.qg_measure(self.ctx, what, out), "qg_measure")
        return tuple(out[:n])

    def plaquette_sums(self):
        return self._measure(MEAS_PLAQUETTE, 2)

    def plaquette_sums_f32(self):
        """plaquette_sums with each plaquette's products and trace in FP32
        (FP32 links; on FP64 links the same values as plaquette_sums)"""
        return self._measure(MEAS_PLAQUETTE_F32, 2)

    def action_sums(self):
        return self._measure(MEAS_ACTION, 2)

    def polyakov_sums(self):
        return self._measure(MEAS_POLYAKOV, 4)

    def wilson_all(self, Rmax, Tmax, fp64_products=True):
        """raw sums of all R x T Wilson loops, array [Rmax][Tmax]"""
        out = np.zeros(Rmax * Tmax)
        self._ck(self.lib.qg_measure_wilson_all(self.ctx, Rmax, Tmax, int(bool(fp64_products)),
                                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                 "qg_measure_wilson_all")
        return out.reshape(Rmax, Tmax)

    def measure_enqueue(self, what):
        """qg_measure_enqueue: the measurement's kernels and result copy on
        the stream, without waiting; returns the ticket for measure_fetch"""
        t = ctypes.c_uint64()
        self._ck(self.lib.qg_measure_enqueue(self.ctx, what, ctypes.byref(t)), "qg_measure_enqueue")
        return t.value

    def measure_fetch(self, ticket):
        """qg_measure_fetch: the values of an enqueued measurement (waits for them)"""
        out = (ctypes.c_double * 4)()
        self._ck(self.lib.qg_measure_fetch(self.ctx, ticket, out), "qg_measure_fetch")
        return tuple(out)

    def measure_all(self, polyakov=False):
        """qg_measure_plaquette_all / qg_measure_polyakov_all: (four totals,
        [profile x, profile y, profile z] each an array [slice][2])"""
        n = list(self.cfg.size)
        out = np.zeros(4 + 2 * (n[0] + n[1] + n[2]))
        fn = self.lib.qg_measure_polyakov_all if polyakov else self.lib.qg_measure_plaquette_all
        self._ck(fn(self.ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "qg_measure_*_all")
        prof, o = [], 4
        for a in range(3):
            prof.append(out[o:o + 2 * n[a]].reshape(-1, 2))
            o += 2 * n[a]
        return tuple(out[:4]), prof

    def fmunu(self, field=0, index1=None, index2=None):
        """raw F_munu sums (qg_measure_fmunu): array [2 generators][3 planes]
        [Re, Im]; field FMUNU_H (xy, xz, yz) or FMUNU_E (xt, yt, zt);
        generators default to the reference's (3, 8) for SU(3), (3, 2) for
        SU(2)"""
        i1 = 3 if index1 is None else index1
        i2 = (8 if self.cfg.group == 3 else 2) if index2 is None else index2
        out = np.zeros(12)
        self._ck(self.lib.qg_measure_fmunu(self.ctx, field, i1, i2, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                 "qg_measure_fmunu")
        return out.reshape(2, 3, 2)

    def action_profile(self, axis):
        """raw per-slice (spatial, temporal) action sums along axis 0..2"""
        out = np.zeros(2 * self.cfg.size[axis])
        self._ck(self.lib.qg_measure_action_profile(self.ctx, axis, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                 "qg_measure_action_profile")
        return out.reshape(-1, 2)

    def polyakov_profile(self, axis):
        """raw per-slice (Re, Im) Polyakov trace sums along axis 0..2"""
        out = np.zeros(2 * self.cfg.size[axis])
        self._ck(self.lib.qg_measure_polyakov_profile(self.ctx, axis,
                                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                 "qg_measure_polyakov_profile")
        return out.reshape(-1, 2)

    def wilson_sum(self, R=None, T=None):
        out = (ctypes.c_double * 1)()
        R = self.cfg.wilson_r if R is None else R
        T = self.cfg.wilson_t if T is None else T
        self._ck(self.lib.qg_measure_wilson(self.ctx, R, T, out), "qg_measure_wilson")
        return out[0]

    def plaquette(self):
        """(Plq_spat, Plq_temp, Plq_total) normalised as lattice_analysis
        does (SU(N)/suncl/suncl.cpp:1357-1373): sum / (3V), range [-N, N]."""
        s, t = self.plaquette_sums()
        V = self.info().sites
        return s / (3 * V), t / (3 * V), (s + t) / (6 * V)

    def polyakov(self):
        """(Re P, Im P, P2, P4) normalised as suncl.cpp:1483-1494,1591-1605."""
        re, im, p2, p4 = self.polyakov_sums()
        n = self.cfg.size[0] * self.cfg.size[1] * self.cfg.size[2]
        N = self.cfg.group
        return re / (n * N), im / (n * N), p2 / (n * N * N), p4 / (n * N ** 4)

    # ---- link table I/O in the reference layout
    def _ref_dtype(self):
        return np.float64 if self.cfg.precision else np.float32

    def download(self):
        a = np.zeros(self.info().ref_elems, dtype=self._ref_dtype())
        self._ck(self.lib.qg_links_download(self.ctx, a.ctypes.data, LAYOUT_REFERENCE), "qg_links_download")
        return a

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=self._ref_dtype())
        if a.size != self.info().ref_elems:
            raise ValueError("link table has %d elements, expected %d" % (a.size, self.info().ref_elems))
        self._ck(self.lib.qg_links_upload(self.ctx, a.ctypes.data, LAYOUT_REFERENCE), "qg_links_upload")

    def prns_download(self, nquads=None):
        n = self.info().prn_quads if nquads is None else nquads
        a = np.zeros(n * 4, dtype=np.float32)
        self._ck(self.lib.qg_prns_download(self.ctx, a.ctypes.data, n), "qg_prns_download")
        return a

    def prns_upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        self._ck(self.lib.qg_prns_upload(self.ctx, a.ctypes.data, a.size // 4), "qg_prns_upload")


class Batch:
    """Many independent lattices updated together (qg_batch): one launch per
    phase over all ensembles, sweep + measurement in one CUDA graph.
    `ensembles` is a list of (size 4-tuple, beta, randseries)."""

    def __init__(self, common, ensembles, max_measurements=0):
        self.lib = load_library()
        self.cfg = common
        self.n = len(ensembles)
        arr = (Ensemble * self.n)()
        for k, (size, beta, series) in enumerate(ensembles):
            for i in range(4):
                arr[k].size[i] = int(size[i])
            arr[k].beta = float(beta)
            arr[k].randseries = int(series)
        self.ens = [(tuple(s), b, r) for s, b, r in ensembles]
        self.b = ctypes.c_void_p()
        rc = self.lib.qg_batch_create(ctypes.byref(common), arr, self.n, int(max_measurements), ctypes.byref(self.b))
        if rc != QG_OK:
            raise QGError("qg_batch_create: %s" % self.lib.qg_last_error(None).decode())

    def _ck(self, rc, what):
        if rc != QG_OK:
            raise QGError("%s: %s" % (what, self.lib.qg_last_error(None).decode()))

    def close(self):
        if self.b:
            self.lib.qg_batch_destroy(self.b)
            self.b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self, start=START_COLD):
        self._ck(self.lib.qg_batch_init(self.b, start), "qg_batch_init")

    def set_shape(self, shape):
        self._ck(self.lib.qg_batch_set_shape(self.b, shape), "qg_batch_set_shape")

    def set_shapes(self, heatbath, overrelax):
        """Pin the batched phase-launch shapes (0 .. BATCH_SHAPES-1) per kind."""
        self._ck(self.lib.qg_batch_set_shapes(self.b, heatbath, overrelax), "qg_batch_set_shapes")

    def shapes(self):
        h, o = ctypes.c_int(), ctypes.c_int()
        self._ck(self.lib.qg_batch_get_shapes(self.b, ctypes.byref(h), ctypes.byref(o)), "qg_batch_get_shapes")
        return h.value, o.value

    def tune(self, reps=4):
        """Pick the fastest batched launch shapes on the live fields (restored);
        returns the measured ms per launch as [(heatbath, overrelaxation)] per shape."""
        t = (ctypes.c_float * (2 * BATCH_SHAPES))()
        self._ck(self.lib.qg_batch_tune(self.b, reps, t), "qg_batch_tune")
        return [(t[2 * v], t[2 * v + 1]) for v in range(BATCH_SHAPES)]

    def set_persistent(self, enable=True):
        """one persistent launch per half-sweep (grid barriers between the
        directions) instead of one launch per phase"""
        self._ck(self.lib.qg_batch_set_persistent(self.b, int(enable)), "qg_batch_set_persistent")

    def set_measure_products(self, fp32=True):
        """plaquette and action series with FP32 products and traces (FP32
        links) instead of the reference's FP64 products"""
        self._ck(self.lib.qg_batch_set_measure_products(self.b, int(fp32)), "qg_batch_set_measure_products")

    def barrier_test(self, skip_block):
        """run one persistent half-sweep in which block skip_block skips its
        first barrier arrival; returns the status code (QG_ERR_CUDA expected)
        and the error text"""
        rc = self.lib.qg_batch_barrier_test(self.b, skip_block)
        return rc, self.lib.qg_last_error(None).decode()

    def run(self, nsweeps, measure_every=0):
        self._ck(self.lib.qg_batch_run(self.b, nsweeps, measure_every), "qg_batch_run")

    def sync(self):
        self._ck(self.lib.qg_batch_sync(self.b), "qg_batch_sync")

    def stream(self):
        s = ctypes.c_void_p()
        self._ck(self.lib.qg_batch_get_stream(self.b, ctypes.byref(s)), "qg_batch_get_stream")
        return s.value

    def series(self):
        """[measurement][ensemble][8] raw sums (plaquette s/t, action s/t,
        Re P, Im P, |P|^2, |P|^4)."""
        n = ctypes.c_uint64()
        self._ck(self.lib.qg_batch_series(self.b, None, 0, ctypes.byref(n)), "qg_batch_series")
        out = np.zeros((n.value, self.n, 8))
        if n.value:
            self._ck(self.lib.qg_batch_series(self.b, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n.value,
                                              ctypes.byref(n)), "qg_batch_series")
        return out

    def download(self, e):
        size = self.ens[e][0]
        V = int(np.prod(size))
        a = self.cfg.row_align if self.cfg.row_align > 0 else 64
        rowsize = (V + a - 1) // a * a
        elems = (12 if self.cfg.group == 3 else 4) * rowsize * 4
        out = np.zeros(elems, dtype=np.float64 if self.cfg.precision else np.float32)
        self._ck(self.lib.qg_batch_links_download(self.b, e, out.ctypes.data_as(ctypes.c_void_p)),
                 "qg_batch_links_download")
        return out

    def info(self):
        v, s, f = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._ck(self.lib.qg_batch_info(self.b, ctypes.byref(v), ctypes.byref(s), ctypes.byref(f)), "qg_batch_info")
        return {"sites": v.value, "sweeps": s.value, "field_bytes": f.value}
