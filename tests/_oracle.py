"""ctypes binding of the CPU oracle (oracle/qg_oracle.c) for the tests.

Test infrastructure only: the oracle is the checker the CUDA path is compared
against, never part of the product.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")


class Cfg(ctypes.Structure):
    _fields_ = [
        ("group", ctypes.c_int),
        ("n", ctypes.c_int * 4),
        ("precision", ctypes.c_int),
        ("rowsize", ctypes.c_int),
        ("prngstep", ctypes.c_int),
        ("nhit", ctypes.c_int),
        ("nhitpar", ctypes.c_int),
        ("beta", ctypes.c_double),
        ("phi", ctypes.c_double),
        ("omega", ctypes.c_double),
        ("gid_mode", ctypes.c_int),
    ]


class Prn(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int),
        ("prns", ctypes.c_void_p),
        ("key0", ctypes.c_uint32),
        ("key1", ctypes.c_uint32),
        ("phase", ctypes.c_uint64),
        ("stream", ctypes.c_void_p),
    ]


def _load():
    src = [os.path.join(ORACLE_DIR, f) for f in ("qg_oracle.c", "qg_oracle_impl.h", "qg_oracle_learned.h",
                                                 "qg_oracle.h")]
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in src):
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    lib.ol_glibc_seeds.argtypes = [ctypes.c_uint32, ctypes.c_int, P(ctypes.c_uint32)]
    lib.ol_ranlux_init.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int]
    lib.ol_ranlux_next.argtypes = [ctypes.c_void_p]
    lib.ol_ranlux_next.restype = ctypes.c_float
    lib.ol_ranlux_states.argtypes = [P(ctypes.c_uint32), ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.ol_ranlux_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.ol_sizeof_ranlux.restype = ctypes.c_int
    lib.ol_philox4x32.argtypes = [P(ctypes.c_uint32), P(ctypes.c_uint32), P(ctypes.c_uint32)]
    lib.ol_philox_prn.argtypes = [P(Prn), ctypes.c_uint32, ctypes.c_uint32, P(ctypes.c_float)]
    for name in ("ol_init_cold", "ol_init_gid", "ol_gramschmidt", "ol_gramschmidt_fp64"):
        getattr(lib, name).argtypes = [P(Cfg), ctypes.c_void_p]
    lib.ol_init_hot_dir.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.ol_phase_hb.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, P(Prn)]
    lib.ol_phase_or.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.ol_plaquette.argtypes = [P(Cfg), ctypes.c_void_p, P(ctypes.c_double)]
    lib.ol_plaquette_f32.argtypes = [P(Cfg), ctypes.c_void_p, P(ctypes.c_double)]
    lib.ol_action.argtypes = [P(Cfg), ctypes.c_void_p, P(ctypes.c_double)]
    lib.ol_polyakov.argtypes = [P(Cfg), ctypes.c_void_p, P(ctypes.c_double)]
    lib.ol_wilson.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.ol_fmunu.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, P(ctypes.c_double)]
    lib.ol_action_profile.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, P(ctypes.c_double)]
    lib.ol_polyakov_profile.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, P(ctypes.c_double)]
    lib.ol_wilson.restype = ctypes.c_double
    lib.ol_local_action_link.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.ol_local_action_link.restype = ctypes.c_double
    fp, dp = P(ctypes.c_float), P(ctypes.c_double)
    lib.ol_expd.argtypes = [ctypes.c_double]
    lib.ol_expd.restype = ctypes.c_double
    lib.ol_mh_features.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, fp]
    lib.ol_mlp_out.argtypes = [fp, fp]
    lib.ol_mlp_out.restype = ctypes.c_float
    lib.ol_mh_phase.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, fp, ctypes.c_double, ctypes.c_int,
                                ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, P(ctypes.c_uint64), dp]
    lib.ol_mh_phase_eps.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, fp, ctypes.c_int,
                                    ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, P(ctypes.c_uint64), dp]
    lib.ol_net_eps.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, fp, ctypes.c_double, fp]
    lib.ol_mh_grad.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, fp, ctypes.c_double,
                               ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, dp, dp]
    lib.ol_mh_loss.argtypes = [P(Cfg), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp, ctypes.c_double,
                               ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]
    lib.ol_mh_loss.restype = ctypes.c_double
    return lib


lib = _load()


def align(n, a):
    return ((n + a - 1) // a) * a


def make_cfg(group=3, dims=(4, 4, 4, 4), precision=1, beta=6.0, nhit=10, nhitpar=1,
             row_align=64, gid_mode=False, phi=0.0, omega=0.0):
    c = Cfg()
    c.group = group
    for i in range(4):
        c.n[i] = dims[i]
    V = dims[0] * dims[1] * dims[2] * dims[3]
    c.precision = precision
    c.rowsize = align(V, row_align)
    c.prngstep = align(V // 2, row_align)
    c.nhit = nhit
    c.nhitpar = nhitpar
    c.beta = beta
    c.phi = phi
    c.omega = omega
    c.gid_mode = 1 if gid_mode else 0
    return c


def volume(c):
    return c.n[0] * c.n[1] * c.n[2] * c.n[3]


def new_table(c):
    planes = 12 if c.group == 3 else 4
    dt = np.float32 if c.precision == 0 else np.float64
    return np.zeros(planes * c.rowsize * 4, dtype=dt)


def vp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def glibc_seeds(series, instances):
    out = np.zeros(instances, dtype=np.uint32)
    lib.ol_glibc_seeds(series, instances, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    return out


class Ranlux:
    """Reference-layout RANLUX batch generator (one state per instance)."""

    def __init__(self, series, instances, nskip=223):
        self.instances = instances
        self.seeds = glibc_seeds(series, instances)
        self.states = ctypes.create_string_buffer(lib.ol_sizeof_ranlux() * instances)
        lib.ol_ranlux_states(self.seeds.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), instances, nskip,
                             self.states)

    def batch(self, samples):
        out = np.zeros(samples * self.instances * 4, dtype=np.float32)
        lib.ol_ranlux_batch(self.states, self.instances, samples, vp(out))
        return out


def prn_samples(c, instances, hot=False):
    """PRNG_samples for one batch (SU(N)/suncl/suncl.cpp:2304-2307, random.cpp:222)."""
    total = c.nhitpar * 3 * c.prngstep * (c.nhit + 1)
    if hot:
        total = c.rowsize * 4 + 3 * c.prngstep * (c.nhit + 1)
    return 1 + (total - 1) // instances


class Stream:
    """One RANLUX stream consumed in order (PRN source mode 2): the reference
    sequential CPU path's generator, seeded as PRNG::initialize_CPU does
    (srand(series), the first rand() mod 2^31-1)."""

    def __init__(self, series, nskip=223):
        self.state = ctypes.create_string_buffer(lib.ol_sizeof_ranlux())
        lib.ol_ranlux_init(self.state, int(glibc_seeds(series, 1)[0]), nskip)


def phase_hb(c, tab, parity, mu, prns=None, philox=None, stream=None):
    src = Prn()
    if stream is not None:
        src.mode = 2
        src.stream = ctypes.cast(stream.state, ctypes.c_void_p)
    elif prns is not None:
        src.mode = 0
        src.prns = prns.ctypes.data
    else:
        src.mode = 1
        src.key0, src.key1, src.phase = philox
    lib.ol_phase_hb(ctypes.byref(c), vp(tab), parity, mu, ctypes.byref(src))


def plaquette(c, tab):
    out = (ctypes.c_double * 2)()
    lib.ol_plaquette(ctypes.byref(c), vp(tab), out)
    return out[0], out[1]


def plaquette_f32(c, tab):
    out = (ctypes.c_double * 2)()
    lib.ol_plaquette_f32(ctypes.byref(c), vp(tab), out)
    return out[0], out[1]


def action(c, tab):
    out = (ctypes.c_double * 2)()
    lib.ol_action(ctypes.byref(c), vp(tab), out)
    return out[0], out[1]


def polyakov(c, tab):
    out = (ctypes.c_double * 4)()
    lib.ol_polyakov(ctypes.byref(c), vp(tab), out)
    return tuple(out)


def wilson(c, tab, R, T):
    return lib.ol_wilson(ctypes.byref(c), vp(tab), R, T)


def fmunu(c, tab, field, i1, i2):
    """F_munu sums as array [2 generators][3 planes][Re, Im]"""
    out = (ctypes.c_double * 12)()
    lib.ol_fmunu(ctypes.byref(c), vp(tab), field, i1, i2, out)
    return np.array(out[:]).reshape(2, 3, 2)


def action_profile(c, tab, axis):
    out = (ctypes.c_double * (2 * c.n[axis]))()
    lib.ol_action_profile(ctypes.byref(c), vp(tab), axis, out)
    return np.array(out[:]).reshape(-1, 2)


def polyakov_profile(c, tab, axis):
    out = (ctypes.c_double * (2 * c.n[axis]))()
    lib.ol_polyakov_profile(ctypes.byref(c), vp(tab), axis, out)
    return np.array(out[:]).reshape(-1, 2)


def philox(ctr, key):
    o = (ctypes.c_uint32 * 4)()
    c4 = (ctypes.c_uint32 * 4)(*ctr)
    k2 = (ctypes.c_uint32 * 2)(*key)
    lib.ol_philox4x32(c4, k2, o)
    return tuple(o)


# ---- learned-proposal Metropolis (SU(3), float links)
CHAIN_KEY1, TRAIN_KEY1 = 0x5D3E1A27, 0x2C1B3A49


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def mh_features(c, tab, gid, mu):
    x = np.zeros(8, dtype=np.float32)
    lib.ol_mh_features(ctypes.byref(c), vp(tab), gid, mu, _fp(x))
    return x


def mh_phase(c, tab, parity, mu, w, eps_max, nhit, key0, phase, key1=CHAIN_KEY1):
    w = np.ascontiguousarray(w, dtype=np.float32)
    acc = ctypes.c_uint64()
    jump = ctypes.c_double()
    lib.ol_mh_phase(ctypes.byref(c), vp(tab), parity, mu, _fp(w), eps_max, nhit, key0, key1, phase,
                    ctypes.byref(acc), ctypes.byref(jump))
    return acc.value, jump.value


def mh_phase_eps(c, tab, parity, mu, eps, nhit, key0, phase, key1=CHAIN_KEY1):
    """one Metropolis phase with the step of the t-th link given as eps[t]"""
    eps = np.ascontiguousarray(eps, dtype=np.float32)
    acc = ctypes.c_uint64()
    jump = ctypes.c_double()
    lib.ol_mh_phase_eps(ctypes.byref(c), vp(tab), parity, mu, _fp(eps), nhit, key0, key1, phase,
                        ctypes.byref(acc), ctypes.byref(jump))
    return acc.value, jump.value


def net_eps(c, tab, parity, mu, w, eps_max):
    """the network's step for every link of a phase (tensor-core definition)"""
    w = np.ascontiguousarray(w, dtype=np.float32)
    e = np.zeros(volume(c) // 2, dtype=np.float32)
    lib.ol_net_eps(ctypes.byref(c), vp(tab), parity, mu, _fp(w), eps_max, _fp(e))
    return e


def mh_grad(c, tab, parity, mu, w, eps_max, key0, phase, key1=TRAIN_KEY1, tc=False):
    """tc: the operand roundings of the tensor-core kernels (BF16); else
    the FP32 network's analytic gradient"""
    w = np.ascontiguousarray(w, dtype=np.float32)
    g = np.zeros(w.size, dtype=np.float64)
    st = (ctypes.c_double * 4)()
    lib.ol_mh_grad(ctypes.byref(c), vp(tab), parity, mu, _fp(w), eps_max, key0, key1, phase, 1 if tc else 0,
                   g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), st)
    return g, list(st)


def mh_loss(c, tab, parity, mu, w, eps_max, key0, phase, key1=TRAIN_KEY1):
    w = np.ascontiguousarray(w, dtype=np.float64)
    return lib.ol_mh_loss(ctypes.byref(c), vp(tab), parity, mu, w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                          eps_max, key0, key1, phase)


# ---- the reference's sequential CPU path (oracle/_ref/ref_cpurun "links")
def table_to_rows(c, tab):
    """reference-layout table -> per (site, dir) the stored rows as the
    reference CPU path keeps them: SU(3) u1..u3, v1..v3 (re, im) = 12
    doubles; SU(2) u1, u2 (re, im) = 4 doubles; site-major, dir fastest"""
    V = volume(c)
    planes = 12 if c.group == 3 else 4
    t = tab.astype(np.float64).reshape(planes, c.rowsize, 4)[:, :V, :]
    if c.group == 2:
        a = t[0:4].transpose(1, 0, 2)                      # [site][dir][x y z w]
        out = np.stack([a[..., 0], a[..., 2], a[..., 1], a[..., 3]], axis=-1)
        return np.ascontiguousarray(out)
    p1, p2, p3 = t[0:4].transpose(1, 0, 2), t[4:8].transpose(1, 0, 2), t[8:12].transpose(1, 0, 2)
    out = np.stack([p1[..., 0], p2[..., 0], p1[..., 1], p2[..., 1], p1[..., 2], p2[..., 2],
                    p3[..., 0], p3[..., 2], p3[..., 1], p3[..., 3], p1[..., 3], p2[..., 3]], axis=-1)
    return np.ascontiguousarray(out)


def rows_to_table(c, rows):
    V = volume(c)
    tab = new_table(c).reshape(-1, c.rowsize, 4)
    if c.group == 2:
        r = rows.reshape(V, 4, 4)
        for d in range(4):
            tab[d, :V, 0], tab[d, :V, 2], tab[d, :V, 1], tab[d, :V, 3] = r[:, d, 0], r[:, d, 1], r[:, d, 2], r[:, d, 3]
        return tab.reshape(-1)
    r = rows.reshape(V, 4, 12)
    for d in range(4):
        x = r[:, d, :]
        tab[d, :V] = np.stack([x[:, 0], x[:, 2], x[:, 4], x[:, 10]], axis=-1)
        tab[d + 4, :V] = np.stack([x[:, 1], x[:, 3], x[:, 5], x[:, 11]], axis=-1)
        tab[d + 8, :V] = np.stack([x[:, 6], x[:, 8], x[:, 7], x[:, 9]], axis=-1)
    return tab.reshape(-1)
