"""Pins the CPU oracle to the reference before anything is checked against it.

* RANLUX: the oracle's generator reproduces, bit for bit, the stream of the
  reference's own host RANLUX (random/random.cpp RL_produce_one_CPU), which
  PRNG::check (random.cpp:339-402) requires GPU instance 0 to equal.
* glibc seeding: RANDSERIES -> instance seeds as PRNG::initialize does.
* Philox4x32-10: the published known-answer vectors of the algorithm.
* Heatbath link by link: fed one RANLUX3 stream in order, the oracle's
  heatbath phases reproduce the links of the reference's sequential CPU
  heatbath (SU(N)/suncpp) to 1e-12 -- Kennedy-Pendleton draws with their
  accept/reject decisions, subgroup embedding and Gram-Schmidt.
* Deterministic INTS=2 mode: the oracle's restatement of the update kernels
  reproduces the plaquettes of the reference's sequential CPU path
  (SU(N)/suncpp) -- to 1e-14 on the closed-form start and to the ~1e-7
  level after sweeps (the CPU path stores its deterministic "random" numbers
  in float, SU(N)/suncpp/su2/update_su2.cpp:44, and sums staple planes in
  another order).
"""
import ctypes
import json
import os
import struct
import subprocess

import numpy as np
import pytest

import _oracle as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))
NSKIP = [24, 48, 97, 223, 389]


def bits(x):
    return struct.unpack("<I", struct.pack("<f", x))[0]


@pytest.mark.parametrize("case", GOLDEN["ranlux"], ids=lambda c: "s%d-lux%d" % (c["randseries"], c["luxury"]))
def test_ranlux_instance0_matches_reference_stream(case):
    seeds = O.glibc_seeds(case["randseries"], 2)
    assert int(seeds[0]) == case["jseed"]
    st = ctypes.create_string_buffer(O.lib.ol_sizeof_ranlux())
    O.lib.ol_ranlux_init(st, int(seeds[0]), NSKIP[case["luxury"]])
    got = [bits(O.lib.ol_ranlux_next(st)) for _ in range(len(case["bits"]))]
    assert got == case["bits"]


def test_ranlux_batch_layout_is_instance_major():
    """ranlux kernel layout: prns[s*instances + i] = 4 consecutive outputs."""
    R = O.Ranlux(54, 8)
    b = R.batch(3).reshape(3, 8, 4)
    seeds = O.glibc_seeds(54, 8)
    for i in (0, 5):
        st = ctypes.create_string_buffer(O.lib.ol_sizeof_ranlux())
        O.lib.ol_ranlux_init(st, int(seeds[i]), 223)
        ref = np.array([O.lib.ol_ranlux_next(st) for _ in range(12)], dtype=np.float32).reshape(3, 4)
        assert np.array_equal(b[:, i, :], ref)


def test_ranlux_values_in_open_unit_interval():
    """PRNG::check_range (random.cpp:403-423)."""
    b = O.Ranlux(99, 64).batch(200)
    assert np.all(b > 0) and np.all(b < 1)


@pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "ref_ranlux")), reason="oracle/_ref not built")
def test_ranlux_live_against_reference_binary():
    out = subprocess.check_output([os.path.join(O.REF_DIR, "ref_ranlux"), "31337", "3", "3000"]).decode().split()
    ref = [bits(float.fromhex(x)) for x in out[4:]]
    seeds = O.glibc_seeds(31337, 1)
    st = ctypes.create_string_buffer(O.lib.ol_sizeof_ranlux())
    O.lib.ol_ranlux_init(st, int(seeds[0]), 223)
    assert [bits(O.lib.ol_ranlux_next(st)) for _ in range(3000)] == ref


def test_philox_known_answers():
    assert O.philox((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert O.philox((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF)) == (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    assert O.philox((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == \
        (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


def run_gid(group, dims, beta, sweeps):
    c = O.make_cfg(group=group, dims=dims, precision=1, beta=beta, gid_mode=True)
    t = O.new_table(c)
    O.lib.ol_init_gid(ctypes.byref(c), O.vp(t))
    V = O.volume(c)
    rows = []
    for s in range(sweeps + 1):
        if s:
            for par in (1, 0):
                for mu in range(4):
                    O.phase_hb(c, t, par, mu, philox=(0, 0, 0))
            O.lib.ol_gramschmidt(ctypes.byref(c), O.vp(t))
        sp, tp = O.plaquette(c, t)
        rows.append((sp / (3 * V), tp / (3 * V)))
    return rows


@pytest.mark.parametrize("case", GOLDEN["gid"], ids=lambda c: "su%d-%s" % (c["group"], "x".join(map(str, c["dims"]))))
def test_gid_mode_matches_reference_cpu_path(case):
    rows = run_gid(case["group"], tuple(case["dims"]), case["beta"], len(case["rows"]) - 1)
    for (sp, tp), ref in zip(rows, case["rows"]):
        tol = 1e-13 if ref[0] == 0 else 2e-7
        assert abs(sp - ref[1]) <= tol * max(1, abs(ref[1])), (ref[0], sp, ref[1])
        assert abs(tp - ref[2]) <= tol * max(1, abs(ref[2])), (ref[0], tp, ref[2])


def test_cold_start_observables_exact():
    """Cold start: Plq = N, P = 1 exactly (a known answer)."""
    for g in (2, 3):
        c = O.make_cfg(group=g, dims=(4, 4, 4, 6), precision=0)
        t = O.new_table(c)
        O.lib.ol_init_cold(ctypes.byref(c), O.vp(t))
        sp, tp = O.plaquette(c, t)
        V = O.volume(c)
        assert sp == 3 * V * g and tp == 3 * V * g
        re, im, p2, p4 = O.polyakov(c, t)
        assert re == 4 * 4 * 4 * g and im == 0


def test_fp32_product_plaquette_against_fp64_products():
    """ol_plaquette_f32 (products and traces in FP32, sums in FP64): exact on
    a cold start; on FP32 links within 1e-6 of the FP64-product plaquette
    (normalised by 3 V N); on FP64 links the FP64 plaquette itself."""
    for g in (2, 3):
        for prec in (0, 1):
            c = O.make_cfg(group=g, dims=(4, 4, 4, 6), precision=prec, beta=5.7)
            t = O.new_table(c)
            O.lib.ol_init_cold(ctypes.byref(c), O.vp(t))
            V = O.volume(c)
            assert O.plaquette_f32(c, t) == (3.0 * V * g, 3.0 * V * g)
            R = O.Ranlux(7, 256)
            n = O.prn_samples(c, 256, hot=True)
            R.batch(n)
            for mu in range(4):
                O.lib.ol_init_hot_dir(ctypes.byref(c), O.vp(t), mu, O.vp(R.batch(n)))
            a, b = O.plaquette_f32(c, t), O.plaquette(c, t)
            if prec:
                assert a == b
            else:
                assert a != b
                assert max(abs(x - y) for x, y in zip(a, b)) / (3 * V * g) <= 1e-6, (a, b)


def test_overrelaxation_preserves_local_action():
    """Microcanonical reflection: Re Tr(U*staple) of each updated link is unchanged."""
    for g in (2, 3):
        c = O.make_cfg(group=g, dims=(4, 4, 4, 4), precision=1, beta=5.7)
        t = O.new_table(c)
        R = O.Ranlux(7, 256)
        n = O.prn_samples(c, 256, hot=True)
        R.batch(n)
        for mu in range(4):
            O.lib.ol_init_hot_dir(ctypes.byref(c), O.vp(t), mu, O.vp(R.batch(n)))
        even = [s for s in range(O.volume(c)) if sum(site_coords(c, s)) % 2 == 0]
        before = [O.lib.ol_local_action_link(ctypes.byref(c), O.vp(t), s, 2) for s in even]
        old = t.copy()
        O.lib.ol_phase_or(ctypes.byref(c), O.vp(t), 0, 2)
        after = [O.lib.ol_local_action_link(ctypes.byref(c), O.vp(t), s, 2) for s in even]
        assert np.allclose(before, after, rtol=0, atol=1e-12)
        assert not np.allclose(old, t)                         # the links did move
        O.lib.ol_phase_or(ctypes.byref(c), O.vp(t), 0, 2)      # SU(2): a reflection is an involution
        if g == 2:
            assert np.allclose(old, t, rtol=0, atol=1e-13)


def site_coords(c, s):
    n1, n2, n3, n4 = c.n
    x = s // (n2 * n3 * n4)
    r = s - x * n2 * n3 * n4
    tt = r // (n2 * n3)
    r -= tt * n2 * n3
    z = r // n2
    return (x, r - z * n2, z, tt)


def test_own_elementary_functions_accuracy():
    """The sin/cos/log routines the update path uses (own Cody-Waite +
    Taylor code; the table-driven log) stay within 2 ulp of the C library:
    on the heatbath's arguments 1 - r, on a log-uniform sweep of the normal
    range and just below and above 1 (where the table's heads cancel)."""
    lib = O.lib
    for n in ("ol_sin", "ol_cos", "ol_logd"):
        getattr(lib, n).argtypes = [ctypes.c_double]
        getattr(lib, n).restype = ctypes.c_double
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-7, 7, 20000), np.float32(rng.uniform(0, 1, 5000)) * np.float32(6.283185307179586)])
    for x in xs:
        for f, g in ((lib.ol_sin, np.sin), (lib.ol_cos, np.cos)):
            a, b = f(float(x)), float(g(x))
            assert abs(a - b) <= 2 * np.spacing(max(abs(b), 1e-300)) + 1e-17, (x, a, b)
    near1 = np.concatenate([1.0 - np.ldexp(1.0, -np.arange(1, 54)), 1.0 + np.ldexp(1.0, -np.arange(1, 53)),
                            1.0 + rng.uniform(-2 ** -6, 2 ** -6, 5000)])
    ys = np.concatenate([1.0 - np.float32(rng.uniform(0, 1, 20000)).astype(np.float64), [2.0 ** -24, 0.5, 1.0],
                         10.0 ** rng.uniform(-300, 300, 20000), near1])
    worst = 0.0
    for y in ys:
        a, b = lib.ol_logd(float(y)), float(np.log(y))
        assert abs(a - b) <= 2 * np.spacing(abs(b)) + 1e-300, (y, a, b)
        if b != 0.0:
            worst = max(worst, abs(a - b) / float(np.spacing(abs(b))))
    print("worst log error: %.2f ulp" % worst)


def test_own_float_sincos_accuracy():
    """The float sin/cos of the FP32 update path (heatbath cos(2 pi r) and
    direction angles, hot start, twist factors): within 2 float ulp of the
    exact value (or 1e-7 absolute near a zero), on the heatbath's arguments
    float(2 pi) * r for r a multiple of 2^-24, on pi * r, and on [-100, 100]"""
    lib = O.lib
    for n in ("ol_sinf_own", "ol_cosf_own"):
        getattr(lib, n).argtypes = [ctypes.c_float]
        getattr(lib, n).restype = ctypes.c_float
    rng = np.random.default_rng(1)
    r = (np.floor(rng.uniform(0, 2 ** 24, 40000)) + 0.5).astype(np.float32) * np.float32(2.0 ** -24)
    xs = np.concatenate([r * np.float32(6.283185307179586), r * np.float32(3.141592653589793),
                         rng.uniform(-100, 100, 20000).astype(np.float32)])
    worst = 0.0
    for x in xs:
        xd = float(np.float32(x))
        for f, g in ((lib.ol_sinf_own, np.sin), (lib.ol_cosf_own, np.cos)):
            a, b = float(f(xd)), float(g(xd))
            tol = max(2 * float(np.spacing(np.float32(abs(b)))), 1e-7)
            worst = max(worst, abs(a - b) / float(np.spacing(np.float32(max(abs(b), 1e-30)))))
            assert abs(a - b) <= tol, (x, a, b)
    print("worst float sin/cos error: %.2f ulp" % worst)


# ---------------------------------------------- heatbath link by link
HB_LINKS = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_heatbath_links.npz"))
HB_CASES = [("su3_b6.0", 3, (4, 4, 2, 4), 6.0), ("su3_b1.5", 3, (4, 4, 2, 4), 1.5),
            ("su2_b2.3", 2, (4, 4, 2, 4), 2.3), ("su2_b0.6", 2, (4, 4, 2, 4), 0.6)]


def _sequential_phases(c, tab, phases, series=54):
    """the oracle's heatbath phases drawing one RANLUX3 stream in order, as
    the reference's sequential CPU path does (PRN source mode 2); returns
    the number of Kennedy-Pendleton numbers drawn"""
    st = O.Stream(series)
    for k in range(phases):
        O.phase_hb(c, tab, 1 - (k // 4) % 2, k % 4, stream=st)
    probe = O.Stream(series)
    n = 0
    # count the stream's consumption by finding where the two states meet
    ref = bytes(st.state)
    while bytes(probe.state) != ref:
        O.lib.ol_ranlux_next(probe.state)
        n += 1
    return n


@pytest.mark.parametrize("case", HB_CASES, ids=lambda c: c[0])
def test_heatbath_links_match_reference_cpu_path(case):
    """The heatbath arithmetic itself against the reference's executed code:
    from the same thermalising start and the same RANLUX3 stream drawn in
    order, one sweep of 8 heatbath phases of the oracle reproduces the links
    of the reference's sequential CPU heatbath (SU(N)/suncpp/su2/
    update_su2.cpp:40-126, su3/update_su3.cpp:40-114; golden file made by
    tests/golden/make_heatbath_links.py) to 1e-12 -- the Kennedy-Pendleton
    log(1-r) draw, its accept/reject decision (the low-coupling cases reject
    often), the direction draw, the subgroup embedding and the per-link
    Gram-Schmidt.  The two sides differ only in rounding order (staple
    association, matrix products, the log and cos routines): measured
    max|dU| <= 4e-15, and 3e-13 for SU(3) at beta = 1.5, where cos(alpha) =
    1 - delta nears -1 and sqrt(1 - cos^2) magnifies last-bit differences."""
    name, group, dims, beta = case
    c = O.make_cfg(group=group, dims=dims, precision=1, beta=beta, row_align=64)
    tab = O.rows_to_table(c, HB_LINKS[name + "_start"])
    drawn = _sequential_phases(c, tab, 8)
    ref = O.rows_to_table(c, HB_LINKS[name + "_ref"])
    d = float(np.max(np.abs(tab - ref)))
    links = O.volume(c) // 2 * 8
    tries_per_link = (drawn - 2 * links * (3 if group == 3 else 1)) / 4.0 / (links * (3 if group == 3 else 1))
    print("%s: max|dU| = %.3g, %.3f Kennedy-Pendleton tries per draw" % (name, d, tries_per_link))
    assert d <= 1e-12
    if beta < 2.0:
        assert tries_per_link > 1.3                  # the rejection path is exercised


@pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "ref_cpurun")), reason="oracle/_ref not built")
@pytest.mark.parametrize("group,beta", [(3, 6.0), (2, 2.3)])
def test_heatbath_links_live_against_reference_binary_8x4(group, beta):
    """The same comparison at the SU(2) run configuration's lattice size (8^4)
    over two sweeps, against the reference binary run live"""
    import tempfile
    dims = (8, 8, 8, 8)
    c = O.make_cfg(group=group, dims=dims, precision=1, beta=beta, row_align=64)
    tab = O.new_table(c)
    O.lib.ol_init_cold(ctypes.byref(c), O.vp(tab))
    for ph in range(8):
        O.phase_hb(c, tab, 1 - (ph // 4) % 2, ph % 4, philox=(9, 0x5D3E1A27, ph))
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        O.table_to_rows(c, tab).tofile(fin)
        subprocess.check_call([os.path.join(O.REF_DIR, "ref_cpurun"), "links", str(group)] +
                              [str(x) for x in dims] + [repr(beta), "54", "16", fin, fout])
        ref = O.rows_to_table(c, np.fromfile(fout, dtype=np.float64))
    _sequential_phases(c, tab, 16)
    d = float(np.max(np.abs(tab - ref)))
    print("SU(%d) 8^4 two sweeps: max|dU| = %.3g" % (group, d))
    assert d <= 1e-12


def test_log_table_is_its_generator_output_and_exact():
    """qg_logtab.h (shared by the device log and the oracle's) is what
    gen_logtab.py writes, c_k is the correctly rounded 1/(1 + k/128), the
    heads are multiples of 2^-32 and head + tail equals -log c_k to within
    2^-60 (checked with Python's decimal logarithm at 40 digits)"""
    import importlib.util
    import tempfile
    from decimal import Decimal, getcontext
    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "qcdgpu_b200", "csrc")
    spec = importlib.util.spec_from_file_location("gen_logtab", os.path.join(csrc, "gen_logtab.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "qg_logtab.h")
        gen.emit(p)
        assert open(p).read() == open(os.path.join(csrc, "qg_logtab.h")).read()
    ln2_hi, ln2_lo, c, lhi, llo = gen.table()
    getcontext().prec = 40
    for k in range(129):
        assert c[k] == 1.0 / (1.0 + k / 128.0)
        assert (lhi[k] * 2.0 ** 32).is_integer()
        err = Decimal(lhi[k]) + Decimal(llo[k]) + Decimal(c[k]).ln()
        assert abs(err) <= Decimal(2) ** -60, (k, err)
    assert (ln2_hi * 2.0 ** 32).is_integer()
    assert abs(Decimal(ln2_hi) + Decimal(ln2_lo) - Decimal(2).ln()) <= Decimal(2) ** -60


@pytest.mark.parametrize("group,beta,prec", [(3, 6.0, 0), (2, 2.3, 0), (3, 6.0, 1), (2, 2.3, 1)])
def test_own_heatbath_arithmetic_against_the_reference_expression(group, beta, prec):
    """How far this build's Kennedy-Pendleton arithmetic (delta with one fused
    multiply-add, its own float cos / sin and table-driven log) moves the
    chain from the reference's expression as written (su3_update_cl.cl:
    619-620: product and sum rounded separately; the C library's cos / sin /
    log standing in for the OpenCL runtime's, whose float cos is itself only
    specified to 4 ulp): one heatbath sweep of a thermalised 8^4 field from
    the same start and Philox stream.  Measured max|dU| 1.2e-6 (SU(3)) and
    3.9e-7 (SU(2)) in FP32, 1e-15 in FP64, no accept decision flipped --
    inside the 2e-6 / 1e-12 one-sweep tolerances (other streams: 4e-7 to
    8e-7 in FP32 after one sweep, up to 2.3e-6 after three)."""
    O.lib.ol_set_reference_arith.argtypes = [ctypes.c_int]
    c = O.make_cfg(group=group, dims=(8, 8, 8, 8), precision=prec, beta=beta, row_align=64)
    t = O.new_table(c)
    O.lib.ol_init_cold(ctypes.byref(c), O.vp(t))
    for ph in range(80):
        O.phase_hb(c, t, 1 - (ph // 4) % 2, ph % 4, philox=(7, 0x5D3E1A27, ph))
    a, b = t.copy(), t.copy()
    try:
        for ph in range(8):
            args = dict(philox=(11, 0x1234567, 1000 + ph))
            O.phase_hb(c, a, 1 - ph // 4, ph % 4, **args)
            O.lib.ol_set_reference_arith(1)
            O.phase_hb(c, b, 1 - ph // 4, ph % 4, **args)
            O.lib.ol_set_reference_arith(0)
    finally:
        O.lib.ol_set_reference_arith(0)
    d = float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64))))
    print("SU(%d) %s: max|dU| = %.3g after one sweep" % (group, "FP64" if prec else "FP32", d))
    assert d <= (1e-12 if prec else 2e-6)
