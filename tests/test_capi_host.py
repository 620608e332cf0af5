"""Host-side checks of the C-ABI library (no GPU needed): it loads, exports
every entry point include/qcdgpu_b200.h declares, and its host-only glibc
seeding reproduces the reference's srand/rand seeding."""
import ctypes
import os
import re

import numpy as np

import _oracle as O
import qcdgpu_b200 as Q

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "qcdgpu_b200.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(qg_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = Q.load_library()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(Q.EXPORTED_SYMBOLS)


def test_glibc_seeding_matches_reference_rand():
    for series in (54, 1, 777, 2 ** 31 - 1):
        assert np.array_equal(Q.glibc_seeds(series, 4096), O.glibc_seeds(series, 4096))


def test_default_config_mirrors_reference_main():
    c = Q.default_config()
    assert c.group == 3 and list(c.size) == [32] * 4 and c.nhit == 10 and c.nhitpar == 1
    assert c.randseries == 54 and c.ranlux_nskip == 223 and c.start == Q.START_COLD
    assert abs(c.beta - 6.5) < 1e-15 and c.wilson_r == 7 and c.wilson_t == 2


def test_create_rejects_bad_configs_without_gpu_side_effects():
    lib = Q.load_library()
    ctx = ctypes.c_void_p()
    for kw in ({"group": 4}, {"size": (4, 3, 4, 4)}, {"randseries": 0}, {"ranlux_nskip": 100}, {"nhit": 0}):
        cfg = Q.default_config(**kw)
        rc = lib.qg_create(ctypes.byref(cfg), ctypes.byref(ctx))
        assert rc == -1 and not ctx.value
        assert lib.qg_last_error(None)
