"""Host-side checks of the C-ABI library (no GPU needed): it loads, exports
every entry point include/qcdgpu_b200.h declares, the header compiles as C
with the integration guide's examples, and its host-only glibc seeding
reproduces the reference's srand/rand seeding."""
import ctypes
import os
import re

import numpy as np
import pytest

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


def test_header_compiles_as_c_and_the_integration_examples_link(tmp_path):
    """include/qcdgpu_b200.h is a plain C header: the two usage examples of
    the integration guide (qg_run from an init.dat; the reference's kernel
    sequence through qg_phase) compile as C11 and link against the library"""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "example.c"
    src.write_text(r"""
#include <stdio.h>
#include "qcdgpu_b200.h"
int run_file(void)
{
    qg_config cfg; qg_run_options opt; qg_run_result res;
    qg_default_config(&cfg); qg_default_run_options(&opt);
    if (qg_parse_init_file("init.dat", &cfg, &opt) || qg_run(&cfg, &opt, &res))
        fprintf(stderr, "%s\n", qg_last_error(NULL));
    return 0;
}
int low_level(qg_config cfg)
{
    qg_ctx *ctx; qg_create(&cfg, &ctx);
    qg_prng_seed(ctx, cfg.randseries);
    qg_init_links(ctx, QG_START_HOT);
    for (int p = 1; p >= 0; --p) for (int d = 0; d < 4; ++d) {
        qg_prng_produce(ctx);
        qg_phase(ctx, p, d, QG_UPDATE_HEATBATH);
    }
    qg_reunitarize(ctx, 0);
    double plq[2]; qg_measure(ctx, QG_MEAS_PLAQUETTE, plq);
    qg_destroy(ctx);
    return 0;
}
int main(void) { return 0; }
""")
    lib = os.path.join(root, "qcdgpu_b200", "lib")
    r = subprocess.run([cc, "-std=c11", "-Wall", "-Werror", "-I", os.path.join(root, "include"), str(src),
                        "-L", lib, "-lqg_sun", "-Wl,-rpath," + lib, "-o", str(tmp_path / "example")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("kw,why", [
    (dict(size=(4, 5, 4, 4)), "even"),                           # N2 odd: no checkerboard
    (dict(size=(1, 4, 4, 4)), "[2, 4096]"),                      # extent below 2
    (dict(size=(8192, 4, 4, 4)), "[2, 4096]"),                   # extent above 4096
    (dict(size=(2048, 2048, 2048, 2)), "2^31"),                  # volume above 2^31 sites
    (dict(group=4), "GROUP"),
    (dict(precision=2), "precision"),
    (dict(nhit=0), "NHIT"),
    (dict(randseries=0), "RANDSERIES 0"),
])
def test_create_rejects_invalid_configurations(kw, why):
    """qg_create refuses configurations the kernels cannot run, before any
    device work (no GPU needed), with the reason in qg_last_error(NULL)"""
    base = dict(group=3, size=(4, 4, 4, 4), precision=0)
    base.update(kw)
    lib = Q.load_library()
    cfg = Q.default_config(**base)
    ctx = ctypes.c_void_p()
    rc = lib.qg_create(ctypes.byref(cfg), ctypes.byref(ctx))
    assert rc == Q.QG_ERR_ARG and not ctx.value
    assert why in lib.qg_last_error(None).decode()
