"""init.dat parsing (host only): the reference's KEY = value format as read
by GPU::get_init_file and applied by model::lattice_get_init_file."""
import os

import pytest

import qcdgpu_b200 as Q


def write(tmp_path, text):
    p = os.path.join(str(tmp_path), "init.dat")
    with open(p, "w") as f:
        f.write(text)
    return p


def test_reference_style_keys(tmp_path):
    p = write(tmp_path, "\tPLATFORM = 0\nDEVICE= 0\nFINISHPATH=./\nOUTPUTPATH=/tmp/out/\nGROUP = 2\nND = 4\n"
                        "LT = 16\nLS = 12\nITER = 50\nNITER = 10\nNHIT = 7\nBETA = 3.5000000000000e+00\nNAV = 50\n"
                        "INTS = 1\nPRNG = RANLUX4\nRANDSERIES = 1234\nGETWILSON = 1\nWILSONR = 10\nWILSONT = 3\n"
                        "PL_LEVEL = 3\nOMEGA = 0.0000000000000e+00\nPHI = 3.000000000000e+00\nFMUNU = 1\n")
    cfg, o = Q.parse_init_file(p)
    assert cfg.group == 2 and list(cfg.size) == [12, 12, 12, 16]
    assert o.iter == 50 and o.niter == 10 and o.nav == 50 and cfg.nhit == 7
    assert cfg.beta == 3.5 and cfg.phi == 3.0 and cfg.omega == 0.0
    assert cfg.start == Q.START_COLD and cfg.prng == Q.PRNG_RANLUX and cfg.ranlux_nskip == 389
    assert cfg.randseries == 1234 and o.get_wilson == 1 and cfg.wilson_r == 10 and cfg.wilson_t == 3
    assert o.pl_level == 3 and o.output_path == b"/tmp/out/" and o.prefix == b"su2-"


def test_comments_whitespace_and_new_keys(tmp_path):
    p = write(tmp_path, "# SU(3) 24^3 x 6 working point\n  L1 = 24   # x\nL2=24\nL3 =24\nL4= 6\nBETA = 5.9\n"
                        "PRECISION = 0\nNOR = 4\nREUNIT_EVERY = 10\nREUNIT_FP64 = 1\nPRNG = PHILOX\nINTS = 2\n"
                        "NHITPAR = 2\nPRNG_INSTANCES = 4096\nROW_ALIGN = 128\n\n")
    cfg, o = Q.parse_init_file(p)
    assert list(cfg.size) == [24, 24, 24, 6] and abs(cfg.beta - 5.9) < 1e-15
    assert cfg.precision == 0 and cfg.n_or == 4 and cfg.reunit_every == 10 and cfg.reunit_fp64 == 1
    assert cfg.prng == Q.PRNG_PHILOX and cfg.start == Q.START_GID and cfg.nhitpar == 2
    assert cfg.prng_instances == 4096 and cfg.row_align == 128


def test_defaults_untouched_without_keys(tmp_path):
    cfg, o = Q.parse_init_file(write(tmp_path, "\n# nothing\n"))
    d = Q.default_config()
    assert list(cfg.size) == list(d.size) and cfg.beta == d.beta and o.iter == 2 and o.niter == 1


@pytest.mark.parametrize("text,msg", [("PRNG = XOR128\n", "XOR128"), ("FOO = 1\n", "FOO"), ("ND = 3\n", "ND")])
def test_errors(tmp_path, text, msg):
    with pytest.raises(Q.QGError, match=msg):
        Q.parse_init_file(write(tmp_path, text))


def test_missing_file():
    with pytest.raises(Q.QGError, match="cannot open"):
        Q.parse_init_file("/nonexistent/init.dat")


def test_fmunu_and_profile_keys(tmp_path):
    """FMUNU / F0MU / TURNOFFFMUNU and the generator keys FMUNU1/2/4/5/6/7
    (suncl.cpp:412-452); PL_LEVEL 3 (Polyakov profiles) is the reference
    main()'s default; ACTIONS_DIFF switches on the action profiles"""
    d = Q.default_run_options()
    assert d.pl_level == 3 and d.fmunu == 0 and d.get_actions_diff == 0
    cfg, o = Q.parse_init_file(write(tmp_path, "FMUNU = 1\nFMUNU4 = 1\nFMUNU6 = 1\nACTIONS_DIFF = 1\n"))
    assert o.fmunu == 1 and o.fmunu_index1 == 4 and o.fmunu_index2 == 6 and o.get_actions_diff == 1
    cfg, o = Q.parse_init_file(write(tmp_path, "FMUNU = 1\nF0MU = 1\nFMUNU1 = 1\nFMUNU2 = 1\n"))
    assert o.fmunu == 2 and o.fmunu_index1 == 2
    cfg, o = Q.parse_init_file(write(tmp_path, "F0MU = 1\nTURNOFFFMUNU = 1\nFMUNU3 = 1\n"))
    assert o.fmunu == 0
    assert d.tune_shapes == 1
    cfg, o = Q.parse_init_file(write(tmp_path, "TUNE = 0\n"))
    assert o.tune_shapes == 0
    assert d.profile == 0
    cfg, o = Q.parse_init_file(write(tmp_path, "PROFILE = 1\n"))
    assert o.profile == 1
