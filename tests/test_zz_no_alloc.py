"""qg_plaquette_noalloc: the allocation-free plaquette/action entry point.

It is meant for callers that may not allocate device memory where they
measure (a framework that owns the memory pool, a loop where cudaMalloc
would synchronise the device).  Here the caller's device buffers come from
torch; the entry point's sums must equal those of the regular path
(qg_measure) on two calls in a row, since every call reuses the library's
fixed scratch array.  Collected last so a failure here cannot hide others.
"""
import ctypes

import numpy as np
import pytest

import qcdgpu_b200 as Q

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("group,precision,dims", [(3, 0, (8, 8, 8, 8)), (3, 1, (4, 6, 4, 8)), (2, 0, (6, 4, 4, 4))])
def test_noalloc_matches_qg_measure_twice(group, precision, dims):
    import torch

    L = Q.Lattice(Q.default_config(group=group, size=dims, precision=precision, start=Q.START_HOT,
                                   prng=Q.PRNG_PHILOX, beta=5.7 if group == 3 else 2.3))
    L.seed()
    L.init()
    L.sweep(2)
    plq = L.plaquette_sums()
    act = L.action_sums()
    table = L.download()
    rowsize = L.info().rowsize
    L.close()
    dev_links = torch.from_numpy(table).to("cuda")
    size = (ctypes.c_int * 4)(*dims)
    lib = Q.load_library()
    for call in range(2):
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.qg_plaquette_noalloc(dev_links.data_ptr(), group, precision, size, rowsize,
                                      5.7 if group == 3 else 2.3, out.data_ptr(), None)
        assert rc == 0, lib.qg_last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = np.array([plq[0], plq[1], act[0], act[1]])
        assert np.allclose(got, ref, rtol=1e-13, atol=1e-9), (call, got, ref)


def test_noalloc_rejects_lattices_beyond_the_scratch():
    import torch

    lib = Q.load_library()
    dummy = torch.zeros(4, dtype=torch.float32, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    size = (ctypes.c_int * 4)(66, 64, 64, 64)
    rc = lib.qg_plaquette_noalloc(dummy.data_ptr(), 3, 0, size, 66 * 64 ** 3, 6.0, out.data_ptr(), None)
    assert rc == Q.QG_ERR_ARG
    assert b"exceeds the fixed scratch" in lib.qg_last_error(None)


def test_noalloc_padded_rows_on_a_side_stream():
    """A table whose planes are padded beyond the site count (rowsize > V),
    read on a caller's stream other than the default one, twice"""
    import torch

    dims, group, precision = (4, 4, 6, 4), 3, 0
    L = Q.Lattice(Q.default_config(group=group, size=dims, precision=precision, start=Q.START_HOT,
                                   prng=Q.PRNG_PHILOX, beta=5.9))
    L.seed()
    L.init()
    L.sweep(1)
    plq, act = L.plaquette_sums(), L.action_sums()
    table = L.download()
    rowsize = L.info().rowsize
    L.close()
    pad = rowsize + 96
    padded = np.zeros(12 * pad * 4, dtype=np.float32)
    padded.reshape(12, pad, 4)[:, :rowsize, :] = table.reshape(12, rowsize, 4)
    side = torch.cuda.Stream()
    lib = Q.load_library()
    size = (ctypes.c_int * 4)(*dims)
    with torch.cuda.stream(side):
        dev_links = torch.from_numpy(padded).to("cuda", non_blocking=False)
        for call in range(2):
            out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
            rc = lib.qg_plaquette_noalloc(dev_links.data_ptr(), group, precision, size, pad, 5.9, out.data_ptr(),
                                          ctypes.c_void_p(side.cuda_stream))
            assert rc == Q.QG_OK, lib.qg_last_error(None)
            side.synchronize()
            got = out.cpu().numpy()
            ref = np.array([plq[0], plq[1], act[0], act[1]])
            assert np.allclose(got, ref, rtol=1e-13, atol=1e-9), (call, got, ref)
