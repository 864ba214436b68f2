"""The allocation-free totals entry point (gam_totals_noalloc), for callers
that cannot call cudaMalloc while they run: called through the C ABI on
device arrays the test owns, its output must equal gam_totals (the handle's
own reduction) within FP64 summation-order round-off, on two calls in a row.
This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from mage_b200 import grids
from mage_b200.gamera import GameraGPU, GamParams, load_library, GAM_EINVAL

pytestmark = pytest.mark.gpu


def test_totals_noalloc_matches_gam_totals():
    import torch

    N = (32, 24, 16)
    g = GameraGPU(GamParams(*N))
    g.set_geometry(grids.warped_periodic_corners(*N))
    g.init_blast_wave()
    g.step_gamera(3)
    ref = g.totals()
    st = g.download_state(old=False)
    vol = g.get_geometry_arrays()["volume"]
    gas_d = torch.from_numpy(np.ascontiguousarray(st["Gas"])).cuda()
    vol_d = torch.from_numpy(np.ascontiguousarray(vol)).cuda()
    out_d = torch.empty(5, dtype=torch.float64, device="cuda")
    L = load_library()
    err = C.create_string_buffer(256)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        out_d.fill_(float("nan"))
        rc = L.gam_totals_noalloc(C.c_void_p(gas_d.data_ptr()), C.c_void_p(vol_d.data_ptr()), *N,
                                  C.c_void_p(out_d.data_ptr()), stream, err, len(err))
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        got = out_d.cpu().numpy()
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-14), (call, got, ref)


def test_totals_noalloc_rejects_oversize_grid():
    L = load_library()
    err = C.create_string_buffer(256)
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.gam_totals_noalloc(dummy, dummy, 8192, 8192, 2, dummy, None, err, len(err))
    assert rc == GAM_EINVAL
    assert b"exceed" in err.value
