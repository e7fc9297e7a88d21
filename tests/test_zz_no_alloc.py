"""The allocation-free mass-budget entry point against the context path.

f3d_mass_volume_noalloc serves callers that cannot allocate device memory
(their device arrays are owned by their own runtime or a pool reserved at
start-up), so it takes only device pointers the caller already holds and
keeps its partial sums in a fixed device array.  The test allocates the
device copies itself (the entry point never does), calls the entry point
twice in a row on the same stream and requires both results to equal
f3d_ads_mass_volume on the same state bit for bit (both paths add the same
cells in the same order with the same compensation).  Around the second
call it checks the property the entry point exists for: the device's free
memory and torch's allocated bytes do not change.  It runs last in the
suite so that a failure here never hides another test.
"""
import ctypes as C

import numpy as np
import pytest

from fall3d_b200 import workloads as W
from fall3d_b200._lib import last_error, lib
from fall3d_b200.ads import Domain

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))).cuda()


def test_mass_volume_noalloc_matches_context_path(built_lib):
    import torch
    wl = W.small_case(40, 30, 12, 5, seed=77)
    g = wl.grid
    c0, a0 = W.random_state(wl, seed=13)
    dom = Domain(g, wl.nbins)
    dom.upload_state(c0, a0)
    ref_total, ref_pb = dom.grid_get_mass_volume(per_bin=True)
    dom.close()

    c_d = _dev(torch, c0)
    d1, d2, d3 = _dev(torch, g.dX1_p), _dev(torch, g.dX2_p), _dev(torch, g.dX3_p)
    pb_d = torch.zeros(wl.nbins, dtype=torch.float64, device="cuda")
    tot_d = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    for call in range(2):
        pb_d.fill_(-1.0)
        tot_d.fill_(-1.0)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        alloc0 = torch.cuda.memory_allocated()
        rc = lib().f3d_mass_volume_noalloc(g.nx, g.ny, g.nz, wl.nbins, vp(c_d), vp(d1), vp(d2),
                                           vp(d3), vp(pb_d), vp(tot_d), C.c_void_p(stream.cuda_stream))
        assert rc == 0, last_error()
        torch.cuda.synchronize()
        if call == 1:  # the first call may load the module (and commit its array)
            assert torch.cuda.mem_get_info()[0] == free0, "device memory changed across the call"
            assert torch.cuda.memory_allocated() == alloc0
        total = float(tot_d.cpu()[0])
        pb = pb_d.cpu().numpy()
        assert total == ref_total, (call, total, ref_total)
        assert np.array_equal(pb, ref_pb), (call, pb, ref_pb)


def test_mass_volume_noalloc_rejects_too_many_bins(built_lib):
    import torch
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(x.data_ptr())
    rc = lib().f3d_mass_volume_noalloc(1, 1, 1, 65, p, p, p, p, p, p, None)
    assert rc == 1
    assert "65 bins exceed" in last_error()
