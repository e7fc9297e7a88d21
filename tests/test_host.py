"""CPU tests of the host side: the Python builders against the C oracle's
restatements, the C ABI's exported symbols, and the replica partition."""
import ctypes as C
import math
import os
import re
import socket
import subprocess

import numpy as np
import pytest

from fall3d_b200 import grid as G
from fall3d_b200 import meteo, source
from fall3d_b200 import workloads as W
from fall3d_b200.replicas import partition_members

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_grid_metrics():
    g = G.build_arakawa_c(10, 8, 6, 10.0, 10.5, 0.0, 0.4, 3000.0, G.uniform_sigma(6))
    d1 = G.REARTH * 0.05 * math.pi / 180.0
    assert np.allclose(g.dX1_p, d1, rtol=1e-15) and np.allclose(g.dX2_b, d1, rtol=1e-15)
    assert np.allclose(g.dX3_b, 500.0) and np.allclose(g.dX3_p, 500.0)
    assert np.allclose(g.Hm1_p, [math.sin((90.0 - lat) * math.pi / 180.0) for lat in g.lat_p])
    assert np.all(g.Hm3_p == 1.0) and g.z_c[3, 4, 6] == 3000.0


def test_grid_vertical_halos_follow_reference():
    sig = np.array([0.0, 0.1, 0.25, 0.45, 0.7, 1.0])
    g = G.build_arakawa_c(4, 4, 5, 0.0, 0.2, 0.0, 0.2, 1000.0, sig)
    # dX3_b(k) = (s(k+1)-s(k)) X3max, k=1..nz; dX3_b(0)=dX3_b(1); dX3_b(nz+1:nz+2)=dX3_b(nz)
    assert np.allclose(g.dX3_b, [100, 100, 150, 200, 250, 300, 300, 300])
    # dX3_p(k) between mass points k, k+1 for k=1..nz-1; halos copy the ends
    mid = 0.5 * (sig[1:] + sig[:-1]) * 1000.0
    inner = np.diff(mid)
    assert np.allclose(g.dX3_p[2:6], inner)
    assert np.allclose(g.dX3_p[:2], inner[0]) and np.allclose(g.dX3_p[6:], inner[-1])


def test_suzuki_matches_oracle(oracle_mod):
    fc = np.array([0.1, 0.3, 0.6])
    z_p, M_p = source.suzuki(100, 2e6, 9000.0, 4.0, 5.0, 150.0, fc)
    z_o, M_o = oracle_mod.suzuki(100, 3, 2e6, 9000.0, 4.0, 5.0, 150.0, fc)
    assert np.array_equal(z_p, z_o) and np.array_equal(M_p, M_o)
    assert abs(M_p.sum() - 2e6) <= 1e-9 * 2e6


def test_source_placement_matches_oracle(oracle_mod):
    wl = W.small_case(30, 24, 12, 4, seed=2)
    g = wl.grid
    rng = np.random.default_rng(5)
    npts = 60
    x = rng.uniform(g.lon_c[0] - 0.1, g.lon_c[-1] + 0.1, npts)
    y = rng.uniform(g.lat_c[0] - 0.1, g.lat_c[-1] + 0.1, npts)
    z = rng.uniform(-100.0, 3500.0, npts)
    M = rng.uniform(0, 10, (4, npts))
    ijk, vals = source.place_source(g, x, y, z, M)
    dense = source.dense_source(g, ijk, vals, 4)
    orc = oracle_mod.Oracle(g, 4)
    ref = orc.place_source(g.lonmin, g.latmin, g.dlon, g.dlat, g.lon_c, g.lat_c, g.z_c, x, y, z, M)
    assert np.array_equal(dense, ref)


@pytest.mark.parametrize("var_id,ptype", [(1, 1), (2, 2), (8, 1), (13, 2), (3, 0)])
def test_perturbation_matches_oracle(oracle_mod, var_id, ptype):
    for v, r in ((5000.0, -0.7), (-3.0, 0.9), (1e6, 1.0)):
        assert source.perturbate(var_id, ptype, v, r, 20.0) == oracle_mod.perturb(var_id, ptype, v, r, 20.0)


def test_stagger_constant_fields_and_ground_zero():
    g = G.build_arakawa_c(6, 5, 4, 0.0, 0.3, 0.0, 0.25, 1000.0)
    uc = np.full((7, 6, 5), 3.0, order="F")
    vc = np.full((7, 6, 5), -2.0, order="F")
    wc = np.zeros((7, 6, 5), order="F")
    meteo.zero_ground(uc, vc, wc)
    u, v, w = meteo.stagger_velocity(uc, vc, wc)
    assert np.allclose(u[:, :, 0], 1.5) and np.allclose(u[:, :, 1:], 3.0)
    assert np.allclose(v[:, :, 1:], -2.0) and np.all(w == 0.0)


def test_capi_exports_every_declared_symbol(built_lib):
    """The shared library loads without a GPU and exports every function the
    header declares (no compute calls are made here)."""
    hdr = open(os.path.join(ROOT, "include", "fall3d_ads.h")).read()
    names = sorted(set(re.findall(r"^int\s+(f3d_\w+)\s*\(", hdr, re.M)))
    assert len(names) >= 25
    lib = C.CDLL(built_lib)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_capi_rejects_bad_arguments_without_gpu(built_lib):
    from fall3d_b200._lib import F3DDims, last_error, lib
    d = F3DDims(0, 4, 4, 2)
    h = C.c_void_p()
    assert lib().f3d_ads_create(C.byref(d), 2, 2, 0, 0, C.byref(h)) == 1
    assert "invalid dims" in last_error()
    d = F3DDims(4, 4, 4, 2)
    assert lib().f3d_ads_create(C.byref(d), 9, 2, 0, 0, C.byref(h)) == 1
    assert "limiter" in last_error()
    # the precision forms' 32-bit pencil offsets: (nx+1)(ny+1)(nz+1) < 2^31
    d = F3DDims(2000, 2000, 600, 2)
    for prec in (1, 2):
        assert lib().f3d_ads_create(C.byref(d), 2, 2, prec, 0, C.byref(h)) == 1
        assert "2^31" in last_error()


def test_partition_members_balances_load():
    costs = [16 * 1.0] * 16 + [32 * 6.0] * 32 + [16 * 27.0] * 16
    owned = [partition_members(costs, 4, r)[0] for r in range(4)]
    assert sorted(sum(owned, [])) == list(range(64))
    loads = partition_members(costs, 4, 0)[1]
    assert max(loads) / min(loads) < 1.05


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_replica_reductions_gloo_two_ranks():
    """world_size-2 gloo run of the replica plumbing: each rank takes its
    share of members, the max/sum reductions agree on both ranks."""
    port = _free_port()
    code = (
        "import os,sys; sys.path.insert(0, %r)\n"
        "import torch.distributed as dist\n"
        "from fall3d_b200.replicas import partition_members, reduce_max, reduce_sum\n"
        "dist.init_process_group('gloo', init_method='tcp://127.0.0.1:%d', rank=int(sys.argv[1]), world_size=2)\n"
        "r = dist.get_rank()\n"
        "mine, _ = partition_members([5., 3., 3., 2., 1.], 2, r)\n"
        "m = reduce_max(10.0 + r, dist); s = reduce_sum(len(mine), dist)\n"
        "assert m == 11.0 and s == 5.0, (m, s)\n"
        "print('ok', r, mine)\n"
        "dist.destroy_process_group()\n" % (ROOT, port))
    procs = [subprocess.Popen([os.environ.get("PYTHON", "python"), "-c", code, str(r)],
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
             for r in range(2)]
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e
        assert o.startswith("ok")
