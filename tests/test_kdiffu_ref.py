"""The oracle's phys_get_kdiffu (or_kdiffu) against a line-by-line Python
transcription of mod_Phys.F90:406-664 with its helpers (:1684-1741), on a
small spherical grid with terrain, for every horizontal and vertical model,
with fields chosen so that every branch is taken (z below and above the
boundary layer, stable and unstable L and Ri, the CMAQ and RAMS floors)."""
import math

import numpy as np

from fall3d_b200 import grid as G

KARMAN, GI = 0.4, 9.81


def _transcription(g, modkh, modkv, kh0, kv0, cs, uc, vc, tvc, pblh, mon, ust):
    nx, ny, nz = g.nx, g.ny, g.nz
    k1 = np.zeros((nx + 4, ny, nz))
    k2 = np.zeros((nx, ny + 4, nz))
    k3 = np.zeros((nx, ny, nz + 4))
    alfa, khf, rkhmin, landac = 0.28, 8000.0, 100.0, 30.0
    khn0 = 4000.0 if g.map_h == 0 else 0.036
    if modkh == 1:
        k1[:], k2[:] = kh0, kh0
    else:
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    dx = g.dX1_p[i + 2] * g.Hm1_p[j]
                    dy = g.dX2_p[j + 2] * g.Hm2_p[j + 2]
                    dudx = 0.5 * (uc[i + 1, j, k] - uc[i, j, k] + uc[i + 1, j + 1, k] - uc[i, j + 1, k]) / dx
                    dvdx = 0.5 * (vc[i + 1, j, k] - vc[i, j, k] + vc[i + 1, j + 1, k] - vc[i, j + 1, k]) / dx
                    dudy = 0.5 * (uc[i, j + 1, k] - uc[i, j, k] + uc[i + 1, j + 1, k] - uc[i + 1, j, k]) / dy
                    dvdy = 0.5 * (vc[i, j + 1, k] - vc[i, j, k] + vc[i + 1, j + 1, k] - vc[i + 1, j, k]) / dy
                    if modkh == 2:
                        kht = alfa * alfa * dx * dy * math.sqrt((dudx - dvdy) ** 2 + (dvdx + dudy) ** 2)
                        khn = khf * (khn0 / (g.Hm1_p[j] * g.dlon)) * (khn0 / (g.Hm2_p[j + 2] * g.dlat))
                        kv = rkhmin if (kht < 1.0 and khn < 1.0) else max(kht * khn / (kht + khn), rkhmin)
                    else:
                        kmh = 0.075 * ((dx * dy) ** (2.0 / 3.0))
                        kv = cs ** 2 * dx * dy * math.sqrt((dudy + dvdx) ** 2 + 2.0 * (dudx ** 2 + dvdy ** 2))
                        kv = max(kv, kmh, rkhmin)
                    k1[i + 2, j, k] = kv
                    k2[i, j + 2, k] = kv
        k1[0], k1[1], k1[nx + 3], k1[nx + 2] = k1[2], k1[2], k1[nx + 1], k1[nx + 1]
        k2[:, 0], k2[:, 1], k2[:, ny + 3], k2[:, ny + 2] = k2[:, 2], k2[:, 2], k2[:, ny + 1], k2[:, ny + 1]
    if modkv == 1:
        k3[:] = kv0
    else:
        zc, hc = g.z_c, g.h_c
        for j in range(ny):
            for i in range(nx):
                hp = (hc[i, j] + hc[i + 1, j] + hc[i, j + 1] + hc[i + 1, j + 1]) / 4.0
                for k in range(nz):
                    zp = (zc[i, j, k] + zc[i + 1, j, k] + zc[i, j + 1, k] + zc[i + 1, j + 1, k] + zc[i, j, k + 1] +
                          zc[i + 1, j, k + 1] + zc[i, j + 1, k + 1] + zc[i + 1, j + 1, k + 1]) / 8.0
                    z = max(0.0, zp - hp)
                    if z < pblh[i, j]:
                        zl = z / mon[i, j]
                        fih = 1.0 / math.sqrt(1.0 - 15.0 * zl) if zl < 0.0 else 1.0 + 5.0 * zl
                        kv = KARMAN * z * ust[i, j] * (1.0 - z / pblh[i, j]) * (1.0 - z / pblh[i, j]) / fih
                        kv = max(0.0, kv)
                    else:
                        lc = 1.0 / (1.0 / (KARMAN * z) + 1.0 / landac)

                        def f4(a, kk):
                            return 0.25 * (a[i, j, kk] + a[i + 1, j, kk] + a[i, j + 1, kk] + a[i + 1, j + 1, kk])
                        z1, z2 = f4(zc, k) - hp, f4(zc, k + 1) - hp
                        u1, v1, u2, v2 = f4(uc, k), f4(vc, k), f4(uc, k + 1), f4(vc, k + 1)
                        umod1, umod2 = math.sqrt(u1 * u1 + v1 * v1), math.sqrt(u2 * u2 + v2 * v2)
                        umod = 0.5 * (umod1 + umod2)
                        tv1, tv2 = f4(tvc, k), f4(tvc, k + 1)
                        um2 = max(umod * umod, 1e-18)
                        ri = GI * (z2 - z1) * (tv2 - tv1) / (um2 * 0.5 * (tv2 + tv1))
                        fc = 1.0 / (1.0 + 10.0 * ri * (1.0 + 8.0 * ri)) if ri > 0.0 else math.sqrt(1.0 - 18.0 * ri)
                        kv = max(0.0, lc * lc * abs((umod2 - umod1) / (z2 - z1)) * fc)
                    k3[i, j, k + 2] = kv
        k3[:, :, 0], k3[:, :, 1] = k3[:, :, 2], k3[:, :, 2]
        k3[:, :, nz + 3], k3[:, :, nz + 2] = k3[:, :, nz + 1], k3[:, :, nz + 1]
    return k1, k2, k3


def kdiffu_case(nx=7, ny=6, nz=8, seed=0):
    rng = np.random.default_rng(seed)
    hc = np.asfortranarray(400.0 * rng.random((nx + 1, ny + 1)))
    g = G.build_arakawa_c(nx, ny, nz, 10.0, 10.0 + 0.1 * nx, 40.0, 40.0 + 0.1 * ny, 6000.0, G.uniform_sigma(nz),
                          h_c=hc, map_v=G.MAP_V_SIGMA_LINEAR_DECAY)
    shp = (nx + 1, ny + 1, nz + 1)
    uc = [np.asfortranarray(rng.uniform(-25, 25, shp)) for _ in range(2)]
    vc = [np.asfortranarray(rng.uniform(-25, 25, shp)) for _ in range(2)]
    # virtual temperature decreasing with height, with inversions in places
    z = np.linspace(0, 1, nz + 1)[None, None, :]
    tvc = [np.asfortranarray(290.0 - 30.0 * z + rng.uniform(-4, 4, shp)) for _ in range(2)]
    pblh = np.asfortranarray(rng.uniform(200.0, 2500.0, (nx, ny)))
    mon = np.asfortranarray(rng.choice([-1.0, 1.0], (nx, ny)) * rng.uniform(10.0, 500.0, (nx, ny)))
    ust = np.asfortranarray(rng.uniform(0.05, 0.8, (nx, ny)))
    return g, uc, vc, tvc, pblh, mon, ust


def test_kdiffu_restatement(oracle_mod):
    g, uc2, vc2, tvc2, pblh, mon, ust = kdiffu_case()
    s = 0.3
    uc, vc, tvc = ((1.0 - s) * a[0] + s * a[1] for a in (uc2, vc2, tvc2))
    orc = oracle_mod.Oracle(g, 1)
    seen = set()
    for modkh in (1, 2, 4):
        for modkv in (1, 3):
            f, k1, k2, k3 = orc.kdiffu(modkh, modkv, g.map_h, 1234.0, 56.0, 0.2275, g.dlon, g.dlat,
                                       uc, vc, tvc, pblh, mon, ust)
            assert f == 0
            r1, r2, r3 = _transcription(g, modkh, modkv, 1234.0, 56.0, 0.2275, uc, vc, tvc, pblh, mon, ust)
            assert np.array_equal(k1, r1) and np.array_equal(k2, r2) and np.array_equal(k3, r3), (modkh, modkv)
            if modkh == 4:
                seen.add(("rams_floor", bool((k1[2:-2] == 100.0).any())))
            if modkv == 3:
                seen.add(("k3_pos", bool((k3 > 0).any())))
    assert ("k3_pos", True) in seen
    # unknown models and mappings are errors, as in the reference
    assert orc.kdiffu(3, 1, g.map_h, 1.0, 1.0, 0.2, g.dlon, g.dlat, uc, vc, tvc, pblh, mon, ust)[0] == 1
    assert orc.kdiffu(1, 2, g.map_h, 1.0, 1.0, 0.2, g.dlon, g.dlat, uc, vc, tvc, pblh, mon, ust)[0] == 1
    assert orc.kdiffu(1, 1, 2, 1.0, 1.0, 0.2, g.dlon, g.dlat, uc, vc, tvc, pblh, mon, ust)[0] == 1
