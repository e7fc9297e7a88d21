"""The oracle's gravity current (or_gc_state, or_add_radial_wind) against a
line-by-line Python transcription of F3D_add_radial_wind
(mod_F3D.F90:1006-1214) with Fortran indices, on a small spherical grid."""
import math

import numpy as np

from fall3d_b200 import workloads as W

PI = 4.0 * math.atan(1.0)
REARTH = 6356000.0


def _transcription(g, P, time, u, v):
    lon, lat, t0, t1, cfr, kent, bv, lam, mfr, htot, rmin_in = P
    if time < t0 or time > t1 or mfr <= 0.0:
        return None
    dx = REARTH * g.Hm1_c[0] * (g.lon_c[0] - g.lon_c[1]) * PI / 180.0
    dy = REARTH * (g.lat_c[0] - g.lat_c[1]) * PI / 180.0
    min_radius = 1.5 * math.sqrt(dx * dx + dy * dy)
    if rmin_in > 0.0:
        min_radius = rmin_in
    tse = time - t0
    q = cfr * math.sqrt(kent) * mfr ** 0.75 / (bv ** 1.25)
    c_gravr = 3.0 * lam * bv * q / (2.0 * PI)
    rg = max((c_gravr * tse ** 2) ** 0.33333, min_radius)
    c_gravu = math.sqrt(2.0 * lam * bv * q / (3.0 * PI))
    cgf = 0.75 * c_gravu * math.sqrt(rg)
    th = c_gravu / (math.sqrt(rg) * lam * bv)
    h_umbr = htot / 1.2
    hmin = max(h_umbr - 0.5 * th, 0.5 * htot)
    hmax = min(h_umbr + 0.5 * th, htot)
    nx, ny, nz = g.nx, g.ny, g.nz
    for j in range(1, ny + 1):              # my_jps..my_jpe
        for i in range(1, nx + 2):          # my_ibs..my_ibe
            deltax = REARTH * g.Hm1_p[j - 1] * (g.lon_c[i - 1] - lon) * PI / 180.0
            deltay = REARTH * (g.lat_p[j - 1] - lat) * PI / 180.0
            radius = math.sqrt(deltax * deltax + deltay * deltay)
            if radius > rg:
                continue
            fu = 0.0 if radius < 1e-3 else deltax / radius / g.Hm1_p[j - 1]
            radius = max(radius, min_radius)
            rvel = fu * cgf / radius * (1.0 + radius ** 2 / (3.0 * rg ** 2))
            for k in range(1, nz + 1):
                zp = g.z_c[i - 1, j - 1, k - 1]
                if hmin <= zp <= hmax:
                    u[i, j - 1, k - 1] = u[i, j - 1, k - 1] + rvel   # u(ibs-1:..) -> offset 1
    for j in range(1, ny + 2):              # my_jbs..my_jbe
        for i in range(1, nx + 1):          # my_ips..my_ipe
            deltax = REARTH * g.Hm1_c[j - 1] * (g.lon_p[i - 1] - lon) * PI / 180.0
            deltay = REARTH * (g.lat_c[j - 1] - lat) * PI / 180.0
            radius = math.sqrt(deltax * deltax + deltay * deltay)
            if radius > rg:
                continue
            fu = 0.0 if radius < 1e-3 else deltay / radius
            radius = max(radius, min_radius)
            rvel = fu * cgf / radius * (1.0 + radius ** 2 / (3.0 * rg ** 2))
            for k in range(1, nz + 1):
                zp = g.z_c[i - 1, j - 1, k - 1]
                if hmin <= zp <= hmax:
                    v[j, i - 1, k - 1] = v[j, i - 1, k - 1] + rvel
    return np.array([q, min_radius, rg, cgf, th, hmin, hmax])


def test_gravity_current_restatement(oracle_mod):
    wl = W.small_case(14, 10, 12, 2, seed=3)
    g = wl.grid
    orc = oracle_mod.Oracle(g, 2)
    for P, time in (([g.lon_c[7], g.lat_p[5], 0.0, 900.0, 430.0, 0.1, 0.02, 0.2, 1e7, 3000.0, 0.0], 700.0),
                    ([g.lon_p[3] + 0.01, g.lat_c[4], 0.0, 900.0, 430.0, 0.1, 0.02, 0.2, 3e6, 2800.0, 4000.0],
                     300.0)):
        u, v, w, _ = orc.current_winds(900.0, 0.0, 3600.0, wl.u12, wl.v12, wl.w12)
        u_t, v_t = u.copy(order="F"), v.copy(order="F")
        act, st = orc.gc_state(P, time)
        ref = _transcription(g, P, time, u_t, v_t)
        assert act and np.array_equal(st, ref)
        orc.add_radial_wind(P, st, u, v)
        assert np.array_equal(u, u_t) and np.array_equal(v, v_t)
        assert not np.array_equal(u, orc.current_winds(900.0, 0.0, 3600.0, wl.u12, wl.v12, wl.w12)[0])
    # outside the window, or without mass flow, the routine returns at once
    P = [g.lon_c[7], g.lat_p[5], 100.0, 900.0, 430.0, 0.1, 0.02, 0.2, 1e7, 3000.0, 0.0]
    assert not orc.gc_state(P, 50.0)[0] and not orc.gc_state(P, 901.0)[0]
    P[8] = 0.0
    assert not orc.gc_state(P, 500.0)[0]
