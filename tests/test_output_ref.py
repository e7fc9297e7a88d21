"""The vectorised restatement of the nc_IO_out_res reductions
(oracle/output_ref.py) against a direct loop transcription of the reference
routines (mod_nc_IO.F90:3400-3446, 3624-3633, 3682-3703, 3828-3858,
3909-3920; grid_p2c and grid_p2c_2D, mod_Grid.F90:1150-1220), on a small
grid with Fortran-style indices (mass points ips..ipe = 1..nx, halo -1..nx+2,
corners 1..nx+1)."""
import numpy as np

from fall3d_b200 import grid as G
from oracle import output_ref


def _loops(c, acum, awet, g, bins, col_du):
    nx, ny, nz, nb = c.shape[0] - 4, c.shape[1] - 4, c.shape[2] - 4, c.shape[3]
    C = lambda i, j, k, b: c[i + 1, j + 1, k + 1, b]          # Fortran index -> array offset
    cs = {}
    for b in range(nb):
        for k in range(-1, nz + 3):
            for j in range(-1, ny + 3):
                jj = max(1, min(j, ny))
                h1, h2 = g.Hm1_p[jj - 1], g.Hm2_p[jj + 1]
                for i in range(-1, nx + 3):
                    ii = max(1, min(i, nx))
                    v = 1e3 * C(i, j, k, b) / (h1 * h2 * g.Hm3_p[ii - 1, jj - 1])
                    cs[i, j, k, b] = max(0.0, v)

    def cc(i, j, k, b):
        return (cs[i, j, k, b] + cs[i - 1, j, k, b] + cs[i, j - 1, k, b] + cs[i - 1, j - 1, k, b] +
                cs[i, j, k - 1, b] + cs[i - 1, j, k - 1, b] + cs[i, j - 1, k - 1, b] +
                cs[i - 1, j - 1, k - 1, b]) / 8.0

    def p2c2d(m):
        h = {(i, j): m[i + 1, j + 1] for i in range(-1, nx + 3) for j in range(-1, ny + 3)}
        for j in range(-1, ny + 3):
            h[0, j] = h[1, j]
            h[nx + 1, j] = h[nx, j]
        for i in range(-1, nx + 3):
            h[i, 0] = h[i, 1]
            h[i, ny + 1] = h[i, ny]
        return lambda i, j: (h[i, j] + h[i - 1, j] + h[i, j - 1] + h[i - 1, j - 1]) / 4.0

    out = {k: np.zeros((nx + 1, ny + 1)) for k in ("con_sur", "col_mass", "cloud_top", "grn_load")}
    acs = [p2c2d(acum[:, :, b]) for b in range(nb)]
    aws = [p2c2d(awet[:, :, b]) for b in range(nb)]
    for j in range(1, ny + 2):
        for i in range(1, nx + 2):
            w = [0.0] * (nz + 1)
            for k in range(1, nz + 2):
                for b in bins:
                    w[k - 1] = w[k - 1] + cc(i, j, k, b)
            z = g.z_c[i - 1, j - 1, :]
            col = 0.0
            for k in range(nz):
                col = col + 0.5 * (w[k] + w[k + 1]) * (z[k + 1] - z[k])
            if col_du:
                col = col / 64.0 * 2.238e3
            top = 0.0
            for k in range(nz, -1, -1):
                if w[k] > 50e-6:
                    top = z[k]
                    break
            grn = 0.0
            for b in bins:
                grn = grn + (acs[b](i, j) + aws[b](i, j))
            out["con_sur"][i - 1, j - 1] = w[0]
            out["col_mass"][i - 1, j - 1] = col
            out["cloud_top"][i - 1, j - 1] = top
            out["grn_load"][i - 1, j - 1] = grn
    return out


def test_output_restatement_matches_loops():
    nx, ny, nz, nb = 7, 5, 4, 3
    rng = np.random.default_rng(0)
    g = G.build_arakawa_c(nx, ny, nz, 10.0, 10.5, 38.0, 38.4, 5000.0, G.uniform_sigma(nz),
                          h_c=np.asfortranarray(300.0 * rng.random((nx + 1, ny + 1))),
                          map_v=G.MAP_V_SIGMA_LINEAR_DECAY)
    c = np.zeros((nx + 4, ny + 4, nz + 4, nb), order="F")
    c[2:-2, 2:-2, 2:-2] = rng.lognormal(-18.0, 3.0, (nx, ny, nz, nb))
    c[2:5, 2:4] = 0.0                # a clear corner region (no cloud top)
    c[6, 5, 3, 0] = -1e-7            # a negative value is clipped
    acum = np.asfortranarray(rng.random((nx + 4, ny + 4, nb)))
    awet = np.asfortranarray(rng.random((nx + 4, ny + 4, nb)))
    for bins, du in (([0, 2], False), ([1], True), ([0, 1, 2], False)):
        ref = _loops(c, acum, awet, g, bins, du)
        got = output_ref.out_species(c, acum, awet, g, bins, col_du=du)
        for k in ref:
            assert np.array_equal(ref[k], got[k]), (bins, k)
        assert 0 < np.count_nonzero(got["cloud_top"]) < got["cloud_top"].size
