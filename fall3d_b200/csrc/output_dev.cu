// output_dev.cu -- the per-species reductions of nc_IO_out_res
// (mod_nc_IO.F90:3206-4335) on the device, so that an output time needs only
// 2-D fields copied to the host instead of the whole state:
//
//   cs  = max(0, 1e3 c / (Hm1 Hm2 Hm3))            g/m3 at mass points (:3400-3419)
//   cc  = 8-point mean of cs at cell corners        grid_p2c (mod_Grid.F90:1150-1181)
//   w   = sum over the species' bins of cc          (in bin order)
//   CON_SUR   = w at the ground level                (:3624-3633)
//   COL_MASS  = sum_k 0.5 (w_k + w_k+1)(z_k+1 - z_k)  g/m2 (:3682-3697), or
//               Dobson units for SO2 (/64 * 2.238e3, :3701-3703); with the
//               bins of diameter <= PM it is the PMxx column load (:3753-3777)
//   CLOUD_TOP = z_c of the highest corner with w > 50 ug/m3, else 0 (:3828-3858)
//   GRN_LOAD  = sum over the species' bins of the 4-point corner means of the
//               dry and wet deposits, grid_p2c_2D (mod_Grid.F90:1190-1220),
//               kg/m2 (:3428-3446, 3909-3920)
//
// Outside the domain the concentration is the state's halo.  Each sweep puts
// its free-flow ghost value in the first halo cell at both ends of its
// pencils (mod_ADS.F90:270,460,676, 1227-1326) and the radionuclide decay scales
// it; the library keeps those layers when asked (gh), else they read as the
// zeros of the initial condition (task_Fall3d.F90:243-248).  Halo cells
// outside in two directions are never written: 0.  The deposits take the
// nearest edge cell, as grid_p2c_2D copies the edge rows into its halo
// (mod_Grid.F90:1203-1206).  Compiled with --fmad=false: the reference's
// summation order, each operation rounded.
#include <cuda_runtime.h>

#include "f3d_common.cuh"
#include "phys_dev.cuh"

namespace f3d {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// cs = max(0, 1e3 c / (Hm1 Hm2 Hm3)) at an interior mass point
__device__ __forceinline__ double cs_interior(const OutArgs& a, int b, int i, int j, int k) {
  const long long q = (((long long)b * a.nz + k) * a.ny + j) * a.nx + i;
  const double c = a.c64 ? a.c64[q]
                         : (a.c32lo ? (double)a.c32[q] + (double)a.c32lo[q] : (double)a.c32[q]);
  const double v = 1e3 * c / (a.hm1[j] * a.hm2[j + 2] * a.hm3[i + (long long)a.nx * j]);
  return v > 0.0 ? v : 0.0;
}

// The interior cs of the selected bins, once per mass point (every value is
// read by the eight corners around it).
__global__ void k_out_cs(OutArgs a) {
  const long long ncell = (long long)a.nx * a.ny * a.nz;
  int nsel = 0;
  for (int b = 0; b < a.nb; ++b) nsel += (int)((a.mask >> b) & 1ull);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ncell * nsel;
       e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e / ncell);
    const long long q = e - (long long)s * ncell;
    int b = 0;
    for (int r = -1; b < a.nb; ++b)  // the s-th selected bin
      if (((a.mask >> b) & 1ull) && ++r == s) break;
    const int i = (int)(q % a.nx);
    const long long t = q / a.nx;
    const int j = (int)(t % a.ny), k = (int)(t / a.ny);
    a.cs[e] = cs_interior(a, b, i, j, k);
  }
}

// cs at mass point (i, j, k) of bin b (its index s among the selected bins),
// i in [-1, nx] and likewise j, k
__device__ __forceinline__ double cs_at(const OutArgs& a, int b, int s, int i, int j, int k) {
  const bool ox = i < 0 || i >= a.nx, oy = j < 0 || j >= a.ny, oz = k < 0 || k >= a.nz;
  double c;
  if (!ox && !oy && !oz) {
    return a.cs[(((long long)s * a.nz + k) * a.ny + j) * a.nx + i];
  } else {
    if ((int)ox + (int)oy + (int)oz > 1 || (!a.gh64 && !a.gh32)) return 0.0;
    long long g;
    if (ox) g = gh_offset(0, i < 0 ? 0 : 1, (long long)k * a.ny + j, a.nx, a.ny, a.nz);
    else if (oy) g = gh_offset(1, j < 0 ? 0 : 1, (long long)k * a.nx + i, a.nx, a.ny, a.nz);
    else g = gh_offset(2, k < 0 ? 0 : 1, (long long)j * a.nx + i, a.nx, a.ny, a.nz);
    g += (long long)b * gh_per_bin(a.nx, a.ny, a.nz);
    c = a.gh64 ? a.gh64[g] : (double)a.gh32[g];
    i = clampi(i, 0, a.nx - 1);  // the metric factors at the clamped index (:3404-3408)
    j = clampi(j, 0, a.ny - 1);
  }
  const double v = 1e3 * c / (a.hm1[j] * a.hm2[j + 2] * a.hm3[i + (long long)a.nx * j]);
  return v > 0.0 ? v : 0.0;
}

__device__ __forceinline__ double g_at(const double* f, const OutArgs& a, int b, int i, int j) {
  i = clampi(i, 0, a.nx - 1);
  j = clampi(j, 0, a.ny - 1);
  return f[((long long)b * a.ny + j) * a.nx + i];
}

__global__ void k_out_columns(OutArgs a) {
  const long long ncol = (long long)(a.nx + 1) * (a.ny + 1);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ncol;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % (a.nx + 1)), j = (int)(e / (a.nx + 1));
    if (a.con_sur || a.col_mass || a.cloud_top) {
      // species sum at every corner level, bins in order (the reference adds
      // whole bins: my_work3d = my_work3d + my_cc(:,:,:,ib)); per bin the
      // levels slide a window, so that level k-1's four mass points are
      // reused from level k's step before
      double* w = a.wbuf + e;
      for (int k = 0; k <= a.nz; ++k) w[ncol * k] = 0.0;
      int s = 0;
      for (int b = 0; b < a.nb; ++b) {
        if (!((a.mask >> b) & 1ull)) continue;
        double p0 = cs_at(a, b, s, i, j, -1), p1 = cs_at(a, b, s, i - 1, j, -1);
        double p2 = cs_at(a, b, s, i, j - 1, -1), p3 = cs_at(a, b, s, i - 1, j - 1, -1);
        for (int k = 0; k <= a.nz; ++k) {
          const double q0 = cs_at(a, b, s, i, j, k), q1 = cs_at(a, b, s, i - 1, j, k);
          const double q2 = cs_at(a, b, s, i, j - 1, k), q3 = cs_at(a, b, s, i - 1, j - 1, k);
          const double cc = (q0 + q1 + q2 + q3 + p0 + p1 + p2 + p3) / 8.0;
          w[ncol * k] = w[ncol * k] + cc;
          p0 = q0;
          p1 = q1;
          p2 = q2;
          p3 = q3;
        }
        ++s;
      }
      double wk = w[0];
      if (a.con_sur) a.con_sur[e] = wk;
      double col = 0.0, top = 0.0;
      if (wk > 50e-6) top = a.zc[e];
      for (int k = 0; k < a.nz; ++k) {
        const double wk1 = w[ncol * (k + 1)];
        const double dz = a.zc[e + ncol * (k + 1)] - a.zc[e + ncol * k];
        col = col + 0.5 * (wk + wk1) * dz;
        if (wk1 > 50e-6) top = a.zc[e + ncol * (k + 1)];
        wk = wk1;
      }
      if (a.col_du) col = col / 64.0 * 2.238e3;
      if (a.col_mass) a.col_mass[e] = col;
      if (a.cloud_top) a.cloud_top[e] = top;
    }
    if (a.grn_load) {
      double g = 0.0;
      for (int b = 0; b < a.nb; ++b) {
        if (!((a.mask >> b) & 1ull)) continue;
        double ac = (g_at(a.acum, a, b, i, j) + g_at(a.acum, a, b, i - 1, j) + g_at(a.acum, a, b, i, j - 1) +
                     g_at(a.acum, a, b, i - 1, j - 1)) /
                    4.0;
        if (a.awet) {
          const double aw = (g_at(a.awet, a, b, i, j) + g_at(a.awet, a, b, i - 1, j) +
                             g_at(a.awet, a, b, i, j - 1) + g_at(a.awet, a, b, i - 1, j - 1)) /
                            4.0;
          ac = ac + aw;
        } else {
          ac = ac + 0.0;
        }
        g = g + ac;
      }
      a.grn_load[e] = g;
    }
  }
}

void launch_out_columns(const OutArgs& a, cudaStream_t st) {
  if (a.con_sur || a.col_mass || a.cloud_top) k_out_cs<<<1184, 256, 0, st>>>(a);
  k_out_columns<<<592, 128, 0, st>>>(a);
}

}  // namespace f3d
