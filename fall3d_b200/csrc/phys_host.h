// phys_host.h -- host-side tables of the after-sweep processes, shared by
// the single-domain library (f3d_capi.cu) and the ensemble (ens.cu).  They
// are evaluated with the host C library, as the CPU restatement evaluates
// them, and handed to the kernels of deposit_dev.cu.
#pragma once
#include <cmath>
#include <cstring>
#include <vector>

#include "phys_dev.cuh"

namespace f3d {

// Wet deposition inputs per column (phys_wet_deposition, mod_Phys.F90:1358-1427):
// P^b, and the number ktop of cells below the boundary-layer top, ho + zp <= pblh
// with ho the terrain and zp the mid height of the cell at the mass point
// (:1404-1414).  Heights grow with k, so those are the first ktop levels.
// Returns false when they do not (the below-PBL cells would not be a prefix).
inline bool wet_tables(int nx, int ny, int nz, double b, const double* pre, const double* pblh,
                       const double* h_c, const double* z_c, std::vector<double>& powpb,
                       std::vector<int>& ktop) {
  const size_t ncol = (size_t)nx * ny;
  powpb.assign(ncol, 0.0);
  ktop.assign(ncol, 0);
  auto HC = [&](int i, int j) { return h_c[i + (size_t)(nx + 1) * j]; };
  auto ZC = [&](int i, int j, int k) { return z_c[i + (size_t)(nx + 1) * (j + (size_t)(ny + 1) * k)]; };
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const size_t ij = i + (size_t)nx * j;
      powpb[ij] = std::pow(pre[ij], b);
      const double ho = 0.25 * (HC(i, j) + HC(i + 1, j) + HC(i, j + 1) + HC(i + 1, j + 1));
      int kt = 0;
      for (int k = 0; k < nz; ++k) {
        const double zp1 = 0.25 * (ZC(i, j, k) + ZC(i + 1, j, k) + ZC(i, j + 1, k) + ZC(i + 1, j + 1, k));
        const double zp2 =
            0.25 * (ZC(i, j, k + 1) + ZC(i + 1, j, k + 1) + ZC(i, j + 1, k + 1) + ZC(i + 1, j + 1, k + 1));
        const double zp = 0.5 * (zp1 + zp2);
        const bool below = ho + zp <= pblh[ij];
        if (below && kt != k) return false;
        if (below) kt = k + 1;
      }
      ktop[ij] = kt;
    }
  return true;
}

// Bins that take wet deposition: particles and radionuclides of diameter
// <= 100 um (mod_F3D.F90:1499-1506).
inline unsigned long long wet_bin_mask(int nb, const int* bin_cat, const double* bin_diam) {
  unsigned long long mask = 0;
  for (int q = 0; q < nb; ++q)
    if ((bin_cat[q] == 1 || bin_cat[q] == 3) && bin_diam[q] <= 1e-4) mask |= 1ull << q;
  return mask;
}

// Radionuclide bins in bin order with their decay constants and, for Y90,
// the Sr90 parent bin (phys_radionuclides, mod_Phys.F90:1216-1299).
struct RadioSpec {
  std::vector<int> bin, parent;
  std::vector<double> kn, pkn;
};

// 0 ok; 1 unequal numbers of Sr90 and Y90 bins; 2 an invalid species
// (*bad_species is set).
inline int radio_spec(int nb, const int* bin_cat, const int* bin_spe, RadioSpec& r, int* bad_species) {
  r = RadioSpec();
  auto rate = [](int spe) {  // mod_Phys.F90:79-83
    switch (spe) {
      case 5: return 1.06e-8;
      case 6: return 9.29e-10;
      case 7: return 1.00e-6;
      case 8: return 7.63e-10;
      case 9: return 2.98e-6;
    }
    return -1.0;
  };
  int ny90 = 0, nsr90 = 0, shift = 0;
  for (int q = 0; q < nb; ++q) {
    if (bin_cat[q] == 3 && bin_spe[q] == 9 && ++ny90 == 1) shift -= q;
    if (bin_cat[q] == 3 && bin_spe[q] == 8 && ++nsr90 == 1) shift += q;
  }
  if (ny90 != nsr90) return 1;
  for (int q = 0; q < nb; ++q) {
    if (bin_cat[q] != 3) continue;
    const double kn = rate(bin_spe[q]);
    if (kn < 0.0) {
      if (bad_species) *bad_species = bin_spe[q];
      return 2;
    }
    const int par = (bin_spe[q] == 9) ? q + shift : -1;
    r.bin.push_back(q);
    r.parent.push_back(par);
    r.kn.push_back(kn);
    r.pkn.push_back(par >= 0 ? rate(bin_spe[par]) : 0.0);
  }
  return 0;
}

// grid_get_mass_sink's serial sum (mod_Grid.F90:1426-1447) over the column
// terms, j outer, i inner, then gl_mass = 0 + the (single) rank's sum.
inline double mass_sink_sum(int nx, int ny, const double* col) {
  double my_mass = 0.0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) my_mass = my_mass + col[i + (size_t)nx * j];
  return 0.0 + my_mass;
}

// Scalars of the gravity current, F3D_add_radial_wind (mod_F3D.F90:978-1226),
// at `time`, with the host C library's sqrt and pow (:1026-1070).  p holds
// {lon, lat, start_time, end_time, c_flow_rate, k_entrain, brunt_vaisala,
// lambda_grav, mass_flow_rate, h_tot, input_min_radius}; lon_c, lat_c and
// hm1_c are the first two corner coordinates and scale factor of the grid.
// Returns false where the routine returns early (outside [start_time,
// end_time] or no mass flow).  st = {vol_flow_rate, min_radius,
// radius_grav, c_grav_factor, th_grav, hmin, hmax}; g receives the scalars
// (the caller sets its device pointers).
inline bool gc_scalars(const double p[11], const double* lon_c, const double* lat_c,
                       const double* hm1_c, double time, GcArgs* g, double st[7]) {
  const double PI = 4.0 * std::atan(1.0), REARTH = 6356000.0;  // mod_KindType.F90:43-44
  std::memset(g, 0, sizeof(*g));
  for (int q = 0; q < 7; ++q) st[q] = 0.0;
  if (time < p[2] || time > p[3] || p[8] <= 0.0) return false;
  double deltax = REARTH * hm1_c[0] * (lon_c[0] - lon_c[1]) * PI / 180.0;
  double deltay = REARTH * (lat_c[0] - lat_c[1]) * PI / 180.0;
  double radius = 1.5 * std::sqrt(deltax * deltax + deltay * deltay);
  double min_radius = radius;  // parallel_max over one rank
  if (p[10] > 0.0) min_radius = p[10];
  const double c_flow_rate = p[4], k_entrain = p[5], brunt_vaisala = p[6], lambda_grav = p[7],
               mass_flow_rate = p[8], h_tot = p[9];
  const double tse = time - p[2];
  const double vol_flow_rate = c_flow_rate * std::sqrt(k_entrain) * std::pow(mass_flow_rate, 0.75) /
                               std::pow(brunt_vaisala, 1.25);
  const double c_gravr = 3.0 * lambda_grav * brunt_vaisala * vol_flow_rate / (2.0 * PI);
  double radius_grav = std::pow(c_gravr * (tse * tse), 0.33333);
  radius_grav = std::fmax(radius_grav, min_radius);
  const double c_gravu = std::sqrt(2.0 * lambda_grav * brunt_vaisala * vol_flow_rate / (3.0 * PI));
  const double c_grav_factor = 0.75 * c_gravu * std::sqrt(radius_grav);
  const double th_grav = c_gravu / (std::sqrt(radius_grav) * lambda_grav * brunt_vaisala);
  const double h_umbr = h_tot / 1.2;
  const double hmin = std::fmax(h_umbr - 0.5 * th_grav, 0.5 * h_tot);
  const double hmax = std::fmin(h_umbr + 0.5 * th_grav, h_tot);
  g->on = 1;
  g->xc = p[0];
  g->yc = p[1];
  g->rearth = REARTH;
  g->pi = PI;
  g->min_radius = min_radius;
  g->radius_grav = radius_grav;
  g->c_grav_factor = c_grav_factor;
  g->hmin = hmin;
  g->hmax = hmax;
  st[0] = vol_flow_rate;
  st[1] = min_radius;
  st[2] = radius_grav;
  st[3] = c_grav_factor;
  st[4] = th_grav;
  st[5] = hmin;
  st[6] = hmax;
  return true;
}

// Boundary halo layers <-> the reference's halo-inclusive state arrays
// my_c(ips-2:ipe+2, jps-2:jpe+2, kps-2:kpe+2, nbins): the first halo cell at
// both ends of every pencil (both halo layers hold it after a sweep,
// mod_ADS.F90:1246,1258,...), in the gh_offset layout (f3d_common.cuh).
inline void gh_gather_ref(int nx_, int ny_, int nz_, int nb_, const double* my_c,
                          std::vector<double>& g) {
  const long long nx = nx_, ny = ny_, nz = nz_, nb = nb_;
  const long long X = nx + 4, Y = ny + 4, Z = nz + 4, per = gh_per_bin(nx_, ny_, nz_);
  g.assign((size_t)(per * nb), 0.0);
  auto at = [&](long long i, long long j, long long k, long long b) {
    return my_c[(i + 2) + X * ((j + 2) + Y * ((k + 2) + Z * b))];
  };
  for (long long b = 0; b < nb; ++b) {
    double* gb = g.data() + b * per;
    for (long long k = 0; k < nz; ++k)
      for (long long j = 0; j < ny; ++j) {
        gb[gh_offset(0, 0, k * ny + j, nx_, ny_, nz_)] = at(-1, j, k, b);
        gb[gh_offset(0, 1, k * ny + j, nx_, ny_, nz_)] = at(nx, j, k, b);
      }
    for (long long k = 0; k < nz; ++k)
      for (long long i = 0; i < nx; ++i) {
        gb[gh_offset(1, 0, k * nx + i, nx_, ny_, nz_)] = at(i, -1, k, b);
        gb[gh_offset(1, 1, k * nx + i, nx_, ny_, nz_)] = at(i, ny, k, b);
      }
    for (long long j = 0; j < ny; ++j)
      for (long long i = 0; i < nx; ++i) {
        gb[gh_offset(2, 0, j * nx + i, nx_, ny_, nz_)] = at(i, j, -1, b);
        gb[gh_offset(2, 1, j * nx + i, nx_, ny_, nz_)] = at(i, j, nz, b);
      }
  }
}

inline void gh_scatter_ref(int nx_, int ny_, int nz_, int nb_, const std::vector<double>& g,
                           double* my_c) {
  const long long nx = nx_, ny = ny_, nz = nz_, nb = nb_;
  const long long X = nx + 4, Y = ny + 4, Z = nz + 4, per = gh_per_bin(nx_, ny_, nz_);
  auto at = [&](long long i, long long j, long long k, long long b) -> double& {
    return my_c[(i + 2) + X * ((j + 2) + Y * ((k + 2) + Z * b))];
  };
  for (long long b = 0; b < nb; ++b) {
    const double* gb = g.data() + b * per;
    for (long long k = 0; k < nz; ++k)
      for (long long j = 0; j < ny; ++j) {
        at(-1, j, k, b) = at(-2, j, k, b) = gb[gh_offset(0, 0, k * ny + j, nx_, ny_, nz_)];
        at(nx, j, k, b) = at(nx + 1, j, k, b) = gb[gh_offset(0, 1, k * ny + j, nx_, ny_, nz_)];
      }
    for (long long k = 0; k < nz; ++k)
      for (long long i = 0; i < nx; ++i) {
        at(i, -1, k, b) = at(i, -2, k, b) = gb[gh_offset(1, 0, k * nx + i, nx_, ny_, nz_)];
        at(i, ny, k, b) = at(i, ny + 1, k, b) = gb[gh_offset(1, 1, k * nx + i, nx_, ny_, nz_)];
      }
    for (long long j = 0; j < ny; ++j)
      for (long long i = 0; i < nx; ++i) {
        at(i, j, -1, b) = at(i, j, -2, b) = gb[gh_offset(2, 0, j * nx + i, nx_, ny_, nz_)];
        at(i, j, nz, b) = at(i, j, nz + 1, b) = gb[gh_offset(2, 1, j * nx + i, nx_, ny_, nz_)];
      }
  }
}

}  // namespace f3d
