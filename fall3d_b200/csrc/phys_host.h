// phys_host.h -- host-side tables of the after-sweep processes, shared by
// the single-domain library (f3d_capi.cu) and the ensemble (ens.cu).  They
// are evaluated with the host C library, as the CPU restatement evaluates
// them, and handed to the kernels of deposit_dev.cu.
#pragma once
#include <cmath>
#include <vector>

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

}  // namespace f3d
