// phys_dev.cuh -- argument blocks of the after-sweep processes and the
// output reductions, shared by their kernels (deposit_dev.cu, output_dev.cu)
// and the host library (f3d_capi.cu).
#pragma once
#include <cuda_runtime.h>

namespace f3d {

// wet deposition, phys_wet_deposition (mod_Phys.F90:1358-1427)
struct WetArgs {
  int nx, ny, nz, nb;
  double dta;              // dt * a
  const double* powpb;     // P^b per column, nx*ny
  const int* ktop;         // cells k < ktop of the column are below the PBL top
  const double* dx3p;      // dX3_p with the reference offset (kps-2)
  double* awet;            // [bin][j][i]
  double* c64;             // exact form state (or null)
  float* c32;              // precision form state (or null)
  unsigned long long mask; // bins that take wet deposition
};

// radioactive decay, phys_radionuclides (mod_Phys.F90:1216-1342)
struct RadioArgs {
  int nx, ny, nz, nr;       // nr radionuclide bins, in bin order
  int bin[64];              // their bin indices
  int parent[64];           // Y90: bin index of the Sr90 parent, else -1
  double fact[64];          // exp(-kn dt) of the bin
  double pfact[64];         // exp(-kn dt) of the parent
  double* c64;
  float* c32;
  double* acum;             // [bin][j][i]
  double* awet;             // [bin][j][i] or null
  double* gh64;             // boundary halo layers (or null): the reference
  float* gh32;              // decays the halo cells of the state as well
  long long ngh;            // halo layer elements per bin
};

// per-species output reductions of nc_IO_out_res (mod_nc_IO.F90:3206-4335)
struct OutArgs {
  int nx, ny, nz, nb;
  unsigned long long mask;  // bins of the species
  int col_du;               // column load in Dobson units (SO2)
  const double* c64;        // state [bin][k][j][i] (one of c64, c32)
  const float* c32;
  const double* acum;       // [bin][j][i]
  const double* awet;       // [bin][j][i] or null
  const double* hm1;        // ny
  const double* hm2;        // ny+4 (jps-2..)
  const double* hm3;        // nx*ny
  const double* zc;         // corner heights (nx+1)(ny+1)(nz+1)
  const double* gh64;       // boundary halo layers, gh_offset layout, or null
  const float* gh32;
  double* con_sur;          // (nx+1)(ny+1) each, or null
  double* col_mass;
  double* cloud_top;
  double* grn_load;
};

void launch_wet(const WetArgs& a, cudaStream_t st);
void launch_radio(const RadioArgs& a, cudaStream_t st);
void launch_out_columns(const OutArgs& a, cudaStream_t st);

}  // namespace f3d
