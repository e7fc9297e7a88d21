// phys_dev.cuh -- argument blocks of the after-sweep processes and the
// output reductions, shared by their kernels (deposit_dev.cu, output_dev.cu)
// and the host library (f3d_capi.cu).
#pragma once
#include <cuda_runtime.h>

#include "f3d_common.cuh"

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
  float* c32lo;            // its low part (compensated precision form), or null
  unsigned long long mask; // bins that take wet deposition
  const double* dt_dev;    // ensemble: the member's device time step (dta = dt * a), or null
  double a;
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
  float* c32lo;             // low part of c32 (compensated precision form), or null
  double* acum;             // [bin][j][i]
  double* awet;             // [bin][j][i] or null
  double* gh64;             // boundary halo layers (or null): the reference
  float* gh32;              // decays the halo cells of the state as well
  long long ngh;            // halo layer elements per bin
  const double* fdev;       // ensemble: the member's {fact[nr], pfact[nr]} in device memory, or null
  int tail;                 // after the z sweep's epilogue: only the daughters' cells and
                            // deposits (set from the parent), and every bin's halo layers
};

// per-species output reductions of nc_IO_out_res (mod_nc_IO.F90:3206-4335)
struct OutArgs {
  int nx, ny, nz, nb;
  unsigned long long mask;  // bins of the species
  int col_du;               // column load in Dobson units (SO2)
  const double* c64;        // state [bin][k][j][i] (one of c64, c32)
  const float* c32;
  const float* c32lo;       // low part of c32 (compensated precision form), or null
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
  double* cs;               // scratch: cs of the selected bins at the interior mass points,
                            // [selected bin][k][j][i], formed once per call
  double* wbuf;             // scratch: species sum at the corners, [k][corner column]
};

// gravity current, F3D_add_radial_wind (mod_F3D.F90:978-1226): the radial
// wind of one time, added to the current winds in the layer [hmin, hmax]
// within radius_grav of the centre (xc, yc).  The scalars are evaluated on
// the host for the step's time.
struct GcArgs {
  int on;
  double xc, yc;
  double rearth, pi;  // REARTH, PI (mod_KindType.F90:43-44)
  double min_radius, radius_grav, c_grav_factor, hmin, hmax;
  const double* lon_c;  // ibs:ibe
  const double* lat_c;  // jbs:jbe
  const double* lon_p;  // ips:ipe
  const double* lat_p;  // jps:jpe
  const double* hm1_p;  // jps:jpe
  const double* hm1_c;  // jbs:jbe
  const double* zc;     // corner heights (nx+1)(ny+1)(nz+1)
};

// rvel of the radial wind at a face of the given offsets (mod_F3D.F90:1148-1164
// for x faces, :1186-1202 for y faces); false where the routine skips it.
// Written operation by operation as the reference evaluates it (compile the
// caller with --fmad=false).
__device__ __forceinline__ bool gc_rvel(const GcArgs& g, double hm1, double dlon, double dlat,
                                        bool xface, double* rvel) {
  const double deltax = g.rearth * hm1 * dlon * g.pi / 180.0;
  const double deltay = g.rearth * dlat * g.pi / 180.0;
  double radius = sqrt(deltax * deltax + deltay * deltay);
  if (radius > g.radius_grav) return false;
  double fu;
  if (radius < 1e-3) fu = 0.0;
  else fu = xface ? deltax / radius / hm1 : deltay / radius;
  radius = fmax(radius, g.min_radius);
  *rvel = fu * g.c_grav_factor / radius *
          (1.0 + radius * radius / (3.0 * (g.radius_grav * g.radius_grav)));
  return true;
}

// x face i (0..nx) of mass row j, level k
__device__ __forceinline__ bool gc_rvel_u(const GcArgs& g, int nx, int ny, int i, int j, int k,
                                          double* rvel) {
  const double zp = g.zc[i + (long long)(nx + 1) * (j + (long long)(ny + 1) * k)];
  if (!(zp >= g.hmin && zp <= g.hmax)) return false;
  return gc_rvel(g, g.hm1_p[j], g.lon_c[i] - g.xc, g.lat_p[j] - g.yc, true, rvel);
}

// y face j (0..ny) of mass column i, level k
__device__ __forceinline__ bool gc_rvel_v(const GcArgs& g, int nx, int ny, int i, int j, int k,
                                          double* rvel) {
  const double zp = g.zc[i + (long long)(nx + 1) * (j + (long long)(ny + 1) * k)];
  if (!(zp >= g.hmin && zp <= g.hmax)) return false;
  return gc_rvel(g, g.hm1_c[j], g.lon_p[i] - g.xc, g.lat_c[j] - g.yc, false, rvel);
}

// diffusion coefficients, phys_get_kdiffu (mod_Phys.F90:406-664): from the
// corner fields of the two meteo snapshots at interpolation factor s, into the
// reference layouts k1(ips-2:ipe+2, jps:jpe, kps:kpe), k2(ips:ipe,
// jps-2:jpe+2, kps:kpe), k3(ips:ipe, jps:jpe, kps-2:kpe+2), unscaled
struct KdArgs {
  int nx, ny, nz, modkh, modkv;  // MOD_CONSTANT 1, CMAQ 2, SIMILARITY 3, RAMS 4
  double kh0, kv0, rams_cs, khn0, dlon, dlat, s;
  const double* uc0;  // corner fields (nx+1)(ny+1)(nz+1), snapshots its and ite
  const double* uc1;
  const double* vc0;
  const double* vc1;
  const double* tvc0;
  const double* tvc1;
  const double* dx1p;  // (nx+4)
  const double* dx2p;  // (ny+4)
  const double* hm1;   // ny
  const double* hm2;   // ny+4
  const double* kmh;   // RAMS: 0.075 (dx dy)^(2/3) per column, nx*ny (host libm)
  const double* pblh;  // nx*ny
  const double* mon;
  const double* ust;
  const double* zc;    // corner heights
  const double* hc;    // (nx+1)(ny+1) terrain at corners
  double* k1;
  double* k2;
  double* k3;
};
void launch_kdiffu(const KdArgs& a, cudaStream_t st);

void launch_wet(const WetArgs& a, cudaStream_t st);
void launch_sink_cols(int nx, int ny, int nb, const double* awet, const double* dx1p,
                      const double* dx2p, double* col, cudaStream_t st);
void launch_radio(const RadioArgs& a, cudaStream_t st);
void launch_out_columns(const OutArgs& a, cudaStream_t st);
// current winds of the step with the radial wind (meteo_dev.cu)
void launch_gc_winds(MemberDev* members, int mi, int nx, int ny, int nz, int fp32, const GcArgs& g,
                     cudaStream_t st);

}  // namespace f3d
