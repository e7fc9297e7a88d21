// f3d_common.cuh -- device-side data layout shared by all FALL3D ADS kernels.
//
// One "member" is one model domain (a serial FALL3D run, or one ensemble
// member).  Every kernel takes a table of members plus a work list, so the
// single-domain drop-in and the batched ensemble run the same code.
//
// HBM layout of a member (interior cells only; ghost cells are rebuilt by
// the free-flow boundary condition inside each sweep, exactly where the
// reference writes them before reading them, mod_ADS.F90:269-271):
//   c     [bin][k][j][i]                     concentration (FP64 or FP32)
//   acum  [bin][j][i]                        ground deposit, FP64 always
//   ux    [snap][k][f=0..nx][j]              x-face wind, j fastest so a warp
//                                            of x-pencils reads it coalesced
//   vy    [snap][k][f=0..ny][i]              y-face wind
//   wz    [snap][f=0..nz][j][i]              z-face wind
//   k1x   [k][p=-1..nx][j]   k2y [k][p=-1..ny][i]   k3z [p=-1..nz][j][i]
//   vs    [bin][f=0..nz][j][i]               settling velocity (scaled)
// Pencils: x-pencil (j,k,bin) lanes over j; y-pencil (i,k,bin) and
// z-pencil (i,j,bin) lanes over i, so y/z loads are fully coalesced.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

namespace f3d {

constexpr double kEps = 1e-12;  // EPSILON, mod_KindType.F90:42

// The precision form's sweeps address a member's cells and faces within one
// bin by 32-bit element offsets: (nx+1)(ny+1)(nz+1) must stay below this.
constexpr long long kMaxPencilSpan = 1LL << 31;
__host__ __device__ inline bool pencil_span_ok(long long nx, long long ny, long long nz) {
  return (nx + 1) * (ny + 1) * (nz + 1) < kMaxPencilSpan;
}

enum Dir { DIR_X = 0, DIR_Y = 1, DIR_Z = 2 };

struct MemberDev {
  int nx, ny, nz, nb;
  // state
  double* c64;
  float* c32;
  double* acum;
  // meteo snapshots (FP64 copies, used by the exact path and the CFL)
  const double* ux[2];
  const double* vy[2];
  const double* wz[2];
  const double* k1x;
  const double* k2y;
  const double* k3z;
  const double* vs;
  // FP64 face data of the exact form, per direction (0 x, 1 y, 2 z):
  //   geo[d][p+1] = {dxp(p), 1/dxp(p), dxb(p), 1/dxb(p)} for p = -1..n-1
  //   kkf[d] = 0.5 (k(f) + k(f-1)) at every face, laid out like the winds
  const double4* geo[3];
  const double* kkf[3];
  // FP32 face data of the precision form (null when unused), one float4 per
  // face and direction, laid out like the winds (x [k][f][j], y [k][f][i],
  // z [f][j][i]): {velocity at its, velocity at ite, 0.5 (k(f) + k(f-1)) /
  // dxp(f-1), 1/dxb(f-1) (0 at f = 0)}, so that a sweep reads a face with a
  // single 16-byte load
  const float4* f4[3];
  const float* vs32;  // [bin][f][j][i]
  // per-step current winds (written by the prep kernel)
  double* ucur;  // [k][f][j]
  double* vcur;  // [k][f][i]
  double* wcur;  // [f][j][i]
  float4* gc4[2];  // precision form with the gravity current: x and y face
                   // data with this step's winds in both velocity slots
  float wfac;       // per-member multiplicative factor on u,v (ensemble), FP32 form
  double wfacd;     // the same factor for the FP64 form and the CFL reduction
  // grid metrics (reference arrays with their halos)
  const double* dx1p;  // (nx+4)   ips-2..ipe+2
  const double* dx1b;  // (nx+3)   ibs-1..ibe+1
  const double* dx2p;
  const double* dx2b;
  const double* dx3p;
  const double* dx3b;
  const double* hm1;  // ny
  const double* hm2;  // ny+4
  const double* hm3;  // nx*ny
  const float* rdx1b32;  // 1/dx_b per axis, FP32 form
  const float* rdx2b32;
  const float* rdx3b32;
  // sparse source: cell index (i + nx*(j + ny*k)), my_s values per bin,
  // cell volume dX dY dZ Hm1 Hm2 Hm3
  int nsrc;
  const int* src_cell;
  const double* src_s;  // [q][bin]
  const double* src_vol;
  // step parameters (device resident so a step can run inside a graph)
  double dt;
  double stime;
  double time;
  double t_its, t_ite;
  int iiter;
  int gc_cur;  // precision form: the x and y sweeps read gc4 (this step's
               // winds with the gravity current) instead of f4
  // flux bookkeeping
  double* flux_part;  // per-block partial sums, [slot][2]
  int part_base[3];   // first partial slot of this member for x, y, z
  int part_count[3];  // number of partial slots (blocks) per direction
  double* flux_tot;   // running totals {W,E,S,N,U,D} and compensations [12]
  double* flux_step;  // this step's increments {W,E,S,N,U,D}
  // boundary halo layers (null unless kept): the free-flow ghost value each
  // sweep puts in the first halo cell at both ends of its pencils, laid out
  // per bin as gh_offset() gives (exact form gh64, precision form gh32)
  double* gh64;
  float* gh32;
  // compensated precision form (null otherwise): the low part of the state,
  // laid out like c32, so that the concentration is c32 + c32lo (about 48
  // bits), and 1/dxb per axis in FP64 ([cell], n entries) for the
  // conservative final update of the sweeps
  float* c32lo;
  const double* rdxb64[3];
  const float2* rdxb2[3];  // the same 1/dxb as an FP32 pair {hi, lo} (~48 bits)
  // Wet deposition and radioactive decay as the z sweep's epilogue
  // (mod_F3D.F90:1493-1520; z is the last sweep of a step): as each cell's
  // final value leaves the march it is scavenged (bins of wet_mask, cells
  // below the column's ktop) and decayed (radionuclide bins), and the
  // column's wet and dry deposits are updated by the thread that owns them.
  // epi_on = 0 leaves both processes to the separate kernels.
  int epi_on;
  unsigned long long wet_mask;       // bins that take wet deposition (0: none)
  double wet_a;                      // lambda = min(1, dt wet_a P^b)
  const double* powpb;               // P^b per column [j][i]
  const int* ktop;                   // cells k < ktop of the column are below the PBL top
  double* awet;                      // wet deposit [bin][j][i] (null without wet deposition)
  const double* radf;                // this step's {exp(-kn dt)[nr], parent's [nr]}, or null
  signed char rad_r[64];             // radionuclide index of each bin, -1 for none
  unsigned long long daughter_mask;  // bins set from their parent after the sweep (Y90)
};

// Host: whether steps run wet deposition and decay as the z sweep's
// epilogue (f3d_set_zsweep_epilogue; on by default).
int zsweep_epilogue();

// The epilogue's per-cell arithmetic, in the order of the separate kernels
// (phys_wet_deposition, then phys_radionuclides): a cell below the PBL top
// adds (dX3_p lambda) c to the column's wet deposit and keeps (1 - lambda) c;
// a radionuclide bin then takes c f.  Every operation is explicitly rounded
// (no contraction), so the fused and the separate paths agree bit for bit.
struct ZEpi {
  double lam;          // wet: min(1, dt a P^b) of the column
  int kt;              // wet: cells below the PBL top (0: no wet deposition)
  const double* dx3p;  // dX3_p with the reference offset (kps-2)
  double aw;           // wet deposit of the column, accumulated in k order
  double f;            // decay factor of the bin
  bool dec;            // the bin decays in the epilogue
  __device__ __forceinline__ double apply(int k, double c) {
    if (k < kt) {
      aw = __dadd_rn(aw, __dmul_rn(__dmul_rn(dx3p[k + 2], lam), c));
      c = __dmul_rn(c, __dsub_rn(1.0, lam));
    }
    return dec ? __dmul_rn(c, f) : c;
  }
  // the FP32 state: each process rounds its result to FP32, as the separate
  // kernels store it
  __device__ __forceinline__ float apply32(int k, float v) {
    if (k < kt) {
      const double c = (double)v;
      aw = __dadd_rn(aw, __dmul_rn(__dmul_rn(dx3p[k + 2], lam), c));
      v = __double2float_rn(__dmul_rn(c, __dsub_rn(1.0, lam)));
    }
    return dec ? __double2float_rn(__dmul_rn((double)v, f)) : v;
  }
};

struct NoEpi {};

// Epilogue parameters of bin b of member m for the column at ij (z sweep).
// A daughter bin (Y90) is overwritten from its parent after the sweep, so its
// epilogue does nothing.
__device__ __forceinline__ ZEpi zepi_setup(const MemberDev& m, int b, long long ij) {
  ZEpi e;
  e.lam = 0.0;
  e.kt = 0;
  e.dx3p = m.dx3p;
  e.aw = 0.0;
  e.f = 1.0;
  e.dec = false;
  const bool daughter = (m.daughter_mask >> b) & 1ull;
  if (((m.wet_mask >> b) & 1ull) && !daughter) {
    const double lam = __dmul_rn(__dmul_rn(m.dt, m.wet_a), m.powpb[ij]);
    e.lam = lam > 1.0 ? 1.0 : lam;
    e.kt = m.ktop[ij];
    e.aw = m.awet[(long long)b * m.nx * m.ny + ij];  // the sum starts from the deposit
  }
  const int r = m.rad_r[b];
  if (m.radf && r >= 0 && !daughter) {
    e.f = m.radf[r];
    e.dec = true;
  }
  return e;
}

// The column's deposits after the march: the wet deposit takes the
// scavenged sum, then both deposits decay with the bin (the dry deposit has
// already taken this step's flux).
__device__ __forceinline__ void zepi_finish(const MemberDev& m, const ZEpi& e, int b, long long ij) {
  const long long q = (long long)b * m.nx * m.ny + ij;
  if (m.awet && (e.kt > 0 || e.dec)) {
    const double w = (e.kt > 0) ? e.aw : m.awet[q];
    m.awet[q] = e.dec ? __dmul_rn(w, e.f) : w;
  }
  if (e.dec) m.acum[q] = __dmul_rn(m.acum[q], e.f);
}

// Precision-form state value of element at (c32, plus c32lo when kept).
__host__ __device__ __forceinline__ double state32(const MemberDev& m, long long at) {
  return m.c32lo ? (double)m.c32[at] + (double)m.c32lo[at] : (double)m.c32[at];
}
// Store v into the precision-form state: rounded to FP32, or split into the
// FP32 pair c32 + c32lo when the compensated state is kept.
__device__ __forceinline__ void set_state32(const MemberDev& m, long long at, double v) {
  const float hi = __double2float_rn(v);
  m.c32[at] = hi;
  if (m.c32lo) m.c32lo[at] = __double2float_rn(v - (double)hi);
}
// Add inc to the precision-form state element at (FP64 add, one rounding).
__device__ __forceinline__ void add_to_state32(const MemberDev& m, long long at, double inc) {
  set_state32(m, at, state32(m, at) + inc);
}

// Boundary halo layers of one bin: x sweep W, E [k][j]; y sweep S, N [k][i];
// z sweep D, U [j][i].  Element of pencil pen (the sweep's spatial pencil
// index) on side s (0 low, 1 high) of direction dir:
__host__ __device__ __forceinline__ long long gh_per_bin(int nx, int ny, int nz) {
  return 2LL * ((long long)ny * nz + (long long)nx * nz + (long long)nx * ny);
}
__host__ __device__ __forceinline__ long long gh_offset(int dir, int side, long long pen, int nx, int ny,
                                                        int nz) {
  const long long ax = (long long)ny * nz, ay = (long long)nx * nz, az = (long long)nx * ny;
  const long long base = (dir == 0) ? 0 : (dir == 1) ? 2 * ax : 2 * (ax + ay);
  const long long n = (dir == 0) ? ax : (dir == 1) ? ay : az;
  return base + side * n + pen;
}

// A block of one sweep: 32 consecutive spatial pencils [pen0, pen0+32) of
// one member, one warp per bin [bin0, bin0 + blockDim/32).  Spatial pencil
// index: x (j + ny k), y (i + nx k), z (i + nx j).  Blocks of the same
// spatial tile are adjacent in the work list, so the face data they share
// is served from L1/L2 instead of DRAM once per bin.
struct WorkItem {
  int member;
  int pen0;
  int bin0;
  int slot;  // flux partial slot
};

// Correctly rounded a/b for a divisor with precomputed y = RN(1/b)
// (Markstein's correction, applied twice so that the second correction
// starts from a faithful quotient; P. Markstein, IBM J. Res. Dev. 34(1),
// 1990).  Numerators below 2^-800 are first scaled by 2^400 (exact) so no
// intermediate is subnormal, and zero numerators return the correctly
// signed zero a*y.  For |b| in [2^-100, 2^100] this is IEEE round-to-nearest
// a/b.  A quotient in the subnormal range (numerators below ~2^-900 only, the
// far fringe of a plume) is rounded a second time by the scaling back; that
// double rounding differs from a single one only when the scaled quotient q
// lies exactly halfway between two subnormals, and then the exact remainder
// sa - q b (one FMA) tells on which side the true quotient lies, so the tie
// is resolved by one subnormal ulp.  No division and no call on any path.
__device__ __forceinline__ double div_rn_recip(double a, double b, double y) {
  const bool tiny = fabs(a) < 0x1p-800;
  const double sa = tiny ? a * 0x1p400 : a;
  double q = sa * y;
  double r = fma(-q, b, sa);
  q = fma(r, y, q);
  r = fma(-q, b, sa);
  q = fma(r, y, q);
  double res = tiny ? q * 0x1p-400 : q;
#ifndef F3D_DIV_TIE
#define F3D_DIV_TIE 1
#endif
  if (F3D_DIV_TIE && tiny) {
    const double rem = fma(-q, b, sa);     // exact: the true quotient is q + rem / b
    const double d = q - res * 0x1p400;    // exact: q's distance from the rounded result
    if (fabs(d) == 0x1p-675 && rem != 0.0 && ((d > 0.0) == ((rem > 0.0) == (b > 0.0))))
      res = res + copysign(0x1p-1074, d);  // a tie the true quotient lies beyond
  }
  return (a == 0.0) ? a * y : res;
}

}  // namespace f3d
