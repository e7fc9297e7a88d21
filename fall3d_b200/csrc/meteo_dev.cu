// meteo_dev.cu -- the compute part of F3D_update_meteo_term
// (mod_F3D.F90:673-944) on the device: from the meteo model's corner winds
// of the two time levels of the interval and the diffusion coefficients at
// mass points, the staggered, scaled fields of the ADS step, written straight
// into the device layouts.
//
//   * ground corner winds are zero (mod_F3D.F90:676-683);
//   * grid_get_stagered_velocity (mod_Grid.F90:685-752): 4-point corner
//     averages at u, v and w faces;
//   * grid_get_scaled_velocity (mod_Grid.F90:761-870): u / Hm1, v / Hm2 at
//     v faces, and for the sigma mappings w = ((w - hx uw) - hy vw) / Hm3
//     with the terrain slopes decayed linearly with height when asked;
//   * the diffusion part of grid_get_scaled_variables (mod_Grid.F90:879-1017):
//     k1 / Hm1^2, k2 / Hm2^2 and for sigma k3 = ((k3 + hx^2 k1) + hy^2 k2) / Hm3^2
//     (with the unscaled k1, k2), vertical halos copied from the edge levels;
//   * the transposes of mod_F3D.F90:931-944 become the output indexing.
//
// Compiled with --fmad=false: every sum and product is rounded separately in
// the reference's order, so the fields equal those built on the host.
#include <cuda_runtime.h>

#include "f3d_common.cuh"
#include "phys_dev.cuh"

namespace f3d {

constexpr int kMapCartesian = 0, kMapSigmaLinearDecay = 2;  // 1: sigma, no decay

struct MetGeo {
  int nx, ny, nz, map_v;
  double X3max;
  const double* X3c;   // corner (w-face) heights above terrain, nz+1
  const double* X3p;   // mass-point heights, nz
  const double* dhdx;  // terrain slopes at mass points, nx*ny
  const double* dhdy;
  const double* hm1;   // ny
  const double* hm2;   // ny+4 (jps-2 .. jpe+2)
  const double* hm3;   // nx*ny
};

#define MGRID(e, total)                                                        \
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (total); \
       e += (long long)gridDim.x * blockDim.x)

// corner value, ground level (k = 0) forced to zero
__device__ __forceinline__ double cw(const double* a, const MetGeo& g, int i, int j, int k) {
  return (k == 0) ? 0.0 : a[i + (long long)(g.nx + 1) * (j + (long long)(g.ny + 1) * k)];
}

// ux[k][f=0..nx][j] of one snapshot
__global__ void k_met_u(MetGeo g, const double* __restrict__ uc, double* __restrict__ ux) {
  const long long tot = (long long)g.nz * (g.nx + 1) * g.ny;
  MGRID(e, tot) {
    const int j = (int)(e % g.ny);
    long long t = e / g.ny;
    const int f = (int)(t % (g.nx + 1));
    const int k = (int)(t / (g.nx + 1));
    const double u = 0.25 * (((cw(uc, g, f, j, k) + cw(uc, g, f, j + 1, k)) + cw(uc, g, f, j, k + 1)) +
                             cw(uc, g, f, j + 1, k + 1));
    ux[e] = u / g.hm1[j];
  }
}

// vy[k][f=0..ny][i] of one snapshot; Hm2 at the face is the mean of the two
// mass points beside it
__global__ void k_met_v(MetGeo g, const double* __restrict__ vc, double* __restrict__ vy) {
  const long long tot = (long long)g.nz * (g.ny + 1) * g.nx;
  MGRID(e, tot) {
    const int i = (int)(e % g.nx);
    long long t = e / g.nx;
    const int f = (int)(t % (g.ny + 1));
    const int k = (int)(t / (g.ny + 1));
    const double v = 0.25 * (((cw(vc, g, i, f, k) + cw(vc, g, i + 1, f, k)) + cw(vc, g, i, f, k + 1)) +
                             cw(vc, g, i + 1, f, k + 1));
    const double h = 0.5 * (g.hm2[f + 2] + g.hm2[f + 1]);
    vy[e] = v / h;
  }
}

// wz[f=0..nz][j][i] of one snapshot
__global__ void k_met_w(MetGeo g, const double* __restrict__ uc, const double* __restrict__ vc,
                        const double* __restrict__ wc, double* __restrict__ wz) {
  const long long tot = (long long)(g.nz + 1) * g.ny * g.nx;
  MGRID(e, tot) {
    const int i = (int)(e % g.nx);
    long long t = e / g.nx;
    const int j = (int)(t % g.ny);
    const int f = (int)(t / g.ny);
    double w = 0.25 * (((cw(wc, g, i, j, f) + cw(wc, g, i + 1, j, f)) + cw(wc, g, i, j + 1, f)) +
                       cw(wc, g, i + 1, j + 1, f));
    if (g.map_v != kMapCartesian) {
      const double uw = 0.25 * (((cw(uc, g, i, j, f) + cw(uc, g, i + 1, j, f)) + cw(uc, g, i, j + 1, f)) +
                                cw(uc, g, i + 1, j + 1, f));
      const double vw = 0.25 * (((cw(vc, g, i, j, f) + cw(vc, g, i + 1, j, f)) + cw(vc, g, i, j + 1, f)) +
                                cw(vc, g, i + 1, j + 1, f));
      const long long ij = i + (long long)g.nx * j;
      double hx = g.dhdx[ij], hy = g.dhdy[ij];
      if (g.map_v == kMapSigmaLinearDecay) {
        const double hz = 1.0 - g.X3c[f] / g.X3max;
        hx = hx * hz;
        hy = hy * hz;
      }
      w = ((w - hx * uw) - hy * vw) / g.hm3[ij];
    }
    wz[e] = w;
  }
}

// k1 (ips-2:ipe+2, jps:jpe, kps:kpe) unscaled -> k1x[k][p=-1..nx][j]
__global__ void k_met_k1(MetGeo g, const double* __restrict__ k1, double* __restrict__ k1x) {
  const long long tot = (long long)g.nz * (g.nx + 2) * g.ny;
  MGRID(e, tot) {
    const int j = (int)(e % g.ny);
    long long t = e / g.ny;
    const int p1 = (int)(t % (g.nx + 2));
    const int k = (int)(t / (g.nx + 2));
    k1x[e] = k1[(p1 + 1) + (long long)(g.nx + 4) * (j + (long long)g.ny * k)] / (g.hm1[j] * g.hm1[j]);
  }
}

// k2 (ips:ipe, jps-2:jpe+2, kps:kpe), i fastest, unscaled -> k2y[k][p=-1..ny][i]
__global__ void k_met_k2(MetGeo g, const double* __restrict__ k2, double* __restrict__ k2y) {
  const long long tot = (long long)g.nz * (g.ny + 2) * g.nx;
  MGRID(e, tot) {
    const int i = (int)(e % g.nx);
    long long t = e / g.nx;
    const int p1 = (int)(t % (g.ny + 2));
    const int k = (int)(t / (g.ny + 2));
    const double h = g.hm2[p1 + 1];
    k2y[e] = k2[i + (long long)g.nx * ((p1 + 1) + (long long)(g.ny + 4) * k)] / (h * h);
  }
}

// k3 (ips:ipe, jps:jpe, kps-2:kpe+2), i fastest, unscaled -> k3z[p=-1..nz][j][i];
// the halo levels take the scaled edge levels
__global__ void k_met_k3(MetGeo g, const double* __restrict__ k1, const double* __restrict__ k2,
                         const double* __restrict__ k3, double* __restrict__ k3z) {
  const long long tot = (long long)(g.nz + 2) * g.ny * g.nx;
  MGRID(e, tot) {
    const int i = (int)(e % g.nx);
    long long t = e / g.nx;
    const int j = (int)(t % g.ny);
    const int p = (int)(t / g.ny) - 1;
    const int k = (p < 0) ? 0 : ((p >= g.nz) ? g.nz - 1 : p);  // level whose value fills p
    const long long ij = i + (long long)g.nx * j;
    double v = k3[i + (long long)g.nx * (j + (long long)g.ny * (k + 2))];
    if (g.map_v != kMapCartesian) {
      double hx = g.dhdx[ij], hy = g.dhdy[ij];
      if (g.map_v == kMapSigmaLinearDecay) {
        const double hz = 1.0 - g.X3p[k] / g.X3max;
        hx = hx * hz;
        hy = hy * hz;
      }
      const double a1 = k1[(i + 2) + (long long)(g.nx + 4) * (j + (long long)g.ny * k)];
      const double a2 = k2[i + (long long)g.nx * ((j + 2) + (long long)(g.ny + 4) * k)];
      v = ((v + hx * hx * a1) + hy * hy * a2) / (g.hm3[ij] * g.hm3[ij]);
    }
    k3z[e] = v;
  }
}

// Constant diffusion (phys_get_kdiffu CONSTANT, mod_Phys.F90:477-480):
// k1 = k2 = kh, k3 = kv at every mass point, written unscaled into the three
// input layouts above.
__global__ void k_met_kconst(int nx, int ny, int nz, double kh, double kv, double* k1, double* k2,
                             double* k3) {
  const long long n1 = (long long)(nx + 4) * ny * nz, n2 = (long long)nx * (ny + 4) * nz,
                  n3 = (long long)nx * ny * (nz + 4);
  MGRID(e, n1 + n2 + n3) {
    if (e < n1) k1[e] = kh;
    else if (e < n1 + n2) k2[e - n1] = kh;
    else k3[e - n1 - n2] = kv;
  }
}

void launch_meteo_corners(const MetGeo& g, const double* uc, const double* vc, const double* wc,
                          const double* k1, const double* k2, const double* k3, double* ux,
                          double* vy, double* wz, double* k1x, double* k2y, double* k3z,
                          cudaStream_t st) {
  const long long ncor = (long long)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  const long long nu = (long long)g.nz * (g.nx + 1) * g.ny, nv = (long long)g.nz * (g.ny + 1) * g.nx,
                  nw = (long long)(g.nz + 1) * g.ny * g.nx;
  for (int s = 0; s < 2; ++s) {
    k_met_u<<<592, 256, 0, st>>>(g, uc + s * ncor, ux + s * nu);
    k_met_v<<<592, 256, 0, st>>>(g, vc + s * ncor, vy + s * nv);
    k_met_w<<<592, 256, 0, st>>>(g, uc + s * ncor, vc + s * ncor, wc + s * ncor, wz + s * nw);
  }
  k_met_k1<<<592, 256, 0, st>>>(g, k1, k1x);
  k_met_k2<<<592, 256, 0, st>>>(g, k2, k2y);
  k_met_k3<<<592, 256, 0, st>>>(g, k1, k2, k3, k3z);
}

// Current winds of a step with the gravity current's radial wind
// (mod_F3D.F90:1437-1445): the exact form adds rvel to the interpolated
// winds the prep kernel wrote (my_u = my_u + rvel, :1171, :1208); the
// precision form writes the interpolated FP64 wind plus rvel, rounded to
// FP32, into both velocity slots of a copy of its face data (gc4), which the
// sweeps then read in place of f4.
__global__ void k_gc_winds(MemberDev* members, int mi, int nx, int ny, int nz, int fp32, GcArgs g) {
  MemberDev& m = members[mi];
  const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)(ny + 1) * nx * nz;
  const double s = m.stime, f = m.wfacd;
  MGRID(e, nu + nv) {
    double rvel = 0.0;
    if (e < nu) {
      const int j = (int)(e % ny);
      const long long t = e / ny;
      const int i = (int)(t % (nx + 1)), k = (int)(t / (nx + 1));
      const bool add = gc_rvel_u(g, nx, ny, i, j, k, &rvel);
      if (!fp32) {
        if (add) m.ucur[e] = m.ucur[e] + rvel;
      } else {
        double u = (1.0 - s) * (f * m.ux[0][e]) + s * (f * m.ux[1][e]);
        if (add) u = u + rvel;
        float4 q = m.f4[0][e];
        q.x = q.y = (float)u;
        m.gc4[0][e] = q;
      }
    } else {
      const long long q = e - nu;
      const int i = (int)(q % nx);
      const long long t = q / nx;
      const int j = (int)(t % (ny + 1)), k = (int)(t / (ny + 1));
      const bool add = gc_rvel_v(g, nx, ny, i, j, k, &rvel);
      if (!fp32) {
        if (add) m.vcur[q] = m.vcur[q] + rvel;
      } else {
        double v = (1.0 - s) * (f * m.vy[0][q]) + s * (f * m.vy[1][q]);
        if (add) v = v + rvel;
        float4 r = m.f4[1][q];
        r.x = r.y = (float)v;
        m.gc4[1][q] = r;
      }
    }
  }
}

void launch_gc_winds(MemberDev* members, int mi, int nx, int ny, int nz, int fp32, const GcArgs& g,
                     cudaStream_t st) {
  k_gc_winds<<<592, 256, 0, st>>>(members, mi, nx, ny, nz, fp32, g);
}

// ---- phys_get_kdiffu (mod_Phys.F90:406-664) -------------------------------
// Thread per mass point; the corner fields are interpolated where read, as
// F3D_update_meteo_term interpolates them first (mod_F3D.F90:760-767).
__device__ __forceinline__ double kd_at(const double* a0, const double* a1, double s, long long q) {
  return (1.0 - s) * a0[q] + s * a1[q];
}

__global__ void k_kdiff_h(KdArgs a) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long NX1 = nx + 1, NY1 = ny + 1;
  const double alfa = 0.28, khf = 8000.0, rkhmin = 100.0;  // :444-446
  MGRID(e, (long long)nx * ny * nz) {
    const int i = (int)(e % nx);
    const long long t = e / nx;
    const int j = (int)(t % ny), k = (int)(t / ny);
    double kv;
    if (a.modkh == 1) {
      kv = a.kh0;
    } else {
      auto C = [&](const double* p0, const double* p1, int ii, int jj) {
        return kd_at(p0, p1, a.s, ii + NX1 * (jj + NY1 * k));
      };
      const double dx = a.dx1p[i + 2] * a.hm1[j];
      const double dy = a.dx2p[j + 2] * a.hm2[j + 2];
      const double u00 = C(a.uc0, a.uc1, i, j), u10 = C(a.uc0, a.uc1, i + 1, j);
      const double u01 = C(a.uc0, a.uc1, i, j + 1), u11 = C(a.uc0, a.uc1, i + 1, j + 1);
      const double v00 = C(a.vc0, a.vc1, i, j), v10 = C(a.vc0, a.vc1, i + 1, j);
      const double v01 = C(a.vc0, a.vc1, i, j + 1), v11 = C(a.vc0, a.vc1, i + 1, j + 1);
      const double dudx = 0.5 * (u10 - u00 + u11 - u01) / dx;
      const double dvdx = 0.5 * (v10 - v00 + v11 - v01) / dx;
      const double dudy = 0.5 * (u01 - u00 + u11 - u10) / dy;
      const double dvdy = 0.5 * (v01 - v00 + v11 - v10) / dy;
      if (a.modkh == 2) {  // CMAQ (:484-499)
        const double kht = alfa * alfa * dx * dy *
                           sqrt((dudx - dvdy) * (dudx - dvdy) + (dvdx + dudy) * (dvdx + dudy));
        const double khn = khf * (a.khn0 / (a.hm1[j] * a.dlon)) * (a.khn0 / (a.hm2[j + 2] * a.dlat));
        if (kht < 1.0 && khn < 1.0) kv = rkhmin;
        else kv = fmax(kht * khn / (kht + khn), rkhmin);
      } else {  // RAMS (:528-550)
        kv = a.rams_cs * a.rams_cs * dx * dy *
             sqrt((dudy + dvdx) * (dudy + dvdx) + 2.0 * (dudx * dudx + dvdy * dvdy));
        kv = fmax(fmax(kv, a.kmh[i + (long long)nx * j]), rkhmin);
      }
    }
    // k1(i, j, k) and its halo copies at the x ends (:501-504); k2 likewise in y
    double* r1 = a.k1 + (long long)(nx + 4) * (j + (long long)ny * k);
    r1[i + 2] = kv;
    if (i == 0) r1[0] = r1[1] = kv;
    if (i == nx - 1) r1[nx + 3] = r1[nx + 2] = kv;
    double* c2 = a.k2 + i + (long long)nx * (long long)(ny + 4) * k;
    c2[(long long)nx * (j + 2)] = kv;
    if (j == 0) c2[0] = c2[nx] = kv;
    if (j == ny - 1) c2[(long long)nx * (ny + 3)] = c2[(long long)nx * (ny + 2)] = kv;
  }
}

__global__ void k_kdiff_v(KdArgs a) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long NX1 = nx + 1, NY1 = ny + 1;
  const double KARMAN = 0.4, GI = 9.81, landac = 30.0;  // mod_KindType.F90:45-46, :447
  MGRID(e, (long long)nx * ny * nz) {
    const int i = (int)(e % nx);
    const long long t = e / nx;
    const int j = (int)(t % ny), k = (int)(t / ny);
    double kv;
    if (a.modkv == 1) {
      kv = a.kv0;
    } else {  // SIMILARITY (:595-645)
      auto Z = [&](int ii, int jj, int kk) { return a.zc[ii + NX1 * (jj + NY1 * kk)]; };
      auto C = [&](const double* p0, const double* p1, int ii, int jj, int kk) {
        return kd_at(p0, p1, a.s, ii + NX1 * (jj + NY1 * kk));
      };
      const double hp = (a.hc[i + NX1 * j] + a.hc[i + 1 + NX1 * j] + a.hc[i + NX1 * (j + 1)] +
                         a.hc[i + 1 + NX1 * (j + 1)]) / 4.0;
      const long long ij = i + (long long)nx * j;
      const double pb = a.pblh[ij], L = a.mon[ij], us = a.ust[ij];
      const double zp = (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k) + Z(i, j, k + 1) +
                         Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1)) / 8.0;
      const double z = fmax(0.0, zp - hp);
      if (z < pb) {
        const double zl = z / L;  // phys_get_Fih (:1702-1721)
        const double fih = (zl < 0.0) ? 1.0 / sqrt(1.0 - 15.0 * zl) : 1.0 + 5.0 * zl;
        kv = KARMAN * z * us * (1.0 - z / pb) * (1.0 - z / pb) / fih;
        kv = fmax(0.0, kv);
      } else {
        double lc = 1.0 / (KARMAN * z) + 1.0 / landac;
        lc = 1.0 / lc;
        double z1 = 0.25 * (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k));
        z1 = z1 - hp;
        double z2 = 0.25 * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1));
        z2 = z2 - hp;
        const double u1 = 0.25 * (C(a.uc0, a.uc1, i, j, k) + C(a.uc0, a.uc1, i + 1, j, k) +
                                  C(a.uc0, a.uc1, i, j + 1, k) + C(a.uc0, a.uc1, i + 1, j + 1, k));
        const double v1 = 0.25 * (C(a.vc0, a.vc1, i, j, k) + C(a.vc0, a.vc1, i + 1, j, k) +
                                  C(a.vc0, a.vc1, i, j + 1, k) + C(a.vc0, a.vc1, i + 1, j + 1, k));
        const double u2 = 0.25 * (C(a.uc0, a.uc1, i, j, k + 1) + C(a.uc0, a.uc1, i + 1, j, k + 1) +
                                  C(a.uc0, a.uc1, i, j + 1, k + 1) + C(a.uc0, a.uc1, i + 1, j + 1, k + 1));
        const double v2 = 0.25 * (C(a.vc0, a.vc1, i, j, k + 1) + C(a.vc0, a.vc1, i + 1, j, k + 1) +
                                  C(a.vc0, a.vc1, i, j + 1, k + 1) + C(a.vc0, a.vc1, i + 1, j + 1, k + 1));
        const double umod1 = sqrt(u1 * u1 + v1 * v1);
        const double umod2 = sqrt(u2 * u2 + v2 * v2);
        const double umod = 0.5 * (umod1 + umod2);
        const double tv1 = 0.25 * (C(a.tvc0, a.tvc1, i, j, k) + C(a.tvc0, a.tvc1, i + 1, j, k) +
                                   C(a.tvc0, a.tvc1, i, j + 1, k) + C(a.tvc0, a.tvc1, i + 1, j + 1, k));
        const double tv2 = 0.25 * (C(a.tvc0, a.tvc1, i, j, k + 1) + C(a.tvc0, a.tvc1, i + 1, j, k + 1) +
                                   C(a.tvc0, a.tvc1, i, j + 1, k + 1) + C(a.tvc0, a.tvc1, i + 1, j + 1, k + 1));
        const double um2 = fmax(umod * umod, 1e-18);  // phys_get_Rib (:1684-1696)
        const double Ri = GI * (z2 - z1) * (tv2 - tv1) / (um2 * 0.5 * (tv2 + tv1));
        double fc;  // phys_get_Fc (:1727-1741)
        if (Ri > 0.0) {
          fc = 1.0 + 10.0 * Ri * (1.0 + 8.0 * Ri);
          fc = 1.0 / fc;
        } else {
          fc = sqrt(1.0 - 18.0 * Ri);
        }
        kv = lc * lc * fabs((umod2 - umod1) / (z2 - z1)) * fc;
        kv = fmax(0.0, kv);
      }
    }
    // k3(i, j, k) and its halo copies at the bottom and top (:647-650)
    const long long pl = (long long)nx * ny;
    double* c3 = a.k3 + i + (long long)nx * j;
    c3[pl * (k + 2)] = kv;
    if (k == 0) c3[0] = c3[pl] = kv;
    if (k == nz - 1) c3[pl * (nz + 3)] = c3[pl * (nz + 2)] = kv;
  }
}

void launch_kdiffu(const KdArgs& a, cudaStream_t st) {
  k_kdiff_h<<<592, 256, 0, st>>>(a);
  k_kdiff_v<<<592, 256, 0, st>>>(a);
}

void launch_meteo_kconst(int nx, int ny, int nz, double kh, double kv, double* k1, double* k2,
                         double* k3, cudaStream_t st) {
  k_met_kconst<<<592, 256, 0, st>>>(nx, ny, nz, kh, kv, k1, k2, k3);
}

}  // namespace f3d
