// ads_fp64.cu -- FP64 "exact" ADS sweeps.  Compiled with --fmad=false so that
// every product and sum is rounded separately, in the reference's order, and
// the result reproduces the reference's FP64 CPU arithmetic bit for bit.
//
// Algorithm (mod_ADS.F90:233-811 + KT_RHS :1057-1120): one thread owns one
// pencil of one bin and marches along it once.  The four RK stages of the
// reference run as a software pipeline: stage s consumes the stage-(s-1)
// value at position q two cells behind stage s-1, because KT_RHS at cell i
// needs its inputs at i-2..i+2.  Each stage keeps a 2-cell window, its last
// face flux and limiter value in registers, so c is read from HBM once and
// written once per sweep with no scratch arrays (the reference copies whole
// pencils into c0/new_c/ini_c at every stage).
#include <cuda_runtime.h>

#include "f3d_common.cuh"

namespace f3d {

// Limiter r(i) from d1 = c(i)-c(i-1), d0 = c(i+1)-c(i)  (mod_ADS.F90:1124-1223)
template <int LIM>
__device__ __forceinline__ double limiter64(double d1, double d0) {
  if (LIM == 1) {
    if (fabs(d0) < kEps) return 1.0;
    double r = d1 / d0;
    return fmax(0.0, fmin(1.0, r));
  } else if (LIM == 2) {
    if (fabs(d0) < kEps) return (fabs(d1) < kEps) ? 0.0 : 2.0;
    double r = d1 / d0;
    double a = fmin(2.0 * r, 1.0), b = fmin(r, 2.0);
    return fmax(fmax(0.0, a), b);
  } else {
    if (fabs(d0) < kEps) return (fabs(d1) < kEps) ? 0.0 : 1.5;
    double r = d1 / d0;
    return 1.5 * (r * r + r) / (r * r + r + 1.0);
  }
}

// Register state of one RK stage walking a pencil.
struct Stage64 {
  double a1;     // a(q-1)
  double a2;     // a(q-2)
  double d1;     // a(q-1) - a(q-2)
  double r2;     // r(q-2)
  double F1;     // advective flux at face q-2
  double P1;     // diffusive flux at face q-2
  double kprev;  // diffusion at cell q-2
};

// Pencil accessors for one sweep direction.
struct Pencil {
  int n;
  long long c_off;     // offset of element 0 in c
  long long c_stride;  // stride between consecutive pencil elements
  const double* vel;   // face velocity, face f at vel[f * vstride]
  long long vstride;
  const double* vsub;  // z only: settling velocity subtracted from vel
  const double* kd;    // diffusion, position p at kd[(p + 1) * kstride]
  long long kstride;
  const double* dxp;   // reference offset: position p at dxp[p + 2]
  const double* dxb;   // reference offset: cell i at dxb[i + 1]
};

__device__ __forceinline__ double face_vel(const Pencil& P, int f) {
  double v = P.vel[f * P.vstride];
  if (P.vsub) v = v - P.vsub[f * P.vstride];
  return v;
}

// Arrival of a(q) at a stage.  Returns true when rhs(q-2) was produced;
// fills face-flux outputs for the boundary faces.
template <int LIM>
__device__ __forceinline__ bool stage_arrive(Stage64& s, const Pencil& P, int q,
                                             double a0, double& rhs,
                                             double& face_flux) {
  double d0 = a0 - s.a1;
  double r1 = limiter64<LIM>(s.d1, d0);
  bool produced = false;
  int f = q - 1;
  if (q >= 1) {
    double u = face_vel(P, f);
    double kf = P.kd[(long long)(f + 1) * P.kstride];
    double cl = s.a2 + 0.5 * s.r2 * s.d1;
    double cr = s.a1 - 0.5 * r1 * d0;
    double F_l = cl * u;
    double F_r = cr * u;
    double F0 = 0.5 * (F_l + F_r) - 0.5 * fabs(u) * (cr - cl);
    double P0 = 0.5 * (kf + s.kprev) * s.d1 / P.dxp[f + 1];
    face_flux = F0 + P0;
    if (q >= 2) {
      double db = P.dxb[q - 1];  // dxb(i), i = q-2
      rhs = (P0 - s.P1) / db - (F0 - s.F1) / db;
      produced = true;
    }
    s.F1 = F0;
    s.P1 = P0;
    s.kprev = kf;
  } else if (q == 0) {
    s.kprev = P.kd[0];  // diffusion at cell -1
  }
  s.a2 = s.a1;
  s.a1 = a0;
  s.d1 = d0;
  s.r2 = r1;
  return produced;
}

// March one pencil: free-flow ghosts, RK4 (or Euler), in-place update.
// Returns the boundary face fluxes of the last stage (flux(1), flux(2)).
template <int LIM, int TM>
__device__ __forceinline__ void march64(double* __restrict__ c, const Pencil& P,
                                        double dt, double& flux_lo,
                                        double& flux_hi) {
  const int n = P.n;
  double* cp = c + P.c_off;
  const long long cs = P.c_stride;
  // free flow ghosts (mod_ADS.F90:1227-1326), bvalue = 0
  double c_first = cp[0];
  double uL = face_vel(P, 0);
  double uR = face_vel(P, n);
  double gL = (uL > 0.0) ? 2.0 * 0.0 - c_first : c_first;
  double gR = 0.0;

  Stage64 S1 = {0, 0, 0, 0, 0, 0, 0}, S2 = S1, S3 = S1, S4 = S1;
  double ch0 = 0, ch1 = 0, ch2 = 0, ch3 = 0, ch4 = 0, ch5 = 0, ch6 = 0;  // c(t-m)
  double nh0 = 0, nh1 = 0, nh2 = 0, nh3 = 0, nh4 = 0, nh5 = 0, nh6 = 0;  // new(t-2-m)
  double ff;
  const double hdt = 0.5 * dt;

  if constexpr (TM == 1) {
    for (int t = -2; t <= n + 1; ++t) {
      double a;
      if (t < 0) a = gL;
      else if (t < n) a = cp[t * cs];
      else a = gR;
      ch2 = ch1; ch1 = ch0; ch0 = a;
      if (t == n - 1) gR = (uR < 0.0) ? 2.0 * 0.0 - a : a;
      double k1;
      if (stage_arrive<LIM>(S1, P, t, a, k1, ff)) {
        cp[(t - 2) * cs] = ch2 + dt * k1;
      }
      if (t == 1) flux_lo = ff;
      if (t == n + 1) flux_hi = ff;
    }
  } else {
#pragma unroll 1
  for (int t = -2; t <= n + 7; ++t) {
    // shift histories
    ch6 = ch5; ch5 = ch4; ch4 = ch3; ch3 = ch2; ch2 = ch1; ch1 = ch0;
    nh6 = nh5; nh5 = nh4; nh4 = nh3; nh3 = nh2; nh2 = nh1; nh1 = nh0;
    // stage 1 arrival at q = t
    double k1 = 0.0;
    bool have1 = false;
    if (t <= n + 1) {
      double a;
      if (t < 0) a = gL;
      else if (t < n) a = cp[t * cs];
      else a = gR;
      ch0 = a;
      if (t == n - 1) gR = (uR < 0.0) ? 2.0 * 0.0 - a : a;
      have1 = stage_arrive<LIM>(S1, P, t, a, k1, ff);
    }
    // stage 2 arrival at q = t-2
    double k2 = 0.0;
    bool have2 = false;
    {
      int q = t - 2;
      if (q >= -2 && q <= n + 1) {
        double a;
        if (q < 0) a = gL;
        else if (q >= n) a = gR;
        else {
          a = ch2 + hdt * k1;
          nh0 = ch2 + dt * k1 / 6.0;
        }
        have2 = stage_arrive<LIM>(S2, P, q, a, k2, ff);
      }
    }
    // stage 3 arrival at q = t-4
    double k3 = 0.0;
    bool have3 = false;
    {
      int q = t - 4;
      if (q >= -2 && q <= n + 1) {
        double a;
        if (q < 0) a = gL;
        else if (q >= n) a = gR;
        else {
          a = ch4 + hdt * k2;
          nh2 = nh2 + dt * k2 / 3.0;
        }
        have3 = stage_arrive<LIM>(S3, P, q, a, k3, ff);
      }
    }
    // stage 4 arrival at q = t-6
    {
      int q = t - 6;
      if (q >= -2 && q <= n + 1) {
        double a;
        if (q < 0) a = gL;
        else if (q >= n) a = gR;
        else {
          a = ch6 + dt * k3;
          nh4 = nh4 + dt * k3 / 3.0;
        }
        double k4;
        if (stage_arrive<LIM>(S4, P, q, a, k4, ff)) {
          cp[(q - 2) * cs] = nh6 + dt * k4 / 6.0;
        }
        if (q == 1) flux_lo = ff;
        if (q == n + 1) flux_hi = ff;
      }
    }
  }
  }
}

// Deterministic block reduction of two doubles (pairwise tree in smem).
__device__ __forceinline__ void block_reduce2(double a, double b, double* out) {
  __shared__ double sa[256], sb[256];
  int t = threadIdx.x;
  sa[t] = a;
  sb[t] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) {
      sa[t] = sa[t] + sa[t + s];
      sb[t] = sb[t] + sb[t + s];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = sa[0];
    out[1] = sb[0];
  }
}

template <int DIR, int LIM, int TM>
__global__ void __launch_bounds__(128) k_sweep64(const MemberDev* __restrict__ members,
                                                 const WorkItem* __restrict__ work) {
  const WorkItem w = work[blockIdx.x];
  const MemberDev& m = members[w.member];
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  const long long npen = (DIR == DIR_X) ? (long long)ny * nz * m.nb
                         : (DIR == DIR_Y) ? (long long)nx * nz * m.nb
                                          : (long long)nx * ny * m.nb;
  const long long pen = (long long)w.pen0 + threadIdx.x;
  double lo = 0.0, hi = 0.0;
  double clo = 0.0, chi = 0.0;  // contributions flux*area*dt
  if (pen < npen) {
    Pencil P;
    double area;
    const double dt = m.dt;
    if (DIR == DIR_X) {
      int j = (int)(pen % ny);
      long long t = pen / ny;
      int k = (int)(t % nz);
      int b = (int)(t / nz);
      P.n = nx;
      P.c_off = (((long long)b * nz + k) * ny + j) * nx;
      P.c_stride = 1;
      P.vel = m.ucur + (long long)k * (nx + 1) * ny + j;
      P.vstride = ny;
      P.vsub = nullptr;
      P.kd = m.k1x + (long long)k * (nx + 2) * ny + j;
      P.kstride = ny;
      P.dxp = m.dx1p;
      P.dxb = m.dx1b;
      area = m.dx3b[k + 1] * m.dx2b[j + 1];
    } else if (DIR == DIR_Y) {
      int i = (int)(pen % nx);
      long long t = pen / nx;
      int k = (int)(t % nz);
      int b = (int)(t / nz);
      P.n = ny;
      P.c_off = ((long long)b * nz + k) * ny * (long long)nx + i;
      P.c_stride = nx;
      P.vel = m.vcur + (long long)k * (ny + 1) * nx + i;
      P.vstride = nx;
      P.vsub = nullptr;
      P.kd = m.k2y + (long long)k * (ny + 2) * nx + i;
      P.kstride = nx;
      P.dxp = m.dx2p;
      P.dxb = m.dx2b;
      area = m.dx3b[k + 1] * m.dx1b[i + 1];
    } else {
      int i = (int)(pen % nx);
      long long t = pen / nx;
      int j = (int)(t % ny);
      int b = (int)(t / ny);
      P.n = nz;
      P.c_off = (long long)b * nz * ny * nx + (long long)j * nx + i;
      P.c_stride = (long long)nx * ny;
      P.vel = m.wcur + (long long)j * nx + i;
      P.vstride = (long long)nx * ny;
      P.vsub = m.vs + (long long)b * (nz + 1) * ny * nx + (long long)j * nx + i;
      P.kd = m.k3z + (long long)j * nx + i;
      P.kstride = (long long)nx * ny;
      P.dxp = m.dx3p;
      P.dxb = m.dx3b;
      area = m.dx2b[j + 1] * m.dx1b[i + 1];
    }
    march64<LIM, TM>(m.c64, P, dt, lo, hi);
    clo = lo * area * dt;
    chi = hi * area * dt;
    if (DIR == DIR_Z) {
      int i = (int)(pen % nx);
      long long t = pen / nx;
      int j = (int)(t % ny);
      int b = (int)(t / ny);
      double* a = m.acum + ((long long)b * ny + j) * nx + i;
      *a = *a + fabs(lo) * dt;
    }
  }
  block_reduce2(clo, chi, m.flux_part + 2 * (long long)w.slot);
}

// Host launchers -------------------------------------------------------------
template <int DIR>
static void launch_dir64(int lim, int tm, const MemberDev* members,
                         const WorkItem* work, int nblocks, cudaStream_t st) {
  dim3 g(nblocks), b(128);
#define F3D_L(L, T) k_sweep64<DIR, L, T><<<g, b, 0, st>>>(members, work)
  if (tm == 1) {
    if (lim == 1) F3D_L(1, 1); else if (lim == 2) F3D_L(2, 1); else F3D_L(3, 1);
  } else {
    if (lim == 1) F3D_L(1, 2); else if (lim == 2) F3D_L(2, 2); else F3D_L(3, 2);
  }
#undef F3D_L
}

void launch_sweep64(int dir, int lim, int tm, const MemberDev* members,
                    const WorkItem* work, int nblocks, cudaStream_t st) {
  if (nblocks <= 0) return;
  if (dir == DIR_X) launch_dir64<DIR_X>(lim, tm, members, work, nblocks, st);
  else if (dir == DIR_Y) launch_dir64<DIR_Y>(lim, tm, members, work, nblocks, st);
  else launch_dir64<DIR_Z>(lim, tm, members, work, nblocks, st);
}

// Per-step preparation: current winds u,v,w = (1-s) x1 + s x2
// (mod_F3D.F90:1437-1439, mod_ADS.F90:667), then the sparse source term
// c += dt*s/vol (mod_F3D.F90:1456-1473).
__global__ void k_prep64(const MemberDev* __restrict__ members, const int* __restrict__ blk_member,
                         const int* __restrict__ blk_first, int mask) {
  const int mi = blk_member[blockIdx.x];
  const MemberDev& m = members[mi];
  const long long nu = (long long)(m.nx + 1) * m.ny * m.nz;
  const long long nv = (long long)(m.ny + 1) * m.nx * m.nz;
  const long long nw = (long long)(m.nz + 1) * m.nx * m.ny;
  const double s = m.stime;
  long long q = (long long)(blockIdx.x - blk_first[mi]) * blockDim.x + threadIdx.x;
  if (q < nu) {
    if (mask & 1) m.ucur[q] = (1.0 - s) * m.ux[0][q] + s * m.ux[1][q];
    return;
  }
  q -= nu;
  if (q < nv) {
    if (mask & 2) m.vcur[q] = (1.0 - s) * m.vy[0][q] + s * m.vy[1][q];
    return;
  }
  q -= nv;
  if (q < nw && (mask & 4)) m.wcur[q] = (1.0 - s) * m.wz[0][q] + s * m.wz[1][q];
}

__global__ void k_source64(const MemberDev* __restrict__ members, int nmembers) {
  for (int mi = blockIdx.y; mi < nmembers; mi += gridDim.y) {
    const MemberDev& m = members[mi];
    const long long tot = (long long)m.nsrc * m.nb;
    const long long ncell = (long long)m.nx * m.ny * m.nz;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
      int q = (int)(e / m.nb), b = (int)(e % m.nb);
      double* cc = m.c64 + (long long)b * ncell + m.src_cell[q];
      *cc = *cc + m.dt * m.src_s[(long long)q * m.nb + b] / m.src_vol[q];
    }
  }
}

void launch_prep64(const MemberDev* members, const int* blk_member, const int* blk_first,
                   int nblocks, int mask, cudaStream_t st) {
  if (nblocks > 0) k_prep64<<<nblocks, 256, 0, st>>>(members, blk_member, blk_first, mask);
}

void launch_source64(const MemberDev* members, int nmembers, cudaStream_t st) {
  dim3 g(8, nmembers < 65535 ? nmembers : 65535);
  k_source64<<<g, 128, 0, st>>>(members, nmembers);
}

}  // namespace f3d
