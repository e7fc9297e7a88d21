// aux_fp64.cu -- FP64 kernels around the sweeps: layout conversion of the
// reference arrays, per-step parameters, boundary-flux reduction, the CFL
// reduction, the mass budget and the settling-velocity solve.  Compiled with
// --fmad=false: every expression keeps the reference's rounding.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "f3d_common.cuh"
#include "step_dev.cuh"
#include "vset.cuh"
#include "phys_dev.cuh"

namespace f3d {

#define GRID_STRIDE(e, total)                                                  \
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (total); \
       e += (long long)gridDim.x * blockDim.x)

// ---- reference layout -> device layout ------------------------------------
// u (ibs-1:ibe+1, jps:jpe, kps:kpe, 2) -> ux[s][k][f=0..nx][j]
__global__ void k_conv_u(const double* __restrict__ in, double* __restrict__ out, int nx, int ny,
                         int nz) {
  const long long tot = 2LL * nz * (nx + 1) * ny;
  GRID_STRIDE(e, tot) {
    int j = (int)(e % ny);
    long long t = e / ny;
    int f = (int)(t % (nx + 1));
    t /= (nx + 1);
    int k = (int)(t % nz);
    int s = (int)(t / nz);
    out[e] = in[(f + 1) + (long long)(nx + 3) * (j + (long long)ny * (k + (long long)nz * s))];
  }
}
// v (jbs-1:jbe+1, ips:ipe, kps:kpe, 2) -> vy[s][k][f=0..ny][i]
__global__ void k_conv_v(const double* __restrict__ in, double* __restrict__ out, int nx, int ny,
                         int nz) {
  const long long tot = 2LL * nz * (ny + 1) * nx;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int f = (int)(t % (ny + 1));
    t /= (ny + 1);
    int k = (int)(t % nz);
    int s = (int)(t / nz);
    out[e] = in[(f + 1) + (long long)(ny + 3) * (i + (long long)nx * (k + (long long)nz * s))];
  }
}
// w (kbs-1:kbe+1, ips:ipe, jps:jpe, 2) -> wz[s][f=0..nz][j][i]
__global__ void k_conv_w(const double* __restrict__ in, double* __restrict__ out, int nx, int ny,
                         int nz) {
  const long long tot = 2LL * (nz + 1) * ny * nx;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    t /= ny;
    int f = (int)(t % (nz + 1));
    int s = (int)(t / (nz + 1));
    out[e] = in[(f + 1) + (long long)(nz + 3) * (i + (long long)nx * (j + (long long)ny * s))];
  }
}
// k1 (ips-2:ipe+2, jps:jpe, kps:kpe) -> k1x[k][p=-1..nx][j]
__global__ void k_conv_k1(const double* __restrict__ in, double* __restrict__ out, int nx, int ny,
                          int nz) {
  const long long tot = (long long)nz * (nx + 2) * ny;
  GRID_STRIDE(e, tot) {
    int j = (int)(e % ny);
    long long t = e / ny;
    int p1 = (int)(t % (nx + 2));
    int k = (int)(t / (nx + 2));
    out[e] = in[(p1 + 1) + (long long)(nx + 4) * (j + (long long)ny * k)];
  }
}
// k2 (jps-2:jpe+2, ips:ipe, kps:kpe) -> k2y[k][p=-1..ny][i]
__global__ void k_conv_k2(const double* __restrict__ in, double* __restrict__ out, int nx, int ny,
                          int nz) {
  const long long tot = (long long)nz * (ny + 2) * nx;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int p1 = (int)(t % (ny + 2));
    int k = (int)(t / (ny + 2));
    out[e] = in[(p1 + 1) + (long long)(ny + 4) * (i + (long long)nx * k)];
  }
}
// k3 (kps-2:kpe+2, ips:ipe, jps:jpe) -> k3z[p=-1..nz][j][i]
__global__ void k_conv_k3(const double* __restrict__ in, double* __restrict__ out, int nx, int ny,
                          int nz) {
  const long long tot = (long long)(nz + 2) * ny * nx;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    int p1 = (int)(t / ny);
    out[e] = in[(p1 + 1) + (long long)(nz + 4) * (i + (long long)nx * j)];
  }
}
// vs (ips:ipe, jps:jpe, kbs-1:kbe+1, nb) -> vs[b][f=0..nz][j][i]
__global__ void k_conv_vs(const double* __restrict__ in, double* __restrict__ out, int nx, int ny,
                          int nz, int nb) {
  const long long tot = (long long)nb * (nz + 1) * ny * nx;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    t /= ny;
    int f = (int)(t % (nz + 1));
    int b = (int)(t / (nz + 1));
    out[e] = in[i + (long long)nx * (j + (long long)ny * ((f + 1) + (long long)(nz + 3) * b))];
  }
}
// c (ips-2:ipe+2, jps-2:jpe+2, kps-2:kpe+2, nb) -> c[b][k][j][i]
__global__ void k_conv_c_in(const double* __restrict__ in, double* __restrict__ out, int nx,
                            int ny, int nz, int nb) {
  const long long tot = (long long)nb * nz * ny * nx;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    t /= ny;
    int k = (int)(t % nz);
    int b = (int)(t / nz);
    out[e] = in[(i + 2) + (long long)(nx + 4) *
                              ((j + 2) + (long long)(ny + 4) * ((k + 2) + (long long)(nz + 4) * b))];
  }
}
// acum (ips-2:ipe+2, jps-2:jpe+2, nb) -> acum[b][j][i]
__global__ void k_conv_acum_in(const double* __restrict__ in, double* __restrict__ out, int nx,
                               int ny, int nb) {
  const long long tot = (long long)nb * ny * nx;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    int b = (int)(t / ny);
    out[e] = in[(i + 2) + (long long)(nx + 4) * ((j + 2) + (long long)(ny + 4) * b)];
  }
}
// device settling velocity [b][f][j][i] -> reference layout with the halo faces
__global__ void k_conv_vs_out(const double* __restrict__ in, double* __restrict__ out, int nx,
                              int ny, int nz, int nb) {
  const long long tot = (long long)nb * (nz + 3) * ny * nx;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    t /= ny;
    int f1 = (int)(t % (nz + 3));
    int b = (int)(t / (nz + 3));
    int f = f1 - 1;
    if (f < 0) f = 0;
    if (f > nz) f = nz;
    out[e] = in[(((long long)b * (nz + 1) + f) * ny + j) * nx + i];
  }
}

void launch_conv(int which, const double* in, double* out, int nx, int ny, int nz, int nb,
                 cudaStream_t st) {
  dim3 g(2048), b(256);
  switch (which) {
    case 0: k_conv_u<<<g, b, 0, st>>>(in, out, nx, ny, nz); break;
    case 1: k_conv_v<<<g, b, 0, st>>>(in, out, nx, ny, nz); break;
    case 2: k_conv_w<<<g, b, 0, st>>>(in, out, nx, ny, nz); break;
    case 3: k_conv_k1<<<g, b, 0, st>>>(in, out, nx, ny, nz); break;
    case 4: k_conv_k2<<<g, b, 0, st>>>(in, out, nx, ny, nz); break;
    case 5: k_conv_k3<<<g, b, 0, st>>>(in, out, nx, ny, nz); break;
    case 6: k_conv_vs<<<g, b, 0, st>>>(in, out, nx, ny, nz, nb); break;
    case 7: k_conv_c_in<<<g, b, 0, st>>>(in, out, nx, ny, nz, nb); break;
    case 8: k_conv_acum_in<<<g, b, 0, st>>>(in, out, nx, ny, nb); break;
    case 9: k_conv_vs_out<<<g, b, 0, st>>>(in, out, nx, ny, nz, nb); break;
    default: break;
  }
}

// ---- FP64 face diffusion 0.5 (k(f) + k(f-1)) (the P term of KT_RHS,
// mod_ADS.F90:1111-1112), once per meteo update, for every face
__global__ void k_face_kk(MemberDev* members, int mi) {
  MemberDev& m = members[mi];
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)(ny + 1) * nx * nz,
                  nw = (long long)(nz + 1) * nx * ny;
  GRID_STRIDE(e, nu + nv + nw) {
    long long q = e;
    if (q < nu) {  // [k][f][j], k1x [k][p+1][j]
      int j = (int)(q % ny);
      long long t = q / ny;
      int f = (int)(t % (nx + 1));
      int k = (int)(t / (nx + 1));
      const double* kk = m.k1x + (long long)k * (nx + 2) * ny + j;
      const_cast<double*>(m.kkf[0])[q] = 0.5 * (kk[(long long)(f + 1) * ny] + kk[(long long)f * ny]);
      continue;
    }
    q -= nu;
    if (q < nv) {  // [k][f][i], k2y [k][p+1][i]
      int i = (int)(q % nx);
      long long t = q / nx;
      int f = (int)(t % (ny + 1));
      int k = (int)(t / (ny + 1));
      const double* kk = m.k2y + (long long)k * (ny + 2) * nx + i;
      const_cast<double*>(m.kkf[1])[q] = 0.5 * (kk[(long long)(f + 1) * nx] + kk[(long long)f * nx]);
      continue;
    }
    q -= nv;
    {  // [f][j][i], k3z [p+1][j][i]
      long long plane = (long long)nx * ny;
      long long ij = q % plane;
      int f = (int)(q / plane);
      const double* kk = m.k3z + ij;
      const_cast<double*>(m.kkf[2])[q] = 0.5 * (kk[(long long)(f + 1) * plane] + kk[(long long)f * plane]);
    }
  }
}
void launch_face_kk(MemberDev* members, int mi, cudaStream_t st) {
  k_face_kk<<<1184, 256, 0, st>>>(members, mi);
}

// ---- per-step parameters (kernel arguments are captured at launch) -------
__global__ void k_set_step(MemberDev* members, int mi, double dt, double time, int iiter) {
  MemberDev& m = members[mi];
  m.dt = dt;
  m.time = time;
  m.iiter = iiter;
  m.stime = (time - m.t_its) / (m.t_ite - m.t_its);  // mod_F3D.F90:1437
}
__global__ void k_set_dt_stime(MemberDev* members, int mi, double dt, double stime) {
  members[mi].dt = dt;
  members[mi].stime = stime;
}
// Per-member step parameters for up to 64 members per launch (arguments are
// copied at launch, so the host arrays may change right after).
struct StepChunk {
  int first, count, iiter;
  double dt[64];
  double time[64];
};
__global__ void k_set_steps(MemberDev* members, StepChunk c) {
  const int q = threadIdx.x;
  if (q < c.count) {
    MemberDev& m = members[c.first + q];
    m.dt = c.dt[q];
    m.time = c.time[q];
    m.iiter = c.iiter;
    m.stime = (c.time[q] - m.t_its) / (m.t_ite - m.t_its);
  }
}
void launch_set_steps(MemberDev* members, int n, const double* dt, const double* time, int iiter,
                      cudaStream_t st) {
  for (int f = 0; f < n; f += 64) {
    StepChunk c;
    c.first = f;
    c.count = (n - f < 64) ? n - f : 64;
    c.iiter = iiter;
    for (int q = 0; q < c.count; ++q) {
      c.dt[q] = dt[f + q];
      c.time[q] = time[f + q];
    }
    k_set_steps<<<1, 64, 0, st>>>(members, c);
  }
}

// Device clock of every member (graph replays need no host input).
__global__ void k_advance_clock(MemberDev* members, int n) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) member_advance(members[q]);
}
void launch_advance_clock(MemberDev* members, int n, cudaStream_t st) {
  k_advance_clock<<<(n + 63) / 64, 64, 0, st>>>(members, n);
}

// dt of each member from its CFL maxima (mod_Grid.F90:1125-1138), in place.
__global__ void k_finalize_dt(MemberDev* members, int n, const double* red, double cfl,
                              double run_end) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) {
    double mx = fmax(fmax(red[3 * q], red[3 * q + 1]), red[3 * q + 2]);
    if (mx > 0.0) mx = 1.0 / mx;
    mx = cfl * mx;
    MemberDev& m = members[q];
    m.dt = fmin(mx, run_end);
  }
}
void launch_finalize_dt(MemberDev* members, int n, const double* red, double cfl, double run_end,
                        cudaStream_t st) {
  k_finalize_dt<<<(n + 63) / 64, 64, 0, st>>>(members, n, red, cfl, run_end);
}

void launch_set_step(MemberDev* members, int mi, double dt, double time, int iiter,
                     cudaStream_t st) {
  k_set_step<<<1, 1, 0, st>>>(members, mi, dt, time, iiter);
}
void launch_set_dt_stime(MemberDev* members, int mi, double dt, double stime, cudaStream_t st) {
  k_set_dt_stime<<<1, 1, 0, st>>>(members, mi, dt, stime);
}

// ---- boundary flux reduction: one block per member ------------------------
// partial slots of each direction are summed pairwise; the step increments go
// to flux_step {W,E,S,N,U,D} and are added to the running totals with a
// Kahan-compensated update.
__global__ void k_flux_reduce(const MemberDev* __restrict__ members, int dirmask) {
  __shared__ double sa[256], sb[256];
  member_flux_reduce(members[blockIdx.x], dirmask, sa, sb);
}
__global__ void k_zero_step(const MemberDev* __restrict__ members) {
  const MemberDev& m = members[blockIdx.x];
  if (threadIdx.x < 6) m.flux_step[threadIdx.x] = 0.0;
}
void launch_flux_reduce(const MemberDev* members, int nmembers, int dirmask, cudaStream_t st) {
  k_flux_reduce<<<nmembers, 256, 0, st>>>(members, dirmask);
}
void launch_zero_step(const MemberDev* members, int nmembers, cudaStream_t st) {
  k_zero_step<<<nmembers, 32, 0, st>>>(members);
}

// ---- CFL: grid_get_time_step (mod_Grid.F90:1026-1141) -----------------------
// Non-negative doubles order like their bit patterns, so an integer atomicMax
// gives the exact maximum independently of the reduction order.
__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

__global__ void k_cfl(const MemberDev* __restrict__ members, int mi, double s, int criterion,
                      double* out3, GcArgs gc) {
  const MemberDev& m = members[mi];
  const int nx = m.nx, ny = m.ny, nz = m.nz, nb = m.nb;
  const long long tot = (long long)nx * ny * nz;
  double d1 = 0.0, d2 = 0.0, d3 = 0.0;
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    int k = (int)(t / ny);
    long long iu = ((long long)k * (nx + 1) + i) * ny + j;
    long long iv = ((long long)k * (ny + 1) + j) * nx + i;
    long long iw = ((long long)k * ny + j) * nx + i;
    const double f = m.wfacd;
    double u = (1.0 - s) * (f * m.ux[0][iu]) + s * (f * m.ux[1][iu]);
    double v = (1.0 - s) * (f * m.vy[0][iv]) + s * (f * m.vy[1][iv]);
    double w = (1.0 - s) * m.wz[0][iw] + s * m.wz[1][iw];
    if (gc.on) {  // the winds the step uses, with the radial wind (mod_F3D.F90:1443-1452)
      double r;
      if (gc_rvel_u(gc, nx, ny, i, j, k, &r)) u = u + r;
      if (gc_rvel_v(gc, nx, ny, i, j, k, &r)) v = v + r;
    }
    double k1 = m.k1x[((long long)k * (nx + 2) + (i + 1)) * ny + j];
    double k2 = m.k2y[((long long)k * (ny + 2) + (j + 1)) * nx + i];
    double k3 = m.k3z[((long long)(k + 1) * ny + j) * nx + i];
    double w_max = -INFINITY;
    for (int b = 0; b < nb; ++b)
      w_max = fmax(w_max, fabs(w - m.vs[(((long long)b * (nz + 1) + k) * ny + j) * nx + i]));
    double dx = m.dx1p[i + 2], dy = m.dx2p[j + 2], dz = m.dx3p[k + 2];
    if (criterion == 1) {
      d1 = fmax(d1, 2.0 * k1 / (dx * dx) + fabs(u) / dx);
      d2 = fmax(d2, 2.0 * k2 / (dy * dy) + fabs(v) / dy);
      d3 = fmax(d3, 2.0 * k3 / (dz * dz) + w_max / dz);
    } else {
      double dtinv = 2.0 * k1 / (dx * dx) + fabs(u) / dx + 2.0 * k2 / (dy * dy) + fabs(v) / dy +
                     2.0 * k3 / (dz * dz) + w_max / dz;
      d1 = fmax(d1, dtinv);
    }
  }
  // warp max then atomics
  for (int o = 16; o > 0; o >>= 1) {
    d1 = fmax(d1, __shfl_xor_sync(0xffffffffu, d1, o));
    d2 = fmax(d2, __shfl_xor_sync(0xffffffffu, d2, o));
    d3 = fmax(d3, __shfl_xor_sync(0xffffffffu, d3, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(out3 + 0, d1);
    atomic_max_pos(out3 + 1, d2);
    atomic_max_pos(out3 + 2, d3);
  }
}
void launch_cfl(const MemberDev* members, int mi, double s, int criterion, double* out3,
                cudaStream_t st, const GcArgs* gc) {
  GcArgs g;
  memset(&g, 0, sizeof(g));
  if (gc) g = *gc;
  k_cfl<<<1184, 256, 0, st>>>(members, mi, s, criterion, out3, g);
}

// ---- mass in the volume: grid_get_mass_volume (mod_Grid.F90:1340-1389) ------
// per bin: pairwise block sums into partials[b][block], then a second pass.
__global__ void k_mass_partial(const MemberDev* __restrict__ members, int mi, int fp32,
                               double* partials) {
  const MemberDev& m = members[mi];
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  const long long ncell = (long long)nx * ny * nz;
  const int b = blockIdx.y;
  __shared__ double sm[256];
  double acc = 0.0, comp = 0.0;  // Neumaier compensated
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ncell;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    int k = (int)(t / ny);
    double c = fp32 ? state32(m, (long long)b * ncell + e) : m.c64[(long long)b * ncell + e];
    double x = c * m.dx1p[i + 2] * m.dx2p[j + 2] * m.dx3p[k + 2];
    double tt = acc + x;
    if (fabs(acc) >= fabs(x)) comp += (acc - tt) + x; else comp += (x - tt) + acc;
    acc = tt;
  }
  sm[threadIdx.x] = acc + comp;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sm[threadIdx.x] = sm[threadIdx.x] + sm[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[(long long)b * gridDim.x + blockIdx.x] = sm[0];
}
__global__ void k_mass_final(const double* partials, int nblk, int nb, double* out) {
  __shared__ double sm[256];
  for (int b = 0; b < nb; ++b) {
    double acc = 0.0, comp = 0.0;
    for (int s = threadIdx.x; s < nblk; s += blockDim.x) {
      double x = partials[(long long)b * nblk + s];
      double tt = acc + x;
      if (fabs(acc) >= fabs(x)) comp += (acc - tt) + x; else comp += (x - tt) + acc;
      acc = tt;
    }
    sm[threadIdx.x] = acc + comp;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sm[threadIdx.x] = sm[threadIdx.x] + sm[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[b] = sm[0];
    __syncthreads();
  }
}
void launch_mass(const MemberDev* members, int mi, int nb, int fp32, double* partials, int nblk,
                 double* out, cudaStream_t st) {
  dim3 g(nblk, nb);
  k_mass_partial<<<g, 256, 0, st>>>(members, mi, fp32, partials);
  k_mass_final<<<1, 256, 0, st>>>(partials, nblk, nb, out);
}

// ---- settling velocity: phys_get_vset_point, see vset.cuh --------------------
__global__ void k_vset_points(int model, int n, const double* diam, const double* rhop,
                              const double* psi, const double* rhoa, const double* visc,
                              double* vset, int* flags, int* iters, int* nfail, int maxit) {
  GRID_STRIDE(q, (long long)n) {
    int it;
    double v;
    int fl = vset_point_dev(diam[q], rhop[q], psi[q], rhoa[q], visc[q], model, &v, &it, maxit);
    vset[q] = v;
    flags[q] = fl;
    if (iters) iters[q] = it;
    if (fl) atomicAdd(nfail, 1);
  }
}
void launch_vset_points(int model, int n, const double* diam, const double* rhop,
                        const double* psi, const double* rhoa, const double* visc, double* vset,
                        int* flags, int* iters, int* nfail, cudaStream_t st) {
  k_vset_points<<<592, 128, 0, st>>>(model, n, diam, rhop, psi, rhoa, visc, vset, flags, iters,
                                      nfail, vset_maxit());
}

// phys_get_vset (mod_Phys.F90:673-740) + vs/Hm3 (mod_Grid.F90:996-1005).
// rhoc, tc corners (nx+1)(ny+1)(nz+1), i fastest.  bins: [diam, rhop, psi]
// in bin_par[3*b..], bin_flags[b] = cat | (aggregate << 8).
__global__ void k_vset_field(MemberDev* members, int mi, int model, const double* rhoc,
                             const double* tc, const double* bin_par, const int* bin_flags,
                             double vset_fac, int* nfail, int maxit) {
  const MemberDev& m = members[mi];
  const int nx = m.nx, ny = m.ny, nz = m.nz, nb = m.nb;
  const long long cx = nx + 1, cy = ny + 1;
  const long long tot = (long long)(nz + 1) * ny * nx * nb;
  double* vs = const_cast<double*>(m.vs);
  GRID_STRIDE(e, tot) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    t /= ny;
    int k = (int)(t % (nz + 1));
    int b = (int)(t / (nz + 1));
#define CO(a, ii, jj) a[(ii) + cx * ((jj) + cy * (long long)k)]
    double rhoa = 0.25 * (CO(rhoc, i, j) + CO(rhoc, i + 1, j) + CO(rhoc, i + 1, j + 1) + CO(rhoc, i, j + 1));
    double ta = 0.25 * (CO(tc, i, j) + CO(tc, i + 1, j) + CO(tc, i + 1, j + 1) + CO(tc, i, j + 1));
#undef CO
    double visa = 1.827e-5 * ((291.15 + 120.0) / (ta + 120.0)) * pow(ta / 291.15, 1.5);
    int fl = bin_flags[b];
    double v = 0.0;
    if ((fl & 0xff) != 2) {
      int it;
      int f = vset_point_dev(bin_par[3 * b], bin_par[3 * b + 1], bin_par[3 * b + 2], rhoa, visa,
                             model, &v, &it, maxit);
      if (f) atomicAdd(nfail, 1);
    }
    if (fl >> 8) v = vset_fac * v;
    v = v / m.hm3[i + (long long)nx * j];
    vs[(((long long)b * (nz + 1) + k) * ny + j) * nx + i] = v;
  }
}
void launch_vset_field(MemberDev* members, int mi, int model, const double* rhoc,
                       const double* tc, const double* bin_par, const int* bin_flags,
                       double vset_fac, int* nfail, cudaStream_t st) {
  k_vset_field<<<1184, 128, 0, st>>>(members, mi, model, rhoc, tc, bin_par, bin_flags, vset_fac,
                                     nfail, vset_maxit());
}

// ---- finite scan: diagnostics of NaN/Inf-poisoned inputs --------------------
// Sets bit `bit` of *mask when any of the n values is NaN or infinite.
template <class T>
__global__ void k_nonfinite(const T* __restrict__ p, long long n, int bit, unsigned int* mask) {
  bool bad = false;
  GRID_STRIDE(e, n) {
    if (!isfinite(p[e])) bad = true;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(mask, 1u << bit);
}
void launch_nonfinite(const double* p, long long n, int bit, unsigned int* mask, cudaStream_t st) {
  if (p && n > 0) k_nonfinite<<<592, 256, 0, st>>>(p, n, bit, mask);
}
void launch_nonfinite(const float* p, long long n, int bit, unsigned int* mask, cudaStream_t st) {
  if (p && n > 0) k_nonfinite<<<592, 256, 0, st>>>(p, n, bit, mask);
}

}  // namespace f3d

namespace f3d {
// ---- ADS_solve_1D (mod_ADS.F90:820-1053) -----------------------------------
// One pencil of n cells in one block: the boundary codes set the ghost cells
// (-1 periodic when the face velocity enters, 0 as given, 1 Dirichlet, 2
// free flow: Dirichlet on inflow, zero gradient on outflow), then RK4 with
// four KT_RHS evaluations (:1057-1120) whose limiter, reconstruction and
// fluxes are computed cell-parallel between block barriers, in the
// reference's operation order (this file is compiled with --fmad=false; the
// divisions are IEEE divisions).  The serial reference's halo swaps are
// no-ops, so the ghosts stay as set.  Arrays (device) with the reference
// offsets: c, dxp, k from ips-2; dxb, u from ibs-1; w (scratch) holds
// c0 (n+4), r (n+4), cl and cr (n+3 each) and k1..k4 (n each).
__device__ void kt_rhs_block(int n, int lim, const double* c, const double* dxp, const double* dxb,
                             const double* u, const double* k, double* r, double* cl, double* cr,
                             double* rhs, double* flux) {
  for (int p = -1 + (int)threadIdx.x; p <= n; p += blockDim.x) {
    const double cm = c[p + 1], c0 = c[p + 2], cp = c[p + 3];
    double rv;
    if (fabs(cp - c0) < kEps) {
      rv = (lim == 1) ? 1.0 : ((fabs(c0 - cm) < kEps) ? 0.0 : (lim == 2 ? 2.0 : 1.5));
    } else {
      const double rr = (c0 - cm) / (cp - c0);
      if (lim == 1) rv = fmax(0.0, fmin(1.0, rr));
      else if (lim == 2) rv = fmax(fmax(0.0, fmin(2.0 * rr, 1.0)), fmin(rr, 2.0));
      else rv = 1.5 * (rr * rr + rr) / (rr * rr + rr + 1.0);
    }
    r[p + 2] = rv;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    r[0] = r[1];          // r(ips-2) = r(ips-1)
    r[n + 3] = r[n + 2];  // r(ipe+2) = r(ipe+1)
  }
  __syncthreads();
  for (int p = -1 + (int)threadIdx.x; p <= n; p += blockDim.x) {
    cr[p + 1] = c[p + 2] - 0.5 * r[p + 2] * (c[p + 3] - c[p + 2]);
    cl[p + 1] = c[p + 1] + 0.5 * r[p + 1] * (c[p + 2] - c[p + 1]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double ui = u[i + 1], up = u[i + 2];
    const double F_m = 0.5 * (cl[i + 1] * ui + cr[i + 1] * ui) - 0.5 * fabs(ui) * (cr[i + 1] - cl[i + 1]);
    const double F_p = 0.5 * (cl[i + 2] * up + cr[i + 2] * up) - 0.5 * fabs(up) * (cr[i + 2] - cl[i + 2]);
    const double P_m = 0.5 * (k[i + 2] + k[i + 1]) * (c[i + 2] - c[i + 1]) / dxp[i + 1];
    const double P_p = 0.5 * (k[i + 3] + k[i + 2]) * (c[i + 3] - c[i + 2]) / dxp[i + 2];
    rhs[i] = -1.0 * (F_p - F_m) / dxb[i + 1] + (P_p - P_m) / dxb[i + 1];
    if (i == 0) flux[0] = F_m + P_m;
    if (i == n - 1) flux[1] = F_p + P_p;
  }
  __syncthreads();
}

__global__ void k_ads_solve_1d(int n, int lim, double* c, const double* dxp, const double* dxb,
                               const double* u, const double* k, double dt, double bv0, double bv1,
                               int bc0, int bc1, double* flux, double* w) {
  double* c0 = w;
  double* r = c0 + (n + 4);
  double* cl = r + (n + 4);
  double* cr = cl + (n + 3);
  double* k1 = cr + (n + 3);
  double* k2 = k1 + n;
  double* k3 = k2 + n;
  double* k4 = k3 + n;
  if (threadIdx.x == 0) {  // boundary conditions (:880-942)
    const double uL = u[1], uR = u[n + 1];
    if (bc0 == -1) {
      if (uL > 0.0) { c[1] = c[n + 1]; c[0] = c[n]; c[n + 2] = c[2]; c[n + 3] = c[3]; }
    } else if (bc0 == 1) {
      c[1] = 2.0 * bv0 - c[2]; c[0] = c[1];
    } else if (bc0 == 2) {
      if (uL > 0.0) c[1] = 2.0 * bv0 - c[2]; else c[1] = c[2];
      c[0] = c[1];
    }
    if (bc1 == -1) {
      if (uR < 0.0) { c[1] = c[n + 1]; c[0] = c[n]; c[n + 2] = c[2]; c[n + 3] = c[3]; }
    } else if (bc1 == 1) {
      c[n + 2] = 2.0 * bv1 - c[n + 1]; c[n + 3] = c[n + 2];
    } else if (bc1 == 2) {
      if (uR < 0.0) c[n + 2] = 2.0 * bv1 - c[n + 1]; else c[n + 2] = c[n + 1];
      c[n + 3] = c[n + 2];
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < n + 4; p += blockDim.x) c0[p] = c[p];  // with the halos (:946)
  __syncthreads();
  kt_rhs_block(n, lim, c0, dxp, dxb, u, k, r, cl, cr, k1, flux);
  for (int i = threadIdx.x; i < n; i += blockDim.x) c0[i + 2] = c[i + 2] + 0.5 * dt * k1[i];
  __syncthreads();
  kt_rhs_block(n, lim, c0, dxp, dxb, u, k, r, cl, cr, k2, flux);
  for (int i = threadIdx.x; i < n; i += blockDim.x) c0[i + 2] = c[i + 2] + 0.5 * dt * k2[i];
  __syncthreads();
  kt_rhs_block(n, lim, c0, dxp, dxb, u, k, r, cl, cr, k3, flux);
  for (int i = threadIdx.x; i < n; i += blockDim.x) c0[i + 2] = c[i + 2] + dt * k3[i];
  __syncthreads();
  kt_rhs_block(n, lim, c0, dxp, dxb, u, k, r, cl, cr, k4, flux);
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    c[i + 2] = c[i + 2] + dt * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]) / 6.0;
}

void launch_ads_solve_1d(int n, int lim, double* c, const double* dxp, const double* dxb,
                         const double* u, const double* k, double dt, const double bvalue[2],
                         const int bcode[2], double* flux, double* work, cudaStream_t st) {
  k_ads_solve_1d<<<1, 256, 0, st>>>(n, lim, c, dxp, dxb, u, k, dt, bvalue[0], bvalue[1], bcode[0],
                                    bcode[1], flux, work);
}
}  // namespace f3d
