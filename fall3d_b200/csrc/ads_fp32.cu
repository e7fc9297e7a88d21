// ads_fp32.cu -- precision form of the ADS sweeps: FP32 state and stencil
// arithmetic, FP64 ground deposit and boundary-flux sums.
//
// Same single-pass pipelined RK march as the FP64 form (see ads_fp64.cu),
// rewritten for throughput:
//  * the limiter is applied division-free as phi(r)*dc, which is what the
//    reconstruction c_l/c_r actually uses (c_r = c - 0.5 phi(r) dc);
//    for superbee with dc > 0 this is max(0, min(2 dm, dc), min(dm, 2 dc))
//    and the mirrored form for dc < 0, with the reference's |dc| < 1e-12
//    special cases (mod_ADS.F90:1170-1183) kept;
//  * diffusion enters through a per-face coefficient kf = 0.5 (k_i + k_i-1) /
//    dxp_i-1 prepared once per meteo update, and 1/dxb per cell;
//  * stage updates use FMA.
#include <cuda_runtime.h>

#include "f3d_common.cuh"

namespace f3d {

constexpr float kEpsF = 1e-12f;

// 0.5 * phi(r) * d0 with r = d1/d0  (d1 = c(i)-c(i-1), d0 = c(i+1)-c(i))
template <int LIM>
__device__ __forceinline__ float half_phid(float d1, float d0) {
  float pd;
  if (LIM == 1) {  // minmod, mod_ADS.F90:1139-1147
    float lo = fminf(d0, d1), hi = fmaxf(d0, d1);
    pd = (d0 > 0.f) ? fmaxf(0.f, lo) : fminf(0.f, hi);
    if (fabsf(d0) < kEpsF) pd = d0;
  } else if (LIM == 2) {  // superbee, mod_ADS.F90:1170-1183
    float t1 = 2.f * d1, t2 = 2.f * d0;
    float pos = fmaxf(fmaxf(0.f, fminf(t1, d0)), fminf(d1, t2));
    float neg = fminf(fminf(0.f, fmaxf(t1, d0)), fmaxf(d1, t2));
    pd = (d0 > 0.f) ? pos : neg;
    if (fabsf(d0) < kEpsF) pd = (fabsf(d1) < kEpsF) ? 0.f : t2;
  } else {  // ospre, mod_ADS.F90:1206-1219: 1.5 (r^2+r)/(r^2+r+1) * d0
    float num = d1 * (d1 + d0);
    float den = fmaf(d1, d1 + d0, d0 * d0);
    pd = 1.5f * num * __frcp_rn(den) * d0;
    if (fabsf(d0) < kEpsF) pd = (fabsf(d1) < kEpsF) ? 0.f : 1.5f * d0;
  }
  return 0.5f * pd;
}

struct Stage32 {
  float a1, a2, d1, h2, G1;
};

struct Pencil32 {
  int n;
  long long c_off, c_stride;
  const float* vel;
  long long vstride;
  const float* vsub;
  const float* kf;  // face coefficient, face f at kf[f * vstride]
  const float* rdxb;
};

__device__ __forceinline__ float face_vel32(const Pencil32& P, int f) {
  float v = __ldg(P.vel + f * P.vstride);
  if (P.vsub) v = v - __ldg(P.vsub + f * P.vstride);
  return v;
}

template <int LIM>
__device__ __forceinline__ bool arrive32(Stage32& s, const Pencil32& P, int q, float a0,
                                         float& rhs, float& face_flux) {
  float d0 = a0 - s.a1;
  float h1 = half_phid<LIM>(s.d1, d0);
  bool produced = false;
  if (q >= 1) {
    int f = q - 1;
    float u = face_vel32(P, f);
    float kf = __ldg(P.kf + f * P.vstride);
    float cl = s.a2 + s.h2;
    float cr = s.a1 - h1;
    float F = 0.5f * fmaf(-fabsf(u), cr - cl, u * (cl + cr));
    float Pd = kf * s.d1;
    face_flux = F + Pd;
    float G0 = Pd - F;
    if (q >= 2) {
      rhs = (G0 - s.G1) * __ldg(P.rdxb + (q - 2));
      produced = true;
    }
    s.G1 = G0;
  }
  s.a2 = s.a1;
  s.a1 = a0;
  s.d1 = d0;
  s.h2 = h1;
  return produced;
}

template <int LIM, int TM>
__device__ __forceinline__ void march32(float* __restrict__ c, const Pencil32& P, float dt,
                                        float& flux_lo, float& flux_hi) {
  const int n = P.n;
  float* cp = c + P.c_off;
  const long long cs = P.c_stride;
  float c_first = cp[0];
  float uL = face_vel32(P, 0), uR = face_vel32(P, n);
  float gL = (uL > 0.f) ? -c_first : c_first;
  float gR = 0.f;
  Stage32 S1 = {0, 0, 0, 0, 0}, S2 = S1, S3 = S1, S4 = S1;
  float ch0 = 0, ch1 = 0, ch2 = 0, ch3 = 0, ch4 = 0, ch5 = 0, ch6 = 0;
  float nh0 = 0, nh1 = 0, nh2 = 0, nh3 = 0, nh4 = 0, nh5 = 0, nh6 = 0;
  float ff = 0.f;
  const float hdt = 0.5f * dt, dt3 = dt * (1.f / 3.f), dt6 = dt * (1.f / 6.f);
  if constexpr (TM == 1) {
    for (int t = -2; t <= n + 1; ++t) {
      float a = (t < 0) ? gL : (t < n) ? cp[t * cs] : gR;
      ch2 = ch1; ch1 = ch0; ch0 = a;
      if (t == n - 1) gR = (uR < 0.f) ? -a : a;
      float k1;
      if (arrive32<LIM>(S1, P, t, a, k1, ff)) cp[(t - 2) * cs] = fmaf(dt, k1, ch2);
      if (t == 1) flux_lo = ff;
      if (t == n + 1) flux_hi = ff;
    }
  } else {
  // prefetch distance 1: the load for t+1 is issued before stage work at t
  float next = c_first;
#pragma unroll 1
  for (int t = -2; t <= n + 7; ++t) {
    ch6 = ch5; ch5 = ch4; ch4 = ch3; ch3 = ch2; ch2 = ch1; ch1 = ch0;
    nh6 = nh5; nh5 = nh4; nh4 = nh3; nh3 = nh2; nh2 = nh1; nh1 = nh0;
    float k1 = 0.f, k2 = 0.f, k3 = 0.f, k4;
    if (t <= n + 1) {
      float a = (t < 0) ? gL : (t < n) ? next : gR;
      if (t + 1 >= 0 && t + 1 < n) next = cp[(t + 1) * cs];
      ch0 = a;
      if (t == n - 1) gR = (uR < 0.f) ? -a : a;
      arrive32<LIM>(S1, P, t, a, k1, ff);
    }
    int q = t - 2;
    if (q >= -2 && q <= n + 1) {
      float a = gL;
      if (q >= n) a = gR;
      else if (q >= 0) {
        a = fmaf(hdt, k1, ch2);
        nh0 = fmaf(dt6, k1, ch2);
      }
      arrive32<LIM>(S2, P, q, a, k2, ff);
    }
    q = t - 4;
    if (q >= -2 && q <= n + 1) {
      float a = gL;
      if (q >= n) a = gR;
      else if (q >= 0) {
        a = fmaf(hdt, k2, ch4);
        nh2 = fmaf(dt3, k2, nh2);
      }
      arrive32<LIM>(S3, P, q, a, k3, ff);
    }
    q = t - 6;
    if (q >= -2 && q <= n + 1) {
      float a = gL;
      if (q >= n) a = gR;
      else if (q >= 0) {
        a = fmaf(dt, k3, ch6);
        nh4 = fmaf(dt3, k3, nh4);
      }
      if (arrive32<LIM>(S4, P, q, a, k4, ff)) cp[(q - 2) * cs] = fmaf(dt6, k4, nh6);
      if (q == 1) flux_lo = ff;
      if (q == n + 1) flux_hi = ff;
    }
  }
  }
}

__device__ __forceinline__ void block_reduce2_f64(double a, double b, double* out) {
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
__global__ void __launch_bounds__(128) k_sweep32(const MemberDev* __restrict__ members,
                                                 const WorkItem* __restrict__ work) {
  const WorkItem w = work[blockIdx.x];
  const MemberDev& m = members[w.member];
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  const long long npen = (DIR == DIR_X) ? (long long)ny * nz * m.nb
                         : (DIR == DIR_Y) ? (long long)nx * nz * m.nb
                                          : (long long)nx * ny * m.nb;
  const long long pen = (long long)w.pen0 + threadIdx.x;
  double clo = 0.0, chi = 0.0;
  if (pen < npen) {
    Pencil32 P;
    double area;
    const double dt = m.dt;
    int i = 0, j = 0, b = 0;
    if (DIR == DIR_X) {
      j = (int)(pen % ny);
      long long t = pen / ny;
      int k = (int)(t % nz);
      b = (int)(t / nz);
      P.n = nx;
      P.c_off = (((long long)b * nz + k) * ny + j) * nx;
      P.c_stride = 1;
      long long fo = (long long)k * (nx + 1) * ny + j;
      P.vel = m.ucur32 + fo;
      P.kf = m.kfx + fo;
      P.vstride = ny;
      P.vsub = nullptr;
      P.rdxb = m.rdx1b32;
      area = m.dx3b[k + 1] * m.dx2b[j + 1];
    } else if (DIR == DIR_Y) {
      i = (int)(pen % nx);
      long long t = pen / nx;
      int k = (int)(t % nz);
      b = (int)(t / nz);
      P.n = ny;
      P.c_off = ((long long)b * nz + k) * ny * (long long)nx + i;
      P.c_stride = nx;
      long long fo = (long long)k * (ny + 1) * nx + i;
      P.vel = m.vcur32 + fo;
      P.kf = m.kfy + fo;
      P.vstride = nx;
      P.vsub = nullptr;
      P.rdxb = m.rdx2b32;
      area = m.dx3b[k + 1] * m.dx1b[i + 1];
    } else {
      i = (int)(pen % nx);
      long long t = pen / nx;
      j = (int)(t % ny);
      b = (int)(t / ny);
      P.n = nz;
      P.c_off = (long long)b * nz * ny * nx + (long long)j * nx + i;
      P.c_stride = (long long)nx * ny;
      long long fo = (long long)j * nx + i;
      P.vel = m.wcur32 + fo;
      P.kf = m.kfz + fo;
      P.vstride = (long long)nx * ny;
      P.vsub = m.vs32 + (long long)b * (nz + 1) * ny * nx + fo;
      P.rdxb = m.rdx3b32;
      area = m.dx2b[j + 1] * m.dx1b[i + 1];
    }
    float lo = 0.f, hi = 0.f;
    march32<LIM, TM>(m.c32, P, (float)dt, lo, hi);
    clo = (double)lo * area * dt;
    chi = (double)hi * area * dt;
    if (DIR == DIR_Z) {
      double* a = m.acum + ((long long)b * ny + j) * nx + i;
      *a = *a + fabs((double)lo) * dt;
    }
  }
  block_reduce2_f64(clo, chi, m.flux_part + 2 * (long long)w.slot);
}

template <int DIR>
static void launch_dir32(int lim, int tm, const MemberDev* members, const WorkItem* work,
                         int nblocks, cudaStream_t st) {
  dim3 g(nblocks), b(128);
#define F3D_L(L, T) k_sweep32<DIR, L, T><<<g, b, 0, st>>>(members, work)
  if (tm == 1) {
    if (lim == 1) F3D_L(1, 1); else if (lim == 2) F3D_L(2, 1); else F3D_L(3, 1);
  } else {
    if (lim == 1) F3D_L(1, 2); else if (lim == 2) F3D_L(2, 2); else F3D_L(3, 2);
  }
#undef F3D_L
}

void launch_sweep32(int dir, int lim, int tm, const MemberDev* members, const WorkItem* work,
                    int nblocks, cudaStream_t st) {
  if (nblocks <= 0) return;
  if (dir == DIR_X) launch_dir32<DIR_X>(lim, tm, members, work, nblocks, st);
  else if (dir == DIR_Y) launch_dir32<DIR_Y>(lim, tm, members, work, nblocks, st);
  else launch_dir32<DIR_Z>(lim, tm, members, work, nblocks, st);
}

// current winds in FP32, scaled by the member's wind factor (u, v only)
__global__ void k_prep32(const MemberDev* __restrict__ members, const int* __restrict__ blk_member,
                         const int* __restrict__ blk_first, int mask) {
  const int mi = blk_member[blockIdx.x];
  const MemberDev& m = members[mi];
  const long long nu = (long long)(m.nx + 1) * m.ny * m.nz;
  const long long nv = (long long)(m.ny + 1) * m.nx * m.nz;
  const long long nw = (long long)(m.nz + 1) * m.nx * m.ny;
  const float s = (float)m.stime, s1 = 1.f - s;
  long long q = (long long)(blockIdx.x - blk_first[mi]) * blockDim.x + threadIdx.x;
  if (q < nu) {
    if (mask & 1) m.ucur32[q] = m.wfac * fmaf(s1, m.ux32[0][q], s * m.ux32[1][q]);
    return;
  }
  q -= nu;
  if (q < nv) {
    if (mask & 2) m.vcur32[q] = m.wfac * fmaf(s1, m.vy32[0][q], s * m.vy32[1][q]);
    return;
  }
  q -= nv;
  if (q < nw && (mask & 4)) m.wcur32[q] = fmaf(s1, m.wz32[0][q], s * m.wz32[1][q]);
}

void launch_prep32(const MemberDev* members, const int* blk_member, const int* blk_first,
                   int nblocks, int mask, cudaStream_t st) {
  if (nblocks > 0) k_prep32<<<nblocks, 256, 0, st>>>(members, blk_member, blk_first, mask);
}

__global__ void k_source32(const MemberDev* __restrict__ members, int nmembers) {
  for (int mi = blockIdx.y; mi < nmembers; mi += gridDim.y) {
    const MemberDev& m = members[mi];
    const long long tot = (long long)m.nsrc * m.nb;
    const long long ncell = (long long)m.nx * m.ny * m.nz;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
      int q = (int)(e / m.nb), b = (int)(e % m.nb);
      float* cc = m.c32 + (long long)b * ncell + m.src_cell[q];
      *cc = (float)((double)*cc + m.dt * m.src_s[(long long)q * m.nb + b] / m.src_vol[q]);
    }
  }
}

void launch_source32(const MemberDev* members, int nmembers, cudaStream_t st) {
  dim3 g(8, nmembers < 65535 ? nmembers : 65535);
  k_source32<<<g, 128, 0, st>>>(members, nmembers);
}

// FP32 field preparation from the FP64 meteo arrays (once per meteo update):
// winds, settling velocity and the face diffusion coefficients
//   kf(f) = 0.5 (k(f) + k(f-1)) / dxp(f-1)         (KT_RHS P term, :1111)
__global__ void k_fp32_fields(MemberDev* members, int mi) {
  MemberDev& m = members[mi];
  const int nx = m.nx, ny = m.ny, nz = m.nz, nb = m.nb;
  const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)(ny + 1) * nx * nz,
                  nw = (long long)(nz + 1) * nx * ny;
  const long long nvs = (long long)nb * nw;
  const long long tot = 2 * nu + 2 * nv + 2 * nw + nu + nv + nw + nvs;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long q = e;
    if (q < 2 * nu) { const_cast<float*>(m.ux32[0])[q] = (float)m.ux[0][q]; continue; }
    q -= 2 * nu;
    if (q < 2 * nv) { const_cast<float*>(m.vy32[0])[q] = (float)m.vy[0][q]; continue; }
    q -= 2 * nv;
    if (q < 2 * nw) { const_cast<float*>(m.wz32[0])[q] = (float)m.wz[0][q]; continue; }
    q -= 2 * nw;
    if (q < nu) {  // x faces: [k][f][j]
      int j = (int)(q % ny);
      long long t = q / ny;
      int f = (int)(t % (nx + 1));
      int k = (int)(t / (nx + 1));
      double kA = m.k1x[((long long)k * (nx + 2) + (f + 1)) * ny + j];
      double kB = m.k1x[((long long)k * (nx + 2) + f) * ny + j];
      const_cast<float*>(m.kfx)[q] = (float)(0.5 * (kA + kB) / m.dx1p[f + 1]);
      continue;
    }
    q -= nu;
    if (q < nv) {  // y faces: [k][f][i]
      int i = (int)(q % nx);
      long long t = q / nx;
      int f = (int)(t % (ny + 1));
      int k = (int)(t / (ny + 1));
      double kA = m.k2y[((long long)k * (ny + 2) + (f + 1)) * nx + i];
      double kB = m.k2y[((long long)k * (ny + 2) + f) * nx + i];
      const_cast<float*>(m.kfy)[q] = (float)(0.5 * (kA + kB) / m.dx2p[f + 1]);
      continue;
    }
    q -= nv;
    if (q < nw) {  // z faces: [f][j][i]
      int i = (int)(q % nx);
      long long t = q / nx;
      int j = (int)(t % ny);
      int f = (int)(t / ny);
      double kA = m.k3z[((long long)(f + 1) * ny + j) * nx + i];
      double kB = m.k3z[((long long)f * ny + j) * nx + i];
      const_cast<float*>(m.kfz)[q] = (float)(0.5 * (kA + kB) / m.dx3p[f + 1]);
      continue;
    }
    q -= nw;
    const_cast<float*>(m.vs32)[q] = (float)m.vs[q];
  }
}

void launch_fp32_fields(MemberDev* members, int mi, cudaStream_t st) {
  k_fp32_fields<<<2048, 256, 0, st>>>(members, mi);
}

}  // namespace f3d
