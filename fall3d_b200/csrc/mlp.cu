// mlp.cu -- learned settling velocity: a 5 -> 64 -> 64 -> 1 tanh network that
// stands in for the fixed-point drag-law solve of phys_get_vset_point
// (mod_Phys.F90:757-954) inside phys_get_vset (mod_Phys.F90:673-740).
//
//   * samples: uniform draws over the training box (the validity envelope
//     widened by a margin), labelled on the device by the model's own FP64
//     iteration (vset_point_dev, the routine the iterative path runs);
//   * training: hand-written FP32 forward/backward kernel over a minibatch,
//     one partial gradient per block reduced in a fixed order, Adam with bias
//     correction and a cosine learning rate, replayed from a CUDA graph;
//   * inference: tcgen05 tensor-core kernel.  Layer 1 (5 -> 64) and layer 3
//     (64 -> 1) run in FP32 on the CUDA cores; layer 2 (64 x 64) runs as
//     three BF16 UMMAs (hi*hi + hi*lo + lo*hi of the split operands) with an
//     FP32 accumulator in tensor memory, which keeps FP32-level accuracy;
//   * cells whose air density or viscosity, or bins whose diameter, density
//     or sphericity, lie outside the envelope take the iteration itself, so
//     they get the iterative path's exact bits.
//
// Network input (features) and output (target), all FP32 on the device:
//   lnAr = ln(g d^3 rhop rhoa / mu^2)             f0 = (lnAr - c) / s
//   f1 = 2 (-log10 psi)^0.5743 / sgmax - 1        (Ganser's shape exponent)
//   f2, f3, f4 = psi, ln d, ln mu mapped linearly to [-1, 1] over the envelope
//   y = (ln Re - ln(Ar K1 / 18)) / 4,  K1 = 3 / (1 + 2 / sqrt(psi)),
// i.e. the log ratio of the particle Reynolds number to its Stokes value, so
//   ln v = 4 y + ln(g d^2 rhop K1 / 18) - ln mu.
//
// Compiled with --fmad=false so that the fallback iteration keeps the
// reference's separately rounded operations; the network arithmetic asks for
// fused multiply-adds explicitly.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <math.h>
#include <string.h>
#include <mutex>
#include <vector>

#include "f3d_common.cuh"
#include "step_dev.cuh"
#include "vset.cuh"

namespace f3d {

int set_error_msg(const char* fmt, ...);

// ---- parameter layout (row-major weights, PyTorch Linear convention) ---------
constexpr int kIn = 5, kHid = 64;
constexpr int kOffW1 = 0;                       // W1[j][i], 64 x 5
constexpr int kOffB1 = kOffW1 + kHid * kIn;     // 320
constexpr int kOffW2 = kOffB1 + kHid;           // 384: W2[j][k], 64 x 64
constexpr int kOffB2 = kOffW2 + kHid * kHid;    // 4480
constexpr int kOffW3 = kOffB2 + kHid;           // 4544
constexpr int kOffB3 = kOffW3 + kHid;           // 4608
constexpr int kNParam = kOffB3 + 1;             // 4609
constexpr int kPartStride = 4612;               // partial gradient + loss, padded
constexpr int kTrainThreads = 128;              // samples per training block
constexpr int kRecF = 8;                        // floats per sample record

// ---- counter-based random numbers --------------------------------------------
// SplitMix64 finaliser (Steele, Lea & Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014) applied to (seed, stream, index).
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b) {
  return mix64(mix64(mix64(seed) ^ a) ^ (b * 0xD1B54A32D192ED03ull));
}
// Uniform double in [0, 1) from the top 53 bits.
__host__ __device__ __forceinline__ double u01(uint64_t h) {
  return (double)(h >> 11) * 0x1p-53;
}

// tanh(x) = 1 - 2 / (exp(2x) + 1): absolute error a few 1e-7, saturates to
// +-1 without overflow (exp -> inf gives 1, exp -> 0 gives -1).
__device__ __forceinline__ float tanh_net(float x) {
  const float e = __expf(2.0f * x);
  return 1.0f - __fdividef(2.0f, e + 1.0f);
}

// ---- envelope and feature normalisation ---------------------------------------
// Coordinates: 0 diameter, 1 particle density, 2 sphericity, 3 air density,
// 4 air viscosity.
struct MlpNorm {
  double lo[5], hi[5];      // validity envelope
  double tlo[5], thi[5];    // training box (envelope widened by the margin)
  float lar_c, lar_sinv;    // f0 = (lnAr - lar_c) * lar_sinv
  float sg_scale;           // f1 = sg * sg_scale - 1
  float psi_lo, psi_sinv;   // f2 = (psi - psi_lo) * psi_sinv - 1
  float lnd_lo, lnd_sinv;   // f3
  float lnmu_lo, lnmu_sinv; // f4
};

__host__ __device__ __forceinline__ double sg_of(double psi) {
  return pow(-log10(psi), 0.5743);
}

// Host: normalisation constants from the envelope.
static MlpNorm make_norm(const double* env, double margin) {
  MlpNorm n;
  for (int c = 0; c < 5; ++c) {
    n.lo[c] = env[2 * c];
    n.hi[c] = env[2 * c + 1];
  }
  // training box: diameter widened in log space, the others linearly;
  // sphericity is capped at 1.
  const double fw = exp(3.0 * margin);
  n.tlo[0] = n.lo[0] / fw;
  n.thi[0] = n.hi[0] * fw;
  for (int c = 1; c < 5; ++c) {
    n.tlo[c] = n.lo[c] * (1.0 - margin);
    n.thi[c] = n.hi[c] * (1.0 + margin);
  }
  if (n.thi[2] > 1.0) n.thi[2] = 1.0;
  const double lar_min = log(9.81) + 3 * log(n.lo[0]) + log(n.lo[1]) + log(n.lo[3]) - 2 * log(n.hi[4]);
  const double lar_max = log(9.81) + 3 * log(n.hi[0]) + log(n.hi[1]) + log(n.hi[3]) - 2 * log(n.lo[4]);
  n.lar_c = (float)(0.5 * (lar_min + lar_max));
  n.lar_sinv = (float)(2.0 / (lar_max - lar_min));
  const double sgmax = sg_of(n.lo[2]);
  n.sg_scale = (float)(sgmax > 0 ? 2.0 / sgmax : 0.0);
  n.psi_lo = (float)n.lo[2];
  n.psi_sinv = (float)(n.hi[2] > n.lo[2] ? 2.0 / (n.hi[2] - n.lo[2]) : 0.0);
  n.lnd_lo = (float)log(n.lo[0]);
  n.lnd_sinv = (float)(2.0 / (log(n.hi[0]) - log(n.lo[0])));
  n.lnmu_lo = (float)log(n.lo[4]);
  n.lnmu_sinv = (float)(2.0 / (log(n.hi[4]) - log(n.lo[4])));
  return n;
}

// Per-bin constants of the features and of the output transform.
struct MlpBin {
  double d, rhop, psi;
  VsetConst k;
  float lar0m;   // ln(g d^3 rhop) - lar_c
  float f1, f2, f3;
  float cout;    // ln(g d^2 rhop K1 / 18)
  int inside;    // d, rhop, psi inside the envelope
  int flags;     // category | aggregate << 8
  int pad;
};

__host__ __device__ __forceinline__ double ln_k1_18(double psi) {
  return log(3.0 / (1.0 + 2.0 / sqrt(psi))) - log(18.0);
}

// Features and the output constant of one (d, rhop, psi, rhoa, mu) point, in
// FP64 (sample generation, gradient entry, host checks).
__host__ __device__ __forceinline__ void point_features(const MlpNorm& n, double d, double rhop,
                                                         double psi, double rhoa, double mu,
                                                         float* f, double* cout) {
  const double lnd = log(d), lnmu = log(mu);
  const double lar = log(9.81) + 3.0 * lnd + log(rhop) + log(rhoa) - 2.0 * lnmu;
  f[0] = (float)((lar - (double)n.lar_c) * (double)n.lar_sinv);
  f[1] = (float)(sg_of(psi) * (double)n.sg_scale - 1.0);
  f[2] = (float)((psi - (double)n.psi_lo) * (double)n.psi_sinv - 1.0);
  f[3] = (float)((lnd - (double)n.lnd_lo) * (double)n.lnd_sinv - 1.0);
  f[4] = (float)((lnmu - (double)n.lnmu_lo) * (double)n.lnmu_sinv - 1.0);
  *cout = log(9.81) + 2.0 * lnd + log(rhop) + ln_k1_18(psi);
}

// ---- sample generation ------------------------------------------------------
// Record q: raw[5 q .. 5 q + 4] = (d, rhop, psi, rhoa, mu) in FP64;
// rec[8 q .. 8 q + 7] = (f0..f4, y, 0, 0) in FP32, y = NaN if the iteration
// did not converge (such samples carry no weight in training).
__global__ void k_mlp_samples(MlpNorm n, int model, long long ns, uint64_t seed, double* raw,
                              float* rec, int* nfail) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ns;
       q += (long long)gridDim.x * blockDim.x) {
    double x[5];
    for (int c = 0; c < 5; ++c) {
      const double u = u01(hash3(seed, (uint64_t)q, (uint64_t)c));
      if (c == 0) x[c] = exp(log(n.tlo[0]) + u * (log(n.thi[0]) - log(n.tlo[0])));
      else x[c] = n.tlo[c] + u * (n.thi[c] - n.tlo[c]);
    }
    double v;
    int it;
    const int fl = vset_point_dev(x[0], x[1], x[2], x[3], x[4], model, &v, &it);
    float f[5];
    double cout;
    point_features(n, x[0], x[1], x[2], x[3], x[4], f, &cout);
    float* r = rec + kRecF * q;
    for (int c = 0; c < 5; ++c) {
      r[c] = f[c];
      raw[5 * q + c] = x[c];
    }
    r[5] = fl ? __int_as_float(0x7fc00000) : (float)(0.25 * (log(v) - cout + log(x[4])));
    r[6] = 0.0f;
    r[7] = 0.0f;
    if (fl) atomicAdd(nfail, 1);
  }
}

// ---- training: forward + backward of one 128-sample block -------------------
// Shared memory (floats): parameters, then per-sample rows (stride kLd) of
// h1, h2, dL/dz2, dL/dz1, the inputs and dL/dy.  Each block writes its partial
// gradient of the mean squared error (and its partial loss) to
// part[blockIdx.x * kPartStride + p]; the sums over blocks are taken in block
// order by the reducer, so training is deterministic.
constexpr int kLd = 68;
constexpr int kTrainSmemFloats = kPartStride + 4 * kTrainThreads * kLd + kTrainThreads * 8 + 2 * kTrainThreads;
constexpr size_t kTrainSmem = sizeof(float) * kTrainSmemFloats;

// FIXED = true: sample s of block b is record b*128+s (valid if < nvalid).
// FIXED = false: the record index is drawn from (seed, step, slot).
template <bool FIXED>
__global__ void __launch_bounds__(kTrainThreads) k_mlp_train(const float* __restrict__ params,
                                                             const float* __restrict__ rec, long long ns,
                                                             uint64_t seed, const int* step_ctr,
                                                             float inv_batch, long long nvalid,
                                                             float* __restrict__ part) {
  extern __shared__ __align__(16) float sm[];
  float* sP = sm;
  float* sH1 = sP + kPartStride;
  float* sH2 = sH1 + kTrainThreads * kLd;
  float* sD2 = sH2 + kTrainThreads * kLd;
  float* sD1 = sD2 + kTrainThreads * kLd;
  float* sX = sD1 + kTrainThreads * kLd;
  float* sE = sX + kTrainThreads * 8;
  float* sL = sE + kTrainThreads;
  const int t = threadIdx.x;
  for (int p = t; p < kNParam; p += kTrainThreads) sP[p] = params[p];

  const long long slot = (long long)blockIdx.x * kTrainThreads + t;
  long long idx;
  bool valid;
  if (FIXED) {
    idx = slot;
    valid = slot < nvalid;
  } else {
    idx = (long long)(hash3(seed, (uint64_t)(*step_ctr), (uint64_t)slot) % (uint64_t)ns);
    valid = true;
  }
  float x[kIn], tgt = 0.0f;
  if (valid) {
    const float4 r0 = *reinterpret_cast<const float4*>(rec + kRecF * idx);
    const float4 r1 = *reinterpret_cast<const float4*>(rec + kRecF * idx + 4);
    x[0] = r0.x; x[1] = r0.y; x[2] = r0.z; x[3] = r0.w; x[4] = r1.x;
    tgt = r1.y;
    if (!(tgt == tgt)) valid = false;  // unlabelled sample
  }
  if (!valid) {
    for (int i = 0; i < kIn; ++i) x[i] = 0.0f;
    tgt = 0.0f;
  }
  __syncthreads();

  // layer 1
  float h1[kHid];
#pragma unroll
  for (int j = 0; j < kHid; ++j) {
    float z = sP[kOffB1 + j];
#pragma unroll
    for (int i = 0; i < kIn; ++i) z = __fmaf_rn(sP[kOffW1 + j * kIn + i], x[i], z);
    h1[j] = tanh_net(z);
  }
#pragma unroll
  for (int j = 0; j < kHid; j += 4)
    *reinterpret_cast<float4*>(sH1 + t * kLd + j) = make_float4(h1[j], h1[j + 1], h1[j + 2], h1[j + 3]);
  // layers 2 and 3
  float y = sP[kOffB3];
  for (int j = 0; j < kHid; ++j) {
    const float4* w = reinterpret_cast<const float4*>(sP + kOffW2 + j * kHid);
    float z0 = sP[kOffB2 + j], z1 = 0.0f;
#pragma unroll
    for (int q = 0; q < kHid / 4; q += 2) {
      const float4 a = w[q], b = w[q + 1];
      z0 = __fmaf_rn(a.x, h1[4 * q], z0);
      z1 = __fmaf_rn(a.y, h1[4 * q + 1], z1);
      z0 = __fmaf_rn(a.z, h1[4 * q + 2], z0);
      z1 = __fmaf_rn(a.w, h1[4 * q + 3], z1);
      z0 = __fmaf_rn(b.x, h1[4 * q + 4], z0);
      z1 = __fmaf_rn(b.y, h1[4 * q + 5], z1);
      z0 = __fmaf_rn(b.z, h1[4 * q + 6], z0);
      z1 = __fmaf_rn(b.w, h1[4 * q + 7], z1);
    }
    const float h2 = tanh_net(z0 + z1);
    sH2[t * kLd + j] = h2;
    y = __fmaf_rn(sP[kOffW3 + j], h2, y);
  }
  const float err = valid ? (y - tgt) : 0.0f;
  const float e = 2.0f * err * inv_batch;
  sE[t] = e;
  sL[t] = err * err * inv_batch;
  // backward through layers 3 and 2
  float dh1[kHid];
#pragma unroll
  for (int k = 0; k < kHid; ++k) dh1[k] = 0.0f;
  for (int j = 0; j < kHid; ++j) {
    const float h2 = sH2[t * kLd + j];
    const float dz = e * sP[kOffW3 + j] * (1.0f - h2 * h2);
    sD2[t * kLd + j] = dz;
    const float4* w = reinterpret_cast<const float4*>(sP + kOffW2 + j * kHid);
#pragma unroll
    for (int q = 0; q < kHid / 4; ++q) {
      const float4 a = w[q];
      dh1[4 * q] = __fmaf_rn(a.x, dz, dh1[4 * q]);
      dh1[4 * q + 1] = __fmaf_rn(a.y, dz, dh1[4 * q + 1]);
      dh1[4 * q + 2] = __fmaf_rn(a.z, dz, dh1[4 * q + 2]);
      dh1[4 * q + 3] = __fmaf_rn(a.w, dz, dh1[4 * q + 3]);
    }
  }
#pragma unroll
  for (int k = 0; k < kHid; k += 4) {
    float4 v;
    v.x = dh1[k] * (1.0f - h1[k] * h1[k]);
    v.y = dh1[k + 1] * (1.0f - h1[k + 1] * h1[k + 1]);
    v.z = dh1[k + 2] * (1.0f - h1[k + 2] * h1[k + 2]);
    v.w = dh1[k + 3] * (1.0f - h1[k + 3] * h1[k + 3]);
    *reinterpret_cast<float4*>(sD1 + t * kLd + k) = v;
  }
#pragma unroll
  for (int i = 0; i < kIn; ++i) sX[t * 8 + i] = x[i];
  __syncthreads();

  float* out = part + (size_t)blockIdx.x * kPartStride;
  // dW2[j][k] = sum_s dz2[s][j] h1[s][k]: a 4 x 8 tile per thread
  {
    const int jb = (t >> 3) * 4, kb = (t & 7) * 4;
    float acc[4][8];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) acc[a][b] = 0.0f;
    for (int s = 0; s < kTrainThreads; ++s) {
      const float4 dz = *reinterpret_cast<const float4*>(sD2 + s * kLd + jb);
      const float4 u = *reinterpret_cast<const float4*>(sH1 + s * kLd + kb);
      const float4 w = *reinterpret_cast<const float4*>(sH1 + s * kLd + 32 + kb);
      const float dzv[4] = {dz.x, dz.y, dz.z, dz.w};
      const float hv[8] = {u.x, u.y, u.z, u.w, w.x, w.y, w.z, w.w};
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = __fmaf_rn(dzv[a], hv[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int k = (b < 4) ? kb + b : 32 + kb + (b - 4);
        out[kOffW2 + (jb + a) * kHid + k] = acc[a][b];
      }
  }
  // the small sums: dW1 (320), db1, db2, dW3 (64 each), db3, loss
  for (int q = t; q < kHid * kIn + 3 * kHid + 2; q += kTrainThreads) {
    float acc = 0.0f;
    int dst;
    if (q < kHid * kIn) {
      const int j = q / kIn, i = q % kIn;
      for (int s = 0; s < kTrainThreads; ++s) acc = __fmaf_rn(sD1[s * kLd + j], sX[s * 8 + i], acc);
      dst = kOffW1 + q;
    } else if (q < kHid * kIn + kHid) {
      const int j = q - kHid * kIn;
      for (int s = 0; s < kTrainThreads; ++s) acc += sD1[s * kLd + j];
      dst = kOffB1 + j;
    } else if (q < kHid * kIn + 2 * kHid) {
      const int j = q - kHid * kIn - kHid;
      for (int s = 0; s < kTrainThreads; ++s) acc += sD2[s * kLd + j];
      dst = kOffB2 + j;
    } else if (q < kHid * kIn + 3 * kHid) {
      const int j = q - kHid * kIn - 2 * kHid;
      for (int s = 0; s < kTrainThreads; ++s) acc = __fmaf_rn(sE[s], sH2[s * kLd + j], acc);
      dst = kOffW3 + j;
    } else if (q == kHid * kIn + 3 * kHid) {
      for (int s = 0; s < kTrainThreads; ++s) acc += sE[s];
      dst = kOffB3;
    } else {
      for (int s = 0; s < kTrainThreads; ++s) acc += sL[s];
      dst = kNParam;  // loss slot
    }
    out[dst] = acc;
  }
}

// Sum of the per-block partials (gradient and loss) in block order.
__global__ void k_mlp_reduce(const float* __restrict__ part, int nblk, float* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > kNParam) return;
  float g = 0.0f;
  for (int b = 0; b < nblk; ++b) g += part[(size_t)b * kPartStride + p];
  out[p] = g;
}

// Adam (Kingma & Ba, 2015) with bias correction and a cosine learning-rate
// schedule from lr_max to lr_min over total_steps.  The step counter lives on
// the device so that a captured graph of many steps can be replayed; the last
// block to finish advances it.
struct AdamArgs {
  float* params;
  float* m;
  float* v;
  const float* part;
  int nblk;
  int* step_ctr;
  unsigned int* done;
  float* loss_hist;
  int total_steps;
  float lr_max, lr_min, beta1, beta2, eps;
};

__global__ void k_mlp_adam(AdamArgs a) {
  const int step = *(volatile int*)a.step_ctr;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kNParam) {
    float g = 0.0f;
    for (int b = 0; b < a.nblk; ++b) g += a.part[(size_t)b * kPartStride + p];
    const float m = a.beta1 * a.m[p] + (1.0f - a.beta1) * g;
    const float v = a.beta2 * a.v[p] + (1.0f - a.beta2) * g * g;
    a.m[p] = m;
    a.v[p] = v;
    const float tstep = (float)(step + 1);
    const float mh = m / (1.0f - powf(a.beta1, tstep));
    const float vh = v / (1.0f - powf(a.beta2, tstep));
    const float frac = fminf((float)step / (float)(a.total_steps > 0 ? a.total_steps : 1), 1.0f);
    const float lr = a.lr_min + 0.5f * (a.lr_max - a.lr_min) * (1.0f + cospif(frac));
    a.params[p] = a.params[p] - lr * mh / (sqrtf(vh) + a.eps);
  } else if (p == kNParam && a.loss_hist && step < a.total_steps) {
    float l = 0.0f;
    for (int b = 0; b < a.nblk; ++b) l += a.part[(size_t)b * kPartStride + kNParam];
    a.loss_hist[step] = l;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(a.done, 1u);
    if (prev == gridDim.x - 1) {
      *a.done = 0u;
      atomicAdd(a.step_ctr, 1);
      __threadfence();
    }
  }
}

// W2 split into BF16 hi and lo parts, packed in the UMMA K-major
// no-swizzle layout: 8-row x 16-byte core matrices, byte offset of
// (row r, column k) = (r/8)*1024 + (k/8)*128 + (r%8)*16 + (k%8)*2.
__host__ __device__ __forceinline__ uint32_t umma_off(int r, int k) {
  return (uint32_t)((r >> 3) * 1024 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__global__ void k_mlp_pack(const float* __restrict__ params, uint8_t* __restrict__ w2pack) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kHid * kHid) return;
  const int j = q / kHid, k = q % kHid;
  const float w = params[kOffW2 + q];
  const __nv_bfloat16 hi = __float2bfloat16_rn(w);
  const __nv_bfloat16 lo = __float2bfloat16_rn(w - __bfloat162float(hi));
  *reinterpret_cast<__nv_bfloat16*>(w2pack + umma_off(j, k)) = hi;
  *reinterpret_cast<__nv_bfloat16*>(w2pack + 8192 + umma_off(j, k)) = lo;
}

// ---- tcgen05 primitives ---------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on an mbarrier phase; false after the limit (error recorded by
// the caller, the kernel then winds down instead of spinning).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          long long limit = kSpinLimit) {
  for (long long s = 0; s < limit; ++s) {
    if (mbar_test(bar, parity)) return true;
    if (s > 64) __nanosleep(32);
  }
  return false;
}
// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (BF16 inputs), FP32 accumulate.
__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0u;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
// Shared-memory matrix descriptor, K-major, no swizzle: start address, leading
// byte offset (between the two 8-column core matrices of a K=16 slice, 128 B),
// stride byte offset (between 8-row groups, 1024 B), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)(1024u >> 4) << 32) | (1ull << 46);
}
// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// ---- inference kernel -----------------------------------------------------------
constexpr int kTile = 128;          // points per tile = UMMA M = threads per CTA
constexpr int kMaxBins = 64;
constexpr uint32_t kTmemCols = 64;  // FP32 accumulator columns (N)
struct InferSmem {
  uint8_t a_hi[16384];              // 128 x 64 BF16, UMMA layout
  uint8_t a_lo[16384];
  uint8_t w_hi[8192];               // 64 x 64 BF16
  uint8_t w_lo[8192];
  float w1[kHid * kIn], b1[kHid], b2[kHid], w3[kHid], b3;
  MlpBin bins[kMaxBins];
  uint64_t mbar;
  uint32_t tmem;
};

struct InferArgs {
  int model;
  int refine;
  MlpNorm norm;
  const float* params;
  const uint8_t* w2pack;
  const MlpBin* bins;
  int nb;
  // field kernel: phys_get_vset over a member's w-faces
  const MemberDev* members;
  int mi;
  const double* rhoc;
  const double* tc;
  double vset_fac;
  // point kernel
  long long npts;
  const double* pd;
  const double* prhop;
  const double* ppsi;
  const double* prhoa;
  const double* pmu;
  double* pout;
  int* pused;
  // counters
  unsigned long long* nfallback;
  int* nfail;
  int* err;
  long long wait_limit;  // polls before a completion wait gives up (kSpinLimit by default)
};

// Settling velocity of arbitrary points (arrays of d, rhop, psi, rhoa, mu):
// the same network and tensor-core layer as the field kernel, features in
// FP64 per point.  Used by f3d_mlp_predict.
__global__ void __launch_bounds__(kTile) k_mlp_vset_points(InferArgs a) {
  extern __shared__ uint8_t smraw[];
  InferSmem& S = *reinterpret_cast<InferSmem*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  const int t = threadIdx.x, warp = t >> 5;
  for (int q = t; q < 16384 / 16; q += kTile)
    reinterpret_cast<uint4*>(S.w_hi)[q] = reinterpret_cast<const uint4*>(a.w2pack)[q];
  for (int q = t; q < kHid * kIn; q += kTile) S.w1[q] = a.params[kOffW1 + q];
  for (int q = t; q < kHid; q += kTile) {
    S.b1[q] = a.params[kOffB1 + q];
    S.b2[q] = a.params[kOffB2 + q];
    S.w3[q] = a.params[kOffW3 + q];
  }
  if (t == 0) S.b3 = a.params[kOffB3];
  if (t == 0) {
    mbar_init(&S.mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    tmem_alloc(&S.tmem, kTmemCols);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t a_hi = smem_addr(S.a_hi), a_lo = smem_addr(S.a_lo);
  const uint32_t w_hi = smem_addr(S.w_hi), w_lo = smem_addr(S.w_lo);
  const long long tot = a.npts;
  const long long ntiles = (tot + kTile - 1) / kTile;
  uint32_t phase = 0;
  bool ok = true;
  unsigned long long nfb = 0;
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long e = tile * kTile + t;
    const bool live = e < tot;
    double d = 1.0, rhop = 1.0, psi = 1.0, rhoa = 1.0, mu = 1.0;
    bool inside = false;
    float f[kIn] = {0.f, 0.f, 0.f, 0.f, 0.f};
    float cout = 0.0f;
    if (live) {
      d = a.pd[e];
      rhop = a.prhop[e];
      psi = a.ppsi[e];
      rhoa = a.prhoa[e];
      mu = a.pmu[e];
      const double x[5] = {d, rhop, psi, rhoa, mu};
      inside = true;
      for (int c = 0; c < 5; ++c) inside = inside && x[c] >= a.norm.lo[c] && x[c] <= a.norm.hi[c];
      double co;
      point_features(a.norm, d, rhop, psi, rhoa, mu, f, &co);
      cout = (float)(co - log(mu));
    }
    // ---- layer 1 (FP32) -> split BF16 operand rows
    {
      uint8_t* rh = S.a_hi + (t >> 3) * 1024 + (t & 7) * 16;
      uint8_t* rl = S.a_lo + (t >> 3) * 1024 + (t & 7) * 16;
#pragma unroll
      for (int c = 0; c < kHid / 8; ++c) {
        uint32_t ph[4], pl[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float h[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int jj = 8 * c + 2 * q + u;
            float z = S.b1[jj];
#pragma unroll
            for (int ii = 0; ii < kIn; ++ii) z = __fmaf_rn(S.w1[jj * kIn + ii], f[ii], z);
            h[u] = tanh_net(z);
          }
          const __nv_bfloat162 hh = __floats2bfloat162_rn(h[0], h[1]);
          const float2 hf = __bfloat1622float2(hh);
          const __nv_bfloat162 ll = __floats2bfloat162_rn(h[0] - hf.x, h[1] - hf.y);
          ph[q] = *reinterpret_cast<const uint32_t*>(&hh);
          pl[q] = *reinterpret_cast<const uint32_t*>(&ll);
        }
        *reinterpret_cast<uint4*>(rh + c * 128) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
        *reinterpret_cast<uint4*>(rl + c * 128) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // ---- layer 2 on the tensor core: D = Ahi Whi^T + Ahi Wlo^T + Alo Whi^T
    if (t == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < kHid / 16; ++ks) {
        const uint32_t off = ks * 256;
        umma_bf16(tmem, umma_desc(a_hi + off), umma_desc(w_hi + off), kIdesc, ks > 0 ? 1u : 0u);
        umma_bf16(tmem, umma_desc(a_hi + off), umma_desc(w_lo + off), kIdesc, 1u);
        umma_bf16(tmem, umma_desc(a_lo + off), umma_desc(w_hi + off), kIdesc, 1u);
      }
      umma_commit(&S.mbar);
    }
    const bool landed = mbar_wait(&S.mbar, phase, a.wait_limit);
    if (!__syncthreads_and(landed)) {  // block-uniform decision
      if (t == 0) atomicExch(a.err, 1);
      ok = false;
      break;
    }
    phase ^= 1u;
    tc_fence_after();
    // ---- epilogue: layer 2 bias + tanh, layer 3, output transform
    float y = S.b3;
#pragma unroll
    for (int c = 0; c < kHid / 16; ++c) {
      float acc[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 16), acc);
      tmem_ld_wait();
#pragma unroll
      for (int q = 0; q < 16; ++q) y = __fmaf_rn(S.w3[c * 16 + q], tanh_net(acc[q] + S.b2[c * 16 + q]), y);
    }
    if (live) {
      double v;
      if (inside) {
        v = (double)expf(__fmaf_rn(4.0f, y, cout));
        if (a.refine) v = vset_steffensen(a.model, v, d, rhop, psi, rhoa, mu, vset_const(a.model, psi));
      } else {
        int it;
        if (vset_point_dev(d, rhop, psi, rhoa, mu, a.model, &v, &it)) atomicAdd(a.nfail, 1);
        ++nfb;
      }
      a.pout[e] = v;
      if (a.pused) a.pused[e] = inside ? 1 : 0;
    }
    // all TMEM reads of this tile complete before the next MMA overwrites D
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  // an MMA in flight lands before its tensor memory is freed (the full limit,
  // whatever the first wait's limit was)
  if (!ok) mbar_wait(&S.mbar, phase, kSpinLimit);
  if (nfb) atomicAdd(a.nfallback, nfb);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// Field kernel of phys_get_vset: one tile = 128 consecutive w-faces (i
// fastest), whose air density, temperature and viscosity are computed once
// and reused for every bin; per bin, layer 1 uses a per-bin constant vector
// (b1 + W1[:, 1:4] f1..f3, computed in the prologue) so that only the two
// air-dependent features (f0, f4) enter per face.  Bins that are gas (zero
// velocity) or outside the envelope (the iteration) skip the tensor core;
// faces whose air lies outside the envelope take the iteration.
struct FieldSmem {
  uint8_t a_hi[16384];
  uint8_t a_lo[16384];
  uint8_t w_hi[8192];
  uint8_t w_lo[8192];
  float w1c0[kHid], w1c4[kHid], b2[kHid], w3[kHid], b3, pad[3];
  float cb[kMaxBins][kHid];
  MlpBin bins[kMaxBins];
  uint64_t mbar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(kTile) k_mlp_vset_field(InferArgs a) {
  extern __shared__ uint8_t smraw[];
  FieldSmem& S = *reinterpret_cast<FieldSmem*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  const int t = threadIdx.x, warp = t >> 5;
  const int nb = a.nb;
  for (int q = t; q < 16384 / 16; q += kTile)
    reinterpret_cast<uint4*>(S.w_hi)[q] = reinterpret_cast<const uint4*>(a.w2pack)[q];
  for (int q = t; q < kHid; q += kTile) {
    S.w1c0[q] = a.params[kOffW1 + q * kIn];
    S.w1c4[q] = a.params[kOffW1 + q * kIn + 4];
    S.b2[q] = a.params[kOffB2 + q];
    S.w3[q] = a.params[kOffW3 + q];
  }
  if (t == 0) S.b3 = a.params[kOffB3];
  for (int q = t; q < nb; q += kTile) S.bins[q] = a.bins[q];
  __syncthreads();
  for (int q = t; q < nb * kHid; q += kTile) {
    const int b = q / kHid, j = q % kHid;
    const MlpBin& B = S.bins[b];
    float z = a.params[kOffB1 + j];
    z = __fmaf_rn(a.params[kOffW1 + j * kIn + 1], B.f1, z);
    z = __fmaf_rn(a.params[kOffW1 + j * kIn + 2], B.f2, z);
    z = __fmaf_rn(a.params[kOffW1 + j * kIn + 3], B.f3, z);
    S.cb[b][j] = z;
  }
  if (t == 0) {
    mbar_init(&S.mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    tmem_alloc(&S.tmem, kTmemCols);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t a_hi = smem_addr(S.a_hi), a_lo = smem_addr(S.a_lo);
  const uint32_t w_hi = smem_addr(S.w_hi), w_lo = smem_addr(S.w_lo);
  const MemberDev* m = a.members + a.mi;
  const unsigned int nx = (unsigned int)m->nx, ny = (unsigned int)m->ny, nz = (unsigned int)m->nz;
  const unsigned int nfaces = nx * ny * (nz + 1);
  const unsigned int ntiles = (nfaces + kTile - 1) / kTile;
  double* vs = const_cast<double*>(m->vs);
  uint32_t phase = 0;
  bool ok = true;
  unsigned long long nfb = 0;
  for (unsigned int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const unsigned int f = tile * kTile + t;
    const bool live = f < nfaces;
    double rhoa = 1.0, ta = 288.0, hm3 = 1.0;
    float lnmu = 0.0f, f0a = 0.0f, f4 = 0.0f;
    bool air_in = false;
    if (live) {
      const unsigned int i = f % nx, r = f / nx, j = r % ny, k = r / ny;
      const size_t cx = nx + 1, cy = ny + 1;
#define CO(arr, ii, jj) arr[(ii) + cx * ((jj) + cy * (size_t)k)]
      rhoa = 0.25 * (CO(a.rhoc, i, j) + CO(a.rhoc, i + 1, j) + CO(a.rhoc, i + 1, j + 1) + CO(a.rhoc, i, j + 1));
      ta = 0.25 * (CO(a.tc, i, j) + CO(a.tc, i + 1, j) + CO(a.tc, i + 1, j + 1) + CO(a.tc, i, j + 1));
#undef CO
      hm3 = m->hm3[i + (size_t)nx * j];
      const double tr = ta / 291.15;
      const double mu = 1.827e-5 * ((291.15 + 120.0) / (ta + 120.0)) * (tr * sqrt(tr));
      air_in = rhoa >= a.norm.lo[3] && rhoa <= a.norm.hi[3] && mu >= a.norm.lo[4] && mu <= a.norm.hi[4];
      const float lnra = __logf((float)rhoa);
      lnmu = __logf((float)mu);
      f0a = (lnra - 2.0f * lnmu) * a.norm.lar_sinv;
      f4 = __fmaf_rn(lnmu - a.norm.lnmu_lo, a.norm.lnmu_sinv, -1.0f);
    }
    bool have_mue = false;
    double mue = 0.0;
    for (int b = 0; b < nb && ok; ++b) {
      const MlpBin& B = S.bins[b];
      const int cat = B.flags & 0xff;
      double v = 0.0;
      bool iterate = false;
      if (cat != 2 && B.inside) {
        // ---- layer 1 -> split BF16 operand row t
        const float f0 = __fmaf_rn(B.lar0m, a.norm.lar_sinv, f0a);
        uint8_t* rh = S.a_hi + (t >> 3) * 1024 + (t & 7) * 16;
        uint8_t* rl = S.a_lo + (t >> 3) * 1024 + (t & 7) * 16;
        const float* cb = S.cb[b];
#pragma unroll
        for (int c = 0; c < kHid / 8; ++c) {
          uint32_t ph[4], pl[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int j0 = 8 * c + 2 * q;
            const float h0 = tanh_net(__fmaf_rn(S.w1c4[j0], f4, __fmaf_rn(S.w1c0[j0], f0, cb[j0])));
            const float h1 = tanh_net(__fmaf_rn(S.w1c4[j0 + 1], f4, __fmaf_rn(S.w1c0[j0 + 1], f0, cb[j0 + 1])));
            const __nv_bfloat162 hh = __floats2bfloat162_rn(h0, h1);
            const float2 hf = __bfloat1622float2(hh);
            const __nv_bfloat162 ll = __floats2bfloat162_rn(h0 - hf.x, h1 - hf.y);
            ph[q] = *reinterpret_cast<const uint32_t*>(&hh);
            pl[q] = *reinterpret_cast<const uint32_t*>(&ll);
          }
          *reinterpret_cast<uint4*>(rh + c * 128) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
          *reinterpret_cast<uint4*>(rl + c * 128) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
          tc_fence_after();
#pragma unroll
          for (int ks = 0; ks < kHid / 16; ++ks) {
            const uint32_t off = ks * 256;
            umma_bf16(tmem, umma_desc(a_hi + off), umma_desc(w_hi + off), kIdesc, ks > 0 ? 1u : 0u);
            umma_bf16(tmem, umma_desc(a_hi + off), umma_desc(w_lo + off), kIdesc, 1u);
            umma_bf16(tmem, umma_desc(a_lo + off), umma_desc(w_hi + off), kIdesc, 1u);
          }
          umma_commit(&S.mbar);
        }
        const bool landed = mbar_wait(&S.mbar, phase, a.wait_limit);
        if (!__syncthreads_and(landed)) {
          if (t == 0) atomicExch(a.err, 1);
          ok = false;
          break;
        }
        phase ^= 1u;
        tc_fence_after();
        float y = S.b3;
#pragma unroll
        for (int c = 0; c < kHid / 16; ++c) {
          float acc[16];
          tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 16), acc);
          tmem_ld_wait();
#pragma unroll
          for (int q = 0; q < 16; ++q) y = __fmaf_rn(S.w3[c * 16 + q], tanh_net(acc[q] + S.b2[c * 16 + q]), y);
        }
        tc_fence_before();  // TMEM reads done before the next bin's MMA
        v = (double)expf(__fmaf_rn(4.0f, y, B.cout - lnmu));
        iterate = !air_in;
      } else if (cat != 2) {
        iterate = true;  // bin outside the envelope
      }
      if (live && cat != 2 && (iterate || a.refine)) {
        if (!have_mue) {
          mue = 1.827e-5 * ((291.15 + 120.0) / (ta + 120.0)) * pow(ta / 291.15, 1.5);
          have_mue = true;
        }
        if (iterate) {
          int it;
          if (vset_point_dev(B.d, B.rhop, B.psi, rhoa, mue, a.model, &v, &it)) atomicAdd(a.nfail, 1);
          ++nfb;
        } else {
          v = vset_steffensen(a.model, v, B.d, B.rhop, B.psi, rhoa, mue, B.k);
        }
      }
      if (live) {
        if (B.flags >> 8) v = a.vset_fac * v;
        vs[(size_t)b * nfaces + f] = v / hm3;
      }
    }
  }
  // an MMA in flight lands before its tensor memory is freed (the full limit,
  // whatever the first wait's limit was)
  if (!ok) mbar_wait(&S.mbar, phase, kSpinLimit);
  if (nfb) atomicAdd(a.nfallback, nfb);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

}  // namespace f3d

using namespace f3d;

// ---- host handle -----------------------------------------------------------------
struct f3d_mlp {
  int device = 0, model = 2;
  double margin = 0.08;
  MlpNorm norm;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float* d_params = nullptr;
  float* d_m = nullptr;
  float* d_v = nullptr;
  uint8_t* d_w2pack = nullptr;
  float* d_part = nullptr;
  int part_blocks = 0;
  float* d_scratch = nullptr;   // gradient entry records / output
  long long scratch_n = 0;
  int* d_step = nullptr;
  unsigned int* d_done = nullptr;
  float* d_loss = nullptr;
  int loss_cap = 0;
  double* d_raw = nullptr;
  float* d_rec = nullptr;
  long long ns = 0;
  int* d_int = nullptr;                    // [0] nfail, [1] err
  unsigned long long* d_u64 = nullptr;     // [0] fallbacks
  MlpBin* d_bins = nullptr;
  int sms = 148, infer_occ = 1;
  size_t infer_smem = 0;
  size_t field_smem = 0;
  int field_occ = 1;
  float last_ms = 0.0f;
  bool packed = false;
};

#define MCK(call)                                                                      \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return set_error_msg("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),     \
                           __FILE__, __LINE__);                                        \
  } while (0)
#define MCKL() MCK(cudaGetLastError())

static int mlp_pack(f3d_mlp* h) {
  k_mlp_pack<<<(kHid * kHid + 255) / 256, 256, 0, h->st>>>(h->d_params, h->d_w2pack);
  MCKL();
  h->packed = true;
  return 0;
}

static void host_init_params(float* p, uint64_t seed) {
  // PyTorch-style Linear initialisation: U(-1/sqrt(fan_in), 1/sqrt(fan_in))
  auto fill = [&](int off, int n, int fan_in, uint64_t stream) {
    const double bound = 1.0 / sqrt((double)fan_in);
    for (int q = 0; q < n; ++q) p[off + q] = (float)((2.0 * u01(hash3(seed, stream, (uint64_t)q)) - 1.0) * bound);
  };
  fill(kOffW1, kHid * kIn, kIn, 1);
  fill(kOffB1, kHid, kIn, 2);
  fill(kOffW2, kHid * kHid, kHid, 3);
  fill(kOffB2, kHid, kHid, 4);
  fill(kOffW3, kHid, kHid, 5);
  fill(kOffB3, 1, kHid, 6);
}

extern "C" int f3d_mlp_destroy(f3d_mlp* h) {
  if (!h) return 0;
  cudaSetDevice(h->device);
  if (h->st) cudaStreamSynchronize(h->st);
  void* bufs[] = {h->d_params, h->d_m, h->d_v, h->d_w2pack, h->d_part, h->d_scratch, h->d_step,
                  h->d_done, h->d_loss, h->d_raw, h->d_rec, h->d_int, h->d_u64, h->d_bins};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return 0;
}

extern "C" int f3d_mlp_create(int model, const double* envelope, double margin, unsigned long long seed,
                              int device, f3d_mlp** out) {
  if (!out) return set_error_msg("f3d_mlp_create: null output");
  *out = nullptr;
  if (model < 1 || model > 7 || model == 4)
    return set_error_msg("f3d_mlp_create: model %d has no iterative solve to replace", model);
  if (!envelope) return set_error_msg("f3d_mlp_create: null envelope");
  for (int c = 0; c < 5; ++c)
    if (!(envelope[2 * c] > 0.0) || !(envelope[2 * c + 1] >= envelope[2 * c]))
      return set_error_msg("f3d_mlp_create: bad envelope for coordinate %d", c);
  if (envelope[0] == envelope[1] || envelope[8] == envelope[9] || envelope[5] > 1.0)
    return set_error_msg("f3d_mlp_create: degenerate diameter/viscosity range or sphericity > 1");
  if (!(margin >= 0.0 && margin < 0.5)) return set_error_msg("f3d_mlp_create: margin must be in [0, 0.5)");
  f3d_mlp* h = new f3d_mlp();
  h->device = device;
  h->model = model;
  h->margin = margin;
  h->norm = make_norm(envelope, margin);
  auto fail = [&](cudaError_t e, const char* what) {
    set_error_msg("f3d_mlp_create: %s: %s", what, cudaGetErrorString(e));
    f3d_mlp_destroy(h);
    return 1;
  };
  cudaError_t e;
  if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(e, "set device");
  if ((e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
  if ((e = cudaEventCreate(&h->ev0)) != cudaSuccess || (e = cudaEventCreate(&h->ev1)) != cudaSuccess)
    return fail(e, "events");
  if ((e = cudaMalloc(&h->d_params, sizeof(float) * kPartStride)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_m, sizeof(float) * kPartStride)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_v, sizeof(float) * kPartStride)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_w2pack, 16384)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_step, sizeof(int) * 2)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_done, sizeof(unsigned int) * 2)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_int, sizeof(int) * 4)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_u64, sizeof(unsigned long long) * 2)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_bins, sizeof(MlpBin) * kMaxBins)) != cudaSuccess)
    return fail(e, "device allocation");
  std::vector<float> p(kPartStride, 0.0f);
  host_init_params(p.data(), seed);
  if ((e = cudaMemcpy(h->d_params, p.data(), sizeof(float) * kPartStride, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e, "upload");
  cudaMemset(h->d_m, 0, sizeof(float) * kPartStride);
  cudaMemset(h->d_v, 0, sizeof(float) * kPartStride);
  cudaMemset(h->d_step, 0, sizeof(int) * 2);
  cudaMemset(h->d_done, 0, sizeof(unsigned int) * 2);
  cudaGetLastError();
  int dev_sms = 0;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
  h->sms = dev_sms > 0 ? dev_sms : 148;
  h->infer_smem = sizeof(InferSmem) + 1024;
  if ((e = cudaFuncSetAttribute(k_mlp_vset_points, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)h->infer_smem)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(k_mlp_train<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kTrainSmem)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(k_mlp_train<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kTrainSmem)) != cudaSuccess)
    return fail(e, "kernel attributes");
  h->field_smem = sizeof(FieldSmem) + 1024;
  if ((e = cudaFuncSetAttribute(k_mlp_vset_field, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)h->field_smem)) != cudaSuccess)
    return fail(e, "kernel attributes");
  // resident CTAs per SM: shared memory (with the 1 KB the runtime reserves
  // per block), registers, and the SM's 512 tensor-memory columns
  {
    int smem_sm = 0;
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    auto occ_of = [&](const void* fn, size_t smem) {
      cudaFuncAttributes fa;
      int regs = 128;
      if (cudaFuncGetAttributes(&fa, fn) == cudaSuccess && fa.numRegs > 0) regs = fa.numRegs;
      int o = smem_sm > 0 ? (int)(smem_sm / (smem + 1024)) : 1;
      const int oreg = 65536 / (regs * kTile);
      if (oreg < o) o = oreg;
      if ((int)(512 / kTmemCols) < o) o = (int)(512 / kTmemCols);
      return o < 1 ? 1 : o;
    };
    h->infer_occ = occ_of((const void*)k_mlp_vset_points, h->infer_smem);
    h->field_occ = occ_of((const void*)k_mlp_vset_field, h->field_smem);
  }
  if (mlp_pack(h)) {
    f3d_mlp_destroy(h);
    return 1;
  }
  if ((e = cudaStreamSynchronize(h->st)) != cudaSuccess) return fail(e, "init");
  *out = h;
  return 0;
}

extern "C" int f3d_mlp_generate(f3d_mlp* h, long long nsamples, unsigned long long seed, long long* nfail) {
  if (!h || nsamples <= 0) return set_error_msg("f3d_mlp_generate: bad arguments");
  MCK(cudaSetDevice(h->device));
  if (nsamples != h->ns) {
    if (h->d_raw) cudaFree(h->d_raw);
    if (h->d_rec) cudaFree(h->d_rec);
    h->d_raw = nullptr;
    h->d_rec = nullptr;
    h->ns = 0;
    MCK(cudaMalloc(&h->d_raw, sizeof(double) * 5 * nsamples));
    MCK(cudaMalloc(&h->d_rec, sizeof(float) * kRecF * nsamples));
    h->ns = nsamples;
  }
  MCK(cudaMemsetAsync(h->d_int, 0, sizeof(int) * 4, h->st));
  k_mlp_samples<<<h->sms * 8, 128, 0, h->st>>>(h->norm, h->model, nsamples, seed, h->d_raw, h->d_rec, h->d_int);
  MCKL();
  int nf = 0;
  MCK(cudaMemcpyAsync(&nf, h->d_int, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  MCK(cudaStreamSynchronize(h->st));
  if (nfail) *nfail = nf;
  return 0;
}

extern "C" int f3d_mlp_get_samples(f3d_mlp* h, long long first, long long n, double* raw, float* rec) {
  if (!h || first < 0 || n < 0 || first + n > h->ns) return set_error_msg("f3d_mlp_get_samples: bad range");
  MCK(cudaSetDevice(h->device));
  if (raw) MCK(cudaMemcpyAsync(raw, h->d_raw + 5 * first, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, h->st));
  if (rec) MCK(cudaMemcpyAsync(rec, h->d_rec + kRecF * first, sizeof(float) * kRecF * n, cudaMemcpyDeviceToHost, h->st));
  MCK(cudaStreamSynchronize(h->st));
  return 0;
}

static int ensure_part(f3d_mlp* h, int nblk) {
  if (nblk <= h->part_blocks) return 0;
  if (h->d_part) cudaFree(h->d_part);
  h->d_part = nullptr;
  h->part_blocks = 0;
  MCK(cudaMalloc(&h->d_part, sizeof(float) * kPartStride * (size_t)nblk));
  h->part_blocks = nblk;
  return 0;
}

extern "C" int f3d_mlp_train(f3d_mlp* h, int steps, int batch, double lr_max, double lr_min,
                             unsigned long long seed, float* loss_hist, float* train_ms) {
  if (!h || steps < 0 || batch <= 0 || batch % kTrainThreads)
    return set_error_msg("f3d_mlp_train: steps >= 0 and batch a positive multiple of %d", kTrainThreads);
  if (h->ns <= 0) return set_error_msg("f3d_mlp_train: no samples (call f3d_mlp_generate first)");
  MCK(cudaSetDevice(h->device));
  const int nblk = batch / kTrainThreads;
  if (ensure_part(h, nblk)) return 1;
  if (steps > h->loss_cap) {
    if (h->d_loss) cudaFree(h->d_loss);
    h->d_loss = nullptr;
    h->loss_cap = 0;
    MCK(cudaMalloc(&h->d_loss, sizeof(float) * steps));
    h->loss_cap = steps;
  }
  // a fresh run of Adam: moments and step counter from zero
  MCK(cudaMemsetAsync(h->d_m, 0, sizeof(float) * kPartStride, h->st));
  MCK(cudaMemsetAsync(h->d_v, 0, sizeof(float) * kPartStride, h->st));
  MCK(cudaMemsetAsync(h->d_step, 0, sizeof(int) * 2, h->st));
  MCK(cudaMemsetAsync(h->d_done, 0, sizeof(unsigned int) * 2, h->st));
  AdamArgs aa;
  aa.params = h->d_params;
  aa.m = h->d_m;
  aa.v = h->d_v;
  aa.part = h->d_part;
  aa.nblk = nblk;
  aa.step_ctr = h->d_step;
  aa.done = h->d_done;
  aa.loss_hist = h->d_loss;
  aa.total_steps = steps;
  aa.lr_max = (float)lr_max;
  aa.lr_min = (float)lr_min;
  aa.beta1 = 0.9f;
  aa.beta2 = 0.999f;
  aa.eps = 1e-8f;
  const float inv_b = 1.0f / (float)batch;
  const int adam_blocks = (kNParam + 1 + 127) / 128;
  auto one_step = [&]() {
    k_mlp_train<false><<<nblk, kTrainThreads, kTrainSmem, h->st>>>(h->d_params, h->d_rec, h->ns, seed, h->d_step,
                                                                   inv_b, 0, h->d_part);
    k_mlp_adam<<<adam_blocks, 128, 0, h->st>>>(aa);
  };
  MCK(cudaEventRecord(h->ev0, h->st));
  const int chunk = 250;
  int done = 0;
  if (steps >= chunk) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    MCK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    for (int q = 0; q < chunk; ++q) one_step();
    cudaError_t ce = cudaStreamEndCapture(h->st, &g);
    if (ce != cudaSuccess) return set_error_msg("f3d_mlp_train: capture failed: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return set_error_msg("f3d_mlp_train: instantiate failed: %s", cudaGetErrorString(ce));
    for (; done + chunk <= steps; done += chunk) {
      ce = cudaGraphLaunch(ge, h->st);
      if (ce != cudaSuccess) break;
    }
    cudaGraphExecDestroy(ge);
    if (ce != cudaSuccess) return set_error_msg("f3d_mlp_train: graph launch failed: %s", cudaGetErrorString(ce));
  }
  for (; done < steps; ++done) one_step();
  MCKL();
  MCK(cudaEventRecord(h->ev1, h->st));
  if (mlp_pack(h)) return 1;
  if (loss_hist && steps)
    MCK(cudaMemcpyAsync(loss_hist, h->d_loss, sizeof(float) * steps, cudaMemcpyDeviceToHost, h->st));
  MCK(cudaStreamSynchronize(h->st));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (train_ms) *train_ms = ms;
  return 0;
}

static int ensure_scratch(f3d_mlp* h, long long nfloats) {
  if (nfloats <= h->scratch_n) return 0;
  if (h->d_scratch) cudaFree(h->d_scratch);
  h->d_scratch = nullptr;
  h->scratch_n = 0;
  MCK(cudaMalloc(&h->d_scratch, sizeof(float) * nfloats));
  h->scratch_n = nfloats;
  return 0;
}

// Gradient of the mean squared error over n given samples (features n x 5,
// targets n) at the current parameters, through the training kernel.
extern "C" int f3d_mlp_gradient(f3d_mlp* h, long long n, const float* feats, const float* targets, float* grad,
                                float* loss) {
  if (!h || n <= 0 || !feats || !targets || !grad) return set_error_msg("f3d_mlp_gradient: bad arguments");
  if (n > (1LL << 24)) return set_error_msg("f3d_mlp_gradient: at most 2^24 samples");
  MCK(cudaSetDevice(h->device));
  const int nblk = (int)((n + kTrainThreads - 1) / kTrainThreads);
  if (ensure_part(h, nblk)) return 1;
  const long long npad = (long long)nblk * kTrainThreads;
  if (ensure_scratch(h, kRecF * npad + kPartStride)) return 1;
  std::vector<float> rec((size_t)(kRecF * npad), 0.0f);
  for (long long q = 0; q < n; ++q) {
    for (int c = 0; c < kIn; ++c) rec[kRecF * q + c] = feats[kIn * q + c];
    rec[kRecF * q + 5] = targets[q];
  }
  MCK(cudaMemcpyAsync(h->d_scratch, rec.data(), sizeof(float) * rec.size(), cudaMemcpyHostToDevice, h->st));
  k_mlp_train<true><<<nblk, kTrainThreads, kTrainSmem, h->st>>>(h->d_params, h->d_scratch, npad, 0, h->d_step,
                                                                1.0f / (float)n, n, h->d_part);
  MCKL();
  float* out = h->d_scratch + kRecF * npad;
  k_mlp_reduce<<<(kNParam + 1 + 127) / 128, 128, 0, h->st>>>(h->d_part, nblk, out);
  MCKL();
  std::vector<float> g(kNParam + 1);
  MCK(cudaMemcpyAsync(g.data(), out, sizeof(float) * (kNParam + 1), cudaMemcpyDeviceToHost, h->st));
  MCK(cudaStreamSynchronize(h->st));
  memcpy(grad, g.data(), sizeof(float) * kNParam);
  if (loss) *loss = g[kNParam];
  return 0;
}

extern "C" int f3d_mlp_get_params(f3d_mlp* h, float* p) {
  if (!h || !p) return set_error_msg("f3d_mlp_get_params: bad arguments");
  MCK(cudaSetDevice(h->device));
  MCK(cudaMemcpyAsync(p, h->d_params, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, h->st));
  MCK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int f3d_mlp_set_params(f3d_mlp* h, const float* p) {
  if (!h || !p) return set_error_msg("f3d_mlp_set_params: bad arguments");
  for (int q = 0; q < kNParam; ++q)
    if (!isfinite(p[q])) return set_error_msg("f3d_mlp_set_params: parameter %d is not finite", q);
  MCK(cudaSetDevice(h->device));
  MCK(cudaMemcpyAsync(h->d_params, p, sizeof(float) * kNParam, cudaMemcpyHostToDevice, h->st));
  if (mlp_pack(h)) return 1;
  MCK(cudaStreamSynchronize(h->st));
  return 0;
}

// Normalisation constants: [lar_c, lar_sinv, sg_scale, psi_lo, psi_sinv, lnd_lo,
// lnd_sinv, lnmu_lo, lnmu_sinv] followed by the training box (lo, hi) x 5.
extern "C" int f3d_mlp_get_norm(f3d_mlp* h, double* out) {
  if (!h || !out) return set_error_msg("f3d_mlp_get_norm: bad arguments");
  const MlpNorm& n = h->norm;
  const float v[9] = {n.lar_c, n.lar_sinv, n.sg_scale, n.psi_lo, n.psi_sinv, n.lnd_lo, n.lnd_sinv, n.lnmu_lo, n.lnmu_sinv};
  for (int q = 0; q < 9; ++q) out[q] = (double)v[q];
  for (int c = 0; c < 5; ++c) {
    out[9 + 2 * c] = n.tlo[c];
    out[10 + 2 * c] = n.thi[c];
  }
  return 0;
}

extern "C" int f3d_mlp_last_ms(f3d_mlp* h, float* ms) {
  if (!h || !ms) return set_error_msg("f3d_mlp_last_ms: bad arguments");
  *ms = h->last_ms;
  return 0;
}

static int infer_launch(f3d_mlp* h, bool field, InferArgs& a, long long tot, cudaStream_t st) {
  a.model = h->model;
  a.norm = h->norm;
  a.params = h->d_params;
  a.w2pack = h->d_w2pack;
  a.nfallback = h->d_u64;
  a.nfail = h->d_int;
  a.err = h->d_int + 1;
  a.wait_limit = wait_limit();
  const long long ntiles = (tot + kTile - 1) / kTile;
  long long grid = (long long)h->sms * h->infer_occ;
  if (grid > ntiles) grid = ntiles;
  if (grid < 1) grid = 1;
  MCK(cudaMemsetAsync(h->d_int, 0, sizeof(int) * 4, st));
  MCK(cudaMemsetAsync(h->d_u64, 0, sizeof(unsigned long long) * 2, st));
  if (field) {
    grid = (long long)h->sms * h->field_occ;
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
  }
  MCK(cudaEventRecord(h->ev0, st));
  if (field) k_mlp_vset_field<<<(int)grid, kTile, h->field_smem, st>>>(a);
  else k_mlp_vset_points<<<(int)grid, kTile, h->infer_smem, st>>>(a);
  MCKL();
  MCK(cudaEventRecord(h->ev1, st));
  return 0;
}

static int infer_finish(f3d_mlp* h, cudaStream_t st, long long* nfallback, int* nfail) {
  int iv[4];
  unsigned long long uv[2];
  MCK(cudaMemcpyAsync(iv, h->d_int, sizeof(iv), cudaMemcpyDeviceToHost, st));
  MCK(cudaMemcpyAsync(uv, h->d_u64, sizeof(uv), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  if (iv[1]) return set_error_msg("mlp inference: tensor-core completion wait timed out");
  if (nfallback) *nfallback = (long long)uv[0];
  if (nfail) *nfail = iv[0];
  return 0;
}

// Settling velocity of n points (host arrays) by the surrogate; points outside
// the envelope take the iteration.  used[q] = 1 where the surrogate answered.
extern "C" int f3d_mlp_predict(f3d_mlp* h, long long n, const double* diam, const double* rhop, const double* psi,
                               const double* rhoa, const double* visc, int refine, double* vset, int* used) {
  if (!h || n < 0 || (n > 0 && (!diam || !rhop || !psi || !rhoa || !visc || !vset)))
    return set_error_msg("f3d_mlp_predict: bad arguments");
  if (n == 0) return 0;
  MCK(cudaSetDevice(h->device));
  double* d = nullptr;
  int* du = nullptr;
  MCK(cudaMalloc(&d, sizeof(double) * 6 * n));
  if (cudaMalloc(&du, sizeof(int) * n) != cudaSuccess) {
    cudaFree(d);
    return set_error_msg("f3d_mlp_predict: device allocation failed");
  }
  int rc = 0;
  const double* src[5] = {diam, rhop, psi, rhoa, visc};
  for (int c = 0; c < 5 && !rc; ++c)
    if (cudaMemcpyAsync(d + c * n, src[c], sizeof(double) * n, cudaMemcpyHostToDevice, h->st) != cudaSuccess)
      rc = set_error_msg("f3d_mlp_predict: upload failed");
  if (!rc) {
    InferArgs a{};
    a.refine = refine;
    a.npts = n;
    a.pd = d;
    a.prhop = d + n;
    a.ppsi = d + 2 * n;
    a.prhoa = d + 3 * n;
    a.pmu = d + 4 * n;
    a.pout = d + 5 * n;
    a.pused = du;
    rc = infer_launch(h, false, a, n, h->st);
  }
  int nfail = 0;
  if (!rc) rc = infer_finish(h, h->st, nullptr, &nfail);
  if (!rc && cudaMemcpy(vset, d + 5 * n, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = set_error_msg("f3d_mlp_predict: download failed");
  if (!rc && used && cudaMemcpy(used, du, sizeof(int) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = set_error_msg("f3d_mlp_predict: download failed");
  cudaFree(d);
  cudaFree(du);
  if (!rc && nfail) {
    set_error_msg("no convergence in vset (%d points)", nfail);
    return 2;
  }
  return rc;
}

namespace f3d {
// phys_get_vset over member mi's w-faces with the surrogate (the ensemble and
// single-domain entry points call this after staging rhoc/tc on the device).
int mlp_vset_field(f3d_mlp* h, const MemberDev* dm, int mi, int nx, int ny, int nz, int nb, const double* drhoc,
                   const double* dtc, const double* diam, const double* rhop, const double* psi,
                   const int* bin_cat, const int* is_aggregate, double vset_fac, int refine, cudaStream_t st,
                   long long* nfallback, int* nfail) {
  if (!h) return set_error_msg("surrogate handle is null");
  if (nb > kMaxBins) return set_error_msg("surrogate vset: at most %d bins", kMaxBins);
  std::vector<MlpBin> bins(nb);
  const MlpNorm& n = h->norm;
  for (int b = 0; b < nb; ++b) {
    MlpBin& B = bins[b];
    memset(&B, 0, sizeof(B));
    B.d = diam[b];
    B.rhop = rhop[b];
    B.psi = psi[b];
    B.flags = bin_cat[b] | ((is_aggregate && is_aggregate[b]) ? (1 << 8) : 0);
    B.inside = B.d >= n.lo[0] && B.d <= n.hi[0] && B.rhop >= n.lo[1] && B.rhop <= n.hi[1] && B.psi >= n.lo[2] &&
               B.psi <= n.hi[2];
    if (B.psi > 0.0) {
      // drag-law bin constants, the same expressions as vset_const
      if (h->model == 2) {
        B.k.rk1 = 3.0 / (1.0 + 2.0 / sqrt(B.psi));
        B.k.rk2 = pow(10.0, 1.8148 * pow(-log10(B.psi), 0.5743));
      }
      if (h->model == 5) {
        const double cd100 = 0.24 * pow(B.psi, -0.828) + 2.0 * sqrt(1.07 - B.psi);
        B.k.a = (1.0 - cd100) / 900.0;
        B.k.b = 1.0 - 1000.0 * B.k.a;
      }
    }
    if (B.inside) {
      const double lnd = log(B.d);
      B.lar0m = (float)(log(9.81) + 3.0 * lnd + log(B.rhop) - (double)n.lar_c);
      B.f1 = (float)(sg_of(B.psi) * (double)n.sg_scale - 1.0);
      B.f2 = (float)((B.psi - (double)n.psi_lo) * (double)n.psi_sinv - 1.0);
      B.f3 = (float)((lnd - (double)n.lnd_lo) * (double)n.lnd_sinv - 1.0);
      B.cout = (float)(log(9.81) + 2.0 * lnd + log(B.rhop) + ln_k1_18(B.psi));
    }
  }
  MCK(cudaMemcpyAsync(h->d_bins, bins.data(), sizeof(MlpBin) * nb, cudaMemcpyHostToDevice, st));
  InferArgs a{};
  a.refine = refine;
  a.bins = h->d_bins;
  a.nb = nb;
  a.members = dm;
  a.mi = mi;
  a.rhoc = drhoc;
  a.tc = dtc;
  a.vset_fac = vset_fac;
  const long long nfaces = (long long)(nz + 1) * ny * nx;
  if (nfaces * nb >= (1LL << 31)) return set_error_msg("surrogate vset: field too large (>= 2^31 faces x bins)");
  if (infer_launch(h, true, a, nfaces, st)) return 1;
  return infer_finish(h, st, nfallback, nfail);
}
}  // namespace f3d
