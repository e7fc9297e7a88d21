// noalloc.cu -- grid_get_mass_volume for callers that cannot allocate.
//
// Some callers cannot let a library call cudaMalloc: a FALL3D port whose
// device arrays are owned by its own runtime (an OpenACC or CUDA Fortran
// data region, a pre-reserved memory pool sized at start-up), or a host
// framework that forbids allocation once its time loop runs.  This entry
// point computes the mass in the volume straight from the caller's device
// arrays and allocates nothing: the per-block partial sums it needs live in
// a fixed file-scope __device__ array (kMaxBins x kBlocks doubles, 148 KiB).
// The CUDA runtime commits that array on a device when it loads this
// library's device code there: at the first call on that device under the
// default lazy module loading (CUDA_MODULE_LOADING=LAZY), or when the
// context is created with eager loading.  From then on the device holds it
// until the context ends.
//
// The array is shared by every call on a device and keeps the last call's
// partials; every call overwrites all the slots it reads, so nothing has to
// be cleared, but two calls that overlap on the GPU (different streams, no
// ordering between them) race on it.
#include <cuda_runtime.h>

#include <cmath>

namespace f3d {
int set_error_msg(const char* fmt, ...);  // f3d_capi.cu

namespace {
constexpr int kMaxBins = 64;
constexpr int kBlocks = 296;  // 2 x 148 SMs, the same grid as the context path
constexpr int kThreads = 256;

__device__ __align__(256) double g_mass_partials[kMaxBins * kBlocks];

// Same cell order and Neumaier accumulation as the context path's
// k_mass_partial, reading the reference layout with its two-cell halos.
__global__ void k_mass_ref_partial(const double* __restrict__ c, int nx, int ny, int nz,
                                   const double* __restrict__ dx1p,
                                   const double* __restrict__ dx2p,
                                   const double* __restrict__ dx3p, double* partials) {
  const long long ncell = (long long)nx * ny * nz;
  const int b = blockIdx.y;
  __shared__ double sm[kThreads];
  double acc = 0.0, comp = 0.0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ncell;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % nx);
    long long t = e / nx;
    int j = (int)(t % ny);
    int k = (int)(t / ny);
    double cv = c[(i + 2) + (long long)(nx + 4) *
                                ((j + 2) + (long long)(ny + 4) * ((k + 2) + (long long)(nz + 4) * b))];
    double x = cv * dx1p[i + 2] * dx2p[j + 2] * dx3p[k + 2];
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

__global__ void k_mass_ref_final(const double* partials, int nblk, int nb, double* per_bin,
                                 double* total) {
  __shared__ double sm[kThreads];
  double tot = 0.0, tcomp = 0.0;
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
    if (threadIdx.x == 0) {
      const double x = sm[0];
      if (per_bin) per_bin[b] = x;
      const double tt = tot + x;
      if (fabs(tot) >= fabs(x)) tcomp += (tot - tt) + x; else tcomp += (x - tt) + tot;
      tot = tt;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = tot + tcomp;
}
}  // namespace
}  // namespace f3d

// Mass in the volume without allocation; see include/fall3d_ads.h.
extern "C" int f3d_mass_volume_noalloc(int nx, int ny, int nz, int nbins, const double* c,
                                       const double* dX1_p, const double* dX2_p,
                                       const double* dX3_p, double* per_bin, double* total,
                                       void* stream) {
  using namespace f3d;
  if (nx < 1 || ny < 1 || nz < 1 || nbins < 1)
    return set_error_msg("f3d_mass_volume_noalloc: invalid sizes %d %d %d %d", nx, ny, nz, nbins);
  if (nbins > kMaxBins)
    return set_error_msg("f3d_mass_volume_noalloc: %d bins exceed the fixed scratch limit of %d "
                         "bins", nbins, kMaxBins);
  if (!c || !dX1_p || !dX2_p || !dX3_p || (!per_bin && !total))
    return set_error_msg("f3d_mass_volume_noalloc: null device pointer");
  // In host code the symbol g_mass_partials is only a stand-in for the
  // device copy; the address a kernel may use comes from
  // cudaGetSymbolAddress, for the current device and its current context.
  // It is looked up on every call (cheap once the module is loaded), so a
  // context that was reset and created again gets its own array's address.
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_mass_partials);
  if (e != cudaSuccess || !p)
    return set_error_msg("f3d_mass_volume_noalloc: cudaGetSymbolAddress failed: %s",
                         cudaGetErrorString(e));
  double* partials = static_cast<double*>(p);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dim3 g(kBlocks, nbins);
  k_mass_ref_partial<<<g, kThreads, 0, st>>>(c, nx, ny, nz, dX1_p, dX2_p, dX3_p, partials);
  k_mass_ref_final<<<1, kThreads, 0, st>>>(partials, kBlocks, nbins, per_bin, total);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error_msg("f3d_mass_volume_noalloc: launch failed: %s", cudaGetErrorString(e));
  return 0;
}
