// f3d_capi.cu -- host side of libfall3d_ads.so: contexts, device buffers,
// uploads in the reference layouts and the step sequence of F3D_time_step.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fall3d_ads.h"
#include "f3d_common.cuh"
#include "phys_dev.cuh"
#include "phys_host.h"

namespace f3d {
// ads_fp64.cu
void launch_sweep64(int dir, int lim, int tm, int epi, const MemberDev* members, const WorkItem* work,
                    int nblocks, int bpb, cudaStream_t st);
void launch_prep64(const MemberDev* members, const int* blk_member, const int* blk_first,
                   int nblocks, int mask, cudaStream_t st);
void launch_source64(const MemberDev* members, int nmembers, cudaStream_t st);
// aux_fp64.cu
void launch_conv(int which, const double* in, double* out, int nx, int ny, int nz, int nb,
                 cudaStream_t st);
void launch_set_step(MemberDev* members, int mi, double dt, double time, int iiter,
                     cudaStream_t st);
void launch_set_dt_stime(MemberDev* members, int mi, double dt, double stime, cudaStream_t st);
void launch_flux_reduce(const MemberDev* members, int nmembers, int dirmask, cudaStream_t st);
void launch_zero_step(const MemberDev* members, int nmembers, cudaStream_t st);
void launch_cfl(const MemberDev* members, int mi, double s, int criterion, double* out3,
                cudaStream_t st, const GcArgs* gc = nullptr);
void launch_mass(const MemberDev* members, int mi, int nb, int fp32, double* partials, int nblk,
                 double* out, cudaStream_t st);
void launch_vset_points(int model, int n, const double* diam, const double* rhop,
                        const double* psi, const double* rhoa, const double* visc, double* vset,
                        int* flags, int* iters, int* nfail, cudaStream_t st);
struct MetGeo {
  int nx, ny, nz, map_v;
  double X3max;
  const double* X3c;
  const double* X3p;
  const double* dhdx;
  const double* dhdy;
  const double* hm1;
  const double* hm2;
  const double* hm3;
};
void launch_meteo_corners(const MetGeo& g, const double* uc, const double* vc, const double* wc,
                          const double* k1, const double* k2, const double* k3, double* ux,
                          double* vy, double* wz, double* k1x, double* k2y, double* k3z,
                          cudaStream_t st);
void launch_meteo_kconst(int nx, int ny, int nz, double kh, double kv, double* k1, double* k2,
                         double* k3, cudaStream_t st);
void launch_gc_winds(MemberDev* members, int mi, int nx, int ny, int nz, int fp32, const GcArgs& g,
                     cudaStream_t st);
int mlp_vset_field(f3d_mlp* h, const MemberDev* dm, int mi, int nx, int ny, int nz, int nb,
                   const double* drhoc, const double* dtc, const double* diam, const double* rhop,
                   const double* psi, const int* bin_cat, const int* is_aggregate, double vset_fac,
                   int refine, cudaStream_t st, long long* nfallback, int* nfail);
void launch_vset_field(MemberDev* members, int mi, int model, const double* rhoc,
                       const double* tc, const double* bin_par, const int* bin_flags,
                       double vset_fac, int* nfail, cudaStream_t st);
void launch_face_kk(MemberDev* members, int mi, cudaStream_t st);
void launch_nonfinite(const double* p, long long n, int bit, unsigned int* mask, cudaStream_t st);
void launch_nonfinite(const float* p, long long n, int bit, unsigned int* mask, cudaStream_t st);
void launch_ads_solve_1d(int n, int lim, double* c, const double* dxp, const double* dxb,
                         const double* u, const double* k, double dt, const double bvalue[2],
                         const int bcode[2], double* flux, double* work, cudaStream_t st);
// ads_fp32.cu
void launch_sweep32(int dir, int lim, int tm, int cmp, int epi, const MemberDev* members,
                    const WorkItem* work, int nblocks, int bpb, cudaStream_t st);
void launch_prep32(const MemberDev* members, const int* blk_member, const int* blk_first,
                   int nblocks, int mask, cudaStream_t st);
void launch_source32(const MemberDev* members, int nmembers, cudaStream_t st);
void launch_fp32_fields(MemberDev* members, int mi, cudaStream_t st);
}  // namespace f3d

using namespace f3d;

// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int set_err(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return 1;
}

namespace f3d {
// Error reporting shared with the other translation units of the library.
int set_error_msg(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return 1;
}
}  // namespace f3d

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                     __LINE__);                                                         \
  } while (0)

#define CKL()                                                                          \
  do {                                                                                 \
    cudaError_t e_ = cudaGetLastError();                                               \
    if (e_ != cudaSuccess)                                                             \
      return set_err("kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, \
                     __LINE__);                                                        \
  } while (0)

static const int kSweepWarps = 4;  // warps per sweep block (128 threads)
static const int kPrepBlock = 256;

struct f3d_ctx {
  int nx = 0, ny = 0, nz = 0, nb = 0, lim = 2, tm = 2, prec = 0, device = 0;
  int cmp = 0;  // precision form with the compensated (hi + lo) state
  cudaStream_t st = nullptr;
  MemberDev hm;            // host mirror of the member descriptor
  MemberDev* dm = nullptr; // device copy
  WorkItem* dwork[3] = {nullptr, nullptr, nullptr};
  int nblk[3] = {0, 0, 0};
  int* dprep_member = nullptr;
  int* dprep_first = nullptr;
  int nprep = 0;
  int bpb = 4;  // bins per sweep block (1, 2 or 4); warps of a block share a spatial tile
  std::vector<void*> allocs;
  double* staging = nullptr;
  size_t staging_elems = 0;
  double* d_red = nullptr;    // reduction scratch (CFL 3 doubles, mass partials)
  int mass_nblk = 148 * 2;
  double* h_pin = nullptr;    // pinned host scratch (fluxes, reductions)
  int* d_nfail = nullptr;
  double t_its = 0.0, t_ite = 1.0;
  bool grid_set = false, meteo_set = false;
  // host copies of the grid (source volumes)
  std::vector<double> dX1_p, dX2_p, dX3_p, Hm1_p, Hm2_p, Hm3_p;
  int src_cap = 0;
  double* d_rhoc_tc = nullptr;
  size_t rhoc_cap = 0;
  // per-phase profiling
  bool prof = false;
  cudaEvent_t ev[8] = {};
  double prof_ms[6] = {0, 0, 0, 0, 0, 0};
  int prof_steps = 0;
  long long launches = 0;  // kernels launched by this context
  // terrain mapping for the on-device meteo term (Cartesian until set)
  int map_v = 0;
  double X3max = 1.0;
  double* d_terrain = nullptr;  // X3_c (nz+1), X3_p (nz), dhdx_p, dhdy_p (nx*ny each)
  double* d_met = nullptr;      // corner winds of two snapshots + unscaled diffusion
  size_t met_cap = 0;
  // wet deposition (after the z sweep) and radioactive decay
  bool wet_on = false;
  double wet_a = 0.0;
  double* d_powpb = nullptr;    // P^b per column
  int* d_ktop = nullptr;        // levels below the boundary-layer top per column
  double* d_awet = nullptr;     // wet deposit [bin][j][i]
  unsigned long long wet_mask = 0;
  double* d_zc = nullptr;       // corner heights for the output reductions
  bool gc_set = false;          // gravity current (f3d_ads_set_gravity_current)
  double gc_p[11] = {};
  std::vector<double> gc_host;  // lon_c, lat_c, lon_p, lat_p, Hm1_c
  double* d_gc_xy = nullptr;    // the same on the device
  double* d_cs = nullptr;       // output reductions: cs of the selected bins
  size_t cs_cap = 0;
  double* d_gh64 = nullptr;     // boundary halo layers (f3d_ads_keep_boundary_halo)
  float* d_gh32 = nullptr;
  double* d_out = nullptr;      // four (nx+1)(ny+1) output fields
  bool radio_on = false;
  std::vector<int> rad_bin, rad_parent;
  std::vector<double> rad_kn, rad_pkn;
  double* d_radf = nullptr;       // z-sweep epilogue: this step's decay factors
  std::vector<double> radf_host;  // their host copy, for the dt they were made for
  double radf_dt = -1.0;
};

template <class T>
static int dalloc(f3d_ctx* c, T** p, size_t n) {
  void* q = nullptr;
  if (n == 0) n = 1;
  CK(cudaMalloc(&q, n * sizeof(T)));
  c->allocs.push_back(q);
  *p = reinterpret_cast<T*>(q);
  return 0;
}

static int upload_member(f3d_ctx* c) {
  CK(cudaMemcpyAsync(c->dm, &c->hm, sizeof(MemberDev), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// Build the work lists: blocks of 128 pencils per direction, one partial
// slot per block.
static int build_work(f3d_ctx* c) {
  long long nsp[3] = {(long long)c->ny * c->nz, (long long)c->nx * c->nz,
                      (long long)c->nx * c->ny};
  const int bpb = c->bpb;
  const int span = 32 * (kSweepWarps / bpb);  // spatial pencils per block
  const int nbg = (c->nb + bpb - 1) / bpb;
  int slot = 0;
  for (int d = 0; d < 3; ++d) {
    const int ng = (int)((nsp[d] + span - 1) / span);
    const int nb = ng * nbg;
    std::vector<WorkItem> w(nb);
    for (int g = 0, q = 0; g < ng; ++g)
      for (int bg = 0; bg < nbg; ++bg, ++q) w[q] = WorkItem{0, span * g, bg * bpb, slot + q};
    c->hm.part_base[d] = slot;
    c->hm.part_count[d] = nb;
    slot += nb;
    if (dalloc(c, &c->dwork[d], (size_t)nb)) return 1;
    CK(cudaMemcpy(c->dwork[d], w.data(), sizeof(WorkItem) * nb, cudaMemcpyHostToDevice));
    c->nblk[d] = nb;
  }
  if (dalloc(c, &c->hm.flux_part, 2 * (size_t)slot)) return 1;
  long long nprep = ((long long)(c->nx + 1) * c->ny * c->nz + (long long)(c->ny + 1) * c->nx * c->nz +
                     (long long)(c->nz + 1) * c->nx * c->ny + kPrepBlock - 1) /
                    kPrepBlock;
  std::vector<int> bm(nprep, 0);
  int first = 0;
  if (dalloc(c, &c->dprep_member, (size_t)nprep)) return 1;
  if (dalloc(c, &c->dprep_first, 1)) return 1;
  CK(cudaMemcpy(c->dprep_member, bm.data(), sizeof(int) * nprep, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->dprep_first, &first, sizeof(int), cudaMemcpyHostToDevice));
  c->nprep = (int)nprep;
  return 0;
}

// ---- bounded waits and the settling-velocity iteration limit -----------------
namespace f3d {
constexpr long long kDefaultWaitLimit = 1LL << 25;  // = kSpinLimit (step_dev.cuh)
static std::atomic<long long> g_wait_limit{kDefaultWaitLimit};
static std::atomic<int> g_vset_maxit{1000};
static std::atomic<int> g_zepi{0};
long long wait_limit() { return g_wait_limit.load(); }
int vset_maxit() { return g_vset_maxit.load(); }
int zsweep_epilogue() { return g_zepi.load(); }
}  // namespace f3d

extern "C" int f3d_set_zsweep_epilogue(int on) {
  g_zepi.store(on ? 1 : 0);
  return 0;
}

extern "C" int f3d_set_wait_limit(long long polls) {
  g_wait_limit.store(polls < 0 ? kDefaultWaitLimit : polls);
  return 0;
}

extern "C" int f3d_set_vset_maxit(int maxit) {
  if (maxit == 0 || maxit < -1) return set_err("f3d_set_vset_maxit: maxit %d (use >= 1, or -1 for 1000)", maxit);
  g_vset_maxit.store(maxit < 0 ? 1000 : maxit);
  return 0;
}

extern "C" int f3d_last_error(char* buf, int len) {
  if (!buf || len <= 0) return 1;
  snprintf(buf, (size_t)len, "%s", g_err.c_str());
  return 0;
}

extern "C" int f3d_ads_create(const f3d_dims* dims, int limiter, int time_marching,
                              int precision, int device, f3d_ctx** out) {
  if (!dims || !out) return set_err("f3d_ads_create: null argument");
  if (dims->nx < 1 || dims->ny < 1 || dims->nz < 1 || dims->nbins < 1)
    return set_err("f3d_ads_create: invalid dims %d %d %d %d", dims->nx, dims->ny, dims->nz,
                   dims->nbins);
  if (limiter < 1 || limiter > 3) return set_err("f3d_ads_create: limiter %d not in 1..3", limiter);
  if (time_marching < 1 || time_marching > 2)
    return set_err("f3d_ads_create: time_marching %d not in 1..2", time_marching);
  if (precision != F3D_PREC_FP64 && precision != F3D_PREC_FP32 && precision != F3D_PREC_FP32C)
    return set_err("f3d_ads_create: precision %d unknown", precision);
  if (precision != F3D_PREC_FP64 && !pencil_span_ok(dims->nx, dims->ny, dims->nz))
    return set_err("f3d_ads_create: grid %d x %d x %d too large for the precision form "
                   "((nx+1)(ny+1)(nz+1) must stay below 2^31); use the FP64 form", dims->nx, dims->ny,
                   dims->nz);
  const int cmp = precision == F3D_PREC_FP32C;
  if (cmp) precision = F3D_PREC_FP32;
  *out = nullptr;
  CK(cudaSetDevice(device));
  f3d_ctx* c = new f3d_ctx();
  c->nx = dims->nx; c->ny = dims->ny; c->nz = dims->nz; c->nb = dims->nbins;
  c->lim = limiter; c->tm = time_marching; c->prec = precision; c->device = device;
  c->cmp = cmp;
  if (const char* e = getenv("F3D_BINS_PER_BLOCK")) {
    int v = atoi(e);
    if (v == 1 || v == 2 || v == 4) c->bpb = v;
  }
  memset(&c->hm, 0, sizeof(MemberDev));
  MemberDev& m = c->hm;
  m.nx = c->nx; m.ny = c->ny; m.nz = c->nz; m.nb = c->nb;
  m.wfac = 1.0f;
  m.wfacd = 1.0;
  const size_t nx = c->nx, ny = c->ny, nz = c->nz, nb = c->nb;
  const size_t ncell = nx * ny * nz;
  int rc = 0;
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return set_err("f3d_ads_create: stream creation failed");
  }
  double* tmp;
  if (precision == F3D_PREC_FP64) rc |= dalloc(c, &m.c64, ncell * nb);
  else rc |= dalloc(c, &m.c32, ncell * nb);
  rc |= dalloc(c, &m.acum, nx * ny * nb);
  rc |= dalloc(c, &tmp, 2 * (nx + 1) * ny * nz); m.ux[0] = tmp; m.ux[1] = tmp + (nx + 1) * ny * nz;
  rc |= dalloc(c, &tmp, 2 * (ny + 1) * nx * nz); m.vy[0] = tmp; m.vy[1] = tmp + (ny + 1) * nx * nz;
  rc |= dalloc(c, &tmp, 2 * (nz + 1) * nx * ny); m.wz[0] = tmp; m.wz[1] = tmp + (nz + 1) * nx * ny;
  rc |= dalloc(c, &tmp, (nx + 2) * ny * nz); m.k1x = tmp;
  rc |= dalloc(c, &tmp, (ny + 2) * nx * nz); m.k2y = tmp;
  rc |= dalloc(c, &tmp, (nz + 2) * nx * ny); m.k3z = tmp;
  rc |= dalloc(c, &tmp, nb * (nz + 1) * nx * ny); m.vs = tmp;
  if (precision == F3D_PREC_FP64) {
    rc |= dalloc(c, &m.ucur, (nx + 1) * ny * nz);
    rc |= dalloc(c, &m.vcur, (ny + 1) * nx * nz);
    rc |= dalloc(c, &m.wcur, (nz + 1) * nx * ny);
    rc |= dalloc(c, &tmp, (nx + 1) * ny * nz); m.kkf[0] = tmp;
    rc |= dalloc(c, &tmp, (ny + 1) * nx * nz); m.kkf[1] = tmp;
    rc |= dalloc(c, &tmp, (nz + 1) * nx * ny); m.kkf[2] = tmp;
    double4* g4;
    rc |= dalloc(c, &g4, nx + 1); m.geo[0] = g4;
    rc |= dalloc(c, &g4, ny + 1); m.geo[1] = g4;
    rc |= dalloc(c, &g4, nz + 1); m.geo[2] = g4;
  } else {
    float* f;
    float4* f4;
    rc |= dalloc(c, &f4, (nx + 1) * ny * nz); m.f4[0] = f4;
    rc |= dalloc(c, &f4, (ny + 1) * nx * nz); m.f4[1] = f4;
    rc |= dalloc(c, &f4, (nz + 1) * nx * ny); m.f4[2] = f4;
    rc |= dalloc(c, &f, nb * (nz + 1) * nx * ny); m.vs32 = f;
    rc |= dalloc(c, &f, nx); m.rdx1b32 = f;
    rc |= dalloc(c, &f, ny); m.rdx2b32 = f;
    rc |= dalloc(c, &f, nz); m.rdx3b32 = f;
    if (cmp) {
      rc |= dalloc(c, &m.c32lo, ncell * nb);
      rc |= dalloc(c, &tmp, nx); m.rdxb64[0] = tmp;
      rc |= dalloc(c, &tmp, ny); m.rdxb64[1] = tmp;
      rc |= dalloc(c, &tmp, nz); m.rdxb64[2] = tmp;
      float2* f2;
      rc |= dalloc(c, &f2, nx); m.rdxb2[0] = f2;
      rc |= dalloc(c, &f2, ny); m.rdxb2[1] = f2;
      rc |= dalloc(c, &f2, nz); m.rdxb2[2] = f2;
    }
  }
  rc |= dalloc(c, &tmp, nx + 4); m.dx1p = tmp;
  rc |= dalloc(c, &tmp, nx + 3); m.dx1b = tmp;
  rc |= dalloc(c, &tmp, ny + 4); m.dx2p = tmp;
  rc |= dalloc(c, &tmp, ny + 3); m.dx2b = tmp;
  rc |= dalloc(c, &tmp, nz + 4); m.dx3p = tmp;
  rc |= dalloc(c, &tmp, nz + 3); m.dx3b = tmp;
  rc |= dalloc(c, &tmp, ny); m.hm1 = tmp;
  rc |= dalloc(c, &tmp, ny + 4); m.hm2 = tmp;
  rc |= dalloc(c, &tmp, nx * ny); m.hm3 = tmp;
  rc |= dalloc(c, &m.flux_tot, 12);
  rc |= dalloc(c, &m.flux_step, 6);
  rc |= dalloc(c, &c->d_red, (size_t)c->mass_nblk * nb + 64);
  rc |= dalloc(c, &c->d_nfail, 4);
  size_t stage = std::max({(nx + 4) * (ny + 4) * (nz + 4) * nb, nx * ny * (nz + 3) * nb,
                           2 * (nx + 3) * ny * nz, 2 * (ny + 3) * nx * nz, 2 * (nz + 3) * nx * ny,
                           (nx + 4) * ny * nz, (ny + 4) * nx * nz, (nz + 4) * nx * ny});
  rc |= dalloc(c, &c->staging, stage);
  c->staging_elems = stage;
  rc |= dalloc(c, &c->dm, 1);
  if (rc == 0) rc |= build_work(c);
  if (rc == 0 && cudaMallocHost(&c->h_pin, 4096) != cudaSuccess) rc = set_err("pinned alloc failed");
  if (rc) {
    std::string keep = g_err;
    f3d_ads_destroy(c);
    g_err = keep;
    return 1;
  }
  CK(cudaMemsetAsync(m.c64 ? (void*)m.c64 : (void*)m.c32, 0,
                     ncell * nb * (m.c64 ? sizeof(double) : sizeof(float)), c->st));
  if (m.c32lo) CK(cudaMemsetAsync(m.c32lo, 0, ncell * nb * sizeof(float), c->st));
  CK(cudaMemsetAsync(m.acum, 0, nx * ny * nb * sizeof(double), c->st));
  CK(cudaMemsetAsync(m.flux_tot, 0, 12 * sizeof(double), c->st));
  CK(cudaMemsetAsync(m.flux_step, 0, 6 * sizeof(double), c->st));
  if (upload_member(c)) return 1;
  *out = c;
  return 0;
}

extern "C" int f3d_ads_destroy(f3d_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  for (void* p : c->allocs) cudaFree(p);
  if (c->d_rhoc_tc) cudaFree(c->d_rhoc_tc);
  if (c->h_pin) cudaFreeHost(c->h_pin);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return 0;
}

static int h2d(f3d_ctx* c, void* dst, const void* src, size_t bytes) {
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->st));
  return 0;
}

extern "C" int f3d_ads_set_grid(f3d_ctx* c, const double* dX1_p, const double* dX1_b,
                                const double* dX2_p, const double* dX2_b, const double* dX3_p,
                                const double* dX3_b, const double* Hm1_p, const double* Hm2_p,
                                const double* Hm3_p) {
  if (!c) return set_err("f3d_ads_set_grid: null context");
  if (!dX1_p || !dX1_b || !dX2_p || !dX2_b || !dX3_p || !dX3_b || !Hm1_p || !Hm2_p || !Hm3_p)
    return set_err("f3d_ads_set_grid: null array");
  CK(cudaSetDevice(c->device));
  MemberDev& m = c->hm;
  const size_t nx = c->nx, ny = c->ny, nz = c->nz;
  if (h2d(c, (void*)m.dx1p, dX1_p, (nx + 4) * 8) || h2d(c, (void*)m.dx1b, dX1_b, (nx + 3) * 8) ||
      h2d(c, (void*)m.dx2p, dX2_p, (ny + 4) * 8) || h2d(c, (void*)m.dx2b, dX2_b, (ny + 3) * 8) ||
      h2d(c, (void*)m.dx3p, dX3_p, (nz + 4) * 8) || h2d(c, (void*)m.dx3b, dX3_b, (nz + 3) * 8) ||
      h2d(c, (void*)m.hm1, Hm1_p, ny * 8) || h2d(c, (void*)m.hm2, Hm2_p, (ny + 4) * 8) ||
      h2d(c, (void*)m.hm3, Hm3_p, nx * ny * 8))
    return 1;
  c->dX1_p.assign(dX1_p, dX1_p + nx + 4);
  c->dX2_p.assign(dX2_p, dX2_p + ny + 4);
  c->dX3_p.assign(dX3_p, dX3_p + nz + 4);
  c->Hm1_p.assign(Hm1_p, Hm1_p + ny);
  c->Hm2_p.assign(Hm2_p, Hm2_p + ny + 4);
  c->Hm3_p.assign(Hm3_p, Hm3_p + nx * ny);
  if (c->prec == F3D_PREC_FP64) {
    // geo[p+1] = {dxp(p), RN(1/dxp(p)), dxb(p), RN(1/dxb(p))}, p = -1..n-1
    // (reference offsets +2 / +1); the reciprocals feed div_rn_recip
    const double* dp[3] = {dX1_p, dX2_p, dX3_p};
    const double* db[3] = {dX1_b, dX2_b, dX3_b};
    const size_t nn[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d) {
      std::vector<double4> g(nn[d] + 1);
      for (size_t q = 0; q <= nn[d]; ++q) {
        double a = dp[d][q + 1], b = db[d][q];
        if (!(std::fabs(a) >= 0x1p-100 && std::fabs(a) <= 0x1p100 && std::fabs(b) >= 0x1p-100 &&
              std::fabs(b) <= 0x1p100))
          return set_err("f3d_ads_set_grid: grid spacing %g / %g outside [2^-100, 2^100]", a, b);
        g[q] = make_double4(a, 1.0 / a, b, 1.0 / b);
      }
      CK(cudaMemcpy((void*)m.geo[d], g.data(), g.size() * sizeof(double4), cudaMemcpyHostToDevice));
    }
  }
  if (c->prec == F3D_PREC_FP32) {
    std::vector<float> r1(nx), r2(ny), r3(nz);
    for (size_t i = 0; i < nx; ++i) r1[i] = (float)(1.0 / dX1_b[i + 1]);
    for (size_t j = 0; j < ny; ++j) r2[j] = (float)(1.0 / dX2_b[j + 1]);
    for (size_t k = 0; k < nz; ++k) r3[k] = (float)(1.0 / dX3_b[k + 1]);
    CK(cudaMemcpy((void*)m.rdx1b32, r1.data(), nx * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void*)m.rdx2b32, r2.data(), ny * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void*)m.rdx3b32, r3.data(), nz * 4, cudaMemcpyHostToDevice));
    if (m.c32lo) {
      std::vector<double> q1(nx), q2(ny), q3(nz);
      for (size_t i = 0; i < nx; ++i) q1[i] = 1.0 / dX1_b[i + 1];
      for (size_t j = 0; j < ny; ++j) q2[j] = 1.0 / dX2_b[j + 1];
      for (size_t k = 0; k < nz; ++k) q3[k] = 1.0 / dX3_b[k + 1];
      CK(cudaMemcpy((void*)m.rdxb64[0], q1.data(), nx * 8, cudaMemcpyHostToDevice));
      CK(cudaMemcpy((void*)m.rdxb64[1], q2.data(), ny * 8, cudaMemcpyHostToDevice));
      CK(cudaMemcpy((void*)m.rdxb64[2], q3.data(), nz * 8, cudaMemcpyHostToDevice));
      const std::vector<double>* qs[3] = {&q1, &q2, &q3};
      for (int d = 0; d < 3; ++d) {
        std::vector<float2> p2(qs[d]->size());
        for (size_t q = 0; q < p2.size(); ++q) {
          const float h = (float)(*qs[d])[q];
          p2[q] = make_float2(h, (float)((*qs[d])[q] - (double)h));
        }
        CK(cudaMemcpy((void*)m.rdxb2[d], p2.data(), p2.size() * sizeof(float2), cudaMemcpyHostToDevice));
      }
    }
  }
  CK(cudaStreamSynchronize(c->st));
  c->grid_set = true;
  return 0;
}

// Upload one reference-layout array through the staging buffer and convert.
static int upload_conv(f3d_ctx* c, int which, const double* host, size_t elems, double* dst) {
  if (elems > c->staging_elems) return set_err("staging buffer too small");
  CK(cudaMemcpyAsync(c->staging, host, elems * 8, cudaMemcpyHostToDevice, c->st));
  launch_conv(which, c->staging, dst, c->nx, c->ny, c->nz, c->nb, c->st);
  CKL();
  CK(cudaStreamSynchronize(c->st));  // the host array may change after return
  return 0;
}

extern "C" int f3d_ads_set_meteo(f3d_ctx* c, const double* u, const double* v, const double* w,
                                 const double* k1, const double* k2, const double* k3,
                                 const double* vs, double t_its, double t_ite) {
  if (!c) return set_err("f3d_ads_set_meteo: null context");
  if (!u || !v || !w || !k1 || !k2 || !k3) return set_err("f3d_ads_set_meteo: null array");
  if (!(t_ite != t_its)) return set_err("f3d_ads_set_meteo: t_ite == t_its");
  CK(cudaSetDevice(c->device));
  MemberDev& m = c->hm;
  const size_t nx = c->nx, ny = c->ny, nz = c->nz, nb = c->nb;
  if (upload_conv(c, 0, u, 2 * (nx + 3) * ny * nz, const_cast<double*>(m.ux[0])) ||
      upload_conv(c, 1, v, 2 * (ny + 3) * nx * nz, const_cast<double*>(m.vy[0])) ||
      upload_conv(c, 2, w, 2 * (nz + 3) * nx * ny, const_cast<double*>(m.wz[0])) ||
      upload_conv(c, 3, k1, (nx + 4) * ny * nz, const_cast<double*>(m.k1x)) ||
      upload_conv(c, 4, k2, (ny + 4) * nx * nz, const_cast<double*>(m.k2y)) ||
      upload_conv(c, 5, k3, (nz + 4) * nx * ny, const_cast<double*>(m.k3z)))
    return 1;
  if (vs && upload_conv(c, 6, vs, nx * ny * (nz + 3) * nb, const_cast<double*>(m.vs))) return 1;
  c->t_its = t_its;
  c->t_ite = t_ite;
  m.t_its = t_its;
  m.t_ite = t_ite;
  if (upload_member(c)) return 1;
  if (c->prec == F3D_PREC_FP32) {
    launch_fp32_fields(c->dm, 0, c->st);
  } else {
    launch_face_kk(c->dm, 0, c->st);
  }
  CKL();
  CK(cudaStreamSynchronize(c->st));
  c->meteo_set = true;
  return 0;
}

extern "C" int f3d_ads_set_terrain(f3d_ctx* c, int map_v, double X3max, const double* X3_c,
                                   const double* X3_p, const double* dhdx_p, const double* dhdy_p) {
  if (!c) return set_err("f3d_ads_set_terrain: null context");
  if (map_v < 0 || map_v > 2) return set_err("f3d_ads_set_terrain: mapping %d not implemented", map_v);
  if (map_v != 0 && (!X3_c || !X3_p || !dhdx_p || !dhdy_p || !(X3max > 0.0)))
    return set_err("f3d_ads_set_terrain: sigma mappings need X3max > 0, X3_c, X3_p and the slopes");
  CK(cudaSetDevice(c->device));
  const size_t nx = c->nx, ny = c->ny, nz = c->nz;
  if (!c->d_terrain && dalloc(c, &c->d_terrain, (nz + 1) + nz + 2 * nx * ny)) return 1;
  if (map_v != 0) {
    CK(cudaMemcpy(c->d_terrain, X3_c, (nz + 1) * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_terrain + nz + 1, X3_p, nz * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_terrain + 2 * nz + 1, dhdx_p, nx * ny * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_terrain + 2 * nz + 1 + nx * ny, dhdy_p, nx * ny * 8, cudaMemcpyHostToDevice));
  }
  c->map_v = map_v;
  c->X3max = map_v != 0 ? X3max : 1.0;
  return 0;
}

// The meteo term from corner fields (F3D_update_meteo_term compute part):
// uploads the corner winds of both snapshots, lets fill_k write the
// unscaled diffusion into dk1..dk3 (reference layouts), then staggers and
// scales on the device.
template <class FillK>
static int meteo_corners_impl(f3d_ctx* c, const char* who, const double* uc, const double* vc,
                              const double* wc, size_t extra, double t_its, double t_ite,
                              FillK fill_k) {
  if (!c) return set_err("%s: null context", who);
  if (!c->grid_set) return set_err("%s: grid not set", who);
  if (!uc || !vc || !wc) return set_err("%s: null corner wind", who);
  if (!(t_ite != t_its)) return set_err("%s: t_ite == t_its", who);
  CK(cudaSetDevice(c->device));
  const size_t nx = c->nx, ny = c->ny, nz = c->nz;
  const size_t ncor = (nx + 1) * (ny + 1) * (nz + 1);
  const size_t n1 = (nx + 4) * ny * nz, n2 = nx * (ny + 4) * nz, n3 = nx * ny * (nz + 4);
  const size_t need = 6 * ncor + n1 + n2 + n3 + extra;
  if (need > c->met_cap) {
    c->d_met = nullptr;  // the old buffer stays in the context's allocation list
    if (dalloc(c, &c->d_met, need)) return 1;
    c->met_cap = need;
  }
  double* duc = c->d_met;
  double* dvc = duc + 2 * ncor;
  double* dwc = dvc + 2 * ncor;
  double* dk1 = dwc + 2 * ncor;
  double* dk2 = dk1 + n1;
  double* dk3 = dk2 + n2;
  double* dextra = dk3 + n3;
  CK(cudaMemcpyAsync(duc, uc, 2 * ncor * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dvc, vc, 2 * ncor * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dwc, wc, 2 * ncor * 8, cudaMemcpyHostToDevice, c->st));
  if (fill_k(duc, dvc, dk1, dk2, dk3, dextra)) return 1;
  MemberDev& m = c->hm;
  MetGeo g;
  g.nx = c->nx;
  g.ny = c->ny;
  g.nz = c->nz;
  g.map_v = c->map_v;
  g.X3max = c->X3max;
  g.X3c = c->d_terrain;
  g.X3p = c->d_terrain ? c->d_terrain + nz + 1 : nullptr;
  g.dhdx = c->d_terrain ? c->d_terrain + 2 * nz + 1 : nullptr;
  g.dhdy = c->d_terrain ? c->d_terrain + 2 * nz + 1 + nx * ny : nullptr;
  g.hm1 = m.hm1;
  g.hm2 = m.hm2;
  g.hm3 = m.hm3;
  launch_meteo_corners(g, duc, dvc, dwc, dk1, dk2, dk3, const_cast<double*>(m.ux[0]),
                       const_cast<double*>(m.vy[0]), const_cast<double*>(m.wz[0]),
                       const_cast<double*>(m.k1x), const_cast<double*>(m.k2y),
                       const_cast<double*>(m.k3z), c->st);
  c->launches += 9;
  CKL();
  c->t_its = t_its;
  c->t_ite = t_ite;
  m.t_its = t_its;
  m.t_ite = t_ite;
  if (upload_member(c)) return 1;
  if (c->prec == F3D_PREC_FP32) {
    launch_fp32_fields(c->dm, 0, c->st);
  } else {
    launch_face_kk(c->dm, 0, c->st);
  }
  CKL();
  CK(cudaStreamSynchronize(c->st));
  c->meteo_set = true;
  return 0;
}

extern "C" int f3d_ads_set_meteo_corners(f3d_ctx* c, const double* uc, const double* vc,
                                         const double* wc, const double* k1, const double* k2,
                                         const double* k3, double kh, double kv, double t_its,
                                         double t_ite) {
  const bool kgiven = k1 || k2 || k3;
  if (kgiven && !(k1 && k2 && k3))
    return set_err("f3d_ads_set_meteo_corners: give all of k1, k2, k3 or none");
  return meteo_corners_impl(
      c, "f3d_ads_set_meteo_corners", uc, vc, wc, 0, t_its, t_ite,
      [&](double*, double*, double* dk1, double* dk2, double* dk3, double*) -> int {
        const size_t nx = c->nx, ny = c->ny, nz = c->nz;
        if (kgiven) {
          CK(cudaMemcpyAsync(dk1, k1, (nx + 4) * ny * nz * 8, cudaMemcpyHostToDevice, c->st));
          CK(cudaMemcpyAsync(dk2, k2, nx * (ny + 4) * nz * 8, cudaMemcpyHostToDevice, c->st));
          CK(cudaMemcpyAsync(dk3, k3, nx * ny * (nz + 4) * 8, cudaMemcpyHostToDevice, c->st));
        } else {
          launch_meteo_kconst(c->nx, c->ny, c->nz, kh, kv, dk1, dk2, dk3, c->st);
          c->launches += 1;
        }
        return 0;
      });
}

extern "C" int f3d_ads_set_meteo_corners_kdiffu(f3d_ctx* c, const double* uc, const double* vc,
                                                const double* wc, const double* tvc,
                                                const double* pblh, const double* mon,
                                                const double* ust, const double* h_c,
                                                const f3d_kdiffu* kd, double t_its, double t_ite) {
  const char* who = "f3d_ads_set_meteo_corners_kdiffu";
  if (!c || !kd) return set_err("%s: null argument", who);
  if (kd->modkh != 1 && kd->modkh != 2 && kd->modkh != 4)
    return set_err("Horizontal diffusion parameterization not implemented ");
  if (kd->modkv != 1 && kd->modkv != 3)
    return set_err("Horizontal diffusion parameterization not implemented ");  // sic, mod_Phys.F90:660
  if (kd->map_h == 2 || kd->map_h == 3) return set_err("Mapping not implemented yet");
  if (kd->map_h != 0 && kd->map_h != 1) return set_err("Incorrect horizontal mapping");
  const bool vsim = kd->modkv == 3;
  if (vsim && (!tvc || !pblh || !mon || !ust || !h_c))
    return set_err("%s: the similarity K needs tvc, pblh, mon, ust and h_c", who);
  if (vsim && !c->d_zc)
    return set_err("%s: corner heights not set (f3d_ads_set_corner_heights)", who);
  const size_t nx = c->grid_set ? c->nx : 0, ny = c->grid_set ? c->ny : 0, nz = c->grid_set ? c->nz : 0;
  const size_t ncor = (nx + 1) * (ny + 1) * (nz + 1), n2d = nx * ny, nc2 = (nx + 1) * (ny + 1);
  const size_t extra = (vsim ? 2 * ncor + 3 * n2d + nc2 : 0) + (kd->modkh == 4 ? n2d : 0);
  return meteo_corners_impl(
      c, who, uc, vc, wc, extra, t_its, t_ite,
      [&](double* duc, double* dvc, double* dk1, double* dk2, double* dk3, double* dx) -> int {
        MemberDev& m = c->hm;
        KdArgs a;
        memset(&a, 0, sizeof(a));
        a.nx = c->nx;
        a.ny = c->ny;
        a.nz = c->nz;
        a.modkh = kd->modkh;
        a.modkv = kd->modkv;
        a.kh0 = kd->kh0;
        a.kv0 = kd->kv0;
        a.rams_cs = kd->rams_cs;
        a.khn0 = kd->map_h == 0 ? 4000.0 : 0.036;  // mod_Phys.F90:449-459
        a.dlon = kd->dlon;
        a.dlat = kd->dlat;
        a.s = kd->s_time;
        a.uc0 = duc;
        a.uc1 = duc + ncor;
        a.vc0 = dvc;
        a.vc1 = dvc + ncor;
        a.dx1p = m.dx1p;
        a.dx2p = m.dx2p;
        a.hm1 = m.hm1;
        a.hm2 = m.hm2;
        a.k1 = dk1;
        a.k2 = dk2;
        a.k3 = dk3;
        a.zc = c->d_zc;
        double* p = dx;
        if (vsim) {
          CK(cudaMemcpyAsync(p, tvc, 2 * ncor * 8, cudaMemcpyHostToDevice, c->st));
          a.tvc0 = p;
          a.tvc1 = p + ncor;
          p += 2 * ncor;
          const double* src[3] = {pblh, mon, ust};
          const double** dst[3] = {&a.pblh, &a.mon, &a.ust};
          for (int q = 0; q < 3; ++q) {
            CK(cudaMemcpyAsync(p, src[q], n2d * 8, cudaMemcpyHostToDevice, c->st));
            *dst[q] = p;
            p += n2d;
          }
          CK(cudaMemcpyAsync(p, h_c, nc2 * 8, cudaMemcpyHostToDevice, c->st));
          a.hc = p;
          p += nc2;
        }
        if (kd->modkh == 4) {  // kmh = 0.075 (dx dy)^(2/3) with the host's pow (mod_Phys.F90:537)
          std::vector<double> dx1(nx + 4), dx2(ny + 4), h1(ny), h2(ny + 4), kmh(n2d);
          CK(cudaMemcpyAsync(dx1.data(), m.dx1p, dx1.size() * 8, cudaMemcpyDeviceToHost, c->st));
          CK(cudaMemcpyAsync(dx2.data(), m.dx2p, dx2.size() * 8, cudaMemcpyDeviceToHost, c->st));
          CK(cudaMemcpyAsync(h1.data(), m.hm1, h1.size() * 8, cudaMemcpyDeviceToHost, c->st));
          CK(cudaMemcpyAsync(h2.data(), m.hm2, h2.size() * 8, cudaMemcpyDeviceToHost, c->st));
          CK(cudaStreamSynchronize(c->st));
          for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
              const double ddx = dx1[i + 2] * h1[j], ddy = dx2[j + 2] * h2[j + 2];
              kmh[i + nx * j] = 0.075 * std::pow(ddx * ddy, 2.0 / 3.0);
            }
          CK(cudaMemcpyAsync(p, kmh.data(), n2d * 8, cudaMemcpyHostToDevice, c->st));
          CK(cudaStreamSynchronize(c->st));  // kmh is freed when this scope ends
          a.kmh = p;
          p += n2d;
        }
        launch_kdiffu(a, c->st);
        c->launches += 2;
        return 0;
      });
}

extern "C" int f3d_ads_set_wet_deposition(f3d_ctx* c, double a, double b, const double* pre,
                                          const double* pblh, const double* h_c, const double* z_c,
                                          const int* bin_cat, const double* bin_diam) {
  if (!c) return set_err("f3d_ads_set_wet_deposition: null context");
  if (!bin_cat) {
    c->wet_on = false;
    return 0;
  }
  if (!pre || !pblh || !h_c || !z_c || !bin_diam) return set_err("f3d_ads_set_wet_deposition: null array");
  if (!c->grid_set) return set_err("f3d_ads_set_wet_deposition: grid not set");
  if (c->nb > 64) return set_err("f3d_ads_set_wet_deposition: at most 64 bins");
  CK(cudaSetDevice(c->device));
  const size_t ncol = (size_t)c->nx * c->ny;
  std::vector<double> powpb;
  std::vector<int> ktop;
  if (!wet_tables(c->nx, c->ny, c->nz, b, pre, pblh, h_c, z_c, powpb, ktop))
    return set_err("f3d_ads_set_wet_deposition: heights not increasing with k");
  if (!c->d_powpb) {
    if (dalloc(c, &c->d_powpb, ncol) || dalloc(c, &c->d_ktop, ncol) ||
        dalloc(c, &c->d_awet, ncol * c->nb))
      return 1;
    CK(cudaMemset(c->d_awet, 0, ncol * c->nb * 8));
  }
  CK(cudaMemcpy(c->d_powpb, powpb.data(), ncol * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_ktop, ktop.data(), ncol * 4, cudaMemcpyHostToDevice));
  c->wet_mask = wet_bin_mask(c->nb, bin_cat, bin_diam);
  c->wet_a = a;
  c->wet_on = true;
  return 0;
}

extern "C" int f3d_ads_set_radionuclides(f3d_ctx* c, const int* bin_cat, const int* bin_spe) {
  if (!c) return set_err("f3d_ads_set_radionuclides: null context");
  c->radio_on = false;
  c->rad_bin.clear();
  c->rad_parent.clear();
  c->rad_kn.clear();
  c->rad_pkn.clear();
  if (!bin_cat || !bin_spe) return 0;
  if (c->nb > 64) return set_err("f3d_ads_set_radionuclides: at most 64 bins");
  RadioSpec r;
  int bad = 0;
  const int rc = radio_spec(c->nb, bin_cat, bin_spe, r, &bad);
  if (rc == 1) return set_err("The number of SR90 and Y90 classes must be equal.");
  if (rc == 2) return set_err("Invalid radionuclide type: species %d", bad);
  c->rad_bin = r.bin;
  c->rad_parent = r.parent;
  c->rad_kn = r.kn;
  c->rad_pkn = r.pkn;
  c->radio_on = !c->rad_bin.empty();
  return 0;
}

extern "C" int f3d_ads_get_awet(f3d_ctx* c, double* my_awet) {
  if (!c || !my_awet) return set_err("f3d_ads_get_awet: null argument");
  const size_t nx = c->nx, ny = c->ny, nb = c->nb;
  std::vector<double> d(nx * ny * nb, 0.0);
  if (c->d_awet) {
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaMemcpy(d.data(), c->d_awet, d.size() * 8, cudaMemcpyDeviceToHost));
  }
  // my_awet(ips-2:ipe+2, jps-2:jpe+2, nbins), halos zero
  std::fill(my_awet, my_awet + (nx + 4) * (ny + 4) * nb, 0.0);
  for (size_t b = 0; b < nb; ++b)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i)
        my_awet[(i + 2) + (nx + 4) * ((j + 2) + (ny + 4) * b)] = d[(b * ny + j) * nx + i];
  return 0;
}

// Boundary halo layers <-> the reference's halo-inclusive state arrays:
// gh_gather_ref / gh_scatter_ref (phys_host.h).
static void gh_gather(const f3d_ctx* c, const double* my_c, std::vector<double>& g) {
  gh_gather_ref(c->nx, c->ny, c->nz, c->nb, my_c, g);
}

static void gh_scatter(const f3d_ctx* c, const std::vector<double>& g, double* my_c) {
  gh_scatter_ref(c->nx, c->ny, c->nz, c->nb, g, my_c);
}

static int gh_upload(f3d_ctx* c, const std::vector<double>& g) {
  MemberDev& m = c->hm;
  if (m.gh64) {
    CK(cudaMemcpy(m.gh64, g.data(), g.size() * 8, cudaMemcpyHostToDevice));
  } else if (m.gh32) {
    std::vector<float> t(g.size());
    for (size_t q = 0; q < g.size(); ++q) t[q] = (float)g[q];
    CK(cudaMemcpy(m.gh32, t.data(), t.size() * 4, cudaMemcpyHostToDevice));
  }
  return 0;
}

extern "C" int f3d_ads_keep_boundary_halo(f3d_ctx* c, int on) {
  if (!c) return set_err("f3d_ads_keep_boundary_halo: null context");
  CK(cudaSetDevice(c->device));
  MemberDev& m = c->hm;
  if (!on) {
    m.gh64 = nullptr;  // the buffers stay with the context until it is destroyed
    m.gh32 = nullptr;
    return upload_member(c);
  }
  const size_t n = (size_t)gh_per_bin(c->nx, c->ny, c->nz) * c->nb;
  if (c->prec == F3D_PREC_FP64) {
    if (!c->d_gh64 && dalloc(c, &c->d_gh64, n)) return 1;
    CK(cudaMemset(c->d_gh64, 0, n * 8));
    m.gh64 = c->d_gh64;
  } else {
    if (!c->d_gh32 && dalloc(c, &c->d_gh32, n)) return 1;
    CK(cudaMemset(c->d_gh32, 0, n * 4));
    m.gh32 = c->d_gh32;
  }
  return upload_member(c);
}

static int check_ready(f3d_ctx* c, const char* who);

// ---- gravity current: F3D_add_radial_wind (mod_F3D.F90:978-1226) ----------
// The scalars of the current for a time, on the host with the C library's
// sqrt and pow (mod_F3D.F90:1026-1070).  Returns false where the routine
// returns early (outside [start_time, end_time] or no mass flow).
static bool gc_args(const f3d_ctx* c, double time, GcArgs* g, double st[7]) {
  if (!c->gc_set) {
    memset(g, 0, sizeof(*g));
    for (int q = 0; q < 7; ++q) st[q] = 0.0;
    return false;
  }
  const double* lon_c = c->gc_host.data();          // layout of f3d_ads_set_gravity_current
  const double* lat_c = lon_c + (c->nx + 1);
  const double* hm1_c = lat_c + (c->ny + 1) + c->nx + c->ny;
  if (!gc_scalars(c->gc_p, lon_c, lat_c, hm1_c, time, g, st)) return false;
  g->lon_c = c->d_gc_xy;
  g->lat_c = g->lon_c + (c->nx + 1);
  g->lon_p = g->lat_c + (c->ny + 1);
  g->lat_p = g->lon_p + c->nx;
  g->hm1_c = g->lat_p + c->ny;
  g->hm1_p = c->hm.hm1;
  g->zc = c->d_zc;
  return true;
}

extern "C" int f3d_ads_set_gravity_current(f3d_ctx* c, const double params[11], const double* lon_c,
                                           const double* lat_c, const double* lon_p,
                                           const double* lat_p, const double* Hm1_c) {
  if (!c || !params) return set_err("f3d_ads_set_gravity_current: null argument");
  if (!c->grid_set) return set_err("f3d_ads_set_gravity_current: grid not set");
  if (!c->d_zc)
    return set_err("f3d_ads_set_gravity_current: corner heights not set (f3d_ads_set_corner_heights)");
  CK(cudaSetDevice(c->device));
  const size_t n = (size_t)(c->nx + 1) + (c->ny + 1) + c->nx + c->ny + (c->ny + 1);
  if (lon_c || lat_c || lon_p || lat_p || Hm1_c) {
    if (!lon_c || !lat_c || !lon_p || !lat_p || !Hm1_c)
      return set_err("f3d_ads_set_gravity_current: give all five coordinate arrays");
    c->gc_host.resize(n);
    double* h = c->gc_host.data();
    const size_t o_lat_c = c->nx + 1, o_lon_p = o_lat_c + c->ny + 1, o_lat_p = o_lon_p + c->nx,
                 o_hm1_c = o_lat_p + c->ny;
    memcpy(h, lon_c, (c->nx + 1) * 8);
    memcpy(h + o_lat_c, lat_c, (c->ny + 1) * 8);
    memcpy(h + o_lon_p, lon_p, c->nx * 8);
    memcpy(h + o_lat_p, lat_p, c->ny * 8);
    memcpy(h + o_hm1_c, Hm1_c, (c->ny + 1) * 8);
    if (!c->d_gc_xy && dalloc(c, &c->d_gc_xy, n)) return 1;
    CK(cudaMemcpy(c->d_gc_xy, h, n * 8, cudaMemcpyHostToDevice));
  } else if (c->gc_host.size() != n) {
    return set_err("f3d_ads_set_gravity_current: coordinates not given");
  }
  if (c->prec == F3D_PREC_FP32 && !c->hm.gc4[0]) {
    MemberDev& m = c->hm;
    if (dalloc(c, &m.gc4[0], (size_t)(c->nx + 1) * c->ny * c->nz) ||
        dalloc(c, &m.gc4[1], (size_t)(c->ny + 1) * c->nx * c->nz))
      return 1;
    if (upload_member(c)) return 1;
  }
  memcpy(c->gc_p, params, sizeof(c->gc_p));
  c->gc_set = true;
  return 0;
}

extern "C" int f3d_ads_gravity_current_time_step(f3d_ctx* c, double time, double stime,
                                                 int criterion, double cfl, double run_end,
                                                 int* active, double* my_dt, double* gl_dt,
                                                 double state[7]) {
  if (check_ready(c, "f3d_ads_gravity_current_time_step")) return 1;
  if (!active || !my_dt || !gl_dt)
    return set_err("f3d_ads_gravity_current_time_step: null output");
  if (criterion != 1 && criterion != 2)
    return set_err("f3d_ads_gravity_current_time_step: criterion %d not in 1..2", criterion);
  GcArgs g;
  double st[7];
  *active = gc_args(c, time, &g, st) ? 1 : 0;
  if (state)
    for (int q = 0; q < 7; ++q) state[q] = st[q];
  if (!*active) return 0;
  CK(cudaSetDevice(c->device));
  CK(cudaMemsetAsync(c->d_red, 0, 3 * sizeof(double), c->st));
  launch_cfl(c->dm, 0, stime, criterion, c->d_red, c->st, &g);
  CKL();
  CK(cudaMemcpyAsync(c->h_pin, c->d_red, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double m = std::max(std::max(c->h_pin[0], c->h_pin[1]), c->h_pin[2]);  // mod_Grid.F90:1125-1127
  if (m > 0.0) m = 1.0 / m;
  m = cfl * m;
  *my_dt = std::min(m, run_end);
  *gl_dt = std::min(m, run_end);
  return 0;
}

extern "C" int f3d_ads_set_corner_heights(f3d_ctx* c, const double* z_c) {
  if (!c || !z_c) return set_err("f3d_ads_set_corner_heights: null argument");
  CK(cudaSetDevice(c->device));
  const size_t n = (size_t)(c->nx + 1) * (c->ny + 1) * (c->nz + 1);
  if (!c->d_zc && dalloc(c, &c->d_zc, n)) return 1;
  CK(cudaMemcpy(c->d_zc, z_c, n * 8, cudaMemcpyHostToDevice));
  return 0;
}

extern "C" int f3d_ads_output_species(f3d_ctx* c, const int* bin_in, int col_du, double* con_sur,
                                      double* col_mass, double* cloud_top, double* grn_load) {
  if (!c || !bin_in) return set_err("f3d_ads_output_species: null argument");
  if (!c->grid_set) return set_err("f3d_ads_output_species: grid not set");
  if (c->nb > 64) return set_err("f3d_ads_output_species: at most 64 bins");
  if ((con_sur || col_mass || cloud_top) && !c->d_zc)
    return set_err("f3d_ads_output_species: corner heights not set (f3d_ads_set_corner_heights)");
  CK(cudaSetDevice(c->device));
  const size_t ncol = (size_t)(c->nx + 1) * (c->ny + 1);
  if (!c->d_out && dalloc(c, &c->d_out, 4 * ncol)) return 1;
  MemberDev& m = c->hm;
  OutArgs a;
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  a.nb = c->nb;
  a.mask = 0;
  for (int q = 0; q < c->nb; ++q)
    if (bin_in[q]) a.mask |= 1ull << q;
  a.col_du = col_du;
  a.c64 = m.c64;
  a.c32 = m.c32;
  a.c32lo = m.c32lo;
  a.acum = m.acum;
  a.awet = c->d_awet;
  a.hm1 = m.hm1;
  a.hm2 = m.hm2;
  a.hm3 = m.hm3;
  a.zc = c->d_zc;
  a.gh64 = m.gh64;
  a.gh32 = m.gh32;
  if (con_sur || col_mass || cloud_top) {
    const size_t ncs = (size_t)__builtin_popcountll(a.mask) * c->nx * c->ny * c->nz;
    const size_t need = ncs + (size_t)(c->nz + 1) * ncol;
    if (need > c->cs_cap) {
      if (dalloc(c, &c->d_cs, need)) return 1;  // the old buffer stays in the allocation list
      c->cs_cap = need;
    }
    a.cs = c->d_cs;
    a.wbuf = c->d_cs + ncs;
  }
  double* outs[4] = {con_sur, col_mass, cloud_top, grn_load};
  double* dev[4];
  for (int q = 0; q < 4; ++q) dev[q] = outs[q] ? c->d_out + q * ncol : nullptr;
  a.con_sur = dev[0];
  a.col_mass = dev[1];
  a.cloud_top = dev[2];
  a.grn_load = dev[3];
  launch_out_columns(a, c->st);
  c->launches += 1;
  CKL();
  for (int q = 0; q < 4; ++q)
    if (outs[q]) CK(cudaMemcpyAsync(outs[q], dev[q], ncol * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int f3d_ads_set_source(f3d_ctx* c, int n, const int* ijk, const double* s) {
  if (!c) return set_err("f3d_ads_set_source: null context");
  if (n < 0 || (n > 0 && (!ijk || !s))) return set_err("f3d_ads_set_source: bad arguments");
  if (!c->grid_set) return set_err("f3d_ads_set_source: grid not set");
  CK(cudaSetDevice(c->device));
  MemberDev& m = c->hm;
  std::vector<int> cell(n);
  std::vector<double> vol(n);
  for (int q = 0; q < n; ++q) {
    int i = ijk[3 * q] - 1, j = ijk[3 * q + 1] - 1, k = ijk[3 * q + 2] - 1;
    if (i < 0 || i >= c->nx || j < 0 || j >= c->ny || k < 0 || k >= c->nz)
      return set_err("f3d_ads_set_source: cell %d (%d,%d,%d) outside the domain", q, i + 1, j + 1,
                     k + 1);
    cell[q] = i + c->nx * (j + c->ny * k);
    // vol = dX*dY*dZ*(Hm1*Hm2*Hm3)   mod_F3D.F90:1466
    double dX = c->dX1_p[i + 2], dY = c->dX2_p[j + 2], dZ = c->dX3_p[k + 2];
    double Hm1 = c->Hm1_p[j], Hm2 = c->Hm2_p[j + 2], Hm3 = c->Hm3_p[i + (size_t)c->nx * j];
    volatile double a = dX * dY;
    volatile double b = a * dZ;
    volatile double h = Hm1 * Hm2;
    volatile double h3 = h * Hm3;
    vol[q] = b * h3;
  }
  if (n > c->src_cap) {
    int cap = std::max(n, 64);
    int* dc;
    double *ds, *dv;
    if (dalloc(c, &dc, (size_t)cap) || dalloc(c, &ds, (size_t)cap * c->nb) ||
        dalloc(c, &dv, (size_t)cap))
      return 1;
    m.src_cell = dc;
    m.src_s = ds;
    m.src_vol = dv;
    c->src_cap = cap;
  }
  if (n > 0) {
    CK(cudaMemcpyAsync((void*)m.src_cell, cell.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync((void*)m.src_s, s, sizeof(double) * n * c->nb, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync((void*)m.src_vol, vol.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  }
  m.nsrc = n;
  return upload_member(c);
}

extern "C" int f3d_ads_set_source_dense(f3d_ctx* c, const double* my_s) {
  if (!c || !my_s) return set_err("f3d_ads_set_source_dense: null argument");
  const size_t nx = c->nx, ny = c->ny, nz = c->nz, nb = c->nb, ncell = nx * ny * nz;
  std::vector<int> ijk;
  std::vector<double> s;
  for (size_t q = 0; q < ncell; ++q) {
    bool any = false;
    for (size_t b = 0; b < nb; ++b) any |= (my_s[q + ncell * b] != 0.0);
    if (!any) continue;
    ijk.push_back((int)(q % nx) + 1);
    ijk.push_back((int)((q / nx) % ny) + 1);
    ijk.push_back((int)(q / (nx * ny)) + 1);
    for (size_t b = 0; b < nb; ++b) s.push_back(my_s[q + ncell * b]);
  }
  return f3d_ads_set_source(c, (int)(ijk.size() / 3), ijk.data(), s.data());
}

extern "C" int f3d_ads_upload_state(f3d_ctx* c, const double* my_c, const double* my_acum) {
  if (!c) return set_err("f3d_ads_upload_state: null context");
  CK(cudaSetDevice(c->device));
  MemberDev& m = c->hm;
  const size_t nx = c->nx, ny = c->ny, nz = c->nz, nb = c->nb;
  if (my_c) {
    if (c->prec == F3D_PREC_FP64) {
      if (upload_conv(c, 7, my_c, (nx + 4) * (ny + 4) * (nz + 4) * nb, m.c64)) return 1;
    } else {
      // convert on the host, rounding to nearest FP32 (compensated form: the
      // pair hi = RN(c), lo = RN(c - hi))
      std::vector<float> tmp(nx * ny * nz * nb), tlo(m.c32lo ? tmp.size() : 0);
      for (size_t b = 0; b < nb; ++b)
        for (size_t k = 0; k < nz; ++k)
          for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
              const size_t q = ((b * nz + k) * ny + j) * nx + i;
              const double v =
                  my_c[(i + 2) + (nx + 4) * ((j + 2) + (ny + 4) * ((k + 2) + (nz + 4) * b))];
              tmp[q] = (float)v;
              if (m.c32lo) tlo[q] = (float)(v - (double)tmp[q]);
            }
      CK(cudaMemcpy(m.c32, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice));
      if (m.c32lo) CK(cudaMemcpy(m.c32lo, tlo.data(), tlo.size() * 4, cudaMemcpyHostToDevice));
    }
  }
  if (my_acum && upload_conv(c, 8, my_acum, (nx + 4) * (ny + 4) * nb, m.acum)) return 1;
  if (my_c && (m.gh64 || m.gh32)) {
    std::vector<double> g;
    gh_gather(c, my_c, g);
    if (gh_upload(c, g)) return 1;
  }
  return 0;
}

extern "C" int f3d_ads_download_state(f3d_ctx* c, double* my_c, double* my_acum) {
  if (!c) return set_err("f3d_ads_download_state: null context");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  MemberDev& m = c->hm;
  const size_t nx = c->nx, ny = c->ny, nz = c->nz, nb = c->nb;
  if (my_c) {
    std::vector<double> tmp(nx * ny * nz * nb);
    if (c->prec == F3D_PREC_FP64) {
      CK(cudaMemcpy(tmp.data(), m.c64, tmp.size() * 8, cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> t32(tmp.size());
      CK(cudaMemcpy(t32.data(), m.c32, t32.size() * 4, cudaMemcpyDeviceToHost));
      for (size_t q = 0; q < t32.size(); ++q) tmp[q] = t32[q];
      if (m.c32lo) {
        CK(cudaMemcpy(t32.data(), m.c32lo, t32.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < t32.size(); ++q) tmp[q] = tmp[q] + (double)t32[q];
      }
    }
    const size_t X = nx + 4, Y = ny + 4, Z = nz + 4;
    for (size_t b = 0; b < nb; ++b)
      for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j) {
          const double* row = &tmp[((b * nz + k) * ny + j) * nx];
          double* dst = &my_c[2 + X * ((j + 2) + Y * ((k + 2) + Z * b))];
          memcpy(dst, row, nx * 8);
          // zero-gradient face ghosts of the final state
          dst[-1] = dst[-2] = row[0];
          dst[nx] = dst[nx + 1] = row[nx - 1];
        }
    for (size_t b = 0; b < nb; ++b)
      for (size_t k = 0; k < nz; ++k)
        for (size_t i = 0; i < nx; ++i) {
          double lo = tmp[((b * nz + k) * ny + 0) * nx + i];
          double hi = tmp[((b * nz + k) * ny + (ny - 1)) * nx + i];
          for (int g = 0; g < 2; ++g) {
            my_c[(i + 2) + X * (g + Y * ((k + 2) + Z * b))] = lo;
            my_c[(i + 2) + X * ((ny + 2 + g) + Y * ((k + 2) + Z * b))] = hi;
          }
        }
    for (size_t b = 0; b < nb; ++b)
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          double lo = tmp[((b * nz + 0) * ny + j) * nx + i];
          double hi = tmp[((b * nz + (nz - 1)) * ny + j) * nx + i];
          for (int g = 0; g < 2; ++g) {
            my_c[(i + 2) + X * ((j + 2) + Y * (g + Z * b))] = lo;
            my_c[(i + 2) + X * ((j + 2) + Y * ((nz + 2 + g) + Z * b))] = hi;
          }
        }
    if (m.gh64 || m.gh32) {  // the kept boundary halo layers replace the zero-gradient ghosts
      std::vector<double> g((size_t)gh_per_bin(c->nx, c->ny, c->nz) * nb);
      if (m.gh64) {
        CK(cudaMemcpy(g.data(), m.gh64, g.size() * 8, cudaMemcpyDeviceToHost));
      } else {
        std::vector<float> t(g.size());
        CK(cudaMemcpy(t.data(), m.gh32, t.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < t.size(); ++q) g[q] = t[q];
      }
      gh_scatter(c, g, my_c);
    }
  }
  if (my_acum) {
    std::vector<double> tmp(nx * ny * nb);
    CK(cudaMemcpy(tmp.data(), m.acum, tmp.size() * 8, cudaMemcpyDeviceToHost));
    for (size_t b = 0; b < nb; ++b)
      for (size_t j = 0; j < ny; ++j)
        memcpy(&my_acum[2 + (nx + 4) * ((j + 2) + (ny + 4) * b)], &tmp[(b * ny + j) * nx], nx * 8);
  }
  return 0;
}

// ---- step ---------------------------------------------------------------
static int enqueue_sweep(f3d_ctx* c, int dir) {
  c->launches += 1;
  if (c->prec == F3D_PREC_FP64)
    launch_sweep64(dir, c->lim, c->tm, c->hm.epi_on, c->dm, c->dwork[dir], c->nblk[dir], c->bpb, c->st);
  else
    launch_sweep32(dir, c->lim, c->tm, c->cmp, c->hm.epi_on, c->dm, c->dwork[dir], c->nblk[dir], c->bpb,
                   c->st);
  CKL();
  return 0;
}

static int enqueue_prep(f3d_ctx* c, int mask) {
  if (c->prec == F3D_PREC_FP64) c->launches += 1;  // the FP32 form interpolates inside the sweeps
  if (c->prec == F3D_PREC_FP64)
    launch_prep64(c->dm, c->dprep_member, c->dprep_first, c->nprep, mask, c->st);
  else
    launch_prep32(c->dm, c->dprep_member, c->dprep_first, c->nprep, mask, c->st);
  CKL();
  return 0;
}

static int enqueue_source(f3d_ctx* c) {
  if (c->hm.nsrc <= 0) return 0;
  c->launches += 1;
  if (c->prec == F3D_PREC_FP64) launch_source64(c->dm, 1, c->st);
  else launch_source32(c->dm, 1, c->st);
  CKL();
  return 0;
}

static int check_ready(f3d_ctx* c, const char* who) {
  if (!c) return set_err("%s: null context", who);
  if (!c->grid_set) return set_err("%s: grid not set", who);
  if (!c->meteo_set) return set_err("%s: meteo not set", who);
  return 0;
}

// Decay factors exp(-kn dt) of the radionuclide bins and of their parents
// (host libm, as the CPU restatement evaluates them).
static void radio_factors(const std::vector<double>& kn, const std::vector<double>& pkn,
                          const std::vector<int>& parent, double dt, double* fact, double* pfact) {
  for (size_t q = 0; q < kn.size(); ++q) {
    fact[q] = exp(-kn[q] * dt);
    pfact[q] = parent[q] >= 0 ? exp(-pkn[q] * dt) : 1.0;
  }
}

// Configure the z sweep's wet deposition and decay epilogue for a step of dt:
// the member descriptor is uploaded when a field changes, the decay factors
// when dt changes.
static int sync_epilogue(f3d_ctx* c, double dt) {
  MemberDev& m = c->hm;
  const bool on = zsweep_epilogue() && (c->wet_on || c->radio_on);
  MemberDev want = m;
  want.epi_on = on ? 1 : 0;
  want.wet_mask = (on && c->wet_on) ? c->wet_mask : 0ull;
  want.wet_a = c->wet_a;
  want.powpb = c->d_powpb;
  want.ktop = c->d_ktop;
  want.awet = c->wet_on ? c->d_awet : nullptr;
  want.radf = nullptr;
  want.daughter_mask = 0ull;
  for (int b = 0; b < 64; ++b) want.rad_r[b] = -1;
  if (on && c->radio_on) {
    const size_t nr = c->rad_bin.size();
    if (!c->d_radf && dalloc(c, &c->d_radf, 2 * 64)) return 1;
    if (c->radf_dt != dt || c->radf_host.size() != 2 * nr) {
      c->radf_host.assign(2 * nr, 1.0);
      radio_factors(c->rad_kn, c->rad_pkn, c->rad_parent, dt, c->radf_host.data(),
                    c->radf_host.data() + nr);
      // from pageable memory: the call returns once the values are staged
      CK(cudaMemcpyAsync(c->d_radf, c->radf_host.data(), 2 * nr * 8, cudaMemcpyHostToDevice, c->st));
      c->radf_dt = dt;
    }
    want.radf = c->d_radf;
    for (size_t q = 0; q < nr; ++q) {
      want.rad_r[c->rad_bin[q]] = (signed char)q;
      if (c->rad_parent[q] >= 0) want.daughter_mask |= 1ull << c->rad_bin[q];
    }
  }
  if (memcmp(&want, &m, sizeof(MemberDev)) != 0) {
    m = want;
    if (upload_member(c)) return 1;
  }
  return 0;
}

// Wet deposition and radioactive decay after the sweeps (mod_F3D.F90:1497-1520).
// With the z sweep's epilogue on, only the daughter bins and the kept halo
// layers are left to k_radio.
static int enqueue_wet_radio(f3d_ctx* c, double dt) {
  MemberDev& m = c->hm;
  if (m.epi_on) {
    bool daughters = false;
    for (int p : c->rad_parent) daughters = daughters || p >= 0;
    if (!c->radio_on || !(daughters || m.gh64 || m.gh32)) return 0;
  }
  if (c->wet_on && !m.epi_on) {
    WetArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = c->nx;
    a.ny = c->ny;
    a.nz = c->nz;
    a.nb = c->nb;
    a.dta = dt * c->wet_a;
    a.powpb = c->d_powpb;
    a.ktop = c->d_ktop;
    a.dx3p = m.dx3p;
    a.awet = c->d_awet;
    a.c64 = m.c64;
    a.c32 = m.c32;
    a.c32lo = m.c32lo;
    a.mask = c->wet_mask;
    launch_wet(a, c->st);
    c->launches += 1;
    CKL();
  }
  if (c->radio_on) {
    RadioArgs r;
    memset(&r, 0, sizeof(r));
    r.nx = c->nx;
    r.ny = c->ny;
    r.nz = c->nz;
    r.nr = (int)c->rad_bin.size();
    for (int q = 0; q < r.nr; ++q) {
      r.bin[q] = c->rad_bin[q];
      r.parent[q] = c->rad_parent[q];
    }
    radio_factors(c->rad_kn, c->rad_pkn, c->rad_parent, dt, r.fact, r.pfact);
    r.tail = m.epi_on;
    r.c64 = m.c64;
    r.c32 = m.c32;
    r.c32lo = m.c32lo;
    r.acum = m.acum;
    r.awet = c->wet_on ? c->d_awet : nullptr;
    r.gh64 = m.gh64;
    r.gh32 = m.gh32;
    r.ngh = gh_per_bin(c->nx, c->ny, c->nz);
    launch_radio(r, c->st);
    c->launches += 1;
    CKL();
  }
  return 0;
}

static int enqueue_step(f3d_ctx* c, double dt, double time, int iiter) {
  // event slots: 0 start, 1 after prep+source, 2..4 after the 1st/2nd/z sweep, 5 end
  auto rec = [&](int k) { if (c->prof) cudaEventRecord(c->ev[k], c->st); };
  rec(0);
  // gravity current at this time; the precision form's sweeps are switched to
  // the precomputed winds before the step's parameters are set on the device
  // (the descriptor upload carries the host's copy of dt and stime)
  GcArgs gc;
  double gst[7];
  const bool gc_on = c->gc_set && gc_args(c, time, &gc, gst);
  const int fp32 = c->prec == F3D_PREC_FP32;
  if (fp32 && c->hm.gc_cur != (gc_on ? 1 : 0)) {
    c->hm.gc_cur = gc_on ? 1 : 0;
    if (upload_member(c)) return 1;
  }
  if (sync_epilogue(c, dt)) return 1;
  launch_set_step(c->dm, 0, dt, time, iiter, c->st);
  c->launches += 1;
  CKL();
  if (enqueue_prep(c, 7)) return 1;
  if (gc_on) {  // F3D_add_radial_wind on the interpolated winds (mod_F3D.F90:1443-1445)
    launch_gc_winds(c->dm, 0, c->nx, c->ny, c->nz, fp32, gc, c->st);
    c->launches += 1;
    CKL();
  }
  if (enqueue_source(c)) return 1;
  rec(1);
  const bool xfirst = (iiter % 2 == 0);  // mod_F3D.F90:1477-1487
  if (enqueue_sweep(c, xfirst ? DIR_X : DIR_Y)) return 1;
  rec(2);
  if (enqueue_sweep(c, xfirst ? DIR_Y : DIR_X)) return 1;
  rec(3);
  if (enqueue_sweep(c, DIR_Z)) return 1;
  rec(4);
  launch_flux_reduce(c->dm, 1, 7, c->st);
  c->launches += 1;
  CKL();
  if (enqueue_wet_radio(c, dt)) return 1;
  rec(5);
  if (c->prof) {
    CK(cudaEventSynchronize(c->ev[5]));
    float t[5];
    for (int k = 0; k < 5; ++k) CK(cudaEventElapsedTime(&t[k], c->ev[k], c->ev[k + 1]));
    c->prof_ms[0] += t[0];
    c->prof_ms[xfirst ? 1 : 2] += t[1];
    c->prof_ms[xfirst ? 2 : 1] += t[2];
    c->prof_ms[3] += t[3];
    c->prof_ms[4] += t[4];
    float tot;
    CK(cudaEventElapsedTime(&tot, c->ev[0], c->ev[5]));
    c->prof_ms[5] += tot;
    c->prof_steps += 1;
  }
  return 0;
}

extern "C" int f3d_ads_set_profiling(f3d_ctx* c, int on) {
  if (!c) return set_err("f3d_ads_set_profiling: null context");
  CK(cudaSetDevice(c->device));
  if (on && !c->ev[0])
    for (auto& e : c->ev) CK(cudaEventCreate(&e));
  c->prof = on != 0;
  for (double& x : c->prof_ms) x = 0.0;
  c->prof_steps = 0;
  return 0;
}

extern "C" int f3d_ads_launch_count(f3d_ctx* c, long long* count) {
  if (!c || !count) return set_err("f3d_ads_launch_count: null argument");
  *count = c->launches;
  return 0;
}

extern "C" int f3d_ads_get_profile(f3d_ctx* c, double ms[6], int* nsteps) {
  if (!c || !ms) return set_err("f3d_ads_get_profile: null argument");
  for (int k = 0; k < 6; ++k) ms[k] = c->prof_ms[k];
  if (nsteps) *nsteps = c->prof_steps;
  return 0;
}

extern "C" int f3d_ads_step(f3d_ctx* c, double dt, double time, int iiter, double fluxes[6]) {
  if (check_ready(c, "f3d_ads_step")) return 1;
  if (!fluxes) return set_err("f3d_ads_step: null fluxes");
  CK(cudaSetDevice(c->device));
  if (enqueue_step(c, dt, time, iiter)) return 1;
  CK(cudaMemcpyAsync(c->h_pin, c->hm.flux_step, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int q = 0; q < 6; ++q) fluxes[q] = fluxes[q] + c->h_pin[q];
  return 0;
}

extern "C" int f3d_ads_step_async(f3d_ctx* c, double dt, double time, int iiter) {
  if (check_ready(c, "f3d_ads_step_async")) return 1;
  CK(cudaSetDevice(c->device));
  return enqueue_step(c, dt, time, iiter);
}

extern "C" int f3d_ads_get_fluxes(f3d_ctx* c, double fluxes[6]) {
  if (!c || !fluxes) return set_err("f3d_ads_get_fluxes: null argument");
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(c->h_pin, c->hm.flux_tot, 12 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemsetAsync(c->hm.flux_tot, 0, 12 * sizeof(double), c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int q = 0; q < 6; ++q) fluxes[q] = fluxes[q] + (c->h_pin[q] - c->h_pin[6 + q]);
  return 0;
}

extern "C" int f3d_ads_synchronize(f3d_ctx* c) {
  if (!c) return set_err("f3d_ads_synchronize: null context");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int f3d_ads_get_stream(f3d_ctx* c, void** stream) {
  if (!c || !stream) return set_err("f3d_ads_get_stream: null argument");
  *stream = (void*)c->st;
  return 0;
}

extern "C" int f3d_ads_update_vcomps(f3d_ctx* c, double stime) {
  if (check_ready(c, "f3d_ads_update_vcomps")) return 1;
  CK(cudaSetDevice(c->device));
  c->hm.stime = stime;
  launch_set_dt_stime(c->dm, 0, 0.0, stime, c->st);
  CKL();
  return enqueue_prep(c, 3);
}

static int solve_dir(f3d_ctx* c, int dir, double dt, double* a, double* b, const char* who) {
  if (check_ready(c, who)) return 1;
  if (!a || !b) return set_err("%s: null flux argument", who);
  CK(cudaSetDevice(c->device));
  if (enqueue_sweep(c, dir)) return 1;
  launch_flux_reduce(c->dm, 1, 1 << dir, c->st);
  CKL();
  CK(cudaMemcpyAsync(c->h_pin, c->hm.flux_step, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  (void)dt;
  if (dir == DIR_X) { *a = *a + c->h_pin[0]; *b = *b + c->h_pin[1]; }
  if (dir == DIR_Y) { *a = *a + c->h_pin[2]; *b = *b + c->h_pin[3]; }
  if (dir == DIR_Z) { *a = *a + c->h_pin[5]; *b = *b + c->h_pin[4]; }
  return 0;
}

// The sweep kernels read dt and stime from the member descriptor; these
// entry points set them (stime only matters for z, whose wind is rebuilt).
extern "C" int f3d_ads_solve_along_x(f3d_ctx* c, double dt, double* W, double* E) {
  if (check_ready(c, "f3d_ads_solve_along_x")) return 1;
  launch_set_dt_stime(c->dm, 0, dt, c->hm.stime, c->st);
  return solve_dir(c, DIR_X, dt, W, E, "f3d_ads_solve_along_x");
}
extern "C" int f3d_ads_solve_along_y(f3d_ctx* c, double dt, double* S, double* N) {
  if (check_ready(c, "f3d_ads_solve_along_y")) return 1;
  launch_set_dt_stime(c->dm, 0, dt, c->hm.stime, c->st);
  return solve_dir(c, DIR_Y, dt, S, N, "f3d_ads_solve_along_y");
}
extern "C" int f3d_ads_solve_along_z(f3d_ctx* c, double dt, double stime, double* D, double* U) {
  if (check_ready(c, "f3d_ads_solve_along_z")) return 1;
  CK(cudaSetDevice(c->device));
  // rebuild the current w at stime (mod_ADS.F90:667) without touching u, v
  c->hm.stime = stime;
  launch_set_dt_stime(c->dm, 0, dt, stime, c->st);
  CKL();
  if (enqueue_prep(c, 4)) return 1;
  return solve_dir(c, DIR_Z, dt, D, U, "f3d_ads_solve_along_z");
}

extern "C" int f3d_ads_add_source(f3d_ctx* c, double dt) {
  if (check_ready(c, "f3d_ads_add_source")) return 1;
  CK(cudaSetDevice(c->device));
  launch_set_dt_stime(c->dm, 0, dt, c->hm.stime, c->st);
  CKL();
  if (enqueue_source(c)) return 1;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int f3d_ads_get_time_step(f3d_ctx* c, double stime, int criterion, double cfl,
                                     double run_end, double* my_dt, double* gl_dt) {
  if (check_ready(c, "f3d_ads_get_time_step")) return 1;
  if (!my_dt || !gl_dt) return set_err("f3d_ads_get_time_step: null output");
  if (criterion != 1 && criterion != 2)
    return set_err("f3d_ads_get_time_step: criterion %d not in 1..2", criterion);
  CK(cudaSetDevice(c->device));
  CK(cudaMemsetAsync(c->d_red, 0, 3 * sizeof(double), c->st));
  launch_cfl(c->dm, 0, stime, criterion, c->d_red, c->st);
  CKL();
  CK(cudaMemcpyAsync(c->h_pin, c->d_red, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double dt1 = c->h_pin[0], dt2 = c->h_pin[1], dt3 = c->h_pin[2];
  double m = std::max(std::max(dt1, dt2), dt3);  // mod_Grid.F90:1125-1127
  if (m > 0.0) m = 1.0 / m;
  m = cfl * m;
  *my_dt = std::min(m, run_end);
  *gl_dt = std::min(m, run_end);
  return 0;
}

// ADS_solve_1D (mod_ADS.F90:820-1053) of one pencil on the device; host
// arrays in the reference layouts (see include/fall3d_ads.h).
extern "C" int f3d_ads_solve_1d(int n, int limiter, double* c, const double* dxp,
                                const double* dxb, const double* u, const double* k, double dt,
                                const double bvalue[2], double flux[2], const int bcode[2],
                                int device) {
  if (n < 2 || !c || !dxp || !dxb || !u || !k || !bvalue || !flux || !bcode)
    return set_err("f3d_ads_solve_1d: bad arguments (n >= 2, no null arrays)");
  if (limiter < 1 || limiter > 3) return set_err("f3d_ads_solve_1d: limiter %d not in 1..3", limiter);
  for (int s = 0; s < 2; ++s)
    if (bcode[s] < -1 || bcode[s] > 2) return set_err("f3d_ads_solve_1d: bcode %d not in -1..2", bcode[s]);
  CK(cudaSetDevice(device));
  const size_t N = (size_t)n;
  const size_t tot = (N + 4) * 3 + (N + 3) * 2 + 2 + (6 * N + 14);
  double* d = nullptr;
  CK(cudaMalloc(&d, tot * sizeof(double)));
  double *dc = d, *dp = dc + N + 4, *dk = dp + N + 4, *db = dk + N + 4, *du = db + N + 3,
         *df = du + N + 3, *dw = df + 2;
  int rc = 0;
  const struct { double* dst; const double* src; size_t n; } up[6] = {
      {dc, c, N + 4}, {dp, dxp, N + 4}, {dk, k, N + 4}, {db, dxb, N + 3}, {du, u, N + 3}, {df, flux, 2}};
  for (int q = 0; q < 6 && !rc; ++q)
    if (cudaMemcpy(up[q].dst, up[q].src, up[q].n * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_err("f3d_ads_solve_1d: upload failed");
  if (!rc) {
    launch_ads_solve_1d(n, limiter, dc, dp, db, du, dk, dt, bvalue, bcode, df, dw, 0);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = set_err("f3d_ads_solve_1d: %s", cudaGetErrorString(e));
  }
  if (!rc && (cudaMemcpy(c, dc, (N + 4) * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
              cudaMemcpy(flux, df, 2 * 8, cudaMemcpyDeviceToHost) != cudaSuccess))
    rc = set_err("f3d_ads_solve_1d: download failed");
  cudaFree(d);
  return rc;
}

// Finite scan of the device-resident inputs and state.  Bits of *mask:
// 1 state, 2 ground deposit, 4 u, 8 v, 16 w (both meteo snapshots),
// 32 k1, 64 k2, 128 k3, 256 settling velocity.
extern "C" int f3d_ads_check_finite(f3d_ctx* c, int* mask) {
  if (!c || !mask) return set_err("f3d_ads_check_finite: null argument");
  CK(cudaSetDevice(c->device));
  const MemberDev& m = c->hm;
  const long long nx = c->nx, ny = c->ny, nz = c->nz, nb = c->nb, ncell = nx * ny * nz;
  unsigned int* dmask = reinterpret_cast<unsigned int*>(c->d_nfail) + 2;
  CK(cudaMemsetAsync(dmask, 0, sizeof(unsigned int), c->st));
  launch_nonfinite(m.c64, ncell * nb, 0, dmask, c->st);
  launch_nonfinite(m.c32, ncell * nb, 0, dmask, c->st);
  launch_nonfinite(m.c32lo, ncell * nb, 0, dmask, c->st);
  launch_nonfinite(m.acum, nx * ny * nb, 1, dmask, c->st);
  launch_nonfinite(m.ux[0], 2 * (nx + 1) * ny * nz, 2, dmask, c->st);
  launch_nonfinite(m.vy[0], 2 * (ny + 1) * nx * nz, 3, dmask, c->st);
  launch_nonfinite(m.wz[0], 2 * (nz + 1) * nx * ny, 4, dmask, c->st);
  launch_nonfinite(m.k1x, (nx + 2) * ny * nz, 5, dmask, c->st);
  launch_nonfinite(m.k2y, (ny + 2) * nx * nz, 6, dmask, c->st);
  launch_nonfinite(m.k3z, (nz + 2) * nx * ny, 7, dmask, c->st);
  launch_nonfinite(m.vs, nb * (nz + 1) * nx * ny, 8, dmask, c->st);
  CKL();
  unsigned int h = 0;
  CK(cudaMemcpyAsync(&h, dmask, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *mask = (int)h;
  return 0;
}

extern "C" int f3d_ads_mass_volume(f3d_ctx* c, double* mass, double* per_bin) {
  if (!c || !mass) return set_err("f3d_ads_mass_volume: null argument");
  if (!c->grid_set) return set_err("f3d_ads_mass_volume: grid not set");
  CK(cudaSetDevice(c->device));
  double* out = c->d_red + (size_t)c->mass_nblk * c->nb;
  if (c->nb > 64) return set_err("f3d_ads_mass_volume: more than 64 bins");
  launch_mass(c->dm, 0, c->nb, c->prec == F3D_PREC_FP32, c->d_red, c->mass_nblk, out, c->st);
  CKL();
  std::vector<double> pb(c->nb);
  CK(cudaMemcpyAsync(c->h_pin, out, c->nb * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double tot = 0.0, comp = 0.0;
  for (int b = 0; b < c->nb; ++b) {
    double x = c->h_pin[b], t = tot + x;
    comp += (std::fabs(tot) >= std::fabs(x)) ? (tot - t) + x : (x - t) + tot;
    tot = t;
    if (per_bin) per_bin[b] = x;
  }
  *mass = tot + comp;
  return 0;
}

extern "C" int f3d_ads_mass_sink(f3d_ctx* c, double* mass) {
  if (!c || !mass) return set_err("f3d_ads_mass_sink: null argument");
  if (!c->grid_set) return set_err("f3d_ads_mass_sink: grid not set");
  if (!c->d_awet) {  // no wet deposition: the sink is 0
    *mass = 0.0 + 0.0;
    return 0;
  }
  CK(cudaSetDevice(c->device));
  const size_t ncol = (size_t)c->nx * c->ny;
  if (!c->d_out && dalloc(c, &c->d_out, 4 * (size_t)(c->nx + 1) * (c->ny + 1))) return 1;
  launch_sink_cols(c->nx, c->ny, c->nb, c->d_awet, c->hm.dx1p, c->hm.dx2p, c->d_out, c->st);
  c->launches += 1;
  CKL();
  std::vector<double> col(ncol);
  CK(cudaMemcpyAsync(col.data(), c->d_out, ncol * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *mass = mass_sink_sum(c->nx, c->ny, col.data());
  return 0;
}

extern "C" int f3d_ads_mass_boundaries(const double fluxes[6], double* ground, double* lateral) {
  if (!fluxes || !ground || !lateral) return set_err("f3d_ads_mass_boundaries: null argument");
  *ground = std::fabs(fluxes[5]);
  *lateral = std::fabs(fluxes[0]) + std::fabs(fluxes[1]) + std::fabs(fluxes[2]) +
             std::fabs(fluxes[3]) + std::fabs(fluxes[4]);
  return 0;
}

extern "C" int f3d_vset_points(int model, int n, const double* diam, const double* rhop,
                               const double* psi, const double* rhoa, const double* visc,
                               double* vset, int* flags, int* iters) {
  if (n < 0) return set_err("f3d_vset_points: n < 0");
  if (n == 0) return 0;
  if (!diam || !rhop || !psi || !rhoa || !visc || !vset || !flags)
    return set_err("f3d_vset_points: null array");
  if (model < 1 || model > 7) return set_err("f3d_vset_points: settling velocity model %d not found", model);
  double* d = nullptr;
  int* fi = nullptr;
  size_t N = (size_t)n;
  if (cudaMalloc(&d, N * 6 * 8) != cudaSuccess) return set_err("f3d_vset_points: device alloc failed");
  if (cudaMalloc(&fi, (N * 2 + 1) * 4) != cudaSuccess) {
    cudaFree(d);
    return set_err("f3d_vset_points: device alloc failed");
  }
  int rc = 0;
  const double* srcs[5] = {diam, rhop, psi, rhoa, visc};
  for (int a = 0; a < 5 && !rc; ++a)
    if (cudaMemcpy(d + a * N, srcs[a], N * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_err("f3d_vset_points: copy failed");
  if (!rc && cudaMemset(fi + 2 * N, 0, 4) != cudaSuccess) rc = set_err("memset failed");
  if (!rc) {
    launch_vset_points(model, n, d, d + N, d + 2 * N, d + 3 * N, d + 4 * N, d + 5 * N, fi,
                       fi + N, fi + 2 * N, 0);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = set_err("f3d_vset_points: %s", cudaGetErrorString(e));
  }
  int nfail = 0;
  if (!rc && (cudaMemcpy(vset, d + 5 * N, N * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
              cudaMemcpy(flags, fi, N * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
              (iters && cudaMemcpy(iters, fi + N, N * 4, cudaMemcpyDeviceToHost) != cudaSuccess) ||
              cudaMemcpy(&nfail, fi + 2 * N, 4, cudaMemcpyDeviceToHost) != cudaSuccess))
    rc = set_err("f3d_vset_points: copy back failed");
  cudaFree(d);
  cudaFree(fi);
  if (rc) return rc;
  if (nfail) {
    set_err("no convergence in vset (%d points)", nfail);
    return 2;
  }
  return 0;
}

// Stage corner air density/temperature and the bin table on the device.
static int stage_vset_inputs(f3d_ctx* c, const double* rhoc, const double* tc, const double* diam,
                             const double* rhop, const double* psi, const int* bin_cat,
                             const int* is_aggregate, double** drho, double** dt, double** dpar,
                             int** dflags) {
  const size_t ncor = (size_t)(c->nx + 1) * (c->ny + 1) * (c->nz + 1);
  size_t need = 2 * ncor + 3 * (size_t)c->nb + (size_t)c->nb;
  if (need > c->rhoc_cap) {
    if (c->d_rhoc_tc) cudaFree(c->d_rhoc_tc);
    c->d_rhoc_tc = nullptr;
    c->rhoc_cap = 0;
    CK(cudaMalloc(&c->d_rhoc_tc, need * 8));
    c->rhoc_cap = need;
  }
  *drho = c->d_rhoc_tc;
  *dt = *drho + ncor;
  *dpar = *dt + ncor;
  *dflags = reinterpret_cast<int*>(*dpar + 3 * c->nb);
  std::vector<double> par(3 * c->nb);
  std::vector<int> fl(c->nb);
  for (int b = 0; b < c->nb; ++b) {
    par[3 * b] = diam[b];
    par[3 * b + 1] = rhop[b];
    par[3 * b + 2] = psi[b];
    fl[b] = bin_cat[b] | ((is_aggregate && is_aggregate[b]) ? (1 << 8) : 0);
  }
  CK(cudaMemcpyAsync(*drho, rhoc, ncor * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(*dt, tc, ncor * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(*dpar, par.data(), par.size() * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(*dflags, fl.data(), fl.size() * 4, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// After a new vs field: FP32 copies, optional download, non-convergence status.
static int finish_vset(f3d_ctx* c, int nfail, double* vs_out) {
  if (c->prec == F3D_PREC_FP32 && c->meteo_set) {
    launch_fp32_fields(c->dm, 0, c->st);
    CKL();
  }
  if (vs_out) {
    size_t n = (size_t)c->nx * c->ny * (c->nz + 3) * c->nb;
    if (n > c->staging_elems) return set_err("staging too small");
    launch_conv(9, c->hm.vs, c->staging, c->nx, c->ny, c->nz, c->nb, c->st);
    CKL();
    CK(cudaMemcpyAsync(vs_out, c->staging, n * 8, cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  if (nfail) {
    set_err("no convergence in vset (%d points)", nfail);
    return 2;
  }
  return 0;
}

extern "C" int f3d_ads_compute_vset(f3d_ctx* c, int model, const double* rhoc, const double* tc,
                                    const double* diam, const double* rhop, const double* psi,
                                    const int* bin_cat, const int* is_aggregate, double vset_fac,
                                    double* vs_out) {
  if (!c) return set_err("f3d_ads_compute_vset: null context");
  if (!c->grid_set) return set_err("f3d_ads_compute_vset: grid not set");
  if (!rhoc || !tc || !diam || !rhop || !psi || !bin_cat)
    return set_err("f3d_ads_compute_vset: null array");
  if (model < 1 || model > 7) return set_err("setling velocity model not found");
  CK(cudaSetDevice(c->device));
  double *drho, *dt, *dpar;
  int* dflags;
  if (stage_vset_inputs(c, rhoc, tc, diam, rhop, psi, bin_cat, is_aggregate, &drho, &dt, &dpar, &dflags))
    return 1;
  CK(cudaMemsetAsync(c->d_nfail, 0, 4, c->st));
  launch_vset_field(c->dm, 0, model, drho, dt, dpar, dflags, vset_fac, c->d_nfail, c->st);
  CKL();
  int nfail = 0;
  CK(cudaMemcpyAsync(c->h_pin, c->d_nfail, 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  memcpy(&nfail, c->h_pin, 4);
  return finish_vset(c, nfail, vs_out);
}

extern "C" int f3d_ads_compute_vset_mlp(f3d_ctx* c, f3d_mlp* h, const double* rhoc, const double* tc,
                                        const double* diam, const double* rhop, const double* psi,
                                        const int* bin_cat, const int* is_aggregate, double vset_fac,
                                        int refine, long long* nfallback, double* vs_out) {
  if (!c || !h) return set_err("f3d_ads_compute_vset_mlp: null handle");
  if (!c->grid_set) return set_err("f3d_ads_compute_vset_mlp: grid not set");
  if (!rhoc || !tc || !diam || !rhop || !psi || !bin_cat)
    return set_err("f3d_ads_compute_vset_mlp: null array");
  CK(cudaSetDevice(c->device));
  double *drho, *dt, *dpar;
  int* dflags;
  if (stage_vset_inputs(c, rhoc, tc, diam, rhop, psi, bin_cat, is_aggregate, &drho, &dt, &dpar, &dflags))
    return 1;
  int nfail = 0;
  if (mlp_vset_field(h, c->dm, 0, c->nx, c->ny, c->nz, c->nb, drho, dt, diam, rhop, psi, bin_cat,
                     is_aggregate, vset_fac, refine, c->st, nfallback, &nfail))
    return 1;
  c->launches += 1;
  return finish_vset(c, nfail, vs_out);
}

extern "C" int f3d_host_alloc(size_t bytes, void** ptr) {
  if (!ptr) return set_err("f3d_host_alloc: null pointer");
  CK(cudaMallocHost(ptr, bytes));
  return 0;
}
extern "C" int f3d_host_free(void* ptr) {
  CK(cudaFreeHost(ptr));
  return 0;
}
