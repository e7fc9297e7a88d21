// ens.cu -- host side of the batched ensemble (f3d_ens_* in fall3d_ads.h).
//
// All members of an ensemble live on one GPU in one member table.  Members of
// a grid class point at the class's grid, meteo and settling-velocity arrays;
// each member owns its concentration, deposit, source, fluxes and clock.  A
// step is either a short sequence of kernels (source, sweeps, flux
// reduction, clock) replayed from CUDA graphs, or one persistent cooperative
// kernel that runs the whole step with bounded grid barriers between phases.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fall3d_ads.h"
#include "f3d_common.cuh"
#include "phys_dev.cuh"
#include "phys_host.h"
#include "step_dev.cuh"

namespace f3d {
int set_error_msg(const char* fmt, ...);
void launch_sweep64(int dir, int lim, int tm, int epi, const MemberDev* members, const WorkItem* work,
                    int nblocks, int bpb, cudaStream_t st);
void launch_sweep32(int dir, int lim, int tm, int cmp, int epi, const MemberDev* members,
                    const WorkItem* work, int nblocks, int bpb, cudaStream_t st);
void launch_prep64(const MemberDev* members, const int* blk_member, const int* blk_first,
                   int nblocks, int mask, cudaStream_t st);
void launch_source64(const MemberDev* members, int nmembers, cudaStream_t st);
void launch_source32(const MemberDev* members, int nmembers, cudaStream_t st);
void launch_conv(int which, const double* in, double* out, int nx, int ny, int nz, int nb,
                 cudaStream_t st);
void launch_flux_reduce(const MemberDev* members, int nmembers, int dirmask, cudaStream_t st);
void launch_cfl(const MemberDev* members, int mi, double s, int criterion, double* out3,
                cudaStream_t st, const GcArgs* gc = nullptr);
void launch_mass(const MemberDev* members, int mi, int nb, int fp32, double* partials, int nblk,
                 double* out, cudaStream_t st);
void launch_vset_field(MemberDev* members, int mi, int model, const double* rhoc,
                       const double* tc, const double* bin_par, const int* bin_flags,
                       double vset_fac, int* nfail, cudaStream_t st);
int mlp_vset_field(f3d_mlp* h, const MemberDev* dm, int mi, int nx, int ny, int nz, int nb,
                   const double* drhoc, const double* dtc, const double* diam, const double* rhop,
                   const double* psi, const int* bin_cat, const int* is_aggregate, double vset_fac,
                   int refine, cudaStream_t st, long long* nfallback, int* nfail);
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
void launch_face_kk(MemberDev* members, int mi, cudaStream_t st);
void launch_gc_winds(MemberDev* members, int mi, int nx, int ny, int nz, int fp32, const GcArgs& g,
                     cudaStream_t st);
void launch_nonfinite(const double* p, long long n, int bit, unsigned int* mask, cudaStream_t st);
void launch_nonfinite(const float* p, long long n, int bit, unsigned int* mask, cudaStream_t st);
void launch_fp32_fields(MemberDev* members, int mi, cudaStream_t st);
void launch_set_steps(MemberDev* members, int n, const double* dt, const double* time, int iiter,
                      cudaStream_t st);
void launch_advance_clock(MemberDev* members, int n, cudaStream_t st);
void launch_finalize_dt(MemberDev* members, int n, const double* red, double cfl, double run_end,
                        cudaStream_t st);
int fused32_smem(int tm, int cmp);
int fused64_smem();
const void* fused32_func(int lim, int tm, int cmp);
const void* fused64_func(int lim, int tm);
}  // namespace f3d

using namespace f3d;

#define ECK(call)                                                                       \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return set_error_msg("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),      \
                           __FILE__, __LINE__);                                         \
  } while (0)
#define ECKL()                                                                          \
  do {                                                                                  \
    cudaError_t e_ = cudaGetLastError();                                                \
    if (e_ != cudaSuccess)                                                              \
      return set_error_msg("kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_),  \
                           __FILE__, __LINE__);                                         \
  } while (0)

namespace {

struct EnsClass {
  int nx = 0, ny = 0, nz = 0;
  int rep = -1;  // a member of the class, used to address class arrays in kernels
  double* ux = nullptr;  // [2][k][f][j]
  double* vy = nullptr;
  double* wz = nullptr;
  double* k1x = nullptr;
  double* k2y = nullptr;
  double* k3z = nullptr;
  double* vs = nullptr;
  double* kkf[3] = {nullptr, nullptr, nullptr};
  double4* geo[3] = {nullptr, nullptr, nullptr};
  float4* f4[3] = {nullptr, nullptr, nullptr};  // FP32 face data (MemberDev::f4)
  float* vs32 = nullptr;
  float* rdx[3] = {nullptr, nullptr, nullptr};
  double* rdx64[3] = {nullptr, nullptr, nullptr};  // compensated form: 1/dxb in FP64
  float2* rdx2[3] = {nullptr, nullptr, nullptr};   // and as FP32 pairs {hi, lo}
  double* dx[6] = {};   // dx1p dx1b dx2p dx2b dx3p dx3b
  double* hm[3] = {};   // hm1 hm2 hm3
  std::vector<double> dX1_p, dX2_p, dX3_p, Hm1_p, Hm2_p, Hm3_p;
  double t_its = 0.0, t_ite = 1.0;
  bool grid_set = false, meteo_set = false;
  int map_v = 0;                 // terrain mapping for the on-device meteo term
  double X3max = 1.0;
  double* terrain = nullptr;     // X3_c, X3_p, dhdx_p, dhdy_p
  double* powpb = nullptr;       // wet deposition: P^b per column
  int* ktop = nullptr;           // and the cells below the boundary-layer top
  bool wet_set = false;
  double* zc = nullptr;          // corner heights (output reductions, gravity current)
  std::vector<double> gc_host;   // lon_c, lat_c, lon_p, lat_p, Hm1_c of the class grid
  double* gc_xy = nullptr;       // the same on the device
};

}  // namespace

struct f3d_ens {
  int ncls = 0, nm = 0, nb = 0, lim = 2, tm = 2, prec = 0, device = 0;
  int cmp = 0;  // precision form with the compensated (hi + lo) state
  int mode = F3D_ENS_MODE_KERNELS, bpb = 4, ctas_per_sm = 0;
  // gravity current per member (F3D_add_radial_wind): parameters and whether set
  std::vector<std::vector<double>> gc_p;
  bool gc_any = false;
  cudaStream_t st = nullptr;
  std::vector<EnsClass> cls;
  std::vector<int> member_class;
  std::vector<MemberDev> hm;
  MemberDev* dm = nullptr;
  std::vector<void*> allocs;
  WorkItem* dwork[3] = {nullptr, nullptr, nullptr};
  int nwork[3] = {0, 0, 0};
  int* dprep_member = nullptr;
  int* dprep_first = nullptr;
  int nprep = 0;
  double* flux_part = nullptr;
  double* flux_tot = nullptr;   // [12 * nm]
  double* flux_step = nullptr;  // [6 * nm]
  double* d_red = nullptr;      // CFL maxima [3 * nm] and mass partials
  int mass_nblk = 296;
  unsigned int* counters = nullptr;  // persistent kernel: 6 phase counters + barrier
  int* d_err = nullptr;
  int* d_nfail = nullptr;
  double* staging = nullptr;
  size_t staging_elems = 0;
  double* h_pin = nullptr;
  size_t h_pin_elems = 0;
  int iiter = 0;
  bool dm_valid = false;  // the device member table has been written once
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  bool graph_ok = false;
  int fused_grid = 0;
  long long launches = 0;
  std::vector<void*> work_allocs;  // rebuilt with the tuning
  cudaEvent_t vev[2] = {nullptr, nullptr};  // around the last class vset kernel
  float vset_ms = 0.0f;
  double* d_met = nullptr;             // corner winds + unscaled diffusion staging
  size_t met_cap = 0;
  bool prof = false;                   // per-phase event timing (no graph)
  cudaEvent_t pev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double prof_ms[5] = {0, 0, 0, 0, 0};  // prep+source, x, y, z, flux+clock
  int prof_steps = 0;
  // wet deposition and radioactive decay after the sweeps (all members)
  bool wet_on = false;
  double wet_a = 0.0;
  unsigned long long wet_mask = 0;
  std::vector<double*> awet;           // per member [bin][j][i]
  bool radio_on = false;
  RadioSpec radio;
  double* d_radfact = nullptr;         // per member {fact[nr], pfact[nr]} for its dt
  size_t radfact_cap = 0;
  double* d_out = nullptr;             // output reductions: 4 (nx+1)(ny+1) fields
  size_t out_cap = 0;
  double* d_cs = nullptr;              // and the cs of the selected bins
  size_t cs_cap = 0;
};

namespace {

template <class T>
int ealloc(f3d_ens* e, T** p, size_t n) {
  void* q = nullptr;
  if (n == 0) n = 1;
  ECK(cudaMalloc(&q, n * sizeof(T)));
  e->allocs.push_back(q);
  *p = reinterpret_cast<T*>(q);
  return 0;
}

void drop_graphs(f3d_ens* e) {
  for (auto& g : e->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  e->graph_ok = false;
}

int update_radio_factors(f3d_ens* e, const double* dt);

// The device owns dt, time, stime and iiter once steps have run (device clock,
// CFL on the device): refresh them in the host mirror before re-uploading it.
int pull_dynamic(f3d_ens* e) {
  if (!e->dm || !e->dm_valid) return 0;
  std::vector<MemberDev> dev(e->nm);
  ECK(cudaStreamSynchronize(e->st));
  ECK(cudaMemcpy(dev.data(), e->dm, sizeof(MemberDev) * e->nm, cudaMemcpyDeviceToHost));
  for (int m = 0; m < e->nm; ++m) {
    e->hm[m].dt = dev[m].dt;
    e->hm[m].time = dev[m].time;
    e->hm[m].stime = dev[m].stime;
    e->hm[m].iiter = dev[m].iiter;
  }
  return 0;
}

int upload_members(f3d_ens* e) {
  if (pull_dynamic(e)) return 1;
  ECK(cudaMemcpyAsync(e->dm, e->hm.data(), sizeof(MemberDev) * e->nm, cudaMemcpyHostToDevice,
                      e->st));
  e->dm_valid = true;
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

// Work lists of the three sweeps.  Items of one class are ordered spatial
// tile -> member -> bin group, so the blocks that read the same class face
// fields at the same place run back to back.  Flux slots stay contiguous
// per member.
int build_work(f3d_ens* e) {
  for (void* p : e->work_allocs) cudaFree(p);
  e->work_allocs.clear();
  const int bpb = e->bpb;
  const int span = 32 * (4 / bpb);
  const int nbg = (e->nb + bpb - 1) / bpb;
  int slot = 0;
  std::vector<std::vector<WorkItem>> lists(3);
  for (int d = 0; d < 3; ++d) {
    for (int mi = 0; mi < e->nm; ++mi) {
      const EnsClass& c = e->cls[e->member_class[mi]];
      long long nsp = d == 0 ? (long long)c.ny * c.nz : d == 1 ? (long long)c.nx * c.nz
                                                               : (long long)c.nx * c.ny;
      const int ng = (int)((nsp + span - 1) / span);
      e->hm[mi].part_base[d] = slot;
      e->hm[mi].part_count[d] = ng * nbg;
      slot += ng * nbg;
    }
    for (int ci = 0; ci < e->ncls; ++ci) {
      const EnsClass& c = e->cls[ci];
      long long nsp = d == 0 ? (long long)c.ny * c.nz : d == 1 ? (long long)c.nx * c.nz
                                                               : (long long)c.nx * c.ny;
      const int ng = (int)((nsp + span - 1) / span);
      for (int g = 0; g < ng; ++g)
        for (int mi = 0; mi < e->nm; ++mi) {
          if (e->member_class[mi] != ci) continue;
          for (int bg = 0; bg < nbg; ++bg)
            lists[d].push_back(WorkItem{mi, span * g, bg * bpb, e->hm[mi].part_base[d] + g * nbg + bg});
        }
    }
  }
  for (int d = 0; d < 3; ++d) {
    void* p = nullptr;
    ECK(cudaMalloc(&p, std::max<size_t>(1, lists[d].size()) * sizeof(WorkItem)));
    e->work_allocs.push_back(p);
    e->dwork[d] = static_cast<WorkItem*>(p);
    ECK(cudaMemcpy(p, lists[d].data(), lists[d].size() * sizeof(WorkItem), cudaMemcpyHostToDevice));
    e->nwork[d] = (int)lists[d].size();
  }
  void* fp = nullptr;
  ECK(cudaMalloc(&fp, 2 * (size_t)std::max(1, slot) * sizeof(double)));
  e->work_allocs.push_back(fp);
  e->flux_part = static_cast<double*>(fp);
  for (int mi = 0; mi < e->nm; ++mi) e->hm[mi].flux_part = e->flux_part;
  // FP64 prep blocks (256 faces each) per member
  std::vector<int> pm, pf(e->nm);
  for (int mi = 0; mi < e->nm; ++mi) {
    const EnsClass& c = e->cls[e->member_class[mi]];
    long long nf = (long long)(c.nx + 1) * c.ny * c.nz + (long long)(c.ny + 1) * c.nx * c.nz +
                   (long long)(c.nz + 1) * c.nx * c.ny;
    pf[mi] = (int)pm.size();
    for (long long q = 0; q < (nf + 255) / 256; ++q) pm.push_back(mi);
  }
  void *a = nullptr, *b = nullptr;
  ECK(cudaMalloc(&a, std::max<size_t>(1, pm.size()) * sizeof(int)));
  ECK(cudaMalloc(&b, std::max<size_t>(1, pf.size()) * sizeof(int)));
  e->work_allocs.push_back(a);
  e->work_allocs.push_back(b);
  ECK(cudaMemcpy(a, pm.data(), pm.size() * sizeof(int), cudaMemcpyHostToDevice));
  ECK(cudaMemcpy(b, pf.data(), pf.size() * sizeof(int), cudaMemcpyHostToDevice));
  e->dprep_member = static_cast<int*>(a);
  e->dprep_first = static_cast<int*>(b);
  e->nprep = (int)pm.size();
  return upload_members(e);
}

}  // namespace

extern "C" int f3d_ens_destroy(f3d_ens* e) {
  if (!e) return 0;
  cudaSetDevice(e->device);
  if (e->st) cudaStreamSynchronize(e->st);
  drop_graphs(e);
  for (void* p : e->work_allocs) cudaFree(p);
  for (void* p : e->allocs) cudaFree(p);
  if (e->d_met) cudaFree(e->d_met);
  if (e->h_pin) cudaFreeHost(e->h_pin);
  for (auto& ev : e->vev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : e->pev)
    if (ev) cudaEventDestroy(ev);
  if (e->st) cudaStreamDestroy(e->st);
  delete e;
  return 0;
}

extern "C" int f3d_ens_create(int nclasses, const f3d_dims* dims, int nmembers,
                              const f3d_ens_member* members, int limiter, int time_marching,
                              int precision, int device, f3d_ens** out) {
  if (!out || !dims || !members || nclasses < 1 || nmembers < 1)
    return set_error_msg("f3d_ens_create: bad arguments");
  if (limiter < 1 || limiter > 3) return set_error_msg("f3d_ens_create: limiter %d not in 1..3", limiter);
  if (time_marching < 1 || time_marching > 2)
    return set_error_msg("f3d_ens_create: time_marching %d not in 1..2", time_marching);
  if (precision != F3D_PREC_FP64 && precision != F3D_PREC_FP32 && precision != F3D_PREC_FP32C)
    return set_error_msg("f3d_ens_create: precision %d unknown", precision);
  const int cmp = precision == F3D_PREC_FP32C;
  if (cmp) precision = F3D_PREC_FP32;
  const int nb = dims[0].nbins;
  for (int c = 0; c < nclasses; ++c)
    if (dims[c].nx < 1 || dims[c].ny < 1 || dims[c].nz < 1 || dims[c].nbins != nb)
      return set_error_msg("f3d_ens_create: class %d dims invalid or bins differ", c);
  for (int c = 0; c < nclasses; ++c)
    if (precision != F3D_PREC_FP64 && !pencil_span_ok(dims[c].nx, dims[c].ny, dims[c].nz))
      return set_error_msg("f3d_ens_create: class %d grid too large for the precision form "
                           "((nx+1)(ny+1)(nz+1) must stay below 2^31)", c);
  for (int m = 0; m < nmembers; ++m)
    if (members[m].grid_class < 0 || members[m].grid_class >= nclasses)
      return set_error_msg("f3d_ens_create: member %d class %d out of range", m, members[m].grid_class);
  *out = nullptr;
  ECK(cudaSetDevice(device));
  f3d_ens* e = new f3d_ens();
  e->ncls = nclasses;
  e->nm = nmembers;
  e->nb = nb;
  e->lim = limiter;
  e->tm = time_marching;
  e->prec = precision;
  e->cmp = cmp;
  e->device = device;
  e->cls.resize(nclasses);
  e->member_class.resize(nmembers);
  e->hm.resize(nmembers);
  int rc = 0;
  if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete e;
    return set_error_msg("f3d_ens_create: stream creation failed");
  }
  const bool f32 = precision == F3D_PREC_FP32;
  size_t stage = 0;
  for (int c = 0; c < nclasses && !rc; ++c) {
    EnsClass& k = e->cls[c];
    k.nx = dims[c].nx;
    k.ny = dims[c].ny;
    k.nz = dims[c].nz;
    const size_t nx = k.nx, ny = k.ny, nz = k.nz;
    const size_t fu = (nx + 1) * ny * nz, fv = (ny + 1) * nx * nz, fw = (nz + 1) * nx * ny;
    rc |= ealloc(e, &k.ux, 2 * fu);
    rc |= ealloc(e, &k.vy, 2 * fv);
    rc |= ealloc(e, &k.wz, 2 * fw);
    rc |= ealloc(e, &k.k1x, (nx + 2) * ny * nz);
    rc |= ealloc(e, &k.k2y, (ny + 2) * nx * nz);
    rc |= ealloc(e, &k.k3z, (nz + 2) * nx * ny);
    rc |= ealloc(e, &k.vs, nb * fw);
    if (!f32) {
      rc |= ealloc(e, &k.kkf[0], fu);
      rc |= ealloc(e, &k.kkf[1], fv);
      rc |= ealloc(e, &k.kkf[2], fw);
      rc |= ealloc(e, &k.geo[0], nx + 1);
      rc |= ealloc(e, &k.geo[1], ny + 1);
      rc |= ealloc(e, &k.geo[2], nz + 1);
    } else {
      rc |= ealloc(e, &k.f4[0], fu);
      rc |= ealloc(e, &k.f4[1], fv);
      rc |= ealloc(e, &k.f4[2], fw);
      rc |= ealloc(e, &k.vs32, nb * fw);
      rc |= ealloc(e, &k.rdx[0], nx);
      rc |= ealloc(e, &k.rdx[1], ny);
      rc |= ealloc(e, &k.rdx[2], nz);
      if (cmp) {
        rc |= ealloc(e, &k.rdx64[0], nx);
        rc |= ealloc(e, &k.rdx64[1], ny);
        rc |= ealloc(e, &k.rdx64[2], nz);
        rc |= ealloc(e, &k.rdx2[0], nx);
        rc |= ealloc(e, &k.rdx2[1], ny);
        rc |= ealloc(e, &k.rdx2[2], nz);
      }
    }
    const size_t dn[6] = {nx + 4, nx + 3, ny + 4, ny + 3, nz + 4, nz + 3};
    for (int q = 0; q < 6; ++q) rc |= ealloc(e, &k.dx[q], dn[q]);
    rc |= ealloc(e, &k.hm[0], ny);
    rc |= ealloc(e, &k.hm[1], ny + 4);
    rc |= ealloc(e, &k.hm[2], nx * ny);
    stage = std::max({stage, (nx + 4) * (ny + 4) * (nz + 4) * nb, nx * ny * (nz + 3) * nb,
                      2 * (nx + 3) * ny * nz, 2 * (ny + 3) * nx * nz, 2 * (nz + 3) * nx * ny,
                      (nx + 4) * ny * nz, (ny + 4) * nx * nz, (nz + 4) * nx * ny,
                      2 * (nx + 1) * (ny + 1) * (nz + 1)});
  }
  rc |= ealloc(e, &e->flux_tot, 12 * (size_t)nmembers);
  rc |= ealloc(e, &e->flux_step, 6 * (size_t)nmembers);
  rc |= ealloc(e, &e->d_red, std::max<size_t>(3 * (size_t)nmembers, (size_t)e->mass_nblk * nb + 64));
  rc |= ealloc(e, &e->counters, 16);
  rc |= ealloc(e, &e->d_err, 1);
  rc |= ealloc(e, &e->d_nfail, 4);
  rc |= ealloc(e, &e->staging, stage + 4 * (size_t)nb);
  e->staging_elems = stage;
  for (int m = 0; m < nmembers && !rc; ++m) {
    const int c = members[m].grid_class;
    e->member_class[m] = c;
    EnsClass& k = e->cls[c];
    if (k.rep < 0) k.rep = m;
    MemberDev& d = e->hm[m];
    memset(&d, 0, sizeof(MemberDev));
    d.nx = k.nx;
    d.ny = k.ny;
    d.nz = k.nz;
    d.nb = nb;
    d.wfac = (float)members[m].wind_factor;
    d.wfacd = members[m].wind_factor;
    const size_t nx = k.nx, ny = k.ny, nz = k.nz, ncell = nx * ny * nz;
    const size_t fu = (nx + 1) * ny * nz, fv = (ny + 1) * nx * nz, fw = (nz + 1) * nx * ny;
    if (f32) rc |= ealloc(e, &d.c32, ncell * nb);
    else rc |= ealloc(e, &d.c64, ncell * nb);
    if (cmp) rc |= ealloc(e, &d.c32lo, ncell * nb);
    rc |= ealloc(e, &d.acum, nx * ny * nb);
    d.ux[0] = k.ux; d.ux[1] = k.ux + fu;
    d.vy[0] = k.vy; d.vy[1] = k.vy + fv;
    d.wz[0] = k.wz; d.wz[1] = k.wz + fw;
    d.k1x = k.k1x; d.k2y = k.k2y; d.k3z = k.k3z; d.vs = k.vs;
    if (!f32) {
      rc |= ealloc(e, &d.ucur, fu);
      rc |= ealloc(e, &d.vcur, fv);
      rc |= ealloc(e, &d.wcur, fw);
      for (int q = 0; q < 3; ++q) { d.kkf[q] = k.kkf[q]; d.geo[q] = k.geo[q]; }
    } else {
      for (int q = 0; q < 3; ++q) d.f4[q] = k.f4[q];
      d.vs32 = k.vs32;
      d.rdx1b32 = k.rdx[0]; d.rdx2b32 = k.rdx[1]; d.rdx3b32 = k.rdx[2];
      for (int q = 0; q < 3; ++q) {
        d.rdxb64[q] = k.rdx64[q];
        d.rdxb2[q] = k.rdx2[q];
      }
    }
    d.dx1p = k.dx[0]; d.dx1b = k.dx[1]; d.dx2p = k.dx[2];
    d.dx2b = k.dx[3]; d.dx3p = k.dx[4]; d.dx3b = k.dx[5];
    d.hm1 = k.hm[0]; d.hm2 = k.hm[1]; d.hm3 = k.hm[2];
    d.flux_tot = e->flux_tot + 12 * (size_t)m;
    d.flux_step = e->flux_step + 6 * (size_t)m;
    d.t_ite = 1.0;
    if (!rc) {
      if (f32) rc |= cudaMemsetAsync(d.c32, 0, ncell * nb * 4, e->st) != cudaSuccess;
      else rc |= cudaMemsetAsync(d.c64, 0, ncell * nb * 8, e->st) != cudaSuccess;
      if (cmp) rc |= cudaMemsetAsync(d.c32lo, 0, ncell * nb * 4, e->st) != cudaSuccess;
      rc |= cudaMemsetAsync(d.acum, 0, nx * ny * nb * 8, e->st) != cudaSuccess;
    }
  }
  if (!rc) {
    rc |= cudaMemsetAsync(e->flux_tot, 0, 12 * (size_t)nmembers * 8, e->st) != cudaSuccess;
    rc |= cudaMemsetAsync(e->flux_step, 0, 6 * (size_t)nmembers * 8, e->st) != cudaSuccess;
    rc |= cudaMemsetAsync(e->d_err, 0, 4, e->st) != cudaSuccess;
    e->h_pin_elems = 16 * (size_t)nmembers + 64;
    rc |= cudaMallocHost(&e->h_pin, e->h_pin_elems * 8) != cudaSuccess;
  }
  if (!rc) rc |= ealloc(e, &e->dm, (size_t)nmembers);
  if (!rc) rc |= build_work(e);
  if (rc) {
    f3d_ens_destroy(e);
    return set_error_msg("f3d_ens_create: device allocation failed (out of memory?)");
  }
  *out = e;
  return 0;
}

extern "C" int f3d_ens_set_class_grid(f3d_ens* e, int ci, const double* dX1_p, const double* dX1_b,
                                      const double* dX2_p, const double* dX2_b,
                                      const double* dX3_p, const double* dX3_b,
                                      const double* Hm1_p, const double* Hm2_p,
                                      const double* Hm3_p) {
  if (!e || ci < 0 || ci >= e->ncls) return set_error_msg("f3d_ens_set_class_grid: bad class");
  if (!dX1_p || !dX1_b || !dX2_p || !dX2_b || !dX3_p || !dX3_b || !Hm1_p || !Hm2_p || !Hm3_p)
    return set_error_msg("f3d_ens_set_class_grid: null array");
  ECK(cudaSetDevice(e->device));
  EnsClass& k = e->cls[ci];
  const size_t nx = k.nx, ny = k.ny, nz = k.nz;
  const double* src[6] = {dX1_p, dX1_b, dX2_p, dX2_b, dX3_p, dX3_b};
  const size_t dn[6] = {nx + 4, nx + 3, ny + 4, ny + 3, nz + 4, nz + 3};
  for (int q = 0; q < 6; ++q) ECK(cudaMemcpy(k.dx[q], src[q], dn[q] * 8, cudaMemcpyHostToDevice));
  ECK(cudaMemcpy(k.hm[0], Hm1_p, ny * 8, cudaMemcpyHostToDevice));
  ECK(cudaMemcpy(k.hm[1], Hm2_p, (ny + 4) * 8, cudaMemcpyHostToDevice));
  ECK(cudaMemcpy(k.hm[2], Hm3_p, nx * ny * 8, cudaMemcpyHostToDevice));
  k.dX1_p.assign(dX1_p, dX1_p + nx + 4);
  k.dX2_p.assign(dX2_p, dX2_p + ny + 4);
  k.dX3_p.assign(dX3_p, dX3_p + nz + 4);
  k.Hm1_p.assign(Hm1_p, Hm1_p + ny);
  k.Hm2_p.assign(Hm2_p, Hm2_p + ny + 4);
  k.Hm3_p.assign(Hm3_p, Hm3_p + nx * ny);
  const double* dp[3] = {dX1_p, dX2_p, dX3_p};
  const double* db[3] = {dX1_b, dX2_b, dX3_b};
  const size_t nn[3] = {nx, ny, nz};
  for (int d = 0; d < 3; ++d) {
    if (e->prec == F3D_PREC_FP64) {
      std::vector<double4> g(nn[d] + 1);
      for (size_t q = 0; q <= nn[d]; ++q) {
        double a = dp[d][q + 1], b = db[d][q];
        if (!(std::fabs(a) >= 0x1p-100 && std::fabs(a) <= 0x1p100 && std::fabs(b) >= 0x1p-100 &&
              std::fabs(b) <= 0x1p100))
          return set_error_msg("f3d_ens_set_class_grid: spacing outside [2^-100, 2^100]");
        g[q] = make_double4(a, 1.0 / a, b, 1.0 / b);
      }
      ECK(cudaMemcpy(k.geo[d], g.data(), g.size() * sizeof(double4), cudaMemcpyHostToDevice));
    } else {
      std::vector<float> r(nn[d]);
      for (size_t q = 0; q < nn[d]; ++q) r[q] = (float)(1.0 / db[d][q + 1]);
      ECK(cudaMemcpy(k.rdx[d], r.data(), nn[d] * 4, cudaMemcpyHostToDevice));
      if (k.rdx64[d]) {
        std::vector<double> r64(nn[d]);
        for (size_t q = 0; q < nn[d]; ++q) r64[q] = 1.0 / db[d][q + 1];
        ECK(cudaMemcpy(k.rdx64[d], r64.data(), nn[d] * 8, cudaMemcpyHostToDevice));
        std::vector<float2> r2(nn[d]);
        for (size_t q = 0; q < nn[d]; ++q) {
          const float h = (float)r64[q];
          r2[q] = make_float2(h, (float)(r64[q] - (double)h));
        }
        ECK(cudaMemcpy(k.rdx2[d], r2.data(), nn[d] * sizeof(float2), cudaMemcpyHostToDevice));
      }
    }
  }
  k.grid_set = true;
  return 0;
}

static int ens_upload_conv(f3d_ens* e, const EnsClass& k, int which, const double* host,
                           size_t elems, double* dst) {
  if (elems > e->staging_elems) return set_error_msg("ensemble staging too small");
  ECK(cudaMemcpyAsync(e->staging, host, elems * 8, cudaMemcpyHostToDevice, e->st));
  launch_conv(which, e->staging, dst, k.nx, k.ny, k.nz, e->nb, e->st);
  e->launches += 1;
  ECKL();
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

static int class_derived_fields(f3d_ens* e, int ci) {
  EnsClass& k = e->cls[ci];
  if (k.rep < 0 || !k.meteo_set) return 0;
  if (e->prec == F3D_PREC_FP32) launch_fp32_fields(e->dm, k.rep, e->st);
  else launch_face_kk(e->dm, k.rep, e->st);
  e->launches += 1;
  ECKL();
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

extern "C" int f3d_ens_set_class_meteo(f3d_ens* e, int ci, const double* u, const double* v,
                                       const double* w, const double* k1, const double* k2,
                                       const double* k3, const double* vs, double t_its,
                                       double t_ite) {
  if (!e || ci < 0 || ci >= e->ncls) return set_error_msg("f3d_ens_set_class_meteo: bad class");
  if (!u || !v || !w || !k1 || !k2 || !k3) return set_error_msg("f3d_ens_set_class_meteo: null array");
  if (!(t_ite != t_its)) return set_error_msg("f3d_ens_set_class_meteo: t_ite == t_its");
  ECK(cudaSetDevice(e->device));
  EnsClass& k = e->cls[ci];
  const size_t nx = k.nx, ny = k.ny, nz = k.nz, nb = e->nb;
  if (ens_upload_conv(e, k, 0, u, 2 * (nx + 3) * ny * nz, k.ux) ||
      ens_upload_conv(e, k, 1, v, 2 * (ny + 3) * nx * nz, k.vy) ||
      ens_upload_conv(e, k, 2, w, 2 * (nz + 3) * nx * ny, k.wz) ||
      ens_upload_conv(e, k, 3, k1, (nx + 4) * ny * nz, k.k1x) ||
      ens_upload_conv(e, k, 4, k2, (ny + 4) * nx * nz, k.k2y) ||
      ens_upload_conv(e, k, 5, k3, (nz + 4) * nx * ny, k.k3z))
    return 1;
  if (vs && ens_upload_conv(e, k, 6, vs, nx * ny * (nz + 3) * nb, k.vs)) return 1;
  k.t_its = t_its;
  k.t_ite = t_ite;
  for (int m = 0; m < e->nm; ++m)
    if (e->member_class[m] == ci) {
      e->hm[m].t_its = t_its;
      e->hm[m].t_ite = t_ite;
    }
  if (upload_members(e)) return 1;
  k.meteo_set = true;
  return class_derived_fields(e, ci);
}

extern "C" int f3d_ens_set_class_terrain(f3d_ens* e, int ci, int map_v, double X3max,
                                         const double* X3_c, const double* X3_p,
                                         const double* dhdx_p, const double* dhdy_p) {
  if (!e || ci < 0 || ci >= e->ncls) return set_error_msg("f3d_ens_set_class_terrain: bad class");
  if (map_v < 0 || map_v > 2) return set_error_msg("f3d_ens_set_class_terrain: mapping %d not implemented", map_v);
  if (map_v != 0 && (!X3_c || !X3_p || !dhdx_p || !dhdy_p || !(X3max > 0.0)))
    return set_error_msg("f3d_ens_set_class_terrain: sigma mappings need X3max > 0, X3_c, X3_p and the slopes");
  ECK(cudaSetDevice(e->device));
  EnsClass& k = e->cls[ci];
  const size_t nx = k.nx, ny = k.ny, nz = k.nz;
  if (!k.terrain && ealloc(e, &k.terrain, (nz + 1) + nz + 2 * nx * ny)) return 1;
  if (map_v != 0) {
    ECK(cudaMemcpy(k.terrain, X3_c, (nz + 1) * 8, cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(k.terrain + nz + 1, X3_p, nz * 8, cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(k.terrain + 2 * nz + 1, dhdx_p, nx * ny * 8, cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(k.terrain + 2 * nz + 1 + nx * ny, dhdy_p, nx * ny * 8, cudaMemcpyHostToDevice));
  }
  k.map_v = map_v;
  k.X3max = map_v != 0 ? X3max : 1.0;
  return 0;
}

extern "C" int f3d_ens_set_class_meteo_corners(f3d_ens* e, int ci, const double* uc, const double* vc,
                                               const double* wc, const double* k1, const double* k2,
                                               const double* k3, double kh, double kv, double t_its,
                                               double t_ite) {
  if (!e || ci < 0 || ci >= e->ncls) return set_error_msg("f3d_ens_set_class_meteo_corners: bad class");
  if (!uc || !vc || !wc) return set_error_msg("f3d_ens_set_class_meteo_corners: null corner wind");
  const bool kgiven = k1 || k2 || k3;
  if (kgiven && !(k1 && k2 && k3))
    return set_error_msg("f3d_ens_set_class_meteo_corners: give all of k1, k2, k3 or none");
  if (!(t_ite != t_its)) return set_error_msg("f3d_ens_set_class_meteo_corners: t_ite == t_its");
  EnsClass& k = e->cls[ci];
  if (!k.grid_set) return set_error_msg("f3d_ens_set_class_meteo_corners: grid not set");
  ECK(cudaSetDevice(e->device));
  const size_t nx = k.nx, ny = k.ny, nz = k.nz;
  const size_t ncor = (nx + 1) * (ny + 1) * (nz + 1);
  const size_t n1 = (nx + 4) * ny * nz, n2 = nx * (ny + 4) * nz, n3 = nx * ny * (nz + 4);
  const size_t need = 6 * ncor + n1 + n2 + n3;
  if (need > e->met_cap) {
    if (e->d_met) {
      ECK(cudaStreamSynchronize(e->st));
      cudaFree(e->d_met);
      e->d_met = nullptr;
      e->met_cap = 0;
    }
    ECK(cudaMalloc(&e->d_met, need * 8));
    e->met_cap = need;
  }
  double* duc = e->d_met;
  double* dvc = duc + 2 * ncor;
  double* dwc = dvc + 2 * ncor;
  double* dk1 = dwc + 2 * ncor;
  double* dk2 = dk1 + n1;
  double* dk3 = dk2 + n2;
  ECK(cudaMemcpyAsync(duc, uc, 2 * ncor * 8, cudaMemcpyHostToDevice, e->st));
  ECK(cudaMemcpyAsync(dvc, vc, 2 * ncor * 8, cudaMemcpyHostToDevice, e->st));
  ECK(cudaMemcpyAsync(dwc, wc, 2 * ncor * 8, cudaMemcpyHostToDevice, e->st));
  if (kgiven) {
    ECK(cudaMemcpyAsync(dk1, k1, n1 * 8, cudaMemcpyHostToDevice, e->st));
    ECK(cudaMemcpyAsync(dk2, k2, n2 * 8, cudaMemcpyHostToDevice, e->st));
    ECK(cudaMemcpyAsync(dk3, k3, n3 * 8, cudaMemcpyHostToDevice, e->st));
  } else {
    launch_meteo_kconst(k.nx, k.ny, k.nz, kh, kv, dk1, dk2, dk3, e->st);
    e->launches += 1;
  }
  MetGeo g;
  g.nx = k.nx;
  g.ny = k.ny;
  g.nz = k.nz;
  g.map_v = k.map_v;
  g.X3max = k.X3max;
  g.X3c = k.terrain;
  g.X3p = k.terrain ? k.terrain + nz + 1 : nullptr;
  g.dhdx = k.terrain ? k.terrain + 2 * nz + 1 : nullptr;
  g.dhdy = k.terrain ? k.terrain + 2 * nz + 1 + nx * ny : nullptr;
  g.hm1 = k.hm[0];
  g.hm2 = k.hm[1];
  g.hm3 = k.hm[2];
  launch_meteo_corners(g, duc, dvc, dwc, dk1, dk2, dk3, k.ux, k.vy, k.wz, k.k1x, k.k2y, k.k3z, e->st);
  e->launches += 9;
  ECKL();
  k.t_its = t_its;
  k.t_ite = t_ite;
  for (int m = 0; m < e->nm; ++m)
    if (e->member_class[m] == ci) {
      e->hm[m].t_its = t_its;
      e->hm[m].t_ite = t_ite;
    }
  if (upload_members(e)) return 1;
  k.meteo_set = true;
  return class_derived_fields(e, ci);
}

// Stage a class's corner air density/temperature and bin table on the device.
static int ens_stage_vset(f3d_ens* e, int ci, const double* rhoc, const double* tc, const double* diam,
                          const double* rhop, const double* psi, const int* bin_cat, const int* is_aggregate,
                          double** drho, double** dtc, double** dpar, int** dflags) {
  EnsClass& k = e->cls[ci];
  ECK(cudaSetDevice(e->device));
  const size_t ncor = (size_t)(k.nx + 1) * (k.ny + 1) * (k.nz + 1);
  if (2 * ncor + 4 * (size_t)e->nb > e->staging_elems + 4 * (size_t)e->nb)
    return set_error_msg("ensemble staging too small for corner fields");
  *drho = e->staging;
  *dtc = *drho + ncor;
  *dpar = *dtc + ncor;
  *dflags = reinterpret_cast<int*>(*dpar + 3 * e->nb);
  std::vector<double> par(3 * e->nb);
  std::vector<int> fl(e->nb);
  for (int b = 0; b < e->nb; ++b) {
    par[3 * b] = diam[b];
    par[3 * b + 1] = rhop[b];
    par[3 * b + 2] = psi[b];
    fl[b] = bin_cat[b] | ((is_aggregate && is_aggregate[b]) ? (1 << 8) : 0);
  }
  ECK(cudaMemcpyAsync(*drho, rhoc, ncor * 8, cudaMemcpyHostToDevice, e->st));
  ECK(cudaMemcpyAsync(*dtc, tc, ncor * 8, cudaMemcpyHostToDevice, e->st));
  ECK(cudaMemcpyAsync(*dpar, par.data(), par.size() * 8, cudaMemcpyHostToDevice, e->st));
  ECK(cudaMemcpyAsync(*dflags, fl.data(), fl.size() * 4, cudaMemcpyHostToDevice, e->st));
  ECK(cudaStreamSynchronize(e->st));
  if (!e->vev[0]) {
    ECK(cudaEventCreate(&e->vev[0]));
    ECK(cudaEventCreate(&e->vev[1]));
  }
  return 0;
}

static int ens_check_vset_args(f3d_ens* e, int ci, const double* rhoc, const double* tc, const double* diam,
                               const double* rhop, const double* psi, const int* bin_cat) {
  if (!e || ci < 0 || ci >= e->ncls) return set_error_msg("f3d_ens_compute_class_vset: bad class");
  if (!rhoc || !tc || !diam || !rhop || !psi || !bin_cat)
    return set_error_msg("f3d_ens_compute_class_vset: null array");
  if (e->cls[ci].rep >= 0 && !e->cls[ci].grid_set)
    return set_error_msg("f3d_ens_compute_class_vset: grid not set");
  return 0;
}

extern "C" int f3d_ens_compute_class_vset(f3d_ens* e, int ci, int model, const double* rhoc,
                                          const double* tc, const double* diam,
                                          const double* rhop, const double* psi,
                                          const int* bin_cat, const int* is_aggregate,
                                          double vset_fac) {
  if (ens_check_vset_args(e, ci, rhoc, tc, diam, rhop, psi, bin_cat)) return 1;
  if (model < 1 || model > 7) return set_error_msg("setling velocity model not found");
  EnsClass& k = e->cls[ci];
  if (k.rep < 0) return 0;
  double *drho, *dtc, *dpar;
  int* dflags;
  if (ens_stage_vset(e, ci, rhoc, tc, diam, rhop, psi, bin_cat, is_aggregate, &drho, &dtc, &dpar, &dflags))
    return 1;
  ECK(cudaMemsetAsync(e->d_nfail, 0, 4, e->st));
  ECK(cudaEventRecord(e->vev[0], e->st));
  launch_vset_field(e->dm, k.rep, model, drho, dtc, dpar, dflags, vset_fac, e->d_nfail, e->st);
  ECKL();
  ECK(cudaEventRecord(e->vev[1], e->st));
  e->launches += 1;
  int nfail = 0;
  ECK(cudaMemcpyAsync(e->h_pin, e->d_nfail, 4, cudaMemcpyDeviceToHost, e->st));
  ECK(cudaStreamSynchronize(e->st));
  memcpy(&nfail, e->h_pin, 4);
  cudaEventElapsedTime(&e->vset_ms, e->vev[0], e->vev[1]);
  if (class_derived_fields(e, ci)) return 1;
  if (nfail) {
    set_error_msg("no convergence in vset (%d points)", nfail);
    return 2;
  }
  return 0;
}

extern "C" int f3d_ens_compute_class_vset_mlp(f3d_ens* e, int ci, f3d_mlp* h, const double* rhoc,
                                              const double* tc, const double* diam,
                                              const double* rhop, const double* psi,
                                              const int* bin_cat, const int* is_aggregate,
                                              double vset_fac, int refine, long long* nfallback) {
  if (ens_check_vset_args(e, ci, rhoc, tc, diam, rhop, psi, bin_cat)) return 1;
  if (!h) return set_error_msg("f3d_ens_compute_class_vset_mlp: null surrogate");
  EnsClass& k = e->cls[ci];
  if (k.rep < 0) return 0;
  double *drho, *dtc, *dpar;
  int* dflags;
  if (ens_stage_vset(e, ci, rhoc, tc, diam, rhop, psi, bin_cat, is_aggregate, &drho, &dtc, &dpar, &dflags))
    return 1;
  int nfail = 0;
  if (mlp_vset_field(h, e->dm, k.rep, k.nx, k.ny, k.nz, e->nb, drho, dtc, diam, rhop, psi, bin_cat,
                     is_aggregate, vset_fac, refine, e->st, nfallback, &nfail))
    return 1;
  e->launches += 1;
  f3d_mlp_last_ms(h, &e->vset_ms);  // the inference kernel alone
  if (class_derived_fields(e, ci)) return 1;
  if (nfail) {
    set_error_msg("no convergence in vset (%d points)", nfail);
    return 2;
  }
  return 0;
}

extern "C" int f3d_ens_vset_ms(f3d_ens* e, float* ms) {
  if (!e || !ms) return set_error_msg("f3d_ens_vset_ms: bad arguments");
  *ms = e->vset_ms;
  return 0;
}

extern "C" int f3d_ens_set_member_source(f3d_ens* e, int mi, int n, const int* ijk,
                                         const double* s) {
  if (!e || mi < 0 || mi >= e->nm) return set_error_msg("f3d_ens_set_member_source: bad member");
  if (n < 0 || (n > 0 && (!ijk || !s))) return set_error_msg("f3d_ens_set_member_source: bad arguments");
  const EnsClass& k = e->cls[e->member_class[mi]];
  if (!k.grid_set) return set_error_msg("f3d_ens_set_member_source: grid not set");
  ECK(cudaSetDevice(e->device));
  MemberDev& m = e->hm[mi];
  std::vector<int> cell(n);
  std::vector<double> vol(n);
  for (int q = 0; q < n; ++q) {
    int i = ijk[3 * q] - 1, j = ijk[3 * q + 1] - 1, kk = ijk[3 * q + 2] - 1;
    if (i < 0 || i >= k.nx || j < 0 || j >= k.ny || kk < 0 || kk >= k.nz)
      return set_error_msg("f3d_ens_set_member_source: cell %d outside the domain", q);
    cell[q] = i + k.nx * (j + k.ny * kk);
    volatile double a = k.dX1_p[i + 2] * k.dX2_p[j + 2];
    volatile double b = a * k.dX3_p[kk + 2];
    volatile double h = k.Hm1_p[j] * k.Hm2_p[j + 2];
    volatile double h3 = h * k.Hm3_p[i + (size_t)k.nx * j];
    vol[q] = b * h3;
  }
  if (n > 0) {
    int* dc;
    double *ds, *dv;
    if (ealloc(e, &dc, (size_t)n) || ealloc(e, &ds, (size_t)n * e->nb) || ealloc(e, &dv, (size_t)n))
      return 1;
    ECK(cudaMemcpy(dc, cell.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(ds, s, sizeof(double) * n * e->nb, cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(dv, vol.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    m.src_cell = dc;
    m.src_s = ds;
    m.src_vol = dv;
  }
  m.nsrc = n;
  return upload_members(e);
}

extern "C" int f3d_ens_upload_member_state(f3d_ens* e, int mi, const double* my_c,
                                           const double* my_acum) {
  if (!e || mi < 0 || mi >= e->nm) return set_error_msg("f3d_ens_upload_member_state: bad member");
  ECK(cudaSetDevice(e->device));
  const EnsClass& k = e->cls[e->member_class[mi]];
  MemberDev& m = e->hm[mi];
  const size_t nx = k.nx, ny = k.ny, nz = k.nz, nb = e->nb;
  if (my_c) {
    if (e->prec == F3D_PREC_FP64) {
      if (ens_upload_conv(e, k, 7, my_c, (nx + 4) * (ny + 4) * (nz + 4) * nb, m.c64)) return 1;
    } else {
      std::vector<float> tmp(nx * ny * nz * nb), tlo(m.c32lo ? tmp.size() : 0);
      for (size_t b = 0; b < nb; ++b)
        for (size_t kk = 0; kk < nz; ++kk)
          for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
              const size_t q = ((b * nz + kk) * ny + j) * nx + i;
              const double v = my_c[(i + 2) + (nx + 4) * ((j + 2) + (ny + 4) * ((kk + 2) + (nz + 4) * b))];
              tmp[q] = (float)v;
              if (m.c32lo) tlo[q] = (float)(v - (double)tmp[q]);
            }
      ECK(cudaMemcpy(m.c32, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice));
      if (m.c32lo) ECK(cudaMemcpy(m.c32lo, tlo.data(), tlo.size() * 4, cudaMemcpyHostToDevice));
    }
  }
  if (my_acum && ens_upload_conv(e, k, 8, my_acum, (nx + 4) * (ny + 4) * nb, m.acum)) return 1;
  if (my_c && (m.gh64 || m.gh32)) {  // the halo cells of the given state
    std::vector<double> g;
    gh_gather_ref(m.nx, m.ny, m.nz, (int)nb, my_c, g);
    if (m.gh64) {
      ECK(cudaMemcpy(m.gh64, g.data(), g.size() * 8, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> t(g.size());
      for (size_t q = 0; q < g.size(); ++q) t[q] = (float)g[q];
      ECK(cudaMemcpy(m.gh32, t.data(), t.size() * 4, cudaMemcpyHostToDevice));
    }
  }
  return 0;
}

extern "C" int f3d_ens_download_member_state(f3d_ens* e, int mi, double* my_c, double* my_acum) {
  if (!e || mi < 0 || mi >= e->nm) return set_error_msg("f3d_ens_download_member_state: bad member");
  ECK(cudaSetDevice(e->device));
  ECK(cudaStreamSynchronize(e->st));
  const EnsClass& k = e->cls[e->member_class[mi]];
  const MemberDev& m = e->hm[mi];
  const size_t nx = k.nx, ny = k.ny, nz = k.nz, nb = e->nb;
  if (my_c) {
    std::vector<double> tmp(nx * ny * nz * nb);
    if (e->prec == F3D_PREC_FP64) {
      ECK(cudaMemcpy(tmp.data(), m.c64, tmp.size() * 8, cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> t32(tmp.size());
      ECK(cudaMemcpy(t32.data(), m.c32, t32.size() * 4, cudaMemcpyDeviceToHost));
      for (size_t q = 0; q < t32.size(); ++q) tmp[q] = t32[q];
      if (m.c32lo) {
        ECK(cudaMemcpy(t32.data(), m.c32lo, t32.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < t32.size(); ++q) tmp[q] = tmp[q] + (double)t32[q];
      }
    }
    for (size_t b = 0; b < nb; ++b)
      for (size_t kk = 0; kk < nz; ++kk)
        for (size_t j = 0; j < ny; ++j)
          memcpy(&my_c[2 + (nx + 4) * ((j + 2) + (ny + 4) * ((kk + 2) + (nz + 4) * b))],
                 &tmp[((b * nz + kk) * ny + j) * nx], nx * 8);
    if (m.gh64 || m.gh32) {  // the kept boundary halo layers
      std::vector<double> g((size_t)gh_per_bin(m.nx, m.ny, m.nz) * nb);
      if (m.gh64) {
        ECK(cudaMemcpy(g.data(), m.gh64, g.size() * 8, cudaMemcpyDeviceToHost));
      } else {
        std::vector<float> t(g.size());
        ECK(cudaMemcpy(t.data(), m.gh32, t.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < t.size(); ++q) g[q] = t[q];
      }
      gh_scatter_ref(m.nx, m.ny, m.nz, (int)nb, g, my_c);
    }
  }
  if (my_acum) {
    std::vector<double> tmp(nx * ny * nb);
    ECK(cudaMemcpy(tmp.data(), m.acum, tmp.size() * 8, cudaMemcpyDeviceToHost));
    for (size_t b = 0; b < nb; ++b)
      for (size_t j = 0; j < ny; ++j)
        memcpy(&my_acum[2 + (nx + 4) * ((j + 2) + (ny + 4) * b)], &tmp[(b * ny + j) * nx], nx * 8);
  }
  return 0;
}

// ---- time step, clock and execution ----------------------------------------
extern "C" int f3d_ens_compute_time_steps(f3d_ens* e, double stime, int criterion, double cfl,
                                          double run_end, double* dt) {
  if (!e) return set_error_msg("f3d_ens_compute_time_steps: null ensemble");
  if (criterion != 1 && criterion != 2)
    return set_error_msg("f3d_ens_compute_time_steps: criterion %d not in 1..2", criterion);
  for (const EnsClass& k : e->cls)
    if (k.rep >= 0 && !k.meteo_set) return set_error_msg("f3d_ens_compute_time_steps: meteo not set");
  ECK(cudaSetDevice(e->device));
  ECK(cudaMemsetAsync(e->d_red, 0, 3 * (size_t)e->nm * sizeof(double), e->st));
  for (int m = 0; m < e->nm; ++m) {
    launch_cfl(e->dm, m, stime, criterion, e->d_red + 3 * (size_t)m, e->st);
    e->launches += 1;
  }
  launch_finalize_dt(e->dm, e->nm, e->d_red, cfl, run_end, e->st);
  e->launches += 1;
  ECKL();
  if (pull_dynamic(e)) return 1;
  std::vector<double> dts(e->nm);
  for (int m = 0; m < e->nm; ++m) dts[m] = e->hm[m].dt;
  if (update_radio_factors(e, dts.data())) return 1;
  if (dt)
    for (int m = 0; m < e->nm; ++m) dt[m] = dts[m];
  return 0;
}

extern "C" int f3d_ens_set_clock(f3d_ens* e, const double* time, int iiter) {
  if (!e || !time) return set_error_msg("f3d_ens_set_clock: null argument");
  ECK(cudaSetDevice(e->device));
  if (pull_dynamic(e)) return 1;
  for (int m = 0; m < e->nm; ++m) {
    MemberDev& d = e->hm[m];
    d.time = time[m];
    d.iiter = iiter;
    d.stime = (time[m] - d.t_its) / (d.t_ite - d.t_its);
  }
  e->iiter = iiter;
  ECK(cudaMemcpyAsync(e->dm, e->hm.data(), sizeof(MemberDev) * e->nm, cudaMemcpyHostToDevice, e->st));
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

extern "C" int f3d_ens_get_clock(f3d_ens* e, double* time, int* iiter) {
  if (!e) return set_error_msg("f3d_ens_get_clock: null ensemble");
  ECK(cudaSetDevice(e->device));
  if (pull_dynamic(e)) return 1;
  if (time)
    for (int m = 0; m < e->nm; ++m) time[m] = e->hm[m].time;
  if (iiter) *iiter = e->hm[0].iiter;
  return 0;
}

extern "C" int f3d_ens_set_tuning(f3d_ens* e, int mode, int bins_per_block, int ctas_per_sm) {
  if (!e) return set_error_msg("f3d_ens_set_tuning: null ensemble");
  if (mode != F3D_ENS_MODE_KERNELS && mode != F3D_ENS_MODE_PERSISTENT)
    return set_error_msg("f3d_ens_set_tuning: mode %d unknown", mode);
  if (bins_per_block != 1 && bins_per_block != 2 && bins_per_block != 4)
    return set_error_msg("f3d_ens_set_tuning: bins_per_block %d not 1, 2 or 4", bins_per_block);
  if (ctas_per_sm < 0 || ctas_per_sm > 16)
    return set_error_msg("f3d_ens_set_tuning: ctas_per_sm %d out of range", ctas_per_sm);
  ECK(cudaSetDevice(e->device));
  ECK(cudaStreamSynchronize(e->st));
  drop_graphs(e);
  e->mode = mode;
  e->ctas_per_sm = ctas_per_sm;
  if (bins_per_block != e->bpb) {
    if (pull_dynamic(e)) return 1;
    e->bpb = bins_per_block;
    if (build_work(e)) return 1;
  }
  return 0;
}

namespace {

int fused_setup(f3d_ens* e, const void** func, int* smem) {
  const bool f32 = e->prec == F3D_PREC_FP32;
  *func = f32 ? fused32_func(e->lim, e->tm, e->cmp) : fused64_func(e->lim, e->tm);
  *smem = f32 ? fused32_smem(e->tm, e->cmp) : fused64_smem();
  ECK(cudaFuncSetAttribute(*func, cudaFuncAttributeMaxDynamicSharedMemorySize, *smem));
  int per_sm = 0;
  ECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, *func, 128, *smem));
  if (per_sm < 1) return set_error_msg("persistent step kernel does not fit on an SM");
  if (e->ctas_per_sm > 0) per_sm = std::min(per_sm, e->ctas_per_sm);
  int nsm = 0;
  ECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device));
  e->fused_grid = per_sm * nsm;
  return 0;
}

// Enqueue one step.  set_host: dt/time come from the host arrays.
// One step on the stream.  ev (profiling only, never while capturing):
// ev[0] before the step, ev[1] after prep/source, ev[2 + q] after the q-th
// sweep of the step's order, ev[5] at the end; in the persistent mode the
// whole step lies between ev[0] and ev[5].
// exp(-kn dt) of every radionuclide bin (and of its Sr90 parent) for each
// member's dt, with the host C library as the CPU restatement evaluates it
// (mod_Phys.F90:1276-1297); read by the decay kernel from device memory, so
// that the captured step graphs pick up a new dt.
int update_radio_factors(f3d_ens* e, const double* dt) {
  if (!e->radio_on) return 0;
  const size_t nr = e->radio.bin.size(), need = 2 * nr * (size_t)e->nm;
  if (need > e->radfact_cap) {
    if (ealloc(e, &e->d_radfact, need)) return 1;
    e->radfact_cap = need;
    drop_graphs(e);
  }
  std::vector<double> f(need);
  for (int m = 0; m < e->nm; ++m)
    for (size_t r = 0; r < nr; ++r) {
      f[2 * nr * m + r] = std::exp(-e->radio.kn[r] * dt[m]);
      f[2 * nr * m + nr + r] = e->radio.parent[r] >= 0 ? std::exp(-e->radio.pkn[r] * dt[m]) : 1.0;
    }
  ECK(cudaMemcpyAsync(e->d_radfact, f.data(), need * 8, cudaMemcpyHostToDevice, e->st));
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

// Configure every member's z-sweep epilogue (wet deposition and decay inside
// the z sweep, f3d_set_zsweep_epilogue); a change re-uploads the descriptors
// and drops the step graphs, whose launches differ.
int sync_epilogue(f3d_ens* e) {
  const bool on = zsweep_epilogue() && (e->wet_on || e->radio_on);
  const size_t nr = e->radio.bin.size();
  bool changed = false;
  for (int m = 0; m < e->nm; ++m) {
    MemberDev& d = e->hm[m];
    const EnsClass& k = e->cls[e->member_class[m]];
    MemberDev w = d;
    const bool wet = on && e->wet_on && k.wet_set;
    w.epi_on = on ? 1 : 0;
    w.wet_mask = wet ? e->wet_mask : 0ull;
    w.wet_a = e->wet_a;
    w.powpb = wet ? k.powpb : nullptr;
    w.ktop = wet ? k.ktop : nullptr;
    w.awet = e->awet.empty() ? nullptr : e->awet[m];
    const bool dec = on && e->radio_on && e->d_radfact;
    w.radf = dec ? e->d_radfact + 2 * nr * (size_t)m : nullptr;
    w.daughter_mask = 0ull;
    for (int b = 0; b < 64; ++b) w.rad_r[b] = -1;
    if (dec)
      for (size_t q = 0; q < nr; ++q) {
        w.rad_r[e->radio.bin[q]] = (signed char)q;
        if (e->radio.parent[q] >= 0) w.daughter_mask |= 1ull << e->radio.bin[q];
      }
    if (memcmp(&w, &d, sizeof(MemberDev)) != 0) {
      d = w;
      changed = true;
    }
  }
  if (changed) {
    drop_graphs(e);
    if (upload_members(e)) return 1;
  }
  return 0;
}

// With the epilogue on, what the z sweep leaves to k_radio: the daughter
// bins, set from their parents, and the kept halo layers.
bool radio_tail_needed(const f3d_ens* e, int m) {
  if (!e->radio_on) return false;
  const MemberDev& d = e->hm[m];
  return d.daughter_mask != 0ull || d.gh64 || d.gh32;
}

// Wet deposition and radioactive decay of every member after its sweeps
// (mod_F3D.F90:1493-1520), one launch each per member, or (epilogue on) the
// remainder of the decay that the z sweep leaves.
int enqueue_wet_radio(f3d_ens* e) {
  for (int m = 0; m < e->nm; ++m) {
    const MemberDev& d = e->hm[m];
    const EnsClass& k = e->cls[e->member_class[m]];
    const double* dt_dev = reinterpret_cast<const double*>(
        reinterpret_cast<const char*>(e->dm + m) + offsetof(MemberDev, dt));
    if (d.epi_on && !radio_tail_needed(e, m)) continue;
    if (e->wet_on && k.wet_set && !d.epi_on) {
      WetArgs a;
      memset(&a, 0, sizeof(a));
      a.nx = d.nx;
      a.ny = d.ny;
      a.nz = d.nz;
      a.nb = e->nb;
      a.dt_dev = dt_dev;
      a.a = e->wet_a;
      a.powpb = k.powpb;
      a.ktop = k.ktop;
      a.dx3p = d.dx3p;
      a.awet = e->awet[m];
      a.c64 = d.c64;
      a.c32 = d.c32;
      a.c32lo = d.c32lo;
      a.mask = e->wet_mask;
      launch_wet(a, e->st);
      e->launches += 1;
    }
    if (e->radio_on) {
      RadioArgs r;
      memset(&r, 0, sizeof(r));
      r.nx = d.nx;
      r.ny = d.ny;
      r.nz = d.nz;
      r.nr = (int)e->radio.bin.size();
      for (int q = 0; q < r.nr; ++q) {
        r.bin[q] = e->radio.bin[q];
        r.parent[q] = e->radio.parent[q];
      }
      r.fdev = e->d_radfact + 2 * (size_t)r.nr * m;
      r.tail = d.epi_on;
      r.c64 = d.c64;
      r.c32 = d.c32;
      r.c32lo = d.c32lo;
      r.acum = d.acum;
      r.gh64 = d.gh64;
      r.gh32 = d.gh32;
      r.ngh = gh_per_bin(d.nx, d.ny, d.nz);
      r.awet = e->awet.empty() ? nullptr : e->awet[m];
      launch_radio(r, e->st);
      e->launches += 1;
    }
  }
  ECKL();
  return 0;
}

int wet_radio_launches(const f3d_ens* e) {
  int n = 0;
  for (int m = 0; m < e->nm; ++m) {
    if (e->hm[m].epi_on) {
      n += radio_tail_needed(e, m) ? 1 : 0;
      continue;
    }
    if (e->wet_on && e->cls[e->member_class[m]].wet_set) ++n;
    if (e->radio_on) ++n;
  }
  return n;
}

int enqueue_step(f3d_ens* e, bool xfirst, bool advance, cudaEvent_t* ev = nullptr,
                 const std::vector<std::pair<int, GcArgs>>* gcl = nullptr) {
  if (ev) ECK(cudaEventRecord(ev[0], e->st));
  // a step with the gravity current runs the per-phase kernels, which take
  // the radial wind between the wind preparation and the sweeps
  if (e->mode == F3D_ENS_MODE_PERSISTENT && !(gcl && !gcl->empty())) {
    const void* func;
    int smem;
    if (fused_setup(e, &func, &smem)) return 1;
    ECK(cudaMemsetAsync(e->counters, 0, 16 * sizeof(unsigned int), e->st));
    FusedArgs a;
    a.members = e->dm;
    a.nmembers = e->nm;
    for (int d = 0; d < 3; ++d) {
      a.work[d] = e->dwork[d];
      a.nwork[d] = e->nwork[d];
    }
    a.prep_member = e->dprep_member;
    a.prep_first = e->dprep_first;
    a.nprep = e->prec == F3D_PREC_FP64 ? e->nprep : 0;
    a.counters = e->counters;
    a.err = e->d_err;
    a.bpb = e->bpb;
    a.wait_limit = wait_limit();
    a.epi = e->hm[0].epi_on;  // the same for every member
    void* args[] = {&a};
    ECK(cudaLaunchCooperativeKernel(func, dim3(e->fused_grid), dim3(128), args, (size_t)smem, e->st));
    e->launches += 1;
    if (enqueue_wet_radio(e)) return 1;
    if (ev) ECK(cudaEventRecord(ev[5], e->st));
    return 0;
  }
  if (e->prec == F3D_PREC_FP64) launch_prep64(e->dm, e->dprep_member, e->dprep_first, e->nprep, 7, e->st);
  if (gcl) {  // F3D_add_radial_wind on the members' interpolated winds (mod_F3D.F90:1443-1445)
    for (const auto& q : *gcl) {
      const MemberDev& m = e->hm[q.first];
      launch_gc_winds(e->dm, q.first, m.nx, m.ny, m.nz, e->prec == F3D_PREC_FP32, q.second, e->st);
      e->launches += 1;
    }
  }
  if (e->prec == F3D_PREC_FP64) launch_source64(e->dm, e->nm, e->st);
  else launch_source32(e->dm, e->nm, e->st);
  e->launches += (e->prec == F3D_PREC_FP64) ? 2 : 1;
  if (ev) ECK(cudaEventRecord(ev[1], e->st));
  const int order[3] = {xfirst ? DIR_X : DIR_Y, xfirst ? DIR_Y : DIR_X, DIR_Z};
  for (int q = 0; q < 3; ++q) {
    const int d = order[q];
    if (e->prec == F3D_PREC_FP64)
      launch_sweep64(d, e->lim, e->tm, e->hm[0].epi_on, e->dm, e->dwork[d], e->nwork[d], e->bpb, e->st);
    else
      launch_sweep32(d, e->lim, e->tm, e->cmp, e->hm[0].epi_on, e->dm, e->dwork[d], e->nwork[d], e->bpb,
                     e->st);
    e->launches += 1;
    if (ev) ECK(cudaEventRecord(ev[2 + q], e->st));
  }
  launch_flux_reduce(e->dm, e->nm, 7, e->st);
  e->launches += 1;
  if (enqueue_wet_radio(e)) return 1;
  if (advance) {
    launch_advance_clock(e->dm, e->nm, e->st);
    e->launches += 1;
  }
  ECKL();
  if (ev) ECK(cudaEventRecord(ev[5], e->st));
  return 0;
}

// Accumulate the phase times of a profiled step (waits for it).
int accumulate_profile(f3d_ens* e, bool xfirst) {
  ECK(cudaEventSynchronize(e->pev[5]));
  float t;
  if (e->mode == F3D_ENS_MODE_PERSISTENT) {
    cudaEventElapsedTime(&t, e->pev[0], e->pev[5]);
    e->prof_ms[1] += t;  // the fused step kernel
  } else {
    const int order[3] = {xfirst ? DIR_X : DIR_Y, xfirst ? DIR_Y : DIR_X, DIR_Z};
    cudaEventElapsedTime(&t, e->pev[0], e->pev[1]);
    e->prof_ms[0] += t;
    for (int q = 0; q < 3; ++q) {
      cudaEventElapsedTime(&t, e->pev[1 + q], e->pev[2 + q]);
      e->prof_ms[1 + order[q]] += t;
    }
    cudaEventElapsedTime(&t, e->pev[4], e->pev[5]);
    e->prof_ms[4] += t;
  }
  e->prof_steps += 1;
  return 0;
}

int build_graphs(f3d_ens* e) {
  drop_graphs(e);
  const int ng = (e->mode == F3D_ENS_MODE_PERSISTENT) ? 1 : 2;
  for (int q = 0; q < ng; ++q) {
    cudaGraph_t g = nullptr;
    ECK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    long long keep = e->launches;
    int rc = enqueue_step(e, q == 0, true);
    cudaError_t ce = cudaStreamEndCapture(e->st, &g);
    e->launches = keep;
    if (rc || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return set_error_msg("step graph capture failed: %s", cudaGetErrorString(ce));
    }
    cudaError_t ie = cudaGraphInstantiate(&e->graph[q], g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return set_error_msg("graph instantiation failed: %s", cudaGetErrorString(ie));
  }
  if (ng == 1) e->graph[1] = nullptr;
  e->graph_ok = true;
  return 0;
}

int kernels_per_step(const f3d_ens* e) {
  if (e->mode == F3D_ENS_MODE_PERSISTENT) return 1 + wet_radio_launches(e);
  return (e->prec == F3D_PREC_FP64 ? 2 : 1) + 3 + 1 + 1 + wet_radio_launches(e);
}

}  // namespace

extern "C" int f3d_ens_run(f3d_ens* e, int nsteps) {
  if (!e || nsteps < 0) return set_error_msg("f3d_ens_run: bad arguments");
  if (e->gc_any)
    return set_error_msg("f3d_ens_run: a member has a gravity current, whose radial wind and time "
                         "step change every step; advance with f3d_ens_step");
  for (const EnsClass& k : e->cls)
    if (k.rep >= 0 && (!k.meteo_set || !k.grid_set)) return set_error_msg("f3d_ens_run: class not ready");
  ECK(cudaSetDevice(e->device));
  if (sync_epilogue(e)) return 1;
  if (e->prof) {
    for (int s = 0; s < nsteps; ++s) {
      const bool xfirst = (e->mode == F3D_ENS_MODE_PERSISTENT) || (e->iiter % 2 == 0);
      if (enqueue_step(e, xfirst, true, e->pev)) return 1;
      if (accumulate_profile(e, xfirst)) return 1;
      e->iiter += 1;
    }
    return 0;
  }
  if (!e->graph_ok && build_graphs(e)) return 1;
  for (int s = 0; s < nsteps; ++s) {
    cudaGraphExec_t g = (e->mode == F3D_ENS_MODE_PERSISTENT) ? e->graph[0] : e->graph[e->iiter & 1];
    ECK(cudaGraphLaunch(g, e->st));
    e->launches += kernels_per_step(e);
    e->iiter += 1;
  }
  return 0;
}

// Boundary halo layers of every member (as f3d_ads_keep_boundary_halo): the
// sweeps keep the free-flow ghost values they compute, the decay decays them,
// and the output reductions and downloads use them instead of zero.
extern "C" int f3d_ens_keep_boundary_halo(f3d_ens* e, int on) {
  if (!e) return set_error_msg("f3d_ens_keep_boundary_halo: null ensemble");
  ECK(cudaSetDevice(e->device));
  for (int mi = 0; mi < e->nm; ++mi) {
    MemberDev& d = e->hm[mi];
    if (!on) {  // the buffers stay with the ensemble until it is destroyed
      d.gh64 = nullptr;
      d.gh32 = nullptr;
      continue;
    }
    const size_t n = (size_t)gh_per_bin(d.nx, d.ny, d.nz) * e->nb;
    if (e->prec == F3D_PREC_FP64) {
      if (!d.gh64 && ealloc(e, &d.gh64, n)) return 1;
      ECK(cudaMemset(d.gh64, 0, n * 8));
    } else {
      if (!d.gh32 && ealloc(e, &d.gh32, n)) return 1;
      ECK(cudaMemset(d.gh32, 0, n * 4));
    }
  }
  drop_graphs(e);
  return upload_members(e);
}

// ---- gravity current per member: F3D_add_radial_wind (mod_F3D.F90:978-1226) --
namespace {
bool ens_gc_args(const f3d_ens* e, int mi, double time, GcArgs* g, double st[7]) {
  const std::vector<double>& p = e->gc_p[mi];
  if (p.empty()) {
    memset(g, 0, sizeof(*g));
    for (int q = 0; q < 7; ++q) st[q] = 0.0;
    return false;
  }
  const EnsClass& k = e->cls[e->member_class[mi]];
  const double* lon_c = k.gc_host.data();
  const double* lat_c = lon_c + (k.nx + 1);
  const double* hm1_c = lat_c + (k.ny + 1) + k.nx + k.ny;
  if (!gc_scalars(p.data(), lon_c, lat_c, hm1_c, time, g, st)) return false;
  g->lon_c = k.gc_xy;
  g->lat_c = g->lon_c + (k.nx + 1);
  g->lon_p = g->lat_c + (k.ny + 1);
  g->lat_p = g->lon_p + k.nx;
  g->hm1_c = g->lat_p + k.ny;
  g->hm1_p = e->hm[mi].hm1;
  g->zc = k.zc;
  return true;
}
}  // namespace

extern "C" int f3d_ens_set_member_gravity_current(f3d_ens* e, int mi, const double params[11],
                                                  const double* lon_c, const double* lat_c,
                                                  const double* lon_p, const double* lat_p,
                                                  const double* Hm1_c) {
  if (!e || mi < 0 || mi >= e->nm) return set_error_msg("f3d_ens_set_member_gravity_current: bad member");
  ECK(cudaSetDevice(e->device));
  if (e->gc_p.empty()) e->gc_p.resize(e->nm);
  if (!params) {  // switch the member's current off
    e->gc_p[mi].clear();
    e->gc_any = false;
    for (const auto& p : e->gc_p) e->gc_any = e->gc_any || !p.empty();
    if (e->hm[mi].gc_cur) {
      e->hm[mi].gc_cur = 0;
      if (upload_members(e)) return 1;
    }
    return 0;
  }
  EnsClass& k = e->cls[e->member_class[mi]];
  if (!k.grid_set) return set_error_msg("f3d_ens_set_member_gravity_current: class grid not set");
  if (!k.zc)
    return set_error_msg("f3d_ens_set_member_gravity_current: corner heights not set "
                         "(f3d_ens_set_class_corner_heights)");
  const size_t n = (size_t)(k.nx + 1) + (k.ny + 1) + k.nx + k.ny + (k.ny + 1);
  if (lon_c || lat_c || lon_p || lat_p || Hm1_c) {
    if (!lon_c || !lat_c || !lon_p || !lat_p || !Hm1_c)
      return set_error_msg("f3d_ens_set_member_gravity_current: give all five coordinate arrays");
    k.gc_host.resize(n);
    double* h = k.gc_host.data();
    const size_t o_lat_c = k.nx + 1, o_lon_p = o_lat_c + k.ny + 1, o_lat_p = o_lon_p + k.nx,
                 o_hm1_c = o_lat_p + k.ny;
    memcpy(h, lon_c, (k.nx + 1) * 8);
    memcpy(h + o_lat_c, lat_c, (k.ny + 1) * 8);
    memcpy(h + o_lon_p, lon_p, k.nx * 8);
    memcpy(h + o_lat_p, lat_p, k.ny * 8);
    memcpy(h + o_hm1_c, Hm1_c, (k.ny + 1) * 8);
    if (!k.gc_xy && ealloc(e, &k.gc_xy, n)) return 1;
    ECK(cudaMemcpy(k.gc_xy, h, n * 8, cudaMemcpyHostToDevice));
  } else if (k.gc_host.size() != n) {
    return set_error_msg("f3d_ens_set_member_gravity_current: the class's coordinates not given");
  }
  MemberDev& m = e->hm[mi];
  if (e->prec == F3D_PREC_FP32 && !m.gc4[0]) {  // this step's x and y face records
    if (ealloc(e, &m.gc4[0], (size_t)(k.nx + 1) * k.ny * k.nz) ||
        ealloc(e, &m.gc4[1], (size_t)(k.ny + 1) * k.nx * k.nz))
      return 1;
    if (upload_members(e)) return 1;
  }
  e->gc_p[mi].assign(params, params + 11);
  e->gc_any = true;
  return 0;
}

extern "C" int f3d_ens_gravity_current_time_steps(f3d_ens* e, const double* times,
                                                  const double* stimes, int criterion, double cfl,
                                                  double run_end, int* active, double* dts) {
  if (!e || !times || !stimes || !active || !dts)
    return set_error_msg("f3d_ens_gravity_current_time_steps: null argument");
  if (criterion != 1 && criterion != 2)
    return set_error_msg("f3d_ens_gravity_current_time_steps: criterion %d not in 1..2", criterion);
  ECK(cudaSetDevice(e->device));
  std::vector<GcArgs> gs(e->nm);
  for (int m = 0; m < e->nm; ++m) {
    double st[7];
    active[m] = ens_gc_args(e, m, times[m], &gs[m], st) ? 1 : 0;
  }
  bool any = false;
  for (int m = 0; m < e->nm; ++m) {
    if (!active[m]) continue;
    any = true;
    ECK(cudaMemsetAsync(e->d_red + 3 * (size_t)m, 0, 3 * sizeof(double), e->st));
    launch_cfl(e->dm, m, stimes[m], criterion, e->d_red + 3 * (size_t)m, e->st, &gs[m]);
  }
  if (!any) return 0;
  ECKL();
  ECK(cudaMemcpyAsync(e->h_pin, e->d_red, 3 * (size_t)e->nm * sizeof(double), cudaMemcpyDeviceToHost,
                      e->st));
  ECK(cudaStreamSynchronize(e->st));
  for (int m = 0; m < e->nm; ++m) {
    if (!active[m]) continue;
    const double* r = e->h_pin + 3 * (size_t)m;
    double x = std::max(std::max(r[0], r[1]), r[2]);  // mod_Grid.F90:1125-1127
    if (x > 0.0) x = 1.0 / x;
    x = cfl * x;
    dts[m] = std::min(x, run_end);
  }
  return 0;
}

// ---- autotuner --------------------------------------------------------------
namespace {
// The candidates: per-phase kernels replayed from CUDA graphs with 4, 2 or 1
// bins per block, and the persistent step kernel with 4 or 2.
const int kTuneCand[F3D_ENS_TUNE_CANDIDATES][3] = {
    {F3D_ENS_MODE_KERNELS, 4, 0},    {F3D_ENS_MODE_KERNELS, 2, 0},
    {F3D_ENS_MODE_KERNELS, 1, 0},    {F3D_ENS_MODE_PERSISTENT, 4, 0},
    {F3D_ENS_MODE_PERSISTENT, 2, 0}};

// Cache file: one line per key, "key mode bpb ctas ms c0 c1 c2 c3 c4"
// (keys are single tokens; later lines of a key win).
bool tune_cache_read(const char* path, const char* key, int tuning[3], double* ms, double* cand) {
  FILE* f = fopen(path, "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (fgets(line, sizeof line, f)) {
    char k[512];
    int t0, t1, t2;
    double m, c[F3D_ENS_TUNE_CANDIDATES];
    if (sscanf(line, "%511s %d %d %d %lf %lf %lf %lf %lf %lf", k, &t0, &t1, &t2, &m, &c[0], &c[1],
               &c[2], &c[3], &c[4]) == 10 &&
        strcmp(k, key) == 0) {
      tuning[0] = t0;
      tuning[1] = t1;
      tuning[2] = t2;
      *ms = m;
      if (cand) memcpy(cand, c, sizeof c);
      found = true;
    }
  }
  fclose(f);
  return found;
}

void tune_cache_write(const char* path, const char* key, const int tuning[3], double ms,
                      const double* cand) {
  std::vector<std::string> keep;
  if (FILE* f = fopen(path, "r")) {
    char line[1024], k[512];
    while (fgets(line, sizeof line, f))
      if (sscanf(line, "%511s", k) == 1 && strcmp(k, key) != 0) keep.push_back(line);
    fclose(f);
  }
  const std::string tmp = std::string(path) + ".tmp";
  FILE* f = fopen(tmp.c_str(), "w");
  if (!f) return;  // an unwritable cache only costs a re-tune
  for (const std::string& l : keep) fputs(l.c_str(), f);
  fprintf(f, "%s %d %d %d %.6f", key, tuning[0], tuning[1], tuning[2], ms);
  for (int q = 0; q < F3D_ENS_TUNE_CANDIDATES; ++q) fprintf(f, " %.6f", cand[q]);
  fputc('\n', f);
  fclose(f);
  rename(tmp.c_str(), path);
}
}  // namespace

extern "C" int f3d_ens_autotune(f3d_ens* e, int steps, const char* cache_file, const char* key,
                                int tuning[3], double* ms_per_step, double* cand_ms) {
  if (!e || !tuning || !ms_per_step || steps < 1)
    return set_error_msg("f3d_ens_autotune: bad arguments");
  if (key && strpbrk(key, " \t\n"))
    return set_error_msg("f3d_ens_autotune: the cache key must be a single token");
  const bool cached = cache_file && key;
  if (cached && tune_cache_read(cache_file, key, tuning, ms_per_step, cand_ms))
    return f3d_ens_set_tuning(e, tuning[0], tuning[1], tuning[2]);
  ECK(cudaSetDevice(e->device));
  cudaEvent_t ev[2];
  ECK(cudaEventCreate(&ev[0]));
  ECK(cudaEventCreate(&ev[1]));
  double ms[F3D_ENS_TUNE_CANDIDATES];
  int best = -1;
  for (int q = 0; q < F3D_ENS_TUNE_CANDIDATES; ++q) {
    ms[q] = -1.0;
    const int* c = kTuneCand[q];
    int derr = 0;
    float el = 0.f;
    // warm-up step (builds the graphs), then `steps` timed steps on the
    // ensemble's stream; a candidate that fails or whose barriers gave up
    // is skipped
    if (f3d_ens_set_tuning(e, c[0], c[1], c[2]) || f3d_ens_run(e, 1) ||
        cudaEventRecord(ev[0], e->st) != cudaSuccess || f3d_ens_run(e, steps) ||
        cudaEventRecord(ev[1], e->st) != cudaSuccess || f3d_ens_status(e, &derr) ||
        cudaEventElapsedTime(&el, ev[0], ev[1]) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (derr) {
      f3d_ens_clear_status(e);
      continue;
    }
    ms[q] = el / steps;
    if (best < 0 || ms[q] < ms[best]) best = q;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (cand_ms) memcpy(cand_ms, ms, sizeof ms);
  if (best < 0) return set_error_msg("f3d_ens_autotune: no configuration ran");
  for (int k = 0; k < 3; ++k) tuning[k] = kTuneCand[best][k];
  *ms_per_step = ms[best];
  if (cached) tune_cache_write(cache_file, key, tuning, ms[best], ms);
  return f3d_ens_set_tuning(e, tuning[0], tuning[1], tuning[2]);
}

extern "C" int f3d_ens_step(f3d_ens* e, const double* dt, const double* time, int iiter,
                            double* fluxes) {
  if (!e || !dt || !time) return set_error_msg("f3d_ens_step: null argument");
  for (const EnsClass& k : e->cls)
    if (k.rep >= 0 && (!k.meteo_set || !k.grid_set)) return set_error_msg("f3d_ens_step: class not ready");
  ECK(cudaSetDevice(e->device));
  if (update_radio_factors(e, dt)) return 1;
  if (sync_epilogue(e)) return 1;
  std::vector<std::pair<int, GcArgs>> gcl;
  if (e->gc_any) {  // the members whose current acts at their time
    bool changed = false;
    for (int m = 0; m < e->nm; ++m) {
      GcArgs g;
      double st[7];
      const bool on = ens_gc_args(e, m, time[m], &g, st);
      if (on) gcl.emplace_back(m, g);
      if (e->prec == F3D_PREC_FP32 && e->hm[m].gc_cur != (on ? 1 : 0)) {
        e->hm[m].gc_cur = on ? 1 : 0;  // the precision form's x/y sweeps read gc4
        changed = true;
      }
    }
    if (changed && upload_members(e)) return 1;
  }
  launch_set_steps(e->dm, e->nm, dt, time, iiter, e->st);
  e->launches += (e->nm + 63) / 64;
  ECKL();
  if (enqueue_step(e, iiter % 2 == 0, false, nullptr, &gcl)) return 1;
  e->iiter = iiter + 1;
  if (fluxes) {
    ECK(cudaMemcpyAsync(e->h_pin, e->flux_step, 6 * (size_t)e->nm * 8, cudaMemcpyDeviceToHost, e->st));
    ECK(cudaStreamSynchronize(e->st));
    for (int q = 0; q < 6 * e->nm; ++q) fluxes[q] = fluxes[q] + e->h_pin[q];
  }
  return 0;
}

extern "C" int f3d_ens_get_fluxes(f3d_ens* e, double* fluxes) {
  if (!e || !fluxes) return set_error_msg("f3d_ens_get_fluxes: null argument");
  ECK(cudaSetDevice(e->device));
  ECK(cudaMemcpyAsync(e->h_pin, e->flux_tot, 12 * (size_t)e->nm * 8, cudaMemcpyDeviceToHost, e->st));
  ECK(cudaMemsetAsync(e->flux_tot, 0, 12 * (size_t)e->nm * 8, e->st));
  ECK(cudaStreamSynchronize(e->st));
  for (int m = 0; m < e->nm; ++m)
    for (int q = 0; q < 6; ++q)
      fluxes[6 * m + q] = fluxes[6 * m + q] + (e->h_pin[12 * m + q] - e->h_pin[12 * m + 6 + q]);
  return 0;
}

extern "C" int f3d_ens_mass_volume(f3d_ens* e, int mi, double* mass) {
  if (!e || !mass || mi < 0 || mi >= e->nm) return set_error_msg("f3d_ens_mass_volume: bad arguments");
  if (e->nb > 64) return set_error_msg("f3d_ens_mass_volume: more than 64 bins");
  ECK(cudaSetDevice(e->device));
  double* out = e->d_red + (size_t)e->mass_nblk * e->nb;
  launch_mass(e->dm, mi, e->nb, e->prec == F3D_PREC_FP32, e->d_red, e->mass_nblk, out, e->st);
  e->launches += 2;
  ECKL();
  ECK(cudaMemcpyAsync(e->h_pin, out, e->nb * 8, cudaMemcpyDeviceToHost, e->st));
  ECK(cudaStreamSynchronize(e->st));
  double tot = 0.0, comp = 0.0;
  for (int b = 0; b < e->nb; ++b) {
    double x = e->h_pin[b], t = tot + x;
    comp += (std::fabs(tot) >= std::fabs(x)) ? (tot - t) + x : (x - t) + tot;
    tot = t;
  }
  *mass = tot + comp;
  return 0;
}

extern "C" int f3d_ens_reset_state(f3d_ens* e) {
  if (!e) return set_error_msg("f3d_ens_reset_state: null ensemble");
  ECK(cudaSetDevice(e->device));
  for (int m = 0; m < e->nm; ++m) {
    const MemberDev& d = e->hm[m];
    const size_t ncell = (size_t)d.nx * d.ny * d.nz, nb = (size_t)e->nb;
    if (d.c32) ECK(cudaMemsetAsync(d.c32, 0, ncell * nb * 4, e->st));
    if (d.c32lo) ECK(cudaMemsetAsync(d.c32lo, 0, ncell * nb * 4, e->st));
    const size_t ngh = (size_t)gh_per_bin(d.nx, d.ny, d.nz) * nb;
    if (d.gh64) ECK(cudaMemsetAsync(d.gh64, 0, ngh * 8, e->st));
    if (d.gh32) ECK(cudaMemsetAsync(d.gh32, 0, ngh * 4, e->st));
    if (d.c64) ECK(cudaMemsetAsync(d.c64, 0, ncell * nb * 8, e->st));
    ECK(cudaMemsetAsync(d.acum, 0, (size_t)d.nx * d.ny * nb * 8, e->st));
  }
  for (int m = 0; m < (int)e->awet.size(); ++m) {
    const MemberDev& d = e->hm[m];
    ECK(cudaMemsetAsync(e->awet[m], 0, (size_t)d.nx * d.ny * e->nb * 8, e->st));
  }
  ECK(cudaMemsetAsync(e->flux_tot, 0, 12 * (size_t)e->nm * 8, e->st));
  ECK(cudaMemsetAsync(e->flux_step, 0, 6 * (size_t)e->nm * 8, e->st));
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

// ---- wet deposition, radioactive decay, output reductions -----------------
extern "C" int f3d_ens_set_class_wet_deposition(f3d_ens* e, int ci, double a, double b, const double* pre,
                                                const double* pblh, const double* h_c, const double* z_c,
                                                const int* bin_cat, const double* bin_diam) {
  if (!e || ci < 0 || ci >= e->ncls) return set_error_msg("f3d_ens_set_class_wet_deposition: bad class");
  if (!bin_cat) {
    e->wet_on = false;
    drop_graphs(e);
    return 0;
  }
  if (!pre || !pblh || !h_c || !z_c || !bin_diam)
    return set_error_msg("f3d_ens_set_class_wet_deposition: null array");
  EnsClass& k = e->cls[ci];
  if (!k.grid_set) return set_error_msg("f3d_ens_set_class_wet_deposition: class grid not set");
  if (e->nb > 64) return set_error_msg("f3d_ens_set_class_wet_deposition: at most 64 bins");
  ECK(cudaSetDevice(e->device));
  std::vector<double> powpb;
  std::vector<int> ktop;
  if (!wet_tables(k.nx, k.ny, k.nz, b, pre, pblh, h_c, z_c, powpb, ktop))
    return set_error_msg("f3d_ens_set_class_wet_deposition: heights not increasing with k");
  const size_t ncol = (size_t)k.nx * k.ny;
  if (!k.powpb && (ealloc(e, &k.powpb, ncol) || ealloc(e, &k.ktop, ncol))) return 1;
  ECK(cudaMemcpy(k.powpb, powpb.data(), ncol * 8, cudaMemcpyHostToDevice));
  ECK(cudaMemcpy(k.ktop, ktop.data(), ncol * 4, cudaMemcpyHostToDevice));
  if (e->awet.empty()) {
    e->awet.assign(e->nm, nullptr);
    for (int m = 0; m < e->nm; ++m) {
      const MemberDev& d = e->hm[m];
      if (ealloc(e, &e->awet[m], (size_t)d.nx * d.ny * e->nb)) return 1;
      ECK(cudaMemset(e->awet[m], 0, (size_t)d.nx * d.ny * e->nb * 8));
    }
  }
  k.wet_set = true;
  e->wet_mask = wet_bin_mask(e->nb, bin_cat, bin_diam);
  e->wet_a = a;
  e->wet_on = true;
  drop_graphs(e);
  return 0;
}

extern "C" int f3d_ens_set_radionuclides(f3d_ens* e, const int* bin_cat, const int* bin_spe) {
  if (!e) return set_error_msg("f3d_ens_set_radionuclides: null ensemble");
  drop_graphs(e);
  e->radio_on = false;
  e->radio = RadioSpec();
  if (!bin_cat || !bin_spe) return 0;
  if (e->nb > 64) return set_error_msg("f3d_ens_set_radionuclides: at most 64 bins");
  int bad = 0;
  const int rc = radio_spec(e->nb, bin_cat, bin_spe, e->radio, &bad);
  if (rc == 1) return set_error_msg("The number of SR90 and Y90 classes must be equal.");
  if (rc == 2) return set_error_msg("Invalid radionuclide type: species %d", bad);
  e->radio_on = !e->radio.bin.empty();
  if (!e->radio_on) return 0;
  ECK(cudaSetDevice(e->device));
  if (pull_dynamic(e)) return 1;
  std::vector<double> dts(e->nm);
  for (int m = 0; m < e->nm; ++m) dts[m] = e->hm[m].dt;
  return update_radio_factors(e, dts.data());
}

extern "C" int f3d_ens_get_member_awet(f3d_ens* e, int mi, double* my_awet) {
  if (!e || !my_awet || mi < 0 || mi >= e->nm) return set_error_msg("f3d_ens_get_member_awet: bad arguments");
  const EnsClass& k = e->cls[e->member_class[mi]];
  const size_t nx = k.nx, ny = k.ny, nb = e->nb;
  std::vector<double> d(nx * ny * nb, 0.0);
  if (!e->awet.empty()) {
    ECK(cudaSetDevice(e->device));
    ECK(cudaStreamSynchronize(e->st));
    ECK(cudaMemcpy(d.data(), e->awet[mi], d.size() * 8, cudaMemcpyDeviceToHost));
  }
  std::fill(my_awet, my_awet + (nx + 4) * (ny + 4) * nb, 0.0);
  for (size_t b = 0; b < nb; ++b)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i)
        my_awet[(i + 2) + (nx + 4) * ((j + 2) + (ny + 4) * b)] = d[(b * ny + j) * nx + i];
  return 0;
}

extern "C" int f3d_ens_mass_sink(f3d_ens* e, int mi, double* mass) {
  if (!e || !mass || mi < 0 || mi >= e->nm) return set_error_msg("f3d_ens_mass_sink: bad arguments");
  if (e->awet.empty()) {
    *mass = 0.0 + 0.0;
    return 0;
  }
  const EnsClass& k = e->cls[e->member_class[mi]];
  ECK(cudaSetDevice(e->device));
  const size_t ncol = (size_t)k.nx * k.ny, need = 4 * (size_t)(k.nx + 1) * (k.ny + 1);
  if (need > e->out_cap) {
    if (ealloc(e, &e->d_out, need)) return 1;
    e->out_cap = need;
  }
  launch_sink_cols(k.nx, k.ny, e->nb, e->awet[mi], e->hm[mi].dx1p, e->hm[mi].dx2p, e->d_out, e->st);
  e->launches += 1;
  ECKL();
  std::vector<double> col(ncol);
  ECK(cudaMemcpyAsync(col.data(), e->d_out, ncol * 8, cudaMemcpyDeviceToHost, e->st));
  ECK(cudaStreamSynchronize(e->st));
  *mass = mass_sink_sum(k.nx, k.ny, col.data());
  return 0;
}

extern "C" int f3d_ens_set_class_corner_heights(f3d_ens* e, int ci, const double* z_c) {
  if (!e || ci < 0 || ci >= e->ncls || !z_c) return set_error_msg("f3d_ens_set_class_corner_heights: bad arguments");
  EnsClass& k = e->cls[ci];
  if (!k.grid_set) return set_error_msg("f3d_ens_set_class_corner_heights: class grid not set");
  ECK(cudaSetDevice(e->device));
  const size_t n = (size_t)(k.nx + 1) * (k.ny + 1) * (k.nz + 1);
  if (!k.zc && ealloc(e, &k.zc, n)) return 1;
  ECK(cudaMemcpy(k.zc, z_c, n * 8, cudaMemcpyHostToDevice));
  return 0;
}

extern "C" int f3d_ens_output_member_species(f3d_ens* e, int mi, const int* bin_in, int col_du,
                                             double* con_sur, double* col_mass, double* cloud_top,
                                             double* grn_load) {
  if (!e || !bin_in || mi < 0 || mi >= e->nm)
    return set_error_msg("f3d_ens_output_member_species: bad arguments");
  if (e->nb > 64) return set_error_msg("f3d_ens_output_member_species: at most 64 bins");
  const EnsClass& k = e->cls[e->member_class[mi]];
  if ((con_sur || col_mass || cloud_top) && !k.zc)
    return set_error_msg("f3d_ens_output_member_species: corner heights not set (f3d_ens_set_class_corner_heights)");
  ECK(cudaSetDevice(e->device));
  const size_t ncol = (size_t)(k.nx + 1) * (k.ny + 1);
  if (4 * ncol > e->out_cap) {
    if (ealloc(e, &e->d_out, 4 * ncol)) return 1;
    e->out_cap = 4 * ncol;
  }
  const MemberDev& d = e->hm[mi];
  OutArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = k.nx;
  a.ny = k.ny;
  a.nz = k.nz;
  a.nb = e->nb;
  for (int q = 0; q < e->nb; ++q)
    if (bin_in[q]) a.mask |= 1ull << q;
  a.col_du = col_du;
  a.c64 = d.c64;
  a.c32 = d.c32;
  a.c32lo = d.c32lo;
  a.acum = d.acum;
  a.awet = e->awet.empty() ? nullptr : e->awet[mi];
  a.hm1 = d.hm1;
  a.hm2 = d.hm2;
  a.hm3 = d.hm3;
  a.zc = k.zc;
  a.gh64 = d.gh64;
  a.gh32 = d.gh32;
  if (con_sur || col_mass || cloud_top) {
    const size_t ncs = (size_t)__builtin_popcountll(a.mask) * k.nx * k.ny * k.nz;
    const size_t need = ncs + (size_t)(k.nz + 1) * ncol;
    if (need > e->cs_cap) {
      if (ealloc(e, &e->d_cs, need)) return 1;
      e->cs_cap = need;
    }
    a.cs = e->d_cs;
    a.wbuf = e->d_cs + ncs;
  }
  double* outs[4] = {con_sur, col_mass, cloud_top, grn_load};
  double* dev[4];
  for (int q = 0; q < 4; ++q) dev[q] = outs[q] ? e->d_out + q * ncol : nullptr;
  a.con_sur = dev[0];
  a.col_mass = dev[1];
  a.cloud_top = dev[2];
  a.grn_load = dev[3];
  launch_out_columns(a, e->st);
  e->launches += 1;
  ECKL();
  for (int q = 0; q < 4; ++q)
    if (outs[q]) ECK(cudaMemcpyAsync(outs[q], dev[q], ncol * 8, cudaMemcpyDeviceToHost, e->st));
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

extern "C" int f3d_ens_set_profiling(f3d_ens* e, int on) {
  if (!e) return set_error_msg("f3d_ens_set_profiling: null ensemble");
  ECK(cudaSetDevice(e->device));
  if (on && !e->pev[0])
    for (auto& ev : e->pev) ECK(cudaEventCreate(&ev));
  e->prof = on != 0;
  for (double& x : e->prof_ms) x = 0.0;
  e->prof_steps = 0;
  return 0;
}

extern "C" int f3d_ens_get_profile(f3d_ens* e, double* ms, int* nsteps) {
  if (!e || !ms) return set_error_msg("f3d_ens_get_profile: null argument");
  for (int q = 0; q < 5; ++q) ms[q] = e->prof_ms[q];
  if (nsteps) *nsteps = e->prof_steps;
  return 0;
}

extern "C" int f3d_ens_synchronize(f3d_ens* e) {
  if (!e) return set_error_msg("f3d_ens_synchronize: null ensemble");
  ECK(cudaSetDevice(e->device));
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

extern "C" int f3d_ens_get_stream(f3d_ens* e, void** stream) {
  if (!e || !stream) return set_error_msg("f3d_ens_get_stream: null argument");
  *stream = (void*)e->st;
  return 0;
}

extern "C" int f3d_ens_launch_count(f3d_ens* e, long long* count) {
  if (!e || !count) return set_error_msg("f3d_ens_launch_count: null argument");
  *count = e->launches;
  return 0;
}

extern "C" int f3d_ens_status(f3d_ens* e, int* device_error) {
  if (!e || !device_error) return set_error_msg("f3d_ens_status: null argument");
  ECK(cudaSetDevice(e->device));
  ECK(cudaStreamSynchronize(e->st));
  ECK(cudaMemcpy(device_error, e->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int f3d_ens_clear_status(f3d_ens* e) {
  if (!e) return set_error_msg("f3d_ens_clear_status: null ensemble");
  ECK(cudaSetDevice(e->device));
  ECK(cudaMemsetAsync(e->d_err, 0, sizeof(int), e->st));
  ECK(cudaStreamSynchronize(e->st));
  return 0;
}

// Finite scan of one member's state and its class's device inputs (bits as
// in f3d_ads_check_finite).
extern "C" int f3d_ens_check_finite(f3d_ens* e, int mi, int* mask) {
  if (!e || !mask || mi < 0 || mi >= e->nm) return set_error_msg("f3d_ens_check_finite: bad arguments");
  ECK(cudaSetDevice(e->device));
  const MemberDev& m = e->hm[mi];
  const long long nx = m.nx, ny = m.ny, nz = m.nz, nb = e->nb, ncell = nx * ny * nz;
  unsigned int* dmask = reinterpret_cast<unsigned int*>(e->d_nfail) + 2;
  ECK(cudaMemsetAsync(dmask, 0, sizeof(unsigned int), e->st));
  launch_nonfinite(m.c64, ncell * nb, 0, dmask, e->st);
  launch_nonfinite(m.c32, ncell * nb, 0, dmask, e->st);
  launch_nonfinite(m.c32lo, ncell * nb, 0, dmask, e->st);
  launch_nonfinite(m.acum, nx * ny * nb, 1, dmask, e->st);
  launch_nonfinite(m.ux[0], 2 * (nx + 1) * ny * nz, 2, dmask, e->st);
  launch_nonfinite(m.vy[0], 2 * (ny + 1) * nx * nz, 3, dmask, e->st);
  launch_nonfinite(m.wz[0], 2 * (nz + 1) * nx * ny, 4, dmask, e->st);
  launch_nonfinite(m.k1x, (nx + 2) * ny * nz, 5, dmask, e->st);
  launch_nonfinite(m.k2y, (ny + 2) * nx * nz, 6, dmask, e->st);
  launch_nonfinite(m.k3z, (nz + 2) * nx * ny, 7, dmask, e->st);
  launch_nonfinite(m.vs, nb * (nz + 1) * nx * ny, 8, dmask, e->st);
  ECKL();
  unsigned int h = 0;
  ECK(cudaMemcpyAsync(&h, dmask, sizeof(h), cudaMemcpyDeviceToHost, e->st));
  ECK(cudaStreamSynchronize(e->st));
  *mask = (int)h;
  return 0;
}
