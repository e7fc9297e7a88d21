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
#include "march.cuh"
#include "step_dev.cuh"

#ifndef F3D_PF64
#define F3D_PF64 1
#endif
#ifndef F3D_V64
#define F3D_V64 1
#endif
// Element offsets along a pencil within one bin: 32-bit with F3D_STRIDE32_64
// (grids with (nx+1)(ny+1)(nz+1) < 2^31), else 64-bit.
#ifndef F3D_STRIDE32_64
#define F3D_STRIDE32_64 0
#endif
#if F3D_STRIDE32_64
typedef int pstride64_t;
#else
typedef long long pstride64_t;
#endif

namespace f3d {

// Limiter r(i) from d1 = c(i)-c(i-1), d0 = c(i+1)-c(i)  (mod_ADS.F90:1124-1223).
// The division is taken only when |d0| >= 1e-12 (a safe divisor otherwise,
// so zero differences never reach the slow path of the division).
template <int LIM>
__device__ __forceinline__ double limiter64(double d1, double d0) {
  const bool small0 = fabs(d0) < kEps;
  const double r = d1 / (small0 ? 1.0 : d0);
  if (LIM == 1) {
    return small0 ? 1.0 : fmax(0.0, fmin(1.0, r));
  } else if (LIM == 2) {
    double a = fmin(2.0 * r, 1.0), b = fmin(r, 2.0);
    double v = fmax(fmax(0.0, a), b);
    return small0 ? ((fabs(d1) < kEps) ? 0.0 : 2.0) : v;
  } else {
    double v = 1.5 * (r * r + r) / (r * r + r + 1.0);
    return small0 ? ((fabs(d1) < kEps) ? 0.0 : 1.5) : v;
  }
}

// Per-pencil operations of the FP64 form, reference operation order.
// EPI (z only): wet deposition and decay applied to each cell as it is
// stored (ZEpi).
template <int LIM, int DIR, bool EPI = false>
struct Ops64 {
  double* cp;
  pstride64_t cs;
  const double* vel;   // current face velocity, face f at vel[f * vs]
  const double* vsub;  // z: settling velocity of the bin at the same faces
  pstride64_t vs;
  const double* kk;    // 0.5 (k(f) + k(f-1)) at face f, same stride
  const double4* geo;  // {dxp(p), 1/dxp(p), dxb(p), 1/dxb(p)} at geo[p + 1]
  int nf;              // cells of the pencil (faces 0..nf)
  double dt, hdt;
  XTile<double> xt;    // x pencils: shared-memory staging of the rows
  ZEpi epi;            // EPI: the column's wet deposition and decay

  __device__ __forceinline__ double load_c(int p) const {
    if constexpr (DIR == DIR_X) {
      return xt.load(p);
    } else {
      // the line of a later position into L1 ahead of its load
      if (F3D_PF64) asm volatile("prefetch.global.L1 [%0];" ::"l"(cp + (pstride64_t)min(p + 8, nf - 1) * cs));
      return cp[p * cs];
    }
  }
  __device__ __forceinline__ double load_last() const { return cp[(pstride64_t)(nf - 1) * cs]; }
  __device__ __forceinline__ void store_c(int p, double v) {
    if constexpr (DIR == DIR_X) xt.store(p, v);
    else if constexpr (EPI) cp[p * cs] = epi.apply(p, v);
    else cp[p * cs] = v;
  }
  __device__ __forceinline__ void stage_init() { if constexpr (DIR == DIR_X) xt.init(); }
  __device__ __forceinline__ void stage_begin(int T0) { if constexpr (DIR == DIR_X) xt.block_begin(T0); }
  __device__ __forceinline__ void stage_end(int T0) { if constexpr (DIR == DIR_X) xt.block_end(T0); }
  __device__ __forceinline__ void stage_finish() { if constexpr (DIR == DIR_X) xt.finish(); }
  __device__ __forceinline__ FaceV<double> face(int f) const {
    if (F3D_PF64) {
      const pstride64_t fp = (pstride64_t)min(f + 8, nf) * vs;
      asm volatile("prefetch.global.L1 [%0];" ::"l"(vel + fp));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(kk + fp));
      if (DIR == DIR_Z) asm volatile("prefetch.global.L1 [%0];" ::"l"(vsub + fp));
    }
    FaceV<double> r;
    r.u = vel[f * vs];
    if (DIR == DIR_Z) r.u = r.u - vsub[f * vs];  // CB%w - my_vs  (mod_ADS.F90:670)
    r.k = kk[f * vs];
    r.r = 0.0;  // the exact form reads its metrics from geo
    return r;
  }
  // face data for the unguarded march (faces outside [0, nf] read the end
  // faces; the right-hand side of a cell outside the pencil is set to 0 in
  // arrive, so its stage values stay the frozen ghost value exactly)
  __device__ __forceinline__ FaceV<double> face_v(int f) const { return face(min(max(f, 0), nf)); }
  // free flow (mod_ADS.F90:1227-1326) with bvalue = 0
  __device__ __forceinline__ double ghost_l(double c0, double uL) const {
    return (uL > 0.0) ? 2.0 * 0.0 - c0 : c0;
  }
  __device__ __forceinline__ double ghost_r(double cn, double uR) const {
    return (uR < 0.0) ? 2.0 * 0.0 - cn : cn;
  }
  // RK4 combinations (mod_ADS.F90:326-390) and Euler (:302)
  __device__ __forceinline__ double euler(double c, double k) const { return c + dt * k; }
  __device__ __forceinline__ double rk_half(double c, double k) const { return c + hdt * k; }
  __device__ __forceinline__ double rk_new1(double c, double k) const {
    return c + div_rn_recip(dt * k, 6.0, 1.0 / 6.0);
  }
  __device__ __forceinline__ double rk_add3(double nw, double k) const {
    return nw + div_rn_recip(dt * k, 3.0, 1.0 / 3.0);
  }
  __device__ __forceinline__ double rk_full(double c, double k) const { return c + dt * k; }
  __device__ __forceinline__ double rk_final(double nw, double k) const {
    return nw + div_rn_recip(dt * k, 6.0, 1.0 / 6.0);
  }

  // KT_RHS at cell q-2 on arrival of a(q) (mod_ADS.F90:1089-1117)
  template <bool G>
  __device__ __forceinline__ void arrive(StageS<double>& s, int q, double a0, FaceV<double> fv,
                                         int p, double& rhs, double& flux) const {
    const double d0 = a0 - s.a1;
    const double r1 = limiter64<LIM>(s.d1, d0);
    if (!G || q >= 1) {
      const double u = fv.u;
      const double cl = s.a2 + 0.5 * s.h2 * s.d1;
      const double cr = s.a1 - 0.5 * r1 * d0;
      const double F_l = cl * u;
      const double F_r = cr * u;
      const double F0 = 0.5 * (F_l + F_r) - 0.5 * fabs(u) * (cr - cl);
      const double4 g = geo[min(max(p + 1, 0), nf)];
      const double P0 = div_rn_recip(fv.k * s.d1, g.x, g.y);
      flux = F0 + P0;
      if (!G || q >= 2) rhs = div_rn_recip(P0 - s.P1, g.z, g.w) - div_rn_recip(F0 - s.F1, g.z, g.w);
      if (!G) rhs = (p >= 0 && p < nf) ? rhs : 0.0;  // ghost cells of the unguarded march
      s.F1 = F0;
      s.P1 = P0;
    }
    s.a2 = s.a1;
    s.a1 = a0;
    s.d1 = d0;
    s.h2 = r1;
  }
};

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

// One pencil of a sweep: march, boundary fluxes, kept ghosts and (z) the
// deposit; EPI adds the wet deposition and decay epilogue (z only).
template <int DIR, int LIM, int TM, bool EPI>
__device__ __forceinline__ void sweep64_pencil(const MemberDev& m, long long pen, int b, bool lane_ok,
                                               int warp, unsigned char* f3d_smem, double& clo,
                                               double& chi) {
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  Ops64<LIM, DIR, EPI> o;
  double area;
  int n, i = 0, j = 0;
  if (DIR == DIR_X) {
    j = (int)(pen % ny);
    int k = (int)(pen / ny);
    n = nx;
    o.cp = m.c64 + (((long long)b * nz + k) * ny + j) * nx;
    o.xt.setup(f3d_smem + warp * XTile<double>::BYTES, lane_ok ? o.cp : nullptr,
               threadIdx.x & 31, nx);
    o.cs = 1;
    long long fo = (long long)k * (nx + 1) * ny + j;
    o.vel = m.ucur + fo;
    o.kk = m.kkf[0] + fo;
    o.vs = ny;
    o.vsub = nullptr;
    area = m.dx3b[k + 1] * m.dx2b[j + 1];
  } else if (DIR == DIR_Y) {
    i = (int)(pen % nx);
    int k = (int)(pen / nx);
    n = ny;
    o.cp = m.c64 + ((long long)b * nz + k) * ny * (long long)nx + i;
    o.cs = nx;
    long long fo = (long long)k * (ny + 1) * nx + i;
    o.vel = m.vcur + fo;
    o.kk = m.kkf[1] + fo;
    o.vs = nx;
    o.vsub = nullptr;
    area = m.dx3b[k + 1] * m.dx1b[i + 1];
  } else {
    i = (int)(pen % nx);
    j = (int)(pen / nx);
    n = nz;
    o.cp = m.c64 + (long long)b * nz * ny * nx + (long long)j * nx + i;
    o.cs = (pstride64_t)nx * ny;
    long long fo = (long long)j * nx + i;
    o.vel = m.wcur + fo;
    o.kk = m.kkf[2] + fo;
    o.vs = (pstride64_t)nx * ny;
    o.vsub = m.vs + (long long)b * (nz + 1) * ny * nx + fo;
    area = m.dx2b[j + 1] * m.dx1b[i + 1];
    if constexpr (EPI) o.epi = zepi_setup(m, b, fo);
  }
  o.geo = m.geo[DIR];
  o.nf = n;
  o.dt = m.dt;
  o.hdt = 0.5 * m.dt;
  // RK4: the edge blocks run the unguarded body (cheaper than the guarded one)
  March<double, Ops64<LIM, DIR, EPI>, TM, (F3D_V64 != 0)> M(o, n);
  M.run();
  const double dt = m.dt;
  if (lane_ok) {
    clo = M.flux_lo * area * dt;
    chi = M.flux_hi * area * dt;
    if (m.gh64) {  // the free-flow ghosts of this pencil (mod_ADS.F90:1227-1326)
      double* g = m.gh64 + (long long)b * gh_per_bin(nx, ny, nz);
      g[gh_offset(DIR, 0, pen, nx, ny, nz)] = M.gL;
      g[gh_offset(DIR, 1, pen, nx, ny, nz)] = M.gR;
    }
  }
  if (DIR == DIR_Z && lane_ok) {
    const long long ij = (long long)j * nx + i;
    double* a = m.acum + (long long)b * ny * nx + ij;
    *a = *a + fabs(M.flux_lo) * dt;  // mod_ADS.F90:791
    if constexpr (EPI) zepi_finish(m, o.epi, b, ij);
  }
}

// One work item of a sweep (per-sweep kernels and the persistent step kernel).
template <int DIR, int LIM, int TM, bool EPI = false>
__device__ __forceinline__ void sweep64_item(const MemberDev* __restrict__ members,
                                             const WorkItem w, int bpb, unsigned char* f3d_smem) {
  const MemberDev& m = members[w.member];
  const long long nsp = (DIR == DIR_X) ? (long long)m.ny * m.nz
                        : (DIR == DIR_Y) ? (long long)m.nx * m.nz : (long long)m.nx * m.ny;
  const int warp = threadIdx.x >> 5;
  const long long pen_raw = (long long)w.pen0 + 32 * (warp / bpb) + (threadIdx.x & 31);
  const long long pen0w = (long long)w.pen0 + 32 * (warp / bpb);
  const int b = w.bin0 + warp % bpb;
  const bool lane_ok = pen_raw < nsp && b < m.nb;
  // x pencils march as a whole warp (the staging is warp-collective); lanes
  // past the end replay the last pencil without storing
  const bool run_it = (DIR == DIR_X) ? (pen0w < nsp && b < m.nb) : lane_ok;
  const long long pen = pen_raw < nsp ? pen_raw : nsp - 1;
  double clo = 0.0, chi = 0.0;  // contributions flux*area*dt
  if (run_it) {
    // the epilogue is a kernel instance of its own (chosen at launch), so
    // that the sweeps without it keep their register allocation
    sweep64_pencil<DIR, LIM, TM, DIR == DIR_Z && EPI>(m, pen, b, lane_ok, warp, f3d_smem, clo, chi);
  }
  block_reduce2(clo, chi, m.flux_part + 2 * (long long)w.slot);
}

// y and z: 3 blocks of 128 threads per SM (168 registers, a few hundred
// bytes spilled), 9-10% faster than 2 blocks at 222-230 registers; x keeps
// the compiler's own choice (2 blocks), 4% faster there than 3.
#ifndef F3D_FP64_MINB
#define F3D_FP64_MINB 3
#endif
template <int DIR, int LIM, int TM, bool EPI = false>
__global__ void __launch_bounds__(128, F3D_FP64_MINB) k_sweep64(const MemberDev* __restrict__ members,
                                                                 const WorkItem* __restrict__ work,
                                                                 int bpb) {
  extern __shared__ __align__(16) unsigned char f3d_smem[];
  sweep64_item<DIR, LIM, TM, EPI>(members, work[blockIdx.x], bpb, f3d_smem);
}
#ifdef F3D_FP64_XMINB
#define F3D_SWEEP64X_BOUNDS __launch_bounds__(128, F3D_FP64_XMINB)
#else
#define F3D_SWEEP64X_BOUNDS __launch_bounds__(128)
#endif
template <int LIM, int TM>
__global__ void F3D_SWEEP64X_BOUNDS k_sweep64x(const MemberDev* __restrict__ members,
                                                  const WorkItem* __restrict__ work, int bpb) {
  extern __shared__ __align__(16) unsigned char f3d_smem[];
  sweep64_item<DIR_X, LIM, TM>(members, work[blockIdx.x], bpb, f3d_smem);
}

// Host launchers -------------------------------------------------------------
template <int DIR, bool EPI = false>
static void launch_dir64(int lim, int tm, const MemberDev* members,
                         const WorkItem* work, int nblocks, int bpb, cudaStream_t st) {
  dim3 g(nblocks), b(128);
  const int smem = (DIR == DIR_X) ? 4 * XTile<double>::BYTES : 0;
  static bool attr_set = false;
  if (!attr_set && smem > 0) {
    cudaFuncSetAttribute(k_sweep64x<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_sweep64x<2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_sweep64x<3, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_sweep64x<1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_sweep64x<2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_sweep64x<3, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr_set = true;
  }
#define F3D_L(L, T)                                                             \
  do {                                                                          \
    if constexpr (DIR == DIR_X) k_sweep64x<L, T><<<g, b, smem, st>>>(members, work, bpb); \
    else k_sweep64<DIR, L, T, EPI><<<g, b, smem, st>>>(members, work, bpb);     \
  } while (0)
  if (tm == 1) {
    if (lim == 1) F3D_L(1, 1); else if (lim == 2) F3D_L(2, 1); else F3D_L(3, 1);
  } else {
    if (lim == 1) F3D_L(1, 2); else if (lim == 2) F3D_L(2, 2); else F3D_L(3, 2);
  }
#undef F3D_L
}

// epi: the z sweep runs the wet deposition and decay epilogue (the members'
// epi_on)
void launch_sweep64(int dir, int lim, int tm, int epi, const MemberDev* members,
                    const WorkItem* work, int nblocks, int bpb, cudaStream_t st) {
  if (nblocks <= 0) return;
  if (dir == DIR_X) launch_dir64<DIR_X>(lim, tm, members, work, nblocks, bpb, st);
  else if (dir == DIR_Y) launch_dir64<DIR_Y>(lim, tm, members, work, nblocks, bpb, st);
  else if (epi) launch_dir64<DIR_Z, true>(lim, tm, members, work, nblocks, bpb, st);
  else launch_dir64<DIR_Z>(lim, tm, members, work, nblocks, bpb, st);
}

// Per-step preparation: current winds u,v,w = (1-s) x1 + s x2
// (mod_F3D.F90:1437-1439, mod_ADS.F90:667), then the sparse source term
// c += dt*s/vol (mod_F3D.F90:1456-1473).
// Current winds of one member: u = (1-s) f u1 + s f u2 with the member's
// wind factor f applied to the snapshots first (the ensemble perturbs the
// meteo winds, task_Fall3d.F90:194-198; f = 1 for a single run leaves the
// values unchanged), w = (1-s) w1 + s w2.  Elements [q0, q0+cnt) of the
// member's concatenated (u, v, w) face list.
__device__ __forceinline__ void prep64_range(const MemberDev& m, long long q0, long long cnt,
                                             int mask) {
  const long long nu = (long long)(m.nx + 1) * m.ny * m.nz;
  const long long nv = (long long)(m.ny + 1) * m.nx * m.nz;
  const long long nw = (long long)(m.nz + 1) * m.nx * m.ny;
  const double s = m.stime, f = m.wfacd;
  for (long long e = threadIdx.x; e < cnt; e += blockDim.x) {
    long long q = q0 + e;
    if (q < nu) {
      if (mask & 1) m.ucur[q] = (1.0 - s) * (f * m.ux[0][q]) + s * (f * m.ux[1][q]);
      continue;
    }
    q -= nu;
    if (q < nv) {
      if (mask & 2) m.vcur[q] = (1.0 - s) * (f * m.vy[0][q]) + s * (f * m.vy[1][q]);
      continue;
    }
    q -= nv;
    if (q < nw && (mask & 4)) m.wcur[q] = (1.0 - s) * m.wz[0][q] + s * m.wz[1][q];
  }
}

__global__ void k_prep64(const MemberDev* __restrict__ members, const int* __restrict__ blk_member,
                         const int* __restrict__ blk_first, int mask) {
  const int mi = blk_member[blockIdx.x];
  prep64_range(members[mi], (long long)(blockIdx.x - blk_first[mi]) * 256, 256, mask);
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

namespace f3d {

__device__ __forceinline__ void source64_all(MemberDev* members, int nmembers) {
  for (int mi = 0; mi < nmembers; ++mi) {
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

template <int DIR, int LIM, int TM, bool EPI = false>
__device__ __noinline__ void sweep64_item_call(MemberDev* members, WorkItem w, int bpb,
                                               unsigned char* smem) {
  sweep64_item<DIR, LIM, TM, EPI>(members, w, bpb, smem);
}

// FP64 form of the persistent step kernel (see k_fused32); the first phase
// also builds each member's current winds.
template <int LIM, int TM>
__global__ void __launch_bounds__(128) k_fused64(FusedArgs a) {
  extern __shared__ __align__(16) unsigned char f3d_smem[];
  __shared__ int slot;
  __shared__ double sa[128], sb[128];
  for (;;) {
    const int it = grab_item(a.counters + 3, &slot);
    if (it >= a.nprep) break;
    const int mi = a.prep_member[it];
    prep64_range(a.members[mi], (long long)(it - a.prep_first[mi]) * 256, 256, 7);
  }
  source64_all(a.members, a.nmembers);
  grid_barrier(a.counters + 6, a.err, a.wait_limit);
  const bool xfirst = (a.members[0].iiter % 2) == 0;
  for (int ph = 0; ph < 3; ++ph) {
    const int dir = (ph == 2) ? 2 : (((ph == 0) == xfirst) ? 0 : 1);
    for (;;) {
      const int it = grab_item(a.counters + ph, &slot);
      if (it >= a.nwork[dir]) break;
      const WorkItem w = a.work[dir][it];
      if (dir == 0) sweep64_item_call<0, LIM, TM>(a.members, w, a.bpb, f3d_smem);
      else if (dir == 1) sweep64_item_call<1, LIM, TM>(a.members, w, a.bpb, f3d_smem);
      else if (a.epi) sweep64_item_call<2, LIM, TM, true>(a.members, w, a.bpb, f3d_smem);
      else sweep64_item_call<2, LIM, TM>(a.members, w, a.bpb, f3d_smem);
    }
    grid_barrier(a.counters + 6, a.err, a.wait_limit);
  }
  for (int mi = blockIdx.x; mi < a.nmembers; mi += gridDim.x) {
    member_flux_reduce(a.members[mi], 7, sa, sb);
    if (threadIdx.x == 0) member_advance(a.members[mi]);
    __syncthreads();
  }
}

int fused64_smem() { return 4 * XTile<double>::BYTES; }

const void* fused64_func(int lim, int tm) {
  if (tm == 1) {
    if (lim == 1) return (const void*)k_fused64<1, 1>;
    if (lim == 2) return (const void*)k_fused64<2, 1>;
    return (const void*)k_fused64<3, 1>;
  }
  if (lim == 1) return (const void*)k_fused64<1, 2>;
  if (lim == 2) return (const void*)k_fused64<2, 2>;
  return (const void*)k_fused64<3, 2>;
}

}  // namespace f3d
