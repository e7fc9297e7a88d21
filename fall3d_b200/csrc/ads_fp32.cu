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

#include <algorithm>

#include "f3d_common.cuh"
// The RK4 march's last block stops after t = n + 7 when that falls in its
// first half (the steps after it store nothing, so the results are the
// same bits).  On the B200 this made the compensated 64-member ensemble
// step 2.4% faster, x and y included (code layout); the FP64 form keeps
// the full block.
#ifndef F3D_HALF_TAIL
#define F3D_HALF_TAIL 1
#endif
#include "march.cuh"
#include "step_dev.cuh"

namespace f3d {

constexpr float kEpsF = 1e-12f;

// Three-input max (one instruction on sm_100).
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ unsigned int sign_bit(float x) { return __float_as_uint(x) & 0x80000000u; }
__device__ __forceinline__ float xor_sign(float x, unsigned int s) {
  return __uint_as_float(__float_as_uint(x) ^ s);
}

#ifndef F3D_LIM_EPS
#define F3D_LIM_EPS 1
#endif
#ifndef F3D_CMP_EFT
#define F3D_CMP_EFT 1
#endif
#ifndef F3D_CMP_XW
#define F3D_CMP_XW 16
#endif
#ifndef F3D_FFORM
#define F3D_FFORM 0
#endif

// 0.5 * phi(r) * d0 with r = d1/d0  (d1 = c(i)-c(i-1), d0 = c(i+1)-c(i)).
// Superbee and minmod are evaluated division-free on x = d1 sign(d0) and
// y = |d0|, so that the sign test of r costs nothing:
//   superbee  0.5 phi d0 = sign(d0) max(0, min(x, y/2), min(x/2, y))
//   minmod    0.5 phi d0 = sign(d0) max(0, min(x, y)) / 2
// (mod_ADS.F90:1124-1187).  The reference's |d0| < 1e-12 branches are kept
// by feeding the general formula a substitute x there: x = 1e30 gives the
// largest slope, y = |d0| (superbee phi = 2; minmod phi = 1, :1139-1140), and
// x = -1 gives 0 (superbee with |d1| < 1e-12 too, :1171-1173).  They decide
// the fluxes in the dilute fringe of the plume, which dominates the early
// ground deposit.  (F3D_LIM_EPS=0 drops them: a half-slope change below
// 1e-12 there, about 8% fewer instructions.)
template <int LIM>
__device__ __forceinline__ float half_phid(float d1, float d0) {
  const unsigned int sg = sign_bit(d0);
  float x = xor_sign(d1, sg);
  const float y = fabsf(d0);
#if F3D_LIM_EPS
  if (LIM == 2) {
    const float xs = (fabsf(d1) < kEpsF) ? -1.f : 1e30f;
    x = (y < kEpsF) ? xs : x;
  } else if (LIM == 1) {
    x = (y < kEpsF) ? 1e30f : x;
  }
#endif
  if (LIM == 1) {  // minmod
    return xor_sign(0.5f * fmaxf(0.f, fminf(x, y)), sg);
  } else if (LIM == 2) {  // superbee
    return xor_sign(max3f(0.f, fminf(x, 0.5f * y), fminf(0.5f * x, y)), sg);
  } else {  // ospre, mod_ADS.F90:1191-1223: 1.5 (r^2+r)/(r^2+r+1) * d0
    float num = d1 * (d1 + d0);
    float den = fmaf(d1, d1 + d0, d0 * d0);
    float pd = 1.5f * num * __frcp_rn(den) * d0;
    if (fabsf(d0) < kEpsF) pd = (fabsf(d1) < kEpsF) ? 0.f : 1.5f * d0;
    return 0.5f * pd;
  }
}

// Prefetch distances (march steps) of the face data and, in y and z, of the
// concentration: the loads themselves stay one step (faces) or four steps
// (concentration) ahead in registers, and the prefetch brings the lines into
// L1 early enough to hide the L2/HBM latency without holding registers.
#ifndef F3D_FACE_PF
#define F3D_FACE_PF 8
#endif
#ifndef F3D_C_PF
#define F3D_C_PF 8
#endif
#ifndef F3D_C_PF_Z
#define F3D_C_PF_Z F3D_C_PF
#endif
#ifndef F3D_FACE_PF_Z
#define F3D_FACE_PF_Z F3D_FACE_PF
#endif
#ifndef F3D_PF_L2
#define F3D_PF_L2 0
#endif
// Element offsets along a pencil (p * stride within one bin of one member,
// and the face offsets likewise): 32-bit, which cuts the index arithmetic of
// the sweeps (4-9% faster); the hosts accept precision-form grids only while
// (nx+1)(ny+1)(nz+1) stays below 2^31 (kMaxPencilSpan).
#ifndef F3D_STRIDE32
#define F3D_STRIDE32 1
#endif
#if F3D_STRIDE32
typedef int pstride_t;
#else
typedef long long pstride_t;
#endif
__device__ __forceinline__ void prefetch_line(const void* p) {
  if (F3D_PF_L2) asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  else asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Per-pencil operations of the precision form.  The current wind is
// interpolated in time on the fly from the two meteo snapshots and scaled by
// the member's wind factor (ensemble perturbation of u, v).
template <int LIM, int DIR, int TM, bool CMP = false, bool EPI = false>
struct Ops32 {
  float* cp;
  pstride_t cs;
  float* lop;          // CMP: low part of the state, same layout and stride as cp
  const double* r64;   // CMP: 1/dxb of the pencil's cells, FP64
  const float2* r2;    // CMP: the same as FP32 pairs {hi, lo}
  float dtf_hi, dtf_lo;  // CMP: weight of the face sums, dt/6 (RK4) or dt (Euler),
                         // as an FP32 pair: folded into the FP32 sums it would scale
                         // the interior transport against the FP64 boundary terms
  const float4* fd;   // face data {u(its), u(ite), kf, 1/dxb(f-1)} (MemberDev::f4)
  const float* vsub;  // z: settling velocity of the bin
  pstride_t vs;
  int nf;  // cells of the pencil (faces 0..nf)
  float s0, s1, wfac;
  float dt, hdt, dt3, dt6;
  // x pencils: shared-memory staging of the rows (the compensated form also
  // stages the low part, in narrower chunks so that both tiles fit)
  static constexpr int XW = CMP ? F3D_CMP_XW : 32;
  XTile<float, (TM == 2) ? 1 : 2, XW> xt;
  XLoTile<XW> lt;
  // EPI (z): the column's wet deposition and decay (an empty struct otherwise)
  std::conditional_t<EPI, ZEpi, NoEpi> epi;

  __device__ __forceinline__ float load_c(int p) const {
    if constexpr (DIR == DIR_X) {
      return xt.load(p);
    } else {
      constexpr int pf = (DIR == DIR_Z) ? F3D_C_PF_Z : F3D_C_PF;
      if constexpr (pf > 0) prefetch_line(cp + (pstride_t)min(p + pf, nf - 1) * cs);
      return cp[p * cs];
    }
  }
  __device__ __forceinline__ float load_last() const { return cp[(pstride_t)(nf - 1) * cs]; }
  __device__ __forceinline__ void store_c(int p, float v) {
    if constexpr (DIR == DIR_X) xt.store(p, v);
    else if constexpr (EPI && !CMP) cp[p * cs] = epi.apply32(p, v);
    else cp[p * cs] = v;  // the compensated pair went through the epilogue in final_cmp
  }
  __device__ __forceinline__ void stage_init() {
    if constexpr (DIR == DIR_X) xt.init();
    if constexpr (DIR == DIR_X && CMP) lt.init();
  }
  __device__ __forceinline__ void stage_begin(int T0) {
    if constexpr (DIR == DIR_X) xt.block_begin(T0);
    if constexpr (DIR == DIR_X && CMP) lt.block_begin(T0);
  }
  __device__ __forceinline__ void stage_end(int T0) {
    if constexpr (DIR == DIR_X) xt.block_end(T0);
    if constexpr (DIR == DIR_X && CMP) lt.block_end(T0);
  }
  __device__ __forceinline__ void stage_finish() {
    if constexpr (DIR == DIR_X) xt.finish();
    if constexpr (DIR == DIR_X && CMP) lt.finish();
  }
  __device__ __forceinline__ FaceV<float> face(int f) const {
    constexpr int fpf = (DIR == DIR_Z) ? F3D_FACE_PF_Z : F3D_FACE_PF;
    if constexpr (fpf > 0) {
      const pstride_t fp = (pstride_t)min(f + fpf, nf) * vs;
      prefetch_line(fd + fp);
      if constexpr (DIR == DIR_Z) prefetch_line(vsub + fp);
    }
    FaceV<float> r;
    const float4 q = __ldg(fd + f * vs);
    float w = fmaf(s0, q.x, s1 * q.y);
#if F3D_FFORM == 1
    if (DIR == DIR_Z) r.u = fmaf(-0.5f, __ldg(vsub + f * vs), w);  // s0, s1 carry the 0.5
    else r.u = wfac * w;                                           // wfac carries the 0.5
#else
    if (DIR == DIR_Z) r.u = w - __ldg(vsub + f * vs);
    else r.u = wfac * w;
#endif
    r.k = q.z;
    r.r = q.w;
    return r;
  }
  // face data for the unguarded march: faces outside [0, nf] read the end
  // face with 1/dxb = 0 (face 0 holds 0 there already), so that the
  // right-hand side of a ghost cell is 0
  __device__ __forceinline__ FaceV<float> face_v(int f) const {
    FaceV<float> r = face(min(max(f, 0), nf));
    if (f > nf) r.r = 0.f;
    return r;
  }
  __device__ __forceinline__ float ghost_l(float c0, float uL) const { return (uL > 0.f) ? -c0 : c0; }
  __device__ __forceinline__ float ghost_r(float cn, float uR) const { return (uR < 0.f) ? -cn : cn; }
  __device__ __forceinline__ float euler(float c, float k) const { return fmaf(dt, k, c); }
  __device__ __forceinline__ float rk_half(float c, float k) const { return fmaf(hdt, k, c); }
  __device__ __forceinline__ float rk_new1(float c, float k) const { return fmaf(dt6, k, c); }
  __device__ __forceinline__ float rk_add3(float nw, float k) const { return fmaf(dt3, k, nw); }
  __device__ __forceinline__ float rk_full(float c, float k) const { return fmaf(dt, k, c); }
  __device__ __forceinline__ float rk_final(float nw, float k) const { return fmaf(dt6, k, nw); }

  // low part of cell p (y, z: global, with an L1 prefetch of a later cell's
  // line; x: the staged tile)
  __device__ __forceinline__ float lo_fetch(int p) {
    if constexpr (DIR == DIR_X) {
      return lt.at(p);
    } else {
      prefetch_line(lop + (pstride_t)min(p + 16, nf - 1) * cs);
      return lop[(pstride_t)p * cs];
    }
  }
  __device__ __forceinline__ void lo_store(int p, float v) {
    if constexpr (DIR == DIR_X) lt.at(p) = v;
    else lop[(pstride_t)p * cs] = v;
  }
  // Compensated final update of cell p (CMP): c(p) = hi + lo advanced by
  // dtf (H(p+1) - H(p)) / dxb(p) and split back into hi + lo.  The difference of
  // the two FP32 face sums is formed exactly and 1/dxb carries ~48 bits, so
  // the cell's change times its volume is the two face sums it shares with
  // its neighbours to ~2^-47: the sweep conserves mass to ~1e-14 of the
  // transported mass, and the state carries ~48 bits.
  __device__ __forceinline__ float final_cmp(float chi, float clo, float hl, float hr, int p) {
#if F3D_CMP_EFT
    // In FP32 pair arithmetic (error-free transformations; every operation
    // explicitly rounded, none contracted):
    //   hr - hl = s + e exactly (Knuth's TwoSum),
    //   X = (s + e) (1/dxb as hi + lo), D = X (dtf as hi + lo), each to ~2^-47
    //   (Dekker's products by FMA),
    //   (chi + clo) + D summed with TwoSum and renormalised to hi + lo.
    const float s = __fsub_rn(hr, hl);
    const float sb = __fsub_rn(s, hr);
    const float e = __fadd_rn(__fsub_rn(hr, __fsub_rn(s, sb)), __fsub_rn(-hl, sb));
    const float2 rr = __ldg(r2 + p);
    const float x = __fmul_rn(s, rr.x);
    float xe = __fmaf_rn(s, rr.x, -x);
    xe = __fmaf_rn(s, rr.y, xe);
    xe = __fmaf_rn(e, rr.x, xe);
    const float d = __fmul_rn(x, dtf_hi);
    float de = __fmaf_rn(x, dtf_hi, -d);
    de = __fmaf_rn(x, dtf_lo, de);
    de = __fmaf_rn(xe, dtf_hi, de);
    const float t = __fadd_rn(chi, d);
    const float tb = __fsub_rn(t, chi);
    float te = __fadd_rn(__fsub_rn(chi, __fsub_rn(t, tb)), __fsub_rn(d, tb));
    te = __fadd_rn(te, __fadd_rn(clo, de));
    float nhi = __fadd_rn(t, te);
    float nlo = __fsub_rn(te, __fsub_rn(nhi, t));
#else
    const double dlt = ((double)hr - (double)hl) * ((double)dtf_hi + (double)dtf_lo) * __ldg(r64 + p);
    const double c64 = ((double)chi + (double)clo) + dlt;
    float nhi = __double2float_rn(c64);
    float nlo = __double2float_rn(c64 - (double)nhi);
#endif
    if constexpr (EPI) {  // the pair is exact in FP64; one split after both processes
      const double v = epi.apply(p, (double)nhi + (double)nlo);
      nhi = __double2float_rn(v);
      nlo = __double2float_rn(__dsub_rn(v, (double)nhi));
    }
    lo_store(p, nlo);
    return nhi;
  }

  // KT right-hand side with G = P - F per face; h = 0.5 phi(r) dc
  template <bool G>
  __device__ __forceinline__ void arrive(StageS<float>& s, int q, float a0, FaceV<float> fv, int p,
                                         float& rhs, float& flux) const {
    const float d0 = a0 - s.a1;
    const float h1 = half_phid<LIM>(s.d1, d0);
    if (!G || q >= 1) {
      const float u = fv.u;
      const float cl = s.a2 + s.h2;
      const float cr = s.a1 - h1;
#if F3D_FFORM == 1
      // fv.u holds 0.5 u: F = 0.5 u (cl + cr) - 0.5 |u| (cr - cl)
      const float F = fmaf(u, cl + cr, -fabsf(u) * (cr - cl));
#else
      // 0.5 u (cl + cr) - 0.5 |u| (cr - cl) in upwind form: u+ cl + u- cr
      const float F = fmaf(fmaxf(u, 0.f), cl, fminf(u, 0.f) * cr);
#endif
      flux = fmaf(fv.k, s.d1, F);        // F + P, the boundary flux
      const float G0 = fmaf(fv.k, s.d1, -F);  // P - F
      if (!G || q >= 2) rhs = (G0 - s.F1) * fv.r;  // fv is face q-1: r = 1/dxb(q-2)
      s.F1 = G0;
    }
    s.a2 = s.a1;
    s.a1 = a0;
    s.d1 = d0;
    s.h2 = h1;
  }
};

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

// One work item (32 pencils x bpb bins of one member) of a sweep; called by
// the per-sweep kernels and by the persistent fused step kernel.  EPI (z
// only): the wet deposition and decay epilogue, a kernel instance of its own
// so that the sweeps without it keep their register allocation.
template <int DIR, int LIM, int TM, bool CMP = false, bool EPI = false>
__device__ __forceinline__ void sweep32_item(const MemberDev* __restrict__ members,
                                             const WorkItem w, int bpb, unsigned char* f3d_smem) {
  const MemberDev& m = members[w.member];
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  const long long nsp = (DIR == DIR_X) ? (long long)ny * nz
                        : (DIR == DIR_Y) ? (long long)nx * nz : (long long)nx * ny;
  const int warp = threadIdx.x >> 5;
  const long long pen_raw = (long long)w.pen0 + 32 * (warp / bpb) + (threadIdx.x & 31);
  const long long pen0w = (long long)w.pen0 + 32 * (warp / bpb);
  const int b = w.bin0 + warp % bpb;
  const bool lane_ok = pen_raw < nsp && b < m.nb;
  const bool run_it = (DIR == DIR_X) ? (pen0w < nsp && b < m.nb) : lane_ok;
  const long long pen = pen_raw < nsp ? pen_raw : nsp - 1;
  double clo = 0.0, chi = 0.0;
  if (run_it) {
    Ops32<LIM, DIR, TM, CMP, EPI> o;
    double area;
    int n, i = 0, j = 0;
    if (DIR == DIR_X) {
      j = (int)(pen % ny);
      int k = (int)(pen / ny);
      n = nx;
      o.cp = m.c32 + (((long long)b * nz + k) * ny + j) * nx;
      constexpr int xbytes = decltype(o.xt)::BYTES + (CMP ? decltype(o.lt)::BYTES : 0);
      o.xt.setup(f3d_smem + warp * xbytes, lane_ok ? o.cp : nullptr, threadIdx.x & 31, nx);
      if constexpr (CMP) {
        o.lop = m.c32lo + (((long long)b * nz + k) * ny + j) * nx;
        o.r64 = m.rdxb64[0];
        o.r2 = m.rdxb2[0];
        o.lt.setup(f3d_smem + warp * xbytes + decltype(o.xt)::BYTES, o.xt.rows,
                   (long long)(m.c32lo - m.c32), threadIdx.x & 31, nx);
      }
      o.cs = 1;
      long long fo = (long long)k * (nx + 1) * ny + j;
      o.fd = (m.gc_cur ? m.gc4[0] : m.f4[0]) + fo;
      o.vs = ny;
      o.vsub = nullptr;
      area = m.dx3b[k + 1] * m.dx2b[j + 1];
    } else if (DIR == DIR_Y) {
      i = (int)(pen % nx);
      int k = (int)(pen / nx);
      n = ny;
      o.cp = m.c32 + ((long long)b * nz + k) * ny * (long long)nx + i;
      if constexpr (CMP) {
        o.lop = m.c32lo + ((long long)b * nz + k) * ny * (long long)nx + i;
        o.r64 = m.rdxb64[1];
        o.r2 = m.rdxb2[1];
      }
      o.cs = nx;
      long long fo = (long long)k * (ny + 1) * nx + i;
      o.fd = (m.gc_cur ? m.gc4[1] : m.f4[1]) + fo;
      o.vs = nx;
      o.vsub = nullptr;
      area = m.dx3b[k + 1] * m.dx1b[i + 1];
    } else {
      i = (int)(pen % nx);
      j = (int)(pen / nx);
      n = nz;
      o.cp = m.c32 + (long long)b * nz * ny * nx + (long long)j * nx + i;
      if constexpr (CMP) {
        o.lop = m.c32lo + (long long)b * nz * ny * nx + (long long)j * nx + i;
        o.r64 = m.rdxb64[2];
        o.r2 = m.rdxb2[2];
      }
      o.cs = (pstride_t)nx * ny;
      long long fo = (long long)j * nx + i;
      o.fd = m.f4[2] + fo;
      o.vs = (pstride_t)nx * ny;
      o.vsub = m.vs32 + (long long)b * (nz + 1) * ny * nx + fo;
      area = m.dx2b[j + 1] * m.dx1b[i + 1];
      if constexpr (EPI) o.epi = zepi_setup(m, b, fo);
    }
    const double dt = m.dt;
    o.s1 = (float)m.stime;
    o.s0 = 1.f - o.s1;
    o.wfac = m.wfac;
    if (DIR != DIR_Z && m.gc_cur) {  // this step's winds in both slots: u = fmaf(1, u, 0 * u)
      o.s0 = 1.f;
      o.s1 = 0.f;
      o.wfac = 1.f;
    }
#if F3D_FFORM == 1
    if (DIR == DIR_Z) {  // the face velocity enters as 0.5 u (exact scaling)
      o.s0 *= 0.5f;
      o.s1 *= 0.5f;
    } else {
      o.wfac *= 0.5f;
    }
#endif
    o.nf = n;
    o.dt = (float)dt;
    o.hdt = 0.5f * o.dt;
    o.dt3 = o.dt * (1.f / 3.f);
    o.dt6 = o.dt * (1.f / 6.f);
    if constexpr (CMP) {
      const double dtf = (TM == 2) ? dt / 6.0 : dt;
      o.dtf_hi = __double2float_rn(dtf);
      o.dtf_lo = __double2float_rn(dtf - (double)o.dtf_hi);
    }
    // the edge blocks run the unguarded body (cheaper than the guarded one)
    March<float, Ops32<LIM, DIR, TM, CMP, EPI>, TM, true, CMP> M(o, n);
    M.run();
    if (lane_ok) {
      clo = (double)M.flux_lo * area * dt;
      chi = (double)M.flux_hi * area * dt;
      if (m.gh32) {  // the free-flow ghosts of this pencil, kept for the output reductions
        float* g = m.gh32 + (long long)b * gh_per_bin(nx, ny, nz);
        g[gh_offset(DIR, 0, pen, nx, ny, nz)] = M.gL;
        g[gh_offset(DIR, 1, pen, nx, ny, nz)] = M.gR;
      }
    }
    if (DIR == DIR_Z) {
      double* a = m.acum + ((long long)b * ny + j) * nx + i;
      *a = *a + fabs((double)M.flux_lo) * dt;
      if constexpr (EPI) zepi_finish(m, o.epi, b, (long long)j * nx + i);
    }
  }
  block_reduce2_f64(clo, chi, m.flux_part + 2 * (long long)w.slot);
}

#ifndef F3D_CMP_BLOCKS
#define F3D_CMP_BLOCKS 4
#endif
#ifndef F3D_CMP_Y_BLOCKS
#define F3D_CMP_Y_BLOCKS 4
#endif
#ifndef F3D_CMP_YZ_BLOCKS
#define F3D_CMP_YZ_BLOCKS 4
#endif
template <int DIR, int LIM, int TM, bool CMP, bool EPI = false>
// 4 blocks of 128 threads per SM (128 registers); with one output buffer the
// RK4 x tiles (4 x 12.6 KB per block) fit 4 blocks as well.  The compensated
// x sweep runs 4 blocks too: at 128 registers it spills a few bytes, and it
// measured 13% faster than 3 blocks at 168 registers.
__global__ void __launch_bounds__(128, CMP ? (DIR == DIR_X ? F3D_CMP_BLOCKS
                                                          : (DIR == DIR_Y ? F3D_CMP_Y_BLOCKS : F3D_CMP_YZ_BLOCKS))
                                              : 4)
    k_sweep32(const MemberDev* __restrict__ members, const WorkItem* __restrict__ work, int bpb) {
  extern __shared__ __align__(16) unsigned char f3d_smem[];
  sweep32_item<DIR, LIM, TM, CMP, EPI>(members, work[blockIdx.x], bpb, f3d_smem);
}

template <int DIR, bool CMP, bool EPI = false>
static void launch_dir32(int lim, int tm, const MemberDev* members, const WorkItem* work,
                         int nblocks, int bpb, cudaStream_t st) {
  dim3 g(nblocks), b(128);
  // RK4 x tiles keep one output buffer (XTile<float, 1>), Euler two; the
  // compensated form stages the low part as well, in chunks of F3D_CMP_XW
  constexpr int cw = CMP ? F3D_CMP_XW : 32;
  constexpr int lob = CMP ? XLoTile<cw>::BYTES : 0;
  const int smem_max = (DIR == DIR_X) ? 4 * (XTile<float, 2, cw>::BYTES + lob) : 0;
  const int smem = (DIR == DIR_X)
                       ? 4 * (((tm == 2) ? XTile<float, 1, cw>::BYTES : XTile<float, 2, cw>::BYTES) + lob)
                       : 0;
  static bool attr_set = false;
  if (!attr_set && smem_max > 0) {
    cudaFuncSetAttribute(k_sweep32<DIR, 1, 1, CMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(k_sweep32<DIR, 2, 1, CMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(k_sweep32<DIR, 3, 1, CMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(k_sweep32<DIR, 1, 2, CMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(k_sweep32<DIR, 2, 2, CMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(k_sweep32<DIR, 3, 2, CMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    attr_set = true;
  }
#define F3D_L(L, T) k_sweep32<DIR, L, T, CMP, EPI><<<g, b, smem, st>>>(members, work, bpb)
  if (tm == 1) {
    if (lim == 1) F3D_L(1, 1); else if (lim == 2) F3D_L(2, 1); else F3D_L(3, 1);
  } else {
    if (lim == 1) F3D_L(1, 2); else if (lim == 2) F3D_L(2, 2); else F3D_L(3, 2);
  }
#undef F3D_L
}

// epi: the z sweep runs the wet deposition and decay epilogue (the members'
// epi_on)
void launch_sweep32(int dir, int lim, int tm, int cmp, int epi, const MemberDev* members,
                    const WorkItem* work, int nblocks, int bpb, cudaStream_t st) {
  if (nblocks <= 0) return;
  if (cmp) {
    if (dir == DIR_X) launch_dir32<DIR_X, true>(lim, tm, members, work, nblocks, bpb, st);
    else if (dir == DIR_Y) launch_dir32<DIR_Y, true>(lim, tm, members, work, nblocks, bpb, st);
    else if (epi) launch_dir32<DIR_Z, true, true>(lim, tm, members, work, nblocks, bpb, st);
    else launch_dir32<DIR_Z, true>(lim, tm, members, work, nblocks, bpb, st);
  } else {
    if (dir == DIR_X) launch_dir32<DIR_X, false>(lim, tm, members, work, nblocks, bpb, st);
    else if (dir == DIR_Y) launch_dir32<DIR_Y, false>(lim, tm, members, work, nblocks, bpb, st);
    else if (epi) launch_dir32<DIR_Z, false, true>(lim, tm, members, work, nblocks, bpb, st);
    else launch_dir32<DIR_Z, false>(lim, tm, members, work, nblocks, bpb, st);
  }
}

void launch_prep32(const MemberDev* members, const int* blk_member, const int* blk_first,
                   int nblocks, int mask, cudaStream_t st) {
  // the precision form interpolates the winds inside the sweeps
  (void)members; (void)blk_member; (void)blk_first; (void)nblocks; (void)mask; (void)st;
}

__global__ void k_source32(const MemberDev* __restrict__ members, int nmembers) {
  for (int mi = blockIdx.y; mi < nmembers; mi += gridDim.y) {
    const MemberDev& m = members[mi];
    const long long tot = (long long)m.nsrc * m.nb;
    const long long ncell = (long long)m.nx * m.ny * m.nz;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
      int q = (int)(e / m.nb), b = (int)(e % m.nb);
      const long long at = (long long)b * ncell + m.src_cell[q];
      add_to_state32(m, at, m.dt * m.src_s[(long long)q * m.nb + b] / m.src_vol[q]);
    }
  }
}

void launch_source32(const MemberDev* members, int nmembers, cudaStream_t st) {
  dim3 g(8, nmembers < 65535 ? nmembers : 65535);
  k_source32<<<g, 128, 0, st>>>(members, nmembers);
}

// FP32 field preparation from the FP64 meteo arrays (once per meteo update):
// the face data {u(its), u(ite), kf, 1/dxb(f-1)} of each direction with
//   kf(f) = 0.5 (k(f) + k(f-1)) / dxp(f-1)         (KT_RHS P term, :1111)
// and the settling velocity.
__global__ void k_fp32_fields(MemberDev* members, int mi) {
  MemberDev& m = members[mi];
  const int nx = m.nx, ny = m.ny, nz = m.nz, nb = m.nb;
  const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)(ny + 1) * nx * nz,
                  nw = (long long)(nz + 1) * nx * ny;
  const long long nvs = (long long)nb * nw;
  const long long tot = nu + nv + nw + nvs;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long q = e;
    if (q < nu) {  // x faces: [k][f][j]
      int j = (int)(q % ny);
      long long t = q / ny;
      int f = (int)(t % (nx + 1));
      int k = (int)(t / (nx + 1));
      double kA = m.k1x[((long long)k * (nx + 2) + (f + 1)) * ny + j];
      double kB = m.k1x[((long long)k * (nx + 2) + f) * ny + j];
      const_cast<float4*>(m.f4[0])[q] =
          make_float4((float)m.ux[0][q], (float)m.ux[1][q], (float)(0.5 * (kA + kB) / m.dx1p[f + 1]),
                      f >= 1 ? m.rdx1b32[f - 1] : 0.f);
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
      const_cast<float4*>(m.f4[1])[q] =
          make_float4((float)m.vy[0][q], (float)m.vy[1][q], (float)(0.5 * (kA + kB) / m.dx2p[f + 1]),
                      f >= 1 ? m.rdx2b32[f - 1] : 0.f);
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
      const_cast<float4*>(m.f4[2])[q] =
          make_float4((float)m.wz[0][q], (float)m.wz[1][q], (float)(0.5 * (kA + kB) / m.dx3p[f + 1]),
                      f >= 1 ? m.rdx3b32[f - 1] : 0.f);
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

namespace f3d {

// Source term of every member, grid-stride over (member, cell, bin).
__device__ __forceinline__ void source32_all(MemberDev* members, int nmembers) {
  for (int mi = 0; mi < nmembers; ++mi) {
    const MemberDev& m = members[mi];
    const long long tot = (long long)m.nsrc * m.nb;
    const long long ncell = (long long)m.nx * m.ny * m.nz;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
      int q = (int)(e / m.nb), b = (int)(e % m.nb);
      const long long at = (long long)b * ncell + m.src_cell[q];
      add_to_state32(m, at, m.dt * m.src_s[(long long)q * m.nb + b] / m.src_vol[q]);
    }
  }
}

// Out-of-line sweep items for the persistent kernel: each direction keeps its
// own register allocation instead of one inlined union of all three.
template <int DIR, int LIM, int TM, bool CMP, bool EPI = false>
__device__ __noinline__ void sweep32_item_call(MemberDev* members, WorkItem w, int bpb,
                                               unsigned char* smem) {
  sweep32_item<DIR, LIM, TM, CMP, EPI>(members, w, bpb, smem);
}

// One whole time step of every member in one persistent kernel: source,
// the two horizontal sweeps (order by iiter parity, mod_F3D.F90:1477-1487),
// the z sweep, boundary-flux reduction and the device clock.  Blocks pull
// work items from per-phase atomic counters (members of uneven size balance
// themselves) and meet at bounded grid barriers between phases.  Launched
// cooperatively so that every block is resident.
template <int LIM, int TM, bool CMP>
#ifndef F3D_FUSED32_BLOCKS
#define F3D_FUSED32_BLOCKS 3
#endif
__global__ void __launch_bounds__(128, F3D_FUSED32_BLOCKS) k_fused32(FusedArgs a) {
  extern __shared__ __align__(16) unsigned char f3d_smem[];
  __shared__ int slot;
  __shared__ double sa[128], sb[128];
  source32_all(a.members, a.nmembers);
  grid_barrier(a.counters + 6, a.err, a.wait_limit);
  const bool xfirst = (a.members[0].iiter % 2) == 0;
  for (int ph = 0; ph < 3; ++ph) {
    const int dir = (ph == 2) ? 2 : (((ph == 0) == xfirst) ? 0 : 1);
    for (;;) {
      const int it = grab_item(a.counters + ph, &slot);
      if (it >= a.nwork[dir]) break;
      const WorkItem w = a.work[dir][it];
      if (dir == 0) sweep32_item_call<0, LIM, TM, CMP>(a.members, w, a.bpb, f3d_smem);
      else if (dir == 1) sweep32_item_call<1, LIM, TM, CMP>(a.members, w, a.bpb, f3d_smem);
      else if (a.epi) sweep32_item_call<2, LIM, TM, CMP, true>(a.members, w, a.bpb, f3d_smem);
      else sweep32_item_call<2, LIM, TM, CMP>(a.members, w, a.bpb, f3d_smem);
    }
    grid_barrier(a.counters + 6, a.err, a.wait_limit);
  }
  for (int mi = blockIdx.x; mi < a.nmembers; mi += gridDim.x) {
    member_flux_reduce(a.members[mi], 7, sa, sb);
    if (threadIdx.x == 0) member_advance(a.members[mi]);
    __syncthreads();
  }
}

// Dynamic shared memory of the persistent kernel: the x sweep's staging of
// this time marching and form, for the 4 warps of a block.
int fused32_smem(int tm, int cmp) {
  if (cmp)
    return 4 * ((tm == 2 ? XTile<float, 1, F3D_CMP_XW>::BYTES : XTile<float, 2, F3D_CMP_XW>::BYTES) +
                XLoTile<F3D_CMP_XW>::BYTES);
  return 4 * (tm == 2 ? XTile<float, 1>::BYTES : XTile<float, 2>::BYTES);
}

template <bool CMP>
static const void* fused32_func_t(int lim, int tm) {
  if (tm == 1) {
    if (lim == 1) return (const void*)k_fused32<1, 1, CMP>;
    if (lim == 2) return (const void*)k_fused32<2, 1, CMP>;
    return (const void*)k_fused32<3, 1, CMP>;
  }
  if (lim == 1) return (const void*)k_fused32<1, 2, CMP>;
  if (lim == 2) return (const void*)k_fused32<2, 2, CMP>;
  return (const void*)k_fused32<3, 2, CMP>;
}

const void* fused32_func(int lim, int tm, int cmp) {
  return cmp ? fused32_func_t<true>(lim, tm) : fused32_func_t<false>(lim, tm);
}

}  // namespace f3d
