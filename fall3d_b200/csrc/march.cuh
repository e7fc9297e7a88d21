// march.cuh -- the pipelined single-pass RK pencil march shared by the FP64
// and FP32 sweep kernels.
//
// One thread owns one pencil of one bin.  KT_RHS at cell i reads cells
// i-2..i+2 (mod_ADS.F90:1057-1120), so RK stage s can run two cells behind
// stage s-1: at march time t, stage s receives its input at q = t - 2(s-1)
// and emits its right-hand side at q - 2.  The pencil is read once and
// written once; the stage inputs the reference keeps in whole-pencil arrays
// (c0, new_c, ini_c) live in registers.
//
// The march runs in blocks of 8 time steps with compile-time ring indices,
// so the per-position histories (input c, new_c accumulator, face data)
// rotate by register renaming.  Blocks entirely inside the steady range
// [8, n-2] (every stage interior) run without edge guards.
#pragma once
#ifndef F3D_COMMON_SKIP
#include "f3d_common.cuh"
#endif

// F3D_HALF_TAIL: the last block of the RK4 V march skips its second half
// when t = n + 7 falls in the first (on in the precision form's sweeps).
#ifndef F3D_HALF_TAIL
#define F3D_HALF_TAIL 0
#endif

namespace f3d {

template <class T>
struct FaceV {
  T u;  // face-normal velocity (z: w - vs of the bin)
  T k;  // diffusion at the face (FP64: 0.5 (k_f + k_f-1); FP32: that / dxp)
  T r;  // FP32 form: 1/dxb of cell f-1, so that the face ring carries it to
        // every stage (stage s at q receives face q-1 and needs cell q-2)
};

// Asynchronous global -> shared copy of one element (cp.async, Ampere and
// later): no register round trip, so the warp keeps computing while the copy
// is in flight.  src_bytes < sizeof(T) zero-fills the destination.
template <class T>
__device__ __forceinline__ void cp_async_elem(T* dst_smem, const T* src, int src_bytes) {
  const unsigned int d = (unsigned int)__cvta_generic_to_shared(dst_smem);
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Per-warp shared-memory staging of x pencils.  The 32 lanes of a warp own
// 32 rows of the x-contiguous concentration; lanes read their own row from a
// transposed tile while the warp moves whole 128-byte row segments between
// HBM and the tile (coalesced).  Input chunks are double-buffered, copied
// with cp.async a chunk ahead and waited for only by the first block that
// reads them, so their latency overlaps W - 8 positions of work.  Output
// chunks are double-buffered (NOUT = 2, any time marching) or, for RK4, held
// in one buffer (NOUT = 1): RK4 writes position p at t = p + 8, so chunk m
// is complete at t = (m+1)W + 7 and chunk m+1's first write comes at
// t = (m+1)W + 8, the block that flushes chunk m before writing.  The
// smaller tile lets more blocks share an SM.
template <class T, int NOUT = 2, int W_ = 128 / (int)sizeof(T)>
struct XTile {
  static constexpr int W = W_;                    // positions per chunk (a multiple of 8)
  static constexpr int LDW = W + 1;               // padded row pitch
  static constexpr int RPI = 32 / W;              // rows per warp instruction
  static constexpr int BYTES = (2 + NOUT) * 32 * LDW * (int)sizeof(T) + 32 * 8;
  T* in;            // [2][32][LDW]
  T* out;           // [NOUT][32][LDW]
  T* const* rows;   // [32] row base pointers, null for lanes without a pencil
  const T* any;     // a valid row of the warp (source address of zero-filled copies)
  int lane, n, next_flush;

  __device__ __forceinline__ void setup(void* base, T* my_row, int lane_, int n_) {
    in = reinterpret_cast<T*>(base);
    out = in + 2 * 32 * LDW;
    T** r = reinterpret_cast<T**>(out + NOUT * 32 * LDW);
    r[lane_] = my_row;
    rows = r;
    lane = lane_;
    n = n_;
    next_flush = 0;
    const unsigned int have = __ballot_sync(0xffffffffu, my_row != nullptr);
    any = have ? reinterpret_cast<const T*>(__shfl_sync(
                     0xffffffffu, reinterpret_cast<unsigned long long>(my_row), __ffs(have) - 1))
               : nullptr;
    __syncwarp();
  }
  // issue the copies of chunk m (one commit group); rows without a pencil and
  // positions past the end are zero-filled
  __device__ __forceinline__ void load_chunk(int m) {
    if (!any) return;
    const int p0 = m * W, sub = lane / W, col = lane % W;
    T* dst = in + (m & 1) * 32 * LDW;
#pragma unroll 8
    for (int r0 = 0; r0 < 32; r0 += RPI) {
      const int r = r0 + sub, p = p0 + col;
      const T* rp = rows[r];
      const bool ok = rp && p < n;
      cp_async_elem(dst + r * LDW + col, ok ? rp + p : any, ok ? (int)sizeof(T) : 0);
    }
    cp_async_commit();
  }
  __device__ __forceinline__ void flush_chunk(int m) {
    const int p0 = m * W, sub = lane / W, col = lane % W;
    const T* src = out + (NOUT == 2 ? (m & 1) : 0) * 32 * LDW;
#pragma unroll 8
    for (int r0 = 0; r0 < 32; r0 += RPI) {
      const int r = r0 + sub, p = p0 + col;
      T* rp = rows[r];
      if (rp && p < n) rp[p] = src[r * LDW + col];
    }
  }
  __device__ __forceinline__ T load(int p) const {
    return in[((p / W) & 1) * 32 * LDW + lane * LDW + (p % W)];
  }
  __device__ __forceinline__ void store(int p, T v) const {
    out[(NOUT == 2 ? ((p / W) & 1) : 0) * 32 * LDW + lane * LDW + (p % W)] = v;
  }
  // hooks driven by the march (warp-uniform)
  __device__ __forceinline__ void init() {
    load_chunk(0);
    cp_async_wait_all();
    __syncwarp();
  }
  __device__ __forceinline__ void block_begin(int T0) {
    // Block T0 reads positions T0+2 .. T0+9 (the march loads c(t+2) at time
    // t).  At T0 = mW every lane is past chunk m-1, so chunk m+1 is copied
    // into its buffer; chunk m+1 is first read by block T0 = (m+1)W - 8,
    // which waits for the copies.
    __syncwarp();
    if (NOUT == 1 && T0 - 8 >= W && (T0 - 8) % W == 0) {
      // single output buffer: chunk (T0-8)/W - 1 is complete, flush it
      // before this block writes the next chunk over it
      flush_chunk((T0 - 8) / W - 1);
      next_flush = (T0 - 8) / W;
      __syncwarp();
    }
    if (T0 >= 0 && T0 % W == 0 && (T0 / W + 1) * W < n) load_chunk(T0 / W + 1);
    if (T0 + 8 >= W && (T0 + 8) % W == 0) cp_async_wait_all();
    __syncwarp();
  }
  __device__ __forceinline__ void block_end(int T0) {
    // chunk m is complete after block (m+1)W and its buffer is rewritten from
    // block (m+2)W on (RK4 writes position p at t = p+8, Euler at t = p+2)
    if (NOUT == 2 && T0 >= W && T0 % W == 0) {
      __syncwarp();
      flush_chunk(T0 / W - 1);
      next_flush = T0 / W;
    }
  }
  __device__ __forceinline__ void finish() {
    cp_async_wait_all();
    __syncwarp();
    for (int m = next_flush; m * W < n; ++m) flush_chunk(m);
  }
};

// Per-warp staging of the low part of the compensated state along x pencils:
// the cells are finalised in place in a two-buffer tile.  With the RK4 march
// the low part of cell p is read at t = p + 7 and written at t = p + 8, so
// chunk m (positions mW .. mW + W - 1) is complete after block T0 = (m+1)W,
// which flushes it and issues the copy of chunk m + 2 into the same buffer;
// that chunk is first read by block T0 = (m+2)W, which waits for it.  The
// rows are those of the state's staging (XTile::rows) shifted by `delta`
// elements (the low part's offset from the state).
template <int W>
struct XLoTile {
  static constexpr int LDW = W + 1;
  static constexpr int BYTES = 2 * 32 * LDW * 4;
  float* buf;            // [2][32][LDW]
  float* const* rows;    // the state's row base pointers
  long long delta;
  int lane, n, next_flush;

  __device__ __forceinline__ void setup(void* base, float* const* rows_, long long delta_, int lane_,
                                        int n_) {
    buf = reinterpret_cast<float*>(base);
    rows = rows_;
    delta = delta_;
    lane = lane_;
    n = n_;
    next_flush = 0;
  }
  __device__ __forceinline__ void load_chunk(int m) {
    const int p0 = m * W, sub = lane / W, col = lane % W;
    float* dst = buf + (m & 1) * 32 * LDW;
    const float* any = nullptr;
    for (int r = 0; r < 32 && !any; ++r)
      if (rows[r]) any = rows[r] + delta;
    if (!any) return;
#pragma unroll 8
    for (int r0 = 0; r0 < 32; r0 += 32 / W) {
      const int r = r0 + sub, p = p0 + col;
      const float* rp = rows[r];
      const bool ok = rp && p < n;
      cp_async_elem(dst + r * LDW + col, ok ? rp + delta + p : any, ok ? 4 : 0);
    }
    cp_async_commit();
  }
  __device__ __forceinline__ void flush_chunk(int m) {
    const int p0 = m * W, sub = lane / W, col = lane % W;
    const float* src = buf + (m & 1) * 32 * LDW;
#pragma unroll 8
    for (int r0 = 0; r0 < 32; r0 += 32 / W) {
      const int r = r0 + sub, p = p0 + col;
      float* rp = rows[r];
      if (rp && p < n) rp[delta + p] = src[r * LDW + col];
    }
  }
  __device__ __forceinline__ float& at(int p) {
    return buf[((p / W) & 1) * 32 * LDW + lane * LDW + (p % W)];
  }
  __device__ __forceinline__ void init() {
    load_chunk(0);
    if (W < n) load_chunk(1);
    cp_async_wait_all();
    __syncwarp();
  }
  __device__ __forceinline__ void block_begin(int T0) {
    if (T0 >= 2 * W && T0 % W == 0) {  // chunk T0/W, issued after block T0 - W
      cp_async_wait_all();
      __syncwarp();
    }
  }
  __device__ __forceinline__ void block_end(int T0) {
    if (T0 >= W && T0 % W == 0) {
      __syncwarp();
      flush_chunk(T0 / W - 1);
      next_flush = T0 / W;
      __syncwarp();
      if ((T0 / W + 1) * W < n) load_chunk(T0 / W + 1);
    }
  }
  __device__ __forceinline__ void finish() {
    cp_async_wait_all();
    __syncwarp();
    for (int m = next_flush; m * W < n; ++m) flush_chunk(m);
  }
};

// Default (no staging) hooks for y and z pencils.
struct NoStage {
  __device__ __forceinline__ void init() {}
  __device__ __forceinline__ void block_begin(int) {}
  __device__ __forceinline__ void block_end(int) {}
  __device__ __forceinline__ void finish() {}
};

template <class T>
struct StageS {
  T a1, a2, d1, h2, F1, P1;  // a(q-1), a(q-2), a(q-1)-a(q-2), limiter at q-2, fluxes at face q-2
};

// Pipeline over a pencil.  Ops supplies (all __device__ __forceinline__):
//   T    load_c(int p)                     concentration at pencil position p
//   T    load_last()                       c(n-1) from memory, before any staging (V)
//   void store_c(int p, T v)
//   FaceV<T> face(int f)                   face data, f in [0, n]
//   T    arrive<G>(StageS&, int q, T a0, FaceV<T> fv, int p, T& rhs, T& flux)
//        -> returns nothing; sets rhs (valid when q >= 2) and flux (face q-1)
//   T    ghost_l(T c0, T uL) / ghost_r(T cn, T uR)  free-flow ghost values
//   rk:  a2 = c + hdt k, new = c + dt6 k, ... provided as methods
//
// V (RK4 only): the edge blocks run an unguarded body instead of the guarded
// one.  Positions outside the pencil arrive as the ghost values (gR is formed
// in the prologue from c(n-1)), and faces outside [1, n] carry 1/dxb = 0
// (Ops::face_v), so the right-hand side of a ghost cell is exactly 0 and its
// stage values stay the ghost value (c + h*0 = c), as the guarded body keeps
// them.  Stores are predicated on the position, the boundary fluxes captured
// by select.  The march starts at t = 0 (see run_v).  This body costs about
// 1.4 steady steps per step against 2.1 for the guarded one, and the edge
// blocks are a third to half of the march on short (z) pencils.
//
// CMP (precision form with a compensated state): instead of accumulating
// new_c per cell, the march accumulates per FACE the RK-weighted sum of the
// stage fluxes, H(f) = G1 + 2 G2 + 2 G3 + G4 (Euler: G1), in hf[f & 7], and
// the final update of cell p is Ops::final_cmp(c(p), H(p), H(p+1), p).  A face
// sum is shared by the two cells it separates, so the mass one cell loses is
// exactly the mass its neighbour gains.  c(p) for that update is taken from
// the input ring at the start of step t = p + 8, before stage 1 overwrites
// its slot; nh is not used.
template <class T, class Ops, int TM, bool V = false, bool CMP = false>
struct March {
  Ops& o;
  const int n;
  T ch[8];           // c(p) at ch[p & 7]
  T nh[8];           // new_c(p) at nh[p & 7] (not used by CMP)
  T hf[8];           // CMP: H(f) at hf[f & 7]
  T lo_next;         // CMP, RK4: the low part of the next cell to finalise,
                     // loaded one step ahead of its use
  FaceV<T> fw[8];    // face(f) at fw[f & 7]
  StageS<T> S1, S2, S3, S4;
  T gL, gR, uR, cn1, cn2, cn3, cn4;
  FaceV<T> fq;       // face(t+1), loaded one step ahead
  T flux_lo, flux_hi;

  __device__ __forceinline__ March(Ops& ops, int n_) : o(ops), n(n_) {}

  template <int U, bool G>
  __device__ __forceinline__ void iter(int t) {
    constexpr int m1 = (U + 7) & 7, m2 = (U + 6) & 7, m3 = (U + 5) & 7, m4 = (U + 4) & 7,
                  m5 = (U + 3) & 7, m6 = (U + 2) & 7, m7 = (U + 1) & 7;
    T k1 = T(0), k2 = T(0), k3 = T(0), k4 = T(0), ff = T(0);
    const T c_fin = ch[U];  // CMP: c(t-8), finalised at the end of this step
    T lo_fin = T(0);
    if constexpr (CMP && TM == 2) {  // its low part, and the next one's load
      lo_fin = lo_next;
      lo_next = o.lo_fetch(min(max(t - 7, 0), n - 1));
    }
    // ---- stage 1: arrival at q = t
    // c(p) is loaded at t = p - 4 and face(f) at t = f - 1 (a four-slot and
    // a one-slot queue in front of the rings), so their latency is hidden
    // behind the work of the intervening positions.
    if (!G || (t >= -2 && t <= n + 1)) {
      T a;
      if (G) {
        a = (t < 0) ? gL : ((t < n) ? cn1 : gR);
        cn1 = cn2;
        cn2 = cn3;
        cn3 = cn4;
        if (t + 4 >= 0 && t + 4 < n) cn4 = o.load_c(t + 4);
        if (t == n - 1) gR = o.ghost_r(a, uR);
        if (t >= 0 && t <= n) fw[U] = fq;
        if (t + 1 >= 0 && t + 1 <= n) fq = o.face(t + 1);
      } else {
        a = cn1;
        cn1 = cn2;
        cn2 = cn3;
        cn3 = cn4;
        cn4 = o.load_c(min(t + 4, n - 1));
        fw[U] = fq;
        fq = o.face(t + 1);
      }
      ch[U] = a;
      o.template arrive<G>(S1, t, a, fw[m1], t - 2, k1, ff);
      if constexpr (CMP) hf[m1] = S1.F1;
    }
    if constexpr (TM == 1) {
      if (!G || (t >= 2 && t <= n + 1)) {
        if constexpr (CMP)
          o.store_c(t - 2, o.final_cmp(ch[m2], o.lo_fetch(t - 2), hf[m2], hf[m1], t - 2));
        else o.store_c(t - 2, o.euler(ch[m2], k1));
      }
      if (G && t == 1) flux_lo = ff;
      if (G && t == n + 1) flux_hi = ff;
      return;
    } else {
    // ---- stage 2: q = t-2
    {
      const int q = t - 2;
      if (!G || (q >= -2 && q <= n + 1)) {
        T a;
        if (G && q < 0) a = gL;
        else if (G && q >= n) a = gR;
        else {
          a = o.rk_half(ch[m2], k1);
          if constexpr (!CMP) nh[m2] = o.rk_new1(ch[m2], k1);
        }
        o.template arrive<G>(S2, q, a, fw[m3], q - 2, k2, ff);
        if constexpr (CMP) hf[m3] = fmaf(T(2), S2.F1, hf[m3]);
      }
    }
    // ---- stage 3: q = t-4
    {
      const int q = t - 4;
      if (!G || (q >= -2 && q <= n + 1)) {
        T a;
        if (G && q < 0) a = gL;
        else if (G && q >= n) a = gR;
        else {
          a = o.rk_half(ch[m4], k2);
          if constexpr (!CMP) nh[m4] = o.rk_add3(nh[m4], k2);
        }
        o.template arrive<G>(S3, q, a, fw[m5], q - 2, k3, ff);
        if constexpr (CMP) hf[m5] = fmaf(T(2), S3.F1, hf[m5]);
      }
    }
    // ---- stage 4: q = t-6, output at t-8
    {
      const int q = t - 6;
      if (!G || (q >= -2 && q <= n + 1)) {
        T a;
        if (G && q < 0) a = gL;
        else if (G && q >= n) a = gR;
        else {
          a = o.rk_full(ch[m6], k3);
          if constexpr (!CMP) nh[m6] = o.rk_add3(nh[m6], k3);
        }
        o.template arrive<G>(S4, q, a, fw[m7], q - 2, k4, ff);
        if constexpr (CMP) {
          hf[m7] = hf[m7] + S4.F1;
          if (!G || (q >= 2)) o.store_c(q - 2, o.final_cmp(c_fin, lo_fin, hf[U], hf[m7], q - 2));
        } else {
          if (!G || (q >= 2)) o.store_c(q - 2, o.rk_final(nh[U], k4));
        }
        if (G && q == 1) flux_lo = ff;
        if (G && q == n + 1) flux_hi = ff;
      }
    }
    }
  }

  // one step of the V march (RK4); the steps of the last block past
  // t = n + 7 run on ghosts and store nothing (cheaper than a branch per step)
  template <int U>
  __device__ __forceinline__ void iter_v(int t) {
    constexpr int m1 = (U + 7) & 7, m2 = (U + 6) & 7, m3 = (U + 5) & 7, m4 = (U + 4) & 7,
                  m5 = (U + 3) & 7, m6 = (U + 2) & 7, m7 = (U + 1) & 7;
    T k1, k2, k3, k4, ff;
    const T c_fin = ch[U];  // CMP: c(t-8), finalised at the end of this step
    T lo_fin = T(0);
    if constexpr (CMP) {  // its low part, and the next one's load
      lo_fin = lo_next;
      lo_next = o.lo_fetch(min(max(t - 7, 0), n - 1));
    }
    {  // stage 1: q = t; c(p) enters the queue at t = p - 4 (positions past
       // the end loaded by a steady block hold c(n-1): arrive as gR)
      const T a = (t < n) ? cn1 : gR;
      cn1 = cn2;
      cn2 = cn3;
      cn3 = cn4;
      const int p = t + 4;
      const T c = o.load_c(min(max(p, 0), n - 1));
      cn4 = (p < 0) ? gL : ((p < n) ? c : gR);
      fw[U] = fq;
      fq = o.face_v(t + 1);
      ch[U] = a;
      o.template arrive<false>(S1, t, a, fw[m1], t - 2, k1, ff);
      if constexpr (CMP) hf[m1] = S1.F1;
    }
    {  // stage 2: q = t-2
      const T a = o.rk_half(ch[m2], k1);
      if constexpr (!CMP) nh[m2] = o.rk_new1(ch[m2], k1);
      o.template arrive<false>(S2, t - 2, a, fw[m3], t - 4, k2, ff);
      if constexpr (CMP) hf[m3] = fmaf(T(2), S2.F1, hf[m3]);
    }
    {  // stage 3: q = t-4
      const T a = o.rk_half(ch[m4], k2);
      if constexpr (!CMP) nh[m4] = o.rk_add3(nh[m4], k2);
      o.template arrive<false>(S3, t - 4, a, fw[m5], t - 6, k3, ff);
      if constexpr (CMP) hf[m5] = fmaf(T(2), S3.F1, hf[m5]);
    }
    {  // stage 4: q = t-6, output at t-8; ff is the flux at face q-1
      const int q = t - 6;
      const T a = o.rk_full(ch[m6], k3);
      if constexpr (!CMP) nh[m6] = o.rk_add3(nh[m6], k3);
      o.template arrive<false>(S4, q, a, fw[m7], q - 2, k4, ff);
      if constexpr (CMP) {
        hf[m7] = hf[m7] + S4.F1;
        if (q - 2 >= 0 && q - 2 < n) o.store_c(q - 2, o.final_cmp(c_fin, lo_fin, hf[U], hf[m7], q - 2));
      } else {
        if (q - 2 >= 0 && q - 2 < n) o.store_c(q - 2, o.rk_final(nh[U], k4));
      }
      flux_lo = (q == 1) ? ff : flux_lo;
      flux_hi = (q == n + 1) ? ff : flux_hi;
    }
  }

  // The first block (t = 0..7, known at compile time): a stage's arrivals at
  // q <= -1 only shape ghost right-hand sides (x 1/dxb = 0), so each stage
  // starts at its arrival q = 0 (t = 2(s-1)) from the state the ghosts leave
  // (a1 = a2 = gL, d1 = 0); nothing is stored before t = 8.
  template <int U>
  __device__ __forceinline__ void iter_head() {
    constexpr int t = U;
    constexpr int m1 = (U + 7) & 7, m2 = (U + 6) & 7, m3 = (U + 5) & 7, m4 = (U + 4) & 7,
                  m5 = (U + 3) & 7, m6 = (U + 2) & 7, m7 = (U + 1) & 7;
    T k1, k2, k3, k4, ff;
    {
      const T a = cn1;
      cn1 = cn2;
      cn2 = cn3;
      cn3 = cn4;
      const int p = t + 4;
      const T c = o.load_c(min(p, n - 1));
      cn4 = (p < n) ? c : gR;
      fw[U] = fq;
      fq = o.face_v(t + 1);
      ch[U] = (t < n) ? a : gR;
      o.template arrive<false>(S1, t, ch[U], fw[m1], t - 2, k1, ff);
      if constexpr (CMP) hf[m1] = S1.F1;
    }
    if constexpr (t >= 2) {
      const T a = o.rk_half(ch[m2], k1);
      if constexpr (!CMP) nh[m2] = o.rk_new1(ch[m2], k1);
      o.template arrive<false>(S2, t - 2, a, fw[m3], t - 4, k2, ff);
      if constexpr (CMP) hf[m3] = fmaf(T(2), S2.F1, hf[m3]);
    }
    if constexpr (t >= 4) {
      const T a = o.rk_half(ch[m4], k2);
      if constexpr (!CMP) nh[m4] = o.rk_add3(nh[m4], k2);
      o.template arrive<false>(S3, t - 4, a, fw[m5], t - 6, k3, ff);
      if constexpr (CMP) hf[m5] = fmaf(T(2), S3.F1, hf[m5]);
    }
    if constexpr (t >= 6) {
      const T a = o.rk_full(ch[m6], k3);
      if constexpr (!CMP) nh[m6] = o.rk_add3(nh[m6], k3);
      o.template arrive<false>(S4, t - 6, a, fw[m7], t - 8, k4, ff);
      if constexpr (CMP) hf[m7] = hf[m7] + S4.F1;
      if constexpr (t == 7) flux_lo = ff;  // face 0 of the last stage
    }
  }

  // The march starts at t = 0 in the state the steps t < 0 would leave: every
  // position below 0 has arrived in every stage as gL (a ghost's right-hand
  // side is 0), the faces below 0 carry 1/dxb = 0, and the queue holds
  // positions 0..3.  The limiter and flux values of those steps feed only
  // ghost right-hand sides, which are multiplied by 1/dxb = 0.
  __device__ __forceinline__ void run_v() {
    o.stage_init();
    const T c0 = o.load_c(0);
    gL = o.ghost_l(c0, o.face(0).u);
    uR = o.face(n).u;
    gR = o.ghost_r(o.load_last(), uR);
    cn1 = c0;
    cn2 = (n > 1) ? o.load_c(1) : gR;
    cn3 = (n > 2) ? o.load_c(2) : gR;
    cn4 = (n > 3) ? o.load_c(3) : gR;
    const FaceV<T> fm = o.face_v(-1);  // face 0's data with 1/dxb = 0
    fq = o.face_v(0);
    flux_lo = flux_hi = T(0);
    S1 = StageS<T>{gL, gL, T(0), T(0), T(0), T(0)};
    S2 = S1;
    S3 = S1;
    S4 = S1;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      ch[u] = gL;
      nh[u] = gL;
      fw[u] = fm;
      if constexpr (CMP) hf[u] = T(0);
    }
    const int t_last = n + 7;
    o.stage_begin(0);
    iter_head<0>();
    iter_head<1>();
    iter_head<2>();
    iter_head<3>();
    iter_head<4>();
    iter_head<5>();
    iter_head<6>();
    iter_head<7>();
    if constexpr (CMP) lo_next = o.lo_fetch(0);  // cell 0 is finalised at t = 8
    o.stage_end(0);
#pragma unroll 1
    for (int T0 = 8; T0 <= t_last; T0 += 8) {
      o.stage_begin(T0);
      if (T0 + 7 <= n - 2) {
        block8<false>(T0);  // interior: the steady body
      } else {
        iter_v<0>(T0);
        iter_v<1>(T0 + 1);
        iter_v<2>(T0 + 2);
        iter_v<3>(T0 + 3);
        // the last block stops at t_last when that is in its first half
        // (steps past t_last store nothing; n is warp-uniform)
        if (!F3D_HALF_TAIL || T0 + 4 <= t_last) {
          iter_v<4>(T0 + 4);
          iter_v<5>(T0 + 5);
          iter_v<6>(T0 + 6);
          iter_v<7>(T0 + 7);
        }
      }
      o.stage_end(T0);
    }
    o.stage_finish();
  }

  template <bool G>
  __device__ __forceinline__ void block8(int T0) {
    iter<0, G>(T0);
    iter<1, G>(T0 + 1);
    iter<2, G>(T0 + 2);
    iter<3, G>(T0 + 3);
    iter<4, G>(T0 + 4);
    iter<5, G>(T0 + 5);
    iter<6, G>(T0 + 6);
    iter<7, G>(T0 + 7);
  }

  __device__ __forceinline__ void run() {
    if constexpr (V && TM == 2) {
      run_v();
      return;
    }
    o.stage_init();
    T c0 = o.load_c(0);
    T uL = o.face(0).u;
    uR = o.face(n).u;
    gL = o.ghost_l(c0, uL);
    gR = T(0);
    cn1 = T(0);
    cn2 = T(0);
    cn3 = c0;  // positions 0 and 1 arrive at t = 0, 1 through the four-slot queue
    cn4 = (n > 1) ? o.load_c(1) : T(0);
    fq = o.face(0);
    flux_lo = flux_hi = T(0);
    S1 = StageS<T>{T(0), T(0), T(0), T(0), T(0), T(0)};
    S2 = S1;
    S3 = S1;
    S4 = S1;
    const int t_last = (TM == 1) ? n + 1 : n + 7;
    // blocks of 8 starting at t = -8 (ring index = t & 7); positions before
    // -2 are skipped inside the guarded body.
    int T0 = -8;
    // the queue is primed for t = -2: c0 and c1 shift down to be consumed
    // at t = 0 and 1, the loads at t = -2, -1 bring c2 and c3
#pragma unroll 1
    for (; T0 <= t_last; T0 += 8) {
      // steady blocks end by n-2: t = n-1 captures the right ghost value
      const bool steady = (TM == 2) ? (T0 >= 8 && T0 + 7 <= n - 2) : (T0 >= 2 && T0 + 7 <= n - 2);
      o.stage_begin(T0);
      if (steady) block8<false>(T0);
      else block8<true>(T0);
      o.stage_end(T0);
    }
    o.stage_finish();
  }
};

}  // namespace f3d
