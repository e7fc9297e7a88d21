// deposit_dev.cu -- the two processes F3D_time_step applies after the sweeps
// (mod_F3D.F90:1493-1520):
//
//   * wet deposition, phys_wet_deposition (mod_Phys.F90:1358-1427): in every
//     column, scavenging coefficient lambda = min(1, dt a P^b) from the
//     precipitation rate P; every cell of a particle or radionuclide bin of
//     diameter <= 100 um below the boundary-layer top loses lambda c, which is
//     added (times dX3_p) to the wet deposit awet, in k order;
//   * radioactive decay, phys_radionuclides (mod_Phys.F90:1216-1342): every
//     radionuclide bin (and its dry and wet deposits) is multiplied by
//     exp(-kn dt); a Y90 bin is then set from its Sr90 parent,
//     c(Y90) = c(Sr90) (1 - exp(-kn_Sr90 dt)), as the reference does (an
//     assignment: the decayed Y90 value is overwritten), with the parent's
//     value as it stands at that point of the bin loop.  The loop covers the
//     halo cells of the state too (my_ips_2h:my_ipe_2h, ...), so the kept
//     boundary halo layers decay with it.
//
// P^b, the boundary-layer test and the decay factors are evaluated on the
// host, with the same C library as the CPU restatement; the kernels do the
// per-cell arithmetic in the reference's order (compiled with --fmad=false).
//
// With the z sweep's epilogue (MemberDev::epi_on) both processes run inside
// the z sweep, cell by cell; k_radio then only sets the daughter bins from
// their parents and decays the kept halo layers (RadioArgs::tail).
#include <cuda_runtime.h>

#include "f3d_common.cuh"
#include "phys_dev.cuh"

namespace f3d {

__global__ void k_wet(WetArgs a) {
  const long long ncol = (long long)a.nx * a.ny;
  const long long tot = ncol * a.nb;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const long long ij = e % ncol;
    const int b = (int)(e / ncol);
    if (!((a.mask >> b) & 1ull)) continue;
    const double dta = a.dt_dev ? *a.dt_dev * a.a : a.dta;
    double lambda = dta * a.powpb[ij];
    if (lambda > 1.0) lambda = 1.0;
    const int kt = a.ktop[ij];
    double aw = a.awet[e];
    for (int k = 0; k < kt; ++k) {
      const long long q = ((long long)b * a.nz + k) * ncol + ij;
      if (a.c64) {
        const double cv = a.c64[q];
        aw = aw + a.dx3p[k + 2] * lambda * cv;
        a.c64[q] = cv * (1.0 - lambda);
      } else if (a.c32lo) {  // compensated pair: FP64 value, split back
        const double cv = (double)a.c32[q] + (double)a.c32lo[q];
        aw = aw + a.dx3p[k + 2] * lambda * cv;
        const double nv = cv * (1.0 - lambda);
        const float hi = __double2float_rn(nv);
        a.c32[q] = hi;
        a.c32lo[q] = __double2float_rn(nv - (double)hi);
      } else {
        const double cv = (double)a.c32[q];
        aw = aw + a.dx3p[k + 2] * lambda * cv;
        a.c32[q] = (float)(cv * (1.0 - lambda));
      }
    }
    a.awet[e] = aw;
  }
}

template <class T>
__device__ __forceinline__ void decay_cell(const RadioArgs& a, T* c, long long q, long long stride,
                                           bool daughters_only = false) {
  for (int r = 0; r < a.nr; ++r) {
    if (daughters_only && a.parent[r] < 0) continue;  // decayed by the z sweep's epilogue
    const double f = a.fdev ? a.fdev[r] : a.fact[r];
    const double pf = a.fdev ? a.fdev[a.nr + r] : a.pfact[r];
    T* p = c + (long long)a.bin[r] * stride + q;
    *p = (T)((double)*p * f);
    if (a.parent[r] >= 0) *p = (T)((double)c[(long long)a.parent[r] * stride + q] * (1.0 - pf));
  }
}

// The same on the compensated pair hi + lo of the precision form.
__device__ __forceinline__ void decay_cell_pair(const RadioArgs& a, float* hi, float* lo, long long q,
                                                long long stride, bool daughters_only = false) {
  for (int r = 0; r < a.nr; ++r) {
    if (daughters_only && a.parent[r] < 0) continue;
    const double f = a.fdev ? a.fdev[r] : a.fact[r];
    const double pf = a.fdev ? a.fdev[a.nr + r] : a.pfact[r];
    const long long at = (long long)a.bin[r] * stride + q;
    double v = ((double)hi[at] + (double)lo[at]) * f;
    if (a.parent[r] >= 0) {
      const long long pa = (long long)a.parent[r] * stride + q;
      v = ((double)hi[pa] + (double)lo[pa]) * (1.0 - pf);
    }
    const float h = __double2float_rn(v);
    hi[at] = h;
    lo[at] = __double2float_rn(v - (double)h);
  }
}

__global__ void k_radio(RadioArgs a) {
  const long long n2 = (long long)a.nx * a.ny, n3 = n2 * a.nz;
  const long long ng = (a.gh64 || a.gh32) ? a.ngh : 0;
  bool daughters = false;
  for (int r = 0; r < a.nr; ++r) daughters = daughters || a.parent[r] >= 0;
  // after the epilogue only the halo layers remain when no bin is a daughter
  const long long e0 = (a.tail && !daughters) ? n3 + n2 : 0;
  const bool dOnly = a.tail != 0;
  for (long long e = e0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n3 + n2 + ng;
       e += (long long)gridDim.x * blockDim.x) {
    if (e < n3) {
      if (a.c64) decay_cell(a, a.c64, e, n3, dOnly);
      else if (a.c32lo) decay_cell_pair(a, a.c32, a.c32lo, e, n3, dOnly);
      else decay_cell(a, a.c32, e, n3, dOnly);
    } else if (e < n3 + n2) {
      const long long q = e - n3;
      decay_cell(a, a.acum, q, n2, dOnly);
      if (a.awet) decay_cell(a, a.awet, q, n2, dOnly);
    } else {  // halo layers: the sweeps' ghosts, not seen by the epilogue
      const long long q = e - n3 - n2;
      if (a.gh64) decay_cell(a, a.gh64, q, ng);
      else decay_cell(a, a.gh32, q, ng);
    }
  }
}

// Column terms of grid_get_mass_sink (mod_Grid.F90:1400-1450): the bins'
// wet deposit summed in bin order, times dX times dY; the host adds the
// columns in the reference's serial order (j outer, i inner).
__global__ void k_sink_cols(int nx, int ny, int nb, const double* awet, const double* dx1p,
                            const double* dx2p, double* col) {
  const long long ncol = (long long)nx * ny;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ncol;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % nx), j = (int)(e / nx);
    double aw = 0.0;
    for (int b = 0; b < nb; ++b) aw = aw + awet[(long long)b * ncol + e];
    col[e] = aw * dx1p[i + 2] * dx2p[j + 2];
  }
}

void launch_sink_cols(int nx, int ny, int nb, const double* awet, const double* dx1p,
                      const double* dx2p, double* col, cudaStream_t st) {
  k_sink_cols<<<296, 256, 0, st>>>(nx, ny, nb, awet, dx1p, dx2p, col);
}

void launch_wet(const WetArgs& a, cudaStream_t st) { k_wet<<<592, 256, 0, st>>>(a); }
void launch_radio(const RadioArgs& a, cudaStream_t st) { k_radio<<<592, 256, 0, st>>>(a); }

}  // namespace f3d
