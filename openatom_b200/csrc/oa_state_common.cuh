// Pieces shared by the state FFT kernels (oa_state.cu: runtime-plan
// kernels for any 2-3-5 length; oa_pencil.cu: two-pass kernels for the
// lengths with a compile-time factorisation).
#pragma once
#include "oa_internal.h"

template <typename R> struct CplxOf { typedef typename OaCplx<R>::T T; };

static __device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum; result valid in thread 0.  Uses 32 doubles of smem.
static __device__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

__host__ __device__ static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <typename C>
__device__ __forceinline__ C herm_x(const C* P, int ldy, int nkx, int nx, int k, int y) {
  // value of the x-spectrum at index k of row y from the stored kx in [0, nkx)
  // (kx < 0 from Hermitian symmetry); DC / Nyquist use the real part only,
  // as a c2r transform does.
  C v = cmk<C>(0.0, 0.0);
  if (k <= nx / 2) {
    if (k < nkx) v = P[k * ldy + y];
    if (k == 0 || 2 * k == nx) v.y = 0;
  } else {
    const int kk = nx - k;
    if (kk < nkx) v = cconj(P[kk * ldy + y]);
  }
  return v;
}

#define OA_PLANE_THREADS 512
#define OA_PLANE_WARPS (OA_PLANE_THREADS / 32)

// EES stencil data for the nonlocal-grid plane modes
struct EesArgs {
  const int* idx;       // [natm][3][order] grid index per axis (a, b, c)
  const double* mn;     // [natm][3][order] B-spline weight per axis
  double* zpart;        // [nstate][natm][order] MODE 2: per-plane Z contributions
  const double* zs;     // [nstate][natm]        MODE 3: scaled Z to scatter
  int natm, order;
  const double* dmn;    // [natm][3][order] derivative weights (with fpart)
  double* fpart;        // [nstate][natm][order][3] MODE 2, null: no atom forces
};


// EES scatter onto one plane of the nonlocal grid (eesEnergyAtmForcRchare,
// cp_ees_nonlocal.C:1480-1720: projPsiRScr[igrid] += z Mn): tile (nx * ny,
// zeroed by the caller) += zs[s][a] Mn_a Mn_b Mn_c over the stencil points
// of every atom whose c-stencil reaches plane z.  One warp per atom.
template <typename R>
__device__ __forceinline__ void ees_scatter_plane(R* tile, int nx, int z, int s, const EesArgs& E, int warp,
                                                  int lane, int nwarp) {
  const int o2 = E.order * E.order;
  for (int a = warp; a < E.natm; a += nwarp) {
    const int* ia = E.idx + (size_t)a * 3 * E.order;
    const double* ma = E.mn + (size_t)a * 3 * E.order;
    int jc = -1;
    for (int j = 0; j < E.order; ++j) if (ia[2 * E.order + j] == z) jc = j;
    if (jc < 0) continue;
    const double zc = E.zs[(size_t)s * E.natm + a] * ma[2 * E.order + jc];
    for (int q = lane; q < o2; q += 32) {
      const int jb = q / E.order, ja = q - jb * E.order;
      atomicAdd(&tile[ia[E.order + jb] * nx + ia[ja]], (R)(zc * ma[E.order + jb] * ma[ja]));
    }
  }
}

// EES Z gather on one plane (eesZmatRchare, cp_ees_nonlocal.C:1238-1352):
// zpart[s][a][jc] = Mn_c(jc) sum over the a-b stencil of tile * Mn_a Mn_b.
// With fpart the plane's share of the atom-force sums of
// eesEnergyAtmForcRchare (1560-1720), before the zs and n / L factors:
// (Mn_c sum tile dMn_a Mn_b, Mn_c sum tile Mn_a dMn_b, dMn_c sum tile Mn_a Mn_b).
template <typename R>
__device__ __forceinline__ void ees_gather_plane(const R* tile, int nx, int z, int s, const EesArgs& E, int warp,
                                                 int lane, int nwarp) {
  const int o2 = E.order * E.order;
  const bool frc = E.fpart != nullptr;
  for (int a = warp; a < E.natm; a += nwarp) {
    const int* ia = E.idx + (size_t)a * 3 * E.order;
    const double* ma = E.mn + (size_t)a * 3 * E.order;
    const double* da = frc ? E.dmn + (size_t)a * 3 * E.order : ma;
    int jc = -1;
    for (int j = 0; j < E.order; ++j) if (ia[2 * E.order + j] == z) jc = j;
    if (jc < 0) continue;
    double acc = 0.0, fx = 0.0, fy = 0.0;
    for (int q = lane; q < o2; q += 32) {
      const int jb = q / E.order, ja = q - jb * E.order;
      const double v = (double)tile[ia[E.order + jb] * nx + ia[ja]];
      acc += v * ma[E.order + jb] * ma[ja];
      if (frc) {
        fx += v * ma[E.order + jb] * da[ja];
        fy += v * da[E.order + jb] * ma[ja];
      }
    }
    acc = warp_sum(acc);
    if (frc) {
      fx = warp_sum(fx);
      fy = warp_sum(fy);
    }
    if (lane == 0) {
      const double mc = ma[2 * E.order + jc];
      E.zpart[((size_t)s * E.natm + a) * E.order + jc] = acc * mc;
      if (frc) {
        double* fp = E.fpart + (((size_t)s * E.natm + a) * E.order + jc) * 3;
        fp[0] = fx * mc;
        fp[1] = fy * mc;
        fp[2] = acc * da[2 * E.order + jc];
      }
    }
  }
}
