// EES local pseudopotential and reciprocal Ewald sum (cp_eext_ees_opt on)
// on one GPU: the B-spline grids of the atom types, their 3-D transform,
// and the atom forces from the back-transformed force grids.  The g-space
// part (energies, V_KS and the force transforms) runs inside the density z
// pass (k_rho_zpass with EesLocArgs, oa_rho.cu).
//
// Replaces:
//   CPLOCAL::eesAtmBsplineRgrp + eesPackGridRchare (cp_hart_ext.C:641-990)  -> k_eesl_spread
//   the RhoRHartExt -> GHartExt transform of sfAtmTypR, exp(+2 pi i m.k/n),
//     and the GHartExt -> RhoRHartExt one of the force grids, exp(-...)
//     (CP_Rho_RHartExt.C:300-330, CP_Rho_GHartExt.C:1018-1060)              -> k_grid_fft2 (two-pass register
//     transforms) or k_grid_fft (runtime plan), one pass per axis
//   CPLOCAL::eesAtmForceRchare, types and Ewald (cp_hart_ext.C:1357-1470)    -> k_eesl_force
// Atom types 2k and 2k+1 share complex grid k (real and imaginary part), so
// one complex transform serves two real ones; the Ewald force grid is folded
// into the per-type grids by the type's charge in g-space.
#include "oa_internal.h"
#include "oa_bspline.cuh"
#include "oa_rdft.cuh"

// One warp per atom: lanes 0..2 build the axis stencils, then the warp adds
// M_a M_b M_c over the order^3 points into the atom type's grid slot.
__global__ void __launch_bounds__(32) k_eesl_spread(const double* __restrict__ pos, const int* __restrict__ atm_type,
                                                    int natm, double box, int na, int nb, int nc, int order,
                                                    size_t gstride, double* __restrict__ zq) {
  __shared__ int sidx[3][16];
  __shared__ double sm[3][16];
  const int a = blockIdx.x, lane = threadIdx.x;
  if (a >= natm) return;
  if (lane < 3) {
    const int ng = lane == 0 ? na : (lane == 1 ? nb : nc);
    ees_bspline_axis(pos[3 * a + lane], box, ng, order, sidx[lane], sm[lane], nullptr);
  }
  __syncwarp();
  const int t = atm_type[a];
  double* g = zq + 2 * (size_t)(t >> 1) * gstride + (t & 1);
  const int n2 = order * order, n3 = n2 * order;
  for (int p = lane; p < n3; p += 32) {
    const int jc = p / n2, r = p - jc * n2, jb = r / order, ja = r - jb * order;
    const double w = sm[0][ja] * sm[1][jb] * sm[2][jc];
    const size_t off = ((size_t)sidx[2][jc] * nb + sidx[1][jb]) * na + sidx[0][ja];
    atomicAdd(g + 2 * off, w);
  }
}

// Batched 1-D transforms along one axis of complex grids [n2][n1][n0]
// (n0 fastest; blockIdx.y = grid), lb lines per block in shared memory.
// Axis 0 lines are contiguous; the strided axes load lb neighbouring lines
// per element so that a warp reads consecutive addresses.
template <int SIGN>
__global__ void __launch_bounds__(OA_NTHREADS) k_grid_fft(double2* __restrict__ grids, size_t gstride, int n0, int n1,
                                                          int n2, int ax, int lb, OaFftPlan p,
                                                          const double2* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = p.n, ld = n + 1;
  double2* stw = (double2*)smem_raw;
  double2* a = stw + ((n + 1) & ~1);
  double2* b = a + (size_t)lb * ld;
  double2* g = grids + (size_t)blockIdx.y * gstride;
  const int nlines = ax == 0 ? n1 * n2 : (ax == 1 ? n0 * n2 : n0 * n1);
  const int l0 = blockIdx.x * lb;
  const int nl = min(lb, nlines - l0);
  const size_t es = ax == 0 ? 1 : (ax == 1 ? (size_t)n0 : (size_t)n0 * n1);
  auto base = [&](int l) -> size_t {
    if (ax == 0) return (size_t)l * n0;
    if (ax == 1) return (size_t)(l / n0) * n0 * n1 + (l % n0);
    return (size_t)l;
  };
  load_twiddles(stw, tw, n);
  for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
    int li, i;
    if (ax == 0) { li = idx / n; i = idx - li * n; } else { i = idx / nl; li = idx - i * nl; }
    a[li * ld + i] = g[base(l0 + li) + (size_t)i * es];
  }
  __syncthreads();
  const double2* r = fft_pingpong<SIGN>(a, b, ld, nl, p, stw);
  for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
    int li, i;
    if (ax == 0) { li = idx / n; i = idx - li * n; } else { i = idx / nl; li = idx - i * nl; }
    g[base(l0 + li) + (size_t)i * es] = r[li * ld + i];
  }
}

// The same passes with the two-pass register transform of the lengths with
// a compile-time factorisation N = N1 N2 (zfft2, oa_rdft.cuh): two block
// barriers per batch of lines instead of one per radix stage.
template <int N1, int N2, int SIGN>
__global__ void __launch_bounds__(OA_NTHREADS) k_grid_fft2(double2* __restrict__ grids, size_t gstride, int n0,
                                                           int n1, int n2, int ax, int lb,
                                                           const double2* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int N = N1 * N2, LD = N + 1;
  double2* stw = (double2*)smem_raw;
  double2* a = stw + ((N + 1) & ~1);
  double2* b = a + (size_t)lb * LD;
  double2* g = grids + (size_t)blockIdx.y * gstride;
  const int nlines = ax == 0 ? n1 * n2 : (ax == 1 ? n0 * n2 : n0 * n1);
  const int l0 = blockIdx.x * lb;
  const int nl = min(lb, nlines - l0);
  const size_t es = ax == 0 ? 1 : (ax == 1 ? (size_t)n0 : (size_t)n0 * n1);
  auto base = [&](int l) -> size_t {
    if (ax == 0) return (size_t)l * n0;
    if (ax == 1) return (size_t)(l / n0) * n0 * n1 + (l % n0);
    return (size_t)l;
  };
  load_twiddles(stw, tw, N);
  for (int idx = threadIdx.x; idx < nl * N; idx += blockDim.x) {
    int li, i;
    if (ax == 0) { li = idx / N; i = idx - li * N; } else { i = idx / nl; li = idx - i * nl; }
    a[li * LD + i] = g[base(l0 + li) + (size_t)i * es];
  }
  __syncthreads();
  zfft2<N1, N2, SIGN>(a, b, LD, nl, stw);
  for (int idx = threadIdx.x; idx < nl * N; idx += blockDim.x) {
    int li, i;
    if (ax == 0) { li = idx / N; i = idx - li * N; } else { i = idx / nl; li = idx - i * nl; }
    g[base(l0 + li) + (size_t)i * es] = a[li * LD + i];
  }
}

// the factorisations of the two-pass grid kernels (N1 <= 16)
#define OA_GRID_LENGTHS(X) \
  X(64, 8, 8) X(75, 15, 5) X(80, 16, 5) X(96, 12, 8) X(100, 10, 10) X(108, 12, 9) X(120, 12, 10) \
  X(128, 16, 8) X(144, 12, 12) X(150, 15, 10) X(160, 16, 10) X(180, 15, 12) X(192, 16, 12) X(200, 10, 20) \
  X(216, 12, 18) X(240, 16, 15) X(256, 16, 16)

// One warp per atom: F_a = -sum over the stencil of grad(M_a M_b M_c) P_t
// with P_t the type's back-transformed force grid (the Ewald part is in it).
__global__ void __launch_bounds__(32) k_eesl_force(const double* __restrict__ pos, const int* __restrict__ atm_type,
                                                   int natm, double box, int na, int nb, int nc, int order,
                                                   size_t gstride, const double* __restrict__ zy,
                                                   double* __restrict__ fout) {
  __shared__ int sidx[3][16];
  __shared__ double sm[3][16], sd[3][16];
  const int a = blockIdx.x, lane = threadIdx.x;
  if (a >= natm) return;
  if (lane < 3) {
    const int ng = lane == 0 ? na : (lane == 1 ? nb : nc);
    ees_bspline_axis(pos[3 * a + lane], box, ng, order, sidx[lane], sm[lane], sd[lane]);
  }
  __syncwarp();
  const int t = atm_type[a];
  const double* g = zy + 2 * (size_t)(t >> 1) * gstride + (t & 1);
  const int n2 = order * order, n3 = n2 * order;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int p = lane; p < n3; p += 32) {
    const int jc = p / n2, r = p - jc * n2, jb = r / order, ja = r - jb * order;
    const size_t off = ((size_t)sidx[2][jc] * nb + sidx[1][jb]) * na + sidx[0][ja];
    const double v = g[2 * off];
    fx += sd[0][ja] * sm[1][jb] * sm[2][jc] * v;
    fy += sm[0][ja] * sd[1][jb] * sm[2][jc] * v;
    fz += sm[0][ja] * sm[1][jb] * sd[2][jc] * v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (lane == 0) {
    fout[3 * a + 0] = -fx * ((double)na / box);
    fout[3 * a + 1] = -fy * ((double)nb / box);
    fout[3 * a + 2] = -fz * ((double)nc / box);
  }
}

// lines per block of k_grid_fft for length n within the shared-memory limit
static int grid_fft_lines(int n) {
  int lb = OA_LB;
  while (lb > 1 && (size_t)(((n + 1) & ~1) + 2 * (size_t)lb * (n + 1)) * sizeof(double2) > (size_t)OA_MAX_SMEM) lb >>= 1;
  return lb;
}

// one axis pass by the two-pass kernel of its length (lines per block so
// that two blocks share an SM); cudaErrorNotSupported for other lengths
template <int SIGN>
static cudaError_t grid_fft2_axis(oa_eesl* L, cudaStream_t s, double2* grids, int ax, int n, const double2* tw) {
  const size_t gs = (size_t)L->na * L->nb * L->nc;
  const int nlines = (int)(gs / n);
  auto go = [&](auto kern, int ps) -> cudaError_t {
    int lb = OA_LB;
    auto bytes = [&](int l) { return (size_t)(((n + 1) & ~1) + (size_t)l * (n + 1) + (size_t)l * ps) * sizeof(double2); };
    while (lb > 2 && bytes(lb) > (size_t)(OA_MAX_SMEM / 2)) lb >>= 1;
    cudaError_t e = oa_smem_limit(kern);
    if (e != cudaSuccess) return e;
    kern<<<dim3((nlines + lb - 1) / lb, L->ngrid), OA_NTHREADS, bytes(lb), s>>>(grids, gs, L->na, L->nb, L->nc, ax,
                                                                             lb, tw);
    return cudaGetLastError();
  };
  switch (n) {
#define OA_GF2(NN, A, B) \
  case NN: return go(k_grid_fft2<A, B, SIGN>, ZLd<A, B>::PS);
    OA_GRID_LENGTHS(OA_GF2)
#undef OA_GF2
    default: return cudaErrorNotSupported;
  }
}

template <int SIGN>
static cudaError_t grid_fft3(oa_eesl* L, cudaStream_t s, double2* grids) {
  const size_t gs = (size_t)L->na * L->nb * L->nc;
  const OaFftPlan* pl[3] = {&L->pa, &L->pb, &L->pc};
  const double2* tw[3] = {L->tw_a, L->tw_b, L->tw_c};
  cudaError_t e = oa_smem_limit(k_grid_fft<SIGN>);
  if (e != cudaSuccess) return e;
  for (int ax = 0; ax < 3; ++ax) {
    const int n = pl[ax]->n;
    e = grid_fft2_axis<SIGN>(L, s, grids, ax, n, tw[ax]);
    if (e != cudaErrorNotSupported) {
      if (e != cudaSuccess) return e;
      continue;
    }
    const int lb = grid_fft_lines(n);
    const int nlines = (int)(gs / n);
    const size_t smem = (size_t)(((n + 1) & ~1) + 2 * (size_t)lb * (n + 1)) * sizeof(double2);
    k_grid_fft<SIGN><<<dim3((nlines + lb - 1) / lb, L->ngrid), OA_NTHREADS, smem, s>>>(
        grids, gs, L->na, L->nb, L->nc, ax, lb, *pl[ax], tw[ax]);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t oa_launch_eesl_front(oa_ctx* c, cudaStream_t s) {
  oa_eesl* L = c->eesl;
  const size_t gs = (size_t)L->na * L->nb * L->nc;
  cudaError_t e = cudaMemsetAsync(L->zq, 0, gs * L->ngrid * sizeof(double2), s);
  if (e != cudaSuccess) return e;
  if (c->ions && (e = cudaMemsetAsync(L->zy, 0, gs * L->ngrid * sizeof(double2), s)) != cudaSuccess) return e;
  k_eesl_spread<<<c->natm, 32, 0, s>>>(c->pos, c->atm_type, c->natm, c->box, L->na, L->nb, L->nc, L->order, gs,
                                       (double*)L->zq);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return grid_fft3<+1>(L, s, L->zq);
}

cudaError_t oa_launch_eesl_forces(oa_ctx* c, cudaStream_t s) {
  oa_eesl* L = c->eesl;
  const size_t gs = (size_t)L->na * L->nb * L->nc;
  cudaError_t e = grid_fft3<-1>(L, s, L->zy);
  if (e != cudaSuccess) return e;
  k_eesl_force<<<c->natm, 32, 0, s>>>(c->pos, c->atm_type, c->natm, c->box, L->na, L->nb, L->nc, L->order, gs,
                                      (const double*)L->zy, c->ions->fpart);
  return cudaGetLastError();
}

void oa_eesl_free(oa_ctx* c) {
  oa_eesl* L = c->eesl;
  if (!L) return;
  void* d[] = {L->tw_a, L->tw_b, L->tw_c, L->ba, L->bb, L->bc, L->zq, L->zy, L->gzvps};
  for (void* p : d)
    if (p) cudaFree(p);
  free(L);
  c->eesl = nullptr;
}
