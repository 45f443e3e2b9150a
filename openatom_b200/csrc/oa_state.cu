// State FFT path of one CP step on one GPU: sphere -> z-lines -> planes ->
// density; V_KS psi -> planes -> z-lines -> sphere forces + EKE.
//
// Replaces the work of these reference entry points for all states at once:
//   CP_State_GSpacePlane::doFFT        (CP_State_GSpacePlane.C:1377)  -> k_state_zfwd
//   FFTcache::expandGSpace/doStpFFTGtoR_Gchare (fftCache.C:460,1133)  -> k_state_zfwd
//   CP_State_GSpacePlane::sendFFTData / RealSpacePlane::unpackFFT
//       (CP_State_GSpacePlane.C:1448, CP_State_RealSpacePlane.C:186) -> z-major line buffer
//   FFTcache::doStpFFTGtoR_Rchare (fftCache.C:1167) + density part of
//       CP_State_RealSpacePlane::doFFT (:349-363) + doReduction (:450) -> k_state_plane_density
//   CP_State_RealSpacePlane::unpackVks (:530-597), doVksFFT (:607),
//       FFTcache::doStpFFTRtoG_Rchare (fftCache.C:1252), sendFPsiToGSP (:663) -> k_state_plane_vks
//   CP_State_GSpacePlane::unpackIFFT/doIFFT (:1530,1581), packGSpace (fftCache.C:517),
//       GStateSlab::addForces (stateSlab.C:239), CPNONLOCAL::CP_eke_calc (cp_eke.C:30) -> k_state_zbwd
//
// HBM layout: coefficients psi[state][g] double2 (AoS re,im as the reference's
// complex); the z-line buffer zbuf[state][z][line] in the compute precision,
// lines padded to ldl so each (state, z) row is one contiguous, aligned run.
#include "oa_internal.h"

template <typename R> struct CplxOf { typedef typename OaCplx<R>::T T; };

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum; result valid in thread 0.  Uses 32 doubles of smem.
__device__ double block_sum(double v, double* sh) {
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

// ---------------------------------------------------------------------------
// z pass, forward: packed sphere -> zero-filled z-lines -> FFT(-) -> zbuf[s][z][l]
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(OA_NTHREADS)
k_state_zfwd(const double2* __restrict__ psi, int ng, int s0,
             const int* __restrict__ line_off, const int* __restrict__ line_nneg,
             const int* __restrict__ line_npos, int nlines,
             typename CplxOf<R>::T* __restrict__ zbuf, int nz, int ldl,
             OaFftPlan pz, const double2* __restrict__ twz) {
  typedef typename CplxOf<R>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ldz = nz + 1;
  C* tw = (C*)smem_raw;
  C* a = tw + align_up(nz, 2);
  C* b = a + OA_LB * ldz;
  const int s = s0 + blockIdx.y;
  const int l0 = blockIdx.x * OA_LB;
  const int nb = min(OA_LB, nlines - l0);
  load_twiddles(tw, twz, nz);
  for (int i = threadIdx.x; i < OA_LB * ldz; i += blockDim.x) a[i] = cmk<C>(0.0, 0.0);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  const double2* ps = psi + (size_t)s * ng;
  for (int lb = warp; lb < nb; lb += nwarp) {
    const int l = l0 + lb;
    const int off = line_off[l], nn = line_nneg[l], np = line_npos[l];
    for (int i = lane; i < nn + np; i += 32) {
      const int kzi = (i < nn) ? (nz - nn + i) : (i - nn);
      const double2 v = ps[off + i];
      a[lb * ldz + kzi] = cmk<C>(v.x, v.y);
    }
  }
  __syncthreads();
  C* r = fft_pingpong<-1>(a, b, ldz, nb, pz, tw);
  C* out = zbuf + (size_t)s * nz * ldl + l0;
  for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
    const int z = idx / OA_LB, lb = idx - z * OA_LB;
    if (lb < nb) out[(size_t)z * ldl + lb] = r[lb * ldz + z];
  }
}

// ---------------------------------------------------------------------------
// plane helpers
// ---------------------------------------------------------------------------
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

// Build W[p][k] = X_{y1}(k) + i X_{y2}(k) for row pairs p in [0, np).
template <typename C>
__device__ void build_pairs(C* W, int ldx, const C* P, int ldy, int nkx, int nx, int ny, int p0, int np) {
  for (int idx = threadIdx.x; idx < np * nx; idx += blockDim.x) {
    const int p = idx / nx, k = idx - p * nx;
    const int y1 = 2 * (p0 + p), y2 = y1 + 1;
    const C a = herm_x(P, ldy, nkx, nx, k, y1);
    C b = cmk<C>(0.0, 0.0);
    if (y2 < ny) b = herm_x(P, ldy, nkx, nx, k, y2);
    C z; z.x = a.x - b.y; z.y = a.y + b.x;
    W[p * ldx + k] = z;
  }
}

// Split W[p][k] = F1(k) + i F2(k) of two real sequences, store k < nkx into P.
template <typename C>
__device__ void split_pairs(const C* W, int ldx, C* P, int ldy, int nkx, int nx, int ny, int p0, int np) {
  typedef decltype(W[0].x) R;
  for (int idx = threadIdx.x; idx < np * nkx; idx += blockDim.x) {
    const int p = idx / nkx, k = idx - p * nkx;
    const int y1 = 2 * (p0 + p), y2 = y1 + 1;
    const C a = W[p * ldx + k];
    const C b = cconj(W[p * ldx + (k == 0 ? 0 : nx - k)]);
    C f1, f2;
    f1.x = (a.x + b.x) * (R)0.5; f1.y = (a.y + b.y) * (R)0.5;
    const R dx = a.x - b.x, dy = a.y - b.y;
    f2.x = dy * (R)0.5; f2.y = -dx * (R)0.5;
    P[k * ldy + y1] = f1;
    if (y2 < ny) P[k * ldy + y2] = f2;
  }
}

struct PlaneSmem {
  size_t tw_x, tw_y, P, W1, W2, tile, red, total;
};

template <typename C, typename T>
static PlaneSmem plane_smem_layout(int nx, int ny, int nkx, int npair, int ychunk, bool tile) {
  PlaneSmem L;
  const int ldx = nx + 1, ldy = ny + 1;
  size_t o = 0;
  L.tw_x = o; o += align_up(nx * sizeof(C), 16);
  L.tw_y = o; o += align_up(ny * sizeof(C), 16);
  L.P = o; o += align_up((size_t)nkx * ldy * sizeof(C), 16);
  size_t wsz = (size_t)npair * ldx;
  if ((size_t)ychunk * ldy > wsz) wsz = (size_t)ychunk * ldy;
  L.W1 = o; o += align_up(wsz * sizeof(C), 16);
  L.W2 = o; o += align_up(wsz * sizeof(C), 16);
  L.tile = o; if (tile) o += align_up((size_t)nx * ny * sizeof(T), 16);
  L.red = o; o += 64 * sizeof(double);
  L.total = o;
  return L;
}

// y FFT of all nkx columns of P, in place, in chunks through W1/W2.
template <int SIGN, typename C>
__device__ void plane_yfft(C* P, int ldy, int nkx, int ychunk, C* W1, C* W2, const OaFftPlan& py, const C* twy) {
  for (int c0 = 0; c0 < nkx; c0 += ychunk) {
    const int nb = min(ychunk, nkx - c0);
    fft_inout<SIGN>(P + c0 * ldy, ldy, P + c0 * ldy, ldy, W1, W2, ldy, nb, py, twy);
  }
}

// ---------------------------------------------------------------------------
// plane pass, forward + density: zbuf row (s, z) -> P[kx][y] -> y FFT(-) ->
// c2r x FFT(-) by row pairs -> rho tile += occ psi(r)^2
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(OA_NTHREADS)
k_state_plane_density(const typename CplxOf<R>::T* __restrict__ zbuf, int nstate, int ldl, int nlines,
                      const int* __restrict__ line_kx, const int* __restrict__ line_ky,
                      int nx, int ny, int nz, int nkx,
                      OaFftPlan px, OaFftPlan py, const double2* __restrict__ twx, const double2* __restrict__ twy,
                      const double* __restrict__ occ, double* __restrict__ rho_part,
                      int ngroup, int npair, int ychunk, PlaneSmem L) {
  typedef typename CplxOf<R>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* stwx = (C*)(smem_raw + L.tw_x);
  C* stwy = (C*)(smem_raw + L.tw_y);
  C* P = (C*)(smem_raw + L.P);
  C* W1 = (C*)(smem_raw + L.W1);
  C* W2 = (C*)(smem_raw + L.W2);
  R* tile = (R*)(smem_raw + L.tile);
  const int ldx = nx + 1, ldy = ny + 1;
  const int z = blockIdx.x, g = blockIdx.y;
  const int nper = (nstate + ngroup - 1) / ngroup;
  const int sb = g * nper, se = min(nstate, sb + nper);
  const int npairs = (ny + 1) / 2;
  load_twiddles(stwx, twx, nx);
  load_twiddles(stwy, twy, ny);
  for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) tile[i] = (R)0;
  for (int s = sb; s < se; ++s) {
    for (int i = threadIdx.x; i < nkx * ldy; i += blockDim.x) P[i] = cmk<C>(0.0, 0.0);
    __syncthreads();
    const C* row = zbuf + ((size_t)s * nz + z) * ldl;
    for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
      int ky = line_ky[l]; if (ky < 0) ky += ny;
      P[line_kx[l] * ldy + ky] = row[l];
    }
    __syncthreads();
    plane_yfft<-1>(P, ldy, nkx, ychunk, W1, W2, py, stwy);
    const R o = (R)occ[s];
    for (int p0 = 0; p0 < npairs; p0 += npair) {
      const int np = min(npair, npairs - p0);
      build_pairs(W1, ldx, P, ldy, nkx, nx, ny, p0, np);
      __syncthreads();
      C* r = fft_pingpong<-1>(W1, W2, ldx, np, px, stwx);
      for (int idx = threadIdx.x; idx < np * nx; idx += blockDim.x) {
        const int p = idx / nx, x = idx - p * nx;
        const int y1 = 2 * (p0 + p);
        const C v = r[p * ldx + x];
        tile[y1 * nx + x] += o * v.x * v.x;
        if (y1 + 1 < ny) tile[(y1 + 1) * nx + x] += o * v.y * v.y;
      }
      __syncthreads();
    }
  }
  __syncthreads();
  double* out = rho_part + ((size_t)g * nz + z) * (size_t)nx * ny;
  for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) out[i] = (double)tile[i];
}

// ---------------------------------------------------------------------------
// plane pass, V_KS: zbuf row -> psi(r) by row pairs -> * V_KS occ -> r2c x
// FFT(+) -> y FFT(+) -> zbuf row (in place)
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(OA_NTHREADS)
k_state_plane_vks(typename CplxOf<R>::T* __restrict__ zbuf, int nstate, int ldl, int nlines,
                  const int* __restrict__ line_kx, const int* __restrict__ line_ky,
                  int nx, int ny, int nz, int nkx,
                  OaFftPlan px, OaFftPlan py, const double2* __restrict__ twx, const double2* __restrict__ twy,
                  const double* __restrict__ occ, const R* __restrict__ vks,
                  int ngroup, int npair, int ychunk, PlaneSmem L) {
  typedef typename CplxOf<R>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* stwx = (C*)(smem_raw + L.tw_x);
  C* stwy = (C*)(smem_raw + L.tw_y);
  C* P = (C*)(smem_raw + L.P);
  C* W1 = (C*)(smem_raw + L.W1);
  C* W2 = (C*)(smem_raw + L.W2);
  R* tile = (R*)(smem_raw + L.tile);
  const int ldx = nx + 1, ldy = ny + 1;
  const int z = blockIdx.x, g = blockIdx.y;
  const int nper = (nstate + ngroup - 1) / ngroup;
  const int sb = g * nper, se = min(nstate, sb + nper);
  const int npairs = (ny + 1) / 2;
  load_twiddles(stwx, twx, nx);
  load_twiddles(stwy, twy, ny);
  const R* vz = vks + (size_t)z * nx * ny;
  for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) tile[i] = vz[i];
  for (int s = sb; s < se; ++s) {
    for (int i = threadIdx.x; i < nkx * ldy; i += blockDim.x) P[i] = cmk<C>(0.0, 0.0);
    __syncthreads();
    C* row = zbuf + ((size_t)s * nz + z) * ldl;
    for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
      int ky = line_ky[l]; if (ky < 0) ky += ny;
      P[line_kx[l] * ldy + ky] = row[l];
    }
    __syncthreads();
    plane_yfft<-1>(P, ldy, nkx, ychunk, W1, W2, py, stwy);
    const R o = (R)occ[s];
    for (int p0 = 0; p0 < npairs; p0 += npair) {
      const int np = min(npair, npairs - p0);
      build_pairs(W1, ldx, P, ldy, nkx, nx, ny, p0, np);
      __syncthreads();
      C* r = fft_pingpong<-1>(W1, W2, ldx, np, px, stwx);
      for (int idx = threadIdx.x; idx < np * nx; idx += blockDim.x) {
        const int p = idx / nx, x = idx - p * nx;
        const int y1 = 2 * (p0 + p);
        C v = r[p * ldx + x];
        v.x *= tile[y1 * nx + x] * o;
        v.y = (y1 + 1 < ny) ? v.y * tile[(y1 + 1) * nx + x] * o : (R)0;
        r[p * ldx + x] = v;
      }
      __syncthreads();
      C* other = (r == W1) ? W2 : W1;
      C* r2 = fft_pingpong<+1>(r, other, ldx, np, px, stwx);
      split_pairs(r2, ldx, P, ldy, nkx, nx, ny, p0, np);
      __syncthreads();
    }
    plane_yfft<+1>(P, ldy, nkx, ychunk, W1, W2, py, stwy);
    for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
      int ky = line_ky[l]; if (ky < 0) ky += ny;
      row[l] = P[line_kx[l] * ldy + ky];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// z pass, backward: zbuf -> FFT(+) -> pack, F = -2/N (x2 for kx>0) + F_NL,
// then CP_eke_calc: F -= occ w g2 psi (g2 <= ecut), EKE partials
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(OA_NTHREADS)
k_state_zbwd(const typename CplxOf<R>::T* __restrict__ zbuf, int nz, int ldl, int nlines,
             const int* __restrict__ line_kx, const int* __restrict__ line_off,
             const int* __restrict__ line_nneg, const int* __restrict__ line_npos,
             OaFftPlan pz, const double2* __restrict__ twz,
             const double2* __restrict__ psi, const double2* __restrict__ fnl, double2* __restrict__ force,
             const double* __restrict__ g2, const double* __restrict__ occ, int ng, int s0,
             double scale, double ecut, double* __restrict__ eke_part, int nblk) {
  typedef typename CplxOf<R>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ldz = nz + 1;
  C* tw = (C*)smem_raw;
  C* a = tw + align_up(nz, 2);
  C* b = a + OA_LB * ldz;
  double* sred = (double*)(b + OA_LB * ldz);
  const int s = s0 + blockIdx.y;
  const int l0 = blockIdx.x * OA_LB;
  const int nb = min(OA_LB, nlines - l0);
  load_twiddles(tw, twz, nz);
  const C* in = zbuf + (size_t)s * nz * ldl + l0;
  for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
    const int z = idx / OA_LB, lb = idx - z * OA_LB;
    if (lb < nb) a[lb * ldz + z] = in[(size_t)z * ldl + lb];
  }
  __syncthreads();
  C* r = fft_pingpong<+1>(a, b, ldz, nb, pz, tw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  const double2* ps = psi + (size_t)s * ng;
  double2* fs = force + (size_t)s * ng;
  const double2* fn = fnl ? fnl + (size_t)s * ng : nullptr;
  const double o = occ[s];
  double ek = 0.0;
  for (int lb = warp; lb < nb; lb += nwarp) {
    const int l = l0 + lb;
    const int off = line_off[l], nn = line_nneg[l], np = line_npos[l];
    const double w = (line_kx[l] == 0) ? 1.0 : 2.0;
    const double sc = scale * w;
    const double wt = o * w;
    for (int i = lane; i < nn + np; i += 32) {
      const int kzi = (i < nn) ? (nz - nn + i) : (i - nn);
      const C v = r[lb * ldz + kzi];
      const int idx = off + i;
      double2 f = make_double2((double)v.x * sc, (double)v.y * sc);
      if (fn) { const double2 q = fn[idx]; f.x += q.x; f.y += q.y; }
      const double gg = g2[idx];
      if (gg <= ecut) {
        const double2 p = ps[idx];
        const double t = wt * gg;
        f.x -= p.x * t; f.y -= p.y * t;
        ek += t * (p.x * p.x + p.y * p.y);
      } else {
        f.x = 0.0; f.y = 0.0;
      }
      fs[idx] = f;
    }
  }
  const double tot = block_sum(ek, sred);
  if (threadIdx.x == 0) eke_part[(size_t)s * nblk + blockIdx.x] = tot;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename R>
static size_t zpass_smem(int nz) {
  typedef typename CplxOf<R>::T C;
  return (align_up(nz, 2) + 2 * (size_t)OA_LB * (nz + 1)) * sizeof(C) + 64 * sizeof(double);
}

template <typename R>
static cudaError_t launch_zfwd(oa_ctx* c, cudaStream_t st, const double2* psi, int s0, int ns) {
  typedef typename CplxOf<R>::T C;
  size_t sm = zpass_smem<R>(c->nz);
  cudaError_t e = cudaFuncSetAttribute(k_state_zfwd<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid((c->nlines + OA_LB - 1) / OA_LB, ns);
  k_state_zfwd<R><<<grid, OA_NTHREADS, sm, st>>>(psi, c->ng, s0, c->line_off, c->line_nneg, c->line_npos,
                                                  c->nlines, (C*)c->zbuf, c->nz, c->ldl, c->plan_z, c->tw_z);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_plane_density(oa_ctx* c, cudaStream_t st) {
  typedef typename CplxOf<R>::T C;
  PlaneSmem L = plane_smem_layout<C, R>(c->nx, c->ny, c->nkx_s, c->npair_s, c->ychunk_s, true);
  cudaError_t e = cudaFuncSetAttribute(k_state_plane_density<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
  if (e != cudaSuccess) return e;
  dim3 grid(c->nz, c->ngroup);
  k_state_plane_density<R><<<grid, OA_NTHREADS, L.total, st>>>(
      (const C*)c->zbuf, c->nstate, c->ldl, c->nlines, c->line_kx, c->line_ky, c->nx, c->ny, c->nz, c->nkx_s,
      c->plan_x, c->plan_y, c->tw_x, c->tw_y, c->occ, c->rho_part, c->ngroup, c->npair_s, c->ychunk_s, L);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_plane_vks(oa_ctx* c, cudaStream_t st) {
  typedef typename CplxOf<R>::T C;
  PlaneSmem L = plane_smem_layout<C, R>(c->nx, c->ny, c->nkx_s, c->npair_s, c->ychunk_s, true);
  cudaError_t e = cudaFuncSetAttribute(k_state_plane_vks<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
  if (e != cudaSuccess) return e;
  dim3 grid(c->nz, c->ngroup);
  k_state_plane_vks<R><<<grid, OA_NTHREADS, L.total, st>>>(
      (C*)c->zbuf, c->nstate, c->ldl, c->nlines, c->line_kx, c->line_ky, c->nx, c->ny, c->nz, c->nkx_s,
      c->plan_x, c->plan_y, c->tw_x, c->tw_y, c->occ, (const R*)c->vks, c->ngroup, c->npair_s, c->ychunk_s, L);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_zbwd(oa_ctx* c, cudaStream_t st, const double2* psi, const double2* fnl,
                               double2* force, int s0, int ns) {
  typedef typename CplxOf<R>::T C;
  size_t sm = zpass_smem<R>(c->nz);
  cudaError_t e = cudaFuncSetAttribute(k_state_zbwd<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid(c->nblk_z, ns);
  k_state_zbwd<R><<<grid, OA_NTHREADS, sm, st>>>(
      (const C*)c->zbuf, c->nz, c->ldl, c->nlines, c->line_kx, c->line_off, c->line_nneg, c->line_npos,
      c->plan_z, c->tw_z, psi, fnl, force, c->g2, c->occ, c->ng, s0, -2.0 / (double)c->npts,
      c->ecut_psi, c->eke_part, c->nblk_z);
  return cudaGetLastError();
}

size_t oa_plane_smem_bytes(int precision, int nx, int ny, int nkx, int npair, int ychunk, bool tile) {
  if (precision == OA_FP64) return plane_smem_layout<double2, double>(nx, ny, nkx, npair, ychunk, tile).total;
  return plane_smem_layout<float2, float>(nx, ny, nkx, npair, ychunk, tile).total;
}

cudaError_t oa_launch_state_zfwd(oa_ctx* c, cudaStream_t s, const double2* psi, int s0, int ns) {
  return c->precision == OA_FP64 ? launch_zfwd<double>(c, s, psi, s0, ns) : launch_zfwd<float>(c, s, psi, s0, ns);
}
cudaError_t oa_launch_state_plane_density(oa_ctx* c, cudaStream_t s) {
  return c->precision == OA_FP64 ? launch_plane_density<double>(c, s) : launch_plane_density<float>(c, s);
}
cudaError_t oa_launch_state_plane_vks(oa_ctx* c, cudaStream_t s) {
  return c->precision == OA_FP64 ? launch_plane_vks<double>(c, s) : launch_plane_vks<float>(c, s);
}
cudaError_t oa_launch_state_zbwd(oa_ctx* c, cudaStream_t s, const double2* psi, const double2* fnl,
                                 double2* force, int s0, int ns) {
  return c->precision == OA_FP64 ? launch_zbwd<double>(c, s, psi, fnl, force, s0, ns)
                                 : launch_zbwd<float>(c, s, psi, fnl, force, s0, ns);
}
