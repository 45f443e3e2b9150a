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

#include "oa_state_common.cuh"

// ---------------------------------------------------------------------------
// z pass, forward: packed sphere -> zero-filled z-lines -> FFT(-) -> zbuf[s][z][l]
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(OA_NTHREADS)
k_state_zfwd(const double2* __restrict__ psi, int ng, int s0,
             const int* __restrict__ line_off, const int* __restrict__ line_nneg,
             const int* __restrict__ line_npos, int nlines,
             typename CplxOf<R>::T* __restrict__ zbuf, int nz, int ldl,
             OaFftPlan pz, const double2* __restrict__ twz, const double2* __restrict__ dyp) {
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
      double2 v = ps[off + i];
      if (dyp) {  // EES projector: projPsiG = conj(dyp psi) (eesProjGchare)
        const double2 d = dyp[off + i];
        v = make_double2(d.x * v.x - d.y * v.y, -(d.y * v.x + d.x * v.y));
      }
      a[lb * ldz + kzi] = cmk<C>(v.x, v.y);
    }
  }
  __syncthreads();
  C* r = (pz.nst & 1) ? b : a;
  for (int lb = warp; lb < nb; lb += nwarp) warp_fft_pingpong<-1>(a + lb * ldz, b + lb * ldz, ldz, 1, pz, tw, lane);
  __syncthreads();
  C* out = zbuf + (size_t)s * nz * ldl + l0;
  for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
    const int z = idx / OA_LB, lb = idx - z * OA_LB;
    if (lb < nb) out[(size_t)z * ldl + lb] = r[lb * ldz + z];
  }
}

// ---------------------------------------------------------------------------
// plane helpers
// ---------------------------------------------------------------------------
struct PlaneSmem {
  size_t tw_x, tw_y, P, tile, wbuf, total;
  int ldw;  // per-warp buffer length (complex elements)
};

// gtile: the density / V_KS plane stays in global memory (the block's own
// rho_part plane, or V_KS read in place) instead of shared memory: the
// layout of planes too large for shared memory (FP64 at 160^3)
template <typename C, typename T>
static PlaneSmem plane_smem_layout(int nx, int ny, int nkx, bool gtile = false) {
  PlaneSmem L;
  const int ldy = ny + 1;
  L.ldw = (nx > ny ? nx : ny) + 1;
  size_t o = 0;
  L.tw_x = o; o += align_up(nx * sizeof(C), 16);
  L.tw_y = o; o += align_up(ny * sizeof(C), 16);
  L.P = o; o += align_up((size_t)nkx * ldy * sizeof(C), 16);
  L.tile = o; o += gtile ? 0 : align_up((size_t)nx * ny * sizeof(T), 16);
  L.wbuf = o; o += align_up((size_t)OA_PLANE_WARPS * 2 * L.ldw * sizeof(C), 16);
  L.total = o;
  return L;
}

// ---------------------------------------------------------------------------
// plane pass for one z-plane and a group of states.  MODE 0 (density):
// zbuf row -> P[kx][y] -> y FFT(-) -> c2r x FFT(-) by row pairs -> tile +=
// occ psi(r)^2.  MODE 1 (V_KS): ... -> psi(r) * V_KS occ -> r2c x FFT(+) ->
// y FFT(+) -> zbuf row (in place).  Every pencil (a y column or an x row
// pair) is owned by one warp; stages synchronise with __syncwarp, the block
// synchronises only between the gather / y / x / y / scatter phases.
// ---------------------------------------------------------------------------
template <typename R, int MODE>
__global__ void __launch_bounds__(OA_PLANE_THREADS)
k_state_plane(typename CplxOf<R>::T* __restrict__ zbuf, int nstate, int ldl, int nlines,
              const int* __restrict__ line_kx, const int* __restrict__ line_ky,
              int nx, int ny, int nz, int nkx,
              OaFftPlan px, OaFftPlan py, const double2* __restrict__ twx, const double2* __restrict__ twy,
              const double* __restrict__ occ, const R* __restrict__ vks, double* __restrict__ rho_part,
              int ngroup, PlaneSmem L, EesArgs E, int gtile) {
  // gtile (MODE 0 / 1 with R = double): the tile is this block's rho_part
  // plane (accumulated in place; each (group, plane) belongs to one block)
  // or the V_KS plane itself
  typedef typename CplxOf<R>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* stwx = (C*)(smem_raw + L.tw_x);
  C* stwy = (C*)(smem_raw + L.tw_y);
  C* P = (C*)(smem_raw + L.P);
  R* tile = (R*)(smem_raw + L.tile);
  if (gtile) {
    if (MODE == 0) tile = (R*)(rho_part + ((size_t)blockIdx.y * nz + blockIdx.x) * (size_t)nx * ny);
    else tile = const_cast<R*>(vks) + (size_t)blockIdx.x * nx * ny;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* wa = (C*)(smem_raw + L.wbuf) + (size_t)warp * 2 * L.ldw;
  C* wb = wa + L.ldw;
  const int ldy = ny + 1, ldw = L.ldw;
  const int z = blockIdx.x, g = blockIdx.y;
  const int nper = (nstate + ngroup - 1) / ngroup;
  const int sb = g * nper, se = min(nstate, sb + nper);
  const int npairs = (ny + 1) / 2;
  load_twiddles(stwx, twx, nx);
  load_twiddles(stwy, twy, ny);
  if (MODE == 0) {
    for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) tile[i] = (R)0;
  } else if (MODE == 1 && !gtile) {
    const R* vz = vks + (size_t)z * nx * ny;
    for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) tile[i] = vz[i];
  }
  for (int s = sb; s < se; ++s) {
    C* row = zbuf + ((size_t)s * nz + z) * ldl;
    if (MODE == 3) {
      // scatter Z M onto this plane (eesEnergyAtmForcRchare: projPsiRScr[igrid] += z Mn)
      for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) tile[i] = (R)0;
      __syncthreads();
      ees_scatter_plane<R>(tile, nx, z, s, E, warp, lane, OA_PLANE_WARPS);
      __syncthreads();
    } else {
      for (int i = threadIdx.x; i < nkx * ldy; i += blockDim.x) P[i] = cmk<C>(0.0, 0.0);
      __syncthreads();
      for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
        int ky = line_ky[l]; if (ky < 0) ky += ny;
        P[line_kx[l] * ldy + ky] = row[l];
      }
      __syncthreads();
      for (int c = warp; c < nkx; c += OA_PLANE_WARPS)
        warp_fft_inout<-1>(P + c * ldy, ldy, P + c * ldy, ldy, wa, wb, ldw, 1, py, stwy, lane);
      __syncthreads();
    }
    const R o = (R)occ[s];
    for (int p = warp; p < npairs; p += OA_PLANE_WARPS) {
      const int y1 = 2 * p, y2 = y1 + 1;
      if (MODE == 3) {
        for (int x = lane; x < nx; x += 32) {
          C zz; zz.x = tile[y1 * nx + x]; zz.y = (y2 < ny) ? tile[y2 * nx + x] : (R)0;
          wa[x] = zz;
        }
        __syncwarp();
        C* r2 = warp_fft_pingpong<+1>(wa, wb, ldw, 1, px, stwx, lane);
        for (int k = lane; k < nkx; k += 32) {
          const C a = r2[k];
          const C b = cconj(r2[k == 0 ? 0 : nx - k]);
          C f1, f2;
          f1.x = (a.x + b.x) * (R)0.5; f1.y = (a.y + b.y) * (R)0.5;
          f2.x = (a.y - b.y) * (R)0.5; f2.y = -(a.x - b.x) * (R)0.5;
          P[k * ldy + y1] = f1;
          if (y2 < ny) P[k * ldy + y2] = f2;
        }
        __syncwarp();
        continue;
      }
      for (int k = lane; k < nx; k += 32) {
        const C a = herm_x(P, ldy, nkx, nx, k, y1);
        C b = cmk<C>(0.0, 0.0);
        if (y2 < ny) b = herm_x(P, ldy, nkx, nx, k, y2);
        C zz; zz.x = a.x - b.y; zz.y = a.y + b.x;
        wa[k] = zz;
      }
      __syncwarp();
      C* r = warp_fft_pingpong<-1>(wa, wb, ldw, 1, px, stwx, lane);
      if (MODE == 0) {
        for (int x = lane; x < nx; x += 32) {
          const C v = r[x];
          tile[y1 * nx + x] += o * v.x * v.x;
          if (y2 < ny) tile[y2 * nx + x] += o * v.y * v.y;
        }
        __syncwarp();
      } else if (MODE == 2) {
        for (int x = lane; x < nx; x += 32) {
          const C v = r[x];
          tile[y1 * nx + x] = v.x;
          if (y2 < ny) tile[y2 * nx + x] = v.y;
        }
        __syncwarp();
      } else {
        for (int x = lane; x < nx; x += 32) {
          C v = r[x];
          v.x *= tile[y1 * nx + x] * o;
          v.y = (y2 < ny) ? v.y * tile[y2 * nx + x] * o : (R)0;
          r[x] = v;
        }
        __syncwarp();
        C* other = (r == wa) ? wb : wa;
        C* r2 = warp_fft_pingpong<+1>(r, other, ldw, 1, px, stwx, lane);
        for (int k = lane; k < nkx; k += 32) {
          const C a = r2[k];
          const C b = cconj(r2[k == 0 ? 0 : nx - k]);
          C f1, f2;
          f1.x = (a.x + b.x) * (R)0.5; f1.y = (a.y + b.y) * (R)0.5;
          f2.x = (a.y - b.y) * (R)0.5; f2.y = -(a.x - b.x) * (R)0.5;
          P[k * ldy + y1] = f1;
          if (y2 < ny) P[k * ldy + y2] = f2;
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (MODE == 2) {
      // Z gather over the stencil points of this plane (eesZmatRchare)
      ees_gather_plane<R>(tile, nx, z, s, E, warp, lane, OA_PLANE_WARPS);
      __syncthreads();
    }
    if (MODE == 1 || MODE == 3) {
      for (int c = warp; c < nkx; c += OA_PLANE_WARPS)
        warp_fft_inout<+1>(P + c * ldy, ldy, P + c * ldy, ldy, wa, wb, ldw, 1, py, stwy, lane);
      __syncthreads();
      for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
        int ky = line_ky[l]; if (ky < 0) ky += ny;
        row[l] = P[line_kx[l] * ldy + ky];
      }
      __syncthreads();
    }
  }
  if (MODE == 0 && !gtile) {
    __syncthreads();
    double* out = rho_part + ((size_t)g * nz + z) * (size_t)nx * ny;
    for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) out[i] = (double)tile[i];
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
             double scale, double ecut, double* __restrict__ eke_part, int nblk,
             const double2* __restrict__ dyp) {
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
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  C* r = (pz.nst & 1) ? b : a;
  for (int lb = warp; lb < nb; lb += nwarp) warp_fft_pingpong<+1>(a + lb * ldz, b + lb * ldz, ldz, 1, pz, tw, lane);
  __syncthreads();
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
      if (dyp) {  // EES psi force (eesPsiForcGspace): F = -w conj(dyp P), Im P = 0 at g = 0
        const double2 d = dyp[idx];
        const double px = (double)v.x;
        const double py = (g2[idx] == 0.0) ? 0.0 : (double)v.y;
        fs[idx] = make_double2(-w * (d.x * px - d.y * py), w * (d.y * px + d.x * py));
        continue;
      }
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

// two-pass kernels (oa_pencil.cu) for the lengths with a compile-time
// factorisation; they return cudaErrorNotSupported otherwise
int oa_pencil_supported(int n);
size_t oa_pencil_plane_smem(int precision, int n, int nkx);
cudaError_t oa_pencil_zfwd(int precision, cudaStream_t st, int n, const double2* psi, int ng, int s0, int ns,
                           const int* off, const int* nneg, const int* npos, int nlines, void* zbuf, int ldl,
                           const double2* tw, const double2* dyp, int zseg, OaCharge qc, int zext);
cudaError_t oa_pencil_zbwd(int precision, cudaStream_t st, int n, const void* zbuf, int ldl, int nlines,
                           const int* lkx, const int* off, const int* nneg, const int* npos, const double2* tw,
                           const double2* psi, const double2* fnl, double2* force, const double* g2,
                           const double* occ, int ng, int s0, int ns, double scale, double ecut, double* eke_part,
                           int nblk, const double2* dyp, OaPlaneOut po, int zseg);
cudaError_t oa_pair_plane(int mode, cudaStream_t st, int n, void* zbuf, int nstate, int nz, int ldl, int nlines,
                          const int* cols, int nkx, const double2* tw, const double* occ, const void* vks,
                          double* rho_part, int ngroup, void* psir, int kymax, double* qpart);
cudaError_t oa_pencil_plane(int precision, int mode, cudaStream_t st, int n, void* zbuf, int nstate, int ldl,
                            int nlines, const int* lkx, const int* lky, int nz, int nkx, const double2* tw,
                            const double* occ, const void* vks, double* rho_part, int ngroup, const EesArgs& E,
                            void* psir);

template <typename R>
static cudaError_t launch_zfwd(oa_ctx* c, cudaStream_t st, const double2* psi, int s0, int ns) {
  typedef typename CplxOf<R>::T C;
  size_t sm = zpass_smem<R>(c->nz);
  cudaError_t e = oa_smem_limit(k_state_zfwd<R>);
  if (e != cudaSuccess) return e;
  dim3 grid((c->nlines + OA_LB - 1) / OA_LB, ns);
  k_state_zfwd<R><<<grid, OA_NTHREADS, sm, st>>>(psi, c->ng, s0, c->line_off, c->line_nneg, c->line_npos,
                                                  c->nlines, (C*)c->zbuf, c->nz, c->ldl, c->plan_z, c->tw_z, nullptr);
  return cudaGetLastError();
}

template <typename R, int MODE>
static cudaError_t launch_plane(oa_ctx* c, cudaStream_t st) {
  typedef typename CplxOf<R>::T C;
  PlaneSmem L = plane_smem_layout<C, R>(c->nx, c->ny, c->nkx_s);
  // FP64 planes beyond shared memory: the tile in global memory
  const int gtile = (L.total > (size_t)OA_MAX_SMEM && sizeof(R) == 8) ? 1 : 0;
  if (gtile) L = plane_smem_layout<C, R>(c->nx, c->ny, c->nkx_s, true);
  if (L.total > (size_t)OA_MAX_SMEM) return cudaErrorNotSupported;
  cudaError_t e = oa_smem_limit(k_state_plane<R, MODE>);
  if (e != cudaSuccess) return e;
  dim3 grid(c->nz, c->ngroup);
  EesArgs E = {nullptr, nullptr, nullptr, nullptr, 0, 0};
  k_state_plane<R, MODE><<<grid, OA_PLANE_THREADS, L.total, st>>>(
      (C*)c->zbuf, c->nstate, c->ldl, c->nlines, c->line_kx, c->line_ky, c->nx, c->ny, c->nz, c->nkx_s,
      c->plan_x, c->plan_y, c->tw_x, c->tw_y, c->occ, (const R*)c->vks, c->rho_part, c->ngroup, L, E, gtile);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_zbwd(oa_ctx* c, cudaStream_t st, const double2* psi, const double2* fnl,
                               double2* force, int s0, int ns) {
  typedef typename CplxOf<R>::T C;
  size_t sm = zpass_smem<R>(c->nz);
  cudaError_t e = oa_smem_limit(k_state_zbwd<R>);
  if (e != cudaSuccess) return e;
  dim3 grid(c->nblk_z, ns);
  k_state_zbwd<R><<<grid, OA_NTHREADS, sm, st>>>(
      (const C*)c->zbuf, c->nz, c->ldl, c->nlines, c->line_kx, c->line_off, c->line_nneg, c->line_npos,
      c->plan_z, c->tw_z, psi, fnl, force, c->g2, c->occ, c->ng, s0, -2.0 / (double)c->npts,
      c->ecut_psi, c->eke_part, c->nblk_z, nullptr);
  return cudaGetLastError();
}

size_t oa_plane_smem_bytes(int precision, int nx, int ny, int nkx) {
  if (nx == ny && oa_pencil_supported(nx)) {
    const size_t p = oa_pencil_plane_smem(precision, nx, nkx);
    if (p > 0 && p <= (size_t)OA_MAX_SMEM) return p;
  }
  if (precision == OA_FP64) {
    const size_t t = plane_smem_layout<double2, double>(nx, ny, nkx).total;
    return t <= (size_t)OA_MAX_SMEM ? t : plane_smem_layout<double2, double>(nx, ny, nkx, true).total;
  }
  return plane_smem_layout<float2, float>(nx, ny, nkx).total;
}

int oa_plane_blocks_per_sm(int precision) {
  int n = 0;
  if (precision == OA_FP64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_state_plane<double, 1>, OA_PLANE_THREADS, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_state_plane<float, 1>, OA_PLANE_THREADS, 0);
  return n;
}

cudaError_t oa_launch_state_zfwd(oa_ctx* c, cudaStream_t s, const double2* psi, int s0, int ns) {
  if (!c->fft_runtime && oa_pencil_supported(c->nz)) {
    // mixed form, all states: the exact charge partials for the density
    // renormalisation ride along
    OaCharge qc = {nullptr, nullptr, nullptr};
    if (c->qpart && s0 == 0 && ns == c->nstate) qc = OaCharge{c->line_kx, c->occ, c->qpart};
    c->qvalid = qc.part ? 1 : 0;
    return oa_pencil_zfwd(c->precision, s, c->nz, psi, c->ng, s0, ns, c->line_off, c->line_nneg, c->line_npos,
                          c->nlines, c->zbuf, c->ldl, c->tw_z, nullptr, c->zseg, qc, c->z_ext);
  }
  c->qvalid = 0;
  return c->precision == OA_FP64 ? launch_zfwd<double>(c, s, psi, s0, ns) : launch_zfwd<float>(c, s, psi, s0, ns);
}
static cudaError_t pencil_plane(oa_ctx* c, cudaStream_t s, int mode, void* psir) {
  if (c->fft_runtime || c->nx != c->ny || !oa_pencil_supported(c->nx)) return cudaErrorNotSupported;
  const EesArgs E = {nullptr, nullptr, nullptr, nullptr, 0, 0};
  return oa_pencil_plane(c->precision, mode, s, c->nx, c->zbuf, c->nstate, c->ldl, c->nlines, c->line_kx,
                         c->line_ky, c->nz, c->nkx_s, c->tw_x, c->occ, c->vks, c->rho_part, c->ngroup, E, psir);
}

// The density pass also stores psi(r) (c->psir) when the two-pass kernels
// run; the V_KS pass then starts from it (MODE 4) instead of redoing the
// forward y and x transforms.  c->psir_valid marks that the last density
// pass stored it.
// In the mixed form with the state-pair kernels (c->pair_cols set) both
// passes run two states per x transform and psi(r) is stored per pair
// (psir_valid 2).
cudaError_t oa_launch_state_plane_density(oa_ctx* c, cudaStream_t s) {
  if (c->pair_cols && c->psir) {
    const cudaError_t e = oa_pair_plane(0, s, c->nx, c->zbuf, c->nstate, c->nz, c->ldl, c->nlines, c->pair_cols,
                                        c->nkx_s, c->tw_x, c->occ, nullptr, c->rho_part, c->ngroup_pair, c->psir,
                                        c->pair_kymax, c->qvalid ? c->qpart2 : nullptr);
    c->psir_valid = e == cudaSuccess ? 2 : 0;
    if (e == cudaSuccess && c->qvalid) c->qvalid = 2;
    c->rho_ngroup = c->ngroup_pair;
    if (e != cudaErrorNotSupported) return e;
  }
  c->rho_ngroup = c->ngroup;
  const cudaError_t e = pencil_plane(c, s, 0, c->psir);
  c->psir_valid = (e == cudaSuccess && c->psir) ? 1 : 0;
  if (e != cudaErrorNotSupported) return e;
  return c->precision == OA_FP64 ? launch_plane<double, 0>(c, s) : launch_plane<float, 0>(c, s);
}
cudaError_t oa_launch_state_plane_vks(oa_ctx* c, cudaStream_t s) {
  if (c->psir_valid == 2)
    return oa_pair_plane(4, s, c->nx, c->zbuf, c->nstate, c->nz, c->ldl, c->nlines, c->pair_cols, c->nkx_s,
                         c->tw_x, c->occ, c->vks, nullptr, c->ngroup_pair, c->psir, c->pair_kymax, nullptr);
  const cudaError_t e = c->psir_valid ? pencil_plane(c, s, 4, c->psir) : pencil_plane(c, s, 1, nullptr);
  if (e != cudaErrorNotSupported) return e;
  return c->precision == OA_FP64 ? launch_plane<double, 1>(c, s) : launch_plane<float, 1>(c, s);
}
cudaError_t oa_launch_state_zbwd(oa_ctx* c, cudaStream_t s, const double2* psi, const double2* fnl,
                                 double2* force, int s0, int ns) {
  c->zb_po_done = 0;
  if (!c->fft_runtime && oa_pencil_supported(c->nz)) {
    const cudaError_t e = oa_pencil_zbwd(c->precision, s, c->nz, c->zbuf, c->ldl, c->nlines, c->line_kx,
                                         c->line_off, c->line_nneg, c->line_npos, c->tw_z, psi, fnl, force, c->g2,
                                         c->occ, c->ng, s0, ns, -2.0 / (double)c->npts, c->ecut_psi, c->eke_part,
                                         c->nblk_z, nullptr, c->zb_po, c->zseg);
    c->zb_po_done = (e == cudaSuccess && c->zb_po.P) ? 1 : 0;
    return e;
  }
  return c->precision == OA_FP64 ? launch_zbwd<double>(c, s, psi, fnl, force, s0, ns)
                                 : launch_zbwd<float>(c, s, psi, fnl, force, s0, ns);
}

// ---------------------------------------------------------------------------
// EES nonlocal path on the nonlocal grid (na, nb, nc)
// ---------------------------------------------------------------------------
template <typename R>
static cudaError_t launch_ees(oa_ctx* c, cudaStream_t st, const double2* psi, double2* fnl) {
  typedef typename CplxOf<R>::T C;
  oa_ees* e = c->ees;
  cudaError_t err;
  const bool pz = !c->fft_runtime && oa_pencil_supported(e->nc) != 0;
  // z pass forward with conj(dyp psi)
  if (pz) {
    err = oa_pencil_zfwd(c->precision, st, e->nc, psi, c->ng, 0, c->nstate, c->line_off, c->line_nneg, c->line_npos,
                         c->nlines, e->zbuf, c->ldl, e->tw_c, e->dyp, c->zseg, OaCharge{nullptr, nullptr, nullptr}, c->z_ext);
    if (err != cudaSuccess) return err;
  } else {
    size_t sm = zpass_smem<R>(e->nc);
    err = oa_smem_limit(k_state_zfwd<R>);
    if (err != cudaSuccess) return err;
    dim3 grid((c->nlines + OA_LB - 1) / OA_LB, c->nstate);
    k_state_zfwd<R><<<grid, OA_NTHREADS, sm, st>>>(psi, c->ng, 0, c->line_off, c->line_nneg, c->line_npos, c->nlines,
                                                    (C*)e->zbuf, e->nc, c->ldl, e->pc, e->tw_c, e->dyp);
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
  }
  PlaneSmem L = plane_smem_layout<C, R>(e->na, e->nb, c->nkx_s);
  EesArgs E = {e->idx, e->mn, e->zpart, e->zs, c->natm_nl, e->order, e->dmn, c->ions ? e->fpart : nullptr};
  dim3 pgrid(e->nc, e->ngroup);
  const bool pp = !c->fft_runtime && e->na == e->nb && oa_pencil_supported(e->na);
  err = cudaErrorNotSupported;
  if (pp)
    err = oa_pencil_plane(c->precision, 2, st, e->na, e->zbuf, c->nstate, c->ldl, c->nlines, c->line_kx, c->line_ky,
                          e->nc, c->nkx_s, e->tw_a, c->occ, nullptr, nullptr, e->ngroup, E, nullptr);
  if (err == cudaErrorNotSupported) {
    err = oa_smem_limit(k_state_plane<R, 2>);
    if (err != cudaSuccess) return err;
    k_state_plane<R, 2><<<pgrid, OA_PLANE_THREADS, L.total, st>>>(
        (C*)e->zbuf, c->nstate, c->ldl, c->nlines, c->line_kx, c->line_ky, e->na, e->nb, e->nc, c->nkx_s, e->pa,
        e->pb, e->tw_a, e->tw_b, c->occ, nullptr, nullptr, e->ngroup, L, E, 0);
    err = cudaGetLastError();
  }
  if (err != cudaSuccess) return err;
  err = oa_launch_ees_zreduce(c, st);
  if (err != cudaSuccess) return err;
  // with ion dynamics: the nonlocal atom forces from the gathered sums and zs
  if (c->ions && (err = oa_launch_ees_atom_force(c, st)) != cudaSuccess) return err;
  err = cudaErrorNotSupported;
  if (pp)
    err = oa_pencil_plane(c->precision, 3, st, e->na, e->zbuf, c->nstate, c->ldl, c->nlines, c->line_kx, c->line_ky,
                          e->nc, c->nkx_s, e->tw_a, c->occ, nullptr, nullptr, e->ngroup, E, nullptr);
  if (err == cudaErrorNotSupported) {
    err = oa_smem_limit(k_state_plane<R, 3>);
    if (err != cudaSuccess) return err;
    k_state_plane<R, 3><<<pgrid, OA_PLANE_THREADS, L.total, st>>>(
        (C*)e->zbuf, c->nstate, c->ldl, c->nlines, c->line_kx, c->line_ky, e->na, e->nb, e->nc, c->nkx_s, e->pa,
        e->pb, e->tw_a, e->tw_b, c->occ, nullptr, nullptr, e->ngroup, L, E, 0);
    err = cudaGetLastError();
  }
  if (err != cudaSuccess) return err;
  if (pz)
    return oa_pencil_zbwd(c->precision, st, e->nc, e->zbuf, c->ldl, c->nlines, c->line_kx, c->line_off,
                          c->line_nneg, c->line_npos, e->tw_c, psi, nullptr, fnl, c->g2, c->occ, c->ng, 0, c->nstate,
                          1.0, c->ecut_psi, c->eke_part, c->nblk_z, e->dyp, OaPlaneOut{nullptr, 0, 0, 0}, 0);
  {
    size_t sm = zpass_smem<R>(e->nc);
    err = oa_smem_limit(k_state_zbwd<R>);
    if (err != cudaSuccess) return err;
    dim3 grid(c->nblk_z, c->nstate);
    k_state_zbwd<R><<<grid, OA_NTHREADS, sm, st>>>(
        (const C*)e->zbuf, e->nc, c->ldl, c->nlines, c->line_kx, c->line_off, c->line_nneg, c->line_npos, e->pc,
        e->tw_c, psi, nullptr, fnl, c->g2, c->occ, c->ng, 0, 1.0, c->ecut_psi, c->eke_part, c->nblk_z, e->dyp);
  }
  return cudaGetLastError();
}

cudaError_t oa_launch_ees(oa_ctx* c, cudaStream_t s, const double2* psi, double2* fnl) {
  return c->precision == OA_FP64 ? launch_ees<double>(c, s, psi, fnl) : launch_ees<float>(c, s, psi, fnl);
}

size_t oa_ees_plane_smem(int precision, int na, int nb, int nkx) { return oa_plane_smem_bytes(precision, na, nb, nkx); }
