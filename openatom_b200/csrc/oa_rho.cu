// Density -> V_KS(r) on one GPU (FP64 in both precision forms; it is one
// grid per step against 2 N_state state transforms).
//
// Replaces:
//   CP_Rho_RealSpacePlane::acceptDensity/handleDensityReduction (CP_Rho_RealSpacePlane.C:398-520)
//     sum of state-group partial densities, probScale = 1/V         -> k_rho_xc
//   CPXCFNCTS::CP_exc_calc (cp_pz_lda.C:23-175), energyComputation (:739) -> k_rho_xc
//   fftRhoRtoRhoG (:831) + Charm forward FFT, rho * volumeFactor   -> k_rho_plane_fwd + k_rho_zpass
//   CP_Rho_GHartExt::HartExtVksG (CP_Rho_GHartExt.C:461) ->
//     CPLOCAL::CP_hart_eext_calc (cp_hart_ext.C:56-431)             -> k_rho_zpass
//   FFTVks (CP_Rho_GHartExt.C:532) + acceptHartVks (CP_Rho_RealSpacePlane.C:1365) -> k_rho_zpass + k_rho_plane_bwd
// Charm-FFT's sign convention is not in the tree; forward exp(-i g.r) and
// backward exp(+i g.r) are the ones under which the e^{+i g.R} structure
// factor of cp_hart_ext.C gives E_ext = integral rho V_loc.
#include "oa_internal.h"
#include "oa_rdft.cuh"

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block sum of NV doubles; results in out[] of thread 0
template <int NV>
__device__ void block_sum_n(double* v, double* sh /* 32*NV */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum_d(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k * 32 + wid] = v[k];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double r = (lane < nw) ? sh[k * 32 + lane] : 0.0;
      v[k] = warp_sum_d(r);
    }
  }
}

__host__ __device__ static inline size_t align_up_r(size_t x, size_t a) { return (x + a - 1) / a * a; }

// ---------------------------------------------------------------------------
// density sum + PZ-LDA
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(OA_NTHREADS)
k_rho_xc(const double* __restrict__ rho_part, int ngroup, size_t npts, double rvol,
         double* __restrict__ rho, double* __restrict__ vxc, double* __restrict__ part) {
  __shared__ double sh[3 * 32];
  // Perdew-Zunger constants (cp_pz_lda.C:46-52)
  const double gamma = -0.14230, beta1 = 1.05290, beta2 = 0.33340;
  const double au = 0.03110, bu = -0.0480, cu = 0.00200, du = -0.01160;
  const double power = 1.0 / 3.0;
  const double rat1 = (7.0 / 6.0) * beta1, rat2 = (4.0 / 3.0) * beta2;
  const double pi = 3.14159265358979323846, fpi = 4.0 * pi;
  double acc[3] = {0.0, 0.0, 0.0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (size_t)gridDim.x * blockDim.x) {
    double r = 0.0;
    for (int g = 0; g < ngroup; ++g) r += rho_part[(size_t)g * npts + i];
    r *= rvol;
    rho[i] = r;
    const double fpin = fpi * r;
    const double rs = pow(3.0 / fpin, power);
    const double sqtrs = sqrt(rs);
    const double xfact = -pow(3.0 * r / pi, power);
    double cfact, mufact;
    if (rs >= 1.0) {
      const double cf1 = 1.0 + beta1 * sqtrs + beta2 * rs;
      const double cf2 = 1.0 + rat1 * sqtrs + rat2 * rs;
      cfact = gamma / cf1;
      mufact = cfact * (cf2 / cf1);
    } else {
      const double lnrs = log(rs);
      cfact = au * lnrs + bu + cu * rs * lnrs + du * rs;
      mufact = au * lnrs + (bu - power * au) + 2.0 * power * cu * rs * lnrs + power * (2.0 * du - cu) * rs;
    }
    acc[0] += xfact * r;
    acc[1] += cfact * r;
    const double v = xfact + mufact;
    acc[2] += v * r;
    vxc[i] = v;
  }
  block_sum_n<3>(acc, sh);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 0] = acc[0];
    part[3 * blockIdx.x + 1] = acc[1];
    part[3 * blockIdx.x + 2] = acc[2];
  }
}

// ---------------------------------------------------------------------------
// plane helpers for the dense density grid (nkx = nx/2 + 1 columns)
// ---------------------------------------------------------------------------
template <typename C>
__device__ __forceinline__ C herm_xd(const C* P, int ldy, int nkx, int nx, int k, int y) {
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

struct RhoPlaneSmem { size_t tw_x, tw_y, P, W1, W2, total; };

static RhoPlaneSmem rho_plane_layout(int nx, int ny, int nkx, int npair, int ychunk) {
  RhoPlaneSmem L;
  const int ldx = nx + 1, ldy = ny + 1;
  size_t o = 0;
  L.tw_x = o; o += align_up_r(nx * sizeof(double2), 16);
  L.tw_y = o; o += align_up_r(ny * sizeof(double2), 16);
  L.P = o; o += align_up_r((size_t)nkx * ldy * sizeof(double2), 16);
  size_t wsz = (size_t)npair * ldx;
  if ((size_t)ychunk * ldy > wsz) wsz = (size_t)ychunk * ldy;
  L.W1 = o; o += align_up_r(wsz * sizeof(double2), 16);
  L.W2 = o; o += align_up_r(wsz * sizeof(double2), 16);
  L.total = o;
  return L;
}

// forward: rho(x,y,z) * V/N -> r2c x (-) by row pairs -> y FFT (-) -> dz[z][k*ny+y]
__global__ void __launch_bounds__(OA_NTHREADS)
k_rho_plane_fwd(const double* __restrict__ rho, double scale, int nx, int ny, int nz, int nkx,
                OaFftPlan px, OaFftPlan py, const double2* __restrict__ twx, const double2* __restrict__ twy,
                double2* __restrict__ dz, int ldl_d, int npair, int ychunk, RhoPlaneSmem L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* stwx = (double2*)(smem_raw + L.tw_x);
  double2* stwy = (double2*)(smem_raw + L.tw_y);
  double2* P = (double2*)(smem_raw + L.P);
  double2* W1 = (double2*)(smem_raw + L.W1);
  double2* W2 = (double2*)(smem_raw + L.W2);
  const int ldx = nx + 1, ldy = ny + 1;
  const int z = blockIdx.x;
  const int npairs = (ny + 1) / 2;
  load_twiddles(stwx, twx, nx);
  load_twiddles(stwy, twy, ny);
  const double* rz = rho + (size_t)z * nx * ny;
  for (int p0 = 0; p0 < npairs; p0 += npair) {
    const int np = min(npair, npairs - p0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < np * nx; idx += blockDim.x) {
      const int p = idx / nx, x = idx - p * nx;
      const int y1 = 2 * (p0 + p), y2 = y1 + 1;
      W1[p * ldx + x] = make_double2(rz[y1 * nx + x] * scale, (y2 < ny) ? rz[y2 * nx + x] * scale : 0.0);
    }
    __syncthreads();
    double2* r = fft_pingpong<-1>(W1, W2, ldx, np, px, stwx);
    for (int idx = threadIdx.x; idx < np * nkx; idx += blockDim.x) {
      const int p = idx / nkx, k = idx - p * nkx;
      const int y1 = 2 * (p0 + p), y2 = y1 + 1;
      const double2 a = r[p * ldx + k];
      const double2 b = cconj(r[p * ldx + (k == 0 ? 0 : nx - k)]);
      P[k * ldy + y1] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
      if (y2 < ny) P[k * ldy + y2] = make_double2(0.5 * (a.y - b.y), -0.5 * (a.x - b.x));
    }
  }
  __syncthreads();
  for (int c0 = 0; c0 < nkx; c0 += ychunk) {
    const int nb = min(ychunk, nkx - c0);
    fft_inout<-1>(P + c0 * ldy, ldy, P + c0 * ldy, ldy, W1, W2, ldy, nb, py, stwy);
  }
  double2* out = dz + (size_t)z * ldl_d;
  for (int idx = threadIdx.x; idx < nkx * ny; idx += blockDim.x) {
    const int k = idx / ny, y = idx - k * ny;
    out[idx] = P[k * ldy + y];
  }
}

// backward: dz[z][k*ny+y] -> y FFT (+) -> c2r x (+) -> vks = V + vxc
template <typename R>
__global__ void __launch_bounds__(OA_NTHREADS)
k_rho_plane_bwd(const double2* __restrict__ dz, int ldl_d, int nx, int ny, int nz, int nkx,
                OaFftPlan px, OaFftPlan py, const double2* __restrict__ twx, const double2* __restrict__ twy,
                const double* __restrict__ vxc, R* __restrict__ vks, int npair, int ychunk, RhoPlaneSmem L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* stwx = (double2*)(smem_raw + L.tw_x);
  double2* stwy = (double2*)(smem_raw + L.tw_y);
  double2* P = (double2*)(smem_raw + L.P);
  double2* W1 = (double2*)(smem_raw + L.W1);
  double2* W2 = (double2*)(smem_raw + L.W2);
  const int ldx = nx + 1, ldy = ny + 1;
  const int z = blockIdx.x;
  const int npairs = (ny + 1) / 2;
  load_twiddles(stwx, twx, nx);
  load_twiddles(stwy, twy, ny);
  const double2* in = dz + (size_t)z * ldl_d;
  for (int idx = threadIdx.x; idx < nkx * ny; idx += blockDim.x) {
    const int k = idx / ny, y = idx - k * ny;
    P[k * ldy + y] = in[idx];
  }
  __syncthreads();
  for (int c0 = 0; c0 < nkx; c0 += ychunk) {
    const int nb = min(ychunk, nkx - c0);
    fft_inout<+1>(P + c0 * ldy, ldy, P + c0 * ldy, ldy, W1, W2, ldy, nb, py, stwy);
  }
  const double* vz = vxc + (size_t)z * nx * ny;
  R* oz = vks + (size_t)z * nx * ny;
  for (int p0 = 0; p0 < npairs; p0 += npair) {
    const int np = min(npair, npairs - p0);
    for (int idx = threadIdx.x; idx < np * nx; idx += blockDim.x) {
      const int p = idx / nx, k = idx - p * nx;
      const int y1 = 2 * (p0 + p), y2 = y1 + 1;
      const double2 a = herm_xd(P, ldy, nkx, nx, k, y1);
      double2 b = make_double2(0.0, 0.0);
      if (y2 < ny) b = herm_xd(P, ldy, nkx, nx, k, y2);
      W1[p * ldx + k] = make_double2(a.x - b.y, a.y + b.x);
    }
    __syncthreads();
    double2* r = fft_pingpong<+1>(W1, W2, ldx, np, px, stwx);
    for (int idx = threadIdx.x; idx < np * nx; idx += blockDim.x) {
      const int p = idx / nx, x = idx - p * nx;
      const int y1 = 2 * (p0 + p), y2 = y1 + 1;
      const double2 v = r[p * ldx + x];
      oz[y1 * nx + x] = (R)(v.x + vz[y1 * nx + x]);
      if (y2 < ny) oz[y2 * nx + x] = (R)(v.y + vz[y2 * nx + x]);
    }
    __syncthreads();
  }
}

struct RhoTypeOff { int off[5]; };

// z pass: FFT(-) -> Hartree + local pseudopotential + Ewald (recip) in G -> FFT(+)
// The structure factor S_t(g) = sum_{a in t} e^{i g.R_a} factorises per
// z-line: pxy[line][a] = e^{i (gx x_a + gy y_a)} is formed once per block in
// shared memory (atoms grouped by type), and each g of the line multiplies
// it by the z phase e^{i gz z_a}.
// In-place z transform of nb lines a[line][z] (row stride ld) for the
// lengths with a compile-time factorisation N = N1 N2 (oa_rdft.cuh): pass A
// (lines fastest) into b [line][k1][n2], pass B back to natural order in a.
template <int N1, int N2> struct ZLd {
  static constexpr int LS = N2 | 1;
  static constexpr int PS = (N1 * LS) | 1;
};
template <int N1, int N2, int SIGN>
__device__ void zfft2(double2* a, double2* b, int ld, int nb, const double2* tw) {
  typedef ZLd<N1, N2> L;
  for (int i = threadIdx.x; i < N2 * nb; i += blockDim.x) {
    const int n2 = i / nb, lb = i - n2 * nb;
    double2 u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) u[n1] = a[lb * ld + N2 * n1 + n2];
    pass_a<N1, N2, SIGN>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) b[lb * L::PS + k1 * L::LS + n2] = u[k1];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 16 * nb; i += blockDim.x) {
    const int lb = i >> 4, k1 = i & 15;
    if (k1 >= N1) continue;
    double2 w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = b[lb * L::PS + k1 * L::LS + n2];
    RDft<N2, SIGN>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) a[lb * ld + k1 + N1 * k2] = w[k2];
  }
  __syncthreads();
}

template <int N1, int N2>
__global__ void __launch_bounds__(OA_NTHREADS, 2)
k_rho_zpass(double2* __restrict__ dz, int ldl_d, int nlines_d, int nx, int ny, int nz,
            OaFftPlan pz, const double2* __restrict__ twz,
            double tpi_l, double vol, double ecut4, double falp2, double gz_term,
            int natm, int ntype, const int* __restrict__ atm_perm, RhoTypeOff toff,
            const double* __restrict__ q_type, const double2* __restrict__ phase, int ktab,
            const double* __restrict__ spl, int nspl, double gmin, double dg,
            double* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ldz = nz + 1;
  constexpr bool TP = N1 > 0;  // two-pass compile-time transforms
  const int ldb = TP ? (ZLd<N1, N2>::PS > ldz ? ZLd<N1, N2>::PS : ldz) : ldz;
  double2* tw = (double2*)smem_raw;
  double2* a = tw + align_up_r(nz, 2);
  double2* b = a + OA_LB * ldz;
  double2* pxy = b + OA_LB * ldb;  // [OA_LB][natm], atoms in type order
  __shared__ double sh[3 * 32];
  const int l0 = blockIdx.x * OA_LB;
  const int nb = min(OA_LB, nlines_d - l0);
  const int nt = 2 * ktab + 1;
  load_twiddles(tw, twz, nz);
  int* zoff = (int*)(pxy + OA_LB * natm);  // [natm]: z-phase row of atom ia (type order)
  for (int ia = threadIdx.x; ia < natm; ia += blockDim.x) zoff[ia] = (atm_perm[ia] * 3 + 2) * nt + ktab;
  for (int idx = threadIdx.x; idx < OA_LB * natm; idx += blockDim.x) {
    const int lb = idx / natm, ia = idx - lb * natm;
    const int l = l0 + lb;
    const int kx = l / ny;
    int ky = l - kx * ny; if (2 * ky >= ny) ky -= ny;
    double2 v = make_double2(0.0, 0.0);
    if (lb < nb && kx <= ktab && abs(ky) <= ktab) {
      const double2* ph = phase + (size_t)atm_perm[ia] * 3 * nt;
      v = cmul(ph[kx + ktab], ph[nt + ky + ktab]);
    }
    pxy[lb * natm + ia] = v;
  }
  for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
    const int zz = idx / OA_LB, lb = idx - zz * OA_LB;
    if (lb < nb) a[lb * ldz + zz] = dz[(size_t)zz * ldl_d + l0 + lb];
  }
  __syncthreads();
  double2* r;
  if constexpr (TP) {
    zfft2<N1, N2, -1>(a, b, ldz, nb, tw);
    r = a;
  } else {
    r = fft_pingpong<-1>(a, b, ldz, nb, pz, tw);
  }
  const double pi = 3.14159265358979323846;
  const double fpi = 4.0 * pi;
  double acc[3] = {0.0, 0.0, 0.0};
  // One thread per (z, group of ZP_L lines): every z-phase load of the atom
  // sums serves ZP_L g-points (the z phase depends on kz and the atom only),
  // and the atoms' z-phase rows are addressed through zoff in shared memory.
  constexpr int ZP_L = 2;
  const int ngrp = (nb + ZP_L - 1) / ZP_L;
  for (int idx = threadIdx.x; idx < ngrp * nz; idx += blockDim.x) {
    const int grp = idx / nz, zz = idx - grp * nz;
    int kz = zz; if (2 * kz >= nz) kz -= nz;
    const double gzv = tpi_l * kz;
    double2 rho[ZP_L], sf_q[ZP_L], vext[ZP_L];
    double g2v[ZP_L], hh[ZP_L], wn[ZP_L];
    int cls[ZP_L], ii[ZP_L];  // cls: 0 outside, 1 g = 0, 2 inside the density sphere
    bool any = false;
#pragma unroll
    for (int j = 0; j < ZP_L; ++j) {
      const int lb = grp * ZP_L + j;
      cls[j] = 0; ii[j] = 1; hh[j] = 0.0; wn[j] = 1.0; g2v[j] = 0.0;
      rho[j] = make_double2(0.0, 0.0);
      sf_q[j] = make_double2(0.0, 0.0);
      vext[j] = make_double2(0.0, 0.0);
      if (lb >= nb) continue;
      const int l = l0 + lb;
      const int kx = l / ny;
      int ky = l - kx * ny; if (2 * ky >= ny) ky -= ny;
      const double gx = tpi_l * kx, gy = tpi_l * ky;
      const double g2 = gx * gx + gy * gy + gzv * gzv;
      g2v[j] = g2;
      rho[j] = r[lb * ldz + zz];
      if (g2 == 0.0) {
        cls[j] = 1;
      } else if (g2 <= ecut4 && abs(kx) <= ktab && abs(ky) <= ktab && abs(kz) <= ktab) {
        cls[j] = 2;
        any = true;
        wn[j] = (kx == 0) ? 1.0 : 2.0;
        // spline interval of the local pseudopotential (CP_get_vpsnow, cp_hart_ext.C:433-480)
        const double g = sqrt(g2);
        int i1 = (int)((g - gmin) / dg + 1.0);
        i1 = min(i1, nspl); i1 = max(i1, 1);
        ii[j] = i1;
        hh[j] = g - ((double)(i1 - 1) * dg + gmin);
      }
    }
    if (any) {
      // structure factors per type, S_t(g) = sum_{a in t} pxy[line][a] e^{i gz z_a},
      // then V_ext = sum_t S_t v_t(|g|) / V and the Ewald charge sum sum_t q_t S_t
      for (int t = 0; t < ntype && t < 4; ++t) {
        double2 st[ZP_L];
#pragma unroll
        for (int j = 0; j < ZP_L; ++j) st[j] = make_double2(0.0, 0.0);
        const double2* pl = pxy + grp * ZP_L * natm;
        for (int ia = toff.off[t]; ia < toff.off[t + 1]; ++ia) {
          const double2 hz = phase[zoff[ia] + kz];
#pragma unroll
          for (int j = 0; j < ZP_L; ++j) {
            const double2 h = cmul(pl[j * natm + ia], hz);
            st[j].x += h.x; st[j].y += h.y;
          }
        }
        const double qa = q_type[t];
#pragma unroll
        for (int j = 0; j < ZP_L; ++j) {
          if (cls[j] != 2) continue;
          sf_q[j].x += qa * st[j].x; sf_q[j].y += qa * st[j].y;
          const double* cc = spl + ((size_t)t * nspl + (ii[j] - 1)) * 4;
          const double vt = (((cc[3] * hh[j] + cc[2]) * hh[j] + cc[1]) * hh[j] + cc[0]) / vol;
          vext[j].x += st[j].x * vt; vext[j].y += st[j].y * vt;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < ZP_L; ++j) {
      const int lb = grp * ZP_L + j;
      if (lb >= nb) continue;
      double2 out = make_double2(0.0, 0.0);
      if (cls[j] == 1) {
        out.x = gz_term;
        acc[1] += gz_term * rho[j].x;
      } else if (cls[j] == 2) {
        const double g2 = g2v[j];
        const double hf = fpi / (g2 * vol);
        acc[0] += hf * (rho[j].x * rho[j].x + rho[j].y * rho[j].y) * wn[j];
        out.x = rho[j].x * hf; out.y = rho[j].y * hf;
        const double ewf = fpi * exp(-g2 / falp2) / (g2 * vol);
        acc[2] += ewf * (sf_q[j].x * sf_q[j].x + sf_q[j].y * sf_q[j].y) * wn[j];
        out.x += vext[j].x; out.y -= vext[j].y;            // vks += conj(vext)
        acc[1] += (rho[j].x * vext[j].x - rho[j].y * vext[j].y) * wn[j];  // Re(rho vext)
      }
      r[lb * ldz + zz] = out;
    }
  }
  __syncthreads();
  double2* r2;
  if constexpr (TP) {
    zfft2<N1, N2, +1>(a, b, ldz, nb, tw);
    r2 = a;
  } else {
    double2* other = (r == a) ? b : a;
    r2 = fft_pingpong<+1>(r, other, ldz, nb, pz, tw);
  }
  for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
    const int zz = idx / OA_LB, lb = idx - zz * OA_LB;
    if (lb < nb) dz[(size_t)zz * ldl_d + l0 + lb] = r2[lb * ldz + zz];
  }
  block_sum_n<3>(acc, sh);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 0] = acc[0];
    part[3 * blockIdx.x + 1] = acc[1];
    part[3 * blockIdx.x + 2] = acc[2];
  }
}

cudaError_t oa_rho2_fwd(cudaStream_t s, int n, int nz, const double* rho, double scale, const double2* tw,
                        double2* dz, int ldl_d);
cudaError_t oa_rho2_bwd(cudaStream_t s, int n, int nz, const double2* dz, int ldl_d, const double2* tw,
                        const double* vxc, void* vks, int fp64);

__global__ void k_phase_tables(const double* __restrict__ pos, int natm, int ktab, double tpi_l, double2* __restrict__ phase) {
  const int nt = 2 * ktab + 1;
  const int total = natm * 3 * nt;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int k = i % nt - ktab;
    const int ax = (i / nt) % 3;
    const int at = i / (3 * nt);
    double sn, cs;
    sincos(tpi_l * (double)k * pos[at * 3 + ax], &sn, &cs);
    phase[i] = make_double2(cs, sn);
  }
}

// ---------------------------------------------------------------------------
size_t oa_rho_plane_smem_bytes(int nx, int ny, int nkx, int npair, int ychunk) {
  return rho_plane_layout(nx, ny, nkx, npair, ychunk).total;
}

cudaError_t oa_launch_rho_xc(oa_ctx* c, cudaStream_t s) {
  const int nblk = 4 * 148;
  k_rho_xc<<<nblk, OA_NTHREADS, 0, s>>>(c->rho_part, c->rho_ngroup, (size_t)c->npts, 1.0 / c->vol, c->rho, c->vxc, c->red);
  return cudaGetLastError();
}

int oa_rho_xc_nblk() { return 4 * 148; }
int oa_rho_z_nblk(const oa_ctx* c) { return (c->nlines_d + OA_LB - 1) / OA_LB; }

cudaError_t oa_launch_phase_tables(oa_ctx* c, cudaStream_t s) {
  const double tpi_l = 2.0 * 3.14159265358979323846 / c->box;
  const int total = c->natm * 3 * (2 * c->kmax_tab + 1);
  k_phase_tables<<<(total + 255) / 256, 256, 0, s>>>(c->pos, c->natm, c->kmax_tab, tpi_l, c->phase);
  return cudaGetLastError();
}

cudaError_t oa_launch_rho_fft_hart(oa_ctx* c, cudaStream_t s) {
  const double tpi_l = 2.0 * 3.14159265358979323846 / c->box;
  cudaError_t e;
  // phase tables exp(i 2 pi k x / L)
  if ((e = oa_launch_phase_tables(c, s)) != cudaSuccess) return e;
  RhoPlaneSmem L = rho_plane_layout(c->nx, c->ny, c->nkx_d, c->npair_d, c->ychunk_d);
  const bool two_pass = c->nx == c->ny;
  e = two_pass ? oa_rho2_fwd(s, c->nx, c->nz, c->rho, c->vol / c->npts, c->tw_x, (double2*)c->dz, c->ldl_d)
               : cudaErrorNotSupported;
  if (e == cudaErrorNotSupported) {
    e = oa_smem_limit(k_rho_plane_fwd);
    if (e != cudaSuccess) return e;
    k_rho_plane_fwd<<<c->nz, OA_NTHREADS, L.total, s>>>(c->rho, c->vol / c->npts, c->nx, c->ny, c->nz, c->nkx_d,
                                                         c->plan_x, c->plan_y, c->tw_x, c->tw_y,
                                                         (double2*)c->dz, c->ldl_d, c->npair_d, c->ychunk_d, L);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return e;
  RhoTypeOff toff;
  for (int t = 0; t < 5; ++t) toff.off[t] = c->type_off[t];
  const int nbz = oa_rho_z_nblk(c);
  auto zpass = [&](auto kern, int ldb) -> cudaError_t {
    const size_t smz =
        (align_up_r(c->nz, 2) + (size_t)OA_LB * (c->nz + 1) + (size_t)OA_LB * ldb + (size_t)OA_LB * c->natm) *
            sizeof(double2) +
        (size_t)c->natm * sizeof(int);  // zoff
    if (smz > (size_t)OA_MAX_SMEM) return cudaErrorNotSupported;
    cudaError_t e2 = oa_smem_limit(kern);
    if (e2 != cudaSuccess) return e2;
    kern<<<nbz, OA_NTHREADS, smz, s>>>((double2*)c->dz, c->ldl_d, c->nlines_d, c->nx, c->ny, c->nz,
                                       c->plan_z, c->tw_z, tpi_l, c->vol, c->ecut_rho,
                                       4.0 * c->alp_ewd * c->alp_ewd, c->gzvps_sum / c->vol,
                                       c->natm, c->ntype, c->atm_perm, toff, c->q_type, c->phase, c->kmax_tab,
                                       c->spl, c->nspl, c->spl_gmin, c->spl_dg,
                                       c->red + 3 * oa_rho_xc_nblk());
    return cudaGetLastError();
  };
  auto ldb2 = [&](int n1, int n2) { const int p = (n1 * (n2 | 1)) | 1; return p > c->nz + 1 ? p : c->nz + 1; };
  switch (c->nz) {
#define OA_ZP(NN, A, B) case NN: e = zpass(k_rho_zpass<A, B>, ldb2(A, B)); break;
    OA_ZP(12, 4, 3) OA_ZP(20, 4, 5) OA_ZP(24, 6, 4) OA_ZP(36, 6, 6) OA_ZP(40, 8, 5) OA_ZP(64, 8, 8)
    OA_ZP(96, 12, 8) OA_ZP(108, 12, 9) OA_ZP(160, 16, 10)
#undef OA_ZP
    default: e = cudaErrorNotSupported; break;
  }
  if (e == cudaErrorNotSupported) e = zpass(k_rho_zpass<0, 0>, c->nz + 1);
  if (e != cudaSuccess) return e;
  if (two_pass) {
    e = oa_rho2_bwd(s, c->nx, c->nz, (const double2*)c->dz, c->ldl_d, c->tw_x, c->vxc, c->vks,
                    c->precision == OA_FP64);
    if (e != cudaErrorNotSupported) return e;
  }
  if (c->precision == OA_FP64) {
    e = oa_smem_limit(k_rho_plane_bwd<double>);
    if (e != cudaSuccess) return e;
    k_rho_plane_bwd<double><<<c->nz, OA_NTHREADS, L.total, s>>>((const double2*)c->dz, c->ldl_d, c->nx, c->ny, c->nz,
                                                                c->nkx_d, c->plan_x, c->plan_y, c->tw_x, c->tw_y,
                                                                c->vxc, (double*)c->vks, c->npair_d, c->ychunk_d, L);
  } else {
    e = oa_smem_limit(k_rho_plane_bwd<float>);
    if (e != cudaSuccess) return e;
    k_rho_plane_bwd<float><<<c->nz, OA_NTHREADS, L.total, s>>>((const double2*)c->dz, c->ldl_d, c->nx, c->ny, c->nz,
                                                               c->nkx_d, c->plan_x, c->plan_y, c->tw_x, c->tw_y,
                                                               c->vxc, (float*)c->vks, c->npair_d, c->ychunk_d, L);
  }
  return cudaGetLastError();
}
