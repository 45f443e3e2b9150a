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

// 16-byte global -> shared copy without a register round trip, so that a
// block's staging copies are all in flight together (the caller commits
// the group and waits for it)
__device__ __forceinline__ void rho_cp16(void* sdst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc));
}
__device__ __forceinline__ void rho_cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void rho_cp_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// density sum + PZ-LDA
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(OA_NTHREADS)
k_rho_xc(const double* __restrict__ rho_part, int ngroup, size_t npts, double rvol, double cfac,
         const double* __restrict__ qscale, double* __restrict__ rho, double* __restrict__ vxc,
         double* __restrict__ part) {
  // cfac = 0 drops the PZ correlation (LYP correlation on, cp_pz_lda.C:66);
  // qscale (mixed form): the renormalisation to the exact electron count
  if (qscale) rvol *= qscale[0];
  __shared__ double sh[3 * 32];
  // Perdew-Zunger constants (cp_pz_lda.C:46-52)
  const double gamma = -0.14230, beta1 = 1.05290, beta2 = 0.33340;
  const double au = 0.03110, bu = -0.0480, cu = 0.00200, du = -0.01160;
  const double power = 1.0 / 3.0;
  const double rat1 = (7.0 / 6.0) * beta1, rat2 = (4.0 / 3.0) * beta2;
  const double pi = 3.14159265358979323846, fpi = 4.0 * pi;
  // rs = (3 / (4 pi r))^(1/3) and -(3 r / pi)^(1/3) from one cube root of
  // r; a negative density gives NaN as the powers do
  const double c_rs = cbrt(3.0 / fpi), c_x = cbrt(3.0 / pi);
  double acc[3] = {0.0, 0.0, 0.0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (size_t)gridDim.x * blockDim.x) {
    double r = 0.0;
    for (int g = 0; g < ngroup; ++g) r += rho_part[(size_t)g * npts + i];
    r *= rvol;
    rho[i] = r;
    const double cr = r >= 0.0 ? cbrt(r) : __longlong_as_double(0x7ff8000000000000LL);
    const double rs = c_rs / cr;
    const double sqtrs = sqrt(rs);
    const double xfact = -c_x * cr;
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
    cfact *= cfac;
    mufact *= cfac;
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
                double2* __restrict__ dz, int ldl_d, int npair, int ychunk, RhoPlaneSmem L, size_t fin,
                size_t fout) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* stwx = (double2*)(smem_raw + L.tw_x);
  double2* stwy = (double2*)(smem_raw + L.tw_y);
  double2* P = (double2*)(smem_raw + L.P);
  double2* W1 = (double2*)(smem_raw + L.W1);
  double2* W2 = (double2*)(smem_raw + L.W2);
  const int ldx = nx + 1, ldy = ny + 1;
  const int z = blockIdx.x;
  const int npairs = (ny + 1) / 2;
  rho += blockIdx.y * fin;
  dz += blockIdx.y * fout;
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
                const double* __restrict__ vxc, R* __restrict__ vks, int npair, int ychunk, RhoPlaneSmem L,
                size_t fin, size_t fout) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* stwx = (double2*)(smem_raw + L.tw_x);
  double2* stwy = (double2*)(smem_raw + L.tw_y);
  double2* P = (double2*)(smem_raw + L.P);
  double2* W1 = (double2*)(smem_raw + L.W1);
  double2* W2 = (double2*)(smem_raw + L.W2);
  const int ldx = nx + 1, ldy = ny + 1;
  const int z = blockIdx.x;
  const int npairs = (ny + 1) / 2;
  dz += blockIdx.y * fin;
  vks += blockIdx.y * fout;
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
  const double* vz = vxc ? vxc + (size_t)z * nx * ny : nullptr;  // null: vks = V
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
      oz[y1 * nx + x] = (R)(v.x + (vz ? vz[y1 * nx + x] : 0.0));
      if (y2 < ny) oz[y2 * nx + x] = (R)(v.y + (vz ? vz[y2 * nx + x] : 0.0));
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

// FORCES: also the atom forces of the local pseudopotential and the
// reciprocal Ewald sum (CP_hart_eext_calc's force loop, cp_hart_ext.C:300-360):
// per g of the block the per-type coefficients
//   A_t = w (Re rho v_t + Re S_q ewf q_t),  B_t = w (-Im rho v_t + Im S_q ewf q_t)
// go to shared memory, then one warp per atom sums
//   F_a += g (A_t Im h_a - B_t Re h_a),  h_a = e^{i g.R_a},
// over the block's g-points into fpart[block][atom][3].
// EES (ees.zq set; eesHartEextGchare / eesEwaldGchare, cp_hart_ext.C:1005-1340):
// the per-type structure factors are b(g) Qhat_t(g), Qhat_t taken from the
// transformed B-spline grids (types 2k, 2k+1 split from complex grid k by
// the conjugate point -g); FORCES writes the per-type force transforms
//   Y_t = v_t conj(rho b) + q_t ewf conj(b) S_q
// (the Ewald part folded in by the type's charge) into ees.zy at g and, for
// kx > 0, their conjugates at -g, instead of reducing over atoms here.
template <int N1, int N2, bool FORCES>
__global__ void __launch_bounds__(OA_NTHREADS, 2)
k_rho_zpass(double2* __restrict__ dz, int ldl_d, int nlines_d, int nx, int ny, int nz,
            OaFftPlan pz, const double2* __restrict__ twz,
            double tpi_l, double vol, double ecut4, double falp2, double gz_term,
            int natm, int ntype, const int* __restrict__ atm_perm, RhoTypeOff toff,
            const double* __restrict__ q_type, const double2* __restrict__ phase, int ktab,
            const double* __restrict__ spl, int nspl, double gmin, double dg,
            double* __restrict__ part, double* __restrict__ fpart, EesLocArgs ees) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ldz = nz + 1;
  const bool use_ees = ees.zq != nullptr;
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
  // FORCES: [OA_LB * nz][ntype] per-type (A, B) coefficients after zoff
  double2* cf = (double2*)(smem_raw + (((size_t)((char*)(zoff + natm) - (char*)smem_raw) + 15) & ~(size_t)15));
  // the density coefficients of the block's lines: every 16-byte copy
  // issued before any is waited for
  for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
    const int zz = idx / OA_LB, lb = idx - zz * OA_LB;
    if (lb < nb) rho_cp16(a + lb * ldz + zz, dz + (size_t)zz * ldl_d + l0 + lb);
  }
  rho_cp_commit();
  for (int ia = threadIdx.x; ia < natm; ia += blockDim.x) zoff[ia] = (atm_perm[ia] * 3 + 2) * nt + ktab;
#pragma unroll 4
  for (int idx = use_ees ? OA_LB * natm : threadIdx.x; idx < OA_LB * natm; idx += blockDim.x) {
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
  rho_cp_wait();
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
    double vtt[ZP_L][4];  // FORCES: v_t(|g|) / V per type
    int cls[ZP_L], ii[ZP_L];  // cls: 0 outside, 1 g = 0, 2 inside the density sphere
    size_t ep[ZP_L], em[ZP_L];  // EES: grid offsets of g and -g
    double2 bgv[ZP_L];          // EES: b(g)
    bool any = false;
#pragma unroll
    for (int j = 0; j < ZP_L; ++j) {
      const int lb = grp * ZP_L + j;
      cls[j] = 0; ii[j] = 1; hh[j] = 0.0; wn[j] = 1.0; g2v[j] = 0.0;
      ep[j] = 0; em[j] = 0;
      bgv[j] = make_double2(0.0, 0.0);
      rho[j] = make_double2(0.0, 0.0);
      sf_q[j] = make_double2(0.0, 0.0);
      vext[j] = make_double2(0.0, 0.0);
      if (lb >= nb) continue;
      const int l = l0 + lb;
      const int kx = l / ny;
      int ky = l - kx * ny; if (2 * ky >= ny) ky -= ny;
      if (use_ees && abs(kx) <= ktab && abs(ky) <= ktab && abs(kz) <= ktab) {
        // kx >= 0 here; |k| <= ktab < n / 2 on each axis of the EES grid
        const int ia = kx, ib = ky < 0 ? ky + ees.nb : ky, ic = kz < 0 ? kz + ees.nc : kz;
        const int iam = kx == 0 ? 0 : ees.na - kx, ibm = ky > 0 ? ees.nb - ky : -ky, icm = kz > 0 ? ees.nc - kz : -kz;
        ep[j] = ((size_t)ic * ees.nb + ib) * ees.na + ia;
        em[j] = ((size_t)icm * ees.nb + ibm) * ees.na + iam;
        bgv[j] = cmul(cmul(ees.ba[ia], ees.bb[ib]), ees.bc[ic]);
      }
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
        if (use_ees) {
          // Qhat_t = (Z +- conj Z(-g)) / (2 or 2i) of grid t / 2, times b(g)
          const double2* zg = ees.zq + (size_t)(t >> 1) * ees.gstride;
#pragma unroll
          for (int j = 0; j < ZP_L; ++j) {
            if (cls[j] != 2) continue;
            const double2 z = zg[ep[j]], zm = zg[em[j]];
            const double2 qh = (t & 1) ? make_double2(0.5 * (z.y + zm.y), 0.5 * (zm.x - z.x))
                                       : make_double2(0.5 * (z.x + zm.x), 0.5 * (z.y - zm.y));
            st[j] = cmul(bgv[j], qh);
          }
        } else {
          const double2* pl = pxy + grp * ZP_L * natm;
          // four z-phase loads in flight per thread (the loop is bound by
          // their latency, not by the multiply-adds)
          // (the force variant, short of registers, takes them one at a time)
          const int a0 = toff.off[t], a1 = toff.off[t + 1];
          int ia = a0;
          for (; !FORCES && ia + 4 <= a1; ia += 4) {
            double2 hz[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) hz[u] = phase[zoff[ia + u] + kz];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
              for (int j = 0; j < ZP_L; ++j) {
                const double2 h = cmul(pl[j * natm + ia + u], hz[u]);
                st[j].x += h.x; st[j].y += h.y;
              }
          }
          for (; ia < a1; ++ia) {
            const double2 hz = phase[zoff[ia] + kz];
#pragma unroll
            for (int j = 0; j < ZP_L; ++j) {
              const double2 h = cmul(pl[j * natm + ia], hz);
              st[j].x += h.x; st[j].y += h.y;
            }
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
          if constexpr (FORCES) vtt[j][t] = vt;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < ZP_L; ++j) {
      const int lb = grp * ZP_L + j;
      if (lb >= nb) continue;
      double2 out = make_double2(0.0, 0.0);
      if (cls[j] == 1) {
        double gzt = gz_term;
        if (use_ees) {
          // sum_t gzvps_t b(0) Qhat_t(0) / V (eesHartEextGchare's g = 0 branch)
          const double b0 = cmul(cmul(ees.ba[0], ees.bb[0]), ees.bc[0]).x;
          gzt = 0.0;
          for (int t = 0; t < ntype && t < 4; ++t) {
            const double2 z0 = ees.zq[(size_t)(t >> 1) * ees.gstride];
            const double yt = ees.gzvps[t] / vol * b0;
            gzt += yt * ((t & 1) ? z0.y : z0.x);
            if constexpr (FORCES) {
              double* w0 = (double*)(ees.zy + (size_t)(t >> 1) * ees.gstride);
              w0[t & 1] = yt * rho[j].x;
            }
          }
        }
        out.x = gzt;
        acc[1] += gzt * rho[j].x;
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
      if (FORCES && use_ees) {
        if (cls[j] == 2) {
          const double g2 = g2v[j];
          const double ewf = fpi * exp(-g2 / falp2) / (g2 * vol);
          const double2 cb = cconj(bgv[j]);
          const double2 rb = cconj(cmul(rho[j], bgv[j]));
          const double2 sqe = cmul(cb, sf_q[j]);
          const bool mirror = l0 + lb >= ny;  // kx > 0
          for (int t0 = 0; t0 < ntype && t0 < 4; t0 += 2) {
            double2 y[2];
            for (int u = 0; u < 2; ++u) {
              const int t = t0 + u;
              y[u] = make_double2(0.0, 0.0);
              if (t < ntype) {
                const double qt = q_type[t] * ewf;
                y[u].x = vtt[j][t] * rb.x + qt * sqe.x;
                y[u].y = vtt[j][t] * rb.y + qt * sqe.y;
              }
            }
            double2* w = ees.zy + (size_t)(t0 >> 1) * ees.gstride;
            w[ep[j]] = make_double2(y[0].x - y[1].y, y[0].y + y[1].x);
            if (mirror) w[em[j]] = make_double2(y[0].x + y[1].y, y[1].x - y[0].y);
          }
        }
      } else if constexpr (FORCES) {
        double2* c2 = cf + ((size_t)lb * nz + zz) * ntype;
        for (int t = 0; t < ntype && t < 4; ++t) {
          double2 ab = make_double2(0.0, 0.0);
          if (cls[j] == 2) {
            const double g2 = g2v[j];
            const double ewf = fpi * exp(-g2 / falp2) / (g2 * vol);
            const double qt = q_type[t];
            ab.x = wn[j] * (rho[j].x * vtt[j][t] + sf_q[j].x * ewf * qt);
            ab.y = wn[j] * (-rho[j].y * vtt[j][t] + sf_q[j].y * ewf * qt);
          }
          c2[t] = ab;
        }
      }
    }
  }
  __syncthreads();
  if (FORCES && !use_ees) {
    // one warp per atom (type order), lanes over the block's (line, plane) points
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int ia = warp; ia < natm; ia += nwarp) {
      int t = 0;
      while (t + 1 < ntype && ia >= toff.off[t + 1]) ++t;
      double fx = 0.0, fy = 0.0, fz = 0.0;
      for (int e = lane; e < nb * nz; e += 32) {
        const int lb = e / nz, zz = e - lb * nz;
        const double2 ab = cf[((size_t)lb * nz + zz) * ntype + t];
        if (ab.x == 0.0 && ab.y == 0.0) continue;
        const int l = l0 + lb;
        const int kx = l / ny;
        int ky = l - kx * ny; if (2 * ky >= ny) ky -= ny;
        int kz = zz; if (2 * kz >= nz) kz -= nz;
        const double2 h = cmul(pxy[lb * natm + ia], phase[zoff[ia] + kz]);
        const double comp = ab.x * h.y - ab.y * h.x;
        fx += tpi_l * kx * comp;
        fy += tpi_l * ky * comp;
        fz += tpi_l * kz * comp;
      }
      fx = warp_sum_d(fx);
      fy = warp_sum_d(fy);
      fz = warp_sum_d(fz);
      if (lane == 0) {
        double* o = fpart + ((size_t)blockIdx.x * natm + atm_perm[ia]) * 3;
        o[0] = fx; o[1] = fy; o[2] = fz;
      }
    }
  }
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

// ---------------------------------------------------------------------------
// BLYP gradient correction (cp_grad_rho_ctrl.C, cp_becke.C; the driver's
// divRhoVksGspace / acceptGradRhoVks / whiteByrdFFT / acceptWhiteByrd,
// CP_Rho_GSpacePlane.C:278-380, CP_Rho_RealSpacePlane.C:1061-1350):
//   k_rho_grad_z   rho(g) -> i g_a rho(g) / V on the density sphere, z^-1
//   (x-y inverse)  -> grad rho(r), three fields
//   k_rho_gga      per point: EGGA density, vxc += df/drho,
//                  h = df/d|grad rho| grad rho / |grad rho|
//   (x-y forward of h / N)
//   k_rho_div_z    z forward of h, i g . h(g) on the sphere, z^-1, and
//                  subtracted from the V_KS z-lines before their x-y inverse
// ---------------------------------------------------------------------------
struct GgaTerm { double f, dfr, dfg; };

// Becke 88 correction to the LDA exchange, spin-unpolarised (becke_gcx_lda,
// cp_becke.C:21-88): per spin rho_s = rho / 2, x = (g / 2) / rho_s^(4/3),
// b = x^2 / (1 + 6 beta x asinh x), f = -2 beta rho_s^(4/3) b;
// df/drho = -(4/3) beta rho_s^(1/3) (b - x b'), df/dg = -beta b'.
__device__ __forceinline__ GgaTerm gga_becke88(double rho, double g) {
  const double beta = 0.0042;
  const double rs = 0.5 * rho;
  const double r13 = cbrt(rs);
  const double r43 = rs * r13;
  const double x = 0.5 * g / r43;
  const double root = sqrt(1.0 + x * x);
  const double ash = log(x + root);
  const double den = 1.0 + 6.0 * beta * x * ash;
  const double b = x * x / den;
  const double q = x / den;
  const double bp = 2.0 * q - 6.0 * beta * q * q * (ash + x / root);
  GgaTerm t;
  t.f = -2.0 * beta * r43 * b;
  t.dfr = -beta * (4.0 / 3.0) * r13 * (b - x * bp);
  t.dfg = -beta * bp;
  return t;
}

// Lee-Yang-Parr correlation, closed shell (lyp_gcc, cp_becke.C:91-172):
// u = rho^(-1/3), D = 1 + d u, omega = exp(-c u) u^11 / D,
// delta = c u + d u / D, A = C_F rho^(8/3) + (5/12 - 7 delta / 72) g^2 - 11 g^2 / 24,
// f = -a rho / D - a b omega A rho^2.
__device__ __forceinline__ GgaTerm gga_lyp(double rho, double g) {
  const double a = 0.049180, b = 0.1320, c = 0.25330, d = 0.3490;
  const double cf = 2.871234000188191;  // C_F = 0.3 (3 pi^2)^(2/3)
  const double u = 1.0 / cbrt(rho);
  const double u2 = u * u;
  const double den = 1.0 + d * u;
  double u11 = u2 * u2;            // u^4
  u11 = u11 * u11 * u2 * u;        // u^11
  const double om = exp(-c * u) * u11 / den;
  const double dl = c * u + d * u / den;
  const double g2 = g * g;
  const double r2 = rho * rho;
  const double r23i = u2;          // rho^(-2/3)
  const double cq = 5.0 / 12.0 - 7.0 * dl / 72.0;
  const double A = cf * r2 / r23i + cq * g2 - 11.0 * g2 / 24.0;  // C_F rho^(8/3) = C_F rho^2 / rho^(-2/3)
  const double dom = om * (c * u + d * u / den - 11.0) / (3.0 * rho);
  const double ddl = -(u / (3.0 * rho)) * (c + d / (den * den));
  const double dA = (8.0 / 3.0) * cf * rho / r23i - (7.0 / 72.0) * ddl * g2;  // d/drho, rho^(5/3) = rho / rho^(-2/3)
  GgaTerm t;
  t.f = -a * rho / den - a * b * om * A * r2;
  t.dfr = -a * (1.0 + (4.0 / 3.0) * d * u) / (den * den) - a * b * (dom * A * r2 + om * (dA * r2 + 2.0 * A * rho));
  t.dfg = -a * b * om * r2 * 2.0 * g * (cq - 11.0 / 24.0);
  return t;
}

// Per point, on rho > rho_cut = gga_cut / 10 (CP_getGGAFunctional): Becke +
// LYP times the switching function s = t^2 (3 - 2 t), t = clamp((rho -
// rho_cut) / (3.9 gga_cut), 0, 1); vxc += d(s f)/drho; grad <- h; block
// partials of the exchange and correlation parts.  h is 0 where
// |grad rho| = 0 (no direction) and below rho_cut.
__global__ void __launch_bounds__(OA_NTHREADS)
k_rho_gga(const double* __restrict__ rho, double* __restrict__ grad, size_t npts, double gga_cut,
          double* __restrict__ vxc, double* __restrict__ part) {
  __shared__ double sh[2 * 32];
  const double rho_cut = 0.1 * gga_cut, heal = 1.0 / (3.9 * gga_cut);
  double acc[2] = {0.0, 0.0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (size_t)gridDim.x * blockDim.x) {
    const double r = rho[i];
    double hx = 0.0, hy = 0.0, hz = 0.0;
    if (r > rho_cut) {
      const double gx = grad[i], gy = grad[npts + i], gz = grad[2 * npts + i];
      const double g2 = gx * gx + gy * gy + gz * gz;
      const double g = sqrt(g2);
      const double t = fmin(fmax((r - rho_cut) * heal, 0.0), 1.0);
      const double sw = t * t * (3.0 - 2.0 * t);
      const double dsw = 6.0 * t * (1.0 - t) * heal;
      const GgaTerm x = gga_becke88(r, g), c = gga_lyp(r, g);
      vxc[i] += (x.dfr + c.dfr) * sw + (x.f + c.f) * dsw;
      acc[0] += x.f * sw;
      acc[1] += c.f * sw;
      if (g2 > 0.0) {
        const double k = (x.dfg + c.dfg) * sw / g;
        hx = gx * k; hy = gy * k; hz = gz * k;
      }
    }
    grad[i] = hx;
    grad[npts + i] = hy;
    grad[2 * npts + i] = hz;
  }
  block_sum_n<2>(acc, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x + 0] = acc[0];
    part[2 * blockIdx.x + 1] = acc[1];
  }
}

// g-vector of element (line lb, plane zz) of a z-pass block and whether it
// is inside the density sphere (the points k_rho_zpass keeps, g = 0 out)
__device__ __forceinline__ bool rho_sphere_g(int l, int zz, int ny, int nz, double tpi_l, double ecut4, int ktab,
                                             double* gx, double* gy, double* gz) {
  const int kx = l / ny;
  int ky = l - kx * ny; if (2 * ky >= ny) ky -= ny;
  int kz = zz; if (2 * kz >= nz) kz -= nz;
  *gx = tpi_l * kx; *gy = tpi_l * ky; *gz = tpi_l * kz;
  const double g2 = *gx * *gx + *gy * *gy + *gz * *gz;
  return g2 != 0.0 && g2 <= ecut4 && abs(kx) <= ktab && abs(ky) <= ktab && abs(kz) <= ktab;
}

// z transform of nb lines in x (ld ldz) with y as scratch; returns the
// buffer holding the result
template <int N1, int N2, int SIGN>
__device__ __forceinline__ double2* zfft_any(double2* x, double2* y, int ldz, int nb, const OaFftPlan& pz,
                                             const double2* tw) {
  if constexpr (N1 > 0) {
    zfft2<N1, N2, SIGN>(x, y, ldz, nb, tw);
    return x;
  } else {
    return fft_pingpong<SIGN>(x, y, ldz, nb, pz, tw);
  }
}

// three buffers of OA_LB lines (row stride ldz, each sized for the
// two-pass scratch layout) after the twiddles
template <int N1, int N2>
__host__ __device__ inline int gga_zbuf_ld(int nz) {
  if constexpr (N1 > 0) {
    const int ps = ZLd<N1, N2>::PS;
    return ps > nz + 1 ? ps : nz + 1;
  } else {
    return nz + 1;
  }
}

template <int N1, int N2>
__global__ void __launch_bounds__(OA_NTHREADS, 2)
k_rho_grad_z(const double2* __restrict__ dz, double2* __restrict__ dzg, size_t fstride, int ldl_d, int nlines_d,
             int ny, int nz, OaFftPlan pz, const double2* __restrict__ twz, double tpi_l, double ecut4, int ktab,
             double rvol) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ldz = nz + 1, lb_sz = OA_LB * gga_zbuf_ld<N1, N2>(nz);
  double2* tw = (double2*)smem_raw;
  double2* bufs[3];
  bufs[0] = tw + align_up_r(nz, 2);
  bufs[1] = bufs[0] + lb_sz;
  bufs[2] = bufs[1] + lb_sz;
  const int l0 = blockIdx.x * OA_LB;
  const int nb = min(OA_LB, nlines_d - l0);
  load_twiddles(tw, twz, nz);
  for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
    const int zz = idx / OA_LB, lb = idx - zz * OA_LB;
    if (lb < nb) rho_cp16(bufs[0] + lb * ldz + zz, dz + (size_t)zz * ldl_d + l0 + lb);
  }
  rho_cp_commit();
  rho_cp_wait();
  __syncthreads();
  double2* r = zfft_any<N1, N2, -1>(bufs[0], bufs[1], ldz, nb, pz, tw);
  __syncthreads();
  double2* x = (r == bufs[0]) ? bufs[1] : bufs[0];
  double2* y = bufs[2];
  for (int a = 0; a < 3; ++a) {
    for (int idx = threadIdx.x; idx < nb * nz; idx += blockDim.x) {
      const int lb = idx / nz, zz = idx - lb * nz;
      double gx, gy, gz;
      const bool in = rho_sphere_g(l0 + lb, zz, ny, nz, tpi_l, ecut4, ktab, &gx, &gy, &gz);
      const double2 v = r[lb * ldz + zz];
      const double f = in ? (a == 0 ? gx : (a == 1 ? gy : gz)) * rvol : 0.0;
      x[lb * ldz + zz] = make_double2(-v.y * f, v.x * f);  // i g_a rho(g) / V
    }
    __syncthreads();
    double2* q = zfft_any<N1, N2, +1>(x, y, ldz, nb, pz, tw);
    __syncthreads();
    double2* out = dzg + a * fstride;
    for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
      const int zz = idx / OA_LB, lb = idx - zz * OA_LB;
      if (lb < nb) out[(size_t)zz * ldl_d + l0 + lb] = q[lb * ldz + zz];
    }
    __syncthreads();
  }
}

template <int N1, int N2>
__global__ void __launch_bounds__(OA_NTHREADS, 2)
k_rho_div_z(double2* __restrict__ dz, const double2* __restrict__ dzh, size_t fstride, int ldl_d, int nlines_d,
            int ny, int nz, OaFftPlan pz, const double2* __restrict__ twz, double tpi_l, double ecut4, int ktab) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ldz = nz + 1, lb_sz = OA_LB * gga_zbuf_ld<N1, N2>(nz);
  double2* tw = (double2*)smem_raw;
  double2* a0 = tw + align_up_r(nz, 2);
  double2* a1 = a0 + lb_sz;
  double2* acc = a1 + lb_sz;
  const int l0 = blockIdx.x * OA_LB;
  const int nb = min(OA_LB, nlines_d - l0);
  load_twiddles(tw, twz, nz);
  for (int idx = threadIdx.x; idx < OA_LB * ldz; idx += blockDim.x) acc[idx] = make_double2(0.0, 0.0);
  for (int a = 0; a < 3; ++a) {
    const double2* in = dzh + a * fstride;
    for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
      const int zz = idx / OA_LB, lb = idx - zz * OA_LB;
      if (lb < nb) rho_cp16(a0 + lb * ldz + zz, in + (size_t)zz * ldl_d + l0 + lb);
    }
    rho_cp_commit();
    rho_cp_wait();
    __syncthreads();
    const double2* r = zfft_any<N1, N2, -1>(a0, a1, ldz, nb, pz, tw);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nb * nz; idx += blockDim.x) {
      const int lb = idx / nz, zz = idx - lb * nz;
      double gx, gy, gz;
      if (rho_sphere_g(l0 + lb, zz, ny, nz, tpi_l, ecut4, ktab, &gx, &gy, &gz)) {
        const double ga = a == 0 ? gx : (a == 1 ? gy : gz);
        const double2 v = r[lb * ldz + zz];
        acc[lb * ldz + zz].x -= v.y * ga;  // += i g_a h_a(g)
        acc[lb * ldz + zz].y += v.x * ga;
      }
    }
    __syncthreads();
  }
  const double2* q = zfft_any<N1, N2, +1>(acc, a0, ldz, nb, pz, tw);
  __syncthreads();
  for (int idx = threadIdx.x; idx < nz * OA_LB; idx += blockDim.x) {
    const int zz = idx / OA_LB, lb = idx - zz * OA_LB;
    if (lb < nb) {
      double2& o = dz[(size_t)zz * ldl_d + l0 + lb];
      const double2 w = q[lb * ldz + zz];
      o.x -= w.x;
      o.y -= w.y;
    }
  }
}

cudaError_t oa_rho2_fwd(cudaStream_t s, int n, int nz, const double* rho, double scale, const double2* tw,
                        double2* dz, int ldl_d, int nf, size_t fin, size_t fout);
cudaError_t oa_rho2_bwd(cudaStream_t s, int n, int nz, const double2* dz, int ldl_d, const double2* tw,
                        const double* vxc, void* vks, int fp64, int nf, size_t fin, size_t fout);

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

// Mixed form: the FP32 transforms scale the density by about 1 - 1.4e-7
// (a uniform gain error); the density is renormalised to the electron count
// of the FP64 coefficients, Q = sum_s occ_s sum_g w |c_sg|^2, against the
// FP32 density's own sum_r rho V/N.  One block, fixed summation order.
__global__ void k_charge_scale(const double* __restrict__ qexact, int n1, const double* __restrict__ q32, int n2,
                               double rnpts, double* __restrict__ scale) {
  __shared__ double sh[2 * 32];
  double v[2] = {0.0, 0.0};
  for (int i = threadIdx.x; i < n1; i += blockDim.x) v[0] += qexact[i];
  for (int i = threadIdx.x; i < n2; i += blockDim.x) v[1] += q32[i];
  block_sum_n<2>(v, sh);
  if (threadIdx.x == 0) scale[0] = (v[1] > 0.0) ? v[0] / (v[1] * rnpts) : 1.0;
}

cudaError_t oa_launch_rho_xc(oa_ctx* c, cudaStream_t s) {
  const int nblk = 4 * 148;
  const bool renorm = c->qvalid == 2;
  if (renorm) {
    k_charge_scale<<<1, 1024, 0, s>>>(c->qpart, c->nq, c->qpart2, c->nq2, 1.0 / (double)c->npts, c->qscale);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  k_rho_xc<<<nblk, OA_NTHREADS, 0, s>>>(c->rho_part, c->rho_ngroup, (size_t)c->npts, 1.0 / c->vol,
                                        c->gga ? 0.0 : 1.0, renorm ? c->qscale : nullptr, c->rho, c->vxc, c->red);
  return cudaGetLastError();
}

int oa_rho_xc_nblk() { return 4 * 148; }
int oa_rho_z_nblk(const oa_ctx* c) { return (c->nlines_d + OA_LB - 1) / OA_LB; }
// offset of the GGA block partials (2 per block of k_rho_gga) in c->red
size_t oa_rho_gga_red_off(const oa_ctx* c) { return (size_t)3 * oa_rho_xc_nblk() + 3 * (size_t)oa_rho_z_nblk(c); }

cudaError_t oa_launch_phase_tables(oa_ctx* c, cudaStream_t s) {
  const double tpi_l = 2.0 * 3.14159265358979323846 / c->box;
  const int total = c->natm * 3 * (2 * c->kmax_tab + 1);
  k_phase_tables<<<(total + 255) / 256, 256, 0, s>>>(c->pos, c->natm, c->kmax_tab, tpi_l, c->phase);
  return cudaGetLastError();
}

// x-y forward transform of nf real fields (stride fin doubles) into density
// z-lines (stride fout double2), two-pass kernels where the length has them
static cudaError_t rho_xy_fwd(oa_ctx* c, cudaStream_t s, const double* src, double scale, double2* dst, int nf,
                              size_t fin, size_t fout) {
  cudaError_t e = c->nx == c->ny ? oa_rho2_fwd(s, c->nx, c->nz, src, scale, c->tw_x, dst, c->ldl_d, nf, fin, fout)
                                 : cudaErrorNotSupported;
  if (e != cudaErrorNotSupported) return e;
  RhoPlaneSmem L = rho_plane_layout(c->nx, c->ny, c->nkx_d, c->npair_d, c->ychunk_d);
  e = oa_smem_limit(k_rho_plane_fwd);
  if (e != cudaSuccess) return e;
  k_rho_plane_fwd<<<dim3(c->nz, nf), OA_NTHREADS, L.total, s>>>(src, scale, c->nx, c->ny, c->nz, c->nkx_d,
                                                                 c->plan_x, c->plan_y, c->tw_x, c->tw_y, dst,
                                                                 c->ldl_d, c->npair_d, c->ychunk_d, L, fin, fout);
  return cudaGetLastError();
}

// x-y inverse of nf fields of density z-lines into real grids (+ vxc when
// not null), in FP64 or the compute precision
static cudaError_t rho_xy_bwd(oa_ctx* c, cudaStream_t s, const double2* src, const double* vxc, void* dst, int fp64,
                              int nf, size_t fin, size_t fout) {
  cudaError_t e = c->nx == c->ny
                      ? oa_rho2_bwd(s, c->nx, c->nz, src, c->ldl_d, c->tw_x, vxc, dst, fp64, nf, fin, fout)
                      : cudaErrorNotSupported;
  if (e != cudaErrorNotSupported) return e;
  RhoPlaneSmem L = rho_plane_layout(c->nx, c->ny, c->nkx_d, c->npair_d, c->ychunk_d);
  const dim3 grid(c->nz, nf);
  if (fp64) {
    e = oa_smem_limit(k_rho_plane_bwd<double>);
    if (e != cudaSuccess) return e;
    k_rho_plane_bwd<double><<<grid, OA_NTHREADS, L.total, s>>>(src, c->ldl_d, c->nx, c->ny, c->nz, c->nkx_d,
                                                               c->plan_x, c->plan_y, c->tw_x, c->tw_y, vxc,
                                                               (double*)dst, c->npair_d, c->ychunk_d, L, fin, fout);
  } else {
    e = oa_smem_limit(k_rho_plane_bwd<float>);
    if (e != cudaSuccess) return e;
    k_rho_plane_bwd<float><<<grid, OA_NTHREADS, L.total, s>>>(src, c->ldl_d, c->nx, c->ny, c->nz, c->nkx_d,
                                                              c->plan_x, c->plan_y, c->tw_x, c->tw_y, vxc,
                                                              (float*)dst, c->npair_d, c->ychunk_d, L, fin, fout);
  }
  return cudaGetLastError();
}

// the two GGA z kernels, two-pass where nz has a factorisation
static cudaError_t gga_z(oa_ctx* c, cudaStream_t s, int div) {
  const double tpi_l = 2.0 * 3.14159265358979323846 / c->box;
  const size_t fst = (size_t)c->nz * c->ldl_d;
  const int nbz = oa_rho_z_nblk(c);
  auto go = [&](auto grad_k, auto div_k, int ld) -> cudaError_t {
    const size_t sm = (align_up_r(c->nz, 2) + (size_t)3 * OA_LB * ld) * sizeof(double2);
    if (sm > (size_t)OA_MAX_SMEM) return cudaErrorNotSupported;
    cudaError_t e2;
    if (div) {
      if ((e2 = oa_smem_limit(div_k)) != cudaSuccess) return e2;
      div_k<<<nbz, OA_NTHREADS, sm, s>>>((double2*)c->dz, (const double2*)c->dzg, fst, c->ldl_d, c->nlines_d, c->ny,
                                         c->nz, c->plan_z, c->tw_z, tpi_l, c->ecut_rho, c->kmax_tab);
    } else {
      if ((e2 = oa_smem_limit(grad_k)) != cudaSuccess) return e2;
      grad_k<<<nbz, OA_NTHREADS, sm, s>>>((const double2*)c->dz, (double2*)c->dzg, fst, c->ldl_d, c->nlines_d,
                                          c->ny, c->nz, c->plan_z, c->tw_z, tpi_l, c->ecut_rho, c->kmax_tab,
                                          1.0 / c->vol);
    }
    return cudaGetLastError();
  };
  cudaError_t e;
  switch (c->nz) {
#define OA_GZ(NN, A, B) \
  case NN: e = go(k_rho_grad_z<A, B>, k_rho_div_z<A, B>, gga_zbuf_ld<A, B>(c->nz)); break;
    OA_GZ(12, 4, 3) OA_GZ(20, 4, 5) OA_GZ(24, 6, 4) OA_GZ(36, 6, 6) OA_GZ(40, 8, 5) OA_GZ(64, 8, 8)
    OA_GZ(96, 12, 8) OA_GZ(108, 12, 9) OA_GZ(160, 16, 10)
#undef OA_GZ
    default: e = cudaErrorNotSupported; break;
  }
  if (e == cudaErrorNotSupported) e = go(k_rho_grad_z<0, 0>, k_rho_div_z<0, 0>, c->nz + 1);
  return e;
}

// BLYP before the Hartree z pass: grad rho, the per-point functional
// (vxc, EGGA partials, h), and h's x-y forward transform into dzg
static cudaError_t gga_front(oa_ctx* c, cudaStream_t s) {
  const size_t fz = (size_t)c->nz * c->ldl_d, fr = (size_t)c->npts;
  cudaError_t e;
  if ((e = gga_z(c, s, 0)) != cudaSuccess) return e;
  if ((e = rho_xy_bwd(c, s, (const double2*)c->dzg, nullptr, c->grad, 1, 3, fz, fr)) != cudaSuccess) return e;
  k_rho_gga<<<oa_rho_xc_nblk(), OA_NTHREADS, 0, s>>>(c->rho, c->grad, fr, c->gga_cut, c->vxc,
                                                      c->red + oa_rho_gga_red_off(c));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return rho_xy_fwd(c, s, c->grad, 1.0 / c->npts, (double2*)c->dzg, 3, fr, fz);
}

cudaError_t oa_launch_rho_fft_hart(oa_ctx* c, cudaStream_t s) {
  const double tpi_l = 2.0 * 3.14159265358979323846 / c->box;
  cudaError_t e;
  // phase tables exp(i 2 pi k x / L)
  if ((e = oa_launch_phase_tables(c, s)) != cudaSuccess) return e;
  if ((e = rho_xy_fwd(c, s, c->rho, c->vol / c->npts, (double2*)c->dz, 1, 0, 0)) != cudaSuccess) return e;
  if (c->gga && (e = gga_front(c, s)) != cudaSuccess) return e;
  RhoTypeOff toff;
  for (int t = 0; t < 5; ++t) toff.off[t] = c->type_off[t];
  const int nbz = oa_rho_z_nblk(c);
  const bool forces = c->ions != nullptr;
  EesLocArgs ees{};
  if (c->eesl) {
    // B-spline grids of the atom types and their transform (and the force
    // grids zeroed) before the z pass reads them
    if ((e = oa_launch_eesl_front(c, s)) != cudaSuccess) return e;
    const oa_eesl* L = c->eesl;
    ees.zq = L->zq;
    ees.zy = forces ? L->zy : nullptr;
    ees.ba = L->ba; ees.bb = L->bb; ees.bc = L->bc;
    ees.gzvps = L->gzvps;
    ees.na = L->na; ees.nb = L->nb; ees.nc = L->nc;
    ees.gstride = (size_t)L->na * L->nb * L->nc;
  }
  auto zpass = [&](auto kern, int ldb) -> cudaError_t {
    size_t smz =
        (align_up_r(c->nz, 2) + (size_t)OA_LB * (c->nz + 1) + (size_t)OA_LB * ldb + (size_t)OA_LB * c->natm) *
            sizeof(double2) +
        (size_t)c->natm * sizeof(int);  // zoff
    if (forces) smz = align_up_r(smz, 16) + (size_t)OA_LB * c->nz * c->ntype * sizeof(double2);
    if (smz > (size_t)OA_MAX_SMEM) return cudaErrorNotSupported;
    cudaError_t e2 = oa_smem_limit(kern);
    if (e2 != cudaSuccess) return e2;
    kern<<<nbz, OA_NTHREADS, smz, s>>>((double2*)c->dz, c->ldl_d, c->nlines_d, c->nx, c->ny, c->nz,
                                       c->plan_z, c->tw_z, tpi_l, c->vol, c->ecut_rho,
                                       4.0 * c->alp_ewd * c->alp_ewd, c->gzvps_sum / c->vol,
                                       c->natm, c->ntype, c->atm_perm, toff, c->q_type, c->phase, c->kmax_tab,
                                       c->spl, c->nspl, c->spl_gmin, c->spl_dg,
                                       c->red + 3 * oa_rho_xc_nblk(), forces ? c->ions->fpart : nullptr, ees);
    return cudaGetLastError();
  };
  auto ldb2 = [&](int n1, int n2) { const int p = (n1 * (n2 | 1)) | 1; return p > c->nz + 1 ? p : c->nz + 1; };
  switch (c->nz) {
#define OA_ZP(NN, A, B)                                                                      \
  case NN:                                                                                   \
    e = forces ? zpass(k_rho_zpass<A, B, true>, ldb2(A, B)) : zpass(k_rho_zpass<A, B, false>, ldb2(A, B)); \
    break;
    OA_ZP(12, 4, 3) OA_ZP(20, 4, 5) OA_ZP(24, 6, 4) OA_ZP(36, 6, 6) OA_ZP(40, 8, 5) OA_ZP(64, 8, 8)
    OA_ZP(96, 12, 8) OA_ZP(108, 12, 9) OA_ZP(160, 16, 10)
#undef OA_ZP
    default: e = cudaErrorNotSupported; break;
  }
  if (e == cudaErrorNotSupported)
    e = forces ? zpass(k_rho_zpass<0, 0, true>, c->nz + 1) : zpass(k_rho_zpass<0, 0, false>, c->nz + 1);
  if (e != cudaSuccess) return e;
  // EES: the force grids back to real space and the atom forces from them
  if (c->eesl && forces && (e = oa_launch_eesl_forces(c, s)) != cudaSuccess) return e;
  // white-byrd: V_KS z-lines -= z^-1 (i g . h(g))
  if (c->gga && (e = gga_z(c, s, 1)) != cudaSuccess) return e;
  return rho_xy_bwd(c, s, (const double2*)c->dz, c->vxc, c->vks, c->precision == OA_FP64, 1, 0, 0);
}
