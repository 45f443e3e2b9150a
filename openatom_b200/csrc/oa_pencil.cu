// Two-pass pencil kernels of the state FFT path, for the grid lengths with a
// compile-time factorisation N = N1 * N2 (oa_rdft.cuh).  Same work and same
// results as the runtime-plan kernels in oa_state.cu (which cover every
// 2-3-5 length), with every pencil transformed as
//   pass A: DFT_N1 in registers + twiddle -> shared memory
//   pass B: DFT_N2 in registers -> destination
// so each pencil makes two shared-memory round trips, all index arithmetic
// is by constants and the small DFTs have constant twiddles.
//
// Reference work replaced (as the oa_state.cu kernels):
//   FFTcache::expandGSpace + doStpFFTGtoR_Gchare (fftCache.C:460, 1133)     -> k_zfwd2
//   FFTcache::doStpFFTGtoR_Rchare (fftCache.C:1167) + density part of
//     CP_State_RealSpacePlane::doFFT/doReduction (:349-363, 450-517)      -> k_plane2<MODE 0>
//   CP_State_RealSpacePlane::unpackVks (:530-597) + doStpFFTRtoG_Rchare
//     (fftCache.C:1252-1319)                                              -> k_plane2<MODE 1>
//   EES eesZmatRchare / eesEnergyAtmForcRchare on the nonlocal grid
//     (cp_ees_nonlocal.C:1238-1352, 1480-1720)                            -> k_plane2<MODE 2, 3>
//   CP_State_GSpacePlane::doIFFT (:1581) + packGSpace (fftCache.C:517) +
//     GStateSlab::addForces (stateSlab.C:239) + CP_eke_calc (cp_eke.C:30)  -> k_zbwd2
#include "oa_rdft.cuh"
#include "oa_state_common.cuh"
#include "oa_planes.cuh"

// Smallest odd stride >= minv, congruent to want (odd) modulo 16 when want >= 0.
__host__ __device__ constexpr int pencil_stride(int minv, int want) {
  int p = minv | 1;
  if (want >= 0)
    while ((p & 15) != want) p += 2;
  return p;
}

// Shared-memory strides (complex elements) of the pass-A -> pass-B buffer
// ([k1][n2] per pencil, row ls1, pencil ps1) and of the inverse B' -> A'
// buffer ([m2][k1], row ls2, pencil ps2).  Bank rule (8-byte elements, 16
// threads per conflict domain): all strides are odd, so 16 threads that
// walk consecutive pencils at the same offset hit 16 distinct banks; and,
// for odd N2, ps1 = N2 and ps2 = N2 ls2 (mod 16), so threads that walk
// (pencil, n2) with n2 fastest address ps1 pencil + n2 = thread (mod 16).
template <int N1, int N2> struct PencilLd {
  static constexpr int ls1 = odd_ld(N2);
  static constexpr int ls2 = odd_ld(N1);
  static constexpr int ps1 = pencil_stride(N1 * ls1, (N2 & 1) ? (N2 & 15) : -1);
  static constexpr int ps2 = pencil_stride(N2 * ls2, (N2 & 1) ? ((N2 * ls2) & 15) : -1);
};

// 16-byte global -> shared copy that completes in the background
__device__ __forceinline__ void zp_cp16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}

// packed index of z-slot z on a line with nn negative and np non-negative kz
// (negative kz first, as the reference's run pairs); -1 outside the sphere
__device__ __forceinline__ int line_slot(int z, int n, int nn, int np) {
  if (z < np) return nn + z;
  if (z >= n - nn) return z - (n - nn);
  return -1;
}

// ---------------------------------------------------------------------------
// z pass forward: packed sphere (optionally conj(dyp psi)) -> FFT(-) of the
// zero-filled z-line -> zbuf[s][z][line].  Block = OA_LB lines of one state.
// BAND: the kz of every line lie in (-N/4, N/4), so the pass-A inputs n1
// in [N1/4, 3 N1/4) are zero (band-pruned first DFT, RDftBand).
// ---------------------------------------------------------------------------
template <typename R, int N1, int N2, bool BAND>
__global__ void __launch_bounds__(OA_NTHREADS)
k_zfwd2(const double2* __restrict__ psi, int ng, int s0, const int* __restrict__ line_off,
        const int* __restrict__ line_nneg, const int* __restrict__ line_npos, int nlines,
        typename CplxOf<R>::T* __restrict__ zbuf, int ldl, const double2* __restrict__ twz,
        const double2* __restrict__ dyp, int zseg, OaCharge qc) {
  typedef typename CplxOf<R>::T C;
  constexpr int N = N1 * N2;
  typedef PencilLd<N1, N2> L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double qsh[32];
  C* tw = (C*)smem_raw;
  C* s1 = tw + align_up(N, 2);
  // zseg > 0: the block's lines are one contiguous run of the coefficients,
  // staged with coalesced loads before pass A gathers from it
  double2* seg = (double2*)(s1 + align_up((size_t)OA_LB * L::ps1, 2));
  const int s = s0 + blockIdx.y;
  const int l0 = blockIdx.x * OA_LB;
  const int nb = min(OA_LB, nlines - l0);
  const double2* ps = psi + (size_t)s * ng;
  const int g0 = zseg > 0 ? line_off[l0] : 0;
  if (zseg > 0) {
    // every 16-byte copy of the run issued before any is waited for
    const int g1 = (l0 + nb < nlines) ? line_off[l0 + nb] : ng;
    for (int i = threadIdx.x; i < g1 - g0; i += blockDim.x) zp_cp16(seg + i, ps + g0 + i);
    asm volatile("cp.async.commit_group;\n" ::);
  }
  load_twiddles(tw, twz, N);
  if (zseg > 0) asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  double q = 0.0;  // charge partial (qc.part)
  for (int it = threadIdx.x; it < nb * N2; it += blockDim.x) {
    const int lb = it / N2, n2 = it - lb * N2;
    const int l = l0 + lb;
    const int off = line_off[l], nn = line_nneg[l], np = line_npos[l];
    const double wq = (qc.part && qc.line_kx[l] != 0) ? 2.0 : 1.0;
    C u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      if (BAND && n1 >= N1 / 4 && n1 < 3 * N1 / 4) {
        u[n1] = cmk<C>(0.0, 0.0);
        continue;
      }
      const int i = line_slot(N2 * n1 + n2, N, nn, np);
      double2 v = make_double2(0.0, 0.0);
      if (i >= 0) {
        v = zseg > 0 ? seg[off - g0 + i] : ps[off + i];
        q += wq * (v.x * v.x + v.y * v.y);
        if (dyp) {  // EES projector: projPsiG = conj(dyp psi) (eesProjGchare)
          const double2 d = dyp[off + i];
          v = make_double2(d.x * v.x - d.y * v.y, -(d.y * v.x + d.x * v.y));
        }
      }
      u[n1] = cmk<C>(v.x, v.y);
    }
    pass_a_band<N1, N2, -1, BAND>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) s1[lb * L::ps1 + k1 * L::ls1 + n2] = u[k1];
  }
  __syncthreads();
  C* out = zbuf + (size_t)s * N * ldl + l0;
  for (int it = threadIdx.x; it < N1 * OA_LB; it += blockDim.x) {
    const int k1 = it / OA_LB, lb = it - k1 * OA_LB;
    if (lb >= nb) continue;
    C w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = s1[lb * L::ps1 + k1 * L::ls1 + n2];
    RDft<N2, -1>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) out[(size_t)(k1 + N1 * k2) * ldl + lb] = w[k2];
  }
  if (qc.part) {
    q = block_sum(q, qsh);
    if (threadIdx.x == 0) qc.part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = qc.occ[s] * q;
  }
}

// ---------------------------------------------------------------------------
// z pass backward: zbuf -> FFT(+) -> pack; F = scale w v (+ F_NL), then
// CP_eke_calc: F -= occ w g2 psi (g2 <= ecut, else F = 0), EKE partials.
// With dyp (EES): F = -w conj(dyp P) instead (eesPsiForcGspace).
// ---------------------------------------------------------------------------
template <typename R, int N1, int N2>
__global__ void __launch_bounds__(OA_NTHREADS)
k_zbwd2(const typename CplxOf<R>::T* __restrict__ zbuf, int ldl, int nlines, const int* __restrict__ line_kx,
        const int* __restrict__ line_off, const int* __restrict__ line_nneg, const int* __restrict__ line_npos,
        const double2* __restrict__ twz, const double2* __restrict__ psi, const double2* __restrict__ fnl,
        double2* __restrict__ force, const double* __restrict__ g2, const double* __restrict__ occ, int ng, int s0,
        double scale, double ecut, double* __restrict__ eke_part, int nblk, const double2* __restrict__ dyp,
        OaPlaneOut po, int zseg) {
  typedef typename CplxOf<R>::T C;
  constexpr int N = N1 * N2;
  typedef PencilLd<N1, N2> L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = (C*)smem_raw;
  C* s1 = tw + align_up(N, 2);
  double* sred = (double*)(s1 + align_up((size_t)OA_LB * L::ps1, 2));
  // zseg > 0: psi and F_NL of the block's lines (one contiguous run) staged
  // with coalesced loads while the z transform runs
  double2* segp = (double2*)(sred + 64);
  double2* segf = segp + zseg;
  const int s = s0 + blockIdx.y;
  const int l0 = blockIdx.x * OA_LB;
  const int nb = min(OA_LB, nlines - l0);
  // this thread's first pass-B item (k1 fastest): its line's packing read
  // now, so that pass B does not wait for it
  const int itB = threadIdx.x;
  const bool hasB = itB < nb * N1;
  int offB = 0, nnB = 0, npB = 0, kxB = 0;
  if (hasB) {
    const int l = l0 + itB / N1;
    offB = line_off[l]; nnB = line_nneg[l]; npB = line_npos[l]; kxB = line_kx[l];
  }
  const int g0 = zseg > 0 ? line_off[l0] : 0;
  if (zseg > 0 && !dyp) {
    const int g1 = (l0 + nb < nlines) ? line_off[l0 + nb] : ng;
    const double2* ps0 = psi + (size_t)s * ng + g0;
    const double2* fn0 = fnl ? fnl + (size_t)s * ng + g0 : nullptr;
    for (int i = threadIdx.x; i < g1 - g0; i += blockDim.x) {
      zp_cp16(segp + i, ps0 + i);
      if (fn0) zp_cp16(segf + i, fn0 + i);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  }
  const C* in = zbuf + (size_t)s * N * ldl + l0;
  // this thread's first pass-A item: its z-line loads go out before the
  // twiddle barrier
  const int itA = threadIdx.x;
  const int n2A = itA / OA_LB, lbA = itA - n2A * OA_LB;
  const bool hasA = itA < N2 * OA_LB && lbA < nb;
  C uA[N1];
  if (hasA) {
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) uA[n1] = in[(size_t)(N2 * n1 + n2A) * ldl + lbA];
  }
  load_twiddles(tw, twz, N);
  __syncthreads();
  if (hasA) {
    pass_a<N1, N2, +1>(uA, n2A, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) s1[lbA * L::ps1 + k1 * L::ls1 + n2A] = uA[k1];
  }
  for (int it = threadIdx.x + blockDim.x; it < N2 * OA_LB; it += blockDim.x) {
    const int n2 = it / OA_LB, lb = it - n2 * OA_LB;
    if (lb >= nb) continue;
    C u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) u[n1] = in[(size_t)(N2 * n1 + n2) * ldl + lb];
    pass_a<N1, N2, +1>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) s1[lb * L::ps1 + k1 * L::ls1 + n2] = u[k1];
  }
  if (zseg > 0 && !dyp) asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  const double2* ps = psi + (size_t)s * ng;
  double2* fs = force + (size_t)s * ng;
  const double2* fn = fnl ? fnl + (size_t)s * ng : nullptr;
  const double o = occ[s];
  double ek = 0.0;
  for (int it = threadIdx.x; it < nb * N1; it += blockDim.x) {
    const int lb = it / N1, k1 = it - lb * N1;
    const int l = l0 + lb;
    const bool first = it == itB;
    const int off = first ? offB : line_off[l];
    const int nn = first ? nnB : line_nneg[l];
    const int np = first ? npB : line_npos[l];
    const double w = ((first ? kxB : line_kx[l]) == 0) ? 1.0 : 2.0;
    const double sc = scale * w;
    const double wt = o * w;
    C v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) v[n2] = s1[lb * L::ps1 + k1 * L::ls1 + n2];
    RDft<N2, +1>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int i = line_slot(k1 + N1 * k2, N, nn, np);
      if (i < 0) continue;
      const int idx = off + i;
      const double gg = g2[idx];
      if (dyp) {
        const double2 d = dyp[idx];
        const double px = (double)v[k2].x;
        const double py = (gg == 0.0) ? 0.0 : (double)v[k2].y;
        fs[idx] = make_double2(-w * (d.x * px - d.y * py), w * (d.y * px + d.x * py));
        continue;
      }
      double2 f = make_double2((double)v[k2].x * sc, (double)v[k2].y * sc);
      if (fn) { const double2 q = zseg > 0 ? segf[idx - g0] : fn[idx]; f.x += q.x; f.y += q.y; }
      if (gg <= ecut) {
        const double2 p = zseg > 0 ? segp[idx - g0] : ps[idx];
        const double t = wt * gg;
        f.x -= p.x * t; f.y -= p.y * t;
        ek += t * (p.x * p.x + p.y * p.y);
      } else {
        f.x = 0.0; f.y = 0.0;
      }
      fs[idx] = f;
      if (po.P) oa_plane_put2(po, s, 2L * idx, f.x, f.y);
    }
  }
  const double tot = block_sum(ek, sred);
  if (threadIdx.x == 0) eke_part[(size_t)s * nblk + blockIdx.x] = tot;
}

// ---------------------------------------------------------------------------
// plane pass, nx = ny = N, for one z-plane and one group of states.
//   MODE 0: zbuf row -> P[kx][y] -> y FFT(-) -> x FFT(-) of row pairs
//           (two-for-one c2r) -> tile += occ psi(r)^2
//   MODE 1: ... x FFT(-) -> psi(r) V_KS occ -> x FFT(+) -> r2c unpack -> y FFT(+)
//           -> zbuf row (in place); V_KS is read from global memory (L2)
//   MODE 2: as MODE 0 but tile = psi(r) (nonlocal grid), then the EES Z gather
//   MODE 3: EES scatter -> tile -> x FFT(+) -> r2c unpack -> y FFT(+) -> zbuf row
//   MODE 4: as MODE 1 from psi(r) stored by MODE 0 (psir) instead of the
//           gather, y FFT(-) and x FFT(-); the zbuf row is output only
// MODE 0 also stores psi(r) to psir when it is given.
// Pencils (y columns, x row pairs) go through in chunks of at most G; the
// block synchronises between the passes.  In MODE 1 the forward DFT_N2, the
// V_KS product and the backward DFT_N2 of an x pencil run back to back in
// the registers of one thread (pass B, then pass B' of the inverse).
// Thread mappings keep shared memory free of bank conflicts (PencilLd):
// y passes and the x pass B walk 16 consecutive pencils (or a whole pencil
// padded to 16 threads) per half-warp; the other passes walk (pencil, index)
// with the index fastest.
// ---------------------------------------------------------------------------
struct Plane2Smem {
  size_t tw, P, tile, s1, s2, total;
  int G;
};

// Threads per block and the blocks per SM that the shared-memory layout aims
// for: the modes that keep a real-space tile (0, 2, 3) run 512 threads with
// two FP32 / one FP64 block per SM; the V_KS mode, which has no tile, runs
// 256 threads with three FP32 / two FP64 blocks per SM.
template <typename R, int MODE> __host__ __device__ constexpr int p2_threads() {
  return (MODE == 1 || MODE == 4) ? 256 : 512;
}
template <typename R, int MODE> __host__ __device__ constexpr int p2_min_blocks() {
  return (MODE == 1 || MODE == 4) ? (sizeof(R) == 4 ? 3 : 2) : (sizeof(R) == 4 ? 2 : 1);
}

template <typename R, int MODE, int N1, int N2>
__global__ void __launch_bounds__(p2_threads<R, MODE>(), p2_min_blocks<R, MODE>())
k_plane2(typename CplxOf<R>::T* __restrict__ zbuf, int nstate, int ldl, int nlines,
         const int* __restrict__ line_kx, const int* __restrict__ line_ky, int nkx,
         const double2* __restrict__ twg, const double* __restrict__ occ, const R* __restrict__ vks,
         double* __restrict__ rho_part, int ngroup, Plane2Smem L, EesArgs E, R* __restrict__ psir) {
  typedef typename CplxOf<R>::T C;
  constexpr int N = N1 * N2;
  constexpr int LDY = N + 1;
  constexpr bool VKS = MODE == 1 || MODE == 4;
  static_assert(N1 <= 16, "pass B pads a pencil to 16 threads");
  typedef PencilLd<N1, N2> LD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = (C*)(smem_raw + L.tw);
  C* P = (C*)(smem_raw + L.P);
  R* tile = (R*)(smem_raw + L.tile);
  C* s1 = (C*)(smem_raw + L.s1);
  C* s2 = (C*)(smem_raw + L.s2);
  const int G = L.G;
  const int z = blockIdx.x, g = blockIdx.y;
  const int nper = (nstate + ngroup - 1) / ngroup;
  const int sb = g * nper, se = min(nstate, sb + nper);
  constexpr int npairs = (N + 1) / 2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const R* vz = VKS ? vks + (size_t)z * N * N : nullptr;
  load_twiddles(tw, twg, N);
  if (MODE == 0) {
    for (int i = threadIdx.x; i < N * N; i += blockDim.x) tile[i] = (R)0;
  }
  __syncthreads();
  // y FFT over the kx columns [0, nkx), in place in P; pencil-fastest
  // mapping padded to 16 columns
  auto y_fft = [&](auto sign_c) {
    constexpr int SG = decltype(sign_c)::value;
    for (int c0 = 0; c0 < nkx; c0 += G) {
      const int gc = min(G, nkx - c0);
      const int gcp = (gc + 15) & ~15;
      for (int it = threadIdx.x; it < gcp * N2; it += blockDim.x) {
        const int n2 = it / gcp, cc = it - n2 * gcp;
        if (cc >= gc) continue;
        const C* col = P + (c0 + cc) * LDY;
        C u[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) u[n1] = col[N2 * n1 + n2];
        pass_a<N1, N2, SG>(u, n2, tw);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) s1[cc * LD::ps1 + k1 * LD::ls1 + n2] = u[k1];
      }
      __syncthreads();
      for (int it = threadIdx.x; it < gcp * N1; it += blockDim.x) {
        const int k1 = it / gcp, cc = it - k1 * gcp;
        if (cc >= gc) continue;
        C* col = P + (c0 + cc) * LDY;
        C w[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) w[n2] = s1[cc * LD::ps1 + k1 * LD::ls1 + n2];
        RDft<N2, SG>::run(w);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) col[k1 + N1 * k2] = w[k2];
      }
      __syncthreads();
    }
  };
  for (int s = sb; s < se; ++s) {
    C* row = zbuf + ((size_t)s * gridDim.x + z) * ldl;
    R* pr = psir ? psir + ((size_t)s * gridDim.x + z) * N * N : nullptr;  // psi(r) of this plane, [y][x]
    if (MODE == 3) {
      for (int i = threadIdx.x; i < N * N; i += blockDim.x) tile[i] = (R)0;
      __syncthreads();
      ees_scatter_plane(tile, N, z, s, E, warp, lane, p2_threads<R, MODE>() / 32);
      __syncthreads();
    } else if (MODE != 4) {
      for (int i = threadIdx.x; i < nkx * LDY; i += blockDim.x) P[i] = cmk<C>(0.0, 0.0);
      __syncthreads();
      for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
        int ky = line_ky[l]; if (ky < 0) ky += N;
        P[line_kx[l] * LDY + ky] = row[l];
      }
      __syncthreads();
      y_fft(std::integral_constant<int, -1>{});
    }
    const R o = (R)occ[s];
    // x pencils: row pairs (y1, y2) as one complex sequence, in balanced chunks
    const int nch = (npairs + G - 1) / G;
    const int gsz = (npairs + nch - 1) / nch;
    for (int p0 = 0; p0 < npairs; p0 += gsz) {
      const int gp = min(gsz, npairs - p0);
      constexpr int SA = (MODE == 3) ? +1 : -1;
      for (int it = threadIdx.x; MODE != 4 && it < gp * N2; it += blockDim.x) {
        const int pp = it / N2, n2 = it - pp * N2;
        const int y1 = 2 * (p0 + pp), y2 = y1 + 1;
        C u[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
          const int k = N2 * n1 + n2;
          C zz;
          if (MODE == 3) {
            zz.x = tile[y1 * N + k];
            zz.y = (y2 < N) ? tile[y2 * N + k] : (R)0;
          } else {
            const C a = herm_x(P, LDY, nkx, N, k, y1);
            C b = cmk<C>(0.0, 0.0);
            if (y2 < N) b = herm_x(P, LDY, nkx, N, k, y2);
            zz.x = a.x - b.y;
            zz.y = a.y + b.x;
          }
          u[n1] = zz;
        }
        pass_a<N1, N2, SA>(u, n2, tw);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) s1[pp * LD::ps1 + k1 * LD::ls1 + n2] = u[k1];
      }
      if (MODE != 4) __syncthreads();
      // pass B: one pencil per 16 threads (k1 < N1 active)
      for (int it = threadIdx.x; it < gp * 16; it += blockDim.x) {
        const int pp = it >> 4, k1 = it & 15;
        if (k1 >= N1) continue;
        const int y1 = 2 * (p0 + pp), y2 = y1 + 1;
        C w[N2];
        if (MODE == 4) {
          // psi(r) of the row pair at x = k1 + N1 k2
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) {
            const int x = k1 + N1 * k2;
            w[k2].x = __ldcs(pr + y1 * N + x);
            w[k2].y = (y2 < N) ? __ldcs(pr + y2 * N + x) : (R)0;
          }
        } else {
#pragma unroll
          for (int n2 = 0; n2 < N2; ++n2) w[n2] = s1[pp * LD::ps1 + k1 * LD::ls1 + n2];
          RDft<N2, SA>::run(w);
        }
        if (MODE == 0) {
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) {
            const int x = k1 + N1 * k2;
            tile[y1 * N + x] += o * w[k2].x * w[k2].x;
            if (y2 < N) tile[y2 * N + x] += o * w[k2].y * w[k2].y;
            if (pr) {
              pr[y1 * N + x] = w[k2].x;
              if (y2 < N) pr[y2 * N + x] = w[k2].y;
            }
          }
        } else if (MODE == 2) {
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) {
            const int x = k1 + N1 * k2;
            tile[y1 * N + x] = w[k2].x;
            if (y2 < N) tile[y2 * N + x] = w[k2].y;
          }
        } else if (MODE == 3) {
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) s2[pp * LD::ps2 + k1 + N1 * k2] = w[k2];
        } else {
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) {
            const int x = k1 + N1 * k2;
            w[k2].x *= __ldg(vz + y1 * N + x) * o;
            w[k2].y = (y2 < N) ? w[k2].y * __ldg(vz + y2 * N + x) * o : (R)0;
          }
          // inverse, first half: DFT_N2(+) over k2, twiddle exp(+2 pi i k1 m2 / N)
          RDft<N2, +1>::run(w);
#pragma unroll
          for (int m2 = 0; m2 < N2; ++m2) {
            const C t = (m2 == 0) ? w[m2] : cmul(w[m2], tw_rt<+1>(tw, k1 * m2));
            s2[pp * LD::ps2 + m2 * LD::ls2 + k1] = t;
          }
        }
      }
      __syncthreads();
      if (VKS) {
        // inverse, second half: DFT_N1(+) over k1 -> natural order in s1
        for (int it = threadIdx.x; it < gp * N2; it += blockDim.x) {
          const int pp = it / N2, m2 = it - pp * N2;
          C u[N1];
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) u[k1] = s2[pp * LD::ps2 + m2 * LD::ls2 + k1];
          RDft<N1, +1>::run(u);
#pragma unroll
          for (int m1 = 0; m1 < N1; ++m1) s1[pp * LD::ps1 + m2 + N2 * m1] = u[m1];
        }
        __syncthreads();
      }
      if (VKS || MODE == 3) {
        // two-for-one r2c unpack of the natural-order result into P[kx][y]
        const C* nat = VKS ? s1 : s2;
        const int pst = VKS ? LD::ps1 : LD::ps2;
        for (int it = threadIdx.x; it < gp * nkx; it += blockDim.x) {
          const int pp = it / nkx, k = it - pp * nkx;
          const int y1 = 2 * (p0 + pp), y2 = y1 + 1;
          const C a = nat[pp * pst + k];
          const C b = cconj(nat[pp * pst + (k == 0 ? 0 : N - k)]);
          C f1, f2;
          f1.x = (a.x + b.x) * (R)0.5; f1.y = (a.y + b.y) * (R)0.5;
          f2.x = (a.y - b.y) * (R)0.5; f2.y = -(a.x - b.x) * (R)0.5;
          P[k * LDY + y1] = f1;
          if (y2 < N) P[k * LDY + y2] = f2;
        }
        __syncthreads();
      }
    }
    if (MODE == 2) {
      ees_gather_plane(tile, N, z, s, E, warp, lane, p2_threads<R, MODE>() / 32);
      __syncthreads();
    }
    if (VKS || MODE == 3) {
      y_fft(std::integral_constant<int, +1>{});
      for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
        int ky = line_ky[l]; if (ky < 0) ky += N;
        row[l] = P[line_kx[l] * LDY + ky];
      }
      __syncthreads();
    }
  }
  if (MODE == 0) {
    double* out = rho_part + ((size_t)g * gridDim.x + z) * (size_t)N * N;
    for (int i = threadIdx.x; i < N * N; i += blockDim.x) out[i] = (double)tile[i];
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Shared-memory layout of k_plane2 for one mode: the per-block budget lets
// the target number of blocks share an SM (p2_min_blocks) when at least 8
// pencils then fit, else fewer blocks; G pencils per chunk.
template <typename C, typename R, int N1, int N2>
static Plane2Smem plane2_layout(int nkx, int mode) {
  constexpr int N = N1 * N2;
  typedef PencilLd<N1, N2> LD;
  const bool need_tile = mode != 1 && mode != 4;
  const bool need_s2 = mode == 1 || mode == 3 || mode == 4;
  Plane2Smem L;
  size_t o = 0;
  L.tw = o; o += align_up(N * sizeof(C), 16);
  L.P = o; o += align_up((size_t)nkx * (N + 1) * sizeof(C), 16);
  L.tile = o; o += need_tile ? align_up((size_t)N * N * sizeof(R), 16) : 0;
  const size_t fixed = o + 32;
  const size_t per = (LD::ps1 + (need_s2 ? LD::ps2 : 0)) * sizeof(C);
  const int want = nkx > (N + 1) / 2 ? nkx : (N + 1) / 2;
  const int target = (mode == 1 || mode == 4) ? (sizeof(R) == 4 ? 3 : 2) : (sizeof(R) == 4 ? 2 : 1);
  long g = 0;
  for (int k = target; k >= 1; --k) {
    size_t budget = (size_t)(228 * 1024) / k - 1024;
    if (budget > (size_t)OA_MAX_SMEM) budget = OA_MAX_SMEM;
    g = fixed < budget ? (long)((budget - fixed) / per) : 0;
    if (g >= 8 || g >= want) break;
  }
  if (g > want) g = want;
  if (g > 0) {  // balanced chunks
    const long nch = (want + g - 1) / g;
    g = (want + nch - 1) / nch;
  }
  L.G = (int)g;
  L.s1 = o; o += align_up((size_t)L.G * LD::ps1 * sizeof(C), 16);
  L.s2 = o; o += need_s2 ? align_up((size_t)L.G * LD::ps2 * sizeof(C), 16) : 0;
  L.total = o;
  return L;
}

template <int N> struct SplitOf { static constexpr int n1 = Split<N>::n1, n2 = Split<N>::n2; };

#define OA_PENCIL_LENGTHS(X) X(12) X(20) X(24) X(36) X(40) X(64) X(96) X(108) X(160)

int oa_pencil_supported(int n) {
#define OA_PS_CASE(NN) if (n == NN) return 1;
  OA_PENCIL_LENGTHS(OA_PS_CASE)
#undef OA_PS_CASE
  return 0;
}

#define OA_PENCIL_DISPATCH(n, CALL)                                  \
  switch (n) {                                                       \
    case 12: return CALL(4, 3);                                      \
    case 20: return CALL(4, 5);                                      \
    case 24: return CALL(6, 4);                                      \
    case 36: return CALL(6, 6);                                      \
    case 40: return CALL(8, 5);                                      \
    case 64: return CALL(8, 8);                                      \
    case 96: return CALL(12, 8);                                     \
    case 108: return CALL(12, 9);                                    \
    case 160: return CALL(16, 10);                                   \
    default: break;                                                  \
  }

// shared memory of the z passes: twiddles, the pass buffer, 64 doubles of
// reduction scratch, and nseg staged coefficient segments of zseg elements
// threads of a z-pass block: one per item of the larger of the two passes
// (N2 x OA_LB pass A items, N1 x OA_LB pass B items), in whole warps, at
// most OA_NTHREADS; smaller blocks than OA_NTHREADS leave room for more
// resident blocks, each with its staged coefficient run in flight
template <int N1, int N2> constexpr int zpass_threads() {
  constexpr int items = (N1 > N2 ? N1 : N2) * OA_LB;
  constexpr int t = (items + 31) / 32 * 32;
  return t < OA_NTHREADS ? t : OA_NTHREADS;
}

template <typename R, int N1, int N2>
static size_t zpass2_smem(int zseg, int nseg) {
  typedef typename CplxOf<R>::T C;
  return (align_up(N1 * N2, 2) + align_up((size_t)OA_LB * PencilLd<N1, N2>::ps1, 2)) * sizeof(C) +
         64 * sizeof(double) + (size_t)nseg * zseg * sizeof(double2);
}

template <typename R, int N1, int N2>
static cudaError_t zfwd2_n(cudaStream_t st, const double2* psi, int ng, int s0, int ns, const int* off,
                           const int* nneg, const int* npos, int nlines, void* zbuf, int ldl, const double2* tw,
                           const double2* dyp, int zseg, OaCharge qc, int zext) {
  typedef typename CplxOf<R>::T C;
  const size_t sm = zpass2_smem<R, N1, N2>(zseg, 1);
  const dim3 grid((nlines + OA_LB - 1) / OA_LB, ns);
  auto launch = [&](auto kern) -> cudaError_t {
    cudaError_t e = oa_smem_limit(kern);
    if (e != cudaSuccess) return e;
    kern<<<grid, zpass_threads<N1, N2>(), sm, st>>>(psi, ng, s0, off, nneg, npos, nlines, (C*)zbuf, ldl, tw, dyp,
                                                    zseg, qc);
    return cudaGetLastError();
  };
  // every line's kz within (-N/4, N/4): the band-pruned first DFT
  if constexpr (N1 % 4 == 0) {
    if (4 * zext <= N1 * N2) return launch(k_zfwd2<R, N1, N2, true>);
  }
  return launch(k_zfwd2<R, N1, N2, false>);
}

template <typename R>
static cudaError_t zfwd2(cudaStream_t st, int n, const double2* psi, int ng, int s0, int ns, const int* off,
                         const int* nneg, const int* npos, int nlines, void* zbuf, int ldl, const double2* tw,
                         const double2* dyp, int zseg, OaCharge qc, int zext) {
#define OA_CALL(A, B) zfwd2_n<R, A, B>(st, psi, ng, s0, ns, off, nneg, npos, nlines, zbuf, ldl, tw, dyp, zseg, qc, zext)
  OA_PENCIL_DISPATCH(n, OA_CALL)
#undef OA_CALL
  return cudaErrorNotSupported;
}

cudaError_t oa_pencil_zfwd(int precision, cudaStream_t st, int n, const double2* psi, int ng, int s0, int ns,
                           const int* off, const int* nneg, const int* npos, int nlines, void* zbuf, int ldl,
                           const double2* tw, const double2* dyp, int zseg, OaCharge qc, int zext) {
  return precision == OA_FP64
             ? zfwd2<double>(st, n, psi, ng, s0, ns, off, nneg, npos, nlines, zbuf, ldl, tw, dyp, zseg, qc, zext)
             : zfwd2<float>(st, n, psi, ng, s0, ns, off, nneg, npos, nlines, zbuf, ldl, tw, dyp, zseg, qc, zext);
}

template <typename R, int N1, int N2>
static cudaError_t zbwd2_n(cudaStream_t st, const void* zbuf, int ldl, int nlines, const int* lkx, const int* off,
                           const int* nneg, const int* npos, const double2* tw, const double2* psi,
                           const double2* fnl, double2* force, const double* g2, const double* occ, int ng, int s0,
                           int ns, double scale, double ecut, double* eke_part, int nblk, const double2* dyp,
                           OaPlaneOut po, int zseg) {
  typedef typename CplxOf<R>::T C;
  if (dyp) zseg = 0;
  const size_t sm = zpass2_smem<R, N1, N2>(zseg, fnl ? 2 : 1);
  cudaError_t e = oa_smem_limit(k_zbwd2<R, N1, N2>);
  if (e != cudaSuccess) return e;
  dim3 grid(nblk, ns);
  k_zbwd2<R, N1, N2><<<grid, zpass_threads<N1, N2>(), sm, st>>>((const C*)zbuf, ldl, nlines, lkx, off, nneg, npos, tw, psi, fnl,
                                                     force, g2, occ, ng, s0, scale, ecut, eke_part, nblk, dyp,
                                                     po, zseg);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t zbwd2(cudaStream_t st, int n, const void* zbuf, int ldl, int nlines, const int* lkx,
                         const int* off, const int* nneg, const int* npos, const double2* tw, const double2* psi,
                         const double2* fnl, double2* force, const double* g2, const double* occ, int ng, int s0,
                         int ns, double scale, double ecut, double* eke_part, int nblk, const double2* dyp,
                         OaPlaneOut po, int zseg) {
#define OA_CALL(A, B)                                                                                          \
  zbwd2_n<R, A, B>(st, zbuf, ldl, nlines, lkx, off, nneg, npos, tw, psi, fnl, force, g2, occ, ng, s0, ns, scale, \
                   ecut, eke_part, nblk, dyp, po, zseg)
  OA_PENCIL_DISPATCH(n, OA_CALL)
#undef OA_CALL
  return cudaErrorNotSupported;
}

cudaError_t oa_pencil_zbwd(int precision, cudaStream_t st, int n, const void* zbuf, int ldl, int nlines,
                           const int* lkx, const int* off, const int* nneg, const int* npos, const double2* tw,
                           const double2* psi, const double2* fnl, double2* force, const double* g2,
                           const double* occ, int ng, int s0, int ns, double scale, double ecut, double* eke_part,
                           int nblk, const double2* dyp, OaPlaneOut po, int zseg) {
  return precision == OA_FP64
             ? zbwd2<double>(st, n, zbuf, ldl, nlines, lkx, off, nneg, npos, tw, psi, fnl, force, g2, occ, ng, s0,
                             ns, scale, ecut, eke_part, nblk, dyp, po, zseg)
             : zbwd2<float>(st, n, zbuf, ldl, nlines, lkx, off, nneg, npos, tw, psi, fnl, force, g2, occ, ng, s0, ns,
                            scale, ecut, eke_part, nblk, dyp, po, zseg);
}

template <typename R, int MODE, int N1, int N2>
static cudaError_t plane2_n(cudaStream_t st, void* zbuf, int nstate, int ldl, int nlines, const int* lkx,
                            const int* lky, int nz, int nkx, const double2* tw, const double* occ, const void* vks,
                            double* rho_part, int ngroup, const EesArgs& E, void* psir) {
  typedef typename CplxOf<R>::T C;
  const Plane2Smem L = plane2_layout<C, R, N1, N2>(nkx, MODE);
  if (L.G < 1 || L.total > (size_t)OA_MAX_SMEM) return cudaErrorNotSupported;
  cudaError_t e =
      oa_smem_limit(k_plane2<R, MODE, N1, N2>);
  if (e != cudaSuccess) return e;
  dim3 grid(nz, ngroup);
  k_plane2<R, MODE, N1, N2><<<grid, p2_threads<R, MODE>(), L.total, st>>>(
      (C*)zbuf, nstate, ldl, nlines, lkx, lky, nkx, tw, occ, (const R*)vks, rho_part, ngroup, L, E, (R*)psir);
  return cudaGetLastError();
}

template <typename R, int MODE>
static cudaError_t plane2(cudaStream_t st, int n, void* zbuf, int nstate, int ldl, int nlines, const int* lkx,
                          const int* lky, int nz, int nkx, const double2* tw, const double* occ, const void* vks,
                          double* rho_part, int ngroup, const EesArgs& E, void* psir) {
#define OA_CALL(A, B) \
  plane2_n<R, MODE, A, B>(st, zbuf, nstate, ldl, nlines, lkx, lky, nz, nkx, tw, occ, vks, rho_part, ngroup, E, psir)
  OA_PENCIL_DISPATCH(n, OA_CALL)
#undef OA_CALL
  return cudaErrorNotSupported;
}

// nx = ny = n; returns cudaErrorNotSupported when n has no two-pass kernel
// or its shared memory does not fit (the caller then uses the runtime-plan
// kernel)
cudaError_t oa_pencil_plane(int precision, int mode, cudaStream_t st, int n, void* zbuf, int nstate, int ldl,
                            int nlines, const int* lkx, const int* lky, int nz, int nkx, const double2* tw,
                            const double* occ, const void* vks, double* rho_part, int ngroup, const EesArgs& E,
                            void* psir) {
#define OA_MODE(M)                                                                                              \
  if (mode == M)                                                                                                \
    return precision == OA_FP64                                                                                 \
               ? plane2<double, M>(st, n, zbuf, nstate, ldl, nlines, lkx, lky, nz, nkx, tw, occ, vks, rho_part, \
                                   ngroup, E, psir)                                                             \
               : plane2<float, M>(st, n, zbuf, nstate, ldl, nlines, lkx, lky, nz, nkx, tw, occ, vks, rho_part,  \
                                  ngroup, E, psir);
  OA_MODE(0) OA_MODE(1) OA_MODE(2) OA_MODE(3) OA_MODE(4)
#undef OA_MODE
  return cudaErrorNotSupported;
}

template <typename C, typename R, int N1, int N2>
static size_t plane2_smem_max(int nkx) {
  size_t m = 0;
  for (int mode = 0; mode < 5; ++mode) {
    const size_t t = plane2_layout<C, R, N1, N2>(nkx, mode).total;
    if (t > m) m = t;
  }
  return m;
}

// largest shared memory of the two-pass plane kernel over its modes; 0 when
// there is none for this length
size_t oa_pencil_plane_smem(int precision, int n, int nkx) {
#define OA_CALL(A, B)                                                                  \
  (precision == OA_FP64 ? plane2_smem_max<double2, double, A, B>(nkx)                  \
                        : plane2_smem_max<float2, float, A, B>(nkx))
  OA_PENCIL_DISPATCH(n, OA_CALL)
#undef OA_CALL
  return 0;
}
