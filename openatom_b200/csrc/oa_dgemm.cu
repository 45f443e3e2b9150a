// Pipelined FP64 tensor-core (DMMA) forward product of the PairCalculator:
//   C[i][j] = alpha sum_k w(k) A[i][k] B[j][k],  w(k) = w_kx0 for k < kx0_cols, else 1
// (PairCalculator::multiplyForward, ckPairCalculator.C:821-933, with the
// reference's DGEMM('T','N') on the 2*ng-double real view of each state).
//
// Split-K over slabs of 32 columns: the kx0 columns [0, kx0_cols) are shared
// out among the first n0 CTAs of a tile and the other columns among the
// remaining nr CTAs, slab t of a region going to CTA t mod (count), so at
// any moment the CTAs stream neighbouring 256-byte pieces of the same rows
// (DRAM pages are opened once, not once per CTA).  Each CTA writes an FP64
// partial of its 128 x 128 output tile; the kx0 weight is applied to the
// first n0 partials in the reduction, so the main loop has no per-column
// weight and, when A and B are the same matrix (the overlap S), one shared
// memory copy of the operand slab serves both sides.  Partials are summed in
// a fixed order: the result does not depend on scheduling.
//
// Main loop: 512 threads, 16 warps of 32 x 32 (4 x 4 DMMA m8n8k4 tiles); K
// slabs of 32 doubles move global -> shared with 16-byte cp.async into a
// ring of STAGES slabs (4 when A and B are one matrix, else 3: 144 / 216 KB),
// so the loads of the next slabs overlap the DMMAs of the current one.
#include "oa_internal.h"

#define DG_TM 128
#define DG_KS 32
#define DG_LD (DG_KS + 4)          // doubles per smem row: conflict-free fragment loads
#define DG_THREADS 512
#define DG_SLAB (DG_TM * DG_LD)    // doubles per operand slab

__device__ __forceinline__ void dg_dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

__device__ __forceinline__ void dg_cp16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;  // src-size 0: the 16 bytes are zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void dg_cp8(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void dg_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void dg_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N)); }

// one operand slab: rows [r0, r0 + 128) of X (row stride K), columns [k0, k0 + 32)
// clipped to [k0, kend) and rows < nrows; 2048 16-byte pieces, 4 per thread
__device__ __forceinline__ void dg_load_slab(double* dst, const double* __restrict__ X, int r0, int nrows, long K,
                                             long k0, long kend) {
#pragma unroll
  for (int q = 0; q < (DG_TM * DG_KS / 2) / DG_THREADS; ++q) {
    const int piece = threadIdx.x + q * DG_THREADS;
    const int r = piece >> 4;            // 16 pieces per row
    const int kk = (piece & 15) * 2;
    const long k = k0 + kk;
    const bool valid = (r0 + r < nrows) && (k < kend);
    const double* src = valid ? X + (size_t)(r0 + r) * K + k : X;
    dg_cp16(dst + r * DG_LD + kk, src, valid);
  }
}

template <bool SAME, int DG_STAGES>
__global__ void __launch_bounds__(DG_THREADS, 1)
k_dgemm_fwd(const double* __restrict__ A, const double* __restrict__ B, int m, int n, long K, long kx0_cols,
            int n0, int nr, double* __restrict__ part, const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  extern __shared__ __align__(16) double dg_smem[];
  double* As = dg_smem;
  double* Bs = SAME ? dg_smem : dg_smem + DG_STAGES * DG_SLAB;
  const int i0 = blockIdx.x * DG_TM, j0 = blockIdx.y * DG_TM;
  const int kb = blockIdx.z;
  // region and slab sequence of this CTA: slabs first, first + stride, ...
  const bool in0 = kb < n0;
  const long rbeg = in0 ? 0 : kx0_cols, rend = in0 ? kx0_cols : K;
  const int first = in0 ? kb : kb - n0, stride = in0 ? n0 : nr;
  const long rslabs = (rend - rbeg + DG_KS - 1) / DG_KS;
  const int nslab = rslabs > first ? (int)((rslabs - first + stride - 1) / stride) : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // A == B (the overlap, one diagonal tile): the 32 x 32 blocks below the
  // diagonal are the transposes of those above, which the reduction mirrors.
  // The ten blocks on and above it go to warps 0-9, so that each SM
  // sub-partition (warp mod 4) issues the DMMAs of at most three.
  int wi = (warp >> 2) * 32, wj = (warp & 3) * 32;
  if (SAME) {
    // 4 bi + bj of the upper blocks 0, 1, 2, 3, 5, 6, 7, 10, 11, 15, one hex digit per warp
    const int u = warp < 10 ? (int)((0xFBA7653210ull >> (4 * warp)) & 15u) : 0;
    wi = (u >> 2) * 32;
    wj = (u & 3) * 32;
  }
  const bool active = (i0 + wi < m) && (j0 + wj < n) && (!SAME || warp < 10);
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) { acc[a][b][0] = 0.0; acc[a][b][1] = 0.0; }
  // prologue: slabs 0 .. STAGES-2
#pragma unroll
  for (int s = 0; s < DG_STAGES - 1; ++s) {
    if (s < nslab) {
      const long k0 = rbeg + ((long)first + (long)s * stride) * DG_KS;
      dg_load_slab(As + s * DG_SLAB, A, i0, m, K, k0, rend);
      if (!SAME) dg_load_slab(Bs + s * DG_SLAB, B, j0, n, K, k0, rend);
    }
    dg_commit();
  }
  for (int s = 0; s < nslab; ++s) {
    dg_wait<DG_STAGES - 2>();
    __syncthreads();
    // refill the stage freed by slab s - 1
    {
      const int sn = s + DG_STAGES - 1;
      if (sn < nslab) {
        const int st = sn % DG_STAGES;
        const long k0 = rbeg + ((long)first + (long)sn * stride) * DG_KS;
        dg_load_slab(As + st * DG_SLAB, A, i0, m, K, k0, rend);
        if (!SAME) dg_load_slab(Bs + st * DG_SLAB, B, j0, n, K, k0, rend);
      }
      dg_commit();
    }
    const double* as = As + (s % DG_STAGES) * DG_SLAB;
    const double* bs = Bs + (s % DG_STAGES) * DG_SLAB;
    if (active) {
#pragma unroll
      for (int k4 = 0; k4 < DG_KS; k4 += 4) {
        double af[4], bf[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) af[q] = as[(wi + q * 8 + (lane >> 2)) * DG_LD + k4 + (lane & 3)];
#pragma unroll
        for (int q = 0; q < 4; ++q) bf[q] = bs[(wj + q * 8 + (lane >> 2)) * DG_LD + k4 + (lane & 3)];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) dg_dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
      }
    }
  }
  dg_wait<0>();
  if (!active) return;
  double* out = part + (size_t)kb * m * n;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = i0 + wi + a * 8 + (lane >> 2);
      const int j = j0 + wj + b * 8 + 2 * (lane & 3);
      if (i < m && j < n) out[(size_t)i * n + j] = acc[a][b][0];
      if (i < m && j + 1 < n) out[(size_t)i * n + j + 1] = acc[a][b][1];
    }
}

// C = alpha (w0 sum_{kb < n0} part[kb] + sum_{kb >= n0} part[kb]).  Block =
// 64 outputs x 4 partial groups (group g sums the partials kb = g mod 4 of
// each range); the groups are combined in a fixed order, so the result does
// not depend on scheduling.
#define DR_COLS 64
#define DR_GROUPS 4
__global__ void __launch_bounds__(DR_COLS * DR_GROUPS)
k_dgemm_fwd_reduce(const double* __restrict__ part, int n0, int nkb, size_t nn, double w0, double alpha,
                   double* __restrict__ C, const int* __restrict__ cond, int sym_n) {
  if (cond && *cond == 0) return;
  __shared__ double s0s[DR_GROUPS][DR_COLS], s1s[DR_GROUPS][DR_COLS];
  const int col = threadIdx.x % DR_COLS, g = threadIdx.x / DR_COLS;
  const size_t i = (size_t)blockIdx.x * DR_COLS + col;
  // sym_n > 0: symmetric n x n result whose partials hold only the 32 x 32
  // blocks on and above the diagonal; (r, c) below reads (c, r)
  size_t src = i;
  if (sym_n > 0 && i < nn) {
    const int r = (int)(i / sym_n), c = (int)(i - (size_t)r * sym_n);
    if ((r >> 5) > (c >> 5)) src = (size_t)c * sym_n + r;
  }
  double s0 = 0.0, s1 = 0.0;
  if (i < nn) {
    for (int k = g; k < n0; k += DR_GROUPS) s0 += __ldcs(part + (size_t)k * nn + src);
    int k = n0 + g;
    for (; k + 3 * DR_GROUPS < nkb; k += 4 * DR_GROUPS) {
      const double a = __ldcs(part + (size_t)k * nn + src);
      const double b = __ldcs(part + (size_t)(k + DR_GROUPS) * nn + src);
      const double c = __ldcs(part + (size_t)(k + 2 * DR_GROUPS) * nn + src);
      const double d = __ldcs(part + (size_t)(k + 3 * DR_GROUPS) * nn + src);
      s1 += a; s1 += b; s1 += c; s1 += d;
    }
    for (; k < nkb; k += DR_GROUPS) s1 += __ldcs(part + (size_t)k * nn + src);
  }
  s0s[g][col] = s0;
  s1s[g][col] = s1;
  __syncthreads();
  if (g == 0 && i < nn) {
    double t0 = 0.0, t1 = 0.0;
#pragma unroll
    for (int q = 0; q < DR_GROUPS; ++q) { t0 += s0s[q][col]; t1 += s1s[q][col]; }
    C[i] = alpha * (w0 * t0 + t1);
  }
}

#define DG_STAGES_SAME 4
#define DG_STAGES_TWO 3
size_t oa_dgemm_fwd_smem(bool same) {
  return same ? (size_t)DG_STAGES_SAME * DG_SLAB * sizeof(double) : (size_t)2 * DG_STAGES_TWO * DG_SLAB * sizeof(double);
}

// Returns cudaErrorNotSupported when the operands do not allow 16-byte
// copies (odd K, odd kx0_cols or unaligned pointers); the caller then uses
// the element-wise kernel.  nkb bounds the partials the caller provides
// (part holds nkb * m * n doubles).
// cond: optional device flag; when it is 0 at run time the launches do nothing
// (the conditional PsiV reset of the native step).
cudaError_t oa_dgemm_fwd(cudaStream_t s, const double* A, const double* B, int m, int n, long K, long kx0_cols,
                         double w_kx0, double alpha, double* part, int nkb, double* C, const int* cond) {
  if ((K & 1) || (kx0_cols & 1) || (((uintptr_t)A | (uintptr_t)B) & 15) || kx0_cols > K || nkb < 2)
    return cudaErrorNotSupported;
  // SM count of the current device (per call: processes may drive GPUs of
  // different sizes)
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0)
    nsm = 148;
  const int ti = (m + DG_TM - 1) / DG_TM, tj = (n + DG_TM - 1) / DG_TM;
  // about one CTA per SM; the kx0 region gets CTAs in proportion to its slabs
  const long s0 = (kx0_cols + DG_KS - 1) / DG_KS, sr = (K - kx0_cols + DG_KS - 1) / DG_KS;
  int nk = nsm / (ti * tj);
  if (nk > nkb) nk = nkb;
  if (nk < 2) nk = 2;
  int n0 = s0 > 0 ? (int)((nk * s0 + s0 + sr - 1) / (s0 + sr)) : 0;  // rounded up: no straggler
  if (s0 > 0 && n0 < 1) n0 = 1;
  if (n0 > s0) n0 = (int)s0;
  int nr = nk - n0;
  if (nr > sr) nr = (int)sr;
  if (sr > 0 && nr < 1) return cudaErrorNotSupported;
  const int nkb_eff = n0 + nr;
  if (nkb_eff < 1 || nkb_eff > nkb) return cudaErrorNotSupported;
  // one shared slab serves both operands only when the single output tile
  // is diagonal (A == B and m, n <= 128)
  const bool same = (A == B) && ti == 1 && tj == 1;
  const size_t sm = oa_dgemm_fwd_smem(same);
  dim3 grid(ti, tj, nkb_eff);
  cudaError_t e;
  if (same) {
    e = oa_smem_limit(k_dgemm_fwd<true, DG_STAGES_SAME>);
    if (e != cudaSuccess) return e;
    k_dgemm_fwd<true, DG_STAGES_SAME><<<grid, DG_THREADS, sm, s>>>(A, B, m, n, K, kx0_cols, n0, nr, part, cond);
  } else {
    e = oa_smem_limit(k_dgemm_fwd<false, DG_STAGES_TWO>);
    if (e != cudaSuccess) return e;
    k_dgemm_fwd<false, DG_STAGES_TWO><<<grid, DG_THREADS, sm, s>>>(A, B, m, n, K, kx0_cols, n0, nr, part, cond);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t mn = (size_t)m * n;
  k_dgemm_fwd_reduce<<<(unsigned)((mn + DR_COLS - 1) / DR_COLS), DR_COLS * DR_GROUPS, 0, s>>>(
      part, n0, nkb_eff, mn, w_kx0, alpha, C, cond, same ? n : 0);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Backward product (PairCalculator::multiplyResult / bwMultiplyHelper /
// bwMultiplyDynOrthoT, ckPairCalculator.C:1201-1468, 1710-2031):
//   out[j][c] = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c]
//   a1(c) = a1_kx0 for c < kx0_cols, else a1_rest
// CTA tile: 128 rows j x 64 columns c, all k; 8 warps of 32 x 32.  The M and
// X slabs of 16 k rows move through a 4-stage cp.async ring; the two terms
// run as one slab sequence.  The first term's sum is scaled by a1(c) in
// registers once it is complete; the second term's M fragments are scaled
// by a2 as they are read, so one accumulator set serves both terms.
// ---------------------------------------------------------------------------
#define DB_TJ 128
#define DB_TC 64
#define DB_KS 16
#define DB_LDM (DB_TJ + 4)
#define DB_LDX (DB_TC + 4)
#define DB_STAGES 4
#define DB_THREADS 256
#define DB_MSLAB (DB_KS * DB_LDM)
#define DB_XSLAB (DB_KS * DB_LDX)

__device__ __forceinline__ void db_load_slab(double* ms, double* xs, const double* __restrict__ M,
                                             const double* __restrict__ X, int nj, int nk, long ncol, int k0,
                                             long c0, int j0) {
  if (nj & 1) {
    // odd nj: the rows of M are not 16-byte aligned; 8-byte pieces, 8 per thread
#pragma unroll
    for (int q = 0; q < (DB_KS * DB_TJ) / DB_THREADS; ++q) {
      const int piece = threadIdx.x + q * DB_THREADS;
      const int kk = piece >> 7, jj = piece & 127;
      const int k = k0 + kk;
      const bool valid = (k < nk) && (j0 + jj < nj);
      dg_cp8(ms + kk * DB_LDM + jj, valid ? M + (size_t)k * nj + j0 + jj : M, valid);
    }
  } else {
    // M rows k0..k0+15, all 128 j: 16 x 64 pieces of 16 B = 1024 -> 4 per thread
#pragma unroll
    for (int q = 0; q < (DB_KS * DB_TJ / 2) / DB_THREADS; ++q) {
      const int piece = threadIdx.x + q * DB_THREADS;
      const int kk = piece >> 6, jj = (piece & 63) * 2;
      const int k = k0 + kk;
      const bool valid = (k < nk) && (j0 + jj < nj);
      dg_cp16(ms + kk * DB_LDM + jj, valid ? M + (size_t)k * nj + j0 + jj : M, valid);
    }
  }
  // X rows k0..k0+15, columns c0..c0+63: 16 x 32 pieces = 512 -> 2 per thread
#pragma unroll
  for (int q = 0; q < (DB_KS * DB_TC / 2) / DB_THREADS; ++q) {
    const int piece = threadIdx.x + q * DB_THREADS;
    const int kk = piece >> 5, cc = (piece & 31) * 2;
    const int k = k0 + kk;
    const long c = c0 + cc;
    const bool valid = (k < nk) && (c < ncol);
    dg_cp16(xs + kk * DB_LDX + cc, valid ? X + (size_t)k * ncol + c : X, valid);
  }
}

// Epilogue options: yadd (optional) adds yadd[j][c] to the result (it may
// be the output array itself: each element is read and written by one
// thread); out2 (optional) receives a second copy of the result when
// *cond2 != 0; vel (optional, when *vcond != 0) receives the finite
// difference (result - previous out) vscale, previous out read by the
// thread that overwrites it.
template <bool TWO>
__global__ void __launch_bounds__(DB_THREADS, 2)
k_dgemm_bwd(const double* __restrict__ M1, const double* __restrict__ X1, double a1_kx0, double a1_rest,
            const double* __restrict__ M2, const double* __restrict__ X2, double a2, int nj, int nk, long ncol,
            long kx0_cols, double* out, const int* __restrict__ cond, const double* yadd, double* __restrict__ out2,
            const int* __restrict__ cond2, OaPlaneOut po, double* __restrict__ vel, double vscale,
            const int* __restrict__ vcond) {
  if (cond && *cond == 0) return;
  const bool dual = out2 && *cond2 != 0;
  const bool velo = vel && *vcond != 0;
  extern __shared__ __align__(16) double db_smem[];
  double* Ms = db_smem;
  double* Xs = db_smem + DB_STAGES * DB_MSLAB;
  const long c0 = (long)blockIdx.x * DB_TC;
  const int j0 = blockIdx.y * DB_TJ;  // rows j0 .. j0 + 127 of the output
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wj = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int nsl = (nk + DB_KS - 1) / DB_KS;
  const int ntot = TWO ? 2 * nsl : nsl;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) { acc[a][b][0] = 0.0; acc[a][b][1] = 0.0; }
  auto issue = [&](int s) {
    const int st = s % DB_STAGES;
    const bool second = TWO && s >= nsl;
    const int k0 = (second ? s - nsl : s) * DB_KS;
    db_load_slab(Ms + st * DB_MSLAB, Xs + st * DB_XSLAB, second ? M2 : M1, second ? X2 : X1, nj, nk, ncol, k0, c0,
                 j0);
  };
  // a1(c) for this thread's output columns
  auto scale_a1 = [&]() {
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const long c = c0 + wc + b * 8 + 2 * (lane & 3) + e;
        const double a1 = (c < kx0_cols) ? a1_kx0 : a1_rest;
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[a][b][e] *= a1;
      }
  };
#pragma unroll
  for (int s = 0; s < DB_STAGES - 1; ++s) {
    if (s < ntot) issue(s);
    dg_commit();
  }
  for (int s = 0; s < ntot; ++s) {
    dg_wait<DB_STAGES - 2>();
    __syncthreads();
    if (s + DB_STAGES - 1 < ntot) issue(s + DB_STAGES - 1);
    dg_commit();
    if (TWO && s == nsl) scale_a1();
    const double sa = (TWO && s >= nsl) ? a2 : 1.0;
    const double* ms = Ms + (s % DB_STAGES) * DB_MSLAB;
    const double* xs = Xs + (s % DB_STAGES) * DB_XSLAB;
#pragma unroll
    for (int k4 = 0; k4 < DB_KS; k4 += 4) {
      double af[4], bf[4];
      // A[j][k] = M[k][j] (row-major 8 x 4 fragment), B[k][c] = X[k][c]
#pragma unroll
      for (int q = 0; q < 4; ++q) af[q] = ms[(k4 + (lane & 3)) * DB_LDM + wj + q * 8 + (lane >> 2)] * sa;
#pragma unroll
      for (int q = 0; q < 4; ++q) bf[q] = xs[(k4 + (lane & 3)) * DB_LDX + wc + q * 8 + (lane >> 2)];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dg_dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
  }
  dg_wait<0>();
  if (!TWO) scale_a1();
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int j = j0 + wj + a * 8 + (lane >> 2);
    if (j >= nj) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const long c = c0 + wc + b * 8 + 2 * (lane & 3);
      const size_t o = (size_t)j * ncol + c;
      if (c + 1 < ncol) {
        double2 v = make_double2(acc[a][b][0], acc[a][b][1]);
        if (yadd) { const double2 y = *(const double2*)(yadd + o); v.x += y.x; v.y += y.y; }
        if (velo) {
          const double2 p = *(const double2*)(out + o);
          *(double2*)(vel + o) = make_double2(fma(v.x, vscale, p.x * -vscale), fma(v.y, vscale, p.y * -vscale));
        }
        *(double2*)(out + o) = v;
        if (dual) *(double2*)(out2 + o) = v;
      } else if (c < ncol) {
        double v = acc[a][b][0];
        if (yadd) v += yadd[o];
        if (velo) vel[o] = fma(v, vscale, out[o] * -vscale);
        out[o] = v;
        if (dual) out2[o] = v;
      }
    }
  }
  if (po.P) {
    // bf16 planes of the tile staged in the (now idle) slab ring, then
    // written as whole 16-byte pieces of 128-byte rows
    constexpr int SPLD = DB_TC + 8;
    __nv_bfloat16* sp = reinterpret_cast<__nv_bfloat16*>(db_smem);
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int jl = wj + a * 8 + (lane >> 2);
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int cl = wc + b * 8 + 2 * (lane & 3);
        __nv_bfloat16 hx[3], hy[3];
        oa_bf16_digits(acc[a][b][0], po.nt, hx);
        oa_bf16_digits(acc[a][b][1], po.nt, hy);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          if (q >= po.nt) break;
          __nv_bfloat162 v2;
          v2.x = hx[q];
          v2.y = hy[q];
          *reinterpret_cast<__nv_bfloat162*>(sp + ((size_t)q * DB_TJ + jl) * SPLD + cl) = v2;
        }
      }
    }
    __syncthreads();
    const size_t pstride = (size_t)po.rows_pad * po.ldp;
    for (int i = threadIdx.x; i < po.nt * DB_TJ * (DB_TC / 8); i += DB_THREADS) {
      const int q = i / (DB_TJ * (DB_TC / 8)), rem = i - q * (DB_TJ * (DB_TC / 8));
      const int jl = rem / (DB_TC / 8), ch = rem - jl * (DB_TC / 8);
      if (j0 + jl >= nj || c0 + ch * 8 >= po.ldp) continue;
      *reinterpret_cast<uint4*>((__nv_bfloat16*)po.P + q * pstride +
                                oa_plane_at(j0 + jl, c0 + ch * 8, po.rows_pad)) =
          *reinterpret_cast<const uint4*>(sp + ((size_t)q * DB_TJ + jl) * SPLD + ch * 8);
    }
  }
}

// Returns cudaErrorNotSupported when the shapes or pointers do not allow the
// copies (odd ncol, unaligned pointers); an odd nj moves M in 8-byte pieces.
// Outputs of more than 128 rows run as row tiles of 128 (grid y).
// po (optional): bf16 planes of out written in the same pass (ncol even).
cudaError_t oa_dgemm_bwd_ex(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                            const double* M2, const double* X2, double a2, int nj, int nk, long ncol, long kx0_cols,
                            double* out, const int* cond, const double* yadd, double* out2, const int* cond2,
                            const OaPlaneOut* po, double* vel, double vscale, const int* vcond) {
  const OaPlaneOut pz = po ? *po : OaPlaneOut{nullptr, 0, 0, 0};
  if (vel && (!vcond || yadd || M2)) return cudaErrorInvalidValue;
  // plane tiles are whole 64-column pieces inside the plane rows
  if (pz.P && ((pz.ldp % DB_TC) || ncol > pz.ldp || nj > pz.rows_pad || pz.nt > 3)) return cudaErrorInvalidValue;
  const uintptr_t al = (uintptr_t)M1 | (uintptr_t)X1 | (uintptr_t)out | (uintptr_t)(M2 ? M2 : M1) |
                       (uintptr_t)(X2 ? X2 : X1) | (uintptr_t)yadd | (uintptr_t)out2 | (uintptr_t)vel;
  if (out2 && !cond2) return cudaErrorInvalidValue;
  if (nj <= 0 || (ncol & 1) || (al & 15) || nk <= 0 || (M2 && !X2)) return cudaErrorNotSupported;
  const size_t sm = (size_t)DB_STAGES * (DB_MSLAB + DB_XSLAB) * sizeof(double);
  // column tiles of 64 by row tiles of 128
  dim3 grid((unsigned)((ncol + DB_TC - 1) / DB_TC), (unsigned)((nj + DB_TJ - 1) / DB_TJ));
  cudaError_t e;
  if (M2) {
    e = oa_smem_limit(k_dgemm_bwd<true>);
    if (e != cudaSuccess) return e;
    k_dgemm_bwd<true><<<grid, DB_THREADS, sm, s>>>(M1, X1, a1_kx0, a1_rest, M2, X2, a2, nj, nk, ncol, kx0_cols, out,
                                                    cond, yadd, out2, cond2, pz, vel, vscale, vcond);
  } else {
    e = oa_smem_limit(k_dgemm_bwd<false>);
    if (e != cudaSuccess) return e;
    k_dgemm_bwd<false><<<grid, DB_THREADS, sm, s>>>(M1, X1, a1_kx0, a1_rest, M2, X2, a2, nj, nk, ncol, kx0_cols,
                                                     out, cond, yadd, out2, cond2, pz, vel, vscale, vcond);
  }
  return cudaGetLastError();
}

cudaError_t oa_dgemm_bwd(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                         const double* M2, const double* X2, double a2, int nj, int nk, long ncol, long kx0_cols,
                         double* out, const int* cond) {
  return oa_dgemm_bwd_ex(s, M1, X1, a1_kx0, a1_rest, M2, X2, a2, nj, nk, ncol, kx0_cols, out, cond, nullptr, nullptr,
                         nullptr, nullptr, nullptr, 0.0, nullptr);
}
