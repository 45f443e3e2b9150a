// FP64-accurate PairCalculator products on the int8 tensor cores (mixed
// form): the overlap S = alpha sum_g w_g Psi~ Psi~^T of the integrated,
// non-orthogonal states and the rotation psi = Psi~ T that orthonormalises
// them.  Both keep FP64 accuracy (relative error about 2^-42 of the largest
// element of a K range), so the mixed step still reaches ||S/2 - I|| at the
// FP64 level while the products run as exact integer MMAs.
//
// Reference work replaced (the FP64 DGEMMs of the symmetric PairCalculator):
//   PairCalculator::multiplyForward, symmetric S (ckPairCalculator.C:821-893)
//     + contributeSubTiles / sumMatrixDouble (:20-53, 938-1016)       -> k_oz_syrk + k_oz_reduce
//   PairCalculator::bwMultiplyHelper, psi = Psi T ('N','N', :1710-1946) -> k_oz_tslice + k_oz_rot
//
// Method (Ozaki's error-free splitting of the operands into digits, run on
// integer matrix units: Ozaki, Ogita, Oishi, Rump, Numer. Algorithms 59
// (2012); Ootomo, Ozaki, Yokota, IJHPCA 38 (2024)).  In a K range whose
// largest |x| is below 2^e every value is written as
//     x = 2^(e-6) (d_0 + d_1 / 128 + ... + d_5 / 128^5) + r,
//     d_q integers in [-64, 64],  |r| <= 2^(e-42),
// the digits stored as int8 ("slices").  A product of two such operands is
//     sum_{s,t} 2^(-7 (s + t)) (D_s^T D_t)   scaled by the two exponents,
// where every D_s^T D_t is exact in int32 (tcgen05.mma.kind::i8).  The
// eight digit levels l = s + t <= 7 (30 digit products) accumulate in eight
// TMEM accumulators of N = 64 columns (all 512 columns) and are combined in
// FP64 in the epilogue.  Levels up to 7, not 5: a value well below its
// range's maximum has leading zero digits, and a product of two such values
// starts at a later level; with eight levels every product keeps at least
// 42 bits of its own magnitude (the off-diagonal entries of T are 1e-3 of
// the diagonal ones, two leading zero digits).
//
// Layout.  The real view of Psi~ [rows][K] (K = 2 ng doubles) is cut into
// 128-column chunks: the kx = 0 columns [0, kA) padded to nA chunks, then the
// rest padded to nB chunks (the kx = 0 weight applies per chunk).  Slices are
// int8 [6][nA + nB][128 rows][128], so that a chunk of one slice is one 16 KB
// TMA box with the 128-byte swizzle, read as the K-major operand of S (rows
// = states, 128 B of K) and as the MN-major operand of the rotation (rows =
// K = states, 128 B of M = g-columns).  Chunks are grouped into R ranges
// (never across the kx = 0 boundary); each range has its own exponent per
// state row, is one split-K unit of S and selects the scaled copy of T the
// rotation uses: T'_r[i][j] = T[i][j] 2^(e_ri - 6), itself split into seven
// digit slices per column j (exponent f_rj), int8 [R][7][128 j][128 i].
//
// Every mbarrier wait is bounded (oa_wait.cuh); on a timeout the block sets
// the device error flag, lets its copies land, frees TMEM and returns.  No
// multicast.
#include <cuda.h>
#include <algorithm>
#include <mutex>
#include <vector>
#include "oa_internal.h"
#include "oa_wait.cuh"

#define OZ_ND 6                 // digits per value of the states
#define OZ_NDT 7                // digits per value of T' (the rotation's other operand)
#define OZ_NL 8                 // digit levels kept (s + t <= 7)
#define OZ_CH 128               // columns per chunk
#define OZ_TILE (128 * OZ_CH)   // bytes of one slice chunk (128 rows)
#define OZ_N 64                 // N of the MMAs
#define OZ_THREADS 128
#define OZ_TLD 132              // padded row of the T' digit staging

__device__ __forceinline__ uint32_t oz_s32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, 128-byte swizzle, sm100 version bit
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
// instruction descriptor of kind::i8: S32 accumulate, signed int8 A and B,
// M = 128, N = OZ_N; a_mn / b_mn select the MN-major operand layouts
__host__ __device__ constexpr uint32_t oz_idesc(int a_mn, int b_mn) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(OZ_N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void oz_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void oz_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(oz_s32(bar)) : "memory");
}
__device__ __forceinline__ void oz_bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(oz_s32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void oz_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(oz_s32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool oz_wait(uint64_t* bar, uint32_t phase) {
  return oa_mbar_wait_bounded(oz_s32(bar), phase);
}
// 4-D tile load {c0, c1, c2, c3} of the map's box into shared memory
__device__ __forceinline__ void oz_tma(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                       uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];"
      :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(oz_s32(bar))
      : "memory");
}
__device__ __forceinline__ void oz_tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void oz_tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void oz_tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(oz_s32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void oz_tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
// 16 consecutive int32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void oz_tmem_ld16(uint32_t taddr, int* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = (int)r[i];
}

// exponent marking a range or column with a non-finite value: the products
// that use it come out NaN (the step's Newton-Schulz check reports it)
#define OZ_BAD 0x40000000

// exponent e with |x| < 2^e for all |x| <= m (0 for m == 0)
__device__ __forceinline__ int oz_exponent(double m) {
  if (!(m > 0.0)) return 0;
  int e;
  frexp(m, &e);  // m = f 2^e, f in [0.5, 1)
  return e;
}
// the ND digits of x 2^(6 - e), |x| < 2^e
template <int ND = OZ_ND>
__device__ __forceinline__ void oz_digits(double x, int e, signed char* d) {
  double t = ldexp(x, 6 - e);
#pragma unroll
  for (int q = 0; q < ND; ++q) {
    const double r = rint(t);
    d[q] = (signed char)(int)r;
    t = (t - r) * 128.0;
  }
}

// chunk-space column -> real-view column (or -1 for padding)
struct OzMap {
  int nA, nB;
  long kA, K;
};
__device__ __forceinline__ long oz_col(const OzMap& m, long cs) {
  if (cs < (long)m.nA * OZ_CH) return cs < m.kA ? cs : -1;
  const long c = m.kA + (cs - (long)m.nA * OZ_CH);
  return c < m.K ? c : -1;
}

// ---------------------------------------------------------------------------
// k_oz_slice: block (range r, row i < rows): stage the range of row i in
// shared memory, its max |x| -> e[r][i], then the six digit slices.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_oz_slice(const double* __restrict__ X, long ldx, OzMap m, const int* __restrict__ rc, int nch,
           signed char* __restrict__ sl, int* __restrict__ ex) {
  extern __shared__ __align__(16) double oz_row[];
  __shared__ double red[8];
  const int r = blockIdx.x, i = blockIdx.y;
  const int c0 = rc[r], c1 = rc[r + 1];
  const long n = (long)(c1 - c0) * OZ_CH;
  const double* xi = X + (size_t)i * ldx;
  double mx = 0.0;
  for (long t = threadIdx.x; t < n; t += blockDim.x) {
    const long c = oz_col(m, (long)c0 * OZ_CH + t);
    const double v = c >= 0 ? xi[c] : 0.0;
    oz_row[t] = v;
    // a NaN or Inf makes the maximum infinite
    mx = isfinite(v) ? fmax(mx, fabs(v)) : (double)INFINITY;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  mx = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, red[w]);
  const bool bad = !isfinite(mx);
  const int e = bad ? 0 : oz_exponent(mx);
  if (threadIdx.x == 0) ex[r * 128 + i] = bad ? OZ_BAD : e;
  // four consecutive columns per thread: one 4-byte store per slice
  const size_t pstride = (size_t)nch * OZ_TILE;
  for (long t = 4 * threadIdx.x; t < n; t += 4 * blockDim.x) {
    signed char d[4][OZ_ND];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (bad) {
#pragma unroll
        for (int q = 0; q < OZ_ND; ++q) d[u][q] = 0;
      } else {
        oz_digits(oz_row[t + u], e, d[u]);
      }
    }
    const long cs = (long)c0 * OZ_CH + t;
    signed char* dst = sl + (size_t)(cs / OZ_CH) * OZ_TILE + (size_t)i * OZ_CH + (cs % OZ_CH);
#pragma unroll
    for (int q = 0; q < OZ_ND; ++q) {
      char4 v;
      v.x = d[0][q]; v.y = d[1][q]; v.z = d[2][q]; v.w = d[3][q];
      *reinterpret_cast<char4*>(dst + q * pstride) = v;
    }
  }
}

// ---------------------------------------------------------------------------
// k_oz_tslice: block r: T'_r[i][j] = T[i][j] 2^(e_ri - 6) for i, j < n, its
// column exponents f[r][j] and seven digit slices tsl[r][q][j][i] (zero
// beyond n).  Seven, not six: each output of the rotation sums 128 products
// whose T' digits are cut relative to the column's largest (diagonal) entry.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
k_oz_tslice(const double* __restrict__ T, int n, const int* __restrict__ ex, signed char* __restrict__ tsl,
            int* __restrict__ fx) {
  // digits staged as [OZ_NDT][128 j][OZ_TLD i]: rows padded to 132 bytes so
  // that the byte writes of 32 threads (32 columns j) fall in 32 banks
  extern __shared__ __align__(16) signed char oz_tb[];
  const int r = blockIdx.x, j = threadIdx.x;
  double mx = 0.0;
  bool bad = false;
  if (j < n)
    for (int i = 0; i < n; ++i) {
      const int e = ex[r * 128 + i];
      const double v = T[(size_t)i * n + j];
      if (e == OZ_BAD || !isfinite(v)) bad = true;
      else mx = fmax(mx, fabs(ldexp(v, e - 6)));
    }
  const int f = oz_exponent(mx);
  fx[r * 128 + j] = bad ? OZ_BAD : f;
  for (int i = 0; i < 128; ++i) {
    signed char d[OZ_NDT];
#pragma unroll
    for (int q = 0; q < OZ_NDT; ++q) d[q] = 0;
    if (!bad && j < n && i < n) oz_digits<OZ_NDT>(ldexp(T[(size_t)i * n + j], ex[r * 128 + i] - 6), f, d);
#pragma unroll
    for (int q = 0; q < OZ_NDT; ++q) oz_tb[(q * 128 + j) * OZ_TLD + i] = d[q];
  }
  __syncthreads();
  // rows of 32 words to global, 32 consecutive words per warp
  int* dst = reinterpret_cast<int*>(tsl + (size_t)r * OZ_NDT * OZ_TILE);
  const int* src = reinterpret_cast<const int*>(oz_tb);
  for (int t = threadIdx.x; t < OZ_NDT * 128 * 32; t += blockDim.x) {
    const int row = t >> 5, w = t & 31;
    dst[t] = src[row * (OZ_TLD / 4) + w];
  }
}

// ---------------------------------------------------------------------------
// k_oz_syrk: CTA (range r, column half h): D_l[i][j] = sum over the range's
// chunks of sum_{s+t=l} d_s[i] d_t[j] for all 128 rows i and the 64 columns
// j of half h, then part[r][i][j] = alpha w_r 2^(e_ri + e_rj - 12) sum_l 2^(-7l) D_l.
// One thread issues the TMA loads (all six slices of a chunk per stage) and
// the MMAs; the B operand is rows [64h, 64h + 64) of the same tile.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(OZ_THREADS, 1)
k_oz_syrk(const __grid_constant__ CUtensorMap tS, const int* __restrict__ rc, int RA, const int* __restrict__ ex,
          int n, double alpha, double w_kx0, int stages, double* __restrict__ part, int* __restrict__ err_flag,
          const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  const int r = blockIdx.x, h = blockIdx.y;
  if (h * OZ_N >= n) return;
  extern __shared__ __align__(1024) unsigned char oz_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)oz_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t stage_bytes = OZ_ND * OZ_TILE;
  uint64_t* full = (uint64_t*)(base + (size_t)stages * stage_bytes);
  uint64_t* empty = full + stages;
  uint32_t* tslot = (uint32_t*)(empty + stages);
  int* okflag = (int*)(tslot + 1);
  int* ecol = okflag + 1;  // [OZ_N]
  const int tid = threadIdx.x, warp = tid >> 5;
  const int c0 = rc[r], nslab = rc[r + 1] - c0;
  constexpr uint32_t ncols = 512;  // eight accumulators of OZ_N columns
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) { oz_bar_init(&full[s], 1); oz_bar_init(&empty[s], 1); }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *okflag = 1;
  }
  if (tid < OZ_N) ecol[tid] = ex[r * 128 + h * OZ_N + tid];
  if (warp == 0) oz_tmem_alloc(tslot, ncols);
  __syncthreads();
  oz_tc_after();
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    constexpr uint32_t idesc = oz_idesc(0, 0);
    const uint32_t sbase = oz_s32(base);
    auto issue = [&](int sl, int st) {
      const uint32_t sb = sbase + st * stage_bytes;
      oz_expect_tx(&full[st], stage_bytes);
#pragma unroll
      for (int q = 0; q < OZ_ND; ++q) oz_tma(sb + q * OZ_TILE, &tS, 0, 0, c0 + sl, q, &full[st]);
    };
    bool ok = true;
    const int pre = nslab < stages ? nslab : stages;
    for (int s = 0; s < pre; ++s) issue(s, s);
    int issued = pre, committed = -1;
    for (int sl = 0; sl < nslab && ok; ++sl) {
      const int st = sl % stages;
      const uint32_t ph = (uint32_t)(sl / stages) & 1u;
      if (!oz_wait(&full[st], ph)) { ok = false; break; }
      oz_tc_after();
      const uint32_t sb = sbase + st * stage_bytes;
      // K-major, 128-byte swizzle: rows 128 B apart, 8-row groups 1024 B
      // apart (SBO); the four K steps of 32 int8 are 32 B apart in a row
#pragma unroll
      for (int ks = 0; ks < OZ_CH / 32; ++ks)
#pragma unroll
        for (int s = 0; s < OZ_ND; ++s)
#pragma unroll
          for (int t = 0; t < OZ_ND; ++t) {
            if (s + t >= OZ_NL) continue;
            const uint64_t da = oz_desc(sb + s * OZ_TILE + ks * 32, 16, 1024);
            const uint64_t db = oz_desc(sb + t * OZ_TILE + h * OZ_N * OZ_CH + ks * 32, 16, 1024);
            // the first MMA into level l = s + t overwrites it: in the first K
            // step of the first chunk, the pair with the smallest s
            // (s = max(0, l - 5))
            const int sfirst = s + t > OZ_ND - 1 ? s + t - (OZ_ND - 1) : 0;
            const uint32_t acc = (sl > 0 || ks > 0 || s > sfirst) ? 1u : 0u;
            oz_mma(tmem + (uint32_t)((s + t) * OZ_N), da, db, idesc, acc);
          }
      oz_commit(&empty[st]);
      committed = sl;
      if (issued < nslab) {
        if (!oz_wait(&empty[st], ph)) { ok = false; break; }
        issue(issued, st);
        ++issued;
      }
    }
    if (ok && nslab > 0) {
      const int sl = nslab - 1;
      if (!oz_wait(&empty[sl % stages], (uint32_t)(sl / stages) & 1u)) ok = false;
    }
    if (!ok) {
      for (int s2 = 0; s2 < stages && s2 < issued; ++s2) {
        const int last = issued - 1 - ((issued - 1 - s2) % stages);
        (void)oz_wait(&full[s2], (uint32_t)(last / stages) & 1u);
      }
      if (committed >= 0) (void)oz_wait(&empty[committed % stages], (uint32_t)(committed / stages) & 1u);
      *okflag = 0;
    }
  }
  __syncthreads();
  oz_tc_after();
  const bool ok = *okflag != 0;
  const int i = warp * 32 + (tid & 31);  // TMEM lane = row i
  const double wr = alpha * (r < RA ? w_kx0 : 1.0);
  const int ei = ex[r * 128 + i];
  double* out = part + ((size_t)r * 128 + i) * 128 + h * OZ_N;
  for (int cb = 0; cb < OZ_N; cb += 16) {
    double v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = 0.0;
    if (ok && nslab > 0) {
#pragma unroll
      for (int l = OZ_NL - 1; l >= 0; --l) {
        int d[16];
        oz_tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(l * OZ_N + cb), d);
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = fma(v[c], 1.0 / 128.0, (double)d[c]);
      }
    }
    // v = sum_l 2^(-7 l) D_l, summed from the smallest level up
#pragma unroll
    for (int c = 0; c < 16; ++c)
      out[cb + c] = (ei == OZ_BAD || ecol[cb + c] == OZ_BAD) ? (double)NAN : wr * ldexp(v[c], ei + ecol[cb + c] - 12);
  }
  if (!ok && tid == 0) atomicExch(err_flag, 1);
  oz_tc_before();
  __syncthreads();
  if (warp == 0) oz_tmem_dealloc(tmem, ncols);
}

// C[i][j] = sum_r part[r][i][j] (i, j < n), in range order
__global__ void k_oz_reduce(const double* __restrict__ part, int R, int n, double* __restrict__ C,
                            const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * n) return;
  const int i = t / n, j = t - i * n;
  double s = 0.0;
  for (int r = 0; r < R; ++r) s += part[((size_t)r * 128 + i) * 128 + j];
  C[(size_t)i * n + j] = s;
}

// ---------------------------------------------------------------------------
// k_oz_rot: CTA (chunk c, column half h): out[j][col] = sum_i T[i][j] X[i][col]
// for the 128 columns of chunk c and j in half h:
//   D_l[k][j] = sum_{s+t=l} sum_i d_s[i][k] b_t[r(c)][j][i],
//   out = 2^(f_rj - 6) sum_l 2^(-7l) D_l,
// A = the slice chunks of X read MN-major (rows = i, 128 B of k), B = the
// digit slices of T'_r read K-major.  Also writes the bf16 planes of out.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(OZ_THREADS, 1)
k_oz_rot(const __grid_constant__ CUtensorMap tS, const __grid_constant__ CUtensorMap tT,
         const int* __restrict__ cr, const int* __restrict__ fx, OzMap m, int n, long ldo,
         double* __restrict__ out, OaPlaneOut po, int* __restrict__ err_flag, const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  const int c = blockIdx.x, h = blockIdx.y;
  if (h * OZ_N >= n) return;
  extern __shared__ __align__(1024) unsigned char oz_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)oz_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t a_bytes = OZ_ND * OZ_TILE, b_bytes = OZ_NDT * OZ_N * 128;
  uint64_t* full = (uint64_t*)(base + a_bytes + b_bytes);
  uint64_t* done = full + 1;
  uint32_t* tslot = (uint32_t*)(done + 1);
  int* okflag = (int*)(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r = cr[c];
  constexpr uint32_t ncols = 512;
  if (tid == 0) {
    oz_bar_init(full, 1);
    oz_bar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *okflag = 1;
  }
  if (warp == 0) oz_tmem_alloc(tslot, ncols);
  __syncthreads();
  oz_tc_after();
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    const uint32_t sa = oz_s32(base), sb = sa + a_bytes;
    oz_expect_tx(full, a_bytes + b_bytes);
#pragma unroll
    for (int q = 0; q < OZ_ND; ++q) oz_tma(sa + q * OZ_TILE, &tS, 0, 0, c, q, full);
#pragma unroll
    for (int q = 0; q < OZ_NDT; ++q) oz_tma(sb + q * OZ_N * 128, &tT, 0, h * OZ_N, q, r, full);
    bool ok = oz_wait(full, 0u);
    if (ok) {
      oz_tc_after();
      // A MN-major: 128-byte rows along i, 8-row K groups 1024 B apart (SBO),
      // K steps of 32 rows 4096 B apart; one 128-wide MN chunk (LBO unused).
      // B K-major as in k_oz_syrk.
      constexpr uint32_t idesc = oz_idesc(1, 0);
#pragma unroll
      for (int ks = 0; ks < 128 / 32; ++ks)
#pragma unroll
        for (int s = 0; s < OZ_ND; ++s)
#pragma unroll
          for (int t = 0; t < OZ_NDT; ++t) {
            if (s + t >= OZ_NL) continue;
            const uint64_t da = oz_desc(sa + s * OZ_TILE + ks * 4096, OZ_TILE, 1024);
            const uint64_t db = oz_desc(sb + t * OZ_N * 128 + ks * 32, 16, 1024);
            const int sfirst = s + t > OZ_NDT - 1 ? s + t - (OZ_NDT - 1) : 0;
            const uint32_t acc = (ks > 0 || s > sfirst) ? 1u : 0u;
            oz_mma(tmem + (uint32_t)((s + t) * OZ_N), da, db, idesc, acc);
          }
      oz_commit(done);
      if (!oz_wait(done, 0u)) ok = false;
    } else {
      // the loads were issued: let them land before the block exits
      (void)oz_wait(full, 0u);
    }
    if (!ok) *okflag = 0;
  }
  __syncthreads();
  oz_tc_after();
  const bool ok = *okflag != 0;
  const int k = warp * 32 + (tid & 31);  // TMEM lane = column k of the chunk
  const long col = oz_col(m, (long)c * OZ_CH + k);
  for (int cb = 0; cb < OZ_N; cb += 16) {
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = 0.0;
    if (ok) {
#pragma unroll
      for (int l = OZ_NL - 1; l >= 0; --l) {
        int d[16];
        oz_tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(l * OZ_N + cb), d);
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = fma(v[q], 1.0 / 128.0, (double)d[q]);
      }
    }
    if (col >= 0) {
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int j = h * OZ_N + cb + q;
        if (j < n) {
          const int f = fx[r * 128 + j];
          const double y = f == OZ_BAD ? (double)NAN : ldexp(v[q], f - 6);
          out[(size_t)j * ldo + col] = y;
          if (po.P) {
            __nv_bfloat16 hd[3];
            oa_bf16_digits(y, po.nt, hd);
            __nv_bfloat16* pb = (__nv_bfloat16*)po.P + oa_plane_at(j, col, po.rows_pad);
            const size_t pstride = (size_t)po.rows_pad * po.ldp;
            for (int qq = 0; qq < po.nt; ++qq) pb[qq * pstride] = hd[qq];
          }
        }
      }
    }
  }
  if (!ok && tid == 0) atomicExch(err_flag, 1);
  oz_tc_before();
  __syncthreads();
  if (warp == 0) oz_tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*OzEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                               const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static OzEncodeFn oz_encoder() {
  static std::once_flag once;
  static OzEncodeFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (OzEncodeFn)p;
    cudaGetLastError();
  });
  return fn;
}

// int8 tensor {128, rows, d2, d3} (128-byte rows), box {128, br, 1, 1}, 128-byte swizzle
static bool oz_map(CUtensorMap* map, const void* P, int rows, long d2, long d3, int br) {
  OzEncodeFn enc = oz_encoder();
  if (!enc || (((uintptr_t)P) & 15) || br > 256 || rows % br) return false;
  const cuuint64_t dims[4] = {128, (cuuint64_t)rows, (cuuint64_t)d2, (cuuint64_t)d3};
  const cuuint64_t strides[3] = {128, (cuuint64_t)rows * 128, (cuuint64_t)rows * 128 * (cuuint64_t)d2};
  const cuuint32_t box[4] = {128, (cuuint32_t)br, 1, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<void*>(P), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

struct oa_oz {
  OzMap map;
  int nch, R, RA, n;
  int* rc;              // [R + 1] first chunk of each range
  int* cr;              // [nch] range of each chunk
  signed char* sl;      // [6][nch][128][128]
  signed char* tsl;     // [R][OZ_NDT][128][128]
  int* ex;              // [R][128]
  int* fx;              // [R][128]
  double* part;         // [R][128][128]
  const double* src;    // the operand the slices hold (for the rotation)
  CUtensorMap tS, tT;
  int stages;
  int maxlen;           // chunks of the longest range
};

static size_t oz_syrk_smem(int stages) { return (size_t)stages * OZ_ND * OZ_TILE + 1024 + 1024; }
static size_t oz_rot_smem() { return (size_t)OZ_ND * OZ_TILE + (size_t)OZ_NDT * OZ_N * 128 + 1024 + 256; }

void oa_oz_free(oa_oz* z) {
  if (!z) return;
  void* p[] = {z->rc, z->cr, z->sl, z->tsl, z->ex, z->fx, z->part};
  for (void* q : p) if (q) cudaFree(q);
  free(z);
}

// Set up the int8 products for n <= 128 states over ng g-points with nkx0
// on the kx = 0 plane; nullptr when not available (the caller keeps FP64).
oa_oz* oa_oz_create(int n, int ng, int nkx0, int nsm) {
  if (n < 1 || n > 128 || !oz_encoder()) return nullptr;
  oa_oz* z = (oa_oz*)calloc(1, sizeof(oa_oz));
  if (!z) return nullptr;
  z->n = n;
  z->map.kA = 2L * nkx0;
  z->map.K = 2L * ng;
  z->map.nA = (int)((z->map.kA + OZ_CH - 1) / OZ_CH);
  z->map.nB = (int)((z->map.K - z->map.kA + OZ_CH - 1) / OZ_CH);
  z->nch = z->map.nA + z->map.nB;
  // about one S CTA per SM: R ranges x 2 column halves (one half up to 64 states)
  const int halves = n > OZ_N ? 2 : 1;
  int R = nsm / halves;
  if (R > z->nch) R = z->nch;
  if (R < 1) R = 1;
  int RA = z->map.nA > 0 ? (int)(((long)R * z->map.nA + z->nch - 1) / z->nch) : 0;
  if (z->map.nA > 0 && RA < 1) RA = 1;
  if (RA > z->map.nA) RA = z->map.nA;
  int RB = R - RA;
  if (z->map.nB > 0 && RB < 1) RB = 1;
  if (RB > z->map.nB) RB = z->map.nB;
  R = RA + RB;
  z->R = R;
  z->RA = RA;
  std::vector<int> rc(R + 1), cr(z->nch);
  for (int a = 0; a <= RA; ++a) rc[a] = (int)((long)z->map.nA * a / (RA > 0 ? RA : 1));
  if (RA == 0) rc[0] = 0;
  for (int b = 0; b <= RB; ++b) rc[RA + b] = z->map.nA + (int)((long)z->map.nB * b / (RB > 0 ? RB : 1));
  for (int q = 0; q < R; ++q)
    for (int c = rc[q]; c < rc[q + 1]; ++c) cr[c] = q;
  int maxlen = 0;
  for (int q = 0; q < R; ++q) maxlen = std::max(maxlen, rc[q + 1] - rc[q]);
  z->maxlen = maxlen;
  bool okm = true;
  okm &= cudaMalloc(&z->rc, (R + 1) * sizeof(int)) == cudaSuccess;
  okm &= cudaMalloc(&z->cr, z->nch * sizeof(int)) == cudaSuccess;
  okm &= cudaMalloc(&z->sl, (size_t)OZ_ND * z->nch * OZ_TILE) == cudaSuccess;
  okm &= cudaMalloc(&z->tsl, (size_t)R * OZ_NDT * OZ_TILE) == cudaSuccess;
  okm &= cudaMalloc(&z->ex, (size_t)R * 128 * sizeof(int)) == cudaSuccess;
  okm &= cudaMalloc(&z->fx, (size_t)R * 128 * sizeof(int)) == cudaSuccess;
  okm &= cudaMalloc(&z->part, (size_t)R * 128 * 128 * sizeof(double)) == cudaSuccess;
  if (!okm) { oa_oz_free(z); cudaGetLastError(); return nullptr; }
  // rows n..127 of the slices stay zero
  okm &= cudaMemset(z->sl, 0, (size_t)OZ_ND * z->nch * OZ_TILE) == cudaSuccess;
  okm &= cudaMemset(z->ex, 0, (size_t)R * 128 * sizeof(int)) == cudaSuccess;
  okm &= cudaMemcpy(z->rc, rc.data(), (R + 1) * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
  okm &= cudaMemcpy(z->cr, cr.data(), z->nch * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
  okm &= oz_map(&z->tS, z->sl, 128, z->nch, OZ_ND, 128);
  okm &= oz_map(&z->tT, z->tsl, 128, OZ_NDT, R, OZ_N);
  z->stages = 0;
  for (int st = 3; st >= 2; --st)
    if (oz_syrk_smem(st) <= (size_t)OA_MAX_SMEM) { z->stages = st; break; }
  okm &= z->stages >= 2 && oz_rot_smem() <= (size_t)OA_MAX_SMEM;
  okm &= (size_t)maxlen * OZ_CH * sizeof(double) <= (size_t)OA_MAX_SMEM;
  if (!okm) { oa_oz_free(z); cudaGetLastError(); return nullptr; }
  return z;
}

size_t oa_oz_bytes(const oa_oz* z) {
  return z ? (size_t)OZ_ND * z->nch * OZ_TILE + (size_t)z->R * OZ_NDT * OZ_TILE + (size_t)z->R * 128 * 128 * 8 : 0;
}

// S = alpha (w_kx0 sum over the kx = 0 columns + sum over the rest) X X^T for
// X [n][2 ng] (row stride ldx), and keep the slices of X for oa_oz_rotate
cudaError_t oa_oz_overlap(oa_oz* z, cudaStream_t s, const double* X, long ldx, double alpha, double w_kx0,
                          double* S, int* err_flag, const int* cond) {
  if (!z) return cudaErrorNotSupported;
  const size_t smem = (size_t)z->maxlen * OZ_CH * sizeof(double);
  cudaError_t e = oa_smem_limit(k_oz_slice);
  if (e != cudaSuccess) return e;
  k_oz_slice<<<dim3(z->R, z->n), 256, smem, s>>>(X, ldx, z->map, z->rc, z->nch, z->sl, z->ex);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  z->src = X;
  e = oa_smem_limit(k_oz_syrk);
  if (e != cudaSuccess) return e;
  k_oz_syrk<<<dim3(z->R, z->n > OZ_N ? 2 : 1), OZ_THREADS, oz_syrk_smem(z->stages), s>>>(
      z->tS, z->rc, z->RA, z->ex, z->n, alpha, w_kx0, z->stages, z->part, err_flag, cond);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int nn = z->n * z->n;
  k_oz_reduce<<<(nn + 255) / 256, 256, 0, s>>>(z->part, z->R, z->n, S, cond);
  return cudaGetLastError();
}

// out[j][c] = sum_i T[i][j] X[i][c] for the X of the last oa_oz_overlap
// (out row stride ldo); po: optional bf16 planes of out
cudaError_t oa_oz_rotate(oa_oz* z, cudaStream_t s, const double* T, const double* X, double* out, long ldo,
                         const OaPlaneOut* po, int* err_flag, const int* cond) {
  if (!z || X != z->src) return cudaErrorNotSupported;
  cudaError_t e = oa_smem_limit(k_oz_tslice);
  if (e != cudaSuccess) return e;
  k_oz_tslice<<<z->R, 128, OZ_NDT * 128 * OZ_TLD, s>>>(T, z->n, z->ex, z->tsl, z->fx);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = oa_smem_limit(k_oz_rot);
  if (e != cudaSuccess) return e;
  k_oz_rot<<<dim3(z->nch, z->n > OZ_N ? 2 : 1), OZ_THREADS, oz_rot_smem(), s>>>(
      z->tS, z->tT, z->cr, z->fx, z->map, z->n, ldo, out, po ? *po : OaPlaneOut{nullptr, 0, 0, 0}, err_flag, cond);
  return cudaGetLastError();
}
