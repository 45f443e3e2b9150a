// Split-BF16 PairCalculator GEMMs fed from bf16 planes, mixed-precision form.
//
// An FP64 matrix X [rows][K] is first written as NT bf16 planes
//   P_q [rows][ldp],  x = P_0 + P_1 (+ P_2),  P_0 = bf16(x), P_1 = bf16(x - P_0), ...
// (k_split_planes; ldp = K rounded up to 64, padding zero).  The GEMMs then
// move 16-byte pieces of the planes straight into the UMMA canonical
// shared-memory layouts with cp.async (no conversion in the main loop) and
// accumulate the cross products P_i Q_j, i + j <= NT - 1, with
// tcgen05.mma kind::f16 into FP32 TMEM accumulators:
//
//   k_pfwd : C[x][y] = alpha sum_k w(k) A[x][k] B[y][k]   (Lambda, the nonlocal Z)
//            PairCalculator::multiplyForward (ckPairCalculator.C:821-893);
//            operands K-major; split-K over CTAs (FP32 partials, FP64 reduce);
//            the kx0 weight is applied to A when its planes are written.
//   k_pbwd : out[j][c] = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c]
//            bwMultiplyHelper / bwMultiplyDynOrthoT (ckPairCalculator.C:1710-2031);
//            operands MN-major (the planes' natural [k][c] and [k][j] order),
//            one TMEM accumulator per term, scaled in the epilogue.
//
// Every mbarrier wait is bounded; on timeout the CTA sets the device error
// flag (read by oa_gpu_check), frees its TMEM and returns.
#include <cuda_bf16.h>
#include "oa_internal.h"

#define P2_KS 32          // K per pipeline stage
#define P2_M 128          // MMA M
#define P2_THREADS 256
#define P2_SPIN_LIMIT (1u << 28)

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ uint32_t p2_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t p2_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // sm_100 descriptor version; base offset 0, SWIZZLE_NONE
  return d;
}

// kind::f16, A/B bf16, D f32, M = 128; a_mn / b_mn select MN-major operands
__host__ __device__ constexpr uint32_t p2_idesc(int n, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(P2_M >> 4) << 24);
}

__device__ __forceinline__ void p2_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void p2_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(p2_smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void p2_mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(p2_smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool p2_mbar_wait(uint64_t* bar, uint32_t phase) {
  const uint32_t a = p2_smem_u32(bar);
  for (uint32_t it = 0; it < P2_SPIN_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(a), "r"(phase) : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void p2_fence_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void p2_tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void p2_tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void p2_tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(p2_smem_u32(slot)), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void p2_tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void p2_tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void p2_cp16(uint32_t sdst, const void* gsrc, bool valid) {
  const int n = valid ? 16 : 0;  // src-size 0: zero fill
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(sdst), "l"(gsrc), "r"(n));
}
__device__ __forceinline__ void p2_cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void p2_cp_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N)); }

// ---------------------------------------------------------------------------
// FP64 -> NT bf16 planes, the columns k < kx0_cols scaled by w_kx0 first (the
// PairCalculator's kx = 0 weight).  Chunks of 8 elements; chunks at or past K
// are written as zeros (the plane padding).
// ---------------------------------------------------------------------------
template <int NT>
__global__ void k_split_planes(const double* __restrict__ X, int rows, long K, long ldx, long kx0_cols, double w_kx0,
                               bf16* __restrict__ P, long ldp) {
  const long cpr = ldp / 8;
  const size_t total = (size_t)rows * cpr;
  const size_t pstride = (size_t)rows * ldp;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(t / cpr);
    const long k0 = (long)(t - (size_t)r * cpr) * 8;
    double x[8];
    const double* src = X + (size_t)r * ldx + k0;
    if (k0 + 8 <= K && ((((uintptr_t)src) & 15) == 0)) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double2 v = __ldcs(reinterpret_cast<const double2*>(src) + e);
        x[2 * e] = v.x; x[2 * e + 1] = v.y;
      }
    } else {
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = (k0 + e < K) ? src[e] : 0.0;
    }
    if (k0 < kx0_cols) {
#pragma unroll
      for (int e = 0; e < 8; ++e) if (k0 + e < kx0_cols) x[e] *= w_kx0;
    }
    bf16 h[NT][8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      double v = x[e];
#pragma unroll
      for (int q = 0; q < NT; ++q) {
        const bf16 b = __float2bfloat16_rn((float)v);
        h[q][e] = b;
        v -= (double)__bfloat162float(b);
      }
    }
#pragma unroll
    for (int q = 0; q < NT; ++q)
      *reinterpret_cast<uint4*>(P + q * pstride + (size_t)r * ldp + k0) = *reinterpret_cast<uint4*>(&h[q][0]);
  }
}

// ---------------------------------------------------------------------------
// forward: part[kb][x][y] (FP32) = sum over this CTA's K slabs of A[x][k] B[y][k]
// K-major canonical layout, per plane tile of R rows x P2_KS:
//   chunk (row r, kc) at kc * (R/8) * 128 + (r/8) * 128 + (r%8) * 16
// ---------------------------------------------------------------------------
template <int NT, int NB>
__global__ void __launch_bounds__(P2_THREADS, 1)
k_pfwd(const bf16* __restrict__ PA, const bf16* __restrict__ PB, int m, int n, long K, long ldp, int nkb,
       int stages, float* __restrict__ part, int* __restrict__ err_flag) {
  extern __shared__ __align__(1024) unsigned char p2_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)p2_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t a_bytes = P2_M * P2_KS * 2, b_bytes = (uint32_t)NB * P2_KS * 2;
  constexpr uint32_t stage_bytes = NT * (a_bytes + b_bytes);
  uint64_t* bars = (uint64_t*)(base + (size_t)stages * stage_bytes);
  uint32_t* tslot = (uint32_t*)(bars + stages);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.y * P2_M, nt0 = blockIdx.z * NB;
  // K slabs kb, kb + nkb, ... : at any moment the CTAs stream neighbouring
  // pieces of the same rows (DRAM pages opened once)
  const int kb = blockIdx.x;
  const long rslabs = (K + P2_KS - 1) / P2_KS;
  const int nslab = rslabs > kb ? (int)((rslabs - kb + nkb - 1) / nkb) : 0;
  constexpr uint32_t ncols = NB <= 32 ? 32 : (NB <= 64 ? 64 : (NB <= 128 ? 128 : 256));
  if (tid == 0)
    for (int s = 0; s < stages; ++s) p2_mbar_init(&bars[s], 1);
  if (warp == 0) p2_tmem_alloc(tslot, ncols);
  p2_fence_async();
  __syncthreads();
  p2_tc_after();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = p2_idesc(NB, 0, 0);
  const uint32_t sbase = p2_smem_u32(base);
  // this thread's 16-byte pieces of a slab (the same for every slab but k0):
  // planes [q][row][k], K-major canonical tile offsets
  constexpr int NA = NT * P2_M * (P2_KS / 8), NTOT = NA + NT * NB * (P2_KS / 8);
  constexpr int J = (NTOT + P2_THREADS - 1) / P2_THREADS;
  const bf16* gsrc[J];
  uint32_t sofs[J];
  uint32_t vmask = 0;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int i = tid + j * P2_THREADS;
    const bool isA = i < NA;
    const int i2 = isA ? i : i - NA;
    const int rows = isA ? P2_M : NB;
    const int q = i2 / (rows * (P2_KS / 8));
    const int rem = i2 - q * rows * (P2_KS / 8);
    const int r = rem % rows, kc = rem / rows;
    const int grow = (isA ? m0 : nt0) + r;
    const bool valid = (i < NTOT) && grow < (isA ? m : n);
    gsrc[j] = valid ? (isA ? PA + (size_t)q * m * ldp : PB + (size_t)q * n * ldp) + (size_t)grow * ldp + kc * 8 : PA;
    sofs[j] = (isA ? q * a_bytes : NT * a_bytes + q * b_bytes) + (uint32_t)kc * (uint32_t)(rows / 8) * 128u +
              (uint32_t)(r >> 3) * 128u + (uint32_t)(r & 7) * 16u;
    if (valid) vmask |= 1u << j;
    if (i >= NTOT) sofs[j] = 0xFFFFFFFFu;
  }
  // the planes are zero-padded to ldp (a multiple of 64): slabs never need a K check
  auto load_slab = [&](int sl, int st) {
    const long k0 = ((long)kb + (long)sl * nkb) * P2_KS;
    const uint32_t sb = sbase + st * stage_bytes;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      if (sofs[j] == 0xFFFFFFFFu) continue;
      const bool v = (vmask >> j) & 1u;
      p2_cp16(sb + sofs[j], v ? (const void*)(gsrc[j] + k0) : (const void*)PA, v);
    }
  };
  for (int s = 0; s < stages - 1; ++s) {
    if (s < nslab) load_slab(s, s);
    p2_cp_commit();
  }
  bool ok = true;
  uint32_t phase_bits = 0;  // bit s: parity of the next completion of bars[s]
  for (int sl = 0; sl < nslab; ++sl) {
    const int st = sl % stages;
    // slabs <= sl have landed: at most stages - 2 newer groups pending
    if (stages == 4) p2_cp_wait<2>(); else p2_cp_wait<1>();
    p2_fence_async();
    __syncthreads();
    if (tid == 0) {
      p2_tc_after();
      const uint32_t sb = sbase + st * stage_bytes;
      constexpr uint32_t lbo_a = (P2_M / 8) * 128, lbo_b = (uint32_t)(NB / 8) * 128;
      bool acc = sl > 0;
#pragma unroll
      for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          if (i + j > NT - 1) continue;
#pragma unroll
          for (int ks = 0; ks < P2_KS / 16; ++ks) {
            const uint64_t da = p2_desc(sb + i * a_bytes + ks * 2 * lbo_a, lbo_a, 128);
            const uint64_t db = p2_desc(sb + NT * a_bytes + j * b_bytes + ks * 2 * lbo_b, lbo_b, 128);
            p2_mma(tmem, da, db, idesc, acc ? 1u : 0u);
            acc = true;
          }
        }
      p2_commit(&bars[st]);
    }
    // refill the stage read by slab sl - 1 once its MMAs are done
    const int sn = sl + stages - 1;
    if (sn < nslab) {
      const int stn = sn % stages;
      if (sl >= 1) {
        const bool w = p2_mbar_wait(&bars[stn], (phase_bits >> stn) & 1u);
        phase_bits ^= 1u << stn;
        if (!__syncthreads_and(w)) { ok = false; break; }
      }
      load_slab(sn, stn);
    }
    p2_cp_commit();
  }
  p2_cp_wait<0>();
  // commits 0 .. nslab - stages - 1 were waited for in the loop
  if (ok) {
    for (int d = (nslab > stages ? nslab - stages : 0); d < nslab; ++d) {
      const int st = d % stages;
      if (!p2_mbar_wait(&bars[st], (phase_bits >> st) & 1u)) { ok = false; break; }
      phase_bits ^= 1u << st;
    }
  }
  ok = __syncthreads_and(ok);
  p2_tc_after();
  // epilogue on all 8 warps: warp w reads TMEM lanes 32 (w % 4) .., columns of half w / 4
  float* out = part + ((size_t)kb * m + m0) * (size_t)n + nt0;
  const int row = (warp & 3) * 32 + (tid & 31);
  constexpr int HALF = NB >= 32 ? NB / 2 : NB;
  const int cbeg = (warp >> 2) * HALF;
  if (cbeg < NB) {
    if (ok && nslab > 0) {
      for (int c0 = cbeg; c0 < cbeg + HALF; c0 += 16) {
        float v[16];
        p2_tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0, v);
        if (m0 + row < m) {
#pragma unroll
          for (int e = 0; e < 16; ++e)
            if (nt0 + c0 + e < n) out[(size_t)row * n + c0 + e] = v[e];
        }
      }
    } else if (m0 + row < m) {
      for (int c = cbeg; c < cbeg + HALF && nt0 + c < n; ++c) out[(size_t)row * n + c] = 0.0f;
    }
  }
  if (!ok && tid == 0) atomicExch(err_flag, 1);
  p2_tc_before();
  __syncthreads();
  if (warp == 0) p2_tmem_dealloc(tmem, ncols);
}

// C = alpha sum_kb part[kb]; 64 outputs x 4 partial groups per block,
// combined in a fixed order
__global__ void __launch_bounds__(256)
k_pfwd_reduce(const float* __restrict__ part, int nkb, size_t nn, double alpha, double* __restrict__ C) {
  __shared__ double s1s[4][64];
  const int col = threadIdx.x & 63, g = threadIdx.x >> 6;
  const size_t i = (size_t)blockIdx.x * 64 + col;
  double s1 = 0.0;
  if (i < nn) {
    int k = g;
    for (; k + 12 < nkb; k += 16) {
      const float a = __ldcs(part + (size_t)k * nn + i);
      const float b = __ldcs(part + (size_t)(k + 4) * nn + i);
      const float c = __ldcs(part + (size_t)(k + 8) * nn + i);
      const float d = __ldcs(part + (size_t)(k + 12) * nn + i);
      s1 += (double)a; s1 += (double)b; s1 += (double)c; s1 += (double)d;
    }
    for (; k < nkb; k += 4) s1 += (double)__ldcs(part + (size_t)k * nn + i);
  }
  s1s[g][col] = s1;
  __syncthreads();
  if (g == 0 && i < nn) C[i] = alpha * (((s1s[0][col] + s1s[1][col]) + s1s[2][col]) + s1s[3][col]);
}

// ---------------------------------------------------------------------------
// backward: CTA = 128 columns c; D_t[c][j] = sum_k X_t[k][c] M_t[k][j] per term
// t in TMEM columns [t nbp, t nbp + nj).  MN-major canonical layout per plane
// tile of MN x P2_KS: chunk (k, group g of 8 MN) at (k/8) * (MN/8) * 128 + g * 128 + (k%8) * 16
// (SBO = 128 between MN groups, LBO = MN/8 * 128 between K groups).
// ---------------------------------------------------------------------------
template <int NT, int NB>
__global__ void __launch_bounds__(P2_THREADS, 1)
k_pbwd(const bf16* __restrict__ PM1, const bf16* __restrict__ PX1, double a1_kx0, double a1_rest,
       const bf16* __restrict__ PM2, const bf16* __restrict__ PX2, double a2, int nj, int nk, long ncol, long ldx,
       long kx0_cols, int stages, double* __restrict__ out, int* __restrict__ err_flag) {
  extern __shared__ __align__(1024) unsigned char p2_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)p2_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t a_bytes = P2_M * P2_KS * 2, b_bytes = (uint32_t)NB * P2_KS * 2;
  constexpr uint32_t stage_bytes = NT * (a_bytes + b_bytes);
  uint64_t* bars = (uint64_t*)(base + (size_t)stages * stage_bytes);
  uint32_t* tslot = (uint32_t*)(bars + stages);
  const int tid = threadIdx.x, warp = tid >> 5;
  const long c0 = (long)blockIdx.x * P2_M;
  const int nterm = PM2 ? 2 : 1;
  constexpr int NBP = NB <= 32 ? 32 : (NB <= 64 ? 64 : 128);  // TMEM columns per term
  const uint32_t ncols = nterm == 1 ? (uint32_t)NBP : (NBP == 128 ? 256u : (uint32_t)(2 * NBP));
  const int kch = (nk + P2_KS - 1) / P2_KS;
  const int nslab = nterm * kch;
  if (tid == 0)
    for (int s = 0; s < stages; ++s) p2_mbar_init(&bars[s], 1);
  if (warp == 0) p2_tmem_alloc(tslot, ncols);
  p2_fence_async();
  __syncthreads();
  p2_tc_after();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = p2_idesc(NB, 1, 1);
  const uint32_t sbase = p2_smem_u32(base);
  // this thread's pieces: (plane q, k row kk of the slab, MN group g); MN-major
  // canonical offsets (kk/8) (MN/8) 128 + g 128 + (kk%8) 16
  constexpr int GA = P2_M / 8, GB = NB / 8;
  constexpr int NA = NT * P2_KS * GA, NTOT = NA + NT * P2_KS * GB;
  constexpr int J = (NTOT + P2_THREADS - 1) / P2_THREADS;
  long goff[J];
  uint32_t sofs[J];
  int kkv[J];
  uint32_t amask = 0, cmask = 0;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int i = tid + j * P2_THREADS;
    const bool isA = i < NA;
    const int i2 = isA ? i : i - NA;
    const int grp = isA ? GA : GB;
    const int q = i2 / (P2_KS * grp);
    const int rem = i2 - q * P2_KS * grp;
    const int kk = rem / grp, g = rem - kk * grp;
    bool cval;
    if (isA) {
      const long c = c0 + g * 8;
      cval = c < ldx;
      goff[j] = (long)q * nk * ldx + (long)kk * ldx + c;
    } else {
      cval = g * 8 < nj;
      goff[j] = (long)q * nk * nj + (long)kk * nj + g * 8;
    }
    kkv[j] = kk;
    sofs[j] = (isA ? q * a_bytes : NT * a_bytes + q * b_bytes) + (uint32_t)(kk >> 3) * (uint32_t)grp * 128u +
              (uint32_t)g * 128u + (uint32_t)(kk & 7) * 16u;
    if (isA) amask |= 1u << j;
    if (cval && i < NTOT) cmask |= 1u << j;
    if (i >= NTOT) sofs[j] = 0xFFFFFFFFu;
  }
  auto load_slab = [&](int sl, int st) {
    const int term = sl / kch;
    const int k0 = (sl - term * kch) * P2_KS;
    const bf16* PX = term ? PX2 : PX1;
    const bf16* PM = term ? PM2 : PM1;
    const uint32_t sb = sbase + st * stage_bytes;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      if (sofs[j] == 0xFFFFFFFFu) continue;
      const bool isA = (amask >> j) & 1u;
      const bool v = ((cmask >> j) & 1u) && (k0 + kkv[j] < nk);
      const bf16* src = isA ? PX + goff[j] + (long)k0 * ldx : PM + goff[j] + (long)k0 * nj;
      p2_cp16(sb + sofs[j], v ? (const void*)src : (const void*)PX1, v);
    }
  };
  for (int s = 0; s < stages - 1; ++s) {
    if (s < nslab) load_slab(s, s);
    p2_cp_commit();
  }
  bool ok = true;
  uint32_t phase_bits = 0;
  for (int sl = 0; sl < nslab; ++sl) {
    const int st = sl % stages;
    if (stages == 4) p2_cp_wait<2>(); else p2_cp_wait<1>();
    p2_fence_async();
    __syncthreads();
    if (tid == 0) {
      p2_tc_after();
      const int term = sl / kch;
      const bool first_of_term = (sl - term * kch) == 0;
      const uint32_t sb = sbase + st * stage_bytes;
      constexpr uint32_t lbo_a = (uint32_t)(P2_M / 8) * 128, lbo_b = (uint32_t)(NB / 8) * 128;
      const uint32_t td = tmem + (uint32_t)(term * NBP);
      bool acc = !first_of_term;
#pragma unroll
      for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          if (i + j > NT - 1) continue;
#pragma unroll
          for (int ks = 0; ks < P2_KS / 16; ++ks) {
            const uint64_t da = p2_desc(sb + i * a_bytes + ks * 2 * lbo_a, lbo_a, 128);
            const uint64_t db = p2_desc(sb + NT * a_bytes + j * b_bytes + ks * 2 * lbo_b, lbo_b, 128);
            p2_mma(td, da, db, idesc, acc ? 1u : 0u);
            acc = true;
          }
        }
      p2_commit(&bars[st]);
    }
    const int sn = sl + stages - 1;
    if (sn < nslab) {
      const int stn = sn % stages;
      if (sl >= 1) {
        const bool w = p2_mbar_wait(&bars[stn], (phase_bits >> stn) & 1u);
        phase_bits ^= 1u << stn;
        if (!__syncthreads_and(w)) { ok = false; break; }
      }
      load_slab(sn, stn);
    }
    p2_cp_commit();
  }
  p2_cp_wait<0>();
  if (ok) {
    for (int d = (nslab > stages ? nslab - stages : 0); d < nslab; ++d) {
      const int st = d % stages;
      if (!p2_mbar_wait(&bars[st], (phase_bits >> st) & 1u)) { ok = false; break; }
      phase_bits ^= 1u << st;
    }
  }
  ok = __syncthreads_and(ok);
  p2_tc_after();
  // epilogue on all 8 warps: warp w reads TMEM lanes 32 (w % 4) .., columns of half w / 4
  const int row = (warp & 3) * 32 + (tid & 31);
  const long c = c0 + row;
  constexpr int HALF = NB >= 32 ? NB / 2 : NB;
  const int jbeg = (warp >> 2) * HALF;
  if (ok && jbeg < NB) {
    const double a1 = (c < kx0_cols) ? a1_kx0 : a1_rest;
    for (int q0 = jbeg; q0 < jbeg + HALF; q0 += 16) {
      float v1[16], v2[16];
      p2_tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)q0, v1);
      if (nterm == 2) p2_tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(NBP + q0), v2);
      if (c < ncol) {
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int j = q0 + e;
          if (j < nj) {
            double r = a1 * (double)v1[e];
            if (nterm == 2) r += a2 * (double)v2[e];
            out[(size_t)j * ncol + c] = r;
          }
        }
      }
    }
  }
  if (!ok && tid == 0) atomicExch(err_flag, 1);
  p2_tc_before();
  __syncthreads();
  if (warp == 0) p2_tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
long oa_plane_ld(long K) { return (K + 63) / 64 * 64; }

cudaError_t oa_split_planes(cudaStream_t s, int nt, const double* X, int rows, long K, long ldx, long kx0_cols,
                            double w_kx0, bf16* P, long ldp) {
  const size_t total = (size_t)rows * (ldp / 8);
  const unsigned nblk = (unsigned)((total + 255) / 256 < 8 * 148 ? (total + 255) / 256 : 8 * 148);
  if (nt == 2) k_split_planes<2><<<nblk, 256, 0, s>>>(X, rows, K, ldx, kx0_cols, w_kx0, P, ldp);
  else k_split_planes<3><<<nblk, 256, 0, s>>>(X, rows, K, ldx, kx0_cols, w_kx0, P, ldp);
  return cudaGetLastError();
}

// N tile of the MMAs: 32, 64 or 128 (one kernel instance each)
static int p2_nb(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : 0)); }

static size_t p2_smem(int nt, int nb, int stages) {
  return (size_t)stages * nt * (P2_M * P2_KS * 2 + (size_t)nb * P2_KS * 2) + 1024 + 256;
}

static int p2_stages(int nt, int nb) {
  for (int st = 4; st >= 3; --st)
    if (p2_smem(nt, nb, st) <= (size_t)OA_MAX_SMEM) return st;
  return 0;
}

// C[m][n] = alpha sum_k A[m][k] B[n][k] from planes PA [nt][m][ldp],
// PB [nt][n][ldp] (any kx0 weight already in the planes); part holds
// max_kb * m * n floats.  NotSupported when the shape does not fit (n > 256).
cudaError_t oa_pfwd(cudaStream_t s, int nt, const bf16* PA, const bf16* PB, int m, int n, long K, long ldp,
                    double alpha, float* part, int max_kb, double* C, int* err_flag, int nsm) {
  const int nb = p2_nb(n);
  if (nb == 0) return cudaErrorNotSupported;
  const int stages = p2_stages(nt, nb);
  if (stages < 3) return cudaErrorNotSupported;
  const int mt = (m + P2_M - 1) / P2_M, ntl = (n + nb - 1) / nb;
  const long sr = (K + P2_KS - 1) / P2_KS;
  int nkb = nsm / (mt * ntl);
  if (nkb > max_kb) nkb = max_kb;
  if (nkb > sr) nkb = (int)sr;
  if (nkb < 1) nkb = 1;
  const size_t sm = p2_smem(nt, nb, stages);
  dim3 grid(nkb, mt, ntl);
  cudaError_t e = cudaErrorNotSupported;
#define OA_PF(NTT, NBB)                                                                                     \
  if (nt == NTT && nb == NBB) {                                                                             \
    e = cudaFuncSetAttribute(k_pfwd<NTT, NBB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);        \
    if (e != cudaSuccess) return e;                                                                         \
    k_pfwd<NTT, NBB><<<grid, P2_THREADS, sm, s>>>(PA, PB, m, n, K, ldp, nkb, stages, part, err_flag);        \
    e = cudaGetLastError();                                                                                 \
  }
  OA_PF(2, 32) OA_PF(2, 64) OA_PF(2, 128) OA_PF(3, 32) OA_PF(3, 64) OA_PF(3, 128)
#undef OA_PF
  if (e != cudaSuccess) return e;
  const size_t mn = (size_t)m * n;
  k_pfwd_reduce<<<(unsigned)((mn + 63) / 64), 256, 0, s>>>(part, nkb, mn, alpha, C);
  return cudaGetLastError();
}

// out[j][c] = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c] from
// planes PX [nt][nk][ldx] and PM [nt][nk][nj].  NotSupported for nj > 128 or
// nj not a multiple of 8.
cudaError_t oa_pbwd(cudaStream_t s, int nt, const bf16* PM1, const bf16* PX1, double a1_kx0, double a1_rest,
                    const bf16* PM2, const bf16* PX2, double a2, int nj, int nk, long ncol, long ldx, long kx0_cols,
                    double* out, int* err_flag) {
  if (nj > 128 || (nj & 7) || ((PM2 == nullptr) != (PX2 == nullptr))) return cudaErrorNotSupported;
  const int nb = p2_nb(nj);
  if (nb == 0) return cudaErrorNotSupported;
  const int stages = p2_stages(nt, nb);
  if (stages < 3) return cudaErrorNotSupported;
  const size_t sm = p2_smem(nt, nb, stages);
  dim3 grid((unsigned)((ncol + P2_M - 1) / P2_M));
  cudaError_t e = cudaErrorNotSupported;
#define OA_PB(NTT, NBB)                                                                                       \
  if (nt == NTT && nb == NBB) {                                                                               \
    e = cudaFuncSetAttribute(k_pbwd<NTT, NBB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);          \
    if (e != cudaSuccess) return e;                                                                           \
    k_pbwd<NTT, NBB><<<grid, P2_THREADS, sm, s>>>(PM1, PX1, a1_kx0, a1_rest, PM2, PX2, a2, nj, nk, ncol, ldx,   \
                                                  kx0_cols, stages, out, err_flag);                           \
    e = cudaGetLastError();                                                                                   \
  }
  OA_PB(2, 32) OA_PB(2, 64) OA_PB(2, 128) OA_PB(3, 32) OA_PB(3, 64) OA_PB(3, 128)
#undef OA_PB
  return e;
}
