// Split-BF16 PairCalculator GEMMs with TMA-fed tcgen05 MMAs, mixed-precision form.
//
// Operand format ("bf16 planes"): an FP64 matrix X [rows][K] becomes NT bf16
// planes x = P_0 + P_1 (+ P_2), P_0 = bf16(x), P_1 = bf16(x - P_0), ...,
// stored K-chunk-major:  P[q][K/8][rows][8]  (K padded with zeros to ldp, a
// multiple of 64).  Element (r, k) sits at ((k/8) rows + r) 16 + (k%8) 2 bytes
// in plane q.  With this order one 3-D TMA box lands as the UMMA canonical
// no-swizzle layout for both uses of a matrix:
//   K-major view (forward GEMM, K = k):    box {8, R rows, 4 k-groups}
//       -> smem [kc][r][8]: SBO 128 (8-row groups), LBO = R 16 (k groups)
//   MN-major view (backward GEMM, MN = k): box {8, 32 rows, G k-groups}
//       -> smem [g][r][8]:  LBO 128 (8-row K groups), SBO = 32 16 = 512 (MN groups)
// (the TMA strides 16 B and rows 16 B grow with the dimension index).
//
//   k_tfwd : C[x][y] = alpha sum_k A[x][k] B[y][k]            (Lambda, the nonlocal Z)
//            PairCalculator::multiplyForward (ckPairCalculator.C:821-893)
//   k_tbwd : out[j][c] = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c]
//            bwMultiplyHelper / bwMultiplyDynOrthoT (ckPairCalculator.C:1710-2031)
//
// One thread issues the TMA loads (mbarrier complete_tx) and the MMAs
// (tcgen05.commit -> mbarrier) over a ring of stages; the block reads the
// FP32 TMEM accumulators in the epilogue.  Every wait is bounded: on timeout
// the block sets the device error flag, waits (bounded) for the copies it
// issued, frees its TMEM and returns.  No multicast.
#include <cuda.h>
#include <cuda_bf16.h>
#include <mutex>
#include "oa_internal.h"

typedef __nv_bfloat16 bf16;

#define TG_KS 32            // K (or k rows) per stage
#define TG_M 128
#define TG_THREADS 128
#define TG_SPIN (1u << 28)

__device__ __forceinline__ uint32_t tg_s32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t tg_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // sm_100 descriptor version; base offset 0, SWIZZLE_NONE
  return d;
}
__host__ __device__ constexpr uint32_t tg_idesc(int n, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TG_M >> 4) << 24);
}
__device__ __forceinline__ void tg_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void tg_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(tg_s32(bar)) : "memory");
}
__device__ __forceinline__ void tg_bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(tg_s32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void tg_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(tg_s32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool tg_wait(uint64_t* bar, uint32_t phase) {
  const uint32_t a = tg_s32(bar);
  for (uint32_t it = 0; it < TG_SPIN; ++it) {
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
// 4-D tile load of a tensor map box into shared memory, completing on bar
__device__ __forceinline__ void tg_tma4(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                        uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];"
      :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(tg_s32(bar))
      : "memory");
}
__device__ __forceinline__ void tg_tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tg_tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tg_tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(tg_s32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tg_tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tg_tmem_ld16(uint32_t taddr, float* v) {
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

// ---------------------------------------------------------------------------
// FP64 [rows][K] (row stride ldx) -> planes P[q][ldp/8][rows_pad][8], columns
// k < kx0_cols scaled by w_kx0 first; padding columns [K, ldp) and rows
// [rows, rows_pad) zero.
// ---------------------------------------------------------------------------
template <int NT>
__global__ void k_split_kc(const double* __restrict__ X, int rows, int rows_pad, long K, long ldx, long kx0_cols,
                           double w_kx0, bf16* __restrict__ P, long ldp, const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  const long ng = ldp / 8;
  const size_t total = (size_t)rows_pad * ng;
  const size_t pstride = (size_t)rows_pad * ldp;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    // t -> (group kg, row r) with r fastest: consecutive threads write
    // consecutive 16-byte pieces of the plane
    const long kg = (long)(t / rows_pad);
    const int r = (int)(t - (size_t)kg * rows_pad);
    const long k0 = kg * 8;
    double x[8];
    const double* src = X + (size_t)r * ldx + k0;
    if (r >= rows) {
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = 0.0;
    } else if (k0 + 8 <= K && ((((uintptr_t)src) & 15) == 0)) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(src) + e);
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
      *reinterpret_cast<uint4*>(P + q * pstride + ((size_t)kg * rows_pad + r) * 8) = *reinterpret_cast<uint4*>(&h[q][0]);
  }
}

// ---------------------------------------------------------------------------
// forward: part[kb][x][y] (FP32) over the K slabs kb, kb + nkb, ... of this CTA
// ---------------------------------------------------------------------------
template <int NT, int NB>
__global__ void __launch_bounds__(TG_THREADS, 1)
k_tfwd(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, int m, int n, long K, int nkb,
       int stages, float* __restrict__ part, int* __restrict__ err_flag, const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  extern __shared__ __align__(1024) unsigned char tg_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)tg_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t a_bytes = TG_M * TG_KS * 2, b_bytes = (uint32_t)NB * TG_KS * 2;
  constexpr uint32_t stage_bytes = NT * (a_bytes + b_bytes);
  uint64_t* full = (uint64_t*)(base + (size_t)stages * stage_bytes);
  uint64_t* empty = full + stages;
  uint32_t* tslot = (uint32_t*)(empty + stages);
  int* okflag = (int*)(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.y * TG_M, n0 = blockIdx.z * NB;
  const int kb = blockIdx.x;
  const long rslabs = (K + TG_KS - 1) / TG_KS;
  const int nslab = rslabs > kb ? (int)((rslabs - kb + nkb - 1) / nkb) : 0;
  constexpr uint32_t ncols = NB <= 32 ? 32 : (NB <= 64 ? 64 : (NB <= 128 ? 128 : 256));
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) { tg_bar_init(&full[s], 1); tg_bar_init(&empty[s], 1); }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *okflag = 1;
  }
  if (warp == 0) tg_tmem_alloc(tslot, ncols);
  __syncthreads();
  tg_tc_after();
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    constexpr uint32_t idesc = tg_idesc(NB, 0, 0);
    const uint32_t sbase = tg_s32(base);
    auto issue_loads = [&](int sl, int st) {
      const int g0 = (kb + sl * nkb) * (TG_KS / 8);
      const uint32_t sb = sbase + st * stage_bytes;
      tg_expect_tx(&full[st], stage_bytes);
#pragma unroll
      for (int q = 0; q < NT; ++q) {
        tg_tma4(sb + q * a_bytes, &tA, 0, m0, g0, q, &full[st]);
        tg_tma4(sb + NT * a_bytes + q * b_bytes, &tB, 0, n0, g0, q, &full[st]);
      }
    };
    bool ok = true;
    const int pre = nslab < stages ? nslab : stages;
    for (int s = 0; s < pre; ++s) issue_loads(s, s);
    int issued = pre;
    for (int sl = 0; sl < nslab && ok; ++sl) {
      const int st = sl % stages;
      const uint32_t ph = (uint32_t)(sl / stages) & 1u;
      if (!tg_wait(&full[st], ph)) { ok = false; break; }
      tg_tc_after();
      const uint32_t sb = sbase + st * stage_bytes;
      constexpr uint32_t lbo_a = TG_M * 16, lbo_b = (uint32_t)NB * 16;
      bool acc = sl > 0;
#pragma unroll
      for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          if (i + j > NT - 1) continue;
#pragma unroll
          for (int ks = 0; ks < TG_KS / 16; ++ks) {
            const uint64_t da = tg_desc(sb + i * a_bytes + ks * 2 * lbo_a, lbo_a, 128);
            const uint64_t db = tg_desc(sb + NT * a_bytes + j * b_bytes + ks * 2 * lbo_b, lbo_b, 128);
            tg_mma(tmem, da, db, idesc, acc ? 1u : 0u);
            acc = true;
          }
        }
      tg_commit(&empty[st]);
      if (issued < nslab) {
        // stage st is free once these MMAs are done
        if (!tg_wait(&empty[st], ph)) { ok = false; break; }
        issue_loads(issued, st);
        ++issued;
      }
    }
    // the last MMAs of every used stage: wait for the final commit of the last slab
    if (ok && nslab > 0) {
      const int sl = nslab - 1;
      if (!tg_wait(&empty[sl % stages], (uint32_t)(sl / stages) & 1u)) ok = false;
    }
    if (!ok) {
      // let the loads already issued land before the block exits
      for (int s2 = 0; s2 < stages; ++s2) (void)tg_wait(&full[s2], 0u);
      *okflag = 0;
    }
  }
  __syncthreads();
  tg_tc_after();
  const bool ok = *okflag != 0;
  float* out = part + ((size_t)kb * m + m0) * (size_t)n + n0;
  const int row = warp * 32 + (tid & 31);
  if (ok && nslab > 0) {
    for (int c0 = 0; c0 < NB; c0 += 16) {
      float v[16];
      tg_tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (m0 + row < m) {
#pragma unroll
        for (int e = 0; e < 16; ++e)
          if (n0 + c0 + e < n) out[(size_t)row * n + c0 + e] = v[e];
      }
    }
  } else if (m0 + row < m) {
    for (int c = 0; c < NB && n0 + c < n; ++c) out[(size_t)row * n + c] = 0.0f;
  }
  if (!ok && tid == 0) atomicExch(err_flag, 1);
  tg_tc_before();
  __syncthreads();
  if (warp == 0) tg_tmem_dealloc(tmem, ncols);
}

__global__ void __launch_bounds__(256)
k_tfwd_reduce(const float* __restrict__ part, int nkb, size_t nn, double alpha, double* __restrict__ C,
              const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  __shared__ double ss[4][64];
  const int col = threadIdx.x & 63, g = threadIdx.x >> 6;
  const size_t i = (size_t)blockIdx.x * 64 + col;
  double s = 0.0;
  if (i < nn) {
    int k = g;
    for (; k + 12 < nkb; k += 16) {
      const float a = __ldcs(part + (size_t)k * nn + i);
      const float b = __ldcs(part + (size_t)(k + 4) * nn + i);
      const float c = __ldcs(part + (size_t)(k + 8) * nn + i);
      const float d = __ldcs(part + (size_t)(k + 12) * nn + i);
      s += (double)a; s += (double)b; s += (double)c; s += (double)d;
    }
    for (; k < nkb; k += 4) s += (double)__ldcs(part + (size_t)k * nn + i);
  }
  ss[g][col] = s;
  __syncthreads();
  if (g == 0 && i < nn) C[i] = alpha * (((ss[0][col] + ss[1][col]) + ss[2][col]) + ss[3][col]);
}

// ---------------------------------------------------------------------------
// backward: CTA = 128 columns c, D_t[c][j] per term t in TMEM columns t NBP ..
// ---------------------------------------------------------------------------
template <int NT, int NB>
__global__ void __launch_bounds__(TG_THREADS, 1)
k_tbwd(const __grid_constant__ CUtensorMap tX1, const __grid_constant__ CUtensorMap tM1,
       const __grid_constant__ CUtensorMap tX2, const __grid_constant__ CUtensorMap tM2, int nterm, double a1_kx0,
       double a1_rest, double a2, int nj, int nk, long ncol, long kx0_cols, int stages, double* out,
       int* __restrict__ err_flag, const double* yadd, const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  extern __shared__ __align__(1024) unsigned char tg_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)tg_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t a_bytes = TG_M * TG_KS * 2, b_bytes = (uint32_t)NB * TG_KS * 2;
  constexpr uint32_t stage_bytes = NT * (a_bytes + b_bytes);
  uint64_t* full = (uint64_t*)(base + (size_t)stages * stage_bytes);
  uint64_t* empty = full + stages;
  uint32_t* tslot = (uint32_t*)(empty + stages);
  int* okflag = (int*)(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const long c0 = (long)blockIdx.x * TG_M;
  constexpr int NBP = NB <= 32 ? 32 : (NB <= 64 ? 64 : 128);
  const uint32_t ncols = nterm == 1 ? (uint32_t)NBP : (NBP == 128 ? 256u : (uint32_t)(2 * NBP));
  const int kch = (nk + TG_KS - 1) / TG_KS;
  const int nslab = nterm * kch;
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) { tg_bar_init(&full[s], 1); tg_bar_init(&empty[s], 1); }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *okflag = 1;
  }
  if (warp == 0) tg_tmem_alloc(tslot, ncols);
  __syncthreads();
  tg_tc_after();
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    constexpr uint32_t idesc = tg_idesc(NB, 1, 1);
    const uint32_t sbase = tg_s32(base);
    const int cg0 = (int)(c0 / 8);
    auto issue_loads = [&](int sl, int st) {
      const int term = sl / kch;
      const int k0 = (sl - term * kch) * TG_KS;
      const CUtensorMap* tx = term ? &tX2 : &tX1;
      const CUtensorMap* tm = term ? &tM2 : &tM1;
      const uint32_t sb = sbase + st * stage_bytes;
      tg_expect_tx(&full[st], stage_bytes);
#pragma unroll
      for (int q = 0; q < NT; ++q) {
        tg_tma4(sb + q * a_bytes, tx, 0, k0, cg0, q, &full[st]);
        tg_tma4(sb + NT * a_bytes + q * b_bytes, tm, 0, k0, 0, q, &full[st]);
      }
    };
    bool ok = true;
    const int pre = nslab < stages ? nslab : stages;
    for (int s = 0; s < pre; ++s) issue_loads(s, s);
    int issued = pre;
    for (int sl = 0; sl < nslab && ok; ++sl) {
      const int st = sl % stages;
      const uint32_t ph = (uint32_t)(sl / stages) & 1u;
      if (!tg_wait(&full[st], ph)) { ok = false; break; }
      tg_tc_after();
      const int term = sl / kch;
      const bool first_of_term = (sl - term * kch) == 0;
      const uint32_t sb = sbase + st * stage_bytes;
      // MN-major: K groups of 8 rows 128 B apart (LBO), MN groups 512 B apart (SBO)
      const uint32_t td = tmem + (uint32_t)(term * NBP);
      bool acc = !first_of_term;
#pragma unroll
      for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          if (i + j > NT - 1) continue;
#pragma unroll
          for (int ks = 0; ks < TG_KS / 16; ++ks) {
            const uint64_t da = tg_desc(sb + i * a_bytes + ks * 256, 128, TG_KS * 16);
            const uint64_t db = tg_desc(sb + NT * a_bytes + j * b_bytes + ks * 256, 128, TG_KS * 16);
            tg_mma(td, da, db, idesc, acc ? 1u : 0u);
            acc = true;
          }
        }
      tg_commit(&empty[st]);
      if (issued < nslab) {
        if (!tg_wait(&empty[st], ph)) { ok = false; break; }
        issue_loads(issued, st);
        ++issued;
      }
    }
    if (ok && nslab > 0) {
      const int sl = nslab - 1;
      if (!tg_wait(&empty[sl % stages], (uint32_t)(sl / stages) & 1u)) ok = false;
    }
    if (!ok) {
      for (int s2 = 0; s2 < stages; ++s2) (void)tg_wait(&full[s2], 0u);
      *okflag = 0;
    }
  }
  __syncthreads();
  tg_tc_after();
  const bool ok = *okflag != 0;
  const int row = warp * 32 + (tid & 31);
  const long c = c0 + row;
  if (ok) {
    const double a1 = (c < kx0_cols) ? a1_kx0 : a1_rest;
    for (int q0 = 0; q0 < NB; q0 += 16) {
      float v1[16], v2[16];
      tg_tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)q0, v1);
      if (nterm == 2) tg_tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(NBP + q0), v2);
      if (c < ncol) {
        // yadd may be out itself: all 16 reads go before the writes
        double ya[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) ya[e] = (yadd && q0 + e < nj) ? yadd[(size_t)(q0 + e) * ncol + c] : 0.0;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int j = q0 + e;
          if (j < nj) {
            double r = a1 * (double)v1[e];
            if (nterm == 2) r += a2 * (double)v2[e];
            out[(size_t)j * ncol + c] = r + ya[e];
          }
        }
      }
    }
  }
  if (!ok && tid == 0) atomicExch(err_flag, 1);
  tg_tc_before();
  __syncthreads();
  if (warp == 0) tg_tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn tg_encoder() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
    cudaGetLastError();
  });
  return fn;
}

// planes P[nt][ldp/8][rows][8] as a 4-D bf16 tensor {8, rows, ldp/8, nt}; box {8, br, bg, 1}
static bool tg_map(CUtensorMap* map, const bf16* P, int nt, int rows, long ldp, int br, int bg) {
  EncodeTiledFn enc = tg_encoder();
  if (!enc || (((uintptr_t)P) & 15)) return false;
  const cuuint64_t dims[4] = {8, (cuuint64_t)rows, (cuuint64_t)(ldp / 8), (cuuint64_t)nt};
  const cuuint64_t strides[3] = {16, (cuuint64_t)rows * 16, (cuuint64_t)rows * (cuuint64_t)ldp * 2};
  const cuuint32_t box[4] = {8, (cuuint32_t)br, (cuuint32_t)bg, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)P, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

int oa_tgemm_available() { return tg_encoder() != nullptr; }

cudaError_t oa_split_kc(cudaStream_t s, int nt, const double* X, int rows, int rows_pad, long K, long ldx,
                        long kx0_cols, double w_kx0, bf16* P, long ldp, const int* cond) {
  if (rows_pad < rows || (ldp & 7)) return cudaErrorInvalidValue;
  const size_t total = (size_t)rows_pad * (ldp / 8);
  const unsigned nblk = (unsigned)((total + 255) / 256 < 8 * 148 ? (total + 255) / 256 : 8 * 148);
  if (nt == 2) k_split_kc<2><<<nblk, 256, 0, s>>>(X, rows, rows_pad, K, ldx, kx0_cols, w_kx0, P, ldp, cond);
  else k_split_kc<3><<<nblk, 256, 0, s>>>(X, rows, rows_pad, K, ldx, kx0_cols, w_kx0, P, ldp, cond);
  return cudaGetLastError();
}

// rows of the planes of an operand the kernels read in boxes of `box` rows
int oa_tg_rows_pad(int rows, int box) { return (rows + box - 1) / box * box; }
int oa_tg_nb(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : 0)); }

static int tg_nb(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : 0)); }
static size_t tg_smem(int nt, int nb, int stages) {
  return (size_t)stages * nt * ((size_t)TG_M * TG_KS * 2 + (size_t)nb * TG_KS * 2) + 1024 + 256;
}
static int tg_stages(int nt, int nb) {
  for (int st = 6; st >= 2; --st)
    if (tg_smem(nt, nb, st) <= (size_t)OA_MAX_SMEM) return st;
  return 0;
}

// C[m][n] = alpha sum_k A[m][k] B[n][k]; PA planes with rows_a rows (a
// multiple of 128), PB with rows_b rows (a multiple of the N tile), both of
// leading size ldp.  NotSupported when the shape or the TMA encoder rules it out.
cudaError_t oa_tfwd(cudaStream_t s, int nt, const bf16* PA, int rows_a, const bf16* PB, int rows_b, int m, int n,
                    long K, long ldp, double alpha, float* part, int max_kb, double* C, int* err_flag, int nsm,
                    const int* cond) {
  const int nb = tg_nb(n);
  if (nb == 0 || m > rows_a || n > rows_b) return cudaErrorNotSupported;
  const int stages = tg_stages(nt, nb);
  if (stages < 2) return cudaErrorNotSupported;
  const int mt = (m + TG_M - 1) / TG_M, ntl = (n + nb - 1) / nb;
  // the planes are padded to whole boxes of rows (oa_tg_rows_pad)
  if (rows_a % TG_M || rows_b % nb || rows_a < m || rows_b < n) return cudaErrorNotSupported;
  CUtensorMap ta, tb;
  if (!tg_map(&ta, PA, nt, rows_a, ldp, TG_M, TG_KS / 8) || !tg_map(&tb, PB, nt, rows_b, ldp, nb, TG_KS / 8))
    return cudaErrorNotSupported;
  const long sr = (K + TG_KS - 1) / TG_KS;
  int nkb = nsm / (mt * ntl);
  if (nkb > max_kb) nkb = max_kb;
  if (nkb > sr) nkb = (int)sr;
  if (nkb < 1) nkb = 1;
  const size_t sm = tg_smem(nt, nb, stages);
  dim3 grid(nkb, mt, ntl);
  cudaError_t e = cudaErrorNotSupported;
#define OA_TF(NTT, NBB)                                                                                     \
  if (nt == NTT && nb == NBB) {                                                                             \
    e = cudaFuncSetAttribute(k_tfwd<NTT, NBB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);        \
    if (e != cudaSuccess) return e;                                                                         \
    k_tfwd<NTT, NBB><<<grid, TG_THREADS, sm, s>>>(ta, tb, m, n, K, nkb, stages, part, err_flag, cond);       \
    e = cudaGetLastError();                                                                                 \
  }
  OA_TF(2, 32) OA_TF(2, 64) OA_TF(2, 128) OA_TF(3, 32) OA_TF(3, 64) OA_TF(3, 128)
#undef OA_TF
  if (e != cudaSuccess) return e;
  const size_t mn = (size_t)m * n;
  k_tfwd_reduce<<<(unsigned)((mn + 63) / 64), 256, 0, s>>>(part, nkb, mn, alpha, C, cond);
  return cudaGetLastError();
}

// out[j][c] = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c]
// (+ yadd[j][c], which may be out itself) from X planes (rows nk, leading
// size ldx) and M planes (rows nk, leading size nj); nk a multiple of 32
// (planes padded with zero rows).  cond: optional device flag, nothing runs
// when it is 0.
cudaError_t oa_tbwd(cudaStream_t s, int nt, const bf16* PM1, const bf16* PX1, double a1_kx0, double a1_rest,
                    const bf16* PM2, const bf16* PX2, double a2, int nj, int nk, long ncol, long ldx, long kx0_cols,
                    double* out, int* err_flag, const double* yadd, const int* cond) {
  const int nb = tg_nb(nj);
  if (nb == 0 || nb != nj || ((PM2 == nullptr) != (PX2 == nullptr)) || nk < TG_KS || (nk % TG_KS)) return cudaErrorNotSupported;
  const int stages = tg_stages(nt, nb);
  if (stages < 2) return cudaErrorNotSupported;
  CUtensorMap tx1, tm1, tx2, tm2;
  if (!tg_map(&tx1, PX1, nt, nk, ldx, TG_KS, TG_M / 8) || !tg_map(&tm1, PM1, nt, nk, nj, TG_KS, nb / 8))
    return cudaErrorNotSupported;
  const int nterm = PM2 ? 2 : 1;
  if (nterm == 2) {
    if (!tg_map(&tx2, PX2, nt, nk, ldx, TG_KS, TG_M / 8) || !tg_map(&tm2, PM2, nt, nk, nj, TG_KS, nb / 8))
      return cudaErrorNotSupported;
  } else {
    tx2 = tx1; tm2 = tm1;
  }
  const size_t sm = tg_smem(nt, nb, stages);
  dim3 grid((unsigned)((ncol + TG_M - 1) / TG_M));
  cudaError_t e = cudaErrorNotSupported;
#define OA_TB(NTT, NBB)                                                                                        \
  if (nt == NTT && nb == NBB) {                                                                                \
    e = cudaFuncSetAttribute(k_tbwd<NTT, NBB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);           \
    if (e != cudaSuccess) return e;                                                                            \
    k_tbwd<NTT, NBB><<<grid, TG_THREADS, sm, s>>>(tx1, tm1, tx2, tm2, nterm, a1_kx0, a1_rest, a2, nj, nk, ncol,  \
                                                  kx0_cols, stages, out, err_flag, yadd, cond);                \
    e = cudaGetLastError();                                                                                    \
  }
  OA_TB(2, 32) OA_TB(2, 64) OA_TB(2, 128) OA_TB(3, 32) OA_TB(3, 64) OA_TB(3, 128)
#undef OA_TB
  return e;
}
