// Split-BF16 PairCalculator GEMMs on the 5th-generation tensor cores
// (tcgen05.mma kind::f16, FP32 accumulator in TMEM), mixed-precision form.
//
// Each FP64 operand element x is split into NT bf16 terms
//   x = t0 + t1 (+ t2),  t0 = bf16(x), t1 = bf16(x - t0), t2 = bf16(x - t0 - t1)
// and the product keeps the cross terms ti*tj with i + j <= NT - 1
// (NT = 2: 3 products, ~2^-16 relative; NT = 3: 6 products, ~2^-24).
// The split happens while staging the FP64 tiles into shared memory, so the
// GEMM reads each FP64 operand from HBM exactly once; these GEMMs are
// HBM-bound on that read, not tensor-bound.
//
//   k_umma_fwd : C[x][y] = alpha sum_k w(k) A[x][k] B[y][k]   (S, Lambda; split-K,
//                FP32 partial per CTA, FP64 reduction in k_umma_fwd_reduce)
//                ckPairCalculator.C:821-893 (multiplyForward)
//   k_umma_bwd : out_j(c) = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c]
//                ckPairCalculator.C:1710-2031 (bwMultiplyHelper, bwMultiplyDynOrthoT)
//
// Shared-memory operand layout: the UMMA canonical K-major, no-swizzle form.
// Core matrix = 8 rows x 16 bytes (8 bf16 along K), rows 16 B apart; row
// groups SBO = 128 B apart; K core-matrix columns LBO = rows/8 * 128 B apart.
#include <cuda_bf16.h>
#include "oa_internal.h"
#include "oa_wait.cuh"

#define UM_KT 64          // K elements per pipeline stage
#define UM_M 128          // MMA M (rows per CTA tile)
#define UM_THREADS 512
#define UM_ITEMS_MAX 4   // staged 8-element chunks per thread per stage (nb <= 128)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, SWIZZLE_NONE
}

// kind::f16, A/B bf16, D f32, both K-major, M = 128
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(UM_M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

// bounded wait on an mbarrier phase (oa_wait.cuh); false when the time limit is hit
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  return oa_mbar_wait_bounded(smem_u32(bar), phase);
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(smem_u32(slot)), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
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

// split 8 doubles into NT bf16 vectors of 8 (16 bytes each)
template <int NT>
__device__ __forceinline__ void split8(const double* x, uint4* out) {
  __nv_bfloat16 t[NT][8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    double r = x[e];
#pragma unroll
    for (int q = 0; q < NT; ++q) {
      const __nv_bfloat16 h = __float2bfloat16_rn((float)r);
      t[q][e] = h;
      r -= (double)__bfloat162float(h);
    }
  }
#pragma unroll
  for (int q = 0; q < NT; ++q) out[q] = *reinterpret_cast<uint4*>(&t[q][0]);
}

// byte offset of the 16-byte chunk (row r, K core column kc) in a tile of R rows
__device__ __forceinline__ uint32_t canon_off(int r, int kc, int rows) {
  return (uint32_t)kc * (uint32_t)(rows / 8) * 128u + (uint32_t)(r >> 3) * 128u + (uint32_t)(r & 7) * 16u;
}

struct UmmaSmem {
  // per stage: NT A tiles [UM_M x UM_KT], NT B tiles [NB x UM_KT] (bf16)
  uint32_t a_bytes, b_bytes, stage_bytes, total;
};

__host__ __device__ inline UmmaSmem umma_smem(int nt, int nb) {
  UmmaSmem L;
  L.a_bytes = UM_M * UM_KT * 2;
  L.b_bytes = (uint32_t)nb * UM_KT * 2;
  L.stage_bytes = (uint32_t)nt * (L.a_bytes + L.b_bytes);
  L.total = 2 * L.stage_bytes + 1024;  // + barriers / TMEM slot, 1 KB aligned base
  return L;
}

// issue the split products of one stage: sum_{i+j<=NT-1} A_i B_j^T
template <int NT>
__device__ __forceinline__ void issue_stage(uint32_t tmem_d, uint32_t sbase, const UmmaSmem& L, int nb, uint32_t idesc,
                                            bool first) {
  const uint32_t lbo_a = (UM_M / 8) * 128, lbo_b = (uint32_t)(nb / 8) * 128;
  bool acc = !first;
#pragma unroll
  for (int i = 0; i < NT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      if (i + j > NT - 1) continue;
      const uint32_t a0 = sbase + i * L.a_bytes;
      const uint32_t b0 = sbase + NT * L.a_bytes + j * L.b_bytes;
#pragma unroll
      for (int ks = 0; ks < UM_KT / 16; ++ks) {
        const uint64_t da = umma_desc(a0 + ks * 2 * lbo_a, lbo_a, 128);
        const uint64_t db = umma_desc(b0 + ks * 2 * lbo_b, lbo_b, 128);
        umma_bf16(tmem_d, da, db, idesc, acc ? 1u : 0u);
        acc = true;
      }
    }
}

// ---------------------------------------------------------------------------
// forward, split-K: part[kb][m-tile rows][n-tile cols] (FP32)
// grid: (num_kblocks, mtiles, ntiles); each CTA loops over its k-tiles
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(UM_THREADS, 1)
k_umma_fwd(const double* __restrict__ A, const double* __restrict__ B, int m, int n, long K, long kx0_cols,
           double w_kx0, int nb, int ktiles_per_cta, float* __restrict__ part, int* __restrict__ err_flag) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const UmmaSmem L = umma_smem(NT, nb);
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(base + 2 * L.stage_bytes);  // [2]
  uint32_t* tslot = (uint32_t*)(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int mt = blockIdx.y, ntile = blockIdx.z;
  const int m0 = mt * UM_M, n0 = ntile * nb;
  const long ktot = (K + UM_KT - 1) / UM_KT;
  const long kt0 = (long)blockIdx.x * ktiles_per_cta;
  const long kt1 = min(ktot, kt0 + ktiles_per_cta);
  const uint32_t ncols = nb <= 32 ? 32 : (nb <= 64 ? 64 : (nb <= 128 ? 128 : 256));
  if (tid == 0) { mbar_init(&bars[0], 1); mbar_init(&bars[1], 1); }
  if (warp == 0) tmem_alloc(tslot, ncols);
  fence_async_smem();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(nb);
  uint32_t phase[2] = {0, 0};
  bool ok = true;
  int nst = 0;
  const int items = (UM_M + nb) * (UM_KT / 8);
  double pre[UM_ITEMS_MAX][8];
  auto load_item = [&](int item, long kt, double* x) {
    const long k0 = kt * UM_KT;
    const bool isA = item < UM_M * (UM_KT / 8);
    const int it2 = isA ? item : item - UM_M * (UM_KT / 8);
    const int rows = isA ? UM_M : nb;
    const int r = it2 % rows, kc = it2 / rows;
    const int grow = (isA ? m0 : n0) + r;
    const double* src = isA ? A : B;
    const long kb0 = k0 + kc * 8;
    if (grow < (isA ? m : n) && kb0 + 8 <= K) {
      const double2* p2 = reinterpret_cast<const double2*>(src + (size_t)grow * K + kb0);
#pragma unroll
      for (int e = 0; e < 4; ++e) { const double2 v = p2[e]; x[2 * e] = v.x; x[2 * e + 1] = v.y; }
    } else {
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const long k = kb0 + e;
        x[e] = (grow < (isA ? m : n) && k < K) ? src[(size_t)grow * K + k] : 0.0;
      }
    }
    if (isA && kb0 < kx0_cols) {
#pragma unroll
      for (int e = 0; e < 8; ++e) if (kb0 + e < kx0_cols) x[e] *= w_kx0;
    }
  };
  auto store_item = [&](int item, unsigned char* sb, const double* x) {
    const bool isA = item < UM_M * (UM_KT / 8);
    const int it2 = isA ? item : item - UM_M * (UM_KT / 8);
    const int rows = isA ? UM_M : nb;
    const int r = it2 % rows, kc = it2 / rows;
    uint4 t[NT];
    split8<NT>(x, t);
    const uint32_t off = canon_off(r, kc, rows);
#pragma unroll
    for (int qq = 0; qq < NT; ++qq) {
      unsigned char* dst = sb + (isA ? qq * L.a_bytes : NT * L.a_bytes + qq * L.b_bytes) + off;
      *reinterpret_cast<uint4*>(dst) = t[qq];
    }
  };
  auto prefetch = [&](long kt) {
#pragma unroll
    for (int q = 0; q < UM_ITEMS_MAX; ++q) {
      const int item = tid + q * UM_THREADS;
      if (item < items) load_item(item, kt, pre[q]);
    }
  };
  if (kt0 < kt1) prefetch(kt0);
  for (long kt = kt0; kt < kt1; ++kt, ++nst) {
    const int s = nst & 1;
    if (nst >= 2) {  // wait until the MMAs that read this buffer are done
      const bool w = mbar_wait(&bars[s], phase[s]);
      if (!__syncthreads_and(w)) { ok = false; break; }
      phase[s] ^= 1;
    }
    unsigned char* sb = base + s * L.stage_bytes;
#pragma unroll
    for (int q = 0; q < UM_ITEMS_MAX; ++q) {
      const int item = tid + q * UM_THREADS;
      if (item < items) store_item(item, sb, pre[q]);
    }
    for (int item = tid + UM_ITEMS_MAX * UM_THREADS; item < items; item += UM_THREADS) {
      double x[8];
      load_item(item, kt, x);
      store_item(item, sb, x);
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      issue_stage<NT>(tmem, smem_u32(sb), L, nb, idesc, nst == 0);
      umma_commit(&bars[s]);
    }
    if (kt + 1 < kt1) prefetch(kt + 1);
  }
  // drain: wait for the last (up to two) committed stages
  if (ok) {
    for (int d = (nst >= 2 ? nst - 2 : 0); d < nst; ++d) {
      const int s = d & 1;
      if (!mbar_wait(&bars[s], phase[s])) { ok = false; break; }
      phase[s] ^= 1;
    }
  }
  ok = __syncthreads_and(ok);
  tc_fence_after();
  float* out = part + ((size_t)blockIdx.x * m + m0) * (size_t)n + n0;
  const int row = (warp & 3) * 32 + (tid & 31);
  if (warp < 4 && ok && nst > 0) {
    for (int c0 = 0; c0 < nb; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (m0 + row < m) {
#pragma unroll
        for (int e = 0; e < 16; ++e)
          if (n0 + c0 + e < n) out[(size_t)row * n + c0 + e] = v[e];
      }
    }
  } else if (warp < 4 && m0 + row < m) {
    for (int c = 0; c < nb && n0 + c < n; ++c) out[(size_t)row * n + c] = 0.0f;
  }
  if (!ok && tid == 0) atomicExch(err_flag, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// C = alpha sum_kb part[kb] in FP64; 64 outputs x 4 partial groups per
// block, groups combined in a fixed order (deterministic)
__global__ void __launch_bounds__(256)
k_umma_fwd_reduce(const float* __restrict__ part, int nkb, size_t nn, double alpha, double* __restrict__ C) {
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
// backward: out[j][c] for a tile of 128 c and nb states j.  Stages run over
// (term, k-chunk of UM_KT states).  A tile rows = c, B tile rows = j, both K = k.
// grid: (ceil(ncol/128), ntiles)
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(UM_THREADS, 1)
k_umma_bwd(const double* __restrict__ M1, const double* __restrict__ X1, double a1_kx0, double a1_rest,
           const double* __restrict__ M2, const double* __restrict__ X2, double a2, int nj, int nk, long ncol,
           long kx0_cols, int nb, double* __restrict__ out, int* __restrict__ err_flag) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const UmmaSmem L = umma_smem(NT, nb);
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(base + 2 * L.stage_bytes);
  uint32_t* tslot = (uint32_t*)(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const long c0 = (long)blockIdx.x * UM_M;
  const int j0 = blockIdx.y * nb;
  const uint32_t ncols = nb <= 32 ? 32 : (nb <= 64 ? 64 : (nb <= 128 ? 128 : 256));
  if (tid == 0) { mbar_init(&bars[0], 1); mbar_init(&bars[1], 1); }
  if (warp == 0) tmem_alloc(tslot, ncols);
  fence_async_smem();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(nb);
  uint32_t phase[2] = {0, 0};
  bool ok = true;
  const int nterm = M2 ? 2 : 1;
  const int kch = (nk + UM_KT - 1) / UM_KT;
  const int nstage = nterm * kch;
  const int items = (UM_M + nb) * (UM_KT / 8);
  double pre[UM_ITEMS_MAX][8];
  auto load_item = [&](int item, int stg, double* x) {
    const int term = stg / kch;
    const int k0 = (stg - term * kch) * UM_KT;
    const double* Mm = term ? M2 : M1;
    const double* Xm = term ? X2 : X1;
    {
      const bool isA = item < UM_M * (UM_KT / 8);
      const int it2 = isA ? item : item - UM_M * (UM_KT / 8);
      const int rows = isA ? UM_M : nb;
      const int r = it2 % rows, kc = it2 / rows;
      if (isA) {
        const long c = c0 + r;
        const double sc = term ? 1.0 : ((c < kx0_cols) ? a1_kx0 : a1_rest);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = k0 + kc * 8 + e;
          x[e] = (c < ncol && k < nk) ? Xm[(size_t)k * ncol + c] * sc : 0.0;
        }
      } else {
        const int j = j0 + r;
        const double sc = term ? a2 : 1.0;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = k0 + kc * 8 + e;
          x[e] = (j < nj && k < nk) ? Mm[(size_t)k * nj + j] * sc : 0.0;
        }
      }
    }
  };
  auto store_item = [&](int item, unsigned char* sb, const double* x) {
    const bool isA = item < UM_M * (UM_KT / 8);
    const int it2 = isA ? item : item - UM_M * (UM_KT / 8);
    const int rows = isA ? UM_M : nb;
    const int r = it2 % rows, kc = it2 / rows;
    uint4 t[NT];
    split8<NT>(x, t);
    const uint32_t off = canon_off(r, kc, rows);
#pragma unroll
    for (int qq = 0; qq < NT; ++qq) {
      unsigned char* dst = sb + (isA ? qq * L.a_bytes : NT * L.a_bytes + qq * L.b_bytes) + off;
      *reinterpret_cast<uint4*>(dst) = t[qq];
    }
  };
  auto prefetch = [&](int stg) {
#pragma unroll
    for (int q = 0; q < UM_ITEMS_MAX; ++q) {
      const int item = tid + q * UM_THREADS;
      if (item < items) load_item(item, stg, pre[q]);
    }
  };
  int nst = 0;
  if (nstage > 0) prefetch(0);
  for (int stg = 0; stg < nstage; ++stg, ++nst) {
    const int s = nst & 1;
    if (nst >= 2) {
      const bool w = mbar_wait(&bars[s], phase[s]);
      if (!__syncthreads_and(w)) { ok = false; break; }
      phase[s] ^= 1;
    }
    unsigned char* sb = base + s * L.stage_bytes;
#pragma unroll
    for (int q = 0; q < UM_ITEMS_MAX; ++q) {
      const int item = tid + q * UM_THREADS;
      if (item < items) store_item(item, sb, pre[q]);
    }
    for (int item = tid + UM_ITEMS_MAX * UM_THREADS; item < items; item += UM_THREADS) {
      double x[8];
      load_item(item, stg, x);
      store_item(item, sb, x);
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      issue_stage<NT>(tmem, smem_u32(sb), L, nb, idesc, nst == 0);
      umma_commit(&bars[s]);
    }
    if (stg + 1 < nstage) prefetch(stg + 1);
  }
  if (ok) {
    for (int d = (nst >= 2 ? nst - 2 : 0); d < nst; ++d) {
      const int s = d & 1;
      if (!mbar_wait(&bars[s], phase[s])) { ok = false; break; }
      phase[s] ^= 1;
    }
  }
  ok = __syncthreads_and(ok);
  tc_fence_after();
  const int row = (warp & 3) * 32 + (tid & 31);
  const long c = c0 + row;
  if (warp < 4 && ok) {
    for (int q0 = 0; q0 < nb; q0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)q0, v);
      if (c < ncol) {
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int j = j0 + q0 + e;
          if (j < nj) out[(size_t)j * ncol + c] = (double)v[e];
        }
      }
    }
  }
  if (!ok && tid == 0) atomicExch(err_flag, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// N tile: the whole N up to 160 (one tile; the two-stage ring of three
// planes still fits shared memory), else tiles of 128
static int umma_nb(int n) {
  int nb = (n + 15) / 16 * 16;
  if (nb > 160) nb = 128;
  if (nb < 16) nb = 16;
  return nb;
}

cudaError_t oa_launch_umma_fwd(cudaStream_t s, int nterm, const double* A, const double* B, int m, int n, long K,
                               long kx0_cols, double w_kx0, double alpha, float* part, int max_kb, double* C,
                               int* err_flag, int nsm) {
  const int nb = umma_nb(n);
  const int mtiles = (m + UM_M - 1) / UM_M, ntiles = (n + nb - 1) / nb;
  const long ktot = (K + UM_KT - 1) / UM_KT;
  int kb = nsm / (mtiles * ntiles);
  if (kb < 1) kb = 1;
  if (kb > max_kb) kb = max_kb;
  const int per = (int)((ktot + kb - 1) / kb);
  kb = (int)((ktot + per - 1) / per);
  const UmmaSmem L = umma_smem(nterm, nb);
  if (L.total > OA_MAX_SMEM) return cudaErrorInvalidValue;
  dim3 grid(kb, mtiles, ntiles);
  cudaError_t e;
  if (nterm == 2) {
    e = oa_smem_limit(k_umma_fwd<2>);
    if (e != cudaSuccess) return e;
    k_umma_fwd<2><<<grid, UM_THREADS, L.total, s>>>(A, B, m, n, K, kx0_cols, w_kx0, nb, per, part, err_flag);
  } else {
    e = oa_smem_limit(k_umma_fwd<3>);
    if (e != cudaSuccess) return e;
    k_umma_fwd<3><<<grid, UM_THREADS, L.total, s>>>(A, B, m, n, K, kx0_cols, w_kx0, nb, per, part, err_flag);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const size_t mn = (size_t)m * n;
  k_umma_fwd_reduce<<<(unsigned)((mn + 63) / 64), 256, 0, s>>>(part, kb, mn, alpha, C);
  return cudaGetLastError();
}

cudaError_t oa_launch_umma_bwd(cudaStream_t s, int nterm, const double* M1, const double* X1, double a1_kx0,
                               double a1_rest, const double* M2, const double* X2, double a2, int nj, int nk,
                               long ncol, long kx0_cols, double* out, int* err_flag) {
  const int nb = umma_nb(nj);
  const UmmaSmem L = umma_smem(nterm, nb);
  if (L.total > OA_MAX_SMEM) return cudaErrorInvalidValue;
  dim3 grid((unsigned)((ncol + UM_M - 1) / UM_M), (nj + nb - 1) / nb);
  cudaError_t e;
  if (nterm == 2) {
    e = oa_smem_limit(k_umma_bwd<2>);
    if (e != cudaSuccess) return e;
    k_umma_bwd<2><<<grid, UM_THREADS, L.total, s>>>(M1, X1, a1_kx0, a1_rest, M2, X2, a2, nj, nk, ncol, kx0_cols, nb,
                                                     out, err_flag);
  } else {
    e = oa_smem_limit(k_umma_bwd<3>);
    if (e != cudaSuccess) return e;
    k_umma_bwd<3><<<grid, UM_THREADS, L.total, s>>>(M1, X1, a1_kx0, a1_rest, M2, X2, a2, nj, nk, ncol, kx0_cols, nb,
                                                     out, err_flag);
  }
  return cudaGetLastError();
}

size_t oa_umma_smem_bytes(int nterm, int n) { return umma_smem(nterm, umma_nb(n)).total; }
int oa_umma_max_kb(int m, int n, int nsm) {
  const int nb = umma_nb(n);
  const int tiles = ((m + UM_M - 1) / UM_M) * ((n + nb - 1) / nb);
  const int kb = nsm / tiles;
  return kb < 1 ? 1 : kb;
}
