// Split-BF16 PairCalculator GEMMs with TMA-fed tcgen05 MMAs, mixed-precision form.
//
// Operand format ("bf16 planes"): an FP64 matrix X [rows][K] becomes NT bf16
// planes x = P_0 + P_1 (+ P_2), P_0 = bf16(x), P_1 = bf16(x - P_0), ...,
// stored in 64-column chunks P[q][ldp/64][rows_pad][64] (K padded with
// zeros to ldp, a multiple of 64; rows padded with zero rows;
// oa_planes.cuh).  Every TMA box is 64 columns (128 bytes) by a run of rows,
// one contiguous piece of memory, loaded with the 128-byte swizzle, which
// lands as the UMMA SWIZZLE_128B canonical layout for both uses of a plane:
//   K-major view (forward GEMM, contiguous = K): box {64 k, R rows}
//       -> R rows of 128 B; 8-row groups 1024 B apart (SBO); the four
//          K = 16 steps of a box start 32 B apart
//   MN-major view (backward GEMM, contiguous = MN): boxes {64 mn, 32 k}
//       -> 32 k rows of 128 B per 64-wide MN chunk; chunks 4096 B apart
//          (LBO), 8-row K groups 1024 B apart (SBO); K = 16 steps 2048 B apart
//
//   k_tfwd : C[x][y] = alpha sum_k A[x][k] B[y][k]            (Lambda, the nonlocal Z)
//            PairCalculator::multiplyForward (ckPairCalculator.C:821-893)
//   k_tbwd : out[j][c] = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c]
//            bwMultiplyHelper / bwMultiplyDynOrthoT (ckPairCalculator.C:1710-2031)
//
// k_tfwd: one thread issues the TMA loads (mbarrier complete_tx) and the
// MMAs (tcgen05.commit -> mbarrier) over a ring of stages; the block reads
// the FP32 TMEM accumulators in the epilogue.  k_tbwd is persistent and
// warp-specialised (below).  Every wait is bounded: on timeout the block
// sets the device error flag, waits (bounded) for the copies it issued,
// frees its TMEM and returns.  No multicast.
#include <cuda.h>
#include <cuda_bf16.h>
#include <mutex>
#include "oa_internal.h"
#include "oa_wait.cuh"

typedef __nv_bfloat16 bf16;

#define TG_KS 32            // k rows per stage (backward)
#define TG_KF 64            // K per stage (forward)
#define TG_M 128
#define TG_THREADS 128

__device__ __forceinline__ uint32_t tg_s32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, SWIZZLE_128B layout (type 2), version 1
__device__ __forceinline__ uint64_t tg_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
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
  return oa_mbar_wait_bounded(tg_s32(bar), phase);
}
// box of 64 columns x the map's rows starting at (row, column chunk ch) of
// plane q, into shared memory, completing on bar (4-D tile load)
__device__ __forceinline__ void tg_tma_box(uint32_t dst, const CUtensorMap* map, int row, int ch, int q,
                                           uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];"
      :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(row), "r"(ch), "r"(q), "r"(tg_s32(bar))
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
// FP64 [rows][K] (row stride ldx) -> planes P[q][ldp/64][rows_pad][64],
// columns k < kx0_cols scaled by w_kx0 first; padding columns [K, ldp) and
// rows [rows, rows_pad) zero.  One thread per 8 consecutive elements of a row.
// ---------------------------------------------------------------------------
template <int NT>
__global__ void k_split_kc(const double* __restrict__ X, int rows, int rows_pad, long K, long ldx, long kx0_cols,
                           double w_kx0, bf16* __restrict__ P, long ldp, const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  const size_t total = (size_t)rows_pad * (ldp / 8);
  const size_t pstride = (size_t)rows_pad * ldp;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    // t -> (64-column chunk, row, 8-column piece), piece fastest: consecutive
    // threads write consecutive 16-byte pieces of the chunked plane
    const size_t per_chunk = (size_t)rows_pad * 8;
    const long ch = (long)(t / per_chunk);
    const int rem = (int)(t - (size_t)ch * per_chunk);
    const int r = rem >> 3;
    const long k0 = ch * 64 + (rem & 7) * 8;
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
      *reinterpret_cast<uint4*>(P + q * pstride + oa_plane_at(r, k0, rows_pad)) = *reinterpret_cast<uint4*>(&h[q][0]);
  }
}

// Failure-detection test hook (oa_gpu_fault_inject): when set, the first
// k_tfwd block (0, 0, 0) to read it takes it back and skips the TMA loads of
// its first stage, so its wait on that stage runs out of time.
__device__ int g_oa_inject_skip_load = 0;

extern "C" oa_status oa_gpu_fault_inject(oa_ctx* c, int kind) {
  if (!c || (kind != 0 && kind != 1)) {
    oa_set_error("kind must be 0 (clear) or 1 (skip one stage's loads)", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  const int v = kind;
  OA_CUDA_TRY(cudaMemcpyToSymbol(g_oa_inject_skip_load, &v, sizeof(int)));
  return OA_OK;
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
  constexpr uint32_t a_bytes = TG_M * TG_KF * 2, b_bytes = (uint32_t)NB * TG_KF * 2;
  constexpr uint32_t stage_bytes = NT * (a_bytes + b_bytes);
  uint64_t* full = (uint64_t*)(base + (size_t)stages * stage_bytes);
  uint64_t* empty = full + stages;
  uint32_t* tslot = (uint32_t*)(empty + stages);
  int* okflag = (int*)(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.y * TG_M, n0 = blockIdx.z * NB;
  const int kb = blockIdx.x;
  const long rslabs = (K + TG_KF - 1) / TG_KF;
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
    const bool skip0 = (blockIdx.x | blockIdx.y | blockIdx.z) == 0 && atomicExch(&g_oa_inject_skip_load, 0) != 0;
    auto issue_loads = [&](int sl, int st) {
      if (skip0 && sl == 0) return;  // injected failure: stage 0 never fills
      const int k0 = (kb + sl * nkb) * TG_KF;
      const uint32_t sb = sbase + st * stage_bytes;
      tg_expect_tx(&full[st], stage_bytes);
#pragma unroll
      for (int q = 0; q < NT; ++q) {
        tg_tma_box(sb + q * a_bytes, &tA, m0, k0 / 64, q, &full[st]);
        tg_tma_box(sb + NT * a_bytes + q * b_bytes, &tB, n0, k0 / 64, q, &full[st]);
      }
    };
    bool ok = true;
    const int pre = nslab < stages ? nslab : stages;
    for (int s = 0; s < pre; ++s) issue_loads(s, s);
    int issued = pre;
    int committed = -1;  // last slab whose MMAs were committed
    for (int sl = 0; sl < nslab && ok; ++sl) {
      const int st = sl % stages;
      const uint32_t ph = (uint32_t)(sl / stages) & 1u;
      if (!tg_wait(&full[st], ph)) { ok = false; break; }
      tg_tc_after();
      const uint32_t sb = sbase + st * stage_bytes;
      // K-major, 128-byte swizzle: rows 128 B apart, 8-row groups 1024 B
      // apart (SBO); K steps of 16 elements 32 B apart inside the rows
      bool acc = sl > 0;
#pragma unroll
      for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          if (i + j > NT - 1) continue;
#pragma unroll
          for (int ks = 0; ks < TG_KF / 16; ++ks) {
            const uint64_t da = tg_desc(sb + i * a_bytes + ks * 32, 16, 1024);
            const uint64_t db = tg_desc(sb + NT * a_bytes + j * b_bytes + ks * 32, 16, 1024);
            tg_mma(tmem, da, db, idesc, acc ? 1u : 0u);
            acc = true;
          }
        }
      tg_commit(&empty[st]);
      committed = sl;
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
      // let the loads already issued land before the block exits: wait for
      // the phase of the last slab issued on each stage
      for (int s2 = 0; s2 < stages && s2 < issued; ++s2) {
        const int last = issued - 1 - ((issued - 1 - s2) % stages);
        if (skip0 && last == 0) continue;  // never issued
        (void)tg_wait(&full[s2], (uint32_t)(last / stages) & 1u);
      }
      // and the MMAs already issued finish before TMEM is freed (the last
      // commit tracks all of them)
      if (committed >= 0) (void)tg_wait(&empty[committed % stages], (uint32_t)(committed / stages) & 1u);
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

// C = alpha sum_kb part[kb]: block of 256 threads = 16 outputs x 16 K-block
// groups; group g sums kb = g, g + 16, ... (all loads issued together),
// then the 16 group sums are added in a fixed order
__global__ void __launch_bounds__(256)
k_tfwd_reduce(const float* __restrict__ part, int nkb, size_t nn, double alpha, double* __restrict__ C,
              const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  __shared__ double ss[16][17];
  const int col = threadIdx.x & 15, g = threadIdx.x >> 4;
  const size_t i = (size_t)blockIdx.x * 16 + col;
  double s = 0.0;
  if (i < nn) {
    int k = g;
    for (; k + 48 < nkb; k += 64) {
      const float a = __ldcs(part + (size_t)k * nn + i);
      const float b = __ldcs(part + (size_t)(k + 16) * nn + i);
      const float c = __ldcs(part + (size_t)(k + 32) * nn + i);
      const float d = __ldcs(part + (size_t)(k + 48) * nn + i);
      s += (double)a; s += (double)b; s += (double)c; s += (double)d;
    }
    for (; k < nkb; k += 16) s += (double)__ldcs(part + (size_t)k * nn + i);
  }
  ss[g][col] = s;
  __syncthreads();
  if (g == 0 && i < nn) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 16; ++q) t += ss[q][col];
    C[i] = alpha * t;
  }
}

// ---------------------------------------------------------------------------
// backward, persistent: CTA b takes the 128-column tiles b, b + grid, ...;
// D_t[c][j] per term t in TMEM.  Warp roles: warp 0 lane 0 issues the TMA
// loads over a ring of stages, warp 1 lane 0 issues the MMAs into one of
// two TMEM accumulators (tile i uses buffer i & 1), warps 2-5 drain the
// other accumulator (TMEM lane quarter warp & 3) to FP64 while the next
// tile's loads and MMAs run.
//   full[s]  : TMA bytes of stage s landed      (producer -> MMA)
//   empty[s] : MMAs reading stage s are done    (MMA commit -> producer)
//   accf[b]  : accumulator b complete           (MMA commit -> epilogue)
//   acce[b]  : accumulator b read out           (4 epilogue warps -> MMA)
// ---------------------------------------------------------------------------
#define TB_THREADS 192

__device__ __forceinline__ void tg_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(tg_s32(bar)) : "memory");
}

template <int NT, int NB>
__global__ void __launch_bounds__(TB_THREADS, 1)
k_tbwd(const __grid_constant__ CUtensorMap tX1, const __grid_constant__ CUtensorMap tM1,
       const __grid_constant__ CUtensorMap tX2, const __grid_constant__ CUtensorMap tM2, int nterm, double a1_kx0,
       double a1_rest, double a2, int nj, int nk, long ncol, long kx0_cols, int stages, double* out,
       int* __restrict__ err_flag, const double* yadd, const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  extern __shared__ __align__(1024) unsigned char tg_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)tg_raw + 1023) & ~(uintptr_t)1023);
  static_assert(NB == 64 || NB == 128, "k_tbwd: N tile of 64 or 128");
  constexpr uint32_t a_bytes = TG_M * TG_KS * 2, b_bytes = (uint32_t)NB * TG_KS * 2;
  constexpr uint32_t stage_bytes = NT * (a_bytes + b_bytes);
  constexpr int NBP = NB;
  constexpr uint32_t ncols = 4 * NBP;  // two accumulators of two terms
  uint64_t* full = (uint64_t*)(base + (size_t)stages * stage_bytes);
  uint64_t* empty = full + stages;
  uint64_t* accf = empty + stages;
  uint64_t* acce = accf + 2;
  uint32_t* tslot = (uint32_t*)(acce + 2);
  volatile int* okflag = (volatile int*)(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long ntile = (ncol + TG_M - 1) / TG_M;
  const int my_tiles = blockIdx.x < ntile ? (int)((ntile - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  const int kch = (nk + TG_KS - 1) / TG_KS;
  const int nslab = nterm * kch;
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) { tg_bar_init(&full[s], 1); tg_bar_init(&empty[s], 1); }
    for (int b = 0; b < 2; ++b) { tg_bar_init(&accf[b], 1); tg_bar_init(&acce[b], 4); }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *okflag = 1;
  }
  if (warp == 0) tg_tmem_alloc(tslot, ncols);
  __syncthreads();
  tg_tc_after();
  const uint32_t tmem = *tslot;
  if (warp == 0) {
    if (lane == 0) {
      // TMA producer
      const uint32_t sbase = tg_s32(base);
      long g = 0;
      bool ok = true;
      for (int i = 0; i < my_tiles && ok; ++i) {
        const int c0 = (int)(((long)blockIdx.x + (long)i * gridDim.x) * TG_M);
        for (int sl = 0; sl < nslab; ++sl, ++g) {
          const int st = (int)(g % stages);
          if (!tg_wait(&empty[st], (uint32_t)((g / stages) & 1) ^ 1u) || !*okflag) { ok = false; break; }
          const int term = sl / kch;
          const int k0 = (sl - term * kch) * TG_KS;
          const CUtensorMap* tx = term ? &tX2 : &tX1;
          const CUtensorMap* tm = term ? &tM2 : &tM1;
          const uint32_t sb = sbase + st * stage_bytes;
          tg_expect_tx(&full[st], stage_bytes);
          // 64-wide MN chunks of 32 k rows, 4096 B each
#pragma unroll
          for (int q = 0; q < NT; ++q) {
            tg_tma_box(sb + q * a_bytes, tx, k0, c0 / 64, q, &full[st]);
            tg_tma_box(sb + q * a_bytes + 4096, tx, k0, c0 / 64 + 1, q, &full[st]);
#pragma unroll
            for (int h = 0; h < NB / 64; ++h) tg_tma_box(sb + NT * a_bytes + q * b_bytes + h * 4096, tm, k0, h, q, &full[st]);
          }
        }
      }
      if (!ok) {
        *okflag = 0;
        // let every issued load land before the block exits: the last
        // issue on stage s is at most one phase ahead of its consumer
        for (int s2 = 0; s2 < stages && s2 < g; ++s2) {
          const long last = g - 1 - ((g - 1 - s2) % stages);
          (void)tg_wait(&full[s2], (uint32_t)((last / stages) & 1));
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      constexpr uint32_t idesc = tg_idesc(NB, 1, 1);
      const uint32_t sbase = tg_s32(base);
      long g = 0;
      bool ok = true;
      for (int i = 0; i < my_tiles && ok; ++i) {
        const int b = i & 1;
        if (!tg_wait(&acce[b], (uint32_t)((i >> 1) & 1) ^ 1u) || !*okflag) { ok = false; break; }
        tg_tc_after();
        for (int sl = 0; sl < nslab; ++sl, ++g) {
          const int st = (int)(g % stages);
          if (!tg_wait(&full[st], (uint32_t)((g / stages) & 1)) || !*okflag) { ok = false; break; }
          tg_tc_after();
          const int term = sl / kch;
          const bool first_of_term = (sl - term * kch) == 0;
          const uint32_t sb = sbase + st * stage_bytes;
          // MN-major, 128-byte swizzle: 64-wide MN chunks 4096 B apart (LBO),
          // 8-row K groups 1024 B apart (SBO); K steps of 16 rows 2048 B apart
          const uint32_t td = tmem + (uint32_t)(b * 2 * NBP + term * NBP);
          bool acc = !first_of_term;
#pragma unroll
          for (int i2 = 0; i2 < NT; ++i2)
#pragma unroll
            for (int j2 = 0; j2 < NT; ++j2) {
              if (i2 + j2 > NT - 1) continue;
#pragma unroll
              for (int ks = 0; ks < TG_KS / 16; ++ks) {
                const uint64_t da = tg_desc(sb + i2 * a_bytes + ks * 2048, 4096, 1024);
                const uint64_t db = tg_desc(sb + NT * a_bytes + j2 * b_bytes + ks * 2048, 4096, 1024);
                tg_mma(td, da, db, idesc, acc ? 1u : 0u);
                acc = true;
              }
            }
          tg_commit(&empty[st]);
        }
        if (!ok) break;
        tg_commit(&accf[b]);
      }
      if (!ok) *okflag = 0;
    }
  } else {
    // epilogue: TMEM lane quarter q = warp & 3 holds columns c0 + 32 q ..
    const int q = warp & 3;
    const int row = q * 32 + lane;
    for (int i = 0; i < my_tiles; ++i) {
      const int b = i & 1;
      if (!tg_wait(&accf[b], (uint32_t)((i >> 1) & 1))) { *okflag = 0; break; }
      tg_tc_after();
      if (!*okflag) break;
      const long c = ((long)blockIdx.x + (long)i * gridDim.x) * TG_M + row;
      const double a1 = (c < kx0_cols) ? a1_kx0 : a1_rest;
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 2 * NBP);
      for (int q0 = 0; q0 < NB; q0 += 16) {
        float v1[16], v2[16];
        tg_tmem_ld16(tbase + (uint32_t)q0, v1);
        if (nterm == 2) tg_tmem_ld16(tbase + (uint32_t)(NBP + q0), v2);
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
      tg_tc_before();
      __syncwarp();
      if (lane == 0) tg_arrive(&acce[b]);
    }
  }
  __syncthreads();
  if (!*okflag && tid == 0) atomicExch(err_flag, 1);
  tg_tc_after();
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

// planes P[nt][ldp/64][rows][64] as a 4-D bf16 tensor {64, rows, ldp/64, nt};
// box {64, br, 1, 1} (128-byte rows, one contiguous piece) with the 128-byte swizzle
static bool tg_map(CUtensorMap* map, const bf16* P, int nt, int rows, long ldp, int br) {
  EncodeTiledFn enc = tg_encoder();
  if (!enc || (((uintptr_t)P) & 15) || (ldp & 63) || br > 256) return false;
  const cuuint64_t dims[4] = {64, (cuuint64_t)rows, (cuuint64_t)(ldp / 64), (cuuint64_t)nt};
  const cuuint64_t strides[3] = {128, (cuuint64_t)rows * 128, (cuuint64_t)rows * (cuuint64_t)ldp * 2};
  const cuuint32_t box[4] = {64, (cuuint32_t)br, 1, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)P, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

int oa_tgemm_available() { return tg_encoder() != nullptr; }

cudaError_t oa_split_kc(cudaStream_t s, int nt, const double* X, int rows, int rows_pad, long K, long ldx,
                        long kx0_cols, double w_kx0, bf16* P, long ldp, const int* cond) {
  if (rows_pad < rows || (ldp & 63)) return cudaErrorInvalidValue;
  const size_t total = (size_t)rows_pad * (ldp / 8);
  const unsigned nblk = (unsigned)((total + 255) / 256 < 8 * 148 ? (total + 255) / 256 : 8 * 148);
  if (nt == 2) k_split_kc<2><<<nblk, 256, 0, s>>>(X, rows, rows_pad, K, ldx, kx0_cols, w_kx0, P, ldp, cond);
  else k_split_kc<3><<<nblk, 256, 0, s>>>(X, rows, rows_pad, K, ldx, kx0_cols, w_kx0, P, ldp, cond);
  return cudaGetLastError();
}

// rows of the planes of an operand the kernels read in boxes of `box` rows
int oa_tg_rows_pad(int rows, int box) { return (rows + box - 1) / box * box; }
int oa_tg_nb(int n) { return n <= 64 ? 64 : (n <= 128 ? 128 : 0); }
// N tile of the forward product: whole N up to 128, else tiles of 128
int oa_tg_nb_fwd(int n) { return n <= 128 ? oa_tg_nb(n) : 128; }

static int tg_nb(int n) { return n <= 64 ? 64 : (n <= 128 ? 128 : 0); }
// forward stages carry TG_KF columns of K, backward stages TG_KS rows of k
static size_t tg_smem(int nt, int nb, int stages, bool fwd) {
  const size_t kk = fwd ? TG_KF : TG_KS;
  return (size_t)stages * nt * ((size_t)TG_M * kk * 2 + (size_t)nb * kk * 2) + 1024 + 256;
}
static int tg_stages(int nt, int nb, bool fwd) {
  for (int st = 6; st >= 2; --st)
    if (tg_smem(nt, nb, st, fwd) <= (size_t)OA_MAX_SMEM) return st;
  return 0;
}

// C[m][n] = alpha sum_k A[m][k] B[n][k]; PA planes with rows_a rows (a
// multiple of 128), PB with rows_b rows (a multiple of the N tile), both of
// leading size ldp.  NotSupported when the shape or the TMA encoder rules it out.
cudaError_t oa_tfwd(cudaStream_t s, int nt, const bf16* PA, int rows_a, const bf16* PB, int rows_b, int m, int n,
                    long K, long ldp, double alpha, float* part, int max_kb, double* C, int* err_flag, int nsm,
                    const int* cond) {
  const int nb = oa_tg_nb_fwd(n);
  if (nb == 0 || m > rows_a || n > rows_b) return cudaErrorNotSupported;
  const int stages = tg_stages(nt, nb, true);
  if (stages < 2) return cudaErrorNotSupported;
  const int mt = (m + TG_M - 1) / TG_M, ntl = (n + nb - 1) / nb;
  // the planes are padded to whole boxes of rows (oa_tg_rows_pad)
  if (rows_a % TG_M || rows_b % nb || rows_a < m || rows_b < n) return cudaErrorNotSupported;
  CUtensorMap ta, tb;
  if (!tg_map(&ta, PA, nt, rows_a, ldp, TG_M) || !tg_map(&tb, PB, nt, rows_b, ldp, nb)) return cudaErrorNotSupported;
  const long sr = (K + TG_KF - 1) / TG_KF;
  int nkb = nsm / (mt * ntl);
  if (nkb > max_kb) nkb = max_kb;
  if (nkb > sr) nkb = (int)sr;
  if (nkb < 1) nkb = 1;
  const size_t sm = tg_smem(nt, nb, stages, true);
  dim3 grid(nkb, mt, ntl);
  cudaError_t e = cudaErrorNotSupported;
#define OA_TF(NTT, NBB)                                                                                     \
  if (nt == NTT && nb == NBB) {                                                                             \
    e = oa_smem_limit(k_tfwd<NTT, NBB>);        \
    if (e != cudaSuccess) return e;                                                                         \
    k_tfwd<NTT, NBB><<<grid, TG_THREADS, sm, s>>>(ta, tb, m, n, K, nkb, stages, part, err_flag, cond);       \
    e = cudaGetLastError();                                                                                 \
  }
  OA_TF(2, 64) OA_TF(2, 128) OA_TF(3, 64) OA_TF(3, 128)
#undef OA_TF
  if (e != cudaSuccess) return e;
  const size_t mn = (size_t)m * n;
  k_tfwd_reduce<<<(unsigned)((mn + 15) / 16), 256, 0, s>>>(part, nkb, mn, alpha, C, cond);
  return cudaGetLastError();
}

// out[j][c] = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c]
// (+ yadd[j][c], which may be out itself) from X planes (rows nk, leading
// size ldx) and M planes (rows nk, leading size oa_tg_nb(nj), zero beyond
// nj); nk a multiple of 32 (planes padded with zero rows).  cond: optional device flag, nothing runs
// when it is 0.
cudaError_t oa_tbwd(cudaStream_t s, int nt, const bf16* PM1, const bf16* PX1, double a1_kx0, double a1_rest,
                    const bf16* PM2, const bf16* PX2, double a2, int nj, int nk, long ncol, long ldx, long kx0_cols,
                    double* out, int* err_flag, const double* yadd, const int* cond) {
  const int nb = tg_nb(nj);
  if (nb == 0 || ((PM2 == nullptr) != (PX2 == nullptr)) || nk < TG_KS || (nk % TG_KS)) return cudaErrorNotSupported;
  const int stages = tg_stages(nt, nb, false);
  if (stages < 2) return cudaErrorNotSupported;
  CUtensorMap tx1, tm1, tx2, tm2;
  if (!tg_map(&tx1, PX1, nt, nk, ldx, TG_KS) || !tg_map(&tm1, PM1, nt, nk, nb, TG_KS)) return cudaErrorNotSupported;
  const int nterm = PM2 ? 2 : 1;
  if (nterm == 2) {
    if (!tg_map(&tx2, PX2, nt, nk, ldx, TG_KS) || !tg_map(&tm2, PM2, nt, nk, nb, TG_KS)) return cudaErrorNotSupported;
  } else {
    tx2 = tx1; tm2 = tm1;
  }
  const size_t sm = tg_smem(nt, nb, stages, false);
  const long ntile = (ncol + TG_M - 1) / TG_M;
  int nsm = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  dim3 grid((unsigned)(ntile < nsm ? ntile : nsm));
  cudaError_t e = cudaErrorNotSupported;
#define OA_TB(NTT, NBB)                                                                                        \
  if (nt == NTT && nb == NBB) {                                                                                \
    e = oa_smem_limit(k_tbwd<NTT, NBB>);           \
    if (e != cudaSuccess) return e;                                                                            \
    k_tbwd<NTT, NBB><<<grid, TB_THREADS, sm, s>>>(tx1, tm1, tx2, tm2, nterm, a1_kx0, a1_rest, a2, nj, nk, ncol,  \
                                                  kx0_cols, stages, out, err_flag, yadd, cond);                \
    e = cudaGetLastError();                                                                                    \
  }
  OA_TB(2, 64) OA_TB(2, 128) OA_TB(3, 64) OA_TB(3, 128)
#undef OA_TB
  return e;
}
