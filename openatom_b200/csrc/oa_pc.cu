// PairCalculator, Ortho and CP integrator work on one GPU, FP64 form.
//
//   PairCalculator::multiplyForward (ckPairCalculator.C:821-893), tile reduce
//     contributeSubTiles + sumMatrixDouble (:938-1016, :20-53)        -> k_pc_fwd_f64 + k_pc_fwd_reduce
//   Ortho::start_calc/do_iteration/step_2/step_3/tolerance_check/collect_error
//     (ortho.C:109-146, 153-266, 848-971)                             -> k_ortho_ns (cooperative)
//   Ortho::acceptSectionLambda Gamma = T Lambda (ortho.C:565-570)     -> k_small_gemm_tn
//   PairCalculator::multiplyResult/bwMultiplyHelper/bwMultiplyDynOrthoT
//     (ckPairCalculator.C:1201-1468, 1710-2031)                       -> k_pc_bwd_f64
//   CPINTEGRATE::CP_integrate_dyn/cp_evolve_vel/get_fictKE (cp_dynamics.C:29-270)
//     + Gamma redundancy sync (CP_State_GSpacePlane.C:2829-2970)     -> k_integrate + k_sync_redundant
//
// Operand layout: every state row is its coefficients as 2*ng contiguous
// doubles (the DGEMM real view).  kx = 0 rows of the reference's 1/sqrt(2),
// sqrt(2) pre-scalings become per-column weights on the first 2*nkx0 doubles.
#include <cooperative_groups.h>
#include "oa_internal.h"

namespace cg = cooperative_groups;

// D = A(8x4, row) * B(4x8, col) + C, FP64 tensor core (DMMA)
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// forward: part[kb][i][j] = sum_{k in chunk kb} w(k) A[i][k] B[j][k]
//   64x64 output tile per block, 4 warps each 32x32 (4x4 DMMA tiles),
//   K staged through shared memory in slabs of 32.
// ---------------------------------------------------------------------------
#define PC_TM 64
#define PC_KS 32
#define PC_LDS (PC_KS + 4)

__global__ void __launch_bounds__(128)
k_pc_fwd_f64(const double* __restrict__ A, const double* __restrict__ B, int m, int n, long K, long kchunk,
             long kx0_cols, double w_kx0, double* __restrict__ part) {
  __shared__ double As[PC_TM * PC_LDS];
  __shared__ double Bs[PC_TM * PC_LDS];
  const int ti = blockIdx.x, tj = blockIdx.y, kb = blockIdx.z;
  const int i0 = ti * PC_TM, j0 = tj * PC_TM;
  const long kbeg = (long)kb * kchunk;
  const long kend = min(K, kbeg + kchunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wi = (warp >> 1) * 32, wj = (warp & 1) * 32;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) { acc[a][b][0] = 0.0; acc[a][b][1] = 0.0; }
  for (long k0 = kbeg; k0 < kend; k0 += PC_KS) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < PC_TM * PC_KS; idx += blockDim.x) {
      const int r = idx / PC_KS, kk = idx - r * PC_KS;
      const long k = k0 + kk;
      double va = 0.0, vb = 0.0;
      if (k < kend) {
        const double w = (k < kx0_cols) ? w_kx0 : 1.0;
        if (i0 + r < m) va = A[(size_t)(i0 + r) * K + k] * w;
        if (j0 + r < n) vb = B[(size_t)(j0 + r) * K + k];
      }
      As[r * PC_LDS + kk] = va;
      Bs[r * PC_LDS + kk] = vb;
    }
    __syncthreads();
#pragma unroll
    for (int k4 = 0; k4 < PC_KS; k4 += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) af[q] = As[(wi + q * 8 + (lane >> 2)) * PC_LDS + k4 + (lane & 3)];
#pragma unroll
      for (int q = 0; q < 4; ++q) bf[q] = Bs[(wj + q * 8 + (lane >> 2)) * PC_LDS + k4 + (lane & 3)];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
  }
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

__global__ void k_pc_fwd_reduce(const double* __restrict__ part, int nkb, size_t nn, double alpha,
                                double* __restrict__ C) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (size_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nkb; ++k) s += part[(size_t)k * nn + i];
    C[i] = alpha * s;
  }
}

// ---------------------------------------------------------------------------
// backward: out[j][c] = a1(c) sum_k M1[k][j] X1[k][c] + a2 sum_k M2[k][j] X2[k][c]
//   a1(c) = a1_kx0 for c < kx0_cols else a1_rest.  Tile: 64 states x 64 cols,
//   4 warps each 32x32; K = n (states) staged in slabs of 32.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
k_pc_bwd_f64(const double* __restrict__ M1, const double* __restrict__ X1, double a1_kx0, double a1_rest,
             const double* __restrict__ M2, const double* __restrict__ X2, double a2,
             int nj, int nk, long ncol, long kx0_cols, double* __restrict__ out) {
  __shared__ double Ms[PC_KS * (PC_TM + 4)];   // [k][j]
  __shared__ double Xs[PC_KS * (PC_TM + 4)];   // [k][c]
  const int LDT = PC_TM + 4;
  const int tj = blockIdx.y;
  const long c0 = (long)blockIdx.x * PC_TM;
  const int j0 = tj * PC_TM;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wj = (warp >> 1) * 32, wc = (warp & 1) * 32;
  double acc1[4][4][2], acc2[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) { acc1[a][b][0] = acc1[a][b][1] = 0.0; acc2[a][b][0] = acc2[a][b][1] = 0.0; }
  for (int term = 0; term < (M2 ? 2 : 1); ++term) {
    const double* M = term ? M2 : M1;
    const double* X = term ? X2 : X1;
    for (int k0 = 0; k0 < nk; k0 += PC_KS) {
      __syncthreads();
      for (int idx = threadIdx.x; idx < PC_KS * PC_TM; idx += blockDim.x) {
        const int kk = idx / PC_TM, r = idx - kk * PC_TM;
        const int k = k0 + kk;
        double vm = 0.0, vx = 0.0;
        if (k < nk) {
          if (j0 + r < nj) vm = M[(size_t)k * nj + j0 + r];
          if (c0 + r < ncol) vx = X[(size_t)k * ncol + c0 + r];
        }
        Ms[kk * LDT + r] = vm;
        Xs[kk * LDT + r] = vx;
      }
      __syncthreads();
#pragma unroll
      for (int k4 = 0; k4 < PC_KS; k4 += 4) {
        double af[4], bf[4];
        // A fragment (row-major 8x4): A[j][k] = M[k][j]
#pragma unroll
        for (int m = 0; m < 4; ++m) af[m] = Ms[(k4 + (lane & 3)) * LDT + wj + m * 8 + (lane >> 2)];
        // B fragment (col-major 4x8): B[k][c] = X[k][c]
#pragma unroll
        for (int m = 0; m < 4; ++m) bf[m] = Xs[(k4 + (lane & 3)) * LDT + wc + m * 8 + (lane >> 2)];
        if (term == 0) {
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) dmma_8x8x4(acc1[a][b][0], acc1[a][b][1], af[a], bf[b]);
        } else {
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) dmma_8x8x4(acc2[a][b][0], acc2[a][b][1], af[a], bf[b]);
        }
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int j = j0 + wj + a * 8 + (lane >> 2);
      const long c = c0 + wc + b * 8 + 2 * (lane & 3);
      if (j >= nj) continue;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const long cc = c + e;
        if (cc < ncol) {
          const double a1 = (cc < kx0_cols) ? a1_kx0 : a1_rest;
          out[(size_t)j * ncol + cc] = a1 * acc1[a][b][e] + a2 * acc2[a][b][e];
        }
      }
    }
}

// ---------------------------------------------------------------------------
// small N x N: C = alpha * A B, FP64; 16 x 16 output tile per block of
// 256 threads (one output each, k in ascending order), K in slabs of 16
// through shared memory
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_small_gemm(const double* __restrict__ A, const double* __restrict__ B, int n, double alpha,
             double* __restrict__ C) {
  __shared__ double sA[16][17], sB[16][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = blockIdx.y * 16, j0 = blockIdx.x * 16;
  double acc = 0.0;
  for (int k0 = 0; k0 < n; k0 += 16) {
    const int ia = i0 + ty, ka = k0 + tx;
    sA[ty][tx] = (ia < n && ka < n) ? A[(size_t)ia * n + ka] : 0.0;
    const int kb = k0 + ty, jb = j0 + tx;
    sB[ty][tx] = (kb < n && jb < n) ? B[(size_t)kb * n + jb] : 0.0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) acc = fma(sA[ty][k], sB[k][tx], acc);
    __syncthreads();
  }
  const int i = i0 + ty, j = j0 + tx;
  if (i < n && j < n) C[(size_t)i * n + j] = alpha * acc;
}

// Several single-block sums in one launch: block b writes
// out[b] = scale[b] * sum_i part[b][i * stride[b] + off[b]], in the order of
// k_sum_partials.
struct SumJobs {
  const double* part[8];
  double* out[8];
  double scale[8];
  int n[8], stride[8], off[8];
};

// ---------------------------------------------------------------------------
// Newton-Schulz S^-1/2 (ortho.C), one cooperative kernel, bounded iterations.
//   B = S/2 (or S for lsda); A = I; repeat:
//     C = 3I - A B;  B <- B C / 2;  A <- C A / 2;
//     err = sqrt(sum (A_old - A_new)^2 / N^2)
//   until err <= tol or iter == max_iter.  status[0] = iterations,
//   status[1] = 1 if converged; errv[0] = err.
// ---------------------------------------------------------------------------
#define NS_TS 32

__device__ void ns_tile_gemm(const double* __restrict__ X, const double* __restrict__ Y, int n, double alpha,
                             double diag, double* __restrict__ Z, int tile, double* sX, double* sY,
                             const double* __restrict__ Aold, double* err_acc) {
  // Z[tile] = alpha * X Y + diag * I ; optional err += (Aold - Z)^2 on the tile
  const int nt = (n + NS_TS - 1) / NS_TS;
  const int ti = tile / nt, tj = tile - ti * nt;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < n; k0 += NS_TS) {
    __syncthreads();
    for (int r = ty; r < NS_TS; r += 8) {
      const int i = ti * NS_TS + r, k = k0 + tx;
      sX[r * (NS_TS + 1) + tx] = (i < n && k < n) ? X[(size_t)i * n + k] : 0.0;
      const int kk = k0 + r, j = tj * NS_TS + tx;
      sY[r * (NS_TS + 1) + tx] = (kk < n && j < n) ? Y[(size_t)kk * n + j] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < NS_TS; ++k) {
      const double y = sY[k * (NS_TS + 1) + tx];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] += sX[(ty + 8 * q) * (NS_TS + 1) + k] * y;
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = ti * NS_TS + ty + 8 * q, j = tj * NS_TS + tx;
    if (i < n && j < n) {
      double v = alpha * acc[q] + ((i == j) ? diag : 0.0);
      Z[(size_t)i * n + j] = v;
      if (Aold) { const double d = Aold[(size_t)i * n + j] - v; *err_acc += d * d; }
    }
  }
}

__global__ void __launch_bounds__(256)
k_ortho_ns(const double* __restrict__ S, int n, double bscale, double tol, int max_iter,
           double* __restrict__ A0, double* __restrict__ A1, double* __restrict__ B0, double* __restrict__ B1,
           double* __restrict__ Cm, double* __restrict__ errpart, double* __restrict__ T,
           int* __restrict__ status, double* __restrict__ errv) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sX[NS_TS * (NS_TS + 1)];
  __shared__ double sY[NS_TS * (NS_TS + 1)];
  __shared__ double sred[32];
  __shared__ int sdone;
  const int nt = (n + NS_TS - 1) / NS_TS;
  const int ntiles = nt * nt;
  const size_t nn = (size_t)n * n;
  // init: A = I, B = S * bscale; max |S - I/bscale| (Ortho::array_diag_max,
  // ortho.h:282-310) for the PsiV tolerance check
  double dmax = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / n), c = (int)(i - (size_t)r * n);
    A0[i] = (r == c) ? 1.0 : 0.0;
    B0[i] = S[i] * bscale;
    const double dv = fabs(S[i] - ((r == c) ? 1.0 / bscale : 0.0));
    dmax = dv > dmax ? dv : dmax;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
  if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = dmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sred[w]);
    errpart[blockIdx.x] = m;
  }
  grid.sync();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double m = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) m = fmax(m, errpart[b]);
    errv[1] = m;
  }
  grid.sync();
  double* A = A0; double* An = A1; double* B = B0; double* Bn = B1;
  int it = 0;
  double err = 1.0;
  while (true) {
    // C = 3I - A B
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
      ns_tile_gemm(A, B, n, -1.0, 3.0, Cm, t, sX, sY, nullptr, nullptr);
    grid.sync();
    // Bn = B C / 2 ; An = C A / 2 with error partials
    double e_loc = 0.0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      ns_tile_gemm(B, Cm, n, 0.5, 0.0, Bn, t, sX, sY, nullptr, nullptr);
      ns_tile_gemm(Cm, A, n, 0.5, 0.0, An, t, sX, sY, A, &e_loc);
    }
    // deterministic per-block partial
    double v = e_loc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sred[w];
      errpart[blockIdx.x] = s;
    }
    grid.sync();
    ++it;
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int b = 0; b < (int)gridDim.x; ++b) s += errpart[b];
      err = sqrt(s / (double)nn);
      sdone = !(err > tol && it < max_iter);
      sred[0] = err;
    }
    __syncthreads();
    err = sred[0];
    const int done = sdone;
    { double* t = A; A = An; An = t; t = B; B = Bn; Bn = t; }
    if (done) break;
    // errpart is rewritten next iteration only after the next grid.sync
    grid.sync();
  }
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (size_t)gridDim.x * blockDim.x) T[i] = A[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    status[0] = it;
    status[1] = (err <= tol) ? 1 : 0;
    errv[0] = err;
  }
}

// ---------------------------------------------------------------------------
// integrator
// ---------------------------------------------------------------------------
// One block per (chunk of OA_INT_CHUNK coefficients, state): every thread
// loads its OA_INT_UNROLL coefficients before it updates them, and writes one
// kinetic-energy partial per block (kepart[state * gridDim.x + chunk]).
#define OA_INT_UNROLL 4
#define OA_INT_CHUNK (256 * OA_INT_UNROLL)
// P_in (optional) replaces P as the coefficients read when *sel != 0 (the
// PsiV reset of the previous step: psi(t) = the orthonormal psi, and the
// velocity is already at t, so no half kick is completed: halfStepEvolve = 0
// of finiteDifferencePsiV, CP_State_GSpacePlane.C:3776).
__global__ void __launch_bounds__(256)
k_integrate(const double2* __restrict__ F, double2* __restrict__ V, double2* P, const double2* P_in,
            const int* __restrict__ sel, const double* __restrict__ cmass, int ng, int nstate, int r0, int r1,
            int iend, double dt, int complete_prev, double* __restrict__ kepart) {
  __shared__ double sh[8];
  const double dt2 = 0.5 * dt;
  const size_t base = (size_t)blockIdx.y * ng;
  const bool reset = P_in && *sel != 0;
  const double2* src = reset ? P_in : P;
  complete_prev = complete_prev && !reset;
  const int i0 = blockIdx.x * OA_INT_CHUNK + threadIdx.x;
  double2 f[OA_INT_UNROLL], v[OA_INT_UNROLL], p[OA_INT_UNROLL];
  double m[OA_INT_UNROLL];
#pragma unroll
  for (int u = 0; u < OA_INT_UNROLL; ++u) {
    const int i = i0 + 256 * u;
    if (i >= r0 && i < ng) {
      f[u] = F[base + i]; v[u] = V[base + i]; p[u] = src[base + i]; m[u] = __ldg(cmass + i);
    }
  }
  double ke = 0.0;
#pragma unroll
  for (int u = 0; u < OA_INT_UNROLL; ++u) {
    const int i = i0 + 256 * u;
    if (i < r0 || i >= ng) continue;
    double2 ff = f[u], vv = v[u], pp = p[u];
    const double h = dt2 / m[u];
    const bool g0 = (i < r1);
    if (g0) { ff.y = 0.0; vv.y = 0.0; }
    if (complete_prev) { vv.x += ff.x * h; vv.y += ff.y * h; if (g0) vv.y = 0.0; }
    const double mk = (i >= r1 && i < iend) ? 2.0 * m[u] : m[u];
    ke += mk * (vv.x * vv.x + vv.y * vv.y);
    vv.x += ff.x * h; vv.y += ff.y * h;
    if (g0) vv.y = 0.0;
    V[base + i] = vv;
    pp.x += vv.x * dt; pp.y += vv.y * dt;
    P[base + i] = pp;
  }
  double w = ke;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = w;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += sh[k];
    kepart[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = 0.5 * s;
  }
}

int oa_integrate_nblk(int ng, int nstate) { return nstate * ((ng + OA_INT_CHUNK - 1) / OA_INT_CHUNK); }

// ---------------------------------------------------------------------------
// Minimisation (cp_min_opt): CPINTEGRATE::CP_fovlap_calc (cp_min_CG.C:128-140)
// -> k_min_fovlap, sum |F|^2 over every stored point; CP_integrate_min_STD
// (cp_min_std.C:17-60, psi += F dt / m) and CP_integrate_min_CG
// (cp_min_CG.C:29-120, conj = conj gamma + F on g^2 <= ecut, psi += conj
// dt / m) -> k_min_step.  Block partial sums in a fixed order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_min_fovlap(const double2* __restrict__ F, size_t n,
                                                    double* __restrict__ part) {
  __shared__ double sh[8];
  double a = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 f = F[i];
    a += f.x * f.x + f.y * f.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

__global__ void k_min_step(const double2* __restrict__ F, double2* __restrict__ conj, double2* __restrict__ P,
                           const double* __restrict__ cmass, const double* __restrict__ g2, double ecut, int ng,
                           size_t n, double gamma, double dt) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % (size_t)ng);
    double2 d = F[t];
    if (conj) {
      double2 c = conj[t];
      if (g2[i] <= ecut) { c.x = c.x * gamma + d.x; c.y = c.y * gamma + d.y; }
      conj[t] = c;
      d = c;
    }
    const double s = dt / cmass[i];
    double2 p = P[t];
    p.x += d.x * s;
    p.y += d.y * s;
    P[t] = p;
  }
}

#define OA_MIN_NBLK 592

cudaError_t oa_launch_min_fovlap(cudaStream_t s, const double2* F, size_t n, double* part) {
  k_min_fovlap<<<OA_MIN_NBLK, 256, 0, s>>>(F, n, part);
  return cudaGetLastError();
}
int oa_min_nblk() { return OA_MIN_NBLK; }

cudaError_t oa_launch_min_step(cudaStream_t s, const double2* F, double2* conj, double2* P, const double* cmass,
                               const double* g2, double ecut, int ng, int nstate, double gamma, double dt) {
  const size_t n = (size_t)nstate * ng;
  k_min_step<<<OA_MIN_NBLK, 256, 0, s>>>(F, conj, P, cmass, g2, ecut, ng, n, gamma, dt);
  return cudaGetLastError();
}

__global__ void k_sync_redundant(double2* __restrict__ P, double2* __restrict__ V, const int* __restrict__ partner,
                                 int nred, int ng, int nstate) {
  const size_t total = (size_t)nstate * nred;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(t / nred), i = (int)(t - (size_t)s * nred);
    const size_t src = (size_t)s * ng + partner[i];
    const size_t dst = (size_t)s * ng + i;
    double2 p = P[src]; p.y = -p.y; P[dst] = p;
    if (V) { double2 v = V[src]; v.y = -v.y; V[dst] = v; }
  }
}

// sum of part[i * stride + off] over i < n in one block: each thread keeps
// four partial sums with four loads in flight, combined in a fixed order
__device__ __forceinline__ double sum_strided_block(const double* __restrict__ part, int n, int stride, int off,
                                                    double* sh) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  const int nb = blockDim.x;
  int i = threadIdx.x;
  for (; i + 3 * nb < n; i += 4 * nb) {
    const double v0 = part[(size_t)i * stride + off];
    const double v1 = part[(size_t)(i + nb) * stride + off];
    const double v2 = part[(size_t)(i + 2 * nb) * stride + off];
    const double v3 = part[(size_t)(i + 3 * nb) * stride + off];
    a0 += v0; a1 += v1; a2 += v2; a3 += v3;
  }
  for (; i < n; i += nb) a0 += part[(size_t)i * stride + off];
  double s = (a0 + a1) + (a2 + a3);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
  return t;
}

__global__ void k_sum_partials(const double* __restrict__ part, int n, int stride, int off, double scale,
                               double* __restrict__ out) {
  // one block: out[0] = scale * sum_i part[i*stride + off]
  __shared__ double sh[32];
  const double t = sum_strided_block(part, n, stride, off, sh);
  if (threadIdx.x == 0) out[0] = scale * t;
}

__global__ void k_sum_partials_multi(SumJobs J) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  const double t = sum_strided_block(J.part[b], J.n[b], J.stride[b], J.off[b], sh);
  if (threadIdx.x == 0) J.out[b][0] = J.scale[b] * t;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
cudaError_t oa_dgemm_fwd(cudaStream_t s, const double* A, const double* B, int m, int n, long K, long kx0_cols,
                         double w_kx0, double alpha, double* part, int nkb, double* C, const int* cond);

cudaError_t oa_launch_pc_fwd_mn(cudaStream_t s, const double* A, const double* B, int m, int n, long K,
                                long kx0_cols, double w_kx0, double alpha, double* part, int nkb, double* C) {
  // pipelined kernel (oa_dgemm.cu) when the operands allow 16-byte copies
  const cudaError_t e2 = oa_dgemm_fwd(s, A, B, m, n, K, kx0_cols, w_kx0, alpha, part, nkb, C, nullptr);
  if (e2 != cudaErrorNotSupported) return e2;
  const long kchunk = ((K + nkb - 1) / nkb + PC_KS - 1) / PC_KS * PC_KS;
  const int nkb_eff = (int)((K + kchunk - 1) / kchunk);
  dim3 grid((m + PC_TM - 1) / PC_TM, (n + PC_TM - 1) / PC_TM, nkb_eff);
  k_pc_fwd_f64<<<grid, 128, 0, s>>>(A, B, m, n, K, kchunk, kx0_cols, w_kx0, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t mn = (size_t)m * n;
  k_pc_fwd_reduce<<<(unsigned)((mn + 255) / 256), 256, 0, s>>>(part, nkb_eff, mn, alpha, C);
  return cudaGetLastError();
}

cudaError_t oa_launch_pc_fwd(cudaStream_t s, const double* A, const double* B, int n, long K, long kx0_cols,
                             double w_kx0, double alpha, double* part, int nkb, double* C) {
  return oa_launch_pc_fwd_mn(s, A, B, n, n, K, kx0_cols, w_kx0, alpha, part, nkb, C);
}

cudaError_t oa_dgemm_bwd(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                         const double* M2, const double* X2, double a2, int nj, int nk, long ncol, long kx0_cols,
                         double* out, const int* cond);

cudaError_t oa_launch_pc_bwd_jk(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                                const double* M2, const double* X2, double a2, int nj, int nk, long ncol,
                                long kx0_cols, double* out) {
  // pipelined kernel (oa_dgemm.cu) when the shapes allow 16-byte copies
  const cudaError_t e2 = oa_dgemm_bwd(s, M1, X1, a1_kx0, a1_rest, M2, X2, a2, nj, nk, ncol, kx0_cols, out, nullptr);
  if (e2 != cudaErrorNotSupported) return e2;
  dim3 grid((unsigned)((ncol + PC_TM - 1) / PC_TM), (nj + PC_TM - 1) / PC_TM);
  k_pc_bwd_f64<<<grid, 128, 0, s>>>(M1, X1, a1_kx0, a1_rest, M2, X2, a2, nj, nk, ncol, kx0_cols, out);
  return cudaGetLastError();
}

cudaError_t oa_launch_pc_bwd(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                             const double* M2, const double* X2, double a2, int n, long ncol, long kx0_cols,
                             double* out) {
  return oa_launch_pc_bwd_jk(s, M1, X1, a1_kx0, a1_rest, M2, X2, a2, n, n, ncol, kx0_cols, out);
}

cudaError_t oa_launch_small_gemm(cudaStream_t s, const double* A, const double* B, int n, double alpha, double* C) {
  dim3 grid((n + 15) / 16, (n + 15) / 16);
  k_small_gemm<<<grid, 256, 0, s>>>(A, B, n, alpha, C);
  return cudaGetLastError();
}

// six reductions of the density / Hartree partials in one launch (see
// oa_gpu_vks_build): entries b < njob of the arrays
cudaError_t oa_launch_sum_partials_multi(cudaStream_t s, int njob, const double* const* part, const int* n,
                                         const int* stride, const int* off, const double* scale, double* const* out) {
  if (njob < 1 || njob > 8) return cudaErrorInvalidValue;
  SumJobs J;
  for (int b = 0; b < njob; ++b) {
    J.part[b] = part[b]; J.out[b] = out[b]; J.scale[b] = scale[b];
    J.n[b] = n[b]; J.stride[b] = stride[b]; J.off[b] = off[b];
  }
  k_sum_partials_multi<<<njob, 512, 0, s>>>(J);
  return cudaGetLastError();
}

int oa_ns_grid(int n, int device) {
  const int nt = (n + NS_TS - 1) / NS_TS;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ortho_ns, 256, 0);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  int g = nt * nt;
  const int cap = per_sm * nsm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return g;
}

cudaError_t oa_launch_ortho_ns_cluster(cudaStream_t s, const double* S, int n, double bscale, double tol,
                                       int max_iter, double* work, double* T, int* status, double* errv, int cs);

// grid > 0: cooperative kernel on grid blocks; grid < 0: the cluster kernel
// (oa_ns.cu) on a cluster of -grid blocks
cudaError_t oa_launch_ortho_ns(cudaStream_t s, const double* S, int n, double bscale, double tol, int max_iter,
                               double* work /* 5 n^2 + grid */, double* T, int* status, double* errv, int grid) {
  if (grid < 0) return oa_launch_ortho_ns_cluster(s, S, n, bscale, tol, max_iter, work, T, status, errv, -grid);
  const size_t nn = (size_t)n * n;
  double* A0 = work; double* A1 = A0 + nn; double* B0 = A1 + nn; double* B1 = B0 + nn; double* Cm = B1 + nn;
  double* errpart = Cm + nn;
  void* args[] = {(void*)&S, (void*)&n, (void*)&bscale, (void*)&tol, (void*)&max_iter, (void*)&A0, (void*)&A1,
                  (void*)&B0, (void*)&B1, (void*)&Cm, (void*)&errpart, (void*)&T, (void*)&status, (void*)&errv};
  return cudaLaunchCooperativeKernel((void*)k_ortho_ns, dim3(grid), dim3(256), args, 0, s);
}

cudaError_t oa_launch_integrate(cudaStream_t s, const double2* F, double2* V, double2* P, const double2* P_in,
                                const int* sel, const double* cmass, int ng, int nstate, int r0, int r1, int iend,
                                double dt, int complete_prev, double* kepart, int nblk) {
  if (nblk != oa_integrate_nblk(ng, nstate) || (P_in && !sel)) return cudaErrorInvalidValue;
  const dim3 grid((ng + OA_INT_CHUNK - 1) / OA_INT_CHUNK, nstate);
  k_integrate<<<grid, 256, 0, s>>>(F, V, P, P_in, sel, cmass, ng, nstate, r0, r1, iend, dt, complete_prev, kepart);
  return cudaGetLastError();
}

cudaError_t oa_launch_sync_redundant(cudaStream_t s, double2* P, double2* V, const int* partner, int nred, int ng,
                                     int nstate) {
  if (nred == 0) return cudaSuccess;
  const size_t total = (size_t)nstate * nred;
  const int nb = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
  k_sync_redundant<<<nb, 256, 0, s>>>(P, V, partner, nred, ng, nstate);
  return cudaGetLastError();
}

cudaError_t oa_launch_sum_partials(cudaStream_t s, const double* part, int n, int stride, int off, double scale,
                                   double* out) {
  k_sum_partials<<<1, 512, 0, s>>>(part, n, stride, off, scale, out);
  return cudaGetLastError();
}
