// Newton-Schulz S^-1/2 on one thread-block cluster (Ortho, ortho.C:109-266,
// 848-971; cp_lowdin.C:180-265), for up to 128 states:
//   B = S bscale, A = I; repeat { C = 3I - A B; B <- B C / 2; A <- C A / 2;
//   err = sqrt(sum (A_old - A_new)^2 / n^2) } until err <= tol or max_iter.
// The cluster's CTAs own the blocks of a 4 x (cs/4) grid over A, B and C
// (global memory, L2 resident); each product block is a row block times a
// column block, staged in shared memory and multiplied with FP64
// tensor-core MMAs (m8n8k4).  The
// phases are separated by cluster barriers, so the kernel is an ordinary
// (graph-capturable) launch; every CTA takes the same convergence decision
// from the same partial sums in the same order.
#include <cooperative_groups.h>
#include "oa_internal.h"

namespace cg = cooperative_groups;

#define NSC_THREADS 512
#define NSC_MAXN 128

__device__ __forceinline__ void nsc_dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

__device__ __forceinline__ void nsc_cp16(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int nb = valid ? 16 : 0;  // src-size 0: zero fill
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(sa), "l"(gmem), "r"(nb));
}

// output blocks of the cluster: rows padded to a multiple of 32, a grid of
// gr = 4 block rows by gc = cs / 4 block columns (blocks of BR x BC)
struct NscGeom { int npad, gc, BR, BC; };
__host__ __device__ inline NscGeom nsc_geom(int n, int cs) {
  NscGeom g;
  g.npad = (n + 31) & ~31;
  g.gc = cs / 4;
  g.BR = g.npad / 4;
  g.BC = g.npad / g.gc;
  return g;
}
// two staged products
static inline size_t nsc_smem_bytes(int n, int cs) {
  const NscGeom g = nsc_geom(n, cs);
  return 2 * ((size_t)g.BR * (g.npad + 4) + (size_t)g.npad * (g.BC + 4)) * sizeof(double);
}

// One or two block products, staged together:
//   Z_p[r0 .. r0+BR)[c0 .. c0+BC) = alpha_p X_p[r0 .. r0+BR)[:] Y_p[:][c0 .. c0+BC) + diag_p I,
// n x n row-major in global memory, zero-padded to npad in shared memory
// (the operands of product p at stage p of Xs / Ys).  err (optional): sum
// over the block of (Aold - Z_p)^2 for the last product.
struct NscProd {
  const double* X;
  const double* Y;
  double* Z;
  double alpha, diag;
};
__device__ __forceinline__ void nsc_gemm_blk(NscProd p0, NscProd p1, int np, int n, const NscGeom& G, int r0, int c0,
                                             double* Xs, double* Ys, const double* __restrict__ Aold, double* err) {
  const int ldx = G.npad + 4, ldy = G.BC + 4;
  const size_t xstage = (size_t)G.BR * ldx, ystage = (size_t)G.npad * ldy;
  __syncthreads();  // the previous products are done with Xs / Ys
  // 16-byte asynchronous copies (n even), zero-filled outside n x n
  const int px = G.npad / 2, pc = G.BC / 2;
  for (int p = 0; p < np; ++p) {
    const double* X = p ? p1.X : p0.X;
    const double* Y = p ? p1.Y : p0.Y;
    double* xs = Xs + p * xstage;
    double* ys = Ys + p * ystage;
    for (int i = threadIdx.x; i < G.BR * px; i += blockDim.x) {
      const int r = i / px, k = (i - r * px) * 2;
      const bool v = (r0 + r < n) && (k < n);
      nsc_cp16(xs + r * ldx + k, v ? X + (size_t)(r0 + r) * n + k : X, v);
    }
    for (int i = threadIdx.x; i < G.npad * pc; i += blockDim.x) {
      const int k = i / pc, j = (i - k * pc) * 2;
      const bool v = (k < n) && (c0 + j < n);
      nsc_cp16(ys + k * ldy + j, v ? Y + (size_t)k * n + c0 + j : Y, v);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rt_n = G.BR / 8, ct_n = G.BC / 8;
  double e = 0.0;
  for (int t = warp; t < np * rt_n * ct_n; t += NSC_THREADS / 32) {
    const int p = t / (rt_n * ct_n), tt = t - p * (rt_n * ct_n);
    const int rt = tt % rt_n, ct = tt / rt_n;
    const double* xr = Xs + p * xstage + (rt * 8 + (lane >> 2)) * ldx + (lane & 3);
    const double* yc = Ys + p * ystage + (lane & 3) * ldy + ct * 8 + (lane >> 2);
    double d0 = 0.0, d1 = 0.0;
    for (int k4 = 0; k4 < G.npad; k4 += 4) nsc_dmma(d0, d1, xr[k4], yc[k4 * ldy]);
    const double alpha = p ? p1.alpha : p0.alpha, diag = p ? p1.diag : p0.diag;
    double* Z = p ? p1.Z : p0.Z;
    const bool chk = Aold && p == np - 1;
    const int i = r0 + rt * 8 + (lane >> 2);
    const int j = c0 + ct * 8 + 2 * (lane & 3);
    if (i < n) {
      if (j < n) {
        const double v = alpha * d0 + (i == j ? diag : 0.0);
        if (chk) { const double d = __ldcg(Aold + (size_t)i * n + j) - v; e += d * d; }
        Z[(size_t)i * n + j] = v;
      }
      if (j + 1 < n) {
        const double v = alpha * d1 + (i == j + 1 ? diag : 0.0);
        if (chk) { const double d = __ldcg(Aold + (size_t)i * n + j + 1) - v; e += d * d; }
        Z[(size_t)i * n + j + 1] = v;
      }
    }
  }
  if (err) *err += e;
}

// deterministic block sum (valid in every thread)
__device__ double nsc_block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < NSC_THREADS / 32; ++w) s += sh[w];
  return s;
}

__device__ double nsc_block_max(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < NSC_THREADS / 32; ++w) s = fmax(s, sh[w]);
  return s;
}

__global__ void __launch_bounds__(NSC_THREADS)
k_ortho_ns_cluster(const double* __restrict__ S, int n, double bscale, double tol, int max_iter,
                   double* __restrict__ A0, double* __restrict__ A1, double* __restrict__ B0,
                   double* __restrict__ B1, double* __restrict__ Cm, double* __restrict__ errpart,
                   double* __restrict__ T, int* __restrict__ status, double* __restrict__ errv) {
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) double nsc_smem[];
  __shared__ double sh[NSC_THREADS / 32];
  const int ncta = (int)cl.num_blocks();
  const int me = (int)cl.block_rank();
  const NscGeom G = nsc_geom(n, ncta);
  const int r0 = (me / G.gc) * G.BR, c0 = (me % G.gc) * G.BC;
  double* Xs = nsc_smem;
  double* Ys = nsc_smem + 2 * (size_t)G.BR * (G.npad + 4);
  const size_t nn = (size_t)n * n;
  // init: A = I, B = S bscale on the own block; max |S - I/bscale|
  double dmax = 0.0;
  for (int i = threadIdx.x; i < G.BR * G.BC; i += blockDim.x) {
    const int r = r0 + i / G.BC, c = c0 + i % G.BC;
    if (r >= n || c >= n) continue;
    const size_t o = (size_t)r * n + c;
    A0[o] = (r == c) ? 1.0 : 0.0;
    B0[o] = S[o] * bscale;
    dmax = fmax(dmax, fabs(S[o] - ((r == c) ? 1.0 / bscale : 0.0)));
  }
  dmax = nsc_block_max(dmax, sh);
  if (threadIdx.x == 0) errpart[me] = dmax;
  __threadfence();
  cl.sync();
  if (me == 0 && threadIdx.x == 0) {
    double m = 0.0;
    for (int b = 0; b < ncta; ++b) m = fmax(m, __ldcg(errpart + b));
    errv[1] = m;
  }
  __threadfence();
  cl.sync();  // errpart is reused below
  double* A = A0; double* An = A1; double* B = B0; double* Bn = B1;
  int it = 0;
  double err = 1.0;
  while (true) {
    // C = 3I - A B (own rows)
    nsc_gemm_blk(NscProd{A, B, Cm, -1.0, 3.0}, NscProd{A, B, Cm, -1.0, 3.0}, 1, n, G, r0, c0, Xs, Ys, nullptr,
                 nullptr);
    __threadfence();
    cl.sync();
    // Bn = B C / 2 ; An = C A / 2 (own rows), with the error partial
    double e = 0.0;
    nsc_gemm_blk(NscProd{B, Cm, Bn, 0.5, 0.0}, NscProd{Cm, A, An, 0.5, 0.0}, 2, n, G, r0, c0, Xs, Ys, A, &e);
    e = nsc_block_sum(e, sh);
    if (threadIdx.x == 0) errpart[me] = e;
    __threadfence();
    cl.sync();
    ++it;
    double ssum = 0.0;
    for (int b = 0; b < ncta; ++b) ssum += __ldcg(errpart + b);
    err = sqrt(ssum / (double)nn);
    const bool done = !(err > tol && it < max_iter);
    { double* t = A; A = An; An = t; t = B; B = Bn; Bn = t; }
    if (done) break;
    // errpart is rewritten only after the next cluster barrier (after the
    // C product), by which time every CTA has read it
  }
  for (int i = threadIdx.x; i < G.BR * G.BC; i += blockDim.x) {
    const int r = r0 + i / G.BC, c = c0 + i % G.BC;
    if (r < n && c < n) T[(size_t)r * n + c] = A[(size_t)r * n + c];
  }
  if (me == 0 && threadIdx.x == 0) {
    status[0] = it;
    status[1] = (err <= tol) ? 1 : 0;
    errv[0] = err;
  }
}

// Cluster size for the Newton-Schulz kernel on this device (16 where the
// device allows non-portable clusters of 16 with the shared memory needed,
// else 8); 0 when n is too large for it.
int oa_ns_cluster_size(int n) {
  if (n < 2 || n > NSC_MAXN || (n & 1)) return 0;  // 16-byte row copies need even n
  for (int cs = 16; cs >= 8; cs /= 2) {
    const size_t sm = nsc_smem_bytes(n, cs);
    if (oa_smem_limit(k_ortho_ns_cluster) != cudaSuccess)
      continue;
    if (cs > 8 && cudaFuncSetAttribute(k_ortho_ns_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                      cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs); cfg.blockDim = dim3(NSC_THREADS); cfg.dynamicSmemBytes = sm;
    cfg.attrs = at; cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, (void*)k_ortho_ns_cluster, &cfg) == cudaSuccess && ncl >= 1) return cs;
    cudaGetLastError();
  }
  return 0;
}

cudaError_t oa_launch_ortho_ns_cluster(cudaStream_t s, const double* S, int n, double bscale, double tol,
                                       int max_iter, double* work, double* T, int* status, double* errv, int cs) {
  const size_t nn = (size_t)n * n;
  double* A0 = work; double* A1 = A0 + nn; double* B0 = A1 + nn; double* B1 = B0 + nn; double* Cm = B1 + nn;
  double* errpart = Cm + nn;
  if (cs != 8 && cs != 16) return cudaErrorInvalidValue;
  const size_t sm = nsc_smem_bytes(n, cs);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(cs); cfg.blockDim = dim3(NSC_THREADS); cfg.dynamicSmemBytes = sm; cfg.stream = s;
  cfg.attrs = at; cfg.numAttrs = 1;
  // the shared-memory limit is a per-function setting: contexts of other
  // sizes in the same process may have changed it since this one was sized
  const cudaError_t e = oa_smem_limit(k_ortho_ns_cluster);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernelEx(&cfg, k_ortho_ns_cluster, S, n, bscale, tol, max_iter, A0, A1, B0, B1, Cm, errpart, T,
                            status, errv);
}
