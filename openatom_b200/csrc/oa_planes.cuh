// bf16 "planes" of an FP64 matrix for the split-BF16 tensor-core GEMMs
// (oa_tgemm.cu): x = P_0 + P_1 (+ P_2), P_0 = bf16(x), P_1 = bf16(x - P_0),
// ..., stored in 64-column chunks, P[q][ldp / 64][rows_pad][64], so that a
// tile of 64 columns and any run of rows is one contiguous piece of memory.
// Kernels that produce such a matrix in FP64 can write its planes in the
// same pass (OaPlaneOut); the digits are the ones k_split_kc computes.
#pragma once
#include <cuda_bf16.h>

struct OaPlaneOut {
  void* P;        // bf16 planes, nullptr = none
  int rows_pad;   // rows per plane
  long ldp;       // leading size (a multiple of 64)
  int nt;         // planes: 2 or 3
};

// offset of element (r, c) in a plane of rows_pad rows
__host__ __device__ __forceinline__ size_t oa_plane_at(int r, long c, int rows_pad) {
  return ((size_t)(c >> 6) * rows_pad + r) * 64 + (size_t)(c & 63);
}

// the nt bf16 digits of v (nt <= 3)
__device__ __forceinline__ void oa_bf16_digits(double v, int nt, __nv_bfloat16* h) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q >= nt) break;
    const __nv_bfloat16 b = __float2bfloat16_rn((float)v);
    h[q] = b;
    v -= (double)__bfloat162float(b);
  }
}

// planes of the pair (x, y) at row r, columns c and c + 1 (c even)
__device__ __forceinline__ void oa_plane_put2(const OaPlaneOut& po, int r, long c, double x, double y) {
  __nv_bfloat16 hx[3], hy[3];
  oa_bf16_digits(x, po.nt, hx);
  oa_bf16_digits(y, po.nt, hy);
  __nv_bfloat16* base = (__nv_bfloat16*)po.P + oa_plane_at(r, c, po.rows_pad);
  const size_t pstride = (size_t)po.rows_pad * po.ldp;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q >= po.nt) break;
    __nv_bfloat162 v;
    v.x = hx[q];
    v.y = hy[q];
    *reinterpret_cast<__nv_bfloat162*>(base + q * pstride) = v;
  }
}
