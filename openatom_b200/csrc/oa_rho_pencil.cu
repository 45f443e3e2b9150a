// Density-grid plane kernels (FP64) for the grid lengths with a
// compile-time factorisation N = N1 * N2 (oa_rdft.cuh): the same work and
// results as k_rho_plane_fwd / k_rho_plane_bwd (oa_rho.cu), with every 1-D
// transform done as two register passes (pass A: DFT_N1 + twiddle, pass B:
// DFT_N2) around one shared-memory exchange, all indexing by constants.
// One block per z plane; the plane moves through two shared-memory regions
// (A, B) of about N^2 / 2 complex values each:
//   forward:  rho(x,y) V/N -> A (row pairs, complex) -> x pass A -> B -> x pass B
//             -> A (natural order) -> r2c unpack -> B [kx][y] -> y pass A -> A
//             -> y pass B -> dz[z][kx ny + y]
//   backward: dz -> A [kx][y] -> y pass A (+) -> B -> y pass B -> A [kx][y]
//             -> c2r x pass A (+) on row pairs -> B -> x pass B -> vks = V + vxc
// Both take several fields at once (gridDim.y, one field per y index at
// fixed strides): the three components of grad rho and of the GGA vector h.
//
// Reference work replaced (as the oa_rho.cu kernels):
//   fftRhoRtoRhoG (CP_Rho_RealSpacePlane.C:831) + the Charm forward FFT   -> k_rho2_fwd
//   FFTVks (CP_Rho_GHartExt.C:532) + acceptHartVks
//     (CP_Rho_RealSpacePlane.C:1365)                                       -> k_rho2_bwd
#include "oa_rdft.cuh"
#include "oa_state_common.cuh"

template <int N1, int N2> struct Rho2Cfg {
  static constexpr int N = N1 * N2;
  static constexpr int NKX = N / 2 + 1;           // stored kx columns
  static constexpr int NPAIR = (N + 1) / 2;       // row pairs of the x transforms
  static constexpr int LD = N | 1;                // row stride of the [kx][y] / [pair][x] arrays
  static constexpr int LS1 = N2 | 1;              // pass A -> B buffer [pencil][k1][n2]
  static constexpr int PS1 = (N1 * LS1) | 1;
  static constexpr int MAXP = NKX > NPAIR ? NKX : NPAIR;
  static constexpr size_t REGION = (size_t)MAXP * (LD > PS1 ? LD : PS1);  // double2 per region
  static constexpr int NT = 512;
};

template <int N1, int N2>
__global__ void __launch_bounds__(512, 1)
k_rho2_fwd(const double* __restrict__ rho, double scale, const double2* __restrict__ twg,
           double2* __restrict__ dz, int ldl_d, size_t fin, size_t fout) {
  typedef Rho2Cfg<N1, N2> CF;
  constexpr int N = CF::N, NKX = CF::NKX, NPAIR = CF::NPAIR, LD = CF::LD, LS1 = CF::LS1, PS1 = CF::PS1;
  constexpr int NT = CF::NT;
  static_assert(N1 <= 16, "pass B pads a pencil to 16 threads");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = (double2*)smem_raw;
  double2* A = tw + ((N + 1) & ~1);
  double2* B = A + CF::REGION;
  const int z = blockIdx.x, tid = threadIdx.x;
  rho += blockIdx.y * fin;
  dz += blockIdx.y * fout;
  for (int i = tid; i < N; i += NT) tw[i] = twg[i];
  // rows y1 = 2p, y2 = 2p + 1 as one complex sequence, scaled by V/N; four
  // items per thread have their loads in flight before any store
  const double* rz = rho + (size_t)z * N * N;
  constexpr int NI = NPAIR * N;
  for (int i0 = tid; i0 < NI; i0 += 4 * NT) {
    double va[4], vb[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * NT;
      va[u] = 0.0;
      vb[u] = 0.0;
      if (i < NI) {
        const int p = i / N, x = i - p * N;
        const int y1 = 2 * p, y2 = y1 + 1;
        va[u] = rz[y1 * N + x];
        if (y2 < N) vb[u] = rz[y2 * N + x];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * NT;
      if (i < NI) {
        const int p = i / N, x = i - p * N;
        A[p * LD + x] = make_double2(va[u] * scale, vb[u] * scale);
      }
    }
  }
  __syncthreads();
  // x pass A (-): pairs fastest
  for (int i = tid; i < N2 * NPAIR; i += NT) {
    const int n2 = i / NPAIR, p = i - n2 * NPAIR;
    double2 u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) u[n1] = A[p * LD + N2 * n1 + n2];
    pass_a<N1, N2, -1>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) B[p * PS1 + k1 * LS1 + n2] = u[k1];
  }
  __syncthreads();
  // x pass B: one pair per 16 lanes -> natural order in A
  for (int i = tid; i < 16 * NPAIR; i += NT) {
    const int p = i >> 4, k1 = i & 15;
    if (k1 >= N1) continue;
    double2 w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = B[p * PS1 + k1 * LS1 + n2];
    RDft<N2, -1>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) A[p * LD + k1 + N1 * k2] = w[k2];
  }
  __syncthreads();
  // two-for-one r2c unpack -> B [kx][y]
  for (int i = tid; i < NPAIR * NKX; i += NT) {
    const int p = i / NKX, k = i - p * NKX;
    const int y1 = 2 * p, y2 = y1 + 1;
    const double2 a = A[p * LD + k];
    const double2 b = cconj(A[p * LD + (k == 0 ? 0 : N - k)]);
    B[k * LD + y1] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
    if (y2 < N) B[k * LD + y2] = make_double2(0.5 * (a.y - b.y), -0.5 * (a.x - b.x));
  }
  __syncthreads();
  // y pass A (-): columns fastest
  for (int i = tid; i < N2 * NKX; i += NT) {
    const int n2 = i / NKX, c = i - n2 * NKX;
    double2 u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) u[n1] = B[c * LD + N2 * n1 + n2];
    pass_a<N1, N2, -1>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) A[c * PS1 + k1 * LS1 + n2] = u[k1];
  }
  __syncthreads();
  // y pass B -> dz[z][kx N + y]
  double2* out = dz + (size_t)z * ldl_d;
  for (int i = tid; i < 16 * NKX; i += NT) {
    const int c = i >> 4, k1 = i & 15;
    if (k1 >= N1) continue;
    double2 w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = A[c * PS1 + k1 * LS1 + n2];
    RDft<N2, -1>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) out[(size_t)c * N + k1 + N1 * k2] = w[k2];
  }
}

template <int N1, int N2, typename R>
__global__ void __launch_bounds__(512, 1)
k_rho2_bwd(const double2* __restrict__ dz, int ldl_d, const double2* __restrict__ twg,
           const double* __restrict__ vxc, R* __restrict__ vks, size_t fin, size_t fout) {
  typedef Rho2Cfg<N1, N2> CF;
  constexpr int N = CF::N, NKX = CF::NKX, NPAIR = CF::NPAIR, LD = CF::LD, LS1 = CF::LS1, PS1 = CF::PS1;
  constexpr int NT = CF::NT;
  static_assert(N1 <= 16, "pass B pads a pencil to 16 threads");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = (double2*)smem_raw;
  double2* A = tw + ((N + 1) & ~1);
  double2* B = A + CF::REGION;
  const int z = blockIdx.x, tid = threadIdx.x;
  dz += blockIdx.y * fin;
  vks += blockIdx.y * fout;
  for (int i = tid; i < N; i += NT) tw[i] = twg[i];
  // the plane's columns staged by cp.async: every 16-byte copy in flight
  // before any is waited for
  const double2* in = dz + (size_t)z * ldl_d;
  for (int i = tid; i < NKX * N; i += NT) {
    const int c = i / N, y = i - c * N;
    const unsigned d = (unsigned)__cvta_generic_to_shared(A + c * LD + y);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(in + i));
  }
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  // y pass A (+): columns fastest
  for (int i = tid; i < N2 * NKX; i += NT) {
    const int n2 = i / NKX, c = i - n2 * NKX;
    double2 u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) u[n1] = A[c * LD + N2 * n1 + n2];
    pass_a<N1, N2, +1>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) B[c * PS1 + k1 * LS1 + n2] = u[k1];
  }
  __syncthreads();
  // y pass B -> A [kx][y]
  for (int i = tid; i < 16 * NKX; i += NT) {
    const int c = i >> 4, k1 = i & 15;
    if (k1 >= N1) continue;
    double2 w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = B[c * PS1 + k1 * LS1 + n2];
    RDft<N2, +1>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) A[c * LD + k1 + N1 * k2] = w[k2];
  }
  __syncthreads();
  // c2r x pass A (+) on row pairs: pairs fastest, Hermitian extension in kx
  for (int i = tid; i < N2 * NPAIR; i += NT) {
    const int n2 = i / NPAIR, p = i - n2 * NPAIR;
    const int y1 = 2 * p, y2 = y1 + 1;
    double2 u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int k = N2 * n1 + n2;
      const double2 a = herm_x(A, LD, NKX, N, k, y1);
      double2 b = make_double2(0.0, 0.0);
      if (y2 < N) b = herm_x(A, LD, NKX, N, k, y2);
      u[n1] = make_double2(a.x - b.y, a.y + b.x);
    }
    pass_a<N1, N2, +1>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) B[p * PS1 + k1 * LS1 + n2] = u[k1];
  }
  __syncthreads();
  // x pass B -> vks = V + vxc (vxc may be null: vks = V)
  const double* vz = vxc ? vxc + (size_t)z * N * N : nullptr;
  R* oz = vks + (size_t)z * N * N;
  for (int i = tid; i < 16 * NPAIR; i += NT) {
    const int p = i >> 4, k1 = i & 15;
    if (k1 >= N1) continue;
    const int y1 = 2 * p, y2 = y1 + 1;
    double2 w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = B[p * PS1 + k1 * LS1 + n2];
    RDft<N2, +1>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int x = k1 + N1 * k2;
      oz[y1 * N + x] = (R)(w[k2].x + (vz ? vz[y1 * N + x] : 0.0));
      if (y2 < N) oz[y2 * N + x] = (R)(w[k2].y + (vz ? vz[y2 * N + x] : 0.0));
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <int N1, int N2>
static size_t rho2_smem() {
  typedef Rho2Cfg<N1, N2> CF;
  return (((size_t)CF::N + 1) / 2 * 2 + 2 * CF::REGION) * sizeof(double2);
}

#define OA_RHO2_DISPATCH(n, CALL)                                    \
  switch (n) {                                                       \
    case 12: return CALL(4, 3);                                      \
    case 20: return CALL(4, 5);                                      \
    case 24: return CALL(6, 4);                                      \
    case 36: return CALL(6, 6);                                      \
    case 40: return CALL(8, 5);                                      \
    case 64: return CALL(8, 8);                                      \
    case 96: return CALL(12, 8);                                     \
    case 108: return CALL(12, 9);                                    \
    default: break;                                                  \
  }

template <int N1, int N2>
static cudaError_t rho2_fwd_n(cudaStream_t s, int nz, const double* rho, double scale, const double2* tw, double2* dz,
                              int ldl_d, int nf, size_t fin, size_t fout) {
  const size_t sm = rho2_smem<N1, N2>();
  if (sm > (size_t)OA_MAX_SMEM) return cudaErrorNotSupported;
  cudaError_t e = oa_smem_limit(k_rho2_fwd<N1, N2>);
  if (e != cudaSuccess) return e;
  k_rho2_fwd<N1, N2><<<dim3(nz, nf), 512, sm, s>>>(rho, scale, tw, dz, ldl_d, fin, fout);
  return cudaGetLastError();
}

template <int N1, int N2>
static cudaError_t rho2_bwd_n(cudaStream_t s, int nz, const double2* dz, int ldl_d, const double2* tw,
                              const double* vxc, void* vks, int fp64, int nf, size_t fin, size_t fout) {
  const size_t sm = rho2_smem<N1, N2>();
  if (sm > (size_t)OA_MAX_SMEM) return cudaErrorNotSupported;
  cudaError_t e;
  if (fp64) {
    e = oa_smem_limit(k_rho2_bwd<N1, N2, double>);
    if (e != cudaSuccess) return e;
    k_rho2_bwd<N1, N2, double><<<dim3(nz, nf), 512, sm, s>>>(dz, ldl_d, tw, vxc, (double*)vks, fin, fout);
  } else {
    e = oa_smem_limit(k_rho2_bwd<N1, N2, float>);
    if (e != cudaSuccess) return e;
    k_rho2_bwd<N1, N2, float><<<dim3(nz, nf), 512, sm, s>>>(dz, ldl_d, tw, vxc, (float*)vks, fin, fout);
  }
  return cudaGetLastError();
}

// nx = ny = n; nf fields at strides fin / fout (elements of the input /
// output type); cudaErrorNotSupported when n has no two-pass kernel or the
// plane does not fit in shared memory (the caller then uses the
// runtime-plan kernels)
cudaError_t oa_rho2_fwd(cudaStream_t s, int n, int nz, const double* rho, double scale, const double2* tw,
                        double2* dz, int ldl_d, int nf, size_t fin, size_t fout) {
#define OA_CALL(A, B) rho2_fwd_n<A, B>(s, nz, rho, scale, tw, dz, ldl_d, nf, fin, fout)
  OA_RHO2_DISPATCH(n, OA_CALL)
#undef OA_CALL
  return cudaErrorNotSupported;
}

cudaError_t oa_rho2_bwd(cudaStream_t s, int n, int nz, const double2* dz, int ldl_d, const double2* tw,
                        const double* vxc, void* vks, int fp64, int nf, size_t fin, size_t fout) {
#define OA_CALL(A, B) rho2_bwd_n<A, B>(s, nz, dz, ldl_d, tw, vxc, vks, fp64, nf, fin, fout)
  OA_RHO2_DISPATCH(n, OA_CALL)
#undef OA_CALL
  return cudaErrorNotSupported;
}
