// State-pair plane kernels of the FP32 state FFT path: the density pass
// (psi(r) of two states per x transform, |psi|^2 summed into registers,
// psi(r) stored) and the V_KS pass that starts from that stored psi(r).
// They do the same work as k_plane2 MODE 0 and MODE 4 (oa_pencil.cu), with
// the two real states of a pair packed into one complex x transform
// (psi_a + i psi_b) instead of two rows of one state, so that
//   - one block moves one plane of two states per iteration with four block
//     barriers (y pass A, y pass B, x pass A, x pass B);
//   - each thread keeps a fixed set of x pass B outputs, so the density of a
//     plane sums in registers over all states of the block, and the inverse
//     twiddles of those outputs sit in registers;
//   - the y pass reads the z-line rows (copied to shared memory with
//     cp.async one pair ahead) through the per-column line runs instead of
//     a zero-filled scatter, and writes the result rows straight back;
//   - every shared-memory access pattern is free of bank conflicts: pass A
//     walks consecutive pencils (odd pencil strides), pass B walks one pencil
//     per 16 lanes (odd element strides).
// psi(r) is stored per pair, [pair][z][y][x] float2 (psi_a, psi_b).
//
// Reference work replaced (as k_plane2):
//   FFTcache::doStpFFTGtoR_Rchare (fftCache.C:1167) + the density part of
//     CP_State_RealSpacePlane::doFFT / doReduction (:349-363, 450-517)     -> k_pair_density
//   CP_State_RealSpacePlane::unpackVks (:530-597) + doStpFFTRtoG_Rchare
//     (fftCache.C:1252-1319)                                               -> k_pair_vks
#include "oa_rdft.cuh"
#include "oa_state_common.cuh"

// x pass B slots (16 lanes per row, N rows) per thread: the smallest count
// that gives a warp-multiple block of at most 640 threads
__host__ __device__ constexpr int pair_xb_waves(int n) {
  for (int w = 1; w <= 8; ++w)
    if ((16 * n) % w == 0 && ((16 * n) / w) % 32 == 0 && (16 * n) / w <= 640) return w;
  return 0;
}

template <int N1, int N2> struct PairCfg {
  static constexpr int N = N1 * N2;
  static constexpr int XBW = pair_xb_waves(N);
  static constexpr int NT = XBW ? 16 * N / XBW : 32;
  static constexpr int LDY = N | 1;           // P[st][kx][LDY]
  static constexpr int LS1 = N2 | 1;          // pass A -> B buffer [pencil][k1][n2]
  static constexpr int PS1 = (N1 * LS1) | 1;
  static constexpr int LS2 = N1;              // inverse B' -> A' buffer [row][m2][k1]
  static constexpr int PS2 = (N2 * N1) | 1;
  static constexpr int NJ = N2 / 2 + 1;       // m2 classes {j, N2 - j}
};

struct PairSmem {
  size_t tw, col, xh, rows, P, S, Sy, total;
  int lr;  // z-line row length in shared memory (float2, even)
};

static __device__ __forceinline__ void pp_cp16(void* sdst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc));
}
static __device__ __forceinline__ void pp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int K> static __device__ __forceinline__ void pp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(K));
}

// x-spectrum value at index k of row y (Hermitian extension of kx in [0, nkx))
template <int N, int LDY>
static __device__ __forceinline__ float2 pp_herm(const float2* P, int nkx, int k, int y) {
  float2 v = make_float2(0.f, 0.f);
  if (k <= N / 2) {
    if (k < nkx) v = P[k * LDY + y];
    if (k == 0 || 2 * k == N) v.y = 0.f;
  } else {
    const int kk = N - k;
    if (kk < nkx) { v = P[kk * LDY + y]; v.y = -v.y; }
  }
  return v;
}

// ---------------------------------------------------------------------------
// density pass: block (z, group) runs the pairs of its group through plane z,
// software-pipelined so that each block barrier separates two phases that
// mix the x work of pair q with the y work of pair q + 1:
//   phase a(q): x pass A (q)  [P -> Sx]   +  y pass A (q+1) [rows -> Sy]
//   phase b(q): x pass B (q)  [Sx -> psi(r), density]  +  y pass B (q+1) [Sy -> P]
// The z-line rows of pair q + 2 arrive by cp.async during both phases.
// ---------------------------------------------------------------------------
template <int N1, int N2, bool BAND>
__global__ void __launch_bounds__(PairCfg<N1, N2>::NT, 1)
k_pair_density(const float2* __restrict__ zbuf, int nstate, int nz, int ldl, int nlines,
               const int4* __restrict__ cols, int nkx, const double2* __restrict__ twg,
               const double* __restrict__ occ, double* __restrict__ rho_part, int ngroup,
               float2* __restrict__ psir, PairSmem L, double* __restrict__ qpart) {
  typedef PairCfg<N1, N2> CF;
  constexpr int N = CF::N, NT = CF::NT, XBW = CF::XBW;
  constexpr int LDY = CF::LDY, LS1 = CF::LS1, PS1 = CF::PS1;
  static_assert(N1 <= 16 && XBW > 0, "pair plane: unsupported factorisation");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw = (float2*)(smem_raw + L.tw);
  int4* col = (int4*)(smem_raw + L.col);
  int2* xh = (int2*)(smem_raw + L.xh);
  float2* rb = (float2*)(smem_raw + L.rows);
  float2* P = (float2*)(smem_raw + L.P);
  float2* Sx = (float2*)(smem_raw + L.S);
  float2* Sy = (float2*)(smem_raw + L.Sy);
  const int tid = threadIdx.x;
  const int z = blockIdx.x, g = blockIdx.y;
  const int npair = (nstate + 1) / 2;
  const int nper = (npair + ngroup - 1) / ngroup;
  const int qb = g * nper, qe = min(npair, qb + nper);
  const int lr = L.lr, nch = lr / 2;
  const int npc = 2 * nkx;
  int lp = 0;
  while ((1 << lp) < npc) ++lp;
  const int ya_slots = N2 << lp;
  constexpr int XA_ITEMS = N2 * N;
  for (int i = tid; i < N; i += NT) tw[i] = make_float2((float)twg[i].x, (float)twg[i].y);
  for (int i = tid; i < nkx; i += NT) col[i] = cols[i];
  // Hermitian table of x pass A, entry n2 * N1 + n1 for kx index k = N2 n1 + n2:
  // {P offset of the stored column (k or N - k), imaginary sign}: +1 stored
  // column, -1 its conjugate, 0 for the real DC / Nyquist terms; offset -1
  // where the spectrum is zero
  for (int i = tid; i < N; i += NT) {
    const int n2 = i / N1, n1 = i - n2 * N1, k = N2 * n1 + n2;
    int off = -1;
    float sg = 0.f;
    if (2 * k <= N) {
      if (k < nkx) { off = k * LDY; sg = (k == 0 || 2 * k == N) ? 0.f : 1.f; }
    } else if (N - k < nkx) {
      off = (N - k) * LDY; sg = -1.f;
    }
    xh[i] = make_int2(off, __float_as_int(sg));
  }
  float dens[XBW][N2];
#pragma unroll
  for (int j = 0; j < XBW; ++j)
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) dens[j][k2] = 0.f;
  auto prefetch = [&](int q, int buf) {
    for (int it = tid; it < 2 * nch; it += NT) {
      const int st = it >= nch ? 1 : 0, ch = it - st * nch;
      const int s = 2 * q + st;
      if (s < nstate) pp_cp16(rb + (size_t)(2 * buf + st) * lr + 2 * ch, zbuf + ((size_t)s * nz + z) * ldl + 2 * ch);
    }
    pp_commit();
  };
  // y pass A, slot sl of pair q (rows in buffer buf): pencil (state, column)
  // fastest in slots of 2^lp per n2; zero outside the column's run
  auto y_a = [&](int q, int buf, int sl) {
    const int n2 = sl >> lp, pc = sl & ((1 << lp) - 1);
    if (pc >= npc) return;
    const int st = pc >= nkx ? 1 : 0, cx = pc - st * nkx;
    const int4 cr = col[cx];
    const float2* r = rb + (size_t)(2 * buf + st) * lr + cr.x;
    const bool live = 2 * q + st < nstate;
    float2 u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      if (BAND && n1 >= N1 / 4 && n1 < 3 * N1 / 4) {  // |ky| >= N/4: outside every column run
        u[n1] = make_float2(0.f, 0.f);
        continue;
      }
      const int i = N2 * n1 + n2;
      const int ky = (2 * i <= N) ? i : i - N;
      const int l = ky - cr.y;
      u[n1] = (live && l >= 0 && l < cr.z) ? r[l] : make_float2(0.f, 0.f);
    }
    pass_a_band<N1, N2, -1, BAND>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) Sy[pc * PS1 + k1 * LS1 + n2] = u[k1];
  };
  // y pass B, slot it: one pencil per 16 lanes -> P[st][kx][y]
  auto y_b = [&](int it) {
    const int pc = it >> 4, k1 = it & 15;
    if (k1 >= N1) return;
    float2 w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = Sy[pc * PS1 + k1 * LS1 + n2];
    RDft<N2, -1>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) P[pc * LDY + k1 + N1 * k2] = w[k2];
  };
  // x pass A, item it: rows fastest (n2 warp-uniform); the pair packs as
  // psi_a + i psi_b, read through the Hermitian table
  auto x_a = [&](int it) {
    const int n2 = it / N, y = it - n2 * N;
    const int2* hx = xh + n2 * N1;
    float2 u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      if (BAND && n1 >= N1 / 4 && n1 < 3 * N1 / 4) {  // N/4 <= kx < 3N/4: zero spectrum
        u[n1] = make_float2(0.f, 0.f);
        continue;
      }
      const int2 t = hx[n1];
      float2 v = make_float2(0.f, 0.f);
      if (t.x >= 0) {
        const float2 a = P[t.x + y], b = P[t.x + nkx * LDY + y];
        const float sg = __int_as_float(t.y);
        v = make_float2(fmaf(-sg, b.y, a.x), fmaf(sg, a.y, b.x));
      }
      u[n1] = v;
    }
    pass_a_band<N1, N2, -1, BAND>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) Sx[y * PS1 + k1 * LS1 + n2] = u[k1];
  };
  if (qb < qe) {
    prefetch(qb, 0);
    if (qb + 1 < qe) { prefetch(qb + 1, 1); pp_wait<1>(); } else { pp_wait<0>(); }
    __syncthreads();
    for (int sl = tid; sl < ya_slots; sl += NT) y_a(qb, 0, sl);
    __syncthreads();
    for (int it = tid; it < 16 * npc; it += NT) y_b(it);
  }
  for (int q = qb; q < qe; ++q) {
    const bool nxt = q + 1 < qe;
    pp_wait<0>();
    __syncthreads();
    if (q + 2 < qe) prefetch(q + 2, (q - qb) & 1);
    // phase a: x pass A (q) + y pass A (q + 1)
    const int na = XA_ITEMS + (nxt ? ya_slots : 0);
    for (int it = tid; it < na; it += NT) {
      if (it < XA_ITEMS) x_a(it);
      else y_a(q + 1, (q + 1 - qb) & 1, it - XA_ITEMS);
    }
    __syncthreads();
    // phase b: x pass B (q), fixed slots per thread (density, psi(r)) + y pass B (q + 1)
    const float o0 = (float)occ[2 * q];
    const float o1 = 2 * q + 1 < nstate ? (float)occ[2 * q + 1] : 0.f;
    float2* pq = psir + ((size_t)q * nz + z) * N * N;
#pragma unroll
    for (int j = 0; j < XBW; ++j) {
      const int it = tid + NT * j;
      const int y = it >> 4, k1 = it & 15;
      if (k1 < N1) {
        float2 w[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) w[n2] = Sx[y * PS1 + k1 * LS1 + n2];
        RDft<N2, -1>::run(w);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          dens[j][k2] += o0 * w[k2].x * w[k2].x + o1 * w[k2].y * w[k2].y;
          __stcs(pq + y * N + k1 + N1 * k2, w[k2]);
        }
      }
    }
    if (nxt)
      for (int it = tid; it < 16 * npc; it += NT) y_b(it);
  }
  double* out = rho_part + ((size_t)g * nz + z) * N * N;
  double q = 0.0;  // this block's share of sum_r occ |psi(r)|^2 (the FP32 charge)
#pragma unroll
  for (int j = 0; j < XBW; ++j) {
    const int it = tid + NT * j;
    const int y = it >> 4, k1 = it & 15;
    if (k1 < N1) {
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        out[y * N + k1 + N1 * k2] = (double)dens[j][k2];
        q += (double)dens[j][k2];
      }
    }
  }
  if (qpart) {
    __shared__ double qsh[32];
    q = block_sum(q, qsh);
    if (tid == 0) qpart[(size_t)g * nz + z] = q;
  }
}

// ---------------------------------------------------------------------------
// V_KS pass from the stored psi(r): psi V_KS occ -> x FFT(+) with the r2c
// unpack of the pair -> y FFT(+) -> the z-line rows of both states.
// Software-pipelined as the density pass, the y work one pair behind:
//   phase a(q): x pass B' (q) [psi(r) -> S2]  +  y pass A' (q-1) [P -> Sy]
//   phase b(q): x pass A' (q) [S2 -> P]       +  y pass B' (q-1) [Sy -> rows]
// ---------------------------------------------------------------------------
template <int N1, int N2>
__global__ void __launch_bounds__(PairCfg<N1, N2>::NT, 1)
k_pair_vks(float2* __restrict__ zbuf, int nstate, int nz, int ldl, const int4* __restrict__ cols, int nkx,
           const double2* __restrict__ twg, const double* __restrict__ occ, const float* __restrict__ vks,
           int ngroup, const float2* __restrict__ psir, PairSmem L) {
  typedef PairCfg<N1, N2> CF;
  constexpr int N = CF::N, NT = CF::NT, XBW = CF::XBW, NJ = CF::NJ;
  // L2 prefetch of a psi(r) pair plane (N^2 float2) in PF_PARTS pieces of
  // PF_BYTES (multiples of 16 bytes)
  constexpr int PF_PARTS = (N * N * 8) % (16 * 8) == 0 ? 8 : ((N * N * 8) % (16 * 4) == 0 ? 4 : 1);
  constexpr int PF_BYTES = N * N * 8 / PF_PARTS;
  static_assert(PF_BYTES % 16 == 0, "psi(r) plane prefetch needs 16-byte pieces");
  constexpr int LDY = CF::LDY, LS1 = CF::LS1, PS1 = CF::PS1, LS2 = CF::LS2, PS2 = CF::PS2;
  static_assert(N1 <= 16 && XBW > 0 && NT % 16 == 0, "pair plane: unsupported factorisation");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw = (float2*)(smem_raw + L.tw);
  int4* col = (int4*)(smem_raw + L.col);
  float2* P = (float2*)(smem_raw + L.P);
  float2* S2 = (float2*)(smem_raw + L.S);
  float2* Sy = (float2*)(smem_raw + L.Sy);
  const int tid = threadIdx.x;
  const int z = blockIdx.x, g = blockIdx.y;
  const int npair = (nstate + 1) / 2;
  const int nper = (npair + ngroup - 1) / ngroup;
  const int qb = g * nper, qe = min(npair, qb + nper);
  const int npc = 2 * nkx;
  int lp = 0;
  while ((1 << lp) < npc) ++lp;
  const int ya_slots = N2 << lp;
  const int kf = tid & 15;  // this thread's k1 in x pass B' (NT is a multiple of 16)
  for (int i = tid; i < N; i += NT) tw[i] = make_float2((float)twg[i].x, (float)twg[i].y);
  for (int i = tid; i < nkx; i += NT) col[i] = cols[i];
  __syncthreads();
  float2 tk[N2];
  const float* vz = vks + (size_t)z * N * N;
  if (kf < N1) {
#pragma unroll
    for (int m2 = 0; m2 < N2; ++m2) tk[m2] = tw_rt<+1>(tw, kf * m2);
  }
  for (int q = qb; q <= qe; ++q) {
    const bool cur = q < qe, prev = q > qb;
    if (q + 1 < qe && tid < PF_PARTS) {
      // the next pair's psi(r) plane heads for L2 while this pair computes
      const char* nxt = (const char*)(psir + ((size_t)(q + 1) * nz + z) * N * N) + (size_t)tid * PF_BYTES;
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(nxt), "r"(PF_BYTES) : "memory");
    }
    __syncthreads();
    // phase a: x pass B' (q) (inverse, first half: DFT_N2(+) over k2,
    // twiddle -> S2[y][m2][k1]) + y pass A' (q - 1)
    if (cur && kf < N1) {
      const bool has1 = 2 * q + 1 < nstate;
      const float o0 = (float)occ[2 * q];
      const float o1 = has1 ? (float)occ[2 * q + 1] : 0.f;
      const float2* pq = psir + ((size_t)q * nz + z) * N * N;
#pragma unroll
      for (int j = 0; j < XBW; ++j) {
        const int y = (tid + NT * j) >> 4;
        float2 w[N2];
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          const float2 p = __ldcs(pq + y * N + kf + N1 * k2);
          const float v = __ldg(vz + y * N + kf + N1 * k2);
          w[k2] = make_float2(p.x * v * o0, p.y * v * o1);
        }
        RDft<N2, +1>::run(w);
        S2[y * PS2 + kf] = w[0];
#pragma unroll
        for (int m2 = 1; m2 < N2; ++m2) S2[y * PS2 + m2 * LS2 + kf] = cmul(w[m2], tk[m2]);
      }
    }
    if (prev) {
      for (int sl = tid; sl < ya_slots; sl += NT) {
        const int n2 = sl >> lp, pc = sl & ((1 << lp) - 1);
        if (pc >= npc) continue;
        float2 u[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) u[n1] = P[pc * LDY + N2 * n1 + n2];
        pass_a<N1, N2, +1>(u, n2, tw);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) Sy[pc * PS1 + k1 * LS1 + n2] = u[k1];
      }
    }
    __syncthreads();
    // phase b: x pass A' (q) (inverse, second half, on the classes
    // {j, N2 - j}; two-for-one unpack of the pair into P[st][kx][y] for
    // kx < nkx) + y pass B' (q - 1) -> the column's z-line run of each state
    if (cur) {
      for (int it = tid; it < NJ * N; it += NT) {
        const int jj = it / N, y = it - jj * N;
        const int ma = jj, mb = (N2 - jj) % N2;
        const bool two = ma != mb;
        float2 za[N1], zb[N1];
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) za[k1] = S2[y * PS2 + ma * LS2 + k1];
        RDft<N1, +1>::run(za);
        if (two) {
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) zb[k1] = S2[y * PS2 + mb * LS2 + k1];
          RDft<N1, +1>::run(zb);
        }
        auto put = [&](int K, float2 a, float2 bp) {
          const float2 b = make_float2(bp.x, -bp.y);
          P[K * LDY + y] = make_float2((a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f);
          P[(nkx + K) * LDY + y] = make_float2((a.y - b.y) * 0.5f, -(a.x - b.x) * 0.5f);
        };
#pragma unroll
        for (int m1 = 0; m1 < N1; ++m1) {
          const int K = ma + N2 * m1;
          if (K < nkx) {
            const float2 pa = (jj == 0) ? za[(N1 - m1) % N1] : (two ? zb[N1 - 1 - m1] : za[N1 - 1 - m1]);
            put(K, za[m1], pa);
          }
          if (two) {
            const int Kb = mb + N2 * m1;
            if (Kb < nkx) put(Kb, zb[m1], za[N1 - 1 - m1]);
          }
        }
      }
    }
    if (prev) {
      const int qp = q - 1;
      const bool has1p = 2 * qp + 1 < nstate;
      for (int it = tid; it < 16 * npc; it += NT) {
        const int pc = it >> 4, k1 = it & 15;
        if (k1 >= N1) continue;
        const int st = pc >= nkx ? 1 : 0, cx = pc - st * nkx;
        if (st == 1 && !has1p) continue;
        float2 w[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) w[n2] = Sy[pc * PS1 + k1 * LS1 + n2];
        RDft<N2, +1>::run(w);
        const int4 cr = col[cx];
        float2* row = zbuf + ((size_t)(2 * qp + st) * nz + z) * ldl + cr.x;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          const int i = k1 + N1 * k2;
          const int ky = (2 * i <= N) ? i : i - N;
          const int l = ky - cr.y;
          if (l >= 0 && l < cr.z) row[l] = w[k2];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <int N1, int N2>
static PairSmem pair_layout(int nkx, int nlines, int mode) {
  typedef PairCfg<N1, N2> CF;
  PairSmem L;
  size_t o = 0;
  L.lr = (nlines + 1) & ~1;
  L.tw = o; o += align_up((size_t)CF::N * sizeof(float2), 16);
  L.col = o; o += align_up((size_t)nkx * sizeof(int4), 16);
  L.xh = o; o += align_up((size_t)CF::N * sizeof(int2), 16);
  L.rows = o; o += mode == 0 ? (size_t)4 * L.lr * sizeof(float2) : 0;
  L.P = o; o += align_up((size_t)2 * nkx * CF::LDY * sizeof(float2), 16);
  // x buffer: Sx [N][PS1] (density) or S2 [N][PS2] (V_KS); y buffer Sy [2 nkx][PS1]
  const size_t sx = (size_t)CF::N * (mode == 0 ? CF::PS1 : CF::PS2);
  L.S = o; o += align_up(sx * sizeof(float2), 16);
  L.Sy = o; o += align_up((size_t)2 * nkx * CF::PS1 * sizeof(float2), 16);
  L.total = o;
  return L;
}

template <int N1, int N2>
static cudaError_t pair_launch(int mode, cudaStream_t st, void* zbuf, int nstate, int nz, int ldl, int nlines,
                               const int* cols, int nkx, const double2* tw, const double* occ, const void* vks,
                               double* rho_part, int ngroup, void* psir, int kymax, double* qpart) {
  typedef PairCfg<N1, N2> CF;
  if (CF::XBW == 0 || N1 > 16 || 2 * nkx > CF::N + 2 || (ldl & 1)) return cudaErrorNotSupported;
  const PairSmem L = pair_layout<N1, N2>(nkx, nlines, mode);
  if (L.total > (size_t)OA_MAX_SMEM) return cudaErrorNotSupported;
  const dim3 grid(nz, ngroup);
  cudaError_t e;
  if (mode == 0) {
    // the forward DFT_N1 inputs in [N1/4, 3 N1/4) are zero when the sphere's
    // kx columns and ky runs stay inside |k| < N/4
    constexpr int N = CF::N;
    const bool band = (N1 % 4 == 0) && 4 * nkx <= N && 4 * (kymax + 1) <= N;
    auto launch = [&](auto kern) -> cudaError_t {
      cudaError_t e2 = oa_smem_limit(kern);
      if (e2 != cudaSuccess) return e2;
      kern<<<grid, CF::NT, L.total, st>>>((const float2*)zbuf, nstate, nz, ldl, nlines, (const int4*)cols, nkx, tw,
                                          occ, rho_part, ngroup, (float2*)psir, L, qpart);
      return cudaGetLastError();
    };
    if constexpr (N1 % 4 == 0) {
      if (band) return launch(k_pair_density<N1, N2, true>);
    }
    return launch(k_pair_density<N1, N2, false>);
  } else {
    e = oa_smem_limit(k_pair_vks<N1, N2>);
    if (e != cudaSuccess) return e;
    k_pair_vks<N1, N2><<<grid, CF::NT, L.total, st>>>((float2*)zbuf, nstate, nz, ldl, (const int4*)cols, nkx, tw,
                                                      occ, (const float*)vks, ngroup, (const float2*)psir, L);
  }
  return cudaGetLastError();
}

#define OA_PAIR_DISPATCH(n, CALL)                                    \
  switch (n) {                                                       \
    case 12: return CALL(4, 3);                                      \
    case 20: return CALL(4, 5);                                      \
    case 24: return CALL(6, 4);                                      \
    case 36: return CALL(6, 6);                                      \
    case 40: return CALL(8, 5);                                      \
    case 64: return CALL(8, 8);                                      \
    case 96: return CALL(12, 8);                                     \
    case 108: return CALL(12, 9);                                    \
    case 160: return CALL(16, 10);                                   \
    default: break;                                                  \
  }

// mode 0: density pass (rho_part[group][z][y][x], psi(r) pairs stored;
// qpart, when not null: [group][z] block sums of sum_r occ |psi(r)|^2);
// mode 4: V_KS pass from those psi(r) pairs.  nx = ny = n; cols = per kx
// column {first line, ky of the first line, line count, 0}; kymax = the
// largest |ky| of the lines.  Returns
// cudaErrorNotSupported when n or the shared memory has no pair kernel.
cudaError_t oa_pair_plane(int mode, cudaStream_t st, int n, void* zbuf, int nstate, int nz, int ldl, int nlines,
                          const int* cols, int nkx, const double2* tw, const double* occ, const void* vks,
                          double* rho_part, int ngroup, void* psir, int kymax, double* qpart) {
#define OA_CALL(A, B)                                                                                          \
  pair_launch<A, B>(mode, st, zbuf, nstate, nz, ldl, nlines, cols, nkx, tw, occ, vks, rho_part, ngroup, psir, kymax, \
                    qpart)
  OA_PAIR_DISPATCH(n, OA_CALL)
#undef OA_CALL
  return cudaErrorNotSupported;
}

// whether the pair kernels cover length n with these sizes (both modes)
int oa_pair_plane_supported(int n, int nkx, int nlines, int ldl) {
#define OA_CALL(A, B)                                                                                     \
  (PairCfg<A, B>::XBW > 0 && 2 * nkx <= PairCfg<A, B>::N + 2 && !(ldl & 1) &&                             \
   pair_layout<A, B>(nkx, nlines, 0).total <= (size_t)OA_MAX_SMEM &&                                      \
   pair_layout<A, B>(nkx, nlines, 4).total <= (size_t)OA_MAX_SMEM)                                        \
      ? 1 : 0
  OA_PAIR_DISPATCH(n, OA_CALL)
#undef OA_CALL
  return 0;
}
