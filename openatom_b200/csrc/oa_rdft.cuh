// Register-resident DFTs with compile-time twiddles, and the two-pass
// ("four-step") factorisation of a pencil of length N = N1 * N2 that the
// pencil kernels (oa_pencil.cu) are built from.
//
// A length-N transform y_k = sum_n x_n exp(SIGN 2 pi i n k / N) is done as
//   pass A (one thread per n2 in [0, N2)):
//     u[n1] = x[N2 n1 + n2];  u = DFT_N1(u);  u[k1] *= exp(SIGN 2 pi i n2 k1 / N)
//   pass B (one thread per k1 in [0, N1)):
//     w[n2] = u_{n2}[k1];     w = DFT_N2(w);  y[k1 + N1 k2] = w[k2]
// with the u's handed from pass A to pass B through shared memory.  The
// small DFTs run entirely in registers: they are Cooley-Tukey recursions on
// radices 4, 2, 3, 5 whose inner twiddles are compile-time constants, so
// each pencil makes two shared-memory round trips instead of one per radix
// stage.  The compile-time cosines and sines are Taylor series evaluated by
// the compiler (ce_sin / ce_cos below), accurate to double rounding.
#pragma once
#include <type_traits>
#include "oa_fft.cuh"

#define OA_PI_D 3.14159265358979323846264338327950288

// sin of x in [-pi/2, pi/2] by its Taylor series (terms to x^41 / 41!).
__host__ __device__ constexpr double ce_sin_core(double x) {
  double term = x, sum = x;
  const double x2 = x * x;
  for (int k = 1; k < 21; ++k) {
    term *= -x2 / (double)((2 * k) * (2 * k + 1));
    sum += term;
  }
  return sum;
}
// sin(x) for x in [-2 pi, 2 pi]: reduce to [-pi, pi], then with
// sin(pi - x) = sin(x) to [-pi/2, pi/2].
__host__ __device__ constexpr double ce_sin(double x) {
  if (x > OA_PI_D) x -= 2.0 * OA_PI_D;
  if (x < -OA_PI_D) x += 2.0 * OA_PI_D;
  if (x > 0.5 * OA_PI_D) x = OA_PI_D - x;
  if (x < -0.5 * OA_PI_D) x = -OA_PI_D - x;
  return ce_sin_core(x);
}
__host__ __device__ constexpr double ce_cos(double x) { return ce_sin(x + 0.5 * OA_PI_D); }

// compile-time loop: f(integral_constant<int, i>) for i in [B, E)
template <int B, int E, typename F>
OA_HD void sfor(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}

// a * exp(SIGN 2 pi i M / N), with the multiples of pi/2 done exactly
template <int N, int SIGN, int M, typename C>
OA_HD C twc(C a) {
  constexpr int m = ((M % N) + N) % N;
  if constexpr (m == 0) {
    return a;
  } else if constexpr (4 * m == N) {
    return cmul_si<SIGN>(a);
  } else if constexpr (2 * m == N) {
    a.x = -a.x;
    a.y = -a.y;
    return a;
  } else if constexpr (4 * m == 3 * N) {
    return cmul_si<-SIGN>(a);
  } else {
    constexpr double ang = (double)SIGN * 2.0 * OA_PI_D * (double)m / (double)N;
    constexpr double c = ce_cos(ang);
    constexpr double s = ce_sin(ang);
    return cmul(a, cmk<C>(c, s));
  }
}

// In-register DFT of length N: v[k] <- sum_n v[n] exp(SIGN 2 pi i n k / N)
template <int N, int SIGN> struct RDft {
  static constexpr int P = (N % 4 == 0) ? 4 : (N % 2 == 0) ? 2 : (N % 3 == 0) ? 3 : 5;
  static constexpr int Q = N / P;
  static_assert(P * Q == N, "RDft: N must factor into 2, 3, 4, 5");
  template <typename C>
  OA_HD static void run(C* v) {
    // n = Q p + q, k = kp + P kq
    C t[N];
    sfor<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      C u[P];
#pragma unroll
      for (int p = 0; p < P; ++p) u[p] = v[Q * p + q];
      RDft<P, SIGN>::run(u);
      sfor<0, P>([&](auto kc) {
        constexpr int kp = decltype(kc)::value;
        t[kp * Q + q] = twc<N, SIGN, q * kp>(u[kp]);
      });
    });
#pragma unroll
    for (int kp = 0; kp < P; ++kp) {
      RDft<Q, SIGN>::run(t + kp * Q);
#pragma unroll
      for (int kq = 0; kq < Q; ++kq) v[kp + P * kq] = t[kp * Q + kq];
    }
  }
};
template <int SIGN> struct RDft<1, SIGN> {
  template <typename C> OA_HD static void run(C*) {}
};
template <int SIGN> struct RDft<2, SIGN> {
  template <typename C> OA_HD static void run(C* v) { dft2<SIGN>(v); }
};
template <int SIGN> struct RDft<3, SIGN> {
  template <typename C> OA_HD static void run(C* v) { dft3<SIGN>(v); }
};
template <int SIGN> struct RDft<4, SIGN> {
  template <typename C> OA_HD static void run(C* v) { dft4<SIGN>(v); }
};
template <int SIGN> struct RDft<5, SIGN> {
  template <typename C> OA_HD static void run(C* v) { dft5<SIGN>(v); }
};

// Two-pass factorisations N = N1 * N2 of the pencil lengths with kernels.
template <int N> struct Split { static constexpr bool ok = false; static constexpr int n1 = 1, n2 = 1; };
#define OA_SPLIT(NN, A, B)                                                   \
  template <> struct Split<NN> {                                             \
    static constexpr bool ok = true;                                         \
    static constexpr int n1 = A, n2 = B;                                     \
  };
OA_SPLIT(12, 4, 3)
OA_SPLIT(20, 4, 5)
OA_SPLIT(24, 6, 4)
OA_SPLIT(36, 6, 6)
OA_SPLIT(40, 8, 5)
OA_SPLIT(64, 8, 8)
OA_SPLIT(96, 12, 8)
OA_SPLIT(108, 12, 9)
OA_SPLIT(160, 16, 10)
#undef OA_SPLIT

// odd leading dimension (complex elements) so that strided accesses by
// consecutive threads fall into distinct shared-memory banks
__host__ __device__ constexpr int odd_ld(int n) { return n | 1; }

// Runtime twiddle exp(SIGN 2 pi i j / N) from the table tw[j] = exp(-2 pi i j / N)
template <int SIGN, typename C>
OA_HD C tw_rt(const C* tw, int j) {
  C t = tw[j];
  if (SIGN > 0) t.y = -t.y;
  return t;
}

// Pass A on one item: u holds x[N2 n1 + n2] for n1 in [0, N1) on entry; on
// exit the twiddled DFT_N1 outputs, ready to be stored at k1.
template <int N1, int N2, int SIGN, typename C>
OA_HD void pass_a(C* u, int n2, const C* tw) {
  RDft<N1, SIGN>::run(u);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1) u[k1] = cmul(u[k1], tw_rt<SIGN>(tw, n2 * k1));
}

// DFT of length N (N % 4 == 0) whose inputs n in [N/4, 3N/4) are zero (the
// sphere of a state occupies |k| < N/4 of its density-sized grid).  Same
// Cooley-Tukey split as RDft<N> (P = 4, Q = N/4, n = Q p + q): every DFT_4
// over p has inputs at p = 0 and p = 3 only, X[kp] = x0 + x3 W^{3 kp}.
template <int N, int SIGN> struct RDftBand {
  static_assert(N % 4 == 0, "RDftBand: N must be a multiple of 4");
  static constexpr int Q = N / 4;
  template <typename C>
  OA_HD static void run(C* v) {
    C t[N];
    sfor<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const C a = v[q], b = v[3 * Q + q];
      C u[4];
      u[0] = cadd(a, b);
      u[1] = cadd(a, cmul_si<-SIGN>(b));
      u[2] = csub(a, b);
      u[3] = cadd(a, cmul_si<SIGN>(b));
      sfor<0, 4>([&](auto kc) {
        constexpr int kp = decltype(kc)::value;
        t[kp * Q + q] = twc<N, SIGN, q * kp>(u[kp]);
      });
    });
#pragma unroll
    for (int kp = 0; kp < 4; ++kp) {
      RDft<Q, SIGN>::run(t + kp * Q);
#pragma unroll
      for (int kq = 0; kq < Q; ++kq) v[kp + 4 * kq] = t[kp * Q + kq];
    }
  }
};

// pass A with the middle band of inputs zero (BAND) or general
template <int N1, int N2, int SIGN, bool BAND, typename C>
OA_HD void pass_a_band(C* u, int n2, const C* tw) {
  if constexpr (BAND) RDftBand<N1, SIGN>::run(u);
  else RDft<N1, SIGN>::run(u);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1) u[k1] = cmul(u[k1], tw_rt<SIGN>(tw, n2 * k1));
}

#ifdef __CUDACC__
// In-place transform of nb lines a[line][n] (row stride ld) for the lengths
// with a compile-time factorisation N = N1 N2, N1 <= 16: pass A (lines
// fastest) into b [line][k1][n2] (row stride ZLd::PS), pass B back to
// natural order in a.  tw: the length-N table exp(-2 pi i k / N) in shared
// memory.  Used by the density z pass and the EES local grid transforms.
template <int N1, int N2> struct ZLd {
  static constexpr int LS = N2 | 1;
  static constexpr int PS = (N1 * LS) | 1;
};
template <int N1, int N2, int SIGN>
__device__ void zfft2(double2* a, double2* b, int ld, int nb, const double2* tw) {
  typedef ZLd<N1, N2> L;
  for (int i = threadIdx.x; i < N2 * nb; i += blockDim.x) {
    const int n2 = i / nb, lb = i - n2 * nb;
    double2 u[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) u[n1] = a[lb * ld + N2 * n1 + n2];
    pass_a<N1, N2, SIGN>(u, n2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) b[lb * L::PS + k1 * L::LS + n2] = u[k1];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 16 * nb; i += blockDim.x) {
    const int lb = i >> 4, k1 = i & 15;
    if (k1 >= N1) continue;
    double2 w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = b[lb * L::PS + k1 * L::LS + n2];
    RDft<N2, SIGN>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) a[lb * ld + k1 + N1 * k2] = w[k2];
  }
  __syncthreads();
}
#endif
