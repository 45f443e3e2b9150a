// Shared-memory batched mixed-radix FFT for the small pencil lengths of the
// CP state and density grids (radices 2, 3, 4, 5; n <= OA_FFT_MAXN).
//
// Algorithm: Stockham autosort (out-of-place per stage, no bit reversal),
// one radix-R butterfly per work item, all threads of the block striding
// over (sequence, butterfly) pairs.  For a stage with radix R after radices
// whose product is Ns:
//   v[r] = in[j + r n/R] * w^(r (j mod Ns)),  w = exp(sign 2 pi i / (Ns R))
//   v    = DFT_R(v)
//   out[(j / Ns) Ns R + (j mod Ns) + r Ns] = v[r]
// Twiddles come from a per-length table tw[k] = exp(-2 pi i k / n) in shared
// memory; sign > 0 uses its conjugate.  This replaces the reference's FFTW2
// plans (src_charm_driver/fft_slab_ctrl/fftCache.C:100-160): FFTW_FORWARD is
// sign -1, FFTW_BACKWARD sign +1, both unnormalised.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define OA_HD __host__ __device__ __forceinline__
#define OA_FFT_MAXST 8
#define OA_FFT_MAXN 512

struct OaFftPlan {
  int n;
  int nst;
  int rad[OA_FFT_MAXST];
};

template <typename R> struct OaCplx;
template <> struct OaCplx<double> { typedef double2 T; };
template <> struct OaCplx<float> { typedef float2 T; };

template <typename C> OA_HD C cmk(double x, double y);
template <> OA_HD double2 cmk<double2>(double x, double y) { return make_double2(x, y); }
template <> OA_HD float2 cmk<float2>(double x, double y) { return make_float2((float)x, (float)y); }

template <typename C> OA_HD C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> OA_HD C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> OA_HD C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename C> OA_HD C cconj(C a) { a.y = -a.y; return a; }
// multiply by sign*i
template <int SIGN, typename C> OA_HD C cmul_si(C a) {
  C r;
  if (SIGN < 0) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
  return r;
}
template <typename C> OA_HD C cscale(C a, decltype(a.x) s) { a.x *= s; a.y *= s; return a; }

// ---------------------------------------------------------------------------
// small DFTs: y_k = sum_r v_r exp(SIGN 2 pi i r k / R)
// ---------------------------------------------------------------------------
template <int SIGN, typename C> OA_HD void dft2(C* v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b); v[1] = csub(a, b);
}
template <int SIGN, typename C> OA_HD void dft4(C* v) {
  C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  C t2 = cadd(v[1], v[3]), t3 = cmul_si<SIGN>(csub(v[1], v[3]));
  v[0] = cadd(t0, t2); v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3); v[3] = csub(t1, t3);
}
template <int SIGN, typename C> OA_HD void dft3(C* v) {
  typedef decltype(v[0].x) R;
  const R c1 = (R)-0.5;
  const R s1 = (R)0.86602540378443864676372317075294;  // sin(2 pi / 3)
  C t = cadd(v[1], v[2]);
  C u = cmul_si<SIGN>(cscale(csub(v[1], v[2]), s1));
  C m = cadd(v[0], cscale(t, c1));
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, u);
  v[2] = csub(m, u);
}
template <int SIGN, typename C> OA_HD void dft5(C* v) {
  typedef decltype(v[0].x) R;
  const R c1 = (R)0.30901699437494742410229341718282;   // cos(2 pi / 5)
  const R c2 = (R)-0.80901699437494742410229341718282;  // cos(4 pi / 5)
  const R s1 = (R)0.95105651629515357211643933337938;   // sin(2 pi / 5)
  const R s2 = (R)0.58778525229247312916870595463907;   // sin(4 pi / 5)
  C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  C m1 = cadd(v[0], cadd(cscale(a1, c1), cscale(a2, c2)));
  C m2 = cadd(v[0], cadd(cscale(a1, c2), cscale(a2, c1)));
  C n1 = cmul_si<SIGN>(cadd(cscale(b1, s1), cscale(b2, s2)));
  C n2 = cmul_si<SIGN>(csub(cscale(b1, s2), cscale(b2, s1)));
  v[0] = cadd(v[0], cadd(a1, a2));
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

template <int RAD, int SIGN, typename C>
__device__ __forceinline__ void stockham_stage(const C* __restrict__ src, int ld_src,
                                               C* __restrict__ dst, int ld_dst,
                                               int n, int Ns, int nb, const C* __restrict__ tw,
                                               int t0, int tstep) {
  const int m = n / RAD;
  const int tstride = n / (Ns * RAD);
  const int total = nb * m;
  for (int w = t0; w < total; w += tstep) {
    const int s = w / m;
    const int j = w - s * m;
    const int k = j % Ns;
    const C* in = src + (size_t)s * ld_src;
    C* out = dst + (size_t)s * ld_dst;
    C v[RAD];
#pragma unroll
    for (int r = 0; r < RAD; ++r) v[r] = in[j + r * m];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < RAD; ++r) {
        C t = tw[k * r * tstride];
        if (SIGN > 0) t = cconj(t);
        v[r] = cmul(v[r], t);
      }
    }
    if (RAD == 2) dft2<SIGN>(v);
    else if (RAD == 3) dft3<SIGN>(v);
    else if (RAD == 4) dft4<SIGN>(v);
    else dft5<SIGN>(v);
    const int d = (j / Ns) * Ns * RAD + k;
#pragma unroll
    for (int r = 0; r < RAD; ++r) out[d + r * Ns] = v[r];
  }
}

template <int SIGN, typename C>
__device__ __forceinline__ void fft_stage_dispatch(int rad, const C* src, int lds, C* dst, int ldd,
                                                   int n, int Ns, int nb, const C* tw, int t0, int tstep) {
  switch (rad) {
    case 2: stockham_stage<2, SIGN>(src, lds, dst, ldd, n, Ns, nb, tw, t0, tstep); break;
    case 3: stockham_stage<3, SIGN>(src, lds, dst, ldd, n, Ns, nb, tw, t0, tstep); break;
    case 4: stockham_stage<4, SIGN>(src, lds, dst, ldd, n, Ns, nb, tw, t0, tstep); break;
    default: stockham_stage<5, SIGN>(src, lds, dst, ldd, n, Ns, nb, tw, t0, tstep); break;
  }
}

// Ping-pong batch FFT: data starts in a (sequence stride ld), b is scratch of
// the same shape.  Returns the buffer holding the result.  Ends with a
// __syncthreads(); the caller must __syncthreads() before it if a was just
// written.
template <int SIGN, typename C>
__device__ C* fft_pingpong(C* a, C* b, int ld, int nb, const OaFftPlan& p, const C* tw) {
  int Ns = 1;
  C* src = a;
  C* dst = b;
  for (int st = 0; st < p.nst; ++st) {
    fft_stage_dispatch<SIGN>(p.rad[st], src, ld, dst, ld, p.n, Ns, nb, tw, threadIdx.x, blockDim.x);
    __syncthreads();
    Ns *= p.rad[st];
    C* t = src; src = dst; dst = t;
  }
  return src;
}

// Warp-cooperative variants: one warp owns the nb sequences, stages are
// separated by __syncwarp() only.
template <int SIGN, typename C>
__device__ C* warp_fft_pingpong(C* a, C* b, int ld, int nb, const OaFftPlan& p, const C* tw, int lane) {
  int Ns = 1;
  C* src = a;
  C* dst = b;
  for (int st = 0; st < p.nst; ++st) {
    fft_stage_dispatch<SIGN>(p.rad[st], src, ld, dst, ld, p.n, Ns, nb, tw, lane, 32);
    __syncwarp();
    Ns *= p.rad[st];
    C* t = src; src = dst; dst = t;
  }
  return src;
}

template <int SIGN, typename C>
__device__ void warp_fft_inout(const C* in, int ld_in, C* out, int ld_out, C* w1, C* w2, int ldw,
                               int nb, const OaFftPlan& p, const C* tw, int lane) {
  int Ns = 1;
  const C* src = in;
  int lds = ld_in;
  C* bufs[2] = {w1, w2};
  for (int st = 0; st < p.nst; ++st) {
    const bool last = (st == p.nst - 1);
    C* dst = last ? out : bufs[st & 1];
    const int ldd = last ? ld_out : ldw;
    fft_stage_dispatch<SIGN>(p.rad[st], src, lds, dst, ldd, p.n, Ns, nb, tw, lane, 32);
    __syncwarp();
    Ns *= p.rad[st];
    src = dst;
    lds = ldd;
  }
}

// FFT from `in` (stride ld_in) to `out` (stride ld_out) with two scratch
// buffers w1, w2 (stride ldw).  in may equal out when nst >= 2.
template <int SIGN, typename C>
__device__ void fft_inout(const C* in, int ld_in, C* out, int ld_out, C* w1, C* w2, int ldw,
                          int nb, const OaFftPlan& p, const C* tw) {
  int Ns = 1;
  const C* src = in;
  int lds = ld_in;
  C* bufs[2] = {w1, w2};
  for (int st = 0; st < p.nst; ++st) {
    const bool last = (st == p.nst - 1);
    C* dst = last ? out : bufs[st & 1];
    const int ldd = last ? ld_out : ldw;
    fft_stage_dispatch<SIGN>(p.rad[st], src, lds, dst, ldd, p.n, Ns, nb, tw, threadIdx.x, blockDim.x);
    __syncthreads();
    Ns *= p.rad[st];
    src = dst;
    lds = ldd;
  }
}

template <typename C>
__device__ __forceinline__ void load_twiddles(C* dst, const double2* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = cmk<C>(src[i].x, src[i].y);
}
