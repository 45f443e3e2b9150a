// C ABI of liboa_gpu: context setup and the per-chare-work entry points.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <vector>
#include <cuda_bf16.h>
#include "oa_internal.h"

// launchers from the other translation units
size_t oa_plane_smem_bytes(int precision, int nx, int ny, int nkx);
int oa_plane_blocks_per_sm(int precision);
size_t oa_rho_plane_smem_bytes(int nx, int ny, int nkx, int npair, int ychunk);
int oa_rho_xc_nblk();
size_t oa_rho_gga_red_off(const oa_ctx* c);
int oa_rho_z_nblk(const oa_ctx* c);
cudaError_t oa_launch_pc_fwd(cudaStream_t s, const double* A, const double* B, int n, long K, long kx0_cols,
                             double w_kx0, double alpha, double* part, int nkb, double* C);
cudaError_t oa_launch_pc_bwd(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                             const double* M2, const double* X2, double a2, int n, long ncol, long kx0_cols,
                             double* out);
cudaError_t oa_launch_small_gemm(cudaStream_t s, const double* A, const double* B, int n, double alpha, double* C);
int oa_ns_grid(int n, int device);
int oa_pencil_supported(int n);
int oa_ns_cluster_size(int n);
cudaError_t oa_launch_ortho_ns(cudaStream_t s, const double* S, int n, double bscale, double tol, int max_iter,
                               double* work, double* T, int* status, double* errv, int grid);
int oa_integrate_nblk(int ng, int nstate);
int oa_pair_plane_supported(int n, int nkx, int nlines, int ldl);
cudaError_t oa_launch_integrate(cudaStream_t s, const double2* F, double2* V, double2* P, const double2* P_in,
                                const int* sel, const double* cmass, int ng, int nstate, int r0, int r1, int iend,
                                double dt, int complete_prev, double* kepart, int nblk);
cudaError_t oa_launch_sync_redundant(cudaStream_t s, double2* P, double2* V, const int* partner, int nred, int ng,
                                     int nstate);
cudaError_t oa_launch_sum_partials_multi(cudaStream_t s, int njob, const double* const* part, const int* n,
                                         const int* stride, const int* off, const double* scale, double* const* out);
cudaError_t oa_launch_sum_partials(cudaStream_t s, const double* part, int n, int stride, int off, double scale,
                                   double* out);
cudaError_t oa_launch_umma_fwd(cudaStream_t s, int nterm, const double* A, const double* B, int m, int n, long K,
                               long kx0_cols, double w_kx0, double alpha, float* part, int max_kb, double* C,
                               int* err_flag, int nsm);
cudaError_t oa_launch_umma_bwd(cudaStream_t s, int nterm, const double* M1, const double* X1, double a1_kx0,
                               double a1_rest, const double* M2, const double* X2, double a2, int nj, int nk,
                               long ncol, long kx0_cols, double* out, int* err_flag);
int oa_umma_max_kb(int m, int n, int nsm);
cudaError_t oa_split_kc(cudaStream_t s, int nt, const double* X, int rows, int rows_pad, long K, long ldx,
                        long kx0_cols, double w_kx0, __nv_bfloat16* P, long ldp, const int* cond = nullptr);
int oa_tg_rows_pad(int rows, int box);
int oa_tg_nb(int n);
int oa_tg_nb_fwd(int n);
cudaError_t oa_tfwd(cudaStream_t s, int nt, const __nv_bfloat16* PA, int rows_a, const __nv_bfloat16* PB, int rows_b,
                    int m, int n, long K, long ldp, double alpha, float* part, int max_kb, double* C, int* err_flag,
                    int nsm, const int* cond = nullptr);
cudaError_t oa_tbwd(cudaStream_t s, int nt, const __nv_bfloat16* PM1, const __nv_bfloat16* PX1, double a1_kx0,
                    double a1_rest, const __nv_bfloat16* PM2, const __nv_bfloat16* PX2, double a2, int nj, int nk,
                    long ncol, long ldx, long kx0_cols, double* out, int* err_flag, const double* yadd = nullptr,
                    const int* cond = nullptr);
cudaError_t oa_launch_pc_fwd_mn(cudaStream_t s, const double* A, const double* B, int m, int n, long K,
                                long kx0_cols, double w_kx0, double alpha, double* part, int nkb, double* C);
cudaError_t oa_launch_pc_bwd_jk(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                                const double* M2, const double* X2, double a2, int nj, int nk, long ncol,
                                long kx0_cols, double* out);
cudaError_t oa_launch_nl_sf(cudaStream_t s, const int* kx, const int* ky, const int* kz, int ng, const int* nl_atm,
                            int natm_nl, const int* atm_type, const double2* phase, int ktab, const double* spl,
                            int nspl, double gmin, double dg, const double* gz0, double tpi_l, double2* sf,
                            const OaPlaneOut* po);
cudaError_t oa_launch_nl_zscale(cudaStream_t s, const double* Z, int nstate, int natm_nl, const int* nl_atm,
                                const int* atm_type, const double* vnorm, double rvol, const double* occ, double* zt,
                                double* enl);

static thread_local char g_err[512] = "";

void oa_set_error(const char* msg, const char* file, int line) {
  snprintf(g_err, sizeof(g_err), "%s (%s:%d)", msg, file, line);
}

extern "C" const char* oa_gpu_last_error(void) { return g_err; }

#define OA_ARG_CHECK(cond, msg)                         \
  do {                                                  \
    if (!(cond)) { oa_set_error(msg, __FILE__, __LINE__); return OA_ERR_BAD_ARG; } \
  } while (0)

// FP64-accurate int8 tensor-core products of the mixed form (oa_ozaki.cu)
struct oa_oz;
oa_oz* oa_oz_create(int n, int ng, int nkx0, int nsm);
void oa_oz_free(oa_oz* z);
size_t oa_oz_bytes(const oa_oz* z);
cudaError_t oa_oz_overlap(oa_oz* z, cudaStream_t s, const double* X, long ldx, double alpha, double w_kx0,
                          double* S, int* err_flag, const int* cond);
cudaError_t oa_oz_rotate(oa_oz* z, cudaStream_t s, const double* T, const double* X, double* out, long ldo,
                         const OaPlaneOut* po, int* err_flag, const int* cond);

// extra per-context PC/Ortho/integrator scratch lives behind the struct
struct oa_ctx_pc {
  double* part;      // split-K partials
  int nkb;
  double* ns_work;   // 5 n^2 + grid
  int ns_grid;        // cooperative Newton-Schulz blocks
  int ns_cluster;     // cluster Newton-Schulz size (0: use the cooperative kernel)
  int* ns_status;    // [2] device
  double* ns_err;    // [1] device
  int* partner;      // [nkx0_red]
  double* cmass;     // [ng]
  double* ke_part;   // integrate partials
  int ke_nblk;
  double* dev_e;     // [8] device energies
  int* h_status;     // pinned
  double* h_vals;    // pinned [16]
  double* mat_a;     // [n][n] scratch
  double* mat_x;     // [n][n] scratch
  double* eye;       // [n][n] identity
  double* vtmp;      // [nstate][ng] complex scratch
  float* upart;      // split-K FP32 partials of the tensor-core forward GEMM
  int umax_kb;
  int umax_cap;      // split-K blocks upart holds
  int nkb_cap;       // split-K blocks part holds
  void* pl_big[3];   // bf16 planes [3][mx][pl_ld] of the big operands (slots below)
  void* pl_ma;       // bf16 planes [3][mx][mx] of the small matrices
  void* pl_mb;
  long pl_ld;
  // what each big slot holds, for reuse inside one native step (pl_cache)
  struct { const double* src; int rows, rows_pad, nt; long K, kx0; double w; bool valid; } pl_key[3];
  int pl_rows;       // row capacity of the big and small plane buffers
  int pl_cache;
  int* err_flag;     // device: set by a kernel whose bounded wait ran out
  int nsm;
  oa_oz* oz;         // int8 overlap / rotation (mixed form, up to 128 states)
};

static oa_ctx_pc* pcx(oa_ctx* c);

struct oa_ctx_full {
  oa_ctx c;
  oa_ctx_pc pc;
};

static oa_ctx_pc* pcx(oa_ctx* c) { return &reinterpret_cast<oa_ctx_full*>(c)->pc; }

// launch grid argument of oa_launch_ortho_ns: -cluster size for the cluster
// kernel, else the cooperative grid
static int ns_launch_grid(const oa_ctx_pc* p) { return p->ns_cluster > 0 ? -p->ns_cluster : p->ns_grid; }

// whether the Newton-Schulz launch can be captured in a CUDA graph
int oa_ns_capturable(oa_ctx* c) { return pcx(c)->ns_cluster > 0; }

static bool make_plan(int n, OaFftPlan* p) {
  p->n = n;
  p->nst = 0;
  int m = n;
  while (m % 4 == 0 && m > 0) { if (p->nst >= OA_FFT_MAXST) return false; p->rad[p->nst++] = 4; m /= 4; }
  const int prim[3] = {2, 3, 5};
  for (int q = 0; q < 3; ++q)
    while (m % prim[q] == 0) { if (p->nst >= OA_FFT_MAXST) return false; p->rad[p->nst++] = prim[q]; m /= prim[q]; }
  return m == 1 && p->nst >= 2 && n <= OA_FFT_MAXN;
}

static double2* make_twiddles(int n) {
  std::vector<double2> h(n);
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    h[k] = make_double2(cos(a), sin(a));
  }
  double2* d = nullptr;
  if (cudaMalloc(&d, n * sizeof(double2)) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), n * sizeof(double2), cudaMemcpyHostToDevice);
  return d;
}

template <typename T>
static cudaError_t upload(T** dst, const T* src, size_t n) {
  cudaError_t e = cudaMalloc(dst, (n ? n : 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  if (n) e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

// Per kx column of the state sphere: the run of z-lines {first line, ky of
// the first line, line count, 0} when the lines of every column are
// consecutive with ky rising by one (the reference's line order) and
// |ky| < ny / 2; false otherwise (the state-pair plane kernels then stay off).
static bool column_runs(const oa_system_desc* d, int nkx, std::vector<int>* out) {
  std::vector<int>& r = *out;
  r.assign((size_t)4 * nkx, 0);
  std::vector<char> seen(nkx, 0);
  int l = 0;
  while (l < d->nlines) {
    const int kx = d->line_kx[l];
    if (kx < 0 || kx >= nkx || seen[kx]) return false;
    seen[kx] = 1;
    int e = l + 1;
    while (e < d->nlines && d->line_kx[e] == kx) {
      if (d->line_ky[e] != d->line_ky[e - 1] + 1) return false;
      ++e;
    }
    if (2 * d->line_ky[l] <= -d->ny || 2 * d->line_ky[e - 1] >= d->ny) return false;
    r[4 * kx] = l; r[4 * kx + 1] = d->line_ky[l]; r[4 * kx + 2] = e - l;
    l = e;
  }
  return true;
}

static int pick_groups(int nz, int nstate, int bps, int nsm, int fixed = 0) {
  // minimise ceil(nz g / (nsm bps)) * (ceil(nstate / g) + fixed): waves of
  // blocks times the items each block runs, plus a fixed per-block cost in
  // items (pipeline fill and drain, twiddle and table loads)
  int best = 1;
  long bestc = -1;
  for (int g = 1; g <= 32 && g <= nstate; ++g) {
    const long waves = (nz * (long)g + (long)nsm * bps - 1) / ((long)nsm * bps);
    const long cost = waves * ((nstate + g - 1) / g + fixed);
    if (bestc < 0 || cost < bestc) { bestc = cost; best = g; }
  }
  return best;
}

extern "C" oa_status oa_gpu_init(const oa_system_desc* d, int precision, oa_ctx** out) {
  OA_ARG_CHECK(d && out, "null argument");
  OA_ARG_CHECK(precision == OA_FP64 || precision == OA_MIXED, "precision must be OA_FP64 or OA_MIXED");
  OA_ARG_CHECK(d->nx > 0 && d->ny > 0 && d->nz > 0 && d->nstate > 0 && d->ng > 0 && d->nlines > 0, "bad sizes");
  OA_ARG_CHECK(d->ntype >= 1 && d->ntype <= 4, "ntype must be 1..4");
  OA_ARG_CHECK(d->natm == 0 || d->atm_type, "null atm_type");
  for (int a = 0; a < d->natm; ++a) OA_ARG_CHECK(d->atm_type[a] >= 0 && d->atm_type[a] < d->ntype, "atom type out of range");
  *out = nullptr;
  oa_ctx_full* F = (oa_ctx_full*)calloc(1, sizeof(oa_ctx_full));
  if (!F) return OA_ERR_CUDA;
  oa_ctx* c = &F->c;
  oa_ctx_pc* p = &F->pc;
  cudaGetDevice(&c->device);
  c->precision = precision;
  c->nx = d->nx; c->ny = d->ny; c->nz = d->nz; c->npts = d->nx * d->ny * d->nz;
  c->ng = d->ng; c->nlines = d->nlines; c->nstate = d->nstate;
  c->ldl = (d->nlines + 31) / 32 * 32;
  c->nkx0 = d->nkx0; c->nkx0_red = d->nkx0_red; c->nkx0_uni = d->nkx0_uni; c->nkx0_zero = d->nkx0_zero;
  c->natm = d->natm; c->ntype = d->ntype;
  c->box = d->box; c->vol = d->box * d->box * d->box;
  c->ecut_psi = d->ecut_psi; c->ecut_rho = d->ecut_rho; c->alp_ewd = d->alp_ewd;
  c->nspl = d->nspl; c->spl_gmin = d->spl_gmin; c->spl_dg = d->spl_dg;
  int mkx = 0;
  for (int l = 0; l < d->nlines; ++l) mkx = d->line_kx[l] > mkx ? d->line_kx[l] : mkx;
  c->nkx_s = mkx + 1;
  c->nkx_d = d->nx / 2 + 1;
  c->nlines_d = c->nkx_d * d->ny;
  c->ldl_d = (c->nlines_d + 31) / 32 * 32;
  const double f = 2.0 * M_PI / d->box;
  c->kmax_tab = (int)floor(sqrt(d->ecut_rho) / f) + 1;
  double gz = 0.0;
  for (int a = 0; a < d->natm; ++a) gz += d->gzvps[d->atm_type[a]];
  c->gzvps_sum = gz;
  for (int t = 0; t < d->ntype; ++t) c->gzvps_t[t] = d->gzvps[t];
  if (!make_plan(d->nx, &c->plan_x) || !make_plan(d->ny, &c->plan_y) || !make_plan(d->nz, &c->plan_z)) {
    oa_set_error("FFT length must be 2^a 3^b 5^c with at least two radix stages and <= 512", __FILE__, __LINE__);
    free(F);
    return OA_ERR_UNSUPPORTED;
  }
  c->npair_d = 16; c->ychunk_d = 16;
  while (oa_rho_plane_smem_bytes(d->nx, d->ny, c->nkx_d, c->npair_d, c->ychunk_d) > OA_MAX_SMEM && c->npair_d > 1) {
    c->npair_d /= 2; c->ychunk_d = c->npair_d;
  }
  c->smem_plane = oa_plane_smem_bytes(precision, d->nx, d->ny, c->nkx_s);
  c->smem_rho_plane = oa_rho_plane_smem_bytes(d->nx, d->ny, c->nkx_d, c->npair_d, c->ychunk_d);
  if (c->smem_plane > OA_MAX_SMEM || c->smem_rho_plane > OA_MAX_SMEM) {
    oa_set_error("grid too large for the shared-memory plane kernels at this precision", __FILE__, __LINE__);
    free(F);
    return OA_ERR_UNSUPPORTED;
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  int bps = (int)(228 * 1024 / (c->smem_plane + 1024));
  {
    const int occ_bps = oa_plane_blocks_per_sm(precision);
    if (occ_bps > 0 && occ_bps < bps) bps = occ_bps;
    if (bps < 1) bps = 1;
  }
  c->ngroup = pick_groups(d->nz, d->nstate, bps, nsm);
  // the state-pair kernels software-pipeline the pairs of a block: a fixed
  // cost of about two pairs per block, which is what the autotuner's
  // measurements over 8-32 water systems on 64^3-108^3 grids imply
  c->ngroup_pair = pick_groups(d->nz, (d->nstate + 1) / 2, 1, nsm, 2);
  c->pair_kymax = 0;
  c->z_ext = 0;
  for (int l = 0; l < d->nlines; ++l) {
    const int a = d->line_ky[l] < 0 ? -d->line_ky[l] : d->line_ky[l];
    c->pair_kymax = a > c->pair_kymax ? a : c->pair_kymax;
    c->z_ext = std::max(c->z_ext, std::max(d->line_nneg[l], d->line_npos[l]));
  }
  c->rho_ngroup = c->ngroup;
  c->nblk_z = (d->nlines + OA_LB - 1) / OA_LB;
  c->zseg = 0;
  {
    bool packed = d->nlines > 0;
    for (int l = 0; l < d->nlines && packed; ++l) {
      const int end = d->line_off[l] + d->line_nneg[l] + d->line_npos[l];
      packed = end == (l + 1 < d->nlines ? d->line_off[l + 1] : d->ng);
    }
    for (int l0 = 0; l0 < d->nlines && packed; l0 += OA_LB) {
      const int g1 = l0 + OA_LB < d->nlines ? d->line_off[l0 + OA_LB] : d->ng;
      c->zseg = std::max(c->zseg, g1 - d->line_off[l0]);
    }
    if (c->zseg > 2048) c->zseg = 0;  // keeps the staged runs within 64 KB
  }

  const size_t csz = precision == OA_FP64 ? sizeof(double2) : sizeof(float2);
  const size_t rsz = precision == OA_FP64 ? sizeof(double) : sizeof(float);
  cudaError_t e = cudaSuccess;
#define TRY(x) do { e = (x); if (e != cudaSuccess) goto fail; } while (0)
  {
    std::vector<double> g2(d->ng);
    std::vector<int> kxv(d->kx, d->kx + d->ng);
    for (int i = 0; i < d->ng; ++i) {
      const double gx = f * d->kx[i], gy = f * d->ky[i], gzz = f * d->kz[i];
      g2[i] = gx * gx + gy * gy + gzz * gzz;
    }
    TRY(upload(&c->line_kx, d->line_kx, d->nlines));
    TRY(upload(&c->line_ky, d->line_ky, d->nlines));
    TRY(upload(&c->line_off, d->line_off, d->nlines));
    TRY(upload(&c->line_nneg, d->line_nneg, d->nlines));
    TRY(upload(&c->line_npos, d->line_npos, d->nlines));
    TRY(upload(&c->kx, kxv.data(), d->ng));
    TRY(upload(&c->g2, g2.data(), d->ng));
    TRY(upload(&c->occ, d->occ, d->nstate));
    TRY(upload(&c->spl, d->spl, (size_t)d->ntype * d->nspl * 4));
    TRY(upload(&c->q_type, d->q_type, d->ntype));
    TRY(upload(&c->atm_type, d->atm_type, d->natm));
    {
      std::vector<int> perm;
      perm.reserve(d->natm);
      for (int t = 0; t < d->ntype; ++t) {
        c->type_off[t] = (int)perm.size();
        for (int a = 0; a < d->natm; ++a)
          if (d->atm_type[a] == t) perm.push_back(a);
      }
      for (int t = d->ntype; t <= 4; ++t) c->type_off[t] = (int)perm.size();
      if ((int)perm.size() != d->natm) { e = cudaErrorInvalidValue; goto fail; }
      TRY(upload(&c->atm_perm, perm.data(), d->natm));
    }
    TRY(upload(&c->pos, d->pos, (size_t)3 * d->natm));
    TRY(upload(&p->partner, d->red_partner, d->nkx0_red));
    TRY(upload(&c->ky, d->ky, d->ng));
    TRY(upload(&c->kz, d->kz, d->ng));
    c->natm_nl = d->natm_nl;
    TRY(upload(&c->nl_atm, d->nl_atm, d->natm_nl));
    TRY(upload(&c->nl_spl, d->nl_spl, d->natm_nl ? (size_t)d->ntype * d->nspl * 4 : 0));
    TRY(upload(&c->nl_vnorm, d->nl_vnorm, d->natm_nl ? d->ntype : 0));
    TRY(upload(&c->nl_gz0, d->nl_gz0, d->natm_nl ? d->ntype : 0));
    TRY(cudaMalloc(&c->sf, ((size_t)d->natm_nl * d->ng + 1) * sizeof(double2)));
    TRY(cudaMalloc(&c->zmat, ((size_t)d->natm_nl * d->nstate + 1) * sizeof(double)));
    TRY(cudaMalloc(&c->zt, ((size_t)d->natm_nl * d->nstate + 1) * sizeof(double)));
    TRY(cudaMalloc(&c->enl, (size_t)d->nstate * sizeof(double)));
    TRY(cudaMalloc(&c->enl_eke, (size_t)d->nstate * sizeof(double)));
    TRY(upload(&p->cmass, d->cmass, d->ng));
    c->tw_x = make_twiddles(d->nx);
    c->tw_y = make_twiddles(d->ny);
    c->tw_z = make_twiddles(d->nz);
    if (!c->tw_x || !c->tw_y || !c->tw_z) { e = cudaErrorMemoryAllocation; goto fail; }
    TRY(cudaMalloc(&c->phase, (size_t)d->natm * 3 * (2 * c->kmax_tab + 1) * sizeof(double2)));
    c->zbuf_bytes = (size_t)d->nstate * d->nz * c->ldl * csz;
    TRY(cudaMalloc(&c->zbuf, c->zbuf_bytes));
    {
      std::vector<int> runs;
      if (precision == OA_MIXED && d->nx == d->ny &&
          oa_pair_plane_supported(d->nx, c->nkx_s, d->nlines, c->ldl) && column_runs(d, c->nkx_s, &runs))
        TRY(upload(&c->pair_cols, runs.data(), runs.size()));
    }
    if (c->pair_cols) {
      // charge partials of the z forward pass (state x 16-line block) and of
      // the pair density pass (group x plane) for the density renormalisation
      c->nq = d->nstate * ((d->nlines + OA_LB - 1) / OA_LB);
      c->nq2 = c->ngroup_pair * d->nz;
      TRY(cudaMalloc(&c->qpart, (size_t)c->nq * sizeof(double)));
      TRY(cudaMalloc(&c->qpart2, (size_t)c->nq2 * sizeof(double)));
      c->nq2_cap = c->nq2;
      TRY(cudaMalloc(&c->qscale, sizeof(double)));
    }
    {
      const int ng = c->ngroup > c->ngroup_pair ? c->ngroup : c->ngroup_pair;
      TRY(cudaMalloc(&c->rho_part, (size_t)ng * c->npts * sizeof(double)));
      c->rho_groups_cap = ng;
    }
    if (d->nx == d->ny && oa_pencil_supported(d->nx))
      TRY(cudaMalloc(&c->psir, (size_t)(d->nstate + 1) / 2 * 2 * c->npts * rsz));
    TRY(cudaMalloc(&c->rho, (size_t)c->npts * sizeof(double)));
    TRY(cudaMalloc(&c->vxc, (size_t)c->npts * sizeof(double)));
    TRY(cudaMalloc(&c->vks, (size_t)c->npts * rsz));
    TRY(cudaMalloc(&c->dz, (size_t)d->nz * c->ldl_d * sizeof(double2)));
    c->red_len = (size_t)5 * oa_rho_xc_nblk() + 3 * (size_t)oa_rho_z_nblk(c) + 64;  // xc, z pass, GGA partials
    c->gga_cut = 5.0e-5;
    TRY(cudaMalloc(&c->red, c->red_len * sizeof(double)));
    TRY(cudaMalloc(&c->eke_part, (size_t)d->nstate * c->nblk_z * sizeof(double)));
    p->nkb = 160;  // split-K partials: about one CTA per SM for a 128 x 128 product
    p->nkb_cap = p->nkb;
    // split-K partials; also the block partials of the minimisation's |F|^2 (>= 1024)
    // (the nonlocal Z product is nstate x natm_nl: more columns than states
    // when there are more nonlocal atoms than states)
    TRY(cudaMalloc(&p->part, std::max((size_t)p->nkb * d->nstate * std::max(d->nstate, d->natm_nl), (size_t)1024) *
                                 sizeof(double)));
    p->ns_grid = oa_ns_grid(d->nstate, c->device);
    p->ns_cluster = oa_ns_cluster_size(d->nstate);
    TRY(cudaMalloc(&p->ns_work, ((size_t)5 * d->nstate * d->nstate + p->ns_grid + 32) * sizeof(double)));
    TRY(cudaMalloc(&p->ns_status, 4 * sizeof(int)));
    TRY(cudaMalloc(&p->ns_err, 2 * sizeof(double)));
    p->ke_nblk = oa_integrate_nblk(d->ng, d->nstate);
    TRY(cudaMalloc(&p->ke_part, p->ke_nblk * sizeof(double)));
    TRY(cudaMalloc(&p->dev_e, 16 * sizeof(double)));
    TRY(cudaMemset(p->dev_e, 0, 16 * sizeof(double)));
    TRY(cudaMalloc(&p->mat_a, (size_t)d->nstate * d->nstate * sizeof(double)));
    TRY(cudaMalloc(&p->mat_x, (size_t)d->nstate * d->nstate * sizeof(double)));
    {
      std::vector<double> eye((size_t)d->nstate * d->nstate, 0.0);
      for (int i = 0; i < d->nstate; ++i) eye[(size_t)i * d->nstate + i] = 1.0;
      TRY(upload(&p->eye, eye.data(), eye.size()));
    }
    TRY(cudaMalloc(&p->vtmp, (size_t)d->nstate * d->ng * sizeof(double2)));
    p->nsm = nsm;
    p->umax_kb = oa_umma_max_kb(d->nstate, d->nstate, nsm);
    {
      const int mx = d->nstate > d->natm_nl ? d->nstate : d->natm_nl;
      const int kbz = oa_umma_max_kb(d->nstate, d->natm_nl > 0 ? d->natm_nl : 1, nsm);
      const size_t need = (size_t)(p->umax_kb > kbz ? p->umax_kb : kbz) * d->nstate * mx;
      TRY(cudaMalloc(&p->upart, need * sizeof(float)));
      p->umax_kb = p->umax_kb > kbz ? p->umax_kb : kbz;
      p->umax_cap = p->umax_kb;
    }
    TRY(cudaMalloc(&p->err_flag, sizeof(int)));
    TRY(cudaMemset(p->err_flag, 0, sizeof(int)));
    {
      const int mx = d->nstate > d->natm_nl ? d->nstate : d->natm_nl;
      p->pl_ld = (2L * d->ng + 63) / 64 * 64;
      p->pl_rows = oa_tg_rows_pad(mx, 128);
      for (int q = 0; q < 3; ++q) {
        TRY(cudaMalloc(&p->pl_big[q], (size_t)3 * p->pl_rows * p->pl_ld * 2));
        // padding rows and columns stay zero: every writer of a slot writes only its rows and columns
        TRY(cudaMemset(p->pl_big[q], 0, (size_t)3 * p->pl_rows * p->pl_ld * 2));
      }
      TRY(cudaMalloc(&p->pl_ma, (size_t)3 * p->pl_rows * p->pl_rows * 2));
      TRY(cudaMalloc(&p->pl_mb, (size_t)3 * p->pl_rows * p->pl_rows * 2));
    }
    TRY(cudaMallocHost(&p->h_status, 4 * sizeof(int)));
    TRY(cudaMallocHost(&p->h_vals, 16 * sizeof(double)));
    TRY(cudaDeviceSynchronize());
  }
#undef TRY
  *out = c;
  return OA_OK;
fail:
  oa_set_error(cudaGetErrorString(e), __FILE__, __LINE__);
  oa_gpu_destroy(c);
  return OA_ERR_CUDA;
}

void oa_step_free(oa_ctx* c);
void oa_ions_free(oa_ctx* c);
static void ees_free(oa_ctx* c);

extern "C" oa_status oa_gpu_destroy(oa_ctx* c) {
  if (!c) return OA_OK;
  oa_step_free(c);
  ees_free(c);
  oa_eesl_free(c);
  oa_ions_free(c);
  oa_ctx_pc* p = pcx(c);
  oa_oz_free(p->oz);
  p->oz = nullptr;
  void* dev[] = {c->line_kx, c->line_ky, c->line_off, c->line_nneg, c->line_npos, c->kx, c->g2, c->tw_x, c->tw_y,
                 c->tw_z, c->spl, c->q_type, c->atm_type, c->atm_perm, c->pos, c->psir, c->pair_cols, c->phase, c->occ, c->zbuf, c->rho_part, c->rho,
                 c->vks, c->vxc, c->dz, c->red, c->eke_part, p->part, p->ns_work, p->ns_status, p->ns_err,
                 p->partner, p->cmass, p->ke_part, p->dev_e, p->mat_a, p->mat_x, p->eye, p->vtmp, p->upart,
                 p->pl_big[0], p->pl_big[1], p->pl_big[2], p->pl_ma, p->pl_mb,
                 p->err_flag, c->ky, c->kz, c->nl_atm, c->nl_spl, c->nl_vnorm, c->nl_gz0, c->sf, c->zmat, c->zt,
                 c->enl, c->enl_eke, c->grad, c->dzg, c->qpart, c->qpart2, c->qscale};
  for (void* q : dev) if (q) cudaFree(q);
  if (p->h_status) cudaFreeHost(p->h_status);
  if (p->h_vals) cudaFreeHost(p->h_vals);
  free(reinterpret_cast<oa_ctx_full*>(c));
  return OA_OK;
}

extern "C" size_t oa_gpu_scratch_bytes(const oa_ctx* c) {
  if (!c) return 0;
  const size_t rsz = c->precision == OA_FP64 ? 8 : 4;
  const int ng = c->ngroup > c->ngroup_pair ? c->ngroup : c->ngroup_pair;
  return c->zbuf_bytes + (size_t)ng * c->npts * 8 + (size_t)c->npts * (16 + rsz) +
         (size_t)c->nz * c->ldl_d * 16 + (c->grad ? (size_t)3 * c->npts * 8 + (size_t)3 * c->nz * c->ldl_d * 16 : 0);
}

extern "C" oa_status oa_gpu_state_fft_fwd(oa_ctx* c, void* stream, const double* psi, double* rho_out) {
  OA_ARG_CHECK(c && psi, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  OA_CUDA_TRY(oa_launch_state_zfwd(c, s, (const double2*)psi, 0, c->nstate));
  OA_CUDA_TRY(oa_launch_state_plane_density(c, s));
  OA_CUDA_TRY(oa_launch_rho_xc(c, s));
  if (rho_out) OA_CUDA_TRY(cudaMemcpyAsync(rho_out, c->rho, (size_t)c->npts * 8, cudaMemcpyDeviceToDevice, s));
  return OA_OK;
}

__global__ void k_to_double(const float* a, double* b, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) b[i] = a[i];
}
__global__ void k_to_float(const double* a, float* b, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

extern "C" oa_status oa_gpu_vks_build(oa_ctx* c, void* stream, double* vks_out) {
  OA_ARG_CHECK(c, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  oa_ctx_pc* p = pcx(c);
  OA_CUDA_TRY(oa_launch_rho_fft_hart(c, s));
  const int nx = oa_rho_xc_nblk(), nzb = oa_rho_z_nblk(c);
  const double vs = c->vol / (double)c->npts;
  // EEXC = (0.75 ex + ec) V/N ; MUXC = sum vxc rho V/N; EGGA = (ex + ec of the
  // gradient correction) V/N, the two halves of each block's partials
  {
    const double* gp = c->red + oa_rho_gga_red_off(c);
    const double* part[8] = {c->red, c->red, c->red, c->red + 3 * nx, c->red + 3 * nx, c->red + 3 * nx, gp, gp + 1};
    const int n[8] = {nx, nx, nx, nzb, nzb, nzb, nx, nx};
    const int stride[8] = {3, 3, 3, 3, 3, 3, 2, 2};
    const int off[8] = {0, 1, 2, 0, 1, 2, 0, 0};
    const double scale[8] = {0.75 * vs, vs, vs, 0.5, 1.0, 0.5, vs, vs};
    double* out[8] = {p->dev_e + 8, p->dev_e + 9, p->dev_e + OA_E_MUXC, p->dev_e + OA_E_EHART,
                      p->dev_e + OA_E_EEXT, p->dev_e + OA_E_EWALD, p->dev_e + 11, p->dev_e + 12};
    OA_CUDA_TRY(oa_launch_sum_partials_multi(s, c->gga ? 8 : 6, part, n, stride, off, scale, out));
    if (!c->gga) OA_CUDA_TRY(cudaMemsetAsync(p->dev_e + 11, 0, 2 * sizeof(double), s));
  }
  if (vks_out) {
    if (c->precision == OA_FP64)
      OA_CUDA_TRY(cudaMemcpyAsync(vks_out, c->vks, (size_t)c->npts * 8, cudaMemcpyDeviceToDevice, s));
    else {
      k_to_double<<<592, 256, 0, s>>>((const float*)c->vks, vks_out, (size_t)c->npts);
      OA_CUDA_TRY(cudaGetLastError());
    }
  }
  return OA_OK;
}

extern "C" oa_status oa_gpu_set_vks(oa_ctx* c, void* stream, const double* vks) {
  OA_ARG_CHECK(c && vks, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (c->precision == OA_FP64)
    OA_CUDA_TRY(cudaMemcpyAsync(c->vks, vks, (size_t)c->npts * 8, cudaMemcpyDeviceToDevice, s));
  else {
    k_to_float<<<592, 256, 0, s>>>(vks, (float*)c->vks, (size_t)c->npts);
    OA_CUDA_TRY(cudaGetLastError());
  }
  return OA_OK;
}

// EKE per state (one block per state, deterministic) = half the weighted sum
__global__ void k_eke_states(const double* part, int nblk, double* eke_state) {
  __shared__ double sh[32];
  const int st = blockIdx.x;
  double sv = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) sv += part[(size_t)st * nblk + i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sv += __shfl_xor_sync(0xffffffffu, sv, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = sv;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
    eke_state[st] = 0.5 * t;
  }
}

extern "C" oa_status oa_gpu_vks_apply_fft_bwd(oa_ctx* c, void* stream, const double* psi, int recompute_fwd,
                                              const double* fnl, double* force, double* eke_out) {
  OA_ARG_CHECK(c && psi && force, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (recompute_fwd) {
    OA_CUDA_TRY(oa_launch_state_zfwd(c, s, (const double2*)psi, 0, c->nstate));
    c->psir_valid = 0;  // the z-line buffer is newer than psi(r)
  }
  OA_CUDA_TRY(oa_launch_state_plane_vks(c, s));
  OA_CUDA_TRY(oa_launch_state_zbwd(c, s, (const double2*)psi, (const double2*)fnl, (double2*)force, 0, c->nstate));
  double* es = eke_out ? eke_out : c->enl_eke;
  k_eke_states<<<c->nstate, 128, 0, s>>>(c->eke_part, c->nblk_z, es);
  OA_CUDA_TRY(cudaGetLastError());
  OA_CUDA_TRY(oa_launch_sum_partials(s, es, c->nstate, 1, 0, 1.0, pcx(c)->dev_e + OA_E_EKE));
  return OA_OK;
}

extern "C" oa_status oa_gpu_pc_forward(oa_ctx* c, void* stream, const double* left, const double* right,
                                       double alpha, double w_kx0, double* C) {
  OA_ARG_CHECK(c && left && right && C, "null argument");
  oa_ctx_pc* p = pcx(c);
  OA_CUDA_TRY(oa_launch_pc_fwd((cudaStream_t)stream, left, right, c->nstate, 2L * c->ng, 2L * c->nkx0, w_kx0, alpha,
                               p->part, p->nkb, C));
  return OA_OK;
}

// The int8 products' buffers (digit slices of psi_t, about 6 bytes per
// coefficient value) are allocated on the first call, so that contexts that
// do not use them pay nothing.
static bool oz_ready(oa_ctx* c) {
  oa_ctx_pc* p = pcx(c);
  if (!p->oz && c->precision == OA_MIXED && c->nstate <= 128)
    p->oz = oa_oz_create(c->nstate, c->ng, c->nkx0, p->nsm);
  return p->oz != nullptr;
}

extern "C" oa_status oa_gpu_pc_overlap_i8(oa_ctx* c, void* stream, const double* psi_t, double alpha,
                                          double w_kx0, double* S) {
  OA_ARG_CHECK(c && psi_t && S, "null argument");
  oa_ctx_pc* p = pcx(c);
  if (!oz_ready(c)) {
    oa_set_error("the int8 overlap needs a mixed-precision context with at most 128 states", __FILE__, __LINE__);
    return OA_ERR_UNSUPPORTED;
  }
  OA_CUDA_TRY(oa_oz_overlap(p->oz, (cudaStream_t)stream, psi_t, 2L * c->ng, alpha, w_kx0, S, p->err_flag, nullptr));
  return OA_OK;
}

extern "C" oa_status oa_gpu_pc_rotate_i8(oa_ctx* c, void* stream, const double* T, const double* psi_t,
                                         double* psi_out) {
  OA_ARG_CHECK(c && T && psi_t && psi_out, "null argument");
  OA_ARG_CHECK(psi_out != psi_t, "psi_out must not alias psi_t");
  oa_ctx_pc* p = pcx(c);
  if (!oz_ready(c)) {
    oa_set_error("the int8 rotation needs a mixed-precision context with at most 128 states", __FILE__, __LINE__);
    return OA_ERR_UNSUPPORTED;
  }
  const cudaError_t e = oa_oz_rotate(p->oz, (cudaStream_t)stream, T, psi_t, psi_out, 2L * c->ng, nullptr,
                                     p->err_flag, nullptr);
  if (e == cudaErrorNotSupported) {
    oa_set_error("oa_gpu_pc_rotate_i8: psi_t is not the operand of the last oa_gpu_pc_overlap_i8", __FILE__,
                 __LINE__);
    return OA_ERR_BAD_ARG;
  }
  OA_CUDA_TRY(e);
  // psi_out changed: planes of psi must be split again when a product needs them
  p->pl_key[0].valid = false;
  return OA_OK;
}


cudaError_t oa_launch_min_fovlap(cudaStream_t s, const double2* F, size_t n, double* part);
int oa_min_nblk();
cudaError_t oa_launch_min_step(cudaStream_t s, const double2* F, double2* conj, double2* P, const double* cmass,
                               const double* g2, double ecut, int ng, int nstate, double gamma, double dt);

extern "C" oa_status oa_gpu_min_fovlap(oa_ctx* c, void* stream, const double* force, double* fovlap_out) {
  OA_ARG_CHECK(c && force && fovlap_out, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  oa_ctx_pc* p = pcx(c);
  const int nb = oa_min_nblk();
  // block partials in the split-K partial buffer (at least nb doubles), summed in a fixed order
  OA_CUDA_TRY(oa_launch_min_fovlap(s, (const double2*)force, (size_t)c->nstate * c->ng, p->part));
  OA_CUDA_TRY(oa_launch_sum_partials(s, p->part, nb, 1, 0, 1.0, p->dev_e + 15));
  OA_CUDA_TRY(cudaMemcpyAsync(p->h_vals + 15, p->dev_e + 15, sizeof(double), cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaStreamSynchronize(s));
  *fovlap_out = p->h_vals[15];
  return OA_OK;
}

extern "C" oa_status oa_gpu_min_step(oa_ctx* c, void* stream, const double* force, double* conj_grad, double* psi,
                                     double gamma, double dt) {
  OA_ARG_CHECK(c && force && psi, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  oa_ctx_pc* p = pcx(c);
  OA_CUDA_TRY(oa_launch_min_step(s, (const double2*)force, (double2*)conj_grad, (double2*)psi, p->cmass, c->g2,
                                 c->ecut_psi, c->ng, c->nstate, gamma, dt));
  // Gamma redundancy sync of psi (computeRedPsi, gspace.ci:692-708)
  OA_CUDA_TRY(oa_launch_sync_redundant(s, (double2*)psi, nullptr, p->partner, c->nkx0_red, c->ng, c->nstate));
  return OA_OK;
}

extern "C" oa_status oa_gpu_ortho_invsqrt(oa_ctx* c, void* stream, const double* S, double* T, double tol,
                                          int max_iter, int* iters_out, double* err_out, double* smax_out) {
  OA_ARG_CHECK(c && S && T && max_iter > 0, "bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  oa_ctx_pc* p = pcx(c);
  OA_CUDA_TRY(oa_launch_ortho_ns(s, S, c->nstate, 0.5, tol, max_iter, p->ns_work, T, p->ns_status, p->ns_err,
                                 ns_launch_grid(p)));
  OA_CUDA_TRY(cudaMemcpyAsync(p->h_status, p->ns_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaMemcpyAsync(p->h_vals, p->ns_err, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaStreamSynchronize(s));
  if (iters_out) *iters_out = p->h_status[0];
  if (err_out) *err_out = p->h_vals[0];
  if (smax_out) *smax_out = p->h_vals[1];
  if (!isfinite(p->h_vals[0])) { oa_set_error("Newton-Schulz residual is not finite", __FILE__, __LINE__); return OA_ERR_NONFINITE; }
  if (!p->h_status[1]) { oa_set_error("Newton-Schulz reached max_iter", __FILE__, __LINE__); return OA_ERR_NOT_CONVERGED; }
  return OA_OK;
}

extern "C" oa_status oa_gpu_pc_backward(oa_ctx* c, void* stream, const double* M1, const double* X1,
                                        double a1_kx0, double a1_rest, const double* M2, const double* X2, double a2,
                                        double* out) {
  OA_ARG_CHECK(c && M1 && X1 && out, "null argument");
  OA_ARG_CHECK((M2 == nullptr) == (X2 == nullptr), "M2 and X2 must both be given or both be NULL");
  OA_ARG_CHECK(out != X1 && out != X2, "out must not alias an input");
  OA_CUDA_TRY(oa_launch_pc_bwd((cudaStream_t)stream, M1, X1, a1_kx0, a1_rest, M2, X2, a2, c->nstate, 2L * c->ng,
                               2L * c->nkx0, out));
  return OA_OK;
}

extern "C" oa_status oa_gpu_small_gemm(oa_ctx* c, void* stream, const double* A, const double* B, double alpha,
                                       double* C) {
  OA_ARG_CHECK(c && A && B && C, "null argument");
  OA_CUDA_TRY(oa_launch_small_gemm((cudaStream_t)stream, A, B, c->nstate, alpha, C));
  return OA_OK;
}

// psi_in / sel (optional): the coefficients are read from psi_in instead of
// psi when *sel != 0 (the native step's deferred PsiV copy)
oa_status oa_integrate_sel(oa_ctx* c, cudaStream_t s, const double* force, double* vpsi, double* psi,
                           const double* psi_in, const int* sel, double dt, int complete_prev, double* fict_ke_out) {
  oa_ctx_pc* p = pcx(c);
  const int r0 = c->nkx0_red, r1 = c->nkx0_red + c->nkx0_zero, iend = c->nkx0_red + c->nkx0_uni;
  OA_CUDA_TRY(oa_launch_integrate(s, (const double2*)force, (double2*)vpsi, (double2*)psi, (const double2*)psi_in,
                                  sel, p->cmass, c->ng, c->nstate, r0, r1, iend, dt, complete_prev, p->ke_part,
                                  p->ke_nblk));
  OA_CUDA_TRY(oa_launch_sum_partials(s, p->ke_part, p->ke_nblk, 1, 0, 1.0, p->dev_e + OA_E_FICT));
  if (fict_ke_out)
    OA_CUDA_TRY(cudaMemcpyAsync(fict_ke_out, p->dev_e + OA_E_FICT, sizeof(double), cudaMemcpyDeviceToDevice, s));
  OA_CUDA_TRY(oa_launch_sync_redundant(s, (double2*)psi, (double2*)vpsi, p->partner, c->nkx0_red, c->ng, c->nstate));
  return OA_OK;
}

extern "C" oa_status oa_gpu_integrate(oa_ctx* c, void* stream, const double* force, double* vpsi, double* psi,
                                      double dt, int complete_prev, double* fict_ke_out) {
  OA_ARG_CHECK(c && force && vpsi && psi, "null argument");
  return oa_integrate_sel(c, (cudaStream_t)stream, force, vpsi, psi, nullptr, nullptr, dt, complete_prev,
                          fict_ke_out);
}

__global__ void k_energy_combine(double* e) {
  // EEXC = 0.75 ex V/N + ec V/N was stored split at [8] and [9], EGGA at [11] and [12]
  e[OA_E_EEXC] = e[8] + e[9];
  e[OA_E_EGGA] = e[11] + e[12];
}

extern "C" oa_status oa_gpu_energies(oa_ctx* c, void* stream, double* out7) {
  OA_ARG_CHECK(c && out7, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  oa_ctx_pc* p = pcx(c);
  k_energy_combine<<<1, 1, 0, s>>>(p->dev_e);
  OA_CUDA_TRY(cudaGetLastError());
  OA_CUDA_TRY(cudaMemcpyAsync(p->h_vals, p->dev_e, 16 * sizeof(double), cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaStreamSynchronize(s));
  out7[0] = p->h_vals[OA_E_EKE];
  out7[1] = p->h_vals[OA_E_EHART];
  out7[2] = p->h_vals[OA_E_EEXT];
  out7[3] = p->h_vals[OA_E_EWALD];
  out7[4] = p->h_vals[OA_E_EEXC];
  out7[5] = p->h_vals[OA_E_MUXC];
  out7[6] = p->h_vals[OA_E_FICT];
  out7[7] = p->h_vals[OA_E_ENL];
  out7[8] = p->h_vals[OA_E_EGGA];
  out7[9] = p->h_vals[OA_E_ION_KE];
  out7[10] = p->h_vals[OA_E_EWALD_REAL];
  return OA_OK;
}

extern "C" oa_status oa_gpu_set_xc(oa_ctx* c, int functional, double gradient_cutoff) {
  OA_ARG_CHECK(c, "null argument");
  if (functional != 0 && functional != 1) {
    oa_set_error("functional must be 0 (PZ-LDA) or 1 (BLYP)", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  if (!(gradient_cutoff > 0.0)) {
    oa_set_error("gradient_cutoff must be > 0", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  if (functional == 1 && !c->grad) {
    OA_CUDA_TRY(cudaMalloc(&c->grad, (size_t)3 * c->npts * sizeof(double)));
    OA_CUDA_TRY(cudaMalloc(&c->dzg, (size_t)3 * c->nz * c->ldl_d * sizeof(double2)));
  }
  c->gga = functional;
  c->gga_cut = gradient_cutoff;
  c->xc_gen += 1;
  return OA_OK;
}

__global__ void k_sym_quarter(const double* A, int n, double* X) {
  const int i = blockIdx.y * 16 + threadIdx.y, j = blockIdx.x * 16 + threadIdx.x;
  if (i < n && j < n) X[(size_t)i * n + j] = 0.25 * (A[(size_t)i * n + j] + A[(size_t)j * n + i]);
}

__global__ void k_copy_cond(double* __restrict__ dst, const double* __restrict__ src, size_t n, const int* cond) {
  if (*cond == 0) return;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}


cudaError_t oa_dgemm_fwd(cudaStream_t s, const double* A, const double* B, int m, int n, long K, long kx0_cols,
                         double w_kx0, double alpha, double* part, int nkb, double* C, const int* cond);
cudaError_t oa_dgemm_bwd_ex(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                            const double* M2, const double* X2, double a2, int nj, int nk, long ncol, long kx0_cols,
                            double* out, const int* cond, const double* yadd, double* out2, const int* cond2,
                            const OaPlaneOut* po = nullptr, double* vel = nullptr, double vscale = 0.0,
                            const int* vcond = nullptr);

#define OA_STEP_CHECK(x) do { const oa_status st_ = (x); if (st_ != OA_OK) return st_; } while (0)

#define OA_ALIGN_TRY(x)                                                                       \
  do {                                                                                        \
    const cudaError_t ea_ = (x);                                                              \
    if (ea_ == cudaErrorNotSupported) {                                                       \
      oa_set_error("coefficient arrays must be 16-byte aligned", __FILE__, __LINE__);         \
      return OA_ERR_BAD_ARG;                                                                  \
    }                                                                                         \
    OA_CUDA_TRY(ea_);                                                                          \
  } while (0)

extern "C" oa_status oa_gpu_set_atoms(oa_ctx* c, void* stream, const double* pos_host) {
  OA_ARG_CHECK(c && pos_host, "null argument");
  OA_CUDA_TRY(cudaMemcpyAsync(c->pos, pos_host, (size_t)3 * c->natm * sizeof(double), cudaMemcpyHostToDevice,
                              (cudaStream_t)stream));
  return OA_OK;
}

// Average device time of each kernel of the step (CUDA events on `stream`),
// for the roofline: ms_out[0..8] = state_zfwd, state_plane_density, rho_xc,
// vks_build (density FFT + Hartree/local + inverse), state_plane_vks,
// state_zbwd, pc_forward (S), pc_backward (two-term), ortho_ns.
static bool oz_ready(oa_ctx* c);
static cudaError_t mixed_fwd(oa_ctx* c, cudaStream_t s, int nt, const double* A, const double* B, int m, int n,
                             long K, long kx0_cols, double w_kx0, double alpha, double* C, int sa, int sb,
                             const int* cond = nullptr);
static cudaError_t mixed_bwd(oa_ctx* c, cudaStream_t s, int nt, const double* M1, const double* X1, double a1_kx0,
                             double a1_rest, const double* M2, const double* X2, double a2, int nj, int nk, long ncol,
                             long kx0_cols, double* out, int s1, int s2, const double* yadd = nullptr,
                             const int* cond = nullptr);

extern "C" oa_status oa_gpu_time_kernels(oa_ctx* c, void* stream, const double* psi, int reps, double* ms_out) {
  OA_ARG_CHECK(c && psi && ms_out && reps > 0, "bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  oa_ctx_pc* p = pcx(c);
  cudaEvent_t e0, e1;
  OA_CUDA_TRY(cudaEventCreate(&e0));
  OA_CUDA_TRY(cudaEventCreate(&e1));
  float ms = 0.f;
  double acc[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int n = c->nstate;
  double* S = p->mat_a;
  double* T = p->mat_x;
  const bool mixed = c->precision == OA_MIXED;
  // the second big operand of the timed products (F, or psi itself)
  double* F = (double*)p->vtmp;
  // an output of the same size: the z-line buffer (at least nstate x nz x
  // nlines complex in the compute precision, which covers nstate x 2 ng doubles)
  double* G = (double*)c->zbuf;
  const long K = 2L * c->ng, K0 = 2L * c->nkx0;
  for (int r = 0; r < reps; ++r) {
#define OA_TIME(slot, call)                                   \
    OA_CUDA_TRY(cudaEventRecord(e0, s));                      \
    OA_CUDA_TRY(call);                                        \
    OA_CUDA_TRY(cudaEventRecord(e1, s));                      \
    OA_CUDA_TRY(cudaEventSynchronize(e1));                    \
    OA_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));           \
    acc[slot] += ms;
    OA_TIME(0, oa_launch_state_zfwd(c, s, (const double2*)psi, 0, n));
    OA_TIME(1, oa_launch_state_plane_density(c, s));
    OA_TIME(2, oa_launch_rho_xc(c, s));
    OA_TIME(3, oa_launch_rho_fft_hart(c, s));
    OA_TIME(4, oa_launch_state_plane_vks(c, s));
    OA_TIME(5, oa_launch_state_zbwd(c, s, (const double2*)psi, nullptr, (double2*)p->vtmp, 0, n));
    OA_TIME(6, oa_launch_pc_fwd(s, psi, psi, n, K, K0, 0.5, 2.0, p->part, p->nkb, S));
    OA_CUDA_TRY(cudaMemcpyAsync(F, psi, (size_t)n * c->ng * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    if (mixed) {
      // the bf16 planes of psi and F are made by their producers in the
      // step: split them once, untimed, and reuse them (plane cache on)
      p->pl_cache = 1;
      p->pl_key[0].valid = p->pl_key[1].valid = false;
      OA_CUDA_TRY(mixed_bwd(c, s, 3, p->eye, psi, -0.5, -1.0, p->eye, F, 1.0, n, n, K, K0, G, 0, 1));
      OA_TIME(7, mixed_bwd(c, s, 3, p->eye, psi, -0.5, -1.0, p->eye, F, 1.0, n, n, K, K0, G, 0, 1));
      OA_TIME(10, mixed_fwd(c, s, 3, psi, F, n, n, K, K0, 1.0, 1.0, T, 0, 1));
      p->pl_cache = 0;
      p->pl_key[0].valid = p->pl_key[1].valid = p->pl_key[2].valid = false;
    } else {
      OA_TIME(7, oa_launch_pc_bwd(s, p->eye, psi, -0.5, -1.0, p->eye, F, 1.0, n, K, K0, G));
      OA_TIME(10, oa_launch_pc_fwd(s, psi, F, n, K, K0, 1.0, 1.0, p->part, p->nkb, T));
    }
    OA_TIME(8, oa_launch_ortho_ns(s, S, n, 0.5, 1e-15, 1000, p->ns_work, T, p->ns_status, p->ns_err,
                                  ns_launch_grid(p)));
    OA_TIME(9, oa_launch_pc_bwd(s, T, psi, 1.0, 1.0, nullptr, nullptr, 0.0, n, K, K0, G));
    if (mixed && oz_ready(c)) {
      // the int8 digit products of S and Psi T, beside the DMMA ones the step uses
      OA_TIME(11, oa_oz_overlap(p->oz, s, psi, K, 2.0, 0.5, S, p->err_flag, nullptr));
      OA_TIME(12, oa_oz_rotate(p->oz, s, T, psi, G, K, nullptr, p->err_flag, nullptr));
    }
#undef OA_TIME
  }
  for (int k = 0; k < 13; ++k) ms_out[k] = acc[k] / reps;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return OA_OK;
}

// Problem sizes a caller needs for byte/flop accounting: out[0..12] =
// nstate, ng, nlines, nz, ldl, ngroup, npts, compute-precision bytes per
// real, nlines_d, kernel launches per CP step of the host runner, state-pair
// plane kernels in use, their state groups, int8 overlap / rotation in use.
extern "C" oa_status oa_gpu_get_tuning(const oa_ctx* c, oa_tuning* t) {
  OA_ARG_CHECK(c && t, "null argument");
  const oa_ctx_pc* p = pcx(const_cast<oa_ctx*>(c));
  t->group_state = c->ngroup;
  t->group_pair = c->ngroup_pair;
  t->dgemm_kblocks = p->nkb;
  t->tgemm_kblocks = p->umax_kb;
  t->fft_path = c->fft_runtime ? 2 : 1;
  return OA_OK;
}

extern "C" oa_status oa_gpu_set_tuning(oa_ctx* c, const oa_tuning* t) {
  OA_ARG_CHECK(c && t, "null argument");
  oa_ctx_pc* p = pcx(c);
  const int npair = (c->nstate + 1) / 2;
  OA_ARG_CHECK(t->group_state >= 0 && t->group_state <= 32 && t->group_state <= c->nstate,
               "group_state must be 1..min(32, nstate) (0 keeps it)");
  OA_ARG_CHECK(t->group_pair >= 0 && t->group_pair <= 32 && t->group_pair <= npair,
               "group_pair must be 1..min(32, state pairs) (0 keeps it)");
  OA_ARG_CHECK(t->dgemm_kblocks == 0 || (t->dgemm_kblocks >= 2 && t->dgemm_kblocks <= p->nkb_cap),
               "dgemm_kblocks must be 2..160 (0 keeps it)");
  OA_ARG_CHECK(t->tgemm_kblocks >= 0 && t->tgemm_kblocks <= p->umax_cap,
               "tgemm_kblocks above the split-K partials allocated at init");
  OA_ARG_CHECK(t->fft_path >= 0 && t->fft_path <= 2, "fft_path must be 1 or 2 (0 keeps it)");
  if (t->fft_path == 2 && c->precision == OA_MIXED) {
    oa_set_error("fft_path 2: the mixed form's state-pair kernels need the two-pass transforms", __FILE__, __LINE__);
    return OA_ERR_UNSUPPORTED;
  }
  const int gs = t->group_state ? t->group_state : c->ngroup;
  const int gp = t->group_pair ? t->group_pair : c->ngroup_pair;
  const int need = gs > gp ? gs : gp;
  if (need > c->rho_groups_cap || (c->pair_cols && gp * c->nz > c->nq2_cap)) {
    OA_CUDA_TRY(cudaDeviceSynchronize());
    if (need > c->rho_groups_cap) {
      double* r = nullptr;
      OA_CUDA_TRY(cudaMalloc(&r, (size_t)need * c->npts * sizeof(double)));
      cudaFree(c->rho_part);
      c->rho_part = r;
      c->rho_groups_cap = need;
    }
    if (c->pair_cols && gp * c->nz > c->nq2_cap) {
      double* q = nullptr;
      OA_CUDA_TRY(cudaMalloc(&q, (size_t)gp * c->nz * sizeof(double)));
      cudaFree(c->qpart2);
      c->qpart2 = q;
      c->nq2_cap = gp * c->nz;
    }
  }
  c->ngroup = gs;
  c->ngroup_pair = gp;
  if (c->pair_cols) c->nq2 = gp * c->nz;
  if (t->dgemm_kblocks) p->nkb = t->dgemm_kblocks;
  if (t->tgemm_kblocks) p->umax_kb = t->tgemm_kblocks;
  if (t->fft_path) c->fft_runtime = t->fft_path == 2 ? 1 : 0;
  c->rho_ngroup = c->ngroup;
  c->psir_valid = 0;
  c->qvalid = 0;
  c->xc_gen += 1;  // the captured step is re-made with the new launch shapes
  return OA_OK;
}

extern "C" oa_status oa_gpu_sizes(const oa_ctx* c, long* out) {
  OA_ARG_CHECK(c && out, "null argument");
  out[0] = c->nstate; out[1] = c->ng; out[2] = c->nlines; out[3] = c->nz; out[4] = c->ldl;
  out[5] = c->ngroup; out[6] = c->npts; out[7] = c->precision == OA_FP64 ? 8 : 4; out[8] = c->nlines_d;
  // kernels of the FP64 oa_gpu_cp_step (an estimate; oa_cp_state.last_kernels counts the
  // graphed step): state_fft_fwd 3 + vks_build 5 + nl_sf 7 + vks_apply 4 + lambda 4 +
  // integrate 3 + S 2 + Newton-Schulz 1 + Psi T 1
  out[9] = 3 + 5 + 7 + 4 + 4 + 3 + 2 + 1 + 1;
  out[10] = c->pair_cols ? 1 : 0;  // state-pair plane kernels in use (mixed form)
  out[11] = c->ngroup_pair;
  out[12] = (c->precision == OA_MIXED && c->nstate <= 128) ? 1 : 0;  // int8 overlap / rotation available
  return OA_OK;
}

typedef __nv_bfloat16 bf16;

// Plane slots of the big operands: the state coefficients, the force or
// second operand, the nonlocal structure factor.
enum { PL_PSI = 0, PL_OTHER = 1, PL_SF = 2 };

// bf16 planes of X [rows][K] (kx0 columns weighted) in a big slot.  Inside a
// native step (pl_cache set) a slot that already holds the same source with
// the same weighting is reused; the step clears the slots whenever the
// sources may have changed.
static cudaError_t ensure_planes(oa_ctx* c, cudaStream_t s, int nt, int slot, const double* X, int rows,
                                 int rows_pad, long K, long kx0_cols, double w_kx0, const int* cond = nullptr) {
  oa_ctx_pc* p = pcx(c);
  if (kx0_cols == 0) w_kx0 = 1.0;
  if (w_kx0 == 1.0) kx0_cols = 0;
  auto& k = p->pl_key[slot];
  if (p->pl_cache && k.valid && k.src == X && k.rows == rows && k.rows_pad == rows_pad && k.nt == nt && k.K == K &&
      k.kx0 == kx0_cols && k.w == w_kx0)
    return cudaSuccess;
  const cudaError_t e =
      oa_split_kc(s, nt, X, rows, rows_pad, K, K, kx0_cols, w_kx0, (bf16*)p->pl_big[slot], p->pl_ld, cond);
  k.src = X; k.rows = rows; k.rows_pad = rows_pad; k.nt = nt; k.K = K; k.kx0 = kx0_cols; k.w = w_kx0;
  k.valid = e == cudaSuccess;
  return e;
}

// Plane reuse inside a native step.  The keys say which FP64 source each
// slot holds planes of; inside a step (pl_cache on) a slot whose key matches
// is not split again.  The psi slot stays valid from step to step: psi
// changes only in Psi T, which writes its planes in the same pass (or at the
// start of a run, oa_planes_psi_refresh).  The other slots are forgotten at
// both ends of a step (their sources change inside it, and a split gated by
// the PsiV flag may not have run).
void oa_planes_step_begin(oa_ctx* c) {
  oa_ctx_pc* p = pcx(c);
  p->pl_cache = 1;
  for (int q = 0; q < 3; ++q)
    if (q != PL_PSI) p->pl_key[q].valid = false;
}
void oa_planes_step_end(oa_ctx* c) {
  oa_ctx_pc* p = pcx(c);
  p->pl_cache = 0;
  for (int q = 0; q < 3; ++q)
    if (q != PL_PSI) p->pl_key[q].valid = false;
}

// slot as the target of a fused plane write of an [rows][2 ng] operand, with
// the padded row count the GEMMs use for it
static bool plane_out(oa_ctx* c, int slot, int rows, int nt, OaPlaneOut* po) {
  oa_ctx_pc* p = pcx(c);
  const int nb = oa_tg_nb(rows);
  if (!p->pl_big[slot] || nb == 0 || !(nt == 2 || nt == 3)) return false;
  const int rp = oa_tg_rows_pad(rows, nb);
  if (rp > p->pl_rows || 2L * c->ng > p->pl_ld) return false;
  *po = OaPlaneOut{p->pl_big[slot], rp, p->pl_ld, nt};
  return true;
}
static void plane_mark(oa_ctx* c, int slot, const double* src, int rows, int rows_pad, int nt) {
  auto& k = pcx(c)->pl_key[slot];
  k.src = src; k.rows = rows; k.rows_pad = rows_pad; k.nt = nt; k.K = 2L * c->ng; k.kx0 = 0; k.w = 1.0;
  k.valid = true;
}

// the next force z pass (oa_launch_state_zbwd) also writes the planes of F
void oa_planes_force_begin(oa_ctx* c, int nt) {
  OaPlaneOut po;
  c->zb_po = plane_out(c, PL_OTHER, c->nstate, nt, &po) ? po : OaPlaneOut{nullptr, 0, 0, 0};
}
void oa_planes_force_end(oa_ctx* c, const double* F) {
  if (c->zb_po.P && c->zb_po_done) plane_mark(c, PL_OTHER, F, c->nstate, c->zb_po.rows_pad, c->zb_po.nt);
  c->zb_po = OaPlaneOut{nullptr, 0, 0, 0};
  c->zb_po_done = 0;
}

// psi planes split afresh (start of a native run)
oa_status oa_planes_psi_refresh(oa_ctx* c, cudaStream_t s, const double* psi, int nt) {
  OaPlaneOut po;
  if (!plane_out(c, PL_PSI, c->nstate, nt, &po)) {
    // no fused psi planes at this size: whatever the slot holds is stale
    pcx(c)->pl_key[PL_PSI].valid = false;
    return OA_OK;
  }
  OA_CUDA_TRY(oa_split_kc(s, nt, psi, c->nstate, po.rows_pad, 2L * c->ng, 2L * c->ng, 0, 1.0, (bf16*)po.P, po.ldp));
  plane_mark(c, PL_PSI, psi, c->nstate, po.rows_pad, nt);
  return OA_OK;
}

// Split-BF16 forward product through bf16 planes (oa_tgemm.cu); the
// element-wise-staging kernels (oa_umma.cu) for shapes the planes path does
// not take.  A: [m][K] (kx0 columns weighted by w_kx0), B: [n][K], in
// plane slots sa and sb.
static cudaError_t mixed_fwd(oa_ctx* c, cudaStream_t s, int nt, const double* A, const double* B, int m, int n,
                             long K, long kx0_cols, double w_kx0, double alpha, double* C, int sa, int sb,
                             const int* cond) {
  oa_ctx_pc* p = pcx(c);
  const int mx = c->nstate > c->natm_nl ? c->nstate : c->natm_nl;
  const int nb = oa_tg_nb_fwd(n);
  const int ra = oa_tg_rows_pad(m, 128), rb = nb ? oa_tg_rows_pad(n, nb) : 0;
  if (nb && m <= mx && n <= mx && K <= p->pl_ld && ra <= p->pl_rows && rb <= p->pl_rows) {
    const bool same = B == A && (w_kx0 == 1.0 || kx0_cols == 0) && ra % nb == 0;
    cudaError_t e = ensure_planes(c, s, nt, sa, A, m, ra, K, kx0_cols, w_kx0, cond);
    if (e != cudaSuccess) return e;
    const bf16* pb = (const bf16*)p->pl_big[sa];
    int rows_b = ra;
    if (!same) {
      if ((e = ensure_planes(c, s, nt, sb, B, n, rb, K, 0, 1.0, cond)) != cudaSuccess) return e;
      pb = (const bf16*)p->pl_big[sb];
      rows_b = rb;
    }
    e = oa_tfwd(s, nt, (const bf16*)p->pl_big[sa], ra, pb, rows_b, m, n, K, p->pl_ld, alpha, p->upart, p->umax_kb, C,
                p->err_flag, p->nsm, cond);
    if (e != cudaErrorNotSupported) return e;
  }
  if (cond) return cudaErrorNotSupported;  // the fallback kernels have no device flag
  return oa_launch_umma_fwd(s, nt, A, B, m, n, K, kx0_cols, w_kx0, alpha, p->upart, p->umax_kb, C, p->err_flag,
                            p->nsm);
}

// Split-BF16 backward product through bf16 planes, with the same fallback;
// X1, X2 in plane slots s1, s2.
static cudaError_t mixed_bwd(oa_ctx* c, cudaStream_t s, int nt, const double* M1, const double* X1, double a1_kx0,
                             double a1_rest, const double* M2, const double* X2, double a2, int nj, int nk, long ncol,
                             long kx0_cols, double* out, int s1, int s2, const double* yadd,
                             const int* cond) {
  oa_ctx_pc* p = pcx(c);
  const int mx = c->nstate > c->natm_nl ? c->nstate : c->natm_nl;
  int nkp = oa_tg_rows_pad(nk, 32);
  {
    // planes of X1 already held with more zero rows (a multiple of 32) serve as they are
    const auto& k = p->pl_key[s1];
    if (p->pl_cache && k.valid && k.src == X1 && k.rows == nk && k.nt == nt && k.K == ncol && k.kx0 == 0 &&
        k.rows_pad > nkp && k.rows_pad % 32 == 0 && k.rows_pad <= p->pl_rows)
      nkp = k.rows_pad;
  }
  const int ldm = oa_tg_nb(nj);  // M planes: leading size of the N tile, zero beyond nj
  if (nj <= mx && nk <= mx && ncol <= p->pl_ld && ldm != 0 && nkp <= p->pl_rows && (!M2 || s1 != s2)) {
    bf16 *pm1 = (bf16*)p->pl_ma, *pm2 = (bf16*)p->pl_mb;
    cudaError_t e = ensure_planes(c, s, nt, s1, X1, nk, nkp, ncol, 0, 1.0, cond);
    if (e == cudaSuccess) e = oa_split_kc(s, nt, M1, nk, nkp, nj, nj, 0, 1.0, pm1, ldm, cond);
    if (e == cudaSuccess && M2) e = ensure_planes(c, s, nt, s2, X2, nk, nkp, ncol, 0, 1.0, cond);
    if (e == cudaSuccess && M2) e = oa_split_kc(s, nt, M2, nk, nkp, nj, nj, 0, 1.0, pm2, ldm, cond);
    if (e != cudaSuccess) return e;
    e = oa_tbwd(s, nt, pm1, (const bf16*)p->pl_big[s1], a1_kx0, a1_rest, M2 ? pm2 : nullptr,
                M2 ? (const bf16*)p->pl_big[s2] : nullptr, a2, nj, nkp, ncol, p->pl_ld, kx0_cols, out, p->err_flag,
                yadd, cond);
    if (e != cudaErrorNotSupported) return e;
  }
  if (cond || yadd) return cudaErrorNotSupported;  // the fallback kernels have neither
  return oa_launch_umma_bwd(s, nt, M1, X1, a1_kx0, a1_rest, M2, X2, a2, nj, nk, ncol, kx0_cols, out, p->err_flag);
}

// v = sign psi / dt under the device flag (and everywhere when cond is
// null): the two halves of finiteDifferencePsiV's v = (psi(t) - psi(t-dt)) / dt
// around the rotation that overwrites psi(t - dt) with psi(t)
__global__ void __launch_bounds__(256) k_fd_velocity(const double2* __restrict__ psi, double2* __restrict__ v,
                                                     size_t n, double scale, int accumulate,
                                                     const int* __restrict__ cond) {
  if (cond && *cond == 0) return;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double2 p = psi[i];
    double2 r = make_double2(p.x * scale, p.y * scale);
    if (accumulate) {
      const double2 o = v[i];
      r.x += o.x;
      r.y += o.y;
    }
    v[i] = r;
  }
}

static cudaError_t fd_velocity(oa_ctx* c, cudaStream_t s, const double* psi, double* vpsi, double scale,
                               int accumulate, const int* cond) {
  const size_t n = (size_t)c->nstate * c->ng;
  k_fd_velocity<<<8 * 148, 256, 0, s>>>((const double2*)psi, (double2*)vpsi, n, scale, accumulate, cond);
  return cudaGetLastError();
}

// psi = psi_t T and, under the device flag, the PsiV reset of the
// reference's default build (finiteDifferencePsiV,
// CP_State_GSpacePlane.C:3741-3800, norb_fin_diff_order 0):
// v = (psi(t) - psi(t - dt)) / dt from the psi the rotation overwrites, and
// T = I.  psi_t = psi is left to the next integration (which reads psi
// under the flag, and then completes no half kick) or to oa_psi_t_settle.
oa_status oa_psi_t_and_psiv(oa_ctx* c, cudaStream_t s, const double* T, double* psi_t, double* psi, double* vpsi,
                            double* Tout, int* flag, int nterm, double dt) {
  oa_ctx_pc* p = pcx(c);
  const int n = c->nstate;
  OaPlaneOut po;
  bool fuse = nterm > 0 && plane_out(c, PL_PSI, n, nterm, &po);
  // the rotation's epilogue writes the velocity under the flag from the psi
  // it overwrites (no separate passes)
  cudaError_t e = oa_dgemm_bwd_ex(s, T, psi_t, 1.0, 1.0, nullptr, nullptr, 0.0, n, n, 2L * c->ng, 2L * c->nkx0, psi,
                                  nullptr, nullptr, nullptr, nullptr, fuse ? &po : nullptr, vpsi, 1.0 / dt, flag);
  if (e == cudaErrorNotSupported) {
    // shapes the tiled kernel does not take: the general kernel, and the psi
    // planes are split again when a product needs them; the velocity in two
    // passes around it
    OA_CUDA_TRY(fd_velocity(c, s, psi, vpsi, -1.0 / dt, 0, flag));
    e = oa_launch_pc_bwd(s, T, psi_t, 1.0, 1.0, nullptr, nullptr, 0.0, n, 2L * c->ng, 2L * c->nkx0, psi);
    OA_CUDA_TRY(e);
    OA_CUDA_TRY(fd_velocity(c, s, psi, vpsi, 1.0 / dt, 1, flag));
    fuse = false;
  } else {
    OA_ALIGN_TRY(e);
  }
  // psi changed: its planes are current only when this pass wrote them (the
  // nonlocal products split psi again otherwise)
  if (fuse) plane_mark(c, PL_PSI, psi, n, po.rows_pad, nterm);
  else pcx(c)->pl_key[PL_PSI].valid = false;
  k_copy_cond<<<16, 256, 0, s>>>(Tout, p->eye, (size_t)n * n, flag);
  OA_CUDA_TRY(cudaGetLastError());
  return OA_OK;
}

// psi_t = psi when the last step's PsiV flag is set: the native steps leave
// that copy to the next integration (which reads psi under the flag), so a
// run ends with it
// dst = src (n 16-byte pieces) when *cond != 0; four pieces in flight per thread
__global__ void __launch_bounds__(256) k_copy_cond16(uint4* __restrict__ dst, const uint4* __restrict__ src, size_t n,
                                                     const int* __restrict__ cond) {
  if (*cond == 0) return;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    uint4 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = __ldcs(src + i + u * stride);
#pragma unroll
    for (int u = 0; u < 4; ++u) __stcs(dst + i + u * stride, v[u]);
  }
  for (; i < n; i += stride) __stcs(dst + i, __ldcs(src + i));
}

oa_status oa_psi_t_settle(oa_ctx* c, cudaStream_t s, const double* psi, double* psi_t, const int* flag) {
  const size_t n = (size_t)c->nstate * c->ng;  // double2 coefficients
  if ((((uintptr_t)psi | (uintptr_t)psi_t) & 15) == 0)
    k_copy_cond16<<<8 * 148, 256, 0, s>>>((uint4*)psi_t, (const uint4*)psi, n, flag);
  else
    k_copy_cond<<<8 * 148, 256, 0, s>>>(psi_t, psi, 2 * n, flag);
  OA_CUDA_TRY(cudaGetLastError());
  return OA_OK;
}

extern "C" oa_status oa_gpu_psiv_reset(oa_ctx* c, void* stream, const double* psi, const double* psi_prev,
                                       double* psi_t, double* vpsi, double dt) {
  OA_ARG_CHECK(c && psi && psi_prev && psi_t && vpsi && dt > 0.0, "null argument or dt <= 0");
  cudaStream_t s = (cudaStream_t)stream;
  OA_CUDA_TRY(fd_velocity(c, s, psi_prev, vpsi, -1.0 / dt, 0, nullptr));
  OA_CUDA_TRY(fd_velocity(c, s, psi, vpsi, 1.0 / dt, 1, nullptr));
  const size_t bytes = (size_t)c->nstate * c->ng * sizeof(double2);
  OA_CUDA_TRY(cudaMemcpyAsync(psi_t, psi, bytes, cudaMemcpyDeviceToDevice, s));
  return OA_OK;
}

extern "C" oa_status oa_gpu_pc_forward_mixed(oa_ctx* c, void* stream, const double* left, const double* right,
                                             double alpha, double w_kx0, int nterm, double* C) {
  OA_ARG_CHECK(c && left && right && C, "null argument");
  OA_ARG_CHECK(nterm == 2 || nterm == 3, "nterm must be 2 or 3");
  oa_ctx_pc* p = pcx(c);
  (void)p;
  OA_CUDA_TRY(mixed_fwd(c, (cudaStream_t)stream, nterm, left, right, c->nstate, c->nstate, 2L * c->ng, 2L * c->nkx0,
                        w_kx0, alpha, C, PL_PSI, PL_OTHER));
  return OA_OK;
}

extern "C" oa_status oa_gpu_pc_backward_mixed(oa_ctx* c, void* stream, const double* M1, const double* X1,
                                              double a1_kx0, double a1_rest, const double* M2, const double* X2,
                                              double a2, int nterm, double* out) {
  OA_ARG_CHECK(c && M1 && X1 && out, "null argument");
  OA_ARG_CHECK((M2 == nullptr) == (X2 == nullptr), "M2 and X2 must both be given or both be NULL");
  OA_ARG_CHECK(out != X1 && out != X2, "out must not alias an input");
  OA_ARG_CHECK(nterm == 2 || nterm == 3, "nterm must be 2 or 3");
  OA_CUDA_TRY(mixed_bwd(c, (cudaStream_t)stream, nterm, M1, X1, a1_kx0, a1_rest, M2, X2, a2, c->nstate, c->nstate,
                        2L * c->ng, 2L * c->nkx0, out, PL_PSI, PL_OTHER));
  return OA_OK;
}

extern "C" oa_status oa_gpu_check(oa_ctx* c, void* stream) {
  OA_ARG_CHECK(c, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  oa_ctx_pc* p = pcx(c);
  OA_CUDA_TRY(cudaMemcpyAsync(p->h_status + 2, p->err_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaStreamSynchronize(s));
  if (p->h_status[2]) {
    // reported once: the flag is cleared for the calls that follow
    OA_CUDA_TRY(cudaMemsetAsync(p->err_flag, 0, sizeof(int), s));
    OA_CUDA_TRY(cudaStreamSynchronize(s));
    oa_set_error("a device wait ran out of time (200 ms) in a tcgen05 product; its output is zero", __FILE__,
                 __LINE__);
    return OA_ERR_CUDA;
  }
  return OA_OK;
}

extern "C" oa_status oa_gpu_nl_sf(oa_ctx* c, void* stream, const double* psi, int nterm, double* fnl_out,
                                  double* enl_out) {
  OA_ARG_CHECK(c && psi && fnl_out, "null argument");
  OA_ARG_CHECK(nterm == 0 || nterm == 2 || nterm == 3, "nterm must be 0, 2 or 3");
  cudaStream_t s = (cudaStream_t)stream;
  oa_ctx_pc* p = pcx(c);
  const int n = c->nstate, na = c->natm_nl;
  if (na == 0) {
    OA_CUDA_TRY(cudaMemsetAsync(fnl_out, 0, (size_t)n * c->ng * sizeof(double2), s));
    OA_CUDA_TRY(cudaMemsetAsync(p->dev_e + OA_E_ENL, 0, sizeof(double), s));
    if (enl_out) OA_CUDA_TRY(cudaMemsetAsync(enl_out, 0, (size_t)n * sizeof(double), s));
    return OA_OK;
  }
  const double tpi_l = 2.0 * M_PI / c->box;
  // inside a native step the phase tables are this step's (vks_build made
  // them from the same positions), and the SF kernel also writes its planes
  if (!p->pl_cache) OA_CUDA_TRY(oa_launch_phase_tables(c, s));
  OaPlaneOut po;
  const bool fuse = nterm > 0 && p->pl_cache && plane_out(c, PL_SF, na, nterm, &po);
  OA_CUDA_TRY(oa_launch_nl_sf(s, c->kx, c->ky, c->kz, c->ng, c->nl_atm, na, c->atm_type, c->phase, c->kmax_tab,
                              c->nl_spl, c->nspl, c->spl_gmin, c->spl_dg, c->nl_gz0, tpi_l, c->sf,
                              fuse ? &po : nullptr));
  if (fuse) plane_mark(c, PL_SF, (const double*)c->sf, na, po.rows_pad, nterm);
  const long K = 2L * c->ng;
  if (nterm == 0)
    OA_CUDA_TRY(oa_launch_pc_fwd_mn(s, psi, (const double*)c->sf, n, na, K, 0, 1.0, 1.0, p->part, p->nkb, c->zmat));
  else
    OA_CUDA_TRY(mixed_fwd(c, s, nterm, psi, (const double*)c->sf, n, na, K, 0, 1.0, 1.0, c->zmat, PL_PSI, PL_SF));
  OA_CUDA_TRY(oa_launch_nl_zscale(s, c->zmat, n, na, c->nl_atm, c->atm_type, c->nl_vnorm, 1.0 / c->vol, c->occ,
                                  c->zt, c->enl));
  if (nterm == 0)
    OA_CUDA_TRY(oa_launch_pc_bwd_jk(s, c->zt, (const double*)c->sf, 1.0, 1.0, nullptr, nullptr, 0.0, n, na, K, 0,
                                    fnl_out));
  else
    OA_CUDA_TRY(mixed_bwd(c, s, nterm, c->zt, (const double*)c->sf, 1.0, 1.0, nullptr, nullptr, 0.0, n, na, K, 0,
                          fnl_out, PL_SF, PL_OTHER));
  OA_CUDA_TRY(oa_launch_sum_partials(s, c->enl, n, 1, 0, 1.0, p->dev_e + OA_E_ENL));
  if (enl_out) OA_CUDA_TRY(cudaMemcpyAsync(enl_out, c->enl, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // ion dynamics: the nonlocal atom forces from the same Z
  if (c->ions) OA_CUDA_TRY(oa_launch_nl_sf_force(c, s, psi));
  return OA_OK;
}

cudaError_t oa_step_ortho_args(oa_ctx* c, double** work, int** status, double** errv, int* grid, double** dev_e,
                               int** h_status, double** h_vals, double** eye) {
  oa_ctx_pc* p = pcx(c);
  *work = p->ns_work; *status = p->ns_status; *errv = p->ns_err; *grid = ns_launch_grid(p); *dev_e = p->dev_e;
  *h_status = p->h_status; *h_vals = p->h_vals; *eye = p->eye;
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// EES nonlocal path
// ---------------------------------------------------------------------------
static void ees_free(oa_ctx* c) {
  oa_ees* e = c->ees;
  if (!e) return;
  void* dev[] = {e->tw_a, e->tw_b, e->tw_c, e->zbuf, e->dyp, e->idx, e->mn, e->zpart, e->zmat, e->zs, e->enl,
                 e->dmn, e->fpart};
  for (void* q : dev) if (q) cudaFree(q);
  free(e);
  c->ees = nullptr;
}

int oa_plane_blocks_per_sm(int precision);

extern "C" oa_status oa_gpu_ees_init(oa_ctx* c, int na, int nb, int nc, int order, const double* dyp_host) {
  OA_ARG_CHECK(c && dyp_host, "null argument");
  OA_ARG_CHECK(order >= 4 && order <= 16 && order % 2 == 0, "EES order must be even, 4..16 (cp_pseudo_ees_order)");
  OA_ARG_CHECK(na >= order && nb >= order && nc >= order, "EES grid smaller than the interpolation order");
  OA_ARG_CHECK(c->natm_nl > 0, "no nonlocal atoms");
  ees_free(c);
  oa_ees* e = (oa_ees*)calloc(1, sizeof(oa_ees));
  if (!e) return OA_ERR_CUDA;
  c->ees = e;
  e->na = na; e->nb = nb; e->nc = nc; e->order = order;
  if (!make_plan(na, &e->pa) || !make_plan(nb, &e->pb) || !make_plan(nc, &e->pc)) {
    ees_free(c);
    oa_set_error("EES grid size must be 2^a 3^b 5^c with at least two radix stages", __FILE__, __LINE__);
    return OA_ERR_UNSUPPORTED;
  }
  int mkx = 0, mky = 0, mkz = 0;
  (void)mky; (void)mkz;
  mkx = c->nkx_s - 1;
  if (2 * mkx + 1 > na) { ees_free(c); oa_set_error("EES grid too small for the state sphere", __FILE__, __LINE__); return OA_ERR_BAD_ARG; }
  const size_t smem = oa_plane_smem_bytes(c->precision, na, nb, c->nkx_s);
  if (smem > OA_MAX_SMEM) { ees_free(c); oa_set_error("EES grid too large for the plane kernel", __FILE__, __LINE__); return OA_ERR_UNSUPPORTED; }
  int bps = (int)(228 * 1024 / (smem + 1024));
  const int occ_bps = oa_plane_blocks_per_sm(c->precision);
  if (occ_bps > 0 && occ_bps < bps) bps = occ_bps;
  if (bps < 1) bps = 1;
  e->ngroup = pick_groups(nc, c->nstate, bps, pcx(c)->nsm);
  cudaError_t err = cudaSuccess;
  const size_t csz = c->precision == OA_FP64 ? sizeof(double2) : sizeof(float2);
#define TRYE(x) do { err = (x); if (err != cudaSuccess) { ees_free(c); oa_set_error(cudaGetErrorString(err), __FILE__, __LINE__); return OA_ERR_CUDA; } } while (0)
  e->tw_a = make_twiddles(na);
  e->tw_b = make_twiddles(nb);
  e->tw_c = make_twiddles(nc);
  if (!e->tw_a || !e->tw_b || !e->tw_c) { ees_free(c); oa_set_error("twiddle allocation failed", __FILE__, __LINE__); return OA_ERR_CUDA; }
  TRYE(cudaMalloc(&e->zbuf, (size_t)c->nstate * nc * c->ldl * csz));
  TRYE(upload(&e->dyp, (const double2*)dyp_host, (size_t)c->ng));
  TRYE(cudaMalloc(&e->idx, (size_t)c->natm_nl * 3 * order * sizeof(int)));
  TRYE(cudaMalloc(&e->mn, (size_t)c->natm_nl * 3 * order * sizeof(double)));
  TRYE(cudaMalloc(&e->zpart, (size_t)c->nstate * c->natm_nl * order * sizeof(double)));
  TRYE(cudaMalloc(&e->zmat, (size_t)c->nstate * c->natm_nl * sizeof(double)));
  TRYE(cudaMalloc(&e->zs, (size_t)c->nstate * c->natm_nl * sizeof(double)));
  TRYE(cudaMalloc(&e->enl, (size_t)c->nstate * sizeof(double)));
  TRYE(cudaMalloc(&e->dmn, (size_t)c->natm_nl * 3 * order * sizeof(double)));
  TRYE(cudaMalloc(&e->fpart, (size_t)c->nstate * c->natm_nl * order * 3 * sizeof(double)));
#undef TRYE
  return OA_OK;
}

// get_bspline_wght1d (set_cp_ewald.C:1237-1325): for m = 0..ngrid-1
// b(m) = exp(2 pi i (n-1) m / K) / sum_{k=1}^{n-1} M_n(k) exp(2 pi i m (k-1) / K),
// M_n at the integers by the cardinal B-spline recursion from M_2.
static std::vector<double2> bspline_factor_1d(int order, int ngrid) {
  std::vector<double> mn(order + 1, 0.0), uk(order + 1, 0.0);
  mn[1] = 1.0;
  for (int k = 1; k <= order; ++k) uk[k] = (double)k;
  for (int n = 3; n <= order; ++n) {
    for (int k = n; k >= 2; --k) mn[k] = (uk[k] * mn[k] + ((double)n - uk[k]) * mn[k - 1]) / (double)(n - 1);
    mn[1] = uk[1] * mn[1] / (double)(n - 1);
  }
  std::vector<double2> b(ngrid);
  for (int m = 0; m < ngrid; ++m) {
    double dr = 0.0, di = 0.0;
    for (int k = 1; k < order; ++k) {
      const double a = 2.0 * M_PI * (double)m * (double)(k - 1) / (double)ngrid;
      dr += cos(a) * mn[k];
      di += sin(a) * mn[k];
    }
    const double an = 2.0 * M_PI * (double)(order - 1) * (double)m / (double)ngrid;
    const double nr = cos(an), ni = sin(an);
    const double den = dr * dr + di * di;
    b[m] = make_double2((nr * dr + ni * di) / den, (ni * dr - nr * di) / den);
  }
  return b;
}

extern "C" oa_status oa_gpu_set_ees_local(oa_ctx* c, int na, int nb, int nc, int order) {
  OA_ARG_CHECK(c, "null context");
  if (na == 0 && nb == 0 && nc == 0) {
    oa_eesl_free(c);
    c->eesl_gen++;
    return OA_OK;
  }
  OA_ARG_CHECK(order >= 4 && order <= 16 && order % 2 == 0, "EES order must be even, 4..16 (cp_pseudo_ees_order)");
  OA_ARG_CHECK(na >= order && nb >= order && nc >= order, "EES grid smaller than the interpolation order");
  OA_ARG_CHECK(na > 2 * c->kmax_tab && nb > 2 * c->kmax_tab && nc > 2 * c->kmax_tab,
               "EES local grid too small for the density sphere (n > 2 kmax_rho)");
  OaFftPlan pa, pb, pc;
  if (!make_plan(na, &pa) || !make_plan(nb, &pb) || !make_plan(nc, &pc)) {
    oa_set_error("EES grid size must be 2^a 3^b 5^c with at least two radix stages and <= 512", __FILE__, __LINE__);
    return OA_ERR_UNSUPPORTED;
  }
  oa_eesl_free(c);
  c->eesl_gen++;
  oa_eesl* L = (oa_eesl*)calloc(1, sizeof(oa_eesl));
  if (!L) return OA_ERR_CUDA;
  c->eesl = L;
  L->na = na; L->nb = nb; L->nc = nc; L->order = order;
  L->ngrid = (c->ntype + 1) / 2;
  L->pa = pa; L->pb = pb; L->pc = pc;
  cudaError_t err = cudaSuccess;
#define TRYL(x) do { err = (x); if (err != cudaSuccess) { oa_eesl_free(c); oa_set_error(cudaGetErrorString(err), __FILE__, __LINE__); return OA_ERR_CUDA; } } while (0)
  L->tw_a = make_twiddles(na);
  L->tw_b = make_twiddles(nb);
  L->tw_c = make_twiddles(nc);
  if (!L->tw_a || !L->tw_b || !L->tw_c) { oa_eesl_free(c); oa_set_error("twiddle allocation failed", __FILE__, __LINE__); return OA_ERR_CUDA; }
  const std::vector<double2> ba = bspline_factor_1d(order, na), bb = bspline_factor_1d(order, nb),
                             bc = bspline_factor_1d(order, nc);
  TRYL(upload(&L->ba, ba.data(), ba.size()));
  TRYL(upload(&L->bb, bb.data(), bb.size()));
  TRYL(upload(&L->bc, bc.data(), bc.size()));
  TRYL(upload(&L->gzvps, c->gzvps_t, (size_t)c->ntype));
  const size_t gbytes = (size_t)L->ngrid * na * nb * nc * sizeof(double2);
  TRYL(cudaMalloc(&L->zq, gbytes));
  TRYL(cudaMalloc(&L->zy, gbytes));
#undef TRYL
  return OA_OK;
}

extern "C" oa_status oa_gpu_nl_ees(oa_ctx* c, void* stream, const double* psi, double* fnl_out, double* enl_out) {
  OA_ARG_CHECK(c && psi && fnl_out, "null argument");
  if (!c->ees) { oa_set_error("oa_gpu_ees_init has not been called", __FILE__, __LINE__); return OA_ERR_BAD_ARG; }
  cudaStream_t s = (cudaStream_t)stream;
  oa_ees* e = c->ees;
  OA_CUDA_TRY(oa_launch_ees_bspline(c, s));
  OA_CUDA_TRY(oa_launch_ees(c, s, (const double2*)psi, (double2*)fnl_out));
  OA_CUDA_TRY(oa_launch_sum_partials(s, e->enl, c->nstate, 1, 0, 1.0, pcx(c)->dev_e + OA_E_ENL));
  if (enl_out) OA_CUDA_TRY(cudaMemcpyAsync(enl_out, e->enl, (size_t)c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, s));
  return OA_OK;
}
