// One whole CP dynamics step in native code: the sequence of
// GSpaceDriver::computeDynamics (src_charm_driver/cp_state_ctrl/gspace.ci:199-324)
// on one GPU, with a single host synchronisation at the end of the step
// (energies, Newton-Schulz status, max|S - 2I|).  The steady-state step
// (iteration > 1, fixed buffers) is captured once into two CUDA graphs
// (forces .. S, and Psi T + the record copies) replayed around the
// cooperative Newton-Schulz launch, which stream capture does not accept;
// a PsiV tolerance reset decided at the end of a step runs eagerly at the
// start of the next one.
#include <string.h>
#include "oa_internal.h"

// entry points of oa_abi.cu used here
extern "C" {
oa_status oa_gpu_state_fft_fwd(oa_ctx* ctx, void* stream, const double* psi, double* rho_out);
oa_status oa_gpu_vks_build(oa_ctx* ctx, void* stream, double* vks_out);
oa_status oa_gpu_nl_sf(oa_ctx* ctx, void* stream, const double* psi, int nterm, double* fnl_out, double* enl_out);
oa_status oa_gpu_vks_apply_fft_bwd(oa_ctx* ctx, void* stream, const double* psi, int recompute_fwd,
                                   const double* fnl, double* force, double* eke_out);
oa_status oa_gpu_pc_forward(oa_ctx* ctx, void* stream, const double* left, const double* right, double alpha,
                            double w_kx0, double* C);
oa_status oa_gpu_pc_forward_mixed(oa_ctx* ctx, void* stream, const double* left, const double* right, double alpha,
                                  double w_kx0, int nterm, double* C);
oa_status oa_gpu_pc_backward(oa_ctx* ctx, void* stream, const double* M1, const double* X1, double a1_kx0,
                             double a1_rest, const double* M2, const double* X2, double a2, double* out);
oa_status oa_gpu_pc_backward_mixed(oa_ctx* ctx, void* stream, const double* M1, const double* X1, double a1_kx0,
                                   double a1_rest, const double* M2, const double* X2, double a2, int nterm,
                                   double* out);
oa_status oa_gpu_small_gemm(oa_ctx* ctx, void* stream, const double* A, const double* B, double alpha, double* C);
oa_status oa_gpu_integrate(oa_ctx* ctx, void* stream, const double* force, double* vpsi, double* psi, double dt,
                           int complete_prev, double* fict_ke_out);
oa_status oa_gpu_psiv_reset(oa_ctx* ctx, void* stream, const double* psi, double* psi_t, double* vpsi);
}

cudaError_t oa_launch_ortho_ns(cudaStream_t s, const double* S, int n, double bscale, double tol, int max_iter,
                               double* work, double* T, int* status, double* errv, int grid);
cudaError_t oa_step_ortho_args(oa_ctx* c, double** work, int** status, double** errv, int* grid, double** dev_e,
                               int** h_status, double** h_vals, double** eye);

struct oa_step_scratch {
  double *F, *F2, *Fnl, *S, *lam, *gam;
  cudaGraphExec_t exec;   // forces .. S
  cudaGraphExec_t exec2;  // Psi T + the record copies
  const void* key[6];
  int key_nterm;
  double key_dt;
  int pending_psiv;
};

static oa_step_scratch* step_scratch(oa_ctx* c) { return (oa_step_scratch*)c->step; }

static oa_status ensure_scratch(oa_ctx* c) {
  if (c->step) return OA_OK;
  oa_step_scratch* s = (oa_step_scratch*)calloc(1, sizeof(oa_step_scratch));
  if (!s) return OA_ERR_CUDA;
  const size_t cb = (size_t)c->nstate * c->ng * sizeof(double2);
  const size_t mb = (size_t)c->nstate * c->nstate * sizeof(double);
  if (cudaMalloc(&s->F, cb) != cudaSuccess || cudaMalloc(&s->F2, cb) != cudaSuccess ||
      cudaMalloc(&s->Fnl, cb) != cudaSuccess || cudaMalloc(&s->S, mb) != cudaSuccess ||
      cudaMalloc(&s->lam, mb) != cudaSuccess || cudaMalloc(&s->gam, mb) != cudaSuccess) {
    oa_set_error("cudaMalloc failed for the step scratch", __FILE__, __LINE__);
    return OA_ERR_CUDA;
  }
  c->step = s;
  return OA_OK;
}

void oa_step_free(oa_ctx* c) {
  oa_step_scratch* s = step_scratch(c);
  if (!s) return;
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->exec2) cudaGraphExecDestroy(s->exec2);
  void* p[] = {s->F, s->F2, s->Fnl, s->S, s->lam, s->gam};
  for (void* q : p) if (q) cudaFree(q);
  free(s);
  c->step = nullptr;
}

#define OA_STEP_TRY(x) do { oa_status st_ = (x); if (st_ != OA_OK) return st_; } while (0)

// Launches of one step up to S (part A); no host synchronisation.
static oa_status launch_step_a(oa_ctx* c, cudaStream_t s, oa_cp_state* st, int complete_prev) {
  oa_step_scratch* w = step_scratch(c);
  const int nt = st->mixed_nterm;
  // forces on the orthonormal psi (computePsiFandVKS, ParticlePlane, combineForcesGetEke)
  OA_STEP_TRY(oa_gpu_state_fft_fwd(c, s, st->psi, nullptr));
  OA_STEP_TRY(oa_gpu_vks_build(c, s, nullptr));
  OA_STEP_TRY(oa_gpu_nl_sf(c, s, st->psi, nt, w->Fnl, nullptr));
  OA_STEP_TRY(oa_gpu_vks_apply_fft_bwd(c, s, st->psi, 0, w->Fnl, w->F, nullptr));
  // constraint force (computeLambdaAndCg): Lambda, Gamma = T Lambda, F' = F T - Psi Gamma
  if (nt) {
    OA_STEP_TRY(oa_gpu_pc_forward_mixed(c, s, st->psi, w->F, 1.0, 1.0, nt, w->lam));
    OA_STEP_TRY(oa_gpu_small_gemm(c, s, st->T, w->lam, 1.0, w->gam));
    OA_STEP_TRY(oa_gpu_pc_backward_mixed(c, s, w->gam, st->psi, -0.5, -1.0, st->T, w->F, 1.0, nt, w->F2));
  } else {
    OA_STEP_TRY(oa_gpu_pc_forward(c, s, st->psi, w->F, 1.0, 1.0, w->lam));
    OA_STEP_TRY(oa_gpu_small_gemm(c, s, st->T, w->lam, 1.0, w->gam));
    OA_STEP_TRY(oa_gpu_pc_backward(c, s, w->gam, st->psi, -0.5, -1.0, st->T, w->F, 1.0, w->F2));
  }
  // integrateModForce
  OA_STEP_TRY(oa_gpu_integrate(c, s, w->F2, st->vpsi, st->psi_t, st->dt, complete_prev, nullptr));
  // computeNewPsi: S (FP64)
  OA_STEP_TRY(oa_gpu_pc_forward(c, s, st->psi_t, st->psi_t, 2.0, 0.5, w->S));
  return OA_OK;
}

// Newton-Schulz: one cooperative launch (kept out of the captured graphs)
static oa_status launch_step_ns(oa_ctx* c, cudaStream_t s, oa_cp_state* st) {
  oa_step_scratch* w = step_scratch(c);
  double *work, *errv, *dev_e, *hv, *eye;
  int *status, *hs, grid;
  OA_CUDA_TRY(oa_step_ortho_args(c, &work, &status, &errv, &grid, &dev_e, &hs, &hv, &eye));
  OA_CUDA_TRY(oa_launch_ortho_ns(s, w->S, c->nstate, 0.5, st->ns_tol, st->ns_max_iter, work, st->T, status, errv,
                                 grid));
  return OA_OK;
}

// psi = psi_t T (FP64) and the record copies (part B)
static oa_status launch_step_b(oa_ctx* c, cudaStream_t s, oa_cp_state* st) {
  double *work, *errv, *dev_e, *hv, *eye;
  int *status, *hs, grid;
  OA_CUDA_TRY(oa_step_ortho_args(c, &work, &status, &errv, &grid, &dev_e, &hs, &hv, &eye));
  OA_STEP_TRY(oa_gpu_pc_backward(c, s, st->T, st->psi_t, 1.0, 1.0, nullptr, nullptr, 0.0, st->psi));
  // one record back to the host: energies [16], NS status [2], errv [2]
  OA_CUDA_TRY(cudaMemcpyAsync(hv, dev_e, 16 * sizeof(double), cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaMemcpyAsync(hs, status, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaMemcpyAsync(hv + 10, errv, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  return OA_OK;
}

extern "C" oa_status oa_gpu_cp_step(oa_ctx* c, void* stream, oa_cp_state* st, double* energies_out) {
  if (!c || !st || !st->psi || !st->psi_t || !st->vpsi || !st->T) {
    oa_set_error("null argument", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  if (!(st->mixed_nterm == 0 || st->mixed_nterm == 2 || st->mixed_nterm == 3)) {
    oa_set_error("mixed_nterm must be 0, 2 or 3", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  OA_STEP_TRY(ensure_scratch(c));
  cudaStream_t s = (cudaStream_t)stream;
  oa_step_scratch* w = step_scratch(c);
  double *work, *errv, *dev_e, *hv, *eye;
  int *status, *hs, grid;
  OA_CUDA_TRY(oa_step_ortho_args(c, &work, &status, &errv, &grid, &dev_e, &hs, &hv, &eye));
  if (w->pending_psiv) {
    OA_STEP_TRY(oa_gpu_psiv_reset(c, s, st->psi, st->psi_t, st->vpsi));
    OA_CUDA_TRY(cudaMemcpyAsync(st->T, eye, (size_t)c->nstate * c->nstate * sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
    w->pending_psiv = 0;
  }
  st->iteration += 1;
  const int complete_prev = st->iteration > 1;
  const void* key[6] = {st->psi, st->psi_t, st->vpsi, st->T, stream, nullptr};
  // the legacy default stream cannot be captured: launch eagerly there
  const bool capturable = s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread;
  bool use_graph = st->use_graph && complete_prev && capturable;
  if (use_graph) {
    const bool same = w->exec && w->exec2 && memcmp(key, w->key, sizeof(key)) == 0 &&
                      w->key_nterm == st->mixed_nterm && w->key_dt == st->dt;
    if (!same) {
      if (w->exec) { cudaGraphExecDestroy(w->exec); w->exec = nullptr; }
      if (w->exec2) { cudaGraphExecDestroy(w->exec2); w->exec2 = nullptr; }
      for (int part = 0; part < 2; ++part) {
        cudaGraph_t g = nullptr;
        OA_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        oa_status r = part == 0 ? launch_step_a(c, s, st, 1) : launch_step_b(c, s, st);
        cudaError_t ce = cudaStreamEndCapture(s, &g);
        if (r != OA_OK) { if (g) cudaGraphDestroy(g); return r; }
        if (ce != cudaSuccess) { oa_set_error(cudaGetErrorString(ce), __FILE__, __LINE__); return OA_ERR_CUDA; }
        ce = cudaGraphInstantiate(part == 0 ? &w->exec : &w->exec2, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { oa_set_error(cudaGetErrorString(ce), __FILE__, __LINE__); return OA_ERR_CUDA; }
      }
      memcpy(w->key, key, sizeof(key));
      w->key_nterm = st->mixed_nterm;
      w->key_dt = st->dt;
    }
    OA_CUDA_TRY(cudaGraphLaunch(w->exec, s));
    OA_STEP_TRY(launch_step_ns(c, s, st));
    OA_CUDA_TRY(cudaGraphLaunch(w->exec2, s));
  } else {
    OA_STEP_TRY(launch_step_a(c, s, st, complete_prev));
    OA_STEP_TRY(launch_step_ns(c, s, st));
    OA_STEP_TRY(launch_step_b(c, s, st));
  }
  OA_CUDA_TRY(cudaStreamSynchronize(s));
  // energies: EKE EHART EEXT EWALD EEXC MUXC FICT ENL, then NS iters, residual, smax
  if (energies_out) {
    energies_out[0] = hv[OA_E_EKE];
    energies_out[1] = hv[OA_E_EHART];
    energies_out[2] = hv[OA_E_EEXT];
    energies_out[3] = hv[OA_E_EWALD];
    energies_out[4] = hv[8] + hv[9];
    energies_out[5] = hv[OA_E_MUXC];
    energies_out[6] = hv[OA_E_FICT];
    energies_out[7] = hv[OA_E_ENL];
    energies_out[8] = (double)hs[0];
    energies_out[9] = hv[10];
    energies_out[10] = hv[11];
  }
  st->last_ns_iters = hs[0];
  st->last_ns_err = hv[10];
  st->last_smax = hv[11];
  if (!(hv[10] == hv[10]) || !(hv[11] == hv[11])) {
    oa_set_error("Newton-Schulz residual is not finite", __FILE__, __LINE__);
    return OA_ERR_NONFINITE;
  }
  if (!hs[1]) {
    oa_set_error("Newton-Schulz reached max_iter", __FILE__, __LINE__);
    return OA_ERR_NOT_CONVERGED;
  }
  if (hv[11] > st->norb_tol) w->pending_psiv = 1;
  return OA_OK;
}
