// Whole CP dynamics steps in native code: the sequence of
// GSpaceDriver::computeDynamics (src_charm_driver/cp_state_ctrl/gspace.ci:199-324)
// on one GPU, ending with the PsiV tolerance reset when max|S - 2I| exceeds
// norb_tol.  The steady-state step (iteration > 1, fixed buffers) is
// captured once into one CUDA graph; with more states than the cluster
// Newton-Schulz kernel takes, into two graphs (PsiV reset .. S, and Psi T +
// the step record) replayed around the cooperative Newton-Schulz launch,
// which stream capture does not accept.  Nothing in a step needs the host: the
// PsiV tolerance check (Ortho::maxCheck, ortho.C:455-475) sets a device
// flag that the conditional reset after Psi T reads, and each step appends
// its energies and Newton-Schulz status to a device record ring.  oa_gpu_cp_run therefore enqueues many steps and
// synchronises once; oa_gpu_cp_step is the one-step case.
#include <stdio.h>
#include <string.h>
#include <vector>
#include "oa_internal.h"

// entry points of oa_abi.cu used here
extern "C" {
oa_status oa_gpu_state_fft_fwd(oa_ctx* ctx, void* stream, const double* psi, double* rho_out);
oa_status oa_gpu_vks_build(oa_ctx* ctx, void* stream, double* vks_out);
oa_status oa_gpu_nl_sf(oa_ctx* ctx, void* stream, const double* psi, int nterm, double* fnl_out, double* enl_out);
oa_status oa_gpu_nl_ees(oa_ctx* ctx, void* stream, const double* psi, double* fnl_out, double* enl_out);
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
}

int oa_ns_capturable(oa_ctx* c);
oa_status oa_integrate_sel(oa_ctx* c, cudaStream_t s, const double* force, double* vpsi, double* psi,
                           const double* psi_in, const int* sel, double dt, int complete_prev, double* fict_ke_out);
oa_status oa_psi_t_settle(oa_ctx* c, cudaStream_t s, const double* psi, double* psi_t, const int* flag);
oa_status oa_psi_t_and_psiv(oa_ctx* c, cudaStream_t s, const double* T, double* psi_t, double* psi, double* vpsi,
                            double* Tout, int* flag, int nterm, double dt);

cudaError_t oa_launch_ortho_ns(cudaStream_t s, const double* S, int n, double bscale, double tol, int max_iter,
                               double* work, double* T, int* status, double* errv, int grid);
cudaError_t oa_step_ortho_args(oa_ctx* c, double** work, int** status, double** errv, int* grid, double** dev_e,
                               int** h_status, double** h_vals, double** eye);

// per-step record: the 16 energy accumulators, NS iterations, converged,
// residual, max|S - 2I|
#define OA_REC 20
#define OA_NREC_OUT 14  // values per step handed back (oa_gpu_cp_step)

// one step record -> EKE EHART EEXT EWALD EEXC MUXC FICT ENL, Newton-Schulz
// iterations, residual, max|S - 2I|, EGGA, ionic KE, real-space Ewald
static void fill_energies(const double* hv, double* eo) {
  eo[0] = hv[OA_E_EKE]; eo[1] = hv[OA_E_EHART]; eo[2] = hv[OA_E_EEXT]; eo[3] = hv[OA_E_EWALD];
  eo[4] = hv[8] + hv[9]; eo[5] = hv[OA_E_MUXC]; eo[6] = hv[OA_E_FICT]; eo[7] = hv[OA_E_ENL];
  eo[8] = hv[16]; eo[9] = hv[18]; eo[10] = hv[19]; eo[11] = hv[11] + hv[12];
  eo[12] = hv[OA_E_ION_KE]; eo[13] = hv[OA_E_EWALD_REAL];
}

struct oa_step_scratch {
  double *F, *F2, *Fnl, *S, *lam, *gam;
  int* flag;              // device: [0] PsiV pending, [1] steps recorded, [2] first error code, [3] its step
  double* ring;           // device: [ring_cap][OA_REC]
  int ring_cap;
  double* ring_host;      // pinned copy of the ring
  int flag_host[4];
  cudaGraphExec_t exec;   // PsiV reset .. S
  cudaGraphExec_t exec2;  // Psi T + the step record
  const void* key[9];
  int key_nterm;
  double key_dt, key_tol;
  int graph_kernels;      // kernel launches of one graphed step (graph nodes + launches outside)
};

static oa_step_scratch* step_scratch(oa_ctx* c) { return (oa_step_scratch*)c->step; }

__global__ void k_set_flag(int* flag) { flag[0] = 1; }

// flag[0] = 1: a PsiV reset is pending from the previous call
static cudaError_t set_flag(cudaStream_t s, int* flag) {
  k_set_flag<<<1, 1, 0, s>>>(flag);
  return cudaGetLastError();
}

void oa_step_free(oa_ctx* c);

static oa_status ensure_scratch(oa_ctx* c) {
  if (c->step) return OA_OK;
  oa_step_scratch* s = (oa_step_scratch*)calloc(1, sizeof(oa_step_scratch));
  if (!s) return OA_ERR_CUDA;
  const size_t cb = (size_t)c->nstate * c->ng * sizeof(double2);
  const size_t mb = (size_t)c->nstate * c->nstate * sizeof(double);
  c->step = s;  // freed by oa_step_free on failure below or at destroy
  if (cudaMalloc(&s->F, cb) != cudaSuccess || cudaMalloc(&s->F2, cb) != cudaSuccess ||
      cudaMalloc(&s->Fnl, cb) != cudaSuccess || cudaMalloc(&s->S, mb) != cudaSuccess ||
      cudaMalloc(&s->lam, mb) != cudaSuccess || cudaMalloc(&s->gam, mb) != cudaSuccess ||
      cudaMalloc(&s->flag, 4 * sizeof(int)) != cudaSuccess || cudaMemset(s->flag, 0, 4 * sizeof(int)) != cudaSuccess) {
    oa_set_error("cudaMalloc failed for the step scratch", __FILE__, __LINE__);
    oa_step_free(c);
    return OA_ERR_CUDA;
  }
  return OA_OK;
}

// record ring of at least n steps (reallocating drops the captured graphs)
static oa_status ensure_ring(oa_ctx* c, int n) {
  oa_step_scratch* s = step_scratch(c);
  if (s->ring_cap >= n) return OA_OK;
  int cap = s->ring_cap > 0 ? s->ring_cap : 64;
  while (cap < n) cap *= 2;
  if (s->ring) cudaFree(s->ring);
  if (s->ring_host) cudaFreeHost(s->ring_host);
  s->ring = nullptr; s->ring_host = nullptr; s->ring_cap = 0;
  if (s->exec) { cudaGraphExecDestroy(s->exec); s->exec = nullptr; }
  if (s->exec2) { cudaGraphExecDestroy(s->exec2); s->exec2 = nullptr; }
  if (cudaMalloc(&s->ring, (size_t)cap * OA_REC * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&s->ring_host, (size_t)cap * OA_REC * sizeof(double)) != cudaSuccess) {
    oa_set_error("allocation of the step record ring failed", __FILE__, __LINE__);
    return OA_ERR_CUDA;
  }
  s->ring_cap = cap;
  return OA_OK;
}

// After Newton-Schulz: the PsiV flag (max|S - 2I| > norb_tol on a good step),
// the first failing step, and the step record.  One thread.
__global__ void k_step_check(const int* __restrict__ status, const double* __restrict__ errv,
                             const double* __restrict__ dev_e, double norb_tol, int* __restrict__ flag,
                             double* __restrict__ ring, int ring_cap) {
  const int k = flag[1];
  const double err = errv[0], smax = errv[1];
  const int code = (!(err == err) || !(smax == smax)) ? 2 : (status[1] ? 0 : 1);
  // set or clear: the flag of the previous step's PsiV reset ends here
  flag[0] = (code == 0 && smax > norb_tol) ? 1 : 0;
  if (code != 0 && flag[2] == 0) { flag[2] = code; flag[3] = k; }
  double* r = ring + (size_t)(k % ring_cap) * OA_REC;
  for (int i = 0; i < 16; ++i) r[i] = dev_e[i];
  r[16] = (double)status[0];
  r[17] = (double)status[1];
  r[18] = err;
  r[19] = smax;
  flag[1] = k + 1;
}

void oa_step_free(oa_ctx* c) {
  oa_step_scratch* s = step_scratch(c);
  if (!s) return;
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->exec2) cudaGraphExecDestroy(s->exec2);
  void* p[] = {s->F, s->F2, s->Fnl, s->S, s->lam, s->gam, s->flag, s->ring};
  for (void* q : p) if (q) cudaFree(q);
  if (s->ring_host) cudaFreeHost(s->ring_host);
  free(s);
  c->step = nullptr;
}

#define OA_STEP_TRY(x) do { oa_status st_ = (x); if (st_ != OA_OK) return st_; } while (0)

void oa_planes_step_begin(oa_ctx* c);
void oa_planes_step_end(oa_ctx* c);
void oa_planes_force_begin(oa_ctx* c, int nt);
void oa_planes_force_end(oa_ctx* c, const double* F);
oa_status oa_planes_psi_refresh(oa_ctx* c, cudaStream_t s, const double* psi, int nt);

// Launches of one step up to S (part A); no host synchronisation.  In the
// mixed form the bf16 planes of psi come from the previous step's Psi T and
// those of F from the force z pass; the structure factor is split once.
static oa_status launch_step_a(oa_ctx* c, cudaStream_t s, oa_cp_state* st, int complete_prev) {
  oa_step_scratch* w = step_scratch(c);
  const int nt = st->mixed_nterm;
  // forces on the orthonormal psi (computePsiFandVKS, ParticlePlane, combineForcesGetEke)
  OA_STEP_TRY(oa_gpu_state_fft_fwd(c, s, st->psi, nullptr));
  OA_STEP_TRY(oa_gpu_vks_build(c, s, nullptr));
  // nonlocal: the EES method once oa_gpu_ees_init enabled it
  // (cp_nonloc_ees_opt; CP_State_ParticlePlane.C:867-1136), else the
  // structure-factor method (StructureFactor.C:35-113)
  if (c->ees) OA_STEP_TRY(oa_gpu_nl_ees(c, s, st->psi, w->Fnl, nullptr));
  else OA_STEP_TRY(oa_gpu_nl_sf(c, s, st->psi, nt, w->Fnl, nullptr));
  if (nt) oa_planes_force_begin(c, nt);
  const oa_status rf = oa_gpu_vks_apply_fft_bwd(c, s, st->psi, 0, w->Fnl, w->F, nullptr);
  oa_planes_force_end(c, w->F);
  OA_STEP_TRY(rf);
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
  // integrateModForce; psi(t) is psi itself after the previous step's PsiV reset
  OA_STEP_TRY(oa_integrate_sel(c, s, w->F2, st->vpsi, st->psi_t, st->psi, w->flag, st->dt, complete_prev, nullptr));
  // ion dynamics: real-space Ewald and the atom integration with this
  // step's forces (AtomsCompute::integrateAtoms); the next step's phase
  // tables, structure factors and B-splines see the new positions
  if (c->ions) {
    double *work, *errv, *dev_e, *hv, *eye;
    int *status, *hs, grid;
    OA_CUDA_TRY(oa_step_ortho_args(c, &work, &status, &errv, &grid, &dev_e, &hs, &hv, &eye));
    OA_CUDA_TRY(oa_launch_ion_step(c, s, dev_e, st->dt, complete_prev));
  }
  // computeNewPsi: S (FP64 DMMA in both forms)
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

// psi = psi_t T (FP64), the PsiV check and the step record (part B)
static oa_status launch_step_b(oa_ctx* c, cudaStream_t s, oa_cp_state* st) {
  oa_step_scratch* w = step_scratch(c);
  double *work, *errv, *dev_e, *hv, *eye;
  int *status, *hs, grid;
  OA_CUDA_TRY(oa_step_ortho_args(c, &work, &status, &errv, &grid, &dev_e, &hs, &hv, &eye));
  k_step_check<<<1, 1, 0, s>>>(status, errv, dev_e, st->norb_tol, w->flag, w->ring, w->ring_cap);
  OA_CUDA_TRY(cudaGetLastError());
  // psi = psi_t T, and the PsiV reset when the check asked for it
  OA_STEP_TRY(oa_psi_t_and_psiv(c, s, st->T, st->psi_t, st->psi, st->vpsi, st->T, w->flag, st->mixed_nterm, st->dt));
  return OA_OK;
}

static oa_status run_steps(oa_ctx* c, void* stream, oa_cp_state* st, int nsteps, const double* pos_host,
                           double* energies_out) {
  if (!c || !st || !st->psi || !st->psi_t || !st->vpsi || !st->T || nsteps < 1) {
    oa_set_error("null argument or nsteps < 1", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  if (!(st->mixed_nterm == 0 || st->mixed_nterm == 2 || st->mixed_nterm == 3)) {
    oa_set_error("mixed_nterm must be 0, 2 or 3", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  OA_STEP_TRY(ensure_scratch(c));
  OA_STEP_TRY(ensure_ring(c, nsteps));
  cudaStream_t s = (cudaStream_t)stream;
  oa_step_scratch* w = step_scratch(c);
  // restart the record count and the error slot; the PsiV flag carries a
  // reset that ended the previous call
  OA_CUDA_TRY(cudaMemsetAsync(w->flag, 0, 4 * sizeof(int), s));
  if (st->psiv_pending) OA_CUDA_TRY(set_flag(s, w->flag));
  // the psi planes of the mixed products, from the psi the caller hands in
  if (st->mixed_nterm) OA_STEP_TRY(oa_planes_psi_refresh(c, s, st->psi, st->mixed_nterm));
  const void* key[9] = {st->psi, st->psi_t, st->vpsi, st->T, stream, w->ring, c->ees,
                        (const void*)(uintptr_t)c->xc_gen, (const void*)(uintptr_t)c->eesl_gen};
  // the legacy default stream cannot be captured: launch eagerly there
  const bool capturable = s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread;
  // the cluster Newton-Schulz kernel is an ordinary launch: then the whole
  // step is one graph; the cooperative one splits it in two
  const bool ns_in_graph = oa_ns_capturable(c) != 0;
  if (pos_host && c->ions) {
    oa_set_error("pos_host with ion dynamics on: the atoms move on the device", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  for (int k = 0; k < nsteps; ++k) {
    if (pos_host)
      OA_CUDA_TRY(cudaMemcpyAsync(c->pos, pos_host + (size_t)k * 3 * c->natm, (size_t)3 * c->natm * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
    st->iteration += 1;
    const int complete_prev = st->iteration > 1;
    const bool use_graph = st->use_graph && complete_prev && capturable;
    if (use_graph) {
      const bool same = w->exec && (ns_in_graph || w->exec2) && memcmp(key, w->key, sizeof(key)) == 0 &&
                        w->key_nterm == st->mixed_nterm && w->key_dt == st->dt && w->key_tol == st->norb_tol;
      if (!same) {
        if (w->exec) { cudaGraphExecDestroy(w->exec); w->exec = nullptr; }
        if (w->exec2) { cudaGraphExecDestroy(w->exec2); w->exec2 = nullptr; }
        int nker = ns_in_graph ? 0 : 1;  // the Newton-Schulz launch between the two graphs
        for (int part = 0; part < (ns_in_graph ? 1 : 2); ++part) {
          cudaGraph_t g = nullptr;
          OA_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
          oa_status r = OA_OK;
          if (part == 0) oa_planes_step_begin(c);
          if (ns_in_graph) {
            r = launch_step_a(c, s, st, 1);
            if (r == OA_OK) r = launch_step_ns(c, s, st);
            if (r == OA_OK) r = launch_step_b(c, s, st);
          } else {
            r = part == 0 ? launch_step_a(c, s, st, 1) : launch_step_b(c, s, st);
          }
          if (ns_in_graph || part == 1 || r != OA_OK) oa_planes_step_end(c);
          cudaError_t ce = cudaStreamEndCapture(s, &g);
          if (r != OA_OK) { if (g) cudaGraphDestroy(g); return r; }
          if (ce != cudaSuccess) { oa_set_error(cudaGetErrorString(ce), __FILE__, __LINE__); return OA_ERR_CUDA; }
          {
            size_t nn = 0;
            if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
              std::vector<cudaGraphNode_t> nodes(nn);
              if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
                for (size_t i = 0; i < nn; ++i) {
                  cudaGraphNodeType t;
                  if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nker;
                }
            }
          }
          ce = cudaGraphInstantiate(part == 0 ? &w->exec : &w->exec2, g, 0);
          cudaGraphDestroy(g);
          if (ce != cudaSuccess) { oa_set_error(cudaGetErrorString(ce), __FILE__, __LINE__); return OA_ERR_CUDA; }
        }
        memcpy(w->key, key, sizeof(key));
        w->graph_kernels = nker;
        w->key_nterm = st->mixed_nterm;
        w->key_dt = st->dt;
        w->key_tol = st->norb_tol;
      }
      OA_CUDA_TRY(cudaGraphLaunch(w->exec, s));
      if (!ns_in_graph) {
        OA_STEP_TRY(launch_step_ns(c, s, st));
        OA_CUDA_TRY(cudaGraphLaunch(w->exec2, s));
      }
    } else {
      oa_planes_step_begin(c);
      oa_status r = launch_step_a(c, s, st, complete_prev);
      if (r == OA_OK) r = launch_step_ns(c, s, st);
      if (r == OA_OK) r = launch_step_b(c, s, st);
      oa_planes_step_end(c);
      OA_STEP_TRY(r);
    }
  }
  OA_STEP_TRY(oa_psi_t_settle(c, s, st->psi, st->psi_t, w->flag));
  OA_CUDA_TRY(cudaMemcpyAsync(w->ring_host, w->ring, (size_t)nsteps * OA_REC * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaMemcpyAsync(w->flag_host, w->flag, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
  OA_CUDA_TRY(cudaStreamSynchronize(s));
  // energies: EKE EHART EEXT EWALD EEXC MUXC FICT ENL, then NS iters, residual, smax, EGGA
  if (energies_out)
    for (int k = 0; k < nsteps; ++k) fill_energies(w->ring_host + (size_t)k * OA_REC, energies_out + (size_t)k * OA_NREC_OUT);
  const double* last = w->ring_host + (size_t)(nsteps - 1) * OA_REC;
  st->last_kernels = (st->use_graph && st->iteration > 1 && w->exec) ? w->graph_kernels : -1;
  st->last_ns_iters = (int)last[16];
  st->last_ns_err = last[18];
  st->last_smax = last[19];
  st->psiv_pending = w->flag_host[0];
  if (w->flag_host[2] != 0) {
    char msg[160];
    snprintf(msg, sizeof(msg), "%s in step %d of %d",
             w->flag_host[2] == 2 ? "Newton-Schulz residual is not finite" : "Newton-Schulz reached max_iter",
             w->flag_host[3] + 1, nsteps);
    oa_set_error(msg, __FILE__, __LINE__);
    return w->flag_host[2] == 2 ? OA_ERR_NONFINITE : OA_ERR_NOT_CONVERGED;
  }
  return OA_OK;
}

// ---------------------------------------------------------------------------
// Batching form: nsys independent systems (replicas, beads, tempering
// systems of any sizes), nsteps CP steps each.  After each system's first
// step, one step of every system is one CUDA graph: the systems' launches
// fork from `stream` onto one stream per system and join back, so the
// kernels of different systems fill the GPU together.
// ---------------------------------------------------------------------------
static oa_status batch_launch_one(oa_ctx* c, cudaStream_t s, oa_cp_state* st, int complete_prev) {
  oa_planes_step_begin(c);
  oa_status r = launch_step_a(c, s, st, complete_prev);
  if (r == OA_OK) r = launch_step_ns(c, s, st);
  if (r == OA_OK) r = launch_step_b(c, s, st);
  oa_planes_step_end(c);
  return r;
}

extern "C" oa_status oa_gpu_cp_run_batch(oa_ctx** ctxs, oa_cp_state** states, int nsys, void* stream, int nsteps,
                                         double* energies_out) {
  if (!ctxs || !states || nsys < 1 || nsteps < 1) {
    oa_set_error("null argument, nsys < 1 or nsteps < 1", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) {
    oa_set_error("the batched run needs a created stream (it is captured into a CUDA graph)", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  for (int i = 0; i < nsys; ++i) {
    oa_ctx* c = ctxs[i];
    oa_cp_state* st = states[i];
    if (!c || !st || !st->psi || !st->psi_t || !st->vpsi || !st->T) {
      oa_set_error("null context or state in the batch", __FILE__, __LINE__);
      return OA_ERR_BAD_ARG;
    }
    if (!(st->mixed_nterm == 0 || st->mixed_nterm == 2 || st->mixed_nterm == 3)) {
      oa_set_error("mixed_nterm must be 0, 2 or 3", __FILE__, __LINE__);
      return OA_ERR_BAD_ARG;
    }
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == c) {
        oa_set_error("a context appears twice in the batch", __FILE__, __LINE__);
        return OA_ERR_BAD_ARG;
      }
    // the whole step must be capturable: the cluster Newton-Schulz kernel
    if (!oa_ns_capturable(c)) {
      oa_set_error("the batched run needs the cluster Newton-Schulz kernel (at most 128 states)", __FILE__,
                   __LINE__);
      return OA_ERR_UNSUPPORTED;
    }
  }
  for (int i = 0; i < nsys; ++i) {
    OA_STEP_TRY(ensure_scratch(ctxs[i]));
    OA_STEP_TRY(ensure_ring(ctxs[i], nsteps));
  }
  std::vector<cudaStream_t> side(nsys, nullptr);
  std::vector<cudaEvent_t> join(nsys, nullptr);
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec = nullptr;
  oa_status ret = OA_OK;
  auto fail = [&](cudaError_t e, int line) {
    oa_set_error(cudaGetErrorString(e), __FILE__, line);
    ret = OA_ERR_CUDA;
  };
  cudaError_t ce = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
  for (int i = 0; i < nsys && ce == cudaSuccess; ++i) {
    ce = cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming);
  }
  if (ce != cudaSuccess) fail(ce, __LINE__);
  // per system: restart the PsiV flag and record count, psi planes from the handed-in psi
  for (int i = 0; i < nsys && ret == OA_OK; ++i) {
    oa_step_scratch* w = step_scratch(ctxs[i]);
    ce = cudaMemsetAsync(w->flag, 0, 4 * sizeof(int), s);
    if (ce == cudaSuccess && states[i]->psiv_pending) ce = set_flag(s, w->flag);
    if (ce != cudaSuccess) { fail(ce, __LINE__); break; }
    if (states[i]->mixed_nterm) ret = oa_planes_psi_refresh(ctxs[i], s, states[i]->psi, states[i]->mixed_nterm);
  }
  int graph_kernels = 0;
  // one step of all systems, launched on the side streams (fork .. join)
  auto step_all = [&](bool steady) -> oa_status {
    cudaError_t e = cudaEventRecord(fork, s);
    if (e != cudaSuccess) { fail(e, __LINE__); return ret; }
    for (int i = 0; i < nsys; ++i) {
      if ((e = cudaStreamWaitEvent(side[i], fork, 0)) != cudaSuccess) { fail(e, __LINE__); return ret; }
      oa_cp_state* st = states[i];
      const int complete_prev = steady ? 1 : (st->iteration > 0);
      const oa_status r = batch_launch_one(ctxs[i], side[i], st, complete_prev);
      if (r != OA_OK) return r;
      if ((e = cudaEventRecord(join[i], side[i])) != cudaSuccess) { fail(e, __LINE__); return ret; }
      if ((e = cudaStreamWaitEvent(s, join[i], 0)) != cudaSuccess) { fail(e, __LINE__); return ret; }
    }
    return OA_OK;
  };
  for (int k = 0; k < nsteps && ret == OA_OK; ++k) {
    bool all_steady = true;
    for (int i = 0; i < nsys; ++i) all_steady = all_steady && states[i]->iteration > 0;
    if (!all_steady) {
      // first steps (no previous half kick) run eagerly
      ret = step_all(false);
    } else {
      if (!exec) {
        cudaGraph_t g = nullptr;
        if ((ce = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
          fail(ce, __LINE__);
          break;
        }
        const oa_status r = step_all(true);
        ce = cudaStreamEndCapture(s, &g);
        if (r != OA_OK) { if (g) cudaGraphDestroy(g); ret = r; break; }
        if (ce != cudaSuccess) { fail(ce, __LINE__); break; }
        size_t nn = 0;
        if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
          std::vector<cudaGraphNode_t> nodes(nn);
          if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
            for (size_t q = 0; q < nn; ++q) {
              cudaGraphNodeType t;
              if (cudaGraphNodeGetType(nodes[q], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++graph_kernels;
            }
        }
        ce = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { fail(ce, __LINE__); break; }
      }
      if ((ce = cudaGraphLaunch(exec, s)) != cudaSuccess) { fail(ce, __LINE__); break; }
    }
    for (int i = 0; i < nsys; ++i) states[i]->iteration += 1;
  }
  // records and flags of every system, one synchronisation
  for (int i = 0; i < nsys && ret == OA_OK; ++i) {
    oa_step_scratch* w = step_scratch(ctxs[i]);
    ret = oa_psi_t_settle(ctxs[i], s, states[i]->psi, states[i]->psi_t, w->flag);
    if (ret != OA_OK) break;
    ce = cudaMemcpyAsync(w->ring_host, w->ring, (size_t)nsteps * OA_REC * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(w->flag_host, w->flag, 4 * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce != cudaSuccess) fail(ce, __LINE__);
  }
  if (ret == OA_OK && (ce = cudaStreamSynchronize(s)) != cudaSuccess) fail(ce, __LINE__);
  if (exec) cudaGraphExecDestroy(exec);
  for (int i = 0; i < nsys; ++i) {
    if (join[i]) cudaEventDestroy(join[i]);
    if (side[i]) cudaStreamDestroy(side[i]);
  }
  if (fork) cudaEventDestroy(fork);
  if (ret != OA_OK) return ret;
  for (int i = 0; i < nsys; ++i) {
    oa_step_scratch* w = step_scratch(ctxs[i]);
    oa_cp_state* st = states[i];
    if (energies_out)
      for (int k = 0; k < nsteps; ++k)
        fill_energies(w->ring_host + (size_t)k * OA_REC, energies_out + ((size_t)i * nsteps + k) * OA_NREC_OUT);
    const double* last = w->ring_host + (size_t)(nsteps - 1) * OA_REC;
    st->last_kernels = graph_kernels > 0 ? graph_kernels : -1;
    st->last_ns_iters = (int)last[16];
    st->last_ns_err = last[18];
    st->last_smax = last[19];
    st->psiv_pending = w->flag_host[0];
    if (w->flag_host[2] != 0) {
      char msg[200];
      snprintf(msg, sizeof(msg), "system %d of the batch: %s in step %d of %d", i,
               w->flag_host[2] == 2 ? "Newton-Schulz residual is not finite" : "Newton-Schulz reached max_iter",
               w->flag_host[3] + 1, nsteps);
      oa_set_error(msg, __FILE__, __LINE__);
      return w->flag_host[2] == 2 ? OA_ERR_NONFINITE : OA_ERR_NOT_CONVERGED;
    }
  }
  return OA_OK;
}

extern "C" oa_status oa_gpu_cp_step(oa_ctx* c, void* stream, oa_cp_state* st, double* energies_out) {
  return run_steps(c, stream, st, 1, nullptr, energies_out);
}

extern "C" oa_status oa_gpu_cp_run(oa_ctx* c, void* stream, oa_cp_state* st, int nsteps, const double* pos_host,
                                   double* energies_out) {
  return run_steps(c, stream, st, nsteps, pos_host, energies_out);
}
