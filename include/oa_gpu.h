/*
 * liboa_gpu — C ABI of the B200 (sm_100a) Car-Parrinello electronic step.
 *
 * Each entry point does, for all states of one system on one GPU, the work of
 * one OpenAtom chare entry method (or PINY physics routine) named beside it.
 * Plain pointers and sizes only.  Arrays called "device" are caller-owned
 * device memory; the context owns its own scratch.  Every call is
 * asynchronous on the given stream unless it says it synchronises.
 *
 * Coefficient layout: double complex AoS (re, im), state-major:
 *   psi[state * ng + ig], the reference's `complex` of ckcomplex.h, with the
 *   g-points ordered as OpenAtom's doublePack state planes (kx = 0 first,
 *   its redundant half first; z-line runs negative kz then non-negative kz),
 *   src_charm_driver/fft_slab_ctrl/stateSlab.C:299-370 and
 *   src_charm_driver/utility/util.C:936-990.
 */
#ifndef OA_GPU_H
#define OA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  OA_OK = 0,
  OA_ERR_BAD_ARG = 1,
  OA_ERR_CUDA = 2,
  OA_ERR_NOT_CONVERGED = 3,
  OA_ERR_NONFINITE = 4,
  OA_ERR_UNSUPPORTED = 5
} oa_status;

typedef enum { OA_FP64 = 0, OA_MIXED = 1 } oa_precision;

typedef struct oa_ctx oa_ctx;

/* Host-side description of one Gamma-point system (read during oa_gpu_init,
 * not retained).  Mirrors what CPcharmParaInfo / the PINY CP singletons hold
 * for the state step (src_piny_physics_v1.0/include/class_defs/allclass_cp.h). */
typedef struct {
  int nx, ny, nz;              /* FFT grid (sizeX, sizeY, sizeZ) */
  int nstate;
  int ng;                      /* half-sphere g-points per state (numPoints) */
  int nlines;                  /* z-lines (numRuns / 2) */
  const int *line_kx, *line_ky;      /* [nlines] */
  const int *line_off;               /* [nlines] packed offset of the line */
  const int *line_nneg, *line_npos;  /* [nlines] run lengths, kz<0 and kz>=0 */
  const int *kx, *ky, *kz;           /* [ng] */
  int nkx0, nkx0_red, nkx0_uni, nkx0_zero;
  const int *red_partner;            /* [nkx0_red] index of -g of each redundant point */
  double box;                  /* cubic cell edge, bohr */
  double ecut_psi;             /* state cutoff on g^2 (Ry), cp_eke.C:50 */
  double ecut_rho;             /* density cutoff on g^2, cp_hart_ext.C:113 */
  const double *occ;           /* [nstate] occupations (1.0 closed shell) */
  const double *cmass;         /* [ng] fictitious masses, cp_control_integrate.C:136 */
  int natm, ntype;
  const double *pos;           /* [natm][3] bohr */
  const int *atm_type;         /* [natm] 0..ntype-1 */
  const double *q_type;        /* [ntype] valence charges */
  const double *gzvps;         /* [ntype] g = 0 local term */
  double alp_ewd;
  int nspl;                    /* local pseudopotential spline (CP_get_vpsnow) */
  double spl_gmin, spl_dg;
  const double *spl;           /* [ntype][nspl][4] */
  /* nonlocal l = 0 KB channel (cppseudo->nonlocal); same spline grid */
  int natm_nl;
  const int *nl_atm;           /* [natm_nl] atom index of each nonlocal atom (map_nl) */
  const double *nl_spl;        /* [ntype][nspl][4] projector spline */
  const double *nl_vnorm;      /* [ntype] vnorm_0 */
  const double *nl_gz0;        /* [ntype] projector at g = 0 (gzvps0) */
} oa_system_desc;

/* Create a context on the current CUDA device.  precision = OA_FP64 (plain
 * form) or OA_MIXED (FP32 state FFT path).  Allocates all scratch. */
oa_status oa_gpu_init(const oa_system_desc *desc, int precision, oa_ctx **out);
oa_status oa_gpu_destroy(oa_ctx *ctx);
const char *oa_gpu_last_error(void);
/* Bytes of device scratch the context holds. */
size_t oa_gpu_scratch_bytes(const oa_ctx *ctx);

/* State FFT g -> r and density.
 * Replaces CP_State_GSpacePlane::doFFT (CP_State_GSpacePlane.C:1377-1445),
 * sendFFTData (:1448), CP_State_RealSpacePlane::unpackFFT/doFFT/doReduction
 * (CP_State_RealSpacePlane.C:186-517) and the density sum of
 * CP_Rho_RealSpacePlane::acceptDensity (CP_Rho_RealSpacePlane.C:398-500).
 * psi: device [nstate][ng] complex.  rho_out (optional, device [nz][ny][nx]
 * doubles) receives rho(r) = sum_s occ_s psi_s(r)^2 / V after the call. */
oa_status oa_gpu_state_fft_fwd(oa_ctx *ctx, void *stream, const double *psi, double *rho_out);

/* V_KS(r) = V_xc + V_H + V_loc from the density of the last state_fft_fwd.
 * Replaces CP_Rho_RealSpacePlane::energyComputation -> CPXCFNCTS::CP_exc_calc
 * (cp_pz_lda.C:23-175), fftRhoRtoRhoG, CP_Rho_GHartExt::HartExtVksG ->
 * CPLOCAL::CP_hart_eext_calc (cp_hart_ext.C:56-431), FFTVks, acceptHartVks.
 * vks_out (optional, device [nz][ny][nx] doubles). */
oa_status oa_gpu_vks_build(oa_ctx *ctx, void *stream, double *vks_out);

/* Set V_KS(r) directly (device doubles [nz][ny][nx]); for callers that build
 * the potential themselves (CP_State_RealSpacePlane::acceptVks). */
oa_status oa_gpu_set_vks(oa_ctx *ctx, void *stream, const double *vks);

/* psi(r) V_KS(r) occ -> back to g-space -> coefficient forces and EKE.
 * Replaces CP_State_RealSpacePlane::unpackVks/doVksFFT/sendFPsiToGSP
 * (:530-725), CP_State_GSpacePlane::unpackIFFT/doIFFT (:1530-1626),
 * combineForcesGetEke (:1634-1746) with GStateSlab::addForces
 * (stateSlab.C:239-268) and CPNONLOCAL::CP_eke_calc (cp_eke.C:30-140).
 * recompute_fwd = 1 redoes the z pass from psi (needed unless the previous
 * call on this context was oa_gpu_state_fft_fwd on the same psi).
 * fnl: optional device [nstate][ng] nonlocal forces added after the x2.
 * force: device [nstate][ng] output.  eke_out: optional device [nstate]. */
oa_status oa_gpu_vks_apply_fft_bwd(oa_ctx *ctx, void *stream, const double *psi, int recompute_fwd,
                                   const double *fnl, double *force, double *eke_out);

/* PairCalculator forward (ckPairCalculator.C:821-893 + the tile reduction
 * to Ortho, :938-1016): C[x][y] = alpha * sum_k w(k) left_x(k) right_y(k)
 * over the real view (2*ng doubles per state); w = w_kx0 on the first
 * 2*nkx0 doubles (kx = 0 plane) and 1 elsewhere.  S: alpha = 2,
 * w_kx0 = 1/2 (sendPsi 1/sqrt2 on both sides); Lambda: alpha = 1, w_kx0 = 1.
 * left, right: device [nstate][ng] complex; C: device [nstate][nstate]. */
oa_status oa_gpu_pc_forward(oa_ctx *ctx, void *stream, const double *left, const double *right,
                            double alpha, double w_kx0, double *C);

/* The symmetric PairCalculator overlap of the mixed form on the int8 tensor
 * cores, S = alpha * sum_k w(k) psi_t_x(k) psi_t_y(k) (the same product as
 * oa_gpu_pc_forward(psi_t, psi_t), ckPairCalculator.C:821-893, with the
 * reduction :938-1016), to FP64 accuracy: psi_t is split into six int8
 * digits per value with one exponent per state and K range, the digit
 * products are exact in int32 and combined in FP64 (relative error about
 * 2^-42 of the largest value of a range).  The digits stay in the context
 * for oa_gpu_pc_rotate_i8.  Mixed-precision contexts with at most 128
 * states (the buffers are allocated on the first call); OA_ERR_UNSUPPORTED
 * otherwise.  Not used by the native step: on B200 its eight digit levels
 * fill all of TMEM with N = 64 accumulators, and at 128 states it is slower
 * than the FP64 DMMA product. */
oa_status oa_gpu_pc_overlap_i8(oa_ctx *ctx, void *stream, const double *psi_t, double alpha, double w_kx0,
                               double *S);

/* psi_out = psi_t T (psi_out_j = sum_i T[i][j] psi_t_i; bwMultiplyHelper
 * 'N','N', ckPairCalculator.C:1710-1946) on the int8 tensor cores, to FP64
 * accuracy, from the digits of psi_t taken by the last
 * oa_gpu_pc_overlap_i8 on this context (OA_ERR_BAD_ARG if psi_t is another
 * array).  T: device [nstate][nstate]; psi_out must not alias psi_t. */
oa_status oa_gpu_pc_rotate_i8(oa_ctx *ctx, void *stream, const double *T, const double *psi_t, double *psi_out);

/* Minimisation (cp_min_opt on; GSpaceDriver::computeMinimization,
 * gspace.ci:85-196).  oa_gpu_min_fovlap: *fovlap_out = sum over every
 * stored point of |force|^2 (CPINTEGRATE::CP_fovlap_calc, cp_min_CG.C:128;
 * its square root is the force magnitude tested against tol_cp_min,
 * CP_State_GSpacePlane.C:110-190); synchronises.  oa_gpu_min_step: one
 * steepest-descent step psi += force dt / m (CP_integrate_min_STD,
 * cp_min_std.C:17-60) when conj_grad is NULL, else one conjugate-gradient
 * step conj = gamma conj + force on g^2 <= ecut, psi += conj dt / m
 * (CP_integrate_min_CG, cp_min_CG.C:29-120), then the Gamma redundancy
 * sync of psi.  force: the constraint-projected force, device [nstate][ng]. */
oa_status oa_gpu_min_fovlap(oa_ctx *ctx, void *stream, const double *force, double *fovlap_out);
oa_status oa_gpu_min_step(oa_ctx *ctx, void *stream, const double *force, double *conj_grad, double *psi,
                          double gamma, double dt);

/* Ortho S -> T = (S/2)^(-1/2) by Newton-Schulz (ortho.C:109-146, 153-266,
 * 848-971; same iteration as CPORTHOG::get_iter_Tmat, cp_lowdin.C:180-265).
 * S, T: device [n][n].  Synchronises the stream to return iterations,
 * residual and smax = max |S - 2I| (Ortho::array_diag_max, ortho.h:282, the
 * quantity Ortho::maxCheck compares with cp_norb_tol); returns
 * OA_ERR_NOT_CONVERGED when max_iter is reached. */
oa_status oa_gpu_ortho_invsqrt(oa_ctx *ctx, void *stream, const double *S, double *T, double tol,
                               int max_iter, int *iters_out, double *err_out, double *smax_out);

/* PairCalculator backward (multiplyResult / bwMultiplyHelper /
 * bwMultiplyDynOrthoT, ckPairCalculator.C:1201-2031), state-row form:
 *   out_j = a1(c) sum_k M1[k][j] X1_k + a2 sum_k M2[k][j] X2_k
 * a1(c) = a1_kx0 on the kx = 0 plane, a1_rest elsewhere.  M2/X2 may be NULL.
 * Orthonormalisation psi = Psi T: M1 = T, a1 = 1.  Dynamics constraint
 * force F' = F T - Psi Gamma (kx=0 Psi term halved by the 1/sqrt2
 * scalings of sendLambda + doLambda): M1 = Gamma, X1 = psi,
 * a1_kx0 = -1/2, a1_rest = -1, M2 = T, X2 = F, a2 = 1.
 * out must not alias X1 or X2. */
oa_status oa_gpu_pc_backward(oa_ctx *ctx, void *stream, const double *M1, const double *X1,
                             double a1_kx0, double a1_rest, const double *M2, const double *X2, double a2,
                             double *out);

/* Mixed-precision PairCalculator forward on the tcgen05 tensor cores: same
 * contract as oa_gpu_pc_forward, operands split into nterm bf16 terms
 * (nterm = 2: 3 products, ~2^-16 relative; nterm = 3: 6 products, ~2^-24),
 * FP32 accumulation per K block, FP64 reduction over K blocks. */
oa_status oa_gpu_pc_forward_mixed(oa_ctx *ctx, void *stream, const double *left, const double *right,
                                  double alpha, double w_kx0, int nterm, double *C);

/* Mixed-precision PairCalculator backward on the tcgen05 tensor cores; same
 * contract as oa_gpu_pc_backward, split as oa_gpu_pc_forward_mixed. */
oa_status oa_gpu_pc_backward_mixed(oa_ctx *ctx, void *stream, const double *M1, const double *X1,
                                   double a1_kx0, double a1_rest, const double *M2, const double *X2, double a2,
                                   int nterm, double *out);

/* Synchronise the stream and report whether any kernel's time-bounded wait
 * (200 ms) ran out (OA_ERR_CUDA with a message) since the last check; the
 * device flag is cleared when it is reported. */
oa_status oa_gpu_check(oa_ctx *ctx, void *stream);

/* Failure-detection test hook, no counterpart in the reference (its
 * failures end in CkAbort / EXIT).  kind 1: the next split-BF16 forward
 * product skips the loads of one pipeline stage in one block, so that
 * block's bounded wait runs out and oa_gpu_check reports it; kind 0 clears
 * the hook.  Acts on the current device. */
oa_status oa_gpu_fault_inject(oa_ctx *ctx, int kind);

/* Small dense C = alpha A B (N x N), e.g. Gamma = T Lambda (ortho.C:565-570). */
oa_status oa_gpu_small_gemm(oa_ctx *ctx, void *stream, const double *A, const double *B, double alpha,
                            double *C);

/* Velocity Verlet on the coefficients (CPINTEGRATE::CP_integrate_dyn,
 * cp_dynamics.C:29-88, cp_evolve_vel :97-210, get_fictKE :218-254) and the
 * Gamma redundancy sync (CP_State_GSpacePlane.C:2829-2970).  complete_prev = 1
 * first completes the previous half kick (iteration > 1).  fict_ke_out:
 * optional device double. */
oa_status oa_gpu_integrate(oa_ctx *ctx, void *stream, const double *force, double *vpsi, double *psi,
                           double dt, int complete_prev, double *fict_ke_out);

/* PsiV tolerance reset of the reference's default build (Ortho::maxCheck,
 * ortho.C:455-475 -> computeNewPsiVFiniteDifference, gspace.ci:290-301;
 * CP_State_GSpacePlane::finiteDifferencePsiV, CP_State_GSpacePlane.C:3741-3800,
 * norb_fin_diff_order 0): psi_t <- psi and v <- (psi - psi_prev) / dt, with
 * psi_prev the orthonormal states of the previous step.  The caller resets
 * its T to the identity, and its next oa_gpu_integrate takes
 * complete_prev = 0 (the velocity is already at t: halfStepEvolve = 0). */
oa_status oa_gpu_psiv_reset(oa_ctx *ctx, void *stream, const double *psi, const double *psi_prev, double *psi_t,
                            double *vpsi, double dt);

/* Copy new atom positions (host [natm][3], bohr) for the next vks_build
 * (the structure-factor phases are rebuilt from them every call). */
oa_status oa_gpu_set_atoms(oa_ctx *ctx, void *stream, const double *pos_host);

/* Average device time (ms, CUDA events on `stream`) of each kernel of the
 * step over `reps` launches on the given orthonormal psi: ms_out[0..10] =
 * state z pass fwd, state plane pass + density, density sum + XC, V_KS build
 * (density FFT, Hartree/local, inverse), state plane pass with V_KS,
 * state z pass bwd + EKE, PairCalculator forward S, PairCalculator
 * backward (two-term, the constraint force), Newton-Schulz, the rotation
 * Psi T, the PairCalculator forward Lambda -- each as the context's form
 * runs it in the step (mixed: the two-term backward and Lambda split-BF16,
 * S and Psi T FP64 DMMA) -- and, for a mixed context of at most 128 states,
 * ms_out[11..12] = the int8 digit products of S and Psi T
 * (oa_gpu_pc_overlap_i8 / oa_gpu_pc_rotate_i8).  ms_out holds 13 values.
 * Clobbers the context's scratch.
 * No reference counterpart (it replaces the Projections user events of
 * e.g. CP_State_GSpacePlane.C:1407-1409). */
oa_status oa_gpu_time_kernels(oa_ctx *ctx, void *stream, const double *psi, int reps, double *ms_out);

/* Runtime tile and schedule choices of a context: what the autotuner
 * (openatom_b200/tuner.py) searches per system size.  No counterpart in the
 * reference, whose decomposition is set by its Charm++ configuration
 * (piny_to_driver/configure.C).  The group, dgemm and fft choices change
 * at most the order of partial sums (results agree to rounding);
 * tgemm_kblocks also sets how many terms each FP32 tensor-core
 * accumulation holds (fewer blocks: longer FP32 sums, larger error), so
 * the autotuner leaves it at the built-in choice, the most the partials
 * allow. */
typedef struct oa_tuning {
  int group_state;   /* state groups of the per-state plane kernels: nz x groups blocks (1..32) */
  int group_pair;    /* state-pair groups of the mixed state-pair plane kernels (1..32) */
  int dgemm_kblocks; /* most split-K blocks of the FP64 tensor-core products (2..160) */
  int tgemm_kblocks; /* most split-K blocks of the split-BF16 tcgen05 products (1..the limit set at init) */
  int fft_path;      /* 1: two-pass register transforms where compiled; 2: runtime-plan shared-memory
                        transforms (FP64 form only: the state-pair kernels are two-pass) */
} oa_tuning;

/* The current choices (after oa_gpu_init: the built-in heuristics). */
oa_status oa_gpu_get_tuning(const oa_ctx *ctx, oa_tuning *out);

/* Set the choices; a field of 0 keeps its value.  Out of range:
 * OA_ERR_BAD_ARG; fft_path 2 in the mixed form: OA_ERR_UNSUPPORTED.  Grows
 * the density partials when a group count grows (synchronising the
 * device first); the next oa_gpu_cp_run re-makes its captured step. */
oa_status oa_gpu_set_tuning(oa_ctx *ctx, const oa_tuning *in);

/* Sizes for byte/flop accounting (see oa_abi.cu): out[0..12]. */
oa_status oa_gpu_sizes(const oa_ctx *ctx, long *out);

/* Nonlocal energy and coefficient forces by the structure-factor method
 * (StructureFactor::computeSF -> CPNONLOCAL::CP_calc_Struct_Fact,
 * cp_struct_fact.C:37-255; CP_State_ParticlePlane::computeZ/reduceZ/getForces,
 * CP_State_ParticlePlane.C:500-760 -> CP_enl_matrix_calc cp_nlmat.C:24-100,
 * CP_enl_atm_forc_calc and CP_enl_force_calc cp_nl_energy_forc.C:29-235).
 * psi: device [nstate][ng]; fnl_out: device [nstate][ng] (the
 * ParticlePlane forces that addForces adds); enl_out: optional device
 * [nstate].  nterm = 0 uses FP64 tensor-core GEMMs, 2 or 3 the split-BF16
 * tcgen05 GEMMs.  The structure factor (FP64) is rebuilt from the current
 * atom positions on every call. */
oa_status oa_gpu_nl_sf(oa_ctx *ctx, void *stream, const double *psi, int nterm, double *fnl_out, double *enl_out);

/* State of one CP dynamics run (caller-owned device buffers). */
typedef struct {
  double *psi_t;        /* [nstate][ng] non-orthogonal coefficients (integrated) */
  double *psi;          /* [nstate][ng] orthonormal coefficients psi_t T */
  double *vpsi;         /* [nstate][ng] coefficient velocities */
  double *T;            /* [nstate][nstate] last Newton-Schulz result */
  int iteration;        /* steps done; the call increments it */
  double dt;            /* time step (a.u.) */
  double ns_tol;        /* invsqr_tolerance (default 1e-15) */
  double norb_tol;      /* cp_norb_tol for the PsiV reset (default 0.003) */
  int ns_max_iter;      /* invsqr_max_iter */
  int mixed_nterm;      /* 0: FP64 GEMMs; 2 or 3: split-BF16 tcgen05 for Lambda, F', nonlocal */
  int use_graph;        /* replay the steady-state step as one CUDA graph */
  int last_ns_iters;    /* out */
  double last_ns_err;   /* out */
  double last_smax;     /* out: max |S - 2I| of this step */
  int last_kernels;     /* out: kernel launches of one step when it replays as a CUDA graph
                           (counted in the captured graph), else -1 */
  int psiv_pending;     /* in/out: the last step ended with a PsiV reset, so the next step
                           completes no half kick (halfStepEvolve = 0); 0 for a new run */
} oa_cp_state;

/* One whole CP dynamics step (GSpaceDriver::computeDynamics,
 * cp_state_ctrl/gspace.ci:199-324): forces, constraint force, Verlet
 * integration, orthonormalisation, in native code with one host
 * synchronisation at the end.  The PsiV reset triggered by max|S - 2I| >
 * norb_tol (Ortho::maxCheck, ortho.C:455-475) is decided on the device and
 * runs at the end of the step, as oa_gpu_psiv_reset would (the velocity
 * from the states before and after the rotation; the next step completes
 * no half kick).  energies_out (optional, host [14]):
 * EKE EHART EEXT EWALD_RECIP EEXC MUXC FICT_KE ENL, Newton-Schulz
 * iterations, residual, max|S - 2I|, EGGA (0 under PZ-LDA), the ionic
 * kinetic energy and the real-space Ewald energy with its self and
 * background terms (both 0 unless oa_gpu_set_ions turned ion dynamics on).  Coefficient arrays must be 16-byte
 * aligned. */
oa_status oa_gpu_cp_step(oa_ctx *ctx, void *stream, oa_cp_state *state, double *energies_out);

/* nsteps CP dynamics steps enqueued back to back with one host
 * synchronisation at the end: the loop of GSpaceDriver::computeDynamics
 * over a trajectory (the reference's per-step energy print,
 * InstanceController::printEnergy*, main/InstanceController.C:373-490,
 * becomes one record per step).  pos_host (optional, host
 * [nsteps][natm][3]) is copied to the atom positions before each step.
 * energies_out (optional, host [nsteps][14]) as oa_gpu_cp_step's.  When the
 * Newton-Schulz iteration fails in a step, the call still runs all nsteps
 * and returns OA_ERR_NOT_CONVERGED or OA_ERR_NONFINITE naming the first
 * failing step in oa_gpu_last_error(); the state is then that of the last
 * step. */
oa_status oa_gpu_cp_run(oa_ctx *ctx, void *stream, oa_cp_state *state, int nsteps, const double *pos_host,
                        double *energies_out);

/* Batching form: nsys independent systems (replicas, PIMD beads, tempering
 * systems; any sizes, one context and one state each) advanced nsteps CP
 * steps each.  After each system's first step, one step of all systems is
 * one CUDA graph: the systems' launches fork from `stream` (a created
 * stream, not the legacy default) onto one stream per system and join
 * back.  Results are those of oa_gpu_cp_run on each system alone.  The
 * reference runs such sets as separate instances (UberCollection /
 * InstanceController, main/InstanceController.C).  energies_out (optional,
 * host [nsys][nsteps][14]).  Needs at most 128 states per system (the whole
 * step captured); a Newton-Schulz failure names the first failing system
 * and step. */
oa_status oa_gpu_cp_run_batch(oa_ctx **ctxs, oa_cp_state **states, int nsys, void *stream, int nsteps,
                              double *energies_out);

/* Allocation-free PairCalculator forward product, for callers that cannot
 * call cudaMalloc (a host framework whose memory pool already holds the
 * device memory, or a latency-critical path that cannot take cudaMalloc's
 * implicit device synchronisation).  Same
 * result as oa_gpu_pc_forward, but it needs no context: the caller passes
 * the sizes (nstate <= 128, ng g-points, nkx0 points on the kx = 0 plane),
 * the device inputs left/right [nstate][ng] complex and the device output
 * C [nstate][nstate].  Its split-K scratch is a fixed 4 MiB device array
 * held by every GPU that loads the library until the process exits; calls
 * whose kernels overlap on one GPU race on it (calls on one stream are
 * ordered).  Larger nstate returns OA_ERR_BAD_ARG.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and
 * caches it for the process (no cudaDeviceReset while the library is
 * loaded).  No counterpart in the reference. */
oa_status oa_gpu_pc_forward_noalloc(void *stream, const double *left, const double *right, int nstate, int ng,
                                    int nkx0, double alpha, double w_kx0, double *C);

/* Set up the EES nonlocal path (cp_nonloc_ees_opt on): nonlocal grid
 * na x nb x nc (2^a 3^b 5^c, each >= order), B-spline order (even, 4..16),
 * and the per-g projector factor dyp(g) = d(g) y00 p(|g|) (host
 * [ng][2] doubles; eesSetEesWghtGgrp cp_ees_nonlocal.C:60-160 and
 * eesProjGchare 594-727).  Allocates the nonlocal-grid scratch. */
oa_status oa_gpu_ees_init(oa_ctx *ctx, int na, int nb, int nc, int order, const double *dyp);

/* Switch the local pseudopotential and the reciprocal Ewald sum to the EES
 * method (cp_eext_ees_opt on; replaces the per-step work of
 * CP_Rho_RHartExt / CP_Rho_GHartExt: eesAtmBsplineRgrp, eesPackGridRchare,
 * eesHartEextGchare, eesEwaldGchare, eesAtmForceRchare,
 * cp_hart_ext.C:641-1470, with eesSetEesWghtGgrp 521-635 and
 * get_bspline_wght1d set_cp_ewald.C:1237-1325 computed here).  Grid
 * na x nb x nc (2^a 3^b 5^c, <= 512, each >= order and > twice the largest
 * |k| of the density sphere; init_eext_ees set_cp_ewald.C:1419-1500 gives
 * the reference's choice), B-spline order even 4..16.  Every later density
 * pass (the stage entry points, oa_gpu_cp_step/run) uses it; with ion
 * dynamics the local and reciprocal Ewald atom forces come from it too.
 * na = nb = nc = 0 switches back to the structure-factor method.
 * Allocates two complex grids per two atom types. */
oa_status oa_gpu_set_ees_local(oa_ctx *ctx, int na, int nb, int nc, int order);

/* Nonlocal energy and coefficient forces by the EES method:
 * eesAtmBsplineRgrp (cp_ees_nonlocal.C:256-593), eesProjGchare + the
 * nonlocal-grid FFT (CP_State_ParticlePlane.C:867-1136), eesZmatRchare
 * (1238-1352) and its plane reduction, eesEnergyAtmForcRchare (1480-1720),
 * the inverse FFT and eesPsiForcGspace (2000-2079).  Same outputs as
 * oa_gpu_nl_sf. */
oa_status oa_gpu_nl_ees(oa_ctx *ctx, void *stream, const double *psi, double *fnl_out, double *enl_out);

/* Energies of the last vks_build / vks_apply_fft_bwd (synchronises):
 * out[0..10] = EKE, EHART, EEXT, EWALD_RECIP, EEXC, MUXC, FICT_KE, ENL, EGGA,
 * ION_KE, EWALD_REAL (the last two from the last native step with ions). */
oa_status oa_gpu_energies(oa_ctx *ctx, void *stream, double *out11);

/* Ion dynamics in the native step (oa_gpu_cp_step / oa_gpu_cp_run): each
 * step computes the forces on the atoms at their current positions -- the
 * local pseudopotential and reciprocal Ewald part of CP_hart_eext_calc
 * (cp_hart_ext.C:56-431, in the density z pass) or of the EES local path
 * (eesAtmForceRchare, cp_hart_ext.C:1357-1470; oa_gpu_set_ees_local), the
 * nonlocal part by the structure-factor method (CP_enl_atm_forc_calc,
 * cp_nl_energy_forc.C:178-235) or the EES method (eesEnergyAtmForcRchare,
 * cp_ees_nonlocal.C:1560-1720; oa_gpu_ees_init), and the real-space Ewald
 * sum of CPRSPACEION::CP_getionforce (cp_ions/cp_rspace_ion.C:25-251) -- and
 * moves them by the NVE integrator of AtomsCompute::integrateAtoms
 * (drv/main/AtomsCompute.C:461-640, integration_drivers.C:17-85): second
 * half kick of the previous step (not on a run's first step), first half
 * kick, drift.  masses: host [natm] in electron masses; vel: host [natm][3]
 * (null: zero).  oa_gpu_cp_run then takes no pos_host. */
oa_status oa_gpu_set_ions(oa_ctx *ctx, const double *masses, const double *vel);

/* Current atom positions and velocities (host [natm][3] each, either may be
 * null); synchronises. */
oa_status oa_gpu_get_ions(oa_ctx *ctx, void *stream, double *pos_out, double *vel_out);

/* Exchange-correlation functional of the density path (the reference's
 * \cp_ggax_typ / \cp_ggac_typ and \gradient_cutoff inputs,
 * interface/sim_params/set_sim_params.C:521-585, 803-808):
 *   functional 0: Perdew-Zunger LDA (CP_exc_calc, cp_pz_lda.C:23-175), the default;
 *   functional 1: BLYP = Slater exchange (the PZ correlation off, cp_pz_lda.C:66)
 *     + the Becke 88 / LYP gradient correction (CP_getGGAFunctional,
 *     cp_grad_rho_ctrl.C:32-190, becke_gcx_lda / lyp_gcc, cp_becke.C) with its
 *     grad rho and white-byrd divergence transforms (CP_Rho_GSpacePlane.C:278-380,
 *     CP_Rho_RealSpacePlane.C:1061-1350); EGGA is reported separately.
 * gradient_cutoff > 0 (the reference's default is 5e-5).  The first BLYP
 * call allocates 3 density grids and 3 density z-line sets. */
oa_status oa_gpu_set_xc(oa_ctx *ctx, int functional, double gradient_cutoff);

#ifdef __cplusplus
}
#endif
#endif
