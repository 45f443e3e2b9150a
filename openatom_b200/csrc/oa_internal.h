// Internal context of liboa_gpu: device tables, plans and scratch for one
// Gamma-point system on one GPU.  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "oa_fft.cuh"
#include "oa_planes.cuh"
#include "../../include/oa_gpu.h"

#define OA_NTHREADS 256
#define OA_LB 16          // z-lines per block in the z passes
#define OA_MAX_SMEM (227 * 1024)

// Raise a kernel's dynamic shared-memory limit to the most a block can have
// beside its static shared memory.  The limit is a per-function setting that
// all launches share (graphs holding systems of several sizes included), so
// it is never lowered to one launch's need.
template <typename K>
static inline cudaError_t oa_smem_limit(K kernel) {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, (const void*)kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(OA_MAX_SMEM - a.sharedSizeBytes));
}

// EES nonlocal path (nonlocal grid na x nb x nc, B-spline order)
struct oa_ees {
  int na, nb, nc, order, ngroup;
  OaFftPlan pa, pb, pc;
  double2 *tw_a, *tw_b, *tw_c;
  void* zbuf;          // [nstate][nc][ldl] compute precision
  double2* dyp;        // [ng] d(g) y00 p(|g|)
  int* idx;            // [natm_nl][3][order]
  double* mn;          // [natm_nl][3][order]
  double* zpart;       // [nstate][natm_nl][order]
  double* zmat;        // [nstate][natm_nl]
  double* zs;          // [nstate][natm_nl]
  double* enl;         // [nstate]
  double* dmn;         // [natm_nl][3][order] B-spline derivative weights (ion dynamics)
  double* fpart;       // [nstate][natm_nl][order][3] per-plane atom-force sums (ion dynamics)
};

// EES local pseudopotential and reciprocal Ewald path (oa_gpu_set_ees_local,
// cp_eext_ees_opt on): grid na x nb x nc, B-spline order; atom types 2k and
// 2k+1 share complex grid k (real and imaginary part)
struct oa_eesl {
  int na, nb, nc, order, ngrid;
  OaFftPlan pa, pb, pc;
  double2 *tw_a, *tw_b, *tw_c;
  double2 *ba, *bb, *bc;   // 1-D B-spline factors b(m), m = 0..n-1 (get_bspline_wght1d)
  double2* zq;             // [ngrid][nc][nb][na]: type grids, then their transform
  double2* zy;             // [ngrid][nc][nb][na]: force transforms, then the force grids
  double* gzvps;           // [ntype]
};

// What the density z pass reads of the EES local path (zq = null: the
// structure-factor path)
struct EesLocArgs {
  const double2* zq;
  double2* zy;             // forces: written at the sphere points (zeroed before)
  const double2 *ba, *bb, *bc;
  const double* gzvps;
  int na, nb, nc;
  size_t gstride;          // na nb nc
};

// Per-block charge partials of the mixed z forward pass: sum over the
// block's coefficients of occ_s w |c|^2 (w = 1 on the kx = 0 lines, whose
// two halves are both stored, 2 elsewhere); part = null: none
struct OaCharge {
  const int* line_kx;
  const double* occ;
  double* part;
};

// Ion dynamics (oa_gpu_set_ions): masses, velocities and the force pieces of
// one step, summed by the integrator in a fixed order
struct oa_ions {
  double* m;        // [natm] electron masses
  double* v;        // [natm][3]
  double* fpart;    // [z-pass blocks][natm][3] local pseudopotential + reciprocal Ewald
  double* fnl;      // [natm][3] nonlocal (structure-factor method)
  double* fr;       // [natm][3] real-space Ewald
  double* er;       // [natm] real-space Ewald energy per atom i (pairs j > i)
  double* y;        // [natm_nl][2 ng] sum_s Z[s][a] psi_s (nonlocal force product)
  int nfpart;       // z-pass blocks
  double self_bgr;  // Ewald self + background terms (constant for fixed charges and box)
};

struct oa_ctx {
  int device;
  int precision;          // OA_FP64 or OA_MIXED
  int nx, ny, nz, npts;
  int ng, nlines, ldl;    // g-points, state z-lines, padded line stride
  int nstate, natm, ntype;
  int nkx0, nkx0_red, nkx0_uni, nkx0_zero;
  int nkx_s;              // state sphere x-columns (max line kx + 1)
  int nkx_d;              // density half-spectrum columns (nx/2 + 1)
  int nlines_d, ldl_d;    // density z-lines (nkx_d * ny) and padded stride
  int ngroup;             // state groups in the plane kernels
  int ngroup_pair;        // pair groups in the state-pair plane kernels
  int rho_ngroup;         // groups summed in rho_part by the last density pass
  int* pair_cols;         // [nkx_s] {first line, ky of the first line, lines, 0}: FP32 pair kernels
  int pair_kymax;         // largest |ky| of the state lines
  int z_ext;              // largest kz count of a state line on either side (max of nneg, npos)
  void* psir;             // psi(r), compute precision: [nstate][nz][ny][nx] (two-pass kernels)
                          // or [nstate/2][nz][ny][nx] pairs (state-pair kernels)
  int psir_valid;         // the last density pass stored psir: 1 per state, 2 per pair
  double box, vol, ecut_psi, ecut_rho, alp_ewd;
  double gzvps_sum;
  int nspl; double spl_gmin, spl_dg;
  int kmax_tab;           // phase table half-width
  OaFftPlan plan_x, plan_y, plan_z;
  // device tables
  int *line_kx, *line_ky, *line_off, *line_nneg, *line_npos;
  int *kx;                // per g-point
  double *g2;             // per g-point
  double2 *tw_x, *tw_y, *tw_z;
  double *spl;            // [ntype][nspl][4]
  double *q_type;         // [ntype]
  int *atm_type;          // [natm]
  int *atm_perm;          // [natm] atom ids grouped by type (stable)
  int type_off[5];        // atoms of type t: atm_perm[type_off[t] .. type_off[t+1])
  double *pos;            // [natm][3]
  double2 *phase;         // [natm][3][2*kmax_tab+1] exp(i 2 pi k x / L)
  double *occ;            // [nstate]
  int *ky, *kz;           // per g-point
  int natm_nl;
  int *nl_atm;            // [natm_nl]
  double *nl_spl, *nl_vnorm, *nl_gz0;
  double2 *sf;            // [natm_nl][ng] structure factor x projector
  double *zmat, *zt, *enl;
  double *enl_eke;        // [nstate] per-state EKE scratch
  // scratch (FFT path precision R; byte sizes)
  void *zbuf;             // [nstate][nz][ldl] C
  size_t zbuf_bytes;
  double *rho_part;       // [ngroup][nz][ny][nx] double (FP64 accumulate)
  double *rho;            // [nz][ny][nx]
  void *vks;              // [nz][ny][nx] R
  double *vxc;            // [nz][ny][nx]
  void *dz;               // [nz][ldl_d] C  (density z-lines)
  double *red;            // reduction partials
  size_t red_len;
  double *eke_part;       // [nstate][nblk_z]
  int nblk_z;
  int zseg;               // longest coefficient run of one z-pass block of
                          // OA_LB lines when the lines are packed back to
                          // back (staged in shared memory), else 0
  double energies[8];
  void *step;             // native-step scratch and captured graph (oa_step.cu)
  oa_ees *ees;            // EES nonlocal path, after oa_gpu_ees_init
  size_t smem_plane, smem_rho_plane;
  OaPlaneOut zb_po;       // bf16 planes the next force z pass also writes (mixed native step), P = nullptr: none
  int zb_po_done;         // the last force z pass wrote them
  int npair_d, ychunk_d;
  // exchange-correlation: gga = 0 Perdew-Zunger LDA, 1 BLYP (Slater
  // exchange + Becke 88 + LYP, oa_gpu_set_xc); gga_cut = \gradient_cutoff
  int gga;
  double gga_cut;
  unsigned xc_gen;        // bumped by every oa_gpu_set_xc (captured step graphs key on it)
  double *grad;           // [3][nz][ny][nx] grad rho, then the GGA vector h (BLYP)
  void *dzg;              // [3][nz][ldl_d] C  z-lines of grad rho / h (BLYP)
  oa_ions *ions;          // ion dynamics, after oa_gpu_set_ions
  oa_eesl *eesl;          // EES local path, after oa_gpu_set_ees_local
  int eesl_gen;           // bumped by every oa_gpu_set_ees_local (captured graphs depend on it)
  int fft_runtime;        // oa_tuning fft_path 2: runtime-plan transforms for the state path
  int rho_groups_cap;     // groups the density partials are allocated for
  int nq2_cap;            // entries of qpart2 allocated
  double gzvps_t[4];      // g = 0 limit of the local part per type
  // mixed form: the FP32 density renormalised to the exact electron count
  // (charge partials of the z forward pass and of the pair density pass)
  double *qpart, *qpart2, *qscale;
  int nq, nq2;
  int qvalid;             // the last density pass wrote both partial sets
};

enum { OA_E_EKE = 0, OA_E_EHART, OA_E_EEXT, OA_E_EWALD, OA_E_EEXC, OA_E_MUXC, OA_E_ENL, OA_E_FICT };
#define OA_E_EGGA 10      // device energy slot of EGGA (slots 8, 9 hold the EEXC halves)
#define OA_E_ION_KE 13    // ionic kinetic energy (ion dynamics)
#define OA_E_EWALD_REAL 14  // real-space Ewald + self + background terms (ion dynamics)
cudaError_t oa_launch_phase_tables(oa_ctx* c, cudaStream_t s);

#define OA_CUDA_TRY(x)                                  \
  do {                                                  \
    cudaError_t e_ = (x);                               \
    if (e_ != cudaSuccess) { oa_set_error(cudaGetErrorString(e_), __FILE__, __LINE__); return OA_ERR_CUDA; } \
  } while (0)

void oa_set_error(const char* msg, const char* file, int line);

// stage launchers (return cudaError_t)
cudaError_t oa_launch_state_zfwd(oa_ctx* c, cudaStream_t s, const double2* psi, int s0, int ns);
cudaError_t oa_launch_state_plane_density(oa_ctx* c, cudaStream_t s);
cudaError_t oa_launch_state_plane_vks(oa_ctx* c, cudaStream_t s);
cudaError_t oa_launch_state_zbwd(oa_ctx* c, cudaStream_t s, const double2* psi, const double2* fnl,
                                 double2* force, int s0, int ns);
cudaError_t oa_launch_rho_xc(oa_ctx* c, cudaStream_t s);
cudaError_t oa_launch_rho_fft_hart(oa_ctx* c, cudaStream_t s);
cudaError_t oa_launch_ees(oa_ctx* c, cudaStream_t s, const double2* psi, double2* fnl);
cudaError_t oa_launch_ees_zreduce(oa_ctx* c, cudaStream_t s);
cudaError_t oa_launch_ees_bspline(oa_ctx* c, cudaStream_t s);
cudaError_t oa_launch_nl_sf_force(oa_ctx* c, cudaStream_t s, const double* psi);
cudaError_t oa_launch_ees_atom_force(oa_ctx* c, cudaStream_t s);
cudaError_t oa_launch_eesl_front(oa_ctx* c, cudaStream_t s);
cudaError_t oa_launch_eesl_forces(oa_ctx* c, cudaStream_t s);
void oa_eesl_free(oa_ctx* c);
cudaError_t oa_launch_ion_step(oa_ctx* c, cudaStream_t s, double* dev_e, double dt, int kick2);
size_t oa_plane_smem_bytes(int precision, int nx, int ny, int nkx);
