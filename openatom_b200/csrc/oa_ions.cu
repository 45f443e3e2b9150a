// Ion side of the CP step: the nonlocal atom forces of the structure-factor
// method, the real-space Ewald sum and the NVE atom integration.
//
// Replaces:
//   CPNONLOCAL::CP_enl_atm_forc_calc (cp_nl_energy_forc.C:178-235) with the
//     derivative structure factors of CP_calc_Struct_Fact (cp_struct_fact.C)  -> GEMM + k_nl_sf_force
//   the atom-force loop of CPNONLOCAL::eesEnergyAtmForcRchare
//     (cp_ees_nonlocal.C:1560-1720), EES nonlocal method                      -> k_ees_atom_force
//     (the per-plane sums come from the Z gather, ees_gather_plane)
//   CPRSPACEION::CP_getionforce (cp_ions/cp_rspace_ion.C:25-251)              -> k_ewald_rspace
//   AtomsCompute::integrateAtoms (drv/main/AtomsCompute.C:461-640) ->
//     ATOMINTEGRATE::integrate_nve_2nd_half / integrate_nve_1st_half
//     (classical_physics/integrate/integration_drivers.C:17-85)             -> k_ion_integrate
// The local pseudopotential and reciprocal Ewald forces come from the
// density z pass (k_rho_zpass<..., true>, oa_rho.cu), one partial per z-pass
// block, or with the EES local path from k_eesl_force (oa_eesl.cu) in the
// first partial.
#include <stdlib.h>
#include <string.h>
#include <vector>
#include "oa_internal.h"

static __device__ __forceinline__ double ion_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// deterministic block sum of 3 values (blockDim.x a multiple of 32, <= 1024);
// the result is valid in thread 0
static __device__ void ion_block_sum3(double v[3], double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = 0; k < 3; ++k) v[k] = ion_warp_sum(v[k]);
  __syncthreads();
  if (lane == 0)
    for (int k = 0; k < 3; ++k) sh[k * 32 + wid] = v[k];
  __syncthreads();
  if (wid == 0)
    for (int k = 0; k < 3; ++k) v[k] = ion_warp_sum(lane < nw ? sh[k * 32 + lane] : 0.0);
}

// F_a = -2 vnorm_a / V sum_g g (Y.x SF.y - Y.y SF.x), Y = sum_s Z[s][a] psi_s:
// dZ/dR_a of SF_a(g) = w p y00 conj(e^{i g.R_a}) is -i g SF_a.  One block per
// nonlocal atom; writes that atom's row of fnl (the others stay zero).
__global__ void k_nl_sf_force(const double2* __restrict__ y, const double2* __restrict__ sf, int ng,
                              const int* __restrict__ kx, const int* __restrict__ ky, const int* __restrict__ kz,
                              double tpi_l, const int* __restrict__ nl_atm, const int* __restrict__ atm_type,
                              const double* __restrict__ vnorm, double rvol, double* __restrict__ fnl) {
  __shared__ double sh[3 * 32];
  const int a = blockIdx.x;
  const double2* ya = y + (size_t)a * ng;
  const double2* sa = sf + (size_t)a * ng;
  double f[3] = {0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < ng; i += blockDim.x) {
    const double2 yy = ya[i], ss = sa[i];
    const double c = yy.x * ss.y - yy.y * ss.x;
    f[0] += kx[i] * c;
    f[1] += ky[i] * c;
    f[2] += kz[i] * c;
  }
  ion_block_sum3(f, sh);
  if (threadIdx.x == 0) {
    const int at = nl_atm[a];
    const double s = -2.0 * vnorm[atm_type[at]] * rvol * tpi_l;
    fnl[3 * at + 0] = s * f[0];
    fnl[3 * at + 1] = s * f[1];
    fnl[3 * at + 2] = s * f[2];
  }
}

// EES nonlocal atom forces (eesEnergyAtmForcRchare's force loop,
// cp_ees_nonlocal.C:1560-1720): F_a = -sum_s zs[s][a] sum over the stencil
// planes of the gathered sums (x n_a / L, y n_b / L, z n_c / L), with zs the
// scaled Z = 2 vnorm / V occ Z.  One block per nonlocal atom.
__global__ void k_ees_atom_force(const double* __restrict__ fpart, const double* __restrict__ zs, int nstate,
                                 int natm_nl, int order, const int* __restrict__ nl_atm, double sa, double sb,
                                 double sc, double* __restrict__ fnl) {
  __shared__ double sh[3 * 32];
  const int a = blockIdx.x;
  double f[3] = {0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < nstate * order; i += blockDim.x) {
    const int s = i / order, jc = i - s * order;
    const double z = zs[(size_t)s * natm_nl + a];
    const double* fp = fpart + (((size_t)s * natm_nl + a) * order + jc) * 3;
    f[0] += z * fp[0];
    f[1] += z * fp[1];
    f[2] += z * fp[2];
  }
  ion_block_sum3(f, sh);
  if (threadIdx.x == 0) {
    const int at = nl_atm[a];
    fnl[3 * at + 0] = -sa * f[0];
    fnl[3 * at + 1] = -sb * f[1];
    fnl[3 * at + 2] = -sc * f[2];
  }
}

// erfc(x) ~ t P(t) e^{-x^2}, t = 1 / (1 + p x), with the polynomial of
// CP_getionforce (cp_rspace_ion.C:36-45); *dq = t^2 e^{-x^2} sum_k k e_k t^(k-1)
static __device__ __forceinline__ double ewald_erfc(double x, double* dq) {
  const double p = 0.3614;
  const double e[9] = {0.2041422096422003, 0.1997535956961481, 0.2213176596405576, 0.03360430734640255,
                       0.4732592578721755, -0.509078520069735, 0.6772631491947646, -0.369912979092217,
                       0.06965131976970335};
  const double t = 1.0 / (1.0 + p * x);
  const double eee = exp(-x * x);
  double poly = 0.0, dpoly = 0.0;
#pragma unroll
  for (int k = 8; k >= 0; --k) {
    poly = poly * t + e[k];
    dpoly = dpoly * t + (k + 1) * e[k];
  }
  *dq = dpoly * t * t * eee;
  return poly * t * eee;
}

// Real-space Ewald on a cubic box: one block per atom i, threads over j;
// the pair (i, j) at its minimum image, within half the box.  fr[i] is the
// force on i from every j; er[i] the energy of the pairs j > i.
__global__ void k_ewald_rspace(const double* __restrict__ pos, const int* __restrict__ atm_type,
                               const double* __restrict__ q_type, int natm, double box, double alp,
                               double* __restrict__ fr, double* __restrict__ er) {
  __shared__ double sh[3 * 32];
  __shared__ double she[32];
  const int i = blockIdx.x;
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
  const double qi = q_type[atm_type[i]];
  const double palp = 0.3614 * alp, talp2 = 2.0 * alp * alp, half = 0.5 * box, rbox = 1.0 / box;
  double f[3] = {0.0, 0.0, 0.0};
  double e = 0.0;
  for (int j = threadIdx.x; j < natm; j += blockDim.x) {
    if (j == i) continue;
    double dx = xi - pos[3 * j], dy = yi - pos[3 * j + 1], dz = zi - pos[3 * j + 2];
    dx -= box * rint(dx * rbox);
    dy -= box * rint(dy * rbox);
    dz -= box * rint(dz * rbox);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double r = sqrt(r2);
    if (r > half) continue;
    const double qij = qi * q_type[atm_type[j]];
    double dq;
    const double ge = ewald_erfc(r * alp, &dq);
    const double dge = dq * palp + talp2 * ge * r;
    const double dv = (ge / r2 + dge / r) * qij / r;
    f[0] += dx * dv;
    f[1] += dy * dv;
    f[2] += dz * dv;
    if (j > i) e += qij * ge / r;
  }
  ion_block_sum3(f, sh);
  e = ion_warp_sum(e);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) she[wid] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += she[w];
    er[i] = t;
    fr[3 * i] = f[0];
    fr[3 * i + 1] = f[1];
    fr[3 * i + 2] = f[2];
  }
}

// NVE atom integration, one block: F = sum of the z-pass partials (fixed
// block order) + nonlocal + real-space Ewald; the second half kick of the
// previous step (kick2), the kinetic energy, the first half kick and the
// drift.  Also the Ewald real-space total: sum_i er[i] + self + background.
__global__ void k_ion_integrate(double* __restrict__ pos, double* __restrict__ v, const double* __restrict__ m,
                                const double* __restrict__ fpart, int nfpart, const double* __restrict__ fnl,
                                const double* __restrict__ fr, const double* __restrict__ er, int natm, double dt,
                                int kick2, double e_self_bgr, double* __restrict__ dev_e) {
  __shared__ double sh[2 * 32];
  double ke = 0.0, ee = 0.0;
  for (int a = threadIdx.x; a < natm; a += blockDim.x) {
    double F[3];
    for (int c = 0; c < 3; ++c) F[c] = fnl[3 * a + c] + fr[3 * a + c];
    for (int b = 0; b < nfpart; ++b)
      for (int c = 0; c < 3; ++c) F[c] += fpart[((size_t)b * natm + a) * 3 + c];
    const double h = 0.5 * dt / m[a];
    double vv[3];
    for (int c = 0; c < 3; ++c) {
      vv[c] = v[3 * a + c];
      if (kick2) vv[c] += h * F[c];
    }
    ke += 0.5 * m[a] * (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]);
    for (int c = 0; c < 3; ++c) {
      vv[c] += h * F[c];
      v[3 * a + c] = vv[c];
      pos[3 * a + c] += dt * vv[c];
    }
    ee += er[a];
  }
  ke = ion_warp_sum(ke);
  ee = ion_warp_sum(ee);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) { sh[wid] = ke; sh[32 + wid] = ee; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double k = 0.0, e = 0.0;
    for (int w = 0; w < nw; ++w) { k += sh[w]; e += sh[32 + w]; }
    dev_e[OA_E_ION_KE] = k;
    dev_e[OA_E_EWALD_REAL] = e + e_self_bgr;
  }
}

cudaError_t oa_launch_pc_bwd_jk(cudaStream_t s, const double* M1, const double* X1, double a1_kx0, double a1_rest,
                                const double* M2, const double* X2, double a2, int nj, int nk, long ncol,
                                long kx0_cols, double* out);

// Y = Z^T psi (FP64 DMMA backward product, Z [nstate][natm_nl]) and the
// per-atom force sums
cudaError_t oa_launch_nl_sf_force(oa_ctx* c, cudaStream_t s, const double* psi) {
  oa_ions* io = c->ions;
  if (!io) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(io->fnl, 0, (size_t)3 * c->natm * sizeof(double), s);
  if (e != cudaSuccess || c->natm_nl == 0) return e;
  const long K = 2L * c->ng;
  e = oa_launch_pc_bwd_jk(s, c->zmat, psi, 1.0, 1.0, nullptr, nullptr, 0.0, c->natm_nl, c->nstate, K, 0, io->y);
  if (e != cudaSuccess) return e;
  k_nl_sf_force<<<c->natm_nl, 256, 0, s>>>((const double2*)io->y, c->sf, c->ng, c->kx, c->ky, c->kz,
                                           2.0 * 3.14159265358979323846 / c->box, c->nl_atm, c->atm_type,
                                           c->nl_vnorm, 1.0 / c->vol, io->fnl);
  return cudaGetLastError();
}

// the self and background Ewald terms of CP_getionforce (cp_rspace_ion.C:218-245)
static double ewald_self_bgr(const oa_ctx* c, const double* q_host) {
  double q2 = 0.0, qs = 0.0;
  for (int a = 0; a < c->natm; ++a) { q2 += q_host[a] * q_host[a]; qs += q_host[a]; }
  const double pi = 3.14159265358979323846, alp = c->alp_ewd;
  const double vself = -(q2 * alp) / sqrt(pi);
  const double vbgr = -(0.5 * qs * qs * pi) / (alp * alp * c->vol);
  // erf(k_cut / 2 alpha) of the finite reciprocal sum, k_cut the density-sphere radius
  const double x = sqrt(c->ecut_rho) / (2.0 * alp);
  const double p = 0.3614;
  const double e[9] = {0.2041422096422003, 0.1997535956961481, 0.2213176596405576, 0.03360430734640255,
                       0.4732592578721755, -0.509078520069735, 0.6772631491947646, -0.369912979092217,
                       0.06965131976970335};
  const double t = 1.0 / (1.0 + p * x);
  double poly = 0.0;
  for (int k = 8; k >= 0; --k) poly = poly * t + e[k];
  const double erfc_x = poly * t * exp(-x * x);
  return vself * (1.0 - erfc_x) + vbgr;
}

cudaError_t oa_launch_ees_atom_force(oa_ctx* c, cudaStream_t s) {
  oa_ions* io = c->ions;
  const oa_ees* e = c->ees;
  cudaError_t err = cudaMemsetAsync(io->fnl, 0, (size_t)3 * c->natm * sizeof(double), s);
  if (err != cudaSuccess) return err;
  if (c->natm_nl == 0) return cudaSuccess;
  k_ees_atom_force<<<c->natm_nl, 128, 0, s>>>(e->fpart, e->zs, c->nstate, c->natm_nl, e->order, c->nl_atm,
                                              (double)e->na / c->box, (double)e->nb / c->box, (double)e->nc / c->box,
                                              io->fnl);
  return cudaGetLastError();
}

// the real-space Ewald sum and the integration, at the end of a step's
// force work (the next step's phase tables see the new positions)
cudaError_t oa_launch_ion_step(oa_ctx* c, cudaStream_t s, double* dev_e, double dt, int kick2) {
  oa_ions* io = c->ions;
  if (!io) return cudaSuccess;
  k_ewald_rspace<<<c->natm, 128, 0, s>>>(c->pos, c->atm_type, c->q_type, c->natm, c->box, c->alp_ewd, io->fr,
                                         io->er);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_ion_integrate<<<1, 256, 0, s>>>(c->pos, io->v, io->m, io->fpart, c->eesl ? 1 : io->nfpart, io->fnl, io->fr,
                                    io->er, c->natm, dt, kick2, io->self_bgr, dev_e);
  return cudaGetLastError();
}

#define OA_ION_TRY(x)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) { oa_set_error(cudaGetErrorString(e_), __FILE__, __LINE__); return OA_ERR_CUDA; } \
  } while (0)

int oa_rho_z_nblk(const oa_ctx* c);

extern "C" oa_status oa_gpu_set_ions(oa_ctx* c, const double* masses, const double* vel) {
  if (!c || !masses) {
    oa_set_error("null argument", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  for (int a = 0; a < c->natm; ++a)
    if (!(masses[a] > 0.0)) {
      oa_set_error("atom masses must be > 0", __FILE__, __LINE__);
      return OA_ERR_BAD_ARG;
    }
  oa_ions* io = c->ions;
  if (!io) {
    io = (oa_ions*)calloc(1, sizeof(oa_ions));
    if (!io) { oa_set_error("out of host memory", __FILE__, __LINE__); return OA_ERR_CUDA; }
    c->ions = io;
    io->nfpart = oa_rho_z_nblk(c);
    OA_ION_TRY(cudaMalloc(&io->m, (size_t)c->natm * sizeof(double)));
    OA_ION_TRY(cudaMalloc(&io->v, (size_t)3 * c->natm * sizeof(double)));
    OA_ION_TRY(cudaMalloc(&io->fpart, (size_t)io->nfpart * 3 * c->natm * sizeof(double)));
    OA_ION_TRY(cudaMalloc(&io->fnl, (size_t)3 * c->natm * sizeof(double)));
    OA_ION_TRY(cudaMalloc(&io->fr, (size_t)3 * c->natm * sizeof(double)));
    OA_ION_TRY(cudaMalloc(&io->er, (size_t)c->natm * sizeof(double)));
    OA_ION_TRY(cudaMalloc(&io->y, ((size_t)2 * c->natm_nl * c->ng + 1) * sizeof(double)));
    OA_ION_TRY(cudaMemset(io->fpart, 0, (size_t)io->nfpart * 3 * c->natm * sizeof(double)));
    // per-atom charges on the host for the self and background terms
    std::vector<int> at(c->natm);
    std::vector<double> qt(c->ntype);
    OA_ION_TRY(cudaMemcpy(at.data(), c->atm_type, (size_t)c->natm * sizeof(int), cudaMemcpyDeviceToHost));
    OA_ION_TRY(cudaMemcpy(qt.data(), c->q_type, (size_t)c->ntype * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<double> q(c->natm);
    for (int a = 0; a < c->natm; ++a) q[a] = qt[at[a]];
    io->self_bgr = ewald_self_bgr(c, q.data());
  }
  OA_ION_TRY(cudaMemcpy(io->m, masses, (size_t)c->natm * sizeof(double), cudaMemcpyHostToDevice));
  if (vel) OA_ION_TRY(cudaMemcpy(io->v, vel, (size_t)3 * c->natm * sizeof(double), cudaMemcpyHostToDevice));
  else OA_ION_TRY(cudaMemset(io->v, 0, (size_t)3 * c->natm * sizeof(double)));
  c->xc_gen += 1;  // the captured step graph gains the ion kernels
  return OA_OK;
}

extern "C" oa_status oa_gpu_get_ions(oa_ctx* c, void* stream, double* pos_out, double* vel_out) {
  if (!c) {
    oa_set_error("null argument", __FILE__, __LINE__);
    return OA_ERR_BAD_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (pos_out) OA_ION_TRY(cudaMemcpyAsync(pos_out, c->pos, (size_t)3 * c->natm * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (vel_out) {
    if (c->ions)
      OA_ION_TRY(cudaMemcpyAsync(vel_out, c->ions->v, (size_t)3 * c->natm * sizeof(double), cudaMemcpyDeviceToHost, s));
    else
      memset(vel_out, 0, (size_t)3 * c->natm * sizeof(double));
  }
  OA_ION_TRY(cudaStreamSynchronize(s));
  return OA_OK;
}

void oa_ions_free(oa_ctx* c) {
  oa_ions* io = c->ions;
  if (!io) return;
  void* d[] = {io->m, io->v, io->fpart, io->fnl, io->fr, io->er, io->y};
  for (void* q : d) if (q) cudaFree(q);
  free(io);
  c->ions = nullptr;
}
