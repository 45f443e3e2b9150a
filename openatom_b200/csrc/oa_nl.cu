// Nonlocal pseudopotential, structure-factor (N^2) method, l = 0 KB channel.
//
//   StructureFactor::computeSF (structure_factor/StructureFactor.C:35-113) ->
//     CPNONLOCAL::CP_calc_Struct_Fact (cp_struct_fact.C:37-255)        -> k_nl_sf
//   CP_State_ParticlePlane::computeZ/reduceZ (CP_State_ParticlePlane.C:500-600) ->
//     CPNONLOCAL::CP_enl_matrix_calc (cp_nlmat.C:24-100)              -> PairCalculator forward GEMM
//   CPNONLOCAL::CP_enl_atm_forc_calc (cp_nl_energy_forc.C:178-235)    -> k_nl_zscale
//   CP_State_ParticlePlane::getForces (:718) ->
//     CPNONLOCAL::CP_enl_force_calc (cp_nl_energy_forc.C:29-110)      -> PairCalculator backward GEMM
//
// SF[a][g] = w_g p_t(|g|) y00 conj(exp(i g.R_a)) is built in FP64 from the
// per-axis phase tables exp(i 2 pi k x_a / L) (the reference's incremental
// e^{i g.R} recursion becomes one product of three table entries).  In the
// mixed form the kernel also writes the bf16 planes of SF (oa_planes.cuh).
#include "oa_internal.h"
#include "oa_bspline.cuh"

__global__ void k_nl_sf(const int* __restrict__ kx, const int* __restrict__ ky, const int* __restrict__ kz, int ng,
                        const int* __restrict__ nl_atm, int natm_nl, const int* __restrict__ atm_type,
                        const double2* __restrict__ phase, int ktab, const double* __restrict__ spl, int nspl,
                        double gmin, double dg, const double* __restrict__ gz0, double tpi_l,
                        double2* __restrict__ sf, OaPlaneOut po) {
  const int a = blockIdx.y;
  const int at = nl_atm[a];
  const int t = atm_type[at];
  const int nt = 2 * ktab + 1;
  const double2* ph = phase + (size_t)at * 3 * nt;
  const double y00 = 0.28209479177387814347;  // 1 / sqrt(4 pi)
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const int x = kx[i], y = ky[i], z = kz[i];
    const double gx = tpi_l * x, gy = tpi_l * y, gzv = tpi_l * z;
    const double g = sqrt(gx * gx + gy * gy + gzv * gzv);
    double p;
    if (g != 0.0) {
      int ii = (int)((g - gmin) / dg) + 1;
      ii = min(ii, nspl); ii = max(ii, 1);
      const double hh = g - ((double)(ii - 1) * dg + gmin);
      const double* cc = spl + ((size_t)t * nspl + (ii - 1)) * 4;
      p = ((cc[3] * hh + cc[2]) * hh + cc[1]) * hh + cc[0];
    } else {
      p = gz0[t];
    }
    const double w = (x == 0) ? 1.0 : 2.0;
    const double2 h = cmul(cmul(ph[x + ktab], ph[nt + y + ktab]), ph[2 * nt + z + ktab]);
    const double s = w * p * y00;
    sf[(size_t)a * ng + i] = make_double2(h.x * s, -h.y * s);
    if (po.P) oa_plane_put2(po, a, 2L * i, h.x * s, -h.y * s);
  }
}

// ENL per state and the scaled, transposed, negated Z for the force GEMM:
// zt[a][s] = -2 vnorm_a / V Z[s][a]
__global__ void k_nl_zscale(const double* __restrict__ Z, int nstate, int natm_nl, const int* __restrict__ nl_atm,
                            const int* __restrict__ atm_type, const double* __restrict__ vnorm, double rvol,
                            const double* __restrict__ occ, double* __restrict__ zt, double* __restrict__ enl) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nstate) return;
  double e = 0.0;
  for (int a = 0; a < natm_nl; ++a) {
    const double vn = vnorm[atm_type[nl_atm[a]]] * rvol;
    const double z = Z[(size_t)s * natm_nl + a];
    e += z * z * vn;
    zt[(size_t)a * nstate + s] = -2.0 * vn * z;
  }
  enl[s] = e * occ[s];
}

cudaError_t oa_launch_nl_sf(cudaStream_t s, const int* kx, const int* ky, const int* kz, int ng, const int* nl_atm,
                            int natm_nl, const int* atm_type, const double2* phase, int ktab, const double* spl,
                            int nspl, double gmin, double dg, const double* gz0, double tpi_l, double2* sf,
                            const OaPlaneOut* po) {
  if (natm_nl == 0) return cudaSuccess;
  dim3 grid((ng + 255) / 256 < 64 ? (ng + 255) / 256 : 64, natm_nl);
  k_nl_sf<<<grid, 256, 0, s>>>(kx, ky, kz, ng, nl_atm, natm_nl, atm_type, phase, ktab, spl, nspl, gmin, dg, gz0,
                               tpi_l, sf, po ? *po : OaPlaneOut{nullptr, 0, 0, 0});
  return cudaGetLastError();
}

cudaError_t oa_launch_nl_zscale(cudaStream_t s, const double* Z, int nstate, int natm_nl, const int* nl_atm,
                                const int* atm_type, const double* vnorm, double rvol, const double* occ, double* zt,
                                double* enl) {
  k_nl_zscale<<<(nstate + 127) / 128, 128, 0, s>>>(Z, nstate, natm_nl, nl_atm, atm_type, vnorm, rvol, occ, zt, enl);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// EES: atom B-splines on the nonlocal grid and the Z reduction
// ---------------------------------------------------------------------------

// CPNONLOCAL::eesAtmBsplineRgrp (cp_ees_nonlocal.C:256-593): cardinal
// B-spline of order n at the fractional grid coordinate of each nonlocal atom,
// per axis, and (dmn not null) its derivative weights for the atom forces.
__global__ void k_ees_bspline(const double* __restrict__ pos, const int* __restrict__ nl_atm, int natm_nl, double box,
                              int na, int nb, int nc, int order, int* __restrict__ idx, double* __restrict__ mn,
                              double* __restrict__ dmn) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= natm_nl * 3) return;
  const int a = t / 3, ax = t - a * 3;
  const int ngrid = ax == 0 ? na : (ax == 1 ? nb : nc);
  const size_t o = ((size_t)a * 3 + ax) * order;
  ees_bspline_axis(pos[nl_atm[a] * 3 + ax], box, ngrid, order, idx + o, mn + o, dmn ? dmn + o : nullptr);
}

// Z = sum over stencil planes; ENL = occ vnorm/V sum Z^2; zs = 2 vnorm/V occ Z
// (eesEnergyAtmForcRchare, cp_ees_nonlocal.C:1480-1560)
__global__ void k_ees_zreduce(const double* __restrict__ zpart, int nstate, int natm_nl, int order,
                              const int* __restrict__ nl_atm, const int* __restrict__ atm_type,
                              const double* __restrict__ vnorm, double rvol, const double* __restrict__ occ,
                              double* __restrict__ zmat, double* __restrict__ zs, double* __restrict__ enl) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nstate) return;
  double e = 0.0;
  for (int a = 0; a < natm_nl; ++a) {
    double z = 0.0;
    for (int j = 0; j < order; ++j) z += zpart[((size_t)s * natm_nl + a) * order + j];
    const double vn = vnorm[atm_type[nl_atm[a]]] * rvol;
    zmat[(size_t)s * natm_nl + a] = z;
    e += z * z * vn;
    zs[(size_t)s * natm_nl + a] = 2.0 * vn * occ[s] * z;
  }
  enl[s] = e * occ[s];
}

cudaError_t oa_launch_ees_bspline(oa_ctx* c, cudaStream_t s) {
  oa_ees* e = c->ees;
  const int n = c->natm_nl * 3;
  k_ees_bspline<<<(n + 127) / 128, 128, 0, s>>>(c->pos, c->nl_atm, c->natm_nl, c->box, e->na, e->nb, e->nc, e->order,
                                                 e->idx, e->mn, c->ions ? e->dmn : nullptr);
  return cudaGetLastError();
}

cudaError_t oa_launch_ees_zreduce(oa_ctx* c, cudaStream_t s) {
  oa_ees* e = c->ees;
  k_ees_zreduce<<<(c->nstate + 127) / 128, 128, 0, s>>>(e->zpart, c->nstate, c->natm_nl, e->order, c->nl_atm,
                                                        c->atm_type, c->nl_vnorm, 1.0 / c->vol, c->occ, e->zmat, e->zs,
                                                        e->enl);
  return cudaGetLastError();
}
