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
// e^{i g.R} recursion becomes one product of three table entries).
#include "oa_internal.h"

__global__ void k_nl_sf(const int* __restrict__ kx, const int* __restrict__ ky, const int* __restrict__ kz, int ng,
                        const int* __restrict__ nl_atm, int natm_nl, const int* __restrict__ atm_type,
                        const double2* __restrict__ phase, int ktab, const double* __restrict__ spl, int nspl,
                        double gmin, double dg, const double* __restrict__ gz0, double tpi_l,
                        double2* __restrict__ sf) {
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
                            int nspl, double gmin, double dg, const double* gz0, double tpi_l, double2* sf) {
  if (natm_nl == 0) return cudaSuccess;
  dim3 grid((ng + 255) / 256 < 64 ? (ng + 255) / 256 : 64, natm_nl);
  k_nl_sf<<<grid, 256, 0, s>>>(kx, ky, kz, ng, nl_atm, natm_nl, atm_type, phase, ktab, spl, nspl, gmin, dg, gz0,
                               tpi_l, sf);
  return cudaGetLastError();
}

cudaError_t oa_launch_nl_zscale(cudaStream_t s, const double* Z, int nstate, int natm_nl, const int* nl_atm,
                                const int* atm_type, const double* vnorm, double rvol, const double* occ, double* zt,
                                double* enl) {
  k_nl_zscale<<<(nstate + 127) / 128, 128, 0, s>>>(Z, nstate, natm_nl, nl_atm, atm_type, vnorm, rvol, occ, zt, enl);
  return cudaGetLastError();
}
