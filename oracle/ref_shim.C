// oracle/_ref shim: serial entry points into the reference's own PINY physics
// routines (compiled from the reference tree by oracle/build_ref.sh), used
// only by the tests to pin the numpy oracle.  TEST INFRASTRUCTURE ONLY.
//
// It defines the PINY singletons the routines read (allclass_*.h
// readonly_cp / readonly_general_data / readonly_mdatoms), fills the fields
// each routine uses from plain arrays, and provides genmatmul_ with the
// DGEMM semantics of src_mathlib/genmatmul.f.
#include "standard_include.h"
#include "ckcomplex.h"
#include "../../../include/Atoms.h"
#include "../../../include/eesDataClass.h"
#include "../class_defs/allclass_gen.h"
#include "../class_defs/allclass_cp.h"
#include "../class_defs/allclass_mdatoms.h"
#include "../class_defs/CP_OPERATIONS/class_cpnonlocal.h"
#include "../class_defs/CP_OPERATIONS/class_cpxcfnctls.h"
#include "../class_defs/CP_OPERATIONS/class_cplocal.h"
#include "../class_defs/CP_OPERATIONS/class_cporthog.h"
#include <vector>

// PINY allocators (friend_lib) as plain malloc/free
void* cmalloc(size_t n, const char*) { return std::malloc(n ? n : 1); }
void cfree(void* p, const char*) { std::free(p); }

// Symbols the compiled files reference on paths the oracle never takes:
// timers, the EISPACK eigen-solver of get_diag_Tmat, the EES B-spline
// setup of the EES Hartree variant, and the wave generator's class.
void cputime(double* t) { *t = 0.0; }
extern "C" void rs_(int*, int*, double*, double*, int*, double*, double*, double*, int*) {
  std::fprintf(stderr, "oracle/_ref: rs_ (EISPACK) is not provided\n");
  std::abort();
}
void get_bspline_wght1d(int, int, double*, double*, double*, double*, double*, double*, double*, double*) {
  std::fprintf(stderr, "oracle/_ref: EES B-spline setup is not provided\n");
  std::abort();
}
GEN_WAVE::GEN_WAVE() {}
GEN_WAVE::~GEN_WAVE() {}

CP readonly_cp;
GENERAL_DATA readonly_general_data;
MDATOMS readonly_mdatoms;

// C(ldz) = alpha op(X) op(Y) + beta C, column-major, op = 'T' for ityp 0
extern "C" void genmatmul_(double* X, int* ldx, int* ityp_x, double* Y, int* ldy, int* ityp_y, double* Z, int* ldz,
                           int* nrz, int* ncz, int* nxy, double* alpha, double* beta) {
  const int m = *nrz, n = *ncz, k = *nxy;
  std::vector<double> out((size_t)m * n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int l = 0; l < k; ++l) {
        const double x = (*ityp_x == 0) ? X[l + (size_t)i * *ldx] : X[i + (size_t)l * *ldx];
        const double y = (*ityp_y == 0) ? Y[j + (size_t)l * *ldy] : Y[l + (size_t)j * *ldy];
        s += x * y;
      }
      out[i + (size_t)j * m] = s;
    }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      double& z = Z[i + (size_t)j * *ldz];
      z = *alpha * out[i + (size_t)j * m] + (*beta == 0.0 ? 0.0 : *beta * z);
    }
}

static void set_cell(double box) {
  GENCELL* gc = &readonly_general_data.gencell;
  for (int i = 1; i <= 9; ++i) gc->hmati[i] = 0.0, gc->hmat[i] = 0.0;
  gc->hmat[1] = gc->hmat[5] = gc->hmat[9] = box;
  gc->hmati[1] = gc->hmati[5] = gc->hmati[9] = 1.0 / box;
  gc->vol = box * box * box;
}

// CPNONLOCAL::CP_eke_calc for one state (cp_eke.C:30-140)
extern "C" void ref_eke(int ncoef, const double* psi, double* forces, const int* kx, const int* ky, const int* kz,
                        const double* g2, double ecut_psi, double occ, int nkx0, double box, double* eke) {
  set_cell(box);
  CPCOEFFS_INFO* ci = &readonly_cp.cpcoeffs_info;
  static double occ_up[2], wkpt[2];
  occ_up[1] = occ; wkpt[1] = 1.0;
  ci->ecut_psi = ecut_psi;
  ci->occ_up = occ_up;
  ci->wght_kpt = wkpt;
  double* g2p[1] = {const_cast<double*>(g2)};
  CPNONLOCAL::CP_eke_calc(ncoef, 0, (complex*)forces, (complex*)const_cast<double*>(psi), const_cast<int*>(kx),
                          const_cast<int*>(ky), const_cast<int*>(kz), g2p, eke, 1, nkx0, 0, 1);
}

// CPXCFNCTS::CP_exc_calc (cp_pz_lda.C:23-175) on an x-padded grid
// [nf3][nf2][2*(nf1/2+1)]
extern "C" void ref_pz_lda(int nf1, int nf2, int nf3, double* density, double* result, double box, double* exc,
                           double* muxc) {
  set_cell(box);
  readonly_cp.cpopts.cp_lyp = 0;
  CPXCFNCTS::CP_exc_calc(nf1 * nf2 * nf3, nf1, nf2, nf3, density, result, exc, muxc, 1);
}

// CPLOCAL::CP_hart_eext_calc (cp_hart_ext.C:56-431) on a list of density
// g-points (kx, ky, kz) with rho(g) given per point; returns vks(g) per point.
extern "C" void ref_hart_eext(int npts, const int* kx, const int* ky, const int* kz, const double* rho, double* vks,
                              int natm, const double* pos, const int* atm_type /* 0-based */, const double* q,
                              int ntype, int nspl, double gmin, double dg, const double* spl /* [ntype][nspl][4] */,
                              const double* gzvps, double alp_ewd, double ecut_ry, double box, double* ehart,
                              double* eext, double* ewd, double* fatm /* [natm][3] */) {
  set_cell(box);
  CP* cp = &readonly_cp;
  CPPSEUDO* ps = &cp->cppseudo;
  MDATOMS* md = &readonly_mdatoms;
  md->mdclatoms_info.natm_tot = natm;
  md->mdatom_maps.natm_typ = ntype;
  std::vector<int> ityp(natm + 1);
  for (int a = 0; a < natm; ++a) ityp[a + 1] = atm_type[a] + 1;
  md->mdatom_maps.iatm_atm_typ = ityp.data();
  ps->nsplin_g = nspl;
  ps->n_rad_max = 1;
  ps->n_ang_max = 0;
  ps->dg_spl = dg;
  ps->gmin_spl = gmin;
  std::vector<double> v0(ntype * nspl + 1), v1(ntype * nspl + 1), v2(ntype * nspl + 1), v3(ntype * nspl + 1);
  for (int t = 0; t < ntype; ++t)
    for (int i = 0; i < nspl; ++i) {
      const double* c = spl + ((size_t)t * nspl + i) * 4;
      const int idx = t * nspl + i + 1;
      v0[idx] = c[0]; v1[idx] = c[1]; v2[idx] = c[2]; v3[idx] = c[3];
    }
  ps->vps0 = v0.data(); ps->vps1 = v1.data(); ps->vps2 = v2.data(); ps->vps3 = v3.data();
  std::vector<double> gz(ntype + 1);
  std::vector<int> lopt(ntype + 1, 0);
  for (int t = 0; t < ntype; ++t) gz[t + 1] = gzvps[t];
  ps->gzvps = gz.data();
  ps->loc_opt = lopt.data();
  cp->cpcoeffs_info.ecut = 0.5 * ecut_ry;
  readonly_general_data.genewald.alp_ewd = alp_ewd;
  std::vector<double> x(natm), y(natm), z(natm), qq(natm), fx(natm, 0.0), fy(natm, 0.0), fz(natm, 0.0);
  for (int a = 0; a < natm; ++a) { x[a] = pos[3 * a]; y[a] = pos[3 * a + 1]; z[a] = pos[3 * a + 2]; qq[a] = q[a]; }
  FastAtoms fa;
  fa.natm = natm; fa.x = x.data(); fa.y = y.data(); fa.z = z.data(); fa.q = qq.data();
  fa.fx = fx.data(); fa.fy = fy.data(); fa.fz = fz.data();
  std::vector<int> index_atm(ntype + 1);
  std::vector<double> vtemp(natm + 1);
  std::vector<complex> ei(natm + 1), ti(natm + 1);
  PSSCRATCH scr;
  scr.index_atm = index_atm.data();
  scr.vtemp = vtemp.data();
  scr.ei_inc = ei.data();
  scr.ti_inc = ti.data();
  std::vector<gridPoint> pts(npts);
  for (int i = 0; i < npts; ++i) { pts[i].d3 = kx[i]; pts[i].d2 = ky[i]; pts[i].d1 = kz[i]; pts[i].offset = i; }
  for (int i = 0; i < 2 * npts; ++i) vks[i] = 0.0;
  CPLOCAL::CP_hart_eext_calc(npts, pts, (complex*)const_cast<double*>(rho), natm, 3, &fa, (complex*)vks, ehart, eext,
                             ewd, 0, &scr, 1);
  if (fatm)
    for (int a = 0; a < natm; ++a) { fatm[3 * a] = fx[a]; fatm[3 * a + 1] = fy[a]; fatm[3 * a + 2] = fz[a]; }
  scr.index_atm = nullptr; scr.vtemp = nullptr; scr.ei_inc = nullptr; scr.ti_inc = nullptr;
}

// CPORTHOG::get_iter_Tmat (cp_lowdin.C:180-265): Schulz iteration, <= 10 iterations
extern "C" void ref_iter_tmat(const double* S, double* T, int n) {
  CPORTHOG::get_iter_Tmat(S, T, n);
}
