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
#include "../class_defs/typedefs_par.h"
#include "../class_defs/CP_OPERATIONS/class_cpnonlocal.h"
#include "../class_defs/CP_OPERATIONS/class_cpxcfnctls.h"
#include "../class_defs/CP_OPERATIONS/class_cplocal.h"
#include "../class_defs/CP_OPERATIONS/class_cporthog.h"
#include "../class_defs/CP_OPERATIONS/class_cpintegrate.h"
#include "../class_defs/CP_OPERATIONS/class_cprspaceion.h"
#include <vector>
#include <cstring>

// y = alpha op(A) x + beta y, A column-major m x n (lda), op = 'T'/'t' or
// 'N'/'n': the BLAS DGEMV / ZGEMV semantics the PINY nonlocal routines call
// (src_mathlib/mathlib.h), written here from the BLAS definition.
extern "C" void dgemv_(char* trans, int* m, int* n, double* alpha, double* A, int* lda, double* x, int* incx,
                       double* beta, double* y, int* incy) {
  const bool t = (*trans == 'T' || *trans == 't');
  const int ny = t ? *n : *m, nx = t ? *m : *n;
  for (int i = 0; i < ny; ++i) {
    double s = 0.0;
    for (int j = 0; j < nx; ++j) {
      const double a = t ? A[j + (size_t)i * *lda] : A[i + (size_t)j * *lda];
      s += a * x[(size_t)j * *incx];
    }
    double& yy = y[(size_t)i * *incy];
    yy = *alpha * s + (*beta == 0.0 ? 0.0 : *beta * yy);
  }
}
extern "C" void zgemv_(char* trans, int* m, int* n, complex* alpha, complex* A, int* lda, complex* x, int* incx,
                       complex* beta, complex* y, int* incy) {
  const bool t = (*trans == 'T' || *trans == 't');
  const int ny = t ? *n : *m, nx = t ? *m : *n;
  for (int i = 0; i < ny; ++i) {
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < nx; ++j) {
      const complex a = t ? A[j + (size_t)i * *lda] : A[i + (size_t)j * *lda];
      const complex b = x[(size_t)j * *incx];
      sr += a.re * b.re - a.im * b.im;
      si += a.re * b.im + a.im * b.re;
    }
    complex& yy = y[(size_t)i * *incy];
    const double yr = yy.re, yi = yy.im;
    const double br = beta->re, bi = beta->im;
    yy.re = alpha->re * sr - alpha->im * si + ((br == 0.0 && bi == 0.0) ? 0.0 : br * yr - bi * yi);
    yy.im = alpha->re * si + alpha->im * sr + ((br == 0.0 && bi == 0.0) ? 0.0 : br * yi + bi * yr);
  }
}

// PINY allocators (friend_lib) as plain malloc/free
void* cmalloc(size_t n, const char*) { return std::malloc(n ? n : 1); }
void cfree(void* p, const char*) { std::free(p); }

// Symbols the compiled files reference on paths the oracle never takes:
// timers, the EISPACK eigen-solver of get_diag_Tmat, the cell determinant
// of the Ewald set-up routines (set_cp_ewald.C is linked for
// get_bspline_wght1d only), and the wave generator's class.
void cputime(double* t) { *t = 0.0; }
extern "C" void rs_(int*, int*, double*, double*, int*, double*, double*, double*, int*) {
  std::fprintf(stderr, "oracle/_ref: rs_ (EISPACK) is not provided\n");
  std::abort();
}
// the input-parsing and Gauss-Hermite routines of control_vps_params.C's
// other functions (make_vps_splin of a LOC / KB type reaches none of them)
#define OA_SHIM_ABSENT(sig)                                                   \
  sig {                                                                       \
    std::fprintf(stderr, "oracle/_ref: %s is not provided\n", #sig);         \
    std::abort();                                                             \
  }
OA_SHIM_ABSENT(void keyarg_barf(DICT_WORD*, char*, char*, int))
OA_SHIM_ABSENT(int** cmall_int_mat(long, long, long, long, const char*))
OA_SHIM_ABSENT(void search_base_vps(char*, CVPS*, DICT_WORD*, int, DICT_WORD**, DICT_WORD*, int, int*))
OA_SHIM_ABSENT(void set_grimme_dict(DICT_WORD**, int*, int))
OA_SHIM_ABSENT(void set_potfun_dict(DICT_WORD**, int*, int))
OA_SHIM_ABSENT(void set_potvps_dict(DICT_WORD**, int*, int))
OA_SHIM_ABSENT(void search_base_grimme(char*, CVPS*, DICT_WORD*, int, DICT_WORD**, DICT_WORD*, int, int*))
OA_SHIM_ABSENT(void limit_gauss_hermite(int*, double*, double*))
OA_SHIM_ABSENT(void weight_node_gauss_hermite(int, double*, double*))
OA_SHIM_ABSENT(double** cmall_mat(long, long, long, long, const char*))
double getdeth(double*) {
  std::fprintf(stderr, "oracle/_ref: getdeth is not provided\n");
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
// [nf3][nf2][2*(nf1/2+1)]; lyp = 1 drops the PZ correlation (LYP on)
extern "C" void ref_pz_lda(int nf1, int nf2, int nf3, double* density, double* result, double box, double* exc,
                           double* muxc, int lyp) {
  set_cell(box);
  readonly_cp.cpopts.cp_lyp = lyp;
  CPXCFNCTS::CP_exc_calc(nf1 * nf2 * nf3, nf1, nf2, nf3, density, result, exc, muxc, 1);
  readonly_cp.cpopts.cp_lyp = 0;
}

// CPXCFNCTS::CP_getGGAFunctional (cp_grad_rho_ctrl.C:32-190) with Becke
// exchange and LYP correlation (cp_becke.C) on x-padded grids
// [nf3][nf2][2*(nf1/2+1)]: vks += df/drho, grad rho (gx, gy, gz) replaced by
// df/d|grad rho| grad rho / |grad rho|, EGGA returned.  The routine keeps
// its healing length in a function-level static, so one process pins one
// gga_cut.
extern "C" double ref_gga(int nf1, int nf2, int nf3, double* density, double* gx, double* gy, double* gz,
                          double* vks, double box, double gga_cut, int becke, int lyp) {
  set_cell(box);
  readonly_cp.cpopts.cp_becke = becke;
  readonly_cp.cpopts.cp_lyp = lyp;
  readonly_cp.cppseudo.gga_cut = gga_cut;
  double e = 0.0;
  CPXCFNCTS::CP_getGGAFunctional(nf1 * nf2 * nf3, nf1, nf2, nf3, density, gx, gy, gz, vks, 0, &e, 1);
  readonly_cp.cpopts.cp_becke = 0;
  readonly_cp.cpopts.cp_lyp = 0;
  return e;
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

// The structure-factor (N^2) nonlocal path for one l = 0 KB channel, all
// states (doublePack, one atom group):
//   CPNONLOCAL::CP_calc_Struct_Fact (cp_struct_fact.C:37-255),
//   CPNONLOCAL::CP_enl_matrix_calc (cp_nlmat.C:24-100, the DGEMV branch),
//   CPNONLOCAL::CP_enl_atm_forc_calc (cp_nl_energy_forc.C:178-235),
//   CPNONLOCAL::CP_enl_force_calc (cp_nl_energy_forc.C:29-110, the DGEMV branch).
// nl_atm: 0-based indices of the nonlocal atoms, grouped by type in type
// order; spl: [ntype][nspl][4] projector spline per type (l = 0);
// vnorm_typ / gz0_typ per type.  Outputs: sf [natm_nl][ng] complex,
// fnl [nstate][ng] complex (starts at zero), zmat [nstate][natm_nl] (the
// scaled Z of CP_enl_atm_forc_calc), enl [nstate], fatm [natm][3].
extern "C" void ref_nl_sf(int ng, const int* kx, const int* ky, const int* kz, int nstate, const double* psi,
                          const double* occ, int natm, const double* pos, const int* atm_type, int ntype,
                          int natm_nl, const int* nl_atm, int nspl, double gmin, double dg, const double* spl,
                          const double* vnorm_typ, const double* gz0_typ, double ecut_ry, double box, double* sf,
                          double* fnl, double* zmat, double* enl, double* fatm) {
  set_cell(box);
  CP* cp = &readonly_cp;
  CPPSEUDO* ps = &cp->cppseudo;
  PSNONLOCAL* nl = &ps->nonlocal;
  cp->cpcoeffs_info.ecut = 0.5 * ecut_ry;
  cp->cpcoeffs_info.ecut_psi = ecut_ry;
  std::vector<double> occ_up(nstate + 1);
  for (int s = 0; s < nstate; ++s) occ_up[s + 1] = occ[s];
  cp->cpcoeffs_info.occ_up = occ_up.data();
  // projector spline, n_ang_max = 0: index (ityp-1) nsplin_g + iii
  ps->nsplin_g = nspl;
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
  std::vector<double> gz0(ntype + 1);
  for (int t = 0; t < ntype; ++t) gz0[t + 1] = gz0_typ[t];
  ps->gzvps0 = gz0.data();
  // nonlocal atom bookkeeping (PSNONLOCAL): one l = 0 channel; the atom types
  // with a projector, in type order, and where their atoms start in the list
  std::vector<int> map_nl(natm_nl + 1), natm_lang(ntype + 1, 0), iatm_str_lang(ntype + 1, 0);
  std::vector<double> vnorm(natm_nl + 1);
  std::vector<int> typ_list;
  for (int i = 0; i < natm_nl; ++i) {
    const int a = nl_atm[i], t = atm_type[a] + 1;
    map_nl[i + 1] = a + 1;
    vnorm[i + 1] = vnorm_typ[t - 1];
    if (natm_lang[t] == 0) { iatm_str_lang[t] = i + 1; typ_list.push_back(t); }
    natm_lang[t]++;
  }
  std::vector<int> natm_typ_lang(2, 0);
  natm_typ_lang[1] = (int)typ_list.size();
  std::vector<std::vector<int>> typ_rows(typ_list.size() + 1, std::vector<int>(2, 0));
  std::vector<int*> iatm_typ_lang(typ_list.size() + 1);
  for (size_t k = 0; k < typ_list.size(); ++k) typ_rows[k + 1][1] = typ_list[k];
  for (size_t k = 0; k <= typ_list.size(); ++k) iatm_typ_lang[k] = typ_rows[k].data();
  nl->natm = natm_nl;
  nl->natm_typ = (int)typ_list.size();
  nl->map_nl = map_nl.data();
  nl->natm_lang = natm_lang.data();
  nl->iatm_str_lang = iatm_str_lang.data();
  nl->natm_typ_lang = natm_typ_lang.data();
  nl->iatm_typ_lang = iatm_typ_lang.data();
  nl->vnorm_0 = vnorm.data();
  // atoms and scratch
  std::vector<double> x(natm), y(natm), z(natm), fx(natm, 0.0), fy(natm, 0.0), fz(natm, 0.0);
  for (int a = 0; a < natm; ++a) { x[a] = pos[3 * a]; y[a] = pos[3 * a + 1]; z[a] = pos[3 * a + 2]; }
  FastAtoms fa;
  fa.natm = natm; fa.x = x.data(); fa.y = y.data(); fa.z = z.data();
  fa.fx = fx.data(); fa.fy = fy.data(); fa.fz = fz.data();
  std::vector<double> sx(natm_nl + 1), sy(natm_nl + 1), sz(natm_nl + 1);
  std::vector<complex> ei(natm_nl + 1), ti(natm_nl + 1);
  PSSCRATCH scr;
  scr.x = sx.data(); scr.y = sy.data(); scr.z = sz.data();
  scr.ei_inc = ei.data(); scr.ti_inc = ti.data();
  std::vector<complex> SFx((size_t)natm_nl * ng), SFy((size_t)natm_nl * ng), SFz((size_t)natm_nl * ng);
  complex* SF = (complex*)sf;
  CPNONLOCAL::CP_calc_Struct_Fact(ng, const_cast<int*>(kx), const_cast<int*>(ky), const_cast<int*>(kz), SF,
                                  SFx.data(), SFy.data(), SFz.data(), &fa, 1, 1, 0, &scr);
  std::vector<complex> zm(natm_nl), zx(natm_nl), zy(natm_nl), zz(natm_nl);
  for (int s = 0; s < nstate; ++s) {
    complex* cs = (complex*)const_cast<double*>(psi) + (size_t)s * ng;
    CPNONLOCAL::CP_enl_matrix_calc(ng, cs, const_cast<int*>(kx), const_cast<int*>(ky), const_cast<int*>(kz), SF,
                                   SFx.data(), SFy.data(), SFz.data(), zm.data(), zx.data(), zy.data(), zz.data(), s,
                                   1, 1, 0);
    double e = 0.0;
    CPNONLOCAL::CP_enl_atm_forc_calc(1, 0, &fa, zm.data(), zx.data(), zy.data(), zz.data(), &e, 1, s);
    enl[s] = e;
    for (int a = 0; a < natm_nl; ++a) zmat[(size_t)s * natm_nl + a] = zm[a].re;
    complex* fs = (complex*)fnl + (size_t)s * ng;
    for (int i = 0; i < ng; ++i) fs[i] = complex(0.0, 0.0);
    CPNONLOCAL::CP_enl_force_calc(zm.data(), ng, const_cast<int*>(kx), const_cast<int*>(ky), const_cast<int*>(kz), SF,
                                  fs, s, 1, 1, 0);
  }
  for (int a = 0; a < natm; ++a) { fatm[3 * a] = fx[a]; fatm[3 * a + 1] = fy[a]; fatm[3 * a + 2] = fz[a]; }
  scr.x = scr.y = scr.z = nullptr;
  scr.ei_inc = scr.ti_inc = nullptr;
  nl->map_nl = nl->natm_lang = nl->iatm_str_lang = nl->natm_typ_lang = nullptr;
  nl->iatm_typ_lang = nullptr;
  nl->vnorm_0 = nullptr;
}

// CPINTEGRATE::CP_integrate_dyn (cp_dynamics.C:29-88) for one state, with
// the coefficient thermostat off (no NHC chunks: cp_isoNHC_update of
// cp_isokin.C loops over zero chunks).  forces, vpsi, psi: ncoef complex;
// cmass: ncoef.  Returns the fictitious KE of get_fictKE.
extern "C" void ref_integrate_dyn(int ncoef, int iteration, double dt, double* forces, double* vpsi, double* psi,
                                  double* cmass, int nkx0_red, int nkx0_uni, int nkx0_zero, double* fict_ke) {
  readonly_general_data.gentimeinfo.dt = dt;
  readonly_general_data.gentimeinfo.bomd_scale = 1.0;
  readonly_cp.cptherm_info.nres_c_nhc = 1;
  readonly_cp.cptherm_info.nyosh_c_nhc = 1;
  double ekeNhc = 0.0, potNHC = 0.0, degfs = 0.0;
  int istr = 0, iend = 0;
  CPINTEGRATE::CP_integrate_dyn(ncoef, 0, iteration, (complex*)forces, (complex*)vpsi, (complex*)psi, cmass, nullptr,
                                nullptr, nullptr, 0, 0, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                nullptr, nullptr, 1.0, fict_ke, nkx0_red, nkx0_uni, nkx0_zero, &ekeNhc, &potNHC,
                                1.0, 1.0, &degfs, &istr, &iend, 1, false, 1.0, 1.0);
}

// CPINTEGRATE::CP_integrate_min_STD (cp_min_std.C:17-60) and
// CP_integrate_min_CG (cp_min_CG.C:29-120) for one state, and
// CP_fovlap_calc (cp_min_CG.C:128-140).
extern "C" void ref_min_step(int ncoef, double* forces, double* conj, double* psi, const int* kx, const int* ky,
                             const int* kz, double* cmass, double dt, double gamma, double box, double ecut_ry) {
  set_cell(box);
  readonly_general_data.gentimeinfo.dt = dt;
  readonly_cp.cpcoeffs_info.ecut_psi = ecut_ry;
  if (conj)
    CPINTEGRATE::CP_integrate_min_CG(ncoef, 0, (complex*)forces, (complex*)conj, (complex*)psi,
                                     const_cast<int*>(kx), const_cast<int*>(ky), const_cast<int*>(kz), cmass, gamma,
                                     0);
  else
    CPINTEGRATE::CP_integrate_min_STD(ncoef, 0, (complex*)forces, (complex*)psi, const_cast<int*>(kx),
                                      const_cast<int*>(ky), const_cast<int*>(kz), cmass, 0);
}
extern "C" double ref_fovlap(int ncoef, double* forces) {
  double f = 0.0;
  CPINTEGRATE::CP_fovlap_calc(ncoef, 0, (complex*)forces, &f);
  return f;
}

// ---------------------------------------------------------------------------
// EES nonlocal, l = 0 KB channel (cp_ees_nonlocal.C), doublePack, Gamma.
// The test runs the routines in three phases with the oracle's nonlocal-grid
// transforms in between (the FFT boundary has no reference implementation
// here):
//   ref_ees_config   the PINY nonlocal setup the routines read (kept here)
//   ref_ees_gproj    eesSetEesWghtGgrp (60-160), eesSplProjectorGgrp
//                    (182-250), eesProjGchare + eesYlmOnD (594-735): d(g),
//                    dyp(g) and projPsiG = conj(dyp psi) of every state
//   ref_ees_rspace   eesAtmBsplineRgrp (256-593), eesZmatRchare (1238-1352)
//                    summed over the planes, eesEnergyAtmForcRchare
//                    (1480-1720) on every plane with its own copy of the
//                    summed zmat: ENL, the scaled zmat, the scattered grid
//                    projPsiRScr and the atom forces
//   ref_ees_psi_forc eesPsiForcGspace (2000-2079)
// Grids are real [nc][nb][na + 2] (the x-padded doublePack plane layout
// the routines index, igrid_b = (ib - 1)(na + 2)).
namespace {
struct EesCfg {
  int ng = 0, na = 0, nb = 0, nc = 0, order = 0, natm = 0, natm_nl = 0, ntyp_nl = 0, ind_g0 = -1, nkx0 = 0;
  double box = 0.0;
  std::vector<int> kx, ky, kz, map_nl, natm_lang, iatm_str_lang, natm_typ_lang, lang_v, mang_v, ityp_v;
  std::vector<std::vector<int>> typ_rows;
  std::vector<int*> iatm_typ_lang;
  std::vector<double> v0, v1, v2, v3, gz0, vpsnorm, occ_up, wkpt, kpt0, pos;
  std::vector<double> d_re, d_im;                  // eesSetEesWghtGgrp
  std::vector<double> h_spl;                       // eesSplProjectorGgrp
  std::vector<int> ind_spl;
  std::vector<double> dyp_re, dyp_im;              // [ntyp_nl][ng]
} g_ees;

void ees_apply() {
  EesCfg& e = g_ees;
  set_cell(e.box);
  CP* cp = &readonly_cp;
  CPPSEUDO* ps = &cp->cppseudo;
  PSNONLOCAL* nl = &ps->nonlocal;
  ps->nsplin_g = (int)(e.v0.size() - 1) / std::max(1, (int)e.gz0.size() - 1);
  ps->n_ang_max = 0;
  ps->n_interp_ps = e.order;
  ps->vps0 = e.v0.data(); ps->vps1 = e.v1.data(); ps->vps2 = e.v2.data(); ps->vps3 = e.v3.data();
  ps->gzvps0 = e.gz0.data();
  ps->vpsnorm = e.vpsnorm.data();
  nl->natm = e.natm_nl;
  nl->n_interp = e.order;
  nl->n_interp2 = e.order * e.order;
  nl->ngrid_a = e.na; nl->ngrid_b = e.nb; nl->ngrid_c = e.nc;
  nl->nfft = e.na * e.nb * e.nc;
  nl->map_nl = e.map_nl.data();
  nl->natm_lang = e.natm_lang.data();
  nl->iatm_str_lang = e.iatm_str_lang.data();
  nl->natm_typ_lang = e.natm_typ_lang.data();
  nl->iatm_typ_lang = e.iatm_typ_lang.data();
  nl->lang_v = e.lang_v.data(); nl->mang_v = e.mang_v.data(); nl->ityp_v = e.ityp_v.data();
  cp->cpewald.doublepack = 1;
  cp->cpewald.akpoint = cp->cpewald.bkpoint = cp->cpewald.ckpoint = e.kpt0.data();
  cp->cpcoeffs_info.nkpoint = 1;
  cp->cpcoeffs_info.igamma_kpt_ind = 1;
  cp->cpcoeffs_info.occ_up = e.occ_up.data();
  cp->cpcoeffs_info.wght_kpt = e.wkpt.data();
  cp->cpylm_cons.rt_fpi = 1.0 / std::sqrt(4.0 * M_PI);
}
}  // namespace

// Set up: g-points (the system's doublePack order, kx = 0 first), states'
// occupations, atoms (nl_atm grouped by type in type order), the l = 0
// projector spline per type [ntype][nspl][4], vnorm and g = 0 value per
// type, the box, the EES grid and the interpolation order.
extern "C" void ref_ees_config(int ng, const int* kx, const int* ky, const int* kz, int nstate, const double* occ,
                               int natm, const double* pos, const int* atm_type, int ntype, int natm_nl,
                               const int* nl_atm, int nspl, double gmin, double dg, const double* spl,
                               const double* vnorm_typ, const double* gz0_typ, double box, int na, int nb, int nc,
                               int order) {
  EesCfg& e = g_ees;
  e = EesCfg();
  e.ng = ng; e.na = na; e.nb = nb; e.nc = nc; e.order = order; e.natm = natm; e.natm_nl = natm_nl; e.box = box;
  e.kx.assign(kx, kx + ng); e.ky.assign(ky, ky + ng); e.kz.assign(kz, kz + ng);
  for (int i = 0; i < ng; ++i) {
    if (kx[i] == 0 && ky[i] == 0 && kz[i] == 0) e.ind_g0 = i;
    if (kx[i] == 0) e.nkx0++;
  }
  e.pos.assign(pos, pos + 3 * natm);
  e.occ_up.assign(nstate + 1, 0.0);
  for (int s = 0; s < nstate; ++s) e.occ_up[s + 1] = occ[s];
  e.wkpt.assign(2, 1.0);
  e.kpt0.assign(2, 0.0);
  e.v0.assign(ntype * nspl + 1, 0.0); e.v1 = e.v0; e.v2 = e.v0; e.v3 = e.v0;
  for (int t = 0; t < ntype; ++t)
    for (int i = 0; i < nspl; ++i) {
      const double* c = spl + ((size_t)t * nspl + i) * 4;
      const int idx = t * nspl + i + 1;
      e.v0[idx] = c[0]; e.v1[idx] = c[1]; e.v2[idx] = c[2]; e.v3[idx] = c[3];
    }
  e.gz0.assign(ntype + 1, 0.0);
  e.vpsnorm.assign(ntype + 1, 0.0);
  for (int t = 0; t < ntype; ++t) { e.gz0[t + 1] = gz0_typ[t]; e.vpsnorm[t + 1] = vnorm_typ[t]; }
  // one l = 0 iteration per atom type with a projector (iter_nl = 1, 2, ...)
  e.map_nl.assign(natm_nl + 1, 0);
  e.natm_lang.assign(ntype + 1, 0);
  e.iatm_str_lang.assign(ntype + 1, 0);
  std::vector<int> typ_list;
  for (int i = 0; i < natm_nl; ++i) {
    const int a = nl_atm[i], t = atm_type[a] + 1;
    e.map_nl[i + 1] = a + 1;
    if (e.natm_lang[t] == 0) { e.iatm_str_lang[t] = i + 1; typ_list.push_back(t); }
    e.natm_lang[t]++;
  }
  e.ntyp_nl = (int)typ_list.size();
  e.natm_typ_lang.assign(2, 0);
  e.natm_typ_lang[1] = e.ntyp_nl;
  e.typ_rows.assign(e.ntyp_nl + 1, std::vector<int>(2, 0));
  for (int k = 0; k < e.ntyp_nl; ++k) e.typ_rows[k + 1][1] = typ_list[k];
  e.iatm_typ_lang.resize(e.ntyp_nl + 1);
  for (int k = 0; k <= e.ntyp_nl; ++k) e.iatm_typ_lang[k] = e.typ_rows[k].data();
  e.lang_v.assign(e.ntyp_nl + 1, 0);
  e.mang_v.assign(e.ntyp_nl + 1, 0);
  e.ityp_v.assign(e.ntyp_nl + 1, 0);
  for (int k = 1; k <= e.ntyp_nl; ++k) e.ityp_v[k] = k;
  readonly_cp.cppseudo.nsplin_g = nspl;
  readonly_cp.cppseudo.dg_spl = dg;
  readonly_cp.cppseudo.gmin_spl = gmin;
}

// d(g) [ng] complex, dyp(g) [ntyp_nl][ng] complex and projPsiG
// [ntyp_nl][nstate][ng] complex for the states psi [nstate][ng].
extern "C" int ref_ees_gproj(int nstate, const double* psi, double* d, double* dyp, double* proj) {
  EesCfg& e = g_ees;
  ees_apply();
  const int ng = e.ng;
  e.d_re.assign(ng, 0.0); e.d_im.assign(ng, 0.0);
  CPNONLOCAL::eesSetEesWghtGgrp(ng, e.kx.data(), e.ky.data(), e.kz.data(), e.d_re.data(), e.d_im.data(), e.na, e.nb,
                                e.nc, e.order);
  e.h_spl.assign(ng, 0.0); e.ind_spl.assign(ng, 0);
  double* hs[1] = {e.h_spl.data()};
  int* is[1] = {e.ind_spl.data()};
  CPNONLOCAL::eesSplProjectorGgrp(ng, e.kx.data(), e.ky.data(), e.kz.data(), hs, is);
  for (int i = 0; i < ng; ++i) { d[2 * i] = e.d_re[i]; d[2 * i + 1] = e.d_im[i]; }
  e.dyp_re.assign((size_t)e.ntyp_nl * ng, 0.0); e.dyp_im = e.dyp_re;
  const int ihave_g0 = e.ind_g0 >= 0 ? 1 : 0;
  for (int it = 1; it <= e.ntyp_nl; ++it) {
    double* yr = e.dyp_re.data() + (size_t)(it - 1) * ng;
    double* yi = e.dyp_im.data() + (size_t)(it - 1) * ng;
    for (int s = 0; s < nstate; ++s) {
      complex* pg = (complex*)proj + ((size_t)(it - 1) * nstate + s) * ng;
      CPNONLOCAL::eesProjGchare(ng, (complex*)const_cast<double*>(psi) + (size_t)s * ng, e.kx.data(), e.ky.data(),
                                e.kz.data(), ihave_g0, e.ind_g0, it, e.d_re.data(), e.d_im.data(), yr, yi, pg, is, hs,
                                s, 0, 0, 1, 0);
    }
    for (int i = 0; i < ng; ++i) {
      dyp[2 * ((size_t)(it - 1) * ng + i)] = yr[i];
      dyp[2 * ((size_t)(it - 1) * ng + i) + 1] = yi[i];
    }
  }
  return e.ntyp_nl;
}

// projPsiR [ntyp_nl][nstate][nc][nb][na + 2] -> zmat (summed over planes,
// unscaled) [ntyp_nl][nstate][natm of the type] laid out per nonlocal atom
// [nstate][natm_nl], enl [nstate], the scattered grid projPsiRScr (same
// shape as projPsiR) and the atom forces fatm [natm][3] (accumulated).
extern "C" void ref_ees_rspace(int nstate, const double* prr, double* zmat, double* enl, double* scr, double* fatm) {
  EesCfg& e = g_ees;
  ees_apply();
  const int n = e.order, n2 = n * n, natm = e.natm, nnl = e.natm_nl;
  const int lda = e.na + 2;
  const size_t plane = (size_t)lda * e.nb, grid = plane * e.nc;
  // PSSCRATCH for the B-spline routine ([j][i] with j = 1..n)
  std::vector<double> aj(n + 1), rn(n + 1), rn1(n + 1), fa(nnl), fb(nnl), fc(nnl);
  std::vector<int> ixa(n + 1), ixb(n + 1), iga(n + 1), igb(n + 1), iat(nnl), ibt(nnl), ict(nnl);
  std::vector<std::vector<int>> gi_a(n + 1, std::vector<int>(nnl)), gi_b = gi_a, gi_c = gi_a;
  std::vector<std::vector<double>> m_a(n + 1, std::vector<double>(nnl)), m_b = m_a, m_c = m_a, u_a = m_a, u_b = m_a,
                                   u_c = m_a, dm_a = m_a, dm_b = m_a, dm_c = m_a;
  auto rows_i = [](std::vector<std::vector<int>>& v) {
    std::vector<int*> p(v.size());
    for (size_t i = 0; i < v.size(); ++i) p[i] = v[i].data();
    return p;
  };
  auto rows_d = [](std::vector<std::vector<double>>& v) {
    std::vector<double*> p(v.size());
    for (size_t i = 0; i < v.size(); ++i) p[i] = v[i].data();
    return p;
  };
  auto pga = rows_i(gi_a), pgb = rows_i(gi_b), pgc = rows_i(gi_c);
  auto pma = rows_d(m_a), pmb = rows_d(m_b), pmc = rows_d(m_c), pua = rows_d(u_a), pub = rows_d(u_b),
       puc = rows_d(u_c), pda = rows_d(dm_a), pdb = rows_d(dm_b), pdc = rows_d(dm_c);
  PSSCRATCH ps;
  ps.aj = aj.data(); ps.rn = rn.data(); ps.rn1 = rn1.data();
  ps.index_a = ixa.data(); ps.index_b = ixb.data(); ps.igrid_at = iga.data(); ps.igrid_bt = igb.data();
  ps.iatemp = iat.data(); ps.ibtemp = ibt.data(); ps.ictemp = ict.data();
  ps.frac_a = fa.data(); ps.frac_b = fb.data(); ps.frac_c = fc.data();
  ps.igrid_a = pga.data(); ps.igrid_b = pgb.data(); ps.igrid_c = pgc.data();
  ps.mn_a = pma.data(); ps.mn_b = pmb.data(); ps.mn_c = pmc.data();
  ps.ua = pua.data(); ps.ub = pub.data(); ps.uc = puc.data();
  ps.dmn_a = pda.data(); ps.dmn_b = pdb.data(); ps.dmn_c = pdc.data();
  // per-plane B-spline data (RPPDATA, [natm_nl][n^2 + 1])
  std::vector<RPPDATA> rpp(e.nc);
  std::vector<RPPDATA*> prpp(e.nc);
  std::vector<std::vector<int>> pidx(e.nc, std::vector<int>(nnl));
  std::vector<std::vector<std::vector<int>>> ig(e.nc, std::vector<std::vector<int>>(nnl, std::vector<int>(n2 + 1)));
  std::vector<std::vector<std::vector<double>>> mn(e.nc, std::vector<std::vector<double>>(nnl, std::vector<double>(n2 + 1)));
  auto dx = mn, dy = mn, dz = mn;
  std::vector<std::vector<int*>> pig(e.nc);
  std::vector<std::vector<double*>> pmn(e.nc), pdx(e.nc), pdy(e.nc), pdz(e.nc);
  for (int p = 0; p < e.nc; ++p) {
    pig[p] = rows_i(ig[p]);
    pmn[p] = rows_d(mn[p]); pdx[p] = rows_d(dx[p]); pdy[p] = rows_d(dy[p]); pdz[p] = rows_d(dz[p]);
    RPPDATA& r = rpp[p];
    r.index = p; r.ngrid_a = e.na; r.ngrid_b = e.nb; r.ngrid_c = e.nc; r.n_interp = n; r.natm = nnl;
    r.plane_index = pidx[p].data();
    r.igrid = pig[p].data();
    r.mn = pmn[p].data(); r.dmn_x = pdx[p].data(); r.dmn_y = pdy[p].data(); r.dmn_z = pdz[p].data();
    r.nBreakJ = nullptr; r.sBreakJ = nullptr;
    prpp[p] = &r;
  }
  std::vector<double> x(natm), y(natm), z(natm), fx(natm, 0.0), fy(natm, 0.0), fz(natm, 0.0);
  for (int a = 0; a < natm; ++a) { x[a] = e.pos[3 * a]; y[a] = e.pos[3 * a + 1]; z[a] = e.pos[3 * a + 2]; }
  FastAtoms at;
  at.natm = natm; at.x = x.data(); at.y = y.data(); at.z = z.data();
  at.fx = fx.data(); at.fy = fy.data(); at.fz = fz.data();
  std::vector<int> allowed(e.nc, 1);
  CPNONLOCAL::eesAtmBsplineRgrp(&at, allowed.data(), prpp.data(), &ps);
  std::vector<double> zp(nnl), zsum(nnl), zcopy(nnl);
  for (int s = 0; s < nstate; ++s) {
    enl[s] = 0.0;
    for (int it = 1; it <= e.ntyp_nl; ++it) {
      const int t = e.iatm_typ_lang[it][1];
      const int na_t = e.natm_lang[t], a0 = e.iatm_str_lang[t] - 1;
      const double* pr = prr + ((size_t)(it - 1) * nstate + s) * grid;
      double* sc = scr + ((size_t)(it - 1) * nstate + s) * grid;
      std::fill(zsum.begin(), zsum.end(), 0.0);
      for (int p = 0; p < e.nc; ++p) {
        CPNONLOCAL::eesZmatRchare(const_cast<double*>(pr) + p * plane, it, zp.data(), rpp[p].igrid, rpp[p].mn,
                                  rpp[p].plane_index, s, p);
        for (int j = 0; j < na_t; ++j) zsum[j] += zp[j];
      }
      for (int j = 0; j < na_t; ++j) zmat[(size_t)s * nnl + a0 + j] = zsum[j];
      for (int p = 0; p < e.nc; ++p) {
        for (int j = 0; j < na_t; ++j) zcopy[j] = zsum[j];
        double ep = 0.0;
        CPNONLOCAL::eesEnergyAtmForcRchare(it, &ep, zcopy.data(), rpp[p].igrid, rpp[p].mn, rpp[p].dmn_x,
                                           rpp[p].dmn_y, rpp[p].dmn_z, const_cast<double*>(pr) + p * plane,
                                           sc + p * plane, rpp[p].plane_index, nullptr, nullptr, p, s, 0, &at);
        if (p == 0) enl[s] += ep;  // every plane computes it; one (the reduction plane) reports it
      }
    }
  }
  for (int a = 0; a < natm; ++a) { fatm[3 * a] += fx[a]; fatm[3 * a + 1] += fy[a]; fatm[3 * a + 2] += fz[a]; }
}

// fPsiG [nstate][ng] complex (accumulated) from projPsiG [ntyp_nl][nstate][ng]
// (the inverse nonlocal-grid transform of projPsiRScr, at the g-points) and
// the dyp of ref_ees_gproj.
extern "C" void ref_ees_psi_forc(int nstate, const double* projg, double* fpsi) {
  EesCfg& e = g_ees;
  ees_apply();
  const int ng = e.ng;
  std::vector<complex> pg(ng);
  std::vector<double> yr(ng), yi(ng);
  for (int it = 1; it <= e.ntyp_nl; ++it)
    for (int s = 0; s < nstate; ++s) {
      const complex* src = (const complex*)projg + ((size_t)(it - 1) * nstate + s) * ng;
      std::copy(src, src + ng, pg.begin());
      std::copy(e.dyp_re.begin() + (size_t)(it - 1) * ng, e.dyp_re.begin() + (size_t)it * ng, yr.begin());
      std::copy(e.dyp_im.begin() + (size_t)(it - 1) * ng, e.dyp_im.begin() + (size_t)it * ng, yi.begin());
      CPNONLOCAL::eesPsiForcGspace(ng, e.ind_g0 >= 0 ? 1 : 0, e.ind_g0, e.nkx0, pg.data(),
                                   (complex*)fpsi + (size_t)s * ng, yr.data(), yi.data(), e.kx.data(), e.ky.data(),
                                   e.kz.data(), s, 0, it, 1, 0);
    }
}

// CPRSPACEION::CP_getionforce (cp_ions/cp_rspace_ion.C:25-251), cubic
// periodic box (iperd 3), no Grimme dispersion: real-space Ewald energy and
// forces, the self term with its erf factor and the background term.
// ecut_ha: the reciprocal Ewald cutoff in Hartree (k_cut = sqrt(2 ecut_ha)).
extern "C" void ref_rspace_ion(int natm, const double* pos, const double* q, double alp_ewd, double ecut_ha,
                               double box, double* e_real, double* e_self, double* e_bgr, double* fatm) {
  set_cell(box);
  GENERAL_DATA* g = &readonly_general_data;
  g->gencell.iperd = 3;
  g->genewald.alp_ewd = alp_ewd;
  g->genewald.ecut = ecut_ha;
  MDATOMS* md = &readonly_mdatoms;
  md->mdclatoms_info.natm_tot = natm;
  md->mdclatoms_info.cp_grimme = 0;
  std::vector<double> x(natm), y(natm), z(natm), qq(q, q + natm), fx(natm, 0.0), fy(natm, 0.0), fz(natm, 0.0);
  for (int a = 0; a < natm; ++a) { x[a] = pos[3 * a]; y[a] = pos[3 * a + 1]; z[a] = pos[3 * a + 2]; }
  FastAtoms fa;
  fa.natm = natm; fa.x = x.data(); fa.y = y.data(); fa.z = z.data(); fa.q = qq.data();
  fa.fx = fx.data(); fa.fy = fy.data(); fa.fz = fz.data();
  PSSCRATCH scr;
  double recip = 0.0, grimme = 0.0;
  CPRSPACEION::CP_getionforce(natm, &fa, 0, 1, e_real, e_self, e_bgr, &recip, &scr, &grimme);
  for (int a = 0; a < natm; ++a) { fatm[3 * a] = fx[a]; fatm[3 * a + 1] = fy[a]; fatm[3 * a + 2] = fz[a]; }
}

void make_vps_splin(char*, int, int, int, int, double, double, double, double, double*, double*, double*, double*,
                    double*, double*, double*, double*, double*, double*, double*, double*, int, int, int, int, int, int,
                    double, int, int, int*, double*, double*);

// make_vps_splin (interface/vps_params/control_vps_params.C:690-1262) for
// one LOC (ivps_label 0) or KB (1) atom type read from a .pseud file, no
// pressure tensor, no dual grid, one radial channel per l.  Outputs per
// angular channel l = 0..n_ang the spline [nspl][4] at vps[l][nspl][4]
// (the local table in the loc_opt slot), gzvps, gzvps0 (l = 0 KB), q and
// vpsnorm[l].
extern "C" int ref_vps_splin(const char* file, int loc_opt, int n_ang, int ivps_label, int nspl, double dg,
                             double gmin_spl, double gmax_spl, double gmin_true, double* vps, double* gzvps,
                             double* gzvps0, double* q, double* vpsnorm) {
  const size_t len = (size_t)(n_ang + 1) * nspl + 1;
  std::vector<double> v0(len, 0.0), v1(len, 0.0), v2(len, 0.0), v3(len, 0.0);
  std::vector<double> nrm(n_ang + 2, 0.0), gz0(2, 0.0);
  double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0, gz = 0.0, qq = 0.0;
  int ngh = 0;
  std::vector<char> name(file, file + std::strlen(file) + 1);
  make_vps_splin(name.data(), loc_opt, n_ang, ivps_label, nspl, dg, gmin_spl, gmax_spl, gmin_true, v0.data(),
                 v1.data(), v2.data(), v3.data(), &d0, &d1, &d2, &d3, &gz, gz0.data(), &qq, nrm.data(), 1, 1, 1, 1, 0,
                 0, 1.0, 1, 0, &ngh, nullptr, nullptr);
  for (int l = 0; l <= n_ang; ++l)
    for (int j = 0; j < nspl; ++j) {
      const size_t i = (size_t)l * nspl + j + 1;
      double* o = vps + ((size_t)l * nspl + j) * 4;
      o[0] = v0[i]; o[1] = v1[i]; o[2] = v2[i]; o[3] = v3[i];
    }
  *gzvps = gz;
  *gzvps0 = gz0[1];
  *q = qq;
  for (int l = 0; l <= n_ang; ++l) vpsnorm[l] = nrm[l + 1];
  return 0;
}

// ---------------------------------------------------------------------------
// EES local pseudopotential and reciprocal Ewald sum (cp_hart_ext.C:492-1470),
// one RhoRHart chare holding the whole grid [nc][nb][lda], lda = 2 (na/2 + 1),
// in three phases with the oracle's transforms between them:
//   ref_eesl_pack    eesAtmBsplineRgrp (641-900) + eesPackGridRchare
//                    (925-990) per type: the real grids sfAtmTypR
//   ref_eesl_gspace  eesSetEesWghtGgrp (521-635), eesHartEextGchare
//                    (1005-1225) over the types, eesEwaldGchare (1241-1340):
//                    energies, vks(g), the per-type force transforms and
//                    the scaled total structure factor
//   ref_eesl_force   eesAtmForceRchare (1357-1470) per type (flag 0) and
//                    for the Ewald grid (flag 1)
namespace {
struct EeslCfg {
  int natm = 0, ntype = 0, na = 0, nb = 0, nc = 0, order = 0, lda = 0;
  double box = 0.0;
  std::vector<double> x, y, z, q, fx, fy, fz;
  std::vector<int> natm_eext;
  std::vector<std::vector<int>> map_rows;
  std::vector<int*> map_eext;
  std::vector<double> q_typ;
  // RHORHARTDATA storage [nc][natm][order^2 + 1]
  std::vector<std::vector<int>> pidx, nsub, itemp;
  std::vector<std::vector<std::vector<int>>> ig;
  std::vector<std::vector<std::vector<double>>> mn, dx, dy, dz;
  std::vector<int*> ppidx, pnsub, pitemp;
  std::vector<std::vector<int*>> pig;
  std::vector<std::vector<double*>> pmn, pdx, pdy, pdz;
  std::vector<int**> ppig;
  std::vector<double**> ppmn, ppdx, ppdy, ppdz;
  RHORHARTDATA rd;
  FastAtoms fa;
} g_eesl;

void eesl_apply() {
  EeslCfg& e = g_eesl;
  set_cell(e.box);
  CPPSEUDO* ps = &readonly_cp.cppseudo;
  ps->n_interp_ps = e.order;
  ps->ngrid_eext_a = e.na; ps->ngrid_eext_b = e.nb; ps->ngrid_eext_c = e.nc;
  ps->natm_typ = e.ntype;
  ps->natm_eext = e.natm_eext.data();
  ps->map_eext = e.map_eext.data();
  ps->q_typ = e.q_typ.data();
  readonly_mdatoms.mdclatoms_info.natm_tot = e.natm;
}
}  // namespace

// Atoms (0-based types, charges), box, EES grid na x nb x nc and order; the
// per-type real grids sfAtmTypR [ntype][nc][nb][lda] are written.
extern "C" void ref_eesl_pack(int natm, const double* pos, const int* atm_type, const double* q, int ntype, double box,
                              int na, int nb, int nc, int order, double* grids) {
  EeslCfg& e = g_eesl;
  e = EeslCfg();
  e.natm = natm; e.ntype = ntype; e.na = na; e.nb = nb; e.nc = nc; e.order = order; e.box = box;
  e.lda = 2 * (na / 2 + 1);
  e.x.resize(natm); e.y.resize(natm); e.z.resize(natm); e.q.assign(q, q + natm);
  e.fx.assign(natm, 0.0); e.fy = e.fx; e.fz = e.fx;
  for (int a = 0; a < natm; ++a) { e.x[a] = pos[3 * a]; e.y[a] = pos[3 * a + 1]; e.z[a] = pos[3 * a + 2]; }
  e.natm_eext.assign(ntype + 2, 0);
  e.map_rows.assign(ntype + 2, std::vector<int>(natm + 1, 0));
  e.q_typ.assign(ntype + 2, 0.0);
  for (int a = 0; a < natm; ++a) {
    const int t = atm_type[a] + 1;
    e.map_rows[t][++e.natm_eext[t]] = a + 1;
    e.q_typ[t] = q[a];
  }
  e.natm_eext[ntype + 1] = natm;  // the Ewald pass runs over all atoms
  for (int a = 0; a < natm; ++a) e.map_rows[ntype + 1][a + 1] = a + 1;
  e.map_eext.resize(ntype + 2);
  for (int t = 0; t <= ntype + 1; ++t) e.map_eext[t] = e.map_rows[t].data();
  eesl_apply();
  const int n = order, n2 = n * n;
  e.pidx.assign(nc, std::vector<int>(natm, 0)); e.nsub = e.pidx;
  e.itemp.assign(nc, std::vector<int>(n + 1, 0));
  e.ig.assign(nc, std::vector<std::vector<int>>(natm, std::vector<int>(n2 + 1, 0)));
  e.mn.assign(nc, std::vector<std::vector<double>>(natm, std::vector<double>(n2 + 1, 0.0)));
  e.dx = e.mn; e.dy = e.mn; e.dz = e.mn;
  e.ppidx.resize(nc); e.pnsub.resize(nc); e.pitemp.resize(nc);
  e.pig.resize(nc); e.pmn.resize(nc); e.pdx.resize(nc); e.pdy.resize(nc); e.pdz.resize(nc);
  e.ppig.resize(nc); e.ppmn.resize(nc); e.ppdx.resize(nc); e.ppdy.resize(nc); e.ppdz.resize(nc);
  for (int c = 0; c < nc; ++c) {
    e.ppidx[c] = e.pidx[c].data(); e.pnsub[c] = e.nsub[c].data(); e.pitemp[c] = e.itemp[c].data();
    e.pig[c].resize(natm); e.pmn[c].resize(natm); e.pdx[c].resize(natm); e.pdy[c].resize(natm); e.pdz[c].resize(natm);
    for (int a = 0; a < natm; ++a) {
      e.pig[c][a] = e.ig[c][a].data(); e.pmn[c][a] = e.mn[c][a].data();
      e.pdx[c][a] = e.dx[c][a].data(); e.pdy[c][a] = e.dy[c][a].data(); e.pdz[c][a] = e.dz[c][a].data();
    }
    e.ppig[c] = e.pig[c].data(); e.ppmn[c] = e.pmn[c].data();
    e.ppdx[c] = e.pdx[c].data(); e.ppdy[c] = e.pdy[c].data(); e.ppdz[c] = e.pdz[c].data();
  }
  RHORHARTDATA& r = e.rd;
  r.xindex = 0; r.yindex = 0;
  r.gridc_start = 0; r.gridc_end = nc; r.gridb_start = 0; r.gridb_end = nb;
  r.mygridc = nc; r.mygridb = nb;
  r.ngrid_a = na; r.ngrid_b = nb; r.ngrid_c = nc; r.n_interp = n; r.natm = natm;
  r.plane_index = e.ppidx.data(); r.nSub = e.pnsub.data(); r.itemp = e.pitemp.data();
  r.igrid = e.ppig.data(); r.mn = e.ppmn.data();
  r.dmn_x = e.ppdx.data(); r.dmn_y = e.ppdy.data(); r.dmn_z = e.ppdz.data();
  // PSSCRATCH ([j][i], j = 1..n)
  std::vector<double> aj(n + 1), rn(n + 1), rn1(n + 1), fa_(natm), fb(natm), fc(natm);
  std::vector<int> iat(natm), ibt(natm), ict(natm);
  std::vector<std::vector<int>> gi_a(n + 1, std::vector<int>(natm)), gi_b = gi_a, gi_c = gi_a;
  std::vector<std::vector<double>> m_a(n + 1, std::vector<double>(natm)), m_b = m_a, m_c = m_a, u_a = m_a, u_b = m_a,
                                   u_c = m_a, dm_a = m_a, dm_b = m_a, dm_c = m_a;
  auto rows_i = [](std::vector<std::vector<int>>& v) {
    std::vector<int*> p(v.size());
    for (size_t i = 0; i < v.size(); ++i) p[i] = v[i].data();
    return p;
  };
  auto rows_d = [](std::vector<std::vector<double>>& v) {
    std::vector<double*> p(v.size());
    for (size_t i = 0; i < v.size(); ++i) p[i] = v[i].data();
    return p;
  };
  auto pga = rows_i(gi_a), pgb = rows_i(gi_b), pgc = rows_i(gi_c);
  auto pma = rows_d(m_a), pmb = rows_d(m_b), pmc = rows_d(m_c), pua = rows_d(u_a), pub = rows_d(u_b),
       puc = rows_d(u_c), pda = rows_d(dm_a), pdb = rows_d(dm_b), pdc = rows_d(dm_c);
  PSSCRATCH ps;
  ps.aj = aj.data(); ps.rn = rn.data(); ps.rn1 = rn1.data();
  ps.iatemp = iat.data(); ps.ibtemp = ibt.data(); ps.ictemp = ict.data();
  ps.frac_a = fa_.data(); ps.frac_b = fb.data(); ps.frac_c = fc.data();
  ps.igrid_a = pga.data(); ps.igrid_b = pgb.data(); ps.igrid_c = pgc.data();
  ps.mn_a = pma.data(); ps.mn_b = pmb.data(); ps.mn_c = pmc.data();
  ps.ua = pua.data(); ps.ub = pub.data(); ps.uc = puc.data();
  ps.dmn_a = pda.data(); ps.dmn_b = pdb.data(); ps.dmn_c = pdc.data();
  FastAtoms& at = e.fa;
  at.natm = natm; at.x = e.x.data(); at.y = e.y.data(); at.z = e.z.data(); at.q = e.q.data();
  at.fx = e.fx.data(); at.fy = e.fy.data(); at.fz = e.fz.data();
  std::vector<RHORHARTDATA> rv(1, r);
  CPLOCAL::eesAtmBsplineRgrp(&at, rv, &ps);
  const size_t gsz = (size_t)nc * nb * e.lda;
  for (int t = 1; t <= ntype; ++t)
    CPLOCAL::eesPackGridRchare(natm, t, grids + (size_t)(t - 1) * gsz, 0, nc, 0, nb, (int)gsz, r.igrid, r.mn,
                               r.plane_index, r.nSub);
  ps.aj = nullptr; ps.rn = nullptr; ps.rn1 = nullptr;
  ps.iatemp = ps.ibtemp = ps.ictemp = nullptr;
  ps.frac_a = ps.frac_b = ps.frac_c = nullptr;
  ps.igrid_a = ps.igrid_b = ps.igrid_c = nullptr;
  ps.mn_a = ps.mn_b = ps.mn_c = ps.ua = ps.ub = ps.uc = ps.dmn_a = ps.dmn_b = ps.dmn_c = nullptr;
}

// Density g-points (kx, ky, kz) with rho(g); local splines per type
// [ntype][nspl][4], gzvps per type, alpha, the state cutoff in Ry.  In:
// sfg [ntype][npts] complex = the transformed grids at the points.  Out:
// vks(g), sfg overwritten by the atom-force transforms, sftot [npts] the
// scaled total structure factor, b [npts] complex, the energies.
extern "C" void ref_eesl_gspace(int npts, const int* kx, const int* ky, const int* kz, const double* rho, double* vks,
                                int nspl, double gmin, double dg, const double* spl, const double* gzvps,
                                double alp_ewd, double ecut_ry, double* sfg, double* sftot, double* b, double* ehart,
                                double* eext, double* ewd) {
  EeslCfg& e = g_eesl;
  eesl_apply();
  CP* cp = &readonly_cp;
  CPPSEUDO* ps = &cp->cppseudo;
  const int ntype = e.ntype;
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
  std::vector<gridPoint> pts(npts);
  for (int i = 0; i < npts; ++i) { pts[i].d3 = kx[i]; pts[i].d2 = ky[i]; pts[i].d1 = kz[i]; pts[i].offset = i; }
  std::vector<double> bre(npts), bim(npts);
  CPLOCAL::eesSetEesWghtGgrp(npts, pts, bre.data(), bim.data(), e.na, e.nb, e.nc, e.order);
  for (int i = 0; i < npts; ++i) { b[2 * i] = bre[i]; b[2 * i + 1] = bim[i]; }
  for (int i = 0; i < 2 * npts; ++i) { vks[i] = 0.0; sftot[i] = 0.0; }
  *ehart = 0.0; *eext = 0.0;
  for (int t = 1; t <= ntype; ++t)
    CPLOCAL::eesHartEextGchare(npts, t, (complex*)const_cast<double*>(rho), (complex*)vks,
                               (complex*)sfg + (size_t)(t - 1) * npts, (complex*)sftot, bre.data(), bim.data(), ehart,
                               eext, pts, nullptr, 0, 1);
  CPLOCAL::eesEwaldGchare(npts, (complex*)sftot, bre.data(), bim.data(), ewd, pts, 0, nullptr, 0, 1);
  ps->vps0 = ps->vps1 = ps->vps2 = ps->vps3 = nullptr;
  ps->gzvps = nullptr;
  ps->loc_opt = nullptr;
}

// Back-transformed grids [ntype][nc][nb][lda] (per type) and [nc][nb][lda]
// (Ewald) -> atom forces [natm][3] (overwritten).
extern "C" void ref_eesl_force(const double* grids, const double* grid_tot, double* fatm) {
  EeslCfg& e = g_eesl;
  eesl_apply();
  std::fill(e.fx.begin(), e.fx.end(), 0.0);
  std::fill(e.fy.begin(), e.fy.end(), 0.0);
  std::fill(e.fz.begin(), e.fz.end(), 0.0);
  RHORHARTDATA& r = e.rd;
  const size_t gsz = (size_t)e.nc * e.nb * e.lda;
  for (int t = 1; t <= e.ntype; ++t)
    CPLOCAL::eesAtmForceRchare(e.natm, &e.fa, t, r.igrid, r.dmn_x, r.dmn_y, r.dmn_z, r.plane_index, r.nSub,
                               const_cast<double*>(grids) + (size_t)(t - 1) * gsz, 0, e.nc, 0, e.nb, 0);
  CPLOCAL::eesAtmForceRchare(e.natm, &e.fa, 1, r.igrid, r.dmn_x, r.dmn_y, r.dmn_z, r.plane_index, r.nSub,
                             const_cast<double*>(grid_tot), 0, e.nc, 0, e.nb, 1);
  for (int a = 0; a < e.natm; ++a) { fatm[3 * a] = e.fx[a]; fatm[3 * a + 1] = e.fy[a]; fatm[3 * a + 2] = e.fz[a]; }
}
