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
#include "../class_defs/CP_OPERATIONS/class_cpintegrate.h"
#include <vector>

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
