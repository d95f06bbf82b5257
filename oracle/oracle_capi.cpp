#include <omp.h>
// CPU ORACLE C API — test infrastructure only (see sod2d_oracle.hpp).  Loaded by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline legs through oracle/oracle.py.
#include "sod2d_oracle.hpp"

using namespace sod_oracle;

extern "C" {

int oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

void oracle_gll(int p, double* xi, double* w) {
  double vn[32];
  zelegl(p, xi, vn);
  welegl(p, xi, vn, w);
}

void oracle_lagrange(const double* xi, double xp, double* l, double* dl) {
  eval_lagrange<double>(xi, xp, l);
  eval_lagrange_deriv<double>(xi, xp, dl);
}

void oracle_shape_tables(const int32_t* atoIJK, double* xgp, double* wgp, double* Ngp, double* dNgp,
                         double* dlxigp_ip, int32_t* invAtoIJK, int32_t* gmshAtoI, int32_t* gmshAtoJ,
                         int32_t* gmshAtoK) {
  shape_tables(atoIJK, xgp, wgp, Ngp, dNgp, dlxigp_ip, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK);
}

void oracle_elem_jacobian(int nelem, int npoin, const int32_t* connec, const double* coord,
                          const double* dNgp, const double* wgp, double* gpvol, double* He) {
  elem_jacobian<double>(nelem, npoin, connec, coord, dNgp, wgp, gpvol, He);
}

// Je(i,j) in Fortran order at i + 3*j; He likewise.
void oracle_cofactor_inverse(const double* Je9, double* He9, double* det) {
  double Je[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Je[i][j] = Je9[i + 3 * j];
  cofactor_inverse<double>(Je, He9, *det);
}

void oracle_lumped_mass(int nelem, int npoin, const int32_t* connec, const double* gpvol, double* Ml) {
  lumped_mass_spectral<double>(nelem, npoin, connec, gpvol, Ml);
}

void oracle_char_length(int nelem, int npoin, const int32_t* connec, const double* coord, double* helem) {
  char_length<double>(nelem, npoin, connec, coord, helem);
}

void oracle_char_length_spectral(int nelem, int npoin, const int32_t* connec, const double* coord,
                                 double* helem_l) {
  char_length_spectral<double>(nelem, npoin, connec, coord, helem_l);
}

void oracle_full_convec_ijk(const ElemCtx* ctx, const double* u, const double* q, const double* rho,
                            const double* pr, const double* E, double* Rmass, double* Rmom, double* Rener) {
  full_convec_ijk(*ctx, u, q, rho, pr, E, Rmass, Rmom, Rener);
}

void oracle_full_convec_ijk_H(const ElemCtx* ctx, const double* u, const double* q, const double* rho,
                              const double* pr, const double* E, double* Rmass, double* Rmom, double* Rener) {
  full_convec_ijk_H(*ctx, u, q, rho, pr, E, Rmass, Rmom, Rener);
}

void oracle_generic_scalar_convec_ijk(const ElemCtx* ctx, const double* q, const double* eta,
                                      const double* u, double* R) {
  generic_scalar_convec_ijk(*ctx, q, eta, u, R);
}

void oracle_full_diffusion_ijk(const ElemCtx* ctx, const Params* P, const double* rho_n, const double* rho,
                               const double* u, const double* Tem, const double* mu_fluid,
                               const double* mu_e, const double* mu_sgs, double* Rmass, double* Rmom,
                               double* Rener) {
  full_diffusion_ijk(*ctx, *P, rho_n, rho, u, Tem, mu_fluid, mu_e, mu_sgs, Rmass, Rmom, Rener);
}

void oracle_smart_visc_spectral(const ElemCtx* ctx, const Params* P, const double* Reta, const double* gpvol,
                                const double* wgp, const double* rho, const double* u, const double* csound,
                                const double* Tem, const double* eta, const double* helem_l,
                                const double* helem, double* mu_e, double* mue_l) {
  smart_visc_spectral(*ctx, *P, Reta, gpvol, wgp, rho, u, csound, Tem, eta, helem_l, helem, mu_e, mue_l);
}

void oracle_sutherland(int npoin, const double* Tem, const double* mu_factor, double* mu_fluid) {
  sutherland_viscosity(npoin, Tem, mu_factor, mu_fluid);
}

double oracle_adapt_dt_cfl(const ElemCtx* ctx, const double* helem, const double* u, const double* csound,
                           double cfl_conv, double cfl_diff, const double* mu_fluid, const double* mu_sgs,
                           const double* rho) {
  return adapt_dt_cfl(*ctx, helem, u, csound, cfl_conv, cfl_diff, mu_fluid, mu_sgs, rho);
}

// Runs nsteps explicit RK4 steps of rk_4_main on the state S (level pos=2 only).  When
// capture is non-null its arrays receive the residuals (after /Ml) of stage capture->stage of
// the first step.  bc non-null selects the non-periodic path with those boundary data.
void oracle_rk_4_main(const ElemCtx* ctx, const Params* P, const double* Ml, const double* mu_factor,
                      const double* gpvol, const double* wgp, const double* helem, const double* helem_l,
                      double dt, int nsteps, State* S, StageCapture* capture, const BcData* bc,
                      const BufferData* buf, const double* source, const WallModelData* wmd) {
  Rk4Scratch W(ctx->npoin);
  for (int s = 0; s < nsteps; ++s)
    rk_4_main(*ctx, *P, Ml, mu_factor, gpvol, wgp, helem, helem_l, dt, *S, W, s == 0 ? capture : nullptr, bc, buf,
              source, wmd);
}

void oracle_wall_model(const ElemCtx* ctx, const WallModelData* wmd, const double* rho, const double* ui,
                       const double* mu_fluid, double* Rdiff) {
  eval_wall_model(*ctx, *wmd, rho, ui, mu_fluid, Rdiff);
}

void oracle_compute_field_derivs(const ElemCtx* ctx, const double* levi, const double* rho, const double* u,
                                 double* gradRho, double* curlU, double* divU, double* Qcrit) {
  compute_field_derivs(*ctx, levi, rho, u, gradRho, curlU, divU, Qcrit);
}

void oracle_update_buffer(int npoin, const BufferData* buf, double* rho, double* q, double* E) {
  update_buffer(npoin, *buf, rho, q, E);
}

void oracle_bc_dirichlet_prim(int npoin, const BcData* bc, double* rho, double* q, double* u, double* pr,
                              double* E) {
  temporary_bc_routine_dirichlet_prim(npoin, *bc, rho, q, u, pr, E);
}

// JVP of temporary_bc_routine_dirichlet_prim in (rho, q, E, u) along (drho, dq, dE, du); u is
// the aux_u the slip branch reads (du may be null: held fixed).  Outputs the new state and its
// tangent.
void oracle_bc_jvp(int npoin, const BcData* bc, const double* rho, const double* q, const double* u,
                   const double* E, const double* drho, const double* dq, const double* dE, const double* du,
                   double* rho_out, double* q_out, double* E_out, double* drho_out, double* dq_out,
                   double* dE_out) {
  const int64_t N = npoin;
  std::vector<Dual> r(N), qq(3 * N), uu(3 * N), pp(N), e(N);
  for (int64_t p = 0; p < N; ++p) { r[p] = Dual(rho[p], drho[p]); e[p] = Dual(E[p], dE[p]); }
  for (int64_t p = 0; p < 3 * N; ++p) { qq[p] = Dual(q[p], dq[p]); uu[p] = Dual(u[p], du ? du[p] : 0.0); }
  temporary_bc_routine_dirichlet_prim_t<Dual>(npoin, *bc, r.data(), qq.data(), uu.data(), pp.data(), e.data());
  for (int64_t p = 0; p < N; ++p) {
    rho_out[p] = r[p].v; drho_out[p] = r[p].d; E_out[p] = e[p].v; dE_out[p] = e[p].d;
  }
  for (int64_t p = 0; p < 3 * N; ++p) { q_out[p] = qq[p].v; dq_out[p] = qq[p].d; }
}

void oracle_bc_fix_dirichlet_residual(int npoin, const BcData* bc, double* Rmass, double* Rmom, double* Rener) {
  bc_fix_dirichlet_residual(npoin, *bc, Rmass, Rmom, Rener);
}

void oracle_bc_fix_dirichlet_residual_entropy(int npoin, const BcData* bc, double* R) {
  bc_fix_dirichlet_residual_entropy(npoin, *bc, R);
}

void oracle_eval_laplacian_mult(const ElemCtx* ctx, const double* p, double* ResP) {
  std::vector<double> aux;
  eval_laplacian_mult(*ctx, p, ResP, aux);
}

void oracle_eval_laplacian_diag(const ElemCtx* ctx, const double* dNgp, double* d) {
  eval_laplacian_diag(*ctx, dNgp, d);
}

int oracle_conjgrad_pressure(const ElemCtx* ctx, const double* dNgp, const double* Rp0, double* R,
                             int maxIter, double tol, double* final_rel) {
  return conjGrad_pressure(*ctx, dNgp, Rp0, R, maxIter, tol, final_rel);
}

// CSR_SpMV_scal as pinned by unitt_CSR_SPMV_scal.f90:14-52: rdom holds 0-based row offsets
// (npoin+1), cdom 1-based column ids.
void oracle_csr_spmv_scal(int npoin, int nzdom, const int32_t* rdom, const int32_t* cdom, const double* Mc,
                          const double* v, double* u) {
  (void)nzdom;
  for (int i = 0; i < npoin; ++i) {
    double s = 0.0;
    for (int k = rdom[i]; k < rdom[i + 1]; ++k) s += Mc[k] * v[cdom[k] - 1];
    u[i] = s;
  }
}

}  // extern "C"

extern "C" {

// Stage RHS (mass, mom x3, energy; /Ml) of rk_4_main without the entropy residual; state in
// (rho, q(npoin,3), E), R out as 5 columns of npoin.  mu_sgs may be null (zero).
void oracle_rhs_stage(const ElemCtx* ctx, const Params* P, const double* Ml, const double* mu_factor,
                      const double* mu_e, const double* mu_sgs, const double* rho, const double* q, const double* E,
                      double* R) {
  std::vector<double> zeros;
  if (!mu_sgs) { zeros.assign((size_t)ctx->nelem * nnode, 0.0); mu_sgs = zeros.data(); }
  rhs_stage_t<double>(*ctx, *P, Ml, mu_factor, mu_e, mu_sgs, rho, q, E, R);
}

// oracle_rhs_stage evaluated in x87 extended precision (inputs and outputs FP64): the rounding
// floor against which the FP64 evaluations are measured on ill-conditioned residuals.
void oracle_rhs_stage_ld(const ElemCtx* ctx, const Params* P, const double* Ml, const double* mu_factor,
                         const double* mu_e, const double* mu_sgs, const double* rho, const double* q,
                         const double* E, double* R) {
  const int64_t N = ctx->npoin;
  std::vector<double> zeros;
  if (!mu_sgs) { zeros.assign((size_t)ctx->nelem * nnode, 0.0); mu_sgs = zeros.data(); }
  std::vector<long double> r(rho, rho + N), qq(q, q + 3 * N), e(E, E + N), out(5 * N);
  rhs_stage_t<long double>(*ctx, *P, Ml, mu_factor, mu_e, mu_sgs, r.data(), qq.data(), e.data(), out.data());
  for (int64_t p = 0; p < 5 * N; ++p) R[p] = (double)out[p];
}

// Exact JVP of oracle_rhs_stage by forward-mode dual numbers: dR = (dR/dU) dU, U = (rho,q,E).
void oracle_rhs_jvp(const ElemCtx* ctx, const Params* P, const double* Ml, const double* mu_factor,
                    const double* mu_e, const double* mu_sgs, const double* rho, const double* q, const double* E,
                    const double* drho, const double* dq, const double* dE, double* R, double* dR,
                    const WallModelData* wmd) {
  const int64_t N = ctx->npoin;
  std::vector<double> zeros;
  if (!mu_sgs) { zeros.assign((size_t)ctx->nelem * nnode, 0.0); mu_sgs = zeros.data(); }
  std::vector<Dual> r(N), qq(3 * N), e(N), out(5 * N);
  for (int64_t p = 0; p < N; ++p) { r[p] = Dual(rho[p], drho[p]); e[p] = Dual(E[p], dE[p]); }
  for (int64_t p = 0; p < 3 * N; ++p) qq[p] = Dual(q[p], dq[p]);
  rhs_stage_t<Dual>(*ctx, *P, Ml, mu_factor, mu_e, mu_sgs, r.data(), qq.data(), e.data(), out.data(), wmd);
  for (int64_t p = 0; p < 5 * N; ++p) { if (R) R[p] = out[p].v; dR[p] = out[p].d; }
}

// Number of arithmetic operations (+ - * /, sqrt and pow as one each) of one oracle_rhs_stage
// evaluation, counted single-threaded with the OpCount type.
double oracle_rhs_opcount(const ElemCtx* ctx, const Params* P, const double* Ml, const double* mu_factor,
                          const double* mu_e, const double* rho, const double* q, const double* E) {
  const int64_t N = ctx->npoin;
  std::vector<double> zeros((size_t)ctx->nelem * nnode, 0.0);
  std::vector<OpCount> r(N), qq(3 * N), e(N), out(5 * N);
  for (int64_t p = 0; p < N; ++p) { r[p] = OpCount(rho[p]); e[p] = OpCount(E[p]); }
  for (int64_t p = 0; p < 3 * N; ++p) qq[p] = OpCount(q[p]);
  const int nt = omp_get_max_threads();
  omp_set_num_threads(1);
  op_count() = 0;
  rhs_stage_t<OpCount>(*ctx, *P, Ml, mu_factor, mu_e, zeros.data(), r.data(), qq.data(), e.data(), out.data());
  const double n = (double)op_count();
  omp_set_num_threads(nt);
  return n;
}

}  // extern "C"

extern "C" {

// Legacy unit-test API (1-based connec, Fortran layouts): see legacy_convec / legacy_mom_diffusion.
void oracle_legacy_mass_convec(int nelem, int ngaus, int npoin, int nnode, int ndime, const int* connec,
                               const double* Ngp, const double* gpcar, const double* gpvol, const double* q, double* R) {
  legacy_convec({nelem, ngaus, npoin, nnode, ndime}, connec, Ngp, gpcar, gpvol, 0, q, nullptr, nullptr, R);
}
void oracle_legacy_mom_convec(int nelem, int ngaus, int npoin, int nnode, int ndime, const int* connec,
                              const double* Ngp, const double* gpcar, const double* gpvol, const double* u,
                              const double* q, const double* pr, double* R) {
  legacy_convec({nelem, ngaus, npoin, nnode, ndime}, connec, Ngp, gpcar, gpvol, 1, q, u, pr, R);
}
void oracle_legacy_ener_convec(int nelem, int ngaus, int npoin, int nnode, int ndime, const int* connec,
                               const double* Ngp, const double* gpcar, const double* gpvol, const double* u,
                               const double* pr, const double* E, double* R) {
  legacy_convec({nelem, ngaus, npoin, nnode, ndime}, connec, Ngp, gpcar, gpvol, 2, u, E, pr, R);
}
void oracle_legacy_mom_diffusion(int nelem, int ngaus, int npoin, int nnode, int ndime, const int* connec,
                                 const double* Ngp, const double* gpcar, const double* gpvol, const double* u,
                                 const double* mu_e, double* R) {
  (void)Ngp;
  legacy_mom_diffusion({nelem, ngaus, npoin, nnode, ndime}, connec, gpcar, gpvol, u, mu_e, R);
}

}  // extern "C"

extern "C" {

double oracle_volavg_ek(const ElemCtx* ctx, const double* Ngp, double rho0, const double* rho, const double* u) {
  return volAvg_EK(*ctx, Ngp, rho0, rho, u);
}
void oracle_visc_dissipation_rate(const ElemCtx* ctx, const double* dNgp, double rho0, const double* mu_fluid,
                                  const double* mu_e, const double* u, double volT, double* eps3) {
  visc_dissipationRate(*ctx, dNgp, rho0, mu_fluid, mu_e, u, volT, eps3);
}

}  // extern "C"
