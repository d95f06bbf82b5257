// Hand-written adjoint (vector-Jacobian product) of the stage RHS and of one RK4 step (sm_100a).
//
// The stage RHS is R(U) = (1/Ml) Gather_e[ gpvol * conv_e(U) + diff_e(U) ] with U = (rho, q, E),
// conv from full_convec_ijk (elem_convec.f90:211-460, energy with h), diff from
// full_diffusion_ijk (elem_diffu.f90:12-198), the stage EOS of time_integ.f90:266-285 and
// Sutherland's law (mod_fluid_viscosity.f90:21-41) - Sutherland is differentiated, the entropy
// viscosity mu_e is frozen at its forward value (it is updated once per step from the state
// after the step, time_integ.f90:492-493), as is dt.
//
// k_rhs_vjp (one element per CTA, one thread per gauss point, FP64) recomputes the forward
// derivative quantities, then runs the reverse sweep:
//   diffusion  output seeds -> D applied along lines (the transpose of pass 2's D^T) ->
//              contravariant-flux adjoints -> stress/heat-flux adjoints
//   convection the split-form combination reversed pointwise
//   both       derivative adjoints mapped back with He^T and D^T along lines to nodal product
//              fields, then the product rule, the EOS and u = q/rho in reverse.
// The energy convection is linear in (h, k) through h + k only (every h term has a k twin with
// the same structure), so the adjoint works with the total enthalpy H = h + k; q (x) u is
// symmetric (rho u_c u_j), so its 9 components reduce to 6 like u (x) u.  The 29 nodal adjoint
// fields go through shared memory in chunks of kChunk fields (3 line arrays each), which keeps
// the CTA at 21 KB of shared memory.
// Element-node adjoints are assembled by the same ordered CSR gather as the forward path.
#include "sod_internal.cuh"
#include <cmath>

namespace sod {
int ensure_step_buffers(SodMesh* m, bool mixed);
int les_in(SodMesh* m, const SodState* s, cudaStream_t st);
int launch_rhs(SodMesh* m, bool mixed, int epb, const double* rho, const double* q0, const double* q1,
               const double* q2, const double* E, const double* mu_factor, const double* musgs_int, cudaStream_t st);

namespace adj {

constexpr double kC1 = 0.000001458;
constexpr double kS = 110.4;
// forward fields staged in shared memory (H = h + k total enthalpy); the products rho H, H u and
// u (x) u are formed from them at the line points
enum { F_RHO = 0, F_H, F_T, F_U0, F_U1, F_U2, F_Q0, F_Q1, F_Q2, NF_FWD };
// nodal adjoint fields receiving D^T line sums: 11 gradient fields, rho H u and H u (divergence),
// q (x) u and u (x) u (symmetric, divergence by rows)
enum { A_RHO = 0, A_P, A_H, A_RH, A_T, A_U0, A_U1, A_U2, A_Q0, A_Q1, A_Q2,
       A_FE0, A_FE1, A_FE2, A_FUE0, A_FUE1, A_FUE2,
       A_F00, A_F01, A_F02, A_F11, A_F12, A_F22,
       A_UU00, A_UU01, A_UU02, A_UU11, A_UU12, A_UU22, NF_ADJ };
constexpr int kChunk = 10;
constexpr int kArrays = 3 * kChunk;  // >= NF_FWD + 6 (forward phase) and >= 6 (seed phase)
static_assert(kArrays >= NF_FWD + 6, "shared arrays");

struct VjpArgs {
  int nelem;
  const int32_t* __restrict__ econn;
  const double* __restrict__ geo;
  const double* __restrict__ mue;        // internal [e][64]
  const double* __restrict__ musgs;      // internal [e][64] frozen SGS viscosity, or null
  const double* __restrict__ rho;
  const double* __restrict__ q0;
  const double* __restrict__ q1;
  const double* __restrict__ q2;
  const double* __restrict__ E;
  const double* __restrict__ mu_factor;
  const double* __restrict__ w;          // seeds / Ml: 5 columns of npoin (mass, mom x3, energy)
  int64_t npoin;
  double* out;                           // [(e*64 + d)*NRES + f] element-node adjoints (rho, q x3, E, 0)
  DMat D;
  DevParams prm;
};

__device__ __forceinline__ void giso_line(const double* f, int i, int j, int k, const double (&D)[NP1][NP1],
                                          double& gx, double& gy, double& gz) {
  gx = D[i][0] * f[sidx(0, j, k)] + D[i][1] * f[sidx(1, j, k)] + D[i][2] * f[sidx(2, j, k)] + D[i][3] * f[sidx(3, j, k)];
  gy = D[j][0] * f[sidx(i, 0, k)] + D[j][1] * f[sidx(i, 1, k)] + D[j][2] * f[sidx(i, 2, k)] + D[j][3] * f[sidx(i, 3, k)];
  gz = D[k][0] * f[sidx(i, j, 0)] + D[k][1] * f[sidx(i, j, 1)] + D[k][2] * f[sidx(i, j, 2)] + D[k][3] * f[sidx(i, j, 3)];
}

// sum_m D[m][i] fx(m,j,k) + D[m][j] fy(i,m,k) + D[m][k] fz(i,j,m)
__device__ __forceinline__ double divT_line(const double* fx, const double* fy, const double* fz, int i, int j, int k,
                                            const double (&D)[NP1][NP1]) {
  double s = 0.0;
#pragma unroll
  for (int m = 0; m < NP1; ++m)
    s += D[m][i] * fx[sidx(m, j, k)] + D[m][j] * fy[sidx(i, m, k)] + D[m][k] * fz[sidx(i, j, m)];
  return s;
}

// symmetric pair (c, j) of each q(x)u / u(x)u field, in enum order 00 01 02 11 12 22
__device__ constexpr int sym_c(int t) { return t < 3 ? 0 : (t < 5 ? 1 : 2); }
__device__ constexpr int sym_j(int t) { return t < 3 ? t : (t < 5 ? t - 2 : 2); }

#ifndef SOD_VJP_MIN_BLOCKS
#define SOD_VJP_MIN_BLOCKS 1  // CTAs per SM the register allocation must allow
#endif
// TOTH: flag_total_enthalpy (energy convection of full_convec_ijk_H)
template <bool TOTH>
__global__ void __launch_bounds__(64, SOD_VJP_MIN_BLOCKS) k_rhs_vjp(const VjpArgs a) {
  __shared__ __align__(16) double sm[kArrays * FSTRIDE];
  __shared__ DMat Ds;
  const int e = blockIdx.x, d = threadIdx.x;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  if (d < 16) Ds.d[d >> 2][d & 3] = a.D.d[d >> 2][d & 3];
  const double* Ge = a.geo + (size_t)e * NGEO * NN;
  double H[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) H[c] = Ge[c * NN + d];
  const double gpv = Ge[9 * NN + d];
  const int n = a.econn[(size_t)e * NN + d];
  const double g = a.prm.gamma, Rg = a.prm.Rgas;
  const double rho = a.rho[n];
  const double qv[3] = {a.q0[n], a.q1[n], a.q2[n]};
  const double Et = a.E[n];
  const double uv[3] = {qv[0] / rho, qv[1] / rho, qv[2] / rho};
  const double umag = uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2];
  const double kk = 0.5 * umag;
  const double p = rho * (g - 1.0) * ((Et / rho) - 0.5 * umag);
  const double h = (g / (g - 1.0)) * p / rho;
  const double T = p / (rho * Rg);
  const double Ht = h + kk;
  const double mf = a.mu_factor[n];
  const double muf = mf * kC1 * (T * sqrt(T)) / (T + kS);
  const double dmuf_dT = mf * kC1 * (1.5 * sqrt(T) * (T + kS) - T * sqrt(T)) / ((T + kS) * (T + kS));
  const double mue = a.mue[(size_t)e * NN + d];
  const double musgs = a.musgs ? a.musgs[(size_t)e * NN + d] : 0.0;
  // elem_diffu.f90: the molecular part of the stress carries rho mu_sgs (mu_fgp), the heat flux
  // Cp/0.9 rho mu_sgs; both enter the reverse sweep through rho
  const double mufgp = muf + rho * musgs;

  // ---------------- forward recompute of the derivative quantities ----------------
  double* Fw = sm;
  Fw[F_RHO * FSTRIDE + s] = rho;
  Fw[F_H * FSTRIDE + s] = Ht;
  Fw[F_T * FSTRIDE + s] = T;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Fw[(F_U0 + c) * FSTRIDE + s] = uv[c];
    Fw[(F_Q0 + c) * FSTRIDE + s] = qv[c];
  }
  __syncthreads();
  auto grad = [&](int f, double* o) {
    double gx, gy, gz;
    giso_line(Fw + f * FSTRIDE, i, j, k, Ds.d, gx, gy, gz);
#pragma unroll
    for (int r = 0; r < 3; ++r) o[r] = H[3 * r] * gx + H[3 * r + 1] * gy + H[3 * r + 2] * gz;
  };
  double gRho[3], gH[3], gRH[3], gT[3], gU[3][3], gQ[3][3];
  grad(F_RHO, gRho); grad(F_H, gH); grad(F_T, gT);
#pragma unroll
  for (int c = 0; c < 3; ++c) { grad(F_U0 + c, gU[c]); grad(F_Q0 + c, gQ[c]); }
  // the product fields rho H, H u_c and u (x) u are formed at the line points from the staged
  // factors (the line weight applied to the first factor), not staged themselves
  double divHu = 0.0, divFuu[3] = {0.0, 0.0, 0.0};
  {
    double gRHi[3];
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      double lRH = 0.0, lHu[3] = {0.0, 0.0, 0.0}, lUU[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      const int x = dir == 0 ? i : (dir == 1 ? j : k);
#pragma unroll
      for (int m = 0; m < NP1; ++m) {
        const int sp = dir == 0 ? sidx(m, j, k) : (dir == 1 ? sidx(i, m, k) : sidx(i, j, m));
        const double w = Ds.d[x][m];
        const double r_ = Fw[F_RHO * FSTRIDE + sp], H_ = Fw[F_H * FSTRIDE + sp];
        const double u_[3] = {Fw[F_U0 * FSTRIDE + sp], Fw[F_U1 * FSTRIDE + sp], Fw[F_U2 * FSTRIDE + sp]};
        const double wH = w * H_;
        lRH += wH * r_;
#pragma unroll
        for (int c = 0; c < 3; ++c) lHu[c] += wH * u_[c];
        const double wu[3] = {w * u_[0], w * u_[1], w * u_[2]};
#pragma unroll
        for (int t = 0; t < 6; ++t) lUU[t] += wu[sym_c(t)] * u_[sym_j(t)];
      }
      gRHi[dir] = lRH;
#pragma unroll
      for (int c = 0; c < 3; ++c) divHu += H[3 * c + dir] * lHu[c];
      // rows of the symmetric u (x) u: row0 = (00,01,02), row1 = (01,11,12), row2 = (02,12,22)
      divFuu[0] += H[dir] * lUU[0] + H[3 + dir] * lUU[1] + H[6 + dir] * lUU[2];
      divFuu[1] += H[dir] * lUU[1] + H[3 + dir] * lUU[3] + H[6 + dir] * lUU[4];
      divFuu[2] += H[dir] * lUU[2] + H[3 + dir] * lUU[4] + H[6 + dir] * lUU[5];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) gRH[r] = H[3 * r] * gRHi[0] + H[3 * r + 1] * gRHi[1] + H[3 * r + 2] * gRHi[2];
  }
  const double divU = gU[0][0] + gU[1][1] + gU[2][2];
  const double divQ = gQ[0][0] + gQ[1][1] + gQ[2][2];
  // diffusion pass 1 (stresses) and the contravariant gradRho / gradT fluxes for pass 2
  const double mut = mufgp + mue;
  double tau[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) tau[r][c] = mut * (gU[r][c] + gU[c][r]);
#pragma unroll
  for (int r = 0; r < 3; ++r) tau[r][r] -= mufgp * (2.0 / 3.0) * divU;
  double* V6 = sm + NF_FWD * FSTRIDE;  // does not overlap the forward fields
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    V6[dir * FSTRIDE + s] = gpv * (H[dir] * gRho[0] + H[3 + dir] * gRho[1] + H[6 + dir] * gRho[2]);
    V6[(3 + dir) * FSTRIDE + s] = gpv * (H[dir] * gT[0] + H[3 + dir] * gT[1] + H[6 + dir] * gT[2]);
  }
  __syncthreads();  // forward fields consumed; V6 complete
  const double divDr = divT_line(V6, V6 + FSTRIDE, V6 + 2 * FSTRIDE, i, j, k, Ds.d);
  const double divDgT = divT_line(V6 + 3 * FSTRIDE, V6 + 4 * FSTRIDE, V6 + 5 * FSTRIDE, i, j, k, Ds.d);

  // ---------------- reverse sweep ----------------
  const int64_t N = a.npoin;
  const double wm = a.w[n], we = a.w[n + 4 * N];
  const double wmo[3] = {a.w[n + N], a.w[n + 2 * N], a.w[n + 3 * N]};
  double rb = 0.0, Hb = 0.0, pb = 0.0, Tb = 0.0, mufb = 0.0;
  double ub[3] = {0, 0, 0}, qb[3] = {0, 0, 0};
  double gRhob[3] = {0, 0, 0}, gPb[3] = {0, 0, 0}, gHb[3] = {0, 0, 0}, gRHb[3] = {0, 0, 0}, gTb[3] = {0, 0, 0};
  double gUb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, gQb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double dFeb = 0.0, dFueb = 0.0, divUb = 0.0, divQb = 0.0;
  double dFb[3] = {0, 0, 0}, dFuub[3] = {0, 0, 0};

  // diffusion outputs (elem_diffu.f90:143-193): nu_e*divD(gradRho), divD(tauU) + kappa*divD(gradT),
  // divD(tau row r); nu_e and kappa belong to the output node
  const double CpPr = a.prm.Cp / a.prm.Prt;
  const double nu_e = a.prm.c_rho * mue / rho;
  const double kappa = muf * CpPr + a.prm.c_ener * mue * CpPr + a.prm.Cp09 * rho * musgs;
  rb += wm * divDr * (-a.prm.c_rho * mue / (rho * rho));
  mufb += we * divDgT * CpPr;
  rb += we * divDgT * a.prm.Cp09 * musgs;
  double* S6 = sm;  // overlaps forward fields only (read before the last barrier), not V6
  S6[0 * FSTRIDE + s] = nu_e * wm;
  S6[1 * FSTRIDE + s] = we;
  S6[2 * FSTRIDE + s] = kappa * we;
#pragma unroll
  for (int r = 0; r < 3; ++r) S6[(3 + r) * FSTRIDE + s] = wmo[r];
  __syncthreads();
  {
    double taub[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int v = 0; v < 6; ++v) {
      double gx, gy, gz;
      giso_line(S6 + v * FSTRIDE, i, j, k, Ds.d, gx, gy, gz);  // adjoint of D^T: D along lines
      double Vb[3];
#pragma unroll
      for (int r = 0; r < 3; ++r) Vb[r] = gpv * (H[3 * r] * gx + H[3 * r + 1] * gy + H[3 * r + 2] * gz);
      if (v == 0) {
#pragma unroll
        for (int r = 0; r < 3; ++r) gRhob[r] += Vb[r];
      } else if (v == 1) {  // tauU_r = sum_c tau_rc u_c
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            taub[r][c] += Vb[r] * uv[c];
            ub[c] += Vb[r] * tau[r][c];
          }
      } else if (v == 2) {
#pragma unroll
        for (int r = 0; r < 3; ++r) gTb[r] += Vb[r];
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) taub[v - 3][c] += Vb[c];
      }
    }
    // tau_rc = (mu_fgp+mue)(du_r/dx_c + du_c/dx_r) - delta_rc mu_fgp 2/3 div u, mu_fgp = muf + rho musgs
    double mufgpb = 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gUb[r][c] += mut * taub[r][c];
        gUb[c][r] += mut * taub[r][c];
        mufgpb += taub[r][c] * (gU[r][c] + gU[c][r]);
      }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      mufgpb += -taub[r][r] * (2.0 / 3.0) * divU;
      divUb += -mufgp * (2.0 / 3.0) * taub[r][r];
    }
    mufb += mufgpb;
    rb += mufgpb * musgs;
  }

  // convection (elem_convec.f90:412-434), seeds times gpvol; energy through H = h + k
  {
    const double mm = gpv * wm, me = gpv * we;
    const double mc[3] = {gpv * wmo[0], gpv * wmo[1], gpv * wmo[2]};
    // mass: 1/2 (div q + rho div u + u . grad rho)
    divQb += 0.5 * mm; rb += 0.5 * divU * mm; divUb += 0.5 * rho * mm;
#pragma unroll
    for (int c = 0; c < 3; ++c) { ub[c] += 0.5 * gRho[c] * mm; gRhob[c] += 0.5 * uv[c] * mm; }
    if constexpr (TOTH) {
      // full_convec_ijk_H (elem_convec.f90:171-177): 1/2 (div((E + p) u) + (E + p) div u
      // + u.grad(E + p)) with E + p = rho H (the same function of rho, q, E)
      dFeb += 0.5 * me;
      rb += 0.5 * Ht * divU * me; Hb += 0.5 * rho * divU * me; divUb += 0.5 * rho * Ht * me;
#pragma unroll
      for (int c = 0; c < 3; ++c) { ub[c] += 0.5 * gRH[c] * me; gRHb[c] += 0.5 * uv[c] * me; }
    } else {
      // energy: 1/4 (H div q + rho H div u + q.grad H + u.grad(rho H) + H u.grad rho
      //              + div(rho H u) + rho div(H u))
      dFeb += 0.25 * me;
      Hb += 0.25 * divQ * me; divQb += 0.25 * Ht * me;
      rb += 0.25 * Ht * divU * me; Hb += 0.25 * rho * divU * me; divUb += 0.25 * rho * Ht * me;
      rb += 0.25 * divHu * me; dFueb += 0.25 * rho * me;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        qb[c] += 0.25 * gH[c] * me; gHb[c] += 0.25 * qv[c] * me;
        ub[c] += 0.25 * gRH[c] * me; gRHb[c] += 0.25 * uv[c] * me;
        Hb += 0.25 * uv[c] * gRho[c] * me; ub[c] += 0.25 * Ht * gRho[c] * me; gRhob[c] += 0.25 * Ht * uv[c] * me;
      }
    }
    // momentum: 1/4 (div(q u) + u div q + q div u + rho div(u u) + u u.grad rho + q.grad u + u.grad q)
    //           + grad p
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double mu_c = mc[c];
      dFb[c] += 0.25 * mu_c;
      ub[c] += 0.25 * divQ * mu_c; divQb += 0.25 * uv[c] * mu_c;
      qb[c] += 0.25 * divU * mu_c; divUb += 0.25 * qv[c] * mu_c;
      rb += 0.25 * divFuu[c] * mu_c; dFuub[c] += 0.25 * rho * mu_c;
      gPb[c] += mu_c;
#pragma unroll
      for (int jd = 0; jd < 3; ++jd) {
        ub[c] += 0.25 * uv[jd] * gRho[jd] * mu_c;
        ub[jd] += 0.25 * uv[c] * gRho[jd] * mu_c;
        gRhob[jd] += 0.25 * uv[c] * uv[jd] * mu_c;
        qb[jd] += 0.25 * gU[c][jd] * mu_c;
        gUb[c][jd] += 0.25 * qv[jd] * mu_c;
        ub[jd] += 0.25 * gQ[c][jd] * mu_c;
        gQb[c][jd] += 0.25 * uv[jd] * mu_c;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      gUb[c][c] += divUb;
      gQb[c][c] += divQb;
    }
  }

  // derivative adjoints -> iso adjoints (He^T) -> D^T line sums, in chunks of kChunk fields
  auto iso3 = [&](int f, double* o) {
    if (f <= A_Q2) {  // gradient fields: sum_r He(r,dir) gb_r
      const double* gb = f == A_RHO ? gRhob : f == A_P ? gPb : f == A_H ? gHb : f == A_RH ? gRHb
                         : f == A_T ? gTb : f <= A_U2 ? gUb[f - A_U0] : gQb[f - A_Q0];
#pragma unroll
      for (int dir = 0; dir < 3; ++dir) o[dir] = H[dir] * gb[0] + H[3 + dir] * gb[1] + H[6 + dir] * gb[2];
    } else if (f <= A_FUE2) {  // component c of a vector whose divergence has adjoint db
      const int c = f <= A_FE2 ? f - A_FE0 : f - A_FUE0;
      const double db = f <= A_FE2 ? dFeb : dFueb;
#pragma unroll
      for (int dir = 0; dir < 3; ++dir) o[dir] = H[3 * c + dir] * db;
    } else {  // symmetric (c,jj) entry: row c takes d/dx_jj, row jj takes d/dx_c
      const int t = f <= A_F22 ? f - A_F00 : f - A_UU00;
      const double* db = f <= A_F22 ? dFb : dFuub;
      const int c = sym_c(t), jj = sym_j(t);
#pragma unroll
      for (int dir = 0; dir < 3; ++dir)
        o[dir] = H[3 * jj + dir] * db[c] + (c != jj ? H[3 * c + dir] * db[jj] : 0.0);
    }
  };
  // nodal product fields -> primitives (product rule at the output node)
  auto apply = [&](int f, double t) {
    if (f == A_RHO) {
      rb += t;
    } else if (f == A_P) {
      pb += t;
    } else if (f == A_H) {
      Hb += t;
    } else if (f == A_RH) {
      rb += Ht * t; Hb += rho * t;
    } else if (f == A_T) {
      Tb += t;
    } else if (f <= A_U2) {
      ub[f - A_U0] += t;
    } else if (f <= A_Q2) {
      qb[f - A_Q0] += t;
    } else if (f <= A_FE2) {  // rho H u_c
      const int c = f - A_FE0;
      rb += Ht * uv[c] * t; Hb += rho * uv[c] * t; ub[c] += rho * Ht * t;
    } else if (f <= A_FUE2) {  // H u_c
      const int c = f - A_FUE0;
      Hb += uv[c] * t; ub[c] += Ht * t;
    } else if (f <= A_F22) {  // q_c u_jj
      const int c = sym_c(f - A_F00), jj = sym_j(f - A_F00);
      qb[c] += uv[jj] * t; ub[jj] += qv[c] * t;
    } else {  // u_c u_jj
      const int c = sym_c(f - A_UU00), jj = sym_j(f - A_UU00);
      ub[c] += uv[jj] * t; ub[jj] += uv[c] * t;
    }
  };
  __syncthreads();  // seed arrays consumed before the chunks overwrite them
#pragma unroll
  for (int c0 = 0; c0 < NF_ADJ; c0 += kChunk) {
#pragma unroll
    for (int f = c0; f < c0 + kChunk && f < NF_ADJ; ++f) {
      double o[3];
      iso3(f, o);
#pragma unroll
      for (int dir = 0; dir < 3; ++dir) sm[((f - c0) * 3 + dir) * FSTRIDE + s] = o[dir];
    }
    __syncthreads();
#pragma unroll
    for (int f = c0; f < c0 + kChunk && f < NF_ADJ; ++f) {
      const double* b = sm + (size_t)(f - c0) * 3 * FSTRIDE;
      apply(f, divT_line(b, b + FSTRIDE, b + 2 * FSTRIDE, i, j, k, Ds.d));
    }
    if (c0 + kChunk < NF_ADJ) __syncthreads();
  }

  // H = h + k; Sutherland, EOS and u = q/rho in reverse (time_integ.f90:266-285,
  // mod_fluid_viscosity.f90:37)
  double hb = Hb, kb = Hb;
  Tb += mufb * dmuf_dT;
  pb += hb * g / ((g - 1.0) * rho);
  rb += -hb * h / rho;
  pb += Tb / (rho * Rg);
  rb += -Tb * T / rho;
  const double Eb = (g - 1.0) * pb;
  rb += -(g - 1.0) * kk * pb;
  kb += -(g - 1.0) * rho * pb;
#pragma unroll
  for (int c = 0; c < 3; ++c) ub[c] += uv[c] * kb;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    qb[c] += ub[c] / rho;
    rb += -uv[c] * ub[c] / rho;
  }
  store_res6<double>(a.out, (size_t)e * NN + d, rb, qb[0], qb[1], qb[2], Eb, 0.0);
}

}  // namespace adj
}  // namespace sod

// ---------------------------------------------------------------------------------------------
// node-side kernels of the adjoint: seeds, ordered gathers, stage states
// ---------------------------------------------------------------------------------------------
namespace sod {
namespace adj {

struct Cols5 {
  const double* c[5];
};
struct MCols5 {
  double* c[5];
};

// w = scale * src / Ml (scale = -dt * coef when dt is given, else 1)
__global__ void k_seed(int64_t N, Cols5 src, const double* __restrict__ Ml, const double* __restrict__ dt,
                       double coef, double* __restrict__ w, MCols5 keep) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const double sc = dt ? -(*dt) * coef : 1.0;
  const double inv = 1.0 / Ml[n];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const double v = src.c[f][n];
    w[f * N + n] = sc * v * inv;
    if (keep.c[f]) keep.c[f][n] = v;
  }
}

// Ordered gather of the element-node adjoints [e][6][64] (ascending element order, like the
// forward assembly), plus extra ([5][npoin], or null); Ybar = sum; out = Ybar (mode 0) or
// acc += Ybar (mode 1, acc = out); when wnext is set: wnext = -dt (cb * ybar + ca * Ybar) / Ml.
__global__ void __launch_bounds__(256) k_gather_vjp(int64_t N, const int32_t* __restrict__ ptr,
                                                    const int32_t* __restrict__ idx, const double* __restrict__ el,
                                                    MCols5 out, int mode, const double* __restrict__ ybar,
                                                    const double* __restrict__ Ml, const double* __restrict__ dt,
                                                    double cb, double ca, double* __restrict__ wnext,
                                                    const double* __restrict__ extra) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double r[5] = {0, 0, 0, 0, 0};
  const int beg = ptr[n], end = ptr[n + 1];
  for (int c = beg; c < end; ++c) {
    double v[6];
    load_res6<double>(el, (size_t)idx[c], v);
#pragma unroll
    for (int f = 0; f < 5; ++f) r[f] += v[f];
  }
  if (extra) {  // the wall model's node-level adjoint
#pragma unroll
    for (int f = 0; f < 5; ++f) r[f] += extra[f * N + n];
  }
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    if (mode == 1) out.c[f][n] += r[f];
    else out.c[f][n] = r[f];
  }
  if (wnext) {
    const double sc = -(*dt) / Ml[n];
#pragma unroll
    for (int f = 0; f < 5; ++f) wnext[f * N + n] = sc * (cb * ybar[f * N + n] + ca * r[f]);
  }
}

// acc += Ybar (the adjoint of a stage state after the boundary routine's adjoint); when wnext
// is set: wnext = -dt (cb * ybar + ca * Ybar) / Ml
__global__ void __launch_bounds__(256) k_accum_seed(int64_t N, const double* __restrict__ Yb, MCols5 acc,
                                                    const double* __restrict__ ybar, const double* __restrict__ Ml,
                                                    const double* __restrict__ dt, double cb, double ca,
                                                    double* __restrict__ wnext) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double r[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    r[f] = Yb[f * N + n];
    acc.c[f][n] += r[f];
  }
  if (wnext) {
    const double sc = -(*dt) / Ml[n];
#pragma unroll
    for (int f = 0; f < 5; ++f) wnext[f * N + n] = sc * (cb * ybar[f * N + n] + ca * r[f]);
  }
}

// stage state: ys = y - coef * dt * gather(rel)/Ml   (time_integ.f90:301-318)
__global__ void __launch_bounds__(256) k_stage_state(int64_t N, const int32_t* __restrict__ ptr,
                                                     const int32_t* __restrict__ idx, const double* __restrict__ el,
                                                     const double* __restrict__ Ml, const double* __restrict__ dt,
                                                     double coef, Cols5 y, const double* __restrict__ src,
                                                     const double* __restrict__ wmc, double* __restrict__ ys) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double r[5] = {0, 0, 0, 0, 0};
  const int beg = ptr[n], end = ptr[n + 1];
  for (int c = beg; c < end; ++c) {
    double v[6];
    load_res6<double>(el, (size_t)idx[c], v);
#pragma unroll
    for (int f = 0; f < 5; ++f) r[f] += v[f];
  }
  // same operation order as the forward stage gather, so the stage states match it bit for bit
  const double ml = Ml[n];
  if (src) {
#pragma unroll
    for (int d = 0; d < 3; ++d) r[1 + d] -= ml * src[d * N + n];
  }
  if (wmc) {
#pragma unroll
    for (int d = 0; d < 3; ++d) r[1 + d] += wmc[d * N + n];
  }
  const double da = (*dt) * coef;
#pragma unroll
  for (int f = 0; f < 5; ++f) ys[f * N + n] = y.c[f][n] - da * (r[f] / ml);
}

// y0 - dt sum_s b_s R_s from the stage states (dt R_1 = 2 (y0 - Y2), dt R_2 = 2 (y0 - Y3),
// dt R_3 = y0 - Y4) and R_4 = gather(rel)/Ml (+ the source term): the forward's updated state at
// nodes the routines do not modify
__global__ void __launch_bounds__(256) k_final_pre(int64_t N, const int32_t* __restrict__ ptr,
                                                   const int32_t* __restrict__ idx, const double* __restrict__ el,
                                                   const double* __restrict__ Ml, const double* __restrict__ dt,
                                                   Cols5 y, const double* __restrict__ Y2,
                                                   const double* __restrict__ Y3, const double* __restrict__ Y4,
                                                   const double* __restrict__ src, const double* __restrict__ wmc,
                                                   double* __restrict__ zf) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double r[5] = {0, 0, 0, 0, 0};
  const int beg = ptr[n], end = ptr[n + 1];
  for (int c = beg; c < end; ++c) {
    double v[6];
    load_res6<double>(el, (size_t)idx[c], v);
#pragma unroll
    for (int f = 0; f < 5; ++f) r[f] += v[f];
  }
  const double ml = Ml[n];
  if (src) {
#pragma unroll
    for (int d = 0; d < 3; ++d) r[1 + d] -= ml * src[d * N + n];
  }
  if (wmc) {
#pragma unroll
    for (int d = 0; d < 3; ++d) r[1 + d] += wmc[d * N + n];
  }
  const double h = (*dt) / 6.0;
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const double y0 = y.c[f][n];
    const double acc = (y0 - Y2[f * N + n]) / 3.0 + 2.0 * (y0 - Y3[f * N + n]) / 3.0 + (y0 - Y4[f * N + n]) / 3.0;
    zf[f * N + n] = y0 - acc - h * (r[f] / ml);
  }
}

static int launch_vjp(SodMesh* m, const double* rho, const double* q0, const double* q1, const double* q2,
                      const double* E, const double* mu_factor, const double* musgs, const double* w, cudaStream_t st) {
  VjpArgs a;
  a.nelem = m->nelem;
  a.econn = m->econn;
  a.geo = m->geo64;
  a.mue = m->mue_int;
  a.musgs = musgs;
  a.rho = rho; a.q0 = q0; a.q1 = q1; a.q2 = q2; a.E = E;
  a.mu_factor = mu_factor;
  a.w = w;
  a.npoin = m->npoin;
  a.out = reinterpret_cast<double*>(m->buf.rel);
  a.D = m->D;
  a.prm = m->prm;
  if (m->prm.total_enthalpy)
    k_rhs_vjp<true><<<m->nelem, NN, 0, st>>>(a);
  else
    k_rhs_vjp<false><<<m->nelem, NN, 0, st>>>(a);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

static int ensure_adj(SodMesh* m, size_t len) {
  if (m->adj_len >= len) return SOD_OK;
  if (m->adj) cudaFree(m->adj);
  m->adj = nullptr;
  m->adj_len = 0;
  SOD_CUDA(cudaMalloc(&m->adj, len * sizeof(double)));
  m->adj_len = len;
  return SOD_OK;
}

static inline unsigned nblk(int64_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace adj
}  // namespace sod

using namespace sod;
using namespace sod::adj;

extern "C" {

int sod_rhs_vjp(SodMesh* m, const double* rho, const double* q, const double* E, const double* mu_e,
                const double* mu_factor, const double* bar_Rmass, const double* bar_Rmom, const double* bar_Rener,
                double* grad_rho, double* grad_q, double* grad_E, sod_stream_t stream) {
  SOD_ARG(m && rho && q && E && mu_e && mu_factor, "inputs null");
  SOD_ARG(bar_Rmass && bar_Rmom && bar_Rener && grad_rho && grad_q && grad_E, "adjoint arrays null");
  if (m->has_slaves) {
    set_error("sod_rhs_vjp on a mesh with periodic slave rows (lpoin_w) is not supported");
    return SOD_ERR_UNSUPPORTED;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  const int64_t N = m->npoin;
  rc = ensure_adj(m, 5 * (size_t)N);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, mu_e, m->mue_int, st);
  if (rc) return rc;
  double* w = m->adj;
  Cols5 src{{bar_Rmass, bar_Rmom, bar_Rmom + N, bar_Rmom + 2 * N, bar_Rener}};
  MCols5 none{{nullptr, nullptr, nullptr, nullptr, nullptr}};
  k_seed<<<nblk(N), 256, 0, st>>>(N, src, m->Ml, nullptr, 1.0, w, none);
  SOD_CHECK_LAUNCH();
  rc = launch_vjp(m, rho, q, q + N, q + 2 * N, E, mu_factor, nullptr, w, st);
  if (rc) return rc;
  const double* wmb = nullptr;
  if (m->wmodel.nw > 0) {
    rc = wall_model_vjp(m, rho, q, E, mu_factor, w, st);
    if (rc) return rc;
    wmb = m->wmodel.wmbar;
  }
  MCols5 out{{grad_rho, grad_q, grad_q + N, grad_q + 2 * N, grad_E}};
  k_gather_vjp<<<nblk(N), 256, 0, st>>>(N, m->n2e_ptr, m->n2e, reinterpret_cast<const double*>(m->buf.rel), out, 0,
                                         nullptr, nullptr, nullptr, 0.0, 0.0, nullptr, wmb);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int sod_rk4_step_vjp(SodMesh* m, const double* rho, const double* q, const double* E, const double* mu_e,
                     const double* mu_sgs, const double* mu_factor, const double* dt_dev, const double* stages,
                     const double* bar_rho, const double* bar_q, const double* bar_E, double* out_rho, double* out_q,
                     double* out_E, sod_stream_t stream) {
  SOD_ARG(m && rho && q && E && mu_e && mu_factor && dt_dev, "inputs null");
  SOD_ARG(bar_rho && bar_q && bar_E && out_rho && out_q && out_E, "adjoint arrays null");
  if (m->has_slaves) {
    set_error("sod_rk4_step_vjp on a mesh with periodic slave rows (lpoin_w) is not supported");
    return SOD_ERR_UNSUPPORTED;
  }
  // boundaries and buffer zone: the routines' adjoints after every stage VJP and on the seed
  const bool has_bc = m->bc.nb > 0, has_zone = m->zone.nb > 0;
  const bool bc = has_bc || has_zone;
  const bool ff = has_bc && m->bc.nff > 0;
  const bool slip = has_bc && m->bc.has_slip;
  // wall model: its forward term in the stage residuals the adjoint rebuilds, its own adjoint in
  // every stage's gather
  const double* wmc = m->wmodel.nw > 0 ? m->wmodel.contrib : nullptr;
  // far-field nodes with a buffer zone: the final routine's input at the lnbn targets from the
  // stage residuals gathered there (the zone changes the stage states the reconstruction uses)
  const bool ffz = ff && has_zone;
  NvtxRange range("sod rk4 step vjp");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  // LES: the step's frozen mu_sgs in the internal layout (the forward re-derives it per step)
  const double* musgs = nullptr;
  if (m->prm.flag_les == 1 && mu_sgs) {
    SodState tmp{};
    tmp.mu_sgs = const_cast<double*>(mu_sgs);
    rc = les_in(m, &tmp, st);
    if (rc) return rc;
    musgs = m->musgs_int;
  }
  const int64_t N = m->npoin;
  // Y = B(Z(y)) for the buffer zone Z and the boundary routine B; adjoint Z^T B^T
  auto pre_stage = [&](double* ys, int stage_of) -> int {
    if (has_zone)
      if (int r = zone_stage(m, ys, st)) return r;
    return has_bc ? bc_stage(m, ys, stage_of, st) : SOD_OK;
  };
  // y: the state the boundary routine read (its far-field nodes' lnbn rows); app: which of the
  // step's five applications (stages 1-4, the update) for the slip walls
  auto pre_adjoint = [&](double* vbar, const double* y, int app) -> int {
    if (has_bc)
      if (int r = bc_adjoint(m, vbar, y, app, st)) return r;
    return has_zone ? zone_adjoint(m, vbar, st) : SOD_OK;
  };
  // scratch: ybar copy | w | (with boundaries: Y1 | Ybar of a stage) | (far-field: the updated
  // state before the routine) | (ys2 ys3 ys4 when the stages are not given)   (5 columns each)
  const size_t base = bc ? (ff ? 25 : 20) : 10;
  rc = ensure_adj(m, (base + (stages ? 0 : 15)) * (size_t)N);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, mu_e, m->mue_int, st);
  if (rc) return rc;
  double* yb = m->adj;
  double* w = m->adj + 5 * N;
  double* y1s = bc ? m->adj + 10 * N : nullptr;   // first stage state B(y0)
  double* Ybs = bc ? m->adj + 15 * N : nullptr;   // adjoint of one stage state
  double* zf = ff ? m->adj + 20 * N : nullptr;     // y0 - dt sum b_s R_s, before the final routine
  const double* ys[3];
  const double* rel = reinterpret_cast<const double*>(m->buf.rel);
  Cols5 y0{{rho, q, q + N, q + 2 * N, E}};
  Cols5 Y1 = y0;
  if (bc) {
    for (int f = 0; f < 5; ++f)
      SOD_CUDA(cudaMemcpyAsync(y1s + f * N, y0.c[f], N * sizeof(double), cudaMemcpyDeviceToDevice, st));
    rc = pre_stage(y1s, 1);
    if (rc) return rc;
    Y1 = Cols5{{y1s, y1s + N, y1s + 2 * N, y1s + 3 * N, y1s + 4 * N}};
  }
  if (stages) {
    for (int t = 0; t < 3; ++t) ys[t] = stages + (size_t)t * 5 * N;
  } else {
    // forward recompute of the stage states (mu_e and dt frozen)
    const int epb = m->tuned_epb[0] ? m->tuned_epb[0] : 2;
    const double acoef[3] = {0.5, 0.5, 1.0};
    Cols5 cur = Y1;
    for (int t = 0; t < 3; ++t) {
      double* b = m->adj + (base + 5 * t) * N;
      if (wmc) {
        rc = wall_model_stage(m, cur.c[0], cur.c[1], cur.c[4], mu_factor, st);
        if (rc) return rc;
      }
      rc = launch_rhs(m, false, epb, cur.c[0], cur.c[1], cur.c[2], cur.c[3], cur.c[4], mu_factor, musgs, st);
      if (rc) return rc;
      if (slip) {
        rc = bc_slip_residuals(m, t + 1, rel, st);
        if (rc) return rc;
      }
      if (ffz) {
        rc = bc_ff_residuals(m, t + 1, rel, st);
        if (rc) return rc;
      }
      k_stage_state<<<nblk(N), 256, 0, st>>>(N, m->n2e_ptr, m->n2e, rel, m->Ml, dt_dev, acoef[t], y0, m->source, wmc,
                                             b);
      SOD_CHECK_LAUNCH();
      if (bc) {
        rc = pre_stage(b, t + 2);
        if (rc) return rc;
      }
      ys[t] = b;
      cur = Cols5{{b, b + N, b + 2 * N, b + 3 * N, b + 4 * N}};
    }
  }
  if (ff || slip) {
    const int epb = m->tuned_epb[0] ? m->tuned_epb[0] : 2;
    if ((slip || ffz) && stages) {
      // the stage residuals at the slip nodes / lnbn targets (the recompute gathered them already)
      for (int t = 0; t < 3; ++t) {
        const double* yt = t == 0 ? y1s : ys[t - 1];
        if (wmc) {
          rc = wall_model_stage(m, yt, yt + N, yt + 4 * N, mu_factor, st);
          if (rc) return rc;
        }
        rc = launch_rhs(m, false, epb, yt, yt + N, yt + 2 * N, yt + 3 * N, yt + 4 * N, mu_factor, musgs, st);
        if (rc) return rc;
        if (slip) {
          rc = bc_slip_residuals(m, t + 1, rel, st);
          if (rc) return rc;
        }
        if (ffz) {
          rc = bc_ff_residuals(m, t + 1, rel, st);
          if (rc) return rc;
        }
      }
    }
    // the updated state the final routine reads, at the far-field nodes' lnbn nodes (interior:
    // there the stage states equal their pre-routine values, so dt R_s = (y0 - Y_{s+1}) / a_{s+1}
    // for s = 1..3); R_4 from one more RHS evaluation at Y4
    const double* y4 = ys[2];
    if (wmc) {
      rc = wall_model_stage(m, y4, y4 + N, y4 + 4 * N, mu_factor, st);
      if (rc) return rc;
    }
    rc = launch_rhs(m, false, epb, y4, y4 + N, y4 + 2 * N, y4 + 3 * N, y4 + 4 * N, mu_factor, musgs, st);
    if (rc) return rc;
    if (ffz) {
      rc = bc_ff_residuals(m, 4, rel, st);
      if (rc) return rc;
      rc = bc_ff_final(m, rho, q, E, dt_dev, zf, st);
      if (rc) return rc;
    } else if (ff) {
      k_final_pre<<<nblk(N), 256, 0, st>>>(N, m->n2e_ptr, m->n2e, rel, m->Ml, dt_dev, y0, ys[0], ys[1], ys[2],
                                           m->source, wmc, zf);
      SOD_CHECK_LAUNCH();
    }
    if (slip) {
      // slip walls: pre-routine rho, q of the five applications and the velocities they read
      rc = bc_slip_residuals(m, 4, rel, st);
      if (rc) return rc;
      rc = bc_slip_prepare(m, rho, q, y1s, ys[0], ys[1], dt_dev, st);
      if (rc) return rc;
    }
  }
  // reverse sweep: kbar4 = -dt/6 ybar, Ybar4 = J4^T kbar4, kbar3 = -dt (ybar/3 + Ybar4), ...
  // (with boundaries ybar is first mapped through the final routine's adjoint)
  Cols5 src{{bar_rho, bar_q, bar_q + N, bar_q + 2 * N, bar_E}};
  MCols5 keep{{yb, yb + N, yb + 2 * N, yb + 3 * N, yb + 4 * N}};
  if (bc) {
    for (int f = 0; f < 5; ++f)
      SOD_CUDA(cudaMemcpyAsync(keep.c[f], src.c[f], N * sizeof(double), cudaMemcpyDeviceToDevice, st));
    rc = pre_adjoint(yb, zf, 4);
    if (rc) return rc;
    src = Cols5{{yb, yb + N, yb + 2 * N, yb + 3 * N, yb + 4 * N}};
    keep = MCols5{{nullptr, nullptr, nullptr, nullptr, nullptr}};
  }
  k_seed<<<nblk(N), 256, 0, st>>>(N, src, m->Ml, dt_dev, 1.0 / 6.0, w, keep);
  SOD_CHECK_LAUNCH();
  keep = MCols5{{yb, yb + N, yb + 2 * N, yb + 3 * N, yb + 4 * N}};
  MCols5 acc{{out_rho, out_q, out_q + N, out_q + 2 * N, out_E}};
  // acc = ybar (copied from the kept columns, so out may alias bar)
  for (int f = 0; f < 5; ++f)
    SOD_CUDA(cudaMemcpyAsync(acc.c[f], keep.c[f], N * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (slip) {
    // the update's slip walls read the velocity q/rho of y0 itself
    rc = bc_slip_push(m, rho, q, out_rho, out_q, st);
    if (rc) return rc;
  }
  const double cb[4] = {1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0, 0.0};
  const double ca[4] = {1.0, 0.5, 0.5, 0.0};
  for (int stage = 4; stage >= 1; --stage) {
    const Cols5 ysrc = stage == 1 ? Y1
                                  : Cols5{{ys[stage - 2], ys[stage - 2] + N, ys[stage - 2] + 2 * N,
                                           ys[stage - 2] + 3 * N, ys[stage - 2] + 4 * N}};
    rc = launch_vjp(m, ysrc.c[0], ysrc.c[1], ysrc.c[2], ysrc.c[3], ysrc.c[4], mu_factor, musgs, w, st);
    if (rc) return rc;
    const double* wmb = nullptr;
    if (wmc) {
      rc = wall_model_vjp(m, ysrc.c[0], ysrc.c[1], ysrc.c[4], mu_factor, w, st);
      if (rc) return rc;
      wmb = m->wmodel.wmbar;
    }
    const int t = 4 - stage;
    if (!bc) {
      k_gather_vjp<<<nblk(N), 256, 0, st>>>(N, m->n2e_ptr, m->n2e, rel, acc, 1, yb, m->Ml, dt_dev, cb[t], ca[t],
                                             stage > 1 ? w : nullptr, wmb);
      SOD_CHECK_LAUNCH();
    } else {
      // Ybar of the post-routine stage state, through the stage routine's adjoint, then accumulated
      MCols5 yc{{Ybs, Ybs + N, Ybs + 2 * N, Ybs + 3 * N, Ybs + 4 * N}};
      k_gather_vjp<<<nblk(N), 256, 0, st>>>(N, m->n2e_ptr, m->n2e, rel, yc, 0, nullptr, nullptr, nullptr, 0.0, 0.0,
                                             nullptr, wmb);
      SOD_CHECK_LAUNCH();
      const double* Ysv = stage == 1 ? y1s : ys[stage - 2];
      if (slip && stage < 4) {
        // stage s + 1's slip walls read the velocity of this stage's post-routine state
        rc = bc_slip_push(m, Ysv, Ysv + N, Ybs, Ybs + N, st);
        if (rc) return rc;
      }
      rc = pre_adjoint(Ybs, Ysv, stage - 1);
      if (rc) return rc;
      k_accum_seed<<<nblk(N), 256, 0, st>>>(N, Ybs, acc, yb, m->Ml, dt_dev, cb[t], ca[t], stage > 1 ? w : nullptr);
      SOD_CHECK_LAUNCH();
    }
  }
  return SOD_OK;
}

int sod_bc_dirichlet_prim_vjp(SodMesh* m, const double* rho, const double* q, const double* E, double* bar_rho,
                              double* bar_q, double* bar_E, sod_stream_t stream) {
  SOD_ARG(m && bar_rho && bar_q && bar_E, "null argument");
  SOD_ARG(m->bc.nb > 0, "no boundary nodes registered (sod_mesh_set_boundaries)");
  if (m->has_slaves) {
    set_error("sod_bc_dirichlet_prim_vjp on a mesh with periodic slave rows (lpoin_w) is not supported");
    return SOD_ERR_UNSUPPORTED;
  }
  SOD_ARG(m->bc.nff == 0 || (rho && q && E), "far-field adjoint needs the state the routine read");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t N = m->npoin;
  int rc = ensure_adj(m, 10 * N);
  if (rc) return rc;
  double* v = m->adj;
  double* y = m->adj + 5 * N;
  const double* bars[3] = {bar_rho, bar_q, bar_E};
  const size_t cnt[3] = {N, 3 * N, N}, off[3] = {0, N, 4 * N};
  for (int t = 0; t < 3; ++t) {
    SOD_CUDA(cudaMemcpyAsync(v + off[t], bars[t], cnt[t] * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (m->bc.nff > 0) {
      const double* ys[3] = {rho, q, E};
      SOD_CUDA(cudaMemcpyAsync(y + off[t], ys[t], cnt[t] * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
  }
  rc = bc_adjoint(m, v, m->bc.nff > 0 ? y : nullptr, -1, st);
  if (rc) return rc;
  double* outs[3] = {bar_rho, bar_q, bar_E};
  for (int t = 0; t < 3; ++t)
    SOD_CUDA(cudaMemcpyAsync(outs[t], v + off[t], cnt[t] * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return SOD_OK;
}

}  // extern "C"
