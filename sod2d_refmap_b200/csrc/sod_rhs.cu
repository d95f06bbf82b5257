// Fused element RHS (KR), deterministic node gather fused with the lumped-mass solve and the
// RK4 stage update (KG), entropy viscosity + CFL dt (KV), and the RK4 step driver (sm_100a).
//
// KR restates, for one CTA-resident tile of EPB elements, the element loops of
//   full_convec_ijk            elem_convec.f90:211-460   (skew-symmetric split convection)
//   full_diffusion_ijk         elem_diffu.f90:12-198     (viscous + heat + artificial mass)
//   generic_scalar_convec_ijk  elem_convec.f90:462-570   (entropy residual)
//   sutherland_viscosity       mod_fluid_viscosity.f90:21-41
//   the stage EOS of rk_4_main time_integ.f90:266-285
// One thread owns one gauss point (= element node, GLL collocation).  Nodal fields are staged
// in shared memory in batches; 1-D derivatives are 4-term line sums with the thread's three
// rows of D held in registers; the weak divergence of the diffusive fluxes is applied as D^T
// to contravariant fluxes precomputed at each gauss point.  Element residuals are written to
// an element-major array and assembled by KG as an ordered CSR gather (no atomics).
//
// This is the FP64 parity path: the reference's formulas in FP64 (R = double).  The mixed
// path (FP32 element arithmetic on deviation fields) is k_rhs_mixed2 in sod_rhs_mixed.cu.
#include "sod_internal.cuh"
#include <cmath>
#include <algorithm>

namespace sod {

template <typename R>
__device__ __forceinline__ void giso(const R* __restrict__ f, int i, int j, int k, const R* Dx, const R* Dy,
                                     const R* Dz, R& gx, R& gy, R& gz) {
  const R* fx = f + 4 * j + PLANE * k;
  const R* fy = f + i + PLANE * k;
  const R* fz = f + i + 4 * j;
  gx = Dx[0] * fx[0] + Dx[1] * fx[1] + Dx[2] * fx[2] + Dx[3] * fx[3];
  gy = Dy[0] * fy[0] + Dy[1] * fy[4] + Dy[2] * fy[8] + Dy[3] * fy[12];
  gz = Dz[0] * fz[0] + Dz[1] * fz[PLANE] + Dz[2] * fz[2 * PLANE] + Dz[3] * fz[3 * PLANE];
}

// physical gradient: g_r = sum_c He(r,c) gI_c
template <typename R>
__device__ __forceinline__ void phys(const R* H, R gx, R gy, R gz, R& o0, R& o1, R& o2) {
  o0 = H[0] * gx + H[1] * gy + H[2] * gz;
  o1 = H[3] * gx + H[4] * gy + H[5] * gz;
  o2 = H[6] * gx + H[7] * gy + H[8] * gz;
}

// divergence of a vector field stored as 3 consecutive smem fields
template <typename R>
__device__ __forceinline__ R divv(const R* f, int i, int j, int k, const R* Dx, const R* Dy, const R* Dz,
                                  const R* H) {
  R s = R(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    R gx, gy, gz;
    giso(f + c * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    s += H[3 * c + 0] * gx + H[3 * c + 1] * gy + H[3 * c + 2] * gz;
  }
  return s;
}

// weak divergence sum_dir sum_m D[m][idx_dir] V_dir(line point m)
template <typename R>
__device__ __forceinline__ R divT(const R* fx, const R* fy, const R* fz, int i, int j, int k, const R* DTx,
                                  const R* DTy, const R* DTz) {
  const R* ax = fx + 4 * j + PLANE * k;
  const R* ay = fy + i + PLANE * k;
  const R* az = fz + i + 4 * j;
  return DTx[0] * ax[0] + DTx[1] * ax[1] + DTx[2] * ax[2] + DTx[3] * ax[3] +
         (DTy[0] * ay[0] + DTy[1] * ay[4] + DTy[2] * ay[8] + DTy[3] * ay[12]) +
         (DTz[0] * az[0] + DTz[1] * az[PLANE] + DTz[2] * az[2 * PLANE] + DTz[3] * az[3 * PLANE]);
}

constexpr int NBUF = 15;  // fields per batch buffer
constexpr int NP2 = 18;   // 6 contravariant fluxes x 3 directions

template <typename R>
constexpr size_t rhs_smem_bytes(int epb) {
  return sizeof(R) * (size_t)epb * (NBUF + NP2) * FSTRIDE;
}

// TOTH: flag_total_enthalpy (energy convection of full_convec_ijk_H)
template <typename R, int EPB, bool TOTH>
__global__ void __launch_bounds__(64 * EPB) k_rhs_fused(const RhsArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* buf_all = reinterpret_cast<R*>(smem_raw);
  const int tid = threadIdx.x;
  const int es = tid >> 6;
  const int d = tid & 63;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4;
  const int e = blockIdx.x * EPB + es;
  const bool active = e < a.nelem;
  const int ee = active ? e : a.nelem - 1;
  R* buf = buf_all + (size_t)es * (NBUF + NP2) * FSTRIDE;
  R* p2 = buf + NBUF * FSTRIDE;
  const int s_me = sidx(i, j, k);
  const R* geo = reinterpret_cast<const R*>(a.geo) + (size_t)ee * NGEO * NN;

  // derivative rows (forward: D[i][m]; transposed: D[m][i])
  R Dx[4], Dy[4], Dz[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    Dx[m] = (R)a.D.d[i][m];
    Dy[m] = (R)a.D.d[j][m];
    Dz[m] = (R)a.D.d[k][m];
  }
  R H[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) H[c] = geo[c * NN + d];
  const R gpv = geo[9 * NN + d];

  // ---- own node: stage EOS (time_integ.f90:266-285) and Sutherland (mod_fluid_viscosity.f90:37)
  const int32_t n = a.econn[(size_t)ee * NN + d];
  const double g = a.prm.gamma;
  const double rho = a.rho[n];
  const double qv[3] = {a.q0[n], a.q1[n], a.q2[n]};
  const double Et = a.E[n];
  // one reciprocal serves the divisions by rho; gamma/(gamma-1) and 1/Rgas come from the host
  const double irho = 1.0 / rho;
  const double uv[3] = {qv[0] * irho, qv[1] * irho, qv[2] * irho};
  const double umag = uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2];
  const double kk = 0.5 * umag;
  const double e_int = Et * irho - 0.5 * umag;
  const double p = rho * (g - 1.0) * e_int;
  const double h = a.prm.g_gm1 * p * irho;
  const double T = p * irho * a.prm.inv_Rgas;
  const double mufac = a.mu_factor[n];
  const R mue = reinterpret_cast<const R*>(a.mue)[(size_t)ee * NN + d];
  const double musgs = a.musgs ? a.musgs[(size_t)ee * NN + d] : 0.0;

  const double eta_full = (rho / (g - 1.0)) * log(p / pow(rho, g));
  const double muf = mufac * kSuthC1 * (T * sqrt(T)) / (T + kSuthS);

  // ---- batch A: primitive and scalar fields
  buf[0 * FSTRIDE + s_me] = (R)rho;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    buf[(1 + c) * FSTRIDE + s_me] = (R)uv[c];
    buf[(4 + c) * FSTRIDE + s_me] = (R)qv[c];
  }
  buf[7 * FSTRIDE + s_me] = (R)p;
  buf[8 * FSTRIDE + s_me] = (R)h;
  buf[9 * FSTRIDE + s_me] = (R)(rho * h);
  buf[10 * FSTRIDE + s_me] = (R)kk;
  buf[11 * FSTRIDE + s_me] = (R)(rho * kk);
  buf[12 * FSTRIDE + s_me] = (R)eta_full;
  buf[13 * FSTRIDE + s_me] = (R)T;
  // flag_total_enthalpy: full_convec_ijk_H differentiates p + E and (E + p) u
  if constexpr (TOTH) buf[14 * FSTRIDE + s_me] = (R)(p + Et);
  __syncthreads();

  R gradRho[3], gradU[3][3], gradQ[3][3], gradP[3], gradH[3], gradRH[3], gradK[3], gradRK[3], gradEta[3], gradT[3];
  R uGradEp = R(0);  // flag_total_enthalpy: sum_c 0.5 u_c d(p + E)/dx_c
  {
    R gx, gy, gz;
    giso(buf + 0 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradRho[0], gradRho[1], gradRho[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      giso(buf + (1 + c) * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
      phys(H, gx, gy, gz, gradU[c][0], gradU[c][1], gradU[c][2]);
      giso(buf + (4 + c) * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
      phys(H, gx, gy, gz, gradQ[c][0], gradQ[c][1], gradQ[c][2]);
    }
    giso(buf + 7 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradP[0], gradP[1], gradP[2]);
    giso(buf + 8 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradH[0], gradH[1], gradH[2]);
    giso(buf + 9 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradRH[0], gradRH[1], gradRH[2]);
    giso(buf + 10 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradK[0], gradK[1], gradK[2]);
    giso(buf + 11 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradRK[0], gradRK[1], gradRK[2]);
    giso(buf + 12 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradEta[0], gradEta[1], gradEta[2]);
    giso(buf + 13 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradT[0], gradT[1], gradT[2]);
    if constexpr (TOTH) {
      R gradEp[3];
      giso(buf + 14 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
      phys(H, gx, gy, gz, gradEp[0], gradEp[1], gradEp[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) uGradEp = uGradEp + R(0.5) * ((R)uv[c] * gradEp[c]);
    }
  }
  const R divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
  const R divQ = gradQ[0][0] + gradQ[1][1] + gradQ[2][2];
  const R rhoR = (R)rho, hR = (R)h, kR = (R)kk, etaR = (R)eta_full;
  const R uR[3] = {(R)uv[0], (R)uv[1], (R)uv[2]};
  const R qR[3] = {(R)qv[0], (R)qv[1], (R)qv[2]};
  const R rhR = (R)(rho * h), rkR = (R)(rho * kk);

  // ---- convective terms available after batch A (elem_convec.f90:412-432)
  R Rm = R(0.5) * (divQ + rhoR * divU);
  R Ren = R(0.25) * (hR * divQ + rhR * divU) + R(0.25) * (kR * divQ + rkR * divU);
  R Rmo[3];
  R Ret = R(0.5) * (etaR * divU);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Rmo[c] = R(0.25) * (uR[c] * divQ + qR[c] * divU) + gradP[c];
    Rm += R(0.5) * (uR[c] * gradRho[c]);
    Ren += R(0.25) * (qR[c] * gradH[c] + uR[c] * gradRH[c] + (hR * uR[c]) * gradRho[c]) +
           R(0.25) * (qR[c] * gradK[c] + uR[c] * gradRK[c] + (kR * uR[c]) * gradRho[c]);
    Ret += R(0.5) * (uR[c] * gradEta[c]);
#pragma unroll
    for (int jd = 0; jd < 3; ++jd)
      Rmo[c] += R(0.25) * ((uR[c] * uR[jd]) * gradRho[jd] + qR[jd] * gradU[c][jd] + uR[jd] * gradQ[c][jd]);
  }

  // ---- diffusion pass 1 (elem_diffu.f90:70-140): stresses and contravariant fluxes
  {
    const R mufgp = (R)(muf + rho * musgs);
    const R mut = mufgp + mue;
    const R twoThirds = R(2.0 / 3.0);
    R tau[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) tau[r][c] = mut * (gradU[r][c] + gradU[c][r]);
#pragma unroll
    for (int r = 0; r < 3; ++r) tau[r][r] = tau[r][r] - mufgp * twoThirds * divU;
    R tauU[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) tauU[r] = tau[r][0] * uR[0] + tau[r][1] * uR[1] + tau[r][2] * uR[2];
    // V-hat_dir = gpvol * sum_r He(r,dir) V_r for V in {gradRho, tauU, gradT, tau row 0,1,2}
    auto emit = [&](int v, R V0, R V1, R V2) {
#pragma unroll
      for (int dir = 0; dir < 3; ++dir)
        p2[(v * 3 + dir) * FSTRIDE + s_me] = gpv * (H[0 + dir] * V0 + H[3 + dir] * V1 + H[6 + dir] * V2);
    };
    emit(0, gradRho[0], gradRho[1], gradRho[2]);
    emit(1, tauU[0], tauU[1], tauU[2]);
    emit(2, gradT[0], gradT[1], gradT[2]);
    emit(3, tau[0][0], tau[0][1], tau[0][2]);
    emit(4, tau[1][0], tau[1][1], tau[1][2]);
    emit(5, tau[2][0], tau[2][1], tau[2][2]);
  }
  __syncthreads();  // batch A reads done

  // ---- batch B: product vectors (rho h u, h u, rho k u, k u, eta u)
  {
    const R sh = (R)h, sk = (R)kk, se = (R)eta_full;
    const R rsh = (R)(rho * h), rsk = (R)(rho * kk);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      buf[(0 + c) * FSTRIDE + s_me] = TOTH ? (R)((Et + p) * uv[c]) : rsh * uR[c];
      buf[(3 + c) * FSTRIDE + s_me] = sh * uR[c];
      buf[(6 + c) * FSTRIDE + s_me] = rsk * uR[c];
      buf[(9 + c) * FSTRIDE + s_me] = sk * uR[c];
      buf[(12 + c) * FSTRIDE + s_me] = se * uR[c];
    }
  }
  __syncthreads();
  {
    const R divFe = divv(buf + 0 * FSTRIDE, i, j, k, Dx, Dy, Dz, H);
    const R divFue = divv(buf + 3 * FSTRIDE, i, j, k, Dx, Dy, Dz, H);
    const R divFk = divv(buf + 6 * FSTRIDE, i, j, k, Dx, Dy, Dz, H);
    const R divFuk = divv(buf + 9 * FSTRIDE, i, j, k, Dx, Dy, Dz, H);
    const R divFeta = divv(buf + 12 * FSTRIDE, i, j, k, Dx, Dy, Dz, H);
    Ren += R(0.25) * (divFe + rhoR * divFue) + R(0.25) * (divFk + rhoR * divFuk);
    Ret += R(0.5) * divFeta;
    if constexpr (TOTH) Ren = R(0.5) * (divFe + (R)(Et + p) * divU) + uGradEp;  // elem_convec.f90:171-177
  }
  __syncthreads();

  // ---- batch C: tensors q x u and u x u (symmetric)
  {
    R sq[3], su[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      sq[c] = (R)qv[c];
      su[c] = (R)uv[c];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) buf[(3 * r + c) * FSTRIDE + s_me] = sq[r] * su[c];
    buf[9 * FSTRIDE + s_me] = su[0] * su[0];
    buf[10 * FSTRIDE + s_me] = su[0] * su[1];
    buf[11 * FSTRIDE + s_me] = su[0] * su[2];
    buf[12 * FSTRIDE + s_me] = su[1] * su[1];
    buf[13 * FSTRIDE + s_me] = su[1] * su[2];
    buf[14 * FSTRIDE + s_me] = su[2] * su[2];
  }
  __syncthreads();
  {
    const int symidx[3][3] = {{9, 10, 11}, {10, 12, 13}, {11, 13, 14}};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      R dF = R(0), dFuu = R(0);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        R gx, gy, gz;
        giso(buf + (3 * r + c) * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
        dF += H[3 * c + 0] * gx + H[3 * c + 1] * gy + H[3 * c + 2] * gz;
        giso(buf + symidx[r][c] * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
        dFuu += H[3 * c + 0] * gx + H[3 * c + 1] * gy + H[3 * c + 2] * gz;
      }
      Rmo[r] += R(0.25) * (dF + rhoR * dFuu);
    }
  }

  // ---- diffusion pass 2 (elem_diffu.f90:142-194): weak divergence with D^T
  R DTx[4], DTy[4], DTz[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    DTx[m] = (R)a.D.d[m][i];
    DTy[m] = (R)a.D.d[m][j];
    DTz[m] = (R)a.D.d[m][k];
  }
  R dv[6];
#pragma unroll
  for (int v = 0; v < 6; ++v)
    dv[v] = divT(p2 + (v * 3 + 0) * FSTRIDE, p2 + (v * 3 + 1) * FSTRIDE, p2 + (v * 3 + 2) * FSTRIDE, i, j, k, DTx,
                 DTy, DTz);
  const R nu_e = (R)a.prm.c_rho * mue * (R)irho;
  const R kappa_e = (R)(muf * a.prm.CpPr) + (R)a.prm.c_ener * mue * (R)a.prm.CpPr + (R)(a.prm.Cp09 * rho * musgs);
  if (active) {
    store_res6<R>(reinterpret_cast<R*>(a.rel), (size_t)e * NN + d, gpv * Rm + nu_e * dv[0], gpv * Rmo[0] + dv[3],
                  gpv * Rmo[1] + dv[4], gpv * Rmo[2] + dv[5], gpv * Ren + (dv[1] + kappa_e * dv[2]), gpv * Ret);
  }
}

// ---------------------------------------------------------------------------------------------
// KG: ordered CSR gather of the element residuals, /Ml, RK accumulate and next stage state.
// STAGE 0 = plain RHS (gather + /Ml into output arrays).  STAGE 4 = final update + EOS.
// ---------------------------------------------------------------------------------------------
struct GatherArgs {
  int npoin;
  int nwork;                      // working nodes (rows with elements): the entropy mean's count
  const int32_t* __restrict__ ptr;
  const int32_t* __restrict__ idx;
  const void* rel;
  const double* __restrict__ Ml;
  const double* __restrict__ dt;  // device scalar, or per-member array when node_member is set
  const int32_t* __restrict__ node_member;
  int member_reduce;              // stage 4: eta sums done by the per-member kernel instead
  double a_next, b_cur;
  // state (level pos=2) columns
  double* y[5];
  double* ys;    // stage state 5*N
  double* rsum;  // 6*N
  // stage-0 outputs
  double* out[6];
  // stage-4 EOS outputs
  double *u0, *u1, *u2, *pr, *Tem, *e_int, *eta, *csound, *machno, *mu_fluid, *Reta;
  const double* mu_factor;
  double gamma, Rgas;
  double* red;              // partials [3*nblocks]
  unsigned int* counter;
  unsigned int* nonfinite;  // raised by stage 4 on a NaN/Inf in the new rho, q, E
  double* scal;             // [0] eta mean, [1] eta norm
  int normalise;
  const double* src;        // momentum source term (npoin,3) or null
  const double* wm;         // wall-model momentum terms (npoin,3) or null
};

__device__ __forceinline__ void block_reduce3(double& s, double& mx, double& mn, double* sh) {
  // warp reduce then smem
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sh[3 * w] = s; sh[3 * w + 1] = mx; sh[3 * w + 2] = mn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    s = sh[0]; mx = sh[1]; mn = sh[2];
    for (int q = 1; q < nw; ++q) { s += sh[3 * q]; mx = fmax(mx, sh[3 * q + 1]); mn = fmin(mn, sh[3 * q + 2]); }
  }
}

#ifndef SOD_KG_MIN_BLOCKS
// resident 256-thread blocks per SM the register budget must allow: 4 leaves 64 registers, no
// spills (7 blocks capped the kernel at 32 registers and spilled 140-244 bytes per thread)
#define SOD_KG_MIN_BLOCKS 4
#endif
template <typename R, int STAGE>
__global__ void __launch_bounds__(256, SOD_KG_MIN_BLOCKS) k_gather_rk(const GatherArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  // a row without elements is a periodic slave (not in lpoin_w): rk_4_main's node loops
  // (time_integ.f90:267-285,445-471) and the lumped solve (mod_solver.f90:23-58) skip it, its
  // residual stays zero and its state untouched; only sutherland_viscosity, which runs over all
  // npoin (time_integ.f90:483-487), re-evaluates its mu_fluid from its own Tem
  const bool inrange = n < a.npoin;
  const bool act = inrange && a.ptr[n + 1] > a.ptr[n];
  if (inrange && !act) {
    if constexpr (STAGE == 0) {
#pragma unroll
      for (int f = 0; f < 6; ++f)
        if (a.out[f]) a.out[f][n] = 0.0;
    } else if constexpr (STAGE == 4) {
      const double T = a.Tem[n];
      a.mu_fluid[n] = a.mu_factor[n] * kSuthC1 * (T * sqrt(T)) / (T + kSuthS);
    }
  }
  double eta_n = 0.0;
  if (act) {
    const R* rel = reinterpret_cast<const R*>(a.rel);
    const size_t N = (size_t)a.npoin;
    // node data independent of the gather, loaded first so their latency overlaps it
    double yv[5], rsv[6];
    if constexpr (STAGE >= 1) {
#pragma unroll
      for (int f = 0; f < 5; ++f) yv[f] = a.y[f][n];
#pragma unroll
      for (int f = 0; f < 6; ++f) rsv[f] = STAGE == 1 ? 0.0 : a.rsum[f * N + n];
    }
    const double ml = a.Ml[n];
    double r[6] = {0, 0, 0, 0, 0, 0};
    const int beg = a.ptr[n], end = a.ptr[n + 1];
    int c = beg;
    // groups of 4 contributions: all loads issued before the (ascending, fixed-order) sums
    for (; c + 4 <= end; c += 4) {
      R v[4][6];
#pragma unroll
      for (int q = 0; q < 4; ++q) load_res6<R>(rel, (size_t)a.idx[c + q], v[q]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int f = 0; f < 6; ++f) r[f] += (double)v[q][f];
    }
    for (; c < end; ++c) {
      R v[6];
      load_res6<R>(rel, (size_t)a.idx[c], v);
#pragma unroll
      for (int f = 0; f < 6; ++f) r[f] += (double)v[f];
    }
    if (a.src) {
      // mom_source_const_vect (elem_source.f90:20-55): - sum_e gpvol s = - Ml s on the momentum
#pragma unroll
      for (int d = 0; d < 3; ++d) r[1 + d] -= ml * a.src[d * N + n];
    }
    if (a.wm) {
      // wall model: the modelled shear added to Rdiff_mom (time_integ.f90:334-357)
#pragma unroll
      for (int d = 0; d < 3; ++d) r[1 + d] += a.wm[d * N + n];
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) r[f] = r[f] / ml;
    if constexpr (STAGE == 0) {
#pragma unroll
      for (int f = 0; f < 6; ++f)
        if (a.out[f]) a.out[f][n] = r[f];
    } else {
      const double dt = a.node_member ? a.dt[a.node_member[n]] : *a.dt;
      double rs[6];
#pragma unroll
      for (int f = 0; f < 6; ++f) rs[f] = rsv[f] + a.b_cur * r[f];
      if constexpr (STAGE < 4) {
#pragma unroll
        for (int f = 0; f < 6; ++f) a.rsum[f * N + n] = rs[f];
        const double da = dt * a.a_next;
#pragma unroll
        for (int f = 0; f < 5; ++f) a.ys[f * N + n] = yv[f] - da * r[f];
      } else {
        // RK update (time_integ.f90:417-426) and EOS at the new level (:445-463)
        double y[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          y[f] = yv[f] - dt * rs[f];
          a.y[f][n] = y[f];
        }
        if (!(isfinite(y[0]) && isfinite(y[1]) && isfinite(y[2]) && isfinite(y[3]) && isfinite(y[4])))
          atomicOr(a.nonfinite, 1u);
        const double g = a.gamma;
        const double rho = y[0];
        const double u0 = y[1] / rho, u1 = y[2] / rho, u2 = y[3] / rho;
        double umag = u0 * u0 + u1 * u1 + u2 * u2;
        const double ei = (y[4] / rho) - 0.5 * umag;
        const double pr = rho * (g - 1.0) * ei;
        const double cs = sqrt(g * pr / rho);
        umag = sqrt(umag);
        const double T = pr / (rho * a.Rgas);
        const double eta = (rho / (g - 1.0)) * log(pr / pow(rho, g));
        a.u0[n] = u0; a.u1[n] = u1; a.u2[n] = u2;
        a.e_int[n] = ei; a.pr[n] = pr; a.csound[n] = cs; a.machno[n] = umag / cs;
        a.Tem[n] = T; a.eta[n] = eta;
        a.mu_fluid[n] = a.mu_factor[n] * kSuthC1 * (T * sqrt(T)) / (T + kSuthS);
        if (a.Reta) a.Reta[n] = -rs[5];
        eta_n = eta;
      }
    }
  }
  if constexpr (STAGE == 4) {
    if (a.member_reduce) return;  // uniform across the grid
    // entropy normalisation (mod_entropy_viscosity.f90:43-66): sum, max, min of eta
    __shared__ double sh[3 * 8];
    __shared__ bool last;
    double s = act ? eta_n : 0.0, mx = act ? eta_n : -1e300, mn = act ? eta_n : 1e300;
    block_reduce3(s, mx, mn, sh);
    if (threadIdx.x == 0) {
      a.red[3 * blockIdx.x] = s;
      a.red[3 * blockIdx.x + 1] = mx;
      a.red[3 * blockIdx.x + 2] = mn;
      __threadfence();
      unsigned int done = atomicAdd(a.counter, 1u);
      last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
      __threadfence();
      // fixed-order final reduction by the last block (deterministic)
      double ts = 0.0, tmx = -1e300, tmn = 1e300;
#pragma unroll 4
      for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        ts += __ldcg(a.red + 3 * b);
        tmx = fmax(tmx, __ldcg(a.red + 3 * b + 1));
        tmn = fmin(tmn, __ldcg(a.red + 3 * b + 2));
      }
      __syncthreads();
      block_reduce3(ts, tmx, tmn, sh);
      if (threadIdx.x == 0) {
        if (a.normalise) {
          const double mean = ts / (double)a.nwork;
          a.scal[0] = mean;
          a.scal[1] = fmax(tmx - mean, mean - tmn);
        } else {
          a.scal[0] = 0.0;
          a.scal[1] = 1.0;
        }
        *a.counter = 0u;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// KV: smart_visc_spectral (mod_entropy_viscosity.f90:68-121) per element with the convertIJK
// filter (mod_filters.f90:42-51), fused with the per-element CFL limits of adapt_dt_cfl
// (mod_time_ops.f90:31-56) and a deterministic min reduction to the next dt.
// ---------------------------------------------------------------------------------------------
struct ViscArgs {
  int nelem;
  const int32_t* __restrict__ econn;
  const double* __restrict__ Reta;
  const double* __restrict__ rho;
  const double* __restrict__ u0;
  const double* __restrict__ u1;
  const double* __restrict__ u2;
  const double* __restrict__ csound;
  const double* __restrict__ Tem;
  const double* __restrict__ mu_fluid;
  const double* __restrict__ musgs;  // [e][64] or null
  const double* __restrict__ helem_l;
  const double* __restrict__ helem;
  const double* __restrict__ jratio;
  const double* __restrict__ scal;   // [0] mean, [1] norm
  double* mue;                       // out FP64 [e][64]
  float* mue32;                      // optional FP32 copy
  double* dt_bits;                   // scratch scalar(s) receiving the min dt (bits, pre-set large)
  const int32_t* __restrict__ elem_member;  // ensemble: member of each element (null = one mesh)
  const double* __restrict__ member_scal;   // ensemble: [member][2] eta mean, norm
  double* dt_out;                    // device scalar (may be null)
  DevParams prm;
};

__device__ __forceinline__ int nb_filter(int x) {
  // natural index of convertIJK(x+1): x=-1 -> 1, 0..3 -> x, 4 -> 1 (reference quirk)
  return (x < 0) ? 1 : ((x > 3) ? 1 : x);
}

constexpr int KV_EPB = 4;

#ifndef SOD_KV_MIN_BLOCKS
#define SOD_KV_MIN_BLOCKS 8  // resident blocks per SM the register budget must allow
#endif
__global__ void __launch_bounds__(64 * KV_EPB, SOD_KV_MIN_BLOCKS) k_visc_dt(const ViscArgs a) {
  __shared__ double ml[KV_EPB][NN];
  __shared__ double fl[KV_EPB][NN];  // filter pass buffer
  __shared__ double wm[KV_EPB][2][5];
  __shared__ double elem_s[KV_EPB][2];  // ced, dt limit of the element
  const int es = threadIdx.x >> 6, d = threadIdx.x & 63;
  const int e = blockIdx.x * KV_EPB + es;
  const bool act = e < a.nelem;
  const int ee = act ? e : a.nelem - 1;
  const int n = a.econn[(size_t)ee * NN + d];
  const double rho = a.rho[n], u0 = a.u0[n], u1 = a.u1[n], u2 = a.u2[n], cs = a.csound[n], T = a.Tem[n];
  // inputs of the second half, loaded before the element reductions so their latency overlaps them
  const double reta_n = a.Reta[n];
  const double hl = a.helem_l[(size_t)ee * NN + d];
  const double vmag = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
  const double he = a.helem[ee];
  // betae node term (mod_entropy_viscosity.f90:90-95)
  const double beta_n = (rho * he) * (a.prm.cmax / (double)P) * (vmag + sqrt(a.prm.Rgas * a.prm.gamma * T));
  // CFL node terms (mod_time_ops.f90:36-50)
  const double umax = fmax(fmax(fabs(u0), fabs(u1)), fabs(u2));
  const double L3n = umax + cs;
  const double musgs = a.musgs ? a.musgs[(size_t)ee * NN + d] : 0.0;
  const double mun = (rho * musgs + a.mu_fluid[n]) / rho;
  // element maxima over the 64 nodes (two warps per element)
  double mV = vmag, mC = cs, mB = beta_n, mL = L3n, mM = mun;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mV = fmax(mV, __shfl_xor_sync(0xffffffffu, mV, o));
    mC = fmax(mC, __shfl_xor_sync(0xffffffffu, mC, o));
    mB = fmax(mB, __shfl_xor_sync(0xffffffffu, mB, o));
    mL = fmax(mL, __shfl_xor_sync(0xffffffffu, mL, o));
    mM = fmax(mM, __shfl_xor_sync(0xffffffffu, mM, o));
  }
  const int wi = d >> 5;
  if ((d & 31) == 0) { wm[es][wi][0] = mV; wm[es][wi][1] = mC; wm[es][wi][2] = mB; wm[es][wi][3] = mL; wm[es][wi][4] = mM; }
  __syncthreads();
  if (d == 0) {
    // shock sensor and cap, once per element (mod_entropy_viscosity.f90:81-84); M**15 as an
    // integer power like the reference
    const double M = fmax(wm[es][0][0], wm[es][1][0]) / fmax(wm[es][0][1], wm[es][1][1]);
    const double M2 = M * M, M4 = M2 * M2, M8 = M4 * M4;
    const double M15 = M8 * M4 * M2 * M;
    const double ceM = fmax(tanh(M15 * 3.141592653589793), a.prm.ce);
    double ced = fmax(1.0 - a.jratio[ee], a.prm.ce);
    elem_s[es][0] = fmax(ced, ceM);
    const double hh = he / (double)(2.0 * P + 1);
    const double L3 = fmax(wm[es][0][3], wm[es][1][3]);
    const double maxMU = fmax(wm[es][0][4], wm[es][1][4]);
    elem_s[es][1] = fmin(a.prm.cfl_conv * hh / L3, a.prm.cfl_diff * (hh * hh) / maxMU);
  }
  __syncthreads();
  const double ced = elem_s[es][0];
  mB = fmax(wm[es][0][2], wm[es][1][2]);
  const int mem = a.elem_member ? a.elem_member[ee] : 0;
  const double norm = a.elem_member ? a.member_scal[2 * mem + 1] : a.scal[1];
  const double R1 = (norm > 0.0) ? rho * fabs(reta_n) / norm : 0.0;
  const double Ve = ced * R1 * hl * hl;
  ml[es][d] = a.prm.cglob * fmin(Ve, mB);
  __syncthreads();
  // 3x3x3 filter with weights (1/4,1/2,1/4) through convertIJK (mod_entropy_viscosity.f90:102-120):
  // the weights and the index map are separable, so it runs as three 3-point passes (xi, eta,
  // zeta) through shared memory, 9 reads per node instead of 27
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4;
  const int ix[3] = {nb_filter(i - 1), i, nb_filter(i + 1)};
  const int jx[3] = {nb_filter(j - 1), j, nb_filter(j + 1)};
  const int kx[3] = {nb_filter(k - 1), k, nb_filter(k + 1)};
  const double w[3] = {0.25, 0.5, 0.25};
  fl[es][d] = w[0] * ml[es][ix[0] + 4 * j + 16 * k] + w[1] * ml[es][d] + w[2] * ml[es][ix[2] + 4 * j + 16 * k];
  __syncthreads();
  // ml's first-pass reads all happened before the barrier above, so it takes the second pass
  ml[es][d] = w[0] * fl[es][i + 4 * jx[0] + 16 * k] + w[1] * fl[es][d] + w[2] * fl[es][i + 4 * jx[2] + 16 * k];
  __syncthreads();
  const double acc = w[0] * ml[es][i + 4 * j + 16 * kx[0]] + w[1] * ml[es][d] + w[2] * ml[es][i + 4 * j + 16 * kx[2]];
  if (act) {
    a.mue[(size_t)e * NN + d] = acc;
    if (a.mue32) a.mue32[(size_t)e * NN + d] = (float)acc;
    // next dt: order-independent min over elements on the bit pattern of a positive double
    if (a.dt_out && d == 0)
      atomicMin(reinterpret_cast<unsigned long long*>(a.dt_bits) + mem,
                (unsigned long long)__double_as_longlong(elem_s[es][1]));
  }
}

// ---------------------------------------------------------------------------------------------
// Host-side launch helpers
// ---------------------------------------------------------------------------------------------
template <typename R, int EPB>
static int set_rhs_attr() {
  SOD_CUDA(cudaFuncSetAttribute(k_rhs_fused<R, EPB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)rhs_smem_bytes<R>(EPB)));
  SOD_CUDA(cudaFuncSetAttribute(k_rhs_fused<R, EPB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)rhs_smem_bytes<R>(EPB)));
  return SOD_OK;
}

int init_kernel_attrs() {
  static bool done = false;
  if (done) return SOD_OK;
  int rc = set_rhs_attr<double, 1>() | set_rhs_attr<double, 2>() | set_rhs_attr<double, 4>() |
           init_rhs_mixed2_attrs();
  if (rc) return SOD_ERR_CUDA;
  done = true;
  return SOD_OK;
}

template <typename R, int EPB>
static int launch_rhs_t(const RhsArgs& a, cudaStream_t st) {
  const size_t smem = rhs_smem_bytes<R>(EPB);
  const int grid = (a.nelem + EPB - 1) / EPB;
  if (a.prm.total_enthalpy)
    k_rhs_fused<R, EPB, true><<<grid, 64 * EPB, smem, st>>>(a);
  else
    k_rhs_fused<R, EPB, false><<<grid, 64 * EPB, smem, st>>>(a);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int launch_rhs(SodMesh* m, bool mixed, int epb, const double* rho, const double* q0, const double* q1,
               const double* q2, const double* E, const double* mu_factor, const double* musgs_int,
               cudaStream_t st) {
  RhsArgs a;
  a.nelem = m->nelem;
  a.econn = m->econn;
  a.geo = mixed ? (const void*)m->geo32 : (const void*)m->geo64;
  a.mue = mixed ? (const void*)m->mue32 : (const void*)m->mue_int;
  a.musgs = musgs_int;
  a.rho = rho; a.q0 = q0; a.q1 = q1; a.q2 = q2; a.E = E;
  a.mu_factor = mu_factor;
  a.rel = m->buf.rel;
  a.D = m->D;
  for (int r = 0; r < NP1; ++r)
    for (int c = 0; c < NP1; ++c) a.Df[r][c] = (float)m->D.d[r][c];
  a.prm = m->prm;
  if (!mixed) {
    switch (epb) {
      case 1: return launch_rhs_t<double, 1>(a, st);
      case 4: return launch_rhs_t<double, 4>(a, st);
      default: return launch_rhs_t<double, 2>(a, st);
    }
  } else {
    return launch_rhs_mixed2(a, epb, st);
  }
}

static const double kA[4] = {0.0, 0.5, 0.5, 1.0};
static const double kB[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};

template <typename R>
static int launch_gather_t(int stage, const GatherArgs& a, cudaStream_t st) {
  const int grid = (a.npoin + 255) / 256;
  switch (stage) {
    case 0: k_gather_rk<R, 0><<<grid, 256, 0, st>>>(a); break;
    case 1: k_gather_rk<R, 1><<<grid, 256, 0, st>>>(a); break;
    case 2: k_gather_rk<R, 2><<<grid, 256, 0, st>>>(a); break;
    case 3: k_gather_rk<R, 3><<<grid, 256, 0, st>>>(a); break;
    default: k_gather_rk<R, 4><<<grid, 256, 0, st>>>(a); break;
  }
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int launch_gather(SodMesh* m, bool mixed, int stage, GatherArgs& a, cudaStream_t st) {
  a.npoin = m->npoin;
  a.nwork = m->npoin_w;
  a.ptr = m->n2e_ptr;
  a.idx = m->n2e;
  a.rel = m->buf.rel;
  a.Ml = m->Ml;
  a.gamma = m->prm.gamma;
  a.Rgas = m->prm.Rgas;
  a.normalise = m->prm.normalise;
  if (!a.ys) a.ys = m->buf.ys;
  a.rsum = m->buf.rsum;
  a.red = m->buf.red;
  a.counter = m->buf.counters + 0;
  a.nonfinite = m->buf.counters + kNonfiniteCounter;
  a.scal = m->buf.scal;
  a.src = m->nmember > 0 ? nullptr : m->source;
  a.wm = (m->nmember > 0 || m->wmodel.nw == 0) ? nullptr : m->wmodel.contrib;
  if (stage >= 1) {
    a.b_cur = kB[stage - 1];
    a.a_next = stage < 4 ? kA[stage] : 0.0;
  }
  return mixed ? launch_gather_t<float>(stage, a, st) : launch_gather_t<double>(stage, a, st);
}

// LES is on for a step when the parameters ask for it and the state carries mu_sgs
static bool les_active(const SodMesh* m, const SodState* s) {
  return m->prm.flag_les == 1 && s->mu_sgs != nullptr && m->musgs_int != nullptr;
}

// mu_sgs (nelem,64) in the reference layout -> internal layout before a step (allocates once)
int les_in(SodMesh* m, const SodState* s, cudaStream_t st) {
  if (!(m->prm.flag_les == 1 && s->mu_sgs)) return SOD_OK;
  if (!m->musgs_int) SOD_CUDA(cudaMalloc(&m->musgs_int, sizeof(double) * (size_t)m->nelem * NN));
  return mesh_ref_to_internal_elem(m, s->mu_sgs, m->musgs_int, st);
}

int les_out(SodMesh* m, const SodState* s, cudaStream_t st) {
  if (!les_active(m, s)) return SOD_OK;
  return mesh_internal_to_ref_elem(m, m->musgs_int, s->mu_sgs, st);
}

int launch_visc_dt(SodMesh* m, const SodState* s, double* dt_out, float* mue32, cudaStream_t st) {
  ViscArgs v;
  v.nelem = m->nelem;
  v.econn = m->econn;
  v.Reta = s->Reta;
  v.rho = s->rho;
  v.u0 = s->u;
  v.u1 = s->u + m->npoin;
  v.u2 = s->u + 2 * (size_t)m->npoin;
  v.csound = s->csound;
  v.Tem = s->Tem;
  v.mu_fluid = s->mu_fluid;
  v.musgs = les_active(m, s) ? m->musgs_int : nullptr;
  v.helem_l = m->helem_l;
  v.helem = m->helem;
  v.jratio = m->jratio;
  v.scal = m->buf.scal;
  v.mue = m->mue_int;
  v.mue32 = mue32;
  const int nm = m->nmember > 0 ? m->nmember : 1;
  v.dt_bits = m->nmember > 0 ? m->member_dt_bits : m->buf.scal + 3;
  v.elem_member = m->nmember > 0 ? m->elem_member : nullptr;
  v.member_scal = m->member_scal;
  v.dt_out = dt_out;
  v.prm = m->prm;
  if (dt_out) SOD_CUDA(cudaMemsetAsync(v.dt_bits, 0x7F, sizeof(double) * nm, st));  // 1.38e306 each
  const int grid = (m->nelem + KV_EPB - 1) / KV_EPB;
  k_visc_dt<<<grid, 64 * KV_EPB, 0, st>>>(v);
  SOD_CHECK_LAUNCH();
  if (dt_out) SOD_CUDA(cudaMemcpyAsync(dt_out, v.dt_bits, sizeof(double) * nm, cudaMemcpyDeviceToDevice, st));
  return SOD_OK;
}

// Ensemble: per-member eta sum/max/min over its contiguous node range, one block per member.
__global__ void __launch_bounds__(512) k_member_eta(const int32_t* __restrict__ off, const double* __restrict__ eta,
                                                    double* scal, int normalise) {
  const int mbr = blockIdx.x;
  const int b = off[mbr], e = off[mbr + 1];
  double s = 0.0, mx = -1e300, mn = 1e300;
  for (int t = b + threadIdx.x; t < e; t += blockDim.x) {
    const double v = eta[t];
    s += v; mx = fmax(mx, v); mn = fmin(mn, v);
  }
  __shared__ double sh[3 * 16];
  block_reduce3(s, mx, mn, sh);
  if (threadIdx.x == 0) {
    if (normalise) {
      const double mean = s / (double)(e - b);
      scal[2 * mbr] = mean;
      scal[2 * mbr + 1] = fmax(mx - mean, mean - mn);
    } else {
      scal[2 * mbr] = 0.0;
      scal[2 * mbr + 1] = 1.0;
    }
  }
}

// Reta scratch when the caller passes none
static double* reta_scratch(SodMesh* m) {
  return m->buf.rsum + 5 * (size_t)m->npoin;  // rsum eta column is dead after stage 4 reads it
}

// One RK4 step on device state (mu_e already in m->mue_int / mue32).  When ev is non-null,
// ev[2*slot] / ev[2*slot+1] bracket each kernel: slots 0-3 KR stages, 4-7 KG stages, 8 KV.
// When stage_store is non-null the stage states Y2, Y3, Y4 (5 columns of npoin each) are
// written there instead of the internal stage buffer (for the adjoint's reverse sweep).
int run_step(SodMesh* m, SodState* s, const double* dt_dev, double* dt_next, bool mixed, cudaStream_t st,
             cudaEvent_t* ev = nullptr, double* stage_store = nullptr) {
  NvtxRange range(mixed ? "sod rk4 step (mixed)" : "sod rk4 step (fp64)");
  const size_t N = m->npoin;
  const int epb = m->tuned_epb[mixed ? 1 : 0] ? m->tuned_epb[mixed ? 1 : 0] : (mixed ? 4 : 2);
  SodState loc = *s;
  const bool les = les_active(m, s);
  double* reta_tmp = nullptr;
  if (!loc.Reta) {
    // stage 4 reads rsum[5] before writing Reta, element-wise, so aliasing is safe
    reta_tmp = reta_scratch(m);
    loc.Reta = reta_tmp;
  }
  int rc;
  // non-periodic path / buffer zone: updateBuffer, then the boundary routine, on every stage
  // state and on the updated state
  const bool bc = m->bc.nb > 0;
  const bool zone = m->zone.nb > 0;
  const bool pre = bc || zone;
  auto pre_stage = [&](double* ys, int stage_of) -> int {
    if (zone)
      if (int r = zone_stage(m, ys, st)) return r;
    return bc ? bc_stage(m, ys, stage_of, st) : SOD_OK;
  };
  if (bc) {
    rc = bc_snapshot_u(m, s->u, st);  // u(:,:,pos) before the update, read by slip walls
    if (rc) return rc;
  }
  for (int stage = 1; stage <= 4; ++stage) {
    double* yin = (stage_store && stage >= 2) ? stage_store + (size_t)(stage - 2) * 5 * N : m->buf.ys;
    if (pre && stage == 1) {
      // the first stage state is the state itself with the routines applied to a copy
      SOD_CUDA(cudaMemcpyAsync(yin, s->rho, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
      SOD_CUDA(cudaMemcpyAsync(yin + N, s->q, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, st));
      SOD_CUDA(cudaMemcpyAsync(yin + 4 * N, s->E, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
      rc = pre_stage(yin, 1);
      if (rc) return rc;
    }
    const bool from_state = stage == 1 && !pre;
    const double* src_rho = from_state ? s->rho : yin;
    const double* src_q0 = from_state ? s->q : yin + N;
    const double* src_q1 = from_state ? s->q + N : yin + 2 * N;
    const double* src_q2 = from_state ? s->q + 2 * N : yin + 3 * N;
    const double* src_E = from_state ? s->E : yin + 4 * N;
    if (m->wmodel.nw > 0) {
      rc = wall_model_stage(m, src_rho, src_q0, src_E, s->mu_factor, st);
      if (rc) return rc;
    }
    if (ev) cudaEventRecord(ev[2 * (stage - 1)], st);
    rc = launch_rhs(m, mixed, epb, src_rho, src_q0, src_q1, src_q2, src_E, s->mu_factor, les ? m->musgs_int : nullptr,
                    st);
    if (rc) return rc;
    if (ev) cudaEventRecord(ev[2 * (stage - 1) + 1], st);
    GatherArgs g{};
    g.dt = dt_dev;
    g.y[0] = s->rho; g.y[1] = s->q; g.y[2] = s->q + N; g.y[3] = s->q + 2 * N; g.y[4] = s->E;
    g.u0 = s->u; g.u1 = s->u + N; g.u2 = s->u + 2 * N;
    g.pr = s->pr; g.Tem = s->Tem; g.e_int = s->e_int; g.eta = s->eta; g.csound = s->csound;
    g.machno = s->machno; g.mu_fluid = s->mu_fluid; g.Reta = loc.Reta; g.mu_factor = s->mu_factor;
    g.node_member = m->nmember > 0 ? m->node_member : nullptr;
    g.member_reduce = m->nmember > 0 ? 1 : 0;
    if (stage_store && stage < 4) g.ys = stage_store + (size_t)(stage - 1) * 5 * N;
    if (ev) cudaEventRecord(ev[2 * (3 + stage)], st);
    rc = launch_gather(m, mixed, stage, g, st);
    if (rc) return rc;
    if (stage == 4 && m->nmember > 0) {
      k_member_eta<<<m->nmember, 512, 0, st>>>(m->member_node_off, s->eta, m->member_scal, m->prm.normalise);
      SOD_CHECK_LAUNCH();
    }
    if (pre) {
      if (stage < 4) {
        double* ynext = (stage_store && stage < 4) ? stage_store + (size_t)(stage - 1) * 5 * N : m->buf.ys;
        rc = pre_stage(ynext, stage + 1);
      } else {
        rc = zone ? zone_final(m, s, st) : SOD_OK;
        if (!rc && bc) rc = bc_final(m, s, loc.Reta, st);
      }
      if (rc) return rc;
    }
    if (ev) cudaEventRecord(ev[2 * (3 + stage) + 1], st);
  }
  if (ev) cudaEventRecord(ev[16], st);
  if (les) {
    // sgs_visc after the step (time_integ.f90:498-506), before the dt of the next step uses it
    // (CFDSolverBase.f90:1592); independent of the entropy viscosity, so it may run first
    rc = launch_sgs(m, s->u, st);
    if (rc) return rc;
  }
  rc = launch_visc_dt(m, &loc, dt_next, mixed ? m->mue32 : nullptr, st);
  if (ev) cudaEventRecord(ev[17], st);
  return rc;
}

}  // namespace sod

using namespace sod;

static int check_state(SodMesh* m, SodState* s) {
  SOD_ARG(m && s, "mesh/state null");
  SOD_ARG(s->rho && s->q && s->E && s->u && s->pr && s->Tem && s->e_int && s->eta && s->csound && s->machno &&
              s->mu_fluid && s->mu_factor && s->mu_e,
          "state arrays must be non-null (Reta optional)");
  return SOD_OK;
}

extern "C" {

int sod_rk4_main(SodMesh* m, SodState* s, const double* dt_dev, double* dt_next_dev, SodPrecision prec,
                 sod_stream_t stream) {
  int rc = check_state(m, s);
  if (rc) return rc;
  SOD_ARG(dt_dev, "dt_dev null");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  cudaStream_t st = (cudaStream_t)stream;
  const bool mixed = prec == SOD_MIXED;
  rc = ensure_step_buffers(m, mixed);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, s->mu_e, m->mue_int, st);
  if (rc) return rc;
  rc = les_in(m, s, st);
  if (rc) return rc;
  if (mixed) {
    rc = launch_copy_f32(m->mue_int, m->mue32, (int64_t)m->nelem * NN, st);
    if (rc) return rc;
  }
  rc = run_step(m, s, dt_dev, dt_next_dev, mixed, st);
  if (rc) return rc;
  rc = les_out(m, s, st);
  if (rc) return rc;
  return mesh_internal_to_ref_elem(m, m->mue_int, s->mu_e, st);
}

int sod_rk4_main_record(SodMesh* m, SodState* s, const double* dt_dev, double* dt_next_dev, double* stages,
                        SodPrecision prec, sod_stream_t stream) {
  int rc = check_state(m, s);
  if (rc) return rc;
  SOD_ARG(dt_dev && stages, "dt_dev/stages null");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  cudaStream_t st = (cudaStream_t)stream;
  const bool mixed = prec == SOD_MIXED;
  rc = ensure_step_buffers(m, mixed);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, s->mu_e, m->mue_int, st);
  if (rc) return rc;
  rc = les_in(m, s, st);
  if (rc) return rc;
  if (mixed) {
    rc = launch_copy_f32(m->mue_int, m->mue32, (int64_t)m->nelem * NN, st);
    if (rc) return rc;
  }
  rc = run_step(m, s, dt_dev, dt_next_dev, mixed, st, nullptr, stages);
  if (rc) return rc;
  rc = les_out(m, s, st);
  if (rc) return rc;
  return mesh_internal_to_ref_elem(m, m->mue_int, s->mu_e, st);
}

int sod_rk4_steps(SodMesh* m, SodState* s, double* dt_dev, int nsteps, SodPrecision prec, sod_stream_t stream) {
  int rc = check_state(m, s);
  if (rc) return rc;
  SOD_ARG(dt_dev && nsteps >= 0, "dt_dev/nsteps");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  cudaStream_t st = (cudaStream_t)stream;
  const bool mixed = prec == SOD_MIXED;
  rc = ensure_step_buffers(m, mixed);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, s->mu_e, m->mue_int, st);
  if (rc) return rc;
  rc = les_in(m, s, st);
  if (rc) return rc;
  if (mixed) {
    rc = launch_copy_f32(m->mue_int, m->mue32, (int64_t)m->nelem * NN, st);
    if (rc) return rc;
  }
  if (nsteps > 0) {
    // capture one step into a graph keyed by (state pointers, dt pointer, precision, epb)
    uint64_t key = (uint64_t)(uintptr_t)s->rho ^ ((uint64_t)(uintptr_t)dt_dev << 1) ^ ((uint64_t)mixed << 63) ^
                   ((uint64_t)(uintptr_t)s->Reta << 3) ^ ((uint64_t)m->tuned_epb[mixed ? 1 : 0] << 56) ^
                   ((uint64_t)(uintptr_t)(les_active(m, s) ? s->mu_sgs : nullptr) << 5);
    auto it = m->graphs.find(key);
    if (it == m->graphs.end()) {
      cudaStream_t cap;
      SOD_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      cudaGraph_t graph;
      int64_t before = g_launches.load();
      SOD_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
      rc = run_step(m, s, dt_dev, dt_dev, mixed, cap);
      cudaError_t ce = cudaStreamEndCapture(cap, &graph);
      cudaStreamDestroy(cap);
      if (rc) return rc;
      if (ce != cudaSuccess) {
        set_error("graph capture failed: %s", cudaGetErrorString(ce));
        return SOD_ERR_CUDA;
      }
      GraphEntry ge;
      ge.nkernels = (int)(g_launches.load() - before);
      g_launches.fetch_sub(ge.nkernels);
      cudaError_t ie = cudaGraphInstantiate(&ge.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        set_error("graph instantiate failed: %s", cudaGetErrorString(ie));
        return SOD_ERR_CUDA;
      }
      it = m->graphs.emplace(key, ge).first;
    }
    for (int t = 0; t < nsteps; ++t) {
      SOD_CUDA(cudaGraphLaunch(it->second.exec, st));
      g_launches.fetch_add(it->second.nkernels);
    }
  }
  rc = les_out(m, s, st);
  if (rc) return rc;
  return mesh_internal_to_ref_elem(m, m->mue_int, s->mu_e, st);
}

int sod_step_profile(SodMesh* m, SodState* s, double* dt_dev, int nsteps, SodPrecision prec, sod_stream_t stream,
                     float* ms_out) {
  int rc = check_state(m, s);
  if (rc) return rc;
  SOD_ARG(dt_dev && nsteps > 0 && ms_out, "dt_dev/nsteps/ms_out");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  cudaStream_t st = (cudaStream_t)stream;
  const bool mixed = prec == SOD_MIXED;
  rc = ensure_step_buffers(m, mixed);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, s->mu_e, m->mue_int, st);
  if (rc) return rc;
  rc = les_in(m, s, st);
  if (rc) return rc;
  if (mixed) {
    rc = launch_copy_f32(m->mue_int, m->mue32, (int64_t)m->nelem * NN, st);
    if (rc) return rc;
  }
  cudaEvent_t ev[18];
  for (int q = 0; q < 18; ++q) SOD_CUDA(cudaEventCreate(&ev[q]));
  double acc[3] = {0, 0, 0};
  for (int t = 0; t < nsteps && rc == SOD_OK; ++t) {
    rc = run_step(m, s, dt_dev, dt_dev, mixed, st, ev);
    if (rc) break;
    if (cudaEventSynchronize(ev[17]) != cudaSuccess) { rc = SOD_ERR_CUDA; break; }
    for (int q = 0; q < 9; ++q) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[2 * q], ev[2 * q + 1]);
      acc[q < 4 ? 0 : (q < 8 ? 1 : 2)] += ms;
    }
  }
  for (int q = 0; q < 18; ++q) cudaEventDestroy(ev[q]);
  if (rc) return rc;
  ms_out[0] = (float)(acc[0] / (4.0 * nsteps));
  ms_out[1] = (float)(acc[1] / (4.0 * nsteps));
  ms_out[2] = (float)(acc[2] / nsteps);
  rc = les_out(m, s, st);
  if (rc) return rc;
  return mesh_internal_to_ref_elem(m, m->mue_int, s->mu_e, st);
}

// Elements-per-CTA autotuner for the fused RHS kernel: times every candidate on the caller's
// state (3 warm-up + 10 timed launches each, CUDA events on the stream) and keeps the fastest
// for this mesh and precision; later steps and newly captured graphs use it.
int sod_set_rhs_config(SodMesh* m, SodPrecision prec, int config) {
  SOD_ARG(m, "mesh null");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  const bool mixed = prec == SOD_MIXED;
  const bool ok = (config == 1 || config == 2 || config == 4 || (mixed && config == 8));
  SOD_ARG(ok || config == 0, "unknown fused-RHS configuration");
  if (m->tuned_epb[mixed ? 1 : 0] != config) {
    for (auto& kv : m->graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    m->graphs.clear();
  }
  m->tuned_epb[mixed ? 1 : 0] = config;
  return SOD_OK;
}

int sod_autotune(SodMesh* m, SodState* s, SodPrecision prec, int* best_epb, float* best_ms, sod_stream_t stream) {
  int rc = check_state(m, s);
  if (rc) return rc;
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  cudaStream_t st = (cudaStream_t)stream;
  const bool mixed = prec == SOD_MIXED;
  rc = ensure_step_buffers(m, mixed);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, s->mu_e, m->mue_int, st);
  if (rc) return rc;
  rc = les_in(m, s, st);
  if (rc) return rc;
  if (mixed) {
    rc = launch_copy_f32(m->mue_int, m->mue32, (int64_t)m->nelem * NN, st);
    if (rc) return rc;
  }
  const size_t N = m->npoin;
  const int fp64_cand[] = {1, 2, 4};
  const int mixed_cand[] = {1, 2, 4, 8};
  const int* cand = mixed ? mixed_cand : fp64_cand;
  const int nc = mixed ? 4 : 3;
  cudaEvent_t e0, e1;
  SOD_CUDA(cudaEventCreate(&e0));
  SOD_CUDA(cudaEventCreate(&e1));
  int best = 0;
  float bms = 1e30f;
  for (int c = 0; c < nc && rc == SOD_OK; ++c) {
    for (int r = 0; r < 3 && rc == SOD_OK; ++r)
      rc = launch_rhs(m, mixed, cand[c], s->rho, s->q, s->q + N, s->q + 2 * N, s->E, s->mu_factor, nullptr, st);
    cudaEventRecord(e0, st);
    for (int r = 0; r < 10 && rc == SOD_OK; ++r)
      rc = launch_rhs(m, mixed, cand[c], s->rho, s->q, s->q + N, s->q + 2 * N, s->E, s->mu_factor, nullptr, st);
    cudaEventRecord(e1, st);
    if (rc) break;
    if (cudaEventSynchronize(e1) != cudaSuccess) { rc = SOD_ERR_CUDA; break; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= 10.f;
    if (ms < bms) { bms = ms; best = cand[c]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  m->tuned_epb[mixed ? 1 : 0] = best;
  if (best_epb) *best_epb = best;
  if (best_ms) *best_ms = bms;
  return SOD_OK;
}

int sod_rhs(SodMesh* m, const double* rho, const double* q, const double* E, const double* mu_e,
            const double* mu_factor, double* Rmass, double* Rmom, double* Rener, double* Reta,
            SodPrecision prec, sod_stream_t stream) {
  SOD_ARG(m && rho && q && E && mu_e && mu_factor, "inputs null");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  cudaStream_t st = (cudaStream_t)stream;
  const bool mixed = prec == SOD_MIXED;
  int rc = ensure_step_buffers(m, mixed);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, mu_e, m->mue_int, st);
  if (rc) return rc;
  if (mixed) {
    rc = launch_copy_f32(m->mue_int, m->mue32, (int64_t)m->nelem * NN, st);
    if (rc) return rc;
  }
  const size_t N = m->npoin;
  const int epb = m->tuned_epb[mixed ? 1 : 0] ? m->tuned_epb[mixed ? 1 : 0] : (mixed ? 4 : 2);
  rc = launch_rhs(m, mixed, epb, rho, q, q + N, q + 2 * N, E, mu_factor, nullptr, st);
  if (rc) return rc;
  GatherArgs g{};
  g.out[0] = Rmass;
  g.out[1] = Rmom ? Rmom : nullptr;
  g.out[2] = Rmom ? Rmom + N : nullptr;
  g.out[3] = Rmom ? Rmom + 2 * N : nullptr;
  g.out[4] = Rener;
  g.out[5] = Reta;
  return launch_gather(m, mixed, 0, g, st);
}

int sod_rk4_main_host(SodMesh* m, SodState* h, double dt_host, double* dt_next_host, SodPrecision prec,
                      sod_stream_t stream) {
  SOD_ARG(m && h, "mesh/state null");
  SOD_ARG(h->rho && h->q && h->E && h->mu_e && h->mu_factor, "host state arrays null");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t N = m->npoin, EN = (size_t)m->nelem * NN;
  // persistent device mirror owned by the mesh
  auto& mv = m->host_mirror;
  const size_t sizes[] = {N, 3 * N, N, 3 * N, N, N, N, N, N, N, N, N, EN, N, 1, EN};
  if (mv.empty()) {
    for (size_t s : sizes) {
      double* p = nullptr;
      SOD_CUDA(cudaMalloc(&p, s * sizeof(double)));
      mv.push_back(p);
    }
  }
  const bool les_h = h->mu_sgs && m->prm.flag_les == 1;
  SodState d{mv[0], mv[1], mv[2], mv[3], mv[4], mv[5], mv[6], mv[7], mv[8], mv[9], mv[10], mv[11], mv[12], mv[13],
             les_h ? mv[15] : nullptr};
  double* ddt = mv[14];
  SOD_CUDA(cudaMemcpyAsync(d.rho, h->rho, N * 8, cudaMemcpyHostToDevice, st));
  SOD_CUDA(cudaMemcpyAsync(d.q, h->q, 3 * N * 8, cudaMemcpyHostToDevice, st));
  SOD_CUDA(cudaMemcpyAsync(d.E, h->E, N * 8, cudaMemcpyHostToDevice, st));
  SOD_CUDA(cudaMemcpyAsync(d.mu_e, h->mu_e, EN * 8, cudaMemcpyHostToDevice, st));
  SOD_CUDA(cudaMemcpyAsync(d.mu_factor, h->mu_factor, N * 8, cudaMemcpyHostToDevice, st));
  SOD_CUDA(cudaMemcpyAsync(ddt, &dt_host, 8, cudaMemcpyHostToDevice, st));
  if (les_h) SOD_CUDA(cudaMemcpyAsync(d.mu_sgs, h->mu_sgs, EN * 8, cudaMemcpyHostToDevice, st));
  struct Pair { double* hst; double* dev; size_t n; };
  Pair outs[] = {{h->rho, d.rho, N}, {h->q, d.q, 3 * N}, {h->E, d.E, N}, {h->u, d.u, 3 * N}, {h->pr, d.pr, N},
                 {h->Tem, d.Tem, N}, {h->e_int, d.e_int, N}, {h->eta, d.eta, N}, {h->csound, d.csound, N},
                 {h->machno, d.machno, N}, {h->mu_fluid, d.mu_fluid, N}, {h->mu_e, d.mu_e, EN},
                 {h->Reta, d.Reta, N}, {les_h ? h->mu_sgs : nullptr, d.mu_sgs, EN}};
  if (m->has_slaves)  // the step leaves slave rows as they are: bring in the rows it will copy back
    for (int i = 3; i < 11; ++i)
      if (outs[i].hst) SOD_CUDA(cudaMemcpyAsync(outs[i].dev, outs[i].hst, outs[i].n * 8, cudaMemcpyHostToDevice, st));
  if (m->has_slaves && h->Reta) SOD_CUDA(cudaMemcpyAsync(d.Reta, h->Reta, N * 8, cudaMemcpyHostToDevice, st));
  int rc = sod_rk4_main(m, &d, ddt, ddt, prec, stream);
  if (rc) return rc;
  for (auto& o : outs)
    if (o.hst) SOD_CUDA(cudaMemcpyAsync(o.hst, o.dev, o.n * 8, cudaMemcpyDeviceToHost, st));
  if (dt_next_host) SOD_CUDA(cudaMemcpyAsync(dt_next_host, ddt, 8, cudaMemcpyDeviceToHost, st));
  if (int rc2 = sync_stream(st)) return rc2;
  bool bad = false;
  if (int rc3 = take_nonfinite(m, st, &bad)) return rc3;
  if (bad) {
    set_error("a non-finite value (NaN/Inf) appeared in rho, q or E during the step");
    return SOD_ERR_NONFINITE;
  }
  return SOD_OK;
}

int sod_smart_visc_spectral(SodMesh* m, const double* Reta, const double* rho, const double* u,
                            const double* csound, const double* Tem, const double* eta, double* mu_e,
                            sod_stream_t stream);
int sod_adapt_dt_cfl(SodMesh* m, const double* u, const double* csound, const double* mu_fluid,
                     const double* mu_sgs, const double* rho, double* dt_dev, sod_stream_t stream);

}  // extern "C"
