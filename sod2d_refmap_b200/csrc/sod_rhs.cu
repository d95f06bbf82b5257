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
#include "sod_step_kernels.cuh"
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

constexpr int NBUF = 13;  // batch-A fields (12, and p + E with flag_total_enthalpy)
constexpr int NP2 = 18;   // 6 contravariant fluxes x 3 directions

template <typename R>
constexpr size_t rhs_smem_bytes(int epb) {
  return sizeof(R) * (size_t)epb * (NBUF + NP2) * FSTRIDE;
}

// One tile of EPB elements (64 threads each) of the fused RHS; smem_raw holds
// rhs_smem_bytes<R>(EPB).  Every thread of the block calls it (it holds block barriers).
// TOTH: flag_total_enthalpy (energy convection of full_convec_ijk_H)
template <typename R, int EPB, bool TOTH>
__device__ __forceinline__ void rhs_fused_tile(const RhsArgs& a, int tile, unsigned char* smem_raw) {
  R* buf_all = reinterpret_cast<R*>(smem_raw);
  const int tid = threadIdx.x;
  const int es = tid >> 6;
  const int d = tid & 63;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4;
  const int e = tile * EPB + es;
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
  // the energy convection is linear in (h, k) and every h term of elem_convec.f90:415-425 has a k
  // twin of the same form: both quartets are evaluated at once on the total enthalpy H = h + k
  const double Ht = h + kk;
  buf[8 * FSTRIDE + s_me] = (R)Ht;
  buf[9 * FSTRIDE + s_me] = (R)(rho * Ht);
  buf[10 * FSTRIDE + s_me] = (R)eta_full;
  buf[11 * FSTRIDE + s_me] = (R)T;
  // flag_total_enthalpy: full_convec_ijk_H differentiates p + E and (E + p) u
  if constexpr (TOTH) buf[12 * FSTRIDE + s_me] = (R)(p + Et);
  __syncthreads();

  R gradRho[3], gradU[3][3], gradQ[3][3], gradP[3], gradH[3], gradRH[3], gradEta[3], gradT[3];
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
    phys(H, gx, gy, gz, gradEta[0], gradEta[1], gradEta[2]);
    giso(buf + 11 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
    phys(H, gx, gy, gz, gradT[0], gradT[1], gradT[2]);
    if constexpr (TOTH) {
      R gradEp[3];
      giso(buf + 12 * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);
      phys(H, gx, gy, gz, gradEp[0], gradEp[1], gradEp[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) uGradEp = uGradEp + R(0.5) * ((R)uv[c] * gradEp[c]);
    }
  }
  const R divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
  const R divQ = gradQ[0][0] + gradQ[1][1] + gradQ[2][2];
  const R rhoR = (R)rho, HR = (R)Ht, etaR = (R)eta_full;
  const R uR[3] = {(R)uv[0], (R)uv[1], (R)uv[2]};
  const R qR[3] = {(R)qv[0], (R)qv[1], (R)qv[2]};
  const R rHR = (R)(rho * Ht);

  // ---- convective terms available after batch A (elem_convec.f90:412-432)
  R Rm = R(0.5) * (divQ + rhoR * divU);
  R Ren = R(0.25) * (HR * divQ + rHR * divU);
  R Rmo[3];
  R Ret = R(0.5) * (etaR * divU);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Rmo[c] = R(0.25) * (uR[c] * divQ + qR[c] * divU) + gradP[c];
    Rm += R(0.5) * (uR[c] * gradRho[c]);
    Ren += R(0.25) * (qR[c] * gradH[c] + uR[c] * gradRH[c] + (HR * uR[c]) * gradRho[c]);
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
  // ---- batches B and C: divergences of the product vectors (rho H u, H u, eta u; (E + p) u with
  // flag_total_enthalpy) and tensors (q x u, u x u).  Every line point m forms its 24 terms
  // D[x][m] f u_c of the line sums from batch A's slots as (D[x][m] u_c) f, so nothing more is
  // staged; the line sums of each direction are folded with He before the next direction.
  {
    R divFe = R(0), divFue = R(0), divFeta = R(0);
    R dF[3] = {R(0), R(0), R(0)}, dFuu[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      const R* Dd = dir == 0 ? Dx : (dir == 1 ? Dy : Dz);
      {
        R gB[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) gB[q] = R(0);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int sp = dir == 0 ? sidx(m, j, k) : (dir == 1 ? sidx(i, m, k) : sidx(i, j, m));
          const R w = Dd[m];
          const R u0 = buf[1 * FSTRIDE + sp], u1 = buf[2 * FSTRIDE + sp], u2 = buf[3 * FSTRIDE + sp];
          const R fe = TOTH ? buf[12 * FSTRIDE + sp] : buf[9 * FSTRIDE + sp];
          const R fh = buf[8 * FSTRIDE + sp];
          const R fet = buf[10 * FSTRIDE + sp];
          // the line weight scales u_c, the factor all 9 products share
          const R wu[3] = {w * u0, w * u1, w * u2};
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            gB[c] += wu[c] * fe;
            gB[3 + c] += wu[c] * fh;
            gB[6 + c] += wu[c] * fet;
          }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const R hc = H[3 * c + dir];
          divFe += hc * gB[c];
          divFue += hc * gB[3 + c];
          divFeta += hc * gB[6 + c];
        }
      }
      {
        R gQ[9], gU[6];
#pragma unroll
        for (int q = 0; q < 9; ++q) gQ[q] = R(0);
#pragma unroll
        for (int q = 0; q < 6; ++q) gU[q] = R(0);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int sp = dir == 0 ? sidx(m, j, k) : (dir == 1 ? sidx(i, m, k) : sidx(i, j, m));
          const R w = Dd[m];
          const R u[3] = {buf[1 * FSTRIDE + sp], buf[2 * FSTRIDE + sp], buf[3 * FSTRIDE + sp]};
          const R q[3] = {buf[4 * FSTRIDE + sp], buf[5 * FSTRIDE + sp], buf[6 * FSTRIDE + sp]};
          const R wu[3] = {w * u[0], w * u[1], w * u[2]};
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) gQ[3 * r + c] += wu[c] * q[r];
          gU[0] += wu[0] * u[0];
          gU[1] += wu[0] * u[1];
          gU[2] += wu[0] * u[2];
          gU[3] += wu[1] * u[1];
          gU[4] += wu[1] * u[2];
          gU[5] += wu[2] * u[2];
        }
        // u x u is symmetric: component (r, c) is the stored product of min(r,c), max(r,c)
        const int symidx[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const R hc = H[3 * c + dir];
            dF[r] += hc * gQ[3 * r + c];
            dFuu[r] += hc * gU[symidx[r][c]];
          }
      }
    }
    Ren += R(0.25) * (divFe + rhoR * divFue);
    Ret += R(0.5) * divFeta;
    if constexpr (TOTH) Ren = R(0.5) * (divFe + (R)(Et + p) * divU) + uGradEp;  // elem_convec.f90:171-177
#pragma unroll
    for (int r = 0; r < 3; ++r) Rmo[r] += R(0.25) * (dF[r] + rhoR * dFuu[r]);
  }
  __syncthreads();  // pass-1 fluxes visible

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

template <typename R, int EPB, bool TOTH>
__global__ void __launch_bounds__(64 * EPB, (EPB >= 6 ? 1 : 6 / EPB)) k_rhs_fused(const RhsArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  rhs_fused_tile<R, EPB, TOTH>(a, blockIdx.x, smem_raw);
}

// One RK stage of the FP64 path in one cooperative launch (persistent blocks): the fused RHS
// over element tiles, then persist_stage_tail (gather / stage update; at stage 4 the entropy
// viscosity and dt).
template <int EPB, bool TOTH>
__global__ void __launch_bounds__(64 * EPB) k_stage_fused(const StageArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ntiles = (p.r.nelem + EPB - 1) / EPB;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    rhs_fused_tile<double, EPB, TOTH>(p.r, t, smem_raw);
    __syncthreads();  // the next tile reuses the shared memory
  }
  persist_stage_tail<double, EPB>(p, smem_raw);
}

// resident 256-thread blocks per SM the register budget must allow.  FP32 residual rows (mixed
// path): 4 blocks, 64 registers, no spill with the predicated groups of 4, 2% faster than full
// groups at 5 blocks (the predicated groups at 5 blocks spilled 76 bytes and ran 4% slower
// than that).  FP64 rows: 5 blocks, 48 registers (48-72 bytes of spill), 1% faster than 4
// blocks; 7 blocks capped the kernel at 32 registers and spilled 140-244 bytes
#ifndef SOD_KG_MIN_BLOCKS
#define SOD_KG_MIN_BLOCKS 4
#endif
#ifndef SOD_KG_MIN_BLOCKS_F64
#define SOD_KG_MIN_BLOCKS_F64 5
#endif
template <typename R, int STAGE>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? SOD_KG_MIN_BLOCKS : SOD_KG_MIN_BLOCKS_F64) k_gather_rk(const GatherArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  double eta_n = 0.0;
  const bool act = gather_rk_node<R, STAGE>(a, n, eta_n);
  if constexpr (STAGE == 4) {
    if (a.member_reduce) return;  // uniform across the grid
    __shared__ double sh[3 * 8];
    gather_eta_reduce(a, act ? eta_n : 0.0, act ? eta_n : -1e300, act ? eta_n : 1e300, sh);
  }
}

#ifndef SOD_KV_MIN_BLOCKS
#define SOD_KV_MIN_BLOCKS 3  // resident 256-thread blocks per SM: 80 registers, no spill (4 blocks: 64 registers with spills, the same time)
#endif
__global__ void __launch_bounds__(32 * KV_WARPS, SOD_KV_MIN_BLOCKS) k_visc_dt(const ViscArgs a) {
  __shared__ double sm[KV_WARPS][KV_WSMEM];
  __shared__ unsigned long long lim[KV_WARPS];
  const int wb = threadIdx.x >> 5, e = blockIdx.x * KV_WARPS + wb;
  // one mesh: one dt atomic per block on the minimum of its elements' limits, instead of one per
  // element on the same address; an ensemble's elements take their member's slot each
  const bool per_elem = a.elem_member != nullptr;
  unsigned long long b = ~0ull;
  if (e < a.nelem) b = visc_dt_warp(a, e, threadIdx.x & 31, sm[wb], per_elem);
  if (!per_elem && a.dt_out) {
    if ((threadIdx.x & 31) == 0) lim[wb] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int q = 1; q < KV_WARPS; ++q) b = min(b, lim[q]);
      if (b != ~0ull) atomicMin(reinterpret_cast<unsigned long long*>(a.dt_bits), b);
    }
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
  SOD_CUDA(cudaFuncSetAttribute(k_stage_fused<EPB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)rhs_smem_bytes<double>(EPB)));
  SOD_CUDA(cudaFuncSetAttribute(k_stage_fused<EPB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)rhs_smem_bytes<double>(EPB)));
  return SOD_OK;
}

// Cooperative launch of one persistent FP64 stage; ctas_per_sm <= 0 asks for the most that fit.
template <int EPB>
static int launch_stage_fused_t(const StageArgs& p, int ctas_per_sm, int* grid_out, cudaStream_t st) {
  const bool toth = p.r.prm.total_enthalpy != 0;
  const void* fn = toth ? (const void*)k_stage_fused<EPB, true> : (const void*)k_stage_fused<EPB, false>;
  const size_t smem = rhs_smem_bytes<double>(EPB);
  int occ = 0, dev = 0, nsm = 0;
  SOD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 64 * EPB, smem));
  SOD_CUDA(cudaGetDevice(&dev));
  SOD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (occ <= 0) {
    set_error("persistent stage kernel: no resident block fits (EPB %d)", EPB);
    return SOD_ERR_UNSUPPORTED;
  }
  const int per = (ctas_per_sm > 0 && ctas_per_sm < occ) ? ctas_per_sm : occ;
  const int ntiles = (p.r.nelem + EPB - 1) / EPB;
  const int grid = std::min(per * nsm, ntiles);
  if (grid_out) *grid_out = grid;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(64 * EPB);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {const_cast<StageArgs*>(&p)};
  SOD_CUDA(cudaLaunchKernelExC(&cfg, fn, args));
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int launch_stage_mixed2(const StageArgs& p, int epb, int ctas_per_sm, int* grid_out, cudaStream_t st);
void stage_mixed2_info(int epb, bool toth, const void** fn, size_t* smem);

// the persistent stage kernel of a configuration and its dynamic shared memory
void persist_kernel_info(bool mixed, int epb, bool toth, const void** fn, size_t* smem) {
  if (mixed) {
    stage_mixed2_info(epb, toth, fn, smem);
    return;
  }
  switch (epb) {
    case 1: *fn = toth ? (const void*)k_stage_fused<1, true> : (const void*)k_stage_fused<1, false>; break;
    case 4: *fn = toth ? (const void*)k_stage_fused<4, true> : (const void*)k_stage_fused<4, false>; break;
    case 8: *fn = toth ? (const void*)k_stage_fused<8, true> : (const void*)k_stage_fused<8, false>; break;
    default: *fn = toth ? (const void*)k_stage_fused<2, true> : (const void*)k_stage_fused<2, false>; epb = 2;
  }
  *smem = rhs_smem_bytes<double>(epb);
}

// One persistent stage launch of either precision
int launch_stage(const StageArgs& p, bool mixed, int epb, int ctas_per_sm, int* grid_out, cudaStream_t st) {
  if (mixed) return launch_stage_mixed2(p, epb, ctas_per_sm, grid_out, st);
  switch (epb) {
    case 1: return launch_stage_fused_t<1>(p, ctas_per_sm, grid_out, st);
    case 4: return launch_stage_fused_t<4>(p, ctas_per_sm, grid_out, st);
    case 8: return launch_stage_fused_t<8>(p, ctas_per_sm, grid_out, st);
    default: return launch_stage_fused_t<2>(p, ctas_per_sm, grid_out, st);
  }
}

int init_kernel_attrs() {
  static bool done = false;
  if (done) return SOD_OK;
  int rc = set_rhs_attr<double, 1>() | set_rhs_attr<double, 2>() | set_rhs_attr<double, 4>() |
           set_rhs_attr<double, 8>() |
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

static RhsArgs make_rhs_args(SodMesh* m, bool mixed, const double* rho, const double* q0, const double* q1,
                             const double* q2, const double* E, const double* mu_factor, const double* musgs_int) {
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
  return a;
}

int launch_rhs(SodMesh* m, bool mixed, int epb, const double* rho, const double* q0, const double* q1,
               const double* q2, const double* E, const double* mu_factor, const double* musgs_int,
               cudaStream_t st) {
  const RhsArgs a = make_rhs_args(m, mixed, rho, q0, q1, q2, E, mu_factor, musgs_int);
  if (!mixed) {
    switch (epb) {
      case 1: return launch_rhs_t<double, 1>(a, st);
      case 4: return launch_rhs_t<double, 4>(a, st);
      case 8: return launch_rhs_t<double, 8>(a, st);
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

static void fill_gather_args(SodMesh* m, int stage, GatherArgs& a) {
  a.npoin = m->npoin;
  a.nwork = m->npoin_w;
  a.slaves = m->has_slaves ? 1 : 0;
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
}

int launch_gather(SodMesh* m, bool mixed, int stage, GatherArgs& a, cudaStream_t st) {
  fill_gather_args(m, stage, a);
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

static ViscArgs make_visc_args(SodMesh* m, const SodState* s, double* dt_out, float* mue32) {
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
  v.dt_bits = m->nmember > 0 ? m->member_dt_bits : m->buf.scal + 3;
  v.elem_member = m->nmember > 0 ? m->elem_member : nullptr;
  v.member_scal = m->member_scal;
  v.dt_out = dt_out;
  v.prm = m->prm;
  return v;
}

int launch_visc_dt(SodMesh* m, const SodState* s, double* dt_out, float* mue32, cudaStream_t st) {
  const ViscArgs v = make_visc_args(m, s, dt_out, mue32);
  const int nm = m->nmember > 0 ? m->nmember : 1;
  if (dt_out) SOD_CUDA(cudaMemsetAsync(v.dt_bits, 0x7F, sizeof(double) * nm, st));  // 1.38e306 each
  const int grid = (m->nelem + KV_WARPS - 1) / KV_WARPS;
  k_visc_dt<<<grid, 32 * KV_WARPS, 0, st>>>(v);
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
  // the FP64 rsum eta column, dead after stage 4 reads it (the mixed path's FP32 accumulators
  // end before it)
  return m->buf.rsum + 5 * (size_t)m->npoin;
}

// The periodic step (no boundaries, buffer zone, wall model, source term or LES) as four
// cooperative launches, one per RK stage: fused RHS, grid barrier, gather / stage update; the
// last one also forms the entropy viscosity and the next dt.  Same arithmetic per element and
// per node as the two-launch path; the entropy sums are blocked by the persistent grid instead,
// so the normalisation can differ from that path's in the last bits.
static int run_step_persist(SodMesh* m, SodState* s, SodState& loc, const double* dt_dev, double* dt_next,
                            bool mixed, int epb, int ctas_per_sm, cudaStream_t st) {
  NvtxRange range(mixed ? "sod rk4 step persistent (mixed)" : "sod rk4 step persistent (fp64)");
  const size_t N = m->npoin;
  StageArgs p{};
  p.g.dt = dt_dev;
  p.g.y[0] = s->rho; p.g.y[1] = s->q; p.g.y[2] = s->q + N; p.g.y[3] = s->q + 2 * N; p.g.y[4] = s->E;
  p.g.u0 = s->u; p.g.u1 = s->u + N; p.g.u2 = s->u + 2 * N;
  p.g.pr = s->pr; p.g.Tem = s->Tem; p.g.e_int = s->e_int; p.g.eta = s->eta; p.g.csound = s->csound;
  p.g.machno = s->machno; p.g.mu_fluid = s->mu_fluid; p.g.Reta = loc.Reta; p.g.mu_factor = s->mu_factor;
  p.g.node_member = m->nmember > 0 ? m->node_member : nullptr;
  p.g.member_reduce = m->nmember > 0 ? 1 : 0;
  p.nmember = m->nmember;
  p.member_node_off = m->member_node_off;
  p.member_scal = m->member_scal;
  p.v = make_visc_args(m, &loc, dt_next, mixed ? m->mue32 : nullptr);
  const int nm = m->nmember > 0 ? m->nmember : 1;
  for (int stage = 1; stage <= 4; ++stage) {
    const double* y = m->buf.ys;
    if (stage == 1)
      p.r = make_rhs_args(m, mixed, s->rho, s->q, s->q + N, s->q + 2 * N, s->E, s->mu_factor, nullptr);
    else
      p.r = make_rhs_args(m, mixed, y, y + N, y + 2 * N, y + 3 * N, y + 4 * N, s->mu_factor, nullptr);
    p.g.ys = nullptr;
    fill_gather_args(m, stage, p.g);
    p.stage = stage;
    if (stage == 4 && dt_next) SOD_CUDA(cudaMemsetAsync(p.v.dt_bits, 0x7F, sizeof(double) * nm, st));
    if (int rc = launch_stage(p, mixed, epb, ctas_per_sm, nullptr, st)) return rc;
    if (stage == 4 && dt_next)
      SOD_CUDA(cudaMemcpyAsync(dt_next, p.v.dt_bits, sizeof(double) * nm, cudaMemcpyDeviceToDevice, st));
  }
  return SOD_OK;
}

// One RK4 step on device state (mu_e already in m->mue_int / mue32).  When ev is non-null,
// ev[2*slot] / ev[2*slot+1] bracket each kernel: slots 0-3 KR stages, 4-7 KG stages, 8 KV.
// When stage_store is non-null the stage states Y2, Y3, Y4 (5 columns of npoin each) are
// written there instead of the internal stage buffer (for the adjoint's reverse sweep).
// state_done (optional) is recorded on st once the new state and its EOS fields are final, before
// the entropy viscosity and dt (and LES's sgs viscosity) that end the step.
int run_step(SodMesh* m, SodState* s, const double* dt_dev, double* dt_next, bool mixed, cudaStream_t st,
             cudaEvent_t* ev = nullptr, double* stage_store = nullptr, cudaEvent_t state_done = nullptr) {
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
  const int pctas = m->persist_ctas[mixed ? 1 : 0];
  if (pctas > 0 && !pre && !les && m->wmodel.nw == 0 && !m->source && !ev && !stage_store) {
    // the one-launch stages form the entropy viscosity inside stage 4: the state is final at the end
    rc = run_step_persist(m, s, loc, dt_dev, dt_next, mixed, epb, pctas, st);
    if (!rc && state_done) SOD_CUDA(cudaEventRecord(state_done, st));
    return rc;
  }
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
  if (state_done) SOD_CUDA(cudaEventRecord(state_done, st));
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

static int rk4_main_impl(SodMesh* m, SodState* s, const double* dt_dev, double* dt_next_dev, SodPrecision prec,
                         sod_stream_t stream, cudaEvent_t state_done);

int sod_rk4_main(SodMesh* m, SodState* s, const double* dt_dev, double* dt_next_dev, SodPrecision prec,
                 sod_stream_t stream) {
  return rk4_main_impl(m, s, dt_dev, dt_next_dev, prec, stream, nullptr);
}

static int rk4_main_impl(SodMesh* m, SodState* s, const double* dt_dev, double* dt_next_dev, SodPrecision prec,
                         sod_stream_t stream, cudaEvent_t state_done) {
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
  rc = run_step(m, s, dt_dev, dt_next_dev, mixed, st, nullptr, nullptr, state_done);
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
  const bool ok = (config == 1 || config == 2 || config == 4 || config == 8);
  SOD_ARG(ok || config == 0, "unknown fused-RHS configuration");
  if (m->tuned_epb[mixed ? 1 : 0] != config) {
    for (auto& kv : m->graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    m->graphs.clear();
  }
  m->tuned_epb[mixed ? 1 : 0] = config;
  return SOD_OK;
}

int sod_set_stage_launch(SodMesh* m, SodPrecision prec, int ctas_per_sm) {
  SOD_ARG(m, "mesh null");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  SOD_ARG(ctas_per_sm >= 0 && ctas_per_sm <= 32, "ctas_per_sm must be in 0..32");
  const int i = prec == SOD_MIXED ? 1 : 0;
  if (m->persist_ctas[i] != ctas_per_sm) {
    for (auto& kv : m->graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    m->graphs.clear();
  }
  m->persist_ctas[i] = ctas_per_sm;
  return SOD_OK;
}

int sod_autotune_table(SodMesh* m, SodPrecision prec, int cap, int32_t* epb, int32_t* ctas_per_sm,
                       float* ms_per_stage) {
  SOD_ARG(m, "mesh null");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  const auto& t = m->tune_table[prec == SOD_MIXED ? 1 : 0];
  const int n = (int)t.size();
  for (int q = 0; q < n && q < cap; ++q) {
    if (epb) epb[q] = t[q].epb;
    if (ctas_per_sm) ctas_per_sm[q] = t[q].ctas;
    if (ms_per_stage) ms_per_stage[q] = t[q].ms;
  }
  return n;
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
  const int cand[] = {1, 2, 4, 8};
  cudaEvent_t e0, e1;
  SOD_CUDA(cudaEventCreate(&e0));
  SOD_CUDA(cudaEventCreate(&e1));
  // One RK stage 1 per trial (fused RHS + gather / stage update into the internal stage buffers;
  // the caller's state is only read).  Two dimensions: elements per CTA, and the launch shape -
  // two launches per stage (ctas 0) or one cooperative launch of c resident CTAs per SM.
  const bool plain = m->bc.nb == 0 && m->zone.nb == 0 && m->wmodel.nw == 0 && !m->source && !les_active(m, s);
  auto& table = m->tune_table[mixed ? 1 : 0];
  table.clear();
  GatherArgs g{};
  g.dt = m->buf.scal + 4;  // any finite scalar: stage 1 scales its stage-state update by it
  SOD_CUDA(cudaMemsetAsync(m->buf.scal + 4, 0, sizeof(double), st));
  g.y[0] = s->rho; g.y[1] = s->q; g.y[2] = s->q + N; g.y[3] = s->q + 2 * N; g.y[4] = s->E;
  g.mu_factor = s->mu_factor;
  g.node_member = nullptr;  // one dt scalar for the timing (an ensemble's per-member dt is not needed)
  auto trial = [&](int epb, int ctas, float* ms_out) -> int {
    int r2 = SOD_OK;
    auto once = [&]() -> int {
      if (ctas == 0) {
        int r3 = launch_rhs(m, mixed, epb, s->rho, s->q, s->q + N, s->q + 2 * N, s->E, s->mu_factor, nullptr, st);
        if (r3) return r3;
        GatherArgs gg = g;
        return launch_gather(m, mixed, 1, gg, st);
      }
      StageArgs p{};
      p.r = make_rhs_args(m, mixed, s->rho, s->q, s->q + N, s->q + 2 * N, s->E, s->mu_factor, nullptr);
      p.g = g;
      fill_gather_args(m, 1, p.g);
      p.stage = 1;
      return launch_stage(p, mixed, epb, ctas, nullptr, st);
    };
    for (int r = 0; r < 3 && r2 == SOD_OK; ++r) r2 = once();
    cudaEventRecord(e0, st);
    for (int r = 0; r < 10 && r2 == SOD_OK; ++r) r2 = once();
    cudaEventRecord(e1, st);
    if (r2) return r2;
    if (cudaEventSynchronize(e1) != cudaSuccess) return SOD_ERR_CUDA;
    cudaEventElapsedTime(ms_out, e0, e1);
    *ms_out /= 10.f;
    return SOD_OK;
  };
  int best = 0, best_ctas = 0;
  float bms = 1e30f, bms_rhs = 1e30f;
  for (int c = 0; c < 4 && rc == SOD_OK; ++c) {
    const int epb = cand[c];
    // the fused RHS alone (reported as best_ms, as before)
    {
      for (int r = 0; r < 3 && rc == SOD_OK; ++r)
        rc = launch_rhs(m, mixed, epb, s->rho, s->q, s->q + N, s->q + 2 * N, s->E, s->mu_factor, nullptr, st);
      cudaEventRecord(e0, st);
      for (int r = 0; r < 10 && rc == SOD_OK; ++r)
        rc = launch_rhs(m, mixed, epb, s->rho, s->q, s->q + N, s->q + 2 * N, s->E, s->mu_factor, nullptr, st);
      cudaEventRecord(e1, st);
      if (rc) break;
      if (cudaEventSynchronize(e1) != cudaSuccess) { rc = SOD_ERR_CUDA; break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      bms_rhs = std::min(bms_rhs, ms / 10.f);
    }
    // launch shapes: two launches, then persistent grids of occ, 3/4 occ and 1/2 occ CTAs per SM
    int shapes[4] = {0, 0, 0, 0}, ns = 1;
    if (plain) {
      const void* fn = nullptr;
      size_t smem = 0;
      persist_kernel_info(mixed, epb, m->prm.total_enthalpy != 0, &fn, &smem);
      int occ = 0;
      if (fn && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 64 * epb, smem) == cudaSuccess && occ > 0) {
        const int opts[3] = {occ, std::max(1, (3 * occ) / 4), std::max(1, occ / 2)};
        for (int o : opts) {
          bool dup = false;
          for (int q = 1; q < ns; ++q) dup |= shapes[q] == o;
          if (!dup) shapes[ns++] = o;
        }
      }
    }
    for (int q = 0; q < ns && rc == SOD_OK; ++q) {
      float ms = 0.f;
      rc = trial(epb, shapes[q], &ms);
      if (rc) break;
      table.push_back(SodMesh::TuneEntry{epb, shapes[q], ms});
      if (ms < bms) { bms = ms; best = epb; best_ctas = shapes[q]; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  const int i = mixed ? 1 : 0;
  if (m->tuned_epb[i] != best || m->persist_ctas[i] != best_ctas) {
    for (auto& kv : m->graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    m->graphs.clear();
  }
  m->tuned_epb[i] = best;
  m->persist_ctas[i] = best_ctas;
  if (best_epb) *best_epb = best;
  if (best_ms) *best_ms = bms_rhs;
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
  // the state fields are copied back on a second stream as soon as the step has formed them, so
  // that the read-back overlaps the entropy viscosity and dt that end the step; mu_e (and mu_sgs)
  // and dt follow on the caller's stream, which then waits for the copies
  if (!m->host_copy_stream) {
    SOD_CUDA(cudaStreamCreateWithFlags(&m->host_copy_stream, cudaStreamNonBlocking));
    SOD_CUDA(cudaEventCreateWithFlags(&m->host_ev_state, cudaEventDisableTiming));
    SOD_CUDA(cudaEventCreateWithFlags(&m->host_ev_copied, cudaEventDisableTiming));
  }
  cudaStream_t cs = m->host_copy_stream;
  int rc = rk4_main_impl(m, &d, ddt, ddt, prec, stream, m->host_ev_state);
  if (rc) return rc;
  SOD_CUDA(cudaStreamWaitEvent(cs, m->host_ev_state, 0));
  for (auto& o : outs) {
    if (!o.hst) continue;
    const bool tail = o.dev == d.mu_e || o.dev == d.mu_sgs;  // written after the state is final
    SOD_CUDA(cudaMemcpyAsync(o.hst, o.dev, o.n * 8, cudaMemcpyDeviceToHost, tail ? st : cs));
  }
  SOD_CUDA(cudaEventRecord(m->host_ev_copied, cs));
  if (dt_next_host) SOD_CUDA(cudaMemcpyAsync(dt_next_host, ddt, 8, cudaMemcpyDeviceToHost, st));
  SOD_CUDA(cudaStreamWaitEvent(st, m->host_ev_copied, 0));
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
