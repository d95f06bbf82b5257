// Mixed-precision fused element RHS with packed FP32 arithmetic (sm_100a FFMA2).
//
// The reference element loops of full_convec_ijk (elem_convec.f90:211-460), full_diffusion_ijk
// (elem_diffu.f90:12-198) and generic_scalar_convec_ijk (elem_convec.f90:462-570) in FP32 on
// deviation fields: each element subtracts FP64 references before the FP32 cast (the values of
// its node 0; for the directly differentiated fields an affine-in-xi reference, see batch A)
// and every product flux is expanded exactly around them, e.g. div(rho H u) = H_r div q +
// div(rho (H - H_r) u), so FP32 rounding acts on small deviations.  Assembly, lumped mass, RK
// state and reductions stay FP64.  The nodal fields are staged in shared memory as float2 pairs: one 8-byte shared load and one packed
// __ffma2_rn serve two fields, and the xi-lines are read as two 16-byte loads.  The energy
// convection is linear in (h, k) and every h term has a k twin of the same form (the two
// skew-symmetric quartets of elem_convec.f90:415-425), so both quartets are evaluated at once
// on the total enthalpy H = h + k: same mathematics, 4 field pairs fewer.  Pairing:
//   batch A  (rho',p') (u0',u1') (u2',q0') (q1',q2') (H',rho H') (eta',T')
//   batch BC (fe,fue)x3 (feta,F0.)x3 (F1.,F2.)x3 (Fuu0.,Fuu1.)x3 (Fuu22,0)
//   pass 2   (gradRho^,tauU^)x3 (gradT^,tauX^)x3 (tauY^,tauZ^)x3   (one slot per direction)
// where fe = rho H' u, fue = H' u, F = (q-q_r) x (u-u_r), Fuu = (u-u_r) x (u-u_r) and ^ marks
// contravariant fluxes.  The batch BC products are not stored: shared memory holds their 9
// factors (5 slots), and each line point forms the 25 weighted products D[x][m] a b from them as
// (D[x][m] a) b; that reads 5 slots per line point instead of 13 (863 instead of 1,226
// shared-memory wavefronts per element) and scales 4 factor pairs per point instead of 13
// products.
#include "sod_internal.cuh"
#include "sod_step_kernels.cuh"
#include <cmath>
#include <algorithm>

namespace sod {
namespace mx2 {

constexpr double kC1 = 0.000001458;
constexpr double kS = 110.4;
constexpr int NA = 6;    // batch A slots (field pairs)
constexpr int NBC = NA + 5;  // batch A + the batch B+C factor slots
constexpr int NP2 = 9;   // pass-2 slots
constexpr int NSLOT = NBC + NP2;
constexpr int NREF = 16 + 36 + 18 + 6;  // node-0 refs, corner values of the batch-A fields, FP32 slopes, 12 FP32 refs

__host__ __device__ constexpr size_t smem_bytes(int epb) {
  return sizeof(double) * (size_t)epb * NREF + sizeof(float2) * (size_t)epb * NSLOT * FSTRIDE;
}

__device__ __forceinline__ float2 F2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 FMA2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 MUL2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 ADD2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// iso derivatives of a field pair: xi-line as two 16-byte loads, eta/zeta lines as 8-byte loads;
// each 4-term line sum as two independent halves (shorter dependency chains)
__device__ __forceinline__ void giso2(const float2* __restrict__ f, int i, int j, int k, const float2* Dx,
                                      const float2* Dy, const float2* Dz, float2& gx, float2& gy, float2& gz) {
  const float2* fx = f + 4 * j + PLANE * k;
  const float4 a01 = *reinterpret_cast<const float4*>(fx);
  const float4 a23 = *reinterpret_cast<const float4*>(fx + 2);
  gx = ADD2(FMA2(Dx[1], make_float2(a01.z, a01.w), MUL2(Dx[0], make_float2(a01.x, a01.y))),
            FMA2(Dx[3], make_float2(a23.z, a23.w), MUL2(Dx[2], make_float2(a23.x, a23.y))));
  const float2* fy = f + i + PLANE * k;
  gy = ADD2(FMA2(Dy[1], fy[4], MUL2(Dy[0], fy[0])), FMA2(Dy[3], fy[12], MUL2(Dy[2], fy[8])));
  const float2* fz = f + i + 4 * j;
  gz = ADD2(FMA2(Dz[1], fz[PLANE], MUL2(Dz[0], fz[0])), FMA2(Dz[3], fz[3 * PLANE], MUL2(Dz[2], fz[2 * PLANE])));
}

// physical gradient component r of a pair: He(r,0) gx + He(r,1) gy + He(r,2) gz
__device__ __forceinline__ float2 physr(const float2* H2, int r, float2 gx, float2 gy, float2 gz) {
  return FMA2(H2[3 * r + 2], gz, FMA2(H2[3 * r + 1], gy, MUL2(H2[3 * r], gx)));
}

// weak divergence of a pair: sum_m D[m][i] fx(m,j,k) + D[m][j] fy(i,m,k) + D[m][k] fz(i,j,m)
__device__ __forceinline__ float2 divT2(const float2* fx, const float2* fy, const float2* fz, int i, int j, int k,
                                        const float2* DTx, const float2* DTy, const float2* DTz) {
  const float2* ax = fx + 4 * j + PLANE * k;
  const float4 a01 = *reinterpret_cast<const float4*>(ax);
  const float4 a23 = *reinterpret_cast<const float4*>(ax + 2);
  float2 s = MUL2(DTx[0], make_float2(a01.x, a01.y));
  s = FMA2(DTx[1], make_float2(a01.z, a01.w), s);
  s = FMA2(DTx[2], make_float2(a23.x, a23.y), s);
  s = FMA2(DTx[3], make_float2(a23.z, a23.w), s);
  const float2* ay = fy + i + PLANE * k;
  float2 t = MUL2(DTy[0], ay[0]);
  t = FMA2(DTy[1], ay[4], t);
  t = FMA2(DTy[2], ay[8], t);
  t = FMA2(DTy[3], ay[12], t);
  const float2* az = fz + i + 4 * j;
  float2 u = MUL2(DTz[0], az[0]);
  u = FMA2(DTz[1], az[PLANE], u);
  u = FMA2(DTz[2], az[2 * PLANE], u);
  u = FMA2(DTz[3], az[3 * PLANE], u);
  return ADD2(ADD2(s, t), u);
}

#ifndef SOD_MX2_MIN_CTAS
#define SOD_MX2_MIN_CTAS 10  // resident 64-thread element groups per SM the register budget must allow
#endif
// One tile of EPB elements (64 threads each); smem_raw holds smem_bytes(EPB).  Every thread of
// the block calls it (it holds block barriers).
// TOTH: flag_total_enthalpy (energy convection of full_convec_ijk_H)
template <int EPB, bool TOTH>
__device__ __forceinline__ void rhs_mixed2_tile(const RhsArgs& a, int tile, unsigned char* smem_raw) {
  double* refs_all = reinterpret_cast<double*>(smem_raw);
  float2* buf_all = reinterpret_cast<float2*>(smem_raw + sizeof(double) * EPB * NREF);
  const int tid = threadIdx.x;
  const int es = tid >> 6;
  const int d = tid & 63;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4;
  const int e = tile * EPB + es;
  const bool active = e < a.nelem;
  const int ee = active ? e : a.nelem - 1;
  double* refs = refs_all + es * NREF;
  float2* buf = buf_all + (size_t)es * NSLOT * FSTRIDE;
  float2* p2 = buf + NBC * FSTRIDE;
  const int s_me = sidx(i, j, k);
  const float* geo = reinterpret_cast<const float*>(a.geo) + (size_t)ee * NGEO * NN;

  float2 Dx[4], Dy[4], Dz[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    Dx[m] = F2(a.Df[i][m]);
    Dy[m] = F2(a.Df[j][m]);
    Dz[m] = F2(a.Df[k][m]);
  }
  float H[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) H[c] = geo[c * NN + d];
  const float gpv = geo[9 * NN + d];
  float2 H2[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) H2[c] = F2(H[c]);

  // ---- own node: stage EOS in FP64 (time_integ.f90:266-285)
  const int32_t n = a.econn[(size_t)ee * NN + d];
  const double g = a.prm.gamma;
  const double rho = a.rho[n];
  const double qv[3] = {a.q0[n], a.q1[n], a.q2[n]};
  const double Et = a.E[n];
  // one FP64 reciprocal serves every division of the EOS (the deviations below need FP64)
  const double irho = 1.0 / rho;
  const double uv[3] = {qv[0] * irho, qv[1] * irho, qv[2] * irho};
  const double umag = uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2];
  const double kk = 0.5 * umag;
  const double e_int = Et * irho - 0.5 * umag;
  const double p = rho * (g - 1.0) * e_int;
  const double h = a.prm.g_gm1 * p * irho;
  const double T = p * irho * a.prm.inv_Rgas;
  const float mufac = (float)a.mu_factor[n];
  const float mue = reinterpret_cast<const float*>(a.mue)[(size_t)ee * NN + d];
  const double musgs = a.musgs ? a.musgs[(size_t)ee * NN + d] : 0.0;

  // element references: FP64 values of local node 0
  if (d == 0) {
    refs[0] = rho; refs[1] = uv[0]; refs[2] = uv[1]; refs[3] = uv[2];
    refs[4] = qv[0]; refs[5] = qv[1]; refs[6] = qv[2]; refs[7] = p; refs[8] = h; refs[9] = kk;
    const double L = log(p) - g * log(rho);
    refs[10] = (rho / (g - 1.0)) * L;
    refs[11] = T;
    refs[12] = L;
    refs[13] = 1.0 / p;
    // FP32 copies of the references, converted once per element
    float* rf = reinterpret_cast<float*>(refs + 16 + 36 + 18);
    rf[0] = (float)rho; rf[1] = (float)uv[0]; rf[2] = (float)uv[1]; rf[3] = (float)uv[2];
    rf[4] = (float)qv[0]; rf[5] = (float)qv[1]; rf[6] = (float)qv[2];
    rf[7] = (float)(h + kk); rf[8] = (float)refs[10]; rf[9] = (float)T;
    rf[10] = (float)(1.0 / rho); rf[11] = (float)refs[13];
  }
  __syncthreads();
  const double r_rho = refs[0], r_p = refs[7], r_h = refs[8], r_k = refs[9], r_T = refs[11],
               r_L = refs[12];
  const double r_u[3] = {refs[1], refs[2], refs[3]};
  const double r_q[3] = {refs[4], refs[5], refs[6]};
  const double s_H = (h - r_h) + (kk - r_k);  // deviation of the total enthalpy H = h + k
  // eta - eta_r = ((rho-rho_r) L_r + rho (L - L_r)) / (gamma-1), L - L_r by log1p of small ratios
  const float drho = (float)(rho - r_rho);
  const float* rf = reinterpret_cast<const float*>(refs + 16 + 36 + 18);  // FP32 references
  const float dpf = (float)(p - r_p);
  const float dL = log1pf(dpf * rf[11]) - a.prm.gamma_f * log1pf(drho * rf[10]);
  const double s_eta = ((double)drho * r_L + rho * (double)dL) * a.prm.inv_gm1;

  // ---- batch A (6 pairs).  The nodal fields differentiated directly (except rho and p, whose
  // rounding does not reach the 1e-7 level of the residuals) get an element reference that is
  // affine in xi: v' = v - sum_d a_d (xi_d + 1), a_d = v(corner_d)/2 (v is the FP64
  // deviation from local node 0, so v = 0 there).  D differentiates linear functions exactly,
  // so D v = D v' + a, and v' (second order in the element size) loses far less to the FP32
  // cast than v.  Product fields (batch B+C) keep the constant node-0 reference, whose exact
  // expansion the discrete product derivative needs.
  const double dev[12] = {rho - r_rho, p - r_p, uv[0] - r_u[0], uv[1] - r_u[1], uv[2] - r_u[2],
                          qv[0] - r_q[0], qv[1] - r_q[1], qv[2] - r_q[2], s_H, rho * s_H, s_eta, T - r_T};
  float vp[12];
  double* crn = refs + 16;  // [dir][12]: values at local nodes (3,0,0), (0,3,0), (0,0,3)
  float2* slopes = reinterpret_cast<float2*>(refs + 16 + 36);  // [dir][6 pairs]: a_dir in FP32
  {
    const int cdir = d == 3 ? 0 : (d == 12 ? 1 : (d == 48 ? 2 : -1));
    if (cdir >= 0) {
#pragma unroll
      for (int f = 0; f < 12; ++f) crn[cdir * 12 + f] = dev[f];
#pragma unroll
      for (int t = 0; t < 6; ++t)
        slopes[cdir * 6 + t] = t == 0 ? make_float2(0.f, 0.f)
                                      : make_float2((float)(0.5 * dev[2 * t]), (float)(0.5 * dev[2 * t + 1]));
    }
  }
  __syncthreads();
  {
    constexpr double kX = 0.44721359549995793928;  // interior GLL nodes of p = 3: +-sqrt(1/5)
    auto xh = [&](int t) {  // (xi_t + 1)/2 of the natural 1-D node order
      return t == 0 ? 0.0 : (t == 1 ? 0.5 * (1.0 - kX) : (t == 2 ? 0.5 * (1.0 + kX) : 1.0));
    };
    const double wx = xh(i), wy = xh(j), wz = xh(k);
    vp[0] = drho;  // rho' and p' keep the constant reference (their rounding is harmless)
    vp[1] = dpf;
#pragma unroll
    for (int f = 2; f < 12; f += 2) {
      const double2 cx = *reinterpret_cast<const double2*>(crn + f);
      const double2 cy = *reinterpret_cast<const double2*>(crn + 12 + f);
      const double2 cz = *reinterpret_cast<const double2*>(crn + 24 + f);
      vp[f] = (float)(dev[f] - (cx.x * wx + cy.x * wy + cz.x * wz));
      vp[f + 1] = (float)(dev[f + 1] - (cx.y * wx + cy.y * wy + cz.y * wz));
    }
#pragma unroll
    for (int t = 0; t < 6; ++t) buf[t * FSTRIDE + s_me] = make_float2(vp[2 * t], vp[2 * t + 1]);
  }
  // FP32 deviations from node 0 = affine deviation + affine part (FP32 FMAs instead of
  // FP64->FP32 conversions, which share the slow XU pipe)
  float su[3], sq[3], sHf, sef, Tf;
  {
    auto xf = [&](int t) {  // xi_t + 1
      return t == 0 ? 0.f : (t == 1 ? 0.55278640450004206f : (t == 2 ? 1.44721359549995794f : 2.f));
    };
    const float2 wx2 = F2(xf(i)), wy2 = F2(xf(j)), wz2 = F2(xf(k));
    float2 lin[6];
#pragma unroll
    for (int t = 1; t < 6; ++t)
      lin[t] = FMA2(slopes[12 + t], wz2, FMA2(slopes[6 + t], wy2, MUL2(slopes[t], wx2)));
    su[0] = vp[2] + lin[1].x; su[1] = vp[3] + lin[1].y; su[2] = vp[4] + lin[2].x;
    sq[0] = vp[5] + lin[2].y; sq[1] = vp[6] + lin[3].x; sq[2] = vp[7] + lin[3].y;
    sHf = vp[8] + lin[4].x;
    sef = vp[10] + lin[5].x;
    Tf = rf[9] + (vp[11] + lin[5].y);
  }
  // factors of the batch B+C products, stored beside batch A: every line point forms its
  // products from them (below), so the element holds 5 factor slots instead of 13 product slots
  buf[(NA + 0) * FSTRIDE + s_me] = make_float2(su[0], su[1]);
  buf[(NA + 1) * FSTRIDE + s_me] = make_float2(su[2], sq[0]);
  buf[(NA + 2) * FSTRIDE + s_me] = make_float2(sq[1], sq[2]);
  buf[(NA + 3) * FSTRIDE + s_me] = make_float2((rf[0] + drho) * sHf, sHf);
  reinterpret_cast<float*>(buf + (NA + 4) * FSTRIDE)[s_me] = sef;
  const float muf = mufac * (float)kC1 * (Tf * sqrtf(Tf)) / (Tf + (float)kS);
  __syncthreads();

  float gradRho[3], gradP[3], gradU[3][3], gradQ[3][3], gradH[3], gradRH[3], gradEta[3], gradT[3];
  {
    float2 gx, gy, gz, o;
#define SOD_PAIR_GRAD(slot, A, B)                                              \
    giso2(buf + (slot) * FSTRIDE, i, j, k, Dx, Dy, Dz, gx, gy, gz);            \
    if ((slot) > 0) {                                                          \
      gx = ADD2(gx, slopes[0 * 6 + (slot)]);                                   \
      gy = ADD2(gy, slopes[1 * 6 + (slot)]);                                   \
      gz = ADD2(gz, slopes[2 * 6 + (slot)]);                                   \
    }                                                                          \
    _Pragma("unroll") for (int r = 0; r < 3; ++r) {                            \
      o = physr(H2, r, gx, gy, gz);                                            \
      A[r] = o.x;                                                              \
      B[r] = o.y;                                                              \
    }
    SOD_PAIR_GRAD(0, gradRho, gradP)
    SOD_PAIR_GRAD(1, gradU[0], gradU[1])
    SOD_PAIR_GRAD(2, gradU[2], gradQ[0])
    SOD_PAIR_GRAD(3, gradQ[1], gradQ[2])
    SOD_PAIR_GRAD(4, gradH, gradRH)
    SOD_PAIR_GRAD(5, gradEta, gradT)
#undef SOD_PAIR_GRAD
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) gradRH[c] += rf[7] * gradRho[c];
  const float divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
  const float divQ = gradQ[0][0] + gradQ[1][1] + gradQ[2][2];
  // node values in FP32 as reference + deviation (float adds instead of FP64->FP32 conversions)
  const float rhoR = rf[0] + drho, HR = rf[7] + sHf;
  const float etaR = rf[8] + sef;
  const float uR[3] = {rf[1] + su[0], rf[2] + su[1], rf[3] + su[2]};
  const float qR[3] = {rf[4] + sq[0], rf[5] + sq[1], rf[6] + sq[2]};
  const float rHR = rhoR * HR;

  // ---- convective terms available after batch A (elem_convec.f90:412-432) + reference parts
  float Rm = 0.5f * (divQ + rhoR * divU);
  float Ren = 0.25f * (HR * divQ + rHR * divU);
  float Rmo[3];
  float Ret = 0.5f * (etaR * divU);
  {
    const float rH = rf[7], re = rf[8];
    Ren += 0.25f * (rH * divQ + rhoR * (rH * divU));
    Ret += 0.5f * (re * divU);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Rmo[c] = 0.25f * (uR[c] * divQ + qR[c] * divU) + gradP[c];
    Rm += 0.5f * (uR[c] * gradRho[c]);
    Ren += 0.25f * (qR[c] * gradH[c] + uR[c] * gradRH[c] + (HR * uR[c]) * gradRho[c]);
    Ret += 0.5f * (uR[c] * gradEta[c]);
    float dF = rf[4 + c] * divU, dFuu = rf[1 + c] * divU;
#pragma unroll
    for (int jd = 0; jd < 3; ++jd) {
      Rmo[c] += 0.25f * ((uR[c] * uR[jd]) * gradRho[jd] + qR[jd] * gradU[c][jd] + uR[jd] * gradQ[c][jd]);
      dF += rf[1 + jd] * gradQ[c][jd];
      dFuu += rf[1 + jd] * gradU[c][jd];
    }
    Rmo[c] += 0.25f * (dF + rhoR * dFuu);
  }

  // ---- diffusion pass 1 (elem_diffu.f90:70-140) -> contravariant flux pairs per direction
  {
    const float mufgp = a.musgs ? muf + (float)(rho * musgs) : muf;
    const float mut = mufgp + mue;
    const float twoThirds = 2.0f / 3.0f;
    float tau[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) tau[r][c] = mut * (gradU[r][c] + gradU[c][r]);
#pragma unroll
    for (int r = 0; r < 3; ++r) tau[r][r] = tau[r][r] - mufgp * twoThirds * divU;
    float tauU[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) tauU[r] = tau[r][0] * uR[0] + tau[r][1] * uR[1] + tau[r][2] * uR[2];
    const float2 g2 = F2(gpv);
    auto emit = [&](int slot0, const float* Va, const float* Vb) {
#pragma unroll
      for (int dir = 0; dir < 3; ++dir) {
        float2 v = MUL2(H2[0 + dir], make_float2(Va[0], Vb[0]));
        v = FMA2(H2[3 + dir], make_float2(Va[1], Vb[1]), v);
        v = FMA2(H2[6 + dir], make_float2(Va[2], Vb[2]), v);
        p2[(slot0 + dir) * FSTRIDE + s_me] = MUL2(g2, v);
      }
    };
    emit(0, gradRho, tauU);
    emit(3, gradT, tau[0]);
    emit(6, tau[1], tau[2]);
  }
  // ---- batch B+C: divergences of the 13 deviation-product pairs
  //   (rho H' u_c, H' u_c) (eta' u_c, q'_0 u'_c) (q'_1 u'_c, q'_2 u'_c) (u'_0 u'_c, u'_1 u'_c) (u'_2 u'_2)
  // with u = u_r + u'.  Each line point m forms its terms D[x][m] a b of the line sums from the
  // factor slots as (D[x][m] a) b (a rounding of the same order as D[x][m] (a b)); per direction
  // the 13 line sums are folded with He at once.
  {
    const float2* f0s = buf + (NA + 0) * FSTRIDE;  // (u'_0, u'_1)
    const float2* f1s = buf + (NA + 1) * FSTRIDE;  // (u'_2, q'_0)
    const float2* f2s = buf + (NA + 2) * FSTRIDE;  // (q'_1, q'_2)
    const float2* f3s = buf + (NA + 3) * FSTRIDE;  // (rho H', H')
    const float* f4s = reinterpret_cast<const float*>(buf + (NA + 4) * FSTRIDE);  // eta' (one float per node)
    const float rU0 = rf[1], rU1 = rf[2], rU2 = rf[3];
    float2 dA = make_float2(0.f, 0.f), dC = dA, dD = dA, dE = dA;
    float dFuu2 = 0.f;
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      float2 g[12];
#pragma unroll
      for (int q = 0; q < 12; ++q) g[q] = make_float2(0.f, 0.f);
      float g12 = 0.f;
      auto point = [&](float2 w, float2 a0, float2 a1, float2 a2, float2 a3, float se) {
        const float su_[3] = {a0.x, a0.y, a1.x};
        const float uR_[3] = {rU0 + a0.x, rU1 + a0.y, rU2 + a1.x};
        // the line weight scales the first factor of each product
        const float2 w3 = MUL2(w, a3), w2 = MUL2(w, a2), w0 = MUL2(w, a0);
        const float2 wsq = MUL2(w, make_float2(se, a1.y));
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          g[c] = FMA2(w3, F2(uR_[c]), g[c]);
          g[3 + c] = FMA2(wsq, make_float2(uR_[c], su_[c]), g[3 + c]);
          g[6 + c] = FMA2(w2, F2(su_[c]), g[6 + c]);
          g[9 + c] = FMA2(w0, F2(su_[c]), g[9 + c]);
        }
        g12 = fmaf(__fmul_rn(w.x, su_[2]), su_[2], g12);
      };
      if (dir == 0) {
        // the xi line of the node: two 16-byte loads per slot
        const int s0 = sidx(0, j, k);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float4 b0 = *reinterpret_cast<const float4*>(f0s + s0 + 2 * h);
          const float4 b1 = *reinterpret_cast<const float4*>(f1s + s0 + 2 * h);
          const float4 b2 = *reinterpret_cast<const float4*>(f2s + s0 + 2 * h);
          const float4 b3 = *reinterpret_cast<const float4*>(f3s + s0 + 2 * h);
          const float2 e4 = *reinterpret_cast<const float2*>(f4s + s0 + 2 * h);  // eta' at both points
          point(Dx[2 * h], make_float2(b0.x, b0.y), make_float2(b1.x, b1.y), make_float2(b2.x, b2.y),
                make_float2(b3.x, b3.y), e4.x);
          point(Dx[2 * h + 1], make_float2(b0.z, b0.w), make_float2(b1.z, b1.w), make_float2(b2.z, b2.w),
                make_float2(b3.z, b3.w), e4.y);
        }
      } else {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int sp = dir == 1 ? sidx(i, m, k) : sidx(i, j, m);
          point(dir == 1 ? Dy[m] : Dz[m], f0s[sp], f1s[sp], f2s[sp], f3s[sp], f4s[sp]);
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 h = H2[3 * c + dir];
        dA = FMA2(h, g[c], dA);
        dC = FMA2(h, g[3 + c], dC);
        dD = FMA2(h, g[6 + c], dD);
        dE = FMA2(h, g[9 + c], dE);
      }
      // row 2 of u' x u' from (Fuu02, Fuu12, Fuu22)
      dFuu2 += H[dir] * g[11].x + H[3 + dir] * g[11].y + H[6 + dir] * g12;
    }
    // dA = (div fe, div fue), dC = (div feta, div F0.), dD = (div F1., div F2.), dE = (div Fuu0., div Fuu1.)
    Ren += 0.25f * (dA.x + rhoR * dA.y);
    Ret += 0.5f * dC.x;
    if constexpr (TOTH) {
      // full_convec_ijk_H (elem_convec.f90:171-177) with E + p = rho H: div(rho H u) =
      // H_r div q + div(rho H' u), and grad(rho H) is gradRH
      Ren = 0.5f * (rf[7] * divQ + dA.x + rHR * divU);
#pragma unroll
      for (int c = 0; c < 3; ++c) Ren += 0.5f * (uR[c] * gradRH[c]);
    }
    Rmo[0] += 0.25f * (dC.y + rhoR * dE.x);
    Rmo[1] += 0.25f * (dD.x + rhoR * dE.y);
    Rmo[2] += 0.25f * (dD.y + rhoR * dFuu2);
  }
  __syncthreads();  // pass-1 fluxes visible

  // ---- diffusion pass 2 (elem_diffu.f90:142-194)
  float2 DTx[4], DTy[4], DTz[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    DTx[m] = F2(a.Df[m][i]);
    DTy[m] = F2(a.Df[m][j]);
    DTz[m] = F2(a.Df[m][k]);
  }
  const float2 vA = divT2(p2 + 0 * FSTRIDE, p2 + 1 * FSTRIDE, p2 + 2 * FSTRIDE, i, j, k, DTx, DTy, DTz);
  const float2 vB = divT2(p2 + 3 * FSTRIDE, p2 + 4 * FSTRIDE, p2 + 5 * FSTRIDE, i, j, k, DTx, DTy, DTz);
  const float2 vC = divT2(p2 + 6 * FSTRIDE, p2 + 7 * FSTRIDE, p2 + 8 * FSTRIDE, i, j, k, DTx, DTy, DTz);
  const float nu_e = a.prm.c_rho_f * mue / rhoR;
  const float CpPr = a.prm.CpPr_f;
  const float kappa_e = muf * CpPr + a.prm.c_ener_f * mue * CpPr + (a.musgs ? a.prm.Cp09_f * rhoR * (float)musgs : 0.f);
  if (active) {
    store_res6<float>(reinterpret_cast<float*>(a.rel), (size_t)e * NN + d, gpv * Rm + nu_e * vA.x,
                      gpv * Rmo[0] + vB.y, gpv * Rmo[1] + vC.x, gpv * Rmo[2] + vC.y,
                      gpv * Ren + (vA.y + kappa_e * vB.x), gpv * Ret);
  }
}

template <int EPB, bool TOTH>
__global__ void __launch_bounds__(64 * EPB, (EPB >= SOD_MX2_MIN_CTAS ? 1 : SOD_MX2_MIN_CTAS / EPB))
    k_rhs_mixed2(const RhsArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  rhs_mixed2_tile<EPB, TOTH>(a, blockIdx.x, smem_raw);
}

// One RK stage of the mixed path in one cooperative launch (persistent blocks): the fused RHS
// over element tiles, then persist_stage_tail (gather / stage update; at stage 4 the entropy
// viscosity and dt).
template <int EPB, bool TOTH>
__global__ void __launch_bounds__(64 * EPB, (EPB >= SOD_MX2_MIN_CTAS ? 1 : SOD_MX2_MIN_CTAS / EPB))
    k_stage_mixed2(const StageArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ntiles = (p.r.nelem + EPB - 1) / EPB;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    rhs_mixed2_tile<EPB, TOTH>(p.r, t, smem_raw);
    __syncthreads();  // the next tile reuses the shared memory
  }
  persist_stage_tail<float, EPB>(p, smem_raw);
}

template <int EPB>
static int set_attr() {
  SOD_CUDA(cudaFuncSetAttribute(k_rhs_mixed2<EPB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_bytes(EPB)));
  SOD_CUDA(cudaFuncSetAttribute(k_rhs_mixed2<EPB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_bytes(EPB)));
  SOD_CUDA(cudaFuncSetAttribute(k_stage_mixed2<EPB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_bytes(EPB)));
  SOD_CUDA(cudaFuncSetAttribute(k_stage_mixed2<EPB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_bytes(EPB)));
  return SOD_OK;
}

// Cooperative launch of one persistent stage; ctas_per_sm <= 0 asks for the most that fit.
template <int EPB>
static int launch_stage(const StageArgs& p, int ctas_per_sm, int* grid_out, cudaStream_t st) {
  const bool toth = p.r.prm.total_enthalpy != 0;
  const void* fn = toth ? (const void*)k_stage_mixed2<EPB, true> : (const void*)k_stage_mixed2<EPB, false>;
  int occ = 0, dev = 0, nsm = 0;
  SOD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 64 * EPB, smem_bytes(EPB)));
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
  cfg.dynamicSmemBytes = smem_bytes(EPB);
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

template <int EPB>
static int launch(const RhsArgs& a, cudaStream_t st) {
  const int grid = (a.nelem + EPB - 1) / EPB;
  if (a.prm.total_enthalpy)
    k_rhs_mixed2<EPB, true><<<grid, 64 * EPB, smem_bytes(EPB), st>>>(a);
  else
    k_rhs_mixed2<EPB, false><<<grid, 64 * EPB, smem_bytes(EPB), st>>>(a);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

}  // namespace mx2

int init_rhs_mixed2_attrs() {
  static bool done = false;
  if (done) return SOD_OK;
  if (mx2::set_attr<1>() || mx2::set_attr<2>() || mx2::set_attr<4>() || mx2::set_attr<8>()) return SOD_ERR_CUDA;
  done = true;
  return SOD_OK;
}

void stage_mixed2_info(int epb, bool toth, const void** fn, size_t* smem) {
  switch (epb) {
    case 1: *fn = toth ? (const void*)mx2::k_stage_mixed2<1, true> : (const void*)mx2::k_stage_mixed2<1, false>; break;
    case 2: *fn = toth ? (const void*)mx2::k_stage_mixed2<2, true> : (const void*)mx2::k_stage_mixed2<2, false>; break;
    case 8: *fn = toth ? (const void*)mx2::k_stage_mixed2<8, true> : (const void*)mx2::k_stage_mixed2<8, false>; break;
    default: *fn = toth ? (const void*)mx2::k_stage_mixed2<4, true> : (const void*)mx2::k_stage_mixed2<4, false>; epb = 4;
  }
  *smem = mx2::smem_bytes(epb);
}

int launch_stage_mixed2(const StageArgs& p, int epb, int ctas_per_sm, int* grid_out, cudaStream_t st) {
  switch (epb) {
    case 1: return mx2::launch_stage<1>(p, ctas_per_sm, grid_out, st);
    case 2: return mx2::launch_stage<2>(p, ctas_per_sm, grid_out, st);
    case 8: return mx2::launch_stage<8>(p, ctas_per_sm, grid_out, st);
    default: return mx2::launch_stage<4>(p, ctas_per_sm, grid_out, st);
  }
}

int launch_rhs_mixed2(const RhsArgs& a, int epb, cudaStream_t st) {
  switch (epb) {
    case 1: return mx2::launch<1>(a, st);
    case 2: return mx2::launch<2>(a, st);
    case 8: return mx2::launch<8>(a, st);
    default: return mx2::launch<4>(a, st);
  }
}

}  // namespace sod
