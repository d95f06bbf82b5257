// Taylor-Green diagnostics on the device: volAvg_EK and visc_dissipationRate
// (mod_analysis.f90:10-144), called by the time loop every few steps (CFDSolverBase.f90:1413-1414,
// 1580-1581) to follow EK(t) and the dissipation rates eps_S (solenoidal, with mu_e), eps_D
// (dilatational) and eps_T = eps_S + eps_D.
//
// One kernel over elements (4 per CTA, one thread per gauss point): the velocity is staged in
// shared memory, its gradient taken with the same line derivatives and He as the RHS, and the
// three integrands and the volume summed per CTA; a one-block kernel adds the CTA partials in a fixed order
// (FP64), so the results do not depend on scheduling.  The reference's constants are kept:
// EK is divided by rho0 (2 * 3.14159)^3, the rates by rho0 * volT.
#include "sod_internal.cuh"

namespace sod {
namespace diag {

constexpr int EPB = 4;

__global__ void __launch_bounds__(64 * EPB) k_diag_elem(int nelem, const int32_t* __restrict__ econn,
                                                       const double* __restrict__ geo, const double* __restrict__ mue,
                                                       const double* __restrict__ rho, const double* __restrict__ u0,
                                                       const double* __restrict__ u1, const double* __restrict__ u2,
                                                       const double* __restrict__ mu_fluid, const DMat D,
                                                       double* __restrict__ partial) {
  __shared__ double us[EPB][3][FSTRIDE];
  __shared__ double red[64 * EPB / 32][4];
  const int es = threadIdx.x >> 6, d = threadIdx.x & 63;
  const int e = blockIdx.x * EPB + es;
  const bool act = e < nelem;
  const int ee = act ? e : nelem - 1;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  const int n = econn[(size_t)ee * NN + d];
  const double uv[3] = {u0[n], u1[n], u2[n]};
#pragma unroll
  for (int c = 0; c < 3; ++c) us[es][c][s] = uv[c];
  const double* G = geo + (size_t)ee * NGEO * NN;
  double H[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) H[c] = G[c * NN + d];
  const double gpv = G[9 * NN + d];
  __syncthreads();
  // gu[c][r] = d u_c / d x_r
  double gu[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double* f = us[es][c];
    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int m = 0; m < NP1; ++m) {
      gx += D.d[i][m] * f[sidx(m, j, k)];
      gy += D.d[j][m] * f[sidx(i, m, k)];
      gz += D.d[k][m] * f[sidx(i, j, m)];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) gu[c][r] = H[3 * r] * gx + H[3 * r + 1] * gy + H[3 * r + 2] * gz;
  }
  const double divu = gu[0][0] + gu[1][1] + gu[2][2];
  // curl u: (d_y u_z - d_z u_y, d_z u_x - d_x u_z, d_x u_y - d_y u_x)
  const double w0 = gu[2][1] - gu[1][2], w1 = gu[0][2] - gu[2][0], w2 = gu[1][0] - gu[0][1];
  const double mf = mu_fluid[n];
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (act) {
    v[0] = gpv * 0.5 * rho[n] * (uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2]);
    v[1] = gpv * (mf + mue[(size_t)e * NN + d]) * (w0 * w0 + w1 * w1 + w2 * w2);
    v[2] = gpv * mf * (divu * divu);
    v[3] = gpv;  // domain volume (CFDSolverBase.f90:1300-1312 sums gpvol the same way)
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) red[w][q] = v[q];
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0.0;
    for (int q = 0; q < 64 * EPB / 32; ++q) t += red[q][threadIdx.x];
    partial[(size_t)blockIdx.x * 4 + threadIdx.x] = t;
  }
}

// out = {EK, eps_S, eps_D, eps_T, volT used}; volT <= 0 selects the summed gpvol
__global__ void k_diag_final(int nblk, const double* __restrict__ partial, double ek_scale, double rho0,
                             double volT, double* __restrict__ out) {
  __shared__ double sh[4][256];
  const int t = threadIdx.x;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = t; b < nblk; b += 256)
    for (int q = 0; q < 4; ++q) a[q] += partial[(size_t)b * 4 + q];
  for (int q = 0; q < 4; ++q) sh[q][t] = a[q];
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h)
      for (int q = 0; q < 4; ++q) sh[q][t] += sh[q][t + h];
    __syncthreads();
  }
  if (t == 0) {
    const double vol = volT > 0.0 ? volT : sh[3][0];
    const double alpha = 1.0 / (rho0 * vol);
    const double eS = sh[1][0] * alpha, eD = (4.0 / 3.0) * sh[2][0] * alpha;
    out[0] = sh[0][0] * ek_scale;
    out[1] = eS;
    out[2] = eD;
    out[3] = eS + eD;
    out[4] = vol;
  }
}

// compute_fieldDerivs (mod_postpro.f90:12-139), element part: per gauss point the physical
// gradient of rho, the reference's curl sum_jk leviCivi(i,j,k) du_j/dx_k, the split divergence
// (div(rho u) + rho div u) / 2 and Q = -1/2 du_i/dx_j du_j/dx_i, written per element node
// [(e*64 + d)*8]: grad rho x3, curl x3, div, Q.  The nodal average over the elements holding a
// node (the reference's atomics, then / lelpn) is the ordered gather below.
struct Levi {
  double e[27];  // leviCivi(i,j,k) at i + 3j + 9k
};

__global__ void __launch_bounds__(64 * EPB) k_fderiv_elem(int nelem, const int32_t* __restrict__ econn,
                                                         const double* __restrict__ geo, const double* __restrict__ rho,
                                                         const double* __restrict__ u0, const double* __restrict__ u1,
                                                         const double* __restrict__ u2, const DMat D, const Levi L,
                                                         double* __restrict__ out) {
  __shared__ double fs[EPB][7][FSTRIDE];  // rho, u x3, rho u x3
  const int es = threadIdx.x >> 6, d = threadIdx.x & 63;
  const int e = blockIdx.x * EPB + es;
  const bool act = e < nelem;
  const int ee = act ? e : nelem - 1;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  const int n = econn[(size_t)ee * NN + d];
  const double r = rho[n];
  const double uv[3] = {u0[n], u1[n], u2[n]};
  fs[es][0][s] = r;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    fs[es][1 + c][s] = uv[c];
    fs[es][4 + c][s] = r * uv[c];
  }
  const double* G = geo + (size_t)ee * NGEO * NN;
  double H[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) H[c] = G[c * NN + d];
  __syncthreads();
  double ph[7][3];  // physical gradient of each staged field: ph[f][r] = d f / d x_r
#pragma unroll
  for (int f = 0; f < 7; ++f) {
    const double* v = fs[es][f];
    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int m = 0; m < NP1; ++m) {
      gx += D.d[i][m] * v[sidx(m, j, k)];
      gy += D.d[j][m] * v[sidx(i, m, k)];
      gz += D.d[k][m] * v[sidx(i, j, m)];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) ph[f][q] = H[3 * q] * gx + H[3 * q + 1] * gy + H[3 * q + 2] * gz;
  }
  if (!act) return;
  double o[8];
#pragma unroll
  for (int q = 0; q < 3; ++q) o[q] = ph[0][q];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double c = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) c += L.e[a + 3 * b + 9 * cc] * ph[1 + b][cc];
    o[3 + a] = c;
  }
  const double divq = ph[4][0] + ph[5][1] + ph[6][2];
  const double divu = ph[1][0] + ph[2][1] + ph[3][2];
  o[6] = 0.5 * (divq + r * divu);
  double qc = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) qc -= 0.5 * (ph[1 + a][b] * ph[1 + b][a]);
  o[7] = qc;
  double4* dst = reinterpret_cast<double4*>(out + ((size_t)e * NN + d) * 8);
  dst[0] = make_double4(o[0], o[1], o[2], o[3]);
  dst[1] = make_double4(o[4], o[5], o[6], o[7]);
}

// nodal average of the element values in ascending element order (deterministic)
__global__ void __launch_bounds__(256) k_fderiv_gather(int npoin, const int32_t* __restrict__ ptr,
                                                       const int32_t* __restrict__ idx, const double* __restrict__ el,
                                                       double* __restrict__ gradRho, double* __restrict__ curlU,
                                                       double* __restrict__ divU, double* __restrict__ Qcrit) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int beg = ptr[n], end = ptr[n + 1];
  for (int c = beg; c < end; ++c) {
    const double4* v = reinterpret_cast<const double4*>(el + (size_t)idx[c] * 8);
    const double4 x = v[0], y = v[1];
    a[0] += x.x; a[1] += x.y; a[2] += x.z; a[3] += x.w;
    a[4] += y.x; a[5] += y.y; a[6] += y.z; a[7] += y.w;
  }
  // lelpn; a row without elements (a periodic slave, outside lpoin_w) keeps the zero the
  // reference's outputs start from (mod_postpro.f90:28-32,127-136)
  const double cnt = end > beg ? (double)(end - beg) : 1.0;
  const size_t N = (size_t)npoin;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    gradRho[n + N * q] = a[q] / cnt;
    curlU[n + N * q] = a[3 + q] / cnt;
  }
  divU[n] = a[6] / cnt;
  Qcrit[n] = a[7] / cnt;
}

}  // namespace diag
}  // namespace sod

using namespace sod;

extern "C" {

int sod_tgv_diagnostics(SodMesh* m, const double* rho, const double* u, const double* mu_fluid,
                        const double* mu_e, double rho0, double volT, double* out_dev, sod_stream_t stream) {
  SOD_ARG(m && rho && u && mu_fluid && mu_e && out_dev, "null argument");
  SOD_ARG(rho0 > 0.0, "rho0 must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, mu_e, m->mue_int, st);
  if (rc) return rc;
  const int nblk = (m->nelem + diag::EPB - 1) / diag::EPB;
  SOD_ARG(m->buf.red_cap >= 4 * (int64_t)nblk, "reduction scratch too small");
  const size_t N = m->npoin;
  diag::k_diag_elem<<<nblk, 64 * diag::EPB, 0, st>>>(m->nelem, m->econn, m->geo64, m->mue_int, rho, u, u + N,
                                                    u + 2 * N, mu_fluid, m->D, m->buf.red);
  SOD_CHECK_LAUNCH();
  const double two_pi = 2.0 * 3.14159;  // the reference's constant (mod_analysis.f90:36)
  const double ek_scale = 1.0 / (rho0 * (two_pi * two_pi * two_pi));
  diag::k_diag_final<<<1, 256, 0, st>>>(nblk, m->buf.red, ek_scale, rho0, volT, out_dev);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int sod_compute_field_derivs(SodMesh* m, const double* rho, const double* u, const double* leviCivi,
                             double* gradRho, double* curlU, double* divU, double* Qcrit, sod_stream_t stream) {
  SOD_ARG(m && rho && u && gradRho && curlU && divU && Qcrit, "null argument");
  SOD_ARG(m->nmember == 0, "field derivatives of an ensemble mesh are not supported");
  cudaStream_t st = (cudaStream_t)stream;
  diag::Levi L{};
  if (leviCivi) {
    for (int q = 0; q < 27; ++q) L.e[q] = leviCivi[q];
  } else {  // CFDSolverBase.f90:1248-1253
    L.e[1 + 3 * 2 + 9 * 0] = 1.0;  L.e[2 + 3 * 1 + 9 * 0] = -1.0;
    L.e[0 + 3 * 2 + 9 * 1] = -1.0; L.e[2 + 3 * 0 + 9 * 1] = 1.0;
    L.e[0 + 3 * 1 + 9 * 2] = 1.0;  L.e[1 + 3 * 0 + 9 * 2] = -1.0;
  }
  const size_t need = (size_t)m->nelem * NN * 8;
  if (m->postpro_len < need) {
    if (m->postpro) cudaFree(m->postpro);
    m->postpro = nullptr;
    m->postpro_len = 0;
    if (cudaMalloc(&m->postpro, need * sizeof(double)) != cudaSuccess) {
      set_error("sod_compute_field_derivs: device allocation failed");
      return SOD_ERR_NOMEM;
    }
    m->postpro_len = need;
  }
  const size_t N = m->npoin;
  const int nblk = (m->nelem + diag::EPB - 1) / diag::EPB;
  diag::k_fderiv_elem<<<nblk, 64 * diag::EPB, 0, st>>>(m->nelem, m->econn, m->geo64, rho, u, u + N, u + 2 * N, m->D,
                                                      L, m->postpro);
  SOD_CHECK_LAUNCH();
  diag::k_fderiv_gather<<<(m->npoin + 255) / 256, 256, 0, st>>>(m->npoin, m->n2e_ptr, m->n2e, m->postpro, gradRho,
                                                                curlU, divU, Qcrit);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

}  // extern "C"
