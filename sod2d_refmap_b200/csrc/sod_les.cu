// LES eddy viscosity (Vreman): sgs_visc (mod_sgs_viscosity.f90:13-125) on the device.
//
// Per element (4 per CTA, one thread per gauss point): the velocity is staged in shared memory
// and differentiated with the same line derivatives and He as the RHS; with hLES = gpvol^(1/3),
// alpha = |grad u|^2 and beta = hLES^2 grad u^T grad u, the point value is
// c_sgs sqrt(max(B(beta), 1e-10) / alpha) where alpha > 1e-10 (B = sum of the principal 2x2
// minors), else the previous mu_sgs; the 3x3x3 convertIJK filter of the entropy viscosity then
// smooths it inside the element.  Element-local, so the update of musgs_int is in place.
#include "sod_internal.cuh"

namespace sod {
namespace les {

constexpr int EPB = 4;

__device__ __forceinline__ int nb_filter(int x) {  // natural index of convertIJK(x+1)
  return (x < 0) ? 1 : ((x > 3) ? 1 : x);
}

__global__ void __launch_bounds__(64 * EPB) k_sgs(int nelem, const int32_t* __restrict__ econn,
                                                 const double* __restrict__ geo, const double* __restrict__ u0,
                                                 const double* __restrict__ u1, const double* __restrict__ u2,
                                                 const DMat D, double c_sgs, double* __restrict__ musgs) {
  __shared__ double us[EPB][3][FSTRIDE];
  __shared__ double ml[EPB][NN];
  const int es = threadIdx.x >> 6, d = threadIdx.x & 63;
  const int e = blockIdx.x * EPB + es;
  const bool act = e < nelem;
  const int ee = act ? e : nelem - 1;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  const int n = econn[(size_t)ee * NN + d];
  us[es][0][s] = u0[n];
  us[es][1][s] = u1[n];
  us[es][2][s] = u2[n];
  const double* G = geo + (size_t)ee * NGEO * NN;
  double H[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) H[c] = G[c * NN + d];
  const double gpv = G[9 * NN + d];
  const double old = musgs[(size_t)ee * NN + d];
  __syncthreads();
  double gu[3][3];  // gu[c][r] = d u_c / d x_r
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
  const double hLES = cbrt(gpv);
  double alpha = 0.0, V[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      V[a][b] = (gu[0][a] * gu[0][b] + gu[1][a] * gu[1][b] + gu[2][a] * gu[2][b]) * (hLES * hLES);
      alpha += gu[a][b] * gu[a][b];
    }
  const double B = V[0][0] * V[1][1] + V[0][0] * V[2][2] + V[1][1] * V[2][2] - V[0][1] * V[0][1] -
                   V[0][2] * V[0][2] - V[1][2] * V[1][2];
  ml[es][d] = alpha > 1.0e-10 ? c_sgs * sqrt(fmax(B, 1.0e-10) / alpha) : old;
  __syncthreads();
  const int ix[3] = {nb_filter(i - 1), i, nb_filter(i + 1)};
  const int jx[3] = {nb_filter(j - 1), j, nb_filter(j + 1)};
  const int kx[3] = {nb_filter(k - 1), k, nb_filter(k + 1)};
  const double w[3] = {0.25, 0.5, 0.25};
  double acc = 0.0;
#pragma unroll
  for (int l = 0; l < 3; ++l)
#pragma unroll
    for (int mm = 0; mm < 3; ++mm)
#pragma unroll
      for (int nn = 0; nn < 3; ++nn) acc = acc + w[l] * w[mm] * w[nn] * ml[es][ix[l] + 4 * jx[mm] + 16 * kx[nn]];
  if (act) musgs[(size_t)e * NN + d] = acc;
}

}  // namespace les

int launch_sgs(SodMesh* m, const double* u, cudaStream_t st) {
  const size_t N = m->npoin;
  const int grid = (m->nelem + les::EPB - 1) / les::EPB;
  les::k_sgs<<<grid, 64 * les::EPB, 0, st>>>(m->nelem, m->econn, m->geo64, u, u + N, u + 2 * N, m->D, m->prm.c_sgs,
                                             m->musgs_int);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

}  // namespace sod
