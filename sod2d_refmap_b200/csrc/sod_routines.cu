// Per-routine entry points with the reference argument lists (sm_100a).  Each keeps the
// reference's inputs independent (e.g. full_convec_ijk takes u and q separately, and the
// energy-like field E as given) and writes fully overwritten nodal outputs.  Element work
// runs one CTA per element (64 threads = gauss points) in FP64, assembly is the same ordered
// CSR gather as the fused path.
#include "sod_internal.cuh"
#include <cmath>

namespace sod {

int launch_visc_dt(SodMesh* m, const SodState* s, double* dt_out, float* mue32, cudaStream_t st);

__device__ __forceinline__ void giso_d(const double* f, int i, int j, int k, const double (&D)[NP1][NP1],
                                       double& gx, double& gy, double& gz) {
  gx = gy = gz = 0.0;
#pragma unroll
  for (int m = 0; m < NP1; ++m) {
    gx += D[i][m] * f[sidx(m, j, k)];
    gy += D[j][m] * f[sidx(i, m, k)];
    gz += D[k][m] * f[sidx(i, j, m)];
  }
}
__device__ __forceinline__ double divT_d(const double* fx, const double* fy, const double* fz, int i, int j, int k,
                                         const double (&D)[NP1][NP1]) {
  double s = 0.0;
#pragma unroll
  for (int m = 0; m < NP1; ++m)
    s += D[m][i] * fx[sidx(m, j, k)] + D[m][j] * fy[sidx(i, m, k)] + D[m][k] * fz[sidx(i, j, m)];
  return s;
}

struct RefArgs {
  int nelem;
  int64_t npoin;
  const int32_t* econn;
  const double* geo;
  DMat D;
  const double *u, *q, *rho, *pr, *E;          // convec / scalar
  const double *rho_n, *Tem, *mu_fluid;         // diffusion
  const double *mue, *musgs;                    // internal layout [e][64]
  double Cp, Pr, c_rho, c_ener;
  double* rel;                                  // [e][6][64]
};

// full_convec_ijk (elem_convec.f90:241-435); TOTH: full_convec_ijk_H (elem_convec.f90:48-187),
// whose energy residual is 0.5 (div((E + p) u) + (E + p) div u + u . grad(E + p)) with E the
// total energy; mass and momentum are the same in both
template <bool TOTH>
__global__ void __launch_bounds__(64) k_convec_ref(const RefArgs a) {
  __shared__ double f[42][FSTRIDE];
  __shared__ DMat Ds;
  const int e = blockIdx.x, d = threadIdx.x;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  if (d < 16) Ds.d[d >> 2][d & 3] = a.D.d[d >> 2][d & 3];
  const int n = a.econn[(int64_t)e * NN + d];
  const int64_t N = a.npoin;
  double u[3], q[3];
  for (int c = 0; c < 3; ++c) { u[c] = a.u[n + N * c]; q[c] = a.q[n + N * c]; }
  const double rho = a.rho[n], El = a.E[n], pr = a.pr[n];
  double kl = 0.0;
  for (int c = 0; c < 3; ++c) kl = kl + u[c] * u[c] * 0.5;
  // fields: 0 rho,1 p,2 E,3 rhoE,4 k,5 rhok, 6-8 u, 9-11 q, 12-14 fe, 15-17 fue, 18-20 fk, 21-23 fuk,
  //         24-32 F=q x u, 33-41 Fuu = u x u
  // TOTH: field 2 holds p + E and fields 12-14 (E + p) u
  f[0][s] = rho; f[1][s] = pr; f[2][s] = TOTH ? pr + El : El; f[3][s] = rho * El; f[4][s] = kl; f[5][s] = rho * kl;
  for (int c = 0; c < 3; ++c) {
    f[6 + c][s] = u[c]; f[9 + c][s] = q[c];
    f[12 + c][s] = TOTH ? (El + pr) * u[c] : rho * El * u[c]; f[15 + c][s] = El * u[c];
    f[18 + c][s] = rho * kl * u[c]; f[21 + c][s] = kl * u[c];
    for (int c2 = 0; c2 < 3; ++c2) { f[24 + 3 * c + c2][s] = q[c] * u[c2]; f[33 + 3 * c + c2][s] = u[c] * u[c2]; }
  }
  __syncthreads();
  const double* G = a.geo + (int64_t)e * NGEO * NN;
  double H[9];
  for (int c = 0; c < 9; ++c) H[c] = G[c * NN + d];
  const double gpv = G[9 * NN + d];
  auto grad = [&](int fi, double* o) {
    double gx, gy, gz;
    giso_d(f[fi], i, j, k, Ds.d, gx, gy, gz);
    for (int r = 0; r < 3; ++r) o[r] = H[3 * r] * gx + H[3 * r + 1] * gy + H[3 * r + 2] * gz;
  };
  double gRho[3], gP[3], gE[3], gRE[3], gk[3], gRk[3], gU[3][3], gQ[3][3];
  grad(0, gRho); grad(1, gP); grad(2, gE); grad(3, gRE); grad(4, gk); grad(5, gRk);
  for (int c = 0; c < 3; ++c) { grad(6 + c, gU[c]); grad(9 + c, gQ[c]); }
  auto divg = [&](int fi) {
    double sdiv = 0.0;
    for (int c = 0; c < 3; ++c) { double g3[3]; grad(fi + c, g3); sdiv += g3[c]; }
    return sdiv;
  };
  const double divFe = divg(12), divFue = divg(15), divFk = divg(18), divFuk = divg(21);
  double divF[3], divFuu[3];
  for (int c = 0; c < 3; ++c) { divF[c] = divg(24 + 3 * c); divFuu[c] = divg(33 + 3 * c); }
  const double divU = gU[0][0] + gU[1][1] + gU[2][2];
  const double divQ = gQ[0][0] + gQ[1][1] + gQ[2][2];
  double Rm = 0.5 * (divQ + rho * divU);
  double Re = TOTH ? 0.5 * (divFe + (El + pr) * divU)
                   : 0.25 * (divFe + El * divQ + rho * El * divU + rho * divFue) +
                         0.25 * (divFk + kl * divQ + rho * kl * divU + rho * divFuk);
  double Rmo[3];
  for (int c = 0; c < 3; ++c) {
    Rmo[c] = 0.25 * (divF[c] + u[c] * divQ + q[c] * divU + rho * divFuu[c]) + gP[c];
    Rm = Rm + 0.5 * (u[c] * gRho[c]);
    if (TOTH)
      Re = Re + 0.5 * (u[c] * gE[c]);
    else
      Re = Re + 0.25 * (q[c] * gE[c] + u[c] * gRE[c] + El * u[c] * gRho[c]) +
           0.25 * (q[c] * gk[c] + u[c] * gRk[c] + kl * u[c] * gRho[c]);
    for (int c2 = 0; c2 < 3; ++c2) Rmo[c] = Rmo[c] + 0.25 * (u[c] * u[c2] * gRho[c2] + q[c2] * gU[c][c2] + u[c2] * gQ[c][c2]);
  }
  double* out = a.rel + (int64_t)e * NRES * NN + d;
  out[0] = gpv * Rm; out[NN] = gpv * Rmo[0]; out[2 * NN] = gpv * Rmo[1]; out[3 * NN] = gpv * Rmo[2];
  out[4 * NN] = gpv * Re; out[5 * NN] = 0.0;
}

// generic_scalar_convec_ijk (elem_convec.f90:488-556)
__global__ void __launch_bounds__(64) k_scalar_ref(const RefArgs a) {
  __shared__ double f[7][FSTRIDE];
  __shared__ DMat Ds;
  const int e = blockIdx.x, d = threadIdx.x;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  if (d < 16) Ds.d[d >> 2][d & 3] = a.D.d[d >> 2][d & 3];
  const int n = a.econn[(int64_t)e * NN + d];
  const int64_t N = a.npoin;
  double u[3];
  for (int c = 0; c < 3; ++c) { u[c] = a.u[n + N * c]; f[1 + c][s] = u[c]; f[4 + c][s] = a.q[n + N * c]; }
  const double eta = a.E[n];
  f[0][s] = eta;
  __syncthreads();
  const double* G = a.geo + (int64_t)e * NGEO * NN;
  double H[9];
  for (int c = 0; c < 9; ++c) H[c] = G[c * NN + d];
  double gx, gy, gz, gE[3], divU = 0.0, divFe = 0.0;
  giso_d(f[0], i, j, k, Ds.d, gx, gy, gz);
  for (int r = 0; r < 3; ++r) gE[r] = H[3 * r] * gx + H[3 * r + 1] * gy + H[3 * r + 2] * gz;
  for (int c = 0; c < 3; ++c) {
    giso_d(f[1 + c], i, j, k, Ds.d, gx, gy, gz);
    divU += H[3 * c] * gx + H[3 * c + 1] * gy + H[3 * c + 2] * gz;
    giso_d(f[4 + c], i, j, k, Ds.d, gx, gy, gz);
    divFe += H[3 * c] * gx + H[3 * c + 1] * gy + H[3 * c + 2] * gz;
  }
  double Re = 0.5 * (divFe + eta * divU);
  for (int c = 0; c < 3; ++c) Re = Re + 0.5 * (u[c] * gE[c]);
  double* out = a.rel + (int64_t)e * NRES * NN + d;
  for (int fld = 0; fld < 5; ++fld) out[fld * NN] = 0.0;
  out[5 * NN] = G[9 * NN + d] * Re;
}

// full_diffusion_ijk (elem_diffu.f90:44-194)
__global__ void __launch_bounds__(64) k_diffusion_ref(const RefArgs a) {
  __shared__ double f[5][FSTRIDE];
  __shared__ double V[18][FSTRIDE];
  __shared__ DMat Ds;
  const int e = blockIdx.x, d = threadIdx.x;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  if (d < 16) Ds.d[d >> 2][d & 3] = a.D.d[d >> 2][d & 3];
  const int n = a.econn[(int64_t)e * NN + d];
  const int64_t N = a.npoin;
  double u[3];
  for (int c = 0; c < 3; ++c) { u[c] = a.u[n + N * c]; f[2 + c][s] = u[c]; }
  f[0][s] = a.rho[n];
  f[1][s] = a.Tem[n];
  const double rhon = a.rho_n[n], muf = a.mu_fluid[n];
  const double mue = a.mue[(int64_t)e * NN + d];
  const double musgs = a.musgs ? a.musgs[(int64_t)e * NN + d] : 0.0;
  __syncthreads();
  const double* G = a.geo + (int64_t)e * NGEO * NN;
  double H[9];
  for (int c = 0; c < 9; ++c) H[c] = G[c * NN + d];
  const double gpv = G[9 * NN + d];
  double gx, gy, gz, gRho[3], gT[3], gU[3][3];
  giso_d(f[0], i, j, k, Ds.d, gx, gy, gz);
  for (int r = 0; r < 3; ++r) gRho[r] = H[3 * r] * gx + H[3 * r + 1] * gy + H[3 * r + 2] * gz;
  giso_d(f[1], i, j, k, Ds.d, gx, gy, gz);
  for (int r = 0; r < 3; ++r) gT[r] = H[3 * r] * gx + H[3 * r + 1] * gy + H[3 * r + 2] * gz;
  for (int c = 0; c < 3; ++c) {
    giso_d(f[2 + c], i, j, k, Ds.d, gx, gy, gz);
    for (int r = 0; r < 3; ++r) gU[c][r] = H[3 * r] * gx + H[3 * r + 1] * gy + H[3 * r + 2] * gz;
  }
  const double divU = gU[0][0] + gU[1][1] + gU[2][2];
  const double mu_fgp = muf + rhon * musgs, mu_egp = mue;
  const double twoThirds = 2.0 / 3.0;
  double tau[3][3], tauU[3];
  for (int r = 0; r < 3; ++r) {
    tauU[r] = 0.0;
    for (int c = 0; c < 3; ++c) {
      tauU[r] = tauU[r] + (mu_fgp + mu_egp) * (gU[r][c] + gU[c][r]) * u[c];
      tau[r][c] = (mu_fgp + mu_egp) * (gU[r][c] + gU[c][r]);
    }
    tauU[r] = tauU[r] - mu_fgp * twoThirds * divU * u[r];
    tau[r][r] = tau[r][r] - mu_fgp * twoThirds * divU;
  }
  const double* Vs[6] = {gRho, tauU, gT, tau[0], tau[1], tau[2]};
  for (int v = 0; v < 6; ++v)
    for (int dir = 0; dir < 3; ++dir)
      V[3 * v + dir][s] = gpv * (H[dir] * Vs[v][0] + H[3 + dir] * Vs[v][1] + H[6 + dir] * Vs[v][2]);
  __syncthreads();
  double dv[6];
  for (int v = 0; v < 6; ++v) dv[v] = divT_d(V[3 * v], V[3 * v + 1], V[3 * v + 2], i, j, k, Ds.d);
  const double nu_e = a.c_rho * mue / rhon;
  const double kappa_e = muf * a.Cp / a.Pr + a.c_ener * mue * a.Cp / a.Pr + a.Cp * rhon * musgs / 0.9;
  double* out = a.rel + (int64_t)e * NRES * NN + d;
  out[0] = nu_e * dv[0];
  out[NN] = dv[3]; out[2 * NN] = dv[4]; out[3 * NN] = dv[5];
  out[4 * NN] = dv[1] + kappa_e * dv[2];
  out[5 * NN] = 0.0;
}

// ordered gather of selected residual fields, optional /Ml
__global__ void k_gather_plain(int npoin, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                               const double* __restrict__ rel, const double* __restrict__ Ml, int f0, int nf,
                               double* o0, double* o1, double* o2, double* o3, double* o4) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  double r[5] = {0, 0, 0, 0, 0};
  for (int c = ptr[n]; c < ptr[n + 1]; ++c) {
    const int pk = idx[c];
    const double* src = rel + (int64_t)(pk >> 6) * NRES * NN + (pk & 63);
    for (int f = 0; f < nf; ++f) r[f] += src[(f0 + f) * NN];
  }
  double* outs[5] = {o0, o1, o2, o3, o4};
  for (int f = 0; f < nf; ++f) {
    double v = Ml ? r[f] / Ml[n] : r[f];
    if (outs[f]) outs[f][n] = v;
  }
}

// lumped_solver_scal/vect over the working nodes (mod_solver.f90:23-58): rows without elements
// (periodic slaves, absent from lpoin_w) are left as they are
__global__ void k_lumped(int64_t npoin, int ncomp, const double* __restrict__ Ml, const int32_t* __restrict__ ptr,
                         double* R) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin * ncomp) return;
  const int64_t n = t % npoin;
  if (ptr[n + 1] > ptr[n]) R[t] = R[t] / Ml[n];
}

__global__ void k_sutherland(int64_t npoin, const double* __restrict__ Tem, const double* __restrict__ mf,
                             double* __restrict__ mu) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin) return;
  const double T = Tem[t];
  mu[t] = mf[t] * 0.000001458 * (T * sqrt(T)) / (T + 110.4);
}

// eta sum/max/min -> scal[0] mean, scal[1] norm (single-block deterministic reduction)
__global__ void __launch_bounds__(1024) k_eta_norm(int64_t npoin, int64_t nwork, const int32_t* __restrict__ ptr,
                                                   const double* __restrict__ eta, double* scal, int normalise) {
  __shared__ double sh[3][32];
  double s = 0.0, mx = -1e300, mn = 1e300;
  for (int64_t t = threadIdx.x; t < npoin; t += blockDim.x) {
    if (ptr[t + 1] == ptr[t]) continue;  // over lpoin_w only (mod_entropy_viscosity.f90:43-62)
    const double v = eta[t];
    s += v; mx = fmax(mx, v); mn = fmin(mn, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = s; sh[1][threadIdx.x >> 5] = mx; sh[2][threadIdx.x >> 5] = mn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    s = sh[0][0]; mx = sh[1][0]; mn = sh[2][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { s += sh[0][w]; mx = fmax(mx, sh[1][w]); mn = fmin(mn, sh[2][w]); }
    if (normalise) {
      const double mean = s / (double)nwork;
      scal[0] = mean;
      scal[1] = fmax(mx - mean, mean - mn);
    } else {
      scal[0] = 0.0;
      scal[1] = 1.0;
    }
  }
}

// adapt_dt_cfl (mod_time_ops.f90:31-57): per-element limits, then a single-block min
__global__ void k_dt_elem(int nelem, int64_t npoin, const int32_t* __restrict__ econn, const double* __restrict__ helem,
                          const double* __restrict__ u, const double* __restrict__ cs, const double* __restrict__ muf,
                          const double* __restrict__ musgs, const double* __restrict__ rho, double cfl_conv,
                          double cfl_diff, double* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  double L3 = 0.0, maxMU = 0.0;
  for (int d = 0; d < NN; ++d) {
    const int n = econn[(int64_t)e * NN + d];
    double um = fabs(u[n]);
    um = fmax(um, fabs(u[n + npoin]));
    um = fmax(um, fabs(u[n + 2 * npoin]));
    L3 = fmax(L3, um + cs[n]);
    const double sg = musgs ? musgs[(int64_t)e * NN + d] : 0.0;
    maxMU = fmax(maxMU, (rho[n] * sg + muf[n]) / rho[n]);
  }
  const double hh = helem[e] / (double)(2.0 * P + 1);
  out[e] = fmin(cfl_conv * hh / L3, cfl_diff * (hh * hh) / maxMU);
}

__global__ void __launch_bounds__(1024) k_min_reduce(int64_t n, const double* __restrict__ v, double* out) {
  __shared__ double sh[32];
  double mn = 100000000000000.0;
  for (int64_t t = threadIdx.x; t < n; t += blockDim.x) mn = fmin(mn, v[t]);
  for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mn;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mn = fmin(mn, sh[w]);
    *out = fmin(sh[0], mn);
  }
}

__global__ void k_csr_spmv_legacy(int npoin, const int32_t* __restrict__ rdom, const int32_t* __restrict__ cdom,
                                  const double* __restrict__ Mc, const double* __restrict__ v, double* __restrict__ u) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= npoin) return;
  double s = 0.0;
  for (int c = rdom[r]; c < rdom[r + 1]; ++c) s += Mc[c] * v[cdom[c] - 1];
  u[r] = s;
}

static int gather_out(SodMesh* m, const double* Ml, int f0, int nf, double* o0, double* o1, double* o2, double* o3,
                      double* o4, cudaStream_t st) {
  k_gather_plain<<<(m->npoin + 255) / 256, 256, 0, st>>>(m->npoin, m->n2e_ptr, m->n2e, (const double*)m->buf.rel, Ml,
                                                          f0, nf, o0, o1, o2, o3, o4);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

static RefArgs ref_args(SodMesh* m) {
  RefArgs a{};
  a.nelem = m->nelem;
  a.npoin = m->npoin;
  a.econn = m->econn;
  a.geo = m->geo64;
  a.D = m->D;
  a.rel = (double*)m->buf.rel;
  a.c_rho = m->prm.c_rho;
  a.c_ener = m->prm.c_ener;
  return a;
}

}  // namespace sod

using namespace sod;

extern "C" {

int sod_full_convec_ijk(SodMesh* m, const double* u, const double* q, const double* rho, const double* pr,
                        const double* E, double* Rmass, double* Rmom, double* Rener, sod_stream_t stream) {
  SOD_ARG(m && u && q && rho && pr && E && Rmass && Rmom && Rener, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  RefArgs a = ref_args(m);
  a.u = u; a.q = q; a.rho = rho; a.pr = pr; a.E = E;
  k_convec_ref<false><<<m->nelem, 64, 0, st>>>(a);
  SOD_CHECK_LAUNCH();
  const size_t N = m->npoin;
  return gather_out(m, nullptr, 0, 5, Rmass, Rmom, Rmom + N, Rmom + 2 * N, Rener, st);
}

int sod_full_convec_ijk_H(SodMesh* m, const double* u, const double* q, const double* rho, const double* pr,
                          const double* E, double* Rmass, double* Rmom, double* Rener, sod_stream_t stream) {
  SOD_ARG(m && u && q && rho && pr && E && Rmass && Rmom && Rener, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  RefArgs a = ref_args(m);
  a.u = u; a.q = q; a.rho = rho; a.pr = pr; a.E = E;
  k_convec_ref<true><<<m->nelem, 64, 0, st>>>(a);
  SOD_CHECK_LAUNCH();
  const size_t N = m->npoin;
  return gather_out(m, nullptr, 0, 5, Rmass, Rmom, Rmom + N, Rmom + 2 * N, Rener, st);
}

int sod_generic_scalar_convec_ijk(SodMesh* m, const double* q, const double* eta, const double* u,
                                  double* Rconvec, sod_stream_t stream) {
  SOD_ARG(m && q && eta && u && Rconvec, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  RefArgs a = ref_args(m);
  a.u = u; a.q = q; a.E = eta;
  k_scalar_ref<<<m->nelem, 64, 0, st>>>(a);
  SOD_CHECK_LAUNCH();
  return gather_out(m, nullptr, 5, 1, Rconvec, nullptr, nullptr, nullptr, nullptr, st);
}

int sod_full_diffusion_ijk(SodMesh* m, double Cp, double Pr, const double* rho_n, const double* rho,
                           const double* u, const double* Tem, const double* mu_fluid, const double* mu_e,
                           const double* mu_sgs, double* Rmass, double* Rmom, double* Rener, sod_stream_t stream) {
  SOD_ARG(m && rho_n && rho && u && Tem && mu_fluid && mu_e && Rmass && Rmom && Rener, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  // element arrays to the internal layout (mu_sgs into the stage scratch of rsum)
  rc = mesh_ref_to_internal_elem(m, mu_e, m->mue_int, st);
  if (rc) return rc;
  double* musgs_int = nullptr;
  if (mu_sgs) {
    SOD_CUDA(cudaMallocAsync((void**)&musgs_int, sizeof(double) * (size_t)m->nelem * NN, st));
    rc = mesh_ref_to_internal_elem(m, mu_sgs, musgs_int, st);
    if (rc) return rc;
  }
  RefArgs a = ref_args(m);
  a.rho_n = rho_n; a.rho = rho; a.u = u; a.Tem = Tem; a.mu_fluid = mu_fluid; a.mue = m->mue_int; a.musgs = musgs_int;
  a.Cp = Cp; a.Pr = Pr;
  k_diffusion_ref<<<m->nelem, 64, 0, st>>>(a);
  SOD_CHECK_LAUNCH();
  if (musgs_int) SOD_CUDA(cudaFreeAsync(musgs_int, st));
  const size_t N = m->npoin;
  return gather_out(m, nullptr, 0, 5, Rmass, Rmom, Rmom + N, Rmom + 2 * N, Rener, st);
}

int sod_lumped_solver(SodMesh* m, double* R, int ncomp, sod_stream_t stream) {
  SOD_ARG(m && R && (ncomp == 1 || ncomp == 3), "lumped solver args");
  int64_t n = (int64_t)m->npoin * ncomp;
  k_lumped<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(m->npoin, ncomp, m->Ml, m->n2e_ptr, R);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int sod_sutherland_viscosity(int32_t npoin, const double* Tem, const double* mu_factor, double* mu_fluid,
                             sod_stream_t stream) {
  SOD_ARG(npoin > 0 && Tem && mu_factor && mu_fluid, "sutherland args");
  k_sutherland<<<(npoin + 255) / 256, 256, 0, (cudaStream_t)stream>>>(npoin, Tem, mu_factor, mu_fluid);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int sod_smart_visc_spectral(SodMesh* m, const double* Reta, const double* rho, const double* u, const double* csound,
                            const double* Tem, const double* eta, double* mu_e, sod_stream_t stream) {
  SOD_ARG(m && Reta && rho && u && csound && Tem && eta && mu_e, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  k_eta_norm<<<1, 1024, 0, st>>>(m->npoin, m->npoin_w, m->n2e_ptr, eta, m->buf.scal, m->prm.normalise);
  SOD_CHECK_LAUNCH();
  SodState s{};
  s.Reta = const_cast<double*>(Reta);
  s.rho = const_cast<double*>(rho);
  s.u = const_cast<double*>(u);
  s.csound = const_cast<double*>(csound);
  s.Tem = const_cast<double*>(Tem);
  s.mu_fluid = const_cast<double*>(rho);  // unused without dt
  rc = launch_visc_dt(m, &s, nullptr, nullptr, st);
  if (rc) return rc;
  return mesh_internal_to_ref_elem(m, m->mue_int, mu_e, st);
}

int sod_adapt_dt_cfl(SodMesh* m, const double* u, const double* csound, const double* mu_fluid,
                     const double* mu_sgs, const double* rho, double* dt_dev, sod_stream_t stream) {
  SOD_ARG(m && u && csound && mu_fluid && rho && dt_dev, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  double* musgs_int = nullptr;
  if (mu_sgs) {
    SOD_CUDA(cudaMallocAsync((void**)&musgs_int, sizeof(double) * (size_t)m->nelem * NN, st));
    rc = mesh_ref_to_internal_elem(m, mu_sgs, musgs_int, st);
    if (rc) return rc;
  }
  double* tmp = (double*)m->buf.rel;  // nelem doubles of scratch
  k_dt_elem<<<(m->nelem + 127) / 128, 128, 0, st>>>(m->nelem, m->npoin, m->econn, m->helem, u, csound, mu_fluid,
                                                     musgs_int, rho, m->prm.cfl_conv, m->prm.cfl_diff, tmp);
  SOD_CHECK_LAUNCH();
  k_min_reduce<<<1, 1024, 0, st>>>(m->nelem, tmp, dt_dev);
  SOD_CHECK_LAUNCH();
  if (musgs_int) SOD_CUDA(cudaFreeAsync(musgs_int, st));
  return SOD_OK;
}

int sod_csr_spmv_scal(int32_t npoin, int32_t nzdom, const int32_t* rdom, const int32_t* cdom, const double* Mc,
                      const double* v, double* u, sod_stream_t stream) {
  SOD_ARG(npoin > 0 && nzdom >= 0 && rdom && cdom && Mc && v && u, "csr args");
  k_csr_spmv_legacy<<<(npoin + 127) / 128, 128, 0, (cudaStream_t)stream>>>(npoin, rdom, cdom, Mc, v, u);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

}  // extern "C"
