// Boundary conditions of the non-periodic path (noBoundaries = .false.): the routines of
// mod_bc_routines.f90 on the device and their place in rk_4_main (time_integ.f90:256-259,
// 299-301, 434-437, 474-477).
//
// The boundary nodes are compacted once (sod_mesh_set_boundaries) into an ascending list with
// their code, lnbn node, normal and buffer velocity; every kernel here runs one thread per
// boundary node.  temporary_bc_routine_dirichlet_prim is two kernels: k_bc_gather copies the
// state of every boundary node's lnbn node first (the reference's first loop), so a boundary
// node whose lnbn node is itself on a boundary reads the value from before the routine, as
// there; k_bc_apply forms the lnbn node's velocity and pressure and overwrites the boundary
// node by code.
//
// Inside a step the stage state is formed by the gather kernel of the previous stage (stage
// 1: a copy of the state) and the routine runs on it before the element kernels evaluate its
// EOS.  The slip branch reads the velocity left in aux_u by the previous stage's EOS (zero at
// stage 1, time_integ.f90:208), which for a boundary node is q/rho of its post-boundary stage
// state: k_bc_apply keeps that per boundary node for the next stage.  After the final update
// the routine reads u(:,:,pos) from before the update (kept at the start of the step), then
// the EOS and Sutherland viscosity of the boundary nodes are re-evaluated, the entropy
// residual is zeroed on no-slip walls and the entropy normalisation (mean and spread of eta,
// mod_entropy_viscosity.f90:43-66) is recomputed from the post-boundary eta.
#include "sod_internal.cuh"
#include <algorithm>
#include <utility>
#include <vector>

namespace sod {
namespace bcd {

constexpr int kMaxNumBouCodes = 10;  // mod_constants.f90:29
constexpr int kFarField = 1, kNonSlipAdiabatic = 3, kNonSlipHot = 4, kNonSlipCold = 5, kSlipAdiabatic = 6,
              kSlipWallModel = 7;  // mod_constants.f90:41-48
constexpr int kBlock = 256;

__device__ __forceinline__ bool no_slip(int c) {
  return c == kNonSlipAdiabatic || c == kNonSlipHot || c == kNonSlipCold;
}

// aux2 = (rho, q x3, E) of each boundary node's lnbn node (mod_bc_routines.f90:41-51)
__global__ void k_bc_gather(int nb, const int32_t* __restrict__ nbr, const double* __restrict__ rho,
                            const double* __restrict__ q, const double* __restrict__ E, size_t N,
                            double* __restrict__ aux2) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const size_t s = (size_t)nbr[b];
  aux2[b] = rho[s];
  aux2[(size_t)nb + b] = q[s];
  aux2[2 * (size_t)nb + b] = q[s + N];
  aux2[3 * (size_t)nb + b] = q[s + 2 * N];
  aux2[4 * (size_t)nb + b] = E[s];
}

struct ApplyArgs {
  int nb;
  size_t N;
  const int32_t* node;
  const int32_t* code;
  const double* normal;  // [3][nb]
  const double* ubuf;    // [3][nb]
  const double* aux2;    // [5][nb]
  double *rho, *q, *E;   // state updated in place (node-indexed)
  const double* uold_b;  // slip branch velocity per boundary node [3][nb], or
  const double* uold_n;  // per node (npoin,3); both null: zero
  double* u_n;           // aux_u / aux_p outputs of the routine (node-indexed), optional
  double* pr_n;
  double* u_post_b;      // q/rho after the routine per boundary node [3][nb], optional
  int eos;               // 1: EOS + Sutherland of the boundary nodes into the outputs below
  double *e_int, *csound, *machno, *Tem, *eta, *mu_fluid;
  const double* mu_factor;
  double* Reta;          // zeroed on no-slip nodes when set
  double gamma, Rgas;
  SodBcParams p;
};

// mod_bc_routines.f90:55-178 (second and third loops) for one boundary node of code c: own =
// (rho, q x3, E) of the node, nb = the same of its lnbn node (copied by the first loop), uo the
// velocity the slip branch reads.  Writes the node's new (rho, q x3, E) to out; uu / pp receive
// the routine's aux_u / aux_p where it sets them (set_u / set_p).
template <typename T> __device__ __forceinline__ T cst(double v);
template <> __device__ __forceinline__ double cst<double>(double v) { return v; }
__device__ __forceinline__ double bsqrt(double a) { return ::sqrt(a); }
__device__ __forceinline__ double bmin(double a, double b) { return ::fmin(a, b); }
__device__ __forceinline__ double bmax(double a, double b) { return ::fmax(a, b); }

// forward-mode dual numbers: the directional derivative of the far-field state (the adjoint)
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)};
}
template <> __device__ __forceinline__ Dual cst<Dual>(double v) { return {v, 0.0}; }
__device__ __forceinline__ Dual bsqrt(Dual a) {
  const double s = ::sqrt(a.v);
  return {s, a.d / (2.0 * s)};
}
__device__ __forceinline__ Dual bmin(Dual a, Dual b) { return a.v <= b.v ? a : b; }
__device__ __forceinline__ Dual bmax(Dual a, Dual b) { return a.v >= b.v ? a : b; }

template <typename T>
__device__ __forceinline__ void bc_point(int c, const T (&own)[5], const T (&nb)[5], const double (&uo)[3],
                                         const double (&nrm)[3], const double (&ub)[3], const SodBcParams& p,
                                         T (&out)[5], T (&uu)[3], T& pp, bool& set_u, bool& set_p) {
  const double gi = p.gamma_inf;
  const T rho2 = nb[0];
  const T q2[3] = {nb[1], nb[2], nb[3]};
  const T E2 = nb[4];
  const T u2[3] = {q2[0] / rho2, q2[1] / rho2, q2[2] / rho2};
  const T p2 = rho2 * cst<T>(gi - 1.0) *
               ((E2 / rho2) - cst<T>(0.5) * ((u2[0] * u2[0]) + (u2[1] * u2[1]) + (u2[2] * u2[2])));
  T r = own[0], e = own[4];
  T qq[3] = {own[1], own[2], own[3]};
  uu[0] = uu[1] = uu[2] = cst<T>(0.0);
  pp = cst<T>(0.0);
  set_u = set_p = false;
  if (c == kFarField) {
    const double E_inf = (p.rho_inf * 0.5 * (p.u_inf * p.u_inf) + p.p_inf / (gi - 1.0));
    const T c2 = bsqrt(cst<T>(gi) * p2 / rho2);
    T sl = bmin(cst<T>(p.u_inf - p.c_inf), u2[0] - c2);
    T sr = bmax(u2[0] + c2, cst<T>(p.u_inf + p.c_inf));
    const T rho_hll = (sr * rho2 - sl * cst<T>(p.rho_inf) + cst<T>(p.rho_inf * p.u_inf) - q2[0]) / (sr - sl);
    const T E_hll = (sr * E2 - sl * cst<T>(E_inf) + cst<T>(p.u_inf * (E_inf + p.p_inf)) - u2[0] * (E2 + p2)) /
                    (sr - sl);
    T qh[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      sl = bmin(cst<T>(ub[d] - p.c_inf), u2[d] - c2);
      sr = bmax(u2[d] + c2, cst<T>(ub[d] + p.c_inf));
      qh[d] = (sr * q2[d] - sl * cst<T>(p.rho_inf) * cst<T>(ub[d]) + cst<T>(p.rho_inf * (ub[d] * ub[d])) -
               u2[d] * q2[d]) / (sr - sl);
    }
    r = rho_hll;
    e = E_hll;
#pragma unroll
    for (int d = 0; d < 3; ++d) qq[d] = qh[d];
#pragma unroll
    for (int d = 0; d < 3; ++d) uu[d] = qq[d] / r;
    pp = r * cst<T>(gi - 1.0) * ((e / r) - cst<T>(0.5) * ((uu[0] * uu[0]) + (uu[1] * uu[1]) + (uu[2] * uu[2])));
    set_u = set_p = true;
  } else if (c == kNonSlipAdiabatic) {
    qq[0] = qq[1] = qq[2] = cst<T>(0.0);
    set_u = true;
    r = cst<T>(p.rho_inf);
  } else if (c == kNonSlipHot || c == kNonSlipCold) {
    qq[0] = qq[1] = qq[2] = cst<T>(0.0);
    set_u = true;
    r = cst<T>(p.p_inf / p.Rgas_inf / (c == kNonSlipHot ? p.T_H : p.T_C));
    e = cst<T>(p.p_inf / (gi - 1.0));
  } else if (c == kSlipWallModel || c == kSlipAdiabatic) {
    e = e - r * cst<T>(0.5) * cst<T>((uo[0] * uo[0]) + (uo[1] * uo[1]) + (uo[2] * uo[2]));
    const T norm = (cst<T>(nrm[0]) * qq[0]) + (cst<T>(nrm[1]) * qq[1]) + (cst<T>(nrm[2]) * qq[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) qq[d] = qq[d] - norm * cst<T>(nrm[d]);
    r = cst<T>(p.rho_inf);
#pragma unroll
    for (int d = 0; d < 3; ++d) uu[d] = qq[d] / r;
    e = e + r * cst<T>(0.5) * ((uu[0] * uu[0]) + (uu[1] * uu[1]) + (uu[2] * uu[2]));
    set_u = true;
  }
  out[0] = r;
  out[1] = qq[0];
  out[2] = qq[1];
  out[3] = qq[2];
  out[4] = e;
}

__global__ void __launch_bounds__(kBlock) k_bc_apply(const ApplyArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nb) return;
  const size_t nb = (size_t)a.nb, N = a.N;
  const size_t n = (size_t)a.node[b];
  const int c = a.code[b];
  double own[5] = {a.rho[n], a.q[n], a.q[n + N], a.q[n + 2 * N], a.E[n]};
  double nbv[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) nbv[f] = a.aux2[f * nb + b];
  double uo[3] = {0.0, 0.0, 0.0};
  if (a.uold_b) {
#pragma unroll
    for (int d = 0; d < 3; ++d) uo[d] = a.uold_b[d * nb + b];
  } else if (a.uold_n) {
#pragma unroll
    for (int d = 0; d < 3; ++d) uo[d] = a.uold_n[n + N * d];
  }
  const double nrm[3] = {a.normal[b], a.normal[nb + b], a.normal[2 * nb + b]};
  const double ubv[3] = {a.ubuf[b], a.ubuf[nb + b], a.ubuf[2 * nb + b]};
  double out[5], uu[3], pp;
  bool set_u, set_p;
  bc_point<double>(c, own, nbv, uo, nrm, ubv, a.p, out, uu, pp, set_u, set_p);
  const double r = out[0], e = out[4];
  const double qq[3] = {out[1], out[2], out[3]};
  a.rho[n] = r;
  a.E[n] = e;
#pragma unroll
  for (int d = 0; d < 3; ++d) a.q[n + N * d] = qq[d];
  if (a.u_post_b) {
#pragma unroll
    for (int d = 0; d < 3; ++d) a.u_post_b[d * nb + b] = qq[d] / r;
  }
  if (a.eos) {
    eos_store(n, N, r, qq, e, a.gamma, a.Rgas, a.u_n, a.pr_n, a.e_int, a.csound, a.machno, a.Tem, a.eta, a.mu_fluid,
              a.mu_factor);
  } else {
    if (a.u_n && set_u) {
#pragma unroll
      for (int d = 0; d < 3; ++d) a.u_n[n + N * d] = uu[d];
    }
    if (a.pr_n && set_p) a.pr_n[n] = pp;
  }
  if (a.Reta && no_slip(c)) a.Reta[n] = 0.0;
}

// Adjoint of the routine, in three steps on vbar, the adjoint of the new state ([5][npoin]
// columns), mapped in place to that of the old state.  (1) Far-field nodes: the new state is
// the HLL state of the lnbn node's old state, so J^T vbar(node) is formed with dual numbers
// (5 directions through bc_point<Dual>) into per-node contributions.  (2) The rows the routine
// overwrites are zeroed: far-field nodes entirely, no-slip nodes in rho and q (adiabatic walls
// keep E, isothermal walls set it), outlet / ABL-top nodes are left alone.  (3) Each lnbn node
// of a far-field node adds the contributions of the far-field nodes that read it, in ascending
// order (deterministic).
__global__ void __launch_bounds__(kBlock) k_bc_ff_adjoint(int nb, const int32_t* __restrict__ node,
                                                          const int32_t* __restrict__ code,
                                                          const int32_t* __restrict__ nbr, size_t N,
                                                          const double* __restrict__ y,
                                                          const double* __restrict__ vbar,
                                                          const double* __restrict__ normal,
                                                          const double* __restrict__ ubuf, const SodBcParams p,
                                                          double* __restrict__ contrib) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb || code[b] != kFarField) return;
  const size_t n = (size_t)node[b], s = (size_t)nbr[b];
  double w[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) w[f] = vbar[f * N + n];
  const double uo[3] = {0.0, 0.0, 0.0};
  const double nrm[3] = {normal[b], normal[(size_t)nb + b], normal[2 * (size_t)nb + b]};
  const double ubv[3] = {ubuf[b], ubuf[(size_t)nb + b], ubuf[2 * (size_t)nb + b]};
  for (int dir = 0; dir < 5; ++dir) {
    Dual own[5], nbd[5], out[5], uu[3], pp;
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      own[f] = Dual{0.0, 0.0};
      nbd[f] = Dual{y[f * N + s], f == dir ? 1.0 : 0.0};
    }
    bool su, sp;
    bc_point<Dual>(kFarField, own, nbd, uo, nrm, ubv, p, out, uu, pp, su, sp);
    double c = 0.0;
#pragma unroll
    for (int f = 0; f < 5; ++f) c += out[f].d * w[f];
    contrib[(size_t)dir * nb + b] = c;
  }
}

// Slip walls: new state (rho_inf, P q, e - rho |uo|^2 / 2 + |P q|^2 / (2 rho_inf)), P = I - n n^T,
// rho, q, e the node's pre-routine values and uo the velocity it read.  Adjoint of the own
// node (rows replaced in place) and of uo (left in ubar for the state uo was read from).
__global__ void __launch_bounds__(kBlock) k_bc_slip_adjoint(int nb, const int32_t* __restrict__ node,
                                                            const int32_t* __restrict__ code,
                                                            const double* __restrict__ normal, size_t N,
                                                            const double* __restrict__ pre,  // [4][nb] rho, q
                                                            const double* __restrict__ uo,   // [3][nb]
                                                            double rho_inf, double* __restrict__ vbar,
                                                            double* __restrict__ ubar) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int c = code[b];
  if (c != kSlipAdiabatic && c != kSlipWallModel) return;
  const size_t n = (size_t)node[b], B = (size_t)nb;
  const double nv[3] = {normal[b], normal[B + b], normal[2 * B + b]};
  const double r = pre[b];
  const double q[3] = {pre[B + b], pre[2 * B + b], pre[3 * B + b]};
  const double u[3] = {uo[b], uo[B + b], uo[2 * B + b]};
  const double qn = nv[0] * q[0] + nv[1] * q[1] + nv[2] * q[2];
  double qp[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) qp[d] = q[d] - qn * nv[d];
  const double eb = vbar[4 * N + n];
  double qb[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) qb[d] = vbar[(1 + d) * N + n];
  const double qbn = nv[0] * qb[0] + nv[1] * qb[1] + nv[2] * qb[2];
  vbar[n] = -0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) * eb;
#pragma unroll
  for (int d = 0; d < 3; ++d) vbar[(1 + d) * N + n] = (qb[d] - qbn * nv[d]) + (qp[d] / rho_inf) * eb;
  // vbar[4N + n] stays eb
#pragma unroll
  for (int d = 0; d < 3; ++d) ubar[(size_t)d * nb + b] = -r * u[d] * eb;
}

// rho and q residuals (gather / Ml, with the source term on q) of one stage at the slip nodes
__global__ void __launch_bounds__(kBlock) k_bc_slip_res(int nb, const int32_t* __restrict__ node,
                                                        const int32_t* __restrict__ code,
                                                        const int32_t* __restrict__ ptr,
                                                        const int32_t* __restrict__ idx,
                                                        const double* __restrict__ el, const double* __restrict__ Ml,
                                                        const double* __restrict__ src,
                                                        const double* __restrict__ wmc, size_t N,
                                                        double* __restrict__ res /*[4][nb]*/) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int c = code[b];
  if (c != kSlipAdiabatic && c != kSlipWallModel) return;
  const size_t n = (size_t)node[b];
  double r[4] = {0.0, 0.0, 0.0, 0.0};
  const int beg = ptr[n], end = ptr[n + 1];
  for (int k = beg; k < end; ++k) {
    const double* v = el + (size_t)idx[k] * NRES;
#pragma unroll
    for (int f = 0; f < 4; ++f) r[f] += v[f];
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
#pragma unroll
  for (int f = 0; f < 4; ++f) res[(size_t)f * nb + b] = r[f] / ml;
}

// pre-routine rho and q of the five applications (stages 1-4: y0 - a_s dt R_{s-1}; the update:
// y0 - dt sum_s b_s R_s, accumulated in the forward's order) and the velocity each reads
// (stage 1: zero; stage s: q/rho of the post-routine stage state s - 1; the update: q/rho of y0)
__global__ void __launch_bounds__(kBlock) k_bc_slip_prepare(int nb, const int32_t* __restrict__ node,
                                                            const int32_t* __restrict__ code, size_t N,
                                                            const double* __restrict__ rho0,
                                                            const double* __restrict__ q0,
                                                            const double* __restrict__ Y1,
                                                            const double* __restrict__ Y2,
                                                            const double* __restrict__ Y3,
                                                            const double* __restrict__ dt,
                                                            const double* __restrict__ res,
                                                            const int32_t* __restrict__ zmap,
                                                            const double* __restrict__ zxi,
                                                            const double* __restrict__ zub, int znb,
                                                            double rho_inf, double* __restrict__ pre,
                                                            double* __restrict__ uo) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int c = code[b];
  if (c != kSlipAdiabatic && c != kSlipWallModel) return;
  const size_t n = (size_t)node[b], B = (size_t)nb;
  const double h = *dt;
  const double a_s[4] = {0.0, 0.5, 0.5, 1.0};
  const double b_s[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const double y = f == 0 ? rho0[n] : q0[(f - 1) * N + n];
    pre[(0 * 4 + f) * B + b] = y;
    double rs = 0.0;
#pragma unroll
    for (int s = 1; s < 4; ++s) pre[((size_t)s * 4 + f) * B + b] = y - h * a_s[s] * res[((size_t)(s - 1) * 4 + f) * B + b];
#pragma unroll
    for (int s = 0; s < 4; ++s) rs = rs + b_s[s] * res[((size_t)s * 4 + f) * B + b];
    pre[((size_t)4 * 4 + f) * B + b] = y - h * rs;
  }
  // with a buffer zone the routine reads the zone-updated state (E is not needed here)
  const int zi = zmap ? zmap[n] : -1;
  if (zi >= 0) {
    for (int a = 0; a < 5; ++a) {
      double r = pre[((size_t)a * 4) * B + b], e = 0.0;
      double qq[3] = {pre[((size_t)a * 4 + 1) * B + b], pre[((size_t)a * 4 + 2) * B + b],
                      pre[((size_t)a * 4 + 3) * B + b]};
      zone_point(zxi, zub, znb, zi, rho_inf, 0.0, r, qq, e);
      pre[((size_t)a * 4) * B + b] = r;
#pragma unroll
      for (int d = 0; d < 3; ++d) pre[((size_t)a * 4 + 1 + d) * B + b] = qq[d];
    }
  }
  const double* from[4] = {nullptr, Y1, Y2, Y3};
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int d = 0; d < 3; ++d)
      uo[((size_t)a * 3 + d) * B + b] = from[a] ? from[a][(1 + d) * N + n] / from[a][n] : 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) uo[((size_t)4 * 3 + d) * B + b] = q0[d * N + n] / rho0[n];
}

// the velocity adjoint ubar of a slip node into the adjoint (vrho, vq) of the state (rho, q) it
// was read from (uo = q / rho at the node)
__global__ void __launch_bounds__(kBlock) k_bc_slip_push(int nb, const int32_t* __restrict__ node,
                                                         const int32_t* __restrict__ code, size_t N,
                                                         const double* __restrict__ rho,
                                                         const double* __restrict__ q,
                                                         const double* __restrict__ ubar, double* __restrict__ vrho,
                                                         double* __restrict__ vq) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int c = code[b];
  if (c != kSlipAdiabatic && c != kSlipWallModel) return;
  const size_t n = (size_t)node[b], B = (size_t)nb;
  const double r = rho[n];
  double s = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double ub = ubar[d * B + b];
    s += (q[d * N + n] / r) * ub;
    vq[d * N + n] += ub / r;
  }
  vrho[n] -= s / r;
}

// residuals (gather / Ml, with the source term on q) of one stage at the far-field lnbn targets
__global__ void __launch_bounds__(kBlock) k_bc_ff_res(int nu, const int32_t* __restrict__ target,
                                                      const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                      const double* __restrict__ el, const double* __restrict__ Ml,
                                                      const double* __restrict__ src,
                                                      const double* __restrict__ wmc, size_t N,
                                                      double* __restrict__ res /*[5][nu]*/) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu) return;
  const size_t n = (size_t)target[u];
  double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int k = ptr[n]; k < ptr[n + 1]; ++k) {
    const double* v = el + (size_t)idx[k] * NRES;
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
#pragma unroll
  for (int f = 0; f < 5; ++f) res[(size_t)f * nu + u] = r[f] / ml;
}

// the state the final routine reads at the far-field lnbn targets: y0 - dt sum_s b_s R_s
// (accumulated in the forward's order), then updateBuffer where the target is in a zone
__global__ void __launch_bounds__(kBlock) k_bc_ff_final(int nu, const int32_t* __restrict__ target, size_t N,
                                                        const double* __restrict__ rho0,
                                                        const double* __restrict__ q0,
                                                        const double* __restrict__ E0,
                                                        const double* __restrict__ dt,
                                                        const double* __restrict__ res,
                                                        const int32_t* __restrict__ zmap,
                                                        const double* __restrict__ zxi,
                                                        const double* __restrict__ zub, int znb, double rho_inf,
                                                        double E_inf, double* __restrict__ zf) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu) return;
  const size_t n = (size_t)target[u], U = (size_t)nu;
  const double b_s[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
  double y[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    double rs = 0.0;
#pragma unroll
    for (int s = 0; s < 4; ++s) rs = rs + b_s[s] * res[((size_t)s * 5 + f) * U + u];
    const double y0 = f == 0 ? rho0[n] : (f == 4 ? E0[n] : q0[(f - 1) * N + n]);
    y[f] = y0 - (*dt) * rs;
  }
  const int zi = zmap ? zmap[n] : -1;
  if (zi >= 0) {
    double qq[3] = {y[1], y[2], y[3]};
    zone_point(zxi, zub, znb, zi, rho_inf, E_inf, y[0], qq, y[4]);
    y[1] = qq[0]; y[2] = qq[1]; y[3] = qq[2];
  }
#pragma unroll
  for (int f = 0; f < 5; ++f) zf[f * N + n] = y[f];
}

__global__ void k_bc_adjoint_mask(int nb, const int32_t* __restrict__ node, const int32_t* __restrict__ code,
                                  size_t N, double* __restrict__ vbar) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int c = code[b];
  const size_t n = (size_t)node[b];
  if (c == kFarField) {
#pragma unroll
    for (int f = 0; f < 5; ++f) vbar[f * N + n] = 0.0;
    return;
  }
  if (!no_slip(c)) return;
#pragma unroll
  for (int f = 0; f < 4; ++f) vbar[f * N + n] = 0.0;
  if (c != kNonSlipAdiabatic) vbar[4 * N + n] = 0.0;
}

__global__ void __launch_bounds__(kBlock) k_bc_ff_scatter(int nu, const int32_t* __restrict__ ptr,
                                                          const int32_t* __restrict__ target,
                                                          const int32_t* __restrict__ bidx, int nb, size_t N,
                                                          const double* __restrict__ contrib,
                                                          double* __restrict__ vbar) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu) return;
  const size_t s = (size_t)target[u];
  const int beg = ptr[u], end = ptr[u + 1];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    double a = 0.0;
    for (int k = beg; k < end; ++k) a += contrib[(size_t)f * nb + bidx[k]];
    vbar[f * N + s] += a;
  }
}

// bc_fix_dirichlet_residual (mod_bc_routines.f90:181-221) and _entropy (:265-291)
__global__ void k_bc_fix(int nb, const int32_t* __restrict__ node, const int32_t* __restrict__ code, size_t N,
                         double* Rmass, double* Rmom, double* Rener, double* R) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int c = code[b];
  if (!no_slip(c)) return;
  const size_t n = (size_t)node[b];
  if (R) R[n] = 0.0;
  if (Rmom) {
    Rmom[n] = 0.0;
    Rmom[n + N] = 0.0;
    Rmom[n + 2 * N] = 0.0;
  }
  if (Rmass) Rmass[n] = 0.0;
  if (Rener && c != kNonSlipAdiabatic) Rener[n] = 0.0;
}

__global__ void k_bc_snapshot(int nb, const int32_t* __restrict__ node, const double* __restrict__ u, size_t N,
                              double* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const size_t n = (size_t)node[b];
#pragma unroll
  for (int d = 0; d < 3; ++d) out[(size_t)d * nb + b] = u[n + N * d];
}

// entropy normalisation from the post-boundary eta: block partials (sum, max, min), then one
// block in a fixed order (deterministic)
__device__ __forceinline__ void reduce3(double& s, double& mx, double& mn, double (*sh)[kBlock / 32]) {
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { sh[0][w] = s; sh[1][w] = mx; sh[2][w] = mn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    s = sh[0][0]; mx = sh[1][0]; mn = sh[2][0];
    for (int q = 1; q < kBlock / 32; ++q) { s += sh[0][q]; mx = fmax(mx, sh[1][q]); mn = fmin(mn, sh[2][q]); }
  }
}

__global__ void __launch_bounds__(kBlock) k_eta_partials(int n, const int32_t* __restrict__ ptr,
                                                         const double* __restrict__ eta, double* red) {
  __shared__ double sh[3][kBlock / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0, mx = -1e300, mn = 1e300;
  if (i < n && ptr[i + 1] > ptr[i]) s = mx = mn = eta[i];  // working nodes only
  reduce3(s, mx, mn, sh);
  if (threadIdx.x == 0) {
    red[3 * blockIdx.x] = s;
    red[3 * blockIdx.x + 1] = mx;
    red[3 * blockIdx.x + 2] = mn;
  }
}

__global__ void __launch_bounds__(kBlock) k_eta_final(int nblk, int npoin, int normalise,
                                                      const double* __restrict__ red, double* scal) {
  __shared__ double sh[3][kBlock / 32];
  double s = 0.0, mx = -1e300, mn = 1e300;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    s += red[3 * b];
    mx = fmax(mx, red[3 * b + 1]);
    mn = fmin(mn, red[3 * b + 2]);
  }
  reduce3(s, mx, mn, sh);
  if (threadIdx.x == 0) {
    if (normalise) {
      const double mean = s / (double)npoin;
      scal[0] = mean;
      scal[1] = fmax(mx - mean, mean - mn);
    } else {
      scal[0] = 0.0;
      scal[1] = 1.0;
    }
  }
}

static int grid_of(int n) { return (n + kBlock - 1) / kBlock; }

static ApplyArgs base_args(SodMesh* m) {
  ApplyArgs a{};
  a.nb = m->bc.nb;
  a.N = (size_t)m->npoin;
  a.node = m->bc.node;
  a.code = m->bc.code;
  a.normal = m->bc.normal;
  a.ubuf = m->bc.ubuf;
  a.aux2 = m->bc.aux2;
  a.gamma = m->prm.gamma;
  a.Rgas = m->prm.Rgas;
  a.p = m->bc.prm;
  return a;
}

static int gather(SodMesh* m, const double* rho, const double* q, const double* E, cudaStream_t st) {
  k_bc_gather<<<grid_of(m->bc.nb), kBlock, 0, st>>>(m->bc.nb, m->bc.nbr, rho, q, E, (size_t)m->npoin, m->bc.aux2);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

}  // namespace bcd

// SOD_ERR_UNSUPPORTED for slip walls without the data of a step application (app < 0) and for
// far-field nodes whose lnbn node is itself a boundary node
int bc_adjoint(SodMesh* m, double* vbar, const double* y, int app, cudaStream_t st) {
  const BcState& B = m->bc;
  if (B.has_slip && (app < 0 || app > 4)) {
    set_error("the slip-wall adjoint needs the velocity the routine read (step adjoint only)");
    return SOD_ERR_UNSUPPORTED;
  }
  if (B.nff > 0 && B.ff_nbr_on_boundary) {
    set_error("far-field adjoint: an lnbn node of a far-field node lies on a boundary");
    return SOD_ERR_UNSUPPORTED;
  }
  const size_t N = m->npoin;
  if (B.has_slip) {
    bcd::k_bc_slip_adjoint<<<bcd::grid_of(B.nb), bcd::kBlock, 0, st>>>(
        B.nb, B.node, B.code, B.normal, N, B.sl_pre + (size_t)app * 4 * B.nb, B.sl_uo + (size_t)app * 3 * B.nb,
        B.prm.rho_inf, vbar, B.sl_ubar);
    SOD_CHECK_LAUNCH();
  }
  if (B.nff > 0) {
    SOD_ARG(y, "far-field adjoint needs the state the routine read");
    bcd::k_bc_ff_adjoint<<<bcd::grid_of(B.nb), bcd::kBlock, 0, st>>>(B.nb, B.node, B.code, B.nbr, N, y, vbar,
                                                                     B.normal, B.ubuf, B.prm, B.ff_contrib);
    SOD_CHECK_LAUNCH();
  }
  bcd::k_bc_adjoint_mask<<<bcd::grid_of(B.nb), bcd::kBlock, 0, st>>>(B.nb, B.node, B.code, N, vbar);
  SOD_CHECK_LAUNCH();
  if (B.nff > 0) {
    bcd::k_bc_ff_scatter<<<bcd::grid_of(B.ff_nu), bcd::kBlock, 0, st>>>(B.ff_nu, B.ff_ptr, B.ff_target, B.ff_b,
                                                                         B.nb, N, B.ff_contrib, vbar);
    SOD_CHECK_LAUNCH();
  }
  return SOD_OK;
}

int bc_slip_residuals(SodMesh* m, int stage, const void* rel, cudaStream_t st) {
  const BcState& B = m->bc;
  bcd::k_bc_slip_res<<<bcd::grid_of(B.nb), bcd::kBlock, 0, st>>>(
      B.nb, B.node, B.code, m->n2e_ptr, m->n2e, reinterpret_cast<const double*>(rel), m->Ml, m->source,
      m->wmodel.nw > 0 ? m->wmodel.contrib : nullptr, (size_t)m->npoin, B.sl_res + (size_t)(stage - 1) * 4 * B.nb);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int bc_slip_prepare(SodMesh* m, const double* rho0, const double* q0, const double* Y1, const double* Y2,
                    const double* Y3, const double* dt_dev, cudaStream_t st) {
  const BcState& B = m->bc;
  const ZoneState& Z = m->zone;
  bcd::k_bc_slip_prepare<<<bcd::grid_of(B.nb), bcd::kBlock, 0, st>>>(
      B.nb, B.node, B.code, (size_t)m->npoin, rho0, q0, Y1, Y2, Y3, dt_dev, B.sl_res, Z.nb > 0 ? Z.zmap : nullptr,
      Z.xi, Z.ub, Z.nb, Z.rho_inf, B.sl_pre, B.sl_uo);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int bc_ff_residuals(SodMesh* m, int stage, const void* rel, cudaStream_t st) {
  const BcState& B = m->bc;
  bcd::k_bc_ff_res<<<bcd::grid_of(B.ff_nu), bcd::kBlock, 0, st>>>(
      B.ff_nu, B.ff_target, m->n2e_ptr, m->n2e, reinterpret_cast<const double*>(rel), m->Ml, m->source,
      m->wmodel.nw > 0 ? m->wmodel.contrib : nullptr, (size_t)m->npoin, B.ff_res + (size_t)(stage - 1) * 5 * B.ff_nu);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int bc_ff_final(SodMesh* m, const double* rho0, const double* q0, const double* E0, const double* dt_dev, double* zf,
                cudaStream_t st) {
  const BcState& B = m->bc;
  const ZoneState& Z = m->zone;
  bcd::k_bc_ff_final<<<bcd::grid_of(B.ff_nu), bcd::kBlock, 0, st>>>(
      B.ff_nu, B.ff_target, (size_t)m->npoin, rho0, q0, E0, dt_dev, B.ff_res, Z.nb > 0 ? Z.zmap : nullptr, Z.xi,
      Z.ub, Z.nb, Z.rho_inf, Z.E_inf, zf);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int bc_slip_push(SodMesh* m, const double* rho, const double* q, double* vrho, double* vq, cudaStream_t st) {
  const BcState& B = m->bc;
  bcd::k_bc_slip_push<<<bcd::grid_of(B.nb), bcd::kBlock, 0, st>>>(B.nb, B.node, B.code, (size_t)m->npoin, rho, q,
                                                                  B.sl_ubar, vrho, vq);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

void bc_free(SodMesh* m) {
  BcState& b = m->bc;
  void* ptrs[] = {b.node, b.code, b.nbr, b.normal, b.ubuf, b.aux2, b.u_stage, b.u_final,
                  b.ff_ptr, b.ff_target, b.ff_b, b.ff_contrib, b.ff_res, b.slip};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  b = BcState{};
}

int bc_snapshot_u(SodMesh* m, const double* u, cudaStream_t st) {
  bcd::k_bc_snapshot<<<bcd::grid_of(m->bc.nb), bcd::kBlock, 0, st>>>(m->bc.nb, m->bc.node, u, (size_t)m->npoin,
                                                                      m->bc.u_final);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

// the routine on stage state ys ([5][npoin]: rho, q x3, E) of stage 1..4
int bc_stage(SodMesh* m, double* ys, int stage, cudaStream_t st) {
  const size_t N = m->npoin;
  if (int rc = bcd::gather(m, ys, ys + N, ys + 4 * N, st)) return rc;
  bcd::ApplyArgs a = bcd::base_args(m);
  a.rho = ys;
  a.q = ys + N;
  a.E = ys + 4 * N;
  a.uold_b = stage == 1 ? nullptr : m->bc.u_stage;  // aux_u is zero before the first stage's EOS
  a.u_post_b = m->bc.u_stage;
  bcd::k_bc_apply<<<bcd::grid_of(m->bc.nb), bcd::kBlock, 0, st>>>(a);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

// the routine on the updated state, boundary-node EOS, entropy residual fix and normalisation
int bc_final(SodMesh* m, SodState* s, double* Reta, cudaStream_t st) {
  if (int rc = bcd::gather(m, s->rho, s->q, s->E, st)) return rc;
  bcd::ApplyArgs a = bcd::base_args(m);
  a.rho = s->rho;
  a.q = s->q;
  a.E = s->E;
  a.uold_b = m->bc.u_final;
  a.eos = 1;
  a.u_n = s->u;
  a.pr_n = s->pr;
  a.e_int = s->e_int;
  a.csound = s->csound;
  a.machno = s->machno;
  a.Tem = s->Tem;
  a.eta = s->eta;
  a.mu_fluid = s->mu_fluid;
  a.mu_factor = s->mu_factor;
  a.Reta = Reta;
  bcd::k_bc_apply<<<bcd::grid_of(m->bc.nb), bcd::kBlock, 0, st>>>(a);
  SOD_CHECK_LAUNCH();
  return eta_stats(m, s->eta, st);
}

int eta_stats(SodMesh* m, const double* eta, cudaStream_t st) {
  const int nblk = bcd::grid_of(m->npoin);
  SOD_ARG(m->buf.red_cap >= 3 * (int64_t)nblk, "reduction scratch too small");
  bcd::k_eta_partials<<<nblk, bcd::kBlock, 0, st>>>(m->npoin, m->n2e_ptr, eta, m->buf.red);
  SOD_CHECK_LAUNCH();
  bcd::k_eta_final<<<1, bcd::kBlock, 0, st>>>(nblk, m->npoin_w, m->prm.normalise, m->buf.red, m->buf.scal);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

}  // namespace sod

using namespace sod;

extern "C" {

int sod_mesh_set_boundaries(SodMesh* m, const int32_t* codes, const int32_t* lnbn, const double* normals,
                            const double* u_buffer, const SodBcParams* bc) {
  SOD_ARG(m, "mesh null");
  SOD_ARG(m->nmember == 0, "boundaries on an ensemble mesh are not supported");
  for (auto& kv : m->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  m->graphs.clear();
  bc_free(m);
  if (!codes) return SOD_OK;
  SOD_ARG(lnbn && bc, "lnbn_nodes and bc parameters required");
  const int N = m->npoin;
  std::vector<int32_t> node, code, nbr;
  for (int n = 0; n < N; ++n) {
    if (codes[n] < bcd::kMaxNumBouCodes) {
      if (m->has_slaves && m->slave_host[n]) {
        set_error("sod_mesh_set_boundaries: boundary code on periodic slave row %d is not supported",
                  n + m->index_base);
        return SOD_ERR_UNSUPPORTED;
      }
      const int32_t s = lnbn[n] - m->index_base;
      SOD_ARG(s >= 0 && s < N, "lnbn_nodes entry out of range");
      node.push_back(n);
      code.push_back(codes[n]);
      nbr.push_back(s);
    }
  }
  const int nb = (int)node.size();
  if (nb == 0) return SOD_OK;
  std::vector<double> nrm((size_t)3 * nb, 0.0), ub((size_t)3 * nb, 0.0);
  for (int b = 0; b < nb; ++b)
    for (int d = 0; d < 3; ++d) {
      if (normals) nrm[(size_t)d * nb + b] = normals[(size_t)node[b] + (size_t)N * d];
      if (u_buffer) ub[(size_t)d * nb + b] = u_buffer[(size_t)node[b] + (size_t)N * d];
    }
  BcState& B = m->bc;
  auto alloc = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
  bool ok = alloc((void**)&B.node, sizeof(int32_t) * nb) && alloc((void**)&B.code, sizeof(int32_t) * nb) &&
            alloc((void**)&B.nbr, sizeof(int32_t) * nb) && alloc((void**)&B.normal, sizeof(double) * 3 * nb) &&
            alloc((void**)&B.ubuf, sizeof(double) * 3 * nb) && alloc((void**)&B.aux2, sizeof(double) * 5 * nb) &&
            alloc((void**)&B.u_stage, sizeof(double) * 3 * nb) && alloc((void**)&B.u_final, sizeof(double) * 3 * nb);
  if (!ok) {
    bc_free(m);
    set_error("sod_mesh_set_boundaries: device allocation failed");
    return SOD_ERR_NOMEM;
  }
  B.nb = nb;
  B.prm = *bc;
  for (int c : code)
    if (c == bcd::kSlipAdiabatic || c == bcd::kSlipWallModel) B.has_slip = true;
  if (B.has_slip) {
    const size_t nbs = (size_t)nb;
    if (!alloc((void**)&B.slip, sizeof(double) * (16 + 20 + 15 + 3) * nbs)) {
      bc_free(m);
      set_error("sod_mesh_set_boundaries: device allocation failed");
      return SOD_ERR_NOMEM;
    }
    B.sl_res = B.slip;
    B.sl_pre = B.sl_res + 16 * nbs;
    B.sl_uo = B.sl_pre + 20 * nbs;
    B.sl_ubar = B.sl_uo + 15 * nbs;
    SOD_CUDA(cudaMemset(B.slip, 0, sizeof(double) * (16 + 20 + 15 + 3) * nbs));
  }
  // far-field adjoint scatter: lnbn targets in ascending node order, readers in ascending order
  {
    std::vector<std::pair<int32_t, int32_t>> tb;  // (target node, boundary index)
    for (int b = 0; b < nb; ++b)
      if (code[b] == bcd::kFarField) {
        tb.emplace_back(nbr[b], b);
        if (codes[nbr[b]] < bcd::kMaxNumBouCodes) B.ff_nbr_on_boundary = true;
      }
    std::sort(tb.begin(), tb.end());
    std::vector<int32_t> ptr{0}, target, bidx;
    for (size_t k = 0; k < tb.size(); ++k) {
      if (k == 0 || tb[k].first != tb[k - 1].first) {
        if (k > 0) ptr.push_back((int32_t)k);
        target.push_back(tb[k].first);
      }
      bidx.push_back(tb[k].second);
    }
    ptr.push_back((int32_t)tb.size());
    B.nff = (int)tb.size();
    B.ff_nu = (int)target.size();
    if (B.nff > 0) {
      if (!(alloc((void**)&B.ff_ptr, sizeof(int32_t) * ptr.size()) &&
            alloc((void**)&B.ff_target, sizeof(int32_t) * target.size()) &&
            alloc((void**)&B.ff_b, sizeof(int32_t) * bidx.size()) &&
            alloc((void**)&B.ff_contrib, sizeof(double) * 5 * (size_t)nb) &&
            alloc((void**)&B.ff_res, sizeof(double) * 20 * target.size()))) {
        bc_free(m);
        set_error("sod_mesh_set_boundaries: device allocation failed");
        return SOD_ERR_NOMEM;
      }
      SOD_CUDA(cudaMemcpy(B.ff_ptr, ptr.data(), sizeof(int32_t) * ptr.size(), cudaMemcpyHostToDevice));
      SOD_CUDA(cudaMemcpy(B.ff_target, target.data(), sizeof(int32_t) * target.size(), cudaMemcpyHostToDevice));
      SOD_CUDA(cudaMemcpy(B.ff_b, bidx.data(), sizeof(int32_t) * bidx.size(), cudaMemcpyHostToDevice));
    }
  }
  SOD_CUDA(cudaMemcpy(B.node, node.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(B.code, code.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(B.nbr, nbr.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(B.normal, nrm.data(), sizeof(double) * 3 * nb, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(B.ubuf, ub.data(), sizeof(double) * 3 * nb, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemset(B.u_stage, 0, sizeof(double) * 3 * nb));
  SOD_CUDA(cudaMemset(B.u_final, 0, sizeof(double) * 3 * nb));
  return SOD_OK;
}

int sod_bc_dirichlet_prim(SodMesh* m, double* rho, double* q, double* u, double* pr, double* E, sod_stream_t stream) {
  SOD_ARG(m && rho && q && u && pr && E, "null argument");
  SOD_ARG(m->bc.nb > 0, "no boundary nodes registered (sod_mesh_set_boundaries)");
  cudaStream_t st = (cudaStream_t)stream;
  if (int rc = bcd::gather(m, rho, q, E, st)) return rc;
  bcd::ApplyArgs a = bcd::base_args(m);
  a.rho = rho;
  a.q = q;
  a.E = E;
  a.uold_n = u;
  a.u_n = u;
  a.pr_n = pr;
  bcd::k_bc_apply<<<bcd::grid_of(m->bc.nb), bcd::kBlock, 0, st>>>(a);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int sod_bc_fix_dirichlet_residual(SodMesh* m, double* Rmass, double* Rmom, double* Rener, sod_stream_t stream) {
  SOD_ARG(m && Rmass && Rmom && Rener, "null argument");
  SOD_ARG(m->bc.nb > 0, "no boundary nodes registered (sod_mesh_set_boundaries)");
  bcd::k_bc_fix<<<bcd::grid_of(m->bc.nb), bcd::kBlock, 0, (cudaStream_t)stream>>>(
      m->bc.nb, m->bc.node, m->bc.code, (size_t)m->npoin, Rmass, Rmom, Rener, nullptr);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int sod_bc_fix_dirichlet_residual_entropy(SodMesh* m, double* R, sod_stream_t stream) {
  SOD_ARG(m && R, "null argument");
  SOD_ARG(m->bc.nb > 0, "no boundary nodes registered (sod_mesh_set_boundaries)");
  bcd::k_bc_fix<<<bcd::grid_of(m->bc.nb), bcd::kBlock, 0, (cudaStream_t)stream>>>(
      m->bc.nb, m->bc.node, m->bc.code, (size_t)m->npoin, nullptr, nullptr, nullptr, R);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

}  // extern "C"
