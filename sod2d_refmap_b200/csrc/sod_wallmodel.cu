// Wall models of rk_4_main (isWallModelOn, time_integ.f90:334-357): evalWallModelReichardt and
// evalWallModelABL (mod_wall_model.f90:12-175, 177-300) add the modelled wall shear to the
// momentum diffusion residual of the wall-model faces' nodes.
//
// Everything geometric is fixed per mesh, so sod_mesh_set_wall_model forms it once on the host,
// as the reference's loop does per call: for each node of each wall-model face, the element
// holding the face (point2elem of an interior face node), the exchange node (the node of that
// element on the opposite face, aligned with the face node), the wall distance
// y = |n . (x_exchange - x_node)| with the node normal n, and the weight |bounorm| wgp_b.  The
// entries are grouped by node (ascending face order inside a node), and one thread per wall
// node evaluates its entries' shear and sums them: the reference's atomic accumulation in a
// fixed order.  tauw, written by every entry in the reference (the last write wins), takes the
// node's last entry.  In the step the kernel reads the stage state (velocity q/rho at the
// exchange node, or the caller's time-averaged walave_u; rho and the Sutherland viscosity of the
// stage EOS at the node) and writes the contribution per node; the node gather adds it to the
// momentum residual before the lumped-mass division.
#include "sod_internal.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace sod {
namespace wm {

constexpr int kBlock = 128;
constexpr int kReichardt = 1, kABL = 2;  // wmles_type_reichardt, wmles_type_abl (mod_constants.f90:51-52)

struct Args {
  int nw;
  const int32_t* __restrict__ wnode;  // wall nodes
  const int32_t* __restrict__ wptr;   // entries of each wall node
  const int32_t* __restrict__ ex;     // exchange node of each entry
  const double* __restrict__ w;       // |bounorm| wgp_b
  const double* __restrict__ nrm;     // [3][nent] normal at the node
  const double* __restrict__ y;       // wall distance
  const double* __restrict__ zo;      // roughness at the node (ABL), per entry
  int nent, type;
  size_t N;
};

// forward-mode dual numbers: the law's derivatives for the adjoint (through the executed
// Newton iterations)
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b) { return {a / b.v, -a * b.d / (b.v * b.v)}; }
__device__ __forceinline__ Dual dexp(Dual a) { const double e = exp(a.v); return {e, e * a.d}; }
__device__ __forceinline__ Dual dlog(Dual a) { return {log(a.v), a.d / a.v}; }
__device__ __forceinline__ Dual dsqrt(Dual a) { const double s = sqrt(a.v); return {s, a.d / (2.0 * s)}; }
__device__ __forceinline__ Dual dabs(Dual a) { return a.v < 0.0 ? -a : a; }
__device__ __forceinline__ Dual dmin(Dual a, Dual b) { return a.v <= b.v ? a : b; }
__device__ __forceinline__ Dual dmax(Dual a, Dual b) { return a.v >= b.v ? a : b; }
__device__ __forceinline__ double dexp(double a) { return exp(a); }
__device__ __forceinline__ double dlog(double a) { return log(a); }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ double dabs(double a) { return fabs(a); }
__device__ __forceinline__ double dmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double dmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ double val(double a) { return a; }
__device__ __forceinline__ double val(Dual a) { return a.v; }

// the wall shear magnitude of one entry (the two laws of mod_wall_model.f90)
template <typename T>
__device__ T shear(int type, T ul, double y, T nul, T rhol, double zo) {
  if (type == kABL) {
    const T uistar = ul * 0.41 / dlog(T{1.0 + y / zo});
    return rhol * uistar * uistar / ul;
  }
  T uistar;
  if (y > 0.0 && val(ul) > 1.0e-10) {
    uistar = dsqrt(ul * nul / y);
    if (val(uistar * y / nul) > 5.0) {
      const double vkinv = 1.0 / 0.41, oneoe = 1.0 / 11.0;
      const T onovu = 1.0 / ul, xmuit = y / nul;
      int itera = 0;
      double parco = 1.0;
      while (parco >= 1.0e-6 && itera < 100) {  // bounded: at most 100 iterations
        itera = itera + 1;
        uistar = dmax(uistar, T{0.0});
        const T yplus = uistar * xmuit;
        const T ypele = yplus * oneoe;
        const T ypel2 = dmin(ypele, T{20.0});
        const T expye = dexp(-ypel2);
        const T yplu2 = dmin(yplus, T{70.0});
        const T expyt = dexp(-yplu2 * 0.33);
        const T firsl = vkinv * dlog(1.0 + 0.4 * yplus);
        const T fdvfr = uistar * (firsl + 7.8 * (1.0 - expye - ypele * expyt)) - ul;
        const T diffd = firsl + vkinv * 0.4 * yplus / (1.0 + 0.4 * yplus) +
                        7.8 * (1.0 - expye * (1.0 - ypele) - ypele * expyt * (2.0 - yplus * 0.33));
        const T devfr = -fdvfr / diffd;
        parco = val(dabs(devfr * onovu));
        uistar = uistar + devfr;
      }
    }
  } else {
    uistar = T{0.0};
  }
  return (val(y * uistar / nul) < 5.0) ? rhol * nul / y : rhol * uistar * uistar / ul;
}

// STATE: rho, q, E are a state's columns (velocity q/rho, viscosity from the EOS + Sutherland);
// otherwise rho, u (3 columns) and mu_fluid are given.  ui, when set, replaces the exchange
// velocity (walave_u).  out: accumulate (+=) or overwrite the node's 3 components.
template <bool STATE>
__global__ void __launch_bounds__(kBlock) k_wall_model(const Args a, const double* __restrict__ rho,
                                                       const double* __restrict__ q, const double* __restrict__ E,
                                                       const double* __restrict__ mu_fluid,
                                                       const double* __restrict__ mu_factor,
                                                       const double* __restrict__ ui, double gamma, double Rgas,
                                                       double* __restrict__ out, int accumulate,
                                                       double* __restrict__ tauw) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nw) return;
  const size_t N = a.N, n = (size_t)a.wnode[t];
  const double rhol = rho[n];
  double mu;
  if constexpr (STATE) {
    const double ir = 1.0 / rhol;
    const double u0 = q[n] * ir, u1 = q[n + N] * ir, u2 = q[n + 2 * N] * ir;
    const double p = rhol * (gamma - 1.0) * (E[n] * ir - 0.5 * (u0 * u0 + u1 * u1 + u2 * u2));
    const double T = p / (rhol * Rgas);
    mu = mu_factor[n] * kSuthC1 * (T * sqrt(T)) / (T + kSuthS);
  } else {
    mu = mu_fluid[n];
  }
  const double nul = mu / rhol;
  double acc[3] = {0.0, 0.0, 0.0}, last[3] = {0.0, 0.0, 0.0};
  for (int k = a.wptr[t]; k < a.wptr[t + 1]; ++k) {
    const size_t x = (size_t)a.ex[k];
    double uiex[3];
    if (ui) {
#pragma unroll
      for (int d = 0; d < 3; ++d) uiex[d] = ui[x + N * d];
    } else if constexpr (STATE) {
#pragma unroll
      for (int d = 0; d < 3; ++d) uiex[d] = q[x + N * d] / rho[x];
    } else {
#pragma unroll
      for (int d = 0; d < 3; ++d) uiex[d] = q[x + N * d];  // q holds u here
    }
    const double nF[3] = {a.nrm[k], a.nrm[(size_t)a.nent + k], a.nrm[2 * (size_t)a.nent + k]};
    const double auxvn = nF[0] * uiex[0] + nF[1] * uiex[1] + nF[2] * uiex[2];
    double tv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) tv[d] = uiex[d] - auxvn * nF[d];
    const double ul = sqrt(tv[0] * tv[0] + tv[1] * tv[1] + tv[2] * tv[2]);
    const double tmag = shear<double>(a.type, ul, a.y[k], nul, rhol, a.zo ? a.zo[k] : 1.0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      acc[d] += a.w[k] * tmag * tv[d];
      last[d] = tmag * tv[d];
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    out[n + N * d] = accumulate ? out[n + N * d] + acc[d] : acc[d];
    if (tauw) tauw[n + N * d] = last[d];
  }
}

// Adjoint of the stage's wall-model term: given the seeds w ([5][npoin], rows 1-3 weigh the
// momentum residual), the transposed Jacobian of sum_k W_k tmag_k tv_k at wall node n with
// respect to the stage state (rho, q, E): the node's own rows (rho through rho_l and nu_l, q and
// E through the EOS temperature of the Sutherland viscosity) into own [5][nw], and the exchange
// velocity q/rho of each entry into ex [4][nent] (rho, q x3; zero with walave_u).  The law's
// derivatives with respect to ul, nu_l and rho_l come from dual numbers through its executed
// iterations.
__global__ void __launch_bounds__(kBlock) k_wall_model_vjp(const Args a, const double* __restrict__ rho,
                                                           const double* __restrict__ q,
                                                           const double* __restrict__ E,
                                                           const double* __restrict__ mu_factor,
                                                           const double* __restrict__ ui,
                                                           const double* __restrict__ w, double gamma, double Rgas,
                                                           double* __restrict__ own, double* __restrict__ ex) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nw) return;
  const size_t N = a.N, n = (size_t)a.wnode[t], NE = (size_t)a.nent, NW = (size_t)a.nw;
  const double rhol = rho[n];
  const double ir = 1.0 / rhol;
  const double qn[3] = {q[n], q[n + N], q[n + 2 * N]};
  const double q2 = qn[0] * qn[0] + qn[1] * qn[1] + qn[2] * qn[2];
  const double u0 = qn[0] * ir, u1 = qn[1] * ir, u2 = qn[2] * ir;
  const double p = rhol * (gamma - 1.0) * (E[n] * ir - 0.5 * (u0 * u0 + u1 * u1 + u2 * u2));
  const double T = p / (rhol * Rgas);
  const double mf = mu_factor[n];
  const double mu = mf * kSuthC1 * (T * sqrt(T)) / (T + kSuthS);
  const double dmu = mf * kSuthC1 * (1.5 * sqrt(T) * (T + kSuthS) - T * sqrt(T)) / ((T + kSuthS) * (T + kSuthS));
  const double nul = mu / rhol;
  const double g[3] = {w[N + n], w[2 * N + n], w[3 * N + n]};
  double nul_b = 0.0, rhol_b = 0.0;
  for (int k = a.wptr[t]; k < a.wptr[t + 1]; ++k) {
    const size_t x = (size_t)a.ex[k];
    double uiex[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) uiex[d] = ui ? ui[x + N * d] : q[x + N * d] / rho[x];
    const double nF[3] = {a.nrm[k], a.nrm[NE + k], a.nrm[2 * NE + k]};
    const double auxvn = nF[0] * uiex[0] + nF[1] * uiex[1] + nF[2] * uiex[2];
    double tv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) tv[d] = uiex[d] - auxvn * nF[d];
    const double ul = sqrt(tv[0] * tv[0] + tv[1] * tv[1] + tv[2] * tv[2]);
    const double zo = a.zo ? a.zo[k] : 1.0, yk = a.y[k];
    const Dual t_ul = shear<Dual>(a.type, Dual{ul, 1.0}, yk, Dual{nul, 0.0}, Dual{rhol, 0.0}, zo);
    const Dual t_nu = shear<Dual>(a.type, Dual{ul, 0.0}, yk, Dual{nul, 1.0}, Dual{rhol, 0.0}, zo);
    const Dual t_rh = shear<Dual>(a.type, Dual{ul, 0.0}, yk, Dual{nul, 0.0}, Dual{rhol, 1.0}, zo);
    const double tmag = t_ul.v;
    const double gt = g[0] * tv[0] + g[1] * tv[1] + g[2] * tv[2];
    const double W = a.w[k];
    nul_b += W * gt * t_nu.d;
    rhol_b += W * gt * t_rh.d;
    double exb[4] = {0.0, 0.0, 0.0, 0.0};
    if (!ui) {
      const double gn = nF[0] * g[0] + nF[1] * g[1] + nF[2] * g[2];
      const double c = ul > 0.0 ? t_ul.d * gt / ul : 0.0;
      double ub[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        // W P (c tv + tmag g), P = I - n n^T (P tv = tv)
        ub[d] = W * (c * tv[d] + tmag * (g[d] - gn * nF[d]));
      }
      const double rx = rho[x];
      exb[0] = -(uiex[0] * ub[0] + uiex[1] * ub[1] + uiex[2] * ub[2]) / rx;
#pragma unroll
      for (int d = 0; d < 3; ++d) exb[1 + d] = ub[d] / rx;
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) ex[(size_t)f * NE + k] = exb[f];
  }
  // own node: rho_l directly and through nu_l = mu(T)/rho; T = (g-1)/R (E/rho - |q|^2/(2 rho^2))
  const double mu_b = nul_b / rhol;
  double rho_b = rhol_b - nul_b * mu / (rhol * rhol);
  const double T_b = mu_b * dmu;
  const double cT = (gamma - 1.0) / Rgas;
  const double E_b = T_b * cT / rhol;
  rho_b += T_b * cT * (-E[n] / (rhol * rhol) + q2 / (rhol * rhol * rhol));
  own[t] = rho_b;
#pragma unroll
  for (int d = 0; d < 3; ++d) own[(1 + d) * NW + t] = -T_b * cT * qn[d] / (rhol * rhol);
  own[4 * NW + t] = E_b;
}

// the adjoint contributions per node in a fixed order: each target (wall node or exchange node)
// sums its own rows and the entries that read it as exchange node; wmbar is [5][npoin]
__global__ void __launch_bounds__(kBlock) k_wall_model_bar(int nt, const int32_t* __restrict__ tnode,
                                                           const int32_t* __restrict__ twall,
                                                           const int32_t* __restrict__ tptr,
                                                           const int32_t* __restrict__ tent, int nw, int nent,
                                                           size_t N, const double* __restrict__ own,
                                                           const double* __restrict__ ex,
                                                           double* __restrict__ wmbar) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nt) return;
  const size_t n = (size_t)tnode[u];
  const int wi = twall[u];
  double acc[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) acc[f] = wi >= 0 ? own[(size_t)f * nw + wi] : 0.0;
  for (int e = tptr[u]; e < tptr[u + 1]; ++e) {
    const size_t k = (size_t)tent[e];
#pragma unroll
    for (int f = 0; f < 4; ++f) acc[f] += ex[(size_t)f * nent + k];
  }
#pragma unroll
  for (int f = 0; f < 5; ++f) wmbar[f * N + n] = acc[f];
}

static Args args_of(const SodMesh* m) {
  const WallModelState& W = m->wmodel;
  Args a{};
  a.nw = W.nw;
  a.wnode = W.wnode;
  a.wptr = W.wptr;
  a.ex = W.ex;
  a.w = W.w;
  a.nrm = W.nrm;
  a.y = W.y;
  a.zo = W.zo;
  a.nent = W.nent;
  a.type = W.type;
  a.N = (size_t)m->npoin;
  return a;
}

}  // namespace wm

int wall_model_stage(SodMesh* m, const double* rho, const double* q0, const double* E, const double* mu_factor,
                     cudaStream_t st) {
  const WallModelState& W = m->wmodel;
  wm::k_wall_model<true><<<(W.nw + wm::kBlock - 1) / wm::kBlock, wm::kBlock, 0, st>>>(
      wm::args_of(m), rho, q0, E, nullptr, mu_factor, W.walave, m->prm.gamma, m->prm.Rgas, W.contrib, 0, W.tauw);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int wall_model_vjp(SodMesh* m, const double* rho, const double* q0, const double* E, const double* mu_factor,
                   const double* w, cudaStream_t st) {
  const WallModelState& W = m->wmodel;
  wm::k_wall_model_vjp<<<(W.nw + wm::kBlock - 1) / wm::kBlock, wm::kBlock, 0, st>>>(
      wm::args_of(m), rho, q0, E, mu_factor, W.walave, w, m->prm.gamma, m->prm.Rgas, W.own_bar, W.ex_bar);
  SOD_CHECK_LAUNCH();
  wm::k_wall_model_bar<<<(W.nt + wm::kBlock - 1) / wm::kBlock, wm::kBlock, 0, st>>>(
      W.nt, W.tnode, W.twall, W.tptr, W.tent, W.nw, W.nent, (size_t)m->npoin, W.own_bar, W.ex_bar, W.wmbar);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

void wall_model_free(SodMesh* m) {
  WallModelState& W = m->wmodel;
  void* ptrs[] = {W.wnode, W.wptr, W.ex, W.w, W.nrm, W.y, W.zo, W.contrib, W.tauw,
                  W.tnode, W.twall, W.tptr, W.tent, W.own_bar, W.ex_bar, W.wmbar};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  W = WallModelState{};
}

}  // namespace sod

using namespace sod;

extern "C" {

int sod_mesh_set_wall_model(SodMesh* m, int32_t type, int32_t nboun, int32_t npbou, const int32_t* bound,
                            const double* bounorm, const double* wgp_b, int32_t numBoundsWM,
                            const int32_t* listBoundsWM, const int32_t* point2elem, const double* coord,
                            const double* normalsAtNodes, const double* zo, const double* walave_u) {
  SOD_ARG(m, "mesh null");
  SOD_ARG(m->nmember == 0, "a wall model on an ensemble mesh is not supported");
  if (m->has_slaves && numBoundsWM > 0) {
    set_error("sod_mesh_set_wall_model on a mesh with periodic slave rows (lpoin_w) is not supported");
    return SOD_ERR_UNSUPPORTED;
  }
  for (auto& kv : m->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  m->graphs.clear();
  wall_model_free(m);
  if (numBoundsWM <= 0) return SOD_OK;
  SOD_ARG(type == wm::kReichardt || type == wm::kABL, "unknown wall-model type");
  SOD_ARG(type == wm::kReichardt || walave_u, "the ABL wall model needs the time-averaged velocity (walave_u)");
  SOD_ARG(type != wm::kABL || zo, "the ABL wall model needs zo");
  SOD_ARG(npbou == NP1 * NP1 && nboun > 0, "faces of 16 nodes expected");
  SOD_ARG(bound && bounorm && wgp_b && listBoundsWM && point2elem && coord && normalsAtNodes, "null argument");
  const int N = m->npoin, E = m->nelem, base = m->index_base;
  // element connectivity in the internal natural order (d = i + 4j + 16k)
  std::vector<int32_t> conn((size_t)E * NN);
  SOD_CUDA(cudaMemcpy(conn.data(), m->econn, sizeof(int32_t) * conn.size(), cudaMemcpyDeviceToHost));
  struct Entry {
    int32_t node, face, ex;
    double w, n[3], y, zo;
  };
  std::vector<Entry> ent;
  ent.reserve((size_t)numBoundsWM * npbou);
  const size_t NB = (size_t)nboun;
  for (int f = 0; f < numBoundsWM; ++f) {
    const int ib = listBoundsWM[f] - base;
    SOD_ARG(ib >= 0 && ib < nboun, "listBoundsWM entry out of range");
    // the element of the face: point2elem of an interior face node (one natural coordinate on
    // an element face, the other two interior), and the face's normal direction there
    int el = -1, dir = -1, side = -1;
    for (int a = 0; a < npbou && el < 0; ++a) {
      const int nd = bound[ib + NB * a] - base;
      SOD_ARG(nd >= 0 && nd < N, "bound entry out of range");
      const int e = point2elem[nd] - base;
      SOD_ARG(e >= 0 && e < E, "point2elem entry out of range");
      for (int d = 0; d < NN; ++d) {
        if (conn[(size_t)e * NN + d] != nd) continue;
        const int c[3] = {d & 3, (d >> 2) & 3, d >> 4};
        int nend = 0, dd = -1;
        for (int r = 0; r < 3; ++r)
          if (c[r] == 0 || c[r] == 3) { ++nend; dd = r; }
        if (nend == 1) { el = e; dir = dd; side = c[dd]; }
        break;
      }
    }
    SOD_ARG(el >= 0, "no interior face node found for a wall-model face");
    for (int a = 0; a < npbou; ++a) {
      const int nd = bound[ib + NB * a] - base;
      int loc = -1;
      for (int d = 0; d < NN; ++d)
        if (conn[(size_t)el * NN + d] == nd) { loc = d; break; }
      SOD_ARG(loc >= 0, "a face node is not a node of the face's element");
      int c[3] = {loc & 3, (loc >> 2) & 3, loc >> 4};
      c[dir] = side == 0 ? 3 : 0;  // the opposite face of the element
      const int xn = conn[(size_t)el * NN + c[0] + 4 * c[1] + 16 * c[2]];
      Entry en{};
      en.node = nd;
      en.face = f;
      en.ex = xn;
      double bm = 0.0;
      for (int r = 0; r < 3; ++r) {
        const double b = bounorm[ib + NB * (size_t)(3 * a + r)];
        bm += b * b;
      }
      en.w = std::sqrt(bm) * wgp_b[a];
      double yy = 0.0;
      for (int r = 0; r < 3; ++r) {
        en.n[r] = normalsAtNodes[nd + (size_t)N * r];
        yy += en.n[r] * (coord[xn + (size_t)N * r] - coord[nd + (size_t)N * r]);
      }
      en.y = std::fabs(yy);
      en.zo = zo ? zo[nd] : 1.0;
      ent.push_back(en);
    }
  }
  std::stable_sort(ent.begin(), ent.end(), [](const Entry& x, const Entry& y) { return x.node < y.node; });
  std::vector<int32_t> wnode, wptr, ex;
  std::vector<double> w, nrm(3 * ent.size()), yv, zv;
  const size_t ne = ent.size();
  for (size_t k = 0; k < ne; ++k) {
    if (k == 0 || ent[k].node != ent[k - 1].node) {
      wnode.push_back(ent[k].node);
      wptr.push_back((int32_t)k);
    }
    ex.push_back(ent[k].ex);
    w.push_back(ent[k].w);
    for (int r = 0; r < 3; ++r) nrm[r * ne + k] = ent[k].n[r];
    yv.push_back(ent[k].y);
    zv.push_back(ent[k].zo);
  }
  wptr.push_back((int32_t)ne);
  WallModelState& W = m->wmodel;
  auto alloc = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
  const size_t nw = wnode.size();
  if (!(alloc((void**)&W.wnode, sizeof(int32_t) * nw) && alloc((void**)&W.wptr, sizeof(int32_t) * (nw + 1)) &&
        alloc((void**)&W.ex, sizeof(int32_t) * ne) && alloc((void**)&W.w, sizeof(double) * ne) &&
        alloc((void**)&W.nrm, sizeof(double) * 3 * ne) && alloc((void**)&W.y, sizeof(double) * ne) &&
        alloc((void**)&W.zo, sizeof(double) * ne) && alloc((void**)&W.contrib, sizeof(double) * 3 * (size_t)N) &&
        alloc((void**)&W.tauw, sizeof(double) * 3 * (size_t)N))) {
    wall_model_free(m);
    set_error("sod_mesh_set_wall_model: device allocation failed");
    return SOD_ERR_NOMEM;
  }
  // adjoint targets: wall nodes and exchange nodes (ascending), with the entries reading each
  // target as exchange node
  std::vector<int32_t> tnode, twall, tptr, tent;
  {
    std::vector<std::pair<int32_t, int32_t>> xe;  // (exchange node, entry)
    for (size_t k = 0; k < ne; ++k) xe.emplace_back(ex[k], (int32_t)k);
    std::sort(xe.begin(), xe.end());
    std::vector<int32_t> all(wnode.begin(), wnode.end());
    for (auto& p : xe) all.push_back(p.first);
    std::sort(all.begin(), all.end());
    all.erase(std::unique(all.begin(), all.end()), all.end());
    size_t xi = 0;
    for (int32_t nd : all) {
      auto it = std::lower_bound(wnode.begin(), wnode.end(), nd);
      tnode.push_back(nd);
      twall.push_back(it != wnode.end() && *it == nd ? (int32_t)(it - wnode.begin()) : -1);
      tptr.push_back((int32_t)tent.size());
      while (xi < xe.size() && xe[xi].first == nd) tent.push_back(xe[xi++].second);
    }
    tptr.push_back((int32_t)tent.size());
  }
  const size_t nt = tnode.size();
  if (!(alloc((void**)&W.tnode, sizeof(int32_t) * nt) && alloc((void**)&W.twall, sizeof(int32_t) * nt) &&
        alloc((void**)&W.tptr, sizeof(int32_t) * (nt + 1)) && alloc((void**)&W.tent, sizeof(int32_t) * (ne + 1)) &&
        alloc((void**)&W.own_bar, sizeof(double) * 5 * nw) && alloc((void**)&W.ex_bar, sizeof(double) * 4 * ne) &&
        alloc((void**)&W.wmbar, sizeof(double) * 5 * (size_t)N))) {
    wall_model_free(m);
    set_error("sod_mesh_set_wall_model: device allocation failed");
    return SOD_ERR_NOMEM;
  }
  SOD_CUDA(cudaMemcpy(W.tnode, tnode.data(), sizeof(int32_t) * nt, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(W.twall, twall.data(), sizeof(int32_t) * nt, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(W.tptr, tptr.data(), sizeof(int32_t) * (nt + 1), cudaMemcpyHostToDevice));
  if (!tent.empty()) SOD_CUDA(cudaMemcpy(W.tent, tent.data(), sizeof(int32_t) * tent.size(), cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemset(W.wmbar, 0, sizeof(double) * 5 * (size_t)N));
  W.nt = (int)nt;
  W.nw = (int)nw;
  W.nent = (int)ne;
  W.type = type;
  W.walave = walave_u;
  SOD_CUDA(cudaMemcpy(W.wnode, wnode.data(), sizeof(int32_t) * nw, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(W.wptr, wptr.data(), sizeof(int32_t) * (nw + 1), cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(W.ex, ex.data(), sizeof(int32_t) * ne, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(W.w, w.data(), sizeof(double) * ne, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(W.nrm, nrm.data(), sizeof(double) * 3 * ne, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(W.y, yv.data(), sizeof(double) * ne, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(W.zo, zv.data(), sizeof(double) * ne, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemset(W.contrib, 0, sizeof(double) * 3 * (size_t)N));
  SOD_CUDA(cudaMemset(W.tauw, 0, sizeof(double) * 3 * (size_t)N));
  return SOD_OK;
}

int sod_wall_model(SodMesh* m, const double* rho, const double* u, const double* mu_fluid, double* Rdiff,
                   double* tauw, sod_stream_t stream) {
  SOD_ARG(m && rho && u && mu_fluid && Rdiff, "null argument");
  SOD_ARG(m->wmodel.nw > 0, "no wall model registered (sod_mesh_set_wall_model)");
  const WallModelState& W = m->wmodel;
  wm::k_wall_model<false><<<(W.nw + wm::kBlock - 1) / wm::kBlock, wm::kBlock, 0, (cudaStream_t)stream>>>(
      wm::args_of(m), rho, u, nullptr, mu_fluid, nullptr, nullptr, 0.0, 0.0, Rdiff, 1, tauw);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

int sod_wall_model_tauw(SodMesh* m, double* tauw, sod_stream_t stream) {
  SOD_ARG(m && tauw, "null argument");
  SOD_ARG(m->wmodel.nw > 0, "no wall model registered (sod_mesh_set_wall_model)");
  SOD_CUDA(cudaMemcpyAsync(tauw, m->wmodel.tauw, sizeof(double) * 3 * (size_t)m->npoin, cudaMemcpyDeviceToDevice,
                           (cudaStream_t)stream));
  return SOD_OK;
}

}  // extern "C"
