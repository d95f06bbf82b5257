// Penalisation buffer zone of rk_4_main (flag_buffer_on): updateBuffer (time_integ.f90:510-589)
// on every stage state (:251) and on the updated state (:429), before the boundary routine.
//
// The zone factor xi of a node depends only on its coordinates and the zone parameters, so it
// is formed once on the host (sod_mesh_set_buffer, the reference's formula in FP64) for the
// nodes inside an enabled zone, which are compacted into an ascending list with their u_buffer;
// each application is one thread per zone node.  Nodes outside every zone have xi = 1, for which
// the reference's update is the identity up to the rounding of u_b rho + (q - u_b rho); they are
// left alone.  After the final update the zone nodes' EOS and Sutherland viscosity are
// re-evaluated and, without boundaries, the entropy normalisation too (the boundary routine's
// final pass recomputes it otherwise).  The update is affine in the state with a constant
// Jacobian (rho' = xi rho + c, q' = xi q + (1 - xi) u_b rho + ..., E' = xi E + c), so its
// adjoint is a fixed per-node map.
//
// The other optional per-node input of rk_4_main, the constant momentum source term, is
// registered here too (sod_mesh_set_source_term); the node gather applies it.
#include "sod_internal.cuh"
#include <cmath>
#include <vector>

namespace sod {
namespace zone {

constexpr int kBlock = 256;
static int grid_of(int n) { return (n + kBlock - 1) / kBlock; }

struct EosArgs {
  double *u, *pr, *e_int, *csound, *machno, *Tem, *eta, *mu_fluid;
  const double* mu_factor;
  double gamma, Rgas;
};

// updateBuffer's loop body (time_integ.f90:580-585) for zone node b: q from the old rho, then E
// and rho
__global__ void __launch_bounds__(kBlock) k_zone_apply(int nb, const int32_t* __restrict__ node,
                                                       const double* __restrict__ xi, const double* __restrict__ ub,
                                                       size_t N, double* rho, double* q, double* E, double rho_inf,
                                                       double E_inf, int eos, EosArgs o) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const size_t n = (size_t)node[b];
  const double x = xi[b];
  const double r = rho[n];
  double qq[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double ur = ub[(size_t)d * nb + b] * r;
    qq[d] = ur + x * (q[n + N * d] - ur);
    q[n + N * d] = qq[d];
  }
  const double e = E_inf + x * (E[n] - E_inf);
  const double rn = rho_inf + x * (r - rho_inf);
  E[n] = e;
  rho[n] = rn;
  if (eos)
    eos_store(n, N, rn, qq, e, o.gamma, o.Rgas, o.u, o.pr, o.e_int, o.csound, o.machno, o.Tem, o.eta, o.mu_fluid,
              o.mu_factor);
}

// transpose of the update's Jacobian on the adjoint columns vbar ([5][npoin]) of zone node b
__global__ void __launch_bounds__(kBlock) k_zone_adjoint(int nb, const int32_t* __restrict__ node,
                                                         const double* __restrict__ xi, const double* __restrict__ ub,
                                                         size_t N, double* vbar) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const size_t n = (size_t)node[b];
  const double x = xi[b];
  double s = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double qb = vbar[(1 + d) * N + n];
    s += ub[(size_t)d * nb + b] * qb;
    vbar[(1 + d) * N + n] = x * qb;
  }
  vbar[n] = x * vbar[n] + (1.0 - x) * s;
  vbar[4 * N + n] = x * vbar[4 * N + n];
}

static int apply(SodMesh* m, double* rho, double* q, double* E, const EosArgs* eos, cudaStream_t st) {
  const ZoneState& z = m->zone;
  EosArgs o{};
  if (eos) o = *eos;
  k_zone_apply<<<grid_of(z.nb), kBlock, 0, st>>>(z.nb, z.node, z.xi, z.ub, (size_t)m->npoin, rho, q, E, z.rho_inf,
                                                 z.E_inf, eos ? 1 : 0, o);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

// the zone factor of one side (time_integ.f90:536 and the five others)
static double side_factor(double xb) {
  const double c1 = 0.01, c2 = 10.0;
  return (1.0 - c1 * xb * xb) * (1.0 - (1.0 - std::exp(c2 * xb * xb)) / (1.0 - std::exp(c2)));
}

}  // namespace zone

int zone_stage(SodMesh* m, double* ys, cudaStream_t st) {
  const size_t N = m->npoin;
  return zone::apply(m, ys, ys + N, ys + 4 * N, nullptr, st);
}

int zone_final(SodMesh* m, SodState* s, cudaStream_t st) {
  zone::EosArgs o{s->u, s->pr, s->e_int, s->csound, s->machno, s->Tem, s->eta, s->mu_fluid, s->mu_factor,
                  m->prm.gamma, m->prm.Rgas};
  if (int rc = zone::apply(m, s->rho, s->q, s->E, &o, st)) return rc;
  return m->bc.nb > 0 ? SOD_OK : eta_stats(m, s->eta, st);
}

int zone_adjoint(SodMesh* m, double* vbar, cudaStream_t st) {
  const ZoneState& z = m->zone;
  zone::k_zone_adjoint<<<zone::grid_of(z.nb), zone::kBlock, 0, st>>>(z.nb, z.node, z.xi, z.ub, (size_t)m->npoin,
                                                                     vbar);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

void zone_free(SodMesh* m) {
  ZoneState& z = m->zone;
  void* ptrs[] = {z.node, z.xi, z.ub, z.zmap};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  z = ZoneState{};
}

}  // namespace sod

using namespace sod;

extern "C" {

int sod_mesh_set_buffer(SodMesh* m, const SodBufferParams* p, const double* coord, const double* u_buffer) {
  SOD_ARG(m, "mesh null");
  SOD_ARG(m->nmember == 0, "a buffer zone on an ensemble mesh is not supported");
  for (auto& kv : m->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  m->graphs.clear();
  zone_free(m);
  if (!p) return SOD_OK;
  SOD_ARG(coord, "coord required");
  SOD_ARG(p->gamma_inf != 1.0, "gamma_inf must differ from 1");
  const int on[6] = {p->on_east, p->on_west, p->on_north, p->on_south, p->on_top, p->on_bottom};
  const double mn[6] = {p->e_min, p->w_min, p->n_min, p->s_min, p->t_min, p->b_min};
  const double sz[6] = {p->e_size, p->w_size, p->n_size, p->s_size, p->t_size, p->b_size};
  for (int f = 0; f < 6; ++f) SOD_ARG(!on[f] || sz[f] != 0.0, "an enabled zone needs a nonzero size");
  const size_t N = m->npoin;
  std::vector<int32_t> node;
  std::vector<double> xi;
  for (size_t n = 0; n < N; ++n) {
    if (m->has_slaves && m->slave_host[n]) continue;  // updateBuffer runs over lpoin_w (time_integ.f90:529)
    double x = 1.0;
    bool in = false;
    for (int f = 0; f < 6; ++f) {
      if (!on[f]) continue;
      const double xs = coord[n + N * (size_t)(f / 2)];  // east/west: x, north/south: y, top/bottom: z
      const bool upper = (f % 2) == 0;                    // east, north, top: beyond the minimum
      if (upper ? xs > mn[f] : xs < mn[f]) {
        const double xb = upper ? (xs - mn[f]) / sz[f] : (mn[f] - xs) / sz[f];
        x = std::fmin(zone::side_factor(xb), x);
        in = true;
      }
    }
    if (in) {
      node.push_back((int32_t)n);
      xi.push_back(x);
    }
  }
  const int nb = (int)node.size();
  if (nb == 0) return SOD_OK;
  std::vector<double> ub((size_t)3 * nb, 0.0);
  if (u_buffer)
    for (int b = 0; b < nb; ++b)
      for (int d = 0; d < 3; ++d) ub[(size_t)d * nb + b] = u_buffer[(size_t)node[b] + N * d];
  ZoneState& z = m->zone;
  auto alloc = [&](void** q, size_t bytes) { return cudaMalloc(q, bytes) == cudaSuccess; };
  if (!(alloc((void**)&z.node, sizeof(int32_t) * nb) && alloc((void**)&z.xi, sizeof(double) * nb) &&
        alloc((void**)&z.ub, sizeof(double) * 3 * nb) && alloc((void**)&z.zmap, sizeof(int32_t) * N))) {
    zone_free(m);
    set_error("sod_mesh_set_buffer: device allocation failed");
    return SOD_ERR_NOMEM;
  }
  z.nb = nb;
  z.rho_inf = p->rho_inf;
  z.E_inf = (p->rho_inf * 0.5 * (p->u_inf * p->u_inf) + p->p_inf / (p->gamma_inf - 1.0));
  SOD_CUDA(cudaMemcpy(z.node, node.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(z.xi, xi.data(), sizeof(double) * nb, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(z.ub, ub.data(), sizeof(double) * 3 * nb, cudaMemcpyHostToDevice));
  {
    std::vector<int32_t> zmap(N, -1);
    for (int b = 0; b < nb; ++b) zmap[node[b]] = b;
    SOD_CUDA(cudaMemcpy(z.zmap, zmap.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
  }
  return SOD_OK;
}

int sod_mesh_set_source_term(SodMesh* m, const double* source_term) {
  SOD_ARG(m, "mesh null");
  SOD_ARG(m->nmember == 0 || !source_term, "a source term on an ensemble mesh is not supported");
  if (m->source != source_term) {
    for (auto& kv : m->graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    m->graphs.clear();
  }
  m->source = source_term;
  return SOD_OK;
}

int sod_update_buffer(SodMesh* m, double* rho, double* q, double* E, sod_stream_t stream) {
  SOD_ARG(m && rho && q && E, "null argument");
  if (m->zone.nb == 0) return SOD_OK;
  return zone::apply(m, rho, q, E, nullptr, (cudaStream_t)stream);
}

}  // extern "C"
