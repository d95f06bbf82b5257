// Ensemble batching: many independent periodic meshes advanced together (sm_100a).
//
// The reference runs an ensemble as separate MPI applications (MPMD colour per member,
// mod_mpi.f90:39-51, TGVMultiSolver.f90:30-60), one solver per process.  Here the members'
// meshes are concatenated into one block-diagonal mesh: every RK stage is ONE fused-RHS launch
// and ONE gather launch over all members, whatever their sizes, and the whole step is captured
// once in a CUDA graph.  What differs per member - the time step, the entropy normalisation
// (mean and max deviation of eta over the member's nodes) and the CFL reduction - is looked up
// through node->member and element->member maps; Reynolds numbers differ through each member's
// own mu_factor.  Members must share the element order and the 1-D derivative table.
#include "sod_internal.cuh"
#include <cstring>
#include <cmath>
#include <vector>

namespace sod {
int run_step(SodMesh* m, SodState* s, const double* dt_dev, double* dt_next, bool mixed, cudaStream_t st,
             cudaEvent_t* ev, double* stage_store, cudaEvent_t state_done);
int launch_visc_dt(SodMesh* m, const SodState* s, double* dt_out, float* mue32, cudaStream_t st);
}  // namespace sod

struct SodBatch {
  SodMesh* mesh = nullptr;          // concatenated mesh (owned)
  int nmember = 0;
  std::vector<int32_t> node_off, elem_off;  // host copies, nmember+1
  SodState st{};                     // device state over all members (owned)
  double* dt = nullptr;              // [nmember] device
  double* ref_mue = nullptr;         // (nelem,64) reference-layout scratch for mu_e get/set
  std::unordered_map<uint64_t, sod::GraphEntry> graphs;
};

namespace sod {
namespace batch {

__global__ void k_offset_copy(const int32_t* __restrict__ src, int32_t* __restrict__ dst, int64_t n, int32_t add) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = src[t] + add;
}
__global__ void k_fill(int32_t* __restrict__ dst, int64_t n, int32_t v) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = v;
}

}  // namespace batch
}  // namespace sod

using namespace sod;
using namespace sod::batch;

static void free_state(SodState& s) {
  double* ptrs[] = {s.rho, s.q, s.E, s.u, s.pr, s.Tem, s.e_int, s.eta, s.csound, s.machno, s.mu_fluid, s.mu_factor,
                    s.mu_e, s.Reta};
  for (double* p : ptrs)
    if (p) cudaFree(p);
}

extern "C" {

void sod_batch_destroy(SodBatch* B) {
  if (!B) return;
  for (auto& kv : B->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  free_state(B->st);
  if (B->dt) cudaFree(B->dt);
  if (B->ref_mue) cudaFree(B->ref_mue);
  if (B->mesh) {
    SodMesh* m = B->mesh;
    void* ptrs[] = {m->node_member, m->elem_member, m->member_node_off, m->member_scal, m->member_dt_bits};
    for (void* p : ptrs)
      if (p) cudaFree(p);
    m->node_member = m->elem_member = m->member_node_off = nullptr;
    m->member_scal = m->member_dt_bits = nullptr;
    sod_mesh_destroy(m);
  }
  delete B;
}

int sod_batch_create(SodMesh* const* meshes, int nmesh, SodBatch** out) {
  SOD_ARG(meshes && nmesh > 0 && out, "meshes/nmesh/out");
  *out = nullptr;
  for (int i = 0; i < nmesh; ++i) SOD_ARG(meshes[i], "null member mesh");
  for (int i = 0; i < nmesh; ++i)
    if (meshes[i]->has_slaves) {
      set_error("sod_batch_create: members with periodic slave rows (lpoin_w) are not supported");
      return SOD_ERR_UNSUPPORTED;
    }
  for (int i = 0; i < nmesh; ++i)
    if (meshes[i]->bc.nb > 0 || meshes[i]->zone.nb > 0 || meshes[i]->source || meshes[i]->wmodel.nw > 0) {
      set_error("sod_batch_create: members with boundaries, a buffer zone, a source term or a wall model are not supported");
      return SOD_ERR_UNSUPPORTED;
    }
  const SodMesh* m0 = meshes[0];
  int64_t E = 0, N = 0;
  SodBatch* B = new SodBatch();
  B->nmember = nmesh;
  B->node_off.assign(nmesh + 1, 0);
  B->elem_off.assign(nmesh + 1, 0);
  for (int i = 0; i < nmesh; ++i) {
    const SodMesh* mi = meshes[i];
    if (std::memcmp(mi->perm_a_of_d, m0->perm_a_of_d, sizeof(m0->perm_a_of_d)) != 0) {
      delete B;
      set_error("invalid argument: member %d has a different element node order", i);
      return SOD_ERR_ARG;
    }
    for (int r = 0; r < NP1; ++r)
      for (int c = 0; c < NP1; ++c)
        if (std::fabs(mi->D.d[r][c] - m0->D.d[r][c]) > 1e-14 * (1.0 + std::fabs(m0->D.d[r][c]))) {
          delete B;
          set_error("invalid argument: member %d has a different derivative table", i);
          return SOD_ERR_ARG;
        }
    E += mi->nelem;
    N += mi->npoin;
    B->node_off[i + 1] = (int32_t)N;
    B->elem_off[i + 1] = (int32_t)E;
  }
  if (E * NN >= ((int64_t)1 << 31) || N >= ((int64_t)1 << 31)) {
    delete B;
    set_error("invalid argument: ensemble too large for int32 indices");
    return SOD_ERR_ARG;
  }
  SodMesh* m = new SodMesh();
  B->mesh = m;
  m->nelem = (int32_t)E;
  m->npoin = (int32_t)N;
  m->device = m0->device;
  m->prm = m0->prm;
  m->D = m0->D;
  std::memcpy(m->wgp_nat, m0->wgp_nat, sizeof(m->wgp_nat));
  std::memcpy(m->perm_a_of_d, m0->perm_a_of_d, sizeof(m->perm_a_of_d));
  std::memcpy(m->perm_d_of_a, m0->perm_d_of_a, sizeof(m->perm_d_of_a));
  m->nmember = nmesh;
  auto fail = [&](const char* what) {
    set_error("sod_batch_create: %s", what);
    sod_batch_destroy(B);
    return SOD_ERR_NOMEM;
  };
#define BALLOC(p, bytes) if (cudaMalloc(&(p), (bytes)) != cudaSuccess) return fail("cudaMalloc " #p)
  BALLOC(m->econn, sizeof(int32_t) * E * NN);
  BALLOC(m->n2e_ptr, sizeof(int32_t) * (N + 1));
  BALLOC(m->n2e, sizeof(int32_t) * E * NN);
  BALLOC(m->geo64, sizeof(double) * E * NGEO * NN);
  BALLOC(m->Ml, sizeof(double) * N);
  BALLOC(m->helem, sizeof(double) * E);
  BALLOC(m->helem_l, sizeof(double) * E * NN);
  BALLOC(m->jratio, sizeof(double) * E);
  BALLOC(m->mue_int, sizeof(double) * E * NN);
  BALLOC(m->a_of_d_dev, sizeof(int32_t) * NN);
  BALLOC(m->node_member, sizeof(int32_t) * N);
  BALLOC(m->elem_member, sizeof(int32_t) * E);
  BALLOC(m->member_node_off, sizeof(int32_t) * (nmesh + 1));
  BALLOC(m->member_scal, sizeof(double) * 2 * nmesh);
  BALLOC(m->member_dt_bits, sizeof(double) * nmesh);
  BALLOC(B->dt, sizeof(double) * nmesh);
  BALLOC(B->ref_mue, sizeof(double) * E * NN);
  {
    double** fields[] = {&B->st.rho, &B->st.E, &B->st.pr, &B->st.Tem, &B->st.e_int, &B->st.eta, &B->st.csound,
                         &B->st.machno, &B->st.mu_fluid, &B->st.mu_factor, &B->st.Reta};
    for (double** f : fields) BALLOC(*f, sizeof(double) * N);
    BALLOC(B->st.q, sizeof(double) * 3 * N);
    BALLOC(B->st.u, sizeof(double) * 3 * N);
    BALLOC(B->st.mu_e, sizeof(double) * E * NN);
  }
#undef BALLOC
  cudaMemcpy(m->a_of_d_dev, m0->a_of_d_dev, sizeof(int32_t) * NN, cudaMemcpyDeviceToDevice);
  cudaMemset(m->mue_int, 0, sizeof(double) * E * NN);
  cudaMemset(B->st.mu_e, 0, sizeof(double) * E * NN);
  cudaMemcpy(m->member_node_off, B->node_off.data(), sizeof(int32_t) * (nmesh + 1), cudaMemcpyHostToDevice);
  int64_t nnz_off = 0;
  for (int i = 0; i < nmesh; ++i) {
    const SodMesh* mi = meshes[i];
    const int64_t eo = B->elem_off[i], no = B->node_off[i], Ei = mi->nelem, Ni = mi->npoin;
    k_offset_copy<<<256, 256>>>(mi->econn, m->econn + eo * NN, Ei * NN, (int32_t)no);
    k_offset_copy<<<256, 256>>>(mi->n2e, m->n2e + eo * NN, Ei * NN, (int32_t)(eo * NN));
    // n2e_ptr of member i shifted by the entries of the members before it (the last entry is
    // written by the next member or, for the last member, below)
    k_offset_copy<<<64, 256>>>(mi->n2e_ptr, m->n2e_ptr + no, Ni + 1, (int32_t)nnz_off);
    nnz_off += Ei * NN;
    cudaMemcpy(m->geo64 + eo * NGEO * NN, mi->geo64, sizeof(double) * Ei * NGEO * NN, cudaMemcpyDeviceToDevice);
    cudaMemcpy(m->Ml + no, mi->Ml, sizeof(double) * Ni, cudaMemcpyDeviceToDevice);
    cudaMemcpy(m->helem + eo, mi->helem, sizeof(double) * Ei, cudaMemcpyDeviceToDevice);
    cudaMemcpy(m->helem_l + eo * NN, mi->helem_l, sizeof(double) * Ei * NN, cudaMemcpyDeviceToDevice);
    cudaMemcpy(m->jratio + eo, mi->jratio, sizeof(double) * Ei, cudaMemcpyDeviceToDevice);
    k_fill<<<64, 256>>>(m->node_member + no, Ni, i);
    k_fill<<<64, 256>>>(m->elem_member + eo, Ei, i);
    g_launches.fetch_add(5);
  }
  cudaError_t err = cudaDeviceSynchronize();
  if (err != cudaSuccess) {
    set_error("sod_batch_create: %s", cudaGetErrorString(err));
    sod_batch_destroy(B);
    return SOD_ERR_CUDA;
  }
  *out = B;
  return SOD_OK;
}

// Host state of one member in the reference layouts (rho, q(N_i,3), E, mu_factor, mu_e(E_i,64)
// required; u(N_i,3), csound, mu_fluid optional - used by sod_batch_adapt_dt).
int sod_batch_set_member(SodBatch* B, int member, const SodState* h) {
  SOD_ARG(B && h && member >= 0 && member < B->nmember, "batch/member/state");
  SOD_ARG(h->rho && h->q && h->E && h->mu_factor && h->mu_e, "rho, q, E, mu_factor, mu_e required");
  const int64_t no = B->node_off[member], Ni = B->node_off[member + 1] - no;
  const int64_t eo = B->elem_off[member], Ei = B->elem_off[member + 1] - eo;
  const int64_t N = B->mesh->npoin, E = B->mesh->nelem;
  SOD_CUDA(cudaMemcpy(B->st.rho + no, h->rho, 8 * Ni, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(B->st.E + no, h->E, 8 * Ni, cudaMemcpyHostToDevice));
  SOD_CUDA(cudaMemcpy(B->st.mu_factor + no, h->mu_factor, 8 * Ni, cudaMemcpyHostToDevice));
  for (int c = 0; c < 3; ++c) {
    SOD_CUDA(cudaMemcpy(B->st.q + c * N + no, h->q + c * Ni, 8 * Ni, cudaMemcpyHostToDevice));
    if (h->u) SOD_CUDA(cudaMemcpy(B->st.u + c * N + no, h->u + c * Ni, 8 * Ni, cudaMemcpyHostToDevice));
  }
  if (h->csound) SOD_CUDA(cudaMemcpy(B->st.csound + no, h->csound, 8 * Ni, cudaMemcpyHostToDevice));
  if (h->mu_fluid) SOD_CUDA(cudaMemcpy(B->st.mu_fluid + no, h->mu_fluid, 8 * Ni, cudaMemcpyHostToDevice));
  for (int a = 0; a < NN; ++a)
    SOD_CUDA(cudaMemcpy(B->st.mu_e + a * E + eo, h->mu_e + a * Ei, 8 * Ei, cudaMemcpyHostToDevice));
  return SOD_OK;
}

int sod_batch_get_member(SodBatch* B, int member, SodState* h) {
  SOD_ARG(B && h && member >= 0 && member < B->nmember, "batch/member/state");
  SOD_CUDA(cudaDeviceSynchronize());
  const int64_t no = B->node_off[member], Ni = B->node_off[member + 1] - no;
  const int64_t eo = B->elem_off[member], Ei = B->elem_off[member + 1] - eo;
  const int64_t N = B->mesh->npoin, E = B->mesh->nelem;
  struct F { double* hst; double* dev; } sc[] = {{h->rho, B->st.rho}, {h->E, B->st.E}, {h->pr, B->st.pr},
      {h->Tem, B->st.Tem}, {h->e_int, B->st.e_int}, {h->eta, B->st.eta}, {h->csound, B->st.csound},
      {h->machno, B->st.machno}, {h->mu_fluid, B->st.mu_fluid}, {h->Reta, B->st.Reta}};
  for (auto& f : sc)
    if (f.hst) SOD_CUDA(cudaMemcpy(f.hst, f.dev + no, 8 * Ni, cudaMemcpyDeviceToHost));
  for (int c = 0; c < 3; ++c) {
    if (h->q) SOD_CUDA(cudaMemcpy(h->q + c * Ni, B->st.q + c * N + no, 8 * Ni, cudaMemcpyDeviceToHost));
    if (h->u) SOD_CUDA(cudaMemcpy(h->u + c * Ni, B->st.u + c * N + no, 8 * Ni, cudaMemcpyDeviceToHost));
  }
  if (h->mu_e)
    for (int a = 0; a < NN; ++a)
      SOD_CUDA(cudaMemcpy(h->mu_e + a * Ei, B->st.mu_e + a * E + eo, 8 * Ei, cudaMemcpyDeviceToHost));
  return SOD_OK;
}

int sod_batch_set_dt(SodBatch* B, const double* dt_host) {
  SOD_ARG(B && dt_host, "batch/dt");
  SOD_CUDA(cudaMemcpy(B->dt, dt_host, sizeof(double) * B->nmember, cudaMemcpyHostToDevice));
  return SOD_OK;
}

int sod_batch_get_dt(SodBatch* B, double* dt_host) {
  SOD_ARG(B && dt_host, "batch/dt");
  SOD_CUDA(cudaMemcpy(dt_host, B->dt, sizeof(double) * B->nmember, cudaMemcpyDeviceToHost));
  return SOD_OK;
}

int sod_batch_mesh(SodBatch* B, SodMesh** mesh) {
  SOD_ARG(B && mesh, "batch/mesh");
  *mesh = B->mesh;
  return SOD_OK;
}

int sod_batch_rk4_steps(SodBatch* B, int nsteps, SodPrecision prec, sod_stream_t stream) {
  SOD_ARG(B && nsteps >= 0, "batch/nsteps");
  SOD_ARG(prec == SOD_FP64 || prec == SOD_MIXED, "precision");
  cudaStream_t st = (cudaStream_t)stream;
  SodMesh* m = B->mesh;
  const bool mixed = prec == SOD_MIXED;
  int rc = ensure_step_buffers(m, mixed);
  if (rc) return rc;
  rc = mesh_ref_to_internal_elem(m, B->st.mu_e, m->mue_int, st);
  if (rc) return rc;
  if (mixed) {
    rc = launch_copy_f32(m->mue_int, m->mue32, (int64_t)m->nelem * NN, st);
    if (rc) return rc;
  }
  if (nsteps > 0) {
    const uint64_t key = ((uint64_t)mixed << 40) ^ ((uint64_t)m->persist_ctas[mixed ? 1 : 0] << 16) ^
                         (uint64_t)m->tuned_epb[mixed ? 1 : 0];
    auto it = B->graphs.find(key);
    if (it == B->graphs.end()) {
      cudaStream_t cap;
      SOD_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      cudaGraph_t graph;
      const int64_t before = g_launches.load();
      SOD_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
      rc = run_step(m, &B->st, B->dt, B->dt, mixed, cap, nullptr, nullptr, nullptr);
      cudaError_t ce = cudaStreamEndCapture(cap, &graph);
      cudaStreamDestroy(cap);
      if (rc) return rc;
      if (ce != cudaSuccess) {
        set_error("batch graph capture failed: %s", cudaGetErrorString(ce));
        return SOD_ERR_CUDA;
      }
      GraphEntry ge;
      ge.nkernels = (int)(g_launches.load() - before);
      g_launches.fetch_sub(ge.nkernels);
      cudaError_t ie = cudaGraphInstantiate(&ge.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        set_error("batch graph instantiate failed: %s", cudaGetErrorString(ie));
        return SOD_ERR_CUDA;
      }
      it = B->graphs.emplace(key, ge).first;
    }
    for (int t = 0; t < nsteps; ++t) {
      SOD_CUDA(cudaGraphLaunch(it->second.exec, st));
      g_launches.fetch_add(it->second.nkernels);
    }
  }
  return mesh_internal_to_ref_elem(m, m->mue_int, B->st.mu_e, st);
}

// Elements-per-CTA autotuning of the fused RHS kernel on the concatenated ensemble.
int sod_batch_autotune(SodBatch* B, SodPrecision prec, int* best_epb, float* best_ms, sod_stream_t stream) {
  SOD_ARG(B, "batch");
  return sod_autotune(B->mesh, &B->st, prec, best_epb, best_ms, stream);
}

// Per-member adapt_dt_cfl (mod_time_ops.f90:11-61) from the members' u, csound, mu_fluid, rho.
int sod_batch_adapt_dt(SodBatch* B, sod_stream_t stream) {
  SOD_ARG(B, "batch");
  cudaStream_t st = (cudaStream_t)stream;
  SodMesh* m = B->mesh;
  int rc = ensure_step_buffers(m, false);
  if (rc) return rc;
  // mu_e is not touched: the viscosity pass writes into a scratch copy
  double* save = m->mue_int;
  m->mue_int = B->ref_mue;
  SodState s = B->st;
  s.Reta = m->buf.rsum;  // zero residual: only the dt part matters here
  SOD_CUDA(cudaMemsetAsync(s.Reta, 0, sizeof(double) * m->npoin, st));
  SOD_CUDA(cudaMemsetAsync(m->member_scal, 0, sizeof(double) * 2 * m->nmember, st));
  rc = launch_visc_dt(m, &s, B->dt, nullptr, st);
  m->mue_int = save;
  return rc;
}

}  // extern "C"
