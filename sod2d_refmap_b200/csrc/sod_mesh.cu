// Mesh upload, deterministic node->element gather map, device geometry (sm_100a).
//
// Geometry kernels restate the reference setup routines on the device:
//   elem_jacobian        jacobian_oper.f90:9-138   (Jacobian by 1-D line derivatives of the
//                                                    element coordinates, cofactor inverse)
//   lumped_mass_spectral mass_matrix.f90:11-43     (as a node-centric CSR gather, no atomics)
//   char_length          mod_geom.f90:13-37        (min corner-edge length, hexa_edges order)
//   char_length_spectral mod_geom.f90:39-66        (min distance to another element node)
#include "sod_internal.cuh"
#include <cstdarg>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <chrono>
#include <thread>

namespace sod {

static thread_local std::string g_err;
std::atomic<int64_t> g_launches{0};
static std::atomic<double> g_wait_timeout_s{0.0};

// Host wait on a stream, given up after the sod_set_wait_timeout limit (0: no limit).  Giving
// up leaves the device work queued; it completes on its own.
int sync_stream(cudaStream_t st) {
  const double lim = g_wait_timeout_s.load();
  if (lim <= 0.0) {
    SOD_CUDA(cudaStreamSynchronize(st));
    return SOD_OK;
  }
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaStreamQuery(st);
    if (e == cudaSuccess) return SOD_OK;
    if (e != cudaErrorNotReady) {
      set_error("stream wait: %s", cudaGetErrorString(e));
      return SOD_ERR_CUDA;
    }
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > lim) {
      set_error("host wait on device work exceeded %.3g s (sod_set_wait_timeout)", lim);
      return SOD_ERR_TIMEOUT;
    }
    std::this_thread::yield();
  }
}

// Reads and clears the non-finite flag the stage-4 gather sets (after the stream's work).
int take_nonfinite(SodMesh* m, cudaStream_t st, bool* flagged) {
  *flagged = false;
  if (!m->buf.counters) return SOD_OK;
  unsigned int h = 0;
  SOD_CUDA(cudaMemcpyAsync(&h, m->buf.counters + kNonfiniteCounter, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                           st));
  if (int rc = sync_stream(st)) return rc;
  if (h) {
    SOD_CUDA(cudaMemsetAsync(m->buf.counters + kNonfiniteCounter, 0, sizeof(unsigned int), st));
    *flagged = true;
  }
  return SOD_OK;
}

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

static const int kSodToNat[NP1] = {0, 3, 1, 2};  // sod2d 1-D index (0-based) -> natural

// ---------------------------------------------------------------------------------------------
// Geometry: one CTA per element, one thread per gauss point d.
// ---------------------------------------------------------------------------------------------
struct GeoArgs {
  int nelem;
  const int32_t* conn_orig;   // internal layout [e*64+d], 0-based ids into coord
  const double* coord;        // (npoin_orig,3) F
  int64_t npoin_orig;
  DMat D;
  double w[NN];               // GLL weight of internal node d
  int corner_d[8];            // internal node of reference local nodes 1..8
  double* geo64;
  double* helem;
  double* helem_l;
  double* jratio;
  int* bad;                   // set to 1 when some detJ <= 0 (inverted or degenerate gauss point)
};

__global__ void __launch_bounds__(64) k_geometry(const GeoArgs a) {
  const int e = blockIdx.x;
  const int d = threadIdx.x;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4;
  __shared__ double X[3][NN];
  __shared__ double red[2][NN];
  const int32_t node = a.conn_orig[(int64_t)e * NN + d];
  for (int c = 0; c < 3; ++c) X[c][d] = a.coord[node + a.npoin_orig * c];
  __syncthreads();
  // Je(r, c) = d x_c / d xi_r by 1-D line derivatives (dNgp is a tensor of 1-D factors with
  // N_a(g) = delta at the GLL collocation points).
  double Je[3][3];
  for (int c = 0; c < 3; ++c) {
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
#pragma unroll
    for (int m = 0; m < NP1; ++m) {
      g0 += a.D.d[i][m] * X[c][m + 4 * j + 16 * k];
      g1 += a.D.d[j][m] * X[c][i + 4 * m + 16 * k];
      g2 += a.D.d[k][m] * X[c][i + 4 * j + 16 * m];
    }
    Je[0][c] = g0; Je[1][c] = g1; Je[2][c] = g2;
  }
  const double det = (Je[0][0] * Je[1][1] * Je[2][2] + Je[0][1] * Je[1][2] * Je[2][0] +
                      Je[0][2] * Je[1][0] * Je[2][1] - Je[2][0] * Je[1][1] * Je[0][2] -
                      Je[2][1] * Je[1][2] * Je[0][0] - Je[2][2] * Je[1][0] * Je[0][1]);
  double b[9];
  b[0] = Je[1][1] * Je[2][2] - Je[2][1] * Je[1][2];
  b[3] = -(Je[1][0] * Je[2][2] - Je[2][0] * Je[1][2]);
  b[6] = Je[1][0] * Je[2][1] - Je[2][0] * Je[1][1];
  b[1] = -(Je[0][1] * Je[2][2] - Je[2][1] * Je[0][2]);
  b[4] = Je[0][0] * Je[2][2] - Je[2][0] * Je[0][2];
  b[7] = -(Je[0][0] * Je[2][1] - Je[2][0] * Je[0][1]);
  b[2] = Je[0][1] * Je[1][2] - Je[1][1] * Je[0][2];
  b[5] = -(Je[0][0] * Je[1][2] - Je[1][0] * Je[0][2]);
  b[8] = Je[0][0] * Je[1][1] - Je[1][0] * Je[0][1];
  if (!(det > 0.0)) atomicOr(a.bad, 1);
  const double inv = 1.0 / det;
  double* G = a.geo64 + (int64_t)e * NGEO * NN;
#pragma unroll
  for (int c = 0; c < 9; ++c) G[c * NN + d] = inv * b[c];
  const double gv = a.w[d] * det;
  G[9 * NN + d] = gv;
  // char_length_spectral: min distance to any other node of the element
  double best = 1000000000000.0;
  for (int o = 0; o < NN; ++o) {
    if (o == d) continue;
    double dx = X[0][d] - X[0][o], dy = X[1][d] - X[1][o], dz = X[2][d] - X[2][o];
    best = fmin(best, sqrt(dx * dx + dy * dy + dz * dz));
  }
  a.helem_l[(int64_t)e * NN + d] = best;
  // min/max of gpvol/wgp (= detJ) over the element
  red[0][d] = det;
  red[1][d] = det;
  __syncthreads();
  if (d == 0) {
    double mn = 1000000.0, mx = 0.0;
    for (int o = 0; o < NN; ++o) { mn = fmin(mn, red[0][o]); mx = fmax(mx, red[1][o]); }
    a.jratio[e] = (mn / mx) * (mn / mx);
    // char_length over the 12 corner edges (hexa_edges, elem_hex.f90:45-75)
    const int ed[12][2] = {{1, 0}, {2, 1}, {3, 2}, {0, 3}, {5, 4}, {6, 5},
                           {7, 6}, {4, 7}, {4, 0}, {5, 1}, {6, 2}, {7, 3}};
    double h = 1000000000000.0;
    for (int q = 0; q < 12; ++q) {
      int p0 = a.corner_d[ed[q][0]], p1 = a.corner_d[ed[q][1]];
      double dx = X[0][p0] - X[0][p1], dy = X[1][p0] - X[1][p1], dz = X[2][p0] - X[2][p1];
      h = fmin(h, sqrt(dx * dx + dy * dy + dz * dz));
    }
    a.helem[e] = h;
  }
}

// Ml(n) = sum of gpvol over the (element, node) pairs of node n, in ascending element order.
__global__ void k_lumped_mass(int npoin, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                              const double* __restrict__ geo64, double* __restrict__ Ml) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  double s = 0.0;
  for (int c = ptr[n]; c < ptr[n + 1]; ++c) {
    int packed = idx[c];
    int e = packed >> 6, d = packed & 63;
    s += geo64[((int64_t)e * NGEO + 9) * NN + d];
  }
  Ml[n] = s;
}

__global__ void k_d2f(const double* __restrict__ s, float* __restrict__ d, int64_t n) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; t < n; t += stride) d[t] = (float)s[t];
}

int launch_copy_f32(const double* src, float* dst, int64_t n, cudaStream_t st) {
  if (n <= 0) return SOD_OK;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_d2f<<<blocks, 256, 0, st>>>(src, dst, n);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

// reference (nelem,64) F layout <-> internal [e*64+d]
__global__ void k_ref2int(int nelem, const int32_t* __restrict__ a_of_d, const double* __restrict__ ref,
                          double* __restrict__ out) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * NN) return;
  int e = (int)(t >> 6), d = (int)(t & 63);
  out[t] = ref[e + (int64_t)nelem * a_of_d[d]];
}
__global__ void k_int2ref(int nelem, const int32_t* __restrict__ a_of_d, const double* __restrict__ in,
                          double* __restrict__ ref) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * NN) return;
  int e = (int)(t >> 6), d = (int)(t & 63);
  ref[e + (int64_t)nelem * a_of_d[d]] = in[t];
}

int mesh_ref_to_internal_elem(SodMesh* m, const double* ref, double* out, cudaStream_t st) {
  int64_t n = (int64_t)m->nelem * NN;
  k_ref2int<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(m->nelem, m->a_of_d_dev, ref, out);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}
int mesh_internal_to_ref_elem(SodMesh* m, const double* in, double* ref, cudaStream_t st) {
  int64_t n = (int64_t)m->nelem * NN;
  k_int2ref<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(m->nelem, m->a_of_d_dev, in, ref);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

// Local node order of the library (natural d = i + 4j + 16k) from the reference's gmshAtoI/J/K
// maps (host arrays, index_base-based), the 1-D derivative matrix from dlxigp_ip and, when given,
// the GLL weights in that order.
int mesh_set_local_tables(SodMesh* m, const int32_t* gI, const int32_t* gJ, const int32_t* gK,
                          const double* dlxigp_ip, const double* wgp, int base) {
  bool seen[NN] = {false};
  for (int a = 0; a < NN; ++a) {
    int si = gI[a] - base, sj = gJ[a] - base, sk = gK[a] - base;
    if (si < 0 || si > 3 || sj < 0 || sj > 3 || sk < 0 || sk > 3) {
      set_error("invalid argument: gmshAto* out of range at local node %d", a);
      return SOD_ERR_ARG;
    }
    int d = kSodToNat[si] + 4 * kSodToNat[sj] + 16 * kSodToNat[sk];
    if (seen[d]) {
      set_error("invalid argument: gmshAto* maps two local nodes to one ijk");
      return SOD_ERR_ARG;
    }
    seen[d] = true;
    m->perm_a_of_d[d] = a;
    m->perm_d_of_a[a] = d;
  }
  // D[mpt][nb] = l'_nb(x_mpt): dlxigp_ip(g, 0, ii) for a gauss point g with natural i = mpt
  for (int mpt = 0; mpt < NP1; ++mpt) {
    int g = m->perm_a_of_d[mpt];  // natural (mpt, 0, 0)
    for (int ii = 0; ii < NP1; ++ii) m->D.d[mpt][kSodToNat[ii]] = dlxigp_ip[g + NN * (0 + 3 * ii)];
  }
  if (wgp)
    for (int d = 0; d < NN; ++d) m->wgp_nat[d] = wgp[m->perm_a_of_d[d]];
  return SOD_OK;
}

int ensure_step_buffers(SodMesh* m, bool mixed) {
  if (int rc = init_kernel_attrs()) return rc;
  StepBuffers& b = m->buf;
  const int64_t N = m->npoin, E = m->nelem;
  if (!b.ys) {
    SOD_CUDA(cudaMalloc(&b.ys, sizeof(double) * 5 * N));
    SOD_CUDA(cudaMalloc(&b.rsum, sizeof(double) * 6 * N));
    b.red_cap = 4 * ((N + 127) / 128 + (E + 1) + 1024);
    SOD_CUDA(cudaMalloc(&b.red, sizeof(double) * b.red_cap));
    SOD_CUDA(cudaMalloc(&b.scal, sizeof(double) * 16));
    SOD_CUDA(cudaMemset(b.scal, 0, sizeof(double) * 16));
    SOD_CUDA(cudaMalloc(&b.counters, sizeof(unsigned int) * 16));
    SOD_CUDA(cudaMemset(b.counters, 0, sizeof(unsigned int) * 16));
    SOD_CUDA(cudaMalloc(&b.mu_fluid, sizeof(double) * N));
  }
  size_t need = (size_t)E * NRES * NN * sizeof(double);  // sized for FP64 (also holds FP32)
  if (b.rel_bytes < need) {
    if (b.rel) cudaFree(b.rel);
    SOD_CUDA(cudaMalloc(&b.rel, need));
    b.rel_bytes = need;
  }
  if (mixed) {
    if (!m->geo32) {
      SOD_CUDA(cudaMalloc(&m->geo32, sizeof(float) * E * NGEO * NN));
      int rc = launch_copy_f32(m->geo64, m->geo32, E * NGEO * NN, 0);
      if (rc) return rc;
    }
    if (!m->mue32) {
      SOD_CUDA(cudaMalloc(&m->mue32, sizeof(float) * E * NN));
      SOD_CUDA(cudaMemset(m->mue32, 0, sizeof(float) * E * NN));
    }
  }
  return SOD_OK;
}

}  // namespace sod

using namespace sod;

extern "C" {

const char* sod_last_error(void) { return sod::g_err.c_str(); }
const char* sod_version(void) { return "sod2d_b200 0.1 (sm_100a)"; }
int64_t sod_launch_count(void) { return sod::g_launches.load(); }

void sod_set_wait_timeout(double seconds) { sod::g_wait_timeout_s.store(seconds > 0.0 ? seconds : 0.0); }

int sod_check_finite(SodMesh* m, sod_stream_t stream) {
  SOD_ARG(m, "mesh null");
  bool bad = false;
  if (int rc = take_nonfinite(m, (cudaStream_t)stream, &bad)) return rc;
  if (bad) {
    set_error("a non-finite value (NaN/Inf) appeared in rho, q or E during a step");
    return SOD_ERR_NONFINITE;
  }
  return SOD_OK;
}

void sod_params_default(SodParams* p) {
  if (!p) return;
  p->gamma_gas = 1.4;
  p->Cp = 1004.0;
  p->Rgas = p->Cp * (p->gamma_gas - 1.0) / p->gamma_gas;
  p->Prt = 0.71;
  p->ce = 0.1;
  p->cmax = 0.5;
  p->cglob = 1.0;
  p->c_rho = 1.0;
  p->c_ener = 1.0;
  p->flag_normalise_entropy = 1;
  p->cfl_conv = 0.5;
  p->cfl_diff = 0.5;
  p->flag_les = 0;
  p->c_sgs = 0.025;
  p->flag_total_enthalpy = 0;
}

static void to_dev_params(const SodParams* s, DevParams* d) {
  d->gamma = s->gamma_gas; d->Rgas = s->Rgas; d->Cp = s->Cp; d->Prt = s->Prt;
  d->ce = s->ce; d->cmax = s->cmax; d->cglob = s->cglob; d->c_rho = s->c_rho; d->c_ener = s->c_ener;
  d->cfl_conv = s->cfl_conv; d->cfl_diff = s->cfl_diff; d->normalise = s->flag_normalise_entropy;
  d->g_gm1 = s->gamma_gas / (s->gamma_gas - 1.0);
  d->inv_gm1 = 1.0 / (s->gamma_gas - 1.0);
  d->inv_Rgas = 1.0 / s->Rgas;
  d->CpPr = s->Cp / s->Prt;
  d->Cp09 = s->Cp / 0.9;
  d->flag_les = s->flag_les;
  d->c_sgs = s->c_sgs;
  d->total_enthalpy = s->flag_total_enthalpy != 0;
  d->gamma_f = (float)s->gamma_gas;
  d->c_rho_f = (float)s->c_rho;
  d->c_ener_f = (float)s->c_ener;
  d->CpPr_f = (float)(s->Cp / s->Prt);
  d->Cp09_f = (float)(s->Cp / 0.9);
}

int sod_mesh_set_params(SodMesh* m, const SodParams* p) {
  SOD_ARG(m && p, "mesh/params null");
  to_dev_params(p, &m->prm);
  // captured step graphs hold the parameters in their kernel arguments
  for (auto& kv : m->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  m->graphs.clear();
  return SOD_OK;
}

void sod_mesh_destroy(SodMesh* m) {
  if (!m) return;
  bc_free(m);
  zone_free(m);
  wall_model_free(m);
  if (m->postpro) cudaFree(m->postpro);
  for (auto& kv : m->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  void* ptrs[] = {m->econn, m->geo64, m->geo32, m->Ml, m->helem, m->helem_l, m->jratio, m->n2e_ptr, m->n2e,
                  m->mue_int, m->mue32, m->a_of_d_dev, m->buf.ys, m->buf.rsum, m->buf.rel, m->buf.red,
                  m->buf.scal, m->buf.counters, m->buf.mu_fluid, m->adj, m->musgs_int};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (double* p : m->host_mirror) cudaFree(p);
  if (m->host_copy_stream) cudaStreamDestroy(m->host_copy_stream);
  if (m->host_ev_state) cudaEventDestroy(m->host_ev_state);
  if (m->host_ev_copied) cudaEventDestroy(m->host_ev_copied);
  delete m;
}

int sod_mesh_create(const SodMeshDesc* desc, const SodParams* params, SodMesh** out) {
  SOD_ARG(desc && out, "desc/out null");
  *out = nullptr;
  SOD_ARG(desc->porder == 3, "porder must be 3 (HEX64)");
  SOD_ARG(desc->nelem > 0 && desc->npoin > 0, "nelem/npoin must be positive");
  SOD_ARG((int64_t)desc->nelem * NN < (int64_t)1 << 31, "nelem*64 must fit int32");
  SOD_ARG(desc->index_base == 0 || desc->index_base == 1, "index_base must be 0 or 1");
  SOD_ARG(desc->connec && desc->dlxigp_ip && desc->wgp && desc->gmshAtoI && desc->gmshAtoJ && desc->gmshAtoK,
          "connec, dlxigp_ip, wgp, gmshAtoI/J/K required");
  const bool have_geo = desc->He && desc->gpvol;
  SOD_ARG(have_geo || (desc->coord_orig && desc->connec_orig && desc->npoin_orig > 0),
          "either He+gpvol or coord_orig+connec_orig+npoin_orig required");
  SOD_ARG(desc->coord_orig || (desc->helem && desc->helem_l), "helem/helem_l need coord_orig when absent");
  const int base = desc->index_base;
  const int E = desc->nelem, N = desc->npoin;
  SodMesh* m = new SodMesh();
  m->nelem = E;
  m->npoin = N;
  m->index_base = base;
  cudaGetDevice(&m->device);
  SodParams dp;
  sod_params_default(&dp);
  to_dev_params(params ? params : &dp, &m->prm);
  {
    const int rc = mesh_set_local_tables(m, desc->gmshAtoI, desc->gmshAtoJ, desc->gmshAtoK, desc->dlxigp_ip, desc->wgp,
                                         base);
    if (rc) {
      delete m;
      return rc;
    }
  }

  auto fail = [&](int rc) { sod_mesh_destroy(m); return rc; };
  // connectivity in internal layout
  std::vector<int32_t> econn((size_t)E * NN);
  for (int e = 0; e < E; ++e)
    for (int d = 0; d < NN; ++d) {
      int32_t v = desc->connec[e + (int64_t)E * m->perm_a_of_d[d]] - base;
      if (v < 0 || v >= N) {
        set_error("invalid argument: connec(%d,%d)=%d out of range", e + base, m->perm_a_of_d[d] + base, v + base);
        return fail(SOD_ERR_ARG);
      }
      econn[(size_t)e * NN + d] = v;
    }
  // CSR node -> (e, d), ascending element order
  std::vector<int32_t> ptr(N + 1, 0), idx((size_t)E * NN);
  for (size_t t = 0; t < econn.size(); ++t) ptr[econn[t] + 1]++;
  for (int n = 0; n < N; ++n) ptr[n + 1] += ptr[n];
  {
    std::vector<int32_t> fillp(ptr.begin(), ptr.end() - 1);
    for (int e = 0; e < E; ++e)
      for (int d = 0; d < NN; ++d) {
        int32_t v = econn[(size_t)e * NN + d];
        idx[fillp[v]++] = e * NN + d;
      }
  }
  // working nodes: lpoin_w when given (rows it does not list are periodic slaves), else all;
  // connec (connecParWork) must reference exactly the working rows
  std::vector<uint8_t> work((size_t)N, desc->lpoin_w ? 0 : 1);
  if (desc->lpoin_w) {
    if (desc->npoin_w <= 0 || desc->npoin_w > N) {
      set_error("invalid argument: npoin_w=%d must be in 1..npoin=%d", desc->npoin_w, N);
      return fail(SOD_ERR_ARG);
    }
    for (int w = 0; w < desc->npoin_w; ++w) {
      const int v = desc->lpoin_w[w] - base;
      if (v < 0 || v >= N || work[v]) {
        set_error("invalid argument: lpoin_w(%d)=%d is out of range or listed twice", w + base, v + base);
        return fail(SOD_ERR_ARG);
      }
      work[v] = 1;
    }
  }
  m->npoin_w = desc->lpoin_w ? desc->npoin_w : N;
  m->has_slaves = m->npoin_w < N;
  if (m->has_slaves) {
    m->slave_host.assign((size_t)N, 0);
    for (int n = 0; n < N; ++n) m->slave_host[n] = work[n] ? 0 : 1;
  }
  for (int n = 0; n < N; ++n) {
    const bool has = ptr[n + 1] > ptr[n];
    if (work[n] && !has) {
      set_error("invalid argument: working node %d is not referenced by any element", n + base);
      return fail(SOD_ERR_ARG);
    }
    if (!work[n] && has) {
      set_error("invalid argument: connec references node %d, which lpoin_w does not list (connec must be "
                "connecParWork: every periodic image replaced by its master)", n + base);
      return fail(SOD_ERR_ARG);
    }
  }
#define ALLOC(p, bytes)                                        \
  do {                                                         \
    if (cudaMalloc(&(p), (bytes)) != cudaSuccess) {            \
      set_error("cudaMalloc of %zu bytes failed", (size_t)(bytes)); \
      return fail(SOD_ERR_NOMEM);                              \
    }                                                          \
  } while (0)
  ALLOC(m->econn, sizeof(int32_t) * E * NN);
  ALLOC(m->n2e_ptr, sizeof(int32_t) * (N + 1));
  ALLOC(m->n2e, sizeof(int32_t) * E * NN);
  ALLOC(m->geo64, sizeof(double) * (size_t)E * NGEO * NN);
  ALLOC(m->Ml, sizeof(double) * N);
  ALLOC(m->helem, sizeof(double) * E);
  ALLOC(m->helem_l, sizeof(double) * E * NN);
  ALLOC(m->jratio, sizeof(double) * E);
  ALLOC(m->mue_int, sizeof(double) * E * NN);
  ALLOC(m->a_of_d_dev, sizeof(int32_t) * NN);
  if (cudaMemcpy(m->econn, econn.data(), sizeof(int32_t) * E * NN, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m->n2e_ptr, ptr.data(), sizeof(int32_t) * (N + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m->n2e, idx.data(), sizeof(int32_t) * E * NN, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m->a_of_d_dev, m->perm_a_of_d, sizeof(int32_t) * NN, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(m->mue_int, 0, sizeof(double) * E * NN) != cudaSuccess) {
    set_error("mesh upload failed: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(SOD_ERR_CUDA);
  }
  // geometry
  if (desc->coord_orig && desc->connec_orig) {
    std::vector<int32_t> co((size_t)E * NN);
    for (int e = 0; e < E; ++e)
      for (int d = 0; d < NN; ++d) {
        int32_t v = desc->connec_orig[e + (int64_t)E * m->perm_a_of_d[d]] - base;
        if (v < 0 || v >= desc->npoin_orig) {
          set_error("invalid argument: connec_orig out of range");
          return fail(SOD_ERR_ARG);
        }
        co[(size_t)e * NN + d] = v;
      }
    int32_t* dco = nullptr;
    double* dxyz = nullptr;
    int* dbad = nullptr;
    ALLOC(dco, sizeof(int32_t) * E * NN);
    ALLOC(dbad, sizeof(int));
    cudaMemset(dbad, 0, sizeof(int));
    if (cudaMalloc(&dxyz, sizeof(double) * 3 * (size_t)desc->npoin_orig) != cudaSuccess) {
      cudaFree(dco);
      set_error("cudaMalloc coord failed");
      return fail(SOD_ERR_NOMEM);
    }
    cudaMemcpy(dco, co.data(), sizeof(int32_t) * E * NN, cudaMemcpyHostToDevice);
    cudaMemcpy(dxyz, desc->coord_orig, sizeof(double) * 3 * (size_t)desc->npoin_orig, cudaMemcpyHostToDevice);
    GeoArgs ga;
    ga.nelem = E; ga.conn_orig = dco; ga.coord = dxyz; ga.npoin_orig = desc->npoin_orig; ga.D = m->D;
    for (int d = 0; d < NN; ++d) ga.w[d] = m->wgp_nat[d];
    for (int c = 0; c < 8; ++c) ga.corner_d[c] = m->perm_d_of_a[c];
    ga.geo64 = m->geo64; ga.helem = m->helem; ga.helem_l = m->helem_l; ga.jratio = m->jratio; ga.bad = dbad;
    k_geometry<<<E, 64>>>(ga);
    g_launches.fetch_add(1);
    cudaError_t err = cudaDeviceSynchronize();
    int hbad = 0;
    cudaMemcpy(&hbad, dbad, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dco);
    cudaFree(dxyz);
    cudaFree(dbad);
    if (err != cudaSuccess) {
      set_error("k_geometry: %s", cudaGetErrorString(err));
      return fail(SOD_ERR_CUDA);
    }
    if (hbad && !(desc->He && desc->gpvol)) {
      set_error("invalid argument: non-positive Jacobian determinant at some gauss point (inverted element)");
      return fail(SOD_ERR_ARG);
    }
  }
  if (have_geo) {
    // caller-provided He/gpvol override the computed ones (reference layouts)
    std::vector<double> g((size_t)E * NGEO * NN);
    for (int e = 0; e < E; ++e)
      for (int d = 0; d < NN; ++d) {
        int a = m->perm_a_of_d[d];
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c)
            g[((size_t)e * NGEO + 3 * r + c) * NN + d] = desc->He[r + 3 * (c + 3 * ((int64_t)a + NN * e))];
        g[((size_t)e * NGEO + 9) * NN + d] = desc->gpvol[a + (int64_t)NN * e];
      }
    if (cudaMemcpy(m->geo64, g.data(), sizeof(double) * g.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("geometry upload failed");
      return fail(SOD_ERR_CUDA);
    }
    // jratio from gpvol/wgp
    std::vector<double> jr(E);
    for (int e = 0; e < E; ++e) {
      double mn = 1000000.0, mx = 0.0;
      for (int a = 0; a < NN; ++a) {
        double v = desc->gpvol[a + (int64_t)NN * e] / desc->wgp[a];
        mn = std::min(mn, v);
        mx = std::max(mx, v);
      }
      jr[e] = (mn / mx) * (mn / mx);
    }
    cudaMemcpy(m->jratio, jr.data(), sizeof(double) * E, cudaMemcpyHostToDevice);
  }
  if (desc->helem) cudaMemcpy(m->helem, desc->helem, sizeof(double) * E, cudaMemcpyHostToDevice);
  if (desc->helem_l) {
    std::vector<double> hl((size_t)E * NN);
    for (int e = 0; e < E; ++e)
      for (int d = 0; d < NN; ++d) hl[(size_t)e * NN + d] = desc->helem_l[e + (int64_t)E * m->perm_a_of_d[d]];
    cudaMemcpy(m->helem_l, hl.data(), sizeof(double) * hl.size(), cudaMemcpyHostToDevice);
  }
  if (desc->Ml) {
    cudaMemcpy(m->Ml, desc->Ml, sizeof(double) * N, cudaMemcpyHostToDevice);
  } else {
    k_lumped_mass<<<(N + 255) / 256, 256>>>(N, m->n2e_ptr, m->n2e, m->geo64, m->Ml);
    g_launches.fetch_add(1);
  }
  cudaError_t err = cudaDeviceSynchronize();
  if (err != cudaSuccess) {
    set_error("mesh create: %s", cudaGetErrorString(err));
    return fail(SOD_ERR_CUDA);
  }
#undef ALLOC
  *out = m;
  return SOD_OK;
}

int sod_mesh_get_geometry(SodMesh* m, double* He, double* gpvol, double* Ml, double* helem, double* helem_l) {
  SOD_ARG(m, "mesh null");
  const int E = m->nelem;
  SOD_CUDA(cudaDeviceSynchronize());
  if (He || gpvol) {
    std::vector<double> g((size_t)E * NGEO * NN);
    SOD_CUDA(cudaMemcpy(g.data(), m->geo64, sizeof(double) * g.size(), cudaMemcpyDeviceToHost));
    for (int e = 0; e < E; ++e)
      for (int d = 0; d < NN; ++d) {
        int a = m->perm_a_of_d[d];
        if (He)
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
              He[r + 3 * (c + 3 * ((int64_t)a + NN * e))] = g[((size_t)e * NGEO + 3 * r + c) * NN + d];
        if (gpvol) gpvol[a + (int64_t)NN * e] = g[((size_t)e * NGEO + 9) * NN + d];
      }
  }
  if (Ml) SOD_CUDA(cudaMemcpy(Ml, m->Ml, sizeof(double) * m->npoin, cudaMemcpyDeviceToHost));
  if (helem) SOD_CUDA(cudaMemcpy(helem, m->helem, sizeof(double) * E, cudaMemcpyDeviceToHost));
  if (helem_l) {
    std::vector<double> hl((size_t)E * NN);
    SOD_CUDA(cudaMemcpy(hl.data(), m->helem_l, sizeof(double) * hl.size(), cudaMemcpyDeviceToHost));
    for (int e = 0; e < E; ++e)
      for (int d = 0; d < NN; ++d) helem_l[e + (int64_t)E * m->perm_a_of_d[d]] = hl[(size_t)e * NN + d];
  }
  return SOD_OK;
}

}  // extern "C"
