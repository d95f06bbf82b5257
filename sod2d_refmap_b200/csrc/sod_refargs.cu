// Per-routine entry points with the reference's complete argument lists (sm_100a).
//
// SOD2D's time loop and its unit tests call full_convec_ijk, full_convec_ijk_H,
// generic_scalar_convec_ijk, full_diffusion_ijk and smart_visc_spectral with the mesh and the
// shape tables in every call (elem_convec.f90:20-33,211-224,462-476; elem_diffu.f90:12-25;
// mod_entropy_viscosity.f90:14-28), its arrays already resident on the device.  These entry
// points take exactly those arguments as device pointers, build a transient device view of the
// mesh from them (the library's element-major connectivity and geometry, and the ordered
// node->element gather map, sorted on the device), run the same kernels as the handle-based
// entry points (so results equal theirs bit for bit), and release the view before returning.
// They allocate per call and wait for their stream; a time loop keeps a SodMesh instead.
#include "sod_internal.cuh"

namespace sod {
namespace refargs {

constexpr int kBlock = 256;

// connec(nelem,64) (reference layout, index_base ids) -> econn[e*64 + d], node counts
__global__ void k_econn(int nelem, int npoin, int base, const int32_t* __restrict__ connec,
                        const int32_t* __restrict__ a_of_d, int32_t* __restrict__ econn, int32_t* __restrict__ cnt,
                        int* flag) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * NN) return;
  const int e = (int)(t / NN), d = (int)(t % NN);
  int v = connec[e + (int64_t)nelem * a_of_d[d]] - base;
  if (v < 0 || v >= npoin) {  // reported after the call; clamped so no access leaves the arrays
    atomicOr(flag, 1);
    v = 0;
  }
  econn[t] = v;
  atomicAdd(&cnt[v], 1);
}

// single-block exclusive scan of cnt[0..n) into ptr[0..n]; cnt becomes the fill cursors (0)
__global__ void __launch_bounds__(1024) k_scan(int n, int32_t* __restrict__ cnt, int32_t* __restrict__ ptr) {
  __shared__ int32_t wsum[32];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int chunk = (n + nthr - 1) / nthr;
  const int beg = min(tid * chunk, n), end = min(beg + chunk, n);
  int32_t s = 0;
  for (int i = beg; i < end; ++i) s += cnt[i];
  int32_t x = s;
  const int lane = tid & 31, w = tid >> 5;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int32_t y = lane < (nthr >> 5) ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t z = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += z;
    }
    wsum[lane] = y;
  }
  __syncthreads();
  int32_t run = x - s + (w > 0 ? wsum[w - 1] : 0);
  for (int i = beg; i < end; ++i) {
    ptr[i] = run;
    run += cnt[i];
    cnt[i] = 0;
  }
  if (tid == nthr - 1) ptr[n] = run;
}

__global__ void k_fill(int nelem, const int32_t* __restrict__ econn, const int32_t* __restrict__ ptr,
                       int32_t* __restrict__ cur, int32_t* __restrict__ idx) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * NN) return;
  const int v = econn[t];
  idx[ptr[v] + atomicAdd(&cur[v], 1)] = (int32_t)t;  // packed e*64 + d
}

// ascending (element, local node) inside each node's list: the order of the host-built map
__global__ void k_sort(int npoin, const int32_t* __restrict__ ptr, int32_t* __restrict__ idx) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  const int b = ptr[n], e = ptr[n + 1];
  for (int q = b + 1; q < e; ++q) {
    const int32_t key = idx[q];
    int r = q - 1;
    while (r >= b && idx[r] > key) {
      idx[r + 1] = idx[r];
      --r;
    }
    idx[r + 1] = key;
  }
}

// He(3,3,64,nelem), gpvol(1,64,nelem) -> geo64[(e*10 + c)*64 + d]; jratio from gpvol / wgp
// (smart_visc_spectral's (minJe/maxJe)^2, mod_entropy_viscosity.f90:71-83)
__global__ void k_geo(int nelem, const double* __restrict__ He, const double* __restrict__ gpvol,
                      const int32_t* __restrict__ a_of_d, double* __restrict__ geo) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * NN) return;
  const int64_t e = t / NN;
  const int d = (int)(t % NN), a = a_of_d[d];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      geo[(e * NGEO + 3 * r + c) * NN + d] = He ? He[r + 3 * (c + 3 * ((int64_t)a + NN * e))] : 0.0;
  geo[(e * NGEO + 9) * NN + d] = gpvol[a + NN * e];
}

__global__ void k_jratio(int nelem, const double* __restrict__ gpvol, const double* __restrict__ wgp,
                         double* __restrict__ jratio) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  double mn = 1000000.0, mx = 0.0;
  for (int a = 0; a < NN; ++a) {
    const double v = gpvol[a + (int64_t)NN * e] / wgp[a];
    mn = fmin(mn, v);
    mx = fmax(mx, v);
  }
  jratio[e] = (mn / mx) * (mn / mx);
}

// lpoin_w must list each row that an element holds exactly once, and no other row
__global__ void k_mark(int npoin_w, int npoin, int base, const int32_t* __restrict__ lpoin_w, int32_t* mark,
                       int* flag) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= npoin_w) return;
  const int v = lpoin_w[w] - base;
  if (v < 0 || v >= npoin) {
    atomicOr(flag, 4);
    return;
  }
  atomicAdd(&mark[v], 1);
}

__global__ void k_check_working(int npoin, const int32_t* __restrict__ mark, const int32_t* __restrict__ ptr,
                                int* flag) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  if (mark[n] > 1) atomicOr(flag, 4);
  if ((mark[n] > 0) != (ptr[n + 1] > ptr[n])) atomicOr(flag, 8);
}

static int grid(int64_t n) { return (int)((n + kBlock - 1) / kBlock); }

}  // namespace refargs

int mesh_from_device_ref(int nelem, int npoin, int base, const int32_t* connec, const double* He,
                         const double* gpvol, const double* dlxigp_ip, const int32_t* invAtoIJK,
                         const int32_t* gI, const int32_t* gJ, const int32_t* gK, const double* wgp,
                         const double* helem_l, const double* helem, int npoin_w, const int32_t* lpoin_w,
                         const SodParams* params, cudaStream_t st, SodMesh** out) {
  using namespace refargs;
  *out = nullptr;
  SOD_ARG(nelem > 0 && npoin > 0 && (int64_t)nelem * NN < ((int64_t)1 << 31), "nelem/npoin out of range");
  SOD_ARG(base == 0 || base == 1, "index_base must be 0 or 1");
  SOD_ARG(connec && gpvol && gI && gJ && gK, "connec, gpvol, gmshAtoI/J/K required");
  SOD_ARG(!lpoin_w || (npoin_w > 0 && npoin_w <= npoin), "npoin_w must be in 1..npoin");
  // the small tables, on the host
  int32_t hI[NN], hJ[NN], hK[NN], hinv[NN];
  double hdl[NN * 3 * NP1] = {0}, hw[NN];
  SOD_CUDA(cudaMemcpyAsync(hI, gI, sizeof(hI), cudaMemcpyDeviceToHost, st));
  SOD_CUDA(cudaMemcpyAsync(hJ, gJ, sizeof(hJ), cudaMemcpyDeviceToHost, st));
  SOD_CUDA(cudaMemcpyAsync(hK, gK, sizeof(hK), cudaMemcpyDeviceToHost, st));
  if (dlxigp_ip) SOD_CUDA(cudaMemcpyAsync(hdl, dlxigp_ip, sizeof(hdl), cudaMemcpyDeviceToHost, st));
  if (invAtoIJK) SOD_CUDA(cudaMemcpyAsync(hinv, invAtoIJK, sizeof(hinv), cudaMemcpyDeviceToHost, st));
  if (wgp) SOD_CUDA(cudaMemcpyAsync(hw, wgp, sizeof(hw), cudaMemcpyDeviceToHost, st));
  if (int rc = sync_stream(st)) return rc;
  SodMesh* m = new SodMesh();
  m->nelem = nelem;
  m->npoin = npoin;
  m->index_base = base;
  cudaGetDevice(&m->device);
  auto fail = [&](int rc) {
    sod_mesh_destroy(m);
    return rc;
  };
  if (int rc = mesh_set_local_tables(m, hI, hJ, hK, hdl, wgp ? hw : nullptr, base)) return fail(rc);
  if (invAtoIJK)  // the reference indexes element lines through invAtoIJK; it must invert the gmshAto maps
    for (int a = 0; a < NN; ++a) {
      const int s = (hI[a] - base) + 4 * ((hJ[a] - base) + 4 * (hK[a] - base));
      if (hinv[s] - base != a) {
        set_error("invalid argument: invAtoIJK does not invert gmshAtoI/J/K at local node %d", a + base);
        return fail(SOD_ERR_ARG);
      }
    }
  SodParams dp;
  sod_params_default(&dp);
  if (int rc = sod_mesh_set_params(m, params ? params : &dp)) return fail(rc);
  const int64_t E = nelem, N = npoin;
  int32_t *cnt = nullptr, *mark = nullptr;
  int* flag = nullptr;
#define RALLOC(p, bytes)                                          \
  do {                                                            \
    if (cudaMalloc((void**)&(p), (bytes)) != cudaSuccess) {       \
      set_error("cudaMalloc of %zu bytes failed", (size_t)(bytes)); \
      cudaFree(cnt); cudaFree(mark); cudaFree(flag);              \
      return fail(SOD_ERR_NOMEM);                                 \
    }                                                             \
  } while (0)
  RALLOC(m->econn, sizeof(int32_t) * E * NN);
  RALLOC(m->n2e_ptr, sizeof(int32_t) * (N + 1));
  RALLOC(m->n2e, sizeof(int32_t) * E * NN);
  RALLOC(m->geo64, sizeof(double) * E * NGEO * NN);
  RALLOC(m->helem, sizeof(double) * E);
  RALLOC(m->helem_l, sizeof(double) * E * NN);
  RALLOC(m->jratio, sizeof(double) * E);
  RALLOC(m->mue_int, sizeof(double) * E * NN);
  RALLOC(m->a_of_d_dev, sizeof(int32_t) * NN);
  RALLOC(cnt, sizeof(int32_t) * (N + 1));
  RALLOC(flag, sizeof(int));
  if (lpoin_w) RALLOC(mark, sizeof(int32_t) * N);
#undef RALLOC
  auto release = [&]() {
    cudaFree(cnt);
    cudaFree(mark);
    cudaFree(flag);
  };
  cudaError_t err = cudaMemcpyAsync(m->a_of_d_dev, m->perm_a_of_d, sizeof(int32_t) * NN, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (N + 1), st);
  if (err == cudaSuccess) err = cudaMemsetAsync(flag, 0, sizeof(int), st);
  if (err == cudaSuccess) err = cudaMemsetAsync(m->mue_int, 0, sizeof(double) * E * NN, st);
  if (err == cudaSuccess && mark) err = cudaMemsetAsync(mark, 0, sizeof(int32_t) * N, st);
  if (err != cudaSuccess) {
    release();
    set_error("mesh view set-up: %s", cudaGetErrorString(err));
    return fail(SOD_ERR_CUDA);
  }
  k_econn<<<grid(E * NN), kBlock, 0, st>>>(nelem, npoin, base, connec, m->a_of_d_dev, m->econn, cnt, flag);
  k_scan<<<1, 1024, 0, st>>>(npoin, cnt, m->n2e_ptr);
  k_fill<<<grid(E * NN), kBlock, 0, st>>>(nelem, m->econn, m->n2e_ptr, cnt, m->n2e);
  k_sort<<<grid(N), kBlock, 0, st>>>(npoin, m->n2e_ptr, m->n2e);
  k_geo<<<grid(E * NN), kBlock, 0, st>>>(nelem, He, gpvol, m->a_of_d_dev, m->geo64);
  g_launches.fetch_add(5);
  if (wgp) {
    k_jratio<<<grid(E), kBlock, 0, st>>>(nelem, gpvol, wgp, m->jratio);
    g_launches.fetch_add(1);
  }
  if (lpoin_w) {
    k_mark<<<grid(npoin_w), kBlock, 0, st>>>(npoin_w, npoin, base, lpoin_w, mark, flag);
    k_check_working<<<grid(N), kBlock, 0, st>>>(npoin, mark, m->n2e_ptr, flag);
    g_launches.fetch_add(2);
  }
  err = cudaGetLastError();
  if (err == cudaSuccess && helem) err = cudaMemcpyAsync(m->helem, helem, sizeof(double) * E, cudaMemcpyDeviceToDevice, st);
  if (err != cudaSuccess) {
    release();
    set_error("mesh view kernels: %s", cudaGetErrorString(err));
    return fail(SOD_ERR_CUDA);
  }
  if (helem_l) {
    if (int rc = mesh_ref_to_internal_elem(m, helem_l, m->helem_l, st)) {
      release();
      return fail(rc);
    }
  }
  int hflag = 0;
  if (int rc = sync_stream(st)) {
    release();
    return fail(rc);
  }
  err = cudaMemcpy(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost);
  release();
  if (err != cudaSuccess) {
    set_error("mesh view flag: %s", cudaGetErrorString(err));
    return fail(SOD_ERR_CUDA);
  }
  if (hflag & 1) {
    set_error("invalid argument: connec holds node ids outside [%d, %d)", base, base + npoin);
    return fail(SOD_ERR_ARG);
  }
  if (hflag & 4) {
    set_error("invalid argument: lpoin_w holds ids out of range or listed twice");
    return fail(SOD_ERR_ARG);
  }
  if (hflag & 8) {
    set_error("invalid argument: lpoin_w must list exactly the nodes that connec references");
    return fail(SOD_ERR_ARG);
  }
  m->npoin_w = lpoin_w ? npoin_w : npoin;
  m->has_slaves = m->npoin_w < npoin;
  *out = m;
  return SOD_OK;
}

}  // namespace sod

using namespace sod;

namespace {
// one call on a transient view: build, run, wait, release
template <class F>
int with_view(int nelem, int npoin, int base, const int32_t* connec, const double* He, const double* gpvol,
              const double* dlxigp_ip, const int32_t* invAtoIJK, const int32_t* gI, const int32_t* gJ,
              const int32_t* gK, cudaStream_t st, F run) {
  SodMesh* m = nullptr;
  int rc = mesh_from_device_ref(nelem, npoin, base, connec, He, gpvol, dlxigp_ip, invAtoIJK, gI, gJ, gK, nullptr,
                                nullptr, nullptr, 0, nullptr, nullptr, st, &m);
  if (rc) return rc;
  rc = run(m);
  const int rw = sync_stream(st);
  sod_mesh_destroy(m);
  return rc ? rc : rw;
}
}  // namespace

extern "C" {

int sod_full_convec_ijk_ref(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                            const double* Ngp, const double* dNgp, const double* He, const double* gpvol,
                            const double* dlxigp_ip, const double* xgp, const int32_t* invAtoIJK,
                            const int32_t* gmshAtoI, const int32_t* gmshAtoJ, const int32_t* gmshAtoK,
                            const double* u, const double* q, const double* rho, const double* pr, const double* E,
                            double* Rmass, double* Rmom, double* Rener, sod_stream_t stream) {
  (void)Ngp; (void)dNgp; (void)xgp;  // collocation: the routine reads only dlxigp_ip and the maps
  SOD_ARG(He && u && q && rho && pr && E && Rmass && Rmom && Rener, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  return with_view(nelem, npoin, index_base, connec, He, gpvol, dlxigp_ip, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK,
                   st, [&](SodMesh* m) { return sod_full_convec_ijk(m, u, q, rho, pr, E, Rmass, Rmom, Rener, stream); });
}

int sod_full_convec_ijk_H_ref(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                              const double* Ngp, const double* dNgp, const double* He, const double* gpvol,
                              const double* dlxigp_ip, const double* xgp, const int32_t* invAtoIJK,
                              const int32_t* gmshAtoI, const int32_t* gmshAtoJ, const int32_t* gmshAtoK,
                              const double* u, const double* q, const double* rho, const double* pr, const double* E,
                              double* Rmass, double* Rmom, double* Rener, sod_stream_t stream) {
  (void)Ngp; (void)dNgp; (void)xgp;
  SOD_ARG(He && u && q && rho && pr && E && Rmass && Rmom && Rener, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  return with_view(nelem, npoin, index_base, connec, He, gpvol, dlxigp_ip, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK,
                   st,
                   [&](SodMesh* m) { return sod_full_convec_ijk_H(m, u, q, rho, pr, E, Rmass, Rmom, Rener, stream); });
}

int sod_generic_scalar_convec_ijk_ref(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                                      const double* Ngp, const double* dNgp, const double* He, const double* gpvol,
                                      const double* dlxigp_ip, const double* xgp, const int32_t* invAtoIJK,
                                      const int32_t* gmshAtoI, const int32_t* gmshAtoJ, const int32_t* gmshAtoK,
                                      const double* q, const double* eta, const double* u, double* Rconvec,
                                      sod_stream_t stream) {
  (void)Ngp; (void)dNgp; (void)xgp;
  SOD_ARG(He && q && eta && u && Rconvec, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  return with_view(nelem, npoin, index_base, connec, He, gpvol, dlxigp_ip, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK,
                   st, [&](SodMesh* m) { return sod_generic_scalar_convec_ijk(m, q, eta, u, Rconvec, stream); });
}

int sod_full_diffusion_ijk_ref(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                               const double* Ngp, const double* He, const double* gpvol, const double* dlxigp_ip,
                               const int32_t* invAtoIJK, const int32_t* gmshAtoI, const int32_t* gmshAtoJ,
                               const int32_t* gmshAtoK, double Cp, double Pr, const double* rho_n, const double* rho,
                               const double* u, const double* Tem, const double* mu_fluid, const double* mu_e,
                               const double* mu_sgs, const double* Ml, double* Rmass, double* Rmom, double* Rener,
                               sod_stream_t stream) {
  (void)Ngp; (void)Ml;  // not read by the routine (elem_diffu.f90:12-198)
  SOD_ARG(He && rho_n && rho && u && Tem && mu_fluid && mu_e && Rmass && Rmom && Rener, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  return with_view(nelem, npoin, index_base, connec, He, gpvol, dlxigp_ip, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK,
                   st, [&](SodMesh* m) {
                     return sod_full_diffusion_ijk(m, Cp, Pr, rho_n, rho, u, Tem, mu_fluid, mu_e, mu_sgs, Rmass, Rmom,
                                                   Rener, stream);
                   });
}

int sod_smart_visc_spectral_ref(int32_t nelem, int32_t npoin, int32_t npoin_w, int32_t index_base,
                                const int32_t* connec, const int32_t* lpoin_w, const double* Reta, const double* Ngp,
                                const double* coord, const double* dNgp, const double* gpvol, const double* wgp,
                                double gamma_gas, const double* rho, const double* u, const double* csound,
                                const double* Tem, const double* eta, const double* helem_l, const double* helem,
                                const double* Ml, double* mu_e, const int32_t* invAtoIJK, const int32_t* gmshAtoI,
                                const int32_t* gmshAtoJ, const int32_t* gmshAtoK, double* mue_l,
                                const SodParams* params, sod_stream_t stream) {
  (void)Ngp; (void)coord; (void)dNgp; (void)Ml; (void)mue_l;  // not read (mod_entropy_viscosity.f90:36-121)
  SOD_ARG(lpoin_w && Reta && wgp && rho && u && csound && Tem && eta && helem_l && helem && mu_e, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  SodParams p;
  if (params) p = *params;
  else sod_params_default(&p);
  p.gamma_gas = gamma_gas;
  // no derivative table: the routine differentiates nothing (dlxigp_ip is not among its arguments)
  SodMesh* m = nullptr;
  int rc = mesh_from_device_ref(nelem, npoin, index_base, connec, nullptr, gpvol, nullptr, invAtoIJK, gmshAtoI,
                                gmshAtoJ, gmshAtoK, wgp, helem_l, helem, npoin_w, lpoin_w, &p, st, &m);
  if (rc) return rc;
  rc = sod_smart_visc_spectral(m, Reta, rho, u, csound, Tem, eta, mu_e, stream);
  const int rw = sync_stream(st);
  sod_mesh_destroy(m);
  return rc ? rc : rw;
}

}  // extern "C"
