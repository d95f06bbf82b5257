// Legacy element-loop API of the unit tests (sm_100a): mass_convec, generic_scalar_convec,
// mom_convec, ener_convec (unitt/unitt_{mass,generic_scalar,mom,ener}_convec/*.f90, arithmetic of
// the companion .m scripts) and mom_diffusion (unitt/unitt_mom_diffu/unitt_mom_diffu.f90, weak
// form with the stress of full_diffusion_ijk).  Generic elements (ndime 2 or 3, nnode and ngaus
// up to 64) described by the caller's gpcar/gpvol/Ngp tables, Fortran layouts, 1-based connec,
// device arrays.  One CTA per element; the element residuals are assembled by a node-ordered
// gather (node -> (element, local node) lists sorted ascending), so results do not depend on
// scheduling.  Scratch is stream-ordered (cudaMallocAsync / cudaFreeAsync).
#include "sod_internal.cuh"

namespace sod {
namespace legacy {

constexpr int kMaxNode = 64;
enum Mode { MASS = 0, MOM = 1, ENER = 2, DIFF = 3 };

struct Args {
  int nelem, ngaus, npoin, nnode, ndime;
  const int32_t* connec;
  const double* Ngp;
  const double* gpcar;
  const double* gpvol;
  const double* f;   // q (mass, mom) / u (ener, diff)
  const double* g;   // u (mom) / E (ener) / mu_e (diff)
  const double* s;   // pr (mom, ener)
  double* rel;       // [(e*nnode + a)*3 + c]
};

template <int MODE>
__global__ void __launch_bounds__(kMaxNode) k_legacy_elem(const Args a) {
  __shared__ double val[kMaxNode][9];  // per Gauss point: divergence(s) or stress tensor
  __shared__ int ip[kMaxNode];
  const int e = blockIdx.x, t = threadIdx.x;
  const int nn = a.nnode, ng = a.ngaus, nd = a.ndime;
  const int64_t np = a.npoin;
  if (t < nn) ip[t] = a.connec[e + (int64_t)a.nelem * t] - 1;
  __syncthreads();
  if (t < ng) {
    const double* car = a.gpcar + (size_t)nd * nn * (t + (size_t)ng * e);
    if (MODE == DIFF) {
      double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // d u_i / d x_j
      for (int b = 0; b < nn; ++b)
        for (int i = 0; i < nd; ++i)
          for (int j = 0; j < nd; ++j) gu[i][j] += car[j + nd * b] * a.f[ip[b] + np * i];
      double divu = 0.0;
      for (int i = 0; i < nd; ++i) divu += gu[i][i];
      const double mu = a.g[e];
      for (int i = 0; i < nd; ++i)
        for (int j = 0; j < nd; ++j)
          val[t][3 * i + j] = mu * (gu[i][j] + gu[j][i]) - (i == j ? mu * (2.0 / 3.0) * divu : 0.0);
    } else {
      const int ncomp = MODE == MOM ? nd : 1;
      for (int c = 0; c < ncomp; ++c) {
        double acc = 0.0;
        for (int b = 0; b < nn; ++b) {
          const int64_t pb = ip[b];
          if (MODE == MASS) {
            for (int d = 0; d < nd; ++d) acc += car[d + nd * b] * a.f[pb + np * d];
          } else if (MODE == ENER) {
            for (int d = 0; d < nd; ++d) acc += car[d + nd * b] * (a.f[pb + np * d] * (a.g[pb] + a.s[pb]));
          } else {
            for (int d = 0; d < nd; ++d) acc += car[d + nd * b] * (a.f[pb + np * c] * a.g[pb + np * d]);
            acc += car[c + nd * b] * a.s[pb];
          }
        }
        val[t][c] = acc;
      }
    }
  }
  __syncthreads();
  if (t < nn) {
    const int ncomp = (MODE == MOM || MODE == DIFF) ? nd : 1;
    double r[3] = {0.0, 0.0, 0.0};
    for (int gp = 0; gp < ng; ++gp) {
      const double vol = a.gpvol[gp + (size_t)ng * e];
      if (MODE == DIFF) {
        const double* car = a.gpcar + (size_t)nd * nn * (gp + (size_t)ng * e);
        for (int i = 0; i < nd; ++i) {
          double acc = 0.0;
          for (int j = 0; j < nd; ++j) acc += car[j + nd * t] * val[gp][3 * i + j];
          r[i] += vol * acc;
        }
      } else {
        const double w = vol * a.Ngp[gp + (size_t)ng * t];
        for (int c = 0; c < ncomp; ++c) r[c] += w * val[gp][c];
      }
    }
    double* o = a.rel + ((size_t)e * nn + t) * 3;
    o[0] = r[0]; o[1] = r[1]; o[2] = r[2];
  }
}

// node -> (element, local node) lists: count, single-block exclusive scan, fill, sort
__global__ void k_count(int nelem, int nnode, const int32_t* connec, int npoin, int* cnt, int* bad) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * nnode) return;
  const int n = connec[t] - 1;  // connec(e, a) at e + nelem*a
  if (n < 0 || n >= npoin) { atomicExch(bad, 1); return; }
  atomicAdd(cnt + n, 1);
}

__global__ void k_scan(int npoin, const int* cnt, int* ptr) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const int chunk = (npoin + 1023) / 1024;
  const int b = t * chunk, e = min(npoin, b + chunk);
  int s = 0;
  for (int i = b; i < e; ++i) s += cnt[i];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    int acc = 0;
    for (int i = 0; i < 1024; ++i) { const int v = part[i]; part[i] = acc; acc += v; }
    ptr[npoin] = acc;
  }
  __syncthreads();
  int acc = part[t];
  for (int i = b; i < e; ++i) { ptr[i] = acc; acc += cnt[i]; }
}

__global__ void k_fill(int nelem, int nnode, const int32_t* connec, const int* ptr, int* cur, int* list) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * nnode) return;
  const int n = connec[t] - 1;
  const int e = (int)(t % nelem), a = (int)(t / nelem);
  list[ptr[n] + atomicAdd(cur + n, 1)] = e * nnode + a;  // packed (element, local node)
}

__global__ void k_sort_gather(int npoin, int ncomp, const int* ptr, int* list, const double* rel, double* R) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  const int b = ptr[n], e = ptr[n + 1];
  for (int i = b + 1; i < e; ++i) {  // ascending (element, local node): a fixed summation order
    const int v = list[i];
    int j = i - 1;
    while (j >= b && list[j] > v) { list[j + 1] = list[j]; --j; }
    list[j + 1] = v;
  }
  double r[3] = {0.0, 0.0, 0.0};
  for (int i = b; i < e; ++i) {
    const double* src = rel + (size_t)list[i] * 3;
    for (int c = 0; c < ncomp; ++c) r[c] += src[c];
  }
  for (int c = 0; c < ncomp; ++c) R[n + (int64_t)npoin * c] = r[c];
}

template <int MODE>
static int run(const Args& in, double* R, cudaStream_t st) {
  SOD_ARG(in.nelem > 0 && in.npoin > 0 && in.nnode > 0 && in.ngaus > 0, "sizes must be positive");
  SOD_ARG(in.nnode <= kMaxNode && in.ngaus <= kMaxNode, "nnode and ngaus must be <= 64");
  SOD_ARG(in.ndime == 2 || in.ndime == 3, "ndime must be 2 or 3");
  SOD_ARG((int64_t)in.nelem * in.nnode < ((int64_t)1 << 31), "nelem*nnode must fit int32");
  SOD_ARG(in.connec && in.gpcar && in.gpvol && in.f && R, "null input");
  SOD_ARG(MODE == DIFF || in.Ngp, "Ngp null");
  SOD_ARG(MODE == MASS || in.g, "second field null");
  SOD_ARG((MODE != MOM && MODE != ENER) || in.s, "pressure null");
  const int64_t EN = (int64_t)in.nelem * in.nnode;
  const int ncomp = (MODE == MOM || MODE == DIFF) ? in.ndime : 1;
  double* rel = nullptr;
  int *cnt = nullptr, *ptr = nullptr, *list = nullptr;
  SOD_CUDA(cudaMallocAsync((void**)&rel, sizeof(double) * 3 * EN, st));
  SOD_CUDA(cudaMallocAsync((void**)&cnt, sizeof(int) * (2 * (size_t)in.npoin + 2), st));  // cnt, cursor, bad flag
  SOD_CUDA(cudaMallocAsync((void**)&ptr, sizeof(int) * ((size_t)in.npoin + 1), st));
  SOD_CUDA(cudaMallocAsync((void**)&list, sizeof(int) * EN, st));
  int* cur = cnt + in.npoin;
  int* bad = cnt + 2 * (size_t)in.npoin;
  int rc = SOD_OK;
  do {
    if (cudaMemsetAsync(cnt, 0, sizeof(int) * (2 * (size_t)in.npoin + 2), st) != cudaSuccess) { rc = SOD_ERR_CUDA; break; }
    const unsigned gE = (unsigned)((EN + 255) / 256);
    k_count<<<gE, 256, 0, st>>>(in.nelem, in.nnode, in.connec, in.npoin, cnt, bad);
    int hbad = 0;
    if (cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) { rc = SOD_ERR_CUDA; break; }
    if (hbad) { set_error("invalid argument: connec entry outside 1..npoin"); rc = SOD_ERR_ARG; break; }
    k_scan<<<1, 1024, 0, st>>>(in.npoin, cnt, ptr);
    k_fill<<<gE, 256, 0, st>>>(in.nelem, in.nnode, in.connec, ptr, cur, list);
    Args a = in;
    a.rel = rel;
    k_legacy_elem<MODE><<<in.nelem, kMaxNode, 0, st>>>(a);
    k_sort_gather<<<(in.npoin + 255) / 256, 256, 0, st>>>(in.npoin, ncomp, ptr, list, rel, R);
    if (cudaGetLastError() != cudaSuccess) { rc = SOD_ERR_CUDA; break; }
    g_launches.fetch_add(5);
  } while (false);
  cudaFreeAsync(rel, st);
  cudaFreeAsync(cnt, st);
  cudaFreeAsync(ptr, st);
  cudaFreeAsync(list, st);
  if (rc == SOD_ERR_CUDA) set_error("CUDA error in a legacy element-loop entry point");
  return rc;
}

}  // namespace legacy
}  // namespace sod

using namespace sod::legacy;

extern "C" {

int sod_legacy_mass_convec(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                           const int32_t* connec, const double* Ngp, const double* gpcar, const double* gpvol,
                           const double* q, double* R, sod_stream_t stream) {
  Args a{nelem, ngaus, npoin, nnode, ndime, connec, Ngp, gpcar, gpvol, q, nullptr, nullptr, nullptr};
  return run<MASS>(a, R, (cudaStream_t)stream);
}

int sod_legacy_generic_scalar_convec(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                                     const int32_t* connec, const double* Ngp, const double* gpcar,
                                     const double* gpvol, const double* q, double* R, sod_stream_t stream) {
  Args a{nelem, ngaus, npoin, nnode, ndime, connec, Ngp, gpcar, gpvol, q, nullptr, nullptr, nullptr};
  return run<MASS>(a, R, (cudaStream_t)stream);
}

int sod_legacy_mom_convec(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                          const int32_t* connec, const double* Ngp, const double* gpcar, const double* gpvol,
                          const double* u, const double* q, const double* pr, double* R, sod_stream_t stream) {
  Args a{nelem, ngaus, npoin, nnode, ndime, connec, Ngp, gpcar, gpvol, q, u, pr, nullptr};
  return run<MOM>(a, R, (cudaStream_t)stream);
}

int sod_legacy_ener_convec(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                           const int32_t* connec, const double* Ngp, const double* gpcar, const double* gpvol,
                           const double* u, const double* pr, const double* E, double* R, sod_stream_t stream) {
  Args a{nelem, ngaus, npoin, nnode, ndime, connec, Ngp, gpcar, gpvol, u, E, pr, nullptr};
  return run<ENER>(a, R, (cudaStream_t)stream);
}

int sod_legacy_mom_diffusion(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                             const int32_t* connec, const double* Ngp, const double* gpcar, const double* gpvol,
                             const double* u, const double* mu_e, double* R, sod_stream_t stream) {
  Args a{nelem, ngaus, npoin, nnode, ndime, connec, Ngp, gpcar, gpvol, u, mu_e, nullptr, nullptr};
  return run<DIFF>(a, R, (cudaStream_t)stream);
}

}  // extern "C"
