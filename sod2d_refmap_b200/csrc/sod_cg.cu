// Incompressible pressure Poisson: assembled CSR operator and Jacobi PCG (sm_100a).
//
// The operator is the pinned stiffness matrix that eval_laplacian_mult (lib_sod2d_incomp
// mod_operators.f90:20-128) applies matrix-free:
//   (K p)_a = sum_e sum_dir sum_{q on the dir-line through a} gpvol_q D[q_dir][a_dir]
//             sum_i He(i,dir,q) (He(q) grad_iso p)_i ,      p(pin) := 0, (K p)(pin) := 0,
// with pin = lpoin_w(1) = node 0 (mod_operators.f90:46-48,125-127).  Its element matrix is
//   K^e_ab = sum_q sum_{dir,dir'} M_q(dir,dir') D[q_dir][a_dir] D[q_dir'][b_dir'],
//   M_q = gpvol_q He_q^T He_q,  a on the dir-line and b on the dir'-line through q,
// so K couples the nodes of an element that share at least one ijk index.  Rows are assembled
// by their owner thread in ascending element order (deterministic, no atomics); the pinned row
// is empty and the pinned column is dropped.  The Jacobi diagonal is the unpinned K_aa, which
// equals eval_laplacian_diag (mod_operators.f90:417-461).
//
// conjGrad_pressure_incomp (mod_solver_incomp.f90:247-434) runs as: fused SpMV + <p,Ap>;
// device scalars alpha; fused x/r/z update with ||r||^2, <r,z-z_old>, <r,z>; device scalars
// beta; p update.  The host reads ||r||^2 each iteration for the stopping test, as the
// reference does after its MPI_Allreduce.  mixed != 0 runs FP32 CG sweeps (FP32 values and
// vectors) inside FP64 residual iterative refinement.
#include "sod_internal.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

struct SodPoisson {
  SodMesh* mesh = nullptr;
  int64_t n = 0, nnz = 0;
  int pin = 0;
  int32_t* rowptr = nullptr;
  int32_t* col = nullptr;
  double* val = nullptr;
  float* val32 = nullptr;
  double* diag = nullptr;
  // CG work vectors (FP64) and inner FP32 vectors
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *zold = nullptr, *b = nullptr;
  float *r32 = nullptr, *p32 = nullptr, *q32 = nullptr, *z32 = nullptr, *zold32 = nullptr, *e32 = nullptr;
  float* diag32 = nullptr;
  double* part = nullptr;   // block partials [4][nblk]
  int nblk = 0;
  double* scal = nullptr;   // device scalars
  double* hscal = nullptr;  // pinned host mirror
};

namespace sod {
namespace cg {

constexpr int kRowThreads = 8;  // threads per CSR row in the SpMV
constexpr int kBlock = 256;

// device scalar slots
enum { S_Q1 = 0, S_Q2, S_T1, S_NUM, S_ALPHA, S_BETA, S_Q1NEW, S_BNORM2, S_COUNT };

struct AsmArgs {
  int n, pin;
  const int32_t* n2e_ptr;
  const int32_t* n2e;
  const int32_t* econn;
  const double* geo;
  const int32_t* rowptr;
  const int32_t* col;
  double* val;
  double* diag;
  DMat D;
};

__device__ __forceinline__ int find_col(const int32_t* c, int lo, int hi, int key) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (c[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void k_assemble(const AsmArgs a) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= a.n) return;
  const int rb = a.rowptr[row], re = a.rowptr[row + 1];
  double dsum = 0.0;
  for (int c = a.n2e_ptr[row]; c < a.n2e_ptr[row + 1]; ++c) {
    const int pk = a.n2e[c];
    const int e = pk >> 6, da = pk & 63;
    const int ac[3] = {da & 3, (da >> 2) & 3, da >> 4};
    const double* G = a.geo + (size_t)e * NGEO * NN;
    const int32_t* conn = a.econn + (size_t)e * NN;
    for (int dir = 0; dir < 3; ++dir) {
      for (int m = 0; m < NP1; ++m) {
        const double c1 = a.D.d[m][ac[dir]];
        if (c1 == 0.0) continue;
        int gc[3] = {ac[0], ac[1], ac[2]};
        gc[dir] = m;
        const int g = gc[0] + 4 * gc[1] + 16 * gc[2];
        double H[9];
        for (int t = 0; t < 9; ++t) H[t] = G[t * NN + g];
        const double gv = G[9 * NN + g];
        for (int dp = 0; dp < 3; ++dp) {
          const double Mq = gv * (H[0 * 3 + dir] * H[0 * 3 + dp] + H[1 * 3 + dir] * H[1 * 3 + dp] +
                                  H[2 * 3 + dir] * H[2 * 3 + dp]);
          for (int np = 0; np < NP1; ++np) {
            const double c2 = a.D.d[gc[dp]][np];
            const double v = Mq * c1 * c2;
            int bc[3] = {gc[0], gc[1], gc[2]};
            bc[dp] = np;
            const int b = bc[0] + 4 * bc[1] + 16 * bc[2];
            if (b == da) dsum += v;
            const int colg = conn[b];
            if (row != a.pin && colg != a.pin) {
              const int pos = find_col(a.col, rb, re, colg);
              a.val[pos] += v;
            }
          }
        }
      }
    }
  }
  a.diag[row] = dsum;
}

template <typename T>
__global__ void k_cast(const double* __restrict__ s, T* __restrict__ d, int64_t n) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    d[t] = (T)s[t];
}

// y = A x (kRowThreads threads per row, fixed-order partial sums) fused with <x, y> partials
template <typename TV, typename TX>
__global__ void __launch_bounds__(kBlock) k_spmv_dot(int n, const int32_t* __restrict__ rowptr,
                                                     const int32_t* __restrict__ col, const TV* __restrict__ val,
                                                     const TX* __restrict__ x, TX* __restrict__ y,
                                                     double* __restrict__ part) {
  const int lane = threadIdx.x & (kRowThreads - 1);
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) / kRowThreads;
  double dot = 0.0;
  TX s = (TX)0;
  if (row < n) {
    const int b = rowptr[row], e = rowptr[row + 1];
    for (int c = b + lane; c < e; c += kRowThreads) s += (TX)val[c] * x[col[c]];
  }
  // every lane takes part in the shuffles (rows past n carry zero)
#pragma unroll
  for (int o = kRowThreads / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, kRowThreads);
  if (row < n && lane == 0) {
    y[row] = s;
    dot = (double)x[row] * (double)s;
  }
  // block partial of <x, y>
  for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, o);
  __shared__ double sh[kBlock / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = dot;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

template <int NP>
__device__ __forceinline__ void block_partials(double (&v)[NP], double* part, int stride) {
  __shared__ double sh[NP][kBlock / 32];
#pragma unroll
  for (int k = 0; k < NP; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < NP; ++k) sh[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      double t = 0.0;
      for (int w = 0; w < kBlock / 32; ++w) t += sh[k][w];
      part[k * stride + blockIdx.x] = t;
    }
}

// r = b - Ax (ax given), z = r/M, p = z; partials ||r||^2, <r,z>
template <typename TV>
__global__ void __launch_bounds__(kBlock) k_cg_init(int n, const TV* __restrict__ b, const TV* __restrict__ ax,
                                                    const TV* __restrict__ M, TV* r, TV* z, TV* p, TV* x,
                                                    double* part, int stride) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (i < n) {
    const TV ri = b[i] - (ax ? ax[i] : (TV)0);
    const TV zi = ri / M[i];
    r[i] = ri; z[i] = zi; p[i] = zi;
    if (x) x[i] = (TV)0;
    v[0] = (double)ri * (double)ri;
    v[1] = (double)ri * (double)zi;
  }
  block_partials<2>(v, part, stride);
}

// x += alpha p; r -= alpha q; z_old = z; z = r/M; partials ||r||^2, <r, z - z_old>, <r, z>
template <typename TV>
__global__ void __launch_bounds__(kBlock) k_cg_update(int n, const double* __restrict__ scal, TV* x, TV* r, TV* z,
                                                      const TV* __restrict__ p, const TV* __restrict__ q,
                                                      const TV* __restrict__ M, double* part, int stride) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[3] = {0.0, 0.0, 0.0};
  if (i < n) {
    const TV alpha = (TV)scal[S_ALPHA];
    x[i] = x[i] + alpha * p[i];
    const TV ri = r[i] - alpha * q[i];
    const TV zo = z[i];
    const TV zi = ri / M[i];
    r[i] = ri; z[i] = zi;
    v[0] = (double)ri * (double)ri;
    v[1] = (double)ri * ((double)zi - (double)zo);
    v[2] = (double)ri * (double)zi;
  }
  block_partials<3>(v, part, stride);
}

template <typename TV>
__global__ void k_cg_pupdate(int n, const double* __restrict__ scal, const TV* __restrict__ z, TV* p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = z[i] + (TV)scal[S_BETA] * p[i];
}

// single-block fixed-order reductions of the partials and the CG scalars
// mode 0: init  (part0 = ||r||^2 -> T1 and BNORM2, part1 = <r,z> -> Q1)
// mode 1: alpha (part0 = <p,Ap> -> Q2, alpha = Q1/Q2)
// mode 2: update(part0 -> T1, part1 -> num, part2 -> Q1new; beta = num/Q1; Q1 = Q1new)
// mode 3: norm  (part0 -> T1)
__global__ void __launch_bounds__(1024) k_cg_scalars(int nblk, const double* __restrict__ part, int stride,
                                                     int mode, double* scal) {
  __shared__ double sh[3][32];
  const int np = mode == 2 ? 3 : (mode == 0 ? 2 : 1);
  double v[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    for (int k = 0; k < np; ++k) v[k] += part[k * stride + b];
  for (int k = 0; k < 3; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) sh[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 3; ++k)
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t[k] += sh[k][w];
    if (mode == 0) {
      scal[S_T1] = t[0]; scal[S_BNORM2] = t[0]; scal[S_Q1] = t[1];
    } else if (mode == 1) {
      scal[S_Q2] = t[0]; scal[S_ALPHA] = scal[S_Q1] / t[0];
    } else if (mode == 2) {
      scal[S_T1] = t[0]; scal[S_NUM] = t[1]; scal[S_BETA] = t[1] / scal[S_Q1]; scal[S_Q1] = t[2];
    } else {
      scal[S_T1] = t[0];
    }
  }
}

// out = a - b with out[pin] = 0 (b may be null)
template <typename T>
__global__ void k_sub_pin(int n, int pin, const T* __restrict__ a, const T* __restrict__ b, T* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (i == pin) ? (T)0 : a[i] - (b ? b[i] : (T)0);
}
__global__ void k_axpy_cast(int n, const float* __restrict__ e, double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += (double)e[i];
}
__global__ void k_add(int n, const double* __restrict__ a, const double* __restrict__ b, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

}  // namespace cg
}  // namespace sod

using namespace sod;
using namespace sod::cg;

static int spmv_grid(int64_t n) { return (int)((n * kRowThreads + kBlock - 1) / kBlock); }

template <typename TV, typename TX>
static int spmv(SodPoisson* P, const TV* val, const TX* x, TX* y, cudaStream_t st) {
  k_spmv_dot<TV, TX><<<spmv_grid(P->n), kBlock, 0, st>>>((int)P->n, P->rowptr, P->col, val, x, y, P->part);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

static int scalars(SodPoisson* P, int nblk, int mode, cudaStream_t st) {
  k_cg_scalars<<<1, 1024, 0, st>>>(nblk, P->part, P->nblk, mode, P->scal);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

static int read_T1(SodPoisson* P, cudaStream_t st, double* T1) {
  SOD_CUDA(cudaMemcpyAsync(P->hscal, P->scal, sizeof(double) * S_COUNT, cudaMemcpyDeviceToHost, st));
  SOD_CUDA(cudaStreamSynchronize(st));
  *T1 = P->hscal[S_T1];
  return SOD_OK;
}

// Jacobi PCG on A e = rhs (vectors TV, values TM) in the reference's iteration order; e starts
// at 0.  Stops when ||r|| < tol * ||r0|| or after max_iter; returns the iteration count.
template <typename TV, typename TM>
static int pcg(SodPoisson* P, const TM* val, const TV* M, const TV* rhs, TV* e, TV* r, TV* z, TV* p, TV* q,
               int max_iter, double tol, cudaStream_t st, int* iters, double* rel) {
  const int n = (int)P->n;
  const int gb = (n + kBlock - 1) / kBlock;
  k_cg_init<TV><<<gb, kBlock, 0, st>>>(n, rhs, (const TV*)nullptr, M, r, z, p, e, P->part, P->nblk);
  SOD_CHECK_LAUNCH();
  if (int rc = scalars(P, gb, 0, st)) return rc;
  double T1 = 0.0;
  if (int rc = read_T1(P, st, &T1)) return rc;
  const double auxB = std::sqrt(P->hscal[S_BNORM2]);
  int it = 0;
  if (auxB == 0.0) {
    *iters = 0;
    *rel = 0.0;
    return SOD_OK;
  }
  for (it = 1; it <= max_iter; ++it) {
    if (int rc = spmv<TM, TV>(P, val, p, q, st)) return rc;
    if (int rc = scalars(P, spmv_grid(n), 1, st)) return rc;
    k_cg_update<TV><<<gb, kBlock, 0, st>>>(n, P->scal, e, r, z, p, q, M, P->part, P->nblk);
    SOD_CHECK_LAUNCH();
    if (int rc = scalars(P, gb, 2, st)) return rc;
    if (int rc = read_T1(P, st, &T1)) return rc;
    if (std::sqrt(T1) < tol * auxB) break;
    k_cg_pupdate<TV><<<gb, kBlock, 0, st>>>(n, P->scal, z, p);
    SOD_CHECK_LAUNCH();
  }
  *iters = it > max_iter ? max_iter : it;
  *rel = std::sqrt(T1) / auxB;
  return SOD_OK;
}

extern "C" {

void sod_poisson_destroy(SodPoisson* P) {
  if (!P) return;
  void* ptrs[] = {P->rowptr, P->col, P->val, P->val32, P->diag, P->x, P->r, P->p, P->q, P->z, P->zold, P->b,
                  P->r32, P->p32, P->q32, P->z32, P->zold32, P->e32, P->diag32, P->part, P->scal};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (P->hscal) cudaFreeHost(P->hscal);
  delete P;
}

int sod_poisson_create(SodMesh* m, SodPoisson** out) {
  SOD_ARG(m && out, "mesh/out null");
  *out = nullptr;
  const int N = m->npoin, E = m->nelem;
  const int pin = 0;
  // host copies of the connectivity and node->element map
  std::vector<int32_t> econn((size_t)E * NN), nptr(N + 1), nidx((size_t)E * NN);
  SOD_CUDA(cudaMemcpy(econn.data(), m->econn, sizeof(int32_t) * econn.size(), cudaMemcpyDeviceToHost));
  SOD_CUDA(cudaMemcpy(nptr.data(), m->n2e_ptr, sizeof(int32_t) * (N + 1), cudaMemcpyDeviceToHost));
  SOD_CUDA(cudaMemcpy(nidx.data(), m->n2e, sizeof(int32_t) * nidx.size(), cudaMemcpyDeviceToHost));
  // local pairs sharing at least one ijk index (the structural nonzeros of K^e)
  std::vector<int> share[NN];
  for (int a = 0; a < NN; ++a)
    for (int b = 0; b < NN; ++b)
      if ((a & 3) == (b & 3) || ((a >> 2) & 3) == ((b >> 2) & 3) || (a >> 4) == (b >> 4)) share[a].push_back(b);
  std::vector<int32_t> rowptr(N + 1, 0);
  std::vector<int32_t> tmp;
  tmp.reserve(1024);
  auto row_cols = [&](int n) {
    tmp.clear();
    if (n == pin) return;
    for (int c = nptr[n]; c < nptr[n + 1]; ++c) {
      const int e = nidx[c] >> 6, da = nidx[c] & 63;
      for (int b : share[da]) {
        const int32_t cg = econn[(size_t)e * NN + b];
        if (cg != pin) tmp.push_back(cg);
      }
    }
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
  };
  for (int n = 0; n < N; ++n) {
    row_cols(n);
    rowptr[n + 1] = rowptr[n] + (int32_t)tmp.size();
    if ((int64_t)rowptr[n + 1] > (int64_t)INT32_MAX - 4096) {
      set_error("Poisson CSR exceeds int32 indices");
      return SOD_ERR_UNSUPPORTED;
    }
  }
  const int64_t nnz = rowptr[N];
  std::vector<int32_t> col(nnz);
  for (int n = 0; n < N; ++n) {
    row_cols(n);
    std::copy(tmp.begin(), tmp.end(), col.begin() + rowptr[n]);
  }
  SodPoisson* P = new SodPoisson();
  P->mesh = m; P->n = N; P->nnz = nnz; P->pin = pin;
  P->nblk = std::max(spmv_grid(N), (N + kBlock - 1) / kBlock);
  auto fail = [&](const char* what) {
    set_error("sod_poisson_create: %s failed", what);
    sod_poisson_destroy(P);
    return SOD_ERR_NOMEM;
  };
#define PALLOC(ptr, bytes) if (cudaMalloc(&(ptr), (bytes)) != cudaSuccess) return fail(#ptr)
  PALLOC(P->rowptr, sizeof(int32_t) * (N + 1));
  PALLOC(P->col, sizeof(int32_t) * (nnz > 0 ? nnz : 1));
  PALLOC(P->val, sizeof(double) * (nnz > 0 ? nnz : 1));
  PALLOC(P->val32, sizeof(float) * (nnz > 0 ? nnz : 1));
  PALLOC(P->diag, sizeof(double) * N);
  PALLOC(P->diag32, sizeof(float) * N);
  for (double** v : {&P->x, &P->r, &P->p, &P->q, &P->z, &P->zold, &P->b}) PALLOC(*v, sizeof(double) * N);
  for (float** v : {&P->r32, &P->p32, &P->q32, &P->z32, &P->zold32, &P->e32}) PALLOC(*v, sizeof(float) * N);
  PALLOC(P->part, sizeof(double) * 4 * P->nblk);
  PALLOC(P->scal, sizeof(double) * S_COUNT);
#undef PALLOC
  if (cudaMallocHost(&P->hscal, sizeof(double) * S_COUNT) != cudaSuccess) return fail("hscal");
  cudaMemcpy(P->rowptr, rowptr.data(), sizeof(int32_t) * (N + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(P->col, col.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice);
  cudaMemset(P->val, 0, sizeof(double) * (nnz > 0 ? nnz : 1));
  AsmArgs a;
  a.n = N; a.pin = pin; a.n2e_ptr = m->n2e_ptr; a.n2e = m->n2e; a.econn = m->econn; a.geo = m->geo64;
  a.rowptr = P->rowptr; a.col = P->col; a.val = P->val; a.diag = P->diag; a.D = m->D;
  k_assemble<<<(N + 127) / 128, 128>>>(a);
  g_launches.fetch_add(1);
  k_cast<float><<<1024, 256>>>(P->val, P->val32, nnz);
  k_cast<float><<<256, 256>>>(P->diag, P->diag32, N);
  g_launches.fetch_add(2);
  cudaError_t err = cudaDeviceSynchronize();
  if (err != cudaSuccess) {
    set_error("Poisson assembly: %s", cudaGetErrorString(err));
    sod_poisson_destroy(P);
    return SOD_ERR_CUDA;
  }
  *out = P;
  return SOD_OK;
}

int sod_poisson_nnz(SodPoisson* P, int64_t* nnz) {
  SOD_ARG(P && nnz, "null argument");
  *nnz = P->nnz;
  return SOD_OK;
}

int sod_poisson_apply(SodPoisson* P, const double* x, double* y, sod_stream_t stream) {
  SOD_ARG(P && x && y, "null argument");
  return spmv<double, double>(P, P->val, x, y, (cudaStream_t)stream);
}

int sod_poisson_diag(SodPoisson* P, double* d, sod_stream_t stream) {
  SOD_ARG(P && d, "null argument");
  SOD_CUDA(cudaMemcpyAsync(d, P->diag, sizeof(double) * P->n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return SOD_OK;
}

int sod_conjgrad_pressure(SodPoisson* P, const double* Rp0, double* R, int max_iter, double tol, int mixed,
                          int* iters_out, double* rel_out, sod_stream_t stream) {
  SOD_ARG(P && Rp0 && R && max_iter > 0 && tol > 0.0, "conjgrad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = (int)P->n;
  const int gb = (n + kBlock - 1) / kBlock;
  // b = R - A x0, b(pin) = 0 (mod_solver_incomp.f90:307-317)
  if (int rc = spmv<double, double>(P, P->val, Rp0, P->q, st)) return rc;
  k_sub_pin<double><<<gb, kBlock, 0, st>>>(n, P->pin, R, P->q, P->b);
  SOD_CHECK_LAUNCH();
  int iters = 0;
  double rel = 0.0;
  if (!mixed) {
    int rc = pcg<double, double>(P, P->val, P->diag, P->b, P->x, P->r, P->z, P->p, P->q, max_iter, tol, st, &iters, &rel);
    if (rc) return rc;
  } else {
    // FP64 residual iterative refinement around FP32 Jacobi-PCG sweeps
    k_cg_init<double><<<gb, kBlock, 0, st>>>(n, P->b, (const double*)nullptr, P->diag, P->r, P->z, P->p, P->x,
                                             P->part, P->nblk);
    SOD_CHECK_LAUNCH();
    if (int rc = scalars(P, gb, 0, st)) return rc;
    double T1 = 0.0;
    if (int rc = read_T1(P, st, &T1)) return rc;
    const double bnorm = std::sqrt(P->hscal[S_BNORM2]);
    rel = bnorm > 0.0 ? 1.0 : 0.0;
    for (int outer = 0; outer < 64 && rel >= tol && iters < max_iter; ++outer) {
      // each FP32 sweep is asked for the remaining reduction, but not below what FP32 resolves
      const double inner_tol = std::max(0.5 * tol / rel, 2e-6);
      k_cast<float><<<gb, kBlock, 0, st>>>(P->r, P->r32, n);
      SOD_CHECK_LAUNCH();
      int it_in = 0;
      double rel_in = 0.0;
      int rc = pcg<float, float>(P, P->val32, P->diag32, P->r32, P->e32, P->zold32, P->z32, P->p32, P->q32,
                                 max_iter - iters, inner_tol, st, &it_in, &rel_in);
      if (rc) return rc;
      iters += it_in;
      k_axpy_cast<<<gb, kBlock, 0, st>>>(n, P->e32, P->x);
      SOD_CHECK_LAUNCH();
      // r = b - A x in FP64, ||r||^2
      if (int rc2 = spmv<double, double>(P, P->val, P->x, P->q, st)) return rc2;
      k_cg_init<double><<<gb, kBlock, 0, st>>>(n, P->b, P->q, P->diag, P->r, P->z, P->p, (double*)nullptr, P->part,
                                               P->nblk);
      SOD_CHECK_LAUNCH();
      if (int rc3 = scalars(P, gb, 3, st)) return rc3;
      if (int rc4 = read_T1(P, st, &T1)) return rc4;
      rel = std::sqrt(T1) / bnorm;
    }
  }
  // R = x0 + x (mod_solver_incomp.f90:428-430)
  k_add<<<gb, kBlock, 0, st>>>(n, Rp0, P->x, R);
  SOD_CHECK_LAUNCH();
  if (iters_out) *iters_out = iters;
  if (rel_out) *rel_out = rel;
  if (rel >= tol) {
    set_error("conjgrad: relative residual %.3e after %d iterations (tol %.1e)", rel, iters, tol);
    return SOD_ERR_NOT_CONVERGED;
  }
  return SOD_OK;
}

}  // extern "C"
