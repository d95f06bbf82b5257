// Incompressible pressure Poisson: matrix-free operator and Jacobi PCG (sm_100a).
//
// The operator is eval_laplacian_mult (lib_sod2d_incomp mod_operators.f90:20-128), applied
// matrix-free as the reference does:
//   (K p)_a = sum_e sum_dir sum_{q on the dir-line through a} D[q_dir][a_dir] F_dir(q),
//   F(q) = gpvol_q He_q^T He_q grad_iso p(q),          p(pin) := 0, (K p)(pin) := 0,
// with pin = lpoin_w(1) = node 0 (mod_operators.f90:46-48,125-127).  The symmetric 3x3
// M_q = gpvol_q He_q^T He_q is formed once per gauss point at setup (6 values: the reference
// re-reads He and gpvol, 10 values, on every product), in FP64 and in an FP32 copy.
//
// One product is two kernels.  k_lap_elem_async: one thread per gauss point, EPB elements per
// group, persistent CTAs (SMs x 3) that stream the metric and connectivity of their next 4
// groups through a cp.async shared-memory ring and gather the next group's p during the
// current group's arithmetic; the element's p goes to shared memory, the three line
// derivatives and F are formed in registers, F goes back to shared memory and the transposed
// line sums give the element residual, stored as rel[e*64 + d].  The kernel is bound by the
// bytes it keeps in flight: one group per CTA (k_lap_elem, the fallback when the occupancy
// query gives no resident CTA) reaches 4.1 TB/s on the same bytes.  k_lap_gather: one thread
// per node sums its element residuals through the node->element CSR in ascending element
// order (deterministic; the reference uses atomics) and adds <p, Kp> to per-block partials.
//
// The Jacobi diagonal is eval_laplacian_diag (mod_operators.f90:417-461): the unpinned K_aa.
//
// conjGrad_pressure_incomp (mod_solver_incomp.f90:247-434) runs as: product + <p,Ap>, whose
// last block forms alpha; fused x/r/z update with ||r||^2, <r,z-z_old>, <r,z>, whose last block
// forms beta and the stop test ||r|| < tol ||r0|| (:393); p update: four launches per iteration.  The stop test, the iteration counter and
// a done flag live on the device, so iterations are replayed in CUDA-graph batches of kBatch
// and the host reads the scalars once per batch; every kernel of an iteration after the
// converged one returns at once, so the iterate and the count are those of a host-tested
// loop.  mixed != 0 runs FP32 CG sweeps (FP32 metric and vectors) inside FP64 residual
// iterative refinement.
#include "sod_internal.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace sod {
namespace cg {

constexpr int kBlock = 256;
constexpr int EPB = 4;      // elements per CTA of the element kernels
constexpr int NSTAGE = 4;   // cp.async ring stages of the streamed element kernel
constexpr int kRingCtas = 3; // its resident CTAs per SM (3 x 64.6 KB shared memory in FP64)
constexpr int kGather = 8;   // residual loads in flight per node in the gather
constexpr int NMET = 6;     // M00, M01, M02, M11, M12, M22
constexpr int kBatch = 16;  // CG iterations per graph replay

// device scalar slots
enum {
  S_Q1 = 0, S_Q2, S_T1, S_NUM, S_ALPHA, S_BETA, S_BNORM2, S_TOL, S_ITER, S_MAXIT, S_DONE, S_COUNT
};

template <typename T>
struct DT {
  T d[NP1][NP1];
};

}  // namespace cg
}  // namespace sod

struct SodPoisson {
  SodMesh* mesh = nullptr;
  int64_t n = 0, nelem = 0;
  int pin = 0;
  double* met = nullptr;   // [e][6][64]  gpvol He^T He
  float* met32 = nullptr;
  double* diag = nullptr;
  float* diag32 = nullptr;
  void* rel = nullptr;     // element residuals [e*64 + d] (double, or float for the FP32 sweeps)
  // CG work vectors (FP64) and inner FP32 vectors
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *b = nullptr;
  float *r32 = nullptr, *p32 = nullptr, *q32 = nullptr, *z32 = nullptr, *e32 = nullptr;
  double* part = nullptr;  // block partials [3][nblk]
  unsigned int* counter = nullptr;  // blocks done, for the last-block scalar reductions
  int red_blocks = 0;               // grid of the node kernels that reduce (8 CTAs per SM)
  int nblk = 0;
  double* scal = nullptr;  // device scalars
  double* hscal = nullptr; // pinned host mirror
  sod::cg::DT<double> D64;
  sod::cg::DT<float> D32;
  cudaGraphExec_t batch[2] = {nullptr, nullptr};  // kBatch iterations: FP64, FP32
  int batch_kernels[2] = {0, 0};
  int ring_grid[2] = {0, 0};  // streamed element-kernel grid: FP64, FP32 (SMs x resident CTAs)
};

namespace sod {
namespace cg {

// M_q = gpvol He^T He at every gauss point (He(r,c) = geo[3r+c])
__global__ void k_metric(int64_t total, const double* __restrict__ geo, double* __restrict__ met,
                         float* __restrict__ met32) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / NN;
    const int d = (int)(t % NN);
    const double* G = geo + e * NGEO * NN;
    double H[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) H[c] = G[c * NN + d];
    const double gv = G[9 * NN + d];
    const int rc[NMET][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
    for (int c = 0; c < NMET; ++c) {
      const int a = rc[c][0], b = rc[c][1];
      const double v = gv * (H[a] * H[b] + H[3 + a] * H[3 + b] + H[6 + a] * H[6 + b]);
      met[(e * NMET + c) * NN + d] = v;
      met32[(e * NMET + c) * NN + d] = (float)v;
    }
  }
}

// Jacobi diagonal K_aa (unpinned), one thread per node over its elements in ascending order
__global__ void k_diag(int n, const int32_t* __restrict__ n2e_ptr, const int32_t* __restrict__ n2e,
                       const double* __restrict__ geo, const DMat D, double* __restrict__ diag,
                       float* __restrict__ diag32) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  double dsum = 0.0;
  for (int c = n2e_ptr[row]; c < n2e_ptr[row + 1]; ++c) {
    const int pk = n2e[c];
    const int e = pk >> 6, da = pk & 63;
    const int ac[3] = {da & 3, (da >> 2) & 3, da >> 4};
    const double* G = geo + (size_t)e * NGEO * NN;
    for (int dir = 0; dir < 3; ++dir) {
      for (int m = 0; m < NP1; ++m) {
        const double c1 = D.d[m][ac[dir]];
        if (c1 == 0.0) continue;
        int gc[3] = {ac[0], ac[1], ac[2]};
        gc[dir] = m;
        const int g = gc[0] + 4 * gc[1] + 16 * gc[2];
        double H[9];
        for (int t = 0; t < 9; ++t) H[t] = G[t * NN + g];
        const double gv = G[9 * NN + g];
        for (int dp = 0; dp < 3; ++dp) {
          // the entry (a, a) needs the dp-line through q to pass through a
          if (dp != dir && m != ac[dir]) continue;
          const double Mq = gv * (H[0 * 3 + dir] * H[0 * 3 + dp] + H[1 * 3 + dir] * H[1 * 3 + dp] +
                                  H[2 * 3 + dir] * H[2 * 3 + dp]);
          dsum += Mq * c1 * D.d[gc[dp]][ac[dp]];
        }
      }
    }
  }
  diag[row] = dsum;
  diag32[row] = (float)dsum;
}

// element residuals of K x (x(pin) read as 0); skipped once the solve is done
template <typename T>
__global__ void __launch_bounds__(64 * EPB) k_lap_elem(int nelem, int pin, const int32_t* __restrict__ econn,
                                                      const T* __restrict__ met, const DT<T> D,
                                                      const T* __restrict__ x, T* __restrict__ rel,
                                                      const double* __restrict__ scal) {
  if (scal && scal[S_DONE] != 0.0) return;
  __shared__ T pl[EPB][FSTRIDE];
  __shared__ T fl[EPB][3][FSTRIDE];
  __shared__ T Ds[NP1][NP1];
  const int es = threadIdx.x >> 6, d = threadIdx.x & 63;
  if (threadIdx.x == 0) {  // constant indices: D stays in the parameter bank
#pragma unroll
    for (int a = 0; a < NP1; ++a)
#pragma unroll
      for (int b = 0; b < NP1; ++b) Ds[a][b] = D.d[a][b];
  }
  const int e = blockIdx.x * EPB + es;
  const bool act = e < nelem;
  const int ee = act ? e : nelem - 1;
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  const int nd = econn[(size_t)ee * NN + d];
  pl[es][s] = nd == pin ? (T)0 : x[nd];
  T M[NMET];
#pragma unroll
  for (int c = 0; c < NMET; ++c) M[c] = met[((size_t)ee * NMET + c) * NN + d];
  __syncthreads();
  T Dx[NP1], Dy[NP1], Dz[NP1], DTx[NP1], DTy[NP1], DTz[NP1];
#pragma unroll
  for (int m = 0; m < NP1; ++m) {
    Dx[m] = Ds[i][m]; Dy[m] = Ds[j][m]; Dz[m] = Ds[k][m];
    DTx[m] = Ds[m][i]; DTy[m] = Ds[m][j]; DTz[m] = Ds[m][k];
  }
  const T* f = pl[es];
  T g0 = (T)0, g1 = (T)0, g2 = (T)0;
#pragma unroll
  for (int m = 0; m < NP1; ++m) {
    g0 += Dx[m] * f[sidx(m, j, k)];
    g1 += Dy[m] * f[sidx(i, m, k)];
    g2 += Dz[m] * f[sidx(i, j, m)];
  }
  fl[es][0][s] = M[0] * g0 + M[1] * g1 + M[2] * g2;
  fl[es][1][s] = M[1] * g0 + M[3] * g1 + M[4] * g2;
  fl[es][2][s] = M[2] * g0 + M[4] * g1 + M[5] * g2;
  __syncthreads();
  T acc = (T)0;
#pragma unroll
  for (int m = 0; m < NP1; ++m) {
    acc += DTx[m] * fl[es][0][sidx(m, j, k)];
    acc += DTy[m] * fl[es][1][sidx(i, m, k)];
    acc += DTz[m] * fl[es][2][sidx(i, j, m)];
  }
  if (act) rel[(size_t)e * NN + d] = acc;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Streamed form of k_lap_elem: persistent CTAs, the metric and connectivity of the next
// NSTAGE element groups copied into a shared-memory ring by cp.async (16-byte chunks, L1
// bypassed), so that several groups' bytes are in flight per CTA, and the p values of the
// next group gathered during the current group's arithmetic.  Same arithmetic and order as
// k_lap_elem (bitwise equal results).  Stage layout: metric [EPB][6][64] T, then
// connectivity [EPB][64] int32.
template <typename T, int NSTAGE>
struct LapRing {
  static constexpr int kMetBytes = EPB * NMET * NN * (int)sizeof(T);
  static constexpr int kConnBytes = EPB * NN * 4;
  static constexpr int kStage = kMetBytes + kConnBytes;
  static constexpr int kBytes = NSTAGE * kStage;
};

template <typename T, int NSTAGE>
__global__ void __launch_bounds__(64 * EPB, kRingCtas) k_lap_elem_async(int nelem, int pin, const int32_t* __restrict__ econn,
                                                            const T* __restrict__ met, const DT<T> D,
                                                            const T* __restrict__ x, T* __restrict__ rel,
                                                            const double* __restrict__ scal) {
  using Ring = LapRing<T, NSTAGE>;
  if (scal && scal[S_DONE] != 0.0) return;
  const int ngroups = (nelem + EPB - 1) / EPB;
  if ((int)blockIdx.x >= ngroups) return;
  extern __shared__ __align__(16) unsigned char ring[];
  __shared__ T pl[EPB][FSTRIDE];
  __shared__ T fl[EPB][3][FSTRIDE];
  __shared__ T Ds[NP1][NP1];
  const int tid = threadIdx.x;
  const int es = tid >> 6, d = tid & 63;
  if (tid == 0) {  // constant indices: D stays in the parameter bank
#pragma unroll
    for (int a = 0; a < NP1; ++a)
#pragma unroll
      for (int b = 0; b < NP1; ++b) Ds[a][b] = D.d[a][b];
  }
  const int i = d & 3, j = (d >> 2) & 3, k = d >> 4, s = sidx(i, j, k);
  // copy the metric and connectivity of the t-th group of this CTA into its stage (all threads)
  auto issue = [&](int t) {
    const int g = blockIdx.x + t * gridDim.x;
    if (g < ngroups) {
      const int nval = min(EPB, nelem - g * EPB);
      unsigned char* st = ring + (t % NSTAGE) * Ring::kStage;
      const unsigned char* gm = reinterpret_cast<const unsigned char*>(met) + (size_t)g * Ring::kMetBytes;
      const int mchunks = nval * NMET * NN * (int)sizeof(T) / 16;
      for (int q = tid; q < mchunks; q += 64 * EPB) cp_async16(st + 16 * q, gm + 16 * (size_t)q);
      const unsigned char* gc = reinterpret_cast<const unsigned char*>(econn) + (size_t)g * EPB * NN * 4;
      const int cchunks = nval * NN * 4 / 16;
      for (int q = tid; q < cchunks; q += 64 * EPB) cp_async16(st + Ring::kMetBytes + 16 * q, gc + 16 * (size_t)q);
    }
    cp_async_commit();
  };
  auto node_of = [&](int t) {  // this thread's node in the t-th group (0 past the last element)
    const int e = (blockIdx.x + t * gridDim.x) * EPB + es;
    const int32_t* cs = reinterpret_cast<const int32_t*>(ring + (t % NSTAGE) * Ring::kStage + Ring::kMetBytes);
    return e < nelem ? cs[es * NN + d] : 0;
  };
  for (int t = 0; t < NSTAGE; ++t) issue(t);
  cp_async_wait<NSTAGE - 1>();  // group 0 landed
  __syncthreads();
  // this thread's D rows, read once for all its groups
  T Dx[NP1], Dy[NP1], Dz[NP1], DTx[NP1], DTy[NP1], DTz[NP1];
#pragma unroll
  for (int m = 0; m < NP1; ++m) {
    Dx[m] = Ds[i][m]; Dy[m] = Ds[j][m]; Dz[m] = Ds[k][m];
    DTx[m] = Ds[m][i]; DTy[m] = Ds[m][j]; DTz[m] = Ds[m][k];
  }
  int nd = node_of(0);
  T xv = nd == pin ? (T)0 : x[nd];
  for (int t = 0;; ++t) {
    const int g = blockIdx.x + t * gridDim.x;
    if (g >= ngroups) break;
    const T* ms = reinterpret_cast<const T*>(ring + (t % NSTAGE) * Ring::kStage) + es * NMET * NN + d;
    T M[NMET];
#pragma unroll
    for (int c = 0; c < NMET; ++c) M[c] = ms[c * NN];
    pl[es][s] = xv;
    cp_async_wait<NSTAGE - 2>();  // this thread's copies of group t + 1 landed
    __syncthreads();              // everyone's copies of group t + 1 and the p line visible
    T xv_n = (T)0;
    if (g + (int)gridDim.x < ngroups) {
      const int ndn = node_of(t + 1);
      xv_n = ndn == pin ? (T)0 : x[ndn];
    }
    const T* f = pl[es];
    T g0 = (T)0, g1 = (T)0, g2 = (T)0;
#pragma unroll
    for (int m = 0; m < NP1; ++m) {
      g0 += Dx[m] * f[sidx(m, j, k)];
      g1 += Dy[m] * f[sidx(i, m, k)];
      g2 += Dz[m] * f[sidx(i, j, m)];
    }
    fl[es][0][s] = M[0] * g0 + M[1] * g1 + M[2] * g2;
    fl[es][1][s] = M[1] * g0 + M[3] * g1 + M[4] * g2;
    fl[es][2][s] = M[2] * g0 + M[4] * g1 + M[5] * g2;
    __syncthreads();  // fluxes visible; stage t no longer read by anyone
    T acc = (T)0;
#pragma unroll
    for (int m = 0; m < NP1; ++m) {
      acc += DTx[m] * fl[es][0][sidx(m, j, k)];
      acc += DTy[m] * fl[es][1][sidx(i, m, k)];
      acc += DTz[m] * fl[es][2][sidx(i, j, m)];
    }
    const int e = g * EPB + es;
    if (e < nelem) rel[(size_t)e * NN + d] = acc;
    issue(t + NSTAGE);  // refill stage t
    xv = xv_n;
  }
  cp_async_wait<0>();  // no copy outlives the CTA
}


// single-block fixed-order reductions of the partials and the CG scalars
// mode 0: init  (part0 = ||r||^2 -> T1 and BNORM2, part1 = <r,z> -> Q1; done if ||b|| = 0)
// mode 1: alpha (part0 = <p,Ap> -> Q2, alpha = Q1/Q2)
// mode 2: update(part0 -> T1, part1 -> num, part2 -> Q1new; beta = num/Q1; Q1 = Q1new;
//                iteration += 1; done if ||r|| < tol ||b|| or the iteration limit is reached)
// mode 3: norm  (part0 -> T1)
// modes 1 and 2 do nothing once done
// Any block size up to 1024 threads; every thread of the block calls it.
__device__ __forceinline__ void cg_scalars_block(int nblk, const double* __restrict__ part, int stride, int mode,
                                                 double* scal) {
  __shared__ double sh[3][32];
  const int np = mode == 2 ? 3 : (mode == 0 ? 2 : 1);
  double v[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    for (int k = 0; k < np; ++k) v[k] += __ldcg(part + k * stride + b);
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
      if (t[0] == 0.0) scal[S_DONE] = 1.0;
    } else if (mode == 1) {
      scal[S_Q2] = t[0]; scal[S_ALPHA] = scal[S_Q1] / t[0];
    } else if (mode == 2) {
      scal[S_T1] = t[0]; scal[S_NUM] = t[1]; scal[S_BETA] = t[1] / scal[S_Q1]; scal[S_Q1] = t[2];
      scal[S_ITER] += 1.0;
      if (sqrt(t[0]) < scal[S_TOL] * sqrt(scal[S_BNORM2]) || scal[S_ITER] >= scal[S_MAXIT]) scal[S_DONE] = 1.0;
    } else {
      scal[S_T1] = t[0];
    }
  }
}

__global__ void __launch_bounds__(1024) k_cg_scalars(int nblk, const double* __restrict__ part, int stride,
                                                     int mode, double* scal) {
  if ((mode == 1 || mode == 2) && scal[S_DONE] != 0.0) return;
  cg_scalars_block(nblk, part, stride, mode, scal);
}

// After a kernel's block partials: the last block to finish reduces them (cg_scalars_block in
// the given mode) in a fixed order, so the CG scalars need no launch of their own.
__device__ __forceinline__ void last_block_scalars(unsigned int* counter, const double* part, int stride, int mode,
                                                   double* scal) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {
    __threadfence();
    cg_scalars_block(gridDim.x, part, stride, mode, scal);
    if (threadIdx.x == 0) *counter = 0u;
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

// y = sum of the element residuals of each node, y(pin) = 0; partials of <x, y>
template <typename T>
__global__ void __launch_bounds__(kBlock) k_lap_gather(int n, int pin, const int32_t* __restrict__ n2e_ptr,
                                                      const int32_t* __restrict__ n2e, const T* __restrict__ rel,
                                                      const T* __restrict__ x, T* __restrict__ y,
                                                      double* __restrict__ part, double* scal, unsigned int* counter) {
  if (scal && scal[S_DONE] != 0.0) return;
  double v[1] = {0.0};
  // grid-stride over the nodes: a grid of a few CTAs per SM keeps the partials (and the last
  // block's reduction of them) short
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T s = (T)0;
    int c = n2e_ptr[i];
    const int c1 = n2e_ptr[i + 1];
    // up to kGather independent loads in flight (a hexahedral vertex has 8 elements), summed in
    // ascending element order
    for (; c < c1; c += kGather) {
      int ix[kGather];
#pragma unroll
      for (int u = 0; u < kGather; ++u) ix[u] = c + u < c1 ? n2e[c + u] : -1;
      T v[kGather];
#pragma unroll
      for (int u = 0; u < kGather; ++u) v[u] = ix[u] >= 0 ? rel[ix[u]] : (T)0;
#pragma unroll
      for (int u = 0; u < kGather; ++u)
        if (ix[u] >= 0) s += v[u];
    }
    if (i == pin) s = (T)0;
    y[i] = s;
    v[0] += (double)x[i] * (double)s;
  }
  block_partials<1>(v, part, 0);
  // inside CG (counter given): <p,Ap> and alpha = <r,z>/<p,Ap> by the last block (mode 1)
  if (counter) last_block_scalars(counter, part, 0, 1, scal);
}

// r = b - Ax (ax may be null), z = r/M, p = z, x = 0 (if given); partials ||r||^2, <r,z>
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
__global__ void __launch_bounds__(kBlock) k_cg_update(int n, double* scal, TV* x, TV* r, TV* z,
                                                      const TV* __restrict__ p, const TV* __restrict__ q,
                                                      const TV* __restrict__ M, double* part, int stride,
                                                      unsigned int* counter) {
  if (scal[S_DONE] != 0.0) return;
  double v[3] = {0.0, 0.0, 0.0};
  const TV alpha = (TV)scal[S_ALPHA];
  auto one = [&](int i) {
    x[i] = x[i] + alpha * p[i];
    const TV ri = r[i] - alpha * q[i];
    const TV zo = z[i];
    const TV zi = ri / M[i];
    r[i] = ri; z[i] = zi;
    v[0] += (double)ri * (double)ri;
    v[1] += (double)ri * ((double)zi - (double)zo);
    v[2] += (double)ri * (double)zi;
  };
  const int gstride = gridDim.x * blockDim.x;
  int i0 = 0;
  if constexpr (sizeof(TV) == 4) {
    // FP32 sweeps: four nodes per thread through 16-byte accesses (a 4-byte load per node keeps
    // too few bytes in flight to reach the HBM rate)
    const int n4 = n >> 2;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n4; t += gstride) {
      float4 xv = reinterpret_cast<const float4*>(x)[t], pv = reinterpret_cast<const float4*>(p)[t];
      float4 rv = reinterpret_cast<const float4*>(r)[t], qv = reinterpret_cast<const float4*>(q)[t];
      float4 zv = reinterpret_cast<const float4*>(z)[t], mv = reinterpret_cast<const float4*>(M)[t];
      float xa[4] = {xv.x, xv.y, xv.z, xv.w}, pa[4] = {pv.x, pv.y, pv.z, pv.w}, ra[4] = {rv.x, rv.y, rv.z, rv.w};
      float qa[4] = {qv.x, qv.y, qv.z, qv.w}, za[4] = {zv.x, zv.y, zv.z, zv.w}, ma[4] = {mv.x, mv.y, mv.z, mv.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        xa[c] = xa[c] + alpha * pa[c];
        const float ri = ra[c] - alpha * qa[c];
        const float zo = za[c];
        const float zi = ri / ma[c];
        ra[c] = ri; za[c] = zi;
        v[0] += (double)ri * (double)ri;
        v[1] += (double)ri * ((double)zi - (double)zo);
        v[2] += (double)ri * (double)zi;
      }
      reinterpret_cast<float4*>(x)[t] = make_float4(xa[0], xa[1], xa[2], xa[3]);
      reinterpret_cast<float4*>(r)[t] = make_float4(ra[0], ra[1], ra[2], ra[3]);
      reinterpret_cast<float4*>(z)[t] = make_float4(za[0], za[1], za[2], za[3]);
    }
    i0 = n4 << 2;
  }
  for (int i = i0 + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gstride) one(i);
  block_partials<3>(v, part, stride);
  // beta, the iteration count and the stop test by the last block (mode 2)
  last_block_scalars(counter, part, stride, 2, scal);
}

template <typename TV>
__global__ void k_cg_pupdate(int n, const double* __restrict__ scal, const TV* __restrict__ z, TV* p) {
  if (scal[S_DONE] != 0.0) return;
  const TV beta = (TV)scal[S_BETA];
  if constexpr (sizeof(TV) == 4) {  // four nodes per thread, 16-byte accesses
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n4 = n >> 2;
    if (t < n4) {
      const float4 zv = reinterpret_cast<const float4*>(z)[t];
      float4 pv = reinterpret_cast<float4*>(p)[t];
      pv.x = zv.x + beta * pv.x; pv.y = zv.y + beta * pv.y; pv.z = zv.z + beta * pv.z; pv.w = zv.w + beta * pv.w;
      reinterpret_cast<float4*>(p)[t] = pv;
    }
    const int i = (n4 << 2) + t;
    if (t < (n & 3)) p[i] = z[i] + beta * p[i];
  } else {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = z[i] + beta * p[i];
  }
}

__global__ void k_cg_setup(double* scal, double tol, int max_iter) {
  scal[S_TOL] = tol;
  scal[S_MAXIT] = (double)max_iter;
  scal[S_ITER] = 0.0;
  scal[S_DONE] = 0.0;
}

// out = a - b with out[pin] = 0 (b may be null)
template <typename T>
__global__ void k_sub_pin(int n, int pin, const T* __restrict__ a, const T* __restrict__ b, T* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (i == pin) ? (T)0 : a[i] - (b ? b[i] : (T)0);
}
__global__ void k_cast32(int n, const double* __restrict__ s, float* __restrict__ d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = (float)s[i];
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

static int node_grid(int64_t n) { return (int)((n + kBlock - 1) / kBlock); }
// grid of the node kernels with reductions (grid-stride loops): a few CTAs per SM
static int red_grid(const SodPoisson* P) { return std::min(P->nblk, P->red_blocks); }

// y = K x with <x, y> block partials (part[0..node_grid(n))); scal != null skips once done and
// then also forms alpha (the CG iteration's scalars) in the gather's last block
template <typename T>
static int lap_apply(SodPoisson* P, const T* x, T* y, double* scal, cudaStream_t st) {
  const SodMesh* m = P->mesh;
  const int E = (int)P->nelem;
  const T* met;
  const DT<T>* D;
  if constexpr (sizeof(T) == 8) {
    met = P->met; D = &P->D64;
  } else {
    met = P->met32; D = &P->D32;
  }
  T* rel = static_cast<T*>(P->rel);
  const int ngroups = (E + EPB - 1) / EPB;
  const int pg = P->ring_grid[sizeof(T) == 8 ? 0 : 1];
  if (pg > 0) {
    k_lap_elem_async<T, NSTAGE><<<std::min(pg, ngroups), 64 * EPB, LapRing<T, NSTAGE>::kBytes, st>>>(
        E, P->pin, m->econn, met, *D, x, rel, scal);
  } else {
    k_lap_elem<T><<<ngroups, 64 * EPB, 0, st>>>(E, P->pin, m->econn, met, *D, x, rel, scal);
  }
  SOD_CHECK_LAUNCH();
  k_lap_gather<T><<<red_grid(P), kBlock, 0, st>>>((int)P->n, P->pin, m->n2e_ptr, m->n2e, rel, x, y, P->part, scal,
                                                  scal ? P->counter : nullptr);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

static int scalars(SodPoisson* P, int nblk, int mode, cudaStream_t st) {
  k_cg_scalars<<<1, 1024, 0, st>>>(nblk, P->part, P->nblk, mode, P->scal);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

static int read_scalars(SodPoisson* P, cudaStream_t st) {
  SOD_CUDA(cudaMemcpyAsync(P->hscal, P->scal, sizeof(double) * S_COUNT, cudaMemcpyDeviceToHost, st));
  return sync_stream(st);
}

template <typename TV>
struct CgVecs {
  const TV* M; TV *e, *r, *z, *p, *q;
};

// FP64: the solve's own vectors; FP32 sweep: its residual overwrites its right-hand side r32
template <typename TV> static CgVecs<TV> vecs(SodPoisson* P);
template <> CgVecs<double> vecs<double>(SodPoisson* P) { return {P->diag, P->x, P->r, P->z, P->p, P->q}; }
template <> CgVecs<float> vecs<float>(SodPoisson* P) { return {P->diag32, P->e32, P->r32, P->z32, P->p32, P->q32}; }

// one CG iteration after the init (matvec, alpha, update, beta + stop test, p update)
template <typename TV>
static int cg_iteration(SodPoisson* P, const CgVecs<TV>& v, cudaStream_t st) {
  const int n = (int)P->n;
  const int gb = node_grid(n);
  if (int rc = lap_apply<TV>(P, v.p, v.q, P->scal, st)) return rc;  // + alpha
  k_cg_update<TV><<<red_grid(P), kBlock, 0, st>>>(n, P->scal, v.e, v.r, v.z, v.p, v.q, v.M, P->part, P->nblk,
                                                  P->counter);  // + beta and the stop test
  SOD_CHECK_LAUNCH();
  k_cg_pupdate<TV><<<sizeof(TV) == 4 ? node_grid((n + 3) / 4) : gb, kBlock, 0, st>>>(n, P->scal, v.z, v.p);
  SOD_CHECK_LAUNCH();
  return SOD_OK;
}

// the graph of kBatch iterations for vector type TV (built once per handle)
template <typename TV>
static int batch_graph(SodPoisson* P, cudaGraphExec_t* exec, int* nkernels) {
  const int slot = sizeof(TV) == 8 ? 0 : 1;
  if (!P->batch[slot]) {
    const CgVecs<TV> v = vecs<TV>(P);
    cudaStream_t cap;
    SOD_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t graph;
    const int64_t before = g_launches.load();
    cudaError_t be = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int rc = SOD_OK;
    if (be == cudaSuccess)
      for (int t = 0; t < kBatch && rc == SOD_OK; ++t) rc = cg_iteration<TV>(P, v, cap);
    cudaError_t ce = be == cudaSuccess ? cudaStreamEndCapture(cap, &graph) : be;
    cudaStreamDestroy(cap);
    const int nk = (int)(g_launches.load() - before);
    g_launches.fetch_sub(nk);
    if (rc) return rc;
    if (ce != cudaSuccess) {
      set_error("CG graph capture failed: %s", cudaGetErrorString(ce));
      return SOD_ERR_CUDA;
    }
    cudaError_t ie = cudaGraphInstantiate(&P->batch[slot], graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      P->batch[slot] = nullptr;
      set_error("CG graph instantiate failed: %s", cudaGetErrorString(ie));
      return SOD_ERR_CUDA;
    }
    P->batch_kernels[slot] = nk;
  }
  *exec = P->batch[slot];
  *nkernels = P->batch_kernels[slot];
  return SOD_OK;
}

// Jacobi PCG on A e = rhs in the reference's iteration order; e starts at 0.  Stops when
// ||r|| < tol * ||r0|| or after max_iter; returns the iteration count and ||r|| / ||r0||.
template <typename TV>
static int pcg(SodPoisson* P, const CgVecs<TV>& v, const TV* rhs, int max_iter, double tol, cudaStream_t st,
               int* iters, double* rel) {
  const int n = (int)P->n;
  const int gb = node_grid(n);
  cudaGraphExec_t exec = nullptr;
  int nk = 0;
  if (int rc = batch_graph<TV>(P, &exec, &nk)) return rc;
  k_cg_setup<<<1, 1, 0, st>>>(P->scal, tol, max_iter);
  SOD_CHECK_LAUNCH();
  k_cg_init<TV><<<gb, kBlock, 0, st>>>(n, rhs, (const TV*)nullptr, v.M, v.r, v.z, v.p, v.e, P->part, P->nblk);
  SOD_CHECK_LAUNCH();
  if (int rc = scalars(P, gb, 0, st)) return rc;
  if (int rc = read_scalars(P, st)) return rc;
  const double auxB = std::sqrt(P->hscal[S_BNORM2]);
  if (auxB == 0.0) {
    *iters = 0;
    *rel = 0.0;
    return SOD_OK;
  }
  // bounded: every replay advances the counter by kBatch until the limit sets done
  for (int guard = 0; guard <= max_iter / kBatch + 1 && P->hscal[S_DONE] == 0.0; ++guard) {
    SOD_CUDA(cudaGraphLaunch(exec, st));
    g_launches.fetch_add(nk);
    if (int rc = read_scalars(P, st)) return rc;
  }
  *iters = (int)P->hscal[S_ITER];
  *rel = std::sqrt(P->hscal[S_T1]) / auxB;
  return SOD_OK;
}

extern "C" {

void sod_poisson_destroy(SodPoisson* P) {
  if (!P) return;
  for (cudaGraphExec_t& g : P->batch)
    if (g) cudaGraphExecDestroy(g);
  void* ptrs[] = {P->met, P->met32, P->diag, P->diag32, P->rel, P->x, P->r, P->p, P->q, P->z, P->b,
                  P->r32, P->p32, P->q32, P->z32, P->e32, P->part, P->scal, P->counter};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (P->hscal) cudaFreeHost(P->hscal);
  delete P;
}

int sod_poisson_create(SodMesh* m, SodPoisson** out) {
  SOD_ARG(m && out, "mesh/out null");
  *out = nullptr;
  if (m->has_slaves) {
    set_error("sod_poisson_create on a mesh with periodic slave rows (lpoin_w) is not supported");
    return SOD_ERR_UNSUPPORTED;
  }
  const int64_t N = m->npoin, E = m->nelem;
  SodPoisson* P = new SodPoisson();
  P->mesh = m; P->n = N; P->nelem = E; P->pin = 0;
  P->nblk = node_grid(N);
  for (int a = 0; a < NP1; ++a)
    for (int b = 0; b < NP1; ++b) {
      P->D64.d[a][b] = m->D.d[a][b];
      P->D32.d[a][b] = (float)m->D.d[a][b];
    }
  auto fail = [&](const char* what) {
    set_error("sod_poisson_create: %s failed", what);
    sod_poisson_destroy(P);
    return SOD_ERR_NOMEM;
  };
#define PALLOC(ptr, bytes) if (cudaMalloc(&(ptr), (bytes)) != cudaSuccess) return fail(#ptr)
  PALLOC(P->met, sizeof(double) * NMET * NN * E);
  PALLOC(P->met32, sizeof(float) * NMET * NN * E);
  PALLOC(P->rel, sizeof(double) * NN * E);
  PALLOC(P->diag, sizeof(double) * N);
  PALLOC(P->diag32, sizeof(float) * N);
  for (double** v : {&P->x, &P->r, &P->p, &P->q, &P->z, &P->b}) PALLOC(*v, sizeof(double) * N);
  for (float** v : {&P->r32, &P->p32, &P->q32, &P->z32, &P->e32}) PALLOC(*v, sizeof(float) * N);
  PALLOC(P->part, sizeof(double) * 3 * P->nblk);
  PALLOC(P->scal, sizeof(double) * S_COUNT);
  PALLOC(P->counter, sizeof(unsigned int));
  if (cudaMemset(P->counter, 0, sizeof(unsigned int)) != cudaSuccess) return fail("counter");
#undef PALLOC
  if (cudaMallocHost(&P->hscal, sizeof(double) * S_COUNT) != cudaSuccess) return fail("hscal");
  {
    int dev = 0, nsm = 0, b64 = 0, b32 = 0;
    SOD_CUDA(cudaGetDevice(&dev));
    SOD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    SOD_CUDA(cudaFuncSetAttribute(k_lap_elem_async<double, NSTAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  LapRing<double, NSTAGE>::kBytes));
    SOD_CUDA(cudaFuncSetAttribute(k_lap_elem_async<float, NSTAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  LapRing<float, NSTAGE>::kBytes));
    SOD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b64, k_lap_elem_async<double, NSTAGE>, 64 * EPB,
                                                           LapRing<double, NSTAGE>::kBytes));
    SOD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b32, k_lap_elem_async<float, NSTAGE>, 64 * EPB,
                                                           LapRing<float, NSTAGE>::kBytes));
    P->ring_grid[0] = nsm * b64;
    P->ring_grid[1] = nsm * b32;
    P->red_blocks = 8 * nsm;
  }
  k_metric<<<1184, 256>>>(E * NN, m->geo64, P->met, P->met32);
  k_diag<<<node_grid(N), kBlock>>>((int)N, m->n2e_ptr, m->n2e, m->geo64, m->D, P->diag, P->diag32);
  g_launches.fetch_add(2);
  cudaError_t err = cudaDeviceSynchronize();
  if (err == cudaSuccess) err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_error("Poisson setup: %s", cudaGetErrorString(err));
    sod_poisson_destroy(P);
    return SOD_ERR_CUDA;
  }
  *out = P;
  return SOD_OK;
}

int sod_poisson_apply(SodPoisson* P, const double* x, double* y, sod_stream_t stream) {
  SOD_ARG(P && x && y, "null argument");
  return lap_apply<double>(P, x, y, nullptr, (cudaStream_t)stream);
}

int sod_poisson_diag(SodPoisson* P, double* d, sod_stream_t stream) {
  SOD_ARG(P && d, "null argument");
  SOD_CUDA(cudaMemcpyAsync(d, P->diag, sizeof(double) * P->n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return SOD_OK;
}

int sod_conjgrad_pressure(SodPoisson* P, const double* Rp0, double* R, int max_iter, double tol, int mixed,
                          int* iters_out, double* rel_out, sod_stream_t stream) {
  SOD_ARG(P && Rp0 && R && max_iter > 0 && tol > 0.0, "conjgrad arguments");
  NvtxRange range("sod conjgrad pressure");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = (int)P->n;
  const int gb = node_grid(n);
  // b = R - A x0, b(pin) = 0 (mod_solver_incomp.f90:307-317)
  if (int rc = lap_apply<double>(P, Rp0, P->q, nullptr, st)) return rc;
  k_sub_pin<double><<<gb, kBlock, 0, st>>>(n, P->pin, R, P->q, P->b);
  SOD_CHECK_LAUNCH();
  int iters = 0;
  double rel = 0.0;
  if (!mixed) {
    int rc = pcg<double>(P, vecs<double>(P), P->b, max_iter, tol, st, &iters, &rel);
    if (rc) return rc;
  } else {
    // FP64 residual iterative refinement around FP32 Jacobi-PCG sweeps
    k_cg_init<double><<<gb, kBlock, 0, st>>>(n, P->b, (const double*)nullptr, P->diag, P->r, P->z, P->p, P->x,
                                             P->part, P->nblk);
    SOD_CHECK_LAUNCH();
    if (int rc = scalars(P, gb, 0, st)) return rc;
    if (int rc = read_scalars(P, st)) return rc;
    const double bnorm = std::sqrt(P->hscal[S_BNORM2]);
    rel = bnorm > 0.0 ? 1.0 : 0.0;
    for (int outer = 0; outer < 64 && rel >= tol && iters < max_iter; ++outer) {
      // each FP32 sweep is asked for the remaining reduction, but not below what FP32 resolves
      const double inner_tol = std::max(0.5 * tol / rel, 2e-6);
      k_cast32<<<gb, kBlock, 0, st>>>(n, P->r, P->r32);
      SOD_CHECK_LAUNCH();
      int it_in = 0;
      double rel_in = 0.0;
      int rc = pcg<float>(P, vecs<float>(P), P->r32, max_iter - iters, inner_tol, st, &it_in, &rel_in);
      if (rc) return rc;
      iters += it_in;
      k_axpy_cast<<<gb, kBlock, 0, st>>>(n, P->e32, P->x);
      SOD_CHECK_LAUNCH();
      // r = b - A x in FP64, ||r||^2
      if (int rc2 = lap_apply<double>(P, P->x, P->q, nullptr, st)) return rc2;
      k_cg_init<double><<<gb, kBlock, 0, st>>>(n, P->b, P->q, P->diag, P->r, P->z, P->p, (double*)nullptr, P->part,
                                               P->nblk);
      SOD_CHECK_LAUNCH();
      if (int rc3 = scalars(P, gb, 3, st)) return rc3;
      if (int rc4 = read_scalars(P, st)) return rc4;
      rel = std::sqrt(P->hscal[S_T1]) / bnorm;
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
