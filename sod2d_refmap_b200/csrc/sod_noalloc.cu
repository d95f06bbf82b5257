// Allocation-free full_convec_ijk for callers that cannot allocate device memory.
//
// Some host codes own every byte of device memory themselves: SOD2D's GPU build hands its
// arrays to the OpenACC runtime (present tables, managed memory) and a host application with
// a fixed device-memory pool may forbid any other cudaMalloc.  Such callers cannot create a
// SodMesh (which allocates geometry, gather map and step buffers).  This entry point takes the
// mesh and field arrays exactly as the reference routine does (device pointers in the
// reference layouts) and keeps its only scratch - the element residuals and the node->element
// gather map - in one file-scope static device array that every GPU loading this library holds
// until the process exits.
//
// Limits and behaviour:
//   * at most kMaxElem elements and kMaxPoin nodes per call; larger sizes return SOD_ERR_ARG;
//   * the scratch array is shared by every call on a device and keeps the last call's contents,
//     so each call clears the counters it needs first; calls that overlap on the GPU (different
//     streams or host threads at the same time) race on it and give wrong results;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//     that device current and caches it; make that first call before any stream capture;
//   * the call waits for its own stream to finish (within sod_set_wait_timeout's limit) so that it
//     can report out-of-range node ids; a wait is not allowed on a stream that is capturing, so on
//     such a stream the call returns SOD_ERR_UNSUPPORTED before it enqueues anything.
#include "sod_internal.cuh"
#include <mutex>

namespace sod {
namespace noalloc {

constexpr int kMaxElem = 4096;
constexpr int kMaxPoin = kMaxElem * NN;
constexpr int kNF = 5;  // mass, mom x3, energy
// byte offsets of the sub-arrays inside the scratch array
constexpr size_t kRelBytes = sizeof(double) * (size_t)kMaxElem * kNF * NN;
constexpr size_t kCntOff = kRelBytes;
constexpr size_t kPtrOff = kCntOff + sizeof(int32_t) * (size_t)(kMaxPoin + 256);
constexpr size_t kIdxOff = kPtrOff + sizeof(int32_t) * (size_t)(kMaxPoin + 256);
constexpr size_t kFlagOff = kIdxOff + sizeof(int32_t) * (size_t)kMaxElem * NN;
constexpr size_t kBytes = kFlagOff + 256;

static __device__ __align__(256) unsigned char g_scratch[kBytes];

struct View {
  double* rel;
  int32_t* cnt;
  int32_t* ptr;
  int32_t* idx;
  int32_t* flag;
};

__host__ __device__ inline View carve(unsigned char* base) {
  View v;
  v.rel = reinterpret_cast<double*>(base);
  v.cnt = reinterpret_cast<int32_t*>(base + kCntOff);
  v.ptr = reinterpret_cast<int32_t*>(base + kPtrOff);
  v.idx = reinterpret_cast<int32_t*>(base + kIdxOff);
  v.flag = reinterpret_cast<int32_t*>(base + kFlagOff);
  return v;
}

__global__ void k_clear(View v, int npoin) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= npoin; t += gridDim.x * blockDim.x) v.cnt[t] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *v.flag = 0;
}

__global__ void k_count(View v, int nelem, int npoin, int base, const int32_t* __restrict__ connec) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * NN) return;
  const int e = (int)(t % nelem), a = (int)(t / nelem);
  const int node = connec[e + (int64_t)nelem * a] - base;
  if (node < 0 || node >= npoin) {
    atomicOr(v.flag, 1);
    return;
  }
  atomicAdd(&v.cnt[node], 1);
}

// single-block exclusive scan cnt -> ptr, then cnt reset to 0 (fill cursors)
__global__ void __launch_bounds__(1024) k_scan(View v, int npoin) {
  __shared__ int32_t warp_tot[32];
  const int nthr = blockDim.x, tid = threadIdx.x;
  const int chunk = (npoin + nthr - 1) / nthr;
  const int beg = min(tid * chunk, npoin), end = min(beg + chunk, npoin);
  int32_t s = 0;
  for (int q = beg; q < end; ++q) s += v.cnt[q];
  // inclusive scan of the per-thread sums
  int32_t x = s;
  const int lane = tid & 31, w = tid >> 5;
  for (int o = 1; o < 32; o <<= 1) {
    int32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    int32_t t = (lane < (nthr >> 5)) ? warp_tot[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  int32_t run = x - s + (w > 0 ? warp_tot[w - 1] : 0);
  for (int q = beg; q < end; ++q) {
    v.ptr[q] = run;
    run += v.cnt[q];
    v.cnt[q] = 0;
  }
  if (tid == nthr - 1) v.ptr[npoin] = run;
}

__global__ void k_fill(View v, int nelem, int npoin, int base, const int32_t* __restrict__ connec) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * NN) return;
  const int e = (int)(t % nelem), a = (int)(t / nelem);
  const int node = connec[e + (int64_t)nelem * a] - base;
  if (node < 0 || node >= npoin) return;
  const int pos = atomicAdd(&v.cnt[node], 1);
  v.idx[v.ptr[node] + pos] = e * NN + a;
}

// ascending (element, local node) order inside each node's list: deterministic assembly order
__global__ void k_sort(View v, int npoin) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  const int b = v.ptr[n], e = v.ptr[n + 1];
  for (int q = b + 1; q < e; ++q) {
    const int32_t key = v.idx[q];
    int r = q - 1;
    while (r >= b && v.idx[r] > key) {
      v.idx[r + 1] = v.idx[r];
      --r;
    }
    v.idx[r + 1] = key;
  }
}

struct Args {
  int nelem, base;
  int64_t npoin;
  const int32_t* connec;     // (nelem,64)
  const double* He;          // (3,3,64,nelem)
  const double* gpvol;       // (1,64,nelem)
  const double* dlxigp_ip;   // (64,3,4)
  const int32_t *gI, *gJ, *gK;
  const double *u, *q, *rho, *pr, *E;
};

__device__ __forceinline__ int nat_of_sod(int s) { return s == 0 ? 0 : (s == 1 ? 3 : s - 1); }
__device__ __forceinline__ int sod_of_nat(int m) { return m == 0 ? 0 : (m == 3 ? 1 : m + 1); }

// full_convec_ijk (elem_convec.f90:241-435) on the reference layouts, one CTA per element,
// thread = local node a; element residuals go to the static scratch.
__global__ void __launch_bounds__(64) k_convec(View v, const Args x) {
  __shared__ double f[42][FSTRIDE];
  const int e = blockIdx.x, a = threadIdx.x;
  int si = x.gI[a] - x.base, sj = x.gJ[a] - x.base, sk = x.gK[a] - x.base;
  if ((unsigned)si > 3u || (unsigned)sj > 3u || (unsigned)sk > 3u) {  // flagged, clamped, no early exit
    atomicOr(v.flag, 2);
    si = sj = sk = 0;
  }
  const int i = nat_of_sod(si), j = nat_of_sod(sj), k = nat_of_sod(sk);
  const int s = sidx(i, j, k);
  int n = x.connec[e + (int64_t)x.nelem * a] - x.base;
  n = (n < 0 || n >= x.npoin) ? 0 : n;  // out-of-range ids were flagged by k_count
  const int64_t N = x.npoin;
  double u[3], q[3];
  for (int c = 0; c < 3; ++c) { u[c] = x.u[n + N * c]; q[c] = x.q[n + N * c]; }
  const double rho = x.rho[n], El = x.E[n], pr = x.pr[n];
  double kl = 0.0;
  for (int c = 0; c < 3; ++c) kl = kl + u[c] * u[c] * 0.5;
  f[0][s] = rho; f[1][s] = pr; f[2][s] = El; f[3][s] = rho * El; f[4][s] = kl; f[5][s] = rho * kl;
  for (int c = 0; c < 3; ++c) {
    f[6 + c][s] = u[c]; f[9 + c][s] = q[c];
    f[12 + c][s] = rho * El * u[c]; f[15 + c][s] = El * u[c];
    f[18 + c][s] = rho * kl * u[c]; f[21 + c][s] = kl * u[c];
    for (int c2 = 0; c2 < 3; ++c2) { f[24 + 3 * c + c2][s] = q[c] * u[c2]; f[33 + 3 * c + c2][s] = u[c] * u[c2]; }
  }
  // this gauss point's 1-D derivative rows, indexed by natural basis position
  double Dx[NP1], Dy[NP1], Dz[NP1];
  for (int m = 0; m < NP1; ++m) {
    const int ii = sod_of_nat(m);
    Dx[m] = x.dlxigp_ip[a + NN * (0 + 3 * ii)];
    Dy[m] = x.dlxigp_ip[a + NN * (1 + 3 * ii)];
    Dz[m] = x.dlxigp_ip[a + NN * (2 + 3 * ii)];
  }
  double H[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) H[3 * r + c] = x.He[r + 3 * (c + 3 * ((int64_t)a + NN * e))];
  const double gpv = x.gpvol[a + (int64_t)NN * e];
  __syncthreads();
  auto grad = [&](int fi, double* o) {
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int m = 0; m < NP1; ++m) {
      gx += Dx[m] * f[fi][sidx(m, j, k)];
      gy += Dy[m] * f[fi][sidx(i, m, k)];
      gz += Dz[m] * f[fi][sidx(i, j, m)];
    }
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
  double Re = 0.25 * (divFe + El * divQ + rho * El * divU + rho * divFue) +
              0.25 * (divFk + kl * divQ + rho * kl * divU + rho * divFuk);
  double Rmo[3];
  for (int c = 0; c < 3; ++c) {
    Rmo[c] = 0.25 * (divF[c] + u[c] * divQ + q[c] * divU + rho * divFuu[c]) + gP[c];
    Rm = Rm + 0.5 * (u[c] * gRho[c]);
    Re = Re + 0.25 * (q[c] * gE[c] + u[c] * gRE[c] + El * u[c] * gRho[c]) +
         0.25 * (q[c] * gk[c] + u[c] * gRk[c] + kl * u[c] * gRho[c]);
    for (int c2 = 0; c2 < 3; ++c2) Rmo[c] = Rmo[c] + 0.25 * (u[c] * u[c2] * gRho[c2] + q[c2] * gU[c][c2] + u[c2] * gQ[c][c2]);
  }
  double* out = v.rel + (int64_t)e * kNF * NN + a;
  out[0] = gpv * Rm; out[NN] = gpv * Rmo[0]; out[2 * NN] = gpv * Rmo[1]; out[3 * NN] = gpv * Rmo[2];
  out[4 * NN] = gpv * Re;
}

__global__ void k_gather(View v, int npoin, double* Rmass, double* Rmom, double* Rener) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  double r[kNF] = {0, 0, 0, 0, 0};
  for (int c = v.ptr[n]; c < v.ptr[n + 1]; ++c) {
    const int pk = v.idx[c];
    const double* src = v.rel + (int64_t)(pk >> 6) * kNF * NN + (pk & 63);
    for (int fld = 0; fld < kNF; ++fld) r[fld] += src[fld * NN];
  }
  Rmass[n] = r[0];
  Rmom[n] = r[1];
  Rmom[n + (int64_t)npoin] = r[2];
  Rmom[n + 2 * (int64_t)npoin] = r[3];
  Rener[n] = r[4];
}

static std::mutex g_mu;
static unsigned char* g_addr[128] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
static int scratch_address(unsigned char** out) {
  int dev = 0;
  SOD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) {
    set_error("device ordinal %d out of range for the allocation-free scratch table", dev);
    return SOD_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) {
      set_error("cudaGetSymbolAddress of the allocation-free scratch failed: %s", cudaGetErrorString(e));
      return SOD_ERR_CUDA;
    }
    g_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_addr[dev];
  return SOD_OK;
}

}  // namespace noalloc
}  // namespace sod

using namespace sod;

extern "C" int sod_full_convec_ijk_noalloc(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                                           const double* He, const double* gpvol, const double* dlxigp_ip,
                                           const int32_t* gmshAtoI, const int32_t* gmshAtoJ, const int32_t* gmshAtoK,
                                           const double* u, const double* q, const double* rho, const double* pr,
                                           const double* E, double* Rmass, double* Rmom, double* Rener,
                                           sod_stream_t stream) {
  using namespace sod::noalloc;
  SOD_ARG(connec && He && gpvol && dlxigp_ip && gmshAtoI && gmshAtoJ && gmshAtoK && u && q && rho && pr && E &&
              Rmass && Rmom && Rener,
          "null argument");
  SOD_ARG(index_base == 0 || index_base == 1, "index_base must be 0 or 1");
  if (nelem <= 0 || npoin <= 0 || nelem > kMaxElem || npoin > kMaxPoin) {
    set_error("invalid argument: sod_full_convec_ijk_noalloc handles 1..%d elements and 1..%d nodes "
              "(got nelem=%d, npoin=%d); use sod_full_convec_ijk for larger meshes",
              kMaxElem, kMaxPoin, nelem, npoin);
    return SOD_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  SOD_CUDA(cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    set_error("sod_full_convec_ijk_noalloc waits for its stream to report bad node ids, which a capturing "
              "stream does not allow");
    return SOD_ERR_UNSUPPORTED;
  }
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  View v = carve(base);
  const int64_t nen = (int64_t)nelem * NN;
  const int gb = (int)((nen + 255) / 256);
  k_clear<<<64, 256, 0, st>>>(v, npoin);
  SOD_CHECK_LAUNCH();
  k_count<<<gb, 256, 0, st>>>(v, nelem, npoin, index_base, connec);
  SOD_CHECK_LAUNCH();
  k_scan<<<1, 1024, 0, st>>>(v, npoin);
  SOD_CHECK_LAUNCH();
  k_fill<<<gb, 256, 0, st>>>(v, nelem, npoin, index_base, connec);
  SOD_CHECK_LAUNCH();
  k_sort<<<(npoin + 255) / 256, 256, 0, st>>>(v, npoin);
  SOD_CHECK_LAUNCH();
  Args x;
  x.nelem = nelem; x.base = index_base; x.npoin = npoin; x.connec = connec; x.He = He; x.gpvol = gpvol;
  x.dlxigp_ip = dlxigp_ip; x.gI = gmshAtoI; x.gJ = gmshAtoJ; x.gK = gmshAtoK;
  x.u = u; x.q = q; x.rho = rho; x.pr = pr; x.E = E;
  k_convec<<<nelem, 64, 0, st>>>(v, x);
  SOD_CHECK_LAUNCH();
  k_gather<<<(npoin + 255) / 256, 256, 0, st>>>(v, npoin, Rmass, Rmom, Rener);
  SOD_CHECK_LAUNCH();
  // bounded wait (sod_set_wait_timeout), then a plain read of the flag once the work is done
  if ((rc = sync_stream(st))) return rc;
  int32_t hflag = 0;
  SOD_CUDA(cudaMemcpy(&hflag, v.flag, sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (hflag & 1) {
    set_error("invalid argument: connec holds node ids outside [%d, %d)", index_base, index_base + npoin);
    return SOD_ERR_ARG;
  }
  if (hflag & 2) {
    set_error("invalid argument: gmshAtoI/J/K hold values outside [%d, %d]", index_base, index_base + 3);
    return SOD_ERR_ARG;
  }
  return SOD_OK;
}
