// Device bodies of the node gather / RK stage update (KG) and of the entropy viscosity + CFL dt
// (KV), shared by their stand-alone kernels (sod_rhs.cu) and by the persistent one-launch-per-
// stage kernels (sod_rhs.cu for FP64, sod_rhs_mixed.cu for the mixed path).  Not part of the ABI.
#pragma once
#include "sod_internal.cuh"
#include <cooperative_groups.h>

namespace sod {

// ---------------------------------------------------------------------------------------------
// KG: ordered CSR gather of the element residuals, /Ml, RK accumulate and next stage state.
// STAGE 0 = plain RHS (gather + /Ml into output arrays).  STAGE 4 = final update + EOS.
// ---------------------------------------------------------------------------------------------
struct GatherArgs {
  int npoin;
  int nwork;                      // working nodes (rows with elements): the entropy mean's count
  int slaves;                     // 1 when some rows have no elements (periodic slave rows)
  const int32_t* __restrict__ ptr;
  const int32_t* __restrict__ idx;
  const void* rel;
  const double* __restrict__ Ml;
  const double* __restrict__ dt;  // device scalar, or per-member array when node_member is set
  const int32_t* __restrict__ node_member;
  int member_reduce;              // stage 4: eta sums done by the per-member kernel instead
  double a_next, b_cur;
  // state (level pos=2) columns
  double* y[5];
  double* ys;    // stage state 5*N
  void* rsum;    // RK accumulators 6*N, stored at the residual precision R: the mixed path's
                 // hold sums of FP32 element residuals, so FP32 storage loses nothing they carry
  // stage-0 outputs
  double* out[6];
  // stage-4 EOS outputs
  double *u0, *u1, *u2, *pr, *Tem, *e_int, *eta, *csound, *machno, *mu_fluid, *Reta;
  const double* mu_factor;
  double gamma, Rgas;
  double* red;              // partials [3*nblocks]
  unsigned int* counter;
  unsigned int* nonfinite;  // raised by stage 4 on a NaN/Inf in the new rho, q, E
  double* scal;             // [0] eta mean, [1] eta norm
  int normalise;
  const double* src;        // momentum source term (npoin,3) or null
  const double* wm;         // wall-model momentum terms (npoin,3) or null
};

// sh: 3 doubles per warp of the block
__device__ __forceinline__ void block_reduce3(double& s, double& mx, double& mn, double* sh) {
  // warp reduce then smem
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sh[3 * w] = s; sh[3 * w + 1] = mx; sh[3 * w + 2] = mn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    s = sh[0]; mx = sh[1]; mn = sh[2];
    for (int q = 1; q < nw; ++q) { s += sh[3 * q]; mx = fmax(mx, sh[3 * q + 1]); mn = fmin(mn, sh[3 * q + 2]); }
  }
}

// One node of KG (n may be past npoin: nothing happens).  Returns whether the node is a working
// node that was updated; at STAGE 4 eta_n receives its new entropy for the normalisation sums.
template <typename R, int STAGE>
__device__ __forceinline__ bool gather_rk_node(const GatherArgs& a, int n, double& eta_n) {
  // a row without elements is a periodic slave (not in lpoin_w): rk_4_main's node loops
  // (time_integ.f90:267-285,445-471) and the lumped solve (mod_solver.f90:23-58) skip it, its
  // residual stays zero and its state untouched; only sutherland_viscosity, which runs over all
  // npoin (time_integ.f90:483-487), re-evaluates its mu_fluid from its own Tem
  const bool inrange = n < a.npoin;
  const bool act = inrange && (!a.slaves || a.ptr[n + 1] > a.ptr[n]);
  if (inrange && !act) {
    if constexpr (STAGE == 0) {
#pragma unroll
      for (int f = 0; f < 6; ++f)
        if (a.out[f]) a.out[f][n] = 0.0;
    } else if constexpr (STAGE == 4) {
      const double T = a.Tem[n];
      a.mu_fluid[n] = a.mu_factor[n] * kSuthC1 * (T * sqrt(T)) / (T + kSuthS);
    }
  }
  if (act) {
    const R* rel = reinterpret_cast<const R*>(a.rel);
    R* rsum = reinterpret_cast<R*>(a.rsum);
    const size_t N = (size_t)a.npoin;
    // node data independent of the gather, loaded first so their latency overlaps it
    double yv[5];
    R rsv[6];      // the accumulators at their stored precision (widened exactly where used)
    if constexpr (STAGE >= 1) {
#pragma unroll
      for (int f = 0; f < 5; ++f) yv[f] = a.y[f][n];
#pragma unroll
      for (int f = 0; f < 6; ++f) rsv[f] = STAGE == 1 ? (R)0 : rsum[f * N + n];
    }
    const double ml = a.Ml[n];
    double r[6] = {0, 0, 0, 0, 0, 0};
    const int beg = a.ptr[n], end = a.ptr[n + 1];
    int c = beg;
    if constexpr (sizeof(R) == 4) {
      // groups of up to 4 contributions (a partial group's missing ones predicated off): all
      // loads of a group issued before its (ascending, fixed-order) sums, so a node with 1-4
      // contributions waits on one chain of index -> residual loads
      for (; c < end; c += 4) {
        R v[4][6];
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (c + q < end) load_res6<R>(rel, (size_t)a.idx[c + q], v[q]);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (c + q < end) {
#pragma unroll
            for (int f = 0; f < 6; ++f) r[f] += (double)v[q][f];
          }
      }
    } else {
      // FP64 residual rows: full groups of 4, then one at a time (a predicated group's 24
      // doubles do not fit the register budget)
      for (; c + 4 <= end; c += 4) {
        R v[4][6];
#pragma unroll
        for (int q = 0; q < 4; ++q) load_res6<R>(rel, (size_t)a.idx[c + q], v[q]);
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int f = 0; f < 6; ++f) r[f] += (double)v[q][f];
      }
      for (; c < end; ++c) {
        R v[6];
        load_res6<R>(rel, (size_t)a.idx[c], v);
#pragma unroll
        for (int f = 0; f < 6; ++f) r[f] += (double)v[f];
      }
    }
    if (a.src) {
      // mom_source_const_vect (elem_source.f90:20-55): - sum_e gpvol s = - Ml s on the momentum
#pragma unroll
      for (int d = 0; d < 3; ++d) r[1 + d] -= ml * a.src[d * N + n];
    }
    if (a.wm) {
      // wall model: the modelled shear added to Rdiff_mom (time_integ.f90:334-357)
#pragma unroll
      for (int d = 0; d < 3; ++d) r[1 + d] += a.wm[d * N + n];
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) r[f] = r[f] / ml;
    if constexpr (STAGE == 0) {
#pragma unroll
      for (int f = 0; f < 6; ++f)
        if (a.out[f]) a.out[f][n] = r[f];
    } else {
      const double dt = a.node_member ? a.dt[a.node_member[n]] : *a.dt;
      double rs[6];
#pragma unroll
      for (int f = 0; f < 6; ++f) rs[f] = (double)rsv[f] + a.b_cur * r[f];
      if constexpr (STAGE < 4) {
#pragma unroll
        for (int f = 0; f < 6; ++f) rsum[f * N + n] = (R)rs[f];
        const double da = dt * a.a_next;
#pragma unroll
        for (int f = 0; f < 5; ++f) a.ys[f * N + n] = yv[f] - da * r[f];
      } else {
        // RK update (time_integ.f90:417-426) and EOS at the new level (:445-463)
        double y[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          y[f] = yv[f] - dt * rs[f];
          a.y[f][n] = y[f];
        }
        if (!(isfinite(y[0]) && isfinite(y[1]) && isfinite(y[2]) && isfinite(y[3]) && isfinite(y[4])))
          atomicOr(a.nonfinite, 1u);
        // one reciprocal of rho serves the divisions by rho, and log(p / rho^gamma) is formed
        // as log p - gamma log rho (no pow): the same quantities to the last bits or so
        const double g = a.gamma;
        const double rho = y[0];
        const double irho = 1.0 / rho;
        const double u0 = y[1] * irho, u1 = y[2] * irho, u2 = y[3] * irho;
        double umag = u0 * u0 + u1 * u1 + u2 * u2;
        const double ei = y[4] * irho - 0.5 * umag;
        const double pr = rho * (g - 1.0) * ei;
        const double cs = sqrt(g * pr * irho);
        umag = sqrt(umag);
        const double T = pr * irho / a.Rgas;
        const double eta = (rho / (g - 1.0)) * (log(pr) - g * log(rho));
        a.u0[n] = u0; a.u1[n] = u1; a.u2[n] = u2;
        a.e_int[n] = ei; a.pr[n] = pr; a.csound[n] = cs; a.machno[n] = umag / cs;
        a.Tem[n] = T; a.eta[n] = eta;
        a.mu_fluid[n] = a.mu_factor[n] * kSuthC1 * (T * sqrt(T)) / (T + kSuthS);
        if (a.Reta) a.Reta[n] = -rs[5];
        eta_n = eta;
      }
    }
  }
  return act;
}

// The STAGE 4 entropy normalisation (mod_entropy_viscosity.f90:43-66) over the grid: block sums
// of (eta, max, min) into red[blockIdx.x], then the last block to finish reduces them in a fixed
// order into scal[0] (mean) and scal[1] (max deviation).  Every thread of the block calls it.
// sh: 3 doubles per warp.
__device__ __forceinline__ void gather_eta_reduce(const GatherArgs& a, double s, double mx, double mn, double* sh) {
  __shared__ bool last;
  // entropy normalisation (mod_entropy_viscosity.f90:43-66): sum, max, min of eta
  block_reduce3(s, mx, mn, sh);
  if (threadIdx.x == 0) {
    a.red[3 * blockIdx.x] = s;
    a.red[3 * blockIdx.x + 1] = mx;
    a.red[3 * blockIdx.x + 2] = mn;
    __threadfence();
    unsigned int done = atomicAdd(a.counter, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    // fixed-order final reduction by the last block (deterministic)
    double ts = 0.0, tmx = -1e300, tmn = 1e300;
#pragma unroll 4
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
      ts += __ldcg(a.red + 3 * b);
      tmx = fmax(tmx, __ldcg(a.red + 3 * b + 1));
      tmn = fmin(tmn, __ldcg(a.red + 3 * b + 2));
    }
    __syncthreads();
    block_reduce3(ts, tmx, tmn, sh);
    if (threadIdx.x == 0) {
      if (a.normalise) {
        const double mean = ts / (double)a.nwork;
        a.scal[0] = mean;
        a.scal[1] = fmax(tmx - mean, mean - tmn);
      } else {
        a.scal[0] = 0.0;
        a.scal[1] = 1.0;
      }
      *a.counter = 0u;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// KV: smart_visc_spectral (mod_entropy_viscosity.f90:68-121) per element with the convertIJK
// filter (mod_filters.f90:42-51), fused with the per-element CFL limits of adapt_dt_cfl
// (mod_time_ops.f90:31-56) and a deterministic min reduction to the next dt.
// ---------------------------------------------------------------------------------------------
struct ViscArgs {
  int nelem;
  const int32_t* __restrict__ econn;
  const double* __restrict__ Reta;
  const double* __restrict__ rho;
  const double* __restrict__ u0;
  const double* __restrict__ u1;
  const double* __restrict__ u2;
  const double* __restrict__ csound;
  const double* __restrict__ Tem;
  const double* __restrict__ mu_fluid;
  const double* __restrict__ musgs;  // [e][64] or null
  const double* __restrict__ helem_l;
  const double* __restrict__ helem;
  const double* __restrict__ jratio;
  const double* __restrict__ scal;   // [0] mean, [1] norm
  double* mue;                       // out FP64 [e][64]
  float* mue32;                      // optional FP32 copy
  double* dt_bits;                   // scratch scalar(s) receiving the min dt (bits, pre-set large)
  const int32_t* __restrict__ elem_member;  // ensemble: member of each element (null = one mesh)
  const double* __restrict__ member_scal;   // ensemble: [member][2] eta mean, norm
  double* dt_out;                    // device scalar (may be null)
  DevParams prm;
};

__device__ __forceinline__ int nb_filter(int x) {
  // natural index of convertIJK(x+1): x=-1 -> 1, 0..3 -> x, 4 -> 1 (reference quirk)
  return (x < 0) ? 1 : ((x > 3) ? 1 : x);
}

constexpr int KV_WARPS = 8;   // elements (one warp each) per block of the stand-alone KV kernel

// Exact maximum of a double over the warp with two 32-bit integer reductions instead of ten
// shuffles: the bit pattern is mapped to an unsigned key of the same order (sign bit flipped for
// non-negative values, all bits for negative ones), the high words are reduced, then the low
// words of the lanes that hold the maximal high word.  Equal to fmax over the lanes for every
// non-NaN input.  A NaN with a clear sign bit (the form the GPU's arithmetic produces) wins
// here, where fmax would drop it; the step's non-finite flag reports such states anyway.
__device__ __forceinline__ double warp_max_f64(double v) {
  const unsigned hi = (unsigned)__double2hiint(v), lo = (unsigned)__double2loint(v);
  const unsigned neg = (unsigned)((int)hi >> 31);
  const unsigned kh = hi ^ (neg | 0x80000000u), kl = lo ^ neg;
  const unsigned mh = __reduce_max_sync(0xffffffffu, kh);
  const unsigned ml = __reduce_max_sync(0xffffffffu, kh == mh ? kl : 0u);
  const unsigned back = (mh & 0x80000000u) ? 0u : 0xffffffffu;   // key of a negative maximum
  return __hiloint2double((int)(mh ^ (back | 0x80000000u)), (int)(ml ^ back));
}

// The larger of two doubles in the key order of warp_max_f64, so that the maximum over a lane's
// two nodes and then over the warp is the one warp_max_f64 gives over all 64 values.
__device__ __forceinline__ double max2_f64(double x, double y) {
  const long long bx = __double_as_longlong(x), by = __double_as_longlong(y);
  const unsigned long long kx = (unsigned long long)bx ^ ((unsigned long long)(bx >> 63) | 0x8000000000000000ull);
  const unsigned long long ky = (unsigned long long)by ^ ((unsigned long long)(by >> 63) | 0x8000000000000000ull);
  return kx >= ky ? x : y;
}

// One element per warp: lane l holds the element nodes d = l and d = l + 32 (k-planes 0-1 and
// 2-3 of d = i + 4j + 16k).  The element maxima are warp reductions, so the element scalars
// (shock sensor, cap, CFL limits) come out warp-uniform on every lane with no shared memory and
// no block barrier; only the filter goes through sm (KV_WSMEM doubles: ml[64], fl[64]) with warp
// barriers.  Returns the bit pattern of the element's dt limit (every lane); with elem_atomic
// lane 0 also takes the atomic minimum into the element's dt slot itself.
constexpr int KV_WSMEM = 2 * NN;
__device__ __forceinline__ unsigned long long visc_dt_warp(const ViscArgs& a, int e, int l, double* sm,
                                                           bool elem_atomic) {
  double* ml = sm;
  double* fl = sm + NN;
  const size_t eb = (size_t)e * NN;
  int nd[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) nd[h] = a.econn[eb + l + 32 * h];
  // element scalars, warp-uniform loads issued with the node gathers
  const double he = a.helem[e];
  const double jr = a.jratio[e];
  const int mem = a.elem_member ? a.elem_member[e] : 0;
  const double norm = a.elem_member ? a.member_scal[2 * mem + 1] : a.scal[1];
  // every node input of both nodes before any arithmetic
  double rho[2], u0[2], u1[2], u2[2], cs[2], T[2], reta[2], hl[2], msg[2], muf[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int n = nd[h];
    rho[h] = a.rho[n]; u0[h] = a.u0[n]; u1[h] = a.u1[n]; u2[h] = a.u2[n];
    cs[h] = a.csound[n]; T[h] = a.Tem[n]; reta[h] = a.Reta[n]; muf[h] = a.mu_fluid[n];
    hl[h] = a.helem_l[eb + l + 32 * h];
    msg[h] = a.musgs ? a.musgs[eb + l + 32 * h] : 0.0;
  }
  double vmag[2], beta[2], L3n[2], mun[2], r1[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    vmag[h] = sqrt(u0[h] * u0[h] + u1[h] * u1[h] + u2[h] * u2[h]);
    // betae node term (mod_entropy_viscosity.f90:90-95)
    beta[h] = (rho[h] * he) * (a.prm.cmax / (double)P) * (vmag[h] + sqrt(a.prm.Rgas * a.prm.gamma * T[h]));
    // CFL node terms (mod_time_ops.f90:36-50)
    const double umax = fmax(fmax(fabs(u0[h]), fabs(u1[h])), fabs(u2[h]));
    L3n[h] = umax + cs[h];
    mun[h] = (rho[h] * msg[h] + muf[h]) / rho[h];
    r1[h] = rho[h] * fabs(reta[h]);
  }
  // element maxima over the 64 nodes
  const double mV = warp_max_f64(max2_f64(vmag[0], vmag[1]));
  const double mC = warp_max_f64(max2_f64(cs[0], cs[1]));
  const double mB = warp_max_f64(max2_f64(beta[0], beta[1]));
  const double L3 = warp_max_f64(max2_f64(L3n[0], L3n[1]));
  const double maxMU = warp_max_f64(max2_f64(mun[0], mun[1]));
  // shock sensor and cap (mod_entropy_viscosity.f90:81-84); M**15 as an integer power like the
  // reference
  const double M = mV / mC;
  const double M2 = M * M, M4 = M2 * M2, M8 = M4 * M4;
  const double M15 = M8 * M4 * M2 * M;
  const double ceM = fmax(tanh(M15 * 3.141592653589793), a.prm.ce);
  const double ced = fmax(fmax(1.0 - jr, a.prm.ce), ceM);
  const double hh = he / (double)(2.0 * P + 1);
  const double limit = fmin(a.prm.cfl_conv * hh / L3, a.prm.cfl_diff * (hh * hh) / maxMU);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const double R1 = (norm > 0.0) ? r1[h] / norm : 0.0;
    const double Ve = ced * R1 * hl[h] * hl[h];
    ml[l + 32 * h] = a.prm.cglob * fmin(Ve, mB);
  }
  __syncwarp();
  // 3x3x3 filter with weights (1/4,1/2,1/4) through convertIJK (mod_entropy_viscosity.f90:102-120):
  // the weights and the index map are separable, so it runs as three 3-point passes (xi, eta,
  // zeta) through shared memory, 9 reads per node instead of 27
  const int i = l & 3, j = (l >> 2) & 3;
  const int ix[3] = {nb_filter(i - 1), i, nb_filter(i + 1)};
  const int jx[3] = {nb_filter(j - 1), j, nb_filter(j + 1)};
  const double w[3] = {0.25, 0.5, 0.25};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = (l >> 4) + 2 * h, d = l + 32 * h;
    fl[d] = w[0] * ml[ix[0] + 4 * j + 16 * k] + w[1] * ml[d] + w[2] * ml[ix[2] + 4 * j + 16 * k];
  }
  __syncwarp();
  // ml's first-pass reads all happened before the barrier above, so it takes the second pass
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = (l >> 4) + 2 * h, d = l + 32 * h;
    ml[d] = w[0] * fl[i + 4 * jx[0] + 16 * k] + w[1] * fl[d] + w[2] * fl[i + 4 * jx[2] + 16 * k];
  }
  __syncwarp();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = (l >> 4) + 2 * h, d = l + 32 * h;
    const int kx[3] = {nb_filter(k - 1), k, nb_filter(k + 1)};
    const double acc = w[0] * ml[i + 4 * j + 16 * kx[0]] + w[1] * ml[d] + w[2] * ml[i + 4 * j + 16 * kx[2]];
    a.mue[eb + d] = acc;
    if (a.mue32) a.mue32[eb + d] = (float)acc;
  }
  __syncwarp();   // the filter's reads are done before a caller reuses sm
  // next dt: order-independent min over elements on the bit pattern of a positive double
  const unsigned long long bits = (unsigned long long)__double_as_longlong(limit);
  if (elem_atomic && a.dt_out && l == 0) atomicMin(reinterpret_cast<unsigned long long*>(a.dt_bits) + mem, bits);
  return bits;
}

// ---------------------------------------------------------------------------------------------
// One RK stage in one cooperative launch: the element RHS over element tiles, a grid barrier,
// the node gather / stage update over all nodes (grid-stride), and at stage 4 a grid barrier,
// the per-member entropy statistics of an ensemble, another barrier and the entropy viscosity
// + CFL dt over element tiles.  The element-RHS phase is the caller's (it differs by precision).
// ---------------------------------------------------------------------------------------------
struct StageArgs {
  RhsArgs r;
  GatherArgs g;
  ViscArgs v;
  int stage;                           // 1..4
  int nmember;                         // ensemble members (0: one mesh)
  const int32_t* __restrict__ member_node_off;  // [nmember+1]
  double* member_scal;                 // [nmember][2]
};

template <typename R, int STAGE>
__device__ __forceinline__ void persist_gather_loop(const GatherArgs& g, double& s, double& mx, double& mn) {
  // two nodes per trip: the persistent grid holds fewer threads than the stand-alone gather, so
  // each thread keeps two independent gathers in flight
  const int stride = gridDim.x * blockDim.x;
  for (int n0 = blockIdx.x * blockDim.x + threadIdx.x; n0 < g.npoin; n0 += 2 * stride) {
    double e0 = 0.0, e1 = 0.0;
    const bool a0 = gather_rk_node<R, STAGE>(g, n0, e0);
    const bool a1 = gather_rk_node<R, STAGE>(g, n0 + stride, e1);
    if (STAGE == 4) {
      if (a0) { s += e0; mx = fmax(mx, e0); mn = fmin(mn, e0); }
      if (a1) { s += e1; mx = fmax(mx, e1); mn = fmin(mn, e1); }
    }
  }
}

// Everything of a stage after its element-RHS phase; EPB elements (64 threads each) per block.
template <typename R, int EPB>
__device__ __forceinline__ void persist_stage_tail(const StageArgs& p, unsigned char* smem_raw) {
  __shared__ double sh[3 * 32];
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  grid.sync();  // every element residual of the stage is written
  double s = 0.0, mx = -1e300, mn = 1e300;
  switch (p.stage) {
    case 1: persist_gather_loop<R, 1>(p.g, s, mx, mn); break;
    case 2: persist_gather_loop<R, 2>(p.g, s, mx, mn); break;
    case 3: persist_gather_loop<R, 3>(p.g, s, mx, mn); break;
    default: persist_gather_loop<R, 4>(p.g, s, mx, mn); break;
  }
  if (p.stage != 4) return;
  if (p.nmember == 0) {
    gather_eta_reduce(p.g, s, mx, mn, sh);
    grid.sync();  // the new state and the entropy statistics are visible
  } else {
    grid.sync();  // the new state is visible
    // per-member entropy statistics over each member's contiguous node range
    for (int mbr = blockIdx.x; mbr < p.nmember; mbr += gridDim.x) {
      const int b = p.member_node_off[mbr], e = p.member_node_off[mbr + 1];
      double ts = 0.0, tmx = -1e300, tmn = 1e300;
      for (int t = b + threadIdx.x; t < e; t += blockDim.x) {
        const double v = p.g.eta[t];
        ts += v; tmx = fmax(tmx, v); tmn = fmin(tmn, v);
      }
      block_reduce3(ts, tmx, tmn, sh);
      if (threadIdx.x == 0) {
        if (p.g.normalise) {
          const double mean = ts / (double)(e - b);
          p.member_scal[2 * mbr] = mean;
          p.member_scal[2 * mbr + 1] = fmax(tmx - mean, mean - tmn);
        } else {
          p.member_scal[2 * mbr] = 0.0;
          p.member_scal[2 * mbr + 1] = 1.0;
        }
      }
      __syncthreads();
    }
    grid.sync();
  }
  // entropy viscosity and the CFL limits, one element per warp (2 EPB per block) at a time; the
  // RHS tile's shared memory (at least 2 KB per 64 threads) holds each warp's KV_WSMEM doubles
  const int wb = threadIdx.x >> 5, nw = 2 * EPB;
  double* sm = reinterpret_cast<double*>(smem_raw) + wb * KV_WSMEM;
  for (int e = blockIdx.x * nw + wb; e < p.v.nelem; e += gridDim.x * nw)
    visc_dt_warp(p.v, e, threadIdx.x & 31, sm, true);
}

}  // namespace sod
