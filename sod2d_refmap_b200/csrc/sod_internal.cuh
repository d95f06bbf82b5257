// Internal declarations of libsod2d_b200 (sm_100a).  Not part of the C ABI.
//
// Device data layout (all element arrays in the library's own natural-ijk local order
// d = i + 4*j + 16*k, i,j,k in ascending-coordinate order 0..3):
//   econn   [e*64 + d]            int32 unique node id
//   geo64   [(e*10 + c)*64 + d]   FP64: c = 0..8 He(i,j) at c = 3*i + j, c = 9 gpvol
//   geo32   same, FP32 copy used by the mixed-precision kernels
//   mue     [e*64 + d]            FP64 entropy viscosity; mue32 FP32 copy
//   helem_l [e*64 + d]            FP64 min node distance; helem [e]
//   n2e_ptr [npoin+1], n2e [64*nelem]  CSR node -> packed (e*64 + d), ascending e
//   Node fields are SoA columns of npoin doubles (the reference's Fortran layout).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <atomic>
#include <mutex>
#include <unordered_map>
#include <vector>
#include "../../include/sod2d_b200.h"
#include <nvtx3/nvToolsExt.h>

namespace sod {

constexpr int P = 3;
constexpr int NP1 = P + 1;
constexpr int NN = NP1 * NP1 * NP1;   // 64 nodes / gauss points per element
constexpr int NGEO = 10;              // 9 He entries + gpvol
constexpr int NRES = 6;               // element residual fields: mass, mom x3, ener, eta
constexpr double kSuthC1 = 0.000001458;  // sutherland_viscosity (mod_fluid_viscosity.f90:21-41)
constexpr double kSuthS = 110.4;
// shared-memory field stride: 4 k-planes of 16 values, plane pitch 22 (bank-conflict free
// for the xi/eta/zeta line reads of a 4x4x2 warp in FP64)
constexpr int PLANE = 22;
constexpr int FSTRIDE = 4 * PLANE;    // 88
__host__ __device__ constexpr int sidx(int i, int j, int k) { return i + 4 * j + PLANE * k; }

void set_error(const char* fmt, ...);

// Host-side NVTX range for the duration of a scope (no device synchronisation; visible to
// Nsight tools, free otherwise).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
extern std::atomic<int64_t> g_launches;

#define SOD_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess) {                                                            \
      ::sod::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
      return SOD_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)

#define SOD_CHECK_LAUNCH()                                                              \
  do {                                                                                  \
    ::sod::g_launches.fetch_add(1, std::memory_order_relaxed);                          \
    cudaError_t _e = cudaGetLastError();                                                \
    if (_e != cudaSuccess) {                                                            \
      ::sod::set_error("%s:%d kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(_e)); \
      return SOD_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)

#define SOD_ARG(cond, msg)                                                              \
  do {                                                                                  \
    if (!(cond)) {                                                                      \
      ::sod::set_error("invalid argument: %s", msg);                                    \
      return SOD_ERR_ARG;                                                               \
    }                                                                                   \
  } while (0)

struct DevParams {
  double gamma, Rgas, Cp, Prt, ce, cmax, cglob, c_rho, c_ener, cfl_conv, cfl_diff;
  int normalise;
  double g_gm1, inv_gm1, inv_Rgas;  // gamma/(gamma-1), 1/(gamma-1), 1/Rgas (host-computed)
  double CpPr, Cp09;                 // Cp/Prt, Cp/0.9 (host-computed)
  // FP32 copies for the mixed kernels (host-converted: FP64->FP32 conversions are slow on the GPU)
  float gamma_f, c_rho_f, c_ener_f, CpPr_f, Cp09_f;  // gamma, c_rho, c_ener, Cp/Prt, Cp/0.9
  int flag_les;
  double c_sgs;
  int total_enthalpy;  // flag_total_enthalpy: energy convection of full_convec_ijk_H
};

// 1-D derivative matrix in natural order: D[m][n] = l_n'(x_m)
struct DMat {
  double d[NP1][NP1];
};

// Arguments of the fused element-RHS kernels.
struct RhsArgs {
  int nelem;
  const int32_t* __restrict__ econn;
  const void* geo;                 // R [e][10][64]
  const void* mue;                 // R [e][64]
  const double* __restrict__ musgs;  // FP64 [e][64] or null
  const double* __restrict__ rho;
  const double* __restrict__ q0;
  const double* __restrict__ q1;
  const double* __restrict__ q2;
  const double* __restrict__ E;
  const double* __restrict__ mu_factor;  // per node
  void* rel;                       // R [(e*64 + d)*6 + f]
  DMat D;
  float Df[NP1][NP1];              // D in FP32 (mixed kernels)
  DevParams prm;
};

// Scratch owned by a mesh for the step pipeline (allocated lazily, sized by npoin/nelem).
// Element residuals of the fused path are node-major: rel[(e*64 + d)*NRES + f], so that one
// gathered contribution (6 fields) is 3 vector loads of contiguous memory.
template <typename R> struct Vec2;
template <> struct Vec2<float> { using T = float2; };
template <> struct Vec2<double> { using T = double2; };
template <typename R>
__device__ __forceinline__ void store_res6(R* rel, size_t node, R a0, R a1, R a2, R a3, R a4, R a5) {
  using V = typename Vec2<R>::T;
  V* o = reinterpret_cast<V*>(rel + node * NRES);
  o[0] = V{a0, a1};
  o[1] = V{a2, a3};
  o[2] = V{a4, a5};
}
template <typename R>
__device__ __forceinline__ void load_res6(const R* rel, size_t node, R (&v)[6]) {
  using V = typename Vec2<R>::T;
  const V* s = reinterpret_cast<const V*>(rel + node * NRES);
  const V x = s[0], y = s[1], z = s[2];
  v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y; v[4] = z.x; v[5] = z.y;
}

struct StepBuffers {
  int64_t npoin = 0, nelem = 0;
  double* ys = nullptr;      // stage state 5*npoin
  double* rsum = nullptr;    // RK accumulators 6*npoin (mass, mom x3, ener, eta); FP64, or FP32 in its first half on the mixed path
  void* rel = nullptr;       // element residuals nelem*6*64 (double or float)
  size_t rel_bytes = 0;
  double* red = nullptr;     // reduction partials
  int64_t red_cap = 0;
  double* scal = nullptr;    // device scalars: [0] eta mean, [1] eta norm, [2] dt, [3] ...
  unsigned int* counters = nullptr;  // last-block-done counters
  double* mu_fluid = nullptr;        // stage Sutherland viscosity scratch (unused by fused path)
};

struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  int nsteps = 0;
  int nkernels = 0;
};

// Boundary data of a non-periodic mesh (sod_bc.cu), compacted to the nb boundary nodes in
// ascending node order; per-boundary-node columns are [field][nb].
struct BcState {
  int nb = 0;
  int32_t* node = nullptr;     // boundary node ids
  int32_t* code = nullptr;     // bou_codes_nodes of each
  int32_t* nbr = nullptr;      // lnbn_nodes of each (0-based)
  double* normal = nullptr;    // [3][nb] normalsAtNodes
  double* ubuf = nullptr;      // [3][nb] u_buffer
  double* aux2 = nullptr;      // [5][nb] state of the lnbn node (rho, q x3, E)
  double* u_stage = nullptr;   // [3][nb] aux_u of the previous stage's EOS
  double* u_final = nullptr;   // [3][nb] u(:,:,pos) at the start of the step
  bool has_slip = false;       // a slip code (6, 7): its new state reads the previous velocity
  // slip-wall adjoint data per boundary node ([..][nb] columns, one allocation): the stage
  // residuals of rho and q (sl_res [4 stages][4]), the pre-routine rho and q of the five
  // applications of a step (sl_pre [5][4]: stages 1-4, then the update), the velocity each one
  // reads (sl_uo [5][3]) and the adjoint of that velocity (sl_ubar [3])
  double* slip = nullptr;
  double *sl_res = nullptr, *sl_pre = nullptr, *sl_uo = nullptr, *sl_ubar = nullptr;
  // far-field nodes (code 1): their lnbn nodes, each with the far-field nodes that read it in
  // ascending order (CSR), for the ordered scatter of the adjoint; the adjoint's per-node
  // contributions [5][nb]
  int nff = 0, ff_nu = 0;
  bool ff_nbr_on_boundary = false;  // an lnbn node of a far-field node is a boundary node
  int32_t* ff_ptr = nullptr;
  int32_t* ff_target = nullptr;
  int32_t* ff_b = nullptr;
  double* ff_contrib = nullptr;
  double* ff_res = nullptr;  // [4 stages][5][ff_nu] residuals at the lnbn targets (with a buffer zone)
  SodBcParams prm{};
};

// Penalisation buffer zone (sod_buffer.cu): the nodes inside an enabled zone in ascending
// order with their relaxation factor xi and u_buffer ([3][nb]).
struct ZoneState {
  int nb = 0;
  int32_t* node = nullptr;
  double* xi = nullptr;
  double* ub = nullptr;
  int32_t* zmap = nullptr;  // [npoin] zone entry of a node, -1 outside every zone
  double rho_inf = 0.0, E_inf = 0.0;
};

// updateBuffer on one node's (rho, q, E) given its zone entry (time_integ.f90:580-585)
__device__ __forceinline__ void zone_point(const double* xi, const double* ub, int znb, int idx, double rho_inf,
                                           double E_inf, double& rho, double (&q)[3], double& E) {
  const double x = xi[idx];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double ur = ub[(size_t)d * znb + idx] * rho;
    q[d] = ur + x * (q[d] - ur);
  }
  E = E_inf + x * (E - E_inf);
  rho = rho_inf + x * (rho - rho_inf);
}

// Wall model (sod_wallmodel.cu): wall nodes, their (face, node) entries grouped by node with
// the exchange node, weight |bounorm| wgp_b, node normal, wall distance and roughness; the
// per-node contribution to the momentum residual [3][npoin] (zero off the walls) and tauw.
struct WallModelState {
  int nw = 0, nent = 0, type = 0;
  int32_t *wnode = nullptr, *wptr = nullptr, *ex = nullptr;
  double *w = nullptr, *nrm = nullptr, *y = nullptr, *zo = nullptr;
  double *contrib = nullptr, *tauw = nullptr;
  const double* walave = nullptr;  // caller's time-averaged velocity (flag_walave), or null
  // adjoint: targets (wall and exchange nodes) with their wall index and reading entries, the
  // per-wall-node and per-entry contributions, and the per-node result [5][npoin] (zero elsewhere)
  int nt = 0;
  int32_t *tnode = nullptr, *twall = nullptr, *tptr = nullptr, *tent = nullptr;
  double *own_bar = nullptr, *ex_bar = nullptr, *wmbar = nullptr;
};

// EOS and Sutherland viscosity of node n at the new level (time_integ.f90:445-463,
// mod_fluid_viscosity.f90:21-41) from its conserved values
__device__ __forceinline__ void eos_store(size_t n, size_t N, double rho, const double (&qq)[3], double e, double g,
                                          double Rgas, double* u_n, double* pr_n, double* e_int, double* csound,
                                          double* machno, double* Tem, double* eta, double* mu_fluid,
                                          const double* mu_factor) {
  const double u0 = qq[0] / rho, u1 = qq[1] / rho, u2 = qq[2] / rho;
  double umag = u0 * u0 + u1 * u1 + u2 * u2;
  const double ei = (e / rho) - 0.5 * umag;
  const double pr = rho * (g - 1.0) * ei;
  const double cs = ::sqrt(g * pr / rho);
  umag = ::sqrt(umag);
  const double T = pr / (rho * Rgas);
  u_n[n] = u0;
  u_n[n + N] = u1;
  u_n[n + 2 * N] = u2;
  e_int[n] = ei;
  pr_n[n] = pr;
  csound[n] = cs;
  machno[n] = umag / cs;
  Tem[n] = T;
  eta[n] = (rho / (g - 1.0)) * log(pr / pow(rho, g));
  mu_fluid[n] = mu_factor[n] * kSuthC1 * (T * ::sqrt(T)) / (T + kSuthS);
}

}  // namespace sod

struct SodMesh {
  int32_t nelem = 0, npoin = 0;
  // working nodes (lpoin_w): rows with elements; the others are periodic slave rows that the
  // node kernels skip (a row works iff n2e_ptr[n+1] > n2e_ptr[n])
  int32_t npoin_w = 0;
  bool has_slaves = false;
  std::vector<uint8_t> slave_host;  // [npoin] 1 on slave rows (only kept when has_slaves)
  int device = 0;
  sod::DevParams prm{};
  sod::DMat D{};
  double wgp_nat[sod::NN];
  int perm_a_of_d[sod::NN];   // reference local node a of library node d
  int perm_d_of_a[sod::NN];
  // device arrays
  int32_t* econn = nullptr;
  double* geo64 = nullptr;
  float* geo32 = nullptr;
  double* Ml = nullptr;
  double* helem = nullptr;
  double* helem_l = nullptr;
  double* jratio = nullptr;  // (minJe/maxJe)^2 per element (smart_visc_spectral :76-83)
  int32_t* n2e_ptr = nullptr;
  int32_t* n2e = nullptr;
  double* mue_int = nullptr;   // internal-layout entropy viscosity (FP64)
  float* mue32 = nullptr;      // FP32 copy
  int32_t* a_of_d_dev = nullptr;  // perm table on device (64)
  sod::StepBuffers buf;
  std::unordered_map<uint64_t, sod::GraphEntry> graphs;
  int tuned_epb[2] = {0, 0};
  // per precision: 0 runs a stage as two launches (fused RHS, gather); n > 0 as one cooperative
  // launch of n resident blocks per SM (the autotuner's choice, or sod_set_rhs_config)
  int persist_ctas[2] = {0, 0};
  struct TuneEntry { int epb, ctas; float ms; };
  std::vector<TuneEntry> tune_table[2];  // the last sod_autotune sweep per precision
  std::vector<double*> host_mirror;  // device buffers of sod_rk4_main_host
  // sod_rk4_main_host's read-back: a stream and two events (created on first use)
  cudaStream_t host_copy_stream = nullptr;
  cudaEvent_t host_ev_state = nullptr, host_ev_copied = nullptr;
  // ensemble members (a SodBatch's concatenated mesh); nmember == 0 for a single mesh
  int nmember = 0;
  int32_t* node_member = nullptr;   // [npoin]
  int32_t* elem_member = nullptr;   // [nelem]
  int32_t* member_node_off = nullptr;  // [nmember+1] contiguous node ranges
  double* member_scal = nullptr;    // [nmember][2] eta mean, eta norm
  double* member_dt_bits = nullptr; // [nmember] scratch for the per-member dt min
  double* musgs_int = nullptr;  // LES: internal-layout SGS viscosity (FP64), allocated on first use
  // adjoint scratch (sod_adjoint.cu): stage states, seeds, accumulators
  double* adj = nullptr;
  size_t adj_len = 0;
  int index_base = 0;          // of the caller's node ids (SodMeshDesc.index_base)
  sod::BcState bc;             // boundaries (nb == 0: periodic path, noBoundaries)
  sod::ZoneState zone;         // buffer zone (nb == 0: flag_buffer_on = .false.)
  const double* source = nullptr;  // caller's constant momentum source term (npoin,3), or null
  sod::WallModelState wmodel;      // wall model (nw == 0: isWallModelOn = .false.)
  double* postpro = nullptr;       // element-node scratch of sod_compute_field_derivs
  size_t postpro_len = 0;
};

namespace sod {
// helpers implemented in sod_mesh.cu
int ensure_step_buffers(SodMesh* m, bool mixed);
int mesh_set_local_tables(SodMesh* m, const int32_t* gI, const int32_t* gJ, const int32_t* gK,
                          const double* dlxigp_ip, const double* wgp, int base);
// a SodMesh built on the device from reference-layout device arrays (sod_refargs.cu): He may be
// null (geometry then holds gpvol only), wgp null (no jratio), helem/helem_l null, lpoin_w null
// (every node works); the caller destroys it with sod_mesh_destroy
int mesh_from_device_ref(int nelem, int npoin, int base, const int32_t* connec, const double* He,
                         const double* gpvol, const double* dlxigp_ip, const int32_t* invAtoIJK,
                         const int32_t* gI, const int32_t* gJ, const int32_t* gK, const double* wgp,
                         const double* helem_l, const double* helem, int npoin_w, const int32_t* lpoin_w,
                         const SodParams* params, cudaStream_t st, SodMesh** out);
int mesh_ref_to_internal_elem(SodMesh* m, const double* ref_dev /*(nelem,64) F*/, double* int_dev,
                              cudaStream_t st);
int mesh_internal_to_ref_elem(SodMesh* m, const double* int_dev, double* ref_dev, cudaStream_t st);
int launch_copy_f32(const double* src, float* dst, int64_t n, cudaStream_t st);
int init_kernel_attrs();
// bounded host wait (sod_set_wait_timeout) and the non-finite flag of the stage-4 gather
constexpr int kNonfiniteCounter = 1;  // index in StepBuffers::counters
int sync_stream(cudaStream_t st);
int take_nonfinite(SodMesh* m, cudaStream_t st, bool* flagged);
// boundary conditions (sod_bc.cu), used by the step pipeline when m->bc.nb > 0
int bc_snapshot_u(SodMesh* m, const double* u, cudaStream_t st);
int bc_stage(SodMesh* m, double* ys, int stage, cudaStream_t st);
int bc_final(SodMesh* m, SodState* s, double* Reta, cudaStream_t st);
// adjoint of the routine in place on vbar ([5][npoin]); y ([5][npoin]) is the state the routine
// read (only its far-field nodes' lnbn rows are used; may be null without far-field nodes);
// app (0-3: stage 1-4, 4: the update) selects the slip-wall data of that application of the
// step (-1: none; slip walls are then refused); the adjoint of the velocity a slip wall read is
// left in bc.sl_ubar
int bc_adjoint(SodMesh* m, double* vbar, const double* y, int app, cudaStream_t st);
// slip-wall adjoint helpers (sod_bc.cu): the rho and q residuals of stage s at the slip nodes
// from the element residuals; the pre-routine states and read velocities of the five
// applications; the velocity adjoint pushed into the adjoint of the state it was read from
int bc_slip_residuals(SodMesh* m, int stage, const void* rel, cudaStream_t st);
int bc_slip_prepare(SodMesh* m, const double* rho0, const double* q0, const double* Y1, const double* Y2,
                    const double* Y3, const double* dt_dev, cudaStream_t st);
int bc_slip_push(SodMesh* m, const double* rho, const double* q, double* vrho, double* vq, cudaStream_t st);
// far-field with a buffer zone: the stage residuals at the lnbn targets, and the updated state
// the final routine reads there (y0 - dt sum b_s R_s, then updateBuffer) into the rows of zf
int bc_ff_residuals(SodMesh* m, int stage, const void* rel, cudaStream_t st);
int bc_ff_final(SodMesh* m, const double* rho0, const double* q0, const double* E0, const double* dt_dev, double* zf,
                cudaStream_t st);
void bc_free(SodMesh* m);
// entropy normalisation (mean and spread of eta) recomputed into buf.scal after a routine that
// changed eta
int eta_stats(SodMesh* m, const double* eta, cudaStream_t st);
// buffer zone (sod_buffer.cu), used by the step pipeline when m->zone.nb > 0: updateBuffer on a
// stage state ([5][npoin]), on the updated state (with the EOS of the zone nodes), and its
// adjoint in place on vbar ([5][npoin])
int zone_stage(SodMesh* m, double* ys, cudaStream_t st);
int zone_final(SodMesh* m, SodState* s, cudaStream_t st);
int zone_adjoint(SodMesh* m, double* vbar, cudaStream_t st);
void zone_free(SodMesh* m);
// wall model (sod_wallmodel.cu) on a stage state: wmodel.contrib <- the wall shear terms
int wall_model_stage(SodMesh* m, const double* rho, const double* q0, const double* E, const double* mu_factor,
                     cudaStream_t st);
void wall_model_free(SodMesh* m);
// adjoint of the stage's wall-model term for seeds w ([5][npoin]) into wmodel.wmbar
int wall_model_vjp(SodMesh* m, const double* rho, const double* q0, const double* E, const double* mu_factor,
                   const double* w, cudaStream_t st);
// packed-FP32 (FFMA2) variant of the mixed fused RHS kernel (sod_rhs_mixed.cu)
int launch_rhs_mixed2(const RhsArgs& a, int epb, cudaStream_t st);
// LES (sod_les.cu): musgs_int <- sgs_visc of the velocity u (3 columns of npoin)
int launch_sgs(SodMesh* m, const double* u, cudaStream_t st);
int init_rhs_mixed2_attrs();
}  // namespace sod
