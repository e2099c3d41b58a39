// capi.cu -- host runtime behind the C ABI (include/aero_b200.h).
//
// Owns no device memory: every device buffer is carved out of the workspace
// the caller binds.  Keeps the A/B buffer parity, the host mirror of the
// step counter and the force-history read cursor, and replays the step
// sequence of two steps as a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/aero_b200.h"
#include "lbm_dispatch.h"
#include "lbm_kernels.cuh"
#include "lbm_les.cuh"
#include "lbm_quad.cuh"

using namespace aero;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CUDA_TRY(expr)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (expr);                                                                 \
    if (e_ != cudaSuccess) return fail(AERO_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

static_assert(kStatsValues == AERO_FIELD_STATS, "field statistics layout");

constexpr uint64_t kAlign = 256;
uint64_t align_up(uint64_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

struct Layout {
  uint64_t P[2], flags, lbits, loff, lc_mask, lc_q, lc_cell, lc_contrib, fin_partial, prof_off, force_const, prof_const,
      prev[2], g[2], U, cs_cell, inflow, recycle, hist, prof_out, counters, stats, stage_link, stage_nb, stage_out,
      lc_contrib2, run_params, total;
};

struct WTab {
  double w[19];
};

// small element-wise kernels for state I/O --------------------------------
__global__ void k_set_i64(int64_t *p, int64_t v) { *p = v; }

// The outlet state is (Q, nz, ny) absolute populations at the boundary and
// (nz, ny, QP) deviations on the device (one 16-byte-aligned row per cell
// row, so a tile's rows are one contiguous copy).
template <class Real>
__global__ void k_prev_in(Real *dst, const double *src, int Q, int QP, int64_t plane, WTab w) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)Q * plane) return;
  const int64_t i = k / plane, r = k - i * plane;
  dst[r * QP + i] = (Real)(src[k] - w.w[i]);
}
template <class Real>
__global__ void k_prev_out(double *dst, const Real *src, int Q, int QP, int64_t plane, WTab w) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)Q * plane) return;
  const int64_t i = k / plane, r = k - i * plane;
  dst[k] = w.w[i] + (double)src[r * QP + i];
}
template <class Real>
__global__ void k_g_in(Real *dst, const double *src, int Qg, int64_t ncells, int64_t cs) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)Qg * ncells) return;
  dst[(k / ncells) * cs + k % ncells] = (Real)src[k];
}
template <class Real>
__global__ void k_g_out(double *dst, const Real *src, int Qg, int64_t ncells, int64_t cs) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)Qg * ncells) return;
  dst[k] = (double)src[(k / ncells) * cs + k % ncells];
}

unsigned blocks_for(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

int aero::set_error(int code, const char *msg) {
  g_err = msg ? msg : "";
  return code;
}

struct AeroBatch;

struct AeroLattice {
  AeroParams prm;
  int Q = 0, QP = 0, Qg = 0;
  int64_t ncells = 0, cs = 0, nwords = 0, prev_plane = 0;
  int nwx = 0, nprof = 0, hist_cap = 4096;
  std::vector<double> force_const, prof_const;  // rest-weight parts of forces / profile
  uint32_t feat = 0;
  // host geometry tables (kept until bind)
  std::vector<uint8_t> solid;
  std::vector<uint32_t> lbits, lc_mask;
  std::vector<int32_t> loff, prof_off;
  std::vector<float> lc_q;
  std::vector<int64_t> lc_cell;
  std::vector<double> cs_cell;
  int64_t n_links = 0;
  bool geometry = false;
  // workspace
  Layout lay{};
  char *ws = nullptr;
  bool bound = false, state_set = false;
  int cur = 0;
  bool old_is_state = false;
  int64_t step_count = 0, read_upto = 0;
  MrtCoeffs<double> mrt{};
  Mrt3Adapted<double> mrt3{};
  WTab w{}, wg{};
  // CUDA graphs of a two-step sequence, one per starting parity
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t pair_exec[2] = {nullptr, nullptr};
  bool use_graphs = true;
  int device = -1;  // device of the bound workspace
  int inflow_ring = 0;            // steps of inflow fields the device holds
  int64_t inflow_upto = 0;        // inflow fields are on the device for steps < inflow_upto
  int recycle_blocks = 0;
  AeroBatch *batch = nullptr;  // batch this lattice is a member of (stepped only by it)
  double cd_norm = 1.0;        // drag normalisation given when it joined the batch
  // step kernel: block shape of k_step (kStepShapeXY), the row-tiled
  // k_step_tiled with its plan, or the two-cells-per-thread k_step_pair
  int step_shape = 0;
  bool tiled = false;
  bool pair = false;
  bool quad = false;
  bool les_fused = false;  // k_step_les: LES velocity stencil in shared memory, no moments pass
  // AA layout: one population buffer updated in place.  Between aero_step
  // calls it holds the post-boundary state (aa_holds_state) in layout cur;
  // a call first collides it in place, then runs its steps, the last of
  // which stores its state instead of colliding it.
  bool aa = false;
  bool aa_holds_state = false;
  int les_chunk = 0;       // planes per block of k_step_les
  int tile_blocks = 0, tile_rows = 0, tiles_per_plane = 0, ntiles = 0;
  uint32_t tile_extra_tx = 0;  // AERO_B200_TEST_STALL_TILES=1 at bind: stages never complete
  // persistent runs (k_run_small) for small lattices; run_stall_block >= 0
  // only under AERO_B200_TEST_STALL_RUN=1 at bind (that block leaves early)
  bool persistent = true;
  int run_stall_block = -1;
  // AERO_B200_GENERIC_KERNELS=1 at bind: no feature-specialised kernels
  bool generic_kernels = false;
  // optional per-kernel event timing (eager launches only)
  bool timing = false;
  std::vector<cudaEvent_t> ev;  // 4 events per timed step
  int64_t timed_steps = 0;
};

namespace {

bool is_f64(const AeroLattice *L) { return L->prm.storage == AERO_STORE_F64; }

// A convective or zero-gradient outlet re-evaluates plane x = nx-2 at the
// outlet cells x = nx-1.  In the AA layout, when nx-2 and nx-1 sit in one warp
// of the step kernel (128-wide blocks along x, so unless nx-1 is a multiple of
// 32) and nothing else reads that plane, the outlet thread takes the post-
// boundary state of nx-2 from its neighbour lane by warp shuffles.
bool aa_outlet_shuffle(const AeroLattice *L) {
  const bool open = L->feat & FEAT_OPEN;
  const bool copy = open && (L->prm.outlet_bc == AERO_OUTLET_CONVECTIVE || L->prm.outlet_bc == AERO_OUTLET_ZEROGRADIENT);
  return copy && !(L->feat & FEAT_RECYCLE) && (L->prm.nx - 1) % 32 != 0;
}

// Whether a step re-evaluates plane x = nx-2 at cells of other warps (the
// outlet when the shuffle does not apply, or the recycling inlet at x = 0):
// in the AA layout its pulled populations are staged before each step.
bool aa_stages_outlet(const AeroLattice *L) {
  const bool open = L->feat & FEAT_OPEN;
  const bool copy = open && (L->prm.outlet_bc == AERO_OUTLET_CONVECTIVE || L->prm.outlet_bc == AERO_OUTLET_ZEROGRADIENT);
  return (copy && !aa_outlet_shuffle(L)) || (L->feat & FEAT_RECYCLE);
}

// Lattices the two-cells-per-thread kernels take: D3Q19, 4- or 2-byte
// storage, even nx (>= 6 in a batch, so that the four edge columns are
// distinct), no body force or scalar lattice (which act on every cell).
bool pair_capable(const AeroLattice *L, int min_nx) {
  return L->prm.dims == 3 && !is_f64(L) && L->prm.nx % 2 == 0 && L->prm.nx >= min_nx &&
         !(L->feat & (FEAT_BODY_FORCE | FEAT_THERMAL));
}

// Lattices the four-cells-per-thread kernel takes: D3Q19, 16-bit storage,
// nx a multiple of 4 (>= 12 where open or recycling columns run per cell),
// no body force or scalar lattice.
bool quad_capable(const AeroLattice *L) {
  const bool edges = L->prm.dims == 3 && (L->feat & (FEAT_OPEN | FEAT_RECYCLE));
  return L->prm.dims == 3 && (L->prm.storage == AERO_STORE_F16 || L->prm.storage == AERO_STORE_BF16) &&
         L->prm.nx % 4 == 0 && L->prm.nx >= (edges ? 12 : 8) && !(L->feat & (FEAT_BODY_FORCE | FEAT_THERMAL));
}

template <class Real>
const Ops<Real> *get_ops(const AeroLattice *L);
template <>
const Ops<double> *get_ops<double>(const AeroLattice *L) {
  return ops_f64(L->prm.dims, L->prm.collision);
}
// The kernel set compiled for this lattice's exact feature word and wall
// type, where there is one (variant k + 1 of kFxSets[k]); else 0, the
// generic kernels.
int kernel_variant(const AeroLattice *L, const Ops<float> **ops = nullptr) {
  if (L->generic_kernels || is_f64(L)) return 0;
  for (int k = 0; k < kFxCount; k++)
    if (const Ops<float> *o = kFxSets[k](L->prm.dims, L->prm.collision, L->prm.storage, L->feat, L->prm.wall_bc)) {
      if (ops) *ops = o;
      return k + 1;
    }
  return 0;
}
template <>
const Ops<float> *get_ops<float>(const AeroLattice *L) {
  const Ops<float> *fx = nullptr;
  if (kernel_variant(L, &fx)) return fx;
  switch (L->prm.storage) {
    case AERO_STORE_F32: return ops_f32(L->prm.dims, L->prm.collision);
    case AERO_STORE_F16: return ops_f16(L->prm.dims, L->prm.collision);
    case AERO_STORE_BF16: return ops_bf16(L->prm.dims, L->prm.collision);
  }
  return nullptr;
}

template <class Real>
StepParams<Real> make_params(const AeroLattice *L, int cur) {
  const AeroParams &a = L->prm;
  StepParams<Real> p;
  std::memset(&p, 0, sizeof(p));
  char *ws = L->ws;
  const int nxt = 1 - cur;
  p.nx = a.nx;
  p.ny = a.ny;
  p.nz = a.nz;
  p.nwx = L->nwx;
  p.cs = L->cs;
  p.ncells = L->ncells;
  p.feat = L->feat;
  p.inlet = a.inlet_bc;
  p.outlet = a.outlet_bc;
  p.wall = a.wall_bc;
  p.sponge_thickness = a.sponge_thickness;
  p.sponge_start = std::max(a.nx - a.sponge_thickness, 0);
  p.tile_rows = L->tile_rows;
  p.batch_rows = L->ncells < kBatchSmallCells ? 1 : kBatchRows;
  p.les_chunk = L->les_chunk > 0 ? L->les_chunk : 1;
  p.tile_extra_tx = L->tile_extra_tx;
  p.tiles_per_plane = L->tiles_per_plane;
  p.ntiles = L->ntiles;
  p.P = ws + L->lay.P[L->aa ? 0 : cur];
  p.Pn = ws + L->lay.P[L->aa ? 0 : nxt];
  p.aa = L->aa ? 1 : 0;
  p.aa_layout = cur;
  p.aa_store_state = 0;
  p.aa_shfl_out = (L->aa && aa_outlet_shuffle(L)) ? 1 : 0;
  p.stage_link = L->aa ? ws + L->lay.stage_link : nullptr;
  p.stage_nb = L->aa ? ws + L->lay.stage_nb : nullptr;
  p.stage_out = (L->aa && aa_stages_outlet(L)) ? ws + L->lay.stage_out : nullptr;
  p.flags = reinterpret_cast<const uint8_t *>(ws + L->lay.flags);
  p.lbits = reinterpret_cast<const uint32_t *>(ws + L->lay.lbits);
  p.loff = reinterpret_cast<const int32_t *>(ws + L->lay.loff);
  p.lc_mask = reinterpret_cast<const uint32_t *>(ws + L->lay.lc_mask);
  p.lc_q = reinterpret_cast<const float *>(ws + L->lay.lc_q);
  p.lc_cell = reinterpret_cast<const int64_t *>(ws + L->lay.lc_cell);
  p.n_lc = (int64_t)L->lc_cell.size();
  p.prev = reinterpret_cast<const Real *>(ws + L->lay.prev[cur]);
  p.prevn = reinterpret_cast<Real *>(ws + L->lay.prev[nxt]);
  p.g = reinterpret_cast<const Real *>(ws + L->lay.g[cur]);
  p.gn = reinterpret_cast<Real *>(ws + L->lay.g[nxt]);
  p.U = reinterpret_cast<const Real *>(ws + L->lay.U);
  p.Uw = reinterpret_cast<Real *>(ws + L->lay.U);
  p.cs_cell = reinterpret_cast<const Real *>(ws + L->lay.cs_cell);
  p.inflow = reinterpret_cast<const Real *>(ws + L->lay.inflow);
  p.inflow_ring = std::max(L->inflow_ring, 1);
  p.recycle_partial = reinterpret_cast<double *>(ws + L->lay.recycle);
  p.recycle_mean = reinterpret_cast<double *>(ws + L->lay.recycle) + L->recycle_blocks;
  p.recycle_ticket = reinterpret_cast<uint32_t *>(p.recycle_mean + 1);
  p.recycle_blocks = L->recycle_blocks;
  p.lc_contrib = reinterpret_cast<double *>(ws + L->lay.lc_contrib);
  p.fin_partial = reinterpret_cast<double *>(ws + L->lay.fin_partial);
  {
    // about 256 link cells per finalisation block (one per thread): the
    // pass is latency-bound, so it spreads over as many SMs as it can use
    const int64_t nlc = (int64_t)L->lc_cell.size();
    const int64_t nb = std::min<int64_t>(std::max<int64_t>((nlc + 255) / 256, 1), kFinalizeMaxBlocks);
    p.fin_blocks = (int32_t)nb;
    p.fin_chunk = (nlc + nb - 1) / nb;
  }
  p.force_const = reinterpret_cast<const double *>(ws + L->lay.force_const);
  p.prof_const = reinterpret_cast<const double *>(ws + L->lay.prof_const);
  p.prof_off = reinterpret_cast<const int32_t *>(ws + L->lay.prof_off);
  p.hist = reinterpret_cast<double *>(ws + L->lay.hist);
  p.prof_out = reinterpret_cast<double *>(ws + L->lay.prof_out);
  p.nprof = L->nprof;
  p.hist_cap = L->hist_cap;
  p.want_profile = 1;
  int64_t *ctr = reinterpret_cast<int64_t *>(ws + L->lay.counters);
  p.step = ctr;
  p.hist_base = ctr + 1;
  p.profile_step = ctr + 4;
  p.fin_ticket = reinterpret_cast<uint32_t *>(ctr + 5);
  p.status = reinterpret_cast<uint32_t *>(ctr + 2);
  p.first_bad_step = reinterpret_cast<unsigned long long *>(ctr + 3);
  const double tau = 1.0 / a.omega;
  const double tp = a.trt_lambda * tau + (1.0 - a.trt_lambda);
  const double tm = (tp * tau - 0.5) / (tp - 0.5);
  p.omega = (Real)a.omega;
  p.u0 = (Real)a.u0;
  p.rho_in = (Real)a.rho_in;
  p.rho_out = (Real)a.rho_out;
  p.pert_amp = (Real)std::max(a.inlet_perturbation, 0.0);
  p.trt_lambda = (Real)a.trt_lambda;
  p.trt_sminus = (Real)(1.0 / tm);
  p.sponge_sigma_max = (Real)a.sponge_strength;
  p.base_nu = (Real)((1.0 / a.omega - 0.5) / 3.0);
  p.les_cs2 = (Real)(a.les_cs * a.les_cs);
  p.wall_u_top = (Real)a.wall_velocity_top;
  p.wall_u_bottom = (Real)a.wall_velocity_bottom;
  p.bf_x = (Real)a.body_force[0];
  p.bf_y = (Real)a.body_force[1];
  p.bf_z = (Real)a.body_force[2];
  p.bf_coeff = (Real)(1.0 - 0.5 / (1.0 / a.omega));
  const double aT = (a.scalar_reduced && a.dims == 3) ? 4.0 : 3.0;
  p.omega_T = (Real)(1.0 / (aT * a.alpha_T + 0.5));
  p.T_hot = (Real)a.T_hot;
  p.T_cold = (Real)a.T_cold;
  p.gbeta = (Real)(a.g_gravity * a.beta);
  p.T_ref = (Real)a.T_ref;
  for (int k = 0; k < 3; k++) p.center[k] = a.center[k];
  // rows r >= 1 of the even block and all odd rows carry the 1/2 of the
  // pair-basis inverse (f_i = (s + t) / 2), folded in here
  for (int k = 0; k < 100; k++) p.mrt.Ae[k] = (Real)(L->mrt.Ae[k] * (k < 10 ? 1.0 : 0.5));
  for (int k = 0; k < 70; k++) p.mrt.Ce[k] = (Real)(L->mrt.Ce[k] * (k < 7 ? 1.0 : 0.5));
  for (int k = 0; k < 81; k++) p.mrt.Ao[k] = (Real)(L->mrt.Ao[k] * 0.5);
  for (int k = 0; k < 27; k++) p.mrt.Co[k] = (Real)(L->mrt.Co[k] * 0.5);
  {
    const Mrt3Adapted<double> &m = L->mrt3;
    for (int k = 0; k < 9; k++) p.mrt3.a1[k] = (Real)m.a1[k];
    for (int k = 0; k < 6; k++) p.mrt3.ca1[k] = (Real)m.ca1[k];
    for (int k = 0; k < 4; k++) {
      p.mrt3.e[k] = (Real)m.e[k];
      p.mrt3.v[k] = (Real)m.v[k];
    }
    for (int k = 0; k < 2; k++) {
      p.mrt3.ce[k] = (Real)m.ce[k];
      p.mrt3.cv[k] = (Real)m.cv[k];
    }
    p.mrt3.t2 = (Real)m.t2;
    p.mrt3.ct2 = (Real)m.ct2;
  }
  return p;
}

dim3 cell_grid(const AeroLattice *L) {
  return dim3(blocks_for(L->prm.nx, kStepBlock), (unsigned)L->prm.ny, (unsigned)L->prm.nz);
}

bool les_active(const AeroLattice *L) { return (L->feat & FEAT_LES) != 0; }

// values per inlet cell and step in the inflow ring: the transverse
// velocities of synthetic inflow (dims - 1), or SEM's (u', v', w')
int inflow_components(const AeroLattice *L) { return (L->feat & FEAT_INFLOW_SEM) ? 3 : L->prm.dims - 1; }

// Launches one step with buffer parity `cur` on stream st.  With timing on,
// events bracket the fused step (moments pass + step kernel, which also
// computes the link-cell force contributions) and the force finalisation.
template <class Real>
int launch_step(AeroLattice *L, int cur, cudaStream_t st, bool timed = false, bool store_state = false) {
  const Ops<Real> *ops = get_ops<Real>(L);
  StepParams<Real> p = make_params<Real>(L, cur);
  p.aa_store_state = store_state ? 1 : 0;
  const dim3 grid = cell_grid(L);
  cudaEvent_t *e = nullptr;
  if (timed) {
    const size_t need = 3 * (size_t)(L->timed_steps + 1);
    while (L->ev.size() < need) {
      cudaEvent_t x;
      CUDA_TRY(cudaEventCreate(&x));
      L->ev.push_back(x);
    }
    e = &L->ev[3 * (size_t)L->timed_steps];
    CUDA_TRY(cudaEventRecord(e[0], st));
  }
  if (L->aa) {
    const int64_t n = (int64_t)L->lc_cell.size() + (aa_stages_outlet(L) ? L->prev_plane : 0);
    if (n > 0) CUDA_TRY(ops->aa_stage(p, blocks_for(n, kStageBlock), st));
    if (L->feat & FEAT_RECYCLE) CUDA_TRY(ops->aa_recycle_mean(p, st));
    if (les_active(L)) CUDA_TRY(ops->aa_moments(p, grid, st));
    CUDA_TRY(ops->aa_step(p, grid, st));
  } else {
    if (L->feat & FEAT_RECYCLE) CUDA_TRY(ops->recycle_mean(p, st));
    if (les_active(L) && !L->les_fused) CUDA_TRY(ops->moments(p, false, grid, st));
    if (L->les_fused)
      CUDA_TRY(ops->step_les(p, st));
    else if (L->tiled)
      CUDA_TRY(ops->step_tiled(p, L->tile_blocks, st));
    else if (L->pair)
      CUDA_TRY(ops->step_pair(p, st));
    else if (L->quad)
      CUDA_TRY(ops->step_quad(p, st));
    else if (L->step_shape != 0)
      CUDA_TRY(ops->step_shaped(p, L->step_shape, st));
    else
      CUDA_TRY(ops->step(p, false, grid, st));
  }
  if (timed) CUDA_TRY(cudaEventRecord(e[1], st));
  CUDA_TRY(ops->finalize(p, st));
  if (timed) {
    CUDA_TRY(cudaEventRecord(e[2], st));
    L->timed_steps++;
  }
  return AERO_OK;
}

// AA layout: the in-place collision of the state the buffer holds (set by
// the host or stored by the previous call's last step), before the steps.
template <class Real>
int aa_collide_state(AeroLattice *L, cudaStream_t st) {
  const Ops<Real> *ops = get_ops<Real>(L);
  const StepParams<Real> p = make_params<Real>(L, L->cur);
  const dim3 grid = cell_grid(L);
  if (les_active(L)) CUDA_TRY(ops->moments(p, true, grid, st));
  CUDA_TRY(ops->step(p, true, grid, st));
  L->aa_holds_state = false;
  return AERO_OK;
}

// Lattices stepped by the persistent runner: small (its point is the launch
// and drain per step that dominate such a lattice), two buffers, the
// per-cell step kernel, and no pass before the step (the LES moments pass of
// BGK / TRT, the recycling mean).
constexpr int64_t kRunSmallCells = (int64_t)1 << 19;
bool run_small_ok(const AeroLattice *L) {
  return L->persistent && !L->aa && !L->batch && !L->timing && !L->tiled && !L->pair && !L->quad &&
         !L->les_fused && L->ncells <= kRunSmallCells && !(les_active(L) && L->prm.collision != AERO_MRT) &&
         !(L->feat & FEAT_RECYCLE);
}

template <class Real>
int launch_run_small(AeroLattice *L, int64_t n, cudaStream_t st) {
  StepParams<Real> pp[2] = {make_params<Real>(L, L->cur), make_params<Real>(L, 1 - L->cur)};
  pp[1].lc_contrib = reinterpret_cast<double *>(L->ws + L->lay.lc_contrib2);
  auto *dpp = reinterpret_cast<StepParams<Real> *>(L->ws + L->lay.run_params);
  // from pageable memory: the copy is staged before the call returns
  CUDA_TRY(cudaMemcpyAsync(dpp, pp, sizeof(pp), cudaMemcpyHostToDevice, st));
  int64_t *ctr = reinterpret_cast<int64_t *>(L->ws + L->lay.counters);
  for (int64_t done = 0; done < n;) {
    const int64_t k = std::min(n - done, kRunMaxSteps);
    if (done > 0) {
      // the next launch starts on the other parameter set when k was odd
      if (k & 1) std::swap(pp[0], pp[1]);
      CUDA_TRY(cudaMemcpyAsync(dpp, pp, sizeof(pp), cudaMemcpyHostToDevice, st));
    }
    CUDA_TRY(cudaMemsetAsync(ctr + 6, 0, 4, st));  // barrier arrivals
    const cudaError_t e = get_ops<Real>(L)->run_small(dpp, L->ncells, k, L->run_stall_block, st);
    if (e != cudaSuccess) return fail(AERO_ERR_CUDA, "persistent run: %s", cudaGetErrorString(e));
    done += k;
  }
  return AERO_OK;
}

template <class Real>
int build_pair_graph(AeroLattice *L, int cur) {
  if (!L->cap_stream) CUDA_TRY(cudaStreamCreateWithFlags(&L->cap_stream, cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamBeginCapture(L->cap_stream, cudaStreamCaptureModeThreadLocal));
  int rc = launch_step<Real>(L, cur, L->cap_stream);
  if (rc == AERO_OK) rc = launch_step<Real>(L, 1 - cur, L->cap_stream);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(L->cap_stream, &graph);
  if (rc != AERO_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return fail(AERO_ERR_CUDA, "stream capture: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&L->pair_exec[cur], graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(AERO_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  return AERO_OK;
}

template <class Real>
int do_steps(AeroLattice *L, int64_t n, cudaStream_t st) {
  if (n >= 2 && run_small_ok(L)) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(st, &cap));
    if (cap == cudaStreamCaptureStatusNone) {
      const int rc = launch_run_small<Real>(L, n, st);
      if (rc != AERO_OK) return rc;
      L->cur ^= (int)(n & 1);
      L->step_count += n;
      L->old_is_state = false;
      return AERO_OK;
    }
  }
  if (L->aa && n > 0 && L->aa_holds_state) {
    const int rc = aa_collide_state<Real>(L, st);
    if (rc != AERO_OK) return rc;
  }
  while (n > 0) {
    // in the AA layout the call's last step stores its state (eager launch)
    const int64_t full = L->aa ? n - 1 : n;
    if (full >= 2 && L->use_graphs && !L->timing) {
      if (!L->pair_exec[L->cur]) {
        const int rc = build_pair_graph<Real>(L, L->cur);
        if (rc != AERO_OK) return rc;
      }
      CUDA_TRY(cudaGraphLaunch(L->pair_exec[L->cur], st));
      n -= 2;
      L->step_count += 2;
    } else {
      const int rc = launch_step<Real>(L, L->cur, st, L->timing, L->aa && n == 1);
      if (rc != AERO_OK) return rc;
      L->cur ^= 1;
      n -= 1;
      L->step_count += 1;
    }
    L->old_is_state = false;
  }
  if (L->aa) L->aa_holds_state = true;
  return AERO_OK;
}

template <class Real>
int finish_set_state(AeroLattice *L, int64_t steps, cudaStream_t st);

template <class Real>
int do_set_state(AeroLattice *L, const double *f, const double *prev, const double *g, int64_t steps,
                 cudaStream_t st) {
  const Ops<Real> *ops = get_ops<Real>(L);
  const int old = 1 - L->cur;
  const dim3 grid = cell_grid(L);
  StepParams<Real> p = make_params<Real>(L, L->cur);
  // raw state into the old buffer, then collide it into the current one (A/B
  // layout); in the AA layout the state goes into the single buffer in
  // layout cur and is collided by the next aero_step
  CUDA_TRY(ops->load_state(p, f, L->ws + L->lay.P[L->aa ? 0 : old], grid, st));
  if (prev) {
    const int64_t n = (int64_t)L->Q * L->prev_plane;
    k_prev_in<Real><<<blocks_for(n, 256), 256, 0, st>>>(reinterpret_cast<Real *>(L->ws + L->lay.prev[L->cur]),
                                                        prev, L->Q, L->QP, L->prev_plane, L->w);
    CUDA_TRY(cudaGetLastError());
  }
  if (g && L->prm.thermal) {
    const int64_t n = (int64_t)L->Qg * L->ncells;
    k_g_in<Real><<<blocks_for(n, 256), 256, 0, st>>>(reinterpret_cast<Real *>(L->ws + L->lay.g[L->cur]), g, L->Qg,
                                                     L->ncells, L->cs);
    CUDA_TRY(cudaGetLastError());
  }
  return finish_set_state<Real>(L, steps, st);
}

// After a state has been written into the old population buffer (and the
// outlet and scalar buffers): the step counter, then the collision of the
// state into the current buffer.
template <class Real>
int finish_set_state(AeroLattice *L, int64_t steps, cudaStream_t st) {
  const Ops<Real> *ops = get_ops<Real>(L);
  const int old = 1 - L->cur;
  const dim3 grid = cell_grid(L);
  int64_t *ctr = reinterpret_cast<int64_t *>(L->ws + L->lay.counters);
  k_set_i64<<<1, 1, 0, st>>>(ctr, steps);
  CUDA_TRY(cudaGetLastError());
  if (L->aa) {
    L->aa_holds_state = true;
  } else {
    StepParams<Real> q = make_params<Real>(L, L->cur);
    q.P = L->ws + L->lay.P[old];
    q.Pn = L->ws + L->lay.P[L->cur];
    if (les_active(L)) CUDA_TRY(ops->moments(q, true, grid, st));
    CUDA_TRY(ops->step(q, true, grid, st));
  }
  L->old_is_state = true;
  L->step_count = steps;
  L->read_upto = steps;
  L->inflow_upto = steps;  // inflow fields are uploaded again from the new step count
  L->state_set = true;
  return AERO_OK;
}

template <class Real>
int do_set_equilibrium(AeroLattice *L, const EqFields &e, int64_t steps, cudaStream_t st) {
  const Ops<Real> *ops = get_ops<Real>(L);
  const int old = 1 - L->cur;
  const StepParams<Real> p = make_params<Real>(L, L->cur);
  Real *prev = reinterpret_cast<Real *>(L->ws + L->lay.prev[L->cur]);
  Real *g = L->prm.thermal ? reinterpret_cast<Real *>(L->ws + L->lay.g[L->cur]) : nullptr;
  CUDA_TRY(ops->init_eq(p, e, L->ws + L->lay.P[L->aa ? 0 : old], prev, g, cell_grid(L), st));
  return finish_set_state<Real>(L, steps, st);
}

// Parameters and mode of the kernels that read the current state: with two
// buffers the state of the last step is evaluated from the previous buffer
// (or read as is after a set state); in the AA layout the buffer holds the
// state itself between calls, in layout cur.
template <class Real>
StepParams<Real> reader_params(const AeroLattice *L, bool *raw) {
  *raw = L->aa ? true : L->old_is_state;
  return make_params<Real>(L, L->aa ? L->cur : 1 - L->cur);
}

template <class Real>
int do_get_state(AeroLattice *L, double *f, double *prev, double *g, int z0, int nzs, cudaStream_t st) {
  const Ops<Real> *ops = get_ops<Real>(L);
  if (f) {
    bool raw = false;
    StepParams<Real> p = reader_params<Real>(L, &raw);
    dim3 grid = cell_grid(L);
    grid.z = (unsigned)nzs;
    CUDA_TRY(ops->state_out(p, f, -1, raw, z0, grid, st));
  }
  if (prev) {
    const int64_t n = (int64_t)L->Q * L->prev_plane;
    k_prev_out<Real><<<blocks_for(n, 256), 256, 0, st>>>(
        prev, reinterpret_cast<const Real *>(L->ws + L->lay.prev[L->cur]), L->Q, L->QP, L->prev_plane, L->w);
    CUDA_TRY(cudaGetLastError());
  }
  if (g && L->prm.thermal) {
    const int64_t n = (int64_t)L->Qg * L->ncells;
    k_g_out<Real><<<blocks_for(n, 256), 256, 0, st>>>(g, reinterpret_cast<const Real *>(L->ws + L->lay.g[L->cur]),
                                                      L->Qg, L->ncells, L->cs);
    CUDA_TRY(cudaGetLastError());
  }
  return AERO_OK;
}

// The per-cell-gather kernel (k_step) is the default: on the 512x256x256
// sphere it is faster than the row-tiled kernel in every storage format.
// AERO_B200_TILES=1 at bind time selects the row-tiled kernel instead,
// where a whole x row fits one shared-memory slab and every row starts on a
// 16-byte boundary (the bulk-copy alignment): tiles of tile_rows rows, a
// persistent grid of resident blocks.
template <class Real>
int plan_tiles(AeroLattice *L, bool force = false) {
  L->tiled = false;
  L->tile_blocks = L->tile_rows = L->tiles_per_plane = L->ntiles = 0;
  const char *want = std::getenv("AERO_B200_TILES");
  if (!force && !(want && want[0] == '1')) return AERO_OK;
  const Ops<Real> *ops = get_ops<Real>(L);
  const AeroParams &a = L->prm;
  const int sb = ops->store_bytes;
  const uintptr_t P0 = reinterpret_cast<uintptr_t>(L->ws + L->lay.P[0]);
  const uintptr_t P1 = reinterpret_cast<uintptr_t>(L->ws + L->lay.P[1]);
  if (((int64_t)a.nx * sb) % 16 != 0 || (L->cs * sb) % 16 != 0 || P0 % 16 != 0 || P1 % 16 != 0) return AERO_OK;
  int per_sm = 0, cap = 0, sms = 0;
  CUDA_TRY(ops->tiled_setup(&per_sm, &cap));
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, L->device));
  if (per_sm < 1 || a.nx > cap) return AERO_OK;
  L->tile_rows = std::max(1, std::min(std::min(a.ny, cap / a.nx), kMaxTileRows));
  L->tiles_per_plane = (a.ny + L->tile_rows - 1) / L->tile_rows;
  const int64_t ntiles = (int64_t)L->tiles_per_plane * a.nz;
  if (ntiles >= ((int64_t)1 << 31)) return AERO_OK;
  L->ntiles = (int)ntiles;
  L->tile_blocks = (int)std::min<int64_t>(ntiles, (int64_t)per_sm * sms);
  L->tiled = true;
  return AERO_OK;
}

int check_params(const AeroParams *a) {
  if (!a) return fail(AERO_ERR_INVALID, "params is NULL");
  if (a->abi_version != AERO_ABI_VERSION)
    return fail(AERO_ERR_INVALID, "abi_version %d != %d", a->abi_version, AERO_ABI_VERSION);
  if (a->dims != 2 && a->dims != 3) return fail(AERO_ERR_INVALID, "dims must be 2 or 3");
  if (a->dims == 2 && a->nz != 1) return fail(AERO_ERR_INVALID, "nz must be 1 in 2D");
  if (a->nx < 3 || a->ny < 2 || a->nz < 1) return fail(AERO_ERR_INVALID, "grid too small (nx>=3, ny>=2)");
  if (a->ny > 65535 || a->nz > 65535) return fail(AERO_ERR_INVALID, "ny and nz must be <= 65535");
  if ((int64_t)a->nx * a->ny * a->nz >= ((int64_t)1 << 31) - 64)
    return fail(AERO_ERR_UNSUPPORTED, "lattices are limited to 2^31 - 64 cells (32-bit cell indices)");
  if (a->storage < 0 || a->storage > 3) return fail(AERO_ERR_INVALID, "unknown storage %d", a->storage);
  if (a->collision < 0 || a->collision > 2) return fail(AERO_ERR_INVALID, "unknown collision %d", a->collision);
  if (!(a->omega > 0.0) || !std::isfinite(a->omega)) return fail(AERO_ERR_INVALID, "omega must be > 0");
  if (a->inlet_bc < 0 || a->inlet_bc > 2) return fail(AERO_ERR_INVALID, "unknown inlet_bc");
  if (a->outlet_bc < 0 || a->outlet_bc > 3) return fail(AERO_ERR_INVALID, "unknown outlet_bc");
  if (a->wall_bc < 0 || a->wall_bc > 3) return fail(AERO_ERR_INVALID, "unknown wall_bc");
  if (a->dims == 3 && (a->inlet_bc == AERO_INLET_PRESSURE || a->outlet_bc == AERO_OUTLET_PRESSURE))
    return fail(AERO_ERR_UNSUPPORTED, "pressure inlet/outlet exist only in 2D");
  if (a->sponge_thickness < 0) return fail(AERO_ERR_INVALID, "sponge_thickness < 0");
  if (a->recycling && (a->dims != 3 || a->streamwise_open))
    return fail(AERO_ERR_INVALID, "recycling is a 3D streamwise mode (streamwise_open must be 0)");
  if (a->inflow_field && a->recycling) return fail(AERO_ERR_INVALID, "inflow_field needs an open inlet");
  if (a->inflow_field < 0 || a->inflow_field > 2 || (a->inflow_field == 2 && a->dims != 3))
    return fail(AERO_ERR_INVALID, "inflow_field is 0, 1 (synthetic inflow) or 2 (SEM, 3D)");
  if (a->inflow_ring < 0 || a->inflow_ring > 65536) return fail(AERO_ERR_INVALID, "inflow_ring must be in 0..65536");
  if (a->hist_capacity < 0) return fail(AERO_ERR_INVALID, "hist_capacity < 0");
  if (a->layout != AERO_LAYOUT_AB && a->layout != AERO_LAYOUT_AA)
    return fail(AERO_ERR_INVALID, "layout must be AERO_LAYOUT_AB or AERO_LAYOUT_AA");
  return AERO_OK;
}

}  // namespace

extern "C" {

int aero_abi_version(void) { return AERO_ABI_VERSION; }

const char *aero_last_error(void) { return g_err.c_str(); }

int aero_lattice_q(const AeroParams *a, int32_t *q, int32_t *qg) {
  if (!a) return fail(AERO_ERR_INVALID, "params is NULL");
  const int Q = a->dims == 2 ? 9 : 19;
  if (q) *q = Q;
  if (qg) *qg = a->thermal ? (a->scalar_reduced ? (a->dims == 2 ? 5 : 7) : Q) : 0;
  return AERO_OK;
}

int aero_create(const AeroParams *params, AeroLattice **out) {
  if (!out) return fail(AERO_ERR_INVALID, "out is NULL");
  *out = nullptr;
  const int rc = check_params(params);
  if (rc != AERO_OK) return rc;
  AeroLattice *L = new AeroLattice();
  L->prm = *params;
  const AeroParams &a = L->prm;
  L->Q = a.dims == 2 ? 9 : 19;
  L->QP = (L->Q + 3) / 4 * 4;
  L->Qg = a.thermal ? (a.scalar_reduced ? (a.dims == 2 ? 5 : 7) : L->Q) : 0;
  L->ncells = (int64_t)a.nx * a.ny * a.nz;
  L->cs = (L->ncells + 63) / 64 * 64;
  L->nwx = (a.nx + 31) / 32;
  L->nwords = (int64_t)a.nz * a.ny * L->nwx;
  L->prev_plane = (int64_t)a.nz * a.ny;
  L->nprof = a.dims == 3 ? a.nz : a.ny;
  L->hist_cap = a.hist_capacity > 0 ? a.hist_capacity : 4096;
  for (int i = 0; i < L->Q; i++) L->w.w[i] = a.dims == 2 ? D2Q9::w[i] : D3Q19::w[i];
  uint32_t f = 0;
  if (a.dims == 2 || a.streamwise_open) f |= FEAT_OPEN;
  if (a.bouzidi) f |= FEAT_BOUZIDI;
  if (a.dims == 3 && (std::fabs(a.body_force[0]) >= 1e-16 || std::fabs(a.body_force[1]) >= 1e-16 ||
                      std::fabs(a.body_force[2]) >= 1e-16))
    f |= FEAT_BODY_FORCE;
  if (a.sponge_thickness > 0 && a.sponge_strength > 0.0) f |= FEAT_SPONGE;
  if (a.les && a.collision != AERO_MRT) {
    f |= FEAT_LES;
    if (a.les_model == AERO_LES_WALE) f |= FEAT_LES_WALE;
  }
  if (a.inflow_field && (a.dims == 2 || a.streamwise_open) && a.inlet_bc == AERO_INLET_VELOCITY) {
    f |= FEAT_INFLOW_FIELD;
    if (a.inflow_field == 2) f |= FEAT_INFLOW_SEM;
    L->inflow_ring = a.inflow_ring > 0 ? a.inflow_ring : 64;
  }
  if (a.recycling) {
    f |= FEAT_RECYCLE;
    L->recycle_blocks = (int)((L->prev_plane + kRecycleBlock - 1) / kRecycleBlock);
  }
  if (a.thermal) {
    f |= FEAT_THERMAL;
    if (a.buoyancy) f |= FEAT_BUOYANCY;
    if (a.scalar_reduced) f |= FEAT_SCALAR_REDUCED;
  }
  L->feat = f;
  L->aa = a.layout == AERO_LAYOUT_AA;
  if (a.collision == AERO_MRT && !build_mrt(a.dims, a.omega, L->mrt, nullptr, nullptr)) {
    delete L;
    return fail(AERO_ERR_INVALID, "MRT operator is not block diagonal in the pair basis");
  }
  if (a.collision == AERO_MRT && a.dims == 3 && !build_mrt3_adapted(a.omega, L->mrt3)) {
    delete L;
    return fail(AERO_ERR_INVALID, "MRT operator does not have the cubic block structure");
  }
  const char *ng = std::getenv("AERO_B200_NO_GRAPHS");
  L->use_graphs = !(ng && ng[0] == '1');
  *out = L;
  return AERO_OK;
}

int aero_set_geometry(AeroLattice *L, const uint8_t *solid, const int32_t *links, const float *q, int64_t n_links,
                      const double *phi) {
  if (!L) return fail(AERO_ERR_INVALID, "lattice is NULL");
  if (L->bound) return fail(AERO_ERR_STATE, "geometry must be set before the workspace is bound");
  if (!solid) return fail(AERO_ERR_INVALID, "solid is NULL");
  if (n_links < 0 || (n_links > 0 && (!links || !q))) return fail(AERO_ERR_INVALID, "bad link list");
  const AeroParams &a = L->prm;
  const int lw = a.dims == 3 ? 4 : 3;
  L->solid.assign(solid, solid + L->ncells);
  for (auto &v : L->solid) v = v ? 1 : 0;
  // group links by cell, keep cells in increasing index order
  std::vector<std::pair<int64_t, int64_t>> order;  // (cell, link index)
  order.reserve((size_t)n_links);
  for (int64_t k = 0; k < n_links; k++) {
    const int32_t *lk = links + k * lw;
    const int i = lk[0];
    const int z = a.dims == 3 ? lk[1] : 0, y = lk[lw - 2], x = lk[lw - 1];
    if (i < 1 || i >= L->Q || x < 0 || x >= a.nx || y < 0 || y >= a.ny || z < 0 || z >= a.nz)
      return fail(AERO_ERR_INVALID, "link %lld out of range", (long long)k);
    const int64_t c = ((int64_t)z * a.ny + y) * a.nx + x;
    if (L->solid[c]) return fail(AERO_ERR_INVALID, "link %lld starts in a solid cell", (long long)k);
    if (!(q[k] > 0.0f) || !(q[k] <= 1.0f)) return fail(AERO_ERR_INVALID, "link %lld has q outside (0, 1]", (long long)k);
    order.emplace_back(c, k);
  }
  std::stable_sort(order.begin(), order.end(), [](const auto &u, const auto &v) { return u.first < v.first; });
  L->lc_cell.clear();
  L->lc_mask.clear();
  L->lc_q.clear();
  for (const auto &e : order) {
    if (L->lc_cell.empty() || L->lc_cell.back() != e.first) {
      L->lc_cell.push_back(e.first);
      L->lc_mask.push_back(0u);
      L->lc_q.insert(L->lc_q.end(), L->Q, 0.5f);
    }
    const int i = links[e.second * lw];
    L->lc_mask.back() |= 1u << i;
    L->lc_q[(L->lc_cell.size() - 1) * L->Q + i] = q[e.second];
  }
  L->n_links = n_links;
  L->lbits.assign((size_t)L->nwords, 0u);
  L->loff.assign((size_t)L->nwords, 0);
  for (size_t k = 0; k < L->lc_cell.size(); k++) {
    const int64_t c = L->lc_cell[k];
    const int x = (int)(c % a.nx);
    const int64_t row = c / a.nx;
    const int64_t word = row * L->nwx + (x >> 5);
    if (L->lbits[word] == 0u) L->loff[word] = (int32_t)k;
    L->lbits[word] |= 1u << (x & 31);
  }
  // profile segments: link cells are sorted by cell index, hence by y (2D) / z (3D)
  L->prof_off.assign(L->nprof + 1, 0);
  {
    size_t k = 0;
    for (int b = 0; b <= L->nprof; b++) {
      while (k < L->lc_cell.size()) {
        const int64_t c = L->lc_cell[k];
        const int bin = a.dims == 3 ? (int)(c / ((int64_t)a.nx * a.ny)) : (int)((c / a.nx) % a.ny);
        if (bin >= b) break;
        k++;
      }
      L->prof_off[b] = (int32_t)k;
    }
  }
  if (n_links > 0) L->feat |= FEAT_OBSTACLE_BB; else L->feat &= ~FEAT_OBSTACLE_BB;
  if ((uint64_t)std::max(L->Q, 3) * (uint64_t)L->cs >= (1ull << 32))
    return fail(AERO_ERR_UNSUPPORTED, "lattice too large: Q x cells must stay below 2^32 (32-bit element offsets)");
  // rest-weight part of the momentum exchange: each link contributes
  // e_i (w_i + w_opp) to F and to its pressure part, and r x that to M
  L->force_const.assign(12, 0.0);
  L->prof_const.assign(3 * (size_t)L->nprof, 0.0);
  for (size_t k = 0; k < L->lc_cell.size(); k++) {
    const int64_t c = L->lc_cell[k];
    const double x = (double)(c % a.nx), y = (double)((c / a.nx) % a.ny), z = (double)(c / ((int64_t)a.nx * a.ny));
    const double r[3] = {x - a.center[0], y - a.center[1], z - a.center[2]};
    const int bin = a.dims == 3 ? (int)z : (int)y;
    for (int i = 1; i < L->Q; i++) {
      if (!((L->lc_mask[k] >> i) & 1u)) continue;
      double e[3], w2;
      if (a.dims == 2) {
        e[0] = D2Q9::ex[i]; e[1] = D2Q9::ey[i]; e[2] = 0.0; w2 = 2.0 * D2Q9::w[i];
      } else {
        e[0] = D3Q19::ex[i]; e[1] = D3Q19::ey[i]; e[2] = D3Q19::ez[i]; w2 = 2.0 * D3Q19::w[i];
      }
      for (int dd = 0; dd < 3; dd++) {
        L->force_const[dd] += e[dd] * w2;
        L->force_const[3 + dd] += e[dd] * w2;
        L->prof_const[3 * bin + dd] += e[dd] * w2;
      }
      L->force_const[9] += (r[1] * e[2] - r[2] * e[1]) * w2;
      L->force_const[10] += (r[2] * e[0] - r[0] * e[2]) * w2;
      L->force_const[11] += (r[0] * e[1] - r[1] * e[0]) * w2;
    }
  }
  L->cs_cell.clear();
  L->feat &= ~FEAT_LES_CS_FIELD;
  if ((L->feat & FEAT_LES) && a.van_driest && phi) {
    L->cs_cell.resize(L->ncells);
    for (int64_t c = 0; c < L->ncells; c++) {
      const double dmp = 1.0 - std::exp(-std::fabs(phi[c]) / a.van_driest_A);
      L->cs_cell[c] = a.les_cs * dmp * dmp;
    }
    L->feat |= FEAT_LES_CS_FIELD;
  }
  // workspace layout
  Layout &y = L->lay;
  const uint64_t sb = is_f64(L) ? 8 : (L->prm.storage == AERO_STORE_F32 ? 4 : 2);
  const uint64_t rb = is_f64(L) ? 8 : 4;
  const uint64_t nlc = L->lc_cell.size();
  uint64_t o = 0;
  auto take = [&](uint64_t bytes) {
    const uint64_t at = o;
    o = align_up(o + std::max<uint64_t>(bytes, 1));
    return at;
  };
  y.P[0] = take(sb * L->Q * L->cs);
  y.P[1] = take(L->aa ? 0 : sb * L->Q * L->cs);  // the AA layout has one buffer
  y.flags = take(L->cs + 32);  // slack for 16-byte-widened tile copies
  y.lbits = take(4 * L->nwords);
  y.loff = take(4 * L->nwords);
  y.lc_mask = take(4 * nlc);
  y.lc_q = take(4 * nlc * L->Q);
  y.lc_cell = take(8 * nlc);
  y.lc_contrib = take(96 * nlc);
  y.fin_partial = take(8 * 12 * (uint64_t)kFinalizeMaxBlocks);
  y.prof_off = take(4 * (L->nprof + 1));
  y.force_const = take(8 * 12);
  y.prof_const = take(24 * (uint64_t)L->nprof);
  y.prev[0] = take(rb * L->QP * L->prev_plane);
  y.prev[1] = take(rb * L->QP * L->prev_plane);
  y.g[0] = take(L->Qg ? rb * L->Qg * L->cs : 0);
  y.g[1] = take(L->Qg ? rb * L->Qg * L->cs : 0);
  y.U = take((L->feat & FEAT_LES) ? rb * 3 * L->cs : 0);
  y.cs_cell = take(L->cs_cell.empty() ? 0 : rb * L->cs);
  y.inflow = take((L->feat & FEAT_INFLOW_FIELD) ? rb * (uint64_t)L->inflow_ring * inflow_components(L) * L->prev_plane
                                                 : 0);
  y.recycle = take((L->feat & FEAT_RECYCLE) ? 8 * (uint64_t)(L->recycle_blocks + 2) : 0);
  y.hist = take(8 * 12 * (uint64_t)L->hist_cap);
  y.prof_out = take(24 * (uint64_t)L->nprof);
  y.counters = take(64);
  // k_field_stats: per-block partials, the combined values, the ticket
  y.stats = take(8 * ((uint64_t)kStatsBlocks * kStatsValues + kStatsValues + 1));
  // AA layout: the staged cross-cell reads of a step
  y.stage_link = take(L->aa ? rb * L->Q * nlc : 0);
  y.stage_nb = take((L->aa && (L->feat & FEAT_BOUZIDI)) ? rb * L->Q * nlc : 0);
  y.stage_out = take((L->aa && aa_stages_outlet(L)) ? rb * L->Q * (uint64_t)L->prev_plane : 0);
  // persistent runs: the odd steps' force terms and the two parameter sets
  y.lc_contrib2 = take(96 * nlc);
  y.run_params = take(2 * (is_f64(L) ? sizeof(StepParams<double>) : sizeof(StepParams<float>)));
  y.total = o;
  L->geometry = true;
  return AERO_OK;
}

int aero_workspace_size(const AeroLattice *L, uint64_t *bytes) {
  if (!L || !bytes) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->geometry) return fail(AERO_ERR_STATE, "aero_set_geometry must come first");
  *bytes = L->lay.total;
  return AERO_OK;
}

int aero_bind_workspace(AeroLattice *L, void *dptr, uint64_t bytes, void *stream) {
  if (!L || !dptr) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->geometry) return fail(AERO_ERR_STATE, "aero_set_geometry must come first");
  if (L->bound) return fail(AERO_ERR_STATE, "workspace already bound");
  if (bytes < L->lay.total) return fail(AERO_ERR_INVALID, "workspace too small: %llu < %llu",
                                        (unsigned long long)bytes, (unsigned long long)L->lay.total);
  if (reinterpret_cast<uintptr_t>(dptr) % kAlign) return fail(AERO_ERR_INVALID, "workspace must be 256-byte aligned");
  cudaPointerAttributes attr;
  CUDA_TRY(cudaPointerGetAttributes(&attr, dptr));
  if (attr.type != cudaMemoryTypeDevice) return fail(AERO_ERR_INVALID, "workspace is not device memory");
  L->device = attr.device;
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  L->ws = static_cast<char *>(dptr);
  auto up = [&](uint64_t off, const void *src, uint64_t n) -> cudaError_t {
    if (n == 0) return cudaSuccess;
    return cudaMemcpyAsync(L->ws + off, src, n, cudaMemcpyHostToDevice, st);
  };
  CUDA_TRY(cudaMemsetAsync(L->ws, 0, L->lay.total, st));
  // first divergent step starts at "never"
  CUDA_TRY(cudaMemsetAsync(L->ws + L->lay.counters + 3 * sizeof(int64_t), 0xff, sizeof(int64_t), st));
  // per-cell flags: solid, and whether the cell has obstacle links
  std::vector<uint8_t> flags(L->solid);
  for (const int64_t c : L->lc_cell) flags[(size_t)c] |= FLAG_LINK;
  CUDA_TRY(up(L->lay.flags, flags.data(), flags.size()));
  CUDA_TRY(up(L->lay.lbits, L->lbits.data(), 4 * L->lbits.size()));
  CUDA_TRY(up(L->lay.loff, L->loff.data(), 4 * L->loff.size()));
  CUDA_TRY(up(L->lay.lc_mask, L->lc_mask.data(), 4 * L->lc_mask.size()));
  CUDA_TRY(up(L->lay.lc_q, L->lc_q.data(), 4 * L->lc_q.size()));
  CUDA_TRY(up(L->lay.lc_cell, L->lc_cell.data(), 8 * L->lc_cell.size()));
  CUDA_TRY(up(L->lay.prof_off, L->prof_off.data(), 4 * L->prof_off.size()));
  CUDA_TRY(up(L->lay.force_const, L->force_const.data(), 8 * L->force_const.size()));
  CUDA_TRY(up(L->lay.prof_const, L->prof_const.data(), 8 * L->prof_const.size()));
  if (!L->cs_cell.empty()) {
    if (is_f64(L)) {
      CUDA_TRY(up(L->lay.cs_cell, L->cs_cell.data(), 8 * L->cs_cell.size()));
    } else {
      std::vector<float> tmp(L->cs_cell.begin(), L->cs_cell.end());
      CUDA_TRY(up(L->lay.cs_cell, tmp.data(), 4 * tmp.size()));
      CUDA_TRY(cudaStreamSynchronize(st));  // tmp goes out of scope
    }
  }
  // host vectors must outlive the async copies
  CUDA_TRY(cudaStreamSynchronize(st));
  const int rc = is_f64(L) ? plan_tiles<double>(L) : plan_tiles<float>(L);
  if (rc != AERO_OK) return rc;
  // Test of the bounded waits of the row-tiled kernel: every stage announces
  // 16 bytes more than its copies deliver, so no stage completes; the waits
  // give up after their limit, raise status bit 1 and the kernel returns.
  const char *stall = std::getenv("AERO_B200_TEST_STALL_TILES");
  L->tile_extra_tx = (stall && stall[0] == '1') ? 16u : 0u;
  // Test of the bounded barrier of persistent runs: cell block 1 leaves
  // before its first barrier, so the others' waits give up after their limit.
  const char *rstall = std::getenv("AERO_B200_TEST_STALL_RUN");
  L->run_stall_block = (rstall && rstall[0] == '1') ? 1 : -1;
  const char *gen = std::getenv("AERO_B200_GENERIC_KERNELS");
  L->generic_kernels = gen && gen[0] == '1';
  L->bound = true;
  return AERO_OK;
}

int aero_set_state(AeroLattice *L, const double *f, const double *prev, const double *g, int64_t steps,
                   void *stream) {
  if (!L || !f) return fail(AERO_ERR_INVALID, "NULL argument");
  if (L->batch) return fail(AERO_ERR_STATE, "the lattice is a batch member; remove it from the batch first");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  if (steps < 0) return fail(AERO_ERR_INVALID, "negative step count");
  if (!L->state_set && !prev && (L->prm.outlet_bc == AERO_OUTLET_CONVECTIVE))
    return fail(AERO_ERR_INVALID, "the first state must include f_outlet_prev");
  if (!L->state_set && !g && L->prm.thermal) return fail(AERO_ERR_INVALID, "the first state must include g");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return is_f64(L) ? do_set_state<double>(L, f, prev, g, steps, st) : do_set_state<float>(L, f, prev, g, steps, st);
}

int aero_set_equilibrium(AeroLattice *L, const double *rho, const double *ux, const double *uy, const double *uz,
                         const double *T, int64_t steps, void *stream) {
  if (!L) return fail(AERO_ERR_INVALID, "NULL argument");
  if (L->batch) return fail(AERO_ERR_STATE, "the lattice is a batch member; remove it from the batch first");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  if (steps < 0) return fail(AERO_ERR_INVALID, "negative step count");
  if (uz && L->prm.dims != 3) return fail(AERO_ERR_INVALID, "uz is a 3D field");
  if (T && !L->prm.thermal) return fail(AERO_ERR_INVALID, "T needs a lattice with a scalar");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const EqFields e{rho, ux, uy, uz, T, L->prm.rho0, L->prm.u0, L->prm.T_ref};
  return is_f64(L) ? do_set_equilibrium<double>(L, e, steps, st) : do_set_equilibrium<float>(L, e, steps, st);
}

int aero_get_state(AeroLattice *L, double *f, double *prev, double *g, void *stream) {
  if (!L) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->state_set) return fail(AERO_ERR_STATE, "no state set");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return is_f64(L) ? do_get_state<double>(L, f, prev, g, 0, L->prm.nz, st)
                    : do_get_state<float>(L, f, prev, g, 0, L->prm.nz, st);
}

int aero_get_state_slab(AeroLattice *L, int32_t z0, int32_t nzs, double *f, void *stream) {
  if (!L || !f) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->state_set) return fail(AERO_ERR_STATE, "no state set");
  if (z0 < 0 || nzs < 1 || z0 + nzs > L->prm.nz) return fail(AERO_ERR_INVALID, "slab outside the grid");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return is_f64(L) ? do_get_state<double>(L, f, nullptr, nullptr, z0, nzs, st)
                    : do_get_state<float>(L, f, nullptr, nullptr, z0, nzs, st);
}

int aero_get_macroscopic(AeroLattice *L, double *out, void *stream) {
  if (!L || !out) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->state_set) return fail(AERO_ERR_STATE, "no state set");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 grid = cell_grid(L);
  bool raw = false;
  if (is_f64(L)) {
    const StepParams<double> p = reader_params<double>(L, &raw);
    CUDA_TRY(get_ops<double>(L)->macro_out(p, out, -1, raw, 0, grid, st));
  } else {
    const StepParams<float> p = reader_params<float>(L, &raw);
    CUDA_TRY(get_ops<float>(L)->macro_out(p, out, -1, raw, 0, grid, st));
  }
  return AERO_OK;
}

int aero_field_stats(AeroLattice *L, int32_t z0, int32_t nzs, double *out, void *stream) {
  if (!L || !out) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->state_set) return fail(AERO_ERR_STATE, "no state set");
  if (z0 < 0 || nzs < 1 || z0 + nzs > L->prm.nz) return fail(AERO_ERR_INVALID, "planes outside the grid");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double *partial = reinterpret_cast<double *>(L->ws + L->lay.stats);
  double *dout = partial + (size_t)kStatsBlocks * kStatsValues;
  uint32_t *ticket = reinterpret_cast<uint32_t *>(dout + kStatsValues);
  // the state of the last step comes from the previous buffers (as in
  // aero_get_macroscopic); the scalar of the last step is the current one
  bool raw = false;
  if (is_f64(L)) {
    const StepParams<double> p = reader_params<double>(L, &raw);
    const double *g = L->prm.thermal ? reinterpret_cast<const double *>(L->ws + L->lay.g[L->cur]) : nullptr;
    CUDA_TRY(get_ops<double>(L)->field_stats(p, g, z0, nzs, -1, raw, partial, ticket, dout, st));
  } else {
    const StepParams<float> p = reader_params<float>(L, &raw);
    const float *g = L->prm.thermal ? reinterpret_cast<const float *>(L->ws + L->lay.g[L->cur]) : nullptr;
    CUDA_TRY(get_ops<float>(L)->field_stats(p, g, z0, nzs, -1, raw, partial, ticket, dout, st));
  }
  CUDA_TRY(cudaMemcpyAsync(out, dout, sizeof(double) * kStatsValues, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return AERO_OK;
}

int aero_params_size(void) { return (int)sizeof(AeroParams); }

int aero_enable_timing(AeroLattice *L, int32_t on) {
  if (!L) return fail(AERO_ERR_INVALID, "NULL argument");
  L->timing = on != 0;
  return AERO_OK;
}

int aero_kernel_times(AeroLattice *L, double *step_ms, double *forces_ms, int64_t *steps, void *stream) {
  if (!L || !step_ms || !forces_ms || !steps) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  CUDA_TRY(cudaSetDevice(L->device));
  CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  double a = 0.0, b = 0.0;
  for (int64_t k = 0; k < L->timed_steps; k++) {
    float t0 = 0.f, t1 = 0.f;
    cudaEvent_t *e = &L->ev[3 * (size_t)k];
    CUDA_TRY(cudaEventElapsedTime(&t0, e[0], e[1]));
    CUDA_TRY(cudaEventElapsedTime(&t1, e[1], e[2]));
    a += t0;
    b += t1;
  }
  *step_ms = a;
  *forces_ms = b;
  *steps = L->timed_steps;
  L->timed_steps = 0;
  return AERO_OK;
}

int aero_step(AeroLattice *L, int64_t n, void *stream) {
  if (!L) return fail(AERO_ERR_INVALID, "NULL argument");
  if (L->batch) return fail(AERO_ERR_STATE, "the lattice is a batch member; it advances with aero_batch_step");
  if (!L->state_set) return fail(AERO_ERR_STATE, "aero_set_state must come first");
  if (n < 0) return fail(AERO_ERR_INVALID, "negative step count");
  if (L->step_count + n - L->read_upto > L->hist_cap)
    return fail(AERO_ERR_CAPACITY, "force history holds %d steps; read it before stepping further", L->hist_cap);
  if ((L->feat & FEAT_INFLOW_FIELD) && L->step_count + n > L->inflow_upto)
    return fail(AERO_ERR_STATE, "inflow fields are on the device up to step %lld; upload them with aero_set_inflow",
                (long long)L->inflow_upto);
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) return AERO_OK;
  // only the last step's force profile can be read (aero_read_profile), so
  // only that step sums it
  int64_t *ctr = reinterpret_cast<int64_t *>(L->ws + L->lay.counters);
  k_set_i64<<<1, 1, 0, st>>>(ctr + 4, L->step_count + n);
  CUDA_TRY(cudaGetLastError());
  return is_f64(L) ? do_steps<double>(L, n, st) : do_steps<float>(L, n, st);
}

int aero_read_forces(AeroLattice *L, double *out, int64_t max_steps, int64_t *n_out, void *stream) {
  if (!L || !out || !n_out) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = std::min(L->step_count - L->read_upto, max_steps);
  const double *hist = reinterpret_cast<const double *>(L->ws + L->lay.hist);
  int64_t done = 0;
  while (done < n) {
    const int64_t slot = (L->read_upto + done) % L->hist_cap;
    const int64_t run = std::min(n - done, (int64_t)L->hist_cap - slot);
    CUDA_TRY(cudaMemcpyAsync(out + done * 12, hist + slot * 12, sizeof(double) * 12 * run, cudaMemcpyDeviceToHost, st));
    done += run;
  }
  CUDA_TRY(cudaStreamSynchronize(st));
  L->read_upto += n;
  *n_out = n;
  return AERO_OK;
}

int aero_read_profile(AeroLattice *L, double *out, void *stream) {
  if (!L || !out) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemcpyAsync(out, L->ws + L->lay.prof_out, 24 * (size_t)L->nprof, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return AERO_OK;
}

int aero_status(AeroLattice *L, uint32_t *status, void *stream) {
  if (!L || !status) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t *ctr = reinterpret_cast<const int64_t *>(L->ws + L->lay.counters);
  CUDA_TRY(cudaMemcpyAsync(status, ctr + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return AERO_OK;
}

int aero_first_bad_step(AeroLattice *L, int64_t *step, void *stream) {
  if (!L || !step) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned long long v = 0;
  CUDA_TRY(cudaMemcpyAsync(&v, L->ws + L->lay.counters + 3 * sizeof(int64_t), sizeof(v), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  *step = v == ~0ull ? -1 : (int64_t)v;
  return AERO_OK;
}

int aero_step_count(const AeroLattice *L, int64_t *steps) {
  if (!L || !steps) return fail(AERO_ERR_INVALID, "NULL argument");
  *steps = L->step_count;
  return AERO_OK;
}

int aero_set_inflow(AeroLattice *L, const double *fields, int64_t first, int64_t n, void *stream) {
  if (!L || (n > 0 && !fields)) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  if (!(L->feat & FEAT_INFLOW_FIELD)) return fail(AERO_ERR_STATE, "the lattice has no inflow field inlet");
  if (n < 0 || first < L->step_count) return fail(AERO_ERR_INVALID, "fields for steps already taken, or n < 0");
  if (first > L->inflow_upto) return fail(AERO_ERR_INVALID, "inflow fields must be uploaded without gaps");
  if (first + n - L->step_count > L->inflow_ring)
    return fail(AERO_ERR_CAPACITY, "the device holds inflow fields for %d steps ahead", L->inflow_ring);
  if (n == 0) return AERO_OK;
  CUDA_TRY(cudaSetDevice(L->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t per = (int64_t)inflow_components(L) * L->prev_plane;  // values per step
  const size_t rb = is_f64(L) ? 8 : 4;
  std::vector<char> host((size_t)(per * n) * rb);
  for (int64_t k = 0; k < per * n; k++) {
    if (rb == 8) reinterpret_cast<double *>(host.data())[k] = fields[k];
    else reinterpret_cast<float *>(host.data())[k] = (float)fields[k];
  }
  char *ring = L->ws + L->lay.inflow;
  for (int64_t k = 0; k < n; k++) {
    const int64_t slot = (first + k) % L->inflow_ring;
    CUDA_TRY(cudaMemcpyAsync(ring + (size_t)(slot * per) * rb, host.data() + (size_t)(k * per) * rb,
                             (size_t)per * rb, cudaMemcpyHostToDevice, st));
  }
  CUDA_TRY(cudaStreamSynchronize(st));  // the staging vector goes out of scope
  L->inflow_upto = std::max(L->inflow_upto, first + n);
  return AERO_OK;
}

int aero_set_step_kernel(AeroLattice *L, int32_t kernel) {
  if (!L) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  if (kernel < 0 || kernel > kStepLes) return fail(AERO_ERR_INVALID, "kernel must be 0..%d", kStepLes);
  if (L->aa && kernel != 0)
    return fail(AERO_ERR_UNSUPPORTED, "the AA layout runs the per-cell step kernel (0) only");
  CUDA_TRY(cudaSetDevice(L->device));
  if (kernel == kStepPair) {
    if (!pair_capable(L, 2))
      return fail(AERO_ERR_UNSUPPORTED,
                  "the two-cell kernel covers D3Q19 with 4- or 2-byte storage, even nx, no body force or scalar "
                  "lattice");
    if (((int64_t)L->prm.ny * L->prm.nz + 31) / 32 > 65535)
      return fail(AERO_ERR_UNSUPPORTED, "the two-cell kernel takes at most 65535 * 32 rows (ny * nz)");
  }
  if (kernel == kStepQuad) {
    if (!quad_capable(L))
      return fail(AERO_ERR_UNSUPPORTED,
                  "the four-cell kernel covers D3Q19 with 16-bit storage, nx a multiple of 4 (>= 12 with an open "
                  "inlet), no body force or scalar lattice");
    if (((int64_t)L->prm.ny * L->prm.nz + kQuadRows - 1) / kQuadRows * ((L->prm.nx / 4 + 127) / 128 * 16 + 1) >=
        ((int64_t)1 << 31))
      return fail(AERO_ERR_UNSUPPORTED, "the four-cell kernel's grid exceeds 2^31 blocks");
  }
  int les_chunk = 0;
  if (kernel == kStepLes) {
    if (!(L->prm.dims == 3 && L->prm.collision != AERO_MRT && les_active(L)))
      return fail(AERO_ERR_UNSUPPORTED, "the fused LES kernel covers D3Q19 BGK / TRT lattices with LES");
    const cudaError_t e =
        is_f64(L) ? get_ops<double>(L)->les_setup() : get_ops<float>(L)->les_setup();
    if (e != cudaSuccess) return fail(AERO_ERR_CUDA, "fused LES kernel set-up: %s", cudaGetErrorString(e));
    // z chunks so that the grid holds about six blocks per SM; at least 8
    // planes a chunk, since each chunk evaluates two planes beyond it
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, L->device));
    const int64_t tiles = (int64_t)((L->prm.nx + kLesTileX - 1) / kLesTileX) * ((L->prm.ny + kLesRows - 1) / kLesRows);
    const int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(L->prm.nz, (6LL * sms + tiles - 1) / tiles));
    les_chunk = (int)((L->prm.nz + chunks - 1) / chunks);
    les_chunk = std::max(les_chunk, std::min(8, L->prm.nz));
  }
  if (kernel == kStepShapes) {
    const int rc = is_f64(L) ? plan_tiles<double>(L, true) : plan_tiles<float>(L, true);
    if (rc != AERO_OK) return rc;
    if (!L->tiled) return fail(AERO_ERR_UNSUPPORTED, "rows of this lattice do not fit the row-tiled kernel");
    L->pair = L->quad = L->les_fused = false;
  } else {
    L->tiled = false;
    L->tile_blocks = L->tile_rows = L->tiles_per_plane = L->ntiles = 0;
    L->pair = kernel == kStepPair;
    L->quad = kernel == kStepQuad;
    L->les_fused = kernel == kStepLes;
    L->les_chunk = les_chunk;
    L->step_shape = (L->pair || L->quad || L->les_fused) ? 0 : kernel;
  }
  // captured step sequences launch the previous kernel
  for (auto &e : L->pair_exec)
    if (e) {
      cudaGraphExecDestroy(e);
      e = nullptr;
    }
  return AERO_OK;
}

int aero_set_persistent(AeroLattice *L, int32_t enable) {
  if (!L) return fail(AERO_ERR_INVALID, "NULL argument");
  L->persistent = enable != 0;
  return AERO_OK;
}

int aero_kernel_variant(const AeroLattice *L, int32_t *variant) {
  if (!L || !variant) return fail(AERO_ERR_INVALID, "NULL argument");
  *variant = kernel_variant(L);
  return AERO_OK;
}

int aero_get_persistent(const AeroLattice *L, int32_t *active) {
  if (!L || !active) return fail(AERO_ERR_INVALID, "NULL argument");
  *active = run_small_ok(L) ? 1 : 0;
  return AERO_OK;
}

int aero_get_step_kernel(const AeroLattice *L, int32_t *kernel) {
  if (!L || !kernel) return fail(AERO_ERR_INVALID, "NULL argument");
  *kernel = L->tiled ? kStepShapes
                    : (L->pair ? kStepPair : (L->quad ? kStepQuad : (L->les_fused ? kStepLes : L->step_shape)));
  return AERO_OK;
}

int aero_step_plan(const AeroLattice *L, int32_t *tiled, int32_t *tile_rows, int32_t *blocks) {
  if (!L) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!L->bound) return fail(AERO_ERR_STATE, "workspace not bound");
  if (tiled) *tiled = L->tiled ? 1 : 0;
  if (tile_rows) *tile_rows = L->tile_rows;
  if (blocks) *blocks = L->tile_blocks;
  return AERO_OK;
}

int aero_destroy(AeroLattice *L) {
  if (!L) return AERO_OK;
  if (L->batch) return fail(AERO_ERR_STATE, "the lattice is a batch member; remove it from the batch first");
  for (auto &e : L->pair_exec)
    if (e) cudaGraphExecDestroy(e);
  if (L->cap_stream) cudaStreamDestroy(L->cap_stream);
  for (auto e : L->ev) cudaEventDestroy(e);
  delete L;
  return AERO_OK;
}

int aero_collide_host(const AeroParams *a, const double *f_in, double *f_out, const uint8_t *solid, int64_t n) {
  const int rc = check_params(a);
  if (rc != AERO_OK) return rc;
  if (!f_in || !f_out || n < 0) return fail(AERO_ERR_INVALID, "bad argument");
  AeroLattice *L = nullptr;
  const int rc2 = aero_create(a, &L);
  if (rc2 != AERO_OK) return rc2;
  StepParams<double> p = make_params<double>(L, 0);
  const int Q = L->Q;
  for (int64_t c = 0; c < n; c++) {
    double d[19];
    for (int i = 0; i < Q; i++) d[i] = f_in[i * n + c] - L->w.w[i];
    const bool sol = solid && solid[c];
    if (a->dims == 2) {
      double (&dd)[9] = *reinterpret_cast<double (*)[9]>(d);
      switch (a->collision) {
        case AERO_BGK: collide<D2Q9, double, COLL_BGK>(p, dd, sol, p.omega, false); break;
        case AERO_TRT: collide<D2Q9, double, COLL_TRT>(p, dd, sol, p.omega, false); break;
        default: collide<D2Q9, double, COLL_MRT>(p, dd, sol, p.omega, false); break;
      }
    } else {
      switch (a->collision) {
        case AERO_BGK: collide<D3Q19, double, COLL_BGK>(p, d, sol, p.omega, false); break;
        case AERO_TRT: collide<D3Q19, double, COLL_TRT>(p, d, sol, p.omega, false); break;
        default: collide<D3Q19, double, COLL_MRT>(p, d, sol, p.omega, false); break;
      }
    }
    for (int i = 0; i < Q; i++) f_out[i * n + c] = L->w.w[i] + d[i];
  }
  aero_destroy(L);
  return AERO_OK;
}

int aero_mrt_operator(int32_t dims, double omega, double *A, double *B) {
  if ((dims != 2 && dims != 3) || !A || !B) return fail(AERO_ERR_INVALID, "bad argument");
  MrtCoeffs<double> tmp;
  if (!build_mrt(dims, omega, tmp, A, B)) return fail(AERO_ERR_INVALID, "MRT operator not block diagonal");
  return AERO_OK;
}

}  // extern "C"

// ==========================================================================
// Batches: many lattices advanced together, one launch per lattice class
// (dimensions, storage, collision) and per step kernel (moments pass, step,
// force finalisation).  The batch owns no device memory either: the caller
// binds a workspace for its plan (parameter arrays, block prefixes, the
// convergence items and results).
// ==========================================================================
namespace {

// Rolling convergence of the drag coefficient on the device, with the rule
// of analyze_convergence (diagnostics.py:87-120): over the last `window`
// steps of Cd = Fx / cd_norm, ratio = std / mean|Cd| (population std);
// converged when ratio < tol, or when mean|Cd| < 1e-12.  One block per
// lattice; out receives (ratio, mean|Cd|, std, converged, steps, status,
// mean Cd) doubles, with ratio = +inf and converged = 0 while fewer than
// `window` steps are in the ring.  status is the lattice's device status word.
constexpr int kConvergeValues = AERO_CONVERGE_VALUES;

struct ConvergeItem {
  const double *hist;
  const int64_t *step;
  const int64_t *hist_base;
  const uint32_t *status;
  double *out;
  double cd_norm;
  int32_t hist_cap;
};

__global__ void __launch_bounds__(kFinalizeBlock) k_converge(const ConvergeItem *__restrict__ items, int n, int W,
                                                              double tol) {
  __shared__ double red[3][kFinalizeBlock / 32];
  if ((int)blockIdx.x >= n) return;
  const ConvergeItem it = items[blockIdx.x];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int64_t steps = *it.step, hb = *it.hist_base;
  if (steps - hb < W || W > it.hist_cap || W < 1) {
    if (t == 0) {
      it.out[0] = __longlong_as_double(0x7ff0000000000000ll);  // +inf
      it.out[1] = 0.0;
      it.out[2] = 0.0;
      it.out[3] = 0.0;
      it.out[4] = (double)steps;
      it.out[5] = (double)*it.status;
      it.out[6] = 0.0;
    }
    return;
  }
  auto block_sum = [&](double v, int j) -> double {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[j][wid] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kFinalizeBlock / 32; w++) s += red[j][w];
    __syncthreads();
    return s;
  };
  double sa = 0.0, sv = 0.0;
  for (int k = t; k < W; k += kFinalizeBlock) {
    const int64_t slot = (steps - W + k - hb) % it.hist_cap;
    const double cd = it.hist[slot * 12] / it.cd_norm;
    sa += fabs(cd);
    sv += cd;
  }
  const double mean_abs = block_sum(sa, 0) / W;
  const double mean = block_sum(sv, 1) / W;
  double sq = 0.0;
  for (int k = t; k < W; k += kFinalizeBlock) {
    const int64_t slot = (steps - W + k - hb) % it.hist_cap;
    const double dv = it.hist[slot * 12] / it.cd_norm - mean;
    sq += dv * dv;
  }
  const double sd = sqrt(block_sum(sq, 2) / W);
  if (t == 0) {
    const bool tiny = mean_abs < 1e-12;
    const double ratio = tiny ? 0.0 : sd / mean_abs;
    it.out[0] = ratio;
    it.out[1] = mean_abs;
    it.out[2] = sd;
    it.out[3] = (tiny || ratio < tol) ? 1.0 : 0.0;
    it.out[4] = (double)steps;
    it.out[5] = (double)*it.status;
    it.out[6] = mean;
  }
}


__global__ void k_set_profile_steps(int64_t *const *ctrs, int n, int64_t delta) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) ctrs[k][4] = ctrs[k][0] + delta;  // profile_step = step + delta
}

struct ClassKey {
  int dims, storage, coll;
  bool pair;    // the members take the two-cells-per-thread layout (k_step_batch_pair)
  int variant;  // the compiled kernel set (kernel_variant)
  bool operator==(const ClassKey &o) const {
    return dims == o.dims && storage == o.storage && coll == o.coll && pair == o.pair && variant == o.variant;
  }
};

struct ClassPlan {
  ClassKey key;
  bool f64;
  const Ops<float> *ops = nullptr;  // the class's kernel table (4- and 2-byte storage)
  int n = 0, n_les = 0;
  int64_t blocks = 0, blocks_les = 0;
  uint64_t params[2] = {0, 0}, first = 0, params_les[2] = {0, 0}, first_les = 0;
  // members with a recycling inlet and their parity at the build: each step
  // launches their plane-mean pass (k_recycle_mean) before the class kernels
  std::vector<std::pair<AeroLattice *, int>> recycle;
};

struct FinPlan {
  int n = 0;
  int64_t blocks = 0;
  uint64_t params[2] = {0, 0}, first = 0;
};

// Members at least this large fill the GPU on their own: they step through
// their single-lattice kernels (the step kernel their autotuning chose, their
// own force finalisation) as branches of the batch graph, which is faster per
// cell than the class kernels' member lookup and parameter copy.  Smaller
// members share the class kernels.
constexpr int64_t kBatchSoloCells = (int64_t)1 << 20;

bool batch_solo(const AeroLattice *L) { return L->ncells >= kBatchSoloCells; }

// In a batch the two-cell kernel runs for 16-bit storage only: measured on
// the 96-case sweep it is 5% faster there and 9% slower with FP32 storage,
// where the per-cell kernel's traffic, not its instructions, sets the pace.
ClassKey class_of(const AeroLattice *L) {
  const bool half = L->prm.storage == AERO_STORE_F16 || L->prm.storage == AERO_STORE_BF16;
  return {L->prm.dims, L->prm.storage, L->prm.collision, half && pair_capable(L, 6), kernel_variant(L)};
}

}  // namespace

struct AeroBatch {
  int max_members = 0;
  std::vector<AeroLattice *> members;
  int device = -1;
  char *ws = nullptr;
  uint64_t ws_bytes = 0;
  bool bound = false, dirty = true;
  int phase = 0;  // parity of the steps taken since the plan was built
  // plan (device offsets into ws)
  std::vector<ClassPlan> classes;
  FinPlan fin[2];  // [0] float members, [1] double members
  std::vector<AeroLattice *> solo;  // members stepped by their own kernels
  std::vector<int> solo_cur;        // their buffer parity when the plan was built
  uint64_t ctr_ptrs = 0, conv_items = 0, conv_out = 0;
  std::vector<char> host_plan;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [steps - 1][phase]
  // branch streams and events of a captured step: the lattice classes run
  // as parallel branches of the graph, joined before the force finalisation
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> branch_done;
  cudaEvent_t fork = nullptr;
};

namespace {

void batch_drop_graphs(AeroBatch *B) {
  for (auto &row : B->graph)
    for (auto &g : row)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
}

uint64_t batch_bytes(int max_members) {
  // Upper bound of batch_build's plan: every member in the step, LES and
  // finalisation lists with the largest parameter block (two parities plus
  // a block prefix each); the one-entry minimum of the LES lists of up to
  // 24 classes and of the two finalisation lists; counters pointers,
  // convergence items and results; 256-byte alignment of every array.
  const uint64_t m = (uint64_t)std::max(max_members, 1);
  const uint64_t sp = sizeof(StepParams<double>);
  const uint64_t kClasses = 2 * 4 * 3 * 2;
  uint64_t b = 3 * m * (2 * sp + 8);
  b += (kClasses + 2) * (2 * sp + 8);
  b += m * (8 + sizeof(ConvergeItem) + kConvergeValues * 8);
  b += kAlign * (6 * kClasses + 6 + 3 + 1);
  return align_up(b);
}

template <class Real>
void put_params(std::vector<char> &buf, uint64_t off, const AeroLattice *L, int parity) {
  const StepParams<Real> p = make_params<Real>(L, parity);
  std::memcpy(buf.data() + off, &p, sizeof(p));
}

// Builds the plan for the current members on the host and uploads it.  The
// parameter array used by step j of a graph is [(phase + j) % 2], and holds
// each member's buffers for its own parity at that step.
int batch_build(AeroBatch *B, cudaStream_t st) {
  B->classes.clear();
  B->fin[0] = FinPlan{};
  B->fin[1] = FinPlan{};
  B->solo.clear();
  B->solo_cur.clear();
  for (AeroLattice *L : B->members) {
    if (batch_solo(L)) {
      B->solo.push_back(L);
      B->solo_cur.push_back(L->cur);
      continue;
    }
    const ClassKey k = class_of(L);
    auto it = std::find_if(B->classes.begin(), B->classes.end(), [&](const ClassPlan &c) { return c.key == k; });
    if (it == B->classes.end()) {
      ClassPlan c;
      c.key = k;
      c.f64 = is_f64(L);
      if (!c.f64) c.ops = get_ops<float>(L);  // the same for every member: the key holds the variant
      B->classes.push_back(c);
      it = B->classes.end() - 1;
    }
    it->n++;
    if (les_active(L)) it->n_les++;
    if (L->feat & FEAT_RECYCLE) it->recycle.emplace_back(L, L->cur);
    B->fin[is_f64(L) ? 1 : 0].n++;
  }
  std::vector<char> &h = B->host_plan;
  h.assign(B->ws_bytes, 0);
  uint64_t o = 0;
  auto take = [&](uint64_t bytes) {
    const uint64_t at = o;
    o = align_up(o + std::max<uint64_t>(bytes, 1));
    return at;
  };
  auto cell_blocks = [](const AeroLattice *L) {
    const int64_t R = L->ncells < kBatchSmallCells ? 1 : kBatchRows;  // as make_params' batch_rows
    const int64_t per_block = R * kStepBlock;                          // consecutive cells of a block
    return (L->ncells + per_block - 1) / per_block;
  };
  auto step_blocks = [&](const AeroLattice *L, bool pair) {
    if (!pair) return cell_blocks(L);
    const PairBatchLayout lay = pair_batch_layout(L->prm.nx, L->prm.ny, L->prm.nz);
    return lay.pair_blocks + lay.edge_blocks;
  };
  for (ClassPlan &c : B->classes) {
    const uint64_t sp = c.f64 ? sizeof(StepParams<double>) : sizeof(StepParams<float>);
    c.params[0] = take(sp * c.n);
    c.params[1] = take(sp * c.n);
    c.first = take(8 * (uint64_t)c.n);
    c.params_les[0] = take(sp * std::max(c.n_les, 1));
    c.params_les[1] = take(sp * std::max(c.n_les, 1));
    c.first_les = take(8 * (uint64_t)std::max(c.n_les, 1));
    int k = 0, kl = 0;
    int64_t blocks = 0, blocks_les = 0;
    for (AeroLattice *L : B->members) {
      if (batch_solo(L) || !(class_of(L) == c.key)) continue;
      for (int j = 0; j < 2; j++) {
        const int par = (L->cur + j) & 1;  // parity at steps with (phase + j') % 2 == j, phase = 0 after a build
        if (c.f64) put_params<double>(h, c.params[j] + sp * k, L, par);
        else put_params<float>(h, c.params[j] + sp * k, L, par);
      }
      std::memcpy(h.data() + c.first + 8 * k, &blocks, 8);
      blocks += step_blocks(L, c.key.pair);
      k++;
      if (les_active(L)) {
        for (int j = 0; j < 2; j++) {
          const int par = (L->cur + j) & 1;
          if (c.f64) put_params<double>(h, c.params_les[j] + sp * kl, L, par);
          else put_params<float>(h, c.params_les[j] + sp * kl, L, par);
        }
        std::memcpy(h.data() + c.first_les + 8 * kl, &blocks_les, 8);
        blocks_les += cell_blocks(L);
        kl++;
      }
    }
    c.blocks = blocks;
    c.blocks_les = blocks_les;
  }
  for (int r = 0; r < 2; r++) {
    FinPlan &f = B->fin[r];
    const uint64_t sp = r ? sizeof(StepParams<double>) : sizeof(StepParams<float>);
    f.params[0] = take(sp * std::max(f.n, 1));
    f.params[1] = take(sp * std::max(f.n, 1));
    f.first = take(8 * (uint64_t)std::max(f.n, 1));
    int k = 0;
    int64_t blocks = 0;
    for (AeroLattice *L : B->members) {
      if (batch_solo(L) || (is_f64(L) ? 1 : 0) != r) continue;
      for (int j = 0; j < 2; j++) {
        const int par = (L->cur + j) & 1;
        if (r) put_params<double>(h, f.params[j] + sp * k, L, par);
        else put_params<float>(h, f.params[j] + sp * k, L, par);
      }
      std::memcpy(h.data() + f.first + 8 * k, &blocks, 8);
      blocks += r ? make_params<double>(L, L->cur).fin_blocks : make_params<float>(L, L->cur).fin_blocks;
      k++;
    }
    f.blocks = blocks;
  }
  const int n = (int)B->members.size();
  B->ctr_ptrs = take(8 * (uint64_t)std::max(n, 1));
  B->conv_items = take(sizeof(ConvergeItem) * std::max(n, 1));
  B->conv_out = take(kConvergeValues * 8 * (uint64_t)std::max(n, 1));
  if (o > B->ws_bytes) return fail(AERO_ERR_CAPACITY, "batch plan needs %llu bytes, workspace has %llu",
                                   (unsigned long long)o, (unsigned long long)B->ws_bytes);
  for (int k = 0; k < n; k++) {
    AeroLattice *L = B->members[k];
    int64_t *ctr = reinterpret_cast<int64_t *>(L->ws + L->lay.counters);
    std::memcpy(h.data() + B->ctr_ptrs + 8 * k, &ctr, 8);
    ConvergeItem ci;
    ci.hist = reinterpret_cast<const double *>(L->ws + L->lay.hist);
    ci.step = ctr;
    ci.hist_base = ctr + 1;
    ci.status = reinterpret_cast<const uint32_t *>(ctr + 2);
    ci.out = reinterpret_cast<double *>(B->ws + B->conv_out) + kConvergeValues * k;
    ci.cd_norm = L->cd_norm;
    ci.hist_cap = L->hist_cap;
    std::memcpy(h.data() + B->conv_items + sizeof(ConvergeItem) * k, &ci, sizeof(ci));
  }
  // pageable source: the call returns once the data is staged, so the host
  // plan may be rebuilt afterwards
  CUDA_TRY(cudaMemcpyAsync(B->ws, h.data(), o, cudaMemcpyHostToDevice, st));
  batch_drop_graphs(B);
  B->phase = 0;
  B->dirty = false;
  return AERO_OK;
}

// Launches one step of every member; `j` selects the parameter arrays.
// With `branches`, every lattice class runs on its own stream forked from st
// and joined back before the finalisation (during capture this makes the
// classes parallel branches of the graph: they touch disjoint lattices).
// `aa_store`: the call's last step, where members in the AA layout store
// their post-boundary state instead of colliding it.
int batch_launch_step(AeroBatch *B, int j, cudaStream_t st, bool branches = false, bool aa_store = false) {
  char *ws = B->ws;
  const size_t nbranch = B->classes.size() + B->solo.size();
  if (branches) {
    while (B->branch.size() < nbranch) {
      cudaStream_t bs;
      cudaEvent_t ev;
      CUDA_TRY(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
      CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      B->branch.push_back(bs);
      B->branch_done.push_back(ev);
    }
    if (!B->fork) CUDA_TRY(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(B->fork, st));
  }
  for (size_t ci = 0; ci < B->classes.size(); ci++) {
    const ClassPlan &c = B->classes[ci];
    cudaStream_t cs = st;
    if (branches) {
      cs = B->branch[ci];
      CUDA_TRY(cudaStreamWaitEvent(cs, B->fork, 0));
    }
    // the recycling members' plane means, as aero_step launches them
    for (const auto &rm : c.recycle) {
      const int par = (rm.second + j) & 1;
      if (c.f64) CUDA_TRY(ops_f64(c.key.dims, c.key.coll)->recycle_mean(make_params<double>(rm.first, par), cs));
      else CUDA_TRY(c.ops->recycle_mean(make_params<float>(rm.first, par), cs));
    }
    if (c.f64) {
      const Ops<double> *ops = ops_f64(c.key.dims, c.key.coll);
      auto *P = reinterpret_cast<const StepParams<double> *>(ws + c.params[j]);
      auto *PL = reinterpret_cast<const StepParams<double> *>(ws + c.params_les[j]);
      if (c.n_les) CUDA_TRY(ops->moments_batch(PL, reinterpret_cast<const int64_t *>(ws + c.first_les), c.n_les,
                                               c.blocks_les, cs));
      CUDA_TRY(ops->step_batch(P, reinterpret_cast<const int64_t *>(ws + c.first), c.n, c.blocks, cs));
    } else {
      const Ops<float> *ops = c.ops;
      auto *P = reinterpret_cast<const StepParams<float> *>(ws + c.params[j]);
      auto *PL = reinterpret_cast<const StepParams<float> *>(ws + c.params_les[j]);
      if (c.n_les) CUDA_TRY(ops->moments_batch(PL, reinterpret_cast<const int64_t *>(ws + c.first_les), c.n_les,
                                               c.blocks_les, cs));
      if (c.key.pair)
        CUDA_TRY(ops->step_batch_pair(P, reinterpret_cast<const int64_t *>(ws + c.first), c.n, c.blocks, cs));
      else
        CUDA_TRY(ops->step_batch(P, reinterpret_cast<const int64_t *>(ws + c.first), c.n, c.blocks, cs));
    }
    if (branches) {
      CUDA_TRY(cudaEventRecord(B->branch_done[ci], cs));
      CUDA_TRY(cudaStreamWaitEvent(st, B->branch_done[ci], 0));
    }
  }
  // large members: their own step and finalisation, at their parity for this step
  for (size_t k = 0; k < B->solo.size(); k++) {
    AeroLattice *L = B->solo[k];
    const size_t bi = B->classes.size() + k;
    cudaStream_t cs = st;
    if (branches) {
      cs = B->branch[bi];
      CUDA_TRY(cudaStreamWaitEvent(cs, B->fork, 0));
    }
    const int par = (B->solo_cur[k] + j) & 1;
    const bool store = L->aa && aa_store;
    const int rc = is_f64(L) ? launch_step<double>(L, par, cs, false, store)
                             : launch_step<float>(L, par, cs, false, store);
    if (rc != AERO_OK) return rc;
    if (branches) {
      CUDA_TRY(cudaEventRecord(B->branch_done[bi], cs));
      CUDA_TRY(cudaStreamWaitEvent(st, B->branch_done[bi], 0));
    }
  }
  // the finalisation kernels do not depend on the lattice class, so any
  // table of the right arithmetic type launches them
  if (B->fin[0].n)
    CUDA_TRY(ops_f32(2, 0)->finalize_batch(reinterpret_cast<const StepParams<float> *>(ws + B->fin[0].params[j]),
                                           reinterpret_cast<const int64_t *>(ws + B->fin[0].first), B->fin[0].n,
                                           B->fin[0].blocks, st));
  if (B->fin[1].n)
    CUDA_TRY(ops_f64(2, 0)->finalize_batch(reinterpret_cast<const StepParams<double> *>(ws + B->fin[1].params[j]),
                                           reinterpret_cast<const int64_t *>(ws + B->fin[1].first), B->fin[1].n,
                                           B->fin[1].blocks, st));
  return AERO_OK;
}

// Graph of `steps` (1 or 2) consecutive steps starting at `phase`.
int batch_graph(AeroBatch *B, int steps, int phase, cudaGraphExec_t *out) {
  cudaGraphExec_t &g = B->graph[steps - 1][phase];
  if (!g) {
    if (!B->cap_stream) CUDA_TRY(cudaStreamCreateWithFlags(&B->cap_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamBeginCapture(B->cap_stream, cudaStreamCaptureModeThreadLocal));
    int rc = AERO_OK;
    const bool branches = B->classes.size() + B->solo.size() > 1;
    for (int j = 0; j < steps && rc == AERO_OK; j++)
      rc = batch_launch_step(B, (phase + j) & 1, B->cap_stream, branches);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(B->cap_stream, &graph);
    if (rc != AERO_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return fail(AERO_ERR_CUDA, "batch capture: %s", cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&g, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(AERO_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(ei));
  }
  *out = g;
  return AERO_OK;
}

}  // namespace

extern "C" {

int aero_batch_create(int32_t max_members, AeroBatch **out) {
  if (!out) return fail(AERO_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (max_members < 1 || max_members > 65536) return fail(AERO_ERR_INVALID, "max_members must be in 1..65536");
  AeroBatch *B = new AeroBatch();
  B->max_members = max_members;
  B->ws_bytes = batch_bytes(max_members);
  *out = B;
  return AERO_OK;
}

int aero_batch_workspace_size(const AeroBatch *B, uint64_t *bytes) {
  if (!B || !bytes) return fail(AERO_ERR_INVALID, "NULL argument");
  *bytes = B->ws_bytes;
  return AERO_OK;
}

int aero_batch_bind_workspace(AeroBatch *B, void *dptr, uint64_t bytes) {
  if (!B || !dptr) return fail(AERO_ERR_INVALID, "NULL argument");
  if (B->bound) return fail(AERO_ERR_STATE, "batch workspace already bound");
  if (bytes < B->ws_bytes) return fail(AERO_ERR_INVALID, "batch workspace too small: %llu < %llu",
                                       (unsigned long long)bytes, (unsigned long long)B->ws_bytes);
  if (reinterpret_cast<uintptr_t>(dptr) % kAlign) return fail(AERO_ERR_INVALID, "workspace must be 256-byte aligned");
  cudaPointerAttributes attr;
  CUDA_TRY(cudaPointerGetAttributes(&attr, dptr));
  if (attr.type != cudaMemoryTypeDevice) return fail(AERO_ERR_INVALID, "workspace is not device memory");
  B->device = attr.device;
  B->ws = static_cast<char *>(dptr);
  B->bound = true;
  return AERO_OK;
}

int aero_batch_add(AeroBatch *B, AeroLattice *L, double cd_norm) {
  if (!B || !L) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!B->bound) return fail(AERO_ERR_STATE, "batch workspace not bound");
  if (!L->state_set) return fail(AERO_ERR_STATE, "the lattice needs a state (aero_set_state) before joining");
  if (L->batch) return fail(AERO_ERR_STATE, "the lattice is already a batch member");
  if (L->device != B->device) return fail(AERO_ERR_INVALID, "the lattice is on another device than the batch");
  if ((int)B->members.size() >= B->max_members) return fail(AERO_ERR_CAPACITY, "batch holds %d members", B->max_members);
  if (!(cd_norm > 0.0) || !std::isfinite(cd_norm)) return fail(AERO_ERR_INVALID, "cd_norm must be > 0");
  if (L->aa && !batch_solo(L))
    return fail(AERO_ERR_UNSUPPORTED,
                "a lattice in the AA layout joins a batch only with at least %lld cells (then it steps on its "
                "own kernels)", (long long)kBatchSoloCells);
  L->batch = B;
  L->cd_norm = cd_norm;
  B->members.push_back(L);
  B->dirty = true;
  return AERO_OK;
}

int aero_batch_remove(AeroBatch *B, AeroLattice *L) {
  if (!B || !L) return fail(AERO_ERR_INVALID, "NULL argument");
  auto it = std::find(B->members.begin(), B->members.end(), L);
  if (it == B->members.end()) return fail(AERO_ERR_INVALID, "the lattice is not a member of this batch");
  B->members.erase(it);
  L->batch = nullptr;
  B->dirty = true;
  return AERO_OK;
}

int aero_batch_size(const AeroBatch *B, int32_t *n) {
  if (!B || !n) return fail(AERO_ERR_INVALID, "NULL argument");
  *n = (int32_t)B->members.size();
  return AERO_OK;
}

int aero_batch_step(AeroBatch *B, int64_t n, void *stream) {
  if (!B) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!B->bound) return fail(AERO_ERR_STATE, "batch workspace not bound");
  if (n < 0) return fail(AERO_ERR_INVALID, "negative step count");
  if (n == 0 || B->members.empty()) return AERO_OK;
  // members with an inflow field inlet read their fields from their own
  // device ring (aero_set_inflow), as when they step alone
  for (size_t k = 0; k < B->members.size(); k++) {
    const AeroLattice *L = B->members[k];
    if ((L->feat & FEAT_INFLOW_FIELD) && L->step_count + n > L->inflow_upto)
      return fail(AERO_ERR_STATE,
                  "member %d: inflow fields are on the device up to step %lld; upload them with aero_set_inflow",
                  (int)k, (long long)L->inflow_upto);
  }
  CUDA_TRY(cudaSetDevice(B->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (B->dirty) {
    const int rc = batch_build(B, st);
    if (rc != AERO_OK) return rc;
  }
  const int nm = (int)B->members.size();
  // only the last step of the call sums the force profiles
  k_set_profile_steps<<<blocks_for(nm, 128), 128, 0, st>>>(reinterpret_cast<int64_t *const *>(B->ws + B->ctr_ptrs),
                                                          nm, n);
  CUDA_TRY(cudaGetLastError());
  // members in the AA layout (all large, so stepped by their own kernels)
  // first collide the state their last call stored, and the call's last
  // step stores theirs: that step runs outside the graphs
  bool any_aa = false;
  for (AeroLattice *L : B->members) {
    if (!L->aa) continue;
    any_aa = true;
    if (L->aa_holds_state) {
      const int rc = is_f64(L) ? aa_collide_state<double>(L, st) : aa_collide_state<float>(L, st);
      if (rc != AERO_OK) return rc;
    }
  }
  int64_t left = any_aa ? n - 1 : n;
  while (left > 0) {
    const int steps = left >= 2 ? 2 : 1;
    cudaGraphExec_t g = nullptr;
    const int rc = batch_graph(B, steps, B->phase, &g);
    if (rc != AERO_OK) return rc;
    CUDA_TRY(cudaGraphLaunch(g, st));
    B->phase = (B->phase + steps) & 1;
    left -= steps;
  }
  if (any_aa) {
    const int rc = batch_launch_step(B, B->phase, st, false, true);
    if (rc != AERO_OK) return rc;
    B->phase ^= 1;
  }
  for (AeroLattice *L : B->members) {
    if (L->aa) L->aa_holds_state = true;
    L->cur ^= (int)(n & 1);
    L->step_count += n;
    L->old_is_state = false;
    // a member's history is a rolling window: unread steps older than the
    // ring are dropped
    L->read_upto = std::max(L->read_upto, L->step_count - (int64_t)L->hist_cap);
  }
  return AERO_OK;
}

int aero_batch_converge(AeroBatch *B, int32_t window, double tol, double *out, void *stream) {
  if (!B || !out) return fail(AERO_ERR_INVALID, "NULL argument");
  if (!B->bound) return fail(AERO_ERR_STATE, "batch workspace not bound");
  if (window < 1) return fail(AERO_ERR_INVALID, "window must be >= 1");
  for (AeroLattice *L : B->members)
    if (window > L->hist_cap) return fail(AERO_ERR_INVALID, "window %d exceeds a member's history ring (%d steps)",
                                          window, L->hist_cap);
  const int nm = (int)B->members.size();
  if (nm == 0) return AERO_OK;
  CUDA_TRY(cudaSetDevice(B->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (B->dirty) {
    const int rc = batch_build(B, st);
    if (rc != AERO_OK) return rc;
  }
  k_converge<<<nm, kFinalizeBlock, 0, st>>>(reinterpret_cast<const ConvergeItem *>(B->ws + B->conv_items), nm,
                                            window, tol);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(out, B->ws + B->conv_out, kConvergeValues * 8 * (size_t)nm, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return AERO_OK;
}

int aero_batch_destroy(AeroBatch *B) {
  if (!B) return AERO_OK;
  for (AeroLattice *L : B->members) L->batch = nullptr;
  batch_drop_graphs(B);
  if (B->cap_stream) cudaStreamDestroy(B->cap_stream);
  for (auto bs : B->branch) cudaStreamDestroy(bs);
  for (auto ev : B->branch_done) cudaEventDestroy(ev);
  if (B->fork) cudaEventDestroy(B->fork);
  delete B;
  return AERO_OK;
}

}  // extern "C"
