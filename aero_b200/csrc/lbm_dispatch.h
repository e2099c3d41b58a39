// lbm_dispatch.h -- per-(lattice, storage, collision) launch tables.
#pragma once
#include <cuda_runtime.h>

#include "lbm_params.h"

namespace aero {

template <class Real>
struct Ops {
  // grid covers (ceil(nx / kStepBlock), ny, nz)
  cudaError_t (*step)(const StepParams<Real> &, bool from_state, dim3 grid, cudaStream_t);
  // regular step with block shape `shape` (kStepShapes); grid from step_grid
  cudaError_t (*step_shaped)(const StepParams<Real> &, int shape, cudaStream_t);
  cudaError_t (*moments)(const StepParams<Real> &, bool from_state, dim3 grid, cudaStream_t);
  cudaError_t (*finalize)(const StepParams<Real> &, cudaStream_t);
  // grid.z = planes written, starting at plane z0; out holds (Q, grid.z, ny, nx)
  cudaError_t (*state_out)(const StepParams<Real> &, double *out, int step_delta, bool raw, int z0, dim3 grid,
                           cudaStream_t);
  cudaError_t (*load_state)(const StepParams<Real> &, const double *in, void *dst, dim3 grid, cudaStream_t);
  // like state_out, but writes rho, ux, uy[, uz] (1 + dims planes) instead of f
  cudaError_t (*macro_out)(const StepParams<Real> &, double *out, int step_delta, bool raw, int z0, dim3 grid,
                           cudaStream_t);
  // row-tiled step (k_step_tiled): persistent grid of `blocks` blocks
  cudaError_t (*step_tiled)(const StepParams<Real> &, int blocks, cudaStream_t);
  // on the current device: raises the kernel's dynamic shared-memory limit and
  // reports resident blocks per SM and the cells one row slab holds
  cudaError_t (*tiled_setup)(int *blocks_per_sm, int *cap_cells);
  // batched kernels over `n` members of one class: params and first (block
  // prefix, n entries) are device arrays; blocks = total grid size
  cudaError_t (*step_batch)(const StepParams<Real> *params, const int64_t *first, int n, int64_t blocks,
                            cudaStream_t);
  cudaError_t (*moments_batch)(const StepParams<Real> *params, const int64_t *first, int n, int64_t blocks,
                               cudaStream_t);
  cudaError_t (*finalize_batch)(const StepParams<Real> *params, const int64_t *first, int n, int64_t blocks,
                                cudaStream_t);
  // mean ux of the recycle plane (3D recycling inlet), before the step kernel
  cudaError_t (*recycle_mean)(const StepParams<Real> &, cudaStream_t);
  // regular step, two cells per thread (k_step_pair; D3Q19, 4-byte
  // arithmetic); cudaErrorNotSupported for other classes
  cudaError_t (*step_pair)(const StepParams<Real> &, cudaStream_t);
  // batched step of a class in the pair layout (k_step_batch_pair; D3Q19,
  // 4-byte arithmetic); blocks = the members' pair_batch_layout blocks
  cudaError_t (*step_batch_pair)(const StepParams<Real> *params, const int64_t *first, int n, int64_t blocks,
                                 cudaStream_t);
  // FP64 field statistics of the current state over planes z0 .. z0+nzs-1
  // (k_field_stats): gcur is the current scalar buffer (NULL without a
  // scalar); partial / ticket are workspace scratch; out (device) receives
  // kStatsValues doubles
  cudaError_t (*field_stats)(const StepParams<Real> &, const Real *gcur, int z0, int nzs, int step_delta, bool raw,
                             double *partial, uint32_t *ticket, double *out, cudaStream_t);
  // equilibrium state of the fields into dst (populations), prev (outlet
  // state, may be NULL) and g (scalar, may be NULL); grid as for step
  cudaError_t (*init_eq)(const StepParams<Real> &, const EqFields &, void *dst, Real *prev, Real *g, dim3 grid,
                         cudaStream_t);
  // regular step, four cells per thread (k_step_quad; D3Q19, 16-bit
  // storage); cudaErrorNotSupported for other classes
  cudaError_t (*step_quad)(const StepParams<Real> &, cudaStream_t);
  // regular step of a D3Q19 BGK / TRT + LES lattice with the LES rate from a
  // shared-memory velocity stencil (k_step_les); cudaErrorNotSupported for
  // other classes.  les_setup raises the kernel's shared-memory limit on the
  // current device.
  cudaError_t (*step_les)(const StepParams<Real> &, cudaStream_t);
  cudaError_t (*les_setup)();
  // AA layout (one buffer updated in place): the staging of the step's
  // cross-cell reads (k_aa_stage, `blocks` x Q blocks), then the recycle mean,
  // moments pass and step kernel reading through the AA access functor
  cudaError_t (*aa_stage)(const StepParams<Real> &, unsigned blocks, cudaStream_t);
  cudaError_t (*aa_recycle_mean)(const StepParams<Real> &, cudaStream_t);
  cudaError_t (*aa_moments)(const StepParams<Real> &, dim3 grid, cudaStream_t);
  cudaError_t (*aa_step)(const StepParams<Real> &, dim3 grid, cudaStream_t);
  // nsteps steps of a small lattice in one cooperative launch (k_run_small):
  // pp (device) = the parameters of the call's even and odd steps; the grid
  // is one finalisation block plus as many cell blocks as ncells needs and
  // the device holds at once; stall_block is -1 (tests: a block that leaves)
  cudaError_t (*run_small)(const StepParams<Real> *pp, int64_t ncells, int64_t nsteps, int stall_block,
                           cudaStream_t);
  int store_bytes;
};

const Ops<float> *ops_f32(int dims, int coll);
const Ops<double> *ops_f64(int dims, int coll);
const Ops<float> *ops_f16(int dims, int coll);
const Ops<float> *ops_bf16(int dims, int coll);
// Kernel sets compiled for one feature word and wall type each
// (lbm_inst_fx_*.cu): the table for a lattice of these dimensions,
// collision, storage, feature word and wall type, or NULL where the set does
// not cover it.  kFxSets lists them; its index + 1 is the variant that
// aero_kernel_variant reports.
using FxLookup = const Ops<float> *(*)(int dims, int coll, int storage, uint32_t feat, int32_t wall);
const Ops<float> *ops_fx_thermal(int dims, int coll, int storage, uint32_t feat, int32_t wall);
const Ops<float> *ops_fx_open2(int dims, int coll, int storage, uint32_t feat, int32_t wall);
const Ops<float> *ops_fx_open3(int dims, int coll, int storage, uint32_t feat, int32_t wall);
const Ops<float> *ops_fx_les2(int dims, int coll, int storage, uint32_t feat, int32_t wall);
const Ops<float> *ops_fx_les3(int dims, int coll, int storage, uint32_t feat, int32_t wall);
constexpr FxLookup kFxSets[] = {&ops_fx_thermal, &ops_fx_open2, &ops_fx_open3, &ops_fx_les2, &ops_fx_les3};
constexpr int kFxCount = (int)(sizeof(kFxSets) / sizeof(kFxSets[0]));

// Block shapes of the per-cell step kernel an autotuner can choose from:
// {threads along x, rows}.  Shape 0 is the default.
constexpr int kStepShapes = 3;
constexpr int kStepShapeXY[kStepShapes][2] = {{128, 1}, {256, 1}, {32, 4}};

// Step kernel ids beyond the shapes: kStepShapes = the row-tiled kernel,
// kStepPair = the two-cells-per-thread kernel, kStepQuad = the four-cells-
// per-thread kernel for 16-bit storage.
constexpr int kStepPair = kStepShapes + 1;
constexpr int kStepQuad = kStepShapes + 2;
// kStepLes = the D3Q19 BGK / TRT step with the LES velocity stencil in
// shared memory (no separate moments pass).
constexpr int kStepLes = kStepShapes + 3;

inline dim3 step_grid(int shape, int nx, int ny, int nz) {
  const int bx = kStepShapeXY[shape][0], by = kStepShapeXY[shape][1];
  return dim3((unsigned)((nx + bx - 1) / bx), (unsigned)((ny + by - 1) / by), (unsigned)nz);
}

bool build_mrt(int dims, double omega, MrtCoeffs<double> &out, double *A_full, double *B_full);
bool build_mrt3_adapted(double omega, Mrt3Adapted<double> &out);
bool mrt_pinv_basis(int dims, double *M_out, double *Minv_out);

// Records the message returned by aero_last_error() and returns code.
int set_error(int code, const char *msg);

}  // namespace aero
