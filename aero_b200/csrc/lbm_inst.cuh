// lbm_inst.cuh -- explicit instantiation of the kernels for one storage type.
// Included by lbm_inst_<storage>.cu with AERO_STORE / AERO_OPS_FN defined.
#pragma once
#include <algorithm>
#include <type_traits>

#include "lbm_dispatch.h"
#include "lbm_kernels.cuh"
#include "lbm_pair.cuh"
#include "lbm_quad.cuh"
#include "lbm_les.cuh"

namespace aero {
inline namespace AERO_KNS {
namespace inst {

template <class L, class S, int COLL>
struct Launch {
  using Real = typename StoreOps<S>::Real;
  static cudaError_t step(const StepParams<Real> &p, bool from_state, dim3 grid, cudaStream_t st) {
    if (from_state)
      k_step<L, S, COLL, true><<<grid, kStepBlock, 0, st>>>(p);
    else
      k_step<L, S, COLL, false><<<grid, kStepBlock, 0, st>>>(p);
    return cudaGetLastError();
  }
  static cudaError_t step_shaped(const StepParams<Real> &p, int shape, cudaStream_t st) {
    const dim3 grid = step_grid(shape, p.nx, p.ny, p.nz);
    switch (shape) {
      case 1:
        k_step<L, S, COLL, false, 256, 1><<<grid, dim3(256, 1), 0, st>>>(p);
        break;
      case 2:
        k_step<L, S, COLL, false, 32, 4><<<grid, dim3(32, 4), 0, st>>>(p);
        break;
      default:
        k_step<L, S, COLL, false, 128, 1><<<grid, dim3(128, 1), 0, st>>>(p);
    }
    return cudaGetLastError();
  }
  static cudaError_t moments(const StepParams<Real> &p, bool from_state, dim3 grid, cudaStream_t st) {
    if (from_state)
      k_moments<L, S, true><<<grid, kStepBlock, 0, st>>>(p);
    else
      k_moments<L, S, false><<<grid, kStepBlock, 0, st>>>(p);
    return cudaGetLastError();
  }
  static cudaError_t finalize(const StepParams<Real> &p, cudaStream_t st) {
    k_finalize<Real><<<p.fin_blocks, kFinalizeBlock, 0, st>>>(p);
    return cudaGetLastError();
  }
  static cudaError_t state_out(const StepParams<Real> &p, double *out, int delta, bool raw, int z0, dim3 grid,
                               cudaStream_t st) {
    const int64_t plane = (int64_t)grid.z * p.ny * p.nx;
    if (raw)
      k_state_out<L, S, true><<<grid, kStepBlock, 0, st>>>(p, out, delta, z0, plane);
    else
      k_state_out<L, S, false><<<grid, kStepBlock, 0, st>>>(p, out, delta, z0, plane);
    return cudaGetLastError();
  }
  static cudaError_t macro_out(const StepParams<Real> &p, double *out, int delta, bool raw, int z0, dim3 grid,
                               cudaStream_t st) {
    const int64_t plane = (int64_t)grid.z * p.ny * p.nx;
    if (raw)
      k_macro_out<L, S, true><<<grid, kStepBlock, 0, st>>>(p, out, delta, z0, plane);
    else
      k_macro_out<L, S, false><<<grid, kStepBlock, 0, st>>>(p, out, delta, z0, plane);
    return cudaGetLastError();
  }
  static cudaError_t load_state(const StepParams<Real> &p, const double *in, void *dst, dim3 grid,
                                cudaStream_t st) {
    k_load_state<L, S><<<grid, kStepBlock, 0, st>>>(p, in, static_cast<S *>(dst));
    return cudaGetLastError();
  }
  static cudaError_t step_tiled(const StepParams<Real> &p, int blocks, cudaStream_t st) {
    k_step_tiled<L, S, COLL><<<blocks, TileCfg<L, S>::threads, TileCfg<L, S>::smem_bytes, st>>>(p);
    return cudaGetLastError();
  }
  static cudaError_t tiled_setup(int *blocks_per_sm, int *cap_cells) {
    cudaError_t e = cudaFuncSetAttribute(k_step_tiled<L, S, COLL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TileCfg<L, S>::smem_bytes);
    if (e != cudaSuccess) return e;
    // without the largest carveout the driver may size shared memory for
    // fewer resident blocks than the occupancy calculation assumes
    e = cudaFuncSetAttribute(k_step_tiled<L, S, COLL>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_step_tiled<L, S, COLL>,
                                                      TileCfg<L, S>::threads, TileCfg<L, S>::smem_bytes);
    *cap_cells = TileCfg<L, S>::cap;
    return e;
  }
  static cudaError_t step_batch(const StepParams<Real> *params, const int64_t *first, int n, int64_t blocks,
                                cudaStream_t st) {
    k_step_batch<L, S, COLL><<<(unsigned)blocks, kStepBlock, 0, st>>>(params, first, n);
    return cudaGetLastError();
  }
  static cudaError_t moments_batch(const StepParams<Real> *params, const int64_t *first, int n, int64_t blocks,
                                   cudaStream_t st) {
    k_moments_batch<L, S><<<(unsigned)blocks, kStepBlock, 0, st>>>(params, first, n);
    return cudaGetLastError();
  }
  static cudaError_t finalize_batch(const StepParams<Real> *params, const int64_t *first, int n, int64_t blocks,
                                    cudaStream_t st) {
    k_finalize_batch<Real><<<(unsigned)blocks, kFinalizeBlock, 0, st>>>(params, first, n);
    return cudaGetLastError();
  }
  static cudaError_t recycle_mean(const StepParams<Real> &p, cudaStream_t st) {
    if constexpr (L::DIMS == 3) {
      k_recycle_mean<L, S><<<p.recycle_blocks, kRecycleBlock, 0, st>>>(p);
      return cudaGetLastError();
    }
    return cudaErrorInvalidValue;  // recycling exists in 3D only
  }
  static cudaError_t step_batch_pair(const StepParams<Real> *params, const int64_t *first, int n, int64_t blocks,
                                     cudaStream_t st) {
    if constexpr (std::is_same<Real, float>::value && L::DIMS == 3) {
      k_step_batch_pair<L, S, COLL><<<(unsigned)blocks, kPairBlock, 0, st>>>(params, first, n);
      return cudaGetLastError();
    } else {
      (void)params;
      (void)first;
      (void)n;
      (void)blocks;
      (void)st;
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t step_pair(const StepParams<Real> &p, cudaStream_t st) {
    if constexpr (std::is_same<Real, float>::value && L::DIMS == 3) {
      k_step_pair<L, S, COLL><<<pair_grid(p), kPairBlock, 0, st>>>(p);
      return cudaGetLastError();
    } else {
      (void)p;
      (void)st;
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t field_stats(const StepParams<Real> &p, const Real *gcur, int z0, int nzs, int delta, bool raw,
                                 double *partial, uint32_t *ticket, double *out, cudaStream_t st) {
    if (raw)
      k_field_stats<L, S, true><<<kStatsBlocks, kStatsBlock, 0, st>>>(p, gcur, z0, nzs, delta, partial, ticket, out);
    else
      k_field_stats<L, S, false><<<kStatsBlocks, kStatsBlock, 0, st>>>(p, gcur, z0, nzs, delta, partial, ticket, out);
    return cudaGetLastError();
  }
  static cudaError_t init_eq(const StepParams<Real> &p, const EqFields &e, void *dst, Real *prev, Real *g,
                             dim3 grid, cudaStream_t st) {
    k_init_equilibrium<L, S><<<grid, kStepBlock, 0, st>>>(p, e, static_cast<S *>(dst), prev, g);
    return cudaGetLastError();
  }
  static cudaError_t step_quad(const StepParams<Real> &p, cudaStream_t st) {
    if constexpr (std::is_same<Real, float>::value && L::DIMS == 3 && sizeof(S) == 2) {
      k_step_quad<L, S, COLL><<<quad_grid(p), kQuadBlock, 0, st>>>(p);
      return cudaGetLastError();
    } else {
      (void)p;
      (void)st;
      return cudaErrorNotSupported;
    }
  }
  static constexpr bool kLesCapable = L::DIMS == 3 && COLL != COLL_MRT;
  static cudaError_t step_les(const StepParams<Real> &p, cudaStream_t st) {
    if constexpr (kLesCapable) {
      const dim3 grid((unsigned)((p.nx + kLesTileX - 1) / kLesTileX), (unsigned)((p.ny + kLesRows - 1) / kLesRows),
                      (unsigned)((p.nz + p.les_chunk - 1) / p.les_chunk));
      k_step_les<L, S, COLL><<<grid, kLesThreads, les_smem_bytes<Real>(), st>>>(p);
      return cudaGetLastError();
    } else {
      (void)p;
      (void)st;
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t les_setup() {
    if constexpr (kLesCapable) {
      return cudaFuncSetAttribute(k_step_les<L, S, COLL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)les_smem_bytes<Real>());
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t aa_stage(const StepParams<Real> &p, unsigned blocks, cudaStream_t st) {
    k_aa_stage<L, S><<<dim3(blocks, L::Q), kStageBlock, 0, st>>>(p);
    return cudaGetLastError();
  }
  static cudaError_t aa_recycle_mean(const StepParams<Real> &p, cudaStream_t st) {
    if constexpr (L::DIMS == 3) {
      k_recycle_mean<L, S, true><<<p.recycle_blocks, kRecycleBlock, 0, st>>>(p);
      return cudaGetLastError();
    }
    return cudaErrorInvalidValue;  // recycling exists in 3D only
  }
  static cudaError_t aa_moments(const StepParams<Real> &p, dim3 grid, cudaStream_t st) {
    k_moments<L, S, false, true><<<grid, kStepBlock, 0, st>>>(p);
    return cudaGetLastError();
  }
  static cudaError_t aa_step(const StepParams<Real> &p, dim3 grid, cudaStream_t st) {
    // one instantiation per read layout: the shifted and the own-cell
    // addressing each compile without the other's branches
    if (p.aa_layout == 0)
      k_step<L, S, COLL, false, kStepBlock, 1, true, 0><<<grid, kStepBlock, 0, st>>>(p);
    else
      k_step<L, S, COLL, false, kStepBlock, 1, true, 1><<<grid, kStepBlock, 0, st>>>(p);
    return cudaGetLastError();
  }
  static cudaError_t run_small(const StepParams<Real> *pp, int64_t ncells, int64_t nsteps, int stall_block,
                               cudaStream_t st) {
    // resident blocks of this instantiation on the current device (every
    // block of a cooperative launch must be resident at once)
    static int per_sm = -1, sms = 0;
    if (per_sm < 0) {
      int dev = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_run_small<L, S, COLL>, kRunBlock, 0);
      if (e != cudaSuccess) {
        per_sm = -1;
        return e;
      }
    }
    const int64_t capacity = (int64_t)per_sm * sms;
    if (capacity < 2) return cudaErrorCooperativeLaunchTooLarge;
    // cell blocks: enough for one cell per thread, at most AERO_RUN_BLOCKS_PER_SM
    // per SM (fewer arrivals at each grid barrier) and what stays resident
    const int64_t cap = std::min<int64_t>(capacity - 1, (int64_t)AERO_RUN_BLOCKS_PER_SM * sms);
    const int64_t cells = std::min<int64_t>((ncells + kRunBlock - 1) / kRunBlock, cap);
    const dim3 grid((unsigned)(1 + cells));
    void *args[] = {(void *)&pp, (void *)&nsteps, (void *)&stall_block};
    return cudaLaunchCooperativeKernel((const void *)k_run_small<L, S, COLL>, grid, dim3(kRunBlock), args, 0, st);
  }
  static constexpr Ops<Real> table = {&step,       &step_shaped, &moments,      &finalize,   &state_out,
                                      &load_state, &macro_out,   &step_tiled,   &tiled_setup, &step_batch,
                                      &moments_batch, &finalize_batch, &recycle_mean, &step_pair,
                                      &step_batch_pair, &field_stats, &init_eq, &step_quad, &step_les, &les_setup, &aa_stage,
                                      &aa_recycle_mean, &aa_moments, &aa_step, &run_small, (int)sizeof(S)};
};

template <class S>
const Ops<typename StoreOps<S>::Real> *lookup(int dims, int coll) {
  if (dims == 2) {
    switch (coll) {
      case COLL_BGK: return &Launch<D2Q9, S, COLL_BGK>::table;
      case COLL_TRT: return &Launch<D2Q9, S, COLL_TRT>::table;
      case COLL_MRT: return &Launch<D2Q9, S, COLL_MRT>::table;
    }
  } else if (dims == 3) {
    switch (coll) {
      case COLL_BGK: return &Launch<D3Q19, S, COLL_BGK>::table;
      case COLL_TRT: return &Launch<D3Q19, S, COLL_TRT>::table;
      case COLL_MRT: return &Launch<D3Q19, S, COLL_MRT>::table;
    }
  }
  return nullptr;
}

}  // namespace inst
}  // namespace AERO_KNS
}  // namespace aero
