// lbm_inst_fx_thermal.cu -- kernels compiled for the thermal channel's feature
// word and wall type: D3Q19 TRT with WALE LES, uniform body force, the D3Q7
// scalar with Boussinesq buoyancy, an obstacle with mid-link bounce-back,
// no-slip walls, streamwise periodic (no inlet, outlet, sponge or Bouzidi).  The step there is
// instruction-bound; with every other feature's branch removed at compile
// time the step chain is shorter and fits the instruction cache better.
// Lattices whose feature word is exactly this one take these kernels
// (capi.cu's get_ops); every other lattice takes the generic ones.
#include "aero_b200.h"
#include "lbm_params.h"

// branches made unreachable by the fixed feature word are expected here
#pragma nv_diag_suppress 128

#define AERO_KNS fx_thermal
#define AERO_FIXED_FEAT                                                                                            \
  (FEAT_BODY_FORCE | FEAT_LES | FEAT_LES_WALE | FEAT_THERMAL | FEAT_BUOYANCY | FEAT_SCALAR_REDUCED |               \
   FEAT_OBSTACLE_BB)
#define AERO_FIXED_WALL WALL_NOSLIP
#include "lbm_inst.cuh"

namespace aero {

const Ops<float> *ops_fx_thermal(int dims, int coll, int storage, uint32_t feat, int32_t wall) {
  if (dims != 3 || coll != COLL_TRT || feat != (uint32_t)(AERO_FIXED_FEAT) || wall != AERO_FIXED_WALL)
    return nullptr;
  switch (storage) {
    case AERO_STORE_F32: return &fx_thermal::inst::Launch<D3Q19, float, COLL_TRT>::table;
    case AERO_STORE_F16: return &fx_thermal::inst::Launch<D3Q19, __half, COLL_TRT>::table;
    case AERO_STORE_BF16: return &fx_thermal::inst::Launch<D3Q19, __nv_bfloat16, COLL_TRT>::table;
  }
  return nullptr;
}

}  // namespace aero
