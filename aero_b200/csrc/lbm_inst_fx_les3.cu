// lbm_inst_fx_les3.cu -- kernels compiled for the 3D wind tunnel with Smagorinsky LES: D3Q19 BGK / TRT with Smagorinsky LES, velocity inlet and outlet planes, an obstacle with mid-link bounce-back, slip walls.  The
// feature word and wall type are fixed, so the other features' branches are
// removed; lattices with exactly this word, wall type, dimension and
// collision (FP32 storage) take these kernels, single lattices and batch
// classes alike (capi.cu).
#include "aero_b200.h"
#include "lbm_params.h"

// branches made unreachable by the fixed feature word are expected here
#pragma nv_diag_suppress 128

#define AERO_KNS fx_les3
#define AERO_FIXED_FEAT (FEAT_OPEN | FEAT_OBSTACLE_BB | FEAT_LES)
#define AERO_FIXED_WALL WALL_SLIP
#include "lbm_inst.cuh"

namespace aero {

const Ops<float> *ops_fx_les3(int dims, int coll, int storage, uint32_t feat, int32_t wall) {
  if (dims != 3 || storage != AERO_STORE_F32 || feat != (uint32_t)(AERO_FIXED_FEAT) || wall != AERO_FIXED_WALL)
    return nullptr;
  switch (coll) {
    case COLL_BGK: return &fx_les3::inst::Launch<D3Q19, float, COLL_BGK>::table;
    case COLL_TRT: return &fx_les3::inst::Launch<D3Q19, float, COLL_TRT>::table;
  }
  return nullptr;
}

}  // namespace aero
