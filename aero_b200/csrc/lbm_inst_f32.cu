// lbm_inst_f32.cu -- kernels instantiated for float population storage.
#include "lbm_inst.cuh"

namespace aero {
const Ops<typename StoreOps<float>::Real> *ops_f32(int dims, int coll) { return inst::lookup<float>(dims, coll); }
}  // namespace aero
