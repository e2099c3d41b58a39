// lbm_inst_f16.cu -- kernels instantiated for __half population storage.
#include "lbm_inst.cuh"

namespace aero {
const Ops<typename StoreOps<__half>::Real> *ops_f16(int dims, int coll) { return inst::lookup<__half>(dims, coll); }
}  // namespace aero
