// lbm_inst_bf16.cu -- kernels instantiated for __nv_bfloat16 population storage.
#include "lbm_inst.cuh"

namespace aero {
const Ops<typename StoreOps<__nv_bfloat16>::Real> *ops_bf16(int dims, int coll) { return inst::lookup<__nv_bfloat16>(dims, coll); }
}  // namespace aero
