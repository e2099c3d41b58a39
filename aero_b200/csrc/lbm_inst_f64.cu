// lbm_inst_f64.cu -- kernels instantiated for double population storage.
#include "lbm_inst.cuh"

namespace aero {
const Ops<typename StoreOps<double>::Real> *ops_f64(int dims, int coll) { return inst::lookup<double>(dims, coll); }
}  // namespace aero
