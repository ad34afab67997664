// k-space pipeline instantiated for float (see p3mg_assign_impl.cuh).
#include "p3mg_assign_impl.cuh"

namespace p3mg {

int kspace_run_f32(Ctx *c) { return assign_impl::run_kspace<float>(c); }
int kspace_batch_f32(Ctx *c, const KspaceBatch &b) { return assign_impl::run_kspace_batch<float>(c, b); }

}  // namespace p3mg
