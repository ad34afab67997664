// k-space pipeline instantiated for float (see p3mg_assign_impl.cuh).
#include "p3mg_assign_impl.cuh"

namespace p3mg {

int kspace_run_f32(Ctx *c) { return assign_impl::run_kspace<float>(c); }

}  // namespace p3mg
