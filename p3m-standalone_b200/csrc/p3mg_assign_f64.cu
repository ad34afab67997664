// k-space pipeline instantiated for double (see p3mg_assign_impl.cuh).
#include "p3mg_assign_impl.cuh"

namespace p3mg {

int kspace_run_f64(Ctx *c) { return assign_impl::run_kspace<double>(c); }

}  // namespace p3mg
