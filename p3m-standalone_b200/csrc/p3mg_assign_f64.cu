// k-space pipeline instantiated for double (see p3mg_assign_impl.cuh).
#include "p3mg_assign_impl.cuh"

namespace p3mg {

int kspace_run_f64(Ctx *c) { return assign_impl::run_kspace<double>(c); }
int kspace_batch_f64(Ctx *c, const KspaceBatch &b) { return assign_impl::run_kspace_batch<double>(c, b); }

}  // namespace p3mg
