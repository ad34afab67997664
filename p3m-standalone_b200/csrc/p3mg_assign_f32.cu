// k-space pipeline instantiated for float (see p3mg_assign_impl.cuh).
#include "p3mg_assign_impl.cuh"

namespace p3mg {

int kspace_run_f32(Ctx *c) { return assign_impl::run_kspace<float>(c); }
int kspace_batch_f32(Ctx *c, const KspaceBatch &b) { return assign_impl::run_kspace_batch<float>(c, b); }
int adjoint_scatter_f32(Ctx *c) { return assign_impl::scatter_any<float, true>(c); }
int adjoint_gather_f32(Ctx *c, const void *Phi, double s, double ge, double *gx, double *gq) {
  return assign_impl::adj_gather_any<float>(c, Phi, s, ge, gx, gq);
}

}  // namespace p3mg
