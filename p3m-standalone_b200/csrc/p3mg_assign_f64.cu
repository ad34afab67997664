// k-space pipeline instantiated for double (see p3mg_assign_impl.cuh).
#include "p3mg_assign_impl.cuh"

namespace p3mg {

int kspace_run_f64(Ctx *c) { return assign_impl::run_kspace<double>(c); }
int kspace_batch_f64(Ctx *c, const KspaceBatch &b) { return assign_impl::run_kspace_batch<double>(c, b); }
int adjoint_scatter_f64(Ctx *c) { return assign_impl::scatter_any<double, true>(c); }
int adjoint_gather_f64(Ctx *c, const void *Phi, double s, double ge, double *gx, double *gq) {
  return assign_impl::adj_gather_any<double>(c, Phi, s, ge, gx, gq);
}

}  // namespace p3mg
