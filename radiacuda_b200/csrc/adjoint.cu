// adjoint.cu -- hand-written adjoint of the relaxation and of the field operator.
#include "internal.cuh"

namespace rb {

int adjoint_solve(Intrc &I, const double *dLdM, double rtol, int max_iter, double *lambda, double *status)
{
  (void)I; (void)dLdM; (void)rtol; (void)max_iter; (void)lambda; (void)status;
  set_error("adjoint not available");
  return RADB200_E_UNSUPPORTED;
}
int adjoint_grad(Intrc &I, const double *lambda, double *dMr, double *dc)
{
  (void)I; (void)lambda; (void)dMr; (void)dc;
  set_error("adjoint not available");
  return RADB200_E_UNSUPPORTED;
}
int field_vjp(Intrc &I, const double *M, const double *pts, int64_t npts, int what, const double *W, double *gM, double *gc)
{
  (void)I; (void)M; (void)pts; (void)npts; (void)what; (void)W; (void)gM; (void)gc;
  set_error("adjoint not available");
  return RADB200_E_UNSUPPORTED;
}
int lu_precond_transposed(Intrc &I, double *x, cudaStream_t st) { (void)I; (void)x; (void)st; return RADB200_E_UNSUPPORTED; }

}  // namespace rb
