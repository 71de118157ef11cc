// krylov.cu -- GMRES (restarted, classical Gram-Schmidt applied twice) on the
// device, and the Newton-Krylov relaxation built on it.
//
// The reference runs GMRES with every dot product round-tripping to the host
// (radgpurlx.cu:2014-2083).  Here the Gram-Schmidt projections of one Arnoldi
// step are fused into one multi-dot kernel (fixed-order partial sums, so the
// iteration is bitwise reproducible) and only the (j+1) projection
// coefficients come back to the host, where the tiny Hessenberg least-squares
// problem is solved with Givens rotations.
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace rb {


static DBuf g_kpart, g_kscal;

// dots[k] = <V_k, w> for k < nv (chunks of MD_MAX)
static int dots_many(double *const *V, int nv, const double *w, int64_t len, double *out)
{
  for (int s = 0; s < nv; s += MD_MAX) {
    DotSet ds;
    ds.nd = std::min(MD_MAX, nv - s);
    for (int k = 0; k < ds.nd; k++) { ds.a[k] = V[s + k]; ds.b[k] = w; }
    RB_TRY(multidot(ds, len, out + s, g_kpart, g_kscal, 0));
  }
  return 0;
}

// y += sum_k c_k V_k (chunks)
static int axpy_many(double *const *V, const double *c, int nv, int64_t len, double *y)
{
  for (int s = 0; s < nv; s += MD_MAX) {
    AxpySet as;
    as.nv = std::min(MD_MAX, nv - s);
    for (int k = 0; k < as.nv; k++) { as.v[k] = V[s + k]; as.c[k] = c[s + k]; }
    RB_TRY(lincomb(as, len, y, 1, 0));
  }
  return 0;
}

static int vscale(double *v, double a, int64_t len)
{
  AxpySet as; as.nv = 1; as.v[0] = v; as.c[0] = a;
  return lincomb(as, len, v, 0, 0);
}

static int vcopy_axpy(double *y, const double *x, double a, const double *z, double b, int64_t len)
{
  AxpySet as; as.nv = 2; as.v[0] = x; as.c[0] = a; as.v[1] = z; as.c[1] = b;
  return lincomb(as, len, y, 0, 0);
}

int gmres(Op &op, int n3, int ld, const double *b, double *x, double rtol, int max_iter, int restart, double *relres,
          int *iters, cudaStream_t)
{
  restart = std::max(1, std::min(restart, 200));
  DBuf Vb, wb, rb_;
  RB_TRY(Vb.alloc((size_t)(restart + 1) * ld * sizeof(double)));
  RB_TRY(wb.alloc((size_t)2 * ld * sizeof(double)));
  // the matvec reads whole padded rows (ld), so the padding must hold zeros
  RB_CUDA(cudaMemset(Vb.p, 0, (size_t)(restart + 1) * ld * sizeof(double)));
  RB_CUDA(cudaMemset(wb.p, 0, (size_t)2 * ld * sizeof(double)));
  std::vector<double *> V(restart + 1);
  for (int k = 0; k <= restart; k++) V[k] = Vb.as<double>() + (size_t)k * ld;
  double *w = wb.as<double>(), *z = w + ld;
  double bnorm;
  {
    double *bb[1] = {(double *)b};
    RB_TRY(dots_many(bb, 1, b, n3, &bnorm));
    bnorm = sqrt(bnorm);
  }
  if (bnorm == 0.0) bnorm = 1.0;
  int total = 0;
  double rel = 1.0;
  while (true) {
    // r = b - A x
    RB_TRY(op.apply(x, w));
    RB_TRY(vcopy_axpy(V[0], b, 1.0, w, -1.0, n3));
    double beta;
    RB_TRY(dots_many(&V[0], 1, V[0], n3, &beta));
    beta = sqrt(beta);
    rel = beta / bnorm;
    if (!std::isfinite(rel)) { set_error("GMRES: non-finite residual"); return RADB200_E_NUMERIC; }
    if (rel <= rtol || total >= max_iter) break;
    RB_TRY(vscale(V[0], 1.0 / beta, n3));
    std::vector<double> H((size_t)(restart + 1) * restart, 0.0), cs(restart), sn(restart), g(restart + 1, 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < restart && total < max_iter; j++, total++) {
      RB_CUDA(cudaMemcpy(z, V[j], n3 * sizeof(double), cudaMemcpyDeviceToDevice));
      RB_TRY(op.precond(z));
      RB_TRY(op.apply(z, w));
      std::vector<double> h(j + 1), h2(j + 1);
      RB_TRY(dots_many(V.data(), j + 1, w, n3, h.data()));
      for (int k = 0; k <= j; k++) h[k] = -h[k];
      RB_TRY(axpy_many(V.data(), h.data(), j + 1, n3, w));
      RB_TRY(dots_many(V.data(), j + 1, w, n3, h2.data()));
      for (int k = 0; k <= j; k++) h2[k] = -h2[k];
      RB_TRY(axpy_many(V.data(), h2.data(), j + 1, n3, w));
      for (int k = 0; k <= j; k++) H[(size_t)k * restart + j] = -(h[k] + h2[k]);
      double hn;
      RB_TRY(dots_many(&w, 1, w, n3, &hn));
      hn = sqrt(hn);
      H[(size_t)(j + 1) * restart + j] = hn;
      // apply previous rotations
      for (int k = 0; k < j; k++) {
        double a = H[(size_t)k * restart + j], c = H[(size_t)(k + 1) * restart + j];
        H[(size_t)k * restart + j] = cs[k] * a + sn[k] * c;
        H[(size_t)(k + 1) * restart + j] = -sn[k] * a + cs[k] * c;
      }
      double a = H[(size_t)j * restart + j], c = H[(size_t)(j + 1) * restart + j];
      double r = hypot(a, c);
      cs[j] = (r == 0.0) ? 1.0 : a / r;
      sn[j] = (r == 0.0) ? 0.0 : c / r;
      H[(size_t)j * restart + j] = r;
      H[(size_t)(j + 1) * restart + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      if (hn > 0.0) {
        RB_CUDA(cudaMemcpy(V[j + 1], w, n3 * sizeof(double), cudaMemcpyDeviceToDevice));
        RB_TRY(vscale(V[j + 1], 1.0 / hn, n3));
      }
      if (fabs(g[j + 1]) / bnorm <= rtol || hn == 0.0) { j++; total++; break; }
    }
    // y = H^-1 g (upper triangular j x j)
    std::vector<double> y(j, 0.0);
    for (int k = j - 1; k >= 0; k--) {
      double s = g[k];
      for (int q = k + 1; q < j; q++) s -= H[(size_t)k * restart + q] * y[q];
      y[k] = s / H[(size_t)k * restart + k];
    }
    RB_CUDA(cudaMemset(z, 0, n3 * sizeof(double)));
    RB_TRY(axpy_many(V.data(), y.data(), j, n3, z));
    RB_TRY(op.precond(z));
    AxpySet as; as.nv = 1; as.v[0] = z; as.c[0] = 1.0;
    RB_TRY(lincomb(as, n3, x, 1, 0));
  }
  *relres = rel;
  *iters = total;
  return 0;
}

}  // namespace rb
