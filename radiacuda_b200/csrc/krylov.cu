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
#include "material.cuh"

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
  restart = std::max(1, std::min(restart, 60));
  DBuf Vb, wb, rb_;
  RB_TRY(Vb.alloc((size_t)(restart + 1) * ld * sizeof(double)));
  RB_TRY(wb.alloc((size_t)2 * ld * sizeof(double)));
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

// ---------------------------------------------------------------------------
// Newton-Krylov relaxation (method 11 of the reference)
// ---------------------------------------------------------------------------
// residual F = M(H) - M with H = N M + H_ext (full field incl. self), D = dM/dH
__global__ void nk_material_kernel(const double *__restrict__ Hfull, const double *__restrict__ M,
                                   const int *__restrict__ kind, const double *__restrict__ mat, int n,
                                   double *__restrict__ F, double *__restrict__ D)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double *m = mat + (size_t)e * RADB200_MAT_STRIDE;
  V3<double> H = mk3<double>(Hfull[3 * e], Hfull[3 * e + 1], Hfull[3 * e + 2]);
  V3<double> Mm = mat_M(kind[e], m, H);
  F[3 * e] = Mm.x - M[3 * e];
  F[3 * e + 1] = Mm.y - M[3 * e + 1];
  F[3 * e + 2] = Mm.z - M[3 * e + 2];
  mat_D(kind[e], m, H, D + 9 * (size_t)e);
}

// block-Jacobi preconditioner P_e = (I - D_e Q_ee)^-1, stored per element
template <typename MT>
__global__ void nk_precond_build(const MT *__restrict__ N, int ld, const double *__restrict__ D, int n, double *__restrict__ P)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double *De = D + 9 * (size_t)e;
  double Q[9], A[9];
  const MT *d = N + (size_t)(3 * e) * ld + 3 * e;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) Q[3 * a + b] = (double)d[(size_t)a * ld + b];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      A[3 * a + b] = (a == b ? 1.0 : 0.0) - (De[3 * a] * Q[b] + De[3 * a + 1] * Q[3 + b] + De[3 * a + 2] * Q[6 + b]);
  inv3x3(A, P + 9 * (size_t)e);
}

__global__ void blockmul_kernel(const double *__restrict__ P, int n, double *__restrict__ v, int transpose)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double *B = P + 9 * (size_t)e;
  double x = v[3 * e], y = v[3 * e + 1], z = v[3 * e + 2];
  if (!transpose) {
    v[3 * e] = B[0] * x + B[1] * y + B[2] * z;
    v[3 * e + 1] = B[3] * x + B[4] * y + B[5] * z;
    v[3 * e + 2] = B[6] * x + B[7] * y + B[8] * z;
  } else {
    v[3 * e] = B[0] * x + B[3] * y + B[6] * z;
    v[3 * e + 1] = B[1] * x + B[4] * y + B[7] * z;
    v[3 * e + 2] = B[2] * x + B[5] * y + B[8] * z;
  }
}

// out = v - D (N v)   given y = N v
__global__ void nk_apply_kernel(const double *__restrict__ v, const double *__restrict__ y, const double *__restrict__ D,
                                int n, double *__restrict__ out)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double *B = D + 9 * (size_t)e;
  for (int a = 0; a < 3; a++)
    out[3 * e + a] = v[3 * e + a] - (B[3 * a] * y[3 * e] + B[3 * a + 1] * y[3 * e + 1] + B[3 * a + 2] * y[3 * e + 2]);
}

struct NKOp : Op {
  Intrc &I;
  const double *D, *P;
  double *tmp;
  NKOp(Intrc &i, const double *d, const double *p, double *t) : I(i), D(d), P(p), tmp(t) {}
  int apply(const double *v, double *out) override
  {
    RB_TRY(run_matvec(I, v, nullptr, 1.0, tmp, 0));
    nk_apply_kernel<<<(I.n + 127) / 128, 128>>>(v, tmp, D, I.n, out);
    return check_launch("nk_apply_kernel");
  }
  int precond(double *v) override
  {
    blockmul_kernel<<<(I.n + 127) / 128, 128>>>(P, I.n, v, 0);
    return check_launch("blockmul_kernel");
  }
};

int relax_newton(Intrc &I, double prec, int max_iter, double *status)
{
  const int n = I.n, n3 = I.n3, ld = I.ld;
  DBuf buf;
  RB_TRY(buf.alloc((size_t)(5 * ld + 18 * (size_t)n) * sizeof(double)));
  RB_CUDA(cudaMemset(buf.p, 0, (size_t)(5 * ld + 18 * (size_t)n) * sizeof(double)));
  double *Hf = buf.as<double>(), *Fv = Hf + ld, *dx = Fv + ld, *tmp = dx + ld, *Mt = tmp + ld;
  double *D = Mt + ld, *P = D + 9 * (size_t)n;
  double *M = I.M.as<double>();
  auto eval = [&](const double *Mx, double *misfit) -> int {
    RB_TRY(run_matvec(I, Mx, I.hext.as<double>(), 1.0, Hf, 0));
    nk_material_kernel<<<(n + 127) / 128, 128>>>(Hf, Mx, I.mat_kind.as<int>(), I.mat.as<double>(), n, Fv, D);
    RB_TRY(check_launch("nk_material_kernel"));
    double s;
    double *fv = Fv;
    RB_TRY(dots_many(&fv, 1, Fv, n3, &s));
    *misfit = sqrt(s / n);
    return 0;
  };
  double misfit;
  RB_TRY(eval(M, &misfit));
  int matvecs = 1, newton = 0;
  if (misfit > prec) {
    // Globalization: Newton from the remanent state overshoots deep into
    // saturation for soft iron (initial chi ~ 1e4).  A short Anderson-mixed
    // Jacobi phase (the method-9 iteration) brings M into the basin first;
    // its iterations count as matvecs.
    double st[4];
    int warm = std::min(300, std::max(1, max_iter / 4));
    double loose = std::max(prec, 1e-3 * std::max(misfit, 1e-12));
    RB_TRY(relax_jacobi(I, loose, warm, 0.0, st));
    matvecs += (int)st[3];
    RB_TRY(eval(M, &misfit));
    matvecs++;
  }
  while (misfit > prec && matvecs < max_iter && newton < 200) {
    newton++;
    if (I.N64.p) nk_precond_build<double><<<(n + 127) / 128, 128>>>(I.N64.as<double>(), ld, D, n, P);
    else nk_precond_build<float><<<(n + 127) / 128, 128>>>(I.N32.as<float>(), ld, D, n, P);
    RB_TRY(check_launch("nk_precond_build"));
    // solve (I - D N) dx = F  (Newton step M+dx); forcing term 0.1 * misfit-relative
    RB_CUDA(cudaMemset(dx, 0, n3 * sizeof(double)));
    NKOp op(I, D, P, tmp);
    double rel;
    int its;
    double eta = std::min(0.1, std::max(1e-3, misfit));
    RB_TRY(gmres(op, n3, ld, Fv, dx, eta, std::max(1, max_iter - matvecs), 40, &rel, &its, 0));
    matvecs += its + 1;
    // backtracking line search on the misfit
    double lam = 1.0, newmis = 0.0;
    for (int ls = 0; ls < 8; ls++) {
      RB_TRY(vcopy_axpy(Mt, M, 1.0, dx, lam, n3));
      RB_TRY(eval(Mt, &newmis));
      matvecs++;
      if (newmis < misfit || ls == 7) break;
      lam *= 0.5;
    }
    RB_CUDA(cudaMemcpy(M, Mt, n3 * sizeof(double), cudaMemcpyDeviceToDevice));
    misfit = newmis;
    if (!std::isfinite(misfit)) { set_error("Newton-Krylov: non-finite residual"); return RADB200_E_NUMERIC; }
  }
  // field of the final state (element fields = full H)
  RB_CUDA(cudaMemcpy(I.H.p, Hf, n3 * sizeof(double), cudaMemcpyDeviceToDevice));
  std::vector<double> hm(n3), hh(n3);
  RB_CUDA(cudaMemcpy(hm.data(), M, n3 * sizeof(double), cudaMemcpyDeviceToHost));
  RB_CUDA(cudaMemcpy(hh.data(), Hf, n3 * sizeof(double), cudaMemcpyDeviceToHost));
  double mm = 0, mh = 0;
  for (int e = 0; e < n; e++) {
    mm = std::max(mm, sqrt(hm[3 * e] * hm[3 * e] + hm[3 * e + 1] * hm[3 * e + 1] + hm[3 * e + 2] * hm[3 * e + 2]));
    mh = std::max(mh, sqrt(hh[3 * e] * hh[3 * e] + hh[3 * e + 1] * hh[3 * e + 1] + hh[3 * e + 2] * hh[3 * e + 2]));
  }
  status[0] = misfit; status[1] = mm; status[2] = mh; status[3] = matvecs;
  return 0;
}

}  // namespace rb
