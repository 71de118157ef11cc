// material.cuh -- per-element constitutive laws on the device.
//
//   linear (isotropic or anisotropic):  M = chi H + Mr
//       radTLinearAnisotropMaterial radmater.h:164-303, radTLinearIsotropMaterial :328-362
//   saturating isotropic formula:       |M| = sum ms_i tanh(ksi_i |H| / ms_i), M || H
//       radTNonlinearIsotropMaterial radmater.h:417-600, radmater.cpp:72-306
//   saturating isotropic table:         |M|(|H|) by cubic Hermite pieces between
//       the points (H_k, M_k) with the table's derivatives dM/dH_k at the nodes,
//       M || H (the same class with gArrayHM, radmater.cpp:618-710)
// Record layout: RADB200_MAT_STRIDE doubles, see include/radb200.h; the
// tables of all elements are rows (H, M, dM/dH) of one array mh.
#pragma once
#include "formulas.cuh"

namespace rb {

__device__ __forceinline__ void inv3x3(const double *A, double *B)
{
  double c0 = A[4] * A[8] - A[5] * A[7], c1 = A[5] * A[6] - A[3] * A[8], c2 = A[3] * A[7] - A[4] * A[6];
  double id = 1.0 / (A[0] * c0 + A[1] * c1 + A[2] * c2);
  B[0] = c0 * id; B[1] = (A[2] * A[7] - A[1] * A[8]) * id; B[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  B[3] = c1 * id; B[4] = (A[0] * A[8] - A[2] * A[6]) * id; B[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  B[6] = c2 * id; B[7] = (A[1] * A[6] - A[0] * A[7]) * id; B[8] = (A[0] * A[4] - A[1] * A[3]) * id;
}

// scalar law f(h) = |M|(|H|) and its derivative (radmater.cpp:279-306)
__device__ __forceinline__ void tanh_law(const double *m, double h, double &f, double &df)
{
  f = 0.0; df = 0.0;
  int n = (int)m[6];
  for (int i = 0; i < n; i++) {
    double ks = m[i], ms = m[3 + i];
    if (ms == 0.0) continue;
    double arg = ks * h / ms;
    double th = tanh(arg);
    f += ms * th;
    df += ks * (1.0 - th * th);  // ks / cosh^2
  }
}

__device__ __forceinline__ double tanh_ksi0(const double *m)
{
  double k = 0.0;
  for (int i = 0; i < (int)m[6]; i++) k += m[i];
  return k;
}

// Tabulated law at |H| = h: m[0] first row of the element's table in mh,
// m[1] its rows.  Below the first point the first M (derivative: the first
// node's); above the last point M continues along the last node's slope for
// M(H) (AbsMvsAbsH_Interpol, radmater.cpp:619-646) while the pair used for
// dM/dH stops there with zero slope (AbsMvsAbsH_FuncAndDer_Interpol,
// :678-710); in between the cubic with the end values and slopes of the piece
// (CubPln, radmater.h:631-639).
__device__ __forceinline__ void table_law(const double *__restrict__ mh, const double *m, double h, bool for_der,
                                          double &f, double &df)
{
  const int L = (int)m[1];
  const double *T = mh + 3 * (size_t)m[0];
  int k = 0;
  while (k < L && T[3 * k] <= h) k++;
  k--;  // last node at or below h
  if (k < 0) { f = T[1]; df = T[2]; return; }
  if (k >= L - 1) {
    const double *t = T + 3 * (L - 1);
    if (for_der) { f = t[1]; df = 0.0; }
    else { f = t[1] + (h - t[0]) * t[2]; df = t[2]; }
    return;
  }
  const double *t = T + 3 * k;
  const double step = t[3] - t[0], is = 1.0 / step, sl = (t[4] - t[1]) * is;
  const double a0 = t[1], a1 = t[2], a2 = (3.0 * sl - 2.0 * t[2] - t[5]) * is, a3 = (-2.0 * sl + t[2] + t[5]) * is * is;
  const double x = h - t[0];
  f = a0 + x * (a1 + x * (a2 + x * a3));
  df = a1 + x * (2.0 * a2 + x * 3.0 * a3);
}

// |M| and |M| / |H| of a saturating law at |H| = h > 0
__device__ __forceinline__ double sat_abs_m(int kind, const double *m, const double *__restrict__ mh, double h)
{
  double f, df;
  if (kind == RADB200_MAT_TABLE) table_law(mh, m, h, false, f, df);
  else tanh_law(m, h, f, df);
  return f;
}

// M(H) for element material (kind, m); mh: the table rows (table laws only)
__device__ __forceinline__ V3<double> mat_M(int kind, const double *m, V3<double> H, const double *__restrict__ mh)
{
  if (kind == RADB200_MAT_LINEAR)
    return mk3<double>(m[0] * H.x + m[1] * H.y + m[2] * H.z + m[9], m[3] * H.x + m[4] * H.y + m[5] * H.z + m[10],
                       m[6] * H.x + m[7] * H.y + m[8] * H.z + m[11]);
  double h = sqrt(H.x * H.x + H.y * H.y + H.z * H.z);
  double ksi;
  if (kind == RADB200_MAT_TABLE) {
    if (h == 0.0) return mk3<double>(m[9], m[10], m[11]);
    ksi = sat_abs_m(kind, m, mh, h) / h;
  } else if (h <= 1e-10) ksi = tanh_ksi0(m);
  else ksi = sat_abs_m(kind, m, mh, h) / h;
  return mk3<double>(ksi * H.x + m[9], ksi * H.y + m[10], ksi * H.z + m[11]);
}

// dM/dH at H (radmater.cpp:206-306; linear: chi tensor)
__device__ __forceinline__ void mat_D(int kind, const double *m, V3<double> H, double *D, const double *__restrict__ mh)
{
  if (kind == RADB200_MAT_LINEAR) {
    for (int k = 0; k < 9; k++) D[k] = m[k];
    return;
  }
  double h0 = sqrt(H.x * H.x + H.y * H.y + H.z * H.z);
  double f, df;
  if (kind == RADB200_MAT_TABLE) {
    if (h0 < 1e-10) { f = 0.0; df = mh[3 * (size_t)m[0] + 2]; }
    else table_law(mh, m, h0, true, f, df);
  } else tanh_law(m, h0, f, df);
  if (h0 < 1e-10) {
    for (int k = 0; k < 9; k++) D[k] = (k % 4 == 0) ? df : 0.0;
    return;
  }
  double ih3 = 1.0 / (h0 * h0 * h0);
  double off = ih3 * (h0 * df - f);
  D[0] = ih3 * ((H.y * H.y + H.z * H.z) * f + H.x * H.x * h0 * df);
  D[4] = ih3 * ((H.x * H.x + H.z * H.z) * f + H.y * H.y * h0 * df);
  D[8] = ih3 * ((H.x * H.x + H.y * H.y) * f + H.z * H.z * h0 * df);
  D[1] = D[3] = off * H.x * H.y;
  D[2] = D[6] = off * H.x * H.z;
  D[5] = D[7] = off * H.y * H.z;
}

// FindNewH: solve H = Hq + Q_ii M(H) for the element's own field.
// Linear: H = (I - Q chi)^-1 (Hq + Q Mr)  (radmater.h:223-231).
// Saturating: damped secant on |H| with at most 15 passes (radmater.cpp:72-164).
__device__ __forceinline__ V3<double> find_new_h(int kind, const double *m, const double *Q, V3<double> Hq,
                                                 V3<double> H0, double prec_e2, const double *__restrict__ mh)
{
  double A[9], Ai[9];
  if (kind == RADB200_MAT_LINEAR) {
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        A[3 * a + b] = (a == b ? 1.0 : 0.0) - (Q[3 * a] * m[b] + Q[3 * a + 1] * m[3 + b] + Q[3 * a + 2] * m[6 + b]);
    inv3x3(A, Ai);
    double rx = Hq.x + Q[0] * m[9] + Q[1] * m[10] + Q[2] * m[11];
    double ry = Hq.y + Q[3] * m[9] + Q[4] * m[10] + Q[5] * m[11];
    double rz = Hq.z + Q[6] * m[9] + Q[7] * m[10] + Q[8] * m[11];
    return mk3<double>(Ai[0] * rx + Ai[1] * ry + Ai[2] * rz, Ai[3] * rx + Ai[4] * ry + Ai[5] * rz,
                       Ai[6] * rx + Ai[7] * ry + Ai[8] * rz);
  }
  double misfit = 3.0;
  double ah = sqrt(H0.x * H0.x + H0.y * H0.y + H0.z * H0.z);
  V3<double> H = H0;
  for (int it = 0; it < 15; it++) {
    double f = 0.0, ksi;
    if (ah <= 1e-10) { ksi = (kind == RADB200_MAT_TABLE) ? mh[3 * (size_t)m[0] + 2] : tanh_ksi0(m); f = 0.0; }
    else { f = sat_abs_m(kind, m, mh, ah); ksi = f / ah; }
    for (int k = 0; k < 9; k++) A[k] = ((k % 4) == 0 ? 1.0 : 0.0) - ksi * Q[k];
    inv3x3(A, Ai);
    H = mk3<double>(Ai[0] * Hq.x + Ai[1] * Hq.y + Ai[2] * Hq.z, Ai[3] * Hq.x + Ai[4] * Hq.y + Ai[5] * Hq.z,
                    Ai[6] * Hq.x + Ai[7] * Hq.y + Ai[8] * Hq.z);
    double nah = sqrt(H.x * H.x + H.y * H.y + H.z * H.z);
    double nmis = f - nah * ksi;
    double am = fabs(misfit), anm = fabs(nmis);
    double pn = am;
    if (nmis * misfit > 0) pn += 0.5 * anm;
    double alpha = pn / (pn + anm);
    ah = alpha * nah + (1.0 - alpha) * ah;
    misfit = f - ah * ksi;
    if (misfit * misfit <= prec_e2) break;
  }
  return H;
}

// Newton polish of the element's implicit field, H = Hq + Q M(H), from
// find_new_h's result: J = I - Q dM/dH, at most 20 steps, each kept only if
// it lowers the residual.  find_new_h stops after 15 passes of a linearly
// converging secant, so its H carries an error that changes from one
// iteration to the next: a Newton iteration on the relaxation as a whole
// falls back to linear convergence on it, and Anderson mixing stalls (a
// 12-element saturating hybrid stopped at a misfit of 4e-5 after 2,000
// Jacobi iterations).  Polished, the fixed-point map is exact to rounding:
// the outer Newton converges quadratically and the Jacobi iteration reaches
// 1e-12 in about a hundred iterations.
__device__ __forceinline__ double implicit_residual(int kind, const double *m, const double *Q, V3<double> Hq,
                                                    V3<double> H, const double *__restrict__ mh, double *r)
{
  const V3<double> M = mat_M(kind, m, H, mh);
  r[0] = H.x - Hq.x - (Q[0] * M.x + Q[1] * M.y + Q[2] * M.z);
  r[1] = H.y - Hq.y - (Q[3] * M.x + Q[4] * M.y + Q[5] * M.z);
  r[2] = H.z - Hq.z - (Q[6] * M.x + Q[7] * M.y + Q[8] * M.z);
  return sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

__device__ __forceinline__ V3<double> polish_h(int kind, const double *m, const double *Q, V3<double> Hq, V3<double> H,
                                               const double *__restrict__ mh)
{
  if (kind == RADB200_MAT_LINEAR) return H;
  double r[3], rn = implicit_residual(kind, m, Q, Hq, H, mh, r);
  for (int it = 0; it < 20; it++) {
    const double hn = sqrt(H.x * H.x + H.y * H.y + H.z * H.z);
    if (!(rn > 1e-16 * fmax(hn, 1e-30))) break;
    double D[9], A[9], Ai[9];
    mat_D(kind, m, H, D, mh);
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        A[3 * a + b] = (a == b ? 1.0 : 0.0) - (Q[3 * a] * D[b] + Q[3 * a + 1] * D[3 + b] + Q[3 * a + 2] * D[6 + b]);
    inv3x3(A, Ai);
    const V3<double> Hn = mk3<double>(H.x - (Ai[0] * r[0] + Ai[1] * r[1] + Ai[2] * r[2]),
                                      H.y - (Ai[3] * r[0] + Ai[4] * r[1] + Ai[5] * r[2]),
                                      H.z - (Ai[6] * r[0] + Ai[7] * r[1] + Ai[8] * r[2]));
    double r2[3];
    const double rn2 = implicit_residual(kind, m, Q, Hq, Hn, mh, r2);
    if (!(rn2 < rn)) break;
    H = Hn;
    rn = rn2;
    r[0] = r2[0]; r[1] = r2[1]; r[2] = r2[2];
  }
  return H;
}

}  // namespace rb
