// adjoint.cu -- hand-written adjoint of the relaxation and of the field operator.
//
// Forward problem (element frames): M solves r(M, p) = M_mat(H_ext + N M) - M = 0.
// For a scalar loss L(M, p), dL/dp = dL/dp|_M + lambda^T dr/dp with
//     (I - D N)^T lambda = dL/dM,        D = dM/dH at the converged H
// (D: radmater.cpp:206-277).  dr/dp = D dH/dp + dM_mat/dp|_H, so with
// mu = D^T lambda the geometric part is mu^T (dH_ext/dp + (dN/dp) M).
//
// Transposed solve.  After a direct (linear) solve the LU factors of
// A = I - chi N are kept: A^T = U^T L^T is solved with the transposed
// diagonal-block inverses and serves as the preconditioner of FP64 GMRES on
// A^T.  Otherwise the system is split with the self blocks Qd (the diagonal
// 3x3 blocks of N):
//     I - D N = P (I - B N'),   P = I - D Qd,   B = P^-1 D,   N' = N - Qd,
// so (I - D N)^T lambda = g  <=>  (I - N'^T B^T) z = g,  lambda = P^-T z:
// GMRES on the transpose of the implicit Jacobi map that the forward
// relaxation iterates (radrlmet.cpp:496-587).
//
// Geometric derivatives.  The cuboid tensor (radrec.cpp:115-283) is a sum
// over the 8 corners: with (X, Y, Z) = q - (ex hx, ey hy, ez hz), R its norm
// and p = ex ey ez,
//     Q_xx = 1/(4 pi) sum p atan(Y Z / (X R)),   Q_xy = -1/(4 pi) sum p log(Z + R)
// (the other entries by permutation; atan branch constants drop out of
// derivatives), so dQ/dq and dQ/dh are corner sums of rational functions of
// X, Y, Z, R.  They are evaluated pair by pair and contracted at once with the
// loss weights; dN/dp is never stored.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "tensor.cuh"
#include "material.cuh"

namespace rb {

// ---- cuboid tensor derivative, contracted -----------------------------------
// w = symmetric weights (xx, yy, zz, xy, xz, yz) of u^T Q m:
//   (u_x m_x, u_y m_y, u_z m_z, u_x m_y + u_y m_x, u_x m_z + u_z m_x, u_y m_z + u_z m_y).
// dq[a] += d(u^T Q m)/dq_a, dh[a] += d(u^T Q m)/dh_a (q relative to the
// centre, h half widths).  A corner whose edge line passes through q is
// skipped (the derivative is singular there).
__device__ __forceinline__ void cuboid_dQ(V3<double> q, V3<double> hd, const double *w, double *dq, double *dh)
{
  // the cuboid form's full-precision pi (radrec.cpp:130), as in the forward cuboid term
  const double C = 1.0 / (4.0 * 3.141592653589793238);
  double gq0 = 0, gq1 = 0, gq2 = 0, gh0 = 0, gh1 = 0, gh2 = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const double ex = (c & 1) ? 1.0 : -1.0, ey = (c & 2) ? 1.0 : -1.0, ez = (c & 4) ? 1.0 : -1.0;
    const double p = ex * ey * ez;
    double X = q.x - ex * hd.x, Y = q.y - ey * hd.y, Z = q.z - ez * hd.z;
    double xx = X * X, yy = Y * Y, zz = Z * Z;
    double sxy = xx + yy, sxz = xx + zz, syz = yy + zz;
    if (!(sxy > 0.0 && sxz > 0.0 && syz > 0.0)) continue;
    // 1/R by rsqrt; the three 1/(a^2 + b^2) from one division of their product
    const double iR = rsqrt(sxy + zz), R = (sxy + zz) * iR;
    const double pxy = sxz * syz, inv3 = 1.0 / (sxy * pxy);
    const double ixy = pxy * inv3, ixz = sxy * syz * inv3, iyz = sxy * sxz * inv3;
    // 1/(Z + R) without cancellation for negative Z: (R - Z)/(X^2 + Y^2), etc.;
    // the divisions of the non-negative cases merged into one
    const double dz = Z >= 0.0 ? Z + R : 1.0, dy = Y >= 0.0 ? Y + R : 1.0, dx = X >= 0.0 ? X + R : 1.0;
    const double invd = 1.0 / (dz * dy * dx);
    const double izr = Z >= 0.0 ? dy * dx * invd : (R - Z) * ixy;
    const double iyr = Y >= 0.0 ? dz * dx * invd : (R - Y) * ixz;
    const double ixr = X >= 0.0 ? dz * dy * invd : (R - X) * iyz;
    double XiR = X * iR, YiR = Y * iR, ZiR = Z * iR;
    double YZ = Y * ZiR, XZ = X * ZiR, XY = X * YiR;
    double gx = -w[0] * YZ * (ixz + ixy) + w[1] * YZ * ixy + w[2] * YZ * ixz;
    double gy = w[0] * XZ * ixy - w[1] * XZ * (iyz + ixy) + w[2] * XZ * iyz;
    double gz = w[0] * XY * ixz + w[1] * XY * iyz - w[2] * XY * (iyz + ixz);
    gx -= w[3] * XiR * izr + w[4] * XiR * iyr + w[5] * iR;
    gy -= w[3] * YiR * izr + w[4] * iR + w[5] * YiR * ixr;
    gz -= w[3] * iR + w[4] * ZiR * iyr + w[5] * ZiR * ixr;
    gq0 += p * gx; gq1 += p * gy; gq2 += p * gz;
    gh0 -= p * ex * gx; gh1 -= p * ey * gy; gh2 -= p * ez * gz;
  }
  dq[0] += C * gq0; dq[1] += C * gq1; dq[2] += C * gq2;
  dh[0] += C * gh0; dh[1] += C * gh1; dh[2] += C * gh2;
}

struct SrcInfo {
  int kind, idx, t0, nt;
  V3<double> c, hd;
  double m0, m1, m2;
};

__device__ __forceinline__ SrcInfo load_src(const GeomView &g, const int *elem_src, const double *m, int j)
{
  SrcInfo s;
  s.kind = __ldg(elem_src + 2 * j);
  s.idx = __ldg(elem_src + 2 * j + 1);
  if (s.kind == 0) {
    s.t0 = __ldg(g.rec_img + 2 * s.idx);
    s.nt = __ldg(g.rec_img + 2 * s.idx + 1);
    const double *r = g.rec + (size_t)s.idx * RADB200_REC_STRIDE;
    s.c = mk3<double>(__ldg(r), __ldg(r + 1), __ldg(r + 2));
    s.hd = mk3<double>(0.5 * __ldg(r + 3), 0.5 * __ldg(r + 4), 0.5 * __ldg(r + 5));
  } else {
    s.t0 = __ldg(g.poly_info + 4 * s.idx + 2);
    s.nt = __ldg(g.poly_info + 4 * s.idx + 3);
    s.c = mk3<double>(0, 0, 0);
    s.hd = s.c;
  }
  s.m0 = __ldg(m + 3 * j); s.m1 = __ldg(m + 3 * j + 1); s.m2 = __ldg(m + 3 * j + 2);
  return s;
}

// One (observer x with lab weight u, source s) pair over all images of s.
//   aM += G^T u           (G: lab field at x per unit source magnetization)
//   ac -= d(u.G m)/dq     (= d/dc of the source centre, object frame)
//   ad += d(u.G m)/dd     (full widths)
//   ax += d(u.G m)/dx     (observer position, lab)
template <bool WANT_M, bool WANT_SRC, bool WANT_OBS, bool RECT_ONLY = false>
__device__ __forceinline__ void pair_adj(const GeomView &g, const SrcInfo &s, V3<double> x, V3<double> u, int what,
                                         double *aM, double *ac, double *ad, double *ax)
{
  for (int t = s.t0; t < s.t0 + s.nt; t++) {
    const double *Tr = g.trf + (size_t)t * RADB200_TRF_STRIDE;
    double r0 = __ldg(Tr), r1 = __ldg(Tr + 1), r2 = __ldg(Tr + 2), r3 = __ldg(Tr + 3), r4 = __ldg(Tr + 4),
           r5 = __ldg(Tr + 5), r6 = __ldg(Tr + 6), r7 = __ldg(Tr + 7), r8 = __ldg(Tr + 8);
    double dx = x.x - __ldg(Tr + 9), dy = x.y - __ldg(Tr + 10), dz = x.z - __ldg(Tr + 11);
    V3<double> q = mk3<double>(r0 * dx + r1 * dy + r2 * dz, r3 * dx + r4 * dy + r5 * dz, r6 * dx + r7 * dy + r8 * dz);
    const double *F = Tr + 12;
    // u~ = F^T u (the weight in the source's object frame)
    double ut0 = __ldg(F) * u.x + __ldg(F + 3) * u.y + __ldg(F + 6) * u.z;
    double ut1 = __ldg(F + 1) * u.x + __ldg(F + 4) * u.y + __ldg(F + 7) * u.z;
    double ut2 = __ldg(F + 2) * u.x + __ldg(F + 5) * u.y + __ldg(F + 8) * u.z;
    if (WANT_M) {
      double Q[9];
      if (RECT_ONLY) cuboid_tensor(g, s.idx, q, Q);
      else elem_tensor(g, s.kind, s.idx, q, Q);
      aM[0] += Q[0] * ut0 + Q[3] * ut1 + Q[6] * ut2;
      aM[1] += Q[1] * ut0 + Q[4] * ut1 + Q[7] * ut2;
      aM[2] += Q[2] * ut0 + Q[5] * ut1 + Q[8] * ut2;
      if (what == 0 && elem_inside(g, RECT_ONLY ? 0 : s.kind, s.idx, q)) { aM[0] += ut0; aM[1] += ut1; aM[2] += ut2; }
    }
    if ((WANT_SRC || WANT_OBS) && s.kind == 0) {
      double w[6] = {ut0 * s.m0, ut1 * s.m1, ut2 * s.m2, ut0 * s.m1 + ut1 * s.m0, ut0 * s.m2 + ut2 * s.m0,
                     ut1 * s.m2 + ut2 * s.m1};
      double dq[3] = {0, 0, 0}, dh[3] = {0, 0, 0};
      cuboid_dQ(mk3<double>(q.x - s.c.x, q.y - s.c.y, q.z - s.c.z), s.hd, w, dq, dh);
      if (WANT_SRC) {
        ac[0] -= dq[0]; ac[1] -= dq[1]; ac[2] -= dq[2];
        ad[0] += 0.5 * dh[0]; ad[1] += 0.5 * dh[1]; ad[2] += 0.5 * dh[2];
      }
      if (WANT_OBS) {
        ax[0] += r0 * dq[0] + r3 * dq[1] + r6 * dq[2];
        ax[1] += r1 * dq[0] + r4 * dq[1] + r7 * dq[2];
        ax[2] += r2 * dq[0] + r5 * dq[1] + r8 * dq[2];
      }
    }
  }
}

constexpr int ADJ_T = 128;

// Thread per source j; observers [k0, k1) of chunk blockIdx.y staged in shared
// memory.  part[chunk][j][9] = (aM, ac, ad).  The kernel waits on FP64
// latency, so the M-gradient variant is held to 168 registers (3 blocks, 12
// warps per SM, a few dozen bytes of spill) instead of 182 (8 warps); the
// variant without it fits 4 blocks at 127.
template <bool WANT_M, bool RECT_ONLY>
__global__ void __launch_bounds__(ADJ_T, WANT_M ? 3 : 4) adj_src_kernel(GeomView g, const int *__restrict__ elem_src,
                                                        const double *__restrict__ m, int n, const double *__restrict__ X,
                                                        const double *__restrict__ U, int nobs, int per_chunk, int what,
                                                        double *__restrict__ part)
{
  __shared__ double sx[ADJ_T * 6];
  int j = blockIdx.x * ADJ_T + threadIdx.x;
  int k0 = blockIdx.y * per_chunk, k1 = min(nobs, k0 + per_chunk);
  SrcInfo s;
  if (j < n) s = load_src(g, elem_src, m, j);
  double aM[3] = {0, 0, 0}, ac[3] = {0, 0, 0}, ad[3] = {0, 0, 0};
  for (int base = k0; base < k1; base += ADJ_T) {
    __syncthreads();
    int k = base + threadIdx.x;
    if (k < k1) {
      for (int a = 0; a < 3; a++) {
        sx[6 * threadIdx.x + a] = X[3 * (size_t)k + a];
        sx[6 * threadIdx.x + 3 + a] = U[3 * (size_t)k + a];
      }
    }
    __syncthreads();
    int cnt = min(ADJ_T, k1 - base);
    if (j < n)
      for (int kk = 0; kk < cnt; kk++) {
        const double *o = sx + 6 * kk;
        pair_adj<WANT_M, true, false, RECT_ONLY>(g, s, mk3<double>(o[0], o[1], o[2]), mk3<double>(o[3], o[4], o[5]), what,
                                                 aM, ac, ad, nullptr);
      }
  }
  if (j < n) {
    double *o = part + ((size_t)blockIdx.y * n + j) * 9;
    for (int a = 0; a < 3; a++) { o[a] = aM[a]; o[3 + a] = ac[a]; o[6 + a] = ad[a]; }
  }
}

// Thread per observer k; sources [j0, j1) of chunk blockIdx.y.
// part[chunk][k][3] = d(u_k . G m)/dx_k.
__global__ void __launch_bounds__(ADJ_T) adj_obs_kernel(GeomView g, const int *__restrict__ elem_src,
                                                        const double *__restrict__ m, int n, const double *__restrict__ X,
                                                        const double *__restrict__ U, int nobs, int per_chunk,
                                                        double *__restrict__ part)
{
  int k = blockIdx.x * ADJ_T + threadIdx.x;
  int j0 = blockIdx.y * per_chunk, j1 = min(n, j0 + per_chunk);
  if (k >= nobs) return;
  V3<double> x = mk3<double>(X[3 * (size_t)k], X[3 * (size_t)k + 1], X[3 * (size_t)k + 2]);
  V3<double> u = mk3<double>(U[3 * (size_t)k], U[3 * (size_t)k + 1], U[3 * (size_t)k + 2]);
  double ax[3] = {0, 0, 0};
  for (int j = j0; j < j1; j++) {
    SrcInfo s = load_src(g, elem_src, m, j);
    if (s.kind != 0) continue;
    pair_adj<false, false, true>(g, s, x, u, 1, nullptr, nullptr, nullptr, ax);
  }
  double *o = part + ((size_t)blockIdx.y * nobs + k) * 3;
  o[0] = ax[0]; o[1] = ax[1]; o[2] = ax[2];
}

// out[i] = sum over chunks of part[c][i], fixed order
__global__ void adj_reduce_kernel(const double *__restrict__ part, int nchunk, int64_t len, double *__restrict__ out)
{
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; c++) s += part[(size_t)c * len + i];
  out[i] = s;
}

// ---- transposed matvec: part[chunk][col] = sum_{rows of chunk} N[row][col] x[row]
template <typename MT> struct Vec16;
template <> struct Vec16<float> {
  static constexpr int V = 4;
  __device__ static void load(const float *p, double *v)
  {
    float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  }
};
template <> struct Vec16<double> {
  static constexpr int V = 2;
  __device__ static void load(const double *p, double *v)
  {
    double2 t = __ldg(reinterpret_cast<const double2 *>(p));
    v[0] = t.x; v[1] = t.y;
  }
};

template <typename MT>
__global__ void __launch_bounds__(ADJ_T) matvec_t_kernel(const MT *__restrict__ N, int ld, int n3,
                                                         const double *__restrict__ x, int rows_per_chunk,
                                                         double *__restrict__ part)
{
  constexpr int V = Vec16<MT>::V;
  int col = (blockIdx.x * ADJ_T + threadIdx.x) * V;
  int r0 = blockIdx.y * rows_per_chunk, r1 = min(n3, r0 + rows_per_chunk);
  if (col >= ld) return;
  double acc[V];
#pragma unroll
  for (int v = 0; v < V; v++) acc[v] = 0.0;
  const MT *p = N + (size_t)r0 * ld + col;
  int r = r0;
  for (; r + 4 <= r1; r += 4, p += 4 * (size_t)ld) {
    double a[4][V];
#pragma unroll
    for (int u = 0; u < 4; u++) Vec16<MT>::load(p + (size_t)u * ld, a[u]);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      double xr = __ldg(x + r + u);
#pragma unroll
      for (int v = 0; v < V; v++) acc[v] = fma(a[u][v], xr, acc[v]);
    }
  }
  for (; r < r1; r++, p += ld) {
    double a[V];
    Vec16<MT>::load(p, a);
    double xr = __ldg(x + r);
#pragma unroll
    for (int v = 0; v < V; v++) acc[v] = fma(a[v], xr, acc[v]);
  }
  double *o = part + (size_t)blockIdx.y * ld + col;
#pragma unroll
  for (int v = 0; v < V; v++) o[v] = acc[v];
}

// ---- per-element coefficients of the transposed operator --------------------
// coef[e] = B^T (9), P^-T (9), Qd^T (9); lu != 0: B^T = chi^T, P^-T = I, Qd^T = 0.
template <typename MT>
__global__ void adj_prep_kernel(const MT *__restrict__ N, int ld, int n, const double *__restrict__ H,
                                const int *__restrict__ kind, const double *__restrict__ mat,
                                const double *__restrict__ mh, int lu, double *__restrict__ coef)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double D[9], *c = coef + (size_t)e * 27;
  mat_D(kind[e], mat + (size_t)e * RADB200_MAT_STRIDE, mk3<double>(H[3 * e], H[3 * e + 1], H[3 * e + 2]), D, mh);
  if (lu) {
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        c[3 * a + b] = D[3 * b + a];
        c[9 + 3 * a + b] = (a == b) ? 1.0 : 0.0;
        c[18 + 3 * a + b] = 0.0;
      }
    return;
  }
  double Q[9], P[9], Pi[9];
  const MT *d = N + (size_t)(3 * e) * ld + 3 * e;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) Q[3 * a + b] = (double)d[(size_t)a * ld + b];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      P[3 * a + b] = (a == b ? 1.0 : 0.0) - (D[3 * a] * Q[b] + D[3 * a + 1] * Q[3 + b] + D[3 * a + 2] * Q[6 + b]);
  inv3x3(P, Pi);
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      double B = Pi[3 * a] * D[b] + Pi[3 * a + 1] * D[3 + b] + Pi[3 * a + 2] * D[6 + b];  // (P^-1 D)_ab
      c[3 * b + a] = B;
      c[9 + 3 * b + a] = Pi[3 * a + b];
      c[18 + 3 * b + a] = Q[3 * a + b];
    }
}

// y_e = C_e x_e for the 3x3 block `which` (0 B^T, 1 P^-T, 2 Qd^T) of coef
__global__ void adj_block_kernel(const double *__restrict__ coef, int which, int n, const double *__restrict__ x,
                                 double *__restrict__ y)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double *C = coef + (size_t)e * 27 + 9 * which;
  double x0 = x[3 * e], x1 = x[3 * e + 1], x2 = x[3 * e + 2];
  y[3 * e] = C[0] * x0 + C[1] * x1 + C[2] * x2;
  y[3 * e + 1] = C[3] * x0 + C[4] * x1 + C[5] * x2;
  y[3 * e + 2] = C[6] * x0 + C[7] * x1 + C[8] * x2;
}

// out_e = v_e - sum_chunks part[.][3e..] + (use_qd ? Qd_e^T t_e : 0)
__global__ void adj_finish_kernel(const double *__restrict__ part, int nchunk, int ld, int n, const double *__restrict__ v,
                                  const double *__restrict__ t, const double *__restrict__ coef, int use_qd,
                                  double *__restrict__ out)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double y[3];
  for (int a = 0; a < 3; a++) {
    double s = 0.0;
    for (int c = 0; c < nchunk; c++) s += part[(size_t)c * ld + 3 * e + a];
    y[a] = s;
  }
  if (use_qd) {
    const double *C = coef + (size_t)e * 27 + 18;
    double t0 = t[3 * e], t1 = t[3 * e + 1], t2 = t[3 * e + 2];
    y[0] -= C[0] * t0 + C[1] * t1 + C[2] * t2;
    y[1] -= C[3] * t0 + C[4] * t1 + C[5] * t2;
    y[2] -= C[6] * t0 + C[7] * t1 + C[8] * t2;
  }
  for (int a = 0; a < 3; a++) out[3 * e + a] = v[3 * e + a] - y[a];
}

// X_e = D_e = dM/dH at H_e, in the layout of a material record's chi slots
__global__ void adj_dmat_kernel(const double *__restrict__ H, const int *__restrict__ kind, const double *__restrict__ mat,
                                const double *__restrict__ mh, int n, double *__restrict__ X)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double D[9];
  mat_D(kind[e], mat + (size_t)e * RADB200_MAT_STRIDE, mk3<double>(H[3 * e], H[3 * e + 1], H[3 * e + 2]), D, mh);
  for (int k = 0; k < 9; k++) X[(size_t)e * RADB200_MAT_STRIDE + k] = D[k];
  for (int k = 9; k < RADB200_MAT_STRIDE; k++) X[(size_t)e * RADB200_MAT_STRIDE + k] = 0.0;
}

// u_e = rowT_e^T D_e^T lambda_e (lab-frame weight of element e's field row)
__global__ void adj_weight_kernel(const double *__restrict__ lambda, const double *__restrict__ H,
                                  const int *__restrict__ kind, const double *__restrict__ mat,
                                  const double *__restrict__ mh, const double *__restrict__ rowT, int n,
                                  double *__restrict__ u)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double D[9];
  mat_D(kind[e], mat + (size_t)e * RADB200_MAT_STRIDE, mk3<double>(H[3 * e], H[3 * e + 1], H[3 * e + 2]), D, mh);
  double l0 = lambda[3 * e], l1 = lambda[3 * e + 1], l2 = lambda[3 * e + 2];
  double mu[3];
  for (int b = 0; b < 3; b++) mu[b] = D[b] * l0 + D[3 + b] * l1 + D[6 + b] * l2;
  const double *R = rowT + (size_t)e * 9;
  for (int b = 0; b < 3; b++) u[3 * e + b] = R[b] * mu[0] + R[3 + b] * mu[1] + R[6 + b] * mu[2];
}

// ---- host side -----------------------------------------------------------------
static int matvec_t(Intrc &I, const double *x, DBuf &part, int *nchunk_out, cudaStream_t st)
{
  const int V = I.N64.p ? 2 : 4;
  int tiles = (I.ld / V + ADJ_T - 1) / ADJ_T;
  int nchunk = std::max(1, std::min(64, (148 * 4 + tiles - 1) / tiles));
  int rows = (I.n3 + nchunk - 1) / nchunk;
  nchunk = (I.n3 + rows - 1) / rows;
  // mixed storage: one more partial slice holds the near residue's D^T x
  const int extra = I.near_nnz > 0 ? 1 : 0;
  RB_TRY(part.alloc((size_t)(nchunk + extra) * I.ld * sizeof(double)));
  dim3 grid(tiles, nchunk);
  if (I.N64.p) matvec_t_kernel<double><<<grid, ADJ_T, 0, st>>>(I.N64.as<double>(), I.ld, I.n3, x, rows, part.as<double>());
  else matvec_t_kernel<float><<<grid, ADJ_T, 0, st>>>(I.N32.as<float>(), I.ld, I.n3, x, rows, part.as<double>());
  RB_TRY(check_launch("matvec_t_kernel"));
  if (extra) {
    double *slice = part.as<double>() + (size_t)nchunk * I.ld;
    RB_CUDA(cudaMemsetAsync(slice, 0, (size_t)I.ld * sizeof(double), st));
    RB_TRY(launch_near_t(I, x, slice, st));
  }
  *nchunk_out = nchunk + extra;
  return 0;
}

struct AdjOp : Op {
  Intrc &I;
  const double *coef;
  double *t;
  DBuf &part;
  int use_lu;
  AdjOp(Intrc &i, const double *c, double *tt, DBuf &p, int lu) : I(i), coef(c), t(tt), part(p), use_lu(lu) {}
  int apply(const double *v, double *out) override
  {
    int nb = (I.n + 127) / 128, nchunk = 0;
    adj_block_kernel<<<nb, 128>>>(coef, 0, I.n, v, t);
    RB_TRY(check_launch("adj_block_kernel"));
    RB_TRY(matvec_t(I, t, part, &nchunk, 0));
    adj_finish_kernel<<<nb, 128>>>(part.as<double>(), nchunk, I.ld, I.n, v, t, coef, !use_lu, out);
    return check_launch("adj_finish_kernel");
  }
  int precond(double *v) override { return use_lu ? lu_precond_transposed(I, v, 0) : 0; }
};

// H = N M + H_ext at the last converged magnetization
static int converged_H(Intrc &I, double *H)
{
  return run_matvec(I, I.lastM.as<double>(), I.hext.as<double>(), 1.0, H, 0);
}

static bool all_linear(const Intrc &I)
{
  for (int k : I.h_mat_kind)
    if (k != RADB200_MAT_LINEAR) return false;
  return true;
}

int adjoint_solve(Intrc &I, const double *dLdM, double rtol, int max_iter, double *lambda, double *status)
{
  auto t0 = std::chrono::steady_clock::now();
  const int n = I.n, n3 = I.n3, ld = I.ld;
  // factors of the forward matrix itself after a direct (linear) solve
  int use_lu = (all_linear(I) && I.last_kind == 1 && I.lu_mode >= 0 && !I.lu_of_d) ? 1 : 0;
  DBuf buf, coef, part;
  RB_TRY(buf.alloc((size_t)4 * ld * sizeof(double)));
  RB_CUDA(cudaMemset(buf.p, 0, (size_t)4 * ld * sizeof(double)));
  double *g = buf.as<double>(), *x = g + ld, *t = x + ld, *H = t + ld;
  RB_CUDA(cudaMemcpy(g, dLdM, n3 * sizeof(double), cudaMemcpyHostToDevice));
  RB_TRY(converged_H(I, H));
  RB_TRY(coef.alloc((size_t)n * 27 * sizeof(double)));
  int nb = (n + 127) / 128;
  double tfac = 0.0;
  if (!use_lu) {
    // factor A = I - D N at the converged state (TF32 tensor cores with FP64
    // refinement for large systems) and precondition the transposed GMRES with
    // A^T = U^T L^T; kept until the next solve.  If the unpivoted factorization
    // breaks down, the block-Jacobi split of the operator is used instead.
    if (I.lu_of_d && I.lu_solve_id == I.solve_id && I.lu_mode >= 0) {
      use_lu = 1;
    } else {
      DBuf X;
      RB_TRY(X.alloc((size_t)n * RADB200_MAT_STRIDE * sizeof(double)));
      adj_dmat_kernel<<<nb, 128>>>(H, I.mat_kind.as<int>(), I.mat.as<double>(), I.mh.as<double>(), n, X.as<double>());
      RB_TRY(check_launch("adj_dmat_kernel"));
      const int mode = n3 >= 3072 ? RADB200_LU_TF32 : RADB200_LU_F64;
      if (lu_build_x(I, mode, X.as<double>(), 1, &tfac) == 0) use_lu = 1;
    }
  }
  if (I.N64.p)
    adj_prep_kernel<double><<<nb, 128>>>(I.N64.as<double>(), ld, n, H, I.mat_kind.as<int>(), I.mat.as<double>(), I.mh.as<double>(), use_lu,
                                         coef.as<double>());
  else
    adj_prep_kernel<float><<<nb, 128>>>(I.N32.as<float>(), ld, n, H, I.mat_kind.as<int>(), I.mat.as<double>(), I.mh.as<double>(), use_lu,
                                        coef.as<double>());
  RB_TRY(check_launch("adj_prep_kernel"));
  AdjOp op(I, coef.as<double>(), t, part, use_lu);
  double relres = 0.0;
  int its = 0;
  RB_TRY(gmres(op, n3, ld, g, x, rtol, max_iter, 60, &relres, &its, 0));
  if (!use_lu) {  // lambda = P^-T z
    adj_block_kernel<<<nb, 128>>>(coef.as<double>(), 1, n, x, t);
    RB_TRY(check_launch("adj_block_kernel"));
    RB_CUDA(cudaMemcpy(lambda, t, n3 * sizeof(double), cudaMemcpyDeviceToHost));
  } else {
    RB_CUDA(cudaMemcpy(lambda, x, n3 * sizeof(double), cudaMemcpyDeviceToHost));
  }
  status[0] = relres;
  status[1] = its;
  status[2] = use_lu;
  status[3] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (!(relres <= rtol)) {
    set_error("adjoint GMRES stopped at relative residual %.3e after %d iterations", relres, its);
    return RADB200_E_NOCONV;
  }
  return 0;
}

// chunking of a (rows x cols) pair loop: grid.x covers rows, grid.y splits cols
static void pair_chunks(int rows, int cols, int *nchunk, int *per_chunk)
{
  int bx = (rows + ADJ_T - 1) / ADJ_T;
  int c = std::max(1, std::min((148 * 8 + bx - 1) / bx, (cols + 31) / 32));
  int per = (cols + c - 1) / c;
  *per_chunk = std::max(per, 1);
  *nchunk = std::max(1, (cols + *per_chunk - 1) / *per_chunk);
}

// per source: [n][9] = (G^T U, -d/dq, d/dd) summed over the observers X
template <bool WANT_M>
static int src_pass(Intrc &I, const double *m, const double *X, const double *U, int nobs, int what, double *out)
{
  int nchunk, per;
  pair_chunks(I.n, nobs, &nchunk, &per);
  DBuf part;
  RB_TRY(part.alloc((size_t)nchunk * I.n * 9 * sizeof(double)));
  dim3 grid((I.n + ADJ_T - 1) / ADJ_T, nchunk);
  // models of cuboids only (the undulators) get the variant without the
  // polyhedron code paths (fewer registers, no spills)
  if (I.geom.n_poly == 0)
    adj_src_kernel<WANT_M, true><<<grid, ADJ_T>>>(I.geom.view(I.fast), I.elem_src.as<int>(), m, I.n, X, U, nobs, per, what,
                                                  part.as<double>());
  else
    adj_src_kernel<WANT_M, false><<<grid, ADJ_T>>>(I.geom.view(I.fast), I.elem_src.as<int>(), m, I.n, X, U, nobs, per,
                                                   what, part.as<double>());
  RB_TRY(check_launch("adj_src_kernel"));
  int64_t len = (int64_t)I.n * 9;
  adj_reduce_kernel<<<(unsigned)((len + 255) / 256), 256>>>(part.as<double>(), nchunk, len, out);
  return check_launch("adj_reduce_kernel");
}

int adjoint_grad(Intrc &I, const double *lambda, double *dMr, double *dchi, double *dc, double *dd)
{
  const int n = I.n, n3 = I.n3, ld = I.ld;
  if (dMr) memcpy(dMr, lambda, n3 * sizeof(double));
  if (!dchi && !dc && !dd) return 0;
  DBuf buf;
  RB_TRY(buf.alloc((size_t)3 * ld * sizeof(double)));
  RB_CUDA(cudaMemset(buf.p, 0, (size_t)3 * ld * sizeof(double)));
  double *lam = buf.as<double>(), *H = lam + ld, *u = H + ld;
  RB_CUDA(cudaMemcpy(lam, lambda, n3 * sizeof(double), cudaMemcpyHostToDevice));
  RB_TRY(converged_H(I, H));
  if (dchi) {
    std::vector<double> hH(n3);
    RB_CUDA(cudaMemcpy(hH.data(), H, n3 * sizeof(double), cudaMemcpyDeviceToHost));
    for (int e = 0; e < n; e++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
          dchi[9 * (size_t)e + 3 * a + b] = I.h_mat_kind[e] == RADB200_MAT_LINEAR ? lambda[3 * e + a] * hH[3 * e + b] : 0.0;
  }
  if (!dc && !dd) return 0;
  int nb = (n + 127) / 128;
  adj_weight_kernel<<<nb, 128>>>(lam, H, I.mat_kind.as<int>(), I.mat.as<double>(), I.mh.as<double>(), I.rowT.as<double>(), n, u);
  RB_TRY(check_launch("adj_weight_kernel"));
  // sources: every element at its converged M; observers: the element centres
  DBuf srcout, obsout, part;
  RB_TRY(srcout.alloc((size_t)n * 9 * sizeof(double)));
  RB_TRY(obsout.alloc((size_t)n * 3 * sizeof(double)));
  RB_TRY(src_pass<false>(I, I.lastM.as<double>(), I.obs.as<double>(), u, n, 1, srcout.as<double>()));
  {
    int nchunk, per;
    pair_chunks(n, n, &nchunk, &per);
    RB_TRY(part.alloc((size_t)nchunk * n * 3 * sizeof(double)));
    dim3 grid((n + ADJ_T - 1) / ADJ_T, nchunk);
    adj_obs_kernel<<<grid, ADJ_T>>>(I.geom.view(I.fast), I.elem_src.as<int>(), I.lastM.as<double>(), n, I.obs.as<double>(),
                                    u, n, per, part.as<double>());
    RB_TRY(check_launch("adj_obs_kernel"));
    int64_t len = (int64_t)n * 3;
    adj_reduce_kernel<<<(unsigned)((len + 255) / 256), 256>>>(part.as<double>(), nchunk, len, obsout.as<double>());
    RB_TRY(check_launch("adj_reduce_kernel"));
  }
  std::vector<double> hs((size_t)n * 9), ho((size_t)n * 3), hu(n3), hobs(n3);
  RB_CUDA(cudaMemcpy(hs.data(), srcout.p, hs.size() * sizeof(double), cudaMemcpyDeviceToHost));
  RB_CUDA(cudaMemcpy(ho.data(), obsout.p, ho.size() * sizeof(double), cudaMemcpyDeviceToHost));
  if (I.has_ext && dc) {
    // gradient of the external field at the centres: central differences of
    // the device field of the external sources (step 1e-4 mm; the error is
    // O(h^2) of a field smooth on the mm scale, and O(eps/h) from rounding)
    const double h = 1e-4;
    RB_CUDA(cudaMemcpy(hu.data(), u, n3 * sizeof(double), cudaMemcpyDeviceToHost));
    RB_CUDA(cudaMemcpy(hobs.data(), I.obs.p, n3 * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<double> P((size_t)n * 18), out((size_t)n * 18);
    for (int e = 0; e < n; e++)
      for (int a = 0; a < 3; a++)
        for (int sgn = 0; sgn < 2; sgn++) {
          double *p = &P[(size_t)18 * e + 6 * a + 3 * sgn];
          for (int b = 0; b < 3; b++) p[b] = hobs[3 * e + b] + (a == b ? (sgn ? -h : h) : 0.0);
        }
    DBuf dP, dO, scratch;
    RB_TRY(dP.upload(P.data(), P.size() * sizeof(double)));
    RB_TRY(dO.alloc(out.size() * sizeof(double)));
    RB_TRY(launch_field(I.xgeom.view(I.fast), dP.as<double>(), (int64_t)n * 6, 1, 0, dO.as<double>(), scratch, 0));
    RB_CUDA(cudaMemcpy(out.data(), dO.p, out.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int e = 0; e < n; e++)
      for (int a = 0; a < 3; a++) {
        const double *fp = &out[(size_t)18 * e + 6 * a], *fm = fp + 3;
        double s = 0.0;
        for (int b = 0; b < 3; b++) s += hu[3 * e + b] * (fp[b] - fm[b]);
        ho[3 * e + a] += s / (2.0 * h);
      }
  }
  for (int e = 0; e < n; e++) {
    bool rect = I.h_elem_src[2 * e] == 0;
    const double *J = &I.h_obsJ[9 * (size_t)e];
    for (int a = 0; a < 3; a++) {
      if (dc) {
        // d obs_e / d c_e = J_e: the observer moves with its element
        double v = hs[9 * (size_t)e + 3 + a] + J[a] * ho[3 * e] + J[3 + a] * ho[3 * e + 1] + J[6 + a] * ho[3 * e + 2];
        dc[3 * e + a] = rect ? v : 0.0;
      }
      if (dd) dd[3 * e + a] = rect ? hs[9 * (size_t)e + 6 + a] : 0.0;
    }
  }
  return 0;
}

int field_vjp(Intrc &I, const double *M, const double *pts, int64_t npts, int what, const double *W, double *gM, double *gc,
              double *gd)
{
  const int n = I.n;
  if (npts > (int64_t)1 << 30) { set_error("field_vjp: too many points"); return RADB200_E_ARG; }
  std::vector<double> hs((size_t)n * 9, 0.0);
  if (npts > 0) {
    DBuf dm, dx, dw, out;
    RB_TRY(dm.upload(M, (size_t)n * 3 * sizeof(double)));
    RB_TRY(dx.upload(pts, (size_t)npts * 3 * sizeof(double)));
    RB_TRY(dw.upload(W, (size_t)npts * 3 * sizeof(double)));
    RB_TRY(out.alloc((size_t)n * 9 * sizeof(double)));
    RB_TRY(src_pass<true>(I, dm.as<double>(), dx.as<double>(), dw.as<double>(), (int)npts, what, out.as<double>()));
    RB_CUDA(cudaMemcpy(hs.data(), out.p, hs.size() * sizeof(double), cudaMemcpyDeviceToHost));
  }
  for (int e = 0; e < n; e++) {
    bool rect = I.h_elem_src[2 * e] == 0;
    for (int a = 0; a < 3; a++) {
      if (gM) gM[3 * e + a] = hs[9 * (size_t)e + a];
      if (gc) gc[3 * e + a] = rect ? hs[9 * (size_t)e + 3 + a] : 0.0;
      if (gd) gd[3 * e + a] = rect ? hs[9 * (size_t)e + 6 + a] : 0.0;
    }
  }
  return 0;
}

}  // namespace rb
