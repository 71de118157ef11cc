// lu_diag.cuh -- factor one diagonal block of the blocked LU (unpivoted) and
// invert both of its triangles, in one CTA.
//
// The block (nb <= DG_N rows and columns) is padded to DG_N x DG_N with the
// identity, which leaves the factors and inverses of the nb x nb part exact
// and puts zeros (and a unit diagonal) outside it.  It lives in shared memory
// in FP64 at row pitch DG_N + 1 (a warp reading one row per lane at a fixed
// column, or a row per warp, hits distinct banks in each half-warp).
//
// Blocked by DG_B = 32.  For each diagonal sub-block b:
//   F  warps 0-3 factor D = S(b,b): warp w holds rows 8w..8w+7 in registers,
//      lane = column.  At step k the warp that owns row k publishes it in
//      shared memory behind a 128-thread named barrier (two alternating row
//      buffers, so one barrier per step suffices) and every warp eliminates
//      column k from its rows below k.
//   I  warps 0-3 invert D's unit-lower triangle by the same forward sweep on
//      the identity, warps 4-7 its upper triangle by a backward sweep, each
//      behind its own named barrier.
//   P  L(i,b) = S(i,b) U_bb^-1 and U(b,j) = L_bb^-1 S(b,j) for i, j > b, in
//      8 x 32 quarter sub-blocks, one per warp; each warp keeps its quarter
//      in registers across a block barrier, so every product has read its
//      inputs before any of them is overwritten.
//   U  S(i,j) -= L(i,b) U(b,j) for i, j > b, quarter sub-blocks over all warps.
// Then the inverses of the whole triangles from the sub-block inverses, in
// place over the factor blocks they consume:
//   Linv(i,j) = -(sum_{j<q<=i} Linv(i,q) L(q,j)) L_jj^-1   columns right to left,
//   Uinv(i,j) = -(sum_{i<=q<j} Uinv(i,q) U(q,j)) U_jj^-1   columns left to right
// (from Linv L = I and Uinv U = I), the last product by shuffles across the
// quarter's lanes.
//
// The serial work is the 3 x 128 pivot steps of F and I (a barrier, a row
// broadcast and 8 FMAs per warp each); everything else is 32 x 32 x 32
// products spread over 32 warps.  No wait depends on anything outside the CTA.
#pragma once

namespace rb {

constexpr int DG_N = 128;                // padded block
constexpr int DG_B = 32;                 // sub-block
constexpr int DG_NS = DG_N / DG_B;       // sub-blocks per side
constexpr int DG_P = DG_N + 1;           // row pitch of the block (doubles)
constexpr int DG_IP = DG_B + 1;          // row pitch of a sub-block inverse
constexpr int DG_T = 1024;               // threads: 32 warps
constexpr int DG_SMEM = (DG_N * DG_P + 2 * DG_NS * DG_B * DG_IP) * (int)sizeof(double);

__device__ __forceinline__ void dg_bar(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// acc[i] += sum_p X[i * ldx + p] * Y[p * ldy + lane] for the 8 rows of a quarter
__device__ __forceinline__ void dg_mac(double (&acc)[8], const double *X, int ldx, const double *Y, int ldy, int lane)
{
#pragma unroll 4
  for (int p = 0; p < DG_B; p++) {
    const double y = Y[p * ldy + lane];
#pragma unroll
    for (int i = 0; i < 8; i++) acc[i] = fma(X[i * ldx + p], y, acc[i]);
  }
}

// acc <- -(acc Y): the quarter's rows are spread over the lanes (lane p holds
// column p), so row entry p comes from lane p by a shuffle
__device__ __forceinline__ void dg_neg_times(double (&acc)[8], const double *Y, int ldy, int lane)
{
  double out[8];
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = 0.0;
#pragma unroll 4
  for (int p = 0; p < DG_B; p++) {
    const double y = Y[p * ldy + lane];
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = fma(__shfl_sync(0xffffffffu, acc[i], p), y, out[i]);
  }
#pragma unroll
  for (int i = 0; i < 8; i++) acc[i] = -out[i];
}

// F: D (pitch DG_P) <- its unit-lower L (strictly below the diagonal) and U;
// warps 0-3, named barrier 1
__device__ __forceinline__ void dg_factor(double *D, double *row, int w, int lane, int *err)
{
  double a[8];
#pragma unroll
  for (int i = 0; i < 8; i++) a[i] = D[(8 * w + i) * DG_P + lane];
  for (int kw = 0; kw < 4; kw++) {
#pragma unroll
    for (int ki = 0; ki < 8; ki++) {
      const int k = 8 * kw + ki;
      double *rb = row + (k & 1) * DG_B;
      if (w == kw) rb[lane] = a[ki];
      dg_bar(1);
      const double u = rb[lane], piv = rb[k];
      if (w == 0 && lane == 0 && !(fabs(piv) > 1e-300)) *err = 1;
      const double ip = 1.0 / piv;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const double l = __shfl_sync(0xffffffffu, a[i], k) * ip;
        if (8 * w + i > k) {
          if (lane == k) a[i] = l;
          else if (lane > k) a[i] = fma(-l, u, a[i]);
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) D[(8 * w + i) * DG_P + lane] = a[i];
}

// I, lower: Out (pitch DG_IP) <- L^-1 of D's unit-lower triangle; warps 0-3, barrier 1
__device__ __forceinline__ void dg_inv_lower(const double *D, double *row, double *Out, int w, int lane)
{
  double b[8];
#pragma unroll
  for (int i = 0; i < 8; i++) b[i] = (8 * w + i == lane) ? 1.0 : 0.0;
  for (int kw = 0; kw < 4; kw++) {
#pragma unroll
    for (int ki = 0; ki < 8; ki++) {
      const int k = 8 * kw + ki;
      double *rb = row + (k & 1) * DG_B;
      if (w == kw) rb[lane] = b[ki];
      dg_bar(1);
      const double x = rb[lane];
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (8 * w + i > k) b[i] = fma(-D[(8 * w + i) * DG_P + k], x, b[i]);
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) Out[(8 * w + i) * DG_IP + lane] = b[i];
}

// I, upper: Out (pitch DG_IP) <- U^-1 of D's upper triangle; warps 4-7 (w = warp - 4), barrier 2
__device__ __forceinline__ void dg_inv_upper(const double *D, double *row, double *Out, int w, int lane)
{
  double b[8];
#pragma unroll
  for (int i = 0; i < 8; i++) b[i] = (8 * w + i == lane) ? 1.0 : 0.0;
  for (int kw = 3; kw >= 0; kw--) {
#pragma unroll
    for (int ki = 7; ki >= 0; ki--) {
      const int k = 8 * kw + ki;
      double *rb = row + (k & 1) * DG_B;
      if (w == kw) {
        b[ki] *= 1.0 / D[k * DG_P + k];
        rb[lane] = b[ki];
      }
      dg_bar(2);
      const double y = rb[lane];
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (8 * w + i < k) b[i] = fma(-D[(8 * w + i) * DG_P + k], y, b[i]);
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) Out[(8 * w + i) * DG_IP + lane] = b[i];
}

// Factor the nb x nb block at (k0, k0) of A (row pitch ld) in place into L\U;
// write L^-1 (unit lower) and U^-1 to rows k0.. of Linv and Uinv (pitch DG_N,
// zero beyond column nb).  err[0] = 1 on a pivot of magnitude <= 1e-300.
template <typename T>
__global__ void __launch_bounds__(DG_T) diag_factor_kernel(T *__restrict__ A, int ld, int k0, int nb, T *__restrict__ Linv,
                                                           T *__restrict__ Uinv, int *__restrict__ err)
{
  extern __shared__ double dg_smem[];
  double *S = dg_smem;                  // DG_N x DG_P
  double *LI = S + DG_N * DG_P;         // DG_NS sub-block inverses of L, DG_B x DG_IP each
  double *UI = LI + DG_NS * DG_B * DG_IP;
  __shared__ double rowL[2 * DG_B], rowU[2 * DG_B];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto blk = [&](int i, int j) { return S + i * DG_B * DG_P + j * DG_B; };
  auto inv = [&](double *X, int i) { return X + i * DG_B * DG_IP; };

  for (int e = tid; e < DG_N * DG_N; e += DG_T) {
    const int r = e / DG_N, c = e % DG_N;
    S[r * DG_P + c] = (r < nb && c < nb) ? (double)A[(size_t)(k0 + r) * ld + k0 + c] : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();

  for (int b = 0; b < DG_NS; b++) {
    if (warp < 4) dg_factor(blk(b, b), rowL, warp, lane, err);
    __syncthreads();
    if (warp < 4) dg_inv_lower(blk(b, b), rowL, inv(LI, b), warp, lane);
    else if (warp < 8) dg_inv_upper(blk(b, b), rowU, inv(UI, b), warp - 4, lane);
    __syncthreads();
    const int m = DG_NS - 1 - b;  // sub-blocks below and right of b
    {
      // P: quarters 0..4m-1 of L(i,b), then 4m..8m-1 of U(b,j)
      double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      double *out = nullptr;
      if (warp < 8 * m) {
        const int s = warp % (4 * m), i = b + 1 + s / 4, q = s % 4;
        if (warp < 4 * m) {
          out = blk(i, b) + 8 * q * DG_P;
          dg_mac(acc, out, DG_P, inv(UI, b), DG_IP, lane);
        } else {
          out = blk(b, i) + 8 * q * DG_P;
          dg_mac(acc, inv(LI, b) + 8 * q * DG_IP, DG_IP, blk(b, i), DG_P, lane);
        }
      }
      __syncthreads();
      if (out)
#pragma unroll
        for (int i = 0; i < 8; i++) out[i * DG_P + lane] = acc[i];
      __syncthreads();
    }
    // U: the trailing sub-blocks
    for (int t = warp; t < 4 * m * m; t += DG_T / 32) {
      const int q = t % 4, s = t / 4, i = b + 1 + s / m, j = b + 1 + s % m;
      double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      dg_mac(acc, blk(i, b) + 8 * q * DG_P, DG_P, blk(b, j), DG_P, lane);
      double *o = blk(i, j) + 8 * q * DG_P;
#pragma unroll
      for (int ii = 0; ii < 8; ii++) o[ii * DG_P + lane] -= acc[ii];
    }
    __syncthreads();
  }

  for (int e = tid; e < nb * nb; e += DG_T) {
    const int r = e / nb, c = e - r * nb;
    A[(size_t)(k0 + r) * ld + k0 + c] = (T)S[r * DG_P + c];
  }

  // the whole inverses: step s takes L's sub-block column DG_NS-2-s and U's s+1
  for (int s = 0; s < DG_NS - 1; s++) {
    const int jl = DG_NS - 2 - s, ju = s + 1;
    const int nl = 4 * (DG_NS - 1 - jl), nu = 4 * ju;
    double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double *out = nullptr;
    if (warp < nl) {
      const int i = jl + 1 + warp / 4, q = warp % 4;
      dg_mac(acc, inv(LI, i) + 8 * q * DG_IP, DG_IP, blk(i, jl), DG_P, lane);
      for (int c = jl + 1; c < i; c++) dg_mac(acc, blk(i, c) + 8 * q * DG_P, DG_P, blk(c, jl), DG_P, lane);
      dg_neg_times(acc, inv(LI, jl), DG_IP, lane);
      out = blk(i, jl) + 8 * q * DG_P;
    } else if (warp < nl + nu) {
      const int i = (warp - nl) / 4, q = (warp - nl) % 4;
      dg_mac(acc, inv(UI, i) + 8 * q * DG_IP, DG_IP, blk(i, ju), DG_P, lane);
      for (int c = i + 1; c < ju; c++) dg_mac(acc, blk(i, c) + 8 * q * DG_P, DG_P, blk(c, ju), DG_P, lane);
      dg_neg_times(acc, inv(UI, ju), DG_IP, lane);
      out = blk(i, ju) + 8 * q * DG_P;
    }
    __syncthreads();
    if (out)
#pragma unroll
      for (int i = 0; i < 8; i++) out[i * DG_P + lane] = acc[i];
    __syncthreads();
  }

  for (int e = tid; e < nb * DG_N; e += DG_T) {
    const int r = e / DG_N, c = e % DG_N;
    double l = 0.0, u = 0.0;
    if (c < nb) {
      const int bi = r / DG_B, bj = c / DG_B;
      if (bi == bj) {
        l = inv(LI, bi)[(r % DG_B) * DG_IP + c % DG_B];
        u = inv(UI, bi)[(r % DG_B) * DG_IP + c % DG_B];
      } else if (bi > bj) {
        l = S[r * DG_P + c];
      } else {
        u = S[r * DG_P + c];
      }
    }
    Linv[(size_t)(k0 + r) * DG_N + c] = (T)l;
    Uinv[(size_t)(k0 + r) * DG_N + c] = (T)u;
  }
}

}  // namespace rb
