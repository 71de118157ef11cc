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
//   F  warps 0-7 factor D = S(b,b) and invert both of its triangles in one
//      sweep: warp w holds rows 4w..4w+3 of D, of L_bb^-1 (starting from the
//      identity) and of an accumulator for U_bb^-1, lane = column.  At step k
//      the warp that owns row k publishes row k of D and of L_bb^-1 in shared
//      memory behind a 256-thread named barrier (two alternating buffers, so
//      one barrier per step suffices); every warp then eliminates column k
//      from its rows of D below k, applies the multipliers to its rows of
//      L_bb^-1 (forward substitution), finishes column k of U_bb^-1 from the
//      accumulator (U^-1(r,k) = -sum_{r<=q<k} U^-1(r,q) U(q,k) / U(k,k)) and
//      adds column k's share to the later columns (row k of U).
//   P  L(i,b) = S(i,b) U_bb^-1 and U(b,j) = L_bb^-1 S(b,j) for i, j > b, in
//      8 x 32 quarter sub-blocks, one per warp; each warp keeps its quarter
//      in registers across a block barrier, so every product has read its
//      inputs before any of them is overwritten.
//   U  S(i,j) -= L(i,b) U(b,j) for i, j > b, quarter sub-blocks: the next
//      diagonal sub-block first, then F of b + 1 on warps 0-7 while warps
//      8-31 update the rest.
// Then the inverses of the whole triangles from the sub-block inverses, in
// place over the factor blocks they consume:
//   Linv(i,j) = -(sum_{j<q<=i} Linv(i,q) L(q,j)) L_jj^-1   columns right to left,
//   Uinv(i,j) = -(sum_{i<=q<j} Uinv(i,q) U(q,j)) U_jj^-1   columns left to right
// (from Linv L = I and Uinv U = I), the last product by shuffles across the
// quarter's lanes.
//
// The serial work is the 128 pivot steps of F (a barrier, two row
// broadcasts and a few FMAs per row each); everything else is 32 x 32 x 32
// products spread over 32 warps.  No wait depends on anything outside the CTA.
#pragma once

namespace rb {

constexpr int DG_N = 128;                // padded block
constexpr int DG_B = 32;                 // sub-block
constexpr int DG_NS = DG_N / DG_B;       // sub-blocks per side
constexpr int DG_P = DG_N + 4;           // row pitch of the block (doubles)
constexpr int DG_IP = DG_B + 4;          // row pitch of a sub-block inverse
constexpr int DG_T = 1024;               // threads: 32 warps
constexpr int DG_SMEM = (DG_N * DG_P + 2 * DG_NS * DG_B * DG_IP) * (int)sizeof(double);

// The 32 x 32 x 32 products run on the FP64 tensor path, mma.sync m8n8k4
// (D = A B + C, A 8 x 4 row-major, B 4 x 8 column-major, FP64 throughout).
// A warp computes one 8 x 32 quarter as four 8 x 8 tiles; its fragments:
//   A(r, c) in lane 4r + c,  B(c, n) in lane 4n + c,  C(r, 2c + i) in lane 4r + c.
// With the pitches above (multiples of 4 doubles, 8 words mod 32) the
// fragment loads of a half-warp hit 16 distinct bank pairs.
struct DgAcc {
  double v[4][2];  // tile t: row lane / 4, columns 8 t + 2 (lane % 4) + i
};

__device__ __forceinline__ void dg_zero(DgAcc &a)
{
#pragma unroll
  for (int t = 0; t < 4; t++) a.v[t][0] = a.v[t][1] = 0.0;
}

// a += X Y: X the quarter's 8 rows (pitch ldx, 32 columns), Y 32 x 32 (pitch ldy)
__device__ __forceinline__ void dg_mac(DgAcc &a, const double *X, int ldx, const double *Y, int ldy, int lane)
{
  const int r = lane >> 2, c = lane & 3;
#pragma unroll
  for (int kk = 0; kk < DG_B / 4; kk++) {
    const double fa = X[r * ldx + 4 * kk + c];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const double fb = Y[(4 * kk + c) * ldy + 8 * t + r];
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(a.v[t][0]), "+d"(a.v[t][1])
                   : "d"(fa), "d"(fb));
    }
  }
}

// O (the quarter's 8 rows, pitch ldo) = s a, or O += s a with add
__device__ __forceinline__ void dg_store(double *O, int ldo, const DgAcc &a, double s, bool add, int lane)
{
  const int r = lane >> 2, c = lane & 3;
#pragma unroll
  for (int t = 0; t < 4; t++) {
    double2 *o = reinterpret_cast<double2 *>(O + r * ldo + 8 * t + 2 * c);
    double2 w = add ? *o : make_double2(0.0, 0.0);
    w.x = fma(s, a.v[t][0], w.x);
    w.y = fma(s, a.v[t][1], w.y);
    *o = w;
  }
}

// F: D (pitch DG_P) <- its unit-lower L (strictly below the diagonal) and U;
// LI, UI (pitch DG_IP) <- L^-1 and U^-1.  Warps 0-7, named barrier 1.
constexpr int DG_FW = 8;               // warps of the sweep
constexpr int DG_FR = DG_B / DG_FW;    // rows per warp
__device__ __forceinline__ void dg_factor(double *D, double *LI, double *UI, double *rowA, double *rowX, int w, int lane,
                                          int *err, double tiny)
{
  double a[DG_FR], x[DG_FR], y[DG_FR];
#pragma unroll
  for (int i = 0; i < DG_FR; i++) {
    a[i] = D[(DG_FR * w + i) * DG_P + lane];
    x[i] = (DG_FR * w + i == lane) ? 1.0 : 0.0;
    y[i] = 0.0;
  }
  for (int kw = 0; kw < DG_FW; kw++) {
#pragma unroll
    for (int ki = 0; ki < DG_FR; ki++) {
      const int k = DG_FR * kw + ki;
      double *ra = rowA + (k & 1) * DG_B, *rx = rowX + (k & 1) * DG_B;
      if (w == kw) {
        ra[lane] = a[ki];
        rx[lane] = x[ki];
      }
      asm volatile("bar.sync 1, %0;" ::"n"(32 * DG_FW) : "memory");
      const double u = ra[lane], piv = ra[k], xk = rx[lane];
      if (w == 0 && lane == 0 && !(fabs(piv) > tiny)) *err = 1;
      const double ip = 1.0 / piv;
#pragma unroll
      for (int i = 0; i < DG_FR; i++) {
        const int r = DG_FR * w + i;
        // column k of D for rows below k (the multipliers), of the U^-1
        // accumulator for the others: one shuffle either way
        const double v = __shfl_sync(0xffffffffu, r > k ? a[i] : y[i], k);
        if (r > k) {
          const double l = v * ip;
          if (lane == k) a[i] = l;
          else if (lane > k) a[i] = fma(-l, u, a[i]);
          x[i] = fma(-l, xk, x[i]);
        } else {
          const double yv = (r < k) ? -v * ip : ip;
          if (lane == k) y[i] = yv;
          else if (lane > k) y[i] = fma(yv, u, y[i]);
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < DG_FR; i++) {
    D[(DG_FR * w + i) * DG_P + lane] = a[i];
    LI[(DG_FR * w + i) * DG_IP + lane] = x[i];
    UI[(DG_FR * w + i) * DG_IP + lane] = y[i];
  }
}

// Factor the nb x nb block at (k0, k0) of A (row pitch ld) in place into L\U;
// write L^-1 (unit lower) and U^-1 to rows k0.. of Linv and Uinv (pitch DG_N,
// zero beyond column nb).  err[0] = 1 on a pivot of magnitude <= tiny (or not
// finite).
template <typename T>
__global__ void __launch_bounds__(DG_T) diag_factor_kernel(T *__restrict__ A, int ld, int k0, int nb, T *__restrict__ Linv,
                                                           T *__restrict__ Uinv, int *__restrict__ err, double tiny)
{
  extern __shared__ double dg_smem[];
  double *S = dg_smem;                  // DG_N x DG_P
  double *LI = S + DG_N * DG_P;         // DG_NS sub-block inverses of L, DG_B x DG_IP each
  double *UI = LI + DG_NS * DG_B * DG_IP;
  __shared__ double rowA[2 * DG_B], rowX[2 * DG_B];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto blk = [&](int i, int j) { return S + i * DG_B * DG_P + j * DG_B; };
  auto inv = [&](double *X, int i) { return X + i * DG_B * DG_IP; };

  for (int e = tid; e < DG_N * DG_N; e += DG_T) {
    const int r = e / DG_N, c = e % DG_N;
    S[r * DG_P + c] = (r < nb && c < nb) ? (double)A[(size_t)(k0 + r) * ld + k0 + c] : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();

  if (warp < DG_FW) dg_factor(blk(0, 0), inv(LI, 0), inv(UI, 0), rowA, rowX, warp, lane, err, tiny);
  for (int b = 0; b < DG_NS; b++) {
    __syncthreads();
    const int m = DG_NS - 1 - b;  // sub-blocks below and right of b
    if (m == 0) break;
    {
      // P: quarters 0..4m-1 of L(i,b), then 4m..8m-1 of U(b,j)
      DgAcc acc;
      dg_zero(acc);
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
      if (out) dg_store(out, DG_P, acc, 1.0, false, lane);
      __syncthreads();
    }
    // U: the next diagonal sub-block first (warps 0-3), then its F on warps
    // 0-7 while warps 8-31 update the other trailing sub-blocks
    if (warp < 4) {
      DgAcc acc;
      dg_zero(acc);
      dg_mac(acc, blk(b + 1, b) + 8 * warp * DG_P, DG_P, blk(b, b + 1), DG_P, lane);
      dg_store(blk(b + 1, b + 1) + 8 * warp * DG_P, DG_P, acc, -1.0, true, lane);
    }
    __syncthreads();
    if (warp < DG_FW) {
      dg_factor(blk(b + 1, b + 1), inv(LI, b + 1), inv(UI, b + 1), rowA, rowX, warp, lane, err, tiny);
    } else {
      for (int t = warp - DG_FW + 4; t < 4 * m * m; t += DG_T / 32 - DG_FW) {
        const int q = t % 4, s = t / 4, i = b + 1 + s / m, j = b + 1 + s % m;  // t < 4: the diagonal sub-block, done
        DgAcc acc;
        dg_zero(acc);
        dg_mac(acc, blk(i, b) + 8 * q * DG_P, DG_P, blk(b, j), DG_P, lane);
        dg_store(blk(i, j) + 8 * q * DG_P, DG_P, acc, -1.0, true, lane);
      }
    }
  }

  for (int e = tid; e < nb * nb; e += DG_T) {
    const int r = e / nb, c = e - r * nb;
    A[(size_t)(k0 + r) * ld + k0 + c] = (T)S[r * DG_P + c];
  }

  // the whole inverses: step s takes L's sub-block column DG_NS-2-s and U's
  // s+1.  Each quarter first forms T = sum (...) in registers; after the
  // barrier it writes T over its own rows of the block it replaces, then
  // multiplies those rows by the diagonal sub-block inverse (only this warp
  // reads them) and writes the negated product.
  for (int s = 0; s < DG_NS - 1; s++) {
    const int jl = DG_NS - 2 - s, ju = s + 1;
    const int nl = 4 * (DG_NS - 1 - jl), nu = 4 * ju;
    DgAcc acc;
    dg_zero(acc);
    double *out = nullptr;
    const double *dinv = nullptr;
    if (warp < nl) {
      const int i = jl + 1 + warp / 4, q = warp % 4;
      dg_mac(acc, inv(LI, i) + 8 * q * DG_IP, DG_IP, blk(i, jl), DG_P, lane);
      for (int c = jl + 1; c < i; c++) dg_mac(acc, blk(i, c) + 8 * q * DG_P, DG_P, blk(c, jl), DG_P, lane);
      out = blk(i, jl) + 8 * q * DG_P;
      dinv = inv(LI, jl);
    } else if (warp < nl + nu) {
      const int i = (warp - nl) / 4, q = (warp - nl) % 4;
      dg_mac(acc, inv(UI, i) + 8 * q * DG_IP, DG_IP, blk(i, ju), DG_P, lane);
      for (int c = i + 1; c < ju; c++) dg_mac(acc, blk(i, c) + 8 * q * DG_P, DG_P, blk(c, ju), DG_P, lane);
      out = blk(i, ju) + 8 * q * DG_P;
      dinv = inv(UI, ju);
    }
    __syncthreads();
    if (out) {
      dg_store(out, DG_P, acc, 1.0, false, lane);
      __syncwarp();
      dg_zero(acc);
      dg_mac(acc, out, DG_P, dinv, DG_IP, lane);
      __syncwarp();
      dg_store(out, DG_P, acc, -1.0, false, lane);
    }
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
