// lu.cu -- dense direct solve of the linear-material relaxation system.
//
// No counterpart in the reference (it only iterates, methods 3-11).  For
// linear laws M_i = X_i H_i + Mr_i the fixed point of the relaxation solves
//     A M = X H_ext + Mr,     A = I - X N      (X = block-diagonal chi)
// A is factored in place by a right-looking blocked LU WITHOUT pivoting:
// with the volume-weighted inner product the demagnetization operator -N is
// positive semi-definite, so A is (close to) positive definite and needs no
// row exchanges; a vanishing pivot is reported as RADB200_E_NUMERIC.
//
// Two levels: outer panels of 1024 columns (768 for the last 30,000 rows),
// 128-wide steps inside.  Step k
// (width nb = 128) inside a panel:
//   1. one CTA factors the diagonal block in shared memory (FP64) and writes
//      the inverses of its unit-lower and upper triangles, L_kk^-1 and U_kk^-1
//      (lu_diag.cuh);
//   2. L21 = A21 U_kk^-1 and the panel's U12 = L_kk^-1 A12 as GEMMs (out of
//      place, then copied back), so the triangular solves of the panel also
//      run on the GEMM engine; a narrow update of the panel's other columns.
// After the panel: its U block row by block forward substitution, then one
// trailing update A22 -= L21 U12 with K = the panel width, split into the next panel's
// columns (main stream) and the rest (a side stream, overlapping the next
// panel's factorization).
//   mode F64  : FP64 factors, GEMMs on the FP64 pipe (CUDA cores).
//   mode mixed: FP32 factors, GEMMs on the tcgen05 tensor cores (FP16
//               operands scaled by powers of two, or TF32; FP32 accumulation,
//               gemm_tc.cu), then right-preconditioned FP64 GMRES on A with
//               the FP64 residual (GMRES-IR).
// Triangular solves with the factors use the stored diagonal-block inverses
// (one persistent launch per sweep, tri_sweep_kernel).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "internal.cuh"
#include "lu_diag.cuh"

namespace rb {

constexpr int LU_NB = 128;  // panel width, also the pitch of the inverse buffers

// A = I - X N, into FP64 or FP32 storage (columns beyond n3 zero)
template <typename T, typename NT>
__global__ void build_A_kernel(const NT *__restrict__ N, const double *__restrict__ mat, int n3, int ld, T *__restrict__ A)
{
  int r = blockIdx.y;
  int e = r / 3, a = r % 3;
  const double *X = mat + (size_t)e * RADB200_MAT_STRIDE;
  double x0 = X[3 * a], x1 = X[3 * a + 1], x2 = X[3 * a + 2];
  const NT *n0 = N + (size_t)(3 * e) * ld;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ld; c += gridDim.x * blockDim.x) {
    double v;
    if (c < n3) v = (r == c ? 1.0 : 0.0) - (x0 * (double)n0[c] + x1 * (double)n0[ld + c] + x2 * (double)n0[2 * (size_t)ld + c]);
    else v = 0.0;
    A[(size_t)r * ld + c] = (T)v;
  }
}

// right-hand side b = X H_ext + Mr
__global__ void build_rhs_kernel(const double *__restrict__ hext, const double *__restrict__ mat, int n, double *__restrict__ b)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double *X = mat + (size_t)e * RADB200_MAT_STRIDE;
  for (int a = 0; a < 3; a++)
    b[3 * e + a] = X[3 * a] * hext[3 * e] + X[3 * a + 1] * hext[3 * e + 1] + X[3 * a + 2] * hext[3 * e + 2] + X[9 + a];
}

// out = x - X y   (A x, given y = N x); transpose != 0: out = x - N^T-side handled by caller
__global__ void apply_A_kernel(const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ mat,
                               int n, double *__restrict__ out)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double *X = mat + (size_t)e * RADB200_MAT_STRIDE;
  for (int a = 0; a < 3; a++)
    out[3 * e + a] = x[3 * e + a] - (X[3 * a] * y[3 * e] + X[3 * a + 1] * y[3 * e + 1] + X[3 * a + 2] * y[3 * e + 2]);
}

// ---- diagonal block: factor (unpivoted) and invert both triangles: one CTA,
// blocked by 32 in shared memory (lu_diag.cuh)
static_assert(DG_N == LU_NB, "the diagonal-block kernel works on LU_NB x LU_NB blocks");

// ---- CUDA-core GEMM: C[m x n] (=|-=) A[m x k] B[k x n]; 64x64 tile, k-slices of 16
template <typename T>
__global__ void __launch_bounds__(256) gemm_simt_kernel(T *__restrict__ C, int ldc, int m, int n, int k,
                                                        const T *__restrict__ A, int lda, const T *__restrict__ B, int ldb,
                                                        int overwrite)
{
  __shared__ T sA[16][64 + 1];
  __shared__ T sB[16][64 + 1];
  int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  int rb = blockIdx.y * 64, cb = blockIdx.x * 64;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0;
  for (int kk = 0; kk < k; kk += 16) {
    for (int e = threadIdx.x; e < 64 * 16; e += 256) {
      int r = e / 16, c = e % 16;
      sA[c][r] = (rb + r < m && kk + c < k) ? A[(size_t)(rb + r) * lda + kk + c] : T(0);
      int kr = e / 64, cc = e % 64;
      sB[kr][cc] = (cb + cc < n && kk + kr < k) ? B[(size_t)(kk + kr) * ldb + cb + cc] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; q++) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = sA[q][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = sB[q][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int gr = rb + ty + 16 * i;
    if (gr >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      int gc = cb + tx + 16 * j;
      if (gc >= n) continue;
      T *d = C + (size_t)gr * ldc + gc;
      if (overwrite) *d = acc[i][j];
      else *d -= acc[i][j];
    }
  }
}

// dst[r][c] = src[r][c] for r < rows, c < cols (row-major, leading dimensions in elements)
template <typename T>
__global__ void copy2d_kernel(T *__restrict__ dst, int ldd, const T *__restrict__ src, int lds, int rows, int cols)
{
  int64_t tot = (int64_t)rows * cols;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(i / cols), c = (int)(i % cols);
    dst[(size_t)r * ldd + c] = src[(size_t)r * lds + c];
  }
}

// host time spent enqueueing each kind of LU work (RADB200_LU_TIMING=2):
// 0 GEMMs of the panel and U block rows, 1 trailing updates, 2 diagonal blocks, 3 copies
static bool g_lu_host_timing = false;
static double g_lu_host[4];
struct LuHostSpan {
  int i;
  std::chrono::steady_clock::time_point t0;
  explicit LuHostSpan(int k) : i(k)
  {
    if (g_lu_host_timing) t0 = std::chrono::steady_clock::now();
  }
  ~LuHostSpan()
  {
    if (g_lu_host_timing) g_lu_host[i] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

template <typename T>
static int copy2d(T *dst, int ldd, const T *src, int lds, int rows, int cols, cudaStream_t st)
{
  LuHostSpan hs(3);
  int64_t tot = (int64_t)rows * cols;
  int nb = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
  copy2d_kernel<T><<<std::max(nb, 1), 256, 0, st>>>(dst, ldd, src, lds, rows, cols);
  return check_launch("copy2d_kernel");
}

template <typename T>
static int gemm(T *C, int ldc, int m, int n, int k, T *A, int lda, const T *B, int ldb, int overwrite, cudaStream_t st,
                int *tc_used)
{
  if (m <= 0 || n <= 0) return 0;
  LuHostSpan hs(0);
  if (sizeof(T) == 4) {
    int used = 0;
    RB_TRY(tc_gemm_f32((float *)C, ldc, m, n, k, (float *)A, lda, (const float *)B, ldb, st, &used, overwrite));
    if (used) { *tc_used = 1; return 0; }
  }
  dim3 grid((n + 63) / 64, (m + 63) / 64);
  if (grid.y > 65535) { set_error("GEMM grid too large"); return RADB200_E_ARG; }
  gemm_simt_kernel<T><<<grid, 256, 0, st>>>(C, ldc, m, n, k, A, lda, B, ldb, overwrite);
  return check_launch("gemm_simt_kernel");
}

// dst = A B where dst is the same memory as A (c_is_a) or as B: in place on
// the tensor cores when they can (tc_gemm_f32_inplace), else into tmp (pitch
// ldt) and copied back
template <typename T>
static int gemm_to(T *dst, int ldd, int m, int n, int k, T *A, int lda, const T *B, int ldb, bool c_is_a, T *tmp,
                   int ldt, cudaStream_t st, int *tc_used)
{
  if (m <= 0 || n <= 0) return 0;
  if (sizeof(T) == 4) {
    LuHostSpan hs(0);
    int used = 0;
    RB_TRY(tc_gemm_f32_inplace((float *)dst, ldd, m, n, k, (float *)A, lda, (const float *)B, ldb, st, &used, c_is_a));
    if (used) { *tc_used = 1; return 0; }
  }
  RB_TRY(gemm<T>(tmp, ldt, m, n, k, A, lda, B, ldb, 1, st, tc_used));
  return copy2d<T>(dst, ldd, tmp, ldt, m, n, st);
}

// ---- triangular solves with the factors (in place on x, FP64) ----
// dot of a 128-wide row (16-byte aligned, zero beyond nb) with xs, across a warp
__device__ __forceinline__ double row128_dot(const float *row, const double *xs, int lane)
{
  float4 v = __ldg(reinterpret_cast<const float4 *>(row) + lane);
  const double *xp = xs + 4 * lane;
  return (double)v.x * xp[0] + (double)v.y * xp[1] + (double)v.z * xp[2] + (double)v.w * xp[3];
}
__device__ __forceinline__ double row128_dot(const double *row, const double *xs, int lane)
{
  double2 v0 = __ldg(reinterpret_cast<const double2 *>(row) + lane);
  double2 v1 = __ldg(reinterpret_cast<const double2 *>(row) + 32 + lane);
  return v0.x * xs[2 * lane] + v0.y * xs[2 * lane + 1] + v1.x * xs[64 + 2 * lane] + v1.y * xs[64 + 2 * lane + 1];
}
__device__ __forceinline__ double warp_sum(double s)
{
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// x[k0:k0+nb] <- Inv_k x[k0:k0+nb]   (Inv = L^-1 or U^-1 of diagonal block k,
// pitch 128 with zero columns beyond nb); warp per row
template <typename T>
__global__ void __launch_bounds__(256) block_matvec_kernel(const T *__restrict__ Inv, int k0, int nb, double *__restrict__ x)
{
  __shared__ double xs[LU_NB];
  if (threadIdx.x < LU_NB) xs[threadIdx.x] = threadIdx.x < nb ? x[k0 + threadIdx.x] : 0.0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = warp; r < nb; r += 8) {
    double s = warp_sum(row128_dot(Inv + (size_t)(k0 + r) * LU_NB, xs, lane));
    if (lane == 0) x[k0 + r] = s;
  }
}

// x[rows r0..r1) -= A[rows, k0:k0+nb] x[k0:k0+nb] (warp per row, 16-byte loads
// when the panel is a full 128 wide)
template <typename T>
__global__ void __launch_bounds__(256) panel_gemv_kernel(const T *__restrict__ A, int ld, int k0, int nb, int r0, int r1,
                                                         double *__restrict__ x)
{
  __shared__ double xs[LU_NB];
  for (int r = threadIdx.x; r < LU_NB; r += blockDim.x) xs[r] = r < nb ? x[k0 + r] : 0.0;
  __syncthreads();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int row = r0 + blockIdx.x * 8 + warp;
  if (row >= r1) return;
  const T *a = A + (size_t)row * ld + k0;
  double s = 0.0;
  if (nb == LU_NB) s = row128_dot(a, xs, lane);
  else
    for (int j = lane; j < nb; j += 32) s += (double)a[j] * xs[j];
  s = warp_sum(s);
  if (lane == 0) x[row] -= s;
}

// ---- transposed solves, A^T = U^T L^T (adjoint) ----
// x[k0:k0+nb] <- Inv_k^T x[k0:k0+nb]
template <typename T>
__global__ void __launch_bounds__(LU_NB) block_matvec_t_kernel(const T *__restrict__ Inv, int k0, int nb, double *__restrict__ x)
{
  __shared__ double xs[LU_NB];
  int r = threadIdx.x;
  if (r < nb) xs[r] = x[k0 + r];
  __syncthreads();
  if (r < nb) {
    double s = 0.0;
    for (int j = 0; j < nb; j++) s += (double)Inv[(size_t)(k0 + j) * LU_NB + r] * xs[j];
    x[k0 + r] = s;
  }
}

// x[c0..c1) -= A[k0:k0+nb, c0..c1)^T x[k0:k0+nb] (thread per column, coalesced rows)
template <typename T>
__global__ void __launch_bounds__(256) panel_gemv_t_kernel(const T *__restrict__ A, int ld, int k0, int nb, int c0, int c1,
                                                           double *__restrict__ x)
{
  __shared__ double xs[LU_NB];
  for (int r = threadIdx.x; r < nb; r += blockDim.x) xs[r] = x[k0 + r];
  __syncthreads();
  int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  const T *a = A + (size_t)k0 * ld + c;
  double s = 0.0;
  for (int r = 0; r < nb; r++) s += (double)a[(size_t)r * ld] * xs[r];
  x[c] -= s;
}

template <typename T>
static int lu_solve_t(const T *A, const T *Linv, const T *Uinv, int n3, int ld, double *x, cudaStream_t st)
{
  // U^T y = x, forward over the block rows of U
  for (int k0 = 0; k0 < n3; k0 += LU_NB) {
    int nb = std::min(LU_NB, n3 - k0);
    block_matvec_t_kernel<T><<<1, LU_NB, 0, st>>>(Uinv, k0, nb, x);
    RB_TRY(check_launch("block_matvec_t_kernel"));
    int rest = k0 + nb;
    if (rest < n3) {
      panel_gemv_t_kernel<T><<<(n3 - rest + 255) / 256, 256, 0, st>>>(A, ld, k0, nb, rest, n3, x);
      RB_TRY(check_launch("panel_gemv_t_kernel"));
    }
  }
  // L^T z = y, backward over the block rows of L
  int last = ((n3 - 1) / LU_NB) * LU_NB;
  for (int k0 = last; k0 >= 0; k0 -= LU_NB) {
    int nb = std::min(LU_NB, n3 - k0);
    block_matvec_t_kernel<T><<<1, LU_NB, 0, st>>>(Linv, k0, nb, x);
    RB_TRY(check_launch("block_matvec_t_kernel"));
    if (k0 > 0) {
      panel_gemv_t_kernel<T><<<(k0 + 255) / 256, 256, 0, st>>>(A, ld, k0, nb, 0, k0, x);
      RB_TRY(check_launch("panel_gemv_t_kernel"));
    }
  }
  return 0;
}

// Optional CUDA-event timing of the trailing updates (A22 -= L21 U12) on the
// stream they are launched on: radb200_update_timing(1) starts collecting,
// radb200_update_stats() returns launches, summed device time, algorithmic
// bytes (C read + written, panels read once) and flops (2 m^2 K) since then.
struct UpdEvents {
  std::vector<cudaEvent_t> ev;
  int used = 0;
  int grow()
  {
    if (2 * used + 2 <= (int)ev.size()) return 0;
    for (int q = 0; q < 512; q++) {
      cudaEvent_t e;
      RB_CUDA(cudaEventCreate(&e));
      ev.push_back(e);
    }
    return 0;
  }
};
static int g_update_timing = 0;
static UpdEvents g_upd_ev;
static double g_upd_bytes = 0.0, g_upd_flops = 0.0;

// Two-level right-looking LU.  Outer panels of LU_OUTER columns; inside a
// panel, 128-wide steps (diagonal block, L21 = A21 U^-1, the panel's own
// U12 = L^-1 A12 and a narrow update of the panel's remaining columns).  The
// panel's U block row for the trailing columns is then solved by block
// forward substitution over its 128-row sub-blocks, and the trailing matrix
// receives ONE update with K = LU_OUTER: the C traffic of the dominant GEMM
// drops by LU_OUTER / 128 against 128-wide steps.
// Outer panel widths: 1024 columns while at least LU_LATE_AT_DEFAULT rows
// remain, then 768.  The trailing GEMMs dominate the early panels (a wider K
// raises their rate: 489 -> 533 TFLOP/s), the main stream's panel chain the
// late ones.  Swept on the 60,000^2 factorization (solve, s): 768 throughout
// 0.494; 1024 then 768 below 20,000 / 30,000 / 40,000 rows 0.482 / 0.481 /
// 0.482; 1280 then 768 0.482; 1536 then 768 0.487; 1024 then 512 0.495;
// 1024 then 640 0.493; 1280 then 1024 0.497.
constexpr int LU_OUTER_DEFAULT = 1024, LU_OUTER_LATE_DEFAULT = 768, LU_LATE_AT_DEFAULT = 30000;
// the outer panel width: LU_OUTER_DEFAULT, or RADB200_LU_OUTER (a multiple of
// 128 from 256 to 2048) for tuning; RADB200_LU_OUTER_LATE (same range) is the
// width once fewer than RADB200_LU_LATE_AT rows remain (tuning: the trailing
// GEMMs dominate the early panels, the panel chain the late ones)
static int lu_width_env(const char *name, int dflt)
{
  const char *e = getenv(name);
  int v = e ? atoi(e) : dflt;
  return (v >= 256 && v <= 2048 && v % LU_NB == 0) ? v : dflt;
}
static int lu_outer()
{
  static int w = 0;
  if (!w) w = lu_width_env("RADB200_LU_OUTER", LU_OUTER_DEFAULT);
  return w;
}
static int lu_outer_at(int remaining)
{
  static int late = 0, at = -1;
  if (!late) {
    late = lu_width_env("RADB200_LU_OUTER_LATE", LU_OUTER_LATE_DEFAULT);
    const char *e = getenv("RADB200_LU_LATE_AT");
    at = e ? std::max(0, atoi(e)) : LU_LATE_AT_DEFAULT;
  }
  return remaining < at ? late : lu_outer();
}

// One-panel look-ahead: the trailing update of outer step k is split into the
// columns of panel k+1 (on the main stream, first) and the rest (on a side
// stream, its grid capped to leave LU_SIDE_FREE_SMS multiprocessors free), so
// that panel k+1 -- its single-CTA diagonal factorizations, narrow GEMMs and
// copies -- is factored on the main stream while the rest of the update runs.
// The main stream waits for the side stream before the U block row of step
// k+1, the only later work that reads or writes the columns the side stream
// updates.  Events order the two streams; nothing waits on the device.
constexpr int LU_SIDE_FREE_SMS = 12;  // swept 4-74 on the 60,000^2 factorization: 12 was fastest;
                                       // with the 1024/768 panels: 6 +9 ms, 20 within 2 ms

struct LuStreams {
  cudaStream_t main = nullptr, side = nullptr;
  cudaEvent_t in = nullptr, upd = nullptr, side_done = nullptr, out = nullptr;
  int init()
  {
    if (main) return 0;
    RB_CUDA(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking));
    RB_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&in, &upd, &side_done, &out}) RB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return 0;
  }
};
static LuStreams g_lu_streams;

template <typename T>
static int lu_factor(Intrc &I, T *A, T *Linv, T *Uinv, T *tmp, int *d_err, double tiny, cudaStream_t st, int *tc_used)
{
  const int n3 = I.n3, ld = I.ld;
  RB_CUDA(cudaFuncSetAttribute(diag_factor_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
  // RADB200_LU_TIMING=1 prints the time of each phase (synchronizes per phase);
  // RADB200_LU_TIMING=2 prints the host's time to enqueue the factorization
  // against its device time (no synchronization inside), which shows whether
  // the launches keep the device fed; RADB200_LU_LOOKAHEAD=0 runs every phase
  // on the caller's stream
  const char *tv = getenv("RADB200_LU_TIMING");
  const int timing_mode = tv ? std::max(1, atoi(tv)) : 0;
  const bool timing = timing_mode == 1;
  cudaEvent_t tq0 = nullptr, tq1 = nullptr;
  auto tq_host = std::chrono::steady_clock::now();
  // RADB200_LU_TIMING=3: events on the main stream between its kinds of work
  // (0 diagonal blocks, 1 L21, 2 U12 in the panel, 3 narrow panel updates,
  // 4 waits for the side stream, 5 U block rows, 6 next panel's update),
  // summed after the factorization: the main stream's critical path by kind
  std::vector<cudaEvent_t> mk_ev;
  std::vector<int> mk_cat;
  if (timing_mode == 2) {
    RB_CUDA(cudaEventCreate(&tq0));
    RB_CUDA(cudaEventCreate(&tq1));
    RB_CUDA(cudaEventRecord(tq0, st));
    tq_host = std::chrono::steady_clock::now();
    g_lu_host_timing = true;
    for (double &h : g_lu_host) h = 0.0;
  }
  const char *la = getenv("RADB200_LU_LOOKAHEAD");
  const bool lookahead = !(la && atoi(la) == 0);
  double tph[4] = {0, 0, 0, 0};
  auto t_last = std::chrono::steady_clock::now();
  auto phase = [&](int p) -> int {
    if (!timing) return 0;
    RB_CUDA(cudaDeviceSynchronize());
    auto t = std::chrono::steady_clock::now();
    tph[p] += std::chrono::duration<double>(t - t_last).count();
    t_last = t;
    return 0;
  };
  cudaStream_t sm = st, ss = st;
  int side_ctas = 0;
  if (lookahead) {
    RB_TRY(g_lu_streams.init());
    sm = g_lu_streams.main;
    ss = g_lu_streams.side;
    RB_CUDA(cudaEventRecord(g_lu_streams.in, st));
    RB_CUDA(cudaStreamWaitEvent(sm, g_lu_streams.in, 0));
    RB_CUDA(cudaStreamWaitEvent(ss, g_lu_streams.in, 0));
    int dev = 0, nsm = 0;
    RB_CUDA(cudaGetDevice(&dev));
    RB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const char *fs = getenv("RADB200_LU_FREE_SMS");  // tuning override
    side_ctas = std::max(1, nsm - ((fs && atoi(fs) > 0) ? atoi(fs) : LU_SIDE_FREE_SMS));
  }
  auto mark = [&](int cat) -> int {
    if (timing_mode != 3) return 0;
    cudaEvent_t e;
    RB_CUDA(cudaEventCreate(&e));
    RB_CUDA(cudaEventRecord(e, sm));
    mk_ev.push_back(e);
    mk_cat.push_back(cat);
    return 0;
  };
  bool side_pending = false;
  auto at = [&](int r, int c) { return A + (size_t)r * ld + c; };
  // C[m x n] -= A B with the update's timing events on stream q
  auto update = [&](T *C, int m, int n, int k, T *Ap, const T *Bp, cudaStream_t q, int slot, int cap) -> int {
    if (m <= 0 || n <= 0) return 0;
    LuHostSpan hs(1);
    if (g_update_timing) {
      RB_TRY(g_upd_ev.grow());
      RB_CUDA(cudaEventRecord(g_upd_ev.ev[2 * g_upd_ev.used], q));
    }
    int used = 0;
    if (sizeof(T) == 4) {
      RB_TRY(tc_gemm_f32((float *)C, ld, m, n, k, (float *)Ap, ld, (const float *)Bp, ld, q, &used, 0, slot, cap));
      if (used) *tc_used = 1;
    }
    if (!used) RB_TRY(gemm<T>(C, ld, m, n, k, Ap, ld, Bp, ld, 0, q, tc_used));
    if (g_update_timing) {
      RB_CUDA(cudaEventRecord(g_upd_ev.ev[2 * g_upd_ev.used + 1], q));
      g_upd_ev.used++;
      // algorithmic bytes: C read + written, the L and U panels read once (as
      // FP16 copies when the tensor cores took FP16 operands)
      const double opb = used == 2 ? 2.0 : (double)sizeof(T);
      g_upd_bytes += (double)sizeof(T) * 2.0 * m * n + opb * ((double)m * k + (double)k * n);
      g_upd_flops += 2.0 * m * n * k;
    }
    return 0;
  };
  for (int K0 = 0, NBe = 0; K0 < n3; K0 += NBe) {
    NBe = std::min(lu_outer_at(n3 - K0), n3 - K0);
    const int pend = K0 + NBe;  // end of the panel's columns
    // ---- factor the panel columns [K0, pend) over rows [K0, n3) (main stream;
    // the previous step updated these columns there first)
    for (int j0 = K0; j0 < pend; j0 += LU_NB) {
      const int jb = std::min(LU_NB, pend - j0);
      {
        LuHostSpan hs(2);
        diag_factor_kernel<T><<<1, DG_T, DG_SMEM, sm>>>(A, ld, j0, jb, Linv, Uinv, d_err, tiny);
        RB_TRY(check_launch("diag_factor_kernel"));
      }
      RB_TRY(mark(0));
      RB_TRY(phase(0));
      const int rest = j0 + jb, m = n3 - rest;
      if (m <= 0) break;
      // L21 = A21 U_jj^-1   (tmp: m x LU_NB)
      RB_TRY(gemm_to<T>(at(rest, j0), ld, m, jb, jb, at(rest, j0), ld, Uinv + (size_t)j0 * LU_NB, LU_NB, true, tmp, LU_NB,
                        sm, tc_used));
      RB_TRY(mark(1));
      const int w = pend - rest;  // panel columns right of this step
      if (w > 0) {
        // U12 inside the panel = L_jj^-1 A12   (tmp: jb x w)
        RB_TRY(gemm_to<T>(at(j0, rest), ld, jb, w, jb, Linv + (size_t)j0 * LU_NB, LU_NB, at(j0, rest), ld, false, tmp, ld,
                          sm, tc_used));
        RB_TRY(mark(2));
        // narrow update of the panel: A[rest:, rest:pend] -= L21 U12
        RB_TRY(gemm<T>(at(rest, rest), ld, m, w, jb, at(rest, j0), ld, at(j0, rest), ld, 0, sm, tc_used));
        RB_TRY(mark(3));
      }
      RB_TRY(phase(1));
    }
    const int T0 = pend, mT = n3 - pend;
    if (mT <= 0) break;
    // the columns right of this panel must carry the previous step's update
    if (side_pending) {
      RB_CUDA(cudaEventRecord(g_lu_streams.side_done, ss));
      RB_CUDA(cudaStreamWaitEvent(sm, g_lu_streams.side_done, 0));
      side_pending = false;
    }
    RB_TRY(mark(4));
    // ---- U block row of the trailing columns: forward substitution with the
    // panel's unit-lower diagonal block, 128 rows at a time
    for (int j0 = K0; j0 < pend; j0 += LU_NB) {
      const int jb = std::min(LU_NB, pend - j0);
      if (j0 > K0) RB_TRY(gemm<T>(at(j0, T0), ld, jb, mT, j0 - K0, at(j0, K0), ld, at(K0, T0), ld, 0, sm, tc_used));
      RB_TRY(gemm_to<T>(at(j0, T0), ld, jb, mT, jb, Linv + (size_t)j0 * LU_NB, LU_NB, at(j0, T0), ld, false, tmp, ld, sm,
                        tc_used));
    }
    RB_TRY(mark(5));
    RB_TRY(phase(2));
    // ---- trailing update A22 -= L21 U12 with K = NBe: the next panel's
    // columns on the main stream, the rest on the side stream
    const int nxt = lookahead ? std::min(lu_outer_at(mT), mT) : mT;  // the next panel's width
    RB_TRY(update(at(T0, T0), mT, nxt, NBe, at(T0, K0), at(K0, T0), sm, 0, 0));
    RB_TRY(mark(6));
    if (mT > nxt) {
      RB_CUDA(cudaEventRecord(g_lu_streams.upd, sm));
      RB_CUDA(cudaStreamWaitEvent(ss, g_lu_streams.upd, 0));
      RB_TRY(update(at(T0, T0 + nxt), mT, mT - nxt, NBe, at(T0, K0), at(K0, T0 + nxt), ss, 1, side_ctas));
      side_pending = true;
    }
    RB_TRY(phase(3));
  }
  if (lookahead) {
    RB_CUDA(cudaEventRecord(g_lu_streams.side_done, ss));
    RB_CUDA(cudaStreamWaitEvent(sm, g_lu_streams.side_done, 0));
    RB_CUDA(cudaEventRecord(g_lu_streams.out, sm));
    RB_CUDA(cudaStreamWaitEvent(st, g_lu_streams.out, 0));
  }
  if (timing)
    fprintf(stderr, "[radb200 LU n=%d %s] diag %.3f s, panel %.3f s, U block rows %.3f s, trailing %.3f s\n", n3,
            sizeof(T) == 4 ? "fp32" : "fp64", tph[0], tph[1], tph[2], tph[3]);
  if (timing_mode == 3 && !mk_ev.empty()) {
    RB_CUDA(cudaEventSynchronize(mk_ev.back()));
    double cat[7] = {0, 0, 0, 0, 0, 0, 0};
    for (size_t i = 1; i < mk_ev.size(); i++) {
      float ms = 0.f;
      RB_CUDA(cudaEventElapsedTime(&ms, mk_ev[i - 1], mk_ev[i]));
      cat[mk_cat[i]] += 1e-3 * ms;
    }
    for (cudaEvent_t e : mk_ev) cudaEventDestroy(e);
    fprintf(stderr,
            "[radb200 LU n=%d %s] main stream: diagonal blocks %.4f s, L21 %.4f s, panel U12 %.4f s, narrow updates "
            "%.4f s, waits for the side stream %.4f s, U block rows %.4f s, next panel's update %.4f s\n",
            n3, sizeof(T) == 4 ? "fp32" : "fp64", cat[0], cat[1], cat[2], cat[3], cat[4], cat[5], cat[6]);
  }
  if (timing_mode == 2) {
    const double host = std::chrono::duration<double>(std::chrono::steady_clock::now() - tq_host).count();
    RB_CUDA(cudaEventRecord(tq1, st));
    RB_CUDA(cudaEventSynchronize(tq1));
    float ms = 0.f;
    RB_CUDA(cudaEventElapsedTime(&ms, tq0, tq1));
    fprintf(stderr,
            "[radb200 LU n=%d %s] host enqueue %.3f s (panel GEMMs %.3f, trailing updates %.3f, diagonal blocks %.3f, "
            "copies %.3f), device %.3f s\n",
            n3, sizeof(T) == 4 ? "fp32" : "fp64", host, g_lu_host[0], g_lu_host[1], g_lu_host[2], g_lu_host[3], 1e-3 * ms);
    g_lu_host_timing = false;
    cudaEventDestroy(tq0);
    cudaEventDestroy(tq1);
  }
  return 0;
}

// ---- triangular sweeps in one launch per factor ---------------------------------
// Forward with the unit-lower factor: x_k = Linv_k (b_k - sum_{j<k} L_kj x_j);
// backward with U: x_k = Uinv_k (b_k - sum_{j>k} U_kj x_j), blocks of 128.
// One persistent launch per sweep: each CTA takes the next block in sweep
// order from an atomic counter, subtracts the products with the blocks already
// solved as their flags appear (streaming its row panel of the factor while
// the chain of blocks advances), applies the diagonal block's inverse, and
// publishes x_k and its flag (release; readers acquire, then read x_j through
// L2).  A CTA waits only on blocks taken before its own by CTAs that are
// running, so every wait ends; each is also bounded by TRI_SPIN polls, after
// which the launch records an error in *err and every CTA returns.
// sync layout: [counter, flags of the blocks]; zeroed before each sweep.
constexpr long long TRI_SPIN = 1ll << 24;

__device__ __forceinline__ int ld_acquire_s32(const int *p)
{
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_s32(int *p, int v)
{
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One lane's slice of a 128-wide row of the factor (or of a diagonal-block
// inverse), loaded ahead of use, and its dot product with xs.
template <typename T> struct RowSlice;
template <> struct RowSlice<float> {
  float4 v;
  __device__ __forceinline__ void set(float4 q) { v = q; }
  __device__ __forceinline__ void load(const float *row, int lane) { v = __ldg(reinterpret_cast<const float4 *>(row) + lane); }
  __device__ __forceinline__ void zero() { v = make_float4(0.f, 0.f, 0.f, 0.f); }
  __device__ __forceinline__ double dot(const double *xs, int lane) const
  {
    const double *xp = xs + 4 * lane;
    return (double)v.x * xp[0] + (double)v.y * xp[1] + (double)v.z * xp[2] + (double)v.w * xp[3];
  }
};
template <> struct RowSlice<double> {
  double2 a, b;
  __device__ __forceinline__ void set(float4) {}  // unused: inverses are staged for float factors only
  __device__ __forceinline__ void load(const double *row, int lane)
  {
    a = __ldg(reinterpret_cast<const double2 *>(row) + lane);
    b = __ldg(reinterpret_cast<const double2 *>(row) + 32 + lane);
  }
  __device__ __forceinline__ void zero() { a = b = make_double2(0.0, 0.0); }
  __device__ __forceinline__ double dot(const double *xs, int lane) const
  {
    return a.x * xs[2 * lane] + a.y * xs[2 * lane + 1] + b.x * xs[64 + 2 * lane] + b.y * xs[64 + 2 * lane + 1];
  }
};

// rows per warp per batch: 8 warps x TRI_ROWS<T> x TRI_BATCH<T> = 128 rows
template <typename T> constexpr int tri_rows() { return sizeof(T) == 4 ? 16 : 8; }

template <typename T, bool UPPER>
__global__ void __launch_bounds__(256, 2) tri_sweep_kernel(const T *__restrict__ A, int ld, const T *__restrict__ Inv, int n3,
                                                        double *x, int *sync, int *err, const float *__restrict__ Msub)
{
  constexpr int NR = tri_rows<T>(), NB = LU_NB / (8 * NR);  // rows per batch, batches
  constexpr bool STAGE_INV = sizeof(T) == 4;  // Inv_k in shared memory (dynamic, LU_NB^2 floats)
  extern __shared__ float4 sinv4[];
  __shared__ double xs[LU_NB], acc_s[LU_NB];
  __shared__ int s_t, s_bad;
  const int nblk = (n3 + LU_NB - 1) / LU_NB;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int *flags = sync + 1;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) { s_t = atomicAdd(sync, 1); s_bad = 0; }
    __syncthreads();
    const int t = s_t;
    if (t >= nblk) return;
    const int k = UPPER ? nblk - 1 - t : t;
    const int k0 = k * LU_NB, nb = min(LU_NB, n3 - k0);
    // this warp's rows: (warp * NB + batch) * NR + i, accumulated in shared
    // memory by the warp's lane 0 (every row belongs to one warp)
    if (threadIdx.x < LU_NB) acc_s[threadIdx.x] = threadIdx.x < nb ? x[k0 + threadIdx.x] : 0.0;
    // with coupling blocks (FP32 factors, Msub): everything but the block
    // before this one in sweep order is done first and multiplied by the
    // inverse while that block is solved; x_k = y_k - M_k x_j then remains
    const bool use_m = STAGE_INV && Msub != nullptr && t > 0;
    // the matrix needed last, on the chain's critical path (M_k, or the
    // diagonal block's inverse): staged now (visible after the barriers
    // below), while the chain is still far from this block
    if constexpr (STAGE_INV) {
      const float *src = use_m ? Msub + (size_t)k * LU_NB * LU_NB : Inv + (size_t)k0 * LU_NB;
      for (int e = threadIdx.x; e < LU_NB * LU_NB / 4; e += blockDim.x) {
        const int r = e / (LU_NB / 4);
        sinv4[e] = (use_m || r < nb) ? __ldg(reinterpret_cast<const float4 *>(src + (size_t)r * LU_NB) + (e % (LU_NB / 4)))
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    const int s_end = use_m ? t - 1 : t;
    for (int s = 0; s < s_end; s++) {
      const int j = UPPER ? nblk - 1 - s : s;
      const int j0 = j * LU_NB, nbj = min(LU_NB, n3 - j0);
      const bool full = (nbj == LU_NB);
      // the tile's first batch is loaded before the wait: it does not depend on x_j
      RowSlice<T> v[NR];
      if (full) {
#pragma unroll
        for (int i = 0; i < NR; i++) {
          const int r = warp * NB * NR + i;
          if (r < nb) v[i].load(A + (size_t)(k0 + r) * ld + j0, lane);
          else v[i].zero();
        }
      }
      if (threadIdx.x == 0) {
        long long it = 0;
        while (ld_acquire_s32(flags + j) == 0) {
          if (++it > TRI_SPIN || ld_acquire_s32(err) != 0) { s_bad = 1; atomicExch(err, 1); break; }
        }
      }
      __syncthreads();  // the flag seen; every warp done with the previous xs
      if (s_bad) return;
      if (threadIdx.x < LU_NB) xs[threadIdx.x] = threadIdx.x < nbj ? __ldcg(x + j0 + threadIdx.x) : 0.0;
      __syncthreads();
      if (full) {
#pragma unroll
        for (int b = 0; b < NB; b++) {
          if (b > 0) {
#pragma unroll
            for (int i = 0; i < NR; i++) {
              const int r = (warp * NB + b) * NR + i;
              if (r < nb) v[i].load(A + (size_t)(k0 + r) * ld + j0, lane);
              else v[i].zero();
            }
          }
#pragma unroll
          for (int i = 0; i < NR; i++) {
            const double w = warp_sum(v[i].dot(xs, lane));
            if (lane == 0) acc_s[(warp * NB + b) * NR + i] -= w;
          }
        }
      } else {
        // the last, partial block: masked columns
#pragma unroll
        for (int b = 0; b < NB; b++)
#pragma unroll
          for (int i = 0; i < NR; i++) {
            const int r = (warp * NB + b) * NR + i;
            double w = 0.0;
            if (r < nb) {
              const T *a = A + (size_t)(k0 + r) * ld + j0;
              for (int c = lane; c < nbj; c += 32) w += (double)a[c] * xs[c];
            }
            w = warp_sum(w);
            if (lane == 0) acc_s[r] -= w;
          }
      }
    }
    if (use_m) {
      // y_k = Inv_k acc into acc_s (Inv_k through L2: off the chain)
      __syncthreads();
      if (threadIdx.x < LU_NB) xs[threadIdx.x] = threadIdx.x < nb ? acc_s[threadIdx.x] : 0.0;
      __syncthreads();
#pragma unroll
      for (int b = 0; b < NB; b++) {
        RowSlice<T> v[NR];
#pragma unroll
        for (int i = 0; i < NR; i++) {
          const int r = (warp * NB + b) * NR + i;
          if (r < nb) v[i].load(Inv + (size_t)(k0 + r) * LU_NB, lane);
          else v[i].zero();
        }
#pragma unroll
        for (int i = 0; i < NR; i++) {
          const int r = (warp * NB + b) * NR + i;
          const double w = warp_sum(v[i].dot(xs, lane));
          if (lane == 0) acc_s[r] = w;
        }
      }
      // the block before this one in sweep order
      const int j = UPPER ? k + 1 : k - 1;
      const int j0 = j * LU_NB, nbj = min(LU_NB, n3 - j0);
      if (threadIdx.x == 0) {
        long long it = 0;
        while (ld_acquire_s32(flags + j) == 0) {
          if (++it > TRI_SPIN || ld_acquire_s32(err) != 0) { s_bad = 1; atomicExch(err, 1); break; }
        }
      }
      __syncthreads();  // the flag seen; every warp done with xs
      if (s_bad) return;
      if (threadIdx.x < LU_NB) xs[threadIdx.x] = threadIdx.x < nbj ? __ldcg(x + j0 + threadIdx.x) : 0.0;
      __syncthreads();
#pragma unroll
      for (int b = 0; b < NB; b++) {
        RowSlice<T> v[NR];
#pragma unroll
        for (int i = 0; i < NR; i++) v[i].set(sinv4[((warp * NB + b) * NR + i) * (LU_NB / 4) + lane]);
#pragma unroll
        for (int i = 0; i < NR; i++) {
          const int r = (warp * NB + b) * NR + i;
          const double w = warp_sum(v[i].dot(xs, lane));
          if (lane == 0 && r < nb) x[k0 + r] = acc_s[r] - w;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        st_release_s32(flags + k, 1);
      }
      continue;
    }
    // x_k = Inv_k acc (rows of Inv beyond nb hold zero columns)
    __syncthreads();
    if (threadIdx.x < LU_NB) xs[threadIdx.x] = threadIdx.x < nb ? acc_s[threadIdx.x] : 0.0;
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; b++) {
      RowSlice<T> v[NR];
#pragma unroll
      for (int i = 0; i < NR; i++) {
        const int r = (warp * NB + b) * NR + i;
        if (STAGE_INV) {
          const float4 q = sinv4[r * (LU_NB / 4) + lane];
          v[i].set(q);
        } else if (r < nb) v[i].load(Inv + (size_t)(k0 + r) * LU_NB, lane);
        else v[i].zero();
      }
#pragma unroll
      for (int i = 0; i < NR; i++) {
        const int r = (warp * NB + b) * NR + i;
        const double w = warp_sum(v[i].dot(xs, lane));
        if (lane == 0 && r < nb) x[k0 + r] = w;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release_s32(flags + k, 1);
    }
  }
}

// Coupling blocks of FP32 factors for the sweeps: Mf[k] = Linv_k L_{k,k-1}
// (k >= 1) and Mb[k] = Uinv_k U_{k,k+1} (k < nblk - 1), 128 x 128 each, rows
// beyond block k's size and columns beyond its neighbour's zero.  With them a
// sweep finishes block k as x_k = y_k - M_k x_j once x_j of the block before
// it (in sweep order) appears, y_k = Inv_k (b_k - the other products) having
// been formed while waiting.  One CTA per block and direction, FP32 products
// of 128 terms, 8 x 8 outputs per thread.
__global__ void __launch_bounds__(256) sweep_m_kernel(const float *__restrict__ A, int ld, const float *__restrict__ Linv,
                                                      const float *__restrict__ Uinv, int n3, float *__restrict__ Mf,
                                                      float *__restrict__ Mb)
{
  __shared__ float sI[LU_NB][33];      // 32 columns of the inverse
  __shared__ float sB[32][LU_NB + 4];  // the matching 32 rows of the coupling block
  const int nblk = (n3 + LU_NB - 1) / LU_NB;
  const int k = blockIdx.x >> 1, upper = blockIdx.x & 1;
  if (upper ? k >= nblk - 1 : k < 1) return;
  const int k0 = k * LU_NB, nb = min(LU_NB, n3 - k0);
  const int j0 = (upper ? k + 1 : k - 1) * LU_NB, nbj = min(LU_NB, n3 - j0);
  const float *Inv = (upper ? Uinv : Linv) + (size_t)k0 * LU_NB;
  float *out = (upper ? Mb : Mf) + (size_t)k * LU_NB * LU_NB;
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int c = 0; c < 8; c++) acc[i][c] = 0.f;
  for (int q0 = 0; q0 < LU_NB; q0 += 32) {
    for (int e = threadIdx.x; e < LU_NB * 32; e += 256) {
      const int r = e / 32, q = e % 32;
      sI[r][q] = r < nb ? Inv[(size_t)r * LU_NB + q0 + q] : 0.f;
      const int qr = e / LU_NB, c = e % LU_NB;
      sB[qr][c] = (q0 + qr < nb && c < nbj) ? A[(size_t)(k0 + q0 + qr) * ld + j0 + c] : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < 32; q++) {
      float a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = sI[tr * 8 + i][q];
#pragma unroll
      for (int c = 0; c < 8; c++) b[c] = sB[q][tc * 8 + c];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int c = 0; c < 8; c++) acc[i][c] = fmaf(a[i], b[c], acc[i][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int c = 0; c < 8; c++) out[(size_t)(tr * 8 + i) * LU_NB + tc * 8 + c] = acc[i][c];
}

// RADB200_TRI_SWEEP=0: the per-block launches below instead (A/B comparisons)
static bool tri_sweep_enabled()
{
  static int on = -1;
  if (on < 0) {
    const char *e = getenv("RADB200_TRI_SWEEP");
    on = (e && atoi(e) == 0) ? 0 : 1;
  }
  return on == 1;
}

// RADB200_SWEEP_M=0: FP32 sweeps without coupling blocks (A/B comparisons)
static bool sweep_m_enabled()
{
  static int on = -1;
  if (on < 0) {
    const char *e = getenv("RADB200_SWEEP_M");
    on = (e && atoi(e) == 0) ? 0 : 1;
  }
  return on == 1;
}

static DBuf g_tri_err;  // allocated with the first factors, before any capture

// the sweeps' counters and flags of an interaction (allocated with its factors,
// so that a captured solve never sees the buffer move)
static int tri_sync_alloc(Intrc &I)
{
  const size_t per = (size_t)(I.n3 + LU_NB - 1) / LU_NB + 1;
  RB_TRY(I.tri_sync.alloc(2 * per * sizeof(int)));
  static bool attr = false;
  if (!attr) {
    const int dyn = LU_NB * LU_NB * (int)sizeof(float);
    RB_CUDA(cudaFuncSetAttribute(tri_sweep_kernel<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    RB_CUDA(cudaFuncSetAttribute(tri_sweep_kernel<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    attr = true;
  }
  if (!g_tri_err.p) {
    RB_TRY(g_tri_err.alloc(sizeof(int)));
    RB_CUDA(cudaMemset(g_tri_err.p, 0, sizeof(int)));
  }
  return 0;
}

template <typename T>
static int lu_solve_sweeps(const T *A, const T *Linv, const T *Uinv, int n3, int ld, double *x, int *sync,
                           const float *Mf, const float *Mb, cudaStream_t st)
{
  const int nblk = (n3 + LU_NB - 1) / LU_NB;
  const size_t per = (size_t)nblk + 1;
  RB_CUDA(cudaMemsetAsync(sync, 0, 2 * per * sizeof(int), st));
  const int grid = std::min(nblk, 148 * 4);
  // FP32 factors: the inverses staged in dynamic shared memory (the limit is
  // raised in tri_sync_alloc, before any capture)
  const size_t dyn = sizeof(T) == 4 ? (size_t)LU_NB * LU_NB * sizeof(float) : 0;
  tri_sweep_kernel<T, false><<<grid, 256, dyn, st>>>(A, ld, Linv, n3, x, sync, g_tri_err.as<int>(), Mf);
  RB_TRY(check_launch("tri_sweep_kernel"));
  tri_sweep_kernel<T, true><<<grid, 256, dyn, st>>>(A, ld, Uinv, n3, x, sync + per, g_tri_err.as<int>(), Mb);
  return check_launch("tri_sweep_kernel");
}

// error flag of the sweeps: 0, or 1 when a wait ran out (then cleared)
int tri_sweep_error(int *flag)
{
  *flag = 0;
  if (!g_tri_err.p) return 0;
  RB_CUDA(cudaMemcpy(flag, g_tri_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (*flag) RB_CUDA(cudaMemset(g_tri_err.p, 0, sizeof(int)));
  return 0;
}

template <typename T>
static int lu_solve(const T *A, const T *Linv, const T *Uinv, int n3, int ld, double *x, int *sync, cudaStream_t st,
                    const float *Mf = nullptr, const float *Mb = nullptr)
{
  if (sync && tri_sweep_enabled()) return lu_solve_sweeps<T>(A, Linv, Uinv, n3, ld, x, sync, Mf, Mb, st);
  for (int k0 = 0; k0 < n3; k0 += LU_NB) {
    int nb = std::min(LU_NB, n3 - k0);
    block_matvec_kernel<T><<<1, 256, 0, st>>>(Linv, k0, nb, x);
    RB_TRY(check_launch("block_matvec_kernel"));
    int rest = k0 + nb;
    if (rest < n3) {
      panel_gemv_kernel<T><<<(n3 - rest + 7) / 8, 256, 0, st>>>(A, ld, k0, nb, rest, n3, x);
      RB_TRY(check_launch("panel_gemv_kernel"));
    }
  }
  int last = ((n3 - 1) / LU_NB) * LU_NB;
  for (int k0 = last; k0 >= 0; k0 -= LU_NB) {
    int nb = std::min(LU_NB, n3 - k0);
    block_matvec_kernel<T><<<1, 256, 0, st>>>(Uinv, k0, nb, x);
    RB_TRY(check_launch("block_matvec_kernel"));
    if (k0 > 0) {
      panel_gemv_kernel<T><<<(k0 + 7) / 8, 256, 0, st>>>(A, ld, k0, nb, 0, k0, x);
      RB_TRY(check_launch("panel_gemv_kernel"));
    }
  }
  return 0;
}

static int lu_solve_direct(Intrc &I, int transposed, double *x, cudaStream_t st)
{
  const int n3 = I.n3, ld = I.ld;
  if (I.lu_mode == RADB200_LU_F64) {
    const double *L = I.LUinv.as<double>(), *U = L + (size_t)n3 * LU_NB;
    return transposed ? lu_solve_t<double>(I.LU64.as<double>(), L, U, n3, ld, x, st)
                      : lu_solve<double>(I.LU64.as<double>(), L, U, n3, ld, x, I.tri_sync.as<int>(), st);
  }
  if (I.lu_mode == RADB200_LU_TF32) {
    const float *L = I.LUinv.as<float>(), *U = L + (size_t)n3 * LU_NB;
    return transposed ? lu_solve_t<float>(I.LU32.as<float>(), L, U, n3, ld, x, st)
                      : lu_solve<float>(I.LU32.as<float>(), L, U, n3, ld, x, I.tri_sync.as<int>(), st,
                                        I.sweep_m.p ? I.sweep_m.as<float>() : nullptr,
                                        I.sweep_m.p ? I.sweep_m.as<float>() + (size_t)((n3 + LU_NB - 1) / LU_NB) * LU_NB * LU_NB
                                                    : nullptr);
  }
  set_error("no LU factors on this interaction");
  return RADB200_E_ARG;
}

// x <- A^-1 x (or A^-T x) with the kept factors.  For systems of 64 blocks
// and more, the ~4 n / 128 small launches of the block sweeps are captured
// once per factorization into a CUDA graph on a fixed buffer and replayed:
// one launch per application.
// RADB200_LU_GRAPH=0 launches the sweeps directly, never capturing them: a
// per-kernel profiler cannot run a launch made into a capturing stream (the
// kernel only becomes a graph node there), so launch lists are taken with it.
static bool lu_graph_enabled()
{
  static int on = -1;
  if (on < 0) {
    const char *e = getenv("RADB200_LU_GRAPH");
    on = (e && atoi(e) == 0) ? 0 : 1;
  }
  return on == 1;
}

static int lu_apply(Intrc &I, int transposed, double *x, cudaStream_t st)
{
  // small systems: a few applications per factorization do not repay a capture
  if (I.n3 < 64 * LU_NB || !lu_graph_enabled()) return lu_solve_direct(I, transposed, x, st);
  cudaGraphExec_t &ex = I.lu_graph[transposed];
  if (!ex) {
    RB_TRY(I.lu_gx.alloc((size_t)I.ld * sizeof(double)));
    cudaStream_t cs;
    RB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    int rc = 0;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
      const long long before = g_launches;
      rc = lu_solve_direct(I, transposed, I.lu_gx.as<double>(), cs);
      I.lu_graph_kernels[transposed] = g_launches - before;
      g_launches = before;  // captured, not launched
      e = cudaStreamEndCapture(cs, &graph);
      if (e == cudaSuccess && rc == 0) e = cudaGraphInstantiate(&ex, graph, 0);
    }
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    if (rc) return rc;
    if (e != cudaSuccess) {
      // no graph: run the sweeps directly (same kernels, launched one by one)
      cudaGetLastError();
      ex = nullptr;
      return lu_solve_direct(I, transposed, x, st);
    }
  }
  const size_t bytes = (size_t)I.n3 * sizeof(double);
  RB_CUDA(cudaMemcpyAsync(I.lu_gx.p, x, bytes, cudaMemcpyDeviceToDevice, st));
  RB_CUDA(cudaGraphLaunch(ex, st));
  g_launches += I.lu_graph_kernels[transposed];
  RB_CUDA(cudaMemcpyAsync(x, I.lu_gx.p, bytes, cudaMemcpyDeviceToDevice, st));
  return 0;
}

int lu_precond(Intrc &I, double *x, cudaStream_t st) { return lu_apply(I, 0, x, st); }

// x <- A^-T x with the kept factors (the adjoint's preconditioner)
int lu_precond_transposed(Intrc &I, double *x, cudaStream_t st) { return lu_apply(I, 1, x, st); }

struct LinOp : Op {
  Intrc &I;
  double *tmp;
  double t_mv = 0.0, t_pc = 0.0;  // seconds in products / sweeps (RADB200_TIMING only)
  LinOp(Intrc &i, double *t) : I(i), tmp(t) {}
  int apply(const double *v, double *out) override
  {
    const double t0 = timing_on() ? (cudaDeviceSynchronize(), now_s()) : 0.0;
    RB_TRY(run_matvec(I, v, nullptr, 1.0, tmp, 0));
    apply_A_kernel<<<(I.n + 127) / 128, 128>>>(v, tmp, I.mat.as<double>(), I.n, out);
    RB_TRY(check_launch("apply_A_kernel"));
    if (t0 > 0.0) { cudaDeviceSynchronize(); t_mv += now_s() - t0; }
    return 0;
  }
  int precond(double *v) override
  {
    const double t0 = timing_on() ? (cudaDeviceSynchronize(), now_s()) : 0.0;
    RB_TRY(lu_precond(I, v, 0));
    if (t0 > 0.0) { cudaDeviceSynchronize(); t_pc += now_s() - t0; }
    return 0;
  }
};

int lu_build(Intrc &I, int mode, double *factor_seconds)
{
  if (I.lu_mode == mode && !I.lu_of_d) { *factor_seconds = 0.0; return 0; }
  return lu_build_x(I, mode, I.mat.as<double>(), 0, factor_seconds);
}

// max |A_ii| (as float bits: non-negative floats order like their bits)
template <typename T>
__global__ void diag_absmax_kernel(const T *__restrict__ A, int ld, int n3, unsigned *__restrict__ out)
{
  float m = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    m = fmaxf(m, (float)fabs((double)A[(size_t)i * ld + i]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

template <typename T>
__global__ void add_diag_kernel(T *__restrict__ A, int ld, int n3, double sigma)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) A[(size_t)i * ld + i] = (T)((double)A[(size_t)i * ld + i] + sigma);
}

// Pivots at or below LU_TINY of the largest |A_ii| stop the unpivoted
// factorization; it is then redone on A + sigma I, sigma = LU_SHIFT of that
// scale (at least LU_SHIFT), and the FP64 GMRES that refines every solve --
// always with the unshifted operator -- takes the shifted factors as its
// preconditioner.  For physical materials (chi >= 0) A is diagonally similar
// to a symmetric positive-definite matrix, so every leading minor is positive
// and the shift is never needed; it covers unphysical inputs (a negative
// susceptibility that zeroes a self block) and rounding.
constexpr double LU_TINY = 1e-12, LU_SHIFT = 1e-3;

int lu_build_x(Intrc &I, int mode, const double *X, int of_d, double *factor_seconds)
{
  auto t0 = std::chrono::steady_clock::now();
  const int n3 = I.n3, ld = I.ld;
  I.lu_mode = -1;
  I.drop_lu_graphs();
  DBuf err;  // [pivot flag, max |A_ii| as float bits]
  dim3 bgrid((ld + 255) / 256 > 64 ? 64 : (ld + 255) / 256, n3);
  int tc_used = 0;
  size_t es = (mode == RADB200_LU_F64) ? sizeof(double) : sizeof(float);
  RB_TRY(I.LUinv.alloc(2 * (size_t)n3 * LU_NB * es));
  RB_TRY(I.lu_scratch.alloc((size_t)std::max((size_t)n3 * LU_NB, (size_t)LU_NB * ld) * es));
  if (mode == RADB200_LU_F64) {
    I.LU32.release();
    RB_TRY(I.LU64.alloc((size_t)n3 * ld * sizeof(double)));
  } else {
    I.LU64.release();
    RB_TRY(I.LU32.alloc((size_t)n3 * ld * sizeof(float)));
  }
  RB_TRY(err.alloc(2 * sizeof(int)));
  double tiny = 0.0;
  I.lu_shift = 0.0;
  int herr = 0, tcflag = 0;
  for (int attempt = 0; attempt < 2; attempt++) {
    RB_CUDA(cudaMemset(err.p, 0, 2 * sizeof(int)));
    unsigned *mx = reinterpret_cast<unsigned *>(err.as<int>() + 1);
    const int nb = std::min((n3 + 255) / 256, 148 * 4);
    if (mode == RADB200_LU_F64) {
      if (I.N64.p) build_A_kernel<double, double><<<bgrid, 256>>>(I.N64.as<double>(), X, n3, ld, I.LU64.as<double>());
      else build_A_kernel<double, float><<<bgrid, 256>>>(I.N32.as<float>(), X, n3, ld, I.LU64.as<double>());
      RB_TRY(check_launch("build_A_kernel"));
      if (attempt) add_diag_kernel<double><<<(n3 + 255) / 256, 256>>>(I.LU64.as<double>(), ld, n3, I.lu_shift);
      else diag_absmax_kernel<double><<<nb, 256>>>(I.LU64.as<double>(), ld, n3, mx);
    } else {
      if (I.N64.p) build_A_kernel<float, double><<<bgrid, 256>>>(I.N64.as<double>(), X, n3, ld, I.LU32.as<float>());
      else build_A_kernel<float, float><<<bgrid, 256>>>(I.N32.as<float>(), X, n3, ld, I.LU32.as<float>());
      RB_TRY(check_launch("build_A_kernel"));
      if (attempt) add_diag_kernel<float><<<(n3 + 255) / 256, 256>>>(I.LU32.as<float>(), ld, n3, I.lu_shift);
      else diag_absmax_kernel<float><<<nb, 256>>>(I.LU32.as<float>(), ld, n3, mx);
    }
    RB_TRY(check_launch(attempt ? "add_diag_kernel" : "diag_absmax_kernel"));
    if (!attempt) {
      unsigned bits = 0;
      RB_CUDA(cudaMemcpy(&bits, mx, sizeof(unsigned), cudaMemcpyDeviceToHost));
      float scale = 0.f;
      memcpy(&scale, &bits, sizeof(float));
      tiny = LU_TINY * (double)scale;
      if (!(tiny > 1e-300)) tiny = 1e-300;
    }
    if (mode == RADB200_LU_F64) {
      double *inv = I.LUinv.as<double>();
      RB_TRY(lu_factor<double>(I, I.LU64.as<double>(), inv, inv + (size_t)n3 * LU_NB, I.lu_scratch.as<double>(),
                               err.as<int>(), tiny, 0, &tc_used));
    } else {
      float *inv = I.LUinv.as<float>();
      RB_TRY(lu_factor<float>(I, I.LU32.as<float>(), inv, inv + (size_t)n3 * LU_NB, I.lu_scratch.as<float>(),
                              err.as<int>(), tiny, 0, &tc_used));
    }
    RB_CUDA(cudaMemcpy(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    RB_TRY(tc_error_flag(&tcflag));
    if (tcflag) { I.lu_mode = -1; set_error("LU: a tensor-core update timed out waiting for its MMAs"); return RADB200_E_TIMEOUT; }
    if (!herr) break;
    I.lu_shift = LU_SHIFT * std::max(1.0, tiny / LU_TINY);
    if (timing_on())
      fprintf(stderr, "RADB200_TIMING LU: pivot at or below %.3e; refactoring A + %.3e I\n", tiny, I.lu_shift);
  }
  if (herr) {
    I.lu_mode = -1;
    I.lu_shift = 0.0;
    set_error("LU: vanishing pivot (A and A + sigma I not factorable without pivoting)");
    return RADB200_E_NUMERIC;
  }
  RB_TRY(tri_sync_alloc(I));
  I.sweep_m.release();
  if (mode != RADB200_LU_F64 && sweep_m_enabled() && n3 > LU_NB) {
    const int nblk = (n3 + LU_NB - 1) / LU_NB;
    RB_TRY(I.sweep_m.alloc(2 * (size_t)nblk * LU_NB * LU_NB * sizeof(float)));
    const float *inv = I.LUinv.as<float>();
    float *Mf = I.sweep_m.as<float>(), *Mb = Mf + (size_t)nblk * LU_NB * LU_NB;
    sweep_m_kernel<<<2 * nblk, 256>>>(I.LU32.as<float>(), ld, inv, inv + (size_t)n3 * LU_NB, n3, Mf, Mb);
    RB_TRY(check_launch("sweep_m_kernel"));
  }
  I.lu_mode = mode;
  I.lu_of_d = of_d;
  I.lu_solve_id = I.solve_id;
  I.lu_tc = tc_used;
  RB_CUDA(cudaDeviceSynchronize());
  *factor_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

int direct_solve(Intrc &I, int mode, double rtol, int max_iter, double *status)
{
  auto t0 = std::chrono::steady_clock::now();
  const int n3 = I.n3, ld = I.ld;
  double tf = 0.0;
  PhaseClock pc;
  RB_TRY(lu_build(I, mode, &tf));
  pc.mark("solve: factors");
  RB_TRY(I.work.alloc((size_t)4 * ld * sizeof(double)));
  double *b = I.work.as<double>(), *tmp = b + ld;
  RB_CUDA(cudaMemset(I.work.p, 0, (size_t)4 * ld * sizeof(double)));
  build_rhs_kernel<<<(I.n + 127) / 128, 128>>>(I.hext.as<double>(), I.mat.as<double>(), I.n, b);
  RB_TRY(check_launch("build_rhs_kernel"));
  RB_CUDA(cudaMemcpy(I.M.p, b, n3 * sizeof(double), cudaMemcpyDeviceToDevice));
  RB_TRY(lu_precond(I, I.M.as<double>(), 0));
  LinOp op(I, tmp);
  double relres = 0.0;
  int its = 0;
  RB_TRY(gmres(op, n3, ld, b, I.M.as<double>(), rtol, max_iter, 30, &relres, &its, 0));
  RB_CUDA(cudaDeviceSynchronize());
  if (timing_on())
    fprintf(stderr, "RADB200_TIMING solve: refinement, %d its: products %.3f ms, sweeps %.3f ms\n", its, 1e3 * op.t_mv,
            1e3 * op.t_pc);
  pc.mark("solve: refinement");
  int tri_err = 0;
  RB_TRY(tri_sweep_error(&tri_err));
  if (tri_err) { set_error("direct solve: a triangular sweep timed out waiting for a block"); return RADB200_E_TIMEOUT; }
  status[0] = relres;
  status[1] = its;
  status[2] = tf;
  status[3] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

}  // namespace rb

extern "C" RADB200_API int radb200_update_timing(int on)
{
  rb::g_update_timing = on;
  rb::g_upd_ev.used = 0;
  rb::g_upd_bytes = 0.0;
  rb::g_upd_flops = 0.0;
  return 0;
}

extern "C" RADB200_API int radb200_update_stats(int64_t *launches, double *seconds, double *bytes, double *flops)
{
  RB_CUDA(cudaDeviceSynchronize());
  double ms_total = 0.0;
  for (int i = 0; i < rb::g_upd_ev.used; i++) {
    float ms = 0.f;
    RB_CUDA(cudaEventElapsedTime(&ms, rb::g_upd_ev.ev[2 * i], rb::g_upd_ev.ev[2 * i + 1]));
    ms_total += ms;
  }
  *launches = rb::g_upd_ev.used;
  *seconds = 1e-3 * ms_total;
  *bytes = rb::g_upd_bytes;
  *flops = rb::g_upd_flops;
  return 0;
}
