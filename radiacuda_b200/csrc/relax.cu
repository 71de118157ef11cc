// relax.cu -- device-resident magnetization relaxation.
//
// Replaces radGPU_RelaxAuto (method 9, reference radgpurlx.cu:799-1349) and
// radGPU_RelaxNK (method 11, :1654-2285).  The reference's hot loop is
//   matvec_add_extfield_kernel (warp per row) -> implicit_solve_kernel ->
//   proposal_residual_kernel -> D2H of the whole residual + host sum.
// Here one kernel does the matvec AND the per-element material step: a warp
// owns the three rows of one element, streams them from HBM with 128-bit
// loads (rows start on 128-byte boundaries), reduces with warp shuffles and
// applies the implicit per-element material solve (FindNewH,
// radmater.cpp:72-164) in its epilogue, writing the proposal M', the element
// field H and the squared step |M' - M|^2.  The misfit (RMS of the undamped
// step, radrlmet.cpp:557-579) is summed on the device in a fixed order, so
// every run is bitwise reproducible.
#include "internal.cuh"
#include "material.cuh"

namespace rb {

template <typename MT> struct VecLoad;
template <> struct VecLoad<float> {
  static constexpr int W = 4;
  __device__ __forceinline__ static void load(const float *p, double *v)
  {
    float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
};
template <> struct VecLoad<double> {
  static constexpr int W = 2;
  __device__ __forceinline__ static void load(const double *p, double *v)
  {
    double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
    v[0] = a.x; v[1] = a.y;
  }
};

// Three-row dot products of element e's rows with x, warp-wide; result in all lanes.
template <typename MT, int U>
__device__ __forceinline__ void rows3_dot(const MT *__restrict__ N, int ld, int e, const double *__restrict__ x,
                                          double &h0, double &h1, double &h2)
{
  constexpr int W = VecLoad<MT>::W;
  const int lane = threadIdx.x & 31;
  const MT *r0 = N + (size_t)(3 * e) * ld;
  const MT *r1 = r0 + ld;
  const MT *r2 = r1 + ld;
  double a0 = 0, a1 = 0, a2 = 0;
  const int step = 32 * W;
  int c = lane * W;
  for (; c + (U - 1) * step < ld; c += U * step) {
    double v0[U][W], v1[U][W], v2[U][W], xv[U][W];
#pragma unroll
    for (int u = 0; u < U; u++) {
      VecLoad<MT>::load(r0 + c + u * step, v0[u]);
      VecLoad<MT>::load(r1 + c + u * step, v1[u]);
      VecLoad<MT>::load(r2 + c + u * step, v2[u]);
#pragma unroll
      for (int w = 0; w < W; w++) xv[u][w] = __ldg(x + c + u * step + w);
    }
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int w = 0; w < W; w++) {
        a0 = fma(v0[u][w], xv[u][w], a0);
        a1 = fma(v1[u][w], xv[u][w], a1);
        a2 = fma(v2[u][w], xv[u][w], a2);
      }
  }
  for (; c < ld; c += step) {
    double v0[W], v1[W], v2[W];
    VecLoad<MT>::load(r0 + c, v0);
    VecLoad<MT>::load(r1 + c, v1);
    VecLoad<MT>::load(r2 + c, v2);
#pragma unroll
    for (int w = 0; w < W; w++) {
      double xv = __ldg(x + c + w);
      a0 = fma(v0[w], xv, a0);
      a1 = fma(v1[w], xv, a1);
      a2 = fma(v2[w], xv, a2);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  h0 = a0; h1 = a1; h2 = a2;
}

constexpr int RLX_WARPS = 8;

// Adds the FP64 near residue of element e's rows (mixed storage) to h,
// warp-wide: lanes take the near entries in turn, then a butterfly reduce.
__device__ __forceinline__ void near_rows3(const NearView &nv, int e, const double *__restrict__ x, double &h0,
                                           double &h1, double &h2)
{
  const int lane = threadIdx.x & 31;
  double a0 = 0, a1 = 0, a2 = 0;
  for (int k = nv.ptr[e] + lane; k < nv.ptr[e + 1]; k += 32) {
    const int j = nv.col[k];
    const double *d = nv.D + 9 * (size_t)k;
    const double x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2];
    a0 += d[0] * x0 + d[1] * x1 + d[2] * x2;
    a1 += d[3] * x0 + d[4] * x1 + d[5] * x2;
    a2 += d[6] * x0 + d[7] * x1 + d[8] * x2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  h0 += a0;
  h1 += a1;
  h2 += a2;
}

// One Jacobi proposal: H = N M + H_ext; per element H' = FindNewH(H - Q_ii M),
// M' = M(H'); writes Mp, Hn, F = M' - M and per-CTA partial sums of |F|^2.
// N holds n rows, or the rows of elements e0 .. e0 + n - 1 of a row block
// (hext, kind, mat, Hn, Mp, F then hold those rows; M is always the full
// magnetization).
template <typename MT>
__global__ void __launch_bounds__(32 * RLX_WARPS) jacobi_kernel(const MT *__restrict__ N, int ld, int n,
                                                               const double *__restrict__ M, const double *__restrict__ hext,
                                                               const int *__restrict__ kind, const double *__restrict__ mat,
                                                               const double *__restrict__ mh,
                                                               double prec_e2, double *__restrict__ Hn,
                                                               double *__restrict__ Mp, double *__restrict__ F,
                                                               double *__restrict__ part, NearView nv, int exact,
                                                               int e0)
{
  __shared__ double ssq[RLX_WARPS];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int e = blockIdx.x * RLX_WARPS + warp;
  double sq = 0.0;
  if (e < n) {
    double h0, h1, h2;
    rows3_dot<MT, 2>(N, ld, e, M, h0, h1, h2);
    if (nv.ptr) near_rows3(nv, e, M, h0, h1, h2);
    if (lane == 0) {
      // row e of a block starting at element e0: its self block is column e0 + e
      double Q[9];
      const int es = e0 + e;
      const MT *d = N + (size_t)(3 * e) * ld + 3 * es;
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Q[3 * a + b] = (double)d[(size_t)a * ld + b];
      double m0 = M[3 * es], m1 = M[3 * es + 1], m2 = M[3 * es + 2];
      V3<double> Hq = mk3<double>(h0 + hext[3 * e] - (Q[0] * m0 + Q[1] * m1 + Q[2] * m2),
                                  h1 + hext[3 * e + 1] - (Q[3] * m0 + Q[4] * m1 + Q[5] * m2),
                                  h2 + hext[3 * e + 2] - (Q[6] * m0 + Q[7] * m1 + Q[8] * m2));
      int k = kind[e];
      const double *mr = mat + (size_t)e * RADB200_MAT_STRIDE;
      V3<double> H0 = mk3<double>(Hn[3 * e], Hn[3 * e + 1], Hn[3 * e + 2]);
      V3<double> H = find_new_h(k, mr, Q, Hq, H0, prec_e2, mh);
      if (exact) H = polish_h(k, mr, Q, Hq, H, mh);
      V3<double> Mn = mat_M(k, mr, H, mh);
      Hn[3 * e] = H.x; Hn[3 * e + 1] = H.y; Hn[3 * e + 2] = H.z;
      Mp[3 * e] = Mn.x; Mp[3 * e + 1] = Mn.y; Mp[3 * e + 2] = Mn.z;
      double f0 = Mn.x - m0, f1 = Mn.y - m1, f2 = Mn.z - m2;
      F[3 * e] = f0; F[3 * e + 1] = f1; F[3 * e + 2] = f2;
      sq = f0 * f0 + f1 * f1 + f2 * f2;
    }
  }
  if (lane == 0) ssq[warp] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < RLX_WARPS; w++) s += ssq[w];
    part[blockIdx.x] = s;
  }
}

// y = N x + b (plain matvec, warp per element, used by NK / refinement / adjoint);
// with nv.ptr set, N is FP32 and the near blocks get their FP64 residue
template <typename MT>
__global__ void __launch_bounds__(32 * RLX_WARPS) matvec_kernel(const MT *__restrict__ N, int ld, int n,
                                                               const double *__restrict__ x, const double *__restrict__ b,
                                                               double alpha, double *__restrict__ y, NearView nv)
{
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int e = blockIdx.x * RLX_WARPS + warp;
  if (e >= n) return;
  double h0, h1, h2;
  rows3_dot<MT, 2>(N, ld, e, x, h0, h1, h2);
  if (nv.ptr) near_rows3(nv, e, x, h0, h1, h2);
  if (lane == 0) {
    double b0 = b ? b[3 * e] : 0.0, b1 = b ? b[3 * e + 1] : 0.0, b2 = b ? b[3 * e + 2] : 0.0;
    y[3 * e] = alpha * h0 + b0;
    y[3 * e + 1] = alpha * h1 + b1;
    y[3 * e + 2] = alpha * h2 + b2;
  }
}

// sum of part[0..n) in a fixed order by one CTA; result to out[0]
__global__ void sum_kernel(const double *__restrict__ part, int n, double *__restrict__ out)
{
  __shared__ double s[256];
  double a = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) a += part[i];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0];
}

// Multi-dot: out[k] = <a_k, b_k> for k < nd, vectors of length len, fixed order.
// part: [gridDim.x][nd] partials.
__global__ void multidot_kernel(DotSet ds, int64_t len, double *__restrict__ part)
{
  __shared__ double red[MD_MAX][8];
  double acc[MD_MAX];
#pragma unroll
  for (int k = 0; k < MD_MAX; k++) acc[k] = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < MD_MAX; k++)
      if (k < ds.nd) acc[k] = fma(ds.a[k][i], ds.b[k][i], acc[k]);
  }
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < MD_MAX; k++) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < ds.nd) {
    double s = 0.0;
    for (int q = 0; q < 8; q++) s += red[threadIdx.x][q];
    part[(size_t)blockIdx.x * ds.nd + threadIdx.x] = s;
  }
}
__global__ void multidot_finish(const double *__restrict__ part, int nb, int nd, double *__restrict__ out)
{
  int k = threadIdx.x;
  if (k >= nd) return;
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += part[(size_t)b * nd + k];
  out[k] = s;
}

__global__ void lincomb_kernel(AxpySet s, int64_t len, double *__restrict__ y, int accumulate)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    double a = accumulate ? y[i] : 0.0;
    for (int k = 0; k < s.nv; k++) a = fma(s.c[k], s.v[k][i], a);
    y[i] = a;
  }
}

// M = Mr of each element (start of a relaxation, radintrc.h:385-395); H = 0
__global__ void reset_kernel(const double *__restrict__ mat, int n, double *__restrict__ M, double *__restrict__ H)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double *m = mat + (size_t)e * RADB200_MAT_STRIDE;
  M[3 * e] = m[9]; M[3 * e + 1] = m[10]; M[3 * e + 2] = m[11];
  H[3 * e] = 0; H[3 * e + 1] = 0; H[3 * e + 2] = 0;
}

// max |M_e| and |H_e| per CTA
__global__ void maxnorm_kernel(const double *__restrict__ M, const double *__restrict__ H, int n, double *__restrict__ out)
{
  __shared__ double sm[256], sh[256];
  double am = 0, ah = 0;
  for (int e = threadIdx.x; e < n; e += 256) {
    double a = sqrt(M[3 * e] * M[3 * e] + M[3 * e + 1] * M[3 * e + 1] + M[3 * e + 2] * M[3 * e + 2]);
    double b = H ? sqrt(H[3 * e] * H[3 * e] + H[3 * e + 1] * H[3 * e + 1] + H[3 * e + 2] * H[3 * e + 2]) : 0.0;
    am = fmax(am, a);
    ah = fmax(ah, b);
  }
  sm[threadIdx.x] = am; sh[threadIdx.x] = ah;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
      sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { out[0] = sm[0]; out[1] = sh[0]; }
}

// ---------------------------------------------------------------------------
// host-side helpers
// ---------------------------------------------------------------------------
struct Ctx {
  Intrc &I;
  cudaStream_t st;
  DBuf part, scal, mdpart;
  Ctx(Intrc &i) : I(i), st(0) {}
};

static int grid_elems(int n) { return (n + RLX_WARPS - 1) / RLX_WARPS; }

// exact: polish each element's implicit field (polish_h) -- the map the
// Newton relaxation differentiates
template <typename MT>
static int jacobi_step(Intrc &I, Ctx &c, const MT *N, double prec_e2, double *misfit, int exact = 0)
{
  int nb = grid_elems(I.n);
  RB_TRY(c.part.alloc((size_t)nb * sizeof(double)));
  RB_TRY(c.scal.alloc(64 * sizeof(double)));
  jacobi_kernel<MT><<<nb, 32 * RLX_WARPS, 0, c.st>>>(N, I.ld, I.n, I.M.as<double>(), I.hext.as<double>(),
                                                      I.mat_kind.as<int>(), I.mat.as<double>(), I.mh.as<double>(), prec_e2,
                                                      I.H.as<double>(), I.Mp.as<double>(), I.F.as<double>(),
                                                      c.part.as<double>(), I.near(), exact, 0);
  RB_TRY(check_launch("jacobi_kernel"));
  sum_kernel<<<1, 256, 0, c.st>>>(c.part.as<double>(), nb, c.scal.as<double>());
  RB_TRY(check_launch("sum_kernel"));
  double s;
  RB_CUDA(cudaMemcpyAsync(&s, c.scal.as<double>(), sizeof(double), cudaMemcpyDeviceToHost, c.st));
  RB_CUDA(cudaStreamSynchronize(c.st));
  *misfit = sqrt(s / I.n);
  return 0;
}

int run_matvec(Intrc &I, const double *x, const double *b, double alpha, double *y, cudaStream_t st)
{
  int nb = grid_elems(I.n);
  if (I.N64.p) matvec_kernel<double><<<nb, 32 * RLX_WARPS, 0, st>>>(I.N64.as<double>(), I.ld, I.n, x, b, alpha, y, NearView());
  else matvec_kernel<float><<<nb, 32 * RLX_WARPS, 0, st>>>(I.N32.as<float>(), I.ld, I.n, x, b, alpha, y, I.near());
  return check_launch("matvec_kernel");
}

int run_matvec_f32(Intrc &I, const double *x, const double *b, double alpha, double *y, cudaStream_t st)
{
  int nb = grid_elems(I.n);
  if (I.N32.p) matvec_kernel<float><<<nb, 32 * RLX_WARPS, 0, st>>>(I.N32.as<float>(), I.ld, I.n, x, b, alpha, y, NearView());
  else matvec_kernel<double><<<nb, 32 * RLX_WARPS, 0, st>>>(I.N64.as<double>(), I.ld, I.n, x, b, alpha, y, NearView());
  return check_launch("matvec_kernel");
}

int multidot(const DotSet &ds, int64_t len, double *host_out, DBuf &part, DBuf &scal, cudaStream_t st)
{
  int nb = 148 * 2;
  RB_TRY(part.alloc((size_t)nb * MD_MAX * sizeof(double)));
  RB_TRY(scal.alloc(64 * sizeof(double)));
  multidot_kernel<<<nb, 256, 0, st>>>(ds, len, part.as<double>());
  RB_TRY(check_launch("multidot_kernel"));
  multidot_finish<<<1, 32, 0, st>>>(part.as<double>(), nb, ds.nd, scal.as<double>());
  RB_TRY(check_launch("multidot_finish"));
  RB_CUDA(cudaMemcpyAsync(host_out, scal.as<double>(), ds.nd * sizeof(double), cudaMemcpyDeviceToHost, st));
  RB_CUDA(cudaStreamSynchronize(st));
  return 0;
}

int lincomb(const AxpySet &s, int64_t len, double *y, int accumulate, cudaStream_t st)
{
  int nb = (int)std::min<int64_t>((len + 255) / 256, 148 * 8);
  if (nb < 1) nb = 1;
  lincomb_kernel<<<nb, 256, 0, st>>>(s, len, y, accumulate);
  return check_launch("lincomb_kernel");
}

// small dense solve (Gaussian elimination with partial pivoting), in place
static int small_solve(std::vector<double> A, std::vector<double> &b, int m)
{
  for (int k = 0; k < m; k++) {
    int p = k;
    for (int i = k + 1; i < m; i++)
      if (fabs(A[i * m + k]) > fabs(A[p * m + k])) p = i;
    if (A[p * m + k] == 0.0) return -1;
    if (p != k) {
      for (int j = 0; j < m; j++) std::swap(A[k * m + j], A[p * m + j]);
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < m; i++) {
      double f = A[i * m + k] / A[k * m + k];
      for (int j = k; j < m; j++) A[i * m + j] -= f * A[k * m + j];
      b[i] -= f * b[k];
    }
  }
  for (int k = m - 1; k >= 0; k--) {
    double s = b[k];
    for (int j = k + 1; j < m; j++) s -= A[k * m + j] * b[j];
    b[k] = s / A[k * m + k];
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Jacobi + Anderson relaxation (methods 3/4/5/8/9/10 reach this fixed point)
// ---------------------------------------------------------------------------
int relax_jacobi(Intrc &I, double prec, int max_iter, double omega0, double *status)
{
  Ctx c(I);
  const int n3 = I.n3;
  const int AM = 6;  // Anderson depth
  RB_TRY(I.work.alloc((size_t)(4 * AM + 4) * I.ld * sizeof(double)));
  double *W = I.work.as<double>();
  RB_CUDA(cudaMemset(W, 0, (size_t)(4 * AM + 4) * I.ld * sizeof(double)));
  double *dX = W;                        // [AM][ld]
  double *dF = W + (size_t)AM * I.ld;    // [AM][ld]
  double *Xprev = W + (size_t)2 * AM * I.ld;
  double *Fprev = Xprev + I.ld;
  double *Mbest = Fprev + I.ld;
  double prec_e2 = prec * prec;
  double omega = (omega0 > 0.0 && omega0 <= 1.0) ? omega0 : 1.0;
  double misfit = 1e30, best = 1e30;
  int hist = 0, head = 0, it = 0;
  std::vector<double> G((size_t)AM * AM, 0.0);
  bool have_prev = false;
  double loc_prec_e2 = prec_e2 / I.n;
  int bad = 0;
  for (it = 1; it <= max_iter; it++) {
    if (I.N64.p) RB_TRY(jacobi_step<double>(I, c, I.N64.as<double>(), loc_prec_e2, &misfit, 1));
    else RB_TRY(jacobi_step<float>(I, c, I.N32.as<float>(), loc_prec_e2, &misfit, 1));
    if (!std::isfinite(misfit)) { set_error("relaxation produced a non-finite misfit"); return RADB200_E_NUMERIC; }
    if (misfit <= prec) {
      // accept the converged proposal (as method 4 stores the new M)
      RB_CUDA(cudaMemcpyAsync(I.M.as<double>(), I.Mp.as<double>(), n3 * sizeof(double), cudaMemcpyDeviceToDevice, c.st));
      break;
    }
    if (misfit < best) {
      best = misfit;
      bad = 0;
    } else if (misfit > 4.0 * best) {
      // divergence guard: drop the history, damp harder
      hist = 0; head = 0; have_prev = false;
      omega = std::max(0.05, 0.5 * omega);
      bad++;
    }
    double *M = I.M.as<double>(), *F = I.F.as<double>();
    if (have_prev) {
      // new differences dX = M - Xprev, dF = F - Fprev into slot head
      AxpySet s1; s1.nv = 2; s1.v[0] = M; s1.c[0] = 1.0; s1.v[1] = Xprev; s1.c[1] = -1.0;
      RB_TRY(lincomb(s1, n3, dX + (size_t)head * I.ld, 0, c.st));
      AxpySet s2; s2.nv = 2; s2.v[0] = F; s2.c[0] = 1.0; s2.v[1] = Fprev; s2.c[1] = -1.0;
      RB_TRY(lincomb(s2, n3, dF + (size_t)head * I.ld, 0, c.st));
      int newslot = head;
      head = (head + 1) % AM;
      if (hist < AM) hist++;
      // Gram row of the new slot and <dF_k, F>
      DotSet ds; ds.nd = 0;
      for (int k = 0; k < hist; k++) {
        int slot = (newslot - k + AM) % AM;
        ds.a[ds.nd] = dF + (size_t)newslot * I.ld; ds.b[ds.nd] = dF + (size_t)slot * I.ld; ds.nd++;
      }
      for (int k = 0; k < hist; k++) {
        int slot = (newslot - k + AM) % AM;
        ds.a[ds.nd] = dF + (size_t)slot * I.ld; ds.b[ds.nd] = F; ds.nd++;
      }
      double dots[2 * MD_MAX];
      RB_TRY(multidot(ds, n3, dots, c.mdpart, c.scal, c.st));
      for (int k = 0; k < hist; k++) {
        int slot = (newslot - k + AM) % AM;
        G[newslot * AM + slot] = G[slot * AM + newslot] = dots[k];
      }
      // gamma = argmin |F - dF gamma|
      std::vector<double> A((size_t)hist * hist), rhs(hist);
      std::vector<int> slots(hist);
      for (int k = 0; k < hist; k++) slots[k] = (newslot - k + AM) % AM;
      double diag = 0.0;
      for (int a = 0; a < hist; a++) diag = std::max(diag, G[slots[a] * AM + slots[a]]);
      for (int a = 0; a < hist; a++) {
        for (int b = 0; b < hist; b++) A[a * hist + b] = G[slots[a] * AM + slots[b]];
        A[a * hist + a] += 1e-10 * diag + 1e-300;
        rhs[a] = dots[hist + a];
      }
      RB_CUDA(cudaMemcpyAsync(Xprev, M, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c.st));
      RB_CUDA(cudaMemcpyAsync(Fprev, F, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c.st));
      if (small_solve(A, rhs, hist) == 0) {
        // M += omega F - sum gamma_k (dX_k + omega dF_k)
        AxpySet s; s.nv = 1 + 2 * hist;
        s.v[0] = F; s.c[0] = omega;
        for (int k = 0; k < hist; k++) {
          s.v[1 + 2 * k] = dX + (size_t)slots[k] * I.ld; s.c[1 + 2 * k] = -rhs[k];
          s.v[2 + 2 * k] = dF + (size_t)slots[k] * I.ld; s.c[2 + 2 * k] = -omega * rhs[k];
        }
        RB_TRY(lincomb(s, n3, M, 1, c.st));
      } else {
        AxpySet s; s.nv = 1; s.v[0] = F; s.c[0] = omega;
        RB_TRY(lincomb(s, n3, M, 1, c.st));
      }
    } else {
      RB_CUDA(cudaMemcpyAsync(Xprev, M, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c.st));
      RB_CUDA(cudaMemcpyAsync(Fprev, F, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c.st));
      have_prev = true;
      AxpySet s; s.nv = 1; s.v[0] = F; s.c[0] = omega;
      RB_TRY(lincomb(s, n3, M, 1, c.st));
    }
    (void)Mbest;
    (void)bad;
  }
  RB_TRY(c.scal.alloc(64 * sizeof(double)));
  maxnorm_kernel<<<1, 256, 0, c.st>>>(I.M.as<double>(), I.H.as<double>(), I.n, c.scal.as<double>());
  RB_TRY(check_launch("maxnorm_kernel"));
  double mm[2];
  RB_CUDA(cudaMemcpy(mm, c.scal.as<double>(), 2 * sizeof(double), cudaMemcpyDeviceToHost));
  status[0] = misfit;
  status[1] = mm[0];
  status[2] = mm[1];
  status[3] = (it > max_iter) ? max_iter : it;
  return 0;
}

// ---------------------------------------------------------------------------
// Newton-Krylov relaxation (method 11 of the reference, radgpurlx.cu:1654-2285)
// ---------------------------------------------------------------------------
// Newton is applied to the fixed-point map Phi of the Jacobi step above
// (per-element implicit material solve), R(M) = Phi(M) - M, rather than to the
// bare residual M(N M + H_ext) - M: for soft iron (chi ~ 1e4) the bare
// residual amplifies every field error by chi and Newton on it diverges from
// any practical start, while Phi already contains the element's own
// demagnetization.  With H_e the element's implicit field and D_e = dM/dH(H_e),
//   dPhi/dM v = B_e ((N v)_e - Q_ee v_e),   B_e = D_e (I - Q_ee D_e)^-1,
// so each Newton step solves (I - dPhi/dM) d = R by GMRES, one matvec per
// Krylov vector, followed by a backtracking line search on the misfit.

template <typename MT>
__global__ void newton_B_kernel(const MT *__restrict__ N, int ld, int n, const double *__restrict__ H,
                                const int *__restrict__ kind, const double *__restrict__ mat,
                                const double *__restrict__ mh, double *__restrict__ B)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double Q[9], D[9], A[9], Ai[9];
  const MT *d = N + (size_t)(3 * e) * ld + 3 * e;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) Q[3 * a + b] = (double)d[(size_t)a * ld + b];
  mat_D(kind[e], mat + (size_t)e * RADB200_MAT_STRIDE, mk3<double>(H[3 * e], H[3 * e + 1], H[3 * e + 2]), D, mh);
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      A[3 * a + b] = (a == b ? 1.0 : 0.0) - (Q[3 * a] * D[b] + Q[3 * a + 1] * D[3 + b] + Q[3 * a + 2] * D[6 + b]);
  inv3x3(A, Ai);
  double *Be = B + 9 * (size_t)e;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      Be[3 * a + b] = D[3 * a] * Ai[b] + D[3 * a + 1] * Ai[3 + b] + D[3 * a + 2] * Ai[6 + b];
}

// out_e = v_e - B_e ((y)_e - Q_ee v_e), y = N v
template <typename MT>
__global__ void newton_apply_kernel(const MT *__restrict__ N, int ld, int n, const double *__restrict__ B,
                                    const double *__restrict__ v, const double *__restrict__ y, double *__restrict__ out)
{
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const MT *d = N + (size_t)(3 * e) * ld + 3 * e;
  double w[3];
  for (int a = 0; a < 3; a++)
    w[a] = y[3 * e + a] - ((double)d[(size_t)a * ld] * v[3 * e] + (double)d[(size_t)a * ld + 1] * v[3 * e + 1] +
                           (double)d[(size_t)a * ld + 2] * v[3 * e + 2]);
  const double *Be = B + 9 * (size_t)e;
  for (int a = 0; a < 3; a++) out[3 * e + a] = v[3 * e + a] - (Be[3 * a] * w[0] + Be[3 * a + 1] * w[1] + Be[3 * a + 2] * w[2]);
}

struct NewtonOp : Op {
  Intrc &I;
  const double *B;
  double *tmp;
  NewtonOp(Intrc &i, const double *b, double *t) : I(i), B(b), tmp(t) {}
  int apply(const double *v, double *out) override
  {
    RB_TRY(run_matvec(I, v, nullptr, 1.0, tmp, 0));
    int nb = (I.n + 127) / 128;
    if (I.N64.p) newton_apply_kernel<double><<<nb, 128>>>(I.N64.as<double>(), I.ld, I.n, B, v, tmp, out);
    else newton_apply_kernel<float><<<nb, 128>>>(I.N32.as<float>(), I.ld, I.n, B, v, tmp, out);
    return check_launch("newton_apply_kernel");
  }
  int precond(double *) override { return 0; }
};

// Krylov settings of the Newton steps; RADB200_NK="c,p,restart,max" overrides
// (tuning aid): forcing term eta = min(0.1, c * misfit^p), GMRES(restart)
// with at most max iterations per step.  On the 6,080-element hybrid
// undulator (saturating poles) to a misfit of 1e-13: 0.3, 0.5, 60, 300 took
// 573 matvecs against 853 for eta = 0.1 misfit with GMRES(50), and larger
// restarts cost more (1,033-1,076).
struct NkParams {
  double eta_c = 0.3, eta_p = 0.5;
  int restart = 60, max_krylov = 300;
};
static NkParams nk_params()
{
  NkParams p;
  const char *e = getenv("RADB200_NK");
  if (e) {
    double c, q;
    int r, m;
    if (sscanf(e, "%lf,%lf,%d,%d", &c, &q, &r, &m) == 4 && c > 0 && q > 0 && r > 0 && m > 0) {
      p.eta_c = c; p.eta_p = q; p.restart = r; p.max_krylov = m;
    }
  }
  return p;
}

int relax_newton(Intrc &I, double prec, int max_iter, double *status)
{
  const NkParams nk = nk_params();
  Ctx c(I);
  const int n = I.n, n3 = I.n3, ld = I.ld;
  DBuf buf;
  RB_TRY(buf.alloc((size_t)(4 * ld + 9 * (size_t)n) * sizeof(double)));
  RB_CUDA(cudaMemset(buf.p, 0, (size_t)(4 * ld + 9 * (size_t)n) * sizeof(double)));
  double *d = buf.as<double>(), *tmp = d + ld, *M0 = tmp + ld, *R0 = M0 + ld, *B = R0 + ld;
  double *M = I.M.as<double>();
  const double loc = prec * prec / n;
  auto step = [&](double *mis) -> int {
    if (I.N64.p) return jacobi_step<double>(I, c, I.N64.as<double>(), loc, mis, 1);
    return jacobi_step<float>(I, c, I.N32.as<float>(), loc, mis, 1);
  };
  double misfit;
  RB_TRY(step(&misfit));
  int matvecs = 1, newton = 0;
  while (misfit > prec && matvecs < max_iter && newton < 100) {
    newton++;
    int nb = (n + 127) / 128;
    if (I.N64.p) newton_B_kernel<double><<<nb, 128>>>(I.N64.as<double>(), ld, n, I.H.as<double>(), I.mat_kind.as<int>(), I.mat.as<double>(), I.mh.as<double>(), B);
    else newton_B_kernel<float><<<nb, 128>>>(I.N32.as<float>(), ld, n, I.H.as<double>(), I.mat_kind.as<int>(), I.mat.as<double>(), I.mh.as<double>(), B);
    RB_TRY(check_launch("newton_B_kernel"));
    RB_CUDA(cudaMemcpy(R0, I.F.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice));
    RB_CUDA(cudaMemcpy(M0, M, n3 * sizeof(double), cudaMemcpyDeviceToDevice));
    RB_CUDA(cudaMemset(d, 0, n3 * sizeof(double)));
    NewtonOp op(I, B, tmp);
    double rel;
    int its;
    double eta = std::min(0.1, std::max(1e-10, nk.eta_c * pow(misfit, nk.eta_p)));
    RB_TRY(gmres(op, n3, ld, R0, d, eta, std::max(1, std::min(nk.max_krylov, max_iter - matvecs)), nk.restart, &rel, &its,
                 0));
    matvecs += its + 1;
    double lam = 1.0, newmis = misfit;
    bool ok = false;
    for (int ls = 0; ls < 6; ls++) {
      AxpySet s; s.nv = 2; s.v[0] = M0; s.c[0] = 1.0; s.v[1] = d; s.c[1] = lam;
      RB_TRY(lincomb(s, n3, M, 0, 0));
      RB_TRY(step(&newmis));
      matvecs++;
      if (std::isfinite(newmis) && newmis < misfit) { ok = true; break; }
      lam *= 0.5;
    }
    if (!ok) {
      // no descent along the Newton direction: restore and fall back to the
      // Anderson-mixed fixed-point iteration for the rest of the budget
      RB_CUDA(cudaMemcpy(M, M0, n3 * sizeof(double), cudaMemcpyDeviceToDevice));
      double st[4];
      RB_TRY(relax_jacobi(I, prec, std::max(1, max_iter - matvecs), 0.0, st));
      matvecs += (int)st[3];
      misfit = st[0];
      break;
    }
    if (timing_on())
      fprintf(stderr, "RADB200_TIMING newton %d: gmres %d its (rel %.2e), step %.3g, misfit %.3e -> %.3e\n", newton, its,
              rel, lam, misfit, newmis);
    misfit = newmis;
  }
  if (misfit <= prec)  // accept the last proposal, as the fixed-point iteration does
    RB_CUDA(cudaMemcpy(M, I.Mp.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice));
  RB_TRY(c.scal.alloc(64 * sizeof(double)));
  maxnorm_kernel<<<1, 256>>>(M, I.H.as<double>(), n, c.scal.as<double>());
  RB_TRY(check_launch("maxnorm_kernel"));
  double mm[2];
  RB_CUDA(cudaMemcpy(mm, c.scal.as<double>(), 2 * sizeof(double), cudaMemcpyDeviceToHost));
  status[0] = misfit; status[1] = mm[0]; status[2] = mm[1]; status[3] = matvecs;
  return 0;
}

// One Jacobi proposal of a row block from the full magnetization M (device):
// Mp and F of its rows, the block's sum of |F_e|^2 to the host.  The implicit
// per-element solve stops at prec^2 / n like relax_jacobi's.
int relax_rows_step(Intrc &I, const double *M, double prec, double *Mp, double *F, double *sq_sum)
{
  Ctx c(I);
  const int nb = grid_elems(I.nr);
  RB_TRY(c.part.alloc((size_t)nb * sizeof(double)));
  RB_TRY(c.scal.alloc(64 * sizeof(double)));
  const double loc = prec * prec / I.n;
  const int *kind = I.mat_kind.as<int>() + I.e0;
  const double *mat = I.mat.as<double>() + (size_t)I.e0 * RADB200_MAT_STRIDE;
  if (I.N64.p)
    jacobi_kernel<double><<<nb, 32 * RLX_WARPS, 0, c.st>>>(I.N64.as<double>(), I.ld, I.nr, M, I.hext.as<double>(), kind, mat,
                                                           I.mh.as<double>(), loc, I.H.as<double>(), Mp, F,
                                                           c.part.as<double>(), NearView(), 1, I.e0);
  else
    jacobi_kernel<float><<<nb, 32 * RLX_WARPS, 0, c.st>>>(I.N32.as<float>(), I.ld, I.nr, M, I.hext.as<double>(), kind, mat,
                                                          I.mh.as<double>(), loc, I.H.as<double>(), Mp, F,
                                                          c.part.as<double>(), NearView(), 1, I.e0);
  RB_TRY(check_launch("jacobi_kernel"));
  sum_kernel<<<1, 256, 0, c.st>>>(c.part.as<double>(), nb, c.scal.as<double>());
  RB_TRY(check_launch("sum_kernel"));
  RB_CUDA(cudaMemcpyAsync(sq_sum, c.scal.as<double>(), sizeof(double), cudaMemcpyDeviceToHost, c.st));
  RB_CUDA(cudaStreamSynchronize(c.st));
  return 0;
}

int relax_reset(Intrc &I)
{
  reset_kernel<<<(I.n + 127) / 128, 128>>>(I.mat.as<double>(), I.n, I.M.as<double>(), I.H.as<double>());
  return check_launch("reset_kernel");
}

}  // namespace rb
