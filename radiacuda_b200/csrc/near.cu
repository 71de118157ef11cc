// near.cu -- the near pairs of mixed storage.
//
// Mixed storage (RADB200_STORE_MIXED) keeps every block of the interaction
// matrix in FP32 and, for the pairs whose elements are close, the FP64
// residue D = N - N32 of the block.  Rounding a block to FP32 costs at most
// 2^-24 of each of its entries, so the absolute error of a row of N x is
// dominated by its largest blocks: the self block and the neighbours, where
// the demagnetizing tensor is O(1), while a block at distance d falls off as
// V / (4 pi d^3).  With the residue of the near blocks added back, the FP64
// operator (refinement residual r = b - A M, transposed products of the
// adjoint) is exact to FP64 rounding there and carries only the FP32
// rounding of far blocks, whose entries are smaller than the self block's by
// the factor (r / d)^3 or more.
//
// Near: some image of element j has its centre within
// factor * (r_i + r_j) of element i's observation point, r the largest
// distance of an element's vertices from its centre (RADB200_NEAR_FACTOR,
// default 1.5).  Found with a uniform grid over the image centres: the host
// bins the centres, a warp per observer row searches its box of cells on the
// device, and two radix sorts give the rows in column order and the entries
// grouped by column for the transposed product.
#include <math.h>
#include <stdlib.h>

#include <algorithm>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "internal.cuh"

namespace rb {

namespace {

// largest distance of the element's vertices from its centre (object frame)
double elem_radius(const RadB200Geom *G, int kind, int idx)
{
  if (kind == 0) {
    const double *r = G->rec + (size_t)idx * RADB200_REC_STRIDE;
    return 0.5 * sqrt(r[3] * r[3] + r[4] * r[4] + r[5] * r[5]);
  }
  const double *c = G->poly + (size_t)idx * RADB200_POLY_STRIDE;
  int f0 = G->poly_info[4 * idx], nf = G->poly_info[4 * idx + 1];
  double rmax = 0.0;
  for (int f = f0; f < f0 + nf; f++) {
    const double *R = G->face + (size_t)f * RADB200_FACE_STRIDE;
    int v0 = G->face_vtx[2 * f], nv = G->face_vtx[2 * f + 1];
    for (int k = 0; k < nv; k++) {
      double x = G->vtx2d[2 * (size_t)(v0 + k)], y = G->vtx2d[2 * (size_t)(v0 + k) + 1], z = R[9];
      // object-frame vertex: R^T (x, y, z)
      double P[3] = {x * R[0] + y * R[3] + z * R[6], x * R[1] + y * R[4] + z * R[7], x * R[2] + y * R[5] + z * R[8]};
      double d = sqrt((P[0] - c[0]) * (P[0] - c[0]) + (P[1] - c[1]) * (P[1] - c[1]) + (P[2] - c[2]) * (P[2] - c[2]));
      rmax = std::max(rmax, d);
    }
  }
  return rmax;
}

}  // namespace

// Uniform grid over the image centres: the host bins them (a counting sort,
// O(images)), the device searches the rows.
struct NearGrid {
  const double *ic;    // [3 * ni] image centres
  const int *iel;      // [ni] element of each image (images of an element are consecutive)
  const int *ifirst;   // [n] first image of each element
  const double *rad;   // [n] element radii
  const int *cstart;   // [ncell + 1]
  const int *cidx;     // [ni] image numbers by cell
  double lo[3];
  double cell, kf, rmax;
  int dim[3];
};

__device__ __forceinline__ bool near_pass(const NearGrid &q, const double *o, double ri, int m, int j)
{
  const double dx = q.ic[3 * m] - o[0], dy = q.ic[3 * m + 1] - o[1], dz = q.ic[3 * m + 2] - o[2];
  const double lim = q.kf * (ri + q.rad[j]);
  return dx * dx + dy * dy + dz * dz <= lim * lim;
}

// a row holds element j once: at its first image that passes
__device__ __forceinline__ bool near_rep(const NearGrid &q, const double *o, double ri, int m, int j)
{
  if (!near_pass(q, o, ri, m, j)) return false;
  for (int m2 = q.ifirst[j]; m2 < m; m2++)
    if (near_pass(q, o, ri, m2, j)) return false;
  return true;
}

// A warp per observer row i: the lanes take the cells of the search box in
// turn.  COUNT: count[i] = entries of row i.  FILL: the entries go to
// key[ptr[i] ...] as (i << 32 | j), in arrival order (sorted afterwards).
template <bool FILL>
__global__ void __launch_bounds__(256) near_rows_kernel(NearGrid q, const double *__restrict__ obs, int n,
                                                        long long *__restrict__ count, const long long *__restrict__ ptr,
                                                        unsigned long long *__restrict__ key)
{
  __shared__ int cursor[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * 8 + w;
  if (i >= n) return;
  const double o[3] = {obs[3 * i], obs[3 * i + 1], obs[3 * i + 2]};
  const double ri = q.rad[i];
  const double R = q.kf * (ri + q.rmax);
  int qlo[3], qn[3];
  for (int a = 0; a < 3; a++) {
    const int l = max(0, (int)floor((o[a] - R - q.lo[a]) / q.cell));
    const int h = min(q.dim[a] - 1, (int)floor((o[a] + R - q.lo[a]) / q.cell));
    qlo[a] = l;
    qn[a] = max(0, h - l + 1);
  }
  const int box = qn[0] * qn[1] * qn[2];
  if (FILL) {
    if (lane == 0) cursor[w] = 0;
    __syncwarp();
  }
  int cnt = 0;
  bool self = false;
  for (int t = lane; t < box; t += 32) {
    const int x = qlo[0] + t % qn[0], y = qlo[1] + (t / qn[0]) % qn[1], z = qlo[2] + t / (qn[0] * qn[1]);
    const size_t c = ((size_t)z * q.dim[1] + y) * q.dim[0] + x;
    for (int k = q.cstart[c]; k < q.cstart[c + 1]; k++) {
      const int m = q.cidx[k], j = q.iel[m];
      if (!near_rep(q, o, ri, m, j)) continue;
      self |= (j == i);
      if (FILL) key[ptr[i] + atomicAdd(&cursor[w], 1)] = ((unsigned long long)i << 32) | (unsigned)j;
      else cnt++;
    }
  }
  // the self block is always near
  const bool has_self = __any_sync(0xffffffffu, self);
  if (FILL) {
    __syncwarp();
    if (lane == 0 && !has_self) key[ptr[i] + cursor[w]] = ((unsigned long long)i << 32) | (unsigned)i;
  } else {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, s);
    if (lane == 0) count[i] = cnt + (has_self ? 0 : 1);
  }
}

// sorted keys -> row / column of each entry; the column keys for the transposed order
__global__ void near_split_kernel(const unsigned long long *__restrict__ key, long long nnz, int *__restrict__ row,
                                  int *__restrict__ col, int *__restrict__ tkey, int *__restrict__ tval)
{
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const unsigned long long v = key[k];
  row[k] = (int)(v >> 32);
  col[k] = (int)(v & 0xffffffffu);
  tkey[k] = (int)(v & 0xffffffffu);
  tval[k] = (int)k;
}

// first entry of each column group (every column holds at least its self entry)
__global__ void near_tptr_kernel(const int *__restrict__ tkey, long long nnz, int n, int *__restrict__ tptr)
{
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  if (p == 0 || tkey[p - 1] != tkey[p]) tptr[tkey[p]] = (int)p;
  if (p == 0) tptr[n] = (int)nnz;
}

__global__ void near_ptr32_kernel(const long long *__restrict__ p64, int n, int *__restrict__ p32)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= n) p32[i] = (int)p64[i];
}

static int bits_for(int n)
{
  int b = 1;
  while ((1ll << b) < (long long)n) b++;
  return b;
}

int build_near(Intrc &I, const RadB200Geom *G, const RadB200Relax *r, const double *obs)
{
  const int n = I.n;
  const char *env = getenv("RADB200_NEAR_FACTOR");
  const double kf = env ? atof(env) : 1.5;
  I.near_factor = kf;
  std::vector<double> rad(n);
  // image centres of every element, element by element
  std::vector<double> ic;
  std::vector<int> iel, ifirst(n);
  for (int e = 0; e < n; e++) {
    int kind = r->elem_src[2 * e], idx = r->elem_src[2 * e + 1];
    rad[e] = elem_radius(G, kind, idx);
    const double *c;
    int t0, nt;
    if (kind == 0) { c = G->rec + (size_t)idx * RADB200_REC_STRIDE; t0 = G->rec_img[2 * idx]; nt = G->rec_img[2 * idx + 1]; }
    else { c = G->poly + (size_t)idx * RADB200_POLY_STRIDE; t0 = G->poly_info[4 * idx + 2]; nt = G->poly_info[4 * idx + 3]; }
    ifirst[e] = (int)iel.size();
    for (int t = t0; t < t0 + nt; t++) {
      const double *T = G->trf + (size_t)t * RADB200_TRF_STRIDE;
      const double s = T[21];
      for (int a = 0; a < 3; a++)
        ic.push_back((T[12 + 3 * a] * c[0] + T[13 + 3 * a] * c[1] + T[14 + 3 * a] * c[2]) / s + T[9 + a]);
      iel.push_back(e);
    }
  }
  const int ni = (int)iel.size();
  std::vector<double> rs(rad);
  std::nth_element(rs.begin(), rs.begin() + n / 2, rs.end());
  const double rmed = std::max(rs[n / 2], 1e-12), rmax = *std::max_element(rad.begin(), rad.end());
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int k = 0; k < ni; k++)
    for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], ic[3 * k + a]); hi[a] = std::max(hi[a], ic[3 * k + a]); }
  // cells of factor * median radius, widened while the grid would hold many
  // more cells than image centres (few elements spread far apart); every
  // centre then lies inside the grid
  double cell = std::max(kf * rmed, 1e-12 * std::max(1.0, rmax));
  double dd[3];
  for (;;) {
    for (int a = 0; a < 3; a++) dd[a] = floor((hi[a] - lo[a]) / cell) + 1.0;
    if (dd[0] * dd[1] * dd[2] <= 8.0 * ni + 64.0) break;
    cell *= 2.0;
  }
  int dim[3] = {(int)dd[0], (int)dd[1], (int)dd[2]};
  auto cell_of = [&](const double *p) {
    int q[3];
    for (int a = 0; a < 3; a++) q[a] = std::min(dim[a] - 1, std::max(0, (int)floor((p[a] - lo[a]) / cell)));
    return ((size_t)q[2] * dim[1] + q[1]) * dim[0] + q[0];
  };
  const size_t ncell = (size_t)dim[0] * dim[1] * dim[2];
  std::vector<int> cstart(ncell + 1, 0), cidx(ni);
  for (int k = 0; k < ni; k++) cstart[cell_of(&ic[3 * k]) + 1]++;
  for (size_t c = 0; c < ncell; c++) cstart[c + 1] += cstart[c];
  {
    std::vector<int> fill(cstart.begin(), cstart.end() - 1);
    for (int k = 0; k < ni; k++) cidx[fill[cell_of(&ic[3 * k])]++] = k;
  }
  DBuf d_ic, d_iel, d_ifirst, d_rad, d_cstart, d_cidx;
  RB_TRY(d_ic.upload(ic.data(), ic.size() * sizeof(double)));
  RB_TRY(d_iel.upload(iel.data(), iel.size() * sizeof(int)));
  RB_TRY(d_ifirst.upload(ifirst.data(), ifirst.size() * sizeof(int)));
  RB_TRY(d_rad.upload(rad.data(), rad.size() * sizeof(double)));
  RB_TRY(d_cstart.upload(cstart.data(), cstart.size() * sizeof(int)));
  RB_TRY(d_cidx.upload(cidx.data(), cidx.size() * sizeof(int)));
  NearGrid q;
  q.ic = d_ic.as<double>(); q.iel = d_iel.as<int>(); q.ifirst = d_ifirst.as<int>(); q.rad = d_rad.as<double>();
  q.cstart = d_cstart.as<int>(); q.cidx = d_cidx.as<int>();
  for (int a = 0; a < 3; a++) { q.lo[a] = lo[a]; q.dim[a] = dim[a]; }
  q.cell = cell; q.kf = kf; q.rmax = rmax;

  // rows: count, scan (64-bit), fill, sort by (row, column)
  DBuf d_count, d_ptr64, tmp;
  RB_TRY(d_count.alloc((size_t)(n + 1) * sizeof(long long)));
  RB_TRY(d_ptr64.alloc((size_t)(n + 1) * sizeof(long long)));
  RB_CUDA(cudaMemset(d_count.p, 0, (size_t)(n + 1) * sizeof(long long)));
  const unsigned rb = (unsigned)((n + 7) / 8);
  near_rows_kernel<false><<<rb, 256>>>(q, I.obs.as<double>(), n, d_count.as<long long>(), nullptr, nullptr);
  RB_TRY(check_launch("near_rows_kernel<count>"));
  size_t tb = 0;
  RB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_count.as<long long>(), d_ptr64.as<long long>(), n + 1));
  RB_TRY(tmp.alloc(std::max<size_t>(tb, 16)));
  RB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, d_count.as<long long>(), d_ptr64.as<long long>(), n + 1));
  long long nnz = 0;
  RB_CUDA(cudaMemcpy(&nnz, d_ptr64.as<long long>() + n, sizeof(long long), cudaMemcpyDeviceToHost));
  if (nnz > (long long)2000000000) { set_error("near list too long (%lld pairs)", nnz); return RADB200_E_NOMEM; }
  DBuf k0, k1;
  RB_TRY(k0.alloc((size_t)nnz * 8));
  RB_TRY(k1.alloc((size_t)nnz * 8));
  near_rows_kernel<true><<<rb, 256>>>(q, I.obs.as<double>(), n, nullptr, d_ptr64.as<long long>(), k0.as<unsigned long long>());
  RB_TRY(check_launch("near_rows_kernel<fill>"));
  const int nb = bits_for(n);
  tb = 0;
  RB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, k0.as<unsigned long long>(), k1.as<unsigned long long>(), (int)nnz, 0,
                                         32 + nb));
  RB_TRY(tmp.alloc(std::max<size_t>(tb, 16)));
  RB_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, k0.as<unsigned long long>(), k1.as<unsigned long long>(), (int)nnz, 0,
                                         32 + nb));
  I.near_nnz = nnz;
  RB_TRY(I.near_ptr.alloc((size_t)(n + 1) * sizeof(int)));
  RB_TRY(I.near_row.alloc((size_t)nnz * sizeof(int)));
  RB_TRY(I.near_col.alloc((size_t)nnz * sizeof(int)));
  RB_TRY(I.near_tptr.alloc((size_t)(n + 1) * sizeof(int)));
  RB_TRY(I.near_tidx.alloc((size_t)nnz * sizeof(int)));
  near_ptr32_kernel<<<(unsigned)((n + 256) / 256), 256>>>(d_ptr64.as<long long>(), n, I.near_ptr.as<int>());
  RB_TRY(check_launch("near_ptr32_kernel"));
  // transposed order: entries grouped by column, rows ascending inside a
  // group (a stable sort of the row-ordered entries by column)
  // the unsorted keys are spent: their buffer holds the two column-key arrays
  int *tkey = (int *)k0.p, *tkey2 = tkey + nnz;
  DBuf d_tval;
  RB_TRY(d_tval.alloc((size_t)nnz * sizeof(int)));
  int *tval = d_tval.as<int>();
  const unsigned eb = (unsigned)((nnz + 255) / 256);
  near_split_kernel<<<eb, 256>>>(k1.as<unsigned long long>(), nnz, I.near_row.as<int>(), I.near_col.as<int>(), tkey, tval);
  RB_TRY(check_launch("near_split_kernel"));
  tb = 0;
  RB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, tkey, tkey2, tval, I.near_tidx.as<int>(), (int)nnz, 0, nb));
  RB_TRY(tmp.alloc(std::max<size_t>(tb, 16)));
  RB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, tkey, tkey2, tval, I.near_tidx.as<int>(), (int)nnz, 0, nb));
  near_tptr_kernel<<<eb, 256>>>(tkey2, nnz, n, I.near_tptr.as<int>());
  RB_TRY(check_launch("near_tptr_kernel"));
  RB_TRY(I.near_D.alloc((size_t)nnz * 9 * sizeof(double)));
  return launch_assemble_near(I.geom.view(I.fast), I.elem_src.as<int>(), I.obs.as<double>(), I.rowT.as<double>(), I.ld,
                              I.N32.as<float>(), I.near_row.as<int>(), I.near_col.as<int>(), nnz, I.near_D.as<double>(), 0);
}

// out[j] += sum_i D_ij^T x_i: a warp per source element j gathers its entries
__global__ void __launch_bounds__(256) near_t_kernel(NearView nv, int n, const double *__restrict__ x,
                                                     double *__restrict__ out)
{
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (j >= n) return;
  double a0 = 0, a1 = 0, a2 = 0;
  for (int q = nv.tptr[j] + lane; q < nv.tptr[j + 1]; q += 32) {
    const int k = nv.tidx[q];
    const int lo = nv.row[k];  // observer of entry k
    const double *d = nv.D + 9 * (size_t)k;
    const double x0 = x[3 * lo], x1 = x[3 * lo + 1], x2 = x[3 * lo + 2];
    a0 += d[0] * x0 + d[3] * x1 + d[6] * x2;
    a1 += d[1] * x0 + d[4] * x1 + d[7] * x2;
    a2 += d[2] * x0 + d[5] * x1 + d[8] * x2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  if (lane == 0) {
    out[3 * j] += a0;
    out[3 * j + 1] += a1;
    out[3 * j + 2] += a2;
  }
}

int launch_near_t(const Intrc &I, const double *x, double *out, cudaStream_t st)
{
  if (I.near_nnz == 0) return 0;
  near_t_kernel<<<(I.n + 7) / 8, 256, 0, st>>>(I.near(), I.n, x, out);
  return check_launch("near_t_kernel");
}

}  // namespace rb
