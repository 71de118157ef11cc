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
// default 1.5).  Found with a uniform grid over the image centres.
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <thread>

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

int build_near(Intrc &I, const RadB200Geom *G, const RadB200Relax *r, const double *obs)
{
  const int n = I.n;
  const char *env = getenv("RADB200_NEAR_FACTOR");
  const double kf = env ? atof(env) : 1.5;
  I.near_factor = kf;
  std::vector<double> rad(n);
  // image centres of every element: (x, y, z, element)
  std::vector<double> ic;
  std::vector<int> iel;
  for (int e = 0; e < n; e++) {
    int kind = r->elem_src[2 * e], idx = r->elem_src[2 * e + 1];
    rad[e] = elem_radius(G, kind, idx);
    const double *c;
    int t0, nt;
    if (kind == 0) { c = G->rec + (size_t)idx * RADB200_REC_STRIDE; t0 = G->rec_img[2 * idx]; nt = G->rec_img[2 * idx + 1]; }
    else { c = G->poly + (size_t)idx * RADB200_POLY_STRIDE; t0 = G->poly_info[4 * idx + 2]; nt = G->poly_info[4 * idx + 3]; }
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
  // grid over the image centres, cell = factor * median radius
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
  auto cell_of = [&](const double *p, int *q) {
    for (int a = 0; a < 3; a++) q[a] = std::min(dim[a] - 1, std::max(0, (int)floor((p[a] - lo[a]) / cell)));
  };
  const size_t ncell = (size_t)dim[0] * dim[1] * dim[2];
  std::vector<int> cstart(ncell + 1, 0), cidx(ni);
  for (int k = 0; k < ni; k++) {
    int q[3];
    cell_of(&ic[3 * k], q);
    cstart[((size_t)q[2] * dim[1] + q[1]) * dim[0] + q[0] + 1]++;
  }
  for (size_t c = 0; c < ncell; c++) cstart[c + 1] += cstart[c];
  {
    std::vector<int> fill(cstart.begin(), cstart.end() - 1);
    for (int k = 0; k < ni; k++) {
      int q[3];
      cell_of(&ic[3 * k], q);
      cidx[fill[((size_t)q[2] * dim[1] + q[1]) * dim[0] + q[0]]++] = k;
    }
  }
  // rows in parallel: each thread owns a contiguous range of observers
  unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::vector<int>> rows(n);
  auto work = [&](int e0, int e1) {
    std::vector<int> seen(n, -1);
    for (int i = e0; i < e1; i++) {
      const double *o = obs + 3 * (size_t)i;
      const double R = kf * (rad[i] + rmax);
      int qlo[3], qhi[3];
      for (int a = 0; a < 3; a++) {
        qlo[a] = std::max(0, (int)floor((o[a] - R - lo[a]) / cell));
        qhi[a] = std::min(dim[a] - 1, (int)floor((o[a] + R - lo[a]) / cell));
      }
      std::vector<int> &row = rows[i];
      for (int z = qlo[2]; z <= qhi[2]; z++)
        for (int y = qlo[1]; y <= qhi[1]; y++)
          for (int x = qlo[0]; x <= qhi[0]; x++) {
            size_t c = ((size_t)z * dim[1] + y) * dim[0] + x;
            for (int k = cstart[c]; k < cstart[c + 1]; k++) {
              int m = cidx[k], j = iel[m];
              if (seen[j] == i) continue;
              const double *p = &ic[3 * (size_t)m];
              double d2 = (p[0] - o[0]) * (p[0] - o[0]) + (p[1] - o[1]) * (p[1] - o[1]) + (p[2] - o[2]) * (p[2] - o[2]);
              double lim = kf * (rad[i] + rad[j]);
              if (d2 <= lim * lim) {
                seen[j] = i;
                row.push_back(j);
              }
            }
          }
      if (seen[i] != i) row.push_back(i);  // the self block is always near
      std::sort(row.begin(), row.end());
    }
  };
  {
    std::vector<std::thread> th;
    int per = (n + (int)nth - 1) / (int)nth;
    for (unsigned t = 0; t < nth; t++) {
      int e0 = (int)t * per, e1 = std::min(n, e0 + per);
      if (e0 < e1) th.emplace_back(work, e0, e1);
    }
    for (auto &t : th) t.join();
  }
  int64_t nnz = 0;
  for (int i = 0; i < n; i++) nnz += (int64_t)rows[i].size();
  if (nnz > (int64_t)2000000000) { set_error("near list too long (%lld pairs)", (long long)nnz); return RADB200_E_NOMEM; }
  I.h_near_ptr.assign(n + 1, 0);
  for (int i = 0; i < n; i++) I.h_near_ptr[i + 1] = I.h_near_ptr[i] + (int)rows[i].size();
  I.h_near_col.resize(nnz);
  std::vector<int> hrow(nnz);
  for (int i = 0; i < n; i++) {
    std::copy(rows[i].begin(), rows[i].end(), I.h_near_col.begin() + I.h_near_ptr[i]);
    std::fill(hrow.begin() + I.h_near_ptr[i], hrow.begin() + I.h_near_ptr[i + 1], i);
  }
  // entries grouped by source element, rows ascending inside a group
  std::vector<int> tptr(n + 1, 0), tidx(nnz);
  for (int64_t k = 0; k < nnz; k++) tptr[I.h_near_col[k] + 1]++;
  for (int j = 0; j < n; j++) tptr[j + 1] += tptr[j];
  {
    std::vector<int> fill(tptr.begin(), tptr.end() - 1);
    for (int64_t k = 0; k < nnz; k++) tidx[fill[I.h_near_col[k]]++] = (int)k;
  }
  I.near_nnz = nnz;
  RB_TRY(I.near_ptr.upload(I.h_near_ptr.data(), (n + 1) * sizeof(int)));
  RB_TRY(I.near_col.upload(I.h_near_col.data(), nnz * sizeof(int)));
  RB_TRY(I.near_tptr.upload(tptr.data(), (n + 1) * sizeof(int)));
  RB_TRY(I.near_tidx.upload(tidx.data(), nnz * sizeof(int)));
  RB_TRY(I.near_D.alloc((size_t)nnz * 9 * sizeof(double)));
  // observer of every entry, for the assembly pass only
  DBuf drow;
  RB_TRY(drow.upload(hrow.data(), nnz * sizeof(int)));
  RB_CUDA(cudaMemset(I.near_D.p, 0, (size_t)nnz * 9 * sizeof(double)));
  return launch_assemble_near(I.geom.view(I.fast), I.elem_src.as<int>(), I.obs.as<double>(), I.rowT.as<double>(), I.ld,
                              I.N32.as<float>(), drow.as<int>(), I.near_col.as<int>(), nnz, I.near_D.as<double>(), 0);
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
    // observer of entry k: the row whose range holds k
    int lo = 0, hi = n;
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (nv.ptr[mid] <= k) lo = mid; else hi = mid;
    }
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
