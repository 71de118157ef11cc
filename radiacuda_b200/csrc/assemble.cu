// assemble.cu -- dense interaction matrix on the device.
//
// Replaces assemble_mixed_kernel / pair_block_dev / store_block_rowmajor of
// the reference plugin (radgpu_asm.cu:68-105, 576-795); the arithmetic
// contract is the reference CPU loop radintrc.cpp:831-877:
//   block(i,j) = (s_i M_i^-1) * sum_images (s M) Q_j(M^-1 (obs_i - V))
// with Q_j the cuboid tensor (radrec.cpp:115-283) or the polyhedron face sum
// (radvlpgn.cpp:441-505, face tensor radplnr2.cpp:367-375).
//
// Layout: row-major [3N x ld], ld = 3N rounded up to 32 elements so every row
// starts on a 128-byte boundary (vectorised, coalesced matvec loads).  A CTA
// owns an 8 x 32 element tile (24 x 96 matrix entries); each thread computes
// one 3x3 block in FP64 (the transcendental-bound part), the CTA stages the
// tile in shared memory and writes it back row by row, fully coalesced.
#include "tensor.cuh"

namespace rb {

constexpr int ATI = 8, ATJ = 32;

// 3x3 block of the interaction of element i (observer) with element j (source).
__device__ __forceinline__ void pair_block(const GeomView &g, const int *elem_src, V3<double> obs, const double *rowT_i,
                                           int j, double *out)
{
  int kind = __ldg(elem_src + 2 * j), idx = __ldg(elem_src + 2 * j + 1);
  int t0, nt;
  if (kind == 0) { t0 = __ldg(g.rec_img + 2 * idx); nt = __ldg(g.rec_img + 2 * idx + 1); }
  else { t0 = __ldg(g.poly_info + 4 * idx + 2); nt = __ldg(g.poly_info + 4 * idx + 3); }
  double B[9];
#pragma unroll
  for (int k = 0; k < 9; k++) B[k] = 0.0;
  for (int t = t0; t < t0 + nt; t++) {
    const double *Tr = g.trf + (size_t)t * RADB200_TRF_STRIDE;
    double dx = obs.x - __ldg(Tr + 9), dy = obs.y - __ldg(Tr + 10), dz = obs.z - __ldg(Tr + 11);
    V3<double> q = mk3<double>(__ldg(Tr + 0) * dx + __ldg(Tr + 1) * dy + __ldg(Tr + 2) * dz,
                               __ldg(Tr + 3) * dx + __ldg(Tr + 4) * dy + __ldg(Tr + 5) * dz,
                               __ldg(Tr + 6) * dx + __ldg(Tr + 7) * dy + __ldg(Tr + 8) * dz);
    double Q[9];
    elem_tensor(g, kind, idx, q, Q);
    const double *F = Tr + 12;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      double f0 = __ldg(F + 3 * a), f1 = __ldg(F + 3 * a + 1), f2 = __ldg(F + 3 * a + 2);
#pragma unroll
      for (int b = 0; b < 3; b++) B[3 * a + b] += f0 * Q[b] + f1 * Q[3 + b] + f2 * Q[6 + b];
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++)
      out[3 * a + b] = rowT_i[3 * a] * B[b] + rowT_i[3 * a + 1] * B[3 + b] + rowT_i[3 * a + 2] * B[6 + b];
}

// rows: the nr observers of obs / rowT; columns: all n source elements
template <typename OutT>
__global__ void __launch_bounds__(256) assemble_kernel(GeomView g, const int *__restrict__ elem_src,
                                                       const double *__restrict__ obs, const double *__restrict__ rowT,
                                                       int nr, int n, int ld, OutT *__restrict__ N)
{
  __shared__ OutT tile[3 * ATI][3 * ATJ + 1];
  int ti = threadIdx.x / ATJ, tj = threadIdx.x % ATJ;
  int i0 = blockIdx.y * ATI, j0 = blockIdx.x * ATJ;
  int i = i0 + ti, j = j0 + tj;
  double blk[9];
#pragma unroll
  for (int k = 0; k < 9; k++) blk[k] = 0.0;
  if (i < nr && j < n) {
    V3<double> o = mk3<double>(__ldg(obs + 3 * i), __ldg(obs + 3 * i + 1), __ldg(obs + 3 * i + 2));
    double R[9];
#pragma unroll
    for (int k = 0; k < 9; k++) R[k] = __ldg(rowT + 9 * (size_t)i + k);
    pair_block(g, elem_src, o, R, j, blk);
  }
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) tile[3 * ti + a][3 * tj + b] = (OutT)blk[3 * a + b];
  __syncthreads();
  const int r3 = 3 * nr, n3 = 3 * n;
  for (int e = threadIdx.x; e < 3 * ATI * 3 * ATJ; e += blockDim.x) {
    int r = e / (3 * ATJ), c = e % (3 * ATJ);
    int gr = 3 * i0 + r, gc = 3 * j0 + c;
    if (gr < r3 && gc < n3) N[(size_t)gr * ld + gc] = tile[r][c];
  }
}

// Sources that are all tetrahedra in the vertex/edge form with one image
// each (a mesh without symmetries): the CTA's 32 source records (tensor
// record and image transform) are staged in shared memory once, instead of
// every pair walking elem_src -> poly_info -> tetidx -> record in global
// memory; the arithmetic and its order are pair_block's, so the blocks are
// the same to the bit.
constexpr int AT_U = TET_REC_TENSOR + 21;  // record, image transform (Minv, V, s M)
union AssembleTetSmem {
  double su[ATJ * AT_U];
  float t32[3 * ATI][3 * ATJ + 1];
  double t64[3 * ATI][3 * ATJ + 1];
};

template <typename OutT>
__global__ void __launch_bounds__(256, 3) assemble_tet_kernel(GeomView g, const int *__restrict__ elem_src,
                                                           const double *__restrict__ obs, const double *__restrict__ rowT,
                                                           int nr, int n, int ld, OutT *__restrict__ N)
{
  __shared__ AssembleTetSmem sm;
  __shared__ int s_rec[ATJ], s_trf[ATJ];
  const int tid = threadIdx.x;
  const int ti = tid / ATJ, tj = tid % ATJ;
  const int i0 = blockIdx.y * ATI, j0 = blockIdx.x * ATJ;
  if (tid < ATJ) {
    const int j = j0 + tid;
    int rec = 0, trf = 0;
    if (j < n) {
      const int idx = __ldg(elem_src + 2 * j + 1);
      rec = __ldg(g.tetidx + idx);
      trf = __ldg(g.poly_info + 4 * idx + 2);
    }
    s_rec[tid] = rec;
    s_trf[tid] = trf;
  }
  __syncthreads();
  for (int e = tid; e < ATJ * AT_U; e += blockDim.x) {
    const int k = e / AT_U, f = e - k * AT_U;
    double v = 0.0;
    if (j0 + k < n)
      v = f < TET_REC_TENSOR ? __ldg(g.tetrec + (size_t)s_rec[k] * TET_REC_TENSOR + f)
                             : __ldg(g.trf + (size_t)s_trf[k] * RADB200_TRF_STRIDE + (f - TET_REC_TENSOR));
    sm.su[e] = v;
  }
  __syncthreads();
  const int i = i0 + ti, j = j0 + tj;
  double blk[9];
#pragma unroll
  for (int k = 0; k < 9; k++) blk[k] = 0.0;
  if (i < nr && j < n) {
    const double *rec = sm.su + tj * AT_U, *Tr = rec + TET_REC_TENSOR;
    const double ox = __ldg(obs + 3 * i), oy = __ldg(obs + 3 * i + 1), oz = __ldg(obs + 3 * i + 2);
    const double dx = ox - Tr[9], dy = oy - Tr[10], dz = oz - Tr[11];
    const V3<double> q = mk3<double>(Tr[0] * dx + Tr[1] * dy + Tr[2] * dz, Tr[3] * dx + Tr[4] * dy + Tr[5] * dz,
                                     Tr[6] * dx + Tr[7] * dy + Tr[8] * dz);
    double Q[9], B[9];
    tet_fast<double, true, true>(rec, q, Q);
    const double *F = Tr + 12;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double f0 = F[3 * a], f1 = F[3 * a + 1], f2 = F[3 * a + 2];
#pragma unroll
      for (int b = 0; b < 3; b++) B[3 * a + b] = 0.0 + (f0 * Q[b] + f1 * Q[3 + b] + f2 * Q[6 + b]);
    }
    const double *R = rowT + 9 * (size_t)i;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double r0 = __ldg(R + 3 * a), r1 = __ldg(R + 3 * a + 1), r2 = __ldg(R + 3 * a + 2);
#pragma unroll
      for (int b = 0; b < 3; b++) blk[3 * a + b] = r0 * B[b] + r1 * B[3 + b] + r2 * B[6 + b];
    }
  }
  __syncthreads();  // every pair done with the staged records: the tile reuses them
  OutT(*tile)[3 * ATJ + 1] = reinterpret_cast<OutT(*)[3 * ATJ + 1]>(sizeof(OutT) == 4 ? (void *)sm.t32 : (void *)sm.t64);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) tile[3 * ti + a][3 * tj + b] = (OutT)blk[3 * a + b];
  __syncthreads();
  const int r3 = 3 * nr, n3 = 3 * n;
  for (int e = tid; e < 3 * ATI * 3 * ATJ; e += blockDim.x) {
    const int r = e / (3 * ATJ), c = e % (3 * ATJ);
    const int gr = 3 * i0 + r, gc = 3 * j0 + c;
    if (gr < r3 && gc < n3) N[(size_t)gr * ld + gc] = tile[r][c];
  }
}

int launch_assemble(const GeomView &g, const int *elem_src, const double *obs, const double *rowT, int nr, int n, int ld,
                    float *N32, double *N64, cudaStream_t st)
{
  if (g.fast && g.all_tets && g.tet_single) {
    dim3 grid((n + ATJ - 1) / ATJ, (nr + ATI - 1) / ATI);
    if (grid.y > 65535) { set_error("too many elements for one assembly grid"); return RADB200_E_ARG; }
    if (N64) {
      assemble_tet_kernel<double><<<grid, 256, 0, st>>>(g, elem_src, obs, rowT, nr, n, ld, N64);
      RB_TRY(check_launch("assemble_tet_kernel<double>"));
    }
    if (N32) {
      if (N64) RB_TRY(launch_round_f32(N64, N32, (size_t)3 * nr * ld, st));
      else {
        assemble_tet_kernel<float><<<grid, 256, 0, st>>>(g, elem_src, obs, rowT, nr, n, ld, N32);
        RB_TRY(check_launch("assemble_tet_kernel<float>"));
      }
    }
    return 0;
  }
  dim3 grid((n + ATJ - 1) / ATJ, (nr + ATI - 1) / ATI);
  if (grid.y > 65535) { set_error("too many elements for one assembly grid"); return RADB200_E_ARG; }
  if (N64) {
    assemble_kernel<double><<<grid, 256, 0, st>>>(g, elem_src, obs, rowT, nr, n, ld, N64);
    RB_TRY(check_launch("assemble_kernel<double>"));
  }
  if (N32) {
    if (N64) {
      // FP32 copy rounded from the FP64 matrix (one rounding, like the reference)
      size_t tot = (size_t)3 * nr * ld;
      RB_TRY(launch_round_f32(N64, N32, tot, st));
    } else {
      assemble_kernel<float><<<grid, 256, 0, st>>>(g, elem_src, obs, rowT, nr, n, ld, N32);
      RB_TRY(check_launch("assemble_kernel<float>"));
    }
  }
  return 0;
}

// FP64 residue of the near pairs of mixed storage: the block computed again
// in FP64 minus its stored FP32 rounding (read back, so the residue is exact
// whatever the compiler did with the first evaluation).
__global__ void __launch_bounds__(128) assemble_near_kernel(GeomView g, const int *__restrict__ elem_src,
                                                            const double *__restrict__ obs, const double *__restrict__ rowT,
                                                            int ld, const float *__restrict__ N32,
                                                            const int *__restrict__ row, const int *__restrict__ col,
                                                            int64_t nnz, double *__restrict__ D)
{
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const int i = row[k], j = col[k];
  V3<double> o = mk3<double>(__ldg(obs + 3 * i), __ldg(obs + 3 * i + 1), __ldg(obs + 3 * i + 2));
  double R[9], blk[9];
#pragma unroll
  for (int q = 0; q < 9; q++) R[q] = __ldg(rowT + 9 * (size_t)i + q);
  pair_block(g, elem_src, o, R, j, blk);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) D[9 * k + 3 * a + b] = blk[3 * a + b] - (double)N32[(size_t)(3 * i + a) * ld + 3 * j + b];
}

int launch_assemble_near(const GeomView &g, const int *elem_src, const double *obs, const double *rowT, int ld,
                         const float *N32, const int *row, const int *col, int64_t nnz, double *D, cudaStream_t st)
{
  if (nnz == 0) return 0;
  assemble_near_kernel<<<(unsigned)((nnz + 127) / 128), 128, 0, st>>>(g, elem_src, obs, rowT, ld, N32, row, col, nnz, D);
  return check_launch("assemble_near_kernel");
}

__global__ void round_f32_kernel(const double *__restrict__ a, float *__restrict__ b, size_t n)
{
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) b[i] = (float)a[i];
}

int launch_round_f32(const double *a, float *b, size_t n, cudaStream_t st)
{
  round_f32_kernel<<<148 * 8, 256, 0, st>>>(a, b, n);
  return check_launch("round_f32_kernel");
}

}  // namespace rb
