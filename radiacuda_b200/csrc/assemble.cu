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
#include "internal.cuh"

namespace rb {

constexpr int ATI = 8, ATJ = 32;

__device__ __forceinline__ void elem_tensor(const GeomView &g, int kind, int idx, V3<double> q, double *Q)
{
  if (kind == 0) {
    const double *r = g.rec + (size_t)idx * RADB200_REC_STRIDE;
    V3<double> qc = mk3<double>(q.x - __ldg(r + 0), q.y - __ldg(r + 1), q.z - __ldg(r + 2));
    V3<double> hd = mk3<double>(0.5 * __ldg(r + 3), 0.5 * __ldg(r + 4), 0.5 * __ldg(r + 5));
    V3<double> Tt, Ss;
    cuboid_TS<double>(qc, hd, g.g, Tt, Ss);  // (q relative to the centre, FP64)
    Q[0] = Tt.x;  Q[1] = -Ss.z; Q[2] = -Ss.y;
    Q[3] = -Ss.z; Q[4] = Tt.y;  Q[5] = -Ss.x;
    Q[6] = -Ss.y; Q[7] = -Ss.x; Q[8] = Tt.z;
    return;
  }
  if (g.fast && __ldg(&g.tp.tinfo[idx].y) >= 0) {  // vertex/edge form
    int ti = __ldg(g.tetidx + idx);
    if (ti >= 0) tet_fast<double, true>(g.tetrec + (size_t)ti * TET_REC_TENSOR, q, Q);
    else poly_fast<double, true>(g.tp, idx, q, Q);
    return;
  }
  const double CH = 1.0 / (4.0 * 3.14159265358979);
  int f0 = __ldg(g.poly_info + 4 * idx), nf = __ldg(g.poly_info + 4 * idx + 1);
#pragma unroll
  for (int k = 0; k < 9; k++) Q[k] = 0.0;
  for (int fi = f0; fi < f0 + nf; fi++) {
    const double *R = g.face + (size_t)fi * RADB200_FACE_STRIDE;
    double r0 = __ldg(R + 0), r1 = __ldg(R + 1), r2 = __ldg(R + 2), r3 = __ldg(R + 3), r4 = __ldg(R + 4),
           r5 = __ldg(R + 5), r6 = __ldg(R + 6), r7 = __ldg(R + 7), r8 = __ldg(R + 8), cz = __ldg(R + 9);
    int v0 = __ldg(g.face_vtx + 2 * fi), nv = __ldg(g.face_vtx + 2 * fi + 1);
    const double *vt = g.vtx2d + 2 * (size_t)v0;
    double cx = 0, cy = 0;
    if (g.g.absr != 0.0 || g.g.relr != 0.0 || g.g.zeror != 0.0) {
      for (int k = 0; k < nv; k++) { cx += __ldg(vt + 2 * k); cy += __ldg(vt + 2 * k + 1); }
      cx /= nv; cy /= nv;
    }
    V3<double> pl = mk3<double>(r0 * q.x + r1 * q.y + r2 * q.z, r3 * q.x + r4 * q.y + r5 * q.z, r6 * q.x + r7 * q.y + r8 * q.z);
    double s0, s1, s2;
    polygon_S<double, double>(vt, nv, cz, cx, cy, pl, g.g, s0, s1, s2);
    // Q += (R^T (-C S)) n^T, n = row 2 of R
    double wx = -CH * (r0 * s0 + r3 * s1 + r6 * s2);
    double wy = -CH * (r1 * s0 + r4 * s1 + r7 * s2);
    double wz = -CH * (r2 * s0 + r5 * s1 + r8 * s2);
    Q[0] += wx * r6; Q[1] += wx * r7; Q[2] += wx * r8;
    Q[3] += wy * r6; Q[4] += wy * r7; Q[5] += wy * r8;
    Q[6] += wz * r6; Q[7] += wz * r7; Q[8] += wz * r8;
  }
}

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

template <typename OutT>
__global__ void __launch_bounds__(256) assemble_kernel(GeomView g, const int *__restrict__ elem_src,
                                                       const double *__restrict__ obs, const double *__restrict__ rowT,
                                                       int n, int ld, OutT *__restrict__ N)
{
  __shared__ OutT tile[3 * ATI][3 * ATJ + 1];
  int ti = threadIdx.x / ATJ, tj = threadIdx.x % ATJ;
  int i0 = blockIdx.y * ATI, j0 = blockIdx.x * ATJ;
  int i = i0 + ti, j = j0 + tj;
  double blk[9];
#pragma unroll
  for (int k = 0; k < 9; k++) blk[k] = 0.0;
  if (i < n && j < n) {
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
  int n3 = 3 * n;
  for (int e = threadIdx.x; e < 3 * ATI * 3 * ATJ; e += blockDim.x) {
    int r = e / (3 * ATJ), c = e % (3 * ATJ);
    int gr = 3 * i0 + r, gc = 3 * j0 + c;
    if (gr < n3 && gc < n3) N[(size_t)gr * ld + gc] = tile[r][c];
  }
}

int launch_assemble(const GeomView &g, const int *elem_src, const double *obs, const double *rowT, int n, int ld,
                    float *N32, double *N64, cudaStream_t st)
{
  dim3 grid((n + ATJ - 1) / ATJ, (n + ATI - 1) / ATI);
  if (grid.y > 65535) { set_error("too many elements for one assembly grid"); return RADB200_E_ARG; }
  if (N64) {
    assemble_kernel<double><<<grid, 256, 0, st>>>(g, elem_src, obs, rowT, n, ld, N64);
    RB_TRY(check_launch("assemble_kernel<double>"));
  }
  if (N32) {
    if (N64) {
      // FP32 copy rounded from the FP64 matrix (one rounding, like the reference)
      size_t tot = (size_t)3 * n * ld;
      RB_TRY(launch_round_f32(N64, N32, tot, st));
    } else {
      assemble_kernel<float><<<grid, 256, 0, st>>>(g, elem_src, obs, rowT, n, ld, N32);
      RB_TRY(check_launch("assemble_kernel<float>"));
    }
  }
  return 0;
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
