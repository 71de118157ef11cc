// field.cu -- B / H / M at observation points from all field sources.
//
// Replaces radGPU_FldKernelT + radGPU_FldRecMagKernel + their partial-sum
// reductions (reference radgpu_fld.cu:381-553, 788-909) and the host coil
// loop (radgpu_fld.cpp:542-617).  Design:
//   - one thread per observation point, FP64 accumulation in registers;
//   - every thread of a CTA walks the same (source, image) unit list, so the
//     source records are warp-uniform loads served by L1 broadcast -- no
//     shared-memory staging is needed because each record feeds hundreds of
//     transcendental operations;
//   - symmetry / orientation images are applied in-kernel (point mapped into
//     the source's own frame, field mapped back with s*M);
//   - coils (arc currents, current cuboids) and background fields run on the
//     device with the magnets;
//   - when there are too few points to fill the GPU, the unit list is split
//     over gridDim.y chunks whose partial sums land in a scratch buffer and
//     are added in a fixed order (bitwise reproducible).
#include "internal.cuh"

namespace rb {

// KIND: 0 cuboid, 1 polyhedron (face-by-face form), 2 polyhedron (vertex/edge
// form where available), 3 arc current, 4 background.  One kernel is compiled
// per kind so each gets the register budget of its own formula.
enum { UK_REC = 0, UK_POLY = 1, UK_POLY_FAST = 2, UK_ARC = 3, UK_BKG = 4, UK_TET = 5 };

template <typename T, int KIND>
__device__ __forceinline__ V3<double> eval_unit(const GeomView &g, int4 u, V3<double> P, int what)
{
  const double *Tr = g.trf + (size_t)u.z * RADB200_TRF_STRIDE;
  // point in the source's own frame: q = M^-1 (P - V)
  double dx = P.x - __ldg(Tr + 9), dy = P.y - __ldg(Tr + 10), dz = P.z - __ldg(Tr + 11);
  V3<double> q = mk3<double>(__ldg(Tr + 0) * dx + __ldg(Tr + 1) * dy + __ldg(Tr + 2) * dz,
                             __ldg(Tr + 3) * dx + __ldg(Tr + 4) * dy + __ldg(Tr + 5) * dz,
                             __ldg(Tr + 6) * dx + __ldg(Tr + 7) * dy + __ldg(Tr + 8) * dz);
  V3<double> f = mk3<double>(0, 0, 0);
  if (KIND == UK_REC) {
    const double *r = g.rec + (size_t)u.y * RADB200_REC_STRIDE;
    double jx = __ldg(r + 9), jy = __ldg(r + 10), jz = __ldg(r + 11);
    V3<double> qc = mk3<double>(q.x - __ldg(r + 0), q.y - __ldg(r + 1), q.z - __ldg(r + 2));
    V3<double> hd = mk3<double>(0.5 * __ldg(r + 3), 0.5 * __ldg(r + 4), 0.5 * __ldg(r + 5));
    if (jx != 0.0 || jy != 0.0 || jz != 0.0) {
      if (what != 2) f = cuboid_J(qc, hd, mk3<double>(jx, jy, jz), g.g);
    } else {
      double mx = __ldg(r + 6), my = __ldg(r + 7), mz = __ldg(r + 8);
      if (what == 2) {
        int in = (fabs(qc.x) < hd.x) && (fabs(qc.y) < hd.y) && (fabs(qc.z) < hd.z);
        if (in) f = mk3<double>(mx, my, mz);
      } else {
        // cuboids stay FP64 in every precision mode, as in the reference (its
        // cuboid kernel radgpu_fld.cu:788-882 has no FP32 variant)
        V3<double> Tt, Ss;
        int in = cuboid_TS<double>(qc, hd, g.g, Tt, Ss);
        double Tx = Tt.x, Ty = Tt.y, Tz = Tt.z, Sx = Ss.x, Sy = Ss.y, Sz = Ss.z;
        f = mk3<double>(Tx * mx - Sz * my - Sy * mz, -Sz * mx + Ty * my - Sx * mz, -Sy * mx - Sx * my + Tz * mz);
        if (what == 0 && in) { f.x += mx; f.y += my; f.z += mz; }
      }
    }
  } else if (KIND == UK_TET) {
    // every polyhedron is a tetrahedron: fixed-topology vertex/edge form only
    const double *pr = g.poly + (size_t)u.y * RADB200_POLY_STRIDE;
    double h[3];
    int in = tet_fast<T, false>(g.tetrec + (size_t)__ldg(g.tetidx + u.y) * TET_REC_FIELD, q, h);
    if (what == 2) f = in ? mk3<double>(__ldg(pr + 3), __ldg(pr + 4), __ldg(pr + 5)) : mk3<double>(0, 0, 0);
    else {
      f = mk3<double>(h[0], h[1], h[2]);
      if (what == 0 && in) { f.x += __ldg(pr + 3); f.y += __ldg(pr + 4); f.z += __ldg(pr + 5); }
    }
  } else if (KIND == UK_POLY_FAST && __ldg(&g.tp.tinfo[u.y].y) >= 0) {
    // vertex/edge form (formulas.cuh: tet_fast for tetrahedra, poly_fast otherwise)
    const double *pr = g.poly + (size_t)u.y * RADB200_POLY_STRIDE;
    double h[3];
    int ti = __ldg(g.tetidx + u.y);
    int in = (ti >= 0) ? tet_fast<T, false>(g.tetrec + (size_t)ti * TET_REC_FIELD, q, h) : poly_fast<T, false>(g.tp, u.y, q, h);
    if (what == 2) f = in ? mk3<double>(__ldg(pr + 3), __ldg(pr + 4), __ldg(pr + 5)) : mk3<double>(0, 0, 0);
    else {
      f = mk3<double>(h[0], h[1], h[2]);
      if (what == 0 && in) { f.x += __ldg(pr + 3); f.y += __ldg(pr + 4); f.z += __ldg(pr + 5); }
    }
  } else if (KIND == UK_POLY || KIND == UK_POLY_FAST) {
    const double *pr = g.poly + (size_t)u.y * RADB200_POLY_STRIDE;
    double mx = __ldg(pr + 3), my = __ldg(pr + 4), mz = __ldg(pr + 5);
    int f0 = __ldg(g.poly_info + 4 * u.y), nf = __ldg(g.poly_info + 4 * u.y + 1);
    // the reference's polygon face form uses this 15-digit pi (radplnr2.cpp:32)
    const double CH = 1.0 / (4.0 * 3.14159265358979);
    int inside = 1;
    double hx = 0, hy = 0, hz = 0;
    for (int fi = f0; fi < f0 + nf; fi++) {
      const double *R = g.face + (size_t)fi * RADB200_FACE_STRIDE;
      double r0 = __ldg(R + 0), r1 = __ldg(R + 1), r2 = __ldg(R + 2), r3 = __ldg(R + 3), r4 = __ldg(R + 4),
             r5 = __ldg(R + 5), r6 = __ldg(R + 6), r7 = __ldg(R + 7), r8 = __ldg(R + 8), cz = __ldg(R + 9);
      // local normal component of M (row 2 of R)
      double mloc = r6 * mx + r7 * my + r8 * mz;
      int v0 = __ldg(g.face_vtx + 2 * fi), nv = __ldg(g.face_vtx + 2 * fi + 1);
      const double *vt = g.vtx2d + 2 * (size_t)v0;
      double cx = 0, cy = 0;
      if (g.g.absr != 0.0 || g.g.relr != 0.0 || g.g.zeror != 0.0) {
        for (int k = 0; k < nv; k++) { cx += __ldg(vt + 2 * k); cy += __ldg(vt + 2 * k + 1); }
        cx /= nv; cy /= nv;
      }
      double plx = r0 * q.x + r1 * q.y + r2 * q.z, ply = r3 * q.x + r4 * q.y + r5 * q.z, plz = r6 * q.x + r7 * q.y + r8 * q.z;
      // the face-by-face form stays in FP64: its products of powers of the edge
      // slope overflow the FP32 range for near-vertical edges
      double s0, s1, s2;
      int in = polygon_S<double, double>(vt, nv, cz, cx, cy, mk3<double>(plx, ply, plz), g.g, s0, s1, s2);
      if (!in) inside = 0;
      if (what != 2) {
        double w = -CH * mloc;
        // H_obj += R^T (w S)
        hx += w * (r0 * s0 + r3 * s1 + r6 * s2);
        hy += w * (r1 * s0 + r4 * s1 + r7 * s2);
        hz += w * (r2 * s0 + r5 * s1 + r8 * s2);
      }
    }
    if (what == 2) f = inside ? mk3<double>(mx, my, mz) : mk3<double>(0, 0, 0);
    else {
      f = mk3<double>(hx, hy, hz);
      if (what == 0 && inside) { f.x += mx; f.y += my; f.z += mz; }
    }
  } else if (KIND == UK_ARC) {
    if (what != 2) f = arc_field(g.arc + (size_t)u.y * RADB200_ARC_STRIDE, q);
  } else {
    if (what != 2) {
      const double *b = g.bkg + 3 * (size_t)u.y;
      f = mk3<double>(__ldg(b), __ldg(b + 1), __ldg(b + 2));
    }
  }
  const double *F = Tr + 12;  // s*M
  return mk3<double>(__ldg(F + 0) * f.x + __ldg(F + 1) * f.y + __ldg(F + 2) * f.z,
                     __ldg(F + 3) * f.x + __ldg(F + 4) * f.y + __ldg(F + 5) * f.z,
                     __ldg(F + 6) * f.x + __ldg(F + 7) * f.y + __ldg(F + 8) * f.z);
}

// Units [ub, ue) of one kind; gridDim.y splits them into chunks.  With one
// chunk the result goes to out directly (accumulate: out += result), else to
// the chunk's slice of the partial buffer.
template <typename T, int KIND>
__global__ void __launch_bounds__(128) field_kernel(GeomView g, const double *__restrict__ pts, int64_t npts, int what,
                                                    double *__restrict__ out, int ub, int ue, int chunk, int accumulate)
{
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int u0 = ub + blockIdx.y * chunk, u1 = min(ue, u0 + chunk);
  bool active = i < npts;
  V3<double> P = mk3<double>(0, 0, 0);
  if (active) P = mk3<double>(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
  double ax = 0, ay = 0, az = 0;
  for (int u = u0; u < u1; u++) {
    int4 un = __ldg(g.units + u);
    V3<double> f = eval_unit<T, KIND>(g, un, P, what);
    ax += f.x; ay += f.y; az += f.z;
  }
  if (active) {
    double *o = out + ((size_t)blockIdx.y * npts + i) * 3;
    if (accumulate) { o[0] += ax; o[1] += ay; o[2] += az; }
    else { o[0] = ax; o[1] = ay; o[2] = az; }
  }
}

// out[i] (=|+=) sum_c partial[c][i], fixed order c = 0..nc-1
__global__ void chunk_reduce_kernel(const double *__restrict__ part, int nc, int64_t n3, double *__restrict__ out, int accumulate)
{
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  double s = accumulate ? out[i] : 0.0;
  for (int c = 0; c < nc; c++) s += part[(size_t)c * n3 + i];
  out[i] = s;
}

// All polyhedra are tetrahedra (fixed-topology vertex/edge form).  A block
// of 128 threads takes 128 PPT points (PPT per thread: with 2, two
// independent evaluation chains to interleave) and walks its unit range in tiles of 32
// units whose records -- tetrahedron record, image transform, magnetization
// -- it first stages in shared memory, so the per-pair reads are
// shared-memory broadcasts.
constexpr int TET_TILE = 32;
constexpr int TET_U = TET_REC_FIELD + 21 + 3;  // record, Minv V sM (21), M (3)
constexpr int TET_UF = 18;                     // float copies: edge lengths (6), face normals (12)

template <typename T>
__device__ __forceinline__ void tet_unit(const double *su, const float *suf, V3<double> P, int what, double *acc)
{
  const double *Tr = su + TET_REC_FIELD, *M = Tr + 21;
  double dx = P.x - Tr[9], dy = P.y - Tr[10], dz = P.z - Tr[11];
  V3<double> q = mk3<double>(Tr[0] * dx + Tr[1] * dy + Tr[2] * dz, Tr[3] * dx + Tr[4] * dy + Tr[5] * dz,
                             Tr[6] * dx + Tr[7] * dy + Tr[8] * dz);
  double h[3];
  int in = tet_fast<T, false, true>(su, q, h, suf);
  V3<double> f;
  if (what == 2) f = in ? mk3<double>(M[0], M[1], M[2]) : mk3<double>(0, 0, 0);
  else {
    f = mk3<double>(h[0], h[1], h[2]);
    if (what == 0 && in) { f.x += M[0]; f.y += M[1]; f.z += M[2]; }
  }
  const double *F = Tr + 12;
  acc[0] += F[0] * f.x + F[1] * f.y + F[2] * f.z;
  acc[1] += F[3] * f.x + F[4] * f.y + F[5] * f.z;
  acc[2] += F[6] * f.x + F[7] * f.y + F[8] * f.z;
}

// PPT points per thread; TPI tetrahedra per iteration of the unit loop (two
// independent evaluation chains interleave when TPI == 2)
template <typename T, int PPT, int TPI = 1>
__global__ void __launch_bounds__(128) field_tet_kernel(GeomView g, const double *__restrict__ pts, int64_t npts, int what,
                                                        double *__restrict__ out, int ub, int ue, int chunk, int accumulate)
{
  __shared__ double su[TET_TILE * TET_U];
  __shared__ float suf[TET_TILE * TET_UF];
  const int tid = threadIdx.x;
  const int64_t i0 = (int64_t)blockIdx.x * (128 * PPT) + tid, i1 = PPT == 2 ? i0 + 128 : npts;
  const int u0 = ub + blockIdx.y * chunk, u1 = min(ue, u0 + chunk);
  V3<double> P0 = mk3<double>(0, 0, 0), P1 = P0;
  if (i0 < npts) P0 = mk3<double>(pts[3 * i0], pts[3 * i0 + 1], pts[3 * i0 + 2]);
  if (i1 < npts) P1 = mk3<double>(pts[3 * i1], pts[3 * i1 + 1], pts[3 * i1 + 2]);
  double a0[3] = {0, 0, 0}, a1[3] = {0, 0, 0};
  for (int base = u0; base < u1; base += TET_TILE) {
    const int cnt = min(TET_TILE, u1 - base);
    __syncthreads();
    for (int e = tid; e < cnt * TET_U; e += 128) {
      const int k = e / TET_U, f = e - k * TET_U;
      const int4 un = __ldg(g.units + base + k);  // {kind, polyhedron, transform, 0}
      double v;
      if (f < TET_REC_FIELD) v = __ldg(g.tetrec + (size_t)__ldg(g.tetidx + un.y) * TET_REC_FIELD + f);
      else if (f < TET_REC_FIELD + 21) v = __ldg(g.trf + (size_t)un.z * RADB200_TRF_STRIDE + (f - TET_REC_FIELD));
      else v = __ldg(g.poly + (size_t)un.y * RADB200_POLY_STRIDE + 3 + (f - TET_REC_FIELD - 21));
      su[e] = v;
    }
    if (sizeof(T) == 4)
      for (int e = tid; e < cnt * TET_UF; e += 128) {
        const int k = e / TET_UF, f = e - k * TET_UF;
        const int4 un = __ldg(g.units + base + k);
        suf[e] = (float)__ldg(g.tetrec + (size_t)__ldg(g.tetidx + un.y) * TET_REC_FIELD + 12 + f);  // rec + 12: lengths, then normals
      }
    __syncthreads();
    if (TPI == 2) {
      int k = 0;
      for (; k + 1 < cnt; k += 2) {
        double b0[3] = {0, 0, 0};
        tet_unit<T>(su + k * TET_U, suf + k * TET_UF, P0, what, a0);
        tet_unit<T>(su + (k + 1) * TET_U, suf + (k + 1) * TET_UF, P0, what, b0);
        a0[0] += b0[0]; a0[1] += b0[1]; a0[2] += b0[2];
      }
      if (k < cnt) tet_unit<T>(su + k * TET_U, suf + k * TET_UF, P0, what, a0);
    } else {
      for (int k = 0; k < cnt; k++) {
        tet_unit<T>(su + k * TET_U, suf + k * TET_UF, P0, what, a0);
        if (PPT == 2) tet_unit<T>(su + k * TET_U, suf + k * TET_UF, P1, what, a1);
      }
    }
  }
  if (i0 < npts) {
    double *o = out + ((size_t)blockIdx.y * npts + i0) * 3;
    if (accumulate) { o[0] += a0[0]; o[1] += a0[1]; o[2] += a0[2]; }
    else { o[0] = a0[0]; o[1] = a0[1]; o[2] = a0[2]; }
  }
  if (i1 < npts) {
    double *o = out + ((size_t)blockIdx.y * npts + i1) * 3;
    if (accumulate) { o[0] += a1[0]; o[1] += a1[1]; o[2] += a1[2]; }
    else { o[0] = a1[0]; o[1] = a1[1]; o[2] = a1[2]; }
  }
}

template <typename T, int PPT, int TPI = 1>
static int launch_tet_ppt(const GeomView &g, const double *d_pts, int64_t npts, int what, double *d_out, int ub, int ue,
                          int accumulate, DBuf &scratch, cudaStream_t st)
{
  int64_t nblk = (npts + 128 * PPT - 1) / (128 * PPT);
  int nu = ue - ub;
  int nchunk = 1;
  const int64_t target = 148 * 6;
  if (nblk < target) nchunk = (int)((target + nblk - 1) / nblk);
  if (nchunk > nu) nchunk = nu;
  if (nchunk > 65535) nchunk = 65535;
  int chunk = (nu + nchunk - 1) / nchunk;
  nchunk = (nu + chunk - 1) / chunk;
  dim3 grid((unsigned)nblk, (unsigned)nchunk);
  if (nchunk == 1) {
    field_tet_kernel<T, PPT, TPI><<<grid, 128, 0, st>>>(g, d_pts, npts, what, d_out, ub, ue, chunk, accumulate);
    return check_launch("field_tet_kernel");
  }
  RB_TRY(scratch.alloc((size_t)nchunk * npts * 3 * sizeof(double)));
  field_tet_kernel<T, PPT, TPI><<<grid, 128, 0, st>>>(g, d_pts, npts, what, scratch.as<double>(), ub, ue, chunk, 0);
  RB_TRY(check_launch("field_tet_kernel"));
  int64_t n3 = npts * 3;
  chunk_reduce_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(scratch.as<double>(), nchunk, n3, d_out, accumulate);
  return check_launch("chunk_reduce_kernel");
}

// points per thread: 1 (more resident warps) or 2 (two interleaved chains);
// RADB200_TET_PPT overrides the default for tuning
template <typename T>
static int launch_tet(const GeomView &g, const double *d_pts, int64_t npts, int what, double *d_out, int ub, int ue,
                      int accumulate, DBuf &scratch, cudaStream_t st)
{
  static int ppt = 0;
  if (!ppt) {
    const char *e = getenv("RADB200_TET_PPT");
    ppt = (e && atoi(e) == 2) ? 2 : (e && atoi(e) == 3) ? 3 : 1;
  }
  if (ppt == 2) return launch_tet_ppt<T, 2>(g, d_pts, npts, what, d_out, ub, ue, accumulate, scratch, st);
  // RADB200_TET_PPT=3: one point, two tetrahedra interleaved per iteration
  if (ppt == 3) return launch_tet_ppt<T, 1, 2>(g, d_pts, npts, what, d_out, ub, ue, accumulate, scratch, st);
  return launch_tet_ppt<T, 1>(g, d_pts, npts, what, d_out, ub, ue, accumulate, scratch, st);
}

template <typename T, int KIND>
static int launch_kind(const GeomView &g, const double *d_pts, int64_t npts, int what, double *d_out, int ub, int ue,
                       int accumulate, DBuf &scratch, cudaStream_t st)
{
  const int TPB = 128;
  int64_t nblk = (npts + TPB - 1) / TPB;
  int nu = ue - ub;
  // split the unit range when the points alone give fewer than ~8 CTAs per SM
  int nchunk = 1;
  const int64_t target = 148 * 8;
  if (nblk < target) nchunk = (int)((target + nblk - 1) / nblk);
  if (nchunk > nu) nchunk = nu;
  if (nchunk > 65535) nchunk = 65535;
  int chunk = (nu + nchunk - 1) / nchunk;
  nchunk = (nu + chunk - 1) / chunk;
  dim3 grid((unsigned)nblk, (unsigned)nchunk);
  if (nchunk == 1) {
    field_kernel<T, KIND><<<grid, TPB, 0, st>>>(g, d_pts, npts, what, d_out, ub, ue, chunk, accumulate);
    return check_launch("field_kernel");
  }
  RB_TRY(scratch.alloc((size_t)nchunk * npts * 3 * sizeof(double)));
  field_kernel<T, KIND><<<grid, TPB, 0, st>>>(g, d_pts, npts, what, scratch.as<double>(), ub, ue, chunk, 0);
  RB_TRY(check_launch("field_kernel"));
  int64_t n3 = npts * 3;
  chunk_reduce_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(scratch.as<double>(), nchunk, n3, d_out, accumulate);
  return check_launch("chunk_reduce_kernel");
}

// RADB200_MESH_FORM=0 evaluates all-tetrahedron models one tetrahedron at a
// time instead of by their unique edges and faces (A/B comparisons)
static bool mesh_form_enabled()
{
  static int on = -1;
  if (on < 0) {
    const char *e = getenv("RADB200_MESH_FORM");
    on = (e && atoi(e) == 0) ? 0 : 1;
  }
  return on == 1;
}

int launch_field(const GeomView &g, const double *d_pts, int64_t npts, int what, int precision, double *d_out,
                 DBuf &scratch, cudaStream_t st)
{
  if (npts <= 0) return 0;
  if ((npts + 127) / 128 > INT32_MAX) { set_error("too many points"); return RADB200_E_ARG; }
  if (g.n_units == 0) {
    RB_CUDA(cudaMemsetAsync(d_out, 0, (size_t)npts * 3 * sizeof(double), st));
    return 0;
  }
  // units are ordered by kind (cuboids, polyhedra, arcs, backgrounds): one launch per kind present
  int acc = 0;
  for (int kind = 0; kind < 4; kind++) {
    int ub = g.ustart[kind], ue = g.ustart[kind + 1];
    if (ue <= ub) continue;
    int rc;
    if (kind == 0)
      rc = launch_kind<double, UK_REC>(g, d_pts, npts, what, d_out, ub, ue, acc, scratch, st);
    // the mesh form in FP64 only: with FP32 terms its largest per-point B
    // error on the 20,000-tetrahedron model was 2.1e-6 against 7.6e-7 for the
    // tetrahedra one by one, at a 1.25x speed-up (1.42x in FP64)
    else if (kind == 1 && g.fast && g.all_tets && g.mesh.n_tiles > 0 && what != 2 && precision != 1 &&
             mesh_form_enabled())
      rc = launch_mesh_field(g, d_pts, npts, what, precision, d_out, acc, scratch, st);
    else if (kind == 1 && g.fast && g.all_tets)
      rc = (precision == 1) ? launch_tet<float>(g, d_pts, npts, what, d_out, ub, ue, acc, scratch, st)
                            : launch_tet<double>(g, d_pts, npts, what, d_out, ub, ue, acc, scratch, st);
    else if (kind == 1 && g.fast)
      rc = (precision == 1) ? launch_kind<float, UK_POLY_FAST>(g, d_pts, npts, what, d_out, ub, ue, acc, scratch, st)
                            : launch_kind<double, UK_POLY_FAST>(g, d_pts, npts, what, d_out, ub, ue, acc, scratch, st);
    else if (kind == 1)
      rc = launch_kind<double, UK_POLY>(g, d_pts, npts, what, d_out, ub, ue, acc, scratch, st);
    else if (kind == 2)
      rc = launch_kind<double, UK_ARC>(g, d_pts, npts, what, d_out, ub, ue, acc, scratch, st);
    else
      rc = launch_kind<double, UK_BKG>(g, d_pts, npts, what, d_out, ub, ue, acc, scratch, st);
    RB_TRY(rc);
    acc = 1;
  }
  return 0;
}

// out_i = rowT_i * in_i  (3x3 per element)
__global__ void rowtrans_kernel(const double *__restrict__ rowT, const double *__restrict__ in, double *__restrict__ out, int n)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *R = rowT + 9 * (size_t)i;
  double x = in[3 * i], y = in[3 * i + 1], z = in[3 * i + 2];
  out[3 * i] = R[0] * x + R[1] * y + R[2] * z;
  out[3 * i + 1] = R[3] * x + R[4] * y + R[5] * z;
  out[3 * i + 2] = R[6] * x + R[7] * y + R[8] * z;
}

int launch_rowtrans_vec(const double *rowT, const double *in, double *out, int n, cudaStream_t st)
{
  if (n <= 0) return 0;
  rowtrans_kernel<<<(n + 127) / 128, 128, 0, st>>>(rowT, in, out, n);
  return check_launch("rowtrans_kernel");
}

// ---------------------------------------------------------------------------
// Relativistic electron trajectories (FldPtcTrj).  The reference integrates
// x(y), x'(y), z(y), z'(y) with the field of the whole source evaluated at
// every Runge-Kutta stage (radTPrtclTrj::TrjEqs, cpp/src/core/radptrj.h:91-105;
// RungeKutta4 / Tabulation / RungeKuttaStep5 / AutoPropagate,
// radptrj.cpp:94-240).  The stages of one trajectory are a dependent chain,
// so one CTA carries one trajectory: at every stage its threads split the
// (source, image) units, the partial fields are reduced in shared memory, and
// every thread then advances an identical copy of the integrator state, so
// the control flow (the step-size control included) stays uniform.  Many
// trajectories run as many CTAs.
// ---------------------------------------------------------------------------
constexpr int TRJ_THREADS = 256;

struct TrjArgs {
  double y0, step, ctm;  // start, tabulation step (mm), charge / momentum (1 / (T mm))
  int np, adaptive, max_steps;
  long long max_evals;   // field evaluations allowed per trajectory (bounds the kernel's run time)
  double prec[4], eps_tol;
};

// B at P from every unit, reduced over the block; every thread gets the sum
__device__ V3<double> trj_block_field(const GeomView &g, V3<double> P, double *red)
{
  double ax = 0, ay = 0, az = 0;
  for (int u = g.ustart[0] + threadIdx.x; u < g.ustart[1]; u += blockDim.x) {
    V3<double> f = eval_unit<double, UK_REC>(g, __ldg(g.units + u), P, 0);
    ax += f.x; ay += f.y; az += f.z;
  }
  for (int u = g.ustart[1] + threadIdx.x; u < g.ustart[2]; u += blockDim.x) {
    V3<double> f = eval_unit<double, UK_POLY>(g, __ldg(g.units + u), P, 0);
    ax += f.x; ay += f.y; az += f.z;
  }
  for (int u = g.ustart[2] + threadIdx.x; u < g.ustart[3]; u += blockDim.x) {
    V3<double> f = eval_unit<double, UK_ARC>(g, __ldg(g.units + u), P, 0);
    ax += f.x; ay += f.y; az += f.z;
  }
  for (int u = g.ustart[3] + threadIdx.x; u < g.ustart[4]; u += blockDim.x) {
    V3<double> f = eval_unit<double, UK_BKG>(g, __ldg(g.units + u), P, 0);
    ax += f.x; ay += f.y; az += f.z;
  }
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_down_sync(0xffffffffu, ax, o);
    ay += __shfl_down_sync(0xffffffffu, ay, o);
    az += __shfl_down_sync(0xffffffffu, az, o);
  }
  int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();  // the previous stage's readers are done with red
  if ((threadIdx.x & 31) == 0) { red[3 * w] = ax; red[3 * w + 1] = ay; red[3 * w + 2] = az; }
  __syncthreads();
  double bx = 0, by = 0, bz = 0;
  for (int k = 0; k < nw; k++) { bx += red[3 * k]; by += red[3 * k + 1]; bz += red[3 * k + 2]; }
  return mk3<double>(bx, by, bz);
}

// dF/dy for F = (x, x', z, z') at longitudinal position s
__device__ void trj_eqs(const GeomView &g, const TrjArgs &a, double s, const double *F, double *dF, double *red,
                        long long &ne)
{
  ne++;
  double xd = F[1], zd = F[3];
  double xdxd = xd * xd, zdzd = zd * zd, xdzd = xd * zd;
  double buf = a.ctm * sqrt(1.0 + xdxd + zdzd);
  V3<double> B = trj_block_field(g, mk3<double>(F[0], s, F[2]), red);
  dF[0] = xd;
  dF[1] = -buf * (zd * B.y - (1.0 + xdxd) * B.z + xdzd * B.x);
  dF[2] = zd;
  dF[3] = buf * (xd * B.y - (1.0 + zdzd) * B.x + xdzd * B.z);
}

// classical fourth-order step of size h from (x, y) with slope dydx
__device__ void trj_rk4(const GeomView &g, const TrjArgs &a, const double *y, const double *dydx, double x, double h,
                        double *yout, double *red, long long &ne)
{
  double hh = 0.5 * h, h6 = h / 6.0, xh = x + hh;
  double yt[4], dyt[4], dym[4];
  for (int i = 0; i < 4; i++) yt[i] = y[i] + hh * dydx[i];
  trj_eqs(g, a, xh, yt, dyt, red, ne);
  for (int i = 0; i < 4; i++) yt[i] = y[i] + hh * dyt[i];
  trj_eqs(g, a, xh, yt, dym, red, ne);
  for (int i = 0; i < 4; i++) {
    yt[i] = y[i] + h * dym[i];
    dym[i] += dyt[i];
  }
  trj_eqs(g, a, x + h, yt, dyt, red, ne);
  for (int i = 0; i < 4; i++) yout[i] = y[i] + h6 * (dydx[i] + dyt[i] + 2.0 * dym[i]);
}

// step-doubling control: one step of size h against two of h/2, accepted when
// the difference over prec, over eps_tol, is at most 1; 0 ok, 1 step too small,
// 2 evaluation budget spent, 3 no acceptable step within the shrink limit
__device__ int trj_step5(const GeomView &g, const TrjArgs &a, double *y, double *dydx, double *x, double htry,
                         double *hdid, double *hnext, double *red, long long &ne)
{
  const double PGROW = -0.2, PSHRNK = -0.25, FCOR = 1.0 / 15.0, SAFETY = 0.9, ERRCON = 6.0e-04;
  double xsav = *x, h = htry, ysav[4], dysav[4], ytemp[4];
  for (int i = 0; i < 4; i++) { ysav[i] = y[i]; dysav[i] = dydx[i]; }
  for (int it = 0; it < 200; it++) {
    if (ne > a.max_evals) return 2;
    double hh = 0.5 * h;
    trj_rk4(g, a, ysav, dysav, xsav, hh, ytemp, red, ne);
    *x = xsav + hh;
    trj_eqs(g, a, *x, ytemp, dydx, red, ne);
    trj_rk4(g, a, ytemp, dydx, *x, hh, y, red, ne);
    *x = xsav + h;
    if (*x == xsav) return 1;
    trj_rk4(g, a, ysav, dysav, xsav, h, ytemp, red, ne);
    double errmax = 0.0;
    for (int i = 0; i < 4; i++) {
      ytemp[i] = y[i] - ytemp[i];
      double t = fabs(ytemp[i] / a.prec[i]);
      if (errmax < t) errmax = t;
    }
    errmax /= a.eps_tol;
    if (errmax <= 1.0) {
      *hdid = h;
      *hnext = (errmax > ERRCON ? SAFETY * h * exp(PGROW * log(errmax)) : 4.0 * h);
      for (int i = 0; i < 4; i++) y[i] += ytemp[i] * FCOR;
      return 0;
    }
    if (!(errmax < 1e300)) return 3;  // non-finite error: no step will be accepted
    h *= SAFETY * exp(PSHRNK * log(errmax));
  }
  return 3;
}

// adaptive propagation of y from x1 to x2; 0 ok, 1 step too small, 2 step limit, 3 failure
__device__ int trj_propagate(const GeomView &g, const TrjArgs &a, double *ystart, double x1, double x2, double h1,
                             double hmin, double *red, long long &ne)
{
  double x = x1, h = (x2 > x1) ? fabs(h1) : -fabs(h1), y[4], dydx[4], hdid, hnext;
  for (int i = 0; i < 4; i++) y[i] = ystart[i];
  for (int n = 1; n <= a.max_steps; n++) {
    trj_eqs(g, a, x, y, dydx, red, ne);
    if ((x + h - x2) * (x + h - x1) > 0.0) h = x2 - x;
    int rc = trj_step5(g, a, y, dydx, &x, h, &hdid, &hnext, red, ne);
    if (rc) return rc;
    if ((x - x2) * (x2 - x1) >= 0.0) {
      for (int i = 0; i < 4; i++) ystart[i] = y[i];
      return 0;
    }
    if (fabs(hnext) <= hmin) return 1;
    h = hnext;
  }
  return 2;
}

// out[(b * np + i) * 5 + (y, x, x', z, z')]; status[b]: 0 ok, else the failure code
__global__ void __launch_bounds__(TRJ_THREADS) trajectory_kernel(GeomView g, TrjArgs a, const double *__restrict__ init,
                                                                double *__restrict__ out, int *__restrict__ status)
{
  __shared__ double red[3 * (TRJ_THREADS / 32)];
  int b = blockIdx.x;
  double Y[4], dY[4];
  for (int k = 0; k < 4; k++) Y[k] = init[4 * b + k];
  double x = a.y0, hmin = 1e-10 * a.step;
  int rc = 0;
  long long ne = 0;
  for (int i = 0; i < a.np; i++) {
    if (!a.adaptive) trj_eqs(g, a, x, Y, dY, red, ne);
    if (threadIdx.x == 0) {
      double *o = out + ((size_t)b * a.np + i) * 5;
      o[0] = x;
      for (int k = 0; k < 4; k++) o[1 + k] = Y[k];
    }
    if (i == a.np - 1 || rc) break;
    double x1 = x + a.step;
    if (a.adaptive) rc = trj_propagate(g, a, Y, x, x1, a.step, hmin, red, ne);
    else trj_rk4(g, a, Y, dY, x, a.step, Y, red, ne);
    x = x1;
    if (rc) {
      // rows after a failed interval repeat the last good state's position with NaN
      for (int j = i + 1; j < a.np && threadIdx.x == 0; j++) {
        double *o = out + ((size_t)b * a.np + j) * 5;
        for (int k = 0; k < 5; k++) o[k] = __longlong_as_double(0x7ff8000000000000LL);
      }
      break;
    }
  }
  if (threadIdx.x == 0) status[b] = rc;
}

int launch_trajectories(const GeomView &g, double energy_gev, const double *d_init, int n_traj, double y0, double y1,
                        int np, const double *prec, double *d_out, int *d_status, cudaStream_t st)
{
  if (n_traj <= 0) return 0;
  TrjArgs a;
  a.y0 = y0;
  a.np = np;
  a.step = (np > 1) ? (y1 - y0) / (double)(np - 1) : 0.0;
  a.ctm = -2.99792458e+05 / (1.e+09 * energy_gev);  // electron charge over momentum
  a.adaptive = prec != nullptr;
  a.max_steps = 5000;
  a.max_evals = 40LL * np + 40000;
  a.eps_tol = 1.0;
  for (int k = 0; k < 4; k++) a.prec[k] = prec ? (prec[k] == 0.0 ? 1e23 : prec[k]) : 1.0;
  trajectory_kernel<<<n_traj, TRJ_THREADS, 0, st>>>(g, a, d_init, d_out, d_status);
  return check_launch("trajectory_kernel");
}

}  // namespace rb
