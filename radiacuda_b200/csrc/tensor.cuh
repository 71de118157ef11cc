// tensor.cuh -- 3x3 field-from-magnetization tensor of one source element.
//
// H(q) = Q(q) m for a uniformly magnetized cuboid (radrec.cpp:115-283) or
// polyhedron (face sum radvlpgn.cpp:441-505 with the face tensor
// radplnr2.cpp:367-375), q in the element's object frame.  Shared by the
// matrix assembly and the adjoint.
#pragma once
#include "internal.cuh"

namespace rb {

// cuboid only: Q at q (object frame) of rectangular record idx
__device__ __forceinline__ void cuboid_tensor(const GeomView &g, int idx, V3<double> q, double *Q)
{
  const double *r = g.rec + (size_t)idx * RADB200_REC_STRIDE;
  V3<double> qc = mk3<double>(q.x - __ldg(r + 0), q.y - __ldg(r + 1), q.z - __ldg(r + 2));
  V3<double> hd = mk3<double>(0.5 * __ldg(r + 3), 0.5 * __ldg(r + 4), 0.5 * __ldg(r + 5));
  V3<double> Tt, Ss;
  cuboid_TS<double>(qc, hd, g.g, Tt, Ss);
  Q[0] = Tt.x;  Q[1] = -Ss.z; Q[2] = -Ss.y;
  Q[3] = -Ss.z; Q[4] = Tt.y;  Q[5] = -Ss.x;
  Q[6] = -Ss.y; Q[7] = -Ss.x; Q[8] = Tt.z;
}

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
  // the reference's polygon face form uses this 15-digit pi (radplnr2.cpp:32)
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

// Is q (object frame) strictly inside the element?  Cuboid: |q - c| < w/2 per
// axis; polyhedron: below every face plane (faces are outward, face-local z).
__device__ __forceinline__ bool elem_inside(const GeomView &g, int kind, int idx, V3<double> q)
{
  if (kind == 0) {
    const double *r = g.rec + (size_t)idx * RADB200_REC_STRIDE;
    return fabs(q.x - __ldg(r + 0)) < 0.5 * __ldg(r + 3) && fabs(q.y - __ldg(r + 1)) < 0.5 * __ldg(r + 4) &&
           fabs(q.z - __ldg(r + 2)) < 0.5 * __ldg(r + 5);
  }
  int f0 = __ldg(g.poly_info + 4 * idx), nf = __ldg(g.poly_info + 4 * idx + 1);
  for (int fi = f0; fi < f0 + nf; fi++) {
    const double *R = g.face + (size_t)fi * RADB200_FACE_STRIDE;
    if (__ldg(R + 6) * q.x + __ldg(R + 7) * q.y + __ldg(R + 8) * q.z >= __ldg(R + 9)) return false;
  }
  return true;
}

}  // namespace rb
