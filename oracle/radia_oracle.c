/*
 * radia_oracle.c -- CPU restatement of the Radia relaxation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only the tests, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this code, and only as the checker.
 * The product (radiacuda_b200) never links, imports or calls it.
 *
 * It restates, in plain C and in FP64 throughout, the reference CPU
 * implementation of:
 *   - the cuboid field / demagnetization tensor   radTRecMag::B_comp,
 *     cpp/src/core/radrec.cpp:49-315 (TransAtans: radg3d.h:938-946)
 *   - the planar polygon face integrals           radTPolygon::B_comp,
 *     cpp/src/core/radplnr2.cpp:29-388 (direct atan2 accumulation, :309-318)
 *   - the polyhedron sum over faces               radTPolyhedron::B_comp_frM,
 *     cpp/src/core/radvlpgn.cpp:441-505
 *   - the arc-current field (trapezoid in phi)    radTArcCur::B_compWithTrapeth,
 *     cpp/src/core/radarccu.cpp:30-236
 *   - image summation of the object tree          radTg3d::NestedFor_B,
 *     cpp/src/core/radg3d.cpp:58-120
 *   - interaction-matrix assembly                 radintrc.cpp:831-877
 *   - external field at element centres           radintrc.cpp:1208-1234
 *   - material laws                               radmater.h:164-600,
 *                                                 radmater.cpp:72-306
 *   - relaxation method 4 (Gauss-Seidel)          radrlmet.cpp:496-587,772-829
 * over the flat geometry arrays of include/radb200.h.  Parity of this file
 * with the reference itself is pinned by tests against the compiled
 * reference module (oracle/_ref) and the committed golden vectors.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/radb200.h"

#define ORC_API __attribute__((visibility("default")))

typedef struct { double x, y, z; } v3;
static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mulm(const double *M, v3 a)
{
  return mk(M[0] * a.x + M[1] * a.y + M[2] * a.z, M[3] * a.x + M[4] * a.y + M[5] * a.z,
            M[6] * a.x + M[7] * a.y + M[8] * a.z);
}
static inline v3 mulmt(const double *M, v3 a)
{
  return mk(M[0] * a.x + M[3] * a.y + M[6] * a.z, M[1] * a.x + M[4] * a.y + M[7] * a.z,
            M[2] * a.x + M[5] * a.y + M[8] * a.z);
}
static inline double dabs(double x) { return x < 0. ? -x : x; }
static inline double sgn(double x) { return x < 0. ? -1. : 1.; }

/* radTConvergRepair::AbsRandMagnitude, radcnvrg.h:85-91 */
typedef struct { double absr, relr, zeror; } guard_t;
static double abs_rand_mag(const guard_t *g, double A)
{
  if (g->absr == 0. && g->relr == 0. && g->zeror == 0.) return 0.;
  double absfromrel = g->relr * A;
  double absmax = (absfromrel < g->absr) ? g->absr : absfromrel;
  return (A != 0.) ? absmax : ((absmax < g->zeror) ? g->zeror : absmax);
}

/* radTg3d::TransAtans, radg3d.h:938-946 */
static double trans_atans(double x, double y, double *pimult)
{
  double buf = 1. - x * y;
  if (buf == 0.) buf = 1.e-50;
  *pimult = ((buf > 0) ? 0. : 1.) * ((x < 0) ? -1. : 1.);
  return (x + y) / buf;
}

/* ------------------------------------------------------------------------
 * Cuboid.  With mode 0 returns the 3x3 tensor Q (H = Q M) of a cuboid of
 * dims d centred at c, at point p (radrec.cpp:115-283, PreRelax branch).
 * With mode 1 (current density J != 0) adds the field of J to *Bj
 * (radrec.cpp:183-281, J branch).  Returns 1 when p is strictly inside.   */
static int recmag_core(v3 c, v3 d, v3 p, const guard_t *g, double *Q, v3 J, v3 *Bj)
{
  const double Pi = 3.141592653589793238;
  v3 pc = sub(p, c);
  v3 hd = mk(0.5 * d.x, 0.5 * d.y, 0.5 * d.z);
  double bx[2], by[2], bz[2];
  for (int ii = 0; ii <= 1; ii++) {
    int eps = ii * 2 - 1;
    bx[ii] = -pc.x + eps * hd.x;
    by[ii] = -pc.y + eps * hd.y;
    bz[ii] = -pc.z + eps * hd.z;
    if (bx[ii] == 0.) bx[ii] = abs_rand_mag(g, hd.x);
    if (by[ii] == 0.) by[ii] = abs_rand_mag(g, hd.y);
    if (bz[ii] == 0.) bz[ii] = abs_rand_mag(g, hd.z);
  }
  double x0 = bx[0], x1 = bx[1], y0 = by[0], y1 = by[1], z0 = bz[0], z1 = bz[1];
  int inside = (x0 * x1 < 0) && (y0 * y1 < 0) && (z0 * z1 < 0);
  double x0e2 = x0 * x0, x1e2 = x1 * x1, y0e2 = y0 * y0, y1e2 = y1 * y1, z0e2 = z0 * z0, z1e2 = z1 * z1;
  double D000 = sqrt(x0e2 + y0e2 + z0e2), D100 = sqrt(x1e2 + y0e2 + z0e2);
  double D010 = sqrt(x0e2 + y1e2 + z0e2), D110 = sqrt(x1e2 + y1e2 + z0e2);
  double D001 = sqrt(x0e2 + y0e2 + z1e2), D101 = sqrt(x1e2 + y0e2 + z1e2);
  double D011 = sqrt(x0e2 + y1e2 + z1e2), D111 = sqrt(x1e2 + y1e2 + z1e2);

  double p1, p2, p3, a1, a2;
  v3 T0, T1;
  a1 = trans_atans(y0 * z0 / (x0 * D000), -y0 * z1 / (x0 * D001), &p1);
  a2 = trans_atans(-y1 * z0 / (x0 * D010), y1 * z1 / (x0 * D011), &p2);
  T0.x = atan(trans_atans(a1, a2, &p3)) + Pi * (p1 + p2 + p3);
  a1 = trans_atans(-y0 * z0 / (x1 * D100), y0 * z1 / (x1 * D101), &p1);
  a2 = trans_atans(y1 * z0 / (x1 * D110), -y1 * z1 / (x1 * D111), &p2);
  T1.x = atan(trans_atans(a1, a2, &p3)) + Pi * (p1 + p2 + p3);
  a1 = trans_atans(x0 * z0 / (y0 * D000), -x0 * z1 / (y0 * D001), &p1);
  a2 = trans_atans(-x1 * z0 / (y0 * D100), x1 * z1 / (y0 * D101), &p2);
  T0.y = atan(trans_atans(a1, a2, &p3)) + Pi * (p1 + p2 + p3);
  a1 = trans_atans(-x0 * z0 / (y1 * D010), x0 * z1 / (y1 * D011), &p1);
  a2 = trans_atans(x1 * z0 / (y1 * D110), -x1 * z1 / (y1 * D111), &p2);
  T1.y = atan(trans_atans(a1, a2, &p3)) + Pi * (p1 + p2 + p3);
  a1 = trans_atans(x0 * y0 / (z0 * D000), -x1 * y0 / (z0 * D100), &p1);
  a2 = trans_atans(-x0 * y1 / (z0 * D010), x1 * y1 / (z0 * D110), &p2);
  T0.z = atan(trans_atans(a1, a2, &p3)) + Pi * (p1 + p2 + p3);
  a1 = trans_atans(-x0 * y0 / (z1 * D001), x1 * y0 / (z1 * D101), &p1);
  a2 = trans_atans(x0 * y1 / (z1 * D011), -x1 * y1 / (z1 * D111), &p2);
  T1.z = atan(trans_atans(a1, a2, &p3)) + Pi * (p1 + p2 + p3);

  double R000 = 10. * abs_rand_mag(g, D000), R010 = 10. * abs_rand_mag(g, D010);
  double R001 = 10. * abs_rand_mag(g, D001), R011 = 10. * abs_rand_mag(g, D011);
  double R100 = 10. * abs_rand_mag(g, D100), R110 = 10. * abs_rand_mag(g, D110);
  double R101 = 10. * abs_rand_mag(g, D101), R111 = 10. * abs_rand_mag(g, D111);

  double z0pD100 = z0 + D100; if (z0pD100 < R100) z0pD100 = 0.5 * (x1e2 + y0e2) / dabs(z0);
  double z1pD101 = z1 + D101; if (z1pD101 < R101) z1pD101 = 0.5 * (x1e2 + y0e2) / dabs(z1);
  double z1pD001 = z1 + D001; if (z1pD001 < R001) z1pD001 = 0.5 * (x0e2 + y0e2) / dabs(z1);
  double z0pD000 = z0 + D000; if (z0pD000 < R000) z0pD000 = 0.5 * (x0e2 + y0e2) / dabs(z0);
  double z0pD010 = z0 + D010; if (z0pD010 < R010) z0pD010 = 0.5 * (x0e2 + y1e2) / dabs(z0);
  double z1pD011 = z1 + D011; if (z1pD011 < R011) z1pD011 = 0.5 * (x0e2 + y1e2) / dabs(z1);
  double z1pD111 = z1 + D111; if (z1pD111 < R111) z1pD111 = 0.5 * (x1e2 + y1e2) / dabs(z1);
  double z0pD110 = z0 + D110; if (z0pD110 < R110) z0pD110 = 0.5 * (x1e2 + y1e2) / dabs(z0);

  double y0pD100 = y0 + D100; if (y0pD100 < R100) y0pD100 = 0.5 * (x1e2 + z0e2) / dabs(y0);
  double y1pD110 = y1 + D110; if (y1pD110 < R110) y1pD110 = 0.5 * (x1e2 + z0e2) / dabs(y1);
  double y1pD010 = y1 + D010; if (y1pD010 < R010) y1pD010 = 0.5 * (x0e2 + z0e2) / dabs(y1);
  double y0pD000 = y0 + D000; if (y0pD000 < R000) y0pD000 = 0.5 * (x0e2 + z0e2) / dabs(y0);
  double y0pD001 = y0 + D001; if (y0pD001 < R001) y0pD001 = 0.5 * (x0e2 + z1e2) / dabs(y0);
  double y1pD011 = y1 + D011; if (y1pD011 < R011) y1pD011 = 0.5 * (x0e2 + z1e2) / dabs(y1);
  double y1pD111 = y1 + D111; if (y1pD111 < R111) y1pD111 = 0.5 * (x1e2 + z1e2) / dabs(y1);
  double y0pD101 = y0 + D101; if (y0pD101 < R101) y0pD101 = 0.5 * (x1e2 + z1e2) / dabs(y0);

  double x0pD010 = x0 + D010; if (x0pD010 < R010) x0pD010 = 0.5 * (y1e2 + z0e2) / dabs(x0);
  double x1pD110 = x1 + D110; if (x1pD110 < R110) x1pD110 = 0.5 * (y1e2 + z0e2) / dabs(x1);
  double x1pD100 = x1 + D100; if (x1pD100 < R100) x1pD100 = 0.5 * (y0e2 + z0e2) / dabs(x1);
  double x0pD000 = x0 + D000; if (x0pD000 < R000) x0pD000 = 0.5 * (y0e2 + z0e2) / dabs(x0);
  double x0pD001 = x0 + D001; if (x0pD001 < R001) x0pD001 = 0.5 * (y0e2 + z1e2) / dabs(x0);
  double x1pD101 = x1 + D101; if (x1pD101 < R101) x1pD101 = 0.5 * (y0e2 + z1e2) / dabs(x1);
  double x1pD111 = x1 + D111; if (x1pD111 < R111) x1pD111 = 0.5 * (y1e2 + z1e2) / dabs(x1);
  double x0pD011 = x0 + D011; if (x0pD011 < R011) x0pD011 = 0.5 * (y1e2 + z1e2) / dabs(x0);

  double qz_a = z0pD100 / z1pD101, qz_b = z1pD001 / z0pD000, qz_c = z0pD010 / z1pD011, qz_d = z1pD111 / z0pD110;
  double qy_a = y0pD100 / y1pD110, qy_b = y1pD010 / y0pD000, qy_c = y0pD001 / y1pD011, qy_d = y1pD111 / y0pD101;
  double qx_a = x0pD010 / x1pD110, qx_b = x1pD100 / x0pD000, qx_c = x0pD001 / x1pD101, qx_d = x1pD111 / x0pD011;
  const double C = 1. / 4. / Pi;

  if (Bj) {
    /* current-density branch, radrec.cpp:183-281 (ConstForJ = 1e-4) */
    double lza = log(qz_a), lzb = log(qz_b), lzc = log(qz_c), lzd = log(qz_d);
    double lya = log(qy_a), lyb = log(qy_b), lyc = log(qy_c), lyd = log(qy_d);
    double lxa = log(qx_a), lxb = log(qx_b), lxc = log(qx_c), lxd = log(qx_d);
    v3 bv = mk(x0 * T0.x + x1 * T1.x + y0 * (lza + lzb) + y1 * (lzc + lzd) + z0 * (lya + lyb) + z1 * (lyc + lyd),
               y0 * T0.y + y1 * T1.y + x0 * (lzc + lzb) + x1 * (lza + lzd) + z0 * (lxa + lxb) + z1 * (lxc + lxd),
               z0 * T0.z + z1 * T1.z + y0 * (lxc + lxb) + y1 * (lxa + lxd) + x0 * (lyc + lyb) + x1 * (lya + lyd));
    v3 cr = mk(J.y * bv.z - J.z * bv.y, J.z * bv.x - J.x * bv.z, J.x * bv.y - J.y * bv.x);
    Bj->x += 0.0001 * cr.x; Bj->y += 0.0001 * cr.y; Bj->z += 0.0001 * cr.z;
    return inside;
  }
  v3 T = add(T0, T1), S;
  S.x = -log(qx_a * qx_b * qx_c * qx_d);
  S.y = -log(qy_a * qy_b * qy_c * qy_d);
  S.z = -log(qz_a * qz_b * qz_c * qz_d);
  T.x *= C; T.y *= C; T.z *= C; S.x *= C; S.y *= C; S.z *= C;
  Q[0] = T.x;  Q[1] = -S.z; Q[2] = -S.y;
  Q[3] = -S.z; Q[4] = T.y;  Q[5] = -S.x;
  Q[6] = -S.y; Q[7] = -S.x; Q[8] = T.z;
  return inside;
}

/* ------------------------------------------------------------------------
 * Planar polygon face integrals (Sx, Sy, Sz) in the face frame at local
 * point (px, py, pz); returns the "point inside frame" flag (z > 0).
 * radTPolygon::B_comp, radplnr2.cpp:29-388, B/H/PreRelax paths.          */
static int polygon_S(const double *vtx, int nv, double coordz, v3 P, const guard_t *g, double *S)
{
  const double Max_k = 1.E+09;
  double cx = 0., cy = 0.;
  for (int k = 0; k < nv; k++) { cx += vtx[2 * k]; cy += vtx[2 * k + 1]; }
  cx /= nv; cy /= nv;
  double arx = abs_rand_mag(g, vtx[0] - cx), ary = abs_rand_mag(g, vtx[1] - cy);
  double arz = abs_rand_mag(g, coordz);
  if (arz < arx) arz = arx;
  if (arz < ary) arz = ary;
  double relr = abs_rand_mag(g, 1.);

  double z = coordz - P.z;
  if (z == 0.) z = arz;
  double ze2 = z * z;
  double f2x = vtx[0] - P.x, f2y = vtx[1] - P.y;
  double addx = -P.x, addy = -P.y;
  double x1 = f2x, y1 = f2y;
  if (x1 == 0.) { x1 = arx; f2x += arx; addx += arx; }
  if (y1 == 0.) { y1 = ary; f2y += ary; addy += ary; }
  double x1e2 = x1 * x1, y1e2 = y1 * y1, x2, y2, x2e2, y2e2;
  double Sx = 0., Sy = 0., sum_atan = 0., arg_logs2 = 1.;
  (void)y1e2;
  for (int i = 0; i < nv; i++) {
    if (i != nv - 1) { x2 = vtx[2 * (i + 1)] + addx; y2 = vtx[2 * (i + 1) + 1] + addy; }
    else { x2 = f2x; y2 = f2y; }
    if (x2 == 0.) { x2 = arx; f2x += arx; addx += arx; }
    if (y2 == 0.) { y2 = ary; f2y += ary; addy += ary; }
    x2e2 = x2 * x2; y2e2 = y2 * y2;
    double x2mx1 = x2 - x1, y2my1 = y2 - y1;
    if (dabs(x2mx1) * Max_k > dabs(y2my1)) {
      double k = y2my1 / x2mx1;
      double b = y1 - k * x1;
      if (b == 0.) {
        b = ary; y1 += ary; x1e2 = x1 * x1; y2my1 -= ary; k = y2my1 / x2mx1;
        f2y += ary; addy += ary;
      }
      double bk = b * k, ke2 = k * k, be2 = b * b, twob = 2. * b;
      double ke2p1 = ke2 + 1.;
      if (ke2p1 == 0.) ke2p1 = relr;
      double sqrtke2p1 = sqrt(ke2p1);
      double kx1 = k * x1, kx2 = k * x2;
      double bpkx1 = y1, bpkx2 = y2;
      double bpkx1e2 = bpkx1 * bpkx1, bpkx2e2 = bpkx2 * bpkx2;
      double kx1mb = -b + kx1, kx2mb = -b + kx2;
      double R1 = sqrt(x1e2 + bpkx1e2 + ze2), R2 = sqrt(x2e2 + bpkx2e2 + ze2);
      double x1e2pze2 = x1e2 + ze2, x2e2pze2 = x2e2 + ze2;
      double bkpx1pke2x1 = bk + ke2p1 * x1, bkpx2pke2x2 = bk + ke2p1 * x2;
      double kze2 = k * ze2, ke2ze2 = k * kze2;
      double ke2ze2mbe2 = ke2ze2 - be2, ke2ze2pbe2 = ke2ze2 + be2;
      double bx1 = b * x1, bx2 = b * x2;
      double R1pbpkx1 = bpkx1 + R1, R2pbpkx2 = bpkx2 + R2;
      const double MaxRelTolToSwitch = 1.E-07;
      double arR2 = 100. * abs_rand_mag(g, R2), arR1 = 100. * abs_rand_mag(g, R1);
      double mR1 = MaxRelTolToSwitch * R1, mR2 = MaxRelTolToSwitch * R2;
      if (arR1 > mR1) arR1 = mR1;
      if (arR2 > mR2) arR2 = mR2;
      if ((R1pbpkx1 < arR1) && (R1 > 100. * arR1) && ((x1e2 + ze2) < bpkx1e2 * MaxRelTolToSwitch))
        R1pbpkx1 = 0.5 * (x1e2 + ze2) / dabs(bpkx1);
      if ((R2pbpkx2 < arR2) && (R2 > 100. * arR2) && ((x2e2 + ze2) < bpkx2e2 * MaxRelTolToSwitch))
        R2pbpkx2 = 0.5 * (x2e2 + ze2) / dabs(bpkx2);
      double A1 = -(ke2ze2pbe2 * (bx1 + kze2) * R1pbpkx1 + kze2 * twob * x1e2pze2);
      double A2 = (ke2ze2pbe2 * kx1mb * R1pbpkx1 + ke2ze2mbe2 * x1e2pze2) * z;
      double A3 = ke2ze2pbe2 * (bx2 + kze2) * R2pbpkx2 + kze2 * twob * x2e2pze2;
      double A4 = (ke2ze2pbe2 * kx2mb * R2pbpkx2 + ke2ze2mbe2 * x2e2pze2) * z;
      sum_atan += atan2(A1 * A4 + A3 * A2, A2 * A4 - A1 * A3);
      double L1 = bkpx1pke2x1 / sqrtke2p1 + R1, L2 = bkpx2pke2x2 / sqrtke2p1 + R2;
      double be2pze2 = be2 + ze2;
      if ((L1 < arR1) && (R1 > 100. * arR1) && ((be2pze2 + 2 * bk * x1) < x1e2 * ke2p1 * MaxRelTolToSwitch))
        L1 = 0.5 * be2pze2 / (dabs(x1) * sqrtke2p1);
      if ((L2 < arR2) && (R2 > 100. * arR2) && ((be2pze2 + 2 * bk * x2) < x2e2 * ke2p1 * MaxRelTolToSwitch))
        L2 = 0.5 * be2pze2 / (dabs(x2) * sqrtke2p1);
      if (L1 == 0.) L1 = 1.e-50;
      if (L2 == 0.) L2 = 1.e-50;
      double sl1 = log(L2 / L1) / sqrtke2p1;
      if (R1pbpkx1 == 0.) R1pbpkx1 = 1.e-50;
      arg_logs2 *= (R2pbpkx2 / R1pbpkx1);
      Sx += -k * sl1;
      Sy += sl1;
    }
    x1 = x2; y1 = y2; x1e2 = x2e2; y1e2 = y2e2;
  }
  if (arg_logs2 <= 0.) arg_logs2 = 1.e-50;
  Sx += log(arg_logs2);
  S[0] = Sx; S[1] = Sy; S[2] = sum_atan;
  return z > 0.;
}

/* Polyhedron tensor Q (H = Q M, object frame) and inside flag
 * (radvlpgn.cpp:441-505; face Q as radplnr2.cpp:367-375).                */
static int poly_q(const RadB200Geom *G, int ip, v3 p, const guard_t *g, double *Q)
{
  const double PI = 3.14159265358979;
  const double CH = 1. / 4. / PI;
  int f0 = G->poly_info[4 * ip], nf = G->poly_info[4 * ip + 1];
  int inside = 1;
  for (int k = 0; k < 9; k++) Q[k] = 0.;
  for (int f = f0; f < f0 + nf; f++) {
    const double *R = G->face + (size_t)f * RADB200_FACE_STRIDE;
    v3 pl = mulm(R, p);
    double S[3];
    int in = polygon_S(G->vtx2d + 2 * (size_t)G->face_vtx[2 * f], G->face_vtx[2 * f + 1], R[9], pl, g, S);
    if (!in) inside = 0;
    /* Q_lab += R^T (col z = -C S) R  =  (R^T (-C S)) n^T with n = row 2 of R */
    v3 w = mulmt(R, mk(-CH * S[0], -CH * S[1], -CH * S[2]));
    const double *n = R + 6;
    Q[0] += w.x * n[0]; Q[1] += w.x * n[1]; Q[2] += w.x * n[2];
    Q[3] += w.y * n[0]; Q[4] += w.y * n[1]; Q[5] += w.y * n[2];
    Q[6] += w.z * n[0]; Q[7] += w.z * n[1]; Q[8] += w.z * n[2];
  }
  return inside;
}

/* ------------------------------------------------------------------------
 * Arc current, radarccu.cpp:30-236 (B and H only).                       */
static v3 arc_field(const double *a, v3 P)
{
  const double Pi = 3.141592653589793238, ZeroTol = 1.E-10, RZ = 1.E-07, SmallPositive = 1.E-10;
  v3 pc = sub(P, mk(a[0], a[1], a[2]));
  double Rmin = a[3], Rmax = a[4], Phimin = a[5], Phimax = a[6], Height = a[7], Jaz = a[8];
  int nsec = (int)a[9];
  double r = sqrt(pc.x * pc.x + pc.y * pc.y + SmallPositive);
  double phi = (pc.y < 0) ? (2 * Pi - acos(pc.x / r)) : acos(pc.x / r);
  double z1 = -Height / 2. - pc.z, z2 = z1 + Height;
  double z1z1 = z1 * z1, z2z2 = z2 * z2, rr = r * r, r1r1 = Rmin * Rmin, r2r2 = Rmax * Rmax;
  double a11 = rr + r1r1 + z1z1, a12 = rr + r1r1 + z2z2, a21 = rr + r2r2 + z1z1, a22 = rr + r2r2 + z2z2;
  double two_r = 2. * r, two_rr1 = two_r * Rmin, two_rr2 = two_r * Rmax;
  int npoi = nsec + 1;
  double step = (Phimax - Phimin + SmallPositive) / (npoi - 1);
  double dphi = Phimin - phi + SmallPositive;
  double SBx = 0., SBy = 0., SBz = 0.;
  for (int i = 0; i < npoi; i++) {
    double cdp = cos(dphi), asdp = dabs(sin(dphi));
    double t1 = two_rr1 * cdp, t2 = two_rr2 * cdp;
    double b11 = fabs(a11 - t1); if (b11 < ZeroTol) b11 = ZeroTol;
    double D11 = sqrt(b11), D12 = sqrt(fabs(a12 - two_rr1 * cdp));
    double b21 = fabs(a21 - t2); if (b21 < ZeroTol) b21 = ZeroTol;
    double D21 = sqrt(b21), D22 = sqrt(fabs(a22 - two_rr2 * cdp));
    double rCos = r * cdp, r1m = Rmin - rCos, r2m = Rmax - rCos;
    double d11 = D11 * RZ, d12 = D12 * RZ, d21 = D21 * RZ, d22 = D22 * RZ;
    double re2s2 = rr * asdp * asdp, zz = z1z1 + re2s2;
    double r1me2 = r1m * r1m, r2me2 = r2m * r2m;
    double u11 = r1m + D11; if ((dabs(u11) < d11) && (zz < r1me2 * RZ)) u11 = 0.5 * zz / dabs(r1m);
    double u12 = r1m + D12; if ((dabs(u12) < d12) && (zz < r1me2 * RZ)) u12 = 0.5 * zz / dabs(r1m);
    double u21 = r2m + D21; if ((dabs(u21) < d21) && (zz < r2me2 * RZ)) u21 = 0.5 * zz / dabs(r2m);
    double u22 = r2m + D22; if ((dabs(u22) < d22) && (zz < r2me2 * RZ)) u22 = 0.5 * zz / dabs(r2m);
    double ln1 = log(u11 / u21), ln2 = log(u22 / u12);
    double rAbsSin = r * asdp;
    double q1 = dabs(r1m) / rAbsSin, q2 = dabs(r2m) / rAbsSin;
    double pm1 = 0., pm2 = 0.;
    double at1 = atan(trans_atans(z2 * q1 / D12, -z1 * q1 / D11, &pm1)) + Pi * pm1;
    double at2 = atan(trans_atans(z1 * q2 / D21, -z2 * q2 / D22, &pm2)) + Pi * pm2;
    double Buf = rAbsSin * (sgn(r1m) * at1 + sgn(r2m) * at2) + z1 * ln1 + z2 * ln2;
    double w11 = z1 + D11, s1 = rr + r1r1 - t1;
    double z1t = z1z1 * RZ, z2t = z2z2 * RZ;
    if ((dabs(w11) < d11) && (s1 < z1t)) w11 = 0.5 * s1 / dabs(z1);
    double w21 = z1 + D21, s2 = rr + r2r2 - t2;
    if ((dabs(w21) < d21) && (s2 < z1t)) w21 = 0.5 * s2 / dabs(z1);
    double w12 = z2 + D12;
    if ((dabs(w12) < d12) && (s1 < z2t)) w12 = 0.5 * s1 / dabs(z2);
    double w22 = z2 + D22;
    if ((dabs(w22) < d22) && (s2 < z2t)) w22 = 0.5 * s2 / dabs(z2);
    double qa = w11 / w12, qb = w22 / w21;
    double php = dphi + phi, cph = cos(php), sph = sin(php);
    double FBxy = D11 - D21 + D22 - D12 + rCos * (ln1 + ln2);
    double FBz = Buf - rCos * log(qa * qb);
    double wgt = (i == 0 || i == npoi - 1) ? 0.5 : 1.0;
    SBx += wgt * cph * FBxy;
    SBy += wgt * sph * FBxy;
    SBz += wgt * FBz;
    dphi += step;
  }
  double fact = 0.0001 * Jaz;
  return mk(fact * step * SBx, fact * step * SBy, fact * step * SBz);
}

/* ------------------------------------------------------------------------
 * Field of all sources at one point.  what: 0 B, 1 H, 2 M.
 * Image sum as radTg3d::NestedFor_B (radg3d.cpp:58-120): each image of a
 * source contributes s*M*F(M^-1 (P - V)).                                  */
static v3 field_at(const RadB200Geom *G, v3 P, int what, const guard_t *g)
{
  v3 acc = mk(0, 0, 0);
  for (int i = 0; i < G->n_rec; i++) {
    const double *r = G->rec + (size_t)i * RADB200_REC_STRIDE;
    v3 c = mk(r[0], r[1], r[2]), d = mk(r[3], r[4], r[5]), m = mk(r[6], r[7], r[8]), J = mk(r[9], r[10], r[11]);
    int jz = (J.x == 0. && J.y == 0. && J.z == 0.);
    int t0 = G->rec_img[2 * i], nt = G->rec_img[2 * i + 1];
    for (int t = t0; t < t0 + nt; t++) {
      const double *T = G->trf + (size_t)t * RADB200_TRF_STRIDE;
      v3 q = mulm(T, sub(P, mk(T[9], T[10], T[11])));
      v3 f = mk(0, 0, 0);
      if (!jz) {
        if (what != 2) { double Q[9]; recmag_core(c, d, q, g, Q, J, &f); }
      } else {
        double Q[9];
        int in = recmag_core(c, d, q, g, Q, J, 0);
        if (what == 2) { if (in) f = m; }
        else {
          f = mulm(Q, m);
          if (what == 0 && in) f = add(f, m);
        }
      }
      acc = add(acc, mulm(T + 12, f));
    }
  }
  for (int i = 0; i < G->n_poly; i++) {
    const double *pr = G->poly + (size_t)i * RADB200_POLY_STRIDE;
    v3 m = mk(pr[3], pr[4], pr[5]);
    if (m.x == 0. && m.y == 0. && m.z == 0.) continue;
    int t0 = G->poly_info[4 * i + 2], nt = G->poly_info[4 * i + 3];
    for (int t = t0; t < t0 + nt; t++) {
      const double *T = G->trf + (size_t)t * RADB200_TRF_STRIDE;
      v3 q = mulm(T, sub(P, mk(T[9], T[10], T[11])));
      double Q[9];
      int in = poly_q(G, i, q, g, Q);
      v3 f;
      if (what == 2) f = in ? m : mk(0, 0, 0);
      else {
        f = mulm(Q, m);
        if (what == 0 && in) f = add(f, m);
      }
      acc = add(acc, mulm(T + 12, f));
    }
  }
  if (what != 2) {
    for (int i = 0; i < G->n_arc; i++) {
      const double *a = G->arc + (size_t)i * RADB200_ARC_STRIDE;
      int t0 = G->arc_img[2 * i], nt = G->arc_img[2 * i + 1];
      for (int t = t0; t < t0 + nt; t++) {
        const double *T = G->trf + (size_t)t * RADB200_TRF_STRIDE;
        v3 q = mulm(T, sub(P, mk(T[9], T[10], T[11])));
        acc = add(acc, mulm(T + 12, arc_field(a, q)));
      }
    }
    for (int i = 0; i < G->n_bkg; i++) {
      const double *b = G->bkg + 3 * (size_t)i;
      int t0 = G->bkg_img[2 * i], nt = G->bkg_img[2 * i + 1];
      for (int t = t0; t < t0 + nt; t++) {
        const double *T = G->trf + (size_t)t * RADB200_TRF_STRIDE;
        acc = add(acc, mulm(T + 12, mk(b[0], b[1], b[2])));
      }
    }
  }
  return acc;
}

ORC_API int orc_field(const RadB200Geom *G, const double *pts, int64_t n, int what, double *out)
{
  guard_t g = {G->abs_rand, G->rel_rand, G->zero_rand};
  for (int64_t i = 0; i < n; i++) {
    v3 f = field_at(G, mk(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), what, &g);
    out[3 * i] = f.x; out[3 * i + 1] = f.y; out[3 * i + 2] = f.z;
  }
  return 0;
}

/* Tensor Q (object frame) of relaxable element e at object-frame point q. */
static void elem_q(const RadB200Geom *G, const RadB200Relax *R, int e, v3 q, const guard_t *g, double *Q)
{
  int kind = R->elem_src[2 * e], idx = R->elem_src[2 * e + 1];
  if (kind == 0) {
    const double *r = G->rec + (size_t)idx * RADB200_REC_STRIDE;
    recmag_core(mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), q, g, Q, mk(0, 0, 0), 0);
  } else {
    poly_q(G, idx, q, g, Q);
  }
}

static void elem_imgs(const RadB200Geom *G, const RadB200Relax *R, int e, int *t0, int *nt, v3 *c)
{
  int kind = R->elem_src[2 * e], idx = R->elem_src[2 * e + 1];
  if (kind == 0) {
    const double *r = G->rec + (size_t)idx * RADB200_REC_STRIDE;
    *t0 = G->rec_img[2 * idx]; *nt = G->rec_img[2 * idx + 1]; *c = mk(r[0], r[1], r[2]);
  } else {
    const double *p = G->poly + (size_t)idx * RADB200_POLY_STRIDE;
    *t0 = G->poly_info[4 * idx + 2]; *nt = G->poly_info[4 * idx + 3]; *c = mk(p[0], p[1], p[2]);
  }
}

static v3 trf_point(const double *T, v3 p)
{ /* M p + V from s*M and s */
  double s = T[21];
  v3 r = mulm(T + 12, p);
  return mk(r.x / s + T[9], r.y / s + T[10], r.z / s + T[11]);
}

/* Dense FP64 interaction matrix, row major [3N x 3N], radintrc.cpp:831-877:
 * block(i,j) = (s_i M_i^-1) * sum_img (s M) Q_j(M^-1 (obs_i - V)).         */
ORC_API int orc_assemble(const RadB200Geom *G, const RadB200Relax *R, double *N)
{
  guard_t g = {G->abs_rand, G->rel_rand, G->zero_rand};
  int n = R->n_elem;
  int64_t ld = 3 * (int64_t)n;
  for (int i = 0; i < n; i++) {
    int ti, nti; v3 ci;
    elem_imgs(G, R, i, &ti, &nti, &ci);
    const double *Ti = G->trf + (size_t)ti * RADB200_TRF_STRIDE;
    v3 obs = trf_point(Ti, ci);
    for (int j = 0; j < n; j++) {
      int tj, ntj; v3 cj;
      elem_imgs(G, R, j, &tj, &ntj, &cj);
      double B[9] = {0};
      for (int t = tj; t < tj + ntj; t++) {
        const double *T = G->trf + (size_t)t * RADB200_TRF_STRIDE;
        v3 q = mulm(T, sub(obs, mk(T[9], T[10], T[11])));
        double Q[9];
        elem_q(G, R, j, q, &g, Q);
        const double *F = T + 12;
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++)
            B[3 * a + b] += F[3 * a] * Q[b] + F[3 * a + 1] * Q[3 + b] + F[3 * a + 2] * Q[6 + b];
      }
      /* row transform s_i M_i^-1 = s_i^2 * M_i^-1 ... stored: Minv, s */
      double si = Ti[21];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          double v = si * (Ti[3 * a] * B[b] + Ti[3 * a + 1] * B[3 + b] + Ti[3 * a + 2] * B[6 + b]);
          N[(3 * (int64_t)i + a) * ld + 3 * (int64_t)j + b] = v;
        }
    }
  }
  return 0;
}

/* External field H at element centres, element frames (radintrc.cpp:1208-1234). */
ORC_API int orc_extfield(const RadB200Geom *G, const RadB200Relax *R, const RadB200Geom *X, double *H)
{
  guard_t g = {X->abs_rand, X->rel_rand, X->zero_rand};
  for (int i = 0; i < R->n_elem; i++) {
    int ti, nti; v3 ci;
    elem_imgs(G, R, i, &ti, &nti, &ci);
    const double *Ti = G->trf + (size_t)ti * RADB200_TRF_STRIDE;
    v3 obs = trf_point(Ti, ci);
    v3 f = field_at(X, obs, 1, &g);
    v3 loc = mulm(Ti, f);
    double si = Ti[21];
    H[3 * i] = si * loc.x; H[3 * i + 1] = si * loc.y; H[3 * i + 2] = si * loc.z;
  }
  return 0;
}

/* ------------------------------------------------------------------------
 * Materials.                                                               */
static int inv3(const double *A, double *B)
{
  double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) + A[2] * (A[3] * A[7] - A[4] * A[6]);
  double id = 1. / det;
  B[0] = (A[4] * A[8] - A[5] * A[7]) * id; B[1] = (A[2] * A[7] - A[1] * A[8]) * id; B[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  B[3] = (A[5] * A[6] - A[3] * A[8]) * id; B[4] = (A[0] * A[8] - A[2] * A[6]) * id; B[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  B[6] = (A[3] * A[7] - A[4] * A[6]) * id; B[7] = (A[1] * A[6] - A[0] * A[7]) * id; B[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return 0;
}

/* Tabulated M(H): linear interpolation between table points, slope of the
 * last segment beyond the table (simplified from AbsMvsAbsH_Interpol).     */
static double table_m(const double *tab, int n, double h, double *dmdh)
{
  if (n <= 1) { *dmdh = 0; return 0; }
  int k = 0;
  while (k < n - 2 && tab[3 * (k + 1)] < h) k++;
  double h0 = tab[3 * k], h1 = tab[3 * (k + 1)], m0 = tab[3 * k + 1], m1 = tab[3 * (k + 1) + 1];
  double s = (m1 - m0) / (h1 - h0);
  *dmdh = s;
  return m0 + s * (h - h0);
}

/* scalar law f(|H|), df/d|H| (radmater.cpp:279-306) */
static void scalar_law(const RadB200Relax *R, int e, double h, double *f, double *df)
{
  const double *m = R->mat + (size_t)e * RADB200_MAT_STRIDE;
  *f = 0.; *df = 0.;
  if (R->mat_kind[e] == RADB200_MAT_TANH) {
    int n = (int)m[6];
    for (int i = 0; i < n; i++) {
      double ks = m[i], ms = m[3 + i];
      if (ms == 0.) continue;
      double arg = ks * h / ms;
      *f += ms * tanh(arg);
      double ch = cosh(arg);
      *df += ks / (ch * ch);
    }
  } else if (R->mat_kind[e] == RADB200_MAT_TABLE) {
    *f = table_m(R->mh_table + 3 * (size_t)m[0], (int)m[1], h, df);
  }
}

ORC_API void orc_material_m(const RadB200Relax *R, int e, const double *H, double *M)
{
  const double *m = R->mat + (size_t)e * RADB200_MAT_STRIDE;
  if (R->mat_kind[e] == RADB200_MAT_LINEAR) {
    v3 r = mulm(m, mk(H[0], H[1], H[2]));
    M[0] = r.x + m[9]; M[1] = r.y + m[10]; M[2] = r.z + m[11];
    return;
  }
  double h = sqrt(H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
  double f, df;
  scalar_law(R, e, h, &f, &df);
  double ksi;
  if (h <= 1e-10) {
    ksi = 0.;
    if (R->mat_kind[e] == RADB200_MAT_TANH) { for (int i = 0; i < (int)m[6]; i++) ksi += m[i]; }
    else ksi = df;
  } else ksi = f / h;
  M[0] = ksi * H[0] + m[9]; M[1] = ksi * H[1] + m[10]; M[2] = ksi * H[2] + m[11];
}

/* FindNewH: linear laws radmater.h:223-231 / 351-359; nonlinear
 * radmater.cpp:72-164 (damped secant on |H|, at most 15 passes).         */
static void find_new_h(const RadB200Relax *R, int e, double *H, const double *Qii, const double *Hq, double prec_e2)
{
  const double *m = R->mat + (size_t)e * RADB200_MAT_STRIDE;
  double A[9], Ai[9];
  if (R->mat_kind[e] == RADB200_MAT_LINEAR) {
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        double s = 0.;
        for (int k = 0; k < 3; k++) s += Qii[3 * a + k] * m[3 * k + b];
        A[3 * a + b] = (a == b ? 1. : 0.) - s;
      }
    inv3(A, Ai);
    v3 rhs = add(mk(Hq[0], Hq[1], Hq[2]), mulm(Qii, mk(m[9], m[10], m[11])));
    v3 r = mulm(Ai, rhs);
    H[0] = r.x; H[1] = r.y; H[2] = r.z;
    return;
  }
  double misfit = 3.;
  double ah = sqrt(H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
  double ksi = 0.;
  for (int it = 0; it < 15; it++) {
    double f = 0., df;
    if (ah <= 1e-10) {
      if (R->mat_kind[e] == RADB200_MAT_TANH) { for (int i = 0; i < (int)m[6]; i++) ksi += m[i]; }
      else { scalar_law(R, e, 0., &f, &df); ksi = df; f = 0.; }
      f = 0.;
    } else {
      scalar_law(R, e, ah, &f, &df);
      ksi = f / ah;
    }
    for (int k = 0; k < 9; k++) A[k] = ((k % 4) == 0 ? 1. : 0.) - ksi * Qii[k];
    inv3(A, Ai);
    v3 r = mulm(Ai, mk(Hq[0], Hq[1], Hq[2]));
    H[0] = r.x; H[1] = r.y; H[2] = r.z;
    double nah = sqrt(r.x * r.x + r.y * r.y + r.z * r.z);
    double nmis = f - nah * ksi;
    double am = fabs(misfit), anm = fabs(nmis);
    double pn = am;
    if (nmis * misfit > 0) pn += 0.5 * anm;
    double po = anm;
    double alpha = pn / (pn + po);
    ah = alpha * nah + (1 - alpha) * ah;
    misfit = f - ah * ksi;
    if (misfit * misfit <= prec_e2) break;
  }
}

/* Relaxation method 4 (radrlmet.cpp:496-587, 772-829) on an FP64 or FP32
 * matrix N (row major, 3N x 3N).  M_io: start value when reset == 0;
 * reset != 0 starts from the remanence (radintrc.h:385-395).
 * status[4]: misfit, max|M|, max|H|, iterations.                           */
ORC_API int orc_relax_m4(const RadB200Relax *R, const double *N64, const float *N32, const double *Hext,
                         double prec, int max_iter, int reset, double *M, double *Hout, double *status)
{
  int n = R->n_elem;
  int64_t ld = 3 * (int64_t)n;
  double *Hn = (double *)calloc(3 * (size_t)n, sizeof(double));
  if (reset)
    for (int e = 0; e < n; e++) {
      const double *m = R->mat + (size_t)e * RADB200_MAT_STRIDE;
      M[3 * e] = m[9]; M[3 * e + 1] = m[10]; M[3 * e + 2] = m[11];
    }
  double prec_e2 = prec * prec, inst = 1.e+23;
  int iters = 0;
  while (inst > prec_e2) {
    if (++iters > max_iter) break;
    double nf = 1. / n;
    double best = prec_e2 * nf;
    double loc = (inst > 1.e+20) ? best : 0.25 * nf * inst;
    if (loc < best) loc = best;
    double sum = 0.;
    for (int i = 0; i < n; i++) {
      double hq[3] = {Hext[3 * i], Hext[3 * i + 1], Hext[3 * i + 2]};
      double acc[3] = {0, 0, 0};
      for (int j = 0; j < n; j++) {
        if (j == i) continue;
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) {
            int64_t ix = (3 * (int64_t)i + a) * ld + 3 * (int64_t)j + b;
            acc[a] += (N64 ? N64[ix] : (double)N32[ix]) * M[3 * j + b];
          }
      }
      for (int a = 0; a < 3; a++) hq[a] += acc[a];
      double Qii[9];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          int64_t ix = (3 * (int64_t)i + a) * ld + 3 * (int64_t)i + b;
          Qii[3 * a + b] = N64 ? N64[ix] : (double)N32[ix];
        }
      find_new_h(R, i, Hn + 3 * i, Qii, hq, loc);
      double Mn[3];
      orc_material_m(R, i, Hn + 3 * i, Mn);
      for (int a = 0; a < 3; a++) {
        double d = Mn[a] - M[3 * i + a];
        sum += d * d;
        M[3 * i + a] = Mn[a];
      }
    }
    inst = sum / n;
  }
  double maxm = 0., maxh = 0.;
  for (int i = 0; i < n; i++) {
    double am = sqrt(M[3 * i] * M[3 * i] + M[3 * i + 1] * M[3 * i + 1] + M[3 * i + 2] * M[3 * i + 2]);
    double ah = sqrt(Hn[3 * i] * Hn[3 * i] + Hn[3 * i + 1] * Hn[3 * i + 1] + Hn[3 * i + 2] * Hn[3 * i + 2]);
    if (am > maxm) maxm = am;
    if (ah > maxh) maxh = ah;
  }
  if (Hout) memcpy(Hout, Hn, 3 * (size_t)n * sizeof(double));
  status[0] = sqrt(inst); status[1] = maxm; status[2] = maxh; status[3] = iters - 1;
  free(Hn);
  return 0;
}

/* dM/dH at H for element e (radmater.cpp:206-277; linear: chi tensor). */
ORC_API void orc_material_dmdh(const RadB200Relax *R, int e, const double *H, double *D)
{
  const double *m = R->mat + (size_t)e * RADB200_MAT_STRIDE;
  if (R->mat_kind[e] == RADB200_MAT_LINEAR) { for (int k = 0; k < 9; k++) D[k] = m[k]; return; }
  double h0 = sqrt(H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
  double f, df;
  scalar_law(R, e, h0, &f, &df);
  if (fabs(h0) < 1e-10) { for (int k = 0; k < 9; k++) D[k] = (k % 4 == 0) ? df : 0.; return; }
  double ih3 = 1. / (h0 * h0 * h0);
  double hx = H[0], hy = H[1], hz = H[2];
  double off = ih3 * (h0 * df - f);
  D[0] = ih3 * ((hy * hy + hz * hz) * f + hx * hx * h0 * df);
  D[4] = ih3 * ((hx * hx + hz * hz) * f + hy * hy * h0 * df);
  D[8] = ih3 * ((hx * hx + hy * hy) * f + hz * hz * h0 * df);
  D[1] = D[3] = off * hx * hy;
  D[2] = D[6] = off * hx * hz;
  D[5] = D[7] = off * hy * hz;
}
