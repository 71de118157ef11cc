// formulas.cuh -- device formulas of the Radia field sources (sm_100a).
//
// Closed forms, restated for the device from the reference CPU code (the GPU
// port of the reference differs in places; the CPU code is the contract):
//   cuboid tensor / current field    radTRecMag::B_comp      radrec.cpp:49-315
//   polygon face integrals           radTPolygon::B_comp     radplnr2.cpp:29-388
//   arc current (trapezoid in phi)   radTArcCur::B_compWithTrapeth radarccu.cpp:30-236
// All functions are templated on the arithmetic type T (double, or float for
// the single-precision field option); guards follow radTConvergRepair
// (radcnvrg.h:85-91) with the magnitudes passed in Guard.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace rb {

template <typename T> struct V3 { T x, y, z; };
template <typename T> __host__ __device__ __forceinline__ V3<T> mk3(T x, T y, T z) { V3<T> r; r.x = x; r.y = y; r.z = z; return r; }

struct Guard { double absr, relr, zeror; };

template <typename T> __device__ __forceinline__ T fabsT(T x) { return x < T(0) ? -x : x; }
__device__ __forceinline__ double logT(double x) { return log(x); }
__device__ __forceinline__ float logT(float x) { return logf(x); }
__device__ __forceinline__ double atanT(double x) { return atan(x); }
__device__ __forceinline__ float atanT(float x) { return atanf(x); }
__device__ __forceinline__ double atan2T(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ float atan2T(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double sqrtT(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrtT(float x) { return sqrtf(x); }

// radTConvergRepair::AbsRandMagnitude (radcnvrg.h:85-91)
template <typename T> __device__ __forceinline__ T abs_rand(const Guard &g, T A)
{
  if (g.absr == 0.0 && g.relr == 0.0 && g.zeror == 0.0) return T(0);
  T fromrel = T(g.relr) * A;
  T amax = (fromrel < T(g.absr)) ? T(g.absr) : fromrel;
  return (A != T(0)) ? amax : ((amax < T(g.zeror)) ? T(g.zeror) : amax);
}

// radTg3d::TransAtans (radg3d.h:938-946)
template <typename T> __device__ __forceinline__ T trans_atans(T x, T y, T &pimult)
{
  T buf = T(1) - x * y;
  if (buf == T(0)) buf = sizeof(T) == 8 ? T(1e-50) : T(1e-30);
  pimult = ((buf > T(0)) ? T(0) : T(1)) * ((x < T(0)) ? T(-1) : T(1));
  return (x + y) / buf;
}

// Sum of four arctangents with branch bookkeeping, as the cuboid formula
// evaluates T0/T1 components (radrec.cpp:117-128).
template <typename T> __device__ __forceinline__ T atan4(T a, T b, T c, T d)
{
  const T Pi = T(3.141592653589793238);
  T p1, p2, p3;
  T u = trans_atans(a, b, p1);
  T v = trans_atans(c, d, p2);
  T w = trans_atans(u, v, p3);
  return atanT(w) + Pi * (p1 + p2 + p3);
}

// Cuboid: q = observation point RELATIVE TO THE CUBOID CENTRE (object frame),
// hd = half dimensions.  Returns 1 if strictly inside.  Writes the symmetric
// tensor entries T = (Txx,Tyy,Tzz) and S = (Sx,Sy,Sz) scaled by 1/(4 pi):
//   Q = [[Tx,-Sz,-Sy],[-Sz,Ty,-Sx],[-Sy,-Sx,Tz]]    (radrec.cpp:265-283)
template <typename T>
__device__ __forceinline__ int cuboid_TS(V3<double> q, V3<double> hd, const Guard &g, V3<T> &Tt, V3<T> &Ss)
{
  // corner offsets in FP64 (exact zeros and guards decided before any rounding to T)
  double dx0 = -q.x - hd.x, dx1 = -q.x + hd.x;
  double dy0 = -q.y - hd.y, dy1 = -q.y + hd.y;
  double dz0 = -q.z - hd.z, dz1 = -q.z + hd.z;
  if (dx0 == 0.0) dx0 = abs_rand(g, hd.x);
  if (dx1 == 0.0) dx1 = abs_rand(g, hd.x);
  if (dy0 == 0.0) dy0 = abs_rand(g, hd.y);
  if (dy1 == 0.0) dy1 = abs_rand(g, hd.y);
  if (dz0 == 0.0) dz0 = abs_rand(g, hd.z);
  if (dz1 == 0.0) dz1 = abs_rand(g, hd.z);
  T x0 = T(dx0), x1 = T(dx1), y0 = T(dy0), y1 = T(dy1), z0 = T(dz0), z1 = T(dz1);
  int inside = (x0 * x1 < T(0)) && (y0 * y1 < T(0)) && (z0 * z1 < T(0));
  T x0e2 = x0 * x0, x1e2 = x1 * x1, y0e2 = y0 * y0, y1e2 = y1 * y1, z0e2 = z0 * z0, z1e2 = z1 * z1;
  T D000 = sqrtT(x0e2 + y0e2 + z0e2), D100 = sqrtT(x1e2 + y0e2 + z0e2);
  T D010 = sqrtT(x0e2 + y1e2 + z0e2), D110 = sqrtT(x1e2 + y1e2 + z0e2);
  T D001 = sqrtT(x0e2 + y0e2 + z1e2), D101 = sqrtT(x1e2 + y0e2 + z1e2);
  T D011 = sqrtT(x0e2 + y1e2 + z1e2), D111 = sqrtT(x1e2 + y1e2 + z1e2);

  T T0x = atan4(y0 * z0 / (x0 * D000), -y0 * z1 / (x0 * D001), -y1 * z0 / (x0 * D010), y1 * z1 / (x0 * D011));
  T T1x = atan4(-y0 * z0 / (x1 * D100), y0 * z1 / (x1 * D101), y1 * z0 / (x1 * D110), -y1 * z1 / (x1 * D111));
  T T0y = atan4(x0 * z0 / (y0 * D000), -x0 * z1 / (y0 * D001), -x1 * z0 / (y0 * D100), x1 * z1 / (y0 * D101));
  T T1y = atan4(-x0 * z0 / (y1 * D010), x0 * z1 / (y1 * D011), x1 * z0 / (y1 * D110), -x1 * z1 / (y1 * D111));
  T T0z = atan4(x0 * y0 / (z0 * D000), -x1 * y0 / (z0 * D100), -x0 * y1 / (z0 * D010), x1 * y1 / (z0 * D110));
  T T1z = atan4(-x0 * y0 / (z1 * D001), x1 * y0 / (z1 * D101), x0 * y1 / (z1 * D011), -x1 * y1 / (z1 * D111));

  T R000 = T(10) * abs_rand(g, D000), R010 = T(10) * abs_rand(g, D010);
  T R001 = T(10) * abs_rand(g, D001), R011 = T(10) * abs_rand(g, D011);
  T R100 = T(10) * abs_rand(g, D100), R110 = T(10) * abs_rand(g, D110);
  T R101 = T(10) * abs_rand(g, D101), R111 = T(10) * abs_rand(g, D111);
  const T h = T(0.5);
  T z0pD100 = z0 + D100; if (z0pD100 < R100) z0pD100 = h * (x1e2 + y0e2) / fabsT(z0);
  T z1pD101 = z1 + D101; if (z1pD101 < R101) z1pD101 = h * (x1e2 + y0e2) / fabsT(z1);
  T z1pD001 = z1 + D001; if (z1pD001 < R001) z1pD001 = h * (x0e2 + y0e2) / fabsT(z1);
  T z0pD000 = z0 + D000; if (z0pD000 < R000) z0pD000 = h * (x0e2 + y0e2) / fabsT(z0);
  T z0pD010 = z0 + D010; if (z0pD010 < R010) z0pD010 = h * (x0e2 + y1e2) / fabsT(z0);
  T z1pD011 = z1 + D011; if (z1pD011 < R011) z1pD011 = h * (x0e2 + y1e2) / fabsT(z1);
  T z1pD111 = z1 + D111; if (z1pD111 < R111) z1pD111 = h * (x1e2 + y1e2) / fabsT(z1);
  T z0pD110 = z0 + D110; if (z0pD110 < R110) z0pD110 = h * (x1e2 + y1e2) / fabsT(z0);

  T y0pD100 = y0 + D100; if (y0pD100 < R100) y0pD100 = h * (x1e2 + z0e2) / fabsT(y0);
  T y1pD110 = y1 + D110; if (y1pD110 < R110) y1pD110 = h * (x1e2 + z0e2) / fabsT(y1);
  T y1pD010 = y1 + D010; if (y1pD010 < R010) y1pD010 = h * (x0e2 + z0e2) / fabsT(y1);
  T y0pD000 = y0 + D000; if (y0pD000 < R000) y0pD000 = h * (x0e2 + z0e2) / fabsT(y0);
  T y0pD001 = y0 + D001; if (y0pD001 < R001) y0pD001 = h * (x0e2 + z1e2) / fabsT(y0);
  T y1pD011 = y1 + D011; if (y1pD011 < R011) y1pD011 = h * (x0e2 + z1e2) / fabsT(y1);
  T y1pD111 = y1 + D111; if (y1pD111 < R111) y1pD111 = h * (x1e2 + z1e2) / fabsT(y1);
  T y0pD101 = y0 + D101; if (y0pD101 < R101) y0pD101 = h * (x1e2 + z1e2) / fabsT(y0);

  T x0pD010 = x0 + D010; if (x0pD010 < R010) x0pD010 = h * (y1e2 + z0e2) / fabsT(x0);
  T x1pD110 = x1 + D110; if (x1pD110 < R110) x1pD110 = h * (y1e2 + z0e2) / fabsT(x1);
  T x1pD100 = x1 + D100; if (x1pD100 < R100) x1pD100 = h * (y0e2 + z0e2) / fabsT(x1);
  T x0pD000 = x0 + D000; if (x0pD000 < R000) x0pD000 = h * (y0e2 + z0e2) / fabsT(x0);
  T x0pD001 = x0 + D001; if (x0pD001 < R001) x0pD001 = h * (y0e2 + z1e2) / fabsT(x0);
  T x1pD101 = x1 + D101; if (x1pD101 < R101) x1pD101 = h * (y0e2 + z1e2) / fabsT(x1);
  T x1pD111 = x1 + D111; if (x1pD111 < R111) x1pD111 = h * (y1e2 + z1e2) / fabsT(x1);
  T x0pD011 = x0 + D011; if (x0pD011 < R011) x0pD011 = h * (y1e2 + z1e2) / fabsT(x0);

  const T C = T(1.0 / (4.0 * 3.141592653589793238));
  // S = -log(product of 4 ratios)  (radrec.cpp:257-260)
  T Sx = -logT((x0pD010 / x1pD110) * (x1pD100 / x0pD000) * (x0pD001 / x1pD101) * (x1pD111 / x0pD011));
  T Sy = -logT((y0pD100 / y1pD110) * (y1pD010 / y0pD000) * (y0pD001 / y1pD011) * (y1pD111 / y0pD101));
  T Sz = -logT((z0pD100 / z1pD101) * (z1pD001 / z0pD000) * (z0pD010 / z1pD011) * (z1pD111 / z0pD110));
  Tt = mk3<T>(C * (T0x + T1x), C * (T0y + T1y), C * (T0z + T1z));
  Ss = mk3<T>(C * Sx, C * Sy, C * Sz);
  return inside;
}

// Field of a current-carrying cuboid (radrec.cpp:183-249, J branch), q
// relative to the centre, J in A/mm^2; returns B (= H) in T.
__device__ __forceinline__ V3<double> cuboid_J(V3<double> q, V3<double> hd, V3<double> J, const Guard &g)
{
  typedef double T;
  T x0 = -q.x - hd.x, x1 = -q.x + hd.x, y0 = -q.y - hd.y, y1 = -q.y + hd.y, z0 = -q.z - hd.z, z1 = -q.z + hd.z;
  if (x0 == 0.) x0 = abs_rand(g, hd.x);
  if (x1 == 0.) x1 = abs_rand(g, hd.x);
  if (y0 == 0.) y0 = abs_rand(g, hd.y);
  if (y1 == 0.) y1 = abs_rand(g, hd.y);
  if (z0 == 0.) z0 = abs_rand(g, hd.z);
  if (z1 == 0.) z1 = abs_rand(g, hd.z);
  T x0e2 = x0 * x0, x1e2 = x1 * x1, y0e2 = y0 * y0, y1e2 = y1 * y1, z0e2 = z0 * z0, z1e2 = z1 * z1;
  T D000 = sqrt(x0e2 + y0e2 + z0e2), D100 = sqrt(x1e2 + y0e2 + z0e2), D010 = sqrt(x0e2 + y1e2 + z0e2), D110 = sqrt(x1e2 + y1e2 + z0e2);
  T D001 = sqrt(x0e2 + y0e2 + z1e2), D101 = sqrt(x1e2 + y0e2 + z1e2), D011 = sqrt(x0e2 + y1e2 + z1e2), D111 = sqrt(x1e2 + y1e2 + z1e2);
  T T0x = atan4(y0 * z0 / (x0 * D000), -y0 * z1 / (x0 * D001), -y1 * z0 / (x0 * D010), y1 * z1 / (x0 * D011));
  T T1x = atan4(-y0 * z0 / (x1 * D100), y0 * z1 / (x1 * D101), y1 * z0 / (x1 * D110), -y1 * z1 / (x1 * D111));
  T T0y = atan4(x0 * z0 / (y0 * D000), -x0 * z1 / (y0 * D001), -x1 * z0 / (y0 * D100), x1 * z1 / (y0 * D101));
  T T1y = atan4(-x0 * z0 / (y1 * D010), x0 * z1 / (y1 * D011), x1 * z0 / (y1 * D110), -x1 * z1 / (y1 * D111));
  T T0z = atan4(x0 * y0 / (z0 * D000), -x1 * y0 / (z0 * D100), -x0 * y1 / (z0 * D010), x1 * y1 / (z0 * D110));
  T T1z = atan4(-x0 * y0 / (z1 * D001), x1 * y0 / (z1 * D101), x0 * y1 / (z1 * D011), -x1 * y1 / (z1 * D111));
  T R000 = 10. * abs_rand(g, D000), R010 = 10. * abs_rand(g, D010), R001 = 10. * abs_rand(g, D001), R011 = 10. * abs_rand(g, D011);
  T R100 = 10. * abs_rand(g, D100), R110 = 10. * abs_rand(g, D110), R101 = 10. * abs_rand(g, D101), R111 = 10. * abs_rand(g, D111);
  T z0pD100 = z0 + D100; if (z0pD100 < R100) z0pD100 = 0.5 * (x1e2 + y0e2) / fabs(z0);
  T z1pD101 = z1 + D101; if (z1pD101 < R101) z1pD101 = 0.5 * (x1e2 + y0e2) / fabs(z1);
  T z1pD001 = z1 + D001; if (z1pD001 < R001) z1pD001 = 0.5 * (x0e2 + y0e2) / fabs(z1);
  T z0pD000 = z0 + D000; if (z0pD000 < R000) z0pD000 = 0.5 * (x0e2 + y0e2) / fabs(z0);
  T z0pD010 = z0 + D010; if (z0pD010 < R010) z0pD010 = 0.5 * (x0e2 + y1e2) / fabs(z0);
  T z1pD011 = z1 + D011; if (z1pD011 < R011) z1pD011 = 0.5 * (x0e2 + y1e2) / fabs(z1);
  T z1pD111 = z1 + D111; if (z1pD111 < R111) z1pD111 = 0.5 * (x1e2 + y1e2) / fabs(z1);
  T z0pD110 = z0 + D110; if (z0pD110 < R110) z0pD110 = 0.5 * (x1e2 + y1e2) / fabs(z0);
  T y0pD100 = y0 + D100; if (y0pD100 < R100) y0pD100 = 0.5 * (x1e2 + z0e2) / fabs(y0);
  T y1pD110 = y1 + D110; if (y1pD110 < R110) y1pD110 = 0.5 * (x1e2 + z0e2) / fabs(y1);
  T y1pD010 = y1 + D010; if (y1pD010 < R010) y1pD010 = 0.5 * (x0e2 + z0e2) / fabs(y1);
  T y0pD000 = y0 + D000; if (y0pD000 < R000) y0pD000 = 0.5 * (x0e2 + z0e2) / fabs(y0);
  T y0pD001 = y0 + D001; if (y0pD001 < R001) y0pD001 = 0.5 * (x0e2 + z1e2) / fabs(y0);
  T y1pD011 = y1 + D011; if (y1pD011 < R011) y1pD011 = 0.5 * (x0e2 + z1e2) / fabs(y1);
  T y1pD111 = y1 + D111; if (y1pD111 < R111) y1pD111 = 0.5 * (x1e2 + z1e2) / fabs(y1);
  T y0pD101 = y0 + D101; if (y0pD101 < R101) y0pD101 = 0.5 * (x1e2 + z1e2) / fabs(y0);
  T x0pD010 = x0 + D010; if (x0pD010 < R010) x0pD010 = 0.5 * (y1e2 + z0e2) / fabs(x0);
  T x1pD110 = x1 + D110; if (x1pD110 < R110) x1pD110 = 0.5 * (y1e2 + z0e2) / fabs(x1);
  T x1pD100 = x1 + D100; if (x1pD100 < R100) x1pD100 = 0.5 * (y0e2 + z0e2) / fabs(x1);
  T x0pD000 = x0 + D000; if (x0pD000 < R000) x0pD000 = 0.5 * (y0e2 + z0e2) / fabs(x0);
  T x0pD001 = x0 + D001; if (x0pD001 < R001) x0pD001 = 0.5 * (y0e2 + z1e2) / fabs(x0);
  T x1pD101 = x1 + D101; if (x1pD101 < R101) x1pD101 = 0.5 * (y0e2 + z1e2) / fabs(x1);
  T x1pD111 = x1 + D111; if (x1pD111 < R111) x1pD111 = 0.5 * (y1e2 + z1e2) / fabs(x1);
  T x0pD011 = x0 + D011; if (x0pD011 < R011) x0pD011 = 0.5 * (y1e2 + z1e2) / fabs(x0);
  T lza = log(z0pD100 / z1pD101), lzb = log(z1pD001 / z0pD000), lzc = log(z0pD010 / z1pD011), lzd = log(z1pD111 / z0pD110);
  T lya = log(y0pD100 / y1pD110), lyb = log(y1pD010 / y0pD000), lyc = log(y0pD001 / y1pD011), lyd = log(y1pD111 / y0pD101);
  T lxa = log(x0pD010 / x1pD110), lxb = log(x1pD100 / x0pD000), lxc = log(x0pD001 / x1pD101), lxd = log(x1pD111 / x0pD011);
  V3<T> bv = mk3<T>(x0 * T0x + x1 * T1x + y0 * (lza + lzb) + y1 * (lzc + lzd) + z0 * (lya + lyb) + z1 * (lyc + lyd),
                    y0 * T0y + y1 * T1y + x0 * (lzc + lzb) + x1 * (lza + lzd) + z0 * (lxa + lxb) + z1 * (lxc + lxd),
                    z0 * T0z + z1 * T1z + y0 * (lxc + lxb) + y1 * (lxa + lxd) + x0 * (lyc + lyb) + x1 * (lya + lyd));
  const T c = 0.0001;
  return mk3<T>(c * (J.y * bv.z - J.z * bv.y), c * (J.z * bv.x - J.x * bv.z), c * (J.x * bv.y - J.y * bv.x));
}

// Planar polygon face integrals (Sx,Sy,Sz) at a point given in the face frame
// (px,py,pz), vertices (counter-clockwise) in shared or global memory.
// Returns 1 when the point is on the inner side of the face plane (z > 0).
// radTPolygon::B_comp, radplnr2.cpp:29-388 (B/H/PreRelax paths).
template <typename T, typename VP>
__device__ __forceinline__ int polygon_S(const VP *vtx, int nv, T coordz, T cx, T cy, V3<T> P,
                                          const Guard &g, T &Sx_o, T &Sy_o, T &Sz_o)
{
  const T Max_k = T(1.E+09);
  T arx = abs_rand(g, T(vtx[0]) - cx), ary = abs_rand(g, T(vtx[1]) - cy);
  T arz = abs_rand(g, coordz);
  if (arz < arx) arz = arx;
  if (arz < ary) arz = ary;
  T relr = abs_rand(g, T(1));
  T z = coordz - P.z;
  if (z == T(0)) z = arz;
  T ze2 = z * z;
  T f2x = T(vtx[0]) - P.x, f2y = T(vtx[1]) - P.y;
  T addx = -P.x, addy = -P.y;
  T x1 = f2x, y1 = f2y;
  if (x1 == T(0)) { x1 = arx; f2x += arx; addx += arx; }
  if (y1 == T(0)) { y1 = ary; f2y += ary; addy += ary; }
  T x1e2 = x1 * x1;
  T Sx = 0, Sy = 0, sum_atan = 0, arg_logs2 = 1;
  const T MaxRel = T(1.E-07);
  const T tiny = sizeof(T) == 8 ? T(1e-50) : T(1e-30);
  for (int i = 0; i < nv; i++) {
    T x2, y2;
    if (i != nv - 1) { x2 = T(vtx[2 * (i + 1)]) + addx; y2 = T(vtx[2 * (i + 1) + 1]) + addy; }
    else { x2 = f2x; y2 = f2y; }
    if (x2 == T(0)) { x2 = arx; f2x += arx; addx += arx; }
    if (y2 == T(0)) { y2 = ary; f2y += ary; addy += ary; }
    T x2e2 = x2 * x2;
    T x2mx1 = x2 - x1, y2my1 = y2 - y1;
    if (fabsT(x2mx1) * Max_k > fabsT(y2my1)) {
      T k = y2my1 / x2mx1;
      T b = y1 - k * x1;
      if (b == T(0)) {
        b = ary; y1 += ary; y2my1 -= ary; k = y2my1 / x2mx1;
        f2y += ary; addy += ary;
      }
      T bk = b * k, ke2 = k * k, be2 = b * b, twob = T(2) * b;
      T ke2p1 = ke2 + T(1);
      if (ke2p1 == T(0)) ke2p1 = relr;
      T sqrtke2p1 = sqrtT(ke2p1);
      T kx1 = k * x1, kx2 = k * x2;
      T bpkx1 = y1, bpkx2 = y2;
      T bpkx1e2 = bpkx1 * bpkx1, bpkx2e2 = bpkx2 * bpkx2;
      T kx1mb = -b + kx1, kx2mb = -b + kx2;
      T R1 = sqrtT(x1e2 + bpkx1e2 + ze2), R2 = sqrtT(x2e2 + bpkx2e2 + ze2);
      T x1e2pze2 = x1e2 + ze2, x2e2pze2 = x2e2 + ze2;
      T bkpx1pke2x1 = bk + ke2p1 * x1, bkpx2pke2x2 = bk + ke2p1 * x2;
      T kze2 = k * ze2, ke2ze2 = k * kze2;
      T ke2ze2mbe2 = ke2ze2 - be2, ke2ze2pbe2 = ke2ze2 + be2;
      T bx1 = b * x1, bx2 = b * x2;
      T R1pbpkx1 = bpkx1 + R1, R2pbpkx2 = bpkx2 + R2;
      T arR2 = T(100) * abs_rand(g, R2), arR1 = T(100) * abs_rand(g, R1);
      T mR1 = MaxRel * R1, mR2 = MaxRel * R2;
      if (arR1 > mR1) arR1 = mR1;
      if (arR2 > mR2) arR2 = mR2;
      if ((R1pbpkx1 < arR1) && (R1 > T(100) * arR1) && ((x1e2 + ze2) < bpkx1e2 * MaxRel))
        R1pbpkx1 = T(0.5) * (x1e2 + ze2) / fabsT(bpkx1);
      if ((R2pbpkx2 < arR2) && (R2 > T(100) * arR2) && ((x2e2 + ze2) < bpkx2e2 * MaxRel))
        R2pbpkx2 = T(0.5) * (x2e2 + ze2) / fabsT(bpkx2);
      T A1 = -(ke2ze2pbe2 * (bx1 + kze2) * R1pbpkx1 + kze2 * twob * x1e2pze2);
      T A2 = (ke2ze2pbe2 * kx1mb * R1pbpkx1 + ke2ze2mbe2 * x1e2pze2) * z;
      T A3 = ke2ze2pbe2 * (bx2 + kze2) * R2pbpkx2 + kze2 * twob * x2e2pze2;
      T A4 = (ke2ze2pbe2 * kx2mb * R2pbpkx2 + ke2ze2mbe2 * x2e2pze2) * z;
      sum_atan += atan2T(A1 * A4 + A3 * A2, A2 * A4 - A1 * A3);
      T L1 = bkpx1pke2x1 / sqrtke2p1 + R1, L2 = bkpx2pke2x2 / sqrtke2p1 + R2;
      T be2pze2 = be2 + ze2;
      if ((L1 < arR1) && (R1 > T(100) * arR1) && ((be2pze2 + T(2) * bk * x1) < x1e2 * ke2p1 * MaxRel))
        L1 = T(0.5) * be2pze2 / (fabsT(x1) * sqrtke2p1);
      if ((L2 < arR2) && (R2 > T(100) * arR2) && ((be2pze2 + T(2) * bk * x2) < x2e2 * ke2p1 * MaxRel))
        L2 = T(0.5) * be2pze2 / (fabsT(x2) * sqrtke2p1);
      if (L1 == T(0)) L1 = tiny;
      if (L2 == T(0)) L2 = tiny;
      T sl1 = logT(L2 / L1) / sqrtke2p1;
      if (R1pbpkx1 == T(0)) R1pbpkx1 = tiny;
      arg_logs2 *= (R2pbpkx2 / R1pbpkx1);
      Sx += -k * sl1;
      Sy += sl1;
    }
    x1 = x2; y1 = y2; x1e2 = x2e2;
  }
  if (arg_logs2 <= T(0)) arg_logs2 = tiny;
  Sx += logT(arg_logs2);
  Sx_o = Sx; Sy_o = Sy; Sz_o = sum_atan;
  return z > T(0);
}

// Arc current field at q (object frame), record a = [cx cy cz rmin rmax
// phimin phimax h j nseg]; trapezoid rule in phi with nseg sectors
// (radTArcCur::B_compWithTrapeth, radarccu.cpp:30-236).
__device__ __forceinline__ V3<double> arc_field(const double *a, V3<double> P)
{
  const double Pi = 3.141592653589793238, ZeroTol = 1.E-10, RZ = 1.E-07, SP = 1.E-10;
  double px = P.x - a[0], py = P.y - a[1], pz = P.z - a[2];
  double Rmin = a[3], Rmax = a[4], Phimin = a[5], Phimax = a[6], Height = a[7], Jaz = a[8];
  int nsec = (int)a[9];
  double r = sqrt(px * px + py * py + SP);
  double phi = (py < 0) ? (2 * Pi - acos(px / r)) : acos(px / r);
  double z1 = -Height / 2. - pz, z2 = z1 + Height;
  double z1z1 = z1 * z1, z2z2 = z2 * z2, rr = r * r, r1r1 = Rmin * Rmin, r2r2 = Rmax * Rmax;
  double a11 = rr + r1r1 + z1z1, a12 = rr + r1r1 + z2z2, a21 = rr + r2r2 + z1z1, a22 = rr + r2r2 + z2z2;
  double two_rr1 = 2. * r * Rmin, two_rr2 = 2. * r * Rmax;
  int npoi = nsec + 1;
  double step = (Phimax - Phimin + SP) / (npoi - 1);
  double dphi = Phimin - phi + SP;
  double SBx = 0., SBy = 0., SBz = 0.;
  for (int i = 0; i < npoi; i++) {
    double sdp, cdp;
    sincos(dphi, &sdp, &cdp);
    double asdp = fabs(sdp);
    double t1 = two_rr1 * cdp, t2 = two_rr2 * cdp;
    double b11 = fabs(a11 - t1); if (b11 < ZeroTol) b11 = ZeroTol;
    double D11 = sqrt(b11), D12 = sqrt(fabs(a12 - t1));
    double b21 = fabs(a21 - t2); if (b21 < ZeroTol) b21 = ZeroTol;
    double D21 = sqrt(b21), D22 = sqrt(fabs(a22 - t2));
    double rCos = r * cdp, r1m = Rmin - rCos, r2m = Rmax - rCos;
    double d11 = D11 * RZ, d12 = D12 * RZ, d21 = D21 * RZ, d22 = D22 * RZ;
    double zz = z1z1 + rr * asdp * asdp;
    double r1me2 = r1m * r1m, r2me2 = r2m * r2m;
    double u11 = r1m + D11; if ((fabs(u11) < d11) && (zz < r1me2 * RZ)) u11 = 0.5 * zz / fabs(r1m);
    double u12 = r1m + D12; if ((fabs(u12) < d12) && (zz < r1me2 * RZ)) u12 = 0.5 * zz / fabs(r1m);
    double u21 = r2m + D21; if ((fabs(u21) < d21) && (zz < r2me2 * RZ)) u21 = 0.5 * zz / fabs(r2m);
    double u22 = r2m + D22; if ((fabs(u22) < d22) && (zz < r2me2 * RZ)) u22 = 0.5 * zz / fabs(r2m);
    double ln1 = log(u11 / u21), ln2 = log(u22 / u12);
    double rAbsSin = r * asdp;
    double q1 = fabs(r1m) / rAbsSin, q2 = fabs(r2m) / rAbsSin;
    double pm1 = 0., pm2 = 0.;
    double at1 = atan(trans_atans(z2 * q1 / D12, -z1 * q1 / D11, pm1)) + Pi * pm1;
    double at2 = atan(trans_atans(z1 * q2 / D21, -z2 * q2 / D22, pm2)) + Pi * pm2;
    double Buf = rAbsSin * ((r1m < 0 ? -1. : 1.) * at1 + (r2m < 0 ? -1. : 1.) * at2) + z1 * ln1 + z2 * ln2;
    double w11 = z1 + D11, s1 = rr + r1r1 - t1;
    double z1t = z1z1 * RZ, z2t = z2z2 * RZ;
    if ((fabs(w11) < d11) && (s1 < z1t)) w11 = 0.5 * s1 / fabs(z1);
    double w21 = z1 + D21, s2 = rr + r2r2 - t2;
    if ((fabs(w21) < d21) && (s2 < z1t)) w21 = 0.5 * s2 / fabs(z1);
    double w12 = z2 + D12;
    if ((fabs(w12) < d12) && (s1 < z2t)) w12 = 0.5 * s1 / fabs(z2);
    double w22 = z2 + D22;
    if ((fabs(w22) < d22) && (s2 < z2t)) w22 = 0.5 * s2 / fabs(z2);
    double php = dphi + phi, sph, cph;
    sincos(php, &sph, &cph);
    double FBxy = D11 - D21 + D22 - D12 + rCos * (ln1 + ln2);
    double FBz = Buf - rCos * log((w11 / w12) * (w22 / w21));
    double wgt = (i == 0 || i == npoi - 1) ? 0.5 : 1.0;
    SBx += wgt * cph * FBxy;
    SBy += wgt * sph * FBxy;
    SBz += wgt * FBz;
    dphi += step;
  }
  double f = 0.0001 * Jaz * step;
  return mk3<double>(f * SBx, f * SBy, f * SBz);
}

// ---------------------------------------------------------------------------
// Polyhedron, vertex/edge form.
//
// The field of a uniformly magnetized polyhedron is that of the surface
// charge sigma_f = M.n_f on its faces:
//   H(q) = 1/(4 pi) sum_f sigma_f I_f,   I_f = int_f (q - r')/|q - r'|^3 dS'
// and for a planar face   I_f = Omega_f n_f + sum_{e in f} nu_{e,f} L_e
// with Omega_f the signed solid angle of the face seen from q (sign of
// n_f.(q - face)), nu_{e,f} the outward in-plane normal of edge e in face f
// and L_e = int_e dl/|q - r'| = log1p(l (Ra + Rb + l) / D),
// D = Ra Rb + ra.rb  (evaluated as |ra x rb|^2 / (Ra Rb - ra.rb) when ra.rb < 0
// to avoid cancellation).  Solid angles per triangle by the Van Oosterom-
// Strackee formula, with the triple product taken from the face's fixed edge
// cross product (ra . m_t, m_t = (vb - va) x (vc - va)) so it does not cancel
// for distant points.  Per tetrahedron this is 4 sqrt, 6 log1p, 4 atan2,
// against 12 edge terms (24 sqrt, 24 log, 12 atan2) of the face-by-face form
// radplnr2.cpp:29-388; both are exact, so they agree to rounding away from
// the edges themselves.
//
// Topology record per polyhedron (built on the host from the face frames):
//   tinfo  = {v0, nv, e0, ne},  tinfo2 = {t0, nt, f0, nf}
//   tv[v]  vertex (object frame)          te[e] = {a, b} (local), tel[e] = l
//   tt[t]  = {a, b, c, f} (local), ttm[t] = m_t
//   tfn[f] = n_f
// Field mode adds per face a_f = sigma_f n_f and per edge g_e = sum_f sigma_f nu_{e,f};
// tensor mode uses per edge G_e = sum_f nu_{e,f} n_f^T (9 doubles).
struct TopoView {
  const int4 *tinfo, *tinfo2;
  const double *tv;     // [V*3]
  const int2 *te;       // [E]
  const double *tel;    // [E]
  const double *teg;    // [E*3] field coefficients g_e (or null)
  const double *teG;    // [E*9] tensor coefficients G_e (or null)
  const int4 *tt;       // [T]
  const double *ttm;    // [T*3]
  const double *tfn;    // [F*3]
  const double *tfa;    // [F*3] field coefficients a_f (or null)
};

constexpr int POLY_NV_FAST = 8;  // vertices handled in registers

template <typename T>
__device__ __forceinline__ T log1pT(T x);
template <> __device__ __forceinline__ double log1pT<double>(double x) { return log1p(x); }
template <> __device__ __forceinline__ float log1pT<float>(float x) { return log1pf(x); }

// Solid angles and edge logs of polyhedron p at q (object frame).
// Accumulates H (field mode, a_f / g_e set) or the tensor Q (tensor mode).
// Returns 1 when q is inside.  T = arithmetic type after the FP64 vertex shift.
template <typename T, bool TENSOR>
__device__ __forceinline__ int poly_fast(const TopoView &tp, int p, V3<double> q, double *out)
{
  const double C = 1.0 / (4.0 * 3.141592653589793238);
  int4 i1 = __ldg(tp.tinfo + p), i2 = __ldg(tp.tinfo2 + p);
  const int v0 = i1.x, nv = i1.y, e0 = i1.z, ne = i1.w, t0 = i2.x, nt = i2.y, f0 = i2.z, nf = i2.w;
  T rx[POLY_NV_FAST], ry[POLY_NV_FAST], rz[POLY_NV_FAST], R[POLY_NV_FAST];
#pragma unroll
  for (int k = 0; k < POLY_NV_FAST; k++) {
    if (k < nv) {
      const double *v = tp.tv + 3 * (size_t)(v0 + k);
      rx[k] = T(__ldg(v) - q.x); ry[k] = T(__ldg(v + 1) - q.y); rz[k] = T(__ldg(v + 2) - q.z);
      R[k] = sqrtT(rx[k] * rx[k] + ry[k] * ry[k] + rz[k] * rz[k]);
    } else {
      rx[k] = ry[k] = rz[k] = R[k] = T(0);
    }
  }
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = 0.0;
  // edges
  for (int e = e0; e < e0 + ne; e++) {
    int2 ab = __ldg(tp.te + e);
    T l = T(__ldg(tp.tel + e));
    T ax = T(0), ay = T(0), az = T(0), Ra = T(0), bx = T(0), by = T(0), bz = T(0), Rb = T(0);
#pragma unroll
    for (int k = 0; k < POLY_NV_FAST; k++) {
      if (k == ab.x) { ax = rx[k]; ay = ry[k]; az = rz[k]; Ra = R[k]; }
      if (k == ab.y) { bx = rx[k]; by = ry[k]; bz = rz[k]; Rb = R[k]; }
    }
    T s = ax * bx + ay * by + az * bz;
    T D;
    if (s >= T(0)) D = Ra * Rb + s;
    else {
      T cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
      D = (cx * cx + cy * cy + cz * cz) / (Ra * Rb - s);
    }
    T L = log1pT<T>(l * (Ra + Rb + l) / D);
    double Ld = (double)L;
    if (TENSOR) {
      const double *G = tp.teG + 9 * (size_t)e;
#pragma unroll
      for (int k = 0; k < 9; k++) acc[k] += Ld * __ldg(G + k);
    } else {
      const double *g = tp.teg + 3 * (size_t)e;
      acc[0] += Ld * __ldg(g); acc[1] += Ld * __ldg(g + 1); acc[2] += Ld * __ldg(g + 2);
    }
  }
  // triangles -> face solid angles
  double omega_tot = 0.0;
  int fcur = -1;
  double om = 0.0;
  for (int t = t0; t <= t0 + nt; t++) {
    int4 tr = (t < t0 + nt) ? __ldg(tp.tt + t) : make_int4(0, 0, 0, -1);
    if (tr.w != fcur) {
      if (fcur >= 0) {  // flush face fcur
        const double *n = tp.tfn + 3 * (size_t)(f0 + fcur);
        if (TENSOR) {
          double n0 = __ldg(n), n1 = __ldg(n + 1), n2 = __ldg(n + 2);
          acc[0] += om * n0 * n0; acc[1] += om * n0 * n1; acc[2] += om * n0 * n2;
          acc[3] += om * n1 * n0; acc[4] += om * n1 * n1; acc[5] += om * n1 * n2;
          acc[6] += om * n2 * n0; acc[7] += om * n2 * n1; acc[8] += om * n2 * n2;
        } else {
          const double *a = tp.tfa + 3 * (size_t)(f0 + fcur);
          acc[0] += om * __ldg(a); acc[1] += om * __ldg(a + 1); acc[2] += om * __ldg(a + 2);
        }
        omega_tot += om;
      }
      fcur = tr.w;
      om = 0.0;
      if (t == t0 + nt) break;
    }
    T xa = 0, ya = 0, za = 0, Ra = 0, xb = 0, yb = 0, zb = 0, Rb = 0, xc = 0, yc = 0, zc = 0, Rc = 0;
#pragma unroll
    for (int k = 0; k < POLY_NV_FAST; k++) {
      if (k == tr.x) { xa = rx[k]; ya = ry[k]; za = rz[k]; Ra = R[k]; }
      if (k == tr.y) { xb = rx[k]; yb = ry[k]; zb = rz[k]; Rb = R[k]; }
      if (k == tr.z) { xc = rx[k]; yc = ry[k]; zc = rz[k]; Rc = R[k]; }
    }
    const double *m = tp.ttm + 3 * (size_t)t;
    T num = xa * T(__ldg(m)) + ya * T(__ldg(m + 1)) + za * T(__ldg(m + 2));
    T den = Ra * Rb * Rc + (xa * xb + ya * yb + za * zb) * Rc + (xa * xc + ya * yc + za * zc) * Rb +
            (xb * xc + yb * yc + zb * zc) * Ra;
    om += 2.0 * (double)atan2T(-num, den);
  }
#pragma unroll
  for (int k = 0; k < (TENSOR ? 9 : 3); k++) out[k] = C * acc[k];
  return omega_tot < -6.283185307179586;
}

// ---------------------------------------------------------------------------
// Tetrahedron, vertex/edge form with a fixed topology: edges (01 02 03 12 13
// 23), faces opposite each vertex, the face cross products m_t oriented
// outward on the host.  No index selection in the inner loop, everything
// unrolled.  Record (object frame), TET_REC_FIELD doubles:
//   [0,12) vertices  [12,18) edge lengths  [18,30) m_t  [30,42) a_f = sigma_f n_f
//   [42,60) g_e = sum_f sigma_f nu_{e,f}
// TET_REC_TENSOR doubles: [0,30) as above, [30,42) n_f, [42,96) G_e (3x3 each).
constexpr int TET_REC_FIELD = 60, TET_REC_TENSOR = 96;
__host__ __device__ constexpr int tet_edge_a(int e) { return e < 3 ? 0 : (e < 5 ? 1 : 2); }
__host__ __device__ constexpr int tet_edge_b(int e) { return e == 0 ? 1 : e == 1 ? 2 : e == 2 ? 3 : e == 3 ? 2 : 3; }
// face f (opposite vertex f) = triangle (a, b, c)
__host__ __device__ constexpr int tet_face_a(int f) { return f == 0 ? 1 : 0; }
__host__ __device__ constexpr int tet_face_b(int f) { return f == 0 ? 2 : (f == 1 ? 2 : 1); }
__host__ __device__ constexpr int tet_face_c(int f) { return f == 3 ? 2 : 3; }
// index of the vertex pair (i < j) in the edge list
__host__ __device__ constexpr int tet_pair(int i, int j) { return i == 0 ? j - 1 : (i == 1 ? j + 1 : 5); }

template <bool SMEM>
__device__ __forceinline__ double rd_rec(const double *p)
{
  if (SMEM) return *p;
  return __ldg(p);
}

// SMEM: the record lives in shared memory (plain loads instead of __ldg).
// recf (T = float, optional): the edge lengths (6) and face normals (12) of
// the record already rounded to float, so that a pair reads them without a
// conversion each (the same values as T(record entry)).
template <typename T, bool TENSOR, bool SMEM = false>
__device__ __forceinline__ int tet_fast(const double *__restrict__ rec, V3<double> q, double *out,
                                        const float *__restrict__ recf = nullptr)
{
  const bool fl = sizeof(T) == 4 && recf != nullptr;
  const double C = 1.0 / (4.0 * 3.141592653589793238);
  T rx[4], ry[4], rz[4], R[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    rx[k] = T(rd_rec<SMEM>(rec + 3 * k) - q.x);
    ry[k] = T(rd_rec<SMEM>(rec + 3 * k + 1) - q.y);
    rz[k] = T(rd_rec<SMEM>(rec + 3 * k + 2) - q.z);
    R[k] = sqrtT(rx[k] * rx[k] + ry[k] * ry[k] + rz[k] * rz[k]);
  }
  T d[6];  // r_i . r_j per edge
#pragma unroll
  for (int e = 0; e < 6; e++) {
    const int a = tet_edge_a(e), b = tet_edge_b(e);
    d[e] = rx[a] * rx[b] + ry[a] * ry[b] + rz[a] * rz[b];
  }
  double acc[TENSOR ? 9 : 3];
#pragma unroll
  for (int k = 0; k < (TENSOR ? 9 : 3); k++) acc[k] = 0.0;
#pragma unroll
  for (int e = 0; e < 6; e++) {
    const int a = tet_edge_a(e), b = tet_edge_b(e);
    T l = fl ? T(recf[e]) : T(rd_rec<SMEM>(rec + 12 + e));
    T D;
    if (d[e] >= T(0)) D = R[a] * R[b] + d[e];
    else {
      T cx = ry[a] * rz[b] - rz[a] * ry[b], cy = rz[a] * rx[b] - rx[a] * rz[b], cz = rx[a] * ry[b] - ry[a] * rx[b];
      D = (cx * cx + cy * cy + cz * cz) / (R[a] * R[b] - d[e]);
    }
    double L = (double)log1pT<T>(l * (R[a] + R[b] + l) / D);
    if (TENSOR) {
#pragma unroll
      for (int k = 0; k < 9; k++) acc[k] += L * rd_rec<SMEM>(rec + 42 + 9 * e + k);
    } else {
#pragma unroll
      for (int k = 0; k < 3; k++) acc[k] += L * rd_rec<SMEM>(rec + 42 + 3 * e + k);
    }
  }
  double omega_tot = 0.0;
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const int a = tet_face_a(f), b = tet_face_b(f), c = tet_face_c(f);
    const T m0 = fl ? T(recf[6 + 3 * f]) : T(rd_rec<SMEM>(rec + 18 + 3 * f));
    const T m1 = fl ? T(recf[7 + 3 * f]) : T(rd_rec<SMEM>(rec + 19 + 3 * f));
    const T m2 = fl ? T(recf[8 + 3 * f]) : T(rd_rec<SMEM>(rec + 20 + 3 * f));
    T num = rx[a] * m0 + ry[a] * m1 + rz[a] * m2;
    T den = R[a] * R[b] * R[c] + d[tet_pair(a, b)] * R[c] + d[tet_pair(a, c)] * R[b] + d[tet_pair(b, c)] * R[a];
    double om = 2.0 * (double)atan2T(-num, den);
    omega_tot += om;
    if (TENSOR) {
      double n0 = rd_rec<SMEM>(rec + 30 + 3 * f), n1 = rd_rec<SMEM>(rec + 31 + 3 * f), n2 = rd_rec<SMEM>(rec + 32 + 3 * f);
      acc[0] += om * n0 * n0; acc[1] += om * n0 * n1; acc[2] += om * n0 * n2;
      acc[3] += om * n1 * n0; acc[4] += om * n1 * n1; acc[5] += om * n1 * n2;
      acc[6] += om * n2 * n0; acc[7] += om * n2 * n1; acc[8] += om * n2 * n2;
    } else {
#pragma unroll
      for (int k = 0; k < 3; k++) acc[k] += om * rd_rec<SMEM>(rec + 30 + 3 * f + k);
    }
  }
#pragma unroll
  for (int k = 0; k < (TENSOR ? 9 : 3); k++) out[k] = C * acc[k];
  return omega_tot < -6.283185307179586;
}

}  // namespace rb
