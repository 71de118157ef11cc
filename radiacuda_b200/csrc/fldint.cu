// fldint.cu -- field integrals along straight lines (rad.FldInt).
//
// The reference integrates element by element (radTg3d::B_genComp,
// cpp/src/core/radg3d.h:907-921): a finite integral is a Newton 3/8 sum whose
// point count doubles until two successive sums differ by less than PrcBInt
// (radTg3d::B_intCompFinNum, cpp/src/core/radg3d.cpp:258-342); the infinite
// one is analytic for blocks (radTRecMag::B_intComp, radrec.cpp:468) and
// polygons (radTPolygon::B_intComp, radplnr2.cpp:390), numeric for arcs
// (radarccu.cpp:461-700) and zero for uniform background fields
// (radarccu.h:306-316).  The sum of those integrals is the integral of the
// total field, which is what is computed here: one adaptive Gauss-Kronrod
// quadrature over the line whose field values come from the device field
// kernels, every refinement level one batched launch over all open panels.
//
// Panel ends are placed where the line enters and leaves each element (the
// field of a magnetized body jumps there), at the projections of elements
// close to the line, and (infinite lines) at the ends of the span covered by
// the geometry, beyond which the two tails are mapped onto [0, 1).
#include <math.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <vector>

#include "internal.cuh"

namespace rb {
namespace {

// 15-point Gauss-Kronrod rule on [-1, 1] with its embedded 7-point Gauss rule
// (Kronrod's extension of Gauss-Legendre; values as tabulated in Piessens et
// al., QUADPACK, Springer 1983).  XGK[1], XGK[3], XGK[5], XGK[7] are the
// Gauss nodes, weighted by WG.
const double XGK[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                       0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                       0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                       0.207784955007898467600689403773245, 0.0};
const double WGK[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                       0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                       0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                       0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
const double WG[4] = {0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                      0.381830050505118944950369775488975, 0.417959183673469387755102040816327};
constexpr int GK_N = 15;

struct Rule {
  double s[GK_N], wk[GK_N], wg[GK_N];
  Rule()
  {
    for (int k = 0; k < 8; k++) {
      double g = (k & 1) ? WG[k >> 1] : 0.0;
      s[k] = -XGK[k];
      wk[k] = WGK[k];
      wg[k] = g;
      s[14 - k] = XGK[k];
      wk[14 - k] = WGK[k];
      wg[14 - k] = g;
    }
  }
};

// Panel of one of three variables: seg 0 the line parameter t (mm from P1
// along u); seg 1 the upper tail t = tb + R x/(1-x); seg 2 the lower tail
// t = ta - R x/(1-x); x in [0, 1].
struct Panel {
  double a, b;
  int seg;
  int evaluated;
  double val[6];
  double err;
  double perr;  // error estimate of the panel this one was split from (0: initial)
  int stall;    // successive splits that did not reduce the error estimate
};

struct LineGeom {
  double p1[3], u[3], len;
  double ta = 0, tb = 0, R = 1;  // span of the geometry along the line, tail scale
  bool any = false;              // some element contributes
  std::vector<double> breaks;    // line parameters of entries, exits and projections
  double amax = 0;               // largest element radius
  double far = 0;                // the tails start this far beyond [ta, tb]
  // far-field model: point dipoles {lab position, mu0 m (T mm^3)}, one per
  // magnetized element image, plus one for all currents together
  std::vector<double> dip;
  double jm[3] = {0, 0, 0}, jc[3] = {0, 0, 0}, jk[3] = {0, 0, 0};  // current moment, centre and net current sums
  int nj = 0;
};

constexpr double MU0_MM = 4e-4 * M_PI;  // mu0 in T mm / A

inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// [t0, t1] of the line a + t b inside the box |p - c| <= h (componentwise)
bool clip_box(const double *a, const double *b, const double *c, const double *h, double &t0, double &t1)
{
  t0 = -INFINITY;
  t1 = INFINITY;
  for (int k = 0; k < 3; k++) {
    double lo = c[k] - h[k] - a[k], hi = c[k] + h[k] - a[k];
    if (fabs(b[k]) < 1e-300) {
      if (lo > 0 || hi < 0) return false;
      continue;
    }
    double x0 = lo / b[k], x1 = hi / b[k];
    if (x0 > x1) std::swap(x0, x1);
    t0 = std::max(t0, x0);
    t1 = std::min(t1, x1);
  }
  return t1 > t0;
}

// object-frame line a + t b of image record T (P_obj = M^-1 (P - V))
void obj_line(const double *T, const LineGeom &L, double *a, double *b)
{
  double d[3] = {L.p1[0] - T[9], L.p1[1] - T[10], L.p1[2] - T[11]};
  for (int r = 0; r < 3; r++) {
    a[r] = T[3 * r] * d[0] + T[3 * r + 1] * d[1] + T[3 * r + 2] * d[2];
    b[r] = T[3 * r] * L.u[0] + T[3 * r + 1] * L.u[1] + T[3 * r + 2] * L.u[2];
  }
}

// lab position of object-frame point c under image T (P = (sM) c / s + V)
void lab_point(const double *T, const double *c, double *out)
{
  for (int r = 0; r < 3; r++)
    out[r] = (T[12 + 3 * r] * c[0] + T[13 + 3 * r] * c[1] + T[14 + 3 * r] * c[2]) / T[21] + T[9 + r];
}

// records the span [proj - rad, proj + rad] of one element image
void add_extent(LineGeom &L, const double *T, const double *c, double rad)
{
  double C[3];
  lab_point(T, c, C);
  double d[3] = {C[0] - L.p1[0], C[1] - L.p1[1], C[2] - L.p1[2]};
  double proj = dot3(d, L.u);
  if (!L.any) {
    L.ta = proj - rad;
    L.tb = proj + rad;
    L.R = rad;
  } else {
    L.ta = std::min(L.ta, proj - rad);
    L.tb = std::max(L.tb, proj + rad);
    L.R = std::max(L.R, rad);
  }
  L.any = true;
  L.amax = std::max(L.amax, rad);
}

// point dipole of magnetic moment mv (M V, T mm^3) at object-frame point c
void add_dipole(LineGeom &L, const double *T, const double *c, const double *mv)
{
  if (mv[0] == 0 && mv[1] == 0 && mv[2] == 0) return;
  double C[3];
  lab_point(T, c, C);
  for (int r = 0; r < 3; r++) L.dip.push_back(C[r]);
  for (int r = 0; r < 3; r++) L.dip.push_back(T[12 + 3 * r] * mv[0] + T[13 + 3 * r] * mv[1] + T[14 + 3 * r] * mv[2]);
}

// current element at object-frame point c: own moment mown (1/2 int (r - c)
// x J dV, A mm^2) and net current K (int J dV, A mm).  Lab images: the
// moment maps like the field (s M), the net current as det(M) s M.  The
// moments of all current elements are summed about the origin as
// 1/2 sum (c x K) + sum mown and re-centred on the mean centre afterwards,
// which is exact for closed circuits (sum K = 0).
void add_current(LineGeom &L, const double *T, const double *c, const double *mown, const double *K)
{
  if (K[0] == 0 && K[1] == 0 && K[2] == 0 && mown[0] == 0 && mown[1] == 0 && mown[2] == 0) return;
  double C[3], m[3], k[3];
  lab_point(T, c, C);
  for (int r = 0; r < 3; r++) {
    m[r] = T[12 + 3 * r] * mown[0] + T[13 + 3 * r] * mown[1] + T[14 + 3 * r] * mown[2];
    k[r] = T[22] * (T[12 + 3 * r] * K[0] + T[13 + 3 * r] * K[1] + T[14 + 3 * r] * K[2]);
  }
  double cxk[3] = {C[1] * k[2] - C[2] * k[1], C[2] * k[0] - C[0] * k[2], C[0] * k[1] - C[1] * k[0]};
  for (int r = 0; r < 3; r++) {
    L.jm[r] += m[r] + 0.5 * cxk[r];
    L.jc[r] += C[r];
    L.jk[r] += k[r];
  }
  L.nj++;
}

// field of the far-field model (B = H outside the sources), T
void dipole_field(const LineGeom &L, const double *p, double *B)
{
  B[0] = B[1] = B[2] = 0;
  const double inv4pi = 0.25 / M_PI;
  for (size_t k = 0; k + 5 < L.dip.size(); k += 6) {
    const double *c = &L.dip[k], *m = &L.dip[k + 3];
    double r[3] = {p[0] - c[0], p[1] - c[1], p[2] - c[2]};
    double r2 = dot3(r, r);
    if (!(r2 > 0)) continue;
    double ir = 1.0 / sqrt(r2), ir3 = ir * ir * ir;
    double mr = dot3(m, r) * ir * ir;
    for (int d = 0; d < 3; d++) B[d] += inv4pi * ir3 * (3.0 * mr * r[d] - m[d]);
  }
}

void scan_geometry(const RadB200Geom *g, LineGeom &L)
{
  const int S = RADB200_TRF_STRIDE;
  double a[3], b[3], t0, t1;
  for (int i = 0; i < g->n_rec; i++) {
    const double *r = g->rec + (size_t)i * RADB200_REC_STRIDE;
    double h[3] = {0.5 * r[3], 0.5 * r[4], 0.5 * r[5]};
    double rad = sqrt(dot3(h, h));
    double vol = r[3] * r[4] * r[5];
    double mv[3] = {r[6] * vol, r[7] * vol, r[8] * vol};          // magnetic moment M V
    double K[3] = {r[9] * vol, r[10] * vol, r[11] * vol};         // net current J V (A mm)
    double zero[3] = {0, 0, 0};
    for (int k = 0; k < g->rec_img[2 * i + 1]; k++) {
      const double *T = g->trf + (size_t)(g->rec_img[2 * i] + k) * S;
      obj_line(T, L, a, b);
      if (clip_box(a, b, r, h, t0, t1)) {
        L.breaks.push_back(t0);
        L.breaks.push_back(t1);
      }
      add_extent(L, T, r, rad);
      add_dipole(L, T, r, mv);
      add_current(L, T, r, zero, K);
    }
  }
  for (int i = 0; i < g->n_poly; i++) {
    const double *c = g->poly + (size_t)i * RADB200_POLY_STRIDE;
    int f0 = g->poly_info[4 * i], nf = g->poly_info[4 * i + 1];
    // vertices p = R^T (x, y, z) of each face (face-local x, y; plane z)
    double rad = 0;
    for (int f = f0; f < f0 + nf; f++) {
      const double *R = g->face + (size_t)f * RADB200_FACE_STRIDE;
      int v0 = g->face_vtx[2 * f], nv = g->face_vtx[2 * f + 1];
      for (int v = v0; v < v0 + nv; v++) {
        double x = g->vtx2d[2 * v], y = g->vtx2d[2 * v + 1];
        double p[3];
        for (int j = 0; j < 3; j++) p[j] = R[j] * x + R[3 + j] * y + R[6 + j] * R[9] - c[j];
        rad = std::max(rad, sqrt(dot3(p, p)));
      }
    }
    // volume and centroid from the tetrahedra (centre, face fan triangle):
    // about its centroid a uniformly magnetized body has no quadrupole moment
    double vol = 0, cen[3] = {0, 0, 0};
    for (int f = f0; f < f0 + nf; f++) {
      const double *R = g->face + (size_t)f * RADB200_FACE_STRIDE;
      int v0 = g->face_vtx[2 * f], nv = g->face_vtx[2 * f + 1];
      double q[3][3];
      auto vert = [&](int v, double *p) {
        double x = g->vtx2d[2 * v], y = g->vtx2d[2 * v + 1];
        for (int j = 0; j < 3; j++) p[j] = R[j] * x + R[3 + j] * y + R[6 + j] * R[9];
      };
      vert(v0, q[0]);
      for (int v = v0 + 1; v + 1 < v0 + nv; v++) {
        vert(v, q[1]);
        vert(v + 1, q[2]);
        double e[3][3];
        for (int a2 = 0; a2 < 3; a2++)
          for (int j = 0; j < 3; j++) e[a2][j] = q[a2][j] - c[j];
        double det = e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) - e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                     e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
        double tv = fabs(det) / 6.0;
        vol += tv;
        for (int j = 0; j < 3; j++) cen[j] += tv * 0.25 * (c[j] + q[0][j] + q[1][j] + q[2][j]);
      }
    }
    if (vol > 0)
      for (int j = 0; j < 3; j++) cen[j] /= vol;
    else
      for (int j = 0; j < 3; j++) cen[j] = c[j];
    double mv[3] = {c[3] * vol, c[4] * vol, c[5] * vol};
    for (int k = 0; k < g->poly_info[4 * i + 3]; k++) {
      const double *T = g->trf + (size_t)(g->poly_info[4 * i + 2] + k) * S;
      obj_line(T, L, a, b);
      // convex body: intersection of the half-spaces on the centre's side
      t0 = -INFINITY;
      t1 = INFINITY;
      bool empty = false;
      for (int f = f0; f < f0 + nf && !empty; f++) {
        const double *R = g->face + (size_t)f * RADB200_FACE_STRIDE;
        double side = dot3(R + 6, c) - R[9];
        double sg = side < 0 ? 1.0 : -1.0;
        double A = sg * (dot3(R + 6, a) - R[9]), B = sg * dot3(R + 6, b);
        if (fabs(B) < 1e-300) {
          if (A > 0) empty = true;
        } else if (B > 0) {
          t1 = std::min(t1, -A / B);
        } else {
          t0 = std::max(t0, -A / B);
        }
      }
      if (!empty && t1 > t0) {
        L.breaks.push_back(t0);
        L.breaks.push_back(t1);
      }
      add_extent(L, T, c, rad);
      add_dipole(L, T, cen, mv);
    }
  }
  for (int i = 0; i < g->n_arc; i++) {
    const double *r = g->arc + (size_t)i * RADB200_ARC_STRIDE;
    double h[3] = {r[4], r[4], 0.5 * r[7]};
    double rad = sqrt(dot3(h, h));
    // azimuthal current j phi^ over rmin..rmax, phimin..phimax, height h about
    // the axis through the centre: net current K = j h (rmax^2 - rmin^2)/2 *
    // (cos p2 - cos p1, sin p2 - sin p1, 0); moment about the centre
    // 1/2 int r x J dV = j h (p2 - p1) (rmax^3 - rmin^3) / 6 z^
    double j = r[8], hh = r[7], p1 = r[5], p2 = r[6];
    double K[3] = {0.5 * j * hh * (r[4] * r[4] - r[3] * r[3]) * (cos(p2) - cos(p1)),
                   0.5 * j * hh * (r[4] * r[4] - r[3] * r[3]) * (sin(p2) - sin(p1)), 0.0};
    double mown[3] = {0, 0, j * hh * (p2 - p1) * (r[4] * r[4] * r[4] - r[3] * r[3] * r[3]) / 6.0};
    for (int k = 0; k < g->arc_img[2 * i + 1]; k++) {
      const double *T = g->trf + (size_t)(g->arc_img[2 * i] + k) * S;
      obj_line(T, L, a, b);
      if (clip_box(a, b, r, h, t0, t1)) {
        L.breaks.push_back(t0);
        L.breaks.push_back(t1);
      }
      add_extent(L, T, r, rad);
      add_current(L, T, r, mown, K);
    }
  }
  if (L.nj) {
    // 1/2 sum c x K about the origin -> about the mean centre c0 (mu0 m, T mm^3)
    double c0[3] = {L.jc[0] / L.nj, L.jc[1] / L.nj, L.jc[2] / L.nj};
    double c0xk[3] = {c0[1] * L.jk[2] - c0[2] * L.jk[1], c0[2] * L.jk[0] - c0[0] * L.jk[2],
                      c0[0] * L.jk[1] - c0[1] * L.jk[0]};
    for (int r = 0; r < 3; r++) L.dip.push_back(c0[r]);
    for (int r = 0; r < 3; r++) L.dip.push_back(MU0_MM * (L.jm[r] - 0.5 * c0xk[r]));
  }
}

// sorted panel ends in [lo, hi]: the ends, the breaks inside and a
// subdivision into nmin panels; ends closer than tol are merged.  The
// subdivision points are moved off the regular grid by fixed fractions of a
// panel (k times the golden ratio, mod 1) so that panel centres, where the
// rule has a node at every bisection level, do not fall on the face planes
// of regularly spaced elements, where the closed-form kernels are singular.
std::vector<double> panel_ends(double lo, double hi, const std::vector<double> &breaks, int nmin)
{
  std::vector<double> e;
  e.reserve(breaks.size() + nmin + 2);
  e.push_back(lo);
  e.push_back(hi);
  for (int k = 1; k < nmin; k++) {
    double f = k * 0.6180339887498949;
    e.push_back(lo + (hi - lo) * (k + 0.3 * (f - floor(f) - 0.5)) / nmin);
  }
  for (double t : breaks)
    if (t > lo && t < hi) e.push_back(t);
  std::sort(e.begin(), e.end());
  double tol = 1e-11 * std::max(hi - lo, 1e-300);
  std::vector<double> out;
  for (double t : e)
    if (out.empty() || t - out.back() > tol) out.push_back(t);
  if (out.back() < hi) out.back() = hi;
  return out;
}

// field of geometry g (uniform background fields already left out of g for
// infinite lines) at n points; what 0 B, 1 H
using PointField = std::function<int(const RadB200Geom *g, const double *pts, int64_t n, int what, double *out)>;

// adaptive Gauss-Kronrod over the panels; what bit 0 B, bit 1 H
int integrate(const RadB200Geom *g, const LineGeom &L, std::vector<Panel> &P, int what, double tol,
              const PointField &fld, double *out, double *status)
{
  static const Rule rule;
  const int MAX_LEVELS = 200;
  const size_t MAX_SPLITS = 1 << 16;  // panels split per level
  const double min_t = 1e-12 * std::max(L.len, L.tb - L.ta + 2 * L.far) + 1e-300, min_x = 1e-12;
  std::vector<double> pts, fb, fh, jac;
  std::vector<int> open;
  double npoints = 0;
  int level = 0;
  bool converged = false, noise_limited = false;
  double total = 0;
  for (; level < MAX_LEVELS; level++) {
    open.clear();
    for (int i = 0; i < (int)P.size(); i++)
      if (!P[i].evaluated) open.push_back(i);
    if (!open.empty()) {
      size_t np = open.size() * GK_N;
      pts.resize(3 * np);
      jac.resize(np);
      fb.assign(3 * np, 0.0);
      fh.assign(3 * np, 0.0);
      size_t nnear = 0;  // panels of seg 0 first: their points go to the point field
      std::stable_sort(open.begin(), open.end(), [&](int x, int y) { return (P[x].seg != 0) < (P[y].seg != 0); });
      for (size_t q = 0; q < open.size(); q++) {
        const Panel &p = P[open[q]];
        if (p.seg == 0) nnear++;
        double c = 0.5 * (p.a + p.b), hw = 0.5 * (p.b - p.a);
        for (int j = 0; j < GK_N; j++) {
          double x = c + hw * rule.s[j], t, J;
          if (p.seg == 0) { t = x; J = 1.0; }
          else {
            double ix = 1.0 / (1.0 - x);
            t = (p.seg == 1) ? L.tb + L.far + L.R * x * ix : L.ta - L.far - L.R * x * ix;
            J = L.R * ix * ix;
          }
          size_t k = q * GK_N + j;
          for (int d = 0; d < 3; d++) pts[3 * k + d] = L.p1[d] + t * L.u[d];
          jac[k] = J * hw;
        }
      }
      size_t nn = nnear * GK_N;
      if (nn && (what & 1)) RB_TRY(fld(g, pts.data(), (int64_t)nn, 0, fb.data()));
      if (nn && (what & 2)) RB_TRY(fld(g, pts.data(), (int64_t)nn, 1, fh.data()));
      for (size_t k = nn; k < np; k++) {
        dipole_field(L, &pts[3 * k], &fb[3 * k]);
        for (int d = 0; d < 3; d++) fh[3 * k + d] = fb[3 * k + d];
      }
      npoints += (double)nn * ((what & 1) + ((what >> 1) & 1));
      for (size_t q = 0; q < open.size(); q++) {
        Panel &p = P[open[q]];
        double K[6] = {0, 0, 0, 0, 0, 0}, G[6] = {0, 0, 0, 0, 0, 0};
        for (int j = 0; j < GK_N; j++) {
          size_t k = q * GK_N + j;
          for (int d = 0; d < 3; d++) {
            double vb = (what & 1) ? fb[3 * k + d] * jac[k] : 0.0;
            double vh = (what & 2) ? fh[3 * k + d] * jac[k] : 0.0;
            K[d] += rule.wk[j] * vb;
            G[d] += rule.wg[j] * vb;
            K[3 + d] += rule.wk[j] * vh;
            G[3 + d] += rule.wg[j] * vh;
          }
        }
        double e = 0;
        bool finite = true;
        for (int d = 0; d < 6; d++) {
          p.val[d] = K[d];
          finite = finite && std::isfinite(K[d]) && std::isfinite(G[d]);
          e = std::max(e, fabs(K[d] - G[d]));
        }
        if (!finite) {
          set_error("field integral: non-finite field on the line");
          return RADB200_E_NUMERIC;
        }
        p.err = e;
        p.evaluated = 1;
        // a half that keeps more than 0.35 of its parent's error estimate did
        // not converge by splitting: after two such generations the panel is
        // at the rounding noise of the field and is not split again
        if (p.perr > 0) p.stall = (e > 0.35 * p.perr) ? p.stall + 1 : 0;
      }
    }
    total = 0;
    double active = 0;  // error in panels that splitting still improves
    double scale = 0;   // sum of |panel integrals|: the size of int |f|
    for (const Panel &p : P) {
      double m = 0;
      for (int d = 0; d < 6; d++) m = std::max(m, fabs(p.val[d]));
      scale += m;
    }
    // a panel whose error estimate stopped shrinking (two generations) and is
    // below 1e-11 of int |f| is at the rounding noise of the field
    auto splittable = [&](const Panel &p) {
      bool noise = p.stall >= 2 && p.err < 1e-11 * scale;
      return !noise && p.b - p.a >= (p.seg == 0 ? min_t : min_x);
    };
    for (const Panel &p : P) {
      total += p.err;
      if (splittable(p)) active += p.err;
    }
    if (total <= tol) { converged = true; break; }
    if (active <= 0.5 * tol) { noise_limited = true; break; }
    // split the fewest improvable panels (largest errors first) that leave at
    // most tol/2 of estimated error in the improvable panels kept
    std::vector<int> order;
    for (size_t i = 0; i < P.size(); i++)
      if (splittable(P[i])) order.push_back((int)i);
    std::sort(order.begin(), order.end(), [&](int x, int y) { return P[x].err > P[y].err; });
    double keep = active;
    std::vector<int> split;
    for (int i : order) {
      if (keep <= 0.5 * tol || split.size() >= MAX_SPLITS) break;
      split.push_back(i);
      keep -= P[i].err;
    }
    for (int i : split) {
      P[i].perr = P[i].err;
      Panel right = P[i];
      double m = 0.5 * (P[i].a + P[i].b);
      P[i].b = m;
      P[i].evaluated = 0;
      right.a = m;
      right.evaluated = 0;
      P.push_back(right);
    }
  }
  for (int d = 0; d < 6; d++) out[d] = 0;
  // sum in line order so that the result does not depend on the split history
  std::sort(P.begin(), P.end(), [](const Panel &x, const Panel &y) {
    return x.seg != y.seg ? x.seg < y.seg : x.a < y.a;
  });
  for (const Panel &p : P)
    for (int d = 0; d < 6; d++) out[d] += p.val[d];
  if (status) {
    status[0] = total;
    status[1] = npoints;
    status[2] = level + (converged ? 1 : 0);
    status[3] = (double)P.size();
    // 1: abs_prec met; 2: the panels left over it are at the field's rounding noise
    status[4] = converged ? 1.0 : (noise_limited ? 2.0 : 0.0);
  }
  return 0;
}

int field_int_impl(const RadB200Geom *g, const PointField &fld, const double *P1, const double *P2, int infinite,
                   int what, double abs_prec, double *out, double *status)
{
  if (!g || !P1 || !P2 || !out || what < 1 || what > 3 || !(abs_prec > 0) || (infinite != 0 && infinite != 1)) {
    set_error("bad field-integral arguments");
    return RADB200_E_ARG;
  }
  for (int d = 0; d < 6; d++) out[d] = 0;
  if (status)
    for (int d = 0; d < 5; d++) status[d] = 0;
  LineGeom L;
  double v[3] = {P2[0] - P1[0], P2[1] - P1[1], P2[2] - P1[2]};
  L.len = sqrt(dot3(v, v));
  for (int d = 0; d < 3; d++) L.p1[d] = P1[d];
  if (!(L.len > 0)) {
    if (infinite) {
      set_error("field integral: the two points defining the line coincide");
      return RADB200_E_ARG;
    }
    if (status) status[4] = 1;
    return 0;  // a finite integral over a zero-length segment
  }
  for (int d = 0; d < 3; d++) L.u[d] = v[d] / L.len;
  RadB200Geom gg = *g;
  if (infinite) gg.n_bkg = 0;  // the reference sets the infinite integral of a uniform field to zero
  scan_geometry(&gg, L);
  std::vector<Panel> P;
  auto add = [&](const std::vector<double> &e, int seg) {
    for (size_t k = 0; k + 1 < e.size(); k++) {
      Panel p{};
      p.a = e[k];
      p.b = e[k + 1];
      p.seg = seg;
      P.push_back(p);
    }
  };
  if (!infinite) {
    add(panel_ends(0.0, L.len, L.breaks, 16), 0);
  } else {
    if (!L.any) {
      if (status) status[4] = 1;
      return 0;
    }
    L.R = std::max(L.R, 0.5 * (L.tb - L.ta));
    add(panel_ends(L.ta, L.tb, L.breaks, 16), 0);
    // Beyond 100 element radii past the span of the geometry the closed-form
    // kernels lose more digits to cancellation than the field has left, and
    // their rounding noise would keep the tails from converging; there the
    // field is that of point dipoles at the element centroids (exact up to
    // relative (radius / distance)^2: a uniformly magnetized body has no
    // quadrupole about its centroid) and of the summed current moment.
    L.far = 100.0 * L.amax;
    std::vector<double> none;
    add(panel_ends(L.ta - L.far, L.ta, none, 8), 0);
    add(panel_ends(L.tb, L.tb + L.far, none, 8), 0);
    add(panel_ends(0.0, 1.0, none, 8), 1);
    add(panel_ends(0.0, 1.0, none, 8), 2);
  }
  return integrate(&gg, L, P, what, abs_prec, fld, out, status);
}

// device point field: points uploaded per refinement level, one launch per quantity
DevGeom g_int_geom;
DBuf g_int_pts, g_int_out, g_int_scratch;
DevGeom g_trj_geom;
DBuf g_trj_init, g_trj_out, g_trj_status;

}  // namespace
}  // namespace rb

using namespace rb;

int radb200_field_int(const RadB200Geom *g, const double *P1, const double *P2, int infinite, int what,
                      int precision, double abs_prec, double *out, double *status)
{
  if (!g || precision < 0 || precision > 2) { set_error("bad field-integral arguments"); return RADB200_E_ARG; }
  auto t0 = std::chrono::steady_clock::now();
  // the geometry handed to the point field is uploaded once, at its first use
  const RadB200Geom *up = nullptr;
  GeomView view{};
  PointField fld = [&](const RadB200Geom *gg, const double *pts, int64_t n, int w, double *res) -> int {
    if (up != gg) {
      RB_TRY(g_int_geom.upload(gg));
      view = g_int_geom.view(precision != 0);
      up = gg;
    }
    size_t b = (size_t)n * 3 * sizeof(double);
    RB_TRY(g_int_pts.upload(pts, b));
    RB_TRY(g_int_out.alloc(b));
    RB_TRY(launch_field(view, g_int_pts.as<double>(), n, w, precision == 1 ? 1 : 0, g_int_out.as<double>(),
                        g_int_scratch, 0));
    RB_CUDA(cudaMemcpy(res, g_int_out.p, b, cudaMemcpyDeviceToHost));
    return 0;
  };
  double st[6];
  RB_TRY(field_int_impl(g, fld, P1, P2, infinite, what, abs_prec, out, st));
  if (status) {
    for (int d = 0; d < 5; d++) status[d] = st[d];
    status[5] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return 0;
}

int radb200_field_int_cb(const RadB200Geom *g, RadB200PointField fn, void *ctx, const double *P1, const double *P2,
                         int infinite, int what, double abs_prec, double *out, double *status)
{
  if (!fn) { set_error("bad field-integral arguments"); return RADB200_E_ARG; }
  auto t0 = std::chrono::steady_clock::now();
  PointField fld = [&](const RadB200Geom *gg, const double *pts, int64_t n, int w, double *res) -> int {
    int rc = fn(ctx, gg, pts, n, w, res);
    if (rc != 0) {
      set_error("field integral: point-field callback returned %d", rc);
      return RADB200_E_ARG;
    }
    return 0;
  };
  double st[6];
  RB_TRY(field_int_impl(g, fld, P1, P2, infinite, what, abs_prec, out, st));
  if (status) {
    for (int d = 0; d < 5; d++) status[d] = st[d];
    status[5] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return 0;
}

int radb200_trajectories(const RadB200Geom *g, double energy_gev, int n_traj, const double *init, double y0, double y1,
                         int np, const double *prec, double *out, int *status)
{
  if (!g || !init || !out || n_traj < 0 || np < 1 || !(energy_gev > 0) || !std::isfinite(y0) || !std::isfinite(y1)) {
    set_error("bad trajectory arguments");
    return RADB200_E_ARG;
  }
  if (n_traj == 0) return 0;
  if ((size_t)n_traj * (size_t)np * 5 > ((size_t)1 << 31)) { set_error("too many trajectory points"); return RADB200_E_ARG; }
  RB_TRY(g_trj_geom.upload(g));
  RB_TRY(g_trj_init.upload(init, (size_t)n_traj * 4 * sizeof(double)));
  size_t ob = (size_t)n_traj * np * 5 * sizeof(double);
  RB_TRY(g_trj_out.alloc(ob));
  RB_TRY(g_trj_status.alloc((size_t)n_traj * sizeof(int)));
  RB_TRY(launch_trajectories(g_trj_geom.view(0), energy_gev, g_trj_init.as<double>(), n_traj, y0, y1, np, prec,
                             g_trj_out.as<double>(), g_trj_status.as<int>(), 0));
  RB_CUDA(cudaMemcpy(out, g_trj_out.p, ob, cudaMemcpyDeviceToHost));
  std::vector<int> st(n_traj);
  RB_CUDA(cudaMemcpy(st.data(), g_trj_status.p, (size_t)n_traj * sizeof(int), cudaMemcpyDeviceToHost));
  int bad = 0, code = 0;
  for (int b = 0; b < n_traj; b++) {
    if (status) status[b] = st[b];
    if (st[b] && !bad) { bad = b + 1; code = st[b]; }
  }
  if (bad) {
    // the reference's messages (radiobuf.cpp:153-154)
    set_error("trajectory %d: %s", bad - 1,
              code == 1 ? "Radia::Error200: Step size is too small in automatic Runge-Kutta integration routine."
                        : "Radia::Error201: Maximum number of steps exceeded in automatic Runge-Kutta integration routine.");
    return RADB200_E_NOCONV;
  }
  return 0;
}
