// mesh.cu -- the field of a tetrahedral mesh by its unique edges and faces.
//
// The vertex/edge form of a uniformly magnetized tetrahedron (tet_fast,
// formulas.cuh) is, at a point q,
//   H(q) = 1/(4 pi) [ sum_edges L_e(q) g_e + sum_faces Omega_f(q) a_f ]
// with L_e = log((R_a + R_b + l) / (R_a + R_b - l)) of the edge's end
// distances, Omega_f the solid angle of the face (Van Oosterom-Strackee) and
// coefficients g_e = sum_f sigma_f nu_{e,f}, a_f = sigma_f n_f,
// sigma_f = M . n_f.  L_e depends on the edge only, and Omega_f changes sign
// with the face's orientation; so for tetrahedra under one image transform
// the sum over tetrahedra equals a sum over their unique edges, with
// G_E = sum of the g_e of the tetrahedra sharing E, and over their unique
// faces, with A_F = sum of s a_f, s = +1 where the tetrahedron's outward
// normal agrees with F's own and -1 where it does not (an inner face between
// magnetizations M1 and M2 carries ((M1 - M2) . n) n).  In a conforming mesh
// each interior face is shared by two tetrahedra and each edge by several,
// so per point this evaluates several times fewer logarithms, arctangents
// and square roots than the tetrahedra one by one.  It is the same sum, term
// for term, as the per-tetrahedron form: B agrees to rounding (5.7e-12 on
// the 20,000-tetrahedron model at 1e6 points in FP64).  Points inside a
// tetrahedron add its magnetization (B), found by a separate inside test that
// only points in a group's bounding box run.  The field dispatch uses this
// form in FP64; the FP32-term variant is compiled but not dispatched (its
// largest per-point error was 2.7x that of the per-tetrahedron FP32 kernel).
#include <math.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <tuple>
#include <unordered_map>

#include "internal.cuh"

namespace rb {

namespace {

struct KeyHash {
  size_t operator()(const std::tuple<long long, long long, long long> &k) const
  {
    uint64_t h = 1469598103934665603ULL;
    for (long long v : {std::get<0>(k), std::get<1>(k), std::get<2>(k)}) {
      h ^= (uint64_t)v;
      h *= 1099511628211ULL;
    }
    return (size_t)h;
  }
};

uint32_t spread10(uint32_t x)
{
  x &= 1023;
  x = (x | (x << 16)) & 0x030000FF;
  x = (x | (x << 8)) & 0x0300F00F;
  x = (x | (x << 4)) & 0x030C30C3;
  x = (x | (x << 2)) & 0x09249249;
  return x;
}

struct MeshHost {
  std::vector<int4> tile;
  std::vector<double> v, e, f;
  std::vector<int4> group;
  std::vector<double> gbox;
  std::vector<int> gtet;
};

// One image transform's tetrahedra (polyhedron indices) into tiles.
void build_group(const std::vector<int> &polys, const std::vector<int> &tetidx, const std::vector<double> &tetrec, int trf,
                 MeshHost &out)
{
  const int nt = (int)polys.size();
  auto rec = [&](int k) { return &tetrec[(size_t)tetidx[polys[k]] * TET_REC_FIELD]; };
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int k = 0; k < nt; k++)
    for (int v = 0; v < 4; v++)
      for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], rec(k)[3 * v + a]); hi[a] = std::max(hi[a], rec(k)[3 * v + a]); }
  const double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
  const double tol = std::max(ext, 1e-300) * 1e-12;
  out.group.push_back(make_int4((int)out.gtet.size(), nt, trf, 0));
  for (int a = 0; a < 3; a++) out.gbox.push_back(lo[a]);
  for (int a = 0; a < 3; a++) out.gbox.push_back(hi[a]);
  out.gtet.insert(out.gtet.end(), polys.begin(), polys.end());
  // unique vertices: copies of one vertex in different tetrahedra are
  // reconstructed from different face frames, so they are merged on a grid of
  // 1e-12 of the mesh's extent (a vertex not merged is only evaluated twice)
  std::unordered_map<std::tuple<long long, long long, long long>, int, KeyHash> vid;
  std::vector<double> V;
  std::vector<int> tv((size_t)nt * 4);
  for (int k = 0; k < nt; k++)
    for (int v = 0; v < 4; v++) {
      const double *p = rec(k) + 3 * v;
      auto key = std::make_tuple(llround((p[0] - lo[0]) / tol), llround((p[1] - lo[1]) / tol), llround((p[2] - lo[2]) / tol));
      auto it = vid.find(key);
      int id;
      if (it == vid.end()) {
        id = (int)(V.size() / 3);
        vid.emplace(key, id);
        V.insert(V.end(), p, p + 3);
      } else id = it->second;
      tv[4 * (size_t)k + v] = id;
    }
  // unique edges and faces with their summed coefficients
  std::unordered_map<uint64_t, int> eid, fid;
  std::vector<double> G;             // 3 per edge
  std::vector<int> ev;               // 2 per edge
  std::vector<double> A, M;          // 3 per face: coefficient, unnormalized normal (own orientation)
  std::vector<int> fv;               // 3 per face
  std::vector<int> te((size_t)nt * 6), tf((size_t)nt * 4);
  for (int k = 0; k < nt; k++) {
    const double *r = rec(k);
    for (int e = 0; e < 6; e++) {
      int a = tv[4 * k + tet_edge_a(e)], b = tv[4 * k + tet_edge_b(e)];
      uint64_t key = ((uint64_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b);
      auto it = eid.find(key);
      int id;
      if (it == eid.end()) {
        id = (int)(ev.size() / 2);
        eid.emplace(key, id);
        ev.push_back(a);
        ev.push_back(b);
        G.insert(G.end(), 3, 0.0);
      } else id = it->second;
      for (int c = 0; c < 3; c++) G[3 * (size_t)id + c] += r[42 + 3 * e + c];
      te[6 * (size_t)k + e] = id;
    }
    for (int f = 0; f < 4; f++) {
      int a = tv[4 * k + tet_face_a(f)], b = tv[4 * k + tet_face_b(f)], c = tv[4 * k + tet_face_c(f)];
      int s0 = std::min(a, std::min(b, c)), s2 = std::max(a, std::max(b, c)), s1 = a + b + c - s0 - s2;
      uint64_t key = ((uint64_t)s0 << 42) | ((uint64_t)s1 << 21) | (uint64_t)s2;
      auto it = fid.find(key);
      int id;
      const double *m = r + 18 + 3 * f;
      if (it == fid.end()) {
        id = (int)(fv.size() / 3);
        fid.emplace(key, id);
        fv.push_back(a);
        fv.push_back(b);
        fv.push_back(c);
        // the face's own orientation: that of the first tetrahedron seen
        const double *pa = &V[3 * (size_t)a], *pb = &V[3 * (size_t)b], *pc = &V[3 * (size_t)c];
        double u[3] = {pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]}, w[3] = {pc[0] - pa[0], pc[1] - pa[1], pc[2] - pa[2]};
        double mm[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
        if (mm[0] * m[0] + mm[1] * m[1] + mm[2] * m[2] < 0) { mm[0] = -mm[0]; mm[1] = -mm[1]; mm[2] = -mm[2]; }
        M.insert(M.end(), mm, mm + 3);
        A.insert(A.end(), 3, 0.0);
      } else id = it->second;
      const double *mm = &M[3 * (size_t)id];
      const double s = (mm[0] * m[0] + mm[1] * m[1] + mm[2] * m[2] < 0) ? -1.0 : 1.0;
      for (int c2 = 0; c2 < 3; c2++) A[3 * (size_t)id + c2] += s * r[30 + 3 * f + c2];
      tf[4 * (size_t)k + f] = id;
    }
  }
  // tetrahedra in Morton order of their centroids; tiles greedily
  std::vector<std::pair<uint32_t, int>> order(nt);
  for (int k = 0; k < nt; k++) {
    uint32_t q[3];
    for (int a = 0; a < 3; a++) {
      double c = 0.25 * (rec(k)[a] + rec(k)[3 + a] + rec(k)[6 + a] + rec(k)[9 + a]);
      q[a] = (uint32_t)std::min(1023.0, std::max(0.0, (c - lo[a]) / std::max(ext, 1e-300) * 1023.0));
    }
    order[k] = std::make_pair(spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2), k);
  }
  std::sort(order.begin(), order.end());
  std::vector<char> eown(ev.size() / 2, 0), fown(fv.size() / 3, 0);
  std::vector<int> slot(V.size() / 3, -1);  // tile-local slot of a vertex in the current tile
  std::vector<int> tverts;                  // vertices of the current tile
  std::vector<int> tedges, tfaces;
  auto flush = [&]() {
    if (tedges.empty() && tfaces.empty()) return;
    int4 t0 = make_int4((int)(out.v.size() / 3), (int)tverts.size(), (int)(out.e.size() / MESH_E), (int)tedges.size());
    int4 t1 = make_int4((int)(out.f.size() / MESH_F), (int)tfaces.size(), trf, 0);
    out.tile.push_back(t0);
    out.tile.push_back(t1);
    for (int v : tverts) out.v.insert(out.v.end(), &V[3 * (size_t)v], &V[3 * (size_t)v] + 3);
    auto len = [&](int a, int b) {
      const double *p = &V[3 * (size_t)a], *q = &V[3 * (size_t)b];
      return sqrt((q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]));
    };
    for (int id : tedges) {
      int a = ev[2 * (size_t)id], b = ev[2 * (size_t)id + 1];
      double r[MESH_E] = {(double)slot[a], (double)slot[b], len(a, b), G[3 * (size_t)id], G[3 * (size_t)id + 1],
                          G[3 * (size_t)id + 2]};
      out.e.insert(out.e.end(), r, r + MESH_E);
    }
    for (int id : tfaces) {
      int a = fv[3 * (size_t)id], b = fv[3 * (size_t)id + 1], c = fv[3 * (size_t)id + 2];
      const double *m = &M[3 * (size_t)id], *pa = &V[3 * (size_t)a];
      double r[MESH_F] = {(double)slot[a], (double)slot[b], (double)slot[c], len(a, b), len(a, c), len(b, c),
                          m[0], m[1], m[2], pa[0] * m[0] + pa[1] * m[1] + pa[2] * m[2],
                          A[3 * (size_t)id], A[3 * (size_t)id + 1], A[3 * (size_t)id + 2]};
      out.f.insert(out.f.end(), r, r + MESH_F);
    }
    for (int v : tverts) slot[v] = -1;
    tverts.clear();
    tedges.clear();
    tfaces.clear();
  };
  for (auto &ok : order) {
    const int k = ok.second;
    int ne_new[6], nf_new[4], nne = 0, nnf = 0;
    for (int e = 0; e < 6; e++)
      if (!eown[te[6 * (size_t)k + e]]) ne_new[nne++] = te[6 * (size_t)k + e];
    for (int f = 0; f < 4; f++)
      if (!fown[tf[4 * (size_t)k + f]]) nf_new[nnf++] = tf[4 * (size_t)k + f];
    if (nne == 0 && nnf == 0) continue;
    // vertices this tetrahedron's new edges and faces need that the tile lacks
    int need = 0;
    for (int v = 0; v < 4; v++)
      if (slot[tv[4 * (size_t)k + v]] < 0) need++;
    if ((int)tverts.size() + need > MESH_VT || (int)tedges.size() + nne > MESH_EMAX ||
        (int)tfaces.size() + nnf > MESH_FMAX)
      flush();
    for (int v = 0; v < 4; v++) {
      int id = tv[4 * (size_t)k + v];
      if (slot[id] < 0) {
        slot[id] = (int)tverts.size();
        tverts.push_back(id);
      }
    }
    for (int q = 0; q < nne; q++) { eown[ne_new[q]] = 1; tedges.push_back(ne_new[q]); }
    for (int q = 0; q < nnf; q++) { fown[nf_new[q]] = 1; tfaces.push_back(nf_new[q]); }
  }
  flush();
}

}  // namespace

int build_mesh(const RadB200Geom *G, const std::vector<int> &tetidx, const std::vector<double> &tetrec, DevGeom &dg)
{
  dg.m_tiles = dg.m_groups = 0;
  // face keys pack three vertex numbers of 21 bits
  if ((int64_t)G->n_poly * 4 >= (1 << 21)) return 0;
  // tetrahedra grouped by image transform: every (polyhedron, image) unit
  std::map<int, std::vector<int>> groups;
  for (int p = 0; p < G->n_poly; p++) {
    if (tetidx[p] < 0) return 0;
    for (int t = 0; t < G->poly_info[4 * p + 3]; t++) groups[G->poly_info[4 * p + 2] + t].push_back(p);
  }
  MeshHost h;
  for (auto &g : groups) build_group(g.second, tetidx, tetrec, g.first, h);
  RB_TRY(dg.m_tile.upload(h.tile.data(), h.tile.size() * sizeof(int4)));
  RB_TRY(dg.m_v.upload(h.v.data(), h.v.size() * sizeof(double)));
  RB_TRY(dg.m_e.upload(h.e.data(), h.e.size() * sizeof(double)));
  RB_TRY(dg.m_f.upload(h.f.data(), h.f.size() * sizeof(double)));
  RB_TRY(dg.m_group.upload(h.group.data(), h.group.size() * sizeof(int4)));
  RB_TRY(dg.m_gbox.upload(h.gbox.data(), h.gbox.size() * sizeof(double)));
  RB_TRY(dg.m_gtet.upload(h.gtet.data(), h.gtet.size() * sizeof(int)));
  dg.m_tiles = (int)(h.tile.size() / 2);
  dg.m_groups = (int)h.group.size();
  return 0;
}

// ---- device ---------------------------------------------------------------------

// dynamic shared memory: the tile's vertices, edges and faces, then every
// thread's distances to the tile's vertices
template <typename T> constexpr size_t mesh_smem()
{
  return sizeof(double) * (MESH_VT * 3 + MESH_EMAX * MESH_E + MESH_FMAX * MESH_F) + sizeof(T) * MESH_VT * 128;
}

template <typename T>
__global__ void __launch_bounds__(128) mesh_field_kernel(GeomView g, const double *__restrict__ pts, int64_t npts,
                                                         double *__restrict__ out, int chunk, int accumulate)
{
  extern __shared__ double smem[];
  double *sv = smem;
  double *se = sv + MESH_VT * 3;
  double *sf = se + MESH_EMAX * MESH_E;
  T(*sR)[128] = reinterpret_cast<T(*)[128]>(sf + MESH_FMAX * MESH_F);
  const int tid = threadIdx.x;
  const int64_t i = (int64_t)blockIdx.x * 128 + tid;
  const MeshView &mv = g.mesh;
  const int t0 = blockIdx.y * chunk, t1 = min(mv.n_tiles, t0 + chunk);
  V3<double> P = mk3<double>(0, 0, 0);
  if (i < npts) P = mk3<double>(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
  const double C = 1.0 / (4.0 * 3.141592653589793238);
  double acc[3] = {0, 0, 0};
  for (int t = t0; t < t1; t++) {
    const int4 ta = __ldg(mv.tile + 2 * t), tb = __ldg(mv.tile + 2 * t + 1);
    __syncthreads();
    for (int k = tid; k < ta.y * 3; k += 128) sv[k] = __ldg(mv.mv + 3 * (size_t)ta.x + k);
    for (int k = tid; k < ta.w * MESH_E; k += 128) se[k] = __ldg(mv.me + (size_t)MESH_E * ta.z + k);
    for (int k = tid; k < tb.y * MESH_F; k += 128) sf[k] = __ldg(mv.mf + (size_t)MESH_F * tb.x + k);
    __syncthreads();
    const double *Tr = g.trf + (size_t)tb.z * RADB200_TRF_STRIDE;
    const double dx = P.x - __ldg(Tr + 9), dy = P.y - __ldg(Tr + 10), dz = P.z - __ldg(Tr + 11);
    const V3<double> q = mk3<double>(__ldg(Tr + 0) * dx + __ldg(Tr + 1) * dy + __ldg(Tr + 2) * dz,
                                     __ldg(Tr + 3) * dx + __ldg(Tr + 4) * dy + __ldg(Tr + 5) * dz,
                                     __ldg(Tr + 6) * dx + __ldg(Tr + 7) * dy + __ldg(Tr + 8) * dz);
    for (int v = 0; v < ta.y; v++) {
      T rx = T(sv[3 * v] - q.x), ry = T(sv[3 * v + 1] - q.y), rz = T(sv[3 * v + 2] - q.z);
      sR[v][tid] = sqrtT(rx * rx + ry * ry + rz * rz);
    }
    double h0 = 0, h1 = 0, h2 = 0;
    for (int e = 0; e < ta.w; e++) {
      const double *r = se + MESH_E * e;
      const int a = (int)r[0], b = (int)r[1];
      const T l = T(r[2]), Ra = sR[a][tid], Rb = sR[b][tid];
      // r_a . r_b from the distances and the edge length
      const T d = T(0.5) * (Ra * Ra + Rb * Rb - l * l);
      T D;
      if (d >= T(0)) D = Ra * Rb + d;
      else {
        // the point sees the edge under more than 90 degrees: Ra Rb + d cancels,
        // use |r_a x r_b|^2 / (Ra Rb - d) from the vectors themselves
        T ax = T(sv[3 * a] - q.x), ay = T(sv[3 * a + 1] - q.y), az = T(sv[3 * a + 2] - q.z);
        T bx = T(sv[3 * b] - q.x), by = T(sv[3 * b + 1] - q.y), bz = T(sv[3 * b + 2] - q.z);
        T cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
        T dd = ax * bx + ay * by + az * bz;
        D = (cx * cx + cy * cy + cz * cz) / (Ra * Rb - dd);
      }
      const double L = (double)log1pT<T>(l * (Ra + Rb + l) / D);
      h0 += L * r[3];
      h1 += L * r[4];
      h2 += L * r[5];
    }
    for (int f = 0; f < tb.y; f++) {
      const double *r = sf + MESH_F * f;
      const int a = (int)r[0], b = (int)r[1], c = (int)r[2];
      const T Ra = sR[a][tid], Rb = sR[b][tid], Rc = sR[c][tid];
      const T lab = T(r[3]), lac = T(r[4]), lbc = T(r[5]);
      const T dab = T(0.5) * (Ra * Ra + Rb * Rb - lab * lab), dac = T(0.5) * (Ra * Ra + Rc * Rc - lac * lac),
              dbc = T(0.5) * (Rb * Rb + Rc * Rc - lbc * lbc);
      // (v_a - q) . m in FP64
      const T num = T(r[9] - (q.x * r[6] + q.y * r[7] + q.z * r[8]));
      const T den = Ra * Rb * Rc + dab * Rc + dac * Rb + dbc * Ra;
      const double om = 2.0 * (double)atan2T(-num, den);
      h0 += om * r[10];
      h1 += om * r[11];
      h2 += om * r[12];
    }
    const double *F = Tr + 12;  // s M: object frame -> lab
    acc[0] += C * (__ldg(F + 0) * h0 + __ldg(F + 1) * h1 + __ldg(F + 2) * h2);
    acc[1] += C * (__ldg(F + 3) * h0 + __ldg(F + 4) * h1 + __ldg(F + 5) * h2);
    acc[2] += C * (__ldg(F + 6) * h0 + __ldg(F + 7) * h1 + __ldg(F + 8) * h2);
  }
  if (i < npts) {
    double *o = out + ((size_t)blockIdx.y * npts + i) * 3;
    if (accumulate) { o[0] += acc[0]; o[1] += acc[1]; o[2] += acc[2]; }
    else { o[0] = acc[0]; o[1] = acc[1]; o[2] = acc[2]; }
  }
}

// B inside a magnet: add the magnetization of the tetrahedron holding the
// point (strictly inside all four face planes), first found, per image.
__global__ void mesh_inside_kernel(GeomView g, const double *__restrict__ pts, int64_t npts, double *__restrict__ out)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const MeshView &mv = g.mesh;
  const V3<double> P = mk3<double>(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
  double add[3] = {0, 0, 0};
  for (int gi = 0; gi < mv.n_groups; gi++) {
    const int4 gr = __ldg(mv.group + gi);
    const double *Tr = g.trf + (size_t)gr.z * RADB200_TRF_STRIDE;
    const double dx = P.x - __ldg(Tr + 9), dy = P.y - __ldg(Tr + 10), dz = P.z - __ldg(Tr + 11);
    const double q[3] = {__ldg(Tr + 0) * dx + __ldg(Tr + 1) * dy + __ldg(Tr + 2) * dz,
                         __ldg(Tr + 3) * dx + __ldg(Tr + 4) * dy + __ldg(Tr + 5) * dz,
                         __ldg(Tr + 6) * dx + __ldg(Tr + 7) * dy + __ldg(Tr + 8) * dz};
    const double *bx = mv.gbox + 6 * (size_t)gi;
    if (q[0] <= bx[0] || q[1] <= bx[1] || q[2] <= bx[2] || q[0] >= bx[3] || q[1] >= bx[4] || q[2] >= bx[5]) continue;
    for (int k = 0; k < gr.y; k++) {
      const int p = __ldg(mv.gtet + gr.x + k);
      const double *rec = g.tetrec + (size_t)__ldg(g.tetidx + p) * TET_REC_FIELD;
      bool in = true;
      for (int f = 0; f < 4 && in; f++) {
        const double *va = rec + 3 * tet_face_a(f), *m = rec + 18 + 3 * f;
        in = (q[0] - va[0]) * m[0] + (q[1] - va[1]) * m[1] + (q[2] - va[2]) * m[2] < 0.0;
      }
      if (!in) continue;
      const double *M = g.poly + (size_t)p * RADB200_POLY_STRIDE + 3;
      const double *F = Tr + 12;
      add[0] += F[0] * M[0] + F[1] * M[1] + F[2] * M[2];
      add[1] += F[3] * M[0] + F[4] * M[1] + F[5] * M[2];
      add[2] += F[6] * M[0] + F[7] * M[1] + F[8] * M[2];
      break;
    }
  }
  out[3 * i] += add[0];
  out[3 * i + 1] += add[1];
  out[3 * i + 2] += add[2];
}

__global__ void mesh_reduce_kernel(const double *__restrict__ part, int nc, int64_t n3, double *__restrict__ out,
                                   int accumulate)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  double s = 0.0;
  for (int c = 0; c < nc; c++) s += part[(size_t)c * n3 + i];
  out[i] = accumulate ? out[i] + s : s;
}

int launch_mesh_field(const GeomView &g, const double *d_pts, int64_t npts, int what, int precision, double *d_out,
                      int accumulate, DBuf &scratch, cudaStream_t st)
{
  const int64_t nblk = (npts + 127) / 128;
  const int nt = g.mesh.n_tiles;
  // split the tiles when the points alone give fewer than ~6 CTAs per SM
  int nchunk = 1;
  const int64_t target = 148 * 6;
  if (nblk < target) nchunk = (int)((target + nblk - 1) / nblk);
  nchunk = std::max(1, std::min(nchunk, std::min(nt, 65535)));
  int chunk = (nt + nchunk - 1) / nchunk;
  nchunk = (nt + chunk - 1) / chunk;
  dim3 grid((unsigned)nblk, (unsigned)nchunk);
  double *dst = d_out;
  int acc = accumulate;
  if (nchunk > 1) {
    RB_TRY(scratch.alloc((size_t)nchunk * npts * 3 * sizeof(double)));
    dst = scratch.as<double>();
    acc = 0;
  }
  static bool attr = false;
  if (!attr) {
    RB_CUDA(cudaFuncSetAttribute(mesh_field_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mesh_smem<float>()));
    RB_CUDA(cudaFuncSetAttribute(mesh_field_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mesh_smem<double>()));
    attr = true;
  }
  if (precision == 1) mesh_field_kernel<float><<<grid, 128, mesh_smem<float>(), st>>>(g, d_pts, npts, dst, chunk, acc);
  else mesh_field_kernel<double><<<grid, 128, mesh_smem<double>(), st>>>(g, d_pts, npts, dst, chunk, acc);
  RB_TRY(check_launch("mesh_field_kernel"));
  if (nchunk > 1) {
    const int64_t n3 = npts * 3;
    mesh_reduce_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(scratch.as<double>(), nchunk, n3, d_out, accumulate);
    RB_TRY(check_launch("mesh_reduce_kernel"));
  }
  if (what == 0) {
    mesh_inside_kernel<<<(unsigned)((npts + 127) / 128), 128, 0, st>>>(g, d_pts, npts, d_out);
    RB_TRY(check_launch("mesh_inside_kernel"));
  }
  return 0;
}

}  // namespace rb
