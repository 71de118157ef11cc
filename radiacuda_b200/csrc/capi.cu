// capi.cu -- the extern "C" boundary of libradb200 (include/radb200.h) and the
// host-side driver state: device geometry, interactions keyed by handle.
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "internal.cuh"

namespace rb {

static char g_err[1024] = "";
long long g_launches = 0;

void set_error(const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int check_launch(const char *what)
{
  g_launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("launch of %s failed: %s", what, cudaGetErrorString(e));
    return RADB200_E_CUDA;
  }
  return 0;
}

// ---- reuse of device blocks ---------------------------------------------------
// Released blocks wait here (after the device is idle, so no kernel still
// uses them) for the next request of their class on the same device: blocks
// above SMALL_MAX by size (a request takes a cached block at most 25% larger),
// up to RADB200_BUFCACHE_GB (default: 40% of the first device's memory; 0
// turns reuse off); smaller blocks by power-of-two class, up to
// RADB200_SMALLCACHE_GB (default 2).  A failed cudaMalloc returns every cached
// block of that device to the driver and tries again;
// radb200_release_cached_memory returns all of them.  Blocks are keyed by
// device ordinal and the pool is guarded by a mutex, so host threads and
// device switches do not mix blocks up.  A large block released when the
// cache is full displaces the least recently released blocks of its device (a
// workload that changes its buffer sizes, e.g. from FP64 to FP32 matrices,
// keeps its new blocks instead of paying cudaMalloc and cudaFree every time).
// The pool is never destroyed (blocks outlive static DBufs).
namespace {
struct BigBlock {
  void *p;
  uint64_t seq;  // release order
};
struct BigPool {
  std::map<int, std::multimap<size_t, BigBlock>> blocks;    // device -> size -> block (large)
  uint64_t seq = 0;
  std::map<int, std::map<size_t, std::vector<void *>>> small;  // device -> class -> blocks
  size_t total = 0, cap = 0, small_total = 0, small_cap = 0;
  bool init = false;
  std::mutex mu;
};
BigPool &big_pool()
{
  static BigPool *bp = new BigPool();
  return *bp;
}
void big_init(BigPool &bp)
{
  if (bp.init) return;
  bp.init = true;
  const char *e = getenv("RADB200_BUFCACHE_GB");
  if (e) bp.cap = (size_t)(atof(e) * 1073741824.0);
  else {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) bp.cap = tot / 10 * 4;
    else cudaGetLastError();
  }
  const char *es = getenv("RADB200_SMALLCACHE_GB");
  bp.small_cap = (size_t)((es ? atof(es) : 2.0) * 1073741824.0);
}
int current_device()
{
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) { cudaGetLastError(); d = 0; }
  return d;
}
// frees the cached blocks of device dev (all devices when dev < 0); caller holds mu
void big_flush(BigPool &bp, int dev)
{
  int cur = current_device();
  for (auto it = bp.blocks.begin(); it != bp.blocks.end();) {
    if (dev >= 0 && it->first != dev) { ++it; continue; }
    if (it->first != cur) cudaSetDevice(it->first);
    for (auto &kv : it->second) { cudaFree(kv.second.p); bp.total -= kv.first; }
    if (it->first != cur) cudaSetDevice(cur);
    it = bp.blocks.erase(it);
  }
  for (auto it = bp.small.begin(); it != bp.small.end();) {
    if (dev >= 0 && it->first != dev) { ++it; continue; }
    if (it->first != cur) cudaSetDevice(it->first);
    for (auto &kv : it->second)
      for (void *q : kv.second) { cudaFree(q); bp.small_total -= kv.first; }
    if (it->first != cur) cudaSetDevice(cur);
    it = bp.small.erase(it);
  }
  cudaGetLastError();
}
size_t small_class(size_t b)
{
  size_t s = 256;
  while (s < b) s <<= 1;
  return s;
}
}  // namespace

void pool_release_all()
{
  BigPool &bp = big_pool();
  std::lock_guard<std::mutex> lk(bp.mu);
  big_flush(bp, -1);
}

void *pool_alloc(size_t b, size_t *got)
{
  BigPool &bp = big_pool();
  std::lock_guard<std::mutex> lk(bp.mu);
  big_init(bp);
  const int dev = current_device();
  size_t want = b;
  if (b <= SMALL_MAX) {
    want = small_class(b);
    auto &cls = bp.small[dev][want];
    if (!cls.empty()) {
      void *p = cls.back();
      cls.pop_back();
      bp.small_total -= want;
      *got = want;
      return p;
    }
  } else {
    auto &mine = bp.blocks[dev];
    auto it = mine.lower_bound(b);
    if (it != mine.end() && it->first <= b + b / 4) {
      void *p = it->second.p;
      *got = it->first;
      bp.total -= it->first;
      mine.erase(it);
      return p;
    }
  }
  void *p = nullptr;
  if (cudaMalloc(&p, want) != cudaSuccess) {
    cudaGetLastError();
    big_flush(bp, dev);
    if (cudaMalloc(&p, want) != cudaSuccess) {
      cudaGetLastError();
      set_error("device allocation of %zu bytes failed", want);
      return nullptr;
    }
  }
  *got = want;
  return p;
}

void pool_free(void *p, size_t b)
{
  BigPool &bp = big_pool();
  std::lock_guard<std::mutex> lk(bp.mu);
  big_init(bp);
  if (b <= SMALL_MAX) {
    if (bp.small_total + b <= bp.small_cap && cudaDeviceSynchronize() == cudaSuccess) {
      bp.small[current_device()][b].push_back(p);
      bp.small_total += b;
      return;
    }
  } else if (b <= bp.cap && cudaDeviceSynchronize() == cudaSuccess) {
    auto &mine = bp.blocks[current_device()];
    while (bp.total + b > bp.cap && !mine.empty()) {  // make room: the oldest blocks go
      auto old = mine.begin();
      for (auto it = mine.begin(); it != mine.end(); ++it)
        if (it->second.seq < old->second.seq) old = it;
      cudaFree(old->second.p);
      bp.total -= old->first;
      mine.erase(old);
    }
    if (bp.total + b <= bp.cap) {
      mine.emplace(b, BigBlock{p, ++bp.seq});
      bp.total += b;
      return;
    }
  }
  cudaGetLastError();
  cudaFree(p);
}


static int validate_geom(const RadB200Geom *G)
{
  if (!G) { set_error("null geometry"); return RADB200_E_ARG; }
  if (G->n_trf < 0 || G->n_rec < 0 || G->n_poly < 0 || G->n_face < 0 || G->n_vtx < 0 || G->n_arc < 0 || G->n_bkg < 0) {
    set_error("negative counts in geometry");
    return RADB200_E_ARG;
  }
  auto chk_img = [&](const int32_t *img, int n, int stride, int off) -> bool {
    for (int i = 0; i < n; i++) {
      int t0 = img[stride * i + off], nt = img[stride * i + off + 1];
      if (t0 < 0 || nt < 1 || (int64_t)t0 + nt > G->n_trf) return false;
    }
    return true;
  };
  if (!chk_img(G->rec_img, G->n_rec, 2, 0) || !chk_img(G->poly_info, G->n_poly, 4, 2) ||
      !chk_img(G->arc_img, G->n_arc, 2, 0) || !chk_img(G->bkg_img, G->n_bkg, 2, 0)) {
    set_error("image range outside the transform table");
    return RADB200_E_ARG;
  }
  for (int i = 0; i < G->n_poly; i++) {
    int f0 = G->poly_info[4 * i], nf = G->poly_info[4 * i + 1];
    if (f0 < 0 || nf < 1 || (int64_t)f0 + nf > G->n_face) { set_error("face range outside the face table"); return RADB200_E_ARG; }
  }
  for (int f = 0; f < G->n_face; f++) {
    int v0 = G->face_vtx[2 * f], nv = G->face_vtx[2 * f + 1];
    if (v0 < 0 || nv < 3 || (int64_t)v0 + nv > G->n_vtx) { set_error("vertex range outside the vertex table"); return RADB200_E_ARG; }
  }
  for (int a = 0; a < G->n_arc; a++)
    if (G->arc[(size_t)a * RADB200_ARC_STRIDE + 9] < 1.0) { set_error("arc needs at least one sector"); return RADB200_E_ARG; }
  return 0;
}

// Vertex/edge topology of every polyhedron, rebuilt from the face frames:
// vertex 3-D positions P = R^T (x, y, coordZ) deduplicated per polyhedron,
// edges shared by two faces, fan triangles of every face, and the
// coefficients of the field (a_f = sigma_f n_f, g_e = sum sigma_f nu_{e,f},
// sigma_f = M.n_f) and of the tensor (G_e = sum nu_{e,f} n_f^T).
struct HostTopo {
  std::vector<int4> tinfo, tinfo2, tt;
  std::vector<int2> te;
  std::vector<double> tv, tel, teg, teG, ttm, tfn, tfa;
  std::vector<int> tetidx;     // per polyhedron: tetrahedron record index or -1
  std::vector<double> tetrec;  // TET_REC_FIELD or TET_REC_TENSOR doubles per tetrahedron
};

// Fixed-topology record of a tetrahedron (formulas.cuh, tet_fast) from its
// deduplicated vertices V[4] and counter-clockwise face loops.
static void build_tet_record(const std::vector<double> &V, const std::vector<std::vector<int>> &loops, const double *M,
                             bool tensor, std::vector<double> &out)
{
  double rec[TET_REC_TENSOR] = {0};
  for (int k = 0; k < 12; k++) rec[k] = V[k];
  for (int e = 0; e < 6; e++) {
    int a = tet_edge_a(e), b = tet_edge_b(e);
    double dx = V[3 * b] - V[3 * a], dy = V[3 * b + 1] - V[3 * a + 1], dz = V[3 * b + 2] - V[3 * a + 2];
    rec[12 + e] = sqrt(dx * dx + dy * dy + dz * dz);
  }
  for (int f = 0; f < 4; f++) {
    // the loop of face f is the one without vertex f
    const std::vector<int> *L = nullptr;
    for (auto &lp : loops)
      if (lp[0] != f && lp[1] != f && lp[2] != f) L = &lp;
    const double *p0 = &V[3 * (*L)[0]], *p1 = &V[3 * (*L)[1]], *p2 = &V[3 * (*L)[2]];
    double u[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]}, w[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    double m[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
    double mn = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    double n[3] = {m[0] / mn, m[1] / mn, m[2] / mn};
    double sigma = M[0] * n[0] + M[1] * n[1] + M[2] * n[2];
    for (int c = 0; c < 3; c++) {
      rec[18 + 3 * f + c] = m[c];
      rec[30 + 3 * f + c] = tensor ? n[c] : sigma * n[c];
    }
    for (int j = 0; j < 3; j++) {  // directed edges of the counter-clockwise loop
      int a = (*L)[j], b = (*L)[(j + 1) % 3];
      double t[3] = {V[3 * b] - V[3 * a], V[3 * b + 1] - V[3 * a + 1], V[3 * b + 2] - V[3 * a + 2]};
      double tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      for (int c = 0; c < 3; c++) t[c] /= tl;
      double nu[3] = {t[1] * n[2] - t[2] * n[1], t[2] * n[0] - t[0] * n[2], t[0] * n[1] - t[1] * n[0]};
      int e = tet_pair(std::min(a, b), std::max(a, b));
      if (tensor) {
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) rec[42 + 9 * e + 3 * r + c] += nu[r] * n[c];
      } else {
        for (int c = 0; c < 3; c++) rec[42 + 3 * e + c] += sigma * nu[c];
      }
    }
  }
  out.insert(out.end(), rec, rec + (tensor ? TET_REC_TENSOR : TET_REC_FIELD));
}

// Polyhedra [pa, pb) into h, their entries of tinfo / tinfo2 / tetidx at
// p - pa and every offset relative to h's own arrays.
static void build_topo_range(const RadB200Geom *G, bool tensor, int pa, int pb, HostTopo &h)
{
  h.tinfo.resize(pb - pa);
  h.tinfo2.resize(pb - pa);
  h.tetidx.assign(pb - pa, -1);
  for (int pg = pa; pg < pb; pg++) {
    const int p = pg - pa;
    int f0 = G->poly_info[4 * pg], nf = G->poly_info[4 * pg + 1];
    const double *M = G->poly + (size_t)pg * RADB200_POLY_STRIDE + 3;
    int v0 = (int)(h.tv.size() / 3), e0 = (int)h.tel.size(), t0 = (int)h.tt.size(), ff0 = (int)(h.tfn.size() / 3);
    // per-polyhedron scratch, reused across polyhedra of this thread (cleared,
    // capacity kept: a 20,000-tetrahedron model otherwise makes ~10^5 small
    // allocations per upload)
    static thread_local std::vector<double> V, Pall;  // local vertices; every face's vertices in 3-D
    static thread_local std::vector<std::vector<int>> loops;
    V.clear();
    Pall.clear();
    loops.resize(nf);  // exactly nf loops: build_tet_record scans all of them
    for (int k = 0; k < nf; k++) loops[k].clear();
    // every face's vertices back in 3-D: P = R^T (x, y, coordZ)
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < nf; k++) {
      const double *R = G->face + (size_t)(f0 + k) * RADB200_FACE_STRIDE;
      int a0 = G->face_vtx[2 * (f0 + k)], na = G->face_vtx[2 * (f0 + k) + 1];
      for (int j = 0; j < na; j++) {
        double x = G->vtx2d[2 * (size_t)(a0 + j)], y = G->vtx2d[2 * (size_t)(a0 + j) + 1], z = R[9];
        double P[3] = {x * R[0] + y * R[3] + z * R[6], x * R[1] + y * R[4] + z * R[7], x * R[2] + y * R[5] + z * R[8]};
        for (int c = 0; c < 3; c++) { lo[c] = std::min(lo[c], P[c]); hi[c] = std::max(hi[c], P[c]); }
        Pall.insert(Pall.end(), P, P + 3);
      }
    }
    // copies of one vertex seen from different face frames differ by rounding
    // of the frames (up to ~1e-7 of the size for sliver faces): merge within
    // 1e-6 of the polyhedron's extent
    double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    const double tol = 1e-6 * ext;
    for (int k = 0, idx = 0; k < nf; k++) {
      int na = G->face_vtx[2 * (f0 + k) + 1];
      for (int j = 0; j < na; j++, idx++) {
        const double *P = &Pall[3 * (size_t)idx];
        int found = -1;
        for (size_t q = 0; q < V.size() / 3; q++) {
          if (fabs(V[3 * q] - P[0]) <= tol && fabs(V[3 * q + 1] - P[1]) <= tol && fabs(V[3 * q + 2] - P[2]) <= tol) {
            found = (int)q;
            break;
          }
        }
        if (found < 0) {
          found = (int)(V.size() / 3);
          V.insert(V.end(), P, P + 3);
        }
        loops[k].push_back(found);
      }
    }
    int nv = (int)(V.size() / 3);
    if (nv == 4 && nf == 4 && loops[0].size() == 3 && loops[1].size() == 3 && loops[2].size() == 3 && loops[3].size() == 3) {
      h.tetidx[p] = (int)(h.tetrec.size() / (tensor ? TET_REC_TENSOR : TET_REC_FIELD));
      build_tet_record(V, loops, M, tensor, h.tetrec);
    }
    if (nv > POLY_NV_FAST) {  // too many vertices for the register form: reference form only
      h.tinfo[p] = make_int4(v0, -1, e0, 0);
      h.tinfo2[p] = make_int4(t0, 0, ff0, 0);
      continue;
    }
    h.tv.insert(h.tv.end(), V.begin(), V.end());
    static thread_local std::vector<int2> edges;
    static thread_local std::vector<double> g_e, G_e;
    edges.clear();
    g_e.clear();
    G_e.clear();
    for (int k = 0; k < nf; k++) {
      const double *R = G->face + (size_t)(f0 + k) * RADB200_FACE_STRIDE;
      double n[3] = {R[6], R[7], R[8]};
      double sigma = M[0] * n[0] + M[1] * n[1] + M[2] * n[2];
      h.tfn.insert(h.tfn.end(), n, n + 3);
      double af[3] = {sigma * n[0], sigma * n[1], sigma * n[2]};
      h.tfa.insert(h.tfa.end(), af, af + 3);
      const std::vector<int> &L = loops[k];
      int m = (int)L.size();
      for (int j = 1; j + 1 < m; j++) {
        const double *a = &V[3 * L[0]], *b = &V[3 * L[j]], *c = &V[3 * L[j + 1]];
        double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        h.tt.push_back(make_int4(L[0], L[j], L[j + 1], k));
        h.ttm.push_back(u[1] * w[2] - u[2] * w[1]);
        h.ttm.push_back(u[2] * w[0] - u[0] * w[2]);
        h.ttm.push_back(u[0] * w[1] - u[1] * w[0]);
      }
      for (int j = 0; j < m; j++) {
        int a = L[j], b = L[(j + 1) % m];
        int lo = std::min(a, b), hi = std::max(a, b);
        int ei = -1;
        for (size_t q = 0; q < edges.size(); q++)
          if (edges[q].x == lo && edges[q].y == hi) { ei = (int)q; break; }
        if (ei < 0) {
          ei = (int)edges.size();
          edges.push_back(make_int2(lo, hi));
          g_e.insert(g_e.end(), 3, 0.0);
          G_e.insert(G_e.end(), 9, 0.0);
        }
        double t[3] = {V[3 * b] - V[3 * a], V[3 * b + 1] - V[3 * a + 1], V[3 * b + 2] - V[3 * a + 2]};
        double tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        for (int c = 0; c < 3; c++) t[c] /= tl;
        double nu[3] = {t[1] * n[2] - t[2] * n[1], t[2] * n[0] - t[0] * n[2], t[0] * n[1] - t[1] * n[0]};
        for (int c = 0; c < 3; c++) g_e[3 * ei + c] += sigma * nu[c];
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) G_e[9 * ei + 3 * r + c] += nu[r] * n[c];
      }
    }
    for (auto &e : edges) {
      h.te.push_back(e);
      const double *a = &V[3 * e.x], *b = &V[3 * e.y];
      h.tel.push_back(sqrt((b[0] - a[0]) * (b[0] - a[0]) + (b[1] - a[1]) * (b[1] - a[1]) + (b[2] - a[2]) * (b[2] - a[2])));
    }
    h.teg.insert(h.teg.end(), g_e.begin(), g_e.end());
    if (tensor) h.teG.insert(h.teG.end(), G_e.begin(), G_e.end());
    h.tinfo[p] = make_int4(v0, nv, e0, (int)edges.size());
    h.tinfo2[p] = make_int4(t0, (int)h.tt.size() - t0, ff0, nf);
  }
}

// All polyhedra, in ranges on up to 16 host threads, joined in order.
static void build_topo(const RadB200Geom *G, bool tensor, HostTopo &h)
{
  const int np = G->n_poly;
  const int nth = std::max(1, std::min({16, (int)std::thread::hardware_concurrency(), np / 512}));
  if (nth <= 1) {
    build_topo_range(G, tensor, 0, np, h);
    return;
  }
  std::vector<HostTopo> part(nth);
  {
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
      th.emplace_back(build_topo_range, G, tensor, (int)((long long)np * t / nth), (int)((long long)np * (t + 1) / nth),
                      std::ref(part[t]));
    for (auto &t : th) t.join();
  }
  const int rs = tensor ? TET_REC_TENSOR : TET_REC_FIELD;
  h = HostTopo();
  for (auto &q : part) {
    const int nv = (int)(h.tv.size() / 3), ne = (int)h.tel.size(), nt = (int)h.tt.size(), nf = (int)(h.tfn.size() / 3);
    const int ntet = (int)(h.tetrec.size() / rs);
    for (auto &a : q.tinfo) h.tinfo.push_back(make_int4(a.x + nv, a.y, a.z + ne, a.w));
    for (auto &a : q.tinfo2) h.tinfo2.push_back(make_int4(a.x + nt, a.y, a.z + nf, a.w));
    for (int t : q.tetidx) h.tetidx.push_back(t >= 0 ? t + ntet : -1);
    h.tt.insert(h.tt.end(), q.tt.begin(), q.tt.end());
    h.te.insert(h.te.end(), q.te.begin(), q.te.end());
    h.tv.insert(h.tv.end(), q.tv.begin(), q.tv.end());
    h.tel.insert(h.tel.end(), q.tel.begin(), q.tel.end());
    h.teg.insert(h.teg.end(), q.teg.begin(), q.teg.end());
    h.teG.insert(h.teG.end(), q.teG.begin(), q.teG.end());
    h.ttm.insert(h.ttm.end(), q.ttm.begin(), q.ttm.end());
    h.tfn.insert(h.tfn.end(), q.tfn.begin(), q.tfn.end());
    h.tfa.insert(h.tfa.end(), q.tfa.begin(), q.tfa.end());
    h.tetrec.insert(h.tetrec.end(), q.tetrec.begin(), q.tetrec.end());
  }
}

int DevGeom::upload(const RadB200Geom *G, bool tensor_coeffs, bool mesh)
{
  RB_TRY(validate_geom(G));
  all_tets = 0;
  tet_single = 0;
  if (G->n_poly > 0) {
    HostTopo h;
    PhaseClock pc;
    build_topo(G, tensor_coeffs, h);
    pc.mark("geometry: topology (host)");
    RB_TRY(tinfo.upload(h.tinfo.data(), h.tinfo.size() * sizeof(int4)));
    RB_TRY(tinfo2.upload(h.tinfo2.data(), h.tinfo2.size() * sizeof(int4)));
    RB_TRY(tv.upload(h.tv.data(), h.tv.size() * sizeof(double)));
    RB_TRY(te.upload(h.te.data(), h.te.size() * sizeof(int2)));
    RB_TRY(tel.upload(h.tel.data(), h.tel.size() * sizeof(double)));
    RB_TRY(teg.upload(h.teg.data(), h.teg.size() * sizeof(double)));
    RB_TRY(teG.upload(h.teG.data(), h.teG.size() * sizeof(double)));
    RB_TRY(tt.upload(h.tt.data(), h.tt.size() * sizeof(int4)));
    RB_TRY(ttm.upload(h.ttm.data(), h.ttm.size() * sizeof(double)));
    RB_TRY(tfn.upload(h.tfn.data(), h.tfn.size() * sizeof(double)));
    RB_TRY(tfa.upload(h.tfa.data(), h.tfa.size() * sizeof(double)));
    RB_TRY(tetidx.upload(h.tetidx.data(), h.tetidx.size() * sizeof(int)));
    RB_TRY(tetrec.upload(h.tetrec.data(), h.tetrec.size() * sizeof(double)));
    all_tets = std::all_of(h.tetidx.begin(), h.tetidx.end(), [](int t) { return t >= 0; }) ? 1 : 0;
    tet_single = all_tets && G->n_rec == 0 && G->n_arc == 0 && G->n_bkg == 0;
    for (int i = 0; i < G->n_poly && tet_single; i++) tet_single = G->poly_info[4 * i + 3] == 1;
    m_tiles = m_groups = 0;
    // field geometry of an all-tetrahedron model: the mesh form (unique edges and faces)
    pc.mark("geometry: topology upload");
    if (all_tets && !tensor_coeffs && mesh) RB_TRY(build_mesh(G, h.tetidx, h.tetrec, *this));
    pc.mark("geometry: mesh form");
  } else {
    m_tiles = m_groups = 0;
  }
  RB_TRY(trf.upload(G->trf, (size_t)G->n_trf * RADB200_TRF_STRIDE * sizeof(double)));
  RB_TRY(rec.upload(G->rec, (size_t)G->n_rec * RADB200_REC_STRIDE * sizeof(double)));
  RB_TRY(rec_img.upload(G->rec_img, (size_t)G->n_rec * 2 * sizeof(int)));
  RB_TRY(poly.upload(G->poly, (size_t)G->n_poly * RADB200_POLY_STRIDE * sizeof(double)));
  RB_TRY(poly_info.upload(G->poly_info, (size_t)G->n_poly * 4 * sizeof(int)));
  RB_TRY(face.upload(G->face, (size_t)G->n_face * RADB200_FACE_STRIDE * sizeof(double)));
  RB_TRY(face_vtx.upload(G->face_vtx, (size_t)G->n_face * 2 * sizeof(int)));
  RB_TRY(vtx2d.upload(G->vtx2d, (size_t)G->n_vtx * 2 * sizeof(double)));
  RB_TRY(arc.upload(G->arc, (size_t)G->n_arc * RADB200_ARC_STRIDE * sizeof(double)));
  RB_TRY(bkg.upload(G->bkg, (size_t)G->n_bkg * 3 * sizeof(double)));
  // unit table: one entry per (source, image); cuboids, polyhedra, arcs, backgrounds
  std::vector<int4> u;
  ustart[0] = 0;
  for (int i = 0; i < G->n_rec; i++)
    for (int t = 0; t < G->rec_img[2 * i + 1]; t++) u.push_back(make_int4(0, i, G->rec_img[2 * i] + t, 0));
  ustart[1] = (int)u.size();
  for (int i = 0; i < G->n_poly; i++)
    for (int t = 0; t < G->poly_info[4 * i + 3]; t++) u.push_back(make_int4(1, i, G->poly_info[4 * i + 2] + t, 0));
  ustart[2] = (int)u.size();
  for (int i = 0; i < G->n_arc; i++)
    for (int t = 0; t < G->arc_img[2 * i + 1]; t++) u.push_back(make_int4(2, i, G->arc_img[2 * i] + t, 0));
  ustart[3] = (int)u.size();
  for (int i = 0; i < G->n_bkg; i++)
    for (int t = 0; t < G->bkg_img[2 * i + 1]; t++) u.push_back(make_int4(3, i, G->bkg_img[2 * i] + t, 0));
  ustart[4] = (int)u.size();
  n_units = (int)u.size();
  RB_TRY(units.upload(u.data(), u.size() * sizeof(int4)));
  n_rec = G->n_rec;
  n_poly = G->n_poly;
  g.absr = G->abs_rand; g.relr = G->rel_rand; g.zeror = G->zero_rand;
  return 0;
}

GeomView DevGeom::view(int fast) const
{
  GeomView v;
  v.trf = trf.as<double>(); v.rec = rec.as<double>(); v.rec_img = rec_img.as<int>();
  v.poly = poly.as<double>(); v.poly_info = poly_info.as<int>(); v.face = face.as<double>();
  v.face_vtx = face_vtx.as<int>(); v.vtx2d = vtx2d.as<double>(); v.arc = arc.as<double>();
  v.bkg = bkg.as<double>(); v.units = units.as<int4>(); v.n_units = n_units; v.g = g;
  for (int k = 0; k < 5; k++) v.ustart[k] = ustart[k];
  v.tp.tinfo = tinfo.as<int4>(); v.tp.tinfo2 = tinfo2.as<int4>(); v.tp.tv = tv.as<double>();
  v.tp.te = te.as<int2>(); v.tp.tel = tel.as<double>(); v.tp.teg = teg.as<double>(); v.tp.teG = teG.as<double>();
  v.tp.tt = tt.as<int4>(); v.tp.ttm = ttm.as<double>(); v.tp.tfn = tfn.as<double>(); v.tp.tfa = tfa.as<double>();
  v.fast = (fast && tinfo.p) ? 1 : 0;
  v.tetidx = tetidx.as<int>();
  v.tetrec = tetrec.as<double>();
  v.all_tets = all_tets;
  v.tet_single = tet_single;
  v.mesh.n_tiles = m_tiles;
  v.mesh.tile = m_tile.as<int4>();
  v.mesh.mv = m_v.as<double>();
  v.mesh.me = m_e.as<double>();
  v.mesh.mf = m_f.as<double>();
  v.mesh.n_groups = m_groups;
  v.mesh.group = m_group.as<int4>();
  v.mesh.gbox = m_gbox.as<double>();
  v.mesh.gtet = m_gtet.as<int>();
  return v;
}

// global state (single device context, like the reference's static caches)
static std::map<int64_t, std::unique_ptr<Intrc>> g_intrc;
static int64_t g_next_handle = 1;
static DBuf g_fld_pts, g_fld_out, g_fld_scratch;
// device copy of the sources of the last field call: its buffers are reused
// by the next call when they are large enough (no allocation, no
// synchronizing free per call; the library is not reentrant)
static DevGeom g_fld_geom;

// interactions over all rows; a row block only serves radb200_relax_rows_step
Intrc *find_intrc(int64_t h)
{
  auto it = g_intrc.find(h);
  if (it == g_intrc.end()) { set_error("unknown interaction handle %lld", (long long)h); return nullptr; }
  if (it->second->nr != it->second->n) {
    set_error("interaction %lld is a row block: only radb200_relax_rows_step and radb200_intrc_free take it", (long long)h);
    return nullptr;
  }
  return it->second.get();
}
static Intrc *find_rows(int64_t h)
{
  auto it = g_intrc.find(h);
  if (it == g_intrc.end()) { set_error("unknown interaction handle %lld", (long long)h); return nullptr; }
  return it->second.get();
}

int relax_jacobi(Intrc &I, double prec, int max_iter, double omega0, double *status);
int relax_newton(Intrc &I, double prec, int max_iter, double *status);
int relax_reset(Intrc &I);
int relax_rows_step(Intrc &I, const double *M, double prec, double *Mp, double *F, double *sq_sum);
int direct_solve(Intrc &I, int mode, double rtol, int max_iter, double *status);
int adjoint_solve(Intrc &I, const double *dLdM, double rtol, int max_iter, double *lambda, double *status);
int adjoint_grad(Intrc &I, const double *lambda, double *dMr, double *dchi, double *dc, double *dd);
int field_vjp(Intrc &I, const double *M, const double *pts, int64_t npts, int what, const double *W, double *gM, double *gc,
              double *gd);

}  // namespace rb

using namespace rb;

namespace rb {
double g_tm[3] = {0.0, 0.0, 0.0};
bool timing_on()
{
  static int on = -1;
  if (on < 0) {
    const char *e = getenv("RADB200_TIMING");
    on = (e && atoi(e) != 0) ? 1 : 0;
  }
  return on == 1;
}
double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
PhaseClock::PhaseClock() : on(timing_on()), t(on ? now_s() : 0.0)
{
  for (int k = 0; k < 3; k++) tm0[k] = g_tm[k];
}
void PhaseClock::mark(const char *what)
{
  if (!on) return;
  cudaDeviceSynchronize();
  const double u = now_s();
  fprintf(stderr, "RADB200_TIMING %-28s %9.3f ms (malloc %.3f, free %.3f, h2d %.3f)\n", what, 1e3 * (u - t),
          1e3 * (g_tm[0] - tm0[0]), 1e3 * (g_tm[1] - tm0[1]), 1e3 * (g_tm[2] - tm0[2]));
  t = u;
  for (int k = 0; k < 3; k++) tm0[k] = g_tm[k];
}
}  // namespace rb

extern "C" {

const char *radb200_last_error(void) { return g_err; }
int radb200_version(void) { return 100; }
int64_t radb200_kernel_launches(void) { return g_launches; }
int radb200_device_sync(void)
{
  RB_CUDA(cudaDeviceSynchronize());
  return 0;
}


int radb200_field_dev(const RadB200Geom *g, const double *d_pts, int64_t npts, int what, int precision, double *d_out)
{
  if (npts < 0 || what < 0 || what > 2 || precision < 0 || precision > 2) { set_error("bad field arguments"); return RADB200_E_ARG; }
  PhaseClock pc;
  // the mesh form serves FP64 B / H only
  RB_TRY(g_fld_geom.upload(g, false, precision != 1 && what != 2));
  pc.mark("field: geometry upload");
  RB_TRY(launch_field(g_fld_geom.view(precision != 0), d_pts, npts, what, precision == 1 ? 1 : 0, d_out, g_fld_scratch, 0));
  RB_CUDA(cudaStreamSynchronize(0));
  pc.mark("field: kernels");
  return 0;
}

int radb200_field(const RadB200Geom *g, const double *pts, int64_t npts, int what, int precision, double *out)
{
  if (npts < 0 || !pts || !out) { set_error("bad field arguments"); return RADB200_E_ARG; }
  if (npts == 0) return 0;
  size_t b = (size_t)npts * 3 * sizeof(double);
  RB_TRY(g_fld_pts.upload(pts, b));
  RB_TRY(g_fld_out.alloc(b));
  RB_TRY(radb200_field_dev(g, g_fld_pts.as<double>(), npts, what, precision, g_fld_out.as<double>()));
  RB_CUDA(cudaMemcpy(out, g_fld_out.p, b, cudaMemcpyDeviceToHost));
  return 0;
}

// FNV-1a over raw bytes: the interaction's geometry stamp
static uint64_t fnv1a(uint64_t h, const void *p, size_t n)
{
  const unsigned char *b = (const unsigned char *)p;
  for (size_t k = 0; k < n; k++) { h ^= b[k]; h *= 1099511628211ULL; }
  return h;
}

// Material records: linear and tanh laws, and tables whose rows lie inside
// mh_table with H ascending (the reference's MatSatIsoTab check,
// radapl2.cpp:152-166) and at least two points.
static int check_materials(const RadB200Relax *r)
{
  for (int e = 0; e < r->n_elem; e++) {
    const int k = r->mat_kind[e];
    if (k < 0 || k > 2) {
      set_error("element %d: unsupported material kind %d", e, k);
      return RADB200_E_UNSUPPORTED;
    }
    if (k != RADB200_MAT_TABLE) continue;
    const double *m = r->mat + (size_t)e * RADB200_MAT_STRIDE;
    const double f = m[0], c = m[1];
    if (!(f >= 0) || !(c >= 2) || f != floor(f) || c != floor(c) || f + c > (double)r->n_mh || !r->mh_table) {
      set_error("element %d: M(H) table rows outside the table array", e);
      return RADB200_E_ARG;
    }
    for (int q = 1; q < (int)c; q++)
      if (!(r->mh_table[3 * ((size_t)f + q)] > r->mh_table[3 * ((size_t)f + q - 1)])) {
        set_error("element %d: M(H) table not ascending in H", e);
        return RADB200_E_ARG;
      }
  }
  return 0;
}

// device copies of the material records and tables
static int upload_materials(Intrc &I, const RadB200Relax *r)
{
  RB_TRY(I.mat_kind.upload(r->mat_kind, (size_t)I.n * sizeof(int)));
  RB_TRY(I.mat.upload(r->mat, (size_t)I.n * RADB200_MAT_STRIDE * sizeof(double)));
  if (r->n_mh > 0) RB_TRY(I.mh.upload(r->mh_table, (size_t)r->n_mh * 3 * sizeof(double)));
  else I.mh.release();
  I.h_mat_kind.assign(r->mat_kind, r->mat_kind + I.n);
  I.h_mat.assign(r->mat, r->mat + (size_t)I.n * RADB200_MAT_STRIDE);
  return 0;
}

// assemble = false builds everything but leaves the matrix zero (a restored
// state fills it)
// rows [e0, e1) of the observer elements (a row block, radb200_intrc_create_rows);
// e1 < 0: all of them
static int intrc_create_impl(const RadB200Geom *elems, const RadB200Relax *r, const RadB200Geom *ext, int storage,
                             int64_t *handle, bool assemble, int e0 = 0, int e1 = -1)
{
  int fast = (storage & RADB200_ASM_FAST) ? 1 : 0;
  storage &= ~RADB200_ASM_FAST;
  if (!elems || !r || !handle || storage < 0 || storage > 2) { set_error("bad arguments"); return RADB200_E_ARG; }
  int n = r->n_elem;
  if (n <= 0) { set_error("no relaxable elements"); return RADB200_E_ARG; }
  for (int e = 0; e < n; e++) {
    int k = r->elem_src[2 * e], idx = r->elem_src[2 * e + 1];
    if ((k == 0 && (idx < 0 || idx >= elems->n_rec)) || (k == 1 && (idx < 0 || idx >= elems->n_poly)) || k < 0 || k > 1) {
      set_error("element %d refers to a missing source", e);
      return RADB200_E_ARG;
    }
  }
  RB_TRY(check_materials(r));
  std::unique_ptr<Intrc> I(new Intrc());
  I->n = n;
  I->n3 = 3 * n;
  I->ld = (I->n3 + 31) / 32 * 32;
  I->storage = storage;
  if (e1 < 0) e1 = n;
  if (e0 < 0 || e1 > n || e0 >= e1) { set_error("row block [%d, %d) outside [0, %d)", e0, e1, n); return RADB200_E_ARG; }
  I->e0 = e0;
  I->nr = e1 - e0;
  if (I->nr != n && storage == RADB200_STORE_MIXED) { set_error("row blocks are stored FP32 or FP64"); return RADB200_E_ARG; }
  const int nr = I->nr;
  PhaseClock pc;
  RB_TRY(I->geom.upload(elems, fast != 0));
  I->fast = fast;
  pc.mark("create: geometry upload");
  // observation points and row transforms from each element's main image
  std::vector<double> obs(3 * (size_t)n), rowT(9 * (size_t)n);
  I->h_obsJ.assign(9 * (size_t)n, 0.0);
  I->h_elem_src.assign(r->elem_src, r->elem_src + 2 * (size_t)n);
  for (int e = 0; e < n; e++) {
    int k = r->elem_src[2 * e], idx = r->elem_src[2 * e + 1];
    int t0;
    const double *c;
    if (k == 0) { t0 = elems->rec_img[2 * idx]; c = elems->rec + (size_t)idx * RADB200_REC_STRIDE; }
    else { t0 = elems->poly_info[4 * idx + 2]; c = elems->poly + (size_t)idx * RADB200_POLY_STRIDE; }
    const double *T = elems->trf + (size_t)t0 * RADB200_TRF_STRIDE;
    double s = T[21];
    for (int a = 0; a < 3; a++) {
      obs[3 * e + a] = (T[12 + 3 * a] * c[0] + T[13 + 3 * a] * c[1] + T[14 + 3 * a] * c[2]) / s + T[9 + a];
      for (int b = 0; b < 3; b++) {
        rowT[9 * e + 3 * a + b] = s * T[3 * a + b];
        I->h_obsJ[9 * e + 3 * a + b] = T[12 + 3 * a + b] / s;
      }
    }
  }
  // observers of the rows held (all of them unless a row block)
  RB_TRY(I->obs.upload(obs.data() + 3 * (size_t)e0, 3 * (size_t)nr * sizeof(double)));
  RB_TRY(I->rowT.upload(rowT.data() + 9 * (size_t)e0, 9 * (size_t)nr * sizeof(double)));
  {
    uint64_t st = 1469598103934665603ULL;
    int32_t hdr[5] = {n, storage, fast, e0, e1};
    st = fnv1a(st, hdr, sizeof(hdr));
    st = fnv1a(st, obs.data(), obs.size() * sizeof(double));
    st = fnv1a(st, rowT.data(), rowT.size() * sizeof(double));
    st = fnv1a(st, r->elem_src, 2 * (size_t)n * sizeof(int32_t));
    st = fnv1a(st, r->mat_kind, (size_t)n * sizeof(int32_t));
    st = fnv1a(st, r->mat, (size_t)n * RADB200_MAT_STRIDE * sizeof(double));
    I->stamp = st;
  }
  RB_TRY(I->elem_src.upload(r->elem_src, 2 * (size_t)n * sizeof(int)));
  RB_TRY(upload_materials(*I, r));
  pc.mark("create: observers, materials");
  size_t nn = (size_t)3 * nr * I->ld;
  // mixed: every block in FP32, the near ones also as their FP64 residue
  if (storage == RADB200_STORE_F64) RB_TRY(I->N64.alloc(nn * sizeof(double)));
  if (storage == RADB200_STORE_F32 || storage == RADB200_STORE_MIXED) RB_TRY(I->N32.alloc(nn * sizeof(float)));
  if (I->N64.p) RB_CUDA(cudaMemsetAsync(I->N64.p, 0, nn * sizeof(double)));
  if (I->N32.p) RB_CUDA(cudaMemsetAsync(I->N32.p, 0, nn * sizeof(float)));
  if (assemble)
    RB_TRY(launch_assemble(I->geom.view(fast), I->elem_src.as<int>(), I->obs.as<double>(), I->rowT.as<double>(), nr, n,
                           I->ld, I->N32.as<float>(), I->N64.as<double>(), 0));
  pc.mark("create: assembly");
  if (storage == RADB200_STORE_MIXED) RB_TRY(build_near(*I, elems, r, obs.data()));
  pc.mark("create: near pairs");
  // external field at element centres, in element frames
  size_t vb = (size_t)I->ld * sizeof(double);
  RB_TRY(I->hext.alloc(vb));
  RB_CUDA(cudaMemset(I->hext.p, 0, vb));
  if (ext && (ext->n_rec + ext->n_poly + ext->n_arc + ext->n_bkg) > 0) {
    DevGeom &xg = I->xgeom;
    RB_TRY(xg.upload(ext));
    I->has_ext = 1;
    DBuf tmp, scratch;
    RB_TRY(tmp.alloc(3 * (size_t)nr * sizeof(double)));
    RB_TRY(launch_field(xg.view(fast), I->obs.as<double>(), nr, 1, 0, tmp.as<double>(), scratch, 0));
    RB_TRY(launch_rowtrans_vec(I->rowT.as<double>(), tmp.as<double>(), I->hext.as<double>(), nr, 0));
  }
  RB_TRY(I->M.alloc(vb)); RB_TRY(I->H.alloc(vb)); RB_TRY(I->Mp.alloc(vb)); RB_TRY(I->F.alloc(vb));
  RB_CUDA(cudaMemset(I->M.p, 0, vb)); RB_CUDA(cudaMemset(I->H.p, 0, vb));
  RB_CUDA(cudaMemset(I->Mp.p, 0, vb)); RB_CUDA(cudaMemset(I->F.p, 0, vb));
  RB_CUDA(cudaDeviceSynchronize());
  pc.mark("create: external field");
  int64_t h = g_next_handle++;
  g_intrc[h] = std::move(I);
  *handle = h;
  return 0;
}

int radb200_intrc_create(const RadB200Geom *elems, const RadB200Relax *r, const RadB200Geom *ext, int storage,
                         int64_t *handle)
{
  return intrc_create_impl(elems, r, ext, storage, handle, true);
}

int radb200_intrc_create_rows(const RadB200Geom *elems, const RadB200Relax *r, const RadB200Geom *ext, int storage,
                              int32_t e0, int32_t e1, int64_t *handle)
{
  if (e1 < 0) { set_error("bad row block"); return RADB200_E_ARG; }
  return intrc_create_impl(elems, r, ext, storage, handle, true, e0, e1);
}

int radb200_relax_rows_step(int64_t handle, const double *d_M, double prec, double *d_Mp_rows, double *d_F_rows,
                            double *d_H_rows, double *sq_sum)
{
  Intrc *I = find_rows(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!d_M || !d_Mp_rows || !d_F_rows || !sq_sum || !(prec > 0)) { set_error("bad arguments"); return RADB200_E_ARG; }
  RB_TRY(relax_rows_step(*I, d_M, prec, d_Mp_rows, d_F_rows, sq_sum));
  if (d_H_rows) RB_CUDA(cudaMemcpy(d_H_rows, I->H.p, 3 * (size_t)I->nr * sizeof(double), cudaMemcpyDeviceToDevice));
  return 0;
}

int radb200_intrc_load(const RadB200Relax *r, const float *N, const double *h_ext, int64_t *handle)
{
  if (!r || !N || !handle || r->n_elem <= 0 || !r->mat_kind || !r->mat) { set_error("bad arguments"); return RADB200_E_ARG; }
  RB_TRY(check_materials(r));
  std::unique_ptr<Intrc> I(new Intrc());
  const int n = r->n_elem;
  I->n = n;
  I->nr = n;
  I->n3 = 3 * n;
  I->ld = (I->n3 + 31) / 32 * 32;
  I->storage = RADB200_STORE_F32;
  I->geom_ok = 0;
  RB_TRY(upload_materials(*I, r));
  const size_t nn = (size_t)I->n3 * I->ld;
  RB_TRY(I->N32.alloc(nn * sizeof(float)));
  RB_CUDA(cudaMemset(I->N32.p, 0, nn * sizeof(float)));
  RB_CUDA(cudaMemcpy2D(I->N32.p, (size_t)I->ld * sizeof(float), N, (size_t)I->n3 * sizeof(float),
                       (size_t)I->n3 * sizeof(float), (size_t)I->n3, cudaMemcpyHostToDevice));
  const size_t vb = (size_t)I->ld * sizeof(double);
  RB_TRY(I->hext.alloc(vb));
  RB_CUDA(cudaMemset(I->hext.p, 0, vb));
  if (h_ext) RB_CUDA(cudaMemcpy(I->hext.p, h_ext, (size_t)I->n3 * sizeof(double), cudaMemcpyHostToDevice));
  RB_TRY(I->M.alloc(vb)); RB_TRY(I->H.alloc(vb)); RB_TRY(I->Mp.alloc(vb)); RB_TRY(I->F.alloc(vb));
  RB_CUDA(cudaMemset(I->M.p, 0, vb)); RB_CUDA(cudaMemset(I->H.p, 0, vb));
  RB_CUDA(cudaMemset(I->Mp.p, 0, vb)); RB_CUDA(cudaMemset(I->F.p, 0, vb));
  {
    uint64_t st = 1469598103934665603ULL;
    int32_t hdr[3] = {n, -1, 0};
    st = fnv1a(st, hdr, sizeof(hdr));
    st = fnv1a(st, r->mat_kind, (size_t)n * sizeof(int32_t));
    st = fnv1a(st, r->mat, (size_t)n * RADB200_MAT_STRIDE * sizeof(double));
    I->stamp = st;
  }
  RB_CUDA(cudaDeviceSynchronize());
  int64_t h = g_next_handle++;
  g_intrc[h] = std::move(I);
  *handle = h;
  return 0;
}

int radb200_intrc_set_materials(int64_t handle, const RadB200Relax *r)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!r || !r->mat_kind || !r->mat || r->n_elem != I->n) { set_error("bad arguments"); return RADB200_E_ARG; }
  RB_TRY(check_materials(r));
  RB_TRY(upload_materials(*I, r));
  // factors and the converged state belong to the old materials
  I->drop_lu_graphs();
  I->lu_mode = -1;
  I->lu_of_d = 0;
  I->last_kind = -1;
  return 0;
}

// ---- saving and restoring the device state of an interaction --------------
namespace {
const char STATE_MAGIC[8] = {'R', 'B', '2', '0', '0', 'I', 'S', '1'};
struct StateHeader {
  char magic[8];
  int32_t n, ld, storage, fast;
  uint64_t stamp;
  int32_t lu_mode, lu_tc, lu_of_d, last_kind;
  int64_t solve_id, lu_solve_id;
  int32_t nsec, pad;
};
enum { SEC_N64 = 1, SEC_N32, SEC_HEXT, SEC_M, SEC_LASTM, SEC_LU64, SEC_LU32, SEC_LUINV, SEC_NEARD };
struct Sec {
  int64_t tag;
  DBuf *buf;
  int64_t bytes;
};

std::vector<Sec> state_sections(Intrc &I)
{
  const int64_t nn = (int64_t)I.n3 * I.ld, vb = (int64_t)I.ld * 8;
  std::vector<Sec> v;
  if (I.N64.p) v.push_back({SEC_N64, &I.N64, nn * 8});
  if (I.N32.p) v.push_back({SEC_N32, &I.N32, nn * 4});
  if (I.near_nnz > 0) v.push_back({SEC_NEARD, &I.near_D, I.near_nnz * 72});
  v.push_back({SEC_HEXT, &I.hext, vb});
  v.push_back({SEC_M, &I.M, vb});
  if (I.last_kind >= 0 && I.lastM.p) v.push_back({SEC_LASTM, &I.lastM, vb});
  if (I.lu_mode >= 0) {
    const int64_t es = (I.lu_mode == RADB200_LU_F64) ? 8 : 4;
    if (I.LU64.p && es == 8) v.push_back({SEC_LU64, &I.LU64, nn * 8});
    if (I.LU32.p && es == 4) v.push_back({SEC_LU32, &I.LU32, nn * 4});
    v.push_back({SEC_LUINV, &I.LUinv, 2 * (int64_t)I.n3 * 128 * es});
  }
  return v;
}
}  // namespace

int radb200_intrc_save(int64_t handle, void *buf, int64_t capacity, int64_t *bytes)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!bytes) { set_error("bad arguments"); return RADB200_E_ARG; }
  std::vector<Sec> secs = state_sections(*I);
  int64_t total = sizeof(StateHeader);
  for (auto &x : secs) total += 16 + x.bytes;
  *bytes = total;
  if (!buf) return 0;
  if (capacity < total) { set_error("state buffer too small: %lld bytes needed", (long long)total); return RADB200_E_ARG; }
  StateHeader h{};
  memcpy(h.magic, STATE_MAGIC, 8);
  h.n = I->n; h.ld = I->ld; h.storage = I->storage; h.fast = I->fast; h.stamp = I->stamp;
  h.lu_mode = I->lu_mode; h.lu_tc = I->lu_tc; h.lu_of_d = I->lu_of_d; h.last_kind = I->last_kind;
  h.solve_id = I->solve_id; h.lu_solve_id = I->lu_solve_id; h.nsec = (int32_t)secs.size();
  char *o = (char *)buf;
  memcpy(o, &h, sizeof(h));
  o += sizeof(h);
  RB_CUDA(cudaDeviceSynchronize());
  for (auto &x : secs) {
    memcpy(o, &x.tag, 8);
    memcpy(o + 8, &x.bytes, 8);
    RB_CUDA(cudaMemcpy(o + 16, x.buf->p, (size_t)x.bytes, cudaMemcpyDeviceToHost));
    o += 16 + x.bytes;
  }
  return 0;
}

int radb200_intrc_restore(const RadB200Geom *elems, const RadB200Relax *r, const RadB200Geom *ext, int storage,
                          const void *buf, int64_t bytes, int64_t *handle)
{
  if (!buf || !handle || bytes < (int64_t)sizeof(StateHeader)) { set_error("bad state buffer"); return RADB200_E_ARG; }
  StateHeader h;
  memcpy(&h, buf, sizeof(h));
  if (memcmp(h.magic, STATE_MAGIC, 8) != 0) { set_error("not a saved interaction state"); return RADB200_E_ARG; }
  int64_t nh = 0;
  RB_TRY(intrc_create_impl(elems, r, ext, storage, &nh, false));
  Intrc *I = find_intrc(nh);
  auto fail = [&](const char *why) {
    g_intrc.erase(nh);
    set_error("saved interaction state: %s", why);
    return RADB200_E_ARG;
  };
  if (h.n != I->n || h.ld != I->ld || h.storage != I->storage || h.fast != I->fast)
    return fail("sizes or storage differ from this geometry");
  if (h.stamp != I->stamp) return fail("geometry stamp differs (other elements, images or materials)");
  const char *p = (const char *)buf + sizeof(h), *end = (const char *)buf + bytes;
  const int64_t nn = (int64_t)I->n3 * I->ld;
  for (int k = 0; k < h.nsec; k++) {
    if (end - p < 16) return fail("truncated");
    int64_t tag, nb;
    memcpy(&tag, p, 8);
    memcpy(&nb, p + 8, 8);
    p += 16;
    if (nb < 0 || end - p < nb) return fail("truncated");
    DBuf *dst = nullptr;
    int64_t want = -1;
    switch (tag) {
      case SEC_N64: dst = &I->N64; want = nn * 8; break;
      case SEC_N32: dst = &I->N32; want = nn * 4; break;
      case SEC_NEARD: dst = &I->near_D; want = I->near_nnz * 72; break;
      case SEC_HEXT: dst = &I->hext; want = (int64_t)I->ld * 8; break;
      case SEC_M: dst = &I->M; want = (int64_t)I->ld * 8; break;
      case SEC_LASTM: dst = &I->lastM; want = (int64_t)I->ld * 8; break;
      case SEC_LU64: dst = &I->LU64; want = nn * 8; break;
      case SEC_LU32: dst = &I->LU32; want = nn * 4; break;
      case SEC_LUINV: dst = &I->LUinv; want = 2 * (int64_t)I->n3 * 128 * ((h.lu_mode == RADB200_LU_F64) ? 8 : 4); break;
      default: return fail("unknown section");
    }
    if (nb != want) return fail("section size differs");
    if (dst->alloc((size_t)nb) != 0) { g_intrc.erase(nh); return RADB200_E_NOMEM; }
    if (cudaMemcpy(dst->p, p, (size_t)nb, cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      g_intrc.erase(nh);
      set_error("saved interaction state: upload failed");
      return RADB200_E_CUDA;
    }
    p += nb;
  }
  I->lu_mode = h.lu_mode;
  I->lu_tc = h.lu_tc;
  I->lu_of_d = h.lu_of_d;
  I->last_kind = h.last_kind;
  I->solve_id = (int)h.solve_id;
  I->lu_solve_id = (int)h.lu_solve_id;
  *handle = nh;
  return 0;
}

int radb200_release_cached_memory(void)
{
  rb::pool_release_all();
  return 0;
}

int radb200_intrc_free(int64_t handle)
{
  auto it = g_intrc.find(handle);
  if (it == g_intrc.end()) { set_error("unknown interaction handle"); return RADB200_E_HANDLE; }
  g_intrc.erase(it);
  return 0;
}

int radb200_intrc_size(int64_t handle, int32_t *n_elem, int32_t *storage)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (n_elem) *n_elem = I->n;
  if (storage) *storage = I->storage;
  return 0;
}

int radb200_intrc_matrix(int64_t handle, int dtype, void *out)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!out || dtype < 0 || dtype > 1) { set_error("bad arguments"); return RADB200_E_ARG; }
  size_t es = dtype ? sizeof(double) : sizeof(float);
  if (dtype == 1 && I->N64.p) {
    RB_CUDA(cudaMemcpy2D(out, I->n3 * es, I->N64.p, I->ld * es, I->n3 * es, I->n3, cudaMemcpyDeviceToHost));
  } else if (dtype == 0 && I->N32.p) {
    RB_CUDA(cudaMemcpy2D(out, I->n3 * es, I->N32.p, I->ld * es, I->n3 * es, I->n3, cudaMemcpyDeviceToHost));
  } else if (dtype == 1 && I->near_nnz > 0) {
    // mixed storage: FP32 blocks plus the FP64 residue of the near ones
    const size_t n3 = (size_t)I->n3;
    std::vector<float> tmp(n3 * n3);
    RB_CUDA(cudaMemcpy2D(tmp.data(), n3 * 4, I->N32.p, I->ld * 4, n3 * 4, n3, cudaMemcpyDeviceToHost));
    double *o = (double *)out;
    for (size_t k = 0; k < n3 * n3; k++) o[k] = tmp[k];
    std::vector<double> D((size_t)I->near_nnz * 9);
    std::vector<int> ptr(I->n + 1), col(I->near_nnz);
    RB_CUDA(cudaMemcpy(D.data(), I->near_D.p, D.size() * sizeof(double), cudaMemcpyDeviceToHost));
    RB_CUDA(cudaMemcpy(ptr.data(), I->near_ptr.p, ptr.size() * sizeof(int), cudaMemcpyDeviceToHost));
    RB_CUDA(cudaMemcpy(col.data(), I->near_col.p, col.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < I->n; i++)
      for (int k = ptr[i]; k < ptr[i + 1]; k++) {
        const int j = col[k];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) o[(3 * (size_t)i + a) * n3 + 3 * j + b] += D[9 * (size_t)k + 3 * a + b];
      }
  } else {
    // convert on the host from whatever is stored
    size_t nn = (size_t)I->n3 * I->n3;
    if (I->N64.p) {
      std::vector<double> tmp(nn);
      RB_CUDA(cudaMemcpy2D(tmp.data(), I->n3 * 8, I->N64.p, I->ld * 8, I->n3 * 8, I->n3, cudaMemcpyDeviceToHost));
      for (size_t k = 0; k < nn; k++) ((float *)out)[k] = (float)tmp[k];
    } else {
      std::vector<float> tmp(nn);
      RB_CUDA(cudaMemcpy2D(tmp.data(), I->n3 * 4, I->N32.p, I->ld * 4, I->n3 * 4, I->n3, cudaMemcpyDeviceToHost));
      for (size_t k = 0; k < nn; k++) ((double *)out)[k] = tmp[k];
    }
  }
  return 0;
}

int radb200_intrc_extfield(int64_t handle, double *out)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  RB_CUDA(cudaMemcpy(out, I->hext.p, I->n3 * sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

int radb200_intrc_set_extfield(int64_t handle, const double *h)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  RB_CUDA(cudaMemcpy(I->hext.p, h, I->n3 * sizeof(double), cudaMemcpyHostToDevice));
  return 0;
}

int radb200_relax(int64_t handle, int method, double prec, int max_iter, int reset, double omega, double *M_io,
                  double *H_out, double *status)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!M_io || !status || max_iter < 0 || !(prec > 0) || method < 0 || method > 1) { set_error("bad relax arguments"); return RADB200_E_ARG; }
  I->solve_id++;
  if (reset) RB_TRY(relax_reset(*I));
  else {
    RB_CUDA(cudaMemcpy(I->M.p, M_io, I->n3 * sizeof(double), cudaMemcpyHostToDevice));
    RB_CUDA(cudaMemset(I->H.p, 0, I->n3 * sizeof(double)));
  }
  if (method == RADB200_RLX_JACOBI) RB_TRY(relax_jacobi(*I, prec, max_iter, omega, status));
  else RB_TRY(relax_newton(*I, prec, max_iter, status));
  RB_CUDA(cudaMemcpy(M_io, I->M.p, I->n3 * sizeof(double), cudaMemcpyDeviceToHost));
  if (H_out) RB_CUDA(cudaMemcpy(H_out, I->H.p, I->n3 * sizeof(double), cudaMemcpyDeviceToHost));
  RB_TRY(I->lastM.alloc(I->ld * sizeof(double)));
  RB_CUDA(cudaMemcpy(I->lastM.p, I->M.p, I->ld * sizeof(double), cudaMemcpyDeviceToDevice));
  I->last_kind = 0;
  return 0;
}

int radb200_direct_solve(int64_t handle, int mode, double rtol, int max_iter, double *M_out, double *status)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!M_out || !status || mode < 0 || mode > 1) { set_error("bad direct-solve arguments"); return RADB200_E_ARG; }
  for (int e = 0; e < I->n; e++)
    if (I->h_mat_kind[e] != RADB200_MAT_LINEAR) { set_error("direct solve needs linear materials"); return RADB200_E_UNSUPPORTED; }
  I->solve_id++;
  RB_TRY(direct_solve(*I, mode, rtol, max_iter, status));
  RB_CUDA(cudaMemcpy(M_out, I->M.p, I->n3 * sizeof(double), cudaMemcpyDeviceToHost));
  RB_TRY(I->lastM.alloc(I->ld * sizeof(double)));
  RB_CUDA(cudaMemcpy(I->lastM.p, I->M.p, I->ld * sizeof(double), cudaMemcpyDeviceToDevice));
  I->last_kind = 1;
  return 0;
}

int radb200_lu_shift(int64_t handle, double *sigma)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!sigma) { set_error("null sigma"); return RADB200_E_ARG; }
  *sigma = I->lu_mode >= 0 ? I->lu_shift : 0.0;
  return 0;
}

int radb200_adjoint_solve(int64_t handle, const double *dLdM, double rtol, int max_iter, double *lambda_out, double *status)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!dLdM || !lambda_out || !status || !(rtol > 0) || max_iter < 1) { set_error("bad adjoint arguments"); return RADB200_E_ARG; }
  if (I->last_kind < 0) { set_error("adjoint: no converged solve on this interaction"); return RADB200_E_ARG; }
  return adjoint_solve(*I, dLdM, rtol, max_iter, lambda_out, status);
}

int radb200_adjoint_grad(int64_t handle, const double *lambda, double *dL_dMr, double *dL_dchi, double *dL_dc,
                         double *dL_dd)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!lambda) { set_error("bad adjoint arguments"); return RADB200_E_ARG; }
  if (I->last_kind < 0) { set_error("adjoint: no converged solve on this interaction"); return RADB200_E_ARG; }
  if (!I->geom_ok && (dL_dc || dL_dd)) { set_error("adjoint: no element geometry (interaction loaded from a matrix)"); return RADB200_E_UNSUPPORTED; }
  return adjoint_grad(*I, lambda, dL_dMr, dL_dchi, dL_dc, dL_dd);
}

int radb200_field_vjp(int64_t handle, const double *M, const double *pts, int64_t npts, int what, const double *W,
                      double *g_M, double *g_c, double *g_d)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!M || !pts || !W || npts < 0 || what < 0 || what > 1) { set_error("bad field_vjp arguments"); return RADB200_E_ARG; }
  if (!I->geom_ok) { set_error("field_vjp: no element geometry (interaction loaded from a matrix)"); return RADB200_E_UNSUPPORTED; }
  return field_vjp(*I, M, pts, npts, what, W, g_M, g_c, g_d);
}

}  // extern "C"
