// capi.cu -- the extern "C" boundary of libradb200 (include/radb200.h) and the
// host-side driver state: device geometry, interactions keyed by handle.
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>

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

int DevGeom::upload(const RadB200Geom *G)
{
  RB_TRY(validate_geom(G));
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
  for (int i = 0; i < G->n_rec; i++)
    for (int t = 0; t < G->rec_img[2 * i + 1]; t++) u.push_back(make_int4(0, i, G->rec_img[2 * i] + t, 0));
  for (int i = 0; i < G->n_poly; i++)
    for (int t = 0; t < G->poly_info[4 * i + 3]; t++) u.push_back(make_int4(1, i, G->poly_info[4 * i + 2] + t, 0));
  for (int i = 0; i < G->n_arc; i++)
    for (int t = 0; t < G->arc_img[2 * i + 1]; t++) u.push_back(make_int4(2, i, G->arc_img[2 * i] + t, 0));
  for (int i = 0; i < G->n_bkg; i++)
    for (int t = 0; t < G->bkg_img[2 * i + 1]; t++) u.push_back(make_int4(3, i, G->bkg_img[2 * i] + t, 0));
  n_units = (int)u.size();
  RB_TRY(units.upload(u.data(), u.size() * sizeof(int4)));
  n_rec = G->n_rec;
  n_poly = G->n_poly;
  g.absr = G->abs_rand; g.relr = G->rel_rand; g.zeror = G->zero_rand;
  return 0;
}

GeomView DevGeom::view() const
{
  GeomView v;
  v.trf = trf.as<double>(); v.rec = rec.as<double>(); v.rec_img = rec_img.as<int>();
  v.poly = poly.as<double>(); v.poly_info = poly_info.as<int>(); v.face = face.as<double>();
  v.face_vtx = face_vtx.as<int>(); v.vtx2d = vtx2d.as<double>(); v.arc = arc.as<double>();
  v.bkg = bkg.as<double>(); v.units = units.as<int4>(); v.n_units = n_units; v.g = g;
  return v;
}

// global state (single device context, like the reference's static caches)
static std::map<int64_t, std::unique_ptr<Intrc>> g_intrc;
static int64_t g_next_handle = 1;
static DBuf g_fld_pts, g_fld_out, g_fld_scratch;

Intrc *find_intrc(int64_t h)
{
  auto it = g_intrc.find(h);
  if (it == g_intrc.end()) { set_error("unknown interaction handle %lld", (long long)h); return nullptr; }
  return it->second.get();
}

int relax_jacobi(Intrc &I, double prec, int max_iter, double omega0, double *status);
int relax_newton(Intrc &I, double prec, int max_iter, double *status);
int relax_reset(Intrc &I);
int direct_solve(Intrc &I, int mode, double rtol, int max_iter, double *status);
int adjoint_solve(Intrc &I, const double *dLdM, double rtol, int max_iter, double *lambda, double *status);
int adjoint_grad(Intrc &I, const double *lambda, double *dMr, double *dc);
int field_vjp(Intrc &I, const double *M, const double *pts, int64_t npts, int what, const double *W, double *gM, double *gc);

}  // namespace rb

using namespace rb;

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
  if (npts < 0 || what < 0 || what > 2 || precision < 0 || precision > 1) { set_error("bad field arguments"); return RADB200_E_ARG; }
  DevGeom dg;
  RB_TRY(dg.upload(g));
  RB_TRY(launch_field(dg.view(), d_pts, npts, what, precision, d_out, g_fld_scratch, 0));
  RB_CUDA(cudaStreamSynchronize(0));
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

int radb200_intrc_create(const RadB200Geom *elems, const RadB200Relax *r, const RadB200Geom *ext, int storage,
                         int64_t *handle)
{
  if (!elems || !r || !handle || storage < 0 || storage > 2) { set_error("bad arguments"); return RADB200_E_ARG; }
  int n = r->n_elem;
  if (n <= 0) { set_error("no relaxable elements"); return RADB200_E_ARG; }
  for (int e = 0; e < n; e++) {
    int k = r->elem_src[2 * e], idx = r->elem_src[2 * e + 1];
    if ((k == 0 && (idx < 0 || idx >= elems->n_rec)) || (k == 1 && (idx < 0 || idx >= elems->n_poly)) || k < 0 || k > 1) {
      set_error("element %d refers to a missing source", e);
      return RADB200_E_ARG;
    }
    if (r->mat_kind[e] < 0 || r->mat_kind[e] > 1) {
      set_error("element %d: unsupported material kind %d", e, r->mat_kind[e]);
      return RADB200_E_UNSUPPORTED;
    }
  }
  std::unique_ptr<Intrc> I(new Intrc());
  I->n = n;
  I->n3 = 3 * n;
  I->ld = (I->n3 + 31) / 32 * 32;
  I->storage = storage;
  RB_TRY(I->geom.upload(elems));
  // observation points and row transforms from each element's main image
  std::vector<double> obs(3 * (size_t)n), rowT(9 * (size_t)n);
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
      for (int b = 0; b < 3; b++) rowT[9 * e + 3 * a + b] = s * T[3 * a + b];
    }
  }
  RB_TRY(I->obs.upload(obs.data(), obs.size() * sizeof(double)));
  RB_TRY(I->rowT.upload(rowT.data(), rowT.size() * sizeof(double)));
  RB_TRY(I->elem_src.upload(r->elem_src, 2 * (size_t)n * sizeof(int)));
  RB_TRY(I->mat_kind.upload(r->mat_kind, (size_t)n * sizeof(int)));
  RB_TRY(I->mat.upload(r->mat, (size_t)n * RADB200_MAT_STRIDE * sizeof(double)));
  I->h_mat_kind.assign(r->mat_kind, r->mat_kind + n);
  I->h_mat.assign(r->mat, r->mat + (size_t)n * RADB200_MAT_STRIDE);
  size_t nn = (size_t)I->n3 * I->ld;
  if (storage == RADB200_STORE_F64 || storage == RADB200_STORE_MIXED) RB_TRY(I->N64.alloc(nn * sizeof(double)));
  if (storage == RADB200_STORE_F32 || storage == RADB200_STORE_MIXED) RB_TRY(I->N32.alloc(nn * sizeof(float)));
  if (I->N64.p) RB_CUDA(cudaMemsetAsync(I->N64.p, 0, nn * sizeof(double)));
  if (I->N32.p) RB_CUDA(cudaMemsetAsync(I->N32.p, 0, nn * sizeof(float)));
  RB_TRY(launch_assemble(I->geom.view(), I->elem_src.as<int>(), I->obs.as<double>(), I->rowT.as<double>(), n, I->ld,
                         I->N32.as<float>(), I->N64.as<double>(), 0));
  // external field at element centres, in element frames
  size_t vb = (size_t)I->ld * sizeof(double);
  RB_TRY(I->hext.alloc(vb));
  RB_CUDA(cudaMemset(I->hext.p, 0, vb));
  if (ext && (ext->n_rec + ext->n_poly + ext->n_arc + ext->n_bkg) > 0) {
    DevGeom xg;
    RB_TRY(xg.upload(ext));
    DBuf tmp, scratch;
    RB_TRY(tmp.alloc(3 * (size_t)n * sizeof(double)));
    RB_TRY(launch_field(xg.view(), I->obs.as<double>(), n, 1, 0, tmp.as<double>(), scratch, 0));
    RB_TRY(launch_rowtrans_vec(I->rowT.as<double>(), tmp.as<double>(), I->hext.as<double>(), n, 0));
  }
  RB_TRY(I->M.alloc(vb)); RB_TRY(I->H.alloc(vb)); RB_TRY(I->Mp.alloc(vb)); RB_TRY(I->F.alloc(vb));
  RB_CUDA(cudaMemset(I->M.p, 0, vb)); RB_CUDA(cudaMemset(I->H.p, 0, vb));
  RB_CUDA(cudaMemset(I->Mp.p, 0, vb)); RB_CUDA(cudaMemset(I->F.p, 0, vb));
  RB_CUDA(cudaDeviceSynchronize());
  int64_t h = g_next_handle++;
  g_intrc[h] = std::move(I);
  *handle = h;
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
  RB_TRY(direct_solve(*I, mode, rtol, max_iter, status));
  RB_CUDA(cudaMemcpy(M_out, I->M.p, I->n3 * sizeof(double), cudaMemcpyDeviceToHost));
  RB_TRY(I->lastM.alloc(I->ld * sizeof(double)));
  RB_CUDA(cudaMemcpy(I->lastM.p, I->M.p, I->ld * sizeof(double), cudaMemcpyDeviceToDevice));
  I->last_kind = 1;
  return 0;
}

int radb200_adjoint_solve(int64_t handle, const double *dLdM, double rtol, int max_iter, double *lambda_out, double *status)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!dLdM || !lambda_out || !status) { set_error("bad adjoint arguments"); return RADB200_E_ARG; }
  return adjoint_solve(*I, dLdM, rtol, max_iter, lambda_out, status);
}

int radb200_adjoint_grad(int64_t handle, const double *lambda, double *dL_dMr, double *dL_dc)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!lambda) { set_error("bad adjoint arguments"); return RADB200_E_ARG; }
  return adjoint_grad(*I, lambda, dL_dMr, dL_dc);
}

int radb200_field_vjp(int64_t handle, const double *M, const double *pts, int64_t npts, int what, const double *W,
                      double *g_M, double *g_c)
{
  Intrc *I = find_intrc(handle);
  if (!I) return RADB200_E_HANDLE;
  if (!M || !pts || !W || npts < 0 || what < 0 || what > 1) { set_error("bad field_vjp arguments"); return RADB200_E_ARG; }
  return field_vjp(*I, M, pts, npts, what, W, g_M, g_c);
}

}  // extern "C"
