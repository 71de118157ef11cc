// radgpu_b200.cpp -- Radia's GPU plugin seam, implemented on libradb200.
//
// Radia's core calls a fixed set of radGPU_* functions when it is compiled
// with RADIA_WITH_CUDA (the core sources themselves are not changed):
//
//   assembly    radGPU_PackGeometryForAsm, radGPU_AssembleMatrix,
//               radGPU_FreeAsmData / FreeSymData / FreeObsQuadData,
//               radGPU_PublishAssembledMatrix, radGPU_DiscardAssembledMatrix
//               (cpp/src/core/radgpu_asm.h:149-187; called from
//               radTInteraction::SetupInteractMatrix, radintrc.cpp:731-805,
//               and radTInteraction::Setup, radintrc.cpp:173-184)
//   relaxation  radGPU_AutoRelax (method 9), radGPU_AutoRelaxNK (method 11)
//               (cpp/src/core/radrlmet.h:700-702; called from
//               radTApplication::MakeAutoRelax, radapl2.cpp:1401-1445)
//   field       radGPU_ComputeField, radGPU_ComputeFieldFromSrcRep
//               (cpp/src/core/radgpu_fld.h:184,198; called from RadFld,
//               radentry.cpp:1073-1134, and radintrc.cpp:1267)
//
// This file takes the place of the reference's radgpu_asm.cpp/.cu,
// radgpurlx.cpp/.cu, radrlmet_gpu.cpp and radgpu_fld.cpp/.cu: it is compiled
// with the core into Radia's own `radia` Python module and links
// libradb200.so.  It walks the core's objects into the flat arrays of
// include/radb200.h; the library does the device work.
//
// Contracts kept from the reference seam:
//   - return codes: the pack returns 1 (take) / 0 (decline), the assembly 0 /
//     -1, the relaxations the iteration count or -1, the field 0 / nonzero;
//     a failure makes the core fall back to its CPU path (or raise Error602
//     under UtiGpuFallback('break')), with the library's message on stderr;
//   - the assembly hands the core a host float[3N x 3N] row-major matrix
//     (RadGPU_AsmResult::matrix_blocks) which the core owns (delete[]), so
//     the CPU consumers (EnsureInteractMatrix, radintrc.cpp:473-525) keep
//     working; the device copy stays resident under the interaction's stamp;
//   - the relaxations write Magn of every element and NewMagnArray /
//     NewFieldArray, and the status (misfit, max |M|, max |H|) the core
//     reports (radrlmet_gpu.cpp:44-49 of the reference glue).
// What differs: symmetry images stay a transform table applied in-kernel;
// coils, backgrounds and images are evaluated on the device (the reference
// falls back to the CPU for coils under a transform, radgpu_fld.cpp:255,281);
// anisotropic linear materials relax on the device (the reference declines
// them, radgpurlx.cpp:169-196).
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "radappl.h"
#include "radarccu.h"
#include "radcast.h"
#include "radg3d.h"
#include "radg3dgr.h"
#include "radgalerkin.h"
#include "radgpu_asm.h"
#include "radgpu_fld.h"
#include "radintrc.h"
#include "radmater.h"
#include "radplnr.h"
#include "radrec.h"
#include "radrlmet.h"
#include "radtrans.h"
#include "radvlpgn.h"

#include "radb200.h"

extern radTApplication rad;
extern radTConvergRepair &radCR;

namespace {

// ---- flat arrays behind one RadB200Geom + RadB200Relax -----------------------
struct Pack {
  std::vector<double> trf, rec, poly, face, vtx2d, arc, bkg;
  std::vector<int32_t> rec_img, poly_info, face_vtx, arc_img, bkg_img;
  std::vector<int32_t> elem_src, mat_kind;
  std::vector<double> mat, mh;
  std::map<std::string, std::pair<int32_t, int32_t>> runs;  // image runs by content
  double rand[3] = {0, 0, 0};
  std::string why;  // reason for declining

  RadB200Geom geom() const
  {
    RadB200Geom g;
    memset(&g, 0, sizeof(g));
    g.n_trf = (int32_t)(trf.size() / RADB200_TRF_STRIDE); g.trf = trf.data();
    g.n_rec = (int32_t)(rec.size() / RADB200_REC_STRIDE); g.rec = rec.data(); g.rec_img = rec_img.data();
    g.n_poly = (int32_t)(poly.size() / RADB200_POLY_STRIDE); g.poly = poly.data(); g.poly_info = poly_info.data();
    g.n_face = (int32_t)(face.size() / RADB200_FACE_STRIDE); g.face = face.data(); g.face_vtx = face_vtx.data();
    g.n_vtx = (int32_t)(vtx2d.size() / 2); g.vtx2d = vtx2d.data();
    g.n_arc = (int32_t)(arc.size() / RADB200_ARC_STRIDE); g.arc = arc.data(); g.arc_img = arc_img.data();
    g.n_bkg = (int32_t)(bkg.size() / 3); g.bkg = bkg.data(); g.bkg_img = bkg_img.data();
    g.abs_rand = rand[0]; g.rel_rand = rand[1]; g.zero_rand = rand[2];
    return g;
  }
  RadB200Relax relax() const
  {
    RadB200Relax r;
    r.n_elem = (int32_t)mat_kind.size();
    r.elem_src = elem_src.data(); r.mat_kind = mat_kind.data(); r.mat = mat.data();
    r.n_mh = (int32_t)(mh.size() / 3); r.mh_table = mh.data();
    return r;
  }
  // Appends a run of image records (deduplicated by content: all elements
  // under the same transformation list share one run).
  void add_run(const std::vector<double> &recs, int32_t *first, int32_t *count)
  {
    std::string key((const char *)recs.data(), recs.size() * sizeof(double));
    auto it = runs.find(key);
    if (it == runs.end()) {
      int32_t f = (int32_t)(trf.size() / RADB200_TRF_STRIDE);
      trf.insert(trf.end(), recs.begin(), recs.end());
      it = runs.emplace(std::move(key), std::make_pair(f, (int32_t)(recs.size() / RADB200_TRF_STRIDE))).first;
    }
    *first = it->second.first;
    *count = it->second.second;
  }
};

// The length-randomization guard magnitudes the closed forms use
// (radTConvergRepair::AbsRandMagnitude, radcnvrg.h:83-89): all zero when
// randomization is off (FldLenRndSw('off')).
void guard_from_core(Pack &p)
{
  if (radCR.ActOnDoubles) { p.rand[0] = radCR.AbsRand; p.rand[1] = radCR.RelRand; p.rand[2] = radCR.ZeroRand; }
  else p.rand[0] = p.rand[1] = p.rand[2] = 0.0;
}

// ---- transforms ----------------------------------------------------------------
// A transform as P -> M P + V, fields F -> s M F (gmTrans, gmtrans.h:22-84).
struct Affine {
  double M[9], Minv[9], V[3], s, det;
};

// Reads a radTrans through its own maps on the unit vectors (exact: every
// product with 0 or 1 is), so identity transforms and subclasses behave as in
// the core.
Affine affine_of(radTrans *T)
{
  Affine a;
  const TVector3d e[3] = {TVector3d(1., 0., 0.), TVector3d(0., 1., 0.), TVector3d(0., 0., 1.)};
  double sM[9];
  for (int k = 0; k < 3; k++) {
    TVector3d m = T->TrBiPoint(e[k]), mi = T->TrBiPoint_inv(e[k]), f = T->TrVectField(e[k]);
    a.M[k] = m.x; a.M[3 + k] = m.y; a.M[6 + k] = m.z;
    a.Minv[k] = mi.x; a.Minv[3 + k] = mi.y; a.Minv[6 + k] = mi.z;
    sM[k] = f.x; sM[3 + k] = f.y; sM[6 + k] = f.z;
  }
  TVector3d v = T->TrPoint(TVector3d(0., 0., 0.));
  a.V[0] = v.x; a.V[1] = v.y; a.V[2] = v.z;
  // s from the field map against the point map (s = +-1 for every Radia transform)
  double num = 0;
  for (int k = 0; k < 9; k++) num += sM[k] * a.M[k];
  a.s = (num < 0) ? -1.0 : 1.0;
  a.det = (double)T->ShowParity();
  return a;
}

Affine affine_identity()
{
  Affine a;
  for (int k = 0; k < 9; k++) a.M[k] = a.Minv[k] = (k % 4 == 0) ? 1.0 : 0.0;
  a.V[0] = a.V[1] = a.V[2] = 0.0;
  a.s = a.det = 1.0;
  return a;
}

// x applied after y
Affine compose(const Affine &x, const Affine &y)
{
  Affine r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double m = 0, mi = 0;
      for (int k = 0; k < 3; k++) { m += x.M[3 * i + k] * y.M[3 * k + j]; mi += y.Minv[3 * i + k] * x.Minv[3 * k + j]; }
      r.M[3 * i + j] = m;
      r.Minv[3 * i + j] = mi;
    }
  for (int i = 0; i < 3; i++)
    r.V[i] = x.M[3 * i] * y.V[0] + x.M[3 * i + 1] * y.V[1] + x.M[3 * i + 2] * y.V[2] + x.V[i];
  r.s = x.s * y.s;
  r.det = x.det * y.det;
  return r;
}

// RADB200_TRF_STRIDE record: M^-1, V, s*M, s, det
void push_record(const Affine &a, std::vector<double> &out)
{
  size_t o = out.size();
  out.resize(o + RADB200_TRF_STRIDE, 0.0);
  double *r = &out[o];
  for (int k = 0; k < 9; k++) { r[k] = a.Minv[k]; r[12 + k] = a.s * a.M[k]; }
  for (int k = 0; k < 3; k++) r[9 + k] = a.V[k];
  r[21] = a.s;
  r[22] = a.det;
}

// All images of a transformation chain (outermost first), in the order of
// radTInteraction::NestedFor_Trans (radintrc.cpp:527-553): a transform of
// multiplicity m contributes its powers 0 .. m-1, the first image (all powers
// zero) is the main one.
typedef std::vector<std::pair<int, Affine>> Chain;
void images_of(const Chain &ch, size_t i, const Affine &base, std::vector<double> &out)
{
  if (i == ch.size()) { push_record(base, out); return; }
  const int mult = ch[i].first;
  const Affine &t = ch[i].second;
  if (mult == 1) { images_of(ch, i + 1, compose(base, t), out); return; }
  images_of(ch, i + 1, base, out);
  Affine cur = base;
  for (int k = 1; k < mult; k++) {
    cur = compose(cur, t);
    images_of(ch, i + 1, cur, out);
  }
}

// ---- sources ---------------------------------------------------------------------
void put3(std::vector<double> &v, const TVector3d &a) { v.push_back(a.x); v.push_back(a.y); v.push_back(a.z); }

// Polyhedron faces in their own frames: radTPolyhedron keeps, per face, the
// polygon in the face plane (2-D vertices, plane z) and the rotation whose
// inverse maps object to face coordinates (FillInVectHandlePgnAndTrans,
// radvlpgn.cpp:350-437; used as TrPoint_inv in B_comp_frM, :441-505).
bool add_poly(Pack &p, radTPolyhedron *ph, const TVector3d &magn, int32_t first, int32_t count)
{
  if (ph->J_IsNotZero) { p.why = "current-carrying polyhedron"; return false; }
  const int f0 = (int)(p.face.size() / RADB200_FACE_STRIDE);
  const int nf = (int)ph->VectHandlePgnAndTrans.size();
  if (nf < 4) { p.why = "polyhedron with fewer than 4 faces"; return false; }
  for (int k = 0; k < nf; k++) {
    radTPolygon *pg = ph->VectHandlePgnAndTrans[k].PgnHndl.rep;
    radTrans *tr = ph->VectHandlePgnAndTrans[k].TransHndl.rep;
    if (!pg || !tr) { p.why = "polyhedron face without polygon"; return false; }
    const int nv = (int)pg->EdgePointsVector.size();
    if (nv < 3) { p.why = "degenerate polyhedron face"; return false; }
    const TVector3d e[3] = {TVector3d(1., 0., 0.), TVector3d(0., 1., 0.), TVector3d(0., 0., 1.)};
    double R[9];
    for (int c = 0; c < 3; c++) {
      TVector3d col = tr->TrBiPoint_inv(e[c]);  // object -> face frame
      R[c] = col.x; R[3 + c] = col.y; R[6 + c] = col.z;
    }
    p.face.insert(p.face.end(), R, R + 9);
    p.face.push_back(pg->CoordZ);
    p.face_vtx.push_back((int32_t)(p.vtx2d.size() / 2));
    p.face_vtx.push_back(nv);
    for (int j = 0; j < nv; j++) { p.vtx2d.push_back(pg->EdgePointsVector[j].x); p.vtx2d.push_back(pg->EdgePointsVector[j].y); }
  }
  put3(p.poly, ph->CentrPoint);
  put3(p.poly, magn);
  p.poly_info.push_back(f0);
  p.poly_info.push_back(nf);
  p.poly_info.push_back(first);
  p.poly_info.push_back(count);
  return true;
}

void add_rec(Pack &p, radTRecMag *r, const TVector3d &magn, int32_t first, int32_t count)
{
  put3(p.rec, r->CentrPoint);
  put3(p.rec, r->Dimensions);
  put3(p.rec, magn);
  put3(p.rec, r->J_IsNotZero ? r->J : TVector3d(0., 0., 0.));
  p.rec_img.push_back(first);
  p.rec_img.push_back(count);
}

// Material record of one element (include/radb200.h, RadB200Relax): the
// linear laws by their instant tensor and remanence (radmater.h:216-219,
// 407-412), the tanh formula by its (ksi_i, ms_i) terms and tables by their
// (H, M, dM/dH) rows (radmater.h:554-580).
bool add_material(Pack &p, radTg3dRelax *el)
{
  radTMaterial *mat = (radTMaterial *)el->MaterHandle.rep;
  if (!mat) { p.why = "element without material"; return false; }
  double r[RADB200_MAT_STRIDE] = {0};
  const int t = mat->Type_Material();
  if (t == 1 || t == 2) {
    TMatrix3d K;
    TVector3d Mr;
    mat->DefineInstantKsiTensor(TVector3d(0., 0., 0.), K, Mr);
    const TVector3d *rows[3] = {&K.Str0, &K.Str1, &K.Str2};
    for (int a = 0; a < 3; a++) { r[3 * a] = rows[a]->x; r[3 * a + 1] = rows[a]->y; r[3 * a + 2] = rows[a]->z; }
    r[9] = Mr.x; r[10] = Mr.y; r[11] = Mr.z;
    p.mat_kind.push_back(RADB200_MAT_LINEAR);
  } else if (t == 3) {
    radTNonlinearIsotropMaterial *nl = dynamic_cast<radTNonlinearIsotropMaterial *>(mat);
    if (!nl) { p.why = "unknown nonlinear material"; return false; }
    int npts = 0, nform = 0;
    nl->GetGPUData_Counts(&npts, &nform);
    if (npts > 0) {
      std::vector<double> H(npts), M(npts), D(npts);
      nl->GetGPUData_Curve(H.data(), M.data(), D.data(), npts);
      r[0] = (double)(p.mh.size() / 3);
      r[1] = (double)npts;
      for (int k = 0; k < npts; k++) { p.mh.push_back(H[k]); p.mh.push_back(M[k]); p.mh.push_back(D[k]); }
      p.mat_kind.push_back(RADB200_MAT_TABLE);
    } else {
      double ms[3], ks[3];
      int len = 0;
      nl->GetGPUData_Formula(ms, ks, &len);
      if (len < 1 || len > 3) { p.why = "nonlinear formula without terms"; return false; }
      for (int k = 0; k < len; k++) { r[k] = ks[k]; r[3 + k] = ms[k]; }
      r[6] = len;
      p.mat_kind.push_back(RADB200_MAT_TANH);
    }
    r[9] = mat->RemMagn.x; r[10] = mat->RemMagn.y; r[11] = mat->RemMagn.z;
  } else {
    p.why = "material law without a device form";
    return false;
  }
  p.mat.insert(p.mat.end(), r, r + RADB200_MAT_STRIDE);
  return true;
}

void say(const char *where, const char *what)
{
  fprintf(stderr, "radiacuda_b200 %s: %s\n", where, what);
}

// ---- device interactions of the core's interactions ----------------------------
// Keyed by radTInteraction::mGpuMatrixStamp.  The core deletes interactions
// without telling the plugin, so residents are bounded: the least recently
// used one is released when more than kMaxResident are held or a new one
// does not fit; a later relaxation of a released one reloads the matrix the
// core keeps on the host.
const int kMaxResident = 8;
struct Resident {
  int64_t handle = 0;
  int n = 0;
  std::vector<int32_t> mat_kind;
  std::vector<double> mat, mh;
  uint64_t used = 0;
};
std::map<unsigned long long, Resident> g_res;
uint64_t g_clock = 0;
struct Pending {
  int64_t handle = 0;
  int n = 0;
  std::vector<int32_t> mat_kind;
  std::vector<double> mat, mh;
};
Pending g_pending;
std::map<const void *, std::unique_ptr<Pack>> g_asm_packs;  // keyed by the core's RadGPU_PolyData

void release_lru()
{
  auto lru = g_res.end();
  for (auto it = g_res.begin(); it != g_res.end(); ++it)
    if (lru == g_res.end() || it->second.used < lru->second.used) lru = it;
  if (lru == g_res.end()) return;
  radb200_intrc_free(lru->second.handle);
  g_res.erase(lru);
}

void drop_pending()
{
  if (g_pending.handle) radb200_intrc_free(g_pending.handle);
  g_pending = Pending();
}

// Runs fn, releasing resident interactions (oldest first) while it runs out
// of device memory.
template <class F> int with_room(F fn)
{
  while ((int)g_res.size() >= kMaxResident) release_lru();
  for (;;) {
    int rc = fn();
    if (rc != RADB200_E_NOMEM || g_res.empty()) return rc;
    release_lru();
  }
}

}  // namespace

// The relaxation pack: everything radb200_relax needs from one interaction.
// (A type of this plugin; radTInteraction names it as the argument type of
// its friends radGPU_PackInteractionData / radGPU_UnpackMagnetization,
// radintrc.h:90-91.)
struct RadGPURelaxData {
  int n = 0;
  unsigned long long stamp = 0;
  Pack mats;                    // mat_kind / mat / mh of the elements
  std::vector<double> M, H, hext;
  bool have_H = false;            // H holds the field at the new M
  const float *matrix = nullptr;  // host matrix, only when it must be uploaded
  std::vector<float> flat;        // flattened InteractMatrix (CPU-assembled)
};

// ---- assembly --------------------------------------------------------------------

int radGPU_PackObsQuadForAsm(radTInteraction *intrct, RadGPU_ObsQuadData *q)
{
  // Collocation only: one observation point per element (its transformed
  // centre, weight 1), which is what the core asks for unless the opt-in
  // volume-averaged assembly is on (radgpu_asm.h:89-125).
  if (!intrct || !q) return 0;
  q->on = 0;
  q->n_elem = intrct->AmOfMainElem;
  return radGalerkinCfg().On ? 0 : 1;
}

int radGPU_PackGeometryForAsm(radTInteraction *I, RadGPU_PolyData *polyData, RadGPU_RecMagData *recData,
                              RadGPU_SymData *symData, RadGPU_ObsQuadData *quadData)
{
  if (!I || !polyData || !recData || !symData || !quadData) return 0;
  if (!radGPU_PackObsQuadForAsm(I, quadData)) return 0;  // volume-averaged assembly: the core's CPU path
  const int N = I->AmOfMainElem;
  if (N <= 0) return 0;
  std::unique_ptr<Pack> p(new Pack());
  guard_from_core(*p);
  int n_rec = 0, total_images = 0;
  for (int i = 0; i < N; i++) {
    radTg3dRelax *el = I->g3dRelaxPtrVect[i];
    // every image of element i, main first, exactly as the core's own loop
    // enumerates them (radintrc.cpp:833, FillInTransPtrVectForElem)
    I->FillInTransPtrVectForElem(i, 'I');
    std::vector<double> recs;
    for (size_t k = 0; k < I->TransPtrVect.size(); k++) push_record(affine_of(I->TransPtrVect[k]), recs);
    I->EmptyTransPtrVect();
    int32_t first = 0, count = 0;
    p->add_run(recs, &first, &count);
    total_images += count;
    radTRecMag *rm = radTCast::RecMagCast(el);
    radTPolyhedron *ph = rm ? nullptr : radTCast::PolyhedronCast(el);
    bool ok;
    if (rm) {
      if (rm->J_IsNotZero) { p->why = "current-carrying relaxable block"; ok = false; }
      else {
        add_rec(*p, rm, el->Magn, first, count);
        p->elem_src.push_back(0);
        p->elem_src.push_back(n_rec++);
        ok = true;
      }
    } else if (ph) {
      ok = add_poly(*p, ph, el->Magn, first, count);
      if (ok) { p->elem_src.push_back(1); p->elem_src.push_back((int32_t)(p->poly.size() / RADB200_POLY_STRIDE) - 1); }
    } else {
      p->why = "element type without a device form (e.g. an extruded polygon)";
      ok = false;
    }
    if (ok) ok = add_material(*p, el);
    if (!ok) {
      say("assembly declined", p->why.c_str());
      return 0;
    }
  }
  // the reference's structs only carry the sizes here; the arrays travel in
  // this plugin's own pack
  polyData->n_elem = N;
  polyData->n_faces_total = (int)(p->face.size() / RADB200_FACE_STRIDE);
  polyData->n_edges_total = (int)(p->vtx2d.size() / 2);
  recData->n_rec = n_rec;
  recData->abs_rand = p->rand[0]; recData->rel_rand = p->rand[1]; recData->zero_rand = p->rand[2];
  recData->act_on_doubles = radCR.ActOnDoubles;
  symData->n_elem = N;
  symData->total_copies = total_images;
  g_asm_packs[polyData] = std::move(p);
  return 1;
}

int radGPU_AssembleMatrix(RadGPU_PolyData *polyData, RadGPU_RecMagData *, RadGPU_SymData *, RadGPU_ObsQuadData *,
                          RadGPU_AsmResult *result)
{
  auto it = g_asm_packs.find(polyData);
  if (it == g_asm_packs.end() || !result) return -1;
  Pack &p = *it->second;
  const RadB200Geom g = p.geom();
  const RadB200Relax r = p.relax();
  const int N = r.n_elem;
  drop_pending();
  int64_t h = 0;
  int rc = with_room([&] { return radb200_intrc_create(&g, &r, nullptr, RADB200_STORE_F32, &h); });
  if (rc != 0) {
    say("assembly failed", radb200_last_error());
    return -1;
  }
  // the core owns a host copy (delete[] in radTInteraction), its CPU
  // consumers read it; the device copy stays resident
  const long long n3 = 3LL * N;
  float *host = new (std::nothrow) float[(size_t)(n3 * n3)];
  if (!host) {
    radb200_intrc_free(h);
    say("assembly failed", "no host memory for the matrix copy");
    return -1;
  }
  rc = radb200_intrc_matrix(h, 0, host);
  if (rc != 0) {
    delete[] host;
    radb200_intrc_free(h);
    say("assembly failed", radb200_last_error());
    return -1;
  }
  result->N = N;
  result->matrix_blocks = host;
  g_pending.handle = h;
  g_pending.n = N;
  g_pending.mat_kind = p.mat_kind;
  g_pending.mat = p.mat;
  g_pending.mh = p.mh;
  return 0;
}

void radGPU_FreeAsmData(RadGPU_PolyData *polyData, RadGPU_RecMagData *, RadGPU_AsmResult *result)
{
  g_asm_packs.erase(polyData);
  if (result && result->matrix_blocks) { delete[] result->matrix_blocks; result->matrix_blocks = nullptr; }
}

void radGPU_FreeObsQuadData(RadGPU_ObsQuadData *) {}

void radGPU_FreeSymData(RadGPU_SymData *) {}

void radGPU_PublishAssembledMatrix(unsigned long long stamp)
{
  if (!g_pending.handle) return;
  auto old = g_res.find(stamp);
  if (old != g_res.end()) { radb200_intrc_free(old->second.handle); g_res.erase(old); }
  Resident &r = g_res[stamp];
  r.handle = g_pending.handle;
  r.n = g_pending.n;
  r.mat_kind.swap(g_pending.mat_kind);
  r.mat.swap(g_pending.mat);
  r.mh.swap(g_pending.mh);
  r.used = ++g_clock;
  g_pending = Pending();
}

void radGPU_DiscardAssembledMatrix() { drop_pending(); }

// ---- relaxation --------------------------------------------------------------------

int radGPU_PackInteractionData(radTInteraction *I, RadGPURelaxData *d, int need_matrix)
{
  const int N = I->AmOfMainElem;
  d->n = N;
  d->stamp = I->mGpuMatrixStamp;
  d->M.resize(3 * (size_t)N);
  d->H.assign(3 * (size_t)N, 0.0);
  d->hext.resize(3 * (size_t)N);
  for (int i = 0; i < N; i++) {
    radTg3dRelax *el = I->g3dRelaxPtrVect[i];
    d->M[3 * i] = el->Magn.x; d->M[3 * i + 1] = el->Magn.y; d->M[3 * i + 2] = el->Magn.z;
    const TVector3d &h = I->ExternFieldArray[i];
    d->hext[3 * i] = h.x; d->hext[3 * i + 1] = h.y; d->hext[3 * i + 2] = h.z;
    if (!add_material(d->mats, el)) {
      say("relaxation declined", d->mats.why.c_str());
      return 0;
    }
    d->mats.elem_src.push_back(0);
    d->mats.elem_src.push_back(i);
  }
  if (!need_matrix) return 1;
  if (I->mAsmMatrix) { d->matrix = I->mAsmMatrix; return 1; }
  if (!I->InteractMatrix) { say("relaxation declined", "the interaction holds no matrix"); return 0; }
  const size_t n3 = 3 * (size_t)N;
  d->flat.resize(n3 * n3);
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      const TMatrix3df &b = I->InteractMatrix[i][j];
      float *r0 = &d->flat[(3 * i) * n3 + 3 * j], *r1 = r0 + n3, *r2 = r1 + n3;
      r0[0] = b.Str0.x; r0[1] = b.Str0.y; r0[2] = b.Str0.z;
      r1[0] = b.Str1.x; r1[1] = b.Str1.y; r1[2] = b.Str1.z;
      r2[0] = b.Str2.x; r2[1] = b.Str2.y; r2[2] = b.Str2.z;
    }
  d->matrix = d->flat.data();
  return 1;
}

void radGPU_UnpackMagnetization(RadGPURelaxData *d, radTInteraction *I)
{
  for (int i = 0; i < d->n; i++) {
    TVector3d m(d->M[3 * i], d->M[3 * i + 1], d->M[3 * i + 2]);
    I->g3dRelaxPtrVect[i]->Magn = m;
    I->NewMagnArray[i] = m;
    if (d->have_H) I->NewFieldArray[i] = TVector3d(d->H[3 * i], d->H[3 * i + 1], d->H[3 * i + 2]);
  }
}

namespace {

// The device interaction of the core's interaction (stamp d.stamp), loaded
// from the host matrix of the pack when it is not resident, with the
// materials of the pack.
int64_t resident_for(RadGPURelaxData &d)
{
  auto it = g_res.find(d.stamp);
  const RadB200Relax r = d.mats.relax();
  if (it != g_res.end() && it->second.n == d.n) {
    Resident &res = it->second;
    res.used = ++g_clock;
    if (res.mat_kind != d.mats.mat_kind || res.mat != d.mats.mat || res.mh != d.mats.mh) {
      if (radb200_intrc_set_materials(res.handle, &r) != 0) { say("relaxation failed", radb200_last_error()); return 0; }
      res.mat_kind = d.mats.mat_kind; res.mat = d.mats.mat; res.mh = d.mats.mh;
    }
    return res.handle;
  }
  if (!d.matrix) { say("relaxation failed", "matrix not resident and not packed"); return 0; }
  int64_t h = 0;
  int rc = with_room([&] { return radb200_intrc_load(&r, d.matrix, d.hext.data(), &h); });
  if (rc != 0) { say("relaxation failed", radb200_last_error()); return 0; }
  Resident &res = g_res[d.stamp];
  res.handle = h; res.n = d.n; res.mat_kind = d.mats.mat_kind; res.mat = d.mats.mat; res.mh = d.mats.mh;
  res.used = ++g_clock;
  return h;
}

bool is_resident(unsigned long long stamp) { return g_res.count(stamp) != 0; }

// Device part of a relaxation of a packed interaction; st: misfit, max |M|,
// max |H|, iterations.
int relax_device(RadGPURelaxData &d, int method, double prec, int max_iter, double omega, double *st)
{
  const int64_t h = resident_for(d);
  if (!h) return -1;
  int rc = radb200_intrc_set_extfield(h, d.hext.data());
  if (rc == 0) rc = radb200_relax(h, method, prec, max_iter, 0, omega, d.M.data(), d.H.data(), st);
  if (rc != 0) {
    say(method == RADB200_RLX_NEWTON ? "method 11 failed" : "method 9 failed", radb200_last_error());
    return -1;
  }
  d.have_H = true;
  return 0;
}

}  // namespace

// Method 9 (radrlmet_gpu.cpp:9-51 of the reference glue): reset M unless
// asked not to, relax on the device, write M, H and the status back.
int radGPU_AutoRelax(radTInteraction *I, double prec, int max_iter, char no_reset, double omega)
{
  if (!I || I->AmOfMainElem <= 0) return 0;
  if (!no_reset) I->ResetM();
  I->ResetAuxParam();
  RadGPURelaxData d;
  if (!radGPU_PackInteractionData(I, &d, is_resident(I->mGpuMatrixStamp) ? 0 : 1)) return -1;
  double st[4] = {0, 0, 0, 0};
  if (relax_device(d, RADB200_RLX_JACOBI, prec, max_iter, omega, st) != 0) return -1;
  radGPU_UnpackMagnetization(&d, I);
  I->RelaxStatusParam.MisfitM = st[0];
  I->RelaxStatusParam.MaxModM = st[1];
  I->RelaxStatusParam.MaxModH = st[2];
  return (int)st[3];
}

// Method 11 (radrlmet_gpu.cpp:55-97): the same with Newton-Krylov.
int radGPU_AutoRelaxNK(radTInteraction *I, double prec, int max_iter, char no_reset, double omega)
{
  if (!I || I->AmOfMainElem <= 0) return 0;
  if (!no_reset) I->ResetM();
  I->ResetAuxParam();
  RadGPURelaxData d;
  if (!radGPU_PackInteractionData(I, &d, is_resident(I->mGpuMatrixStamp) ? 0 : 1)) return -1;
  double st[4] = {0, 0, 0, 0};
  if (relax_device(d, RADB200_RLX_NEWTON, prec, max_iter, omega, st) != 0) return -1;
  radGPU_UnpackMagnetization(&d, I);
  I->RelaxStatusParam.MisfitM = st[0];
  I->RelaxStatusParam.MaxModM = st[1];
  I->RelaxStatusParam.MaxModH = st[2];
  return (int)st[3];
}

// ---- field -----------------------------------------------------------------------------
namespace {

// Depth-first walk of an object tree in the core's order: containers iterate
// their members in handle order (radTGroup::GroupMapOfHandlers), the
// transformation list of every object is appended to its parent's (front =
// outermost, radg3d.h:871-875).
bool walk(radTg3d *g, Chain &chain, Pack &p)
{
  const size_t base = chain.size();
  for (auto &pr : g->g3dListOfTransform) {
    radTrans *t = radTCast::TransCast(pr.Handler_g.rep);
    if (!t) { p.why = "transformation list entry is not a transformation"; return false; }
    chain.push_back(std::make_pair(pr.m, affine_of(t)));
  }
  bool ok = true;
  if (radTGroup *grp = radTCast::GroupCast(g)) {
    for (auto &kv : grp->GroupMapOfHandlers) {
      radTg3d *c = radTCast::g3dCast(kv.second.rep);
      if (!c) { p.why = "container member is not a 3-D object"; ok = false; break; }
      if (!(ok = walk(c, chain, p))) break;
    }
  } else {
    std::vector<double> recs;
    images_of(chain, 0, affine_identity(), recs);
    int32_t first = 0, count = 0;
    p.add_run(recs, &first, &count);
    if (radTg3dRelax *el = radTCast::g3dRelaxCast(g)) {
      if (radTRecMag *rm = radTCast::RecMagCast(el)) add_rec(p, rm, el->Magn, first, count);
      else if (radTPolyhedron *ph = radTCast::PolyhedronCast(el)) ok = add_poly(p, ph, el->Magn, first, count);
      else { p.why = "object without a device field form (e.g. an extruded polygon)"; ok = false; }
    } else if (radTArcCur *a = dynamic_cast<radTArcCur *>(g)) {
      if (a->BasedOnPrecLevel) { p.why = "arc segmented by precision level"; ok = false; }
      else {
        const double r[RADB200_ARC_STRIDE] = {a->CircleCentrPoint.x, a->CircleCentrPoint.y, a->CircleCentrPoint.z,
                                              a->R_min, a->R_max, a->Phi_min, a->Phi_max, a->Height, a->J_azim,
                                              (double)(a->NumberOfSectors > 0 ? a->NumberOfSectors : 1)};
        p.arc.insert(p.arc.end(), r, r + RADB200_ARC_STRIDE);
        p.arc_img.push_back(first);
        p.arc_img.push_back(count);
      }
    } else if (radTBackgroundFieldSource *b = dynamic_cast<radTBackgroundFieldSource *>(g)) {
      put3(p.bkg, b->BackgrB);
      p.bkg_img.push_back(first);
      p.bkg_img.push_back(count);
    } else {
      p.why = "object without a device field form";
      ok = false;
    }
  }
  chain.resize(base);
  return ok;
}

int field_of(radTg3d *g, double *pts, int np, double *out, int use_gpu)
{
  if (!g || !pts || !out || np <= 0) return -1;
  Pack p;
  guard_from_core(p);
  Chain chain;
  if (!walk(g, chain, p)) {
    say("field declined", p.why.c_str());
    return -1;
  }
  const RadB200Geom geom = p.geom();
  // use_gpu 1: FP64 with the reference's face-by-face polygon form; 2: FP32
  // terms with FP64 offsets and sums (the reference's fp32 face kernel)
  int rc = radb200_field(&geom, pts, np, 0, use_gpu == 2 ? 1 : 0, out);
  if (rc != 0) {
    say("field failed", radb200_last_error());
    return -1;
  }
  return 0;
}

}  // namespace

int radGPU_ComputeField(int indObj, double *arCoord, int nP, double *arB, int use_gpu)
{
  auto it = rad.GlobalMapOfHandlers.find(indObj);
  if (it == rad.GlobalMapOfHandlers.end()) return -1;  // the core's CPU path reports the bad key
  return field_of(radTCast::g3dCast(it->second.rep), arCoord, nP, arB, use_gpu);
}

int radGPU_ComputeFieldFromSrcRep(void *srcRepPtr, double *arCoord, int nP, double *arB, int use_gpu)
{
  return field_of(radTCast::g3dCast((radTg *)srcRepPtr), arCoord, nP, arB, use_gpu);
}

// ---- exports beyond the reference seam -------------------------------------------------
// Capabilities the reference has no GPU path for, on interactions made by
// rad.RlxPre: the device direct solve of a linear model (no counterpart in
// the reference) through its element handle.
extern "C" {

// Solves (I - X N) M = X H_ext + Mr of the interaction with handle key on
// the device (radb200_direct_solve: mode 0 FP64 LU, 1 TF32 tensor-core LU +
// FP64 GMRES-IR) and writes the magnetization back into the elements, as a
// relaxation would.  status [4]: as radb200_direct_solve.  Returns 0, or a
// negative RADB200_E_* code (message from radb200_last_error).
__attribute__((visibility("default"))) int radB200_DirectSolve(int key, int mode, double rtol, int max_iter,
                                                                double *status)
{
  radThg hg;
  if (!rad.ValidateElemKey(key, hg)) return RADB200_E_HANDLE;
  radTInteraction *I = radTCast::InteractCast(hg.rep);
  if (!I || !status) return RADB200_E_ARG;
  RadGPURelaxData d;
  if (!radGPU_PackInteractionData(I, &d, is_resident(I->mGpuMatrixStamp) ? 0 : 1)) return RADB200_E_UNSUPPORTED;
  if (d.n <= 0) return RADB200_E_ARG;
  const int64_t h = resident_for(d);
  if (!h) return RADB200_E_NOMEM;
  int rc = radb200_intrc_set_extfield(h, d.hext.data());
  if (rc == 0) rc = radb200_direct_solve(h, mode, rtol, max_iter, d.M.data(), status);
  if (rc != 0) return rc;
  radGPU_UnpackMagnetization(&d, I);
  return 0;
}
}
