// internal.cuh -- shared declarations of the libradb200 translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "../../include/radb200.h"
#include "formulas.cuh"

namespace rb {

// ---- errors / bookkeeping --------------------------------------------------
void set_error(const char *fmt, ...);
extern long long g_launches;          // kernels launched by this library
int check_launch(const char *what);   // cudaGetLastError after a launch

#define RB_CUDA(x)                                                                  \
  do {                                                                              \
    cudaError_t e_ = (x);                                                           \
    if (e_ != cudaSuccess) {                                                        \
      ::rb::set_error("%s:%d %s: %s", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
      return RADB200_E_CUDA;                                                        \
    }                                                                               \
  } while (0)
// RADB200_TIMING=1 prints the phases of interaction creation and field
// calls on stderr; each mark synchronizes the device first, so a phase
// includes its kernels.  Off: a mark costs one branch.
struct PhaseClock {
  bool on;
  double t;
  double tm0[3];
  PhaseClock();
  void mark(const char *what);
};
bool timing_on();
double now_s();
extern double g_tm[3];  // seconds in cudaMalloc, cudaFree, cudaMemcpy of DBufs (timing on)

#define RB_TRY(x)            \
  do {                       \
    int r_ = (x);            \
    if (r_ != 0) return r_;  \
  } while (0)

// ---- device buffers ----------------------------------------------------------
// Every DBuf block comes from a per-device pool (pool_alloc / pool_free in
// capi.cu).  Blocks above SMALL_MAX have their exact size and are reused by
// any request up to 25% smaller (an interaction's 10-60 GB of matrix and
// factors would otherwise be unmapped and mapped again by every
// create/free); smaller ones are rounded up to a power of two and reused by
// class.  cudaMalloc and cudaFree on a busy device can each take tens of
// milliseconds (cudaFree also synchronizes), which for the dozens of small
// buffers of an interaction adds up to a large share of its assembly.
constexpr size_t BIG_BLOCK = (size_t)256 << 20;
constexpr size_t SMALL_MAX = BIG_BLOCK / 2;
void *pool_alloc(size_t b, size_t *got);  // nullptr on failure (error set)
void pool_free(void *p, size_t b);
void pool_release_all();

struct DBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DBuf() {}
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { release(); }
  void release()
  {
    if (p) {
      const double t0 = timing_on() ? now_s() : 0.0;
      pool_free(p, bytes);
      if (t0 > 0.0) g_tm[1] += now_s() - t0;
    }
    p = nullptr;
    bytes = 0;
  }
  int alloc(size_t b)
  {
    if (b <= bytes && p) return 0;
    release();
    if (b == 0) return 0;
    const double t0 = timing_on() ? now_s() : 0.0;
    size_t got = 0;
    p = pool_alloc(b, &got);
    if (t0 > 0.0) g_tm[0] += now_s() - t0;
    if (!p) return RADB200_E_NOMEM;
    bytes = got;
    return 0;
  }
  int upload(const void *h, size_t b)
  {
    RB_TRY(alloc(b));
    const double t0 = timing_on() ? now_s() : 0.0;
    if (b) RB_CUDA(cudaMemcpy(p, h, b, cudaMemcpyHostToDevice));
    if (t0 > 0.0) g_tm[2] += now_s() - t0;
    return 0;
  }
  template <typename T> T *as() const { return (T *)p; }
};

// ---- tetrahedral meshes by their unique vertices, edges and faces -----------
// The vertex/edge form sums, per tetrahedron, a logarithm per edge and a
// solid angle per face.  Tetrahedra of a mesh share vertices, edges and
// faces, and the sum is linear in the per-edge and per-face coefficients, so
// the field of all tetrahedra under one image transform is evaluated once per
// UNIQUE edge (coefficients G summed over the tetrahedra sharing it) and per
// unique face (A = sum of s a_f, s = +-1 the face's orientation in each
// tetrahedron against the face's own).  Tiles group spatially close
// tetrahedra: up to MESH_VT vertices whose distances to the point are
// computed once per tile, and the edges and faces the tile owns (each unique
// edge or face belongs to exactly one tile).
constexpr int MESH_VT = 32, MESH_EMAX = 128, MESH_FMAX = 160;
constexpr int MESH_E = 6;   // edge record: a, b (tile-local vertices), l, G (3)
constexpr int MESH_F = 13;  // face record: a, b, c, l_ab, l_ac, l_bc, m (3, unnormalized normal), v_a . m, A (3)
struct MeshView {
  int n_tiles = 0;
  const int4 *tile = nullptr;   // [2 per tile] {first vertex slot, vertices, first edge, edges}, {first face, faces, transform, 0}
  const double *mv = nullptr;   // tile-local vertices, 3 doubles per slot (object frame of the transform)
  const double *me = nullptr;   // [edges * MESH_E]
  const double *mf = nullptr;   // [faces * MESH_F]
  int n_groups = 0;
  const int4 *group = nullptr;  // {first entry of gtet, tetrahedra, transform, 0}
  const double *gbox = nullptr; // [groups * 6] bounding box (lo, hi) in the transform's object frame
  const int *gtet = nullptr;    // polyhedron index of every tetrahedron of each group
};

// ---- geometry on the device --------------------------------------------------
// Kernel-side view (passed by value).  Mirrors RadB200Geom plus a unit table:
// one unit per (source, image), kinds 0 cuboid, 1 polyhedron, 2 arc, 3 background.
struct GeomView {
  const double *trf;
  const double *rec;
  const int *rec_img;
  const double *poly;
  const int *poly_info;
  const double *face;
  const int *face_vtx;
  const double *vtx2d;
  const double *arc;
  const double *bkg;
  const int4 *units;  // {kind, source, transform, 0}, ordered by kind
  int n_units;
  int ustart[5];      // first unit of each kind (cuboid, polyhedron, arc, background), end
  Guard g;
  TopoView tp;        // vertex/edge form of the polyhedra (tinfo.y < 0: not available)
  const int *tetidx;  // per polyhedron: tetrahedron record or -1
  const double *tetrec;
  int all_tets;       // every polyhedron has a tetrahedron record
  int tet_single;     // ... and the sources are only those tetrahedra, one image each
  int fast;           // 1: evaluate polyhedra in the vertex/edge form
  MeshView mesh;      // all-tetrahedron models: unique edges and faces (n_tiles 0: none)
};

struct DevGeom {
  DBuf trf, rec, rec_img, poly, poly_info, face, face_vtx, vtx2d, arc, bkg, units;
  // polyhedron topology (vertex/edge form), see TopoView in formulas.cuh
  DBuf tinfo, tinfo2, tv, te, tel, teg, teG, tt, ttm, tfn, tfa;
  DBuf tetidx, tetrec;  // fixed-topology tetrahedron records (tet_fast)
  DBuf m_tile, m_v, m_e, m_f, m_group, m_gbox, m_gtet;  // mesh form (MeshView)
  int m_tiles = 0, m_groups = 0;
  int n_units = 0, n_rec = 0, n_poly = 0;
  int ustart[5] = {0, 0, 0, 0, 0};
  int all_tets = 0, tet_single = 0;
  Guard g{0, 0, 0};
  int upload(const RadB200Geom *G, bool tensor_coeffs = false, bool mesh = true);
  GeomView view(int fast = 0) const;
};

// ---- near blocks of mixed storage ------------------------------------------
// With RADB200_STORE_MIXED every block is stored in FP32 and the pairs within
// the near range additionally keep their FP64 residue D = N(FP64) - N32, in
// CSR by observer element (ptr, col, D [nnz][9]) and indexed by source element
// for the transposed product (tptr, tidx: entry numbers grouped by column).
struct NearView {
  const int *ptr = nullptr;
  const int *col = nullptr;
  const double *D = nullptr;
  const int *tptr = nullptr;
  const int *tidx = nullptr;
  const int *row = nullptr;  // observer element of each entry
};

// ---- interaction state -------------------------------------------------------
struct Intrc {
  int n = 0;        // elements
  int e0 = 0;       // first observer row held (row blocks; 0 otherwise)
  int nr = 0;       // observer rows held: n, or e1 - e0 for a row block
  int n3 = 0;       // 3n
  int ld = 0;       // padded leading dimension of N (multiple of 32)
  int storage = 0;
  int fast = 0;     // polyhedra in the vertex/edge form
  int geom_ok = 1;  // 0: loaded from a matrix assembled elsewhere (no element geometry)
  DevGeom geom;     // relaxable elements (object frames, images)
  DBuf elem_src, obs, rowT;           // [2n] int, [3n] obs points, [9n] s*Minv of main image
  DBuf N32, N64;                      // [n3 x ld]
  DBuf near_ptr, near_row, near_col, near_D, near_tptr, near_tidx;  // mixed storage: FP64 residue of near pairs
  int64_t near_nnz = 0;
  double near_factor = 0.0;           // near range: centre distance <= factor * (r_i + r_j)
  NearView near() const
  {
    NearView v;
    if (near_nnz > 0) {
      v.ptr = near_ptr.as<int>(); v.col = near_col.as<int>(); v.D = near_D.as<double>();
      v.tptr = near_tptr.as<int>(); v.tidx = near_tidx.as<int>(); v.row = near_row.as<int>();
    }
    return v;
  }
  DBuf hext;                          // [ld]
  DBuf mat_kind, mat, mh;             // materials
  std::vector<int> h_mat_kind;
  std::vector<double> h_mat;
  // solver work buffers
  DBuf M, H, Mp, F, part, work;
  // LU factors (row-major [n3 x ld]) and solve state
  DBuf LU32, LU64, lu_scratch;
  DBuf LUinv;                         // [2][3N x 128] inverses of the diagonal blocks (L, then U)
  DBuf tri_sync;                      // counters and flags of the one-launch triangular sweeps
  DBuf sweep_m;                       // FP32 factors: per block Linv_k L_{k,k-1}, then Uinv_k U_{k,k+1} (128 x 128 each)
  int lu_tc = 0;                      // the factorization ran on the tensor cores
  int lu_mode = -1;                   // factors valid for this mode (-1 none)
  int lu_of_d = 0;                    // 1: the factors are of I - D N at the converged state of solve lu_solve_id
  double lu_shift = 0.0;              // sigma when the factors are of A + sigma I (a pivot fell below the threshold)
  int lu_solve_id = -1;
  int solve_id = 0;                   // counts relaxations / direct solves on this interaction
  uint64_t stamp = 0;                 // hash of the element records, frames and materials
  DBuf lastM, lastH;                  // converged state of the last solve
  int last_kind = -1;                 // 0 relax, 1 direct
  // adjoint: external sources (kept for the gradient of H_ext at the centres),
  // element kinds and d(obs_e)/d(centre_e) of each element's main image
  DevGeom xgeom;
  int has_ext = 0;
  std::vector<int> h_elem_src;        // [2n]
  std::vector<double> h_obsJ;         // [9n] row-major
  // the triangular solves with the current factors, captured once as CUDA
  // graphs ([0] A^-1, [1] A^-T) acting on lu_gx; dropped when the factors change
  cudaGraphExec_t lu_graph[2] = {nullptr, nullptr};
  long long lu_graph_kernels[2] = {0, 0};  // kernels per replay (launch counter)
  DBuf lu_gx;
  void drop_lu_graphs()
  {
    for (auto &g : lu_graph)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }
  ~Intrc() { drop_lu_graphs(); }
};

// ---- small vector helpers (relax.cu) ---------------------------------------
constexpr int MD_MAX = 16;
struct DotSet {            // out[k] = <a_k, b_k>
  const double *a[MD_MAX];
  const double *b[MD_MAX];
  int nd;
};
struct AxpySet {           // y = (accumulate ? y : 0) + sum_k c_k v_k
  const double *v[MD_MAX];
  double c[MD_MAX];
  int nv;
};
int multidot(const DotSet &ds, int64_t len, double *host_out, DBuf &part, DBuf &scal, cudaStream_t st);
int lincomb(const AxpySet &s, int64_t len, double *y, int accumulate, cudaStream_t st);
int run_matvec(Intrc &I, const double *x, const double *b, double alpha, double *y, cudaStream_t st);
int run_matvec_f32(Intrc &I, const double *x, const double *b, double alpha, double *y, cudaStream_t st);
int launch_round_f32(const double *a, float *b, size_t n, cudaStream_t st);

// linear operator + preconditioner for GMRES (krylov.cu)
struct Op {
  virtual int apply(const double *v, double *out) = 0;  // out = A v
  virtual int precond(double *v) = 0;                   // v <- P v
  virtual ~Op() {}
};
int gmres(Op &op, int n3, int ld, const double *b, double *x, double rtol, int max_iter, int restart, double *relres,
          int *iters, cudaStream_t st);
int lu_precond(Intrc &I, double *x, cudaStream_t st);
int relax_jacobi(Intrc &I, double prec, int max_iter, double omega0, double *status);
int lu_precond_transposed(Intrc &I, double *x, cudaStream_t st);
// factor A = I - X N with X [n x RADB200_MAT_STRIDE] (3x3 in the first 9
// slots) into the interaction's LU buffers; of_d marks factors of I - D N
int lu_build_x(Intrc &I, int mode, const double *X, int of_d, double *factor_seconds);

// TF32 tensor-core GEMM update (gemm_tc.cu); *used = 0 when the shape is not
// supported and the caller must fall back to the CUDA-core GEMM.
// C[m x n] -= A[m x k] B[k x n] (overwrite != 0: C = A B), FP32 row-major,
// any k, leading dimensions multiples of 4, 16-byte aligned pointers, C not
// aliasing A or B.  A is rounded to TF32 in place.
// slot selects one of two B^T scratch buffers (updates on two streams must use
// different slots); max_ctas > 0 caps the persistent grid
int tc_gemm_f32(float *C, int ldc, int m, int n, int k, float *A, int lda, const float *B, int ldb, cudaStream_t st,
                int *used, int overwrite = 0, int slot = 0, int max_ctas = 0);
int tc_gemm_f32_inplace(float *C, int ldc, int m, int n, int k, float *A, int lda, const float *B, int ldb,
                        cudaStream_t st, int *used, bool c_is_a, int slot = 0);
int tc_error_flag(int *flag);  // 2 when a tensor-core CTA hit its wait limit

// ---- kernels (launch wrappers) ---------------------------------------------
int launch_field(const GeomView &g, const double *d_pts, int64_t npts, int what, int precision,
                 double *d_out, DBuf &scratch, cudaStream_t st);
int launch_assemble(const GeomView &g, const int *elem_src, const double *obs, const double *rowT, int nr, int n,
                    int ld, float *N32, double *N64, cudaStream_t st);
int launch_rowtrans_vec(const double *rowT, const double *in, double *out, int n, cudaStream_t st);
// mesh form of an all-tetrahedron geometry from its tetrahedron records
// (mesh.cu); tetidx[p] = record of polyhedron p
int build_mesh(const RadB200Geom *G, const std::vector<int> &tetidx, const std::vector<double> &tetrec, DevGeom &dg);
// field of the tetrahedra in the mesh form, all units of kind polyhedron
// (what 0 B, 1 H; mesh.cu)
int launch_mesh_field(const GeomView &g, const double *d_pts, int64_t npts, int what, int precision, double *d_out,
                      int accumulate, DBuf &scratch, cudaStream_t st);
// near lists of mixed storage from the element geometry (host, near.cu);
// obs: [3n] element centres (main images)
int build_near(Intrc &I, const RadB200Geom *elems, const RadB200Relax *r, const double *obs);
// FP64 residue of the near pairs: D[k] = block(row[k], col[k]) - N32 (assemble.cu)
int launch_assemble_near(const GeomView &g, const int *elem_src, const double *obs, const double *rowT, int ld,
                         const float *N32, const int *row, const int *col, int64_t nnz, double *D, cudaStream_t st);
// out[j] += sum over near entries (i, j) of D_ij^T x_i (near.cu)
int launch_near_t(const Intrc &I, const double *x, double *out, cudaStream_t st);
// electron trajectories, one CTA each (field.cu); prec NULL: one RK4 step per
// tabulation interval, else step-doubling control with these [4] accuracies
int launch_trajectories(const GeomView &g, double energy_gev, const double *d_init, int n_traj, double y0, double y1,
                        int np, const double *prec, double *d_out, int *d_status, cudaStream_t st);

}  // namespace rb
