/*
 * radb200.h -- C-ABI of the B200 (sm_100a) relaxation hot path for Radia.
 *
 * This library replaces Radia's CUDA plugin layer (the radGPU_* seam between
 * radTInteraction / radTApplication and the device) with a new implementation:
 *   - interaction-matrix assembly     (replaces radGPU_AssembleMatrix,
 *                                       cpp/src/core/radgpu_asm.h:166-173)
 *   - magnetization relaxation        (replaces radGPU_RelaxAuto / radGPU_RelaxNK,
 *                                       cpp/src/core/radgpurlx.h:69-87)
 *   - dense direct solve, adjoint     (no counterpart in the reference)
 *   - B/H field evaluation            (replaces radGPU_ComputeField,
 *                                       cpp/src/core/radgpu_fld.h:107-198, and
 *                                       the host coil loop radgpu_fld.cpp:542-617)
 *
 * Every entry point takes plain pointers and sizes.  Geometry is handed over
 * as flat arrays (RadB200Geom), which is what the reference's packers
 * (radGPU_PackGeometryForAsm radgpu_asm.cpp:206-444, CollectElementsRecursive
 * radgpu_fld.cpp:194-317) produce from the object tree; the difference is that
 * symmetry / orientation images stay a separate transform table which the
 * kernels apply in-kernel instead of duplicating records on the host.
 *
 * Conventions (identical to the reference): lengths in mm, B, H and M in
 * Tesla (mu0*H), current density in A/mm^2.  All functions return 0 on
 * success and a negative RADB200_E* code on failure; radb200_last_error()
 * returns a message.  No function aborts or traps.  The library is not
 * reentrant (one global device context, like the reference's static caches).
 */
#ifndef RADB200_H
#define RADB200_H

#include <stdint.h>

#if defined(__GNUC__)
#define RADB200_API __attribute__((visibility("default")))
#else
#define RADB200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------- */
#define RADB200_OK            0
#define RADB200_E_ARG        -1   /* bad argument / size                     */
#define RADB200_E_CUDA       -2   /* CUDA runtime error                      */
#define RADB200_E_NOMEM      -3   /* device allocation failed / too large    */
#define RADB200_E_HANDLE     -4   /* unknown interaction handle              */
#define RADB200_E_NUMERIC    -5   /* non-finite result / breakdown           */
#define RADB200_E_NOCONV     -6   /* iteration cap reached before tolerance  */
#define RADB200_E_TIMEOUT    -7   /* a bounded device wait ran out           */
#define RADB200_E_UNSUPPORTED -8  /* feature not available for this input    */

/* ---- image transform record -------------------------------------------
 * One record per (source, image).  Mirrors gmTrans (ext/genmath/gmtrans.h:22-84):
 * an image maps a point of the source's own frame to the lab frame as
 * P_lab = M*P + V and a field vector as F_lab = s*M*F (TrVectField).
 * Stored as RADB200_TRF_STRIDE doubles:
 *   [0..8]   M^-1 (row major)      P_obj = M^-1 * (P_lab - V)
 *   [9..11]  V
 *   [12..20] s*M (row major)       field map object frame -> lab frame
 *   [21]     s                     [22] det(M)    [23] unused               */
#define RADB200_TRF_STRIDE 24

/* ---- source records ------------------------------------------------------ */
#define RADB200_REC_STRIDE  12  /* cx cy cz  wx wy wz  mx my mz  jx jy jz      */
#define RADB200_POLY_STRIDE 6   /* centre xyz (vertex mean), magnetization xyz */
#define RADB200_FACE_STRIDE 10  /* R (9, object -> face-local rows), coordZ    */
#define RADB200_ARC_STRIDE  10  /* cx cy cz rmin rmax phimin phimax h j nseg   */

typedef struct RadB200Geom {
  int32_t n_trf;             /* transform table                              */
  const double *trf;         /* [n_trf * RADB200_TRF_STRIDE]                 */

  int32_t n_rec;             /* rectangular blocks: radTRecMag (M and/or J)  */
  const double *rec;         /* [n_rec * RADB200_REC_STRIDE], object frame   */
  const int32_t *rec_img;    /* [n_rec * 2] first transform, image count     */

  int32_t n_poly;            /* polyhedra: radTPolyhedron                    */
  const double *poly;        /* [n_poly * RADB200_POLY_STRIDE]               */
  const int32_t *poly_info;  /* [n_poly * 4] first face, faces, first trf, images */
  int32_t n_face;
  const double *face;        /* [n_face * RADB200_FACE_STRIDE]               */
  const int32_t *face_vtx;   /* [n_face * 2] first 2-D vertex, vertex count  */
  int32_t n_vtx;
  const double *vtx2d;       /* [n_vtx * 2] counter-clockwise, face frame    */

  int32_t n_arc;             /* arc currents: radTArcCur, trapezoid in phi   */
  const double *arc;         /* [n_arc * RADB200_ARC_STRIDE]                 */
  const int32_t *arc_img;    /* [n_arc * 2]                                  */

  int32_t n_bkg;             /* uniform background fields: ObjBckg           */
  const double *bkg;         /* [n_bkg * 3]                                  */
  const int32_t *bkg_img;    /* [n_bkg * 2]                                  */

  /* length-randomization guard magnitudes (radTConvergRepair,
   * cpp/src/core/radcnvrg.h:29-92); all zero after FldLenRndSw('off'). */
  double abs_rand, rel_rand, zero_rand;
} RadB200Geom;

/* ---- relaxable elements and materials -----------------------------------
 * Element e is source rec[elem_src[2e+1]] (elem_src[2e]==0) or
 * poly[elem_src[2e+1]] (elem_src[2e]==1).  Its FIRST image is its main
 * transform (all symmetry powers zero, radintrc.cpp:557-573); magnetization
 * and field of the relaxation live in that frame (the element's own frame).
 * Material record, RADB200_MAT_STRIDE doubles per element:
 *   kind 0 (linear):   [0..8] chi tensor, [9..11] Mr          (radmater.h:164-362)
 *   kind 1 (tanh):     [0..2] ksi_i, [3..5] ms_i, [6] count, [9..11] Mr
 *                      |M| = sum ms_i tanh(ksi_i |H| / ms_i)  (radmater.h:417-600)
 *   kind 2 (table):    [0] first row, [1] rows (>= 2, H ascending) of
 *                      mh_table (H, M, dM/dH), [9..11] Mr; |M|(|H|) cubic
 *                      between the rows (radmater.cpp:618-710), M || H     */
#define RADB200_MAT_STRIDE 12
#define RADB200_MAT_LINEAR 0
#define RADB200_MAT_TANH   1
#define RADB200_MAT_TABLE  2

typedef struct RadB200Relax {
  int32_t n_elem;
  const int32_t *elem_src;   /* [n_elem * 2] kind (0 rec, 1 poly), index     */
  const int32_t *mat_kind;   /* [n_elem]                                     */
  const double *mat;         /* [n_elem * RADB200_MAT_STRIDE]                */
  int32_t n_mh;
  const double *mh_table;    /* [n_mh * 3]  H, M, dM/dH                      */
} RadB200Relax;

/* ---- general ------------------------------------------------------------- */
RADB200_API const char *radb200_last_error(void);
RADB200_API int radb200_version(void);                      /* 100 * major + minor       */
/* Number of this library's kernels launched since load (all entry points). */
RADB200_API int64_t radb200_kernel_launches(void);
RADB200_API int radb200_device_sync(void);
/* Profiling hook, no counterpart in the reference: CUDA-event timing of the
 * dense LU's trailing updates on their own stream.  radb200_update_timing(1)
 * starts collecting (and clears), 0 stops; radb200_update_stats returns the
 * launches timed, their summed device seconds, algorithmic bytes (C read and
 * written, panels read once) and flops (2 m^2 K per update) since then.      */
RADB200_API int radb200_update_timing(int on);
RADB200_API int radb200_update_stats(int64_t *launches, double *seconds, double *bytes, double *flops);
/* Diagnostics, no counterpart in the reference: measured FMA throughput of
 * the FP64 (fp64 != 0) or FP32 pipe of the current device in TFLOP/s, the
 * roofline denominator of the transcendental-bound assembly / field kernels. */
RADB200_API int radb200_measure_fma_peak(int fp64, double *tflops);
/* Diagnostics, no counterpart in the reference: runs (once) the self-test of
 * the LU's tcgen05 GEMM kernels against a CUDA-core GEMM.
 * state: 0 tensor-core path disabled, 1 the cp.async-fed kernel (TF32) in
 * use, 2 the TMA-fed kernel with TF32 operands, 3 the TMA-fed kernel with
 * FP16 operands scaled per row and column; err: max relative deviation seen
 * by the first kernel of the chain.                                         */
RADB200_API int radb200_tc_selftest(int *state, double *err);

/* ---- field evaluation ------------------------------------------------------
 * Replaces radGPU_ComputeField (radgpu_fld.h:183-198) and the reference's
 * host coil loop.  what: 0 = B, 1 = H, 2 = M (magnetization at the point).
 * precision: 0 = FP64 with the reference's face-by-face polygon form;
 * 1 = FP32 terms (FP64 vertex offsets and accumulation; the reference's
 * use_gpu == 2); 2 = FP64 with the vertex/edge polyhedron form.  pts/out are HOST arrays [npts*3]; the
 * call copies them to and from the device.                                   */
RADB200_API int radb200_field(const RadB200Geom *g, const double *pts, int64_t npts,
                  int what, int precision, double *out);
/* No counterpart in the reference: field evaluation for callers that cannot
 * allocate device memory (code running while another part of the process
 * captures a CUDA graph, real-time loops that must stay off the allocator,
 * hosts that hand the library fixed device arenas).  EVERY array is in device
 * memory: the pointer fields of *g, pts and out; the struct itself and its
 * counts are on the host.  FP64, face-by-face polyhedron form.  The call
 * allocates nothing: its only scratch is a static 3 MiB device array that
 * every GPU it runs on keeps until exit.  The driver maps that array when the
 * first call on a device looks up its address (lazy module loading), so the
 * first call can fail for lack of device memory: make it at set-up, outside
 * any stream capture.  At most 16,384 points per call; larger counts are
 * rejected with RADB200_E_ARG.  Calls that overlap on the GPU share the
 * scratch and race: serialize them.  Runs on the calling thread's per-thread
 * default stream (cudaStreamPerThread) and synchronizes it before returning. */
RADB200_API int radb200_field_noalloc(const RadB200Geom *g, const double *d_pts, int64_t npts,
                                      int what, double *d_out);
/* Same, with pts/out already in device memory (cudaStream 0 ordering).      */
RADB200_API int radb200_field_dev(const RadB200Geom *g, const double *d_pts, int64_t npts,
                      int what, int precision, double *d_out);

/* ---- field integrals along a straight line ---------------------------------
 * Replaces radTApplication::ComputeFieldInt (cpp/src/core/radapl3.cpp:356-385),
 * which RadFldInt (cpp/src/lib/radentry.cpp:1310-1325) and radpy FldInt
 * (cpp/src/clients/python/radpy.cpp:2501-2531) call.
 *   P1, P2     [3] host points on the line (mm).
 *   infinite   0: integral from P1 to P2; 1: over the whole line through P1
 *              and P2 (uniform background fields contribute zero there, as in
 *              the reference, radarccu.h:306-316).
 *   what       bit 0: integral of B into out[0..2]; bit 1: of H into out[3..5].
 *   precision  as radb200_field.
 *   abs_prec   absolute accuracy in T mm (the reference's PrcBInt, FldCmpCrt;
 *              its default is 1e-3): adaptive Gauss-Kronrod panels are split
 *              until the sum of their error estimates is below it.
 *   out        [6] host.
 *   status     [6] host or NULL: error estimate (T mm), field points
 *              evaluated, refinement levels, panels, 1 if abs_prec was met
 *              (2 if the panels still above it stopped converging at the
 *              rounding noise of the field, 0 if the level cap was hit),
 *              seconds.                                                       */
RADB200_API int radb200_field_int(const RadB200Geom *g, const double *P1, const double *P2, int infinite,
                                  int what, int precision, double abs_prec, double *out, double *status);
/* Relativistic electron trajectories in the field of g: replaces
 * radTApplication::ComputeParticleTrajectory (cpp/src/core/radapl3.cpp:639-672)
 * behind RadFldPtcTrj / radpy FldPtcTrj (radpy.cpp:2537-2569).
 *   energy_gev  electron energy (GeV).
 *   init        [n_traj * 4] host: x, dx/dy, z, dz/dy at y0 (mm, rad).
 *   y0, y1, np  tabulation y0 + k (y1 - y0) / (np - 1), k = 0 .. np-1.
 *   prec        NULL: one fourth-order Runge-Kutta step per interval (the
 *               reference's default); else [4] accuracies of x, x', z, z'
 *               (the reference's PrcCoord, PrcAngle, PrcCoord, PrcAngle)
 *               for its step-doubling control, 0 meaning none.
 *   out         [n_traj * np * 5] host: y, x, dx/dy, z, dz/dy per point.
 *   status      [n_traj] host or NULL: 0, or 1 step too small (Error200),
 *               2 step limit (Error201), 3 no acceptable step.
 * One CTA per trajectory (the stages of one trajectory are a chain); many
 * trajectories in one call run concurrently.  Returns RADB200_E_NOCONV when
 * any trajectory failed.                                                    */
RADB200_API int radb200_trajectories(const RadB200Geom *g, double energy_gev, int n_traj, const double *init,
                                     double y0, double y1, int np, const double *prec, double *out, int *status);
/* The same quadrature around a caller-supplied point field (no device use):
 * fn(ctx, g', pts, npts, what, out) must write the field (what 0 B, 1 H) of
 * geometry g' at npts host points and return 0; g' is g with the background
 * fields removed for infinite lines.  No counterpart in the reference.      */
typedef int (*RadB200PointField)(void *ctx, const RadB200Geom *g, const double *pts, int64_t npts, int what,
                                 double *out);
RADB200_API int radb200_field_int_cb(const RadB200Geom *g, RadB200PointField fn, void *ctx, const double *P1,
                                     const double *P2, int infinite, int what, double abs_prec, double *out,
                                     double *status);

/* ---- interaction (assembly + solver state) ---------------------------------
 * Replaces radGPU_PackGeometryForAsm + radGPU_AssembleMatrix +
 * radGPU_PublishAssembledMatrix (radgpu_asm.h:149-187): assembles the dense
 * 3N x 3N interaction matrix (block (i,j) = H in element i's frame at i's
 * centre from unit magnetization of element j, images folded in,
 * radintrc.cpp:831-877) and the external field from every non-relaxable
 * source (radintrc.cpp:1208-1234) into device memory, where it stays for the
 * solves.  storage: 0 = FP32 matrix (the reference's layout),
 * 1 = FP64 matrix, 2 = mixed: every block in FP32 and, for the near pairs
 * (an image of element j within RADB200_NEAR_FACTOR (default 1.5) times the
 * sum of the two elements' radii of element i's centre; the self block
 * always), the FP64 residue of the block, which the refinement residual,
 * the relaxation and the adjoint's transposed products add back in FP64.
 * ext may be NULL (no external sources).                                     */
#define RADB200_STORE_F32   0
#define RADB200_STORE_F64   1
#define RADB200_STORE_MIXED 2
/* OR-ed into storage: polyhedron blocks by the vertex/edge form (solid angles
 * + edge logarithms, exact like the face-by-face form of the reference but
 * with ~4x fewer transcendentals); cuboid blocks are unaffected.            */
#define RADB200_ASM_FAST    16
RADB200_API int radb200_intrc_create(const RadB200Geom *elems, const RadB200Relax *r,
                         const RadB200Geom *ext, int storage, int64_t *handle);
RADB200_API int radb200_intrc_free(int64_t handle);
/* Row block of an interaction, for a relaxation split over devices: the rows
 * of observer elements e0 .. e1-1 against every source element (3 (e1-e0) x
 * 3N, FP32 or FP64 storage), with the external field of those rows.  The
 * reference relaxes on one device (radgpurlx.cu); this has no counterpart
 * there.  The handle serves radb200_relax_rows_step and radb200_intrc_free
 * only; every other call rejects it.                                         */
RADB200_API int radb200_intrc_create_rows(const RadB200Geom *elems, const RadB200Relax *r,
                              const RadB200Geom *ext, int storage, int32_t e0, int32_t e1,
                              int64_t *handle);
/* One Jacobi proposal of a row block (the step of RADB200_RLX_JACOBI): from
 * the full magnetization d_M [3N] (device), H = N_rows M + H_ext, each row
 * element's implicit field H' and M' = M(H'); writes d_Mp_rows = M',
 * d_F_rows = M' - M and, unless NULL, d_H_rows = H' of its rows
 * [3 (e1-e0)] (device), and *sq_sum = sum |F_e|^2 over them (host).  The
 * block keeps each row element's field as the start of its next implicit
 * solve.                                                                     */
RADB200_API int radb200_relax_rows_step(int64_t handle, const double *d_M, double prec,
                            double *d_Mp_rows, double *d_F_rows, double *d_H_rows,
                            double *sq_sum);
/* Device blocks are kept for reuse when released: those above 128 MB
 * (matrices, factors) up to RADB200_BUFCACHE_GB (environment; default 40% of
 * the device's memory, 0 = off), so that repeated create / free cycles do
 * not unmap and remap tens of GB each time; smaller ones by power-of-two
 * class up to RADB200_SMALLCACHE_GB (default 2).  No counterpart in the
 * reference.  This call returns every kept block to the driver.             */
RADB200_API int radb200_release_cached_memory(void);
/* Save / restore the device state of an interaction (the solution state that
 * UtiDmp / UtiDmpPrs would carry across processes, radintrc.cpp:1516,1946 of
 * the reference dump the object tree only): the matrix as stored, the
 * external field, the current and last converged magnetization and, when
 * valid, the LU factors with their diagonal-block inverses.
 * radb200_intrc_save: *bytes = size of the state; with buf != NULL and
 * capacity >= that size the state is written there (host memory).
 * radb200_intrc_restore: creates a new interaction from the same geometry,
 * relaxation records, external sources and storage flags WITHOUT assembling
 * and loads the state into it; the geometry stamp (a hash of element centres,
 * frames, sources and materials) and the sizes must match the saved ones,
 * else RADB200_E_ARG.                                                        */
RADB200_API int radb200_intrc_save(int64_t handle, void *buf, int64_t capacity, int64_t *bytes);
RADB200_API int radb200_intrc_restore(const RadB200Geom *elems, const RadB200Relax *r, const RadB200Geom *ext,
                                      int storage, const void *buf, int64_t bytes, int64_t *handle);
RADB200_API int radb200_intrc_size(int64_t handle, int32_t *n_elem, int32_t *storage);
/* Copy the interaction matrix (row major, 3N x 3N) to a host buffer, as FP32
 * or FP64 (dtype 0 / 1), and the external field H_ext [3N].                 */
RADB200_API int radb200_intrc_matrix(int64_t handle, int dtype, void *out);
RADB200_API int radb200_intrc_extfield(int64_t handle, double *out);
/* Replace the external field (e.g. after a source update, RlxUpdSrc).       */
RADB200_API int radb200_intrc_set_extfield(int64_t handle, const double *h_ext);
/* Create an interaction from a matrix assembled elsewhere: replaces the
 * host flatten + upload of radGPU_PackInteractionData (radgpurlx.cpp:25-62,
 * radgpurlx.h:90-96), used when Radia's CPU assembly built the matrix.
 * N: host [3N x 3N] FP32 row major (radTInteraction::mAsmMatrix layout,
 * radintrc.h:99-115); h_ext: host [3N] or NULL (zero).  The interaction has
 * no element geometry: relaxation and direct solves work, the geometric
 * adjoint terms (dL_dc, dL_dd, radb200_field_vjp) return
 * RADB200_E_UNSUPPORTED.                                                     */
RADB200_API int radb200_intrc_load(const RadB200Relax *r, const float *N, const double *h_ext, int64_t *handle);
/* Replace the materials of an interaction (same elements); drops its LU
 * factors.  The reference re-reads each element's material at every
 * relaxation (radgpurlx.cpp:104-196), so a MatApl between RlxPre and RlxAuto
 * takes effect; this is the device side of that.                            */
RADB200_API int radb200_intrc_set_materials(int64_t handle, const RadB200Relax *r);

/* ---- relaxation ------------------------------------------------------------
 * Replaces radGPU_AutoRelax (method 9) and radGPU_AutoRelaxNK (method 11),
 * radrlmet_gpu.cpp:9-99.  method:
 *   RADB200_RLX_JACOBI   device-resident under-relaxed Jacobi with per-element
 *                        implicit material solve and Anderson mixing
 *                        (methods 4/9/10 of the reference reach the same
 *                        fixed point);
 *   RADB200_RLX_NEWTON   Newton-Krylov with right-preconditioned GMRES (method 11).
 * M_io: [3N] magnetization in each element's frame; read when reset == 0,
 * always written.  H_out: [3N] or NULL.  status: [4] = misfit (RMS of the last
 * undamped step, T), max|M|, max|H|, iterations (radsend.cpp:1009-1024).   */
#define RADB200_RLX_JACOBI 0
#define RADB200_RLX_NEWTON 1
RADB200_API int radb200_relax(int64_t handle, int method, double prec, int max_iter,
                  int reset, double omega, double *M_io, double *H_out,
                  double *status);

/* ---- dense direct solve (linear materials) --- no counterpart in the reference.
 * Solves (I - X N) M = X H_ext + Mr by a blocked unpivoted LU of
 * A = I - X N on the device, then FP64 GMRES on A (the FP64 operator) with
 * the factors as right preconditioner, to rtol.  mode: RADB200_LU_F64 = FP64
 * factors; RADB200_LU_TF32 = FP32 factors whose updates run on the tcgen05
 * tensor cores (FP16 operands scaled per row and column by powers of two, or
 * TF32 operands; FP32 accumulation).  A pivot at or below 1e-12 of the
 * largest |A_ii| makes the factorization restart on A + sigma I (sigma = 1e-3
 * of that scale, at least 1e-3); GMRES still solves with A, so the shifted
 * factors only precondition it (radb200_lu_shift reports sigma).  For
 * chi >= 0 this never happens.  The factorization is kept with the
 * interaction for later solves (adjoint).  status: [4] = final relative FP64
 * residual, refinement (GMRES) iterations, factor seconds, total seconds.
 * RADB200_E_NUMERIC when A + sigma I also meets such a pivot.               */
#define RADB200_LU_F64  0
#define RADB200_LU_TF32 1
RADB200_API int radb200_direct_solve(int64_t handle, int mode, double rtol, int max_iter,
                         double *M_out, double *status);

/* The diagonal shift sigma of the interaction's current factorization: 0 when
 * the factors are of A itself.                                               */
RADB200_API int radb200_lu_shift(int64_t handle, double *sigma);

/* ---- adjoint --- no counterpart in the reference.
 * Given the converged magnetization of the last solve and dL/dM [3N] (each
 * element's frame), solves the transposed system (I - D N)^T lambda = dL/dM
 * with D = dM/dH at the converged state (radmater.cpp:206-277) and returns
 * lambda [3N], by FP64 GMRES on the transposed operator preconditioned with
 * A^T = U^T L^T: the kept factors of the direct solve (linear materials), or
 * otherwise a factorization of A = I - D N (on the tensor cores above 3,072
 * unknowns), kept until the next solve.  status: [4] = final relative
 * residual, GMRES iterations, 1 if LU-preconditioned (0: block-Jacobi split
 * after a factorization breakdown), seconds.                                */
RADB200_API int radb200_adjoint_solve(int64_t handle, const double *dLdM, double rtol,
                          int max_iter, double *lambda_out, double *status);

/* Sensitivities of a scalar loss through the converged solve, given lambda
 * from radb200_adjoint_solve.  Every output is per element, may be NULL:
 *   dL_dMr  [3N]  w.r.t. the remanence Mr of each element's material (element
 *                 frame) with the susceptibility tensor held fixed: lambda;
 *   dL_dchi [9N]  w.r.t. the 3x3 susceptibility tensor of linear elements,
 *                 lambda_e H_e^T (H at the converged state); chaining it
 *                 through chi(Mr) = chi_perp I + (chi_par - chi_perp) L L^T,
 *                 L = Mr/|Mr| (radmater.h:292-303) gives the easy-axis term;
 *   dL_dc   [3N]  w.r.t. the centre of each RECTANGULAR element (object
 *                 frame of the element), from lambda^T D (dN/dc) M + the
 *                 gradient of H_ext at the centres; zero for polyhedra;
 *   dL_dd   [3N]  w.r.t. the dimensions (full widths) of each rectangular
 *                 element, from lambda^T D (dN/dd) M; zero for polyhedra.
 * dN/dc and dN/dd are the analytic derivatives of the cuboid tensor,
 * recomputed pair by pair (images included), never stored.  Terms of the
 * loss that depend on the parameters directly (a field loss at fixed points)
 * come from radb200_field_vjp and are added by the caller.                   */
RADB200_API int radb200_adjoint_grad(int64_t handle, const double *lambda, double *dL_dMr, double *dL_dchi,
                                     double *dL_dc, double *dL_dd);

/* Field-operator part of the adjoint.  F = B (what 0) or H (what 1) at pts
 * [npts*3] from the relaxable elements of this interaction magnetized by M
 * [3N] (element frames).  Given W = dL/dF [npts*3], returns (any may be NULL)
 *   g_M [3N]  = (dF/dM)^T W;
 *   g_c [3N]  = d(W.F)/d(centre) of each rectangular element, M fixed;
 *   g_d [3N]  = d(W.F)/d(dimensions) of each rectangular element, M fixed.  */
RADB200_API int radb200_field_vjp(int64_t handle, const double *M, const double *pts, int64_t npts, int what,
                                  const double *W, double *g_M, double *g_c, double *g_d);

#ifdef __cplusplus
}
#endif
#endif /* RADB200_H */
