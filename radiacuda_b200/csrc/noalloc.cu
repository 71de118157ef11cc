// noalloc.cu -- field evaluation that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured elsewhere in the process, real-time loops that must not hit
// the allocator's locks or its fragmentation, and hosts that hand this
// library fixed device arenas (a simulation framework's memory pool, an
// embedded controller with all memory reserved at start-up).  For them,
// radb200_field_noalloc evaluates B / H / M like radb200_field_dev but takes
// EVERY array in device memory -- the geometry arrays of RadB200Geom included
// -- and keeps its only scratch (per-chunk partial sums) in the file-scope
// array below.
//
// The scratch holds RADB200_NOALLOC_MAX_CHUNKS x RADB200_NOALLOC_MAX_POINTS x 3
// doubles (3 MiB) on every GPU this entry point runs on, until the process
// exits.  With lazy module loading (the CUDA default since 12.2) the driver
// maps it on the first call on each device, when this file looks up its
// address: that first call can fail for lack of device memory, so make it at
// set-up, outside any stream capture.  Every call shares the scratch and it
// keeps the last call's contents; each call overwrites the slices it reads.
// Calls that overlap on the GPU (two host threads, or two streams) race on
// it: serialize them.  The work runs on the calling thread's per-thread
// default stream, which does not synchronize with other blocking streams
// (a capture running on one of them elsewhere in the process is not
// disturbed), and the call waits for it before returning.
#include "internal.cuh"

#define RADB200_NOALLOC_MAX_POINTS 16384
#define RADB200_NOALLOC_MAX_CHUNKS 8

namespace rb {

static __device__ __align__(256) double g_noalloc_scratch[RADB200_NOALLOC_MAX_CHUNKS * RADB200_NOALLOC_MAX_POINTS * 3];

// device address of g_noalloc_scratch per device ordinal (host-side symbols are
// stand-ins, not device addresses); filled by the first call on each device,
// and looked up again if the cached address no longer belongs to this device
// (a caller that reset the device with cudaDeviceReset)
static double *g_noalloc_addr[64];

// Field of source s of the concatenated list [cuboids, polyhedra, arcs,
// backgrounds] at P, all images; the face-by-face polyhedron form in FP64.
__device__ V3<double> noalloc_source(const RadB200Geom &G, const Guard &gd, int s, V3<double> P, int what)
{
  int kind, idx, t0, nt;
  if (s < G.n_rec) { kind = 0; idx = s; t0 = G.rec_img[2 * idx]; nt = G.rec_img[2 * idx + 1]; }
  else if ((s -= G.n_rec) < G.n_poly) { kind = 1; idx = s; t0 = G.poly_info[4 * idx + 2]; nt = G.poly_info[4 * idx + 3]; }
  else if ((s -= G.n_poly) < G.n_arc) { kind = 2; idx = s; t0 = G.arc_img[2 * idx]; nt = G.arc_img[2 * idx + 1]; }
  else { s -= G.n_arc; kind = 3; idx = s; t0 = G.bkg_img[2 * idx]; nt = G.bkg_img[2 * idx + 1]; }
  V3<double> acc = mk3<double>(0, 0, 0);
  for (int t = t0; t < t0 + nt; t++) {
    const double *Tr = G.trf + (size_t)t * RADB200_TRF_STRIDE;
    double dx = P.x - Tr[9], dy = P.y - Tr[10], dz = P.z - Tr[11];
    V3<double> q = mk3<double>(Tr[0] * dx + Tr[1] * dy + Tr[2] * dz, Tr[3] * dx + Tr[4] * dy + Tr[5] * dz,
                               Tr[6] * dx + Tr[7] * dy + Tr[8] * dz);
    V3<double> f = mk3<double>(0, 0, 0);
    if (kind == 0) {
      const double *r = G.rec + (size_t)idx * RADB200_REC_STRIDE;
      V3<double> qc = mk3<double>(q.x - r[0], q.y - r[1], q.z - r[2]);
      V3<double> hd = mk3<double>(0.5 * r[3], 0.5 * r[4], 0.5 * r[5]);
      if (r[9] != 0.0 || r[10] != 0.0 || r[11] != 0.0) {
        if (what != 2) f = cuboid_J(qc, hd, mk3<double>(r[9], r[10], r[11]), gd);
      } else if (what == 2) {
        if (fabs(qc.x) < hd.x && fabs(qc.y) < hd.y && fabs(qc.z) < hd.z) f = mk3<double>(r[6], r[7], r[8]);
      } else {
        V3<double> Tt, Ss;
        int in = cuboid_TS<double>(qc, hd, gd, Tt, Ss);
        f = mk3<double>(Tt.x * r[6] - Ss.z * r[7] - Ss.y * r[8], -Ss.z * r[6] + Tt.y * r[7] - Ss.x * r[8],
                        -Ss.y * r[6] - Ss.x * r[7] + Tt.z * r[8]);
        if (what == 0 && in) { f.x += r[6]; f.y += r[7]; f.z += r[8]; }
      }
    } else if (kind == 1) {
      const double *pr = G.poly + (size_t)idx * RADB200_POLY_STRIDE;
      // the reference's polygon face form uses this 15-digit pi (radplnr2.cpp:32)
      const double C = 1.0 / (4.0 * 3.14159265358979);
      int f0 = G.poly_info[4 * idx], nf = G.poly_info[4 * idx + 1], inside = 1;
      double hx = 0, hy = 0, hz = 0;
      for (int fi = f0; fi < f0 + nf; fi++) {
        const double *R = G.face + (size_t)fi * RADB200_FACE_STRIDE;
        int v0 = G.face_vtx[2 * fi], nv = G.face_vtx[2 * fi + 1];
        const double *vt = G.vtx2d + 2 * (size_t)v0;
        double cx = 0, cy = 0;
        if (gd.absr != 0.0 || gd.relr != 0.0 || gd.zeror != 0.0) {
          for (int k = 0; k < nv; k++) { cx += vt[2 * k]; cy += vt[2 * k + 1]; }
          cx /= nv; cy /= nv;
        }
        V3<double> pl = mk3<double>(R[0] * q.x + R[1] * q.y + R[2] * q.z, R[3] * q.x + R[4] * q.y + R[5] * q.z,
                                    R[6] * q.x + R[7] * q.y + R[8] * q.z);
        double s0, s1, s2;
        if (!polygon_S<double, double>(vt, nv, R[9], cx, cy, pl, gd, s0, s1, s2)) inside = 0;
        double w = -C * (R[6] * pr[3] + R[7] * pr[4] + R[8] * pr[5]);
        hx += w * (R[0] * s0 + R[3] * s1 + R[6] * s2);
        hy += w * (R[1] * s0 + R[4] * s1 + R[7] * s2);
        hz += w * (R[2] * s0 + R[5] * s1 + R[8] * s2);
      }
      if (what == 2) f = inside ? mk3<double>(pr[3], pr[4], pr[5]) : mk3<double>(0, 0, 0);
      else {
        f = mk3<double>(hx, hy, hz);
        if (what == 0 && inside) { f.x += pr[3]; f.y += pr[4]; f.z += pr[5]; }
      }
    } else if (kind == 2) {
      if (what != 2) f = arc_field(G.arc + (size_t)idx * RADB200_ARC_STRIDE, q);
    } else if (what != 2) {
      f = mk3<double>(G.bkg[3 * idx], G.bkg[3 * idx + 1], G.bkg[3 * idx + 2]);
    }
    const double *F = Tr + 12;
    acc.x += F[0] * f.x + F[1] * f.y + F[2] * f.z;
    acc.y += F[3] * f.x + F[4] * f.y + F[5] * f.z;
    acc.z += F[6] * f.x + F[7] * f.y + F[8] * f.z;
  }
  return acc;
}

// chunk c = blockIdx.y sums sources [c*chunk, (c+1)*chunk) into scratch slice c
__global__ void __launch_bounds__(128) noalloc_field_kernel(RadB200Geom G, Guard gd, const double *__restrict__ pts,
                                                            int npts, int what, int nsrc, int chunk, double *scratch)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  int s0 = blockIdx.y * chunk, s1 = min(nsrc, s0 + chunk);
  V3<double> P = mk3<double>(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
  double ax = 0, ay = 0, az = 0;
  for (int s = s0; s < s1; s++) {
    V3<double> f = noalloc_source(G, gd, s, P, what);
    ax += f.x; ay += f.y; az += f.z;
  }
  double *o = scratch + ((size_t)blockIdx.y * npts + i) * 3;
  o[0] = ax; o[1] = ay; o[2] = az;
}

// out[i] = sum over chunks in a fixed order
__global__ void noalloc_reduce_kernel(const double *scratch, int nchunk, int n3, double *__restrict__ out)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; c++) s += scratch[(size_t)c * n3 + i];
  out[i] = s;
}

}  // namespace rb

using namespace rb;

extern "C" RADB200_API int radb200_field_noalloc(const RadB200Geom *g, const double *d_pts, int64_t npts, int what,
                                                 double *d_out)
{
  if (!g || npts < 0 || what < 0 || what > 2 || (npts > 0 && (!d_pts || !d_out))) {
    set_error("radb200_field_noalloc: bad arguments");
    return RADB200_E_ARG;
  }
  if (npts > RADB200_NOALLOC_MAX_POINTS) {
    set_error("radb200_field_noalloc: %lld points exceed the static scratch limit of %d points per call "
              "(split the call, or use radb200_field_dev)", (long long)npts, RADB200_NOALLOC_MAX_POINTS);
    return RADB200_E_ARG;
  }
  if (npts == 0) return 0;
  int dev = 0;
  RB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { set_error("radb200_field_noalloc: device ordinal out of range"); return RADB200_E_ARG; }
  if (g_noalloc_addr[dev]) {
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, g_noalloc_addr[dev]) != cudaSuccess || pa.type != cudaMemoryTypeDevice ||
        pa.device != dev) {
      cudaGetLastError();
      g_noalloc_addr[dev] = nullptr;
    }
  }
  if (!g_noalloc_addr[dev]) {
    // set-up, once per device, with that device current: the device address of the scratch
    void *p = nullptr;
    RB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = (double *)p;
  }
  const cudaStream_t st = cudaStreamPerThread;
  double *scratch = g_noalloc_addr[dev];
  int nsrc = g->n_rec + g->n_poly + g->n_arc + g->n_bkg;
  int n3 = (int)npts * 3;
  if (nsrc == 0) {
    RB_CUDA(cudaMemsetAsync(d_out, 0, (size_t)n3 * sizeof(double), st));
    RB_CUDA(cudaStreamSynchronize(st));
    return 0;
  }
  // as many source chunks as fit the scratch, up to ~8 CTAs per SM in total
  int nblk = (int)((npts + 127) / 128);
  int nchunk = std::max(1, std::min(RADB200_NOALLOC_MAX_CHUNKS, (148 * 8 + nblk - 1) / nblk));
  nchunk = std::min(nchunk, nsrc);
  int chunk = (nsrc + nchunk - 1) / nchunk;
  nchunk = (nsrc + chunk - 1) / chunk;
  Guard gd{g->abs_rand, g->rel_rand, g->zero_rand};
  noalloc_field_kernel<<<dim3(nblk, nchunk), 128, 0, st>>>(*g, gd, d_pts, (int)npts, what, nsrc, chunk, scratch);
  RB_TRY(check_launch("noalloc_field_kernel"));
  noalloc_reduce_kernel<<<(n3 + 255) / 256, 256, 0, st>>>(scratch, nchunk, n3, d_out);
  RB_TRY(check_launch("noalloc_reduce_kernel"));
  RB_CUDA(cudaStreamSynchronize(st));
  return 0;
}
