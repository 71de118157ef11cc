// gemm_tc.cu -- TF32 tensor-core (tcgen05, TMEM accumulator) GEMM updates of
// the blocked LU:   C[m x n] -= A[m x k] * B[k x n]   (or C = A B),
// all FP32 row-major inside the LU matrix (leading dimension ld), any k.
//
// Persistent CTAs of 8 warps loop over 128 x 256 tiles of C (one CTA per SM,
// 192 KB of staged operands):
//   0. A is rounded to TF32 (round to nearest) in place and B is transposed
//      to K-major with the same rounding, once per call, so the tensor core
//      reads exact TF32 values (in the LU, A is always an L panel or an
//      inverse, which the factorization keeps at TF32 accuracy anyway);
//   1. K runs in chunks of 64 through two shared-memory stages: cp.async
//      brings chunk g+1 of A (128 x 64) and B^T (256 x 64) into one stage,
//      in the canonical no-swizzle UMMA layout (8-row x 16-byte core
//      matrices), while the tensor core works on chunk g in the other;
//   2. one elected thread issues 8 tcgen05.mma.kind::tf32 (M=128, N=256,
//      K=8) per chunk into 256 TMEM columns and commits them to an mbarrier;
//      at a tile's first chunk every thread loads the 128 C values of its row
//      segment, which stay in registers through the K loop;
//   3. after the last chunk each thread reads its accumulators with
//      tcgen05.ld and stores C - AB, while the next tile's first chunk lands.
// Waits on the mbarrier are bounded: on timeout the CTA raises an error flag,
// waits for its own copies, frees its TMEM and returns (the host then falls
// back to the CUDA-core GEMM and reports the error).
//
// Layouts (byte offsets inside one stage's A / B^T buffers, chunk-local k):
//   (row/8)*2048 + (k/4)*128 + (row%8)*16 + (k%4)*4, both operands K-major
//   descriptor of MMA step s: start + 256 s, LBO 128 (next k group),
//   SBO 2048 (next 8 rows).  B arrives row-major k x n and is transposed to
//   n x k in global memory first (k*n*8 bytes, small against the m*n*8 of C;
//   the MMA reads tf32 operands K-major only).
// The first use runs a self-test against the CUDA-core GEMM (ragged m, n, k,
// several tiles and chunks per CTA) and keeps the tensor-core path only if it
// agrees to TF32 accuracy.
#include <cuda.h>
#include <cuda_fp16.h>
#include <math.h>
#include <stdlib.h>

#include <vector>

#include "internal.cuh"

namespace rb {

constexpr int TC_BM = 128, TC_BN = 256;
constexpr int TC_KC = 64;                       // K chunk per pipeline stage
constexpr int TC_THREADS = 256;
constexpr int TC_STAGE_A = TC_BM * TC_KC * 4;   // 32 KB
constexpr int TC_STAGE_B = TC_BN * TC_KC * 4;   // 64 KB
constexpr int TC_STAGE = TC_STAGE_A + TC_STAGE_B;
constexpr int TC_SMEM = 2 * TC_STAGE + 1024;      // two stages + alignment slack
constexpr long long TC_SPIN_LIMIT = 1ll << 22;  // ~0.3 s of polling; the MMAs of a tile take microseconds

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ float to_tf32(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  // base offset 0, lbo mode 0, layout type 0 (no swizzle)
  return d;
}

// instruction descriptor: F32 accumulate, TF32 A/B, A K-major, B N- or K-major, M=128, N=256
__host__ __device__ constexpr uint32_t umma_idesc(int b_mn_major)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | (0u << 15) | ((uint32_t)b_mn_major << 16) | ((uint32_t)(TC_BN >> 3) << 17) |
         ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

// 16-byte cp.async of this thread's share of K chunk [k0, k0 + 64) of A
// (rows row0..) and B^T (rows col0..) into one stage, in the K-major
// core-matrix layout: offset (row / 8) * 2048 + (k / 4) * 128 + (row % 8) * 16.
// Lanes -> (row % 8, 4 consecutive k-groups): global reads are 64-byte runs,
// shared writes bank-conflict free.  Zero-filled past m, n and k.
__device__ __forceinline__ void tc_issue_chunk(uint32_t sa, uint32_t sb, const float *__restrict__ A, int lda,
                                               const float *__restrict__ Bt, int ldbt, int m, int n, int k, int k0,
                                               int row0, int col0, int tid)
{
  constexpr int NA = (TC_BM / 8) * (TC_KC / 4) * 8, NB = (TC_BN / 8) * (TC_KC / 4) * 8;
#pragma unroll 4
  for (int it = tid; it < NA; it += TC_THREADS) {
    int rr = it & 7, rest = it >> 3;
    int kc = rest & (TC_KC / 4 - 1), rg = rest / (TC_KC / 4);
    int gr = row0 + rg * 8 + rr, kk = k0 + kc * 4;
    uint32_t bytes = (gr < m && kk < k) ? (uint32_t)(min(4, k - kk) * 4) : 0u;
    const float *src = bytes ? A + (size_t)gr * lda + kk : A;
    cp_async16(sa + rg * 2048 + kc * 128 + rr * 16, src, bytes);
  }
#pragma unroll 4
  for (int it = tid; it < NB; it += TC_THREADS) {
    int nr = it & 7, rest = it >> 3;
    int kc = rest & (TC_KC / 4 - 1), ngp = rest / (TC_KC / 4);
    int gc = col0 + ngp * 8 + nr, kk = k0 + kc * 4;
    uint32_t bytes = (gc < n && kk < k) ? (uint32_t)(min(4, k - kk) * 4) : 0u;
    const float *src = bytes ? Bt + (size_t)gc * ldbt + kk : Bt;
    cp_async16(sb + ngp * 2048 + kc * 128 + nr * 16, src, bytes);
  }
}

// overwrite == 0: C -= A B;  overwrite == 1: C = A B.  C must not alias A or B.
// Tile order of the persistent grid: bands of TC_TILE_GROUP n-tiles, and
// inside a band the n-tiles fastest, then the rows.  The CTAs running at any
// moment then cover about (grid / 16) row blocks of one 16-tile band, so the
// band's B^T slice (16 x 256 x K) stays in L2 for the whole band and the A
// panel is streamed once per band, instead of the whole B^T panel once per
// row of tiles when a row is wider than L2 holds (60,000 columns: 120 MB).
constexpr int TC_TILE_GROUP = 16;
__device__ __forceinline__ void tile_rc(int t, int tiles_m, int tiles_n, int &row0, int &col0)
{
  const int band = t / (TC_TILE_GROUP * tiles_m);
  const int n0 = band * TC_TILE_GROUP;
  const int gw = min(TC_TILE_GROUP, tiles_n - n0);
  const int r = t - band * TC_TILE_GROUP * tiles_m;
  row0 = (r / gw) * TC_BM;
  col0 = (n0 + r % gw) * TC_BN;
}

// Bt = B^T (n x ldbt, K contiguous).  Persistent: CTA b handles tiles b,
// b + gridDim.x, ... in the banded order of tile_rc.
// Every tile runs ceil(k / 64) chunks through a two-stage pipeline: chunk g+1
// is copied into the other stage while the MMAs of chunk g run; the tile's C
// values are loaded into registers at its first chunk and consumed at its
// last, so their latency hides behind the whole K loop.
__global__ void __launch_bounds__(TC_THREADS, 1) tc_update_kernel(float *__restrict__ C, int ldc, int m, int n, int k,
                                                                  const float *__restrict__ A, int lda,
                                                                  const float *__restrict__ Bt, int ldbt,
                                                                  int *__restrict__ err, int overwrite)
{
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *sbase = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int timed_out;
  __shared__ int abort_cta;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_n = (n + TC_BN - 1) / TC_BN, tiles_m = (m + TC_BM - 1) / TC_BM;
  const int ntiles = tiles_n * tiles_m;
  const int nch = (k + TC_KC - 1) / TC_KC;
  // once any CTA of this launch (or an earlier one) has timed out, the rest
  // return at once (decided by one thread so the whole CTA leaves together)
  if (tid == 0) abort_cta = *(volatile int *)err;
  __syncthreads();
  if (abort_cta != 0 || (int)blockIdx.x >= ntiles || nch < 1) return;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)), "r"(TC_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    timed_out = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  const uint32_t s0 = smem_u32(sbase);
  // my tiles: blockIdx.x + i * gridDim.x; global chunk g = i * nch + c
  const int my_tiles = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int G = my_tiles * nch;
  uint32_t phase = 0;
  const int q = warp & 3, hc = warp >> 2;
  const int r = q * 32 + lane;
  float4 cv[32];

  {  // chunk 0 into stage 0
    const int t0 = blockIdx.x;
    int r0, c0;
    tile_rc(t0, tiles_m, tiles_n, r0, c0);
    tc_issue_chunk(s0, s0 + TC_STAGE_A, A, lda, Bt, ldbt, m, n, k, 0, r0, c0, tid);
  }
  for (int g = 0; g < G; g++) {
    const int i = g / nch, c = g - i * nch;
    const int tile = blockIdx.x + i * gridDim.x;
    int row0, col0;
    tile_rc(tile, tiles_m, tiles_n, row0, col0);
    const int st = g & 1;
    unsigned char *sa = sbase + st * TC_STAGE, *sb = sa + TC_STAGE_A;
    // ---- this chunk's operands (already TF32 values): wait for the copies
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // ---- MMAs of the chunk (one thread): 8 steps of K = 8
    if (tid == 0) {
      const uint32_t idesc = umma_idesc(0);
      const uint32_t ua = smem_u32(sa), ub = smem_u32(sb);
#pragma unroll
      for (int s = 0; s < TC_KC / 8; s++) {
        uint64_t da = umma_desc(ua + 256u * s, 128u, 2048u);
        uint64_t db = umma_desc(ub + 256u * s, 128u, 2048u);
        uint32_t acc = (c > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&mbar))
                   : "memory");
    }
    // ---- next chunk into the other stage (its last reader, chunk g-1, is complete)
    if (g + 1 < G) {
      const int i1 = (g + 1) / nch, c1 = (g + 1) - i1 * nch;
      const int t1 = blockIdx.x + i1 * gridDim.x;
      const uint32_t so = s0 + (st ^ 1) * TC_STAGE;
      int r1, c1b;
      tile_rc(t1, tiles_m, tiles_n, r1, c1b);
      tc_issue_chunk(so, so + TC_STAGE_A, A, lda, Bt, ldbt, m, n, k, c1 * TC_KC, r1, c1b, tid);
    }
    // ---- first chunk of a tile: this thread's C values (row r, 128 columns)
    if (c == 0) {
      const int gr = row0 + r, gcb = col0 + hc * 128;
#pragma unroll
      for (int j = 0; j < 32; j++) {
        int gc = gcb + 4 * j;
        cv[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!overwrite && gr < m) {
          const float *src = C + (size_t)gr * ldc + gc;
          if (gc + 3 < n) cv[j] = *reinterpret_cast<const float4 *>(src);
          else if (gc < n) {
            cv[j].x = src[0];
            if (gc + 1 < n) cv[j].y = src[1];
            if (gc + 2 < n) cv[j].z = src[2];
          }
        }
      }
    }
    // ---- bounded wait for the chunk's MMAs
    {
      uint32_t done = 0;
      long long spins = 0;
      while (!done) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(&mbar)), "r"(phase)
            : "memory");
        if (!done && ++spins > TC_SPIN_LIMIT) {
          timed_out = 1;
          break;
        }
      }
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (timed_out) break;
    if (c != nch - 1) continue;

    // ---- last chunk: epilogue, TMEM -> registers -> C (warp w: TMEM lanes 32 (w % 4), columns 128 (w / 4))
    const int gr = row0 + r, gcb = col0 + hc * 128;
#pragma unroll
    for (int cb = 0; cb < 128; cb += 16) {
      uint32_t v[16];
      uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(hc * 128 + cb);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
            "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (gr < m) {
#pragma unroll
        for (int j4 = 0; j4 < 4; j4++) {
          const int j = cb / 4 + j4;
          const int gc = gcb + 4 * j;
          float4 t = make_float4(__uint_as_float(v[4 * j4]), __uint_as_float(v[4 * j4 + 1]), __uint_as_float(v[4 * j4 + 2]),
                                 __uint_as_float(v[4 * j4 + 3]));
          float4 o = overwrite ? t : make_float4(cv[j].x - t.x, cv[j].y - t.y, cv[j].z - t.z, cv[j].w - t.w);
          float *dst = C + (size_t)gr * ldc + gc;
          if (gc + 3 < n) *reinterpret_cast<float4 *>(dst) = o;
          else if (gc < n) {
            dst[0] = o.x;
            if (gc + 1 < n) dst[1] = o.y;
            if (gc + 2 < n) dst[2] = o.z;
          }
        }
      }
    }
    // TMEM reads done before the next tile's first MMAs overwrite the accumulators
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  // no copies may still be landing in shared memory when the CTA exits
  asm volatile("cp.async.wait_all;" ::: "memory");
  if (timed_out && tid == 0) atomicExch(err, 2);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN));
}

// ---- TMA variant ---------------------------------------------------------------
// Same tiles and epilogue, but the operands come in by TMA: per K chunk of 32
// one 2-D bulk tensor load of A (32 x 128) and one of B^T (32 x 256), written
// by the copy engine in the 128-byte-swizzled K-major layout (8-row x 128-byte
// atoms, 1024-byte aligned) and completed on the stage's "full" mbarrier with
// a transaction count.  One lane of a producer warp issues the loads and the
// MMAs through TM_NST stages (loads run TM_NST - 1 chunks ahead; a stage is
// refilled once the MMAs that read it have committed to its "empty"
// mbarrier) into two alternating TMEM accumulators; 8 epilogue warps load C
// and write the results.  Descriptors: start address of the atom + 32 bytes
// per K=8 step, SBO 1024, layout 128B swizzle.
constexpr int TM_KC = 32;
constexpr int TM_NST = 4;
constexpr int TM_STAGE_A = TC_BM * TM_KC * 4;   // 16 KB
constexpr int TM_STAGE_B = TC_BN * TM_KC * 4;   // 32 KB
constexpr int TM_STAGE = TM_STAGE_A + TM_STAGE_B;
constexpr int TM_SMEM_W = 8 * 32 * 32 * 4;  // one 32 x 32 transpose buffer per epilogue warp (XOR-swizzled columns)
constexpr int TM_SMEM = TM_NST * TM_STAGE + 1024 + TM_SMEM_W;

__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;             // leading byte offset: not used by swizzled K-major operands
  d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset: 8 rows x 128 bytes
  d |= (uint64_t)1 << 46;             // descriptor version for sm_100
  d |= (uint64_t)2 << 61;             // layout: 128-byte swizzle
  return d;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ int tm_wait(uint32_t bar, uint32_t parity)
{
  uint32_t done = 0;
  long long spins = 0;
  while (!done) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (!done && ++spins > TC_SPIN_LIMIT) return 0;
  }
  return 1;
}

constexpr int TM_THREADS = 288;  // warps 0-7: epilogue; warp 8: TMA loads and MMAs


// Warp-specialised: warp 8 (one lane) streams the chunks of all of the CTA's
// tiles through the operand stages into two TMEM accumulators (columns
// 0-255 and 256-511, alternating per tile) and commits each finished tile to
// that buffer's "full" barrier; warps 0-7 drain a finished buffer (C loaded
// beforehand, C - AB stored) and arrive on its "empty" barrier, so the MMAs
// of tile i+1 run while tile i is written back.  Every wait is bounded.
// F16: the operands are FP16 copies scaled by powers of two (*scale holds
// 1 / (sA sB), applied to the accumulator in the epilogue): kind::f16 MMAs of
// K = 16 (32 bytes of a 128-byte row, as the TF32 K = 8 step), 64 elements
// per stage row instead of 32, so a stage feeds twice the flops.
template <bool F16>
__global__ void __launch_bounds__(TM_THREADS, 1) tc_update_tma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                                      const __grid_constant__ CUtensorMap tmB,
                                                                      float *__restrict__ C, int ldc, int m, int n, int k,
                                                                      int *__restrict__ err, int overwrite,
                                                                      const float *__restrict__ row_scale,
                                                                      const float *__restrict__ col_scale)
{
  constexpr int KC = F16 ? 2 * TM_KC : TM_KC;  // K elements per stage
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *sbase = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ uint64_t full[TM_NST], empty[TM_NST], accf[2], acce[2];
  __shared__ uint32_t tmem_base_s;
  __shared__ int timed_out;
  __shared__ int abort_cta;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_n = (n + TC_BN - 1) / TC_BN, tiles_m = (m + TC_BM - 1) / TC_BM;
  const int ntiles = tiles_n * tiles_m;
  const int nch = (k + KC - 1) / KC;
  if (tid == 0) abort_cta = *(volatile int *)err;
  __syncthreads();
  if (abort_cta != 0 || (int)blockIdx.x >= ntiles || nch < 1) return;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(2 * TC_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int b = 0; b < TM_NST; b++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[b])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[b])));
    }
    for (int b = 0; b < 2; b++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accf[b])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 256;" ::"r"(smem_u32(&acce[b])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    timed_out = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  const uint32_t s0 = smem_u32(sbase);
  const int my_tiles = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;

  if (warp == 8) {
    // ---------------- producer: TMA loads and MMAs (lane 0) ----------------
    int issued = 0, consumed = 0;
    if (lane == 0) {
      const int G = my_tiles * nch;
      auto issue = [&](int gg) {
        const int ii = gg / nch, cc = gg - ii * nch;
        const int tt = blockIdx.x + ii * gridDim.x;
        const uint32_t so = s0 + (gg % TM_NST) * TM_STAGE, fb = smem_u32(&full[gg % TM_NST]);
        mbar_expect_tx(fb, (uint32_t)TM_STAGE);
        int rr, ccol;
        tile_rc(tt, tiles_m, tiles_n, rr, ccol);
        tma_load_2d(so, &tmA, cc * KC, rr, fb);
        tma_load_2d(so + TM_STAGE_A, &tmB, cc * KC, ccol, fb);
      };
      for (; issued < TM_NST - 1 && issued < G; issued++) issue(issued);
      // F16: A and B formats 0 (f16); TF32: 2 (tf32)
      const uint32_t idesc = F16 ? (umma_idesc(0) & ~((7u << 7) | (7u << 10))) : umma_idesc(0);
      for (int i = 0; i < my_tiles && !timed_out; i++) {
        const int buf = i & 1;
        // the epilogue of tile i - 2 has released this accumulator buffer
        if (i >= 2 && !tm_wait(smem_u32(&acce[buf]), (uint32_t)(((i - 2) / 2) & 1))) { timed_out = 1; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t dacc = tmem + (uint32_t)(buf * TC_BN);
        for (int c = 0; c < nch; c++) {
          const int g = i * nch + c, st = g % TM_NST;
          if (!tm_wait(smem_u32(&full[st]), (uint32_t)((g / TM_NST) & 1))) { timed_out = 1; break; }
          consumed++;
          const uint32_t ua = s0 + st * TM_STAGE, ub = ua + TM_STAGE_A;
#pragma unroll
          for (int s = 0; s < TM_KC / 8; s++) {
            uint64_t da = umma_desc_sw128(ua + 32u * s);
            uint64_t db = umma_desc_sw128(ub + 32u * s);
            uint32_t acc = (c > 0 || s > 0) ? 1u : 0u;
            if (F16)
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dacc),
                  "l"(da), "l"(db), "r"(idesc), "r"(acc));
            else
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dacc),
                  "l"(da), "l"(db), "r"(idesc), "r"(acc));
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_u32(&empty[st]))
                       : "memory");
          if (issued < G) {
            const int old = issued - TM_NST;  // the chunk whose stage is refilled
            if (old >= 0 && !tm_wait(smem_u32(&empty[old % TM_NST]), (uint32_t)((old / TM_NST) & 1))) {
              timed_out = 1;
              break;
            }
            issue(issued++);
          }
        }
        if (timed_out) break;
        // the tile's accumulators are complete once everything issued so far is
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&accf[buf]))
                     : "memory");
      }
      // after a timeout: wait (bounded) for bulk copies still in flight
      for (int j = consumed; j < issued; j++) tm_wait(smem_u32(&full[j % TM_NST]), (uint32_t)((j / TM_NST) & 1));
    }
    __syncwarp();
  } else {
    // ---------------- epilogue: warps 0-7 ----------------
    // Warp (q, hc) owns rows q*32.. of the tile (its TMEM lane quarter) and
    // the column half hc*128.., in four 32-column slices.  C is read and
    // written row-contiguous: lane l takes 4 columns, (l % 8) * 4.., of row
    // (l / 8) of every group of 4 rows, so a warp instruction covers four
    // full 128-byte lines.  The accumulator rows arrive lane = row
    // (tcgen05.ld 32x32b) and are turned around through a 32 x 32 shared
    // buffer per warp in 16-byte groups: group g of row r sits at group
    // position g ^ (r % 8), so the row-wise group writes and the column-wise
    // group reads of each 8-lane phase hit all 32 banks once.  The tile's C values are loaded before its
    // accumulator is waited on.
    const int q = warp & 3, hc = warp >> 2;
    float *W = reinterpret_cast<float *>(sbase + TM_NST * TM_STAGE) + warp * 32 * 32;
    const int lr = lane >> 3, lc = (lane & 7) * 4;
    for (int i = 0; i < my_tiles; i++) {
      const int tile = blockIdx.x + i * gridDim.x;
      int row0, col0;
      tile_rc(tile, tiles_m, tiles_n, row0, col0);
      const int buf = i & 1;
      const int rbase = row0 + q * 32, cbase = col0 + hc * 128;
      // C slice sl (8 float4 per thread) for rows rbase + 4 rr + lr, columns cbase + 32 sl + lc ..:
      // slices 0 and 1 are loaded before the accumulator wait, slice sl + 2
      // while slice sl is written back
      auto load_slice = [&](float4 *cs, int sl) {
#pragma unroll
        for (int rr = 0; rr < 8; rr++) {
          const int gr = rbase + 4 * rr + lr, gc = cbase + 32 * sl + lc;
          cs[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (!overwrite && gr < m) {
            const float *src = C + (size_t)gr * ldc + gc;
            if (gc + 3 < n) cs[rr] = *reinterpret_cast<const float4 *>(src);
            else if (gc < n) {
              cs[rr].x = src[0];
              if (gc + 1 < n) cs[rr].y = src[1];
              if (gc + 2 < n) cs[rr].z = src[2];
            }
          }
        }
      };
      auto store_slice = [&](const float4 *cs, int sl) {
        // FP16 operands: the accumulator carries the row and column factors
        // (read only for columns inside C: the factors hold n + 8 entries)
        const int gcs = cbase + 32 * sl + lc;
        const float4 csc = (F16 && gcs < n) ? __ldg(reinterpret_cast<const float4 *>(col_scale + gcs))
                                            : make_float4(1.f, 1.f, 1.f, 1.f);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          uint32_t v[16];
          const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * TC_BN + hc * 128 + sl * 32 + h * 16);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
                "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
              : "r"(taddr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int c4 = 0; c4 < 4; c4++)
            *reinterpret_cast<float4 *>(W + lane * 32 + (((h * 4 + c4) ^ (lane & 7)) << 2)) =
                make_float4(__uint_as_float(v[4 * c4]), __uint_as_float(v[4 * c4 + 1]), __uint_as_float(v[4 * c4 + 2]),
                            __uint_as_float(v[4 * c4 + 3]));
        }
        __syncwarp();
#pragma unroll
        for (int rr = 0; rr < 8; rr++) {
          const int rl = 4 * rr + lr;
          float4 t = *reinterpret_cast<const float4 *>(W + rl * 32 + (((lane & 7) ^ (rl & 7)) << 2));
          const int gr = rbase + rl, gc = cbase + 32 * sl + lc;
          if (gr < m) {
            if (F16) {
              const float rsc = __ldg(row_scale + gr);
              t.x *= rsc * csc.x;
              t.y *= rsc * csc.y;
              t.z *= rsc * csc.z;
              t.w *= rsc * csc.w;
            }
            const float4 c4 = cs[rr];
            const float4 o = overwrite ? t : make_float4(c4.x - t.x, c4.y - t.y, c4.z - t.z, c4.w - t.w);
            float *dst = C + (size_t)gr * ldc + gc;
            if (gc + 3 < n) *reinterpret_cast<float4 *>(dst) = o;
            else if (gc < n) {
              dst[0] = o.x;
              if (gc + 1 < n) dst[1] = o.y;
              if (gc + 2 < n) dst[2] = o.z;
            }
          }
        }
        __syncwarp();  // the next slice overwrites W
      };
      float4 c0[8], c1[8], c2[8], c3[8];
      load_slice(c0, 0);
      load_slice(c1, 1);
      if (!tm_wait(smem_u32(&accf[buf]), (uint32_t)((i / 2) & 1))) { timed_out = 1; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      store_slice(c0, 0);
      load_slice(c2, 2);
      store_slice(c1, 1);
      load_slice(c3, 3);
      store_slice(c2, 2);
      store_slice(c3, 3);
      // this thread's reads of the buffer are done: release it to the producer
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acce[buf])) : "memory");
    }
  }
  if (timed_out && tid == 0) atomicExch(err, 2);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_BN));
}

// CUDA-core reference for the self-test: C -= A B or C = A B (FP32 inputs
// rounded to TF32 like the tensor path)
__global__ void tc_ref_kernel(float *C, int ld, int m, int n, int k, const float *A, const float *B, int overwrite)
{
  int r = blockIdx.y, c = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m || c >= n) return;
  float s = 0.f;
  for (int q = 0; q < k; q++) s = fmaf(to_tf32(A[(size_t)r * ld + q]), to_tf32(B[(size_t)q * ld + c]), s);
  C[(size_t)r * ld + c] = overwrite ? s : C[(size_t)r * ld + c] - s;
}

static int g_tc_state = -1;   // -1 untested, 0 disabled, 1 enabled
static int g_tc_tma = 0;      // 1: the TMA-fed kernel (TF32 operands) passed the self-test; 2: also with FP16 operands
static double g_tc_err = -1.0;
static DBuf g_tc_err_flag;

// A[r][c] <- TF32(A[r][c]) for r < m, c < k, in place
__global__ void tc_round_kernel(float *__restrict__ A, int lda, int m, int k)
{
  int64_t tot = (int64_t)m * k;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(i / k), c = (int)(i - (int64_t)r * k);
    float *p = A + (size_t)r * lda + c;
    *p = to_tf32(*p);
  }
}

// Bt[c][r] = TF32(B[r][c]) for r < k, c < n (32 x 32 tiles through shared memory)
__global__ void tc_transpose_kernel(const float *__restrict__ B, int ldb, int k, int n, float *__restrict__ Bt, int ldbt)
{
  __shared__ float t[32][33];
  int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    int r = r0 + i, c = c0 + threadIdx.x;
    if (r < k && c < n) t[i][threadIdx.x] = B[(size_t)r * ldb + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    int c = c0 + i, r = r0 + threadIdx.x;
    if (r < k && c < n) Bt[(size_t)c * ldbt + r] = to_tf32(t[threadIdx.x][i]);
  }
}

// ---- FP16 operands: power-of-two scaling against the FP16 range -------------
// max |A| (m x k) and max |B| (k x n) into mx[0], mx[1] (float bits; non-
// negative floats order as unsigned integers)
// the power of two that brings max |x| to at most 2^14 (1 for an all-zero operand)
__device__ __forceinline__ float f16_scale(unsigned maxbits)
{
  const float mxv = __uint_as_float(maxbits);
  if (!(mxv > 0.f) || !isfinite(mxv)) return 1.f;
  int e;
  frexpf(mxv, &e);  // mxv < 2^e
  return ldexpf(1.f, 14 - e);
}

// Ah[r][c] = FP16(s_r A[r][c]) for c < k, 0 for k <= c < kp, with s_r the
// power of two that brings row r's largest magnitude to at most 2^14; irs[r] =
// 1 / s_r (exact).  A warp per row: the maximum, then the conversion (the row
// is read again from L1/L2).
__global__ void tc_f16_rows_kernel(const float *__restrict__ A, int lda, int m, int k, __half *__restrict__ Ah, int kp,
                                   float *__restrict__ irs)
{
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < m; r += nw) {
    const float *row = A + (size_t)r * lda;
    float mx = 0.f;
    for (int c = lane; c < k; c += 32) mx = fmaxf(mx, fabsf(row[c]));
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const float sr = f16_scale(__float_as_uint(mx));
    if (lane == 0) irs[r] = 1.f / sr;
    __half2 *dst = reinterpret_cast<__half2 *>(Ah + (size_t)r * kp);
    for (int c2 = lane; c2 < kp / 2; c2 += 32) {
      const int c = 2 * c2;
      dst[c2] = __floats2half2_rn(c < k ? sr * row[c] : 0.f, c + 1 < k ? sr * row[c + 1] : 0.f);
    }
  }
}

// Bth[c][r] = FP16(t_c B[r][c]) (n x kp, K contiguous), with t_c the power of
// two that brings column c's largest magnitude to at most 2^14; ics[c] = 1 / t_c.
// A block of 32 x 8 threads per 32 columns: the column maxima, then the
// columns turned around 32 rows at a time through shared memory.
__global__ void tc_f16_transpose_kernel(const float *__restrict__ B, int ldb, int k, int n, __half *__restrict__ Bth,
                                        int kp, float *__restrict__ ics)
{
  __shared__ float t[32][33];
  __shared__ float red[8][32];
  __shared__ float sc[32];
  const int c0 = blockIdx.x * 32, tx = threadIdx.x, ty = threadIdx.y;
  const int c = c0 + tx;
  float mx = 0.f;
  if (c < n)
    for (int r = ty; r < k; r += 8) mx = fmaxf(mx, fabsf(B[(size_t)r * ldb + c]));
  red[ty][tx] = mx;
  __syncthreads();
  if (ty == 0) {
    for (int i = 1; i < 8; i++) mx = fmaxf(mx, red[i][tx]);
    const float tc = f16_scale(__float_as_uint(mx));
    sc[tx] = tc;
    if (c < n) ics[c] = 1.f / tc;
  }
  __syncthreads();
  for (int r0 = 0; r0 < kp; r0 += 32) {
    for (int i = ty; i < 32; i += 8) {
      const int r = r0 + i;
      t[i][tx] = (r < k && c < n) ? B[(size_t)r * ldb + c] : 0.f;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
      const int cc = c0 + i, r = r0 + tx;
      if (cc < n && r < kp) Bth[(size_t)cc * kp + r] = __float2half_rn(sc[i] * t[tx][i]);
    }
    __syncthreads();
  }
}

// B^T scratch, [n x ldbt] floats, ldbt = k rounded up to 4; one per slot so
// that updates on two streams (the LU's look-ahead) never share it
static DBuf g_tc_bt_slots[2];
// FP16 path, per slot: A and B^T copies, the row and column factors
static DBuf g_tc_ah_slots[2], g_tc_bh_slots[2], g_tc_rs_slots[2], g_tc_cs_slots[2];

// cudaFuncSetAttribute once per kernel and device (a driver call per launch
// showed up in the LU's host enqueue time)
template <typename K>
static int set_smem_once(K kernel, int bytes, int which)
{
  static bool done[3][64] = {};
  int dev = 0;
  RB_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && done[which][dev]) return 0;
  RB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  if (dev >= 0 && dev < 64) done[which][dev] = true;
  return 0;
}


// max_ctas > 0 caps the persistent grid (the self-test uses it to make every
// CTA loop over several tiles)
typedef CUresult (*TensorMapEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                      const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda)
static TensorMapEncodeFn tensor_map_encoder()
{
  static TensorMapEncodeFn fn = nullptr;
  static int tried = 0;
  if (!tried) {
    tried = 1;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (TensorMapEncodeFn)p;
    cudaGetLastError();
  }
  return fn;
}

// 2-D FP32 map of a row-major rows x cols matrix (pitch ld floats), boxes of
// 32 columns x box_rows rows, 128-byte swizzle, zero fill outside
static int encode_map(CUtensorMap *map, const void *base, int rows, int cols, int ld, int box_rows, bool f16 = false)
{
  TensorMapEncodeFn enc = tensor_map_encoder();
  if (!enc) return RADB200_E_UNSUPPORTED;
  // 128-byte rows of the box: 32 FP32 or 64 FP16 elements
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * (f16 ? 2u : 4u)};
  cuuint32_t box[2] = {(cuuint32_t)(f16 ? 2 * TM_KC : TM_KC), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)base, dims,
                   strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("tensor map encoding failed (%d)", (int)r);
    return RADB200_E_UNSUPPORTED;
  }
  return 0;
}

static int launch_tc(float *C, int ldc, int m, int n, int k, float *A, int lda, const float *B, int ldb,
                     cudaStream_t st, int overwrite = 0, int max_ctas = 0, int use_tma = -1, int slot = 0)
{
  DBuf &g_tc_bt = g_tc_bt_slots[slot & 1];
  if (use_tma < 0) use_tma = g_tc_tma;
  long long tiles = (long long)((n + TC_BN - 1) / TC_BN) * ((m + TC_BM - 1) / TC_BM);
  if (tiles > (1ll << 30) || k < 1 || k > (1 << 20)) { set_error("tensor-core update shape out of range"); return RADB200_E_ARG; }
  const int ldbt = (k + 3) / 4 * 4;
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    RB_CUDA(cudaGetDevice(&dev));
    RB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  }
  int grid = (int)std::min<long long>(tiles, max_ctas > 0 ? max_ctas : nsm);
  if (use_tma == 2) {
    // FP16 operands, each row of A and each column of B scaled by a power of
    // two into range (A and B are left as they are)
    const int kp = (k + 7) / 8 * 8;
    DBuf &ah = g_tc_ah_slots[slot & 1], &bh = g_tc_bh_slots[slot & 1];
    DBuf &rs = g_tc_rs_slots[slot & 1], &cs = g_tc_cs_slots[slot & 1];
    RB_TRY(ah.alloc((size_t)m * kp * sizeof(__half)));
    RB_TRY(bh.alloc((size_t)n * kp * sizeof(__half)));
    RB_TRY(rs.alloc((size_t)m * sizeof(float)));
    RB_TRY(cs.alloc((size_t)(n + 8) * sizeof(float)));  // the epilogue reads 4 at a time past a ragged end
    const int nra = (int)std::min<int64_t>(((int64_t)m + 7) / 8, 148 * 16);
    tc_f16_rows_kernel<<<std::max(nra, 1), 256, 0, st>>>(A, lda, m, k, ah.as<__half>(), kp, rs.as<float>());
    RB_TRY(check_launch("tc_f16_rows_kernel"));
    tc_f16_transpose_kernel<<<(n + 31) / 32, dim3(32, 8), 0, st>>>(B, ldb, k, n, bh.as<__half>(), kp, cs.as<float>());
    RB_TRY(check_launch("tc_f16_transpose_kernel"));
    CUtensorMap ma, mb;
    RB_TRY(encode_map(&ma, ah.p, m, k, kp, TC_BM, true));
    RB_TRY(encode_map(&mb, bh.p, n, k, kp, TC_BN, true));
    RB_TRY(set_smem_once(tc_update_tma_kernel<true>, TM_SMEM, 0));
    tc_update_tma_kernel<true><<<grid, TM_THREADS, TM_SMEM, st>>>(ma, mb, C, ldc, m, n, k, g_tc_err_flag.as<int>(),
                                                                  overwrite, rs.as<float>(), cs.as<float>());
    return check_launch("tc_update_tma_kernel<f16>");
  }
  RB_TRY(g_tc_bt.alloc((size_t)n * ldbt * sizeof(float)));
  {
    int64_t tot = (int64_t)m * k;
    int nb = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
    tc_round_kernel<<<std::max(nb, 1), 256, 0, st>>>(A, lda, m, k);
    RB_TRY(check_launch("tc_round_kernel"));
  }
  tc_transpose_kernel<<<dim3((n + 31) / 32, (k + 31) / 32), dim3(32, 8), 0, st>>>(B, ldb, k, n, g_tc_bt.as<float>(), ldbt);
  RB_TRY(check_launch("tc_transpose_kernel"));
  if (use_tma) {
    CUtensorMap ma, mb;
    RB_TRY(encode_map(&ma, A, m, k, lda, TC_BM));
    RB_TRY(encode_map(&mb, g_tc_bt.as<float>(), n, k, ldbt, TC_BN));
    RB_TRY(set_smem_once(tc_update_tma_kernel<false>, TM_SMEM, 1));
    tc_update_tma_kernel<false><<<grid, TM_THREADS, TM_SMEM, st>>>(ma, mb, C, ldc, m, n, k, g_tc_err_flag.as<int>(),
                                                                   overwrite, nullptr, nullptr);
    return check_launch("tc_update_tma_kernel");
  }
  RB_TRY(set_smem_once(tc_update_kernel, TC_SMEM, 2));
  tc_update_kernel<<<grid, TC_THREADS, TC_SMEM, st>>>(C, ldc, m, n, k, A, lda, g_tc_bt.as<float>(), ldbt,
                                                      g_tc_err_flag.as<int>(), overwrite);
  return check_launch("tc_update_kernel");
}

// One self-test case: a random m x n x k update inside an ld-wide buffer
// (A = rows k.. cols 0..k-1, B = rows 0..k-1 cols k.., C = rows k.. cols k..)
// on 2 CTAs, so each CTA loops over several tiles and K chunks; returns the
// relative max deviation from the CUDA-core reference in *err, or sets
// *timeout when an MMA completion wait ran out.
static int tc_selftest_case(int m, int n, int k, int overwrite, int use_tma, double *err, int *timeout)
{
  const int ld = ((k + n + 3) / 4) * 4;
  std::vector<float> h((size_t)(m + k) * ld);
  unsigned s = 12345u + (unsigned)(m * 7 + n * 13 + k);
  for (auto &x : h) { s = s * 1664525u + 1013904223u; x = (float)((s >> 8) * (1.0 / 16777216.0) - 0.5); }
  DBuf buf, ref;
  RB_TRY(buf.alloc(h.size() * 4));
  RB_TRY(ref.alloc(h.size() * 4));
  float *A = buf.as<float>() + (size_t)k * ld, *Bm = buf.as<float>() + k, *C = buf.as<float>() + (size_t)k * ld + k;
  float *Ar = ref.as<float>() + (size_t)k * ld, *Br = ref.as<float>() + k, *Cr = ref.as<float>() + (size_t)k * ld + k;
  RB_CUDA(cudaMemcpy(ref.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
  RB_CUDA(cudaMemcpy(buf.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
  tc_ref_kernel<<<dim3((n + 127) / 128, m), 128>>>(Cr, ld, m, n, k, Ar, Br, overwrite);
  RB_TRY(check_launch("tc_ref_kernel"));
  RB_CUDA(cudaMemset(g_tc_err_flag.p, 0, sizeof(int)));
  int rc = launch_tc(C, ld, m, n, k, A, ld, Bm, ld, 0, overwrite, 2, use_tma);
  if (rc == RADB200_E_UNSUPPORTED) {  // no tensor-map encoder: nothing was launched
    *err = 1.0;
    *timeout = 0;
    return 0;
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (rc != 0 || e != cudaSuccess) {
    cudaGetLastError();
    set_error("tensor-core self-test launch failed: %s", cudaGetErrorString(e));
    return e != cudaSuccess ? RADB200_E_CUDA : rc;
  }
  int flag = 0;
  RB_CUDA(cudaMemcpy(&flag, g_tc_err_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
  *timeout = flag != 0;
  std::vector<float> cref(h.size()), ctc(h.size());
  RB_CUDA(cudaMemcpy(cref.data(), ref.p, h.size() * 4, cudaMemcpyDeviceToHost));
  RB_CUDA(cudaMemcpy(ctc.data(), buf.p, h.size() * 4, cudaMemcpyDeviceToHost));
  double maxd = 0.0, maxr = 0.0;
  for (size_t i = 0; i < ctc.size(); i++) {
    maxd = std::max(maxd, (double)fabs(ctc[i] - cref[i]));
    maxr = std::max(maxr, (double)fabs(cref[i]));
  }
  *err = maxd / maxr;
  return 0;
}

// Keeps the tensor-core path only if every case matches the CUDA-core
// reference to TF32 accuracy: K of 4 chunks of 32 (120) and of 10 (300),
// ragged m and n, and the overwrite form the LU panels use.  The cp.async-fed
// kernel is tested first, then the TMA-fed kernel with TF32 operands, then
// with scaled FP16 operands (the same 11-bit significand as TF32 inside the
// scaled range); each is used only if it and the ones before it pass every
// case.  RADB200_TC_F16=0 stops at the TF32 TMA kernel (A/B comparisons).
static int tc_selftest()
{
  RB_TRY(g_tc_err_flag.alloc(sizeof(int)));
  g_tc_state = 0;
  g_tc_tma = 0;
  g_tc_err = 0.0;
  const char *ef = getenv("RADB200_TC_F16");
  const int last = (ef && atoi(ef) == 0) ? 1 : 2;
  const int cases[3][4] = {{300, 400, 120, 0}, {300, 300, 300, 0}, {260, 290, 64, 1}};
  for (int use_tma = 0; use_tma <= last; use_tma++) {
    double worst = 0.0;
    for (auto &cs : cases) {
      double err = 1.0;
      int timeout = 0;
      RB_TRY(tc_selftest_case(cs[0], cs[1], cs[2], cs[3], use_tma, &err, &timeout));
      if (timeout) {  // an MMA or copy never completed: leave this kernel off
        set_error("tensor-core self-test: a completion wait timed out (%s kernel)",
                  use_tma == 2 ? "TMA FP16" : use_tma ? "TMA" : "cp.async");
        RB_CUDA(cudaMemset(g_tc_err_flag.p, 0, sizeof(int)));  // the kernels before it may still run
        return 0;
      }
      worst = std::max(worst, err);
    }
    if (!(worst < 1e-4)) return 0;
    if (use_tma) g_tc_tma = use_tma;
    else { g_tc_state = 1; g_tc_err = worst; }
  }
  return 0;
}

int tc_gemm_f32(float *C, int ldc, int m, int n, int k, float *A, int lda, const float *B, int ldb, cudaStream_t st,
                int *used, int overwrite, int slot, int max_ctas)
{
  *used = 0;
  static const bool no_tc = getenv("RADB200_NO_TC") != nullptr;
  if (no_tc) return 0;
  if (k < 1 || m <= 0 || n <= 0 || (ldc % 4) || (lda % 4) || (ldb % 4) || ((uintptr_t)C & 15) || ((uintptr_t)A & 15) ||
      ((uintptr_t)B & 15))
    return 0;
  if (g_tc_state < 0) RB_TRY(tc_selftest());
  if (g_tc_state <= 0) return 0;
  RB_TRY(g_tc_err_flag.alloc(sizeof(int)));
  RB_TRY(launch_tc(C, ldc, m, n, k, A, lda, B, ldb, st, overwrite, max_ctas, -1, slot));
  *used = g_tc_tma == 2 ? 2 : 1;  // 2: the operands went to the tensor cores as FP16
  return 0;
}

// C = A B where C is the same memory as A (c_is_a, n <= TC_BN: every row
// tile of C is written by the one CTA that reads those rows of A, after its
// MMAs have consumed them; with FP16 operands A is read from its converted
// copy anyway) or as B (B is transposed or converted into scratch before the
// update runs).  Only the TMA-fed kernels give these guarantees: with the
// cp.async kernel or no tensor cores *used = 0 and the caller goes out of place.
int tc_gemm_f32_inplace(float *C, int ldc, int m, int n, int k, float *A, int lda, const float *B, int ldb,
                        cudaStream_t st, int *used, bool c_is_a, int slot)
{
  *used = 0;
  if (g_tc_state < 0) RB_TRY(tc_selftest());
  if (g_tc_state <= 0 || g_tc_tma == 0) return 0;
  if (c_is_a && n > TC_BN) return 0;
  return tc_gemm_f32(C, ldc, m, n, k, A, lda, B, ldb, st, used, 1, slot, 0);
}

int tc_error_flag(int *flag)
{
  *flag = 0;
  if (!g_tc_err_flag.p) return 0;
  RB_CUDA(cudaMemcpy(flag, g_tc_err_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
  return 0;
}

}  // namespace rb

extern "C" RADB200_API int radb200_tc_selftest(int *state, double *err)
{
  if (rb::g_tc_state < 0) RB_TRY(rb::tc_selftest());
  *state = rb::g_tc_state + rb::g_tc_tma;  // 0 off, 1 cp.async-fed kernel, 2 TMA-fed kernel, 3 with FP16 operands
  *err = rb::g_tc_err;
  return 0;
}
