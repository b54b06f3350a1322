// Trailing update of the FP32 factorization on the 5th-generation tensor cores.
//
// One CTA per 128 x 128 tile of the trailing lower triangle of a front,
// C -= P_i P_j^T with P the solved panel rows over the K range of the step's
// deferred group (update_k_range: up to defer x 128 columns):
//   * operands are staged by all 256 threads from the panel (global) into
//     shared memory in the canonical K-major, no-swizzle UMMA layout
//     (8-row x 16-byte core matrices), split into TF32 hi / lo parts;
//   * one elected thread issues tcgen05.mma.kind::tf32 (M = N = 128, K = 8)
//     with the accumulator in tensor memory: hi*hi + hi*lo + lo*hi per K step
//     (3xTF32, ~FP32 accuracy) or hi*hi only (1xTF32);
//   * K runs in stages of 16 with two shared-memory buffers: the MMAs of one
//     stage overlap the loads of the next, tcgen05.commit on an mbarrier frees
//     a buffer;
//   * the epilogue reads the accumulator with tcgen05.ld (warp w sees TMEM
//     lanes 32 (w mod 4) ..; warps 4-7 take the upper 64 columns) and
//     subtracts it from C in place (column-major panel / update matrix, rows
//     across lanes: coalesced).
// Every mbarrier wait is bounded (~1 s); on expiry the kernel raises err[0],
// waits once more (bounded, ~8 s: MMAs finish in microseconds) for its MMAs,
// frees its tensor memory and returns.  err[1] != 0 is a test request: before
// any MMA, every CTA waits on an mbarrier that nothing arrives at, with a
// ~1 ms limit, so the expiry path runs without any fault.
//
// k_update_tcq (deferral depth 1, the default schedule) takes its operands
// already split: the step's TRSM writes the solved rows once as TF32 hi / lo
// blocks in the UMMA layout (packed_offset), so the main loop does no SIMT
// work per element.  Warp-specialised, one tile per CTA, two CTAs per SM:
//   * warp 0 (one thread): 1D bulk copies (cp.async.bulk, no multicast) of
//     each 16-column stage of A and B (16 KB each, hi and lo of two K = 8
//     chunks) into a three-stage ring, completion by mbarrier transaction
//     count; a stage is reused once the MMAs that read it have committed;
//   * warp 1 (one thread): waits for a stage, issues its tcgen05.mma
//     (3xTF32 or 1xTF32), commits to the stage's empty barrier, and at the end
//     to the accumulator barrier;
//   * all eight warps load their C elements before the main loop (the loads
//     fly while the MMAs run), wait for the accumulator and subtract it.
// Every wait is bounded; a wait that expires sets a shared abort flag that
// the other roles' waits also watch, raises err[0], and the CTA drains its
// copies and MMAs (bounded) before freeing its tensor memory.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "kernels.cuh"

namespace mfd {
namespace {

constexpr int kTcTile = 128;
constexpr int kTcK = 16;                                   // K per stage: 2 MMAs of K = 8
constexpr int kTcThreads = 256;
constexpr uint32_t kSbo = (kTcK / 4) * 128;                // bytes between 8-row groups
constexpr uint32_t kOpBytes = kTcTile * kTcK * 4;          // one 128 x 16 fp32 operand: 8 KB
constexpr uint32_t kStageBytes = 4 * kOpBytes;             // A hi, A lo, B hi, B lo
constexpr uint32_t kTmemCols = 128;                        // fp32 accumulator 128 lanes x 128 columns
constexpr size_t kTcSmem = 2 * (size_t)kStageBytes + 1024 + 64;
constexpr int kPairs = kTcTile * (kTcK / 4) / kTcThreads;  // (row, k-quad) pairs per thread per operand

// byte offset of element (row, k) (k a multiple of 4) in a 128 x kTcK operand:
// k-cores of 16 B adjacent (128 B apart), 8-row groups kSbo apart
__device__ __forceinline__ uint32_t op_offset(int row, int k) {
  return (uint32_t)((row >> 3) * kSbo + (row & 7) * 16 + (k >> 2) * 128);
}

// UMMA shared-memory descriptor (sm_100): start address, leading byte offset
// (between the two 16-byte k-cores of one K = 8 step), stride byte offset
// (between 8-row groups), version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((kSbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: D = f32 (bits 4-5), A = B = tf32 (bits 7-9, 10-12),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcTile >> 3) << 17) |
                            ((uint32_t)(kTcTile >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

constexpr long long kWaitLimit = 1ll << 31;        // cycles (~1.1 s at 1.965 GHz)
constexpr long long kDrainLimit = 1ll << 34;       // the final wait for issued MMAs
constexpr long long kProbeLimit = 1ll << 21;       // the test request's wait (~1 ms)

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit = kWaitLimit) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  return __uint_as_float(h);
}

__global__ void __launch_bounds__(kTcThreads, 2) k_update_tc(DevFronts F, const int32_t* list, int step,
                                                             float* panel, float* upool, int split, int32_t* err,
                                                             int blo, int bhi, int defer) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  const int c0 = step * kFactB;
  if (c0 >= nc) return;
  const int w = min(kFactB, nc - c0);
  const int base = c0 + w;
  const int nrem = nf - base;
  if (nrem <= 0) return;
  const int T = (nrem + kTcTile - 1) / kTcTile;
  int ti, tj, kbeg, kend;
  if (!select_tile(T, kTcTile, blo, bhi, blockIdx.x, ti, tj)) return;
  if (!update_k_range(nc, step, defer, tj, kTcTile, kbeg, kend)) return;
  const int K = kend - kbeg;                        // panel columns [kbeg, kend) of the front
  const int i0 = base + ti * kTcTile, j0 = base + tj * kTcTile;
  const bool diag = ti == tj;
  float* P = panel + F.panel_off[f];
  float* U = upool + F.u_off[f];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // 1024-byte aligned stage area, then two mbarriers, the TMEM address slot
  // and the test request's mbarrier
  const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  unsigned char* sm = smem_raw + pad;
  const uint32_t sb = raw + pad;
  const uint32_t mbar0 = sb + 2 * kStageBytes, mbar1 = mbar0 + 8, mbar_probe = mbar0 + 24;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + 2 * kStageBytes + 16);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sb + 2 * kStageBytes + 16),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar0));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_probe));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  pdl_wait();                       // the panel rows are the preceding TRSM's output
  pdl_trigger();

  const int nch = (K + kTcK - 1) / kTcK;
  bool ok = true;
  int issued = 0;                                   // stages whose MMAs were committed
  if (err[1]) ok = __syncthreads_and(mbar_wait(mbar_probe, 0, kProbeLimit)) != 0;   // test request: expires
  for (int c = 0; c < nch; ++c) {
    const int buf = c & 1;
    const uint32_t mb = buf ? mbar1 : mbar0;
    if (c >= 2 && ok) ok = __syncthreads_and(mbar_wait(mb, ((c - 2) >> 1) & 1)) != 0;
    if (!ok) break;
    unsigned char* st = sm + buf * kStageBytes;
    // stage: (row, k-quad) pairs; all global loads first, then split and store
    float x[2][kPairs][4];
#pragma unroll
    for (int op = 0; op < 2; ++op)
#pragma unroll
      for (int u = 0; u < kPairs; ++u) {
        const int pr = tid + u * kTcThreads;
        const int row = pr & (kTcTile - 1), kk = c * kTcK + 4 * (pr >> 7);
        const int grow = (op == 0 ? i0 : j0) + row;
        const bool need = op == 0 || !diag;
#pragma unroll
        for (int e = 0; e < 4; ++e)
          x[op][u][e] = (need && grow < nf && kk + e < K) ? P[grow + (size_t)(kbeg + kk + e) * nf] : 0.0f;
      }
#pragma unroll
    for (int op = 0; op < 2; ++op) {
      if (op == 1 && diag) break;
#pragma unroll
      for (int u = 0; u < kPairs; ++u) {
        const int pr = tid + u * kTcThreads;
        const uint32_t off = op_offset(pr & (kTcTile - 1), 4 * (pr >> 7));
        float4 hi, lo;
        if (split) {
          hi = make_float4(tf32_hi(x[op][u][0]), tf32_hi(x[op][u][1]), tf32_hi(x[op][u][2]), tf32_hi(x[op][u][3]));
          lo = make_float4(x[op][u][0] - hi.x, x[op][u][1] - hi.y, x[op][u][2] - hi.z, x[op][u][3] - hi.w);
        } else {
          hi = make_float4(x[op][u][0], x[op][u][1], x[op][u][2], x[op][u][3]);
          lo = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        *reinterpret_cast<float4*>(st + (2 * op) * kOpBytes + off) = hi;
        *reinterpret_cast<float4*>(st + (2 * op + 1) * kOpBytes + off) = lo;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      const uint32_t aH = sb + buf * kStageBytes, aL = aH + kOpBytes;
      const uint32_t bH = diag ? aH : aH + 2 * kOpBytes, bL = diag ? aL : aH + 3 * kOpBytes;
#pragma unroll
      for (int k8 = 0; k8 < kTcK / 8; ++k8) {
        const uint32_t o = k8 * 256;          // two 16-byte k-cores per K = 8 step
        mma_tf32(tmem, smem_desc(aH + o), smem_desc(bH + o), (c > 0 || k8 > 0) ? 1u : 0u);
        if (split) {
          mma_tf32(tmem, smem_desc(aH + o), smem_desc(bL + o), 1u);
          mma_tf32(tmem, smem_desc(aL + o), smem_desc(bH + o), 1u);
        }
      }
      mma_commit(mb);
    }
    issued = c + 1;
  }
  if (ok) ok = __syncthreads_and(mbar_wait((nch - 1) & 1 ? mbar1 : mbar0, ((nch - 1) >> 1) & 1)) != 0;
  fence_after_sync();
  if (ok) {
    const int q = warp & 3, half = warp >> 2;
    const int gi = i0 + 32 * q + lane;
#pragma unroll 1
    for (int part = 0; part < 2; ++part) {
      const int col0 = 64 * half + 32 * part;
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)col0, v);
      // all 32 loads of C before any store: independent accesses in flight
      const bool row_ok = gi < nf;
      float cur[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int gj = j0 + col0 + j;
        cur[j] = (row_ok && gj < nf && gi >= gj)
                     ? (gj < nc ? P[gi + (size_t)gj * nf] : U[(gi - nc) + (size_t)(gj - nc) * nr])
                     : 0.0f;
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int gj = j0 + col0 + j;
        if (row_ok && gj < nf && gi >= gj) {
          const float r = cur[j] - __uint_as_float(v[j]);
          if (gj < nc) P[gi + (size_t)gj * nf] = r;
          else U[(gi - nc) + (size_t)(gj - nc) * nr] = r;
        }
      }
    }
  } else {
    if (tid == 0) atomicExch(err, 1);
    // MMAs may still be in flight: one more bounded wait for the last commit (it covers all earlier MMAs)
    if (issued > 0) mbar_wait((issued - 1) & 1 ? mbar1 : mbar0, ((issued - 1) >> 1) & 1, kDrainLimit);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// ---- packed-operand variant --------------------------------------------------------
constexpr uint32_t kQChunkBytes = kTcTile * 8 * 4;              // one 128 x 8 hi (or lo) block: 4 KB
constexpr int kQStageChunks = 2;                                 // K = 16 per stage
constexpr uint32_t kQOpStage = kQStageChunks * 2 * kQChunkBytes; // 16 KB: hi, lo of two chunks
constexpr int kQStages = 3;
constexpr uint32_t kQStageBytes = 2 * kQOpStage;                 // A, B
constexpr uint32_t kQBarOff = kQStages * kQStageBytes;           // 96 KB of stages
constexpr size_t kQSmem = (size_t)kQBarOff + 128 + 1024;
constexpr uint32_t kQSbo = 256;                                  // between 8-row groups of a K = 8 block

__device__ __forceinline__ uint64_t smem_desc_q(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((kQSbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// bounded wait that also gives up when another role raised the CTA's abort flag
__device__ __forceinline__ bool mbar_wait_ab(uint32_t mbar, uint32_t parity, volatile int* abort_flag,
                                             long long limit) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (*abort_flag) return false;
    if (clock64() - t0 > limit) {
      *abort_flag = 1;
      return false;
    }
  }
}

__global__ void __launch_bounds__(kTcThreads, 2) k_update_tcq(DevFronts F, const int32_t* list, int step,
                                                              const float* __restrict__ q, float* panel,
                                                              float* upool, int split, int32_t* err, int blo,
                                                              int bhi) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int f = list[blockIdx.y];
  const int nc = F.nc[f], nr = F.nr[f], nf = nc + nr;
  const int c0 = step * kFactB;
  if (c0 >= nc) return;
  const int w = min(kFactB, nc - c0);
  const int base = c0 + w;
  const int nrem = nf - base;
  if (nrem <= 0) return;
  const int T = (nrem + kTcTile - 1) / kTcTile;
  int ti, tj, kbeg, kend;
  if (!select_tile(T, kTcTile, blo, bhi, blockIdx.x, ti, tj)) return;
  if (!update_k_range(nc, step, 1, tj, kTcTile, kbeg, kend)) return;
  const int nchunk = (kend - kbeg + 7) / 8;         // K = 8 chunks of the packed operands
  const int nst = (nchunk + kQStageChunks - 1) / kQStageChunks;
  const int i0 = base + ti * kTcTile, j0 = base + tj * kTcTile;
  const bool diag = ti == tj;
  float* P = panel + F.panel_off[f];
  float* U = upool + F.u_off[f];
  const float* QA = q + F.q_off[f] + (int64_t)ti * packed_block_elems();
  const float* QB = q + F.q_off[f] + (int64_t)tj * packed_block_elems();

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  unsigned char* sm = smem_raw + pad;
  const uint32_t sb = raw + pad;
  // barriers: full[3] at +0, empty[3] at +24, accumulator at +48, test probe at +56;
  // TMEM address slot at +64, abort flag at +72
  const uint32_t bar = sb + kQBarOff;
  const uint32_t bar_acc = bar + 48, bar_probe = bar + 56;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kQBarOff + 64);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + kQBarOff + 72);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(bar + 64),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < 8; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar + 8 * i));
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  pdl_wait();                       // the packed rows and C are the preceding kernels' output
  pdl_trigger();

  // this thread's C elements: row gi, columns j0 + 64 half + 32 part + [0, 32); part 0 is
  // loaded now (in flight during the MMAs), part 1 after part 0 is stored
  const int qr = warp & 3, half = warp >> 2;
  const int gi = i0 + 32 * qr + lane;
  const bool row_ok = gi < nf;
  // a tile wholly inside the matrix, below the diagonal and wholly in the panel or wholly in
  // the update matrix takes unpredicated accesses through one base and stride (the per-element
  // select of the general path keeps its loads from flying together)
  const bool full = i0 + kTcTile <= nf && j0 + kTcTile <= nf && i0 >= j0 + kTcTile && (j0 + kTcTile <= nc || j0 >= nc);
  const int ldc = j0 < nc ? nf : nr;
  float* Cb = (j0 < nc ? P + (size_t)j0 * nf : U + (size_t)(j0 - nc) * nr - nc) + gi;   // C(gi, j0 + j) = Cb[j ldc]
  float cur[64];
  if (full) {                       // both parts now
    const float* c = Cb + (size_t)(64 * half) * ldc;
#pragma unroll
    for (int j = 0; j < 64; ++j) cur[j] = c[(size_t)j * ldc];
  }
  auto load_c = [&](int part) {     // the general path, one part at a time
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int gj = j0 + 64 * half + 32 * part + j;
      cur[32 * part + j] = (row_ok && gj < nf && gi >= gj)
                               ? (gj < nc ? P[gi + (size_t)gj * nf] : U[(gi - nc) + (size_t)(gj - nc) * nr])
                               : 0.0f;
    }
  };
  if (!full) load_c(0);

  if (err[1]) {                     // test request: every CTA waits on a barrier nothing arrives at
    if (tid == 0) mbar_wait_ab(bar_probe, 0, abort_flag, kProbeLimit);
  }
  __syncthreads();
  int produced = 0;
  if (warp == 0 && lane == 0 && !*abort_flag) {
    for (int c = 0; c < nst; ++c) {
      const int s = c % kQStages;
      if (c >= kQStages && !mbar_wait_ab(bar + 24 + 8 * s, ((c / kQStages) - 1) & 1, abort_flag, kWaitLimit)) break;
      const int nck = min(kQStageChunks, nchunk - c * kQStageChunks);
      const uint32_t opb = (uint32_t)nck * 2 * kQChunkBytes;
      const uint32_t fb = bar + 8 * s;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(diag ? opb : 2 * opb)
                   : "memory");
      const uint32_t dA = sb + s * kQStageBytes;
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dA),
                   "l"(QA + (int64_t)c * kQStageChunks * 2048), "r"(opb), "r"(fb)
                   : "memory");
      if (!diag)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         dA + kQOpStage),
                     "l"(QB + (int64_t)c * kQStageChunks * 2048), "r"(opb), "r"(fb)
                     : "memory");
      produced = c + 1;
    }
  } else if (warp == 1 && lane == 0) {
    bool any = false;
    for (int c = 0; c < nst; ++c) {
      const int s = c % kQStages;
      if (!mbar_wait_ab(bar + 8 * s, (c / kQStages) & 1, abort_flag, kWaitLimit)) break;
      fence_after_sync();
      const int nck = min(kQStageChunks, nchunk - c * kQStageChunks);
      const uint32_t aS = sb + s * kQStageBytes, bS = diag ? aS : aS + kQOpStage;
      for (int j = 0; j < nck; ++j) {
        const uint32_t aH = aS + j * 2 * kQChunkBytes, aL = aH + kQChunkBytes;
        const uint32_t bH = bS + j * 2 * kQChunkBytes, bL = bH + kQChunkBytes;
        mma_tf32(tmem, smem_desc_q(aH), smem_desc_q(bH), (c > 0 || j > 0) ? 1u : 0u);
        if (split) {
          mma_tf32(tmem, smem_desc_q(aH), smem_desc_q(bL), 1u);
          mma_tf32(tmem, smem_desc_q(aL), smem_desc_q(bH), 1u);
        }
      }
      mma_commit(bar + 24 + 8 * s);
      any = true;
    }
    if (any)
      mma_commit(bar_acc);          // completes when every MMA issued above has
    else
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar_acc) : "memory");
  }
  __syncwarp();
  // the accumulator barrier always completes: the MMA thread commits to it, or arrives when it issued nothing
  const bool acc_ok = mbar_wait_ab(bar_acc, 0, abort_flag, kDrainLimit) || mbar_wait(bar_acc, 0, kDrainLimit);
  fence_after_sync();
  const bool ok = __syncthreads_and(acc_ok && !*abort_flag) != 0;
  if (ok) {
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      const int col0 = 64 * half + 32 * part;
      if (part == 1 && !full) load_c(1);
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(32 * qr) << 16) + (uint32_t)col0, v);
      if (full) {
        float* c = Cb + (size_t)col0 * ldc;
#pragma unroll
        for (int j = 0; j < 32; ++j) c[(size_t)j * ldc] = cur[32 * part + j] - __uint_as_float(v[j]);
        continue;
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int gj = j0 + col0 + j;
        if (row_ok && gj < nf && gi >= gj) {
          const float r = cur[32 * part + j] - __uint_as_float(v[j]);
          if (gj < nc) P[gi + (size_t)gj * nf] = r;
          else U[(gi - nc) + (size_t)(gj - nc) * nr] = r;
        }
      }
    }
  } else {
    if (tid == 0) atomicExch(err, 1);
    // copies still landing: wait (bounded) for every stage the producer issued and nobody consumed
    if (warp == 0 && lane == 0)
      for (int c = max(0, produced - kQStages); c < produced; ++c)
        mbar_wait(bar + 8 * (c % kQStages), (c / kQStages) & 1, kDrainLimit);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

cudaError_t prepare_update_tcq() {
  return cudaFuncSetAttribute(k_update_tcq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQSmem);
}

int launch_update_tcq(const DevFronts& F, const int32_t* list, int count, int step, int T128, const float* q,
                      float* panel, float* upool, int split, int32_t* err, cudaStream_t st, UpdBand band, bool pdl) {
  const int g = update_grid(T128, kTcTile, band);
  if (count <= 0 || g <= 0) return 0;
  launch_k(k_update_tcq, dim3(g, count), dim3(kTcThreads), kQSmem, st, pdl, F, list, step, q, panel, upool, split,
           err, band.blo, band.bhi);
  return 1;
}

cudaError_t prepare_update_tc() {
  return cudaFuncSetAttribute(k_update_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
}

int launch_update_tc(const DevFronts& F, const int32_t* list, int count, int step, int T128, float* panel,
                     float* upool, int split, int32_t* err, cudaStream_t st, UpdBand band, int defer, bool pdl) {
  const int g = update_grid(T128, kTcTile, band);
  if (count <= 0 || g <= 0) return 0;
  launch_k(k_update_tc, dim3(g, count), dim3(kTcThreads), kTcSmem, st, pdl, F, list, step, panel, upool, split, err,
           band.blo, band.bhi, defer);
  return 1;
}

}  // namespace mfd
