// Factorization of dense fronts without any device allocation.
//
// Some callers cannot call cudaMalloc: code that runs while its process holds
// all device memory in its own arena (a Fortran driver or framework that
// reserved HBM up front and sub-allocates it itself), or a latency-critical
// loop that must not take the CUDA allocator's lock or trigger its implicit
// synchronisation.  mfd_factor_fronts_noalloc serves them: the caller passes
// the fronts in one device buffer it already owns, and the only scratch the
// blocked factorization needs -- one inverted 128x128 diagonal block per front
// and the small front tables -- lives in the file-scope array below, which
// every GPU that loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mfdag.h"
#include "kernels.cuh"
#include "plan.hpp"

namespace mfd {
namespace {

constexpr int kMaxFronts = MFD_NOALLOC_MAX_FRONTS;
constexpr size_t kInvElems = (size_t)kMaxFronts * kFactB * kFactB;      // L11^{-1} blocks (FP64)
constexpr size_t kTableWords = 8 * kMaxFronts + 8;                        // front tables, in 8-byte words
constexpr size_t kScratchElems = kInvElems + kTableWords;

// The only scratch of the no-allocation path: kMaxFronts x 128 x 128 doubles
// (1 MiB for 8 fronts) plus the front tables.  In host code this name is a
// host-side stand-in, not a device address; the device address comes from
// cudaGetSymbolAddress in scratch_on_device().
static __device__ __align__(256) double g_noalloc_scratch[kScratchElems];

std::mutex g_mu;
double* g_addr[256] = {};
thread_local std::string g_msg;

// Once per device, with that device current: look up the device address of the
// scratch array and opt the kernels into their shared-memory carve-out.
int scratch_on_device(int dev, double** out) {
  if (dev < 0 || dev >= 256) return MFD_E_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      g_msg = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return MFD_E_CUDA;
    }
    e = prepare_kernels();
    if (e != cudaSuccess) {
      g_msg = std::string("kernel attributes: ") + cudaGetErrorString(e);
      return MFD_E_CUDA;
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return MFD_OK;
}

}  // namespace
}  // namespace mfd

using namespace mfd;

extern "C" __attribute__((visibility("default"))) int mfd_factor_fronts_noalloc(
    double* fronts, int32_t count, const int64_t* panel_off, const int64_t* update_off, const int32_t* nf,
    const int32_t* nc, int32_t* info, void* stream) {
  if (!fronts || !panel_off || !update_off || !nf || !nc || !info) {
    g_msg = "null argument";
    return MFD_E_ARG;
  }
  if (count < 1 || count > kMaxFronts) {
    g_msg = "count must be between 1 and MFD_NOALLOC_MAX_FRONTS (" + std::to_string(kMaxFronts) + ")";
    return MFD_E_ARG;
  }
  int maxnc = 0;
  for (int i = 0; i < count; ++i) {
    if (nc[i] < 1 || nf[i] < nc[i] || panel_off[i] < 0 || update_off[i] < 0) {
      g_msg = "front " + std::to_string(i) + ": need 1 <= nc <= nf and non-negative offsets";
      return MFD_E_ARG;
    }
    maxnc = nc[i] > maxnc ? nc[i] : maxnc;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // A capture cannot record the host table copy or the info read-back below,
  // so a capturing stream is refused before anything is issued on it.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    g_msg = "cannot query the stream's capture status";
    return MFD_E_ARG;
  }
  if (cap != cudaStreamCaptureStatusNone) {
    g_msg = "the stream is being captured into a CUDA graph; this entry point cannot be captured";
    return MFD_E_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { g_msg = "no current device"; return MFD_E_CUDA; }
  double* scratch = nullptr;
  int rc = scratch_on_device(dev, &scratch);
  if (rc) return rc;

  // front tables in the scratch tail: nc, nr, first, list | panel_off, u_off | info per front
  struct Tables {
    int32_t nc[kMaxFronts], nr[kMaxFronts], first[kMaxFronts], list[kMaxFronts];
    int64_t poff[kMaxFronts], uoff[kMaxFronts];
    int32_t info[kMaxFronts];
  } t;
  static_assert(sizeof(Tables) <= kTableWords * sizeof(double), "table area too small");
  std::memset(&t, 0, sizeof(t));
  for (int i = 0; i < count; ++i) {
    t.nc[i] = nc[i];
    t.nr[i] = nf[i] - nc[i];
    t.first[i] = 0;
    t.list[i] = i;
    t.poff[i] = panel_off[i];
    t.uoff[i] = update_off[i];
  }
  for (int i = 0; i < kMaxFronts; ++i) t.info[i] = INT_MAX;   // the array keeps the last call's contents
  Tables* dt = reinterpret_cast<Tables*>(scratch + kInvElems);
  cudaError_t e = cudaMemcpyAsync(dt, &t, sizeof(t), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) { g_msg = cudaGetErrorString(e); return MFD_E_CUDA; }

  DevFronts F{};
  F.nc = dt->nc;
  F.nr = dt->nr;
  F.first = dt->first;
  F.panel_off = dt->poff;
  F.u_off = dt->uoff;
  const int32_t* list = dt->list;
  int32_t* dinfo = dt->info;                         // slot i: front i's first bad pivot (list[i] = i)
  const int steps = (maxnc + kFactB - 1) / kFactB;
  for (int s = 0; s < steps; ++s) {
    int rows = 0, tiles = 0;                         // TRSM row blocks, update tiles per side
    for (int i = 0; i < count; ++i) {
      if (nc[i] <= s * kFactB) continue;
      int w = nc[i] - s * kFactB < kFactB ? nc[i] - s * kFactB : kFactB;
      int nrem = nf[i] - s * kFactB - w;
      int rb = (nrem + kTrRowsH - 1) / kTrRowsH, T = (nrem + kUpdTile - 1) / kUpdTile;
      rows = rb > rows ? rb : rows;
      tiles = T > tiles ? T : tiles;
    }
    // fronts whose columns are exhausted return at once inside the kernels
    launch_potrf<double>(F, list, count, s, fronts, scratch, dinfo, st, false, 1);
    launch_trsm<double>(F, list, count, s, rows, fronts, scratch, 0, st);
    launch_update<double>(F, list, count, s, tiles, 0, fronts, fronts, 0, st);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) { g_msg = cudaGetErrorString(e); return MFD_E_CUDA; }
  int32_t hinfo[kMaxFronts];
  e = cudaMemcpyAsync(hinfo, dinfo, sizeof(int32_t) * count, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) { g_msg = cudaGetErrorString(e); return MFD_E_CUDA; }
  for (int i = 0; i < count; ++i) info[i] = hinfo[i] == INT_MAX ? 0 : hinfo[i];
  return MFD_OK;
}

extern "C" __attribute__((visibility("default"))) const char* mfd_noalloc_last_error(void) { return g_msg.c_str(); }
