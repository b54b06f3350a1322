// Input formats ahead of the analysis: the Matrix Market reader and the
// COO -> CCS conversion of the reference's driver (example.f90:63-145), the
// conversion on the GPU, and direct CSR input to the handle API.
//
//  * mfd_mm_read (host): coordinate file, '%' header lines skipped, then
//    "n n nnz" and nnz lines "row col value" (read_data, example.f90:63-93).
//  * mfd_coo_to_ccs (device): the reference's two counting sorts (by row,
//    then by column, example.f90:95-145) give, in each column, the rows in
//    ascending order and entries with equal (row, col) in reverse input order.
//    Here: one stable radix sort of the keys (col, row) taken over the
//    entries in reverse input order, which yields exactly that order.
//  * mfd_analyze_csr: a lower-triangle or full symmetric CSR (0- or 1-based)
//    becomes the lower CCS on the device, the reference's analysis runs on it,
//    and the handle's value sources are re-pointed at the CSR positions, so
//    mfd_factorize takes the values in the caller's CSR order.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mfdag.h"
#include "kernels.cuh"

namespace mfd {
// defined in api.cu
int handle_set_value_map(mfd_handle* h, const int32_t* d_map, int64_t a_len);
int set_error(int code, const std::string& msg);

namespace {

#define CKI(call)                                                                                             \
  do {                                                                                                        \
    cudaError_t e_ = (call);                                                                                  \
    if (e_ != cudaSuccess)                                                                                    \
      return set_error(e_ == cudaErrorMemoryAllocation ? MFD_E_NOMEM : MFD_E_CUDA,                             \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                                   \
  } while (0)

template <typename T>
struct DMem {
  T* p = nullptr;
  ~DMem() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

bool on_device(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// key of input entry nnz-1-i (reverse input order): column in the high half,
// row in the low half (both 1-based); payload: the input position
__global__ void k_coo_keys(const int32_t* row, const int32_t* col, int64_t nnz, uint64_t* key, int32_t* pos) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = nnz - 1 - i;
    key[i] = ((uint64_t)(uint32_t)col[k] << 32) | (uint32_t)row[k];
    pos[i] = (int32_t)k;
  }
}

// sorted keys -> CCS rows, values and per-column counts
__global__ void k_ccs_rows(const uint64_t* key, const int32_t* pos, const double* val, int64_t nnz, int32_t* ccs_row,
                           double* ccs_val, int32_t* count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = key[i];
    ccs_row[i] = (int32_t)(uint32_t)(k & 0xffffffffu);
    if (ccs_val) ccs_val[i] = val[pos[i]];
    atomicAdd(&count[(int32_t)(k >> 32) - 1], 1);
  }
}

// column pointers (1-based) from the exclusive scan of the counts
__global__ void k_col_ptr(const int32_t* scan, int32_t n, int64_t nnz, int32_t* ccs_col) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j <= n; j += (int64_t)gridDim.x * blockDim.x)
    ccs_col[j] = j < n ? scan[j] + 1 : (int32_t)(nnz + 1);
}

// entries with an index outside 1..n (the conversion's input contract)
__global__ void k_coo_check(const int32_t* row, const int32_t* col, int64_t nnz, int32_t n, int32_t* bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x)
    if (row[i] < 1 || row[i] > n || col[i] < 1 || col[i] > n) atomicExch(bad, 1);
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096)); }

// Device conversion; every pointer is a device pointer.  val / ccs_val may be
// null (structure only); pos_out (may be null) receives, for every CCS entry,
// its position in the input.
int coo_to_ccs_device(int32_t n, int64_t nnz, const int32_t* row, const int32_t* col, const double* val,
                      int32_t* ccs_col, int32_t* ccs_row, double* ccs_val, int32_t* pos_out, cudaStream_t st) {
  if (n < 1 || nnz < 0 || nnz >= INT32_MAX) return set_error(MFD_E_ARG, "coo_to_ccs: need n >= 1 and nnz < 2^31");
  DMem<int32_t> bad;
  CKI(bad.alloc(1));
  CKI(cudaMemsetAsync(bad.p, 0, sizeof(int32_t), st));
  if (nnz > 0) k_coo_check<<<grid_for(nnz), 256, 0, st>>>(row, col, nnz, n, bad.p);
  int32_t hbad = 0;
  CKI(cudaMemcpyAsync(&hbad, bad.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CKI(cudaStreamSynchronize(st));
  if (hbad) return set_error(MFD_E_ARG, "coo_to_ccs: an index lies outside 1..n");
  DMem<uint64_t> k_in, k_out;
  DMem<int32_t> p_in, p_out, cnt, scan;
  CKI(k_in.alloc(nnz));
  CKI(k_out.alloc(nnz));
  CKI(p_in.alloc(nnz));
  CKI(p_out.alloc(nnz));
  CKI(cnt.alloc(n));
  CKI(scan.alloc(n));
  if (nnz > 0) k_coo_keys<<<grid_for(nnz), 256, 0, st>>>(row, col, nnz, k_in.p, p_in.p);
  // sort on the bits the keys use: 32 row bits + the column's bits
  int cbits = 1;
  while (cbits < 31 && (1ll << cbits) <= (long long)n) ++cbits;
  size_t tmp_bytes = 0;
  CKI(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, k_in.p, k_out.p, p_in.p, p_out.p, (int)nnz, 0, 32 + cbits,
                                      st));
  DMem<unsigned char> tmp;
  CKI(tmp.alloc(tmp_bytes));
  CKI(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, k_in.p, k_out.p, p_in.p, p_out.p, (int)nnz, 0, 32 + cbits,
                                      st));
  CKI(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * n, st));
  if (nnz > 0) k_ccs_rows<<<grid_for(nnz), 256, 0, st>>>(k_out.p, p_out.p, val, nnz, ccs_row, ccs_val, cnt.p);
  size_t scan_bytes = 0;
  CKI(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt.p, scan.p, n, st));
  DMem<unsigned char> stmp;
  CKI(stmp.alloc(scan_bytes));
  CKI(cub::DeviceScan::ExclusiveSum(stmp.p, scan_bytes, cnt.p, scan.p, n, st));
  k_col_ptr<<<grid_for(n + 1), 256, 0, st>>>(scan.p, n, nnz, ccs_col);
  if (pos_out && nnz > 0) CKI(cudaMemcpyAsync(pos_out, p_out.p, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, st));
  CKI(cudaGetLastError());
  CKI(cudaStreamSynchronize(st));
  return MFD_OK;
}

}  // namespace
}  // namespace mfd

using namespace mfd;

extern "C" {
#pragma GCC visibility push(default)

int mfd_mm_read(const char* path, mfd_coo* out) {
  if (!path || !out) return set_error(MFD_E_ARG, "mfd_mm_read: null argument");
  std::memset(out, 0, sizeof(*out));
  FILE* fp = std::fopen(path, "r");
  if (!fp) return set_error(MFD_E_ARG, std::string("cannot open: ") + path);
  std::string line;
  char buf[4096];
  bool pattern = false, have_size = false;
  long long n1 = 0, n2 = 0, nz = 0, k = 0;
  int rc = MFD_OK;
  while (std::fgets(buf, sizeof(buf), fp)) {
    if (buf[0] == '%') {                                   // banner and comments (read_data skips them)
      std::string h(buf);
      for (auto& c : h) c = (char)std::tolower((unsigned char)c);
      if (h.rfind("%%matrixmarket", 0) == 0) {
        if (h.find("coordinate") == std::string::npos || h.find("complex") != std::string::npos) {
          rc = set_error(MFD_E_ARG, "mfd_mm_read: only real / integer / pattern coordinate files");
          break;
        }
        pattern = h.find("pattern") != std::string::npos;
      }
      continue;
    }
    char* s = buf;
    while (*s && std::isspace((unsigned char)*s)) ++s;
    if (!*s) continue;                                     // blank line
    if (!have_size) {
      if (std::sscanf(s, "%lld %lld %lld", &n1, &n2, &nz) != 3 || n1 < 1 || n1 != n2 || nz < 0 || n1 > INT32_MAX) {
        rc = set_error(MFD_E_ARG, "mfd_mm_read: bad size line (need a square matrix: n n nnz)");
        break;
      }
      have_size = true;
      out->n = (int32_t)n1;
      out->nnz = nz;
      out->row = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max<long long>(nz, 1)));
      out->col = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max<long long>(nz, 1)));
      out->val = static_cast<double*>(std::malloc(sizeof(double) * std::max<long long>(nz, 1)));
      if (!out->row || !out->col || !out->val) {
        rc = set_error(MFD_E_NOMEM, "mfd_mm_read: out of host memory");
        break;
      }
      continue;
    }
    if (k >= nz) break;
    long long r = 0, c = 0;
    double v = 1.0;
    const int got = pattern ? std::sscanf(s, "%lld %lld", &r, &c) : std::sscanf(s, "%lld %lld %lf", &r, &c, &v);
    if (got != (pattern ? 2 : 3) || r < 1 || r > n1 || c < 1 || c > n1) {
      rc = set_error(MFD_E_ARG, "mfd_mm_read: bad entry line " + std::to_string(k + 1));
      break;
    }
    out->row[k] = (int32_t)r;
    out->col[k] = (int32_t)c;
    out->val[k] = v;
    ++k;
  }
  std::fclose(fp);
  if (rc == MFD_OK && (!have_size || k != nz))
    rc = set_error(MFD_E_ARG, "mfd_mm_read: file ends before its " + std::to_string(nz) + " entries");
  if (rc != MFD_OK) mfd_coo_free(out);
  return rc;
}

void mfd_coo_free(mfd_coo* coo) {
  if (!coo) return;
  std::free(coo->row);
  std::free(coo->col);
  std::free(coo->val);
  std::memset(coo, 0, sizeof(*coo));
}

int mfd_coo_to_ccs(int32_t n, int64_t nnz, const int32_t* row, const int32_t* col, const double* val,
                   int32_t* ccs_col, int32_t* ccs_row, double* ccs_val, int32_t device) {
  if (!row || !col || !ccs_col || !ccs_row || (val && !ccs_val) || (!val && ccs_val))
    return set_error(MFD_E_ARG, "mfd_coo_to_ccs: null argument");
  CKI(cudaSetDevice(device));
  cudaStream_t st;
  CKI(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{st};
  const bool din = on_device(row), dout = on_device(ccs_row);
  // stage host arrays on the device
  DMem<int32_t> drow, dcol, dccol, dcrow;
  DMem<double> dval, dcval;
  const int32_t *r = row, *c = col;
  const double* v = val;
  if (!din) {
    CKI(drow.alloc(nnz));
    CKI(dcol.alloc(nnz));
    CKI(cudaMemcpyAsync(drow.p, row, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
    CKI(cudaMemcpyAsync(dcol.p, col, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
    r = drow.p;
    c = dcol.p;
    if (val) {
      CKI(dval.alloc(nnz));
      CKI(cudaMemcpyAsync(dval.p, val, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
      v = dval.p;
    }
  }
  int32_t *oc = ccs_col, *orow = ccs_row;
  double* ov = ccs_val;
  if (!dout) {
    CKI(dccol.alloc((size_t)n + 1));
    CKI(dcrow.alloc(nnz));
    oc = dccol.p;
    orow = dcrow.p;
    if (val) {
      CKI(dcval.alloc(nnz));
      ov = dcval.p;
    }
  }
  int rc = coo_to_ccs_device(n, nnz, r, c, v, oc, orow, ov, nullptr, st);
  if (rc) return rc;
  if (!dout) {
    CKI(cudaMemcpyAsync(ccs_col, oc, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost, st));
    if (nnz > 0) CKI(cudaMemcpyAsync(ccs_row, orow, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
    if (val && nnz > 0) CKI(cudaMemcpyAsync(ccs_val, ov, sizeof(double) * nnz, cudaMemcpyDeviceToHost, st));
    CKI(cudaStreamSynchronize(st));
  }
  return MFD_OK;
}

int mfd_analyze_csr(mfd_handle** h, int32_t n, const int32_t* csr_ptr, const int32_t* csr_col, int32_t base,
                    const int32_t* order_perm, const mfd_options* opt) {
  if (!h || !csr_ptr || !csr_col || n < 1 || (base != 0 && base != 1))
    return set_error(MFD_E_ARG, "mfd_analyze_csr: null argument, n < 1 or base not 0 / 1");
  const int64_t len = (int64_t)csr_ptr[n] - csr_ptr[0];
  if (len < 1 || len >= INT32_MAX || csr_ptr[0] != base) return set_error(MFD_E_ARG, "mfd_analyze_csr: bad row pointers");
  // the lower triangle as COO (1-based) with each entry's CSR position
  std::vector<int32_t> cr, cc, cpos;
  cr.reserve(len);
  cc.reserve(len);
  cpos.reserve(len);
  for (int32_t i = 0; i < n; ++i) {
    if (csr_ptr[i + 1] < csr_ptr[i]) return set_error(MFD_E_ARG, "mfd_analyze_csr: row pointers decrease");
    for (int32_t k = csr_ptr[i] - base; k < csr_ptr[i + 1] - base; ++k) {
      const int32_t j = csr_col[k] - base;
      if (j < 0 || j >= n) return set_error(MFD_E_ARG, "mfd_analyze_csr: column index outside the matrix");
      if (j > i) continue;                                  // upper triangle: the symmetric copy is in the lower one
      cr.push_back(i + 1);
      cc.push_back(j + 1);
      cpos.push_back(k);
    }
  }
  const int64_t nnz = (int64_t)cr.size();
  int dev = opt ? opt->device : 0;
  CKI(cudaSetDevice(dev));
  cudaStream_t st;
  CKI(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{st};
  DMem<int32_t> drow, dcol, dccol, dcrow, dpos, dmap;
  CKI(drow.alloc(nnz));
  CKI(dcol.alloc(nnz));
  CKI(dccol.alloc((size_t)n + 1));
  CKI(dcrow.alloc(nnz));
  CKI(dpos.alloc(nnz));
  CKI(dmap.alloc(nnz));
  CKI(cudaMemcpyAsync(drow.p, cr.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
  CKI(cudaMemcpyAsync(dcol.p, cc.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
  CKI(cudaMemcpyAsync(dmap.p, cpos.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
  int rc = coo_to_ccs_device(n, nnz, drow.p, dcol.p, nullptr, dccol.p, dcrow.p, nullptr, dpos.p, st);
  if (rc) return rc;
  std::vector<int32_t> ccol((size_t)n + 1), crow(nnz), pos(nnz);
  CKI(cudaMemcpyAsync(ccol.data(), dccol.p, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost, st));
  CKI(cudaMemcpyAsync(crow.data(), dcrow.p, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
  CKI(cudaMemcpyAsync(pos.data(), dpos.p, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
  CKI(cudaStreamSynchronize(st));
  // CCS entry k is COO entry pos[k], which is CSR entry cpos[pos[k]]
  std::vector<int32_t> map(nnz);
  for (int64_t k = 0; k < nnz; ++k) map[k] = cpos[pos[k]];
  rc = mfd_analyze(h, n, ccol.data(), crow.data(), order_perm, opt);
  if (rc) return rc;
  CKI(cudaMemcpyAsync(dmap.p, map.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
  CKI(cudaStreamSynchronize(st));
  rc = handle_set_value_map(*h, dmap.p, len);
  if (rc) {
    mfd_destroy(*h);
    *h = nullptr;
  }
  return rc;
}

#pragma GCC visibility pop
}  // extern "C"
