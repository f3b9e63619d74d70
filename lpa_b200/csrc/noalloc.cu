// One synchronous label-propagation iteration that allocates nothing.
//
// Some callers cannot allocate device memory. Examples: code running under a
// strict device-memory budget that is already fully spent, a caller that owns
// every buffer through its own pool, or a context where cudaMalloc is not
// permitted. lpa_create allocates all of its buffers, so it is unusable there.
// This entry point takes the compressed graph and both label buffers as
// caller-owned device memory and runs the two-pass path: decode into a CSR,
// then count. Its only working memory is one static device array,
// g_noalloc_scratch (kScratchBytes), which every GPU that loads the library
// holds until exit. Degrees, offsets, the decoded ids and three counters live
// there.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress, with that device current, and keeps it. The library
// loads its device code lazily, so that first call is also when the device
// claims the 16 MiB array and loads these kernels: make it before the caller
// spends its memory budget, and before any stream capture. The address is
// kept for the life of the process; a reset of the device's primary context
// (cudaDeviceReset) is not supported afterwards.
//
// Sharing: every call uses the same array, which keeps the last call's
// contents. The counters are cleared at the start of every call. Calls whose
// work overlaps on the GPU (other streams, other host threads) race on the
// array.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "noalloc.cuh"
#include "lpa_capi.h"

using namespace lpa_dev;

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;  // 16 MiB
constexpr int kMaxDevices = 64;

// File-scope scratch. In host code this name is a host-side stand-in, not a
// device address: kernels get the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};

lpa_status scratch_for_current_device(unsigned char **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return LPA_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) return LPA_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      // loading the module that holds the array is what allocates it
      return e == cudaErrorMemoryAllocation ? LPA_ERR_OOM : LPA_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return LPA_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" lpa_status lpa_iterate_noalloc(const lpa_graph_desc *g, const uint32_t *labels_in, uint32_t *labels_out,
                                          uint32_t cms_threshold, void *stream, uint64_t *changed_out) {
  if (!g || !labels_in || !labels_out || labels_in == labels_out) return LPA_ERR_INVALID_ARG;
  const uint64_t n = g->num_vertices, n_c = g->num_compressed;
  if (n == 0 || n > 0xFFFFFFFEull || n_c > n || !g->vertices) return LPA_ERR_INVALID_ARG;
  if (n_c && (!g->words || !g->offsets || g->num_words < 4)) return LPA_ERR_INVALID_ARG;
  if (n > n_c && !g->small_offset) return LPA_ERR_INVALID_ARG;
  // fixed part of the scratch: counters, degrees, offsets; the rest holds ids
  const size_t off_stats = 0, off_err = 64, off_deg = 256;
  const size_t off_arc = align256(off_deg + size_t(n) * 4);
  const size_t off_ids = align256(off_arc + size_t(n_c + 1) * 8);
  if (off_ids >= kScratchBytes) return LPA_ERR_CAPACITY;  // too many vertices for the scratch
  const size_t ids_cap = (kScratchBytes - off_ids) / 4;

  unsigned char *base = nullptr;
  lpa_status st = scratch_for_current_device(&base);
  if (st != LPA_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  NoAllocArgs a{};
  a.g.words = g->words;
  a.g.offsets = g->offsets;
  a.g.vertices = g->vertices;
  a.g.small_off = g->small_offset;
  a.g.small_nbr = g->small_graph;
  a.g.n = n;
  a.g.n_c = n_c;
  a.stats = reinterpret_cast<unsigned long long *>(base + off_stats);
  a.err = reinterpret_cast<uint32_t *>(base + off_err);
  a.deg = reinterpret_cast<uint32_t *>(base + off_deg);
  a.g.deg = a.deg;
  a.arc_off = reinterpret_cast<uint64_t *>(base + off_arc);
  a.ids = reinterpret_cast<uint32_t *>(base + off_ids);
  a.lab_in = labels_in;
  a.lab_out = labels_out;
  a.cms_thr = cms_threshold;

  a.small_arcs = g->num_small_arcs;

  auto fail = [](cudaError_t e) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? LPA_ERR_OOM : LPA_ERR_CUDA;
  };
  cudaError_t e = cudaSuccess;
  if (n_c) {  // the stream must hold every vertex's bits plus 4 words of padding
    uint64_t total_bits = 0;
    e = cudaMemcpyAsync(&total_bits, g->offsets + n_c, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(e);
    if ((total_bits + 31) / 32 + 4 > g->num_words) return LPA_ERR_INVALID_ARG;
    a.total_bits = total_bits;
  }
  e = cudaMemsetAsync(base, 0, 256, s);  // counters and error word start at zero
  if (e != cudaSuccess) return fail(e);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_na_degrees<<<sms * 8, 256, 0, s>>>(a);
  if (n_c) k_na_scan<<<1, 1024, 0, s>>>(a);
  unsigned long long stats[3] = {0, 0, 0};
  uint32_t err = 0;
  e = cudaMemcpyAsync(stats, a.stats, sizeof(stats), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err, a.err, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(e);
  if (err) return LPA_ERR_BAD_STREAM;
  // limits: the decoded ids must fit the scratch; one warp counts every vertex
  // exactly (degree <= 1023), so a vertex that would need the sketch is refused
  if (stats[2] > ids_cap) return LPA_ERR_CAPACITY;
  if (stats[1] > kV1MaxDeg || (cms_threshold != 0 && stats[1] >= cms_threshold)) return LPA_ERR_CAPACITY;
  if (n_c) k_na_decode<<<sms * 8, 256, 0, s>>>(a);
  e = cudaFuncSetAttribute(k_na_count, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes));
  if (e != cudaSuccess) return fail(e);
  k_na_count<<<sms * 2, kThreads, kSmemBytes, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(e);
  e = cudaMemcpyAsync(stats, a.stats, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err, a.err, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(e);
  if (err == kErrCapacity) return LPA_ERR_CAPACITY;
  if (err) return LPA_ERR_BAD_STREAM;
  if (changed_out) *changed_out = stats[0];
  return LPA_OK;
}
