// Stream compaction that allocates no device memory.
//
// gc_compact keeps the look-back scratch of its single-pass scan (a ticket counter, a
// finish counter, an error word, a sequence tag and one status word per 4096-item chunk)
// in a gc_scan_state, whose device memory the library obtains with cudaMalloc.  Some callers cannot allow that: code that must keep a fixed device-memory
// footprint (a serving process whose memory is carved up in advance, or one that runs next
// to other jobs on a shared GPU), and code that cannot afford the implicit device-wide
// synchronisation that cudaMalloc / cudaFree may cause while other work is in flight.
//
// gc_compact_noalloc runs the same compaction kernel (k_scan in gcut_scan.cu) with its
// scratch in a fixed array compiled into this library, so it never allocates.  That array
// exists once on every GPU that loads the library and stays there until the process exits.
#include <mutex>

#include "gcut_internal.h"

namespace {

constexpr int kChunkItems = 4096;  // items per look-back chunk of k_scan
constexpr int kChunks = GC_COMPACT_NOALLOC_MAX_N / kChunkItems;
static_assert(GC_COMPACT_NOALLOC_MAX_N % kChunkItems == 0, "whole chunks");

// Words 0-1 hold four int32 counters (ticket, done, error, sequence tag); words 2.. hold one
// look-back status per chunk.  (2 + 1024) * 8 bytes = 8208 bytes.
static __device__ __align__(256) unsigned long long g_compact_scratch[2 + kChunks];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

int noalloc_fail(int code, const char* msg) { return gcut::set_last_error(code, msg); }

// Device address of the scratch array on the current device.  The host-side name of a
// __device__ variable is only a stand-in: it must be translated once per device with the
// device current, and the translated address is what the kernel gets.
int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(GC_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(GC_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    // every kernel of the library is loaded here, once per device, so a later call never
    // loads one lazily (inside a stream capture or next to other threads' launches)
    gcut::preload_kernels();
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_compact_scratch);
    if (e != cudaSuccess || !p) return noalloc_fail(GC_ERR_CUDA, "cudaGetSymbolAddress of the compaction scratch failed");
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return GC_OK;
}

}  // namespace

extern "C" int gc_compact_noalloc(const int32_t* flags, int32_t* list, int32_t* length, int n,
                                  void* stream) {
  gcut::set_last_error(GC_OK, "");
  if (n < 0 || !length || (n > 0 && (!flags || !list)))
    return noalloc_fail(GC_ERR_INVALID, "gc_compact_noalloc: bad argument");
  if (n > GC_COMPACT_NOALLOC_MAX_N)
    return noalloc_fail(GC_ERR_INVALID,
                        "gc_compact_noalloc: n exceeds GC_COMPACT_NOALLOC_MAX_N (4194304 items); "
                        "use gc_compact for larger inputs");
  if (n > 0 && flags == list) return noalloc_fail(GC_ERR_INVALID, "gc_compact_noalloc: list must not alias flags");
  void* base = nullptr;
  const int r = scratch_address(&base);
  if (r != GC_OK) return r;
  cudaStream_t s = (cudaStream_t)stream;
  const int nch = gcut::scan_chunks(n);
  // Every call shares the array and finds the previous call's contents there: the counters
  // and the status words this call will read start at zero.
  if (cudaMemsetAsync(base, 0, sizeof(unsigned long long) * (2 + nch), s) != cudaSuccess)
    return noalloc_fail(GC_ERR_CUDA, "gc_compact_noalloc: clearing the scratch failed");
  gcut::ScanState st{};
  int32_t* words = static_cast<int32_t*>(base);
  st.ticket = words;
  st.done = words + 1;
  st.err = words + 2;
  st.seq = reinterpret_cast<uint32_t*>(words + 3);
  st.status = static_cast<unsigned long long*>(base) + 2;
  st.max_chunks = kChunks;
  const int rc = gcut::launch_scan(gcut::GC_SCAN_MODE_COMPACT, flags, nullptr, nullptr, nullptr,
                                   list, length, n, 0, 0, 0, 0, 0, st, s);
  if (rc != GC_OK) return noalloc_fail(rc, "gc_compact_noalloc: kernel launch failed");
  return GC_OK;
}
