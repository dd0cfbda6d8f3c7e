// C ABI of libgcut.so: tile pools, the solve loop and the data-parallel primitives.
//
// The host loop mirrors GraphCut.cut (GraphCut.pyx:348-418) at a coarser grain: where the
// reference enqueues ~30 kernels and blocks on ~5 device->host reads per push iteration,
// a cycle here is `pulses_per_relabel` x {discharge, edge-relabel + list rebuild} and one
// exact global relabel, all enqueued without a host wait; the host reads one int (the
// active-tile count) per cycle and one per few BFS rounds.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "gcut_internal.h"

using namespace gcut;

namespace {

thread_local std::string g_err;

int fail(int code, const char* msg) {
  g_err = msg;
  return code;
}

// Serialises CUDA-graph construction and destruction across the handles of the process.
std::mutex& graph_build_mutex() {
  static std::mutex mu;
  return mu;
}

int cuda_fail(cudaError_t e, const char* where) {
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  return GC_ERR_CUDA;
}

#define CK(call)                                   \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

#define RK(call)                                   \
  do {                                             \
    int _r = (call);                               \
    if (_r != GC_OK) {                             \
      if (g_err.empty()) g_err = #call;            \
      return _r;                                   \
    }                                              \
  } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  return cudaMalloc((void**)p, n * sizeof(T) + 16);
}

struct ScanBuffers {
  ScanState st{};
  cudaError_t alloc(int max_chunks) {
    cudaError_t e;
    if ((e = cudaMalloc((void**)&st.status, sizeof(unsigned long long) * max_chunks))) return e;
    if ((e = cudaMalloc((void**)&st.ticket, 4 * sizeof(int32_t)))) return e;
    st.done = st.ticket + 1;
    st.err = st.ticket + 2;
    st.seq = (uint32_t*)(st.ticket + 3);
    st.max_chunks = max_chunks;
    if ((e = cudaMemset(st.status, 0, sizeof(unsigned long long) * max_chunks))) return e;
    if ((e = cudaMemset(st.ticket, 0, 4 * sizeof(int32_t)))) return e;
    uint32_t one = 1;
    if ((e = cudaMemcpy(st.seq, &one, sizeof(one), cudaMemcpyHostToDevice))) return e;
    // The clears above run on the legacy default stream, which does not order itself
    // with non-blocking streams: finish them before any caller stream uses the state.
    return cudaStreamSynchronize(cudaStreamLegacy);
  }
  void release() {
    if (st.status) cudaFree(st.status);
    if (st.ticket) cudaFree(st.ticket);
    st = ScanState{};
  }
};

}  // namespace

// ------------------------------------------------------------------------------------
// Small pinned host blocks (control words and accumulators copied back after a solve).
// Page-locking host memory costs milliseconds per call, so blocks come from a
// process-wide slab, allocated 64 at a time and recycled; larger requests (batch pools
// with many images) get their own allocation.  Portable: usable from every device.
// ------------------------------------------------------------------------------------
namespace {
constexpr size_t kPinBlock = 1024;
constexpr int kPinPerChunk = 64;
std::mutex g_pin_mu;
std::vector<char*> g_pin_free;

void* pinned_take(size_t bytes) {
  void* p = nullptr;
  if (bytes > kPinBlock) return cudaHostAlloc(&p, bytes, cudaHostAllocPortable) ? nullptr : p;
  std::lock_guard<std::mutex> lock(g_pin_mu);
  if (g_pin_free.empty()) {
    char* c = nullptr;
    if (cudaHostAlloc((void**)&c, kPinBlock * kPinPerChunk, cudaHostAllocPortable)) {
      cudaGetLastError();
      return nullptr;
    }
    for (int i = kPinPerChunk - 1; i >= 0; --i) g_pin_free.push_back(c + (size_t)i * kPinBlock);
  }
  p = g_pin_free.back();
  g_pin_free.pop_back();
  return p;
}

void pinned_give(void* p, size_t bytes) {
  if (!p) return;
  if (bytes > kPinBlock) { cudaFreeHost(p); return; }
  std::lock_guard<std::mutex> lock(g_pin_mu);
  g_pin_free.push_back(static_cast<char*>(p));
}

// Sub-buffers of one device allocation, each 256-byte aligned.  Run once with base ==
// nullptr to size the arena, then with the allocation to place the buffers.
struct Carve {
  char* base = nullptr;
  size_t off = 0;
  template <class T>
  void take(T** out, size_t n) {
    off = (off + 255) & ~(size_t)255;
    *out = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += n * sizeof(T);
  }
};
}  // namespace

// ------------------------------------------------------------------------------------
// Tile pool: one or more images, all solved together.  Every device buffer of the pool
// lives in one allocation (the arena), cleared once at creation.
// ------------------------------------------------------------------------------------
struct Pool {
  int device = 0;
  gc_opts opts{};
  std::vector<ImageDesc> imgs;
  int nt = 0;
  PoolView P{};
  int32_t* tl = nullptr;       // current t-links per pixel (tile planes)
  int32_t* list = nullptr;     // active / frontier tile list
  int32_t* counts = nullptr;   // [0] list length
  ImageAcc* acc = nullptr;     // per image
  ScanBuffers scan;            // look-back state (inside the arena)
  char* arena = nullptr;       // every device buffer of the pool
  size_t arena_bytes = 0;
  bool own_arena = true;       // false: caller-owned memory (gc_create_in)
  cudaEvent_t done_ev = nullptr;   // recorded after every call's work (see track)
  void* pin = nullptr;         // pinned block holding h_count, h_ctl, h_acc
  size_t pin_bytes = 0;
  int32_t* h_count = nullptr;  // pinned
  int32_t* h_ctl = nullptr;    // pinned copy of the control words
  unsigned long long* lab_slot = nullptr;     // device: output buffer of the in-graph labels
  unsigned long long* h_labslot = nullptr;    // pinned: its source word (inside h_count's slot)
  uint8_t* lab_slot_val = nullptr;            // what lab_slot holds
  bool use_graph = true;
  ImageAcc* h_acc = nullptr;   // pinned
  int grid_dis = 0, grid_warps = 0, sms = 1;
  unsigned long long* dsum = nullptr;     // device: sum of |dI|^2 (gc_upload_rgba)
  int32_t* ntab = nullptr;                // device: n-link thresholds (gc_upload_rgba)
  bool uploaded = false, solved = false, edited = false, collect = false;
  bool list_valid = false, bfs_fresh = false;
  // per image: uploaded, solved since its upload or last edit, edited since its last solve
  std::vector<uint8_t> img_up, img_solved, img_edited;
  bool dynamic = false;        // a session pool: images open and close at run time
  // the selection block (ranges, modes, counts) in device memory and its pinned mirror
  char* d_sel = nullptr;
  char* h_sel = nullptr;
  size_t sel_bytes = 0;
  std::vector<int32_t> sel_key, sel_last;   // a selection; the one last copied to the device
  int32_t* trace_words = nullptr;   // device: trace on/off and entry count (P.trace_ctl when on)
  bool graph_warm = false;          // the last graph solve ran the warm variant
  gc_stats stats{};
  // profiling: event pairs around every launch, tiles processed per kernel kind
  bool prof = false;
  unsigned long long* ktiles = nullptr;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, size_t>> ev_used;   // (kind, index of the start event)
  gc_kernel_prof kprof[GC_NKERN]{};

  template <class F>
  int timed(int kind, cudaStream_t s, F&& launch) {
    kprof[kind].launches++;
    if (kind != K_LABELS) stats.launches++;   // the labels are not a kernel of the solve
    if (!prof) return launch();
    size_t i = ev_used.size() * 2;
    while (ev_pool.size() < i + 2) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      ev_pool.push_back(e);
    }
    CK(cudaEventRecord(ev_pool[i], s));
    int r = launch();
    CK(cudaEventRecord(ev_pool[i + 1], s));
    ev_used.push_back({kind, i});
    return r;
  }
  int prof_begin(cudaStream_t s) {
    for (auto& k : kprof) k = gc_kernel_prof{};
    ev_used.clear();
    if (prof) {
      CK(cudaMemsetAsync(ktiles, 0, sizeof(unsigned long long) * GC_NKERN, s));
      P.ktiles = ktiles;
    } else {
      P.ktiles = nullptr;
    }
    return GC_OK;
  }
  int prof_end(cudaStream_t s) {
    if (!prof) return GC_OK;
    CK(cudaStreamSynchronize(s));
    for (auto& u : ev_used) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev_pool[u.second], ev_pool[u.second + 1]));
      kprof[u.first].ms += ms;
    }
    unsigned long long t[GC_NKERN];
    CK(cudaMemcpy(t, ktiles, sizeof(t), cudaMemcpyDeviceToHost));
    for (int k = 0; k < GC_NKERN; ++k) kprof[k].tiles = (int64_t)t[k];
    ev_used.clear();
    return GC_OK;
  }
  // staging for host uploads (allocated on first use) and label reads (in the arena,
  // single-image handles)
  int32_t* stage = nullptr;
  uint8_t* lstage = nullptr;
  int32_t* pts = nullptr;      // stroke points (device, in the arena)

  ~Pool() { release(); }

  // marks the end of the work a call enqueued on s; gc_destroy of a handle in caller-owned
  // memory waits for it before the caller may reuse that memory
  void track(cudaStream_t s) {
    if (done_ev) cudaEventRecord(done_ev, s);
  }

  void release() {
    if (done_ev) {
      if (!own_arena) cudaEventSynchronize(done_ev);
      cudaEventDestroy(done_ev);
      done_ev = nullptr;
    }
    release_graphs();
    if (stage) cudaFree(stage);   // host-upload staging, allocated on first use
    if (arena && own_arena) cudaFree(arena);
    pinned_give(pin, pin_bytes);
    for (auto e : ev_pool) cudaEventDestroy(e);
    ev_pool.clear();
    arena = nullptr;
    pin = nullptr;
    ktiles = nullptr;
    scan.st = ScanState{};
    P = PoolView{};
    tl = list = counts = stage = pts = nullptr;
    acc = nullptr; lstage = nullptr; h_count = nullptr; h_ctl = nullptr; h_acc = nullptr;
    dsum = nullptr; ntab = nullptr; d_sel = nullptr; h_sel = nullptr;
    lab_slot = nullptr; h_labslot = nullptr; lab_slot_val = nullptr;
    trace_words = nullptr;
  }

  // places every device buffer of the pool (see Carve)
  void layout(Carve& c) {
    const size_t px = (size_t)nt * GC_TILE_PX;
    int32_t** planes[] = {&P.exc, &P.hgt, &P.cap[0], &P.cap[1], &P.cap[2], &P.cap[3], &tl};
    for (auto** p : planes) c.take(p, px);
    c.take(&P.nbr, nt);
    c.take(&P.mcan, (size_t)nt * 128);
    c.take(&P.msink, (size_t)nt * 32);
    c.take(&P.mexc, (size_t)nt * 32);
    c.take(&P.mreach, (size_t)nt * 32);
    int32_t** small[] = {&P.touched, &P.act_int, &P.mark[0], &P.mark[1], &P.tact, &P.img_of,
                         &P.queue[0], &P.queue[1], &P.inq[0], &P.inq[1], &P.mdirty};
    for (auto** p : small) c.take(p, nt);
    c.take(&P.qcount, 2);
    c.take(&P.fq[0], nt);
    c.take(&P.fq[1], nt);
    c.take(&P.fcount, 2);
    c.take(&P.img_live, imgs.size());
    c.take(&P.img_hit, imgs.size());
    c.take(&P.img_mode, imgs.size());
    c.take(&d_sel, sel_bytes);
    if (d_sel) {
      P.nsel = reinterpret_cast<int32_t*>(d_sel);
      P.sel = reinterpret_cast<int4*>(d_sel + 16);
      P.sel_mode = reinterpret_cast<int32_t*>(P.sel + imgs.size());
    }
    c.take(&P.tpos, nt);
    c.take(&P.rcnt, 2);
    c.take(&P.ctl, CTL_N);
    c.take(&acc, imgs.size());
    c.take(&ktiles, GC_NKERN);
    c.take(&P.trace, 2 * GC_TRACE_MAX);
    c.take(&P.trace_ctl, 2);
    // look-back slots: the scan uses one per 4096 items, the list rebuild one per 1024 tiles
    const int chunks = scan_chunks(nt) > nt / 1024 + 1 ? scan_chunks(nt) : nt / 1024 + 1;
    c.take(&scan.st.status, chunks);
    c.take(&scan.st.ticket, 4);
    scan.st.max_chunks = chunks;
    c.take(&pts, 2 * 1024);
    c.take(&dsum, 1);
    c.take(&ntab, GC_NLINK_LEVELS);
    c.take(&lab_slot, 1);
    if (imgs.size() == 1) c.take(&lstage, (size_t)imgs[0].W * imgs[0].H);
  }

  // image descriptors and the arena size (host only, no CUDA calls)
  int describe(int n, const int* W, const int* H) {
    if (n <= 0 || !W || !H) return fail(GC_ERR_INVALID, "no images");
    nt = 0;
    imgs.clear();
    for (int i = 0; i < n; ++i) {
      if (W[i] <= 0 || H[i] <= 0 || W[i] > (1 << 16) || H[i] > (1 << 16))
        return fail(GC_ERR_INVALID, "image size out of range");
      ImageDesc d{W[i], H[i], (W[i] + 31) / 32, (H[i] + 31) / 32, nt};
      long long tiles = (long long)d.tw * d.th;
      if (nt + tiles > (1 << 26)) return fail(GC_ERR_INVALID, "pool too large");
      nt += (int)tiles;
      imgs.push_back(d);
    }
    return finish_describe();
  }

  // a session pool: room for max_tiles tiles and max_images images, none open yet
  int describe_dynamic(int max_tiles, int max_images) {
    if (max_tiles < 1 || max_tiles > (1 << 26) || max_images < 1 || max_images > (1 << 16))
      return fail(GC_ERR_INVALID, "session pool size out of range");
    nt = max_tiles;
    imgs.assign(max_images, ImageDesc{0, 0, 0, 0, 0});
    dynamic = true;
    return finish_describe();
  }

  int finish_describe() {
    P.nt = nt;
    P.nimg = (int)imgs.size();
    // selection block: counts (16 bytes), one int4 range and one mode per image
    sel_bytes = 16 + imgs.size() * (sizeof(int4) + sizeof(int32_t));
    Carve sizing;
    layout(sizing);
    arena_bytes = sizing.off + 256;   // slack after the last buffer
    return GC_OK;
  }

  // ext: caller-owned device memory of ext_bytes (256-byte aligned), or null to allocate
  int create(int n, const int* W, const int* H, const gc_opts* o, void* ext = nullptr,
             size_t ext_bytes = 0) {
    opts = *o;
    RK(describe(n, W, H));
    return create_common(ext, ext_bytes);
  }

  // a session pool of max_tiles tiles and max_images image slots
  int create_dynamic(int max_tiles, int max_images, const gc_opts* o, void* ext = nullptr,
                     size_t ext_bytes = 0) {
    opts = *o;
    RK(describe_dynamic(max_tiles, max_images));
    return create_common(ext, ext_bytes);
  }

  int create_common(void* ext, size_t ext_bytes) {
    device = opts.device;
    use_graph = opts.use_graph != 0;
    img_up.assign(imgs.size(), 0);
    img_solved.assign(imgs.size(), 0);
    img_edited.assign(imgs.size(), 0);
    if (ext) {
      if ((reinterpret_cast<uintptr_t>(ext) & 255) != 0) return fail(GC_ERR_INVALID, "arena not 256-byte aligned");
      if (ext_bytes < arena_bytes) return fail(GC_ERR_INVALID, "arena smaller than gc_arena_bytes");
    }
    CK(cudaSetDevice(device));
    cudaError_t e = cudaSuccess;
    if (ext) {
      arena = static_cast<char*>(ext);
      own_arena = false;
    } else {
      e = cudaMalloc((void**)&arena, arena_bytes);
      if (e == cudaErrorMemoryAllocation) { cudaGetLastError(); arena = nullptr; release(); return fail(GC_ERR_OOM, "device allocation failed"); }
      if (e) { arena = nullptr; release(); return cuda_fail(e, "pool allocation"); }
    }
    e = cudaEventCreateWithFlags(&done_ev, cudaEventDisableTiming);
    if (e) { done_ev = nullptr; release(); return cuda_fail(e, "event"); }
    Carve place{arena, 0};
    layout(place);
    // tracing starts off: the kernels see a null trace_ctl and skip the mark without a load
    trace_words = P.trace_ctl;
    P.trace_ctl = nullptr;
    list = P.queue[0];
    counts = P.qcount;
    scan.st.done = scan.st.ticket + 1;
    scan.st.err = scan.st.ticket + 2;
    scan.st.seq = (uint32_t*)(scan.st.ticket + 3);
    // the per-image sums follow the control words in the arena (256 bytes of them) and in
    // the pinned block, so one copy brings both back
    static_assert(sizeof(int32_t) * CTL_N == 256, "control words fill one 256-byte slot");
    if (reinterpret_cast<char*>(acc) != reinterpret_cast<char*>(P.ctl) + 256) {
      release();
      return fail(GC_ERR_INTERNAL, "arena layout");
    }
    // pinned: counts, control words, per-image sums, then the selection mirror
    const size_t acc_end = (512 + imgs.size() * sizeof(ImageAcc) + 15) & ~(size_t)15;
    pin_bytes = acc_end + sel_bytes;
    pin = pinned_take(pin_bytes);
    if (!pin) { release(); return fail(GC_ERR_OOM, "pinned host allocation failed"); }
    h_count = static_cast<int32_t*>(pin);
    h_labslot = reinterpret_cast<unsigned long long*>(static_cast<char*>(pin) + 128);
    h_ctl = reinterpret_cast<int32_t*>(static_cast<char*>(pin) + 256);
    h_acc = reinterpret_cast<ImageAcc*>(static_cast<char*>(pin) + 512);
    {   // the kernel that ends a graph solve writes the results here itself (no copy node)
      void* dptr = nullptr;
      if (cudaHostGetDevicePointer(&dptr, h_ctl, 0) == cudaSuccess && dptr)
        P.host_out = static_cast<int32_t*>(dptr);
      else
        cudaGetLastError();
    }
    h_sel = static_cast<char*>(pin) + acc_end;
    // every buffer starts at zero; the look-back tag starts at 1
    CK(cudaMemset(arena, 0, arena_bytes));
    if (!dynamic) {   // a session pool sets its tiles up as images open
      std::vector<int4> nb(nt);
      for (const auto& d : imgs)
        for (int ty = 0; ty < d.th; ++ty)
          for (int tx = 0; tx < d.tw; ++tx) {
            int t = d.tile0 + ty * d.tw + tx;
            nb[t] = make_int4(ty > 0 ? t - d.tw : -1, ty < d.th - 1 ? t + d.tw : -1,
                              tx > 0 ? t - 1 : -1, tx < d.tw - 1 ? t + 1 : -1);
          }
      CK(cudaMemcpy(P.nbr, nb.data(), sizeof(int4) * nt, cudaMemcpyHostToDevice));
    }
    const uint32_t one = 1;
    CK(cudaMemcpy(scan.st.seq, &one, sizeof(one), cudaMemcpyHostToDevice));
    // These clears were issued on the legacy default stream, which non-blocking streams
    // (torch's, for one) do not wait for: an upload on such a stream could otherwise run
    // first and have its masks, tile sums and flow accumulator zeroed afterwards.
    CK(cudaStreamSynchronize(cudaStreamLegacy));
    grid_dis = occupancy_discharge(device);
    grid_warps = occupancy_warps(device);
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    return GC_OK;
  }

  int upload(int i, const int32_t* up, const int32_t* down, const int32_t* left,
             const int32_t* right, const int32_t* excess, cudaStream_t s) {
    if (i < 0 || i >= (int)imgs.size()) return fail(GC_ERR_INVALID, "image index");
    if (!up || !down || !left || !right || !excess) return fail(GC_ERR_INVALID, "null plane");
    CK(cudaSetDevice(device));
    CK(cudaMemsetAsync(acc + i, 0, sizeof(ImageAcc), s));
    P.ktiles = nullptr;
    RK(timed(K_UPLOAD, s, [&] { return launch_upload(P, imgs[i], i, up, down, left, right, excess, tl, acc, s); }));
    uploaded_image(i);
    return GC_OK;
  }

  // Capacities from an RGBA image (n-links) and int32 t-links, all on the device with no
  // host wait.  lambda == 0: the exp weighting, whose scale comes from the mean |dI|^2 over
  // all 4-neighbour pairs (k_dsum sums it exactly, k_nlink_table turns it into the weight
  // thresholds); lambda > 0: the reference's weighting with that LAMBDA.
  int upload_rgba(int i, const uint32_t* rgba, const int32_t* excess, int lambda, cudaStream_t s) {
    if (i < 0 || i >= (int)imgs.size()) return fail(GC_ERR_INVALID, "image index");
    if (!rgba || !excess) return fail(GC_ERR_INVALID, "null plane");
    if (lambda < 0 || lambda > GC_NLINK_MAX_LAMBDA) return fail(GC_ERR_INVALID, "lambda out of range");
    CK(cudaSetDevice(device));
    const ImageDesc& im = imgs[i];
    if (lambda == 0) {
      const long long npairs = (long long)(im.H - 1) * im.W + (long long)im.H * (im.W - 1);
      CK(cudaMemsetAsync(dsum, 0, sizeof(unsigned long long), s));
      RK(launch_dsum(rgba, im.W, im.H, dsum, sms, s));
      RK(launch_nlink_table(dsum, npairs, ntab, s));
    }
    CK(cudaMemsetAsync(acc + i, 0, sizeof(ImageAcc), s));
    P.ktiles = nullptr;
    RK(timed(K_UPLOAD, s, [&] {
      return launch_upload_rgba(P, im, i, rgba, excess, lambda ? nullptr : ntab, lambda, tl, acc, s);
    }));
    uploaded_image(i);
    return GC_OK;
  }

  void uploaded_image(int i) {
    img_up[i] = 1;
    img_solved[i] = 0;
    img_edited[i] = 0;
    uploaded = true;
    solved = false;
    edited = false;
    list_valid = false;
    bfs_fresh = false;
  }

  void edited_image(int i) {
    img_edited[i] = 1;
    img_solved[i] = 0;
    edited = true;
    bfs_fresh = false;
  }

  // Writes the selection of a solve (the listed images, in order) to the pinned mirror and
  // queues its copy to the device.  An image is fresh (mode 1: trivial labelling, no flood
  // before its first pulses) right after its upload, else it continues from its previous
  // flow (mode 2); initial_relabel makes every image mode 2.  *any_warm: some image is mode 2.
  // Repeated solves of the same images (every solve of a one-image handle) find the
  // selection already on the device and skip both copies.
  int set_selection(const int* idx, int n, bool* any_warm, cudaStream_t s) {
    // n, selected tiles, then per range: first tile, tiles, first selected index, image, mode
    sel_key.assign(2 + 5 * (size_t)n, 0);
    long long start = 0;
    bool warm = false;
    for (int k = 0; k < n; ++k) {
      const int i = idx[k];
      const ImageDesc& im = imgs[i];
      const int tiles = im.tw * im.th;
      int32_t* e = &sel_key[2 + 5 * (size_t)k];
      e[0] = im.tile0;
      e[1] = tiles;
      e[2] = (int)start;
      e[3] = i;
      e[4] = (opts.initial_relabel || img_solved[i] || img_edited[i]) ? 2 : 1;
      warm |= e[4] == 2;
      start += tiles;
    }
    if (start > nt) return fail(GC_ERR_INTERNAL, "selection larger than the pool");
    sel_key[0] = n;
    sel_key[1] = (int)start;
    *any_warm = warm;
    if (sel_key == sel_last) return GC_OK;
    // the previous copy out of the pinned mirror finished with the previous (synchronous) solve
    int32_t* cnt = reinterpret_cast<int32_t*>(h_sel);
    int4* rng = reinterpret_cast<int4*>(h_sel + 16);
    int32_t* mode = reinterpret_cast<int32_t*>(rng + imgs.size());
    cnt[0] = n;
    cnt[1] = (int)start;
    for (int k = 0; k < n; ++k) {
      const int32_t* e = &sel_key[2 + 5 * (size_t)k];
      rng[k] = make_int4(e[0], e[1], e[2], e[3]);
      mode[k] = e[4];
    }
    // one copy: counts, the n ranges, then (at their fixed place) the modes
    sel_last.clear();   // unknown until both copies are queued
    CK(cudaMemcpyAsync(d_sel, h_sel, 16 + sizeof(int4) * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(P.sel_mode, mode, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
    sel_last.swap(sel_key);
    return GC_OK;
  }

  int select_all(bool* any_warm, cudaStream_t s) {
    std::vector<int> all(imgs.size());
    for (size_t i = 0; i < imgs.size(); ++i) all[i] = (int)i;
    return set_selection(all.data(), (int)all.size(), any_warm, s);
  }

  // exact BFS distances to the sink pixels (global relabel); sets tact.  h: condition
  // handle when captured into a graph (0: host-driven rounds)
  int global_relabel(cudaStream_t s, int first = 1) {
    RK(timed(K_MASKS, s, [&] { return launch_masks(P, grid_warps, s); }));
    RK(timed(K_BFS_FIRST, s, [&] { return launch_bfs_round(P, first, 0, grid_warps, s); }));
    return frontier_rounds(s, /*flood=*/false);
  }

  // host-driven rounds over the marked tiles until a round finds none; the host reads
  // the control words once per batch of rounds
  int frontier_rounds(cudaStream_t s, bool flood, int abort_hit = 0) {
    int batch = 4;
    while (true) {
      for (int k = 0; k < batch; ++k) {
        if (flood) RK(timed(K_FLOOD, s, [&] { return launch_flood_round(P, 0, abort_hit, 0, acc, grid_warps, s); }));
        else RK(timed(K_BFS, s, [&] { return launch_bfs_round(P, 0, 0, grid_warps, s); }));
      }
      RK(read_ctl(s));
      if (h_ctl[CTL_ERR] == 1) return fail(GC_ERR_NOT_CONVERGED, "BFS round cap reached");
      if (h_ctl[CTL_LASTCNT] == 0) break;
      batch = batch < 32 ? batch * 2 : 32;
    }
    return GC_OK;
  }

  int read_ctl(cudaStream_t s) {
    CK(cudaMemcpyAsync(h_ctl, P.ctl, sizeof(int32_t) * CTL_N, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return GC_OK;
  }

  int compact(const int32_t* flags, int32_t* clear, cudaStream_t s) {
    return timed(K_COMPACT, s, [&] {
      return launch_scan(GC_SCAN_MODE_COMPACT, flags, nullptr, clear, nullptr, list, counts, nt,
                         0, 0, 0, 0, 0, scan.st, s);
    });
  }

  int read_count(cudaStream_t s, int* n) {
    CK(cudaMemcpyAsync(h_count, counts, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *n = h_count[0];
    return GC_OK;
  }

  int check_device_error(cudaStream_t s) {
    int32_t err = 0;
    CK(cudaMemcpyAsync(&h_count[1], scan.st.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    err = h_count[1];
    if (err) {
      cudaMemsetAsync(scan.st.err, 0, sizeof(int32_t), s);
      return fail(GC_ERR_INTERNAL, "a bounded device-side wait gave up");
    }
    return GC_OK;
  }

  // Solves every image of a fixed pool.
  // Work queued right behind a solve, before the host waits for it (the labels of
  // gc_solve_labels): it needs only the solve's device results, so it follows the solve
  // without a host round trip in between.
  using After = std::function<int(cudaStream_t)>;

  int solve(cudaStream_t s, const After* after = nullptr) {
    std::vector<int> all(imgs.size());
    for (size_t i = 0; i < imgs.size(); ++i) all[i] = (int)i;
    return solve_images(all.data(), (int)all.size(), s, after);
  }

  // Solves the listed images together (distinct, uploaded); the pool's other images keep
  // their state and results.
  int solve_images(const int* idx, int n, cudaStream_t s, const After* after = nullptr,
                   int lmode = 0, uint8_t* lbuf = nullptr) {
    if (n < 1 || !idx) return fail(GC_ERR_INVALID, "no images to solve");
    std::vector<uint8_t> seen(imgs.size(), 0);
    for (int k = 0; k < n; ++k) {
      const int i = idx[k];
      if (i < 0 || i >= (int)imgs.size() || seen[i]) return fail(GC_ERR_INVALID, "bad image list");
      if (!img_up[i]) return fail(GC_ERR_STATE, "solve before upload");
      seen[i] = 1;
    }
    CK(cudaSetDevice(device));
    stats = gc_stats{};
    bool warm = false;
    RK(set_selection(idx, n, &warm, s));
    const bool host = prof || collect || !use_graph;
    int r = host ? solve_host(s, warm) : solve_graph(s, warm, after, lmode, lbuf);
    if (r) return r;
    if (host && after) {   // the host-driven solve has finished: queue the work and wait
      RK((*after)(s));
      CK(cudaStreamSynchronize(s));
    }
    RK(finish_check(s, idx, n, /*err_in_ctl=*/true));
    for (int k = 0; k < n; ++k) {
      img_solved[idx[k]] = 1;
      img_edited[idx[k]] = 0;
    }
    return GC_OK;
  }

  // Host-driven solve (profiling, stats collection): same kernels, host decides the loops.
  //
  // The solve (both paths) over the selected images: the images that continue from a
  // previous flow (warm) are flooded first, and those whose flood reaches a sink pixel get a
  // global relabel; freshly uploaded images start from the trivial labelling.  Then, while
  // tiles are active: pulses of discharge, a mask rebuild, the flood of the live images with
  // its termination check, and for the images that are not solved a global relabel and the
  // next active-tile list.  The last flood of every image is its canonical cut, so no
  // separate flood phase follows.
  int solve_host(cudaStream_t s, bool warm) {
    RK(prof_begin(s));
    RK(launch_ctl_begin(P, opts.max_bfs_rounds, opts.max_cycles, acc, s));
    int n = 0;
    if (warm) {
      RK(flood_phase(s, /*mode=*/3));   // its first round rebuilds the masks of edited tiles
      RK(timed(K_COMPACT, s, [&] { return launch_flood_check(P, 1, 0, 0, s); }));
      RK(read_ctl(s));
      if (h_ctl[CTL_LEFT] > 0) RK(bfs_phase(s));
    }
    RK(timed(K_COMPACT, s, [&] { return launch_active_list(P, scan.st, list, counts, 0, 0, 2, 0, acc, 2 * sms, s); }));
    RK(read_count(s, &n));
    for (int cycle = 0; n > 0; ++cycle) {
      if (cycle >= opts.max_cycles) return fail(GC_ERR_NOT_CONVERGED, "cycle cap reached before the cut was final");
      stats.cycles++;
      for (int p = 0; p < opts.pulses_per_relabel; ++p) {
        if (collect) {
          RK(read_ctl(s));
          CK(cudaMemcpy(h_count, P.qcount, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost));
          stats.tiles_discharged += h_count[h_ctl[CTL_PULSE] & 1];
        }
        RK(timed(K_DISCHARGE, s, [&] { return launch_discharge(P, opts.discharge_iters, grid_dis, s); }));
        stats.pulses++;
      }
      RK(flood_phase(s, /*mode=*/2));   // its first round rebuilds the masks of changed tiles
      RK(timed(K_COMPACT, s, [&] { return launch_flood_check(P, 0, 0, 0, s); }));
      RK(read_ctl(s));
      n = 0;
      if (h_ctl[CTL_LEFT] > 0) {
        RK(bfs_phase(s));
        RK(timed(K_COMPACT, s, [&] { return launch_active_list(P, scan.st, list, counts, 1, 1, 1, 0, acc, 2 * sms, s); }));
        RK(read_count(s, &n));
      }
    }
    CK(cudaMemcpyAsync(h_acc, acc, sizeof(ImageAcc) * imgs.size(), cudaMemcpyDeviceToHost, s));
    RK(read_ctl(s));
    RK(prof_end(s));
    return GC_OK;
  }

  // global relabel of the live images: first round, then frontier rounds until none is left
  int bfs_phase(cudaStream_t s) {
    RK(timed(K_BFS_FIRST, s, [&] { return launch_bfs_round(P, 2, 0, grid_warps, s); }));
    return frontier_rounds(s, /*flood=*/false);
  }

  // flood of every image (mode 1) or of the live images (mode 2), to its end
  int flood_phase(cudaStream_t s, int mode) {
    RK(timed(K_FLOOD_FIRST, s, [&] { return launch_flood_round(P, mode, 1, 0, acc, grid_warps, s); }));
    return frontier_rounds(s, /*flood=*/true, /*abort_hit=*/1);
  }

  // ---- CUDA graph solve: the whole solve is one graph launch.  The loops are WHILE nodes
  // whose conditions are set on the device (frontier rounds by their last CTA, cycles by
  // k_ctl_cycle), so the host waits once, at the end.
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};   // [relabel_first]
  cudaGraph_t graph[2] = {nullptr, nullptr};
  // Solve graphs that end with the labels of a pool's one image (gc_solve_labels), [warm]
  // [packed]: the labels start right after the solve's last kernel instead of after the
  // graph has left its loop nodes and ended.  Their kernels read the output buffer from a
  // device word (lab_slot), which is set from the pinned h_labslot when the caller's buffer
  // changes, so the graphs stay as built.
  cudaGraphExec_t lexec[2][2] = {};
  cudaGraph_t lgraph[2][2] = {};
  int bl_mode = 0;   // during a build: the labels the graph ends with (0 none, 1 bytes, 2 packed)

  template <class F>
  int capture(cudaGraph_t g, std::vector<cudaGraphNode_t>& leaves, F&& fn) {
    CK(cudaStreamBeginCaptureToGraph(cap_stream, g, leaves.empty() ? nullptr : leaves.data(),
                                     nullptr, leaves.size(), cudaStreamCaptureModeThreadLocal));
    const int r = fn(cap_stream);
    cudaStreamCaptureStatus st;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    const cudaError_t e1 = cudaStreamGetCaptureInfo(cap_stream, &st, nullptr, nullptr, &deps, &nd);
    std::vector<cudaGraphNode_t> nl(deps, deps + (e1 == cudaSuccess ? nd : 0));
    cudaGraph_t out = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(cap_stream, &out);
    if (r) return r;
    if (e1) return cuda_fail(e1, "cudaStreamGetCaptureInfo");
    if (e2) return cuda_fail(e2, "cudaStreamEndCapture");
    if (!nl.empty()) leaves = nl;
    return GC_OK;
  }

  int add_cond(cudaGraph_t g, std::vector<cudaGraphNode_t>& leaves,
               cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, cudaGraph_t* body) {
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, leaves.empty() ? nullptr : leaves.data(), leaves.size(), &p));
    *body = p.conditional.phGraph_out[0];
    leaves.assign(1, node);
    return GC_OK;
  }
  int add_while(cudaGraph_t g, std::vector<cudaGraphNode_t>& leaves,
                cudaGraphConditionalHandle h, cudaGraph_t* body) {
    return add_cond(g, leaves, h, cudaGraphCondTypeWhile, body);
  }
  int add_if(cudaGraph_t g, std::vector<cudaGraphNode_t>& leaves,
             cudaGraphConditionalHandle h, cudaGraph_t* body) {
    return add_cond(g, leaves, h, cudaGraphCondTypeIf, body);
  }

  // The kernels read a conditional handle of value 0 as "not launched from a graph" (the
  // host-driven loop passes 0).  The runtime does not promise that 0 is never a valid handle,
  // so a handle that comes out as 0 is left unused in the graph and another one is created.
  int cond_handle(cudaGraphConditionalHandle* h, cudaGraph_t g) {
    for (int tries = 0; tries < 4; ++tries) {
      CK(cudaGraphConditionalHandleCreate(h, g, 0, 0));
      if (*h != 0) return GC_OK;
    }
    return fail(GC_ERR_INTERNAL, "cudaGraphConditionalHandleCreate gave only handle 0");
  }

  // A labels node of the pool's one image, into the buffer held in lab_slot.  first: the
  // node after the first cycle's flood (it writes only when that cycle ended the solve).
  int capture_labels(cudaGraph_t g, std::vector<cudaGraphNode_t>& L, int first) {
    return capture(g, L, [&](cudaStream_t cs) {
      return bl_mode == 2 ? launch_labels_packed(P, imgs[0], nullptr, cs, first, lab_slot, 4 * sms)
                          : launch_labels_out(P, imgs[0], nullptr, cs, first, lab_slot, 4 * sms);
    });
  }

  // Appends to g: flood first round (mode) + WHILE(frontier rounds) + the check, then
  // IF(images left) { global relabel [+ the next cycle's active list (bump = count_cycle =
  // 1)] }.  all: the warm prologue's flood (the solve does not end at its check; the first
  // active list that follows decides).  first_cycle: the first cycle of a fresh solve, which
  // runs ahead of the solve loop: the loop and its handle sit inside the IF body, after the
  // list, so a solve that ends after one cycle never enters or leaves a loop node (each
  // conditional node a solve passes costs several microseconds of device time).
  int graph_cycle_tail(cudaGraph_t g, std::vector<cudaGraphNode_t>& L, int mode, int all,
                       int bump, cudaGraphConditionalHandle hmain, bool first_cycle = false) {
    cudaGraphConditionalHandle hf, hbfs, hb;
    RK(cond_handle(&hf, g));
    RK(cond_handle(&hbfs, g));
    // the round that ends the flood runs the flood check (retires the solved images, sets
    // the IF condition below and, when none is left, ends the solve loop and publishes)
    const cudaGraphConditionalHandle hm = all ? 0 : hmain;
    const int publish = all ? 0 : 1;
    RK(capture(g, L, [&](cudaStream_t cs) {
      return launch_flood_round(P, mode, 1, hf, acc, grid_warps, cs, all, hbfs, hm, publish);
    }));
    cudaGraph_t bf;
    RK(add_while(g, L, hf, &bf));
    {
      std::vector<cudaGraphNode_t> Lf;
      RK(capture(bf, Lf, [&](cudaStream_t cs) {
        return launch_flood_round(P, 0, 1, hf, acc, grid_warps, cs, all, hbfs, hm, publish);
      }));
    }
    // a graph that ends with the labels: they follow the first cycle's flood on a branch of
    // their own (writing only when its check ended the solve), beside the IF node
    std::vector<cudaGraphNode_t> Lq = L;
    if (first_cycle && bl_mode) RK(capture_labels(g, Lq, 1));
    cudaGraph_t bi;
    RK(add_if(g, L, hbfs, &bi));
    if (first_cycle && bl_mode) L.push_back(Lq[0]);   // what follows waits for both
    std::vector<cudaGraphNode_t> Li;
    RK(cond_handle(&hb, bi));
    RK(capture(bi, Li, [&](cudaStream_t cs) { return launch_bfs_round(P, 2, hb, grid_warps, cs); }));
    cudaGraph_t bb;
    RK(add_while(bi, Li, hb, &bb));
    {
      std::vector<cudaGraphNode_t> Lb;
      RK(capture(bb, Lb, [&](cudaStream_t cs) { return launch_bfs_round(P, 0, hb, grid_warps, cs); }));
    }
    if (!bump) return GC_OK;   // the first list of a solve follows the IF node
    cudaGraphConditionalHandle hl = hmain;
    if (first_cycle) RK(cond_handle(&hl, bi));   // the solve loop's handle, in the IF body
    RK(capture(bi, Li, [&](cudaStream_t cs) {
      return launch_active_list(P, scan.st, list, counts, 1, 1, 1, hl, acc, 2 * sms, cs);
    }));
    if (!first_cycle) return GC_OK;
    RK(add_solve_loop(bi, Li, hl));
    // the labels of a solve that went on past its first cycle, after its loop
    return bl_mode ? capture_labels(bi, Li, 0) : GC_OK;
  }

  // WHILE(hloop) { pulses x discharge, then the cycle's flood, check and relabel, and the
  // next active list, which sets hloop }
  int add_solve_loop(cudaGraph_t g, std::vector<cudaGraphNode_t>& L,
                     cudaGraphConditionalHandle hloop) {
    cudaGraph_t bm;
    RK(add_while(g, L, hloop, &bm));
    std::vector<cudaGraphNode_t> Lm;
    RK(capture(bm, Lm, [&](cudaStream_t cs) { return launch_pulses(cs); }));
    return graph_cycle_tail(bm, Lm, /*mode=*/2, /*all=*/0, /*bump=*/1, hloop);
  }

  int launch_pulses(cudaStream_t s) {
    for (int p = 0; p < opts.pulses_per_relabel; ++p)
      RK(launch_discharge(P, opts.discharge_iters, grid_dis, s));
    return GC_OK;
  }

  // Builds the solve graph of a variant into *gout / *eout; with bl_mode set, the graph
  // ends with the labels of the pool's one image.
  int build_graph(int variant, cudaGraph_t* gout, cudaGraphExec_t* eout) {
    // One graph construction at a time in the process (building, instantiating and
    // destroying graphs with nested conditional nodes from several threads at once was the
    // suspected trigger of an intermittent fault under concurrent serving).
    std::lock_guard<std::mutex> lock(graph_build_mutex());
    if (!cap_stream) CK(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    *gout = g;
    std::vector<cudaGraphNode_t> L;
    if (!variant) {
      // fresh images only: the prologue and the first active list (one CTA for a small
      // pool), then the first cycle unrolled, with the solve loop inside its IF node.  The
      // list sets no condition: an empty one leaves nothing for the pulses, the flood finds
      // no live image and its check ends the solve.
      if (nt <= begin_list_max_tiles()) {
        RK(capture(g, L, [&](cudaStream_t cs) {
          return launch_begin_list(P, opts.max_bfs_rounds, opts.max_cycles, acc, list, counts, 0, cs);
        }));
      } else {
        RK(capture(g, L, [&](cudaStream_t cs) {
          RK(launch_ctl_begin(P, opts.max_bfs_rounds, opts.max_cycles, acc, cs));
          return launch_active_list(P, scan.st, list, counts, 0, 0, 2, 0, acc, 2 * sms, cs);
        }));
      }
      RK(capture(g, L, [&](cudaStream_t cs) { return launch_pulses(cs); }));
      RK(graph_cycle_tail(g, L, /*mode=*/2, /*all=*/0, /*bump=*/1, 0, /*first_cycle=*/true));
    } else {
      cudaGraphConditionalHandle hmain;
      RK(cond_handle(&hmain, g));
      RK(capture(g, L, [&](cudaStream_t cs) { return launch_ctl_begin(P, opts.max_bfs_rounds, opts.max_cycles, acc, cs); }));
      // images that continue from a previous flow: flood them; relabel the ones not solved
      RK(graph_cycle_tail(g, L, /*mode=*/3, /*all=*/1, /*bump=*/0, hmain));
      RK(capture(g, L, [&](cudaStream_t cs) {   // the first active list (fresh and live images)
        return launch_active_list(P, scan.st, list, counts, 0, 0, 2, hmain, acc, 2 * sms, cs);
      }));
      RK(add_solve_loop(g, L, hmain));
    }
    if (bl_mode && variant) RK(capture_labels(g, L, 0));   // (fresh: inside the IF node)
    if (!P.host_out) {   // else the kernel that ends the solve wrote them already
      RK(capture(g, L, [&](cudaStream_t cs) {
        // control words and per-image sums are adjacent on both sides: one copy
        CK(cudaMemcpyAsync(h_ctl, P.ctl, sizeof(int32_t) * CTL_N + sizeof(ImageAcc) * imgs.size(),
                           cudaMemcpyDeviceToHost, cs));
        return GC_OK;
      }));
    }
    CK(cudaGraphInstantiate(eout, g, 0));
    // upload the executable graph here, under the construction lock, rather than implicitly
    // at its first launch next to other threads' graph work
    CK(cudaGraphUpload(*eout, cap_stream));
    CK(cudaStreamSynchronize(cap_stream));
    return GC_OK;
  }


  // variant 1: some selected image continues from a previous flow (the graph floods first).
  // lmode 1 / 2: the graph that ends with the labels (bytes / packed) of the pool's one
  // image, into lbuf.
  int solve_graph(cudaStream_t s, bool warm, const After* after = nullptr, int lmode = 0,
                  uint8_t* lbuf = nullptr) {
    const int v = warm ? 1 : 0;
    cudaGraphExec_t* ex = lmode ? &lexec[v][lmode - 1] : &gexec[v];
    cudaGraph_t* gr = lmode ? &lgraph[v][lmode - 1] : &graph[v];
    if (!*ex) {
      bl_mode = lmode;
      const int r = build_graph(v, gr, ex);
      bl_mode = 0;
      if (r) {
        if (*ex) { cudaGraphExecDestroy(*ex); *ex = nullptr; }
        if (*gr) { cudaGraphDestroy(*gr); *gr = nullptr; }
        return r;
      }
    }
    if (lmode && lab_slot_val != lbuf) {   // the labels kernels read their buffer from here
      *h_labslot = (unsigned long long)(uintptr_t)lbuf;
      CK(cudaMemcpyAsync(lab_slot, h_labslot, sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
      lab_slot_val = lbuf;
    }
    P.ktiles = nullptr;
    graph_warm = warm;
    CK(cudaGraphLaunch(*ex, s));
    if (after) RK((*after)(s));
    CK(cudaStreamSynchronize(s));
    stats.launches = -1;  // inside the graph; see gc_stats
    return GC_OK;
  }

  void release_graphs() {
    std::lock_guard<std::mutex> lock(graph_build_mutex());
    for (int v = 0; v < 2; ++v) {
      if (gexec[v]) cudaGraphExecDestroy(gexec[v]);
      if (graph[v]) cudaGraphDestroy(graph[v]);
      gexec[v] = nullptr;
      graph[v] = nullptr;
      for (int m = 0; m < 2; ++m) {
        if (lexec[v][m]) cudaGraphExecDestroy(lexec[v][m]);
        if (lgraph[v][m]) cudaGraphDestroy(lgraph[v][m]);
        lexec[v][m] = nullptr;
        lgraph[v][m] = nullptr;
      }
    }
    if (cap_stream) cudaStreamDestroy(cap_stream);
    cap_stream = nullptr;
  }

  // errors and results common to both paths (h_acc / h_ctl are filled and synchronised).
  // err_in_ctl: the solve's active lists brought the scan state's error word back with the
  // control words, so no separate read (and host round trip) is needed
  int finish_check(cudaStream_t s, const int* idx = nullptr, int n = 0, bool err_in_ctl = false) {
    if (!err_in_ctl) {
      RK(check_device_error(s));
    } else if (h_ctl[CTL_SCANERR]) {
      CK(cudaMemsetAsync(scan.st.err, 0, sizeof(int32_t), s));
      return fail(GC_ERR_INTERNAL, "a bounded device-side wait gave up");
    }
    if (h_ctl[CTL_ERR] == 1) return fail(GC_ERR_NOT_CONVERGED, "BFS round cap reached");
    if (h_ctl[CTL_ERR] == 2) return fail(GC_ERR_NOT_CONVERGED, "cycle cap reached before the cut was final");
    if (h_ctl[CTL_ERR] == 3) return fail(GC_ERR_INTERNAL, "a bounded wait for a tile copy gave up");
    if (h_ctl[CTL_ERR] == 4) {
      char msg[96];
      snprintf(msg, sizeof(msg), "self-check: worklist value %d out of range (site %d)",
               h_ctl[CTL_BAD], h_ctl[CTL_BADWHERE]);
      return fail(GC_ERR_INTERNAL, msg);
    }
    for (int k = 0; k < (idx ? n : (int)imgs.size()); ++k)
      if (h_acc[idx ? idx[k] : k].bad_caps) return fail(GC_ERR_INVALID, "negative capacity in the upload");
    stats.bfs_rounds = h_ctl[CTL_BFS_TOTAL];
    stats.flood_rounds = h_ctl[CTL_FLOOD_TOTAL];
    if (stats.launches < 0) {  // graph solve: count the kernel nodes that ran
      stats.cycles = h_ctl[CTL_CYCLES];
      stats.pulses = stats.cycles * opts.pulses_per_relabel;
      // the prologue (k_begin_list also builds the first active list), the active lists,
      // the pulses and every BFS / flood round (the flood check runs inside the last round)
      const bool begin_list = !graph_warm && nt <= begin_list_max_tiles();
      stats.launches = (begin_list ? 0 : 1) + h_ctl[CTL_NACT] + stats.pulses +
                       stats.bfs_rounds + stats.flood_rounds;
    }
    for (int k = 0; k < (idx ? n : (int)imgs.size()); ++k) {
      img_solved[idx ? idx[k] : k] = 1;
      img_edited[idx ? idx[k] : k] = 0;
    }
    solved = true;
    edited = false;
    return GC_OK;
  }

  // manual stepping (gc_push / gc_relabel / gc_start_bfs / gc_is_completed)
  int step_push(cudaStream_t s) {
    if (!uploaded) return fail(GC_ERR_STATE, "push before upload");
    if (!list_valid) {
      RK(compact(P.tact, nullptr, s));
      RK(launch_ctl_cycle(P, counts, 0, 0, s));
      list_valid = true;
    }
    solved = false;
    bfs_fresh = false;
    img_solved.assign(imgs.size(), 0);
    img_edited.assign(imgs.size(), 1);   // the next solve starts by flooding
    return launch_discharge(P, opts.discharge_iters, grid_dis, s);
  }
  int step_relabel(cudaStream_t s) {
    if (!uploaded) return fail(GC_ERR_STATE, "relabel before upload");
    solved = false;
    bfs_fresh = false;
    list_valid = true;
    img_solved.assign(imgs.size(), 0);
    img_edited.assign(imgs.size(), 1);
    RK(launch_edge_relabel_build(P, list, counts, scan.st, s));
    return launch_ctl_cycle(P, counts, 0, 0, s);
  }
  int step_start_bfs(cudaStream_t s) {
    if (!uploaded) return fail(GC_ERR_STATE, "startBfs before upload");
    bool warm;
    RK(select_all(&warm, s));
    RK(launch_ctl_begin(P, opts.max_bfs_rounds, opts.max_cycles, acc, s));
    RK(global_relabel(s));
    RK(compact(P.tact, nullptr, s));
    RK(launch_ctl_cycle(P, counts, 0, 0, s));
    list_valid = true;
    bfs_fresh = true;
    return GC_OK;
  }
  int step_is_completed(int* done, cudaStream_t s) {
    if (!bfs_fresh) return fail(GC_ERR_STATE, "isCompleted is valid right after startBfs");
    int n;
    RK(read_count(s, &n));
    *done = n == 0;
    if (*done) {
      RK(launch_acc_reset(acc, (int)imgs.size(), s));
      RK(launch_flood_round(P, 1, 0, 0, acc, grid_warps, s));
      RK(frontier_rounds(s, /*flood=*/true));
      CK(cudaMemcpyAsync(h_acc, acc, sizeof(ImageAcc) * imgs.size(), cudaMemcpyDeviceToHost, s));
      RK(read_ctl(s));
      RK(finish_check(s));
    }
    return GC_OK;
  }

  int flow(int i, int64_t* out) {
    if (i < 0 || i >= (int)imgs.size() || !out) return fail(GC_ERR_INVALID, "bad argument");
    if (!img_solved[i]) return fail(GC_ERR_STATE, "flow before solve");
    *out = (int64_t)(h_acc[i].sumpos_t - h_acc[i].sumpos_e);
    return GC_OK;
  }

  int labels(int i, uint8_t* out, cudaStream_t s) {
    if (i < 0 || i >= (int)imgs.size() || !out) return fail(GC_ERR_INVALID, "bad argument");
    if (!img_solved[i]) return fail(GC_ERR_STATE, "labels before solve");
    CK(cudaSetDevice(device));
    return timed(K_LABELS, s, [&] { return launch_labels_out(P, imgs[i], out, s); });
  }

  // device-side trace: on/off and a fresh start (ordered on the stream)
  int set_trace(int on, cudaStream_t s) {
    CK(cudaSetDevice(device));
    int32_t* w = reinterpret_cast<int32_t*>(static_cast<char*>(pin) + 64);
    CK(cudaStreamSynchronize(s));   // the words' previous copy has been read
    w[0] = on ? 1 : 0;
    w[1] = 0;
    CK(cudaMemcpyAsync(trace_words, w, 2 * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    // the kernels take the trace words as an argument (null when off, so an untraced solve
    // pays no load for it): switching rebuilds the solve graphs at their next use
    int32_t* want = on ? trace_words : nullptr;
    if (P.trace_ctl != want) {
      if (done_ev) CK(cudaEventSynchronize(done_ev));   // no solve graph of ours in flight
      P.trace_ctl = want;
      release_graphs();
    }
    return GC_OK;
  }

  int get_trace(unsigned long long* out, int max, int* n, cudaStream_t s) {
    if (!n || max < 0 || (max > 0 && !out)) return fail(GC_ERR_INVALID, "bad argument");
    CK(cudaSetDevice(device));
    int32_t cnt[2];
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpy(cnt, trace_words, sizeof(cnt), cudaMemcpyDeviceToHost));
    const int have = cnt[1] < GC_TRACE_MAX ? cnt[1] : GC_TRACE_MAX;
    *n = cnt[1];
    const int k = have < max ? have : max;
    if (k > 0) CK(cudaMemcpy(out, P.trace, sizeof(unsigned long long) * 2 * k, cudaMemcpyDeviceToHost));
    return GC_OK;
  }

  int labels_packed(int i, uint8_t* out, cudaStream_t s) {
    if (i < 0 || i >= (int)imgs.size() || !out) return fail(GC_ERR_INVALID, "bad argument");
    if (!img_solved[i]) return fail(GC_ERR_STATE, "labels before solve");
    CK(cudaSetDevice(device));
    return timed(K_LABELS, s, [&] { return launch_labels_packed(P, imgs[i], out, s); });
  }

  // Solves the listed images and writes their labels (bit-packed or one byte per pixel) to
  // outs[k], with one host wait for both.
  int solve_labels(const int* idx, int n, uint8_t* const* outs, bool packed, cudaStream_t s) {
    if (n < 1 || !idx || !outs) return fail(GC_ERR_INVALID, "bad argument");
    for (int k = 0; k < n; ++k)
      if (!outs[k]) return fail(GC_ERR_INVALID, "null label buffer");
    // a pool of one image solved by graph: the solve graph itself ends with the labels
    if (n == 1 && imgs.size() == 1 && idx[0] == 0 && use_graph && !prof && !collect)
      return solve_images(idx, n, s, nullptr, packed ? 2 : 1, outs[0]);
    const After after = [&](cudaStream_t cs) {
      for (int k = 0; k < n; ++k) {
        const ImageDesc& im = imgs[idx[k]];
        RK(timed(K_LABELS, cs, [&] {
          return packed ? launch_labels_packed(P, im, outs[k], cs) : launch_labels_out(P, im, outs[k], cs);
        }));
      }
      return GC_OK;
    };
    return solve_images(idx, n, s, &after);
  }
};

struct gc_handle {
  Pool pool;
};

struct gcb_handle {
  Pool pool;
};

struct gcp_handle {
  Pool pool;
  std::vector<uint8_t> open;   // slot is open
};

// ------------------------------------------------------------------------------------
// Look-back state of the stand-alone primitives (gc_scan_state).  The reference gives every
// tile list its own StreamCompact and PrefixSum objects (IncrementalTileList.pyx:74,
// StreamCompact.pyx:39, PrefixSum.pyx:46); here every such object owns one state, so calls
// from different objects on different streams never share tickets or status words.  A state
// passed as NULL selects one shared state per device.
//
// The device error word is sticky: a launch that gives up a look-back wait (or whose scatter
// index is out of range) sets it and it stays set until the host reports it.  After each
// launch the word is copied into pinned host memory on the caller's stream; the next call on
// the state returns GC_ERR_INTERNAL once that copy has landed with a non-zero word, and
// gc_scan_state_error reads it synchronously.
// ------------------------------------------------------------------------------------
struct gc_scan_state {
  int device = 0;
  ScanBuffers buf;
  int32_t* h_err = nullptr;     // pinned mirror of the device error word
  cudaEvent_t ev = nullptr;     // the last mirror copy
  bool pending = false;
  std::mutex mu;                // one call at a time on a state
  ~gc_scan_state() {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    if (ev) { cudaEventSynchronize(ev); cudaEventDestroy(ev); }
    buf.release();
    if (h_err) cudaFreeHost(h_err);
    cudaSetDevice(cur);
  }
};

namespace {
constexpr int kDefaultScanChunks = 1 << 16;   // the shared per-device state: 2^28 items

int scan_state_init(gc_scan_state* S, int device, int chunks) {
  S->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e) return cuda_fail(e, "cudaSetDevice");
  preload_kernels();
  e = S->buf.alloc(chunks);
  if (e) { cudaGetLastError(); return e == cudaErrorMemoryAllocation ? fail(GC_ERR_OOM, "scan state") : cuda_fail(e, "scan state"); }
  e = cudaHostAlloc((void**)&S->h_err, sizeof(int32_t), cudaHostAllocPortable);
  if (e) { S->h_err = nullptr; cudaGetLastError(); return fail(GC_ERR_OOM, "pinned host allocation failed"); }
  *S->h_err = 0;
  e = cudaEventCreateWithFlags(&S->ev, cudaEventDisableTiming);
  if (e) { S->ev = nullptr; return cuda_fail(e, "event"); }
  return GC_OK;
}

std::mutex g_scan_mu;
std::unordered_map<int, gc_scan_state*> g_scan;   // shared per-device states (never freed)

// The state a primitive runs on (the caller's, or the device's shared one), with the device
// made current.
int resolve_scan_state(gc_scan_state* S, gc_scan_state** out) {
  if (S) {
    cudaError_t e = cudaSetDevice(S->device);
    if (e) return cuda_fail(e, "cudaSetDevice");
    *out = S;
    return GC_OK;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e) return cuda_fail(e, "cudaGetDevice");
  std::lock_guard<std::mutex> lock(g_scan_mu);
  auto it = g_scan.find(dev);
  if (it == g_scan.end()) {
    gc_scan_state* n = new (std::nothrow) gc_scan_state();
    if (!n) return fail(GC_ERR_OOM, "host allocation");
    const int r = scan_state_init(n, dev, kDefaultScanChunks);
    if (r) { delete n; return r; }
    it = g_scan.emplace(dev, n).first;
  }
  *out = it->second;
  return GC_OK;
}

// An error recorded by an earlier launch whose mirror copy has landed (no wait).
int scan_state_take_error(gc_scan_state* S, cudaStream_t s) {
  if (!S->pending || cudaEventQuery(S->ev) != cudaSuccess) { cudaGetLastError(); return GC_OK; }
  S->pending = false;
  if (*S->h_err == 0) return GC_OK;
  const int code = *S->h_err;
  *S->h_err = 0;
  CK(cudaMemsetAsync(S->buf.st.err, 0, sizeof(int32_t), s));
  return fail(GC_ERR_INTERNAL, code == 1 ? "an earlier call on this scan state gave up a bounded look-back wait"
                                         : "an earlier call on this scan state computed an out-of-range index");
}

// After a launch: mirror the error word into pinned memory on the caller's stream.
int scan_state_track(gc_scan_state* S, cudaStream_t s) {
  CK(cudaMemcpyAsync(S->h_err, S->buf.st.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaEventRecord(S->ev, s));
  S->pending = true;
  return GC_OK;
}

// Runs one primitive launch on a state: reports an earlier error, launches, mirrors.
template <class F>
int with_scan_state(gc_scan_state* state, cudaStream_t s, F&& launch) {
  gc_scan_state* S = nullptr;
  RK(resolve_scan_state(state, &S));
  std::lock_guard<std::mutex> lock(S->mu);
  RK(scan_state_take_error(S, s));
  const int r = launch(S->buf.st);
  if (r) return r == GC_ERR_INVALID ? fail(r, "input larger than the scan state holds") : fail(r, "launch failed");
  return scan_state_track(S, s);
}
}  // namespace

int gcut::set_last_error(int code, const char* msg) {
  g_err = msg;
  return code;
}

extern "C" {

const char* gc_last_error(void) { return g_err.c_str(); }

int gc_opts_default(gc_opts* o) {
  if (!o) return fail(GC_ERR_INVALID, "null opts");
  o->device = 0;
  // autotuned (cl-util_b200/autotune.py) on synthetic grids: 3 in-tile iterations x 2
  // discharge launches between exact global relabels is the best of the offline grid at
  // 2048^2 and 4096^2 and within a few percent of the best on smaller grids
  o->discharge_iters = 3;
  o->pulses_per_relabel = 2;
  o->initial_relabel = 0;
  o->max_cycles = 100000;
  o->max_bfs_rounds = 1 << 20;
  o->use_graph = 1;
  return GC_OK;
}

static int check_opts(const gc_opts* o) {
  if (o->discharge_iters < 1 || o->pulses_per_relabel < 1 || o->max_cycles < 1 || o->max_bfs_rounds < 1)
    return fail(GC_ERR_INVALID, "invalid options");
  return GC_OK;
}

int gc_create(int width, int height, const gc_opts* opts, gc_handle** out) {
  g_err.clear();
  if (!out) return fail(GC_ERR_INVALID, "null out");
  *out = nullptr;
  gc_opts o;
  if (opts) o = *opts; else gc_opts_default(&o);
  RK(check_opts(&o));
  gc_handle* h = new (std::nothrow) gc_handle();
  if (!h) return fail(GC_ERR_OOM, "host allocation");
  int w[1] = {width}, hh[1] = {height};
  int r = h->pool.create(1, w, hh, &o);
  if (r) { delete h; return r; }
  *out = h;
  return GC_OK;
}

int gc_arena_bytes(int width, int height, int64_t* bytes) {
  g_err.clear();
  if (!bytes) return fail(GC_ERR_INVALID, "null out");
  Pool p;
  int w[1] = {width}, hh[1] = {height};
  RK(p.describe(1, w, hh));
  *bytes = (int64_t)p.arena_bytes;
  return GC_OK;
}

int gc_create_in(int width, int height, const gc_opts* opts, void* arena, int64_t bytes,
                 gc_handle** out) {
  g_err.clear();
  if (!out) return fail(GC_ERR_INVALID, "null out");
  *out = nullptr;
  if (!arena || bytes <= 0) return fail(GC_ERR_INVALID, "null arena");
  gc_opts o;
  if (opts) o = *opts; else gc_opts_default(&o);
  RK(check_opts(&o));
  gc_handle* h = new (std::nothrow) gc_handle();
  if (!h) return fail(GC_ERR_OOM, "host allocation");
  int w[1] = {width}, hh[1] = {height};
  int r = h->pool.create(1, w, hh, &o, arena, (size_t)bytes);
  if (r) { delete h; return r; }
  *out = h;
  return GC_OK;
}

int gc_destroy(gc_handle* h) {
  if (!h) return GC_OK;
  cudaSetDevice(h->pool.device);
  delete h;
  return GC_OK;
}

int gc_size(const gc_handle* h, int* w, int* hh) {
  if (!h || !w || !hh) return fail(GC_ERR_INVALID, "null argument");
  *w = h->pool.imgs[0].W;
  *hh = h->pool.imgs[0].H;
  return GC_OK;
}

int gc_upload(gc_handle* h, const int32_t* up, const int32_t* down, const int32_t* left,
              const int32_t* right, const int32_t* excess, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  const int r = h->pool.upload(0, up, down, left, right, excess, (cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_upload_host(gc_handle* h, const int32_t* up, const int32_t* down, const int32_t* left,
                   const int32_t* right, const int32_t* excess, void* stream) {
  g_err.clear();
  if (!h || !up || !down || !left || !right || !excess) return fail(GC_ERR_INVALID, "null argument");
  Pool& p = h->pool;
  CK(cudaSetDevice(p.device));
  const size_t n = (size_t)p.imgs[0].W * p.imgs[0].H;
  if (!p.stage) {
    cudaError_t e = cudaMalloc((void**)&p.stage, 5 * n * sizeof(int32_t));
    if (e) { p.stage = nullptr; cudaGetLastError(); return fail(GC_ERR_OOM, "staging buffer"); }
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int32_t* src[5] = {up, down, left, right, excess};
  for (int k = 0; k < 5; ++k)
    CK(cudaMemcpyAsync(p.stage + k * n, src[k], n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  int r = p.upload(0, p.stage, p.stage + n, p.stage + 2 * n, p.stage + 3 * n, p.stage + 4 * n, s);
  p.track(s);
  if (r) return r;
  CK(cudaStreamSynchronize(s));
  return GC_OK;
}

static int upload_rgba_dev(gc_handle* h, const uint32_t* rgba, const int32_t* excess, int lambda,
                           void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  const int r = h->pool.upload_rgba(0, rgba, excess, lambda, (cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

static int upload_rgba_host(gc_handle* h, const uint32_t* rgba, const int32_t* excess, int lambda,
                            void* stream) {
  g_err.clear();
  if (!h || !rgba || !excess) return fail(GC_ERR_INVALID, "null argument");
  Pool& p = h->pool;
  CK(cudaSetDevice(p.device));
  const size_t n = (size_t)p.imgs[0].W * p.imgs[0].H;
  if (!p.stage) {
    cudaError_t e = cudaMalloc((void**)&p.stage, 5 * n * sizeof(int32_t));
    if (e) { p.stage = nullptr; cudaGetLastError(); return fail(GC_ERR_OOM, "staging buffer"); }
  }
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t* img = reinterpret_cast<const uint32_t*>(p.stage);
  CK(cudaMemcpyAsync(p.stage, rgba, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(p.stage + n, excess, n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  int r = p.upload_rgba(0, img, p.stage + n, lambda, s);
  p.track(s);
  if (r) return r;
  CK(cudaStreamSynchronize(s));
  return GC_OK;
}

int gc_upload_rgba(gc_handle* h, const uint32_t* rgba, const int32_t* excess, void* stream) {
  return upload_rgba_dev(h, rgba, excess, 0, stream);
}

int gc_upload_rgba_host(gc_handle* h, const uint32_t* rgba, const int32_t* excess,
                        void* stream) {
  return upload_rgba_host(h, rgba, excess, 0, stream);
}

int gc_upload_rgba_lambda(gc_handle* h, const uint32_t* rgba, const int32_t* excess,
                          int32_t lambda, void* stream) {
  if (lambda < 1) return fail(GC_ERR_INVALID, "lambda out of range");
  return upload_rgba_dev(h, rgba, excess, lambda, stream);
}

int gc_upload_rgba_lambda_host(gc_handle* h, const uint32_t* rgba, const int32_t* excess,
                               int32_t lambda, void* stream) {
  if (lambda < 1) return fail(GC_ERR_INVALID, "lambda out of range");
  return upload_rgba_host(h, rgba, excess, lambda, stream);
}

int gc_solve(gc_handle* h, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  const int r = h->pool.solve((cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_solve_labels(gc_handle* h, uint8_t* labels, int packed, void* stream) {
  g_err.clear();
  if (!h || !labels) return fail(GC_ERR_INVALID, "null argument");
  const int zero = 0;
  const int r = h->pool.solve_labels(&zero, 1, &labels, packed != 0, (cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_flow(gc_handle* h, int64_t* flow) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  return h->pool.flow(0, flow);
}

int gc_labels(gc_handle* h, uint8_t* labels, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  const int r = h->pool.labels(0, labels, (cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_labels_host(gc_handle* h, uint8_t* labels, void* stream) {
  g_err.clear();
  if (!h || !labels) return fail(GC_ERR_INVALID, "null argument");
  Pool& p = h->pool;
  CK(cudaSetDevice(p.device));
  const size_t n = (size_t)p.imgs[0].W * p.imgs[0].H;
  cudaStream_t s = (cudaStream_t)stream;
  RK(p.labels(0, p.lstage, s));
  CK(cudaMemcpyAsync(labels, p.lstage, n, cudaMemcpyDeviceToHost, s));
  p.track(s);
  CK(cudaStreamSynchronize(s));
  return GC_OK;
}

int gc_labels_packed(gc_handle* h, uint8_t* bits, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  const int r = h->pool.labels_packed(0, bits, (cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_labels_packed_host(gc_handle* h, uint8_t* bits, void* stream) {
  g_err.clear();
  if (!h || !bits) return fail(GC_ERR_INVALID, "null argument");
  Pool& p = h->pool;
  CK(cudaSetDevice(p.device));
  const size_t n = (size_t)p.imgs[0].H * ((p.imgs[0].W + 7) / 8);   // fits the label staging
  cudaStream_t s = (cudaStream_t)stream;
  RK(p.labels_packed(0, p.lstage, s));
  CK(cudaMemcpyAsync(bits, p.lstage, n, cudaMemcpyDeviceToHost, s));
  p.track(s);
  CK(cudaStreamSynchronize(s));
  return GC_OK;
}

int gc_edit_tlinks(gc_handle* h, const int32_t* idx, const int32_t* value, int n, void* stream) {
  g_err.clear();
  if (!h || n < 0 || (n > 0 && (!idx || !value))) return fail(GC_ERR_INVALID, "bad argument");
  Pool& p = h->pool;
  if (!p.uploaded) return fail(GC_ERR_STATE, "edit before upload");
  CK(cudaSetDevice(p.device));
  RK(launch_edit(p.P, p.imgs[0], 0, idx, value, n, p.tl, p.acc, (cudaStream_t)stream));
  p.track((cudaStream_t)stream);
  p.edited_image(0);
  return GC_OK;
}

int gc_edit_stroke(gc_handle* h, const int32_t* xs, const int32_t* ys, int npts, int radius,
                   int32_t value, void* stream) {
  g_err.clear();
  if (!h || !xs || !ys || npts < 1 || npts > 1024 || radius < 0 || radius > 4096)
    return fail(GC_ERR_INVALID, "bad stroke");
  Pool& p = h->pool;
  if (!p.uploaded) return fail(GC_ERR_STATE, "edit before upload");
  CK(cudaSetDevice(p.device));
  std::vector<int32_t> pts(2 * npts);
  for (int k = 0; k < npts; ++k) { pts[2 * k] = xs[k]; pts[2 * k + 1] = ys[k]; }
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(p.pts, pts.data(), pts.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  RK(launch_stroke(p.P, p.imgs[0], 0, p.pts, pts.data(), npts, radius, value, p.tl, p.acc, s));
  p.track(s);
  CK(cudaStreamSynchronize(s));  // pts (host vector) must outlive the copy
  p.edited_image(0);
  return GC_OK;
}

int gc_edit_brush(gc_handle* h, const int32_t* xs, const int32_t* ys, int npts, int radius,
                  int32_t value, void* stream) {
  g_err.clear();
  if (!h || !xs || !ys || npts < 1 || npts > 1024 || radius > 1024)
    return fail(GC_ERR_INVALID, "bad brush stroke");
  Pool& p = h->pool;
  if (!p.uploaded) return fail(GC_ERR_STATE, "edit before upload");
  CK(cudaSetDevice(p.device));
  std::vector<int32_t> pts(2 * npts);
  for (int k = 0; k < npts; ++k) { pts[2 * k] = xs[k]; pts[2 * k + 1] = ys[k]; }
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(p.pts, pts.data(), pts.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  RK(launch_brush(p.P, p.imgs[0], 0, p.pts, pts.data(), npts, radius, value, p.tl, p.acc, s));
  p.track(s);
  CK(cudaStreamSynchronize(s));  // pts (host vector) must outlive the copy
  p.edited_image(0);
  return GC_OK;
}

int gc_download_state(gc_handle* h, int32_t* excess, int32_t* height, int32_t* up,
                      int32_t* down, int32_t* left, int32_t* right, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  Pool& p = h->pool;
  CK(cudaSetDevice(p.device));
  cudaStream_t s = (cudaStream_t)stream;
  const int32_t* planes[6] = {p.P.exc, p.P.hgt, p.P.cap[0], p.P.cap[1], p.P.cap[2], p.P.cap[3]};
  int32_t* outs[6] = {excess, height, up, down, left, right};
  for (int k = 0; k < 6; ++k)
    if (outs[k]) RK(launch_state_out(p.P, p.imgs[0], planes[k], outs[k], s));
  p.track(s);
  return GC_OK;
}

int gc_push(gc_handle* h, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  const int r = h->pool.step_push((cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_relabel(gc_handle* h, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  const int r = h->pool.step_relabel((cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_start_bfs(gc_handle* h, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  const int r = h->pool.step_start_bfs((cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_is_completed(gc_handle* h, int* completed, void* stream) {
  g_err.clear();
  if (!h || !completed) return fail(GC_ERR_INVALID, "null argument");
  const int r = h->pool.step_is_completed(completed, (cudaStream_t)stream);
  h->pool.track((cudaStream_t)stream);
  return r;
}

int gc_set_trace(gc_handle* h, int on, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  return h->pool.set_trace(on, (cudaStream_t)stream);
}

int gc_get_trace(gc_handle* h, uint64_t* entries, int max_entries, int* n, void* stream) {
  g_err.clear();
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  return h->pool.get_trace(reinterpret_cast<unsigned long long*>(entries), max_entries, n,
                           (cudaStream_t)stream);
}

int gcb_set_trace(gcb_handle* b, int on, void* stream) {
  g_err.clear();
  if (!b) return fail(GC_ERR_INVALID, "null handle");
  return b->pool.set_trace(on, (cudaStream_t)stream);
}

int gcb_get_trace(gcb_handle* b, uint64_t* entries, int max_entries, int* n, void* stream) {
  g_err.clear();
  if (!b) return fail(GC_ERR_INVALID, "null handle");
  return b->pool.get_trace(reinterpret_cast<unsigned long long*>(entries), max_entries, n,
                           (cudaStream_t)stream);
}

int gc_get_stats(const gc_handle* h, gc_stats* st) {
  if (!h || !st) return fail(GC_ERR_INVALID, "null argument");
  *st = h->pool.stats;
  return GC_OK;
}

int gc_set_profile(gc_handle* h, int on) {
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  h->pool.prof = on != 0;
  return GC_OK;
}

int gc_get_profile(const gc_handle* h, gc_kernel_prof* out, int n) {
  if (!h || !out || n < 0) return fail(GC_ERR_INVALID, "bad argument");
  for (int k = 0; k < n && k < GC_NKERN; ++k) out[k] = h->pool.kprof[k];
  return GC_OK;
}

const char* gc_kernel_name(int kind) {
  static const char* names[GC_NKERN] = {"upload", "discharge", "edge_relabel_build", "bfs_first",
                                        "bfs", "flood_first", "flood", "compact", "labels",
                                        "masks"};
  return kind >= 0 && kind < GC_NKERN ? names[kind] : "";
}

int gc_set_collect_stats(gc_handle* h, int on) {
  if (!h) return fail(GC_ERR_INVALID, "null handle");
  h->pool.collect = on != 0;
  return GC_OK;
}

// ---- primitives -------------------------------------------------------------------
int gc_scan_state_create(int device, int max_items, gc_scan_state** out) {
  g_err.clear();
  if (!out || max_items < 0) return fail(GC_ERR_INVALID, "bad argument");
  *out = nullptr;
  gc_scan_state* S = new (std::nothrow) gc_scan_state();
  if (!S) return fail(GC_ERR_OOM, "host allocation");
  // chunks of the widest launch on max_items: the scan's (4096 items each), at least two
  // (the look-back self-test uses two)
  int chunks = scan_chunks(max_items);
  if (chunks < 2) chunks = 2;
  const int r = scan_state_init(S, device, chunks);
  if (r) { delete S; return r; }
  *out = S;
  return GC_OK;
}

int gc_scan_state_destroy(gc_scan_state* S) {
  if (!S) return GC_OK;
  std::lock_guard<std::mutex> lock(g_scan_mu);
  for (auto& kv : g_scan)
    if (kv.second == S) return fail(GC_ERR_INVALID, "the shared per-device state is not destroyed");
  delete S;
  return GC_OK;
}

int gc_scan_state_error(gc_scan_state* state, int* err, void* stream) {
  g_err.clear();
  if (!err) return fail(GC_ERR_INVALID, "null argument");
  gc_scan_state* S = nullptr;
  RK(resolve_scan_state(state, &S));
  std::lock_guard<std::mutex> lock(S->mu);
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(S->h_err, S->buf.st.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *err = *S->h_err;
  S->pending = false;
  if (*err) {
    *S->h_err = 0;
    CK(cudaMemsetAsync(S->buf.st.err, 0, sizeof(int32_t), s));
    CK(cudaStreamSynchronize(s));
  }
  return GC_OK;
}

int gc_scan_state_selftest(gc_scan_state* state, int spins, int* err, void* stream) {
  g_err.clear();
  if (spins < 1) return fail(GC_ERR_INVALID, "bad argument");
  gc_scan_state* S = nullptr;
  RK(resolve_scan_state(state, &S));
  {
    std::lock_guard<std::mutex> lock(S->mu);
    ScanState st = S->buf.st;
    st.spin_limit = spins;
    const int r = launch_lookback_selftest(st, (cudaStream_t)stream);
    if (r) return fail(r, "self-test launch failed");
    if (!err) return scan_state_track(S, (cudaStream_t)stream);   // reported like any error
  }
  return gc_scan_state_error(S, err, stream);
}

int gc_scan_exclusive(gc_scan_state* state, const int32_t* in, int32_t* out, int32_t* total,
                      int n, void* stream) {
  g_err.clear();
  if (n < 0 || (n > 0 && (!in || !out)) || !total) return fail(GC_ERR_INVALID, "bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  return with_scan_state(state, s, [&](const ScanState& st) {
    return launch_scan(GC_SCAN_MODE_SCAN, in, nullptr, nullptr, out, nullptr, total, n, 0, 0, 0,
                       0, 0, st, s);
  });
}

int gc_compact(gc_scan_state* state, const int32_t* flags, int32_t* list, int32_t* length,
               int n, void* stream) {
  g_err.clear();
  if (n < 0 || (n > 0 && (!flags || !list)) || !length) return fail(GC_ERR_INVALID, "bad argument");
  if (n > 0 && flags == list) return fail(GC_ERR_INVALID, "list must not alias flags");
  cudaStream_t s = (cudaStream_t)stream;
  return with_scan_state(state, s, [&](const ScanState& st) {
    return launch_scan(GC_SCAN_MODE_COMPACT, flags, nullptr, nullptr, nullptr, list, length, n, 0,
                       0, 0, 0, 0, st, s);
  });
}

int gc_tiles_build(gc_scan_state* state, const int32_t* tiles, int op, int32_t operand,
                   int32_t* list, int32_t* length, int n, void* stream) {
  g_err.clear();
  if (n < 0 || (n > 0 && (!tiles || !list)) || !length || op < 0 || op > 4)
    return fail(GC_ERR_INVALID, "bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  return with_scan_state(state, s, [&](const ScanState& st) {
    return launch_scan(GC_SCAN_MODE_FLAG, tiles, nullptr, nullptr, nullptr, list, length, n, op,
                       operand, 0, 0, 0, st, s);
  });
}

int gc_tiles_build_logical(gc_scan_state* state, const int32_t* tiles, const int32_t* tiles2,
                           int op1, int32_t a1, int op2, int32_t a2, int logical, int32_t* list,
                           int32_t* length, int n, void* stream) {
  g_err.clear();
  if (n < 0 || (n > 0 && (!tiles || !tiles2 || !list)) || !length || op1 < 0 || op1 > 4 ||
      op2 < 0 || op2 > 4 || logical < 0 || logical > 1)
    return fail(GC_ERR_INVALID, "bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  return with_scan_state(state, s, [&](const ScanState& st) {
    return launch_scan(GC_SCAN_MODE_LOGICAL, tiles, tiles2, nullptr, nullptr, list, length, n,
                       op1, a1, op2, a2, logical, st, s);
  });
}

int gc_tiles_incorporate(int32_t* tiles, const int32_t* tiles2, int op1, int32_t a1, int op2,
                         int32_t a2, int logical, int32_t iteration, int n, void* stream) {
  g_err.clear();
  if (n < 0 || (n > 0 && (!tiles || !tiles2)) || op1 < 0 || op1 > 4 || op2 < 0 || op2 > 4 ||
      logical < 0 || logical > 1)
    return fail(GC_ERR_INVALID, "bad argument");
  return launch_increment_logical(tiles, tiles2, tiles, n, op1, op2, a1, a2, logical, iteration,
                                  (cudaStream_t)stream);
}

int gc_tiles_fill(int32_t* tiles, int32_t value, int n, void* stream) {
  g_err.clear();
  if (n < 0 || (n > 0 && !tiles)) return fail(GC_ERR_INVALID, "bad argument");
  return launch_fill(tiles, n, value, (cudaStream_t)stream);
}

int gc_view_colorize(const int32_t* values, int values_w, int values_h, int cell_w, int cell_h,
                     int width, int height, const float* ramp, const uint32_t* base,
                     uint32_t* out, void* stream) {
  g_err.clear();
  if (values_w < 0 || values_h < 0 || cell_w < 1 || cell_h < 1 || width < 0 || height < 0)
    return fail(GC_ERR_INVALID, "gc_view_colorize: bad size");
  if (!ramp) return fail(GC_ERR_INVALID, "gc_view_colorize: null ramp");
  for (int k = 0; k < 9; ++k)
    if (!std::isfinite(ramp[k])) return fail(GC_ERR_INVALID, "gc_view_colorize: ramp not finite");
  if ((long long)width * height > 0 && (!out || ((long long)values_w * values_h > 0 && !values)))
    return fail(GC_ERR_INVALID, "gc_view_colorize: null pointer");
  const int r = launch_view_colorize(values, values_w, values_h, cell_w, cell_h, width, height,
                                     ramp, base, out, (cudaStream_t)stream);
  return r == GC_OK ? GC_OK : fail(r, "gc_view_colorize: launch failed");
}

int gc_tiles_view(const int32_t* tiles, int tiles_w, int tiles_h, int tile_w, int tile_h,
                  int32_t iteration, int width, int height, uint32_t* out, void* stream) {
  g_err.clear();
  if (tiles_w < 0 || tiles_h < 0 || tile_w < 1 || tile_h < 1 || width < 0 || height < 0)
    return fail(GC_ERR_INVALID, "gc_tiles_view: bad size");
  if ((long long)width * height > 0 && (!out || ((long long)tiles_w * tiles_h > 0 && !tiles)))
    return fail(GC_ERR_INVALID, "gc_tiles_view: null pointer");
  const int r = launch_tiles_view(tiles, tiles_w, tiles_h, tile_w, tile_h, iteration, width,
                                  height, out, (cudaStream_t)stream);
  return r == GC_OK ? GC_OK : fail(r, "gc_tiles_view: launch failed");
}

// ---- batch ------------------------------------------------------------------------
int gcb_create(int n, const int* widths, const int* heights, const gc_opts* opts,
               gcb_handle** out) {
  g_err.clear();
  if (!out) return fail(GC_ERR_INVALID, "null out");
  *out = nullptr;
  gc_opts o;
  if (opts) o = *opts; else gc_opts_default(&o);
  RK(check_opts(&o));
  gcb_handle* b = new (std::nothrow) gcb_handle();
  if (!b) return fail(GC_ERR_OOM, "host allocation");
  int r = b->pool.create(n, widths, heights, &o);
  if (r) { delete b; return r; }
  *out = b;
  return GC_OK;
}

int gcb_destroy(gcb_handle* b) {
  if (!b) return GC_OK;
  cudaSetDevice(b->pool.device);
  delete b;
  return GC_OK;
}

int gcb_upload(gcb_handle* b, int i, const int32_t* up, const int32_t* down,
               const int32_t* left, const int32_t* right, const int32_t* excess, void* stream) {
  g_err.clear();
  if (!b) return fail(GC_ERR_INVALID, "null handle");
  Pool& p = b->pool;
  int r = p.upload(i, up, down, left, right, excess, (cudaStream_t)stream);
  return r;
}

int gcb_solve(gcb_handle* b, void* stream) {
  g_err.clear();
  if (!b) return fail(GC_ERR_INVALID, "null handle");
  return b->pool.solve((cudaStream_t)stream);
}

int gcb_flow(gcb_handle* b, int i, int64_t* flow) {
  g_err.clear();
  if (!b) return fail(GC_ERR_INVALID, "null handle");
  return b->pool.flow(i, flow);
}

int gcb_labels(gcb_handle* b, int i, uint8_t* labels, void* stream) {
  g_err.clear();
  if (!b) return fail(GC_ERR_INVALID, "null handle");
  return b->pool.labels(i, labels, (cudaStream_t)stream);
}

int gcb_set_profile(gcb_handle* b, int on) {
  if (!b) return fail(GC_ERR_INVALID, "null handle");
  b->pool.prof = on != 0;
  return GC_OK;
}

int gcb_get_profile(const gcb_handle* b, gc_kernel_prof* out, int n) {
  if (!b || !out || n < 0) return fail(GC_ERR_INVALID, "bad argument");
  for (int k = 0; k < n && k < GC_NKERN; ++k) out[k] = b->pool.kprof[k];
  return GC_OK;
}

int gcb_get_stats(const gcb_handle* b, gc_stats* st) {
  if (!b || !st) return fail(GC_ERR_INVALID, "null argument");
  *st = b->pool.stats;
  return GC_OK;
}

// ---- session pools -----------------------------------------------------------------
int gcp_arena_bytes(int max_tiles, int max_sessions, int64_t* bytes) {
  g_err.clear();
  if (!bytes) return fail(GC_ERR_INVALID, "null out");
  Pool p;
  RK(p.describe_dynamic(max_tiles, max_sessions));
  *bytes = (int64_t)p.arena_bytes;
  return GC_OK;
}

static int gcp_make(int max_tiles, int max_sessions, const gc_opts* opts, void* arena,
                    int64_t bytes, gcp_handle** out) {
  g_err.clear();
  if (!out) return fail(GC_ERR_INVALID, "null out");
  *out = nullptr;
  gc_opts o;
  if (opts) o = *opts; else gc_opts_default(&o);
  RK(check_opts(&o));
  gcp_handle* h = new (std::nothrow) gcp_handle();
  if (!h) return fail(GC_ERR_OOM, "host allocation");
  int r = h->pool.create_dynamic(max_tiles, max_sessions, &o, arena, (size_t)bytes);
  if (r) { delete h; return r; }
  h->open.assign(max_sessions, 0);
  *out = h;
  return GC_OK;
}

int gcp_create(int max_tiles, int max_sessions, const gc_opts* opts, gcp_handle** out) {
  return gcp_make(max_tiles, max_sessions, opts, nullptr, 0, out);
}

int gcp_create_in(int max_tiles, int max_sessions, const gc_opts* opts, void* arena,
                  int64_t bytes, gcp_handle** out) {
  if (!arena || bytes <= 0) return fail(GC_ERR_INVALID, "null arena");
  return gcp_make(max_tiles, max_sessions, opts, arena, bytes, out);
}

int gcp_destroy(gcp_handle* p) {
  if (!p) return GC_OK;
  cudaSetDevice(p->pool.device);
  delete p;
  return GC_OK;
}

static int gcp_slot(gcp_handle* p, int slot, bool must_be_open) {
  if (!p) return fail(GC_ERR_INVALID, "null handle");
  if (slot < 0 || slot >= (int)p->open.size()) return fail(GC_ERR_INVALID, "slot out of range");
  if (must_be_open && !p->open[slot]) return fail(GC_ERR_STATE, "slot not open");
  return GC_OK;
}

int gcp_open(gcp_handle* p, int slot, int width, int height, int tile0, void* stream) {
  g_err.clear();
  RK(gcp_slot(p, slot, false));
  if (p->open[slot]) return fail(GC_ERR_STATE, "slot already open");
  if (width < 1 || height < 1 || width > (1 << 16) || height > (1 << 16))
    return fail(GC_ERR_INVALID, "image size out of range");
  Pool& pool = p->pool;
  const ImageDesc d{width, height, (width + 31) / 32, (height + 31) / 32, tile0};
  const long long tiles = (long long)d.tw * d.th;
  if (tile0 < 0 || tile0 + tiles > pool.nt) return fail(GC_ERR_INVALID, "tile range outside the pool");
  for (size_t k = 0; k < p->open.size(); ++k) {   // no two open slots share a tile
    if (!p->open[k]) continue;
    const ImageDesc& o = pool.imgs[k];
    const long long a0 = o.tile0, a1 = o.tile0 + (long long)o.tw * o.th;
    if (tile0 < a1 && a0 < tile0 + tiles) return fail(GC_ERR_INVALID, "tile range overlaps an open slot");
  }
  CK(cudaSetDevice(pool.device));
  pool.imgs[slot] = d;
  RK(launch_image_tiles(pool.P, d, slot, (cudaStream_t)stream));
  pool.img_up[slot] = pool.img_solved[slot] = pool.img_edited[slot] = 0;
  p->open[slot] = 1;
  pool.track((cudaStream_t)stream);
  return GC_OK;
}

int gcp_close(gcp_handle* p, int slot) {
  g_err.clear();
  RK(gcp_slot(p, slot, true));
  p->open[slot] = 0;
  p->pool.img_up[slot] = p->pool.img_solved[slot] = 0;
  return GC_OK;
}

int gcp_upload(gcp_handle* p, int slot, const int32_t* up, const int32_t* down,
               const int32_t* left, const int32_t* right, const int32_t* excess, void* stream) {
  g_err.clear();
  RK(gcp_slot(p, slot, true));
  const int r = p->pool.upload(slot, up, down, left, right, excess, (cudaStream_t)stream);
  p->pool.track((cudaStream_t)stream);
  return r;
}

int gcp_upload_rgba(gcp_handle* p, int slot, const uint32_t* rgba, const int32_t* excess,
                    void* stream) {
  g_err.clear();
  RK(gcp_slot(p, slot, true));
  const int r = p->pool.upload_rgba(slot, rgba, excess, 0, (cudaStream_t)stream);
  p->pool.track((cudaStream_t)stream);
  return r;
}

static int gcp_edit(gcp_handle* p, int slot, const int32_t* xs, const int32_t* ys, int npts,
                    int radius, int32_t value, bool brush, void* stream) {
  g_err.clear();
  RK(gcp_slot(p, slot, true));
  if (!xs || !ys || npts < 1 || npts > 1024 || radius > (brush ? 1024 : 4096) ||
      (!brush && radius < 0))
    return fail(GC_ERR_INVALID, "bad stroke");
  Pool& pool = p->pool;
  if (!pool.img_up[slot]) return fail(GC_ERR_STATE, "edit before upload");
  CK(cudaSetDevice(pool.device));
  std::vector<int32_t> pts(2 * npts);
  for (int k = 0; k < npts; ++k) { pts[2 * k] = xs[k]; pts[2 * k + 1] = ys[k]; }
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(pool.pts, pts.data(), pts.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (brush)
    RK(launch_brush(pool.P, pool.imgs[slot], slot, pool.pts, pts.data(), npts, radius, value, pool.tl, pool.acc, s));
  else
    RK(launch_stroke(pool.P, pool.imgs[slot], slot, pool.pts, pts.data(), npts, radius, value, pool.tl, pool.acc, s));
  pool.track(s);
  CK(cudaStreamSynchronize(s));  // pts (host vector) must outlive the copy
  pool.edited_image(slot);
  return GC_OK;
}

int gcp_edit_stroke(gcp_handle* p, int slot, const int32_t* xs, const int32_t* ys, int npts,
                    int radius, int32_t value, void* stream) {
  return gcp_edit(p, slot, xs, ys, npts, radius, value, false, stream);
}

int gcp_edit_brush(gcp_handle* p, int slot, const int32_t* xs, const int32_t* ys, int npts,
                   int radius, int32_t value, void* stream) {
  return gcp_edit(p, slot, xs, ys, npts, radius, value, true, stream);
}

int gcp_solve(gcp_handle* p, const int* slots, int n, void* stream) {
  g_err.clear();
  if (!p || !slots || n < 1) return fail(GC_ERR_INVALID, "bad argument");
  for (int k = 0; k < n; ++k) RK(gcp_slot(p, slots[k], true));
  const int r = p->pool.solve_images(slots, n, (cudaStream_t)stream);
  p->pool.track((cudaStream_t)stream);
  return r;
}

int gcp_solve_labels(gcp_handle* p, const int* slots, int n, uint8_t* const* labels, int packed,
                     void* stream) {
  g_err.clear();
  if (!p || !slots || !labels || n < 1) return fail(GC_ERR_INVALID, "bad argument");
  for (int k = 0; k < n; ++k) RK(gcp_slot(p, slots[k], true));
  const int r = p->pool.solve_labels(slots, n, labels, packed != 0, (cudaStream_t)stream);
  p->pool.track((cudaStream_t)stream);
  return r;
}

int gcp_flow(gcp_handle* p, int slot, int64_t* flow) {
  g_err.clear();
  RK(gcp_slot(p, slot, true));
  return p->pool.flow(slot, flow);
}

int gcp_labels(gcp_handle* p, int slot, uint8_t* labels, void* stream) {
  g_err.clear();
  RK(gcp_slot(p, slot, true));
  const int r = p->pool.labels(slot, labels, (cudaStream_t)stream);
  p->pool.track((cudaStream_t)stream);
  return r;
}

int gcp_labels_packed(gcp_handle* p, int slot, uint8_t* bits, void* stream) {
  g_err.clear();
  RK(gcp_slot(p, slot, true));
  const int r = p->pool.labels_packed(slot, bits, (cudaStream_t)stream);
  p->pool.track((cudaStream_t)stream);
  return r;
}

int gcp_set_trace(gcp_handle* p, int on, void* stream) {
  g_err.clear();
  if (!p) return fail(GC_ERR_INVALID, "null handle");
  return p->pool.set_trace(on, (cudaStream_t)stream);
}

int gcp_get_trace(gcp_handle* p, uint64_t* entries, int max_entries, int* n, void* stream) {
  g_err.clear();
  if (!p) return fail(GC_ERR_INVALID, "null handle");
  return p->pool.get_trace(reinterpret_cast<unsigned long long*>(entries), max_entries, n,
                           (cudaStream_t)stream);
}

int gcp_get_stats(const gcp_handle* p, gc_stats* st) {
  if (!p || !st) return fail(GC_ERR_INVALID, "null argument");
  *st = p->pool.stats;
  return GC_OK;
}

}  // extern "C"
