// api.cpp -- the C ABI of scarl_b200 (include/scarl.h): contexts, device
// workspace, cached per-grid plans (twiddles, spectrum tables and the FP64
// spectral normalisation), host<->device staging, and the dispatch of every
// entry point onto the sm_100a kernels.  No CPU fallback: every numerical
// entry point runs on the GPU or returns an error.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/scarl.h"
#include "h5io.h"
#include "host_maps.h"
#include "scarl_internal.h"

using namespace scarl;

namespace {

constexpr double kPiRef = 3.1415926535898;  // SRC_F/constants_ScaRL.f90:5

struct Buf {
  void* p = nullptr;
  size_t n = 0;
};

struct PaddedPlan {
  int dt = 4;
  int amp = AMP_SEPARABLE;
  double expo = 0.0;
  double norm = 1.0;
  Buf tabs;
  const void* t[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

struct Mark {
  std::string name;
  cudaEvent_t a, b;
};

// One batched launch of an ensemble: the realisations that share the line
// length N of a pass, launched with variant var.
struct EnsGroup {
  int pass = 1, N = 0, var = 0;
  std::vector<int> items;  // realisations, largest first
  std::vector<int> start;  // block offsets (items.size() + 1)
  BatchMap m{};
};

// Plan of the most recent ensemble (list of shapes) of a context.
struct EnsPlan {
  std::string key;
  int dt = 4, n = 0;
  bool split = false;  // FP32 with the split-BF16 tensor-core pass 1 where its z length has one
  std::vector<GenArgs> args;  // host copies of the device argument blocks
  std::vector<size_t> off;    // first element of each field in the output
  size_t total = 0;           // elements of all fields
  Buf work, dargs, dmap, tmp;
  std::vector<EnsGroup> groups;  // pass-major
  bool uploaded = false, tuned = false, graph_failed = false;
  cudaGraphExec_t exec = nullptr;
};

// A few host threads that copy a staged chunk into the caller's pageable
// memory in parallel (memory bandwidth and first-touch page faults of a fresh
// destination are shared among them).  run(f) calls f(p) for every part p <
// parts(), part 0 on the calling thread, and returns when all are done.
class HostPool {
 public:
  explicit HostPool(int workers) {
    for (int i = 0; i < workers; ++i) th_.emplace_back([this, i] { loop(i + 1); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (std::thread& t : th_) t.join();
  }
  int parts() const { return (int)th_.size() + 1; }
  void run(const std::function<void(int)>& f) {
    {
      std::lock_guard<std::mutex> g(m_);
      f_ = &f;
      pending_ = (int)th_.size();
      ++gen_;
    }
    cv_.notify_all();
    f(0);
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [&] { return pending_ == 0; });
    f_ = nullptr;
  }

 private:
  void loop(int p) {
    long seen = 0;
    for (;;) {
      const std::function<void(int)>* f;
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        f = f_;
      }
      (*f)(p);
      std::lock_guard<std::mutex> g(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* f_ = nullptr;
  int pending_ = 0;
  long gen_ = 0;
  bool stop_ = false;
};

// pageable host output: chunks of kRingChunk bytes through kRingSlots pinned
// slots, for outputs of at least kRingMin bytes
constexpr int kRingSlots = 4;
constexpr size_t kRingChunk = (size_t)32 << 20;
constexpr size_t kRingMin = (size_t)8 << 20;

}  // namespace

struct scarl_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  size_t budget = 0, used = 0;
  std::string err;
  Buf work, tile, stage_out, stage_in, stage_in2, tabs, dtabs, part, t1, t2, sk, pmpw;
  Buf status;  // device word raised by kernels whose bounded waits expired
  Buf mom;     // FP64 partial pairs of the streamed moments (pass 3) and their sum
  int wait_test = 0;  // test hook of the bounded tensor-core waits
  void* pin = nullptr;
  size_t pin_n = 0;
  cudaEvent_t pin_ev = nullptr;
  // device -> pinned host copies of finished z slabs, overlapped with the
  // generation of the remaining tiles
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> slab_ev;
  Buf targs;  // argument blocks and block maps of the tiles batched in passes 1-2
  // pinned ring and copy threads of pageable host outputs
  char* ring = nullptr;
  cudaEvent_t ring_ev[kRingSlots] = {};
  HostPool* hpool = nullptr;
  std::map<std::string, PaddedPlan> plans;
  std::map<long long, Buf> twiddles;
  std::map<int, Buf> dct_tabs;
  bool profile = false;
  long long launches = 0;
  unsigned long long h2d = 0, d2h = 0;
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> pool;
  std::vector<std::string> porder;
  std::map<std::string, std::pair<double, long long>> pstats;
  std::map<long long, int> tune;          // (dtype, pass, N) -> launch variant
  std::map<std::string, bool> tuned_shapes;
  EnsPlan* ens = nullptr;
  // learned padding model: FP32 master parameters, Adam moments, gradient,
  // BF16 copies
  Buf mlp_p, mlp_m, mlp_v, mlp_g, mlp_wb;
  bool mlp_ready = false;
  int mlp_step = 0;
};

namespace {

int fail(scarl_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(ctx, SCARL_EDEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define RC(call)                     \
  do {                               \
    int r_ = (call);                 \
    if (r_ != SCARL_OK) return r_;   \
  } while (0)

int ensure(scarl_ctx* ctx, Buf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.n >= bytes) return SCARL_OK;
  const size_t want = bytes;
  if (ctx->used - b.n + want > ctx->budget)
    return fail(ctx, SCARL_ENOMEM, "device memory budget exceeded (" + std::to_string(want) + " bytes requested)");
  if (b.p) {
    cudaFree(b.p);
    ctx->used -= b.n;
    b.p = nullptr;
    b.n = 0;
  }
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return fail(ctx, SCARL_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  b.n = want;
  ctx->used += want;
  return SCARL_OK;
}

void release(scarl_ctx* ctx, Buf& b) {
  if (b.p) {
    cudaFree(b.p);
    ctx->used -= b.n;
  }
  b.p = nullptr;
  b.n = 0;
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool is_pinned_host(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Pinned host staging for small tables; waits for the previous upload.
int pinned(scarl_ctx* ctx, size_t bytes, void** out) {
  if (ctx->pin_ev) CK(cudaEventSynchronize(ctx->pin_ev));
  if (ctx->pin_n < bytes) {
    if (ctx->pin) cudaFreeHost(ctx->pin);
    ctx->pin = nullptr;
    ctx->pin_n = 0;
    CK(cudaMallocHost(&ctx->pin, bytes));
    ctx->pin_n = bytes;
  }
  *out = ctx->pin;
  return SCARL_OK;
}

int upload_pinned(scarl_ctx* ctx, void* dst, size_t bytes) {
  CK(cudaMemcpyAsync(dst, ctx->pin, bytes, cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d += bytes;
  if (!ctx->pin_ev) CK(cudaEventCreateWithFlags(&ctx->pin_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ctx->pin_ev, ctx->stream));
  return SCARL_OK;
}

// ---- profiling: events around each launch while enabled ----
cudaEvent_t pool_event(scarl_ctx* ctx) {
  if (!ctx->pool.empty()) {
    cudaEvent_t e = ctx->pool.back();
    ctx->pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

struct Prof {
  scarl_ctx* c;
  bool on;
  Mark m;
  Prof(scarl_ctx* ctx, const char* name, int nlaunch = 1) : c(ctx), on(ctx->profile) {
    c->launches += nlaunch;
    if (on) {
      m.name = name;
      m.a = pool_event(c);
      m.b = pool_event(c);
      cudaEventRecord(m.a, c->stream);
    }
  }
  ~Prof() {
    if (on) {
      cudaEventRecord(m.b, c->stream);
      c->marks.push_back(m);
    }
  }
};

void flush_marks(scarl_ctx* ctx) {
  if (ctx->marks.empty()) return;
  cudaEventSynchronize(ctx->marks.back().b);
  for (Mark& m : ctx->marks) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, m.a, m.b);
    auto it = ctx->pstats.find(m.name);
    if (it == ctx->pstats.end()) {
      ctx->porder.push_back(m.name);
      ctx->pstats[m.name] = {0.0, 0};
    }
    ctx->pstats[m.name].first += ms;
    ctx->pstats[m.name].second += 1;
    ctx->pool.push_back(m.a);
    ctx->pool.push_back(m.b);
  }
  ctx->marks.clear();
}

int begin(scarl_ctx* ctx) {
  if (!ctx) return SCARL_EINVAL;
  CK(cudaSetDevice(ctx->device));
  return SCARL_OK;
}

// Output destination on the device: the caller's pointer or the staging
// buffer, copied back by finish_out.
int out_dev(scarl_ctx* ctx, void* user, size_t bytes, void** dev, bool* host) {
  if (!user) return fail(ctx, SCARL_EINVAL, "null output pointer");
  *host = !is_device_ptr(user);
  if (!*host) {
    *dev = user;
    return SCARL_OK;
  }
  RC(ensure(ctx, ctx->stage_out, bytes));
  *dev = ctx->stage_out.p;
  return SCARL_OK;
}

// Reads and clears the device status word (the stream must be idle).
int check_status(scarl_ctx* ctx) {
  if (!ctx->status.p) return SCARL_OK;
  int st = 0;
  CK(cudaMemcpy(&st, ctx->status.p, sizeof st, cudaMemcpyDeviceToHost));
  if (st == 0) return SCARL_OK;
  CK(cudaMemset(ctx->status.p, 0, sizeof st));
  return fail(ctx, SCARL_ETIMEOUT, "a bounded tensor-core or copy wait expired; the output is invalid");
}

// Device -> pageable host copy through the pinned ring: the DMA fills the
// next slots while the host threads move a finished slot into the caller's
// memory (a direct copy into pageable memory runs at a fraction of the link
// rate, and into a fresh allocation it also takes every page fault on one
// thread).  A piece is h runs of w <= kRingChunk bytes, `pitch` apart, from
// byte offset off of both the device and the host buffer; its copy waits for
// the event `after` when one is given.
struct RingPiece {
  size_t off, w, h;
  cudaEvent_t after;
};

// The ring's slots, their events (the last DMA into or out of each slot) and
// the host copy threads, created on first use.
int ring_init(scarl_ctx* ctx) {
  if (!ctx->ring) CK(cudaMallocHost((void**)&ctx->ring, kRingSlots * kRingChunk));
  for (cudaEvent_t& e : ctx->ring_ev)
    if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (!ctx->hpool) {
    // SCARL_HOST_COPY_THREADS (copy threads including the caller), else up
    // to 12 of the host's hardware threads
    const unsigned hc = std::thread::hardware_concurrency();
    int n = (int)std::min(12u, std::max(hc, 1u));
    if (const char* v = std::getenv("SCARL_HOST_COPY_THREADS")) n = std::max(1, std::min(64, std::atoi(v)));
    ctx->hpool = new HostPool(n - 1);
  }
  return SCARL_OK;
}

// dst[a, b) = src[a, b) for the part of [0, len) that pool part p owns.
void pool_memcpy(HostPool* pool, char* dst, const char* src, size_t len) {
  const int parts = pool->parts();
  const size_t part = ((len + parts - 1) / parts + 63) / 64 * 64;
  pool->run([&](int p) {
    const size_t a = std::min(len, (size_t)p * part), b = std::min(len, a + part);
    if (b > a) std::memcpy(dst + a, src + a, b - a);
  });
}

int ring_copy(scarl_ctx* ctx, void* user, const void* dev, size_t pitch, const std::vector<RingPiece>& pieces,
              cudaStream_t s) {
  RC(ring_init(ctx));
  char* dst = static_cast<char*>(user);
  const char* src = static_cast<const char*>(dev);
  const size_t np = pieces.size();
  auto enqueue = [&](size_t i) -> int {
    const RingPiece& q = pieces[i];
    char* slot = ctx->ring + (i % kRingSlots) * kRingChunk;
    CK(cudaStreamWaitEvent(s, ctx->ring_ev[i % kRingSlots], 0));  // an earlier upload may still read it
    if (q.after) CK(cudaStreamWaitEvent(s, q.after, 0));
    if (q.h == 1) CK(cudaMemcpyAsync(slot, src + q.off, q.w, cudaMemcpyDeviceToHost, s));
    else CK(cudaMemcpy2DAsync(slot, q.w, src + q.off, pitch, q.w, q.h, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(ctx->ring_ev[i % kRingSlots], s));
    return SCARL_OK;
  };
  for (size_t i = 0; i < std::min(np, (size_t)kRingSlots); ++i) RC(enqueue(i));
  size_t total = 0;
  for (size_t i = 0; i < np; ++i) {
    const RingPiece& q = pieces[i];
    CK(cudaEventSynchronize(ctx->ring_ev[i % kRingSlots]));
    const char* from = ctx->ring + (i % kRingSlots) * kRingChunk;
    const size_t len = q.w * q.h;
    const int parts = ctx->hpool->parts();
    const size_t part = ((len + parts - 1) / parts + 63) / 64 * 64;
    ctx->hpool->run([&](int p) {
      // packed bytes [a, b) of the slot, run by run
      size_t a = std::min(len, (size_t)p * part);
      const size_t b = std::min(len, a + part);
      while (a < b) {
        const size_t r = a / q.w, x = a % q.w, n = std::min(b - a, q.w - x);
        std::memcpy(dst + q.off + r * pitch + x, from + a, n);
        a += n;
      }
    });
    total += len;
    if (i + kRingSlots < np) RC(enqueue(i + kRingSlots));
  }
  ctx->d2h += total;
  return SCARL_OK;
}

// Host -> device copy of a caller's buffer on the context's stream.  Pageable
// buffers of kRingMin bytes and more go through the pinned ring: host threads
// fill a slot while the DMA empties the previous ones.
int copy_in(scarl_ctx* ctx, void* dst, const void* user, size_t bytes) {
  if (bytes < kRingMin || is_pinned_host(user)) {
    CK(cudaMemcpyAsync(dst, user, bytes, cudaMemcpyHostToDevice, ctx->stream));
    ctx->h2d += bytes;
    return SCARL_OK;
  }
  RC(ring_init(ctx));
  const char* src = static_cast<const char*>(user);
  char* d = static_cast<char*>(dst);
  for (size_t off = 0, i = 0; off < bytes; off += kRingChunk, ++i) {
    const int slot = (int)(i % kRingSlots);
    const size_t len = std::min(kRingChunk, bytes - off);
    char* sl = ctx->ring + slot * kRingChunk;
    CK(cudaEventSynchronize(ctx->ring_ev[slot]));  // the slot's last DMA is done
    pool_memcpy(ctx->hpool, sl, src + off, len);
    CK(cudaMemcpyAsync(d + off, sl, len, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->ring_ev[slot], ctx->stream));
  }
  ctx->h2d += bytes;
  return SCARL_OK;
}

// Contiguous bytes as ring pieces of at most one slot each.
std::vector<RingPiece> ring_contiguous(size_t bytes) {
  std::vector<RingPiece> v;
  for (size_t off = 0; off < bytes; off += kRingChunk) v.push_back({off, std::min(kRingChunk, bytes - off), 1, nullptr});
  return v;
}

// Rows [y0, y1) of planes [z0, z1) (x rows of `row` bytes, planes of `plane`
// bytes) as ring pieces that wait for event e: whole row runs of several
// planes per piece, or parts of one plane's run when a run exceeds a slot.
void ring_box(std::vector<RingPiece>& v, size_t row, size_t plane, int y0, int y1, int z0, int z1,
              cudaEvent_t e) {
  if (y1 <= y0 || z1 <= z0) return;
  const size_t w = (size_t)(y1 - y0) * row;
  if (w <= kRingChunk) {
    const int per = (int)std::max<size_t>(1, kRingChunk / w);
    for (int z = z0; z < z1; z += per)
      v.push_back({(size_t)z * plane + (size_t)y0 * row, w, (size_t)std::min(per, z1 - z), e});
  } else {
    const int per = (int)std::max<size_t>(1, kRingChunk / row);
    for (int z = z0; z < z1; ++z)
      for (int y = y0; y < y1; y += per)
        v.push_back({(size_t)z * plane + (size_t)y * row, (size_t)std::min(per, y1 - y) * row, 1, e});
  }
}

int finish_out(scarl_ctx* ctx, void* user, const void* dev, size_t bytes, bool host) {
  if (host) {
    if (bytes >= kRingMin && !is_pinned_host(user)) {
      RC(ring_copy(ctx, user, dev, 0, ring_contiguous(bytes), ctx->stream));
    } else {
      CK(cudaMemcpyAsync(user, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
      ctx->d2h += bytes;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    RC(check_status(ctx));
  }
  CK(cudaGetLastError());
  return SCARL_OK;
}

// Output copied back in boxes while later tiles are generated.  Tiles run
// x fastest, then y, then z; with ystart(ty) = (Np_y - Np_ovlp_y) ty
// (ystart(0) = 0, ystart(Ty) = L_y) and zstart likewise, the box
// [ystart(ty), ystart(ty + 1)) x [zstart(tz), zstart(tz + 1)) (all x) is only
// covered by tile rows (ty, tz), (ty - 1, tz), (ty, tz - 1) and
// (ty - 1, tz - 1), so it is final once row (ty, tz) is blended.  Its
// device -> host copy (one strided 2D copy: a run of whole y rows per z
// plane) runs on a second stream that waits for the row.
struct SlabCopier {
  scarl_ctx* ctx = nullptr;
  char* user = nullptr;
  const char* dev = nullptr;
  size_t row = 0;    // bytes of one x row
  size_t plane = 0;  // bytes of one z plane
  int nev = 0;
  bool on = false;
};

int slab_begin(scarl_ctx* ctx, SlabCopier& c, void* user, const void* dev, size_t row, int Ly) {
  c.ctx = ctx;
  c.user = static_cast<char*>(user);
  c.dev = static_cast<const char*>(dev);
  c.row = row;
  c.plane = row * (size_t)Ly;
  c.on = true;
  if (!ctx->copy_stream) CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  return SCARL_OK;
}

// Rows [y0, y1) of planes [z0, z1) are final once the work queued so far on
// the context's stream completes.
int slab_copy(SlabCopier& c, int y0, int y1, int z0, int z1) {
  scarl_ctx* ctx = c.ctx;
  if (!c.on || y1 <= y0 || z1 <= z0) return SCARL_OK;
  if ((int)ctx->slab_ev.size() <= c.nev) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->slab_ev.push_back(e);
  }
  cudaEvent_t e = ctx->slab_ev[c.nev++];
  CK(cudaEventRecord(e, ctx->stream));
  CK(cudaStreamWaitEvent(ctx->copy_stream, e, 0));
  const size_t o = (size_t)z0 * c.plane + (size_t)y0 * c.row, w = (size_t)(y1 - y0) * c.row;
  CK(cudaMemcpy2DAsync(c.user + o, c.plane, c.dev + o, c.plane, w, (size_t)(z1 - z0),
                       cudaMemcpyDeviceToHost, ctx->copy_stream));
  ctx->d2h += w * (size_t)(z1 - z0);
  return SCARL_OK;
}

// Waits for every queued copy (also on error paths: the copies write the
// caller's memory).
int slab_end(SlabCopier& c) {
  scarl_ctx* ctx = c.ctx;
  if (!c.on) return SCARL_OK;
  c.on = false;
  CK(cudaStreamSynchronize(ctx->copy_stream));
  return SCARL_OK;
}

// The context's device status word (allocated and cleared on first use).
int ensure_status(scarl_ctx* ctx) {
  if (!ctx->status.p) {
    RC(ensure(ctx, ctx->status, 16));
    CK(cudaMemset(ctx->status.p, 0, 16));
  }
  return SCARL_OK;
}

// dtype argument of the padded generator: SCARL_F32 / SCARL_F64, optionally
// SCARL_F32 | SCARL_SPLIT_BF16 (or SCARL_SPLIT_BF16_X).
int parse_dtype(scarl_ctx* ctx, int dtype, int* dt, int* split) {
  // bit 0: pass 1's z DFT on the tensor cores; bit 1: pass 3's x DFT too
  *split = (dtype & SCARL_SPLIT_BF16_X) ? 3 : (dtype & SCARL_SPLIT_BF16) ? 1 : 0;
  *dt = dtype & ~(SCARL_SPLIT_BF16 | SCARL_SPLIT_BF16_X);
  if (*dt != SCARL_F32 && *dt != SCARL_F64)
    return fail(ctx, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64 (SCARL_F32 | SCARL_SPLIT_BF16)");
  if (*split && *dt != SCARL_F32) return fail(ctx, SCARL_EINVAL, "SCARL_SPLIT_BF16 applies to SCARL_F32 only");
  return SCARL_OK;
}

// Input on the device: the caller's pointer or a copy in buf.
int in_dev(scarl_ctx* ctx, Buf& buf, const void* user, size_t bytes, const void** dev) {
  if (!user) {
    *dev = nullptr;
    return SCARL_OK;
  }
  if (is_device_ptr(user)) {
    *dev = user;
    return SCARL_OK;
  }
  RC(ensure(ctx, buf, bytes));
  RC(copy_in(ctx, buf.p, user, bytes));
  *dev = buf.p;
  return SCARL_OK;
}

int default_pad(int Np) {
  int p = 1;
  while (p < 2 * Np) p <<= 1;
  return p;
}
int round_up(int a, int m) { return (a + m - 1) / m * m; }

// e^{2 pi i m / P}, m < P, rounded from long double.
int twiddles(scarl_ctx* ctx, int P, int dt, const void** out) {
  const long long key = (long long)P * 16 + dt;
  auto it = ctx->twiddles.find(key);
  if (it != ctx->twiddles.end()) {
    *out = it->second.p;
    return SCARL_OK;
  }
  Buf b;
  RC(ensure(ctx, b, (size_t)P * 2 * dt));
  std::vector<double> d(2 * (size_t)P);
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int m = 0; m < P; ++m) {
    const long double a = 2.0L * pi * (long double)m / (long double)P;
    d[2 * m] = (double)cosl(a);
    d[2 * m + 1] = (double)sinl(a);
  }
  if (dt == 8) {
    CK(cudaMemcpy(b.p, d.data(), d.size() * 8, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(d.begin(), d.end());
    CK(cudaMemcpy(b.p, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
  }
  ctx->twiddles[key] = b;
  *out = b.p;
  return SCARL_OK;
}

double freq(int k, int P, double dx) {
  const int s = (2 * k <= P) ? k : k - P;
  return (double)s / ((double)P * dx);
}

// Spectrum tables and the FP64 spectral normalisation of one padded grid.
int padded_plan(scarl_ctx* ctx, int dt, const int P[3], const double dx[3],
                const double corrL[3], int corrMod, double nu, int normalise,
                PaddedPlan** out) {
  char key[512];
  std::snprintf(key, sizeof key, "%d|%d,%d,%d|%a,%a,%a|%a,%a,%a|%d|%a|%d", dt, P[0], P[1], P[2],
                dx[0], dx[1], dx[2], corrL[0], corrL[1], corrL[2], corrMod, nu, normalise);
  auto it = ctx->plans.find(key);
  if (it != ctx->plans.end()) {
    *out = &it->second;
    return SCARL_OK;
  }
  PaddedPlan pl;
  pl.dt = dt;
  const int Hx = P[0] / 2 + 1;
  const int n[3] = {Hx, P[1], P[2]};
  std::vector<double> r[3];
  double craw2 = 0.0;
  if (corrMod == SCARL_CM_GAUSSIAN) {
    pl.amp = AMP_SEPARABLE;
    for (int d = 0; d < 3; ++d) {
      const double dk = 1.0 / ((double)P[d] * dx[d]);
      r[d].resize(n[d]);
      for (int k = 0; k < n[d]; ++k) {
        const double f = freq(k, P[d], dx[d]);
        r[d][k] = std::sqrt(corrL[d] * dk) * std::exp(-M_PI * corrL[d] * corrL[d] * f * f / 2.0);
      }
    }
  } else {
    const double v = (corrMod == SCARL_CM_EXPONENTIAL) ? 0.5 : nu;
    const double sc = std::tgamma(v) / (2.0 * std::sqrt(M_PI) * std::tgamma(v + 0.5));
    double a[3], dk3 = 1.0;
    for (int d = 0; d < 3; ++d) {
      a[d] = corrL[d] * sc;
      dk3 *= 1.0 / ((double)P[d] * dx[d]);
    }
    const double C = 8.0 * std::pow(M_PI, 1.5) * std::tgamma(v + 1.5) / std::tgamma(v) * a[0] * a[1] * a[2];
    craw2 = C * dk3;
    pl.expo = -(v + 1.5) / 2.0;
    pl.amp = (v == 0.5) ? AMP_RECIP : AMP_POW;
    for (int d = 0; d < 3; ++d) {
      r[d].resize(n[d]);
      for (int k = 0; k < n[d]; ++k) {
        const double f = freq(k, P[d], dx[d]);
        r[d][k] = 4.0 * M_PI * M_PI * a[d] * a[d] * f * f;
      }
    }
  }
  // FP64 normalisation sum on the GPU over the full periodic grid.
  double norm = 1.0;
  if (normalise) {
    Buf t64;
    const size_t tot = (size_t)n[0] + n[1] + n[2];
    RC(ensure(ctx, t64, tot * 8));
    std::vector<double> h;
    h.insert(h.end(), r[0].begin(), r[0].end());
    h.insert(h.end(), r[1].begin(), r[1].end());
    h.insert(h.end(), r[2].begin(), r[2].end());
    CK(cudaMemcpy(t64.p, h.data(), tot * 8, cudaMemcpyHostToDevice));
    const double* d0 = (const double*)t64.p;
    const double* d1 = d0 + n[0];
    const double* d2 = d1 + n[1];
    GenArgs ga;
    std::memset(&ga, 0, sizeof ga);
    for (int d = 0; d < 3; ++d) ga.P[d] = P[d];
    ga.Hx = Hx;
    ga.amp = pl.amp;
    ga.expo = pl.expo;
    ga.qx = d0; ga.qy = d1; ga.qz = d2;
    const int nb = spectrum_sum_blocks();
    RC(ensure(ctx, ctx->part, (size_t)nb * 8));
    {
      Prof pr(ctx, "spectrum_sum");
      CK(launch_spectrum_sum(ga, d0, d1, d2, craw2, (double*)ctx->part.p, nb, ctx->stream));
    }
    std::vector<double> parts(nb);
    CK(cudaMemcpyAsync(parts.data(), ctx->part.p, (size_t)nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    release(ctx, t64);
    norm = 0.0;
    for (double p : parts) norm += p;
    if (!(norm > 0.0)) return fail(ctx, SCARL_EINVAL, "spectrum sums to zero on this grid");
  }
  pl.norm = norm;
  // Device tables in the pass precision.
  const double inv = 1.0 / std::sqrt(norm);
  std::vector<double> tab;
  std::vector<size_t> off(6, 0);
  auto push = [&](int slot, const std::vector<double>& v) {
    off[slot] = tab.size();
    tab.insert(tab.end(), v.begin(), v.end());
  };
  std::vector<double> ax(Hx);
  for (int k = 0; k < Hx; ++k) {
    const double g = (k == 0 || 2 * k == P[0]) ? 1.0 : M_SQRT1_2;
    ax[k] = (pl.amp == AMP_SEPARABLE ? r[0][k] : std::sqrt(craw2)) * g * inv;
  }
  push(0, ax);
  if (pl.amp == AMP_SEPARABLE) {
    push(1, r[1]);
    push(2, r[2]);
  } else {
    push(3, r[0]);
    push(4, r[1]);
    push(5, r[2]);
  }
  RC(ensure(ctx, pl.tabs, tab.size() * dt));
  if (dt == 8) {
    CK(cudaMemcpy(pl.tabs.p, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(tab.begin(), tab.end());
    CK(cudaMemcpy(pl.tabs.p, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
  }
  for (int s = 0; s < 6; ++s) pl.t[s] = (const char*)pl.tabs.p + off[s] * dt;
  if (pl.amp == AMP_SEPARABLE) pl.t[3] = pl.t[4] = pl.t[5] = nullptr;
  else pl.t[1] = pl.t[2] = nullptr;
  auto ins = ctx->plans.emplace(key, pl);
  *out = &ins.first->second;
  return SCARL_OK;
}

int pm_powers(scarl_ctx* ctx, const uint32_t** out) {
  if (!ctx->pmpw.p) {
    RC(ensure(ctx, ctx->pmpw, 64 * 4));
    uint32_t h[64];
    uint64_t b = 16807;
    for (int i = 0; i < 64; ++i) {
      h[i] = (uint32_t)b;
      b = (b * b) % 2147483647ull;
    }
    CK(cudaMemcpy(ctx->pmpw.p, h, sizeof h, cudaMemcpyHostToDevice));
  }
  *out = (const uint32_t*)ctx->pmpw.p;
  return SCARL_OK;
}

// One Park-Miller step with Schrage's factorisation (SRC_F/normal_ScaRL.f90:827-833).
int32_t schrage(int32_t seed) {
  int32_t k = seed / 127773;
  seed = 16807 * (seed - k * 127773) - k * 2836;
  if (seed < 0) seed += 2147483647;
  return seed;
}

int run_passes(scarl_ctx* ctx, int dt, const GenArgs& a) {
  {
    const bool tc = a.split && dt == 4 && a.spec == SPEC_PHILOX && gen_z_tc_supported(a.P[2]);
    Prof p(ctx, tc ? "k_gen_z_tc" : "k_gen_z");
    CK(launch_gen_pass(dt, 1, a, ctx->stream));
  }
  {
    Prof p(ctx, "k_mid_y");
    CK(launch_gen_pass(dt, 2, a, ctx->stream));
  }
  {
    Prof p(ctx, c2r_x_tc_used(dt, a) ? "k_c2r_x_tc" : "k_c2r_x");
    CK(launch_gen_pass(dt, 3, a, ctx->stream));
  }
  return SCARL_OK;
}

// Passes 1 and 2 of k tiles of one sample (same padded grid and tile shape,
// one work buffer each) as one batched launch per pass: a pass over one tile
// ends with a partial last wave (the persistent tensor-core pass 1 of the
// 513^3 headline: 2700 items on 296 CTAs), over k tiles the waves pack.
// Each tile computes exactly what its single launch computes.  grp[j] must
// have its Philox schedule filled.
int run_passes12_batched(scarl_ctx* ctx, int dt, const GenArgs* grp, int k) {
  const GenArgs& a0 = grp[0];
  const bool tc = a0.split && dt == 4 && a0.spec == SPEC_PHILOX && gen_z_tc_supported(a0.P[2]);
  const int nb1 = tc ? gen_z_tc_items(a0) : gen_pass_blocks(dt, 1, a0.var[0], a0);
  const int nb2 = gen_pass_blocks(dt, 2, a0.var[1], a0);
  if (nb1 < 1 || nb2 < 1) return fail(ctx, SCARL_EUNSUPPORTED, "no batched launch for this grid");
  if ((long long)nb1 * k > 2147483647LL || (long long)nb2 * k > 2147483647LL)
    return fail(ctx, SCARL_EINVAL, "too many blocks for one batched launch");
  // [k GenArgs][k items][k + 1 pass-1 offsets][k + 1 pass-2 offsets]
  const size_t ab = (size_t)k * sizeof(GenArgs), bytes = ab + (size_t)(3 * k + 2) * sizeof(int);
  RC(ensure(ctx, ctx->targs, bytes));
  void* pin;
  RC(pinned(ctx, bytes, &pin));
  std::memcpy(pin, grp, ab);
  int* h = reinterpret_cast<int*>(static_cast<char*>(pin) + ab);
  for (int j = 0; j < k; ++j) h[j] = j;
  for (int j = 0; j <= k; ++j) {
    h[k + j] = j * nb1;
    h[2 * k + 1 + j] = j * nb2;
  }
  RC(upload_pinned(ctx, ctx->targs.p, bytes));
  const GenArgs* dargs = static_cast<const GenArgs*>(ctx->targs.p);
  const int* di = reinterpret_cast<const int*>(static_cast<const char*>(ctx->targs.p) + ab);
  const BatchMap m1{dargs, di, di + k, k, k * nb1};
  const BatchMap m2{dargs, di, di + 2 * k + 1, k, k * nb2};
  {
    Prof p(ctx, tc ? "k_gen_z_tc" : "k_gen_z");
    CK(tc ? launch_gen_z_tc_batch(a0, m1, ctx->stream) : launch_gen_pass_batch(dt, 1, a0.var[0], a0, m1, ctx->stream));
  }
  {
    Prof p(ctx, "k_mid_y");
    CK(launch_gen_pass_batch(dt, 2, a0.var[1], a0, m2, ctx->stream));
  }
  return SCARL_OK;
}

int check_grid(scarl_ctx* ctx, const int P[3], const int Np[3]) {
  for (int d = 0; d < 3; ++d) {
    if (Np[d] < 1) return fail(ctx, SCARL_EINVAL, "Np must be >= 1");
    if (!fft_length_supported(P[d]))
      return fail(ctx, SCARL_EUNSUPPORTED,
                  "padded grid lengths must lie in [8, 2048] and be a power of two or 3, 5 or 7 "
                  "times a power of two >= 16");
    if (P[d] < Np[d]) return fail(ctx, SCARL_EINVAL, "padded grid smaller than the tile");
  }
  return SCARL_OK;
}

long long tune_key(int dt, int pass, int N) { return ((long long)dt * 8 + pass) * 100000 + N; }

// Tuning cache file: lines "dtype pass N variant".
void tune_load(scarl_ctx* ctx, const char* path) {
  if (!path || !*path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  int dt, pass, N, v;
  while (std::fscanf(f, "%d %d %d %d", &dt, &pass, &N, &v) == 4)
    if ((dt == 4 || dt == 8) && pass >= 1 && pass <= 3 && v >= 0 && v < gen_variant_count(dt, pass))
      ctx->tune[tune_key(dt, pass, N)] = v;
  std::fclose(f);
}

void tune_save(scarl_ctx* ctx, const char* path) {
  if (!path || !*path) return;
  FILE* f = std::fopen(path, "w");
  if (!f) return;
  for (const auto& kv : ctx->tune) {
    const long long k = kv.first;
    const int N = (int)(k % 100000), dp = (int)(k / 100000);
    std::fprintf(f, "%d %d %d %d\n", dp / 8, dp % 8, N, kv.second);
  }
  std::fclose(f);
}

// Common GenArgs of the padded passes for one tile.
int gen_args(scarl_ctx* ctx, int dt, const int P[3], const int Np[3], GenArgs* a) {
  std::memset(a, 0, sizeof *a);
  for (int d = 0; d < 3; ++d) {
    a->P[d] = P[d];
    a->Nout[d] = Np[d];
  }
  a->Hx = P[0] / 2 + 1;
  a->Hpad = round_up(a->Hx, 16);
  RC(ensure_status(ctx));
  a->status = (int*)ctx->status.p;
  a->wait_test = ctx->wait_test;
  const size_t wbytes = (size_t)a->Hpad * P[1] * Np[2] * 2 * dt;
  RC(ensure(ctx, ctx->work, wbytes));
  a->work = ctx->work.p;
  RC(twiddles(ctx, P[2], dt, &a->tw_z));
  RC(twiddles(ctx, P[1], dt, &a->tw_y));
  RC(twiddles(ctx, P[0], dt, &a->tw_x));
  const int Nl[3] = {P[2], P[1], P[0] / 2};
  for (int p = 0; p < 3; ++p) {
    auto it = ctx->tune.find(tune_key(dt, p + 1, Nl[p]));
    a->var[p] = it == ctx->tune.end() ? gen_default_variant(dt, p + 1, *a) : it->second;
  }
  return SCARL_OK;
}

void set_plan(GenArgs* a, const PaddedPlan* pl) {
  a->spec = SPEC_PHILOX;
  a->amp = pl->amp;
  a->expo = pl->expo;
  a->ax = pl->t[0];
  a->ay = pl->t[1];
  a->az = pl->t[2];
  a->qx = pl->t[3];
  a->qy = pl->t[4];
  a->qz = pl->t[5];
}

// Times every valid launch variant of the three passes on grid P / tile Np
// (CUDA events, best of 3 after one warm-up) and keeps the fastest per
// (dtype, pass, line length) in the context.
int autotune_shape(scarl_ctx* ctx, int dt, const int P[3], const int Np[3], int corrMod, double nu,
                   const double xStep[3], const double corrL[3]) {
  PaddedPlan* pl;
  RC(padded_plan(ctx, dt, P, xStep, corrL, corrMod, nu, 1, &pl));
  GenArgs a;
  RC(gen_args(ctx, dt, P, Np, &a));
  set_plan(&a, pl);
  const size_t n = (size_t)Np[0] * Np[1] * Np[2];
  RC(ensure(ctx, ctx->tile, n * dt));
  a.epi.mode = 0;
  a.epi.out = ctx->tile.p;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int Nl[3] = {P[2], P[1], P[0] / 2};
  for (int pass = 1; pass <= 3; ++pass) {
    int best = 0;
    float best_ms = 1e30f;
    for (int v = 0; v < gen_variant_count(dt, pass); ++v) {
      GenArgs b = a;
      b.var[pass - 1] = v;
      cudaError_t e = launch_gen_pass(dt, pass, b, ctx->stream);
      if (e != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      float tmin = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0, ctx->stream);
        launch_gen_pass(dt, pass, b, ctx->stream);
        cudaEventRecord(e1, ctx->stream);
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        tmin = std::min(tmin, ms);
      }
      if (tmin < best_ms) {
        best_ms = tmin;
        best = v;
      }
    }
    ctx->tune[tune_key(dt, pass, Nl[pass - 1])] = best;
    a.var[pass - 1] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaGetLastError());
  return SCARL_OK;
}

// Marginal parameters exactly as SRC_F/main_ScaRL.f90:1371-1389.
int marginal_params(scarl_ctx* ctx, int margiFirst, double avg, double std_dev, double* s,
                    double* mu) {
  double nv, na;
  if (margiFirst == SCARL_FOM_GAUSSIAN) {
    nv = std_dev * std_dev;
    na = avg;
  } else if (margiFirst == SCARL_FOM_LOGNORMAL) {
    if (avg <= 0.0)
      return fail(ctx, SCARL_EINVAL, "ERROR - when using lognormal fieldAvg should be a positive number");
    const double cv = std_dev / avg;
    nv = std::log(1.0 + cv * cv);
    na = std::log(avg) - nv / 2.0;
  } else {
    return fail(ctx, SCARL_EINVAL, "First-order marginal not detected");
  }
  *s = std::sqrt(nv);
  *mu = na;
  return SCARL_OK;
}

// ---------------------------------------------------------------------------
// Ensembles of uneven grids: per pass, one batched launch per line length.
// ---------------------------------------------------------------------------
void ens_free(scarl_ctx* ctx) {
  EnsPlan* e = ctx->ens;
  if (!e) return;
  if (e->exec) cudaGraphExecDestroy(e->exec);
  for (Buf* b : {&e->work, &e->dargs, &e->dmap, &e->tmp}) release(ctx, *b);
  delete e;
  ctx->ens = nullptr;
}

// Block offsets of a group for launch variant v (host).
// Pass-1 groups of a split-precision plan whose z length has a tensor-core kernel.
bool ens_tc(const EnsPlan* e, const EnsGroup& g) {
  return e->split && e->dt == 4 && g.pass == 1 && gen_z_tc_supported(g.N);
}

cudaError_t ens_launch_group(const EnsPlan* e, const EnsGroup& g, int v, const BatchMap& m,
                             cudaStream_t s) {
  const GenArgs& rep = e->args[g.items[0]];
  if (ens_tc(e, g)) return launch_gen_z_tc_batch(rep, m, s);
  return launch_gen_pass_batch(e->dt, g.pass, v, rep, m, s);
}

int ens_starts(scarl_ctx* ctx, const EnsPlan* e, const EnsGroup& g, int v, std::vector<int>* st) {
  st->assign(1, 0);
  for (int i : g.items) {
    const int nb = ens_tc(e, g) ? gen_z_tc_items(e->args[i]) : gen_pass_blocks(e->dt, g.pass, v, e->args[i]);
    if (nb < 0) return SCARL_EUNSUPPORTED;
    if ((long long)st->back() + nb > 2147483647LL)
      return fail(ctx, SCARL_EINVAL, "ensemble too large for one launch");
    st->push_back(st->back() + nb);
  }
  return SCARL_OK;
}

// Uploads every group's item list and block offsets (after the stream has
// drained, since launches in flight read them).
int ens_maps(scarl_ctx* ctx, EnsPlan* e) {
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<int> h;
  std::vector<size_t> pos;
  for (EnsGroup& g : e->groups) {
    RC(ens_starts(ctx, e, g, g.var, &g.start));
    pos.push_back(h.size());
    h.insert(h.end(), g.items.begin(), g.items.end());
    h.insert(h.end(), g.start.begin(), g.start.end());
  }
  RC(ensure(ctx, e->dmap, h.size() * sizeof(int)));
  CK(cudaMemcpy(e->dmap.p, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
  ctx->h2d += h.size() * sizeof(int);
  const int* base = static_cast<const int*>(e->dmap.p);
  for (size_t k = 0; k < e->groups.size(); ++k) {
    EnsGroup& g = e->groups[k];
    g.m.args = static_cast<const GenArgs*>(e->dargs.p);
    g.m.items = base + pos[k];
    g.m.start = base + pos[k] + g.items.size();
    g.m.n = (int)g.items.size();
    g.m.total = g.start.back();
  }
  return SCARL_OK;
}

int ens_build(scarl_ctx* ctx, int dt, int split, int n, const int* Np, const double* dx,
              const double* cl, int corrMod, double nu, int policy, double tol,
              const std::string& key) {
  CK(cudaStreamSynchronize(ctx->stream));
  ens_free(ctx);
  RC(ensure_status(ctx));
  EnsPlan* e = new EnsPlan();
  ctx->ens = e;
  e->dt = dt;
  e->split = split != 0;
  e->n = n;
  e->args.resize(n);
  e->off.resize(n);
  std::vector<size_t> woff(n);
  size_t wtot = 0, tot = 0;
  for (int i = 0; i < n; ++i) {
    const int* np = Np + 3 * i;
    int P[3];
    if (pad_size(policy, corrMod, nu, cl + 3 * i, dx + 3 * i, np, tol, P) != SCARL_OK)
      return fail(ctx, SCARL_EINVAL, "no padded grid for realisation " + std::to_string(i));
    RC(check_grid(ctx, P, np));
    PaddedPlan* pl;
    RC(padded_plan(ctx, dt, P, dx + 3 * i, cl + 3 * i, corrMod, nu, 1, &pl));
    GenArgs& a = e->args[i];
    std::memset(&a, 0, sizeof a);
    for (int d = 0; d < 3; ++d) {
      a.P[d] = P[d];
      a.Nout[d] = np[d];
    }
    a.Hx = P[0] / 2 + 1;
    a.Hpad = round_up(a.Hx, 16);
    RC(twiddles(ctx, P[2], dt, &a.tw_z));
    RC(twiddles(ctx, P[1], dt, &a.tw_y));
    RC(twiddles(ctx, P[0], dt, &a.tw_x));
    set_plan(&a, pl);
    a.split = split;
    a.status = (int*)ctx->status.p;
    a.epi.mode = 0;
    woff[i] = wtot;
    wtot += ((size_t)a.Hpad * P[1] * np[2] * 2 * dt + 255) / 256 * 256;
    e->off[i] = tot;
    tot += (size_t)np[0] * np[1] * np[2];
  }
  RC(ensure(ctx, e->work, wtot));
  for (int i = 0; i < n; ++i) e->args[i].work = static_cast<char*>(e->work.p) + woff[i];
  e->total = tot;
  RC(ensure(ctx, e->dargs, (size_t)n * sizeof(GenArgs)));
  // groups: per pass, realisations by line length; largest realisations first
  // inside a group, groups with more blocks first
  for (int pass = 1; pass <= 3; ++pass) {
    std::map<int, std::vector<int>> by;
    for (int i = 0; i < n; ++i) {
      const GenArgs& a = e->args[i];
      by[pass == 1 ? a.P[2] : (pass == 2 ? a.P[1] : a.P[0] / 2)].push_back(i);
    }
    std::vector<EnsGroup> gs;
    for (auto& kv : by) {
      EnsGroup g;
      g.pass = pass;
      g.N = kv.first;
      g.items = kv.second;
      std::stable_sort(g.items.begin(), g.items.end(), [&](int x, int y) {
        const int* p = e->args[x].Nout;
        const int* q = e->args[y].Nout;
        return (long long)p[0] * p[1] * p[2] > (long long)q[0] * q[1] * q[2];
      });
      auto it = ctx->tune.find(tune_key(dt, pass, g.N));
      g.var = it == ctx->tune.end() ? gen_default_variant(dt, pass, e->args[g.items[0]]) : it->second;
      std::vector<int> st;
      if (ens_starts(ctx, e, g, g.var, &st) != SCARL_OK) g.var = 0;
      RC(ens_starts(ctx, e, g, g.var, &st));
      g.start = st;
      gs.push_back(g);
    }
    std::stable_sort(gs.begin(), gs.end(), [](const EnsGroup& x, const EnsGroup& y) {
      return x.start.back() > y.start.back();
    });
    e->groups.insert(e->groups.end(), gs.begin(), gs.end());
  }
  RC(ens_maps(ctx, e));
  e->key = key;
  return SCARL_OK;
}

const char* kBatchName[3] = {"k_gen_z_batch", "k_mid_y_batch", "k_c2r_x_batch"};

int ens_launch(scarl_ctx* ctx, EnsPlan* e) {
  for (EnsGroup& g : e->groups) {
    Prof p(ctx, ens_tc(e, g) ? "k_gen_z_tc_batch" : kBatchName[g.pass - 1]);
    CK(ens_launch_group(e, g, g.var, g.m, ctx->stream));
  }
  return SCARL_OK;
}

// Records the plan's launches into a CUDA graph; on any failure the plan
// keeps launching eagerly.
void ens_capture(scarl_ctx* ctx, EnsPlan* e) {
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGetLastError();
    e->graph_failed = true;
    return;
  }
  bool ok = true;
  for (EnsGroup& gr : e->groups)
    if (ens_launch_group(e, gr, gr.var, gr.m, ctx->stream) !=
        cudaSuccess)
      ok = false;
  if (cudaStreamEndCapture(ctx->stream, &g) != cudaSuccess) ok = false;
  if (ok && cudaGraphInstantiate(&e->exec, g, 0) != cudaSuccess) {
    e->exec = nullptr;
    ok = false;
  }
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    cudaGetLastError();
    e->graph_failed = true;
  }
}

// Times every valid variant of every group (CUDA events, best of 3 after a
// warm-up launch) and keeps the fastest.  The field is regenerated by the
// caller afterwards.
int ens_tune(scarl_ctx* ctx, EnsPlan* e) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  for (EnsGroup& g : e->groups) {
    if (ens_tc(e, g)) continue;  // the tensor-core pass has one launch shape
    int best = g.var;
    float best_ms = 1e30f;
    for (int v = 0; v < gen_variant_count(e->dt, g.pass); ++v) {
      std::vector<int> st;
      if (ens_starts(ctx, e, g, v, &st) != SCARL_OK) continue;
      CK(cudaStreamSynchronize(ctx->stream));
      RC(ensure(ctx, e->tmp, st.size() * sizeof(int)));
      CK(cudaMemcpy(e->tmp.p, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice));
      BatchMap m = g.m;
      m.start = static_cast<const int*>(e->tmp.p);
      m.total = st.back();
      if (ens_launch_group(e, g, v, m, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      float tmin = 1e30f;
      for (int rep_i = 0; rep_i < 3; ++rep_i) {
        CK(cudaEventRecord(e0, ctx->stream));
        CK(ens_launch_group(e, g, v, m, ctx->stream));
        CK(cudaEventRecord(e1, ctx->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        tmin = std::min(tmin, ms);
      }
      if (tmin < best_ms) {
        best_ms = tmin;
        best = v;
      }
    }
    g.var = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e->exec) {
    cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
  }
  return ens_maps(ctx, e);
}

// Blend tables of every tile: per tile, per axis lo[Np], hi[Np] (doubles)
// then flags[Np] (bytes), uploaded once.
struct BlendTabs {
  size_t dbl_off[64][3];
  size_t flag_off[64][3];
};

int upload_blend_tables(scarl_ctx* ctx, const scarl_layout& lay, int partitionType,
                        std::vector<BlendAxis>* axes) {
  // per tile and axis: lo, hi, sqrt(lo*hi) as doubles; sqrt(lo*hi) as
  // floats; flags as bytes -- three sections of one upload
  const int nb = lay.nb_tiles;
  size_t nsum = 0;
  for (int d = 0; d < 3; ++d) nsum += (size_t)lay.Np[d];
  const size_t dbytes = 3 * nsum * 8 * nb;
  const size_t fbytes = (nsum * 4 * nb + 15) / 16 * 16;
  const size_t bbytes = (nsum * nb + 15) / 16 * 16;
  const size_t total = dbytes + fbytes + bbytes;
  void* hp;
  RC(pinned(ctx, total, &hp));
  RC(ensure(ctx, ctx->tabs, total));
  double* hd = (double*)hp;
  float* hf = (float*)((char*)hp + dbytes);
  uint8_t* hb = (uint8_t*)hp + dbytes + fbytes;
  const char* dbase = (const char*)ctx->tabs.p;
  axes->resize((size_t)nb * 3);
  size_t od = 0, of = 0;
  for (int r = 0; r < nb; ++r) {
    int pos[3];
    get_topo_pos(r, lay.topo_shape, pos);
    for (int d = 0; d < 3; ++d) {
      const int Np = lay.Np[d];
      double* lo = hd + od;
      double* hi = lo + Np;
      double* sw = hi + Np;
      pou_axis_tables(Np, lay.Np_ovlp[d], pos[d], lay.topo_shape[d], partitionType, lo, hi);
      for (int x = 0; x < Np; ++x) {
        sw[x] = std::sqrt(lo[x] * hi[x]);
        hf[of + x] = (float)sw[x];
      }
      blend_axis_flags(Np, lay.Np_ovlp[d], pos[d], lay.topo_shape[d], hb + of);
      BlendAxis& ax = (*axes)[(size_t)r * 3 + d];
      ax.lo = (const double*)(dbase + od * 8);
      ax.hi = (const double*)(dbase + (od + Np) * 8);
      ax.sw64 = (const double*)(dbase + (od + 2 * (size_t)Np) * 8);
      ax.sw32 = (const float*)(dbase + dbytes + of * 4);
      ax.flags = (const uint8_t*)(dbase + dbytes + fbytes + of);
      od += 3 * (size_t)Np;
      of += (size_t)Np;
    }
  }
  RC(upload_pinned(ctx, ctx->tabs.p, total));
  return SCARL_OK;
}

int dct_table(scarl_ctx* ctx, int N, const double** out) {
  auto it = ctx->dct_tabs.find(N);
  if (it != ctx->dct_tabs.end()) {
    *out = (const double*)it->second.p;
    return SCARL_OK;
  }
  Buf b;
  RC(ensure(ctx, b, (size_t)4 * N * 8));
  std::vector<double> c(4 * (size_t)N);
  for (int m = 0; m < 4 * N; ++m) c[m] = std::cos(M_PI * (double)m / (2.0 * (double)N));
  CK(cudaMemcpy(b.p, c.data(), c.size() * 8, cudaMemcpyHostToDevice));
  ctx->dct_tabs[N] = b;
  *out = (const double*)b.p;
  return SCARL_OK;
}

// gen_std_gauss_FFT on the device into dev_out (Np doubles).
// full_z: the spectrum spans every kz (gen_Std_Gauss_FFT_MPI,
// SRC_F/fftw_ScaRL.f90:469-476), else the (Np/2)^3 octant.
int dct_tile(scarl_ctx* ctx, double* dev_out, const int Np[3], const double xRange[3],
             const double corrL[3], const double* phi_dev, const double* gamma_dev,
             uint32_t key, bool full_z = false) {
  DctArgs a;
  std::memset(&a, 0, sizeof a);
  size_t ktot = 1, t1n, t2n;
  std::vector<double> ex;
  for (int d = 0; d < 3; ++d) {
    a.Np[d] = Np[d];
    a.K[d] = (full_z && d == 2) ? Np[d] : Np[d] / 2;
    a.corrL[d] = corrL[d];
    ktot *= (size_t)a.K[d];
  }
  t1n = (size_t)Np[0] * a.K[1] * a.K[2];
  t2n = (size_t)Np[0] * Np[1] * a.K[2];
  // per-axis exp(-PI k^2) factors, SRC_F/fftw_ScaRL.f90:300-326
  std::vector<double> h;
  size_t off[3];
  for (int d = 0; d < 3; ++d) {
    off[d] = h.size();
    const double delta_x = xRange[d] / (double)(Np[d] - 1);
    const double k_max = 1.0 / delta_x;
    const double dk = k_max / (double)(Np[d] - 1);
    for (int i = 0; i < a.K[d]; ++i) {
      const double kp = (double)i * dk / corrL[d];
      h.push_back(std::exp(-kPiRef * (kp * kp)));
    }
  }
  h.push_back(0.0);
  void* hp;
  RC(pinned(ctx, h.size() * 8, &hp));
  std::memcpy(hp, h.data(), h.size() * 8);
  RC(ensure(ctx, ctx->dtabs, h.size() * 8));
  RC(upload_pinned(ctx, ctx->dtabs.p, h.size() * 8));
  const double* dt = (const double*)ctx->dtabs.p;
  a.cx = dt + off[0];
  a.cy = dt + off[1];
  a.cz = dt + off[2];
  RC(ensure(ctx, ctx->sk, std::max<size_t>(ktot, 1) * 8));
  RC(ensure(ctx, ctx->t1, std::max<size_t>(t1n, 1) * 8));
  RC(ensure(ctx, ctx->t2, std::max<size_t>(t2n, 1) * 8));
  a.sk = (double*)ctx->sk.p;
  a.t1 = (double*)ctx->t1.p;
  a.t2 = (double*)ctx->t2.p;
  a.out = dev_out;
  a.phi = phi_dev;
  a.gamma = gamma_dev;
  a.k0 = key;
  a.k1 = 0;
  a.stream = 0;
  for (int d = 0; d < 3; ++d) RC(dct_table(ctx, Np[d], &a.ctab[d]));
  Prof p(ctx, "k_dct_literal", 4);
  CK(launch_dct_literal(a, ctx->stream));
  return SCARL_OK;
}

// Literal Shino GenArgs for one tile (SRC_F/fftw_ScaRL.f90:157-255).
int shino_args(scarl_ctx* ctx, const int Np[3], const double xRange[3], const double corrL[3],
               int seed, GenArgs* a) {
  int sz_c[3], sz[3];
  double dk[3];
  shino_sizes(Np, xRange, corrL, sz_c, sz, dk);
  RC(check_grid(ctx, sz_c, Np));
  RC(gen_args(ctx, 8, sz_c, Np, a));
  a->spec = SPEC_SHINO;
  for (int d = 0; d < 3; ++d) {
    a->sz[d] = sz[d];
    a->de[d] = ((kPiRef * kPiRef) / 2.0) * (dk[d] * dk[d]);
  }
  a->shino_scale = std::sqrt(8.0);
  a->shino_f = 2.0 * std::sqrt((dk[0] * dk[1]) * dk[2]);
  const int32_t s0 = (int32_t)((uint32_t)seed + 1000000u);
  a->pm_s1 = (uint32_t)schrage(s0);
  RC(pm_powers(ctx, &a->pm_pw));
  return SCARL_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ---------------------------------------------------------------------------
// Learned padding: labels, features, the MLP's host side.
// ---------------------------------------------------------------------------
constexpr double kLearnTol = 0.01;       // covariance error the labels hold
constexpr double kLearnMargin = 0.25;    // safety margin on predictions (log2 units)

// Matern / Gaussian axis description for the label kernels.
PadLabelIn label_in(int corrMod, double nu, double ell_pts, int N) {
  PadLabelIn c;
  c.N = N;
  c.ell = ell_pts;
  if (corrMod == SCARL_CM_GAUSSIAN) {
    c.kind = 1;
    c.nu = 0.0;
    c.q = 0.0;
  } else {
    const double v = corrMod == SCARL_CM_EXPONENTIAL ? 0.5 : nu;
    const double a = ell_pts * std::tgamma(v) / (2.0 * std::sqrt(M_PI) * std::tgamma(v + 0.5));
    c.kind = 2;
    c.nu = v;
    c.q = 4.0 * M_PI * M_PI * a * a;
  }
  return c;
}

// Network inputs of one axis (16 values; the trained range is l/N in
// [0.01, 0.3], N in [64, 256], nu in [0.3, 1.5]).
void mlp_feat(int corrMod, double nu, double ell_pts, int N, float* f) {
  for (int i = 0; i < kMlpIn; ++i) f[i] = 0.f;
  const double r = ell_pts / (double)N;
  f[0] = (float)(4.0 * r);
  f[1] = (float)(std::log2(r) / 4.0);
  f[2] = (float)(std::log2((double)N) - 7.0);
  f[3] = (float)(std::log2(ell_pts) / 4.0);
  f[4] = corrMod == SCARL_CM_GAUSSIAN ? 1.f : 0.f;
  f[5] = corrMod == SCARL_CM_EXPONENTIAL ? 1.f : 0.f;
  f[6] = corrMod == SCARL_CM_VON_KARMAN ? 1.f : 0.f;
  f[7] = corrMod == SCARL_CM_VON_KARMAN ? (float)(nu - 0.9) : 0.f;
}

bool mlp_in_range(int corrMod, double nu, double ell_pts, int N) {
  const double r = ell_pts / (double)N;
  if (!(r >= 0.008 && r <= 0.32) || N < 48 || N > 320) return false;
  if (corrMod == SCARL_CM_VON_KARMAN && !(nu >= 0.28 && nu <= 1.55)) return false;
  return corrMod >= 1 && corrMod <= 3;
}

int mlp_alloc(scarl_ctx* ctx) {
  for (Buf* b : {&ctx->mlp_p, &ctx->mlp_m, &ctx->mlp_v, &ctx->mlp_g})
    RC(ensure(ctx, *b, (size_t)kMlpParams * 4));
  RC(ensure(ctx, ctx->mlp_wb, (size_t)kMlpParams * 2));
  return SCARL_OK;
}

// Inputs (FP32 host rows of 16) as BF16 on the device, in ctx->stage_in.
int mlp_inputs(scarl_ctx* ctx, const float* X, int n, const void** dev) {
  RC(ensure(ctx, ctx->stage_in2, (size_t)n * kMlpIn * 4));
  RC(ensure(ctx, ctx->stage_in, (size_t)n * kMlpIn * 2));
  CK(cudaMemcpyAsync(ctx->stage_in2.p, X, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d += (size_t)n * kMlpIn * 4;
  CK(launch_to_bf16((const float*)ctx->stage_in2.p, ctx->stage_in.p, n * kMlpIn, ctx->stream));
  ctx->launches += 1;
  *dev = ctx->stage_in.p;
  return SCARL_OK;
}

// ---------------------------------------------------------------------------
// HDF5 / XDMF output of a sample (SRC_F/write_output.f90).
// ---------------------------------------------------------------------------
std::string f25(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%25.10f", v);
  return b;
}

std::string dim_text(const int n[3]) {  // slowest first, SRC_F/write_output.f90:488-497
  return std::to_string(n[2]) + " " + std::to_string(n[1]) + " " + std::to_string(n[0]);
}

std::string pad5(int r) {  // num2str(rank, 5)
  char b[32];
  std::snprintf(b, sizeof b, "%05d", r);
  return b;
}

// write_XMF_elements (SRC_F/write_output.f90:455-559)
bool xmf_elements(const std::string& path, const std::string& h5name, const double xMin[3],
                  const double xMax[3], const int n[3], const std::string& ds, int prec) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  double st[3];
  for (int d = 0; d < 3; ++d) st[d] = (xMax[d] - xMin[d]) / (double)(n[d] - 1);
  const std::string dt = dim_text(n);
  std::fprintf(f, "<?xml version=\"1.0\" ?>\n<Xdmf Version=\"2.0\">\n <Domain>\n");
  std::fprintf(f, "   <DataItem Name=\"RF_1\" Format=\"HDF\" DataType=\"Float\" Precision=\"%d\" Dimensions=\"%s\">\n", prec, dt.c_str());
  std::fprintf(f, "        ./%s:/%s\n   </DataItem>\n", h5name.c_str(), ds.c_str());
  std::fprintf(f, "  <Grid GridType=\"Collection\" CollectionType=\"Spatial\">\n   <Grid Name=\"Group1\">\n");
  std::fprintf(f, "     <Topology TopologyType=\"3DCoRectMesh\" Dimensions=\"%s\"/>\n", dt.c_str());
  std::fprintf(f, "     <Geometry GeometryType=\"ORIGIN_DXDYDZ\">\n");
  std::fprintf(f, "   <DataItem Name=\"origin\" Format=\"XML\" DataType=\"Float\" Precision=\"8\" Dimensions=\"3\">\n");
  for (int d = 2; d >= 0; --d) std::fprintf(f, " %s\n", f25(xMin[d]).c_str());
  std::fprintf(f, "   </DataItem>\n   <DataItem Name=\"step\" Format=\"XML\" DataType=\"Float\" Precision=\"8\" Dimensions=\"3\">\n");
  for (int d = 2; d >= 0; --d) std::fprintf(f, " %s\n", f25(st[d]).c_str());
  std::fprintf(f, "   </DataItem>\n     </Geometry>\n");
  std::fprintf(f, "     <Attribute Name=\"RF1\" Center=\"Node\" AttributeType=\"Scalar\">\n       <DataItem Reference=\"XML\">\n");
  std::fprintf(f, "         /Xdmf/Domain/DataItem[@Name=\"RF_1\"]\n       </DataItem>\n     </Attribute>\n");
  std::fprintf(f, "   </Grid>\n  </Grid>\n </Domain>\n</Xdmf>\n");
  return std::fclose(f) == 0;
}

// write_XMF_global (SRC_F/write_output.f90:564-656)
bool xmf_global(const std::string& path, const std::vector<std::string>& h5list,
                const std::vector<std::array<double, 3>>& c0, const double xStep[3], const int n[3],
                int prec) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  const std::string dt = dim_text(n);
  const int np = (int)h5list.size();
  std::fprintf(f, "<?xml version=\"1.0\" ?>\n<Xdmf Version=\"2.0\">\n <Domain>\n");
  for (int i = 0; i < np; ++i) {
    std::fprintf(f, "   <DataItem Name=\"RF_1_p%d\" Format=\"HDF\" DataType=\"Float\" Precision=\"%d\" Dimensions=\"%s\">\n", i, prec, dt.c_str());
    std::fprintf(f, "        ./%s:/sample_1_p%d\n   </DataItem>\n", h5list[i].c_str(), i);
  }
  std::fprintf(f, "  <Grid GridType=\"Collection\" CollectionType=\"Spatial\">\n");
  for (int i = 0; i < np; ++i) {
    std::fprintf(f, "   <Grid Name=\"Proc_%d\">\n", i);
    std::fprintf(f, "     <Topology TopologyType=\"3DCoRectMesh\" Dimensions=\"%s\"/>\n", dt.c_str());
    std::fprintf(f, "     <Geometry GeometryType=\"ORIGIN_DXDYDZ\">\n");
    std::fprintf(f, "   <DataItem Name=\"origin\" Format=\"XML\" DataType=\"Float\" Precision=\"8\" Dimensions=\"3\">\n");
    for (int d = 2; d >= 0; --d) std::fprintf(f, " %s\n", f25(c0[i][d]).c_str());
    std::fprintf(f, "   </DataItem>\n   <DataItem Name=\"step\" Format=\"XML\" DataType=\"Float\" Precision=\"8\" Dimensions=\"3\">\n");
    for (int d = 2; d >= 0; --d) std::fprintf(f, " %s\n", f25(xStep[d]).c_str());
    std::fprintf(f, "   </DataItem>\n     </Geometry>\n");
    std::fprintf(f, "     <Attribute Name=\"RF_1\" Center=\"Node\" AttributeType=\"Scalar\">\n       <DataItem Reference=\"XML\">\n");
    std::fprintf(f, "         /Xdmf/Domain/DataItem[@Name=\"RF_1_p%d\"]\n       </DataItem>\n     </Attribute>\n", i);
    std::fprintf(f, "   </Grid>\n");
  }
  std::fprintf(f, "  </Grid>\n </Domain>\n</Xdmf>\n");
  return std::fclose(f) == 0;
}

// Root attributes of write_HDF5_attributes (SRC_F/write_output.f90:722-813),
// in its order.
std::vector<h5::Attr> sample_attrs(const scarl_sample* s, const scarl_layout& lay,
                                   const double xMaxEff[3]) {
  std::vector<h5::Attr> a;
  const int nb = lay.nb_tiles, ndim = 3, nmc = 1, method = SCARL_FFT, seed = s->seedBase;
  a.push_back(h5::attr_i32("nb_procs", &nb, 1, true));
  a.push_back(h5::attr_i32("nDim", &ndim, 1, true));
  a.push_back(h5::attr_i32("Nmc", &nmc, 1, true));
  a.push_back(h5::attr_i32("method", &method, 1, true));
  a.push_back(h5::attr_i32("seedStart", &seed, 1, true));
  a.push_back(h5::attr_i32("corrMod", &s->corrMod, 1, true));
  a.push_back(h5::attr_i32("margiFirst", &s->margiFirst, 1, true));
  a.push_back(h5::attr_i32("nFields", lay.topo_shape, 3));
  a.push_back(h5::attr_i32("Np", lay.Np, 3));
  a.push_back(h5::attr_i32("Np_ovlp", lay.Np_ovlp, 3));
  a.push_back(h5::attr_i32("L", lay.L, 3));
  double ov[3];
  for (int d = 0; d < 3; ++d) ov[d] = (double)(lay.Np_ovlp[d] - 1) * lay.xStep[d];  // main_ScaRL.f90:460
  a.push_back(h5::attr_f64("xMinGlob", s->xMinGlob, 3));
  a.push_back(h5::attr_f64("xMaxGlob", xMaxEff, 3));
  a.push_back(h5::attr_f64("xStep", lay.xStep, 3));
  a.push_back(h5::attr_f64("corrL", s->corrL, 3));
  a.push_back(h5::attr_f64("overlap", ov, 3));
  return a;
}

// "times" (ranks x labels, one rank here) and "time_labels" (20-character
// Fortran strings), write_time_on_hdf5 (SRC_F/write_output.f90:819-911).
void time_datasets(const char* labels, const double* times, int nt, std::vector<h5::Dataset>* ds) {
  if (nt <= 0 || !times) return;
  h5::Dataset t;
  t.name = "times";
  t.kind = h5::F64;
  t.dims = {1, (uint64_t)nt};
  t.nbytes = (uint64_t)nt * 8;
  std::vector<double> tv(times, times + nt);
  t.write = [tv](FILE* f) { return std::fwrite(tv.data(), 8, tv.size(), f) == tv.size(); };
  ds->push_back(t);
  h5::Dataset l;
  l.name = "time_labels";
  l.kind = h5::STR;
  l.strsize = 20;
  l.dims = {(uint64_t)nt};
  l.nbytes = (uint64_t)nt * 20;
  std::string lv((size_t)nt * 20, ' ');
  if (labels)
    for (int i = 0; i < nt; ++i)
      for (int c = 0; c < 20 && labels[i * 20 + c]; ++c) lv[(size_t)i * 20 + c] = labels[i * 20 + c];
  l.write = [lv](FILE* f) { return std::fwrite(lv.data(), 1, lv.size(), f) == lv.size(); };
  ds->push_back(l);
}

// Writes the block [o, o + n) of a column-major field of extent L to f,
// staging through pinned memory when the field is on the device.
bool write_block(scarl_ctx* ctx, FILE* f, const void* field, bool dev, int dt, const int L[3],
                 const int o[3], const int n[3]) {
  const size_t line = (size_t)n[0] * dt;
  const bool whole = o[0] == 0 && o[1] == 0 && o[2] == 0 && n[0] == L[0] && n[1] == L[1] && n[2] == L[2];
  if (!dev) {
    const char* p = static_cast<const char*>(field);
    if (whole) return std::fwrite(p, 1, line * n[1] * n[2], f) == line * n[1] * n[2];
    for (int z = 0; z < n[2]; ++z)
      for (int y = 0; y < n[1]; ++y) {
        const size_t at = ((size_t)(o[2] + z) * L[1] + (o[1] + y)) * L[0] + o[0];
        if (std::fwrite(p + at * dt, 1, line, f) != line) return false;
      }
    return true;
  }
  const size_t plane = line * n[1];
  const size_t zper = std::max<size_t>(1, ((size_t)64 << 20) / plane);
  void* pin;
  if (pinned(ctx, std::min<size_t>(zper, n[2]) * plane, &pin) != SCARL_OK) return false;
  for (int z0 = 0; z0 < n[2]; z0 += (int)zper) {
    const int nz = (int)std::min<size_t>(zper, (size_t)(n[2] - z0));
    for (int z = 0; z < nz; ++z) {
      const char* src = static_cast<const char*>(field) +
                        (((size_t)(o[2] + z0 + z) * L[1] + o[1]) * L[0] + o[0]) * dt;
      if (cudaMemcpy2DAsync(static_cast<char*>(pin) + (size_t)z * plane, line, src, (size_t)L[0] * dt,
                            line, n[1], cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
        return false;
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return false;
    ctx->d2h += plane * nz;
    if (std::fwrite(pin, 1, plane * nz, f) != plane * nz) return false;
  }
  return true;
}

// ===========================================================================
extern "C" {

const char* scarl_version(void) { return "scarl_b200 0.1 (sm_100a)"; }

int scarl_ctx_create(int device, size_t budget_bytes, scarl_ctx** out) {
  if (!out) return SCARL_EINVAL;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return SCARL_EDEVICE;
  }
  if (device < 0 || device >= n) return SCARL_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return SCARL_EDEVICE;
  scarl_ctx* c = new scarl_ctx();
  c->device = device;
  if (budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    budget_bytes = fr / 10 * 9;
  }
  c->budget = budget_bytes;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return SCARL_EDEVICE;
  }
  c->own_stream = true;
  tune_load(c, std::getenv("SCARL_TUNE_CACHE"));
  *out = c;
  return SCARL_OK;
}

int scarl_ctx_destroy(scarl_ctx* ctx) {
  if (!ctx) return SCARL_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  flush_marks(ctx);
  for (Buf* b : {&ctx->work, &ctx->targs, &ctx->tile, &ctx->stage_out, &ctx->stage_in, &ctx->stage_in2,
                 &ctx->tabs, &ctx->dtabs, &ctx->part, &ctx->t1, &ctx->t2, &ctx->sk, &ctx->pmpw,
                 &ctx->status, &ctx->mom})
    release(ctx, *b);
  for (auto& kv : ctx->plans) release(ctx, kv.second.tabs);
  for (auto& kv : ctx->twiddles) release(ctx, kv.second);
  for (auto& kv : ctx->dct_tabs) release(ctx, kv.second);
  ens_free(ctx);
  for (Buf* b : {&ctx->mlp_p, &ctx->mlp_m, &ctx->mlp_v, &ctx->mlp_g, &ctx->mlp_wb}) release(ctx, *b);
  for (cudaEvent_t e : ctx->pool) cudaEventDestroy(e);
  if (ctx->pin_ev) cudaEventDestroy(ctx->pin_ev);
  if (ctx->pin) cudaFreeHost(ctx->pin);
  for (cudaEvent_t e : ctx->slab_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->ring_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->ring) cudaFreeHost(ctx->ring);
  delete ctx->hpool;
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return SCARL_OK;
}

const char* scarl_last_error(const scarl_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int scarl_ctx_set_stream(scarl_ctx* ctx, void* s) {
  RC(begin(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  if (s) {
    ctx->stream = (cudaStream_t)s;
    ctx->own_stream = false;
  } else {
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  return SCARL_OK;
}

int scarl_sync(scarl_ctx* ctx) {
  RC(begin(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  RC(check_status(ctx));
  return SCARL_OK;
}

int scarl_tc_wait_test(scarl_ctx* ctx, int enable) {
  if (!ctx) return SCARL_EINVAL;
  ctx->wait_test = enable ? 1 : 0;
  return SCARL_OK;
}

int scarl_counters(scarl_ctx* ctx, long long* launches, unsigned long long* h2d_bytes,
                   unsigned long long* d2h_bytes) {
  if (!ctx) return SCARL_EINVAL;
  if (launches) *launches = ctx->launches;
  if (h2d_bytes) *h2d_bytes = ctx->h2d;
  if (d2h_bytes) *d2h_bytes = ctx->d2h;
  return SCARL_OK;
}

int scarl_autotune(scarl_ctx* ctx, int dtype, int corrMod, double nu, const int P[3],
                   const int Np[3], const double xStep[3], const double corrL[3],
                   const char* cache_path) {
  RC(begin(ctx));
  if (!P || !Np || !xStep || !corrL) return fail(ctx, SCARL_EINVAL, "null argument");
  if (dtype != SCARL_F32 && dtype != SCARL_F64) return fail(ctx, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64");
  RC(check_grid(ctx, P, Np));
  tune_load(ctx, cache_path);
  RC(autotune_shape(ctx, dtype, P, Np, corrMod, nu, xStep, corrL));
  tune_save(ctx, cache_path);
  return SCARL_OK;
}

int scarl_tune_get(scarl_ctx* ctx, int dtype, int pass, int N, int* variant) {
  if (!ctx || !variant || pass < 1 || pass > 3) return SCARL_EINVAL;
  auto it = ctx->tune.find(tune_key(dtype, pass, N));
  *variant = it == ctx->tune.end() ? -1 : it->second;
  return SCARL_OK;
}

int scarl_tune_set(scarl_ctx* ctx, int dtype, int pass, int N, int variant) {
  if (!ctx || pass < 1 || pass > 3 || (dtype != SCARL_F32 && dtype != SCARL_F64)) return SCARL_EINVAL;
  if (variant == -1) {  // forget the choice: the default variant runs again
    ctx->tune.erase(tune_key(dtype, pass, N));
    return SCARL_OK;
  }
  if (variant < 0 || variant >= gen_variant_count(dtype, pass)) return SCARL_EINVAL;
  ctx->tune[tune_key(dtype, pass, N)] = variant;
  return SCARL_OK;
}

int scarl_profile(scarl_ctx* ctx, int enable) {
  RC(begin(ctx));
  flush_marks(ctx);
  if (enable == 2) {  // reset
    ctx->pstats.clear();
    ctx->porder.clear();
    return SCARL_OK;
  }
  ctx->profile = enable != 0;
  return SCARL_OK;
}

int scarl_profile_read(scarl_ctx* ctx, int idx, char* name, size_t name_len, double* total_ms,
                       long long* launches) {
  RC(begin(ctx));
  flush_marks(ctx);
  if (idx < 0 || idx >= (int)ctx->porder.size()) return SCARL_EINVAL;
  const std::string& k = ctx->porder[idx];
  if (name && name_len) std::snprintf(name, name_len, "%s", k.c_str());
  if (total_ms) *total_ms = ctx->pstats[k].first;
  if (launches) *launches = ctx->pstats[k].second;
  return SCARL_OK;
}

// ---- host-only ----
int scarl_verify_inputs(const scarl_sample* s, int gen_meth, char* msg, size_t len) {
  if (!s) return SCARL_EINVAL;
  return verify_inputs(s, gen_meth, msg, len);
}

int scarl_decide_topo_shape(int nb_procs, const int L[3], const int Np_ovlp[3],
                            long long ppbi, int topo[3]) {
  if (nb_procs < 1 || !L || !Np_ovlp || !topo) return SCARL_EINVAL;
  decide_topo_shape(nb_procs, L, Np_ovlp, ppbi, topo);
  return SCARL_OK;
}

int scarl_get_topo_pos(int rank, const int shape[3], int pos[3]) {
  if (!shape || !pos || shape[0] < 1 || shape[1] < 1 || shape[2] < 1) return SCARL_EINVAL;
  get_topo_pos(rank, shape, pos);
  return SCARL_OK;
}

int scarl_get_topo_rank(const int shape[3], const int pos[3]) {
  if (!shape || !pos) return -1;
  return get_topo_rank(shape, pos);
}

int scarl_sample_layout(const scarl_sample* s, int gen_meth, int nb_procs, const int* topo_in,
                        scarl_layout* out) {
  if (!s || !out) return SCARL_EINVAL;
  return sample_layout(s, gen_meth, nb_procs, topo_in, out);
}

int scarl_tile_geometry(const scarl_layout* lay, const double xMin[3], int rank, scarl_tile* t) {
  if (!lay || !xMin || !t || rank < 0 || rank >= lay->nb_tiles) return SCARL_EINVAL;
  tile_geometry(lay, xMin, rank, t);
  return SCARL_OK;
}

int scarl_unity_partition_weights(const int Np[3], const int No[3], int partitionType,
                                  const int pos[3], const int shape[3], double* w) {
  if (!Np || !No || !pos || !shape || !w) return SCARL_EINVAL;
  unity_partition_weights(Np, No, partitionType, pos, shape, w);
  return SCARL_OK;
}

int scarl_shino_sizes(const int Np[3], const double xRange[3], const double corrL[3],
                      int sz_c[3], int sz_Sk[3], double delta_k[3]) {
  if (!Np || !xRange || !corrL || !sz_c || !sz_Sk || !delta_k) return SCARL_EINVAL;
  shino_sizes(Np, xRange, corrL, sz_c, sz_Sk, delta_k);
  return SCARL_OK;
}

int scarl_pad_size(int policy, int corrMod, double nu, const double corrL[3],
                   const double xStep[3], const int Np[3], double tol, int P[3]) {
  if (!corrL || !xStep || !Np || !P) return SCARL_EINVAL;
  return pad_size(policy, corrMod, nu, corrL, xStep, Np, tol, P);
}

double scarl_axis_correlation(int corrMod, double nu, double l, double r) {
  return axis_correlation(corrMod, nu, l, r);
}

int scarl_read_config(const char* path, int* gen_meth, int* c_info_file, int* d_sample,
                      int* one_file, int* one_hdf_ds, char* input_file, size_t len) {
  if (!path || !gen_meth || !c_info_file || !d_sample || !one_file || !one_hdf_ds) return SCARL_EINVAL;
  return read_config(path, gen_meth, c_info_file, d_sample, one_file, one_hdf_ds, input_file, len);
}

int scarl_read_extra_config(const char* path, int* found, int topo[3]) {
  if (!path || !found || !topo) return SCARL_EINVAL;
  return read_extra_config(path, found, topo);
}

int scarl_read_input(const char* path, char* folder, size_t flen, int* nSamples,
                     scarl_sample* samples, int max_samples) {
  if (!path || !nSamples) return SCARL_EINVAL;
  return read_input(path, folder, flen, nSamples, samples, max_samples);
}

int scarl_read_input_sem(const char* folder, char* out_folder, size_t flen, int* nSamples,
                         scarl_sample* samples, int max_samples) {
  if (!nSamples) return SCARL_EINVAL;
  return read_input_sem(folder, out_folder, flen, nSamples, samples, max_samples);
}

int scarl_rebuild_corrL(const double* SkTot, const int L[3], const double xStep[3],
                        double corrL_out[3]) {
  if (!SkTot || !L || !xStep || !corrL_out) return SCARL_EINVAL;
  int off = 0;
  for (int d = 0; d < 3; ++d) {
    const int nk = L[d] / 2;
    if (nk < 1) return SCARL_EINVAL;
    double s = 0.0;
    for (int t = 0; t < nk; ++t) s += SkTot[off + t];
    corrL_out[d] = 2.0 * (s - ((SkTot[off] + SkTot[off + nk - 1]) / 2.0)) * xStep[d];
    off += nk;
  }
  return SCARL_OK;
}

// ---- Stat_ScaRL front end ----
int scarl_stat_file(scarl_ctx* ctx, const char* res_path, const char* dset_name, int calc_corrL,
                    double* globalAvg, double* globalStdDev, double* corrL_out) {
  RC(begin(ctx));
  if (!res_path || !dset_name || !globalAvg || !globalStdDev) return fail(ctx, SCARL_EINVAL, "null argument");
  h5::RObject root;
  std::vector<h5::RObject> ds;
  std::string err;
  int rc = h5::read_file(res_path, &root, &ds, &err);
  if (rc) return fail(ctx, rc == 5 ? SCARL_EUNSUPPORTED : (rc == 6 ? SCARL_EIO : SCARL_EINVAL), err);
  const h5::RObject* d = nullptr;
  for (const auto& o : ds)
    if (o.name == dset_name) d = &o;
  if (!d || !d->is_dataset || d->kind == h5::STR)
    return fail(ctx, SCARL_EINVAL, std::string("no numeric dataset ") + dset_name + " in " + res_path);
  if (d->dims.size() != 3) return fail(ctx, SCARL_EUNSUPPORTED, "the sample dataset must be 3D");
  auto find = [&](const char* n) -> const h5::Attr* {
    for (const auto& a : root.attrs)
      if (a.name == n) return &a;
    return nullptr;
  };
  // read_RF_h5_File_Attributes (SRC_F/Stat_ScaRL/main_Stat.f90:133-194)
  const char* needed[] = {"nb_procs", "nDim", "Nmc", "method", "seedStart", "corrMod", "margiFirst",
                          "nFields", "Np", "Np_ovlp", "L", "xMinGlob", "xMaxGlob", "xStep", "corrL",
                          "overlap"};
  for (const char* n : needed)
    if (!find(n)) return fail(ctx, SCARL_EINVAL, std::string("attribute ") + n + " missing in " + res_path);
  const h5::Attr* xs = find("xStep");
  if (xs->kind != h5::F64 || xs->data.size() != 24) return fail(ctx, SCARL_EINVAL, "xStep must hold 3 doubles");
  double xStep[3];
  std::memcpy(xStep, xs->data.data(), 24);
  const int L[3] = {(int)d->dims[2], (int)d->dims[1], (int)d->dims[0]};
  const size_t n = (size_t)L[0] * L[1] * L[2];
  const int dt = d->kind == h5::F32 ? SCARL_F32 : SCARL_F64;
  // read_RF_h5_File_Table: the whole dataset, then one upload
  std::vector<double> h64;
  std::vector<float> h32;
  if (dt == SCARL_F64) h64.resize(n);
  else h32.resize(n);
  if (h5::read_values(res_path, *d, dt == SCARL_F64 ? h64.data() : nullptr,
                      dt == SCARL_F32 ? h32.data() : nullptr, &err))
    return fail(ctx, SCARL_EIO, err);
  RC(ensure(ctx, ctx->tile, n * dt));
  RC(copy_in(ctx, ctx->tile.p, dt == SCARL_F64 ? (const void*)h64.data() : (const void*)h32.data(), n * dt));
  double evA = 0.0, evS = 0.0;
  RC(scarl_moments(ctx, ctx->tile.p, dt, (long long)n, 1, &evA, &evS, globalAvg, globalStdDev));
  std::vector<h5::Attr> stats;
  stats.push_back(h5::attr_f64("globalAvg", globalAvg, 1, true));
  stats.push_back(h5::attr_f64("globalStdDev", globalStdDev, 1, true));
  stats.push_back(h5::attr_f64("evntAvg", &evA, 1));
  stats.push_back(h5::attr_f64("evntStdDev", &evS, 1));
  if (calc_corrL) {
    std::vector<double> sk((size_t)L[0] / 2 + L[1] / 2 + L[2] / 2);
    double cl[3];
    RC(scarl_rebuild_sk(ctx, ctx->tile.p, dt, L, *globalAvg, *globalStdDev, 1, sk.data()));
    RC(scarl_rebuild_corrL(sk.data(), L, xStep, cl));
    if (corrL_out) std::memcpy(corrL_out, cl, sizeof cl);
    stats.push_back(h5::attr_f64("corrL_out", cl, 3));
    size_t off = 0;
    for (int k = 0; k < 3; ++k) {
      const int nk = L[k] / 2;
      stats.push_back(h5::attr_f64("Sk_" + std::to_string(k + 1), sk.data() + off, nk));
      off += (size_t)nk;
    }
    // write_StatisticsOnH5 on the result file (main_Stat.f90:90-96)
    if (h5::append_root_attrs(res_path, stats, &err)) return fail(ctx, SCARL_EIO, err);
  }
  // makeStatFile (main_Stat.f90:635-790): folder/STAT_<file> with the
  // sample's attributes, the result file's size in MB and the statistics
  const std::string rp = res_path;
  const size_t slash = rp.find_last_of('/');
  const std::string folder = slash == std::string::npos ? std::string(".") : rp.substr(0, slash);
  const std::string fname = slash == std::string::npos ? rp : rp.substr(slash + 1);
  double mb = 0.0;
  if (FILE* f = std::fopen(res_path, "rb")) {
    std::fseek(f, 0, SEEK_END);
    mb = (double)std::ftell(f) / (1024.0 * 1024.0);
    std::fclose(f);
  }
  std::vector<h5::Attr> out;
  for (const char* nme : {"nb_procs", "nDim", "Nmc", "method", "seedStart", "corrMod", "margiFirst"})
    out.push_back(*find(nme));
  out.push_back(h5::attr_f64("old_file_mb_size", &mb, 1, true));
  for (const char* nme : {"nFields", "Np", "Np_ovlp", "L", "xMinGlob", "xMaxGlob", "xStep", "corrL", "overlap"})
    out.push_back(*find(nme));
  out.insert(out.end(), stats.begin(), stats.end());
  if (h5::write_file(folder + "/STAT_" + fname, out, {}, &err)) return fail(ctx, SCARL_EIO, err);
  return SCARL_OK;
}

// ---- learned padding ----
int scarl_pad_labels(scarl_ctx* ctx, int n, const int* corrMod, const double* nu,
                     const double* ell_pts, const int* N, int* P, int* W, int* saturated) {
  RC(begin(ctx));
  if (n < 1 || !corrMod || !ell_pts || !N || !P || !W) return fail(ctx, SCARL_EINVAL, "null argument");
  std::vector<PadLabelIn> in(n);
  for (int i = 0; i < n; ++i) {
    if (N[i] < 2 || N[i] > 256 || !(ell_pts[i] > 0.0) || corrMod[i] < 1 || corrMod[i] > 3)
      return fail(ctx, SCARL_EINVAL, "label inputs: N in [2, 256], l > 0, corrMod 1..3");
    in[i] = label_in(corrMod[i], nu ? nu[i] : 0.5, ell_pts[i], N[i]);
  }
  RC(ensure(ctx, ctx->t1, (size_t)n * sizeof(PadLabelIn)));
  RC(ensure(ctx, ctx->t2, (size_t)n * sizeof(PadLabelOut)));
  CK(cudaMemcpyAsync(ctx->t1.p, in.data(), (size_t)n * sizeof(PadLabelIn), cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d += (size_t)n * sizeof(PadLabelIn);
  {
    Prof p(ctx, "k_pad_labels");
    CK(launch_pad_labels((const PadLabelIn*)ctx->t1.p, (PadLabelOut*)ctx->t2.p, n, kLearnTol, ctx->stream));
  }
  std::vector<PadLabelOut> out(n);
  CK(cudaMemcpyAsync(out.data(), ctx->t2.p, (size_t)n * sizeof(PadLabelOut), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->d2h += (size_t)n * sizeof(PadLabelOut);
  for (int i = 0; i < n; ++i) {
    P[i] = out[i].P;
    W[i] = out[i].W;
    if (saturated) saturated[i] = out[i].saturated;
  }
  return SCARL_OK;
}

int scarl_pad_error(scarl_ctx* ctx, int n, const int* corrMod, const double* nu,
                    const double* ell_pts, const int* N, const int* P, double* err) {
  RC(begin(ctx));
  if (n < 1 || !corrMod || !ell_pts || !N || !P || !err) return fail(ctx, SCARL_EINVAL, "null argument");
  std::vector<PadLabelIn> in(n);
  for (int i = 0; i < n; ++i) {
    if (N[i] < 2 || N[i] > 256 || P[i] < N[i] || P[i] > 8192 || !(ell_pts[i] > 0.0) || corrMod[i] < 1 || corrMod[i] > 3)
      return fail(ctx, SCARL_EINVAL, "error inputs: N in [2, 256], N <= P <= 8192, l > 0");
    in[i] = label_in(corrMod[i], nu ? nu[i] : 0.5, ell_pts[i], N[i]);
  }
  RC(ensure(ctx, ctx->t1, (size_t)n * (sizeof(PadLabelIn) + sizeof(int))));
  RC(ensure(ctx, ctx->t2, (size_t)n * 8));
  CK(cudaMemcpyAsync(ctx->t1.p, in.data(), (size_t)n * sizeof(PadLabelIn), cudaMemcpyHostToDevice, ctx->stream));
  int* dP = (int*)((char*)ctx->t1.p + (size_t)n * sizeof(PadLabelIn));
  CK(cudaMemcpyAsync(dP, P, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d += (size_t)n * (sizeof(PadLabelIn) + sizeof(int));
  {
    Prof p(ctx, "k_pad_error");
    CK(launch_pad_error((const PadLabelIn*)ctx->t1.p, dP, (double*)ctx->t2.p, n, ctx->stream));
  }
  CK(cudaMemcpyAsync(err, ctx->t2.p, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->d2h += (size_t)n * 8;
  return SCARL_OK;
}

int scarl_mlp_features(int n, const int* corrMod, const double* nu, const double* ell_pts,
                       const int* N, float* X) {
  if (n < 0 || (n && (!corrMod || !ell_pts || !N || !X))) return SCARL_EINVAL;
  for (int i = 0; i < n; ++i) {
    if (!(ell_pts[i] > 0.0) || N[i] < 1) return SCARL_EINVAL;
    mlp_feat(corrMod[i], nu ? nu[i] : 0.5, ell_pts[i], N[i], X + (size_t)i * kMlpIn);
  }
  return SCARL_OK;
}

int scarl_mlp_targets(int n, const double* ell_pts, const int* N, const int* P, const int* W,
                      float* T) {
  if (n < 0 || (n && (!ell_pts || !N || !P || !W || !T))) return SCARL_EINVAL;
  for (int i = 0; i < n; ++i) {
    const double d = std::max(1, P[i] - N[i] + 1);
    T[2 * i] = (float)std::log2(d / ell_pts[i]);
    T[2 * i + 1] = (float)std::log2((double)std::max(W[i], 1) / ell_pts[i]);
  }
  return SCARL_OK;
}

int scarl_mlp_init(scarl_ctx* ctx, uint64_t seed) {
  RC(begin(ctx));
  RC(mlp_alloc(ctx));
  std::vector<float> p(kMlpParams, 0.f);
  uint64_t st = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
  auto next = [&]() {  // splitmix64
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  auto normal = [&]() {
    const double u1 = ((next() >> 11) + 0.5) * 0x1p-53, u2 = ((next() >> 11) + 0.5) * 0x1p-53;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
  };
  const int H = kMlpHidden, I = kMlpIn, O = kMlpOut;
  size_t o = 0;
  for (int i = 0; i < H * I; ++i) p[o++] = (float)(normal() * std::sqrt(2.0 / 8.0));  // 8 live inputs
  o += H;
  for (int i = 0; i < H * H; ++i) p[o++] = (float)(normal() * std::sqrt(2.0 / H));
  o += H;
  for (int i = 0; i < O * H; ++i) p[o++] = (float)(normal() * std::sqrt(1.0 / H));
  CK(cudaMemcpy(ctx->mlp_p.p, p.data(), (size_t)kMlpParams * 4, cudaMemcpyHostToDevice));
  CK(cudaMemset(ctx->mlp_m.p, 0, (size_t)kMlpParams * 4));
  CK(cudaMemset(ctx->mlp_v.p, 0, (size_t)kMlpParams * 4));
  CK(cudaMemset(ctx->mlp_g.p, 0, (size_t)kMlpParams * 4));
  CK(launch_to_bf16((const float*)ctx->mlp_p.p, ctx->mlp_wb.p, kMlpParams, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->h2d += (size_t)kMlpParams * 4;
  ctx->mlp_ready = true;
  ctx->mlp_step = 0;
  return SCARL_OK;
}

int scarl_mlp_params(scarl_ctx* ctx, float* get, const float* set) {
  RC(begin(ctx));
  if (set) {
    RC(mlp_alloc(ctx));
    CK(cudaMemcpy(ctx->mlp_p.p, set, (size_t)kMlpParams * 4, cudaMemcpyHostToDevice));
    CK(cudaMemset(ctx->mlp_m.p, 0, (size_t)kMlpParams * 4));
    CK(cudaMemset(ctx->mlp_v.p, 0, (size_t)kMlpParams * 4));
    CK(cudaMemset(ctx->mlp_g.p, 0, (size_t)kMlpParams * 4));
    CK(launch_to_bf16((const float*)ctx->mlp_p.p, ctx->mlp_wb.p, kMlpParams, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->mlp_ready = true;
    ctx->mlp_step = 0;
  }
  if (get) {
    if (!ctx->mlp_ready) return fail(ctx, SCARL_EINVAL, "no model: call scarl_mlp_init or set parameters");
    CK(cudaMemcpy(get, ctx->mlp_p.p, (size_t)kMlpParams * 4, cudaMemcpyDeviceToHost));
  }
  return SCARL_OK;
}

int scarl_mlp_grad(scarl_ctx* ctx, const float* X, const float* T, int n, float* grad, double* loss) {
  RC(begin(ctx));
  if (!ctx->mlp_ready) return fail(ctx, SCARL_EINVAL, "no model");
  if (n < 1 || !X || !T || !grad || !loss) return fail(ctx, SCARL_EINVAL, "null argument");
  const void* xb;
  RC(mlp_inputs(ctx, X, n, &xb));
  RC(ensure(ctx, ctx->tile, (size_t)n * kMlpOut * 4));
  CK(cudaMemcpyAsync(ctx->tile.p, T, (size_t)n * kMlpOut * 4, cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d += (size_t)n * kMlpOut * 4;
  RC(ensure(ctx, ctx->part, 8));
  CK(cudaMemsetAsync(ctx->part.p, 0, 8, ctx->stream));
  CK(cudaMemsetAsync(ctx->mlp_g.p, 0, (size_t)kMlpParams * 4, ctx->stream));
  {
    Prof p(ctx, "k_mlp_train");
    CK(launch_mlp_train(xb, (const float*)ctx->tile.p, n, ctx->mlp_wb.p, (const float*)ctx->mlp_p.p,
                        (float*)ctx->mlp_g.p, (double*)ctx->part.p, ctx->stream));
  }
  CK(cudaMemcpyAsync(grad, ctx->mlp_g.p, (size_t)kMlpParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(loss, ctx->part.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemsetAsync(ctx->mlp_g.p, 0, (size_t)kMlpParams * 4, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SCARL_OK;
}

int scarl_mlp_train(scarl_ctx* ctx, const float* X, const float* T, int n, int steps, float lr,
                    double* loss_hist) {
  RC(begin(ctx));
  if (!ctx->mlp_ready) return fail(ctx, SCARL_EINVAL, "no model: call scarl_mlp_init first");
  if (n < 1 || steps < 1 || !X || !T || !(lr > 0.f)) return fail(ctx, SCARL_EINVAL, "bad training arguments");
  const void* xb;
  RC(mlp_inputs(ctx, X, n, &xb));
  RC(ensure(ctx, ctx->tile, (size_t)n * kMlpOut * 4));
  CK(cudaMemcpyAsync(ctx->tile.p, T, (size_t)n * kMlpOut * 4, cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d += (size_t)n * kMlpOut * 4;
  RC(ensure(ctx, ctx->part, (size_t)steps * 8));
  CK(cudaMemsetAsync(ctx->part.p, 0, (size_t)steps * 8, ctx->stream));
  CK(cudaMemsetAsync(ctx->mlp_g.p, 0, (size_t)kMlpParams * 4, ctx->stream));
  for (int t = 0; t < steps; ++t) {
    {
      Prof p(ctx, "k_mlp_train");
      CK(launch_mlp_train(xb, (const float*)ctx->tile.p, n, ctx->mlp_wb.p, (const float*)ctx->mlp_p.p,
                          (float*)ctx->mlp_g.p, (double*)ctx->part.p + t, ctx->stream));
    }
    Prof p(ctx, "k_mlp_adam");
    CK(launch_mlp_adam((float*)ctx->mlp_p.p, (float*)ctx->mlp_g.p, (float*)ctx->mlp_m.p,
                       (float*)ctx->mlp_v.p, ctx->mlp_wb.p, lr, ++ctx->mlp_step, ctx->stream));
  }
  if (loss_hist) {
    CK(cudaMemcpyAsync(loss_hist, ctx->part.p, (size_t)steps * 8, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->d2h += (size_t)steps * 8;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return SCARL_OK;
}

int scarl_mlp_predict(scarl_ctx* ctx, const float* X, int n, float* Y) {
  RC(begin(ctx));
  if (!ctx->mlp_ready) return fail(ctx, SCARL_EINVAL, "no model");
  if (n < 1 || !X || !Y) return fail(ctx, SCARL_EINVAL, "null argument");
  const void* xb;
  RC(mlp_inputs(ctx, X, n, &xb));
  RC(ensure(ctx, ctx->tile, (size_t)n * kMlpOut * 4));
  {
    Prof p(ctx, "k_mlp_infer");
    CK(launch_mlp_infer(xb, n, ctx->mlp_wb.p, (const float*)ctx->mlp_p.p, (float*)ctx->tile.p, ctx->stream));
  }
  CK(cudaMemcpyAsync(Y, ctx->tile.p, (size_t)n * kMlpOut * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->d2h += (size_t)n * kMlpOut * 4;
  return SCARL_OK;
}

int scarl_pad_size_learned(scarl_ctx* ctx, int corrMod, double nu, const double corrL[3],
                           const double xStep[3], const int Np[3], int P[3], int W[3],
                           int* fallback) {
  RC(begin(ctx));
  if (!corrL || !xStep || !Np || !P) return fail(ctx, SCARL_EINVAL, "null argument");
  int full[3];
  RC(pad_size(SCARL_PAD_FULL, corrMod, nu, corrL, xStep, Np, 0.0, full) == SCARL_OK ? SCARL_OK : SCARL_EINVAL);
  double ell[3];
  bool ok = ctx->mlp_ready;
  float X[3 * kMlpIn], Y[3 * kMlpOut];
  for (int d = 0; d < 3; ++d) {
    ell[d] = corrL[d] / xStep[d];
    ok = ok && mlp_in_range(corrMod, nu, ell[d], Np[d]);
    mlp_feat(corrMod, nu, ell[d], Np[d], X + d * kMlpIn);
  }
  if (ok) RC(scarl_mlp_predict(ctx, X, 3, Y));
  int fb = ok ? 0 : 1;
  for (int d = 0; d < 3; ++d) {
    if (!ok) {
      P[d] = full[d];
      if (W) W[d] = Np[d];
      continue;
    }
    const double D = ell[d] * std::exp2((double)Y[2 * d] + kLearnMargin);
    const double need = (double)Np[d] - 1.0 + std::ceil(D);
    // the smallest length the generator runs (powers of two and 3, 5, 7
    // times a power of two >= 16) that covers the prediction
    int p = std::max(8, Np[d]);
    while (p <= 2048 && ((double)p < need || !fft_length_supported(p))) ++p;
    if (p > full[d] || p > 2048 || !std::isfinite(D)) {
      p = full[d];
      fb |= 2;
    }
    P[d] = p;
    if (W) {
      const double w = std::ceil(ell[d] * std::exp2((double)Y[2 * d + 1] + kLearnMargin));
      W[d] = (int)std::min<double>((double)Np[d], std::max(2.0, std::isfinite(w) ? w : (double)Np[d]));
    }
  }
  if (fallback) *fallback = fb;
  return SCARL_OK;
}

// ---- output files ----
int scarl_write_sample_h5(scarl_ctx* ctx, const char* folder, const char* output_name,
                          const void* field, int dtype, const scarl_sample* s,
                          const scarl_layout* lay, int one_file, int one_hdf_ds,
                          const char* time_labels, const double* times, int ntimes) {
  if (ctx) RC(begin(ctx));
  if (!folder || !output_name || !field || !s || !lay) return fail(ctx, SCARL_EINVAL, "null argument");
  if (dtype != SCARL_F32 && dtype != SCARL_F64) return fail(ctx, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64");
  const bool dev = is_device_ptr(field);
  if (dev && !ctx) return SCARL_EINVAL;  // device fields are copied through a context
  if (lay->nb_tiles < 1 || lay->nb_tiles != lay->topo_shape[0] * lay->topo_shape[1] * lay->topo_shape[2])
    return fail(ctx, SCARL_EINVAL, "inconsistent layout");
  const h5::Kind kind = dtype == SCARL_F64 ? h5::F64 : h5::F32;
  const std::string dir = std::string(folder) + "/";
  const std::string name = output_name;
  const int nb = lay->nb_tiles;
  std::vector<scarl_tile> tiles(nb);
  for (int r = 0; r < nb; ++r) tile_geometry(lay, s->xMinGlob, r, &tiles[r]);
  double xMaxEff[3];  // main_ScaRL.f90:462-467 (xMaxGlob re-derived from the last tile)
  for (int d = 0; d < 3; ++d) xMaxEff[d] = tiles[nb - 1].coord_N[d];
  const std::vector<h5::Attr> root = sample_attrs(s, *lay, xMaxEff);
  std::string err;
  auto tile_dataset = [&](int r, bool pos) {
    h5::Dataset d;
    d.name = "sample_1_p" + std::to_string(r);
    d.kind = kind;
    d.dims = {(uint64_t)lay->Np[2], (uint64_t)lay->Np[1], (uint64_t)lay->Np[0]};
    d.nbytes = (uint64_t)lay->Np[0] * lay->Np[1] * lay->Np[2] * dtype;
    d.attrs.push_back(h5::attr_f64("xMin", tiles[r].coord_0, 3));
    d.attrs.push_back(h5::attr_f64("xMax", tiles[r].coord_N, 3));
    if (pos) {
      d.attrs.push_back(h5::attr_i32("pos_0", tiles[r].pos_0, 3));
      d.attrs.push_back(h5::attr_i32("pos_N", tiles[r].pos_N, 3));
    }
    int o[3];
    for (int k = 0; k < 3; ++k) o[k] = tiles[r].pos_0[k] - 1;
    const int* Np = lay->Np;
    const int* L = lay->L;
    d.write = [=](FILE* f) { return write_block(ctx, f, field, dev, dtype, L, o, Np); };
    return d;
  };
  if (one_file && one_hdf_ds) {  // write_hdf5_multi_proc_3D_1ds
    std::vector<h5::Dataset> ds;
    h5::Dataset d;
    d.name = "samples";
    d.kind = kind;
    d.dims = {(uint64_t)lay->L[2], (uint64_t)lay->L[1], (uint64_t)lay->L[0]};
    d.nbytes = (uint64_t)lay->L[0] * lay->L[1] * lay->L[2] * dtype;
    const int one[3] = {1, 1, 1};
    d.attrs.push_back(h5::attr_f64("xMin", tiles[0].coord_0, 3));
    d.attrs.push_back(h5::attr_f64("xMax", xMaxEff, 3));
    d.attrs.push_back(h5::attr_i32("pos_0", one, 3));
    d.attrs.push_back(h5::attr_i32("pos_N", lay->L, 3));
    const int zero[3] = {0, 0, 0};
    const int* L = lay->L;
    d.write = [=](FILE* f) { return write_block(ctx, f, field, dev, dtype, L, zero, L); };
    ds.push_back(d);
    time_datasets(time_labels, times, ntimes, &ds);
    if (h5::write_file(dir + name + ".h5", root, ds, &err)) return fail(ctx, SCARL_EIO, err);
    if (!xmf_elements(dir + name + ".xmf", name + ".h5", tiles[0].coord_0, xMaxEff, lay->L, "samples", dtype))
      return fail(ctx, SCARL_EIO, "cannot write " + dir + name + ".xmf");
    return SCARL_OK;
  }
  std::vector<std::string> h5list(nb);
  std::vector<std::array<double, 3>> c0(nb);
  for (int r = 0; r < nb; ++r)
    for (int d = 0; d < 3; ++d) c0[r][d] = tiles[r].coord_0[d];
  if (one_file) {  // write_hdf5_multi_proc_3D: one dataset per tile
    std::vector<h5::Dataset> ds;
    for (int r = 0; r < nb; ++r) ds.push_back(tile_dataset(r, true));
    time_datasets(time_labels, times, ntimes, &ds);
    if (h5::write_file(dir + name + ".h5", root, ds, &err)) return fail(ctx, SCARL_EIO, err);
    for (int r = 0; r < nb; ++r) h5list[r] = name + ".h5";
  } else {  // write_hdf5_single_proc_3D: one file per tile
    for (int r = 0; r < nb; ++r) {
      const std::string base = name + "_proc_" + pad5(r);
      std::vector<h5::Dataset> ds = {tile_dataset(r, false)};
      time_datasets(time_labels, times, ntimes, &ds);
      if (h5::write_file(dir + base + ".h5", root, ds, &err)) return fail(ctx, SCARL_EIO, err);
      if (!xmf_elements(dir + base + ".xmf", base + ".h5", tiles[r].coord_0, tiles[r].coord_N, lay->Np,
                        "sample_1_p" + std::to_string(r), dtype))
        return fail(ctx, SCARL_EIO, "cannot write " + dir + base + ".xmf");
      h5list[r] = base + ".h5";
    }
  }
  if (!xmf_global(dir + name + ".xmf", h5list, c0, lay->xStep, lay->Np, dtype))
    return fail(ctx, SCARL_EIO, "cannot write " + dir + name + ".xmf");
  return SCARL_OK;
}

// write_constant_field (SRC_F/write_output.f90:144-178): a 2 x 2 x 2 field of
// avg with the attribute values the reference gives it.
int scarl_write_constant_field_h5(const char* folder, const char* output_name,
                                  const double xMinGlob[3], const double xMaxGlob[3], double avg) {
  if (!folder || !output_name || !xMinGlob || !xMaxGlob) return SCARL_EINVAL;
  const std::string dir = std::string(folder) + "/", name = output_name;
  const int one = 1, three = 3, m1 = -1;
  const int ones[3] = {1, 1, 1}, twos[3] = {2, 2, 2}, zeros[3] = {0, 0, 0};
  double xStep[3];
  for (int d = 0; d < 3; ++d) xStep[d] = xMaxGlob[d] - xMinGlob[d];
  const double neg[3] = {-1.0, -1.0, -1.0}, zero3[3] = {0.0, 0.0, 0.0};
  std::vector<h5::Attr> root;
  root.push_back(h5::attr_i32("nb_procs", &one, 1, true));
  root.push_back(h5::attr_i32("nDim", &three, 1, true));
  root.push_back(h5::attr_i32("Nmc", &one, 1, true));
  root.push_back(h5::attr_i32("method", &m1, 1, true));
  root.push_back(h5::attr_i32("seedStart", &m1, 1, true));
  root.push_back(h5::attr_i32("corrMod", &m1, 1, true));
  root.push_back(h5::attr_i32("margiFirst", &m1, 1, true));
  root.push_back(h5::attr_i32("nFields", ones, 3));
  root.push_back(h5::attr_i32("Np", twos, 3));
  root.push_back(h5::attr_i32("Np_ovlp", zeros, 3));
  root.push_back(h5::attr_i32("L", twos, 3));
  root.push_back(h5::attr_f64("xMinGlob", xMinGlob, 3));
  root.push_back(h5::attr_f64("xMaxGlob", xMaxGlob, 3));
  root.push_back(h5::attr_f64("xStep", xStep, 3));
  root.push_back(h5::attr_f64("corrL", neg, 3));
  root.push_back(h5::attr_f64("overlap", zero3, 3));
  h5::Dataset d;
  d.name = "samples";
  d.kind = h5::F64;
  d.dims = {2, 2, 2};
  d.nbytes = 64;
  d.attrs.push_back(h5::attr_f64("xMin", xMinGlob, 3));
  d.attrs.push_back(h5::attr_f64("xMax", xMaxGlob, 3));
  d.write = [avg](FILE* f) {
    const double v[8] = {avg, avg, avg, avg, avg, avg, avg, avg};
    return std::fwrite(v, 8, 8, f) == 8;
  };
  std::string err;
  if (h5::write_file(dir + name + ".h5", root, {d}, &err)) return SCARL_EIO;
  if (!xmf_elements(dir + name + ".xmf", name + ".h5", xMinGlob, xMaxGlob, twos, "samples", 8))
    return SCARL_EIO;
  return SCARL_OK;
}

static int copy_msg(char* msg, size_t len, const std::string& m) {
  if (msg && len) {
    std::snprintf(msg, len, "%s", m.c_str());
  }
  return 0;
}

int scarl_h5_overwrite_dataset(const char* path, const char* name, const void* data,
                               unsigned long long nbytes, char* msg, size_t msg_len) {
  if (!path || !name || !data) return SCARL_EINVAL;
  std::string err;
  const int rc = h5::overwrite_dataset(path, name, data, nbytes, &err);
  if (rc) {
    copy_msg(msg, msg_len, err);
    return rc == 6 ? SCARL_EIO : (rc == 5 ? SCARL_EUNSUPPORTED : SCARL_EINVAL);
  }
  return SCARL_OK;
}

int scarl_h5_list(const char* path, char* names, size_t len, char* msg, size_t msg_len) {
  if (!path || !names || !len) return SCARL_EINVAL;
  h5::RObject root;
  std::vector<h5::RObject> ds;
  std::string err;
  const int rc = h5::read_file(path, &root, &ds, &err);
  if (rc) {
    copy_msg(msg, msg_len, err);
    return rc == 5 ? SCARL_EUNSUPPORTED : (rc == 6 ? SCARL_EIO : SCARL_EINVAL);
  }
  std::string all;
  for (const auto& d : ds) all += d.name + "\n";
  if (all.size() + 1 > len) {
    copy_msg(msg, msg_len, "name buffer too small");
    return SCARL_EINVAL;
  }
  std::memcpy(names, all.c_str(), all.size() + 1);
  return SCARL_OK;
}

int scarl_h5_read_dataset(const char* path, const char* name, void* out, int dtype,
                          long long dims[3], int* rank, char* msg, size_t msg_len) {
  if (!path || !name || !dims || !rank) return SCARL_EINVAL;
  h5::RObject root;
  std::vector<h5::RObject> ds;
  std::string err;
  const int rc = h5::read_file(path, &root, &ds, &err);
  if (rc) {
    copy_msg(msg, msg_len, err);
    return rc == 5 ? SCARL_EUNSUPPORTED : (rc == 6 ? SCARL_EIO : SCARL_EINVAL);
  }
  for (const auto& d : ds) {
    if (d.name != name) continue;
    if (d.dims.size() > 3) {
      copy_msg(msg, msg_len, "datasets of rank > 3 are not supported");
      return SCARL_EUNSUPPORTED;
    }
    *rank = (int)d.dims.size();
    for (int k = 0; k < 3; ++k) dims[k] = 1;
    for (int k = 0; k < *rank; ++k) dims[k] = (long long)d.dims[*rank - 1 - k];  // column-major order
    if (!out) return SCARL_OK;
    if (dtype != SCARL_F32 && dtype != SCARL_F64) return SCARL_EINVAL;
    if (h5::read_values(path, d, dtype == SCARL_F64 ? (double*)out : nullptr,
                        dtype == SCARL_F32 ? (float*)out : nullptr, &err)) {
      copy_msg(msg, msg_len, err);
      return SCARL_EIO;
    }
    return SCARL_OK;
  }
  copy_msg(msg, msg_len, std::string("no dataset ") + name);
  return SCARL_EINVAL;
}

int scarl_h5_read_attr(const char* path, const char* object, const char* name, double* out,
                       int max_count, int* count, char* msg, size_t msg_len) {
  if (!path || !name || !count) return SCARL_EINVAL;
  h5::RObject root;
  std::vector<h5::RObject> ds;
  std::string err;
  const int rc = h5::read_file(path, &root, &ds, &err);
  if (rc) {
    copy_msg(msg, msg_len, err);
    return rc == 5 ? SCARL_EUNSUPPORTED : (rc == 6 ? SCARL_EIO : SCARL_EINVAL);
  }
  const h5::RObject* o = nullptr;
  if (!object || !*object) o = &root;
  for (const auto& d : ds)
    if (object && d.name == object) o = &d;
  if (!o) {
    copy_msg(msg, msg_len, std::string("no object ") + (object ? object : ""));
    return SCARL_EINVAL;
  }
  for (const auto& a : o->attrs) {
    if (a.name != name) continue;
    if (a.kind == h5::STR) {
      copy_msg(msg, msg_len, "string attribute");
      return SCARL_EUNSUPPORTED;
    }
    const int es = a.kind == h5::F64 ? 8 : 4;
    const int n = (int)(a.data.size() / es);
    *count = n;
    for (int i = 0; i < n && i < max_count && out; ++i) {
      if (a.kind == h5::F64) std::memcpy(&out[i], &a.data[(size_t)i * 8], 8);
      else if (a.kind == h5::F32) { float f; std::memcpy(&f, &a.data[(size_t)i * 4], 4); out[i] = f; }
      else { int32_t v; std::memcpy(&v, &a.data[(size_t)i * 4], 4); out[i] = v; }
    }
    return SCARL_OK;
  }
  copy_msg(msg, msg_len, std::string("no attribute ") + name);
  return SCARL_EINVAL;
}

// ---- generation ----
int scarl_gen_std_gauss_fft(scarl_ctx* ctx, double* data, const int Np[3], const double xRange[3],
                            const double corrL[3], int corrMod, int seed, int rank,
                            const double* phiK, const double* gammaK) {
  RC(begin(ctx));
  if (!data || !Np || !xRange || !corrL) return fail(ctx, SCARL_EINVAL, "null argument");
  if (corrMod != SCARL_CM_GAUSSIAN) return fail(ctx, SCARL_EINVAL, "ERROR: Correlation model not implemented");
  for (int d = 0; d < 3; ++d)
    if (Np[d] < 2) return fail(ctx, SCARL_EINVAL, "Np must be >= 2");
  const size_t n = (size_t)Np[0] * Np[1] * Np[2];
  const size_t nk = (size_t)(Np[0] / 2) * (Np[1] / 2) * (Np[2] / 2);
  void* dev;
  bool host;
  RC(out_dev(ctx, data, n * 8, &dev, &host));
  const void *phi = nullptr, *gam = nullptr;
  RC(in_dev(ctx, ctx->stage_in, phiK, nk * 8, &phi));
  RC(in_dev(ctx, ctx->stage_in2, gammaK, nk * 8, &gam));
  RC(dct_tile(ctx, (double*)dev, Np, xRange, corrL, (const double*)phi, (const double*)gam,
              (uint32_t)((uint32_t)seed + (uint32_t)rank)));
  return finish_out(ctx, data, dev, n * 8, host);
}

int scarl_gen_std_gauss_fft_mpi(scarl_ctx* ctx, double* data, const double xRange[3],
                                const double corrL[3], int corrMod, int seed, int rank,
                                const int L[3], const int Np[3], const double* phiK,
                                const double* gammaK) {
  RC(begin(ctx));
  if (!data || !xRange || !corrL || !L || !Np) return fail(ctx, SCARL_EINVAL, "null argument");
  if (corrMod != SCARL_CM_GAUSSIAN) return fail(ctx, SCARL_EINVAL, "ERROR: Correlation model not implemented");
  for (int d = 0; d < 3; ++d) {
    if (L[d] < 2) return fail(ctx, SCARL_EINVAL, "L must be >= 2");
    if (Np[d] != L[d])
      return fail(ctx, SCARL_EUNSUPPORTED, "the global transform runs on one GPU: Np must equal L (one rank)");
  }
  const size_t n = (size_t)L[0] * L[1] * L[2];
  const size_t nk = (size_t)(L[0] / 2) * (L[1] / 2) * L[2];
  void* dev;
  bool host;
  RC(out_dev(ctx, data, n * 8, &dev, &host));
  const void *phi = nullptr, *gam = nullptr;
  RC(in_dev(ctx, ctx->stage_in, phiK, nk * 8, &phi));
  RC(in_dev(ctx, ctx->stage_in2, gammaK, nk * 8, &gam));
  RC(dct_tile(ctx, (double*)dev, L, xRange, corrL, (const double*)phi, (const double*)gam,
              (uint32_t)((uint32_t)seed + (uint32_t)rank), true));
  return finish_out(ctx, data, dev, n * 8, host);
}

int scarl_gen_std_gauss_shino_fft(scarl_ctx* ctx, double* data, const int Np[3],
                                  const double xRange[3], const double corrL[3],
                                  const int ppcl[3], int corrMod, int seed, int rank) {
  (void)ppcl;
  (void)rank;
  RC(begin(ctx));
  if (!data || !Np || !xRange || !corrL) return fail(ctx, SCARL_EINVAL, "null argument");
  if (corrMod != SCARL_CM_GAUSSIAN)
    return fail(ctx, SCARL_EUNSUPPORTED, "the Shino generator has only the Gaussian model (SRC_F/spectra_ScaRL.f90:119-137 is commented out)");
  for (int d = 0; d < 3; ++d)
    if (Np[d] < 2 || !(corrL[d] > 0.0)) return fail(ctx, SCARL_EINVAL, "Np >= 2 and corrL > 0 required");
  const size_t n = (size_t)Np[0] * Np[1] * Np[2];
  void* dev;
  bool host;
  RC(out_dev(ctx, data, n * 8, &dev, &host));
  GenArgs a;
  RC(shino_args(ctx, Np, xRange, corrL, seed, &a));
  a.epi.mode = 0;
  a.epi.out = dev;
  RC(run_passes(ctx, 8, a));
  return finish_out(ctx, data, dev, n * 8, host);
}

int scarl_gen_padded(scarl_ctx* ctx, void* out, int dtype_in, const int Np[3], const int pad[3],
                     const double xStep[3], const double corrL[3], int corrMod, double nu,
                     int normalise, uint64_t seed, uint32_t stream, const void* xi) {
  RC(begin(ctx));
  if (!out || !Np || !xStep || !corrL) return fail(ctx, SCARL_EINVAL, "null argument");
  int dtype, split;
  RC(parse_dtype(ctx, dtype_in, &dtype, &split));
  if (corrMod < 1 || corrMod > 3) return fail(ctx, SCARL_EINVAL, "ERROR: Correlation model not implemented");
  if (corrMod == SCARL_CM_VON_KARMAN && !(nu > 0.0)) return fail(ctx, SCARL_EINVAL, "nu must be > 0");
  int P[3];
  for (int d = 0; d < 3; ++d) {
    P[d] = (pad && pad[d] > 0) ? pad[d] : default_pad(Np[d]);
    if (!(xStep[d] > 0.0) || !(corrL[d] > 0.0)) return fail(ctx, SCARL_EINVAL, "xStep and corrL must be > 0");
  }
  RC(check_grid(ctx, P, Np));
  const size_t n = (size_t)Np[0] * Np[1] * Np[2];
  void* dev;
  bool host;
  RC(out_dev(ctx, out, n * dtype, &dev, &host));
  PaddedPlan* pl;
  RC(padded_plan(ctx, dtype, P, xStep, corrL, corrMod, nu, normalise, &pl));
  GenArgs a;
  RC(gen_args(ctx, dtype, P, Np, &a));
  set_plan(&a, pl);
  a.split = split;
  a.k0 = (uint32_t)seed;
  a.k1 = (uint32_t)(seed >> 32);
  a.stream = stream;
  if (xi) {
    const size_t nm = (size_t)a.Hx * P[1] * P[2];
    RC(in_dev(ctx, ctx->stage_in, xi, nm * 2 * dtype, &a.xi));
    a.spec = SPEC_INJECT;
  }
  a.epi.mode = 0;
  a.epi.out = dev;
  RC(run_passes(ctx, dtype, a));
  return finish_out(ctx, out, dev, n * dtype, host);
}

int scarl_ensemble_draw(uint64_t seed, long long first, int n, const int* choices, int nchoices,
                        double lmin, double lmax, int* Np, double* corrL) {
  return ensemble_draw(seed, first, n, choices, nchoices, lmin, lmax, Np, corrL);
}

int scarl_gen_ensemble(scarl_ctx* ctx, void* out, int dtype_in, int n, const int* Np,
                       const double* xStep, const double* corrL, int corrMod, double nu,
                       int pad_policy, double pad_tol, const uint64_t* seeds,
                       const uint32_t* streams, int margiFirst, double avg, double std_dev,
                       int flags) {
  RC(begin(ctx));
  if (!out || !Np || !xStep || !corrL) return fail(ctx, SCARL_EINVAL, "null argument");
  if (n < 1 || n > 65536) return fail(ctx, SCARL_EINVAL, "ensemble size must be in [1, 65536]");
  int dtype, split;
  RC(parse_dtype(ctx, dtype_in, &dtype, &split));
  if (corrMod < 1 || corrMod > 3) return fail(ctx, SCARL_EINVAL, "ERROR: Correlation model not implemented");
  if (corrMod == SCARL_CM_VON_KARMAN && !(nu > 0.0)) return fail(ctx, SCARL_EINVAL, "nu must be > 0");
  if (pad_policy != SCARL_PAD_FULL && pad_policy != SCARL_PAD_AUTO && pad_policy != SCARL_PAD_SMOOTH)
    return fail(ctx, SCARL_EINVAL, "unknown padding policy");
  if (margiFirst < 0 || margiFirst > 2) return fail(ctx, SCARL_EINVAL, "First-order marginal not detected");
  const double tol = pad_tol > 0.0 ? pad_tol : 1e-3;
  std::string key;
  {
    char b[160];
    std::snprintf(b, sizeof b, "%d|%d|%a|%d|%a|%d", dtype_in, corrMod, nu, pad_policy, tol, n);
    key = b;
    key.reserve(key.size() + (size_t)n * 96);
    for (int i = 0; i < n; ++i) {
      for (int d = 0; d < 3; ++d) {
        if (Np[3 * i + d] < 1) return fail(ctx, SCARL_EINVAL, "Np must be >= 1");
        if (!(xStep[3 * i + d] > 0.0) || !(corrL[3 * i + d] > 0.0))
          return fail(ctx, SCARL_EINVAL, "xStep and corrL must be > 0");
      }
      std::snprintf(b, sizeof b, "|%d,%d,%d,%a,%a,%a,%a,%a,%a", Np[3 * i], Np[3 * i + 1],
                    Np[3 * i + 2], xStep[3 * i], xStep[3 * i + 1], xStep[3 * i + 2], corrL[3 * i],
                    corrL[3 * i + 1], corrL[3 * i + 2]);
      key += b;
    }
  }
  if (!ctx->ens || ctx->ens->key != key)
    RC(ens_build(ctx, dtype, split, n, Np, xStep, corrL, corrMod, nu, pad_policy, tol, key));
  EnsPlan* e = ctx->ens;
  void* dev;
  bool host;
  RC(out_dev(ctx, out, e->total * dtype, &dev, &host));
  double ms = 1.0, mu = 0.0;
  if (margiFirst) RC(marginal_params(ctx, margiFirst, avg, std_dev, &ms, &mu));
  bool changed = !e->uploaded;
  for (int i = 0; i < n; ++i) {
    GenArgs& a = e->args[i];
    const uint64_t sd = seeds ? seeds[i] : (uint64_t)i;
    const uint32_t k0 = (uint32_t)sd, k1 = (uint32_t)(sd >> 32), st = streams ? streams[i] : 0u;
    void* o = static_cast<char*>(dev) + e->off[i] * dtype;
    if (a.k0 != k0 || a.k1 != k1 || a.stream != st || a.epi.out != o || a.epi.marginal != margiFirst ||
        a.epi.ms != ms || a.epi.mmu != mu) {
      a.k0 = k0;
      a.k1 = k1;
      a.stream = st;
      a.epi.out = o;
      a.epi.marginal = margiFirst;
      a.epi.ms = ms;
      a.epi.mmu = mu;
      changed = true;
    }
  }
  if (changed) {
    for (int i = 0; i < n; ++i) philox_schedule(&e->args[i]);
    const size_t bytes = (size_t)n * sizeof(GenArgs);
    void* pin;
    RC(pinned(ctx, bytes, &pin));
    std::memcpy(pin, e->args.data(), bytes);
    RC(upload_pinned(ctx, e->dargs.p, bytes));
    e->uploaded = true;
  }
  if ((flags & SCARL_ENS_AUTOTUNE) && !e->tuned) {
    RC(ens_tune(ctx, e));
    e->tuned = true;
  }
  const bool graph = !(flags & SCARL_ENS_NO_GRAPH) && !ctx->profile && !e->graph_failed;
  if (graph && e->exec) {
    CK(cudaGraphLaunch(e->exec, ctx->stream));
    ctx->launches += (long long)e->groups.size();
  } else {
    RC(ens_launch(ctx, e));
    if (graph) ens_capture(ctx, e);
  }
  return finish_out(ctx, out, dev, e->total * dtype, host);
}

int scarl_generate_sample(scarl_ctx* ctx, const scarl_sample* s, const scarl_gen_opts* o_in,
                          void* global) {
  RC(begin(ctx));
  if (!s || !global) return fail(ctx, SCARL_EINVAL, "null argument");
  scarl_gen_opts o;
  std::memset(&o, 0, sizeof o);
  if (o_in) o = *o_in;
  const int gen = o.generator ? o.generator : SCARL_GEN_PADDED;
  int dt, split;
  RC(parse_dtype(ctx, o.dtype ? o.dtype : SCARL_F32, &dt, &split));
  if (gen != SCARL_GEN_PADDED && dt != SCARL_F64)
    return fail(ctx, SCARL_EUNSUPPORTED, "the reference generators (DCT, Shino) run in FP64 only");
  const int gm = o.gen_meth ? o.gen_meth : SCARL_FFT;
  if (gm != SCARL_FFT && gm != SCARL_FFT_MPI) return fail(ctx, SCARL_EINVAL, "ERROR! Generation Method not implemented");
  if (gm == SCARL_FFT_MPI && gen == SCARL_GEN_SHINO)
    return fail(ctx, SCARL_EUNSUPPORTED, "the Shino generator has no global (FFT_MPI) form");
  char msg[256];
  if (verify_inputs(s, gm, msg, sizeof msg) != SCARL_OK) return fail(ctx, SCARL_EINVAL, msg);
  if (gen != SCARL_GEN_PADDED && s->corrMod != SCARL_CM_GAUSSIAN)
    return fail(ctx, SCARL_EINVAL, "ERROR: Correlation model not implemented");
  const int nb_procs = o.nb_procs > 0 ? o.nb_procs : 1;
  const bool topo_given = o.topo_shape[0] > 0 && o.topo_shape[1] > 0 && o.topo_shape[2] > 0;
  scarl_layout lay;
  if (sample_layout(s, gm, nb_procs, topo_given ? o.topo_shape : nullptr, &lay) != SCARL_OK)
    return fail(ctx, SCARL_EINVAL, "ERROR! procs grid dimensions do not agree with the total number of procs");
  if (gm == SCARL_FFT_MPI) {
    // the slabs of the FFTW-MPI layout form one global transform on the GPU:
    // a single tile of the re-fitted grid, no partition of unity
    for (int d = 0; d < 3; ++d) {
      lay.Np[d] = lay.L[d];
      lay.Np_ovlp[d] = 0;
      lay.topo_shape[d] = 1;
    }
    lay.nb_tiles = 1;
  }
  for (int d = 0; d < 3; ++d)
    if (lay.Np_ovlp[d] < 0) return fail(ctx, SCARL_EUNSUPPORTED, "negative overlap (discontinuous mesh) is not supported");
  if (lay.nb_tiles > 4096) return fail(ctx, SCARL_EINVAL, "too many tiles");
  const size_t ng = (size_t)lay.L[0] * lay.L[1] * lay.L[2];
  void* dev;
  bool host;
  RC(out_dev(ctx, global, ng * dt, &dev, &host));
  if (o.moments && (gen == SCARL_GEN_DCT || o.normalize_field))
    return fail(ctx, SCARL_EUNSUPPORTED,
                "streamed moments need the padded or Shino generator without normalize_field");
  if (s->std_dev == 0.0) {  // write_constant_field, SRC_F/main_ScaRL.f90:145-155
    if (o.moments) {
      o.moments[0] = s->avg * (double)ng;
      o.moments[1] = s->avg * s->avg * (double)ng;
    }
    if (dt == 8) {
      CK(cudaMemsetAsync(dev, 0, ng * 8, ctx->stream));
      RC(launch_marginal(8, dev, (int64_t)ng, 1, 0.0, s->avg, ctx->stream) == cudaSuccess ? SCARL_OK : SCARL_EDEVICE);
    } else {
      CK(cudaMemsetAsync(dev, 0, ng * 4, ctx->stream));
      RC(launch_marginal(4, dev, (int64_t)ng, 1, 0.0, s->avg, ctx->stream) == cudaSuccess ? SCARL_OK : SCARL_EDEVICE);
    }
    return finish_out(ctx, global, dev, ng * dt, host);
  }
  double ms, mmu;
  RC(marginal_params(ctx, s->margiFirst, s->avg, s->std_dev, &ms, &mmu));
  std::vector<BlendAxis> axes;
  RC(upload_blend_tables(ctx, lay, 1, &axes));
  Epilogue epi;
  std::memset(&epi, 0, sizeof epi);
  epi.mode = 1;
  epi.out = dev;
  for (int d = 0; d < 3; ++d) epi.L[d] = lay.L[d];
  epi.marginal = o.normalize_field ? 0 : s->margiFirst;
  epi.ms = ms;
  epi.mmu = mmu;
  epi.apply_pou = gm == SCARL_FFT ? 1 : 0;
  const size_t ntile = (size_t)lay.Np[0] * lay.Np[1] * lay.Np[2];
  const size_t nk = (size_t)(lay.Np[0] / 2) * (lay.Np[1] / 2) *
                    (gm == SCARL_FFT_MPI ? lay.Np[2] : lay.Np[2] / 2);
  PaddedPlan* pl = nullptr;
  int P[3];
  if (gen == SCARL_GEN_PADDED) {
    int Pp[3];
    const double tol = o.pad_tol > 0.0 ? o.pad_tol : 1e-3;
    if (o.pad_policy == SCARL_PAD_LEARNED) {
      RC(scarl_pad_size_learned(ctx, s->corrMod, s->nu, s->corrL, lay.xStep, lay.Np, Pp, nullptr, nullptr));
    } else if (pad_size(o.pad_policy, s->corrMod, s->nu, s->corrL, lay.xStep, lay.Np, tol, Pp) != SCARL_OK) {
      return fail(ctx, SCARL_EINVAL, "invalid padding policy or tolerance");
    }
    for (int d = 0; d < 3; ++d) P[d] = o.pad[d] > 0 ? o.pad[d] : Pp[d];
    RC(check_grid(ctx, P, lay.Np));
    for (int d = 0; d < 3; ++d)
      if (!(s->corrL[d] > 0.0)) return fail(ctx, SCARL_EINVAL, "corrL must be > 0");
    RC(padded_plan(ctx, dt, P, lay.xStep, s->corrL, s->corrMod, s->nu, !o.no_spectral_normalisation, &pl));
    if (o.autotune) {
      char key[128];
      std::snprintf(key, sizeof key, "%d|%d,%d,%d|%d,%d,%d", dt, P[0], P[1], P[2], lay.Np[0], lay.Np[1], lay.Np[2]);
      if (!ctx->tuned_shapes[key]) {
        RC(autotune_shape(ctx, dt, P, lay.Np, s->corrMod, s->nu, lay.xStep, s->corrL));
        ctx->tuned_shapes[key] = true;
        tune_save(ctx, std::getenv("SCARL_TUNE_CACHE"));
      }
    }
  }
  if (gen == SCARL_GEN_DCT) {
    for (int d = 0; d < 3; ++d)
      if (lay.Np[d] < 2) return fail(ctx, SCARL_EINVAL, "Np must be >= 2");
    RC(ensure(ctx, ctx->tile, ntile * 8));
  }
  const void* phi_all = nullptr;
  if (gen == SCARL_GEN_DCT && o.phiK)
    RC(in_dev(ctx, ctx->stage_in, o.phiK, nk * lay.nb_tiles * 8, &phi_all));
  // pinned host output over several rows of tiles: finished boxes stream
  // back while the later rows are generated
  SlabCopier slabs;
  const bool stream_out = host && !o.normalize_field && lay.topo_shape[1] * lay.topo_shape[2] > 1 &&
                          is_pinned_host(global);
  if (stream_out) RC(slab_begin(ctx, slabs, global, dev, (size_t)lay.L[0] * dt, lay.L[1]));
  // pageable host output of kRingMin bytes and more over several rows of
  // tiles: the same boxes pass through the pinned ring, starting while the
  // later rows are generated
  const size_t row_b = (size_t)lay.L[0] * dt, plane_b = row_b * lay.L[1];
  const bool ring_out = host && !stream_out && !o.normalize_field &&
                        lay.topo_shape[1] * lay.topo_shape[2] > 1 && ng * dt >= kRingMin && row_b <= kRingChunk;
  std::vector<RingPiece> ring_pieces;
  size_t ring_nev = 0;
  auto row_start = [&](int d, int tp) {  // first plane (d = 1: y, 2: z) of the box of tile row tp
    return tp >= lay.topo_shape[d] ? lay.L[d] : std::min(lay.L[d], (lay.Np[d] - lay.Np_ovlp[d]) * tp);
  };
  // padded tiles whose pass 1 runs on the tensor cores (a persistent kernel,
  // whose per-tile launches end with a partial wave): passes 1-2 batched over
  // groups of up to kb tiles, one work buffer each (at most kBatchWork bytes
  // of them); pass 3 per tile, in order.  The CUDA-core passes gain nothing
  // from batching (measured: the FP32 pass 1 is slower batched) and run per tile.
  constexpr size_t kBatchWork = (size_t)4 << 30;
  int kb = 1;
  size_t wtile = 0;
  if (gen == SCARL_GEN_PADDED && lay.nb_tiles > 1 && split && dt == 4 && gen_z_tc_supported(P[2])) {
    wtile = (size_t)round_up(P[0] / 2 + 1, 16) * P[1] * lay.Np[2] * 2 * dt;
    kb = (int)std::min<size_t>((size_t)lay.nb_tiles, std::max<size_t>(1, kBatchWork / wtile));
    // an output streamed to the host takes one row of tiles per group, so
    // that the first boxes are final (and copied) early
    if (stream_out || ring_out) kb = std::min(kb, lay.topo_shape[0]);
    if (kb > 1 && ensure(ctx, ctx->work, wtile * kb) != SCARL_OK) kb = 1;  // budget: one tile at a time
  }
  std::vector<GenArgs> grp;
  double* mom_base = nullptr;
  size_t mom_cnt = 0;
  auto padded_args = [&](int r, GenArgs* a) -> int {
    scarl_tile t;
    tile_geometry(&lay, s->xMinGlob, r, &t);
    RC(gen_args(ctx, dt, P, lay.Np, a));
    set_plan(a, pl);
    a->split = split;
    a->k0 = (uint32_t)s->seedBase + 1u + (uint32_t)r;
    a->k1 = 0;
    a->stream = o.stream;
    a->epi = epi;
    for (int d = 0; d < 3; ++d) {
      a->epi.off[d] = t.pos_0[d] - 1;
      a->epi.ax[d] = axes[(size_t)r * 3 + d];
    }
    a->epi.mom = mom_base ? mom_base + 2 * mom_cnt * (size_t)r : nullptr;
    return SCARL_OK;
  };
  // streamed moments: tile r's pass 3 writes mom_cnt FP64 partial pairs at
  // mom_base + 2 mom_cnt r, summed in a fixed order after the last tile
  if (o.moments) {
    GenArgs a0;
    if (gen == SCARL_GEN_PADDED) {
      RC(padded_args(0, &a0));
    } else {
      scarl_tile t0;
      tile_geometry(&lay, s->xMinGlob, 0, &t0);
      RC(shino_args(ctx, lay.Np, t0.xRange, s->corrL, (int32_t)((uint32_t)s->seedBase + 1u), &a0));
    }
    const int c = gen_pass3_partials(gen == SCARL_GEN_PADDED ? dt : 8, a0.var[2], a0);
    if (c < 1) return fail(ctx, SCARL_EDEVICE, "no pass-3 launch for the streamed moments");
    mom_cnt = (size_t)c;
    RC(ensure(ctx, ctx->mom, (2 * mom_cnt * lay.nb_tiles + 2 + 2 * (size_t)pair_sum_parts()) * sizeof(double)));
    mom_base = static_cast<double*>(ctx->mom.p);
  }
  // the moments' pair sum, queued after the last tile; read once the stream is idle
  auto moments_sum = [&]() -> int {
    if (!mom_base) return SCARL_OK;
    CK(launch_pair_sum(mom_base, (int64_t)(mom_cnt * lay.nb_tiles), mom_base + 2 * mom_cnt * lay.nb_tiles + 2,
                       mom_base + 2 * mom_cnt * lay.nb_tiles, ctx->stream));
    return SCARL_OK;
  };
  auto moments_read = [&]() -> int {
    if (!mom_base) return SCARL_OK;
    CK(cudaMemcpyAsync(o.moments, mom_base + 2 * mom_cnt * lay.nb_tiles, 2 * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SCARL_OK;
  };
  const int rc_tiles = [&]() -> int {
    for (int r = 0; r < lay.nb_tiles; ++r) {
      scarl_tile t;
      tile_geometry(&lay, s->xMinGlob, r, &t);
      const int32_t seedStart = (int32_t)((uint32_t)s->seedBase + 1u + (uint32_t)r);
      Epilogue e = epi;
      for (int d = 0; d < 3; ++d) {
        e.off[d] = t.pos_0[d] - 1;
        e.ax[d] = axes[(size_t)r * 3 + d];
      }
      if (gen == SCARL_GEN_PADDED && kb > 1) {
        if (r % kb == 0) {
          const int k = std::min(kb, lay.nb_tiles - r);
          grp.resize(k);
          for (int j = 0; j < k; ++j) {
            RC(padded_args(r + j, &grp[j]));
            grp[j].work = static_cast<char*>(ctx->work.p) + wtile * j;
            philox_schedule(&grp[j]);
          }
          RC(run_passes12_batched(ctx, dt, grp.data(), k));
        }
        Prof p(ctx, c2r_x_tc_used(dt, grp[r % kb]) ? "k_c2r_x_tc" : "k_c2r_x");
        CK(launch_gen_pass(dt, 3, grp[r % kb], ctx->stream));
      } else if (gen == SCARL_GEN_PADDED) {
        GenArgs a;
        RC(padded_args(r, &a));
        RC(run_passes(ctx, dt, a));
      } else if (gen == SCARL_GEN_SHINO) {
        GenArgs a;
        RC(shino_args(ctx, lay.Np, t.xRange, s->corrL, seedStart, &a));
        a.epi = e;
        a.epi.mom = mom_base ? mom_base + 2 * mom_cnt * (size_t)r : nullptr;
        RC(run_passes(ctx, 8, a));
      } else {
        const double* phi = phi_all ? (const double*)phi_all + nk * r : nullptr;
        RC(dct_tile(ctx, (double*)ctx->tile.p, lay.Np, t.xRange, s->corrL, phi, nullptr, (uint32_t)seedStart,
                    gm == SCARL_FFT_MPI));
        Prof p(ctx, "k_blend_tile");
        CK(launch_blend_tile(8, ctx->tile.p, lay.Np, e, ctx->stream));
      }
      if ((stream_out || ring_out) && t.topo_pos[0] == lay.topo_shape[0] - 1) {
        const int ty = t.topo_pos[1], tz = t.topo_pos[2];
        if (stream_out) {
          RC(slab_copy(slabs, row_start(1, ty), row_start(1, ty + 1), row_start(2, tz), row_start(2, tz + 1)));
        } else {
          if (ctx->slab_ev.size() <= ring_nev) {
            cudaEvent_t ev;
            CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            ctx->slab_ev.push_back(ev);
          }
          cudaEvent_t ev = ctx->slab_ev[ring_nev++];
          CK(cudaEventRecord(ev, ctx->stream));
          ring_box(ring_pieces, row_b, plane_b, row_start(1, ty), row_start(1, ty + 1), row_start(2, tz),
                   row_start(2, tz + 1), ev);
        }
      }
    }
    return SCARL_OK;
  }();
  const int rc_slabs = slab_end(slabs);
  RC(rc_tiles);
  RC(rc_slabs);
  RC(moments_sum());
  if (ring_out) {
    if (!ctx->copy_stream) CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    const int rc_ring = ring_copy(ctx, global, dev, plane_b, ring_pieces, ctx->copy_stream);
    CK(cudaStreamSynchronize(ctx->copy_stream));
    RC(rc_ring);
    CK(cudaStreamSynchronize(ctx->stream));
    RC(check_status(ctx));
    RC(moments_read());
    CK(cudaGetLastError());
    return SCARL_OK;
  }
  if (stream_out) {
    CK(cudaStreamSynchronize(ctx->stream));
    RC(check_status(ctx));
    RC(moments_read());
    CK(cudaGetLastError());
    return SCARL_OK;
  }
  if (o.normalize_field) {
    double avg, sd;
    RC(scarl_normalize_field(ctx, dev, dt, (long long)ng, &avg, &sd));
    Prof p(ctx, "k_marginal");
    CK(launch_marginal(dt, dev, (int64_t)ng, s->margiFirst, ms, mmu, ctx->stream));
  }
  RC(finish_out(ctx, global, dev, ng * dt, host));
  return moments_read();
}

// ---- post steps ----
int scarl_apply_unity_partition(scarl_ctx* ctx, double* field, const int Np[3],
                                const int No[3], int partitionType, const int pos[3],
                                const int shape[3]) {
  RC(begin(ctx));
  if (!field || !Np || !No || !pos || !shape) return fail(ctx, SCARL_EINVAL, "null argument");
  const size_t n = (size_t)Np[0] * Np[1] * Np[2];
  void* dev;
  bool host = !is_device_ptr(field);
  if (host) {
    RC(ensure(ctx, ctx->stage_out, n * 8));
    dev = ctx->stage_out.p;
    RC(copy_in(ctx, dev, field, n * 8));
  } else {
    dev = field;
  }
  const size_t nd = 2 * ((size_t)Np[0] + Np[1] + Np[2]);
  void* hp;
  RC(pinned(ctx, nd * 8, &hp));
  RC(ensure(ctx, ctx->tabs, nd * 8));
  double* h = (double*)hp;
  BlendAxis ax[3];
  size_t od = 0;
  for (int d = 0; d < 3; ++d) {
    pou_axis_tables(Np[d], No[d], pos[d], shape[d], partitionType, h + od, h + od + Np[d]);
    ax[d].lo = (const double*)ctx->tabs.p + od;
    ax[d].hi = (const double*)ctx->tabs.p + od + Np[d];
    ax[d].flags = nullptr;
    ax[d].sw64 = nullptr;
    ax[d].sw32 = nullptr;
    od += 2 * (size_t)Np[d];
  }
  RC(upload_pinned(ctx, ctx->tabs.p, nd * 8));
  {
    Prof p(ctx, "k_apply_pou");
    CK(launch_apply_pou(8, dev, Np, ax, ctx->stream));
  }
  return finish_out(ctx, field, dev, n * 8, host);
}

int scarl_add_overlap(scarl_ctx* ctx, double* tiles, const int Np[3], const int No[3],
                      const int shape[3]) {
  RC(begin(ctx));
  if (!tiles || !Np || !No || !shape) return fail(ctx, SCARL_EINVAL, "null argument");
  for (int d = 0; d < 3; ++d)
    if (shape[d] < 1 || No[d] > Np[d] || No[d] < 0) return fail(ctx, SCARL_EINVAL, "invalid topology or overlap");
  const size_t n = (size_t)Np[0] * Np[1] * Np[2] * shape[0] * shape[1] * shape[2];
  RC(ensure(ctx, ctx->tile, n * 8));
  void* dev;
  bool host = !is_device_ptr(tiles);
  if (host) {
    RC(ensure(ctx, ctx->stage_out, n * 8));
    dev = ctx->stage_out.p;
    RC(copy_in(ctx, dev, tiles, n * 8));
  } else {
    dev = tiles;
  }
  CK(cudaMemcpyAsync(ctx->tile.p, dev, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  {
    Prof p(ctx, "k_add_overlap");
    CK(launch_add_overlap((const double*)ctx->tile.p, (double*)dev, Np, No, shape, ctx->stream));
  }
  return finish_out(ctx, tiles, dev, n * 8, host);
}

int scarl_multivariate_transformation(scarl_ctx* ctx, void* field, int dtype, long long n,
                                      double avg, double std_dev, int margiFirst) {
  RC(begin(ctx));
  if (!field || n < 0) return fail(ctx, SCARL_EINVAL, "null argument");
  if (dtype != SCARL_F32 && dtype != SCARL_F64) return fail(ctx, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64");
  double ms, mu;
  RC(marginal_params(ctx, margiFirst, avg, std_dev, &ms, &mu));
  void* dev;
  bool host = !is_device_ptr(field);
  if (host) {
    RC(ensure(ctx, ctx->stage_out, (size_t)n * dtype));
    dev = ctx->stage_out.p;
    RC(copy_in(ctx, dev, field, (size_t)n * dtype));
  } else {
    dev = field;
  }
  {
    Prof p(ctx, "k_marginal");
    CK(launch_marginal(dtype, dev, n, margiFirst, ms, mu, ctx->stream));
  }
  return finish_out(ctx, field, dev, (size_t)n * dtype, host);
}

static int sums(scarl_ctx* ctx, const void* dev, int dtype, long long xN, int nmc,
                std::vector<double>* s, std::vector<double>* s2) {
  const int nb = sums_blocks(xN);
  RC(ensure(ctx, ctx->part, (size_t)nb * nmc * 2 * 8));
  {
    Prof p(ctx, "k_sums");
    CK(launch_sums(dtype, dev, xN, nmc, (double*)ctx->part.p, nb, ctx->stream));
  }
  std::vector<double> h((size_t)nb * nmc * 2);
  CK(cudaMemcpyAsync(h.data(), ctx->part.p, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  s->assign(nmc, 0.0);
  s2->assign(nmc, 0.0);
  for (int e = 0; e < nmc; ++e)
    for (int b = 0; b < nb; ++b) {
      (*s)[e] += h[((size_t)e * nb + b) * 2];
      (*s2)[e] += h[((size_t)e * nb + b) * 2 + 1];
    }
  return SCARL_OK;
}

int scarl_normalize_field(scarl_ctx* ctx, void* field, int dtype, long long n, double* avg,
                          double* sd) {
  RC(begin(ctx));
  if (!field || n <= 0) return fail(ctx, SCARL_EINVAL, "null argument");
  if (dtype != SCARL_F32 && dtype != SCARL_F64) return fail(ctx, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64");
  void* dev;
  bool host = !is_device_ptr(field);
  if (host) {
    RC(ensure(ctx, ctx->stage_out, (size_t)n * dtype));
    dev = ctx->stage_out.p;
    RC(copy_in(ctx, dev, field, (size_t)n * dtype));
  } else {
    dev = field;
  }
  std::vector<double> s, s2;
  RC(sums(ctx, dev, dtype, n, 1, &s, &s2));
  const double a = s[0] / (double)n;
  {
    Prof p(ctx, "k_affine");
    CK(launch_affine(dtype, dev, n, a, 1.0, ctx->stream));
  }
  RC(sums(ctx, dev, dtype, n, 1, &s, &s2));
  const double sdv = std::sqrt(s2[0] / (double)n);
  {
    Prof p(ctx, "k_affine");
    CK(launch_affine(dtype, dev, n, 0.0, sdv, ctx->stream));
  }
  if (avg) *avg = a;
  if (sd) *sd = sdv;
  return finish_out(ctx, field, dev, (size_t)n * dtype, host);
}

// ---- estimators ----
int scarl_moments(scarl_ctx* ctx, const void* field, int dtype, long long xN, int nmc,
                  double* evntAvg, double* evntStd, double* gAvg, double* gStd) {
  RC(begin(ctx));
  if (!field || xN <= 0 || nmc <= 0) return fail(ctx, SCARL_EINVAL, "invalid argument");
  if (dtype != SCARL_F32 && dtype != SCARL_F64) return fail(ctx, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64");
  const void* dev;
  RC(in_dev(ctx, ctx->stage_in, field, (size_t)xN * nmc * dtype, &dev));
  std::vector<double> s, s2;
  RC(sums(ctx, dev, dtype, xN, nmc, &s, &s2));
  double S = 0.0, S2 = 0.0;
  for (int e = 0; e < nmc; ++e) {
    const double a = s[e] / (double)xN;
    if (evntAvg) evntAvg[e] = a;
    if (evntStd) evntStd[e] = std::sqrt(s2[e] / (double)xN - a * a);
    S += s[e];
    S2 += s2[e];
  }
  const double ga = S / (double)(xN * nmc);
  if (gAvg) *gAvg = ga;
  if (gStd) *gStd = std::sqrt(S2 / (double)(xN * nmc) - ga * ga);
  return SCARL_OK;
}

// sums: (sum f, sum f^2) of the field when already known (streamed from the
// generator), so that the moment pass is skipped; NULL = run it.
static int axis_cov_impl(scarl_ctx* ctx, const void* field, int dtype, const int L[3], int maxlag,
                         const double* known_mean, const double* sums, double* mean, double* var,
                         double* cov) {
  RC(begin(ctx));
  if (!field || !L || !mean || !var || !cov) return fail(ctx, SCARL_EINVAL, "null argument");
  if (dtype != SCARL_F32 && dtype != SCARL_F64) return fail(ctx, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64");
  if (maxlag < 0) return fail(ctx, SCARL_EINVAL, "maxlag must be >= 0");
  int Nc[3];
  for (int d = 0; d < 3; ++d) {
    if (L[d] < 1 || maxlag >= L[d]) return fail(ctx, SCARL_EINVAL, "maxlag must be below every extent");
    // smallest padded line M = 2 N >= L + maxlag with a covariance kernel for N
    static const int kCovN[] = {4, 8, 16, 32, 64, 128, 256, 320, 384, 512, 640, 768, 1024, 1280,
                                1536, 2048};
    Nc[d] = 0;
    for (int c : kCovN)
      if (2 * c >= L[d] + maxlag) {
        Nc[d] = c;
        break;
      }
    if (!Nc[d]) return fail(ctx, SCARL_EUNSUPPORTED, "L[d] + maxlag must be <= 4096");
  }
  const size_t n = (size_t)L[0] * L[1] * L[2];
  const void* dev;
  RC(in_dev(ctx, ctx->stage_in, field, n * dtype, &dev));
  // mean (FP64 sums)
  double s1 = 0.0;
  if (sums) {
    s1 = sums[0];
  } else {
    const int nb = sums_blocks((int64_t)n);
    RC(ensure(ctx, ctx->part, (size_t)nb * 2 * 8));
    {
      Prof p(ctx, "k_sums");
      CK(launch_sums(dtype, dev, (int64_t)n, 1, (double*)ctx->part.p, nb, ctx->stream));
    }
    std::vector<double> h((size_t)nb * 2);
    CK(cudaMemcpyAsync(h.data(), ctx->part.p, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->d2h += h.size() * 8;
    for (int b = 0; b < nb; ++b) s1 += h[2 * (size_t)b];
  }
  const double sample_mean = s1 / (double)n;
  const double mu = known_mean ? *known_mean : sample_mean;
  // per axis: power pass, FP64 lag sums
  const int H = maxlag + 1;
  int nblk[3];
  size_t pbytes = 0;
  for (int d = 0; d < 3; ++d) {
    nblk[d] = axis_power_blocks(dtype, L, d, Nc[d]);
    if (nblk[d] < 1) return fail(ctx, SCARL_EDEVICE, "no launch configuration for the covariance pass");
    pbytes = std::max(pbytes, (size_t)nblk[d] * (Nc[d] + 1) * 8);
  }
  RC(ensure(ctx, ctx->t1, pbytes));
  RC(ensure(ctx, ctx->t2, (size_t)(2048 + 1) * 8 + (size_t)3 * H * 8));
  RC(ensure_status(ctx));  // the bounded copy waits of the power pass report here
  double* bins = (double*)ctx->t2.p;
  double* S = bins + 2048 + 1;
  for (int d = 0; d < 3; ++d) {
    const void* tw;
    const void* tw64;
    RC(twiddles(ctx, 2 * Nc[d], dtype, &tw));
    RC(twiddles(ctx, 2 * Nc[d], 8, &tw64));
    {
      Prof p(ctx, "k_axis_power");
      CK(launch_axis_power(dtype, dev, L, d, Nc[d], mu, tw, (double*)ctx->t1.p, nblk[d], ctx->stream,
                           (int*)ctx->status.p));
    }
    {
      Prof p(ctx, "k_cov_lags", 2);
      CK(launch_cov_lags((const double*)ctx->t1.p, nblk[d], Nc[d], maxlag, (const double*)tw64, bins,
                         S + (size_t)d * H, ctx->stream));
    }
  }
  std::vector<double> hs((size_t)3 * H);
  CK(cudaMemcpyAsync(hs.data(), S, hs.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->d2h += hs.size() * 8;
  RC(check_status(ctx));
  for (int d = 0; d < 3; ++d)
    for (int lag = 0; lag < H; ++lag) {
      const double pairs = (double)(L[d] - lag) * (double)(n / (size_t)L[d]);
      cov[(size_t)d * H + lag] = hs[(size_t)d * H + lag] / pairs;
    }
  *mean = sample_mean;
  *var = cov[0];
  return SCARL_OK;
}

int scarl_axis_cov(scarl_ctx* ctx, const void* field, int dtype, const int L[3], int maxlag,
                   const double* known_mean, double* mean, double* var, double* cov) {
  return axis_cov_impl(ctx, field, dtype, L, maxlag, known_mean, nullptr, mean, var, cov);
}

int scarl_axis_cov_sums(scarl_ctx* ctx, const void* field, int dtype, const int L[3], int maxlag,
                        const double sums[2], double* mean, double* var, double* cov) {
  if (!sums) return fail(ctx, SCARL_EINVAL, "null argument");
  return axis_cov_impl(ctx, field, dtype, L, maxlag, nullptr, sums, mean, var, cov);
}

int scarl_rebuild_sk(scarl_ctx* ctx, const void* field, int dtype, const int L[3], double avg,
                     double stdDev, int tukey_literal, double* SkTot) {
  RC(begin(ctx));
  if (!field || !L || !SkTot) return fail(ctx, SCARL_EINVAL, "null argument");
  if (dtype != SCARL_F32 && dtype != SCARL_F64) return fail(ctx, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64");
  for (int d = 0; d < 3; ++d)
    if (L[d] < 2 || L[d] > 4096) return fail(ctx, SCARL_EUNSUPPORTED, "line length must be in [2, 4096]");
  if (!(stdDev > 0.0)) return fail(ctx, SCARL_EINVAL, "stdDev must be > 0");
  const size_t n = (size_t)L[0] * L[1] * L[2];
  const void* dev;
  RC(in_dev(ctx, ctx->stage_in, field, n * dtype, &dev));
  const double r = (double)0.1f;  // SRC_F/Stat_ScaRL/statistics_RF.f90:277
  int off = 0;
  for (int d = 0; d < 3; ++d) {
    const int nl = L[d];
    const int nkeep = nl / 2;
    std::vector<double> w(nl);
    for (int i = 0; i < nl; ++i) {  // statistics_RF.f90:325-351
      const double ratio = (double)i / (double)(nl - 1);
      w[i] = 1.0;
      if (tukey_literal) {
        if (ratio < r) w[i] = 1.0 / 2.0 * (1 + std::cos(2.0 * kPiRef / r * (ratio - r / 2.0)));
        else if (ratio > r) w[i] = 1.0 / 2.0 * (1 + std::cos(2.0 * kPiRef / r * (ratio - 1.0 + r / 2.0)));
      } else {
        if (ratio < r / 2.0) w[i] = 1.0 / 2.0 * (1 + std::cos(2.0 * M_PI / r * (ratio - r / 2.0)));
        else if (ratio > 1.0 - r / 2.0) w[i] = 1.0 / 2.0 * (1 + std::cos(2.0 * M_PI / r * (ratio - 1.0 + r / 2.0)));
      }
    }
    void* hp;
    RC(pinned(ctx, (size_t)nl * 8, &hp));
    std::memcpy(hp, w.data(), (size_t)nl * 8);
    RC(ensure(ctx, ctx->tabs, (size_t)nl * 8));
    RC(upload_pinned(ctx, ctx->tabs.p, (size_t)nl * 8));
    const int np = lag_cov_parts(L, d);
    RC(ensure(ctx, ctx->part, (size_t)np * std::max(nkeep, 1) * 8));
    {
      Prof p(ctx, "k_lag_cov");
      CK(launch_lag_cov(dtype, dev, L, d, avg, stdDev, (const double*)ctx->tabs.p, nkeep,
                        (double*)ctx->part.p, np, ctx->stream));
    }
    std::vector<double> h((size_t)np * nkeep);
    CK(cudaMemcpyAsync(h.data(), ctx->part.p, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double nlines = (double)(n / (size_t)nl);
    for (int m = 0; m < nkeep; ++m) {
      double s = 0.0;
      for (int b = 0; b < np; ++b) s += h[(size_t)b * nkeep + m];
      SkTot[off + m] = s / ((double)nl * nlines);
    }
    off += nkeep;
  }
  return SCARL_OK;
}

}  // extern "C"
