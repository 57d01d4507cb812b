// nb_stage.cu -- copies between large pageable host arrays and device memory through pinned
// staging buffers, the host CPU copy split over several threads.
//
// The drop-in operators take host (numpy) arrays like the reference's petprj, whose
// osem_rec copies ~1.8 GB of sinograms and sensitivity images from pageable memory on
// every call (prj/src/prj_module.cu:613-839, recon.cu:334-419).  A pageable cudaMemcpy goes
// through one driver-side bounce buffer filled by one CPU thread.  Here each chunk of the
// source is copied into one of a ring of pinned buffers by several host threads at once
// while the DMA engine moves the previous chunk, so the copy runs at the speed of a
// multi-threaded memcpy instead of a single-threaded one.
//
// The staging ring (NB_STAGE_SLOTS pinned buffers of NB_STAGE_CHUNK bytes) is allocated on
// the first call on a device and kept until the process exits.  Calls on one device are
// serialised by a mutex.  Host -> device: like a pageable-source cudaMemcpyAsync, a call
// returns once the whole source has been read into staging memory (the caller may reuse it
// at once); the DMAs themselves are ordered on the caller's stream.  Device -> host: the
// copy is ordered after the stream's earlier work and the call returns when the host array
// holds the data; while the host threads unpack one chunk the DMA engine fills the next.
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "nb_internal.cuh"

#define NB_STAGE_SLOTS 8
#define NB_STAGE_CHUNK ((size_t)8 << 20)

namespace {

struct Stage {
  unsigned char *buf[NB_STAGE_SLOTS] = {};
  cudaEvent_t done[NB_STAGE_SLOTS] = {};
  bool ready = false;
  std::mutex mu;
};

Stage g_stage[64];
std::mutex g_init_mu;

int stage_init(Stage &s) {
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (s.ready) return NB_OK;
  for (int k = 0; k < NB_STAGE_SLOTS; k++) {
    NB_CUDA(cudaHostAlloc((void **)&s.buf[k], NB_STAGE_CHUNK, cudaHostAllocPortable));
    NB_CUDA(cudaEventCreateWithFlags(&s.done[k], cudaEventDisableTiming));
  }
  s.ready = true;
  return NB_OK;
}

int copy_threads() {
  const unsigned hc = std::thread::hardware_concurrency();
  const int n = hc == 0 ? 4 : (int)hc;
  return n > 16 ? 16 : n;
}

// A pool of copy threads, started on first use and kept for the life of the process (they
// sleep on a condition variable between copies; starting threads for every chunk cost as
// much as the copy of a small chunk).  run() splits one memcpy into parts, hands them to
// the workers, copies a part itself and returns when every part is done.  Callers hold
// their device's staging mutex; the pool serialises callers of different devices.
class CopyPool {
 public:
  explicit CopyPool(int nthr) {
    for (int t = 0; t < nthr - 1; t++) std::thread([this] { work(); }).detach();
  }
  void run(unsigned char *dst, const unsigned char *src, size_t n, int nparts) {
    std::lock_guard<std::mutex> one(call_mu_);
    const size_t part = ((n / nparts) + 4095) & ~(size_t)4095;
    {
      std::lock_guard<std::mutex> lk(mu_);
      dst_ = dst;
      src_ = src;
      n_ = n;
      part_ = part;
      next_ = 0;
      left_ = (n + part - 1) / part;
      ++gen_;
    }
    cv_.notify_all();
    take();
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [this] { return left_ == 0; });
  }

 private:
  // copy parts until none is left to start
  void take() {
    for (;;) {
      size_t k, off, len;
      unsigned char *d;
      const unsigned char *s;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (next_ * part_ >= n_) return;
        k = next_++;
        off = k * part_;
        len = off + part_ < n_ ? part_ : n_ - off;
        d = dst_;
        s = src_;
      }
      memcpy(d + off, s + off, len);
      std::lock_guard<std::mutex> lk(mu_);
      if (--left_ == 0) done_.notify_all();
    }
  }
  void work() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
      }
      take();
    }
  }
  std::mutex call_mu_, mu_;
  std::condition_variable cv_, done_;
  unsigned char *dst_ = nullptr;
  const unsigned char *src_ = nullptr;
  size_t n_ = 0, part_ = 1, next_ = 0, left_ = 0;
  uint64_t gen_ = 0;
};

CopyPool &copy_pool() {
  static CopyPool *p = new CopyPool(copy_threads());  // never destroyed: workers outlive exit
  return *p;
}

// memcpy of n bytes split over nthr parts copied by the pool and the calling thread
void par_copy(unsigned char *dst, const unsigned char *src, size_t n, int nthr) {
  if (nthr <= 1 || n < ((size_t)1 << 20)) {
    memcpy(dst, src, n);
    return;
  }
  copy_pool().run(dst, src, n, nthr);
}

}  // namespace

extern "C" int nb_copy_h2d(void *dst, const void *src, size_t bytes, void *stream) {
  NB_RANGE("nb_copy_h2d");
  NB_REQUIRE(bytes == 0 || (dst && src), "nb_copy_h2d: NULL pointer");
  if (bytes == 0) return NB_OK;
  int dev = 0;
  NB_CUDA(cudaGetDevice(&dev));
  NB_REQUIRE(dev >= 0 && dev < 64, "nb_copy_h2d: device index above 63");
  Stage &s = g_stage[dev];
  int st = stage_init(s);
  if (st) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  const int nthr = copy_threads();
  std::lock_guard<std::mutex> lk(s.mu);
  unsigned char *d = static_cast<unsigned char *>(dst);
  const unsigned char *h = static_cast<const unsigned char *>(src);
  int slot = 0;
  for (size_t off = 0; off < bytes; off += NB_STAGE_CHUNK) {
    const size_t n = bytes - off < NB_STAGE_CHUNK ? bytes - off : NB_STAGE_CHUNK;
    // the slot's previous DMA (this call's or an earlier one's) must have left the buffer
    NB_CUDA(cudaEventSynchronize(s.done[slot]));
    par_copy(s.buf[slot], h + off, n, nthr);
    NB_CUDA(cudaMemcpyAsync(d + off, s.buf[slot], n, cudaMemcpyHostToDevice, cs));
    NB_CUDA(cudaEventRecord(s.done[slot], cs));
    slot = (slot + 1) % NB_STAGE_SLOTS;
  }
  return NB_OK;
}

extern "C" int nb_copy_d2h(void *dst, const void *src, size_t bytes, void *stream) {
  NB_RANGE("nb_copy_d2h");
  NB_REQUIRE(bytes == 0 || (dst && src), "nb_copy_d2h: NULL pointer");
  if (bytes == 0) return NB_OK;
  int dev = 0;
  NB_CUDA(cudaGetDevice(&dev));
  NB_REQUIRE(dev >= 0 && dev < 64, "nb_copy_d2h: device index above 63");
  Stage &s = g_stage[dev];
  int st = stage_init(s);
  if (st) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  const int nthr = copy_threads();
  std::lock_guard<std::mutex> lk(s.mu);
  unsigned char *h = static_cast<unsigned char *>(dst);
  const unsigned char *d = static_cast<const unsigned char *>(src);
  const size_t nchunk = (bytes + NB_STAGE_CHUNK - 1) / NB_STAGE_CHUNK;
  // keep up to NB_STAGE_SLOTS chunks in flight; unpack them in order
  size_t issued = 0;
  auto issue = [&](size_t c) -> cudaError_t {
    const int slot = (int)(c % NB_STAGE_SLOTS);
    const size_t off = c * NB_STAGE_CHUNK;
    const size_t n = bytes - off < NB_STAGE_CHUNK ? bytes - off : NB_STAGE_CHUNK;
    cudaError_t e = cudaEventSynchronize(s.done[slot]);  // an earlier use of the slot
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.buf[slot], d + off, n, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaEventRecord(s.done[slot], cs);
    return e;
  };
  for (; issued < nchunk && issued < NB_STAGE_SLOTS; issued++) NB_CUDA(issue(issued));
  for (size_t c = 0; c < nchunk; c++) {
    const int slot = (int)(c % NB_STAGE_SLOTS);
    const size_t off = c * NB_STAGE_CHUNK;
    const size_t n = bytes - off < NB_STAGE_CHUNK ? bytes - off : NB_STAGE_CHUNK;
    NB_CUDA(cudaEventSynchronize(s.done[slot]));
    par_copy(h + off, s.buf[slot], n, nthr);
    if (issued < nchunk) NB_CUDA(issue(issued++));
  }
  return NB_OK;
}
