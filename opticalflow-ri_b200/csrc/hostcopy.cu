// Host-side copies of the host-buffer calls.
//
// A call with numpy frames (the reference's own call pattern) moves each frame into a
// pinned staging buffer before its asynchronous upload and each result out of one after
// its download.  One core's memcpy moves ~16 GB/s, so four 4 MB planes cost ~1 ms per
// 1024^2 pair, more than the uploads themselves.  of_host_copy splits a large copy over a
// small persistent pool of threads (the caller copies one slice itself).  Python reaches
// it through ctypes, which releases the interpreter lock for the call.
#include <string.h>
#include <unistd.h>

#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"

namespace {

class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool* p = new CopyPool();  // never destroyed: workers may outlive static teardown
    return *p;
  }
  bool usable() const { return getpid() == pid_; }  // a forked child has none of the workers
  void copy(char* dst, const char* src, size_t bytes) {
    std::lock_guard<std::mutex> one(call_mu_);  // one pooled copy at a time
    {
      std::lock_guard<std::mutex> g(mu_);
      dst_ = dst;
      src_ = src;
      bytes_ = bytes;
      pending_ = (int)workers_.size();
      ++gen_;
    }
    cv_.notify_all();
    part(0);
    std::unique_lock<std::mutex> g(mu_);
    done_.wait(g, [&] { return pending_ == 0; });
  }

 private:
  CopyPool() : pid_(getpid()) {
    unsigned hc = std::thread::hardware_concurrency();
    int n = hc > 1 ? (int)(hc / 2) : 1;
    if (n > 8) n = 8;
    parts_ = n;
    for (int i = 1; i < n; i++) workers_.emplace_back([this, i] { loop(i); });
    for (auto& t : workers_) t.detach();
  }
  void part(int i) const {
    size_t per = (bytes_ + parts_ - 1) / parts_;
    per = (per + 4095) & ~(size_t)4095;  // page-aligned slices
    const size_t b = (size_t)i * per;
    if (b >= bytes_) return;
    const size_t e = b + per < bytes_ ? b + per : bytes_;
    memcpy(dst_ + b, src_ + b, e - b);
  }
  void loop(int i) {
    unsigned seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> g(mu_);
      cv_.wait(g, [&] { return gen_ != seen; });
      seen = gen_;
      g.unlock();
      part(i);
      g.lock();
      if (--pending_ == 0) done_.notify_one();
    }
  }

  const pid_t pid_;
  int parts_ = 1;
  std::vector<std::thread> workers_;
  std::mutex call_mu_, mu_;
  std::condition_variable cv_, done_;
  char* dst_ = nullptr;
  const char* src_ = nullptr;
  size_t bytes_ = 0;
  int pending_ = 0;
  unsigned gen_ = 0;
};

}  // namespace

extern "C" int of_host_copy(void* dst, const void* src, size_t bytes) {
  OF_REQUIRE(bytes == 0 || (dst && src), "of_host_copy: null buffer");
  OF_REQUIRE(bytes == 0 || (const char*)dst + bytes <= (const char*)src || (const char*)src + bytes <= (const char*)dst,
             "of_host_copy: the buffers overlap");
  if (bytes < ((size_t)1 << 20) || !CopyPool::get().usable()) {
    if (bytes) memcpy(dst, src, bytes);
    return OF_OK;
  }
  CopyPool::get().copy(static_cast<char*>(dst), static_cast<const char*>(src), bytes);
  return OF_OK;
}
