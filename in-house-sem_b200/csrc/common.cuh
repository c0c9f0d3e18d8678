// Shared host/device infrastructure of the insem B200 backend: status
// handling behind the C ABI, device buffers, launch checks and the
// IEEE-ordered float helpers every kernel uses.
//
// Arithmetic contract: the reference's float build on x86-64 rounds every
// product and sum separately (no FMA contraction; the INSEM_STRICT_FP build
// is bit-identical to the default one there).  All kernels therefore build
// their sums from __fmul_rn / __fadd_rn (never contracted), in the order the
// reference writes them, and the library is compiled with -fmad=false so
// that double arithmetic (Stacey solves, receivers, energy) is not
// contracted either.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <set>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/insem_cuda.h"

namespace insem_b200 {

// ------------------------------------------------------------------ errors
// Error carrying a C-ABI status code; thrown inside the library and turned
// into a return code plus thread-local message at the boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

void set_last_error(const std::string& msg);
const char* last_error();

#define INSEM_REQUIRE(cond, code, msg)                                          \
  do {                                                                          \
    if (!(cond)) throw ::insem_b200::Error((code), std::string(msg));           \
  } while (0)

#define CUDA_CHECK(expr)                                                        \
  do {                                                                          \
    cudaError_t err__ = (expr);                                                 \
    if (err__ != cudaSuccess)                                                   \
      throw ::insem_b200::Error(INSEM_CUDA_ERR_CUDA,                            \
                                std::string(#expr) + ": " + cudaGetErrorString(err__)); \
  } while (0)

#define CUDA_LAUNCH_CHECK()                                                     \
  do {                                                                          \
    cudaError_t err__ = cudaGetLastError();                                     \
    if (err__ != cudaSuccess)                                                   \
      throw ::insem_b200::Error(INSEM_CUDA_ERR_CUDA, std::string("kernel launch at ") + __FILE__ + ":" + \
                                std::to_string(__LINE__) + ": " + cudaGetErrorString(err__)); \
  } while (0)

// Runs `fn` and converts exceptions to a status code (C-ABI wrapper).
template <class Fn>
int guarded(Fn&& fn) {
  try {
    fn();
    set_last_error("");
    return INSEM_CUDA_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host memory allocation failed");
    return INSEM_CUDA_ERR_NOMEM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return INSEM_CUDA_ERR_INVALID;
  }
}

// ------------------------------------------------------------ device memory
// Device memory comes from the current device's default stream-ordered pool,
// in the legacy stream's order, and freed memory stays in the pool: freeing
// does not wait for the whole device (as cudaFree does) and does not hand
// memory back to the system, so solves can come and go while others run.
// An owner frees memory only after its own stream has finished with it.
inline void keep_pool_memory(int device) {
  static std::mutex mu;
  static std::set<int> done;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(device)) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done.insert(device);
}

// Allocates `bytes` on the current device; usable on every stream on return.
inline void* device_alloc(std::size_t bytes) {
  int device = 0;
  CUDA_CHECK(cudaGetDevice(&device));
  keep_pool_memory(device);
  void* p = nullptr;
  const cudaError_t e = cudaMallocAsync(&p, bytes, nullptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(INSEM_CUDA_ERR_NOMEM, "device allocation of " + std::to_string(bytes) +
                                          " bytes failed: " + cudaGetErrorString(e));
  }
  CUDA_CHECK(cudaStreamSynchronize(nullptr));
  return p;
}

// Returns memory to the pool (the current device must be the one it came from).
inline void device_free(void* p) {
  if (p) cudaFreeAsync(p, nullptr);
}

// Owning device buffer.  Allocation failures report INSEM_CUDA_ERR_NOMEM.
template <class T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(std::size_t n) { resize(n); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_;
      n_ = o.n_;
      o.p_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  void resize(std::size_t n) {
    release();
    if (n == 0) return;
    p_ = static_cast<T*>(device_alloc(n * sizeof(T)));
    n_ = n;
  }
  void upload(const T* host, std::size_t n) {
    resize(n);
    if (n) {
      CUDA_CHECK(cudaMemcpy(p_, host, n * sizeof(T), cudaMemcpyHostToDevice));
      // a copy from pageable memory may return before its DMA has landed;
      // consumers run on other (non-blocking) streams
      CUDA_CHECK(cudaStreamSynchronize(nullptr));
    }
  }
  void upload(const std::vector<T>& v) { upload(v.data(), v.size()); }
  // For buffers only stream `s` uses: (re)allocates from the pool and copies
  // in s's order, without waiting for the legacy stream (a new size frees the
  // old memory, which `s` must no longer be using).
  void upload_async(const std::vector<T>& v, cudaStream_t s) {
    if (v.size() != n_) {
      release();
      if (!v.empty()) {
        int device = 0;
        CUDA_CHECK(cudaGetDevice(&device));
        keep_pool_memory(device);
        void* p = nullptr;
        const cudaError_t e = cudaMallocAsync(&p, v.size() * sizeof(T), s);
        if (e != cudaSuccess) {
          cudaGetLastError();
          throw Error(INSEM_CUDA_ERR_NOMEM, "device allocation of " + std::to_string(v.size() * sizeof(T)) +
                                                " bytes failed: " + cudaGetErrorString(e));
        }
        p_ = static_cast<T*>(p);
        n_ = v.size();
      }
    }
    if (!v.empty()) CUDA_CHECK(cudaMemcpyAsync(p_, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void zero(cudaStream_t s = nullptr) {
    if (n_) CUDA_CHECK(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
  }
  std::vector<T> download() const {
    std::vector<T> out(n_);
    if (n_) CUDA_CHECK(cudaMemcpy(out.data(), p_, n_ * sizeof(T), cudaMemcpyDeviceToHost));
    return out;
  }
  T* get() { return p_; }
  const T* get() const { return p_; }
  std::size_t size() const { return n_; }
  std::size_t bytes() const { return n_ * sizeof(T); }

 private:
  void release() {
    device_free(p_);
    p_ = nullptr;
    n_ = 0;
  }
  T* p_ = nullptr;
  std::size_t n_ = 0;
};

// Copies a host array given by pointer and count (nullptr allowed when n == 0).
template <class T>
std::vector<T> host_vec(const T* p, std::size_t n) {
  if (n == 0) return {};
  INSEM_REQUIRE(p != nullptr, INSEM_CUDA_ERR_INVALID, "null array pointer for a non-empty array");
  return std::vector<T>(p, p + n);
}

// Makes `device` current for the lifetime of the guard.
class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    CUDA_CHECK(cudaGetDevice(&old_));
    if (device != old_) CUDA_CHECK(cudaSetDevice(device));
  }
  ~DeviceGuard() { cudaSetDevice(old_); }

 private:
  int old_ = 0;
};

// ------------------------------------------------- IEEE-ordered arithmetic
// Round-to-nearest operations that the compiler never fuses: sums and
// products are evaluated exactly as the reference writes them.
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }
// Grid of a grid-stride loop over n items (at most 16 CTAs per SM of a B200).
inline int grid_for(int64_t n, int threads = 256) {
  const int64_t g = (n + threads - 1) / threads;
  return static_cast<int>(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace insem_b200
