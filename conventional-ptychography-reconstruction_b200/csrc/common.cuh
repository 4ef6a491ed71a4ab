// common.cuh -- shared device helpers for the ptychography kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/ptycho_b200.h"

#define PTY_DEVI __device__ __forceinline__

PTY_DEVI float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
PTY_DEVI float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
PTY_DEVI float2 c_mul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
PTY_DEVI float2 c_mulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
PTY_DEVI float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
PTY_DEVI float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
PTY_DEVI float2 c_negif(float2 a, int odd) { return odd ? make_float2(-a.x, -a.y) : a; }
// acc += a * conj(b), as two FMAs per component
PTY_DEVI void c_fma_conj(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, fmaf(a.y, b.y, acc.x));
  acc.y = fmaf(a.y, b.x, fmaf(-a.x, b.y, acc.y));
}

// Record an error code in a device status word (first writer wins; never cleared).
PTY_DEVI void pty_raise(int32_t* status, int code) {
  if (status) atomicCAS(reinterpret_cast<int*>(status), 0, code);
}

static inline bool pty_aligned(const void* p, size_t a) {
  return (reinterpret_cast<uintptr_t>(p) % a) == 0;
}
static inline size_t pty_align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
__host__ __device__ constexpr size_t pty_align_up_c(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Per-device cache of a launch set-up value that is computed once per device
// (a resident-CTA count, an SM count, "the shared-memory attribute is set");
// 0 means not yet known.  Entries are atomics, so host threads may race on
// them: two threads that both miss compute and store the same value.  A
// device reset drops a kernel's shared-memory attribute, so a launcher that
// caches "attribute set" clears its entry and sets it again when a launch is
// refused (static storage: every entry starts at 0).
constexpr int kPtyMaxDevices = 64;
struct PtyDevCache {
  std::atomic<int> v[kPtyMaxDevices];
  // the cached value of the current device, or 0; dev_out receives the device
  int get(int* dev_out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kPtyMaxDevices) {
      *dev_out = -1;
      return 0;
    }
    *dev_out = dev;
    return v[dev].load(std::memory_order_relaxed);
  }
  void put(int dev, int x) {
    if (dev >= 0 && dev < kPtyMaxDevices) v[dev].store(x, std::memory_order_relaxed);
  }
};
