// abi_util.h - host-side argument checks, status reporting and launch
// accounting shared by every C-ABI entry point.
//
// The checks restate the reference runtime's binding/dispatch validation
// (vendor/cuda-webshader/runtime/runtime.js:18-22 scalar finiteness,
// :323-325 record size and writable aliasing, :352 workgroup limits) for raw
// device pointers whose sizes follow from the ABI.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/arbor.h"

namespace arbor {

void set_error(const char* fmt, ...);
std::atomic<uint64_t>& launch_counter();

inline void count_launch(uint64_t n = 1) { launch_counter().fetch_add(n, std::memory_order_relaxed); }

// One binding: base pointer, size in bytes, writable flag, required alignment.
struct Binding {
  const void* ptr;
  size_t bytes;
  bool writable;
  size_t align;
  const char* name;
};

// Null / alignment / writable-aliasing checks over one entry's bindings.
template <int N>
inline int check_bindings(const char* entry, const Binding (&b)[N]) {
  for (int i = 0; i < N; i++) {
    if (b[i].ptr == nullptr) {
      set_error("%s: buffer %s is NULL", entry, b[i].name);
      return ARBOR_ERR_NULL;
    }
    if ((reinterpret_cast<uintptr_t>(b[i].ptr) % b[i].align) != 0) {
      set_error("%s: buffer %s is not %zu-byte aligned", entry, b[i].name, b[i].align);
      return ARBOR_ERR_ALIGN;
    }
  }
  for (int i = 0; i < N; i++)
    for (int j = i + 1; j < N; j++) {
      if (!b[i].writable && !b[j].writable) continue;
      uintptr_t a0 = reinterpret_cast<uintptr_t>(b[i].ptr), a1 = a0 + b[i].bytes;
      uintptr_t c0 = reinterpret_cast<uintptr_t>(b[j].ptr), c1 = c0 + b[j].bytes;
      if (a0 < c1 && c0 < a1) {
        set_error("%s: writable buffer aliasing across bindings %s and %s is rejected", entry, b[i].name, b[j].name);
        return ARBOR_ERR_ALIAS;
      }
    }
  return ARBOR_OK;
}

// Image size checks: negative is an error, zero is a no-op (the runtime
// skips a dispatch with a zero workgroup count), more than 65535 workgroups
// of 8 pixels per dimension is an error, and the pixel index must fit int32.
inline int check_image(const char* entry, int width, int height, bool* empty) {
  *empty = false;
  if (width < 0 || height < 0) {
    set_error("%s: width and height must be non-negative (got %d x %d)", entry, width, height);
    return ARBOR_ERR_VALUE;
  }
  if (width == 0 || height == 0) {
    *empty = true;
    return ARBOR_OK;
  }
  if ((width + 7) / 8 > 65535 || (height + 7) / 8 > 65535) {
    set_error("%s: %d x %d needs more than 65535 workgroups per dimension", entry, width, height);
    return ARBOR_ERR_LIMIT;
  }
  if ((uint64_t)width * (uint64_t)height * 4u > 0x7fffffffull) {
    set_error("%s: %d x %d exceeds the 2^31 float index range of one image buffer", entry, width, height);
    return ARBOR_ERR_LIMIT;
  }
  return ARBOR_OK;
}

inline int check_launch(const char* entry) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: launch failed: %s", entry, cudaGetErrorString(e));
    return ARBOR_ERR_CUDA;
  }
  return ARBOR_OK;
}

constexpr size_t kB = 4u * 2109u * 20u;
constexpr size_t kP = 4u * 32768u * 24u;
constexpr size_t kKeys = 4u * 32768u;
constexpr size_t kNodes = 4u * 65536u * 8u;
constexpr size_t kC = 4u * 64u;
constexpr size_t kI = 4u * 32u;
inline size_t image_bytes(int w, int h) { return (size_t)w * (size_t)h * 16u; }
inline size_t pixel_bytes(int w, int h) { return (size_t)w * (size_t)h * 4u; }

}  // namespace arbor
