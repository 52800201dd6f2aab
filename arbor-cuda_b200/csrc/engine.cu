// engine.cu - the C++ host: status reporting and the Engine, which restates
// the reference's browser engine (src/engine.js) over the C-ABI entries:
// buffer ownership (:22, :40), generate (:27-34), resize (:35-43),
// frame (:45-53), inspect (:55) and dispose (:57).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "abi_util.h"

namespace arbor {

namespace {
thread_local char g_error[512] = "";
std::atomic<uint64_t> g_launches{0};
}  // namespace

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}
std::atomic<uint64_t>& launch_counter() { return g_launches; }

int launch_sort(uint32_t* Keys, uint32_t* Order, void* scratch, cudaStream_t stream);

}  // namespace arbor

using namespace arbor;

extern "C" const char* arbor_last_error(void) { return g_error; }

extern "C" const char* arbor_status_name(int status) {
  switch (status) {
    case ARBOR_OK: return "ARBOR_OK";
    case ARBOR_ERR_NULL: return "ARBOR_ERR_NULL";
    case ARBOR_ERR_VALUE: return "ARBOR_ERR_VALUE";
    case ARBOR_ERR_ALIGN: return "ARBOR_ERR_ALIGN";
    case ARBOR_ERR_ALIAS: return "ARBOR_ERR_ALIAS";
    case ARBOR_ERR_LIMIT: return "ARBOR_ERR_LIMIT";
    case ARBOR_ERR_CUDA: return "ARBOR_ERR_CUDA";
    case ARBOR_ERR_TIMEOUT: return "ARBOR_ERR_TIMEOUT";
    case ARBOR_ERR_STATE: return "ARBOR_ERR_STATE";
    case ARBOR_ERR_NO_DEVICE: return "ARBOR_ERR_NO_DEVICE";
    default: return "ARBOR_ERR_UNKNOWN";
  }
}

extern "C" int arbor_device_ready(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return 0;
  }
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return 0;
  return major == 10 ? 1 : 0;
}

extern "C" uint64_t arbor_launch_count(void) { return g_launches.load(); }

// ------------------------------------------------------------------ Engine --
struct arbor_engine {
  cudaStream_t stream = nullptr;
  bool single = false;
  bool disposed = false;
  bool timing = false;
  int width = 0, height = 0, seed = -1;
  uint64_t frames = 0;
  arbor_engine_buffers buf{};
  void* scratch = nullptr;
  float* staging = nullptr;  // pinned copy of the input record
  cudaEvent_t input_done = nullptr;
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float ms_build = 0, ms_vis = 0, ms_light = 0, ms_resolve = 0;
  uint64_t scene_bytes = 0, image_bytes_total = 0;
};

namespace {

int cuda_fail(const char* what, cudaError_t e) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  return ARBOR_ERR_CUDA;
}
#define ARBOR_CUDA(call)                                   \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(#call, e_);    \
  } while (0)

void free_images(arbor_engine* e) {
  cudaFree(e->buf.Hit);
  cudaFree(e->buf.Linear);
  cudaFree(e->buf.Guide);
  cudaFree(e->buf.Filtered);
  cudaFree(e->buf.History);
  cudaFree(e->buf.Pixels);
  e->buf.Hit = e->buf.Linear = e->buf.Guide = e->buf.Filtered = e->buf.History = nullptr;
  e->buf.Pixels = nullptr;
  e->image_bytes_total = 0;
}

int live(arbor_engine* e, const char* what) {
  if (e == nullptr) {
    set_error("%s: engine is NULL", what);
    return ARBOR_ERR_NULL;
  }
  if (e->disposed) {
    set_error("%s: renderer was disposed", what);
    return ARBOR_ERR_STATE;
  }
  return ARBOR_OK;
}

// Resolution rounding and limits of src/engine.js:36-37; the binding limit
// is the 256 MiB per storage binding the reference runtime requests
// (runtime.js, GpuRuntime.create).
int round_size(int width, int height, int* w, int* h) {
  if (width <= 0 || height <= 0) {
    set_error("Invalid render dimensions.");
    return ARBOR_ERR_VALUE;
  }
  int64_t rw = ((int64_t)width + 63) / 64 * 64, rh = ((int64_t)height + 7) / 8 * 8;
  if (rw < 320) rw = 320;
  if (rh < 192) rh = 192;
  if (rw > 16384 || rh > 16384 || rw * rh * 16 > 268435456) {
    set_error("Resolution exceeds the adapter limits. Choose a lower width.");
    return ARBOR_ERR_LIMIT;
  }
  *w = (int)rw;
  *h = (int)rh;
  return ARBOR_OK;
}

}  // namespace

extern "C" int arbor_engine_resize(arbor_engine* e, int width, int height) {
  if (int s = live(e, "arbor_engine_resize")) return s;
  int w, h;
  if (int s = round_size(width, height, &w, &h)) return s;
  if (w == e->width && h == e->height) return ARBOR_OK;
  ARBOR_CUDA(cudaStreamSynchronize(e->stream));
  free_images(e);
  size_t img = (size_t)w * h * 16, px = (size_t)w * h * 4;
  ARBOR_CUDA(cudaMalloc(&e->buf.Hit, img));
  ARBOR_CUDA(cudaMalloc(&e->buf.Linear, img));
  ARBOR_CUDA(cudaMalloc(&e->buf.Guide, img));
  ARBOR_CUDA(cudaMalloc(&e->buf.Filtered, img));
  ARBOR_CUDA(cudaMalloc(&e->buf.History, img));
  ARBOR_CUDA(cudaMalloc(&e->buf.Pixels, px));
  ARBOR_CUDA(cudaMemsetAsync(e->buf.History, 0, img, e->stream));
  ARBOR_CUDA(cudaMemsetAsync(e->buf.Pixels, 0, px, e->stream));
  e->image_bytes_total = img * 5 + px;
  e->width = w;
  e->height = h;
  return ARBOR_OK;
}

extern "C" int arbor_engine_generate(arbor_engine* e, int seed) {
  if (int s = live(e, "arbor_engine_generate")) return s;
  if (seed < 0 || seed > 1000000) {
    set_error("Seed must be an integer from 0 to 1,000,000.");
    return ARBOR_ERR_VALUE;
  }
  if (e->timing) ARBOR_CUDA(cudaEventRecord(e->ev[0], e->stream));
  if (int s = arbor_buildScene(seed, e->buf.B, e->buf.P, e->buf.Keys, e->buf.Order, e->buf.Nodes, e->buf.C, e->scratch, e->stream)) return s;
  if (e->buf.History) ARBOR_CUDA(cudaMemsetAsync(e->buf.History, 0, (size_t)e->width * e->height * 16, e->stream));
  if (e->timing) {
    ARBOR_CUDA(cudaEventRecord(e->ev[1], e->stream));
    ARBOR_CUDA(cudaEventSynchronize(e->ev[1]));
    ARBOR_CUDA(cudaEventElapsedTime(&e->ms_build, e->ev[0], e->ev[1]));
  }
  e->seed = seed;
  return ARBOR_OK;
}

extern "C" int arbor_engine_create(arbor_engine** out, int width, int height, int seed, int single_tree, arbor_stream stream) {
  if (out == nullptr) {
    set_error("arbor_engine_create: out is NULL");
    return ARBOR_ERR_NULL;
  }
  *out = nullptr;
  if (!arbor_device_ready()) {
    set_error("arbor_engine_create: no sm_100 CUDA device is available");
    return ARBOR_ERR_NO_DEVICE;
  }
  int w, h;
  if (int s = round_size(width, height, &w, &h)) return s;
  if (seed < 0 || seed > 1000000) {
    set_error("Seed must be an integer from 0 to 1,000,000.");
    return ARBOR_ERR_VALUE;
  }
  arbor_engine* e = new (std::nothrow) arbor_engine();
  if (e == nullptr) {
    set_error("arbor_engine_create: out of host memory");
    return ARBOR_ERR_LIMIT;
  }
  e->stream = stream;
  e->single = single_tree != 0;
  auto fail = [&](int s) {
    arbor_engine_destroy(e);
    return s;
  };
  cudaError_t ce;
  if ((ce = cudaMalloc(&e->buf.B, kB)) != cudaSuccess) return fail(cuda_fail("cudaMalloc B", ce));
  if ((ce = cudaMalloc(&e->buf.P, kP)) != cudaSuccess) return fail(cuda_fail("cudaMalloc P", ce));
  if ((ce = cudaMalloc(&e->buf.Keys, kKeys)) != cudaSuccess) return fail(cuda_fail("cudaMalloc Keys", ce));
  if ((ce = cudaMalloc(&e->buf.Order, kKeys)) != cudaSuccess) return fail(cuda_fail("cudaMalloc Order", ce));
  if ((ce = cudaMalloc(&e->buf.Nodes, kNodes)) != cudaSuccess) return fail(cuda_fail("cudaMalloc Nodes", ce));
  if ((ce = cudaMalloc(&e->buf.C, kC)) != cudaSuccess) return fail(cuda_fail("cudaMalloc C", ce));
  if ((ce = cudaMalloc(&e->buf.I, kI)) != cudaSuccess) return fail(cuda_fail("cudaMalloc I", ce));
  if ((ce = cudaMalloc(&e->scratch, arbor_sort_scratch_bytes())) != cudaSuccess) return fail(cuda_fail("cudaMalloc scratch", ce));
  if ((ce = cudaMallocHost(&e->staging, kI)) != cudaSuccess) return fail(cuda_fail("cudaMallocHost input", ce));
  if ((ce = cudaEventCreateWithFlags(&e->input_done, cudaEventDisableTiming)) != cudaSuccess) return fail(cuda_fail("cudaEventCreate", ce));
  for (auto& ev : e->ev)
    if ((ce = cudaEventCreate(&ev)) != cudaSuccess) return fail(cuda_fail("cudaEventCreate", ce));
  memset(e->staging, 0, kI);
  // Device buffers start zeroed, as WebGPU buffers do.
  if ((ce = cudaMemsetAsync(e->buf.B, 0, kB, stream)) != cudaSuccess) return fail(cuda_fail("cudaMemsetAsync", ce));
  if ((ce = cudaMemsetAsync(e->buf.Nodes, 0, kNodes, stream)) != cudaSuccess) return fail(cuda_fail("cudaMemsetAsync", ce));
  if ((ce = cudaMemsetAsync(e->buf.I, 0, kI, stream)) != cudaSuccess) return fail(cuda_fail("cudaMemsetAsync", ce));
  if ((ce = cudaMemsetAsync(e->buf.C, 0, kC, stream)) != cudaSuccess) return fail(cuda_fail("cudaMemsetAsync", ce));
  e->scene_bytes = kB + kP + 2 * kKeys + kNodes;
  if (int s = arbor_engine_resize(e, w, h)) return fail(s);
  if (int s = arbor_engine_generate(e, seed)) return fail(s);
  if ((ce = cudaStreamSynchronize(stream)) != cudaSuccess) return fail(cuda_fail("cudaStreamSynchronize", ce));
  *out = e;
  return ARBOR_OK;
}

extern "C" int arbor_engine_set_input(arbor_engine* e, const float* input32) {
  if (int s = live(e, "arbor_engine_set_input")) return s;
  if (input32 == nullptr) {
    set_error("arbor_engine_set_input: input is NULL");
    return ARBOR_ERR_NULL;
  }
  for (int i = 0; i < 32; i++)
    if (!std::isfinite(input32[i])) {
      set_error("arbor_engine_set_input: input[%d] must be finite", i);
      return ARBOR_ERR_VALUE;
    }
  // The previous frame's upload must have left the staging buffer.
  ARBOR_CUDA(cudaEventSynchronize(e->input_done));
  memcpy(e->staging, input32, kI);
  return ARBOR_OK;
}

extern "C" int arbor_engine_set_state(arbor_engine* e, const float* state64) {
  if (int s = live(e, "arbor_engine_set_state")) return s;
  if (state64 == nullptr) {
    set_error("arbor_engine_set_state: state is NULL");
    return ARBOR_ERR_NULL;
  }
  for (int i = 0; i < 64; i++)
    if (!std::isfinite(state64[i])) {
      set_error("arbor_engine_set_state: state[%d] must be finite", i);
      return ARBOR_ERR_VALUE;
    }
  ARBOR_CUDA(cudaMemcpyAsync(e->buf.C, state64, kC, cudaMemcpyHostToDevice, e->stream));
  ARBOR_CUDA(cudaStreamSynchronize(e->stream));
  return ARBOR_OK;
}

extern "C" int arbor_engine_set_timing(arbor_engine* e, int enabled) {
  if (int s = live(e, "arbor_engine_set_timing")) return s;
  e->timing = enabled != 0;
  return ARBOR_OK;
}

extern "C" int arbor_engine_frame(arbor_engine* e, float dt) {
  if (int s = live(e, "arbor_engine_frame")) return s;
  if (!std::isfinite(dt)) {
    set_error("arbor_engine_frame: dt must be finite");
    return ARBOR_ERR_VALUE;
  }
  float delta = fmaxf(0.0f, fminf(0.1f, dt));
  const arbor_engine_buffers& b = e->buf;
  cudaStream_t s = e->stream;
  ARBOR_CUDA(cudaMemcpyAsync(b.I, e->staging, kI, cudaMemcpyHostToDevice, s));
  ARBOR_CUDA(cudaEventRecord(e->input_done, s));
  if (e->timing) ARBOR_CUDA(cudaEventRecord(e->ev[1], s));
  // Visibility (src/engine.js:48)
  if (int r = arbor_updateCamera(b.C, b.I, b.P, delta, e->width, e->height, s)) return r;
  int r = e->single ? arbor_traceTreePixels(b.P, b.Nodes, b.Order, b.C, b.Hit, e->width, e->height, s)
                    : arbor_tracePixels(b.P, b.Nodes, b.Order, b.C, b.Hit, e->width, e->height, s);
  if (r) return r;
  if (e->timing) ARBOR_CUDA(cudaEventRecord(e->ev[2], s));
  // Materials and light (:49)
  r = e->single ? arbor_shadeTreePixels(b.P, b.Nodes, b.Order, b.C, b.Hit, b.Linear, b.Guide, e->width, e->height, s)
                : arbor_shadePixels(b.P, b.Nodes, b.Order, b.C, b.Hit, b.Linear, b.Guide, e->width, e->height, s);
  if (r) return r;
  if (e->timing) ARBOR_CUDA(cudaEventRecord(e->ev[3], s));
  // Progressive resolve (:50), filter and resolve fused.
  if ((r = arbor_filterResolve(b.Linear, b.Guide, b.Hit, b.Filtered, b.History, b.Pixels, b.C, e->width, e->height, s))) return r;
  if (e->timing) {
    ARBOR_CUDA(cudaEventRecord(e->ev[4], s));
    ARBOR_CUDA(cudaEventSynchronize(e->ev[4]));
    ARBOR_CUDA(cudaEventElapsedTime(&e->ms_vis, e->ev[1], e->ev[2]));
    ARBOR_CUDA(cudaEventElapsedTime(&e->ms_light, e->ev[2], e->ev[3]));
    ARBOR_CUDA(cudaEventElapsedTime(&e->ms_resolve, e->ev[3], e->ev[4]));
  }
  e->frames++;
  return ARBOR_OK;
}

extern "C" int arbor_engine_inspect(arbor_engine* e, arbor_engine_info* info) {
  if (int s = live(e, "arbor_engine_inspect")) return s;
  if (info == nullptr) {
    set_error("arbor_engine_inspect: info is NULL");
    return ARBOR_ERR_NULL;
  }
  ARBOR_CUDA(cudaMemcpyAsync(info->camera, e->buf.C, kC, cudaMemcpyDeviceToHost, e->stream));
  ARBOR_CUDA(cudaStreamSynchronize(e->stream));
  info->width = e->width;
  info->height = e->height;
  info->seed = e->seed;
  info->single_tree = e->single ? 1 : 0;
  info->frames = e->frames;
  info->scene_bytes = e->scene_bytes;
  info->allocated_bytes = e->scene_bytes + kC + kI + arbor_sort_scratch_bytes() + e->image_bytes_total;
  info->launches_per_frame = 6;  // updateCamera, trace, shadow setup + shadow pass + compose (shadePixels), filterResolve
  info->ms_build = e->ms_build;
  info->ms_visibility = e->ms_vis;
  info->ms_lighting = e->ms_light;
  info->ms_resolve = e->ms_resolve;
  return ARBOR_OK;
}

extern "C" int arbor_engine_buffers_get(arbor_engine* e, arbor_engine_buffers* out) {
  if (int s = live(e, "arbor_engine_buffers_get")) return s;
  if (out == nullptr) {
    set_error("arbor_engine_buffers_get: out is NULL");
    return ARBOR_ERR_NULL;
  }
  *out = e->buf;
  return ARBOR_OK;
}

extern "C" int arbor_engine_read_pixels(arbor_engine* e, uint32_t* host, size_t count) {
  if (int s = live(e, "arbor_engine_read_pixels")) return s;
  if (host == nullptr) {
    set_error("arbor_engine_read_pixels: host is NULL");
    return ARBOR_ERR_NULL;
  }
  if (count < (size_t)e->width * e->height) {
    set_error("arbor_engine_read_pixels: %zu elements cannot hold %d x %d pixels", count, e->width, e->height);
    return ARBOR_ERR_LIMIT;
  }
  ARBOR_CUDA(cudaMemcpyAsync(host, e->buf.Pixels, (size_t)e->width * e->height * 4, cudaMemcpyDeviceToHost, e->stream));
  ARBOR_CUDA(cudaStreamSynchronize(e->stream));
  return ARBOR_OK;
}

extern "C" int arbor_engine_dispose(arbor_engine* e) {
  if (e == nullptr) return ARBOR_OK;
  if (e->disposed) return ARBOR_OK;
  cudaStreamSynchronize(e->stream);
  e->disposed = true;
  free_images(e);
  cudaFree(e->buf.B);
  cudaFree(e->buf.P);
  cudaFree(e->buf.Keys);
  cudaFree(e->buf.Order);
  cudaFree(e->buf.Nodes);
  cudaFree(e->buf.C);
  cudaFree(e->buf.I);
  cudaFree(e->scratch);
  e->buf = arbor_engine_buffers{};
  e->scratch = nullptr;
  if (e->staging) cudaFreeHost(e->staging);
  e->staging = nullptr;
  if (e->input_done) cudaEventDestroy(e->input_done);
  e->input_done = nullptr;
  for (auto& ev : e->ev) {
    if (ev) cudaEventDestroy(ev);
    ev = nullptr;
  }
  return ARBOR_OK;
}

extern "C" int arbor_engine_destroy(arbor_engine* e) {
  if (e == nullptr) return ARBOR_OK;
  arbor_engine_dispose(e);
  delete e;
  return ARBOR_OK;
}

// ------------------------------------------------------------ image files --
// Binary PPM exactly as the harness writes it (tests/native_harness.cpp:53):
// "P6\n<w> <h>\n255\n", then R, G, B bytes per pixel (R is Pixels' low byte).
extern "C" int arbor_write_ppm(const char* path, const uint32_t* pixels, int width, int height) {
  if (path == nullptr || pixels == nullptr) {
    set_error("arbor_write_ppm: path and pixels must not be NULL");
    return ARBOR_ERR_NULL;
  }
  if (width <= 0 || height <= 0) {
    set_error("arbor_write_ppm: %d x %d is not an image", width, height);
    return ARBOR_ERR_VALUE;
  }
  FILE* f = fopen(path, "wb");
  if (f == nullptr) {
    set_error("arbor_write_ppm: cannot open %s", path);
    return ARBOR_ERR_VALUE;
  }
  fprintf(f, "P6\n%d %d\n255\n", width, height);
  std::vector<unsigned char> row((size_t)width * 3);
  bool ok = true;
  for (int y = 0; y < height && ok; y++) {
    for (int x = 0; x < width; x++) {
      const uint32_t p = pixels[(size_t)y * width + x];
      row[3 * x] = (unsigned char)(p & 255u);
      row[3 * x + 1] = (unsigned char)((p >> 8) & 255u);
      row[3 * x + 2] = (unsigned char)((p >> 16) & 255u);
    }
    ok = fwrite(row.data(), 1, row.size(), f) == row.size();
  }
  if (fclose(f) != 0) ok = false;
  if (!ok) {
    set_error("arbor_write_ppm: write to %s failed", path);
    return ARBOR_ERR_VALUE;
  }
  return ARBOR_OK;
}

// Portable float map of an RGBA float image (Linear, Guide, Filtered, ...):
// "PF\n<w> <h>\n-1.0\n", then little-endian float RGB rows, bottom row first.
extern "C" int arbor_write_pfm(const char* path, const float* rgba, int width, int height) {
  if (path == nullptr || rgba == nullptr) {
    set_error("arbor_write_pfm: path and rgba must not be NULL");
    return ARBOR_ERR_NULL;
  }
  if (width <= 0 || height <= 0) {
    set_error("arbor_write_pfm: %d x %d is not an image", width, height);
    return ARBOR_ERR_VALUE;
  }
  FILE* f = fopen(path, "wb");
  if (f == nullptr) {
    set_error("arbor_write_pfm: cannot open %s", path);
    return ARBOR_ERR_VALUE;
  }
  fprintf(f, "PF\n%d %d\n-1.0\n", width, height);
  std::vector<float> row((size_t)width * 3);
  bool ok = true;
  for (int y = height - 1; y >= 0 && ok; y--) {
    for (int x = 0; x < width; x++)
      for (int c = 0; c < 3; c++) row[3 * x + c] = rgba[((size_t)y * width + x) * 4 + c];
    ok = fwrite(row.data(), sizeof(float), row.size(), f) == row.size();
  }
  if (fclose(f) != 0) ok = false;
  if (!ok) {
    set_error("arbor_write_pfm: write to %s failed", path);
    return ARBOR_ERR_VALUE;
  }
  return ARBOR_OK;
}

// The engine's current Pixels as a PPM (Renderer::save, native_harness.cpp:53).
extern "C" int arbor_engine_save_ppm(arbor_engine* e, const char* path) {
  if (int s = live(e, "arbor_engine_save_ppm")) return s;
  std::vector<uint32_t> px((size_t)e->width * e->height);
  if (int s = arbor_engine_read_pixels(e, px.data(), px.size())) return s;
  return arbor_write_ppm(path, px.data(), e->width, e->height);
}
