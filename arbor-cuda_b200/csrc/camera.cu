// camera.cu - initCamera / updateCamera (Arbor.cu:179-182): single-thread
// kernels that write the 64-float camera/state record C.
//
// C fields: 0..2 eye, 3 display distance, 4..6 look-at point, 8 time,
// 9 sample index, 10 history reset, 11 wind amplitude, 12/13 sun azimuth /
// elevation, 14 FOV scale, 15 view mode, 16/17 yaw/pitch, 20 exposure,
// 22 shadows, 24 frame counter, 31 world seed, 32/33 width/height.
#include <cmath>
#include <mutex>

#include "abi_util.h"
#include "arbor_math.cuh"

namespace arbor {
namespace {

// Arbor.cu:179
__device__ void fps_pose(float* C, f3 eye, float yaw, float pitch) {
  C[16] = yaw;
  C[17] = pitch;
  C[27] = yaw;
  C[28] = pitch;
  st3(C, 0, eye);
  float cp = xcos(pitch);
  f3 f = norm3(mk(xsin(yaw) * cp, xsin(pitch), xcos(yaw) * cp));
  st3(C, 4, eye + f);
  C[3] = 1.0f;
  C[18] = 1.0f;
}
// Arbor.cu:180
__device__ void view_preset(float* C, int preset) {
  if (preset == 1) fps_pose(C, mk(2.0f, 1.72f, 18.0f), kPi, 0.0f);
  if (preset == 2) fps_pose(C, mk(-1.4f, 1.72f, 7.0f), kPi * 0.94f, 0.02f);
  if (preset == 3) fps_pose(C, mk(8.0f, 1.72f, -3.0f), kPi * 0.55f, -0.02f);
  if (preset == 4) fps_pose(C, mk(-11.0f, 1.72f, -7.0f), 0.65f, 0.03f);
  if (preset == 5) fps_pose(C, mk(0.0f, 12.0f, 72.0f), kPi, -0.12f);
  C[9] = 0.0f;
  C[10] = 1.0f;
}
// Arbor.cu:181
__global__ void init_camera_kernel(float* C, int seed) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int i = 0; i < 64; i++) C[i] = 0.0f;
  C[12] = -0.45f;
  C[13] = 0.63f;
  C[14] = 0.90f;
  C[20] = 1.18f;
  C[22] = 1.0f;
  C[23] = 1.0f;
  C[31] = (float)seed;
  C[44] = 1.0f;
  fps_pose(C, mk(2.0f, 1.72f, 18.0f), kPi, 0.0f);
}
// Arbor.cu:182
__global__ void update_camera_kernel(float* C, const float* I, float delta, int width, int height) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  C[10] = 0.0f;
  C[24] += 1.0f;
  float dt = clampf(delta, 0.0f, 0.1f);
  f3 old = ld3(C, 0);
  if (I[5] > 0.0f) view_preset(C, (int)I[5]);
  if (I[7] > 0.0f) {
    C[11] = C[11] > 0.0f ? 0.0f : 0.60f;
    C[10] = 1.0f;
  }
  if (I[9] > 0.0f) {
    C[15] = (float)(((int)C[15] + 1) % 4);
    C[10] = 1.0f;
  }
  if (I[10] > 0.0f) {
    C[22] = 1.0f - C[22];
    C[10] = 1.0f;
  }
  if (I[8] != 0.0f) {
    C[12] += I[8] * dt * 0.6f;
    C[10] = 1.0f;
  }
  if (I[12] != 0.0f) {
    C[20] = clampf(C[20] + I[12] * dt, 0.25f, 3.0f);
    C[10] = 1.0f;
  }
  if (C[11] > 0.0f) {
    C[8] += dt;
    C[10] = 1.0f;
  }
  C[16] -= I[0] * 0.00225f;
  C[17] = clampf(C[17] - I[1] * 0.0020f, -1.45f, 1.45f);
  float yaw = C[16];
  float cp = xcos(C[17]);
  f3 look = norm3(mk(xsin(yaw) * cp, xsin(C[17]), xcos(yaw) * cp));
  f3 walkF = norm3(mk(xsin(yaw), 0.0f, xcos(yaw)));
  f3 right = norm3(mk(walkF.z, 0.0f, -walkF.x));
  float speed = (I[16] > 0.5f ? 10.5f : 4.2f);
  f3 move = walkF * I[15] + right * I[13];
  if (dot3(move, move) > 0.0001f) move = norm3(move) * speed * dt;
  f3 eye = ld3(C, 0) + move;
  eye.y = 1.72f;
  st3(C, 0, eye);
  st3(C, 4, eye + look);
  C[27] = C[16];
  C[28] = C[17];
  C[3] = 1.0f;
  C[18] = 1.0f;
  if (length3(eye - old) > 0.000001f || I[0] != 0.0f || I[1] != 0.0f) C[10] = 1.0f;
  if (C[32] != (float)width || C[33] != (float)height) {
    C[10] = 1.0f;
    C[32] = (float)width;
    C[33] = (float)height;
  }
  C[9] = C[10] > 0.5f ? 0.0f : fminf(255.0f, C[9] + 1.0f);
}

// Sample index and history reset for progressive sampling, as the harness
// writes them before each sample (tests/native_harness.cpp:62).
__global__ void set_sample_kernel(float* C, int sample, int reset) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  C[9] = (float)sample;
  C[10] = reset ? 1.0f : 0.0f;
}

// The forest instance table of world seed ws, one Instance per tree: the
// table the trace and shade kernels use (built in shared memory by the shade
// passes' block prologues, read from the registry by the persistent passes).
__global__ void forest_instances_kernel(Instance* out, int ws, const WorldTrig* trig) {
  const float4* yaw_trig = world_trig_of(trig, ws);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < kForest) out[t] = make_instance(t, ws, yaw_trig);
}

// A registry slot's instance table, from the slot's own sines and cosines.
__global__ void slot_instances_kernel(WorldTrig* slot, int ws) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < kForest) slot->inst[t] = make_instance(t, ws, slot->v);
}

// Per-device registry of world-seed yaw tables (WorldTrig).  Slots are
// written once, data before header, and never reused, so a kernel running
// on another stream meanwhile reads either a complete slot or none.
struct TrigRegistry {
  WorldTrig* dev = nullptr;
  int used = 0;
  int seeds[kTrigSlots];
};
constexpr int kMaxDevices = 64;
std::mutex g_trig_mu;
TrigRegistry g_trig[kMaxDevices];

int current_device() {
  int d = 0;
  return cudaGetDevice(&d) == cudaSuccess && d >= 0 && d < kMaxDevices ? d : -1;
}

}  // namespace

const WorldTrig* world_trig() {
  const int d = current_device();
  if (d < 0) return nullptr;
  std::lock_guard<std::mutex> lock(g_trig_mu);
  return g_trig[d].dev;
}

void register_world_seed(int ws, cudaStream_t stream) {
  const int d = current_device();
  if (d < 0) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (cs != cudaStreamCaptureStatusNone) return;  // no allocation or copy inside a capture
  std::lock_guard<std::mutex> lock(g_trig_mu);
  TrigRegistry& r = g_trig[d];
  for (int i = 0; i < r.used; i++)
    if (r.seeds[i] == ws) return;
  if (r.used == kTrigSlots) return;  // full: later seeds keep make_instance's values
  if (r.dev == nullptr) {
    if (cudaMalloc(&r.dev, sizeof(WorldTrig) * kTrigSlots) != cudaSuccess) {
      cudaGetLastError();
      r.dev = nullptr;
      return;
    }
    if (cudaMemset(r.dev, 0, sizeof(WorldTrig) * kTrigSlots) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(r.dev);
      r.dev = nullptr;
      return;
    }
  }
  // The harness's values: yaw as forestYaw computes it (float arithmetic,
  // Arbor.cu:66), then the C library's cosf/sinf of -yaw and yaw
  // (Arbor.cu:67-69).
  static float4 v[kForest];
  for (int t = 0; t < kForest; t++) {
    const float yaw = forest_yaw(t, ws);
    const float a = -yaw;
    v[t] = make_float4(::cosf(a), ::sinf(a), ::cosf(yaw), ::sinf(yaw));
  }
  WorldTrig* dst = r.dev + r.used;
  const int header[2] = {ws, 1};
  if (cudaMemcpyAsync(dst->v, v, sizeof(v), cudaMemcpyHostToDevice, stream) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  // then the instance table from those values, on the device (the same
  // make_instance as every block prologue)
  slot_instances_kernel<<<(kForest + 127) / 128, 128, 0, stream>>>(dst, ws);
  count_launch();
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess ||
      cudaMemcpyAsync(dst, header, sizeof(header), cudaMemcpyHostToDevice, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  r.seeds[r.used++] = ws;
}

}  // namespace arbor

using namespace arbor;

extern "C" int arbor_forestInstances(int world_seed, float* instances, arbor_stream stream) {
  static_assert(sizeof(Instance) == ARBOR_INSTANCE_FLOATS * 4, "Instance record layout");
  const Binding b[] = {{instances, (size_t)kForest * sizeof(Instance), true, 16, "instances"}};
  if (int s = check_bindings("arbor_forestInstances", b)) return s;
  register_world_seed(world_seed, stream);
  forest_instances_kernel<<<(kForest + 127) / 128, 128, 0, stream>>>(reinterpret_cast<Instance*>(instances), world_seed, world_trig());
  count_launch();
  return check_launch("arbor_forestInstances");
}

extern "C" int arbor_setSample(float* C, int sample, int reset, arbor_stream stream) {
  const Binding b[] = {{C, kC, true, 4, "C"}};
  if (int s = check_bindings("arbor_setSample", b)) return s;
  if (sample < 0 || sample > 16777216) {
    set_error("arbor_setSample: sample %d outside 0..2^24 (C[9] is a float)", sample);
    return ARBOR_ERR_VALUE;
  }
  set_sample_kernel<<<1, 1, 0, stream>>>(C, sample, reset);
  count_launch();
  return check_launch("arbor_setSample");
}

extern "C" int arbor_initCamera(float* C, const float* P, int seed, arbor_stream stream) {
  const Binding b[] = {{C, kC, true, 4, "C"}, {P, kP, false, 4, "P"}};
  if (int s = check_bindings("arbor_initCamera", b)) return s;
  register_world_seed(seed, stream);
  init_camera_kernel<<<1, 1, 0, stream>>>(C, seed);
  count_launch();
  return check_launch("arbor_initCamera");
}
extern "C" int arbor_updateCamera(float* C, const float* I, const float* P, float delta, int width, int height, arbor_stream stream) {
  const Binding b[] = {{C, kC, true, 4, "C"}, {I, kI, false, 4, "I"}, {P, kP, false, 4, "P"}};
  if (int s = check_bindings("arbor_updateCamera", b)) return s;
  if (!std::isfinite(delta)) {
    set_error("arbor_updateCamera: scalar 'delta' must be finite");
    return ARBOR_ERR_VALUE;
  }
  update_camera_kernel<<<1, 1, 0, stream>>>(C, I, delta, width, height);
  count_launch();
  return check_launch("arbor_updateCamera");
}
