// render_common.cuh - per-block camera constants, the pixel tiling and the
// block prologue shared by the trace/shade kernels and the work-counting
// kernel.
#pragma once
#include "warpbatch.cuh"

namespace arbor {
namespace {

constexpr int kTile = 16;
constexpr int kBlock = 256;

// Per-frame camera constants (Arbor.cu:45-51), computed once per block.
struct Camera {
  f3 ro, f, r, up, sun;
  float jx, jy, c14;
  float time, wind;
  int ws, sample;
  float mode, shadows;
};
__device__ __forceinline__ void load_camera(const float* C, Camera& cam) {
  cam.ro = ld3(C, 0);
  int sample = (int)C[9];
  cam.sample = sample;
  cam.jx = halton(sample + 1, 2) - 0.5f;
  cam.jy = halton(sample + 1, 3) - 0.5f;
  cam.f = norm3(ld3(C, 4) - ld3(C, 0));
  cam.r = norm3(cross3(cam.f, mk(0.0f, 1.0f, 0.0f)));
  cam.up = cross3(cam.r, cam.f);
  cam.c14 = C[14];
  cam.time = C[8];
  cam.wind = C[11];
  cam.ws = (int)C[31];
  cam.mode = C[15];
  cam.shadows = C[22];
  // sunC (Arbor.cu:48)
  cam.sun = norm3(mk(xcos(C[12]) * xcos(C[13]), xsin(C[13]), xsin(C[12]) * xcos(C[13])));
}
__device__ __forceinline__ f3 camera_ray(const Camera& cam, int x, int y, int width, int height) {
  float u = ((float)x + 0.5f + cam.jx - (float)width * 0.5f) / (float)height;
  float v = ((float)height * 0.5f - (float)y - 0.5f - cam.jy) / (float)height;
  return norm3(cam.f + cam.r * (u * cam.c14) + cam.up * (v * cam.c14));
}
// Pixel of thread `t` in a 16x16 tile made of 8x4 warp sub-tiles.
__device__ __forceinline__ void tile_pixel(int t, int& x, int& y) {
  int warp = t >> 5, lane = t & 31;
  x = blockIdx.x * kTile + (warp & 1) * 8 + (lane & 7);
  y = blockIdx.y * kTile + (warp >> 1) * 4 + (lane >> 3);
}
// Block prologue: camera constants and (forest scenes) the instance table,
// its yaw sines and cosines from the world-seed registry `trig` where it has
// the scene's seed.
__device__ __forceinline__ void block_setup(const float* C, Camera& cam, Instance* inst, bool forest, const WorldTrig* trig) {
  if (threadIdx.x == 0) load_camera(C, cam);
  if (forest) {
    const int ws = (int)C[31];
    const float4* yaw_trig = world_trig_of(trig, ws);
    for (int t = threadIdx.x; t < kForest; t += blockDim.x) inst[t] = make_instance(t, ws, yaw_trig);
  }
  __syncthreads();
}

}  // namespace
}  // namespace arbor
