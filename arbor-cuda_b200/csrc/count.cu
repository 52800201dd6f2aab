// count.cu - work counting for the trace and shade roofline models.
//
// Compiles the product's traversal and intersection code a second time with
// the work-event hooks enabled, into kernels that record, per thread, how
// many times each event of arbor_scene.cuh's WorkEvent list happened: the
// primary rays of tracePixels, and the shading (normals) and shadow-ray
// segments of shadePixels.  The product kernels (render.cu) are compiled
// without the hooks; these passes run outside any timed region and only to
// size the work one frame does.
#include <cstdint>

namespace arbor {
__device__ uint32_t* g_work_slots;
__device__ __forceinline__ void count_event(int event) {
  uint32_t gtid = (blockIdx.y * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x;
  g_work_slots[gtid * 16u + (uint32_t)event] += 1u;
}
}  // namespace arbor
#define ARBOR_COUNT(event) ::arbor::count_event(event)

#include "abi_util.h"
#include "passes.cuh"

namespace arbor {
namespace {

template <bool kForestScene>
__global__ void __launch_bounds__(kBlock) trace_work_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                            const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                            const WorldTrig* __restrict__ trig,
                                                            int width, int height) {
  __shared__ Camera cam;
  __shared__ Instance inst[kForestScene ? kForest : 1];
  block_setup(C, cam, inst, kForestScene, trig);
  int x, y;
  tile_pixel(threadIdx.x, x, y);
  if (x >= width || y >= height) return;
  count_event(kEvRay);
  f3 ro = cam.ro;
  f3 rd = camera_ray(cam, x, y, width, height);
  float ground = rd.y < -0.00001f ? -ro.y / rd.y : kFar;
  float cone = cam.c14 / (float)height;
  float best = ground > 0.0f ? ground : kFar;
  int tree = -1;
  if (kForestScene) {
    trace_forest(P, Nodes, Order, inst, ro, rd, cone, cam.time, cam.wind, best, &tree, false);
  } else {
    count_event(kEvTree);
    trace_tree(P, Nodes, Order, ro, rd, cone, cam.time, cam.wind, best, -1, false);
  }
}

// shadePixels' work for the given Hit records: the shading of each pixel
// (surface normals evaluate the wood field) and its shadow segments
// (lightVisibility, Arbor.cu:271-274: up to four traces of 36 m toward the
// sun, continuing through leaves).
template <bool kForestScene>
__global__ void __launch_bounds__(kBlock) shade_work_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                            const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                            const WorldTrig* __restrict__ trig,
                                                            const float* __restrict__ Hit, int width, int height) {
  __shared__ Camera cam;
  __shared__ Instance inst[kForestScene ? kForest : 1];
  block_setup(C, cam, inst, kForestScene, trig);
  int x, y;
  tile_pixel(threadIdx.x, x, y);
  if (x >= width || y >= height) return;
  Shading sh;
  shade_pre<kForestScene>(P, cam, inst, __ldg(reinterpret_cast<const float4*>(Hit) + y * width + x), x, y, width, height, sh);
  if (sh.final || !sh.shadow) return;
  f3 o = sh.origin;
  for (int j = 0; j < 4; j++) {
    count_event(kEvSegment);
    int tree = -1;
    f2 h = kForestScene ? trace_forest(P, Nodes, Order, inst, o, sh.light, 0.0001f, cam.time, cam.wind, 36.0f, &tree, true)
                        : trace_tree(P, Nodes, Order, o, sh.light, 0.0001f, cam.time, cam.wind, 36.0f, -1, true);
    int id = (int)h.y;
    if (id < 0 || ldg4(P, id * 6).w != 1.0f) break;
    o = o + sh.light * (h.x + 0.0018f);
  }
}

}  // namespace
}  // namespace arbor

using namespace arbor;

extern "C" size_t arbor_trace_work_slots(int width, int height) {
  if (width <= 0 || height <= 0) return 0;
  size_t blocks = (size_t)((width + kTile - 1) / kTile) * (size_t)((height + kTile - 1) / kTile);
  return blocks * kBlock * 16u;
}

extern "C" int arbor_traceWork(const float* P, const float* Nodes, const uint32_t* Order, const float* C, int width, int height, int single_tree,
                               uint32_t* slots, arbor_stream stream) {
  const char* name = "arbor_traceWork";
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  size_t nslots = empty ? 0 : arbor_trace_work_slots(width, height);
  const Binding b[] = {{P, kP, false, 16, "P"},
                       {Nodes, kNodes, false, 16, "Nodes"},
                       {Order, kKeys, false, 4, "Order"},
                       {C, kC, false, 4, "C"},
                       {slots, nslots * 4, true, 4, "slots"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  if (cudaMemsetAsync(slots, 0, nslots * 4, stream) != cudaSuccess) return check_launch(name);
  if (cudaMemcpyToSymbolAsync(g_work_slots, &slots, sizeof(slots), 0, cudaMemcpyHostToDevice, stream) != cudaSuccess) return check_launch(name);
  dim3 grid((width + kTile - 1) / kTile, (height + kTile - 1) / kTile);
  if (single_tree)
    trace_work_kernel<false><<<grid, kBlock, 0, stream>>>(P, Nodes, Order, C, world_trig(), width, height);
  else
    trace_work_kernel<true><<<grid, kBlock, 0, stream>>>(P, Nodes, Order, C, world_trig(), width, height);
  count_launch();
  return check_launch(name);
}

extern "C" int arbor_shadeWork(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, int width, int height,
                               int single_tree, uint32_t* slots, arbor_stream stream) {
  const char* name = "arbor_shadeWork";
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  size_t nslots = empty ? 0 : arbor_trace_work_slots(width, height);
  const Binding b[] = {{P, kP, false, 16, "P"},
                       {Nodes, kNodes, false, 16, "Nodes"},
                       {Order, kKeys, false, 4, "Order"},
                       {C, kC, false, 4, "C"},
                       {Hit, image_bytes(width, height), false, 16, "Hit"},
                       {slots, nslots * 4, true, 4, "slots"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  if (cudaMemsetAsync(slots, 0, nslots * 4, stream) != cudaSuccess) return check_launch(name);
  if (cudaMemcpyToSymbolAsync(g_work_slots, &slots, sizeof(slots), 0, cudaMemcpyHostToDevice, stream) != cudaSuccess) return check_launch(name);
  dim3 grid((width + kTile - 1) / kTile, (height + kTile - 1) / kTile);
  if (single_tree)
    shade_work_kernel<false><<<grid, kBlock, 0, stream>>>(P, Nodes, Order, C, world_trig(), Hit, width, height);
  else
    shade_work_kernel<true><<<grid, kBlock, 0, stream>>>(P, Nodes, Order, C, world_trig(), Hit, width, height);
  count_launch();
  return check_launch(name);
}
