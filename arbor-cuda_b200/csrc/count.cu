// count.cu - work counting for the trace roofline model.
//
// Compiles the product's traversal and intersection code a second time with
// the work-event hooks enabled, into a kernel that records, per thread, how
// many times each event of arbor_scene.cuh's WorkEvent list happened.  The
// product trace kernel (render.cu) is compiled without the hooks; this pass
// runs outside any timed region and only to size the work one frame does.
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
#include "render_common.cuh"

namespace arbor {
namespace {

template <bool kForestScene>
__global__ void __launch_bounds__(kBlock) trace_work_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                            const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                            int width, int height) {
  __shared__ Camera cam;
  __shared__ Instance inst[kForestScene ? kForest : 1];
  block_setup(C, cam, inst, kForestScene);
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
    trace_work_kernel<false><<<grid, kBlock, 0, stream>>>(P, Nodes, Order, C, width, height);
  else
    trace_work_kernel<true><<<grid, kBlock, 0, stream>>>(P, Nodes, Order, C, width, height);
  count_launch();
  return check_launch(name);
}
