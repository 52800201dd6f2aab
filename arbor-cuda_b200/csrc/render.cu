// render.cu - per-frame image passes: tracePixels, shadePixels,
// filterLighting, resolvePixels (Arbor.cu:252-304) and their single-tree and
// fused variants, with their C-ABI entry points.
//
// Launch shapes: the trace and the shade's shadow pass are persistent (2
// CTAs per SM, lanes taking pixels of 8x4 blocks as their rays finish); the
// shade's compose pass runs 256-thread blocks over 16x16 pixel tiles.  The
// persistent passes read the 324-entry forest instance table from the
// world-seed registry (pass_instances); the compose blocks build it in shared
// memory once.  Every table entry equals what the reference's forest helpers
// recompute per ray (Arbor.cu:57-69).
#include <algorithm>

#include "abi_util.h"
#include "passes.cuh"

namespace arbor {
namespace {

// ---------------------------------------------------------------- kernels --
// The instance table of a persistent pass: the registry slot's (global
// memory) when the host registered the world seed, else one built in the
// dynamic shared memory of the CTA's last two warp batches, whose warps then
// leave (kTableWarps warps trace).  Every thread of the block calls it.
constexpr int kTableWarps = kBlock / 32 - 2;
static_assert(2 * sizeof(WarpBatch) >= sizeof(Instance) * kForest, "two warp batches hold an instance table");
__device__ __forceinline__ const Instance* pass_instances(const WorldTrig* trig, int ws, float4* smem, bool& leave) {
  const WorldTrig* slot = world_slot_of(trig, ws);
  leave = false;
  if (slot != nullptr) return slot->inst;
  Instance* table = reinterpret_cast<Instance*>(reinterpret_cast<WarpBatch*>(smem) + kTableWarps);
  for (int t = threadIdx.x; t < kForest; t += blockDim.x) table[t] = make_instance(t, ws);
  __syncthreads();
  leave = (int)(threadIdx.x >> 5) >= kTableWarps;
  return table;
}

// Persistent form of the trace: a grid of (SMs x 2) CTAs, each taking every
// gridDim.x-th 8x4-pixel block of the image, its lanes taking pixels as
// their rays finish (batch_run_pool).
template <bool kForestScene>
__global__ void __launch_bounds__(kBlock, 2) trace_pool_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                               const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                               const WorldTrig* __restrict__ trig,
                                                               float* __restrict__ Hit, int width, int height) {
  extern __shared__ float4 batch_smem[];
  WarpBatch& b = reinterpret_cast<WarpBatch*>(batch_smem)[threadIdx.x >> 5];
  __shared__ Camera cam;
  __shared__ int next;
  if (threadIdx.x == 0) next = 0;
  block_setup(C, cam, nullptr, false, nullptr);
  bool leave = false;
  const Instance* inst = kForestScene ? pass_instances(trig, cam.ws, batch_smem, leave) : nullptr;
  if (leave) return;
  const TraceCtx c{P, Nodes, Order, inst, cam.c14 / (float)height, cam.time, cam.wind, true, kForestScene};
  const int bx = (width + 7) / 8;
  const PixelPool pool{&next, width, height, bx, bx * ((height + 3) / 4)};
  trace_pool(c, cam, b, Hit, pool);
}

// shadePixels in two passes.  The shadow pass is persistent like the trace:
// lanes take pixels from a pool and trace their shadow segments, writing the
// visibility into Linear; with sun shadows off it returns at once.
template <bool kForestScene>
__global__ void __launch_bounds__(kBlock, 2) shadow_pool_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                                const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                                const WorldTrig* __restrict__ trig,
                                                                const float* __restrict__ Guide, float* __restrict__ Linear, int width, int height) {
  extern __shared__ float4 batch_smem[];
  WarpBatch& b = reinterpret_cast<WarpBatch*>(batch_smem)[threadIdx.x >> 5];
  __shared__ Camera cam;
  __shared__ int next;
  if (threadIdx.x == 0) next = 0;
  block_setup(C, cam, nullptr, false, nullptr);
  if (!(cam.shadows > 0.5f)) return;
  bool leave = false;
  const Instance* inst = kForestScene ? pass_instances(trig, cam.ws, batch_smem, leave) : nullptr;
  if (leave) return;
  const TraceCtx c{P, Nodes, Order, inst, 0.0001f, cam.time, cam.wind, false, kForestScene};
  const int bx = (width + 7) / 8;
  const PixelPool pool{&next, width, height, bx, bx * ((height + 3) / 4)};
  staged_shadow_pool(c, b, Guide, Linear, pool);
}

// Stages each pixel's shadow ray for the shadow pass (origin into Linear,
// direction into Guide; both are overwritten by the compose pass); with sun
// shadows off it returns at once.
__global__ void __launch_bounds__(kBlock) shadow_setup_kernel(const float* __restrict__ C, const float* __restrict__ Hit, float* __restrict__ Linear,
                                                              float* __restrict__ Guide, int width, int height) {
  __shared__ Camera cam;
  block_setup(C, cam, nullptr, false, nullptr);
  if (!(cam.shadows > 0.5f)) return;
  int x, y;
  tile_pixel_at(threadIdx.x, blockIdx.x * kTile, blockIdx.y * kTile, kTile, x, y);
  if (x < width && y < height) shadow_setup_px(cam, Hit, Linear, Guide, x, y, width, height);
}

// The compose pass: one pixel per thread, the surface terms and the colour
// with the shadow pass's visibility; 4 CTAs per SM (64 registers) hide its
// memory latency better than 3 (measured 0.557 -> 0.530 ms at 1080p).
template <bool kForestScene>
__global__ void __launch_bounds__(kBlock, 4) shade_compose_kernel(const float* __restrict__ P, const float* __restrict__ C,
                                                                  const WorldTrig* __restrict__ trig, const float* __restrict__ Hit,
                                                                  float* __restrict__ Linear, float* __restrict__ Guide, float* __restrict__ Normal,
                                                                  int width, int height) {
  __shared__ Camera cam;
  __shared__ Instance inst[kForestScene ? kForest : 1];
  block_setup(C, cam, inst, kForestScene, trig);
  int x, y;
  tile_pixel_at(threadIdx.x, blockIdx.x * kTile, blockIdx.y * kTile, kTile, x, y);
  if (x < width && y < height) shade_compose_px<kForestScene>(P, cam, inst, Hit, Linear, Guide, Normal, x, y, width, height);
}

// ------------------------------------------------ forest of several species --
// The reference's 324 instances all share one resident tree (README.md:8,
// docs/ARCHITECTURE.md:5).  These kernels trace and shade a forest whose
// instance t keeps the reference's transform, wind phase and tint but takes
// its geometry (its own records and BVH) from scene of[t]; P, Nodes and Order
// hold the scenes back to back.  The 2D DDA, bounding spheres and every
// per-instance step are the reference's; only the scene a tree's traversal
// and tests read changes.  With every of[t] = 0 the results equal
// arbor_tracePixels / arbor_shadePixels on scene 0.
struct SpeciesMap {
  uint8_t of[kForest];
};
__device__ __forceinline__ void species_setup(Instance* inst, const SpeciesMap& m) {
  for (int t = threadIdx.x; t < kForest; t += blockDim.x) inst[t].species = m.of[t];
  __syncthreads();
}

__global__ void __launch_bounds__(kBlock, 2) trace_species_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                                  const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                                  const WorldTrig* __restrict__ trig,
                                                                  float* __restrict__ Hit, int width, int height, const SpeciesMap map) {
  extern __shared__ float4 batch_smem[];
  WarpBatch& b = reinterpret_cast<WarpBatch*>(batch_smem)[threadIdx.x >> 5];
  __shared__ Camera cam;
  __shared__ uint8_t of[kForest];
  __shared__ int next;
  if (threadIdx.x == 0) next = 0;
  for (int t = threadIdx.x; t < kForest; t += blockDim.x) of[t] = map.of[t];
  block_setup(C, cam, nullptr, false, nullptr);
  bool leave = false;
  const Instance* inst = pass_instances(trig, cam.ws, batch_smem, leave);
  if (leave) return;
  const TraceCtx c{P, Nodes, Order, inst, cam.c14 / (float)height, cam.time, cam.wind, true, true, true, of};
  const int bx = (width + 7) / 8;
  const PixelPool pool{&next, width, height, bx, bx * ((height + 3) / 4)};
  trace_pool(c, cam, b, Hit, pool);
}

__global__ void __launch_bounds__(kBlock, 2) shadow_species_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                                   const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                                   const WorldTrig* __restrict__ trig,
                                                                   const float* __restrict__ Guide, float* __restrict__ Linear, int width, int height,
                                                                   const SpeciesMap map) {
  extern __shared__ float4 batch_smem[];
  WarpBatch& b = reinterpret_cast<WarpBatch*>(batch_smem)[threadIdx.x >> 5];
  __shared__ Camera cam;
  __shared__ uint8_t of[kForest];
  __shared__ int next;
  if (threadIdx.x == 0) next = 0;
  for (int t = threadIdx.x; t < kForest; t += blockDim.x) of[t] = map.of[t];
  block_setup(C, cam, nullptr, false, nullptr);
  if (!(cam.shadows > 0.5f)) return;
  bool leave = false;
  const Instance* inst = pass_instances(trig, cam.ws, batch_smem, leave);
  if (leave) return;
  const TraceCtx c{P, Nodes, Order, inst, 0.0001f, cam.time, cam.wind, false, true, true, of};
  const int bx = (width + 7) / 8;
  const PixelPool pool{&next, width, height, bx, bx * ((height + 3) / 4)};
  staged_shadow_pool(c, b, Guide, Linear, pool);
}

__global__ void __launch_bounds__(kBlock, 4) shade_compose_species_kernel(const float* __restrict__ P, const float* __restrict__ C,
                                                                          const WorldTrig* __restrict__ trig,
                                                                          const float* __restrict__ Hit, float* __restrict__ Linear,
                                                                          float* __restrict__ Guide, int width, int height, const SpeciesMap map) {
  __shared__ Camera cam;
  __shared__ Instance inst[kForest];
  block_setup(C, cam, inst, true, trig);
  species_setup(inst, map);
  int x, y;
  tile_pixel_at(threadIdx.x, blockIdx.x * kTile, blockIdx.y * kTile, kTile, x, y);
  if (x < width && y < height) shade_compose_px<true, true>(P, cam, inst, Hit, Linear, Guide, nullptr, x, y, width, height);
}

// tracePixels and shadePixels with the reference's traversal as written
// (Arbor.cu:220-289): one ray per thread over 16x16-pixel CTAs, candidates
// tested in visiting order, children nearest entry first, no warp batching.
// Slower forms kept to check that the batched passes' order does not change
// a result (the in-order entry points).
template <bool kForestScene>
__global__ void __launch_bounds__(kBlock) trace_inorder_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                               const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                               const WorldTrig* __restrict__ trig,
                                                               float* __restrict__ Hit, int width, int height) {
  __shared__ Camera cam;
  __shared__ Instance inst[kForestScene ? kForest : 1];
  block_setup(C, cam, inst, kForestScene, trig);
  int x, y;
  tile_pixel(threadIdx.x, x, y);
  if (x >= width || y >= height) return;
  const f3 ro = cam.ro;
  const f3 rd = camera_ray(cam, x, y, width, height);
  const float ground = rd.y < -0.00001f ? -ro.y / rd.y : kFar;
  const float cone = cam.c14 / (float)height;
  const float best = ground > 0.0f ? ground : kFar;
  int tree = -1;
  const f2 h = kForestScene ? trace_forest(P, Nodes, Order, inst, ro, rd, cone, cam.time, cam.wind, best, &tree, false)
                            : trace_tree(P, Nodes, Order, ro, rd, cone, cam.time, cam.wind, best, -1, false);
  reinterpret_cast<float4*>(Hit)[y * width + x] = make_float4(h.x, h.y, (float)tree, cam.c14 * h.x / (float)height);
}

template <bool kForestScene>
__global__ void __launch_bounds__(kBlock) shade_inorder_kernel(const float* __restrict__ P, const float* __restrict__ Nodes,
                                                               const uint32_t* __restrict__ Order, const float* __restrict__ C,
                                                               const WorldTrig* __restrict__ trig,
                                                               const float* __restrict__ Hit, float* __restrict__ Linear,
                                                               float* __restrict__ Guide, int width, int height) {
  __shared__ Camera cam;
  __shared__ Instance inst[kForestScene ? kForest : 1];
  block_setup(C, cam, inst, kForestScene, trig);
  int x, y;
  tile_pixel(threadIdx.x, x, y);
  if (x >= width || y >= height) return;
  const int pixel = y * width + x;
  Shading sh;
  shade_pre<kForestScene>(P, cam, inst, __ldg(reinterpret_cast<const float4*>(Hit) + pixel), x, y, width, height, sh);
  f3 vis = mk(1.0f, 1.0f, 1.0f);
  if (!sh.final && sh.shadow) {
    // lightVisibility (Arbor.cu:271-274)
    f3 trans = mk(1.0f, 1.0f, 1.0f);
    f3 o = sh.origin;
    for (int j = 0; j < 4; j++) {
      int tree = -1;
      const f2 h = kForestScene ? trace_forest(P, Nodes, Order, inst, o, sh.light, 0.0001f, cam.time, cam.wind, 36.0f, &tree, true)
                                : trace_tree(P, Nodes, Order, o, sh.light, 0.0001f, cam.time, cam.wind, 36.0f, -1, true);
      const int id = (int)h.y;
      if (id < 0) {
        vis = trans;
        break;
      }
      if (ldg4(P, id * 6).w != 1.0f) {
        vis = mk(0.0f, 0.0f, 0.0f);
        break;
      }
      trans = trans * mk(0.18f, 0.29f, 0.065f);
      o = o + sh.light * (h.x + 0.0018f);
      if (j == 3) vis = trans;
    }
  }
  const f3 col = shade_post(sh, vis);
  reinterpret_cast<float4*>(Linear)[pixel] = make_float4(col.x, col.y, col.z, 1.0f);
  reinterpret_cast<float4*>(Guide)[pixel] = make_float4(sh.guide.x, sh.guide.y, sh.guide.z, 1.0f);
}

// filterLighting (+ resolvePixels) of one 32x16 tile per CTA, its halo
// staged from global memory; 4 CTAs per SM.
template <bool kResolve>
__global__ void __launch_bounds__(kFX * kFT, 4) filter_kernel(const float* __restrict__ Linear, const float* __restrict__ Guide,
                                                              const float* __restrict__ Hit, float* __restrict__ Filtered,
                                                              float* __restrict__ History, uint32_t* __restrict__ Pixels,
                                                              const float* __restrict__ C, int width, int height) {
  __shared__ FilterTile s;
  filter_tile<kResolve>(s, Linear, Guide, Hit, Filtered, History, Pixels, kResolve ? C[9] : 0.0f, kResolve ? C[10] : 0.0f, C[15],
                        kResolve ? C[20] : 0.0f, width, height, blockIdx.x * kFX, blockIdx.y * kFY);
}

// resolvePixels alone (Arbor.cu:304): 32x8-pixel CTAs, one pixel per thread.
constexpr int kRX = 32, kRY = 8;
__global__ void __launch_bounds__(kRX * kRY) resolve_kernel(const float* __restrict__ Filtered, float* __restrict__ History,
                                                            uint32_t* __restrict__ Pixels, const float* __restrict__ C, int width,
                                                            int height) {
  const int x = blockIdx.x * kRX + threadIdx.x, y = blockIdx.y * kRY + threadIdx.y;
  if (x >= width || y >= height) return;
  float4 f = __ldg(reinterpret_cast<const float4*>(Filtered) + y * width + x);
  const float count = sample_count(C[9], C[10]);
  resolve_px(mk(f.x, f.y, f.z), History, Pixels, count, 1.0f / (count + 1.0f), C[20], vig_coord(x, width), vig_coord(y, height), y * width + x);
}

// Dynamic shared memory of a 256-thread CTA: one WarpBatch per warp.
constexpr size_t kBatchSmem = sizeof(WarpBatch) * (kBlock / 32);

// Opt a kernel in to kBatchSmem of dynamic shared memory, once per device.
inline bool batch_smem_ready(const void* kernel) {
  static const void* done[64][8] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  for (int i = 0; i < 8; i++) {
    if (done[dev][i] == kernel) return true;
    if (done[dev][i] == nullptr) {
      if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmem) != cudaSuccess) return false;
      done[dev][i] = kernel;
      return true;
    }
  }
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmem) == cudaSuccess;
}

dim3 pixel_grid(int w, int h) { return dim3((w + kTile - 1) / kTile, (h + kTile - 1) / kTile); }

// Persistent grid: 2 CTAs per SM (the register and shared-memory limit of
// the batched tracer), or one CTA per 8x4 block when the image has fewer.
dim3 pool_grid(int w, int h) {
  static int sms[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (sms[dev] == 0 && cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms[dev] = 148;
  const long blocks = (long)((w + 7) / 8) * ((h + 3) / 4);
  return dim3((unsigned)std::min<long>(blocks, 2L * sms[dev]));
}
dim3 filter_grid(int w, int h) { return dim3((w + kFX - 1) / kFX, (h + kFY - 1) / kFY); }

// filterLighting (+ resolvePixels) over width x height: one 32x16 tile per CTA.
int launch_filter(const char* name, bool resolve, const float* Linear, const float* Guide, const float* Hit, float* Filtered, float* History,
                  uint32_t* Pixels, const float* C, int width, int height, cudaStream_t stream) {
  if (resolve)
    filter_kernel<true><<<filter_grid(width, height), dim3(kFX, kFT), 0, stream>>>(Linear, Guide, Hit, Filtered, History, Pixels, C, width, height);
  else
    filter_kernel<false><<<filter_grid(width, height), dim3(kFX, kFT), 0, stream>>>(Linear, Guide, Hit, Filtered, nullptr, nullptr, C, width,
                                                                                    height);
  count_launch();
  return check_launch(name);
}
dim3 resolve_grid(int w, int h) { return dim3((w + kRX - 1) / kRX, (h + kRY - 1) / kRY); }

int trace_entry(const char* name, bool forest, const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int width,
                int height, cudaStream_t stream) {
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  const Binding b[] = {{P, kP, false, 16, "P"},
                       {Nodes, kNodes, false, 16, "Nodes"},
                       {Order, kKeys, false, 4, "Order"},
                       {C, kC, false, 4, "C"},
                       {Hit, empty ? 0 : image_bytes(width, height), true, 16, "Hit"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  if (!batch_smem_ready(forest ? (const void*)trace_pool_kernel<true> : (const void*)trace_pool_kernel<false>)) {
    set_error("%s: cannot reserve %zu bytes of shared memory per CTA", name, kBatchSmem);
    return ARBOR_ERR_CUDA;
  }
  if (forest)
    trace_pool_kernel<true><<<pool_grid(width, height), kBlock, kBatchSmem, stream>>>(P, Nodes, Order, C, world_trig(), Hit, width, height);
  else
    trace_pool_kernel<false><<<pool_grid(width, height), kBlock, kBatchSmem, stream>>>(P, Nodes, Order, C, world_trig(), Hit, width, height);
  count_launch();
  return check_launch(name);
}

int shade_entry(const char* name, bool forest, const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit,
                float* Linear, float* Guide, int width, int height, cudaStream_t stream, float* Normal = nullptr) {
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  size_t img = empty ? 0 : image_bytes(width, height);
  const Binding b[] = {{P, kP, false, 16, "P"},         {Nodes, kNodes, false, 16, "Nodes"}, {Order, kKeys, false, 4, "Order"},
                       {C, kC, false, 4, "C"},          {Hit, img, false, 16, "Hit"},        {Linear, img, true, 16, "Linear"},
                       {Guide, img, true, 16, "Guide"}};
  if (int s = check_bindings(name, b)) return s;
  if (Normal != nullptr) {
    const Binding g[] = {{P, kP, false, 16, "P"}, {Hit, img, false, 16, "Hit"}, {Linear, img, true, 16, "Linear"},
                         {Guide, img, true, 16, "Guide"}, {Normal, img, true, 16, "Normal"}};
    if (int s = check_bindings(name, g)) return s;
  }
  if (empty) return ARBOR_OK;
  if (!batch_smem_ready(forest ? (const void*)shadow_pool_kernel<true> : (const void*)shadow_pool_kernel<false>)) {
    set_error("%s: cannot reserve %zu bytes of shared memory per CTA", name, kBatchSmem);
    return ARBOR_ERR_CUDA;
  }
  // Shadow segments in a persistent pass whose loop holds only the tracer
  // (its code stays small), then the shading of every pixel.
  shadow_setup_kernel<<<pixel_grid(width, height), kBlock, 0, stream>>>(C, Hit, Linear, Guide, width, height);
  if (forest) {
    shadow_pool_kernel<true><<<pool_grid(width, height), kBlock, kBatchSmem, stream>>>(P, Nodes, Order, C, world_trig(), Guide, Linear, width, height);
    shade_compose_kernel<true><<<pixel_grid(width, height), kBlock, 0, stream>>>(P, C, world_trig(), Hit, Linear, Guide, Normal, width, height);
  } else {
    shadow_pool_kernel<false><<<pool_grid(width, height), kBlock, kBatchSmem, stream>>>(P, Nodes, Order, C, world_trig(), Guide, Linear, width, height);
    shade_compose_kernel<false><<<pixel_grid(width, height), kBlock, 0, stream>>>(P, C, world_trig(), Hit, Linear, Guide, Normal, width, height);
  }
  count_launch(3);
  return check_launch(name);
}

// Checks of a forest-of-species call: 1..256 scenes, every instance on one
// of them.  Fills `map`.
int species_args(const char* name, int n_species, const int* species_of, SpeciesMap& map) {
  if (n_species < 1 || n_species > ARBOR_MAX_SPECIES) {
    set_error("%s: n_species %d outside 1..%d", name, n_species, ARBOR_MAX_SPECIES);
    return ARBOR_ERR_VALUE;
  }
  if (species_of == nullptr) {
    set_error("%s: species_of is NULL", name);
    return ARBOR_ERR_NULL;
  }
  for (int t = 0; t < kForest; t++) {
    if (species_of[t] < 0 || species_of[t] >= n_species) {
      set_error("%s: species_of[%d] = %d outside 0..%d", name, t, species_of[t], n_species - 1);
      return ARBOR_ERR_VALUE;
    }
    map.of[t] = (uint8_t)species_of[t];
  }
  return ARBOR_OK;
}

}  // namespace
}  // namespace arbor

using namespace arbor;

extern "C" int arbor_traceSpeciesPixels(const float* P, const float* Nodes, const uint32_t* Order, int n_species, const int* species_of,
                                        const float* C, float* Hit, int width, int height, arbor_stream stream) {
  const char* name = "arbor_traceSpeciesPixels";
  SpeciesMap map;
  if (int s = species_args(name, n_species, species_of, map)) return s;
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  const size_t n = (size_t)n_species;
  const Binding b[] = {{P, n * kP, false, 16, "P"},
                       {Nodes, n * kNodes, false, 16, "Nodes"},
                       {Order, n * kKeys, false, 4, "Order"},
                       {C, kC, false, 4, "C"},
                       {Hit, empty ? 0 : image_bytes(width, height), true, 16, "Hit"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  if (!batch_smem_ready((const void*)trace_species_kernel)) {
    set_error("%s: cannot reserve %zu bytes of shared memory per CTA", name, kBatchSmem);
    return ARBOR_ERR_CUDA;
  }
  trace_species_kernel<<<pool_grid(width, height), kBlock, kBatchSmem, stream>>>(P, Nodes, Order, C, world_trig(), Hit, width, height, map);
  count_launch();
  return check_launch(name);
}
extern "C" int arbor_shadeSpeciesPixels(const float* P, const float* Nodes, const uint32_t* Order, int n_species, const int* species_of,
                                        const float* C, const float* Hit, float* Linear, float* Guide, int width, int height, arbor_stream stream) {
  const char* name = "arbor_shadeSpeciesPixels";
  SpeciesMap map;
  if (int s = species_args(name, n_species, species_of, map)) return s;
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  const size_t n = (size_t)n_species;
  const size_t img = empty ? 0 : image_bytes(width, height);
  const Binding b[] = {{P, n * kP, false, 16, "P"},  {Nodes, n * kNodes, false, 16, "Nodes"}, {Order, n * kKeys, false, 4, "Order"},
                       {C, kC, false, 4, "C"},      {Hit, img, false, 16, "Hit"},             {Linear, img, true, 16, "Linear"},
                       {Guide, img, true, 16, "Guide"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  if (!batch_smem_ready((const void*)shadow_species_kernel)) {
    set_error("%s: cannot reserve %zu bytes of shared memory per CTA", name, kBatchSmem);
    return ARBOR_ERR_CUDA;
  }
  shadow_setup_kernel<<<pixel_grid(width, height), kBlock, 0, stream>>>(C, Hit, Linear, Guide, width, height);
  shadow_species_kernel<<<pool_grid(width, height), kBlock, kBatchSmem, stream>>>(P, Nodes, Order, C, world_trig(), Guide, Linear, width, height, map);
  shade_compose_species_kernel<<<pixel_grid(width, height), kBlock, 0, stream>>>(P, C, world_trig(), Hit, Linear, Guide, width, height, map);
  count_launch(3);
  return check_launch(name);
}

extern "C" int arbor_tracePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int width, int height,
                                 arbor_stream stream) {
  return trace_entry("arbor_tracePixels", true, P, Nodes, Order, C, Hit, width, height, stream);
}
extern "C" int arbor_traceTreePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int width, int height,
                                     arbor_stream stream) {
  return trace_entry("arbor_traceTreePixels", false, P, Nodes, Order, C, Hit, width, height, stream);
}
extern "C" int arbor_shadePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, float* Linear,
                                 float* Guide, int width, int height, arbor_stream stream) {
  return shade_entry("arbor_shadePixels", true, P, Nodes, Order, C, Hit, Linear, Guide, width, height, stream);
}
extern "C" int arbor_shadeGBuffer(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, float* Linear,
                                  float* Guide, float* Normal, int width, int height, arbor_stream stream) {
  if (Normal == nullptr && width > 0 && height > 0) {
    set_error("arbor_shadeGBuffer: buffer Normal is NULL");
    return ARBOR_ERR_NULL;
  }
  return shade_entry("arbor_shadeGBuffer", true, P, Nodes, Order, C, Hit, Linear, Guide, width, height, stream, Normal);
}
extern "C" int arbor_shadeTreePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, float* Linear,
                                     float* Guide, int width, int height, arbor_stream stream) {
  return shade_entry("arbor_shadeTreePixels", false, P, Nodes, Order, C, Hit, Linear, Guide, width, height, stream);
}
extern "C" int arbor_tracePixelsInOrder(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int width,
                                        int height, int single_tree, arbor_stream stream) {
  const char* name = "arbor_tracePixelsInOrder";
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  const Binding b[] = {{P, kP, false, 16, "P"},
                       {Nodes, kNodes, false, 16, "Nodes"},
                       {Order, kKeys, false, 4, "Order"},
                       {C, kC, false, 4, "C"},
                       {Hit, empty ? 0 : image_bytes(width, height), true, 16, "Hit"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  if (single_tree)
    trace_inorder_kernel<false><<<pixel_grid(width, height), kBlock, 0, stream>>>(P, Nodes, Order, C, world_trig(), Hit, width, height);
  else
    trace_inorder_kernel<true><<<pixel_grid(width, height), kBlock, 0, stream>>>(P, Nodes, Order, C, world_trig(), Hit, width, height);
  count_launch();
  return check_launch(name);
}
extern "C" int arbor_shadePixelsInOrder(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit,
                                        float* Linear, float* Guide, int width, int height, int single_tree, arbor_stream stream) {
  const char* name = "arbor_shadePixelsInOrder";
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  size_t img = empty ? 0 : image_bytes(width, height);
  const Binding b[] = {{P, kP, false, 16, "P"},         {Nodes, kNodes, false, 16, "Nodes"}, {Order, kKeys, false, 4, "Order"},
                       {C, kC, false, 4, "C"},          {Hit, img, false, 16, "Hit"},        {Linear, img, true, 16, "Linear"},
                       {Guide, img, true, 16, "Guide"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  if (single_tree)
    shade_inorder_kernel<false><<<pixel_grid(width, height), kBlock, 0, stream>>>(P, Nodes, Order, C, world_trig(), Hit, Linear, Guide, width, height);
  else
    shade_inorder_kernel<true><<<pixel_grid(width, height), kBlock, 0, stream>>>(P, Nodes, Order, C, world_trig(), Hit, Linear, Guide, width, height);
  count_launch();
  return check_launch(name);
}
extern "C" int arbor_filterLighting(const float* Linear, const float* Guide, const float* Hit, float* Filtered, const float* C, int width,
                                    int height, arbor_stream stream) {
  const char* name = "arbor_filterLighting";
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  size_t img = empty ? 0 : image_bytes(width, height);
  const Binding b[] = {{Linear, img, false, 16, "Linear"},
                       {Guide, img, false, 16, "Guide"},
                       {Hit, img, false, 16, "Hit"},
                       {Filtered, img, true, 16, "Filtered"},
                       {C, kC, false, 4, "C"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  return launch_filter(name, false, Linear, Guide, Hit, Filtered, nullptr, nullptr, C, width, height, stream);
}
extern "C" int arbor_resolvePixels(const float* Filtered, float* History, uint32_t* Pixels, const float* C, int width, int height,
                                   arbor_stream stream) {
  const char* name = "arbor_resolvePixels";
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  size_t img = empty ? 0 : image_bytes(width, height);
  const Binding b[] = {{Filtered, img, false, 16, "Filtered"},
                       {History, img, true, 16, "History"},
                       {Pixels, empty ? 0 : pixel_bytes(width, height), true, 4, "Pixels"},
                       {C, kC, false, 4, "C"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  resolve_kernel<<<resolve_grid(width, height), dim3(kRX, kRY), 0, stream>>>(Filtered, History, Pixels, C, width, height);
  count_launch();
  return check_launch(name);
}
extern "C" int arbor_filterResolve(const float* Linear, const float* Guide, const float* Hit, float* Filtered, float* History, uint32_t* Pixels,
                                   const float* C, int width, int height, arbor_stream stream) {
  const char* name = "arbor_filterResolve";
  bool empty;
  if (int s = check_image(name, width, height, &empty)) return s;
  size_t img = empty ? 0 : image_bytes(width, height);
  const Binding b[] = {{Linear, img, false, 16, "Linear"},     {Guide, img, false, 16, "Guide"},
                       {Hit, img, false, 16, "Hit"},           {Filtered, img, true, 16, "Filtered"},
                       {History, img, true, 16, "History"},    {Pixels, empty ? 0 : pixel_bytes(width, height), true, 4, "Pixels"},
                       {C, kC, false, 4, "C"}};
  if (int s = check_bindings(name, b)) return s;
  if (empty) return ARBOR_OK;
  return launch_filter(name, true, Linear, Guide, Hit, Filtered, History, Pixels, C, width, height, stream);
}

