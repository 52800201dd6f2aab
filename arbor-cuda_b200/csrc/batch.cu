// batch.cu - batched multi-view rendering.
//
// Many views (each with its own resolution, camera record C and resident
// scene) render in one CUDA graph launch of five kernels:
//
//   batch_setup_kernel        per view: camera constants, the forest
//                             instance table and the filter/resolve scalars
//                             of its C record; resets the queues
//   batch_pool_kernel<trace>  persistent warps walk the views; in each, their
//                             lanes take pixels from the view's own queue as
//                             their rays finish and run tracePixels
//                             (Arbor.cu:252)
//   batch_pool_kernel<shadow> the same for the shadow segments of
//                             shadePixels (Arbor.cu:271-274)
//   batch_compose_kernel      persistent CTAs pull tiles of every view from
//                             one global queue: shadePixels' colours
//                             (Arbor.cu:277-289) with that visibility
//   batch_filter_kernel       persistent CTAs pull 32x8 tiles and run the
//                             fused filterLighting + resolvePixels
//                             (Arbor.cu:292-304)
//
// Every per-pixel value is computed by the same device code as the
// single-image entries (passes.cuh), so a view renders as
// arbor_tracePixels + arbor_shadePixels + arbor_filterResolve render it with
// the same C, apart from the order in which exactly equal hit distances are
// met (the warp batch groups rays by tile; see warpbatch.cuh).
//
// The autotuner times the trace, shadow and compose kernels on a sample of
// the views for each compose tile shape (16x16 or 32x8), CTAs per SM (1 or
// 2), view order (as given, or the largest views first) and warp-batch queue
// depth (12 or 16 candidates per lane), and keeps the fastest.
#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "abi_util.h"
#include "passes.cuh"

namespace arbor {
namespace {

// Work queues (global counters) of one render: the compose tiles, the filter
// tiles, then one pixel queue per view for the trace pass and one per view
// for the shadow pass.
constexpr int kQueueCompose = 0, kQueueFilter = 1, kViewQueues = 2;

struct BatchView {
  const float* P;
  const float* Nodes;
  const uint32_t* Order;
  float* Hit;
  float* Linear;
  float* Guide;
  float* Filtered;
  float* History;
  uint32_t* Pixels;
  int width, height;
};

__global__ void __launch_bounds__(kBlock) batch_setup_kernel(const float* __restrict__ Cs, const WorldTrig* __restrict__ trig, Camera* __restrict__ cams,
                                                             float4* __restrict__ scal, Instance* __restrict__ insts, int* __restrict__ counters) {
  const int v = blockIdx.x;
  if (threadIdx.x == 0) {
    counters[kViewQueues + v] = 0;
    counters[kViewQueues + gridDim.x + v] = 0;
  }
  const float* C = Cs + v * 64;
  if (threadIdx.x == 0) {
    Camera cam;
    load_camera(C, cam);
    cams[v] = cam;
    scal[v] = make_float4(C[9], C[10], C[15], C[20]);
  }
  const int ws = (int)C[31];
  const float4* yaw_trig = world_trig_of(trig, ws);
  for (int t = threadIdx.x; t < kForest; t += blockDim.x) insts[v * kForest + t] = make_instance(t, ws, yaw_trig);
  if (v == 0 && threadIdx.x < kViewQueues) counters[threadIdx.x] = 0;
}

// tracePixels (kShadow false) or the shadow segments of shadePixels (true,
// visibility into Linear) of every listed view.  Each warp walks the views in
// order and joins each one's pixel queue; its lanes take the view's next
// pixels as their rays finish, so warps of any CTA share a view's work and
// move on independently.  The view's camera and instance table are read from
// global memory (the values setup wrote).
template <int Q, bool kShadow>
__global__ void __launch_bounds__(kBlock, 2) batch_pool_kernel(const BatchView* __restrict__ views, const Camera* __restrict__ cams,
                                                               const Instance* __restrict__ insts, const int* __restrict__ list, int n_list,
                                                               int* __restrict__ queues) {
  using WB = WarpBatchQ<Q>;
  extern __shared__ float4 batch_smem[];
  WB& b = reinterpret_cast<WB*>(batch_smem)[threadIdx.x >> 5];
  for (int i = 0; i < n_list; i++) {
    const int v = __ldg(list + i);
    const Camera& cam = cams[v];
    if (kShadow && !(cam.shadows > 0.5f)) continue;
    const BatchView view = views[v];
    const int bx = (view.width + 7) / 8;
    const ViewPool pool{queues + v, view.width, view.height, bx, bx * ((view.height + 3) / 4)};
    Ray r;
    if (kShadow) {
      const TraceCtx c{view.P, view.Nodes, view.Order, insts + (size_t)v * kForest, 0.0001f, cam.time, cam.wind, false, true};
      ShadowPolicy policy{&c, &cam, view.Hit, view.Linear, view.width, view.height, 0, 0};
      batch_run_pool(c, r, b, policy, pool);
    } else {
      const TraceCtx c{view.P, view.Nodes, view.Order, insts + (size_t)v * kForest, cam.c14 / (float)view.height, cam.time, cam.wind, true, true};
      PrimaryPolicy policy{&cam, view.Hit, view.width, view.height, 0};
      batch_run_pool(c, r, b, policy, pool);
    }
  }
}

// shadePixels' colours of each tile, one pixel per thread, with the shadow
// pass's visibility (4 CTAs per SM, as the single-image compose pass).
__global__ void __launch_bounds__(kBlock, 4) batch_compose_kernel(const BatchView* __restrict__ views, const Camera* __restrict__ cams,
                                                               const Instance* __restrict__ insts, const int4* __restrict__ tiles,
                                                               int n_tiles, int tw, int* __restrict__ counter) {
  __shared__ Camera cam;
  __shared__ Instance inst[kForest];
  __shared__ int s_tile;
  int cur = -1;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= n_tiles) break;
    const int4 td = __ldg(tiles + t);
    if (td.x != cur) {  // uniform across the CTA
      cur = td.x;
      if (threadIdx.x == 0) cam = cams[cur];
      for (int k = threadIdx.x; k < kForest; k += blockDim.x) inst[k] = insts[cur * kForest + k];
      __syncthreads();
    }
    const BatchView v = views[cur];
    int x, y;
    tile_pixel_at(threadIdx.x, td.y, td.z, tw, x, y);
    if (x < v.width && y < v.height) shade_compose_px<true>(v.P, cam, inst, v.Hit, v.Linear, v.Guide, nullptr, x, y, v.width, v.height);
    __syncthreads();  // every thread has read s_tile, cam and inst
  }
}

__global__ void __launch_bounds__(kFX * kFT) batch_filter_kernel(const BatchView* __restrict__ views, const float4* __restrict__ scal,
                                                                 const int4* __restrict__ tiles, int n_tiles, int* __restrict__ counter) {
  __shared__ FilterTile s;
  __shared__ int s_tile;
  const int tid = threadIdx.y * kFX + threadIdx.x;
  for (;;) {
    if (tid == 0) s_tile = atomicAdd(counter, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= n_tiles) break;
    const int4 td = __ldg(tiles + t);
    const BatchView v = views[td.x];
    const float4 sc = scal[td.x];
    filter_tile<true>(s, v.Linear, v.Guide, v.Hit, v.Filtered, v.History, v.Pixels, sc.x, sc.y, sc.z, sc.w, v.width, v.height, td.y, td.z);
    __syncthreads();  // the tile's shared memory and s_tile are free again
  }
}

template <int Q>
constexpr size_t batch_smem_bytes() {
  return sizeof(WarpBatchQ<Q>) * (kBlock / 32);
}

int cuda_fail(const char* what, cudaError_t e) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  return ARBOR_ERR_CUDA;
}
#define BATCH_CUDA(call)                                \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(#call, e_); \
  } while (0)

constexpr size_t align256(size_t n) { return (n + 255) / 256 * 256; }
constexpr size_t kOffP = align256(kB), kOffKeys = kOffP + align256(kP), kOffOrder = kOffKeys + align256(kKeys),
                 kOffNodes = kOffOrder + align256(kKeys), kSceneStride = kOffNodes + align256(kNodes);
constexpr int kMaxViews = 65536;
constexpr int kMaxScenes = 1024;

bool valid_config(const arbor_batch_config& c) {
  return (c.tile_width == 16 || c.tile_width == 32) && (c.ctas_per_sm == 1 || c.ctas_per_sm == 2) && (c.order == 0 || c.order == 1) &&
         (c.queue == 12 || c.queue == 16);
}

}  // namespace
}  // namespace arbor

using namespace arbor;

struct arbor_batch {
  cudaStream_t user = nullptr;  // the caller's stream; work is ordered after it
  cudaStream_t own = nullptr;   // capture and launch stream
  cudaEvent_t joined = nullptr, done = nullptr;
  int n_scenes = 0, n_views = 0, sms = 0;
  std::vector<int> seeds, vw, vh, vscene;
  std::vector<uint64_t> offset;  // first pixel of each view in the image arenas
  uint64_t total_px = 0;
  char* scenes = nullptr;      // n_scenes x {B, P, Keys, Order, Nodes}
  float* images = nullptr;     // Hit | Linear | Guide | Filtered | History, total_px float4 each
  uint32_t* pixels = nullptr;  // total_px
  float* C = nullptr;          // n_views x 64
  float* staging = nullptr;    // pinned host copy of C
  BatchView* views = nullptr;
  Camera* cams = nullptr;
  float4* scal = nullptr;
  Instance* insts = nullptr;
  int* counters = nullptr;     // work queues: kViewQueues tile queues, then 2 pixel queues per view
  int* vlist = nullptr;        // views the shadow pass walks, in order
  int4* tiles = nullptr;       // trace/shade tiles, then filter tiles
  int n_ts = 0, n_filter = 0;
  size_t tile_capacity = 0;
  void* scratch = nullptr;     // radix-sort scratch of the scene builds
  arbor_batch_config cfg{16, 2, 0, 16};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t renders = 0;
  uint64_t allocated = 0;
};

namespace {

float* image(arbor_batch* b, int which, int v) { return b->images + ((uint64_t)which * b->total_px + b->offset[v]) * 4; }
char* scene_base(arbor_batch* b, int s) { return b->scenes + (size_t)s * kSceneStride; }

// Trace/shade tiles of tw x (256/tw) pixels of the listed views, in order.
void trace_tiles(const arbor_batch* b, const std::vector<int>& order, int tw, std::vector<int4>& out) {
  const int th = kBlock / tw;
  for (int v : order)
    for (int y0 = 0; y0 < b->vh[v]; y0 += th)
      for (int x0 = 0; x0 < b->vw[v]; x0 += tw) out.push_back(make_int4(v, x0, y0, 0));
}
void filter_tiles(const arbor_batch* b, std::vector<int4>& out) {
  for (int v = 0; v < b->n_views; v++)
    for (int y0 = 0; y0 < b->vh[v]; y0 += kFY)
      for (int x0 = 0; x0 < b->vw[v]; x0 += kFX) out.push_back(make_int4(v, x0, y0, 0));
}
std::vector<int> view_order(const arbor_batch* b, const std::vector<int>& subset, int order) {
  std::vector<int> o = subset;
  if (order == 1)
    std::stable_sort(o.begin(), o.end(), [&](int a, int c) { return (uint64_t)b->vw[a] * b->vh[a] > (uint64_t)b->vw[c] * b->vh[c]; });
  return o;
}

int launch_setup(arbor_batch* b, cudaStream_t s) {
  batch_setup_kernel<<<b->n_views, kBlock, 0, s>>>(b->C, world_trig(), b->cams, b->scal, b->insts, b->counters);
  return check_launch("batch_setup_kernel");
}

// The trace pass over the listed views.
int launch_trace(arbor_batch* b, const arbor_batch_config& cfg, int n_list, cudaStream_t s) {
  const dim3 grid(b->sms * cfg.ctas_per_sm);
  int* queues = b->counters + kViewQueues;
  if (cfg.queue == 12)
    batch_pool_kernel<12, false><<<grid, kBlock, batch_smem_bytes<12>(), s>>>(b->views, b->cams, b->insts, b->vlist, n_list, queues);
  else
    batch_pool_kernel<16, false><<<grid, kBlock, batch_smem_bytes<16>(), s>>>(b->views, b->cams, b->insts, b->vlist, n_list, queues);
  return check_launch("batch_pool_kernel");
}

// shadePixels: the shadow pass over the listed views, then the compose pass
// over the tile list.
int launch_shade(arbor_batch* b, const arbor_batch_config& cfg, const int4* tiles, int n_tiles, int n_list, cudaStream_t s) {
  const dim3 grid(b->sms * cfg.ctas_per_sm);
  int* queues = b->counters + kViewQueues + b->n_views;
  if (cfg.queue == 12)
    batch_pool_kernel<12, true><<<grid, kBlock, batch_smem_bytes<12>(), s>>>(b->views, b->cams, b->insts, b->vlist, n_list, queues);
  else
    batch_pool_kernel<16, true><<<grid, kBlock, batch_smem_bytes<16>(), s>>>(b->views, b->cams, b->insts, b->vlist, n_list, queues);
  if (int st = check_launch("batch_pool_kernel")) return st;
  batch_compose_kernel<<<b->sms * 8, kBlock, 0, s>>>(b->views, b->cams, b->insts, tiles, n_tiles, cfg.tile_width,
                                                     b->counters + kQueueCompose);
  return check_launch("batch_compose_kernel");
}

int launch_trace_shade(arbor_batch* b, const arbor_batch_config& cfg, const int4* tiles, int n_tiles, int n_list, cudaStream_t s) {
  if (int st = launch_trace(b, cfg, n_list, s)) return st;
  return launch_shade(b, cfg, tiles, n_tiles, n_list, s);
}

// Rebuild the tile and view lists for cfg and capture setup -> trace ->
// shadow -> compose -> filter.
int configure(arbor_batch* b, const arbor_batch_config& cfg) {
  std::vector<int> all(b->n_views);
  std::iota(all.begin(), all.end(), 0);
  std::vector<int4> t;
  const std::vector<int> order = view_order(b, all, cfg.order);
  trace_tiles(b, order, cfg.tile_width, t);
  const int n_ts = (int)t.size();
  filter_tiles(b, t);
  if (t.size() > b->tile_capacity) {
    set_error("arbor_batch: %zu tiles exceed the tile list capacity %zu", t.size(), b->tile_capacity);
    return ARBOR_ERR_LIMIT;
  }
  BATCH_CUDA(cudaStreamSynchronize(b->own));
  BATCH_CUDA(cudaMemcpyAsync(b->tiles, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice, b->own));
  BATCH_CUDA(cudaMemcpyAsync(b->vlist, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, b->own));
  BATCH_CUDA(cudaStreamSynchronize(b->own));
  b->n_ts = n_ts;
  b->n_filter = (int)t.size() - n_ts;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  BATCH_CUDA(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal));
  int st = launch_setup(b, b->own);
  if (!st) st = launch_trace_shade(b, cfg, b->tiles, b->n_ts, b->n_views, b->own);
  if (!st) {
    batch_filter_kernel<<<b->sms * 8, dim3(kFX, kFT), 0, b->own>>>(b->views, b->scal, b->tiles + b->n_ts, b->n_filter,
                                                                   b->counters + kQueueFilter);
    st = check_launch("batch_filter_kernel");
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->own, &g);
  if (st) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) return cuda_fail("cudaStreamEndCapture", e);
  b->graph = g;
  BATCH_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->cfg = cfg;
  return ARBOR_OK;
}

int live(arbor_batch* b, const char* what) {
  if (b == nullptr) {
    set_error("%s: batch is NULL", what);
    return ARBOR_ERR_NULL;
  }
  return ARBOR_OK;
}

int check_cameras(const float* C, int n, const char* what) {
  for (int v = 0; v < n; v++)
    for (int i = 0; i < 64; i++)
      if (!std::isfinite(C[(size_t)v * 64 + i])) {
        set_error("%s: view %d camera value C[%d] must be finite", what, v, i);
        return ARBOR_ERR_VALUE;
      }
  return ARBOR_OK;
}

// Order the batch's stream after the caller's.
int join_user(arbor_batch* b) {
  BATCH_CUDA(cudaEventRecord(b->joined, b->user));
  BATCH_CUDA(cudaStreamWaitEvent(b->own, b->joined, 0));
  return ARBOR_OK;
}
// Order the caller's stream after the batch's.
int join_back(arbor_batch* b) {
  BATCH_CUDA(cudaEventRecord(b->done, b->own));
  BATCH_CUDA(cudaStreamWaitEvent(b->user, b->done, 0));
  return ARBOR_OK;
}

}  // namespace

extern "C" int arbor_batch_create(arbor_batch** out, const int* seeds, int n_scenes, const arbor_batch_view* views, int n_views,
                                  arbor_stream stream) {
  if (out == nullptr || seeds == nullptr || views == nullptr) {
    set_error("arbor_batch_create: out, seeds and views must not be NULL");
    return ARBOR_ERR_NULL;
  }
  *out = nullptr;
  if (n_scenes < 1 || n_scenes > kMaxScenes || n_views < 1 || n_views > kMaxViews) {
    set_error("arbor_batch_create: need 1..%d scenes and 1..%d views (got %d, %d)", kMaxScenes, kMaxViews, n_scenes, n_views);
    return ARBOR_ERR_VALUE;
  }
  for (int s = 0; s < n_scenes; s++)
    if (seeds[s] < 0 || seeds[s] > 1000000) {
      set_error("Seed must be an integer from 0 to 1,000,000.");
      return ARBOR_ERR_VALUE;
    }
  uint64_t total = 0;
  for (int v = 0; v < n_views; v++) {
    const arbor_batch_view& w = views[v];
    if (w.scene < 0 || w.scene >= n_scenes) {
      set_error("arbor_batch_create: view %d names scene %d of %d", v, w.scene, n_scenes);
      return ARBOR_ERR_VALUE;
    }
    bool empty = false;
    if (int s = check_image("arbor_batch_create", w.width, w.height, &empty)) return s;
    if (empty) {
      set_error("arbor_batch_create: view %d is empty (%d x %d)", v, w.width, w.height);
      return ARBOR_ERR_VALUE;
    }
    if (int s = check_cameras(w.C, 1, "arbor_batch_create")) return s;
    total += (uint64_t)w.width * w.height;
  }
  if (!arbor_device_ready()) {
    set_error("arbor_batch_create: no sm_100 CUDA device is available");
    return ARBOR_ERR_NO_DEVICE;
  }
  arbor_batch* b = new (std::nothrow) arbor_batch();
  if (b == nullptr) {
    set_error("arbor_batch_create: out of host memory");
    return ARBOR_ERR_LIMIT;
  }
  auto fail = [&](int s) {
    arbor_batch_destroy(b);
    return s;
  };
  b->user = stream;
  b->n_scenes = n_scenes;
  b->n_views = n_views;
  b->seeds.assign(seeds, seeds + n_scenes);
  b->total_px = total;
  uint64_t off = 0;
  size_t tiles = 0;
  for (int v = 0; v < n_views; v++) {
    const size_t w = (size_t)views[v].width, h = (size_t)views[v].height;
    b->vw.push_back(views[v].width);
    b->vh.push_back(views[v].height);
    b->vscene.push_back(views[v].scene);
    b->offset.push_back(off);
    off += (uint64_t)w * h;
    // the most tiles either trace tile shape needs, plus the filter tiles
    tiles += std::max((w + 15) / 16 * ((h + 15) / 16), (w + 31) / 32 * ((h + 7) / 8)) + (w + kFX - 1) / kFX * ((h + kFY - 1) / kFY);
  }
  b->tile_capacity = tiles;
  int dev = 0;
  cudaError_t ce;
  if ((ce = cudaGetDevice(&dev)) != cudaSuccess) return fail(cuda_fail("cudaGetDevice", ce));
  if ((ce = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return fail(cuda_fail("cudaDeviceGetAttribute", ce));
  if ((ce = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking)) != cudaSuccess) return fail(cuda_fail("cudaStreamCreate", ce));
  if ((ce = cudaEventCreateWithFlags(&b->joined, cudaEventDisableTiming)) != cudaSuccess) return fail(cuda_fail("cudaEventCreate", ce));
  if ((ce = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming)) != cudaSuccess) return fail(cuda_fail("cudaEventCreate", ce));
  {
    const void* kernels[] = {(const void*)batch_pool_kernel<12, false>, (const void*)batch_pool_kernel<12, true>,
                             (const void*)batch_pool_kernel<16, false>, (const void*)batch_pool_kernel<16, true>};
    const int bytes[] = {(int)batch_smem_bytes<12>(), (int)batch_smem_bytes<12>(), (int)batch_smem_bytes<16>(), (int)batch_smem_bytes<16>()};
    for (int k = 0; k < 4; k++)
      if ((ce = cudaFuncSetAttribute(kernels[k], cudaFuncAttributeMaxDynamicSharedMemorySize, bytes[k])) != cudaSuccess)
        return fail(cuda_fail("cudaFuncSetAttribute", ce));
  }
  const size_t scene_bytes = kSceneStride * n_scenes, image_bytes = total * 16 * 5, pixel_bytes = total * 4;
  struct Alloc {
    void** p;
    size_t bytes;
  } allocs[] = {
      {(void**)&b->scenes, scene_bytes},
      {(void**)&b->images, image_bytes},
      {(void**)&b->pixels, pixel_bytes},
      {(void**)&b->C, (size_t)n_views * kC},
      {(void**)&b->views, (size_t)n_views * sizeof(BatchView)},
      {(void**)&b->cams, (size_t)n_views * sizeof(Camera)},
      {(void**)&b->scal, (size_t)n_views * sizeof(float4)},
      {(void**)&b->insts, (size_t)n_views * kForest * sizeof(Instance)},
      {(void**)&b->counters, (size_t)(kViewQueues + 2 * n_views) * sizeof(int)},
      {(void**)&b->vlist, (size_t)n_views * sizeof(int)},
      {(void**)&b->tiles, tiles * sizeof(int4)},
      {&b->scratch, arbor_sort_scratch_bytes()},
  };
  for (const Alloc& a : allocs) {
    if ((ce = cudaMalloc(a.p, a.bytes)) != cudaSuccess) return fail(cuda_fail("cudaMalloc (batch)", ce));
    b->allocated += a.bytes;
  }
  if ((ce = cudaMallocHost(&b->staging, (size_t)n_views * kC)) != cudaSuccess) return fail(cuda_fail("cudaMallocHost", ce));
  if (int st = join_user(b)) return fail(st);
  if ((ce = cudaMemsetAsync(b->images, 0, image_bytes, b->own)) != cudaSuccess) return fail(cuda_fail("cudaMemsetAsync", ce));
  if ((ce = cudaMemsetAsync(b->pixels, 0, pixel_bytes, b->own)) != cudaSuccess) return fail(cuda_fail("cudaMemsetAsync", ce));
  for (int s = 0; s < n_scenes; s++) {
    char* base = scene_base(b, s);
    if ((ce = cudaMemsetAsync(base, 0, kB, b->own)) != cudaSuccess) return fail(cuda_fail("cudaMemsetAsync", ce));
    if ((ce = cudaMemsetAsync(base + kOffNodes, 0, kNodes, b->own)) != cudaSuccess) return fail(cuda_fail("cudaMemsetAsync", ce));
    int st = arbor_buildScene(seeds[s], (float*)base, (float*)(base + kOffP), (uint32_t*)(base + kOffKeys), (uint32_t*)(base + kOffOrder),
                              (float*)(base + kOffNodes), nullptr, b->scratch, b->own);
    if (st) return fail(st);
  }
  std::vector<BatchView> hv(n_views);
  for (int v = 0; v < n_views; v++) {
    char* base = scene_base(b, b->vscene[v]);
    hv[v] = BatchView{(const float*)(base + kOffP), (const float*)(base + kOffNodes), (const uint32_t*)(base + kOffOrder),
                      image(b, 0, v), image(b, 1, v), image(b, 2, v), image(b, 3, v), image(b, 4, v), b->pixels + b->offset[v],
                      b->vw[v], b->vh[v]};
    memcpy(b->staging + (size_t)v * 64, views[v].C, kC);
  }
  if ((ce = cudaMemcpyAsync(b->views, hv.data(), hv.size() * sizeof(BatchView), cudaMemcpyHostToDevice, b->own)) != cudaSuccess)
    return fail(cuda_fail("cudaMemcpyAsync", ce));
  if ((ce = cudaMemcpyAsync(b->C, b->staging, (size_t)n_views * kC, cudaMemcpyHostToDevice, b->own)) != cudaSuccess)
    return fail(cuda_fail("cudaMemcpyAsync", ce));
  if ((ce = cudaStreamSynchronize(b->own)) != cudaSuccess) return fail(cuda_fail("cudaStreamSynchronize", ce));
  if (int st = configure(b, b->cfg)) return fail(st);
  *out = b;
  return ARBOR_OK;
}

extern "C" int arbor_batch_set_cameras(arbor_batch* b, const float* C, int n_views) {
  if (int s = live(b, "arbor_batch_set_cameras")) return s;
  if (C == nullptr) {
    set_error("arbor_batch_set_cameras: C is NULL");
    return ARBOR_ERR_NULL;
  }
  if (n_views != b->n_views) {
    set_error("arbor_batch_set_cameras: %d records for a batch of %d views", n_views, b->n_views);
    return ARBOR_ERR_VALUE;
  }
  if (int s = check_cameras(C, n_views, "arbor_batch_set_cameras")) return s;
  // The previous upload must have left the staging buffer.
  BATCH_CUDA(cudaStreamSynchronize(b->own));
  memcpy(b->staging, C, (size_t)n_views * kC);
  if (int s = join_user(b)) return s;
  BATCH_CUDA(cudaMemcpyAsync(b->C, b->staging, (size_t)n_views * kC, cudaMemcpyHostToDevice, b->own));
  return join_back(b);
}

extern "C" int arbor_batch_configure(arbor_batch* b, const arbor_batch_config* cfg) {
  if (int s = live(b, "arbor_batch_configure")) return s;
  if (cfg == nullptr) {
    set_error("arbor_batch_configure: cfg is NULL");
    return ARBOR_ERR_NULL;
  }
  if (!valid_config(*cfg)) {
    set_error("arbor_batch_configure: tile_width 16|32, ctas_per_sm 1|2, order 0|1, queue 12|16 (got %d %d %d %d)", cfg->tile_width,
              cfg->ctas_per_sm, cfg->order, cfg->queue);
    return ARBOR_ERR_VALUE;
  }
  if (int s = join_user(b)) return s;
  return configure(b, *cfg);
}

extern "C" int arbor_batch_get_config(arbor_batch* b, arbor_batch_config* cfg) {
  if (int s = live(b, "arbor_batch_get_config")) return s;
  if (cfg == nullptr) {
    set_error("arbor_batch_get_config: cfg is NULL");
    return ARBOR_ERR_NULL;
  }
  *cfg = b->cfg;
  return ARBOR_OK;
}

extern "C" int arbor_batch_render(arbor_batch* b) {
  if (int s = live(b, "arbor_batch_render")) return s;
  if (int s = join_user(b)) return s;
  BATCH_CUDA(cudaGraphLaunch(b->exec, b->own));
  count_launch(5);
  b->renders++;
  return join_back(b);
}

extern "C" int arbor_batch_profile(arbor_batch* b, float* ms4) {
  if (int s = live(b, "arbor_batch_profile")) return s;
  if (ms4 == nullptr) {
    set_error("arbor_batch_profile: ms4 is NULL");
    return ARBOR_ERR_NULL;
  }
  // The graph's kernels launched one by one, with an event between the
  // stages (the shade stage is the shadow and compose kernels).
  cudaEvent_t ev[5] = {};
  int status = ARBOR_OK;
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) status = cuda_fail("cudaEventCreate", cudaGetLastError());
  if (status == ARBOR_OK) status = join_user(b);
  if (status == ARBOR_OK) {
    cudaEventRecord(ev[0], b->own);
    status = launch_setup(b, b->own);
    cudaEventRecord(ev[1], b->own);
  }
  if (status == ARBOR_OK) {
    status = launch_trace(b, b->cfg, b->n_views, b->own);
    cudaEventRecord(ev[2], b->own);
  }
  if (status == ARBOR_OK) {
    status = launch_shade(b, b->cfg, b->tiles, b->n_ts, b->n_views, b->own);
    cudaEventRecord(ev[3], b->own);
  }
  if (status == ARBOR_OK) {
    batch_filter_kernel<<<b->sms * 8, dim3(kFX, kFT), 0, b->own>>>(b->views, b->scal, b->tiles + b->n_ts, b->n_filter,
                                                                   b->counters + kQueueFilter);
    status = check_launch("batch_filter_kernel");
    cudaEventRecord(ev[4], b->own);
  }
  if (status == ARBOR_OK) {
    count_launch(5);
    cudaError_t ce = cudaEventSynchronize(ev[4]);
    if (ce != cudaSuccess) status = cuda_fail("cudaEventSynchronize", ce);
    for (int k = 0; k < 4 && status == ARBOR_OK; k++) cudaEventElapsedTime(&ms4[k], ev[k], ev[k + 1]);
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (status == ARBOR_OK) status = join_back(b);
  return status;
}

extern "C" int arbor_batch_autotune(arbor_batch* b, int sample_views, arbor_batch_config* best, float* ms_table) {
  if (int s = live(b, "arbor_batch_autotune")) return s;
  // Views spread evenly over the batch (all of them when sample_views <= 0).
  std::vector<int> subset;
  const int n = (sample_views <= 0 || sample_views >= b->n_views) ? b->n_views : sample_views;
  for (int k = 0; k < n; k++) subset.push_back((int)((int64_t)k * b->n_views / n));
  const arbor_batch_config keep = b->cfg;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BATCH_CUDA(cudaEventCreate(&e0));
  BATCH_CUDA(cudaEventCreate(&e1));
  int status = join_user(b), slot = 0;
  float best_ms = -1.0f;
  arbor_batch_config chosen = keep;
  for (int tw : {16, 32})
    for (int ctas : {1, 2})
      for (int order : {0, 1})
        for (int q : {12, 16}) {
          const arbor_batch_config cfg{tw, ctas, order, q};
          std::vector<int4> t;
          const std::vector<int> vo = view_order(b, subset, order);
          trace_tiles(b, vo, tw, t);
          float ms = 0.0f;
          if (status == ARBOR_OK) {
            // the previous candidate's kernels must be done with the tile list
            cudaError_t ce = cudaStreamSynchronize(b->own);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(b->tiles, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice, b->own);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(b->vlist, vo.data(), vo.size() * sizeof(int), cudaMemcpyHostToDevice, b->own);
            if (ce != cudaSuccess) status = cuda_fail("autotune tile upload", ce);
            // one untimed run, then one timed run
            for (int rep = 0; rep < 2 && status == ARBOR_OK; rep++) {
              if ((status = launch_setup(b, b->own))) break;
              if (rep == 1 && (ce = cudaEventRecord(e0, b->own)) != cudaSuccess) status = cuda_fail("cudaEventRecord", ce);
              if (status || (status = launch_trace_shade(b, cfg, b->tiles, (int)t.size(), (int)vo.size(), b->own))) break;
              if (rep == 1 && (ce = cudaEventRecord(e1, b->own)) != cudaSuccess) status = cuda_fail("cudaEventRecord", ce);
            }
            if (status == ARBOR_OK) {
              if ((ce = cudaEventSynchronize(e1)) != cudaSuccess)
                status = cuda_fail("cudaEventSynchronize", ce);
              else
                cudaEventElapsedTime(&ms, e0, e1);
            }
            count_launch(8);  // two runs of setup, trace, shadow, compose
          }
          if (ms_table) ms_table[slot] = ms;
          slot++;
          if (status == ARBOR_OK && (best_ms < 0.0f || ms < best_ms)) {
            best_ms = ms;
            chosen = cfg;
          }
        }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status) {
    configure(b, keep);
    return status;
  }
  if (int s = configure(b, chosen)) return s;
  if (best) *best = chosen;
  return join_back(b);
}

extern "C" int arbor_batch_view_buffers(arbor_batch* b, int view, arbor_engine_buffers* out) {
  if (int s = live(b, "arbor_batch_view_buffers")) return s;
  if (out == nullptr) {
    set_error("arbor_batch_view_buffers: out is NULL");
    return ARBOR_ERR_NULL;
  }
  if (view < 0 || view >= b->n_views) {
    set_error("arbor_batch_view_buffers: view %d of %d", view, b->n_views);
    return ARBOR_ERR_VALUE;
  }
  char* base = scene_base(b, b->vscene[view]);
  *out = arbor_engine_buffers{(float*)base, (float*)(base + kOffP), (uint32_t*)(base + kOffKeys), (uint32_t*)(base + kOffOrder),
                              (float*)(base + kOffNodes), b->C + (size_t)view * 64, nullptr, image(b, 0, view), image(b, 1, view),
                              image(b, 2, view), image(b, 3, view), image(b, 4, view), b->pixels + b->offset[view]};
  return ARBOR_OK;
}

extern "C" int arbor_batch_inspect(arbor_batch* b, arbor_batch_info* info) {
  if (int s = live(b, "arbor_batch_inspect")) return s;
  if (info == nullptr) {
    set_error("arbor_batch_inspect: info is NULL");
    return ARBOR_ERR_NULL;
  }
  info->n_scenes = b->n_scenes;
  info->n_views = b->n_views;
  info->total_pixels = b->total_px;
  info->allocated_bytes = b->allocated;
  info->trace_tiles = b->n_ts;
  info->filter_tiles = b->n_filter;
  info->renders = b->renders;
  info->launches_per_render = 5;
  info->config = b->cfg;
  return ARBOR_OK;
}

extern "C" int arbor_batch_read_pixels(arbor_batch* b, uint32_t* host, size_t count) {
  if (int s = live(b, "arbor_batch_read_pixels")) return s;
  if (host == nullptr) {
    set_error("arbor_batch_read_pixels: host is NULL");
    return ARBOR_ERR_NULL;
  }
  if (count < b->total_px) {
    set_error("arbor_batch_read_pixels: %zu elements cannot hold %llu pixels", count, (unsigned long long)b->total_px);
    return ARBOR_ERR_LIMIT;
  }
  if (int s = join_user(b)) return s;
  BATCH_CUDA(cudaMemcpyAsync(host, b->pixels, b->total_px * 4, cudaMemcpyDeviceToHost, b->own));
  BATCH_CUDA(cudaStreamSynchronize(b->own));
  return ARBOR_OK;
}

extern "C" int arbor_batch_destroy(arbor_batch* b) {
  if (b == nullptr) return ARBOR_OK;
  if (b->own) cudaStreamSynchronize(b->own);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  void* bufs[] = {b->scenes, b->images, b->pixels, b->C, b->views, b->cams, b->scal, b->insts, b->counters, b->vlist, b->tiles, b->scratch};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (b->staging) cudaFreeHost(b->staging);
  if (b->joined) cudaEventDestroy(b->joined);
  if (b->done) cudaEventDestroy(b->done);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
  return ARBOR_OK;
}
