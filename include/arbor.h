/*
 * arbor.h - C ABI of the B200-native Arbor render path.
 *
 * Drop-in for the reference's 12 kernel entry points.  Each entry keeps the
 * buffer order, element types and scalars of the reference's kernel metadata
 * (generated/<entry>.json "bindings"/"scalars", generated/manifest.json) and
 * the reference kernel's semantics (Arbor.cu, cited per entry).  The engine
 * (src/engine.js:26-53) bound buffers and dispatched workgroups through
 * Kernel.bind + ComputeBatch.dispatch (vendor/cuda-webshader/runtime/
 * runtime.js:279,347); here the caller passes device pointers and a CUDA
 * stream, and the callee derives the grid.
 *
 * Conventions
 *  - All buffers are caller-owned device memory with the ABI sizes below.
 *    Entry points never allocate or free caller buffers.
 *  - Every entry returns an arbor_status (0 = ARBOR_OK).  No exception or
 *    abort crosses the ABI.  arbor_last_error() gives a message for the
 *    calling thread's most recent failure.
 *  - Calls on one stream execute in issue order, as the reference's
 *    dispatches inside one pass do (docs/ARCHITECTURE.md:19).
 *  - Argument checks mirror runtime.js: non-finite scalars
 *    (runtime.js:18-22), writable aliasing across bindings (runtime.js:325),
 *    workgroup counts above 65535 (runtime.js:352); plus null and
 *    misaligned pointers, which a WebGPU binding cannot express.
 *  - A launch error is reported as ARBOR_ERR_CUDA; the kernel itself runs
 *    asynchronously on `stream`.
 */
#ifndef ARBOR_H
#define ARBOR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define ARBOR_API __attribute__((visibility("default")))
#else
#define ARBOR_API
#endif

/* Same type as cudaStream_t; NULL is the legacy default stream. */
typedef struct CUstream_st* arbor_stream;

/* ABI constants (kernels/common.cu:2-12, src/engine.js:2). */
#define ARBOR_CAPACITY 32768
#define ARBOR_NODE_COUNT 65536
#define ARBOR_PS 24
#define ARBOR_CS 20
#define ARBOR_CURVES 2109
#define ARBOR_WOOD_COUNT 5124
#define ARBOR_LEAF_COUNT 24192
#define ARBOR_ROCK_COUNT 96
#define ARBOR_OBJECT_COUNT 29412
#define ARBOR_FOREST_SIDE 18
#define ARBOR_FOREST_COUNT 324

/* Buffer sizes in elements (src/engine.js:22,40). */
#define ARBOR_B_FLOATS (ARBOR_CURVES * ARBOR_CS)
#define ARBOR_P_FLOATS (ARBOR_CAPACITY * ARBOR_PS)
#define ARBOR_NODES_FLOATS (ARBOR_NODE_COUNT * 8)
#define ARBOR_C_FLOATS 64
#define ARBOR_I_FLOATS 32
/* Hit, Linear, Guide, Filtered, History: width*height*4 floats.
 * Pixels: width*height uint32 (RGBA8, R in the low byte). */

typedef enum arbor_status {
  ARBOR_OK = 0,
  ARBOR_ERR_NULL = 1,          /* a required pointer is NULL */
  ARBOR_ERR_VALUE = 2,         /* a scalar is non-finite or out of range */
  ARBOR_ERR_ALIGN = 3,         /* a buffer is not 16-byte aligned */
  ARBOR_ERR_ALIAS = 4,         /* a writable buffer overlaps another binding */
  ARBOR_ERR_LIMIT = 5,         /* grid above 65535 workgroups per dimension, or
                                  a size above a stated maximum */
  ARBOR_ERR_CUDA = 6,          /* a CUDA runtime call failed */
  ARBOR_ERR_TIMEOUT = 7,       /* a bounded device wait gave up */
  ARBOR_ERR_STATE = 8,         /* object disposed or in the wrong state */
  ARBOR_ERR_NO_DEVICE = 9      /* no CUDA device is available */
} arbor_status;

/* Message for the calling thread's last failing call ("" if none). */
ARBOR_API const char* arbor_last_error(void);
/* Human-readable name of a status code. */
ARBOR_API const char* arbor_status_name(int status);
/* 1 when this library was built for sm_100a and a device is present. */
ARBOR_API int arbor_device_ready(void);
/* Number of kernels this library has launched in this process (all entries,
 * all threads).  Tests and the benchmark use it to count launches. */
ARBOR_API uint64_t arbor_launch_count(void);

/* ---------------------------------------------------------------------------
 * The 12 reference entry points.
 * ------------------------------------------------------------------------- */

/* One generation of branch curves into B (Arbor.cu:76-102; bindings B rw;
 * scalars level, seed).  Levels 0..4 launch 9/12/72/288/1728 threads as the
 * harness does (tests/native_harness.cpp:45); any other level runs the level-4
 * thread count with the reference kernel's fall-through semantics. */
ARBOR_API int arbor_growTree(float* B, int level, int seed, arbor_stream stream);

/* 32768 primitive records (Arbor.cu:103-131; bindings B r, P w; scalar seed). */
ARBOR_API int arbor_makePrimitives(const float* B, float* P, int seed, arbor_stream stream);

/* 30-bit Morton key per primitive centroid and identity order
 * (Arbor.cu:138-139; bindings P r, Keys w, Order w). */
ARBOR_API int arbor_makeKeys(const float* P, uint32_t* Keys, uint32_t* Order, arbor_stream stream);

/* One bitonic compare-exchange stage over (key, index) (Arbor.cu:140;
 * bindings Keys rw, Order rw; scalars distance, span).  distance must lie in
 * 0..32767 (a larger one indexes past the 32768 records). */
ARBOR_API int arbor_sortPass(uint32_t* Keys, uint32_t* Order, int distance, int span, arbor_stream stream);

/* Leaf nodes 32768+i from Morton order (Arbor.cu:141; bindings P r, Order r,
 * Nodes w). */
ARBOR_API int arbor_makeBounds(const float* P, const uint32_t* Order, float* Nodes, arbor_stream stream);

/* One BVH level: parents first..2*first-1 (Arbor.cu:142; bindings Nodes rw;
 * scalar first).  first must lie in 0..16384. */
ARBOR_API int arbor_reduceBounds(float* Nodes, int first, arbor_stream stream);

/* Camera/state record defaults (Arbor.cu:181; bindings C w, P r; scalar seed). */
ARBOR_API int arbor_initCamera(float* C, const float* P, int seed, arbor_stream stream);

/* Input record -> camera state (Arbor.cu:182; bindings C rw, I r, P r;
 * scalars delta (finite), width, height). */
ARBOR_API int arbor_updateCamera(float* C, const float* I, const float* P, float delta, int width, int height, arbor_stream stream);

/* Progressive sampling control (no reference kernel; the harness writes these
 * fields directly before each sample, tests/native_harness.cpp:62):
 * C[9] = sample, C[10] = reset ? 1 : 0.  sample must lie in 0..2^24. */
ARBOR_API int arbor_setSample(float* C, int sample, int reset, arbor_stream stream);

/* Primary hit per pixel: Hit[4*px] = {t, primId, treeId, footprint}
 * (Arbor.cu:252; bindings P, Nodes, Order, C r; Hit w; scalars width, height). */
ARBOR_API int arbor_tracePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int width, int height, arbor_stream stream);

/* Radiance and albedo per pixel, sun shadows when C[22] > 0.5
 * (Arbor.cu:277-289; bindings P, Nodes, Order, C, Hit r; Linear, Guide w). */
ARBOR_API int arbor_shadePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, float* Linear, float* Guide, int width, int height, arbor_stream stream);

/* 5x5 same-surface demodulated filter (Arbor.cu:292-302; bindings Linear,
 * Guide, Hit r; Filtered w; C r). */
ARBOR_API int arbor_filterLighting(const float* Linear, const float* Guide, const float* Hit, float* Filtered, const float* C, int width, int height, arbor_stream stream);

/* Progressive mean, ACES, gamma, vignette, RGBA8 (Arbor.cu:303-304; bindings
 * Filtered r, History rw, Pixels w, C r). */
ARBOR_API int arbor_resolvePixels(const float* Filtered, float* History, uint32_t* Pixels, const float* C, int width, int height, arbor_stream stream);

/* ---------------------------------------------------------------------------
 * Fused and extra entry points (no single reference counterpart).
 * ------------------------------------------------------------------------- */

/* Stable LSD radix sort of (Keys, Order) by key: the same (key, index) order
 * as the reference's 120 bitonic sortPass stages (src/engine.js:31) and the
 * harness's std::sort of pairs (tests/native_harness.cpp:47), provided Order
 * holds increasing indices on entry, as makeKeys leaves it.  `scratch` is
 * caller-owned device memory of at least arbor_sort_scratch_bytes() bytes. */
ARBOR_API size_t arbor_sort_scratch_bytes(void);
ARBOR_API int arbor_sortKeys(uint32_t* Keys, uint32_t* Order, void* scratch, arbor_stream stream);

/* arbor_sortKeys without a scratch argument, for callers that cannot
 * allocate device memory (no reference counterpart).  Sorts the first `count`
 * (Keys, Order) pairs, count <= 32768, in the same order arbor_sortKeys
 * gives; a larger count returns ARBOR_ERR_LIMIT.  It allocates nothing: its
 * ping-pong buffer is a fixed 256 KB array inside the library, which every
 * GPU that loads the library keeps until the process exits.  A call outside
 * stream capture looks up that array's device address (cudaGetSymbolAddress);
 * a call during capture reuses the address its device's last call outside
 * capture found, so make one call on a device before capturing, and again
 * after a device reset (which can move the array).  All calls
 * share the one array: calls that overlap on the GPU (different streams, no
 * ordering between them) race and corrupt each other's results. */
ARBOR_API int arbor_sortKeysNoAlloc(uint32_t* Keys, uint32_t* Order, int count, arbor_stream stream);

/* Makes leaf nodes (as makeBounds) and all 15 parent levels (as the 15
 * reduceBounds dispatches, src/engine.js:32) in two launches. */
ARBOR_API int arbor_buildBounds(const float* P, const uint32_t* Order, float* Nodes, arbor_stream stream);

/* The whole scene build of src/engine.js:27-33 for one seed: growTree x5,
 * makePrimitives, makeKeys, sort, makeBounds, reduceBounds x15, initCamera.
 * Bit-identical Keys/Order/Nodes to the reference sequence given the same P.
 * B must be zeroed by the caller before the first build (the reference's
 * buffers start zeroed); `scratch` as for arbor_sortKeys.  C may be NULL to
 * leave the camera untouched. */
ARBOR_API int arbor_buildScene(int seed, float* B, float* P, uint32_t* Keys, uint32_t* Order, float* Nodes, float* C, void* scratch, arbor_stream stream);

/* Single-tree scene (no reference counterpart; mirrors the harness's direct
 * traceTree use at tests/native_harness.cpp:84): the resident tree traced
 * with an identity instance.  Hit.treeId is -1; shading uses the tree-local
 * normal, no per-tree tint, and shadow rays through the same tree. */
ARBOR_API int arbor_traceTreePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int width, int height, arbor_stream stream);
ARBOR_API int arbor_shadeTreePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, float* Linear, float* Guide, int width, int height, arbor_stream stream);
/* tracePixels / shadePixels (single_tree = 0) or their single-tree forms
 * (single_tree != 0) with the reference's traversal as written: one ray per
 * thread, candidate primitives tested in visiting order, children nearest
 * entry first (Arbor.cu:220-289).  Same buffers and results as the entries
 * above; slower.  They exist to check that the batched passes' visiting
 * order does not change a result.  No counterpart in the reference (which
 * has only this order). */
ARBOR_API int arbor_tracePixelsInOrder(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int width, int height, int single_tree, arbor_stream stream);
ARBOR_API int arbor_shadePixelsInOrder(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, float* Linear, float* Guide, int width, int height, int single_tree, arbor_stream stream);

/* A forest of several species (no reference counterpart: the reference's
 * 324 instances all share one resident tree, README.md:8,
 * docs/ARCHITECTURE.md:5).  Instance t keeps the reference's transform, wind
 * phase and tint (forestPos/Scale/Yaw/Seed of t, Arbor.cu:57-69) but takes
 * its geometry - its own records and its own BVH - from scene species_of[t]
 * (host array of ARBOR_FOREST_COUNT ints in 0..n_species-1).  P, Nodes and
 * Order hold n_species scenes back to back (each the ABI size: 32768*24,
 * 65536*8 and 32768 elements), e.g. n_species arbor_buildScene results with
 * different seeds.  Hit.primId is a record id of the hit instance's scene.
 * The 2D DDA and bounding spheres are the reference's.  With every
 * species_of[t] = 0 the results equal arbor_tracePixels / arbor_shadePixels
 * on scene 0.  n_species at most ARBOR_MAX_SPECIES. */
#define ARBOR_MAX_SPECIES 256
ARBOR_API int arbor_traceSpeciesPixels(const float* P, const float* Nodes, const uint32_t* Order, int n_species, const int* species_of, const float* C, float* Hit, int width, int height, arbor_stream stream);
ARBOR_API int arbor_shadeSpeciesPixels(const float* P, const float* Nodes, const uint32_t* Order, int n_species, const int* species_of, const float* C, const float* Hit, float* Linear, float* Guide, int width, int height, arbor_stream stream);

/* shadePixels (Arbor.cu:277-289) that also writes the shading normal of
 * each pixel (world space, facing the camera; zero for sky) into Normal
 * (W*H float4, .w = 0): the G-buffer the learned denoiser reads.  No
 * reference counterpart: the reference keeps the normal inside shadePixels. */
ARBOR_API int arbor_shadeGBuffer(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, float* Linear, float* Guide, float* Normal, int width, int height, arbor_stream stream);

/* filterLighting followed by resolvePixels in one launch; writes Filtered,
 * History and Pixels exactly as the two separate entries do. */
ARBOR_API int arbor_filterResolve(const float* Linear, const float* Guide, const float* Hit, float* Filtered, float* History, uint32_t* Pixels, const float* C, int width, int height, arbor_stream stream);

/* The forest instance table of a world seed (C[31]): per tree t of the
 * 18x18 grid, the values the reference's forest helpers compute on the fly
 * (forestSeed, forestPos, forestScale, forestYaw, the wind phase;
 * Arbor.cu:57-69, 279), as the trace and shade kernels hold them.  Writes
 * ARBOR_FOREST_COUNT records of ARBOR_INSTANCE_FLOATS 4-byte words:
 * {pos.x, pos.z, scale, sphere centre y = 4.4 scale, sphere radius = 6.6
 * scale, cos(-yaw), sin(-yaw), cos(yaw), sin(yaw), phase, seed (int32), 0}.
 * Inspection helper; no single reference counterpart. */
#define ARBOR_INSTANCE_FLOATS 12
ARBOR_API int arbor_forestInstances(int world_seed, float* instances, arbor_stream stream);

/* Profiling helper (no reference counterpart): counts the traversal and
 * intersection events one tracePixels (single_tree = 0) or traceTreePixels
 * (single_tree != 0) launch performs, per thread, into `slots` (caller-owned,
 * arbor_trace_work_slots(width, height) uint32 values: 16 per thread, events
 * in the order ray, cell, tree, node, wood, march, bark, wood-shadow, leaf,
 * newton-start, newton, stone, segment).  It runs the same code compiled with
 * counters and writes no Hit. */
ARBOR_API size_t arbor_trace_work_slots(int width, int height);
ARBOR_API int arbor_traceWork(const float* P, const float* Nodes, const uint32_t* Order, const float* C, int width, int height, int single_tree, uint32_t* slots, arbor_stream stream);
/* The same count for one shadePixels launch on the given Hit records: the
 * shading's own events (surface normals) and, per shadow segment toward the
 * sun, event 12 (segment) plus its traversal and primitive-test events. */
ARBOR_API int arbor_shadeWork(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, int width, int height, int single_tree, uint32_t* slots, arbor_stream stream);

/* ---------------------------------------------------------------------------
 * Engine: the C++ host of src/engine.js (generate / resize / frame /
 * inspect / dispose) over the entries above.
 * ------------------------------------------------------------------------- */
typedef struct arbor_engine arbor_engine;

typedef struct arbor_engine_buffers {
  float* B; float* P; uint32_t* Keys; uint32_t* Order; float* Nodes; float* C; float* I;
  float* Hit; float* Linear; float* Guide; float* Filtered; float* History; uint32_t* Pixels;
} arbor_engine_buffers;

typedef struct arbor_engine_info {
  int width, height, seed, single_tree;
  uint64_t frames;
  uint64_t allocated_bytes;     /* all engine device buffers */
  uint64_t scene_bytes;         /* B + P + Keys + Order + Nodes (src/engine.js:55) */
  uint32_t launches_per_frame;  /* kernels one arbor_engine_frame launches */
  float camera[64];             /* copy of C after the last frame */
  float ms_build, ms_visibility, ms_lighting, ms_resolve; /* last timed phases */
} arbor_engine_info;

/* Creates an engine on the current device: allocates the ABI buffers for
 * width x height (rounded as src/engine.js:36: width up to a multiple of 64,
 * at least 320; height up to a multiple of 8, at least 192) and builds the
 * scene for `seed` (integer 0..1,000,000, src/engine.js:28).  single_tree != 0
 * selects the one-tree scene. */
ARBOR_API int arbor_engine_create(arbor_engine** out, int width, int height, int seed, int single_tree, arbor_stream stream);
ARBOR_API int arbor_engine_generate(arbor_engine* e, int seed);
ARBOR_API int arbor_engine_resize(arbor_engine* e, int width, int height);
/* Copies a 32-float input record (host memory) into I for the next frame. */
ARBOR_API int arbor_engine_set_input(arbor_engine* e, const float* input32);
/* Overwrites the 64-float camera/state record C from host memory, as the
 * harness writes Renderer::c directly (tests/native_harness.cpp:61-62). */
ARBOR_API int arbor_engine_set_state(arbor_engine* e, const float* state64);
/* One frame: updateCamera, trace, shade, filter+resolve (src/engine.js:45-53). */
ARBOR_API int arbor_engine_frame(arbor_engine* e, float dt);
/* Per-phase CUDA-event timing of subsequent frames on/off. */
ARBOR_API int arbor_engine_set_timing(arbor_engine* e, int enabled);
ARBOR_API int arbor_engine_inspect(arbor_engine* e, arbor_engine_info* info);
ARBOR_API int arbor_engine_buffers_get(arbor_engine* e, arbor_engine_buffers* out);
/* Copies Pixels to host memory (width*height uint32) on the engine stream
 * and waits for it. */
ARBOR_API int arbor_engine_read_pixels(arbor_engine* e, uint32_t* host, size_t count);
/* Releases the engine's device memory (src/engine.js:57); the handle stays
 * valid and every later call on it returns ARBOR_ERR_STATE. */
ARBOR_API int arbor_engine_dispose(arbor_engine* e);
/* Disposes (if needed) and frees the handle. */
ARBOR_API int arbor_engine_destroy(arbor_engine* e);
/* Writes the engine's Pixels as a binary PPM, as the harness's
 * Renderer::save does (tests/native_harness.cpp:53). */
ARBOR_API int arbor_engine_save_ppm(arbor_engine* e, const char* path);

/* Image files from host memory.  PPM: "P6\n<w> <h>\n255\n" then R, G, B
 * bytes per pixel, R being Pixels' low byte (native_harness.cpp:53).  PFM
 * (no reference counterpart; float dumps of Linear, Guide, Filtered or a
 * denoised image): "PF\n<w> <h>\n-1.0\n" then little-endian float RGB rows,
 * bottom row first. */
ARBOR_API int arbor_write_ppm(const char* path, const uint32_t* pixels, int width, int height);
ARBOR_API int arbor_write_pfm(const char* path, const float* rgba, int width, int height);


/* ---------------------------------------------------------------------------
 * Batched rendering: many views of many resident scenes, each view with its
 * own resolution and camera/state record, rendered by one CUDA graph launch
 * (a per-view setup kernel, persistent trace and shade kernels and a
 * persistent filter+resolve kernel, all pulling tiles from global queues).
 * No reference counterpart: the reference renders one view per frame
 * (src/engine.js:45-53).  Each view renders as arbor_tracePixels +
 * arbor_shadePixels + arbor_filterResolve render it on the same scene and C.
 * Forest scenes only.
 * ------------------------------------------------------------------------- */
typedef struct arbor_batch arbor_batch;

typedef struct arbor_batch_view {
  int scene;        /* index into the seeds array given to arbor_batch_create */
  int width, height;
  int reserved;
  float C[64];      /* camera/state record (Arbor.cu:179-182 layout); C[31] is the forest's world seed */
} arbor_batch_view;

typedef struct arbor_batch_config {
  int tile_width;   /* shading (compose) tile: 16 (16x16 pixels) or 32 (32x8 pixels) */
  int ctas_per_sm;  /* persistent CTAs per SM: 1 or 2 */
  int order;        /* view order of every pass: 0 as given, 1 largest views first */
  int queue;        /* warp-batch queue depth, candidates per lane: 12 or 16 */
} arbor_batch_config;

typedef struct arbor_batch_info {
  int n_scenes, n_views;
  uint64_t total_pixels;
  uint64_t allocated_bytes;
  int trace_tiles, filter_tiles;
  uint64_t renders;
  uint32_t launches_per_render;   /* kernels in the graph */
  arbor_batch_config config;
} arbor_batch_info;

/* Builds every scene (seeds: integers 0..1,000,000) and allocates every
 * view's Hit/Linear/Guide/Filtered/History/Pixels on the current device.
 * The batch works on a stream of its own, ordered after `stream` at each
 * call, and `stream` is ordered after the work each call queues.  Default
 * configuration: 16x16 tiles, 2 CTAs/SM, view order, queue depth 16 (the
 * single-image kernels' depth). */
ARBOR_API int arbor_batch_create(arbor_batch** out, const int* seeds, int n_scenes, const arbor_batch_view* views, int n_views, arbor_stream stream);
/* Replaces every view's camera record (n_views x 64 floats, host memory). */
ARBOR_API int arbor_batch_set_cameras(arbor_batch* b, const float* C, int n_views);
ARBOR_API int arbor_batch_configure(arbor_batch* b, const arbor_batch_config* cfg);
ARBOR_API int arbor_batch_get_config(arbor_batch* b, arbor_batch_config* cfg);
/* Times the trace, shadow and compose kernels of every configuration (16, ordered by
 * tile_width, ctas_per_sm, order, queue, the last varying fastest) on
 * `sample_views` views spread over the batch (all when <= 0), writes the
 * times to ms_table (nullable, 16 floats), keeps the fastest and returns it
 * in best (nullable).  The sample renders overwrite those views' Hit,
 * Linear and Guide. */
ARBOR_API int arbor_batch_autotune(arbor_batch* b, int sample_views, arbor_batch_config* best, float* ms_table);
/* Renders every view: one graph launch. */
ARBOR_API int arbor_batch_render(arbor_batch* b);
/* Renders every view with the graph's kernels launched one by one and writes
 * each stage's duration (CUDA events, ms) to ms4: setup, trace, shade (the
 * shadow and compose kernels), filter+resolve. */
ARBOR_API int arbor_batch_profile(arbor_batch* b, float* ms4);
/* Device buffers of one view (its scene's records, its C record and images). */
ARBOR_API int arbor_batch_view_buffers(arbor_batch* b, int view, arbor_engine_buffers* out);
ARBOR_API int arbor_batch_inspect(arbor_batch* b, arbor_batch_info* info);
/* Copies every view's Pixels, view after view, into host memory and waits. */
ARBOR_API int arbor_batch_read_pixels(arbor_batch* b, uint32_t* host, size_t count);
ARBOR_API int arbor_batch_destroy(arbor_batch* b);


/* ---------------------------------------------------------------------------
 * Learned denoiser (no reference counterpart; the reference's denoiser is
 * filterLighting, Arbor.cu:292-302, which stays available): a 4-level
 * convolutional encoder-decoder (channels 32/64/96/128, 3x3 kernels, leaky
 * ReLU) over 16 BF16 feature channels per pixel (log(1 + radiance), albedo,
 * normal, log(1 + depth), log(1 + filterLighting's radiance)), predicting
 * log(1 + radiance) as a correction of a base image (filterLighting's
 * output at the same sample count).  BF16 weights and activations, tensor-core products
 * accumulated in FP32, FP32 master weights and Adam moments; trained and
 * run by this library's own forward and backward kernels.  Image sizes are
 * multiples of 8.  All calls run on the stream given at creation.
 * ------------------------------------------------------------------------- */
typedef struct arbor_denoiser arbor_denoiser;

/* Creates the network (He-normal weights from `seed`) with working buffers
 * for up to max_batch images of max_width x max_height pixels. */
ARBOR_API int arbor_denoiser_create(arbor_denoiser** out, int max_batch, int max_width, int max_height, uint32_t seed, arbor_stream stream);
ARBOR_API int arbor_denoiser_param_count(arbor_denoiser* d, size_t* count);
/* FP32 parameters, layer after layer: weights [cout][3][3][cin], then biases. */
ARBOR_API int arbor_denoiser_get_params(arbor_denoiser* d, float* host, size_t count);
ARBOR_API int arbor_denoiser_set_params(arbor_denoiser* d, const float* host, size_t count);
/* Packs one image's features (W*H*16 BF16, as uint16_t) from the 1-spp
 * Linear, Guide (albedo), Normal (arbor_shadeGBuffer), Hit (depth) and
 * Filtered (filterLighting of that sample). */
ARBOR_API int arbor_denoiser_features(const float* Linear, const float* Guide, const float* Normal, const float* Hit, const float* Filtered, int width, int height, uint16_t* features, arbor_stream stream);
/* One Adam step on a batch: features (batch images back to back), the base
 * image the network corrects (Filtered) and the target Linear (float4 per
 * pixel); L1 loss in log(1 + radiance).  loss (host, nullable) receives the
 * batch's mean loss before the step, after the step completes. */
ARBOR_API int arbor_denoiser_train_step(arbor_denoiser* d, const uint16_t* features, const float* base, const float* target, int batch, int width, int height, float lr, float* loss);
/* The gradient train_step would apply, without applying it: the loss's
 * gradient with respect to every parameter (count >= param_count floats,
 * host memory, the get_params layout) and the loss (host, nullable); the
 * parameters and the Adam state are unchanged. */
ARBOR_API int arbor_denoiser_gradient(arbor_denoiser* d, const uint16_t* features, const float* base, const float* target, int batch, int width, int height, float* grad, size_t count, float* loss);
/* Denoised Linear (float4 per pixel, .w = 1) of one image:
 * exp(log(1 + base) + network) - 1. */
ARBOR_API int arbor_denoiser_infer(arbor_denoiser* d, const uint16_t* features, const float* base, float* denoised, int width, int height);
/* Forward convolutions on tcgen05 (1, the default) or on mma.sync (0). */
ARBOR_API int arbor_denoiser_set_backend(arbor_denoiser* d, int tcgen05);
/* Training loss in log(1 + radiance): mean absolute difference
 * (ARBOR_LOSS_L1, the default) or mean squared difference (ARBOR_LOSS_L2). */
#define ARBOR_LOSS_L1 0
#define ARBOR_LOSS_L2 1
ARBOR_API int arbor_denoiser_set_loss(arbor_denoiser* d, int kind);
/* Waits for the stream and reports ARBOR_ERR_TIMEOUT if a tensor-core
 * convolution gave up waiting for its MMAs since the last check. */
ARBOR_API int arbor_denoiser_check(arbor_denoiser* d);
ARBOR_API int arbor_denoiser_destroy(arbor_denoiser* d);
/* sum = scale * sum + x over `count` floats (progressive sample means). */
ARBOR_API int arbor_accumulate(float* sum, const float* x, size_t count, float scale, arbor_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* ARBOR_H */
