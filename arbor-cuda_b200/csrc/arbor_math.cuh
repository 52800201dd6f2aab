// arbor_math.cuh - device math shared by every Arbor kernel.
//
// Each helper restates one reference helper (Arbor.cu:17-69) with the same
// floating-point operation order.  All translation units are compiled with
// -fmad=false and IEEE division/sqrt, so + - * / sqrt match the reference's
// CPU execution bit for bit; only the transcendental functions differ.
//
// Two transcendental flavours:
//   xsin/xcos/xpow/xexp  float result of the double-precision function, i.e.
//                        correctly rounded except in astronomically rare
//                        cases.  Used where a value is computed a few times
//                        per pixel or per scene (generation, camera, instance
//                        table, sun direction, sky, tone curve), so those
//                        values agree with a correctly rounded CPU libm.
//                        The per-tree yaw sines and cosines come from the
//                        host's libm instead (WorldTrig below).
//   sinf/cosf/expf/powf/atan2f  CUDA's single-precision functions, used in
//                        the inner loops (SDF march, Newton solve, bark).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace arbor {

constexpr float kPi = 3.14159265359f;
constexpr float kFar = 100000.0f;
constexpr int kCapacity = 32768;
constexpr int kNodeCount = 65536;
constexpr int kPS = 24;
constexpr int kCS = 20;
constexpr int kCurves = 2109;
constexpr int kWood = 5124;
constexpr int kLeaf = 24192;
constexpr int kRock = 96;
constexpr int kObjects = 29412;
constexpr int kSide = 18;
constexpr int kForest = 324;
constexpr float kSpacing = 28.0f;

struct f3 {
  float x, y, z;
};
struct f2 {
  float x, y;
};

__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float b) { return {a.x * b, a.y * b, a.z * b}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, float b) { return {a.x / b, a.y / b, a.z / b}; }

__device__ __forceinline__ float clampf(float x, float a, float b) { return fminf(b, fmaxf(a, x)); }
__device__ __forceinline__ float sat(float x) { return clampf(x, 0.0f, 1.0f); }
__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + (b - a) * t; }
__device__ __forceinline__ float fracf(float a) { return a - floorf(a); }
__device__ __forceinline__ float smooth(float a, float b, float x) {
  float t = sat((x - a) / (b - a));
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross3(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ float length3(f3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ f3 norm3(f3 a) { return a / fmaxf(0.0000001f, length3(a)); }
__device__ __forceinline__ f3 min3(f3 a, f3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__device__ __forceinline__ f3 max3(f3 a, f3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__device__ __forceinline__ f3 mix3(f3 a, f3 b, float t) { return a + (b - a) * t; }
__device__ __forceinline__ f3 ld3(const float* a, int i) { return {a[i], a[i + 1], a[i + 2]}; }
__device__ __forceinline__ void st3(float* a, int i, f3 v) { a[i] = v.x; a[i + 1] = v.y; a[i + 2] = v.z; }
__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }

// Correctly rounded (to within double rounding) float transcendentals.
__device__ __forceinline__ float xsin(float x) { return (float)sin((double)x); }
__device__ __forceinline__ float xcos(float x) { return (float)cos((double)x); }
__device__ __forceinline__ float xpow(float x, float y) { return (float)pow((double)x, (double)y); }
__device__ __forceinline__ float xexp(float x) { return (float)exp((double)x); }

// Integer hash and uniforms (Arbor.cu:32-34).  Products wrap like the
// reference's int arithmetic; they are written unsigned to keep that defined.
__host__ __device__ __forceinline__ uint32_t hashU(uint32_t x) {
  x ^= x >> 16;
  x *= 2146121005u;
  x ^= x >> 15;
  x *= 2221713035u;
  x ^= x >> 16;
  return x;
}
__host__ __device__ __forceinline__ float unit24(uint32_t h) { return (float)(h & 16777215u) / 16777216.0f; }
__host__ __device__ __forceinline__ float rnd(int n, int seed) { return unit24(hashU((uint32_t)n ^ hashU((uint32_t)seed))); }
// rnd with the seed hash precomputed: rndh(n, hashU(seed)) == rnd(n, seed).
__device__ __forceinline__ float rndh(int n, uint32_t hseed) { return unit24(hashU((uint32_t)n ^ hseed)); }
__device__ __forceinline__ int hcell(int x, int y) { return (int)((uint32_t)x * 1973u + (uint32_t)y * 9277u); }
__device__ __forceinline__ float hash2(int x, int y, int seed) { return rnd(hcell(x, y), seed); }

// Value noise (Arbor.cu:35).  `hseed` = hashU(seed).
__device__ __forceinline__ float noise_h(float x, float y, uint32_t hseed) {
  int ix = (int)floorf(x);
  int iy = (int)floorf(y);
  float fx = fracf(x);
  float fy = fracf(y);
  fx = fx * fx * (3.0f - 2.0f * fx);
  fy = fy * fy * (3.0f - 2.0f * fy);
  return lerpf(lerpf(rndh(hcell(ix, iy), hseed), rndh(hcell(ix + 1, iy), hseed), fx),
               lerpf(rndh(hcell(ix, iy + 1), hseed), rndh(hcell(ix + 1, iy + 1), hseed), fx), fy);
}
__device__ __forceinline__ float noise(float x, float y, int seed) { return noise_h(x, y, hashU((uint32_t)seed)); }
// Arbor.cu:36
__device__ __forceinline__ float noise3(f3 p, int seed) {
  int iz = (int)floorf(p.z);
  float f = fracf(p.z);
  f = f * f * (3.0f - 2.0f * f);
  int s0 = (int)((uint32_t)seed + (uint32_t)iz * 131u);
  int s1 = (int)((uint32_t)seed + (uint32_t)(iz + 1) * 131u);
  return lerpf(noise(p.x, p.y, s0), noise(p.x, p.y, s1), f);
}

// Slab test (Arbor.cu:37-38).  box_span_inv takes the three invSafe values
// precomputed: the reference recomputes them per call with the same result.
__device__ __forceinline__ float inv_safe(float x) {
  return fabsf(x) < 0.00000001f ? (x < 0.0f ? -100000000.0f : 100000000.0f) : 1.0f / x;
}
__device__ __forceinline__ f3 inv3(f3 rd) { return {inv_safe(rd.x), inv_safe(rd.y), inv_safe(rd.z)}; }
__device__ __forceinline__ f2 box_span_inv(f3 ro, f3 inv, f3 lo, f3 hi) {
  f3 a = (lo - ro) * inv;
  f3 b = (hi - ro) * inv;
  f3 mn = min3(a, b);
  f3 mx = max3(a, b);
  return {fmaxf(mn.x, fmaxf(mn.y, mn.z)), fminf(mx.x, fminf(mx.y, mx.z))};
}
__device__ __forceinline__ f2 box_span(f3 ro, f3 rd, f3 lo, f3 hi) { return box_span_inv(ro, inv3(rd), lo, hi); }

// Arbor.cu:39
__device__ __forceinline__ f3 basisU(f3 n) {
  return norm3(cross3(fabsf(n.y) < 0.91f ? mk(0.0f, 1.0f, 0.0f) : mk(0.0f, 0.0f, 1.0f), n));
}
// Arbor.cu:44 - C1 footprint band weight.
__device__ __forceinline__ float band_weight(float period, float footprint) {
  return 1.0f - smooth(period * 0.12f, period * 0.65f, footprint);
}
// Arbor.cu:49
__device__ __forceinline__ uint32_t pack_rgb(f3 c) {
  uint32_t r = (uint32_t)(sat(c.x) * 255.0f + 0.5f);
  uint32_t g = (uint32_t)(sat(c.y) * 255.0f + 0.5f);
  uint32_t b = (uint32_t)(sat(c.z) * 255.0f + 0.5f);
  return r | (g << 8) | (b << 16) | 4278190080u;
}
// Arbor.cu:50
__device__ __forceinline__ float halton(int n, int base) {
  float f = 1.0f;
  float r = 0.0f;
  for (int j = 0; j < 12; j++) {
    if (n <= 0) break;
    f /= (float)base;
    r += f * (float)(n % base);
    n /= base;
  }
  return r;
}

// Forest instancing (Arbor.cu:57-66).
__host__ __device__ __forceinline__ int forest_seed(int tree, int ws) {
  return (int)(hashU((uint32_t)tree * 92821u + (uint32_t)ws * 68917u + 17u) & 1048575u);
}
__device__ __forceinline__ f3 forest_pos(int tree, int ws) {
  int x = tree % kSide - kSide / 2;
  int z = tree / kSide - kSide / 2;
  int s = forest_seed(tree, ws);
  float jx = (rnd(1, s) - 0.5f) * 10.0f;
  float jz = (rnd(2, s) - 0.5f) * 10.0f;
  float warpX = (noise((float)x * 0.19f, (float)z * 0.19f, ws + 311) - 0.5f) * 3.0f;
  float warpZ = (noise((float)x * 0.19f + 17.0f, (float)z * 0.19f - 9.0f, ws + 733) - 0.5f) * 3.0f;
  return mk((float)x * kSpacing + jx + warpX, 0.0f, (float)z * kSpacing + jz + warpZ);
}
__device__ __forceinline__ float forest_scale(int tree, int ws) { return 0.72f + rnd(3, forest_seed(tree, ws)) * 0.62f; }
__host__ __device__ __forceinline__ float forest_yaw(int tree, int ws) { return rnd(4, forest_seed(tree, ws)) * kPi * 2.0f; }

// One forest instance, precomputed per tree: every value is what the
// reference's forest helpers (Arbor.cu:57-69, 246-247, 279-282) compute on
// the fly, so using the table changes no result.
struct Instance {
  float px, pz;    // forestPos x, z (y is 0)
  float sc;        // forestScale
  float cy, rad;   // bounding sphere centre y = 4.4*sc, radius = 6.6*sc
  float lc, ls;    // cos/sin of -yaw (world -> local)
  float wc, wsn;   // cos/sin of +yaw (local normal -> world)
  float phase;     // wind phase
  int seed;        // forestSeed
  int species;     // scene of this instance in a forest of several species (0: the one resident scene)
};
__device__ __forceinline__ Instance make_instance(int tree, int ws) {
  Instance t;
  f3 p = forest_pos(tree, ws);
  t.px = p.x;
  t.pz = p.z;
  t.sc = forest_scale(tree, ws);
  t.cy = 4.4f * t.sc;
  t.rad = 6.6f * t.sc;
  float yaw = forest_yaw(tree, ws);
  float a = -yaw;
  t.lc = xcos(a);
  t.ls = xsin(a);
  t.wc = xcos(yaw);
  t.wsn = xsin(yaw);
  t.seed = forest_seed(tree, ws);
  t.phase = (float)(t.seed & 8191) * 0.0017f;
  t.species = 0;
  return t;
}
// Arbor.cu:67-69
// The per-tree yaw sines and cosines of a world seed as the reference
// harness computes them: sinf/cosf of the host's C library (Arbor.cu:67-69
// compiled for the CPU).  That library's single-precision sine and cosine are
// not correctly rounded: for about 3 % of the trees one of the four values is
// one unit in the last place away from make_instance's correctly rounded
// one, which turns the tree by that much and changes hit IDs along its
// silhouettes.  The host fills a registry slot per world seed
// (register_world_seed, camera.cu) with these values and the whole instance
// table built from them; block prologues take the values from it, and the
// persistent trace and shadow passes read the slot's table in place (global
// memory, L1/L2-resident) instead of building one in shared memory, which
// leaves their warp batches the room for deeper queues.  A seed without a
// slot keeps make_instance's values.
constexpr int kTrigSlots = 64;
struct WorldTrig {
  int ws, ready;          // world seed; 1 once the values below are in place
  int pad[2];
  float4 v[kForest];      // per tree: cos(-yaw), sin(-yaw), cos(yaw), sin(yaw)
  Instance inst[kForest]; // make_instance(t, ws, v) of every tree
};
// Host: the registry of the current device (nullptr if it cannot be
// allocated) and the registration of a world seed (a no-op for a seed already
// present, with the registry full, or while `stream` is being captured).
const WorldTrig* world_trig();
void register_world_seed(int ws, cudaStream_t stream);

// Block-wide: the registry slot of world seed ws, or nullptr.  Every thread
// of the block calls it (it synchronises the block; blockDim.x >= 64).
__device__ __forceinline__ const WorldTrig* world_slot_of(const WorldTrig* trig, int ws) {
  __shared__ int slot;
  if (threadIdx.x == 0) slot = -1;
  __syncthreads();
  if (trig != nullptr && threadIdx.x < kTrigSlots) {
    const volatile WorldTrig* s = trig + threadIdx.x;
    if (s->ready == 1 && s->ws == ws) atomicMax(&slot, (int)threadIdx.x);
  }
  __syncthreads();
  return slot >= 0 ? trig + slot : nullptr;
}
// Block-wide: the registry's sines and cosines for world seed ws, or nullptr.
__device__ __forceinline__ const float4* world_trig_of(const WorldTrig* trig, int ws) {
  const WorldTrig* s = world_slot_of(trig, ws);
  return s != nullptr ? s->v : nullptr;
}
// make_instance with the registry's sines and cosines where it has them.
__device__ __forceinline__ Instance make_instance(int tree, int ws, const float4* yaw_trig) {
  Instance t = make_instance(tree, ws);
  if (yaw_trig != nullptr) {
    const float4 q = yaw_trig[tree];
    t.lc = q.x;
    t.ls = q.y;
    t.wc = q.z;
    t.wsn = q.w;
  }
  return t;
}

__device__ __forceinline__ f3 to_local_point(f3 p, const Instance& t) {
  f3 q = mk(p.x - t.px, p.y - 0.0f, p.z - t.pz);
  return mk(q.x * t.lc - q.z * t.ls, q.y, q.x * t.ls + q.z * t.lc) / t.sc;
}
__device__ __forceinline__ f3 to_local_dir(f3 d, const Instance& t) {
  return norm3(mk(d.x * t.lc - d.z * t.ls, d.y, d.x * t.ls + d.z * t.lc));
}
__device__ __forceinline__ f3 to_world_normal(f3 n, const Instance& t) {
  return norm3(mk(n.x * t.wc - n.z * t.wsn, n.y, n.x * t.wsn + n.z * t.wc));
}

}  // namespace arbor
