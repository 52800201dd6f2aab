// build.cu - scene build: growTree, makePrimitives, makeKeys, sortPass,
// makeBounds, reduceBounds (Arbor.cu:75-142) as drop-in entries, plus the
// fused build (grow all levels in one CTA; primitives and keys in one pass;
// a stable LSD radix sort in place of 120 bitonic stages; all 15 BVH levels
// in two launches).
//
// Generation uses correctly rounded sin/cos/pow (xsin/xcos/xpow) and
// -fmad=false, so B and P agree with a correctly rounded CPU libm; keys,
// order and every node depend only on + - * / min max of P and are
// bit-identical to the reference for identical P.
#include "abi_util.h"
#include "arbor_scene.cuh"

namespace arbor {
namespace {

// ------------------------------------------------------------- growTree --
__device__ __forceinline__ f3 curve_at(const float* B, int id, float t) {
  int b = id * kCS;
  float q = 1.0f - t;
  return ld3(B, b) * (q * q * q) + ld3(B, b + 3) * (3.0f * q * q * t) + ld3(B, b + 6) * (3.0f * q * t * t) + ld3(B, b + 9) * (t * t * t);
}
__device__ __forceinline__ f3 curve_tangent(const float* B, int id, float t) {
  int b = id * kCS;
  float q = 1.0f - t;
  return norm3((ld3(B, b + 3) - ld3(B, b)) * (q * q) + (ld3(B, b + 6) - ld3(B, b + 3)) * (2.0f * q * t) + (ld3(B, b + 9) - ld3(B, b + 6)) * (t * t));
}
__device__ __forceinline__ float curve_radius(const float* B, int id, float t) { return lerpf(B[id * kCS + 12], B[id * kCS + 13], t); }
// Arbor.cu:75
__device__ __forceinline__ void store_curve(float* B, int id, f3 a, f3 b, f3 c, f3 d, float ra, float rb, float arc, int seed) {
  int o = id * kCS;
  st3(B, o, a);
  st3(B, o + 3, b);
  st3(B, o + 6, c);
  st3(B, o + 9, d);
  B[o + 12] = ra;
  B[o + 13] = rb;
  B[o + 14] = arc;
  B[o + 15] = (float)seed;
  B[o + 16] = length3(d - a);
}
// One thread of growTree (Arbor.cu:76-102).
__device__ void grow_one(float* B, int level, int seed, int i) {
  if (level == 0) {
    if (i == 0)
      store_curve(B, 0, mk(0.0f, -0.15f, 0.0f), mk(-0.22f, 1.1f, 0.16f), mk(0.23f, 2.9f, -0.19f), mk(0.04f, 4.2f, 0.05f), 0.68f, 0.23f, 0.0f, seed);
    if (i < 8) {
      float a = (float)i * kPi * 0.25f + (rnd(i, seed) - 0.5f) * 0.5f;
      f3 d = mk(xcos(a), 0.0f, xsin(a));
      float len = 2.0f + rnd(i + 10, seed) * 1.4f;
      f3 p = d * 0.32f + mk(0.0f, 0.27f, 0.0f);
      store_curve(B, i + 1, p, d * 0.8f + mk(0.0f, 0.10f, 0.0f), d * (len * 0.68f) + mk(0.0f, -0.06f, 0.0f), d * len + mk(0.0f, -0.16f, 0.0f), 0.235f,
                  0.012f, 0.0f, seed + i * 37);
    }
    return;
  }
  if (level == 1 && i < 12) {
    float t = 0.31f + 0.65f * (float)i / 11.0f;
    float a = (float)i * 2.399963f + 0.31f;
    float r = rnd(i + 37, seed);
    float len = 3.2f + 2.1f * r;
    f3 base = curve_at(B, 0, t);
    f3 d = mk(xcos(a), 0.0f, xsin(a));
    f3 side = mk(-d.z, 0.0f, d.x);
    f3 end = base + d * (len * (0.87f - 0.30f * t)) + mk(0.0f, len * (0.60f + 0.40f * t), 0.0f) + side * ((r - 0.5f) * 1.2f);
    float ra = curve_radius(B, 0, t) * (0.46f + 0.13f * r);
    store_curve(B, 9 + i, base, base + d * (len * 0.29f) + mk(0.0f, len * 0.12f, 0.0f), end - d * (len * 0.17f) - mk(0.0f, len * 0.26f, 0.0f), end, ra,
                ra * 0.14f, B[14] + t * 4.2f, seed + i * 19);
    return;
  }
  int count = level == 2 ? 72 : (level == 3 ? 288 : 1728);
  if (i >= count) return;
  int children = level == 2 ? 6 : (level == 3 ? 4 : 6);
  int offset = level == 2 ? 21 : (level == 3 ? 93 : 381);
  int parentOffset = level == 2 ? 9 : (level == 3 ? 21 : 93);
  int parent = parentOffset + i / children;
  int child = i % children;
  float h = rnd(i + level * 730, seed);
  float t = 0.23f + 0.72f * ((float)child + 0.35f) / (float)children;
  f3 p = curve_at(B, parent, t);
  f3 tangent = curve_tangent(B, parent, t);
  f3 u = basisU(tangent);
  f3 v = cross3(tangent, u);
  float angle = (float)child * 2.399963f + h * 0.8f;
  f3 lateral = u * xcos(angle) + v * xsin(angle);
  f3 d = norm3(tangent * 0.52f + lateral * (level == 4 ? 0.64f : 0.80f) + mk(0.0f, 0.26f, 0.0f));
  float len = level == 2 ? 1.65f + 1.10f * h : (level == 3 ? 0.85f + 0.65f * h : 0.43f + 0.37f * h);
  len *= 0.84f + 0.25f * (1.0f - t);
  f3 end = p + d * len + mk(0.0f, len * 0.16f, 0.0f);
  float radius = curve_radius(B, parent, t) * (level == 4 ? 0.30f : 0.40f);
  radius = fmaxf(level == 4 ? 0.0035f : 0.008f, radius);
  store_curve(B, offset + i, p, p + tangent * (len * 0.25f) + lateral * (len * 0.11f), end - d * (len * 0.28f) + mk(0.0f, len * 0.05f, 0.0f), end, radius,
              radius * (level == 4 ? 0.30f : 0.22f), B[parent * kCS + 14] + t * B[parent * kCS + 16], seed + (offset + i) * 31);
}
__host__ __device__ __forceinline__ int grow_threads(int level) {
  return level == 0 ? 9 : level == 1 ? 12 : level == 2 ? 72 : level == 3 ? 288 : 1728;
}
__global__ void grow_kernel(float* __restrict__ B, int level, int seed, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) grow_one(B, level, seed, i);
}
// All five generations in one CTA; __syncthreads orders each level after its
// parents, as the reference's separate dispatches do.
__global__ void __launch_bounds__(1024) grow_all_kernel(float* __restrict__ B, int seed) {
  for (int level = 0; level < 5; level++) {
    int n = grow_threads(level);
    for (int i = threadIdx.x; i < n; i += blockDim.x) grow_one(B, level, seed, i);
    __syncthreads();
  }
}

// ------------------------------------------------------- makePrimitives --
// One primitive record (Arbor.cu:103-131) in registers.
struct Rec {
  float v[24];
};
__device__ void prim_one(const float* B, int seed, int i, Rec& R) {
#pragma unroll
  for (int j = 0; j < 24; j++) R.v[j] = 0.0f;
  R.v[3] = -1.0f;
  if (i >= kObjects) return;
  if (i < kWood) {
    int c, segment, segments;
    if (i < 12) { c = 0; segment = i; segments = 12; }
    else if (i < 60) { c = 1 + (i - 12) / 6; segment = (i - 12) % 6; segments = 6; }
    else if (i < 156) { c = 9 + (i - 60) / 8; segment = (i - 60) % 8; segments = 8; }
    else if (i < 516) { c = 21 + (i - 156) / 5; segment = (i - 156) % 5; segments = 5; }
    else if (i < 1668) { c = 93 + (i - 516) / 4; segment = (i - 516) % 4; segments = 4; }
    else { c = 381 + (i - 1668) / 2; segment = (i - 1668) % 2; segments = 2; }
    float t0 = (float)segment / (float)segments;
    float t1 = (float)(segment + 1) / (float)segments;
    f3 a = curve_at(B, c, t0), e = curve_at(B, c, t1);
    R.v[0] = a.x; R.v[1] = a.y; R.v[2] = a.z; R.v[3] = 0.0f;
    R.v[4] = e.x; R.v[5] = e.y; R.v[6] = e.z;
    R.v[7] = curve_radius(B, c, t0);
    R.v[11] = curve_radius(B, c, t1);
    R.v[15] = B[c * kCS + 15];
    float arclength = B[c * kCS + 14];
    for (int j = 0; j < 12; j++)
      if (j < segment) arclength += length3(curve_at(B, c, (float)(j + 1) / (float)segments) - curve_at(B, c, (float)j / (float)segments));
    R.v[16] = arclength;
    R.v[17] = (float)c;
    R.v[18] = B[c * kCS + 12];
    f3 bu = basisU(curve_tangent(B, c, 0.0f));
    R.v[8] = bu.x; R.v[9] = bu.y; R.v[10] = bu.z;
    return;
  }
  if (i < kWood + kLeaf) {
    int leaf = i - kWood;
    int twig = leaf / 14;
    int k = leaf % 14;
    int c = 381 + twig;
    float h = rnd(leaf + 13, seed);
    float t = 0.16f + 0.81f * ((float)k + 0.4f) / 14.0f;
    f3 anchor = curve_at(B, c, t);
    f3 axis = curve_tangent(B, c, t);
    f3 bu = basisU(axis);
    f3 bv = cross3(axis, bu);
    float angle = (float)k * 2.399963f + rnd(twig, seed) * 6.28f;
    f3 out = norm3(bu * xcos(angle) + bv * xsin(angle));
    f3 u = norm3(out * 0.82f + axis * 0.35f + mk(0.0f, 0.20f, 0.0f));
    f3 normal = norm3(mk(0.0f, 1.0f, 0.0f) + out * (0.20f + h * 0.38f));
    f3 v = norm3(cross3(normal, u));
    normal = norm3(cross3(u, v));
    R.v[0] = anchor.x; R.v[1] = anchor.y; R.v[2] = anchor.z; R.v[3] = 1.0f;
    R.v[4] = u.x; R.v[5] = u.y; R.v[6] = u.z;
    R.v[7] = 0.145f + 0.075f * h;
    R.v[8] = v.x; R.v[9] = v.y; R.v[10] = v.z;
    R.v[11] = R.v[7] * (0.34f + 0.07f * rnd(leaf + 37, seed));
    R.v[12] = normal.x; R.v[13] = normal.y; R.v[14] = normal.z;
    R.v[15] = (float)(leaf + seed * 11);
    R.v[16] = 0.023f + 0.024f * rnd(leaf + 149, seed);
    R.v[17] = 0.013f + 0.016f * h;
    R.v[18] = (rnd(leaf + 777, seed) - 0.5f) * 0.10f;
    R.v[19] = (float)twig;
    return;
  }
  int rock = i - kWood - kLeaf;
  float a = rnd(rock * 3 + 1, seed) * 6.2831853f;
  float r = 0.8f + 4.5f * sqrtf(rnd(rock * 3 + 2, seed));
  float size = 0.045f + 0.19f * xpow(rnd(rock + 371, seed), 3.0f);
  R.v[0] = xcos(a) * r; R.v[1] = size * 0.30f - 0.015f; R.v[2] = xsin(a) * r; R.v[3] = 2.0f;
  R.v[4] = size; R.v[5] = size * 0.55f; R.v[6] = size * (0.7f + rnd(rock + 16, seed) * 0.5f);
  R.v[15] = (float)(rock + seed);
}
__device__ __forceinline__ void store_rec(float* P, int i, const Rec& R) {
  float4* d = reinterpret_cast<float4*>(P) + i * 6;
#pragma unroll
  for (int k = 0; k < 6; k++) d[k] = make_float4(R.v[4 * k], R.v[4 * k + 1], R.v[4 * k + 2], R.v[4 * k + 3]);
}
// Arbor.cu:138
__device__ __forceinline__ uint32_t spread10(uint32_t x) {
  x &= 1023u;
  x = (x | (x << 16)) & 50331903u;
  x = (x | (x << 8)) & 50393103u;
  x = (x | (x << 4)) & 51130563u;
  x = (x | (x << 2)) & 153391689u;
  return x;
}
// Morton key of one record (Arbor.cu:139).
__device__ __forceinline__ uint32_t morton_key(float4 r0, float4 r1, float p7, float p11, float p16) {
  if (r0.w < 0.0f) return 4294967295u;
  f3 lo, hi;
  prim_bounds(r0, r1, p7, p11, p16, lo, hi);
  f3 p = (lo + hi) * 0.5f;
  uint32_t x = (uint32_t)(sat((p.x + 12.0f) / 24.0f) * 1023.0f);
  uint32_t y = (uint32_t)(sat((p.y + 1.0f) / 18.0f) * 1023.0f);
  uint32_t z = (uint32_t)(sat((p.z + 12.0f) / 24.0f) * 1023.0f);
  return spread10(x) | (spread10(y) << 1) | (spread10(z) << 2);
}
__global__ void __launch_bounds__(128) prims_kernel(const float* __restrict__ B, float* __restrict__ P, int seed) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCapacity) return;
  Rec R;
  prim_one(B, seed, i, R);
  store_rec(P, i, R);
}
__global__ void __launch_bounds__(128) keys_kernel(const float* __restrict__ P, uint32_t* __restrict__ Keys, uint32_t* __restrict__ Order) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCapacity) return;
  Order[i] = (uint32_t)i;
  float4 r0 = ldg4(P, i * 6), r1 = ldg4(P, i * 6 + 1), r2 = ldg4(P, i * 6 + 2), r4 = ldg4(P, i * 6 + 4);
  Keys[i] = morton_key(r0, r1, r1.w, r2.w, r4.x);
}
// makePrimitives and makeKeys fused: the key is computed from the record
// still in registers (the same float values the reference reads back).
__global__ void __launch_bounds__(128) prims_keys_kernel(const float* __restrict__ B, float* __restrict__ P, uint32_t* __restrict__ Keys,
                                                         uint32_t* __restrict__ Order, int seed) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCapacity) return;
  Rec R;
  prim_one(B, seed, i, R);
  store_rec(P, i, R);
  Order[i] = (uint32_t)i;
  Keys[i] = morton_key(make_float4(R.v[0], R.v[1], R.v[2], R.v[3]), make_float4(R.v[4], R.v[5], R.v[6], R.v[7]), R.v[7], R.v[11], R.v[16]);
}

// ------------------------------------------------------------- sortPass --
// One bitonic stage (Arbor.cu:140).
__global__ void __launch_bounds__(128) sort_pass_kernel(uint32_t* __restrict__ Keys, uint32_t* __restrict__ Order, int distance, int span) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCapacity) return;
  int j = i ^ distance;
  if (j <= i) return;
  uint32_t a = Keys[i], b = Keys[j], ia = Order[i], ib = Order[j];
  bool greater = a > b || (a == b && ia > ib);
  bool ascending = (i & span) == 0;
  if (greater == ascending) {
    Keys[i] = b;
    Keys[j] = a;
    Order[i] = ib;
    Order[j] = ia;
  }
}

// ----------------------------------------------------------- radix sort --
// Stable LSD radix sort of 32768 (key, value) pairs, 8 bits per pass, one
// launch per pass.  Each of the 16 CTAs ranks 2048 consecutive elements; it
// obtains the global digit offsets by counting all 32768 digits itself (a
// 128 KB L2-resident read), so no inter-CTA synchronisation is needed.
// Ranks within a CTA are stable: warps own consecutive 32-element groups,
// lanes rank among equal digits with __match_any_sync.
constexpr int kSortCtas = 16;
constexpr int kSortThreads = 1024;
constexpr int kSortPerCta = kCapacity / kSortCtas;  // 2048

__global__ void __launch_bounds__(kSortThreads) radix_pass_kernel(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                                  uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int shift) {
  __shared__ uint32_t before[256];
  __shared__ uint32_t total[256];
  __shared__ uint32_t base[256];
  __shared__ uint32_t wcnt[kSortThreads / 32][256];
  const int tid = threadIdx.x;
  const int start = blockIdx.x * kSortPerCta;
  if (tid < 256) {
    before[tid] = 0;
    total[tid] = 0;
  }
  __syncthreads();
  for (int e = tid; e < kCapacity; e += kSortThreads) {
    uint32_t d = (__ldg(kin + e) >> shift) & 255u;
    atomicAdd(&total[d], 1u);
    if (e < start) atomicAdd(&before[d], 1u);
  }
  __syncthreads();
  // Exclusive scan of the digit totals (one warp, 8 digits per lane).
  if (tid < 32) {
    uint32_t local[8], s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      local[k] = s;
      s += total[tid * 8 + k];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t n = __shfl_up_sync(0xffffffffu, incl, o);
      if (tid >= o) incl += n;
    }
    uint32_t excl = incl - s;
#pragma unroll
    for (int k = 0; k < 8; k++) base[tid * 8 + k] = excl + local[k] + before[tid * 8 + k];
  }
  const int warp = tid >> 5, lane = tid & 31;
  const uint32_t lt = (1u << lane) - 1u;
  for (int round = 0; round < kSortPerCta / kSortThreads; round++) {
    for (int k = tid; k < (kSortThreads / 32) * 256; k += kSortThreads) (&wcnt[0][0])[k] = 0;
    __syncthreads();
    int e = start + round * kSortThreads + tid;
    uint32_t key = __ldg(kin + e), val = __ldg(vin + e);
    uint32_t d = (key >> shift) & 255u;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t rank = __popc(peers & lt);
    if (rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (tid < 256) {
      uint32_t run = base[tid];
      for (int w = 0; w < kSortThreads / 32; w++) {
        uint32_t c = wcnt[w][tid];
        wcnt[w][tid] = run;
        run += c;
      }
      base[tid] = run;
    }
    __syncthreads();
    uint32_t pos = wcnt[warp][d] + rank;
    kout[pos] = key;
    vout[pos] = val;
    __syncthreads();
  }
}

// ---------------------------------------------------- makeBounds / reduce --
// Leaf record of one Order slot (Arbor.cu:141): {boundLow, active, boundHigh,
// id}.  An id outside the 32768 records (invalid input) is given the bounds
// of an unused record instead of reading out of bounds.
__device__ __forceinline__ void leaf_record(const float* P, uint32_t uid, float4& lo4, float4& hi4) {
  if (uid >= (uint32_t)kCapacity) {
    lo4 = make_float4(kFar, kFar, kFar, 0.0f);
    hi4 = make_float4(-kFar, -kFar, -kFar, (float)(int)uid);
    return;
  }
  int id = (int)uid;
  float4 r0 = ldg4(P, id * 6), r1 = ldg4(P, id * 6 + 1), r2 = ldg4(P, id * 6 + 2), r4 = ldg4(P, id * 6 + 4);
  f3 lo, hi;
  prim_bounds(r0, r1, r1.w, r2.w, r4.x, lo, hi);
  lo4 = make_float4(lo.x, lo.y, lo.z, r0.w >= 0.0f ? 1.0f : 0.0f);
  hi4 = make_float4(hi.x, hi.y, hi.z, (float)id);
}
__global__ void __launch_bounds__(128) bounds_kernel(const float* __restrict__ P, const uint32_t* __restrict__ Order, float* __restrict__ Nodes) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCapacity) return;
  float4 lo, hi;
  leaf_record(P, __ldg(Order + i), lo, hi);
  float4* n = reinterpret_cast<float4*>(Nodes) + (kCapacity + i) * 2;
  n[0] = lo;
  n[1] = hi;
}
// Parent = union of the two children (Arbor.cu:142).
__device__ __forceinline__ void merge(float4 alo, float4 ahi, float4 clo, float4 chi, float4& plo, float4& phi) {
  plo = make_float4(fminf(alo.x, clo.x), fminf(alo.y, clo.y), fminf(alo.z, clo.z), alo.w + clo.w);
  phi = make_float4(fmaxf(ahi.x, chi.x), fmaxf(ahi.y, chi.y), fmaxf(ahi.z, chi.z), -1.0f);
}
__global__ void __launch_bounds__(128) reduce_kernel(float* __restrict__ Nodes, int first) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= first) return;
  int node = first + i;
  float4* n = reinterpret_cast<float4*>(Nodes);
  float4 plo, phi;
  merge(n[node * 4], n[node * 4 + 1], n[node * 4 + 2], n[node * 4 + 3], plo, phi);
  n[node * 2] = plo;
  n[node * 2 + 1] = phi;
}
// Leaves and the ten levels above them: CTA k owns leaves 1024k..1024k+1023
// and reduces them in shared memory down to its subtree root, node 32+k.
constexpr int kLeavesPerCta = 1024;
__global__ void __launch_bounds__(kLeavesPerCta) subtree_kernel(const float* __restrict__ P, const uint32_t* __restrict__ Order,
                                                                float* __restrict__ Nodes) {
  __shared__ float4 slo[kLeavesPerCta], shi[kLeavesPerCta];
  const int tid = threadIdx.x;
  const int leaf = blockIdx.x * kLeavesPerCta + tid;
  float4* n = reinterpret_cast<float4*>(Nodes);
  float4 lo, hi;
  leaf_record(P, __ldg(Order + leaf), lo, hi);
  n[(kCapacity + leaf) * 2] = lo;
  n[(kCapacity + leaf) * 2 + 1] = hi;
  slo[tid] = lo;
  shi[tid] = hi;
  __syncthreads();
  int width = kLeavesPerCta / 2;
  int levelFirst = kCapacity / 2;  // heap index of the first node of this level
  while (width >= 1) {
    float4 plo, phi;
    if (tid < width) merge(slo[2 * tid], shi[2 * tid], slo[2 * tid + 1], shi[2 * tid + 1], plo, phi);
    __syncthreads();
    if (tid < width) {
      slo[tid] = plo;
      shi[tid] = phi;
      int node = levelFirst + blockIdx.x * width + tid;
      n[node * 2] = plo;
      n[node * 2 + 1] = phi;
    }
    __syncthreads();
    width >>= 1;
    levelFirst >>= 1;
  }
}
// The top five levels: nodes 1..31 from the 32 subtree roots.
__global__ void __launch_bounds__(32) top_kernel(float* __restrict__ Nodes) {
  float4* n = reinterpret_cast<float4*>(Nodes);
  for (int first = 16; first >= 1; first >>= 1) {
    int i = threadIdx.x;
    if (i < first) {
      int node = first + i;
      float4 plo, phi;
      merge(n[node * 4], n[node * 4 + 1], n[node * 4 + 2], n[node * 4 + 3], plo, phi);
      n[node * 2] = plo;
      n[node * 2 + 1] = phi;
    }
    __syncwarp();
    __threadfence_block();
  }
}

int grid_of(int n, int block) { return (n + block - 1) / block; }

}  // namespace

// Host helpers reused by the engine and the fused build.
int launch_sort(uint32_t* Keys, uint32_t* Order, void* scratch, cudaStream_t stream) {
  uint32_t* k2 = static_cast<uint32_t*>(scratch);
  uint32_t* v2 = k2 + kCapacity;
  for (int pass = 0; pass < 4; pass++) {
    bool even = (pass & 1) == 0;
    radix_pass_kernel<<<kSortCtas, kSortThreads, 0, stream>>>(even ? Keys : k2, even ? Order : v2, even ? k2 : Keys, even ? v2 : Order, pass * 8);
  }
  count_launch(4);
  return check_launch("arbor_sortKeys");
}
int launch_bounds_build(const float* P, const uint32_t* Order, float* Nodes, cudaStream_t stream) {
  subtree_kernel<<<kCapacity / kLeavesPerCta, kLeavesPerCta, 0, stream>>>(P, Order, Nodes);
  top_kernel<<<1, 32, 0, stream>>>(Nodes);
  count_launch(2);
  return check_launch("arbor_buildBounds");
}
int launch_grow_all(float* B, int seed, cudaStream_t stream) {
  grow_all_kernel<<<1, 1024, 0, stream>>>(B, seed);
  count_launch();
  return check_launch("grow");
}
int launch_prims_keys(const float* B, float* P, uint32_t* Keys, uint32_t* Order, int seed, cudaStream_t stream) {
  prims_keys_kernel<<<grid_of(kCapacity, 128), 128, 0, stream>>>(B, P, Keys, Order, seed);
  count_launch();
  return check_launch("primitives");
}

}  // namespace arbor

using namespace arbor;

extern "C" int arbor_growTree(float* B, int level, int seed, arbor_stream stream) {
  const Binding b[] = {{B, kB, true, 4, "B"}};
  if (int s = check_bindings("arbor_growTree", b)) return s;
  int n = grow_threads(level);
  grow_kernel<<<grid_of(n, 64), 64, 0, stream>>>(B, level, seed, n);
  count_launch();
  return check_launch("arbor_growTree");
}
extern "C" int arbor_makePrimitives(const float* B, float* P, int seed, arbor_stream stream) {
  const Binding b[] = {{B, kB, false, 4, "B"}, {P, kP, true, 16, "P"}};
  if (int s = check_bindings("arbor_makePrimitives", b)) return s;
  prims_kernel<<<grid_of(kCapacity, 128), 128, 0, stream>>>(B, P, seed);
  count_launch();
  return check_launch("arbor_makePrimitives");
}
extern "C" int arbor_makeKeys(const float* P, uint32_t* Keys, uint32_t* Order, arbor_stream stream) {
  const Binding b[] = {{P, kP, false, 16, "P"}, {Keys, kKeys, true, 4, "Keys"}, {Order, kKeys, true, 4, "Order"}};
  if (int s = check_bindings("arbor_makeKeys", b)) return s;
  keys_kernel<<<grid_of(kCapacity, 128), 128, 0, stream>>>(P, Keys, Order);
  count_launch();
  return check_launch("arbor_makeKeys");
}
extern "C" int arbor_sortPass(uint32_t* Keys, uint32_t* Order, int distance, int span, arbor_stream stream) {
  const Binding b[] = {{Keys, kKeys, true, 4, "Keys"}, {Order, kKeys, true, 4, "Order"}};
  if (int s = check_bindings("arbor_sortPass", b)) return s;
  if (distance < 0 || distance >= kCapacity) {
    set_error("arbor_sortPass: distance %d outside 0..%d indexes past the records", distance, kCapacity - 1);
    return ARBOR_ERR_VALUE;
  }
  sort_pass_kernel<<<grid_of(kCapacity, 128), 128, 0, stream>>>(Keys, Order, distance, span);
  count_launch();
  return check_launch("arbor_sortPass");
}
extern "C" int arbor_makeBounds(const float* P, const uint32_t* Order, float* Nodes, arbor_stream stream) {
  const Binding b[] = {{P, kP, false, 16, "P"}, {Order, kKeys, false, 4, "Order"}, {Nodes, kNodes, true, 16, "Nodes"}};
  if (int s = check_bindings("arbor_makeBounds", b)) return s;
  bounds_kernel<<<grid_of(kCapacity, 128), 128, 0, stream>>>(P, Order, Nodes);
  count_launch();
  return check_launch("arbor_makeBounds");
}
extern "C" int arbor_reduceBounds(float* Nodes, int first, arbor_stream stream) {
  const Binding b[] = {{Nodes, kNodes, true, 16, "Nodes"}};
  if (int s = check_bindings("arbor_reduceBounds", b)) return s;
  if (first < 0 || first > kCapacity / 2) {
    set_error("arbor_reduceBounds: first %d outside 0..%d indexes past the node records", first, kCapacity / 2);
    return ARBOR_ERR_VALUE;
  }
  if (first == 0) return ARBOR_OK;
  reduce_kernel<<<grid_of(first, 128), 128, 0, stream>>>(Nodes, first);
  count_launch();
  return check_launch("arbor_reduceBounds");
}
extern "C" size_t arbor_sort_scratch_bytes(void) { return 2u * kCapacity * sizeof(uint32_t); }
extern "C" int arbor_sortKeys(uint32_t* Keys, uint32_t* Order, void* scratch, arbor_stream stream) {
  const Binding b[] = {{Keys, kKeys, true, 4, "Keys"}, {Order, kKeys, true, 4, "Order"}, {scratch, arbor_sort_scratch_bytes(), true, 4, "scratch"}};
  if (int s = check_bindings("arbor_sortKeys", b)) return s;
  return launch_sort(Keys, Order, scratch, stream);
}
extern "C" int arbor_buildBounds(const float* P, const uint32_t* Order, float* Nodes, arbor_stream stream) {
  const Binding b[] = {{P, kP, false, 16, "P"}, {Order, kKeys, false, 4, "Order"}, {Nodes, kNodes, true, 16, "Nodes"}};
  if (int s = check_bindings("arbor_buildBounds", b)) return s;
  return launch_bounds_build(P, Order, Nodes, stream);
}
extern "C" int arbor_initCamera(float* C, const float* P, int seed, arbor_stream stream);
extern "C" int arbor_buildScene(int seed, float* B, float* P, uint32_t* Keys, uint32_t* Order, float* Nodes, float* C, void* scratch,
                                arbor_stream stream) {
  const Binding b[] = {{B, kB, true, 4, "B"},
                       {P, kP, true, 16, "P"},
                       {Keys, kKeys, true, 4, "Keys"},
                       {Order, kKeys, true, 4, "Order"},
                       {Nodes, kNodes, true, 16, "Nodes"},
                       {scratch, arbor_sort_scratch_bytes(), true, 4, "scratch"}};
  if (int s = check_bindings("arbor_buildScene", b)) return s;
  if (C != nullptr) {
    const Binding c[] = {{C, kC, true, 4, "C"}, {B, kB, true, 4, "B"}, {P, kP, true, 16, "P"}, {Nodes, kNodes, true, 16, "Nodes"},
                         {Keys, kKeys, true, 4, "Keys"}, {Order, kKeys, true, 4, "Order"}, {scratch, arbor_sort_scratch_bytes(), true, 4, "scratch"}};
    if (int s = check_bindings("arbor_buildScene", c)) return s;
  }
  register_world_seed(seed, stream);  // a forest built from `seed` has world seed `seed` (initCamera sets C[31])
  if (int s = launch_grow_all(B, seed, stream)) return s;
  if (int s = launch_prims_keys(B, P, Keys, Order, seed, stream)) return s;
  if (int s = launch_sort(Keys, Order, scratch, stream)) return s;
  if (int s = launch_bounds_build(P, Order, Nodes, stream)) return s;
  if (C != nullptr) return arbor_initCamera(C, P, seed, stream);
  return ARBOR_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free sort.
//
// Some callers cannot allocate device memory: a host that, like the
// reference's engine (src/engine.js:22,40), owns every buffer and binds only
// the ABI records to the kernels has no scratch buffer to hand to
// arbor_sortKeys, and a frame loop running under a fixed memory budget may
// not call cudaMalloc at all.  arbor_sortKeysNoAlloc sorts the same way as
// arbor_sortKeys but takes its ping-pong buffer from the file-scope array
// below, so it allocates nothing.  The array is part of the library image:
// every GPU that loads the library holds its 256 KB until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace arbor {
namespace {

constexpr int kNoAllocMaxPairs = kCapacity;  // largest count the array holds
static __device__ __align__(256) uint32_t g_noalloc_sort_scratch[2 * kNoAllocMaxPairs];

// One 8-bit LSD pass over the first n pairs (n <= kNoAllocMaxPairs), the
// same stable ranking as radix_pass_kernel with the tail beyond n masked.
__global__ void __launch_bounds__(kSortThreads) radix_pass_n_kernel(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                                    uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int shift, int n) {
  __shared__ uint32_t before[256];
  __shared__ uint32_t total[256];
  __shared__ uint32_t base[256];
  __shared__ uint32_t wcnt[kSortThreads / 32][256];
  const int tid = threadIdx.x;
  const int start = blockIdx.x * kSortPerCta;
  if (tid < 256) {
    before[tid] = 0;
    total[tid] = 0;
  }
  __syncthreads();
  for (int e = tid; e < n; e += kSortThreads) {
    uint32_t d = (__ldg(kin + e) >> shift) & 255u;
    atomicAdd(&total[d], 1u);
    if (e < start) atomicAdd(&before[d], 1u);
  }
  __syncthreads();
  if (tid < 32) {
    uint32_t local[8], s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      local[k] = s;
      s += total[tid * 8 + k];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (tid >= o) incl += v;
    }
    uint32_t excl = incl - s;
#pragma unroll
    for (int k = 0; k < 8; k++) base[tid * 8 + k] = excl + local[k] + before[tid * 8 + k];
  }
  const int warp = tid >> 5, lane = tid & 31;
  const uint32_t lt = (1u << lane) - 1u;
  for (int round = 0; round < kSortPerCta / kSortThreads; round++) {
    for (int k = tid; k < (kSortThreads / 32) * 256; k += kSortThreads) (&wcnt[0][0])[k] = 0;
    __syncthreads();
    int e = start + round * kSortThreads + tid;
    bool live = e < n;
    uint32_t key = live ? __ldg(kin + e) : 0u, val = live ? __ldg(vin + e) : 0u;
    uint32_t d = live ? ((key >> shift) & 255u) : 256u;  // 256 marks the masked tail
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t rank = __popc(peers & lt);
    if (live && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (tid < 256) {
      uint32_t run = base[tid];
      for (int w = 0; w < kSortThreads / 32; w++) {
        uint32_t c = wcnt[w][tid];
        wcnt[w][tid] = run;
        run += c;
      }
      base[tid] = run;
    }
    __syncthreads();
    if (live) {
      uint32_t pos = wcnt[warp][d] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
  }
}

// Device address of the scratch array on each device.  A call outside stream
// capture looks it up again (a device reset reloads the library's module,
// and the array may then sit elsewhere); a call during capture uses the
// address its device's last call outside capture found.
std::mutex g_noalloc_mutex;
uint32_t* g_noalloc_ptr[64] = {};

int noalloc_scratch(cudaStream_t stream, uint32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("arbor_sortKeysNoAlloc: cudaGetDevice failed: %s", cudaGetErrorString(e));
    return ARBOR_ERR_CUDA;
  }
  if (dev < 0 || dev >= 64) {
    set_error("arbor_sortKeysNoAlloc: device %d is beyond the 64 devices this library tracks", dev);
    return ARBOR_ERR_LIMIT;
  }
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess) {
    (void)cudaGetLastError();  // the query's own error; treat the stream as capturing
    capture = cudaStreamCaptureStatusActive;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_ptr[dev] == nullptr || capture == cudaStreamCaptureStatusNone) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_sort_scratch);
    if (e != cudaSuccess || ptr == nullptr) {
      set_error("arbor_sortKeysNoAlloc: cudaGetSymbolAddress of the scratch array failed: %s", cudaGetErrorString(e));
      return ARBOR_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = static_cast<uint32_t*>(ptr);
  }
  *out = g_noalloc_ptr[dev];
  return ARBOR_OK;
}

}  // namespace
}  // namespace arbor

extern "C" int arbor_sortKeysNoAlloc(uint32_t* Keys, uint32_t* Order, int count, arbor_stream stream) {
  const char* name = "arbor_sortKeysNoAlloc";
  if (count < 0) {
    set_error("%s: count %d is negative", name, count);
    return ARBOR_ERR_VALUE;
  }
  if (count > kNoAllocMaxPairs) {
    set_error("%s: count %d exceeds the %d pairs its fixed scratch array holds", name, count, kNoAllocMaxPairs);
    return ARBOR_ERR_LIMIT;
  }
  const Binding b[] = {{Keys, (size_t)count * 4u, true, 4, "Keys"}, {Order, (size_t)count * 4u, true, 4, "Order"}};
  if (int s = check_bindings(name, b)) return s;
  if (count == 0) return ARBOR_OK;
  uint32_t* scratch = nullptr;
  if (int s = noalloc_scratch(stream, &scratch)) return s;
  uint32_t* k2 = scratch;
  uint32_t* v2 = scratch + kNoAllocMaxPairs;
  int ctas = (count + kSortPerCta - 1) / kSortPerCta;
  for (int pass = 0; pass < 4; pass++) {
    bool even = (pass & 1) == 0;
    radix_pass_n_kernel<<<ctas, kSortThreads, 0, stream>>>(even ? Keys : k2, even ? Order : v2, even ? k2 : Keys, even ? v2 : Order, pass * 8,
                                                           count);
  }
  count_launch(4);
  return check_launch(name);
}
