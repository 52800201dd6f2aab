// TEST INFRASTRUCTURE ONLY - exports the reference's own CPU execution of the
// Arbor kernels under the same oracle_* names as oracle/arbor_oracle.c.
//
// Built by oracle/Makefile into oracle/_ref/libarbor_ref.so straight from the
// reference's sources: this file includes tests/native_harness.cpp (which
// includes ../Arbor.cu with the harness's host shim, native_harness.cpp:15-33)
// with its main() renamed.  Nothing of the reference is copied here; the
// kernels run exactly as the harness runs them, one simulated thread at a
// time, with the harness's OpenMP row schedule (native_harness.cpp:36-39).
//
// The one composition that the reference lacks, the single-tree scene (one
// resident tree with an identity instance), is built here from the
// reference's own traceTree/objectNormal/surfaceColor/... exactly as the
// forest passes use them (Arbor.cu:252, 277-289).
#define main arbor_harness_main
#include "native_harness.cpp"
#undef main

#include <omp.h>

#define EXPORT extern "C" __attribute__((visibility("default")))

namespace {
template <class F> void each_thread(int n, int block, F f) {
  for (int i = 0; i < n; i++) {
    blockDim = {unsigned(block), 1, 1};
    blockIdx = {unsigned(i / block), 0, 0};
    threadIdx = {unsigned(i % block), 0, 0};
    f();
  }
}
template <class F> void each_pixel(int w, int y0, int y1, F f) {
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < w; x++) {
      blockDim = {8, 8, 1};
      blockIdx = {unsigned(x / 8), unsigned(y / 8), 0};
      threadIdx = {unsigned(x % 8), unsigned(y % 8), 0};
      f();
    }
}

// Single-tree primary hit: tracePixels (Arbor.cu:252) with traceTree in
// place of traceForest.
void trace_single(const float* P, const float* Nodes, const unsigned* Order, const float* C, float* Hit, int w, int h, int x, int y) {
  int b = (y * w + x) * 4;
  float3 ro = cameraPos(C);
  float3 rd = cameraRay(C, x, y, w, h);
  float ground = rd.y < -0.00001f ? -ro.y / rd.y : FAR;
  float2 r = traceTree(P, Nodes, Order, ro, rd, C[14] / (float)h, C[8], C[11], ground > 0.0f ? ground : FAR, -1, false);
  Hit[b] = r.x; Hit[b + 1] = r.y; Hit[b + 2] = -1.0f; Hit[b + 3] = C[14] * r.x / (float)h;
}
float3 visibility_single(const float* P, const float* Nodes, const unsigned* Order, float3 p, float3 direction, float time, float wind) {
  float3 transmission = make_float3(1.0f, 1.0f, 1.0f);
  float3 ro = p;
  for (int j = 0; j < 4; j++) {
    float2 h = traceTree(P, Nodes, Order, ro, direction, 0.0001f, time, wind, 36.0f, -1, true);
    int id = (int)h.y;
    if (id < 0) break;
    if (P[id * PS + 3] != 1.0f) return make_float3(0.0f, 0.0f, 0.0f);
    transmission = transmission * make_float3(0.18f, 0.29f, 0.065f);
    ro = ro + direction * (h.x + 0.0018f);
  }
  return transmission;
}
// Single-tree shading: shadePixels (Arbor.cu:277-289) with the identity
// instance (local point = world point, no per-tree tint, phase 0).
void shade_single(const float* P, const float* Nodes, const unsigned* Order, const float* C, const float* Hit, float* Linear, float* Guide, int width, int height, int x, int y) {
  int pixel = y * width + x; int b = pixel * 4;
  float t = Hit[b]; int id = (int)Hit[b + 1];
  float3 ro = cameraPos(C); float3 rd = cameraRay(C, x, y, width, height); float3 sun = sunC(C);
  float3 col = sky(rd, sun); float3 guide = make_float3(1.0f, 1.0f, 1.0f);
  if (t < FAR) {
    float3 p = ro + rd * t; float fp = fmaxf(0.000005f, Hit[b + 3]);
    float3 n = make_float3(0.0f, 1.0f, 0.0f);
    if (id >= 0) n = objectNormal(P, id, p, fp, C[8], C[11]);
    bool leaf = id >= 0 && P[id * PS + 3] == 1.0f;
    if (dot3(n, rd) > 0.0f) n = n * -1.0f;
    if (id < 0) {
      float e = fmaxf(0.001f, fp);
      float nx = (noise((p.x + e) * 18.0f, p.z * 18.0f, 133) - noise((p.x - e) * 18.0f, p.z * 18.0f, 133)) * 0.18f;
      float nz = (noise(p.x * 18.0f, (p.z + e) * 18.0f, 133) - noise(p.x * 18.0f, (p.z - e) * 18.0f, 133)) * 0.18f;
      n = norm3(make_float3(nx, 1.0f, nz));
    }
    float3 albedo = surfaceColor(P, id, p, fp, C[8], C[11]);
    guide = albedo;
    int sample = (int)C[9];
    float r1 = rnd(pixel + sample * 1823, 991); float r2 = rnd(pixel + sample * 971, 731);
    float3 su = basisU(sun); float3 sv = cross3(sun, su);
    float angle = r1 * 6.28318f; float disk = sqrtf(r2) * 0.012f;
    float3 light = norm3(sun + su * (cosf(angle) * disk) + sv * (sinf(angle) * disk));
    float offset = id >= 0 ? 0.0014f : 0.004f;
    float3 visibility = make_float3(1.0f, 1.0f, 1.0f);
    if (C[22] > 0.5f) visibility = visibility_single(P, Nodes, Order, p + light * offset, light, C[8], C[11]);
    float nl = sat(dot3(n, light)); float back = sat(-dot3(n, light));
    float3 direct = albedo * (nl / PI);
    if (leaf) { float vein = leafVein(P, id, p, fp, C[8], C[11]); direct = direct + albedo * (back * (0.75f - 0.25f * vein) + powf(sat(dot3(rd, light)), 9.0f) * 0.12f); }
    float spec = specGGX(n, rd * -1.0f, light, leaf ? 0.39f : 0.82f);
    direct = direct + make_float3(spec, spec, spec);
    float ao = 1.0f;
    float3 ambient = make_float3(0.30f, 0.37f, 0.45f) * (0.45f + 0.55f * sat(n.y)) * ao + make_float3(0.08f, 0.068f, 0.035f) * sat(-n.y);
    if (leaf) ambient = ambient + make_float3(0.04f, 0.055f, 0.022f) * ao;
    col = direct * visibility * make_float3(4.8f, 4.2f, 3.1f) + albedo * ambient;
    float haze = 1.0f - expf(-t * 0.0018f);
    col = mix3(col, sky(rd, sun), haze);
    if (C[15] == 1.0f) { float w0 = bandWeight(0.065f, fp); float w1 = bandWeight(0.005f, fp); float w2 = bandWeight(0.001f, fp); col = make_float3(w0 * 0.80f, w1 * 0.85f, w2 * 0.9f); }
    if (C[15] == 2.0f) { float hh = rnd(id + 177 + (-1 + 1) * 71, 32); col = id < 0 ? make_float3(0.10f, 0.10f, 0.10f) : (leaf ? make_float3(0.1f, 0.3f + hh * 0.5f, 0.17f) : make_float3(0.47f + hh * 0.3f, 0.25f, 0.10f)); }
    if (C[15] == 3.0f) col = n * 0.5f + make_float3(0.5f, 0.5f, 0.5f);
  }
  write3(Linear, b, col); Linear[b + 3] = 1.0f; write3(Guide, b, guide); Guide[b + 3] = 1.0f;
}
}  // namespace

EXPORT int oracle_is_f64() { return 0; }
EXPORT void oracle_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
EXPORT int oracle_max_threads() { return omp_get_max_threads(); }
EXPORT void oracle_growTree(float* B, int level, int seed) {
  int n = level == 0 ? 9 : level == 1 ? 12 : level == 2 ? 72 : level == 3 ? 288 : 1728;
  each_thread(n, 128, [&] { growTree(B, level, seed); });
}
EXPORT void oracle_makePrimitives(const float* B, float* P, int seed) { each_thread(CAPACITY, 128, [&] { makePrimitives(B, P, seed); }); }
EXPORT void oracle_makeKeys(const float* P, unsigned* Keys, unsigned* Order) { each_thread(CAPACITY, 128, [&] { makeKeys(P, Keys, Order); }); }
EXPORT void oracle_sortPass(unsigned* Keys, unsigned* Order, int distance, int span) { each_thread(CAPACITY, 128, [&] { sortPass(Keys, Order, distance, span); }); }
// The harness's own independent sort of (key, index) pairs (native_harness.cpp:47).
EXPORT void oracle_sortPairs(unsigned* Keys, unsigned* Order, int n) {
  std::vector<std::pair<unsigned, unsigned>> a;
  for (int i = 0; i < n; i++) a.push_back({Keys[i], Order[i]});
  std::sort(a.begin(), a.end());
  for (int i = 0; i < n; i++) { Keys[i] = a[i].first; Order[i] = a[i].second; }
}
EXPORT void oracle_makeBounds(const float* P, const unsigned* Order, float* Nodes) { each_thread(CAPACITY, 128, [&] { makeBounds(P, Order, Nodes); }); }
EXPORT void oracle_reduceBounds(float* Nodes, int first) { each_thread(first, 128, [&] { reduceBounds(Nodes, first); }); }
EXPORT void oracle_initCamera(float* C, const float* P, int seed) { scalar(); initCamera(C, P, seed); }
EXPORT void oracle_updateCamera(float* C, const float* I, const float* P, float delta, int width, int height) { scalar(); updateCamera(C, I, P, delta, width, height); }
EXPORT void oracle_tracePixels(const float* P, const float* Nodes, const unsigned* Order, const float* C, float* Hit, int w, int h, int y0, int y1, int single) {
  if (single) {
#pragma omp parallel for schedule(dynamic, 2)
    for (int y = y0; y < y1; y++)
      for (int x = 0; x < w; x++) trace_single(P, Nodes, Order, C, Hit, w, h, x, y);
    return;
  }
  each_pixel(w, y0, y1, [&] { tracePixels(P, Nodes, Order, C, Hit, w, h); });
}
EXPORT void oracle_shadePixels(const float* P, const float* Nodes, const unsigned* Order, const float* C, const float* Hit, float* Linear, float* Guide, int w, int h, int y0, int y1, int single) {
  if (single) {
#pragma omp parallel for schedule(dynamic, 2)
    for (int y = y0; y < y1; y++)
      for (int x = 0; x < w; x++) shade_single(P, Nodes, Order, C, Hit, Linear, Guide, w, h, x, y);
    return;
  }
  each_pixel(w, y0, y1, [&] { shadePixels(P, Nodes, Order, C, Hit, Linear, Guide, w, h); });
}
EXPORT void oracle_filterLighting(const float* Linear, const float* Guide, const float* Hit, float* Filtered, const float* C, int w, int h, int y0, int y1) {
  each_pixel(w, y0, y1, [&] { filterLighting(Linear, Guide, Hit, Filtered, C, w, h); });
}
EXPORT void oracle_resolvePixels(const float* Filtered, float* History, unsigned* Pixels, const float* C, int w, int h, int y0, int y1) {
  each_pixel(w, y0, y1, [&] { resolvePixels(Filtered, History, Pixels, C, w, h); });
}
EXPORT void oracle_tracePixelList(const float* P, const float* Nodes, const unsigned* Order, const float* C, float* Hit, int w, int h, const int* xy, int n, int single) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < n; i++) {
    int x = xy[2 * i], y = xy[2 * i + 1];
    if (single) { trace_single(P, Nodes, Order, C, Hit, w, h, x, y); continue; }
    blockDim = {8, 8, 1};
    blockIdx = {unsigned(x / 8), unsigned(y / 8), 0};
    threadIdx = {unsigned(x % 8), unsigned(y % 8), 0};
    tracePixels(P, Nodes, Order, C, Hit, w, h);
  }
}
EXPORT void oracle_traceTreeRay(const float* P, const float* Nodes, const unsigned* Order, const float* ro, const float* rd, float cone, float time, float wind, float best, int ignore, int shadows, float* out) {
  float2 r = traceTree(P, Nodes, Order, make_float3(ro[0], ro[1], ro[2]), make_float3(rd[0], rd[1], rd[2]), cone, time, wind, best, ignore, shadows != 0);
  out[0] = r.x; out[1] = r.y;
}
EXPORT float oracle_objectT(const float* P, int id, const float* ro, const float* rd, float fp, float time, float wind, int refine) {
  return objectT(P, id, make_float3(ro[0], ro[1], ro[2]), make_float3(rd[0], rd[1], rd[2]), fp, time, wind, refine != 0);
}
EXPORT float oracle_leafT(const float* P, int id, const float* ro, const float* rd, float fp, float time, float wind) {
  return leafT(P, id, make_float3(ro[0], ro[1], ro[2]), make_float3(rd[0], rd[1], rd[2]), fp, time, wind);
}
EXPORT void oracle_boxSpan(const float* ro, const float* rd, const float* lo, const float* hi, float* out) {
  float2 s = boxSpan(make_float3(ro[0], ro[1], ro[2]), make_float3(rd[0], rd[1], rd[2]), make_float3(lo[0], lo[1], lo[2]), make_float3(hi[0], hi[1], hi[2]));
  out[0] = s.x; out[1] = s.y;
}
EXPORT void oracle_bounds(const float* P, int id, float* lo, float* hi) {
  float3 a = boundLow(P, id), b = boundHigh(P, id);
  lo[0] = a.x; lo[1] = a.y; lo[2] = a.z; hi[0] = b.x; hi[1] = b.y; hi[2] = b.z;
}
EXPORT float oracle_barkCut(const float* P, int id, const float* p, float fp) { return barkCut(P, id, make_float3(p[0], p[1], p[2]), fp); }
EXPORT float oracle_bandWeight(float period, float fp) { return bandWeight(period, fp); }
EXPORT float oracle_rnd(int n, int seed) { return rnd(n, seed); }
EXPORT int oracle_forestSeed(int tree, int ws) { return forestSeed(tree, ws); }
EXPORT void oracle_forestInstance(int tree, int ws, float* out) {
  float3 p = forestPos(tree, ws);
  out[0] = p.x; out[1] = p.y; out[2] = p.z;
  out[3] = forestScale(tree, ws); out[4] = forestYaw(tree, ws);
  out[5] = (float)(forestSeed(tree, ws) & 8191) * 0.0017f;
}
// The harness's Renderer constructor sequence (native_harness.cpp:45-48), for
// the recorded BOUNDS line (docs/native-checks.log:2).
EXPORT void oracle_harnessBuild(int seed, float* B, float* P, unsigned* Keys, unsigned* Order, float* Nodes) {
  Renderer r(seed);
  std::copy(r.branches.begin(), r.branches.end(), B);
  std::copy(r.prims.begin(), r.prims.end(), P);
  std::copy(r.keys.begin(), r.keys.end(), Keys);
  std::copy(r.order.begin(), r.order.end(), Order);
  std::copy(r.nodes.begin(), r.nodes.end(), Nodes);
}
// The harness's own PPM writer (Renderer::save, native_harness.cpp:53) on the
// given pixels, to pin the library's PPM output to it byte for byte.
EXPORT void oracle_harnessSave(const unsigned* pixels, int width, int height, const char* path) {
  Renderer r(1788);
  r.resize(width, height);
  std::copy(pixels, pixels + (size_t)width * height, r.pixels.begin());
  r.save(path);
}
EXPORT void oracle_exhaustiveRay(const float* P, const float* ro, const float* rd, float cone, float* out) {
  float3 o = make_float3(ro[0], ro[1], ro[2]), d = make_float3(rd[0], rd[1], rd[2]);
  float nearest = FAR; int winner = -1;
  for (int id = 0; id < OBJECT_COUNT; id++) {
    auto a = boxSpan(o, d, boundLow(P, id), boundHigh(P, id));
    if (a.y < std::max(.0001f, a.x) || a.x > nearest) continue;
    float fp = std::max(.000005f, cone * std::max(.05f, a.x));
    float t = objectT(P, id, o, d, fp, 0, 0, true);
    if (t < nearest) { nearest = t; winner = id; }
  }
  out[0] = nearest; out[1] = (float)winner;
}
EXPORT void oracle_harnessRay(int ray, float* ro, float* rd) {
  float3 o = {rnd(ray, 198) * 24 - 12, 1 + rnd(ray, 31) * 14, rnd(ray, 78) * 24 - 12};
  float3 target = {rnd(ray, 211) * 10 - 5, 2 + rnd(ray, 433) * 8, rnd(ray, 123) * 10 - 5};
  float3 d = norm3(target - o);
  ro[0] = o.x; ro[1] = o.y; ro[2] = o.z; rd[0] = d.x; rd[1] = d.y; rd[2] = d.z;
}
EXPORT void oracle_footprintSweep(const float* P, int id, float* out) {
  bool mono = true, finite = true; float last = 1; float jump = 0;
  auto point = read3(P, id * PS) + make_float3(0.0f, 0.0f, P[id * PS + 7]);
  float prev = barkCut(P, id, point, .000001f);
  for (int i = 0; i < 10000; i++) {
    float f = 0.000001f * powf(100000.0f, float(i) / 9999);
    float w = bandWeight(.065f, f); mono &= w <= last + 1e-7f; last = w;
    float cut = barkCut(P, id, point, f); jump = std::max(jump, std::abs(cut - prev)); prev = cut; finite &= std::isfinite(cut);
  }
  out[0] = jump; out[1] = mono ? 1.0f : 0.0f; out[2] = finite ? 1.0f : 0.0f;
}
EXPORT void oracle_leafPair(const float* P, int k, float* out) {
  int id = WOOD_COUNT + k * 431; int b = id * PS;
  auto u = read3(P, b + 4); auto n = read3(P, b + 12);
  auto p = read3(P, b) + u * (P[b + 16] + P[b + 7] * .5f) + n * .10f; auto rd = n * -1.0f;
  out[0] = leafT(P, id, p, rd, .00001f, 0, 0); out[1] = leafT(P, id, p, rd, .05f, 0, 0);
}
namespace {
template <class F> void each_listed_row(int w, const int* rows, int n, F f) {
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < n; i++)
    for (int x = 0; x < w; x++) {
      int y = rows[i];
      blockDim = {8, 8, 1};
      blockIdx = {unsigned(x / 8), unsigned(y / 8), 0};
      threadIdx = {unsigned(x % 8), unsigned(y % 8), 0};
      f(x, y);
    }
}
}  // namespace
EXPORT void oracle_frameRows(const float* P, const float* Nodes, const unsigned* Order, const float* C, float* Hit, float* Linear, float* Guide,
                             float* Filtered, float* History, unsigned* Pixels, int w, int h, const int* rows, int n, int single) {
  each_listed_row(w, rows, n, [&](int x, int y) {
    if (single) trace_single(P, Nodes, Order, C, Hit, w, h, x, y); else tracePixels(P, Nodes, Order, C, Hit, w, h);
  });
  each_listed_row(w, rows, n, [&](int x, int y) {
    if (single) shade_single(P, Nodes, Order, C, Hit, Linear, Guide, w, h, x, y); else shadePixels(P, Nodes, Order, C, Hit, Linear, Guide, w, h);
  });
  each_listed_row(w, rows, n, [&](int, int) { filterLighting(Linear, Guide, Hit, Filtered, C, w, h); });
  each_listed_row(w, rows, n, [&](int, int) { resolvePixels(Filtered, History, Pixels, C, w, h); });
}
