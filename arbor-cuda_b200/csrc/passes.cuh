// passes.cuh - per-tile device code of the image passes, shared by the
// single-image kernels (render.cu) and the batched renderer (batch.cu):
// the trace and shade of one tile of pixels, the shading functions
// (Arbor.cu:256-289) and the filter / resolve of one tile (Arbor.cu:292-304).
#pragma once
#include "render_common.cuh"

namespace arbor {
namespace {

// A CTA's 256 threads cover a tile of tw x (256 / tw) pixels (tw = 16 or 32)
// made of 8x4-pixel warps.
__device__ __forceinline__ void tile_pixel_at(int t, int x0, int y0, int tw, int& x, int& y) {
  int warp = t >> 5, lane = t & 31, across = tw >> 3;
  x = x0 + (warp % across) * 8 + (lane & 7);
  y = y0 + (warp / across) * 4 + (lane >> 3);
}

// ---------------------------------------------------------------- trace --
// Primary rays (tracePixels); each warp's primitive tests run warp-batched
// (warpbatch.cuh).
struct PrimaryPolicy {
  static constexpr int kRefill = 8;  // idle lanes that trigger a refill (measured best of 1-16)
  const Camera* cam;
  float* Hit;
  int width, height, pixel;
  // The primary ray of pixel (x, y) with the ground plane as its initial
  // nearest hit (tracePixels, Arbor.cu:252).
  __device__ __forceinline__ void start(const TraceCtx& c, Ray& r, int x, int y) {
    pixel = y * width + x;
    f3 rd = camera_ray(*cam, x, y, width, height);
    float ground = rd.y < -0.00001f ? -cam->ro.y / rd.y : kFar;
    ray_begin(c, r, cam->ro, rd, ground > 0.0f ? ground : kFar);
  }
  __device__ __forceinline__ void done(Ray& r) {
    reinterpret_cast<float4*>(Hit)[pixel] = make_float4(r.best, r.found, (float)r.foundTree, cam->c14 * r.best / (float)height);
    r.phase = kPhIdle;
  }
};

// Primary rays of every pixel of a persistent CTA's pool.
template <class WB>
__device__ __forceinline__ void trace_pool(const TraceCtx& c, const Camera& cam, WB& b, float* __restrict__ Hit, const PixelPool& pool) {
  PrimaryPolicy policy{&cam, Hit, pool.width, pool.height, 0};
  Ray r;
  batch_run_pool(c, r, b, policy, pool);
}

// ---------------------------------------------------------------- shade --
// Arbor.cu:256
__device__ f3 sky(f3 rd, f3 sun) {
  float h = sat(rd.y);
  f3 c = mix3(mk(0.75f, 0.79f, 0.77f), mk(0.19f, 0.35f, 0.54f), xpow(h, 0.48f));
  float warm = xpow(sat(dot3(rd, sun)), 32.0f);
  c = c + mk(0.48f, 0.26f, 0.075f) * warm;
  float disc = smooth(0.99996f, 0.999984f, dot3(rd, sun));
  c = c + mk(8.0f, 6.7f, 4.9f) * disc;
  float clouds = noise(rd.x * 5.0f / (0.2f + h), rd.z * 5.0f / (0.2f + h), 231);
  float veil = smooth(0.62f, 0.81f, clouds) * smooth(0.02f, 0.18f, h) * 0.38f;
  return mix3(c, mk(1.1f, 1.10f, 1.05f), veil);
}
// Arbor.cu:257-263
__device__ f3 bark_color(const float* P, int id, f3 p, float footprint) {
  Wood w = load_wood(P, id);
  f3 q = p - w.a;
  float z = dot3(q, w.d);
  float theta = atan2f(dot3(q, w.v), dot3(q, w.u));
  float arc = w.arc0 + z;
  f3 coord = mk(cosf(theta) * 9.0f, sinf(theta) * 9.0f, arc * 7.0f);
  float mottle = noise3(p * 3.0f, 714);
  float rough = noise3(coord, w.seed);
  float t = sat(dot3(p - w.a, w.ab) / fmaxf(0.000001f, w.abab));
  float amp = fminf(0.021f, lerpf(w.ra, w.rb, t) * 0.055f);
  float cut = bark_cut(w, p, footprint, band_weight(0.010f, footprint), band_weight(0.0025f, footprint)) / fmaxf(0.00001f, amp);
  f3 c = mix3(mk(0.10f, 0.075f, 0.050f), mk(0.25f, 0.21f, 0.16f), 0.25f + rough * 0.62f);
  c = c * (0.75f + 0.35f * mottle);
  c = c * (1.0f - 0.62f * smooth(0.28f, 0.85f, cut));
  float moss = smooth(0.52f, 0.72f, noise3(p * 5.0f, 189)) * (1.0f - smooth(0.15f, 1.4f, p.y));
  c = mix3(c, mk(0.045f, 0.064f, 0.018f), moss * 0.62f);
  float lichen = smooth(0.65f, 0.77f, noise3(p * 23.0f, 27)) * smooth(0.25f, 0.65f, noise3(p * 90.0f, 712)) * band_weight(0.018f, footprint);
  c = mix3(c, mk(0.31f, 0.33f, 0.23f), lichen * 0.5f);
  float grain = (noise3(coord * 15.0f, w.seed) - 0.5f) * band_weight(0.0025f, footprint);
  return c * (1.0f + grain * 0.38f);
}
// Arbor.cu:264
__device__ float leaf_vein(const Leaf& l, f3 p, float footprint) {
  f3 q = p - l.origin;
  float x = dot3(q, l.u) - l.stem;
  float y = dot3(q, l.v);
  float len = l.len;
  float mid = xexp(-fabsf(y) / fmaxf(0.00065f, footprint * 0.55f));
  float fy = fracf((x - fabsf(y) * 0.70f) / len * 7.0f);
  float dd = fminf(fy, 1.0f - fy) * len / 7.0f;
  float lateral = xexp(-dd / fmaxf(0.00033f, footprint * 0.5f));
  return sat(mid * 0.82f + lateral * 0.48f) * band_weight(0.003f, footprint);
}
// Arbor.cu:265-268
__device__ f3 leaf_color(const Leaf& l, f3 p, float fp) {
  float h = rnd(l.seed, 887);
  f3 q = p - l.origin;
  float x = dot3(q, l.u) - l.stem;
  if (x < 0.0f) return mk(0.17f, 0.15f, 0.048f);
  float y = dot3(q, l.v);
  float v = leaf_vein(l, p, fp);
  f3 c = mix3(mk(0.035f, 0.11f, 0.008f), mk(0.15f, 0.255f, 0.025f), h);
  c = mix3(c, mk(0.22f, 0.26f, 0.055f), v * 0.57f);
  float speck = (noise(x * 700.0f, y * 700.0f, l.seed) - 0.5f) * band_weight(0.0017f, fp);
  float edge = smooth(0.78f, 1.0f, fabsf(y) / fmaxf(0.001f, leaf_width(x, l.len, l.width, band_weight(0.002f, fp))));
  c = c * (1.0f + speck * 0.27f);
  c = mix3(c, mk(0.23f, 0.20f, 0.05f), edge * 0.22f);
  return c;
}
// Arbor.cu:269
__device__ f3 ground_color(f3 p, float fp) {
  float a = noise(p.x * 3.0f, p.z * 3.0f, 819);
  float b = noise(p.x * 15.0f, p.z * 15.0f, 28);
  float r = sqrtf(p.x * p.x + p.z * p.z);
  float soil = 1.0f - smooth(4.1f, 6.8f, r + noise(p.x, p.z, 13));
  f3 grass = mix3(mk(0.085f, 0.115f, 0.035f), mk(0.23f, 0.24f, 0.092f), a);
  f3 dirt = mix3(mk(0.075f, 0.055f, 0.035f), mk(0.16f, 0.13f, 0.080f), b);
  float moss = smooth(0.53f, 0.73f, a);
  dirt = mix3(dirt, mk(0.049f, 0.079f, 0.022f), moss * 0.72f);
  float grit = (noise(p.x * 200.0f, p.z * 200.0f, 127) - 0.5f) * band_weight(0.007f, fp);
  return mix3(grass, dirt, soil) * (1.0f + grit * 0.40f);
}
// Arbor.cu:231-234
__device__ f3 object_normal(const float* P, int id, f3 p, float fp, float time, float wind) {
  int type = (int)ldg4(P, id * 6).w;
  if (type == 0) {
    Wood w = load_wood(P, id);
    float fine = band_weight(0.010f, fp), grain = band_weight(0.0025f, fp);
    float e = fmaxf(0.000035f, fminf(0.0005f, fp * 0.18f));
    f3 dx = mk(e, 0.0f, 0.0f), dy = mk(0.0f, e, 0.0f), dz = mk(0.0f, 0.0f, e);
    return norm3(mk(wood_field(w, p + dx, fp, fine, grain) - wood_field(w, p - dx, fp, fine, grain),
                    wood_field(w, p + dy, fp, fine, grain) - wood_field(w, p - dy, fp, fine, grain),
                    wood_field(w, p + dz, fp, fine, grain) - wood_field(w, p - dz, fp, fine, grain)));
  }
  if (type == 1) {
    Leaf l = load_leaf(P, id, time, wind);
    f3 q = p - l.origin;
    float x = dot3(q, l.u) - l.stem;
    float y = dot3(q, l.v);
    if (x < 0.0f) {
      f3 centre = l.origin + l.u * (x + l.stem);
      return norm3(p - centre);
    }
    const float e = 0.0002f;
    float hw2 = l.width * l.width, bw = band_weight(0.007f, fp);
    float a = (leaf_height(x + e, y, l.len, hw2, l.curl, l.twist, bw) - leaf_height(x - e, y, l.len, hw2, l.curl, l.twist, bw)) / (2.0f * e);
    float c = (leaf_height(x, y + e, l.len, hw2, l.curl, l.twist, bw) - leaf_height(x, y - e, l.len, hw2, l.curl, l.twist, bw)) / (2.0f * e);
    return norm3(l.n - l.u * a - l.v * c);
  }
  f3 q = p - xyz(ldg4(P, id * 6));
  f3 h = xyz(ldg4(P, id * 6 + 1));
  return norm3(mk(q.x / (h.x * h.x), q.y / (h.y * h.y), q.z / (h.z * h.z)));
}
// Arbor.cu:270
__device__ f3 surface_color(const float* P, int id, f3 p, float fp, float time, float wind) {
  if (id < 0) return ground_color(p, fp);
  float4 r0 = ldg4(P, id * 6);
  int type = (int)r0.w;
  if (type == 0) return bark_color(P, id, p, fp);
  if (type == 1) return leaf_color(load_leaf(P, id, time, wind), p, fp);
  float f = noise3(p * 42.0f, (int)ldg4(P, id * 6 + 3).w);
  return mix3(mk(0.09f, 0.10f, 0.086f), mk(0.31f, 0.30f, 0.24f), f);
}
// Arbor.cu:276
__device__ float spec_ggx(f3 n, f3 v, f3 l, float rough) {
  f3 h = norm3(v + l);
  float nh = sat(dot3(n, h));
  float nv = fmaxf(0.002f, sat(dot3(n, v)));
  float nl = sat(dot3(n, l));
  float vh = sat(dot3(v, h));
  float a = rough * rough;
  float aa = a * a;
  float den = nh * nh * (aa - 1.0f) + 1.0f;
  float D = aa / (kPi * den * den);
  float k = (rough + 1.0f) * (rough + 1.0f) * 0.125f;
  float G = nv / (nv * (1.0f - k) + k) * nl / (nl * (1.0f - k) + k);
  float F = 0.035f + 0.965f * xpow(1.0f - vh, 5.0f);
  return D * G * F / (4.0f * nv + 0.0001f);
}

// shadePixels (Arbor.cu:277-289) is split at the sun-visibility call:
// shade_pre computes everything before it, the shadow segments are traced by
// the warp tracer, shade_post composes the colour.  Each value is computed
// with the reference's operations in the reference's order; the colour
// before haze is (direct * visibility) * (4.8, 4.2, 3.1) + albedo * ambient.
struct Shading {
  f3 direct, ambientTerm, skyc, guide, origin, light, debug;
  f3 normal;    // shading normal (zero for sky), the G-buffer normal
  float haze;
  bool final;   // colour is `debug` (sky pixel or debug view mode): no visibility needed
  bool shadow;  // visibility must be traced
};

// The pixel's light direction: the sun jittered inside its disk by the
// pixel's and sample's hashes (Arbor.cu:282).
__device__ __forceinline__ f3 sun_sample(const Camera& cam, int pixel) {
  const f3 sun = cam.sun;
  int sample = cam.sample;
  float r1 = rnd((int)((uint32_t)pixel + (uint32_t)sample * 1823u), 991);
  float r2 = rnd((int)((uint32_t)pixel + (uint32_t)sample * 971u), 731);
  f3 su = basisU(sun);
  f3 sv = cross3(sun, su);
  float angle = r1 * 6.28318f;
  float disk = sqrtf(r2) * 0.012f;
  return norm3(sun + su * (xcos(angle) * disk) + sv * (xsin(angle) * disk));
}
// The first shadow segment's origin, off the surface along the light
// (Arbor.cu:283).
__device__ __forceinline__ f3 shadow_origin(f3 p, f3 light, int id) {
  float offset = id >= 0 ? 0.0014f : 0.004f;
  return p + light * offset;
}

// The single-tree scene uses the identity instance: tree-local point and
// normal, phase 0, no tint.
template <bool kForestScene>
__device__ __noinline__ void shade_pre(const float* P, const Camera& cam, const Instance* inst, float4 hit, int x, int y, int width, int height,
                          Shading& o) {
  int pixel = y * width + x;
  float t = hit.x;
  int id = (int)hit.y;
  int tree = (int)hit.z;
  // IDs past the record / instance ranges cannot come from tracePixels; such
  // input is shaded as ground rather than read out of bounds.
  if (id >= kCapacity) id = -1;
  if (tree >= kForest) tree = -1;
  f3 ro = cam.ro;
  f3 rd = camera_ray(cam, x, y, width, height);
  f3 sun = cam.sun;
  o.skyc = sky(rd, sun);
  o.guide = mk(1.0f, 1.0f, 1.0f);
  o.shadow = false;
  o.normal = mk(0.0f, 0.0f, 0.0f);
  if (!(t < kFar)) {
    o.final = true;
    o.debug = o.skyc;
    return;
  }
  f3 p = ro + rd * t;
  float fp = fmaxf(0.000005f, hit.w);
  f3 localP = p;
  f3 n = mk(0.0f, 1.0f, 0.0f);
  float localFp = fp;
  float phase = 0.0f;
  const float time = cam.time, wind = cam.wind;
  if (kForestScene) {
    if (id >= 0 && tree >= 0) {
      const Instance& it = inst[tree];
      localP = to_local_point(p, it);
      localFp = fp / it.sc;
      phase = it.phase;
      n = to_world_normal(object_normal(P, id, localP, localFp, time + phase, wind), it);
    }
  } else if (id >= 0) {
    n = object_normal(P, id, localP, localFp, time, wind);
  }
  bool leaf = id >= 0 && ldg4(P, id * 6).w == 1.0f;
  if (dot3(n, rd) > 0.0f) n = n * -1.0f;
  if (id < 0) {
    float e = fmaxf(0.001f, fp);
    uint32_t h133 = hashU(133u);
    float nx = (noise_h((p.x + e) * 18.0f, p.z * 18.0f, h133) - noise_h((p.x - e) * 18.0f, p.z * 18.0f, h133)) * 0.18f;
    float nz = (noise_h(p.x * 18.0f, (p.z + e) * 18.0f, h133) - noise_h(p.x * 18.0f, (p.z - e) * 18.0f, h133)) * 0.18f;
    n = norm3(mk(nx, 1.0f, nz));
  }
  o.normal = n;
  f3 albedo = surface_color(P, id, id >= 0 ? localP : p, localFp, time + phase, wind);
  if (kForestScene && tree >= 0) {
    int ts = inst[tree].seed;
    float hue = rnd(8, ts);
    float age = rnd(9, ts);
    float season = rnd(10, ts);
    float dark = 0.76f + age * 0.38f;
    f3 tint = mk(0.88f + 0.22f * hue, 0.84f + 0.28f * (1.0f - fabsf(hue - 0.55f)), 0.72f + 0.25f * (1.0f - hue));
    if (leaf)
      tint = mix3(tint, mk(1.12f, 0.88f, 0.48f), smooth(0.78f, 0.98f, season) * 0.38f);
    else
      tint = mix3(tint, mk(0.78f, 0.66f, 0.53f), season * 0.18f);
    albedo = albedo * tint * dark;
  }
  o.guide = albedo;
  if (cam.mode == 1.0f || cam.mode == 2.0f || cam.mode == 3.0f) {
    // Debug views replace the colour whatever the lighting (Arbor.cu:286).
    o.final = true;
    if (cam.mode == 1.0f) {
      float w0 = band_weight(0.065f, localFp);
      float w1 = band_weight(0.005f, localFp);
      float w2 = band_weight(0.001f, localFp);
      o.debug = mk(w0 * 0.80f, w1 * 0.85f, w2 * 0.9f);
    } else if (cam.mode == 2.0f) {
      float hh = rnd(id + 177 + (tree + 1) * 71, 32);
      o.debug = id < 0 ? mk(0.10f, 0.10f, 0.10f) : (leaf ? mk(0.1f, 0.3f + hh * 0.5f, 0.17f) : mk(0.47f + hh * 0.3f, 0.25f, 0.10f));
    } else {
      o.debug = n * 0.5f + mk(0.5f, 0.5f, 0.5f);
    }
    return;
  }
  o.final = false;
  const f3 light = sun_sample(cam, pixel);
  o.light = light;
  o.origin = shadow_origin(p, light, id);
  o.shadow = cam.shadows > 0.5f;
  float nl = sat(dot3(n, light));
  float back = sat(-dot3(n, light));
  f3 direct = albedo * (nl / kPi);
  if (leaf) {
    float vein = leaf_vein(load_leaf(P, id, time + phase, wind), localP, localFp);
    direct = direct + albedo * (back * (0.75f - 0.25f * vein) + xpow(sat(dot3(rd, light)), 9.0f) * 0.12f);
  }
  float spec = spec_ggx(n, rd * -1.0f, light, leaf ? 0.39f : 0.82f);
  o.direct = direct + mk(spec, spec, spec);
  float ao = 1.0f;
  f3 ambient = mk(0.30f, 0.37f, 0.45f) * (0.45f + 0.55f * sat(n.y)) * ao + mk(0.08f, 0.068f, 0.035f) * sat(-n.y);
  if (leaf) ambient = ambient + mk(0.04f, 0.055f, 0.022f) * ao;
  o.ambientTerm = albedo * ambient;
  o.haze = 1.0f - xexp(-t * 0.0018f);
}
__device__ __forceinline__ f3 shade_post(const Shading& o, f3 visibility) {
  if (o.final) return o.debug;
  f3 col = o.direct * visibility * mk(4.8f, 4.2f, 3.1f) + o.ambientTerm;
  return mix3(col, o.skyc, o.haze);
}

// Whether shadePixels traces a shadow ray for a pixel whose hit distance is
// t: a surface hit (not sky), no debug view, sun shadows on (Arbor.cu:283,
// 286).  The shadow setup pass stages a ray exactly where this holds, and the
// compose pass reads the shadow pass's visibility exactly where it holds.
__device__ __forceinline__ bool traces_shadow(const Camera& cam, float t) {
  return t < kFar && !(cam.mode == 1.0f || cam.mode == 2.0f || cam.mode == 3.0f) && cam.shadows > 0.5f;
}

// The shadow ray of pixel (x, y), when shadePixels traces one.  The same
// values shade_pre computes for the pixel.
__device__ __forceinline__ bool shadow_ray(const Camera& cam, float4 hit, int x, int y, int width, int height, f3& origin, f3& light) {
  const float t = hit.x;
  int id = (int)hit.y;
  if (id >= kCapacity) id = -1;
  if (!traces_shadow(cam, t)) return false;
  const f3 p = cam.ro + camera_ray(cam, x, y, width, height) * t;
  light = sun_sample(cam, y * width + x);
  origin = shadow_origin(p, light, id);
  return true;
}

// Shadow segments alone (Arbor.cu:271-274), for the persistent shadow pass:
// a pixel's visibility toward the sun is written to Vis (the Linear buffer,
// which the compose pass then overwrites with the colour); pixels without a
// shadow ray are left alone.
struct ShadowPolicy {
  static constexpr int kRefill = 8;
  const TraceCtx* ctx;
  const Camera* cam;
  const float* Hit;
  float* Vis;
  int width, height;
  int pixel, seg;
  f3 trans, origin, light;
  __device__ __forceinline__ void start(const TraceCtx& c, Ray& r, int x, int y) {
    pixel = y * width + x;
    if (shadow_ray(*cam, __ldg(reinterpret_cast<const float4*>(Hit) + pixel), x, y, width, height, origin, light)) {
      trans = mk(1.0f, 1.0f, 1.0f);
      seg = 0;
      ray_begin(c, r, origin, light, 36.0f);
    } else {
      r.phase = kPhIdle;
    }
  }
  __device__ __forceinline__ void write(f3 v) { reinterpret_cast<float4*>(Vis)[pixel] = make_float4(v.x, v.y, v.z, 1.0f); }
  __device__ __forceinline__ void done(Ray& r) {
    int id = (int)r.found;
    if (id < 0) {
      write(trans);
    } else if (ldg4(scene_P(*ctx, tree_species(*ctx, r.foundTree)), id * 6).w != 1.0f) {
      write(mk(0.0f, 0.0f, 0.0f));
    } else {
      trans = trans * mk(0.18f, 0.29f, 0.065f);
      origin = origin + light * (r.best + 0.0018f);
      if (++seg < 4) {
        ray_begin(*ctx, r, origin, light, 36.0f);
        return;
      }
      write(trans);
    }
    r.phase = kPhIdle;
  }
};

// Shadow segments of every pixel of a persistent CTA's pool.
template <class WB>
__device__ __forceinline__ void shadow_pool(const TraceCtx& c, const Camera& cam, WB& b, const float* __restrict__ Hit, float* __restrict__ Vis,
                                            const PixelPool& pool) {
  ShadowPolicy policy{&c, &cam, Hit, Vis, pool.width, pool.height, 0, 0};
  Ray r;
  batch_run_pool(c, r, b, policy, pool);
}

// The same shadow segments with each pixel's ray staged in memory by the
// setup pass (shadow_setup_px): origin in Vis (w = 1 when the pixel has a
// shadow ray), direction in Dir.  The tracer's loop then holds no camera or
// sun-sampling code.
struct StagedShadowPolicy {
  static constexpr int kRefill = 8;
  const TraceCtx* ctx;
  const float* Dir;
  float* Vis;
  int width, height;
  int pixel, seg;
  f3 trans, origin, light;
  __device__ __forceinline__ void start(const TraceCtx& c, Ray& r, int x, int y) {
    pixel = y * width + x;
    const float4 o = reinterpret_cast<const float4*>(Vis)[pixel];
    if (o.w == 1.0f) {
      origin = mk(o.x, o.y, o.z);
      light = xyz(__ldg(reinterpret_cast<const float4*>(Dir) + pixel));
      trans = mk(1.0f, 1.0f, 1.0f);
      seg = 0;
      ray_begin(c, r, origin, light, 36.0f);
    } else {
      r.phase = kPhIdle;
    }
  }
  __device__ __forceinline__ void write(f3 v) { reinterpret_cast<float4*>(Vis)[pixel] = make_float4(v.x, v.y, v.z, 1.0f); }
  __device__ __forceinline__ void done(Ray& r) {
    int id = (int)r.found;
    if (id < 0) {
      write(trans);
    } else if (ldg4(scene_P(*ctx, tree_species(*ctx, r.foundTree)), id * 6).w != 1.0f) {
      write(mk(0.0f, 0.0f, 0.0f));
    } else {
      trans = trans * mk(0.18f, 0.29f, 0.065f);
      origin = origin + light * (r.best + 0.0018f);
      if (++seg < 4) {
        ray_begin(*ctx, r, origin, light, 36.0f);
        return;
      }
      write(trans);
    }
    r.phase = kPhIdle;
  }
};

// Stage pixel (x, y)'s shadow ray for StagedShadowPolicy: origin and w = 1
// into Vis and the direction into Dir, or Vis.w = 0 without a shadow ray.
__device__ __forceinline__ void shadow_setup_px(const Camera& cam, const float* __restrict__ Hit, float* __restrict__ Vis, float* __restrict__ Dir,
                                                int x, int y, int width, int height) {
  const int pixel = y * width + x;
  f3 origin, light;
  if (shadow_ray(cam, __ldg(reinterpret_cast<const float4*>(Hit) + pixel), x, y, width, height, origin, light)) {
    reinterpret_cast<float4*>(Vis)[pixel] = make_float4(origin.x, origin.y, origin.z, 1.0f);
    reinterpret_cast<float4*>(Dir)[pixel] = make_float4(light.x, light.y, light.z, 0.0f);
  } else {
    reinterpret_cast<float4*>(Vis)[pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
}

// Staged shadow segments of every pixel of a persistent CTA's pool.
template <class WB>
__device__ __forceinline__ void staged_shadow_pool(const TraceCtx& c, WB& b, const float* __restrict__ Dir, float* __restrict__ Vis,
                                                   const PixelPool& pool) {
  StagedShadowPolicy policy{&c, Dir, Vis, pool.width, pool.height, 0, 0};
  Ray r;
  batch_run_pool(c, r, b, policy, pool);
}

// shadePixels' colour of pixel (x, y) (Arbor.cu:277-289), its visibility
// read from Linear where the shadow pass traced one.  kSpecies: a forest of
// several species, P holding one scene per species back to back; the hit
// instance's scene is shaded.
template <bool kForestScene, bool kSpecies = false>
__device__ __forceinline__ void shade_compose_px(const float* __restrict__ P, const Camera& cam, const Instance* inst, const float* __restrict__ Hit,
                                                 float* __restrict__ Linear, float* __restrict__ Guide, float* __restrict__ Normal, int x, int y,
                                                 int width, int height) {
  const int pixel = y * width + x;
  const float4 hit = __ldg(reinterpret_cast<const float4*>(Hit) + pixel);
  if (kSpecies) {
    const int tree = (int)hit.z;
    if (tree >= 0 && tree < kForest) P += (size_t)inst[tree].species * (kCapacity * kPS);
  }
  Shading sh;
  shade_pre<kForestScene>(P, cam, inst, hit, x, y, width, height, sh);
  f3 vis = mk(1.0f, 1.0f, 1.0f);
  if (traces_shadow(cam, hit.x)) vis = xyz(reinterpret_cast<const float4*>(Linear)[pixel]);
  const f3 col = shade_post(sh, vis);
  reinterpret_cast<float4*>(Linear)[pixel] = make_float4(col.x, col.y, col.z, 1.0f);
  reinterpret_cast<float4*>(Guide)[pixel] = make_float4(sh.guide.x, sh.guide.y, sh.guide.z, 1.0f);
  if (Normal) reinterpret_cast<float4*>(Normal)[pixel] = make_float4(sh.normal.x, sh.normal.y, sh.normal.z, 0.0f);
}

// ------------------------------------------------------ filter / resolve --
// A filter tile is kFX x kFY output pixels, computed by kFX x kFT threads
// (threadIdx.x, threadIdx.y), each thread a vertical pair of pixels.
constexpr int kFX = 32, kFY = 16, kFT = kFY / 2, kHalo = 2;
constexpr int kSX = kFX + 2 * kHalo, kSY = kFY + 2 * kHalo;

// Arbor.cu:303
__device__ __forceinline__ float aces(float x) { return sat((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f)); }

// The filter and resolve keep the transcendental / conversion unit (which
// runs divisions' reciprocals, exp2/log2 and int<->float conversions at an
// eighth of the FMA rate) for the IEEE divisions the reference's results
// need; truncations and floors of small values are taken in FP32 adds with
// directed rounding instead: for |v| < 2^22, v + 1.5 * 2^23 lies in
// [2^23, 2^24), where consecutive floats are consecutive integers, so the
// sum rounded toward zero / toward minus infinity is 1.5 * 2^23 + trunc(v) /
// + floor(v) exactly, and the integer difference of the bit patterns is that
// integer.
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;

// Vignette coordinate of column x of a width-pixel image (row y of a height
// one): ((float)x / (float)width - 0.5) * 2 (Arbor.cu:304).
__device__ __forceinline__ float vig_coord(int x, int width) { return ((float)x / (float)width - 0.5f) * 2.0f; }

// One channel of resolvePixels' output byte (Arbor.cu:304, packRGB :49):
// byte = (uint)(t), t = sat(pow(aces(c), 1/2.2) * vig) * 255 + 0.5, with the
// power taken as the float of the double-precision pow (xpow) and aces with
// IEEE division.  The byte changes only where t crosses an integer.  The fast
// path evaluates t with an approximate division in aces (within 2 ulp) and
// the hardware exp2/log2 power (__powf: relative error below 1e-6 wherever
// the power is above 1e-3, and an absolute error below 1e-9 under it), so its
// t is within 3e-4 of the exact t; where it lies within 1e-3 of an integer
// the exact t decides.  Same bytes as the exact evaluation, far fewer
// instructions.  t lies in [0.5, 255.5], so its floor is taken with kMagic.
__device__ __forceinline__ uint32_t gamma_byte(float c, float vig) {
  const float a = sat(__fdividef(c * (2.51f * c + 0.03f), c * (2.43f * c + 0.59f) + 0.14f));
  float t = sat(__powf(a, 1.0f / 2.2f) * vig) * 255.0f + 0.5f;
  float fl = __fadd_rd(t, kMagic);  // kMagic + floor(t)
  const float fr = t - (fl - kMagic);
  // (|c| >= 1e18 also takes the exact path: there the approximate division's
  // denominator can pass 2^126, where __fdividef returns 0.)
  if (fr < 1e-3f || fr > 1.0f - 1e-3f || !(fabsf(c) < 1e18f)) {
    t = sat(xpow(aces(c), 1.0f / 2.2f) * vig) * 255.0f + 0.5f;
    fl = __fadd_rd(t, kMagic);
  }
  return (uint32_t)(__float_as_int(fl) - kMagicBits);
}

// Arbor.cu:304, one pixel i: `current` is the filtered colour; count is the
// sample count (C[10] > 0.5 ? 0 : C[9]) and inv = 1 / (count + 1), the same
// for every pixel; u, v the pixel's vignette coordinates (vig_coord).
__device__ __forceinline__ void resolve_px(f3 current, float* __restrict__ History, uint32_t* __restrict__ Pixels, float count, float inv,
                                           float exposure, float u, float v, int i) {
  f3 mean = current;
  if (!(count < 0.5f)) mean = mix3(xyz(reinterpret_cast<const float4*>(History)[i]), current, inv);
  reinterpret_cast<float4*>(History)[i] = make_float4(mean.x, mean.y, mean.z, count + 1.0f);
  const f3 col = mean * exposure;
  const float vig = 1.0f - 0.09f * (u * u + v * v);
  Pixels[i] = gamma_byte(col.x, vig) | (gamma_byte(col.y, vig) << 8) | (gamma_byte(col.z, vig) << 16) | 4278190080u;
}
__device__ __forceinline__ float sample_count(float c9, float c10) { return c10 > 0.5f ? 0.0f : c9; }

// Same-surface 5x5 demodulated filter (Arbor.cu:292-302) of one kFX x kFY
// tile, staged with a 2-pixel halo in shared memory so each input pixel is
// read from HBM once per tile.  Each halo pixel is staged once as its depth,
// its surface key and its demodulated colour Linear / (Guide + 0.02): the
// same conversions and IEEE quotients the reference evaluates per neighbour,
// evaluated once per pixel.  The surface key packs (int) primitive id + 1 and
// (int) tree id + 1 into 16 bits each, so one integer compare decides "same
// primitive and same tree"; a tile holding an id or tree id outside
// -1..65534 (never written by tracePixels) is filtered by the reference's
// per-neighbour loop instead (filter_px_direct).  Each thread filters a
// vertical pair of pixels: their 5x5 windows share 20 taps, loaded once.
// Each pixel's taps are accumulated in the reference's order (rows, then
// columns) with its weights as constants; tiles whose halo lies inside the
// image skip the bounds test.  kResolve fuses resolvePixels on the filtered
// value.
struct FilterTile {
  int2 key[kSY][kSX];      // depth bits, packed surface key
  float4 demod[kSY][kSX];  // Linear / (Guide + 0.02)
  float w[6];              // weights of r^2 = 0, 1, 2, 4, 5, 8
  float u[kFX], v[kFY];    // vignette coordinates of the tile's columns and rows
};

// Weight of tap (j, k), from the staged exp(-0.3 r^2) values (compile-time index).
__device__ __forceinline__ float tap_weight(const float (&w)[6], int j, int k) {
  const int r2 = j * j + k * k;
  return w[r2 == 0 ? 0 : r2 == 1 ? 1 : r2 == 2 ? 2 : r2 == 4 ? 3 : r2 == 5 ? 4 : 5];
}

// The centre pixel of a filter pass and its running sums.
struct FilterCentre {
  int key;
  float depth, tol;
  f3 sum;
  float weight;
};

// One tap of one centre: accept a neighbour with the same surface key and
// |depth difference| not above the tolerance (Arbor.cu:297-299).
__device__ __forceinline__ void filter_tap(FilterCentre& c, int2 q, const float4* demod, float wt) {
  if (q.y != c.key || fabsf(__int_as_float(q.x) - c.depth) > c.tol) return;
  const float4 d = *demod;
  c.sum = c.sum + mk(d.x, d.y, d.z) * wt;
  c.weight += wt;
}

// The taps of a vertical pixel pair centred at shared-memory (cx, cy) and
// (cx, cy + 1), image (x, y) and (x, y + 1): rows cy - 2 .. cy + 3 are read
// once; row r feeds pixel 0 as tap row r - cy and pixel 1 as tap row
// r - cy - 1.
template <bool kEdge>
__device__ __forceinline__ void filter_pair(const FilterTile& s, int cx, int cy, int x, int y, int width, int height, const float (&w)[6],
                                            FilterCentre& p0, FilterCentre& p1, bool live0, bool live1) {
#pragma unroll
  for (int r = -2; r <= 3; r++)
#pragma unroll
    for (int k = -2; k <= 2; k++) {
      const int2 q = s.key[cy + r][cx + k];
      const float4* d = &s.demod[cy + r][cx + k];
      if (kEdge) {
        const int xx = x + k, yy = y + r;
        if (xx < 0 || xx >= width || yy < 0 || yy >= height) continue;
      }
      if (r <= 2 && live0) filter_tap(p0, q, d, tap_weight(w, r, k));
      if (r >= -1 && live1) filter_tap(p1, q, d, tap_weight(w, r - 1, k));
    }
}

// filterLighting of pixel (x, y) straight from global memory, in the
// reference's per-neighbour form (Arbor.cu:292-302): the path for tiles whose
// ids do not fit the packed key.
__device__ __noinline__ f3 filter_px_direct(const float* __restrict__ Linear, const float* __restrict__ Guide, const float* __restrict__ Hit,
                                            int x, int y, int width, int height) {
  const int i = y * width + x;
  const float4 lc = __ldg(reinterpret_cast<const float4*>(Linear) + i);
  const float4 gc = __ldg(reinterpret_cast<const float4*>(Guide) + i);
  const float4 hc = __ldg(reinterpret_cast<const float4*>(Hit) + i);
  f3 col = mk(lc.x, lc.y, lc.z);
  const f3 base = mk(gc.x, gc.y, gc.z) + mk(0.02f, 0.02f, 0.02f);
  f3 sum = mk(0.0f, 0.0f, 0.0f);
  float weight = 0.0f;
  const int id = (int)hc.y, tree = (int)hc.z;
  const float tol = fmaxf(0.005f, hc.w * 6.0f);
  for (int j = -2; j <= 2; j++)
    for (int k = -2; k <= 2; k++) {
      const int xx = x + k, yy = y + j;
      if (xx < 0 || yy < 0 || xx >= width || yy >= height) continue;
      const int q = yy * width + xx;
      const float4 h = __ldg(reinterpret_cast<const float4*>(Hit) + q);
      if ((int)h.y != id || (int)h.z != tree || fabsf(h.x - hc.x) > tol) continue;
      const float wt = xexp(-(float)(j * j + k * k) * 0.30f);  // the staged weights' values
      const float4 l = __ldg(reinterpret_cast<const float4*>(Linear) + q);
      const float4 g = __ldg(reinterpret_cast<const float4*>(Guide) + q);
      sum = sum + mk(l.x / (g.x + 0.02f), l.y / (g.y + 0.02f), l.z / (g.z + 0.02f)) * wt;
      weight += wt;
    }
  if (weight > 0.0f) col = mix3(col, (sum / weight) * base, 0.86f);
  return col;
}

// Packed surface key of a Hit record: (int) id + 1 and (int) tree + 1 in 16
// bits each, or -1 (never a packed key) unless both lie in [0, 65535) or are
// exactly -1 (what tracePixels writes); the truncations are kMagic adds
// rounded toward zero.
__device__ __forceinline__ bool key_range(float v) { return (v >= 0.0f || v == -1.0f) && v < 65535.0f; }
__device__ __forceinline__ int surface_key(float id_f, float tree_f) {
  if (!key_range(id_f) || !key_range(tree_f)) return -1;
  const int id = __float_as_int(__fadd_rz(id_f, kMagic)) - kMagicBits, tree = __float_as_int(__fadd_rz(tree_f, kMagic)) - kMagicBits;
  return (id + 1) | ((tree + 1) << 16);
}

// Filter weights expf(-(j*j+k*k)*0.30f) for r^2 = 0, 1, 2, 4, 5, 8, staged by
// the first six threads.
__device__ __forceinline__ void filter_weights(FilterTile& s, int tid) {
  if (tid < 6) {
    const int r2[6] = {0, 1, 2, 4, 5, 8};
    s.w[tid] = xexp(-(float)r2[tid] * 0.30f);
  }
}

// One staged halo pixel: its depth bits, packed key and demodulated colour.
// Returns false when its ids do not fit the packed key.
__device__ __forceinline__ bool filter_stage_px(FilterTile& s, int sy, int sx, float4 h, float4 l, float4 g) {
  const int key = surface_key(h.y, h.z);
  s.key[sy][sx] = make_int2(__float_as_int(h.x), key);
  s.demod[sy][sx] = make_float4(l.x / (g.x + 0.02f), l.y / (g.y + 0.02f), l.z / (g.z + 0.02f), 0.0f);
  return key >= 0;
}

// Stage a tile's halo from global memory.  Returns (uniformly over the CTA)
// whether some staged id does not fit the packed key.
// All of a thread's staging loads are issued before any is used, so their
// latencies overlap.  The vignette coordinates of the tile's columns and
// rows are computed once here (kResolve).
template <bool kResolve>
__device__ __forceinline__ bool filter_stage_global(FilterTile& s, const float* __restrict__ Linear, const float* __restrict__ Guide,
                                                    const float* __restrict__ Hit, int width, int height, int x0, int y0, int tid) {
  filter_weights(s, tid);
  if (kResolve) {
    if (tid >= 32 && tid < 32 + kFX) s.u[tid - 32] = vig_coord(x0 + tid - 32, width);
    if (tid >= 64 && tid < 64 + kFY) s.v[tid - 64] = vig_coord(y0 + tid - 64, height);
  }
  const int hx0 = x0 - kHalo, hy0 = y0 - kHalo;
  constexpr int kPer = (kSX * kSY + kFX * kFT - 1) / (kFX * kFT);
  float4 hv[kPer], lv[kPer], gv[kPer];
  bool in[kPer];
#pragma unroll
  for (int n = 0; n < kPer; n++) {
    const int k = tid + n * kFX * kFT;
    const int sy = k / kSX, sx = k - sy * kSX;
    const int gx = hx0 + sx, gy = hy0 + sy;
    in[n] = k < kSX * kSY && gx >= 0 && gy >= 0 && gx < width && gy < height;
    if (in[n]) {
      const int q = gy * width + gx;
      hv[n] = __ldg(reinterpret_cast<const float4*>(Hit) + q);
      lv[n] = __ldg(reinterpret_cast<const float4*>(Linear) + q);
      gv[n] = __ldg(reinterpret_cast<const float4*>(Guide) + q);
    }
  }
  bool unpacked = false;
#pragma unroll
  for (int n = 0; n < kPer; n++) {
    const int k = tid + n * kFX * kFT;
    const int sy = k / kSX, sx = k - sy * kSX;
    if (in[n]) unpacked |= !filter_stage_px(s, sy, sx, hv[n], lv[n], gv[n]);
  }
  return __syncthreads_or(unpacked);
}

// The centre values of a pair's pixel e, read from global memory.
struct CentreGlobal {
  const float* Linear;
  const float* Guide;
  const float* Hit;
  int i0, width;
  __device__ __forceinline__ int index(int e) const { return e ? i0 + width : i0; }
  __device__ __forceinline__ float4 linear(int e) const { return __ldg(reinterpret_cast<const float4*>(Linear) + index(e)); }
  __device__ __forceinline__ float4 guide(int e) const { return __ldg(reinterpret_cast<const float4*>(Guide) + index(e)); }
  __device__ __forceinline__ float footprint(int e) const { return __ldg(Hit + 4 * index(e) + 3); }
};

// Filter the staged tile: each thread its vertical pair of pixels, then
// (kResolve) resolvePixels on the filtered values.
template <bool kResolve, class Centre>
__device__ __forceinline__ void filter_finish(const FilterTile& s, bool unpacked, const Centre& ctr, const float* __restrict__ Linear,
                                              const float* __restrict__ Guide, const float* __restrict__ Hit, float* __restrict__ Filtered,
                                              float* __restrict__ History, uint32_t* __restrict__ Pixels, float c9, float c10, float c15, float c20,
                                              int width, int height, int x0, int y0) {
  const float w[6] = {s.w[0], s.w[1], s.w[2], s.w[3], s.w[4], s.w[5]};
  const int x = x0 + threadIdx.x, y = y0 + 2 * threadIdx.y;
  if (x >= width || y >= height) return;
  const float count = sample_count(c9, c10);
  const float inv = kResolve ? 1.0f / (count + 1.0f) : 0.0f;
  const int cx = threadIdx.x + kHalo, cy = 2 * threadIdx.y + kHalo;
  const bool has1 = y + 1 < height;
  const int i0 = y * width + x, i1 = i0 + width;
  const bool filter = c15 < 0.5f;
  FilterCentre p[2];
  bool live[2];
#pragma unroll
  for (int e = 0; e < 2; e++) {
    const int2 kc = s.key[cy + e][cx];
    p[e].key = kc.y;
    p[e].depth = __int_as_float(kc.x);
    p[e].sum = mk(0.0f, 0.0f, 0.0f);
    p[e].weight = 0.0f;
    live[e] = filter && (e == 0 || has1) && p[e].depth < kFar;
    p[e].tol = live[e] ? fmaxf(0.005f, ctr.footprint(e) * 6.0f) : 0.0f;
  }
  f3 col[2];
  if (!unpacked) {
    const bool interior = x0 >= kHalo && y0 >= kHalo && x0 + kFX + kHalo <= width && y0 + kFY + kHalo <= height;
    if (live[0] || live[1]) {
      if (interior)
        filter_pair<false>(s, cx, cy, x, y, width, height, w, p[0], p[1], live[0], live[1]);
      else
        filter_pair<true>(s, cx, cy, x, y, width, height, w, p[0], p[1], live[0], live[1]);
    }
#pragma unroll
    for (int e = 0; e < 2; e++) {
      if (e == 1 && !has1) break;
      const float4 lc = ctr.linear(e);
      col[e] = mk(lc.x, lc.y, lc.z);
      if (live[e] && p[e].weight > 0.0f) {
        const float4 gc = ctr.guide(e);
        const f3 base = mk(gc.x, gc.y, gc.z) + mk(0.02f, 0.02f, 0.02f);
        col[e] = mix3(col[e], (p[e].sum / p[e].weight) * base, 0.86f);
      }
    }
  } else {
#pragma unroll
    for (int e = 0; e < 2; e++) {
      if (e == 1 && !has1) break;
      if (live[e]) {
        col[e] = filter_px_direct(Linear, Guide, Hit, x, y + e, width, height);
      } else {
        const float4 lc = ctr.linear(e);
        col[e] = mk(lc.x, lc.y, lc.z);
      }
    }
  }
#pragma unroll
  for (int e = 0; e < 2; e++) {
    if (e == 1 && !has1) break;
    reinterpret_cast<float4*>(Filtered)[e ? i1 : i0] = make_float4(col[e].x, col[e].y, col[e].z, 1.0f);
    if (kResolve) resolve_px(col[e], History, Pixels, count, inv, c20, s.u[threadIdx.x], s.v[2 * threadIdx.y + e], e ? i1 : i0);
  }
}

template <bool kResolve>
__device__ __forceinline__ void filter_tile(FilterTile& s, const float* __restrict__ Linear, const float* __restrict__ Guide,
                                            const float* __restrict__ Hit, float* __restrict__ Filtered, float* __restrict__ History,
                                            uint32_t* __restrict__ Pixels, float c9, float c10, float c15, float c20, int width, int height,
                                            int x0, int y0) {
  const int tid = threadIdx.y * kFX + threadIdx.x;
  const bool unpacked = filter_stage_global<kResolve>(s, Linear, Guide, Hit, width, height, x0, y0, tid);
  const int i0 = (y0 + 2 * (int)threadIdx.y) * width + x0 + (int)threadIdx.x;
  const CentreGlobal ctr{Linear, Guide, Hit, i0, width};
  filter_finish<kResolve>(s, unpacked, ctr, Linear, Guide, Hit, Filtered, History, Pixels, c9, c10, c15, c20, width, height, x0, y0);
}

}  // namespace
}  // namespace arbor
