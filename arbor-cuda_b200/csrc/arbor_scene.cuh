// arbor_scene.cuh - surface fields, intersections and BVH traversal.
//
// Device restatement of the reference's surface/trace functions
// (Arbor.cu:132-133, 148-174, 186-251).  Per-primitive invariants (frames,
// seed hashes, column counts, footprint band weights) are hoisted out of the
// march / Newton loops; each hoisted value is the exact value the reference
// recomputes on every iteration, so results are unchanged.
#pragma once
#include "arbor_math.cuh"

// Work-event hooks.  They compile to nothing in the product kernels; the
// work-counting translation unit (count.cu) defines ARBOR_COUNT before
// including this header to tally the events the trace roofline model weighs.
#ifndef ARBOR_COUNT
#define ARBOR_COUNT(event) ((void)0)
#endif

namespace arbor {

enum WorkEvent {
  kEvRay = 0,          // primary ray set up
  kEvCell = 1,         // forest DDA cell with its bounding-sphere test
  kEvTree = 2,         // tree entered (local transform + root test)
  kEvNode = 3,         // BVH node box test
  kEvWood = 4,         // primary wood test (frame, tube, bounds)
  kEvMarch = 5,        // SDF march step (one woodField)
  kEvBarkFull = 6,     // bark relief past its footprint early-out
  kEvWoodShadow = 7,   // shadow-ray wood tube test
  kEvLeaf = 8,         // leaf test (frame, petiole tube, box clip)
  kEvNewtonStart = 9,  // leaf test that reaches the Newton solve
  kEvNewton = 10,      // Newton iteration (five height-field evaluations)
  kEvStone = 11,       // stone ellipsoid test
  kEvSegment = 12,     // shadow-ray segment toward the sun (forest or tree trace set up)
  kEvCount = 13
};

// ------------------------------------------------------------ records --
__device__ __forceinline__ float4 ldg4(const float* base, int index4) {
  return __ldg(reinterpret_cast<const float4*>(base) + index4);
}

// Per-type bounds (Arbor.cu:132-133) from the first five floats of interest.
__device__ __forceinline__ void prim_bounds(float4 r0, float4 r1, float p7, float p11, float p16, f3& lo, f3& hi) {
  int type = (int)r0.w;
  if (type < 0) {
    lo = mk(kFar, kFar, kFar);
    hi = mk(-kFar, -kFar, -kFar);
    return;
  }
  f3 a = xyz(r0);
  f3 b = xyz(r1);
  if (type == 0) {
    float r = fmaxf(p7, p11) + 0.002f;
    lo = min3(a, b) - mk(r, r, r);
    hi = max3(a, b) + mk(r, r, r);
    return;
  }
  if (type == 2) {
    lo = a - b;
    hi = a + b;
    return;
  }
  float radius = p7 + p16 + 0.025f;
  lo = a - mk(radius, radius, radius);
  hi = a + mk(radius, radius, radius);
}

// --------------------------------------------------------------- wood --
struct Wood {
  f3 a, end, ab;
  float abab, ra, rb;
  // bark frame and constants (woodUV / barkCut, Arbor.cu:148-151)
  f3 d, u, v;
  float arc0;
  int columns, seed;
  uint32_t hs, hs31, hs731;
};
__device__ __forceinline__ Wood load_wood(const float* P, int id) {
  float4 r0 = ldg4(P, id * 6 + 0), r1 = ldg4(P, id * 6 + 1), r2 = ldg4(P, id * 6 + 2);
  float4 r3 = ldg4(P, id * 6 + 3), r4 = ldg4(P, id * 6 + 4);
  Wood w;
  w.a = xyz(r0);
  w.end = xyz(r1);
  w.ra = r1.w;
  w.rb = r2.w;
  w.ab = w.end - w.a;
  w.abab = dot3(w.ab, w.ab);
  f3 initial = xyz(r2);
  w.d = norm3(w.end - w.a);
  w.u = norm3(initial - w.d * dot3(initial, w.d));
  w.v = cross3(w.d, w.u);
  w.arc0 = r4.x;                       // P[b+16]
  w.seed = (int)r3.w;                  // P[b+15]
  w.columns = (int)fmaxf(7.0f, floorf(r4.z * 2.0f * kPi / 0.065f + 0.5f));  // P[b+18]
  w.hs = hashU((uint32_t)w.seed);
  w.hs31 = hashU((uint32_t)(w.seed + 31));
  w.hs731 = hashU((uint32_t)(w.seed + 731));
  return w;
}
// Voronoi bark relief (Arbor.cu:149-169).  fine/grain are the footprint
// band weights of the 10 mm and 2.5 mm bands (constant per call).
// kMarch: the SDF march of the intersection test, whose angular terms take
// the hardware sine/cosine (below); shading and normals (kMarch false) keep
// the accurate functions.
template <bool kMarch = false>
__device__ __forceinline__ float bark_cut(const Wood& w, f3 p, float fp, float fine, float grain) {
  f3 pa = p - w.a;
  float along = sat(dot3(pa, w.ab) / fmaxf(0.000001f, w.abab));
  float radius = lerpf(w.ra, w.rb, along);
  float amp = fminf(0.021f, radius * 0.055f);
  float period = radius * 2.0f * kPi / (float)w.columns;
  float coarse = band_weight(period, fp);
  if (coarse < 0.000001f && fine < 0.000001f) return amp * 0.32f;
  ARBOR_COUNT(kEvBarkFull);
  float z = dot3(pa, w.d);
  float theta = atan2f(dot3(pa, w.v), dot3(pa, w.u));
  float arc = w.arc0 + z;
  // In the march the relief's angular terms use the hardware sine/cosine
  // (absolute error about 2^-21 per unit of argument magnitude: below 1e-4
  // for the arguments here, |x| < 700): they shift the Voronoi plates by far
  // less than a footprint, and the relief enters the SDF scaled by
  // amp <= 0.021.  The whole-frame IDs and distances stay within the
  // contract (tests pin them).
  float st, ct, x, y;
  if (kMarch) {
    st = __sinf(theta);
    ct = __cosf(theta);
    x = (theta / (2.0f * kPi) + 0.5f) * (float)w.columns + 0.32f * __sinf(arc * 6.7f + ct * 3.0f) + 0.15f * __sinf(arc * 19.0f + st * 2.0f);
    y = arc / 0.19f + 0.25f * __sinf(theta * 7.0f) + 0.1f * __sinf(theta * 19.0f);
  } else {
    st = sinf(theta);
    ct = cosf(theta);
    x = (theta / (2.0f * kPi) + 0.5f) * (float)w.columns + 0.32f * sinf(arc * 6.7f + ct * 3.0f) + 0.15f * sinf(arc * 19.0f + st * 2.0f);
    y = arc / 0.19f + 0.25f * sinf(theta * 7.0f) + 0.1f * sinf(theta * 19.0f);
  }
  int ix = (int)floorf(x);
  int iy = (int)floorf(y);
  int wrapped[3];
#pragma unroll
  for (int k = -1; k <= 1; k++) {
    int cell = ix + k;
    wrapped[k + 1] = ((cell % w.columns) + w.columns) % w.columns;
  }
  float first = 100.0f, second = 100.0f;
#pragma unroll
  for (int j = -1; j <= 1; j++) {
#pragma unroll
    for (int k = -1; k <= 1; k++) {
      int cell = ix + k;
      int wr = wrapped[k + 1];
      float xx = (float)cell + 0.18f + 0.64f * rndh(hcell(wr, iy + j), w.hs) - x;
      float yy = (float)(iy + j) + 0.18f + 0.64f * rndh(hcell(wr + w.columns, iy + j), w.hs31) - y;
      float dd = xx * xx + yy * yy;
      if (dd < first) {
        second = first;
        first = dd;
      } else if (dd < second) {
        second = dd;
      }
    }
  }
  float gap = sqrtf(second) - sqrtf(first);
  float fissure = 1.0f - smooth(0.015f, 0.17f, gap);
  float plates = fissure * fissure;
  f3 coord = mk(ct * 9.0f, st * 9.0f, arc * 23.0f);
  float splinter = noise3(coord, w.seed);
  float pores = noise3(coord * 4.0f, w.seed + 731);
  return amp * clampf(0.32f + coarse * (plates - 0.37f) * 0.69f + fine * (splinter - 0.5f) * 0.24f + grain * (pores - 0.5f) * 0.08f, 0.005f, 1.0f);
}
// Wood SDF (Arbor.cu:170).
template <bool kMarch = false>
__device__ __forceinline__ float wood_field(const Wood& w, f3 p, float fp, float fine, float grain) {
  float t = sat(dot3(p - w.a, w.ab) / fmaxf(0.0000001f, w.abab));
  float radius = lerpf(w.ra, w.rb, t);
  return length3(p - w.a - w.ab * t) - radius + bark_cut<kMarch>(w, p, fp, fine, grain);
}

// --------------------------------------------------------------- leaf --
struct Leaf {
  f3 origin, u, v, n;
  float stem, len, width, curl, twist;
  int seed;  // P[b+15]
};
// Wind-rotated frame (Arbor.cu:171-172).
__device__ __forceinline__ Leaf load_leaf(const float* P, int id, float time, float wind) {
  float4 r0 = ldg4(P, id * 6 + 0), r1 = ldg4(P, id * 6 + 1), r2 = ldg4(P, id * 6 + 2);
  float4 r3 = ldg4(P, id * 6 + 3), r4 = ldg4(P, id * 6 + 4);
  Leaf l;
  l.origin = xyz(r0);
  f3 u = xyz(r1);
  f3 n = xyz(r3);
  l.len = r1.w;
  l.v = xyz(r2);
  l.width = r2.w;
  l.seed = (int)r3.w;
  l.stem = r4.x;
  l.curl = r4.y;
  l.twist = r4.z;
  if (wind == 0.0f) {
    // Still air: the rotation angle is wind * (finite) = +-0, so cos = 1 and
    // sin = +-0 and the reference's u*cos + n*sin, n*cos - u*sin are u and n
    // exactly (up to the sign of a zero component).
    l.u = u;
    l.n = n;
    return l;
  }
  float phase = (float)(l.seed % 8192) * 0.618f;
  float a = wind * (0.11f * sinf(time * 2.1f + phase) + 0.045f * sinf(time * 5.8f + phase * 1.7f));
  float ca = cosf(a), sa = sinf(a);
  l.u = u * ca + n * sa;
  l.n = n * ca - u * sa;
  return l;
}
// Leaf outline (Arbor.cu:173); bw002 = band_weight(0.002, fp).
__device__ __forceinline__ float leaf_width(float u, float length, float halfWidth, float bw002) {
  float q = sat(u / length);
  float s = sinf(kPi * q);
  float lobes = 0.77f + 0.23f * cosf(q * kPi * 10.0f + 0.45f);
  float fine = bw002 * 0.015f * sinf(q * kPi * 160.0f);
  return halfWidth * powf(fmaxf(0.0f, s), 0.72f) * (lobes + fine);
}
// Leaf height field (Arbor.cu:174); bw007 = band_weight(0.007, fp),
// hw2 = halfWidth * halfWidth.
__device__ __forceinline__ float leaf_height(float u, float v, float len, float hw2, float curl, float twist, float bw007) {
  float q = clampf(u / len, -0.2f, 1.2f);
  float s = sinf(kPi * q);
  float coarse = curl * s + twist * (q - 0.4f) * v + 0.009f * (v * v / hw2) * s;
  float mid = 0.0012f * expf(-fabsf(v) / 0.005f) * s * bw007;
  return coarse + mid;
}
// leaf_height in parts, for the Newton stage's five evaluations at
// (u, v), (u +- e, v), (u, v +- e): the along-blade terms of one u and the
// across-blade terms of one v are each computed once and shared.  Each
// height is assembled with exactly leaf_height's operations.  The iterations
// take the hardware sine and exponential (absolute errors near 1e-6 for these
// arguments, |x| < 4, against a height scale of centimetres); they only steer
// the iterate - the acceptance test at the end (leaf_height, leaf_width)
// evaluates the accurate functions.
struct LeafU {
  float q, s;
};
struct LeafV {
  float vv, ev;  // v * v / hw2, expf(-|v| / 0.005)
};
__device__ __forceinline__ LeafU leaf_u(float u, float len) {
  const float q = clampf(u / len, -0.2f, 1.2f);
  return {q, __sinf(kPi * q)};
}
__device__ __forceinline__ LeafV leaf_v(float v, float hw2) { return {v * v / hw2, __expf(-fabsf(v) / 0.005f)}; }
__device__ __forceinline__ float leaf_height_parts(const LeafU& a, float v, const LeafV& b, float curl, float twist, float bw007) {
  float coarse = curl * a.s + twist * (a.q - 0.4f) * v + 0.009f * b.vv * a.s;
  float mid = 0.0012f * b.ev * a.s * bw007;
  return coarse + mid;
}

// ------------------------------------------------------- intersections --
// Arbor.cu:186
__device__ __forceinline__ float sphere_t(f3 ro, f3 rd, f3 p, float radius) {
  f3 q = ro - p;
  float b = dot3(q, rd);
  float c = dot3(q, q) - radius * radius;
  float d = b * b - c;
  if (d < 0.0f) return kFar;
  float t = -b - sqrtf(d);
  if (t <= 0.0001f) t = -b + sqrtf(d);
  return t > 0.0001f ? t : kFar;
}
// Tapered tube plus joint caps (Arbor.cu:188-191).
__device__ __forceinline__ float tube_t(f3 ro, f3 rd, f3 a, f3 b, float ra, float rb) {
  f3 axis = b - a;
  float len = length3(axis);
  axis = axis / fmaxf(len, 0.000001f);
  f3 q = ro - a;
  float z = dot3(q, axis);
  float dz = dot3(rd, axis);
  float k = (rb - ra) / fmaxf(0.000001f, len);
  f3 v = q - axis * z;
  f3 d = rd - axis * dz;
  float radius = ra + k * z;
  float aa = dot3(d, d) - k * k * dz * dz;
  float bb = dot3(v, d) - radius * k * dz;
  float cc = dot3(v, v) - radius * radius;
  float best = fminf(sphere_t(ro, rd, a, ra), sphere_t(ro, rd, b, rb));
  float disc = bb * bb - aa * cc;
  if (disc >= 0.0f && fabsf(aa) > 0.0000001f) {
    float sq = sqrtf(disc);
#pragma unroll
    for (int j = 0; j < 2; j++) {
      float t = (-bb + (j == 0 ? -1.0f : 1.0f) * sq) / aa;
      float h = z + t * dz;
      if (t > 0.0001f && h >= 0.0f && h <= len) best = fminf(best, t);
    }
  }
  return best;
}
// Wood hit (Arbor.cu:192-202): mean-radius tube for shadow rays, bounded
// SDF march seeded by the analytic tube for primary rays.
static __device__ __noinline__ float wood_t(const float* P, int id, f3 ro, f3 rd, float footprint, bool refine) {
  if (!refine) {
    ARBOR_COUNT(kEvWoodShadow);
    float4 r0 = ldg4(P, id * 6 + 0), r1 = ldg4(P, id * 6 + 1), r2 = ldg4(P, id * 6 + 2);
    float p7 = r1.w, p11 = r2.w;
    float ra = p7 - fminf(0.021f, p7 * 0.055f) * 0.32f;
    float rb = p11 - fminf(0.021f, p11 * 0.055f) * 0.32f;
    return tube_t(ro, rd, xyz(r0), xyz(r1), ra, rb);
  }
  ARBOR_COUNT(kEvWood);
  Wood w = load_wood(P, id);
  float t = tube_t(ro, rd, w.a, w.end, w.ra, w.rb);
  if (t >= kFar) return kFar;
  f3 lo, hi;
  {
    float r = fmaxf(w.ra, w.rb) + 0.002f;
    lo = min3(w.a, w.end) - mk(r, r, r);
    hi = max3(w.a, w.end) + mk(r, r, r);
  }
  f2 span = box_span(ro, rd, lo, hi);
  float eps = fmaxf(0.000025f, fminf(0.00025f, footprint * 0.13f));
  float fine = band_weight(0.010f, footprint);
  float grain = band_weight(0.0025f, footprint);
  for (int k = 0; k < 64; k++) {
    ARBOR_COUNT(kEvMarch);
    float f = wood_field<true>(w, ro + rd * t, footprint, fine, grain);
    if (f < eps) return t;
    t += fmaxf(eps * 0.35f, f * 0.27f);
    if (t > span.y) return kFar;
  }
  return kFar;
}
// Curved-leaf intersection (Arbor.cu:203-218), in two parts so the
// wavefront tracer can run them as separate compacted stages: leaf_clip does
// the frame, the petiole tube and the leaf-box clip; leaf_newton does the
// seven Newton steps and the acceptance test.  leaf_t chains them and is the
// reference's leafT.
struct LeafSolve {
  float x, y, z, dx, dy, dz;  // ray in the leaf frame
  float t, spanx, spany;      // Newton start and the clipped interval
};
// The leaf's blade shape (P[b+7], P[b+11], P[b+17], P[b+18]), re-read by
// the Newton stage from the record rather than carried with the solve.
struct LeafShape {
  float len, width, curl, twist;
};
__device__ __forceinline__ LeafShape leaf_shape(const float* P, int id) {
  return {__ldg(P + id * 24 + 7), __ldg(P + id * 24 + 11), __ldg(P + id * 24 + 17), __ldg(P + id * 24 + 18)};
}
// `tube` is the petiole tube's result.  Returns true when the leaf box is hit
// and the Newton solve must run; otherwise the result is `tube`.
__device__ __forceinline__ bool leaf_clip(const float* P, int id, f3 ro, f3 rd, float time, float wind, LeafSolve& s, float& tube) {
  ARBOR_COUNT(kEvLeaf);
  Leaf l = load_leaf(P, id, time, wind);
  f3 q = ro - l.origin;
  s.x = dot3(q, l.u) - l.stem;
  s.y = dot3(q, l.v);
  s.z = dot3(q, l.n);
  s.dx = dot3(rd, l.u);
  s.dy = dot3(rd, l.v);
  s.dz = dot3(rd, l.n);
  tube = tube_t(ro, rd, l.origin, l.origin + l.u * l.stem, 0.0011f, 0.00065f);
  f2 span = box_span(mk(s.x, s.y, s.z), mk(s.dx, s.dy, s.dz), mk(-0.001f, -l.width, -0.035f), mk(l.len + 0.001f, l.width, 0.065f));
  if (span.y < fmaxf(0.0001f, span.x)) return false;
  ARBOR_COUNT(kEvNewtonStart);
  float t = fabsf(s.dz) > 0.000001f ? -s.z / s.dz : (span.x + span.y) * 0.5f;
  s.t = clampf(t, fmaxf(0.0001f, span.x), span.y);
  s.spanx = span.x;
  s.spany = span.y;
  return true;
}
// leaf_clip out of line, for the primary-ray passes: a smaller warp loop
// there (1080p trace 11.0 -> 10.5 ms); the shadow-segment passes keep it
// inlined (out of line they ran 3x slower).
static __device__ __noinline__ bool leaf_clip_outlined(const float* P, int id, f3 ro, f3 rd, float time, float wind, LeafSolve& s, float& tube) {
  return leaf_clip(P, id, ro, rd, time, wind, s, tube);
}
// The Newton stage; `best` is the petiole tube's result.
__device__ __forceinline__ float leaf_newton(const LeafSolve& s, const LeafShape& sh, float best, float footprint) {
  const float x = s.x, y = s.y, z = s.z, dx = s.dx, dy = s.dy, dz = s.dz;
  float t = s.t;
  float hw2 = sh.width * sh.width;
  float bw007 = band_weight(0.007f, footprint);
  for (int k = 0; k < 7; k++) {
    ARBOR_COUNT(kEvNewton);
    float xx = x + dx * t;
    float yy = y + dy * t;
    const float e = 0.00015f;
    const LeafU u0 = leaf_u(xx, sh.len), up = leaf_u(xx + e, sh.len), um = leaf_u(xx - e, sh.len);
    const LeafV v0 = leaf_v(yy, hw2), vp = leaf_v(yy + e, hw2), vm = leaf_v(yy - e, hw2);
    float height = leaf_height_parts(u0, yy, v0, sh.curl, sh.twist, bw007);
    float f = z + dz * t - height;
    float hx = (leaf_height_parts(up, yy, v0, sh.curl, sh.twist, bw007) - leaf_height_parts(um, yy, v0, sh.curl, sh.twist, bw007)) / (2.0f * e);
    float hy = (leaf_height_parts(u0, yy + e, vp, sh.curl, sh.twist, bw007) - leaf_height_parts(u0, yy - e, vm, sh.curl, sh.twist, bw007)) / (2.0f * e);
    float deriv = dz - hx * dx - hy * dy;
    if (fabsf(deriv) < 0.00001f) break;
    t -= clampf(f / deriv, -0.13f, 0.13f);
    t = clampf(t, s.spanx, s.spany);
  }
  float xx = x + dx * t;
  float yy = y + dy * t;
  float err = fabsf(z + dz * t - leaf_height(xx, yy, sh.len, hw2, sh.curl, sh.twist, bw007));
  if (t > 0.0001f && xx > 0.0f && xx < sh.len && err < 0.0003f && fabsf(yy) < leaf_width(xx, sh.len, sh.width, band_weight(0.002f, footprint)))
    best = fminf(best, t);
  return best;
}
static __device__ __noinline__ float leaf_t(const float* P, int id, f3 ro, f3 rd, float footprint, float time, float wind) {
  LeafSolve s;
  float tube;
  if (!leaf_clip(P, id, ro, rd, time, wind, s, tube)) return tube;
  return leaf_newton(s, leaf_shape(P, id), tube, footprint);
}
// Arbor.cu:219
__device__ __forceinline__ float object_t(const float* P, int id, f3 ro, f3 rd, float footprint, float time, float wind, bool refine) {
  float4 r0 = ldg4(P, id * 6 + 0);
  int type = (int)r0.w;
  if (type < 0) return kFar;
  if (type == 0) return wood_t(P, id, ro, rd, footprint, refine);
  if (type == 1) return leaf_t(P, id, ro, rd, footprint, time, wind);
  ARBOR_COUNT(kEvStone);
  f3 h = xyz(ldg4(P, id * 6 + 1));
  f3 q = ro - xyz(r0);
  f3 p = mk(q.x / h.x, q.y / h.y, q.z / h.z);
  f3 d = mk(rd.x / h.x, rd.y / h.y, rd.z / h.z);
  float aa = dot3(d, d);
  float bb = dot3(p, d);
  float cc = dot3(p, p) - 1.0f;
  float disc = bb * bb - aa * cc;
  if (disc < 0.0f) return kFar;
  float t = (-bb - sqrtf(disc)) / aa;
  return t > 0.0001f ? t : kFar;
}

// -------------------------------------------------------- traversal --
// Heap-BVH traversal with the reference's visiting order (Arbor.cu:220-230):
// nearest hit child first, the other deferred, a node accepted when its
// count is positive, span.y >= max(1e-4, span.x) and span.x < best.
//
// The reference keeps deferred nodes on a 32-entry stack and re-tests each
// popped node against the current best.  In a heap-indexed tree the deferred
// node at depth L is always the sibling of the current path's depth-L
// ancestor, so one bit per depth (`pending`) replaces the stack: popping the
// deepest pending bit yields exactly the node the stack would pop, and the
// popped node is re-tested the same way.  No local memory is used.
//
// A child reached by descent is not re-tested: the reference's re-test of it
// repeats the child test just made with the same best, so it always passes;
// its span.x (the leaf footprint input) is carried instead.
__device__ __forceinline__ bool node_accept_span(float4 lo, float4 hi, f3 ro, f3 inv, float best, f2& s) {
  ARBOR_COUNT(kEvNode);
  s = box_span_inv(ro, inv, xyz(lo), xyz(hi));
  return lo.w > 0.0f && s.y >= fmaxf(0.0001f, s.x) && s.x < best;
}
__device__ __forceinline__ bool node_accept(float4 lo, float4 hi, f3 ro, f3 inv, float best, float& spanx) {
  f2 s;
  const bool ok = node_accept_span(lo, hi, ro, inv, best, s);
  spanx = s.x;
  return ok;
}
__device__ __forceinline__ f2 trace_tree(const float* P, const float* Nodes, const uint32_t* Order, f3 ro, f3 rd, float cone, float time,
                                         float wind, float best, int ignore, bool shadows) {
  const f3 inv = inv3(rd);
  int found = -1;
  int node = 1;
  int depth = 0;
  uint32_t pending = 0;
  float spanx;
  if (!node_accept(ldg4(Nodes, 2), ldg4(Nodes, 3), ro, inv, best, spanx)) return {best, -1.0f};
  for (int visit = 1; visit < kNodeCount; visit++) {
    bool descended = false;
    if (node < kCapacity) {
      int left = node * 2;
      float4 llo = ldg4(Nodes, left * 2), lhi = ldg4(Nodes, left * 2 + 1);
      float4 rlo = ldg4(Nodes, left * 2 + 2), rhi = ldg4(Nodes, left * 2 + 3);
      float lx, rx;
      bool lh = node_accept(llo, lhi, ro, inv, best, lx);
      bool rh = node_accept(rlo, rhi, ro, inv, best, rx);
      if (lh || rh) {
        depth++;
        if (lh && rh) {
          bool l = lx < rx;
          pending |= 1u << depth;
          node = l ? left : left + 1;
          spanx = l ? lx : rx;
        } else if (lh) {
          node = left;
          spanx = lx;
        } else {
          node = left + 1;
          spanx = rx;
        }
        descended = true;
      }
    } else {
      uint32_t uid = __ldg(Order + (node - kCapacity));
      int id = (int)uid;
      // An Order entry past the 32768 records (invalid input) is skipped
      // rather than read out of bounds.
      if (id != ignore && uid < (uint32_t)kCapacity) {
        float footprint = fmaxf(0.000005f, cone * fmaxf(0.05f, spanx));
        float t = object_t(P, id, ro, rd, footprint, time, wind, !shadows);
        if (t < best) {
          best = t;
          found = id;
        }
      }
    }
    if (descended) continue;
    // Pop deferred siblings, deepest first, until one is still accepted.
    bool resumed = false;
    while (pending != 0u && visit < kNodeCount) {
      int level = 31 - __clz(pending);
      pending &= ~(1u << level);
      node = (node >> (depth - level)) ^ 1;
      depth = level;
      visit++;
      if (node_accept(ldg4(Nodes, node * 2), ldg4(Nodes, node * 2 + 1), ro, inv, best, spanx)) {
        resumed = true;
        break;
      }
    }
    if (!resumed) break;
  }
  return {best, (float)found};
}

// Forest 2D DDA (Arbor.cu:235-251) over a per-block instance table.
__device__ __forceinline__ f2 trace_forest(const float* P, const float* Nodes, const uint32_t* Order, const Instance* inst, f3 ro, f3 rd,
                                           float cone, float time, float wind, float best, int* treeOut, bool shadows) {
  int foundTree = -1;
  float found = -1.0f;
  const float half = (float)kSide * kSpacing * 0.5f;
  f2 worldSpan = box_span(ro, rd, mk(-half, -1.2f, -half), mk(half, 13.5f, half));
  float enter = fmaxf(0.0f, worldSpan.x);
  float exit = fminf(best, worldSpan.y);
  if (exit < enter) {
    *treeOut = -1;
    return {best, -1.0f};
  }
  f3 pos = ro + rd * (enter + 0.0002f);
  int ix = (int)floorf(pos.x / kSpacing + (float)kSide * 0.5f + 0.5f);
  int iz = (int)floorf(pos.z / kSpacing + (float)kSide * 0.5f + 0.5f);
  int sx = rd.x >= 0.0f ? 1 : -1;
  int sz = rd.z >= 0.0f ? 1 : -1;
  float invx = inv_safe(rd.x);
  float invz = inv_safe(rd.z);
  float bx = ((float)(ix - kSide / 2) + (sx > 0 ? 0.5f : -0.5f)) * kSpacing;
  float bz = ((float)(iz - kSide / 2) + (sz > 0 ? 0.5f : -0.5f)) * kSpacing;
  float tx = (bx - ro.x) * invx;
  float tz = (bz - ro.z) * invz;
  float dx = kSpacing * fabsf(invx);
  float dz = kSpacing * fabsf(invz);
  for (int step = 0; step < 48; step++) {
    if (ix < 0 || iz < 0 || ix >= kSide || iz >= kSide) break;
    int tree = iz * kSide + ix;
    ARBOR_COUNT(kEvCell);
    const Instance& it = inst[tree];
    float broad = sphere_t(ro, rd, mk(it.px + 0.0f, 0.0f + it.cy, it.pz + 0.0f), it.rad);
    if (broad < best) {
      ARBOR_COUNT(kEvTree);
      f3 lr = to_local_point(ro, it);
      f3 ld = to_local_dir(rd, it);
      f2 h = trace_tree(P, Nodes, Order, lr, ld, cone / it.sc, time + it.phase, wind, best / it.sc, -1, shadows);
      if (h.y >= 0.0f && h.x * it.sc < best) {
        best = h.x * it.sc;
        found = h.y;
        foundTree = tree;
      }
    }
    float next = tx < tz ? tx : tz;
    if (next > exit || next > best) break;
    if (tx < tz) {
      ix += sx;
      tx += dx;
    } else {
      iz += sz;
      tz += dz;
    }
  }
  *treeOut = foundTree;
  return {best, found};
}

}  // namespace arbor
