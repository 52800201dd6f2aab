/*
 * TEST INFRASTRUCTURE ONLY - the CPU oracle for the Arbor render path.
 *
 * A plain-C restatement of the reference's per-thread CUDA-C math
 * (reference: Arbor.cu, which is kernels/{common,tree,cache,surface,camera,
 * trace,shade}.cu concatenated) executed as scalar loops on the host, the way
 * tests/native_harness.cpp:35-39 executes it.  Every function cites the
 * reference line it restates.  The operation order of each floating-point
 * expression follows the reference exactly, because bit-identical results
 * against the reference harness (built from its own sources into oracle/_ref
 * by oracle/Makefile) are the pin for this file.
 *
 * Two instantiations are built from this one file:
 *   liboracle.so    real == float   (bit-exact restatement, -ffp-contract=off)
 *   liboracle64.so  real == double  (the FP64 rerun of the same formulas; the
 *                                    constants stay the reference's f32 values,
 *                                    buffers stay f32)
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * this code, and only as the checker.  No product path links it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_F64
typedef double real;
#define SQRT sqrt
#define SIN sin
#define COS cos
#define POW pow
#define EXP exp
#define ATAN2 atan2
#define FLOOR floor
#define FABS fabs
#define FMIN fmin
#define FMAX fmax
#else
typedef float real;
#define SQRT sqrtf
#define SIN sinf
#define COS cosf
#define POW powf
#define EXP expf
#define ATAN2 atan2f
#define FLOOR floorf
#define FABS fabsf
#define FMIN fminf
#define FMAX fmaxf
#endif

/* ABI constants (Arbor.cu:5-15, 54-56). */
#define K_PI 3.14159265359f
#define K_FAR 100000.0f
#define K_CAPACITY 32768
#define K_NODES 65536
#define K_PS 24
#define K_CS 20
#define K_WOOD 5124
#define K_LEAF 24192
#define K_ROCK 96
#define K_OBJECTS 29412
#define K_SIDE 18
#define K_SPACING 28.0f

typedef struct { real x, y, z; } v3;
typedef struct { real x, y; } v2;

static inline v3 V(real x, real y, real z) { v3 r = {x, y, z}; return r; }
static inline v2 V2(real x, real y) { v2 r = {x, y}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 vscale(v3 a, real s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 vdivs(v3 a, real s) { return V(a.x / s, a.y / s, a.z / s); }
/* Arbor.cu:17-31 */
static inline real clampr(real x, real a, real b) { return FMIN(b, FMAX(a, x)); }
static inline real sat(real x) { return clampr(x, 0.0f, 1.0f); }
static inline real lerpr(real a, real b, real t) { return a + (b - a) * t; }
static inline real fracr(real a) { return a - FLOOR(a); }
static inline real smoothr(real a, real b, real x) { real t = sat((x - a) / (b - a)); return t * t * (3.0f - 2.0f * t); }
static inline real dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline real len3(v3 a) { return SQRT(dot(a, a)); }
static inline v3 unit(v3 a) { return vdivs(a, FMAX(0.0000001f, len3(a))); }
static inline v3 vmin(v3 a, v3 b) { return V(FMIN(a.x, b.x), FMIN(a.y, b.y), FMIN(a.z, b.z)); }
static inline v3 vmax(v3 a, v3 b) { return V(FMAX(a.x, b.x), FMAX(a.y, b.y), FMAX(a.z, b.z)); }
static inline v3 mixv(v3 a, v3 b, real t) { return vadd(a, vscale(vsub(b, a), t)); }
static inline v3 ld3(const float* a, int i) { return V(a[i], a[i + 1], a[i + 2]); }
static inline void st3(float* a, int i, v3 v) { a[i] = (float)v.x; a[i + 1] = (float)v.y; a[i + 2] = (float)v.z; }

/* Integer hash and derived uniforms (Arbor.cu:32-34).  The products are taken
 * in unsigned arithmetic: the same bits as the reference's wrapping int
 * multiply, without signed-overflow UB in C. */
static inline uint32_t hashu(uint32_t x) { x ^= x >> 16; x *= 2146121005u; x ^= x >> 15; x *= 2221713035u; x ^= x >> 16; return x; }
static inline real rnd(int n, int seed) { return (real)(float)(hashu((uint32_t)n ^ hashu((uint32_t)seed)) & 16777215u) / 16777216.0f; }
static inline int imad(int a, int b, int c) { return (int)((uint32_t)a * (uint32_t)b + (uint32_t)c); }
static inline real hash2(int x, int y, int seed) { return rnd((int)((uint32_t)x * 1973u + (uint32_t)y * 9277u), seed); }
/* Value noise (Arbor.cu:35-36). */
static real noise2(real x, real y, int seed) {
  int ix = (int)FLOOR(x), iy = (int)FLOOR(y);
  real fx = fracr(x), fy = fracr(y);
  fx = fx * fx * (3.0f - 2.0f * fx);
  fy = fy * fy * (3.0f - 2.0f * fy);
  return lerpr(lerpr(hash2(ix, iy, seed), hash2(ix + 1, iy, seed), fx),
               lerpr(hash2(ix, iy + 1, seed), hash2(ix + 1, iy + 1, seed), fx), fy);
}
static real noise3(v3 p, int seed) {
  int iz = (int)FLOOR(p.z);
  real f = fracr(p.z);
  f = f * f * (3.0f - 2.0f * f);
  return lerpr(noise2(p.x, p.y, imad(iz, 131, seed)), noise2(p.x, p.y, imad(iz + 1, 131, seed)), f);
}
/* Slab test (Arbor.cu:37-38). */
static inline real inv_safe(real x) { return FABS(x) < 0.00000001f ? (x < 0.0f ? -100000000.0f : 100000000.0f) : 1.0f / x; }
static v2 box_span(v3 ro, v3 rd, v3 lo, v3 hi) {
  v3 inv = V(inv_safe(rd.x), inv_safe(rd.y), inv_safe(rd.z));
  v3 a = vmul(vsub(lo, ro), inv), b = vmul(vsub(hi, ro), inv);
  v3 mn = vmin(a, b), mx = vmax(a, b);
  return V2(FMAX(mn.x, FMAX(mn.y, mn.z)), FMIN(mx.x, FMIN(mx.y, mx.z)));
}
/* Arbor.cu:39 */
static inline v3 basis_u(v3 n) { return unit(cross(FABS(n.y) < 0.91f ? V(0.0f, 1.0f, 0.0f) : V(0.0f, 0.0f, 1.0f), n)); }
/* Cubic Bezier of curve `id` (Arbor.cu:40-42). */
static v3 bezier(const float* B, int id, real t) {
  int b = id * K_CS; real q = 1.0f - t;
  v3 r = vscale(ld3(B, b), q * q * q);
  r = vadd(r, vscale(ld3(B, b + 3), 3.0f * q * q * t));
  r = vadd(r, vscale(ld3(B, b + 6), 3.0f * q * t * t));
  return vadd(r, vscale(ld3(B, b + 9), t * t * t));
}
static v3 bezier_dir(const float* B, int id, real t) {
  int b = id * K_CS; real q = 1.0f - t;
  v3 r = vscale(vsub(ld3(B, b + 3), ld3(B, b)), q * q);
  r = vadd(r, vscale(vsub(ld3(B, b + 6), ld3(B, b + 3)), 2.0f * q * t));
  return unit(vadd(r, vscale(vsub(ld3(B, b + 9), ld3(B, b + 6)), t * t)));
}
static inline real bezier_radius(const float* B, int id, real t) { return lerpr(B[id * K_CS + 12], B[id * K_CS + 13], t); }
/* Footprint band weight (Arbor.cu:44). */
static inline real band(real period, real footprint) { return 1.0f - smoothr(period * 0.12f, period * 0.65f, footprint); }
/* Camera helpers (Arbor.cu:45-51). */
static inline v3 cam_pos(const float* C) { return ld3(C, 0); }
static inline v3 cam_fwd(const float* C) { return unit(vsub(ld3(C, 4), ld3(C, 0))); }
static inline v3 cam_right(const float* C) { return unit(cross(cam_fwd(C), V(0.0f, 1.0f, 0.0f))); }
static v3 sun_dir(const float* C) { return unit(V(COS(C[12]) * COS(C[13]), SIN(C[13]), SIN(C[12]) * COS(C[13]))); }
static uint32_t pack_rgba(v3 c) {
  uint32_t r = (uint32_t)(float)(sat(c.x) * 255.0f + 0.5f);
  uint32_t g = (uint32_t)(float)(sat(c.y) * 255.0f + 0.5f);
  uint32_t b = (uint32_t)(float)(sat(c.z) * 255.0f + 0.5f);
  return r | (g << 8) | (b << 16) | 4278190080u;
}
static real radical_inverse(int n, int base) {
  real f = 1.0f, r = 0.0f;
  for (int j = 0; j < 12; j++) { if (n <= 0) break; f /= (real)base; r += f * (real)(n % base); n /= base; }
  return r;
}
static v3 primary_dir(const float* C, int x, int y, int width, int height) {
  int sample = (int)C[9];
  real jx = radical_inverse(sample + 1, 2) - 0.5f, jy = radical_inverse(sample + 1, 3) - 0.5f;
  real u = ((real)x + 0.5f + jx - (real)width * 0.5f) / (real)height;
  real v = ((real)height * 0.5f - (real)y - 0.5f - jy) / (real)height;
  v3 f = cam_fwd(C), r = cam_right(C), up = cross(r, f);
  return unit(vadd(vadd(f, vscale(r, u * C[14])), vscale(up, v * C[14])));
}

/* Forest instancing (Arbor.cu:57-69). */
static inline int tree_seed(int tree, int ws) { return (int)(hashu((uint32_t)tree * 92821u + (uint32_t)ws * 68917u + 17u) & 1048575u); }
static v3 tree_pos(int tree, int ws) {
  int x = tree % K_SIDE - K_SIDE / 2, z = tree / K_SIDE - K_SIDE / 2, s = tree_seed(tree, ws);
  real jx = (rnd(1, s) - 0.5f) * 10.0f, jz = (rnd(2, s) - 0.5f) * 10.0f;
  real wx = (noise2((real)x * 0.19f, (real)z * 0.19f, ws + 311) - 0.5f) * 3.0f;
  real wz = (noise2((real)x * 0.19f + 17.0f, (real)z * 0.19f - 9.0f, ws + 733) - 0.5f) * 3.0f;
  return V((real)x * K_SPACING + jx + wx, 0.0f, (real)z * K_SPACING + jz + wz);
}
static inline real tree_scale(int tree, int ws) { return 0.72f + rnd(3, tree_seed(tree, ws)) * 0.62f; }
static inline real tree_yaw(int tree, int ws) { return rnd(4, tree_seed(tree, ws)) * K_PI * 2.0f; }
static v3 to_local_point(v3 p, int tree, int ws) {
  v3 q = vsub(p, tree_pos(tree, ws)); real a = -tree_yaw(tree, ws); real c = COS(a), s = SIN(a); real sc = tree_scale(tree, ws);
  return vdivs(V(q.x * c - q.z * s, q.y, q.x * s + q.z * c), sc);
}
static v3 to_local_dir(v3 d, int tree, int ws) {
  real a = -tree_yaw(tree, ws); real c = COS(a), s = SIN(a);
  return unit(V(d.x * c - d.z * s, d.y, d.x * s + d.z * c));
}
static v3 to_world_normal(v3 n, int tree, int ws) {
  real a = tree_yaw(tree, ws); real c = COS(a), s = SIN(a);
  return unit(V(n.x * c - n.z * s, n.y, n.x * s + n.z * c));
}

/* ---------------------------------------------------------------- TREE -- */
/* Arbor.cu:75 */
static void put_curve(float* B, int id, v3 a, v3 b, v3 c, v3 d, real ra, real rb, real arc, int seed) {
  int o = id * K_CS;
  st3(B, o, a); st3(B, o + 3, b); st3(B, o + 6, c); st3(B, o + 9, d);
  B[o + 12] = (float)ra; B[o + 13] = (float)rb; B[o + 14] = (float)arc; B[o + 15] = (float)seed; B[o + 16] = (float)len3(vsub(d, a));
}
/* One thread of growTree (Arbor.cu:76-102). */
static void grow_one(float* B, int level, int seed, int i) {
  if (level == 0) {
    if (i == 0) put_curve(B, 0, V(0.0f, -0.15f, 0.0f), V(-0.22f, 1.1f, 0.16f), V(0.23f, 2.9f, -0.19f), V(0.04f, 4.2f, 0.05f), 0.68f, 0.23f, 0.0f, seed);
    if (i < 8) {
      real a = (real)i * K_PI * 0.25f + (rnd(i, seed) - 0.5f) * 0.5f;
      v3 d = V(COS(a), 0.0f, SIN(a));
      real len = 2.0f + rnd(i + 10, seed) * 1.4f;
      v3 p = vadd(vscale(d, 0.32f), V(0.0f, 0.27f, 0.0f));
      put_curve(B, i + 1, p, vadd(vscale(d, 0.8f), V(0.0f, 0.10f, 0.0f)), vadd(vscale(d, len * 0.68f), V(0.0f, -0.06f, 0.0f)),
                vadd(vscale(d, len), V(0.0f, -0.16f, 0.0f)), 0.235f, 0.012f, 0.0f, seed + i * 37);
    }
    return;
  }
  if (level == 1 && i < 12) {
    real t = 0.31f + 0.65f * (real)i / 11.0f;
    real a = (real)i * 2.399963f + 0.31f;
    real r = rnd(i + 37, seed);
    real len = 3.2f + 2.1f * r;
    v3 base = bezier(B, 0, t);
    v3 d = V(COS(a), 0.0f, SIN(a));
    v3 side = V(-d.z, 0.0f, d.x);
    v3 end = vadd(vadd(vadd(base, vscale(d, len * (0.87f - 0.30f * t))), V(0.0f, len * (0.60f + 0.40f * t), 0.0f)), vscale(side, (r - 0.5f) * 1.2f));
    real ra = bezier_radius(B, 0, t) * (0.46f + 0.13f * r);
    put_curve(B, 9 + i, base, vadd(vadd(base, vscale(d, len * 0.29f)), V(0.0f, len * 0.12f, 0.0f)),
              vsub(vsub(end, vscale(d, len * 0.17f)), V(0.0f, len * 0.26f, 0.0f)), end, ra, ra * 0.14f, B[14] + t * 4.2f, seed + i * 19);
    return;
  }
  int count = level == 2 ? 72 : (level == 3 ? 288 : 1728);
  if (i >= count) return;
  int children = level == 2 ? 6 : (level == 3 ? 4 : 6);
  int offset = level == 2 ? 21 : (level == 3 ? 93 : 381);
  int parent_offset = level == 2 ? 9 : (level == 3 ? 21 : 93);
  int parent = parent_offset + i / children, child = i % children;
  real h = rnd(i + level * 730, seed);
  real t = 0.23f + 0.72f * ((real)child + 0.35f) / (real)children;
  v3 p = bezier(B, parent, t), tangent = bezier_dir(B, parent, t);
  v3 u = basis_u(tangent), v = cross(tangent, u);
  real angle = (real)child * 2.399963f + h * 0.8f;
  v3 lateral = vadd(vscale(u, COS(angle)), vscale(v, SIN(angle)));
  v3 d = unit(vadd(vadd(vscale(tangent, 0.52f), vscale(lateral, level == 4 ? 0.64f : 0.80f)), V(0.0f, 0.26f, 0.0f)));
  real len = level == 2 ? 1.65f + 1.10f * h : (level == 3 ? 0.85f + 0.65f * h : 0.43f + 0.37f * h);
  len *= 0.84f + 0.25f * (1.0f - t);
  v3 end = vadd(vadd(p, vscale(d, len)), V(0.0f, len * 0.16f, 0.0f));
  real radius = bezier_radius(B, parent, t) * (level == 4 ? 0.30f : 0.40f);
  radius = FMAX(level == 4 ? 0.0035f : 0.008f, radius);
  put_curve(B, offset + i, p, vadd(vadd(p, vscale(tangent, len * 0.25f)), vscale(lateral, len * 0.11f)),
            vadd(vsub(end, vscale(d, len * 0.28f)), V(0.0f, len * 0.05f, 0.0f)), end, radius,
            radius * (level == 4 ? 0.30f : 0.22f), B[parent * K_CS + 14] + t * B[parent * K_CS + 16], seed + (offset + i) * 31);
}
/* One thread of makePrimitives (Arbor.cu:103-131). */
static void prim_one(const float* B, float* P, int seed, int i) {
  int b = i * K_PS;
  for (int j = 0; j < K_PS; j++) P[b + j] = 0.0f;
  P[b + 3] = -1.0f;
  if (i >= K_OBJECTS) return;
  if (i < K_WOOD) {
    int c, seg, segs;
    if (i < 12) { c = 0; seg = i; segs = 12; }
    else if (i < 60) { c = 1 + (i - 12) / 6; seg = (i - 12) % 6; segs = 6; }
    else if (i < 156) { c = 9 + (i - 60) / 8; seg = (i - 60) % 8; segs = 8; }
    else if (i < 516) { c = 21 + (i - 156) / 5; seg = (i - 156) % 5; segs = 5; }
    else if (i < 1668) { c = 93 + (i - 516) / 4; seg = (i - 516) % 4; segs = 4; }
    else { c = 381 + (i - 1668) / 2; seg = (i - 1668) % 2; segs = 2; }
    real t0 = (real)seg / (real)segs, t1 = (real)(seg + 1) / (real)segs;
    st3(P, b, bezier(B, c, t0)); P[b + 3] = 0.0f; st3(P, b + 4, bezier(B, c, t1));
    P[b + 7] = (float)bezier_radius(B, c, t0); P[b + 11] = (float)bezier_radius(B, c, t1);
    P[b + 15] = B[c * K_CS + 15];
    real arc = B[c * K_CS + 14];
    for (int j = 0; j < 12; j++)
      if (j < seg) arc += len3(vsub(bezier(B, c, (real)(j + 1) / (real)segs), bezier(B, c, (real)j / (real)segs)));
    P[b + 16] = (float)arc; P[b + 17] = (float)c; P[b + 18] = B[c * K_CS + 12];
    st3(P, b + 8, basis_u(bezier_dir(B, c, 0.0f)));
    return;
  }
  if (i < K_WOOD + K_LEAF) {
    int leaf = i - K_WOOD, twig = leaf / 14, k = leaf % 14, c = 381 + twig;
    real h = rnd(leaf + 13, seed);
    real t = 0.16f + 0.81f * ((real)k + 0.4f) / 14.0f;
    v3 anchor = bezier(B, c, t), axis = bezier_dir(B, c, t), bu = basis_u(axis), bv = cross(axis, bu);
    real angle = (real)k * 2.399963f + rnd(twig, seed) * 6.28f;
    v3 out = unit(vadd(vscale(bu, COS(angle)), vscale(bv, SIN(angle))));
    v3 u = unit(vadd(vadd(vscale(out, 0.82f), vscale(axis, 0.35f)), V(0.0f, 0.20f, 0.0f)));
    v3 normal = unit(vadd(V(0.0f, 1.0f, 0.0f), vscale(out, 0.20f + h * 0.38f)));
    v3 v = unit(cross(normal, u));
    normal = unit(cross(u, v));
    st3(P, b, anchor); P[b + 3] = 1.0f; st3(P, b + 4, u);
    P[b + 7] = (float)(0.145f + 0.075f * h);
    st3(P, b + 8, v);
    P[b + 11] = (float)(P[b + 7] * (0.34f + 0.07f * rnd(leaf + 37, seed)));
    st3(P, b + 12, normal);
    P[b + 15] = (float)(leaf + seed * 11);
    P[b + 16] = (float)(0.023f + 0.024f * rnd(leaf + 149, seed));
    P[b + 17] = (float)(0.013f + 0.016f * h);
    P[b + 18] = (float)((rnd(leaf + 777, seed) - 0.5f) * 0.10f);
    P[b + 19] = (float)twig;
    return;
  }
  int rock = i - K_WOOD - K_LEAF;
  real a = rnd(rock * 3 + 1, seed) * 6.2831853f;
  real r = 0.8f + 4.5f * SQRT(rnd(rock * 3 + 2, seed));
  real size = 0.045f + 0.19f * POW(rnd(rock + 371, seed), 3.0f);
  st3(P, b, V(COS(a) * r, size * 0.30f - 0.015f, SIN(a) * r));
  P[b + 3] = 2.0f;
  st3(P, b + 4, V(size, size * 0.55f, size * (0.7f + rnd(rock + 16, seed) * 0.5f)));
  P[b + 15] = (float)(rock + seed);
}
/* Per-type bounds (Arbor.cu:132-133). */
static v3 bound_lo(const float* P, int id) {
  int b = id * K_PS, type = (int)P[b + 3];
  if (type < 0) return V(K_FAR, K_FAR, K_FAR);
  v3 a = ld3(P, b);
  if (type == 0) { real r = FMAX(P[b + 7], P[b + 11]) + 0.002f; return vsub(vmin(a, ld3(P, b + 4)), V(r, r, r)); }
  if (type == 2) return vsub(a, ld3(P, b + 4));
  real radius = P[b + 7] + P[b + 16] + 0.025f;
  return vsub(a, V(radius, radius, radius));
}
static v3 bound_hi(const float* P, int id) {
  int b = id * K_PS, type = (int)P[b + 3];
  if (type < 0) return V(-K_FAR, -K_FAR, -K_FAR);
  v3 a = ld3(P, b);
  if (type == 0) { real r = FMAX(P[b + 7], P[b + 11]) + 0.002f; return vadd(vmax(a, ld3(P, b + 4)), V(r, r, r)); }
  if (type == 2) return vadd(a, ld3(P, b + 4));
  real radius = P[b + 7] + P[b + 16] + 0.025f;
  return vadd(a, V(radius, radius, radius));
}

/* --------------------------------------------------------------- CACHE -- */
/* Arbor.cu:138 */
static inline uint32_t bits10(uint32_t x) {
  x &= 1023u; x = (x | (x << 16)) & 50331903u; x = (x | (x << 8)) & 50393103u;
  x = (x | (x << 4)) & 51130563u; x = (x | (x << 2)) & 153391689u; return x;
}
/* Arbor.cu:139 */
static void key_one(const float* P, uint32_t* Keys, uint32_t* Order, int i) {
  Order[i] = (uint32_t)i;
  if (P[i * K_PS + 3] < 0.0f) { Keys[i] = 4294967295u; return; }
  v3 p = vscale(vadd(bound_lo(P, i), bound_hi(P, i)), 0.5f);
  uint32_t x = (uint32_t)(float)(sat((p.x + 12.0f) / 24.0f) * 1023.0f);
  uint32_t y = (uint32_t)(float)(sat((p.y + 1.0f) / 18.0f) * 1023.0f);
  uint32_t z = (uint32_t)(float)(sat((p.z + 12.0f) / 24.0f) * 1023.0f);
  Keys[i] = bits10(x) | (bits10(y) << 1) | (bits10(z) << 2);
}

/* --------------------------------------------------------------- SURFACE -- */
/* Arbor.cu:148 */
static v2 wood_uv(const float* P, int id, v3 p) {
  int b = id * K_PS; v3 a = ld3(P, b); v3 d = unit(vsub(ld3(P, b + 4), a)); v3 init = ld3(P, b + 8);
  v3 u = unit(vsub(init, vscale(d, dot(init, d)))); v3 v = cross(d, u); v3 q = vsub(p, a);
  real z = dot(q, d); real theta = ATAN2(dot(q, v), dot(q, u));
  return V2(theta, P[b + 16] + z);
}
/* Voronoi bark relief (Arbor.cu:149-169). */
static real bark_relief(const float* P, int id, v3 p, real fp) {
  int b = id * K_PS; v3 a = ld3(P, b); v3 d = vsub(ld3(P, b + 4), a);
  real along = sat(dot(vsub(p, a), d) / FMAX(0.000001f, dot(d, d)));
  real radius = lerpr(P[b + 7], P[b + 11], along);
  real amp = FMIN(0.021f, radius * 0.055f);
  int columns = (int)FMAX(7.0f, FLOOR(P[b + 18] * 2.0f * K_PI / 0.065f + 0.5f));
  real period = radius * 2.0f * K_PI / (real)columns;
  real coarse = band(period, fp), fine = band(0.010f, fp), grain = band(0.0025f, fp);
  if (coarse < 0.000001f && fine < 0.000001f) return amp * 0.32f;
  v2 uv = wood_uv(P, id, p); real theta = uv.x, arc = uv.y; int seed = (int)P[b + 15];
  real x = (theta / (2.0f * K_PI) + 0.5f) * (real)columns + 0.32f * SIN(arc * 6.7f + COS(theta) * 3.0f) + 0.15f * SIN(arc * 19.0f + SIN(theta) * 2.0f);
  real y = arc / 0.19f + 0.25f * SIN(theta * 7.0f) + 0.1f * SIN(theta * 19.0f);
  int ix = (int)FLOOR(x), iy = (int)FLOOR(y);
  real first = 100.0f, second = 100.0f;
  for (int j = -1; j <= 1; j++)
    for (int k = -1; k <= 1; k++) {
      int cell = ix + k; int wrapped = ((cell % columns) + columns) % columns;
      real xx = (real)cell + 0.18f + 0.64f * hash2(wrapped, iy + j, seed) - x;
      real yy = (real)(iy + j) + 0.18f + 0.64f * hash2(wrapped + columns, iy + j, seed + 31) - y;
      real dd = xx * xx + yy * yy;
      if (dd < first) { second = first; first = dd; } else if (dd < second) second = dd;
    }
  real gap = SQRT(second) - SQRT(first);
  real fissure = 1.0f - smoothr(0.015f, 0.17f, gap);
  real plates = fissure * fissure;
  v3 coord = V(COS(theta) * 9.0f, SIN(theta) * 9.0f, arc * 23.0f);
  real splinter = noise3(coord, seed), pores = noise3(vscale(coord, 4.0f), seed + 731);
  return amp * clampr(0.32f + coarse * (plates - 0.37f) * 0.69f + fine * (splinter - 0.5f) * 0.24f + grain * (pores - 0.5f) * 0.08f, 0.005f, 1.0f);
}
/* Wood signed distance (Arbor.cu:170). */
static real wood_sdf(const float* P, int id, v3 p, real fp) {
  int b = id * K_PS; v3 a = ld3(P, b); v3 ab = vsub(ld3(P, b + 4), a);
  real t = sat(dot(vsub(p, a), ab) / FMAX(0.0000001f, dot(ab, ab)));
  real radius = lerpr(P[b + 7], P[b + 11], t);
  return len3(vsub(vsub(p, a), vscale(ab, t))) - radius + bark_relief(P, id, p, fp);
}
/* Wind-rotated leaf frame (Arbor.cu:171-172). */
static real leaf_angle(const float* P, int b, real time, real wind) {
  real phase = (real)(((int)P[b + 15]) % 8192) * 0.618f;
  return wind * (0.11f * SIN(time * 2.1f + phase) + 0.045f * SIN(time * 5.8f + phase * 1.7f));
}
static v3 leaf_axis_u(const float* P, int id, real time, real wind) {
  int b = id * K_PS; v3 u = ld3(P, b + 4), n = ld3(P, b + 12); real a = leaf_angle(P, b, time, wind);
  return vadd(vscale(u, COS(a)), vscale(n, SIN(a)));
}
static v3 leaf_axis_n(const float* P, int id, real time, real wind) {
  int b = id * K_PS; v3 u = ld3(P, b + 4), n = ld3(P, b + 12); real a = leaf_angle(P, b, time, wind);
  return vsub(vscale(n, COS(a)), vscale(u, SIN(a)));
}
/* Leaf outline and height field (Arbor.cu:173-174). */
static real leaf_width(real u, real length, real half_width, real fp) {
  real q = sat(u / length); real s = SIN(K_PI * q);
  real lobes = 0.77f + 0.23f * COS(q * K_PI * 10.0f + 0.45f);
  real fine = band(0.002f, fp) * 0.015f * SIN(q * K_PI * 160.0f);
  return half_width * POW(FMAX(0.0f, s), 0.72f) * (lobes + fine);
}
static real leaf_height(real u, real v, real len, real hw, real curl, real twist, real fp) {
  real q = clampr(u / len, -0.2f, 1.2f); real s = SIN(K_PI * q);
  real coarse = curl * s + twist * (q - 0.4f) * v + 0.009f * (v * v / (hw * hw)) * s;
  real mid = 0.0012f * EXP(-FABS(v) / 0.005f) * s * band(0.007f, fp);
  return coarse + mid;
}

/* --------------------------------------------------------------- CAMERA -- */
/* Arbor.cu:179 */
static void pose(float* C, v3 eye, real yaw, real pitch) {
  C[16] = (float)yaw; C[17] = (float)pitch; C[27] = (float)yaw; C[28] = (float)pitch;
  st3(C, 0, eye);
  real cp = COS(pitch);
  v3 f = unit(V(SIN(yaw) * cp, SIN(pitch), COS(yaw) * cp));
  st3(C, 4, vadd(eye, f));
  C[3] = 1.0f; C[18] = 1.0f;
}
/* Arbor.cu:180 */
static void preset(float* C, int which) {
  if (which == 1) pose(C, V(2.0f, 1.72f, 18.0f), K_PI, 0.0f);
  if (which == 2) pose(C, V(-1.4f, 1.72f, 7.0f), K_PI * 0.94f, 0.02f);
  if (which == 3) pose(C, V(8.0f, 1.72f, -3.0f), K_PI * 0.55f, -0.02f);
  if (which == 4) pose(C, V(-11.0f, 1.72f, -7.0f), 0.65f, 0.03f);
  if (which == 5) pose(C, V(0.0f, 12.0f, 72.0f), K_PI, -0.12f);
  C[9] = 0.0f; C[10] = 1.0f;
}

/* ---------------------------------------------------------------- TRACE -- */
/* Arbor.cu:186 */
static real sphere_hit(v3 ro, v3 rd, v3 p, real radius) {
  v3 q = vsub(ro, p); real b = dot(q, rd); real c = dot(q, q) - radius * radius; real d = b * b - c;
  if (d < 0.0f) return K_FAR;
  real t = -b - SQRT(d);
  if (t <= 0.0001f) t = -b + SQRT(d);
  return t > 0.0001f ? t : K_FAR;
}
/* Tapered tube plus spherical caps (Arbor.cu:188-191). */
static real tube_hit(v3 ro, v3 rd, v3 a, v3 b, real ra, real rb) {
  v3 axis = vsub(b, a); real len = len3(axis); axis = vdivs(axis, FMAX(len, 0.000001f));
  v3 q = vsub(ro, a); real z = dot(q, axis), dz = dot(rd, axis);
  real k = (rb - ra) / FMAX(0.000001f, len);
  v3 v = vsub(q, vscale(axis, z)), d = vsub(rd, vscale(axis, dz));
  real radius = ra + k * z;
  real aa = dot(d, d) - k * k * dz * dz, bb = dot(v, d) - radius * k * dz, cc = dot(v, v) - radius * radius;
  real best = FMIN(sphere_hit(ro, rd, a, ra), sphere_hit(ro, rd, b, rb));
  real disc = bb * bb - aa * cc;
  if (disc >= 0.0f && FABS(aa) > 0.0000001f) {
    for (int j = 0; j < 2; j++) {
      real t = (-bb + (j == 0 ? -1.0f : 1.0f) * SQRT(disc)) / aa;
      real h = z + t * dz;
      if (t > 0.0001f && h >= 0.0f && h <= len) best = FMIN(best, t);
    }
  }
  return best;
}
/* Arbor.cu:192-202 */
static real wood_hit(const float* P, int id, v3 ro, v3 rd, real fp, int refine) {
  int b = id * K_PS; v3 a = ld3(P, b), end = ld3(P, b + 4);
  if (!refine) {
    real ra = P[b + 7] - FMIN(0.021f, P[b + 7] * 0.055f) * 0.32f;
    real rb = P[b + 11] - FMIN(0.021f, P[b + 11] * 0.055f) * 0.32f;
    return tube_hit(ro, rd, a, end, ra, rb);
  }
  real t = tube_hit(ro, rd, a, end, P[b + 7], P[b + 11]);
  if (t >= K_FAR) return K_FAR;
  v2 span = box_span(ro, rd, bound_lo(P, id), bound_hi(P, id));
  real eps = FMAX(0.000025f, FMIN(0.00025f, fp * 0.13f));
  for (int k = 0; k < 64; k++) {
    real f = wood_sdf(P, id, vadd(ro, vscale(rd, t)), fp);
    if (f < eps) return t;
    t += FMAX(eps * 0.35f, f * 0.27f);
    if (t > span.y) return K_FAR;
  }
  return K_FAR;
}
/* Curved-leaf Newton solve (Arbor.cu:203-218). */
static real leaf_hit(const float* P, int id, v3 ro, v3 rd, real fp, real time, real wind) {
  int b = id * K_PS; v3 origin = ld3(P, b);
  v3 u = leaf_axis_u(P, id, time, wind), v = ld3(P, b + 8), n = leaf_axis_n(P, id, time, wind);
  real stem = P[b + 16], len = P[b + 7], width = P[b + 11];
  v3 q = vsub(ro, origin);
  real x = dot(q, u) - stem, y = dot(q, v), z = dot(q, n);
  real dx = dot(rd, u), dy = dot(rd, v), dz = dot(rd, n);
  real best = tube_hit(ro, rd, origin, vadd(origin, vscale(u, stem)), 0.0011f, 0.00065f);
  v2 span = box_span(V(x, y, z), V(dx, dy, dz), V(-0.001f, -width, -0.035f), V(len + 0.001f, width, 0.065f));
  if (span.y < FMAX(0.0001f, span.x)) return best;
  real t = FABS(dz) > 0.000001f ? -z / dz : (span.x + span.y) * 0.5f;
  t = clampr(t, FMAX(0.0001f, span.x), span.y);
  real c17 = P[b + 17], c18 = P[b + 18];
  for (int k = 0; k < 7; k++) {
    real xx = x + dx * t, yy = y + dy * t;
    real height = leaf_height(xx, yy, len, width, c17, c18, fp);
    real f = z + dz * t - height;
    real e = 0.00015f;
    real hx = (leaf_height(xx + e, yy, len, width, c17, c18, fp) - leaf_height(xx - e, yy, len, width, c17, c18, fp)) / (2.0f * e);
    real hy = (leaf_height(xx, yy + e, len, width, c17, c18, fp) - leaf_height(xx, yy - e, len, width, c17, c18, fp)) / (2.0f * e);
    real deriv = dz - hx * dx - hy * dy;
    if (FABS(deriv) < 0.00001f) break;
    t -= clampr(f / deriv, -0.13f, 0.13f);
    t = clampr(t, span.x, span.y);
  }
  real xx = x + dx * t, yy = y + dy * t;
  real err = FABS(z + dz * t - leaf_height(xx, yy, len, width, c17, c18, fp));
  if (t > 0.0001f && xx > 0.0f && xx < len && FABS(yy) < leaf_width(xx, len, width, fp) && err < 0.0003f) best = FMIN(best, t);
  return best;
}
/* Arbor.cu:219 */
static real object_hit(const float* P, int id, v3 ro, v3 rd, real fp, real time, real wind, int refine) {
  int b = id * K_PS, type = (int)P[b + 3];
  if (type < 0) return K_FAR;
  if (type == 0) return wood_hit(P, id, ro, rd, fp, refine);
  if (type == 1) return leaf_hit(P, id, ro, rd, fp, time, wind);
  v3 h = ld3(P, b + 4), q = vsub(ro, ld3(P, b));
  v3 p = V(q.x / h.x, q.y / h.y, q.z / h.z), d = V(rd.x / h.x, rd.y / h.y, rd.z / h.z);
  real aa = dot(d, d), bb = dot(p, d), cc = dot(p, p) - 1.0f;
  real disc = bb * bb - aa * cc;
  if (disc < 0.0f) return K_FAR;
  real t = (-bb - SQRT(disc)) / aa;
  return t > 0.0001f ? t : K_FAR;
}
/* Stack traversal of the heap BVH, nearest child first (Arbor.cu:220-230). */
static v2 walk_tree(const float* P, const float* N, v3 ro, v3 rd, real cone, real time, real wind, real best, int ignore, int shadows, const uint32_t* Order) {
  int stack[32], top = 0, node = 1, found = -1;
  for (int visit = 0; visit < K_NODES; visit++) {
    if (node <= 0) break;
    int b = node * 8;
    v2 span = box_span(ro, rd, ld3(N, b), ld3(N, b + 4));
    int hit = N[b + 3] > 0.0f && span.y >= FMAX(0.0001f, span.x) && span.x < best;
    if (hit && node < K_CAPACITY) {
      int left = node * 2, right = left + 1, lb = left * 8, rb = right * 8;
      v2 ls = box_span(ro, rd, ld3(N, lb), ld3(N, lb + 4));
      v2 rs = box_span(ro, rd, ld3(N, rb), ld3(N, rb + 4));
      int lh = N[lb + 3] > 0.0f && ls.y >= FMAX(0.0001f, ls.x) && ls.x < best;
      int rh = N[rb + 3] > 0.0f && rs.y >= FMAX(0.0001f, rs.x) && rs.x < best;
      if (lh && rh) { int l = ls.x < rs.x; stack[top++] = l ? right : left; node = l ? left : right; continue; }
      if (lh) { node = left; continue; }
      if (rh) { node = right; continue; }
    } else if (hit) {
      int id = (int)Order[node - K_CAPACITY];
      if (id != ignore) {
        real fp = FMAX(0.000005f, cone * FMAX(0.05f, span.x));
        real t = object_hit(P, id, ro, rd, fp, time, wind, !shadows);
        if (t < best) { best = t; found = id; }
      }
    }
    node = 0;
    if (top > 0) node = stack[--top];
  }
  return V2(best, (real)found);
}
/* Arbor.cu:231-234 */
static v3 object_normal(const float* P, int id, v3 p, real fp, real time, real wind) {
  int b = id * K_PS, type = (int)P[b + 3];
  if (type == 0) {
    real e = FMAX(0.000035f, FMIN(0.0005f, fp * 0.18f));
    v3 ex = V(e, 0.0f, 0.0f), ey = V(0.0f, e, 0.0f), ez = V(0.0f, 0.0f, e);
    return unit(V(wood_sdf(P, id, vadd(p, ex), fp) - wood_sdf(P, id, vsub(p, ex), fp),
                  wood_sdf(P, id, vadd(p, ey), fp) - wood_sdf(P, id, vsub(p, ey), fp),
                  wood_sdf(P, id, vadd(p, ez), fp) - wood_sdf(P, id, vsub(p, ez), fp)));
  }
  if (type == 1) {
    v3 u = leaf_axis_u(P, id, time, wind), v = ld3(P, b + 8), n = leaf_axis_n(P, id, time, wind);
    v3 q = vsub(p, ld3(P, b));
    real x = dot(q, u) - P[b + 16], y = dot(q, v);
    if (x < 0.0f) { v3 centre = vadd(ld3(P, b), vscale(u, x + P[b + 16])); return unit(vsub(p, centre)); }
    real e = 0.0002f;
    real a = (leaf_height(x + e, y, P[b + 7], P[b + 11], P[b + 17], P[b + 18], fp) - leaf_height(x - e, y, P[b + 7], P[b + 11], P[b + 17], P[b + 18], fp)) / (2.0f * e);
    real c = (leaf_height(x, y + e, P[b + 7], P[b + 11], P[b + 17], P[b + 18], fp) - leaf_height(x, y - e, P[b + 7], P[b + 11], P[b + 17], P[b + 18], fp)) / (2.0f * e);
    return unit(vsub(vsub(n, vscale(u, a)), vscale(v, c)));
  }
  v3 q = vsub(p, ld3(P, b)), h = ld3(P, b + 4);
  return unit(V(q.x / (h.x * h.x), q.y / (h.y * h.y), q.z / (h.z * h.z)));
}
/* A forest of several species (no reference counterpart; the reference keeps
 * one resident tree for all 324 instances, README.md:8): instance t keeps the
 * reference's transform, phase and tint (forestPos/Scale/Yaw/Seed of t) but
 * takes its geometry from scene of[t] of the set.  NULL = the reference's
 * forest, every instance on the one resident scene. */
typedef struct {
  const float* const* P;
  const float* const* N;
  const uint32_t* const* Order;
  const int* of;  /* K_FOREST species indices */
} species_set;
#define SP_P(sp, tree, base) ((sp) ? (sp)->P[(sp)->of[tree]] : (base))
#define SP_N(sp, tree, base) ((sp) ? (sp)->N[(sp)->of[tree]] : (base))
#define SP_O(sp, tree, base) ((sp) ? (sp)->Order[(sp)->of[tree]] : (base))

/* Forest 2D DDA with per-tree bounding spheres (Arbor.cu:235-251).  The
 * single-tree mode (no forest counterpart in the reference) traces the
 * resident tree with an identity instance, as the harness's BVH check does at
 * tests/native_harness.cpp:84. */
static v2 walk_forest(const float* P, const float* N, const uint32_t* Order, v3 ro, v3 rd, real cone, real time, real wind, real best, int ws, int* tree_out, int shadows, const species_set* sp) {
  int found_tree = -1; real found = -1.0f;
  real half = (real)K_SIDE * K_SPACING * 0.5f;
  v2 world = box_span(ro, rd, V(-half, -1.2f, -half), V(half, 13.5f, half));
  real enter = FMAX(0.0f, world.x), exit_t = FMIN(best, world.y);
  if (exit_t < enter) { *tree_out = -1; return V2(best, -1.0f); }
  v3 pos = vadd(ro, vscale(rd, enter + 0.0002f));
  int ix = (int)FLOOR(pos.x / K_SPACING + (real)K_SIDE * 0.5f + 0.5f);
  int iz = (int)FLOOR(pos.z / K_SPACING + (real)K_SIDE * 0.5f + 0.5f);
  int sx = rd.x >= 0.0f ? 1 : -1, sz = rd.z >= 0.0f ? 1 : -1;
  real invx = inv_safe(rd.x), invz = inv_safe(rd.z);
  real bx = ((real)(ix - K_SIDE / 2) + (sx > 0 ? 0.5f : -0.5f)) * K_SPACING;
  real bz = ((real)(iz - K_SIDE / 2) + (sz > 0 ? 0.5f : -0.5f)) * K_SPACING;
  real tx = (bx - ro.x) * invx, tz = (bz - ro.z) * invz;
  real dx = K_SPACING * FABS(invx), dz = K_SPACING * FABS(invz);
  for (int step = 0; step < 48; step++) {
    if (ix < 0 || iz < 0 || ix >= K_SIDE || iz >= K_SIDE) break;
    int tree = iz * K_SIDE + ix;
    real sc = tree_scale(tree, ws);
    v3 centre = vadd(tree_pos(tree, ws), V(0.0f, 4.4f * sc, 0.0f));
    real radius = 6.6f * sc;
    real broad = sphere_hit(ro, rd, centre, radius);
    if (broad < best) {
      v3 lr = to_local_point(ro, tree, ws), ld = to_local_dir(rd, tree, ws);
      real phase = (real)(tree_seed(tree, ws) & 8191) * 0.0017f;
      v2 h = walk_tree(SP_P(sp, tree, P), SP_N(sp, tree, N), lr, ld, cone / sc, time + phase, wind, best / sc, -1, shadows, SP_O(sp, tree, Order));
      if (h.y >= 0.0f && h.x * sc < best) { best = h.x * sc; found = h.y; found_tree = tree; }
    }
    real next = tx < tz ? tx : tz;
    if (next > exit_t || next > best) break;
    if (tx < tz) { ix += sx; tx += dx; } else { iz += sz; tz += dz; }
  }
  *tree_out = found_tree;
  return V2(best, found);
}
static v2 walk_scene(const float* P, const float* N, const uint32_t* Order, v3 ro, v3 rd, real cone, real time, real wind, real best, int ws, int* tree_out, int shadows, int single, const species_set* sp) {
  if (!single) return walk_forest(P, N, Order, ro, rd, cone, time, wind, best, ws, tree_out, shadows, sp);
  *tree_out = -1;
  return walk_tree(P, N, ro, rd, cone, time, wind, best, -1, shadows, Order);
}
/* One pixel of tracePixels (Arbor.cu:252). */
static void trace_px(const float* P, const float* N, const uint32_t* Order, const float* C, float* Hit, int w, int h, int x, int y, int single, const species_set* sp) {
  int b = (y * w + x) * 4;
  v3 ro = cam_pos(C), rd = primary_dir(C, x, y, w, h);
  real ground = rd.y < -0.00001f ? -ro.y / rd.y : K_FAR;
  int tree = -1;
  v2 r = walk_scene(P, N, Order, ro, rd, C[14] / (real)h, C[8], C[11], ground > 0.0f ? ground : K_FAR, (int)C[31], &tree, 0, single, sp);
  Hit[b] = (float)r.x; Hit[b + 1] = (float)r.y; Hit[b + 2] = (float)tree; Hit[b + 3] = (float)(C[14] * r.x / (real)h);
}

/* ---------------------------------------------------------------- SHADE -- */
/* Arbor.cu:256 */
static v3 sky(v3 rd, v3 sun) {
  real h = sat(rd.y);
  v3 c = mixv(V(0.75f, 0.79f, 0.77f), V(0.19f, 0.35f, 0.54f), POW(h, 0.48f));
  real warm = POW(sat(dot(rd, sun)), 32.0f);
  c = vadd(c, vscale(V(0.48f, 0.26f, 0.075f), warm));
  real disc = smoothr(0.99996f, 0.999984f, dot(rd, sun));
  c = vadd(c, vscale(V(8.0f, 6.7f, 4.9f), disc));
  real clouds = noise2(rd.x * 5.0f / (0.2f + h), rd.z * 5.0f / (0.2f + h), 231);
  real veil = smoothr(0.62f, 0.81f, clouds) * smoothr(0.02f, 0.18f, h) * 0.38f;
  return mixv(c, V(1.1f, 1.10f, 1.05f), veil);
}
/* Arbor.cu:257-263 */
static v3 bark_albedo(const float* P, int id, v3 p, real fp) {
  int b = id * K_PS, seed = (int)P[b + 15];
  v2 uv = wood_uv(P, id, p);
  v3 coord = V(COS(uv.x) * 9.0f, SIN(uv.x) * 9.0f, uv.y * 7.0f);
  real mottle = noise3(vscale(p, 3.0f), 714), rough = noise3(coord, seed);
  v3 d = vsub(ld3(P, b + 4), ld3(P, b));
  real t = sat(dot(vsub(p, ld3(P, b)), d) / FMAX(0.000001f, dot(d, d)));
  real amp = FMIN(0.021f, lerpr(P[b + 7], P[b + 11], t) * 0.055f);
  real cut = bark_relief(P, id, p, fp) / FMAX(0.00001f, amp);
  v3 c = mixv(V(0.10f, 0.075f, 0.050f), V(0.25f, 0.21f, 0.16f), 0.25f + rough * 0.62f);
  c = vscale(c, 0.75f + 0.35f * mottle);
  c = vscale(c, 1.0f - 0.62f * smoothr(0.28f, 0.85f, cut));
  real moss = smoothr(0.52f, 0.72f, noise3(vscale(p, 5.0f), 189)) * (1.0f - smoothr(0.15f, 1.4f, p.y));
  c = mixv(c, V(0.045f, 0.064f, 0.018f), moss * 0.62f);
  real lichen = smoothr(0.65f, 0.77f, noise3(vscale(p, 23.0f), 27)) * smoothr(0.25f, 0.65f, noise3(vscale(p, 90.0f), 712)) * band(0.018f, fp);
  c = mixv(c, V(0.31f, 0.33f, 0.23f), lichen * 0.5f);
  real grain = (noise3(vscale(coord, 15.0f), seed) - 0.5f) * band(0.0025f, fp);
  return vscale(c, 1.0f + grain * 0.38f);
}
/* Arbor.cu:264 */
static real vein(const float* P, int id, v3 p, real fp, real time, real wind) {
  int b = id * K_PS; v3 q = vsub(p, ld3(P, b));
  real x = dot(q, leaf_axis_u(P, id, time, wind)) - P[b + 16], y = dot(q, ld3(P, b + 8)), len = P[b + 7];
  real mid = EXP(-FABS(y) / FMAX(0.00065f, fp * 0.55f));
  real fy = fracr((x - FABS(y) * 0.70f) / len * 7.0f);
  real dd = FMIN(fy, 1.0f - fy) * len / 7.0f;
  real lateral = EXP(-dd / FMAX(0.00033f, fp * 0.5f));
  return sat(mid * 0.82f + lateral * 0.48f) * band(0.003f, fp);
}
/* Arbor.cu:265-268 */
static v3 leaf_albedo(const float* P, int id, v3 p, real fp, real time, real wind) {
  int b = id * K_PS; real h = rnd((int)P[b + 15], 887);
  v3 q = vsub(p, ld3(P, b));
  real x = dot(q, leaf_axis_u(P, id, time, wind)) - P[b + 16];
  if (x < 0.0f) return V(0.17f, 0.15f, 0.048f);
  real y = dot(q, ld3(P, b + 8));
  real v = vein(P, id, p, fp, time, wind);
  v3 c = mixv(V(0.035f, 0.11f, 0.008f), V(0.15f, 0.255f, 0.025f), h);
  c = mixv(c, V(0.22f, 0.26f, 0.055f), v * 0.57f);
  real speck = (noise2(x * 700.0f, y * 700.0f, (int)P[b + 15]) - 0.5f) * band(0.0017f, fp);
  real edge = smoothr(0.78f, 1.0f, FABS(y) / FMAX(0.001f, leaf_width(x, P[b + 7], P[b + 11], fp)));
  c = vscale(c, 1.0f + speck * 0.27f);
  return mixv(c, V(0.23f, 0.20f, 0.05f), edge * 0.22f);
}
/* Arbor.cu:269 */
static v3 ground_albedo(v3 p, real fp) {
  real a = noise2(p.x * 3.0f, p.z * 3.0f, 819), b = noise2(p.x * 15.0f, p.z * 15.0f, 28);
  real r = SQRT(p.x * p.x + p.z * p.z);
  real soil = 1.0f - smoothr(4.1f, 6.8f, r + noise2(p.x, p.z, 13));
  v3 grass = mixv(V(0.085f, 0.115f, 0.035f), V(0.23f, 0.24f, 0.092f), a);
  v3 dirt = mixv(V(0.075f, 0.055f, 0.035f), V(0.16f, 0.13f, 0.080f), b);
  real moss = smoothr(0.53f, 0.73f, a);
  dirt = mixv(dirt, V(0.049f, 0.079f, 0.022f), moss * 0.72f);
  real grit = (noise2(p.x * 200.0f, p.z * 200.0f, 127) - 0.5f) * band(0.007f, fp);
  return vscale(mixv(grass, dirt, soil), 1.0f + grit * 0.40f);
}
/* Arbor.cu:270 */
static v3 albedo_of(const float* P, int id, v3 p, real fp, real time, real wind) {
  if (id < 0) return ground_albedo(p, fp);
  int b = id * K_PS, type = (int)P[b + 3];
  if (type == 0) return bark_albedo(P, id, p, fp);
  if (type == 1) return leaf_albedo(P, id, p, fp, time, wind);
  real f = noise3(vscale(p, 42.0f), (int)P[b + 15]);
  return mixv(V(0.09f, 0.10f, 0.086f), V(0.31f, 0.30f, 0.24f), f);
}
/* Sun visibility through at most four segments (Arbor.cu:271-274). */
static v3 sun_visibility(const float* P, const float* N, const uint32_t* Order, v3 p, v3 dir, real time, real wind, int ws, int single, const species_set* sp) {
  v3 trans = V(1.0f, 1.0f, 1.0f); v3 ro = p;
  for (int j = 0; j < 4; j++) {
    int tree = -1;
    v2 h = walk_scene(P, N, Order, ro, dir, 0.0001f, time, wind, 36.0f, ws, &tree, 1, single, sp);
    int id = (int)h.y;
    if (id < 0) break;
    if (SP_P(sp, tree, P)[id * K_PS + 3] != 1.0f) return V(0.0f, 0.0f, 0.0f);
    trans = vmul(trans, V(0.18f, 0.29f, 0.065f));
    ro = vadd(ro, vscale(dir, h.x + 0.0018f));
  }
  return trans;
}
/* Arbor.cu:276 */
static real ggx(v3 n, v3 v, v3 l, real rough) {
  v3 h = unit(vadd(v, l));
  real nh = sat(dot(n, h)), nv = FMAX(0.002f, sat(dot(n, v))), nl = sat(dot(n, l)), vh = sat(dot(v, h));
  real a = rough * rough, aa = a * a;
  real den = nh * nh * (aa - 1.0f) + 1.0f;
  real D = aa / (K_PI * den * den);
  real k = (rough + 1.0f) * (rough + 1.0f) * 0.125f;
  real G = nv / (nv * (1.0f - k) + k) * nl / (nl * (1.0f - k) + k);
  real F = 0.035f + 0.965f * POW(1.0f - vh, 5.0f);
  return D * G * F / (4.0f * nv + 0.0001f);
}
/* The surface point of a hit pixel and its shading normal, facing the
 * camera (Arbor.cu:278-280: the first steps of shadePixels). */
typedef struct { v3 p, lp, n; real fp, lfp, phase; int leaf; } surface;
static surface shade_surface(const float* P, const float* C, const float* Hit, v3 ro, v3 rd, int b, int single) {
  surface s;
  real t = Hit[b]; int id = (int)Hit[b + 1], tree = (int)Hit[b + 2];
  int ws = (int)C[31];
  v3 p = vadd(ro, vscale(rd, t));
  real fp = FMAX(0.000005f, Hit[b + 3]);
  v3 lp = p, n = V(0.0f, 1.0f, 0.0f);
  real lfp = fp, phase = 0.0f;
  if (id >= 0 && tree >= 0) {
    real sc = tree_scale(tree, ws);
    lp = to_local_point(p, tree, ws); lfp = fp / sc;
    phase = (real)(tree_seed(tree, ws) & 8191) * 0.0017f;
    n = to_world_normal(object_normal(P, id, lp, lfp, C[8] + phase, C[11]), tree, ws);
  } else if (id >= 0 && single) {
    n = object_normal(P, id, lp, lfp, C[8], C[11]);
  }
  s.leaf = id >= 0 && P[id * K_PS + 3] == 1.0f;
  if (dot(n, rd) > 0.0f) n = vscale(n, -1.0f);
  if (id < 0) {
    real e = FMAX(0.001f, fp);
    real nx = (noise2((p.x + e) * 18.0f, p.z * 18.0f, 133) - noise2((p.x - e) * 18.0f, p.z * 18.0f, 133)) * 0.18f;
    real nz = (noise2(p.x * 18.0f, (p.z + e) * 18.0f, 133) - noise2(p.x * 18.0f, (p.z - e) * 18.0f, 133)) * 0.18f;
    n = unit(V(nx, 1.0f, nz));
  }
  s.p = p; s.lp = lp; s.n = n; s.fp = fp; s.lfp = lfp; s.phase = phase;
  return s;
}
/* One pixel of shadePixels (Arbor.cu:277-289). */
static void shade_px(const float* Pw, const float* N, const uint32_t* Order, const float* C, const float* Hit, float* Linear, float* Guide, int w, int hgt, int x, int y, int single, const species_set* sp) {
  int pixel = y * w + x, b = pixel * 4;
  real t = Hit[b]; int id = (int)Hit[b + 1], tree = (int)Hit[b + 2];
  v3 ro = cam_pos(C), rd = primary_dir(C, x, y, w, hgt), sun = sun_dir(C);
  v3 col = sky(rd, sun), guide = V(1.0f, 1.0f, 1.0f);
  int ws = (int)C[31];
  /* the hit instance's scene (its species' scene in a forest of several) */
  const float* P = (tree >= 0 && tree < K_SIDE * K_SIDE) ? SP_P(sp, tree, Pw) : Pw;
  if (t < K_FAR) {
    surface s = shade_surface(P, C, Hit, ro, rd, b, single);
    v3 p = s.p, lp = s.lp, n = s.n;
    real fp = s.fp, lfp = s.lfp, phase = s.phase;
    int leaf = s.leaf;
    (void)fp;
    v3 albedo = albedo_of(P, id, id >= 0 ? lp : p, lfp, C[8] + phase, C[11]);
    if (tree >= 0) {
      int ts = tree_seed(tree, ws);
      real hue = rnd(8, ts), age = rnd(9, ts), season = rnd(10, ts);
      real dark = 0.76f + age * 0.38f;
      v3 tint = V(0.88f + 0.22f * hue, 0.84f + 0.28f * (1.0f - FABS(hue - 0.55f)), 0.72f + 0.25f * (1.0f - hue));
      if (leaf) tint = mixv(tint, V(1.12f, 0.88f, 0.48f), smoothr(0.78f, 0.98f, season) * 0.38f);
      else tint = mixv(tint, V(0.78f, 0.66f, 0.53f), season * 0.18f);
      albedo = vscale(vmul(albedo, tint), dark);
    }
    guide = albedo;
    int sample = (int)C[9];
    real r1 = rnd(imad(sample, 1823, pixel), 991), r2 = rnd(imad(sample, 971, pixel), 731);
    v3 su = basis_u(sun), sv = cross(sun, su);
    real angle = r1 * 6.28318f, disk = SQRT(r2) * 0.012f;
    v3 light = unit(vadd(vadd(sun, vscale(su, COS(angle) * disk)), vscale(sv, SIN(angle) * disk)));
    real offset = id >= 0 ? 0.0014f : 0.004f;
    v3 vis = V(1.0f, 1.0f, 1.0f);
    if (C[22] > 0.5f) vis = sun_visibility(Pw, N, Order, vadd(p, vscale(light, offset)), light, C[8], C[11], ws, single, sp);
    real nl = sat(dot(n, light)), back = sat(-dot(n, light));
    v3 direct = vscale(albedo, nl / K_PI);
    if (leaf) {
      real vv = vein(P, id, lp, lfp, C[8] + phase, C[11]);
      direct = vadd(direct, vscale(albedo, back * (0.75f - 0.25f * vv) + POW(sat(dot(rd, light)), 9.0f) * 0.12f));
    }
    real spec = ggx(n, vscale(rd, -1.0f), light, leaf ? 0.39f : 0.82f);
    direct = vadd(direct, V(spec, spec, spec));
    real ao = 1.0f;
    v3 ambient = vadd(vscale(vscale(V(0.30f, 0.37f, 0.45f), 0.45f + 0.55f * sat(n.y)), ao), vscale(V(0.08f, 0.068f, 0.035f), sat(-n.y)));
    if (leaf) ambient = vadd(ambient, vscale(V(0.04f, 0.055f, 0.022f), ao));
    col = vadd(vmul(vmul(direct, vis), V(4.8f, 4.2f, 3.1f)), vmul(albedo, ambient));
    real haze = 1.0f - EXP(-t * 0.0018f);
    col = mixv(col, sky(rd, sun), haze);
    if (C[15] == 1.0f) {
      real w0 = band(0.065f, lfp), w1 = band(0.005f, lfp), w2 = band(0.001f, lfp);
      col = V(w0 * 0.80f, w1 * 0.85f, w2 * 0.9f);
    }
    if (C[15] == 2.0f) {
      real hh = rnd(id + 177 + (tree + 1) * 71, 32);
      col = id < 0 ? V(0.10f, 0.10f, 0.10f) : (leaf ? V(0.1f, 0.3f + hh * 0.5f, 0.17f) : V(0.47f + hh * 0.3f, 0.25f, 0.10f));
    }
    if (C[15] == 3.0f) col = vadd(vscale(n, 0.5f), V(0.5f, 0.5f, 0.5f));
  }
  st3(Linear, b, col); Linear[b + 3] = 1.0f;
  st3(Guide, b, guide); Guide[b + 3] = 1.0f;
}
/* Same-surface 5x5 demodulated filter (Arbor.cu:292-302). */
static void filter_px(const float* Linear, const float* Guide, const float* Hit, float* Filtered, const float* C, int w, int h, int x, int y) {
  int b = (y * w + x) * 4;
  v3 col = ld3(Linear, b), base = vadd(ld3(Guide, b), V(0.02f, 0.02f, 0.02f)), sum = V(0.0f, 0.0f, 0.0f);
  real weight = 0.0f; int id = (int)Hit[b + 1]; real depth = Hit[b];
  if (depth < K_FAR && C[15] < 0.5f) {
    for (int j = -2; j <= 2; j++)
      for (int k = -2; k <= 2; k++) {
        int xx = x + k, yy = y + j;
        if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
        int q = (yy * w + xx) * 4;
        if ((int)Hit[q + 1] != id || (int)Hit[q + 2] != (int)Hit[b + 2] || FABS(Hit[q] - depth) > FMAX(0.005f, Hit[b + 3] * 6.0f)) continue;
        real wt = EXP(-(real)(j * j + k * k) * 0.30f);
        v3 c = ld3(Linear, q), g = vadd(ld3(Guide, q), V(0.02f, 0.02f, 0.02f));
        sum = vadd(sum, vscale(V(c.x / g.x, c.y / g.y, c.z / g.z), wt));
        weight += wt;
      }
    if (weight > 0.0f) col = mixv(col, vmul(vdivs(sum, weight), base), 0.86f);
  }
  st3(Filtered, b, col); Filtered[b + 3] = 1.0f;
}
/* Arbor.cu:303 */
static inline real aces_curve(real x) { return sat((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f)); }
/* Progressive mean, ACES, gamma, vignette, RGBA8 (Arbor.cu:304). */
static void resolve_px(const float* Filtered, float* History, uint32_t* Pixels, const float* C, int w, int h, int x, int y) {
  int i = y * w + x, b = i * 4;
  v3 cur = ld3(Filtered, b);
  real count = C[10] > 0.5f ? 0.0f : C[9];
  v3 mean = count < 0.5f ? cur : mixv(ld3(History, b), cur, 1.0f / (count + 1.0f));
  st3(History, b, mean); History[b + 3] = (float)(count + 1.0f);
  v3 col = vscale(mean, C[20]);
  col = V(aces_curve(col.x), aces_curve(col.y), aces_curve(col.z));
  col = V(POW(col.x, 1.0f / 2.2f), POW(col.y, 1.0f / 2.2f), POW(col.z, 1.0f / 2.2f));
  real u = ((real)x / (real)w - 0.5f) * 2.0f, v = ((real)y / (real)h - 0.5f) * 2.0f;
  col = vscale(col, 1.0f - 0.09f * (u * u + v * v));
  Pixels[i] = pack_rgba(col);
}

/* ============================================================ EXPORTS == */
/* Same exported names in this library and in oracle/_ref/libarbor_ref.so,
 * so one Python wrapper drives either. */
#define EXPORT __attribute__((visibility("default")))

EXPORT int oracle_is_f64(void) {
#ifdef ORACLE_F64
  return 1;
#else
  return 0;
#endif
}
EXPORT void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
EXPORT int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
/* Thread counts per growth level as the harness dispatches them
 * (tests/native_harness.cpp:45). */
EXPORT void oracle_growTree(float* B, int level, int seed) {
  int n = level == 0 ? 9 : level == 1 ? 12 : level == 2 ? 72 : level == 3 ? 288 : 1728;
  for (int i = 0; i < n; i++) grow_one(B, level, seed, i);
}
EXPORT void oracle_makePrimitives(const float* B, float* P, int seed) { for (int i = 0; i < K_CAPACITY; i++) prim_one(B, P, seed, i); }
EXPORT void oracle_makeKeys(const float* P, uint32_t* Keys, uint32_t* Order) { for (int i = 0; i < K_CAPACITY; i++) key_one(P, Keys, Order, i); }
/* One bitonic compare-exchange stage over all threads (Arbor.cu:140). */
EXPORT void oracle_sortPass(uint32_t* Keys, uint32_t* Order, int distance, int span) {
  for (int i = 0; i < K_CAPACITY; i++) {
    int j = i ^ distance;
    if (j <= i) continue;
    uint32_t a = Keys[i], b = Keys[j], ia = Order[i], ib = Order[j];
    int greater = a > b || (a == b && ia > ib), ascending = (i & span) == 0;
    if (greater == ascending) { Keys[i] = b; Keys[j] = a; Order[i] = ib; Order[j] = ia; }
  }
}
/* Independent (key, index) sort, the harness's std::sort of pairs
 * (tests/native_harness.cpp:47): a stable LSD radix sort by key over pairs
 * already in index order yields the same lexicographic order. */
EXPORT void oracle_sortPairs(uint32_t* Keys, uint32_t* Order, int n) {
  uint32_t* k2 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
  uint32_t* o2 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
  /* order-preserving tie break: sort by index first, then stably by key */
  for (int pass = 0; pass < 2; pass++) {
    uint32_t* key = pass == 0 ? Order : Keys;
    for (int shift = 0; shift < 32; shift += 8) {
      size_t cnt[257] = {0};
      for (int i = 0; i < n; i++) cnt[((key[i] >> shift) & 255u) + 1]++;
      for (int d = 0; d < 256; d++) cnt[d + 1] += cnt[d];
      for (int i = 0; i < n; i++) { size_t at = cnt[(key[i] >> shift) & 255u]++; k2[at] = Keys[i]; o2[at] = Order[i]; }
      memcpy(Keys, k2, sizeof(uint32_t) * (size_t)n); memcpy(Order, o2, sizeof(uint32_t) * (size_t)n);
    }
  }
  free(k2); free(o2);
}
/* Arbor.cu:141 */
EXPORT void oracle_makeBounds(const float* P, const uint32_t* Order, float* Nodes) {
  for (int i = 0; i < K_CAPACITY; i++) {
    int id = (int)Order[i], b = (K_CAPACITY + i) * 8;
    st3(Nodes, b, bound_lo(P, id)); st3(Nodes, b + 4, bound_hi(P, id));
    Nodes[b + 3] = P[id * K_PS + 3] >= 0.0f ? 1.0f : 0.0f;
    Nodes[b + 7] = (float)id;
  }
}
/* Arbor.cu:142 */
EXPORT void oracle_reduceBounds(float* Nodes, int first) {
  for (int i = 0; i < first; i++) {
    int b = (first + i) * 8, a = b * 2, c = a + 8;
    st3(Nodes, b, vmin(ld3(Nodes, a), ld3(Nodes, c)));
    st3(Nodes, b + 4, vmax(ld3(Nodes, a + 4), ld3(Nodes, c + 4)));
    Nodes[b + 3] = Nodes[a + 3] + Nodes[c + 3];
    Nodes[b + 7] = -1.0f;
  }
}
/* Arbor.cu:181 */
EXPORT void oracle_initCamera(float* C, const float* P, int seed) {
  (void)P;
  for (int i = 0; i < 64; i++) C[i] = 0.0f;
  C[12] = -0.45f; C[13] = 0.63f; C[14] = 0.90f; C[20] = 1.18f; C[22] = 1.0f; C[23] = 1.0f; C[31] = (float)seed; C[44] = 1.0f;
  pose(C, V(2.0f, 1.72f, 18.0f), K_PI, 0.0f);
}
/* Arbor.cu:182 */
EXPORT void oracle_updateCamera(float* C, const float* I, const float* P, float delta, int width, int height) {
  (void)P;
  C[10] = 0.0f; C[24] += 1.0f;
  real dt = clampr(delta, 0.0f, 0.1f);
  v3 old = ld3(C, 0);
  if (I[5] > 0.0f) preset(C, (int)I[5]);
  if (I[7] > 0.0f) { C[11] = C[11] > 0.0f ? 0.0f : 0.60f; C[10] = 1.0f; }
  if (I[9] > 0.0f) { C[15] = (float)(((int)C[15] + 1) % 4); C[10] = 1.0f; }
  if (I[10] > 0.0f) { C[22] = 1.0f - C[22]; C[10] = 1.0f; }
  if (I[8] != 0.0f) { C[12] = (float)(C[12] + I[8] * dt * 0.6f); C[10] = 1.0f; }
  if (I[12] != 0.0f) { C[20] = (float)clampr(C[20] + I[12] * dt, 0.25f, 3.0f); C[10] = 1.0f; }
  if (C[11] > 0.0f) { C[8] = (float)(C[8] + dt); C[10] = 1.0f; }
  C[16] = (float)(C[16] - I[0] * 0.00225f);
  C[17] = (float)clampr(C[17] - I[1] * 0.0020f, -1.45f, 1.45f);
  real yaw = C[16], cp = COS(C[17]);
  v3 look = unit(V(SIN(yaw) * cp, SIN(C[17]), COS(yaw) * cp));
  v3 walk = unit(V(SIN(yaw), 0.0f, COS(yaw)));
  v3 right = unit(V(walk.z, 0.0f, -walk.x));
  real speed = I[16] > 0.5f ? 10.5f : 4.2f;
  v3 move = vadd(vscale(walk, I[15]), vscale(right, I[13]));
  if (dot(move, move) > 0.0001f) move = vscale(vscale(unit(move), speed), dt);
  v3 eye = vadd(ld3(C, 0), move);
  eye.y = 1.72f;
  st3(C, 0, eye); st3(C, 4, vadd(eye, look));
  C[27] = C[16]; C[28] = C[17]; C[3] = 1.0f; C[18] = 1.0f;
  if (len3(vsub(eye, old)) > 0.000001f || I[0] != 0.0f || I[1] != 0.0f) C[10] = 1.0f;
  if (C[32] != (float)width || C[33] != (float)height) { C[10] = 1.0f; C[32] = (float)width; C[33] = (float)height; }
  C[9] = C[10] > 0.5f ? 0.0f : fminf(255.0f, C[9] + 1.0f);
}
/* Image passes over rows [y0, y1), OpenMP over rows with the harness's
 * schedule (tests/native_harness.cpp:36-39).  `single` selects the one-tree
 * identity-instance scene instead of the 324-tree forest. */
EXPORT void oracle_tracePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int w, int h, int y0, int y1, int single) {
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < w; x++) trace_px(P, Nodes, Order, C, Hit, w, h, x, y, single, NULL);
}
EXPORT void oracle_shadePixels(const float* P, const float* Nodes, const uint32_t* Order, const float* C, const float* Hit, float* Linear, float* Guide, int w, int h, int y0, int y1, int single) {
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < w; x++) shade_px(P, Nodes, Order, C, Hit, Linear, Guide, w, h, x, y, single, NULL);
}
/* tracePixels / shadePixels over a forest of several species: instance t
 * takes its geometry from scene of[t] (P[of[t]], Nodes[of[t]],
 * Order[of[t]]), everything else as in the reference's forest (rows
 * y0..y1-1).  No reference counterpart: the reference's instances all share
 * one resident tree (README.md:8, docs/ARCHITECTURE.md:5); with every of[t]
 * equal this is its tracePixels / shadePixels. */
EXPORT void oracle_tracePixelsSpecies(const float* const* P, const float* const* N, const uint32_t* const* Order, const int* of, const float* C,
                                      float* Hit, int w, int h, int y0, int y1) {
  species_set sp = {P, N, Order, of};
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < w; x++) trace_px(P[0], N[0], Order[0], C, Hit, w, h, x, y, 0, &sp);
}
EXPORT void oracle_shadePixelsSpecies(const float* const* P, const float* const* N, const uint32_t* const* Order, const int* of, const float* C,
                                      const float* Hit, float* Linear, float* Guide, int w, int h, int y0, int y1) {
  species_set sp = {P, N, Order, of};
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < w; x++) shade_px(P[0], N[0], Order[0], C, Hit, Linear, Guide, w, h, x, y, 0, &sp);
}
/* The shading normal shadePixels computes for each pixel (world space,
 * facing the camera), zero for sky pixels: rows y0..y1-1 of Normal (w*h
 * float4, .w = 0).  The reference keeps this value inside shadePixels; its
 * view mode 3 writes it as n * 0.5 + 0.5 (Arbor.cu:286). */
EXPORT void oracle_shadeNormals(const float* P, const float* C, const float* Hit, float* Normal, int w, int h, int y0, int y1, int single) {
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < w; x++) {
      int b = (y * w + x) * 4;
      v3 n = V(0.0f, 0.0f, 0.0f);
      if (Hit[b] < K_FAR) n = shade_surface(P, C, Hit, cam_pos(C), primary_dir(C, x, y, w, h), b, single).n;
      st3(Normal, b, n); Normal[b + 3] = 0.0f;
    }
}
EXPORT void oracle_filterLighting(const float* Linear, const float* Guide, const float* Hit, float* Filtered, const float* C, int w, int h, int y0, int y1) {
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < w; x++) filter_px(Linear, Guide, Hit, Filtered, C, w, h, x, y);
}
EXPORT void oracle_resolvePixels(const float* Filtered, float* History, uint32_t* Pixels, const float* C, int w, int h, int y0, int y1) {
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < w; x++) resolve_px(Filtered, History, Pixels, C, w, h, x, y);
}
/* Single pixels at explicit coordinates (used for the FP64 rerun of
 * mismatching pixels). */
EXPORT void oracle_tracePixelList(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, int w, int h, const int* xy, int n, int single) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < n; i++) trace_px(P, Nodes, Order, C, Hit, w, h, xy[2 * i], xy[2 * i + 1], single, NULL);
}
/* Function-level probes (the harness's checks at tests/native_harness.cpp:84-92). */
EXPORT void oracle_traceTreeRay(const float* P, const float* Nodes, const uint32_t* Order, const float* ro, const float* rd, float cone, float time, float wind, float best, int ignore, int shadows, float* out) {
  v2 r = walk_tree(P, Nodes, V(ro[0], ro[1], ro[2]), V(rd[0], rd[1], rd[2]), cone, time, wind, best, ignore, shadows, Order);
  out[0] = (float)r.x; out[1] = (float)r.y;
}
EXPORT float oracle_objectT(const float* P, int id, const float* ro, const float* rd, float fp, float time, float wind, int refine) {
  return (float)object_hit(P, id, V(ro[0], ro[1], ro[2]), V(rd[0], rd[1], rd[2]), fp, time, wind, refine);
}
EXPORT float oracle_leafT(const float* P, int id, const float* ro, const float* rd, float fp, float time, float wind) {
  return (float)leaf_hit(P, id, V(ro[0], ro[1], ro[2]), V(rd[0], rd[1], rd[2]), fp, time, wind);
}
EXPORT void oracle_boxSpan(const float* ro, const float* rd, const float* lo, const float* hi, float* out) {
  v2 s = box_span(V(ro[0], ro[1], ro[2]), V(rd[0], rd[1], rd[2]), V(lo[0], lo[1], lo[2]), V(hi[0], hi[1], hi[2]));
  out[0] = (float)s.x; out[1] = (float)s.y;
}
EXPORT void oracle_bounds(const float* P, int id, float* lo, float* hi) {
  v3 a = bound_lo(P, id), b = bound_hi(P, id);
  lo[0] = (float)a.x; lo[1] = (float)a.y; lo[2] = (float)a.z; hi[0] = (float)b.x; hi[1] = (float)b.y; hi[2] = (float)b.z;
}
EXPORT float oracle_barkCut(const float* P, int id, const float* p, float fp) { return (float)bark_relief(P, id, V(p[0], p[1], p[2]), fp); }
EXPORT float oracle_bandWeight(float period, float fp) { return (float)band(period, fp); }
EXPORT float oracle_rnd(int n, int seed) { return (float)rnd(n, seed); }
EXPORT int oracle_forestSeed(int tree, int ws) { return tree_seed(tree, ws); }
/* Per-tree instance: pos.xyz, scale, yaw, phase (Arbor.cu:57-66, 247). */
EXPORT void oracle_forestInstance(int tree, int ws, float* out) {
  v3 p = tree_pos(tree, ws);
  out[0] = (float)p.x; out[1] = (float)p.y; out[2] = (float)p.z;
  out[3] = (float)tree_scale(tree, ws); out[4] = (float)tree_yaw(tree, ws);
  out[5] = (float)((real)(tree_seed(tree, ws) & 8191) * 0.0017f);
}
/* Exhaustive nearest hit over all objects, the harness's BVH cross-check
 * (tests/native_harness.cpp:85). */
EXPORT void oracle_exhaustiveRay(const float* P, const float* ro, const float* rd, float cone, float* out) {
  v3 o = V(ro[0], ro[1], ro[2]), d = V(rd[0], rd[1], rd[2]);
  real nearest = K_FAR; int winner = -1;
  for (int id = 0; id < K_OBJECTS; id++) {
    v2 a = box_span(o, d, bound_lo(P, id), bound_hi(P, id));
    if (a.y < FMAX(0.0001f, a.x) || a.x > nearest) continue;
    real fp = FMAX(0.000005f, cone * FMAX(0.05f, a.x));
    real t = object_hit(P, id, o, d, fp, 0.0f, 0.0f, 1);
    if (t < nearest) { nearest = t; winner = id; }
  }
  out[0] = (float)nearest; out[1] = (float)winner;
}
/* The harness's check inputs and sweeps (tests/native_harness.cpp:83, 89-92),
 * computed in this library's own arithmetic. */
EXPORT void oracle_harnessRay(int ray, float* ro, float* rd) {
  v3 o = V(rnd(ray, 198) * 24.0f - 12.0f, 1.0f + rnd(ray, 31) * 14.0f, rnd(ray, 78) * 24.0f - 12.0f);
  v3 target = V(rnd(ray, 211) * 10.0f - 5.0f, 2.0f + rnd(ray, 433) * 8.0f, rnd(ray, 123) * 10.0f - 5.0f);
  v3 d = unit(vsub(target, o));
  ro[0] = (float)o.x; ro[1] = (float)o.y; ro[2] = (float)o.z;
  rd[0] = (float)d.x; rd[1] = (float)d.y; rd[2] = (float)d.z;
}
EXPORT void oracle_footprintSweep(const float* P, int id, float* out) {
  int mono = 1, finite = 1; real last = 1.0f, jump = 0.0f;
  v3 point = vadd(ld3(P, id * K_PS), V(0.0f, 0.0f, P[id * K_PS + 7]));
  real prev = bark_relief(P, id, point, 0.000001f);
  for (int i = 0; i < 10000; i++) {
    real f = 0.000001f * POW(100000.0f, (real)i / 9999);
    real w = band(0.065f, f);
    mono &= w <= last + 1e-7f; last = w;
    real cut = bark_relief(P, id, point, f);
    real dj = FABS(cut - prev); if (dj > jump) jump = dj;
    prev = cut; finite &= isfinite(cut) ? 1 : 0;
  }
  out[0] = (float)jump; out[1] = (float)mono; out[2] = (float)finite;
}
EXPORT void oracle_leafPair(const float* P, int k, float* out) {
  int id = K_WOOD + k * 431, b = id * K_PS;
  v3 u = ld3(P, b + 4), n = ld3(P, b + 12);
  v3 p = vadd(vadd(ld3(P, b), vscale(u, P[b + 16] + P[b + 7] * 0.5f)), vscale(n, 0.10f));
  v3 rd = vscale(n, -1.0f);
  out[0] = (float)leaf_hit(P, id, p, rd, 0.00001f, 0.0f, 0.0f);
  out[1] = (float)leaf_hit(P, id, p, rd, 0.05f, 0.0f, 0.0f);
}
/* One frame (trace, shade, filter, resolve) over a list of rows: each pass is
 * one OpenMP loop over the listed rows with the harness's schedule, so a
 * sample of rows spread over the image keeps every host thread busy. */
EXPORT void oracle_frameRows(const float* P, const float* Nodes, const uint32_t* Order, const float* C, float* Hit, float* Linear, float* Guide,
                             float* Filtered, float* History, uint32_t* Pixels, int w, int h, const int* rows, int n, int single) {
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < n; i++)
    for (int x = 0; x < w; x++) trace_px(P, Nodes, Order, C, Hit, w, h, x, rows[i], single, NULL);
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < n; i++)
    for (int x = 0; x < w; x++) shade_px(P, Nodes, Order, C, Hit, Linear, Guide, w, h, x, rows[i], single, NULL);
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < n; i++)
    for (int x = 0; x < w; x++) filter_px(Linear, Guide, Hit, Filtered, C, w, h, x, rows[i]);
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < n; i++)
    for (int x = 0; x < w; x++) resolve_px(Filtered, History, Pixels, C, w, h, x, rows[i]);
}
