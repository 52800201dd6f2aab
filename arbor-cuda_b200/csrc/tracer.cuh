// tracer.cuh - forest ray state machine.
//
// One ray per lane, advanced through the phases of the reference's
// traceForest/traceTree (Arbor.cu:220-251):
//
//   DDA   one forest cell: bounding-sphere test, tree entry, cell advance
//   TREE  one BVH step: test both children of an accepted interior node,
//         descend nearest-first, or pop a deferred sibling
//   LEAF  the ray sits at an accepted leaf (a candidate primitive)
//   TREE_END  the tree has no accepted node left (finish_tree folds it in)
//   DONE  the ray's result is final
//
// Every step makes the reference's tests on the same values (same cells,
// same nodes, same acceptance tests).  For primary rays the order differs:
// of two accepted children the reference descends first into the one the ray
// enters first; here it is the one whose span inside the ray's range (entry
// clamped at the ray origin) has the nearer midpoint, which finds near hits
// sooner and prunes more.  The result is the nearest hit over the accepted
// leaf boxes whatever the order (warpbatch.cuh gives the argument), as long
// as each hit lies inside its primitive's box; between exactly equal hit
// distances (leaves sharing a petiole base, wood segments sharing a joint)
// the one the reference meets first is kept (ref_before).  Shadow segments
// keep the reference's order: with the midpoint order their visibility
// differed from the reference's on a few pixels of a 1080p forest frame.
#pragma once
#include "arbor_scene.cuh"

namespace arbor {

enum RayPhase : int { kPhDDA = 0, kPhTree = 1, kPhLeaf = 2, kPhDone = 3, kPhIdle = 4, kPhBlocked = 5, kPhTreeEnd = 6 };

struct Ray {
  f3 ro, rd;        // world ray
  float best;       // world-space nearest t so far
  float found;      // primitive id of best (as the reference's float), -1
  int foundTree;    // tree of best, -1
  // forest DDA (Arbor.cu:241-248)
  int ix, iz, sx, sz, step;
  float tx, tz, dx, dz, exit;
  // the tree being traversed, in its local frame (Arbor.cu:247)
  int tree;
  f3 lro, lrd, linv;
  float lcone, lbest, ltime, lsc;
  int lfound;       // lbest's leaf slot (primary rays) or record id (shadow segments), -1
  int node, depth;
  uint32_t pending;
  float spanx;
  int phase;
  int species;      // scene of the tree being traversed (forest of several species; 0 otherwise)
};

struct TraceCtx {
  const float* P;
  const float* Nodes;
  const uint32_t* Order;
  const Instance* inst;   // forest instance table (the world-seed registry's, or shared memory)
  float cone, time, wind;
  bool refine;            // primary rays: wood refined by the SDF march, their own visiting order,
                          // ties settled by ref_before; false for shadow segments
  bool forest;            // false: the single-tree scene (identity instance)
  bool species = false;   // true: a forest of several species, P / Nodes / Order holding one scene
                          // per species back to back, instance t on scene species_of[t] (or
                          // inst[t].species when species_of is null)
  const uint8_t* species_of = nullptr;
};

// The scene of tree `tree` (0 unless the forest has several species).
__device__ __forceinline__ int tree_species(const TraceCtx& c, int tree) {
  if (!c.species || tree < 0) return 0;
  return c.species_of != nullptr ? (int)c.species_of[tree] : c.inst[tree].species;
}

// The records of scene `s` (s = 0 unless the forest has several species).
__device__ __forceinline__ const float* scene_P(const TraceCtx& c, int s) { return c.species ? c.P + (size_t)s * (kCapacity * kPS) : c.P; }
__device__ __forceinline__ const float* scene_nodes(const TraceCtx& c, int s) {
  return c.species ? c.Nodes + (size_t)s * (kNodeCount * 8) : c.Nodes;
}
__device__ __forceinline__ const uint32_t* scene_order(const TraceCtx& c, int s) { return c.species ? c.Order + (size_t)s * kCapacity : c.Order; }

__device__ __forceinline__ void load_node(const TraceCtx& c, const Ray& r, int n, float4& lo, float4& hi) {
  const float* nodes = scene_nodes(c, r.species);
  lo = ldg4(nodes, 2 * n);
  hi = ldg4(nodes, 2 * n + 1);
}

// Tree entry with the root test (Arbor.cu:221-223).  Returns true when the
// root is accepted and traversal starts.
__device__ __forceinline__ bool enter_tree(const TraceCtx& c, Ray& r) {
  r.lfound = -1;
  r.node = 1;
  r.depth = 0;
  r.pending = 0u;
  float4 lo, hi;
  load_node(c, r, 1, lo, hi);
  return node_accept(lo, hi, r.lro, r.linv, r.lbest, r.spanx);
}

// After a cell's tree: next crossing, exit test, advance (Arbor.cu:248).
__device__ __forceinline__ void dda_advance(Ray& r) {
  float next = r.tx < r.tz ? r.tx : r.tz;
  if (next > r.exit || next > r.best) {
    r.phase = kPhDone;
    return;
  }
  if (r.tx < r.tz) {
    r.ix += r.sx;
    r.tx += r.dx;
  } else {
    r.iz += r.sz;
    r.tz += r.dz;
  }
  r.step++;
  r.phase = kPhDDA;
}

// The tree is exhausted: fold its local result into the world result
// (Arbor.cu:247 for the forest; traceTree's return for the single tree).
__device__ __forceinline__ void finish_tree(const TraceCtx& c, Ray& r) {
  if (!c.forest) {
    r.best = r.lbest;
    r.found = r.lfound >= 0 && c.refine ? (float)__ldg(scene_order(c, r.species) + r.lfound) : (float)r.lfound;
    r.phase = kPhDone;
    return;
  }
  if (r.lfound >= 0 && r.lbest * r.lsc < r.best) {
    r.best = r.lbest * r.lsc;
    r.found = c.refine ? (float)__ldg(scene_order(c, r.species) + r.lfound) : (float)r.lfound;
    r.foundTree = r.tree;
  }
  dda_advance(r);
}

// Begin a trace of (ro, rd) with initial nearest `best` (Arbor.cu:236-244).
__device__ __forceinline__ void ray_begin(const TraceCtx& c, Ray& r, f3 ro, f3 rd, float best) {
  r.ro = ro;
  r.rd = rd;
  r.best = best;
  r.found = -1.0f;
  r.foundTree = -1;
  r.tree = -1;
  r.species = 0;
  if (!c.forest) {
    r.lro = ro;
    r.lrd = rd;
    r.linv = inv3(rd);
    r.lcone = c.cone;
    r.lbest = best;
    r.ltime = c.time;
    r.lsc = 1.0f;
    r.phase = enter_tree(c, r) ? kPhTree : kPhDone;
    if (r.phase == kPhDone) finish_tree(c, r);
    return;
  }
  const float half = (float)kSide * kSpacing * 0.5f;
  f2 worldSpan = box_span(ro, rd, mk(-half, -1.2f, -half), mk(half, 13.5f, half));
  float enter = fmaxf(0.0f, worldSpan.x);
  r.exit = fminf(best, worldSpan.y);
  if (r.exit < enter) {
    r.phase = kPhDone;
    return;
  }
  f3 pos = ro + rd * (enter + 0.0002f);
  r.ix = (int)floorf(pos.x / kSpacing + (float)kSide * 0.5f + 0.5f);
  r.iz = (int)floorf(pos.z / kSpacing + (float)kSide * 0.5f + 0.5f);
  r.sx = rd.x >= 0.0f ? 1 : -1;
  r.sz = rd.z >= 0.0f ? 1 : -1;
  float invx = inv_safe(rd.x);
  float invz = inv_safe(rd.z);
  float bx = ((float)(r.ix - kSide / 2) + (r.sx > 0 ? 0.5f : -0.5f)) * kSpacing;
  float bz = ((float)(r.iz - kSide / 2) + (r.sz > 0 ? 0.5f : -0.5f)) * kSpacing;
  r.tx = (bx - ro.x) * invx;
  r.tz = (bz - ro.z) * invz;
  r.dx = kSpacing * fabsf(invx);
  r.dz = kSpacing * fabsf(invz);
  r.step = 0;
  r.phase = kPhDDA;
}

// One forest cell (Arbor.cu:245-247).
__device__ __forceinline__ void dda_step(const TraceCtx& c, Ray& r) {
  if (r.step >= 48 || r.ix < 0 || r.iz < 0 || r.ix >= kSide || r.iz >= kSide) {
    r.phase = kPhDone;
    return;
  }
  int tree = r.iz * kSide + r.ix;
  ARBOR_COUNT(kEvCell);
  const Instance& it = c.inst[tree];
  float broad = sphere_t(r.ro, r.rd, mk(it.px + 0.0f, 0.0f + it.cy, it.pz + 0.0f), it.rad);
  if (broad < r.best) {
    ARBOR_COUNT(kEvTree);
    r.tree = tree;
    r.lro = to_local_point(r.ro, it);
    r.lrd = to_local_dir(r.rd, it);
    r.linv = inv3(r.lrd);
    r.lcone = c.cone / it.sc;
    r.lbest = r.best / it.sc;
    r.ltime = c.time + it.phase;
    r.lsc = it.sc;
    if (c.species) r.species = tree_species(c, tree);
    if (enter_tree(c, r)) {
      r.phase = kPhTree;
      return;
    }
    finish_tree(c, r);  // root rejected: traceTree returns (best, -1)
    return;
  }
  dda_advance(r);
}

// Entry distances of the deferred siblings of one lane, one per BVH level
// 1-15 (a sibling is deferred below the root only), in shared memory with a
// stride of 32 floats (the warp's lanes side by side).
struct SiblingSpans {
  float* lane;  // &spans[0][lane] of a [15][32] array
  __device__ __forceinline__ float& at(int level) const { return lane[(level - 1) * 32]; }
};

// Pop deferred siblings, deepest first, until one is still accepted (the
// reference's stack pop and re-test, Arbor.cu:223, 227).  A sibling is
// deferred only when its box test passed, and of that test only the
// comparison span.x < best depends on the ray's state, so the re-test is
// that comparison on the span.x recorded at the push: the same decision as
// reloading the node and repeating the slab test, without the load.
__device__ __forceinline__ bool pop_next(Ray& r, const SiblingSpans& sib) {
  while (r.pending != 0u) {
    int level = 31 - __clz(r.pending);
    r.pending &= ~(1u << level);
    r.node = (r.node >> (r.depth - level)) ^ 1;
    r.depth = level;
    const float sx = sib.at(level);
    if (sx < r.lbest) {
      r.spanx = sx;
      return true;
    }
  }
  return false;
}

// True when leaf slot a comes before leaf slot b in the reference's visiting
// order of this tree (Arbor.cu:224-225): a depth-first order in which, at
// every node, the child with the smaller entry span.x goes first (the left
// one only when its entry is strictly smaller).  The two leaves part at their
// lowest common ancestor, so the order is that node's decision, made again
// here on the same values (ro, inv: the tree-local ray).  Ties are rare; the
// function stays out of line, away from the traversal's instruction stream.
static __device__ __noinline__ bool ref_before_at(const float* __restrict__ Nodes, f3 ro, f3 inv, int a, int b) {
  int na = a + kCapacity, nb = b + kCapacity;
  while ((na >> 1) != (nb >> 1)) {
    na >>= 1;
    nb >>= 1;
  }
  const int left = na & ~1;
  const float4 llo = ldg4(Nodes, 2 * left), lhi = ldg4(Nodes, 2 * left + 1);
  const float4 rlo = ldg4(Nodes, 2 * left + 2), rhi = ldg4(Nodes, 2 * left + 3);
  const float lx = box_span_inv(ro, inv, xyz(llo), xyz(lhi)).x;
  const float rx = box_span_inv(ro, inv, xyz(rlo), xyz(rhi)).x;
  return (na == left) == (lx < rx);
}
__device__ __forceinline__ bool ref_before(const TraceCtx& c, const Ray& r, int a, int b) {
  return ref_before_at(scene_nodes(c, r.species), r.lro, r.linv, a, b);
}

// One interior step (Arbor.cu:224-225, 227).
__device__ __forceinline__ void tree_step(const TraceCtx& c, Ray& r, const SiblingSpans& sib) {
  if (r.node >= kCapacity) {
    r.phase = kPhLeaf;
    return;
  }
  int left = r.node * 2;
  float4 llo, lhi, rlo, rhi;
  load_node(c, r, left, llo, lhi);
  load_node(c, r, left + 1, rlo, rhi);
  f2 ls, rs;
  bool lh = node_accept_span(llo, lhi, r.lro, r.linv, r.lbest, ls);
  bool rh = node_accept_span(rlo, rhi, r.lro, r.linv, r.lbest, rs);
  const float lx = ls.x, rx = rs.x;
  if (lh || rh) {
    r.depth++;
    if (lh && rh) {
      // Primary rays: the child whose span inside the ray's range (entry
      // clamped at the origin) has the nearer midpoint first.  Shadow
      // segments: the reference's order, the nearer entry first.
      const bool l = c.refine ? fmaxf(lx, 0.0f) + ls.y < fmaxf(rx, 0.0f) + rs.y : lx < rx;
      r.pending |= 1u << r.depth;
      sib.at(r.depth) = l ? rx : lx;
      r.node = l ? left : left + 1;
      r.spanx = l ? lx : rx;
    } else if (lh) {
      r.node = left;
      r.spanx = lx;
    } else {
      r.node = left + 1;
      r.spanx = rx;
    }
    if (r.node >= kCapacity) r.phase = kPhLeaf;
    return;
  }
  if (pop_next(r, sib)) {
    r.phase = r.node >= kCapacity ? kPhLeaf : kPhTree;
    return;
  }
  // The tree is exhausted.  The driver folds the tree's result in
  // (finish_tree) once every test it queued for this tree has come back.
  r.phase = kPhTreeEnd;
}

}  // namespace arbor
