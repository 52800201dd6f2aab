// warpbatch.cuh - warp-batched primitive tests for forest rays.
//
// The reference tests one candidate primitive at a time inside its BVH loop
// (Arbor.cu:226).  On a GPU that serialises a warp: the rare, long tests
// (the leaf Newton solve, the bark SDF march) run with one or two lanes
// active.  Here each lane traverses on its own (tracer.cuh) and, instead of
// testing a candidate, queues it (up to Q per lane) and keeps
// traversing; when every lane is blocked (queue full, tree finished, ray
// done) the warp runs all queued tests as compacted jobs - leaf clips, then
// Newton solves of the clips that pass, wood tests and the rest - one job per
// lane, and each lane applies its results in candidate order.
//
// Why results do not change: the primitive surfaces lie inside their own
// bounding boxes (the leaf-frame box, petiole, bark relief and ellipsoid are
// built inside boundLow/boundHigh, Arbor.cu:132-133), so a hit t is not below
// the box's entry span.x, and the reference only prunes boxes with span.x >=
// best.  A primitive it prunes then cannot beat its final answer, and the
// answer is the nearest hit over the accepted leaf boxes whatever the order
// of the tests.  (Where a hit does fall before its box's entry, the reference
// can prune the box after a farther hit while this pass keeps the nearer
// one: 2 pixels of a 1080p forest frame, measured against the in-order
// entry points.)  Traversing past a queued candidate with
// the not-yet-updated best only adds tests that cannot win; the footprint of
// each test depends only on its own box (Arbor.cu:226).  Between exactly
// equal t values the reference keeps the one it meets first; batch_apply
// decides such ties by the reference's visiting order (ref_before).  The DDA
// advance and tree hand-over wait for all results, so they use the
// reference's best.
#pragma once
#include "tracer.cuh"

namespace arbor {

constexpr int kQueue = 16;       // candidates a lane may queue: the most at which a 256-thread CTA's 8 warp
                                 // batches (111 KB) still leave 2 CTAs per SM, the instance table read from
                                 // global memory (on the 1080p forest walk, shadow segments 10 % faster at
                                 // 12 than at 8 and 5 % faster again at 16; primary rays 6 % and 4 %)
constexpr int kNewtonCap = 64;   // pending Newton solves per warp
enum JobClass : int { kJobLeaf = 0, kJobWood = 1, kJobMisc = 2, kJobNone = 3 };

// Per-warp shared-memory batch for a queue depth of Q candidates per lane.
template <int Q>
struct WarpBatchQ {
  static constexpr int kQ = Q;
  static constexpr int kWarpJobs = 32 * Q;
  float4 rayO[32];             // owner lane's local ray origin and wind time
  float4 rayD[32];             // owner lane's local ray direction
  int rayS[32];                // owner lane's scene (forest of several species)
  LeafSolve solve[kNewtonCap];
  int prim[kWarpJobs];         // lane-major queue: lane * Q + k (leaf slot, then record id)
  float fp[kWarpJobs];
  float res[kWarpJobs];
  signed char cls[kWarpJobs];  // test class of a queued candidate (JobClass)
  short slot[kWarpJobs];       // leaf slot of a queued candidate (primary rays)
  short job[kWarpJobs];        // compacted job list: leaf clips, wood tests, the rest
  short solveJob[kNewtonCap];
  float sib[15][32];           // deferred siblings' span.x, BVH levels 1-15 (SiblingSpans)
};
using WarpBatch = WarpBatchQ<kQueue>;

// Advance one lane until its queue is full, its tree is finished with tests
// pending, or its ray is done.
template <class WB>
__device__ __forceinline__ void batch_advance(const TraceCtx& c, Ray& r, WB& b, int lane, int& nq) {
  const SiblingSpans sib{&b.sib[0][lane]};
  while (r.phase == kPhDDA || r.phase == kPhTree || r.phase == kPhLeaf || r.phase == kPhTreeEnd) {
    if (r.phase == kPhDDA) {
      dda_step(c, r);
      continue;
    }
    if (r.phase == kPhTree) {
      tree_step(c, r, sib);
      continue;
    }
    if (r.phase == kPhTreeEnd) {
      if (nq > 0) return;  // the tree's queued tests must come back first
      finish_tree(c, r);
      continue;
    }
    // an accepted leaf: queue its slot (the Order entry and the record are
    // read when the warp runs its tests, off the traversal's load chain)
    int q = lane * WB::kQ + nq++;
    b.prim[q] = r.node - kCapacity;
    if (c.refine) b.slot[q] = (short)(r.node - kCapacity);
    b.fp[q] = fmaxf(0.000005f, r.lcone * fmaxf(0.05f, r.spanx));
    if (nq == WB::kQ) {
      r.phase = kPhBlocked;  // resume with the pop once results are in
      return;
    }
    if (pop_next(r, sib)) {
      r.phase = r.node >= kCapacity ? kPhLeaf : kPhTree;
    } else {
      r.phase = kPhTreeEnd;  // the tree's queued tests must come back first
      return;
    }
  }
}

// Run every queued test of the warp.  All 32 lanes call it together.
template <class WB>
__device__ __forceinline__ void batch_tests(const TraceCtx& c, const Ray& r, WB& b, int lane, int nq) {
  const unsigned full = 0xffffffffu;
  const unsigned lt = (1u << lane) - 1u;
  if (nq > 0) {
    b.rayO[lane] = make_float4(r.lro.x, r.lro.y, r.lro.z, r.ltime);
    b.rayD[lane] = make_float4(r.lrd.x, r.lrd.y, r.lrd.z, 0.0f);
    if (c.species) b.rayS[lane] = r.species;
  }
  // Resolve each queued leaf slot to its record and test class: leaf clip,
  // wood (tube + SDF march, primary rays), the rest (stones, shadow-ray wood,
  // unused records) or none (an Order entry past the records, skipped and
  // not read).  Per-lane counts by class, scanned across the warp.
  int nl = 0, nw = 0, nm = 0;
  for (int k = 0; k < nq; k++) {
    const int q = lane * WB::kQ + k;
    const uint32_t uid = __ldg(scene_order(c, r.species) + b.prim[q]);
    int cls = kJobNone;
    if (uid < (uint32_t)kCapacity) {
      const int t = (int)ldg4(scene_P(c, r.species), (int)uid * 6).w;
      cls = t == 1 ? kJobLeaf : (t == 0 && c.refine) ? kJobWood : kJobMisc;
    } else {
      b.res[q] = kFar;
    }
    b.prim[q] = (int)uid;
    b.cls[q] = (signed char)cls;
    nl += cls == kJobLeaf;
    nw += cls == kJobWood;
    nm += cls == kJobMisc;
  }
  int sl = nl, sw = nw, sm = nm;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int a = __shfl_up_sync(full, sl, o), d = __shfl_up_sync(full, sw, o), e = __shfl_up_sync(full, sm, o);
    if (lane >= o) {
      sl += a;
      sw += d;
      sm += e;
    }
  }
  const int totL = __shfl_sync(full, sl, 31), totW = __shfl_sync(full, sw, 31), totM = __shfl_sync(full, sm, 31);
  int ol = sl - nl, ow = totL + sw - nw, om = totL + totW + sm - nm;
  for (int k = 0; k < nq; k++) {
    int q = lane * WB::kQ + k;
    int cls = b.cls[q];
    if (cls == kJobLeaf)
      b.job[ol++] = (short)q;
    else if (cls == kJobWood)
      b.job[ow++] = (short)q;
    else if (cls == kJobMisc)
      b.job[om++] = (short)q;
  }
  __syncwarp();
  // Leaf clips, 32 jobs at a time while fewer than 32 Newton solves are
  // pending; the clips that pass queue a Newton solve; a full pass of 32
  // solves (or the rest, once every clip is done) runs at the single call site
  // of leaf_newton below.
  int nN = 0;
  for (int base = 0;;) {
    if (base < totL && nN < 32) {
      int j = base + lane;
      bool solve = false;
      LeafSolve ls;
      int q = 0;
      if (j < totL) {
        q = b.job[j];
        int owner = q / WB::kQ;
        float4 o = b.rayO[owner], d = b.rayD[owner];
        float tube;
        const float* P = scene_P(c, c.species ? b.rayS[owner] : 0);
        solve = c.refine ? leaf_clip_outlined(P, b.prim[q], mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), o.w, c.wind, ls, tube)
                         : leaf_clip(P, b.prim[q], mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), o.w, c.wind, ls, tube);
        b.res[q] = tube;  // the result, or the Newton stage's starting best
      }
      unsigned m = __ballot_sync(full, solve);
      if (solve) {
        int pos = nN + __popc(m & lt);
        b.solve[pos] = ls;
        b.solveJob[pos] = (short)q;
      }
      nN += __popc(m);
      base += 32;
      __syncwarp();
      continue;
    }
    if (nN == 0) break;
    const int run = nN < 32 ? nN : 32;
    if (lane < run) {
      int qn = b.solveJob[lane];
      b.res[qn] = leaf_newton(b.solve[lane], leaf_shape(scene_P(c, c.species ? b.rayS[qn / WB::kQ] : 0), b.prim[qn]), b.res[qn], b.fp[qn]);
    }
    __syncwarp();
    if (lane < nN - run) {
      b.solve[lane] = b.solve[run + lane];
      b.solveJob[lane] = b.solveJob[run + lane];
    }
    nN -= run;
    __syncwarp();
  }
  // wood tests (tube + SDF march)
  for (int base = 0; base < totW; base += 32) {
    int j = base + lane;
    if (j < totW) {
      int q = b.job[totL + j];
      int owner = q / WB::kQ;
      float4 o = b.rayO[owner], d = b.rayD[owner];
      b.res[q] = wood_t(scene_P(c, c.species ? b.rayS[owner] : 0), b.prim[q], mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), b.fp[q], true);
    }
  }
  // stones, shadow-ray wood and unused records
  for (int base = 0; base < totM; base += 32) {
    int j = base + lane;
    if (j < totM) {
      int q = b.job[totL + totW + j];
      int owner = q / WB::kQ;
      float4 o = b.rayO[owner], d = b.rayD[owner];
      b.res[q] = object_t(scene_P(c, c.species ? b.rayS[owner] : 0), b.prim[q], mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), b.fp[q], o.w, c.wind,
                          c.refine);
    }
  }
  __syncwarp();
}

// Apply a lane's results and resume it.  A nearer hit replaces the best.  For
// primary rays (visited in their own order) an exactly equal one replaces it
// when the reference meets it first, so the kept primitive does not depend on
// the order of visits or tests; shadow segments visit in the reference's
// order, in which the first of equal hits is kept as it is.
template <class WB>
__device__ __forceinline__ void batch_apply(const TraceCtx& c, Ray& r, WB& b, int lane, int& nq) {
  for (int k = 0; k < nq; k++) {
    const int q = lane * WB::kQ + k;
    const float t = b.res[q];
    if (c.refine) {
      const int slot = b.slot[q];
      if (t < r.lbest || (t == r.lbest && r.lfound >= 0 && ref_before(c, r, slot, r.lfound))) {
        r.lbest = t;
        r.lfound = slot;
      }
    } else if (t < r.lbest) {
      r.lbest = t;
      r.lfound = b.prim[q];
    }
  }
  nq = 0;
  if (r.phase == kPhBlocked) {
    if (pop_next(r, SiblingSpans{&b.sib[0][lane]}))
      r.phase = r.node >= kCapacity ? kPhLeaf : kPhTree;
    else
      finish_tree(c, r);
  } else if (r.phase == kPhTreeEnd) {
    finish_tree(c, r);
  }
}

// Drive one warp's rays to completion.  Policy::done(r) is called for a
// finished ray and either starts a new trace on r or sets it idle.
template <class WB, class Policy>
__device__ __forceinline__ void batch_run(const TraceCtx& c, Ray& r, WB& b, Policy& policy) {
  const int lane = threadIdx.x & 31;
  int nq = 0;
  for (;;) {
    for (;;) {
      batch_advance(c, r, b, lane, nq);
      if (r.phase != kPhDone) break;
      policy.done(r);
    }
    const bool pending = nq > 0;
    if (!__any_sync(0xffffffffu, pending)) break;  // every lane idle
    batch_tests(c, r, b, lane, nq);
    batch_apply(c, r, b, lane, nq);
  }
}

// The pixels of a persistent CTA: the 8x4-pixel blocks blockIdx.x,
// blockIdx.x + gridDim.x, blockIdx.x + 2 gridDim.x, ... of a width x height
// image, handed out one pixel at a time, in block order, from a counter in
// shared memory.
struct PixelPool {
  int* next;  // shared-memory counter of pixels handed out by this CTA
  int width, height, blocks_x, blocks;
};

// Collective (all 32 lanes): hand the next pixels to the lanes in `idle`.
// Returns true for a lane that received a pixel inside the image; `past` is
// set for every lane once the CTA's blocks are used up.
__device__ __forceinline__ bool pool_take(const PixelPool& pool, unsigned idle, int lane, int& x, int& y, bool& past) {
  const unsigned full = 0xffffffffu;
  int base = 0;
  if (lane == 0) base = atomicAdd(pool.next, __popc(idle));
  base = __shfl_sync(full, base, 0);
  bool got = false, beyond = false;
  if (idle & (1u << lane)) {
    const int idx = base + __popc(idle & ((1u << lane) - 1u));
    const int block = (int)blockIdx.x + (idx >> 5) * (int)gridDim.x;
    if (block >= pool.blocks) {
      beyond = true;
    } else {
      const int by = block / pool.blocks_x, bx = block - by * pool.blocks_x;
      x = bx * 8 + (idx & 7);
      y = by * 4 + ((idx >> 3) & 3);
      got = x < pool.width && y < pool.height;
    }
  }
  past = __any_sync(full, beyond);
  return got;
}

// The pixels of one image shared by every CTA that works on it: its 8x4
// blocks 0, 1, 2, ... handed out one pixel at a time from a counter in
// global memory (the batched renderer's per-view pools).
struct ViewPool {
  int* next;  // global counter of pixels handed out for this image
  int width, height, blocks_x, blocks;
};

// ViewPool form of pool_take (same contract).
__device__ __forceinline__ bool pool_take(const ViewPool& pool, unsigned idle, int lane, int& x, int& y, bool& past) {
  const unsigned full = 0xffffffffu;
  int base = 0;
  if (lane == 0) base = atomicAdd(pool.next, __popc(idle));
  base = __shfl_sync(full, base, 0);
  bool got = false, beyond = false;
  if (idle & (1u << lane)) {
    const int idx = base + __popc(idle & ((1u << lane) - 1u));
    const int block = idx >> 5;
    if (block >= pool.blocks) {
      beyond = true;
    } else {
      const int by = block / pool.blocks_x, bx = block - by * pool.blocks_x;
      x = bx * 8 + (idx & 7);
      y = by * 4 + ((idx >> 3) & 3);
      got = x < pool.width && y < pool.height;
    }
  }
  past = __any_sync(full, beyond);
  return got;
}

// Drive one warp through a pixel pool: lanes whose rays are finished take
// the next pixels (Policy::start begins a ray, or finishes the pixel at
// once), so no lane waits for the slowest ray of a fixed tile.  Policy::done
// is called for a finished ray and either continues it (a new trace on r) or
// sets it idle.
template <class WB, class Policy, class Pool>
__device__ __forceinline__ void batch_run_pool(const TraceCtx& c, Ray& r, WB& b, Policy& policy, const Pool& pool) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int nq = 0;
  bool drained = false;
  r.phase = kPhIdle;
  for (;;) {
    if (!drained) {
      const unsigned idle = __ballot_sync(full, r.phase == kPhIdle);
      // Refill once Policy::kRefill lanes are idle (or all are): a policy
      // whose start is long (shading) runs it with more lanes together.
      if (idle && (__popc(idle) >= Policy::kRefill || idle == full)) {
        int x = 0, y = 0;
        bool past = false;
        const bool got = pool_take(pool, idle, lane, x, y, past);
        drained = past;
        if (got) policy.start(c, r, x, y);
      }
    }
    for (;;) {
      batch_advance(c, r, b, lane, nq);
      if (r.phase != kPhDone) break;
      policy.done(r);
    }
    const bool pending = nq > 0;
    if (!__any_sync(full, pending)) {
      // every lane is idle: take more pixels, or stop when none are left
      if (drained) break;
      continue;
    }
    batch_tests(c, r, b, lane, nq);
    batch_apply(c, r, b, lane, nq);
  }
}

}  // namespace arbor
