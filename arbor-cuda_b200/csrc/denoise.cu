// denoise.cu - the learned denoiser: a 4-level convolutional encoder-decoder
// (U-Net, channels 32/64/96/128, 3x3 kernels) over the 1-spp radiance and
// the albedo / normal / depth G-buffer, trained and run on the GPU by the
// kernels in this file.  No reference counterpart: the reference's only
// denoiser is filterLighting (Arbor.cu:292-302), which stays available.
//
// Arithmetic: activations and weights in BF16, tensor-core products
// accumulated in FP32 (tcgen05.mma with TMEM accumulators for the forward
// convolutions and the backward data pass, except the data pass of the two
// widest decoder inputs (160 and 224 channels) and the weight gradients,
// which use mma.sync m16n8k16), FP32 master
// weights, biases, gradients and Adam moments.  Activations are NHWC with channel counts that
// are multiples of 16.
//
// Kernels:
//   conv_tc_kernel  the forward 3x3 convolutions on tcgen05 (TMEM
//                   accumulators), used by inference and training
//   conv_kernel     3x3 convolution as an implicit GEMM: a CTA computes an
//                   8x8-pixel tile (partial at the image edge) for 16, 32 or
//                   64 output channels; input halo
//                   and weights are staged in shared memory 16 or 32 input
//                   channels at a time.  The same kernel runs the backward
//                   data pass on rotated, transposed weights, with the
//                   previous layer's activation derivative in its epilogue.
//   wgrad_kernel    weight gradients: a GEMM over pixels of the output
//                   gradient and the shifted input; each CTA writes its
//                   pixel range's partial sums, reduce_kernel adds the
//                   partials in a fixed order (deterministic gradients)
//   pool / upcat    2x2 average pooling and its backward pass; the backward
//                   pass of nearest upsampling + skip concatenation (the
//                   forward concatenation is read in place by the decoder
//                   convolutions), with activation derivatives
//   loss, adam, features, output: elementwise
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "abi_util.h"
#include "arbor_math.cuh"

namespace arbor {
namespace {

typedef __nv_bfloat16 bf16;
constexpr float kSlope = 0.1f;  // leaky ReLU
constexpr int kFeat = 16;       // input feature channels (13 used)
constexpr int kOutC = 16;       // output channels (3 used)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n" : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n" : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ------------------------------------------------------------ convolution --
struct ConvArgs {
  const bf16* x;      // input NHWC, cin channels
  const bf16* wt;     // weights [cout][9][cin]
  const float* bias;  // nullable
  void* y;            // output NHWC, cout channels (bf16, or fp32 when y_fp32)
  const bf16* mask;   // nullable: multiply by the leaky-ReLU derivative at mask (NHWC, cout channels)
  int cin, cout, n, h, w;
  int act;            // leaky ReLU on the output
  int y_fp32;
  // Optional second input: channels [cs, cin) are x2 (cin - cs channels) at
  // half resolution, upsampled by nearest neighbour, and x holds channels
  // [0, cs) - the decoder's concatenation, read without being stored.
  const bf16* x2;
  int cs;
};

// Address of input channels [c, c + 8) of pixel (img, gy, gx).
__device__ __forceinline__ const bf16* conv_in(const bf16* x, const bf16* x2, int cin, int cs, int h, int w, int img, int gy, int gx, int c) {
  if (x2 == nullptr) return x + ((size_t)(img * h + gy) * w + gx) * cin + c;
  if (c < cs) return x + ((size_t)(img * h + gy) * w + gx) * cs + c;
  return x2 + ((size_t)(img * (h >> 1) + (gy >> 1)) * (w >> 1) + (gx >> 1)) * (cin - cs) + (c - cs);
}

// smem layout of one stage: halo [100][KC+8], weights [NT*8*9][KC+8] (bf16)
template <int KC, int NT>
constexpr int conv_smem_bytes() {
  return (100 + NT * 8 * 9) * (KC + 8) * 2;
}

template <int KC, int NT>
__global__ void __launch_bounds__(128) conv_kernel(ConvArgs a) {
  extern __shared__ uint4 conv_smem[];
  constexpr int RS = KC + 8;  // row stride (elements): 16-byte aligned rows, staggered banks
  bf16* halo = reinterpret_cast<bf16*>(conv_smem);
  bf16* wts = halo + 100 * RS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_x = (a.w + 7) >> 3;
  const int ty = blockIdx.x / tiles_x, tx = blockIdx.x - ty * tiles_x;
  const int co0 = blockIdx.y * NT * 8;
  const int img = blockIdx.z;
  float acc[NT][4];
#pragma unroll
  for (int i = 0; i < NT; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0f;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (int c0 = 0; c0 < a.cin; c0 += KC) {
    // input halo: 10x10 pixels x KC channels, zero outside the image
    for (int v = tid; v < 100 * (KC / 8); v += 128) {
      const int pix = v / (KC / 8), part = v - pix * (KC / 8);
      const int hy = pix / 10, hx = pix - hy * 10;
      const int gy = ty * 8 + hy - 1, gx = tx * 8 + hx - 1;
      uint4 val = zero;
      if (gy >= 0 && gy < a.h && gx >= 0 && gx < a.w)
        val = *reinterpret_cast<const uint4*>(conv_in(a.x, a.x2, a.cin, a.cs, a.h, a.w, img, gy, gx, c0 + part * 8));
      *reinterpret_cast<uint4*>(halo + pix * RS + part * 8) = val;
    }
    // weights: NT*8 output channels x 9 taps x KC input channels
    for (int v = tid; v < NT * 8 * 9 * (KC / 8); v += 128) {
      const int row = v / (KC / 8), part = v - row * (KC / 8);
      const int co = co0 + row / 9, tap = row - (row / 9) * 9;
      uint4 val = zero;
      if (co < a.cout) val = *reinterpret_cast<const uint4*>(a.wt + ((size_t)co * 9 + tap) * a.cin + c0 + part * 8);
      *reinterpret_cast<uint4*>(wts + row * RS + part * 8) = val;
    }
    __syncthreads();
#pragma unroll 1
    for (int tap = 0; tap < 9; tap++) {
      const int dy = tap / 3, dx = tap - dy * 3;
#pragma unroll
      for (int kk = 0; kk < KC / 16; kk++) {
        uint32_t a0, a1, a2, a3;
        {
          const int r = lane & 15, koff = (lane >> 4) * 8;
          const int hp = (2 * warp + (r >> 3) + dy) * 10 + (r & 7) + dx;
          ldsm_x4(smem_u32(halo + hp * RS + kk * 16 + koff), a0, a1, a2, a3);
        }
#pragma unroll
        for (int nt = 0; nt < NT; nt += 2) {
          const int mi = lane >> 3;
          const int col = (nt + (mi >> 1)) * 8 + (lane & 7);
          uint32_t b0, b1, b2, b3;
          ldsm_x4(smem_u32(wts + (col * 9 + tap) * RS + kk * 16 + (mi & 1) * 8), b0, b1, b2, b3);
          mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
          mma_bf16(acc[nt + 1], a0, a1, a2, a3, b2, b3);
        }
      }
    }
    __syncthreads();
  }
  // epilogue: bias, activation or activation derivative, store
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; nt++) {
    const int co = co0 + nt * 8 + 2 * t;
    if (co >= a.cout) continue;
    const float b0 = a.bias ? a.bias[co] : 0.0f, b1 = a.bias ? a.bias[co + 1] : 0.0f;
#pragma unroll
    for (int hh = 0; hh < 2; hh++) {
      const int r = g + 8 * hh;
      const int gy = ty * 8 + 2 * warp + (r >> 3), gx = tx * 8 + (r & 7);
      if (gy >= a.h || gx >= a.w) continue;  // partial tile at the image edge
      const size_t p = (size_t)(img * a.h + gy) * a.w + gx;
      float v0 = acc[nt][2 * hh] + b0, v1 = acc[nt][2 * hh + 1] + b1;
      if (a.act) {
        v0 = v0 > 0.0f ? v0 : v0 * kSlope;
        v1 = v1 > 0.0f ? v1 : v1 * kSlope;
      }
      if (a.mask) {
        const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(a.mask + p * a.cout + co);
        if (!(__bfloat162float(m.x) > 0.0f)) v0 *= kSlope;
        if (!(__bfloat162float(m.y) > 0.0f)) v1 *= kSlope;
      }
      if (a.y_fp32)
        *reinterpret_cast<float2*>(reinterpret_cast<float*>(a.y) + p * a.cout + co) = make_float2(v0, v1);
      else
        *reinterpret_cast<__nv_bfloat162*>(reinterpret_cast<bf16*>(a.y) + p * a.cout + co) = __floats2bfloat162_rn(v0, v1);
    }
  }
}

// ------------------------------------------- tcgen05 convolution (sm_100a) --
// The same 3x3 convolution on the 5th-generation tensor cores: a CTA of 4
// warps computes R consecutive output rows of a 128-pixel column segment for
// all N output channels.  Per chunk of CC input channels it stages the R + 2
// input rows (130 pixels with the halo) and the chunk's weights in shared
// memory with cp.async (two stage buffers: chunk c + 1 loads while chunk c's
// MMAs run), in the K-major, non-swizzled core-matrix layout the
// MMA reads (8 rows of 16 bytes per core matrix): the A operand of output row
// r and tap (dy, dx) is staged row r + dy shifted by dx, so one 128-row
// descriptor per (row, tap) needs no copy.  One thread issues tcgen05.mma
// (M = 128, N, K = 16, BF16 inputs, FP32 accumulators in TMEM, one N-column
// block per output row) for R rows x 9 taps x CC/16 steps and commits to an
// mbarrier; every thread waits (bounded) for a chunk's MMAs before its stage
// buffer is refilled.  The epilogue reads the accumulators with tcgen05.ld (warp w owns
// TMEM lanes 32w..32w+31 = pixels 32w..32w+31 of the segment), applies bias
// and activation and stores BF16 or FP32.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  // start address, leading / stride byte offsets (16-byte units), version 1,
  // no swizzle (layout type 0)
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
         (1ull << 46);
}
template <int N>
constexpr uint32_t umma_idesc() {
  // FP32 accumulator, BF16 A and B, both K-major, N >> 3, M = 128 >> 4
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
constexpr int pow2_cols(int c) { return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512; }
template <int N, int CC, int R>
constexpr int conv_tc_stage_bytes() {
  return (CC / 8) * (R + 2) * 130 * 16 + 9 * (CC / 8) * N * 16;
}
template <int N, int CC, int R>
constexpr int conv_tc_smem_bytes() {
  return 2 * conv_tc_stage_bytes<N, CC, R>() + N * 4 + 16;  // two stages, biases, mbarrier, TMEM slot
}

// Bounded wait on an mbarrier phase; false when it did not complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (int i = 0; i < (1 << 20); i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
  // a 16-byte copy, or 16 zero bytes when !valid (src-size 0)
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

template <int N, int CC, int R>
__global__ void __launch_bounds__(128) conv_tc_kernel(ConvArgs a, int* err) {
  extern __shared__ __align__(128) uint8_t tc_smem[];
  constexpr int KU = CC / 8;                    // 16-byte K units per chunk
  constexpr int ROWS = R + 2;                   // staged input rows
  constexpr int HALO_B = KU * ROWS * 130 * 16;
  constexpr int STAGE_B = conv_tc_stage_bytes<N, CC, R>();
  constexpr uint32_t LBO_A = ROWS * 130 * 16;   // next K unit of the staged rows
  constexpr uint32_t LBO_B = N * 16;            // next K unit of the weights
  constexpr int COLS = pow2_cols(R * N);
  float* bias_s = reinterpret_cast<float*>(tc_smem + 2 * STAGE_B);
  uint64_t* bar = reinterpret_cast<uint64_t*>(bias_s + N);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_x = (a.w + 127) >> 7, rows_y = (a.h + R - 1) / R;
  int t = blockIdx.x;
  const int tx = t % tiles_x;
  t /= tiles_x;
  const int y0 = (t % rows_y) * R, img = t / rows_y;
  const int x0 = tx * 128;
  const uint32_t bar_a = smem_u32(bar);
  const uint32_t smem_a = smem_u32(tc_smem);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)), "r"(COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_a), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  for (int i = tid; i < N; i += 128) bias_s[i] = a.bias && i < a.cout ? a.bias[i] : 0.0f;
  // Stage the operands of the chunk starting at channel c0 into stage buffer sb.
  auto stage = [&](int c0, int sb) {
    const uint32_t halo_a = smem_a + sb * STAGE_B, wts_a = halo_a + HALO_B;
    for (int v = tid; v < ROWS * 130 * KU; v += 128) {
      const int k = v % KU, rh = v / KU;
      const int r = rh / 130, hx = rh - r * 130;
      const int gy = y0 + r - 1, gx = x0 + hx - 1;
      const bool in = gy >= 0 && gy < a.h && gx >= 0 && gx < a.w;
      const bf16* src = in ? conv_in(a.x, a.x2, a.cin, a.cs, a.h, a.w, img, gy, gx, c0 + k * 8) : a.x;
      cp_async16(halo_a + ((k * ROWS + r) * 130 + hx) * 16, src, in);
    }
    for (int v = tid; v < 9 * KU * N; v += 128) {
      const int k = v % KU, q = v / KU;
      const int tap = q % 9, n = q / 9;
      const bool in = n < a.cout;
      const bf16* src = in ? a.wt + ((size_t)n * 9 + tap) * a.cin + c0 + k * 8 : a.wt;
      cp_async16(wts_a + ((tap * KU + k) * N + n) * 16, src, in);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;
  const int chunks = a.cin / CC;
  bool ok = true;
  stage(0, 0);
  for (int c = 0; c < chunks && ok; c++) {
    // The chunk c-1 MMAs must be done before their buffer takes chunk c+1.
    if (c > 0) ok = __syncthreads_and(mbar_wait(bar_a, (uint32_t)((c - 1) & 1)) ? 1 : 0) != 0;
    if (!ok) break;
    if (c + 1 < chunks) {
      stage((c + 1) * CC, (c + 1) & 1);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // chunk c's copies are in
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    // make the staged operands visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t idesc = umma_idesc<N>();
      const uint32_t halo_a = smem_a + (c & 1) * STAGE_B, wts_a = halo_a + HALO_B;
      // descriptors advance by address only (16-byte units in the low bits)
      const uint64_t da0 = umma_desc(halo_a, LBO_A, 128), db0 = umma_desc(wts_a, LBO_B, 128);
      uint32_t acc = c > 0 ? 1u : 0u;
#pragma unroll
      for (int r = 0; r < R; r++) {
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
#pragma unroll
          for (int st = 0; st < CC / 16; st++) {
            const uint64_t da = da0 + (uint64_t)((((2 * st * ROWS + r + tap / 3) * 130 + tap % 3) * 16) >> 4);
            const uint64_t db = db0 + (uint64_t)(((tap * KU + 2 * st) * N * 16) >> 4);
            const uint32_t acc_rt = (tap > 0 || st > 0) ? 1u : acc;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + (uint32_t)(r * N)),
                "l"(da), "l"(db), "r"(idesc), "r"(acc_rt));
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar_a) : "memory");
    }
  }
  // the last chunk's MMAs (bounded, uniform outcome)
  if (ok) ok = __syncthreads_and(mbar_wait(bar_a, (uint32_t)((chunks - 1) & 1)) ? 1 : 0) != 0;
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const int gx = x0 + warp * 32 + lane;  // this thread's TMEM lane = pixel of the segment
#pragma unroll 1
    for (int r = 0; r < R; r++) {
      const int gy = y0 + r;
      const size_t p = (size_t)(img * a.h + gy) * a.w + gx;
#pragma unroll 1
      for (int col = 0; col < N; col += 16) {
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]),
              "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(r * N + col)));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (gx < a.w && gy < a.h) {
          float f[16];
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const int co = col + j;
            float x = __uint_as_float(v[j]) + bias_s[co];
            if (a.act) x = x > 0.0f ? x : x * kSlope;
            if (a.mask && !(__bfloat162float(a.mask[p * a.cout + co]) > 0.0f)) x *= kSlope;
            f[j] = x;
          }
          if (a.y_fp32) {
            float4* o = reinterpret_cast<float4*>(reinterpret_cast<float*>(a.y) + p * a.cout + col);
#pragma unroll
            for (int j = 0; j < 4; j++) o[j] = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
          } else {
            uint4* o = reinterpret_cast<uint4*>(reinterpret_cast<bf16*>(a.y) + p * a.cout + col);
            uint32_t w[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
              const __nv_bfloat162 b2 = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
              w[j] = *reinterpret_cast<const uint32_t*>(&b2);
            }
            o[0] = make_uint4(w[0], w[1], w[2], w[3]);
            o[1] = make_uint4(w[4], w[5], w[6], w[7]);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(COLS));
}

// Row-streaming form for the layers whose weights fit in shared memory
// with a 5-row input ring: a CTA keeps all 9 x CIN x N weights resident and
// walks down its rows of one 128-pixel column segment.  Per output row y it
// starts loading input row y + 2 (all CIN channels, cp.async) into the ring,
// waits for row y + 1, one thread issues the row's 9 x CIN/16 MMAs into one
// of two TMEM accumulators, and the 4 warps run the previous row's epilogue
// while those MMAs execute; each input row is read from memory once per
// segment.
template <int N, int CIN>
constexpr int conv_row_smem_bytes() {
  return 9 * (CIN / 8) * N * 16 + 5 * (CIN / 8) * 130 * 16 + N * 4 + 32;
}

template <int N, int CIN>
__global__ void __launch_bounds__(128) conv_row_kernel(ConvArgs a, int rows_per_cta, int* err) {
  extern __shared__ __align__(128) uint8_t rs_smem[];
  constexpr int KU = CIN / 8;
  constexpr int W_B = 9 * KU * N * 16;
  constexpr int SLOT_B = KU * 130 * 16;        // one staged input row
  constexpr uint32_t LBO_A = 130 * 16;         // next K unit within a staged row
  constexpr uint32_t LBO_B = N * 16;           // next K unit of the weights
  constexpr int COLS = pow2_cols(2 * N);
  const uint32_t smem_a = smem_u32(rs_smem);
  const uint32_t wts_a = smem_a, ring_a = smem_a + W_B;
  float* bias_s = reinterpret_cast<float*>(rs_smem + W_B + 5 * SLOT_B);
  uint64_t* bar = reinterpret_cast<uint64_t*>(bias_s + N);  // two mbarriers, one per accumulator
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_x = (a.w + 127) >> 7, groups = (a.h + rows_per_cta - 1) / rows_per_cta;
  int t = blockIdx.x;
  const int tx = t % tiles_x;
  t /= tiles_x;
  const int y_begin = (t % groups) * rows_per_cta, img = t / groups;
  const int y_end = y_begin + rows_per_cta < a.h ? y_begin + rows_per_cta : a.h;
  const int x0 = tx * 128;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)), "r"(COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar + 1)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  for (int i = tid; i < N; i += 128) bias_s[i] = a.bias && i < a.cout ? a.bias[i] : 0.0f;
  // weights: unit (tap, k, n)
  for (int v = tid; v < 9 * KU * N; v += 128) {
    const int k = v % KU, q = v / KU;
    const int tap = q % 9, n = q / 9;
    const bool in = n < a.cout;
    cp_async16(wts_a + ((tap * KU + k) * N + n) * 16, in ? a.wt + ((size_t)n * 9 + tap) * a.cin + k * 8 : a.wt, in);
  }
  // input row gy into its ring slot (gy + 5) % 5: unit (k, hx)
  auto load_row = [&](int gy) {
    const uint32_t slot = ring_a + ((gy + 5) % 5) * SLOT_B;
    for (int v = tid; v < 130 * KU; v += 128) {
      const int k = v % KU, hx = v / KU;
      const int gx = x0 + hx - 1;
      const bool in = gy >= 0 && gy < a.h && gx >= 0 && gx < a.w;
      const bf16* src = in ? conv_in(a.x, a.x2, a.cin, a.cs, a.h, a.w, img, gy, gx, k * 8) : a.x;
      cp_async16(slot + (k * 130 + hx) * 16, src, in);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  load_row(y_begin - 1);
  load_row(y_begin);
  load_row(y_begin + 1);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc<N>();
  bool ok = true;
  // epilogue of output row y from accumulator (y - y_begin) & 1
  auto epilogue = [&](int y) {
    const int b = (y - y_begin) & 1;
    const bool done = mbar_wait(smem_u32(bar + b), (uint32_t)(((y - y_begin) >> 1) & 1));
    ok = __syncthreads_and(done ? 1 : 0) != 0;
    if (!ok) return;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const int gx = x0 + warp * 32 + lane;
    const size_t p = (size_t)(img * a.h + y) * a.w + gx;
#pragma unroll 1
    for (int col = 0; col < N; col += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]),
            "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * N + col)));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (gx < a.w) {
        float f[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
          float x = __uint_as_float(v[j]) + bias_s[col + j];
          if (a.act) x = x > 0.0f ? x : x * kSlope;
          if (a.mask && !(__bfloat162float(a.mask[p * a.cout + col + j]) > 0.0f)) x *= kSlope;
          f[j] = x;
        }
        if (a.y_fp32) {
          float4* o = reinterpret_cast<float4*>(reinterpret_cast<float*>(a.y) + p * a.cout + col);
#pragma unroll
          for (int j = 0; j < 4; j++) o[j] = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
        } else {
          uint4* o = reinterpret_cast<uint4*>(reinterpret_cast<bf16*>(a.y) + p * a.cout + col);
          uint32_t w[8];
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const __nv_bfloat162 b2 = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
            w[j] = *reinterpret_cast<const uint32_t*>(&b2);
          }
          o[0] = make_uint4(w[0], w[1], w[2], w[3]);
          o[1] = make_uint4(w[4], w[5], w[6], w[7]);
        }
      }
    }
    // the accumulator is read out before its next MMAs are issued
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  };
  for (int y = y_begin; y < y_end && ok; y++) {
    // Row y + 2's slot held row y - 3, last read by output row y - 2, whose
    // MMAs completed before its epilogue (the previous iteration).
    load_row(y + 2);
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // rows up to y + 1 are in
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t acc_t = tmem + (uint32_t)(((y - y_begin) & 1) * N);
      const uint64_t db0 = umma_desc(wts_a, LBO_B, 128);
#pragma unroll
      for (int tap = 0; tap < 9; tap++) {
        const int dy = tap / 3, dx = tap - dy * 3;
        const uint64_t da0 = umma_desc(ring_a + ((y - 1 + dy + 5) % 5) * SLOT_B, LBO_A, 128);
#pragma unroll
        for (int st = 0; st < CIN / 16; st++) {
          const uint64_t da = da0 + (uint64_t)(((2 * st * 130 + dx) * 16) >> 4);
          const uint64_t db = db0 + (uint64_t)(((tap * KU + 2 * st) * N * 16) >> 4);
          const uint32_t acc = (tap > 0 || st > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(acc_t),
              "l"(da), "l"(db), "r"(idesc), "r"(acc));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar + ((y - y_begin) & 1)))
                   : "memory");
    }
    if (y > y_begin) epilogue(y - 1);
  }
  if (ok && y_end > y_begin) epilogue(y_end - 1);
  if (!ok && tid == 0) atomicExch(err, 1);
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(COLS));
}

// ------------------------------------------------------- weight gradient --
// dW[co][tap][ci] += sum over pixels p of dY[p][co] * X[p + tap offset][ci].
// CTA: 64 output channels (4 warps x 16) x CI (16 or 32) input channels of
// one tap, over a contiguous range of pixels, 32 at a time.
struct WgradArgs {
  const bf16* dy;  // NHWC, cout channels
  const bf16* x;   // NHWC, cin channels (or cs channels with x2, as ConvArgs)
  float* dw;       // partial sums: [gridDim.x][cout][9][cin], one slice per pixel range
  int cin, cout, n, h, w;
  int pixels_per_cta;
  const bf16* x2;
  int cs;
};

template <int CI>
__global__ void __launch_bounds__(128) wgrad_kernel(WgradArgs a) {
  constexpr int KP = 32;   // pixels per stage
  constexpr int NT = CI / 8;
  constexpr int DS = 64 + 8, XS = CI + 8;
  __shared__ __align__(16) bf16 dys[KP * DS];
  __shared__ __align__(16) bf16 xs[KP * XS];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int co0 = blockIdx.y * 64;
  const int chunks = a.cin / CI;
  const int tap = blockIdx.z / chunks, ci0 = (blockIdx.z - tap * chunks) * CI;
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;
  const long total = (long)a.n * a.h * a.w;
  const long p_begin = (long)blockIdx.x * a.pixels_per_cta;
  const long p_end = p_begin + a.pixels_per_cta < total ? p_begin + a.pixels_per_cta : total;
  float acc[NT][4];
#pragma unroll
  for (int i = 0; i < NT; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0f;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (long pb = p_begin; pb < p_end; pb += KP) {
    // dY rows: KP pixels x 64 channels
    for (int v = tid; v < KP * 8; v += 128) {
      const int r = v >> 3, part = v & 7;
      const long p = pb + r;
      const int co = co0 + part * 8;
      uint4 val = zero;
      if (p < p_end && co < a.cout) val = *reinterpret_cast<const uint4*>(a.dy + p * a.cout + co);
      *reinterpret_cast<uint4*>(dys + r * DS + part * 8) = val;
    }
    // shifted X rows: KP pixels x CI channels
    for (int v = tid; v < KP * (CI / 8); v += 128) {
      const int r = v / (CI / 8), part = v - r * (CI / 8);
      const long p = pb + r;
      uint4 val = zero;
      if (p < p_end) {
        const int img = (int)(p / ((long)a.h * a.w));
        const int rem = (int)(p - (long)img * a.h * a.w);
        const int y = rem / a.w + dy, xx = rem % a.w + dx;
        if (y >= 0 && y < a.h && xx >= 0 && xx < a.w)
          val = *reinterpret_cast<const uint4*>(conv_in(a.x, a.x2, a.cin, a.cs, a.h, a.w, img, y, xx, ci0 + part * 8));
      }
      *reinterpret_cast<uint4*>(xs + r * XS + part * 8) = val;
    }
    __syncthreads();
#pragma unroll
    for (int kb = 0; kb < KP; kb += 16) {
      const int mi = lane >> 3, row = lane & 7;
      uint32_t a0, a1, a2, a3;
      // A[m = co][k = pixel] from dY rows (pixel-major): transposed loads
      ldsm_x4_t(smem_u32(dys + (kb + (mi >> 1) * 8 + row) * DS + warp * 16 + (mi & 1) * 8), a0, a1, a2, a3);
#pragma unroll
      for (int nt = 0; nt < NT; nt += 2) {
        uint32_t b0, b1, b2, b3;
        ldsm_x4_t(smem_u32(xs + (kb + (mi & 1) * 8 + row) * XS + (nt + (mi >> 1)) * 8), b0, b1, b2, b3);
        mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
        mma_bf16(acc[nt + 1], a0, a1, a2, a3, b2, b3);
      }
    }
    __syncthreads();
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; nt++) {
#pragma unroll
    for (int hh = 0; hh < 2; hh++) {
      const int co = co0 + warp * 16 + g + 8 * hh;
      if (co >= a.cout) continue;
      const int ci = ci0 + nt * 8 + 2 * t;
      float* d = a.dw + (size_t)blockIdx.x * a.cout * 9 * a.cin + ((size_t)co * 9 + tap) * a.cin + ci;
      d[0] = acc[nt][2 * hh];
      d[1] = acc[nt][2 * hh + 1];
    }
  }
}

// Partial bias gradients: db[blockIdx.x][co] = sum over this block's pixels of dY[p][co]
__global__ void bgrad_kernel(const bf16* __restrict__ dy, float* __restrict__ db, int cout, long pixels) {
  __shared__ float part[256];
  const int tid = threadIdx.x;
  const int lanes = 256 / cout * cout;  // threads that own a channel
  float s = 0.0f;
  if (tid < lanes) {
    const int co = tid % cout;
    for (long p = (long)blockIdx.x * (256 / cout) + tid / cout; p < pixels; p += (long)gridDim.x * (256 / cout))
      s += __bfloat162float(dy[p * cout + co]);
  }
  part[tid] = s;
  __syncthreads();
  if (tid < cout) {
    float t = 0.0f;
    for (int k = tid; k < lanes; k += cout) t += part[k];
    db[(size_t)blockIdx.x * cout + tid] = t;
  }
}

// g[i] += sum over s = 0 .. splits - 1, in that order, of part[s * n + i]:
// the partial sums of wgrad_kernel / bgrad_kernel folded in a fixed order.
__global__ void reduce_kernel(const float* __restrict__ part, float* __restrict__ g, long n, int splits) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int k = 0; k < splits; k++) s += part[(size_t)k * n + i];
    g[i] += s;
  }
}

// --------------------------------------------------- pooling and concat --
// All four move 8 channels (16 bytes) per thread; channel counts are
// multiples of 16.
__device__ __forceinline__ void unpack8(uint4 v, float (&f)[8]) {
  const __nv_bfloat162* b = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const float2 t = __bfloat1622float2(b[j]);
    f[2 * j] = t.x;
    f[2 * j + 1] = t.y;
  }
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint4 v;
  __nv_bfloat162* b = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
  for (int j = 0; j < 4; j++) b[j] = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
  return v;
}

__global__ void pool_kernel(const bf16* __restrict__ x, bf16* __restrict__ y, int n, int h, int w, int c) {
  const int c8 = c / 8;
  const long total = (long)n * (h / 2) * (w / 2) * c8;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c8);
    long q = i / c8;
    const int X = (int)(q % (w / 2));
    q /= (w / 2);
    const int Y = (int)(q % (h / 2));
    const int img = (int)(q / (h / 2));
    const uint4* b = reinterpret_cast<const uint4*>(x + ((size_t)(img * h + 2 * Y) * w + 2 * X) * c) + ch;
    float s[8], t[8];
    unpack8(b[0], s);
    unpack8(b[c8], t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] += t[j];
    unpack8(b[(size_t)w * c8], t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] += t[j];
    unpack8(b[(size_t)w * c8 + c8], t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] = 0.25f * (s[j] + t[j]);
    reinterpret_cast<uint4*>(y)[i] = pack8(s);
  }
}

// d(skip)[p] = (0.25 * d(pooled)[parent] + dcat[p]) * act'(skip[p])
__global__ void pool_back_kernel(const bf16* __restrict__ dpool, const bf16* __restrict__ dcat, const bf16* __restrict__ skip,
                                 bf16* __restrict__ dx, int n, int h, int w, int c) {
  const int c8 = c / 8;
  const long total = (long)n * h * w * c8;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c8);
    long q = i / c8;
    const int x = (int)(q % w);
    q /= w;
    const int y = (int)(q % h);
    const int img = (int)(q / h);
    float g[8], d[8], m[8];
    unpack8(reinterpret_cast<const uint4*>(dpool + ((size_t)(img * (h / 2) + y / 2) * (w / 2) + x / 2) * c)[ch], g);
    unpack8(reinterpret_cast<const uint4*>(dcat)[i], d);
    unpack8(reinterpret_cast<const uint4*>(skip)[i], m);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      g[j] = 0.25f * g[j] + d[j];
      if (!(m[j] > 0.0f)) g[j] *= kSlope;
    }
    reinterpret_cast<uint4*>(dx)[i] = pack8(g);
  }
}

// dcat -> d(skip part) unmasked (dskip), d(low)[q] = sum of its 4 children's gradients * act'(low[q])
__global__ void upcat_back_kernel(const bf16* __restrict__ dcat, const bf16* __restrict__ low, bf16* __restrict__ dskip,
                                  bf16* __restrict__ dlow, int n, int h, int w, int cs, int cl) {
  const int c8 = (cs + cl) / 8, s8 = cs / 8, l8 = cl / 8;
  const long skip_total = (long)n * h * w * s8;
  const long low_total = (long)n * (h / 2) * (w / 2) * l8;
  const uint4* dc = reinterpret_cast<const uint4*>(dcat);
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < skip_total + low_total; i += (long)gridDim.x * blockDim.x) {
    if (i < skip_total) {
      const long p = i / s8;
      reinterpret_cast<uint4*>(dskip)[i] = dc[p * c8 + (i - p * s8)];
    } else {
      const long j = i - skip_total;
      const int ch = (int)(j % l8);
      long q = j / l8;
      const int X = (int)(q % (w / 2));
      q /= (w / 2);
      const int Y = (int)(q % (h / 2));
      const int img = (int)(q / (h / 2));
      const size_t b = ((size_t)(img * h + 2 * Y) * w + 2 * X) * c8 + s8 + ch;
      float g[8], t[8], m[8];
      unpack8(dc[b], g);
      unpack8(dc[b + c8], t);
#pragma unroll
      for (int k = 0; k < 8; k++) g[k] += t[k];
      unpack8(dc[b + (size_t)w * c8], t);
#pragma unroll
      for (int k = 0; k < 8; k++) g[k] += t[k];
      unpack8(dc[b + (size_t)w * c8 + c8], t);
      unpack8(reinterpret_cast<const uint4*>(low)[j], m);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        g[k] += t[k];
        if (!(m[k] > 0.0f)) g[k] *= kSlope;
      }
      reinterpret_cast<uint4*>(dlow)[j] = pack8(g);
    }
  }
}

// ----------------------------------------------------------- elementwise --
// Features of one pixel: log(1 + radiance), albedo, normal,
// log(1 + depth) / 4, log(1 + filterLighting's radiance).
__global__ void features_kernel(const float4* __restrict__ lin, const float4* __restrict__ gui, const float4* __restrict__ nrm,
                                const float4* __restrict__ hit, const float4* __restrict__ fil, bf16* __restrict__ f, long pixels) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (long)gridDim.x * blockDim.x) {
    const float4 l = lin[p], g = gui[p], n = nrm[p], h = hit[p], q = fil[p];
    const float depth = fminf(fmaxf(h.x, 0.0f), 1.0e4f);
    float v[kFeat] = {log1pf(fmaxf(l.x, 0.0f)), log1pf(fmaxf(l.y, 0.0f)), log1pf(fmaxf(l.z, 0.0f)), g.x, g.y, g.z, n.x, n.y, n.z,
                      log1pf(depth) * 0.25f, log1pf(fmaxf(q.x, 0.0f)), log1pf(fmaxf(q.y, 0.0f)), log1pf(fmaxf(q.z, 0.0f)),
                      0.0f, 0.0f, 0.0f};
    __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(f + p * kFeat);
#pragma unroll
    for (int k = 0; k < kFeat / 2; k++) o[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
  }
}

// Loss in log(1 + radiance), prediction = log(1 + base) + out[0:3]: mean
// absolute difference (l2 = false) or mean squared difference (l2 = true).
__global__ void loss_kernel(const float* __restrict__ out, const float4* __restrict__ noisy, const float4* __restrict__ target,
                            bf16* __restrict__ dout, float* __restrict__ loss, long pixels, float scale, bool l2) {
  __shared__ float part[256];
  float s = 0.0f;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (long)gridDim.x * blockDim.x) {
    const float4 nz = noisy[p], tg = target[p];
    const float nv[3] = {nz.x, nz.y, nz.z}, tv[3] = {tg.x, tg.y, tg.z};
    __nv_bfloat162* d = reinterpret_cast<__nv_bfloat162*>(dout + p * kOutC);
    float g[kOutC] = {};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float diff = log1pf(fmaxf(nv[c], 0.0f)) + out[p * kOutC + c] - log1pf(fmaxf(tv[c], 0.0f));
      if (l2) {
        s += diff * diff;
        g[c] = 2.0f * scale * diff;
      } else {
        s += fabsf(diff);
        g[c] = diff > 0.0f ? scale : (diff < 0.0f ? -scale : 0.0f);
      }
    }
#pragma unroll
    for (int k = 0; k < kOutC / 2; k++) d[k] = __floats2bfloat162_rn(g[2 * k], g[2 * k + 1]);
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, part[0]);
}

__global__ void output_kernel(const float* __restrict__ out, const float4* __restrict__ noisy, float4* __restrict__ den, long pixels) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (long)gridDim.x * blockDim.x) {
    const float4 nz = noisy[p];
    const float* o = out + p * kOutC;
    den[p] = make_float4(expm1f(log1pf(fmaxf(nz.x, 0.0f)) + o[0]), expm1f(log1pf(fmaxf(nz.y, 0.0f)) + o[1]),
                         expm1f(log1pf(fmaxf(nz.z, 0.0f)) + o[2]), 1.0f);
  }
}

__global__ void accumulate_kernel(float* __restrict__ sum, const float* __restrict__ x, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) sum[i] += x[i];
}
__global__ void scale_kernel(float* __restrict__ x, long n, float s) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] *= s;
}

// ------------------------------------------------------------- parameters --
// One layer's parameters inside the flat FP32 arrays: weights [cout][9][cin]
// at woff, biases at boff.
struct LayerParams {
  int cin, cout;
  long woff, boff;
};

// Hash-based normal deviates (Box-Muller over two hashed uniforms).
__device__ __forceinline__ float hash_uniform(uint32_t i, uint32_t seed) {
  uint32_t h = hashU(i * 2654435761u ^ hashU(seed));
  return ((float)(h >> 8) + 0.5f) * (1.0f / 16777216.0f);
}
__global__ void init_kernel(float* __restrict__ w, long count, float stdev, uint32_t seed) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
    const float u1 = hash_uniform((uint32_t)(2 * i), seed), u2 = hash_uniform((uint32_t)(2 * i + 1), seed);
    w[i] = stdev * sqrtf(-2.0f * logf(u1)) * cosf(6.2831853f * u2);
  }
}

// Adam on the flat parameters; writes the BF16 forward weights and the
// rotated, transposed BF16 weights of the backward data pass.
struct AdamArgs {
  float* p;
  float* g;
  float* m;
  float* v;
  long count;
  float lr, b1, b2, eps, c1, c2;  // c1 = 1 - b1^t, c2 = 1 - b2^t
};
__global__ void adam_kernel(AdamArgs a) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.count; i += (long)gridDim.x * blockDim.x) {
    const float g = a.g[i];
    const float m = a.b1 * a.m[i] + (1.0f - a.b1) * g;
    const float v = a.b2 * a.v[i] + (1.0f - a.b2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    a.p[i] -= a.lr * (m / a.c1) / (sqrtf(v / a.c2) + a.eps);
    a.g[i] = 0.0f;
  }
}
// wf[co][tap][ci] = p[woff + ...]; wb[ci][8 - tap][co] = the same value
__global__ void cast_kernel(const float* __restrict__ p, bf16* __restrict__ wf, bf16* __restrict__ wb, int cin, int cout) {
  const long total = (long)cout * 9 * cin;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ci = (int)(i % cin);
    const long q = i / cin;
    const int tap = (int)(q % 9);
    const int co = (int)(q / 9);
    const bf16 v = __float2bfloat16(p[i]);
    wf[i] = v;
    wb[((size_t)ci * 9 + (8 - tap)) * cout + co] = v;
  }
}

int cuda_fail(const char* what, cudaError_t e) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  return ARBOR_ERR_CUDA;
}
#define DN_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(#call, e_); \
  } while (0)

dim3 ew_grid(long n) {
  long b = (n + 255) / 256;
  return dim3((unsigned)(b < 8192 ? (b > 0 ? b : 1) : 8192));
}

}  // namespace
}  // namespace arbor

using namespace arbor;

// The network: 15 convolutions.
namespace {
constexpr int kLayers = 15;
// (cin, cout, leaky ReLU) of each convolution, in forward order
constexpr int kSpec[kLayers][3] = {
    {kFeat, 32, 1}, {32, 32, 1},      // encoder level 0
    {32, 64, 1},    {64, 64, 1},      // level 1
    {64, 96, 1},    {96, 96, 1},      // level 2
    {96, 128, 1},   {128, 128, 1},    // level 3
    {224, 96, 1},   {96, 96, 1},      // decoder level 2 (96 skip + 128 up)
    {160, 64, 1},   {64, 64, 1},      // level 1 (64 + 96)
    {96, 32, 1},    {32, 32, 1},      // level 0 (32 + 64)
    {32, kOutC, 0},                   // output (3 of 16 channels used)
};
// activation tensors
enum Act {
  aF, aE0a, aE0, aP1, aE1a, aE1, aP2, aE2a, aE2, aP3, aB3a, aB3, aC2, aD2a, aD2, aC1, aD1a, aD1, aC0, aD0a, aD0, kActs
};
struct ActSpec {
  int level, channels;
};
constexpr ActSpec kAct[kActs] = {{0, kFeat}, {0, 32}, {0, 32}, {1, 32}, {1, 64},  {1, 64}, {2, 64}, {2, 96}, {2, 96}, {3, 96}, {3, 128},
                                 {3, 128},   {2, 224}, {2, 96}, {2, 96}, {1, 160}, {1, 64}, {1, 64}, {0, 96}, {0, 32}, {0, 32}};
// input and output tensor of each convolution (the output layer writes `out`)
constexpr int kIn[kLayers] = {aF, aE0a, aP1, aE1a, aP2, aE2a, aP3, aB3a, aC2, aD2a, aC1, aD1a, aC0, aD0a, aD0};
constexpr int kOut[kLayers] = {aE0a, aE0, aE1a, aE1, aE2a, aE2, aB3a, aB3, aD2a, aD2, aD1a, aD1, aD0a, aD0, -1};
// decoder inputs read as (skip, level below) without storing the concatenation
constexpr int kCat[kLayers][2] = {{-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}, {aE2, aB3}, {-1, -1},
                                  {aE1, aD2}, {-1, -1}, {aE0, aD1}, {-1, -1}, {-1, -1}};
}  // namespace

struct arbor_denoiser {
  cudaStream_t stream = nullptr;
  int max_batch = 0, max_w = 0, max_h = 0;
  long param_count = 0;
  LayerParams layer[kLayers];
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // FP32 parameters, gradients, moments
  bf16 *wf = nullptr, *wb = nullptr;                              // BF16 forward / backward-data weights
  long wf_off[kLayers];
  bf16* act[kActs] = {};
  bf16* grad[kActs] = {};
  bf16* dcat[3] = {};     // skip gradients from the concat, levels 0..2
  float* out = nullptr;   // network output, kOutC FP32 channels
  bf16* dout = nullptr;
  float* loss = nullptr;  // device scalar
  float loss_host = 0.0f;
  int* err = nullptr;     // device flag: a tcgen05 wait gave up
  float* part = nullptr;  // partial weight / bias gradients of one layer (wgrad_kernel, bgrad_kernel)
  size_t part_floats = 0;
  bool tc = true;         // forward convolutions on tcgen05
  bool l2 = false;        // training loss: squared (true) or absolute (false) difference in log(1 + radiance)
  long steps = 0;
  size_t allocated = 0;
};

namespace {

long level_pixels(const arbor_denoiser* d, int level, int batch, int w, int h) { return (long)batch * (w >> level) * (h >> level); }

int launch_conv(const ConvArgs& a, cudaStream_t s) {
  const dim3 grid((unsigned)(((a.w + 7) / 8) * ((a.h + 7) / 8)), 1, (unsigned)a.n);
  const int kc = a.cin % 32 == 0 ? 32 : 16;
  const int nt = a.cout % 64 == 0 ? 8 : (a.cout % 32 == 0 ? 4 : 2);
  dim3 g = grid;
  g.y = (unsigned)(a.cout / (nt * 8));
#define DN_CONV(KC, NT)                                                                                                 \
  do {                                                                                                                  \
    static bool ready = false;                                                                                          \
    if (!ready) {                                                                                                       \
      if (cudaFuncSetAttribute(conv_kernel<KC, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, conv_smem_bytes<KC, NT>()) != \
          cudaSuccess)                                                                                                  \
        return cuda_fail("cudaFuncSetAttribute (conv)", cudaGetLastError());                                            \
      ready = true;                                                                                                     \
    }                                                                                                                   \
    conv_kernel<KC, NT><<<g, 128, conv_smem_bytes<KC, NT>(), s>>>(a);                                                   \
  } while (0)
  if (kc == 32 && nt == 8) DN_CONV(32, 8);
  else if (kc == 32 && nt == 4) DN_CONV(32, 4);
  else if (kc == 32 && nt == 2) DN_CONV(32, 2);
  else if (kc == 16 && nt == 8) DN_CONV(16, 8);
  else if (kc == 16 && nt == 4) DN_CONV(16, 4);
  else DN_CONV(16, 2);
#undef DN_CONV
  count_launch();
  return check_launch("conv_kernel");
}

// The forward convolutions on tcgen05 (cout 16..128).  R rows per CTA keep
// R x N TMEM columns within 256, so two CTAs per SM fit the 512 columns.
// Shared memory per CTA is padded so that the CTAs one SM can hold never ask
// for more than its 512 TMEM columns together (an allocation then never
// waits on another CTA).
template <int N, int CC, int R>
constexpr int conv_tc_launch_smem() {
  constexpr int need = conv_tc_smem_bytes<N, CC, R>();
  constexpr int floor_b = 228 * 1024 / (512 / pow2_cols(R * N) + 1) + 1024;
  return need > floor_b ? need : floor_b;
}
template <int N, int CC, int R>
int launch_tc(const ConvArgs& a, int* err, cudaStream_t s) {
  static_assert(pow2_cols(R * N) <= 256, "TMEM budget");
  constexpr int smem = conv_tc_launch_smem<N, CC, R>();
  static_assert(smem <= 227 * 1024, "shared memory per CTA");
  static bool ready = false;
  if (!ready) {
    if (cudaFuncSetAttribute(conv_tc_kernel<N, CC, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return cuda_fail("cudaFuncSetAttribute (conv_tc)", cudaGetLastError());
    ready = true;
  }
  const dim3 grid((unsigned)(((a.w + 127) / 128) * ((a.h + R - 1) / R) * a.n));
  conv_tc_kernel<N, CC, R><<<grid, 128, smem, s>>>(a, err);
  count_launch();
  return check_launch("conv_tc_kernel");
}
// Row-streaming launch: rows per CTA chosen so the grid fills the SMs once
// at the occupancy the shared memory allows (TMEM: 2 x N columns per CTA).
template <int N, int CIN>
int launch_row(const ConvArgs& a, int* err, cudaStream_t s) {
  constexpr int need = conv_row_smem_bytes<N, CIN>();
  constexpr int floor_b = 228 * 1024 / (512 / pow2_cols(2 * N) + 1) + 1024;
  constexpr int smem = need > floor_b ? need : floor_b;
  static_assert(smem <= 227 * 1024, "shared memory per CTA");
  static bool ready = false;
  static int sms = 0;
  if (!ready) {
    if (cudaFuncSetAttribute(conv_row_kernel<N, CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return cuda_fail("cudaFuncSetAttribute (conv_row)", cudaGetLastError());
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
    ready = true;
  }
  const int per_sm = std::max(1, 228 * 1024 / (smem + 1024));
  const long segs = (long)((a.w + 127) / 128) * a.n;
  long rows = ((long)a.h * segs + (long)sms * per_sm - 1) / ((long)sms * per_sm);
  if (rows < 4) rows = 4;
  if (rows > a.h) rows = a.h;
  const dim3 grid((unsigned)(segs * ((a.h + rows - 1) / rows)));
  conv_row_kernel<N, CIN><<<grid, 128, smem, s>>>(a, (int)rows, err);
  count_launch();
  return check_launch("conv_row_kernel");
}

bool tc_shape(const ConvArgs& a) { return a.cout == 16 || a.cout == 32 || a.cout == 64 || a.cout == 96 || a.cout == 128; }
int launch_conv_tc(const ConvArgs& a, int* err, cudaStream_t s) {
  // Layers whose weights and a 5-row ring fit in shared memory at 2 or more
  // CTAs per SM stream rows (measured 11-19 % faster per layer); 96 -> 32,
  // at 1 CTA per SM, was 2.3x slower that way and keeps the chunked form,
  // as do the layers whose weights do not fit.
  if (a.cout == 32 && a.cin == 16) return launch_row<32, 16>(a, err, s);
  if (a.cout == 32 && a.cin == 32) return launch_row<32, 32>(a, err, s);
  if (a.cout == 16 && a.cin == 32) return launch_row<16, 32>(a, err, s);
  if (a.cout == 64 && a.cin == 32) return launch_row<64, 32>(a, err, s);
  if (a.cout == 64 && a.cin == 64) return launch_row<64, 64>(a, err, s);
  if (a.cout == 96 && a.cin == 64) return launch_row<96, 64>(a, err, s);
  switch (a.cout) {
    case 16: return launch_tc<16, 16, 8>(a, err, s);
    case 32: return launch_tc<32, 16, 8>(a, err, s);
    case 64: return launch_tc<64, 16, 4>(a, err, s);
    case 96: return launch_tc<96, 16, 2>(a, err, s);
    default: return launch_tc<128, 16, 2>(a, err, s);
  }
}

// Pixel ranges of one layer's weight-gradient GEMM: about 1184 CTAs (8 per
// SM) over (cout / 64) x 9 x (cin / ci_tile) tiles, ranges of >= 256 pixels.
long wgrad_per(long pixels, int cin, int cout) {
  const int ci_tile = cin % 32 == 0 ? 32 : 16;
  const int base = ((cout + 63) / 64) * 9 * (cin / ci_tile);
  long split = 1184 / base;
  if (split < 1) split = 1;
  long per = (pixels + split - 1) / split;
  per = (per + 31) / 32 * 32;
  if (per < 256) per = 256;
  return per;
}
// Largest number of pixel ranges wgrad_per gives for any pixel count.
long wgrad_max_splits(int cin, int cout) {
  const int ci_tile = cin % 32 == 0 ? 32 : 16;
  const long base = ((cout + 63) / 64) * 9 * (cin / ci_tile);
  return std::max(1L, 1184 / base) + 1;
}
constexpr int kBgradBlocks = 1184;

// dw += the layer's weight gradient: partial sums per pixel range into
// `part`, then folded in range order (the same sums whatever the schedule).
int launch_wgrad(const bf16* dy, const bf16* x, const bf16* x2, int cs, float* dw, float* part, size_t part_floats, int cin, int cout, int n,
                 int h, int w, cudaStream_t s) {
  WgradArgs a{dy, x, part, cin, cout, n, h, w, 0, x2, cs};
  const long pixels = (long)n * h * w;
  const int ci_tile = cin % 32 == 0 ? 32 : 16;
  const long per = wgrad_per(pixels, cin, cout);
  a.pixels_per_cta = (int)per;
  const long splits = (pixels + per - 1) / per;
  const long size = (long)cout * 9 * cin;
  if ((size_t)(splits * size) > part_floats) {
    set_error("launch_wgrad: %ld partial gradients exceed the %zu-float buffer", splits * size, part_floats);
    return ARBOR_ERR_LIMIT;
  }
  const dim3 grid((unsigned)splits, (unsigned)((cout + 63) / 64), (unsigned)(9 * (cin / ci_tile)));
  if (ci_tile == 32)
    wgrad_kernel<32><<<grid, 128, 0, s>>>(a);
  else
    wgrad_kernel<16><<<grid, 128, 0, s>>>(a);
  reduce_kernel<<<ew_grid(size), 256, 0, s>>>(part, dw, size, (int)splits);
  count_launch(2);
  return check_launch("wgrad_kernel");
}

int check_size(const char* what, int batch, int w, int h, const arbor_denoiser* d) {
  if (batch < 1 || w < 8 || h < 8 || w % 8 || h % 8) {
    set_error("%s: batch >= 1 and width, height multiples of 8 are required (got %d x %d x %d)", what, batch, w, h);
    return ARBOR_ERR_VALUE;
  }
  if ((long)batch * w * h > (long)d->max_batch * d->max_w * d->max_h) {
    set_error("%s: %d x %d x %d pixels exceed the %d x %d x %d the denoiser was created for", what, batch, w, h, d->max_batch, d->max_w,
              d->max_h);
    return ARBOR_ERR_LIMIT;
  }
  return ARBOR_OK;
}

int cast_weights(arbor_denoiser* d) {
  for (int l = 0; l < kLayers; l++) {
    const LayerParams& L = d->layer[l];
    cast_kernel<<<ew_grid((long)L.cout * 9 * L.cin), 256, 0, d->stream>>>(d->p + L.woff, d->wf + d->wf_off[l], d->wb + d->wf_off[l], L.cin,
                                                                          L.cout);
    count_launch();
  }
  return check_launch("cast_kernel");
}

// Forward pass over `features` (batch x h x w x 16 BF16); the output lands in d->out.
int forward(arbor_denoiser* d, const bf16* features, int batch, int w, int h) {
  cudaStream_t s = d->stream;
  const bf16* in[kActs];
  for (int k = 0; k < kActs; k++) in[k] = d->act[k];
  in[aF] = features;
  auto conv = [&](int l) {
    const LayerParams& L = d->layer[l];
    const int lv = kAct[kIn[l]].level;
    ConvArgs a{in[kIn[l]], d->wf + d->wf_off[l], d->p + L.boff,
               kOut[l] < 0 ? (void*)d->out : (void*)d->act[kOut[l]], nullptr, L.cin, L.cout, batch, h >> lv, w >> lv, kSpec[l][2],
               kOut[l] < 0 ? 1 : 0, nullptr, 0};
    if (kCat[l][0] >= 0) {  // a decoder input: read the skip and the upsampled level below in place
      a.x = d->act[kCat[l][0]];
      a.x2 = d->act[kCat[l][1]];
      a.cs = kAct[kCat[l][0]].channels;
    }
    return d->tc && tc_shape(a) ? launch_conv_tc(a, d->err, s) : launch_conv(a, s);
  };
  auto pool = [&](int src, int dst) {
    const int lv = kAct[src].level;
    const long n = level_pixels(d, lv + 1, batch, w, h) * kAct[src].channels / 8;
    pool_kernel<<<ew_grid(n), 256, 0, s>>>(d->act[src], d->act[dst], batch, h >> lv, w >> lv, kAct[src].channels);
    count_launch();
    return check_launch("pool_kernel");
  };
  int st;
  if ((st = conv(0)) || (st = conv(1)) || (st = pool(aE0, aP1)) || (st = conv(2)) || (st = conv(3)) || (st = pool(aE1, aP2)) ||
      (st = conv(4)) || (st = conv(5)) || (st = pool(aE2, aP3)) || (st = conv(6)) || (st = conv(7)) || (st = conv(8)) ||
      (st = conv(9)) || (st = conv(10)) || (st = conv(11)) || (st = conv(12)) || (st = conv(13)) || (st = conv(14)))
    return st;
  return ARBOR_OK;
}

// Backward pass from d->dout; accumulates into d->g.
int backward(arbor_denoiser* d, const bf16* features, int batch, int w, int h) {
  cudaStream_t s = d->stream;
  auto x_of = [&](int l) -> const bf16* { return kIn[l] == aF ? features : d->act[kIn[l]]; };
  // weight and bias gradients of layer l from dY (its pre-activation gradient)
  auto wgrad = [&](int l, const bf16* dy) {
    const LayerParams& L = d->layer[l];
    const int lv = kAct[kIn[l]].level;
    const bool cat = kCat[l][0] >= 0;
    if (int st = launch_wgrad(dy, cat ? d->act[kCat[l][0]] : x_of(l), cat ? d->act[kCat[l][1]] : nullptr, cat ? kAct[kCat[l][0]].channels : 0,
                              d->g + L.woff, d->part, d->part_floats, L.cin, L.cout, batch, h >> lv, w >> lv, s))
      return st;
    const long px = level_pixels(d, lv, batch, w, h);
    const unsigned blocks = (unsigned)std::min<long>(kBgradBlocks, (px * L.cout + 255) / 256 + 1);
    bgrad_kernel<<<blocks, 256, 0, s>>>(dy, d->part, L.cout, px);
    reduce_kernel<<<1, 256, 0, s>>>(d->part, d->g + L.boff, L.cout, (int)blocks);
    count_launch(2);
    return check_launch("bgrad_kernel");
  };
  // input gradient of layer l: conv of dY with the rotated, transposed
  // weights; mask_act: the input's activation derivative (or -1: none)
  auto dgrad = [&](int l, const bf16* dy, bf16* dx, int mask_act) {
    const LayerParams& L = d->layer[l];
    const int lv = kAct[kIn[l]].level;
    ConvArgs a{dy, d->wb + d->wf_off[l], nullptr, dx, mask_act >= 0 ? d->act[mask_act] : nullptr, L.cout, L.cin, batch, h >> lv, w >> lv, 0, 0,
               nullptr, 0};
    // tcgen05 where the output width has a tensor-core kernel (all but the
    // 160- and 224-channel decoder inputs); the same K = 16 accumulation order
    // as the mma.sync kernel.
    return d->tc && tc_shape(a) ? launch_conv_tc(a, d->err, s) : launch_conv(a, s);
  };
  auto upcat_back = [&](int cat, int skip_level, int low) {
    const int lv = kAct[cat].level;
    const int cs = kAct[cat].channels - kAct[low].channels, cl = kAct[low].channels;
    const long n = (level_pixels(d, lv, batch, w, h) * cs + level_pixels(d, lv + 1, batch, w, h) * cl) / 8;
    upcat_back_kernel<<<ew_grid(n), 256, 0, s>>>(d->grad[cat], d->act[low], d->dcat[skip_level], d->grad[low], batch, h >> lv, w >> lv, cs,
                                                 cl);
    count_launch();
    return check_launch("upcat_back_kernel");
  };
  auto pool_back = [&](int pooled, int skip, int skip_level) {
    const int lv = kAct[skip].level;
    const long n = level_pixels(d, lv, batch, w, h) * kAct[skip].channels / 8;
    pool_back_kernel<<<ew_grid(n), 256, 0, s>>>(d->grad[pooled], d->dcat[skip_level], d->act[skip], d->grad[skip], batch, h >> lv, w >> lv,
                                                kAct[skip].channels);
    count_launch();
    return check_launch("pool_back_kernel");
  };
  int st;
  // decoder level 0
  if ((st = wgrad(14, d->dout)) || (st = dgrad(14, d->dout, d->grad[aD0], aD0))) return st;
  if ((st = wgrad(13, d->grad[aD0])) || (st = dgrad(13, d->grad[aD0], d->grad[aD0a], aD0a))) return st;
  if ((st = wgrad(12, d->grad[aD0a])) || (st = dgrad(12, d->grad[aD0a], d->grad[aC0], -1))) return st;
  if ((st = upcat_back(aC0, 0, aD1))) return st;
  // decoder level 1
  if ((st = wgrad(11, d->grad[aD1])) || (st = dgrad(11, d->grad[aD1], d->grad[aD1a], aD1a))) return st;
  if ((st = wgrad(10, d->grad[aD1a])) || (st = dgrad(10, d->grad[aD1a], d->grad[aC1], -1))) return st;
  if ((st = upcat_back(aC1, 1, aD2))) return st;
  // decoder level 2
  if ((st = wgrad(9, d->grad[aD2])) || (st = dgrad(9, d->grad[aD2], d->grad[aD2a], aD2a))) return st;
  if ((st = wgrad(8, d->grad[aD2a])) || (st = dgrad(8, d->grad[aD2a], d->grad[aC2], -1))) return st;
  if ((st = upcat_back(aC2, 2, aB3))) return st;
  // bottleneck
  if ((st = wgrad(7, d->grad[aB3])) || (st = dgrad(7, d->grad[aB3], d->grad[aB3a], aB3a))) return st;
  if ((st = wgrad(6, d->grad[aB3a])) || (st = dgrad(6, d->grad[aB3a], d->grad[aP3], -1))) return st;
  if ((st = pool_back(aP3, aE2, 2))) return st;
  // encoder level 2
  if ((st = wgrad(5, d->grad[aE2])) || (st = dgrad(5, d->grad[aE2], d->grad[aE2a], aE2a))) return st;
  if ((st = wgrad(4, d->grad[aE2a])) || (st = dgrad(4, d->grad[aE2a], d->grad[aP2], -1))) return st;
  if ((st = pool_back(aP2, aE1, 1))) return st;
  // encoder level 1
  if ((st = wgrad(3, d->grad[aE1])) || (st = dgrad(3, d->grad[aE1], d->grad[aE1a], aE1a))) return st;
  if ((st = wgrad(2, d->grad[aE1a])) || (st = dgrad(2, d->grad[aE1a], d->grad[aP1], -1))) return st;
  if ((st = pool_back(aP1, aE0, 0))) return st;
  // encoder level 0
  if ((st = wgrad(1, d->grad[aE0])) || (st = dgrad(1, d->grad[aE0], d->grad[aE0a], aE0a))) return st;
  if ((st = wgrad(0, d->grad[aE0a]))) return st;
  return ARBOR_OK;
}

int live(arbor_denoiser* d, const char* what) {
  if (d == nullptr) {
    set_error("%s: denoiser is NULL", what);
    return ARBOR_ERR_NULL;
  }
  return ARBOR_OK;
}

}  // namespace

extern "C" int arbor_denoiser_create(arbor_denoiser** out, int max_batch, int max_width, int max_height, uint32_t seed, arbor_stream stream) {
  if (out == nullptr) {
    set_error("arbor_denoiser_create: out is NULL");
    return ARBOR_ERR_NULL;
  }
  *out = nullptr;
  if (max_batch < 1 || max_width < 8 || max_height < 8 || max_width % 8 || max_height % 8) {
    set_error("arbor_denoiser_create: batch >= 1 and width, height multiples of 8 are required (got %d x %d x %d)", max_batch, max_width,
              max_height);
    return ARBOR_ERR_VALUE;
  }
  if ((long)max_batch * max_width * max_height > (1L << 26)) {
    set_error("arbor_denoiser_create: %d x %d x %d pixels exceed 2^26", max_batch, max_width, max_height);
    return ARBOR_ERR_LIMIT;
  }
  if (!arbor_device_ready()) {
    set_error("arbor_denoiser_create: no sm_100 CUDA device is available");
    return ARBOR_ERR_NO_DEVICE;
  }
  arbor_denoiser* d = new (std::nothrow) arbor_denoiser();
  if (d == nullptr) {
    set_error("arbor_denoiser_create: out of host memory");
    return ARBOR_ERR_LIMIT;
  }
  auto fail = [&](int s) {
    arbor_denoiser_destroy(d);
    return s;
  };
  d->stream = stream;
  d->max_batch = max_batch;
  d->max_w = max_width;
  d->max_h = max_height;
  long off = 0, woff = 0;
  for (int l = 0; l < kLayers; l++) {
    LayerParams& L = d->layer[l];
    L.cin = kSpec[l][0];
    L.cout = kSpec[l][1];
    L.woff = off;
    off += (long)L.cout * 9 * L.cin;
    L.boff = off;
    off += L.cout;
    d->wf_off[l] = woff;
    woff += (long)L.cout * 9 * L.cin;
  }
  d->param_count = off;
  cudaError_t ce;
  auto alloc = [&](void** ptr, size_t bytes) {
    ce = cudaMalloc(ptr, bytes);
    if (ce == cudaSuccess) d->allocated += bytes;
    return ce == cudaSuccess;
  };
  const size_t pb = (size_t)off * 4;
  if (!alloc((void**)&d->p, pb) || !alloc((void**)&d->g, pb) || !alloc((void**)&d->m, pb) || !alloc((void**)&d->v, pb) ||
      !alloc((void**)&d->wf, (size_t)woff * 2) || !alloc((void**)&d->wb, (size_t)woff * 2) || !alloc((void**)&d->loss, 4) ||
      !alloc((void**)&d->err, 4))
    return fail(cuda_fail("cudaMalloc (denoiser parameters)", ce));
  const long px0 = (long)max_batch * max_width * max_height;
  for (int k = 0; k < kActs; k++) {
    const size_t bytes = (size_t)(px0 >> (2 * kAct[k].level)) * kAct[k].channels * 2;
    const bool concat = k == aC0 || k == aC1 || k == aC2;  // read in place by the decoder convolutions, never stored
    if (k != aF && !concat && !alloc((void**)&d->act[k], bytes)) return fail(cuda_fail("cudaMalloc (denoiser activations)", ce));
    if (!alloc((void**)&d->grad[k], bytes)) return fail(cuda_fail("cudaMalloc (denoiser gradients)", ce));
  }
  const int skips[3] = {aE0, aE1, aE2};
  for (int lv = 0; lv < 3; lv++)
    if (!alloc((void**)&d->dcat[lv], (size_t)(px0 >> (2 * lv)) * kAct[skips[lv]].channels * 2))
      return fail(cuda_fail("cudaMalloc (denoiser concat gradients)", ce));
  if (!alloc((void**)&d->out, (size_t)px0 * kOutC * 4) || !alloc((void**)&d->dout, (size_t)px0 * kOutC * 2))
    return fail(cuda_fail("cudaMalloc (denoiser output)", ce));
  for (int l = 0; l < kLayers; l++) {
    const LayerParams& L = d->layer[l];
    d->part_floats = std::max(d->part_floats, (size_t)(wgrad_max_splits(L.cin, L.cout) * L.cout * 9 * L.cin));
    d->part_floats = std::max(d->part_floats, (size_t)kBgradBlocks * L.cout);
  }
  if (!alloc((void**)&d->part, d->part_floats * 4)) return fail(cuda_fail("cudaMalloc (denoiser partial gradients)", ce));
  // He-normal weights (the output layer 10x smaller), zero biases and moments
  if ((ce = cudaMemsetAsync(d->err, 0, 4, stream)) != cudaSuccess || (ce = cudaMemsetAsync(d->p, 0, pb, stream)) != cudaSuccess ||
      (ce = cudaMemsetAsync(d->g, 0, pb, stream)) != cudaSuccess ||
      (ce = cudaMemsetAsync(d->m, 0, pb, stream)) != cudaSuccess || (ce = cudaMemsetAsync(d->v, 0, pb, stream)) != cudaSuccess)
    return fail(cuda_fail("cudaMemsetAsync", ce));
  for (int l = 0; l < kLayers; l++) {
    const LayerParams& L = d->layer[l];
    const float stdev = sqrtf(2.0f / (9.0f * L.cin)) * (l == kLayers - 1 ? 0.1f : 1.0f);
    init_kernel<<<ew_grid((long)L.cout * 9 * L.cin), 256, 0, stream>>>(d->p + L.woff, (long)L.cout * 9 * L.cin, stdev, seed * 977u + l);
    count_launch();
  }
  if (int st = cast_weights(d)) return fail(st);
  if ((ce = cudaStreamSynchronize(stream)) != cudaSuccess) return fail(cuda_fail("cudaStreamSynchronize", ce));
  *out = d;
  return ARBOR_OK;
}

namespace {
// A tcgen05 wait that gave up leaves its flag set: report it (and clear it).
int check_err(arbor_denoiser* d, const char* what) {
  int e = 0;
  DN_CUDA(cudaMemcpyAsync(&e, d->err, 4, cudaMemcpyDeviceToHost, d->stream));
  DN_CUDA(cudaStreamSynchronize(d->stream));
  if (e) {
    cudaMemsetAsync(d->err, 0, 4, d->stream);
    set_error("%s: a tensor-core convolution timed out waiting for its MMAs", what);
    return ARBOR_ERR_TIMEOUT;
  }
  return ARBOR_OK;
}
}  // namespace

extern "C" int arbor_denoiser_set_backend(arbor_denoiser* d, int tcgen05) {
  if (int s = live(d, "arbor_denoiser_set_backend")) return s;
  d->tc = tcgen05 != 0;
  return ARBOR_OK;
}

extern "C" int arbor_denoiser_set_loss(arbor_denoiser* d, int kind) {
  if (int s = live(d, "arbor_denoiser_set_loss")) return s;
  if (kind != ARBOR_LOSS_L1 && kind != ARBOR_LOSS_L2) {
    set_error("arbor_denoiser_set_loss: kind must be ARBOR_LOSS_L1 (0) or ARBOR_LOSS_L2 (1), got %d", kind);
    return ARBOR_ERR_VALUE;
  }
  d->l2 = kind == ARBOR_LOSS_L2;
  return ARBOR_OK;
}

extern "C" int arbor_denoiser_param_count(arbor_denoiser* d, size_t* count) {
  if (int s = live(d, "arbor_denoiser_param_count")) return s;
  if (count == nullptr) {
    set_error("arbor_denoiser_param_count: count is NULL");
    return ARBOR_ERR_NULL;
  }
  *count = (size_t)d->param_count;
  return ARBOR_OK;
}

extern "C" int arbor_denoiser_get_params(arbor_denoiser* d, float* host, size_t count) {
  if (int s = live(d, "arbor_denoiser_get_params")) return s;
  if (host == nullptr || count < (size_t)d->param_count) {
    set_error("arbor_denoiser_get_params: need room for %ld floats", d->param_count);
    return host == nullptr ? ARBOR_ERR_NULL : ARBOR_ERR_LIMIT;
  }
  DN_CUDA(cudaMemcpyAsync(host, d->p, (size_t)d->param_count * 4, cudaMemcpyDeviceToHost, d->stream));
  DN_CUDA(cudaStreamSynchronize(d->stream));
  return ARBOR_OK;
}

extern "C" int arbor_denoiser_set_params(arbor_denoiser* d, const float* host, size_t count) {
  if (int s = live(d, "arbor_denoiser_set_params")) return s;
  if (host == nullptr || count != (size_t)d->param_count) {
    set_error("arbor_denoiser_set_params: expected %ld floats", d->param_count);
    return host == nullptr ? ARBOR_ERR_NULL : ARBOR_ERR_VALUE;
  }
  for (size_t i = 0; i < count; i++)
    if (!std::isfinite(host[i])) {
      set_error("arbor_denoiser_set_params: parameter %zu is not finite", i);
      return ARBOR_ERR_VALUE;
    }
  DN_CUDA(cudaMemcpyAsync(d->p, host, count * 4, cudaMemcpyHostToDevice, d->stream));
  if (int st = cast_weights(d)) return st;
  DN_CUDA(cudaStreamSynchronize(d->stream));
  return ARBOR_OK;
}

extern "C" int arbor_denoiser_features(const float* Linear, const float* Guide, const float* Normal, const float* Hit, const float* Filtered,
                                       int width, int height, uint16_t* features, arbor_stream stream) {
  bool empty;
  if (int s = check_image("arbor_denoiser_features", width, height, &empty)) return s;
  const size_t img = empty ? 0 : image_bytes(width, height);
  const Binding b[] = {{Linear, img, false, 16, "Linear"},
                       {Guide, img, false, 16, "Guide"},
                       {Normal, img, false, 16, "Normal"},
                       {Hit, img, false, 16, "Hit"},
                       {Filtered, img, false, 16, "Filtered"},
                       {features, (size_t)width * height * kFeat * 2, true, 16, "features"}};
  if (int s = check_bindings("arbor_denoiser_features", b)) return s;
  if (empty) return ARBOR_OK;
  const long px = (long)width * height;
  features_kernel<<<ew_grid(px), 256, 0, stream>>>(reinterpret_cast<const float4*>(Linear), reinterpret_cast<const float4*>(Guide),
                                                   reinterpret_cast<const float4*>(Normal), reinterpret_cast<const float4*>(Hit),
                                                   reinterpret_cast<const float4*>(Filtered), reinterpret_cast<bf16*>(features), px);
  count_launch();
  return check_launch("arbor_denoiser_features");
}

extern "C" int arbor_denoiser_train_step(arbor_denoiser* d, const uint16_t* features, const float* base, const float* target, int batch,
                                         int width, int height, float lr, float* loss) {
  if (int s = live(d, "arbor_denoiser_train_step")) return s;
  if (features == nullptr || base == nullptr || target == nullptr) {
    set_error("arbor_denoiser_train_step: features, base and target must not be NULL");
    return ARBOR_ERR_NULL;
  }
  if (int s = check_size("arbor_denoiser_train_step", batch, width, height, d)) return s;
  if (!(lr > 0.0f) || !std::isfinite(lr)) {
    set_error("arbor_denoiser_train_step: lr must be positive and finite");
    return ARBOR_ERR_VALUE;
  }
  cudaStream_t s = d->stream;
  const bf16* f = reinterpret_cast<const bf16*>(features);
  if (int st = forward(d, f, batch, width, height)) return st;
  const long px = (long)batch * width * height;
  DN_CUDA(cudaMemsetAsync(d->loss, 0, 4, s));
  loss_kernel<<<ew_grid(px), 256, 0, s>>>(d->out, reinterpret_cast<const float4*>(base), reinterpret_cast<const float4*>(target), d->dout,
                                          d->loss, px, 1.0f / (float)(px * 3), d->l2);
  count_launch();
  if (int st = check_launch("loss_kernel")) return st;
  if (int st = backward(d, f, batch, width, height)) return st;
  d->steps++;
  const float b1 = 0.9f, b2 = 0.999f;
  AdamArgs a{d->p, d->g, d->m, d->v, d->param_count, lr, b1, b2, 1e-8f, 1.0f - powf(b1, (float)d->steps), 1.0f - powf(b2, (float)d->steps)};
  adam_kernel<<<ew_grid(d->param_count), 256, 0, s>>>(a);
  count_launch();
  if (int st = check_launch("adam_kernel")) return st;
  if (int st = cast_weights(d)) return st;
  if (loss) {
    DN_CUDA(cudaMemcpyAsync(&d->loss_host, d->loss, 4, cudaMemcpyDeviceToHost, s));
    DN_CUDA(cudaStreamSynchronize(s));
    *loss = d->loss_host / (float)(px * 3);
    return check_err(d, "arbor_denoiser_train_step");
  }
  return ARBOR_OK;
}

extern "C" int arbor_denoiser_gradient(arbor_denoiser* d, const uint16_t* features, const float* base, const float* target, int batch,
                                       int width, int height, float* grad, size_t count, float* loss) {
  if (int s = live(d, "arbor_denoiser_gradient")) return s;
  if (features == nullptr || base == nullptr || target == nullptr || grad == nullptr) {
    set_error("arbor_denoiser_gradient: features, base, target and grad must not be NULL");
    return ARBOR_ERR_NULL;
  }
  if (count < (size_t)d->param_count) {
    set_error("arbor_denoiser_gradient: need room for %ld floats", d->param_count);
    return ARBOR_ERR_LIMIT;
  }
  if (int s = check_size("arbor_denoiser_gradient", batch, width, height, d)) return s;
  cudaStream_t s = d->stream;
  const bf16* f = reinterpret_cast<const bf16*>(features);
  if (int st = forward(d, f, batch, width, height)) return st;
  const long px = (long)batch * width * height;
  DN_CUDA(cudaMemsetAsync(d->loss, 0, 4, s));
  loss_kernel<<<ew_grid(px), 256, 0, s>>>(d->out, reinterpret_cast<const float4*>(base), reinterpret_cast<const float4*>(target), d->dout,
                                          d->loss, px, 1.0f / (float)(px * 3), d->l2);
  count_launch();
  if (int st = check_launch("loss_kernel")) return st;
  if (int st = backward(d, f, batch, width, height)) return st;
  DN_CUDA(cudaMemcpyAsync(grad, d->g, (size_t)d->param_count * 4, cudaMemcpyDeviceToHost, s));
  DN_CUDA(cudaMemcpyAsync(&d->loss_host, d->loss, 4, cudaMemcpyDeviceToHost, s));
  // the gradient buffer starts the next step at zero, as after an Adam step
  DN_CUDA(cudaMemsetAsync(d->g, 0, (size_t)d->param_count * 4, s));
  DN_CUDA(cudaStreamSynchronize(s));
  if (loss) *loss = d->loss_host / (float)(px * 3);
  return check_err(d, "arbor_denoiser_gradient");
}

extern "C" int arbor_denoiser_infer(arbor_denoiser* d, const uint16_t* features, const float* base, float* denoised, int width, int height) {
  if (int s = live(d, "arbor_denoiser_infer")) return s;
  if (features == nullptr || base == nullptr || denoised == nullptr) {
    set_error("arbor_denoiser_infer: features, base and denoised must not be NULL");
    return ARBOR_ERR_NULL;
  }
  if (int s = check_size("arbor_denoiser_infer", 1, width, height, d)) return s;
  if (int st = forward(d, reinterpret_cast<const bf16*>(features), 1, width, height)) return st;
  const long px = (long)width * height;
  output_kernel<<<ew_grid(px), 256, 0, d->stream>>>(d->out, reinterpret_cast<const float4*>(base), reinterpret_cast<float4*>(denoised), px);
  count_launch();
  return check_launch("output_kernel");
}

extern "C" int arbor_denoiser_check(arbor_denoiser* d) {
  if (int s = live(d, "arbor_denoiser_check")) return s;
  return check_err(d, "arbor_denoiser_check");
}

extern "C" int arbor_denoiser_destroy(arbor_denoiser* d) {
  if (d == nullptr) return ARBOR_OK;
  if (d->stream) cudaStreamSynchronize(d->stream);
  void* bufs[] = {d->p, d->g, d->m, d->v, d->wf, d->wb, d->out, d->dout, d->loss, d->err, d->part, d->dcat[0], d->dcat[1], d->dcat[2]};
  for (void* p : bufs)
    if (p) cudaFree(p);
  for (int k = 0; k < kActs; k++) {
    if (d->act[k]) cudaFree(d->act[k]);
    if (d->grad[k]) cudaFree(d->grad[k]);
  }
  delete d;
  return ARBOR_OK;
}

extern "C" int arbor_accumulate(float* sum, const float* x, size_t count, float scale, arbor_stream stream) {
  if (sum == nullptr || x == nullptr) {
    set_error("arbor_accumulate: sum and x must not be NULL");
    return count == 0 ? ARBOR_OK : ARBOR_ERR_NULL;
  }
  if (!std::isfinite(scale)) {
    set_error("arbor_accumulate: scale must be finite");
    return ARBOR_ERR_VALUE;
  }
  if (count == 0) return ARBOR_OK;
  if (scale != 1.0f) {
    scale_kernel<<<ew_grid((long)count), 256, 0, stream>>>(sum, (long)count, scale);
    count_launch();
  }
  accumulate_kernel<<<ew_grid((long)count), 256, 0, stream>>>(sum, x, (long)count);
  count_launch();
  return check_launch("arbor_accumulate");
}
