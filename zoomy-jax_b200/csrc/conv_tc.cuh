// 3x3 convolution as an implicit GEMM on the 5th-generation tensor cores
// (tcgen05.mma, kind::f16 with bf16 operands, float32 accumulation in TMEM).
//
// GEMM view of one output tile: M = 128 pixels (an 8-wide by 16-tall block;
// GEMM row m is pixel (x0 + m % 8, y0 + m / 8)), N = output channels rounded
// up to 16, K = 9 taps x input channels rounded up to 16.  No im2col copy is
// made: the input tile with its one-pixel halo (10 x 18 pixels) is staged once
// in shared memory in the canonical no-swizzle K-major layout,
//   byte(chunk, q) = chunk * (180 * 16) + q * 16,   q = halo pixel (y * 10 + x),
// 8 consecutive channels (one 16-byte core-matrix row) per (chunk, q), so the
// A operand of tap (dy, dx) is the same buffer with its descriptor start moved
// by (dy * 10 + dx) * 16 bytes: rows of one 8-pixel line are 16 bytes apart
// (the core matrix), successive lines 160 bytes apart (stride byte offset),
// the two 8-channel halves of a K=16 step 2880 bytes apart (leading byte
// offset).  The weights sit next to it as [tap][chunk][n][8 channels].  One
// thread issues the 9 * Cin/16 MMAs of a tile and commits them to an
// mbarrier; the four warps then read the accumulator rows they own out of TMEM
// (tcgen05.ld 32x32b), add the bias, apply tanh and store float32 planes.
// CTAs are persistent over the tiles; the weights are staged once per CTA.
//
// Every wait is bounded: on a timeout the kernel raises a flag in the error
// word, skips the tile's stores, and still releases its TMEM columns.
#pragma once

#include <cuda.h>   // CUtensorMap (the type only; the encoder is fetched at run time)
#include <cuda_bf16.h>
#include <stdint.h>

namespace zb {
namespace unet {

constexpr int TCX = 8, TCY = 16;            // output tile (M = 128)
constexpr int THX = TCX + 2, THY = TCY + 2; // halo tile
constexpr int THP = THX * THY;              // 180 halo pixels
constexpr int TC_THREADS = 128;
constexpr unsigned TC_SPIN_LIMIT = 1u << 24;

__host__ __device__ constexpr int pad16(int c) { return (c + 15) & ~15; }

// How input channels [0, cin_a) are read: as stored, as the nearest-neighbour
// 2x upsampling of a half-resolution field (the U-Net's up(m2)), or as the 2x2
// average of a double-resolution field (pool(e2)); the last two replace the
// materialised upsampled / pooled activations.  Channels [cin_a, cin) are read
// as stored from the second source.
enum { SRC_DIRECT = 0, SRC_UP = 1, SRC_POOL = 2 };

__device__ __forceinline__ float src_at(const float* __restrict__ inA, int cin_a,
                                        const float* __restrict__ inB, int mode_a, int ci, int b,
                                        int B, int H, int W, int yy, int xx) {
  if (ci < cin_a) {
    if (mode_a == SRC_UP) {
      const int h = H >> 1, w = W >> 1;
      return inA[((size_t)ci * B + b) * h * w + (size_t)(yy >> 1) * w + (xx >> 1)];
    }
    if (mode_a == SRC_POOL) {
      const int w = 2 * W;
      const float* q = inA + ((size_t)ci * B + b) * (size_t)(2 * H) * w + (size_t)(2 * yy) * w + 2 * xx;
      return 0.25f * (q[0] + q[1] + q[w] + q[w + 1]);
    }
    return inA[((size_t)ci * B + b) * H * W + (size_t)yy * W + xx];
  }
  return inB[((size_t)(ci - cin_a) * B + b) * H * W + (size_t)yy * W + xx];
}

__host__ __device__ inline size_t tc_smem_bytes(int cinp, int coutp) {
  return (size_t)cinp * THP * 2 + (size_t)9 * cinp * coutp * 2 + 64;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// canonical K-major, no-swizzle shared-memory matrix descriptor (sm_100)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version for sm_100
  // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
  return d;
}

// instruction descriptor: D f32, A and B bf16, both K-major, M = 128, N
__device__ __forceinline__ uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t"
      "}\n"
      :
      : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Activation of the tensor-core epilogues: act 0 none, 1 tanhf, 2 tanh on the
// SFU (tanh.approx.f32), whose maximum relative error, about 2^-11 per the PTX
// ISA, sits below the bf16 rounding every activation takes before the next
// layer reads it.  The smoother application uses 2; training keeps 1, so its
// gradients stay those of the exact activation.
__device__ __forceinline__ float tanh_sfu(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// out[co][b][y][x] = act(bias[co] + sum_ci sum_tap w[co][ci][tap] in[ci][b][y+dy-1][x+dx-1])
// with the input channels [0, cin_a) from inA (read per mode_a, see src_at)
// and [cin_a, cin) from inB, the input rounded to bf16, zero padding at the
// image border.  err (may be null)
// receives 1 when an mbarrier wait timed out.
__global__ void __launch_bounds__(TC_THREADS)
conv3x3_tc(const float* __restrict__ inA, int cin_a, const float* __restrict__ inB, int cin,
           const __nv_bfloat16* __restrict__ w, const float* __restrict__ bias,
           float* __restrict__ out, int cout, int B, int H, int W, int act, int mode_a,
           int tmem_cols, unsigned* err) {
  extern __shared__ __align__(128) unsigned char tc_sm[];
  const int cinp = pad16(cin), coutp = pad16(cout);
  const int nch = cinp / 8;
  unsigned char* sA = tc_sm;
  unsigned char* sB = tc_sm + (size_t)cinp * THP * 2;
  unsigned long long* mbar = (unsigned long long*)(sB + (size_t)9 * cinp * coutp * 2);
  uint32_t* tmem_slot = (uint32_t*)(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // weights: [tap][chunk][n][8] bf16, zero outside (cout, cin)
  for (int e = tid; e < 9 * nch * coutp; e += TC_THREADS) {
    const int n = e % coutp;
    const int rest = e / coutp;
    const int ch = rest % nch, tap = rest / nch;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ci = ch * 8 + k;
      v[k] = (n < cout && ci < cin) ? w[((size_t)n * cin + ci) * 9 + tap] : __float2bfloat16(0.0f);
    }
    *(uint4*)(sB + ((size_t)(tap * nch + ch) * coutp + n) * 16) = *(const uint4*)v;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t mbar_a = smem_u32(mbar);
  const uint32_t sA_a = smem_u32(sA), sB_a = smem_u32(sB);
  const uint32_t idesc = tc_idesc(coutp);
  const size_t plane = (size_t)B * H * W;
  const int tiles_x = (W + TCX - 1) / TCX, tiles_y = (H + TCY - 1) / TCY;
  const int ntiles = tiles_x * tiles_y * B;
  uint32_t parity = 0;
  bool failed = false;

  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int b = t / (tiles_x * tiles_y);
    const int r = t - b * tiles_x * tiles_y;
    const int x0 = (r % tiles_x) * TCX, y0 = (r / tiles_x) * TCY;
    const size_t img = (size_t)b * H * W;
    // halo tile: one thread per (chunk, halo pixel), 8 channels -> 16 bytes
    for (int e = tid; e < nch * THP; e += TC_THREADS) {
      const int q = e % THP, ch = e / THP;
      const int yy = y0 - 1 + q / THX, xx = x0 - 1 + q % THX;
      __align__(16) __nv_bfloat16 v[8];
      const bool inside = yy >= 0 && yy < H && xx >= 0 && xx < W;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int ci = ch * 8 + k;
        const float f = (inside && ci < cin)
                            ? src_at(inA, cin_a, inB, mode_a, ci, b, B, H, W, yy, xx) : 0.0f;
        v[k] = __float2bfloat16_rn(f);
      }
      *(uint4*)(sA + ((size_t)ch * THP + q) * 16) = *(const uint4*)v;
    }
    // make the generic-proxy stores visible to the tensor core's async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      uint32_t acc = 0;
      for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3, dx = tap % 3;
        for (int g = 0; g < cinp / 16; ++g) {
          const uint32_t a = sA_a + (uint32_t)(2 * g) * (THP * 16) + (uint32_t)(dy * THX + dx) * 16;
          const uint32_t bb = sB_a + (uint32_t)((tap * nch + 2 * g) * coutp) * 16;
          tc_mma(tmem, tc_desc(a, THP * 16, THX * 16), tc_desc(bb, coutp * 16, 128), idesc, acc);
          acc = 1;
        }
      }
      tc_commit(mbar_a);
    }
    // wait for the tile's MMAs (bounded); the CTA agrees on the outcome so
    // every warp takes the same path through the collective TMEM loads
    bool done = false;
    for (unsigned it = 0; it < TC_SPIN_LIMIT; ++it) {
      if (mbar_try_wait(mbar_a, parity)) { done = true; break; }
    }
    parity ^= 1u;
    if (__syncthreads_or(done ? 0 : 1)) {
      failed = true;
      if (err && tid == 0) atomicExch(err, 1u);
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w owns accumulator rows (pixels) 32w .. 32w+31
    const int m = warp * 32 + lane;
    const int x = x0 + (m % TCX), y = y0 + (m / TCX);
    const bool store = x < W && y < H;
    for (int c0 = 0; c0 < coutp; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int co = c0 + i;
        if (store && co < cout) {
          float s = v[i] + (bias ? bias[co] : 0.0f);
          if (act == 1) s = tanhf(s);
          else if (act == 2) s = tanh_sfu(s);
          out[(size_t)co * plane + img + (size_t)y * W + x] = s;
        }
      }
    }
    // TMEM reads and smem reads of this tile complete before the next tile
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (failed) {
    // give an in-flight MMA a bounded chance to land before releasing TMEM
    for (unsigned it = 0; it < TC_SPIN_LIMIT; ++it)
      if (mbar_try_wait(mbar_a, parity ^ 1u)) break;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols)
                 : "memory");
  }
}

// ── the chunked bf16 activation layout (inference) ──────────────────────────
// An activation of C channels (C a multiple of 8) on B images H x W is stored
// as C / 8 chunks, chunk-major: byte ((chunk * B + b) * H * W + y * W + x) * 16
// holds channels 8 chunk .. 8 chunk + 7 of pixel (b, y, x) as bf16.  A pixel's
// chunk is then one 16-byte core-matrix row of the MMA's A operand, and a row
// of pixels is contiguous, so a tile's halo is staged with coalesced 16-byte
// cp.async copies (zero-filled outside the image) instead of per-thread
// float32 gathers; the producing layer writes it in its epilogue.  Values are
// the float32 activations rounded to bf16 once (the rounding the planar
// kernel applies when it stages them), so a network run through this layout
// gives the same bits as through conv3x3_tc.
constexpr int CBX = 16, CBY = 16;            // output region: two 8 x 16 M tiles
constexpr int CHX = CBX + 2, CHY = CBY + 2;  // halo region
constexpr int CHP = CHX * CHY;               // 324 halo pixels
// NTH = 256 (wide layers): eight warps stage the halo, and warps w and w + 4
// read TMEM lane quarter w of M tiles 0 and 1 in the epilogue; NTH = 128:
// four warps, each reading its lane quarter of both tiles.  Measured, one
// 1024^2 application: (24, 48) 0.473 ms with 128 threads everywhere, 0.448
// with 256 everywhere, 0.440 with 256 for the layers of six or more input
// chunks only (what the launcher takes); (8, 16) 0.249 / 0.255 / 0.247.
constexpr int CB_WIDE_CHUNKS = 6;
// one staged chunk: the 18 x 18 halo pixels x 16 bytes, its stride rounded up
// to 128 bytes (the alignment of a tensor-copy destination)
constexpr int CB_CHUNK_BYTES = CHP * 16;                            // 5184
constexpr int CB_CHUNK_STRIDE = ((CB_CHUNK_BYTES + 127) / 128) * 128;  // 5248

// staged chunks, weights, two mbarriers and the TMEM slot
__host__ __device__ inline size_t cb8_smem_bytes(int cinp, int coutp) {
  return (size_t)(cinp / 8) * CB_CHUNK_STRIDE + (size_t)9 * cinp * coutp * 2 + 64;
}

// TMA: a 4-D tiled tensor copy of one chunk's halo box into shared memory,
// completing on an mbarrier (no multicast)
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];"
      :
      : "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
        "r"(mbar)
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}

// Output forms of conv3x3_cb8.
enum { CB_OUT_CHUNKED = 0, CB_OUT_F32 = 1 };

// out = act(bias + conv3x3(in)) with in = [A (chA chunks; mode_a SRC_DIRECT
// at H x W or SRC_UP: the nearest 2x upsampling of an H/2 x W/2 field), then
// B (chB chunks at H x W)], cin real channels (the rest of the chunks and the
// padding to 16 read as zeros).  out_form CB_OUT_CHUNKED: out holds cout / 8
// chunks; pool (may be null) also receives the 2x2 average of the float32
// activation (H/2 x W/2 chunks, the average of conv3x3_tc's SRC_POOL loader,
// in its summation order).  CB_OUT_F32: out is float32 planes [co][b][y][x].
// H and W even.  act != 0: tanh on the SFU (the inference activation, act 2
// of conv3x3_tc).
// Staging: the chunks read as stored (A in SRC_DIRECT mode when tma_a, B when
// tma_b) arrive by TMA, one 4-D box (8 channels x 18 x 18 pixels x 1 image
// chunk) per chunk on the maps tm_a / tm_b (out-of-image pixels are filled
// with zeros by the copy), issued by one thread and completed on an mbarrier;
// the upsampled chunks of SRC_UP keep 16-byte cp.async copies (their address
// map is not a box); the padding chunks are zeroed once.  Staged chunk ch sits
// at ch * CB_CHUNK_STRIDE from the start of dynamic shared memory; a CTA whose
// dynamic shared memory does not start on 128 bytes (the alignment a tensor
// copy's destination needs) stages everything by cp.async instead.  (Aligning
// the area at run time, 128 bytes more per CTA, measured 5-8 % slower.)
template <int NTH>
__global__ void __launch_bounds__(NTH)
conv3x3_cb8(const uint4* __restrict__ inA, int chA, int mode_a, const uint4* __restrict__ inB,
            int chB, int cin, const __nv_bfloat16* __restrict__ w, const float* __restrict__ bias,
            void* __restrict__ out, uint4* __restrict__ pool, int cout, int out_form, int B,
            int H, int W, int act, int tmem_cols, unsigned* err,
            const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
            int tma_a_req, int tma_b_req) {
  extern __shared__ __align__(1024) unsigned char tc_sm[];
  const int cinp = pad16(cin), coutp = pad16(cout);
  const int nch = cinp / 8;
  unsigned char* sA = tc_sm;   // staged chunks
  unsigned char* sB = sA + (size_t)nch * CB_CHUNK_STRIDE;
  const bool tma_aligned = (smem_u32(tc_sm) & 127u) == 0u;
  const int tma_a = tma_a_req && tma_aligned, tma_b = tma_b_req && tma_aligned;
  unsigned long long* mbar = (unsigned long long*)(sB + (size_t)9 * cinp * coutp * 2);
  uint32_t* tmem_slot = (uint32_t*)(mbar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // the padding chunks past A and B read as zeros; nothing writes them again
  for (int e = tid; e < (nch - chA - chB) * (CB_CHUNK_STRIDE / 16); e += NTH)
    ((uint4*)(sA + (size_t)(chA + chB) * CB_CHUNK_STRIDE))[e] = make_uint4(0u, 0u, 0u, 0u);

  // weights: [tap][chunk][n][8] bf16, zero outside (cout, cin)
  for (int e = tid; e < 9 * nch * coutp; e += NTH) {
    const int n = e % coutp;
    const int rest = e / coutp;
    const int ch = rest % nch, tap = rest / nch;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ci = ch * 8 + k;
      v[k] = (n < cout && ci < cin) ? w[((size_t)n * cin + ci) * 9 + tap] : __float2bfloat16(0.0f);
    }
    *(uint4*)(sB + ((size_t)(tap * nch + ch) * coutp + n) * 16) = *(const uint4*)v;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar + 1)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t mbar_a = smem_u32(mbar);
  const uint32_t mbar_t = smem_u32(mbar + 1);   // the TMA copies of a region
  const uint32_t sA_a = smem_u32(sA), sB_a = smem_u32(sB);
  const uint32_t idesc = tc_idesc(coutp);
  const size_t npix = (size_t)B * H * W;
  const int H2 = H >> 1, W2 = W >> 1;
  const int rx = (W + CBX - 1) / CBX, ry = (H + CBY - 1) / CBY;
  const int nreg = rx * ry * B;
  const int ntma = (tma_a ? chA : 0) + (tma_b ? chB : 0);
  uint32_t parity = 0, tparity = 0;
  bool failed = false;
  // issue the staging of region t: the box-shaped chunks by TMA (the box
  // starts one pixel up and left of the region; the innermost coordinate, the
  // channel, is always 0), the rest by 16-byte cp.async copies (zero outside
  // the image), as one cp.async group
  auto issue_stage = [&](int t) {
    const int b = t / (rx * ry);
    const int rr = t - b * rx * ry;
    const int x0 = (rr % rx) * CBX, y0 = (rr / rx) * CBY;
    if (tid == 0 && ntma > 0) {
      mbar_expect_tx(mbar_t, (uint32_t)ntma * CB_CHUNK_BYTES);
      if (tma_a)
        for (int ch = 0; ch < chA; ++ch)
          tma_load_4d(sA_a + (uint32_t)ch * CB_CHUNK_STRIDE, &tm_a, 0, x0 - 1, y0 - 1,
                      ch * B + b, mbar_t);
      if (tma_b)
        for (int ch = 0; ch < chB; ++ch)
          tma_load_4d(sA_a + (uint32_t)(chA + ch) * CB_CHUNK_STRIDE, &tm_b, 0, x0 - 1, y0 - 1,
                      ch * B + b, mbar_t);
    }
    // the rest: one 16-byte cp.async copy per (chunk, halo pixel), zero
    // outside the image
    const int cp_lo = tma_a ? chA : 0, cp_hi = chA + (tma_b ? 0 : chB);
    for (int e = cp_lo * CHP + tid; e < cp_hi * CHP; e += NTH) {
      const int ch = e / CHP, q = e - ch * CHP;
      const int yy = y0 - 1 + q / CHX, xx = x0 - 1 + q % CHX;
      const bool inside = yy >= 0 && yy < H && xx >= 0 && xx < W;
      const uint4* src = inA;
      uint32_t bytes = 0;
      if (inside && ch < chA) {
        src = mode_a == SRC_UP
                  ? inA + ((size_t)ch * B + b) * H2 * W2 + (size_t)(yy >> 1) * W2 + (xx >> 1)
                  : inA + ((size_t)ch * B + b) * H * W + (size_t)yy * W + xx;
        bytes = 16;
      } else if (inside && ch < chA + chB) {
        src = inB + ((size_t)(ch - chA) * B + b) * H * W + (size_t)yy * W + xx;
        bytes = 16;
      }
      cp_async16(sA_a + (uint32_t)ch * CB_CHUNK_STRIDE + (uint32_t)q * 16, src, bytes);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // with TMA copies the next region's staging is issued as soon as this
  // region's MMAs have read the chunks, so it lands during the epilogue;
  // layers staged by cp.async alone (a fallback) stage at the top of each
  // region.  Measured, one 1024^2 application against the cp.async staging
  // at the top of each region: (24, 48) 0.443 -> 0.423 ms, (8, 16) 0.248 ->
  // 0.244 ms.
  const bool early = ntma > 0;
  if (early && (int)blockIdx.x < nreg) issue_stage(blockIdx.x);
  for (int t = blockIdx.x; t < nreg; t += gridDim.x) {
    const int b = t / (rx * ry);
    const int rr = t - b * rx * ry;
    const int x0 = (rr % rx) * CBX, y0 = (rr / rx) * CBY;
    const size_t img = (size_t)b * H * W;
    if (!early) issue_stage(t);
    // region t's copies
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (ntma > 0) {
      bool landed = false;
      for (unsigned it = 0; it < TC_SPIN_LIMIT; ++it)
        if (mbar_try_wait(mbar_t, tparity)) { landed = true; break; }
      tparity ^= 1u;
      if (__syncthreads_or(landed ? 0 : 1)) {
        failed = true;
        if (err && tid == 0) atomicExch(err, 1u);
        break;
      }
    }
    // make the cp.async copies visible to the tensor core's async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      // M tile i: pixels x0 + 8 i .. x0 + 8 i + 7 of the region's 16 rows,
      // accumulator columns [i coutp, (i + 1) coutp)
      for (int i = 0; i < 2; ++i) {
        uint32_t acc = 0;
        for (int tap = 0; tap < 9; ++tap) {
          const int dy = tap / 3, dx = tap % 3;
          for (int g = 0; g < cinp / 16; ++g) {
            const uint32_t a = sA_a + (uint32_t)(2 * g) * CB_CHUNK_STRIDE +
                               (uint32_t)(dy * CHX + dx + 8 * i) * 16;
            const uint32_t bb = sB_a + (uint32_t)((tap * nch + 2 * g) * coutp) * 16;
            tc_mma(tmem + (uint32_t)(i * coutp), tc_desc(a, CB_CHUNK_STRIDE, CHX * 16),
                   tc_desc(bb, coutp * 16, 128), idesc, acc);
            acc = 1;
          }
        }
      }
      tc_commit(mbar_a);
    }
    bool done = false;
    for (unsigned it = 0; it < TC_SPIN_LIMIT; ++it) {
      if (mbar_try_wait(mbar_a, parity)) { done = true; break; }
    }
    parity ^= 1u;
    if (__syncthreads_or(done ? 0 : 1)) {
      failed = true;
      if (err && tid == 0) atomicExch(err, 1u);
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // the MMAs have read the staged chunks: the next region's copies land
    // while this region's epilogue runs
    if (early && t + (int)gridDim.x < nreg) issue_stage(t + gridDim.x);
    // epilogue: warp w owns accumulator rows 32 (w % 4) .. 32 (w % 4) + 31 of
    // M tile w / 4 (NTH = 256), or of both tiles (NTH = 128)
    const int m = (warp & 3) * 32 + lane;
    for (int i = (NTH == 256 ? warp >> 2 : 0); i < (NTH == 256 ? (warp >> 2) + 1 : 2); ++i) {
      const int x = x0 + 8 * i + (m % 8), y = y0 + m / 8;
      const bool store = x < W && y < H;
      // the 2x2 block's top-left lane (even x, even y) writes the pooled pixel
      const bool pstore = store && ((m & 1) == 0) && (((m >> 3) & 1) == 0);
      for (int c0 = 0; c0 < coutp; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(i * coutp + c0), v);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int co = c0 + k;
          if (co < cout) {   // padding columns are never stored
            float s = v[k] + (bias ? bias[co] : 0.0f);
            if (act) s = tanh_sfu(s);   // the inference kernel: tanh on the SFU
            v[k] = s;
          }
        }
        if (out_form == CB_OUT_F32) {
#pragma unroll
          for (int k = 0; k < 16; ++k)
            if (store && c0 + k < cout)
              ((float*)out)[(size_t)(c0 + k) * npix + img + (size_t)y * W + x] = v[k];
          continue;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int chunk = c0 / 8 + h;
          if (chunk * 8 >= cout) continue;   // uniform
          __align__(16) __nv_bfloat16 o[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) o[k] = __float2bfloat16_rn(v[8 * h + k]);
          if (store)
            ((uint4*)out)[((size_t)chunk * B + b) * H * W + (size_t)y * W + x] = *(const uint4*)o;
          if (pool) {
            __align__(16) __nv_bfloat16 pv[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const float a0 = v[8 * h + k];
              const float a1 = __shfl_down_sync(0xffffffffu, a0, 1);
              const float a2 = __shfl_down_sync(0xffffffffu, a0, 8);
              const float a3 = __shfl_down_sync(0xffffffffu, a0, 9);
              pv[k] = __float2bfloat16_rn(0.25f * (((a0 + a1) + a2) + a3));
            }
            if (pstore)
              pool[((size_t)chunk * B + b) * H2 * W2 + (size_t)(y >> 1) * W2 + (x >> 1)] =
                  *(const uint4*)pv;
          }
        }
      }
    }
    // TMEM reads and shared-memory reads of this region complete before the next
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (failed) {
    // give copies and MMAs still in flight a bounded chance to land before
    // the shared memory and the TMEM columns are released (a phase that
    // already completed returns at once)
    if (ntma > 0)
      for (unsigned it = 0; it < TC_SPIN_LIMIT; ++it)
        if (mbar_try_wait(mbar_t, tparity ^ 1u)) break;
    for (unsigned it = 0; it < TC_SPIN_LIMIT; ++it)
      if (mbar_try_wait(mbar_a, parity ^ 1u)) break;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols)
                 : "memory");
  }
}

}  // namespace unet
}  // namespace zb
