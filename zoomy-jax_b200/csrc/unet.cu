// Learned multigrid smoother: a small convolutional U-Net with bf16 weights
// and float32 accumulation, its training kernels (forward, backward, Adam) and
// its use as the level-0 smoother of the pressure V-cycle.
//
// The reference's learned V-cycle (zoomy_jax/gnn_blueprint/
// vcycle_structured_gnn.py:74-122, 145-200; graph_mp_multibranch.py:9-16;
// trained by train_vcycle_structured_poisson.py:168-306) smooths each level
// with tanh message-passing layers over the residual.  On a Cartesian grid the
// same local learned operator is a convolution; here it is a two-level U-Net:
//
//   in  = [r / s, c / cmax]                  (2 channels; s = RMS of r)
//   e1  = tanh(conv3x3(in,  2  -> C1))        level 0
//   e2  = tanh(conv3x3(e1,  C1 -> C1))
//   m1  = tanh(conv3x3(pool2(e2), C1 -> C2))  level 1 (2x2 average pool)
//   m2  = tanh(conv3x3(m1,  C2 -> C2))
//   o1  = tanh(conv3x3([up2(m2), e2], C2+C1 -> C1))   (nearest upsample)
//   out = conv3x3(o1, C1 -> 1)
//   correction = s * dx^2 / c * out           (1-homogeneous in r)
//
// with c the cell mean of the four face coefficients.  Activations are
// channel planes [C][B][H][W] in float32; weights [Cout][Cin][3][3] in bf16
// (the training keeps a float32 master copy and rounds it to bf16 for every
// forward, so the gradients are those of the bf16 network).  Convolutions are
// direct: a 16x16 pixel tile with a 1-pixel halo per 8-channel input chunk in
// shared memory, one thread per output pixel with all output channels in
// registers.  Zero padding at image borders.
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "conv_tc.cuh"

namespace zb {
namespace unet {

constexpr int TS = 16;          // pixel tile side
constexpr int NTT = TS * TS;    // threads per conv CTA
constexpr int CCH = 8;          // input channels per shared-memory chunk
constexpr int NT = 256;

enum { ACT_NONE = 0, ACT_TANH = 1, ACT_TANH_SFU = 2 };   // see conv_tc.cuh


// out[co][b][y][x] = act(bias[co] + sum_ci sum_tap w[co][ci][tap] in[ci][b][y+dy][x+dx])
// input channels may come from two planes sets (the concatenation): channels
// [0, cin_a) from inA, [cin_a, cin) from inB
template <int COUT>
__global__ void __launch_bounds__(NTT)
conv3x3_fwd(const float* __restrict__ inA, int cin_a, const float* __restrict__ inB, int cin,
            const __nv_bfloat16* __restrict__ w, const float* __restrict__ bias,
            float* __restrict__ out, int B, int H, int W, int act, int mode_a) {
  __shared__ float sin_[CCH][TS + 2][TS + 2];
  __shared__ float sw[COUT][CCH][9];
  const int tx = threadIdx.x % TS, ty = threadIdx.x / TS;
  const int x0 = blockIdx.x * TS, y0 = blockIdx.y * TS, b = blockIdx.z;
  const int x = x0 + tx, y = y0 + ty;
  const size_t plane = (size_t)B * H * W;
  const size_t img = (size_t)b * H * W;
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) acc[co] = bias ? bias[co] : 0.0f;
  for (int c0 = 0; c0 < cin; c0 += CCH) {
    const int nc = min(CCH, cin - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < CCH * (TS + 2) * (TS + 2); e += NTT) {
      const int cc = e / ((TS + 2) * (TS + 2));
      const int rr = e - cc * (TS + 2) * (TS + 2);
      const int yy = y0 - 1 + rr / (TS + 2), xx = x0 - 1 + rr % (TS + 2);
      float v = 0.0f;
      if (cc < nc && yy >= 0 && yy < H && xx >= 0 && xx < W)
        v = src_at(inA, cin_a, inB, mode_a, c0 + cc, b, B, H, W, yy, xx);
      sin_[cc][rr / (TS + 2)][rr % (TS + 2)] = v;
    }
    for (int e = threadIdx.x; e < COUT * CCH * 9; e += NTT) {
      const int co = e / (CCH * 9), rem = e - co * CCH * 9;
      const int cc = rem / 9, tap = rem - cc * 9;
      sw[co][cc][tap] = cc < nc ? __bfloat162float(w[((size_t)co * cin + c0 + cc) * 9 + tap]) : 0.0f;
    }
    __syncthreads();
    for (int cc = 0; cc < nc; ++cc) {
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const float v = sin_[cc][ty + tap / 3][tx + tap % 3];
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] = fmaf(sw[co][cc][tap], v, acc[co]);
      }
    }
  }
  if (x < W && y < H) {
#pragma unroll
    for (int co = 0; co < COUT; ++co) {
      const float v = act != ACT_NONE ? tanhf(acc[co]) : acc[co];   // exact reference
      out[(size_t)co * plane + img + (size_t)y * W + x] = v;
    }
  }
}

// dW[co][ci][tap] += sum_p dout[co](p) in[ci](p + tap); dbias[co] += sum_p dout
// one CTA per (16x16 tile, image); each thread owns weight entries and walks
// the tile's pixels from shared memory
__global__ void __launch_bounds__(NTT)
conv3x3_wgrad(const float* __restrict__ inA, int cin_a, const float* __restrict__ inB, int cin,
              const float* __restrict__ dout, int cout, float* __restrict__ dw,
              float* __restrict__ dbias, int B, int H, int W, int mode_a) {
  __shared__ float sin_[CCH][TS + 2][TS + 2];
  __shared__ float sd[8][TS * TS];
  const int x0 = blockIdx.x * TS, y0 = blockIdx.y * TS, b = blockIdx.z;
  const size_t plane = (size_t)B * H * W;
  const size_t img = (size_t)b * H * W;
  for (int co0 = 0; co0 < cout; co0 += 8) {
    const int nco = min(8, cout - co0);
    __syncthreads();
    for (int e = threadIdx.x; e < 8 * TS * TS; e += NTT) {
      const int c = e / (TS * TS), pp = e - c * TS * TS;
      const int yy = y0 + pp / TS, xx = x0 + pp % TS;
      sd[c][pp] = (c < nco && yy < H && xx < W)
                      ? dout[(size_t)(co0 + c) * plane + img + (size_t)yy * W + xx] : 0.0f;
    }
    __syncthreads();
    if (dbias != nullptr && threadIdx.x < nco) {
      float s = 0.0f;
      for (int pp = 0; pp < TS * TS; ++pp) s += sd[threadIdx.x][pp];
      atomicAdd(&dbias[co0 + threadIdx.x], s);
    }
    for (int c0 = 0; c0 < cin; c0 += CCH) {
      const int nc = min(CCH, cin - c0);
      __syncthreads();
      for (int e = threadIdx.x; e < CCH * (TS + 2) * (TS + 2); e += NTT) {
        const int cc = e / ((TS + 2) * (TS + 2));
        const int rr = e - cc * (TS + 2) * (TS + 2);
        const int yy = y0 - 1 + rr / (TS + 2), xx = x0 - 1 + rr % (TS + 2);
        float v = 0.0f;
        if (cc < nc && yy >= 0 && yy < H && xx >= 0 && xx < W)
          v = src_at(inA, cin_a, inB, mode_a, c0 + cc, b, B, H, W, yy, xx);
        sin_[cc][rr / (TS + 2)][rr % (TS + 2)] = v;
      }
      __syncthreads();
      // entries: nco x nc x 9 <= 8 * 8 * 9 = 576 over 256 threads
      for (int e = threadIdx.x; e < nco * nc * 9; e += NTT) {
        const int c = e / (nc * 9), rem = e - c * nc * 9;
        const int cc = rem / 9, tap = rem - cc * 9;
        const int dy = tap / 3, dx = tap % 3;
        float s = 0.0f;
        for (int pp = 0; pp < TS * TS; ++pp) s += sd[c][pp] * sin_[cc][pp / TS + dy][pp % TS + dx];
        atomicAdd(&dw[((size_t)(co0 + c) * cin + c0 + cc) * 9 + tap], s);
      }
    }
  }
}

// transposed, flipped weights for the data gradient: wt[ci][co][8 - tap]
__global__ void flip_weights(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wt,
                             int cout, int cin) {
  for (int e = blockIdx.x * NT + threadIdx.x; e < cout * cin * 9; e += gridDim.x * NT) {
    const int co = e / (cin * 9), rem = e - co * cin * 9;
    const int ci = rem / 9, tap = rem - ci * 9;
    wt[((size_t)ci * cout + co) * 9 + (8 - tap)] = w[e];
  }
}

// g *= (1 - y^2) (tanh derivative), in place on the gradient
__global__ void tanh_back(float* __restrict__ g, const float* __restrict__ y, size_t n) {
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT)
    g[k] *= 1.0f - y[k] * y[k];
}

__global__ void avgpool2_back(const float* __restrict__ gout, float* __restrict__ gin, int C,
                              int B, int H, int W) {
  const int Wo = W / 2, Ho = H / 2;
  const size_t n = (size_t)C * B * H * W;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT) {
    const int xx = (int)(k % W);
    const size_t t = k / W;
    const int yy = (int)(t % H);
    const size_t cb = t / H;
    gin[k] = 0.25f * gout[cb * (size_t)Ho * Wo + (size_t)(yy / 2) * Wo + xx / 2];
  }
}

__global__ void upsample2_back(const float* __restrict__ gout, float* __restrict__ gin, int C,
                               int B, int H, int W) {
  const int Ho = H / 2, Wo = W / 2;
  const size_t n = (size_t)C * B * Ho * Wo;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT) {
    const int xo = (int)(k % Wo);
    const size_t t = k / Wo;
    const int yo = (int)(t % Ho);
    const size_t cb = t / Ho;
    const float* src = gout + cb * (size_t)H * W;
    gin[k] = src[(size_t)(2 * yo) * W + 2 * xo] + src[(size_t)(2 * yo) * W + 2 * xo + 1] +
             src[(size_t)(2 * yo + 1) * W + 2 * xo] + src[(size_t)(2 * yo + 1) * W + 2 * xo + 1];
  }
}

__global__ void add_inplace(float* __restrict__ a, const float* __restrict__ b, size_t n) {
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT)
    a[k] += b[k];
}

__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, __nv_bfloat16* __restrict__ wb, int n,
                            float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int k = blockIdx.x * NT + threadIdx.x; k < n; k += gridDim.x * NT) {
    const float g0 = g[k];
    const float gk = isfinite(g0) ? g0 : 0.0f;   // a non-finite entry is skipped
    const float mk = b1 * m[k] + (1.0f - b1) * gk;
    const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float wk = w[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    w[k] = wk;
    wb[k] = __float2bfloat16(wk);
  }
}

}  // namespace unet
}  // namespace zb

// ── features, scaling, patch operator, loss ─────────────────────────────────
namespace zb {
namespace unet {

// per image b: s[b] = sqrt(mean r^2) (tiny floor so a zero residual stays
// zero), as a two-stage deterministic reduction: P partial sums per image
// (grid (P, B)), then one warp per image adds them in a fixed order
constexpr int RMS_PARTS = 1024;   // partial-sum slots in the workspace

__global__ void rms_part_kernel(const float* __restrict__ r, size_t npix, int P,
                                float* __restrict__ part) {
  __shared__ float red[NT / 32];
  const int b = blockIdx.y, p = blockIdx.x;
  float acc = 0.0f;
  for (size_t k = (size_t)p * NT + threadIdx.x; k < npix; k += (size_t)P * NT) {
    const float v = r[(size_t)b * npix + k];
    acc += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int i = 0; i < NT / 32; ++i) t += red[i];
    part[b * P + p] = t;
  }
}

__global__ void rms_final_kernel(const float* __restrict__ part, int P, size_t npix,
                                 float* __restrict__ s) {
  const int b = blockIdx.x;
  float t = 0.0f;
  for (int p = threadIdx.x; p < P; p += 32) t += part[b * P + p];
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (threadIdx.x == 0) s[b] = fmaxf(sqrtf(t / (float)npix), 1e-30f);
}

static void rms(const float* r, int B, size_t npix, float* part, float* s, cudaStream_t st) {
  int P = (int)std::min<size_t>(256, std::max<size_t>(1, npix / (NT * 16)));
  P = std::max(1, std::min(P, RMS_PARTS / std::max(1, B)));
  rms_part_kernel<<<dim3(P, B), NT, 0, st>>>(r, npix, P, part);
  rms_final_kernel<<<B, 32, 0, st>>>(part, P, npix, s);
}

// cell coefficient of image b's cell (i, j) from its faces: cx (B, H+1, W),
// cy (B, H, W+1)
__device__ __forceinline__ float cell_c(const float* cx, const float* cy, int b, int H, int W,
                                        int i, int j) {
  const float* ax = cx + (size_t)b * (H + 1) * W;
  const float* ay = cy + (size_t)b * H * (W + 1);
  return 0.25f * (ax[(size_t)i * W + j] + ax[(size_t)(i + 1) * W + j] +
                  ay[(size_t)i * (W + 1) + j] + ay[(size_t)i * (W + 1) + j + 1]);
}

__global__ void features_kernel(const float* __restrict__ r, const float* __restrict__ s,
                                const float* __restrict__ cx, const float* __restrict__ cy,
                                int B, int H, int W, float inv_cmax, float* __restrict__ in) {
  const size_t npix = (size_t)H * W, n = (size_t)B * npix;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT) {
    const int b = (int)(k / npix);
    const size_t p = k - (size_t)b * npix;
    const int i = (int)(p / W), j = (int)(p - (size_t)i * W);
    in[k] = r[k] / s[b];
    in[n + k] = cell_c(cx, cy, b, H, W, i, j) * inv_cmax;
  }
}

// the same two input channels as one chunk of the chunked bf16 layout
// (channels 2..7 zero), each rounded as the planar kernel rounds them
__global__ void features_cb8_kernel(const float* __restrict__ r, const float* __restrict__ s,
                                    const float* __restrict__ cx, const float* __restrict__ cy,
                                    int B, int H, int W, float inv_cmax, uint4* __restrict__ in) {
  const size_t npix = (size_t)H * W, n = (size_t)B * npix;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT) {
    const int b = (int)(k / npix);
    const size_t p = k - (size_t)b * npix;
    const int i = (int)(p / W), j = (int)(p - (size_t)i * W);
    __align__(16) __nv_bfloat16 v[8];
    v[0] = __float2bfloat16_rn(r[k] / s[b]);
    v[1] = __float2bfloat16_rn(cell_c(cx, cy, b, H, W, i, j) * inv_cmax);
#pragma unroll
    for (int c = 2; c < 8; ++c) v[c] = __float2bfloat16_rn(0.0f);
    in[k] = *(const uint4*)v;
  }
}

// y = x_in + s dx^2 / c * out   (x_in may be null; y may alias x_in)
__global__ void scale_out_kernel(const float* __restrict__ out, const float* __restrict__ s,
                                 const float* __restrict__ cx, const float* __restrict__ cy,
                                 int B, int H, int W, float dx2, const float* x_in, float* y) {
  const size_t npix = (size_t)H * W, n = (size_t)B * npix;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT) {
    const int b = (int)(k / npix);
    const size_t p = k - (size_t)b * npix;
    const int i = (int)(p / W), j = (int)(p - (size_t)i * W);
    const float v = s[b] * dx2 / cell_c(cx, cy, b, H, W, i, j) * out[k];
    y[k] = x_in ? x_in[k] + v : v;
  }
}

__device__ __forceinline__ float xg(const float* x, int H, int W, int i, int j, float self) {
  return (i < 0 || i >= H || j < 0 || j >= W) ? -self : x[(size_t)i * W + j];
}

// res = f - A x per image (Dirichlet ghost -x), with x null meaning zero
__global__ void patch_residual(const float* __restrict__ f, const float* __restrict__ x,
                               const float* __restrict__ cx, const float* __restrict__ cy,
                               int B, int H, int W, float idx2, float* __restrict__ res) {
  const size_t npix = (size_t)H * W, n = (size_t)B * npix;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT) {
    const int b = (int)(k / npix);
    const size_t p = k - (size_t)b * npix;
    const int i = (int)(p / W), j = (int)(p - (size_t)i * W);
    float ax = 0.0f;
    if (x) {
      const float* xb = x + (size_t)b * npix;
      const float* ax_ = cx + (size_t)b * (H + 1) * W;
      const float* ay_ = cy + (size_t)b * H * (W + 1);
      const float xc = xb[p];
      ax = (ax_[(size_t)(i + 1) * W + j] * (xc - xg(xb, H, W, i + 1, j, xc)) +
            ax_[(size_t)i * W + j] * (xc - xg(xb, H, W, i - 1, j, xc)) +
            ay_[(size_t)i * (W + 1) + j + 1] * (xc - xg(xb, H, W, i, j + 1, xc)) +
            ay_[(size_t)i * (W + 1) + j] * (xc - xg(xb, H, W, i, j - 1, xc))) * idx2;
    }
    res[k] = f[k] - ax;
  }
}

// loss terms per image: lnum[b] = a_b . b_b, lden[b] = c_b . d_b (residual
// loss: a = b = res, c = d = r; energy loss: a = res, b = A res, c = e,
// d = A e).  An image whose denominator is not a positive finite number above
// 1e-30 (a patch without signal) is left out of the loss and its gradient.
__global__ void loss_kernel(const float* __restrict__ a_, const float* __restrict__ b_,
                            const float* __restrict__ c_, const float* __restrict__ d_, int B,
                            size_t npix, float* __restrict__ lnum, float* __restrict__ lden) {
  __shared__ float red[2][NT / 32];
  const int b = blockIdx.x;
  float a = 0.0f, c = 0.0f;
  for (size_t k = threadIdx.x; k < npix; k += NT) {
    const size_t q = (size_t)b * npix + k;
    a += a_[q] * b_[q];
    c += c_[q] * d_[q];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = a; red[1][threadIdx.x >> 5] = c; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float ta = 0.0f, tc = 0.0f;
    for (int i = 0; i < NT / 32; ++i) { ta += red[0][i]; tc += red[1][i]; }
    lnum[b] = ta;
    lden[b] = tc;
  }
}

__device__ __forceinline__ bool loss_counts(float den) { return den > 1e-30f && den < 3e38f; }

__global__ void loss_total(const float* lnum, const float* lden, int B, double* out) {
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int b = 0; b < B; ++b)
      if (loss_counts(lden[b])) t += (double)lnum[b] / (double)lden[b];
    *out = t / B;
  }
}

// A x per image (Dirichlet ghost -x)
__global__ void patch_apply(const float* __restrict__ x, const float* __restrict__ cx,
                            const float* __restrict__ cy, int B, int H, int W, float idx2,
                            float* __restrict__ out) {
  const size_t npix = (size_t)H * W, n = (size_t)B * npix;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT) {
    const int b = (int)(k / npix);
    const size_t p = k - (size_t)b * npix;
    const int i = (int)(p / W), j = (int)(p - (size_t)i * W);
    const float* xb = x + (size_t)b * npix;
    const float* ax_ = cx + (size_t)b * (H + 1) * W;
    const float* ay_ = cy + (size_t)b * H * (W + 1);
    const float xc = xb[p];
    out[k] = (ax_[(size_t)(i + 1) * W + j] * (xc - xg(xb, H, W, i + 1, j, xc)) +
              ax_[(size_t)i * W + j] * (xc - xg(xb, H, W, i - 1, j, xc)) +
              ay_[(size_t)i * (W + 1) + j + 1] * (xc - xg(xb, H, W, i, j + 1, xc)) +
              ay_[(size_t)i * (W + 1) + j] * (xc - xg(xb, H, W, i, j - 1, xc))) * idx2;
  }
}

__global__ void sub_kernel(const float* __restrict__ a, const float* __restrict__ b, size_t n,
                           float* __restrict__ out) {
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT)
    out[k] = a[k] - b[k];
}

// dL/dout = -2 (A res)_b / (B den_b) * s_b dx^2 / c   (A symmetric); ar holds
// A res (energy loss) or is null, in which case A res is formed here from res
__global__ void loss_grad_kernel(const float* __restrict__ res, const float* __restrict__ ar_in,
                                 const float* __restrict__ cx, const float* __restrict__ cy,
                                 const float* __restrict__ lden, const float* __restrict__ s,
                                 int B, int H, int W, float idx2, float dx2,
                                 float* __restrict__ dout) {
  const size_t npix = (size_t)H * W, n = (size_t)B * npix;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < n; k += (size_t)gridDim.x * NT) {
    const int b = (int)(k / npix);
    const size_t p = k - (size_t)b * npix;
    const int i = (int)(p / W), j = (int)(p - (size_t)i * W);
    float ar;
    if (ar_in) {
      ar = ar_in[k];
    } else {
      const float* rb = res + (size_t)b * npix;
      const float* ax_ = cx + (size_t)b * (H + 1) * W;
      const float* ay_ = cy + (size_t)b * H * (W + 1);
      const float rc = rb[p];
      ar = (ax_[(size_t)(i + 1) * W + j] * (rc - xg(rb, H, W, i + 1, j, rc)) +
            ax_[(size_t)i * W + j] * (rc - xg(rb, H, W, i - 1, j, rc)) +
            ay_[(size_t)i * (W + 1) + j + 1] * (rc - xg(rb, H, W, i, j + 1, rc)) +
            ay_[(size_t)i * (W + 1) + j] * (rc - xg(rb, H, W, i, j - 1, rc))) * idx2;
    }
    const float den = lden[b];
    const float c = cell_c(cx, cy, b, H, W, i, j);
    dout[k] = loss_counts(den) ? -2.0f * ar / ((float)B * den) * s[b] * dx2 / c : 0.0f;
  }
}

// ── network plumbing ────────────────────────────────────────────────────────
struct Net {
  int c1, c2;
  size_t off_w[6], off_b[6];
  int cin[6], cout[6];
  size_t nw, nb;
};

static Net net_layout(int c1, int c2) {
  Net n;
  const int ci[6] = {2, c1, c1, c2, c1 + c2, c1};
  const int co[6] = {c1, c1, c2, c2, c1, 1};
  size_t w = 0, b = 0;
  for (int l = 0; l < 6; ++l) {
    n.cin[l] = ci[l];
    n.cout[l] = co[l];
    n.off_w[l] = w;
    n.off_b[l] = b;
    w += (size_t)co[l] * ci[l] * 9;
    b += (size_t)co[l];
  }
  n.c1 = c1;
  n.c2 = c2;
  n.nw = w;
  n.nb = b;
  return n;
}

// channel pairs with an instantiated convolution for every layer and for the
// data gradient of the concatenation layer (c1 + c2 output channels)
static bool valid_channels(int c1, int c2) {
  return (c1 == 8 && c2 == 16) || (c1 == 16 && c2 == 16) || (c1 == 16 && c2 == 32) ||
         (c1 == 24 && c2 == 48);
}

// which convolution runs the forward and data-gradient passes: 0 = the
// CUDA-core direct convolution (float32 operands, kept as the exactness
// reference); 1 (default) = the tcgen05 implicit GEMM (bf16 operands), the
// smoother application's forward through the chunked bf16 layout
// (conv3x3_cb8) and training through the float32 planar staging
// (conv3x3_tc); 2 = the tcgen05 GEMM with the planar staging everywhere (the
// same bits as 1)
static int g_conv_impl = 1;
static __device__ unsigned g_unet_err;

static unsigned* unet_err_word() {
  static std::atomic<unsigned*> ptrs[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!ptrs[dev].load()) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_unet_err) != cudaSuccess) return nullptr;
    ptrs[dev].store((unsigned*)p);
  }
  return ptrs[dev].load();
}

static int conv_tc_launch(const float* inA, int cin_a, const float* inB, int cin,
                          const __nv_bfloat16* w, const float* bias, float* out, int cout, int B,
                          int H, int W, int act, int mode_a, cudaStream_t st) {
  const int cinp = pad16(cin), coutp = pad16(cout);
  if (coutp > 256 || cinp > 256) return ZB_E_UNSUPPORTED;
  int cols = 32;
  while (cols < coutp) cols *= 2;
  static std::atomic<int> sms[64];
  static std::atomic<bool> attr[64];
  int dev = 0;
  ZB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return ZB_E_CUDA;
  if (!sms[dev].load()) {
    int v = 0;
    ZB_CUDA_TRY(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    sms[dev].store(v);
  }
  if (!attr[dev].load()) {
    ZB_CUDA_TRY(cudaFuncSetAttribute(conv3x3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     227 * 1024));
    attr[dev].store(true);
  }
  // resident CTAs of one SM must never ask for more than its 512 TMEM
  // columns: pad the shared memory so that at most 512 / cols fit
  const int smem_sm = 228 * 1024, per_cta_reserved = 1024;
  const int by_tmem = 512 / cols, by_threads = 2048 / TC_THREADS;
  size_t smem = tc_smem_bytes(cinp, coutp);
  if (by_tmem < by_threads) {
    const size_t floor_bytes = (size_t)(smem_sm / (by_tmem + 1) - per_cta_reserved + 16);
    smem = std::max(smem, floor_bytes);
  }
  if (smem > 227 * 1024) return ZB_E_UNSUPPORTED;
  const int fit = std::min(by_threads, (int)(smem_sm / (smem + per_cta_reserved)));
  const long long ntiles =
      (long long)((W + TCX - 1) / TCX) * ((H + TCY - 1) / TCY) * B;
  const int grid = (int)std::max<long long>(1, std::min<long long>(ntiles, (long long)sms[dev] * std::max(1, fit)));
  conv3x3_tc<<<grid, TC_THREADS, smem, st>>>(inA, cin_a, inB, cin, w, bias, out, cout, B, H, W,
                                             act, mode_a, cols, unet_err_word());
  return zb_launch_check();
}

// cuTensorMapEncodeTiled from the driver, fetched once through the runtime
// (no link against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static std::atomic<void*> fn{nullptr};
  void* f = fn.load();
  if (!f) {
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f)
      return nullptr;
    fn.store(f);
  }
  return (PFN_cuTensorMapEncodeTiled_v12000)f;
}

// The halo-box map of a chunked activation: dimensions (8 channels, W, H,
// chunks x B) with byte strides (16, 16 W, 16 H W), box (8, 18, 18, 1); pixels
// outside the image read as zeros.  The base is 16-byte aligned and every
// stride a multiple of 16, as the encoder requires.
static bool cb8_map(CUtensorMap* m, const uint4* base, int nchunks, int B, int H, int W) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc || !base || ((uintptr_t)base & 15u)) return false;
  const cuuint64_t dims[4] = {8, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)nchunks * B};
  const cuuint64_t strides[3] = {16, (cuuint64_t)W * 16, (cuuint64_t)H * W * 16};
  const cuuint32_t box[4] = {8, (cuuint32_t)CHX, (cuuint32_t)CHY, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)base, dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// conv3x3_cb8 over B images H x W (see conv_tc.cuh); resident CTAs are capped
// so that their TMEM columns (two M tiles of coutp each) fit in 512
static int conv_cb8_launch(const uint4* inA, int chA, int mode_a, const uint4* inB, int chB,
                           int cin, const __nv_bfloat16* w, const float* bias, void* out,
                           uint4* pool, int cout, int out_form, int B, int H, int W, int act,
                           cudaStream_t st) {
  const int cinp = pad16(cin), coutp = pad16(cout);
  if (2 * coutp > 256 || cinp > 256 || chA + chB > cinp / 8) return ZB_E_UNSUPPORTED;
  int cols = 32;
  while (cols < 2 * coutp) cols *= 2;
  static std::atomic<int> sms[64];
  static std::atomic<bool> attr[64];
  int dev = 0;
  ZB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return ZB_E_CUDA;
  if (!sms[dev].load()) {
    int v = 0;
    ZB_CUDA_TRY(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    sms[dev].store(v);
  }
  if (!attr[dev].load()) {
    ZB_CUDA_TRY(cudaFuncSetAttribute(conv3x3_cb8<128>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    ZB_CUDA_TRY(cudaFuncSetAttribute(conv3x3_cb8<256>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    attr[dev].store(true);
  }
  const int nth = cinp / 8 >= CB_WIDE_CHUNKS ? 256 : 128;
  const int smem_sm = 228 * 1024, per_cta_reserved = 1024;
  const int by_tmem = 512 / cols, by_threads = 2048 / nth;
  size_t smem = cb8_smem_bytes(cinp, coutp);
  if (by_tmem < by_threads) {
    const size_t floor_bytes = (size_t)(smem_sm / (by_tmem + 1) - per_cta_reserved + 16);
    smem = std::max(smem, floor_bytes);
  }
  if (smem > 227 * 1024) return ZB_E_UNSUPPORTED;
  const int fit = std::min(by_threads, (int)(smem_sm / (smem + per_cta_reserved)));
  const long long nreg = (long long)((W + CBX - 1) / CBX) * ((H + CBY - 1) / CBY) * B;
  const int grid = (int)std::max<long long>(
      1, std::min<long long>(nreg, (long long)sms[dev] * std::max(1, fit)));
  // tensor maps of the sources read as stored (the upsampled source, and one
  // whose map cannot be encoded, stay on the cp.async copies)
  CUtensorMap tm_a, tm_b;
  std::memset(&tm_a, 0, sizeof(tm_a));
  std::memset(&tm_b, 0, sizeof(tm_b));
  const int tma_a = (mode_a == SRC_DIRECT && chA > 0 && cb8_map(&tm_a, inA, chA, B, H, W)) ? 1 : 0;
  const int tma_b = (chB > 0 && cb8_map(&tm_b, inB, chB, B, H, W)) ? 1 : 0;
  if (nth == 256)
    conv3x3_cb8<256><<<grid, 256, smem, st>>>(inA, chA, mode_a, inB, chB, cin, w, bias, out,
                                              pool, cout, out_form, B, H, W, act, cols,
                                              unet_err_word(), tm_a, tm_b, tma_a, tma_b);
  else
    conv3x3_cb8<128><<<grid, 128, smem, st>>>(inA, chA, mode_a, inB, chB, cin, w, bias, out,
                                              pool, cout, out_form, B, H, W, act, cols,
                                              unet_err_word(), tm_a, tm_b, tma_a, tma_b);
  return zb_launch_check();
}

static int conv(const float* inA, int cin_a, const float* inB, int cin,
                const __nv_bfloat16* w, const float* bias, float* out, int cout, int B, int H,
                int W, int act, cudaStream_t st, int mode_a = SRC_DIRECT) {
  if (g_conv_impl >= 1)
    return conv_tc_launch(inA, cin_a, inB, cin, w, bias, out, cout, B, H, W, act, mode_a, st);
  dim3 grid((W + TS - 1) / TS, (H + TS - 1) / TS, B);
  switch (cout) {
#define ZB_CONV(N) case N: conv3x3_fwd<N><<<grid, NTT, 0, st>>>(inA, cin_a, inB, cin, w, bias, out, B, H, W, act, mode_a); break;
    ZB_CONV(1) ZB_CONV(8) ZB_CONV(16) ZB_CONV(24) ZB_CONV(32) ZB_CONV(48) ZB_CONV(72)
#undef ZB_CONV
    default: return ZB_E_UNSUPPORTED;
  }
  return zb_launch_check();
}

static int wgrad(const float* inA, int cin_a, const float* inB, int cin, const float* dout,
                 int cout, float* dw, float* db, int B, int H, int W, cudaStream_t st,
                 int mode_a = SRC_DIRECT) {
  dim3 grid((W + TS - 1) / TS, (H + TS - 1) / TS, B);
  conv3x3_wgrad<<<grid, NTT, 0, st>>>(inA, cin_a, inB, cin, dout, cout, dw, db, B, H, W, mode_a);
  return zb_launch_check();
}

static int gridn(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + NT - 1) / NT, 148 * 16)); }

// activation buffers (floats) for a batch of B images H x W
struct Acts {
  float *in, *e1, *e2, *m1, *m2, *o1, *out, *s, *part;
  // training: gradients and scratch
  float *d_e1, *d_e2, *d_p, *d_m1, *d_m2, *d_cat, *d_o1, *d_out, *res, *lnum, *lden, *tmp;
  __nv_bfloat16* wflip;
};

static size_t acts_floats(const Net& n, int B, int H, int W, bool train) {
  const size_t N0 = (size_t)B * H * W, N1 = (size_t)B * (H / 2) * (W / 2);
  // in (2), e1, e2 (c1 each), m1, m2 (c2 each, half resolution), o1 (c1), out
  size_t f = 2 * N0 + 2 * (size_t)n.c1 * N0 + 2 * (size_t)n.c2 * N1 + (size_t)n.c1 * N0 + N0 +
             512 + RMS_PARTS;
  if (train)
    f += 2 * (size_t)n.c1 * N0 + (size_t)n.c1 * N1 + 2 * (size_t)n.c2 * N1 +
         (size_t)(n.c1 + n.c2) * N0 + (size_t)n.c1 * N0 + N0 + N0 + 1024 +
         (size_t)n.c1 * N0 + (n.nw + 64);   // tmp + flipped weights (bf16 fits in floats)
  return f;
}

static Acts acts_split(const Net& n, void* base, int B, int H, int W, bool train) {
  const size_t N0 = (size_t)B * H * W, N1 = (size_t)B * (H / 2) * (W / 2);
  float* f = (float*)base;
  Acts a;
  std::memset(&a, 0, sizeof(a));
  a.in = f; f += 2 * N0;
  a.e1 = f; f += (size_t)n.c1 * N0;
  a.e2 = f; f += (size_t)n.c1 * N0;
  a.m1 = f; f += (size_t)n.c2 * N1;
  a.m2 = f; f += (size_t)n.c2 * N1;
  a.o1 = f; f += (size_t)n.c1 * N0;
  a.out = f; f += N0;
  a.s = f; f += 512;   // per-image RMS, batch <= 512
  a.part = f; f += RMS_PARTS;
  if (train) {
    a.d_e1 = f; f += (size_t)n.c1 * N0;
    a.d_e2 = f; f += (size_t)n.c1 * N0;
    a.d_p = f; f += (size_t)n.c1 * N1;
    a.d_m1 = f; f += (size_t)n.c2 * N1;
    a.d_m2 = f; f += (size_t)n.c2 * N1;
    a.d_cat = f; f += (size_t)(n.c1 + n.c2) * N0;
    a.d_o1 = f; f += (size_t)n.c1 * N0;
    a.d_out = f; f += N0;
    a.res = f; f += N0;
    a.lnum = f; f += 512;
    a.lden = f; f += 512;
    a.tmp = f; f += (size_t)n.c1 * N0;
    a.wflip = (__nv_bfloat16*)f;
  }
  return a;
}

// forward of the network from a.in; weights bf16, biases float32
static int forward(const Net& n, const Acts& a, const __nv_bfloat16* w, const float* b, int B, int H,
                   int W, cudaStream_t st, int act = ACT_TANH) {
  const int H1 = H / 2, W1 = W / 2;
  int rc;
  if ((rc = conv(a.in, 2, nullptr, 2, w + n.off_w[0], b + n.off_b[0], a.e1, n.c1, B, H, W, act, st))) return rc;
  if ((rc = conv(a.e1, n.c1, nullptr, n.c1, w + n.off_w[1], b + n.off_b[1], a.e2, n.c1, B, H, W, act, st))) return rc;
  // pool(e2) and up(m2) are read through the convolutions' loaders, never stored
  if ((rc = conv(a.e2, n.c1, nullptr, n.c1, w + n.off_w[2], b + n.off_b[2], a.m1, n.c2, B, H1, W1, act, st, SRC_POOL))) return rc;
  if ((rc = conv(a.m1, n.c2, nullptr, n.c2, w + n.off_w[3], b + n.off_b[3], a.m2, n.c2, B, H1, W1, act, st))) return rc;
  if ((rc = conv(a.m2, n.c2, a.e2, n.c2 + n.c1, w + n.off_w[4], b + n.off_b[4], a.o1, n.c1, B, H, W, act, st, SRC_UP))) return rc;
  if ((rc = conv(a.o1, n.c1, nullptr, n.c1, w + n.off_w[5], b + n.off_b[5], a.out, 1, B, H, W, ACT_NONE, st))) return rc;
  return zb_launch_check();
}

// Inference forward in the chunked bf16 layout (conv3x3_cb8), the same bits as
// forward(): the activations live where the float32 ones would (the chunked
// tensors take fewer bytes); e2's epilogue also writes pool(e2), o1 reads
// up(m2) through its loader.  The network output goes to a.out (float32).
struct ActsCB8 {
  uint4 *in, *e1, *e2, *e2p, *m1, *m2, *o1;
};

static bool acts_cb8(const Net& n, const Acts& a, int B, int H, int W, ActsCB8* c) {
  const size_t N0 = (size_t)B * H * W, N1 = (size_t)B * (H / 2) * (W / 2);
  uint4* p = (uint4*)a.in;
  c->in = p; p += N0;
  c->e1 = p; p += (size_t)(n.c1 / 8) * N0;
  c->e2 = p; p += (size_t)(n.c1 / 8) * N0;
  c->e2p = p; p += (size_t)(n.c1 / 8) * N1;
  c->m1 = p; p += (size_t)(n.c2 / 8) * N1;
  c->m2 = p; p += (size_t)(n.c2 / 8) * N1;
  c->o1 = p; p += (size_t)(n.c1 / 8) * N0;
  return (const void*)p <= (const void*)a.out && (((uintptr_t)a.in) & 15u) == 0;
}

static int forward_cb8(const Net& n, const Acts& a, const ActsCB8& c, const __nv_bfloat16* w,
                       const float* b, int B, int H, int W, cudaStream_t st) {
  const int H1 = H / 2, W1 = W / 2, k1 = n.c1 / 8, k2 = n.c2 / 8;
  int rc;
  if ((rc = conv_cb8_launch(c.in, 1, SRC_DIRECT, nullptr, 0, 2, w + n.off_w[0], b + n.off_b[0],
                            c.e1, nullptr, n.c1, CB_OUT_CHUNKED, B, H, W, ACT_TANH_SFU, st))) return rc;
  if ((rc = conv_cb8_launch(c.e1, k1, SRC_DIRECT, nullptr, 0, n.c1, w + n.off_w[1], b + n.off_b[1],
                            c.e2, c.e2p, n.c1, CB_OUT_CHUNKED, B, H, W, ACT_TANH_SFU, st))) return rc;
  if ((rc = conv_cb8_launch(c.e2p, k1, SRC_DIRECT, nullptr, 0, n.c1, w + n.off_w[2], b + n.off_b[2],
                            c.m1, nullptr, n.c2, CB_OUT_CHUNKED, B, H1, W1, ACT_TANH_SFU, st))) return rc;
  if ((rc = conv_cb8_launch(c.m1, k2, SRC_DIRECT, nullptr, 0, n.c2, w + n.off_w[3], b + n.off_b[3],
                            c.m2, nullptr, n.c2, CB_OUT_CHUNKED, B, H1, W1, ACT_TANH_SFU, st))) return rc;
  if ((rc = conv_cb8_launch(c.m2, k2, SRC_UP, c.e2, k1, n.c2 + n.c1, w + n.off_w[4], b + n.off_b[4],
                            c.o1, nullptr, n.c1, CB_OUT_CHUNKED, B, H, W, ACT_TANH_SFU, st))) return rc;
  if ((rc = conv_cb8_launch(c.o1, k1, SRC_DIRECT, nullptr, 0, n.c1, w + n.off_w[5], b + n.off_b[5],
                            a.out, nullptr, 1, CB_OUT_F32, B, H, W, ACT_NONE, st))) return rc;
  return zb_launch_check();
}

// data gradient through conv layer l: din (cin channels) from dout (cout)
static int data_grad(const Net& n, int l, const __nv_bfloat16* w, __nv_bfloat16* wflip,
                     const float* dout, float* din, int B, int H, int W, cudaStream_t st) {
  const int ci = n.cin[l], co = n.cout[l];
  flip_weights<<<gridn((size_t)ci * co * 9), NT, 0, st>>>(w + n.off_w[l], wflip, co, ci);
  return conv(dout, co, nullptr, co, wflip, nullptr, din, ci, B, H, W, ACT_NONE, st);
}

}  // namespace unet
}  // namespace zb

using namespace zb;
using namespace zb::unet;

extern "C" {

int zb_unet_conv_impl(int impl) {
  const int prev = g_conv_impl;
  if (impl == 0 || impl == 1 || impl == 2) g_conv_impl = impl;
  return prev;
}

int zb_unet_status(int clear) {
  unsigned* p = unet_err_word();
  if (!p) return ZB_E_CUDA;
  unsigned v = 0;
  ZB_CUDA_TRY(cudaMemcpy(&v, p, sizeof(v), cudaMemcpyDeviceToHost));
  if (clear && v) {
    const unsigned z = 0;
    ZB_CUDA_TRY(cudaMemcpy(p, &z, sizeof(z), cudaMemcpyHostToDevice));
  }
  return (int)v;
}

size_t zb_unet_param_count(int c1, int c2, size_t* n_weights, size_t* n_biases) {
  if (!valid_channels(c1, c2)) return 0;
  const Net n = net_layout(c1, c2);
  if (n_weights) *n_weights = n.nw;
  if (n_biases) *n_biases = n.nb;
  return n.nw + n.nb;
}

size_t zb_smoother_workspace_bytes(int c1, int c2, int nx, int ny) {
  if (!valid_channels(c1, c2) || nx < 2 || ny < 2 || (nx & 1) || (ny & 1)) return 0;
  return acts_floats(net_layout(c1, c2), 1, nx, ny, false) * sizeof(float) + 256;
}

int zb_smoother_apply(const zb_smoother* smo, const float* f, const float* x_in, float* x_out,
                      const float* cx, const float* cy, float* r_scratch, int nx, int ny,
                      double dx, int pre, zb_stream_t stream) {
  (void)pre;
  if (!smo || !f || !x_out || !cx || !cy || !r_scratch) return ZB_E_ARG;
  if (!valid_channels(smo->c1, smo->c2) || (nx & 1) || (ny & 1)) return ZB_E_ARG;
  if (nx > smo->max_nx || ny > smo->max_ny || !smo->act ||
      smo->act_bytes < zb_smoother_workspace_bytes(smo->c1, smo->c2, nx, ny))
    return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const Net n = net_layout(smo->c1, smo->c2);
  const Acts a = acts_split(n, smo->act, 1, nx, ny, false);
  const float idx2 = (float)(1.0 / (dx * dx));
  const size_t N0 = (size_t)nx * ny;
  patch_residual<<<gridn(N0), NT, 0, st>>>(f, x_in, cx, cy, 1, nx, ny, idx2, r_scratch);
  rms(r_scratch, 1, N0, a.part, a.s, st);
  int rc;
  ActsCB8 c;
  if (g_conv_impl == 1 && acts_cb8(n, a, 1, nx, ny, &c)) {
    features_cb8_kernel<<<gridn(N0), NT, 0, st>>>(r_scratch, a.s, cx, cy, 1, nx, ny,
                                                  1.0f / smo->cmax, c.in);
    rc = forward_cb8(n, a, c, (const __nv_bfloat16*)smo->w, smo->b, 1, nx, ny, st);
  } else {
    features_kernel<<<gridn(N0), NT, 0, st>>>(r_scratch, a.s, cx, cy, 1, nx, ny,
                                              1.0f / smo->cmax, a.in);
    rc = forward(n, a, (const __nv_bfloat16*)smo->w, smo->b, 1, nx, ny, st, ACT_TANH_SFU);
  }
  if (rc) return rc;
  scale_out_kernel<<<gridn(N0), NT, 0, st>>>(a.out, a.s, cx, cy, 1, nx, ny, (float)(dx * dx),
                                             x_in, x_out);
  return zb_launch_check();
}

size_t zb_unet_train_workspace_bytes(int c1, int c2, int batch, int n) {
  if (!valid_channels(c1, c2) || batch < 1 || batch > 512 || n < 4 || (n & 1)) return 0;
  return acts_floats(net_layout(c1, c2), batch, n, n, true) * sizeof(float) + 256;
}

int zb_unet_forward(const zb_unet_trainer* t, const float* r, const float* cx, const float* cy,
                    double dx, float* y, zb_stream_t stream) {
  if (!t || !r || !cx || !cy || !y || !valid_channels(t->c1, t->c2)) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const Net n = net_layout(t->c1, t->c2);
  const Acts a = acts_split(n, t->act, t->batch, t->n, t->n, true);
  const int B = t->batch, H = t->n, W = t->n;
  const size_t N0 = (size_t)B * H * W;
  rms(r, B, (size_t)H * W, a.part, a.s, st);
  features_kernel<<<gridn(N0), NT, 0, st>>>(r, a.s, cx, cy, B, H, W, 1.0f / t->cmax, a.in);
  int rc = forward(n, a, (const __nv_bfloat16*)t->w_bf16, t->b_master, B, H, W, st);
  if (rc) return rc;
  scale_out_kernel<<<gridn(N0), NT, 0, st>>>(a.out, a.s, cx, cy, B, H, W, (float)(dx * dx),
                                             nullptr, y);
  return zb_launch_check();
}

int zb_unet_backward(const zb_unet_trainer* t, const float* r, const float* target,
                     const float* cx, const float* cy, double dx, double* loss_out,
                     zb_stream_t stream) {
  if (!t || !r || !cx || !cy || !valid_channels(t->c1, t->c2)) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const Net n = net_layout(t->c1, t->c2);
  const Acts a = acts_split(n, t->act, t->batch, t->n, t->n, true);
  const int B = t->batch, H = t->n, W = t->n, H1 = H / 2, W1 = W / 2;
  const size_t N0 = (size_t)B * H * W, N1 = (size_t)B * H1 * W1;
  const float idx2 = (float)(1.0 / (dx * dx)), dx2 = (float)(dx * dx);
  const __nv_bfloat16* w = (const __nv_bfloat16*)t->w_bf16;
  int rc;
  // forward (keeps activations), y into a.tmp
  if ((rc = zb_unet_forward(t, r, cx, cy, dx, a.tmp, stream))) return rc;
  if (target) {
    // energy loss: res = e - y, (res . A res) / (e . A e); A res -> d_out,
    // A e -> tmp (y is no longer needed once res is formed)
    sub_kernel<<<gridn(N0), NT, 0, st>>>(target, a.tmp, N0, a.res);
    patch_apply<<<gridn(N0), NT, 0, st>>>(a.res, cx, cy, B, H, W, idx2, a.d_out);
    patch_apply<<<gridn(N0), NT, 0, st>>>(target, cx, cy, B, H, W, idx2, a.tmp);
    loss_kernel<<<B, NT, 0, st>>>(a.res, a.d_out, target, a.tmp, B, (size_t)H * W, a.lnum, a.lden);
    if (loss_out) loss_total<<<1, 32, 0, st>>>(a.lnum, a.lden, B, loss_out);
    loss_grad_kernel<<<gridn(N0), NT, 0, st>>>(a.res, a.d_out, cx, cy, a.lden, a.s, B, H, W, idx2,
                                               dx2, a.d_out);
  } else {
    patch_residual<<<gridn(N0), NT, 0, st>>>(r, a.tmp, cx, cy, B, H, W, idx2, a.res);
    loss_kernel<<<B, NT, 0, st>>>(a.res, a.res, r, r, B, (size_t)H * W, a.lnum, a.lden);
    if (loss_out) loss_total<<<1, 32, 0, st>>>(a.lnum, a.lden, B, loss_out);
    loss_grad_kernel<<<gridn(N0), NT, 0, st>>>(a.res, nullptr, cx, cy, a.lden, a.s, B, H, W, idx2,
                                               dx2, a.d_out);
  }
  cudaMemsetAsync(t->g_w, 0, n.nw * sizeof(float), st);
  cudaMemsetAsync(t->g_b, 0, n.nb * sizeof(float), st);
  float* gw = t->g_w;
  float* gb = t->g_b;
  // out = conv(o1)
  if ((rc = wgrad(a.o1, n.c1, nullptr, n.c1, a.d_out, 1, gw + n.off_w[5], gb + n.off_b[5], B, H, W, st))) return rc;
  if ((rc = data_grad(n, 5, w, a.wflip, a.d_out, a.d_o1, B, H, W, st))) return rc;
  tanh_back<<<gridn((size_t)n.c1 * N0), NT, 0, st>>>(a.d_o1, a.o1, (size_t)n.c1 * N0);
  // o1 = tanh(conv([u, e2]))
  if ((rc = wgrad(a.m2, n.c2, a.e2, n.c2 + n.c1, a.d_o1, n.c1, gw + n.off_w[4], gb + n.off_b[4], B, H, W, st, SRC_UP))) return rc;
  if ((rc = data_grad(n, 4, w, a.wflip, a.d_o1, a.d_cat, B, H, W, st))) return rc;
  // d_cat = [du (c2), de2_b (c1)]
  upsample2_back<<<gridn((size_t)n.c2 * N1), NT, 0, st>>>(a.d_cat, a.d_m2, n.c2, B, H, W);
  tanh_back<<<gridn((size_t)n.c2 * N1), NT, 0, st>>>(a.d_m2, a.m2, (size_t)n.c2 * N1);
  if ((rc = wgrad(a.m1, n.c2, nullptr, n.c2, a.d_m2, n.c2, gw + n.off_w[3], gb + n.off_b[3], B, H1, W1, st))) return rc;
  if ((rc = data_grad(n, 3, w, a.wflip, a.d_m2, a.d_m1, B, H1, W1, st))) return rc;
  tanh_back<<<gridn((size_t)n.c2 * N1), NT, 0, st>>>(a.d_m1, a.m1, (size_t)n.c2 * N1);
  if ((rc = wgrad(a.e2, n.c1, nullptr, n.c1, a.d_m1, n.c2, gw + n.off_w[2], gb + n.off_b[2], B, H1, W1, st, SRC_POOL))) return rc;
  if ((rc = data_grad(n, 2, w, a.wflip, a.d_m1, a.d_p, B, H1, W1, st))) return rc;
  avgpool2_back<<<gridn((size_t)n.c1 * N0), NT, 0, st>>>(a.d_p, a.d_e2, n.c1, B, H, W);
  add_inplace<<<gridn((size_t)n.c1 * N0), NT, 0, st>>>(a.d_e2, a.d_cat + (size_t)n.c2 * N0,
                                                       (size_t)n.c1 * N0);
  tanh_back<<<gridn((size_t)n.c1 * N0), NT, 0, st>>>(a.d_e2, a.e2, (size_t)n.c1 * N0);
  if ((rc = wgrad(a.e1, n.c1, nullptr, n.c1, a.d_e2, n.c1, gw + n.off_w[1], gb + n.off_b[1], B, H, W, st))) return rc;
  if ((rc = data_grad(n, 1, w, a.wflip, a.d_e2, a.d_e1, B, H, W, st))) return rc;
  tanh_back<<<gridn((size_t)n.c1 * N0), NT, 0, st>>>(a.d_e1, a.e1, (size_t)n.c1 * N0);
  if ((rc = wgrad(a.in, 2, nullptr, 2, a.d_e1, n.c1, gw + n.off_w[0], gb + n.off_b[0], B, H, W, st))) return rc;
  return zb_launch_check();
}

int zb_unet_adam(const zb_unet_trainer* t, float lr, int step, zb_stream_t stream) {
  if (!t || step < 1 || !valid_channels(t->c1, t->c2)) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const Net n = net_layout(t->c1, t->c2);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  adam_kernel<<<gridn(n.nw), NT, 0, st>>>(t->w_master, t->m_w, t->v_w, t->g_w,
                                          (__nv_bfloat16*)t->w_bf16, (int)n.nw, lr, b1, b2, eps,
                                          c1, c2);
  // biases stay float32: the bf16 shadow is only written for the weights
  adam_kernel<<<gridn(n.nb), NT, 0, st>>>(t->b_master, t->m_b, t->v_b, t->g_b,
                                          (__nv_bfloat16*)t->b_shadow, (int)n.nb, lr, b1, b2,
                                          eps, c1, c2);
  return zb_launch_check();
}

}  // extern "C"
