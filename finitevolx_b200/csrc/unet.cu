// Learned coarse-grid preconditioner: a 4-level U-Net (16/16/32/32
// channels) with hand-written forward, backward and Adam kernels.
//
// Tensors are FP32 [B, C, h, w]; convolution weights are [Cout, Cin, 3, 3]
// with FP32 master copies for training and BF16 copies for the forward pass
// (BF16 weights, FP32 accumulation).  One conv layer reads its input through
// an optional 2x2 average pool (from a 2h x 2w tensor) or a nearest 2x
// upsample (from an h/2 x w/2 tensor), adds a bias and an optional skip
// tensor, and applies ReLU.  The reference has no learned component; this
// is new work measured against its multigrid preconditioner.
#include "fvx_common.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <type_traits>
#include <vector>

namespace fvx {
namespace nn {

enum InMode { IN_DIRECT = 0, IN_POOL = 1, IN_UP = 2 };
constexpr int TILE = 16;           // 16 x 16 output pixels per block
constexpr int THREADS = TILE * TILE;
constexpr int CMAX = 32;

// value of the conv input (channel plane ``src`` of the source tensor) at
// conv-grid pixel (y, x); zero outside [0, h) x [0, w)
DEV float in_at(const float* src, int mode, int h, int w, int y, int x) {
  if (y < 0 || y >= h || x < 0 || x >= w) return 0.f;
  if (mode == IN_DIRECT) return src[(size_t)y * w + x];
  if (mode == IN_POOL) {
    const int W2 = 2 * w;
    const float* p = src + (size_t)(2 * y) * W2 + 2 * x;
    return 0.25f * ((p[0] + p[1]) + (p[W2] + p[W2 + 1]));
  }
  return src[(size_t)(y >> 1) * (w >> 1) + (x >> 1)];  // IN_UP
}

// in_at through L2 only (ld.global.cg): for tensors the kernel before wrote,
// read after grid_dep_wait by a programmatic dependent.
DEV float in_at_l2(const float* src, int mode, int h, int w, int y, int x) {
  if (y < 0 || y >= h || x < 0 || x >= w) return 0.f;
  if (mode == IN_DIRECT) return __ldcg(src + (size_t)y * w + x);
  if (mode == IN_POOL) {
    const int W2 = 2 * w;
    const float* p = src + (size_t)(2 * y) * W2 + 2 * x;
    return 0.25f * ((__ldcg(p) + __ldcg(p + 1)) + (__ldcg(p + W2) + __ldcg(p + W2 + 1)));
  }
  return __ldcg(src + (size_t)(y >> 1) * (w >> 1) + (x >> 1));  // IN_UP
}

__host__ __device__ __forceinline__ size_t src_plane(int mode, int h, int w) {
  return mode == IN_DIRECT ? (size_t)h * w : (mode == IN_POOL ? (size_t)4 * h * w : (size_t)(h / 2) * (w / 2));
}

// y = act(W * in + b [+ skip]) for one conv layer.
// Latency-oriented: a T x T pixel tile per block with every
// input channel staged in shared memory by one cooperative load (one
// barrier), each thread accumulating CPT output channels of one pixel.
// Small tiles give enough blocks for single-field inference on coarse grids.
// Launched as a programmatic dependent of the previous layer (inference), a
// block stages the weights before waiting for that layer's output; the
// layer's input, skip tensor and scale (written by the kernels before) are
// read after the wait through L2, from pointers not marked __restrict__.
// Inference hooks of the first and last layers (null elsewhere): with
// x0_src, input channel 0 is x0_src * scale[1] (the network input f / s
// formed while the tile loads); with out_mask, the output is
// (y * (scale[0] * sigma)) * out_mask (the coarse correction s sigma m y).
struct ConvHooks {
  const float* x0_src = nullptr;
  const float* scale = nullptr;
  const float* out_mask = nullptr;
  float sigma = 1.f;
};

template <int COUT, int CPT, int T>
__global__ void __launch_bounds__(T * T * (COUT / CPT))
conv_tile_kernel(const float* in, int mode, int cin, const __nv_bfloat16* __restrict__ wb,
                 const float* __restrict__ bias, const float* skip, float* __restrict__ out, int h, int w, int relu,
                 ConvHooks hk) {
  constexpr int NT = T * T * (COUT / CPT);
  constexpr int TW = T + 2;
  extern __shared__ __align__(16) float sm[];
  float* ws = sm;                     // [cin * 9][COUT]
  float* tile = sm + cin * 9 * COUT;  // [cin][TW][TW]
  const int b = blockIdx.z;
  const int x0 = blockIdx.x * T, y0 = blockIdx.y * T;
  const int tid = threadIdx.x;
  // staging in batches of 16 per thread so the loads overlap
  const int nw = cin * 9 * COUT;
  for (int k0 = tid; k0 < nw; k0 += 16 * NT) {
    float v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int k = k0 + u * NT;
      const int co = k % COUT, rest = k / COUT;
      v[u] = k < nw ? __bfloat162float(wb[(size_t)co * cin * 9 + rest]) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u)
      if (k0 + u * NT < nw) ws[k0 + u * NT] = v[u];
  }
  grid_dep_wait();  // the input (and skip) come from the previous kernel
  const size_t sp = src_plane(mode, h, w);
  const float* inb = in + (size_t)b * cin * sp;
  const int nt = cin * TW * TW;
  const float x0s = hk.x0_src ? __ldcg(hk.scale + 1) : 0.f;
  for (int k0 = tid; k0 < nt; k0 += 16 * NT) {
    float v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int k = k0 + u * NT;
      const int ci = k / (TW * TW), r = k - ci * (TW * TW);
      const int ly = r / TW, lx = r - ly * TW;
      if (hk.x0_src && ci == 0)
        v[u] = k < nt ? in_at_l2(hk.x0_src, mode, h, w, y0 - 1 + ly, x0 - 1 + lx) * x0s : 0.f;
      else
        v[u] = k < nt ? in_at_l2(inb + ci * sp, mode, h, w, y0 - 1 + ly, x0 - 1 + lx) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u)
      if (k0 + u * NT < nt) tile[k0 + u * NT] = v[u];
  }
  __syncthreads();
  grid_dep_launch();
  const int p = tid % (T * T), co0 = (tid / (T * T)) * CPT;
  const int ty = p / T, tx = p % T;
  float acc[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) acc[c] = 0.f;
  for (int ci = 0; ci < cin; ++ci) {
    const float* tl = tile + ci * TW * TW + ty * TW + tx;
    const float* wc = ws + ci * 9 * COUT + co0;
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const float v = tl[(t / 3) * TW + t % 3];
      const float* wr = wc + t * COUT;
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] = fmaf(wr[c], v, acc[c]);
    }
  }
  const int y = y0 + ty, x = x0 + tx;
  if (y >= h || x >= w) return;
  const size_t plane = (size_t)h * w, base = (size_t)b * COUT * plane + (size_t)y * w + x;
  const float os = hk.out_mask ? __ldcg(hk.scale) * hk.sigma : 0.f;
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int co = co0 + c;
    float v = acc[c] + bias[co];
    if (skip) v += __ldcg(skip + base + co * plane);
    if (relu) v = fmaxf(v, 0.f);
    if (hk.out_mask) v = (v * os) * hk.out_mask[(size_t)y * w + x];
    out[base + co * plane] = v;
  }
}

template <int COUT, int CPT, int T>
static int launch_conv_tile(const float* in, int mode, int batch, int cin, const __nv_bfloat16* wb,
                            const float* bias, const float* skip, float* out, int h, int w, int relu,
                            cudaStream_t st, bool pdl, ConvHooks hk) {
  constexpr int NT = T * T * (COUT / CPT);
  const size_t smem = ((size_t)cin * 9 * COUT + (size_t)cin * (T + 2) * (T + 2)) * sizeof(float);
  static fvx_once_per_device attr;  // per instantiation; the largest use needs > 48 KB
  if (fvx_once_on_device(attr, [] {
        const int max_smem = (CMAX * 9 * COUT + CMAX * (T + 2) * (T + 2)) * (int)sizeof(float);
        return fvx_set_max_smem(conv_tile_kernel<COUT, CPT, T>, max_smem);
      }))
    return FVX_ERR_CUDA;
  dim3 g((w + T - 1) / T, (h + T - 1) / T, batch);
  if (pdl) {
    if (fvx_launch_pdl(conv_tile_kernel<COUT, CPT, T>, g, dim3(NT), smem, st, in, mode, cin, wb, bias, skip, out, h,
                       w, relu, hk) != cudaSuccess)
      return FVX_ERR_CUDA;
  } else {
    conv_tile_kernel<COUT, CPT, T><<<g, NT, smem, st>>>(in, mode, cin, wb, bias, skip, out, h, w, relu, hk);
  }
  return fvx_cuda_status();
}

// The network's last three layers in one kernel (single-field inference):
// the half-resolution decoder conv (nearest upsample of the quarter-
// resolution tensor, 32 -> 16, + skip, ReLU) on the 6 x 6 half-resolution
// pixels the next conv's upsampled input touches, the full-resolution
// decoder conv (16 -> 16, + skip, ReLU) on the 8 x 8 output tile and a
// one-pixel ring around it, both kept in shared memory, then the output
// conv (16 -> 1) and the output hook on the tile.  The halo values are
// recomputed by the neighbouring tiles (2.25x and 1.56x those two layers'
// products, for two launches and two tensor round trips fewer); every value
// is summed in the same order as conv_tile_kernel, so the result equals the
// layer-by-layer form.
constexpr int kDT = 8;                 // output tile (full resolution)
constexpr int kDR = kDT + 2;           // full-resolution decoder ring
constexpr int kDH = kDT / 2 + 2;       // half-resolution decoder pixels per side
constexpr int kDQ = kDH / 2 + 1;       // quarter-resolution input pixels per side
constexpr int kDThreads = 512;
__global__ void __launch_bounds__(kDThreads)
conv_d1_d0_out_kernel(const float* a4, const float* a1, const float* a0, const __nv_bfloat16* __restrict__ w5,
                      const float* __restrict__ b5, const __nv_bfloat16* __restrict__ w6,
                      const float* __restrict__ b6, const __nv_bfloat16* __restrict__ w7,
                      const float* __restrict__ b7, float* __restrict__ out, int h, int w, ConvHooks hk) {
  constexpr int C4 = 32, C = 16;
  __shared__ float ws5[C4 * 9 * C];        // [ci * 9][co]
  __shared__ float ws6[C * 9 * C];
  __shared__ float ws7[C * 9];
  __shared__ float t4[C4][kDQ][kDQ];       // quarter-resolution input, origin (y0 / 4 - 1, x0 / 4 - 1)
  __shared__ float t1[C][kDH][kDH];        // half-resolution skip, origin (y0 / 2 - 1, x0 / 2 - 1)
  __shared__ float t5[C][kDH][kDH];        // half-resolution decoder output, same origin
  __shared__ float td[C][kDR][kDR];        // full-resolution decoder output, origin (y0 - 1, x0 - 1)
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * kDT, y0 = blockIdx.y * kDT;
  const int h1 = h >> 1, w1 = w >> 1, h2 = h >> 2, w2 = w >> 2;
  const int H0 = (y0 >> 1) - 1, G0 = (x0 >> 1) - 1;  // half-resolution origin
  const int Q0 = (y0 >> 2) - 1, P0 = (x0 >> 2) - 1;  // quarter-resolution origin
  for (int k = tid; k < C4 * 9 * C; k += kDThreads) {
    const int co = k % C, rest = k / C;
    ws5[k] = __bfloat162float(w5[(size_t)co * C4 * 9 + rest]);
  }
  for (int k = tid; k < C * 9 * C; k += kDThreads) {
    const int co = k % C, rest = k / C;
    ws6[k] = __bfloat162float(w6[(size_t)co * C * 9 + rest]);
  }
  for (int k = tid; k < C * 9; k += kDThreads) ws7[k] = __bfloat162float(w7[k]);
  grid_dep_wait();  // the decoder's inputs come from the kernels before
  {
    constexpr int N4 = C4 * kDQ * kDQ, N1 = C * kDH * kDH;
    float v[3];
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      const int k = tid + u * kDThreads;
      v[u] = 0.f;
      if (k < N4) {
        const int ci = k / (kDQ * kDQ), r = k - ci * (kDQ * kDQ);
        const int ly = r / kDQ, lx = r - ly * kDQ;
        v[u] = in_at_l2(a4 + (size_t)ci * h2 * w2, IN_DIRECT, h2, w2, Q0 + ly, P0 + lx);
      } else if (k < N4 + N1) {
        const int kk = k - N4;
        const int ci = kk / (kDH * kDH), r = kk - ci * (kDH * kDH);
        const int ly = r / kDH, lx = r - ly * kDH;
        v[u] = in_at_l2(a1 + (size_t)ci * h1 * w1, IN_DIRECT, h1, w1, H0 + ly, G0 + lx);
      }
    }
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      const int k = tid + u * kDThreads;
      if (k < N4) (&t4[0][0][0])[k] = v[u];
      else if (k < N4 + N1) (&t1[0][0][0])[k - N4] = v[u];
    }
  }
  __syncthreads();
  grid_dep_launch();
  // half-resolution decoder conv: 36 pixels x 8 groups of 2 channels
  if (tid < kDH * kDH * (C / 2)) {
    constexpr int CPT = 2;
    const int p = tid % (kDH * kDH), co0 = (tid / (kDH * kDH)) * CPT;
    const int hy = p / kDH, hx = p % kDH;
    const int Y = H0 + hy, X = G0 + hx;
    float acc[CPT] = {0.f, 0.f};
    for (int ci = 0; ci < C4; ++ci) {
      const float* wc = ws5 + ci * 9 * C + co0;
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const int yy = Y - 1 + t / 3, xx = X - 1 + t % 3;
        const float v = (yy >= 0 && yy < h1 && xx >= 0 && xx < w1) ? t4[ci][(yy >> 1) - Q0][(xx >> 1) - P0] : 0.f;
        const float* wr = wc + t * C;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = fmaf(wr[c], v, acc[c]);
      }
    }
    const bool inside = Y >= 0 && Y < h1 && X >= 0 && X < w1;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int co = co0 + c;
      float v = 0.f;  // never read: the next conv's upsampled input is zero off the grid
      if (inside) v = fmaxf((acc[c] + b5[co]) + t1[co][hy][hx], 0.f);
      t5[co][hy][hx] = v;
    }
  }
  __syncthreads();
  // full-resolution decoder conv on the 10 x 10 ring region: 100 pixels x 4 groups of 4 channels
  if (tid < kDR * kDR * (C / 4)) {
    constexpr int CPT = 4;
    const int p = tid % (kDR * kDR), co0 = (tid / (kDR * kDR)) * CPT;
    const int ry = p / kDR, rx = p % kDR;
    const int y = y0 - 1 + ry, x = x0 - 1 + rx;
    float acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.f;
    for (int ci = 0; ci < C; ++ci) {
      const float* wc = ws6 + ci * 9 * C + co0;
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const int yy = y - 1 + t / 3, xx = x - 1 + t % 3;
        const float v = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? t5[ci][(yy >> 1) - H0][(xx >> 1) - G0] : 0.f;
        const float* wr = wc + t * C;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = fmaf(wr[c], v, acc[c]);
      }
    }
    const bool inside = y >= 0 && y < h && x >= 0 && x < w;
    const size_t base = inside ? (size_t)y * w + x : 0, plane = (size_t)h * w;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int co = co0 + c;
      float v = 0.f;  // the output conv reads zero outside the grid
      if (inside) v = fmaxf((acc[c] + b6[co]) + __ldcg(a0 + base + co * plane), 0.f);
      td[co][ry][rx] = v;
    }
  }
  __syncthreads();
  // output conv on the 8 x 8 tile
  if (tid < kDT * kDT) {
    const int ty = tid / kDT, tx = tid % kDT;
    const int y = y0 + ty, x = x0 + tx;
    float acc = 0.f;
    for (int ci = 0; ci < C; ++ci) {
#pragma unroll
      for (int t = 0; t < 9; ++t) acc = fmaf(ws7[ci * 9 + t], td[ci][ty + t / 3][tx + t % 3], acc);
    }
    if (y < h && x < w) {
      const size_t base = (size_t)y * w + x;
      float v = acc + b7[0];
      const float os = __ldcg(hk.scale) * hk.sigma;
      v = (v * os) * hk.out_mask[base];
      out[base] = v;
    }
  }
}

// The network's first two layers in one kernel (single-field inference): the
// input conv (3 -> 16, ReLU; channel 0 = f / s as it loads) on the fine
// pixels under a 4 x 4 tile of the half-resolution grid and its one-pixel
// ring, kept in shared memory (the block writes its own 8 x 8 of it, the
// decoder's skip tensor), then 2 x 2 average pooling and the second conv
// (16 -> 16, ReLU) on the tile.  The ring's values are recomputed by the
// neighbouring tiles (2.25x the first layer's 27 products per output for one
// launch and one tensor read fewer); every value is summed in the same order
// as conv_tile_kernel, so the result equals the two-launch form.
constexpr int kE1T = 4, kE1R = kE1T + 2, kE0R = 2 * kE1R, kE0IN = kE0R + 2;
constexpr int kE01Threads = 288;
__global__ void __launch_bounds__(kE01Threads)
conv_e0_e1_kernel(const float* x, const float* f, const __nv_bfloat16* __restrict__ w0,
                  const float* __restrict__ b0, const __nv_bfloat16* __restrict__ w1, const float* __restrict__ b1,
                  float* __restrict__ a0, float* __restrict__ a1, int h, int w, const float* scale) {
  constexpr int C0 = 3, C1 = 16;
  __shared__ float ws0[C0 * 9 * C1];          // [ci * 9][co]
  __shared__ float ws1[C1 * 9 * C1];
  __shared__ float tx[C0][kE0IN][kE0IN];      // input, origin (2 Y0 - 3, 2 X0 - 3)
  __shared__ float t0[C1][kE0R][kE0R];        // first layer's output, origin (2 Y0 - 2, 2 X0 - 2)
  __shared__ float tp[C1][kE1R][kE1R];        // pooled, origin (Y0 - 1, X0 - 1)
  const int tid = threadIdx.x;
  const int h1 = h >> 1, w1n = w >> 1;
  const int X0 = blockIdx.x * kE1T, Y0 = blockIdx.y * kE1T;
  const int fy0 = 2 * Y0 - 2, fx0 = 2 * X0 - 2;
  for (int k = tid; k < C0 * 9 * C1; k += kE01Threads) {
    const int co = k % C1, rest = k / C1;
    ws0[k] = __bfloat162float(w0[(size_t)co * C0 * 9 + rest]);
  }
  for (int k = tid; k < C1 * 9 * C1; k += kE01Threads) {
    const int co = k % C1, rest = k / C1;
    ws1[k] = __bfloat162float(w1[(size_t)co * C1 * 9 + rest]);
  }
  grid_dep_wait();  // f and the scale come from the kernels before
  const size_t plane = (size_t)h * w;
  const float rs = __ldcg(scale + 1);
  {
    constexpr int NIN = C0 * kE0IN * kE0IN;
    float v[3];
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      const int k = tid + u * kE01Threads;
      v[u] = 0.f;
      if (k < NIN) {
        const int ci = k / (kE0IN * kE0IN), r = k - ci * (kE0IN * kE0IN);
        const int ly = r / kE0IN, lx = r - ly * kE0IN;
        v[u] = ci == 0 ? in_at_l2(f, IN_DIRECT, h, w, fy0 - 1 + ly, fx0 - 1 + lx) * rs
                       : in_at_l2(x + ci * plane, IN_DIRECT, h, w, fy0 - 1 + ly, fx0 - 1 + lx);
      }
    }
#pragma unroll
    for (int u = 0; u < 3; ++u)
      if (tid + u * kE01Threads < NIN) (&tx[0][0][0])[tid + u * kE01Threads] = v[u];
  }
  __syncthreads();
  grid_dep_launch();
  // first layer on the 12 x 12 fine region: 144 pixels x 2 groups of 8 channels
  {
    constexpr int CPT = 8;
    const int p = tid % (kE0R * kE0R), co0 = (tid / (kE0R * kE0R)) * CPT;
    const int ry = p / kE0R, rx = p % kE0R;
    const int y = fy0 + ry, xg = fx0 + rx;
    float acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.f;
    for (int ci = 0; ci < C0; ++ci) {
      const float* wc = ws0 + ci * 9 * C1 + co0;
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const float v = tx[ci][ry + t / 3][rx + t % 3];
        const float* wr = wc + t * C1;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = fmaf(wr[c], v, acc[c]);
      }
    }
    const bool inside = y >= 0 && y < h && xg >= 0 && xg < w;
    const bool own = ry >= 2 && ry < 2 + 2 * kE1T && rx >= 2 && rx < 2 + 2 * kE1T;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int co = co0 + c;
      const float v = fmaxf(acc[c] + b0[co], 0.f);
      t0[co][ry][rx] = v;
      if (inside && own) a0[(size_t)co * plane + (size_t)y * w + xg] = v;
    }
  }
  __syncthreads();
  // 2 x 2 average pooling (zero off the half-resolution grid)
  for (int k = tid; k < C1 * kE1R * kE1R; k += kE01Threads) {
    const int ci = k / (kE1R * kE1R), r = k - ci * (kE1R * kE1R);
    const int ly = r / kE1R, lx = r - ly * kE1R;
    const int Y = Y0 - 1 + ly, X = X0 - 1 + lx;
    float v = 0.f;
    if (Y >= 0 && Y < h1 && X >= 0 && X < w1n)
      v = 0.25f * ((t0[ci][2 * ly][2 * lx] + t0[ci][2 * ly][2 * lx + 1]) +
                   (t0[ci][2 * ly + 1][2 * lx] + t0[ci][2 * ly + 1][2 * lx + 1]));
    tp[ci][ly][lx] = v;
  }
  __syncthreads();
  // second layer on the 4 x 4 tile: 16 pixels x 16 channels
  if (tid < kE1T * kE1T * C1) {
    const int p = tid % (kE1T * kE1T), co = tid / (kE1T * kE1T);
    const int ty = p / kE1T, tx_ = p % kE1T;
    const int Y = Y0 + ty, X = X0 + tx_;
    float acc = 0.f;
    for (int ci = 0; ci < C1; ++ci) {
#pragma unroll
      for (int t = 0; t < 9; ++t) acc = fmaf(ws1[(ci * 9 + t) * C1 + co], tp[ci][ty + t / 3][tx_ + t % 3], acc);
    }
    if (Y < h1 && X < w1n) a1[(size_t)co * h1 * w1n + (size_t)Y * w1n + X] = fmaxf(acc + b1[co], 0.f);
  }
}

// G = dL/d(pre-activation) = dY * (y > 0) (or dY when the layer is linear);
// dskip += G.
DEV float4 relu_mask4(float4 d, float4 yv, int relu) {
  if (relu) {
    d.x = yv.x > 0.f ? d.x : 0.f;
    d.y = yv.y > 0.f ? d.y : 0.f;
    d.z = yv.z > 0.f ? d.z : 0.f;
    d.w = yv.w > 0.f ? d.w : 0.f;
  }
  return d;
}
// g = dL/dy masked by the ReLU (y > 0), dskip += g.  Four elements per
// access and two accesses per trip when every pointer is 16-byte aligned
// (each trip's loads issued before its stores); else one element at a time.
__global__ void act_grad_kernel(const float* dy, const float* y, float* g, float* dskip, size_t n, int relu) {
  const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (size_t)gridDim.x * blockDim.x;
  const bool v4 = (((uintptr_t)dy | (uintptr_t)y | (uintptr_t)g | (uintptr_t)dskip) & 15) == 0;
  size_t head = 0;
  if (v4) {
    const size_t n4 = n / 4;
    const float4* dy4 = (const float4*)dy;
    const float4* y4 = (const float4*)y;
    float4* g4 = (float4*)g;
    float4* s4 = (float4*)dskip;
    for (size_t k = t0; k < n4; k += 2 * stride) {
      const size_t k2 = k + stride;
      const bool two = k2 < n4;
      const float4 d0 = dy4[k], y0 = y4[k];
      float4 d1 = make_float4(0.f, 0.f, 0.f, 0.f), y1 = d1, a0 = d1, a1 = d1;
      if (two) { d1 = dy4[k2]; y1 = y4[k2]; }
      if (dskip) {
        a0 = s4[k];
        if (two) a1 = s4[k2];
      }
      const float4 v0 = relu_mask4(d0, y0, relu), v1 = relu_mask4(d1, y1, relu);
      g4[k] = v0;
      if (two) g4[k2] = v1;
      if (dskip) {
        s4[k] = make_float4(a0.x + v0.x, a0.y + v0.y, a0.z + v0.z, a0.w + v0.w);
        if (two) s4[k2] = make_float4(a1.x + v1.x, a1.y + v1.y, a1.z + v1.z, a1.w + v1.w);
      }
    }
    head = n4 * 4;
  }
  for (size_t k = head + t0; k < n; k += stride) {
    const float v = relu ? (y[k] > 0.f ? dy[k] : 0.f) : dy[k];
    g[k] = v;
    if (dskip) dskip[k] += v;
  }
}

// dXin[b, ci, p] = sum_co sum_t W[co][ci][t] G[b, co, p - (t - 1)] (the conv's
// adjoint on the conv-input grid), W the BF16 weights the forward pass used.
template <int CIN>
__global__ void __launch_bounds__(THREADS)
conv_bwd_data_kernel(const float* __restrict__ g, int cout, const __nv_bfloat16* __restrict__ wb,
                     float* __restrict__ dxin, int h, int w) {
  __shared__ float tile[TILE + 2][TILE + 2];
  __shared__ float ws[CMAX * 9 * CIN];
  const int b = blockIdx.z;
  const int x0 = blockIdx.x * TILE, y0 = blockIdx.y * TILE;
  const int tx = threadIdx.x % TILE, ty = threadIdx.x / TILE;
  for (int k = threadIdx.x; k < cout * 9 * CIN; k += THREADS) {
    // ws[(co*9 + t)*CIN + ci] = W[co][ci][t]
    const int ci = k % CIN, rest = k / CIN, co = rest / 9, t = rest % 9;
    ws[k] = __bfloat162float(wb[((size_t)co * CIN + ci) * 9 + t]);
  }
  float acc[CIN];
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.f;
  const size_t plane = (size_t)h * w;
  const float* gb = g + (size_t)b * cout * plane;
  for (int co = 0; co < cout; ++co) {
    __syncthreads();
    for (int k = threadIdx.x; k < (TILE + 2) * (TILE + 2); k += THREADS) {
      const int ly = k / (TILE + 2), lx = k % (TILE + 2);
      const int yy = y0 - 1 + ly, xx = x0 - 1 + lx;
      tile[ly][lx] = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? gb[co * plane + (size_t)yy * w + xx] : 0.f;
    }
    __syncthreads();
    // input pixel p receives G at p - (t - 1): tile offset (2 - dy, 2 - dx)
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const float v = tile[ty + 2 - t / 3][tx + 2 - t % 3];
      const float* wr = ws + (co * 9 + t) * CIN;
#pragma unroll
      for (int ci = 0; ci < CIN; ++ci) acc[ci] = fmaf(wr[ci], v, acc[ci]);
    }
  }
  const int y = y0 + ty, x = x0 + tx;
  if (y >= h || x >= w) return;
  const size_t base = (size_t)b * CIN * plane + (size_t)y * w + x;
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) dxin[base + ci * plane] = acc[ci];
}

// Batched 3x3 convolution for training (many samples):
//   out[b][co] = act(sum_ci sum_t W[co][ci][t] in~[b][ci](p + shift t) + bias[co] (+ skip)),
// in~ the mode-transformed input.  A block covers a TH x 32 pixel tile of
// one sample and every output channel; a thread owns 8 consecutive pixels
// of one row x 8 output channels (64 FMA accumulators), walks the input
// channels in chunks of 8 staged in shared memory, and per (channel, tap
// row) loads one 10-value input window and per tap 8 weights as two
// float4: 33 shared loads per 576 FMAs.  WT = bf16: the forward weights
// W[co][ci][9]; WT = float: any [co][ci][9] FP32 table (the data gradient's
// transposed, flipped weights).  bias and skip may be null.
constexpr int kBcPX = 8, kBcCO = 8, kBcTW = 32, kBcKC = 8, kBcPitch = kBcTW + 2;
template <int COUT> struct BcCfg {
  static constexpr int NCG = COUT / kBcCO;        // channel groups
  static constexpr int TH = THREADS / (4 * NCG);   // tile rows (4 threads cover a row of 32 pixels)
  static constexpr int IN_FLOATS = kBcKC * (TH + 2) * kBcPitch;
  static_assert(IN_FLOATS % 4 == 0, "the weight table starts 16-byte aligned");
};
template <int COUT>
static size_t bc_smem(int cin, bool adjoint = false) {
  const size_t main = (size_t)BcCfg<COUT>::IN_FLOATS + (size_t)cin * 9 * COUT;
  const size_t adj = adjoint ? (size_t)COUT * BcCfg<COUT>::TH * (kBcTW + 1) : 0;  // the adjoint epilogue's tile
  return (main > adj ? main : adj) * sizeof(float);
}

// Adjoint epilogue of the data gradient: the tile's 8 channels of dX (in
// shared memory, [8][TH][EP]) go straight into the gradient of the layer's
// source, dsrc += T^T dX, instead of through a dX tensor: IN_DIRECT adds
// them, IN_POOL spreads each value / 4 over its 2 x 2 source pixels, IN_UP
// gathers each source pixel's 2 x 2 children (the tile holds whole groups:
// y0 and x0 even, h and w even).  Every dsrc element is updated by one
// thread, in the order of the separate adjoint pass.  A thread takes runs of
// 4 destination pixels along a row (float4 read-modify-writes when aligned)
// and issues the loads of 4 runs before any store.
template <int COUT, int TH, int EP>
DEV void conv_batch_adjoint(const float* e, float* dsrc, int amode, int b, int grp, int y0, int x0, int h, int w) {
  // destination runs per channel: rows x (columns / 4) of the tile's image
  // in dsrc (IN_POOL: two source rows per tile row, each 8 wide per run of 4)
  const bool up = amode == IN_UP, pool = amode == IN_POOL;
  const int drows = up ? TH / 2 : TH, druns = up ? kBcTW / 8 : kBcTW / 4;
  const int dh = up ? h >> 1 : (pool ? 2 * h : h), dw = up ? w >> 1 : (pool ? 2 * w : w);
  const bool v4 = (dw & 3) == 0 && ((uintptr_t)dsrc & 15) == 0;
  const int n = kBcCO * drows * druns;
  for (int base = threadIdx.x; base < n; base += 4 * THREADS) {
    float4 add[4][2];
    float4 cur[4][2];
    size_t off[4];
    int valid[4], dxs[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = base + u * THREADS;
      valid[u] = 0;
      if (k >= n) continue;
      const int q = k / (drows * druns), rem = k - q * (drows * druns);
      const int rr = rem / druns, j = rem - rr * druns;
      const size_t pl = (size_t)b * COUT + grp * kBcCO + q;
      int dy, dx;  // first destination pixel of the run
      if (up) {
        dy = (y0 >> 1) + rr;
        dx = (x0 >> 1) + 4 * j;
        const float* c = e + (q * TH + 2 * rr) * EP + 8 * j;
        float v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] = (c[2 * i] + c[2 * i + 1]) + (c[EP + 2 * i] + c[EP + 2 * i + 1]);
        add[u][0] = make_float4(v[0], v[1], v[2], v[3]);
        add[u][1] = make_float4(0.f, 0.f, 0.f, 0.f);
      } else {
        const float* c = e + (q * TH + rr) * EP + 4 * j;
        if (pool) {
          dy = 2 * (y0 + rr);
          dx = 2 * (x0 + 4 * j);
          const float a0 = 0.25f * c[0], a1 = 0.25f * c[1], a2 = 0.25f * c[2], a3 = 0.25f * c[3];
          add[u][0] = make_float4(a0, a0, a1, a1);
          add[u][1] = make_float4(a2, a2, a3, a3);
        } else {
          dy = y0 + rr;
          dx = x0 + 4 * j;
          add[u][0] = make_float4(c[0], c[1], c[2], c[3]);
          add[u][1] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
      if (dy >= dh || dx >= dw) continue;
      dxs[u] = dx;
      valid[u] = (v4 && dx + (pool ? 8 : 4) <= dw) ? 2 : 1;
      off[u] = (pl * dh + dy) * dw + dx;
      if (valid[u] == 2) {
        cur[u][0] = *(const float4*)(dsrc + off[u]);
        if (pool) {
          cur[u][1] = *(const float4*)(dsrc + off[u] + 4);
        }
      }
    }
    // IN_POOL also needs the second source row: loaded with the first
    float4 cur2[4][2];
    if (pool) {
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (valid[u] == 2) {
          cur2[u][0] = *(const float4*)(dsrc + off[u] + dw);
          cur2[u][1] = *(const float4*)(dsrc + off[u] + dw + 4);
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (valid[u] == 2) {
        const int nv = pool ? 2 : 1;
        for (int h2 = 0; h2 < nv; ++h2) {
          float4 a = cur[u][h2];
          const float4 d = add[u][h2];
          a.x += d.x; a.y += d.y; a.z += d.z; a.w += d.w;
          *(float4*)(dsrc + off[u] + 4 * h2) = a;
          if (pool) {
            float4 a2 = cur2[u][h2];
            a2.x += d.x; a2.y += d.y; a2.z += d.z; a2.w += d.w;
            *(float4*)(dsrc + off[u] + dw + 4 * h2) = a2;
          }
        }
      } else if (valid[u] == 1) {
        // ragged or unaligned run: element by element, inside the row
        const float4 d0 = add[u][0], d1 = add[u][1];
        const float vals[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
        const int len = pool ? 8 : 4;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          if (i >= len || dxs[u] + i >= dw) break;
          dsrc[off[u] + i] += vals[i];
          if (pool) dsrc[off[u] + dw + i] += vals[i];
        }
      }
    }
  }
}

template <int COUT, typename WT>
__global__ void __launch_bounds__(THREADS)
conv_batch_kernel(const float* __restrict__ in, int mode, int cin, const WT* __restrict__ wt,
                  const float* __restrict__ bias, const float* __restrict__ skip, float* __restrict__ out, int h,
                  int w, int relu, int amode) {
  using C = BcCfg<COUT>;
  constexpr int TH = C::TH, NCG = C::NCG;
  extern __shared__ __align__(16) float bsm[];
  float* xin = bsm;               // [kBcKC][TH + 2][kBcPitch], origin (y0 - 1, x0 - 1)
  float* ws = bsm + C::IN_FLOATS;  // [cin][9][COUT]
  const int tid = threadIdx.x;
  const int g = tid % NCG, c = (tid / NCG) % 4, r = tid / (4 * NCG);
  const int b = blockIdx.z, x0 = blockIdx.x * kBcTW, y0 = blockIdx.y * TH;
  for (int k = tid; k < cin * 9 * COUT; k += THREADS) {
    const int co = k % COUT, rest = k / COUT;  // rest = ci * 9 + t
    if constexpr (std::is_same<WT, float>::value) ws[k] = wt[(size_t)co * cin * 9 + rest];
    else ws[k] = __bfloat162float(wt[(size_t)co * cin * 9 + rest]);
  }
  float acc[kBcPX][kBcCO];
#pragma unroll
  for (int p = 0; p < kBcPX; ++p)
#pragma unroll
    for (int q = 0; q < kBcCO; ++q) acc[p][q] = 0.f;
  const size_t sp = src_plane(mode, h, w);
  const float* inb = in + (size_t)b * cin * sp;
  for (int c0 = 0; c0 < cin; c0 += kBcKC) {
    const int kc = cin - c0 < kBcKC ? cin - c0 : kBcKC;
    __syncthreads();  // the previous chunk's reads are done
    stage8(
        kc * (TH + 2) * kBcPitch,
        [&](int k) {
          const int cc = k / ((TH + 2) * kBcPitch), q = k - cc * ((TH + 2) * kBcPitch);
          const int ly = q / kBcPitch, lx = q - ly * kBcPitch;
          return in_at(inb + (size_t)(c0 + cc) * sp, mode, h, w, y0 - 1 + ly, x0 - 1 + lx);
        },
        [&](int k, float v) { xin[k] = v; });
    __syncthreads();
    for (int cc = 0; cc < kc; ++cc) {
      const float* xr = xin + (cc * (TH + 2) + r) * kBcPitch + c * kBcPX;
      const float* wr = ws + (size_t)(c0 + cc) * 9 * COUT + g * kBcCO;
#pragma unroll
      for (int dy = 0; dy < 3; ++dy) {
        float row[kBcPX + 2];
#pragma unroll
        for (int j = 0; j < kBcPX + 2; j += 2) {
          const float2 v = *(const float2*)(xr + dy * kBcPitch + j);
          row[j] = v.x;
          row[j + 1] = v.y;
        }
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
          const float4 wa = *(const float4*)(wr + (dy * 3 + dx) * COUT);
          const float4 wb = *(const float4*)(wr + (dy * 3 + dx) * COUT + 4);
          const float wv[kBcCO] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
          for (int p = 0; p < kBcPX; ++p)
#pragma unroll
            for (int q = 0; q < kBcCO; ++q) acc[p][q] = fmaf(row[p + dx], wv[q], acc[p][q]);
        }
      }
    }
  }
  // epilogue: each group of 8 output channels passes through shared memory
  // ([8][TH][33], reusing the input tile) so that the stores and the skip
  // loads run along whole tile rows, four pixels per thread
  constexpr int EP = kBcTW + 1;
  static_assert(kBcCO * TH * EP <= C::IN_FLOATS, "epilogue staging fits the input tile");
  if (amode >= 0) {
    // data gradient: every channel of the tile into shared memory at once
    // ([COUT][TH][EP], launched with room for it), then dsrc += T^T dX
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kBcCO; ++q)
#pragma unroll
      for (int p = 0; p < kBcPX; ++p) xin[((g * kBcCO + q) * TH + r) * EP + c * kBcPX + p] = acc[p][q];
    __syncthreads();
    for (int grp = 0; grp < NCG; ++grp)
      conv_batch_adjoint<COUT, TH, EP>(xin + grp * kBcCO * TH * EP, out, amode, b, grp, y0, x0, h, w);
    return;
  }
  const bool v4 = (w & 3) == 0 && (((uintptr_t)out | (uintptr_t)skip) & 15) == 0;
  for (int grp = 0; grp < NCG; ++grp) {
    __syncthreads();
    if (g == grp) {
#pragma unroll
      for (int q = 0; q < kBcCO; ++q)
#pragma unroll
        for (int p = 0; p < kBcPX; ++p) xin[(q * TH + r) * EP + c * kBcPX + p] = acc[p][q];
    }
    __syncthreads();
    for (int k = tid; k < kBcCO * TH * (kBcTW / 4); k += THREADS) {
      const int q = k / (TH * (kBcTW / 4)), rem = k - q * (TH * (kBcTW / 4));
      const int rr = rem / (kBcTW / 4), x4 = (rem - rr * (kBcTW / 4)) * 4;
      const int co = grp * kBcCO + q, y = y0 + rr, x = x0 + x4;
      if (y >= h || x >= w) continue;
      const float bq = bias ? bias[co] : 0.f;
      const float* e = xin + (q * TH + rr) * EP + x4;
      float v[4] = {e[0] + bq, e[1] + bq, e[2] + bq, e[3] + bq};
      const size_t o = (((size_t)b * COUT + co) * h + y) * w + x;
      if (v4 && x + 4 <= w) {
        if (skip) {
          const float4 s = *(const float4*)(skip + o);
          v[0] += s.x; v[1] += s.y; v[2] += s.z; v[3] += s.w;
        }
        if (relu) {
#pragma unroll
          for (int j = 0; j < 4; ++j) v[j] = fmaxf(v[j], 0.f);
        }
        *(float4*)(out + o) = make_float4(v[0], v[1], v[2], v[3]);
      } else {
        for (int j = 0; j < 4 && x + j < w; ++j) {
          float t = v[j];
          if (skip) t += skip[o + j];
          if (relu) t = fmaxf(t, 0.f);
          out[o + j] = t;
        }
      }
    }
  }
}

// The data gradient's weights for conv_batch_kernel: wt[ci][co][t] =
// W[co][ci][8 - t] (input pixel p receives G at p - shift t).
__global__ void flip_transpose_kernel(const __nv_bfloat16* __restrict__ wb, int cin, int cout,
                                      float* __restrict__ wt) {
  const int n = cin * cout * 9;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int ci = k / (cout * 9), rest = k - ci * (cout * 9), co = rest / 9, t = rest - co * 9;
    wt[k] = __bfloat162float(wb[((size_t)co * cin + ci) * 9 + (8 - t)]);
  }
}

// Adjoint of the input transform: dsrc += T^T dxin.
__global__ void in_adjoint_kernel(const float* dxin, float* dsrc, int mode, int bc, int h, int w) {
  // bc = B * Cin planes; conv grid h x w
  const size_t sp = src_plane(mode, h, w);
  const size_t n = (size_t)bc * sp;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const size_t pl = k / sp, r = k - pl * sp;
    const float* d = dxin + pl * (size_t)h * w;
    float v;
    if (mode == IN_DIRECT) v = d[r];
    else if (mode == IN_POOL) {  // source (Y, X) on the 2h x 2w grid
      const int Y = (int)(r / (2 * w)), X = (int)(r % (2 * w));
      v = 0.25f * d[(size_t)(Y >> 1) * w + (X >> 1)];
    } else {  // IN_UP: source (Y, X) on the h/2 x w/2 grid gathers its 4 children
      const int w2 = w / 2;
      const int Y = (int)(r / w2), X = (int)(r % w2);
      const float* c = d + (size_t)(2 * Y) * w + 2 * X;
      v = (c[0] + c[1]) + (c[w] + c[w + 1]);
    }
    dsrc[k] += v;
  }
}

// dW and db partials.  dW[co][ci][t] = sum over samples and pixels of
// G[co](p) Xin[ci](p + shift t), db[co] = sum of G[co]: a contraction over
// B h w pixels with Cout x Cin x 9 outputs.  Block j of P accumulates the
// (sample, 16 x 16 tile) items j, j + P, j + 2P, ... in registers, in that
// order; a thread owns COT output channels x one input channel x the nine
// taps and a residue class of the tile's rows, walking each row with a 3 x 3
// window of the input that gains one column per pixel (per pixel: COT + 3
// shared loads for 9 COT FMAs).  The row classes are summed at the end in a
// fixed order and the block writes its partial row [Cout Cin 9 | Cout]:
// every partial, and the fixed-order sum over P that follows, is run-to-run
// identical.
// store(k, load(k)) for k < n over the block, eight loads in flight per
// thread (all issued before any is stored), so staging a tile costs about
// n / (8 THREADS) memory latencies instead of n / THREADS.
template <typename L, typename S>
DEV void stage8(int n, L load, S store) {
  for (int base = threadIdx.x; base < n; base += 8 * THREADS) {
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = base + u * THREADS;
      v[u] = k < n ? load(k) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = base + u * THREADS;
      if (k < n) store(k, v[u]);
    }
  }
}

constexpr int kWgradRows = 592;  // P at most: four partial rows per SM
constexpr int kWgradGS = TILE * TILE + 1;                   // padded G row
constexpr int kWgradXS = ((TILE + 2) * (TILE + 2)) | 1;     // padded input plane (odd: ci spreads over banks)

struct WgradShape {
  int ncog, ot, pg;  // channel groups, threads per row class, row classes
};
__host__ __device__ inline WgradShape wgrad_shape(int cin, int cout, int cot) {
  WgradShape s;
  s.ncog = (cout + cot - 1) / cot;
  s.ot = s.ncog * cin;
  s.pg = THREADS / s.ot < TILE ? THREADS / s.ot : TILE;
  return s;
}
static size_t wgrad_smem(int cin, int cout, int cot) {
  const WgradShape s = wgrad_shape(cin, cout, cot);
  const size_t stage = (size_t)s.ncog * cot * kWgradGS + (size_t)cin * kWgradXS;
  const size_t comb = (size_t)s.pg * s.ot * cot * 10;
  return (stage > comb ? stage : comb) * sizeof(float);
}
// Output channels per thread: 2 while Cout / 2 x Cin threads fit the block
// (fewer registers, four blocks per SM), else 4 (always fits: 8 x 32); 1
// for a single output channel.
static int wgrad_cot(int cin, int cout) {
  if (cout == 1) return 1;
  return wgrad_shape(cin, cout, 2).ot <= THREADS ? 2 : 4;
}
// Largest dynamic shared memory a COT instantiation is launched with.
static size_t wgrad_smem_max(int cot) {
  size_t m = 0;
  for (int ci = 1; ci <= CMAX; ++ci)
    for (int co = 1; co <= CMAX; ++co)
      if (wgrad_cot(ci, co) == cot) m = std::max(m, wgrad_smem(ci, co, cot));
  return m;
}

template <int COT>
__global__ void __launch_bounds__(THREADS)
conv_wgrad_kernel(const float* __restrict__ in, int mode, int cin, const float* __restrict__ g, int cout, int h,
                  int w, int batch, float* __restrict__ part) {
  extern __shared__ float wsm[];
  const WgradShape S = wgrad_shape(cin, cout, COT);
  const int coutp = S.ncog * COT;
  float* gs = wsm;                          // [coutp][kWgradGS]
  float* xs = wsm + (size_t)coutp * kWgradGS;  // [cin][kWgradXS], (TILE+2)^2 used
  const int tid = threadIdx.x;
  const int pg = tid / S.ot, r = tid - pg * S.ot;
  const int cog = r / cin, ci = r - cog * cin;
  const bool act = pg < S.pg;
  float acc[COT][9], accb[COT];
#pragma unroll
  for (int j = 0; j < COT; ++j) {
    accb[j] = 0.f;
#pragma unroll
    for (int t = 0; t < 9; ++t) acc[j][t] = 0.f;
  }
  const int tx = (w + TILE - 1) / TILE, ty = (h + TILE - 1) / TILE;
  const int nitems = tx * ty * batch;
  const size_t plane = (size_t)h * w, sp = src_plane(mode, h, w);
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int b = it / (tx * ty), rr = it - b * (tx * ty);
    const int y0 = (rr / tx) * TILE, x0 = (rr - (rr / tx) * tx) * TILE;
    __syncthreads();  // the previous item's reads are done
    stage8(
        coutp * TILE * TILE,
        [&](int k) {
          const int co = k / (TILE * TILE), p = k - co * (TILE * TILE);
          const int y = y0 + p / TILE, x = x0 + p % TILE;
          return (co < cout && y < h && x < w) ? g[((size_t)b * cout + co) * plane + (size_t)y * w + x] : 0.f;
        },
        [&](int k, float v) { gs[(k / (TILE * TILE)) * kWgradGS + k % (TILE * TILE)] = v; });
    const float* inb = in + (size_t)b * cin * sp;
    stage8(
        cin * (TILE + 2) * (TILE + 2),
        [&](int k) {
          const int c = k / ((TILE + 2) * (TILE + 2)), q = k - c * ((TILE + 2) * (TILE + 2));
          const int ly = q / (TILE + 2), lx = q - ly * (TILE + 2);
          return in_at(inb + c * sp, mode, h, w, y0 - 1 + ly, x0 - 1 + lx);
        },
        [&](int k, float v) {
          const int c = k / ((TILE + 2) * (TILE + 2));
          xs[c * kWgradXS + (k - c * ((TILE + 2) * (TILE + 2)))] = v;
        });
    __syncthreads();
    if (act) {
      const float* gp = gs + (size_t)cog * COT * kWgradGS;
      const float* xp = xs + (size_t)ci * kWgradXS;
      for (int py = pg; py < TILE; py += S.pg) {
        // window columns c0, c1 (and c2 loaded per pixel) of rows py .. py+2
        const float* xr = xp + py * (TILE + 2);
        float a0 = xr[0], a1 = xr[TILE + 2], a2 = xr[2 * (TILE + 2)];
        float b0 = xr[1], b1 = xr[TILE + 3], b2 = xr[2 * (TILE + 2) + 1];
#pragma unroll 4
        for (int px = 0; px < TILE; ++px) {
          const float c0 = xr[px + 2], c1 = xr[TILE + 2 + px + 2], c2 = xr[2 * (TILE + 2) + px + 2];
#pragma unroll
          for (int j = 0; j < COT; ++j) {
            const float gv = gp[j * kWgradGS + py * TILE + px];
            acc[j][0] = fmaf(gv, a0, acc[j][0]);
            acc[j][1] = fmaf(gv, b0, acc[j][1]);
            acc[j][2] = fmaf(gv, c0, acc[j][2]);
            acc[j][3] = fmaf(gv, a1, acc[j][3]);
            acc[j][4] = fmaf(gv, b1, acc[j][4]);
            acc[j][5] = fmaf(gv, c1, acc[j][5]);
            acc[j][6] = fmaf(gv, a2, acc[j][6]);
            acc[j][7] = fmaf(gv, b2, acc[j][7]);
            acc[j][8] = fmaf(gv, c2, acc[j][8]);
            accb[j] += gv;
          }
          a0 = b0; a1 = b1; a2 = b2;
          b0 = c0; b1 = c1; b2 = c2;
        }
      }
    }
  }
  // row classes summed in a fixed order through shared memory
  __syncthreads();
  float* comb = wsm;  // [pg][ot][COT * 10]
  if (act) {
    float* c = comb + ((size_t)pg * S.ot + r) * (COT * 10);
#pragma unroll
    for (int j = 0; j < COT; ++j) {
#pragma unroll
      for (int t = 0; t < 9; ++t) c[j * 10 + t] = acc[j][t];
      c[j * 10 + 9] = accb[j];
    }
  }
  __syncthreads();
  if (tid < S.ot) {
    float* row = part + (size_t)blockIdx.x * ((size_t)cout * cin * 9 + cout);
    for (int j = 0; j < COT; ++j) {
      const int co = cog * COT + j;
      if (co >= cout) break;
      for (int t = 0; t < 10; ++t) {
        float s = 0.f;
        for (int q = 0; q < S.pg; ++q) s += comb[((size_t)q * S.ot + r) * (COT * 10) + j * 10 + t];
        if (t < 9) row[((size_t)co * cin + ci) * 9 + t] = s;
        else if (ci == 0) row[(size_t)cout * cin * 9 + co] = s;
      }
    }
  }
}

// Sum of the P partial rows (fixed order) into dW (the first nw entries of
// a row) and db (the rest): a block per 32 consecutive entries, its eight
// warps taking the rows in residue classes mod 8, then the eight class sums
// in order.
__global__ void __launch_bounds__(256)
reduce_rows_kernel(const float* __restrict__ part, int nrows, int len, int nw, float* dw, float* db) {
  __shared__ float sh[8][32];
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int k = blockIdx.x * 32 + lane;
  float s = 0.f;
  if (k < len)
    for (int j = wq; j < nrows; j += 8) s += part[(size_t)j * len + k];
  sh[wq][lane] = s;
  __syncthreads();
  if (wq == 0 && k < len) {
    float t = sh[0][lane];
#pragma unroll
    for (int q = 1; q < 8; ++q) t += sh[q][lane];
    if (k < nw) dw[k] = t;
    else db[k - nw] = t;
  }
}

// L = sum(mask * (pred - target)^2) / sum(mask); dpred = 2 mask (pred - target) / sum(mask)
// (mask of sample b at mask + b * mstride)
__global__ void mse_kernel(const float* pred, const float* target, const float* mask, size_t mstride, size_t plane,
                           int batch, float* dpred, double* loss_acc, double msum) {
  double acc = 0.0;
  const size_t n = plane * batch;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const size_t b = k / plane;
    const float m = mask ? mask[b * mstride + (k - b * plane)] : 1.f;
    const float d = (pred[k] - target[k]) * m;
    dpred[k] = (float)(2.0 * d / msum);
    acc += (double)d * d;
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss_acc, acc / msum);
}

// Adam (Kingma & Ba 2015) on FP32 master weights, refreshing the BF16 copy.
__global__ void adam_kernel(float* wgt, __nv_bfloat16* wb, const float* grad, float* m, float* v, int n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float g = grad[k];
    const float mk = b1 * m[k] + (1.f - b1) * g;
    const float vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    const float wk = wgt[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    wgt[k] = wk;
    if (wb) wb[k] = __float2bfloat16_rn(wk);
  }
}

__global__ void to_bf16_kernel(const float* src, __nv_bfloat16* dst, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    dst[k] = __float2bfloat16_rn(src[k]);
}

static int blocks_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace nn
}  // namespace fvx

using namespace fvx;
using namespace fvx::nn;

template <int COUT, typename WT>
static int launch_conv_batch(const float* in, int mode, int batch, int cin, const WT* wt, const float* bias,
                             const float* skip, float* out, int h, int w, int relu, cudaStream_t st,
                             int amode = -1) {
  static fvx_once_per_device attr;  // per instantiation; 32 input channels need > 48 KB
  if (fvx_once_on_device(attr, [] {
        return fvx_set_max_smem(conv_batch_kernel<COUT, WT>, (int)bc_smem<COUT>(CMAX, true));
      }))
    return FVX_ERR_CUDA;
  const dim3 g((w + kBcTW - 1) / kBcTW, (h + BcCfg<COUT>::TH - 1) / BcCfg<COUT>::TH, batch);
  conv_batch_kernel<COUT, WT><<<g, THREADS, bc_smem<COUT>(cin, amode >= 0), st>>>(in, mode, cin, wt, bias, skip, out,
                                                                                  h, w, relu, amode);
  return fvx_cuda_status();
}
// Training batches (several samples, grids of 32 x 32 and up) take the
// register-blocked batch kernel; single samples (inference) the tile kernels.
static bool conv_batch_ok(int batch, int h, int w, int cout) {
  return batch > 1 && h >= 32 && w >= 32 && (cout == 16 || cout == 32);
}

// One conv layer; pdl: launched as a programmatic dependent of the kernel
// before it, which must not have written the weights or biases (the kernel
// reads them before waiting for it).
static int conv_fwd(const float* in, int mode, int batch, int cin, const void* w_bf16, const float* bias,
                    const float* skip, float* out, int cout, int h, int w, int relu, cudaStream_t st, bool pdl,
                    ConvHooks hk = ConvHooks{}) {
  if (!in || !w_bf16 || !bias || !out) return FVX_ERR_ARG;
  if (cin < 1 || cin > CMAX || batch < 1 || h < 1 || w < 1 || mode < 0 || mode > 2) return FVX_ERR_SHAPE;
  if ((mode == IN_UP) && ((h % 2) || (w % 2))) return FVX_ERR_SHAPE;
  const __nv_bfloat16* wb = (const __nv_bfloat16*)w_bf16;
  if (!pdl && !hk.x0_src && !hk.scale && !hk.out_mask && conv_batch_ok(batch, h, w, cout))
    return cout == 16 ? launch_conv_batch<16>(in, mode, batch, cin, wb, bias, skip, out, h, w, relu, st)
                      : launch_conv_batch<32>(in, mode, batch, cin, wb, bias, skip, out, h, w, relu, st);
  // 8 x 8 tiles with 4 or 8 output channels per thread while that gives at
  // least one block per SM; else 4 x 4 tiles with 1 or 2 channels per
  // thread (256 threads, 4-8x the blocks) for the coarse levels
  const bool big = (size_t)((h + 7) / 8) * ((w + 7) / 8) * batch >= 148;
  switch (cout) {
    case 1:
      return big ? launch_conv_tile<1, 1, 8>(in, mode, batch, cin, wb, bias, skip, out, h, w, relu, st, pdl, hk)
                 : launch_conv_tile<1, 1, 4>(in, mode, batch, cin, wb, bias, skip, out, h, w, relu, st, pdl, hk);
    case 16:
      return big ? launch_conv_tile<16, 4, 8>(in, mode, batch, cin, wb, bias, skip, out, h, w, relu, st, pdl, hk)
                 : launch_conv_tile<16, 1, 4>(in, mode, batch, cin, wb, bias, skip, out, h, w, relu, st, pdl, hk);
    case 32:
      return big ? launch_conv_tile<32, 8, 8>(in, mode, batch, cin, wb, bias, skip, out, h, w, relu, st, pdl, hk)
                 : launch_conv_tile<32, 2, 4>(in, mode, batch, cin, wb, bias, skip, out, h, w, relu, st, pdl, hk);
    default: return FVX_ERR_SHAPE;
  }
}

extern "C" int fvx_nn_conv_fwd(const float* in, int mode, int batch, int cin, const void* w_bf16, const float* bias,
                               const float* skip, float* out, int cout, int h, int w, int relu, void* stream) {
  return conv_fwd(in, mode, batch, cin, w_bf16, bias, skip, out, cout, h, w, relu, fvx_stream(stream), false);
}

// Backward of one conv layer (wb: the BF16 weights of the forward pass).
// dy: dL/dy (post-activation); y: the layer's output (for the ReLU mask).  Writes g (scratch [B, Cout, h, w]), adds the
// skip gradient into dskip (if non-null), adds the input gradient into
// dsrc (if non-null; dxin scratch [B, Cin, h, w]), and writes dW, db.
// part: scratch of nblocks * Cout * (Cin * 9 + 1) floats.
extern "C" int fvx_nn_conv_bwd_blocks(int batch, int h, int w);
extern "C" int fvx_nn_conv_bwd(const float* in, int mode, int batch, int cin, const void* wb, const float* dy,
                               const float* y, int cout, int h, int w, int relu, float* g, float* dskip, float* dxin,
                               float* dsrc, float* dw, float* db, float* part, void* stream) {
  if (!in || !wb || !dy || !y || !g || !dw || !db || !part) return FVX_ERR_ARG;
  const __nv_bfloat16* wf = (const __nv_bfloat16*)wb;
  if (cin < 1 || cin > CMAX || cout < 1 || cout > CMAX) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  const size_t n = (size_t)batch * cout * h * w;
  act_grad_kernel<<<blocks_for(n), 256, 0, st>>>(dy, y, g, dskip, n, relu);
  dim3 gr((w + TILE - 1) / TILE, (h + TILE - 1) / TILE, batch);
  // weight and bias gradients: P partial rows, then their fixed-order sum
  static fvx_once_per_device attr;
  if (fvx_once_on_device(attr, [] {
        return fvx_set_max_smem(conv_wgrad_kernel<4>, (int)wgrad_smem_max(4)) &&
               fvx_set_max_smem(conv_wgrad_kernel<2>, (int)wgrad_smem_max(2)) &&
               fvx_set_max_smem(conv_wgrad_kernel<1>, (int)wgrad_smem_max(1));
      }))
    return FVX_ERR_CUDA;
  const int nrows = fvx_nn_conv_bwd_blocks(batch, h, w);
  const int cot = wgrad_cot(cin, cout);
  const size_t wsm = wgrad_smem(cin, cout, cot);
  if (cot == 4) conv_wgrad_kernel<4><<<nrows, THREADS, wsm, st>>>(in, mode, cin, g, cout, h, w, batch, part);
  else if (cot == 2) conv_wgrad_kernel<2><<<nrows, THREADS, wsm, st>>>(in, mode, cin, g, cout, h, w, batch, part);
  else conv_wgrad_kernel<1><<<nrows, THREADS, wsm, st>>>(in, mode, cin, g, cout, h, w, batch, part);
  const int len = cout * (cin * 9 + 1);
  reduce_rows_kernel<<<(len + 31) / 32, 256, 0, st>>>(part, nrows, len, cout * cin * 9, dw, db);
  if (dsrc) {
    if (!dxin) return FVX_ERR_ARG;
    if (conv_batch_ok(batch, h, w, cin) && (mode != IN_UP || ((h | w) & 1) == 0)) {
      // the data gradient as a convolution of G with the transposed,
      // flipped weights (staged in the partial-row scratch, whose sum is
      // done), its epilogue adding T^T dX into dsrc (no dX tensor)
      flip_transpose_kernel<<<blocks_for((size_t)cin * cout * 9), 256, 0, st>>>(wf, cin, cout, part);
      const int rc = cin == 16 ? launch_conv_batch<16>(g, IN_DIRECT, batch, cout, (const float*)part, nullptr, nullptr,
                                                        dsrc, h, w, 0, st, mode)
                               : launch_conv_batch<32>(g, IN_DIRECT, batch, cout, (const float*)part, nullptr, nullptr,
                                                        dsrc, h, w, 0, st, mode);
      if (rc) return rc;
    } else {
      switch (cin) {
        case 1: conv_bwd_data_kernel<1><<<gr, THREADS, 0, st>>>(g, cout, wf, dxin, h, w); break;
        case 2: conv_bwd_data_kernel<2><<<gr, THREADS, 0, st>>>(g, cout, wf, dxin, h, w); break;
        case 3: conv_bwd_data_kernel<3><<<gr, THREADS, 0, st>>>(g, cout, wf, dxin, h, w); break;
        case 16: conv_bwd_data_kernel<16><<<gr, THREADS, 0, st>>>(g, cout, wf, dxin, h, w); break;
        case 32: conv_bwd_data_kernel<32><<<gr, THREADS, 0, st>>>(g, cout, wf, dxin, h, w); break;
        default: return FVX_ERR_SHAPE;
      }
      const size_t sp = src_plane(mode, h, w);
      in_adjoint_kernel<<<blocks_for((size_t)batch * cin * sp), 256, 0, st>>>(dxin, dsrc, mode, batch * cin, h, w);
    }
  }
  return fvx_cuda_status();
}

// Number of partial rows a conv_bwd call writes (scratch sizing): one per
// (sample, 16 x 16 tile) item, at most kWgradRows.
extern "C" int fvx_nn_conv_bwd_blocks(int batch, int h, int w) {
  const long long items = (long long)((w + TILE - 1) / TILE) * ((h + TILE - 1) / TILE) * batch;
  return (int)(items < kWgradRows ? (items < 1 ? 1 : items) : kWgradRows);
}

extern "C" int fvx_nn_mse(const float* pred, const float* target, const float* mask, long long plane, int batch,
                          float* dpred, double* loss_dev, double mask_sum, void* stream) {
  if (!pred || !target || !dpred || !loss_dev || mask_sum <= 0) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  cudaMemsetAsync(loss_dev, 0, sizeof(double), st);
  mse_kernel<<<blocks_for((size_t)plane * batch), 256, 0, st>>>(pred, target, mask, 0, (size_t)plane, batch, dpred,
                                                                 loss_dev, mask_sum);
  return fvx_cuda_status();
}

extern "C" int fvx_nn_adam(float* w, void* w_bf16, const float* grad, float* m, float* v, int n, double lr,
                           double beta1, double beta2, double eps, int step, void* stream) {
  if (!w || !grad || !m || !v || n < 0 || step < 1) return FVX_ERR_ARG;
  const float c1 = (float)(1.0 - pow(beta1, step)), c2 = (float)(1.0 - pow(beta2, step));
  adam_kernel<<<blocks_for((size_t)n), 256, 0, fvx_stream(stream)>>>(w, (__nv_bfloat16*)w_bf16, grad, m, v, n,
                                                                      (float)lr, (float)beta1, (float)beta2,
                                                                      (float)eps, c1, c2);
  return fvx_cuda_status();
}

extern "C" int fvx_nn_to_bf16(const float* src, void* dst, int n, void* stream) {
  if (!src || !dst || n < 0) return FVX_ERR_ARG;
  to_bf16_kernel<<<blocks_for((size_t)n), 256, 0, fvx_stream(stream)>>>(src, (__nv_bfloat16*)dst, n);
  return fvx_cuda_status();
}

// ===========================================================================
// The network object: parameters, Adam state, activations and scratch for up
// to batch_max samples on an h x w grid (h, w multiples of 8).
//
//   x  [B, 3, h, w]      input: f / s, level mask, log coefficient
//   E0 conv 3->16, ReLU                       a0 [16, h]
//   E1 pool, conv 16->16, ReLU                a1 [16, h/2]
//   E2 pool, conv 16->32, ReLU                a2 [32, h/4]
//   E3 pool, conv 32->32, ReLU                a3 [32, h/8]
//   D2 upsample a3, conv 32->32, + a2, ReLU   a4 [32, h/4]
//   D1 upsample a4, conv 32->16, + a1, ReLU   a5 [16, h/2]
//   D0 upsample a5, conv 16->16, + a0, ReLU   a6 [16, h]
//   OUT conv 16->1, linear                    y  [1, h]
//
// Parameters are one flat FP32 vector (layer by layer: W[Cout][Cin][3][3]
// then b[Cout]); the forward pass uses its BF16 copy.
// ===========================================================================
namespace fvx {
namespace nn {

struct LayerDef {
  int cin, cout, mode, in, skip, out, div, relu;
};
// activation slots: 0 x, 1 a0, 2 a1, 3 a2, 4 a3, 5 a4, 6 a5, 7 a6, 8 y
constexpr int kSlots = 9;
constexpr int kSlotC[kSlots] = {3, 16, 16, 32, 32, 32, 16, 16, 1};
constexpr int kSlotDiv[kSlots] = {0, 0, 1, 2, 3, 2, 1, 0, 0};
constexpr int kLayers = 8;
constexpr LayerDef kNet[kLayers] = {
    {3, 16, IN_DIRECT, 0, -1, 1, 0, 1},  {16, 16, IN_POOL, 1, -1, 2, 1, 1}, {16, 32, IN_POOL, 2, -1, 3, 2, 1},
    {32, 32, IN_POOL, 3, -1, 4, 3, 1},   {32, 32, IN_UP, 4, 3, 5, 2, 1},    {32, 16, IN_UP, 5, 2, 6, 1, 1},
    {16, 16, IN_UP, 6, 1, 7, 0, 1},      {16, 1, IN_DIRECT, 7, -1, 8, 0, 0},
};

static size_t layer_params(const LayerDef& L) { return (size_t)L.cout * L.cin * 9 + L.cout; }
static size_t total_params() {
  size_t n = 0;
  for (const LayerDef& L : kNet) n += layer_params(L);
  return n;
}

constexpr int kRmsThreads = 1024;
// s = sqrt(sum(f^2 m) / max(sum m, 1)), stored as [s, 1/s] (1/s = 0 when
// s = 0), by one block (the coarse level has tens of thousands of cells):
// FP64 partial sums per thread, then a fixed-order tree, so the result is
// deterministic.  Launched as a programmatic dependent of the kernel that
// wrote f (read after the wait, through L2).
__global__ void __launch_bounds__(kRmsThreads) rms_kernel(const float* f, const float* mask, size_t n,
                                                          float* scale) {
  __shared__ double sh[2][kRmsThreads / 32];
  double a = 0.0, c = 0.0;
  grid_dep_wait();
  // eight cells' loads in flight per thread before they are accumulated (in
  // the same order as a one-at-a-time loop)
  for (size_t k0 = threadIdx.x; k0 < n; k0 += 8 * kRmsThreads) {
    float fv[8], mv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const size_t k = k0 + (size_t)u * kRmsThreads;
      fv[u] = k < n ? __ldcg(f + k) : 0.f;
      mv[u] = k < n ? mask[k] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const double m = mv[u];
      a += (double)fv[u] * fv[u] * m;
      c += m;
    }
  }
  grid_dep_launch();  // the first layer may stage its weights
  for (int o = 16; o; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = a; sh[1][threadIdx.x >> 5] = c; }
  __syncthreads();
  if (threadIdx.x < 32) {
    a = sh[0][threadIdx.x];
    c = sh[1][threadIdx.x];
    for (int o = 16; o; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (threadIdx.x == 0) {
      const double s = sqrt(a / (c > 1.0 ? c : 1.0));
      scale[0] = (float)s;
      scale[1] = s > 0.0 ? (float)(1.0 / s) : 0.f;
    }
  }
}

// ---- single-launch inference -----------------------------------------------
// The whole coarse solve -- the RMS s of f over wet cells, the eight conv
// layers, the output scaling -- as one cooperative launch of one CTA per SM.
// Every layer's weights are staged in shared memory once, while the RMS
// partial sums run; the layers are phases separated by grid barriers.  A
// layer's activations go to the same slots as in the layer-by-layer pass and
// are read back through L2 only (ld.global.cg), so no SM sees a stale L1
// line of a tensor another SM wrote in the same launch.  Each output is
// summed in the same order as conv_tile_kernel (input channels outer, taps
// inner, one fmaf chain per output channel).
constexpr int kInferThreads = 512;
constexpr int kWeightFloats = 3 * 9 * 16 + 16 * 9 * 16 + 16 * 9 * 32 + 32 * 9 * 32 + 32 * 9 * 32 + 32 * 9 * 16 +
                              16 * 9 * 16 + 16 * 9 * 1;
constexpr int kTileFloats = 8 * 16 * 10 * 10;  // largest phase: OUT, 8 tiles of 16 x 10 x 10
constexpr int kInferSmem = (kWeightFloats + kTileFloats) * (int)sizeof(float);

struct InferArgs {
  const float* f;        // right-hand side at the level [h, w]
  float* u;              // output [h, w]
  const float* x;        // input slot: channel 1 mask, channel 2 log c (channel 0 formed from f)
  float* act[kSlots];
  const __nv_bfloat16* wb;          // all BF16 weights, layer by layer (with the biases' gaps)
  const float* B[kLayers];          // each layer's FP32 biases
  const float* mask;
  float* scale;          // [s, 1/s] (written for inspection)
  double* part;          // RMS partials [gridDim.x][2]
  unsigned* bar;         // [0] arrivals, [1] generation
  int* err;              // set when a barrier wait ran out
  long long wait_cycles;
  int stall;             // CTA 0 never arrives at the first barrier (the timeout test)
  float sigma;
  int h, w;
};

DEV unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Returns true once every CTA of the grid has arrived (their global writes
// before the barrier visible to all); false when the wait ran past `limit`
// SM cycles, after raising the error flag: the CTA must return.  The last
// CTA to arrive resets the arrival count and advances the generation word,
// so the state is ready for the next barrier and the next launch.
DEV bool grid_barrier(unsigned* bar, int* err, long long limit) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = ld_acquire_u32(bar + 1);  // cannot advance before this CTA arrives
    __threadfence();
    int ok = 1;
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const long long t0 = clock64();
      while (ld_acquire_u32(bar + 1) == g) {
        if (clock64() - t0 > limit) {
          ok = 0;
          atomicExch(err, 1);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// in_at through L2 only (the source may have been written in this launch).
template <int MODE>
DEV float in_at_cg(const float* src, int h, int w, int y, int x) {
  if (y < 0 || y >= h || x < 0 || x >= w) return 0.f;
  if constexpr (MODE == IN_DIRECT) return __ldcg(src + (size_t)y * w + x);
  if constexpr (MODE == IN_POOL) {
    const int W2 = 2 * w;
    const float* p = src + (size_t)(2 * y) * W2 + 2 * x;
    return 0.25f * ((__ldcg(p) + __ldcg(p + 1)) + (__ldcg(p + W2) + __ldcg(p + W2 + 1)));
  }
  return __ldcg(src + (size_t)(y >> 1) * (w >> 1) + (x >> 1));
}

// One conv layer over the whole grid: T x T output tiles, COUT / CPT
// threads per pixel (CPT output channels each), kInferThreads / (T T COUT /
// CPT) tiles per CTA pass; ws: the layer's weights in shared memory as
// [cin * 9][COUT].  x0_src / out_mask: the first and last layers' hooks of
// conv_tile_kernel (input channel 0 = x0_src * x0s; output (y * os) *
// out_mask).
template <int MODE, int COUT, int CPT, int T>
DEV void infer_conv(const float* in, int cin, const float* ws, const float* __restrict__ bias, const float* skip,
                    float* out, int h, int w, int relu, const float* x0_src, float x0s,
                    const float* __restrict__ out_mask, float os, float* tile) {
  constexpr int NT = kInferThreads, TW = T + 2, GROUPS = COUT / CPT, TPT = T * T * GROUPS;
  static_assert(COUT % CPT == 0 && NT % TPT == 0, "tile threads must divide the block");
  constexpr int TPI = NT / TPT;
  constexpr int U = 8;  // loads in flight per thread while a tile is staged
  const int tid = threadIdx.x;
  const int per = cin * TW * TW, tot = TPI * per;
  const int tx_n = (w + T - 1) / T, ntiles = tx_n * ((h + T - 1) / T);
  const size_t sp = src_plane(MODE, h, w);
  const int slot = tid / TPT, r = tid - slot * TPT;
  const int p = r % (T * T), co0 = (r / (T * T)) * CPT;
  const int ty = p / T, tx = p % T;
  const size_t plane = (size_t)h * w;
  for (int t0 = blockIdx.x * TPI; t0 < ntiles; t0 += gridDim.x * TPI) {
    __syncthreads();  // the previous pass is done with the tiles
    for (int k0 = tid; k0 < tot; k0 += U * NT) {
      float v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u * NT;
        const int s = k / per, kk = k - s * per;
        const int tt = t0 + s;
        v[u] = 0.f;
        if (k < tot && tt < ntiles) {
          const int ci = kk / (TW * TW), rr = kk - ci * (TW * TW);
          const int ly = rr / TW, lx = rr - ly * TW;
          const int gy = (tt / tx_n) * T - 1 + ly, gx = (tt % tx_n) * T - 1 + lx;
          v[u] = (x0_src && ci == 0) ? in_at_cg<MODE>(x0_src, h, w, gy, gx) * x0s
                                     : in_at_cg<MODE>(in + ci * sp, h, w, gy, gx);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (k0 + u * NT < tot) tile[k0 + u * NT] = v[u];
    }
    __syncthreads();
    const int tt = t0 + slot;
    if (tt >= ntiles) continue;
    const int y = (tt / tx_n) * T + ty, x = (tt % tx_n) * T + tx;
    const float* tb = tile + slot * per;
    float acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.f;
    for (int ci = 0; ci < cin; ++ci) {
      const float* tl = tb + ci * TW * TW + ty * TW + tx;
      const float* wc = ws + ci * 9 * COUT + co0;
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const float v = tl[(t / 3) * TW + t % 3];
        const float* wr = wc + t * COUT;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = fmaf(wr[c], v, acc[c]);
      }
    }
    if (y >= h || x >= w) continue;
    const size_t base = (size_t)y * w + x;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int co = co0 + c;
      float v = acc[c] + bias[co];
      if (skip) v += __ldcg(skip + base + co * plane);
      if (relu) v = fmaxf(v, 0.f);
      if (out_mask) v = (v * os) * out_mask[base];
      out[base + co * plane] = v;
    }
  }
}

static_assert(kNet[0].cin == 3 && kNet[1].cin == 16 && kNet[2].cin == 16 && kNet[3].cin == 32 &&
                  kNet[4].cin == 32 && kNet[5].cin == 32 && kNet[6].cin == 16 && kNet[7].cin == 16 &&
                  kNet[0].cout == 16 && kNet[1].cout == 16 && kNet[2].cout == 32 && kNet[3].cout == 32 &&
                  kNet[4].cout == 32 && kNet[5].cout == 16 && kNet[6].cout == 16 && kNet[7].cout == 1,
              "unet_infer_kernel's layer table follows kNet");

__global__ void __launch_bounds__(kInferThreads, 1) unet_infer_kernel(InferArgs a) {
  extern __shared__ __align__(16) float ism[];
  __shared__ double red[2][kInferThreads / 32];
  __shared__ float sc[2];
  float* tile = ism + kWeightFloats;
  const int h = a.h, w = a.w;
  const size_t plane = (size_t)h * w;
  // every layer's weights, [cin * 9][cout] per layer: coalesced BF16 reads
  // (8 in flight per thread), transposed as they are stored
  {
    constexpr int kCin[kLayers] = {3, 16, 16, 32, 32, 32, 16, 16}, kCout[kLayers] = {16, 16, 32, 32, 32, 16, 16, 1};
    int wo = 0;        // shared-memory offset of the layer
    size_t go = 0;     // parameter offset of the layer
#pragma unroll
    for (int l = 0; l < kLayers; ++l) {
      const int cin = kCin[l], cout = kCout[l], k9 = cin * 9, n = cout * k9;
      for (int k0 = threadIdx.x; k0 < n; k0 += 8 * kInferThreads) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int k = k0 + u * kInferThreads;
          v[u] = k < n ? __bfloat162float(a.wb[go + k]) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int k = k0 + u * kInferThreads;  // k = co * k9 + rest
          if (k < n) {
            const int co = k / k9, rest = k - co * k9;
            ism[wo + rest * cout + co] = v[u];
          }
        }
      }
      wo += n;
      go += (size_t)n + cout;
    }
  }
  // RMS: FP64 partial sums over one contiguous chunk per CTA, then every
  // CTA adds the partials in CTA order (the same s everywhere)
  {
    const size_t chunk = (plane + gridDim.x - 1) / gridDim.x;
    const size_t c0 = (size_t)blockIdx.x * chunk, c1 = c0 + chunk < plane ? c0 + chunk : plane;
    double q2 = 0.0, cm = 0.0;
    for (size_t c = c0 + threadIdx.x; c < c1; c += kInferThreads) {
      const double m = a.mask[c], fv = a.f[c];
      q2 += fv * fv * m;
      cm += m;
    }
    for (int o = 16; o; o >>= 1) {
      q2 += __shfl_xor_sync(0xffffffffu, q2, o);
      cm += __shfl_xor_sync(0xffffffffu, cm, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = q2; red[1][threadIdx.x >> 5] = cm; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t2 = 0.0, tc = 0.0;
      for (int i = 0; i < kInferThreads / 32; ++i) { t2 += red[0][i]; tc += red[1][i]; }
      a.part[2 * blockIdx.x] = t2;
      a.part[2 * blockIdx.x + 1] = tc;
    }
  }
  if (a.stall && blockIdx.x == 0) return;  // never arrives: the others' waits run out
  if (!grid_barrier(a.bar, a.err, a.wait_cycles)) return;
  if (threadIdx.x < 32) {
    double t2 = 0.0, tc = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) {
      t2 += __ldcg(a.part + 2 * i);
      tc += __ldcg(a.part + 2 * i + 1);
    }
    for (int o = 16; o; o >>= 1) {
      t2 += __shfl_xor_sync(0xffffffffu, t2, o);
      tc += __shfl_xor_sync(0xffffffffu, tc, o);
    }
    if (threadIdx.x == 0) {
      const double s = sqrt(t2 / (tc > 1.0 ? tc : 1.0));
      sc[0] = (float)s;
      sc[1] = s > 0.0 ? (float)(1.0 / s) : 0.f;
      if (blockIdx.x == 0) { a.scale[0] = sc[0]; a.scale[1] = sc[1]; }
    }
  }
  __syncthreads();
  const float s = sc[0], rs = sc[1];
  constexpr int o0 = 0, o1 = o0 + 3 * 9 * 16, o2 = o1 + 16 * 9 * 16, o3 = o2 + 16 * 9 * 32, o4 = o3 + 32 * 9 * 32,
                o5 = o4 + 32 * 9 * 32, o6 = o5 + 32 * 9 * 16, o7 = o6 + 16 * 9 * 16;
  const long long lim = a.wait_cycles;
  infer_conv<IN_DIRECT, 16, 2, 8>(a.x, 3, ism + o0, a.B[0], nullptr, a.act[1], h, w, 1, a.f, rs, nullptr, 0.f,
                                  tile);
  if (!grid_barrier(a.bar, a.err, lim)) return;
  infer_conv<IN_POOL, 16, 1, 4>(a.act[1], 16, ism + o1, a.B[1], nullptr, a.act[2], h >> 1, w >> 1, 1, nullptr, 0.f,
                                nullptr, 0.f, tile);
  if (!grid_barrier(a.bar, a.err, lim)) return;
  infer_conv<IN_POOL, 32, 1, 4>(a.act[2], 16, ism + o2, a.B[2], nullptr, a.act[3], h >> 2, w >> 2, 1, nullptr, 0.f,
                                nullptr, 0.f, tile);
  if (!grid_barrier(a.bar, a.err, lim)) return;
  infer_conv<IN_POOL, 32, 1, 4>(a.act[3], 32, ism + o3, a.B[3], nullptr, a.act[4], h >> 3, w >> 3, 1, nullptr, 0.f,
                                nullptr, 0.f, tile);
  if (!grid_barrier(a.bar, a.err, lim)) return;
  infer_conv<IN_UP, 32, 1, 4>(a.act[4], 32, ism + o4, a.B[4], a.act[3], a.act[5], h >> 2, w >> 2, 1, nullptr, 0.f,
                              nullptr, 0.f, tile);
  if (!grid_barrier(a.bar, a.err, lim)) return;
  infer_conv<IN_UP, 16, 1, 4>(a.act[5], 32, ism + o5, a.B[5], a.act[2], a.act[6], h >> 1, w >> 1, 1, nullptr, 0.f,
                              nullptr, 0.f, tile);
  if (!grid_barrier(a.bar, a.err, lim)) return;
  infer_conv<IN_UP, 16, 2, 8>(a.act[6], 16, ism + o6, a.B[6], a.act[1], a.act[7], h, w, 1, nullptr, 0.f, nullptr,
                              0.f, tile);
  if (!grid_barrier(a.bar, a.err, lim)) return;
  infer_conv<IN_DIRECT, 1, 1, 8>(a.act[7], 16, ism + o7, a.B[7], nullptr, a.u, h, w, 0, nullptr, 0.f, a.mask,
                                 s * a.sigma, tile);
}

}  // namespace nn
}  // namespace fvx

struct fvx_unet {
  int h = 0, w = 0, batch_max = 0;
  size_t n_params = 0;
  float *wf = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16* wb = nullptr;
  float* act[kSlots] = {};   // activations, batch_max samples
  float* dact[kSlots] = {};  // their gradients (slots 1..8)
  float *g = nullptr, *dxin = nullptr, *part = nullptr;
  double* loss = nullptr;
  // inference on one field: level mask, scale [s, 1/s], output scale sigma
  float* mask = nullptr;
  float* scale = nullptr;
  float sigma = 1.f;
  // single-launch inference: grid barrier state, error flag, RMS partials
  unsigned* bar = nullptr;
  int* err = nullptr;
  double* rms_part = nullptr;
  int infer_grid = 0;
  long long wait_cycles = 4000000000LL;  // ~2 s at the boost clock
  int stall = 0;
  std::vector<void*> allocs;
};

static size_t slot_elems(const fvx_unet* n, int s, int batch) {
  const int d = kSlotDiv[s];
  return (size_t)batch * kSlotC[s] * (size_t)(n->h >> d) * (size_t)(n->w >> d);
}

static void unet_free(fvx_unet* n) {
  for (void* p : n->allocs) cudaFree(p);
  n->allocs.clear();
}

extern "C" long long fvx_unet_num_params(void) { return (long long)total_params(); }

extern "C" int fvx_unet_create(int h, int w, int batch_max, fvx_unet** out) {
  if (!out) return FVX_ERR_ARG;
  *out = nullptr;
  if (h < 8 || w < 8 || (h % 8) || (w % 8) || batch_max < 1) return FVX_ERR_SHAPE;
  fvx_unet* n = new fvx_unet();
  n->h = h; n->w = w; n->batch_max = batch_max;
  n->n_params = total_params();
  bool ok = true;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes < 16 ? 16 : bytes) != cudaSuccess) { ok = false; return nullptr; }
    n->allocs.push_back(p);
    cudaMemset(p, 0, bytes < 16 ? 16 : bytes);
    return p;
  };
  const size_t P = n->n_params;
  n->wf = (float*)alloc(P * 4);
  n->grad = (float*)alloc(P * 4);
  n->m = (float*)alloc(P * 4);
  n->v = (float*)alloc(P * 4);
  n->wb = (__nv_bfloat16*)alloc(P * 2);
  for (int s = 0; s < kSlots; ++s) {
    n->act[s] = (float*)alloc(slot_elems(n, s, batch_max) * 4);
    if (s > 0) n->dact[s] = (float*)alloc(slot_elems(n, s, batch_max) * 4);
  }
  // scratch: G [B, Cout, conv grid], dXin [B, Cin, conv grid], weight partials
  size_t gmax = 0, xmax = 0, pmax = 0;
  for (const LayerDef& L : kNet) {
    const int hh = h >> L.div, ww = w >> L.div;
    gmax = std::max(gmax, (size_t)batch_max * L.cout * hh * ww);
    xmax = std::max(xmax, (size_t)batch_max * L.cin * hh * ww);
    const size_t nblk = (size_t)fvx_nn_conv_bwd_blocks(batch_max, hh, ww);
    pmax = std::max(pmax, nblk * L.cout * ((size_t)L.cin * 9 + 1));
  }
  n->g = (float*)alloc(gmax * 4);
  n->dxin = (float*)alloc(xmax * 4);
  n->part = (float*)alloc(pmax * 4);
  n->loss = (double*)alloc(8);
  n->mask = (float*)alloc((size_t)h * w * 4);
  n->scale = (float*)alloc(16);
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      fvx_set_max_smem(unet_infer_kernel, kInferSmem) == false ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, unet_infer_kernel, kInferThreads, kInferSmem) !=
          cudaSuccess ||
      occ < 1)
    ok = false;
  n->infer_grid = sms;  // one CTA per SM: every CTA resident (cooperative launch)
  n->bar = (unsigned*)alloc(16);
  n->err = (int*)alloc(16);
  n->rms_part = (double*)alloc((size_t)2 * (sms > 0 ? sms : 1) * sizeof(double));
  if (!ok || cudaDeviceSynchronize() != cudaSuccess) {
    unet_free(n);
    delete n;
    return FVX_ERR_CUDA;
  }
  *out = n;
  return FVX_OK;
}

extern "C" int fvx_unet_destroy(fvx_unet* n) {
  if (!n) return FVX_OK;
  cudaDeviceSynchronize();
  unet_free(n);
  delete n;
  return fvx_cuda_status();
}

// Copy ``count`` floats at ``offset`` of one of the network's buffers
// (0 FP32 master parameters, 1 their gradient, 2 input x [batch_max, 3, h,
// w], 3 output y [batch_max, 1, h, w], 4 the inference scale pair [s, 1/s]
// of the last coarse solve) from ``src`` and/or to ``dst`` (host or device
// pointers; NULL skips that direction).
extern "C" int fvx_unet_io(fvx_unet* n, int which, long long offset, long long count, const void* src, void* dst,
                           void* stream) {
  if (!n || which < 0 || which > 4 || offset < 0 || count < 0) return FVX_ERR_ARG;
  float* buf = which == 0 ? n->wf : which == 1 ? n->grad : which == 2 ? n->act[0] : which == 3 ? n->act[8] : n->scale;
  const size_t len = which < 2 ? n->n_params : which == 4 ? 2 : slot_elems(n, which == 2 ? 0 : 8, n->batch_max);
  if ((size_t)(offset + count) > len) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  if (src) cudaMemcpyAsync(buf + offset, src, (size_t)count * 4, cudaMemcpyDefault, st);
  if (dst) cudaMemcpyAsync(dst, buf + offset, (size_t)count * 4, cudaMemcpyDefault, st);
  return fvx_cuda_status();
}

// Refresh the BF16 copy after the master parameters were written.
extern "C" int fvx_unet_sync_params(fvx_unet* n, void* stream) {
  if (!n) return FVX_ERR_ARG;
  return fvx_nn_to_bf16(n->wf, n->wb, (int)n->n_params, stream);
}

// pdl: each layer launched as a programmatic dependent of the kernel before
// it (inference only: no kernel between the layers writes the weights).
// coarse_f / coarse_u (inference on one field): the first layer forms
// f / s from coarse_f as it loads, the last writes s sigma m y to coarse_u.
static_assert(kNet[5].cin == 32 && kNet[5].cout == 16 && kNet[5].mode == IN_UP && kNet[5].skip == 2 &&
                  kNet[5].relu == 1 && kNet[5].div == 1 && kNet[6].cin == 16 && kNet[6].cout == 16 &&
                  kNet[6].mode == IN_UP && kNet[6].in == kNet[5].out && kNet[6].skip == 1 && kNet[6].relu == 1 &&
                  kNet[7].cin == 16 && kNet[7].cout == 1 && kNet[7].mode == IN_DIRECT && kNet[7].skip < 0 &&
                  kNet[7].relu == 0 && kNet[7].in == kNet[6].out,
              "conv_d1_d0_out_kernel computes layers 5, 6 and 7 of kNet");

static_assert(kNet[0].cin == 3 && kNet[0].cout == 16 && kNet[0].mode == IN_DIRECT && kNet[0].skip < 0 &&
                  kNet[0].relu == 1 && kNet[1].cin == 16 && kNet[1].cout == 16 && kNet[1].mode == IN_POOL &&
                  kNet[1].skip < 0 && kNet[1].relu == 1 && kNet[1].in == kNet[0].out,
              "conv_e0_e1_kernel computes layers 0 and 1 of kNet");

// coarse_u (single-field inference, batch 1): the first two layers run as
// one conv_e0_e1_kernel launch and the last three as one
// conv_d1_d0_out_kernel launch.
static int unet_forward(fvx_unet* n, int batch, cudaStream_t st, bool pdl = false, const float* coarse_f = nullptr,
                        float* coarse_u = nullptr) {
  size_t off = 0;
  int l0 = 0;
  if (coarse_u && coarse_f) {
    const LayerDef& L0 = kNet[0];
    const LayerDef& L1 = kNet[1];
    const size_t off1 = layer_params(L0);
    const dim3 g((n->w / 2) / kE1T, (n->h / 2) / kE1T);
    if (fvx_launch_pdl(conv_e0_e1_kernel, g, dim3(kE01Threads), 0, st, (const float*)n->act[0], coarse_f,
                       (const __nv_bfloat16*)n->wb, (const float*)(n->wf + (size_t)L0.cout * L0.cin * 9),
                       (const __nv_bfloat16*)(n->wb + off1), (const float*)(n->wf + off1 + (size_t)L1.cout * L1.cin * 9),
                       n->act[L0.out], n->act[L1.out], n->h, n->w, (const float*)n->scale) != cudaSuccess)
      return FVX_ERR_CUDA;
    off = off1 + layer_params(L1);
    l0 = 2;
  }
  for (int l = l0; l < kLayers; ++l) {
    const LayerDef& L = kNet[l];
    if (coarse_u && l == kLayers - 3) {
      const LayerDef& L6 = kNet[l + 1];
      const LayerDef& L7 = kNet[l + 2];
      const size_t off6 = off + layer_params(L), off7 = off6 + layer_params(L6);
      ConvHooks hk;
      hk.out_mask = n->mask;
      hk.scale = n->scale;
      hk.sigma = n->sigma;
      const dim3 g(n->w / kDT, n->h / kDT);
      if (fvx_launch_pdl(conv_d1_d0_out_kernel, g, dim3(kDThreads), 0, st, (const float*)n->act[L.in],
                         (const float*)n->act[L.skip], (const float*)n->act[L6.skip],
                         (const __nv_bfloat16*)(n->wb + off), (const float*)(n->wf + off + (size_t)L.cout * L.cin * 9),
                         (const __nv_bfloat16*)(n->wb + off6),
                         (const float*)(n->wf + off6 + (size_t)L6.cout * L6.cin * 9),
                         (const __nv_bfloat16*)(n->wb + off7),
                         (const float*)(n->wf + off7 + (size_t)L7.cout * L7.cin * 9), coarse_u, n->h, n->w,
                         hk) != cudaSuccess)
        return FVX_ERR_CUDA;
      return fvx_cuda_status();
    }
    const int hh = n->h >> L.div, ww = n->w >> L.div;
    const __nv_bfloat16* W = n->wb + off;
    const float* wf_b = n->wf + off + (size_t)L.cout * L.cin * 9;  // biases stay FP32
    ConvHooks hk;
    float* dst = n->act[L.out];
    if (coarse_f && l == 0) { hk.x0_src = coarse_f; hk.scale = n->scale; }
    if (coarse_u && l == kLayers - 1) { hk.out_mask = n->mask; hk.scale = n->scale; hk.sigma = n->sigma; dst = coarse_u; }
    int rc = conv_fwd(n->act[L.in], L.mode, batch, L.cin, W, wf_b, L.skip >= 0 ? n->act[L.skip] : nullptr, dst,
                      L.cout, hh, ww, L.relu, st, pdl, hk);
    if (rc) return rc;
    off += layer_params(L);
  }
  return FVX_OK;
}

// y = net(x) on the first ``batch`` samples of the x buffer.
extern "C" int fvx_unet_forward(fvx_unet* n, int batch, void* stream) {
  if (!n) return FVX_ERR_ARG;
  if (batch < 1 || batch > n->batch_max) return FVX_ERR_SHAPE;
  return unet_forward(n, batch, fvx_stream(stream));
}

// grad = dL/dparams given dL/dy (in the y-gradient buffer, or copied from
// ``dy`` when non-null), after a forward pass on the same batch.
static int unet_backward(fvx_unet* n, int batch, cudaStream_t st) {
  for (int s = 1; s < 8; ++s) cudaMemsetAsync(n->dact[s], 0, slot_elems(n, s, batch) * 4, st);
  size_t offs[kLayers];
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) { offs[l] = off; off += layer_params(kNet[l]); }
  for (int l = kLayers - 1; l >= 0; --l) {
    const LayerDef& L = kNet[l];
    const int hh = n->h >> L.div, ww = n->w >> L.div;
    float* dw = n->grad + offs[l];
    float* db = dw + (size_t)L.cout * L.cin * 9;
    int rc = fvx_nn_conv_bwd(n->act[L.in], L.mode, batch, L.cin, n->wb + offs[l], n->dact[L.out], n->act[L.out],
                             L.cout, hh, ww, L.relu, n->g, L.skip >= 0 ? n->dact[L.skip] : nullptr, n->dxin,
                             L.in > 0 ? n->dact[L.in] : nullptr, dw, db, n->part, st);
    if (rc) return rc;
  }
  return fvx_cuda_status();
}

extern "C" int fvx_unet_backward(fvx_unet* n, int batch, const float* dy, void* stream) {
  if (!n) return FVX_ERR_ARG;
  if (batch < 1 || batch > n->batch_max) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  if (dy) cudaMemcpyAsync(n->dact[8], dy, slot_elems(n, 8, batch) * 4, cudaMemcpyDeviceToDevice, st);
  return unet_backward(n, batch, st);
}

// One Adam step on a batch already in the x buffer:
//   L = sum_b sum_p m_b(p) (y_b(p) - target_b(p))^2 / (batch h w),
// m_b = channel 1 of x (the level mask).  loss_out (device double, may be
// NULL) receives L.
extern "C" int fvx_unet_train_step(fvx_unet* n, int batch, const float* target, double lr, double beta1,
                                   double beta2, double eps, int step, double* loss_out, void* stream) {
  if (!n || !target || step < 1) return FVX_ERR_ARG;
  if (batch < 1 || batch > n->batch_max) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  int rc = unet_forward(n, batch, st);
  if (rc) return rc;
  const size_t plane = (size_t)n->h * n->w;
  cudaMemsetAsync(n->loss, 0, sizeof(double), st);
  mse_kernel<<<blocks_for(plane * batch), 256, 0, st>>>(n->act[8], target, n->act[0] + plane, 3 * plane, plane, batch,
                                                        n->dact[8], n->loss, (double)plane * batch);
  if ((rc = unet_backward(n, batch, st))) return rc;
  if ((rc = fvx_nn_adam(n->wf, n->wb, n->grad, n->m, n->v, (int)n->n_params, lr, beta1, beta2, eps, step, st)))
    return rc;
  if (loss_out) cudaMemcpyAsync(loss_out, n->loss, sizeof(double), cudaMemcpyDeviceToDevice, st);
  return fvx_cuda_status();
}

// Inference set-up for one field: the mask and coefficient channels of x
// (sample 0), the mask applied to the output, and the output scale sigma.
extern "C" int fvx_unet_set_level(fvx_unet* n, const float* mask, const float* logc, double sigma, void* stream) {
  if (!n || !mask || !logc) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  const size_t plane = (size_t)n->h * n->w;
  cudaMemcpyAsync(n->mask, mask, plane * 4, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(n->act[0] + plane, mask, plane * 4, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(n->act[0] + 2 * plane, logc, plane * 4, cudaMemcpyDeviceToDevice, st);
  n->sigma = (float)sigma;
  return fvx_cuda_status();
}

// The coarse solve of fvx_unet_coarse in one cooperative launch
// (unet_infer_kernel).  No host synchronisation; a barrier wait that ran
// out shows in fvx_unet_check.
extern "C" int fvx_unet_coarse_fused(void* ctx, const void* f, void* u, void* stream) {
  fvx_unet* n = (fvx_unet*)ctx;
  if (!n || !f || !u) return FVX_ERR_ARG;
  InferArgs a;
  a.f = (const float*)f;
  a.u = (float*)u;
  a.x = n->act[0];
  for (int s = 0; s < kSlots; ++s) a.act[s] = n->act[s];
  a.wb = n->wb;
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    a.B[l] = n->wf + off + (size_t)kNet[l].cout * kNet[l].cin * 9;
    off += layer_params(kNet[l]);
  }
  a.mask = n->mask;
  a.scale = n->scale;
  a.part = n->rms_part;
  a.bar = n->bar;
  a.err = n->err;
  a.wait_cycles = n->wait_cycles;
  a.stall = n->stall;
  a.sigma = n->sigma;
  a.h = n->h;
  a.w = n->w;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(n->infer_grid);
  cfg.blockDim = dim3(kInferThreads);
  cfg.dynamicSmemBytes = kInferSmem;
  cfg.stream = fvx_stream(stream);
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, unet_infer_kernel, a) != cudaSuccess) return FVX_ERR_CUDA;
  return fvx_cuda_status();
}

// FVX_ERR_TIMEOUT (and the barrier state and flag cleared) when a barrier
// wait of the single-launch inference ran out since the last check.
// Synchronises the device.
extern "C" int fvx_unet_check(fvx_unet* n) {
  if (!n) return FVX_ERR_ARG;
  int e = 0;
  if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost) !=
                                                    cudaSuccess)
    return FVX_ERR_CUDA;
  if (!e) return FVX_OK;
  if (cudaMemset(n->bar, 0, 16) != cudaSuccess || cudaMemset(n->err, 0, 16) != cudaSuccess) return FVX_ERR_CUDA;
  return FVX_ERR_TIMEOUT;
}

// Bound (SM cycles) on each barrier wait of the single-launch inference.
extern "C" int fvx_unet_set_wait_limit(fvx_unet* n, long long cycles) {
  if (!n || cycles < 1) return FVX_ERR_ARG;
  n->wait_cycles = cycles;
  return FVX_OK;
}

// stall != 0: CTA 0 of the next launches never arrives at the first
// barrier, so the other CTAs' waits run out (the timeout test).
extern "C" int fvx_unet_inject_stall(fvx_unet* n, int stall) {
  if (!n) return FVX_ERR_ARG;
  n->stall = stall != 0;
  return FVX_OK;
}

// Coarse solver callback (fvx_precond_fn, ctx = the network): u = s sigma
// m net([f / s, m, log c]) with s the RMS of f over wet cells, as a chain of
// per-layer launches (the RMS kernel, then conv_tile_kernel per layer, each
// a programmatic dependent of the one before).  Launches only; no host
// synchronisation.
extern "C" int fvx_unet_coarse(void* ctx, const void* f, void* u, void* stream) {
  fvx_unet* n = (fvx_unet*)ctx;
  if (!n || !f || !u) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  const size_t plane = (size_t)n->h * n->w;
  if (fvx_launch_pdl(rms_kernel, dim3(1), dim3(kRmsThreads), 0, st, (const float*)f, (const float*)n->mask, plane,
                     n->scale) != cudaSuccess)
    return FVX_ERR_CUDA;
  // the first layer forms f / s, the last writes s sigma m y into u
  int rc = unet_forward(n, 1, st, true, (const float*)f, (float*)u);
  if (rc) return rc;
  return fvx_cuda_status();
}
