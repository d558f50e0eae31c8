// Mask2D construction on the device (mask/cartesian.py:584-739,
// mask/utils.py:42-546, mask/base.py:60-105).  Integer / boolean work only,
// so every output is bit-exact with the reference's NumPy construction.
#include "fvx_common.cuh"

namespace fvx {

DEV bool hb(const uint8_t* h, int j, int i, int ny, int nx) {
  return j >= 0 && j < ny && i >= 0 && i < nx && h[(size_t)j * nx + i] != 0;
}

// Staggered masks with the trailing-pad (positive half-step) convention:
// pool_bool thresholds 3/4 (both of two), 1/8 (any of four), 7/8 (all four)
// reduce exactly to the AND / OR forms below.  Corner wall flags, the
// 4-level classification (two cross dilations of land) and the irregular
// strict-corner flag (pool3 > 1/18  <=>  any wet strict corner in the 3x3).
__global__ void mask_build_kernel(const uint8_t* __restrict__ h, int ny, int nx, uint8_t* u, uint8_t* v,
                                  uint8_t* xy, uint8_t* xys, uint8_t* ywall, uint8_t* xwall,
                                  uint8_t* convex, uint8_t* valid, int32_t* cls, uint8_t* irr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= ny) return;
  size_t c = (size_t)j * nx + i;
  auto H = [&](int jj, int ii) { return hb(h, jj, ii, ny, nx); };
  bool uu = H(j, i) && H(j, i + 1);
  bool vv = H(j, i) && H(j + 1, i);
  bool un = H(j + 1, i) && H(j + 1, i + 1);  // u[j+1, i], zero past the last row
  bool ve = H(j, i + 1) && H(j + 1, i + 1);  // v[j, i+1], zero past the last column
  bool c4[4] = {H(j, i), H(j, i + 1), H(j + 1, i), H(j + 1, i + 1)};
  bool any4 = c4[0] || c4[1] || c4[2] || c4[3];
  bool all4 = c4[0] && c4[1] && c4[2] && c4[3];
  u[c] = uu;
  v[c] = vv;
  xy[c] = any4;
  xys[c] = all4;
  bool yw = any4 && (!uu || !un);
  bool xw = any4 && (!vv || !ve);
  ywall[c] = yw;
  xwall[c] = xw;
  convex[c] = yw && xw;
  valid[c] = any4 && uu && un && vv && ve;
  // classification: land dilated once (cross) and twice (diamond radius 2),
  // both with a zero border.
  bool wet = H(j, i);
  bool d1 = false, d2 = false;
  for (int dj = -2; dj <= 2; ++dj)
    for (int di = -2; di <= 2; ++di) {
      int r = abs(dj) + abs(di);
      if (r > 2) continue;
      int jj = j + dj, ii = i + di;
      if (jj < 0 || jj >= ny || ii < 0 || ii >= nx) continue;
      bool land = h[(size_t)jj * nx + ii] == 0;
      if (land) {
        d2 = true;
        if (r <= 1) d1 = true;
      }
    }
  int k = 0;
  if (wet && d1) k = 1;
  else if (wet && d2) k = 2;
  else if (wet) k = 3;
  cls[c] = k;
  // irregular boundary of the strict corner mask, interior cells only
  bool ir = false;
  if (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2 && !all4) {
    for (int dj = -1; dj <= 1 && !ir; ++dj)
      for (int di = -1; di <= 1; ++di) {
        int jj = j + dj, ii = i + di;
        if (H(jj, ii) && H(jj, ii + 1) && H(jj + 1, ii) && H(jj + 1, ii + 1)) { ir = true; break; }
      }
  }
  irr[c] = ir;
}

// count_contiguous (mask/utils.py:385-468): run length of wet cells starting
// at each cell, scanning one line per thread.
__global__ void count_rows_kernel(const uint8_t* __restrict__ m, int ny, int nx, int32_t* pos, int32_t* neg) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny) return;
  const uint8_t* r = m + (size_t)j * nx;
  int32_t* P = pos + (size_t)j * nx;
  int32_t* Ng = neg + (size_t)j * nx;
  int32_t run = 0;
  for (int i = nx - 1; i >= 0; --i) { run = r[i] ? run + 1 : 0; P[i] = run; }
  run = 0;
  for (int i = 0; i < nx; ++i) { run = r[i] ? run + 1 : 0; Ng[i] = run; }
}
__global__ void count_cols_kernel(const uint8_t* __restrict__ m, int ny, int nx, int32_t* pos, int32_t* neg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx) return;
  int32_t run = 0;
  for (int j = ny - 1; j >= 0; --j) { size_t c = (size_t)j * nx + i; run = m[c] ? run + 1 : 0; pos[c] = run; }
  run = 0;
  for (int j = 0; j < ny; ++j) { size_t c = (size_t)j * nx + i; run = m[c] ? run + 1 : 0; neg[c] = run; }
}

// make_sponge (mask/utils.py:471-546), float32 ramps multiplied y then x.
__global__ void sponge_kernel(float* out, int ny, int nx, float w) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= ny) return;
  float ry, rx;
  if (w <= 0.f) { ry = rx = 1.f; }
  else {
    float fj = (float)j, fi = (float)i;
    ry = fminf(fmaxf(fminf(fj, (float)(ny - 1) - fj) / w, 0.f), 1.f);
    rx = fminf(fmaxf(fminf(fi, (float)(nx - 1) - fi) / w, 0.f), 1.f);
  }
  out[(size_t)j * nx + i] = (1.0f * ry) * rx;
}

// get_adaptive_masks (mask/cartesian.py:495-553): largest stencil size s in
// ``sizes`` with pos >= s/2 and neg >= s/2, one uint8 mask per size.
__global__ void adaptive_masks_kernel(const int32_t* __restrict__ pos, const int32_t* __restrict__ neg,
                                      size_t n, const int32_t* sizes_sorted, int nsizes, uint8_t* out) {
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  int p = pos[c], q = neg[c], ms = 0;
  for (int k = 0; k < nsizes; ++k) {
    int hw = sizes_sorted[k] / 2;
    if (p >= hw && q >= hw) ms = sizes_sorted[k];
  }
  for (int k = 0; k < nsizes; ++k) out[(size_t)k * n + c] = (ms == sizes_sorted[k]);
}

// Packed advection tier codes for the (2, 4, 6) hierarchy of Advection2D
// (advection/advection.py:55, :318-324): bits 0-1 x, bits 2-3 y.
__global__ void tier_codes_kernel(const int32_t* xp, const int32_t* xn, const int32_t* yp,
                                  const int32_t* yn, size_t n, uint8_t* out) {
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  auto code = [](int p, int q) {
    int k = 0;
    if (p >= 1 && q >= 1) k = 1;
    if (p >= 2 && q >= 2) k = 2;
    if (p >= 3 && q >= 3) k = 3;
    return k;
  };
  out[c] = (uint8_t)(code(xp[c], xn[c]) | (code(yp[c], yn[c]) << 2));
}

// Row-major compaction of a flag array into (row, col) lists, preserving
// np.where order: per-row counts, one-block scan, per-row ordered writes.
__global__ void row_count_kernel(const uint8_t* f, int ny, int nx, int32_t* cnt) {
  int j = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  if (j >= ny) return;
  int s = 0;
  for (int i = lane; i < nx; i += 32) s += f[(size_t)j * nx + i] != 0;
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) cnt[j] = s;
}
__global__ void exclusive_scan_kernel(const int32_t* cnt, int n, int32_t* off, int32_t* total) {
  __shared__ int32_t part[1024];
  int t = threadIdx.x;
  int per = (n + 1023) / 1024;
  int lo = t * per, hi = min(n, lo + per);
  int s = 0;
  for (int k = lo; k < hi; ++k) s += cnt[k];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    int acc = 0;
    for (int k = 0; k < 1024; ++k) { int v = part[k]; part[k] = acc; acc += v; }
    *total = acc;
  }
  __syncthreads();
  int acc = part[t];
  for (int k = lo; k < hi; ++k) { off[k] = acc; acc += cnt[k]; }
}
__global__ void row_write_kernel(const uint8_t* f, int ny, int nx, const int32_t* off, int32_t* rows,
                                 int32_t* cols) {
  int j = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  if (j >= ny) return;
  int base = off[j];
  for (int i0 = 0; i0 < nx; i0 += 32) {
    int i = i0 + lane;
    bool flag = i < nx && f[(size_t)j * nx + i] != 0;
    unsigned b = __ballot_sync(0xffffffffu, flag);
    if (flag) {
      int p = base + __popc(b & ((1u << lane) - 1u));
      rows[p] = j;
      cols[p] = i;
    }
    base += __popc(b);
  }
}

}  // namespace fvx

using namespace fvx;

extern "C" int fvx_mask2d_build(const uint8_t* h, int ny, int nx, uint8_t* u, uint8_t* v, uint8_t* xy,
                                uint8_t* xy_strict, uint8_t* y_wall, uint8_t* x_wall, uint8_t* convex,
                                uint8_t* valid, int32_t* classification, uint8_t* irr_flag,
                                int32_t* x_pos, int32_t* x_neg, int32_t* y_pos, int32_t* y_neg,
                                float* sponge, int sponge_width, void* stream) {
  if (!h || !u || !v || !xy || !xy_strict || !y_wall || !x_wall || !convex || !valid || !classification ||
      !irr_flag || !x_pos || !x_neg || !y_pos || !y_neg)
    return FVX_ERR_ARG;
  if (ny < 1 || nx < 1) return FVX_ERR_SHAPE;
  if (sponge_width < 0) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);
  mask_build_kernel<<<g, b, 0, st>>>(h, ny, nx, u, v, xy, xy_strict, y_wall, x_wall, convex, valid,
                                     classification, irr_flag);
  count_rows_kernel<<<(ny + 127) / 128, 128, 0, st>>>(h, ny, nx, x_pos, x_neg);
  count_cols_kernel<<<(nx + 127) / 128, 128, 0, st>>>(h, ny, nx, y_pos, y_neg);
  if (sponge) sponge_kernel<<<g, b, 0, st>>>(sponge, ny, nx, (float)sponge_width);
  return fvx_cuda_status();
}

extern "C" int fvx_count_contiguous(const uint8_t* m, int ny, int nx, int axis, int32_t* pos, int32_t* neg,
                                    void* stream) {
  if (!m || !pos || !neg) return FVX_ERR_ARG;
  if (ny < 1 || nx < 1) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  if (axis == 1) count_rows_kernel<<<(ny + 127) / 128, 128, 0, st>>>(m, ny, nx, pos, neg);
  else if (axis == 0) count_cols_kernel<<<(nx + 127) / 128, 128, 0, st>>>(m, ny, nx, pos, neg);
  else return FVX_ERR_ARG;
  return fvx_cuda_status();
}

extern "C" int fvx_adaptive_masks(const int32_t* pos, const int32_t* neg, int64_t n, const int32_t* sizes_sorted,
                                  int nsizes, uint8_t* out, void* stream) {
  if (!pos || !neg || !sizes_sorted || !out) return FVX_ERR_ARG;
  if (n < 0 || nsizes < 1 || nsizes > 16) return FVX_ERR_SHAPE;
  if (n == 0) return FVX_OK;
  adaptive_masks_kernel<<<(unsigned)((n + 255) / 256), 256, 0, fvx_stream(stream)>>>(pos, neg, (size_t)n,
                                                                                      sizes_sorted, nsizes, out);
  return fvx_cuda_status();
}

extern "C" int fvx_tier_codes(const int32_t* x_pos, const int32_t* x_neg, const int32_t* y_pos,
                              const int32_t* y_neg, int64_t n, uint8_t* out, void* stream) {
  if (!x_pos || !x_neg || !y_pos || !y_neg || !out) return FVX_ERR_ARG;
  if (n < 0) return FVX_ERR_SHAPE;
  if (n == 0) return FVX_OK;
  tier_codes_kernel<<<(unsigned)((n + 255) / 256), 256, 0, fvx_stream(stream)>>>(x_pos, x_neg, y_pos, y_neg,
                                                                                  (size_t)n, out);
  return fvx_cuda_status();
}

// Compacts flags into row-major (rows, cols).  ``work`` holds 2*ny+1 int32:
// per-row counts, offsets and the total (read back by the caller to size
// the lists; rows/cols must hold ny*nx entries).
extern "C" int fvx_compact_flags(const uint8_t* flags, int ny, int nx, int32_t* work, int32_t* rows,
                                 int32_t* cols, void* stream) {
  if (!flags || !work || !rows || !cols) return FVX_ERR_ARG;
  if (ny < 1 || nx < 1) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  int32_t* cnt = work;
  int32_t* off = work + ny;
  int32_t* total = work + 2 * ny;
  row_count_kernel<<<(ny + 7) / 8, 256, 0, st>>>(flags, ny, nx, cnt);
  exclusive_scan_kernel<<<1, 1024, 0, st>>>(cnt, ny, off, total);
  row_write_kernel<<<(ny + 7) / 8, 256, 0, st>>>(flags, ny, nx, off, rows, cols);
  return fvx_cuda_status();
}
