// Ensemble of multi-layer QG models with uneven grid sizes and layer
// counts, one RK3-SSP step for every member per call.
//
// Member model (built from finitevolX's pieces; the reference has no
// multi-layer time stepper): layers k = 1..nl of PV q_k on an (n+2)^2 grid
// with one ghost ring (periodic q, Dirichlet psi), inverted through vertical
// modes -- q_m = sum_l L2M[m][l] q_l (vertical_modes.py:193-227), one DST-I
// Helmholtz solve per mode with lambda_m = 1/Rd_m^2 (elliptic.py:390-542),
// psi_k = sum_m M2L[k][m] psi_m (:230-263) -- and each layer stepped with the
// 1.5-layer tendency (advection of q_k by its geostrophic velocity plus
// beta v_k, scripts/qg_1p5_layer.py:454-487) in rk3_ssp_step
// (timestepping/explicit_rk.py:74-121).
//
// Per RK stage: for each grid-size group, one kernel mixes the layers of
// every member into modes and writes them as the split DST operand, one
// batched tensor-core DST chain solves all modes of the group (per-mode
// lambda), one kernel mixes modes back into layer streamfunctions; then ONE
// persistent launch runs the fused stage on every tile of every layer of
// every member, CTAs pulling (field, tile) items from an atomic work queue
// (largest fields first).  All launches are stream-ordered with no host
// synchronisation, so a host can capture whole steps in a CUDA graph.
#include "qg_stage.cuh"

#include <algorithm>
#include <numeric>
#include <vector>

struct fvx_dst_plan;
extern "C" int fvx_dst_plan_create(int ny, int nx, double dx, double dy, int batch_max, const double* lambdas,
                                   int n_lambda, int want_fp64, fvx_dst_plan** out);
extern "C" int fvx_dst_plan_destroy(fvx_dst_plan* p);
extern "C" int fvx_dst_solve_presplit_f32(fvx_dst_plan* p, float* psi, long long psi_bstride, long long psi_ld,
                                          int batch, void* stream);
extern "C" int fvx_dst_workspace(fvx_dst_plan* p, void** w1_hi, void** w1_lo);
extern "C" int fvx_dst_operand_layout(fvx_dst_plan* p);
extern "C" int fvx_dst_refine_f32(fvx_dst_plan* p, const float* rhs, long long rhs_bstride, long long rhs_ld,
                                  float* psi, long long psi_bstride, long long psi_ld, int batch, int passes,
                                  void* stream);

namespace fvx {
namespace ens {

constexpr int TXE = 64, TYE = 16;
constexpr int kMaxLayers = 3;
// Modes with lambda L^2 below this (deformation radius above ~L / 45) are
// weakly screened: their streamfunction is dominated by the largest scales,
// and the velocity differences amplify the split DST chain's ~1e-5 relative
// psi error past the FP32 step bar (a NumPy emulation of the chain: 5e-5 ..
// 2.6e-4 one-step q error for 64^2 .. 1024^2 members with Rd 670 km or
// lambda = 0, 2.4e-6 for Ld = 40 km in 5120 km at 2048^2).  They take the
// FP64-residual refinement pass; strongly screened modes do not need it.
constexpr double kWeakScreening = 2000.0;

struct FieldDesc {
  qg::StageArgs a[3];  // the three RK stages
  int tiles_x, tile0;  // tiles per row, first queue index
};

struct ModeDesc {      // batch entry: sum_l c[l] q_l (interior of a [n+2]^2 field)
  const float* q[kMaxLayers];
  float c[kMaxLayers];
  int nl;
};

struct LayerDesc {     // psi_k = sum_m c[m] psi_mode[b[m]]
  float* psi;
  int b[kMaxLayers];
  float c[kMaxLayers];
  int nl;
};

// Persistent fused-stage kernel over every tile of every field.  The tile's
// field arguments are read from shared memory: a register copy stays live
// across the whole tile body (WENO5: 63 registers against the single-field
// kernel's 40, four resident blocks per SM instead of six).
template <int S>
__global__ void __launch_bounds__(qg::THREADS, 6)
ens_stage_kernel(const FieldDesc* __restrict__ fields, int nfields, int stage, int total, unsigned* counter) {
  extern __shared__ __align__(16) uint8_t sm[];
  __shared__ int item;
  __shared__ qg::StageArgs sa;
  for (;;) {
    if (threadIdx.x == 0) item = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int t = item;
    __syncthreads();
    if (t >= total) break;
    int lo = 0, hi = nfields - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (fields[mid].tile0 <= t) lo = mid;
      else hi = mid - 1;
    }
    if (threadIdx.x == 0) sa = fields[lo].a[stage];
    __syncthreads();
    const qg::StageArgs& A = sa;
    const int lt = t - fields[lo].tile0;
    const int ty = lt / fields[lo].tiles_x, tx = lt - ty * fields[lo].tiles_x;
    qg::stage_tile<float, S, TXE, TYE>(A, sm, tx * TXE, ty * TYE);
    __syncthreads();
  }
}

// Layers -> modes, written split into bf16 hi/lo (x de-interleaved when
// perm) and, when fm is not null, as FP32 in natural order (the right-hand
// side of the refinement residual).  Grid (row blocks of kMixRows rows,
// modes): each block reads its mode's descriptor once.
constexpr int kMixRows = 8;
__global__ void __launch_bounds__(256)
ens_mode_split_kernel(const ModeDesc* __restrict__ md, int n, __nv_bfloat16* hi, __nv_bfloat16* lo, int perm,
                      float* __restrict__ fm) {
  const int b = blockIdx.y;
  const ModeDesc d = md[b];
  const size_t plane = (size_t)n * n;
  const int y1 = min(n, (int)(blockIdx.x + 1) * kMixRows);
  for (int y = blockIdx.x * kMixRows; y < y1; ++y) {
    const size_t grow = (size_t)(y + 1) * (n + 2) + 1, orow = (size_t)b * plane + (size_t)y * n;
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
      const size_t g = grow + x;
      float v = d.c[0] * d.q[0][g];
#pragma unroll
      for (int l = 1; l < kMaxLayers; ++l)
        if (l < d.nl) v += d.c[l] * d.q[l][g];
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      const int xs = perm ? ((x & 1) ? (n >> 1) + (x >> 1) : (x >> 1)) : x;
      hi[orow + xs] = h;
      lo[orow + xs] = __float2bfloat16_rn(v - __bfloat162float(h));
      if (fm) fm[orow + x] = v;
    }
  }
}

// Modes -> layers: psi_k = sum_m c[m] psi_mode[b[m]].  Grid (row blocks of
// kMixRows rows, layers).
__global__ void __launch_bounds__(256)
ens_layer_mix_kernel(const LayerDesc* __restrict__ ld, int n, const float* __restrict__ psim) {
  const LayerDesc d = ld[blockIdx.y];
  const size_t plane = (size_t)n * n;
  const int y1 = min(n, (int)(blockIdx.x + 1) * kMixRows);
  for (int y = blockIdx.x * kMixRows; y < y1; ++y) {
    const size_t r0 = (size_t)y * n;
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
      const size_t r = r0 + x;
      float v = d.c[0] * psim[(size_t)d.b[0] * plane + r];
#pragma unroll
      for (int m = 1; m < kMaxLayers; ++m)
        if (m < d.nl) v += d.c[m] * psim[(size_t)d.b[m] * plane + r];
      d.psi[r] = v;
    }
  }
}

}  // namespace ens
}  // namespace fvx

using namespace fvx;
using namespace fvx::ens;

struct fvx_ens {
  int method = 5;
  int refine = 1;  // FP64-residual refinement passes per DST solve
  int nm = 0, nfields = 0, total_tiles = 0, blocks = 0, grid = 0;
  size_t smem = 0;
  std::vector<int> n, nl;
  std::vector<float*> q, y1, y2, psi;  // per field (member-major, layer-minor)
  std::vector<int> field0;             // first field of each member
  struct Group {
    int n = 0, B = 0, nlay = 0;
    fvx_dst_plan* plan = nullptr;
    float* psim = nullptr;
    float* fm = nullptr;  // FP32 modes (refinement right-hand side)
    int nref = 0;         // the first nref batch entries are the weakly screened modes that take refinement
    ModeDesc* md[3] = {nullptr, nullptr, nullptr};
    LayerDesc* ld = nullptr;
    __nv_bfloat16 *hi = nullptr, *lo = nullptr;
    int perm = 0;
  };
  std::vector<Group> groups;
  // one stream per size group after the first: the groups' DST chains are
  // independent, and the small groups alone would leave most SMs idle
  std::vector<cudaStream_t> gst;
  std::vector<cudaEvent_t> gdone;
  cudaEvent_t fork = nullptr;
  FieldDesc* fd = nullptr;
  unsigned* counter = nullptr;
  std::vector<void*> allocs;
};

static void ens_free(fvx_ens* e) {
  for (auto& g : e->groups)
    if (g.plan) fvx_dst_plan_destroy(g.plan);
  for (cudaStream_t s : e->gst)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t ev : e->gdone)
    if (ev) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  e->gst.clear();
  e->gdone.clear();
  e->fork = nullptr;
  for (void* p : e->allocs) cudaFree(p);
  e->allocs.clear();
}

template <int S>
static int ens_stage_smem_and_blocks(int blocks_per_sm, int* blocks, size_t* smem) {
  *smem = qg::smem_bytes<float, S, TXE, TYE>();
  static fvx_once_per_device attr;
  const int bytes = (int)*smem;
  if (fvx_once_on_device(attr, [bytes] { return fvx_set_max_smem(ens_stage_kernel<S>, bytes); }))
    return FVX_ERR_CUDA;
  int occ = 0, dev = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ens_stage_kernel<S>, qg::THREADS, *smem) != cudaSuccess ||
      cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess)
    return FVX_ERR_CUDA;
  const int per = blocks_per_sm > 0 ? std::min(blocks_per_sm, std::max(occ, 1)) : std::max(occ, 1);
  *blocks = per * sms;
  return FVX_OK;
}

template <int S>
static int ens_stage_launch(fvx_ens* e, int stage, cudaStream_t st) {
  if (e->grid <= 0) {  // resolved once (occupancy query) per object and setting
    int rc = ens_stage_smem_and_blocks<S>(e->blocks, &e->grid, &e->smem);
    if (rc) return rc;
  }
  const int blocks = e->grid;
  const size_t smem = e->smem;
  cudaMemsetAsync(e->counter, 0, sizeof(unsigned), st);
  ens_stage_kernel<S><<<blocks, qg::THREADS, smem, st>>>(e->fd, e->nfields, stage, e->total_tiles, e->counter);
  return fvx_cuda_status();
}

static int ens_stage_dispatch(fvx_ens* e, int stage, cudaStream_t st) {
  switch (e->method) {
    case FVX_UPWIND1: return ens_stage_launch<FVX_UPWIND1>(e, stage, st);
    case FVX_WENO3: return ens_stage_launch<FVX_WENO3>(e, stage, st);
    case FVX_WENO5: return ens_stage_launch<FVX_WENO5>(e, stage, st);
    case FVX_WENOZ5: return ens_stage_launch<FVX_WENOZ5>(e, stage, st);
    case FVX_VAN_LEER: return ens_stage_launch<FVX_VAN_LEER>(e, stage, st);
    default: return FVX_ERR_METHOD;
  }
}

// n, nl: per member; l2m, m2l: per member nl*nl row-major, concatenated;
// lam: per member nl (mode lambdas); dx, dy, dt: per member.  n must be a
// multiple of 8 (the tensor-core DST).  method: 1 upwind1, 4 weno3, 5 weno5,
// 6 wenoz5, 10 van_leer.
extern "C" int fvx_ens_create(int n_members, const int* n, const int* nl, const double* l2m, const double* m2l,
                              const double* lam, const double* dx, const double* dy, const double* dt, double beta,
                              int method, fvx_ens** out) {
  if (!out || !n || !nl || !l2m || !m2l || !lam || !dx || !dy || !dt || n_members < 1) return FVX_ERR_ARG;
  *out = nullptr;
  if (method != FVX_UPWIND1 && method != FVX_WENO3 && method != FVX_WENO5 && method != FVX_WENOZ5 &&
      method != FVX_VAN_LEER)
    return FVX_ERR_METHOD;
  for (int m = 0; m < n_members; ++m)
    if (n[m] < 8 || n[m] % 8 || nl[m] < 1 || nl[m] > kMaxLayers) return FVX_ERR_SHAPE;
  fvx_ens* e = new fvx_ens();
  e->method = method;
  e->nm = n_members;
  e->n.assign(n, n + n_members);
  e->nl.assign(nl, nl + n_members);
  bool ok = true;
  auto A = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (ok && cudaMalloc(&p, bytes) == cudaSuccess) {
      e->allocs.push_back(p);
      cudaMemset(p, 0, bytes);
      return p;
    }
    ok = false;
    return nullptr;
  };
  // fields
  std::vector<int> coff(n_members + 1, 0);  // offsets into the concatenated nl*nl matrices
  for (int m = 0; m < n_members; ++m) coff[m + 1] = coff[m] + nl[m] * nl[m];
  std::vector<int> loff(n_members + 1, 0);
  for (int m = 0; m < n_members; ++m) loff[m + 1] = loff[m] + nl[m];
  for (int m = 0; m < n_members; ++m) {
    e->field0.push_back((int)e->q.size());
    const size_t full = (size_t)(n[m] + 2) * (n[m] + 2), inter = (size_t)n[m] * n[m];
    for (int k = 0; k < nl[m]; ++k) {
      e->q.push_back((float*)A(full * 4));
      e->y1.push_back((float*)A(full * 4));
      e->y2.push_back((float*)A(full * 4));
      e->psi.push_back((float*)A(inter * 4));
    }
  }
  e->nfields = (int)e->q.size();
  if (!ok) { ens_free(e); delete e; return FVX_ERR_CUDA; }
  // size groups: modes batched per grid size
  std::vector<int> sizes(e->n);
  std::sort(sizes.begin(), sizes.end());
  sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
  std::vector<std::vector<int>> batch_of(n_members);  // batch index of each member mode within its group
  for (int sz : sizes) {
    fvx_ens::Group g;
    g.n = sz;
    std::vector<double> lams;
    std::vector<ModeDesc> md[3];
    std::vector<LayerDesc> ld;
    double gdx = 0, gdy = 0;
    // batch order: the weakly screened modes (lambda L^2 < kWeakScreening,
    // L = n dx the domain width) first, so a refinement pass covers a prefix
    // of the batch; then the rest
    for (int m = 0; m < n_members; ++m)
      if (n[m] == sz) batch_of[m].assign(nl[m], -1);
    for (int pass = 0; pass < 2; ++pass)
    for (int m = 0; m < n_members; ++m) {
      if (n[m] != sz) continue;
      if (gdx == 0) { gdx = dx[m]; gdy = dy[m]; }
      if (dx[m] != gdx || dy[m] != gdy) { ens_free(e); delete e; return FVX_ERR_ARG; }  // one spacing per size
      const double L = sz * fmax(dx[m], dy[m]);
      for (int mo = 0; mo < nl[m]; ++mo) {
        const bool weak = lam[loff[m] + mo] * L * L < kWeakScreening;
        if (weak != (pass == 0)) continue;
        if (weak) ++g.nref;
        batch_of[m][mo] = g.B++;
        lams.push_back(lam[loff[m] + mo]);
        for (int s = 0; s < 3; ++s) {
          ModeDesc d{};
          d.nl = nl[m];
          for (int l = 0; l < nl[m]; ++l) {
            const int f = e->field0[m] + l;
            d.q[l] = s == 0 ? e->q[f] : (s == 1 ? e->y1[f] : e->y2[f]);
            d.c[l] = (float)l2m[coff[m] + mo * nl[m] + l];
          }
          md[s].push_back(d);
        }
      }
    }
    for (int m = 0; m < n_members; ++m) {
      if (n[m] != sz) continue;
      for (int k = 0; k < nl[m]; ++k) {
        LayerDesc d{};
        d.psi = e->psi[e->field0[m] + k];
        d.nl = nl[m];
        for (int mo = 0; mo < nl[m]; ++mo) {
          d.b[mo] = batch_of[m][mo];
          d.c[mo] = (float)m2l[coff[m] + k * nl[m] + mo];
        }
        ld.push_back(d);
      }
    }
    g.nlay = (int)ld.size();
    int rc = fvx_dst_plan_create(sz, sz, gdx, gdy, g.B, lams.data(), (int)lams.size(), 0, &g.plan);
    if (rc) { ens_free(e); delete e; return rc; }
    void *hi = nullptr, *lo = nullptr;
    if ((rc = fvx_dst_workspace(g.plan, &hi, &lo))) {
      fvx_dst_plan_destroy(g.plan);
      ens_free(e); delete e; return rc;
    }
    g.hi = (__nv_bfloat16*)hi;
    g.lo = (__nv_bfloat16*)lo;
    g.perm = fvx_dst_operand_layout(g.plan);
    g.psim = (float*)A((size_t)g.B * sz * sz * 4);
    g.fm = (float*)A((size_t)g.B * sz * sz * 4);
    for (int s = 0; s < 3; ++s) {
      g.md[s] = (ModeDesc*)A(md[s].size() * sizeof(ModeDesc));
      if (ok) cudaMemcpy(g.md[s], md[s].data(), md[s].size() * sizeof(ModeDesc), cudaMemcpyHostToDevice);
    }
    g.ld = (LayerDesc*)A(ld.size() * sizeof(LayerDesc));
    if (ok) cudaMemcpy(g.ld, ld.data(), ld.size() * sizeof(LayerDesc), cudaMemcpyHostToDevice);
    e->groups.push_back(g);
    if (!ok) { ens_free(e); delete e; return FVX_ERR_CUDA; }
  }
  // work queue: fields ordered by size (largest first), tiles numbered consecutively
  std::vector<int> order(e->nfields);
  std::iota(order.begin(), order.end(), 0);
  std::vector<int> fmember(e->nfields);
  for (int m = 0; m < n_members; ++m)
    for (int k = 0; k < nl[m]; ++k) fmember[e->field0[m] + k] = m;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[fmember[a]] > n[fmember[b]]; });
  std::vector<FieldDesc> fd(e->nfields);
  int t0 = 0;
  for (int i = 0; i < e->nfields; ++i) {
    const int f = order[i], m = fmember[f];
    const int N = n[m] + 2;
    FieldDesc d{};
    d.tiles_x = (N + TXE - 1) / TXE;
    d.tile0 = t0;
    t0 += d.tiles_x * ((N + TYE - 1) / TYE);
    const double a[3] = {0.0, 0.75, 1.0 / 3.0}, b[3] = {1.0, 0.25, 2.0 / 3.0}, c[3] = {1.0, 0.25, 2.0 / 3.0};
    const float* qs[3] = {e->q[f], e->y1[f], e->y2[f]};
    float* outp[3] = {e->y1[f], e->y2[f], e->q[f]};
    for (int s = 0; s < 3; ++s) {
      qg::StageArgs& A2 = d.a[s];
      A2 = qg::StageArgs{};
      A2.qs = qs[s];
      A2.qn = s == 0 ? nullptr : e->q[f];
      A2.psi = e->psi[f];
      A2.forcing = nullptr;
      A2.out = outp[s];
      A2.split_hi = nullptr;
      A2.split_lo = nullptr;
      A2.split_layout = 0;
      A2.ny = N; A2.nx = N;
      A2.a = a[s]; A2.b = b[s]; A2.c = c[s] * dt[m];
      A2.dx = dx[m]; A2.dy = dy[m]; A2.beta = beta;
      A2.drag = 0.0; A2.visc = 0.0;
      A2.periodic = 1;
      A2.write_ghost = s == 2 ? 1 : 0;
    }
    fd[i] = d;
  }
  e->total_tiles = t0;
  e->fd = (FieldDesc*)A(fd.size() * sizeof(FieldDesc));
  e->counter = (unsigned*)A(sizeof(unsigned));
  if (ok) cudaMemcpy(e->fd, fd.data(), fd.size() * sizeof(FieldDesc), cudaMemcpyHostToDevice);
  if (!ok || cudaDeviceSynchronize() != cudaSuccess) { ens_free(e); delete e; return FVX_ERR_CUDA; }
  *out = e;
  return FVX_OK;
}

extern "C" int fvx_ens_destroy(fvx_ens* e) {
  if (!e) return FVX_OK;
  cudaDeviceSynchronize();
  ens_free(e);
  delete e;
  return fvx_cuda_status();
}

// Copy layer ``layer`` of member ``member`` ([n+2][n+2] FP32, ghost ring
// included) from ``src`` and/or to ``dst`` (host or device pointers).
extern "C" int fvx_ens_io(fvx_ens* e, int member, int layer, const void* src, void* dst, void* stream) {
  if (!e || member < 0 || member >= e->nm || layer < 0 || layer >= e->nl[member]) return FVX_ERR_ARG;
  float* q = e->q[e->field0[member] + layer];
  const size_t bytes = (size_t)(e->n[member] + 2) * (e->n[member] + 2) * sizeof(float);
  cudaStream_t st = fvx_stream(stream);
  if (src) cudaMemcpyAsync(q, src, bytes, cudaMemcpyDefault, st);
  if (dst) cudaMemcpyAsync(dst, q, bytes, cudaMemcpyDefault, st);
  return fvx_cuda_status();
}

// Persistent stage grid: CTAs per SM (0 = as many as fit).
extern "C" int fvx_ens_set_blocks_per_sm(fvx_ens* e, int blocks_per_sm) {
  if (!e || blocks_per_sm < 0) return FVX_ERR_ARG;
  e->blocks = blocks_per_sm;
  e->grid = 0;
  return FVX_OK;
}

// Launches of one step (for the caller's launch count).
extern "C" int fvx_ens_launches_per_step(fvx_ens* e) {
  if (!e) return -1;
  // per stage: per group (mode split + 4 DST products + layer mix, plus
  // refine passes x (residual + 4 products) when the group has weakly
  // screened modes) + counter reset + stage kernel
  int per = 0;
  for (const auto& g : e->groups) per += 6 + (g.nref ? 5 * e->refine : 0);
  return 3 * (per + 2);
}

// FP64-residual refinement passes per DST solve (default 1; 0 leaves the
// split chain's ~1e-5 relative error in psi).
extern "C" int fvx_ens_set_refine(fvx_ens* e, int passes) {
  if (!e || passes < 0 || passes > 4) return FVX_ERR_ARG;
  e->refine = passes;
  return FVX_OK;
}

// n_steps RK3-SSP steps of every member.
extern "C" int fvx_ens_step(fvx_ens* e, int n_steps, void* stream) {
  if (!e || n_steps < 0) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  const int ng = (int)e->groups.size();
  if (e->gst.size() + 1 < (size_t)ng) {  // created on first use, on the caller's device
    for (int k = (int)e->gst.size(); k < ng - 1; ++k) {
      cudaStream_t s2 = nullptr;
      cudaEvent_t ev = nullptr;
      if (cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        return FVX_ERR_CUDA;
      e->gst.push_back(s2);
      e->gdone.push_back(ev);
    }
    if (!e->fork && cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) return FVX_ERR_CUDA;
  }
  for (int it = 0; it < n_steps; ++it)
    for (int s = 0; s < 3; ++s) {
      // fork: group 0 on the caller's stream, the others on their own
      if (ng > 1 && cudaEventRecord(e->fork, st) != cudaSuccess) return FVX_ERR_CUDA;
      for (int k = 0; k < ng; ++k) {
        auto& g = e->groups[k];
        cudaStream_t gs = k == 0 ? st : e->gst[k - 1];
        if (k > 0 && cudaStreamWaitEvent(gs, e->fork, 0) != cudaSuccess) return FVX_ERR_CUDA;
        ens_mode_split_kernel<<<dim3((g.n + kMixRows - 1) / kMixRows, g.B), 256, 0, gs>>>(
            g.md[s], g.n, g.hi, g.lo, g.perm, e->refine ? g.fm : nullptr);
        const long long plane = (long long)g.n * g.n;
        int rc = fvx_dst_solve_presplit_f32(g.plan, g.psim, plane, g.n, g.B, gs);
        if (rc) return rc;
        if (e->refine && g.nref &&
            (rc = fvx_dst_refine_f32(g.plan, g.fm, plane, g.n, g.psim, plane, g.n, g.nref, e->refine, gs)))
          return rc;
        ens_layer_mix_kernel<<<dim3((g.n + kMixRows - 1) / kMixRows, g.nlay), 256, 0, gs>>>(g.ld, g.n, g.psim);
        if (k > 0 && cudaEventRecord(e->gdone[k - 1], gs) != cudaSuccess) return FVX_ERR_CUDA;
      }
      for (int k = 1; k < ng; ++k)  // join before the stage kernel reads every psi
        if (cudaStreamWaitEvent(st, e->gdone[k - 1], 0) != cudaSuccess) return FVX_ERR_CUDA;
      int rc = ens_stage_dispatch(e, s, st);
      if (rc) return rc;
    }
  return fvx_cuda_status();
}
