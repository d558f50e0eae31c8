// Dirichlet Helmholtz solver by dense DST-I matrix products on the
// tcgen05 tensor cores (sm_100a).
//
// Restates spectraldiffx v0.0.10 ``solve_helmholtz_dst`` (re-exported at
// finitevolX solvers/spectral.py:14-98; math in docs/elliptic_solvers.md:
// 55-76): psi = IDST2(DST2(f) / Lambda) with Lambda[j,i] = ey[j] + ex[i] -
// lambda and ey[j] = -4/dy^2 sin^2(pi (j+1) / (2 (Ny+1))).  With the DST-I
// matrix S[j,k] = sin(pi (j+1)(k+1) / (N+1)) (symmetric), scipy's
// unnormalised DST-I is 2 S and its inverse S / (N+1), so
//   psi = 4 / ((Ny+1)(Nx+1)) * S_y ((S_y f S_x) ./ Lambda) S_x.
//
// The four products run as one GEMM shape, C = X S (X row-major, S
// symmetric, so both operands are K-major), whose epilogue stores C
// transposed: the chain Q -> (Q S_x)^T -> (S_y Q S_x ./ Lambda) ->
// (. S_x)^T -> psi needs no transpose kernels and every operand is a
// K-major TMA tile.  Precision: 3xBF16 split (X = Xh + Xl, S = Sh + Sl,
// C = Xh Sh + Xh Sl + Xl Sh) with FP32 accumulation in TMEM; the epilogue
// writes the next product's operand already split into bf16 hi/lo.  An FP64
// SIMT form of the same chain is the correctness path, and the FP64 solve
// recovers full accuracy by iterative refinement with an FP64 residual.
#include "fvx_common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <cstdio>
#include <vector>

namespace fvx {
namespace dst {

typedef __nv_bfloat16 bf16;

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 2;
constexpr int A_TILE = BM * BK * 2;                        // 16 KiB
constexpr int B_TILE = BN * BK * 2;                        // 32 KiB
constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE;       // 96 KiB
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr int THREADS = 192;                               // TMA warp, MMA warp, 4 epilogue warps
constexpr long long kWaitCycles = 4000000000LL;            // default bound on every spin-wait (~2 s)

enum EpiMode { EPI_SPLIT = 0, EPI_F32 = 1, EPI_F64 = 2, EPI_F64_ACC = 3, EPI_F32_ACC = 4 };

struct Epi {
  int mode;
  int rows_per_batch;      // R: row m of C is (batch m / R, r = m % R)
  int m_total;             // M
  int n_cols;              // valid N
  void* out0;              // hi / f32 / f64 output
  void* out1;              // lo output (split mode)
  long long batch_stride;  // elements between batches in the output
  long long ld;            // elements between consecutive n rows of the (transposed) output
  int off_n, off_r;        // index offsets into the output (e.g. a ghost ring)
  double alpha;
  const float* inv_eig;    // [n_eig][N][R] scale 1/Lambda, or null
  const double* inv_eig64;
  int n_eig;               // batch b uses grid b % n_eig
  int* err;
  int perm_r = 0;          // store r at its even/odd de-interleaved position (the next product's layout)
  int tma_out = 0;         // even/odd kernel: stage the tile in shared memory, TMA bulk-tensor stores
  long long wait_cycles = kWaitCycles;  // bound on every barrier wait of the main loop and epilogue
  int stall = 0;           // fault injection for tests: the producer issues no loads, so the
                           // MMA warp's first wait runs out (nothing is ever in flight)
};

// ---- PTX helpers ----------------------------------------------------------
DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

DEV void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count));
}
DEV void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
DEV bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after ``limit`` SM cycles (default ~2 s), raises the
// CTA abort flag and the global error flag instead of spinning forever.
DEV bool mbar_wait(uint32_t a, uint32_t parity, volatile int* abort_flag, int* err, long long limit = kWaitCycles) {
  long long t0 = clock64();
  while (!mbar_try(a, parity)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > limit) {
      *abort_flag = 1;
      if (err) atomicExch(err, 1);
      return false;
    }
  }
  return true;
}
// Wait for phase ``parity`` of barrier ``a`` regardless of the abort flag,
// bounded by the default limit: used after an abort so that no copy or MMA
// issued earlier is still in flight when the CTA frees TMEM and exits.
DEV void mbar_drain(uint32_t a, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(a, parity))
    if (clock64() - t0 > kWaitCycles) return;
}
// The loads issued for ring slots issued-stages .. issued-1 (the last one
// into each stage) have landed.
DEV void drain_ring(uint32_t full0, int stages, int issued) {
  for (int k = issued > stages ? issued - stages : 0; k < issued; ++k)
    mbar_drain(full0 + 8u * (uint32_t)(k % stages), (uint32_t)((k / stages) & 1));
}
DEV void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1)
      : "memory");
}
DEV void tma_store_3d(const CUtensorMap* map, uint32_t src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                   (uint64_t)map),
               "r"(src), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
DEV void tma_store_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
DEV void prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}
DEV void tma_store_commit_wait() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
// A-operand collector buffer (tcgen05.mma .collector::a::*): an MMA with
// COLL_FILL keeps the A tile it reads from shared memory in the tensor
// core's collector; the next MMA, with COLL_LASTUSE and the same A
// descriptor, takes A from there instead of shared memory and frees it.
// The split products reuse A_hi this way (A_hi B_hi, then A_hi B_lo).
enum { COLL_NONE = 0, COLL_FILL = 1, COLL_LASTUSE = 2 };
#define FVX_UMMA(GROUP, QUAL)                                                      \
  asm volatile(                                                                    \
      "{\n\t.reg .pred p;\n\t"                                                     \
      "setp.ne.b32 p, %4, 0;\n\t"                                                  \
      "tcgen05.mma.cta_group::" GROUP ".kind::f16" QUAL " [%0], %1, %2, %3, p;\n\t}" \
      ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate))
template <int COLL = COLL_NONE>
DEV void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  if constexpr (COLL == COLL_FILL) FVX_UMMA("1", ".collector::a::fill");
  else if constexpr (COLL == COLL_LASTUSE) FVX_UMMA("1", ".collector::a::lastuse");
  else FVX_UMMA("1", "");
}
DEV void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// ---- CTA-pair (cta_group::2) forms ----------------------------------------
DEV uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// The same shared-memory variable in CTA `rank` of the cluster.
DEV uint32_t map_to_rank(uint32_t a, uint32_t rank) {
  uint32_t o;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(o) : "r"(a), "r"(rank));
  return o;
}
// Every thread of both CTAs (the non-.aligned form: callers may arrive from
// diverged lanes).
DEV void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire;" ::: "memory");
}
// Tile load into this CTA's shared memory whose completion is counted on the
// pair leader's barrier `bar` (a shared::cluster address).  No multicast.
DEV void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
      "%4}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1)
      : "memory");
}
// M = 256 product over the pair: A rows 0-127 from the leader's shared
// memory, 128-255 from the peer's; B's N columns split in halves likewise.
template <int COLL = COLL_NONE>
DEV void umma_bf16_pair(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  if constexpr (COLL == COLL_FILL) FVX_UMMA("2", ".collector::a::fill");
  else if constexpr (COLL == COLL_LASTUSE) FVX_UMMA("2", ".collector::a::lastuse");
  else FVX_UMMA("2", "");
}
#undef FVX_UMMA
// Arrive on barrier `bar` of both CTAs of the pair once the issued MMAs end.
DEV void umma_commit_pair(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          bar),
      "h"((uint16_t)3)
      : "memory");
}
DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
DEV void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
DEV void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row core
// groups 1024 B apart (SBO), sm_100 descriptor version 1.
DEV uint64_t sdesc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// The same for 64-byte rows (32 bf16 of K): 64-byte swizzle, 8-row groups
// 512 B apart.
DEV uint64_t sdesc_sw64(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}
template <int BKT> DEV uint64_t sdesc_k(uint32_t saddr) {
  if constexpr (BKT == 64) return sdesc_sw128(saddr);
  else return sdesc_sw64(saddr);
}
// Instruction descriptor: kind::f16 with BF16 A/B, FP32 accumulator,
// both operands K-major, M = 128, N = 256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);

// ---- epilogue store ---------------------------------------------------------
// Position of index r in the even/odd de-interleaved layout of a length-R
// axis: evens first (r / 2), then odds (R / 2 + r / 2).
DEV int deinterleave(int r, int R) { return (r & 1) ? (R >> 1) + (r >> 1) : (r >> 1); }

DEV void epi_store(const Epi& ep, int b, int r, int n, float acc) {
  const int rs = ep.perm_r ? deinterleave(r, ep.rows_per_batch) : r;
  long long idx = (long long)b * ep.batch_stride + (long long)(n + ep.off_n) * ep.ld + (rs + ep.off_r);
  switch (ep.mode) {
    case EPI_SPLIT: {
      float x = acc * (float)ep.alpha;
      if (ep.inv_eig) x *= ep.inv_eig[((long long)(b % ep.n_eig) * ep.n_cols + n) * ep.rows_per_batch + r];
      bf16 hi = __float2bfloat16_rn(x);
      bf16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
      ((bf16*)ep.out0)[idx] = hi;
      ((bf16*)ep.out1)[idx] = lo;
      break;
    }
    case EPI_F32: {
      float x = acc * (float)ep.alpha;
      if (ep.inv_eig) x *= ep.inv_eig[((long long)(b % ep.n_eig) * ep.n_cols + n) * ep.rows_per_batch + r];
      ((float*)ep.out0)[idx] = x;
      break;
    }
    case EPI_F64:
      ((double*)ep.out0)[idx] = (double)acc * ep.alpha;
      break;
    case EPI_F32_ACC:
      ((float*)ep.out0)[idx] += acc * (float)ep.alpha;
      break;
    default:
      ((double*)ep.out0)[idx] += (double)acc * ep.alpha;
      break;
  }
}

// ---- the tcgen05 GEMM -------------------------------------------------------
__global__ void __launch_bounds__(THREADS, 1)
gemm_split_bf16_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                       const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl, int K,
                       Epi ep) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);  // full[S], empty[S], acc
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 1);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int KT = (K + BK - 1) / BK;
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[STAGES + s]); };
  const uint32_t accb = smem_u32(&bars[2 * STAGES]);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) { mbar_init(full(s), 1); mbar_init(empty(s), 1); }
    mbar_init(accb, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // CTAs start their K loop at different blocks so the ones that share an
  // A or B tile do not all read the same L2 lines at the same time
  const int kshift = (int)((blockIdx.x * 5u + blockIdx.y * 3u) % (unsigned)KT);
  if (warp == 0 && lane == 0) {
    // TMA producer (with ep.stall: no loads, for the timeout test)
    int issued = 0;
    for (int kt = 0; kt < KT && !ep.stall; ++kt) {
      const int s = kt % STAGES;
      if (kt >= STAGES && !mbar_wait(empty(s), ((kt / STAGES) - 1) & 1, abort_flag, ep.err, ep.wait_cycles)) break;
      mbar_expect_tx(full(s), STAGE_BYTES);
      const uint32_t base = smem_u32(smem + s * STAGE_BYTES);
      const int kc = ((kt + kshift) % KT) * BK;
      tma_load_2d(base, &mAh, full(s), kc, m0);
      tma_load_2d(base + A_TILE, &mAl, full(s), kc, m0);
      tma_load_2d(base + 2 * A_TILE, &mBh, full(s), kc, n0);
      tma_load_2d(base + 2 * A_TILE + B_TILE, &mBl, full(s), kc, n0);
      issued = kt + 1;
    }
    drain_ring(full(0), STAGES, issued);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: three split products per 16-wide K step
    bool ok = true;
    for (int kt = 0; kt < KT && ok; ++kt) {
      const int s = kt % STAGES;
      ok = mbar_wait(full(s), (kt / STAGES) & 1, abort_flag, ep.err, ep.wait_cycles);
      if (!ok) break;
      tc_fence_after();
      const uint32_t base = smem_u32(smem + s * STAGE_BYTES);
      const uint64_t ah = sdesc_sw128(base), al = sdesc_sw128(base + A_TILE);
      const uint64_t bh = sdesc_sw128(base + 2 * A_TILE), bl = sdesc_sw128(base + 2 * A_TILE + B_TILE);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint64_t o = (uint64_t)(kk * 32 >> 4);
        umma_bf16<COLL_FILL>(tmem, ah + o, bh + o, kIdesc, (kt | kk) != 0);
        umma_bf16<COLL_LASTUSE>(tmem, ah + o, bl + o, kIdesc, 1u);
        umma_bf16(tmem, al + o, bh + o, kIdesc, 1u);
      }
      umma_commit(empty(s));
    }
    umma_commit(accb);  // also issued after an abort so the epilogue never waits on MMAs in flight
  } else if (warp >= 2) {
    // epilogue: TMEM -> registers -> transposed global stores
    const int wq = warp & 3;
    const int row = wq * 32 + lane;
    const int m = m0 + row;
    const bool mvalid = m < ep.m_total;
    const int b = mvalid ? m / ep.rows_per_batch : 0;
    const int r = mvalid ? m - b * ep.rows_per_batch : 0;
    if (mbar_wait(accb, 0, abort_flag, ep.err, ep.wait_cycles)) {
      tc_fence_after();
      if (!*abort_flag) {
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
          uint32_t v[32];
          tmem_ld32(tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)c0, v);
          tmem_wait_ld();
          if (mvalid) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const int n = n0 + c0 + j;
              if (n < ep.n_cols) epi_store(ep, b, r, n, __uint_as_float(v[j]));
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    if (lane == 0) mbar_drain(accb, 0);  // the MMAs issued before an abort have completed
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
  }
}

// ---- even/odd DST-I product ---------------------------------------------------
// S[N-1-j][k] = (-1)^k S[j][k] and S is symmetric, so for C = X S (N even)
//   P[:, k] = sum_{j even} X[:, j] S[j, k],  Q[:, k] = sum_{j odd} X[:, j] S[j, k]
//   C[:, k] = P + Q,  C[:, N-1-k] = P - Q      (k < N/2)
// which halves the multiply work.  X arrives with its columns de-interleaved
// (evens then odds), so the even and odd halves are plain column ranges of
// one TMA tensor; B_P[k][j'] = S[2j'][k] and B_Q[k][j'] = S[2j'+1][k] are
// N/2 x N/2 K-major tables.  Each CTA owns a 128-row x 128-k tile of P and
// of Q (TMEM columns 0-127 and 128-255); the k loop alternates P and Q
// blocks through a 3-stage TMA ring of 64 KiB stages.
constexpr int SBN = 128;
// Ring geometry for a K block of BKT elements: 192 KiB of stages (3 of 64
// KiB for BKT = 64, 6 of 32 KiB for BKT = 32; the smaller stages keep more
// loads in flight).
template <int BKT> struct SymCfg {
  static constexpr int A_T = BM * BKT * 2, B_T = SBN * BKT * 2;
  static constexpr int STAGE = 2 * A_T + 2 * B_T;
  static constexpr int STAGES = (3 * 64) / BKT;
  static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
  static_assert(STAGES * STAGE >= 2 * 2 * 2 * 8192 * 2, "epilogue staging fits in the operand ring");
};
constexpr uint32_t kIdesc128 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SBN >> 3) << 17) |
                               ((uint32_t)(BM >> 4) << 24);
// TMA warp, MMA warp and 16 epilogue warps in four groups of four (one warp
// per TMEM lane quadrant, warp % 4); group g converts columns 32g..32g+31 of
// P and Q.  Four warps per scheduler hide the epilogue's TMEM, conversion
// and store latencies (the epilogue does not overlap the main loop: one
// tile per CTA).
constexpr int EPI_GROUPS = 4;
constexpr int EPI_COLS = SBN / EPI_GROUPS;  // 32 columns per group
constexpr int S_THREADS = 64 + 128 * EPI_GROUPS;

DEV void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
DEV void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Epilogue of the even/odd product, run by the 16 epilogue warps of a CTA
// (warps 2-17): P and Q of this CTA's 128 rows from TMEM (columns 0-127 and
// 128-255) become C[:, k] = P + Q and C[:, K-1-k] = P - Q, scaled, divided
// by Lambda when the plan asks, and stored (staged in shared memory and
// written by TMA when ep.tma_out, else by scattered stores).
DEV void sym_epilogue(uint8_t* smem, uint32_t tmem, uint32_t accb, int m0, int n0, int K, const Epi& ep,
                      volatile int* abort_flag, const CUtensorMap* mO0, const CUtensorMap* mO1, int warp,
                      int lane) {
  const int KH = K >> 1;
  const int wq = warp & 3;
  const int grp = (warp - 2) >> 2;
  const int cbeg = grp * EPI_COLS;  // this group's columns
  const int row = wq * 32 + lane;
  const int m = m0 + row;
  const bool mvalid = m < ep.m_total;
  const int b = mvalid ? m / ep.rows_per_batch : 0;
  const int r = mvalid ? m - b * ep.rows_per_batch : 0;
  const uint32_t lanes = (uint32_t)(wq * 32) << 16;
  if (ep.tma_out) {
    // Tile staged in the idle operand ring (all MMAs have completed), then
    // written by TMA bulk-tensor stores.  The host enables this only when
    // R is a multiple of 128 and the outputs satisfy TMA's alignment, so
    // the tile has one batch index b and starts at an even r0.
    const int R = ep.rows_per_batch;
    const int bb = m0 / R, r0 = m0 - bb * R;
    const int be = bb % ep.n_eig;
    const float alpha = (float)ep.alpha;
    const bool scaled = ep.alpha != 1.0;
    const int half = row & 1, rl = row >> 1;
    const float* ie = ep.inv_eig ? ep.inv_eig + (long long)be * ep.n_cols * R + (r0 + row) : nullptr;
    // 1/Lambda while the main loop runs: the first 16 columns' values into
    // registers, the next 16 columns' lines into L2
    float ivp[16], ivm[16];
    if (ie) {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int k = n0 + cbeg + j;
        ivp[j] = __ldg(ie + (long long)k * R);
        ivm[j] = __ldg(ie + (long long)(K - 1 - k) * R);
      }
      const float* base = ie - row + wq * 32;  // the warp's first row
      const int k = n0 + cbeg + 16 + (lane & 15);
      prefetch_l2(base + (long long)((lane < 16) ? k : K - 1 - k) * R);
    }
    const bool ok = mbar_wait(accb, 0, abort_flag, ep.err, ep.wait_cycles);
    if (ok) tc_fence_after();
    grid_dep_launch();  // the next kernel may start its set-up while this tile drains
    const bool go = ok && !*abort_flag;
    // 16 columns per step; each step's stores run while the group converts
    // the next step's columns
#pragma unroll 1
    for (int sc = 0; sc < EPI_COLS; sc += 16) {
      const int c0 = cbeg + sc;
      if (go) {
        if (ie && sc) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int k = n0 + c0 + j;
            ivp[j] = __ldg(ie + (long long)k * R);
            ivm[j] = __ldg(ie + (long long)(K - 1 - k) * R);
          }
        }
        uint32_t vp[16], vq[16];
        tmem_ld16(tmem + lanes + (uint32_t)c0, vp);
        tmem_ld16(tmem + lanes + (uint32_t)(SBN + c0), vq);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int kl = c0 + j;
          const float P = __uint_as_float(vp[j]), Q = __uint_as_float(vq[j]);
          float xp = P + Q, xm = P - Q;
          if (scaled) { xp *= alpha; xm *= alpha; }
          if (ie) {
            xp *= ivp[j];
            xm *= ivm[j];
          }
          if (ep.mode == EPI_SPLIT) {
            // boxes [which][half][hi/lo][128 n][64 r] bf16
            bf16* box = (bf16*)smem;
            // both values of the pair converted by one packed cvt
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(xp, xm);
            const __nv_bfloat162 l2 = __floats2bfloat162_rn(xp - __low2float(h2), xm - __high2float(h2));
            const int op = kl * 64 + rl, om = (127 - kl) * 64 + rl;
            box[((0 * 2 + half) * 2 + 0) * 8192 + op] = h2.x;
            box[((0 * 2 + half) * 2 + 1) * 8192 + op] = l2.x;
            box[((1 * 2 + half) * 2 + 0) * 8192 + om] = h2.y;
            box[((1 * 2 + half) * 2 + 1) * 8192 + om] = l2.y;
          } else {
            // boxes [which][128 n][128 r] fp32
            float* box = (float*)smem;
            box[kl * 128 + row] = xp;
            box[16384 + (127 - kl) * 128 + row] = xm;
          }
        }
      }
      // the step's 16 columns of every box are complete once the group's
      // four warps (one per 32-row quadrant) pass: its first thread writes
      // them (16-row sub-boxes) with TMA
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("bar.sync %0, 128;" ::"r"(2 + grp) : "memory");
      if (go && lane == 0 && (warp & 3) == 2) {
        const uint32_t sb = smem_u32(smem);
        if (ep.mode == EPI_SPLIT) {
          for (int which = 0; which < 2; ++which)
            for (int hf = 0; hf < 2; ++hf)
              for (int hl = 0; hl < 2; ++hl) {
                const int brow = which ? 112 - c0 : c0;  // first box row of the step's columns
                const uint32_t src = sb + (uint32_t)((((which * 2 + hf) * 2 + hl) * 8192 + brow * 64) * 2);
                const int x = (hf ? (R >> 1) : 0) + (r0 >> 1);
                const int y = (which ? K - n0 - SBN : n0) + brow;
                tma_store_3d(hl ? mO1 : mO0, src, x, y, bb);
              }
        } else {
          tma_store_3d(mO0, sb + (uint32_t)(c0 * 128 * 4), r0, n0 + c0, bb);
          tma_store_3d(mO0, sb + (uint32_t)((16384 + (112 - c0) * 128) * 4), r0, K - n0 - SBN + 112 - c0, bb);
        }
        tma_store_commit();
      }
    }
    // shared memory stays allocated until the stores have read it
    if (go && lane == 0 && (warp & 3) == 2) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
  } else {
    const bool ok = mbar_wait(accb, 0, abort_flag, ep.err, ep.wait_cycles);
    if (ok) tc_fence_after();
    grid_dep_launch();
    if (ok && !*abort_flag) {
#pragma unroll 1
      for (int sc = 0; sc < EPI_COLS; sc += 16) {
        const int c0 = cbeg + sc;
        uint32_t vp[16], vq[16];
        tmem_ld16(tmem + lanes + (uint32_t)c0, vp);
        tmem_ld16(tmem + lanes + (uint32_t)(SBN + c0), vq);
        tmem_wait_ld();
        if (mvalid) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int k = n0 + c0 + j;
            if (k < KH) {
              const float P = __uint_as_float(vp[j]), Q = __uint_as_float(vq[j]);
              epi_store(ep, b, r, k, P + Q);
              epi_store(ep, b, r, K - 1 - k, P - Q);
            }
          }
        }
      }
    }
  }
}

template <int BKT>
__global__ void __launch_bounds__(S_THREADS, 1)
gemm_sym_bf16_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                     const __grid_constant__ CUtensorMap mPh, const __grid_constant__ CUtensorMap mPl,
                     const __grid_constant__ CUtensorMap mQh, const __grid_constant__ CUtensorMap mQl,
                     const __grid_constant__ CUtensorMap mO0, const __grid_constant__ CUtensorMap mO1, int K,
                     Epi ep) {
  using C = SymCfg<BKT>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + C::STAGES * C::STAGE);  // full[S], empty[S], acc
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * C::STAGES + 1);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * SBN;
  const int KH = K >> 1;
  const int KT = 2 * ((KH + BKT - 1) / BKT);  // P and Q blocks alternate
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[C::STAGES + s]); };
  const uint32_t accb = smem_u32(&bars[2 * C::STAGES]);

  if (threadIdx.x == 0) {
    // descriptor fetches overlap the barrier and TMEM set-up
    prefetch_map(&mAh); prefetch_map(&mAl); prefetch_map(&mPh);
    prefetch_map(&mPl); prefetch_map(&mQh); prefetch_map(&mQl);
    if (ep.tma_out) { prefetch_map(&mO0); prefetch_map(&mO1); }
    for (int s = 0; s < C::STAGES; ++s) { mbar_init(full(s), 1); mbar_init(empty(s), 1); }
    mbar_init(accb, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * SBN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // staggered start (an even shift keeps the P / Q alternation)
  const int kshift = 2 * (int)((blockIdx.x * 5u + blockIdx.y * 3u) % (unsigned)(KT / 2));
  if (warp == 0 && lane == 0) {
    // B blocks (the DST tables) of the first ring fill before waiting for
    // the previous kernel; A (its output) only after
    auto load_b = [&](int kt0) {
      const int s = kt0 % C::STAGES;
      mbar_expect_tx(full(s), C::STAGE);
      const uint32_t base = smem_u32(smem + s * C::STAGE);
      const int kt = (kt0 + kshift) % KT;
      const int kb = kt >> 1;
      const bool odd = kt & 1;
      tma_load_2d(base + 2 * C::A_T, odd ? &mQh : &mPh, full(s), kb * BKT, n0);
      tma_load_2d(base + 2 * C::A_T + C::B_T, odd ? &mQl : &mPl, full(s), kb * BKT, n0);
    };
    const int KTL = ep.stall ? 0 : KT;  // ep.stall: no loads (the timeout test)
    for (int kt0 = 0; kt0 < KTL && kt0 < C::STAGES; ++kt0) load_b(kt0);
    grid_dep_wait();
    int issued = 0;
    for (int kt0 = 0; kt0 < KTL; ++kt0) {
      const int s = kt0 % C::STAGES;
      if (kt0 >= C::STAGES) {
        if (!mbar_wait(empty(s), ((kt0 / C::STAGES) - 1) & 1, abort_flag, ep.err, ep.wait_cycles)) break;
        load_b(kt0);
      }
      const uint32_t base = smem_u32(smem + s * C::STAGE);
      const int kt = (kt0 + kshift) % KT;
      const int ac = ((kt & 1) ? KH : 0) + (kt >> 1) * BKT;
      tma_load_2d(base, &mAh, full(s), ac, m0);
      tma_load_2d(base + C::A_T, &mAl, full(s), ac, m0);
      issued = kt0 + 1;
    }
    drain_ring(full(0), C::STAGES, issued);
  } else if (warp == 1 && lane == 0) {
    bool ok = true;
    for (int kt0 = 0; kt0 < KT && ok; ++kt0) {
      const int s = kt0 % C::STAGES;
      ok = mbar_wait(full(s), (kt0 / C::STAGES) & 1, abort_flag, ep.err, ep.wait_cycles);
      if (!ok) break;
      tc_fence_after();
      const uint32_t base = smem_u32(smem + s * C::STAGE);
      const uint64_t ah = sdesc_k<BKT>(base), al = sdesc_k<BKT>(base + C::A_T);
      const uint64_t bh = sdesc_k<BKT>(base + 2 * C::A_T), bl = sdesc_k<BKT>(base + 2 * C::A_T + C::B_T);
      const int kt = (kt0 + kshift) % KT;
      const uint32_t d = tmem + ((kt & 1) ? (uint32_t)SBN : 0u);
      const bool first = kt0 < 2;  // the first P block and the first Q block overwrite
#pragma unroll
      for (int kk = 0; kk < BKT / 16; ++kk) {
        const uint64_t o = (uint64_t)(kk * 32 >> 4);
        umma_bf16<COLL_FILL>(d, ah + o, bh + o, kIdesc128, !(first && kk == 0));
        umma_bf16<COLL_LASTUSE>(d, ah + o, bl + o, kIdesc128, 1u);
        umma_bf16(d, al + o, bh + o, kIdesc128, 1u);
      }
      umma_commit(empty(s));
    }
    umma_commit(accb);
  } else if (warp >= 2) {
    sym_epilogue(smem, tmem, accb, m0, n0, K, ep, abort_flag, &mO0, &mO1, warp, lane);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    if (lane == 0) mbar_drain(accb, 0);  // the MMAs issued before an abort have completed
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * SBN));
  }
}

// The even/odd product on CTA pairs (cta_group::2): the two CTAs of a
// cluster own rows m0..m0+127 and m0+128..m0+255 of one 256-row tile and
// share its B blocks, each CTA loading 64 of the 128 table rows.  Per stage
// a CTA moves 48 KiB (its A hi/lo, half of B hi/lo) instead of 64 KiB, and
// its tensor core reads 6 KiB of shared memory per 128x128x16 product
// instead of 8 KiB: shared-memory bandwidth bounds the single-CTA main
// loop.  The leader (rank 0) issues the M = 256 MMAs; both CTAs' TMA loads
// complete on the leader's full barriers; each MMA commit arrives on both
// CTAs' empty barriers.  The epilogue is per CTA (its own TMEM lanes).
constexpr int P_STAGES = 4;
constexpr int P_A_TILE = BM * BK * 2;                       // 16 KiB
constexpr int P_B_TILE = (SBN / 2) * BK * 2;                // 8 KiB
constexpr int P_STAGE = 2 * P_A_TILE + 2 * P_B_TILE;        // 48 KiB
constexpr int P_SMEM = P_STAGES * P_STAGE + 1024 + 256;
constexpr uint32_t kIdescPair = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SBN >> 3) << 17) |
                                ((uint32_t)((2 * BM) >> 4) << 24);
static_assert(P_STAGES * P_STAGE >= 2 * 2 * 2 * 8192 * 2, "epilogue staging fits in the operand ring");

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(S_THREADS, 1)
gemm_sym_pair_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                     const __grid_constant__ CUtensorMap mPh, const __grid_constant__ CUtensorMap mPl,
                     const __grid_constant__ CUtensorMap mQh, const __grid_constant__ CUtensorMap mQl,
                     const __grid_constant__ CUtensorMap mO0, const __grid_constant__ CUtensorMap mO1, int K,
                     Epi ep) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + P_STAGES * P_STAGE);  // full[S], empty[S], acc
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * P_STAGES + 1);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * SBN;
  const int KH = K >> 1;
  const int KT = 2 * ((KH + BK - 1) / BK);  // P and Q blocks alternate
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[P_STAGES + s]); };
  const uint32_t accb = smem_u32(&bars[2 * P_STAGES]);

  if (threadIdx.x == 0) {
    // descriptor fetches overlap the barrier and TMEM set-up
    prefetch_map(&mAh); prefetch_map(&mAl); prefetch_map(&mPh);
    prefetch_map(&mPl); prefetch_map(&mQh); prefetch_map(&mQl);
    if (ep.tma_out) { prefetch_map(&mO0); prefetch_map(&mO1); }
    for (int s = 0; s < P_STAGES; ++s) { mbar_init(full(s), 1); mbar_init(empty(s), 1); }
    mbar_init(accb, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {  // the same warp in both CTAs, as the paired allocation requires
    __syncwarp();
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * SBN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  cluster_sync_all();  // both CTAs' barriers initialised before any cross-CTA arrive
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // staggered start, the same for both CTAs of the pair (an even shift
  // keeps the P / Q alternation)
  const int kshift = 2 * (int)(((blockIdx.x >> 1) * 5u + blockIdx.y * 3u) % (unsigned)(KT / 2));
  if (warp == 0 && lane == 0) {
    // B blocks of the first ring fill before waiting for the previous
    // kernel; A (its output) only after
    const int brow = n0 + (int)rank * (SBN / 2);
    auto load_b = [&](int kt0) {
      const int s = kt0 % P_STAGES;
      if (rank == 0) mbar_expect_tx(full(s), 2 * P_STAGE);
      const uint32_t fb = map_to_rank(full(s), 0);
      const uint32_t base = smem_u32(smem + s * P_STAGE);
      const int kt = (kt0 + kshift) % KT;
      const int kb = kt >> 1;
      const bool odd = kt & 1;
      tma_load_2d_pair(base + 2 * P_A_TILE, odd ? &mQh : &mPh, fb, kb * BK, brow);
      tma_load_2d_pair(base + 2 * P_A_TILE + P_B_TILE, odd ? &mQl : &mPl, fb, kb * BK, brow);
    };
    for (int kt0 = 0; kt0 < KT && kt0 < P_STAGES; ++kt0) load_b(kt0);
    grid_dep_wait();
    for (int kt0 = 0; kt0 < KT; ++kt0) {
      const int s = kt0 % P_STAGES;
      if (kt0 >= P_STAGES) {
        if (!mbar_wait(empty(s), ((kt0 / P_STAGES) - 1) & 1, abort_flag, ep.err, ep.wait_cycles)) break;
        load_b(kt0);
      }
      const uint32_t fb = map_to_rank(full(s), 0);
      const uint32_t base = smem_u32(smem + s * P_STAGE);
      const int kt = (kt0 + kshift) % KT;
      const int ac = ((kt & 1) ? KH : 0) + (kt >> 1) * BK;
      tma_load_2d_pair(base, &mAh, fb, ac, m0);
      tma_load_2d_pair(base + P_A_TILE, &mAl, fb, ac, m0);
    }
  } else if (warp == 1 && lane == 0) {
    if (rank == 0) {
      bool ok = true;
      for (int kt0 = 0; kt0 < KT && ok; ++kt0) {
        const int s = kt0 % P_STAGES;
        ok = mbar_wait(full(s), (kt0 / P_STAGES) & 1, abort_flag, ep.err, ep.wait_cycles);
        if (!ok) break;
        tc_fence_after();
        const uint32_t base = smem_u32(smem + s * P_STAGE);
        const uint64_t ah = sdesc_sw128(base), al = sdesc_sw128(base + P_A_TILE);
        const uint64_t bh = sdesc_sw128(base + 2 * P_A_TILE), bl = sdesc_sw128(base + 2 * P_A_TILE + P_B_TILE);
        const int kt = (kt0 + kshift) % KT;
        const uint32_t d = tmem + ((kt & 1) ? (uint32_t)SBN : 0u);
        const bool first = kt0 < 2;  // the first P block and the first Q block overwrite
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          const uint64_t o = (uint64_t)(kk * 32 >> 4);
          umma_bf16_pair<COLL_FILL>(d, ah + o, bh + o, kIdescPair, !(first && kk == 0));
          umma_bf16_pair<COLL_LASTUSE>(d, ah + o, bl + o, kIdescPair, 1u);
          umma_bf16_pair(d, al + o, bh + o, kIdescPair, 1u);
        }
        umma_commit_pair(empty(s));
      }
      umma_commit_pair(accb);
    }
  } else if (warp >= 2) {
    sym_epilogue(smem, tmem, accb, m0, n0, K, ep, abort_flag, &mO0, &mO1, warp, lane);
  }
  tc_fence_before();
  cluster_sync_all();  // no CTA frees TMEM or exits while its peer may still signal it
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * SBN));
  }
}

// ---- FP64 SIMT GEMM with the same transposed-store epilogue (correctness path)
// TDT x TDT output tiles, 256 threads, each (TDT / 16)^2 outputs; every
// output's FMA chain runs over k in order, so the tile size does not change
// the result.  The largest tile that still gives at least one CTA per SM is
// used (64, else 32, else 16).
template <int TDT> struct F64Cfg {
  // k-block: small tiles stage long k-blocks (few dependent load round trips
  // per output); large tiles are bound by their FMAs
  static constexpr int DK = TDT == 16 ? 128 : 16;
};
template <int TDT>
__global__ void __launch_bounds__(256)
gemm_f64_kernel(const double* A, int lda, const double* __restrict__ S, int lds, int M, int N, int K, Epi ep) {
  constexpr int R = TDT / 16, DK = F64Cfg<TDT>::DK, NL = TDT * DK / 256;  // loads per thread per operand
  static_assert(TDT * DK % 256 == 0, "whole loads per thread");
  __shared__ double As[DK][TDT + 1];
  __shared__ double Ss[DK][TDT + 1];
  // launched as a programmatic dependent: A (and the output) belong to the
  // kernel before until the wait; A is then read through L2 (__ldcg, no
  // restrict), so no load of it can be placed before the wait
  grid_dep_wait();
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * TDT, n0 = blockIdx.x * TDT;
  double acc[R][R] = {};
  for (int k0 = 0; k0 < K; k0 += DK) {
    {  // every load of the k-block in flight before any is stored
      double va[NL], vs[NL];
#pragma unroll
      for (int u = 0; u < NL; ++u) {
        const int t = threadIdx.x + u * 256;
        const int mm = t / DK, kk = t % DK, gm = m0 + mm, gk = k0 + kk;
        va[u] = (gm < M && gk < K) ? __ldcg(A + (long long)gm * lda + gk) : 0.0;
        const int kk2 = t / TDT, nn = t % TDT, gk2 = k0 + kk2, gn = n0 + nn;
        vs[u] = (gk2 < K && gn < N) ? S[(long long)gk2 * lds + gn] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < NL; ++u) {
        const int t = threadIdx.x + u * 256;
        As[t % DK][t / DK] = va[u];
        Ss[t / TDT][t % TDT] = vs[u];
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < DK; ++kk) {
      double a[R], s[R];
#pragma unroll
      for (int i = 0; i < R; ++i) { a[i] = As[kk][ty + 16 * i]; s[i] = Ss[kk][tx + 16 * i]; }
#pragma unroll
      for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < R; ++j) acc[i][j] = fma(a[i], s[j], acc[i][j]);
    }
    __syncthreads();
  }
  // the next kernel may launch while this one stores its results
  grid_dep_launch();
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
    const int b = m / ep.rows_per_batch, r = m - b * ep.rows_per_batch;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      double x = acc[i][j] * ep.alpha;
      if (ep.inv_eig64) x *= ep.inv_eig64[((long long)(b % ep.n_eig) * ep.n_cols + n) * ep.rows_per_batch + r];
      long long idx = (long long)b * ep.batch_stride + (long long)(n + ep.off_n) * ep.ld + (r + ep.off_r);
      if (ep.mode == EPI_F64_ACC) ((double*)ep.out0)[idx] += x;
      else if (ep.mode == EPI_F32) ((float*)ep.out0)[idx] = (float)x;
      else ((double*)ep.out0)[idx] = x;
    }
  }
}

// ---- input split / copy / residual kernels ---------------------------------
// perm: store x at its de-interleaved position (the even/odd product's
// operand layout).
template <typename T>
__global__ void split_input_kernel(const T* __restrict__ in, long long bstride, long long ld, int ny, int nx,
                                   int batch, bf16* __restrict__ hi, bf16* __restrict__ lo, double scale,
                                   int perm = 0) {
  // rows of the [batch][ny][nx] input over the grid, (even, odd) pairs of a
  // row over the threads: no 64-bit divisions, and with perm the two halves
  // of the de-interleaved row are written by consecutive threads
  const int rows = batch * ny, half = (nx + 1) >> 1;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    const int b = r / ny, y = r - b * ny;
    const T* src = in + (long long)b * bstride + (long long)y * ld;
    const long long o = (long long)r * nx;
    for (int p = threadIdx.x; p < half; p += blockDim.x) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int x = 2 * p + e;
        if (x >= nx) break;
        const float v = (float)((double)src[x] * scale);
        const bf16 h = __float2bfloat16_rn(v);
        const long long d = o + (perm ? (e ? (nx >> 1) + p : p) : x);
        hi[d] = h;
        lo[d] = __float2bfloat16_rn(v - __bfloat162float(h));
      }
    }
  }
}

template <typename T>
__global__ void copy_in_f64_kernel(const T* in, long long bstride, long long ld, int ny, int nx, int batch,
                                   double* __restrict__ out) {
  // rows of the [batch][ny][nx] input over the grid, a row's elements over
  // the threads (no per-element divisions).  Launched as a programmatic
  // dependent: the input is the previous kernel's output, read after the
  // wait through L2.
  grid_dep_wait();
  const int rows = batch * ny;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    const int b = r / ny, y = r - b * ny;
    const T* src = in + (long long)b * bstride + (long long)y * ld;
    double* dst = out + (long long)r * nx;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) dst[x] = (double)__ldcg(src + x);
  }
  grid_dep_launch();
}
static int copy_rows_grid(long long rows) { return (int)(rows < 148 * 16 ? (rows < 1 ? 1 : rows) : 148 * 16); }

__global__ void zero_f64_kernel(double* p, long long bstride, long long ld, int ny, int nx, int batch) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)batch * ny * nx;
  for (; k < n; k += (long long)gridDim.x * blockDim.x) {
    long long b = k / ((long long)ny * nx);
    long long rem = k - b * ny * nx;
    int y = (int)(rem / nx), x = (int)(rem - (long long)y * nx);
    p[b * bstride + (long long)y * ld + x] = 0.0;
  }
}

DEV double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// r = f - (lap - lambda) psi (5-point, zero outside), FP64; writes r split
// into bf16 hi/lo (the next correction's GEMM operand, scaled by 1/rscale)
// and accumulates sum r^2, sum f^2, sum psi^2, sum |A|^2-weighted norm parts
// into norms[0..3] with warp-shuffle reductions.
template <typename T, typename PT>
__global__ void residual_kernel(const T* __restrict__ f, long long fb, long long fld, const PT* __restrict__ psi,
                                long long pb, long long pld, int ny, int nx, int batch, double dx, double dy,
                                const double* __restrict__ lam, int nlam, bf16* __restrict__ hi,
                                bf16* __restrict__ lo, double* norms, int perm) {
  // a row (b, y) per block iteration, its x over the threads: no 64-bit
  // index divisions
  double s_r = 0, s_f = 0, s_p = 0;
  const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy);
  const int rows = batch * ny;
  for (int row = blockIdx.x; row < rows; row += gridDim.x) {
    const int b = row / ny, y = row - b * ny;
    const double lb = lam[b % nlam];
    const PT* P = psi + b * pb + (long long)y * pld;
    const T* F = f + b * fb + (long long)y * fld;
    const long long o0 = (long long)row * nx;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
      const PT* Px = P + x;
      const double c = (double)Px[0];
      const double e = x + 1 < nx ? (double)Px[1] : 0.0, w = x > 0 ? (double)Px[-1] : 0.0;
      const double nn = y + 1 < ny ? (double)Px[pld] : 0.0, s = y > 0 ? (double)Px[-pld] : 0.0;
      const double lap = ((e - 2.0 * c) + w) * idx2 + ((nn - 2.0 * c) + s) * idy2;
      const double fv = (double)F[x];
      const double r = fv - (lap - lb * c);
      const float rv = (float)r;
      const bf16 h = __float2bfloat16_rn(rv);
      const long long o = o0 + (perm ? deinterleave(x, nx) : x);
      hi[o] = h;
      lo[o] = __float2bfloat16_rn(rv - __bfloat162float(h));
      s_r += r * r;
      s_f += fv * fv;
      s_p += c * c;
    }
  }
  if (!norms) return;
  s_r = warp_sum(s_r);
  s_f = warp_sum(s_f);
  s_p = warp_sum(s_p);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&norms[0], s_r);
    atomicAdd(&norms[1], s_f);
    atomicAdd(&norms[2], s_p);
  }
}

static int residual_grid(int rows) { return rows < 148 * 16 ? rows : 148 * 16; }

// ---- host side ----------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 2-D bf16 tensor map over [outer][inner] (inner contiguous), box
// {BK, box_outer}, 128-byte swizzle, zero fill out of bounds.
static bool make_map(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint32_t box_outer,
                     uint32_t box_inner = BK) {
  auto enc = encode_fn();
  if (!enc) return false;
  if (((uintptr_t)base & 15) != 0 || (inner * 2) % 16 != 0) return false;
  if (box_inner != 64 && box_inner != 32) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {inner * 2};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE,
                   box_inner == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// C[M, N] = X[M, K] S[K, N] (S symmetric, given as hi/lo rows of length K).
static int gemm_split(const bf16* Xh, const bf16* Xl, int M, int K, const bf16* Sh, const bf16* Sl, int N,
                      const Epi& ep, cudaStream_t st) {
  static fvx_once_per_device attr;
  if (fvx_once_on_device(attr, [] { return fvx_set_max_smem(gemm_split_bf16_kernel, SMEM_BYTES); }))
    return FVX_ERR_CUDA;
  CUtensorMap a_h, a_l, b_h, b_l;
  if (!make_map(&a_h, Xh, K, M, BM) || !make_map(&a_l, Xl, K, M, BM) || !make_map(&b_h, Sh, K, N, BN) ||
      !make_map(&b_l, Sl, K, N, BN))
    return FVX_ERR_ARG;
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  if (grid.y > 65535) return FVX_ERR_SHAPE;
  gemm_split_bf16_kernel<<<grid, THREADS, SMEM_BYTES, st>>>(a_h, a_l, b_h, b_l, K, ep);
  return fvx_cuda_status();
}

// 3-D tensor map over an epilogue output [B][N][R] (R innermost, row pitch
// ld, batch pitch bs, in elements), box {box_r, 128, 1}, no swizzle.
static bool make_out_map(CUtensorMap* map, void* base, bool f32, uint64_t R, uint64_t N, uint64_t B, long long ld,
                         long long bs, uint32_t box_r) {
  auto enc = encode_fn();
  if (!enc) return false;
  const uint64_t es = f32 ? 4 : 2;
  if (((uintptr_t)base & 15) != 0 || ((uint64_t)ld * es) % 16 != 0 || (B > 1 && ((uint64_t)bs * es) % 16 != 0))
    return false;
  cuuint64_t dims[3] = {R, N, B};
  cuuint64_t strides[2] = {(cuuint64_t)ld * es, (cuuint64_t)(B > 1 ? bs : ld * (long long)N) * es};
  cuuint32_t box[3] = {box_r, 16, 1};  // one 16-column step of an epilogue group
  cuuint32_t estr[3] = {1, 1, 1};
  return enc(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Which even/odd kernel runs (fvx_dst_kernel_config): 0 = single CTAs with
// 64-element K blocks (default), 1 = CTA pairs (row counts that are
// multiples of 256), 2 = single CTAs with 32-element K blocks.
static int g_sym_kernel = 0;

// C[M, K] = X[M, K] S[K, K] by the even/odd product; X's columns
// de-interleaved; P/Q: the [K/2][K/2] hi/lo tables.  Needs K % 256 == 0.
static int gemm_sym(const bf16* Xh, const bf16* Xl, int M, int K, const bf16* Ph, const bf16* Pl, const bf16* Qh,
                    const bf16* Ql, const Epi& ep_in, cudaStream_t st) {
  Epi ep = ep_in;
  static fvx_once_per_device attr;
  if (fvx_once_on_device(attr, [] {
        return fvx_set_max_smem(gemm_sym_bf16_kernel<64>, SymCfg<64>::SMEM) &&
               fvx_set_max_smem(gemm_sym_bf16_kernel<32>, SymCfg<32>::SMEM);
      }))
    return FVX_ERR_CUDA;
  if (K % (2 * SBN) != 0) return FVX_ERR_SHAPE;
  const int KH = K / 2;
  const uint32_t bki = g_sym_kernel == 2 ? 32 : 64;  // K block of the single-CTA forms
  CUtensorMap a_h, a_l, p_h, p_l, q_h, q_l;
  if (!make_map(&a_h, Xh, K, M, BM, bki) || !make_map(&a_l, Xl, K, M, BM, bki) ||
      !make_map(&p_h, Ph, KH, KH, SBN, bki) || !make_map(&p_l, Pl, KH, KH, SBN, bki) ||
      !make_map(&q_h, Qh, KH, KH, SBN, bki) || !make_map(&q_l, Ql, KH, KH, SBN, bki))
    return FVX_ERR_ARG;
  // staged TMA stores for the split and FP32 outputs when their layout allows
  CUtensorMap o0, o1;
  memset(&o0, 0, sizeof(o0));
  memset(&o1, 0, sizeof(o1));
  ep.tma_out = 0;
  const int R = ep.rows_per_batch;
  if ((ep.mode == EPI_SPLIT || ep.mode == EPI_F32) && R % BM == 0 && M % R == 0 && ep.off_n == 0 &&
      ep.off_r == 0 && ep.n_cols == K && (ep.mode == EPI_F32 || ep.perm_r)) {
    const uint64_t B = (uint64_t)(M / R);
    bool okm = ep.mode == EPI_SPLIT
                   ? make_out_map(&o0, ep.out0, false, R, K, B, ep.ld, ep.batch_stride, 64) &&
                         make_out_map(&o1, ep.out1, false, R, K, B, ep.ld, ep.batch_stride, 64)
                   : make_out_map(&o0, ep.out0, true, R, K, B, ep.ld, ep.batch_stride, 128);
    ep.tma_out = okm ? 1 : 0;
  }
  if (M % (2 * BM) == 0 && g_sym_kernel == 1) {
    // CTA pairs: B blocks of 64 table rows per CTA
    static fvx_once_per_device pattr;
    if (fvx_once_on_device(pattr, [] { return fvx_set_max_smem(gemm_sym_pair_kernel, P_SMEM); }))
      return FVX_ERR_CUDA;
    CUtensorMap p2h, p2l, q2h, q2l;
    if (!make_map(&p2h, Ph, KH, KH, SBN / 2) || !make_map(&p2l, Pl, KH, KH, SBN / 2) ||
        !make_map(&q2h, Qh, KH, KH, SBN / 2) || !make_map(&q2l, Ql, KH, KH, SBN / 2))
      return FVX_ERR_ARG;
    dim3 grid(M / BM, KH / SBN);
    if (grid.y > 65535) return FVX_ERR_SHAPE;
    if (fvx_launch_pdl(gemm_sym_pair_kernel, grid, dim3(S_THREADS), P_SMEM, st, a_h, a_l, p2h, p2l, q2h, q2l, o0,
                       o1, K, ep) != cudaSuccess)
      return FVX_ERR_CUDA;
    return fvx_cuda_status();
  }
  dim3 grid(KH / SBN, (M + BM - 1) / BM);
  if (grid.y > 65535) return FVX_ERR_SHAPE;
  // programmatic launch: the kernel's set-up and its first table loads
  // overlap the previous kernel's tail (the producer waits before reading X)
  const cudaError_t le =
      bki == 32 ? fvx_launch_pdl(gemm_sym_bf16_kernel<32>, grid, dim3(S_THREADS), SymCfg<32>::SMEM, st, a_h, a_l, p_h,
                                 p_l, q_h, q_l, o0, o1, K, ep)
                : fvx_launch_pdl(gemm_sym_bf16_kernel<64>, grid, dim3(S_THREADS), SymCfg<64>::SMEM, st, a_h, a_l, p_h,
                                 p_l, q_h, q_l, o0, o1, K, ep);
  if (le != cudaSuccess) return FVX_ERR_CUDA;
  return fvx_cuda_status();
}

static int gemm_f64(const double* A, int lda, int M, int K, const double* S, int N, const Epi& ep, cudaStream_t st) {
  auto tiles = [&](int t) { return (long long)((N + t - 1) / t) * ((M + t - 1) / t); };
  const int t = tiles(64) >= 148 ? 64 : (tiles(32) >= 148 ? 32 : 16);
  dim3 grid((N + t - 1) / t, (M + t - 1) / t);
  if (grid.y > 65535) return FVX_ERR_SHAPE;
  // programmatic dependent launch: the set-up overlaps the previous
  // kernel's tail (the kernel waits before touching its data)
  cudaError_t e;
  if (t == 64) e = fvx_launch_pdl(gemm_f64_kernel<64>, grid, dim3(256), 0, st, A, lda, S, N, M, N, K, ep);
  else if (t == 32) e = fvx_launch_pdl(gemm_f64_kernel<32>, grid, dim3(256), 0, st, A, lda, S, N, M, N, K, ep);
  else e = fvx_launch_pdl(gemm_f64_kernel<16>, grid, dim3(256), 0, st, A, lda, S, N, M, N, K, ep);
  if (e != cudaSuccess) return FVX_ERR_CUDA;
  return fvx_cuda_status();
}

static int grid1d(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

}  // namespace dst
}  // namespace fvx

using namespace fvx;
using namespace fvx::dst;

struct fvx_dst_plan {
  int ny, nx, batch_max, n_lam;
  int kind = FVX_SPECTRAL_DST;  // transform pair (fvx_spectral_plan_create)
  double dx, dy;
  double cfin = 1.0;            // scale of the last product
  bool split_ok;
  std::vector<double> lam_host;
  double* lam_dev = nullptr;
  bf16 *Sxh = nullptr, *Sxl = nullptr, *Syh = nullptr, *Syl = nullptr;
  bool sym = false;  // even/odd products (nx, ny multiples of 256); operands x/y de-interleaved
  bf16 *xPh = nullptr, *xPl = nullptr, *xQh = nullptr, *xQl = nullptr;  // [nx/2][nx/2]
  bf16 *yPh = nullptr, *yPl = nullptr, *yQh = nullptr, *yQl = nullptr;  // [ny/2][ny/2]
  double *Sx64 = nullptr, *Sy64 = nullptr;
  // inverse-transform operands (DCT-II, periodic); the DST-I plan reuses S
  bf16 *Ixh = nullptr, *Ixl = nullptr, *Iyh = nullptr, *Iyl = nullptr;
  double *Ix64 = nullptr, *Iy64 = nullptr;
  float* inv32 = nullptr;   // [n_lam][ny][nx]
  double* inv64 = nullptr;  // [n_lam][ny][nx]
  bf16 *W1h = nullptr, *W1l = nullptr, *W2h = nullptr, *W2l = nullptr;
  double *V1 = nullptr, *V2 = nullptr;  // FP64 chain work
  double* norms = nullptr;              // [4]
  int* err = nullptr;
  long long wait_cycles = kWaitCycles;  // fvx_dst_plan_set_wait_limit
  int stall = 0;                        // fvx_dst_plan_inject_stall (tests only)
};

static void dst_free(fvx_dst_plan* p) {
  void* ptrs[] = {p->lam_dev, p->Sxh, p->Sxl, p->Syh, p->Syl, p->Sx64, p->Sy64, p->inv32, p->inv64,
                  p->W1h,     p->W1l, p->W2h, p->W2l, p->V1,  p->V2,  p->norms, p->err,
                  p->xPh,     p->xPl, p->xQh, p->xQl, p->yPh, p->yPl, p->yQh,   p->yQl,
                  p->Ixh,     p->Ixl, p->Iyh, p->Iyl, p->Ix64, p->Iy64};
  for (void* q : ptrs)
    if (q) cudaFree(q);
}

// Transform pairs of one axis of length n: forward T[k][j] (coefficient k
// of sample j) and inverse Tinv[j][k] (sample j from coefficient k), FP64,
// row-major, with the 1-D eigenvalues of the 3-point second difference they
// diagonalise.
//   DST-I  (Dirichlet, n interior points): T = sin(pi (j+1)(k+1)/(n+1)),
//          Tinv = T (the 2/(n+1) factors go to the last product's scale),
//          e_k = -4/h^2 sin^2(pi (k+1) / (2(n+1)))
//   DCT-II (Neumann, cell-centred): T = cos(pi k (2j+1) / (2n)),
//          Tinv[j][k] = w_k T[k][j], w_0 = 1/n, w_k = 2/n,
//          e_k = -4/h^2 sin^2(pi k / (2n))
//   periodic: the real Hartley basis T = cos(2 pi k j / n) + sin(2 pi k j / n)
//          (symmetric, T T = n I, and it diagonalises the periodic second
//          difference because e_k = e_{n-k}), Tinv = T / n,
//          e_k = -4/h^2 sin^2(pi k / n)
// Arguments are reduced exactly in integers before the FP64 sin / cos.
static void transform_pair(int kind, int n, double h, std::vector<double>& T, std::vector<double>& Ti,
                           std::vector<double>& e) {
  T.assign((size_t)n * n, 0.0);
  Ti.assign((size_t)n * n, 0.0);
  e.assign(n, 0.0);
  for (int k = 0; k < n; ++k) {
    double sarg;
    if (kind == FVX_SPECTRAL_DST) sarg = M_PI * (k + 1) / (2.0 * (n + 1));
    else if (kind == FVX_SPECTRAL_DCT) sarg = M_PI * k / (2.0 * n);
    else sarg = M_PI * k / (double)n;
    const double sv = std::sin(sarg);
    e[k] = -4.0 / (h * h) * sv * sv;
    for (int j = 0; j < n; ++j) {
      double t;
      if (kind == FVX_SPECTRAL_DST) {
        const long long q = ((long long)(j + 1) * (k + 1)) % (2LL * (n + 1));
        t = std::sin(M_PI * (double)q / (double)(n + 1));
      } else if (kind == FVX_SPECTRAL_DCT) {
        const long long q = ((long long)k * (2 * j + 1)) % (4LL * n);
        t = std::cos(M_PI * (double)q / (2.0 * n));
      } else {
        const long long q = ((long long)k * j) % (long long)n;
        const double a = 2.0 * M_PI * (double)q / (double)n;
        t = std::cos(a) + std::sin(a);
      }
      T[(size_t)k * n + j] = t;
      double w = 1.0;
      if (kind == FVX_SPECTRAL_DCT) w = (k == 0 ? 1.0 : 2.0) / n;
      else if (kind == FVX_SPECTRAL_PERIODIC) w = 1.0 / n;
      Ti[(size_t)j * n + k] = w * t;
    }
  }
}

extern "C" int fvx_spectral_plan_create(int kind, int ny, int nx, double dx, double dy, int batch_max,
                                        const double* lambdas, int n_lambda, int want_fp64, fvx_dst_plan** out);

extern "C" int fvx_dst_plan_create(int ny, int nx, double dx, double dy, int batch_max, const double* lambdas,
                                   int n_lambda, int want_fp64, fvx_dst_plan** out) {
  return fvx_spectral_plan_create(FVX_SPECTRAL_DST, ny, nx, dx, dy, batch_max, lambdas, n_lambda, want_fp64, out);
}

extern "C" int fvx_spectral_plan_create(int kind, int ny, int nx, double dx, double dy, int batch_max,
                                        const double* lambdas, int n_lambda, int want_fp64, fvx_dst_plan** out) {
  if (!out || !lambdas) return FVX_ERR_ARG;
  *out = nullptr;
  if (kind != FVX_SPECTRAL_DST && kind != FVX_SPECTRAL_DCT && kind != FVX_SPECTRAL_PERIODIC) return FVX_ERR_METHOD;
  if (ny < 1 || nx < 1 || batch_max < 1 || n_lambda < 1) return FVX_ERR_SHAPE;
  fvx_dst_plan* p = new fvx_dst_plan();
  p->kind = kind;
  p->ny = ny; p->nx = nx; p->dx = dx; p->dy = dy; p->batch_max = batch_max; p->n_lam = n_lambda;
  p->lam_host.assign(lambdas, lambdas + n_lambda);
  p->split_ok = (nx % 8 == 0) && (ny % 8 == 0);
  p->sym = kind == FVX_SPECTRAL_DST && p->split_ok && nx % (2 * SBN) == 0 && ny % (2 * SBN) == 0;
  p->cfin = kind == FVX_SPECTRAL_DST ? 4.0 / ((double)(ny + 1) * (double)(nx + 1)) : 1.0;
  const bool dst = kind == FVX_SPECTRAL_DST;
  const size_t plane = (size_t)ny * nx, work = plane * batch_max;
  bool ok = true;
  auto A = [&](void** q, size_t bytes) { if (ok && cudaMalloc(q, bytes) != cudaSuccess) ok = false; };
  A((void**)&p->lam_dev, sizeof(double) * n_lambda);
  A((void**)&p->Sx64, sizeof(double) * nx * nx);
  A((void**)&p->Sy64, sizeof(double) * ny * ny);
  if (!dst) {
    A((void**)&p->Ix64, sizeof(double) * nx * nx);
    A((void**)&p->Iy64, sizeof(double) * ny * ny);
  }
  A((void**)&p->inv32, sizeof(float) * plane * n_lambda);
  A((void**)&p->inv64, sizeof(double) * plane * n_lambda);
  A((void**)&p->norms, sizeof(double) * 4);
  A((void**)&p->err, sizeof(int));
  if (p->split_ok) {
    A((void**)&p->Sxh, sizeof(bf16) * nx * nx); A((void**)&p->Sxl, sizeof(bf16) * nx * nx);
    A((void**)&p->Syh, sizeof(bf16) * ny * ny); A((void**)&p->Syl, sizeof(bf16) * ny * ny);
    if (!dst) {
      A((void**)&p->Ixh, sizeof(bf16) * nx * nx); A((void**)&p->Ixl, sizeof(bf16) * nx * nx);
      A((void**)&p->Iyh, sizeof(bf16) * ny * ny); A((void**)&p->Iyl, sizeof(bf16) * ny * ny);
    }
    A((void**)&p->W1h, sizeof(bf16) * work); A((void**)&p->W1l, sizeof(bf16) * work);
    A((void**)&p->W2h, sizeof(bf16) * work); A((void**)&p->W2l, sizeof(bf16) * work);
  }
  if (p->sym) {
    const size_t hx = (size_t)(nx / 2) * (nx / 2), hy = (size_t)(ny / 2) * (ny / 2);
    A((void**)&p->xPh, sizeof(bf16) * hx); A((void**)&p->xPl, sizeof(bf16) * hx);
    A((void**)&p->xQh, sizeof(bf16) * hx); A((void**)&p->xQl, sizeof(bf16) * hx);
    A((void**)&p->yPh, sizeof(bf16) * hy); A((void**)&p->yPl, sizeof(bf16) * hy);
    A((void**)&p->yQh, sizeof(bf16) * hy); A((void**)&p->yQl, sizeof(bf16) * hy);
  }
  if (want_fp64 || !p->split_ok) {
    A((void**)&p->V1, sizeof(double) * work);
    A((void**)&p->V2, sizeof(double) * work);
  }
  if (!ok) { dst_free(p); delete p; return FVX_ERR_CUDA; }
  // host-side tables in FP64.  Operands: the tensor-core products read B
  // as [out][in] (T itself for the forward, Tinv for the inverse); the FP64
  // products read [in][out] (the transposes).
  std::vector<double> Tx, Tix, ex, Ty, Tiy, ey;
  transform_pair(kind, nx, dx, Tx, Tix, ex);
  transform_pair(kind, ny, dy, Ty, Tiy, ey);
  auto transpose = [](const std::vector<double>& M, int n) {
    std::vector<double> R(M.size());
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) R[(size_t)b * n + a] = M[(size_t)a * n + b];
    return R;
  };
  const std::vector<double> Sx = Tx, Sy = Ty;  // split operands [out][in]
  std::vector<double> inv64(plane * n_lambda);
  std::vector<float> inv32(plane * n_lambda);
  for (int l = 0; l < n_lambda; ++l)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        // the null mode (Neumann / periodic Poisson) gets 0: the zero-mean solution
        const double d = (ey[j] + ex[i]) - lambdas[l];
        const double v = d == 0.0 ? 0.0 : 1.0 / d;
        inv64[(size_t)l * plane + (size_t)j * nx + i] = v;
        inv32[(size_t)l * plane + (size_t)j * nx + i] = (float)v;
      }
  cudaMemcpy(p->lam_dev, lambdas, sizeof(double) * n_lambda, cudaMemcpyHostToDevice);
  {
    const std::vector<double> fx = transpose(Tx, nx), fy = transpose(Ty, ny);
    cudaMemcpy(p->Sx64, fx.data(), sizeof(double) * fx.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(p->Sy64, fy.data(), sizeof(double) * fy.size(), cudaMemcpyHostToDevice);
    if (!dst) {
      const std::vector<double> ix = transpose(Tix, nx), iy = transpose(Tiy, ny);
      cudaMemcpy(p->Ix64, ix.data(), sizeof(double) * ix.size(), cudaMemcpyHostToDevice);
      cudaMemcpy(p->Iy64, iy.data(), sizeof(double) * iy.size(), cudaMemcpyHostToDevice);
    }
  }
  cudaMemcpy(p->inv64, inv64.data(), sizeof(double) * inv64.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(p->inv32, inv32.data(), sizeof(float) * inv32.size(), cudaMemcpyHostToDevice);
  if (p->split_ok) {
    auto split = [](const std::vector<double>& S, std::vector<bf16>& h, std::vector<bf16>& l) {
      h.resize(S.size());
      l.resize(S.size());
      for (size_t k = 0; k < S.size(); ++k) {
        h[k] = __float2bfloat16_rn((float)S[k]);
        l[k] = __float2bfloat16_rn((float)(S[k] - (double)__bfloat162float(h[k])));
      }
    };
    std::vector<bf16> h, l;
    split(Sx, h, l);
    cudaMemcpy(p->Sxh, h.data(), sizeof(bf16) * h.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(p->Sxl, l.data(), sizeof(bf16) * l.size(), cudaMemcpyHostToDevice);
    split(Sy, h, l);
    cudaMemcpy(p->Syh, h.data(), sizeof(bf16) * h.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(p->Syl, l.data(), sizeof(bf16) * l.size(), cudaMemcpyHostToDevice);
    if (!dst) {
      split(Tix, h, l);
      cudaMemcpy(p->Ixh, h.data(), sizeof(bf16) * h.size(), cudaMemcpyHostToDevice);
      cudaMemcpy(p->Ixl, l.data(), sizeof(bf16) * l.size(), cudaMemcpyHostToDevice);
      split(Tiy, h, l);
      cudaMemcpy(p->Iyh, h.data(), sizeof(bf16) * h.size(), cudaMemcpyHostToDevice);
      cudaMemcpy(p->Iyl, l.data(), sizeof(bf16) * l.size(), cudaMemcpyHostToDevice);
    }
    if (p->sym) {
      // B_P[k][j'] = S[2j'][k], B_Q[k][j'] = S[2j'+1][k] for k, j' < n/2
      auto halves = [&](const std::vector<double>& S, int n, bf16* Ph, bf16* Pl, bf16* Qh, bf16* Ql) {
        const int hn = n / 2;
        std::vector<double> P((size_t)hn * hn), Q((size_t)hn * hn);
        for (int k = 0; k < hn; ++k)
          for (int j = 0; j < hn; ++j) {
            P[(size_t)k * hn + j] = S[(size_t)(2 * j) * n + k];
            Q[(size_t)k * hn + j] = S[(size_t)(2 * j + 1) * n + k];
          }
        std::vector<bf16> hh, ll;
        split(P, hh, ll);
        cudaMemcpy(Ph, hh.data(), sizeof(bf16) * hh.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(Pl, ll.data(), sizeof(bf16) * ll.size(), cudaMemcpyHostToDevice);
        split(Q, hh, ll);
        cudaMemcpy(Qh, hh.data(), sizeof(bf16) * hh.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(Ql, ll.data(), sizeof(bf16) * ll.size(), cudaMemcpyHostToDevice);
      };
      halves(Sx, nx, p->xPh, p->xPl, p->xQh, p->xQl);
      halves(Sy, ny, p->yPh, p->yPl, p->yQh, p->yQl);
    }
  }
  cudaMemset(p->err, 0, sizeof(int));
  if (cudaDeviceSynchronize() != cudaSuccess) { dst_free(p); delete p; return FVX_ERR_CUDA; }
  *out = p;
  return FVX_OK;
}

extern "C" int fvx_dst_plan_destroy(fvx_dst_plan* p) {
  if (!p) return FVX_ERR_ARG;
  cudaDeviceSynchronize();
  dst_free(p);
  delete p;
  return fvx_cuda_status();
}

// Device error flag of the plan's kernels (1 = a bounded wait gave up).
// Synchronises the stream.
extern "C" int fvx_dst_plan_check(fvx_dst_plan* p, void* stream) {
  if (!p) return FVX_ERR_ARG;
  int e = 0;
  cudaStream_t st = fvx_stream(stream);
  if (cudaMemcpyAsync(&e, p->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return FVX_ERR_CUDA;
  if (e && (cudaMemsetAsync(p->err, 0, sizeof(int), st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess))
    return FVX_ERR_CUDA;  // reported once, then cleared for the plan's next solves
  return e ? FVX_ERR_TIMEOUT : FVX_OK;
}

// Bound on every barrier wait of the plan's tensor-core products, in SM
// clock cycles (default 4e9, about 2 s at 1.97 GHz); a wait that runs out
// ends its CTA without trapping and sets the flag fvx_dst_plan_check reads.
extern "C" int fvx_dst_plan_set_wait_limit(fvx_dst_plan* p, long long cycles) {
  if (!p || cycles < 1000) return FVX_ERR_ARG;
  p->wait_cycles = cycles;
  return FVX_OK;
}

// Fault injection for tests: while on, the products' producer warps issue
// no loads, so their MMA warps wait on barriers that nothing will complete,
// run out after the wait limit and abort (no copy or MMA is in flight).
extern "C" int fvx_dst_plan_inject_stall(fvx_dst_plan* p, int on) {
  if (!p) return FVX_ERR_ARG;
  p->stall = on ? 1 : 0;
  return FVX_OK;
}

static Epi make_epi(fvx_dst_plan* p, int mode, int R, int M, int N, void* o0, void* o1, long long bstride,
                    long long ld, int off_n, int off_r, double alpha, bool eig) {
  Epi e;
  e.mode = mode; e.rows_per_batch = R; e.m_total = M; e.n_cols = N; e.out0 = o0; e.out1 = o1;
  e.batch_stride = bstride; e.ld = ld; e.off_n = off_n; e.off_r = off_r; e.alpha = alpha;
  e.inv_eig = eig ? p->inv32 : nullptr; e.inv_eig64 = eig ? p->inv64 : nullptr; e.n_eig = p->n_lam;
  e.err = p->err;
  e.wait_cycles = p->wait_cycles;
  e.stall = p->stall;
  return e;
}

// The split-BF16 chain on operands already split into W1 ([B][ny][nx]).
// Output: mode EPI_F32 / EPI_F64 / EPI_F64_ACC into ``out`` with batch
// stride ``ob`` and row pitch ``old`` (interior [B][ny][nx] view).
static int chain_split(fvx_dst_plan* p, int B, int out_mode, void* out, long long ob, long long old,
                       cudaStream_t st) {
  const int ny = p->ny, nx = p->nx;
  const double c = p->cfin;
  const bool dst = p->kind == FVX_SPECTRAL_DST;
  const bf16 *Ixh = dst ? p->Sxh : p->Ixh, *Ixl = dst ? p->Sxl : p->Ixl;
  const bf16 *Iyh = dst ? p->Syh : p->Iyh, *Iyl = dst ? p->Syl : p->Iyl;
  int rc;
  if (p->sym) {
    // even/odd products; every intermediate is stored de-interleaved along
    // the next product's contraction axis, the result in natural order
    Epi e1 = make_epi(p, EPI_SPLIT, ny, B * ny, nx, p->W2h, p->W2l, (long long)nx * ny, ny, 0, 0, 1.0, false);
    e1.perm_r = 1;
    if ((rc = gemm_sym(p->W1h, p->W1l, B * ny, nx, p->xPh, p->xPl, p->xQh, p->xQl, e1, st))) return rc;
    Epi e2 = make_epi(p, EPI_SPLIT, nx, B * nx, ny, p->W1h, p->W1l, (long long)ny * nx, nx, 0, 0, 1.0, true);
    e2.perm_r = 1;
    if ((rc = gemm_sym(p->W2h, p->W2l, B * nx, ny, p->yPh, p->yPl, p->yQh, p->yQl, e2, st))) return rc;
    if ((rc = gemm_sym(p->W1h, p->W1l, B * ny, nx, p->xPh, p->xPl, p->xQh, p->xQl, e1, st))) return rc;
    Epi e4 = make_epi(p, out_mode, nx, B * nx, ny, out, nullptr, ob, old, 0, 0, c, false);
    return gemm_sym(p->W2h, p->W2l, B * nx, ny, p->yPh, p->yPl, p->yQh, p->yQl, e4, st);
  }
  // 1: (Q S_x)^T -> W2 [B][nx][ny]
  Epi e1 = make_epi(p, EPI_SPLIT, ny, B * ny, nx, p->W2h, p->W2l, (long long)nx * ny, ny, 0, 0, 1.0, false);
  if ((rc = gemm_split(p->W1h, p->W1l, B * ny, nx, p->Sxh, p->Sxl, nx, e1, st))) return rc;
  // 2: (S_y Q S_x) ./ Lambda -> W1 [B][ny][nx]
  Epi e2 = make_epi(p, EPI_SPLIT, nx, B * nx, ny, p->W1h, p->W1l, (long long)ny * nx, nx, 0, 0, 1.0, true);
  // inv_eig is indexed [n][r] = [y'][x'] = the [ny][nx] grid
  if ((rc = gemm_split(p->W2h, p->W2l, B * nx, ny, p->Syh, p->Syl, ny, e2, st))) return rc;
  // 3: inverse along x -> W2
  if ((rc = gemm_split(p->W1h, p->W1l, B * ny, nx, Ixh, Ixl, nx, e1, st))) return rc;
  // 4: inverse along y, scaled -> out [B][ny][nx]
  Epi e4 = make_epi(p, out_mode, nx, B * nx, ny, out, nullptr, ob, old, 0, 0, c, false);
  return gemm_split(p->W2h, p->W2l, B * nx, ny, Iyh, Iyl, ny, e4, st);
}

static int chain_f64(fvx_dst_plan* p, int B, int out_mode, void* out, long long ob, long long old, cudaStream_t st) {
  const int ny = p->ny, nx = p->nx;
  const double c = p->cfin;
  const bool dst = p->kind == FVX_SPECTRAL_DST;
  const double* Ix = dst ? p->Sx64 : p->Ix64;
  const double* Iy = dst ? p->Sy64 : p->Iy64;
  int rc;
  Epi e1 = make_epi(p, EPI_F64, ny, B * ny, nx, p->V2, nullptr, (long long)nx * ny, ny, 0, 0, 1.0, false);
  if ((rc = gemm_f64(p->V1, nx, B * ny, nx, p->Sx64, nx, e1, st))) return rc;
  Epi e2 = make_epi(p, EPI_F64, nx, B * nx, ny, p->V1, nullptr, (long long)ny * nx, nx, 0, 0, 1.0, true);
  if ((rc = gemm_f64(p->V2, ny, B * nx, ny, p->Sy64, ny, e2, st))) return rc;
  if ((rc = gemm_f64(p->V1, nx, B * ny, nx, Ix, nx, e1, st))) return rc;
  Epi e4 = make_epi(p, out_mode, nx, B * nx, ny, out, nullptr, ob, old, 0, 0, c, false);
  return gemm_f64(p->V2, ny, B * nx, ny, Iy, ny, e4, st);
}

// FP32 solve through the split-BF16 tensor-core chain.  rhs / psi are
// interior views: element (b, y, x) at ptr[b*bstride + y*ld + x].
extern "C" int fvx_dst_solve_f32(fvx_dst_plan* p, const float* rhs, long long rhs_bstride, long long rhs_ld,
                                 float* psi, long long psi_bstride, long long psi_ld, int batch, void* stream) {
  if (!p || !rhs || !psi) return FVX_ERR_ARG;
  if (batch < 1 || batch > p->batch_max) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  long long n = (long long)batch * p->ny * p->nx;
  if (!p->split_ok) {  // sizes the TMA tiles cannot address: FP64 SIMT chain, FP32 output
    if (fvx_launch_pdl(copy_in_f64_kernel<float>, dim3(copy_rows_grid((long long)batch * p->ny)), dim3(256), 0, st,
                       rhs, rhs_bstride, rhs_ld, p->ny, p->nx, batch, p->V1) != cudaSuccess)
      return FVX_ERR_CUDA;
    int rc0 = fvx_cuda_status();
    if (rc0) return rc0;
    return chain_f64(p, batch, EPI_F32, psi, psi_bstride, psi_ld, st);
  }
  split_input_kernel<float><<<grid1d(n), 256, 0, st>>>(rhs, rhs_bstride, rhs_ld, p->ny, p->nx, batch, p->W1h,
                                                        p->W1l, 1.0, p->sym ? 1 : 0);
  int rc = fvx_cuda_status();
  if (rc) return rc;
  return chain_split(p, batch, EPI_F32, psi, psi_bstride, psi_ld, st);
}

// Same chain on operands the caller already split into the plan's first
// workspace (fvx_dst_workspace); used by the fused QG stage kernel.
extern "C" int fvx_dst_solve_presplit_f32(fvx_dst_plan* p, float* psi, long long psi_bstride, long long psi_ld,
                                          int batch, void* stream) {
  if (!p || !psi) return FVX_ERR_ARG;
  if (batch < 1 || batch > p->batch_max || !p->split_ok) return FVX_ERR_SHAPE;
  return chain_split(p, batch, EPI_F32, psi, psi_bstride, psi_ld, fvx_stream(stream));
}

// FP64-residual iterative refinement of an FP32 result: ``passes`` times,
// r = rhs - (lap - lambda) psi evaluated in FP64 from the FP32 rhs and psi,
// split into the chain's operand, and psi += the chain's solve of r.  One
// pass takes the split chain's ~1e-5 relative error (16-bit hi + lo
// intermediates) to the FP32 rounding of psi.  Stream-ordered, no host
// synchronisation (capturable).  Dirichlet plans with split-capable sizes.
extern "C" int fvx_dst_refine_f32(fvx_dst_plan* p, const float* rhs, long long rhs_bstride, long long rhs_ld,
                                  float* psi, long long psi_bstride, long long psi_ld, int batch, int passes,
                                  void* stream) {
  if (!p || !rhs || !psi || passes < 0) return FVX_ERR_ARG;
  if (batch < 1 || batch > p->batch_max || !p->split_ok) return FVX_ERR_SHAPE;
  if (p->kind != FVX_SPECTRAL_DST) return FVX_ERR_METHOD;
  cudaStream_t st = fvx_stream(stream);
  for (int it = 0; it < passes; ++it) {
    residual_kernel<float, float><<<residual_grid(batch * p->ny), 256, 0, st>>>(rhs, rhs_bstride, rhs_ld, psi, psi_bstride, psi_ld,
                                                              p->ny, p->nx, batch, p->dx, p->dy, p->lam_dev,
                                                              p->n_lam, p->W1h, p->W1l, nullptr, p->sym ? 1 : 0);
    int rc = fvx_cuda_status();
    if (rc) return rc;
    if ((rc = chain_split(p, batch, EPI_F32_ACC, psi, psi_bstride, psi_ld, st))) return rc;
  }
  return FVX_OK;
}

// FP64 chain on the input the caller already wrote into the plan's FP64
// workspace (fvx_dst_workspace_f64; the FP64 QG stage kernel writes it):
// the FP64 solve without its input copy.  psi: FP64 interior view.
extern "C" int fvx_dst_solve_presplit_f64(fvx_dst_plan* p, double* psi, long long psi_bstride, long long psi_ld,
                                          int batch, void* stream) {
  if (!p || !psi || !p->V1) return FVX_ERR_ARG;
  if (batch < 1 || batch > p->batch_max) return FVX_ERR_SHAPE;
  return chain_f64(p, batch, EPI_F64, psi, psi_bstride, psi_ld, fvx_stream(stream));
}

// The FP64 chain's input workspace: [batch_max][ny][nx] doubles, natural
// layout (what fvx_dst_solve_presplit_f64 reads).
extern "C" int fvx_dst_workspace_f64(fvx_dst_plan* p, void** v1) {
  if (!p || !v1) return FVX_ERR_ARG;
  *v1 = p->V1;
  return p->V1 ? FVX_OK : FVX_ERR_SHAPE;
}

// Layout of the chain's first operand (the fvx_dst_workspace buffers): 0
// natural [b][y][x]; 1 x de-interleaved, x stored at x / 2 (even x) or
// nx / 2 + x / 2 (odd x) -- the even/odd products of plans whose ny and nx
// are multiples of 256.
extern "C" int fvx_dst_operand_layout(fvx_dst_plan* p) { return p ? (p->sym ? 1 : 0) : -1; }

extern "C" int fvx_dst_workspace(fvx_dst_plan* p, void** w1_hi, void** w1_lo) {
  if (!p || !w1_hi || !w1_lo) return FVX_ERR_ARG;
  *w1_hi = p->W1h;
  *w1_lo = p->W1l;
  return p->split_ok ? FVX_OK : FVX_ERR_SHAPE;
}

// FP64 solve.  method 0: FP64 SIMT chain (one pass).  method 1: split-BF16
// chain + iterative refinement on the FP64 residual until the normwise
// backward error ||r|| / (||A|| ||psi|| + ||f||) <= tol (||A|| the 2-norm
// bound 8/h^2 + lambda) or max_iter passes.  info (host, may be null):
// [passes, backward error, ||r||/||f||].
extern "C" int fvx_dst_solve_f64(fvx_dst_plan* p, const double* rhs, long long rhs_bstride, long long rhs_ld,
                                 double* psi, long long psi_bstride, long long psi_ld, int batch, int method,
                                 double tol, int max_iter, double* info, void* stream) {
  if (!p || !rhs || !psi) return FVX_ERR_ARG;
  if (batch < 1 || batch > p->batch_max) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  const int ny = p->ny, nx = p->nx;
  long long n = (long long)batch * ny * nx;
  int rc;
  if (method == 0 || !p->split_ok) {
    if (!p->V1) return FVX_ERR_ARG;
    if (fvx_launch_pdl(copy_in_f64_kernel<double>, dim3(copy_rows_grid((long long)batch * ny)), dim3(256), 0, st,
                       rhs, rhs_bstride, rhs_ld, ny, nx, batch, p->V1) != cudaSuccess)
      return FVX_ERR_CUDA;
    if ((rc = fvx_cuda_status())) return rc;
    rc = chain_f64(p, batch, EPI_F64, psi, psi_bstride, psi_ld, st);
    if (info) { info[0] = 1; info[1] = -1; info[2] = -1; }
    return rc;
  }
  if (p->kind != FVX_SPECTRAL_DST) return FVX_ERR_METHOD;  // refinement: Dirichlet residual only
  double lam_max = 0;
  for (double l : p->lam_host) lam_max = fmax(lam_max, fabs(l));
  const double anorm = 4.0 / (p->dx * p->dx) + 4.0 / (p->dy * p->dy) + lam_max;
  zero_f64_kernel<<<grid1d(n), 256, 0, st>>>(psi, psi_bstride, psi_ld, ny, nx, batch);
  split_input_kernel<double><<<grid1d(n), 256, 0, st>>>(rhs, rhs_bstride, rhs_ld, ny, nx, batch, p->W1h, p->W1l, 1.0,
                                                         p->sym ? 1 : 0);
  if ((rc = fvx_cuda_status())) return rc;
  double be = 1, rr = 1;
  int it = 0;
  for (it = 1; it <= max_iter; ++it) {
    if ((rc = chain_split(p, batch, EPI_F64_ACC, psi, psi_bstride, psi_ld, st))) return rc;
    cudaMemsetAsync(p->norms, 0, sizeof(double) * 4, st);
    residual_kernel<double, double><<<residual_grid(batch * ny), 256, 0, st>>>(rhs, rhs_bstride, rhs_ld, psi, psi_bstride, psi_ld, ny, nx,
                                                        batch, p->dx, p->dy, p->lam_dev, p->n_lam, p->W1h, p->W1l,
                                                        p->norms, p->sym ? 1 : 0);
    double h[4];
    if (cudaMemcpyAsync(h, p->norms, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return FVX_ERR_CUDA;
    const double rn = sqrt(h[0]), fn = sqrt(h[1]), pn = sqrt(h[2]);
    be = rn / (anorm * pn + fn + 1e-300);
    rr = rn / (fn + 1e-300);
    if (be <= tol) break;
  }
  if (info) { info[0] = it > max_iter ? max_iter : it; info[1] = be; info[2] = rr; }
  return be <= tol ? FVX_OK : FVX_ERR_NOT_CONVERGED;
}

// One product of the split chain on the plan's workspaces, for timing the
// tensor-core GEMM in isolation: which 0 = (W1 S_x)^T -> W2, 1 = (W2 S_y) ./
// Lambda -> W1.  Operands are whatever the workspaces currently hold.
extern "C" int fvx_dst_kernel_config(int kind) {
  if (kind < 0) return g_sym_kernel;
  if (kind > 2) return FVX_ERR_ARG;
  g_sym_kernel = kind;
  return FVX_OK;
}

extern "C" int fvx_dst_gemm_step(fvx_dst_plan* p, int which, int batch, void* stream) {
  if (!p || !p->split_ok) return FVX_ERR_ARG;
  if (batch < 1 || batch > p->batch_max) return FVX_ERR_SHAPE;
  const int ny = p->ny, nx = p->nx;
  cudaStream_t st = fvx_stream(stream);
  if (which == 0) {
    Epi e1 = make_epi(p, EPI_SPLIT, ny, batch * ny, nx, p->W2h, p->W2l, (long long)nx * ny, ny, 0, 0, 1.0, false);
    if (p->sym) {
      e1.perm_r = 1;
      return gemm_sym(p->W1h, p->W1l, batch * ny, nx, p->xPh, p->xPl, p->xQh, p->xQl, e1, st);
    }
    return gemm_split(p->W1h, p->W1l, batch * ny, nx, p->Sxh, p->Sxl, nx, e1, st);
  }
  if (which == 1) {
    Epi e2 = make_epi(p, EPI_SPLIT, nx, batch * nx, ny, p->W1h, p->W1l, (long long)ny * nx, nx, 0, 0, 1.0, true);
    if (p->sym) {
      e2.perm_r = 1;
      return gemm_sym(p->W2h, p->W2l, batch * nx, ny, p->yPh, p->yPl, p->yQh, p->yQl, e2, st);
    }
    return gemm_split(p->W2h, p->W2l, batch * nx, ny, p->Syh, p->Syl, ny, e2, st);
  }
  return FVX_ERR_ARG;
}

// ===========================================================================
// Allocation-free FP32 DST Helmholtz solve.
//
// Some callers cannot call cudaMalloc at solve time: a framework custom call
// (an XLA FFI handler, for instance) where the framework owns every byte of
// device memory and a library-side allocation would bypass its allocator
// and its limits; a host that budgets all device memory up front and
// forbids allocation once it runs; or a latency-critical loop that cannot
// afford cudaMalloc's implicit device synchronisation.  For them,
// fvx_dst_solve_noalloc_f32 runs the same 3xBF16 tensor-core chain as
// fvx_dst_solve_f32 without a plan: its scratch (DST matrices, inverse
// eigenvalue grid, two split operand buffers and an error flag) lives in the
// file-scope array below, which every GPU that loads this library holds
// until the process exits.  The caller still passes rhs and psi.
//
// Limits and rules:
//   * ny and nx (interior sizes) must be multiples of 8 and at most
//     kNoAllocMaxN = 256, batch 1, one lambda; larger sizes return
//     FVX_ERR_SHAPE (1) and touch nothing.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current);
//     make that first call before any stream capture.
//   * Every call shares the one array and overwrites it (tables, operands
//     and the error flag are rewritten or cleared by each call), so calls
//     that overlap on the GPU -- on different streams, or from different
//     host threads -- race and corrupt each other's results.
// ===========================================================================
namespace fvx {
namespace dst {

constexpr int kNoAllocMaxN = 256;
constexpr size_t kNaPlane = (size_t)kNoAllocMaxN * kNoAllocMaxN;
// bf16: S_x hi/lo, S_y hi/lo, W1 hi/lo, W2 hi/lo (8 planes); f32 1/Lambda;
// int error flag (padded to 256 bytes)
constexpr size_t kNoAllocBytes = 8 * kNaPlane * sizeof(bf16) + kNaPlane * sizeof(float) + 256;

static __device__ __align__(256) unsigned char g_dst_noalloc_scratch[kNoAllocBytes];

// DST-I matrices (split into bf16 hi/lo) and 1/Lambda for one (ny, nx, dx,
// dy, lambda), computed in FP64 on the device.
__global__ void noalloc_tables_kernel(int ny, int nx, double dx, double dy, double lam, bf16* sxh, bf16* sxl,
                                      bf16* syh, bf16* syl, float* inv) {
  const int n2 = nx * nx, m2 = ny * ny, p = ny * nx;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n2 + m2 + p; k += gridDim.x * blockDim.x) {
    if (k < n2 + m2) {
      const bool isx = k < n2;
      const int n = isx ? nx : ny, kk = isx ? k : k - n2;
      const int j = kk / n, c = kk - j * n;
      const long long q = ((long long)(j + 1) * (c + 1)) % (2LL * (n + 1));
      const double s = sinpi((double)q / (double)(n + 1));
      const bf16 h = __float2bfloat16_rn((float)s);
      const bf16 l = __float2bfloat16_rn((float)(s - (double)__bfloat162float(h)));
      (isx ? sxh : syh)[kk] = h;
      (isx ? sxl : syl)[kk] = l;
    } else {
      const int kk = k - n2 - m2, j = kk / nx, i = kk - j * nx;
      const double sy = sinpi((double)(j + 1) / (2.0 * (ny + 1)));
      const double sx = sinpi((double)(i + 1) / (2.0 * (nx + 1)));
      const double ey = -4.0 / (dy * dy) * sy * sy, ex = -4.0 / (dx * dx) * sx * sx;
      const double d = (ey + ex) - lam;
      inv[kk] = d == 0.0 ? 0.f : (float)(1.0 / d);  // the plan's rule: a zero eigenvalue divides out as 0
    }
  }
}

}  // namespace dst
}  // namespace fvx

#include <mutex>

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[128] = {nullptr};

// The device address of the scratch array on the current device (looked up
// on first use when ``setup``), or null.
static unsigned char* noalloc_base(bool setup) {
  using namespace fvx::dst;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return nullptr;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev] && setup) {
    // Load this file's module on the current device first (with lazy module
    // loading nothing may have loaded it yet), then look up the array.
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, noalloc_tables_kernel) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_dst_noalloc_scratch) != cudaSuccess || !ptr) {
      cudaGetLastError();
      return nullptr;
    }
    g_noalloc_addr[dev] = ptr;
  }
  return (unsigned char*)g_noalloc_addr[dev];
}

// The error flag inside the scratch array (after the eight bf16 planes and
// the 1/Lambda grid).
static int* noalloc_err(unsigned char* base) {
  using namespace fvx::dst;
  return (int*)((float*)((bf16*)base + 8 * kNaPlane) + kNaPlane);
}

extern "C" int fvx_dst_solve_noalloc_f32(const float* rhs, long long rhs_ld, float* psi, long long psi_ld, int ny,
                                         int nx, double dx, double dy, double lambda, void* stream) {
  using namespace fvx::dst;
  if (!rhs || !psi) return FVX_ERR_ARG;
  if (ny < 8 || nx < 8 || ny > kNoAllocMaxN || nx > kNoAllocMaxN || ny % 8 || nx % 8) return FVX_ERR_SHAPE;
  unsigned char* base = noalloc_base(true);
  if (!base) return FVX_ERR_CUDA;
  cudaStream_t st = fvx_stream(stream);
  bf16* pl = (bf16*)base;
  bf16 *sxh = pl, *sxl = pl + kNaPlane, *syh = pl + 2 * kNaPlane, *syl = pl + 3 * kNaPlane;
  bf16 *w1h = pl + 4 * kNaPlane, *w1l = pl + 5 * kNaPlane, *w2h = pl + 6 * kNaPlane, *w2l = pl + 7 * kNaPlane;
  float* inv = (float*)(pl + 8 * kNaPlane);
  int* err = noalloc_err(base);
  if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return FVX_ERR_CUDA;
  const int total = nx * nx + ny * ny + ny * nx;
  noalloc_tables_kernel<<<(total + 255) / 256, 256, 0, st>>>(ny, nx, dx, dy, lambda, sxh, sxl, syh, syl, inv);
  split_input_kernel<float><<<grid1d((long long)ny * nx), 256, 0, st>>>(rhs, 0, rhs_ld, ny, nx, 1, w1h, w1l, 1.0);
  int rc = fvx_cuda_status();
  if (rc) return rc;
  auto epi = [&](int mode, int R, int M, int N, void* o0, void* o1, long long bs, long long ld, double alpha,
                 bool eig) {
    Epi e;
    e.mode = mode; e.rows_per_batch = R; e.m_total = M; e.n_cols = N; e.out0 = o0; e.out1 = o1;
    e.batch_stride = bs; e.ld = ld; e.off_n = 0; e.off_r = 0; e.alpha = alpha;
    e.inv_eig = eig ? inv : nullptr; e.inv_eig64 = nullptr; e.n_eig = 1; e.err = err;
    return e;
  };
  const double c = 4.0 / ((double)(ny + 1) * (double)(nx + 1));
  if ((rc = gemm_split(w1h, w1l, ny, nx, sxh, sxl, nx, epi(EPI_SPLIT, ny, ny, nx, w2h, w2l, (long long)nx * ny, ny, 1.0, false), st)))
    return rc;
  if ((rc = gemm_split(w2h, w2l, nx, ny, syh, syl, ny, epi(EPI_SPLIT, nx, nx, ny, w1h, w1l, (long long)ny * nx, nx, 1.0, true), st)))
    return rc;
  if ((rc = gemm_split(w1h, w1l, ny, nx, sxh, sxl, nx, epi(EPI_SPLIT, ny, ny, nx, w2h, w2l, (long long)nx * ny, ny, 1.0, false), st)))
    return rc;
  return gemm_split(w2h, w2l, nx, ny, syh, syl, ny, epi(EPI_F32, nx, nx, ny, psi, nullptr, 0, psi_ld, c, false), st);
}

// Reports whether a bounded wait inside the tensor-core products of the last
// allocation-free solve on this device gave up (the solve then returned
// FVX_OK but psi is incomplete): copies the scratch array's error flag to
// the host on ``stream`` and waits for it.  FVX_ERR_TIMEOUT if it is set,
// FVX_OK if it is clear or no allocation-free solve ran on this device.
extern "C" int fvx_dst_noalloc_check(void* stream) {
  unsigned char* base = noalloc_base(false);
  if (!base) return FVX_OK;
  int e = 0;
  cudaStream_t st = fvx_stream(stream);
  if (cudaMemcpyAsync(&e, noalloc_err(base), sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return FVX_ERR_CUDA;
  return e ? FVX_ERR_TIMEOUT : FVX_OK;
}
