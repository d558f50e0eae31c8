// Shared definitions for the finitevolx_b200 CUDA library (sm_100a).
//
// Conventions (same as finitevolX): fields are row-major [Ny, Nx] arrays
// with a one-cell ghost ring; U[j,i] sits at i+1/2, V[j,i] at j+1/2 and
// X[j,i] at the north-east corner of T[j,i].  Every entry point takes
// caller-owned device pointers and a cudaStream_t, allocates nothing on the
// hot path, and returns an int status (fvx_status below).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#define DEV __device__ __forceinline__

enum fvx_status {
  FVX_OK = 0,
  FVX_ERR_SHAPE = 1,      // a size or stride is out of the supported range
  FVX_ERR_METHOD = 2,     // unknown scheme / operator code
  FVX_ERR_DTYPE = 3,      // unsupported dtype combination
  FVX_ERR_CUDA = 4,       // a CUDA runtime call failed
  FVX_ERR_NOT_CONVERGED = 5,
  FVX_ERR_ARG = 6,        // a required pointer is null or an argument is invalid
  FVX_ERR_TIMEOUT = 7,    // a bounded device-side wait gave up
};

// Advection schemes (Advection2D method strings, advection/advection.py:360-368).
enum fvx_scheme {
  FVX_NAIVE = 0,
  FVX_UPWIND1 = 1,
  FVX_UPWIND2 = 2,
  FVX_UPWIND3 = 3,
  FVX_WENO3 = 4,
  FVX_WENO5 = 5,
  FVX_WENOZ5 = 6,
  FVX_WENO7 = 7,
  FVX_WENO9 = 8,
  FVX_MINMOD = 9,
  FVX_VAN_LEER = 10,
  FVX_SUPERBEE = 11,
  FVX_MC = 12,
  FVX_WENOZ3 = 13,  // face-flux only (Reconstruction2D.wenoz3_x/_y)
  FVX_NUM_SCHEMES = 14,
};

// Rectangular spectral Helmholtz solvers (solvers/spectral.py:105-128 bc
// names "dst", "dct", "fft").
enum fvx_spectral_kind {
  FVX_SPECTRAL_DST = 0,       // Dirichlet, DST-I
  FVX_SPECTRAL_DCT = 1,       // Neumann, DCT-II
  FVX_SPECTRAL_PERIODIC = 2,  // periodic (FFT), as the real Hartley pair
};

static inline int fvx_cuda_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FVX_OK : FVX_ERR_CUDA;
}

static inline cudaStream_t fvx_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Function attributes (cudaFuncSetAttribute) apply to the current device
// only, and one process may drive several GPUs from several host threads:
// a set-up step that must run once per device keeps one of these per site.
struct fvx_once_per_device {
  std::mutex mu;
  bool done[128] = {};
};

// Runs set() (returns true on success) the first time it is reached with a
// given device current; FVX_ERR_CUDA if set() fails (it runs again next time).
template <typename Fn>
static inline int fvx_once_on_device(fvx_once_per_device& once, Fn&& set) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return FVX_ERR_CUDA;
  std::lock_guard<std::mutex> lock(once.mu);
  if (once.done[dev]) return FVX_OK;
  if (!set()) return FVX_ERR_CUDA;
  once.done[dev] = true;
  return FVX_OK;
}

// cudaFuncAttributeMaxDynamicSharedMemorySize = bytes, once per device.
template <typename K>
static inline bool fvx_set_max_smem(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
}

// ---- programmatic dependent launch ------------------------------------------
// A kernel launched with fvx_launch_pdl may start while the kernel before it
// on the stream is still running (once every CTA of that kernel has executed
// grid_dep_launch or exited).  Such a kernel must execute grid_dep_wait --
// which returns when the previous kernel has completed and its writes are
// visible -- before it reads anything the previous kernel wrote or writes
// anything it may still read.  Without the launch attribute both
// instructions return at once.
#ifdef __CUDACC__
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
static inline cudaError_t fvx_launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                         cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
#endif

// Preconditioner / coarse-solver callback: z = M rho on the given stream;
// returns a status.
typedef int (*fvx_precond_fn)(void* ctx, const void* rho, void* z, void* stream);

template <typename T>
DEV T ldg(const T* p) { return __ldg(p); }
