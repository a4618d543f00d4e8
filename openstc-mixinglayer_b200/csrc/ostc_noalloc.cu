// ostc_noalloc.cu -- ostc_residual_noalloc: residual norms of two caller-owned states with no device
// allocation at all.
//
// Some callers cannot call cudaMalloc: hosts whose device memory is planned up front and handed out
// by their own pool (allocating behind the pool's back breaks its accounting and can fail once the
// pool holds the whole GPU), loops that must not take the implicit device synchronisation of an
// allocation, and code that runs while another thread captures a CUDA graph in global mode.  This
// entry point needs only the two states the caller already owns and returns four numbers; its
// scratch (per-block partial sums and the final result) lives in a file-scope __device__ array that
// every GPU loading the library holds until the process exits.
#include "ostc.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

namespace ostc {
void set_free_error(const std::string &msg);
}

namespace {

constexpr int kThreads = 256;
constexpr long long kNodesPerBlock = (long long)kThreads * OSTC_NOALLOC_NODES_PER_THREAD;
constexpr int kMaxBlocks = OSTC_NOALLOC_MAX_BLOCKS;

// partial sums [kMaxBlocks][4], then the four RMS results
static __device__ __align__(256) double g_residual_scratch[kMaxBlocks * 4 + 4];

// One block reduces a contiguous chunk of kNodesPerBlock nodes: squared changes of rho, |V|, p, T
// (compute_square_of_dbv, TimeAdvanceFunc.cu:21-37), warp shuffles then shared memory.
__global__ void __launch_bounds__(kThreads) k_res_partial(const double *__restrict__ bn, const double *__restrict__ bo,
                                                          long long n, double *scratch) {
  double acc[4] = {0, 0, 0, 0};
  const long long beg = (long long)blockIdx.x * kNodesPerBlock;
  const long long end = beg + kNodesPerBlock < n ? beg + kNodesPerBlock : n;
  for (long long p = beg + threadIdx.x; p < end; p += kThreads) {
    const double un = bn[n + p], vn = bn[2 * n + p], wn = bn[3 * n + p];
    const double uo = bo[n + p], vo = bo[2 * n + p], wo = bo[3 * n + p];
    const double d0 = bn[p] - bo[p];
    const double d1 = sqrt(un * un + vn * vn + wn * wn) - sqrt(uo * uo + vo * vo + wo * wo);
    const double d2 = bn[4 * n + p] - bo[4 * n + p];
    const double d3 = bn[5 * n + p] - bo[5 * n + p];
    acc[0] += d0 * d0;
    acc[1] += d1 * d1;
    acc[2] += d2 * d2;
    acc[3] += d3 * d3;
  }
  __shared__ double red[kThreads / 32][4];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
  if ((threadIdx.x & 31) == 0)
    for (int q = 0; q < 4; ++q) red[threadIdx.x >> 5][q] = acc[q];
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0;
    for (int w = 0; w < kThreads / 32; ++w) t += red[w][threadIdx.x];
    scratch[(long long)blockIdx.x * 4 + threadIdx.x] = t;
  }
}

// Fixed-order sum of the partials (deterministic for a given size), RMS over the node count.
__global__ void k_res_final(double *scratch, int nblocks, long long n) {
  const int q = threadIdx.x;
  if (q >= 4) return;
  double t = 0;
  for (int b = 0; b < nblocks; ++b) t += scratch[b * 4 + q];
  scratch[kMaxBlocks * 4 + q] = sqrt(t / (double)n);
}

std::mutex g_mu;
constexpr int kMaxDevices = 64;
// per device: the array's device address and the id of the context it was resolved in.  A context
// made anew (after cudaDeviceReset, or a primary context released and retained again) loads the
// module anew, so the address is looked up again whenever the current context's id differs.
double *g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

// id of the current context (cuCtxGetId: unique over the process lifetime), through the driver entry
// point the runtime hands out, so the library needs no link against the driver library
bool current_context_id(unsigned long long *id) {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void *a = nullptr, *b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qb != cudaDriverEntryPointSuccess)
      return false;
    get_current = reinterpret_cast<GetCurrent>(a);
    get_id = reinterpret_cast<GetId>(b);
  }
  CUcontext c = nullptr;
  return get_current(&c) == CUDA_SUCCESS && c && get_id(c, id) == CUDA_SUCCESS;
}

}  // namespace

extern "C" int ostc_residual_noalloc(const double *bv_new, const double *bv_old, long long n_nodes, double res[4],
                                     void *stream) {
  if (!bv_new || !bv_old || !res) {
    ostc::set_free_error("ostc_residual_noalloc: null pointer argument");
    return OSTC_EINVAL;
  }
  if (n_nodes <= 0 || n_nodes > OSTC_NOALLOC_MAX_NODES) {
    ostc::set_free_error("ostc_residual_noalloc: n_nodes = " + std::to_string(n_nodes) +
                         " outside 1.." + std::to_string((long long)OSTC_NOALLOC_MAX_NODES) +
                         " (the static scratch holds partial sums for at most that many nodes)");
    return OSTC_EINVAL;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    ostc::set_free_error("ostc_residual_noalloc: no current CUDA device");
    return OSTC_ECUDA;
  }
  // no context may be current yet (cudaGetDevice does not make one); the symbol lookup below binds
  // the device's primary context, after which its id is read
  unsigned long long ctx_id = 0;
  const bool have_ctx = current_context_id(&ctx_id);
  double *scratch = nullptr;
  {
    // first call on each device (and in each new context): resolve the device address of the static
    // array (host code may not use the symbol itself; it is only a host-side stand-in)
    std::lock_guard<std::mutex> lock(g_mu);
    if (!have_ctx || !g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx_id) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_residual_scratch);
      if (e != cudaSuccess || !p) {
        ostc::set_free_error(std::string("ostc_residual_noalloc: cudaGetSymbolAddress failed: ") +
                             cudaGetErrorString(e));
        return OSTC_ECUDA;
      }
      if (!have_ctx && !current_context_id(&ctx_id)) {
        ostc::set_free_error("ostc_residual_noalloc: cannot identify the current CUDA context");
        return OSTC_ECUDA;
      }
      g_scratch_ptr[dev] = static_cast<double *>(p);
      g_scratch_ctx[dev] = ctx_id;
    }
    scratch = g_scratch_ptr[dev];
  }
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nblocks = (int)((n_nodes + kNodesPerBlock - 1) / kNodesPerBlock);
  k_res_partial<<<nblocks, kThreads, 0, st>>>(bv_new, bv_old, n_nodes, scratch);
  k_res_final<<<1, 32, 0, st>>>(scratch, nblocks, n_nodes);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(res, scratch + kMaxBlocks * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    ostc::set_free_error(std::string("ostc_residual_noalloc: ") + cudaGetErrorString(e));
    return OSTC_ECUDA;
  }
  return OSTC_OK;
}
