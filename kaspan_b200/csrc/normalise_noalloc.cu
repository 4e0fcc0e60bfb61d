// kspn_normalise_noalloc: the canonical relabel of kspn_normalise for
// callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc when they need this step: an
// application whose device memory is already handed out by its own pool or
// caching allocator (a new cudaMalloc can fail or fragment that pool), or a
// latency-critical loop that cannot afford the device-wide synchronisation a
// cudaMalloc/cudaFree pair may cause.  They also cannot hold a kspn_context,
// whose workspace is allocated on first use.  This entry point needs neither:
// its scratch is a fixed file-scope device array, sized for at most
// KSPN_NOALLOC_MAX_N vertices, which every GPU that loads the library keeps
// until the process exits (4 MiB + 256 B).
//
// Rules of use (also stated in include/kspn.h):
//  * n <= KSPN_NOALLOC_MAX_N, else KSPN_ERR_INVALID_ARGUMENT and nothing runs;
//  * the first call on a device looks up the array's device address for that
//    device (cudaGetSymbolAddress) -- make that first call before any stream
//    capture;
//  * all calls share the one array: calls whose work overlaps on the GPU
//    (different streams, or different host threads on one device) race and
//    corrupt each other's result; serialise them;
//  * the call waits for its stream to finish (it reads back an error word);
//  * an id >= n is reported as KSPN_ERR_INVALID_ARGUMENT after the ids < n
//    were relabelled (the array is left partly relabelled).
// Each call rewrites the part of the array it uses before reading it, so
// nothing left by an earlier call leaks into the result.
#include "kspn_internal.cuh"

#include <mutex>

namespace {

constexpr uint32_t NOALLOC_THREADS = 256;
constexpr uint32_t NOALLOC_ERR     = KSPN_NOALLOC_MAX_N; // index of the error word

// scratch[r] = smallest vertex carrying id r; scratch[NOALLOC_ERR] = error word
static __device__ __align__(256) uint32_t g_noalloc_scratch[KSPN_NOALLOC_MAX_N + 64];

// Device address of g_noalloc_scratch per device, looked up once each.
constexpr int   MAX_DEVICES = 64;
std::mutex      g_setup_mutex;
uint32_t*       g_scratch_ptr[MAX_DEVICES] = {};

int
scratch_for_current_device(uint32_t** out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
    cudaGetLastError();
    return KSPN_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    // the symbol's name is only a host-side stand-in; the kernels need the
    // address of this device's copy
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return KSPN_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_scratch_ptr[dev];
  return KSPN_OK;
}

__global__ void
k_noalloc_init(uint32_t n, uint32_t* __restrict__ scratch)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) scratch[i] = kspn::UNDECIDED;
  if (blockIdx.x == 0 && threadIdx.x == 0) scratch[NOALLOC_ERR] = 0;
}

__global__ void
k_noalloc_min(uint32_t n, uint32_t const* __restrict__ id, uint32_t* __restrict__ scratch)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t const r = id[v];
    if (r >= n) {
      scratch[NOALLOC_ERR] = 1;
      continue;
    }
    if (v < __ldcg(scratch + r)) atomicMin(scratch + r, v);
  }
}

__global__ void
k_noalloc_apply(uint32_t n, uint32_t* __restrict__ id, uint32_t const* __restrict__ scratch)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t const r = id[v];
    if (r < n) id[v] = scratch[r];
  }
}

} // namespace

extern "C" int
kspn_normalise_noalloc(uint32_t n, uint32_t* d_scc_id, void* stream)
{
  if (n > KSPN_NOALLOC_MAX_N) return KSPN_ERR_INVALID_ARGUMENT;
  if (n == 0) return KSPN_OK;
  if (!d_scc_id) return KSPN_ERR_INVALID_ARGUMENT;
  uint32_t* scratch = nullptr;
  int const rc      = scratch_for_current_device(&scratch);
  if (rc != KSPN_OK) return rc;
  cudaStream_t const s    = static_cast<cudaStream_t>(stream);
  unsigned const     grid = (n + NOALLOC_THREADS - 1) / NOALLOC_THREADS < 148u * 8 ? (n + NOALLOC_THREADS - 1) / NOALLOC_THREADS : 148u * 8;
  k_noalloc_init<<<grid, NOALLOC_THREADS, 0, s>>>(n, scratch);
  k_noalloc_min<<<grid, NOALLOC_THREADS, 0, s>>>(n, d_scc_id, scratch);
  k_noalloc_apply<<<grid, NOALLOC_THREADS, 0, s>>>(n, d_scc_id, scratch);
  if (cudaGetLastError() != cudaSuccess) return KSPN_ERR_CUDA;
  uint32_t err = 0;
  if (cudaMemcpyAsync(&err, scratch + NOALLOC_ERR, sizeof(err), cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return KSPN_ERR_CUDA;
  }
  // ids >= n were left as they were; the ids < n are relabelled
  return err ? KSPN_ERR_INVALID_ARGUMENT : KSPN_OK;
}
