// Canonical contact sort for callers that cannot allocate device memory.
//
// The batch path sorts each scene's contacts with k_csort, whose key scratch (when the keys do not
// fit shared memory) is part of the batch's device arena, allocated by steel_batch_create. Some
// callers cannot call cudaMalloc at all: a robot controller running a fixed-rate loop, where
// cudaMalloc and cudaFree can block and synchronise the whole device for an unbounded time, and a
// host engine that hands all device memory out of its own pool, sized at start-up, leaving nothing
// for a library to allocate. Such a caller owns its input and output buffers and only needs the
// sort. steel_sort_contacts_noalloc gives it that sort with its key scratch in a file-scope
// __device__ array of fixed size (STEEL_NOALLOC_MAX_CONTACTS keys of 16 bytes, 1 MiB), which every
// GPU that loads this library holds until the process exits. The call allocates nothing. Up to
// NOALLOC_SMEM_KEYS padded keys sort in the kernel's static shared memory instead.
//
// The array is shared by every call on a device and keeps the last call's keys. Each launch
// writes every key slot it later reads (real keys, then padding up to the next power of two)
// before the sort reads any, so nothing has to start at zero. Calls whose kernels overlap on the
// GPU (different streams, or several host threads) race on the array and corrupt each other's
// output; the caller must order them, for example on one stream.
//
// The array's device address is looked up with cudaGetSymbolAddress once per CUDA context: the
// first call made in a context (a device's primary context, again after cudaDeviceReset) does the
// look-up, so make that first call before any stream capture. Later calls compare the current
// context's id with the cached one (cuCtxGetId through the runtime's driver entry points) and reuse
// the address.
#include <cuda.h>

#include <mutex>
#include <string>

#include "../../include/steel_b200.h"
#include "contact_key.cuh"

namespace steel {

int set_last_error(int code, const std::string& msg);

namespace {

constexpr uint32_t NOALLOC_THREADS = 1024;
constexpr uint32_t NOALLOC_SMEM_KEYS = 2048;  // 32 KiB of static shared memory
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) uint4 g_sort_scratch[STEEL_NOALLOC_MAX_CONTACTS];

// Same order as k_csort: keys of the n raw records (record c at raw[5c..5c+4], its shape-mu vec4
// at raw[5n + c]), bitonic sort of the power-of-two padded key array, then a gather of the
// records in key order. One block; `gkeys` is the device address of g_sort_scratch, used when the
// padded keys do not fit the block's shared array.
__global__ void __launch_bounds__(NOALLOC_THREADS)
    k_csort_noalloc(const float4* __restrict__ raw, uint32_t nc, float4* __restrict__ out, uint4* gkeys) {
  __shared__ uint4 sk[NOALLOC_SMEM_KEYS];
  uint32_t n2 = 1u;
  while (n2 < nc) n2 <<= 1u;
  uint4* keys = n2 <= NOALLOC_SMEM_KEYS ? sk : gkeys;
  for (uint32_t q = threadIdx.x; q < n2; q += blockDim.x)
    keys[q] = q < nc ? contact_key(raw, q) : make_uint4(0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu);
  __syncthreads();
  for (uint32_t k = 2u; k <= n2; k <<= 1u) {
    for (uint32_t j = k >> 1u; j > 0u; j >>= 1u) {
      for (uint32_t q = threadIdx.x; q < n2 / 2u; q += blockDim.x) {
        uint32_t i = 2u * j * (q / j) + q % j, l = i + j;
        uint4 a = keys[i], b = keys[l];
        if (key_gt(a, b) == ((i & k) == 0u)) { keys[i] = b; keys[l] = a; }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) {
    uint32_t c = keys[i].w;
#pragma unroll
    for (uint32_t q = 0; q < 5u; q++) out[i * 5u + q] = raw[c * 5u + q];
    out[nc * 5u + i] = raw[nc * 5u + c];
  }
}

std::mutex g_setup_mu;
struct ScratchSlot {
  unsigned long long ctx_id = 0;  // cuCtxGetId of the context the address belongs to (ids start at 1)
  uint4* ptr = nullptr;
};
ScratchSlot g_scratch[MAX_DEVICES];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the calling thread's current context (0 when it cannot be read).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    (void)cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_sort_scratch on `dev`, which must be the current device. Looked up in the
// first call of each context and cached with the context's id; a new context (after
// cudaDeviceReset, or a primary context released and retained again) looks it up again. When the
// id cannot be read the address is looked up on every call.
int scratch_address(int dev, uint4** out) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  const unsigned long long id = current_context_id();
  ScratchSlot& slot = g_scratch[dev];
  if (!slot.ptr || id == 0 || slot.ctx_id != id) {
    uint4* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_sort_scratch);
    if (e != cudaSuccess)
      return set_last_error(STEEL_E_CUDA, std::string("steel_sort_contacts_noalloc: scratch address: ") +
                                               cudaGetErrorString(e));
    slot.ptr = p;
    slot.ctx_id = id;
  }
  *out = slot.ptr;
  return STEEL_OK;
}

// A pointer the current device can dereference (device, managed or mapped host memory).
bool device_visible(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeDevice) return a.device == dev;
  return (a.type == cudaMemoryTypeManaged || a.type == cudaMemoryTypeHost) && a.devicePointer == p;
}

}  // namespace
}  // namespace steel

extern "C" int steel_sort_contacts_noalloc(const float* raw, uint32_t n, float* sorted, void* stream) {
  using namespace steel;
  const char* fn = "steel_sort_contacts_noalloc: ";
  if (n > STEEL_NOALLOC_MAX_CONTACTS)
    return set_last_error(STEEL_E_CAPACITY, std::string(fn) + std::to_string(n) + " contacts exceed the maximum of " +
                                                std::to_string(STEEL_NOALLOC_MAX_CONTACTS) +
                                                " held by the static sort scratch");
  if (n == 0) return STEEL_OK;
  if (!raw || !sorted) return set_last_error(STEEL_E_INVALID, std::string(fn) + "null buffer");
  if ((reinterpret_cast<uintptr_t>(raw) | reinterpret_cast<uintptr_t>(sorted)) & 15u)
    return set_last_error(STEEL_E_INVALID, std::string(fn) + "buffers must be 16-byte aligned");
  const uintptr_t bytes = 96ull * n, r0 = reinterpret_cast<uintptr_t>(raw), s0 = reinterpret_cast<uintptr_t>(sorted);
  if (r0 < s0 + bytes && s0 < r0 + bytes)
    return set_last_error(STEEL_E_INVALID, std::string(fn) + "input and output buffers overlap");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_last_error(STEEL_E_NODEVICE, std::string(fn) + cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES)
    return set_last_error(STEEL_E_INVALID, std::string(fn) + "device ordinal beyond " + std::to_string(MAX_DEVICES));
  if (!device_visible(raw, dev) || !device_visible(sorted, dev))
    return set_last_error(STEEL_E_INVALID, std::string(fn) + "buffers must be memory the current device can access");
  uint4* keys = nullptr;
  if (int rc = scratch_address(dev, &keys)) return rc;
  k_csort_noalloc<<<1, NOALLOC_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float4*>(raw), n, reinterpret_cast<float4*>(sorted), keys);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_last_error(STEEL_E_CUDA, std::string(fn) + "launch: " + cudaGetErrorString(e));
  return STEEL_OK;
}
