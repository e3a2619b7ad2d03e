// Allocation-free Morton ordering: the engine's particle sort (the same key
// and stable radix-sort kernels as tpm_compute_forces) with its scratch in a
// fixed device array compiled into the library, for callers that cannot
// allocate device memory themselves.
//
// Who needs it: a host code that manages all of the GPU's memory through its
// own pool (EUNHA keeps its particles in its own arena) cannot let a library
// call cudaMalloc behind its back: the pool may already hold the whole device,
// and a library allocation escapes its accounting. Time-critical loops are the
// other case: cudaMalloc and cudaFree synchronise the device, which stalls
// every stream the caller keeps busy.
//
// The scratch array below is reserved on every GPU that loads this library
// and stays reserved until the process exits. It holds the second key/index
// buffer of the ping-pong sort and the per-tile digit histograms. Every call
// reuses it and it keeps whatever the previous call left; nothing in it has
// to start at zero, because each pass writes every histogram entry and every
// buffer element it later reads. Two calls whose work overlaps on the GPU
// (different streams, or different host threads on one device) use the same
// array and corrupt each other's results: serialise them.
#include <stdio.h>

#include <mutex>

#include "engine_internal.cuh"
#include "tpm_engine.h"

namespace {

constexpr int64_t kMaxParticles = TPM_NOALLOC_MAX_PARTICLES;
constexpr int64_t kMaxTiles = (kMaxParticles + tpm::kSortTile - 1) / tpm::kSortTile;
constexpr size_t kKeysBytes = sizeof(uint64_t) * kMaxParticles;
constexpr size_t kValsBytes = sizeof(uint32_t) * kMaxParticles;
constexpr size_t kHistBytes = sizeof(uint32_t) * 256 * (kMaxTiles + 1);
constexpr size_t kTotalBytes = kKeysBytes + kValsBytes + kHistBytes + sizeof(uint32_t) * 256;

// The scratch: one array per device, laid out as keys | indices | histograms
// | digit totals. Its name, used in host code, is only a host-side handle;
// the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_sort_scratch[kTotalBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {nullptr};

// The device address of this device's scratch, looked up once per device
// with that device current (the calling thread's current device). It is kept
// for the life of the process: after a cudaDeviceReset the module is loaded
// again in a new context and the kept address would be stale, so the entry
// point is documented as not for use on a device after its reset.
cudaError_t scratch_for_device(int dev, unsigned char **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char *>(g_scratch_addr[dev]);
  return cudaSuccess;
}

// failures are reported through tpm_last_error()
int noalloc_fail(int code, const char *msg, cudaError_t e = cudaSuccess) {
  char buf[256];
  if (e != cudaSuccess)
    snprintf(buf, sizeof(buf), "%s: %s", msg, cudaGetErrorString(e));
  else
    snprintf(buf, sizeof(buf), "%s", msg);
  tpm::set_last_error(buf);
  return code;
}

}  // namespace

extern "C" {

int tpm_morton_order_noalloc(const uint32_t *pos, int64_t np, int32_t n_mesh, uint64_t *keys,
                             uint32_t *perm, void *stream) {
  if (!pos || !keys || !perm) return noalloc_fail(TPM_E_ARG, "NULL device pointer");
  if (np < 1) return noalloc_fail(TPM_E_ARG, "np must be at least 1");
  if (np > kMaxParticles)
    return noalloc_fail(TPM_E_ARG, "np exceeds TPM_NOALLOC_MAX_PARTICLES (the fixed scratch size)");
  if (n_mesh < 16 || n_mesh > 4096) return noalloc_fail(TPM_E_ARG, "n_mesh outside [16, 4096]");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(TPM_E_NODEV, "no current CUDA device", e);
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(TPM_E_ARG, "device index beyond the supported range");
  unsigned char *base = nullptr;
  e = scratch_for_device(dev, &base);
  if (e != cudaSuccess) return noalloc_fail(TPM_E_CUDA, "cudaGetSymbolAddress of the scratch array failed", e);

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint64_t *key_alt = reinterpret_cast<uint64_t *>(base);
  uint32_t *val_alt = reinterpret_cast<uint32_t *>(base + kKeysBytes);
  tpm::SortScratch scr;
  scr.hist = reinterpret_cast<uint32_t *>(base + kKeysBytes + kValsBytes);
  scr.dtotal = reinterpret_cast<uint32_t *>(base + kKeysBytes + kValsBytes + kHistBytes);
  scr.cap_tiles = kMaxTiles;

  tpm::MeshGeom g = tpm::make_geom(n_mesh);
  // keys start in the scratch buffers; the sort has an odd number of passes,
  // so the sorted pairs end in the caller's buffers
  tpm::launch_make_keys(pos, np, (uint32_t)n_mesh, g.sub_bits, key_alt, val_alt, st);
  uint64_t *k = key_alt;
  uint32_t *v = val_alt;
  tpm::radix_sort_pairs(&k, &v, keys, perm, np, kKeyBits, scr, st, nullptr);
  if (k != keys) {
    e = cudaMemcpyAsync(keys, k, sizeof(uint64_t) * np, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(perm, v, sizeof(uint32_t) * np, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return noalloc_fail(TPM_E_CUDA, "copy of the sorted pairs failed", e);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(TPM_E_CUDA, "kernel launch failed", e);
  return 0;
}

}  // extern "C"
