// A dense entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc at all: real-time threads that may not take the
// driver's allocation locks, plugin hosts that own the device heap and forbid
// allocations behind their back, and embedded integrations whose memory budget is
// fixed before the process starts.  For them, de_dense_noalloc_dev runs the same
// dense pipeline as de_dense_dev, with its workspace taken from a file-scope device
// array instead of a caller allocation.
//
// The array is kNoAllocBytes (16 MiB) per device, held by every GPU that loads this
// library until the process exits.  A pair whose workspace (de_dense_workspace_bytes)
// exceeds it is refused with DE_ERR_ARG; at the default census window that covers,
// for example, 320x240 at up to 64 disparities.  The array's head is the pipeline's
// status word, read back with de_workspace_status(NULL, stream, &status).
//
// The array's device address is resolved once per device and kept for the life of
// the process, so a device reset (cudaDeviceReset) while the library is loaded is not
// supported: calls after one would use a stale address.

#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "de_internal.h"

namespace {

constexpr size_t kNoAllocBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};   // device address of the array, per device

// Host code may not use g_noalloc_scratch's name as an address: on the host it is a
// stand-in symbol.  The device address is looked up once per device, with that
// device current.
int scratch_for_current_device(void** out, int* dev_out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  *dev_out = dev;
  if (e != cudaSuccess) return -1;
  if (dev < 0 || dev >= kMaxDevices) return -2;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return -1;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return 0;
}

int scratch_error(int why, int dev) {
  if (why == -2)
    return de::set_error(DE_ERR_UNSUPPORTED,
                         "device %d: the no-allocation entry point supports devices 0..%d",
                         dev, kMaxDevices - 1);
  return de::set_error(DE_ERR_CUDA, "cannot resolve the no-allocation scratch on device %d: %s",
                       dev, cudaGetErrorString(cudaGetLastError()));
}

}  // namespace

extern "C" int de_dense_noalloc_dev(const de_cfg* cfg, const de_pair* pair, void* stream) {
  if (!pair) return de::set_error(DE_ERR_ARG, "pair is NULL");
  size_t need = 0;
  int rc = de_dense_workspace_bytes(cfg, pair, 1, &need);
  if (rc) return rc;
  if (need > kNoAllocBytes)
    return de::set_error(DE_ERR_ARG,
                         "%dx%d needs %zu workspace bytes; the no-allocation scratch holds %zu",
                         pair->W, pair->H, need, kNoAllocBytes);
  void* scratch = nullptr;
  int dev = 0;
  if (const int why = scratch_for_current_device(&scratch, &dev)) return scratch_error(why, dev);
  return de_dense_dev(cfg, pair, 1, scratch, kNoAllocBytes, stream);
}

namespace de {

// The status word at the head of the array, for de_workspace_status(NULL, ...).
int noalloc_status_word(void** out) {
  int dev = 0;
  if (const int why = scratch_for_current_device(out, &dev)) return scratch_error(why, dev);
  return DE_OK;
}

}  // namespace de
