// soapb_noalloc.cu -- the fixed scratch array behind soapb_descriptor_noalloc.
//
// Some callers cannot let a library call cudaMalloc while they run: molecular
// dynamics codes that reserve the GPU's memory in their own pool at start-up
// (a driver allocation then fails, or eats into memory they have promised
// elsewhere), and codes whose time step must not synchronise the device, which
// cudaMalloc and cudaFree may do.  For them the descriptor's per-call scratch
// -- the CSR offsets, mask bits, error word, work counters and the pair rows
// that the pair kernel writes and the site kernel reads -- lives in one array
// of static device memory, sized once here, instead of in buffers that grow
// on demand.
//
// Every GPU that loads this library holds the array until the process exits.
// All calls on a device share it, and it keeps the last call's contents:
// the entry point clears what must start at zero (the work counters) and
// writes everything else before reading it.  Calls whose work overlaps on the
// GPU (two streams, two host threads, two contexts on one device) race on the
// array; serialise them.

#include <cuda_runtime.h>

#include <mutex>

#include "../../include/soap_b200.h"
#include "soapb_internal.h"

// The scratch.  In host code this name stands for the array but is not its
// device address: the address comes from cudaGetSymbolAddress, per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SOAPB_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_addr[kMaxDevices];  // device address of the array, per device; null until set up
}  // namespace

namespace soapb {

// The array's device address on `device`, which must be the current device.
// The first call on a device looks the address up (the set-up); later calls
// return the cached value.  Allocates nothing.
cudaError_t noalloc_scratch(int device, unsigned char **addr, size_t *bytes) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[device]) {
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return e;
    if (cur != device) return cudaErrorInvalidDevice;
    unsigned char *ptr = nullptr;
    e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[device] = ptr;
  }
  *addr = g_addr[device];
  *bytes = sizeof(g_noalloc_scratch);
  return cudaSuccess;
}

}  // namespace soapb
