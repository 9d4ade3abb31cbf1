// dpt_noalloc.cu - drift_pt_run_noalloc: the PT round loop without any device allocation.
//
// drift_pt_run needs a scratch workspace (error flag, per-round energy publication buffer and
// its round tags, which are also the grid-wide synchronisation) that the caller allocates. Some callers cannot allocate device memory at
// all: code that runs after a framework has reserved the device's memory for its own pool, hosts
// whose allocation policy forbids cudaMalloc outside start-up (real-time or embedded loops), and
// foreign-language bindings that only receive pointers to buffers someone else owns. For them
// this entry point uses a scratch array compiled into the library instead.
//
// The scratch array is a file-scope __device__ variable, so every GPU that loads the library holds
// kNoAllocBytes (about 128 KiB) of it until the process exits. On the host its name is only a
// stand-in symbol, never a device address: the device address is looked up with
// cudaGetSymbolAddress while the device is current. The first call on a device does that set-up;
// later calls look it up again unless their stream is being captured (then the address found by the
// device's previous call is used), so an address cached before a device reset is never used after
// it. drift_pt_noalloc_check reads the array's error flag, the one drift_pt_check reads from a
// caller's workspace.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "../../include/drift_pt.h"
#include "dpt_internal.h"

namespace {

// drift_pt_workspace_bytes(DRIFT_PT_NOALLOC_MAX_REPLICAS): 256-byte header + 32 bytes per replica
constexpr size_t kNoAllocBytes = 256 + 32 * (size_t)DRIFT_PT_NOALLOC_MAX_REPLICAS;

// offset of the int error flag in a workspace (drift_pt_run sets it when a bounded wait gives up)
constexpr size_t kErrFlagOffset = 8;

std::mutex g_mu;
std::vector<void*> g_scratch_addr;  // device address of the scratch array, per device ordinal

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of the scratch array on the current device.
static int scratch_address(void* stream, void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return dpt::set_error(DRIFT_PT_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs);
  if (e != cudaSuccess) return dpt::set_error(DRIFT_PT_ECUDA, "cudaStreamIsCapturing: %s", cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_mu);
  if ((int)g_scratch_addr.size() <= dev) g_scratch_addr.resize(dev + 1, nullptr);
  if (!g_scratch_addr[dev] || cs == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return dpt::set_error(DRIFT_PT_ECUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", dev,
                            cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_run_noalloc(const DriftPtDeviceProblem* prob, const DriftPtRunArgs* args,
                                    DriftPtDeviceState* state, void* stream) {
  dpt::clear_error();
  if (!args) return dpt::set_error(DRIFT_PT_EINVAL, "run args are NULL");
  if (args->n_replicas < 1 || args->n_replicas > DRIFT_PT_NOALLOC_MAX_REPLICAS)
    return dpt::set_error(DRIFT_PT_EUNSUPPORTED,
                          "drift_pt_run_noalloc handles 1..%d replicas (got %d); use drift_pt_run with a "
                          "caller-provided workspace for more",
                          DRIFT_PT_NOALLOC_MAX_REPLICAS, args->n_replicas);
  size_t need = 0;
  int rc = drift_pt_workspace_bytes(args->n_replicas, &need);
  if (rc) return rc;
  if (need > kNoAllocBytes)
    return dpt::set_error(DRIFT_PT_EUNSUPPORTED, "scratch of %zu bytes exceeds the built-in %zu", need, kNoAllocBytes);
  void* scratch = nullptr;
  rc = scratch_address(stream, &scratch);
  if (rc) return rc;
  // drift_pt_run clears the whole scratch (error flag, published energies, round tags) at the
  // start of every launch, so the contents left by the previous call do not matter.
  return drift_pt_run(prob, args, state, scratch, kNoAllocBytes, stream);
}

extern "C" int drift_pt_noalloc_check(void* stream) {
  dpt::clear_error();
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return dpt::set_error(DRIFT_PT_ECUDA, "stream synchronize: %s", cudaGetErrorString(e));
  int flag = 0;
  // a synchronous copy out of the array by its symbol (no staging buffer, nothing allocated)
  e = cudaMemcpyFromSymbol(&flag, g_noalloc_scratch, sizeof flag, kErrFlagOffset, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return dpt::set_error(DRIFT_PT_ECUDA, "error flag read: %s", cudaGetErrorString(e));
  if (flag)
    return dpt::set_error(DRIFT_PT_ETIMEOUT, "a bounded in-kernel wait timed out (flag %d); the state is incomplete",
                          flag);
  return DRIFT_PT_OK;
}
