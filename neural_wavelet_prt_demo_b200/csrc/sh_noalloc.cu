// SH projection entry point that allocates no device memory.
//
// nwprt_sh_project needs a caller-provided workspace for its per-block partial sums.
// Some callers cannot produce one: a real-time frame loop that must never hit
// cudaMalloc/cudaFree (they can synchronise the whole device and stall the frame), or an
// embedding host that reserves all device memory up front and forbids allocations it
// does not account for.  nwprt_sh_project_static serves them: its partial sums live in a
// file-scope __device__ array of fixed size that every GPU loading this library holds
// until the process exits.
//
// Host code never uses the array's name as a device address (in host code that name is
// only a host-side stand-in).  Instead, the first call on each device, with that device
// current, looks up the array's device address with cudaGetSymbolAddress and caches it;
// that first call should therefore come before any stream capture.  The cached address
// belongs to the device's current primary context: a host application that calls
// cudaDeviceReset after using this entry point must not call it again in that process.
// Every device holds its own instance of the array.  All calls on one device share that
// instance and it keeps the previous call's contents: every partial sum a call reads is
// written earlier in the same call, so nothing needs clearing, but calls that overlap on
// the same device (for example on two streams) race on it and must be serialised by the
// caller.  Calls on different devices do not race.
#include <mutex>

#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

// Largest supported cubemap face: S = 128, i.e. 6*128*128 texels in 256-texel blocks,
// 243 partial sums (81 coefficients x RGB) per block.
constexpr int kStaticMaxFace = 128;
constexpr size_t kStaticScratchFloats = (size_t)(6 * kStaticMaxFace * kStaticMaxFace / 256) * 243;

static __device__ __align__(256) float g_sh_scratch[kStaticScratchFloats];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
float* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_sh_scratch on the current device (looked up once per device).
float* scratch_on_current_device() {
  int dev = 0;
  NWPRT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) fail(NWPRT_UNSUPPORTED, "device ordinal beyond the static scratch table");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    NWPRT_CUDA(cudaGetSymbolAddress(&p, g_sh_scratch));
    if (!p) fail(NWPRT_CUDA_ERROR, "cudaGetSymbolAddress returned a null address for the SH scratch");
    g_scratch_ptr[dev] = static_cast<float*>(p);
  }
  return g_scratch_ptr[dev];
}

}  // namespace
}  // namespace nwprt

using namespace nwprt;

extern "C" nwprt_status nwprt_sh_project_static(const float* faces, int S, float* L, void* stream) {
  try {
    if (!faces || !L) fail(NWPRT_INVALID_ARG, "nwprt_sh_project_static: null pointer");
    if (S < 1 || S > kStaticMaxFace)
      fail(NWPRT_INVALID_ARG,
           "nwprt_sh_project_static: face size must be in [1, 128]; larger cubemaps need "
           "nwprt_sh_project with a caller workspace");
    if (sh_project_workspace_bytes(S) > kStaticScratchFloats * sizeof(float))
      fail(NWPRT_INVALID_ARG, "nwprt_sh_project_static: static scratch too small for this face size");
    float* scratch = scratch_on_current_device();
    launch_sh_project(faces, S, L, scratch, (cudaStream_t)stream);
    return NWPRT_OK;
  } catch (const Error& e) {
    set_thread_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    set_thread_error(e.what());
    return NWPRT_CUDA_ERROR;
  }
}
