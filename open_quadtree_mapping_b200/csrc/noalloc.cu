// qm_upsample_noalloc: the upsampling stage (row solve, then column solve)
// with its intermediate buffer in a fixed device array of this library
// instead of a caller-provided workspace.
//
// Who needs it: a host that cannot hand out device memory per call - a
// plugin whose host owns no CUDA allocator, or a real-time loop that must
// not call cudaMalloc/cudaFree after start-up (both synchronise the device
// and can stall the tracking thread for milliseconds).  The entry point
// itself allocates nothing, on the device or through any library.
//
// The scratch holds the row pass's (smoothed depth, smoothed indicator) pair
// per pixel, 8 bytes, for at most QM_UPSAMPLE_NOALLOC_MAX_PIXELS pixels
// (8 MiB).  Nothing in it has to start at zero: the row pass writes every
// pixel of the image before the column pass reads it.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress, which may load this
// library's device code on that device; make that first call before any
// stream capture begins.  Later calls reuse the address while the same CUDA
// context is current; a call under another context (after cudaDeviceReset,
// or with a context the host created and made current itself) looks it up
// again, because the module, and so the array, may sit elsewhere there.
//
// All calls on one device share the one array: two calls whose work can
// overlap on the device (different streams, or different host threads
// without ordering) race on it and both outputs are undefined.  Serialise
// them, e.g. issue them on one stream.
#include <cuda.h>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "engine.h"

namespace qm
{
namespace
{

constexpr size_t kScratchPixels = QM_UPSAMPLE_NOALLOC_MAX_PIXELS;

__device__ __align__(256) float2 g_upsample_scratch[kScratchPixels];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;

// The scratch address of each device, with the id of the context it was
// looked up under (0: none yet).
struct ScratchAddr
{
  unsigned long long ctx_id;
  float2 *ptr;
};
ScratchAddr g_scratch_of_device[kMaxDevices] = {};

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Unique id of the context current on this thread, 0 when none is current
// or the driver cannot say (then the address is looked up on every call).
unsigned long long current_context_id()
{
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved)
  {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
    resolved = true;
  }
  if (!get_current || !get_id)
    return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// Device address of the scratch array on the current device, looked up once
// per device and context.
float2 *scratch_for_current_device()
{
  int dev = -1;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    throw CudaError{QM_ERR_INVALID_ARG, "qm_upsample_noalloc: device ordinal out of range"};
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  ScratchAddr &slot = g_scratch_of_device[dev];
  const unsigned long long ctx = current_context_id();
  if (ctx != 0 && slot.ctx_id == ctx && slot.ptr != nullptr)
    return slot.ptr;
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_upsample_scratch);
  if (e != cudaSuccess || p == nullptr)
  {
    cudaGetLastError();
    throw CudaError{QM_ERR_CUDA, std::string("qm_upsample_noalloc: cudaGetSymbolAddress: ") +
                                     cudaGetErrorString(e)};
  }
  // the lookup may have made the device's primary context current
  slot.ctx_id = ctx != 0 ? ctx : current_context_id();
  slot.ptr = static_cast<float2 *>(p);
  return slot.ptr;
}

void fail_if(bool bad, const char *msg)
{
  if (bad)
    throw CudaError{QM_ERR_INVALID_ARG, msg};
}

int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

} // namespace
} // namespace qm

extern "C" int qm_upsample_noalloc(const float *sparse, const uint8_t *img, size_t img_pitch,
                                   int width, int height, const qm_params *p, float *dense,
                                   void *stream)
{
  using namespace qm;
  try
  {
    fail_if(width < 16 || height < 8 || width > kMaxRowLen || height > kMaxColLen,
            "qm_upsample_noalloc: image size must be within 16 x 8 .. 4096 x 2048");
    fail_if(width % 16 != 0 || height % 8 != 0,
            "qm_upsample_noalloc: width must be a multiple of 16 and height of 8");
    if ((size_t)width * (size_t)height > kScratchPixels)
    {
      char msg[192];
      std::snprintf(msg, sizeof(msg),
                    "qm_upsample_noalloc: %d x %d = %zu pixels exceeds the static scratch "
                    "of %zu pixels; use qm_upsample with a workspace",
                    width, height, (size_t)width * (size_t)height, kScratchPixels);
      throw CudaError{QM_ERR_INVALID_ARG, msg};
    }
    fail_if(!sparse || !img || !dense || img_pitch < (size_t)width,
            "qm_upsample_noalloc: bad argument");
    qm_params q;
    if (p)
      q = *p;
    else
      qm_params_default(&q);
    const std::string err = validate(q);
    fail_if(!err.empty(), err.c_str());

    float2 *scratch = scratch_for_current_device();

    Batch B;
    std::memset(&B, 0, sizeof(B));
    B.njobs = 1;
    JobDesc &J = B.one;
    J.W = width;
    J.H = height;
    J.D = q.num_hyp;
    J.F = 1;
    J.ref = img;
    J.ref_pitch = (int)img_pitch;
    J.sparse = const_cast<float *>(sparse);
    J.dense = dense;
    J.rowres = scratch;
    const KParams kp = kparams(q);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    launch_row_solve(B, cdiv(height, kRowWarps), kp, q.arith, width, s);
    launch_col_solve(B, cdiv(width, kColLines), kp, q.arith, height, s);
    check(cudaGetLastError(), "kernel launch");
    set_error("");
    return QM_OK;
  }
  catch (const CudaError &e)
  {
    set_error(e.msg);
    return e.status;
  }
  catch (...)
  {
    set_error("qm_upsample_noalloc: unexpected error");
    return QM_ERR_CUDA;
  }
}
