// Forward rasterization for callers that must not allocate device memory.
//
// Some hosts of this rasterizer cannot call cudaMalloc: a viewer or render plugin living inside
// an application that reserves all device memory up front and forbids further allocation, or a
// fixed-budget real-time loop in which cudaMalloc (which may synchronise the whole device) would
// stall every other stream.  omnigs_lonlat_forward_noalloc serves them: the caller passes only
// the inputs and outputs of omnigs_lonlat_forward, and the geometry / image / binning state lives
// in one file-scope __device__ array of kNoallocScratchBytes (16 MiB), which every GPU that loads
// this library holds until the process exits.
//
// Limits (checked before any work): at most kNoallocMaxGaussians Gaussians and
// kNoallocMaxPixels pixels; the instances must fit the part of the array left after the geometry
// and image state (about 400k instances at the maximum P and image size).  An instance count
// that does not fit is detected on the device and reported as OMNIGS_ERR_CAPACITY.
//
// All calls share the one array, and each call leaves its state there; the forward clears every
// word it relies on being zero before using it.  Two calls whose work overlaps on the GPU (for
// example on two streams) race on the array and must not be issued.
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/omnigs_b200.h"
#include "kernels.h"
#include "layout.h"

namespace omnigs {
namespace {

constexpr size_t kNoallocScratchBytes = size_t(16) << 20;
constexpr int kNoallocMaxGaussians = 32768;
constexpr int64_t kNoallocMaxPixels = 512 * 512;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

int noalloc_fail(int code, const std::string& msg) {
  set_last_error(msg.c_str());  // reported by omnigs_last_error()
  return code;
}

// Device address of g_noalloc_scratch on the current device.  In host code the array's name is
// only a host-side stand-in, so the address is looked up once per device (with that device
// current) and cached.
int scratch_address(void** out) {
  static std::mutex mu;
  static void* addr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return noalloc_fail(OMNIGS_ERR_CUDA, "omnigs_lonlat_forward_noalloc: no current CUDA device");
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return noalloc_fail(OMNIGS_ERR_CUDA, std::string("omnigs_lonlat_forward_noalloc: cudaGetSymbolAddress "
                                                       "failed: ") + cudaGetErrorString(e));
    addr[dev] = p;
  }
  *out = addr[dev];
  return OMNIGS_OK;
}

}  // namespace
}  // namespace omnigs

using namespace omnigs;

extern "C" int omnigs_lonlat_forward_noalloc(const OmnigsLonlatForwardArgs* a, int* num_rendered,
                                             omnigs_stream_t stream) {
  if (a == nullptr || num_rendered == nullptr)
    return noalloc_fail(OMNIGS_ERR_INVALID_ARGUMENT, "omnigs_lonlat_forward_noalloc: NULL argument");
  if (a->P > kNoallocMaxGaussians)
    return noalloc_fail(OMNIGS_ERR_INVALID_ARGUMENT,
                        "omnigs_lonlat_forward_noalloc: P = " + std::to_string(a->P) +
                            " exceeds the no-allocation limit of " + std::to_string(kNoallocMaxGaussians) +
                            " Gaussians; use omnigs_lonlat_forward with caller-allocated buffers");
  if ((int64_t)a->W * a->H > kNoallocMaxPixels)
    return noalloc_fail(OMNIGS_ERR_INVALID_ARGUMENT,
                        "omnigs_lonlat_forward_noalloc: " + std::to_string(a->W) + "x" + std::to_string(a->H) +
                            " exceeds the no-allocation limit of " + std::to_string(kNoallocMaxPixels) +
                            " pixels; use omnigs_lonlat_forward with caller-allocated buffers");
  void* base = nullptr;
  if (int rc = scratch_address(&base)) return rc;
  const size_t geom_bytes = omnigs_lonlat_geom_bytes(a->P < 0 ? 0 : a->P);
  const size_t image_bytes = a->W > 0 && a->H > 0 ? omnigs_lonlat_image_bytes(a->W, a->H) : 0;
  const size_t image_off = align_up(geom_bytes);
  const size_t binning_off = align_up(image_off + image_bytes);
  if (binning_off + omnigs_lonlat_binning_bytes(0) > kNoallocScratchBytes)
    return noalloc_fail(OMNIGS_ERR_INVALID_ARGUMENT,
                        "omnigs_lonlat_forward_noalloc: the scene's state does not fit the scratch array");
  unsigned char* scratch = static_cast<unsigned char*>(base);
  void* geom = scratch;
  void* image = scratch + image_off;
  void* binning = scratch + binning_off;
  const size_t binning_bytes = kNoallocScratchBytes - binning_off;
  int rc = omnigs_lonlat_forward(a, geom, geom_bytes, binning, binning_bytes, image, image_bytes, stream);
  if (rc) return rc;
  uint32_t status = 0;
  rc = omnigs_lonlat_read_status(geom, num_rendered, &status, stream);
  if (rc) return rc;
  if (status & OMNIGS_STATUS_CAPACITY)
    return noalloc_fail(OMNIGS_ERR_CAPACITY,
                        "omnigs_lonlat_forward_noalloc: " + std::to_string(*num_rendered) +
                            " instances exceed the " +
                            std::to_string(omnigs_lonlat_binning_capacity(binning_bytes)) +
                            " that fit the scratch array");
  if (status != 0)
    return noalloc_fail(OMNIGS_ERR_DEVICE, "omnigs_lonlat_forward_noalloc: device status " + std::to_string(status));
  return OMNIGS_OK;
}
