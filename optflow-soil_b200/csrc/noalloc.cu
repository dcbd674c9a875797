// noalloc.cu -- the guard's connected-component pass for callers that cannot allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc: a runtime whose pool allocator owns every device
// allocation of the process, or an embedded host that must not grow device memory after start-up. ofc_large_components_noalloc gives them the large-component mask of the
// guard (track._large_components, python/optflow_ref/track.py:45-53) with its union-find scratch in a fixed
// file-scope device array instead of engine-owned buffers: the caller passes device inputs and outputs, and
// the call makes no allocation of any kind.
#include <mutex>

#include "kernels.cuh"

namespace {

// parent[] and size[] of the union-find: OFC_NOALLOC_MAX_PIXELS ints each, 8 MiB that every device which loads
// this library holds until the process exits
__device__ __align__(256) int g_ccl_scratch[2 * (size_t)OFC_NOALLOC_MAX_PIXELS];

std::mutex g_scratch_mu;
int* g_scratch_ptr[128] = {};  // device address of g_ccl_scratch, per device ordinal

void set_msg(char* err, size_t len, const char* m) {
  if (!err || !len) return;
  size_t n = 0;
  while (m[n] && n + 1 < len) {
    err[n] = m[n];
    n++;
  }
  err[n] = 0;
}

}  // namespace

extern "C" int ofc_large_components_noalloc(const uint8_t* d_mask, size_t w, size_t h, double min_area,
                                            uint8_t* d_out, void* stream, char* err, size_t errlen) {
  if (!d_mask || !d_out || w < 1 || h < 1) {
    set_msg(err, errlen, "ofc_large_components_noalloc: null buffer or empty image");
    return OFC_ERR_ARG;
  }
  if (w > (size_t)OFC_NOALLOC_MAX_PIXELS || h > (size_t)OFC_NOALLOC_MAX_PIXELS ||
      w * h > (size_t)OFC_NOALLOC_MAX_PIXELS) {
    std::string m = "ofc_large_components_noalloc: " + std::to_string(w) + " x " + std::to_string(h) +
                    " pixels exceed its fixed scratch of " + std::to_string((size_t)OFC_NOALLOC_MAX_PIXELS) +
                    " pixels; use ofc_finish or an engine call for larger images";
    set_msg(err, errlen, m.c_str());
    return OFC_ERR_WINDOW;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 128) {
    set_msg(err, errlen, e != cudaSuccess ? cudaGetErrorString(e) : "device ordinal out of range");
    return OFC_ERR_DEVICE;
  }
  int* scratch = nullptr;
  {
    // once per device, with that device current: the host-side symbol is not a device address
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
      e = cudaGetSymbolAddress((void**)&g_scratch_ptr[dev], g_ccl_scratch);
      if (e != cudaSuccess) {
        g_scratch_ptr[dev] = nullptr;
        set_msg(err, errlen, cudaGetErrorString(e));
        return OFC_ERR_DEVICE;
      }
    }
    scratch = g_scratch_ptr[dev];
  }
  // an error left pending by the caller's own earlier work would otherwise be reported as this call's failure
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::string m = std::string("ofc_large_components_noalloc: a CUDA error was pending before this call: ") +
                    cudaGetErrorString(e);
    set_msg(err, errlen, m.c_str());
    return OFC_ERR_DEVICE;
  }
  try {
    // k_ccl_init rewrites parent[] and zeroes size[] over the first w * h entries: no state of an earlier call
    // survives into this one
    ofc::launch_large_components(d_mask, (int)w, (int)h, min_area, scratch, scratch + OFC_NOALLOC_MAX_PIXELS, d_out,
                                 (cudaStream_t)stream);
  } catch (const ofc::Error& x) {
    set_msg(err, errlen, x.what());
    return x.status;
  }
  return OFC_OK;
}
