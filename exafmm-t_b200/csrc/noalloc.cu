// noalloc.cu -- xfmm_gradient_p2p_noalloc: the direct potential + gradient evaluation of
// xfmm_gradient_p2p with its packed-body scratch in one fixed, file-scope device array instead of
// device memory allocated on every call.
//
// Which callers cannot allocate, and why:
//   - a time-stepping or serving loop that keeps other streams of the device busy: cudaMalloc and
//     cudaFree can synchronise the whole device, so an allocation per call stalls that other work
//     at every step;
//   - a process whose device memory is handed out once at start-up (another framework's caching
//     allocator holds the rest of the device): a fresh allocation in the middle of a run can fail
//     or fragment that pool.
// The array below is part of this library's module image, so it is reserved on a device when the
// module is loaded there, not by this entry point.
//
// Set-up: the first call on each device looks the array's address up with cudaGetSymbolAddress,
// with that device current, and keeps it per device; that first call may load the module on the
// device, so make it before any stream capture begins.  Later calls on that device only launch.
//
// Limits and rules:
//   - scratch: the packed sources (40 bytes each) and targets (32 bytes each), each region rounded
//     up to 256 bytes, must fit in XFMM_NOALLOC_SCRATCH_BYTES; larger sizes are rejected with
//     XFMM_ERR_ARG before anything is launched;
//   - all pointers are device (or managed) memory of the current device; host pointers are
//     rejected;
//   - nothing in the scratch has to start at zero: the packing kernels write every entry that the
//     evaluation kernel reads.  `out` is accumulated into, as by xfmm_gradient_p2p, so it must hold
//     the values to add to (zeros for the plain result);
//   - the work is queued on `stream` and the call returns without waiting;
//   - there is one scratch array per device: calls that overlap on one device (two streams, two
//     host threads) write the same scratch and race.  Order them, e.g. on one stream.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>

#include "xfmm_internal.h"

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[XFMM_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::atomic<uintptr_t> g_scratch_addr[kMaxDevices];  // 0 until the device's first call

// Address of g_noalloc_scratch on the current device (looked up once per device; racing first calls
// look up the same address, so no lock is needed).
unsigned char* scratch_of_current_device() {
  int dev = -1;
  XCUDA(cudaGetDevice(&dev));
  XREQUIRE(dev >= 0 && dev < kMaxDevices, XFMM_ERR_UNSUPPORTED, "device ordinal beyond the no-alloc scratch table");
  uintptr_t a = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!a) {
    void* p = nullptr;
    XCUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    XREQUIRE(p != nullptr, XFMM_ERR_CUDA, "cudaGetSymbolAddress returned a null scratch address");
    a = (uintptr_t)p;
    g_scratch_addr[dev].store(a, std::memory_order_release);
  }
  return (unsigned char*)a;
}

void require_device_pointer(const void* p, int dev, const char* what) {
  cudaPointerAttributes at{};
  XCUDA(cudaPointerGetAttributes(&at, p));
  const bool ok = at.type == cudaMemoryTypeManaged || (at.type == cudaMemoryTypeDevice && at.device == dev);
  if (!ok)
    throw xfmm::Error(XFMM_ERR_ARG, std::string("xfmm_gradient_p2p_noalloc: ") + what +
                                        " is not device memory of the current device");
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" xfmm_status xfmm_gradient_p2p_noalloc(int kernel, double k_re, double k_im, int precision,
                                                 const double* src_xyz, int64_t nsrc, const double* q,
                                                 const double* trg_xyz, int64_t ntrg, double* out, void* stream) {
  try {
    XREQUIRE(kernel >= 0 && kernel <= 2, XFMM_ERR_ARG, "unknown kernel");
    XREQUIRE(nsrc >= 0 && ntrg >= 0, XFMM_ERR_ARG, "negative size");
    XREQUIRE(precision == XFMM_FP64 || precision == XFMM_MIXED, XFMM_ERR_ARG, "unknown precision");
    if (ntrg == 0) return XFMM_OK;
    XREQUIRE(src_xyz && q && trg_xyz && out, XFMM_ERR_ARG, "null argument");
    // scratch layout: sources (x, y, z, Re q) | Im q of the sources | targets (x, y, z, 0)
    constexpr int64_t kMaxBodies = (int64_t)XFMM_NOALLOC_SCRATCH_BYTES / 32;
    const int64_t ns1 = nsrc > 0 ? nsrc : 1;
    size_t need = 0, o_qim = 0, o_t4 = 0;
    if (nsrc <= kMaxBodies && ntrg <= kMaxBodies) {
      o_qim = round256((size_t)ns1 * sizeof(double4));
      o_t4 = o_qim + round256((size_t)ns1 * sizeof(double));
      need = o_t4 + round256((size_t)ntrg * sizeof(double4));
    }
    if (need == 0 || need > (size_t)XFMM_NOALLOC_SCRATCH_BYTES) {
      char msg[256];
      std::snprintf(msg, sizeof msg,
                    "xfmm_gradient_p2p_noalloc: nsrc=%lld and ntrg=%lld need more than its fixed scratch of %u "
                    "bytes (40 bytes per source, 32 per target); use xfmm_gradient_p2p",
                    (long long)nsrc, (long long)ntrg, (unsigned)XFMM_NOALLOC_SCRATCH_BYTES);
      throw xfmm::Error(XFMM_ERR_ARG, msg);
    }
    int dev = -1;
    XCUDA(cudaGetDevice(&dev));
    require_device_pointer(src_xyz, dev, "src_xyz");
    require_device_pointer(q, dev, "q");
    require_device_pointer(trg_xyz, dev, "trg_xyz");
    require_device_pointer(out, dev, "out");
    unsigned char* base = scratch_of_current_device();
    xfmm::gradient_p2p_scratch(kernel, k_re, k_im, precision, src_xyz, nsrc, q, trg_xyz, ntrg, out,
                               reinterpret_cast<double4*>(base), reinterpret_cast<double*>(base + o_qim),
                               reinterpret_cast<double4*>(base + o_t4), (cudaStream_t)stream);
    return XFMM_OK;
  } catch (const xfmm::Error& e) {
    xfmm::set_last_error(e.msg.c_str());
    return (xfmm_status)e.code;
  } catch (...) {
    xfmm::set_last_error("xfmm_gradient_p2p_noalloc: unexpected failure");
    return XFMM_ERR_CUDA;
  }
}
