// ov_noalloc.cu - the direct Biot-Savart point query for callers that cannot
// allocate device memory (ov_direct_points_noalloc, include/openvort_b200.h).
//
// The same kernels as ov_state_eval_points' direct sum run with their scratch
// (the segment table and the per-image partial sums) in one file-scope
// device array of fixed size instead of cudaMalloc'd buffers.  Every GPU
// that loads the library holds that array until the process exits.
#include <mutex>

#include "openvort_b200.h"
#include "ov_internal.h"

namespace {

constexpr size_t kSegBytes = sizeof(double) * 6 * (size_t)OV_NOALLOC_MAX_NODES;
constexpr size_t kFwdBytes = sizeof(int) * (size_t)OV_NOALLOC_MAX_NODES;
constexpr size_t kPartBytes = sizeof(double) * 3 * (size_t)OV_NOALLOC_MAX_POINT_IMAGES;
constexpr size_t kImgBytes = sizeof(double) * 3 * (size_t)OV_NOALLOC_MAX_POINTS;
constexpr size_t kScratchBytes = kSegBytes + kFwdBytes + kPartBytes + kImgBytes;

// Scratch shared by every call on a device.  Host code must not use this
// name as an address: it is a host-side stand-in; the device address comes
// from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_scratch on the current device, looked up on the first
// call per device (with that device current) and kept for the life of the
// process; a cudaDeviceReset of that device makes the kept address stale,
// which the entry point's documentation rules out.
bool scratch_address(unsigned char** out) {
  int dev = -1;
  if (!ov_cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return false;
  if (dev < 0 || dev >= kMaxDevices) {
    ov_set_error(OV_ERR_INVALID, "ov_direct_points_noalloc: device %d beyond %d", dev, kMaxDevices);
    return false;
  }
  std::lock_guard<std::mutex> lk(g_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (!ov_cuda_ok(cudaGetSymbolAddress(&p, g_scratch), "cudaGetSymbolAddress")) return false;
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
  return true;
}

}  // namespace

// Params of the tangle header and globals, as the reference-named calls use
bool ov_capture_header_params(const struct tangle_state* t, OvParams& P);

extern "C" int ov_direct_points_noalloc(const struct tangle_state* header, const double* d_pos,
                                        const int* d_links, const int* d_status, int npts,
                                        const double* d_pts, const int* d_skip, double* d_out,
                                        void* stream) {
  ov_clear_error();
  if (!header || header->N < 0 || npts < 0 || (header->N > 0 && (!d_pos || !d_links || !d_status)) ||
      (npts > 0 && (!d_pts || !d_out))) {
    ov_set_error(OV_ERR_INVALID, "ov_direct_points_noalloc: null or negative argument");
    return OV_ERR_INVALID;
  }
  const int n = header->N;
  if (n > OV_NOALLOC_MAX_NODES) {
    ov_set_error(OV_ERR_INVALID, "ov_direct_points_noalloc: %d nodes exceed the %d the scratch holds",
                 n, OV_NOALLOC_MAX_NODES);
    return OV_ERR_INVALID;
  }
  if (npts > OV_NOALLOC_MAX_POINTS) {
    ov_set_error(OV_ERR_INVALID, "ov_direct_points_noalloc: %d points exceed the %d the scratch holds",
                 npts, OV_NOALLOC_MAX_POINTS);
    return OV_ERR_INVALID;
  }
  const int nimg = header->bimg.n;
  if ((long long)npts * (nimg + 1) > OV_NOALLOC_MAX_POINT_IMAGES) {
    ov_set_error(OV_ERR_INVALID,
                 "ov_direct_points_noalloc: %d points x %d images exceed the %d partial sums the scratch holds",
                 npts, nimg + 1, OV_NOALLOC_MAX_POINT_IMAGES);
    return OV_ERR_INVALID;
  }
  if (npts == 0) return OV_OK;
  OvParams P;
  if (!ov_capture_header_params(header, P)) return ov_last_error();
  unsigned char* base = nullptr;
  if (!scratch_address(&base)) return ov_last_error();
  double* seg = reinterpret_cast<double*>(base);
  int* fwd = reinterpret_cast<int*>(base + kSegBytes);
  double* part = reinterpret_cast<double*>(base + kSegBytes + kFwdBytes);
  double* img = reinterpret_cast<double*>(base + kSegBytes + kFwdBytes + kPartBytes);
  // every scratch element a kernel reads is written earlier in this call, so
  // nothing has to start at zero
  if (!ov_direct_points_scratch(static_cast<cudaStream_t>(stream), P, d_pos,
                                reinterpret_cast<const int2*>(d_links),
                                reinterpret_cast<const int2*>(d_status), n, npts, d_pts, d_skip, seg,
                                fwd, part, d_out, img))
    return ov_last_error();
  return OV_OK;
}
