// n3ds_stroke_forward_static: the reference stroke_forward operator with its scratch
// (prepared per-stroke records) in a fixed file-scope device array instead of a
// caller-provided workspace, so the call allocates nothing and needs no buffer from
// the caller.
//
// Scratch: g_scratch below, sized for N3DS_STATIC_MAX_STROKES strokes with the same
// layout n3ds_stroke_forward uses (status word, records, culling arrays, reduction
// slots). Nothing in it has to start at zero: the prep kernel rewrites every record
// and culling entry that the evaluation kernel reads, on every call.
//
// One scratch per device: two calls in flight on the same device at once (on
// different streams or host threads) race on it. Calls on one stream are ordered.
//
// The first call on a device (with that device current) looks up the array's device
// address with cudaGetSymbolAddress, which may load the module; that one-time setup
// is not a stream operation, so a caller that records the call into a stream capture
// makes one call on that device before capturing. The address is kept for the life
// of the process: after cudaDeviceReset (which rebuilds the device's context and
// modules) this entry point must not be called again.
#include <mutex>
#include <string>

#include "../../include/n3ds.h"
#include "n3ds_record.cuh"

namespace n3ds {
int report_error(int code, const std::string& msg);  // sets n3ds_last_error (n3ds_capi.cu)
}

namespace {

// The layout n3ds_stroke_forward uses for N3DS_STATIC_MAX_STROKES strokes (one formula
// for both, built from the record and slot sizes).
constexpr size_t kScratchBytes = n3ds::stroke_workspace_bytes(N3DS_STATIC_MAX_STROKES);
static_assert(kScratchBytes >= n3ds::stroke_workspace_bytes(N3DS_STATIC_MAX_STROKES),
              "static scratch must hold the stroke workspace of N3DS_STATIC_MAX_STROKES strokes");
static_assert(kScratchBytes % 256 == 0, "static scratch keeps the workspace's 256-byte blocks aligned");

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_scratch for the current device (looked up once per device).
int scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return n3ds::report_error(N3DS_ERR_INVALID, "device ordinal " + std::to_string(dev) + " is beyond the " +
                                                    std::to_string(kMaxDevices) + " devices this entry point tracks");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
      return n3ds::report_error(N3DS_ERR_CUDA, std::string("cudaGetSymbolAddress(g_scratch): ") + cudaGetErrorString(e));
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return N3DS_OK;
}

}  // namespace

extern "C" int n3ds_stroke_forward_static(float* alpha_out, float* color_out, float* sdf_out, float* texcoord_out,
                                          int64_t n_texcoord,
                                          const float* x, const float* radius, const float* viewdir,
                                          const float* shape_params, const float* color_params, int64_t n_points,
                                          int64_t n_viewdirs, int64_t n_strokes, int64_t n_shape_params,
                                          int64_t n_color_params, uint32_t sdf_id, uint32_t color_id,
                                          float sdf_delta, int use_laplace_transform, int inv_scale_radius,
                                          n3ds_stream_t stream) {
  if (n_strokes > N3DS_STATIC_MAX_STROKES)
    return n3ds::report_error(N3DS_ERR_INVALID, "n_strokes " + std::to_string(n_strokes) +
                                                    " exceeds the static scratch of n3ds_stroke_forward_static (" +
                                                    std::to_string(N3DS_STATIC_MAX_STROKES) +
                                                    " strokes); use n3ds_stroke_forward with a workspace");
  if (n3ds_stroke_workspace_bytes(n_strokes) > kScratchBytes)
    return n3ds::report_error(N3DS_ERR_INVALID, "static scratch smaller than the stroke workspace layout");
  void* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  return n3ds_stroke_forward(alpha_out, color_out, sdf_out, texcoord_out, n_texcoord, x, radius, viewdir, shape_params,
                             color_params, n_points, n_viewdirs, n_strokes, n_shape_params, n_color_params, sdf_id,
                             color_id, sdf_delta, use_laplace_transform, inv_scale_radius, scratch, kScratchBytes,
                             stream);
}
