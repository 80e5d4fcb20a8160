// Allocation-free plane-Couette norm: dnsb_couette_norm_noalloc.
//
// Some callers cannot allocate device memory: a JAX/XLA FFI handler runs
// inside memory that XLA's allocator already owns (a cudaMalloc there can
// fail or stall the runtime).  Such callers also cannot create a
// dnsb_couette context (creation allocates its workspace).  This entry
// point computes the same quantity as dnsb_couette_norm -- the reference's
// sqrt(Simpson_y(sum conj(v) k_metric v) / ly) -- from the caller's field
// alone, keeping its per-mode partial sums in a file-scope device array of
// fixed size instead of context workspace.
//
// Limits and sharing:
//   * at most kNoallocMaxModes = 32768 (kz, kx) modes, i.e. (nz-1)*(nx/2);
//     larger fields are rejected with DNSB_ERR_ARG;
//   * the array lives on every GPU that loads the library until the process
//     exits (256 KiB per device);
//   * every call uses the same array: calls that may overlap on the GPU
//     (different streams without ordering) race and must be serialised by
//     the caller.  Each call writes every partial it later reads, so no
//     clearing is needed between calls and a previous call's leftovers are
//     never used.
//   * host code cannot use the array's name as a device address.  The first
//     call on each device looks the address up with cudaGetSymbolAddress
//     (with that device current) and caches it together with the unique ID
//     of the CUDA context it came from.  A later call from a different
//     context on that device (after cudaDeviceReset, or with another
//     driver-API context current) repeats the look-up, so a stale address
//     is never used.  Do that first call on a device (and the first call
//     after a reset) before any stream capture.
#include <cuda.h>  // CUcontext / CUresult types; the driver functions are
                   // fetched at run time, the library does not link libcuda
#include <mutex>
#include <string>

#include "../../include/dnsb.h"
#include "solver.cuh"

namespace dnsb {

constexpr int kNoallocMaxModes = 32768;
constexpr int kNoallocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoallocMaxModes];

// One warp per mode: sum over the 3 components and y of W_y k_metric |v|^2,
// with the CGL grid y_j = -cos(j pi / (ny-1)) (plane_couette.py:73-77) and
// composite Simpson weights on non-uniform panels (cartesian.py:106-140)
// evaluated in the kernel.
__global__ void couette_mode_norm2_kernel(const double2* __restrict__ v, int nm,
                                          int nkx, int ny, double* partials) {
  const int lane = threadIdx.x & 31;
  const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (m >= nm) return;
  const double km = (m % nkx == 0) ? 1.0 : 2.0;
  const long long cs = (long long)nm * ny;
  const long long mo = (long long)m * ny;
  const double pi = 3.14159265358979323846;
  double acc = 0.0;
  for (int y = lane; y < ny; y += 32) {
    // Simpson weight of point y: contributions of the panels touching it.
    double W = 0.0;
    for (int i = (y % 2 == 0 ? y - 2 : y - 1); i <= y; i += 2) {
      if (i < 0 || i + 2 > ny - 1) continue;
      const double y0 = -cos(i * pi / (ny - 1));
      const double y1 = -cos((i + 1) * pi / (ny - 1));
      const double y2 = -cos((i + 2) * pi / (ny - 1));
      const double h0 = y1 - y0, h1 = y2 - y1;
      const double hs = h0 + h1, hp = h0 * h1, r = h0 / h1;
      if (y == i) W += (hs / 6) * (2 - 1 / r);
      else if (y == i + 1) W += (hs / 6) * (hs * hs / hp);
      else W += (hs / 6) * (2 - r);
    }
    const double2 a = v[mo + y], b = v[cs + mo + y], c = v[2 * cs + mo + y];
    acc += W * km * ((a.x * a.x + a.y * a.y) + (b.x * b.x + b.y * b.y) +
                     (c.x * c.x + c.y * c.y));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) partials[m] = acc;
}

}  // namespace dnsb

namespace {

std::mutex g_noalloc_mutex;

struct NoallocAddress {
  unsigned long long ctx_id = 0;  // context the address belongs to (0: none)
  double* ptr = nullptr;
};
NoallocAddress g_noalloc_addr[dnsb::kNoallocMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique ID of the current context (IDs are never reused within a process);
// 0 if the driver does not provide one.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool fetched = false;
  if (!fetched) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    fetched = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
      get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

}  // namespace

extern "C" int dnsb_couette_norm_noalloc(const void* v, int nx, int ny, int nz,
                                         double ly, double* out_dev,
                                         void* stream) {
  using namespace dnsb;
  if (!v || !out_dev) return set_last_error(DNSB_ERR_ARG, "null argument");
  if (nx < 2 || nz < 2 || nx % 2 || nz % 2 || ny < 3 || ny % 2 == 0 || !(ly > 0))
    return set_last_error(DNSB_ERR_ARG,
                           "nx, nz must be even, ny odd (Simpson rule), ly > 0");
  const long long nm = (long long)(nz - 1) * (nx / 2);
  if (nm > kNoallocMaxModes)
    return set_last_error(DNSB_ERR_ARG,
                          "(nz-1)*(nx/2) exceeds the 32768 modes of the static "
                          "scratch of dnsb_couette_norm_noalloc");
  int dev = 0;
  const cudaError_t de = cudaGetDevice(&dev);
  if (de != cudaSuccess)
    return set_last_error(DNSB_ERR_CUDA,
                          std::string("cudaGetDevice: ") + cudaGetErrorString(de));
  if (dev < 0 || dev >= kNoallocMaxDevices)
    return set_last_error(DNSB_ERR_ARG,
                          "device ordinal " + std::to_string(dev) +
                              " beyond the 64 devices dnsb_couette_norm_noalloc "
                              "keeps scratch addresses for");
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    const unsigned long long ctx_id = current_context_id();
    NoallocAddress& a = g_noalloc_addr[dev];
    if (!a.ptr || ctx_id == 0 || a.ctx_id != ctx_id) {
      // First call on this device, or from another context than the cached
      // address came from: host code needs the symbol's device address in
      // the current context; the array's host-side name is not one.
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
      if (e != cudaSuccess || !p)
        return set_last_error(DNSB_ERR_CUDA,
                              std::string("cudaGetSymbolAddress: ") +
                                  cudaGetErrorString(e));
      a.ptr = static_cast<double*>(p);
      a.ctx_id = ctx_id;
    }
    scratch = a.ptr;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int warps = 4;
  const int grid = (int)((nm + warps - 1) / warps);
  couette_mode_norm2_kernel<<<grid, 32 * warps, 0, st>>>(
      static_cast<const double2*>(v), (int)nm, nx / 2, ny, scratch);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = launch_finalize(scratch, (int)nm, out_dev, 1.0 / ly, 1, st);
  count_launches(2);
  if (e != cudaSuccess)
    return set_last_error(DNSB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return DNSB_OK;
}
