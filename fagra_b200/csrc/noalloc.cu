// fg_bal_cost_noalloc: the BAL objective (sum over observations of
// 0.5 |projection - pixel|^2) evaluated with no device allocation at all.
//
// Who needs it: callers whose device memory is owned entirely by someone else
// — a framework's caching allocator, a real-time pipeline that reserves its
// whole memory budget up front, or an optimizer held to a warmed
// no-allocation contract — cannot let a library call cudaMalloc behind their
// back. fg_bal_cost goes through a problem handle that owns device buffers;
// this entry point takes every input and the output as caller-provided device
// pointers and keeps its scratch (per-camera rotations, per-block partial
// sums, the arrival counter) in one file-scope __device__ array instead.
//
// Limits and sharing: the scratch holds at most FG_NOALLOC_MAX_CAMERAS
// cameras; larger problems are rejected with FG_INVALID_OPTIONS. Every GPU
// that loads the library keeps this array (about 2.4 MB) until the process
// exits. All calls share it and it keeps the previous call's contents, so the
// counter is cleared at the start of every call, and calls whose work
// overlaps on the GPU (different streams, or different host threads without
// ordering) race on it and must not be issued concurrently.
#include "common.cuh"
#include "bal.cuh"
#include "kernels.cuh"
#include <mutex>

namespace fg {

constexpr int64_t NOALLOC_MAX_CAMERAS = 16384;
constexpr int NOALLOC_MAX_BLOCKS = 1024;
// [per-camera prep: 18 doubles x max cameras | partials: 3 x max blocks | counter]
constexpr size_t NOALLOC_DOUBLES = 18 * NOALLOC_MAX_CAMERAS + 3 * NOALLOC_MAX_BLOCKS + 2;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

namespace {
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {};  // device address of the scratch, per device

// Once per device, with that device current: the device address of the array.
fg_status noalloc_scratch(int device, double** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_ptr[device] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[device];
  return FG_OK;
}
}  // namespace

// Same arithmetic as k_bal_cost, with observation indices bounds-checked on the
// device (they come straight from the caller): an out-of-range index counts as
// an invalid evaluation instead of being read.
__global__ void k_bal_cost_noalloc(int64_t nc, int64_t np, int64_t no, const uint32_t* oc, const uint32_t* op,
                                   const double* px, const double* cams, const double* pts, const double* prep,
                                   double* partials, unsigned* counter, double* out) {
  double hi = 0, lo = 0, bad = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < no; k += (int64_t)gridDim.x * blockDim.x) {
    uint32_t c = oc[k], pi = op[k];
    if ((int64_t)c >= nc || (int64_t)pi >= np) {
      bad = 1;
      continue;
    }
    double X[3] = {pts[3 * (int64_t)pi], pts[3 * (int64_t)pi + 1], pts[3 * (int64_t)pi + 2]};
    ObsEval o = bal_eval(prep + 18 * (int64_t)c, cams + 9 * (int64_t)c, X);
    double r0 = o.pixel[0] - px[2 * k], r1 = o.pixel[1] - px[2 * k + 1];
    double v = 0.5 * (r0 * r0 + r1 * r1);
    if (!o.ok || !isfinite(v)) bad = 1;
    else dd_add(hi, lo, v, 0.0);
  }
  for (int o = 16; o > 0; o >>= 1) {
    double h2 = __shfl_down_sync(0xffffffffu, hi, o), l2 = __shfl_down_sync(0xffffffffu, lo, o);
    double b2 = __shfl_down_sync(0xffffffffu, bad, o);
    dd_add(hi, lo, h2, l2);
    bad = fmax(bad, b2);
  }
  __shared__ double sh[32][3];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { sh[warp][0] = hi; sh[warp][1] = lo; sh[warp][2] = bad; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nw = (blockDim.x + 31) >> 5;
    for (int w = 1; w < nw; ++w) {
      dd_add(hi, lo, sh[w][0], sh[w][1]);
      bad = fmax(bad, sh[w][2]);
    }
    partials[3 * blockIdx.x] = hi;
    partials[3 * blockIdx.x + 1] = lo;
    partials[3 * blockIdx.x + 2] = bad;
  }
  if (arrive_last(counter)) {
    if (threadIdx.x == 0) {
      double H = 0, Lo = 0, B = 0;
      for (unsigned b = 0; b < gridDim.x; ++b) {
        dd_add(H, Lo, ((volatile double*)partials)[3 * b], ((volatile double*)partials)[3 * b + 1]);
        B = fmax(B, ((volatile double*)partials)[3 * b + 2]);
      }
      out[0] = H + Lo;
      out[1] = B;
      *counter = 0;
    }
  }
}

}  // namespace fg

using namespace fg;

FG_API fg_status fg_bal_cost_noalloc(size_t cameras, size_t points, size_t observations, const double* camera_params,
                                     const double* point_params, const uint32_t* obs_camera,
                                     const uint32_t* obs_point, const double* obs_pixel, double* out, int device,
                                     void* stream) {
  if (!out) return FG_NULL_ARGUMENT;
  if ((cameras && !camera_params) || (points && !point_params) ||
      (observations && (!obs_camera || !obs_point || !obs_pixel)))
    return FG_NULL_ARGUMENT;
  if (cameras > (size_t)NOALLOC_MAX_CAMERAS) {
    set_error("fg_bal_cost_noalloc: at most 16384 cameras fit the fixed scratch array");
    return FG_INVALID_OPTIONS;
  }
  FG_TRY(select_device(device));
  double* scratch = nullptr;
  FG_TRY(noalloc_scratch(device, &scratch));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* prep = scratch;
  double* partials = scratch + 18 * NOALLOC_MAX_CAMERAS;
  unsigned* counter = reinterpret_cast<unsigned*>(partials + 3 * NOALLOC_MAX_BLOCKS);
  FG_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), st));
  if (cameras) FG_LAUNCH(k_bal_camera_prep, grid_for(cameras, 128), 128, 0, st, (int64_t)cameras, camera_params, prep);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  unsigned g = std::min<unsigned>(grid_for(std::max<size_t>(observations, 1), 256),
                                  (unsigned)std::min(4 * std::max(sms, 1), NOALLOC_MAX_BLOCKS));
  FG_LAUNCH(k_bal_cost_noalloc, g, 256, 0, st, (int64_t)cameras, (int64_t)points, (int64_t)observations, obs_camera,
            obs_point, obs_pixel, camera_params, point_params, prep, partials, counter, out);
  return FG_OK;
}
