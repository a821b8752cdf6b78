// The allocation-free Chebyshev smoothing entry point (its scratch in a file-scope device array).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.h"
#include "kern_vec.cuh"

using namespace hfk;

// =================================================================================================
// Allocation-free Chebyshev smoothing
//
// hfk_chebyshev_smooth allocates its three work vectors (residual, product, direction) on every
// call. This variant takes them from one file-scope device array instead, so that a caller whose
// device memory is fixed after set-up (a host that draws every GPU buffer from a pre-sized pool, or
// an application that forbids further allocation once its solver is built, since cudaMalloc and
// cudaFree synchronise the device and may fail once memory is committed) can smooth without any
// allocation. The array is sized for HFK_NOALLOC_MAX_DOFS free dofs and is held on every GPU that
// loads the library until the process exits.
// =================================================================================================
namespace {

static __device__ __align__(256) double g_noalloc_cheb_scratch[3 * (size_t)HFK_NOALLOC_MAX_DOFS];

constexpr int kNoAllocMaxDevices = 64;
double* g_noalloc_cheb_addr[kNoAllocMaxDevices] = {nullptr};
std::mutex g_noalloc_mutex;

// Device address of the scratch array on the current device (resolved once per device).
double* noalloc_scratch_on(int device) {
  HFK_REQUIRE(device >= 0 && device < kNoAllocMaxDevices, HFK_ERR_UNSUPPORTED, "device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_cheb_addr[device]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_cheb_scratch);
    if (e != cudaSuccess || !ptr)
      throw Error{HFK_ERR_CUDA, std::string("HyperFEMKernels: cudaGetSymbolAddress of the smoother scratch failed: ") +
                                    cudaGetErrorString(e)};
    g_noalloc_cheb_addr[device] = static_cast<double*>(ptr);
  }
  return g_noalloc_cheb_addr[device];
}

// smooth! (src/smoothers.jl:116-146) on caller-provided work vectors r, z, d (same kernels and
// recurrence as cheb_smooth_dev)
void cheb_smooth_on(hfk_problem* p, double* r, double* z, double* d, double a, double b, int degree, const double* rhs,
                    double* x, bool zero_guess, double* residual) {
  const int64_t n = p->nfree;
  const double th = (b + a) / 2, de = (b - a) / 2, sg = th / de;
  if (!zero_guess) mf_apply_dev(p, x, z);
  cheb_start_kernel<double><<<vec_grid(p->nblocks), 256, 0, p->stream>>>(p->nblocks, p->bdofs.p, p->Binv.p, rhs, z, r,
                                                                         d, x, 1.0 / th, zero_guess ? 1 : 0);
  check_launch(p);
  double rho = 1.0 / sg;
  for (int i = 1; i <= degree; ++i) {
    if (i == degree && !residual) break;
    mf_apply_dev(p, d, z);
    const bool last = i == degree;
    double c1 = 0, c2 = 0, rn = 0;
    if (!last) {
      rn = 1.0 / (2 * sg - rho);
      c1 = rn * rho;
      c2 = 2 * rn / de;
    }
    cheb_step_kernel<double><<<vec_grid(p->nblocks), 256, 0, p->stream>>>(p->nblocks, p->bdofs.p, p->Binv.p, z, r, d, x,
                                                                          c1, c2, last ? 0 : 1);
    check_launch(p);
    if (last) break;
    rho = rn;
  }
  if (residual) HFK_CUDA(cudaMemcpyAsync(residual, r, n * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
}

}  // namespace

extern "C" int hfk_chebyshev_smooth_noalloc(hfk_problem* p, double a, double b, int degree, const double* rhs,
                                            double* x, int zero_guess, double* residual) {
  HFK_API_BEGIN
  HFK_REQUIRE(p && rhs && x && degree >= 1 && b > a, HFK_ERR_ARG, "invalid argument");
  HFK_REQUIRE(p->nfree <= (int64_t)HFK_NOALLOC_MAX_DOFS, HFK_ERR_ARG,
              "hfk_chebyshev_smooth_noalloc supports at most " + std::to_string((long long)HFK_NOALLOC_MAX_DOFS) +
                  " free dofs (this operator has " + std::to_string((long long)p->nfree) +
                  "); use hfk_chebyshev_smooth");
  HFK_REQUIRE(is_device_ptr(rhs) && is_device_ptr(x) && (!residual || is_device_ptr(residual)), HFK_ERR_ARG,
              "hfk_chebyshev_smooth_noalloc takes device pointers only (staging host data would allocate)");
  HFK_REQUIRE(is_device_ptr_on(rhs, p->device) && is_device_ptr_on(x, p->device) &&
                  (!residual || is_device_ptr_on(residual, p->device)),
              HFK_ERR_ARG, "hfk_chebyshev_smooth_noalloc: rhs, x and residual must be memory of the operator's GPU");
  HFK_REQUIRE(p->prepared, HFK_ERR_STATE, "the matrix-free Jacobian has not been prepared (call hfk_mf_prepare)");
  HFK_REQUIRE(p->nblocks > 0 && p->blocks_ok, HFK_ERR_STATE, "blocks not built (call hfk_blocks_update)");
  int dev = 0;
  HFK_CUDA(cudaGetDevice(&dev));
  HFK_REQUIRE(dev == p->device, HFK_ERR_STATE, "the current device is not the operator's device");
  double* scratch = noalloc_scratch_on(dev);
  const int64_t n = p->nfree;
  double* r = scratch;
  double* z = scratch + n;
  double* d = scratch + 2 * n;
  // the array keeps the previous call's values: start from zeros
  HFK_CUDA(cudaMemsetAsync(scratch, 0, 3 * n * sizeof(double), p->stream));
  // no autotuning inside this call: the tuner's candidate launches, events and host copies are
  // work the caller did not ask for (a product not tuned yet runs with the default shape)
  struct NoTune {
    hfk_problem* p;
    bool old;
    ~NoTune() { p->no_tune = old; }
  } guard{p, p->no_tune};
  p->no_tune = true;
  cheb_smooth_on(p, r, z, d, a, b, degree, rhs, x, zero_guess != 0, residual);
  HFK_CUDA(cudaStreamSynchronize(p->stream));
  HFK_API_END
}

