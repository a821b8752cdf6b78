// Helpers and internal entry points shared by the engine's translation units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "devcache.h"
#include "hfk_internal.h"

namespace hfk {

template <typename R>
struct CellIO;

inline int sm_count() {
  static PerDeviceValue g_sm_count;
  int dev = 0;
  cudaGetDevice(&dev);
  return g_sm_count.get(dev, [dev] {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
  });
}
inline int vec_grid(int64_t n, int threads = 256) {
  int64_t g = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)sm_count() * 8));
}

// ---- pointer classification: device-accessible or host ---------------------------------------
inline bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device memory of GPU `device` (or managed memory, which every GPU can reach)
inline bool is_device_ptr_on(const void* p, int device) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == device);
}

// An input vector on the device: the caller's device pointer, or a copy of host data in `stage`
template <typename T>
const T* dev_in(const T* p, size_t n, DBuf<T>& stage, cudaStream_t s) {
  if (!p) return nullptr;
  if (is_device_ptr(p)) return p;
  stage.resize(std::max(stage.n, n));
  if (n) HFK_CUDA(cudaMemcpyAsync(stage.p, p, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return stage.p;
}
// An output vector: device pointer written directly, or staged and copied back by `finish_out`
template <typename T>
T* dev_out(T* p, size_t n, DBuf<T>& stage) {
  if (is_device_ptr(p)) return p;
  stage.resize(std::max(stage.n, n));
  return stage.p;
}
template <typename T>
void finish_out(T* p, const T* d, size_t n, cudaStream_t s) {
  if (p != d && n) {
    HFK_CUDA(cudaMemcpyAsync(p, d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    HFK_CUDA(cudaStreamSynchronize(s));
  }
}

inline void check_launch(hfk_problem* p) {
  p->launches++;
  HFK_CUDA(cudaGetLastError());
}

// Kernel timing: an event before and after an element-kernel launch sequence (only with timing on)
inline void ktimer_mark(hfk_problem* p) {
  if (!p->ktiming) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;  // no event nodes in captured graphs
  if (cudaStreamIsCapturing(p->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  if (p->kev_used == p->kev.size()) {
    cudaEvent_t e;
    HFK_CUDA(cudaEventCreate(&e));
    p->kev.push_back(e);
  }
  HFK_CUDA(cudaEventRecord(p->kev[p->kev_used++], p->stream));
}

// Raise a kernel's dynamic shared-memory limit on the current device to at least `smem` (`limit`
// records, per device, what was set).
template <typename K>
void raise_smem_limit(K kernel, size_t smem, PerDeviceLimit& limit) {
  int dev = 0;
  HFK_CUDA(cudaGetDevice(&dev));
  limit.raise(dev, smem, [&] {
    HFK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  });
}

// ---- internal entry points defined in hfk_api.cu ----------------------------------------------
void color_cells(hfk_problem* p);                 // color_cells (src/coloring.jl:4-28)
void pattern_build_dev(hfk_problem* p);           // sparsity / cell_positions! (src/assembly.jl:773-899)
bool use_atomic_scatter(const hfk_problem* p);    // the scatter policy of the cell kernels
void mf_apply_dev(hfk_problem* p, const double* dx, double* y);  // y = J dx (device vectors)
CellData cell_data(const hfk_problem* p, const int32_t* cells, int ncells_list);  // the kernels' view

// ---- defined in jv_tc.cu: the FP32 product of Q2 cells on the tensor cores (kern_jv_tc.cuh) ----
constexpr int JV_TC_WARPS = 4;  // warps per CTA (128 cells)
void launch_jv_tc(hfk_problem* p, const int32_t* cells, int ncl, const CellIO<float>& io);

}  // namespace hfk
