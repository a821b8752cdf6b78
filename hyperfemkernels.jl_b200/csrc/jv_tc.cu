// The tensor-core FP32 matrix-free product of Q2 cells (kern_jv_tc.cuh): its per-problem tables and
// its launch. A translation unit of its own, so that the kernel is compiled once.
#include <cuda_runtime.h>

#include "engine.h"
#include "kern_jv_tc.cuh"

namespace hfk {

void launch_jv_tc(hfk_problem* p, const int32_t* cells, int ncl, const CellIO<float>& io) {
  if (!p->tc_tabs.p) {  // the B operands, once per problem (the reference gradients do not change)
    p->tc_tabs.resize(TC_TAB_FLOATS);
    tc_tables_kernel<<<16, 256, 0, p->stream>>>(p->dNt.p, p->tc_tabs.p);
    check_launch(p);
  }
  if (!p->tc_err.p) {
    p->tc_err.resize(1);
    p->tc_err.zero(p->stream);
  }
  static PerDeviceLimit attr;
  raise_smem_limit(jv_tc_kernel, TC_SMEM, attr);
  const int grid = (ncl + TC_CELLS - 1) / TC_CELLS;
  if (grid == 0) return;
  jv_tc_kernel<<<grid, TC_CELLS, TC_SMEM, p->stream>>>(cell_data(p, cells, ncl), p->tc_tabs.p, io, p->tc_err.p);
  check_launch(p);
}

}  // namespace hfk
