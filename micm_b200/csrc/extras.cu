// extras.cu -- autotuner, CUDA-graph replay and adjoint entry points.
#include "runtime.hpp"

extern "C"
{
  int micmb_autotune(micmb_solver*, micmb_state*, double, const char*, micmb_fused_config*)
  {
    return MICMB_ERR_UNSUPPORTED;
  }
  int micmb_solve_graph(micmb_solver*, micmb_state*, double, int32_t)
  {
    return MICMB_ERR_UNSUPPORTED;
  }
}
