// mathcheck.cu -- micmb_math_eval: the correctly rounded exp, log10 and pow
// the kernels use (crmath.cuh), evaluated element-wise on the host or by a
// kernel, so tests can pin both against exactly rounded values and against
// each other.
#include "runtime.hpp"

namespace micmb
{
  namespace
  {
    __host__ __device__ inline double EvalOne(int32_t fn, double x, double y)
    {
      switch (fn)
      {
        case MICMB_MATH_EXP: return cr_exp(x);
        case MICMB_MATH_LOG10: return cr_log10(x);
        default: return cr_pow(x, y);
      }
    }

    __global__ void k_math_eval(int32_t fn, const double* x, const double* y, double* out, int64_t n)
    {
      const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (i < n)
        out[i] = EvalOne(fn, x[i], y ? y[i] : 0.0);
    }
  }  // namespace
}  // namespace micmb

using namespace micmb;

extern "C" int micmb_math_eval(int32_t function, const double* x, const double* y, double* out, int64_t n,
                               int32_t on_device)
{
  return GuardCall([&] {
    if (function < MICMB_MATH_EXP || function > MICMB_MATH_POW || n < 0 || (n > 0 && (!x || !out)) ||
        (function == MICMB_MATH_POW && n > 0 && !y))
      throw Error(MICMB_ERR_INVALID_ARGUMENT, "unknown function, negative size or missing array");
    if (!on_device)
    {
      for (int64_t i = 0; i < n; ++i)
        out[i] = EvalOne(function, x[i], y ? y[i] : 0.0);
      return;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
      cudaGetLastError();
      throw Error(MICMB_ERR_NO_DEVICE, "no CUDA device");
    }
    if (n == 0)
      return;
    const int block = 256;
    k_math_eval<<<(unsigned)((n + block - 1) / block), block>>>(function, x, y, out, n);
    MICMB_CUDA(cudaGetLastError());
    MICMB_CUDA(cudaDeviceSynchronize());
  });
}
