// noalloc.cu -- micmb_normalized_error_noalloc: the global NormalizedError of
// micmb_normalized_error computed without allocating anything.
//
// Scratch lives in one file-scope device array of fixed size (per-cell sums
// for at most kNoAllocMaxCells cells, plus one slot for the total).  The host
// looks up its address with cudaGetSymbolAddress once per device and caches
// it.  Nothing in the scratch has to start at zero: every slot a call reads is
// written earlier in the same call.  There is one scratch area per device, so
// two calls that overlap in time on the same device (different streams or
// host threads) race on it; callers serialise them.  The cached address
// belongs to the device's primary context: after cudaDeviceReset (or any
// reset of that context) the array is gone and the cached address is stale,
// so the entry point must not be called in a process after such a reset.
#include "runtime.hpp"

#include <cmath>
#include <mutex>

namespace micmb
{
  namespace
  {
    constexpr int64_t kNoAllocMaxCells = 65536;
    constexpr int kMaxDevices = 64;
    constexpr int kBlock = 256;

    // [0, kNoAllocMaxCells): per-cell sums of squared scaled errors; [kNoAllocMaxCells]: their total
    static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxCells + 1];

    std::mutex g_addr_mutex;
    double* g_addr[kMaxDevices] = { nullptr };

    double* ScratchAddress(int device)
    {
      if (device < 0 || device >= kMaxDevices)
        throw Error(MICMB_ERR_UNSUPPORTED, "device ordinal out of range for the fixed scratch table");
      std::lock_guard<std::mutex> lock(g_addr_mutex);
      if (!g_addr[device])
      {
        void* p = nullptr;
        MICMB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_addr[device] = static_cast<double*>(p);
      }
      return g_addr[device];
    }

    __device__ __forceinline__ size_t cell_base(int64_t c, int32_t L, int32_t ncol)
    {
      return (size_t)(c / L) * (size_t)L * (size_t)ncol + (size_t)(c % L);
    }

    // per-cell sum of squared scaled errors in species order, as the per-cell
    // error of micmb_normalized_error forms it
    __global__ void k_error_cells_fixed(int32_t S, const double* y, const double* ynew, const double* err,
                                        const double* atol, double rtol, int64_t n, int32_t L, double* cells)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= n)
        return;
      const size_t bs = cell_base(c, L, S);
      double sum = 0.0;
      for (int32_t i = 0; i < S; ++i)
        sum += scaled_sq(y[bs + (size_t)i * L], ynew[bs + (size_t)i * L], err[bs + (size_t)i * L], atol[i], rtol);
      cells[c] = sum;
    }

    // total over cells in cell order (the order micmb_normalized_error adds them in)
    __global__ void k_sum_in_order(const double* cells, int64_t n, double* total)
    {
      double s = 0.0;
      for (int64_t c = 0; c < n; ++c)
        s += cells[c];
      *total = s;
    }
  }  // namespace
}  // namespace micmb

using namespace micmb;

extern "C" int micmb_normalized_error_noalloc(micmb_solver* solver, micmb_state* state, double* global_out)
{
  return GuardCall([&] {
    if (!solver || !state || state->solver != solver || !global_out)
      throw Error(MICMB_ERR_INVALID_ARGUMENT, "state does not belong to this solver, or no output");
    micmb_state& st = *state;
    const int64_t n = st.n_cells;
    if (n > kNoAllocMaxCells)
      throw Error(MICMB_ERR_INVALID_ARGUMENT, "more cells than the fixed scratch holds (at most 65536)");
    if (!st.ynew.p || !st.forcing0.p)
      throw Error(MICMB_ERR_INVALID_ARGUMENT,
                  "upload MICMB_BUF_SCRATCH_Y and MICMB_BUF_FORCING first (this call allocates nothing)");
    MICMB_CUDA(cudaSetDevice(solver->device));
    double* scratch = ScratchAddress(solver->device);
    const int32_t S = solver->mech->S;
    if (n > 0)
    {
      k_error_cells_fixed<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, st.stream>>>(
          S, st.variables.as<double>(), st.ynew.as<double>(), st.forcing0.as<double>(), st.atol.as<double>(),
          st.rtol, n, st.L, scratch);
      MICMB_CUDA(cudaGetLastError());
    }
    k_sum_in_order<<<1, 1, 0, st.stream>>>(scratch, n, scratch + kNoAllocMaxCells);
    MICMB_CUDA(cudaGetLastError());
    double sum = 0.0;
    MICMB_CUDA(cudaMemcpyAsync(&sum, scratch + kNoAllocMaxCells, sizeof(double), cudaMemcpyDeviceToHost, st.stream));
    MICMB_CUDA(cudaStreamSynchronize(st.stream));
    *global_out = error_from_sum(sum, (double)(n * S > 0 ? n * S : 1));
  });
}
