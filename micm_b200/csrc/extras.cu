// extras.cu -- autotuner and CUDA-graph replay of the fused solve.
#include "runtime.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace micmb
{
  namespace
  {
    template<class F>
    int GuardX(F&& f)
    {
      return GuardCall(std::forward<F>(f));
    }

    void NeedX(bool ok, const char* what)
    {
      if (!ok)
        throw Error(MICMB_ERR_INVALID_ARGUMENT, what);
    }

    // cache key: tables, tableau and the GPU (SM count, shared memory)
    std::string TuneKey(const micmb_solver& s)
    {
      char buf[128];
      std::snprintf(buf, sizeof(buf), "%016llx:%d:%d:%zu", (unsigned long long)s.mech->hash, s.params.stages,
                    s.sm_count, s.smem_optin);
      return buf;
    }

    bool ReadCache(const char* path, const std::string& key, micmb_fused_config& cfg)
    {
      if (!path)
        return false;
      std::ifstream in(path);
      std::string line;
      bool found = false;
      while (std::getline(in, line))
      {
        std::istringstream ls(line);
        std::string k;
        micmb_fused_config c{};
        if (ls >> k >> c.cells_per_cta >> c.lu_in_shared >> c.ctas_per_sm >> c.ring_slots >> c.variant && k == key)
        {
          cfg = c;  // the last entry for a key wins
          found = true;
        }
      }
      return found;
    }

    void AppendCache(const char* path, const std::string& key, const micmb_fused_config& c)
    {
      if (!path)
        return;
      std::ofstream out(path, std::ios::app);
      out << key << ' ' << c.cells_per_cta << ' ' << c.lu_in_shared << ' ' << c.ctas_per_sm << ' ' << c.ring_slots
          << ' ' << c.variant << '\n';
    }

    // enqueue UpdateStateParameters + fused Solve (no host synchronisation)
    void EnqueueStep(micmb_solver& s, micmb_state& st, double dt)
    {
      LaunchRateConstants(s, st);
      SolveFused(s, st, dt, nullptr, nullptr, nullptr, nullptr);
    }

    void CheckFusedError(micmb_state& st)
    {
      int32_t err_flag = 0;
      MICMB_CUDA(cudaStreamSynchronize(st.stream));
      MICMB_CUDA(cudaMemcpy(&err_flag, st.counters.as<char>() + 16, sizeof(int32_t), cudaMemcpyDeviceToHost));
      if (err_flag)
        throw Error(MICMB_ERR_TIMEOUT, "fused kernel: a pipeline wait timed out");
    }

    bool SameConfig(const micmb_fused_config& a, const micmb_fused_config& b)
    {
      return a.cells_per_cta == b.cells_per_cta && a.lu_in_shared == b.lu_in_shared &&
             a.ctas_per_sm == b.ctas_per_sm && a.ring_slots == b.ring_slots && a.variant == b.variant;
    }
  }  // namespace
}  // namespace micmb

using namespace micmb;

extern "C"
{
  // Times each candidate configuration on (a prefix of) the state's own cells
  // and keeps the fastest.  The state's variables are restored afterwards.
  int micmb_autotune(micmb_solver* solver, micmb_state* state, double dt, const char* cache_path,
                     micmb_fused_config* chosen)
  {
    return GuardX([&] {
      NeedX(solver && state && state->solver == solver, "state does not belong to this solver");
      NeedX(dt > 0 && std::isfinite(dt), "time step must be positive and finite");
      MICMB_CUDA(cudaSetDevice(solver->device));
      const std::string key = TuneKey(*solver);
      micmb_fused_config best{};
      if (ReadCache(cache_path, key, best))
      {
        solver->fused = best;
        if (chosen)
          *chosen = best;
        return;
      }
      micmb_state& st = *state;
      const micmb_fused_config candidates[] = {
        { 0, 1, 0, 2, 0 }, { 0, 1, 0, 4, 0 },  // streamed, LU in shared memory
        { 0, 0, 0, 2, 0 }, { 0, 0, 0, 4, 0 },  // streamed, LU in global slots, as many cells as fit
        { 6, 0, 0, 4, 0 }, { 4, 0, 0, 4, 0 },  // streamed, fewer cells per CTA
        { 0, 1, 0, 0, 1 }, { 0, 0, 0, 0, 1 },  // direct
        { 0, 0, 0, 0, 2 }, { 0, 0, 12, 0, 2 },  // one cell per thread: 32-, 40-, 64- and 96-register builds
        { 0, 0, 8, 0, 2 }, { 0, 0, 5, 0, 2 },
      };
      // tune each candidate on enough cells to fill every SM a few times over:
      // a few warps per SM for the warp-per-cell variants, up to 1024 threads
      // per SM for the thread-per-cell variant; compare cells per second
      auto trial_cells = [&](const micmb_fused_config& c) {
        const int64_t per_sm = c.variant == 2 ? 2 * 1024 : 12 * 8;
        return std::min<int64_t>(st.n_cells, (int64_t)solver->sm_count * per_sm);
      };
      DeviceMemory saved(st.variables.bytes);
      MICMB_CUDA(cudaMemcpyAsync(saved.p, st.variables.p, st.variables.bytes, cudaMemcpyDeviceToDevice, st.stream));
      cudaEvent_t e0, e1;
      MICMB_CUDA(cudaEventCreate(&e0));
      MICMB_CUDA(cudaEventCreate(&e1));
      const micmb_fused_config before = solver->fused;
      const bool verbose = std::getenv("MICMB_AUTOTUNE_VERBOSE") != nullptr;
      // cells per second of one configuration over the first `cells` cells (best of `reps`)
      auto rate_of = [&](const micmb_fused_config& c, int64_t cells, int reps) {
        solver->fused = c;
        st.solve_limit = cells;
        float ms_min = -1.0f;
        for (int rep = 0; rep < reps; ++rep)
        {
          MICMB_CUDA(cudaMemcpyAsync(st.variables.p, saved.p, st.variables.bytes, cudaMemcpyDeviceToDevice,
                                     st.stream));
          MICMB_CUDA(cudaEventRecord(e0, st.stream));
          SolveFused(*solver, st, dt, nullptr, nullptr, nullptr, nullptr);
          MICMB_CUDA(cudaEventRecord(e1, st.stream));
          CheckFusedError(st);
          float ms = 0.0f;
          MICMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          ms_min = (ms_min < 0.0f || ms < ms_min) ? ms : ms_min;
        }
        const double rate = 1e3 * (double)cells / std::max(ms_min, 1e-3f);
        if (verbose)
          std::fprintf(stderr, "micmb_autotune: variant %d cells_per_cta %d lu_in_shared %d ring_slots %d "
                               "ctas_per_sm %d: %lld cells in %.3f ms -> %.0f cells/s\n",
                       c.variant, c.cells_per_cta, c.lu_in_shared, c.ring_slots, c.ctas_per_sm, (long long)cells,
                       ms_min, rate);
        return rate;
      };
      try
      {
        // stage 1: every candidate on a short trial, best configuration of each variant
        micmb_fused_config best_of[3];
        double rate_of_best[3] = { -1.0, -1.0, -1.0 };
        // a mechanism beyond 16-bit byte offsets has no streamed schedule (variant
        // 0 would run the direct kernel), beyond 16-bit positions no warp tables
        const bool has_stream = solver->dev.has_warp && solver->stream_blocks.p;
        for (const auto& c : candidates)
        {
          if ((c.variant == 0 && !has_stream) || (c.variant == 1 && !solver->dev.has_warp))
            continue;
          const double r = rate_of(c, trial_cells(c), 2);
          if (r > rate_of_best[c.variant])
          {
            rate_of_best[c.variant] = r;
            best_of[c.variant] = c;
          }
        }
        // stage 2: the variants' winners on the state itself (up to 2^20 cells).  Cells
        // take very different step counts, so how long the last cells keep the GPU
        // busy depends on how many cells each resident warp or thread gets; a short
        // trial cannot show that for the thread-per-cell variant.
        const double lead = std::max(rate_of_best[0], std::max(rate_of_best[1], rate_of_best[2]));
        const int64_t full = std::min<int64_t>(st.n_cells, (int64_t)1 << 20);
        double best_rate = -1.0;
        for (int v = 0; v < 3; ++v)
        {
          if (rate_of_best[v] < 0.0 || (v == 1 && rate_of_best[v] < 0.5 * lead))
            continue;
          const double r = rate_of(best_of[v], full, 1);
          if (r > best_rate)
          {
            best_rate = r;
            best = best_of[v];
          }
        }
      }
      catch (...)
      {
        st.solve_limit = 0;
        solver->fused = before;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
      }
      st.solve_limit = 0;
      MICMB_CUDA(cudaMemcpyAsync(st.variables.p, saved.p, st.variables.bytes, cudaMemcpyDeviceToDevice, st.stream));
      MICMB_CUDA(cudaStreamSynchronize(st.stream));
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      solver->fused = best;
      AppendCache(cache_path, key, best);
      if (chosen)
        *chosen = best;
    });
  }

  // n_repeats x (UpdateStateParameters + fused Solve): the first repeat runs
  // eagerly (allocating the working set), is then captured once into a CUDA
  // graph for this state, dt and configuration, and the graph is replayed.
  int micmb_solve_graph(micmb_solver* solver, micmb_state* state, double dt, int32_t n_repeats)
  {
    return GuardX([&] {
      NeedX(solver && state && state->solver == solver, "state does not belong to this solver");
      NeedX(dt > 0 && std::isfinite(dt), "time step must be positive and finite");
      NeedX(n_repeats >= 0, "n_repeats must be >= 0");
      MICMB_CUDA(cudaSetDevice(solver->device));
      micmb_state& st = *state;
      int32_t done = 0;
      const bool reuse = st.graph_exec && st.graph_dt == dt && SameConfig(st.graph_config, solver->fused);
      if (!reuse && n_repeats > 0)
      {
        if (st.graph_exec)
        {
          MICMB_CUDA(cudaGraphExecDestroy(st.graph_exec));
          st.graph_exec = nullptr;
        }
        EnqueueStep(*solver, st, dt);
        CheckFusedError(st);
        ++done;
        cudaGraph_t graph = nullptr;
        MICMB_CUDA(cudaStreamBeginCapture(st.stream, cudaStreamCaptureModeRelaxed));
        try
        {
          EnqueueStep(*solver, st, dt);
        }
        catch (...)
        {
          cudaStreamEndCapture(st.stream, &graph);
          if (graph)
            cudaGraphDestroy(graph);
          throw;
        }
        MICMB_CUDA(cudaStreamEndCapture(st.stream, &graph));
        const cudaError_t ie = cudaGraphInstantiate(&st.graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        MICMB_CUDA(ie);
        st.graph_dt = dt;
        st.graph_config = solver->fused;
      }
      for (; done < n_repeats; ++done)
        MICMB_CUDA(cudaGraphLaunch(st.graph_exec, st.stream));
      CheckFusedError(st);
    });
  }
}
