// fused_stream.cu -- the persistent fused solve with the mechanism's schedule
// streamed through shared memory.
//
// A CTA has W consumer warps and one producer warp.  Each consumer warp owns
// one grid cell (state, stage vectors, rate constants and LU factor in its
// slice of shared memory) and runs that cell's adaptive Rosenbrock solve; all
// W consumers walk the same per-attempt sequence of table blocks in lockstep.
// The producer warp streams those blocks (forcing and -J gathers, LU, the
// triangular solves of every stage) from global memory into a ring of
// shared-memory slots with bulk asynchronous copies (TMA) completed on
// mbarriers, so each table byte crosses L2 once per CTA attempt and every
// consumer lane reads its operand indices from shared memory.  Cells that
// finish hand their warp the next unsolved cell from a global atomic counter;
// the CTA runs while any of its warps has a cell.
#include "pipeline.cuh"
#include "runtime.hpp"
#include "stream_engine.cuh"

#include <algorithm>

namespace micmb
{
  namespace
  {
    using namespace stream;
    constexpr int kWarp = 32;
    constexpr int kMaxSlots = 8;
    constexpr int kMaxConsumers = 12;  // consumer warps per CTA (register file: 13 warps x 32 x 157)
    constexpr int kBlockBytes = kStreamBlockBytes;

    __device__ __forceinline__ size_t cell_base(int64_t c, int32_t L, int32_t ncol)
    {
      return (size_t)(c / L) * (size_t)L * (size_t)ncol + (size_t)(c % L);
    }

    __host__ __device__ inline int32_t RoundUp2(int32_t v)
    {
      return (v + 1) & ~1;
    }


    struct StreamArgs
    {
      const uint8_t* blocks;          // kBlockBytes apart
      const int32_t* block_bytes;     // bytes to copy per block
      const int32_t* attempt_blocks;  // block ids in the order one attempt consumes them
      int32_t n_attempt_blocks;
      int32_t n_slots;
      int32_t f_n, j_n, lu_n, fw_n, bw_n;  // blocks per phase
      int32_t* error_flag;
      const double* coef;                  // negated gather coefficients
      int32_t n_coef;
    };

    struct Layout
    {
      int32_t VS, KS, SC, LUS, per_warp;  // doubles (LUS = 0: the LU lives in a global slot)
      int32_t coef_offset;                // bytes from smem start: coefficient table (CTA-wide)
      int32_t ring_offset;
      int32_t bar_offset;
      int32_t flag_offset;
      int32_t total_bytes;
    };

    __host__ __device__ inline Layout MakeLayout(int32_t S, int32_t R, int32_t stages, int32_t n_info, int32_t nnz,
                                                 int32_t n_coef, int32_t warps, int32_t slots, bool lu_shared)
    {
      Layout l;
      const int32_t scratch_cols = R > n_info ? R : n_info;
      l.VS = RoundUp2(S + 2);  // slot S holds 0, slot S + 1 holds 1
      l.KS = RoundUp2(R > 0 ? R : 1);
      l.SC = RoundUp2(scratch_cols + 1);
      l.LUS = lu_shared ? RoundUp2(nnz + 1) : 0;
      l.per_warp = l.VS * (4 + stages) + l.KS + l.SC + l.LUS;  // 1/a_ii shares Fc's slot
      l.coef_offset = Pad16(l.per_warp * 8 * warps);
      l.ring_offset = Pad16(l.coef_offset + 8 * n_coef);
      l.bar_offset = l.ring_offset + slots * kBlockBytes;
      l.flag_offset = l.bar_offset + 2 * slots * 8;
      l.total_bytes = l.flag_offset + 2 * 16 * 4 + 16;
      return l;
    }

    // consumer side of the slot ring
    struct Ring
    {
      const uint8_t* slots;
      uint64_t* full;
      uint64_t* empty;
      int32_t ns;
      uint32_t count;
      volatile int32_t* abort;

      __device__ const uint8_t* acquire()
      {
        const int32_t s = (int32_t)(count % (uint32_t)ns);
        const uint32_t parity = (count / (uint32_t)ns) & 1u;
        bool ok = *abort == 0 && mbar_wait(full + s, parity);
        ok = __all_sync(0xffffffffu, ok);
        if (!ok)
        {
          *abort = 1;
          return nullptr;
        }
        return slots + (size_t)s * kBlockBytes;
      }

      __device__ void release(int lane)
      {
        __syncwarp();
        if (lane == 0)
          mbar_arrive(empty + (count % (uint32_t)ns));
        ++count;
      }
    };

    template<int KIND>
    __device__ __forceinline__ void consume(Ring& ring, int32_t n_blocks, bool active, const double* X,
                                            const double* Yv, double* out, double* inv, double alpha, int lane)
    {
      double acc[4] = { 0.0, 0.0, 0.0, 0.0 };
      for (int32_t b = 0; b < n_blocks; ++b)
      {
        const uint8_t* blk = ring.acquire();
        if (blk && active)
          blk_run<KIND>(blk, X, Yv, out, inv, alpha, acc, lane);
        ring.release(lane);
      }
    }

    __device__ __forceinline__ void count_attempt(CellCtl& cc, const DevParams& P)
    {
      cc.decompositions += 1;
      cc.solves += P.stages;
      for (int32_t s = 1; s < P.stages; ++s)
        cc.function_calls += P.new_f[s] ? 1 : 0;
    }

    struct WarpCell
    {
      int32_t cell;
      bool have;
      bool need_f0;
      int32_t n_ckpt;
      CellCtl c;
    };

    template<int W>
    __global__ void __launch_bounds__((W + 1) * 32, 1)
        k_fused_stream(DevMech M, DevParams P, StepBounds B, FusedArgs A, StreamArgs SA, Layout LY)
    {
      extern __shared__ __align__(128) uint8_t sm[];
      const int warp = threadIdx.x >> 5;
      const int lane = threadIdx.x & 31;
      const int32_t S = M.S, R = M.R, L = A.L;
      const int32_t ns = SA.n_slots;
      uint8_t* ring_slots = sm + LY.ring_offset;
      uint64_t* full = reinterpret_cast<uint64_t*>(sm + LY.bar_offset);
      uint64_t* empty = full + ns;
      // work flags, double-buffered by attempt parity ([0,W) and [16,16+W)), then abort
      int32_t* flags = reinterpret_cast<int32_t*>(sm + LY.flag_offset);
      volatile int32_t* abort_flag = flags + 32;
      uint32_t round = 0;
      const uint32_t all_threads = (W + 1) * 32;

      if (threadIdx.x == 0)
      {
        for (int32_t s = 0; s < ns; ++s)
        {
          mbar_init(full + s, 1);
          mbar_init(empty + s, W);
        }
        *abort_flag = 0;
        fence_barrier_init();
      }
      double* coefs = reinterpret_cast<double*>(sm + LY.coef_offset);
      for (int32_t i = threadIdx.x; i < SA.n_coef; i += blockDim.x)
        coefs[i] = SA.coef[i];
      __syncthreads();

      if (warp == W)
      {
        // ---------------- producer warp ----------------
        uint32_t issued = 0;
        for (;;)
        {
          named_barrier(1, all_threads);  // consumers have decided whether to run another attempt
          bool any = false;
          for (int w = 0; w < W; ++w)
            any |= flags[(round & 1u) * 16 + w] != 0;
          ++round;
          if (!any || *abort_flag)
            break;
          if (lane == 0)
          {
            for (int32_t j = 0; j < SA.n_attempt_blocks; ++j)
            {
              const int32_t s = (int32_t)(issued % (uint32_t)ns);
              if (issued >= (uint32_t)ns)
              {
                const uint32_t parity = ((issued / (uint32_t)ns) - 1u) & 1u;
                if (*abort_flag || !mbar_wait(empty + s, parity))
                {
                  *abort_flag = 1;
                  break;
                }
              }
              const int32_t b = SA.attempt_blocks[j];
              const uint32_t bytes = (uint32_t)SA.block_bytes[b];
              mbar_arrive_expect_tx(full + s, bytes);
              bulk_copy_g2s(ring_slots + (size_t)s * kBlockBytes, SA.blocks + (size_t)b * kBlockBytes, bytes,
                            full + s);
              ++issued;
            }
          }
          __syncwarp();
        }
        // let every issued copy land before the CTA exits
        if (lane == 0)
        {
          const uint32_t first = issued > (uint32_t)ns ? issued - (uint32_t)ns : 0u;
          for (uint32_t i = first; i < issued; ++i)
            mbar_wait(full + (i % (uint32_t)ns), (i / (uint32_t)ns) & 1u);
        }
        if (*abort_flag && lane == 0)
          atomicExch(SA.error_flag, 1);
        return;
      }

      // ---------------- consumer warps ----------------
      const int32_t VS = LY.VS;
      double* base = reinterpret_cast<double*>(sm) + (size_t)warp * LY.per_warp;
      double* Y = base;
      double* Yn = Y + VS;
      double* F0 = Yn + VS;
      double* Fc = F0 + VS;
      double* inv = Fc;  // 1/a_ii lives only inside the LU, Fc only inside the stages
      double* K = Fc + VS;
      double* kk = K + (size_t)P.stages * VS;
      double* scr = kk + LY.KS;
      double* LU = LY.LUS ? scr + LY.SC
                          : A.lu_global + ((size_t)blockIdx.x * W + warp) * (size_t)A.lu_slot_stride;
      if (lane == 0)
      {
        for (int32_t st = 0; st < P.stages; ++st)
          K[(size_t)st * VS + S] = 0.0;
        Y[S] = 0.0;
        Yn[S] = 0.0;
        Y[S + 1] = 1.0;
        Yn[S + 1] = 1.0;
        scr[M.scratch_zero] = 0.0;
        LU[M.nnz] = 0.0;
      }
      __syncwarp();

      Ring ring{ ring_slots, full, empty, ns, 0u, abort_flag };
      long long acc_stats[8] = { 0 };
      WarpCell wc;
      wc.have = false;
      wc.need_f0 = false;
      wc.cell = 0;
      wc.n_ckpt = 0;
      ctl_init(wc.c, B);

      // write the finished cell, then claim cells until one needs work or the queue is empty
      auto finish_and_claim = [&](bool finished_one) {
        for (;;)
        {
          if (finished_one)
          {
            const size_t by = cell_base(wc.cell, L, S);
            for (int32_t i = lane; i < S; i += kWarp)
            {
              const double v = Y[i];
              A.variables_out[by + (size_t)i * L] = (v < 0.0) ? 0.0 : v;
            }
            if (lane == 0)
            {
              if (A.cell_status)
                A.cell_status[wc.cell] = wc.c.state;
              if (A.cell_accepted)
                A.cell_accepted[wc.cell] = A.ckpt_y ? wc.n_ckpt : wc.c.accepted;
              acc_stats[0] += wc.c.function_calls;
              acc_stats[1] += wc.c.jacobian_updates;
              acc_stats[2] += wc.c.number_of_steps;
              acc_stats[3] += wc.c.accepted;
              acc_stats[4] += wc.c.rejected;
              acc_stats[5] += wc.c.decompositions;
              acc_stats[6] += wc.c.solves;
              acc_stats[7] += (wc.c.state == MICMB_SOLVER_CONVERGED) ? 0 : 1;
            }
            __syncwarp();
            finished_one = false;
          }
          int32_t cell = 0;
          if (lane == 0)
            cell = atomicAdd(A.next_cell, 1);
          cell = __shfl_sync(0xffffffffu, cell, 0);
          if (cell >= A.n_cells)
          {
            wc.have = false;
            return;
          }
          wc.cell = cell;
          wc.have = true;
          wc.n_ckpt = 0;
          const size_t by = cell_base(cell, L, S);
          const size_t bk = cell_base(cell, L, R);
          for (int32_t i = lane; i < S; i += kWarp)
            Y[i] = A.variables_in[by + (size_t)i * L];
          for (int32_t r = lane; r < R; r += kWarp)
            kk[r] = A.rate_constants[bk + (size_t)r * L];
          __syncwarp();
          ctl_init(wc.c, B);
          if (ctl_begin_step(wc.c, P, B))
          {
            wc.c.function_calls += 1;
            wc.c.jacobian_updates += 1;
            wc.need_f0 = true;
            return;
          }
          finished_one = true;  // a cell with nothing to do (dt already covered)
        }
      };

      finish_and_claim(false);
      if (lane == 0)
        flags[(round & 1u) * 16 + warp] = wc.have ? 1 : 0;
      named_barrier(1, all_threads);

      for (;;)
      {
        bool any = false;
        for (int w = 0; w < W; ++w)
          any |= flags[(round & 1u) * 16 + w] != 0;
        ++round;
        if (!any || *abort_flag)
          break;
        const bool act = wc.have;
        // initial forcing F0 = f(Y) for cells starting a step
        const bool do_f0 = act && wc.need_f0;
        if (do_f0)
        {
          if (M.rate_desc)
            reaction_rates_narrow<kWarp>(M, Unit{ kk }, Unit{ Y }, Unit{ scr }, lane);
          else
            reaction_rates<kWarp>(M, Unit{ kk }, Unit{ Y }, Unit{ scr }, lane);
          __syncwarp();
        }
        consume<kGather>(ring, SA.f_n, do_f0, scr, coefs, F0, nullptr, 0.0, lane);
        __syncwarp();
        // alpha I - J at Y, then LU
        const double H = wc.c.H;
        const double alpha = 1.0 / (H * P.gamma0);
        if (act)
        {
          if (M.drate_desc)
            jacobian_rates_narrow<kWarp>(M, Unit{ kk }, Unit{ Y }, Unit{ scr }, lane);
          else
            jacobian_rates<kWarp>(M, Unit{ kk }, Unit{ Y }, Unit{ scr }, lane);
          __syncwarp();
        }
        consume<kGather>(ring, SA.j_n, act, scr, coefs, LU, nullptr, alpha, lane);
        __syncwarp();
        consume<kLU>(ring, SA.lu_n, act, LU, LU, LU, inv, 0.0, lane);
        __syncwarp();
        const double* Fsrc = F0;
        for (int32_t st = 0; st < P.stages; ++st)
        {
          const int32_t sc = st * (st - 1) / 2;
          if (st > 0 && P.new_f[st])
          {
            if (act)
            {
              for (int32_t i = lane; i < S; i += kWarp)
              {
                double v = Y[i];
                for (int32_t j = 0; j < st; ++j)
                  v += P.a[sc + j] * K[(size_t)j * VS + i];
                Yn[i] = v;
              }
              __syncwarp();
              if (M.rate_desc)
                reaction_rates_narrow<kWarp>(M, Unit{ kk }, Unit{ Yn }, Unit{ scr }, lane);
              else
                reaction_rates<kWarp>(M, Unit{ kk }, Unit{ Yn }, Unit{ scr }, lane);
              __syncwarp();
            }
            consume<kGather>(ring, SA.f_n, act, scr, coefs, Fc, nullptr, 0.0, lane);
            __syncwarp();
            Fsrc = Fc;
          }
          double* Ks = K + (size_t)st * VS;
          if (act)
          {
            double coh[6];
            for (int32_t j = 0; j < st; ++j)
              coh[j] = P.c[sc + j] / H;
            for (int32_t i = lane; i < S; i += kWarp)
            {
              double v = Fsrc[i];
              for (int32_t j = 0; j < st; ++j)
                v += coh[j] * K[(size_t)j * VS + i];
              Ks[i] = v;
            }
          }
          __syncwarp();
          consume<kSolve>(ring, SA.fw_n, act, LU, Ks, Ks, nullptr, 0.0, lane);
          __syncwarp();
          consume<kSolveDiv>(ring, SA.bw_n, act, LU, Ks, Ks, nullptr, 0.0, lane);
          __syncwarp();
        }
        if (act && !*abort_flag)
        {
          // error norm in species order (micm's order): stripe by stripe, the
          // lanes' terms added in lane order
          double sum = 0.0;
          for (int32_t base = 0; base < S; base += kWarp)
          {
            const int32_t i = base + lane;
            double q = 0.0;
            if (i < S)
            {
              double v = Y[i];
              double e = 0.0;
              for (int32_t st = 0; st < P.stages; ++st)
              {
                const double kv = K[(size_t)st * VS + i];
                v += P.m[st] * kv;
                e += P.e[st] * kv;
              }
              Yn[i] = v;
              q = scaled_sq(Y[i], v, e, A.atol[i], A.rtol);
            }
            sum = warp_seq_add(sum, q, (S - base < kWarp) ? S - base : kWarp);
          }
          const double error = error_from_sum(sum, (double)S);
          count_attempt(wc.c, P);
          const double h_used = wc.c.H;
          const int res = ctl_after_error(wc.c, P, B, error);
          __syncwarp();
          if (res == 1)
          {
            if (A.ckpt_y)
            {
              double* dst = A.ckpt_y + ((size_t)wc.cell * A.max_ckpt + wc.n_ckpt) * S;
              for (int32_t i = lane; i < S; i += kWarp)
                dst[i] = Y[i];
              if (A.ckpt_k)
              {
                double* kd = A.ckpt_k + ((size_t)wc.cell * A.max_ckpt + wc.n_ckpt) * (size_t)P.stages * S;
                for (int32_t st = 0; st < P.stages; ++st)
                  for (int32_t i = lane; i < S; i += kWarp)
                    kd[(size_t)st * S + i] = K[(size_t)st * VS + i];
              }
              if (lane == 0)
                A.ckpt_h[(size_t)wc.cell * A.max_ckpt + wc.n_ckpt] = h_used;
              ++wc.n_ckpt;
            }
            for (int32_t i = lane; i < S; i += kWarp)
              Y[i] = Yn[i];
            __syncwarp();
            bool more = ctl_begin_step(wc.c, P, B);
            if (more && A.ckpt_y && wc.n_ckpt >= A.max_ckpt)
            {
              wc.c.state = MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS;
              more = false;
            }
            if (more)
            {
              wc.c.function_calls += 1;
              wc.c.jacobian_updates += 1;
              wc.need_f0 = true;
            }
            else
              finish_and_claim(true);
          }
          else if (res == 0)
            wc.need_f0 = false;
          else
            finish_and_claim(true);
        }
        if (lane == 0)
          flags[(round & 1u) * 16 + warp] = wc.have ? 1 : 0;
        named_barrier(1, all_threads);
      }
      if (lane == 0)
        for (int q = 0; q < 8; ++q)
          if (acc_stats[q])
            atomicAdd(A.stats + q, (unsigned long long)acc_stats[q]);
    }

    template<int W>
    void Launch(micmb_solver& s, micmb_state& st, const FusedArgs& A, const StreamArgs& SA, const Layout& LY,
                int64_t grid)
    {
      auto kernel = k_fused_stream<W>;
      MICMB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, LY.total_bytes));
      const StepBounds B = step_bounds(s.params, st.dt_for_launch);
      kernel<<<(unsigned)grid, (W + 1) * 32, LY.total_bytes, st.stream>>>(s.dev, s.params, B, A, SA, LY);
      MICMB_CUDA(cudaGetLastError());
    }
  }  // namespace

  int StreamWarpsPerCta(const micmb_solver& s, int slots, int cap, bool lu_shared)
  {
    const auto& m = *s.mech;
    for (int w = std::min(cap > 0 ? cap : kMaxConsumers, kMaxConsumers); w >= 1; --w)
    {
      const Layout l = MakeLayout(m.S, m.R, s.params.stages, (int32_t)m.info_rxn.size(), m.nnz, s.n_stream_coef, w,
                                  slots, lu_shared);
      if ((size_t)l.total_bytes <= s.smem_optin)
        return w;
    }
    return 0;
  }

  bool StreamVariantApplies(const micmb_solver& s)
  {
    if (!s.dev.has_warp || !s.stream_blocks.p)
      return false;
    const int slots = std::max(2, std::min(kMaxSlots, s.fused.ring_slots > 0 ? s.fused.ring_slots : 4));
    return StreamWarpsPerCta(s, slots, s.fused.cells_per_cta, s.fused.lu_in_shared != 0) >= 1;
  }

  bool SolveFusedStream(micmb_solver& s, micmb_state& st, double dt, const FusedArgs& A_in)
  {
    const auto& m = *s.mech;
    if (!StreamVariantApplies(s))
      return false;
    const int slots = std::max(2, std::min(kMaxSlots, s.fused.ring_slots > 0 ? s.fused.ring_slots : 4));
    const bool lu_shared = s.fused.lu_in_shared != 0;
    const int W = StreamWarpsPerCta(s, slots, s.fused.cells_per_cta, lu_shared);
    const Layout LY =
        MakeLayout(m.S, m.R, s.params.stages, (int32_t)m.info_rxn.size(), m.nnz, s.n_stream_coef, W, slots, lu_shared);
    // per-attempt block order: F0 forcing, -J, LU, then per stage [forcing], forward, backward
    std::vector<int32_t> order;
    auto add = [&](const StreamPhase& ph) {
      for (int32_t b = 0; b < ph.n_blocks; ++b)
        order.push_back(ph.first_block + b);
    };
    add(m.stream.forcing);
    add(m.stream.jacobian);
    add(m.stream.lu);
    for (int32_t stg = 0; stg < s.params.stages; ++stg)
    {
      if (stg > 0 && s.params.new_f[stg])
        add(m.stream.forcing);
      add(m.stream.fwd);
      add(m.stream.bwd);
    }
    if (order != st.attempt_order_host)
    {
      // uploaded once per tableau, so repeated launches (and graph captures) copy nothing
      MICMB_CUDA(cudaStreamSynchronize(st.stream));  // no earlier launch still reads the old order
      if (st.attempt_order.bytes < order.size() * sizeof(int32_t))
        st.attempt_order = DeviceMemory(order.size() * sizeof(int32_t));
      MICMB_CUDA(cudaMemcpy(st.attempt_order.p, order.data(), order.size() * sizeof(int32_t),
                            cudaMemcpyHostToDevice));
      st.attempt_order_host = order;
    }
    StreamArgs SA{};
    SA.blocks = s.stream_blocks.as<const uint8_t>();
    SA.block_bytes = s.stream_block_bytes.as<const int32_t>();
    SA.attempt_blocks = st.attempt_order.as<const int32_t>();
    SA.n_attempt_blocks = (int32_t)order.size();
    SA.n_slots = slots;
    SA.f_n = m.stream.forcing.n_blocks;
    SA.j_n = m.stream.jacobian.n_blocks;
    SA.lu_n = m.stream.lu.n_blocks;
    SA.fw_n = m.stream.fwd.n_blocks;
    SA.bw_n = m.stream.bwd.n_blocks;
    SA.error_flag = reinterpret_cast<int32_t*>(st.counters.as<char>() + 16);
    SA.coef = s.stream_coef.as<const double>();
    SA.n_coef = s.n_stream_coef;
    int64_t grid = (int64_t)s.sm_count * (s.fused.ctas_per_sm > 0 ? s.fused.ctas_per_sm : 1);
    grid = std::max<int64_t>(1, std::min<int64_t>(grid, (A_in.n_cells + W - 1) / W));
    FusedArgs A = A_in;
    if (!lu_shared)
    {
      const int64_t slots_needed = grid * W;
      const int64_t stride = ((int64_t)m.nnz + 2 + 31) & ~31ll;
      if (st.lu_slot_count < slots_needed * stride || !st.lu_slots.p)
      {
        st.lu_slots = DeviceMemory(sizeof(double) * (size_t)(slots_needed * stride));
        st.lu_slot_count = slots_needed * stride;
      }
      A.lu_global = st.lu_slots.as<double>();
      A.lu_slot_stride = stride;
    }
    st.dt_for_launch = dt;
    switch (W)
    {
      case 1: Launch<1>(s, st, A, SA, LY, grid); break;
      case 2: Launch<2>(s, st, A, SA, LY, grid); break;
      case 3: Launch<3>(s, st, A, SA, LY, grid); break;
      case 4: Launch<4>(s, st, A, SA, LY, grid); break;
      case 5: Launch<5>(s, st, A, SA, LY, grid); break;
      case 6: Launch<6>(s, st, A, SA, LY, grid); break;
      case 7: Launch<7>(s, st, A, SA, LY, grid); break;
      case 8: Launch<8>(s, st, A, SA, LY, grid); break;
      case 9: Launch<9>(s, st, A, SA, LY, grid); break;
      case 10: Launch<10>(s, st, A, SA, LY, grid); break;
      case 11: Launch<11>(s, st, A, SA, LY, grid); break;
      default: Launch<kMaxConsumers>(s, st, A, SA, LY, grid); break;
    }
    return true;
  }
}  // namespace micmb
