// capi.cu -- the extern "C" boundary (include/micmb.h): handle management,
// device table upload, host<->device copies and dispatch to the kernels.
// No exception crosses the boundary; failures become a status code plus a
// thread-local message.
#include "runtime.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace micmb
{
  thread_local std::string g_last_error;

  void CudaCheck(cudaError_t e, const char* what)
  {
    if (e != cudaSuccess)
    {
      const int code = (e == cudaErrorMemoryAllocation) ? MICMB_ERR_OUT_OF_MEMORY
                       : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? MICMB_ERR_NO_DEVICE
                                                                                       : MICMB_ERR_CUDA;
      throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
  }

  DeviceMemory::DeviceMemory(size_t b)
      : bytes(b)
  {
    if (b)
      CudaCheck(cudaMalloc(&p, b), "cudaMalloc");
  }

  DeviceMemory::~DeviceMemory()
  {
    if (p)
      cudaFree(p);
  }

  DeviceMemory& DeviceMemory::operator=(DeviceMemory&& o) noexcept
  {
    if (this != &o)
    {
      if (p)
        cudaFree(p);
      p = o.p;
      bytes = o.bytes;
      o.p = nullptr;
      o.bytes = 0;
    }
    return *this;
  }

  DevParams ToDevParams(const micmb_rosenbrock_params& p)
  {
    if (p.stages < 1 || p.stages > 6)
      throw Error(MICMB_ERR_INVALID_ARGUMENT, "stages must be 1..6");
    DevParams d{};
    d.stages = p.stages;
    d.max_steps = p.max_number_of_steps;
    d.round_off = p.round_off;
    d.factor_min = p.factor_min;
    d.factor_max = p.factor_max;
    d.rejection_factor_decrease = p.rejection_factor_decrease;
    d.safety_factor = p.safety_factor;
    d.h_min_param = p.h_min;
    d.h_max_param = p.h_max;
    d.h_start_param = p.h_start;
    for (int i = 0; i < 6; ++i)
    {
      d.new_f[i] = p.new_function_evaluation[i];
      d.m[i] = p.m[i];
      d.e[i] = p.e[i];
    }
    for (int i = 0; i < 15; ++i)
    {
      d.a[i] = p.a[i];
      d.c[i] = p.c[i];
    }
    d.inv_order = 1 / p.estimator_of_local_order;
    d.gamma0 = p.gamma[0];
    d.cinit_max_iter = p.constraint_init_max_iterations;
    d.cinit_tol = p.constraint_init_tolerance;
    return d;
  }

  namespace
  {
    // packs host arrays into one device allocation (256-byte aligned pieces)
    struct Packer
    {
      std::vector<char> bytes;
      template<class T>
      size_t add(const std::vector<T>& v)
      {
        size_t off = (bytes.size() + 255) & ~size_t(255);
        bytes.resize(off + std::max<size_t>(v.size() * sizeof(T), sizeof(T)), 0);
        if (!v.empty())
          std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
        return off;
      }
    };

    struct SchedOffsets
    {
      size_t ls, tg, ax, ts, ta, tb, tab, item, item_j = 0;
      int32_t n_levels;
    };

    SchedOffsets AddSchedule(Packer& pk, const LevelSchedule& s)
    {
      SchedOffsets o;
      o.ls = pk.add(s.level_start);
      o.tg = pk.add(s.item_target);
      o.ax = pk.add(s.item_aux);
      o.ts = pk.add(s.term_start);
      o.ta = pk.add(s.term_a);
      o.tb = pk.add(s.term_b);
      std::vector<int32_t> tab(2 * s.term_a.size());
      for (size_t t = 0; t < s.term_a.size(); ++t)
      {
        tab[2 * t] = s.term_a[t];
        tab[2 * t + 1] = s.term_b[t];
      }
      o.tab = pk.add(tab);
      std::vector<int32_t> item(4 * s.item_target.size());
      for (size_t it = 0; it < s.item_target.size(); ++it)
      {
        item[4 * it] = s.item_target[it];
        item[4 * it + 1] = s.term_start[it];
        item[4 * it + 2] = s.term_start[it + 1];
        item[4 * it + 3] = s.item_aux[it];
      }
      o.item = pk.add(item);
      o.n_levels = s.n_levels();
      return o;
    }

    struct WarpOffsets
    {
      size_t lcs, ch, it, tm, cf;
      int32_t n_levels;
      bool has_coef;
    };

    WarpOffsets AddWarp(Packer& pk, const WarpTable& w)
    {
      WarpOffsets o;
      o.lcs = pk.add(w.level_chunk_start);
      o.ch = pk.add(w.chunk);
      o.it = pk.add(w.item);
      o.tm = pk.add(w.term);
      o.cf = pk.add(w.coef);
      o.n_levels = w.n_levels;
      o.has_coef = !w.coef.empty();
      return o;
    }

    DevWarpTable ResolveWarp(const char* base, const WarpOffsets& o)
    {
      DevWarpTable d;
      d.n_levels = o.n_levels;
      d.level_chunk_start = reinterpret_cast<const int32_t*>(base + o.lcs);
      d.chunk = reinterpret_cast<const int4*>(base + o.ch);
      d.item = reinterpret_cast<const uint32_t*>(base + o.it);
      d.term = reinterpret_cast<const uint32_t*>(base + o.tm);
      d.coef = o.has_coef ? reinterpret_cast<const double*>(base + o.cf) : nullptr;
      return d;
    }

    struct BlockedOffsets
    {
      size_t bl, tg, ax, op;
      int32_t n_blocks;
    };

    BlockedOffsets AddBlocked(Packer& pk, const BlockedSchedule& b)
    {
      BlockedOffsets o;
      o.bl = pk.add(b.block);
      o.tg = pk.add(b.target);
      o.ax = pk.add(b.aux);
      o.op = pk.add(b.op);
      o.n_blocks = b.n_blocks;
      return o;
    }

    DevBlocked ResolveBlocked(const char* base, const BlockedOffsets& o)
    {
      DevBlocked d;
      d.n_blocks = o.n_blocks;
      d.block = reinterpret_cast<const int4*>(base + o.bl);
      d.target = reinterpret_cast<const int4*>(base + o.tg);
      d.aux = reinterpret_cast<const int4*>(base + o.ax);
      d.op = reinterpret_cast<const uint4*>(base + o.op);
      return d;
    }

    DevSchedule Resolve(const char* base, const SchedOffsets& o)
    {
      DevSchedule d;
      d.n_levels = o.n_levels;
      d.level_start = reinterpret_cast<const int32_t*>(base + o.ls);
      d.target = reinterpret_cast<const int32_t*>(base + o.tg);
      d.aux = reinterpret_cast<const int32_t*>(base + o.ax);
      d.term_start = reinterpret_cast<const int32_t*>(base + o.ts);
      d.ta = reinterpret_cast<const int32_t*>(base + o.ta);
      d.tb = reinterpret_cast<const int32_t*>(base + o.tb);
      d.tab = reinterpret_cast<const int2*>(base + o.tab);
      d.item = reinterpret_cast<const int4*>(base + o.item);
      d.item_j = o.item_j ? reinterpret_cast<const int4*>(base + o.item_j) : nullptr;
      return d;
    }

    void UploadTables(micmb_solver& s)
    {
      const CompiledMechanism& m = *s.mech;
      Packer pk;
      std::vector<int32_t> kind(m.R), pcol(m.R), nmult(m.R);
      std::vector<double> rp((size_t)m.R * MICMB_RATE_PARAM_STRIDE), mult((size_t)m.R * MICMB_MAX_PARAMETERIZED * 4);
      for (int32_t r = 0; r < m.R; ++r)
      {
        kind[r] = m.rates[r].kind;
        pcol[r] = m.rates[r].param_col;
        nmult[r] = m.rates[r].n_mult;
        for (int i = 0; i < MICMB_RATE_PARAM_STRIDE; ++i)
          rp[(size_t)r * MICMB_RATE_PARAM_STRIDE + i] = m.rates[r].p[i];
        for (int i = 0; i < MICMB_MAX_PARAMETERIZED; ++i)
          for (int q = 0; q < 4; ++q)
            mult[((size_t)r * MICMB_MAX_PARAMETERIZED + i) * 4 + q] = m.rates[r].mult[i][q];
      }
      std::vector<int32_t> diag_row_of(m.nnz, -1);
      for (int32_t i = 0; i < m.S; ++i)
        diag_row_of[m.diag_pos[i]] = i;
      const size_t o_kind = pk.add(kind), o_rp = pk.add(rp), o_pcol = pk.add(pcol), o_nm = pk.add(nmult),
                   o_mult = pk.add(mult);
      const size_t o_rs = pk.add(m.react_start), o_ri = pk.add(m.react_ids);
      const size_t o_ps = pk.add(m.prod_start), o_pi = pk.add(m.prod_ids), o_py = pk.add(m.prod_yield);
      const size_t o_fs = pk.add(m.f_start), o_fr = pk.add(m.f_rxn), o_fc = pk.add(m.f_coef);
      const size_t o_ir = pk.add(m.info_rxn), o_ids = pk.add(m.info_dep_start), o_idi = pk.add(m.info_dep_ids);
      const size_t o_js = pk.add(m.j_start), o_ji = pk.add(m.j_info), o_jc = pk.add(m.j_coef);
      const size_t o_dp = pk.add(m.diag_pos), o_dro = pk.add(diag_row_of);
      const SchedOffsets lu = AddSchedule(pk, m.lu), fw = AddSchedule(pk, m.fwd), bw = AddSchedule(pk, m.bwd),
                         fwt = AddSchedule(pk, m.fwd_t), bwt = AddSchedule(pk, m.bwd_t);
      const SchedOffsets lus = AddSchedule(pk, m.lu_serial), fws = AddSchedule(pk, m.fwd_serial),
                         bws = AddSchedule(pk, m.bwd_serial), fwts = AddSchedule(pk, m.fwd_t_serial),
                         bwts = AddSchedule(pk, m.bwd_t_serial);
      // the serial LU's per-item Jacobian gather range and diagonal rows
      SchedOffsets lus_j = lus;
      {
        const auto& ls = m.lu_serial;
        std::vector<int32_t> ij(4 * ls.item_target.size());
        for (size_t it = 0; it < ls.item_target.size(); ++it)
        {
          const int32_t e = ls.item_target[it], aux = ls.item_aux[it];
          ij[4 * it] = diag_row_of[e];
          ij[4 * it + 1] = m.j_start[e];
          ij[4 * it + 2] = m.j_start[e + 1];
          ij[4 * it + 3] = aux >= 0 ? diag_row_of[aux] : -1;
        }
        lus_j.item_j = pk.add(ij);
      }
      std::vector<double> jterm(2 * m.j_info.size());
      for (size_t t = 0; t < m.j_info.size(); ++t)
      {
        jterm[2 * t] = m.j_coef[t];
        int64_t bits = (int64_t)(uint32_t)m.j_info[t];
        std::memcpy(&jterm[2 * t + 1], &bits, sizeof bits);
      }
      const size_t o_jt = pk.add(jterm);
      const size_t o_rd = pk.add(m.rate_desc), o_drd = pk.add(m.drate_desc);
      // algebraic constraints
      std::vector<int32_t> con4, con2;
      std::vector<double> conp;
      for (const auto& cd : m.constraints)
      {
        con4.insert(con4.end(), { cd.kind, cd.row, cd.t0, cd.t1 });
        con2.insert(con2.end(), { cd.n_react, cd.keq });
        conp.insert(conp.end(), cd.p, cd.p + 4);
      }
      const size_t o_con = pk.add(con4), o_con2 = pk.add(con2), o_conp = pk.add(conp);
      const size_t o_ctc = pk.add(m.c_term_col), o_ctf = pk.add(m.c_term_coef), o_mass = pk.add(m.mass);
      const size_t o_cjs = pk.add(m.cj_start), o_cjt = pk.add(m.cj_term);
      BlockedOffsets blu{}, bfw{}, bbw{};
      if (m.has_blocked)
      {
        blu = AddBlocked(pk, m.lu_blocked);
        bfw = AddBlocked(pk, m.fwd_blocked);
        bbw = AddBlocked(pk, m.bwd_blocked);
      }
      WarpOffsets wl{}, wf{}, wb{}, wft{}, wbt{}, wfo{}, wj{};
      if (m.has_warp_tables)
      {
        wl = AddWarp(pk, m.w_lu);
        wf = AddWarp(pk, m.w_fwd);
        wb = AddWarp(pk, m.w_bwd);
        wft = AddWarp(pk, m.w_fwd_t);
        wbt = AddWarp(pk, m.w_bwd_t);
        wfo = AddWarp(pk, m.w_forcing);
        wj = AddWarp(pk, m.w_jacobian);
      }
      if (m.has_warp_tables && !m.stream.block_bytes.empty())
      {
        s.stream_blocks = DeviceMemory(m.stream.bytes.size());
        MICMB_CUDA(cudaMemcpy(s.stream_blocks.p, m.stream.bytes.data(), m.stream.bytes.size(),
                              cudaMemcpyHostToDevice));
        s.stream_block_bytes = DeviceMemory(m.stream.block_bytes.size() * sizeof(int32_t));
        MICMB_CUDA(cudaMemcpy(s.stream_block_bytes.p, m.stream.block_bytes.data(),
                              m.stream.block_bytes.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        s.n_stream_coef = (int32_t)m.stream.coef_table.size();
        s.stream_coef = DeviceMemory(m.stream.coef_table.size() * sizeof(double));
        MICMB_CUDA(cudaMemcpy(s.stream_coef.p, m.stream.coef_table.data(),
                              m.stream.coef_table.size() * sizeof(double), cudaMemcpyHostToDevice));
      }
      s.tables = DeviceMemory(pk.bytes.size());
      MICMB_CUDA(cudaMemcpy(s.tables.p, pk.bytes.data(), pk.bytes.size(), cudaMemcpyHostToDevice));
      std::vector<double> ones(std::max<int32_t>(m.R, 1), 1.0);
      s.scale_dev = DeviceMemory(ones.size() * sizeof(double));
      MICMB_CUDA(cudaMemcpy(s.scale_dev.p, ones.data(), ones.size() * sizeof(double), cudaMemcpyHostToDevice));
      const char* b = s.tables.as<const char>();
      DevMech& d = s.dev;
      d.S = m.S;
      d.R = m.R;
      d.P = m.P;
      d.nnz = m.nnz;
      d.n_info = (int32_t)m.info_rxn.size();
      d.rate_kind = reinterpret_cast<const int32_t*>(b + o_kind);
      d.rate_p = reinterpret_cast<const double*>(b + o_rp);
      d.rate_param_col = reinterpret_cast<const int32_t*>(b + o_pcol);
      d.rate_n_mult = reinterpret_cast<const int32_t*>(b + o_nm);
      d.rate_mult = reinterpret_cast<const double*>(b + o_mult);
      d.rate_scale = s.scale_dev.as<const double>();
      d.react_start = reinterpret_cast<const int32_t*>(b + o_rs);
      d.react_ids = reinterpret_cast<const int32_t*>(b + o_ri);
      d.prod_start = reinterpret_cast<const int32_t*>(b + o_ps);
      d.prod_ids = reinterpret_cast<const int32_t*>(b + o_pi);
      d.prod_yield = reinterpret_cast<const double*>(b + o_py);
      d.f_start = reinterpret_cast<const int32_t*>(b + o_fs);
      d.f_rxn = reinterpret_cast<const int32_t*>(b + o_fr);
      d.f_coef = reinterpret_cast<const double*>(b + o_fc);
      d.info_rxn = reinterpret_cast<const int32_t*>(b + o_ir);
      d.info_dep_start = reinterpret_cast<const int32_t*>(b + o_ids);
      d.info_dep_ids = reinterpret_cast<const int32_t*>(b + o_idi);
      d.j_start = reinterpret_cast<const int32_t*>(b + o_js);
      d.j_info = reinterpret_cast<const int32_t*>(b + o_ji);
      d.j_coef = reinterpret_cast<const double*>(b + o_jc);
      d.jterm = reinterpret_cast<const JTerm*>(b + o_jt);
      d.diag_pos = reinterpret_cast<const int32_t*>(b + o_dp);
      d.diag_row_of = reinterpret_cast<const int32_t*>(b + o_dro);
      d.lu = Resolve(b, lu);
      d.fwd = Resolve(b, fw);
      d.bwd = Resolve(b, bw);
      d.fwd_t = Resolve(b, fwt);
      d.bwd_t = Resolve(b, bwt);
      d.lu_s = Resolve(b, lus_j);
      d.fwd_s = Resolve(b, fws);
      d.bwd_s = Resolve(b, bws);
      d.fwd_t_s = Resolve(b, fwts);
      d.bwd_t_s = Resolve(b, bwts);
      // the register-blocked LU and solves are opt-in: on the 210-species
      // mechanism they measured slower than the serial schedules (the operand
      // re-reads they remove hit L1, and their accesses spread over more DRAM pages)
      const char* blk = std::getenv("MICMB_BLOCKED_SCHEDULES");
      d.has_blocked = (m.has_blocked && blk && blk[0] == '1') ? 1 : 0;
      d.n_constraints = (int32_t)m.constraints.size();
      d.n_eq = m.n_eq;
      d.n_cterms = (int32_t)m.c_term_col.size();
      d.con = reinterpret_cast<const int4*>(b + o_con);
      d.con_eq = reinterpret_cast<const int2*>(b + o_con2);
      d.con_p = reinterpret_cast<const double*>(b + o_conp);
      d.ct_col = reinterpret_cast<const int32_t*>(b + o_ctc);
      d.ct_coef = reinterpret_cast<const double*>(b + o_ctf);
      d.mass = reinterpret_cast<const double*>(b + o_mass);
      d.cj_start = reinterpret_cast<const int32_t*>(b + o_cjs);
      d.cj_term = reinterpret_cast<const int32_t*>(b + o_cjt);
      if (m.has_blocked)
      {
        d.lu_b = ResolveBlocked(b, blu);
        d.fwd_b = ResolveBlocked(b, bfw);
        d.bwd_b = ResolveBlocked(b, bbw);
      }
      s.diag_row_of = d.diag_row_of;
      d.has_warp = m.has_warp_tables ? 1 : 0;
      d.scratch_zero = m.scratch_zero;
      if (m.has_warp_tables)
      {
        d.w_lu = ResolveWarp(b, wl);
        d.w_fwd = ResolveWarp(b, wf);
        d.w_bwd = ResolveWarp(b, wb);
        d.w_fwd_t = ResolveWarp(b, wft);
        d.w_bwd_t = ResolveWarp(b, wbt);
        d.w_forcing = ResolveWarp(b, wfo);
        d.w_jacobian = ResolveWarp(b, wj);
      }
      d.rate_desc = m.rate_desc.empty() ? nullptr : reinterpret_cast<const int4*>(b + o_rd);
      d.drate_desc = m.drate_desc.empty() ? nullptr : reinterpret_cast<const int4*>(b + o_drd);
    }

    template<class F>
    int Guard(F&& f)
    {
      return GuardCall<MICMB_ERR_INVALID_ARGUMENT>(std::forward<F>(f));
    }

    void Need(bool ok, const char* what)
    {
      if (!ok)
        throw Error(MICMB_ERR_INVALID_ARGUMENT, what);
    }

    // buffer descriptor: device pointer and number of doubles
    std::pair<double*, size_t> BufferOf(micmb_state& st, int32_t which)
    {
      const auto& m = *st.solver->mech;
      switch (which)
      {
        case MICMB_BUF_VARIABLES: return { st.variables.as<double>(), st.variables.bytes / sizeof(double) };
        case MICMB_BUF_CUSTOM_PARAMS: return { st.custom_params.as<double>(), (size_t)st.n_pad * m.P };
        case MICMB_BUF_RATE_CONSTANTS: return { st.rate_constants.as<double>(), (size_t)st.n_pad * m.R };
        case MICMB_BUF_CONDITIONS: return { st.conditions.as<double>(), (size_t)st.n_pad * 3 };
        case MICMB_BUF_ABSOLUTE_TOLERANCE: return { st.atol.as<double>(), (size_t)m.S };
        case MICMB_BUF_JACOBIAN: EnsurePlainBuffers(st); return { st.jacobian.as<double>(), (size_t)st.n_pad * m.nnz };
        case MICMB_BUF_FORCING: EnsurePlainBuffers(st); return { st.forcing0.as<double>(), (size_t)st.n_pad * m.S };
        case MICMB_BUF_SCRATCH_Y: EnsurePlainBuffers(st); return { st.ynew.as<double>(), (size_t)st.n_pad * m.S };
      }
      throw Error(MICMB_ERR_INVALID_ARGUMENT, "unknown buffer id");
    }

    void SetDevice(const micmb_solver& s)
    {
      MICMB_CUDA(cudaSetDevice(s.device));
    }
  }  // namespace
}  // namespace micmb

using namespace micmb;

extern "C"
{
  const char* micmb_last_error(void)
  {
    return g_last_error.c_str();
  }

  int micmb_mechanism_create(const micmb_mechanism_desc* desc, micmb_mechanism** out)
  {
    return Guard([&] {
      Need(desc && out, "null argument");
      auto* h = new micmb_mechanism{ Compile(*desc) };
      *out = h;
    });
  }

  void micmb_mechanism_destroy(micmb_mechanism* mech)
  {
    delete mech;
  }

  int micmb_mechanism_get_info(const micmb_mechanism* mech, micmb_mechanism_info* out)
  {
    return Guard([&] {
      Need(mech && out, "null argument");
      const auto& m = mech->m;
      out->n_species = m.S;
      out->n_reactions = m.R;
      out->n_custom_params = m.P;
      out->jacobian_nnz = m.nnz;
      out->jacobian_nnz_unfilled = (int32_t)m.pattern_unfilled.size();
      out->lu_updates = m.lu_updates;
      out->lu_lower = m.lu_lower;
      out->n_jacobian_terms = (int32_t)m.j_info.size();
      out->n_forcing_terms = (int32_t)m.f_rxn.size();
      out->n_jacobian_infos = (int32_t)m.info_rxn.size();
      out->lu_levels = m.lu.n_levels();
      out->forward_levels = m.fwd.n_levels();
      out->backward_levels = m.bwd.n_levels();
      out->blocked_schedules = m.has_blocked ? 1 : 0;
      out->lu_blocked_ops = (int32_t)(m.lu_blocked.op.size() / 4);
    });
  }

  int micmb_mechanism_species_columns(const micmb_mechanism* mech, int32_t* out)
  {
    return Guard([&] {
      Need(mech && out, "null argument");
      std::copy(mech->m.species_column.begin(), mech->m.species_column.end(), out);
    });
  }

  int micmb_mechanism_reaction_columns(const micmb_mechanism* mech, int32_t* out)
  {
    return Guard([&] {
      Need(mech && out, "null argument");
      std::copy(mech->m.reaction_column.begin(), mech->m.reaction_column.end(), out);
    });
  }

  int micmb_mechanism_custom_param_columns(const micmb_mechanism* mech, int32_t* out)
  {
    return Guard([&] {
      Need(mech && out, "null argument");
      std::copy(mech->m.param_column.begin(), mech->m.param_column.end(), out);
    });
  }

  int micmb_mechanism_jacobian_pattern(const micmb_mechanism* mech, int32_t* rows, int32_t* cols)
  {
    return Guard([&] {
      Need(mech && rows && cols, "null argument");
      std::copy(mech->m.nz_row.begin(), mech->m.nz_row.end(), rows);
      std::copy(mech->m.nz_col.begin(), mech->m.nz_col.end(), cols);
    });
  }

  int micmb_mechanism_jacobian_pattern_unfilled(const micmb_mechanism* mech, int32_t* rows, int32_t* cols)
  {
    return Guard([&] {
      Need(mech && rows && cols, "null argument");
      for (size_t i = 0; i < mech->m.pattern_unfilled.size(); ++i)
      {
        rows[i] = mech->m.pattern_unfilled[i].first;
        cols[i] = mech->m.pattern_unfilled[i].second;
      }
    });
  }

  int micmb_mechanism_stream_stats(const micmb_mechanism* mech, int64_t* out)
  {
    return Guard([&] {
      Need(mech && out, "null argument");
      const auto& m = mech->m;
      if (!m.has_warp_tables)
        throw Error(MICMB_ERR_UNSUPPORTED, "no streamed schedule for this mechanism");
      const StreamPhase* ph[7] = { &m.stream.forcing, &m.stream.jacobian, &m.stream.lu, &m.stream.fwd,
                                   &m.stream.bwd,     &m.stream.fwd_t,    &m.stream.bwd_t };
      const LevelSchedule* sch[7] = { nullptr, nullptr, &m.lu, &m.fwd, &m.bwd, &m.fwd_t, &m.bwd_t };
      for (int p = 0; p < 7; ++p)
      {
        int64_t segs = 0, steps = 0;
        for (int32_t b = ph[p]->first_block; b < ph[p]->first_block + ph[p]->n_blocks; ++b)
        {
          const uint8_t* blk = m.stream.bytes.data() + (size_t)b * kStreamBlockBytes;
          int32_t nseg = 0;
          std::memcpy(&nseg, blk, 4);
          const uint8_t* q = blk + 16;
          for (int32_t g = 0; g < nseg; ++g)
          {
            int32_t d[4];
            std::memcpy(d, q, 16);
            steps += d[0];
            q += d[2];
          }
          segs += nseg;
        }
        out[p * 4 + 0] = ph[p]->n_blocks;
        out[p * 4 + 1] = segs;
        out[p * 4 + 2] = steps;
        out[p * 4 + 3] = sch[p] ? (int64_t)sch[p]->term_a.size()
                                : (int64_t)(p == 0 ? m.f_rxn.size() : m.j_info.size());
      }
    });
  }

  uint64_t micmb_mechanism_hash(const micmb_mechanism* mech)
  {
    return mech ? mech->m.hash : 0;
  }

  int micmb_rosenbrock_params_default(int32_t kind, micmb_rosenbrock_params* out)
  {
    return Guard([&] {
      Need(out != nullptr, "null argument");
      micmb_rosenbrock_params p{};
      p.max_number_of_steps = 1000;
      p.constraint_init_max_iterations = 10;  // rosenbrock_solver_parameters.hpp:43-44
      p.constraint_init_tolerance = 1e-10;
      p.round_off = 2.220446049250313080847e-16;  // std::numeric_limits<double>::epsilon()
      p.factor_min = 0.2;
      p.factor_max = 6;
      p.rejection_factor_decrease = 0.1;
      p.safety_factor = 0.9;
      // Published tableaus (Hairer & Wanner; Sandu et al. 1997), as tabulated in
      // micm's rosenbrock_solver_parameters.hpp:152-434.
      switch (kind)
      {
        case 2:
        {
          const double g = 1.0 + 1.0 / 1.41421356237309504880;  // 1 + 1/sqrt(2)
          p.stages = 2;
          p.a[0] = 1.0 / g;
          p.c[0] = -2.0 / g;
          for (int i = 0; i < 6; ++i)
            p.new_function_evaluation[i] = 1;
          p.m[0] = (3.0) / (2.0 * g);
          p.m[1] = (1.0) / (2.0 * g);
          p.e[0] = 1.0 / (2.0 * g);
          p.e[1] = 1.0 / (2.0 * g);
          p.estimator_of_local_order = 2.0;
          p.alpha[1] = 1.0;
          p.gamma[0] = g;
          p.gamma[1] = -g;
          break;
        }
        case 3:
          p.stages = 3;
          p.a[0] = 1;
          p.a[1] = 1;
          p.c[0] = -0.10156171083877702091975600115545e+01;
          p.c[1] = 0.40759956452537699824805835358067e+01;
          p.c[2] = 0.92076794298330791242156818474003e+01;
          p.new_function_evaluation[0] = 1;
          p.new_function_evaluation[1] = 1;
          p.m[0] = 0.1e+01;
          p.m[1] = 0.61697947043828245592553615689730e+01;
          p.m[2] = -0.42772256543218573326238373806514;
          p.e[0] = 0.5;
          p.e[1] = -0.29079558716805469821718236208017e+01;
          p.e[2] = 0.22354069897811569627360909276199;
          p.estimator_of_local_order = 3;
          p.alpha[1] = 0.43586652150845899941601945119356;
          p.alpha[2] = 0.43586652150845899941601945119356;
          p.gamma[0] = 0.43586652150845899941601945119356;
          p.gamma[1] = 0.24291996454816804366592249683314;
          p.gamma[2] = 0.21851380027664058511513169485832e+01;
          break;
        case 4:
          p.stages = 4;
          p.a[0] = 0.2000000000000000E+01;
          p.a[1] = 0.1867943637803922E+01;
          p.a[2] = 0.2344449711399156;
          p.a[3] = p.a[1];
          p.a[4] = p.a[2];
          p.c[0] = -0.7137615036412310E+01;
          p.c[1] = 0.2580708087951457E+01;
          p.c[2] = 0.6515950076447975;
          p.c[3] = -0.2137148994382534E+01;
          p.c[4] = -0.3214669691237626;
          p.c[5] = -0.6949742501781779;
          p.new_function_evaluation[0] = 1;
          p.new_function_evaluation[1] = 1;
          p.new_function_evaluation[2] = 1;
          p.m[0] = 0.2255570073418735E+01;
          p.m[1] = 0.2870493262186792;
          p.m[2] = 0.4353179431840180;
          p.m[3] = 0.1093502252409163E+01;
          p.e[0] = -0.2815431932141155;
          p.e[1] = -0.7276199124938920E-01;
          p.e[2] = -0.1082196201495311;
          p.e[3] = -0.1093502252409163E+01;
          p.estimator_of_local_order = 4.0;
          p.alpha[1] = 0.1145640000000000E+01;
          p.alpha[2] = 0.6552168638155900;
          p.alpha[3] = p.alpha[2];
          p.gamma[0] = 0.5728200000000000;
          p.gamma[1] = -0.1769193891319233E+01;
          p.gamma[2] = 0.7592633437920482;
          p.gamma[3] = -0.1049021087100450;
          break;
        case 40:
          p.stages = 4;
          p.a[1] = 2.0;
          p.a[3] = 2.0;
          p.a[5] = 1.0;
          p.c[0] = 4.0;
          p.c[1] = 1.0;
          p.c[2] = -1.0;
          p.c[3] = 1.0;
          p.c[4] = -1.0;
          p.c[5] = -(8.0 / 3.0);
          p.new_function_evaluation[0] = 1;
          p.new_function_evaluation[2] = 1;
          p.new_function_evaluation[3] = 1;
          p.m[0] = 2.0;
          p.m[2] = 1.0;
          p.m[3] = 1.0;
          p.e[3] = 1.0;
          p.estimator_of_local_order = 3.0;
          p.alpha[2] = 1.0;
          p.alpha[3] = 1.0;
          p.gamma[0] = 0.5;
          p.gamma[1] = 1.5;
          break;
        case 60:
          p.stages = 6;
          p.alpha[1] = 0.386;
          p.alpha[2] = 0.210;
          p.alpha[3] = 0.630;
          p.alpha[4] = 1.000;
          p.alpha[5] = 1.000;
          p.gamma[0] = 0.2500000000000000;
          p.gamma[1] = -0.1043000000000000;
          p.gamma[2] = 0.1035000000000000;
          p.gamma[3] = -0.3620000000000023E-01;
          p.a[0] = 0.1544000000000000E+01;
          p.a[1] = 0.9466785280815826;
          p.a[2] = 0.2557011698983284;
          p.a[3] = 0.3314825187068521E+01;
          p.a[4] = 0.2896124015972201E+01;
          p.a[5] = 0.9986419139977817;
          p.a[6] = 0.1221224509226641E+01;
          p.a[7] = 0.6019134481288629E+01;
          p.a[8] = 0.1253708332932087E+02;
          p.a[9] = -0.6878860361058950;
          p.a[10] = p.a[6];
          p.a[11] = p.a[7];
          p.a[12] = p.a[8];
          p.a[13] = p.a[9];
          p.a[14] = 1.0;
          p.c[0] = -0.5668800000000000E+01;
          p.c[1] = -0.2430093356833875E+01;
          p.c[2] = -0.2063599157091915;
          p.c[3] = -0.1073529058151375;
          p.c[4] = -0.9594562251023355E+01;
          p.c[5] = -0.2047028614809616E+02;
          p.c[6] = 0.7496443313967647E+01;
          p.c[7] = -0.1024680431464352E+02;
          p.c[8] = -0.3399990352819905E+02;
          p.c[9] = 0.1170890893206160E+02;
          p.c[10] = 0.8083246795921522E+01;
          p.c[11] = -0.7981132988064893E+01;
          p.c[12] = -0.3152159432874371E+02;
          p.c[13] = 0.1631930543123136E+02;
          p.c[14] = -0.6058818238834054E+01;
          p.m[0] = p.a[6];
          p.m[1] = p.a[7];
          p.m[2] = p.a[8];
          p.m[3] = p.a[9];
          p.m[4] = 1.0;
          p.m[5] = 1.0;
          p.e[5] = 1.0;
          for (int i = 0; i < 6; ++i)
            p.new_function_evaluation[i] = 1;
          p.estimator_of_local_order = 4.0;
          break;
        default: throw Error(MICMB_ERR_INVALID_ARGUMENT, "unknown tableau kind (use 2, 3, 4, 40 or 60)");
      }
      *out = p;
    });
  }

  int micmb_solver_create(const micmb_mechanism* mech, const micmb_rosenbrock_params* params, micmb_solver** out)
  {
    return Guard([&] {
      Need(mech && params && out, "null argument");
      int count = 0;
      cudaError_t e = cudaGetDeviceCount(&count);
      if (e != cudaSuccess || count == 0)
        throw Error(MICMB_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
      auto s = std::make_unique<micmb_solver>();
      MICMB_CUDA(cudaGetDevice(&s->device));
      cudaDeviceProp prop{};
      MICMB_CUDA(cudaGetDeviceProperties(&prop, s->device));
      if (prop.major < 10)
        throw Error(MICMB_ERR_UNSUPPORTED, "this library is built for sm_100a (B200) only");
      s->sm_count = prop.multiProcessorCount;
      s->smem_optin = prop.sharedMemPerBlockOptin;
      s->mech = std::make_shared<CompiledMechanism>(mech->m);
      s->host_params = *params;
      s->params = ToDevParams(*params);
      UploadTables(*s);
      *out = s.release();
    });
  }

  void micmb_solver_destroy(micmb_solver* solver)
  {
    delete solver;
  }

  int micmb_solver_set_params(micmb_solver* solver, const micmb_rosenbrock_params* params)
  {
    return Guard([&] {
      Need(solver && params, "null argument");
      solver->params = ToDevParams(*params);
      solver->host_params = *params;
    });
  }

  int micmb_solver_set_rate_scale(micmb_solver* solver, const double* scale)
  {
    return Guard([&] {
      Need(solver && scale, "null argument");
      SetDevice(*solver);
      const auto& m = *solver->mech;
      std::vector<double> by_col(std::max<int32_t>(m.R, 1), 1.0);
      for (int32_t r = 0; r < m.R; ++r)
        by_col[m.reaction_column[r]] = scale[r];
      MICMB_CUDA(cudaMemcpy(solver->scale_dev.p, by_col.data(), by_col.size() * sizeof(double),
                            cudaMemcpyHostToDevice));
    });
  }

  int micmb_solver_set_fused_config(micmb_solver* solver, const micmb_fused_config* config)
  {
    return Guard([&] {
      Need(solver && config, "null argument");
      Need(config->cells_per_cta >= 0 && config->cells_per_cta <= 12, "cells_per_cta must be 0..12");
      Need(config->ring_slots >= 0 && config->ring_slots <= 8, "ring_slots must be 0..8");
      Need(config->variant >= 0 && config->variant <= 2,
           "variant must be 0 (streamed), 1 (direct) or 2 (one cell per thread)");
      solver->fused = *config;
    });
  }

  int micmb_solver_get_fused_config(micmb_solver* solver, micmb_fused_config* config)
  {
    return Guard([&] {
      Need(solver && config, "null argument");
      *config = solver->fused;
    });
  }

  int micmb_state_create(micmb_solver* solver, int64_t n_cells, int32_t vector_length, micmb_state** out)
  {
    return Guard([&] {
      Need(solver && out, "null argument");
      Need(n_cells >= 0, "negative cell count");
      Need(vector_length >= 1 && vector_length <= 4096, "vector length must be 1..4096");
      SetDevice(*solver);
      const auto& m = *solver->mech;
      auto st = std::make_unique<micmb_state>();
      st->solver = solver;
      st->n_cells = n_cells;
      st->L = vector_length;
      st->n_groups = (n_cells + vector_length - 1) / vector_length;
      st->n_pad = st->n_groups * vector_length;
      MICMB_CUDA(cudaStreamCreateWithFlags(&st->own_stream, cudaStreamNonBlocking));
      st->stream = st->own_stream;
      st->variables = DeviceMemory(st->dense_bytes(m.S));
      st->custom_params = DeviceMemory(st->dense_bytes(std::max<int32_t>(m.P, 1)));
      st->rate_constants = DeviceMemory(st->dense_bytes(std::max<int32_t>(m.R, 1)));
      st->keq = DeviceMemory(st->dense_bytes(std::max<int32_t>(m.n_eq, 1)));
      st->conditions = DeviceMemory(st->dense_bytes(3));
      st->atol = DeviceMemory(sizeof(double) * m.S);
      st->counters = DeviceMemory(256);
      MICMB_CUDA(cudaMallocHost(&st->host_counters, 64));
      MICMB_CUDA(cudaMemsetAsync(st->variables.p, 0, st->variables.bytes, st->stream));
      MICMB_CUDA(cudaMemsetAsync(st->custom_params.p, 0, st->custom_params.bytes, st->stream));
      MICMB_CUDA(cudaMemsetAsync(st->rate_constants.p, 0, st->rate_constants.bytes, st->stream));
      MICMB_CUDA(cudaMemsetAsync(st->conditions.p, 0, st->conditions.bytes, st->stream));
      std::vector<double> atol(m.S, 1e-3);  // SolverBuilder default (solver_builder.inl:208)
      MICMB_CUDA(cudaMemcpyAsync(st->atol.p, atol.data(), sizeof(double) * m.S, cudaMemcpyHostToDevice, st->stream));
      MICMB_CUDA(cudaStreamSynchronize(st->stream));
      *out = st.release();
    });
  }

  void micmb_state_destroy(micmb_state* state)
  {
    if (!state)
      return;
    cudaSetDevice(state->solver->device);
    if (state->stream)
      cudaStreamSynchronize(state->stream);
    if (state->host_counters)
      cudaFreeHost(state->host_counters);
    if (state->graph_exec)
      cudaGraphExecDestroy(state->graph_exec);
    if (state->own_stream)
      cudaStreamDestroy(state->own_stream);
    delete state;
  }

  int micmb_state_set_stream(micmb_state* state, void* stream)
  {
    return Guard([&] {
      Need(state != nullptr, "null argument");
      state->stream = stream ? static_cast<cudaStream_t>(stream) : state->own_stream;
    });
  }

  int micmb_state_synchronize(micmb_state* state)
  {
    return Guard([&] {
      Need(state != nullptr, "null argument");
      MICMB_CUDA(cudaStreamSynchronize(state->stream));
    });
  }

  int micmb_state_upload(micmb_state* state, int32_t buffer, const double* host)
  {
    return Guard([&] {
      Need(state && host, "null argument");
      SetDevice(*state->solver);
      auto b = BufferOf(*state, buffer);
      MICMB_CUDA(cudaMemcpyAsync(b.first, host, b.second * sizeof(double), cudaMemcpyHostToDevice, state->stream));
      MICMB_CUDA(cudaStreamSynchronize(state->stream));
    });
  }

  int micmb_state_download(micmb_state* state, int32_t buffer, double* host)
  {
    return Guard([&] {
      Need(state && host, "null argument");
      SetDevice(*state->solver);
      auto b = BufferOf(*state, buffer);
      MICMB_CUDA(cudaMemcpyAsync(host, b.first, b.second * sizeof(double), cudaMemcpyDeviceToHost, state->stream));
      MICMB_CUDA(cudaStreamSynchronize(state->stream));
    });
  }

  int micmb_state_device_buffer(micmb_state* state, int32_t buffer, double** ptr, int64_t* count)
  {
    return Guard([&] {
      Need(state && ptr && count, "null argument");
      auto b = BufferOf(*state, buffer);
      *ptr = b.first;
      *count = (int64_t)b.second;
    });
  }

  int micmb_state_set_relative_tolerance(micmb_state* state, double rtol)
  {
    return Guard([&] {
      Need(state != nullptr, "null argument");
      Need(rtol > 0, "relative tolerance must be positive");
      state->rtol = rtol;
    });
  }

  int micmb_update_state_parameters(micmb_solver* solver, micmb_state* state)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      SetDevice(*solver);
      LaunchRateConstants(*solver, *state);
    });
  }

  int micmb_solve(micmb_solver* solver, micmb_state* state, double dt, int32_t method, int32_t step_control,
                  micmb_solver_stats* stats, int32_t* per_cell_status, int32_t* per_cell_accepted)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      Need(dt > 0 && std::isfinite(dt), "time step must be positive and finite");
      Need(method == MICMB_METHOD_PLAIN || method == MICMB_METHOD_FUSED, "unknown method");
      Need(step_control == MICMB_STEP_GLOBAL || step_control == MICMB_STEP_PER_CELL, "unknown step control");
      SetDevice(*solver);
      if (method == MICMB_METHOD_FUSED)
      {
        Need(step_control == MICMB_STEP_PER_CELL, "the fused method solves each cell independently (per-cell step control)");
        SolveFused(*solver, *state, dt, stats, per_cell_status, per_cell_accepted, nullptr);
      }
      else
        SolvePlain(*solver, *state, dt, step_control, stats, per_cell_status, per_cell_accepted);
    });
  }

  int micmb_state_set_global_exchange(micmb_state* state, micmb_allgather_fn fn, void* user, int32_t world,
                                      int64_t total_cells)
  {
    return Guard([&] {
      Need(state != nullptr, "no state");
      if (!fn)
      {
        state->gx_fn = nullptr;
        state->gx_user = nullptr;
        state->gx_world = 1;
        state->gx_total_cells = 0;
        return;
      }
      Need(world >= 1 && world <= 65536, "world must be 1..65536");
      Need(total_cells >= state->n_cells, "total_cells must count every rank's cells");
      SetDevice(*state->solver);
      if (!state->gx_buf.p || state->gx_buf.bytes < sizeof(double) * (size_t)(1 + world))
        state->gx_buf = DeviceMemory(sizeof(double) * (size_t)(1 + world));
      state->gx_fn = fn;
      state->gx_user = user;
      state->gx_world = world;
      state->gx_total_cells = total_cells;
    });
  }

  int micmb_backward_euler_params_default(micmb_backward_euler_params* out)
  {
    return Guard([&] {
      Need(out != nullptr, "no output");
      DefaultBackwardEulerParams(out);
    });
  }

  int micmb_solve_backward_euler(micmb_solver* solver, micmb_state* state, double dt,
                                 const micmb_backward_euler_params* params, int32_t step_control,
                                 micmb_solver_stats* stats, int32_t* per_cell_status, int32_t* per_cell_accepted)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      Need(dt > 0 && std::isfinite(dt), "time step must be positive and finite");
      Need(step_control == MICMB_STEP_GLOBAL || step_control == MICMB_STEP_PER_CELL, "unknown step control");
      SetDevice(*solver);
      micmb_backward_euler_params p;
      if (params)
        p = *params;
      else
        DefaultBackwardEulerParams(&p);
      SolveBackwardEuler(*solver, *state, dt, p, step_control, stats, per_cell_status, per_cell_accepted);
    });
  }

  int micmb_set_adjoint_memory_limit(micmb_solver* solver, int64_t bytes)
  {
    return Guard([&] {
      Need(solver != nullptr, "no solver");
      Need(bytes >= 0, "memory limit must be >= 0");
      solver->adjoint_memory_limit = bytes;
    });
  }

  int micmb_solve_adjoint(micmb_solver* solver, micmb_state* state, double dt, const double* dloss_dy_final,
                          double* dloss_dy0, double* dloss_dlogk, int32_t max_checkpoints,
                          micmb_solver_stats* stats)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      Need(dloss_dy_final != nullptr, "dloss_dy_final is required");
      Need(dt > 0 && std::isfinite(dt), "time step must be positive and finite");
      Need(max_checkpoints >= 1, "max_checkpoints must be at least 1");
      SetDevice(*solver);
      micmb_state& st = *state;
      const auto& m = *solver->mech;
      const int64_t n = st.n_cells;
      const size_t var_bytes = st.variables.bytes;
      if (!st.adj_y0.p || st.adj_y0.bytes < var_bytes)
      {
        st.adj_y0 = DeviceMemory(var_bytes);
        st.adj_ybar = DeviceMemory(var_bytes);
      }
      // The forward pass (streamed or thread variant) stores each accepted
      // step's stage vectors beside the checkpoint, so the backward sweep (one
      // cell per thread) rebuilds only the LU factor.
      const micmb_fused_config tuned = solver->fused;
      // the direct kernel keeps no stage vectors; it also runs when variant 0 is
      // configured but the mechanism has no streamed schedule: use the thread variant
      if (tuned.variant == 1 || (tuned.variant == 0 && !StreamVariantApplies(*solver)))
        solver->fused = micmb_fused_config{ 0, 0, 0, 0, 2 };
      struct Restore
      {
        micmb_solver* s;
        micmb_fused_config c;
        ~Restore() { s->fused = c; }
      } restore{ solver, tuned };
      if (!st.adj_kbar_cells.p || st.adj_kbar_cells.bytes < sizeof(double) * (size_t)std::max<int64_t>(n * m.R, 1))
      {
        st.adj_kbar_cells = DeviceMemory(sizeof(double) * (size_t)std::max<int64_t>(n * m.R, 1));
        st.adj_kbar = DeviceMemory(sizeof(double) * (size_t)std::max<int32_t>(m.R, 1));
      }
      if (!st.status.p)
        st.status = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(n, 1));
      if (!st.accepted.p)
        st.accepted = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(n, 1));
      // per-thread working sets do not shrink with the chunk: size them first
      const int64_t ws = std::max(FusedThreadWorkspaceDoubles(*solver, n), AdjointThreadWorkspaceDoubles(*solver, n));
      if (!st.thread_ws.p || st.thread_ws.bytes < (size_t)ws * sizeof(double))
      {
        st.thread_ws = DeviceMemory();
        st.thread_ws = DeviceMemory((size_t)ws * sizeof(double));
      }

      // Checkpoints take max_checkpoints * (S + 1) doubles per cell, the stored
      // stage vectors max_checkpoints * stages * S more.  Cells are solved and
      // swept in chunks (multiples of L) that fit the memory limit; when stored
      // stages would leave a chunk smaller than the cells the forward kernel
      // keeps resident, the stages are recomputed in the sweep instead.
      const int64_t per_cell_y = (int64_t)max_checkpoints * (m.S + 1) * (int64_t)sizeof(double);
      const int64_t per_cell_k = (int64_t)max_checkpoints * solver->params.stages * m.S * (int64_t)sizeof(double);
      int64_t budget = solver->adjoint_memory_limit;
      if (budget <= 0)
      {
        size_t free_b = 0, total_b = 0;
        MICMB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t held = st.adj_ckpt_y.bytes + st.adj_ckpt_h.bytes + st.adj_ckpt_k.bytes;
        budget = (int64_t)(0.8 * (double)(free_b + held));
      }
      const int64_t L = st.L;
      // equal chunks (multiples of L) of at most budget / per_cell cells; 0 if one group does not fit
      auto balanced_chunk = [&](int64_t per_cell) -> int64_t {
        const int64_t most = budget / per_cell / L * L;
        if (most < 1 || n < 1)
          return most < 1 ? 0 : std::max<int64_t>(n, 1);
        const int64_t parts = (n + most - 1) / most;
        return std::min<int64_t>(n, ((n + parts - 1) / parts + L - 1) / L * L);
      };
      const int64_t busy = std::min<int64_t>(n, FusedThreadResidentCells(*solver));
      int64_t chunk = balanced_chunk(per_cell_y + per_cell_k);
      bool store_k = true;
      if (chunk < busy && balanced_chunk(per_cell_y) > chunk)
      {
        chunk = balanced_chunk(per_cell_y);
        store_k = false;
      }
      if (n > 0 && chunk < 1)
        throw Error(MICMB_ERR_OUT_OF_MEMORY, "adjoint checkpoints of one cell group exceed the memory limit");
      chunk = std::max<int64_t>(chunk, 1);
      const int64_t ck = (int64_t)max_checkpoints * chunk * m.S;
      if (!store_k)
        st.adj_ckpt_k = DeviceMemory();
      if (!st.adj_ckpt_y.p || st.adj_ckpt_capacity < ck || (store_k && st.adj_ckpt_k.bytes < sizeof(double) *
                                                                                  (size_t)ck * solver->params.stages))
      {
        st.adj_ckpt_y = DeviceMemory();
        st.adj_ckpt_h = DeviceMemory();
        st.adj_ckpt_k = DeviceMemory();
        st.adj_ckpt_y = DeviceMemory(sizeof(double) * (size_t)std::max<int64_t>(ck, 1));
        st.adj_ckpt_h = DeviceMemory(sizeof(double) * (size_t)std::max<int64_t>((int64_t)max_checkpoints * chunk, 1));
        if (store_k)
          st.adj_ckpt_k = DeviceMemory(sizeof(double) * (size_t)std::max<int64_t>(ck * solver->params.stages, 1));
        st.adj_ckpt_capacity = ck;
      }
      MICMB_CUDA(cudaMemcpyAsync(st.adj_y0.p, st.variables.p, var_bytes, cudaMemcpyDeviceToDevice, st.stream));
      MICMB_CUDA(cudaMemcpyAsync(st.adj_ybar.p, dloss_dy_final, var_bytes, cudaMemcpyHostToDevice, st.stream));
      micmb_solver_stats total{};
      total.state = MICMB_SOLVER_CONVERGED;
      for (int64_t begin = 0; begin < n; begin += chunk)
      {
        const int64_t count = std::min<int64_t>(chunk, n - begin);
        FusedArgs adj{};
        adj.n_cells = count;
        adj.variables_in = st.variables.as<double>() + (size_t)begin * m.S;
        adj.variables_out = st.variables.as<double>() + (size_t)begin * m.S;
        adj.rate_constants = st.rate_constants.as<double>() + (size_t)begin * m.R;
        adj.cell_status = st.status.as<int32_t>() + begin;
        adj.cell_accepted = st.accepted.as<int32_t>() + begin;
        adj.ckpt_y = st.adj_ckpt_y.as<double>();
        adj.ckpt_h = st.adj_ckpt_h.as<double>();
        adj.ckpt_k = store_k ? st.adj_ckpt_k.as<double>() : nullptr;
        adj.max_ckpt = max_checkpoints;
        micmb_solver_stats cs{};
        SolveFused(*solver, st, dt, stats ? &cs : nullptr, nullptr, nullptr, &adj);
        LaunchAdjoint(*solver, st, max_checkpoints, begin, count);
        if (stats)
        {
          total.function_calls += cs.function_calls;
          total.jacobian_updates += cs.jacobian_updates;
          total.number_of_steps += cs.number_of_steps;
          total.accepted += cs.accepted;
          total.rejected += cs.rejected;
          total.decompositions += cs.decompositions;
          total.solves += cs.solves;
          total.cells_not_converged += cs.cells_not_converged;
          if (total.state == MICMB_SOLVER_CONVERGED)
            total.state = cs.state;
        }
      }
      ReduceAdjointParameters(*solver, st);
      if (stats)
      {
        total.final_time = dt;
        *stats = total;
      }
      if (dloss_dy0)
        MICMB_CUDA(cudaMemcpyAsync(dloss_dy0, st.adj_ybar.p, var_bytes, cudaMemcpyDeviceToHost, st.stream));
      std::vector<double> kcol(std::max<int32_t>(m.R, 1));
      if (dloss_dlogk && m.R > 0)
        MICMB_CUDA(cudaMemcpyAsync(kcol.data(), st.adj_kbar.p, sizeof(double) * m.R, cudaMemcpyDeviceToHost,
                                   st.stream));
      MICMB_CUDA(cudaStreamSynchronize(st.stream));
      if (dloss_dlogk)
        for (int32_t r = 0; r < m.R; ++r)
          dloss_dlogk[r] = kcol[m.reaction_column[r]];
    });
  }

  int micmb_add_forcing_terms(micmb_solver* solver, micmb_state* state)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      SetDevice(*solver);
      LaunchAddForcing(*solver, *state);
      MICMB_CUDA(cudaStreamSynchronize(state->stream));
    });
  }

  int micmb_subtract_jacobian_terms(micmb_solver* solver, micmb_state* state)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      SetDevice(*solver);
      LaunchSubtractJacobian(*solver, *state);
      MICMB_CUDA(cudaStreamSynchronize(state->stream));
    });
  }

  int micmb_alpha_minus_jacobian(micmb_solver* solver, micmb_state* state, double alpha)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      SetDevice(*solver);
      LaunchAlphaMinusJacobian(*solver, *state, alpha);
      MICMB_CUDA(cudaStreamSynchronize(state->stream));
    });
  }

  int micmb_lu_decompose(micmb_solver* solver, micmb_state* state)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      SetDevice(*solver);
      LaunchDecompose(*solver, *state);
      MICMB_CUDA(cudaStreamSynchronize(state->stream));
    });
  }

  int micmb_linear_solve(micmb_solver* solver, micmb_state* state)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      SetDevice(*solver);
      LaunchLinearSolve(*solver, *state);
      MICMB_CUDA(cudaStreamSynchronize(state->stream));
    });
  }

  int micmb_normalized_error(micmb_solver* solver, micmb_state* state, double* global_out, double* per_cell_out)
  {
    return Guard([&] {
      Need(solver && state && state->solver == solver, "state does not belong to this solver");
      SetDevice(*solver);
      NormalizedError(*solver, *state, global_out, per_cell_out);
    });
  }
}
