// mechanism.cpp -- symbolic compile (see mechanism.hpp).
#include "mechanism.hpp"

#include <algorithm>
#include <array>
#include <map>
#include <cstring>
#include <cmath>
#include <numeric>
#include <set>
#include <stdexcept>

namespace micmb
{
  namespace
  {
    constexpr double kAvogadro = 6.02214076e23;           // micm::constants::AVOGADRO_CONSTANT
    constexpr double kBoltzmann = 1.380649e-23;           // micm::constants::BOLTZMANN_CONSTANT
    constexpr double kGas = kBoltzmann * kAvogadro;       // micm::constants::GAS_CONSTANT
    constexpr double kPi = 3.14159265358979323846;

    void Require(bool ok, const std::string& what)
    {
      if (!ok)
        throw std::runtime_error(what);
    }

    // One output value (LU entry, solution component, forcing, -J entry) with
    // its ordered terms.  term_dep[t] lists the items whose final values term
    // t reads; final_dep lists the items the finalisation reads (the pivot
    // 1/a_kk of an L entry).
    struct RawItem
    {
      int32_t target;
      int32_t aux;
      std::vector<std::pair<int32_t, int32_t>> terms;
      std::vector<std::vector<int32_t>> term_dep;
      std::vector<int32_t> final_dep;
    };

    // "As soon as possible" level schedule that keeps every item's terms in
    // their original order.  Term t of an item can be applied once its
    // operands are final (and after the item's earlier terms), so an item is
    // cut into work units, one per level in which it gains terms; each unit
    // reloads the partial sum from memory and stores it back (an exact round
    // trip), and only the last unit finalises (pivot scaling, reciprocal,
    // division).  Long dot products then overlap the levels that produce
    // their operands instead of running after all of them.  Items must be
    // visited in a dependency-respecting order.
    LevelSchedule Schedule(const std::vector<RawItem>& items)
    {
      const int32_t n = (int32_t)items.size();
      std::vector<int32_t> final_level(n, 0);
      struct Unit
      {
        int32_t level, item, t0, t1;
        bool final;
      };
      std::vector<Unit> units;
      int32_t max_level = 0;
      for (int32_t i = 0; i < n; ++i)
      {
        const RawItem& it = items[i];
        const int32_t m = (int32_t)it.terms.size();
        int32_t unit_start = 0, unit_level = -1, prefix = 0;
        for (int32_t t = 0; t < m; ++t)
        {
          int32_t d = 0;
          for (int32_t dep : it.term_dep[t])
          {
            if (dep >= i)
              throw std::runtime_error("schedule: dependency visited after its user");
            d = std::max(d, final_level[dep] + 1);
          }
          prefix = std::max(prefix, d);
          if (t == 0)
            unit_level = prefix;
          else if (prefix > unit_level)
          {
            units.push_back({ unit_level, i, unit_start, t, false });
            unit_start = t;
            unit_level = prefix;
          }
        }
        int32_t fin = 0;
        for (int32_t dep : it.final_dep)
        {
          if (dep >= i)
            throw std::runtime_error("schedule: dependency visited after its user");
          fin = std::max(fin, final_level[dep] + 1);
        }
        if (m == 0)
        {
          units.push_back({ fin, i, 0, 0, true });
          final_level[i] = fin;
        }
        else if (fin <= unit_level)
        {
          units.push_back({ unit_level, i, unit_start, m, true });
          final_level[i] = unit_level;
        }
        else
        {
          units.push_back({ unit_level, i, unit_start, m, false });
          units.push_back({ fin, i, m, m, true });
          final_level[i] = fin;
        }
        max_level = std::max(max_level, final_level[i]);
      }
      // by level, then longer term lists first so lanes finish together
      std::stable_sort(units.begin(), units.end(), [](const Unit& a, const Unit& b) {
        if (a.level != b.level)
          return a.level < b.level;
        return (a.t1 - a.t0) > (b.t1 - b.t0);
      });
      LevelSchedule s;
      s.level_start.assign(n ? max_level + 2 : 1, 0);
      for (const Unit& u : units)
        s.level_start[u.level + 1]++;
      for (int32_t l = 0; l + 1 < (int32_t)s.level_start.size(); ++l)
        s.level_start[l + 1] += s.level_start[l];
      s.term_start.push_back(0);
      for (const Unit& u : units)
      {
        const RawItem& it = items[u.item];
        s.item_target.push_back(it.target);
        s.item_aux.push_back(u.final ? it.aux : -2);  // -2: partial sum, no finalisation
        for (int32_t t = u.t0; t < u.t1; ++t)
        {
          s.term_a.push_back(it.terms[t].first);
          s.term_b.push_back(it.terms[t].second);
        }
        s.term_start.push_back((int32_t)s.term_a.size());
      }
      return s;
    }

    // One thread visiting every item in order, each with all of its terms:
    // one level, no partial sums (the order the items were built in already
    // respects their dependencies).
    LevelSchedule SerialSchedule(const std::vector<RawItem>& items)
    {
      LevelSchedule s;
      s.level_start = { 0, (int32_t)items.size() };
      s.term_start.push_back(0);
      for (const RawItem& it : items)
      {
        s.item_target.push_back(it.target);
        s.item_aux.push_back(it.aux);
        for (const auto& t : it.terms)
        {
          s.term_a.push_back(t.first);
          s.term_b.push_back(t.second);
        }
        s.term_start.push_back((int32_t)s.term_a.size());
      }
      return s;
    }

    // Lane-interleave a level schedule (see WarpTable).  `meta(i)` packs item i,
    // `pack(t)` packs term t, `coef` (optional) is per term; padding terms
    // are `dummy` with coefficient 0.  `cls(i)` (0 or kSegRecip) keeps items
    // that finalise differently in separate chunks; chunk_flags records it.
    template<class Meta, class Pack, class Cls>
    WarpTable BuildWarp(const LevelSchedule& s, Meta meta, Pack pack, uint32_t dummy, const std::vector<double>* coef,
                        Cls cls)
    {
      WarpTable w;
      w.dummy = dummy;
      w.n_levels = s.n_levels();
      w.level_chunk_start.push_back(0);
      for (int32_t l = 0; l < w.n_levels; ++l)
      {
        // items of the level, class by class, each class longest first (the schedule's order)
        std::vector<int32_t> order;
        for (int32_t i = s.level_start[l]; i < s.level_start[l + 1]; ++i)
          order.push_back(i);
        std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return cls(a) < cls(b); });
        for (size_t first = 0; first < order.size();)
        {
          const int32_t c = cls(order[first]);
          size_t last = first;
          while (last < order.size() && last - first < 32 && cls(order[last]) == c)
            ++last;
          const int32_t n = (int32_t)(last - first);
          int32_t T = 0;
          for (size_t q = first; q < last; ++q)
            T = std::max(T, s.term_start[order[q] + 1] - s.term_start[order[q]]);
          w.chunk.push_back((int32_t)w.term.size());
          w.chunk.push_back(T);
          w.chunk.push_back((int32_t)w.item.size());
          w.chunk.push_back(n);
          w.chunk_flags.push_back(c);
          for (size_t q = first; q < last; ++q)
            w.item.push_back(meta(order[q]));
          const size_t base = w.term.size();
          w.term.resize(base + (size_t)T * 32, dummy);
          if (coef)
            w.coef.resize(base + (size_t)T * 32, 0.0);
          for (size_t q = first; q < last; ++q)
          {
            const int32_t i = order[q];
            for (int32_t t = s.term_start[i]; t < s.term_start[i + 1]; ++t)
            {
              const size_t at = base + (size_t)(t - s.term_start[i]) * 32 + (q - first);
              w.term[at] = pack(t);
              if (coef)
                w.coef[at] = (*coef)[t];
            }
          }
          first = last;
        }
        w.level_chunk_start.push_back((int32_t)(w.chunk.size() / 4));
      }
      return w;
    }

    // one-level schedule of independent gather items (forcing / -J)
    LevelSchedule GatherSchedule(const std::vector<int32_t>& start, const std::vector<int32_t>& idx,
                                 const std::vector<double>& cf, std::vector<double>& coef_out)
    {
      std::vector<RawItem> items;
      const int32_t n = (int32_t)start.size() - 1;
      for (int32_t i = 0; i < n; ++i)
      {
        RawItem it;
        it.target = i;
        it.aux = -1;
        for (int32_t t = start[i]; t < start[i + 1]; ++t)
        {
          it.terms.push_back({ idx[t], t });  // term_b carries the coefficient index
          it.term_dep.emplace_back();
        }
        items.push_back(std::move(it));
      }
      LevelSchedule s = Schedule(items);
      coef_out.resize(s.term_b.size());
      for (size_t t = 0; t < s.term_b.size(); ++t)
        coef_out[t] = cf[s.term_b[t]];
      return s;
    }

    inline int32_t Pad16(int32_t b)
    {
      return (b + 15) & ~15;
    }

    // index of -c in the stream's coefficient table (entry 0 stays +0 for padding)
    uint32_t InternCoef(StreamProgram& P, std::map<uint64_t, uint32_t>& seen, double c)
    {
      if (P.coef_table.empty())
        P.coef_table.push_back(0.0);
      const double v = -c;
      uint64_t bits;
      std::memcpy(&bits, &v, sizeof(bits));
      auto it = seen.find(bits);
      if (it != seen.end())
        return it->second;
      const uint32_t idx = (uint32_t)P.coef_table.size();
      if (idx > 0xFFFFu)
        throw std::runtime_error("too many distinct coefficients for the streamed schedule");
      P.coef_table.push_back(v);
      seen.emplace(bits, idx);
      return idx;
    }

    // operand pair of 16-bit element indices -> pair of 16-bit byte offsets
    inline uint32_t ToBytes(uint32_t v)
    {
      return (((v & 0xFFFFu) * 8u) & 0xFFFFu) | ((((v >> 16) * 8u) & 0xFFFFu) << 16);
    }

    // Re-cut one warp table into stream blocks (see StreamProgram).  Weighted
    // gathers (w.coef non-empty) get their coefficients interned in the table.
    void AppendStreamPhase(StreamProgram& P, std::map<uint64_t, uint32_t>& seen, const WarpTable& w,
                           StreamPhase& ph)
    {
      const bool has_coef = !w.coef.empty();
      if (P.coef_table.empty())
        P.coef_table.push_back(0.0);
      const int32_t B = kStreamBlockBytes;
      int32_t n_blocks = (int32_t)P.block_bytes.size();
      ph.first_block = n_blocks;
      int32_t used = 16;  // header
      int32_t n_segs = 0;
      auto block_ptr = [&]() { return P.bytes.data() + (size_t)n_blocks * B; };
      auto open_block = [&]() {
        P.bytes.resize((size_t)(n_blocks + 1) * B, 0);
        used = 16;
        n_segs = 0;
      };
      auto close_block = [&]() {
        std::memcpy(block_ptr(), &n_segs, sizeof(int32_t));
        P.block_bytes.push_back(used);
        ++n_blocks;
      };
      open_block();
      auto packed = [&](size_t at) -> uint32_t {
        if (!has_coef)
          return w.term[at];
        const double c = w.coef[at];
        uint64_t bits;
        std::memcpy(&bits, &c, sizeof(bits));
        const uint32_t cidx = bits == 0 ? 0u : InternCoef(P, seen, c);
        return (w.term[at] & 0xFFFFu) | (cidx << 16);
      };
      const uint32_t pad_term = has_coef ? (w.dummy & 0xFFFFu) : w.dummy;  // coefficient entry 0 is +0
      // term t of lane `lane` in chunk ch (padding past the chunk's own length)
      auto term_of = [&](int32_t ch, int32_t lane, int32_t t) -> uint32_t {
        const int32_t base = w.chunk[4 * ch + 0], T = w.chunk[4 * ch + 1], n = w.chunk[4 * ch + 3];
        return (t < T && lane < n) ? packed((size_t)base + (size_t)t * 32 + lane) : pad_term;
      };
      for (int32_t l = 0; l < w.n_levels; ++l)
      {
        const int32_t c_end = w.level_chunk_start[l + 1];
        for (int32_t ch = w.level_chunk_start[l]; ch < c_end;)
        {
          // Up to four chunks of similar length run side by side (U = 4: one
          // accumulator per chunk in every lane); a chunk much longer than the
          // next one runs alone, four terms per step (U = 1).
          const int32_t T0 = w.chunk[4 * ch + 1];
          const int32_t cflags = w.chunk_flags[ch];
          auto joins = [&](int32_t c) {
            return c < c_end && w.chunk_flags[c] == cflags && T0 <= 2 * w.chunk[4 * c + 1] + 2;
          };
          int32_t U = 1, width = 1;
          if (T0 <= kWideMaxSteps && joins(ch + 1))
          {
            U = 4;
            while (width < 4 && joins(ch + width))
              ++width;
          }
          const int32_t T = T0, n = w.chunk[4 * ch + 3];
          const bool last_in_level = (ch + width == c_end);
          const int32_t fixed = 16 + Pad16(4 * n * U);
          const int32_t per_group = 16 * n;
          const int32_t step_quantum = (U == 1) ? 4 : 1;  // terms per uint4 and lane
          int32_t t0 = 0;
          bool first_seg = true;
          for (;;)
          {
            const int32_t avail = B - used;
            int32_t tseg = 0;
            if (avail >= fixed)
              tseg = std::min(T - t0, step_quantum * ((avail - fixed) / per_group));
            const bool fits = avail >= fixed && (tseg > 0 || T == t0);
            if (!fits)
            {
              if (n_segs == 0)
                throw std::runtime_error("stream block too small for one table segment");
              close_block();
              open_block();
              continue;
            }
            const int32_t groups = (tseg + step_quantum - 1) / step_quantum;
            const int32_t seg_bytes = fixed + per_group * groups;
            uint8_t* seg = block_ptr() + used;
            int32_t flags = (first_seg ? kSegFirst : 0) | cflags;
            const bool last_seg = (t0 + tseg == T);
            if (last_seg)
              flags |= kSegLast;
            if (last_seg && last_in_level)
              flags |= kSegLevelEnd;
            const int32_t desc[4] = { tseg, n | (flags << 8) | (U << 16), seg_bytes, 0 };
            std::memcpy(seg, desc, 16);
            uint32_t* items = reinterpret_cast<uint32_t*>(seg + 16);
            for (int32_t u = 0; u < U; ++u)
              for (int32_t lane = 0; lane < n; ++lane)
              {
                const int32_t c = ch + u;
                const bool real = u < width && lane < w.chunk[4 * c + 3];
                uint32_t it = kNoItem;
                if (real)
                {
                  it = w.item[(size_t)w.chunk[4 * c + 2] + lane];
                  it = (it & 0xFFFF0000u) | (((it & 0xFFFFu) * 8u) & 0xFFFFu);
                }
                items[u * n + lane] = it;
              }
            uint32_t* terms = reinterpret_cast<uint32_t*>(seg + fixed);
            for (int32_t g = 0; g < groups; ++g)
              for (int32_t lane = 0; lane < n; ++lane)
                for (int32_t k = 0; k < 4; ++k)
                {
                  uint32_t v = pad_term;
                  if (U == 1)
                  {
                    const int32_t t = t0 + 4 * g + k;
                    if (t < T)
                      v = term_of(ch, lane, t);
                  }
                  else if (k < width)
                    v = term_of(ch + k, lane, t0 + g);
                  terms[(g * n + lane) * 4 + k] = ToBytes(v);
                }
            used += seg_bytes;
            ++n_segs;
            t0 += tseg;
            first_seg = false;
            if (last_seg)
              break;
          }
          ch += width;
        }
      }
      close_block();
      ph.n_blocks = n_blocks - ph.first_block;
    }

    uint64_t Fnv(uint64_t h, const void* data, size_t bytes)
    {
      const unsigned char* p = static_cast<const unsigned char*>(data);
      for (size_t i = 0; i < bytes; ++i)
      {
        h ^= p[i];
        h *= 1099511628211ull;
      }
      return h;
    }
    template<class T>
    uint64_t FnvVec(uint64_t h, const std::vector<T>& v)
    {
      return v.empty() ? h : Fnv(h, v.data(), v.size() * sizeof(T));
    }

    // ------------------------------------------------------------------
    // register-blocked serial schedules (mechanism.hpp BlockedSchedule)
    // ------------------------------------------------------------------
    using PosMap = std::map<std::pair<int32_t, int32_t>, int32_t>;

    // One block: slots' targets and, per slot, its terms as (shared index,
    // per-slot operand) in increasing shared-index order.
    void EmitBlock(BlockedSchedule& b, int32_t kind, int32_t diag_slot, int32_t pivot,
                   const std::vector<int32_t>& targets, const std::vector<int32_t>& aux,
                   const std::vector<std::vector<std::pair<int32_t, int32_t>>>& terms,
                   const std::vector<std::vector<int32_t>>& order_keys)
    {
      // union of the slots' terms, ordered by each slot's own term order (the
      // order keys increase along every slot's list, so one merged order
      // serves all slots)
      std::map<int32_t, std::pair<int32_t, std::array<int32_t, kBlockSlots>>> ops;  // key -> shared, slot operands
      for (size_t sl = 0; sl < targets.size(); ++sl)
        for (size_t t = 0; t < terms[sl].size(); ++t)
        {
          auto f = ops.find(order_keys[sl][t]);
          if (f == ops.end())
          {
            std::array<int32_t, kBlockSlots> none;
            none.fill(-1);
            f = ops.emplace(order_keys[sl][t], std::make_pair(terms[sl][t].first, none)).first;
          }
          if (f->second.first != terms[sl][t].first)
            throw std::runtime_error("blocked schedule: slots disagree on a shared operand");
          f->second.second[sl] = terms[sl][t].second;
        }
      const int32_t first_op = (int32_t)(b.op.size() / 4);
      for (const auto& kv : ops)
      {
        int32_t mask = 0;
        uint32_t p[kBlockSlots] = { 0, 0, 0, 0 };
        for (int32_t sl = 0; sl < kBlockSlots; ++sl)
          if (kv.second.second[sl] >= 0)
          {
            mask |= 1 << sl;
            p[sl] = (uint32_t)kv.second.second[sl];
          }
        b.op.push_back(kv.second.first);
        b.op.push_back(mask);
        b.op.push_back((int32_t)(p[0] | (p[1] << 16)));
        b.op.push_back((int32_t)(p[2] | (p[3] << 16)));
      }
      b.block.push_back(first_op);
      b.block.push_back((int32_t)ops.size());
      b.block.push_back((int32_t)targets.size() | (kind << 4) | ((diag_slot + 1) << 8));
      b.block.push_back(pivot);
      for (int32_t sl = 0; sl < kBlockSlots; ++sl)
      {
        b.target.push_back(sl < (int32_t)targets.size() ? targets[sl] : -1);
        b.aux.push_back(sl < (int32_t)aux.size() ? aux[sl] : -1);
      }
      ++b.n_blocks;
    }

    // The LU of step 8 (Crout entries, pivot by pivot: the U row, then the L
    // column) in blocks of up to kBlockSlots entries of one row or column.
    BlockedSchedule BlockLu(int32_t S, const std::vector<std::set<int32_t>>& row_cols,
                            const std::vector<std::set<int32_t>>& col_rows, const PosMap& position)
    {
      auto pos = [&](int32_t r, int32_t c) { return position.at({ r, c }); };
      BlockedSchedule b;
      for (int32_t mn = 0; mn < S; ++mn)
      {
        std::vector<int32_t> u_cols, l_rows;
        for (int32_t k : row_cols[mn])
          if (k >= mn)
            u_cols.push_back(k);
        for (int32_t j : col_rows[mn])
          if (j > mn)
            l_rows.push_back(j);
        for (int32_t kind : { kBlockU, kBlockL })
        {
          const std::vector<int32_t>& list = kind == kBlockU ? u_cols : l_rows;
          for (size_t c0 = 0; c0 < list.size(); c0 += kBlockSlots)
          {
            std::vector<int32_t> targets, none;
            std::vector<std::vector<std::pair<int32_t, int32_t>>> terms;
            std::vector<std::vector<int32_t>> keys;
            int32_t diag_slot = -1;
            for (size_t q = c0; q < std::min(list.size(), c0 + kBlockSlots); ++q)
            {
              const int32_t j = kind == kBlockU ? mn : list[q];
              const int32_t k = kind == kBlockU ? list[q] : mn;
              if (j == k)
                diag_slot = (int32_t)targets.size();
              targets.push_back(pos(j, k));
              terms.emplace_back();
              keys.emplace_back();
              const int32_t lim = std::min(j, k);
              for (int32_t i : row_cols[j])
              {
                if (i >= lim)
                  break;
                auto f = position.find({ i, k });
                if (f == position.end())
                  continue;
                // term a_ji * a_ik: U row shares a_{mn,i}, L column shares a_{i,mn}
                if (kind == kBlockU)
                  terms.back().push_back({ pos(j, i), f->second });
                else
                  terms.back().push_back({ f->second, pos(j, i) });
                keys.back().push_back(i);
              }
            }
            EmitBlock(b, kind, diag_slot, mn, targets, none, terms, keys);
          }
        }
      }
      return b;
    }

    // A triangular solve in blocks of up to kBlockSlots rows of one
    // dependency level (rows of a level do not read each other).  forward:
    // rows ascending, terms j < i; backward: rows descending, terms j > i,
    // then the division by the diagonal.
    BlockedSchedule BlockSolve(int32_t S, const std::vector<std::set<int32_t>>& row_cols, const PosMap& position,
                               bool forward)
    {
      auto pos = [&](int32_t r, int32_t c) { return position.at({ r, c }); };
      std::vector<int32_t> level(S, 0);
      int32_t max_level = 0;
      for (int32_t v = 0; v < S; ++v)
      {
        const int32_t i = forward ? v : S - 1 - v;
        int32_t l = 0;
        for (int32_t j : row_cols[i])
          if (forward ? j < i : j > i)
            l = std::max(l, level[j] + 1);
        level[i] = l;
        max_level = std::max(max_level, l);
      }
      BlockedSchedule b;
      for (int32_t l = 0; l <= max_level; ++l)
      {
        std::vector<int32_t> rows;
        for (int32_t v = 0; v < S; ++v)
        {
          const int32_t i = forward ? v : S - 1 - v;
          if (level[i] == l)
            rows.push_back(i);
        }
        for (size_t c0 = 0; c0 < rows.size(); c0 += kBlockSlots)
        {
          std::vector<int32_t> targets, aux;
          std::vector<std::vector<std::pair<int32_t, int32_t>>> terms;
          std::vector<std::vector<int32_t>> keys;
          for (size_t q = c0; q < std::min(rows.size(), c0 + kBlockSlots); ++q)
          {
            const int32_t i = rows[q];
            targets.push_back(i);
            aux.push_back(forward ? -1 : pos(i, i));
            terms.emplace_back();
            keys.emplace_back();
            for (int32_t j : row_cols[i])
              if (forward ? j < i : j > i)
              {
                terms.back().push_back({ j, pos(i, j) });
                keys.back().push_back(j);
              }
          }
          EmitBlock(b, kBlockSolve, -1, -1, targets, aux, terms, keys);
        }
      }
      return b;
    }

    // Host check that the blocked forms give the serial forms' bits on random
    // values (the same IEEE operations in the same order per entry).
    bool BlockedMatchesSerial(const CompiledMechanism& m)
    {
      const int32_t S = m.S, nnz = m.nnz;
      std::vector<double> A0(nnz), x0(S);
      uint64_t st = 0x9E3779B97F4A7C15ull;
      auto rnd = [&]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return ((double)(st >> 11) / 9007199254740992.0) * 2.0 - 1.0;
      };
      for (auto& v : A0)
        v = rnd();
      for (int32_t i = 0; i < S; ++i)
        A0[m.diag_pos[i]] = 4.0 + (double)S + rnd();
      for (auto& v : x0)
        v = rnd();
      std::vector<int32_t> diag_row(nnz, -1);
      for (int32_t i = 0; i < S; ++i)
        diag_row[m.diag_pos[i]] = i;
      // serial LU (lu_decompose with one lane)
      std::vector<double> A = A0, inv(S, 0.0);
      const LevelSchedule& ls = m.lu_serial;
      for (size_t it = 0; it < ls.item_target.size(); ++it)
      {
        const int32_t e = ls.item_target[it];
        double v = A[e];
        for (int32_t t = ls.term_start[it]; t < ls.term_start[it + 1]; ++t)
          v -= A[ls.term_a[t]] * A[ls.term_b[t]];
        const int32_t aux = ls.item_aux[it];
        if (aux >= 0)
          v *= inv[diag_row[aux]];
        A[e] = v;
        if (aux != -2 && diag_row[e] >= 0)
          inv[diag_row[e]] = 1.0 / v;
      }
      // blocked LU
      std::vector<double> B = A0, binv(S, 0.0);
      const BlockedSchedule& bl = m.lu_blocked;
      for (int32_t k = 0; k < bl.n_blocks; ++k)
      {
        const int32_t* blk = &bl.block[4 * k];
        const int32_t n = blk[2] & 0xF, kind = (blk[2] >> 4) & 0xF, diag = (blk[2] >> 8) - 1;
        double acc[kBlockSlots] = { 0, 0, 0, 0 };
        for (int32_t sl = 0; sl < n; ++sl)
          acc[sl] = B[bl.target[4 * k + sl]];
        for (int32_t o = blk[0]; o < blk[0] + blk[1]; ++o)
        {
          const int32_t* op = &bl.op[4 * o];
          const double sh = B[op[0]];
          const uint32_t p01 = (uint32_t)op[2], p23 = (uint32_t)op[3];
          const uint32_t p[4] = { p01 & 0xFFFFu, p01 >> 16, p23 & 0xFFFFu, p23 >> 16 };
          for (int32_t sl = 0; sl < kBlockSlots; ++sl)
            if (op[1] & (1 << sl))
              acc[sl] -= (kind == kBlockU ? sh * B[p[sl]] : B[p[sl]] * sh);
        }
        for (int32_t sl = 0; sl < n; ++sl)
        {
          double v = acc[sl];
          if (kind == kBlockL)
            v *= binv[blk[3]];
          B[bl.target[4 * k + sl]] = v;
          if (sl == diag)
            binv[blk[3]] = 1.0 / v;
        }
      }
      for (int32_t e = 0; e < nnz; ++e)
        if (std::memcmp(&A[e], &B[e], sizeof(double)) != 0)
          return false;
      // solves on the factor
      for (int fw = 1; fw >= 0; --fw)
      {
        const LevelSchedule& ss = fw ? m.fwd_serial : m.bwd_serial;
        const BlockedSchedule& bs = fw ? m.fwd_blocked : m.bwd_blocked;
        std::vector<double> x = x0, y = x0;
        for (size_t it = 0; it < ss.item_target.size(); ++it)
        {
          const int32_t i = ss.item_target[it];
          double v = x[i];
          for (int32_t t = ss.term_start[it]; t < ss.term_start[it + 1]; ++t)
            v -= A[ss.term_a[t]] * x[ss.term_b[t]];
          const int32_t aux = ss.item_aux[it];
          x[i] = aux >= 0 ? v / A[aux] : v;
        }
        for (int32_t k = 0; k < bs.n_blocks; ++k)
        {
          const int32_t* blk = &bs.block[4 * k];
          const int32_t n = blk[2] & 0xF;
          double acc[kBlockSlots] = { 0, 0, 0, 0 };
          for (int32_t sl = 0; sl < n; ++sl)
            acc[sl] = y[bs.target[4 * k + sl]];
          for (int32_t o = blk[0]; o < blk[0] + blk[1]; ++o)
          {
            const int32_t* op = &bs.op[4 * o];
            const double sh = y[op[0]];
            const uint32_t p01 = (uint32_t)op[2], p23 = (uint32_t)op[3];
            const uint32_t p[4] = { p01 & 0xFFFFu, p01 >> 16, p23 & 0xFFFFu, p23 >> 16 };
            for (int32_t sl = 0; sl < kBlockSlots; ++sl)
              if (op[1] & (1 << sl))
                acc[sl] -= A[p[sl]] * sh;
          }
          for (int32_t sl = 0; sl < n; ++sl)
          {
            const int32_t aux = bs.aux[4 * k + sl];
            y[bs.target[4 * k + sl]] = aux >= 0 ? acc[sl] / A[aux] : acc[sl];
          }
        }
        for (int32_t i = 0; i < S; ++i)
          if (std::memcmp(&x[i], &y[i], sizeof(double)) != 0)
            return false;
      }
      return true;
    }
  }  // namespace

  std::vector<int32_t> DiagonalMarkowitz(int32_t n, const std::vector<std::pair<int32_t, int32_t>>& nonzeros)
  {
    // Same selection rule and tie-break as micm's sparse Markowitz scan: the
    // live node with the smallest (row_deg-1)*(col_deg-1), computed in
    // unsigned 64-bit arithmetic (micm::Index), first index wins ties.
    std::vector<std::set<int32_t>> out(n), in(n);
    for (const auto& e : nonzeros)
    {
      out[e.first].insert(e.second);
      in[e.second].insert(e.first);
    }
    std::vector<uint64_t> row_deg(n), col_deg(n);
    for (int32_t v = 0; v < n; ++v)
    {
      row_deg[v] = out[v].size();
      col_deg[v] = in[v].size();
    }
    std::vector<char> alive(n, 1);
    std::vector<int32_t> perm;
    perm.reserve(n);
    for (int32_t step = 0; step < n; ++step)
    {
      int32_t pivot = n;
      uint64_t best = ~0ull;
      for (int32_t v = 0; v < n; ++v)
      {
        if (!alive[v])
          continue;
        const uint64_t cost = (row_deg[v] - 1ull) * (col_deg[v] - 1ull);
        if (pivot == n || cost < best)
        {
          best = cost;
          pivot = v;
        }
      }
      perm.push_back(pivot);
      alive[pivot] = 0;
      std::vector<int32_t> cols, ins;
      for (int32_t c : out[pivot])
        if (c != pivot && alive[c])
          cols.push_back(c);
      for (int32_t i : in[pivot])
        if (i != pivot && alive[i])
          ins.push_back(i);
      for (int32_t i : ins)
        for (int32_t c : cols)
          if (out[i].insert(c).second)
          {
            ++row_deg[i];
            in[c].insert(i);
            ++col_deg[c];
          }
      for (int32_t c : cols)
      {
        in[c].erase(pivot);
        --col_deg[c];
      }
      for (int32_t i : ins)
      {
        out[i].erase(pivot);
        --row_deg[i];
      }
    }
    return perm;
  }

  CompiledMechanism Compile(const micmb_mechanism_desc& d)
  {
    Require(d.n_species > 0, "mechanism has no species");
    Require(d.n_reactions >= 0, "negative reaction count");
    Require(d.n_species < 32768, "too many species (limit 32767)");
    const int32_t S = d.n_species, R = d.n_reactions;
    Require(R == 0 || (d.rate_type && d.rate_params && d.reactant_start && d.product_start),
            "null mechanism arrays");
    for (int32_t r = 0; r < R; ++r)
    {
      Require(d.rate_type[r] >= 0 && d.rate_type[r] <= MICMB_RATE_SURFACE,
              "reaction " + std::to_string(r) + ": unsupported rate-constant kind");
      Require(d.reactant_start[r] <= d.reactant_start[r + 1] && d.product_start[r] <= d.product_start[r + 1],
              "reaction " + std::to_string(r) + ": bad reactant/product offsets");
      int nparam = 0;
      for (int32_t i = d.reactant_start[r]; i < d.reactant_start[r + 1]; ++i)
      {
        const int32_t s = d.reactant_species[i];
        Require(s < S && (s >= 0 || -s - 1 < d.n_parameterized),
                "reaction " + std::to_string(r) + ": reactant index out of range");
        if (s < 0)
          ++nparam;
      }
      Require(nparam <= MICMB_MAX_PARAMETERIZED,
              "reaction " + std::to_string(r) + ": more parameterized reactants than supported");
      for (int32_t i = d.product_start[r]; i < d.product_start[r + 1]; ++i)
        Require(d.product_species[i] >= 0 && d.product_species[i] < S,
                "reaction " + std::to_string(r) + ": product index out of range");
    }

    CompiledMechanism m;
    m.S = S;
    m.R = R;

    // 1. stable sort by rate-constant kind (solver_builder.inl:274-329)
    std::vector<int32_t> order(R);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return d.rate_type[a] < d.rate_type[b]; });
    m.reaction_column.assign(R, 0);
    for (int32_t i = 0; i < R; ++i)
      m.reaction_column[order[i]] = i;

    // 2. species columns (solver_builder.inl:78-119)
    m.species_column.resize(S);
    std::iota(m.species_column.begin(), m.species_column.end(), 0);
    auto collect_nonzeros = [&](const std::vector<int32_t>& col) {
      std::set<std::pair<int32_t, int32_t>> ids;
      for (int32_t r = 0; r < R; ++r)
      {
        std::vector<int32_t> re, pr;
        for (int32_t i = d.reactant_start[r]; i < d.reactant_start[r + 1]; ++i)
          if (d.reactant_species[i] >= 0)
            re.push_back(col[d.reactant_species[i]]);
        for (int32_t i = d.product_start[r]; i < d.product_start[r + 1]; ++i)
          pr.push_back(col[d.product_species[i]]);
        for (int32_t ind : re)
        {
          for (int32_t dep : re)
            ids.insert({ dep, ind });
          for (int32_t dep : pr)
            ids.insert({ dep, ind });
        }
      }
      return ids;
    };
    if (d.reorder_state)
    {
      auto ids = collect_nonzeros(m.species_column);
      std::vector<std::pair<int32_t, int32_t>> nz(ids.begin(), ids.end());
      auto perm = DiagonalMarkowitz(S, nz);
      for (int32_t i = 0; i < S; ++i)
        m.species_column[perm[i]] = i;
    }

    // 2b. algebraic constraints (constraint_set.hpp:90-160): the algebraic
    //     species' rows become algebraic (mass-matrix diagonal 0)
    m.mass.assign(S, 1.0);
    std::vector<char> algebraic(S, 0);
    Require(d.n_constraints >= 0, "negative constraint count");
    if (d.n_constraints > 0)
    {
      Require(d.constraint_type && d.constraint_species && d.constraint_term_start && d.constraint_n_reactants &&
                  d.constraint_params,
              "constraint arrays missing");
      Require(d.constraint_term_start[0] == 0, "constraint_term_start[0] must be 0");
      const int32_t n_terms = d.constraint_term_start[d.n_constraints];
      Require(n_terms == 0 || (d.constraint_term_species && d.constraint_term_coef), "constraint terms missing");
      for (int32_t c = 0; c < d.n_constraints; ++c)
      {
        CompiledMechanism::ConstraintDef cd;
        cd.kind = d.constraint_type[c];
        Require(cd.kind == MICMB_CONSTRAINT_LINEAR || cd.kind == MICMB_CONSTRAINT_EQUILIBRIUM, "unknown constraint kind");
        const int32_t sp = d.constraint_species[c];
        Require(sp >= 0 && sp < S, "constraint algebraic species out of range");
        cd.row = m.species_column[sp];
        Require(!algebraic[cd.row], "a species is the algebraic variable of two constraints");
        algebraic[cd.row] = 1;
        m.mass[cd.row] = 0.0;
        const int32_t a = d.constraint_term_start[c], b = d.constraint_term_start[c + 1];
        Require(a <= b && b <= n_terms && b > a, "constraint terms out of order or empty");
        cd.t0 = (int32_t)m.c_term_col.size();
        for (int32_t t = a; t < b; ++t)
        {
          const int32_t ts = d.constraint_term_species[t];
          Require(ts >= 0 && ts < S, "constraint term species out of range");
          m.c_term_col.push_back(m.species_column[ts]);
          m.c_term_coef.push_back(d.constraint_term_coef[t]);
        }
        cd.t1 = (int32_t)m.c_term_col.size();
        cd.n_react = cd.kind == MICMB_CONSTRAINT_EQUILIBRIUM ? d.constraint_n_reactants[c] : 0;
        Require(cd.n_react >= 0 && cd.n_react <= b - a, "equilibrium reactant count out of range");
        for (int i = 0; i < 4; ++i)
          cd.p[i] = d.constraint_params[4 * (size_t)c + i];
        if (cd.kind == MICMB_CONSTRAINT_EQUILIBRIUM)
          cd.keq = m.n_eq++;
        m.constraints.push_back(cd);
      }
    }

    // 3. rate definitions and reactant/product tables by rate column
    int32_t next_param = 0;
    m.param_column.assign(R, -1);
    m.rates.resize(R);
    m.react_start.push_back(0);
    m.prod_start.push_back(0);
    for (int32_t rc = 0; rc < R; ++rc)
    {
      const int32_t r = order[rc];
      RateDef& def = m.rates[rc];
      def.kind = d.rate_type[r];
      def.input_index = r;
      const double* p = d.rate_params + (size_t)r * MICMB_RATE_PARAM_STRIDE;
      for (int i = 0; i < MICMB_RATE_PARAM_STRIDE; ++i)
        def.p[i] = p[i];
      switch (def.kind)
      {
        case MICMB_RATE_BRANCHED:
        {
          // ReactionRateConstantStore::BuildFrom precomputation (reaction_rate_store.hpp:268-281):
          // p = [branch, X, Y, a0, n] -> [branch, X, Y, a0, n, k0, z]
          const double n = std::floor(p[4]);
          const double k0 = 2.0e-22 * kAvogadro * 1.0e-6 * std::exp(n);
          const double air_ref = 2.45e19 / kAvogadro * 1.0e6;
          const double a = k0 * air_ref;
          const double b = 0.43 * std::pow(293.0 / 298.0, -8.0);
          const double A_val = a / (1.0 + a / b) * std::pow(0.41, 1.0 / (1.0 + std::pow(std::log10(a / b), 2.0)));
          def.p[5] = k0;
          def.p[6] = A_val * (1.0 - p[3]) / p[3];
          break;
        }
        case MICMB_RATE_TAYLOR_SERIES:
          Require(p[5] >= 1 && p[5] <= 16, "TaylorSeries needs 1..16 coefficients");
          break;
        case MICMB_RATE_USER_DEFINED:
          def.param_col = next_param;
          next_param += 1;
          break;
        case MICMB_RATE_SURFACE:
          // p = [D_g, MW, gamma] -> [D_g, 8R/(pi MW), gamma] (reaction_rate_store.hpp:300-314)
          Require(p[1] > 0, "surface reaction needs a positive molecular weight");
          def.p[1] = 8.0 * kGas / (kPi * p[1]);
          def.param_col = next_param;
          next_param += 2;
          break;
        default: break;
      }
      m.param_column[r] = def.param_col;
      for (int32_t i = d.reactant_start[r]; i < d.reactant_start[r + 1]; ++i)
      {
        const int32_t s = d.reactant_species[i];
        if (s >= 0)
          m.react_ids.push_back(m.species_column[s]);
        else
        {
          const double* c = d.parameterized_coef + 4 * (size_t)(-s - 1);
          for (int q = 0; q < 4; ++q)
            def.mult[def.n_mult][q] = c[q];
          def.n_mult++;
        }
      }
      m.react_start.push_back((int32_t)m.react_ids.size());
      for (int32_t i = d.product_start[r]; i < d.product_start[r + 1]; ++i)
      {
        m.prod_ids.push_back(m.species_column[d.product_species[i]]);
        m.prod_yield.push_back(d.product_yield[i]);
      }
      m.prod_start.push_back((int32_t)m.prod_ids.size());
    }
    m.P = next_param;

    // 4. Jacobian infos: (independent column, process) stably sorted by column
    //    (process_set.hpp:329-391)
    std::vector<std::pair<int32_t, int32_t>> columns;
    for (int32_t rc = 0; rc < R; ++rc)
      for (int32_t i = m.react_start[rc]; i < m.react_start[rc + 1]; ++i)
        columns.push_back({ m.react_ids[i], rc });
    std::stable_sort(columns.begin(), columns.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    m.info_dep_start.push_back(0);
    for (const auto& c : columns)
    {
      m.info_ind.push_back(c.first);
      m.info_rxn.push_back(c.second);
      bool found = false;
      for (int32_t i = m.react_start[c.second]; i < m.react_start[c.second + 1]; ++i)
      {
        if (m.react_ids[i] == c.first && !found)
        {
          found = true;
          continue;
        }
        m.info_dep_ids.push_back(m.react_ids[i]);
      }
      m.info_dep_start.push_back((int32_t)m.info_dep_ids.size());
    }

    // 5. sparsity: ProcessSet::NonZeroJacobianElements + diagonal, then LU fill
    std::set<std::pair<int32_t, int32_t>> nz;
    for (int32_t rc = 0; rc < R; ++rc)
      for (int32_t i = m.react_start[rc]; i < m.react_start[rc + 1]; ++i)
      {
        const int32_t ind = m.react_ids[i];
        for (int32_t j = m.react_start[rc]; j < m.react_start[rc + 1]; ++j)
          nz.insert({ m.react_ids[j], ind });
        for (int32_t j = m.prod_start[rc]; j < m.prod_start[rc + 1]; ++j)
          nz.insert({ m.prod_ids[j], ind });
      }
    for (int32_t i = 0; i < S; ++i)
      nz.insert({ i, i });
    if (!m.constraints.empty())
    {
      // kinetic entries of algebraic rows go (solver_builder.inl:377-389); the
      // constraints' own entries and diagonals come in
      for (auto it = nz.begin(); it != nz.end();)
        it = algebraic[it->first] ? nz.erase(it) : std::next(it);
      for (const CompiledMechanism::ConstraintDef& cd : m.constraints)
      {
        nz.insert({ cd.row, cd.row });
        for (int32_t t = cd.t0; t < cd.t1; ++t)
          nz.insert({ cd.row, m.c_term_col[t] });
      }
    }
    m.pattern_unfilled.assign(nz.begin(), nz.end());
    std::vector<std::set<int32_t>> row_cols(S), col_rows(S);
    for (const auto& e : nz)
    {
      row_cols[e.first].insert(e.second);
      col_rows[e.second].insert(e.first);
    }
    for (int32_t i = 0; i < S; ++i)
    {
      std::vector<int32_t> U(row_cols[i].upper_bound(i), row_cols[i].end());
      std::vector<int32_t> Lr(col_rows[i].upper_bound(i), col_rows[i].end());
      for (int32_t k : U)
        for (int32_t j : Lr)
          if (row_cols[j].insert(k).second)
            col_rows[k].insert(j);
    }
    for (int32_t i = 0; i < S; ++i)
      for (int32_t j : row_cols[i])
      {
        m.position[{ i, j }] = (int32_t)m.nz_row.size();
        m.nz_row.push_back(i);
        m.nz_col.push_back(j);
      }
    m.nnz = (int32_t)m.nz_row.size();
    Require(m.nnz < (1 << 30), "Jacobian too large");
    m.diag_pos.resize(S);
    for (int32_t i = 0; i < S; ++i)
      m.diag_pos[i] = m.position.at({ i, i });
    auto pos = [&](int32_t r, int32_t c) { return m.position.at({ r, c }); };

    // 6. forcing gather per species (process_set.hpp:524-590 order)
    {
      std::vector<std::vector<std::pair<int32_t, double>>> terms(S);
      for (int32_t rc = 0; rc < R; ++rc)
      {
        for (int32_t i = m.react_start[rc]; i < m.react_start[rc + 1]; ++i)
          terms[m.react_ids[i]].push_back({ rc, -1.0 });
        for (int32_t i = m.prod_start[rc]; i < m.prod_start[rc + 1]; ++i)
          terms[m.prod_ids[i]].push_back({ rc, m.prod_yield[i] });
      }
      m.f_start.push_back(0);
      for (int32_t s = 0; s < S; ++s)
      {
        if (algebraic[s])
          terms[s].clear();  // the constraint's residual replaces the row
        for (const auto& t : terms[s])
        {
          m.f_rxn.push_back(t.first);
          m.f_coef.push_back(t.second);
        }
        m.f_start.push_back((int32_t)m.f_rxn.size());
      }
    }

    // 7. -J gather per nonzero (process_set.hpp:594-670 order)
    {
      std::vector<std::vector<std::pair<int32_t, double>>> terms(m.nnz);
      for (int32_t info = 0; info < (int32_t)m.info_rxn.size(); ++info)
      {
        const int32_t ind = m.info_ind[info], rc = m.info_rxn[info];
        // process terms of algebraic rows are skipped (process_set.hpp:623-660)
        for (int32_t i = m.info_dep_start[info]; i < m.info_dep_start[info + 1]; ++i)
          if (!algebraic[m.info_dep_ids[i]])
            terms[pos(m.info_dep_ids[i], ind)].push_back({ info, 1.0 });
        if (!algebraic[ind])
          terms[pos(ind, ind)].push_back({ info, 1.0 });
        for (int32_t i = m.prod_start[rc]; i < m.prod_start[rc + 1]; ++i)
          if (!algebraic[m.prod_ids[i]])
            terms[pos(m.prod_ids[i], ind)].push_back({ info, -m.prod_yield[i] });
      }
      m.j_start.push_back(0);
      for (int32_t e = 0; e < m.nnz; ++e)
      {
        for (const auto& t : terms[e])
        {
          m.j_info.push_back(t.first);
          m.j_coef.push_back(t.second);
        }
        m.j_start.push_back((int32_t)m.j_info.size());
      }
    }

    // 7b. constraint Jacobian positions, and per position the constraint
    //     terms it receives in micm's order (constraint order; an equilibrium
    //     constraint's reactants, then its products)
    m.cj_start.assign(1, 0);
    if (!m.constraints.empty())
    {
      m.c_term_pos.resize(m.c_term_col.size());
      std::vector<std::vector<int32_t>> at(m.nnz);
      for (const CompiledMechanism::ConstraintDef& cd : m.constraints)
        for (int32_t t = cd.t0; t < cd.t1; ++t)
        {
          m.c_term_pos[t] = pos(cd.row, m.c_term_col[t]);
          at[m.c_term_pos[t]].push_back(t);
        }
      for (int32_t e = 0; e < m.nnz; ++e)
      {
        for (int32_t t : at[e])
          m.cj_term.push_back(t);
        m.cj_start.push_back((int32_t)m.cj_term.size());
      }
    }

    // 8. LU in Crout form (same per-entry update order as
    //    lu_decomposition_mozart_in_place.inl:171-210)
    {
      std::vector<RawItem> items;
      std::map<int32_t, int32_t> item_of_pos;
      for (int32_t mn = 0; mn < S; ++mn)
      {
        auto add = [&](int32_t j, int32_t k) {
          RawItem it;
          it.target = pos(j, k);
          it.aux = j > k ? pos(k, k) : -1;
          const int32_t lim = std::min(j, k);
          for (int32_t i : row_cols[j])
          {
            if (i >= lim)
              break;
            auto f = m.position.find({ i, k });
            if (f == m.position.end())
              continue;
            it.terms.push_back({ pos(j, i), f->second });
            it.term_dep.push_back({ item_of_pos.at(pos(j, i)), item_of_pos.at(f->second) });
          }
          if (j > k)
          {
            it.final_dep.push_back(item_of_pos.at(pos(k, k)));
            m.lu_lower++;
          }
          m.lu_updates += (int32_t)it.terms.size();
          item_of_pos[it.target] = (int32_t)items.size();
          items.push_back(std::move(it));
        };
        for (int32_t k : row_cols[mn])
          if (k >= mn)
            add(mn, k);
        for (int32_t j : col_rows[mn])
          if (j > mn)
            add(j, mn);
      }
      m.lu = Schedule(items);
      m.lu_serial = SerialSchedule(items);
    }

    // 9. triangular solves (linear_solver_in_place.inl:49-103, 113-167) and
    //    their transposes for the adjoint
    {
      std::vector<RawItem> f, b, ft, bt;
      for (int32_t i = 0; i < S; ++i)
      {
        RawItem it;
        it.target = i;
        it.aux = -1;
        for (int32_t j : row_cols[i])
        {
          if (j >= i)
            break;
          it.terms.push_back({ pos(i, j), j });
          it.term_dep.push_back({ j });
        }
        f.push_back(std::move(it));
      }
      m.fwd = Schedule(f);
      m.fwd_serial = SerialSchedule(f);
      // backward: visit i = S-1 .. 0; item index v = S-1-i
      for (int32_t v = 0; v < S; ++v)
      {
        const int32_t i = S - 1 - v;
        RawItem it;
        it.target = i;
        it.aux = pos(i, i);
        for (int32_t j : row_cols[i])
          if (j > i)
          {
            it.terms.push_back({ pos(i, j), j });
            it.term_dep.push_back({ S - 1 - j });
          }
        b.push_back(std::move(it));
      }
      m.bwd = Schedule(b);
      m.bwd_serial = SerialSchedule(b);
      for (int32_t i = 0; i < S; ++i)
      {
        RawItem it;
        it.target = i;
        it.aux = pos(i, i);
        for (int32_t j : col_rows[i])
        {
          if (j >= i)
            break;
          it.terms.push_back({ pos(j, i), j });
          it.term_dep.push_back({ j });
        }
        ft.push_back(std::move(it));
      }
      m.fwd_t = Schedule(ft);
      m.fwd_t_serial = SerialSchedule(ft);
      for (int32_t v = 0; v < S; ++v)
      {
        const int32_t i = S - 1 - v;
        RawItem it;
        it.target = i;
        it.aux = -1;
        for (int32_t j : col_rows[i])
          if (j > i)
          {
            it.terms.push_back({ pos(j, i), j });
            it.term_dep.push_back({ S - 1 - j });
          }
        bt.push_back(std::move(it));
      }
      m.bwd_t = Schedule(bt);
      m.bwd_t_serial = SerialSchedule(bt);
    }

    // 9b. register-blocked serial forms (16-bit slot operands), kept only when
    //     they reproduce the serial forms bit for bit
    if (m.nnz <= 0xFFFF && S <= 0xFFFF)
    {
      m.lu_blocked = BlockLu(S, row_cols, col_rows, m.position);
      m.fwd_blocked = BlockSolve(S, row_cols, m.position, true);
      m.bwd_blocked = BlockSolve(S, row_cols, m.position, false);
      m.has_blocked = BlockedMatchesSerial(m);
      if (!m.has_blocked)
        m.lu_blocked = m.fwd_blocked = m.bwd_blocked = BlockedSchedule{};
    }

    // 10. warp-interleaved tables for the fused kernel (16-bit operand positions)
    const int32_t scratch_cols = std::max<int32_t>(R, (int32_t)m.info_rxn.size());
    m.scratch_zero = scratch_cols;
    if (m.nnz + 1 <= 0xFFFF && S + 1 < 0x7FFF && scratch_cols + 1 <= 0xFFFF)
    {
      const uint32_t NZ = (uint32_t)m.nnz, SV = (uint32_t)S;
      auto pack2 = [](uint32_t a, uint32_t b) { return a | (b << 16); };
      m.w_lu = BuildWarp(
          m.lu,
          [&](int32_t i) {
            const int32_t e = m.lu.item_target[i];
            const int32_t j = m.nz_row[e], k = m.nz_col[e];
            uint32_t hi = (j < k) ? 0xFFFFu : (j == k ? (0x8000u | (uint32_t)j) : (uint32_t)k);
            if (m.lu.item_aux[i] == -2)
              hi = 0xFFFEu;  // partial sum
            return (uint32_t)e | (hi << 16);
          },
          [&](int32_t t) { return pack2((uint32_t)m.lu.term_a[t], (uint32_t)m.lu.term_b[t]); }, pack2(NZ, NZ),
          nullptr, [&](int32_t i) {
            const int32_t e = m.lu.item_target[i];
            return (m.lu.item_aux[i] != -2 && m.nz_row[e] == m.nz_col[e]) ? kSegRecip : 0;
          });
      auto solve_table = [&](const LevelSchedule& s) {
        return BuildWarp(
            s,
            [&](int32_t i) {
              const uint32_t hi = s.item_aux[i] == -2 ? 0xFFFEu : (s.item_aux[i] < 0 ? 0xFFFFu : (uint32_t)s.item_aux[i]);
              return (uint32_t)s.item_target[i] | (hi << 16);
            },
            [&](int32_t t) { return pack2((uint32_t)s.term_a[t], (uint32_t)s.term_b[t]); }, pack2(NZ, SV), nullptr,
            [](int32_t) { return 0; });
      };
      m.w_fwd = solve_table(m.fwd);
      m.w_bwd = solve_table(m.bwd);
      m.w_fwd_t = solve_table(m.fwd_t);
      m.w_bwd_t = solve_table(m.bwd_t);
      std::vector<double> fco, jco;
      const LevelSchedule fs = GatherSchedule(m.f_start, m.f_rxn, m.f_coef, fco);
      m.w_forcing = BuildWarp(
          fs, [&](int32_t i) { return (uint32_t)fs.item_target[i] | (0xFFFFu << 16); },
          [&](int32_t t) { return (uint32_t)fs.term_a[t]; }, (uint32_t)m.scratch_zero, &fco,
          [](int32_t) { return 0; });
      const LevelSchedule js = GatherSchedule(m.j_start, m.j_info, m.j_coef, jco);
      m.w_jacobian = BuildWarp(
          js,
          [&](int32_t i) {
            const int32_t e = js.item_target[i];
            const uint32_t hi = (m.nz_row[e] == m.nz_col[e]) ? (0x8000u | (uint32_t)m.nz_row[e]) : 0xFFFFu;
            return (uint32_t)e | (hi << 16);
          },
          [&](int32_t t) { return (uint32_t)js.term_a[t]; }, (uint32_t)m.scratch_zero, &jco,
          [](int32_t) { return 0; });
      m.has_warp_tables = true;
      bool narrow = true;
      for (int32_t r = 0; r < R; ++r)
        narrow &= (m.react_start[r + 1] - m.react_start[r]) <= 3;
      if (narrow)
      {
        const int32_t one = S + 1;
        m.rate_desc.assign((size_t)4 * R, one);
        for (int32_t r = 0; r < R; ++r)
          for (int32_t i = m.react_start[r]; i < m.react_start[r + 1]; ++i)
            m.rate_desc[(size_t)4 * r + (i - m.react_start[r])] = m.react_ids[i];
        const int32_t ni = (int32_t)m.info_rxn.size();
        m.drate_desc.assign((size_t)4 * ni, one);
        for (int32_t i = 0; i < ni; ++i)
        {
          m.drate_desc[(size_t)4 * i] = m.info_rxn[i];
          for (int32_t d = m.info_dep_start[i]; d < m.info_dep_start[i + 1]; ++d)
            m.drate_desc[(size_t)4 * i + 1 + (d - m.info_dep_start[i])] = m.info_dep_ids[d];
        }
      }
      std::map<uint64_t, uint32_t> seen;
      m.stream = StreamProgram{};
      AppendStreamPhase(m.stream, seen, m.w_forcing, m.stream.forcing);
      AppendStreamPhase(m.stream, seen, m.w_jacobian, m.stream.jacobian);
      AppendStreamPhase(m.stream, seen, m.w_lu, m.stream.lu);
      AppendStreamPhase(m.stream, seen, m.w_fwd, m.stream.fwd);
      AppendStreamPhase(m.stream, seen, m.w_bwd, m.stream.bwd);
      AppendStreamPhase(m.stream, seen, m.w_fwd_t, m.stream.fwd_t);
      AppendStreamPhase(m.stream, seen, m.w_bwd_t, m.stream.bwd_t);
      // operands are addressed by 16-bit byte offsets from their array
      const int64_t limit = 0xFFFF / 8;
      if (m.nnz + 1 >= limit || S + 2 >= limit || scratch_cols + 1 >= limit ||
          (int64_t)m.stream.coef_table.size() >= limit)
        m.stream = StreamProgram{};
    }

    // 11. hash of everything the device sees
    uint64_t h = 1469598103934665603ull;
    h = Fnv(h, &m.S, sizeof(m.S));
    h = Fnv(h, &m.R, sizeof(m.R));
    h = FnvVec(h, m.nz_row);
    h = FnvVec(h, m.nz_col);
    h = FnvVec(h, m.react_ids);
    h = FnvVec(h, m.prod_ids);
    h = FnvVec(h, m.prod_yield);
    for (const auto& r : m.rates)
      h = Fnv(h, &r.kind, sizeof(r.kind));
    h = FnvVec(h, m.c_term_col);
    h = FnvVec(h, m.c_term_coef);
    for (const auto& cd : m.constraints)
    {
      h = Fnv(h, &cd.kind, sizeof(cd.kind));
      h = Fnv(h, &cd.row, sizeof(cd.row));
      h = Fnv(h, cd.p, sizeof(cd.p));
    }
    m.hash = h;
    return m;
  }
}  // namespace micmb
