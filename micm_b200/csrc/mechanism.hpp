// mechanism.hpp -- symbolic compile of a chemical mechanism for the B200 solver.
//
// Reproduces micm's numbering exactly, so every column and nonzero lines up
// with the reference solver:
//   * reactions stably sorted by rate-constant kind (solver_builder.inl:274-329)
//   * species order from diagonal Markowitz reordering of the Jacobian
//     sparsity (linear_solver.inl:30-124, solver_builder.inl:78-119)
//   * Jacobian sparsity (process_set.hpp:425-457) plus the diagonal
//     (util/jacobian.hpp:15-32), LU fill (lu_decomposition_mozart_in_place.inl:121-169)
//   * custom-parameter columns (solver_builder.inl:129-188)
// and then emits the device work lists in *gather* form with level schedules:
// every output value (forcing of a species, -J nonzero, LU nonzero, solution
// component) is one item whose terms are summed in exactly the order micm's
// scatter loops apply them, so a single lane can own an item and the result
// does not depend on how items are spread over lanes.
#pragma once

#include "../../include/micmb.h"

#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace micmb
{
  struct LevelSchedule
  {
    // items are grouped by level; level l holds items [level_start[l], level_start[l+1])
    std::vector<int32_t> level_start;
    std::vector<int32_t> item_target;  // value written by the item
    std::vector<int32_t> item_aux;     // diagonal position / -1
    std::vector<int32_t> term_start;   // [n_items + 1]
    std::vector<int32_t> term_a;       // first operand position
    std::vector<int32_t> term_b;       // second operand position
    int32_t n_items() const
    {
      return (int32_t)item_target.size();
    }
    int32_t n_levels() const
    {
      return level_start.empty() ? 0 : (int32_t)level_start.size() - 1;
    }
  };

  // A level schedule re-laid out for a 32-lane warp: the items of a level are
  // cut into chunks of 32 consecutive items (one per lane); the terms of a
  // chunk are stored lane-interleaved, term t of lane l at base + 32 t + l,
  // padded to the chunk's longest item with terms that read zero slots, so
  // one 128-byte line feeds a whole warp step.  Operands are 16-bit
  // positions packed in one 32-bit word.
  struct WarpTable
  {
    int32_t n_levels = 0;
    std::vector<int32_t> level_chunk_start;  // [n_levels + 1]
    std::vector<int32_t> chunk;              // [n_chunks * 4]: term base, T, first item, n items
    std::vector<uint32_t> item;              // packed item metadata
    std::vector<uint32_t> term;              // packed operand pair (a | b << 16)
    std::vector<double> coef;                // per-term coefficient (gathers with weights)
    uint32_t dummy = 0;                      // padding term (operands that hold 0)
    std::vector<int32_t> chunk_flags;        // [n_chunks]: extra segment flags (kSegRecip)
  };

  // The warp tables re-cut into fixed-size blocks for bulk (TMA) streaming
  // into a shared-memory ring.  Every term of every phase has one form,
  //   acc = acc - X[a] * Y[b],   packed as a | b << 16,
  // with X, Y chosen by the phase: LU (X = Y = factor), triangular solves
  // (X = factor, Y = vector), weighted gathers (X = rates, Y = the table of
  // negated coefficients `coef_table`; acc + c*w and acc - (-c)*w round
  // identically).  A block holds a 16-byte header (segment count) followed by
  // segments laid end to end:
  //   int4 {T, n | flags << 8 | U << 16, segment bytes, 0}
  //   uint32 items[U][n]           (padded to 16 bytes; kNoItem = empty slot)
  //   U = 1: uint4 terms[ceil(T/4)][n]  (lane l's terms 4g..4g+3 at g*n + l)
  //   U = 4: uint4 terms[T][n]          (term t of lane l's four items at t*n + l)
  // With U = 4 every lane carries four independent sums.  Lanes with fewer
  // than T terms are padded with products that are exactly +0 (operands
  // that hold 0), which leave every sum bit-identical.  A chunk whose terms
  // do not fit in the rest of a block continues in the next block
  // (FIRST/LAST flags; U = 1 splits fall on 4-term boundaries); LEVEL_END
  // marks the end of a dependency level (the warp synchronises there).
  constexpr int32_t kStreamBlockBytes = 8192;
  // kSegRecip: every item of the segment is a diagonal LU entry (store the
  // pivot and its reciprocal); all other LU items store sum * (1/a_kk or 1).
  constexpr int32_t kSegFirst = 1, kSegLast = 2, kSegLevelEnd = 4, kSegRecip = 8;
  constexpr uint32_t kNoItem = 0xFFFFFFFFu;
  constexpr int32_t kWideMaxSteps = 48;  // longest chunk run four-wide

  struct StreamPhase
  {
    int32_t first_block = 0;
    int32_t n_blocks = 0;
  };

  struct StreamProgram
  {
    std::vector<uint8_t> bytes;          // all blocks, each kStreamBlockBytes apart
    std::vector<int32_t> block_bytes;    // used bytes per block (multiple of 16)
    std::vector<double> coef_table;      // negated gather coefficients; entry 0 is +0
    StreamPhase forcing, jacobian, lu, fwd, bwd, fwd_t, bwd_t;
  };

  // Register-blocked serial forms for one thread per cell.  Items that share
  // an operand are grouped in blocks of up to kBlockSlots entries held in
  // registers; each op of a block loads the shared operand once and updates
  // the accumulators of the entries that use it, in increasing order of the
  // shared index, so every entry's terms come in the serial schedule's order
  // and every result is bit-identical to it.
  //   LU:     the U-row entries of one pivot row (shared a_{mn,i}) or the
  //           L-column entries of one pivot column (shared a_{i,mn}).
  //   solves: up to kBlockSlots rows of one dependency level (shared x_j).
  // block[4b..4b+3] = {first op, n ops, n slots | kind << 4 | (diag slot + 1) << 8, pivot row}
  // target[4b + s] = the entry (LU position or vector row) of slot s, -1 if unused
  // aux[4b + s]    = backward solve: position of the slot row's diagonal
  // op[4o..4o+3]   = {shared index, slot mask, slot 0 | slot 1 << 16, slot 2 | slot 3 << 16}
  constexpr int32_t kBlockSlots = 4;
  constexpr int32_t kBlockU = 0, kBlockL = 1, kBlockSolve = 2;
  struct BlockedSchedule
  {
    int32_t n_blocks = 0;
    std::vector<int32_t> block, target, aux, op;
  };

  struct RateDef
  {
    int32_t kind = 0;
    double p[MICMB_RATE_PARAM_STRIDE] = { 0 };  // derived parameters, see rates.cuh
    int32_t param_col = -1;                     // first custom-parameter column
    int32_t input_index = 0;                    // reaction index in the input description
    int32_t n_mult = 0;                         // parameterized reactants
    double mult[MICMB_MAX_PARAMETERIZED][4] = { { 0 } };
  };

  struct CompiledMechanism
  {
    int32_t S = 0;  // species (state columns)
    int32_t R = 0;  // reactions (rate columns)
    int32_t P = 0;  // custom parameters
    std::vector<int32_t> species_column;   // system species -> column
    std::vector<int32_t> reaction_column;  // input reaction -> rate column
    std::vector<int32_t> param_column;     // input reaction -> first custom column or -1
    std::vector<RateDef> rates;            // [R] by rate column

    // reactants / products per rate column, state columns (parameterized excluded)
    std::vector<int32_t> react_start, react_ids;
    std::vector<int32_t> prod_start, prod_ids;
    std::vector<double> prod_yield;

    // Jacobian: unfilled pattern and LU-filled pattern (row-major storage order)
    std::vector<std::pair<int32_t, int32_t>> pattern_unfilled;
    std::vector<int32_t> nz_row, nz_col;  // filled, storage order
    std::map<std::pair<int32_t, int32_t>, int32_t> position;
    std::vector<int32_t> diag_pos;  // [S]
    int32_t nnz = 0;

    // ProcessSet jacobian infos (process_set.hpp:329-391): (independent column, rate column)
    std::vector<int32_t> info_rxn, info_ind;
    std::vector<int32_t> info_dep_start, info_dep_ids;  // dependent reactants per info

    // forcing gather: item = species (target column), terms (rate column, coefficient)
    std::vector<int32_t> f_start, f_rxn;
    std::vector<double> f_coef;
    // -J gather: item = nonzero position, terms (info index, coefficient)
    std::vector<int32_t> j_start, j_info;
    std::vector<double> j_coef;

    LevelSchedule lu;      // Crout form: target a_jk, aux = diag pos of column k for j > k
    LevelSchedule fwd;     // L y = b (unit diagonal): target row i, terms (L_ij pos, j)
    LevelSchedule bwd;     // U x = y: target row i, aux = U_ii pos, terms (U_ij pos, j)
    LevelSchedule fwd_t;   // U^T w = g: target i, aux = U_ii pos, terms (U_ji pos, j)
    LevelSchedule bwd_t;   // L^T z = w: target i, terms (L_ji pos, j)
    // the same LU and solves as single-level lists in visiting order, every
    // item whole (no partial sums): the order one thread per cell runs them
    LevelSchedule lu_serial, fwd_serial, bwd_serial, fwd_t_serial, bwd_t_serial;
    // register-blocked forms of lu_serial, fwd_serial, bwd_serial (empty
    // unless every position fits 16 bits and the host check passed)
    bool has_blocked = false;
    BlockedSchedule lu_blocked, fwd_blocked, bwd_blocked;

    // warp-interleaved forms for the fused kernel (empty when the mechanism
    // exceeds 16-bit positions); dummy operands: LU slot nnz, vector slot S,
    // scratch slot `scratch_zero`, all holding 0.0
    bool has_warp_tables = false;
    int32_t scratch_zero = 0;
    // Fixed-width product lists for the fused kernels: rate_desc[4r..4r+2] are
    // the reactant columns of reaction r, drate_desc[4i] the rate column and
    // [4i+1..4i+3] the dependent columns of info i, padded with column S + 1
    // (a slot holding 1.0; multiplying by it is exact).  Empty unless every
    // reaction has at most three reactants.
    std::vector<int32_t> rate_desc, drate_desc;
    WarpTable w_lu, w_fwd, w_bwd, w_fwd_t, w_bwd_t, w_forcing, w_jacobian;
    StreamProgram stream;

    // algebraic constraints (DAE form; constraint_set.hpp).  Each replaces the
    // ODE row of its algebraic species: process terms are left out of that
    // row's forcing and -J gathers, the constraint residual G overwrites the
    // forcing, and -dG/dy fills the row's Jacobian entries.
    struct ConstraintDef
    {
      int32_t kind = 0;     // MICMB_CONSTRAINT_*
      int32_t row = 0;      // state column of the algebraic species
      int32_t t0 = 0, t1 = 0;  // terms [t0, t1) of c_term_*
      int32_t n_react = 0;  // equilibrium: leading reactant terms
      int32_t keq = -1;     // equilibrium: index of its K_eq among the cell's K_eq values
      double p[4] = { 0, 0, 0, 0 };
    };
    std::vector<ConstraintDef> constraints;  // input order
    std::vector<int32_t> c_term_col;         // state column of each term
    std::vector<double> c_term_coef;         // coefficient / stoichiometry
    std::vector<int32_t> c_term_pos;         // LU position of (row, term column)
    std::vector<double> mass;                // [S] mass-matrix diagonal: 1 ODE row, 0 algebraic row
    int32_t n_eq = 0;                        // equilibrium constraints
    // per LU position, the constraint terms whose derivative it receives, in
    // the order micm applies them (constraint order, reactants then products)
    std::vector<int32_t> cj_start, cj_term;

    int32_t lu_updates = 0;
    int32_t lu_lower = 0;
    uint64_t hash = 0;
  };

  // Throws std::runtime_error on invalid input.
  CompiledMechanism Compile(const micmb_mechanism_desc& desc);

  // Markowitz reorder of a square 0/1 pattern given as per-row column sets;
  // returns perm with perm[new] = old (linear_solver.inl:30-124).
  std::vector<int32_t> DiagonalMarkowitz(int32_t n, const std::vector<std::pair<int32_t, int32_t>>& nonzeros);
}  // namespace micmb
