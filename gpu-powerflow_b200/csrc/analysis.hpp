// analysis.hpp -- one-time host analysis of a power-flow case.
//
// Two stages, both value independent and run once per grid:
//
//  1. Jacobian analysis: bus <-> Jacobian index tables, the CSR pattern of the
//     2x2-block Jacobian and the per-Ybus-entry scatter maps.  Same arrays as
//     the reference's make_jacobian_indexing / JacobianPatternGenerator /
//     JacobianMapBuilder (cuPF/cpp/src/newton_solver/ops/jacobian/
//     jacobian_analysis.cpp:257-445).
//
//  2. Symbolic factorisation plan of the Jacobian pattern: METIS nested
//     dissection (seed 42), elimination tree, symbolic Cholesky fill of
//     A + A^T, relaxed panels (cap = max_panel_width), multifrontal fronts with
//     their extend-add maps, panel levels, the dense front layout and the
//     per-entry front position a_pos.  Same arrays as the reference's
//     BuildPlanSeed / AnalyzeMultifrontal (custom_linear_solver/src/analyze/
//     pipeline.cpp:199-332, analyze/plan/lower.cu:572-644).
//
// On top of that plan, build_factor_program() derives the engine's own
// scenario-interleaved factor program (row assembly lists, storage offsets,
// level work lists) that the CUDA kernels consume.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace cupf_b200 {

struct JacobianAnalysis {
  int32_t n_bus = 0, n_pv = 0, n_pq = 0, n_pvpq = 0, dim = 0, nnz = 0;
  std::vector<int32_t> row_pvpq, row_pq;  // bus -> J row (angle/P, magnitude/Q), -1 absent
  std::vector<int32_t> row_ptr, col_idx;  // CSR pattern, columns sorted per row
  std::vector<int32_t> map11, map21, map12, map22;      // per Ybus entry (CSR order)
  std::vector<int32_t> diag11, diag21, diag12, diag22;  // per bus
  bool every_slot_mapped = false;  // true when each J slot receives exactly one Ybus entry
};

// Throws std::invalid_argument on bad indices.
JacobianAnalysis analyze_jacobian(int32_t n_bus, const int32_t* indptr, const int32_t* indices,
                                  const int32_t* pv, int32_t n_pv, const int32_t* pq, int32_t n_pq);

struct SymbolicOptions {
  int max_panel_width = 8;   // relaxed-panel cap (clamped to [1, 64])
  bool serial_nd = true;     // one METIS_NodeND call; false = separator recursion
  int metis_seed = 42;
  bool use_matching = false;  // structural (Hopcroft-Karp) column matching
  // separator recursion (serial_nd = false): depth and base-case sizes, the
  // small one below 20,000 vertices (SolverConfig::parallel_nd_*, solver.hpp:44-46)
  int par_nd_depth = 4, par_nd_base_small = 4000, par_nd_base_large = 20000;
};

struct SymbolicPlan {
  int32_t n = 0, nnz = 0;
  // ordering
  std::vector<int32_t> graph_xadj, graph_adjncy;  // A + A^T without the diagonal
  std::vector<int32_t> perm, iperm;               // perm[new] = old row; iperm[old col] = new col
  std::vector<int32_t> row_iperm, col_perm;       // iperm[old row] = new row; col_perm[new] = old col
  std::vector<int32_t> row_to_col;                // structural matching (empty without)
  std::vector<int32_t> sym_col_ptr, sym_row_idx;  // relabelled graph
  // elimination tree + fill
  std::vector<int32_t> parent;
  std::vector<int32_t> Lp, Li;                    // per-column sets, rows ascending
  // panels and fronts
  int32_t num_panels = 0;
  std::vector<int32_t> panel_first, panel_ncols, panel_width, panel_of;
  std::vector<int32_t> front_ptr, front_rows, panel_parent, asm_ptr, asm_idx, asm_local;
  // levels (panel e-tree depth from the leaves)
  int32_t num_levels = 0;
  std::vector<int32_t> plevel, level_ptr, plcols_level;
  // dense front layout of the reference (arena offsets) and entry positions
  std::vector<int32_t> front_off;
  int64_t front_total = 0;
  std::vector<int32_t> a_pos_csr;  // per Jacobian CSR entry: front_off[p] + r * fsz + c
  std::vector<int32_t> a_owner;    // per Jacobian CSR entry: owning panel
  std::vector<int32_t> a_row, a_col;  // per Jacobian CSR entry: position inside the front
};

// Per-front structure as CSV text (the columns of the reference's
// MaybeDumpFronts, custom_linear_solver/src/analyze/pipeline.cpp:162-193):
// q,p,fsz,nc,uc,level,parent,asm_len,extend_elems, one row per panel, levels
// leaves first and each level's panels in ascending order (plcols_level).
std::string fronts_csv(const SymbolicPlan& sp);

SymbolicPlan analyze_symbolic(int32_t n, const int32_t* row_ptr, const int32_t* col_idx,
                              const SymbolicOptions& opt);

// ---------------------------------------------------------------------------
// Engine factor program (scenario-interleaved, one warp per front x 32 scenarios)
// ---------------------------------------------------------------------------
struct FactorProgram {
  int32_t P = 0, dim = 0, nnz = 0, num_levels = 0;
  int32_t max_fsz = 0, max_nc = 0;
  std::vector<int32_t> fsz, nc, first;            // per panel
  std::vector<int32_t> front_ptr, front_rows;     // per panel rows (permuted indices)
  std::vector<int64_t> u_off, l_off, cb_off;      // element offsets: U rows, L21, CB(+rhs col)
  int64_t u_total = 0, l_total = 0, cb_total = 0;
  // A sources per front row: entries [arow_ptr[fr], arow_ptr[fr+1]) with
  // (Jacobian CSR position, front column)
  std::vector<int32_t> arow_ptr, arow_q, arow_col;
  // CB sources per front row: (child panel, row inside the child's CB)
  std::vector<int32_t> crow_ptr, crow_child, crow_r;
  std::vector<int32_t> asm_local;                 // child CB index -> parent front position
  std::vector<int32_t> asm_ptr;
  std::vector<int32_t> level_ptr, level_fronts;   // fronts by level, bucket-sorted inside a level
  std::vector<int32_t> level_max_fsz;
  std::vector<int32_t> perm, iperm;          // row order; column inverse
  std::vector<int32_t> row_iperm, col_perm;  // row inverse; column order
  std::vector<int32_t> parent_panel;
  std::vector<int32_t> nchildren;
  // Dense-front assembly program: for front p, entries [fe_ptr[p], fe_ptr[p+1])
  // give a destination inside the (fsz x (fsz + 1)) front (last column = rhs)
  // and a source: kind (bits 62-63) 0 = Jacobian CSR position, 1 = CB element
  // (global index), 2 = mismatch row (pivot-order index).  Sorted by
  // destination, stable (J entries, mismatch rows, then children in order);
  // fe_split
  // (kFeChunks + 1 per front) cuts the list at destination boundaries into
  // chunks that different warps can accumulate without sharing a destination.
  std::vector<int64_t> fe_ptr;
  std::vector<int32_t> fe_dst;
  std::vector<int64_t> fe_src;
  std::vector<int64_t> fe_split;
  // Launch records in level order (24 int32 per front): fs, nc, first, p,
  // fe start, u_off, l_off, cb_off (int64 as two int32), the 8 fe_split cuts
  // relative to the fe start, front_ptr.
  std::vector<int32_t> front_meta;
};

constexpr int kFeChunks = 8;
constexpr int kFeKindShift = 62;

FactorProgram build_factor_program(const SymbolicPlan& sp);

}  // namespace cupf_b200
