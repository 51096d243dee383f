// ref_symbolic.cu -- the REFERENCE's own symbolic analysis, run on the host
// (TEST INFRASTRUCTURE ONLY).
//
// This translation unit compiles the reference's Analyze sources where they
// lie (custom_linear_solver/src/analyze/...) and calls their internal steps in
// the order of BuildPlanSeed (custom_linear_solver/src/analyze/pipeline.cpp:
// 199-332) and AnalyzeMultifrontal (analyze/plan/lower.cu:572-644).  The three
// device steps of that pipeline (BuildCscFromCsrDevice, BuildSymmetricGraph-
// Device, PermuteCscDevice; pattern_kernels.cu:171-403) and the a_pos kernel
// (lower.cu:35-62) have no host entry point, so this driver performs the same
// transformations on the host:
//   * CSR -> CSC with rows ascending inside each column (one of the orders the
//     device scatter can produce; the order never reaches a compared array);
//   * A + A^T adjacency = sorted unique directed edge keys, diagonal dropped;
//   * column relabel new_col = iperm[old_col], rows through iperm;
//   * a_pos[q] = front_off + r * fsz + c, reported in CSR order.
// With structural matching (use_matching), the reference's own
// StructuralMatchingFromCsc (pipeline.cpp:77-160) runs on that CSC, the rows
// follow the ND order and the columns their matched rows, the permuted CSC
// maps rows through row_iperm and columns through iperm (PermuteCscDeviceRc,
// pattern_kernels.cu:405-460), and the Etree / fill graph is A' + A'^T of the
// permuted matrix (pipeline.cpp:265-272).
// Everything else -- METIS ND, Etree, FillPattern, RelaxedPanels,
// ComputeMultifrontalSymbolic, panel levels, subtree/tier orders, assembly
// map, arena layout -- is the reference's code.
#include <unistd.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "analyze/pattern/pattern_kernels.cu"
#include "analyze/plan/lower.cu"
#include "analyze/pipeline.cpp"
#include "internal/plan/multifrontal_plan.cu"

namespace {

struct RefSymbolic {
  std::map<std::string, std::vector<int>> arrays;
  std::map<std::string, std::string> texts;
};

// The reference's MaybeDumpFronts (pipeline.cpp:162-193) writes to a path;
// its output is read back as text.
std::string dump_fronts_text(const custom_linear_solver::plan::MultifrontalPlan& plan) {
  char path[] = "/tmp/ref_fronts_XXXXXX";
  const int fd = mkstemp(path);
  if (fd < 0) return std::string();
  close(fd);
  custom_linear_solver::plan::MaybeDumpFronts(plan, path);
  std::string text;
  if (FILE* f = std::fopen(path, "r")) {
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, k);
    std::fclose(f);
  }
  std::remove(path);
  return text;
}

}  // namespace

extern "C" {

void* ref_symbolic_run_p(int n, const int* csr_row_ptr, const int* csr_col_idx, int max_panel_width,
                         int parallel_nd, int float_front, int use_matching, int nd_depth, int nd_base_small,
                         int nd_base_large) {
  using namespace custom_linear_solver;
  using namespace custom_linear_solver::plan;
  namespace sym = custom_linear_solver::symbolic;
  auto* out = new RefSymbolic();
  auto& A = out->arrays;
  const int nnz = csr_row_ptr[n];

  // 1. CSR -> CSC (+ source_pos)
  std::vector<int> cp(n + 1, 0), ci(nnz), src(nnz);
  for (int k = 0; k < nnz; ++k) cp[csr_col_idx[k] + 1]++;
  for (int c = 0; c < n; ++c) cp[c + 1] += cp[c];
  {
    std::vector<int> cur(cp.begin(), cp.end());
    for (int r = 0; r < n; ++r)
      for (int k = csr_row_ptr[r]; k < csr_row_ptr[r + 1]; ++k) {
        const int q = cur[csr_col_idx[k]]++;
        ci[q] = r;
        src[q] = k;
      }
  }
  // 2. symmetric graph (A + A^T, no diagonal), sorted unique neighbours
  std::vector<unsigned long long> keys;
  keys.reserve(2 * (size_t)nnz);
  for (int c = 0; c < n; ++c)
    for (int q = cp[c]; q < cp[c + 1]; ++q) {
      const int r = ci[q];
      if (r == c) continue;
      keys.push_back((unsigned long long)r * n + c);
      keys.push_back((unsigned long long)c * n + r);
    }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  std::vector<int> xadj(n + 1, 0), adjncy(keys.size());
  for (size_t i = 0; i < keys.size(); ++i) {
    xadj[(int)(keys[i] / n) + 1]++;
    adjncy[i] = (int)(keys[i] % n);
  }
  for (int v = 0; v < n; ++v) xadj[v + 1] += xadj[v];
  A["graph_xadj"] = xadj;
  A["graph_adjncy"] = adjncy;

  std::vector<int> row_to_col;
  if (use_matching) {
    if (!StructuralMatchingFromCsc(n, cp, ci, row_to_col)) {
      delete out;
      return nullptr;
    }
    A["row_to_col"] = row_to_col;
  }

  // 3. METIS nested dissection (reference code, seed 42)
  std::vector<int> perm(n, 0);
  {
    std::vector<int> gx = xadj, ga = adjncy;
    if (!reordering::MetisNdFromGraph(n, gx, ga, perm, parallel_nd != 0, 42, nd_depth, nd_base_small,
                                      nd_base_large)) {
      delete out;
      return nullptr;
    }
  }
  std::vector<int> iperm(n), row_iperm(n);
  if (use_matching) {
    std::vector<int> col_perm(n);
    for (int k = 0; k < n; ++k) col_perm[k] = row_to_col[perm[k]];
    for (int k = 0; k < n; ++k) iperm[col_perm[k]] = k;
    A["col_perm"] = col_perm;
  } else {
    for (int k = 0; k < n; ++k) iperm[perm[k]] = k;
  }
  for (int k = 0; k < n; ++k) row_iperm[perm[k]] = k;
  A["perm"] = perm;
  A["iperm"] = iperm;
  A["row_iperm"] = row_iperm;

  // 4. permuted CSC (new column iperm[old], rows through row_iperm, order kept)
  std::vector<int> ocp(n + 1, 0), oci(nnz), osrc(nnz);
  for (int c = 0; c < n; ++c) ocp[iperm[c] + 1] = cp[c + 1] - cp[c];
  for (int c = 0; c < n; ++c) ocp[c + 1] += ocp[c];
  for (int c = 0; c < n; ++c) {
    const int nc = iperm[c];
    for (int off = 0; off < cp[c + 1] - cp[c]; ++off) {
      oci[ocp[nc] + off] = row_iperm[ci[cp[c] + off]];
      osrc[ocp[nc] + off] = src[cp[c] + off];
    }
  }

  // 5. symmetric pattern for Etree / fill: relabelled (reference static
  // helper), or with matching A' + A'^T of the permuted CSC, sorted unique
  std::vector<int> scp, sri;
  if (use_matching) {
    std::vector<unsigned long long> ok;
    ok.reserve(2 * (size_t)nnz);
    for (int c = 0; c < n; ++c)
      for (int q = ocp[c]; q < ocp[c + 1]; ++q) {
        const int r = oci[q];
        if (r == c) continue;
        ok.push_back((unsigned long long)r * n + c);
        ok.push_back((unsigned long long)c * n + r);
      }
    std::sort(ok.begin(), ok.end());
    ok.erase(std::unique(ok.begin(), ok.end()), ok.end());
    scp.assign(n + 1, 0);
    sri.resize(ok.size());
    for (size_t i = 0; i < ok.size(); ++i) {
      scp[(int)(ok[i] / n) + 1]++;
      sri[i] = (int)(ok[i] % n);
    }
    for (int v = 0; v < n; ++v) scp[v + 1] += scp[v];
  } else {
    PermuteSymmetricPattern(n, xadj, adjncy, perm, iperm, scp, sri);
  }
  A["sym_col_ptr"] = scp;
  A["sym_row_idx"] = sri;

  // 6-7. elimination tree and fill pattern (reference)
  std::vector<int> parent = sym::Etree(n, scp.data(), sri.data());
  std::vector<int> Lp, Li;
  sym::FillPattern(n, scp.data(), sri.data(), parent, Lp, Li);
  A["parent"] = parent;
  A["Lp"] = Lp;
  A["Li"] = Li;
  std::vector<int> Li_sorted = Li;
  for (int j = 0; j < n; ++j) std::sort(Li_sorted.begin() + Lp[j], Li_sorted.begin() + Lp[j + 1]);
  A["Li_sorted"] = Li_sorted;

  // 8. AnalyzeMultifrontal steps (lower.cu:584-635, reference helpers)
  std::vector<int> colcount(n);
  for (int j = 0; j < n; ++j) colcount[j] = Lp[j + 1] - Lp[j];
  const int eff = ComputeEffectivePanelWidth(n, max_panel_width, float_front != 0);
  const sym::PanelPartition panels = sym::RelaxedPanels(n, parent, colcount, eff);
  const sym::MultifrontalSymbolic sf = sym::ComputeMultifrontalSymbolic(n, Lp, Li, panels);
  const int P = panels.num_panels;
  A["panel_first"] = panels.first;
  A["panel_ncols"] = panels.ncols;
  A["panel_width"] = panels.width;
  A["panel_of"] = panels.panel_of;
  A["front_ptr"] = sf.front_ptr;
  A["front_rows"] = sf.front_rows;
  A["panel_parent"] = sf.panel_parent;
  A["asm_ptr"] = sf.asm_ptr;
  A["asm_idx"] = sf.asm_idx;

  MultifrontalPlan plan;
  plan.num_rows = n;
  plan.nnz = nnz;
  plan.num_panels = P;
  plan.h_front_ptr = sf.front_ptr;
  plan.h_ncols = panels.ncols;
  plan.h_panel_parent = sf.panel_parent;
  plan.h_asm_ptr = sf.asm_ptr;
  std::vector<int> plevel;
  const int num_plevels = BuildPanelLevels(plan, sf, P, plevel);
  std::vector<int> plcols(P);
  {
    std::vector<int> next(plan.panel_level_ptr.begin(), plan.panel_level_ptr.end());
    for (int p = 0; p < P; ++p) plcols[next[plevel[p]]++] = p;
  }
  plan.h_plcols = plcols;
  out->texts["fronts_csv_level"] = dump_fronts_text(plan);  // the analyze_fronts_only dump
  A["plevel"] = plevel;
  A["panel_level_ptr"] = plan.panel_level_ptr;
  A["plcols_level"] = plcols;
  std::vector<int> front_off;
  long total = 0;
  LayoutFrontArena(plan, sf, P, front_off, total);
  A["front_off"] = front_off;
  A["front_total"] = {(int)total};
  const bool fp64 = float_front == 0;
  PartitionSubtrees(plan, sf, plcols, P, num_plevels, fp64, false);
  A["plcols"] = plcols;
  A["spine_panels"] = plan.h_spine_panels;
  A["spine_start_level"] = {plan.spine_start_level};
  A["subtree_roots"] = plan.h_subtree_roots;
  A["subtree_of_panel"] = plan.h_subtree_of_panel;
  A["subtree_level_off"] = plan.h_subtree_level_off;
  A["subtree_level_cnt"] = plan.h_subtree_level_cnt;
  A["subtree_level_tier_off"] = plan.h_subtree_level_tier_off;
  BuildTierOrder(plan, sf, plcols, P, num_plevels, fp64);
  A["plcols_tier"] = plan.h_plcols_tier;
  A["level_tier_off"] = plan.h_level_tier_off;
  A["asm_local"] = BuildAssemblyMap(plan, sf, P);
  out->texts["fronts_csv_full"] = dump_fronts_text(plan);  // the full analysis's dump

  // a_pos (formula of BuildAPosDevice, lower.cu:35-62), reported in CSR order
  std::vector<int> a_pos_csr(nnz, -1);
  for (int j = 0; j < n; ++j)
    for (int q = ocp[j]; q < ocp[j + 1]; ++q) {
      const int i = oci[q];
      const int mn = std::min(i, j), mx = std::max(i, j);
      const int owner = panels.panel_of[mn];
      const int first = panels.first[owner];
      const int nc = panels.ncols[owner];
      const int fb = sf.front_ptr[owner], fe = sf.front_ptr[owner + 1];
      const int fsz = fe - fb;
      const int mn_l = mn - first;
      int mx_l;
      if (mx < first + nc) {
        mx_l = mx - first;
      } else {
        mx_l = (int)(std::lower_bound(sf.front_rows.begin() + fb, sf.front_rows.begin() + fe, mx) -
                     (sf.front_rows.begin() + fb));
      }
      const int ri = (i < j) ? mn_l : mx_l;
      const int cc = (i < j) ? mx_l : mn_l;
      a_pos_csr[osrc[q]] = front_off[owner] + ri * fsz + cc;
    }
  A["a_pos_csr"] = a_pos_csr;
  return out;
}

// SolverConfig defaults for the parallel-ND knobs (solver.hpp:44-46)
void* ref_symbolic_run_m(int n, const int* csr_row_ptr, const int* csr_col_idx, int max_panel_width,
                         int parallel_nd, int float_front, int use_matching) {
  return ref_symbolic_run_p(n, csr_row_ptr, csr_col_idx, max_panel_width, parallel_nd, float_front, use_matching, 4,
                            4000, 20000);
}

void* ref_symbolic_run(int n, const int* csr_row_ptr, const int* csr_col_idx, int max_panel_width,
                       int parallel_nd, int float_front) {
  return ref_symbolic_run_m(n, csr_row_ptr, csr_col_idx, max_panel_width, parallel_nd, float_front, 0);
}

int ref_symbolic_len(void* h, const char* name) {
  auto* s = static_cast<RefSymbolic*>(h);
  auto it = s->arrays.find(name);
  return it == s->arrays.end() ? -1 : (int)it->second.size();
}

int ref_symbolic_copy(void* h, const char* name, int* dst) {
  auto* s = static_cast<RefSymbolic*>(h);
  auto it = s->arrays.find(name);
  if (it == s->arrays.end()) return -1;
  if (!it->second.empty()) std::memcpy(dst, it->second.data(), sizeof(int) * it->second.size());
  return 0;
}

int ref_symbolic_names(void* h, char* buf, int cap) {
  auto* s = static_cast<RefSymbolic*>(h);
  std::string all;
  for (auto& kv : s->arrays) {
    all += kv.first;
    all += ',';
  }
  if ((int)all.size() + 1 > cap) return -1;
  std::memcpy(buf, all.c_str(), all.size() + 1);
  return 0;
}

// Text outputs ("fronts_csv_level", "fronts_csv_full"): returns the length,
// copying it (with a terminating NUL) when buf has room; -1 if unknown.
int ref_symbolic_text(void* h, const char* name, char* buf, int cap) {
  auto* s = static_cast<RefSymbolic*>(h);
  auto it = s->texts.find(name);
  if (it == s->texts.end()) return -1;
  const int len = (int)it->second.size();
  if (buf && cap > len) std::memcpy(buf, it->second.c_str(), (size_t)len + 1);
  return len;
}

void ref_symbolic_free(void* h) { delete static_cast<RefSymbolic*>(h); }

}  // extern "C"
