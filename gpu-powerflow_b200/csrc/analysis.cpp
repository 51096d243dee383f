// analysis.cpp -- Jacobian analysis and symbolic multifrontal plan (host).
//
// Each function restates one step of the reference's analysis; the file:line
// it follows is given at the function.  The arrays produced are compared
// element for element with the reference's own code in the test suite.
#include "analysis.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>

#include "metis_api.hpp"

namespace cupf_b200 {

// ===========================================================================
// Jacobian analysis (cuPF/cpp/src/newton_solver/ops/jacobian/jacobian_analysis.cpp)
// ===========================================================================

namespace {

// Slot of (row, col) in a row-sorted CSR pattern, -1 if absent
// (jacobian_analysis.cpp:143-174: linear scan or binary search, same result).
int32_t slot_of(const std::vector<int32_t>& rp, const std::vector<int32_t>& ci, int32_t dim, int32_t r,
                int32_t c) {
  if (r < 0 || c < 0 || r >= dim || c >= dim) return -1;
  auto b = ci.begin() + rp[r], e = ci.begin() + rp[r + 1];
  auto it = std::lower_bound(b, e, c);
  return (it != e && *it == c) ? static_cast<int32_t>(it - ci.begin()) : -1;
}

}  // namespace

JacobianAnalysis analyze_jacobian(int32_t n_bus, const int32_t* indptr, const int32_t* indices,
                                  const int32_t* pv, int32_t n_pv, const int32_t* pq, int32_t n_pq) {
  // Index tables (make_jacobian_indexing, jacobian_analysis.cpp:257-307): PV
  // buses own one angle row/column, PQ buses an angle and a magnitude one.
  if (n_bus <= 0 || n_pv < 0 || n_pq < 0 || n_pv + n_pq <= 0)
    throw std::invalid_argument("make_jacobian_indexing: invalid dimensions");
  if ((n_pv > 0 && !pv) || (n_pq > 0 && !pq)) throw std::invalid_argument("pv/pq must not be null");
  JacobianAnalysis ja;
  ja.n_bus = n_bus;
  ja.n_pv = n_pv;
  ja.n_pq = n_pq;
  ja.n_pvpq = n_pv + n_pq;
  ja.dim = ja.n_pvpq + n_pq;
  ja.row_pvpq.assign(n_bus, -1);
  ja.row_pq.assign(n_bus, -1);
  for (int32_t i = 0; i < n_pv; ++i) {
    if (pv[i] < 0 || pv[i] >= n_bus) throw std::invalid_argument("make_jacobian_indexing: pv bus index out of range");
    ja.row_pvpq[pv[i]] = i;
  }
  for (int32_t i = 0; i < n_pq; ++i) {
    if (pq[i] < 0 || pq[i] >= n_bus) throw std::invalid_argument("make_jacobian_indexing: pq bus index out of range");
    ja.row_pvpq[pq[i]] = n_pv + i;
    ja.row_pq[pq[i]] = ja.n_pvpq + i;
  }

  // Pattern (JacobianPatternGenerator::generate, jacobian_analysis.cpp:310-386):
  // every Ybus coupling of buses (a, b) puts the angle/magnitude columns of b
  // into the angle/magnitude rows of a; Ybus is walked as its strict upper
  // triangle mirrored plus the diagonal, then each row is sorted and deduped.
  std::vector<std::vector<int32_t>> rows(ja.dim);
  auto couple = [&](int32_t a, int32_t b) {
    const int32_t ra = ja.row_pvpq[a], qa = ja.row_pq[a];
    const int32_t cb = ja.row_pvpq[b], qb = ja.row_pq[b];
    if (ra >= 0 && cb >= 0) rows[ra].push_back(cb);
    if (qa >= 0 && cb >= 0) rows[qa].push_back(cb);
    if (ra >= 0 && qb >= 0) rows[ra].push_back(qb);
    if (qa >= 0 && qb >= 0) rows[qa].push_back(qb);
  };
  for (int32_t r = 0; r < n_bus; ++r) {
    for (int32_t k = indptr[r]; k < indptr[r + 1]; ++k) {
      const int32_t c = indices[k];
      if (c < 0 || c >= n_bus) throw std::invalid_argument("Ybus column index out of range");
      if (c > r) {
        couple(r, c);
        couple(c, r);
      }
    }
  }
  for (int32_t b = 0; b < n_bus; ++b) couple(b, b);
  ja.row_ptr.assign(ja.dim + 1, 0);
  for (int32_t r = 0; r < ja.dim; ++r) {
    auto& v = rows[r];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    ja.row_ptr[r + 1] = ja.row_ptr[r] + static_cast<int32_t>(v.size());
  }
  ja.nnz = ja.row_ptr[ja.dim];
  ja.col_idx.reserve(ja.nnz);
  for (auto& v : rows) ja.col_idx.insert(ja.col_idx.end(), v.begin(), v.end());

  // Scatter maps (JacobianMapBuilder::build, jacobian_analysis.cpp:389-445).
  const int32_t nnz_y = indptr[n_bus];
  ja.map11.assign(nnz_y, -1);
  ja.map21.assign(nnz_y, -1);
  ja.map12.assign(nnz_y, -1);
  ja.map22.assign(nnz_y, -1);
  ja.diag11.assign(n_bus, -1);
  ja.diag21.assign(n_bus, -1);
  ja.diag12.assign(n_bus, -1);
  ja.diag22.assign(n_bus, -1);
  std::vector<int32_t> hits(ja.nnz, 0);
  for (int32_t r = 0; r < n_bus; ++r) {
    for (int32_t k = indptr[r]; k < indptr[r + 1]; ++k) {
      const int32_t c = indices[k];
      const int32_t ra = ja.row_pvpq[r], qa = ja.row_pq[r];
      const int32_t cb = ja.row_pvpq[c], qb = ja.row_pq[c];
      ja.map11[k] = (ra >= 0 && cb >= 0) ? slot_of(ja.row_ptr, ja.col_idx, ja.dim, ra, cb) : -1;
      ja.map21[k] = (qa >= 0 && cb >= 0) ? slot_of(ja.row_ptr, ja.col_idx, ja.dim, qa, cb) : -1;
      ja.map12[k] = (ra >= 0 && qb >= 0) ? slot_of(ja.row_ptr, ja.col_idx, ja.dim, ra, qb) : -1;
      ja.map22[k] = (qa >= 0 && qb >= 0) ? slot_of(ja.row_ptr, ja.col_idx, ja.dim, qa, qb) : -1;
      for (int32_t s : {ja.map11[k], ja.map21[k], ja.map12[k], ja.map22[k]})
        if (s >= 0) hits[s]++;
      if (r == c) {
        ja.diag11[r] = ja.map11[k];
        ja.diag21[r] = ja.map21[k];
        ja.diag12[r] = ja.map12[k];
        ja.diag22[r] = ja.map22[k];
      }
    }
  }
  ja.every_slot_mapped = std::all_of(hits.begin(), hits.end(), [](int32_t h) { return h == 1; });
  return ja;
}

// ===========================================================================
// Nested-dissection ordering (custom_linear_solver/src/analyze/reorder/metis_nd.cpp)
// ===========================================================================

namespace {

using Graph = std::pair<std::vector<idx_t>, std::vector<idx_t>>;  // (xadj, adjncy)

// METIS keeps its random-number state in globals: two engines analysing at the
// same time from different threads would race and could get different
// orderings, so every METIS call holds this lock.
std::mutex g_metis_mutex;

void metis_options(idx_t* opt, int seed) {
  METIS_SetDefaultOptions(opt);
  opt[METIS_OPTION_NUMBERING] = 0;
  opt[METIS_OPTION_SEED] = seed;
}

// Leaf of the recursion: one METIS_NodeND call, natural order for trivial or
// edgeless graphs and on failure (metis_nd.cpp:71-103).
std::vector<int32_t> nodend(const Graph& g, int seed) {
  const int32_t n = static_cast<int32_t>(g.first.size()) - 1;
  std::vector<int32_t> perm(std::max(n, 0));
  std::iota(perm.begin(), perm.end(), 0);
  if (n <= 1 || g.second.empty()) return perm;
  idx_t nv = n;
  idx_t opt[METIS_NOPTIONS];
  metis_options(opt, seed);
  std::vector<idx_t> xa(g.first), ad(g.second), p(n), ip(n);
  int st;
  {
    std::lock_guard<std::mutex> lock(g_metis_mutex);
    st = METIS_NodeND(&nv, xa.data(), ad.data(), nullptr, opt, p.data(), ip.data());
  }
  if (st != METIS_OK) return perm;
  for (int32_t i = 0; i < n; ++i) perm[i] = static_cast<int32_t>(p[i]);
  return perm;
}

// Sub-graph on the vertices with part[v] == which, vertices in ascending
// order, only edges inside the part kept (metis_nd.cpp:27-61).
Graph induced(const Graph& g, const std::vector<idx_t>& part, idx_t which, std::vector<int32_t>& map) {
  const int32_t n = static_cast<int32_t>(g.first.size()) - 1;
  std::vector<int32_t> g2l(n, -1);
  map.clear();
  for (int32_t v = 0; v < n; ++v)
    if (part[v] == which) {
      g2l[v] = static_cast<int32_t>(map.size());
      map.push_back(v);
    }
  Graph s;
  s.first.assign(map.size() + 1, 0);
  for (size_t l = 0; l < map.size(); ++l) {
    const int32_t v = map[l];
    for (idx_t p = g.first[v]; p < g.first[v + 1]; ++p)
      if (part[g.second[p]] == which) s.second.push_back(g2l[g.second[p]]);
    s.first[l + 1] = static_cast<idx_t>(s.second.size());
  }
  return s;
}

// Separator recursion (metis_nd.cpp:110-172): order part 0, then part 1, then
// the separator.  Each METIS call reseeds from its options, so running the two
// halves one after the other gives the ordering a thread-safe parallel run does.
std::vector<int32_t> nd_recurse(const Graph& g, int depth, int base_thr, int seed) {
  const int32_t n = static_cast<int32_t>(g.first.size()) - 1;
  if (depth <= 0 || n < base_thr || g.second.empty()) return nodend(g, seed);
  idx_t nv = n, sep = 0;
  std::vector<idx_t> part(n);
  idx_t opt[METIS_NOPTIONS];
  metis_options(opt, seed);
  std::vector<idx_t> xa(g.first), ad(g.second);
  int st;
  {
    std::lock_guard<std::mutex> lock(g_metis_mutex);
    st = METIS_ComputeVertexSeparator(&nv, xa.data(), ad.data(), nullptr, opt, &sep, part.data());
  }
  if (st != METIS_OK) return nodend(g, seed);
  std::vector<int32_t> m0, m1;
  const Graph g0 = induced(g, part, 0, m0);
  const Graph g1 = induced(g, part, 1, m1);
  if (m0.empty() || m1.empty()) return nodend(g, seed);
  const std::vector<int32_t> p0 = nd_recurse(g0, depth - 1, base_thr, seed);
  const std::vector<int32_t> p1 = nd_recurse(g1, depth - 1, base_thr, seed);
  std::vector<int32_t> perm;
  perm.reserve(n);
  for (int32_t i : p0) perm.push_back(m0[i]);
  for (int32_t i : p1) perm.push_back(m1[i]);
  for (int32_t v = 0; v < n; ++v)
    if (part[v] == 2) perm.push_back(v);
  return perm;
}

// RunNdOnGraph (metis_nd.cpp:241-278) with the reference's parallel-ND knobs
// (recursion depth; base-case size base_small below 20,000 vertices, else
// base_large; defaults 4, 4000, 20000).
std::vector<int32_t> nd_order(const std::vector<int32_t>& xadj, const std::vector<int32_t>& adjncy, int n,
                              bool serial, int seed, int depth, int base_small, int base_large) {
  std::vector<int32_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  if (n <= 1 || adjncy.empty()) return perm;
  Graph g{std::vector<idx_t>(xadj.begin(), xadj.end()), std::vector<idx_t>(adjncy.begin(), adjncy.end())};
  if (!serial) {
    const int base_thr = n < 20000 ? base_small : base_large;
    return nd_recurse(g, depth, base_thr, seed);
  }
  return nodend(g, seed);
}

// Perfect structural matching row -> column by Hopcroft-Karp, in the search
// order of StructuralMatchingFromCsc (analyze/pipeline.cpp:77-160): rows keep
// their columns in ascending order; each phase runs a BFS from all unmatched
// rows, then a depth-first augmentation from every unmatched row in row
// order, trying its columns in order and restarting at the first column on
// every call.  The depth-first search runs on an explicit stack (paths may be
// as long as n).  Returns false when no perfect matching exists.
bool structural_matching(int32_t n, const int32_t* row_ptr, const int32_t* col_idx, std::vector<int32_t>& row_to_col) {
  // row -> columns ascending (the CSR may hold them in any order)
  std::vector<int32_t> rp(n + 1, 0), adj;
  {
    std::vector<std::vector<int32_t>> rows(n);
    for (int32_t r = 0; r < n; ++r)
      for (int32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k)
        if (col_idx[k] >= 0 && col_idx[k] < n) rows[r].push_back(col_idx[k]);
    for (int32_t r = 0; r < n; ++r) {
      std::sort(rows[r].begin(), rows[r].end());
      rp[r + 1] = rp[r] + static_cast<int32_t>(rows[r].size());
      adj.insert(adj.end(), rows[r].begin(), rows[r].end());
    }
  }
  for (int32_t r = 0; r < n; ++r)
    if (rp[r + 1] == rp[r]) return false;
  row_to_col.assign(n, -1);
  std::vector<int32_t> col_to_row(n, -1), dist(n, -1), q;
  q.reserve(n);
  auto bfs = [&]() {
    q.clear();
    bool found = false;
    for (int32_t r = 0; r < n; ++r) {
      if (row_to_col[r] < 0) {
        dist[r] = 0;
        q.push_back(r);
      } else {
        dist[r] = -1;
      }
    }
    for (size_t h = 0; h < q.size(); ++h) {
      const int32_t r = q[h];
      for (int32_t p = rp[r]; p < rp[r + 1]; ++p) {
        const int32_t rr = col_to_row[adj[p]];
        if (rr < 0) {
          found = true;
        } else if (dist[rr] < 0) {
          dist[rr] = dist[r] + 1;
          q.push_back(rr);
        }
      }
    }
    return found;
  };
  struct Frame {
    int32_t r, p;
  };
  std::vector<Frame> st;
  auto augment = [&](int32_t r0) {
    st.clear();
    st.push_back({r0, rp[r0]});
    while (!st.empty()) {
      Frame& f = st.back();
      if (f.p == rp[f.r + 1]) {  // every column tried: this row is a dead end
        dist[f.r] = -1;
        st.pop_back();
        if (!st.empty()) ++st.back().p;
        continue;
      }
      const int32_t c = adj[f.p];
      const int32_t rr = col_to_row[c];
      if (rr < 0) {  // free column: flip the path
        for (size_t k = st.size(); k-- > 0;) {
          const int32_t cc = adj[st[k].p];
          row_to_col[st[k].r] = cc;
          col_to_row[cc] = st[k].r;
        }
        return true;
      }
      if (dist[rr] == dist[f.r] + 1)
        st.push_back({rr, rp[rr]});
      else
        ++f.p;
    }
    return false;
  };
  int32_t matched = 0;
  while (bfs())
    for (int32_t r = 0; r < n; ++r)
      if (row_to_col[r] < 0 && augment(r)) ++matched;
  return matched == n;
}

}  // namespace

// ===========================================================================
// Symbolic plan
// ===========================================================================

std::string fronts_csv(const SymbolicPlan& sp) {
  std::string out = "q,p,fsz,nc,uc,level,parent,asm_len,extend_elems\n";
  char line[160];
  for (int32_t L = 0; L + 1 < (int32_t)sp.level_ptr.size(); ++L)
    for (int32_t q = sp.level_ptr[L]; q < sp.level_ptr[L + 1]; ++q) {
      const int32_t p = sp.plcols_level[q];
      const int32_t fsz = sp.front_ptr[p + 1] - sp.front_ptr[p];
      const int32_t nc = sp.panel_ncols[p];
      const int32_t uc = fsz - nc;
      const int32_t parent = sp.panel_parent.empty() ? -1 : sp.panel_parent[p];
      const int32_t asm_len = sp.asm_ptr.empty() ? 0 : sp.asm_ptr[p + 1] - sp.asm_ptr[p];
      const long long extend = parent >= 0 ? (long long)uc * uc : 0;
      std::snprintf(line, sizeof line, "%d,%d,%d,%d,%d,%d,%d,%d,%lld\n", q, p, fsz, nc, uc, L, parent, asm_len,
                    extend);
      out += line;
    }
  return out;
}

SymbolicPlan analyze_symbolic(int32_t n, const int32_t* row_ptr, const int32_t* col_idx, const SymbolicOptions& opt) {
  if (n <= 0) throw std::invalid_argument("analyze_symbolic: empty matrix");
  SymbolicPlan sp;
  sp.n = n;
  sp.nnz = row_ptr[n];

  // A + A^T without the diagonal, neighbours ascending: the METIS input of
  // BuildSymmetricGraphDevice (analyze/pattern/pattern_kernels.cu:171-252).
  {
    std::vector<std::vector<int32_t>> adj(n);
    for (int32_t r = 0; r < n; ++r)
      for (int32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
        const int32_t c = col_idx[k];
        if (c < 0 || c >= n) throw std::invalid_argument("analyze_symbolic: column index out of range");
        if (c == r) continue;
        adj[r].push_back(c);
        adj[c].push_back(r);
      }
    sp.graph_xadj.assign(n + 1, 0);
    for (int32_t v = 0; v < n; ++v) {
      auto& a = adj[v];
      std::sort(a.begin(), a.end());
      a.erase(std::unique(a.begin(), a.end()), a.end());
      sp.graph_xadj[v + 1] = sp.graph_xadj[v] + static_cast<int32_t>(a.size());
      sp.graph_adjncy.insert(sp.graph_adjncy.end(), a.begin(), a.end());
    }
  }

  // Optional structural matching, computed before the ordering as the
  // reference does (pipeline.cpp:222-233).
  if (opt.use_matching && !structural_matching(n, row_ptr, col_idx, sp.row_to_col))
    throw std::runtime_error("analyze_symbolic: structural matching requested but no perfect matching exists");

  // Ordering (pipeline.cpp:236-258).  perm orders the rows; the columns
  // follow the rows, or with a matching the matched column of each row:
  // col_perm[k] = row_to_col[perm[k]], iperm = col_perm^-1.
  sp.perm = nd_order(sp.graph_xadj, sp.graph_adjncy, n, opt.serial_nd, opt.metis_seed, opt.par_nd_depth,
                     opt.par_nd_base_small, opt.par_nd_base_large);
  sp.row_iperm.assign(n, 0);
  for (int32_t k = 0; k < n; ++k) sp.row_iperm[sp.perm[k]] = k;
  if (opt.use_matching) {
    sp.col_perm.assign(n, 0);
    for (int32_t k = 0; k < n; ++k) sp.col_perm[k] = sp.row_to_col[sp.perm[k]];
    sp.iperm.assign(n, 0);
    for (int32_t k = 0; k < n; ++k) sp.iperm[sp.col_perm[k]] = k;
  } else {
    sp.col_perm = sp.perm;
    sp.iperm = sp.row_iperm;
  }

  if (opt.use_matching) {
    // The permuted matrix is no longer structurally symmetric: its A + A^T
    // graph is built afresh, neighbours ascending (pipeline.cpp:265-272 with
    // BuildSymmetricGraphDevice on the ordered pattern).
    std::vector<std::vector<int32_t>> adj(n);
    for (int32_t r = 0; r < n; ++r)
      for (int32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
        const int32_t i = sp.row_iperm[r], j = sp.iperm[col_idx[k]];
        if (i == j) continue;
        adj[i].push_back(j);
        adj[j].push_back(i);
      }
    sp.sym_col_ptr.assign(n + 1, 0);
    for (int32_t v = 0; v < n; ++v) {
      auto& a = adj[v];
      std::sort(a.begin(), a.end());
      a.erase(std::unique(a.begin(), a.end()), a.end());
      sp.sym_col_ptr[v + 1] = sp.sym_col_ptr[v] + static_cast<int32_t>(a.size());
      sp.sym_row_idx.insert(sp.sym_row_idx.end(), a.begin(), a.end());
    }
  } else {
    // Relabelled graph: new column k holds old column perm[k], rows through
    // iperm, in the old adjacency order (PermuteSymmetricPattern, pipeline.cpp:47-72).
    sp.sym_col_ptr.assign(n + 1, 0);
    for (int32_t k = 0; k < n; ++k) {
      const int32_t o = sp.perm[k];
      sp.sym_col_ptr[k + 1] = sp.sym_col_ptr[k] + (sp.graph_xadj[o + 1] - sp.graph_xadj[o]);
    }
    sp.sym_row_idx.resize(sp.sym_col_ptr[n]);
    for (int32_t k = 0; k < n; ++k) {
      const int32_t o = sp.perm[k];
      int32_t w = sp.sym_col_ptr[k];
      for (int32_t p = sp.graph_xadj[o]; p < sp.graph_xadj[o + 1]; ++p)
        sp.sym_row_idx[w++] = sp.iperm[sp.graph_adjncy[p]];
    }
  }

  // Elimination tree with path compression (symbolic/elimination_tree.cpp:67-88).
  const auto& scp = sp.sym_col_ptr;
  const auto& sri = sp.sym_row_idx;
  sp.parent.assign(n, -1);
  {
    std::vector<int32_t> anc(n, -1);
    for (int32_t k = 0; k < n; ++k)
      for (int32_t p = scp[k]; p < scp[k + 1]; ++p) {
        int32_t i = sri[p];
        while (i != -1 && i < k) {
          const int32_t up = anc[i];
          anc[i] = k;
          if (up == -1) sp.parent[i] = k;
          i = up;
        }
      }
  }

  // Fill of L (symbolic Cholesky by column merge, elimination_tree.cpp:365-434):
  // struct(j) = {j} u {i > j adjacent to j} u (struct(child) \ {child}).
  {
    std::vector<std::vector<int32_t>> kids(n);
    for (int32_t j = 0; j < n; ++j)
      if (sp.parent[j] >= 0) kids[sp.parent[j]].push_back(j);
    std::vector<std::vector<int32_t>> cols(n);
    std::vector<int32_t> mark(n, -1);
    for (int32_t j = 0; j < n; ++j) {
      auto& s = cols[j];
      mark[j] = j;
      s.push_back(j);
      for (int32_t p = scp[j]; p < scp[j + 1]; ++p) {
        const int32_t i = sri[p];
        if (i > j && mark[i] != j) {
          mark[i] = j;
          s.push_back(i);
        }
      }
      for (int32_t c : kids[j])
        for (int32_t i : cols[c])
          if (i != c && mark[i] != j) {
            mark[i] = j;
            s.push_back(i);
          }
      std::sort(s.begin(), s.end());
    }
    sp.Lp.assign(n + 1, 0);
    for (int32_t j = 0; j < n; ++j) sp.Lp[j + 1] = sp.Lp[j] + static_cast<int32_t>(cols[j].size());
    sp.Li.reserve(sp.Lp[n]);
    for (auto& c : cols) sp.Li.insert(sp.Li.end(), c.begin(), c.end());
  }

  // Relaxed panels: greedy merge along single-child chains j -> j + 1 up to
  // cap columns (symbolic/supernode.cpp:104-141; cap clamp lower.cu:123-131).
  {
    const int cap = std::min(64, std::max(1, opt.max_panel_width));
    sp.panel_of.assign(n, -1);
    for (int32_t j = 0; j < n;) {
      const int32_t start = j;
      int32_t sz = 1, w = sp.Lp[j + 1] - sp.Lp[j];
      while (j + 1 < n && sz < cap && sp.parent[j] == j + 1) {
        ++j;
        ++sz;
        w = std::max(w, sp.Lp[j + 1] - sp.Lp[j]);
      }
      const int32_t id = sp.num_panels++;
      sp.panel_first.push_back(start);
      sp.panel_ncols.push_back(sz);
      sp.panel_width.push_back(w);
      for (int32_t c = start; c <= j; ++c) sp.panel_of[c] = id;
      ++j;
    }
  }
  const int32_t P = sp.num_panels;

  // Fronts: sorted union of the member columns' structures; the pivots come
  // first, the contribution-block rows follow (symbolic/multifrontal.cpp:224-320).
  {
    sp.front_ptr.assign(P + 1, 0);
    std::vector<int32_t> mark(n, -1);
    std::vector<int32_t> rows;
    for (int32_t p = 0; p < P; ++p) {
      rows.clear();
      const int32_t f = sp.panel_first[p], l = f + sp.panel_ncols[p];
      for (int32_t j = f; j < l; ++j)
        for (int32_t q = sp.Lp[j]; q < sp.Lp[j + 1]; ++q) {
          const int32_t i = sp.Li[q];
          if (mark[i] != p) {
            mark[i] = p;
            rows.push_back(i);
          }
        }
      std::sort(rows.begin(), rows.end());
      sp.front_rows.insert(sp.front_rows.end(), rows.begin(), rows.end());
      sp.front_ptr[p + 1] = static_cast<int32_t>(sp.front_rows.size());
    }
    sp.panel_parent.assign(P, -1);
    sp.asm_ptr.assign(P + 1, 0);
    for (int32_t p = 0; p < P; ++p) {
      const int32_t s = sp.front_ptr[p], nc = sp.panel_ncols[p];
      const int32_t fsz = sp.front_ptr[p + 1] - s;
      if (fsz > nc) sp.panel_parent[p] = sp.panel_of[sp.front_rows[s + nc]];
      sp.asm_ptr[p + 1] = sp.asm_ptr[p] + (fsz - nc);
    }
    sp.asm_idx.assign(sp.asm_ptr[P], -1);
    for (int32_t p = 0; p < P; ++p) {
      const int32_t par = sp.panel_parent[p];
      if (par < 0) continue;
      const int32_t ps = sp.front_ptr[par], pe = sp.front_ptr[par + 1];
      const int32_t pf = sp.panel_first[par], pl = pf + sp.panel_ncols[par];
      int32_t a = sp.asm_ptr[p];
      for (int32_t k = sp.front_ptr[p] + sp.panel_ncols[p]; k < sp.front_ptr[p + 1]; ++k, ++a) {
        const int32_t r = sp.front_rows[k];
        if (r >= pf && r < pl) {
          sp.asm_idx[a] = ps + (r - pf);
        } else {
          auto b = sp.front_rows.begin() + ps, e = sp.front_rows.begin() + pe;
          auto it = std::lower_bound(b, e, r);
          if (it != e && *it == r) sp.asm_idx[a] = static_cast<int32_t>(it - sp.front_rows.begin());
        }
      }
    }
    // parent-local extend-add positions (BuildAssemblyMap, lower.cu:450-463)
    sp.asm_local.assign(sp.asm_idx.size(), 0);
    for (int32_t p = 0; p < P; ++p) {
      const int32_t par = sp.panel_parent[p];
      const int32_t base = par >= 0 ? sp.front_ptr[par] : 0;
      for (int32_t a = sp.asm_ptr[p]; a < sp.asm_ptr[p + 1]; ++a) sp.asm_local[a] = sp.asm_idx[a] - base;
    }
  }

  // Levels: a panel sits one above its highest child; panel ids grow towards
  // the root so one forward pass suffices (BuildPanelLevels, lower.cu:176-197).
  sp.plevel.assign(P, 0);
  for (int32_t p = 0; p < P; ++p) {
    const int32_t par = sp.panel_parent[p];
    if (par >= 0) sp.plevel[par] = std::max(sp.plevel[par], sp.plevel[p] + 1);
  }
  for (int32_t p = 0; p < P; ++p) sp.num_levels = std::max(sp.num_levels, sp.plevel[p] + 1);
  sp.level_ptr.assign(sp.num_levels + 1, 0);
  for (int32_t p = 0; p < P; ++p) sp.level_ptr[sp.plevel[p] + 1]++;
  for (int32_t L = 0; L < sp.num_levels; ++L) sp.level_ptr[L + 1] += sp.level_ptr[L];
  sp.plcols_level.assign(P, 0);
  {
    std::vector<int32_t> next(sp.level_ptr.begin(), sp.level_ptr.end() - 1);
    for (int32_t p = 0; p < P; ++p) sp.plcols_level[next[sp.plevel[p]]++] = p;
  }

  // Dense front layout: offsets are the prefix sum of fsz^2 in panel order
  // (LayoutFrontArena, lower.cu:137-157).
  sp.front_off.assign(P + 1, 0);
  int64_t total = 0;
  for (int32_t p = 0; p < P; ++p) {
    const int64_t fsz = sp.front_ptr[p + 1] - sp.front_ptr[p];
    sp.front_off[p] = static_cast<int32_t>(total);
    total += fsz * fsz;
    if (total > (int64_t(1) << 30)) throw std::runtime_error("analyze_symbolic: front arena exceeds 2^30 elements");
  }
  sp.front_off[P] = static_cast<int32_t>(total);
  sp.front_total = total;

  // Entry positions: entry (i, j) of P_r A P_c^T belongs to the panel of min(i, j);
  // inside the front its row and column are the local indices of i and j
  // (BuildAPosDevice, lower.cu:35-62), reported per CSR entry.
  sp.a_pos_csr.assign(sp.nnz, -1);
  sp.a_owner.assign(sp.nnz, -1);
  sp.a_row.assign(sp.nnz, -1);
  sp.a_col.assign(sp.nnz, -1);
  for (int32_t r = 0; r < n; ++r)
    for (int32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
      const int32_t i = sp.row_iperm[r], j = sp.iperm[col_idx[k]];
      const int32_t mn = std::min(i, j), mx = std::max(i, j);
      const int32_t owner = sp.panel_of[mn];
      const int32_t first = sp.panel_first[owner], nc = sp.panel_ncols[owner];
      const int32_t fb = sp.front_ptr[owner], fe = sp.front_ptr[owner + 1];
      const int32_t fsz = fe - fb;
      const int32_t mn_l = mn - first;
      const int32_t mx_l = (mx < first + nc)
                               ? (mx - first)
                               : static_cast<int32_t>(std::lower_bound(sp.front_rows.begin() + fb,
                                                                       sp.front_rows.begin() + fe, mx) -
                                                      (sp.front_rows.begin() + fb));
      const int32_t ri = (i < j) ? mn_l : mx_l;
      const int32_t cc = (i < j) ? mx_l : mn_l;
      sp.a_owner[k] = owner;
      sp.a_row[k] = ri;
      sp.a_col[k] = cc;
      sp.a_pos_csr[k] = sp.front_off[owner] + ri * fsz + cc;
    }
  return sp;
}

// ===========================================================================
// Engine factor program
// ===========================================================================

FactorProgram build_factor_program(const SymbolicPlan& sp) {
  FactorProgram fp;
  const int32_t P = sp.num_panels;
  fp.P = P;
  fp.dim = sp.n;
  fp.nnz = sp.nnz;
  fp.num_levels = sp.num_levels;
  fp.front_ptr = sp.front_ptr;
  fp.front_rows = sp.front_rows;
  fp.asm_local = sp.asm_local;
  fp.asm_ptr = sp.asm_ptr;
  fp.perm = sp.perm;
  fp.iperm = sp.iperm;
  fp.row_iperm = sp.row_iperm;
  fp.col_perm = sp.col_perm;
  fp.parent_panel = sp.panel_parent;
  fp.fsz.resize(P);
  fp.nc.resize(P);
  fp.first = sp.panel_first;
  fp.u_off.assign(P + 1, 0);
  fp.l_off.assign(P + 1, 0);
  fp.cb_off.assign(P + 1, 0);
  fp.nchildren.assign(P, 0);
  for (int32_t p = 0; p < P; ++p) {
    const int32_t fsz = sp.front_ptr[p + 1] - sp.front_ptr[p];
    const int32_t nc = sp.panel_ncols[p];
    const int32_t uc = fsz - nc;
    fp.fsz[p] = fsz;
    fp.nc[p] = nc;
    fp.max_fsz = std::max(fp.max_fsz, fsz);
    fp.max_nc = std::max(fp.max_nc, nc);
    fp.u_off[p + 1] = fp.u_off[p] + int64_t(nc) * fsz;
    fp.l_off[p + 1] = fp.l_off[p] + int64_t(uc) * nc;
    fp.cb_off[p + 1] = fp.cb_off[p] + int64_t(uc) * (uc + 1);
    if (sp.panel_parent[p] >= 0) fp.nchildren[sp.panel_parent[p]]++;
  }
  fp.u_total = fp.u_off[P];
  fp.l_total = fp.l_off[P];
  fp.cb_total = fp.cb_off[P];

  const int32_t nrows = sp.front_ptr[P];
  // A sources per front row, from the entry positions (owner, r, c)
  {
    std::vector<std::vector<std::pair<int32_t, int32_t>>> lists(nrows);
    for (int32_t q = 0; q < sp.nnz; ++q) {
      const int32_t fr = sp.front_ptr[sp.a_owner[q]] + sp.a_row[q];
      lists[fr].push_back({sp.a_col[q], q});
    }
    fp.arow_ptr.assign(nrows + 1, 0);
    for (int32_t fr = 0; fr < nrows; ++fr) {
      auto& l = lists[fr];
      std::sort(l.begin(), l.end());
      for (auto& e : l) {
        fp.arow_col.push_back(e.first);
        fp.arow_q.push_back(e.second);
      }
      fp.arow_ptr[fr + 1] = static_cast<int32_t>(fp.arow_q.size());
    }
  }
  // CB sources per front row: child c's CB row r lands on parent row asm_local
  {
    std::vector<std::vector<std::pair<int32_t, int32_t>>> lists(nrows);
    for (int32_t c = 0; c < P; ++c) {
      const int32_t par = sp.panel_parent[c];
      if (par < 0) continue;
      for (int32_t a = sp.asm_ptr[c]; a < sp.asm_ptr[c + 1]; ++a) {
        const int32_t pos = sp.asm_local[a];
        if (pos < 0) throw std::runtime_error("build_factor_program: extend-add row missing in parent front");
        lists[sp.front_ptr[par] + pos].push_back({c, a - sp.asm_ptr[c]});
      }
    }
    fp.crow_ptr.assign(nrows + 1, 0);
    for (int32_t fr = 0; fr < nrows; ++fr) {
      for (auto& e : lists[fr]) {
        fp.crow_child.push_back(e.first);
        fp.crow_r.push_back(e.second);
      }
      fp.crow_ptr[fr + 1] = static_cast<int32_t>(fp.crow_child.size());
    }
  }
  // Dense-front assembly entries (sorted by destination) and warp chunks.
  {
    fp.fe_ptr.assign(P + 1, 0);
    fp.fe_split.assign((size_t)P * (kFeChunks + 1), 0);
    std::vector<std::vector<int32_t>> owned(P);
    for (int32_t q = 0; q < sp.nnz; ++q) owned[sp.a_owner[q]].push_back(q);
    std::vector<std::vector<int32_t>> kids(P);
    for (int32_t c = 0; c < P; ++c)
      if (sp.panel_parent[c] >= 0) kids[sp.panel_parent[c]].push_back(c);
    struct Ent {
      int32_t dst;
      int64_t src;
    };
    std::vector<Ent> ents;
    for (int32_t p = 0; p < P; ++p) {
      ents.clear();
      const int32_t fs = fp.fsz[p], nc = fp.nc[p], rw = fs + 1;
      for (int32_t q : owned[p]) ents.push_back({sp.a_row[q] * rw + sp.a_col[q], (int64_t)q});
      for (int32_t i = 0; i < nc; ++i)
        ents.push_back({i * rw + fs, (int64_t(2) << kFeKindShift) | (int64_t)(sp.panel_first[p] + i)});
      for (int32_t c : kids[p]) {
        const int32_t ucc = fp.fsz[c] - fp.nc[c];
        const int32_t* al = sp.asm_local.data() + sp.asm_ptr[c];
        for (int32_t r = 0; r < ucc; ++r)
          for (int32_t cc = 0; cc <= ucc; ++cc) {
            const int32_t col = cc < ucc ? al[cc] : fs;
            const int64_t idx = fp.cb_off[c] + (int64_t)r * (ucc + 1) + cc;
            ents.push_back({al[r] * rw + col, (int64_t(1) << kFeKindShift) | idx});
          }
      }
      std::stable_sort(ents.begin(), ents.end(), [](const Ent& a, const Ent& b) { return a.dst < b.dst; });
      const int64_t base = (int64_t)fp.fe_dst.size();
      for (const Ent& e : ents) {
        fp.fe_dst.push_back(e.dst);
        fp.fe_src.push_back(e.src);
      }
      fp.fe_ptr[p + 1] = (int64_t)fp.fe_dst.size();
      // chunk cuts at destination boundaries, about equal entry counts
      const int64_t n = (int64_t)ents.size();
      int64_t* split = fp.fe_split.data() + (size_t)p * (kFeChunks + 1);
      split[0] = base;
      for (int w = 1; w < kFeChunks; ++w) {
        int64_t cut = std::max<int64_t>(split[w - 1] - base, n * w / kFeChunks);
        while (cut > 0 && cut < n && ents[cut].dst == ents[cut - 1].dst) ++cut;
        split[w] = base + std::min(cut, n);
      }
      split[kFeChunks] = base + n;
    }
  }
  // Level work lists, fronts ordered by size inside a level so that warps of
  // one block tend to take the same code path.
  fp.level_ptr = sp.level_ptr;
  fp.level_fronts = sp.plcols_level;
  fp.level_max_fsz.assign(sp.num_levels, 0);
  for (int32_t L = 0; L < sp.num_levels; ++L) {
    auto b = fp.level_fronts.begin() + sp.level_ptr[L], e = fp.level_fronts.begin() + sp.level_ptr[L + 1];
    std::stable_sort(b, e, [&](int32_t a, int32_t c) { return fp.fsz[a] < fp.fsz[c]; });
    for (auto it = b; it != e; ++it) fp.level_max_fsz[L] = std::max(fp.level_max_fsz[L], fp.fsz[*it]);
  }
  // Per-front launch records in level order (24 int32 each, one
  // 96-byte line per front): everything a front kernel needs before staging.
  fp.front_meta.assign((size_t)P * 24, 0);
  for (int32_t q = 0; q < P; ++q) {
    const int32_t p = fp.level_fronts[q];
    int32_t* m = fp.front_meta.data() + (size_t)q * 24;
    m[0] = fp.fsz[p];
    m[1] = fp.nc[p];
    m[2] = fp.first[p];
    m[3] = p;
    const int64_t wide[4] = {fp.fe_ptr[p], fp.u_off[p], fp.l_off[p], fp.cb_off[p]};
    std::memcpy(m + 4, wide, sizeof(wide));
    const int64_t* split = fp.fe_split.data() + (size_t)p * (kFeChunks + 1);
    for (int w = 1; w <= kFeChunks; ++w) m[11 + w] = (int32_t)(split[w] - split[0]);
    m[20] = fp.front_ptr[p];
  }
  return fp;
}

}  // namespace cupf_b200
