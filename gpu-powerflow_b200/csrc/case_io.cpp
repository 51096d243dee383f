// case_io.cpp -- reader of the reference's dump-case directory format.
//
// A case directory holds (benchmark/common/matpower_data.py:341-359 writes it):
//   dump_Ybus.mtx   MatrixMarket coordinate complex, general or symmetric
//   dump_Sbus.txt   one "re im" pair per bus
//   dump_V.txt      one "re im" pair per bus (start voltage)
//   dump_pv.txt     one bus index per line
//   dump_pq.txt     one bus index per line
//   dump_Vref.txt   optional: reference solution, "re im" per bus
// Lines whose first non-blank character is '#' or '%' and blank lines are
// skipped.  Reading follows cuPF/tests/dump_case_loader.cpp:45-232: a
// symmetric file mirrors every off-diagonal entry, entries are ordered by
// (row, col) and duplicates summed, the result is CSR with sorted columns, and
// the same messages are raised for the same defects.  Duplicates are summed
// in file order (stable ordering).
#include <algorithm>
#include <cctype>
#include <complex>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cupf_b200.h"

struct pf_case_s {
  std::string name;
  int32_t rows = 0, cols = 0;
  std::vector<int32_t> indptr, indices, pv, pq;
  std::vector<std::complex<double>> ybus, sbus, v0, vref;
  bool has_vref = false;
};

namespace {

namespace fs = std::filesystem;
using Case = pf_case_s;

thread_local std::string g_case_error;

bool skip_line(const std::string& line) {
  for (char ch : line)
    if (!std::isspace(static_cast<unsigned char>(ch))) return ch == '#' || ch == '%';
  return true;
}

bool payload(std::ifstream& in, std::string& line) {
  while (std::getline(in, line))
    if (!skip_line(line)) return true;
  return false;
}

std::ifstream open_or_throw(const fs::path& p) {
  std::ifstream in(p);
  if (!in) throw std::runtime_error("Failed to open " + p.string());
  return in;
}

std::vector<std::complex<double>> read_pairs(const fs::path& p) {
  std::ifstream in = open_or_throw(p);
  std::vector<std::complex<double>> out;
  std::string line;
  while (payload(in, line)) {
    std::istringstream ss(line);
    double re = 0.0, im = 0.0;
    if (!(ss >> re >> im)) throw std::runtime_error("Malformed complex vector entry in " + p.string());
    out.emplace_back(re, im);
  }
  return out;
}

std::vector<int32_t> read_ints(const fs::path& p) {
  std::ifstream in = open_or_throw(p);
  std::vector<int32_t> out;
  std::string line;
  while (payload(in, line)) {
    std::istringstream ss(line);
    int32_t v = 0;
    if (!(ss >> v)) throw std::runtime_error("Malformed integer entry in " + p.string());
    out.push_back(v);
  }
  return out;
}

void read_ybus(const fs::path& p, Case& c) {
  std::ifstream in = open_or_throw(p);
  std::string head;
  if (!std::getline(in, head)) throw std::runtime_error("Missing MatrixMarket header in " + p.string());
  for (char& ch : head) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
  if (head.find("matrixmarket") == std::string::npos || head.find("coordinate") == std::string::npos ||
      head.find("complex") == std::string::npos)
    throw std::runtime_error("Unsupported MatrixMarket format in " + p.string());
  const bool mirror = head.find("symmetric") != std::string::npos;

  std::string line;
  if (!payload(in, line)) throw std::runtime_error("Unexpected end of file while reading " + p.string());
  int32_t nnz = 0;
  {
    std::istringstream ss(line);
    if (!(ss >> c.rows >> c.cols >> nnz)) throw std::runtime_error("Malformed MatrixMarket dimensions in " + p.string());
  }
  struct Entry {
    int32_t r, c;
    std::complex<double> v;
  };
  std::vector<Entry> ent;
  ent.reserve((size_t)std::max(nnz, 0) * (mirror ? 2 : 1));
  for (int32_t k = 0; k < nnz; ++k) {
    if (!payload(in, line)) throw std::runtime_error("Unexpected end of file while reading " + p.string());
    std::istringstream ss(line);
    int32_t r1 = 0, c1 = 0;
    double re = 0.0, im = 0.0;
    if (!(ss >> r1 >> c1 >> re >> im)) throw std::runtime_error("Malformed MatrixMarket entry in " + p.string());
    ent.push_back({r1 - 1, c1 - 1, {re, im}});
    if (mirror && r1 != c1) ent.push_back({c1 - 1, r1 - 1, {re, im}});
  }
  std::stable_sort(ent.begin(), ent.end(),
                   [](const Entry& a, const Entry& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
  std::vector<Entry> merged;
  merged.reserve(ent.size());
  for (const Entry& e : ent) {
    if (!merged.empty() && merged.back().r == e.r && merged.back().c == e.c)
      merged.back().v += e.v;
    else
      merged.push_back(e);
  }
  c.indptr.assign((size_t)std::max(c.rows, 0) + 1, 0);
  for (const Entry& e : merged) {
    if (e.r < 0 || e.r >= c.rows || e.c < 0 || e.c >= c.cols)
      throw std::runtime_error("Matrix entry out of bounds in " + p.string());
    ++c.indptr[(size_t)e.r + 1];
  }
  for (int32_t r = 0; r < c.rows; ++r) c.indptr[(size_t)r + 1] += c.indptr[(size_t)r];
  // merged is row-major sorted, so the CSR arrays are its columns in order
  c.indices.resize(merged.size());
  c.ybus.resize(merged.size());
  for (size_t k = 0; k < merged.size(); ++k) {
    c.indices[k] = merged[k].c;
    c.ybus[k] = merged[k].v;
  }
}

Case* load(const fs::path& dir) {
  if (!fs::exists(dir)) throw std::runtime_error("Case directory does not exist: " + dir.string());
  auto c = std::make_unique<Case>();
  c->name = dir.filename().string();
  read_ybus(dir / "dump_Ybus.mtx", *c);
  c->sbus = read_pairs(dir / "dump_Sbus.txt");
  c->v0 = read_pairs(dir / "dump_V.txt");
  c->pv = read_ints(dir / "dump_pv.txt");
  c->pq = read_ints(dir / "dump_pq.txt");
  if (c->rows <= 0 || c->cols <= 0) throw std::runtime_error("Loaded case has invalid Ybus dimensions");
  if (c->rows != c->cols) throw std::runtime_error("Ybus must be square");
  if ((int32_t)c->sbus.size() != c->rows) throw std::runtime_error("Sbus size does not match Ybus rows");
  if ((int32_t)c->v0.size() != c->rows) throw std::runtime_error("V0 size does not match Ybus rows");
  if (fs::exists(dir / "dump_Vref.txt")) {
    c->vref = read_pairs(dir / "dump_Vref.txt");
    if ((int32_t)c->vref.size() != c->rows) throw std::runtime_error("Vref size does not match Ybus rows");
    c->has_vref = true;
  }
  return c.release();
}

void copy_complex(const std::vector<std::complex<double>>& v, double* out) {
  if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(std::complex<double>));
}

}  // namespace

extern "C" {

pf_status pf_case_load(const char* case_dir, pf_case* out) {
  if (!out) return PF_INVALID_ARGUMENT;
  *out = nullptr;
  if (!case_dir) {
    g_case_error = "case_dir must not be null";
    return PF_INVALID_ARGUMENT;
  }
  try {
    *out = load(fs::path(case_dir));
    g_case_error.clear();
    return PF_OK;
  } catch (const std::exception& e) {
    g_case_error = e.what();
    return PF_RUNTIME_ERROR;
  }
}

const char* pf_case_last_error(void) { return g_case_error.c_str(); }

pf_status pf_case_dims(pf_case c, int32_t* rows, int32_t* cols, int32_t* nnz, int32_t* n_pv, int32_t* n_pq,
                       int32_t* has_vref) {
  if (!c) return PF_INVALID_ARGUMENT;
  if (rows) *rows = c->rows;
  if (cols) *cols = c->cols;
  if (nnz) *nnz = (int32_t)c->ybus.size();
  if (n_pv) *n_pv = (int32_t)c->pv.size();
  if (n_pq) *n_pq = (int32_t)c->pq.size();
  if (has_vref) *has_vref = c->has_vref ? 1 : 0;
  return PF_OK;
}

const char* pf_case_name(pf_case c) { return c ? c->name.c_str() : ""; }

pf_status pf_case_copy(pf_case c, int32_t* indptr, int32_t* indices, double* ybus, double* sbus, double* v0,
                       int32_t* pv, int32_t* pq, double* vref) {
  if (!c) return PF_INVALID_ARGUMENT;
  if (vref && !c->has_vref) return PF_INVALID_ARGUMENT;
  if (indptr) std::memcpy(indptr, c->indptr.data(), c->indptr.size() * sizeof(int32_t));
  if (indices && !c->indices.empty()) std::memcpy(indices, c->indices.data(), c->indices.size() * sizeof(int32_t));
  copy_complex(c->ybus, ybus);
  copy_complex(c->sbus, sbus);
  copy_complex(c->v0, v0);
  if (pv && !c->pv.empty()) std::memcpy(pv, c->pv.data(), c->pv.size() * sizeof(int32_t));
  if (pq && !c->pq.empty()) std::memcpy(pq, c->pq.data(), c->pq.size() * sizeof(int32_t));
  copy_complex(c->vref, vref);
  return PF_OK;
}

void pf_case_destroy(pf_case c) { delete c; }

}  // extern "C"
