// NASTRAN bulk-data (BDF) mesh input for the shell path: the part of
// TACSMeshLoader::scanBDFFile / getAssemblerCreatorData
// (include/mesh/TACSMeshLoader.h:188-225, :762-...) that the reference's
// createFromBDF (include/assembler.h:92-115) uses.
//   GRID / GRID*           node coordinates (CP and CD frames must be 0)
//   CQUAD4 / CQUADR (/ *)  4-node shells; nodes G1 G2 G3 G4 (around the
//                          element) are stored in tensor order G1 G2 G4 G3
//   SPC / SPC*             constrained DOFs (digits 1..6) of the listed nodes
// Small-field (8-column), large-field (keyword with '*', 16-column fields on
// two lines) and free-field (comma separated) entries are read, with
// continuation lines ('+' / '*' leading field, or a blank first field).
// Nodes are numbered by ascending file id, elements by ascending file id;
// NASTRAN reals without 'E' ("1.5-3" = 1.5e-3) are accepted. Other element
// cards are an error for the shell path.
#include <algorithm>
#include <array>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "gf_internal.h"

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

// NASTRAN real: "1.5-3" / "-2.+4" / "3.0E-2" / "7" / "" (0)
bool bdf_real(const std::string& f, double* out) {
  std::string s = trim(f);
  if (s.empty()) {
    *out = 0.0;
    return true;
  }
  // an exponent sign that is not at the start and not after E/D
  for (size_t k = 1; k < s.size(); k++) {
    const char c = s[k], p = (char)std::toupper((unsigned char)s[k - 1]);
    if ((c == '+' || c == '-') && p != 'E' && p != 'D') {
      s.insert(k, "E");
      break;
    }
  }
  for (auto& c : s)
    if (c == 'D' || c == 'd') c = 'E';
  char* end = nullptr;
  *out = std::strtod(s.c_str(), &end);
  return end && *end == '\0';
}

bool bdf_int(const std::string& f, long* out) {
  const std::string s = trim(f);
  if (s.empty()) {
    *out = 0;
    return true;
  }
  char* end = nullptr;
  *out = std::strtol(s.c_str(), &end, 10);
  return end && *end == '\0';
}

// One bulk-data entry: its keyword and data fields (continuations merged;
// the continuation markers are dropped).
struct Entry {
  std::string key;
  std::vector<std::string> f;
};

// fields of one physical line, without the keyword field
void split_line(const std::string& line, bool large, std::vector<std::string>& out,
                bool* free_field) {
  if (line.find(',') != std::string::npos) {
    *free_field = true;
    size_t a = 0;
    bool first = true;
    while (a <= line.size()) {
      size_t b = line.find(',', a);
      if (b == std::string::npos) b = line.size();
      if (!first) out.push_back(line.substr(a, b - a));
      first = false;
      a = b + 1;
    }
    return;
  }
  *free_field = false;
  const size_t w = large ? 16 : 8, nf = large ? 4 : 8;
  for (size_t k = 0; k < nf; k++) {
    const size_t a = 8 + k * w;
    out.push_back(a < line.size() ? line.substr(a, std::min(w, line.size() - a)) : std::string());
  }
}

bool is_continuation(const std::string& line) {
  if (line.empty()) return false;
  if (line[0] == '+' || line[0] == '*' || line[0] == ',') return true;
  // a blank first field (small or large)
  return line.size() > 0 && trim(line.substr(0, std::min<size_t>(8, line.size()))).empty() &&
         !trim(line).empty();
}

}  // namespace

struct gf_bdf_mesh_impl {
  gf_bdf_mesh pub{};
  std::vector<int32_t> conn, bcs, comp;
  std::vector<double> xpts;
};

extern "C" {

gf_status gf_bdf_read(const char* path, gf_bdf_mesh** out) {
  if (!path || !out) return GF_INVALID_ARG;
  std::ifstream in(path);
  if (!in) {
    ::gf::set_last_error_text(std::string("gf_bdf_read: cannot open ") + path);
    return GF_INVALID_ARG;
  }
  std::vector<std::string> lines;
  {
    std::string l;
    while (std::getline(in, l)) {
      if (!l.empty() && l.back() == '\r') l.pop_back();
      for (auto& c : l)
        if (c == '\t') c = ' ';
      lines.push_back(l);
    }
  }
  // bulk data: after BEGIN BULK when present, up to ENDDATA
  size_t start = 0;
  for (size_t k = 0; k < lines.size(); k++)
    if (lines[k].compare(0, 10, "BEGIN BULK") == 0) {
      start = k + 1;
      break;
    }
  std::vector<Entry> entries;
  for (size_t k = start; k < lines.size(); k++) {
    const std::string& l = lines[k];
    if (l.empty() || l[0] == '$') continue;
    if (l.compare(0, 7, "ENDDATA") == 0 || l.compare(0, 8, "END BULK") == 0) break;
    bool free_field = false;
    if (is_continuation(l) && !entries.empty()) {
      const bool large = l[0] == '*';
      std::vector<std::string> f;
      split_line(l, large, f, &free_field);
      auto& e = entries.back();
      e.f.insert(e.f.end(), f.begin(), f.end());
      continue;
    }
    Entry e;
    std::string key = l.find(',') != std::string::npos ? l.substr(0, l.find(',')) : l.substr(0, 8);
    key = trim(key);
    const bool large = !key.empty() && key.back() == '*';
    if (large) key.pop_back();
    for (auto& c : key) c = (char)std::toupper((unsigned char)c);
    e.key = key;
    split_line(l, large, e.f, &free_field);
    entries.push_back(std::move(e));
  }
  // GRID: id, cp, x1, x2, x3, cd
  std::map<long, int> node_of;  // file id -> (later) index
  std::vector<std::pair<long, std::array<double, 3>>> grids;
  struct Quad {
    long eid, pid, g[4];
  };
  std::vector<Quad> quads;
  std::vector<std::pair<long, int>> spcs;  // (file node id, dof 0..5)
  for (const auto& e : entries) {
    auto fld = [&](size_t i) { return i < e.f.size() ? e.f[i] : std::string(); };
    if (e.key == "GRID") {
      long id, cp = 0, cd = 0;
      double x[3];
      if (!bdf_int(fld(0), &id) || !bdf_int(fld(1), &cp) || !bdf_real(fld(2), &x[0]) ||
          !bdf_real(fld(3), &x[1]) || !bdf_real(fld(4), &x[2]) || !bdf_int(fld(5), &cd) ||
          cp != 0 || cd != 0) {
        ::gf::set_last_error_text("gf_bdf_read: unreadable GRID entry (or CP / CD frame not 0)");
        return GF_INVALID_ARG;
      }
      grids.push_back({id, {x[0], x[1], x[2]}});
    } else if (e.key == "CQUAD4" || e.key == "CQUADR") {
      Quad q;
      bool ok = bdf_int(fld(0), &q.eid) && bdf_int(fld(1), &q.pid);
      for (int a = 0; a < 4 && ok; a++) ok = bdf_int(fld(2 + a), &q.g[a]) && q.g[a] > 0;
      if (!ok) {
        ::gf::set_last_error_text("gf_bdf_read: unreadable " + e.key + " entry");
        return GF_INVALID_ARG;
      }
      quads.push_back(q);
    } else if (e.key == "SPC") {
      // SID, then (G, C, D) triples
      for (size_t t = 1; t < e.f.size(); t += 3) {
        long g;
        if (!bdf_int(fld(t), &g)) break;
        if (g <= 0) continue;
        for (char c : trim(fld(t + 1)))
          if (c >= '1' && c <= '6') spcs.push_back({g, c - '1'});
      }
    } else if (e.key.compare(0, 1, "C") == 0 &&
               (e.key == "CTRIA3" || e.key == "CQUAD8" || e.key == "CQUAD9" || e.key == "CQUAD" ||
                e.key == "CHEXA" || e.key == "CTETRA" || e.key == "CBAR")) {
      ::gf::set_last_error_text("gf_bdf_read: element " + e.key +
                                " is not a 4-node shell (CQUAD4 / CQUADR)");
      return GF_INVALID_ARG;
    }
  }
  std::sort(grids.begin(), grids.end(),
            [](const auto& a, const auto& b) { return a.first < b.first; });
  for (size_t k = 0; k < grids.size(); k++) {
    if (k && grids[k].first == grids[k - 1].first) {
      ::gf::set_last_error_text("gf_bdf_read: duplicate GRID id " + std::to_string(grids[k].first));
      return GF_INVALID_ARG;
    }
    node_of[grids[k].first] = (int)k;
  }
  std::sort(quads.begin(), quads.end(), [](const Quad& a, const Quad& b) { return a.eid < b.eid; });
  auto* m = new gf_bdf_mesh_impl();
  m->xpts.resize(3 * grids.size());
  for (size_t k = 0; k < grids.size(); k++)
    for (int d = 0; d < 3; d++) m->xpts[3 * k + d] = grids[k].second[d];
  for (const auto& q : quads) {
    int idx[4];
    for (int a = 0; a < 4; a++) {
      auto it = node_of.find(q.g[a]);
      if (it == node_of.end()) {
        ::gf::set_last_error_text("gf_bdf_read: element " + std::to_string(q.eid) +
                                  " uses missing GRID " + std::to_string(q.g[a]));
        delete m;
        return GF_INVALID_ARG;
      }
      idx[a] = it->second;
    }
    // G1 G2 G3 G4 around the element -> tensor order G1 G2 G4 G3
    m->conn.insert(m->conn.end(), {idx[0], idx[1], idx[3], idx[2]});
    m->comp.push_back((int32_t)q.pid);
  }
  for (const auto& sc : spcs) {
    auto it = node_of.find(sc.first);
    if (it == node_of.end()) {
      ::gf::set_last_error_text("gf_bdf_read: SPC on missing GRID " + std::to_string(sc.first));
      delete m;
      return GF_INVALID_ARG;
    }
    m->bcs.push_back(6 * it->second + sc.second);
  }
  std::sort(m->bcs.begin(), m->bcs.end());
  m->bcs.erase(std::unique(m->bcs.begin(), m->bcs.end()), m->bcs.end());
  m->pub.num_nodes = (int32_t)grids.size();
  m->pub.num_elements = (int32_t)quads.size();
  m->pub.num_bcs = (int32_t)m->bcs.size();
  m->pub.conn = m->conn.data();
  m->pub.xpts = m->xpts.data();
  m->pub.bcs = m->bcs.data();
  m->pub.component = m->comp.data();
  m->pub.impl = m;
  *out = &m->pub;
  return GF_OK;
}

gf_status gf_bdf_free(gf_bdf_mesh* mesh) {
  if (mesh) delete static_cast<gf_bdf_mesh_impl*>(mesh->impl);
  return GF_OK;
}

}  // extern "C"
