// Hypergraph files in the formats the reference's programs read and write.
//
//   HM_FMT_ESCHER  dynamicHyperGraph input/*.txt: one hyperedge per line,
//                  space-separated vertex ids >= 1; empty lines and lines
//                  starting with '#' are skipped, a non-positive id is an
//                  error (utils/utils.cpp:88-130, written by :66-85).
//                  Vertex v becomes node v - 1.
//   HM_FMT_MOCHY   MoCHy: one hyperedge per line, comma-separated node ids
//                  >= 0; a node repeated within a line counts once
//                  (MoCHy-master/read_data.cpp:8-45; the reference driver
//                  writes it from 1-based ids as id - 1,
//                  figureGeneration/figure7/figure7.cu:279-294).
//   HM_FMT_THYME   THyMe: "n1,n2,...<TAB>time" per line, node ids >= 0
//                  (THyMe-main/code/read_data.cpp:22-57). THyMe reads the
//                  time as a double; here it must be an integer (int64).
//                  THyMe shuffles the lines it reads; hyperedge i here is
//                  line i.
// n_nodes of a graph read from a file is its largest node id + 1.
#include <algorithm>
#include <cerrno>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <string>
#include <vector>

#include "hm_internal.h"

namespace {

bool parse_id(const char*& p, const char* end, long long& v) {
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  if (p >= end) return false;
  char* q = nullptr;
  errno = 0;
  v = std::strtoll(p, &q, 10);
  if (q == p || errno) return false;
  p = q;
  return true;
}

int read_file(const char* path, int format, hm_hostgraph* g) {
  std::ifstream in(path);
  if (!in.is_open()) return hm::set_error(HM_ERR_INVALID, "cannot open %s", path);
  g->offsets.assign(1, 0);
  std::string line;
  uint64_t line_no = 0;
  uint64_t max_node = 0;
  bool any = false;
  std::vector<uint32_t> row;
  while (std::getline(in, line)) {
    ++line_no;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    row.clear();
    if (format == HM_FMT_ESCHER) {
      if (line.empty() || line[0] == '#') continue;
      const char* p = line.c_str();
      const char* end = p + line.size();
      long long v;
      while (parse_id(p, end, v)) {
        if (v <= 0 || v > (1ll << 32))
          return hm::set_error(HM_ERR_INVALID, "%s:%" PRIu64 ": vertex id %lld is not in [1, 2^32]", path, line_no, v);
        row.push_back((uint32_t)(v - 1));
      }
      while (p < end && (*p == ' ' || *p == '\t')) ++p;
      if (p != end) return hm::set_error(HM_ERR_INVALID, "%s:%" PRIu64 ": not a vertex id list", path, line_no);
      if (row.empty()) continue;
    } else {
      std::string nodes = line;
      if (format == HM_FMT_THYME) {
        const size_t tab = line.find('\t');
        if (tab == std::string::npos)
          return hm::set_error(HM_ERR_INVALID, "%s:%" PRIu64 ": expected 'nodes<TAB>time'", path, line_no);
        nodes = line.substr(0, tab);
        const char* t = line.c_str() + tab + 1;
        char* q = nullptr;
        errno = 0;
        const double d = std::strtod(t, &q);
        if (q == t || errno || !std::isfinite(d) || d != std::floor(d) || std::fabs(d) > 9.0e18)
          return hm::set_error(HM_ERR_INVALID, "%s:%" PRIu64 ": time is not an integer", path, line_no);
        g->times.push_back((int64_t)d);
      } else if (line.empty()) {
        continue;  // a trailing empty line
      }
      const char* p = nodes.c_str();
      const char* end = p + nodes.size();
      for (;;) {
        long long v;
        if (!parse_id(p, end, v) || v < 0 || v >= (1ll << 32))
          return hm::set_error(HM_ERR_INVALID, "%s:%" PRIu64 ": bad node id", path, line_no);
        bool seen = false;  // repeated ids within a line count once
        for (uint32_t x : row) seen |= (x == (uint32_t)v);
        if (!seen) row.push_back((uint32_t)v);
        while (p < end && (*p == ' ' || *p == '\r')) ++p;
        if (p == end) break;
        if (*p != ',') return hm::set_error(HM_ERR_INVALID, "%s:%" PRIu64 ": expected ','", path, line_no);
        ++p;
      }
    }
    for (uint32_t v : row) max_node = std::max<uint64_t>(max_node, v);
    any = any || !row.empty();
    g->members.insert(g->members.end(), row.begin(), row.end());
    g->offsets.push_back(g->members.size());
  }
  if (g->offsets.size() - 1 >= (1ull << 32)) return hm::set_error(HM_ERR_LIMIT, "%s: too many hyperedges", path);
  if (any && max_node + 1 >= (1ull << 32)) return hm::set_error(HM_ERR_LIMIT, "%s: node ids reach 2^32", path);
  g->n_nodes = any ? (uint32_t)(max_node + 1) : 0;
  return HM_OK;
}

}  // namespace

extern "C" int hm_hostgraph_read(const char* path, int format, hm_hostgraph** out) {
  if (!path || !out) return hm::set_error(HM_ERR_INVALID, "hm_hostgraph_read: NULL argument");
  *out = nullptr;
  if (format != HM_FMT_ESCHER && format != HM_FMT_MOCHY && format != HM_FMT_THYME)
    return hm::set_error(HM_ERR_INVALID, "hm_hostgraph_read: unknown format %d", format);
  try {
    auto* g = new hm_hostgraph();
    const int rc = read_file(path, format, g);
    if (rc < 0) {
      delete g;
      return rc;
    }
    *out = g;
    return HM_OK;
  } catch (const std::bad_alloc&) {
    return hm::set_error(HM_ERR_NOMEM, "hm_hostgraph_read: host allocation failed");
  }
}

extern "C" int hm_hostgraph_from_csr(const uint64_t* offsets, const uint32_t* members, uint32_t n_edges,
                                     uint32_t n_nodes, const int64_t* times, hm_hostgraph** out) {
  if (!out || (n_edges && !offsets) || (n_edges && offsets[n_edges] && !members))
    return hm::set_error(HM_ERR_INVALID, "hm_hostgraph_from_csr: NULL argument");
  *out = nullptr;
  try {
    auto* g = new hm_hostgraph();
    g->n_nodes = n_nodes;
    if (n_edges) {
      g->offsets.assign(offsets, offsets + n_edges + 1);
      g->members.assign(members, members + offsets[n_edges]);
      if (times) g->times.assign(times, times + n_edges);
    } else {
      g->offsets.assign(1, 0);
    }
    *out = g;
    return HM_OK;
  } catch (const std::bad_alloc&) {
    return hm::set_error(HM_ERR_NOMEM, "hm_hostgraph_from_csr: host allocation failed");
  }
}

extern "C" int hm_hostgraph_write(const hm_hostgraph* g, const char* path, int format) {
  if (!g || !path) return hm::set_error(HM_ERR_INVALID, "hm_hostgraph_write: NULL argument");
  if (format != HM_FMT_ESCHER && format != HM_FMT_MOCHY && format != HM_FMT_THYME)
    return hm::set_error(HM_ERR_INVALID, "hm_hostgraph_write: unknown format %d", format);
  const size_t n = g->offsets.empty() ? 0 : g->offsets.size() - 1;
  if (format == HM_FMT_THYME && g->times.size() != n)
    return hm::set_error(HM_ERR_INVALID, "hm_hostgraph_write: THyMe files need one time per hyperedge");
  FILE* f = std::fopen(path, "w");
  if (!f) return hm::set_error(HM_ERR_INVALID, "cannot write %s", path);
  const char sep = format == HM_FMT_ESCHER ? ' ' : ',';
  for (size_t e = 0; e < n; ++e) {
    if (g->offsets[e] == g->offsets[e + 1] && format != HM_FMT_ESCHER) continue;  // as the reference writers do
    for (uint64_t i = g->offsets[e]; i < g->offsets[e + 1]; ++i) {
      if (i > g->offsets[e]) std::fputc(sep, f);
      std::fprintf(f, "%" PRIu64, (uint64_t)g->members[i] + (format == HM_FMT_ESCHER ? 1 : 0));
    }
    if (format == HM_FMT_THYME) std::fprintf(f, "\t%" PRId64, g->times[e]);
    std::fputc('\n', f);
  }
  const bool ok = std::fflush(f) == 0 && !std::ferror(f);
  std::fclose(f);
  return ok ? HM_OK : hm::set_error(HM_ERR_INVALID, "write to %s failed", path);
}
