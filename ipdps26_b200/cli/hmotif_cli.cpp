// hmotif: command-line driver over the engine's C ABI, with the reference
// driver's arguments and flow (dynamicHyperGraph/src/main.cu:304-350,
// utils/utils.cpp:135-309):
//
//   hmotif <num_hyperedges> <max_vertices_per_hyperedge> <min_vertex_id>
//          <max_vertex_id> <payload_capacity> [alignment=4]
//          [-totalChanges N] [-insertionPercentage P] [-deletionPercentage P]
//          [--save-generated[=FILE]]
//   hmotif <payload_capacity> [alignment=4] --input=FILE [...]
//
// It builds the store, prints the 30 static class counts, applies one
// synthetic update batch (deletions of the last hyperedges, insertions drawn
// like the generated ones, freed ids reused first) and prints the exact
// change of the counts. payload_capacity and alignment are accepted for
// compatibility; the store has no fixed capacity.
//
// The temporal driver's flags (temporalDynamicHMotif/src/main.cu:262-372,
// utils/utils.cpp:13-40): --temporal counts the strictly increasing 30
// classes of a three-layer window whose layers all hold the graph, then of
// the window whose newest layer holds the graph after the batch, and prints
// the first counts and the difference; --temporal-synthetic uses the
// reference's fixed three-hyperedge window instead; --temporal-deltas=PATH
// applies "A|R <hyperedge> <vertices>" lines to the newer window's newest
// layer (in generate/input mode after rotating the older window so that its
// newest layer holds the graph after the batch too).
//
// Additions: --input-dir=DIR (default input, as the reference),
// --input-format=escher|mochy|thyme, --seed=S (the reference seeds with the
// time), --mochy (print MoCHy's 26 motifs as "motif i: c"),
// --temporal-delta=D (THyMe input: print THyMe's 96 motifs), --device=N,
// --no-update.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <set>
#include <string>
#include <vector>

#include "hmotif.h"

namespace {

struct Args {
  long long num_hyperedges = 0, max_vertices = 0, min_vertex = 0, max_vertex = 0, payload_capacity = 0,
            alignment = 4;
  long long total_changes = 5;
  double insertion_pct = 50.0, deletion_pct = 50.0;
  std::string input, input_dir = "input", save_name;
  bool save_generated = false;
  int format = HM_FMT_ESCHER;
  unsigned long long seed = 0;
  bool mochy = false, no_update = false;
  long long temporal_delta = -1;
  bool temporal = false, temporal_synthetic = false;
  std::string temporal_deltas;
  int device = 0;
};

void usage(const char* prog) {
  std::fprintf(stderr,
               "Usage (generate mode): %s <num_hyperedges> <max_vertices_per_hyperedge> <min_vertex_id> "
               "<max_vertex_id> <payload_capacity> [alignment=4] [-totalChanges N] [-insertionPercentage P] "
               "[-deletionPercentage P] [--save-generated[=FILE]]\n"
               "Usage (input mode):    %s <payload_capacity> [alignment=4] --input=FILE [-totalChanges N] "
               "[-insertionPercentage P] [-deletionPercentage P]\n"
               "Options: --input-dir=DIR --input-format=escher|mochy|thyme --seed=S --mochy --temporal-delta=D "
               "--temporal [--temporal-synthetic] [--temporal-deltas=PATH] --device=N --no-update\n",
               prog, prog);
}

bool pos_int(const std::string& s, long long& v) {
  char* e = nullptr;
  const long long x = std::strtoll(s.c_str(), &e, 10);
  if (s.empty() || *e || x <= 0) return false;
  v = x;
  return true;
}

bool nonneg_double(const std::string& s, double& v) {
  char* e = nullptr;
  const double x = std::strtod(s.c_str(), &e);
  if (s.empty() || *e || !(x >= 0.0)) return false;
  v = x;
  return true;
}

// Returns 0 on success, 1 on a usage error (message printed).
int parse(int argc, char** argv, Args& a) {
  if (argc < 2) {
    usage(argv[0]);
    return 1;
  }
  std::vector<std::string> pos;
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    auto value = [&](const char* name, std::string& out) -> bool {  // "-name V", "-name=V", "--name..."
      for (const std::string pre : {std::string("-") + name, std::string("--") + name}) {
        if (s == pre) {
          if (i + 1 >= argc) return false;
          out = argv[++i];
          return true;
        }
        if (s.rfind(pre + "=", 0) == 0) {
          out = s.substr(pre.size() + 1);
          return true;
        }
      }
      return false;
    };
    std::string v;
    if (s == "-h" || s == "--help") {
      usage(argv[0]);
      return 1;
    } else if (s.rfind("--input=", 0) == 0) {
      a.input = s.substr(8);
      if (a.input.empty()) {
        std::fprintf(stderr, "Error: --input requires a file name under %s/\n", a.input_dir.c_str());
        return 1;
      }
    } else if (s == "--save-generated") {
      a.save_generated = true;
    } else if (s.rfind("--save-generated=", 0) == 0) {
      a.save_generated = true;
      a.save_name = s.substr(17);
      if (a.save_name.empty()) {
        std::fprintf(stderr, "Error: --save-generated requires a non-empty file name when using '=' form\n");
        return 1;
      }
    } else if (value("totalChanges", v)) {
      if (!pos_int(v, a.total_changes)) {
        std::fprintf(stderr, "Error: totalChanges must be a positive integer\n");
        return 1;
      }
    } else if (value("insertionPercentage", v)) {
      if (!nonneg_double(v, a.insertion_pct)) {
        std::fprintf(stderr, "Error: insertionPercentage must be a non-negative number\n");
        return 1;
      }
    } else if (value("deletionPercentage", v)) {
      if (!nonneg_double(v, a.deletion_pct)) {
        std::fprintf(stderr, "Error: deletionPercentage must be a non-negative number\n");
        return 1;
      }
    } else if (s.rfind("--input-dir=", 0) == 0) {
      a.input_dir = s.substr(12);
    } else if (s.rfind("--input-format=", 0) == 0) {
      const std::string f = s.substr(15);
      if (f == "escher") a.format = HM_FMT_ESCHER;
      else if (f == "mochy") a.format = HM_FMT_MOCHY;
      else if (f == "thyme") a.format = HM_FMT_THYME;
      else {
        std::fprintf(stderr, "Error: unknown input format '%s'\n", f.c_str());
        return 1;
      }
    } else if (s.rfind("--seed=", 0) == 0) {
      a.seed = std::strtoull(s.c_str() + 7, nullptr, 10);
    } else if (s == "--mochy") {
      a.mochy = true;
    } else if (s == "--no-update") {
      a.no_update = true;
    } else if (s == "--temporal") {
      a.temporal = true;
    } else if (s == "--temporal-synthetic") {
      a.temporal_synthetic = true;
    } else if (s.rfind("--temporal-deltas=", 0) == 0) {
      a.temporal_deltas = s.substr(18);
    } else if (s.rfind("--temporal-delta=", 0) == 0) {
      long long d;
      if (!pos_int(s.substr(17), d)) {
        std::fprintf(stderr, "Error: temporal-delta must be a positive integer\n");
        return 1;
      }
      a.temporal_delta = d;
    } else if (s.rfind("--device=", 0) == 0) {
      a.device = std::atoi(s.c_str() + 9);
    } else {
      pos.push_back(s);
    }
  }
  if (!a.input.empty()) {
    if (pos.empty() || pos.size() > 2) {
      std::fprintf(stderr, "Error: input mode expects <payload_capacity> [alignment=4] plus --input=FILE\n");
      usage(argv[0]);
      return 1;
    }
    if (!pos_int(pos[0], a.payload_capacity) || (pos.size() == 2 && !pos_int(pos[1], a.alignment))) {
      std::fprintf(stderr, "Error: payload_capacity and alignment must be positive integers\n");
      return 1;
    }
    if (a.save_generated) {
      std::printf("Warning: --save-generated is ignored when --input is provided.\n");
      a.save_generated = false;
    }
  } else {
    if (pos.size() < 5 || pos.size() > 6) {
      std::fprintf(stderr,
                   "Error: generate mode expects <num_hyperedges> <max_vertices_per_hyperedge> <min_vertex_id> "
                   "<max_vertex_id> <payload_capacity> [alignment=4]\n");
      usage(argv[0]);
      return 1;
    }
    if (!pos_int(pos[0], a.num_hyperedges) || !pos_int(pos[1], a.max_vertices) || !pos_int(pos[2], a.min_vertex) ||
        !pos_int(pos[3], a.max_vertex) || !pos_int(pos[4], a.payload_capacity) ||
        (pos.size() == 6 && !pos_int(pos[5], a.alignment))) {
      std::fprintf(stderr, "Error: all generate-mode numeric arguments must be positive integers\n");
      return 1;
    }
    if (a.min_vertex >= a.max_vertex) {
      std::fprintf(stderr, "Error: min_vertex_id must be less than max_vertex_id\n");
      return 1;
    }
    if (a.max_vertices > HM_MAX_EDGE_SIZE || a.max_vertices > a.max_vertex - a.min_vertex + 1) {
      std::fprintf(stderr, "Error: max_vertices_per_hyperedge must be at most %d and fit the vertex range\n",
                   HM_MAX_EDGE_SIZE);
      return 1;
    }
  }
  if (a.insertion_pct + a.deletion_pct <= 0.0) {
    std::fprintf(stderr,
                 "Error: insertionPercentage and deletionPercentage must be non-negative, and their sum must be > 0\n");
    return 1;
  }
  if (a.temporal_delta > 0 && a.format != HM_FMT_THYME) {
    std::fprintf(stderr, "Error: --temporal-delta needs --input-format=thyme\n");
    return 1;
  }
  if (a.temporal && a.temporal_delta > 0) {
    std::fprintf(stderr, "Error: --temporal (three-layer window) and --temporal-delta (THyMe) exclude each other\n");
    return 1;
  }
  return 0;
}

// n hyperedges of 1..m distinct vertices uniform in [r1, r2], as 0-based
// node ids (vertex v is node v - 1): the reference generator's distribution
// (src/graphGeneration.cpp:10-29) from a seeded engine.
void generate(std::mt19937_64& rng, long long n, long long m, long long r1, long long r2,
              std::vector<uint64_t>& off, std::vector<uint32_t>& mem) {
  std::uniform_int_distribution<long long> size(1, m), vert(r1, r2);
  for (long long i = 0; i < n; ++i) {
    const long long k = size(rng);
    std::set<long long> s;
    while ((long long)s.size() < k) s.insert(vert(rng));
    for (long long v : s) mem.push_back((uint32_t)(v - 1));
    off.push_back(mem.size());
  }
}

int fail(const char* what) {
  std::fprintf(stderr, "Error: %s: %s\n", what, hm_last_error());
  return 2;
}

void print30(const char* title, const uint64_t* c) {
  std::printf("%s (30 bins): ", title);
  for (int i = 0; i < HM_N_STATIC_CLASSES; ++i) std::printf("%llu%c", (unsigned long long)c[i], i + 1 < 30 ? ' ' : '\n');
}

using Rows = std::vector<std::vector<uint32_t>>;

int set_layer(hm_window* w, int layer, const Rows& rows) {
  std::vector<uint64_t> off(1, 0);
  std::vector<uint32_t> mem;
  for (const auto& r : rows) {
    mem.insert(mem.end(), r.begin(), r.end());
    off.push_back(mem.size());
  }
  return hm_window_set_layer(w, layer, off.data(), mem.data(), (uint32_t)rows.size());
}

// The three-layer strictly increasing count of the temporal driver. base is
// the graph, updated the graph after the batch (deleted rows empty, inserted
// rows at their ids); the synthetic window replaces both.
int temporal_windows(const Args& a, hm_ctx* ctx, uint32_t n_nodes, const Rows& base, const Rows& updated) {
  // the reference's fixed window: Older = Middle = Newest = {1,2},{2,3},{1,3};
  // the newer window's Newest is {1,2},{2,3},{1,2,3} (vertex v is node v - 1)
  const Rows syn = {{0, 1}, {1, 2}, {0, 2}}, syn_new = {{0, 1}, {1, 2}, {0, 1, 2}};
  const uint32_t wn = std::max<uint32_t>(n_nodes, 3);
  hm_window *ow = nullptr, *nw = nullptr;
  if (hm_window_create(ctx, wn, &ow) < 0 || hm_window_create(ctx, wn, &nw) < 0) {
    hm_window_destroy(ow);
    return fail("creating the temporal windows");
  }
  int rc = 0;
  uint64_t c_old[HM_N_STATIC_CLASSES], c_new[HM_N_STATIC_CLASSES];
  const Rows& older = a.temporal_synthetic ? syn : base;
  const Rows& newest = a.temporal_synthetic ? syn_new : updated;
  do {
    if (set_layer(ow, HM_LAYER_OLDER, older) < 0 || set_layer(ow, HM_LAYER_MIDDLE, older) < 0 ||
        set_layer(ow, HM_LAYER_NEWEST, older) < 0) {
      rc = fail("building the older window");
      break;
    }
    if (hm_window_count30(ow, c_old) < 0) {
      rc = fail("temporal count");
      break;
    }
    print30("Temporal strict-inc counts", c_old);
    if (set_layer(nw, HM_LAYER_OLDER, older) < 0 || set_layer(nw, HM_LAYER_MIDDLE, older) < 0 ||
        set_layer(nw, HM_LAYER_NEWEST, newest) < 0) {
      rc = fail("building the newer window");
      break;
    }
    if (!a.temporal_deltas.empty()) {
      if (!a.temporal_synthetic &&
          (hm_window_rotate(ow) < 0 || set_layer(ow, HM_LAYER_NEWEST, updated) < 0 || hm_window_count30(ow, c_old) < 0)) {
        rc = fail("rotating the older window");
        break;
      }
      if (hm_window_apply_deltas_file(nw, a.temporal_deltas.c_str()) < 0) {
        rc = fail("applying the temporal deltas");
        break;
      }
    }
    if (hm_window_count30(nw, c_new) < 0) {
      rc = fail("temporal count");
      break;
    }
    std::printf("Temporal strict-inc delta (30 bins): ");
    for (int i = 0; i < HM_N_STATIC_CLASSES; ++i)
      std::printf("%lld%c", (long long)(c_new[i] - c_old[i]), i + 1 < 30 ? ' ' : '\n');
  } while (false);
  hm_window_destroy(ow);
  hm_window_destroy(nw);
  return rc;
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  if (parse(argc, argv, a)) return 1;
  std::mt19937_64 rng(a.seed);
  std::vector<uint64_t> off(1, 0);
  std::vector<uint32_t> mem;
  std::vector<int64_t> times;
  uint32_t n_nodes = 0;
  if (!a.input.empty()) {
    const std::string path = a.input_dir + "/" + a.input;
    hm_hostgraph* hg = nullptr;
    if (hm_hostgraph_read(path.c_str(), a.format, &hg) < 0) return fail("reading the input");
    hm_hostgraph_info info;
    hm_hostgraph_view(hg, &info);
    off.assign(info.offsets, info.offsets + info.n_edges + 1);
    mem.assign(info.members, info.members + info.n_members);
    if (info.timestamps) times.assign(info.timestamps, info.timestamps + info.n_edges);
    n_nodes = info.n_nodes;
    hm_hostgraph_free(hg);
    if (info.n_edges == 0) {
      std::fprintf(stderr, "Error: input file contains no hyperedges: %s\n", path.c_str());
      return 1;
    }
    std::printf("Loaded hypergraph from %s (%u hyperedges, %u nodes)\n", path.c_str(), info.n_edges, n_nodes);
    a.num_hyperedges = info.n_edges;
    a.max_vertices = 0;
    a.min_vertex = 1;
    a.max_vertex = n_nodes;
    for (uint32_t e = 0; e < info.n_edges; ++e) a.max_vertices = std::max<long long>(a.max_vertices, off[e + 1] - off[e]);
    if (a.max_vertices > HM_MAX_EDGE_SIZE) a.max_vertices = HM_MAX_EDGE_SIZE;
    if (a.max_vertex < 2) a.max_vertex = 2;
  } else {
    generate(rng, a.num_hyperedges, a.max_vertices, a.min_vertex, a.max_vertex, off, mem);
    n_nodes = (uint32_t)a.max_vertex;
    std::printf("Generated %lld hyperedges over vertices [%lld, %lld] (seed %llu)\n", a.num_hyperedges, a.min_vertex,
                a.max_vertex, a.seed);
    if (a.save_generated) {
      const std::string path = a.input_dir + "/" + (a.save_name.empty() ? "generated_hypergraph.txt" : a.save_name);
      hm_hostgraph* hg = nullptr;
      if (hm_hostgraph_from_csr(off.data(), mem.data(), (uint32_t)(off.size() - 1), n_nodes, nullptr, &hg) < 0 ||
          hm_hostgraph_write(hg, path.c_str(), HM_FMT_ESCHER) < 0) {
        hm_hostgraph_free(hg);
        return fail("saving the generated hypergraph");
      }
      hm_hostgraph_free(hg);
      std::printf("Saved generated hypergraph to %s\n", path.c_str());
    }
  }
  const uint32_t n_edges = (uint32_t)(off.size() - 1);

  hm_ctx* ctx = nullptr;
  if (hm_ctx_create(a.device, 0, &ctx) < 0) return fail("creating the device context");
  int rc = 0;
  hm_graph* g = nullptr;
  if (a.temporal_delta > 0) {
    if (times.size() != n_edges) return fail("the input has no times");
    if (hm_graph_build(ctx, off.data(), mem.data(), n_edges, n_nodes, times.data(), &g) < 0) return fail("build");
    uint64_t c96[HM_N_TEMPORAL_MOTIFS];
    if (hm_count_temporal(g, a.temporal_delta, c96) < 0) return fail("temporal count");
    for (int i = 0; i < HM_N_TEMPORAL_MOTIFS; ++i) std::printf("motif %d: %llu\n", i + 1, (unsigned long long)c96[i]);
    hm_graph_destroy(g);
    hm_ctx_destroy(ctx);
    return 0;
  }
  Rows base(n_edges);
  for (uint32_t e = 0; e < n_edges; ++e) base[e].assign(mem.begin() + off[e], mem.begin() + off[e + 1]);
  Rows updated = base;
  if (hm_graph_build(ctx, off.data(), mem.data(), n_edges, n_nodes, nullptr, &g) < 0) return fail("build");
  uint64_t c30[HM_N_STATIC_CLASSES];
  if (hm_count_static30(g, c30) < 0) return fail("count");
  print30("Motif counts", c30);
  if (a.mochy) {
    uint64_t c26[HM_N_STATIC_MOTIFS];
    if (hm_count_static(g, c26) < 0) return fail("count");
    for (int i = 0; i < HM_N_STATIC_MOTIFS; ++i) std::printf("motif %d: %llu\n", i + 1, (unsigned long long)c26[i]);
  }
  if (!a.no_update) {
    // buildSyntheticUpdateBatch (src/main.cu:159-236): sizes from the
    // percentages, the rounding remainder to the larger share, deletions
    // capped at the hyperedge count; the last hyperedges are deleted.
    long long n_del = std::llround((double)a.total_changes * (a.deletion_pct / 100.0));
    long long n_ins = std::llround((double)a.total_changes * (a.insertion_pct / 100.0));
    const long long diff = a.total_changes - (n_del + n_ins);
    if (diff) (a.insertion_pct >= a.deletion_pct ? n_ins : n_del) += diff;
    if (n_del < 0) n_del = 0;
    if (n_ins < 0) n_ins = 0;
    if (n_del > n_edges) {
      n_del = n_edges;
      n_ins = std::max<long long>(0, a.total_changes - n_del);
    }
    if (n_del == 0 && n_ins == 0) n_ins = a.total_changes;
    std::printf("Synthetic update batch sizes -> deletes: %lld, inserts: %lld (totalChanges=%lld)\n", n_del, n_ins,
                a.total_changes);
    std::vector<uint32_t> dels;
    for (long long k = n_del - 1; k >= 0; --k) dels.push_back((uint32_t)(n_edges - 1 - k));
    std::vector<uint64_t> ioff(1, 0);
    std::vector<uint32_t> imem;
    generate(rng, n_ins, a.max_vertices, a.min_vertex, a.max_vertex, ioff, imem);
    for (uint32_t& v : imem)
      if (v >= n_nodes) v = n_nodes - 1;  // input mode: keep draws inside the file's node range
    std::vector<uint32_t> ids(std::max<long long>(n_ins, 1));
    int64_t d30[HM_N_STATIC_CLASSES];
    if (hm_graph_apply_batch(g, dels.data(), (uint32_t)dels.size(), ioff.data(), imem.data(), (uint32_t)n_ins,
                             ids.data(), d30) < 0)
      return fail("update batch");
    std::printf("Inserted ids (1-based):");
    for (long long i = 0; i < n_ins; ++i) std::printf(" %u", ids[i] + 1);
    for (uint32_t d : dels) updated[d].clear();
    for (long long i = 0; i < n_ins; ++i) {
      if (ids[i] >= updated.size()) updated.resize(ids[i] + 1);
      updated[ids[i]].assign(imem.begin() + ioff[i], imem.begin() + ioff[i + 1]);
    }
    std::printf("\nMotif delta counts (30 bins): ");
    for (int i = 0; i < HM_N_STATIC_CLASSES; ++i) std::printf("%lld%c", (long long)d30[i], i + 1 < 30 ? ' ' : '\n');
    if (hm_count_static30(g, c30) < 0) return fail("count");
    print30("Motif counts after the batch", c30);
  }
  if (a.temporal) rc = temporal_windows(a, ctx, n_nodes, base, updated);
  hm_graph_destroy(g);
  hm_ctx_destroy(ctx);
  return rc;
}
