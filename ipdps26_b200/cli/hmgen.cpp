// hmgen: writes a seeded synthetic workload (or its first n hyperedges) as a
// text file in one of the reference programs' formats. Host code only: it is
// built from the generator and file-format sources with g++ and links no CUDA,
// so a process that must not map the engine (the timed run of the reference's
// own counters) can still produce exactly the engine's inputs.
//
//   hmgen static   SEED N_NODES N_EDGES K_MIN K_MAX SIZE_EXP POP_EXP Q DEDUPE PREFIX OUT [FORMAT]
//   hmgen temporal SEED N_NODES N_EDGES K_MIN K_MAX SIZE_EXP POP_EXP Q DEDUPE
//                  BURST_RATE EVENTS_PER_BURST GAP_MEAN SPAN PREFIX OUT
//
// PREFIX = 0 writes every hyperedge, else the first PREFIX of them (the same
// node universe). FORMAT is "mochy" (default; MoCHy-master/read_data.cpp:8-45)
// or "escher" (dynamicHyperGraph/utils/utils.cpp:88-130); temporal workloads
// are written as THyMe input (THyMe-main/code/read_data.cpp:22-57).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "hmotif.h"

namespace {

int usage() {
  std::fprintf(stderr,
               "usage: hmgen static SEED N_NODES N_EDGES K_MIN K_MAX SIZE_EXP POP_EXP Q DEDUPE PREFIX OUT [mochy|escher]\n"
               "       hmgen temporal SEED N_NODES N_EDGES K_MIN K_MAX SIZE_EXP POP_EXP Q DEDUPE "
               "BURST_RATE EVENTS_PER_BURST GAP_MEAN SPAN PREFIX OUT\n");
  return 2;
}

int fail(const char* what, int status) {
  std::fprintf(stderr, "hmgen: %s: %s (%s)\n", what, hm_last_error(), hm_status_string(status));
  return 1;
}

// The first `prefix` hyperedges of g (all of them when prefix is 0 or larger).
int write_prefix(const hm_hostgraph* g, uint32_t prefix, const char* path, int format) {
  hm_hostgraph_info info;
  int s = hm_hostgraph_view(g, &info);
  if (s < 0) return fail("view", s);
  const uint32_t n = prefix && prefix < info.n_edges ? prefix : info.n_edges;
  hm_hostgraph* sub = nullptr;
  s = hm_hostgraph_from_csr(info.offsets, info.members, n, info.n_nodes, info.timestamps, &sub);
  if (s < 0) return fail("prefix", s);
  s = hm_hostgraph_write(sub, path, format);
  hm_hostgraph_free(sub);
  if (s < 0) return fail("write", s);
  std::printf("%u %u\n", n, info.n_nodes);
  return 0;
}

bool parse_gen(char** a, hm_gen_params* p) {
  char* end = nullptr;
  p->seed = std::strtoull(a[0], &end, 10);
  p->n_nodes = (uint32_t)std::strtoul(a[1], &end, 10);
  p->n_edges = (uint32_t)std::strtoul(a[2], &end, 10);
  p->k_min = (uint32_t)std::strtoul(a[3], &end, 10);
  p->k_max = (uint32_t)std::strtoul(a[4], &end, 10);
  p->size_exp = std::strtod(a[5], &end);
  p->pop_exp = std::strtod(a[6], &end);
  p->pop_offset = std::strtod(a[7], &end);
  p->dedupe = std::atoi(a[8]);
  p->permute_nodes = 1;
  return p->n_nodes > 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) return usage();
  const std::string mode = argv[1];
  hm_gen_params p;
  std::memset(&p, 0, sizeof(p));
  hm_hostgraph* g = nullptr;
  if (mode == "static") {
    if (argc != 13 && argc != 14) return usage();
    if (!parse_gen(argv + 2, &p)) return usage();
    int format = HM_FMT_MOCHY;
    if (argc == 14) {
      if (!std::strcmp(argv[13], "escher")) format = HM_FMT_ESCHER;
      else if (std::strcmp(argv[13], "mochy")) return usage();
    }
    const int s = hm_gen_static(&p, &g);
    if (s < 0) return fail("generate", s);
    const int r = write_prefix(g, (uint32_t)std::strtoul(argv[11], nullptr, 10), argv[12], format);
    hm_hostgraph_free(g);
    return r;
  }
  if (mode == "temporal") {
    if (argc != 17) return usage();
    if (!parse_gen(argv + 2, &p)) return usage();
    hm_burst_params b;
    b.burst_rate = std::strtod(argv[11], nullptr);
    b.events_per_burst = (uint32_t)std::strtoul(argv[12], nullptr, 10);
    b.gap_mean = std::strtod(argv[13], nullptr);
    b.span = std::strtoll(argv[14], nullptr, 10);
    const int s = hm_gen_temporal(&p, &b, &g);
    if (s < 0) return fail("generate", s);
    const int r = write_prefix(g, (uint32_t)std::strtoul(argv[15], nullptr, 10), argv[16], HM_FMT_THYME);
    hm_hostgraph_free(g);
    return r;
  }
  return usage();
}
