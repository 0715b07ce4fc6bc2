// Harness around the reference's own vertex-triad counters (TEST
// INFRASTRUCTURE ONLY: builds the checker). Compiled by build_ref.sh with
// -DHM_TYPE=1, 2 or 3 and the reference tree on the include path, it includes
// temporalDynamicHMotif/src/typeN.cpp where it lies (its main renamed) and
// runs that file's countTypeNMotifs on a MoCHy-format input (0-based node ids
// per line), printing the count. Node v becomes vertex v + 1 and every
// hyperedge is sorted and deduplicated, as the reference's generator makes
// them.
#define main hm_reference_type_main
#if HM_TYPE == 1
#include "src/type1.cpp"
#elif HM_TYPE == 2
#include "src/type2.cpp"
#else
#include "src/type3.cpp"
#endif
#undef main

#include <algorithm>
#include <fstream>
#include <sstream>
#include <string>

int main(int argc, char** argv) {
  if (argc != 2) return 2;
  std::ifstream in(argv[1]);
  std::vector<std::vector<int>> h2v;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty()) continue;
    std::vector<int> row;
    std::stringstream ss(line);
    std::string tok;
    while (std::getline(ss, tok, ',')) row.push_back(std::stoi(tok) + 1);
    std::sort(row.begin(), row.end());
    row.erase(std::unique(row.begin(), row.end()), row.end());
    h2v.push_back(row);
  }
#if HM_TYPE == 1
  std::printf("%lld\n", countType1Motifs(h2v));
#elif HM_TYPE == 2
  std::printf("%lld\n", countType2Motifs(h2v, vertex2hyperedge(h2v)));
#else
  std::printf("%lld\n", countType3Motifs(h2v, vertex2hyperedge(h2v)));
#endif
  return 0;
}
