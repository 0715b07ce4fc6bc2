"""The reference-shaped C++ shim (include/hmotif_cbst.hpp) run on the GPU: a
program written against the reference's host interface (flat 1-based
payloads with 0 pads, 1-based keys, computeMotifCounts, an erase + insert
batch with its delta, keyed insert (fillCBST) and unfill with their deltas,
the three-layer temporal ring and its delta file)
prints counts that equal the oracle's."""
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

PROGRAM = r"""
#include <cstdio>
#include <fstream>
#include <vector>

#include "hmotif_cbst.hpp"

static void print(const char* title, const std::vector<int64_t>& c) {
  std::printf("%s:", title);
  for (int64_t x : c) std::printf(" %lld", (long long)x);
  std::printf("\n");
}

int main(int argc, char** argv) {
  // argv[1]: "n" then n lines "k v1 .. vk" (1-based vertices); argv[2]: delta file
  std::ifstream in(argv[1]);
  int n = 0, maxv = 0;
  in >> n;
  std::vector<int> starts, flat;
  for (int i = 0; i < n; ++i) {
    int k;
    in >> k;
    starts.push_back((int)flat.size());
    for (int j = 0; j < k; ++j) {
      int v;
      in >> v;
      flat.push_back(v);
      if (v > maxv) maxv = v;
    }
    while (flat.size() % 4) flat.push_back(0);  // the reference's alignment padding
  }
  hm::Context ctx(0);
  hm::HypergraphStore store(ctx, "H2V");
  store.construct(starts.data(), n, flat.data(), (int)flat.size(), (uint32_t)maxv + 1);
  auto c = hm::computeMotifCounts(store, false);
  print("static", std::vector<int64_t>(c.begin(), c.end()));
  // erase the last three keys, insert two records: {1,2,3} and {2,maxv}
  std::vector<int64_t> d;
  auto keys = store.update({n - 2, n - 1, n}, {1, 2, 3, 2, maxv}, {3, 5}, &d);
  print("delta", d);
  std::printf("keys: %d %d\n", keys[0], keys[1]);
  c = hm::computeMotifCounts(store, false);
  print("after", std::vector<int64_t>(c.begin(), c.end()));
  // CBSTOperations::insert(insertKeys, insertPayload, insertPrefixSizes) is
  // fillCBST: values appended to existing keys, which keep their ids
  store.insert({1, 2}, {maxv, 3, 1}, {2, 3}, &d);
  print("fill_delta", d);
  c = hm::computeMotifCounts(store, false);
  print("after_fill", std::vector<int64_t>(c.begin(), c.end()));
  store.unfill({1}, {maxv}, {1}, &d);
  print("unfill_delta", d);
  c = hm::computeMotifCounts(store, false);
  print("after_unfill", std::vector<int64_t>(c.begin(), c.end()));

  std::vector<int> tkeys;
  for (int i = 0; i < n; ++i) tkeys.push_back(i + 1);
  hm::TemporalWindow w(ctx, (uint32_t)maxv), w2(ctx, (uint32_t)maxv);
  for (auto l : {hm::TemporalLayer::Older, hm::TemporalLayer::Middle, hm::TemporalLayer::Newest}) {
    w.construct(l, tkeys.data(), starts.data(), n, flat.data(), (int)flat.size());
    w2.construct(l, tkeys.data(), starts.data(), n, flat.data(), (int)flat.size());
  }
  std::vector<int64_t> t;
  hm::computeTemporalMotifCountsStrictInc(w, t);
  print("window", t);
  if (!hm::applyTemporalDeltasFromFile(argv[2], w2)) return 3;
  w2.fill(hm::TemporalLayer::Newest, {n - 2}, {maxv}, {1});
  hm::computeTemporalMotifCountsStrictIncDelta(w, w2, t);
  print("window_delta", t);
  return 0;
}
"""


def _csr(rows):
    off = np.zeros(len(rows) + 1, np.uint64)
    off[1:] = np.cumsum([len(r) for r in rows])
    return off, np.array([v for r in rows for v in r], np.uint32)


def _line(out, title):
    m = re.search(r"^" + re.escape(title) + r":((?: -?\d+)*)$", out, flags=re.M)
    assert m, out
    return [int(x) for x in m.group(1).split()]


def test_reference_shaped_program_matches_oracle(tmp_path):
    from ipdps26_b200 import gen
    from oracle import oracle

    cxx = shutil.which("g++")
    assert cxx, "g++ is needed to build the shim program"
    src = tmp_path / "shim_prog.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "shim_prog"
    r = subprocess.run([cxx, "-O1", "-std=c++17", f"-I{ROOT / 'include'}", str(src), "-o", str(exe),
                        f"-L{ROOT / 'ipdps26_b200'}", "-lhmotif", f"-Wl,-rpath,{ROOT / 'ipdps26_b200'}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    h = gen.static(gen.params(41, 60, 150, 2, 9, 2.5, 1.2, 5.0))
    rows = [[int(v) + 1 for v in h.edge(i)] for i in range(h.n_edges)]  # 1-based vertices
    n, maxv = len(rows), max(max(r) for r in rows)
    (tmp_path / "g.txt").write_text(f"{n}\n" + "".join(f"{len(r)} {' '.join(map(str, r))}\n" for r in rows))
    # edits of the newest layer's last hyperedges (strictly increasing triples end there)
    (tmp_path / "d.txt").write_text(f"A {n - 1} 1 {maxv}\nR {n} {rows[n - 1][0]}\n")
    r = subprocess.run([str(exe), str(tmp_path / "g.txt"), str(tmp_path / "d.txt")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    out = r.stdout

    # the store uses payload values as node ids
    before = oracle.static30(*_csr(rows), maxv + 1)
    after_rows = rows[: n - 3] + [[1, 2, 3], [2, maxv]]
    after = oracle.static30(*_csr(after_rows), maxv + 1)
    assert _line(out, "static") == before.tolist()
    assert _line(out, "after") == after.tolist()
    assert _line(out, "delta") == (after.astype(np.int64) - before.astype(np.int64)).tolist()
    assert _line(out, "keys") == [n - 2, n - 1]  # freed keys reused, ascending
    # keyed fill of keys 1 and 2, then unfill of key 1 (keys are 1-based)
    filled = [list(r) for r in after_rows]
    filled[0] = sorted(set(filled[0]) | {maxv, 3})
    filled[1] = sorted(set(filled[1]) | {1})
    after_fill = oracle.static30(*_csr(filled), maxv + 1)
    assert _line(out, "after_fill") == after_fill.tolist()
    assert _line(out, "fill_delta") == (after_fill.astype(np.int64) - after.astype(np.int64)).tolist()
    unfilled = [list(r) for r in filled]
    unfilled[0] = sorted(set(unfilled[0]) - {maxv})
    after_unfill = oracle.static30(*_csr(unfilled), maxv + 1)
    assert _line(out, "after_unfill") == after_unfill.tolist()
    assert _line(out, "unfill_delta") == (after_unfill.astype(np.int64) - after_fill.astype(np.int64)).tolist()

    # the window: vertex v is node v - 1 in constructs, fills and delta files alike
    layer = [[v - 1 for v in r] for r in rows]
    newest = [list(r) for r in layer]
    newest[n - 2] = sorted(set(newest[n - 2]) | {0, maxv - 1})
    newest[n - 1] = sorted(set(newest[n - 1]) - {rows[n - 1][0] - 1})
    newest[n - 3] = sorted(set(newest[n - 3]) | {maxv - 1})
    base = oracle.strictinc30([_csr(layer)] * 3)
    new = oracle.strictinc30([_csr(layer), _csr(layer), _csr(newest)])
    assert base.sum() > 0 and np.any(new != base)
    assert _line(out, "window") == base.tolist()
    assert _line(out, "window_delta") == (new.astype(np.int64) - base.astype(np.int64)).tolist()
