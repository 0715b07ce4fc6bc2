"""The C ABI library loads and exports every entry point include/*.h declares."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(hm_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["hm_ctx_create", "hm_graph_build", "hm_count_static", "hm_graph_query"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from ipdps26_b200 import _lib

    missing = [n for n in declared_functions() if not hasattr(_lib.lib, n)]
    assert not missing, f"symbols declared in include/*.h but not exported: {missing}"


def test_status_strings():
    from ipdps26_b200._lib import lib

    assert lib.hm_status_string(0) == b"ok"
    assert b"invalid" in lib.hm_status_string(-1)


def test_no_device_means_clean_error():
    """Without a GPU, creating a context fails with a status, never exits."""
    import torch

    if torch.cuda.is_available():
        return
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HmError

    try:
        engine.Context(0)
    except HmError as e:
        assert e.status < 0
    else:
        raise AssertionError("context creation succeeded without a device")


def test_cpp_shim_compiles_and_links(tmp_path):
    """The reference-shaped C++ shim (include/hmotif_cbst.hpp) builds against
    the library (linking only; nothing runs without a GPU)."""
    import shutil
    import subprocess

    cxx = shutil.which("g++")
    if cxx is None:
        return
    src = tmp_path / "use_shim.cpp"
    src.write_text(
        '#include "hmotif_cbst.hpp"\n'
        "int main(int argc, char**) {\n"
        "  if (argc < 99) return 0;  // link check only\n"
        "  hm::Context ctx(0);\n"
        "  hm::HypergraphStore s(ctx, \"H2V\");\n"
        "  int starts[2] = {0, 4}; int flat[8] = {1, 2, 0, 0, 2, 3, 0, 0};\n"
        "  s.construct(starts, 2, flat, 8, 4);\n"
        "  s.set_schedule(s.autotune().best ? s.schedule() : hm_schedule{128, 2048, 128, 2048});\n"
        "  auto c = hm::computeMotifCounts(s);\n"
        "  std::vector<int64_t> d; s.update({1}, {1, 3}, {2}, &d);\n"
        "  s.findAndPrint({1, 2});\n"
        "  hm::TemporalWindow w(ctx, 3), w2(ctx, 3);\n"
        "  int keys[3] = {1, 2, 3}, st[3] = {0, 2, 4}, L[6] = {1, 2, 2, 3, 1, 3};\n"
        "  for (auto l : {hm::TemporalLayer::Older, hm::TemporalLayer::Middle, hm::TemporalLayer::Newest})\n"
        "    w.construct(l, keys, st, 3, L, 6);\n"
        "  w.fill(hm::TemporalLayer::Newest, {3}, {2}, {1});\n"
        "  w.unfill(hm::TemporalLayer::Newest, {3}, {1}, {1});\n"
        "  w.rotate(); w.resetNewest();\n"
        "  bool ok = hm::applyTemporalDeltasFromFile(\"d.txt\", w2) && w.size(hm::TemporalLayer::Older) == 3;\n"
        "  std::vector<int64_t> t; hm::computeTemporalMotifCountsStrictIncDelta(w, w2, t);\n"
        "  hm::computeTemporalMotifCountsStrictInc(w, t);\n"
        "  if (!ok) return 3;\n"
        "  return (int)c[0];\n"
        "}\n")
    out = tmp_path / "use_shim"
    r = subprocess.run([cxx, "-std=c++17", f"-I{ROOT / 'include'}", str(src), "-o", str(out),
                        f"-L{ROOT / 'ipdps26_b200'}", "-lhmotif", f"-Wl,-rpath,{ROOT / 'ipdps26_b200'}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert subprocess.run([str(out)]).returncode == 0


def test_struct_layouts_match_ctypes(tmp_path):
    """The ctypes mirrors in engine.py have the C structs' sizes and field
    offsets (checked by compiling a probe against include/hmotif.h)."""
    import ctypes as C
    import shutil
    import subprocess

    from ipdps26_b200 import engine

    cc = shutil.which("gcc")
    if cc is None:
        return
    structs = {
        "hm_graph_info_t": engine.GraphInfo, "hm_traffic_t": engine.Traffic, "hm_timings_t": engine.Timings,
        "hm_serve_config": engine.ServeConfig, "hm_serve_result": engine.ServeResult,
        "hm_serve_stats_t": engine.ServeStats, "hm_schedule": engine.Schedule, "hm_tune_report": engine.TuneReport,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "hmotif.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run([cc, f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, f, v = ln.split()
        got[(cname, f)] = int(v)
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_status_constants_match_header():
    from ipdps26_b200 import _lib

    text = (ROOT / "include" / "hmotif.h").read_text()
    for m in re.finditer(r"#define (HM_(?:OK|ERR_\w+))\s+\(?(-?\d+)\)?", text):
        assert getattr(_lib, m.group(1)) == int(m.group(2)), m.group(1)
