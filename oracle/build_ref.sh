#!/usr/bin/env bash
# Compiles the reference's own exact CPU counters, straight from the reference
# sources, into oracle/_ref/ (git-ignored). These are the pins for the C
# restatement in hm_oracle.c and the timed CPU baseline. Nothing is copied:
# g++ reads the sources where they lie.
#   MoCHy-master/main_exact.cpp       -> _ref/mochy_exact
#   MoCHy-master/main_exact_par.cpp   -> _ref/mochy_exact_par   (OpenMP)
#   THyMe-main/code/main_thyme.cpp    -> _ref/thyme
#   THyMe-main/code/main_thymeP.cpp   -> _ref/thymeP            (OpenMP)
#   temporalDynamicHMotif/src/type{1,2,3}.cpp, through the harness
#   ref_types.cpp (its main renamed), with graphGeneration.cpp and utils/
#                                     -> _ref/type1, type2, type3
set -euo pipefail
REF=${HM_REFERENCE_ROOT:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -d "$REF/MoCHy-master" ] || [ ! -d "$REF/THyMe-main/code" ]; then
  echo "build_ref.sh: reference tree not found at $REF; keeping existing _ref/" >&2
  exit 0
fi
mkdir -p "$OUT"
# The system g++ carries libgomp; a bare $CXX from the environment may not.
CXX=${HM_REF_CXX:-$( [ -x /usr/bin/g++ ] && echo /usr/bin/g++ || echo g++ )}
$CXX -O3 -std=c++11 -o "$OUT/mochy_exact" "$REF/MoCHy-master/main_exact.cpp"
$CXX -O3 -std=c++11 -fopenmp -o "$OUT/mochy_exact_par" "$REF/MoCHy-master/main_exact_par.cpp"
$CXX -O3 -std=c++11 -o "$OUT/thyme" "$REF/THyMe-main/code/main_thyme.cpp"
$CXX -O3 -std=c++11 -fopenmp -o "$OUT/thymeP" "$REF/THyMe-main/code/main_thymeP.cpp"
TD="$REF/temporalDynamicHMotif"
if [ -d "$TD/src" ]; then
  for t in 1 2 3; do
    $CXX -O2 -std=c++17 -DHM_TYPE=$t -I"$TD" -o "$OUT/type$t" "$HERE/ref_types.cpp" "$TD/src/graphGeneration.cpp" \
      "$TD/utils/utils.cpp" "$TD/utils/printUtils.cpp" "$TD/utils/flatten.cpp"
  done
  # The reference's strictly increasing temporal counter (CUDA) with its store,
  # through the harness ref_strictinc.cu -> _ref/strictinc (sm_100a).
  # operations.cu uses std::sort without including <algorithm>; the header is
  # pre-included rather than the source changed.
  NVCC=${NVCC:-$(command -v nvcc || echo /usr/local/cuda/bin/nvcc)}
  if [ -x "$NVCC" ]; then
    "$NVCC" -std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a --pre-include algorithm \
      -I"$TD/include" -I"$TD/kernel" \
      -o "$OUT/strictinc" "$HERE/ref_strictinc.cu" "$TD/src/temporal_count.cu" "$TD/src/temporal_structure.cpp" \
      "$TD/structure/operations.cu" "$TD/kernel/insert_reuse.cu" "$TD/kernel/unfill.cu" "$TD/kernel/payload.cu" \
      "$TD/kernel/build_tree.cu" "$TD/kernel/delete_avail.cu" "$TD/kernel/find.cu" "$TD/utils/flatten.cpp" \
      "$TD/utils/utils.cpp" "$TD/utils/printUtils.cpp" "$TD/src/graphGeneration.cpp" 2>/dev/null ||
      echo "build_ref.sh: the strict-increasing counter did not build; its parity test will skip" >&2
  fi
fi
# The reference's own datasets with known outputs, copied verbatim for the
# parity tests (refdata.py): MoCHy's dblp sample and THyMe's email-Enron with
# its shipped results at delta = 86,400,000.
mkdir -p "$OUT/data"
for f in MoCHy-master/dblp_graph.txt THyMe-main/data/email-Enron-full/email-Enron-full.txt \
    THyMe-main/results/email-Enron-full_86400000.000000_thyme.txt \
    THyMe-main/results/email-Enron-full_86400000.000000_thymeP.txt \
    THyMe-main/results/email-Enron-full_86400000.000000_dp.txt; do
  if [ -f "$REF/$f" ]; then cp "$REF/$f" "$OUT/data/"; fi
done
echo "build_ref.sh: built $(ls "$OUT" | tr '\n' ' ')"
