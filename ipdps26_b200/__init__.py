"""B200 hypergraph motif engine: exact MoCHy 26-motif and THyMe 96-motif
counts over a device-resident dynamic hypergraph store.

The compute path is libhmotif.so (hand-written sm_100a CUDA behind the C ABI
in include/hmotif.h). Submodules:
  engine  - Python view of the C ABI (context, graph, counts, batches)
  gen     - seeded synthetic workloads
  build   - nvcc build recipe for libhmotif.so
Importing ``engine`` or ``gen`` loads the library and fails loudly if it is
missing; this package module itself loads nothing so that ``build`` can run
before the library exists.
"""

__all__ = ["engine", "gen", "build"]
