"""eggpu_b200 — a B200-native PageRank engine behind EasyGraph's ``eg.pagerank``.

Layers (host side mirrors the reference's PageRank path):
  * ``eggpu_b200.api``         ``pagerank(G, alpha, weight, max_iter, tol, personalization)``,
                               the drop-in for easygraph/functions/centrality/pagerank.py:12-72
  * ``eggpu_b200.backend``     prepared-graph cache and dense read-only results, the mirror of
                               easygraph/utils/gpu_eggpu_backend.py:254-348,636-704,1595-1821
  * ``eggpu_b200.bulk``        ``eggpu-csr-v1`` bulk CSR graphs (read_eggpu_csr)
  * ``eggpu_b200._native``     ctypes binding of libegpr.so (include/egpr.h)
  * ``eggpu_b200.synth``       seeded R-MAT / Erdos-Renyi workloads
  * ``eggpu_b200.serving``     continuous-batching request loop

The native library is imported lazily so that ``eggpu_b200.synth`` and the build
script work before ``libegpr.so`` exists; any solve fails loudly without it.
"""

__all__ = ["pagerank", "pagerank_batch", "install", "PreparedGraph"]


def __getattr__(name):
    if name in ("pagerank", "pagerank_batch", "install"):
        from . import api as _pr

        return getattr(_pr, name)
    if name == "PreparedGraph":
        from ._native import PreparedGraph

        return PreparedGraph
    raise AttributeError(name)
