"""``pagerank`` — the drop-in for EasyGraph's public PageRank entry.

Mirrors easygraph/functions/centrality/pagerank.py:12-72 (argument defaults,
environment defaults, multigraph rejection, empty graph -> ``{}``) and the
dispatch of :161-179, with two deliberate changes taken from the engine's
contract: an added ``personalization`` argument (appended last, so positional
callers are unaffected) and no silent CPU fallback — with
``EASYGRAPH_ENABLE_GPU`` on, a native failure raises.

:func:`install` puts this implementation behind an installed easygraph:
``easygraph.utils.gpu_eggpu_backend.pagerank`` (what the reference dispatch
calls under ``EASYGRAPH_ENABLE_GPU=TRUE``) and ``eg.pagerank`` itself (to
accept ``personalization``).  With the GPU switch off the installed wrapper
calls easygraph's own CPU implementation, as the reference does.
"""

from __future__ import annotations

import os

from . import backend

_TRUE_VALUES = {"1", "TRUE", "ON", "YES"}


def gpu_runtime_enabled():
    """easygraph/utils/gpu_runtime.py:10-11."""
    return os.environ.get("EASYGRAPH_ENABLE_GPU", "").strip().upper() in _TRUE_VALUES


def gpu_strict_errors():
    """easygraph/utils/gpu_runtime.py:14-15."""
    return os.environ.get("EASYGRAPH_GPU_STRICT_ERRORS", "").strip().upper() in _TRUE_VALUES


try:  # the reference's exception type when easygraph is importable
    from easygraph.utils.exception import EasyGraphNotImplemented  # type: ignore
except Exception:  # noqa: BLE001
    class EasyGraphNotImplemented(Exception):
        """Raised for graph types PageRank does not support (multigraphs)."""


def _effective_limits(max_iter, tol):
    """pagerank.py:45-52: env defaults EASYGRAPH_CPU_PR_MAX_ITER (200) and
    EASYGRAPH_CPU_PR_TOL (1e-6); max_iter >= 1, tol >= 0."""
    if max_iter is None:
        max_iter_eff = max(1, int(os.environ.get("EASYGRAPH_CPU_PR_MAX_ITER", "200")))
    else:
        max_iter_eff = max(1, int(max_iter))
    if tol is None:
        tol_eff = max(0.0, float(os.environ.get("EASYGRAPH_CPU_PR_TOL", "1e-6")))
    else:
        tol_eff = max(0.0, float(tol))
    return max_iter_eff, tol_eff


def _check_graph(G):
    is_multi = getattr(G, "is_multigraph", None)
    if callable(is_multi) and is_multi():
        raise EasyGraphNotImplemented("not implemented for multigraph type")


def pagerank(G, alpha=0.85, weight=None, max_iter=None, tol=None, personalization=None):
    """PageRank of every node of G on the GPU.

    G is an easygraph Graph/DiGraph (or any graph exposing ``nodes``,
    ``_adj``, ``is_directed()``, ``cache``) or a bulk CSR graph from
    :func:`eggpu_b200.bulk.read_eggpu_csr`.  Undirected graphs count each
    edge in both directions.  ``personalization`` (dict node -> weight >= 0,
    or an n-vector in node order) replaces the uniform teleport vector after
    normalisation; dangling mass is still spread uniformly.  Returns a
    read-only node -> float Mapping in node order (``dict(result)`` for a
    mutable copy).
    """
    _check_graph(G)
    max_iter_eff, tol_eff = _effective_limits(max_iter, tol)
    if len(G) == 0:
        return {}
    return backend.pagerank(G, alpha=alpha, max_iter=max_iter_eff, eps=tol_eff, weight=weight,
                            personalization=personalization)


def pagerank_batch(G, personalizations, alpha=0.85, weight=None, max_iter=None, tol=None):
    """Personalised PageRank for k teleport vectors in one batched solve; a list of Mappings."""
    _check_graph(G)
    max_iter_eff, tol_eff = _effective_limits(max_iter, tol)
    if len(G) == 0:
        return [{} for _ in range(len(personalizations))]
    return backend.pagerank_batch(G, personalizations, alpha=alpha, max_iter=max_iter_eff, eps=tol_eff,
                                  weight=weight)


_INSTALLED = {}


def install():
    """Routes an importable easygraph's PageRank through this engine.

    Returns True if easygraph was found and patched.  Patches:
      * easygraph.utils.gpu_eggpu_backend.pagerank(G, alpha, max_iter, eps, weight)
      * easygraph.functions.centrality.pagerank.pagerank and easygraph.pagerank,
        wrapped to accept ``personalization`` and to use this engine when
        EASYGRAPH_ENABLE_GPU is on (easygraph's own CPU code otherwise; C++
        graphs keep easygraph's routing to its C++ CPU PageRank).
    """
    import importlib

    try:
        import easygraph as eg  # type: ignore
        # the submodule itself: in easygraph the package attribute
        # easygraph.functions.centrality.pagerank is the re-exported function
        pr_mod = importlib.import_module("easygraph.functions.centrality.pagerank")
        eb = importlib.import_module("easygraph.utils.gpu_eggpu_backend")
    except Exception:  # noqa: BLE001
        return False
    if _INSTALLED:
        return True
    original = pr_mod.pagerank

    def backend_pagerank(G, alpha=0.85, max_iter=200, eps=1e-6, weight=None):
        return backend.pagerank(G, alpha=alpha, max_iter=max_iter, eps=eps, weight=weight)

    def eg_pagerank(G, alpha=0.85, weight=None, max_iter=None, tol=None, personalization=None):
        # C++ graphs (cflag) keep the reference's routing to cpp_pagerank
        # through its hybrid decorator (easygraph/utils/decorators.py:140-163),
        # with the GPU switch on or off; only a personalised solve, which that
        # path does not offer, comes to this engine.
        if getattr(G, "cflag", 0) and personalization is None:
            return original(G, alpha=alpha, weight=weight, max_iter=max_iter, tol=tol)
        if gpu_runtime_enabled():
            return pagerank(G, alpha=alpha, weight=weight, max_iter=max_iter, tol=tol,
                            personalization=personalization)
        if personalization is not None:
            raise ValueError("personalization needs the GPU engine (EASYGRAPH_ENABLE_GPU=TRUE)")
        return original(G, alpha=alpha, weight=weight, max_iter=max_iter, tol=tol)

    _INSTALLED.update(original=original, backend=eb.pagerank)
    eb.pagerank = backend_pagerank
    pr_mod.pagerank = eg_pagerank
    eg.pagerank = eg_pagerank
    # the re-exports of the function on the package path
    for path in ("functions", "functions.centrality"):
        obj = eg
        for part in path.split("."):
            obj = getattr(obj, part, None)
            if obj is None:
                break
        if obj is not None and getattr(obj, "pagerank", None) is original:
            try:
                obj.pagerank = eg_pagerank
            except Exception:  # noqa: BLE001
                pass
    return True
