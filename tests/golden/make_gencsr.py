"""Writes tests/golden/gencsr_ref.npz: out-edge CSRs made by the reference's
own C++ graph code.

Each case is an easygraph graph built by the reference's Python package (node
and edge insertion orders shuffled, undirected duplicates and self-loops
included, weights on part of the edges), converted by the reference's
build_digraph / build_graph (cpp_easygraph/classes/graph_convert.cpp:72-134)
and turned into a CSR by Graph::gen_CSR (cpp_easygraph/classes/graph.cpp:
719-886), compiled from the reference sources by oracle/Makefile.gencsr into
oracle/_ref/.  The fixture keeps the insertion orders, so the tests rebuild the
same graphs without the reference.

    python tests/golden/make_gencsr.py [REFERENCE_ROOT]
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT))


def cases():
    """(name, directed, nodes in insertion order, edges (u, v) in insertion order,
    per-edge weight or nan for an edge without the attribute, weight key)."""
    from eggpu_b200 import synth

    rng = np.random.Generator(np.random.PCG64(12))
    out = []
    for directed in (True, False):
        g = synth.rmat(scale=12, edgefactor=8, seed=12 + directed)
        src = np.repeat(np.arange(g.n), np.diff(g.V))
        edges = np.stack([src, g.E], 1)
        if not directed:  # both directions, duplicates and self-loops, as a caller adds them
            extra = edges[rng.random(len(edges)) < 0.3][:, ::-1]
            loops = np.repeat(rng.integers(0, g.n, 40)[:, None], 2, 1)
            edges = np.concatenate([edges, extra, loops])
        edges = edges[rng.permutation(len(edges))]
        nodes = rng.permutation(g.n)
        w = np.where(rng.random(len(edges)) < 0.8, rng.integers(1, 64, len(edges)) / 16.0, np.nan)
        kind = "digraph" if directed else "graph"
        out.append((f"rmat12_{kind}", directed, nodes, edges, None, None))
        out.append((f"rmat12_{kind}_weighted", directed, nodes, edges, w, "weight"))
    # nodes that are only edge endpoints come after the listed ones
    out.append(("endpoints_only", True, np.array([7, 3]), np.array([[3, 9], [9, 7], [11, 3], [7, 7]]), None, None))
    return out


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else None
    sys.argv = sys.argv[:1] if ref_root is None else [sys.argv[0], ref_root]
    import make_golden

    subprocess.run(["make", "-s", "-f", str(ROOT / "oracle" / "Makefile.gencsr"),
                    f"REFERENCE_ROOT={make_golden.REF_ROOT}"], check=True, cwd=str(ROOT))
    eg, _ = make_golden._import_reference()
    sys.path.insert(0, str(ROOT / "oracle" / "_ref"))
    import _ref_gencsr

    arrays = {}
    for name, directed, nodes, edges, w, key in cases():
        G = eg.DiGraph() if directed else eg.Graph()
        G.add_nodes([int(v) for v in nodes])
        if w is None:
            G.add_edges([(int(a), int(b)) for a, b in edges])
        else:
            G.add_edges([(int(a), int(b)) for a, b in edges],
                        edges_attr=[{} if np.isnan(x) else {key: float(x)} for x in w])
        V, E, W = _ref_gencsr.gen_csr(G, directed, key)
        arrays[f"{name}/directed"] = np.array([directed])
        arrays[f"{name}/nodes"] = np.asarray(nodes, np.int32)
        arrays[f"{name}/edges"] = np.asarray(edges, np.int32)
        if w is not None:
            arrays[f"{name}/w"] = np.asarray(w, np.float64)
        arrays[f"{name}/V"] = V
        arrays[f"{name}/E"] = E
        if W is not None:
            arrays[f"{name}/W"] = W
    np.savez_compressed(HERE / "gencsr_ref.npz", **arrays)
    print("wrote", HERE / "gencsr_ref.npz", sorted({k.split("/")[0] for k in arrays}))


if __name__ == "__main__":
    main()
