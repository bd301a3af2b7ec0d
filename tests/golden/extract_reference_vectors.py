"""Extract the golden vectors of the reference's own unit tests into ``reference_vectors.json``.

    python tests/golden/extract_reference_vectors.py <path of the reference checkout>

(or set ``PACMAP_REFERENCE`` to that path). The tests never read the reference at run time: they use the
committed JSON.

Sources (beamform/pacmap-rs v0.2.6):
  * src/gradient.rs:162-195  test_pacmap_grad: y, pairs, weights -> 11x2 gradient incl. loss;
  * src/adam.rs:71-103       test_update_embedding_adam (file lines);
  * src/weights.rs:89-114    test_find_weight (file lines);
  * src/distance.rs:125-190  test_scale_dist / test_scale_dist_large;
  * src/knn.rs:259-324       exact-kNN known answers (normal case, duplicates, negatives).
"""
from __future__ import annotations

import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PACMAP_REFERENCE", "")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")


def _read(rel: str) -> str:
    if not REF:
        raise SystemExit("give the reference checkout's path as the first argument (or in PACMAP_REFERENCE)")
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def _array_literal(src: str, name: str, start: int = 0):
    """Parse `let [mut] name[: T] = array![ ... ];` (1-D or 2-D numeric) starting at offset `start`."""
    m = re.compile(r"let\s+(?:mut\s+)?" + re.escape(name) + r"\b[^=]*=\s*array!\[").search(src, start)
    if m is None:
        raise KeyError(name)
    i, depth = m.end(), 1
    while depth:
        depth += {"[": 1, "]": -1}.get(src[i], 0)
        i += 1
    body = re.sub(r"//[^\n]*", "", src[m.end():i - 1])
    rows = re.findall(r"\[([^\[\]]*)\]", body)
    num = r"-?\d+(?:\.\d+)?(?:[eE][-+]?\d+)?"
    if rows:
        return [[float(v) for v in re.findall(num, r)] for r in rows], i
    return [float(v) for v in re.findall(num, body)], i


def _scalar(src: str, name: str, start: int = 0) -> float:
    m = re.compile(r"let\s+" + re.escape(name) + r"\s*=\s*(-?\d+(?:\.\d+)?(?:[eE][-+]?\d+)?)").search(src, start)
    if m is None:
        raise KeyError(name)
    return float(m.group(1))


def main() -> int:
    out = {"source": "beamform/pacmap-rs v0.2.6 unit tests"}

    g = _read("src/gradient.rs")
    out["gradient"] = {
        "cite": "src/gradient.rs:162-195",
        "y": _array_literal(g, "y_test")[0],
        "pair_neighbors": _array_literal(g, "pair_neighbors")[0],
        "pair_mn": _array_literal(g, "pair_mn")[0],
        "pair_fp": _array_literal(g, "pair_fp")[0],
        "w_neighbors": _scalar(g, "w_neighbors"),
        "w_mn": _scalar(g, "w_mn"),
        "w_fp": _scalar(g, "w_fp"),
        "expected": _array_literal(g, "grad_python")[0],
        "eps": 1e-6,
    }

    a = _read("src/adam.rs")
    t0 = a.index("fn test_update_embedding_adam")
    out["adam"] = {
        "cite": "src/adam.rs:69-117 (file lines)",
        "y": _array_literal(a, "y", t0)[0],
        "grad": _array_literal(a, "grad", t0)[0],
        "beta1": _scalar(a, "beta1", t0),
        "beta2": _scalar(a, "beta2", t0),
        "lr": _scalar(a, "lr", t0),
        "itr": int(_scalar(a, "itr", t0)),
        "y_expected": _array_literal(a, "y_expected", t0)[0],
        "m_expected": _array_literal(a, "m_expected", t0)[0],
        "v_expected": _array_literal(a, "v_expected", t0)[0],
        "eps": 1e-6,
    }

    w = _read("src/weights.rs")
    calls = re.findall(r"let\s+w\d+\s*=\s*find_weights\(w_mn_init,\s*(\d+),\s*(\d+),\s*(\d+)\);", w)
    vals = re.findall(r"assert_abs_diff_eq!\(w\d+\.(w_mn|w_neighbors|w_fp),\s*(-?\d+(?:\.\d+)?)\)", w)
    cases = []
    for ci, (itr, p1, p2) in enumerate(calls):
        triple = {k: float(v) for k, v in vals[3 * ci:3 * ci + 3]}
        cases.append({"itr": int(itr), "p1": int(p1), "p2": int(p2), **triple})
    out["weights"] = {"cite": "src/weights.rs:89-114 (file lines)", "w_mn_init": _scalar(w, "w_mn_init"),
                      "cases": cases}

    d = _read("src/distance.rs")
    s0 = d.index("fn test_scale_dist()")
    s1 = d.index("fn test_scale_dist_large()")
    out["scale_dist_small"] = {
        "cite": "src/distance.rs:120-133",
        "knn_distances": _array_literal(d, "knn_distances", s0)[0],
        "sig": _array_literal(d, "sig", s0)[0],
        "neighbors": _array_literal(d, "neighbors", s0)[0],
        "expected": _array_literal(d, "expected", s0)[0],
        "exact": True,
    }
    out["scale_dist_large"] = {
        "cite": "src/distance.rs:135-190",
        "knn_distances": _array_literal(d, "knn_distances", s1)[0],
        "sig": _array_literal(d, "sig", s1)[0],
        "neighbors": _array_literal(d, "neighbors", s1)[0],
        "expected": _array_literal(d, "expected", s1)[0],
        "eps": 1e-6,
    }

    k = _read("src/knn.rs")
    knn_cases = {}
    for test in ("test_normal_case", "test_duplicate_embeddings", "test_negative_components"):
        t = k.index(f"fn {test}")
        emb = _array_literal(k, "embeddings", t)[0]
        kk = int(_scalar(k, "k", t))
        block_end = k.index("check_neighbors_and_distances", t)
        exp_src = k[k.index("let expected", t):block_end]
        expected = []
        for pm in re.finditer(r"\((\d+),\s*vec!\[((?:\([^)]*\),?\s*)*)\]\)", exp_src):
            pairs = re.findall(r"\((\d+),\s*([A-Z0-9_.]+)\)", pm.group(2))
            conv = []
            for idx, val in pairs:
                conv.append([int(idx), 0.7071067811865476 if val == "FRAC_1_SQRT_2" else float(val)])
            expected.append([int(pm.group(1)), conv])
        knn_cases[test] = {"embeddings": emb, "k": kk, "expected": expected}
    out["knn"] = {"cite": "src/knn.rs:257-324 (compare as index-sorted sets, distances eps 1e-4)",
                  "cases": knn_cases}

    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
