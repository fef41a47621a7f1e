"""Writes tests/golden/pcg_kat.json: the known-answer cases of the reference's
tests/octree-pipelined-pcg.test.ts, restated as data plus expected outcomes.

The reference cannot run here (TypeScript, no Node), so the expected values are
recomputed with independent methods: the conventional PCG the reference test
itself compares against (octree-pipelined-pcg.test.ts:17-40) and numpy's dense
solve.  Every case cites the test it comes from.

    python tests/golden/make_golden.py
"""
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def conventional_pcg(A, inv_diag, b):
    """octree-pipelined-pcg.test.ts:17-40: plain PCG, stops when ||r|| < 1e-13."""
    A = np.asarray(A, float)
    x = np.zeros(len(b))
    r = np.array(b, float)
    z = inv_diag * r
    d = z.copy()
    g = float(r @ z)
    for _ in range(len(b)):
        q = A @ d
        a = g / float(d @ q)
        x += a * d
        r -= a * q
        z = inv_diag * r
        gn = float(r @ z)
        if math.sqrt(float(r @ r)) < 1e-13:
            break
        d = z + (gn / g) * d
        g = gn
    return x


def main():
    cases = []
    # octree-pipelined-pcg.test.ts:42-70
    A = [[7, -2, 0, 0, 0], [-2, 6, -1, 0, 0], [0, -1, 5, -1, 0], [0, 0, -1, 4, -1], [0, 0, 0, -1, 3]]
    b = [1.25, -0.75, 2.5, 0.125, -1.5]
    inv = 1.0 / np.diag(np.asarray(A, float))
    cases.append({
        "name": "conventional-spd-5x5", "source": "tests/octree-pipelined-pcg.test.ts:42-70",
        "A": A, "b": b, "preconditioner": "jacobi", "max_iterations": 10, "relative_tolerance": 1e-12,
        "expect": {"accepted": True, "max_iterations_used": 5, "reductions": "2*iterations (min 1)",
                   "solution": conventional_pcg(A, inv, b).tolist(), "solution_tol": 2e-12,
                   "dense_solution": np.linalg.solve(np.asarray(A, float), b).tolist()},
    })
    # octree-pipelined-pcg.test.ts:72-97
    n = 17
    fw = [0.75 + ((f * 13) % 11) / 9 for f in range(n + 1)]
    M = np.zeros((n, n))
    for r in range(n):
        M[r, r] = fw[r] + fw[r + 1] + 0.2
        if r > 0:
            M[r, r - 1] = -fw[r]
        if r + 1 < n:
            M[r, r + 1] = -fw[r + 1]
    man = np.array([math.sin((r + 1) * 0.37) + 0.2 * math.cos((r + 1) * 0.91) for r in range(n)])
    cases.append({
        "name": "manufactured-poisson-17", "source": "tests/octree-pipelined-pcg.test.ts:72-97",
        "A": M.tolist(), "b": (M @ man).tolist(), "preconditioner": "jacobi", "max_iterations": 40,
        "relative_tolerance": 5e-13,
        "expect": {"accepted": True, "reductions": "2*iterations", "solution": man.tolist(), "solution_tol": 2e-11},
    })
    # octree-pipelined-pcg.test.ts:99-114
    A2 = np.array([[3.0, -1.0], [-1.0, 2.0]])
    sol = np.array([0.75, -1.25])
    cases.append({
        "name": "initial-guess-accepted", "source": "tests/octree-pipelined-pcg.test.ts:99-114",
        "A": A2.tolist(), "b": (A2 @ sol).tolist(), "preconditioner": "identity", "initial_guess": sol.tolist(),
        "relative_tolerance": 1e-14,
        "expect": {"accepted": True, "iterations": 0, "reductions": 1, "residual_norm": 0.0},
    })
    # octree-pipelined-pcg.test.ts:116-127
    cases.append({
        "name": "non-linear-preconditioner", "source": "tests/octree-pipelined-pcg.test.ts:116-127",
        "A": [[4, -1, 0], [-1, 3, -1], [0, -1, 2]], "b": [1, 2, -1], "preconditioner": "v*abs(v)",
        "expect": {"accepted": False, "failure": "preconditioner-is-not-linear", "iterations": 0, "reductions": 0},
    })
    # octree-pipelined-pcg.test.ts:129-147
    cases.append({
        "name": "indefinite-operator", "source": "tests/octree-pipelined-pcg.test.ts:129-136",
        "A": [[1, 0], [0, -1]], "b": [1, 0], "preconditioner": "identity",
        "expect": {"accepted": False, "failure": "operator-is-not-positive", "iterations": 0},
    })
    cases.append({
        "name": "exhausted-budget", "source": "tests/octree-pipelined-pcg.test.ts:138-147",
        "A": [[4, -1, 0], [-1, 4, -1], [0, -1, 3]], "b": [1, 2, 3], "preconditioner": "identity",
        "max_iterations": 1, "relative_tolerance": 1e-15,
        "expect": {"accepted": False, "failure": "maximum-iterations", "iterations": 1, "reductions": 2},
    })
    # octree-pipelined-pcg.test.ts:149-165
    cases.append({
        "name": "malformed-inputs", "source": "tests/octree-pipelined-pcg.test.ts:149-165",
        "raises": [{"b": [1, "nan"], "match": "non-finite"},
                   {"b": [1, 2], "initial_guess": [0], "match": "length 2"},
                   {"b": [1], "relative_tolerance": -1, "match": "non-negative"}],
    })
    with open(os.path.join(HERE, "pcg_kat.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=1)


if __name__ == "__main__":
    main()
