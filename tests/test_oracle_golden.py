"""The oracle's PCG recurrence against the reference's known-answer tests
(tests/octree-pipelined-pcg.test.ts, restated in tests/golden/pcg_kat.json)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import pcg
from oracle.oracle import pcg_dense

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pcg_kat.json")))
CASES = {c["name"]: c for c in GOLDEN["cases"]}


def _maps(case):
    A = np.asarray(case["A"], float)
    op = lambda v: (A @ np.asarray(v, float)).tolist()
    kind = case.get("preconditioner", "identity")
    if kind == "jacobi":
        inv = 1.0 / np.diag(A)
        pre = lambda v: (inv * np.asarray(v, float)).tolist()
    elif kind == "v*abs(v)":
        pre = lambda v: [x * abs(x) for x in v]
    else:
        pre = None
    return A, op, pre


def _solve_py(case):
    A, op, pre = _maps(case)
    return pcg.solve(case["b"], op, pre, initial_guess=case.get("initial_guess"),
                     maximum_iterations=case.get("max_iterations"),
                     relative_tolerance=case.get("relative_tolerance", 1e-10))


@pytest.mark.parametrize("name", ["conventional-spd-5x5", "manufactured-poisson-17", "initial-guess-accepted",
                                  "non-linear-preconditioner", "indefinite-operator", "exhausted-budget"])
def test_python_restatement_matches_reference_assertions(name):
    case = CASES[name]
    exp = case["expect"]
    res = _solve_py(case)
    assert res.accepted == exp["accepted"], res.failure
    if "failure" in exp:
        assert res.failure == exp["failure"]
    if "iterations" in exp:
        assert res.iterations == exp["iterations"]
    if exp.get("reductions") == "2*iterations (min 1)":
        assert res.reductions == max(1, 2 * res.iterations)
        assert len(res.history) == res.iterations + 1
    elif exp.get("reductions") == "2*iterations":
        assert res.reductions == 2 * res.iterations
        assert [h[0] for h in res.history] == list(range(len(res.history)))
    elif "reductions" in exp:
        assert res.reductions == exp["reductions"]
    if "max_iterations_used" in exp:
        assert res.iterations <= exp["max_iterations_used"]
    if "solution" in exp:
        assert max(abs(a - b) for a, b in zip(res.solution, exp["solution"])) < exp["solution_tol"]
        assert res.residual_norm <= res.stopping_threshold
    if "residual_norm" in exp:
        assert res.residual_norm == exp["residual_norm"]
    if name == "exhausted-budget":
        assert res.residual_norm > res.stopping_threshold


def test_python_restatement_rejects_malformed_inputs():
    op = lambda v: v
    for spec in CASES["malformed-inputs"]["raises"]:
        b = [float(x) for x in spec["b"]]
        with pytest.raises(ValueError, match=spec["match"]):
            pcg.solve(b, op, initial_guess=spec.get("initial_guess"),
                      relative_tolerance=spec.get("relative_tolerance", 1e-10))


@pytest.mark.parametrize("name", ["conventional-spd-5x5", "manufactured-poisson-17", "initial-guess-accepted",
                                  "exhausted-budget"])
def test_cpp_oracle_recurrence_matches_reference_assertions(name):
    """The C++ recurrence behind the grid oracle (no map audit in C++; audits are Python's)."""
    case = CASES[name]
    exp = case["expect"]
    A = np.asarray(case["A"], float)
    minv = 1.0 / np.diag(A) if case.get("preconditioner") == "jacobi" else None
    x, info = pcg_dense(A, case["b"], minv=minv, x0=case.get("initial_guess"),
                        max_iter=case.get("max_iterations", len(case["b"])),
                        rel_tol=case.get("relative_tolerance", 1e-10))
    assert (info["failure_name"] is None) == exp["accepted"]
    if "failure" in exp:
        assert info["failure_name"] == exp["failure"]
    if "iterations" in exp:
        assert info["iterations"] == exp["iterations"]
    if exp.get("reductions") == "2*iterations (min 1)":
        assert info["reductions"] == max(1, 2 * info["iterations"])
    elif exp.get("reductions") == "2*iterations":
        assert info["reductions"] == 2 * info["iterations"]
    elif "reductions" in exp:
        assert info["reductions"] == exp["reductions"]
    if "solution" in exp:
        assert np.abs(x - np.asarray(exp["solution"])).max() < exp["solution_tol"]
    py = _solve_py(case)
    assert py.iterations == info["iterations"]
    np.testing.assert_allclose(x, py.solution, rtol=0, atol=1e-13 * max(1.0, np.abs(x).max()))


def test_golden_fixture_generator_is_reproducible(tmp_path):
    import importlib.util
    import shutil
    src = os.path.join(os.path.dirname(__file__), "golden", "make_golden.py")
    spec = importlib.util.spec_from_file_location("mg", src)
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    mg.HERE = str(tmp_path)
    mg.main()
    regen = json.load(open(tmp_path / "pcg_kat.json"))
    assert regen == GOLDEN
