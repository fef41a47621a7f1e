"""Direct-curvature PCG restated in Python (test infrastructure only: the oracle).

Follows solveOctreePipelinedPCG in
lib/methods/octree-shared/octree-pipelined-pcg.ts:305-594, with the linear-map
audit (:184-230), the Neumaier dot (:146-158) and the merged reduction
(:232-265).  Pure-Python loops: for the small known-answer systems of the
reference's tests/octree-pipelined-pcg.test.ts only.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field


def neumaier_dot(a, b) -> float:
    s, c = 0.0, 0.0
    for x, y in zip(a, b):
        p = x * y
        n = s + p
        c += (s - n) + p if abs(s) >= abs(p) else (p - n) + s
        s = n
    return s + c


def norm(v) -> float:
    return math.sqrt(max(0.0, neumaier_dot(v, v)))


def _close(a, b, tol) -> bool:
    return abs(a - b) <= tol * max(1.0, abs(a), abs(b))


def _finite_map(fn, x):
    out = fn(list(x))
    if out is None or len(out) != len(x):
        return None
    out = [float(v) for v in out]
    if not all(math.isfinite(v) for v in out):
        return None
    return out


def _probes(n):
    first = [((i * 17 + 5) % 23) - 11 for i in range(n)]
    second = [((i * 29 + 3) % 19) - 9 for i in range(n)]
    return [float(v) for v in first], [float(v) for v in second]


def _audit(fn, n, tol, role):
    first, second = _probes(n)
    comb = [a - 0.375 * b for a, b in zip(first, second)]
    fi, fi2, se, co, ze = (_finite_map(fn, v) for v in (first, first, second, comb, [0.0] * n))
    if None in (fi, fi2, se, co, ze):
        return "non-finite-map-output"
    exp = [a - 0.375 * b for a, b in zip(fi, se)]
    if not (all(_close(a, b, tol) for a, b in zip(fi, fi2)) and all(_close(a, b, tol) for a, b in zip(co, exp))
            and all(_close(a, 0.0, tol) for a in ze)):
        return f"{role}-is-not-linear"
    if not _close(neumaier_dot(first, se), neumaier_dot(second, fi), tol):
        return f"{role}-is-not-symmetric"
    if not (neumaier_dot(first, fi) > 0 and neumaier_dot(second, se) > 0):
        return f"{role}-is-not-positive"
    return None


def _merge(r, z, az=None):
    def acc(s, c, v):
        n = s + v
        return n, c + ((s - n) + v if abs(s) >= abs(v) else (v - n) + s)
    g = gc = d = dc = rr = rc = 0.0
    for k in range(len(r)):
        g, gc = acc(g, gc, r[k] * z[k])
        if az is not None:
            d, dc = acc(d, dc, z[k] * az[k])
        rr, rc = acc(rr, rc, r[k] * r[k])
    return g + gc, d + dc, rr + rc


@dataclass
class Result:
    accepted: bool
    solution: list
    residual: list
    converged: bool
    iterations: int
    reductions: int
    residual_norm: float
    stopping_threshold: float
    failure: str | None = None
    history: list = field(default_factory=list)


def solve(rhs, apply_operator, apply_preconditioner=None, initial_guess=None, maximum_iterations=None,
          relative_tolerance=1e-10, absolute_tolerance=0.0, validate=True, validation_tolerance=2e-12) -> Result:
    n = len(rhs)
    if n < 1:
        raise ValueError("Pipelined PCG requires at least one row")
    b = [float(v) for v in rhs]
    if not all(math.isfinite(v) for v in b):
        raise ValueError("right-hand side contains a non-finite value")
    if initial_guess is not None and len(initial_guess) != n:
        raise ValueError(f"initial guess must have length {n}")
    x = [float(v) for v in initial_guess] if initial_guess is not None else [0.0] * n
    maxit = n if maximum_iterations is None else maximum_iterations
    for name, v in (("relativeTolerance", relative_tolerance), ("absoluteTolerance", absolute_tolerance)):
        if not math.isfinite(v) or v < 0:
            raise ValueError(f"{name} must be finite and non-negative")
    prec = apply_preconditioner or (lambda v: v)

    def reject(res, it, red, thr, failure, hist):
        return Result(False, x, res, False, it, red, norm(res), thr, failure, hist)

    if validate:
        f = _audit(apply_operator, n, validation_tolerance, "operator")
        if f:
            return reject(list(b), 0, 0, 0.0, f, [])
        f = _audit(prec, n, validation_tolerance, "preconditioner")
        if f:
            ax = _finite_map(apply_operator, x) or [0.0] * n
            return reject([bi - ai for bi, ai in zip(b, ax)], 0, 0, 0.0, f, [])
    ax = _finite_map(apply_operator, x)
    r = [bi - ai for bi, ai in zip(b, ax)]
    bnorm = norm(b)
    thr = max(absolute_tolerance, relative_tolerance * max(bnorm, 5e-324))
    z = _finite_map(prec, r)
    az = _finite_map(apply_operator, z)
    g, d, rr = _merge(r, z, az)
    red, it = 1, 0
    rec = math.sqrt(max(0.0, rr))
    hist = [(0, red, rec)]
    if rec <= thr:
        return Result(True, x, r, True, 0, red, rec, thr, None, hist)
    if not (g > 0):
        return reject(r, it, red, thr, "non-positive-preconditioned-residual", hist)
    if not (d > 0):
        return reject(r, it, red, thr, "non-positive-direction-curvature", hist)
    alpha = g / d
    dirn, adir = list(z), list(az)
    while it < maxit:
        for k in range(n):
            x[k] += alpha * dirn[k]
            r[k] -= alpha * adir[k]
        it += 1
        z = _finite_map(prec, r)
        gn, _, rr = _merge(r, z)
        red += 1
        rec = math.sqrt(max(0.0, rr))
        hist.append((it, red, rec))
        if rec <= thr:
            ax = _finite_map(apply_operator, x)
            tr = [bi - ai for bi, ai in zip(b, ax)]
            if norm(tr) > thr:
                return reject(tr, it, red, thr, "true-residual-validation", hist)
            return Result(True, x, tr, True, it, red, norm(tr), thr, None, hist)
        if not (gn > 0):
            return reject(r, it, red, thr, "non-positive-preconditioned-residual", hist)
        if it >= maxit:
            ax = _finite_map(apply_operator, x)
            return reject([bi - ai for bi, ai in zip(b, ax)], it, red, thr, "maximum-iterations", hist)
        beta = gn / g
        dirn = [zk + beta * dk for zk, dk in zip(z, dirn)]
        adir = _finite_map(apply_operator, dirn)
        den = neumaier_dot(dirn, adir)
        red += 1
        if not (den > 0):
            return reject(r, it, red, thr, "non-positive-direction-curvature", hist)
        alpha = gn / den
        g = gn
    ax = _finite_map(apply_operator, x)
    return reject([bi - ai for bi, ai in zip(b, ax)], it, red, thr, "maximum-iterations", hist)
