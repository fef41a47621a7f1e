"""Parity of the CUDA tall-cell projection against the float64 tall-cell oracle (GPU)."""
import numpy as np
import pytest

from fluid_b200 import configs
from fluid_b200.tall import TallProjector
from oracle import tall as oracle

pytestmark = pytest.mark.gpu

REL_L2_PRESSURE = 1e-5
REL_RES = 1e-6
# The tall layout's weakest mode (a near-constant pressure offset, coupled to the
# free surface through tall cells hundreds of rows high) lets a relative
# residual of 1e-6 leave a pressure error of about 2e-5 against the float64
# solution (measured at 256^2 x 1024: 2.0e-5 at 1e-6, 2.5e-6 at 1e-8, with the
# true residual evaluated in float64).  The parity tests therefore solve to
# 1e-7; the bench states the float64 error at its 1e-6 operating point.
REL_RES_PARITY = 1e-7

CASES = {
    "waves12x10": lambda: configs.tall_waves(12, 10, 64, 16, seed=21, mean=30, amp_max=4, lam=(4, 16),
                                             quality="balanced"),
    "waves20x14_b24": lambda: configs.tall_waves(20, 14, 96, 24, seed=22, mean=50, amp_max=6, lam=(6, 30),
                                                 quality="high"),
}


def _pair(s):
    tp = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
    tp.upload_state(s.vof, s.u, s.v, s.w)
    g = oracle.TallGrid(s.nx, s.fine_ny, s.nz, s.band, s.bases)
    g.set_state(s.vof, s.u, s.v, s.w)
    return tp, g


@pytest.mark.parametrize("name", sorted(CASES))
def test_tall_labels_rhs_operator(name):
    s = CASES[name]()
    tp, g = _pair(s)
    tp.prepare(s.dt)
    lab_o = g.liquid_samples()
    np.testing.assert_array_equal(tp.labels(0).reshape(lab_o.shape), lab_o.astype(np.uint8))
    b_o = g.rhs().reshape(tp.shape)
    b_d = tp.rhs()
    assert np.abs(b_d - b_o).max() <= 1e-5 * np.abs(b_o).max()
    A = g.operator()
    rng = np.random.default_rng(3)
    p = (rng.normal(size=tp.shape) * lab_o).astype(np.float32)
    ap_o = (A @ p.ravel().astype(np.float64)) * lab_o.ravel()
    ap_d = tp.apply_operator(p).ravel()
    assert np.linalg.norm(ap_d - ap_o) <= 1e-6 * np.linalg.norm(ap_o)


@pytest.mark.parametrize("name", sorted(CASES))
def test_tall_project_matches_oracle(name):
    s = CASES[name]()
    tp, g = _pair(s)
    rec = tp.project(s.dt, rel_tol=REL_RES_PARITY)
    assert rec["status_name"] == "OK", rec
    assert rec["true_rel_residual"] <= REL_RES_PARITY
    assert rec["levels"] >= 2
    p_o, _, _ = g.solve()
    p_d = tp.pressure().ravel().astype(np.float64)
    assert np.linalg.norm(p_d - p_o) <= REL_L2_PRESSURE * np.linalg.norm(p_o)
    u_o, v_o, w_o = g.grad_subtract(p_o)
    p_si, u, v, w = tp.download()
    scale = max(np.abs(u_o).max(), np.abs(v_o).max(), np.abs(w_o).max())
    for dev, ref in ((u, u_o), (v, v_o), (w, w_o)):
        assert np.abs(dev - ref).max() <= 1e-4 * scale
    assert rec["max_div_after"] <= 1e-5 * rec["max_div_before"], rec


@pytest.fixture(scope="module")
def full_size_tall():
    """The 256^2 x 1024 wave tank (2.23M samples) with its float64 operator and
    right-hand side assembled by the oracle from the dense faces."""
    s = configs.tall_waves()
    A, b = oracle.assemble_fp64(s.nx, s.fine_ny, s.nz, s.band, s.bases, s.vof, s.u, s.v, s.w)
    return s, A, b


def fp64_solution(tp, s, A, b, max_steps=12):
    """The float64 solution of the oracle's system A x = b by iterative
    refinement: float64 residuals with the oracle's operator, corrections from
    the device MGPCG.  Returns x and ||b - A x|| / ||b|| (certified in float64)."""
    x = np.zeros_like(b)
    nb = np.linalg.norm(b)
    rel = 1.0
    for _ in range(max_steps):
        r = b - A @ x
        rel = np.linalg.norm(r) / nb
        if rel <= 1e-12:
            break
        e, rec = tp.solve_rhs(s.dt, r.astype(np.float32), rel_tol=REL_RES)
        assert rec["status_name"] in ("OK", "NONCONVERGENCE"), rec
        x += e.ravel().astype(np.float64)
    return x, rel


def test_tall_full_size_labels_rhs_operator(full_size_tall):
    s, A, b = full_size_tall
    tp = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
    tp.upload_state(s.vof, s.u, s.v, s.w)
    tp.prepare(s.dt)
    # liquid samples: vof > 0.5 on active band rows; a tall segment follows its bottom sample
    rows = configs.tall_sample_rows(s.bases, s.band)
    lab = (s.vof > 0.5) & (rows < s.fine_ny)
    lab[:, 1, :] = lab[:, 0, :]
    np.testing.assert_array_equal(tp.labels(0).reshape(lab.shape), lab.astype(np.uint8))
    b_d = tp.rhs().ravel()
    assert np.abs(b_d - b).max() <= 1e-5 * np.abs(b).max()
    p = (np.random.default_rng(3).normal(size=tp.shape) * lab).astype(np.float32)
    ap_o = A @ p.ravel().astype(np.float64)
    ap_d = tp.apply_operator(p).ravel()
    assert np.linalg.norm(ap_d - ap_o) <= 1e-6 * np.linalg.norm(ap_o)
    tp.destroy()


@pytest.fixture(scope="module")
def full_size_tall_solution(full_size_tall):
    """The float64 solution of the full-size system (iterative refinement with
    float32-level device corrections), certified by its float64 residual."""
    s, A, b = full_size_tall
    tp = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
    tp.upload_state(s.vof, s.u, s.v, s.w)
    x, rel = fp64_solution(tp, s, A, b)
    tp.destroy()
    assert rel <= 1e-12, rel
    return x


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
def test_tall_full_size_matches_fp64(full_size_tall, full_size_tall_solution, precision):
    """The 2.23M-sample projection with every level storage type against the
    float64 solution of the oracle's independently assembled system: receipts
    at the 1e-6 operating point, divergence over represented band cells
    reduced by 1e-4, and at the parity tolerance pressure rel-L2 <= 1e-5.
    Levels 1-2 are grid levels here, so fp16 / bf16 change their storage."""
    s, A, b = full_size_tall
    x = full_size_tall_solution
    tp = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho, precision=precision)
    tp.upload_state(s.vof, s.u, s.v, s.w)
    rec = tp.project(s.dt, rel_tol=REL_RES)
    assert rec["status_name"] == "OK", rec
    assert rec["true_rel_residual"] <= REL_RES
    assert rec["levels"] == 7
    assert rec["max_div_after"] <= 1e-4 * rec["max_div_before"], rec
    tp.upload_state(s.vof, s.u, s.v, s.w)
    rec = tp.project(s.dt, rel_tol=REL_RES_PARITY)
    assert rec["status_name"] == "OK", rec
    p_d = tp.pressure().ravel().astype(np.float64)
    err = np.linalg.norm(p_d - x) / np.linalg.norm(x)
    assert err <= REL_L2_PRESSURE, (precision, err)
    tp.destroy()


@pytest.mark.parametrize("shape,precision", [((20, 20, 96, 24), "fp32"), ((64, 64, 128, 16), "fp16")])
def test_tall_sliced_projection_matches_one_call(shape, precision):
    """begin + continue in slices of 3 iterations + end (the one-iteration graph
    replayed) gives the one-call result (the whole loop as one graph) bit for
    bit; the 64^2 case has grid level 1 in fp16."""
    nx, nz, fny, band = shape
    s = configs.tall_waves(nx, nz, fny, band, seed=2, mean=fny // 2, amp_max=4, lam=(8, 32))
    a = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho, precision=precision)
    a.upload_state(s.vof, s.u, s.v, s.w)
    ra = a.project(s.dt, rel_tol=1e-6)
    b = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho, precision=precision)
    b.upload_state(s.vof, s.u, s.v, s.w)
    b.project_begin(s.dt, rel_tol=1e-6)
    slices = 1
    while not b.project_continue(3):
        slices += 1
    rb = b.project_end()
    assert slices >= 2
    assert ra["iterations"] == rb["iterations"] and rb["status_name"] == "OK"
    np.testing.assert_array_equal(a.pressure(), b.pressure())
    a.destroy()
    b.destroy()


def test_tall_direct_launches_match_the_graphs():
    """With graphs off (one launch per kernel, as a profiler needs) the solve
    runs the same kernels in the same order: same iterations, same bits."""
    s = configs.tall_waves(48, 40, 128, 16, seed=4, mean=64, amp_max=4, lam=(8, 32))
    a = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
    a.upload_state(s.vof, s.u, s.v, s.w)
    ra = a.project(s.dt, rel_tol=1e-6)
    b = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
    b.set_graphs(False)
    b.upload_state(s.vof, s.u, s.v, s.w)
    rb = b.project(s.dt, rel_tol=1e-6)
    assert ra["status_name"] == rb["status_name"] == "OK"
    assert ra["iterations"] == rb["iterations"]
    np.testing.assert_array_equal(a.pressure(), b.pressure())
    b.set_graphs(True)
    b.upload_state(s.vof, s.u, s.v, s.w)
    rc = b.project(s.dt, rel_tol=1e-6)
    assert rc["iterations"] == ra["iterations"]
    np.testing.assert_array_equal(a.pressure(), b.pressure())
    a.destroy()
    b.destroy()
