"""Parity of the CUDA tall-cell projection against the float64 tall-cell oracle (GPU)."""
import numpy as np
import pytest

from fluid_b200 import configs
from fluid_b200.tall import TallProjector
from oracle import tall as oracle

pytestmark = pytest.mark.gpu

REL_L2_PRESSURE = 1e-5
REL_RES = 1e-6

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
    rec = tp.project(s.dt, rel_tol=REL_RES)
    assert rec["status_name"] == "OK", rec
    assert rec["true_rel_residual"] <= REL_RES
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


def test_tall_full_size_waves_converge():
    s = configs.tall_waves()
    tp = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
    tp.upload_state(s.vof, s.u, s.v, s.w)
    rec = tp.project(s.dt, rel_tol=REL_RES)
    assert rec["status_name"] == "OK", rec
    assert rec["true_rel_residual"] <= REL_RES
    assert rec["levels"] == 7
    assert rec["max_div_after"] <= 1e-4 * rec["max_div_before"], rec


def test_tall_sliced_projection_matches_one_call():
    """begin + continue in slices of 3 iterations + end gives the one-call result bit for bit."""
    s = configs.tall_waves(20, 20, 96, 24, seed=2, mean=50, amp_max=4, lam=(8, 32))
    a = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
    a.upload_state(s.vof, s.u, s.v, s.w)
    ra = a.project(s.dt, rel_tol=1e-6)
    b = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
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
