"""Embedded solids (cut cells) on the device against the float64 oracle (GPU)."""
import numpy as np
import pytest

from fluid_b200 import BatchProjector, PressureProjector, configs
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

REL_L2_PRESSURE = 1e-5
DIV_RATIO = 1e-6
REL_RES = 1e-6

SCENES = {
    "ramp_ball_48x40x44": lambda: configs.solid_scene(48, 40, 44, seed=3),
    "ramp_ball_static_37x30x26": lambda: configs.solid_scene(37, 30, 26, seed=5, sphere_velocity=(0.0, 0.0, 0.0)),
    "ramp_ball_open_top_40x32x36": lambda: configs.solid_scene(40, 32, 36, seed=7, open_top=True),
}


def _pair(sc, precision="fp32"):
    s = sc.state
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, s.open_top, precision)
    pp.upload_solids(*sc.solids())
    pp.upload_state(s.vof, s.u, s.v, s.w)
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho, s.open_top)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    o.set_solids(*sc.solids())
    return pp, o


@pytest.mark.parametrize("name", sorted(SCENES))
def test_solid_labels_faces_and_levels_bit_exact(name):
    sc = SCENES[name]()
    pp, o = _pair(sc)
    pp.prepare(sc.state.dt)
    for l in range(o.num_levels):
        assert pp.level_dims(l) == o.level_dims(l)[0]
        np.testing.assert_array_equal(pp.level_faces(l).view(np.uint32), o.level_faces(l).view(np.uint32),
                                      err_msg=f"face fractions level {l}")
        lab_d, phi_d, diag_d = pp.level(l)
        lab_o, phi_o, diag_o = o.level(l)
        np.testing.assert_array_equal(lab_d, lab_o, err_msg=f"labels level {l}")
        np.testing.assert_array_equal(phi_d.view(np.uint32), phi_o.view(np.uint32), err_msg=f"phi level {l}")
        np.testing.assert_allclose(diag_d, diag_o, rtol=2e-6, atol=1e-12, err_msg=f"diag level {l}")
    pp.destroy()


@pytest.mark.parametrize("name", sorted(SCENES))
def test_solid_rhs_operator_and_vcycle(name):
    sc = SCENES[name]()
    pp, o = _pair(sc)
    pp.prepare(sc.state.dt)
    b_o, _ = o.rhs()
    assert np.abs(pp.rhs() - b_o).max() <= 1e-6 * np.abs(b_o).max()
    lab, _, _ = o.level(0)
    rng = np.random.default_rng(5)
    p = (rng.normal(size=lab.shape) * lab).astype(np.float32)
    ap_o = o.apply(p.astype(np.float64))
    assert np.linalg.norm(pp.apply_operator(p) - ap_o) <= 1e-6 * np.linalg.norm(ap_o)
    for pre in (1, 2):
        z = pp.apply_vcycle(p, pre, pre)
        zo = o.vcycle(p.astype(np.float64), pre, pre)
        assert np.linalg.norm(z - zo) <= 2e-5 * np.linalg.norm(zo), pre
    pp.destroy()


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("name", sorted(SCENES))
def test_solid_projection_matches_fp64_oracle(name, precision):
    """Pressure within rel-L2 1e-5 of the float64 solve, the weighted divergence
    reduced by 1e-6, projected faces within 1e-4 of the oracle's (closed faces
    carry the solids' velocity exactly)."""
    sc = SCENES[name]()
    pp, o = _pair(sc, precision)
    rec = pp.project(sc.state.dt, rel_tol=REL_RES, rel_tol_inf=0.5 * DIV_RATIO)
    assert rec["status_name"] == "OK", rec
    assert rec["true_rel_residual"] <= REL_RES
    assert rec["max_div_after"] <= DIV_RATIO * rec["max_div_before"], rec
    p_ref, info = o.solve_mgpcg(1e-12, 0.0, 400, 2, 2)
    assert info["converged"] == 1.0
    x = pp.pressure_cells().astype(np.float64)
    assert np.linalg.norm(x - p_ref) <= REL_L2_PRESSURE * np.linalg.norm(p_ref)
    (uo, vo, wo), _ = o.grad_subtract(p_ref)
    _, u, v, w = pp.download()
    scale = max(np.abs(uo).max(), np.abs(vo).max(), np.abs(wo).max())
    for dev, ref in ((u, uo), (v, vo), (w, wo)):
        assert np.abs(dev - ref).max() <= 1e-4 * scale
    closed = np.clip(sc.fy, 0, 1) <= 1e-6
    closed[:, 0, :] = False
    if not sc.state.open_top:
        closed[:, -1, :] = False
    np.testing.assert_array_equal(v[closed], sc.usy[closed])
    pp.destroy()


def test_solid_batch_is_identical_to_singles_and_rejects_mixing():
    scenes = [configs.solid_scene(32, 28, 30, seed=11), configs.solid_scene(40, 24, 36, seed=12)]
    singles, handles = [], []
    for sc in scenes:
        pp, _ = _pair(sc)
        rec = pp.project(sc.state.dt, rel_tol=REL_RES)
        assert rec["status_name"] == "OK"
        singles.append((rec, pp.pressure_cells()))
        pp.destroy()
    for sc in scenes:
        pp, _ = _pair(sc)
        handles.append(pp)
    B = BatchProjector(handles)
    recs = B.project([sc.state.dt for sc in scenes], rel_tol=REL_RES)
    for (rs, ps), rb, pp in zip(singles, recs, handles):
        assert rb["iterations"] == rs["iterations"]
        np.testing.assert_array_equal(pp.pressure_cells(), ps)
    B.destroy()
    s = configs.random_small(24, 20, 28, seed=5)
    plain = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho)
    plain.upload_state(s.vof, s.u, s.v, s.w)
    with pytest.raises(ValueError, match="embedded solids"):
        BatchProjector([handles[0], plain])
    for pp in handles + [plain]:
        pp.destroy()


def test_all_open_solids_give_the_plain_solution():
    """Open fractions of 1 (face-weighted per-pass kernels) solve the same
    system as the handle without solids (fused kernels), to the solver tolerance."""
    s = configs.dam_break_32()
    plain = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho)
    plain.upload_state(s.vof, s.u, s.v, s.w)
    r0 = plain.project(s.dt, rel_tol=1e-9)
    solid = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho)
    ones = lambda a: np.ones_like(a, np.float32)
    solid.upload_solids(np.ones_like(s.vof), ones(s.u), ones(s.v), ones(s.w))
    solid.upload_state(s.vof, s.u, s.v, s.w)
    r1 = solid.project(s.dt, rel_tol=1e-9)
    assert r0["status_name"] == r1["status_name"] == "OK"
    np.testing.assert_array_equal(plain.level(0)[0], solid.level(0)[0])
    x0, x1 = plain.pressure_cells().astype(np.float64), solid.pressure_cells().astype(np.float64)
    assert np.linalg.norm(x1 - x0) <= 1e-7 * np.linalg.norm(x0)
    plain.destroy()
    solid.destroy()
