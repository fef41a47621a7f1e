"""Parity of the CUDA uniform-grid projection against the float64 oracle (GPU)."""
import numpy as np
import pytest

from fluid_b200 import BatchProjector, PipelinedBatchProjector, PressureProjector, configs
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

REL_L2_PRESSURE = 1e-5      # pressure vs the float64 oracle (required tolerance)
DIV_RATIO = 1e-6            # max post-projection divergence / max pre-projection divergence
REL_RES = 1e-6


def _pair(s, precision="fp32"):
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, s.open_top, precision)
    pp.upload_state(s.vof, s.u, s.v, s.w)
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho, s.open_top)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    return pp, o


CASES = {
    "dam32": lambda: configs.dam_break_32(),
    "odd37x50x29": lambda: configs.random_small(37, 50, 29, seed=11),
    "semi2x64x48": lambda: configs.random_small(2, 64, 48, seed=12),
    "open_top24": lambda: configs.random_small(24, 24, 24, seed=13, open_top=True),
    "thin40x8x24": lambda: configs.random_small(40, 8, 24, seed=14),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_labels_and_level_maps_bit_exact(name):
    s = CASES[name]()
    pp, o = _pair(s)
    pp.prepare(s.dt)
    assert o.num_levels == len([1 for _ in range(o.num_levels)])
    for l in range(o.num_levels):
        (dims, _, _) = o.level_dims(l)
        assert pp.level_dims(l) == dims
        lab_d, phi_d, diag_d = pp.level(l)
        lab_o, phi_o, diag_o = o.level(l)
        np.testing.assert_array_equal(lab_d, lab_o, err_msg=f"labels level {l}")
        np.testing.assert_array_equal(phi_d.view(np.uint32), phi_o.view(np.uint32), err_msg=f"phi level {l}")
        np.testing.assert_allclose(diag_d, diag_o, rtol=2e-6, atol=1e-12, err_msg=f"diag level {l}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_rhs_and_operator(name):
    s = CASES[name]()
    pp, o = _pair(s)
    pp.prepare(s.dt)
    b_o, _ = o.rhs()
    b_d = pp.rhs()
    scale = np.abs(b_o).max()
    assert np.abs(b_d - b_o).max() <= 1e-6 * scale
    lab, _, _ = o.level(0)
    rng = np.random.default_rng(5)
    p = (rng.normal(size=lab.shape) * lab).astype(np.float32)
    ap_d = pp.apply_operator(p)
    ap_o = o.apply(p.astype(np.float64))
    assert np.linalg.norm(ap_d - ap_o) <= 1e-6 * np.linalg.norm(ap_o)


@pytest.mark.parametrize("name", ["dam32", "odd37x50x29", "semi2x64x48", "open_top24"])
def test_vcycle_matches_oracle_and_is_symmetric(name):
    s = CASES[name]()
    pp, o = _pair(s)
    pp.prepare(s.dt)
    lab, _, _ = o.level(0)
    rng = np.random.default_rng(7)
    x = (rng.normal(size=lab.shape) * lab).astype(np.float32)
    y = (rng.normal(size=lab.shape) * lab).astype(np.float32)
    for pre in (1, 2):
        zx = pp.apply_vcycle(x, pre, pre)
        zo = o.vcycle(x.astype(np.float64), pre, pre)
        assert np.linalg.norm(zx - zo) <= 2e-5 * np.linalg.norm(zo), pre
        zy = pp.apply_vcycle(y, pre, pre)
        a, b = float(np.dot(x.ravel().astype(np.float64), zy.ravel())), float(np.dot(zx.ravel().astype(np.float64), y.ravel()))
        assert abs(a - b) <= 1e-5 * np.sqrt(abs(np.dot(x.ravel(), zx.ravel()) * np.dot(y.ravel(), zy.ravel())))


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
@pytest.mark.parametrize("name", ["dam32", "odd37x50x29", "semi2x64x48", "open_top24"])
def test_fcycle_matches_oracle(name, precision):
    """One full cycle (cycle = 1's preconditioner) against the float64 full
    cycle of the oracle with the same first block level."""
    s = CASES[name]()
    pp, o = _pair(s, precision)
    pp.prepare(s.dt)
    lab, _, _ = o.level(0)
    x = (np.random.default_rng(8).normal(size=lab.shape) * lab).astype(np.float32)
    tol = 2e-5 if precision == "fp32" else 3e-3
    for pre in (1, 2):
        z, fb = pp.apply_fcycle(x, pre, pre)
        assert 1 <= fb < o.num_levels or (o.num_levels == 1 and fb == 0)
        zo = o.fcycle(x.astype(np.float64), pre, pre, fb)
        assert np.linalg.norm(z - zo) <= tol * np.linalg.norm(zo), (pre, fb)


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("name", ["dam32", "odd37x50x29", "open_top24", "semi2x64x48"])
def test_project_full_cycle_matches_oracle(name, precision):
    """The full cycle under flexible CG meets the same parity bars as the
    V-cycle solve, in the iterations of the float64 flexible PCG (within one)."""
    s = CASES[name]()
    pp, o = _pair(s, precision)
    rec = pp.project(s.dt, rel_tol=REL_RES, rel_tol_inf=0.5 * DIV_RATIO, cycle="f")
    _check_projection(s, precision, rec, pp, o)
    _, fb = pp.apply_fcycle(np.zeros(o.level(0)[0].shape, np.float32))
    _, info = o.solve_fcg(REL_RES, 0.0, 300, 1, 1, fb)
    assert info["converged"] == 1.0
    if precision == "fp32":
        assert abs(rec["iterations"] - info["iterations"]) <= 1, (rec["iterations"], info)


def _check_projection(s, precision, rec, pp, o, p_ref=None):
    assert rec["status_name"] == "OK", rec
    assert rec["true_rel_residual"] <= REL_RES
    assert rec["l2_div_after"] <= DIV_RATIO * rec["l2_div_before"], rec
    if p_ref is None:
        p_ref, info = o.solve_mgpcg(1e-12, 0.0, 300, 2, 2)
        assert info["converged"] == 1.0
    x = pp.pressure_cells().astype(np.float64)
    err = np.linalg.norm(x - p_ref) / np.linalg.norm(p_ref)
    assert err <= REL_L2_PRESSURE, (precision, err)
    assert rec["max_div_after"] <= DIV_RATIO * rec["max_div_before"], rec
    (uo, vo, wo), orec = o.grad_subtract(p_ref)
    p_si, u, v, w = pp.download()
    scale = max(np.abs(uo).max(), np.abs(vo).max(), np.abs(wo).max())
    for dev, ref in ((u, uo), (v, vo), (w, wo)):
        assert np.abs(dev - ref).max() <= 1e-4 * scale
    np.testing.assert_allclose(p_si, o.pressure_si(p_ref).astype(np.float32) * (x != 0),
                               rtol=0, atol=1e-4 * np.abs(o.pressure_si(p_ref)).max())
    return err


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("name", ["dam32", "odd37x50x29", "open_top24"])
def test_project_matches_oracle(name, precision):
    s = CASES[name]()
    pp, o = _pair(s, precision)
    # the max-norm criterion leaves room for the float32 rounding of the stored velocities
    rec = pp.project(s.dt, rel_tol=REL_RES, rel_tol_inf=0.5 * DIV_RATIO)
    _check_projection(s, precision, rec, pp, o)


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
@pytest.mark.parametrize("name", ["dam32", "semi2x64x48"])
def test_project_two_sweep_schedule(name, precision):
    """Two sweeps down and up run the per-pass grid kernels instead of the fused ones."""
    s = CASES[name]()
    pp, o = _pair(s, precision)
    rec = pp.project(s.dt, rel_tol=REL_RES, rel_tol_inf=0.5 * DIV_RATIO, pre_sweeps=2, post_sweeps=2)
    _check_projection(s, precision, rec, pp, o)


@pytest.mark.parametrize("name", ["dam32", "odd37x50x29", "open_top24"])
def test_project_at_l2_tolerance(name):
    """At the benchmark's operating point (L2 criterion only) the max-norm ratio stays near 1e-6."""
    s = CASES[name]()
    pp, o = _pair(s)
    rec = pp.project(s.dt, rel_tol=REL_RES)
    assert rec["status_name"] == "OK", rec
    assert rec["true_rel_residual"] <= REL_RES
    assert rec["l2_div_after"] <= DIV_RATIO * rec["l2_div_before"], rec
    assert rec["max_div_after"] <= 3 * DIV_RATIO * rec["max_div_before"], rec


def test_all_liquid_box_nullspace():
    n = 16
    rng = np.random.default_rng(3)
    vof = np.ones((n, n, n), np.float32)
    s = configs.GridState(n, n, n, 1.0 / n, 1 / 60, vof, *configs.velocities(vof, rng, 1 / 60, "gauss", 0.2))
    pp, o = _pair(s)
    rec = pp.project(s.dt, rel_tol=REL_RES, rel_tol_inf=0.5 * DIV_RATIO)
    assert rec["status_name"] == "OK", rec
    p_ref, info = o.solve_mgpcg(1e-12, 0.0, 300, 2, 2)
    x = pp.pressure_cells().astype(np.float64)
    x -= x.mean()
    assert np.linalg.norm(x - p_ref) <= REL_L2_PRESSURE * np.linalg.norm(p_ref)
    assert rec["max_div_after"] <= DIV_RATIO * rec["max_div_before"]


def test_nonfinite_input_keeps_previous_pressure():
    s = configs.dam_break_32()
    pp, _ = _pair(s)
    rec = pp.project(s.dt)
    assert rec["status_name"] == "OK"
    p0, u0, v0, w0 = pp.download()
    bad = s.vof.copy()
    bad[3, 3, 3] = np.nan
    pp.upload_state(bad, u0, v0, w0)
    rec2 = pp.project(s.dt)
    assert rec2["status_name"] == "NONFINITE"
    p1, _, _, _ = pp.download()
    np.testing.assert_array_equal(p0, p1)


def test_iteration_cap_reports_nonconvergence():
    s = configs.dam_break_32()
    pp, _ = _pair(s)
    rec = pp.project(s.dt, rel_tol=1e-12, max_iters=2)
    assert rec["status_name"] == "NONCONVERGENCE"
    assert rec["iterations"] == 2


@pytest.mark.parametrize("tuning", [None, {"parts": 3}])
def test_batch_is_identical_to_single(tuning):
    """Uneven lattices (a semi-coarsened one and a tiny one among them) give each
    single solve's bits in a batch, also split into concurrent parts."""
    import dataclasses
    # a different dt per instance, so each part must receive its own instances' dts
    states = [dataclasses.replace(s, dt=s.dt * (1.0 + 0.25 * k)) for k, s in enumerate(
        configs.random_small(n[0], n[1], n[2], seed=20 + k)
        for k, n in enumerate([(24, 30, 28), (37, 25, 41), (16, 16, 16), (48, 20, 33), (2, 64, 48), (4, 4, 4)]))]
    singles = []
    for s in states:
        pp = PressureProjector((s.nx, s.ny, s.nz), s.h)
        pp.upload_state(s.vof, s.u, s.v, s.w)
        singles.append((pp.project(s.dt), pp.pressure_cells(), pp.download()[0]))
    pps = []
    for s in states:
        pp = PressureProjector((s.nx, s.ny, s.nz), s.h)
        pp.upload_state(s.vof, s.u, s.v, s.w)
        pps.append(pp)
    batch = BatchProjector(pps, tuning=tuning)
    recs = batch.project([s.dt for s in states])
    for (r1, x1, p1), r2, pp in zip(singles, recs, pps):
        assert r2["status_name"] == "OK"
        assert r1["iterations"] == r2["iterations"]
        np.testing.assert_array_equal(x1, pp.pressure_cells())
        np.testing.assert_array_equal(p1, pp.download()[0])   # pressure in Pa carries each instance's dt


def test_batch_of_thirteen_is_identical_to_singles():
    """Thirteen 64x48x64 grids fill the GPU as a batch, so the column kernels take
    long z chunks; each grid alone takes short chunks to fill the GPU by itself.
    Halo cells repeat their owner's arithmetic and the dot products fold over
    fixed tiles, so pressures and iteration counts agree bit for bit."""
    states = [configs.random_small(64, 48, 64, seed=60 + k) for k in range(13)]
    singles = []
    for s in states:
        pp = PressureProjector((s.nx, s.ny, s.nz), s.h, precision="fp16")
        pp.upload_state(s.vof, s.u, s.v, s.w)
        singles.append((pp.project(s.dt), pp.pressure_cells()))
        pp.destroy()
    pps = []
    for s in states:
        pp = PressureProjector((s.nx, s.ny, s.nz), s.h, precision="fp16")
        pp.upload_state(s.vof, s.u, s.v, s.w)
        pps.append(pp)
    batch = BatchProjector(pps)
    recs = batch.project([s.dt for s in states])
    for (r1, x1), r2, pp in zip(singles, recs, pps):
        assert r2["status_name"] == "OK"
        assert r1["iterations"] == r2["iterations"]
        np.testing.assert_array_equal(x1, pp.pressure_cells())
    batch.destroy()
    for pp in pps:
        pp.destroy()


@pytest.mark.parametrize("tuning", [None, {"parts": 2}])
def test_pipelined_ticks_match_synchronous_batches(tuning):
    """Four ticks of three lattices through PipelinedBatchProjector (two streams,
    two ticks in flight, pinned host buffers) give the receipts and the p, u, v, w
    of BatchProjector.project on each tick's inputs, bit for bit."""
    import torch
    dims = [(40, 32, 36), (24, 20, 26), (33, 17, 29)]
    ticks = [[configs.random_small(nx, ny, nz, seed=300 + 10 * t + k) for k, (nx, ny, nz) in enumerate(dims)]
             for t in range(4)]
    s0 = ticks[0]

    def make_set():
        return [PressureProjector((s.nx, s.ny, s.nz), s.h, precision="fp16") for s in s0]

    ref = []
    pps = make_set()
    batch = BatchProjector(pps)
    for states in ticks:
        for pp, s in zip(pps, states):
            pp.upload_state(s.vof, s.u, s.v, s.w)
        recs = batch.project([s.dt for s in states])
        ref.append((recs, [pp.download() for pp in pps]))
    batch.destroy()
    for pp in pps:
        pp.destroy()

    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    sets = [make_set(), make_set()]
    for st, ps in zip(streams, sets):
        for pp in ps:
            pp.set_stream(st.cuda_stream)
    pipe = PipelinedBatchProjector(sets, tuning=tuning)

    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory().numpy()

    ins = [[tuple(pinned(a) for a in (s.vof, s.u, s.v, s.w)) for s in states] for states in ticks]
    outs = [[tuple(pinned(np.zeros(shp, np.float32)) for shp in
                   ((nz, ny, nx), (nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)))
             for (nx, ny, nz) in dims] for _ in ticks]
    tickets = [pipe.submit(ins[t], outs[t], [s.dt for s in ticks[t]]) for t in range(len(ticks))]
    for t, ticket in enumerate(tickets):
        recs = pipe.result(ticket)
        ref_recs, ref_fields = ref[t]
        for r1, r2 in zip(ref_recs, recs):
            assert r2["status_name"] == "OK"
            assert r1["iterations"] == r2["iterations"]
        for f1, f2 in zip(ref_fields, outs[t]):
            for a, b in zip(f1, f2):
                np.testing.assert_array_equal(a, b)
    with pytest.raises(KeyError):
        pipe.result(tickets[0])
    pipe.destroy()
    for ps in sets:
        for pp in ps:
            pp.destroy()


def test_handles_created_large_first_solve_alone():
    """Kernel limits are process-wide: creating a small handle after a large one must not
    break the large one's own solve (shared-memory limits are never lowered)."""
    big = configs.random_small(120, 72, 100, seed=31)
    small = configs.random_small(24, 20, 26, seed=32)
    handles = []
    for prec in ("fp32", "fp16"):
        pb = PressureProjector((big.nx, big.ny, big.nz), big.h, precision=prec)
        ps = PressureProjector((small.nx, small.ny, small.nz), small.h, precision=prec)
        pb.upload_state(big.vof, big.u, big.v, big.w)
        ps.upload_state(small.vof, small.u, small.v, small.w)
        rb = pb.project(big.dt)
        rs = ps.project(small.dt)
        assert rb["status_name"] == "OK" and rs["status_name"] == "OK", (rb, rs)
        assert rb["true_rel_residual"] <= REL_RES and rs["true_rel_residual"] <= REL_RES
        handles += [pb, ps]


@pytest.fixture(scope="module")
def full_size_dam_spheres():
    """The 128x96x128 dam break with 16 spheres and its float64 oracle (MGPCG to
    rel-res 1e-12), shared by the full-size parity tests."""
    s = configs.dam_spheres()
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    p_ref, info = o.solve_mgpcg(1e-12, 0.0, 300, 2, 2)
    assert info["converged"] == 1.0
    return s, o, p_ref


def test_full_size_dam_spheres_labels_rhs_operator(full_size_dam_spheres):
    """Labels, level sets and level maps bit-exact on all 7 levels; b and A p
    against the oracle at the full 1.57M-cell size."""
    s, o, _ = full_size_dam_spheres
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho)
    pp.upload_state(s.vof, s.u, s.v, s.w)
    pp.prepare(s.dt)
    assert o.num_levels == 7
    for l in range(o.num_levels):
        assert pp.level_dims(l) == o.level_dims(l)[0]
        lab_d, phi_d, diag_d = pp.level(l)
        lab_o, phi_o, diag_o = o.level(l)
        np.testing.assert_array_equal(lab_d, lab_o, err_msg=f"labels level {l}")
        np.testing.assert_array_equal(phi_d.view(np.uint32), phi_o.view(np.uint32), err_msg=f"phi level {l}")
        np.testing.assert_allclose(diag_d, diag_o, rtol=2e-6, atol=1e-12, err_msg=f"diag level {l}")
    b_o, _ = o.rhs()
    assert np.abs(pp.rhs() - b_o).max() <= 1e-6 * np.abs(b_o).max()
    lab, _, _ = o.level(0)
    p = (np.random.default_rng(3).normal(size=lab.shape) * lab).astype(np.float32)
    ap_o = o.apply(p.astype(np.float64))
    assert np.linalg.norm(pp.apply_operator(p) - ap_o) <= 1e-6 * np.linalg.norm(ap_o)
    pp.destroy()


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
def test_full_size_dam_spheres_matches_fp64_oracle(full_size_dam_spheres, precision):
    """The 1.57M-cell projection with every level precision against the float64
    oracle: pressure rel-L2 <= 1e-5, max divergence <= 1e-6 of its pre-projection
    value, projected faces and Pa pressure as in the small-lattice parity tests.
    At the L2-only operating point the receipts meet the L2 bars too."""
    s, o, p_ref = full_size_dam_spheres
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, precision=precision)
    pp.upload_state(s.vof, s.u, s.v, s.w)
    rec = pp.project(s.dt, rel_tol=REL_RES, rel_tol_inf=0.5 * DIV_RATIO)
    assert rec["levels"] == 7
    _check_projection(s, precision, rec, pp, o, p_ref=p_ref)
    pp.upload_state(s.vof, s.u, s.v, s.w)   # the projection overwrote the velocities
    rec = pp.project(s.dt, rel_tol=REL_RES)
    assert rec["status_name"] == "OK", rec
    assert rec["true_rel_residual"] <= REL_RES
    assert rec["l2_div_after"] <= DIV_RATIO * rec["l2_div_before"], rec
    err = np.linalg.norm(pp.pressure_cells().astype(np.float64) - p_ref) / np.linalg.norm(p_ref)
    assert err <= REL_L2_PRESSURE, (precision, err)
    pp.destroy()


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_full_size_dam_spheres_full_cycle_matches_fp64_oracle(full_size_dam_spheres, precision):
    """The full-cycle solve at 128x96x128 against the float64 solution, with
    fewer iterations than the V-cycle solve of the same system."""
    s, o, p_ref = full_size_dam_spheres
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, precision=precision)
    pp.upload_state(s.vof, s.u, s.v, s.w)
    rec_v = pp.project(s.dt, rel_tol=REL_RES, rel_tol_inf=0.5 * DIV_RATIO)
    pp.upload_state(s.vof, s.u, s.v, s.w)
    rec = pp.project(s.dt, rel_tol=REL_RES, rel_tol_inf=0.5 * DIV_RATIO, cycle="f")
    _check_projection(s, precision, rec, pp, o, p_ref=p_ref)
    assert rec["iterations"] < rec_v["iterations"], (rec["iterations"], rec_v["iterations"])
    pp.destroy()


def test_batch_layouts_give_the_same_bits_and_autotune_keeps_the_fastest():
    """Every batch layout (box shapes, column z chunks, fill counts, concurrent parts) gives the
    default layout's pressures and iteration counts bit for bit; the autotuner's
    choice is never slower than the default it measured."""
    from fluid_b200 import autotune
    from fluid_b200.projector import batch_tuning
    states = [configs.random_small(64, 48, 64, seed=90 + k) for k in range(13)]
    pps = [PressureProjector((s.nx, s.ny, s.nz), s.h, precision="fp16") for s in states]

    def restore():
        for pp, s in zip(pps, states):
            pp.upload_state(s.vof, s.u, s.v, s.w)

    dts = [s.dt for s in states]
    layouts = [None, dict(chunk_planes=8), dict(chunk_planes=64, fill_tiles=148), dict(box_shape=4, chunk_planes=16),
               dict(fill_tiles=4096), dict(parts=2), dict(parts=3, chunk_planes=32)]
    ref = None
    for lay in layouts:
        b = BatchProjector(pps, tuning=lay)
        restore()
        recs = b.project(dts)
        got = ([r["iterations"] for r in recs], [pp.pressure_cells() for pp in pps])
        b.destroy()
        assert all(r["status_name"] == "OK" for r in recs), lay
        if ref is None:
            ref = got
            continue
        assert got[0] == ref[0], lay
        for a, c in zip(got[1], ref[1]):
            np.testing.assert_array_equal(a, c, err_msg=str(lay))
    cands = tuple(dict(batch_tuning(**lay).as_dict()) for lay in [dict(), dict(chunk_planes=8), dict(fill_tiles=148)])
    res = autotune.autotune_batch(pps, dts, restore, layouts=cands, parts=(2,), sweeps=((1, 1), (2, 2)), repeats=1)
    assert res.ms <= res.default_ms
    assert len(res.table) == 5 and res.sweeps in ((1, 1), (2, 2))
    for pp in pps:
        pp.destroy()


def test_batch_rejects_handles_on_different_streams():
    """A batch orders all of its work on one stream, while each handle's uploads,
    downloads and release use the handle's own stream.  Handles on different
    streams are rejected at batch creation, and a member moved to another stream
    afterwards is rejected at the next batch call, so neither can race the solve."""
    import torch
    states = [configs.random_small(16, 12, 20, seed=900 + k) for k in range(2)]
    pps = [PressureProjector((s.nx, s.ny, s.nz), s.h) for s in states]
    for pp, s in zip(pps, states):
        pp.upload_state(s.vof, s.u, s.v, s.w)
    side = torch.cuda.Stream()
    pps[1].set_stream(side.cuda_stream)
    with pytest.raises(ValueError, match="share one stream"):
        BatchProjector(pps)
    pps[1].set_stream(0)   # back on the default stream, like pps[0]
    batch = BatchProjector(pps)
    recs = batch.project([s.dt for s in states])
    assert all(r["status_name"] == "OK" for r in recs)
    pps[0].set_stream(side.cuda_stream)
    with pytest.raises(ValueError, match="no longer matches"):
        batch.project([s.dt for s in states])
    pps[0].set_stream(0)
    assert all(r["status_name"] == "OK" for r in batch.project([s.dt for s in states]))
    batch.destroy()
    for pp in pps:
        pp.destroy()


def test_consecutive_steps_converge_with_default_options():
    """Steps whose input is the previous step's projected velocity plus gravity
    have a smooth right-hand side about 20x smaller than the first step's; with
    the recursive float32 residual alone CG stalled above 1e-6 for 200+
    iterations.  With the default options (float64 true residual every 4
    iterations) every step converges in a handful of V-cycles, and the pressure
    stays within the float64 oracle's tolerance."""
    s0 = configs.dam_spheres()
    carrier = PressureProjector((s0.nx, s0.ny, s0.nz), s0.h, s0.rho)

    def carry(st):
        carrier.upload_state(st.vof, st.u, st.v, st.w)
        rec = carrier.project(st.dt)
        assert rec["status_name"] == "OK", rec
        return carrier.download()[1:]
    states = configs.dam_spheres_sequence(4, carry)
    carrier.destroy()
    for precision in ("fp32", "fp16"):
        pp = PressureProjector((s0.nx, s0.ny, s0.nz), s0.h, s0.rho, precision=precision)
        for st in states[1:]:
            pp.upload_state(st.vof, st.u, st.v, st.w)
            rec = pp.project(st.dt)
            assert rec["status_name"] == "OK", (precision, rec)
            assert rec["iterations"] <= 30, (precision, rec)
            assert rec["true_rel_residual"] <= REL_RES
        o = Oracle(st.nx, st.ny, st.nz, st.h, st.rho)
        o.set_state(st.vof, st.u, st.v, st.w, st.dt)
        p_ref, _ = o.solve_mgpcg(1e-12, 0.0, 300, 2, 2)
        err = np.linalg.norm(pp.pressure_cells().astype(np.float64) - p_ref) / np.linalg.norm(p_ref)
        assert err <= REL_L2_PRESSURE, (precision, err)
        pp.destroy()
