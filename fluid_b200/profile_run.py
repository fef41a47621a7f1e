"""A few projections of a named workload with direct kernel launches, for profilers.

Kernels inside the solve's CUDA graphs (conditional WHILE nodes) are not visible
to ncu, so this runs the same solves with one launch per kernel (the profiling
mode of the library) and prints one line per solve:

  python -m fluid_b200.profile_run --workload dam --solves 3
  python -m fluid_b200.profile_run --workload tall --solves 1
  python -m fluid_b200.profile_run --workload batch --solves 2

dam   : 128x96x128 dam break + 16 spheres, fp16 levels (the bench's secondary uniform workload)
tall  : 256^2 columns x 1024 rows, band 32 (the bench's tall-cell workload)
batch : the bench's 64 uneven uniform grids in one batched solve
transport : CM12 density transport steps on the 128x96x128 transport lattice (one launch per kernel always)
extrap : velocity extrapolation of the projected 128x96x128 dam break + 16 spheres
atlas : the sparse brick atlas of a 256x192x256 pool with 40 drops (8508 bricks), V-cycle PCG
"""
from __future__ import annotations

import argparse

from . import BatchProjector, PressureProjector, configs
from .tall import TallProjector


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["dam", "tall", "batch", "transport", "atlas", "extrap"], default="dam")
    ap.add_argument("--solves", type=int, default=2)
    ap.add_argument("--precision", default="fp16", choices=["fp32", "fp16", "bf16"])
    args = ap.parse_args()
    if args.workload == "dam":
        s = configs.dam_spheres()
        pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, precision=args.precision)
        pp.set_profiling(True)
        for _ in range(args.solves):
            pp.upload_state(s.vof, s.u, s.v, s.w)
            r = pp.project(s.dt, rel_tol=1e-6)
            print(r["status_name"], r["iterations"], flush=True)
    elif args.workload == "tall":
        s = configs.tall_waves()
        tp = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho)
        tp.set_graphs(False)
        for _ in range(args.solves):
            tp.upload_state(s.vof, s.u, s.v, s.w)
            r = tp.project(s.dt, rel_tol=1e-6)
            print(r["status_name"], r["iterations"], flush=True)
    elif args.workload == "extrap":
        s = configs.dam_spheres()
        pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, precision=args.precision)
        pp.upload_state(s.vof, s.u, s.v, s.w)
        pp.project(s.dt, rel_tol=1e-6)
        _, u, v, w = pp.download()
        for _ in range(args.solves):
            pp.upload_state(s.vof, u, v, w)
            print("filled", pp.extrapolate_velocity(), flush=True)
    elif args.workload == "atlas":
        from .atlas import AtlasProjector, bricks_from_dense
        s = configs.atlas_scene(256, 192, 256, seed=11, drops=40)
        coords = configs.atlas_bricks(s.vof)
        dens, faces = bricks_from_dense(s.vof, s.u, s.v, s.w, coords)
        A = AtlasProjector((s.nx, s.ny, s.nz), s.h, s.rho)
        A.set_graphs(False)
        for _ in range(args.solves):
            A.upload(coords, dens, faces)
            r = A.project(s.dt, rel_tol=1e-6)
            print(r["status_name"], r["iterations"], flush=True)
    elif args.workload == "transport":
        s = configs.transport_scene(128, 96, 128, seed=21, cells_per_step=2.5)
        pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, s.open_top)
        pp.upload_state(s.vof, s.u, s.v, s.w)
        for _ in range(args.solves):
            r = pp.transport_density(s.dt)
            print("mass", r["mass_before"], r["mass_after"], flush=True)
    else:
        insts = configs.batch_instances()
        pps = [PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, precision=args.precision) for s in insts]
        B = BatchProjector(pps)
        B.set_profiling(True)
        for _ in range(args.solves):
            for p, s in zip(pps, insts):
                p.upload_state(s.vof, s.u, s.v, s.w)
            recs = B.project([s.dt for s in insts], rel_tol=1e-6)
            print(sum(r["status_name"] == "OK" for r in recs), max(r["iterations"] for r in recs), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
