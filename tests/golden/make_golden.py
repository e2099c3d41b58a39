"""Generate the golden fixtures that pin the oracle and the CUDA engine.

Run in a container that has the Aero reference checked out (read-only is
fine) and Numba installed:

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py \
        --reference <path to an Aero checkout>

It imports the reference's own ``aero`` package and records, for a set of
small seeded cases covering every hot-path feature, the initial state, the
state after N ``_step()`` calls, the per-step coefficient histories and the
last force profile.  It also records the reference's lattice/MRT tables and
bit-exact geometry (masks, link lists, q values) for the benchmark
configurations: in full for the 2D channel, as SHA-256 digests for the large
3D grids.

The fixtures are written to ``tests/golden/*.npz`` and committed; nothing at
test time reads the reference.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import zlib
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def _digest(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a)
    h = hashlib.sha256()
    h.update(str(a.dtype).encode())
    h.update(str(a.shape).encode())
    h.update(a.tobytes())
    return h.hexdigest()


CASES_2D = [
    # name, geometry, solver kwargs, steps
    ("c2d_bgk_noslip_zerograd", ("cyl", 4.5, 0.3, 0.5),
     dict(collision="bgk", wall_bc="noslip", outlet_bc="zerogradient"), 40),
    ("c2d_bgk_slip_convective_pert", ("cyl", 4.5, 0.3, 0.5),
     dict(collision="bgk", wall_bc="slip", outlet_bc="convective", inlet_perturbation=0.1), 40),
    ("c2d_trt_noslip_smag", ("cyl", 4.5, 0.3, 0.5),
     dict(_tau=0.8, collision="trt", trt_lambda=0.25, wall_bc="noslip", outlet_bc="convective",
          les=True, les_cs=0.16, van_driest=True, van_driest_A=5.0), 40),
    ("c2d_mrt_slip_sponge", ("cyl", 4.5, 0.3, 0.5),
     dict(collision="mrt", wall_bc="slip", outlet_bc="convective", sponge_thickness=8,
          sponge_strength=0.1, les=True), 40),
    ("c2d_bgk_wale_bouzidi", ("cyl", 4.5, 0.3, 0.5),
     dict(collision="bgk", wall_bc="noslip", outlet_bc="zerogradient", les=True,
          les_model="wale", les_cs=0.3, bouzidi=True), 40),
    ("c2d_trt_bouzidi_moving", ("cyl", 4.5, 0.3, 0.5),
     dict(_tau=0.8, collision="trt", trt_lambda=3.0 / 16.0, wall_bc="moving", wall_velocity_top=0.03,
          wall_velocity_bottom=-0.01, outlet_bc="convective", bouzidi=True), 40),
    ("c2d_bgk_pressure", ("cyl", 4.5, 0.3, 0.5),
     dict(collision="bgk", wall_bc="noslip", inlet_bc="pressure", outlet_bc="pressure",
          rho_in=1.002, rho_out=0.999), 40),
    ("c2d_bgk_thermal", ("cyl", 4.5, 0.3, 0.5),
     dict(collision="bgk", wall_bc="noslip", outlet_bc="zerogradient", thermal=True,
          alpha_T=0.02, buoyancy=True, g_gravity=1e-3, beta=0.5, T_ref=0.5), 40),
    ("c2d_bgk_rect_on_wall", ("rect", 8.0, 6.0, 0.35, 2.0 / 24.0),
     dict(collision="bgk", wall_bc="noslip", outlet_bc="convective", bouzidi=True), 40),
    ("c2d_mrt_smag_bouzidi_noslip", ("cyl", 5.0, 0.3, 0.45),
     dict(collision="mrt", wall_bc="noslip", outlet_bc="zerogradient", bouzidi=True,
          les=True), 40),
    ("c2d_bgk_synthetic_inflow", ("cyl", 4.5, 0.3, 0.5),
     dict(collision="bgk", wall_bc="noslip", outlet_bc="convective", synthetic_inflow=True,
          synthetic_inflow_intensity=0.05, synthetic_inflow_seed=77), 40),
]

CASES_3D = [
    ("c3d_bgk_slip_convective", ("sph", 3.0, 0.3, 0.5, 0.5),
     dict(collision="bgk", wall_bc="slip", outlet_bc="convective"), 12),
    ("c3d_mrt_smag_bouzidi_sponge", ("sph", 3.0, 0.3, 0.5, 0.5),
     dict(collision="mrt", wall_bc="slip", outlet_bc="convective", les=True, les_cs=0.1,
          bouzidi=True, sponge_thickness=6), 12),
    ("c3d_trt_wale_periodic_bodyforce_thermal", ("box", 4.0, 4.0, 100.0, 0.4, 2.0 / 10.0, 0.5),
     dict(_tau=0.75, collision="trt", trt_lambda=3.0 / 16.0, les=True, les_model="wale", les_cs=0.3,
          streamwise_bc="periodic", body_force_x=1e-5, wall_bc="noslip", thermal=True,
          T_hot=1.0, T_cold=0.0, alpha_T=0.01, buoyancy=True, g_gravity=1e-3, beta=1.0,
          T_ref=0.5), 12),
    ("c3d_bgk_noslip_zerograd_pert", ("sph", 3.0, 0.3, 0.5, 0.5),
     dict(collision="bgk", wall_bc="noslip", outlet_bc="zerogradient", inlet_perturbation=0.2), 12),
    ("c3d_trt_moving_smag_vandriest", ("sph", 3.0, 0.3, 0.5, 0.5),
     dict(_tau=0.8, collision="trt", wall_bc="moving", wall_velocity_top=0.02, wall_velocity_bottom=0.01,
          outlet_bc="convective", les=True, les_cs=0.2, van_driest=True, van_driest_A=3.0,
          bouzidi=True), 12),
    ("c3d_mrt_noslip_zerograd", ("sph", 3.5, 0.35, 0.45, 0.55),
     dict(collision="mrt", wall_bc="noslip", outlet_bc="zerogradient"), 12),
    ("c3d_bgk_smag_bodyforce_open", ("sph", 3.0, 0.3, 0.5, 0.5),
     dict(collision="bgk", wall_bc="slip", outlet_bc="convective", les=True, les_cs=0.16,
          body_force_x=2e-5, body_force_y=-1e-5), 12),
    ("c3d_bgk_synthetic_inflow", ("sph", 3.0, 0.3, 0.5, 0.5),
     dict(collision="bgk", wall_bc="slip", outlet_bc="convective", synthetic_inflow=True,
          synthetic_inflow_intensity=0.05, synthetic_inflow_seed=91), 12),
    ("c3d_bgk_sem_inlet", ("sph", 3.0, 0.3, 0.5, 0.5),
     dict(collision="bgk", wall_bc="slip", outlet_bc="convective", sem_inlet=True, sem_Tu=0.05,
          sem_L_int=3.0, sem_N=40), 12),
    ("c3d_mrt_recycling_sponge_bodyforce", ("sph", 3.0, 0.3, 0.5, 0.5),
     dict(collision="mrt", wall_bc="noslip", streamwise_bc="recycling", sponge_thickness=4,
          body_force_x=1e-5, bouzidi=True), 12),
]


def _geometry_2d(spec, ny, nx):
    from aero.geometry.cylinder import Cylinder
    from aero.geometry.rectangle import Rectangle
    if spec[0] == "cyl":
        g = Cylinder(radius=spec[1], cx_frac=spec[2], cy_frac=spec[3])
    else:
        g = Rectangle(width=spec[1], height=spec[2], cx_frac=spec[3], cy_frac=spec[4])
    return g, g.mark_solid(ny, nx), g.sdf_field(ny, nx)


def _geometry_3d(spec, nz, ny, nx):
    from aero.geometry3d.sphere import Sphere
    from aero.geometry3d.box import Box
    if spec[0] == "sph":
        g = Sphere(radius=spec[1], cx_frac=spec[2], cy_frac=spec[3], cz_frac=spec[4])
    else:
        g = Box(width=spec[1], height=spec[2], depth=spec[3], cx_frac=spec[4], cy_frac=spec[5],
                cz_frac=spec[6])
    return g, g.mark_solid(nz, ny, nx), g.sdf_field(nz, ny, nx)


def run_case_2d(name, spec, kw, steps, out):
    from aero.lbm.solver import Solver
    from aero.lbm.d2q9 import compute_feq
    ny, nx = 24, 48
    geom, solid, phi = _geometry_2d(spec, ny, nx)
    D = geom.reference_length()
    u0 = 0.05
    kw = dict(kw)
    tau = kw.pop("_tau", 3.0 * (u0 * D / 30.0) + 0.5)
    omega = 1.0 / tau
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    s = Solver(Ny=ny, Nx=nx, solid=solid, omega=omega, u0=u0, D=D, backend="numba",
               phi=phi, **kw)
    rho = 1.0 + 1e-3 * rng.uniform(-1, 1, (ny, nx))
    ux = u0 + 2e-3 * rng.uniform(-1, 1, (ny, nx))
    uy = 2e-3 * rng.uniform(-1, 1, (ny, nx))
    s.f = np.ascontiguousarray(compute_feq(rho, ux, uy))
    if s.g is not None:
        T0 = 0.5 + 0.05 * rng.uniform(-1, 1, (ny, nx))
        s.g = np.ascontiguousarray(s._w[:, None, None] * T0[None])
    f0 = s.f.copy()
    g0 = None if s.g is None else s.g.copy()
    hist = {k: [] for k in ("Cd", "Cl", "Cm", "Cd_p", "Cd_v")}
    for _ in range(steps):
        cd, cl = s._step()
        hist["Cd"].append(cd)
        hist["Cl"].append(cl)
        hist["Cm"].append(s._last_cm)
        hist["Cd_p"].append(s._last_cd_p)
        hist["Cd_v"].append(s._last_cd_v)
    prof = s._last_force_profile
    rec = dict(
        dims=2, nx=nx, ny=ny, nz=1, omega=omega, u0=u0, D=D, steps=steps,
        kwargs=json.dumps(kw), solid=solid, phi=phi, f0=f0, f=s.f,
        f_outlet_prev=s._f_outlet_prev, links=s.surface_links, q_vals=s.q_vals,
        profile=np.array([prof["fx"], prof["fy"]]),
        **{f"hist_{k}": np.array(v) for k, v in hist.items()},
    )
    if g0 is not None:
        rec["g0"] = g0
        rec["g"] = s.g
    np.savez_compressed(out / f"{name}.npz", **rec)


def run_case_3d(name, spec, kw, steps, out):
    from aero.lbm.solver3d import Solver3D
    from aero.lbm.d3q19 import compute_feq_3d
    nz, ny, nx = 8, 10, 18
    geom, solid, phi = _geometry_3d(spec, nz, ny, nx)
    D = geom.reference_length()
    u0 = 0.05
    kw = dict(kw)
    tau = kw.pop("_tau", 3.0 * (u0 * D / 20.0) + 0.5)
    omega = 1.0 / tau
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    s = Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, omega=omega, u0=u0, D=D, backend="numba",
                 phi=phi, **kw)
    shp = (nz, ny, nx)
    rho = 1.0 + 1e-3 * rng.uniform(-1, 1, shp)
    ux = u0 + 2e-3 * rng.uniform(-1, 1, shp)
    uy = 2e-3 * rng.uniform(-1, 1, shp)
    uz = 2e-3 * rng.uniform(-1, 1, shp)
    s.f = np.ascontiguousarray(compute_feq_3d(rho, ux, uy, uz))
    if s.g is not None:
        T0 = 0.5 + 0.05 * rng.uniform(-1, 1, shp)
        s.g = np.ascontiguousarray(s._w_np[:, None, None, None] * T0[None])
    f0 = s.f.copy()
    g0 = None if s.g is None else s.g.copy()
    keys = ("Cd", "Cly", "Clz", "Cmx", "Cmy", "Cmz", "Cd_p", "Cd_v")
    hist = {k: [] for k in keys}
    for _ in range(steps):
        cd, cly, clz = s._step()
        hist["Cd"].append(cd)
        hist["Cly"].append(cly)
        hist["Clz"].append(clz)
        hist["Cmx"].append(s._last_cmx)
        hist["Cmy"].append(s._last_cmy)
        hist["Cmz"].append(s._last_cmz)
        hist["Cd_p"].append(s._last_cd_p)
        hist["Cd_v"].append(s._last_cd_v)
    prof = s._last_spanwise_profile
    rec = dict(
        dims=3, nx=nx, ny=ny, nz=nz, omega=omega, u0=u0, D=D, steps=steps,
        kwargs=json.dumps(kw), solid=solid, phi=phi, f0=f0, f=s.f,
        f_outlet_prev=s._f_outlet_prev, links=s.surface_links, q_vals=s.q_vals,
        profile=np.array([prof["fx"], prof["fy"], prof["fz"]]),
        **{f"hist_{k}": np.array(v) for k, v in hist.items()},
    )
    if g0 is not None:
        rec["g0"] = g0
        rec["g"] = s.g
    np.savez_compressed(out / f"{name}.npz", **rec)


def tables(out):
    from aero.lbm.d2q9 import E, W, OPP
    from aero.lbm.d3q19 import E3, W3, OPP3, Y_MIR3
    from aero.lbm.mrt2d import M9, M9_inv, build_s_vec
    from aero.lbm.mrt3d import M19, M19_inv, build_s3_vec
    from aero.lbm.trt2d import trt_taus
    omegas = np.array([1.0 / 0.56, 1.0 / 0.5048, 1.0 / 0.53, 1.2, 1.7])
    np.savez_compressed(
        out / "tables.npz", E=E, W=W, OPP=OPP, E3=E3, W3=W3, OPP3=OPP3, Y_MIR3=Y_MIR3,
        M9=M9, M9_inv=M9_inv, M19=M19, M19_inv=M19_inv, omegas=omegas,
        s9=np.array([build_s_vec(o) for o in omegas]),
        s19=np.array([build_s3_vec(o) for o in omegas]),
        trt=np.array([[trt_taus(o, lam) for lam in (0.25, 3.0 / 16.0)] for o in omegas]),
    )


def geometry_fixtures(out):
    """Bit-exact geometry pins for the benchmark configurations."""
    from aero.geometry.cylinder import Cylinder
    from aero.geometry.rectangle import Rectangle
    from aero.geometry3d.sphere import Sphere
    from aero.geometry3d.box import Box
    from aero.lbm.boundary import build_surface_links
    from aero.lbm.boundary3d import build_surface_links_3d
    rec = {}
    # 2D channel (400x200, r=20 at (100,100)), with and without Bouzidi q.
    cyl = Cylinder(radius=20, cx_frac=0.25, cy_frac=0.5)
    solid = cyl.mark_solid(200, 400)
    phi = cyl.sdf_field(200, 400)
    links, q = build_surface_links(solid, phi)
    rec["c1_solid"] = np.packbits(solid)
    rec["c1_links"] = links
    rec["c1_q"] = q
    rec["c1_phi_digest"] = np.array(_digest(phi))
    # 3D sphere 512x256x256, r=16 at (96,128,128), Bouzidi q from its SDF.
    sph = Sphere(radius=16, cx_frac=96 / 512, cy_frac=0.5, cz_frac=0.5)
    solid = sph.mark_solid(256, 256, 512)
    phi = sph.sdf_field(256, 256, 512)
    links, q = build_surface_links_3d(solid, phi)
    rec["c2_solid_digest"] = np.array(_digest(solid))
    rec["c2_n_solid"] = np.array(int(solid.sum()))
    rec["c2_links_digest"] = np.array(_digest(links))
    rec["c2_q_digest"] = np.array(_digest(q))
    rec["c2_n_links"] = np.array(len(links))
    del solid, phi
    # 3D box obstacle 256x128x128: width 24, height 24, depth 128 at x 64..88, y 0..24.
    box = Box(width=24, height=24, depth=128, cx_frac=76 / 256, cy_frac=12 / 128, cz_frac=0.5)
    solid = box.mark_solid(128, 128, 256)
    links, q = build_surface_links_3d(solid, None)
    rec["c3_solid_digest"] = np.array(_digest(solid))
    rec["c3_n_solid"] = np.array(int(solid.sum()))
    rec["c3_links_digest"] = np.array(_digest(links))
    rec["c3_q_digest"] = np.array(_digest(q))
    rec["c3_n_links"] = np.array(len(links))
    # A spread of smaller shapes in full (masks, links, q).
    rng = np.random.default_rng(7)
    small = []
    for k in range(6):
        nx = int(rng.choice(np.arange(64, 161, 16)))
        ny = nx // 2
        if k % 2 == 0:
            g = Cylinder(radius=float(rng.uniform(4, 10)), cx_frac=float(rng.uniform(0.2, 0.4)),
                         cy_frac=float(rng.uniform(0.4, 0.6)))
        else:
            h = float(rng.uniform(4, 10))
            g = Rectangle(width=2 * h, height=2 * h, cx_frac=float(rng.uniform(0.2, 0.4)),
                          cy_frac=float(rng.uniform(0.4, 0.6)))
        s = g.mark_solid(ny, nx)
        p = g.sdf_field(ny, nx)
        l, qq = build_surface_links(s, p)
        small.append(dict(kind="cyl" if k % 2 == 0 else "rect", nx=nx, ny=ny,
                          params=[float(v) for v in vars(g).values()]))
        rec[f"s2_{k}_solid"] = np.packbits(s)
        rec[f"s2_{k}_links"] = l
        rec[f"s2_{k}_q"] = qq
    for k in range(4):
        nx = int(rng.choice(np.arange(32, 65, 8)))
        ny = nz = nx // 2
        if k % 2 == 0:
            g = Sphere(radius=float(rng.uniform(3, 6)), cx_frac=float(rng.uniform(0.2, 0.4)),
                       cy_frac=float(rng.uniform(0.4, 0.6)), cz_frac=float(rng.uniform(0.4, 0.6)))
        else:
            g = Box(width=float(rng.uniform(4, 10)), height=float(rng.uniform(4, 10)),
                    depth=float(rng.uniform(4, 10)), cx_frac=float(rng.uniform(0.2, 0.4)),
                    cy_frac=float(rng.uniform(0.3, 0.6)), cz_frac=float(rng.uniform(0.3, 0.6)))
        s = g.mark_solid(nz, ny, nx)
        p = g.sdf_field(nz, ny, nx)
        l, qq = build_surface_links_3d(s, p)
        small.append(dict(kind="sph" if k % 2 == 0 else "box", nx=nx, ny=ny, nz=nz,
                          params=[float(v) for v in vars(g).values()]))
        rec[f"s3_{k}_solid"] = np.packbits(s)
        rec[f"s3_{k}_links"] = l
        rec[f"s3_{k}_q"] = qq
    rec["small_meta"] = np.array(json.dumps(small))
    np.savez_compressed(out / "geometry.npz", **rec)


def checkpoint_fixtures(out):
    """Checkpoints written by the reference's own save_checkpoint
    (solver.py:638-686, solver3d.py:727-780), one 2D and one 3D thermal case,
    each after `n1` steps from a seeded state, plus the state and histories
    the reference reaches `n2` steps after it and the names of the
    reference constructors' keyword arguments."""
    import inspect

    from aero.lbm.d2q9 import compute_feq
    from aero.lbm.d3q19 import compute_feq_3d
    from aero.lbm.solver import Solver
    from aero.lbm.solver3d import Solver3D

    specs = [
        ("2d", Solver, ("cyl", 4.5, 0.3, 0.5), (24, 48),
         dict(collision="bgk", wall_bc="noslip", outlet_bc="convective", bouzidi=True, thermal=True,
              alpha_T=0.02, buoyancy=True, g_gravity=1e-3, beta=0.5, T_ref=0.5), 0.6, 10, 15),
        ("3d", Solver3D, ("box", 4.0, 4.0, 100.0, 0.4, 2.0 / 10.0, 0.5), (8, 10, 18),
         dict(collision="trt", trt_lambda=3.0 / 16.0, les=True, les_model="wale", les_cs=0.3,
              streamwise_bc="periodic", body_force_x=1e-5, wall_bc="noslip", thermal=True, T_hot=1.0,
              T_cold=0.0, alpha_T=0.01, buoyancy=True, g_gravity=1e-3, beta=1.0, T_ref=0.5), 0.75, 6, 8),
    ]
    for tag, cls, spec, shape, kw, tau, n1, n2 in specs:
        rng = np.random.default_rng(zlib.crc32(f"ckpt_{tag}".encode()))
        if tag == "2d":
            geom, solid, phi = _geometry_2d(spec, *shape)
            s = cls(Ny=shape[0], Nx=shape[1], solid=solid, omega=1.0 / tau, u0=0.05, D=geom.reference_length(),
                    backend="numba", phi=phi, **kw)
            rho = 1.0 + 1e-3 * rng.uniform(-1, 1, shape)
            s.f = np.ascontiguousarray(compute_feq(rho, 0.05 + 2e-3 * rng.uniform(-1, 1, shape),
                                                   2e-3 * rng.uniform(-1, 1, shape)))
            w = s._w
        else:
            geom, solid, phi = _geometry_3d(spec, *shape)
            s = cls(Nz=shape[0], Ny=shape[1], Nx=shape[2], solid=solid, omega=1.0 / tau, u0=0.05,
                    D=geom.reference_length(), backend="numba", phi=phi, **kw)
            rho = 1.0 + 1e-3 * rng.uniform(-1, 1, shape)
            s.f = np.ascontiguousarray(compute_feq_3d(rho, 0.05 + 2e-3 * rng.uniform(-1, 1, shape),
                                                      2e-3 * rng.uniform(-1, 1, shape),
                                                      2e-3 * rng.uniform(-1, 1, shape)))
            w = s._w_np
        T0 = 0.5 + 0.05 * rng.uniform(-1, 1, shape)
        s.g = np.ascontiguousarray(w.reshape((-1,) + (1,) * len(shape)) * T0[None])
        s.run(n1, check_every=n1 + 1, verbose=False)
        s.save_checkpoint(str(out / f"ckpt_ref_{tag}.npz"))
        s.run(n2, check_every=n2 + 1, verbose=False)
        hist = {k: np.array(getattr(s, k), dtype=np.float64) for k in
                (("Cd_history", "Cl_history", "Cm_history") if tag == "2d" else
                 ("Cd_history", "Cly_history", "Clz_history", "Cmx_history", "Cmy_history", "Cmz_history"))}
        names = [n for n in inspect.signature(cls.__init__).parameters if n != "self"]
        np.savez_compressed(out / f"ckpt_cont_{tag}.npz", f=s.f, f_outlet_prev=s._f_outlet_prev, g=s.g,
                            step_count=np.array(s.step_count), n2=np.array(n2),
                            ctor_params=np.array(json.dumps(names)), **hist)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the Aero checkout")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    sys.path.insert(0, str(pathlib.Path(args.reference).resolve()))
    out = HERE
    tables(out)
    for name, spec, kw, steps in CASES_2D:
        if args.only and args.only not in name:
            continue
        run_case_2d(name, spec, kw, steps, out)
        print("wrote", name, flush=True)
    for name, spec, kw, steps in CASES_3D:
        if args.only and args.only not in name:
            continue
        run_case_3d(name, spec, kw, steps, out)
        print("wrote", name, flush=True)
    if not args.only:
        geometry_fixtures(out)
        print("wrote geometry", flush=True)
    if not args.only or "ckpt" in args.only:
        checkpoint_fixtures(out)
        print("wrote checkpoints", flush=True)


if __name__ == "__main__":
    main()
