"""Generate the golden vectors in tests/golden/*.npz by executing the EDGE
reference's own Python sources (sim/*.py, util/taichi_utils.py and the step
kernels of run_edge.py / run_ed4.py / run_ed8.py / run_ge.py / run_efm.py) on
tiny seeded grids.

Taichi 1.7.3 is not installable here, so the sources run on the numpy
emulation of the Taichi subset they use (``_taichi_emu/taichi``); it keeps
Taichi's float32 arithmetic, pass-by-reference ``ti.template()`` function
parameters and serial parallel-for semantics.  The fixtures therefore pin the
oracle and the CUDA kernels to the reference's own code paths, not to Taichi's
code generator (FMA contraction and atomic ordering differ, which the tests
absorb through their tolerances).

Run from the repository root in a container that has the reference checked
out (it is read-only there)::

    python tests/golden/make_golden.py [--ref /root/reference] [--only NAME] [--force]

Each fixture is an .npz of float32/int32 arrays; ``meta_*`` entries hold the
scalars (dx, dt, epsilon, iteration counts).
"""
import argparse
import ast
import contextlib
import io
import os
import re
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

ap = argparse.ArgumentParser()
ap.add_argument("--ref", default="/root/reference")
ap.add_argument("--only", default=None)
ap.add_argument("--force", action="store_true")
args = ap.parse_args()

sys.path.insert(0, os.path.join(HERE, "_taichi_emu"))
sys.path.insert(1, args.ref)

import taichi as ti  # noqa: E402  (the emulation)

ti.init(arch=ti.cpu, debug=False, default_fp=ti.f32)

import util.taichi_utils as tu  # noqa: E402
import sim.hermite as H  # noqa: E402
import sim.mgpcg as MG  # noqa: E402
import sim.mgpcg_solid as MGS  # noqa: E402
import sim.lp as LP  # noqa: E402
import sim.init_conditions as IC  # noqa: E402

F32 = np.float32


def load_driver_kernels(fname, names, extra_globals):
    """Compile selected top-level functions of a run_*.py driver (which is a
    script and cannot be imported) in a namespace that provides the module
    globals those kernels read."""
    path = os.path.join(args.ref, fname)
    tree = ast.parse(open(path).read(), path)
    defs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    missing = set(names) - {d.name for d in defs}
    assert not missing, missing
    mod = ast.Module(body=defs, type_ignores=[])
    ns = {}
    exec("from util.taichi_utils import *\nfrom sim.hermite import *", ns)
    ns.update(extra_globals)
    exec(compile(mod, path, "exec"), ns)
    return ns


# ---------------------------------------------------------------------------
# seeded inputs
# ---------------------------------------------------------------------------
def smooth_noise(rng, shape, dx, nmodes=4, amp=1.0):
    """Sum of a few random plane waves sampled at the cell/face positions of
    ``shape`` (float64 -> float32)."""
    idx = np.indices(shape).astype(np.float64)
    out = np.zeros(shape)
    for _ in range(nmodes):
        k = rng.uniform(0.5, 2.5, size=3) * 2 * np.pi
        ph = rng.uniform(0, 2 * np.pi)
        a = rng.normal()
        out += a * np.sin(k[0] * idx[0] * dx + k[1] * idx[1] * dx + k[2] * idx[2] * dx + ph)
    out *= amp / max(1e-9, np.abs(out).max())
    return out.astype(F32)


def vfield(shape):
    return ti.Vector.field(3, float, shape=shape)


def sfield(shape):
    return ti.field(float, shape=shape)


def from_np(arr, vec=None):
    arr = np.ascontiguousarray(arr, dtype=F32)
    if vec is None:
        f = sfield(arr.shape)
    else:
        f = ti.Vector.field(vec, float, shape=arr.shape[:-1])
    f.from_numpy(arr)
    return f


class Grid:
    def __init__(self, res, dx):
        self.res = tuple(res)
        nx, ny, nz = res
        self.dx = F32(dx)
        self.X = vfield(res)
        self.X_x = vfield((nx + 1, ny, nz))
        self.X_y = vfield((nx, ny + 1, nz))
        self.X_z = vfield((nx, ny, nz + 1))
        tu.center_coords_func(self.X, dx)
        tu.x_coords_func(self.X_x, dx)
        tu.y_coords_func(self.X_y, dx)
        tu.z_coords_func(self.X_z, dx)

    def faces(self):
        nx, ny, nz = self.res
        return [(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)]


def velocity(rng, g, amp=1.0):
    return [from_np(smooth_noise(rng, s, float(g.dx), amp=amp)) for s in g.faces()]


def map_state(rng, g, with_dT=True, with_d2T=False):
    """A non-identity backward map: psi = X + small smooth displacement, with
    T and dT perturbed around the identity / zero."""
    res = g.res
    dx = float(g.dx)
    X = g.X.to_numpy()
    psi = X + 0.4 * dx * np.stack([smooth_noise(rng, res, dx) for _ in range(3)], -1)
    T = [np.eye(3, dtype=F32)[c][None, None, None, :] + 0.08 * np.stack(
        [smooth_noise(rng, res, dx) for _ in range(3)], -1) for c in range(3)]
    out = {"psi": from_np(psi, 3), "T": [from_np(t, 3) for t in T]}
    if with_dT:
        out["dT"] = [from_np(0.6 * np.stack([smooth_noise(rng, res, dx) for _ in range(3)], -1), 3)
                     for _ in range(3)]
    if with_d2T:
        out["d2T"] = [from_np(0.5 * smooth_noise(rng, res, dx)) for _ in range(3)]
    return out


def smoke_field(rng, g):
    return from_np(rng.uniform(0, 1, size=g.res + (4,)), 4)


def dt_for(u, g, cfl=0.5):
    m = max(float(np.abs(f.to_numpy()).max()) for f in u)
    return F32(cfl * float(g.dx) / m)


def save(name, **arrays):
    out = {}
    for k, v in arrays.items():
        if isinstance(v, (ti.Field,)):
            v = v.to_numpy()
        out[k] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"  wrote {name}.npz ({sum(a.nbytes for a in out.values()) / 1024:.1f} KiB raw)")


def fixture(fn):
    FIXTURES.append(fn)
    return fn


FIXTURES = []
G_SMALL = ((8, 6, 5), 1.0 / 6.0)


# ---------------------------------------------------------------------------
# fixtures
# ---------------------------------------------------------------------------
@fixture
def interp_points():
    """B-spline, trilinear and Hermite point samplers (taichi_utils.py:120-341,
    hermite.py:65-607) at random points, some outside the grid (clamps)."""
    rng = np.random.default_rng(101)
    g = Grid(*G_SMALL)
    u = velocity(rng, g)
    ms = map_state(rng, g, with_dT=True, with_d2T=True)
    smoke = smoke_field(rng, g)
    L = np.array(g.res) * float(g.dx)
    npts = 96
    P = rng.uniform(-0.15, 1.0, size=(npts, 3)) * (L + 0.3)
    P[:8] = rng.uniform(0, 1, size=(8, 3)) * L  # keep a few strictly inside
    pts = from_np(P, 3)
    outs = {k: sfield((npts,)) for k in ["i2x", "i2y", "i2z"]}
    g2 = {k: vfield((npts,)) for k in ["g2x", "g2y", "g2z"]}
    macv = vfield((npts,))
    macg_v = vfield((npts,))
    macg_g = [vfield((npts,)) for _ in range(3)]
    lin = ti.Vector.field(4, float, shape=(npts,))
    mn = ti.Vector.field(4, float, shape=(npts,))
    mx = ti.Vector.field(4, float, shape=(npts,))
    h_fd = vfield((npts,))
    hg_fd = [vfield((npts,)) for _ in range(3)]
    hg_fd_v = vfield((npts,))
    h_garm = vfield((npts,))
    hg_garm = [vfield((npts,)) for _ in range(3)]
    hg_garm_v = vfield((npts,))
    h_full = vfield((npts,))
    hg_full = [vfield((npts,)) for _ in range(3)]
    hg_full_v = vfield((npts,))
    u_x, u_y, u_z = u
    psi = ms["psi"]
    T_x, T_y, T_z = ms["T"]
    dT_x, dT_y, dT_z = ms["dT"]
    d2T_x, d2T_y, d2T_z = ms["d2T"]
    dx = g.dx

    @ti.kernel
    def run(dx: float):
        for I in ti.grouped(pts):
            p = pts[I]
            outs["i2x"][I] = tu.interp_2(u_x, p, dx, BL_x=0.0, BL_y=0.5, BL_z=0.5)
            outs["i2y"][I] = tu.interp_2(u_y, p, dx, BL_x=0.5, BL_y=0.0, BL_z=0.5)
            outs["i2z"][I] = tu.interp_2(u_z, p, dx, BL_x=0.5, BL_y=0.5, BL_z=0.0)
            v, gr = tu.interp_grad_2(u_x, p, dx, BL_x=0.0, BL_y=0.5, BL_z=0.5)
            g2["g2x"][I] = gr
            v, gr = tu.interp_grad_2(u_y, p, dx, BL_x=0.5, BL_y=0.0, BL_z=0.5)
            g2["g2y"][I] = gr
            v, gr = tu.interp_grad_2(u_z, p, dx, BL_x=0.5, BL_y=0.5, BL_z=0.0)
            g2["g2z"][I] = gr
            macv[I] = tu.interp_u_MAC(u_x, u_y, u_z, p, dx)
            vv, gg = tu.interp_u_MAC_grad(u_x, u_y, u_z, p, dx)
            macg_v[I] = vv
            macg_g[0][I] = gg[0, :]
            macg_g[1][I] = gg[1, :]
            macg_g[2][I] = gg[2, :]
            lin[I] = tu.interp_1(smoke, p, dx)
            a, b = tu.sample_min_max_1(smoke, p, dx)
            mn[I] = a
            mx[I] = b
            h_fd[I] = ti.Vector([H.interp_hermite_fd_unroll(psi, 0, T_x, p, dx),
                                 H.interp_hermite_fd_unroll(psi, 1, T_y, p, dx),
                                 H.interp_hermite_fd_unroll(psi, 2, T_z, p, dx)])
            a0, b0 = H.interp_grad_hermite_fd_unroll(psi, 0, T_x, p, dx)
            a1, b1 = H.interp_grad_hermite_fd_unroll(psi, 1, T_y, p, dx)
            a2, b2 = H.interp_grad_hermite_fd_unroll(psi, 2, T_z, p, dx)
            hg_fd_v[I] = ti.Vector([a0, a1, a2])
            hg_fd[0][I] = b0
            hg_fd[1][I] = b1
            hg_fd[2][I] = b2
            h_garm[I] = ti.Vector([H.interp_hermite_garm_fd_unroll(psi, 0, T_x, dT_x, p, dx),
                                   H.interp_hermite_garm_fd_unroll(psi, 1, T_y, dT_y, p, dx),
                                   H.interp_hermite_garm_fd_unroll(psi, 2, T_z, dT_z, p, dx)])
            a0, b0 = H.interp_grad_hermite_garm_fd_unroll(psi, 0, T_x, dT_x, p, dx)
            a1, b1 = H.interp_grad_hermite_garm_fd_unroll(psi, 1, T_y, dT_y, p, dx)
            a2, b2 = H.interp_grad_hermite_garm_fd_unroll(psi, 2, T_z, dT_z, p, dx)
            hg_garm_v[I] = ti.Vector([a0, a1, a2])
            hg_garm[0][I] = b0
            hg_garm[1][I] = b1
            hg_garm[2][I] = b2
            h_full[I] = ti.Vector([H.interp_hermite(psi, 0, T_x, dT_x, d2T_x, p, dx),
                                   H.interp_hermite(psi, 1, T_y, dT_y, d2T_y, p, dx),
                                   H.interp_hermite(psi, 2, T_z, dT_z, d2T_z, p, dx)])
            a0, b0 = H.interp_grad_hermite(psi, 0, T_x, dT_x, d2T_x, p, dx)
            a1, b1 = H.interp_grad_hermite(psi, 1, T_y, dT_y, d2T_y, p, dx)
            a2, b2 = H.interp_grad_hermite(psi, 2, T_z, dT_z, d2T_z, p, dx)
            hg_full_v[I] = ti.Vector([a0, a1, a2])
            hg_full[0][I] = b0
            hg_full[1][I] = b1
            hg_full[2][I] = b2

    run(dx)
    save("interp_points", meta_dx=dx, res=np.array(g.res), pts=pts, u_x=u_x, u_y=u_y, u_z=u_z,
         smoke=smoke, psi=psi, T_x=T_x, T_y=T_y, T_z=T_z, dT_x=dT_x, dT_y=dT_y, dT_z=dT_z,
         d2T_x=d2T_x, d2T_y=d2T_y, d2T_z=d2T_z,
         interp2_x=outs["i2x"], interp2_y=outs["i2y"], interp2_z=outs["i2z"],
         grad2_x=g2["g2x"], grad2_y=g2["g2y"], grad2_z=g2["g2z"],
         mac_v=macv, macg_v=macg_v, macg_gx=macg_g[0], macg_gy=macg_g[1], macg_gz=macg_g[2],
         lin=lin, minv=mn, maxv=mx,
         herm_fd=h_fd, hermg_fd_v=hg_fd_v, hermg_fd_x=hg_fd[0], hermg_fd_y=hg_fd[1], hermg_fd_z=hg_fd[2],
         herm_garm=h_garm, hermg_garm_v=hg_garm_v, hermg_garm_x=hg_garm[0], hermg_garm_y=hg_garm[1],
         hermg_garm_z=hg_garm[2],
         herm_full=h_full, hermg_full_v=hg_full_v, hermg_full_x=hg_full[0], hermg_full_y=hg_full[1],
         hermg_full_z=hg_full[2])


@fixture
def march_edge():
    """EDGE march advect_psi_garm_ed4_fusion_unroll (hermite.py:1427-1521)."""
    rng = np.random.default_rng(202)
    g = Grid(*G_SMALL)
    u = velocity(rng, g)
    ms = map_state(rng, g)
    dt = dt_for(u, g)
    eps = F32(0.025 * float(g.dx))
    inputs = {"psi": ms["psi"].to_numpy(), **{f"T_{a}": ms["T"][i].to_numpy() for i, a in enumerate("xyz")},
              **{f"dT_{a}": ms["dT"][i].to_numpy() for i, a in enumerate("xyz")}}
    tmp = [vfield(g.res) for _ in range(7)]
    H.advect_psi_garm_ed4_fusion_unroll(*tmp, ms["psi"], *ms["T"], *ms["dT"], *u, g.X, g.dx, dt, eps)
    save("march_edge", meta_dx=g.dx, meta_dt=dt, meta_eps=eps, res=np.array(g.res),
         u_x=u[0], u_y=u[1], u_z=u[2], **{"in_" + k: v for k, v in inputs.items()},
         out_psi=ms["psi"], out_T_x=ms["T"][0], out_T_y=ms["T"][1], out_T_z=ms["T"][2],
         out_dT_x=ms["dT"][0], out_dT_y=ms["dT"][1], out_dT_z=ms["dT"][2])


@fixture
def march_ed4():
    """ED4 march advect_ps_hermite_ed4_fd_unroll (hermite.py:1375-1395)."""
    rng = np.random.default_rng(303)
    g = Grid(*G_SMALL)
    u = velocity(rng, g)
    ms = map_state(rng, g, with_dT=False)
    dt = dt_for(u, g)
    eps = F32(0.025 * float(g.dx))
    inputs = {"psi": ms["psi"].to_numpy(), **{f"T_{a}": ms["T"][i].to_numpy() for i, a in enumerate("xyz")}}
    pts = [vfield(g.res) for _ in range(4)]
    H.advect_ps_hermite_ed4_fd_unroll(*pts, ms["psi"], *ms["T"], *u, g.X, g.dx, dt, eps)
    save("march_ed4", meta_dx=g.dx, meta_dt=dt, meta_eps=eps, res=np.array(g.res),
         u_x=u[0], u_y=u[1], u_z=u[2], **{"in_" + k: v for k, v in inputs.items()},
         out_psi=ms["psi"], out_T_x=ms["T"][0], out_T_y=ms["T"][1], out_T_z=ms["T"][2])


@fixture
def march_ed8():
    """ED8 march advect_ps_hermite_ed8 (hermite.py:1290-1338) followed by the
    face split split_psi_hermite (run_ed8.py:191-224)."""
    rng = np.random.default_rng(404)
    g = Grid(*G_SMALL)
    u = velocity(rng, g)
    ms = map_state(rng, g, with_dT=True, with_d2T=True)
    dt = dt_for(u, g)
    eps = F32(0.025 * float(g.dx))
    inputs = {"psi": ms["psi"].to_numpy(), **{f"T_{a}": ms["T"][i].to_numpy() for i, a in enumerate("xyz")},
              **{f"dT_{a}": ms["dT"][i].to_numpy() for i, a in enumerate("xyz")},
              **{f"d2T_{a}": ms["d2T"][i].to_numpy() for i, a in enumerate("xyz")}}
    pts = [vfield(g.res) for _ in range(8)]
    H.advect_ps_hermite_ed8(*pts, ms["psi"], *ms["T"], *ms["dT"], *ms["d2T"], *u, g.X, g.dx, dt, eps)
    fx, fy, fz = g.faces()
    Tf = [vfield(fx), vfield(fy), vfield(fz)]
    Pf = [vfield(fx), vfield(fy), vfield(fz)]
    ns = load_driver_kernels("run_ed8.py", ["split_psi_hermite"], dict(
        T_x=Tf[0], T_y=Tf[1], T_z=Tf[2], psi_x=Pf[0], psi_y=Pf[1], psi_z=Pf[2],
        psi_ed=ms["psi"], T_x_ed=ms["T"][0], T_y_ed=ms["T"][1], T_z_ed=ms["T"][2],
        dT_x_ed=ms["dT"][0], dT_y_ed=ms["dT"][1], dT_z_ed=ms["dT"][2],
        d2T_x_ed=ms["d2T"][0], d2T_y_ed=ms["d2T"][1], d2T_z_ed=ms["d2T"][2],
        X_x=g.X_x, X_y=g.X_y, X_z=g.X_z, dx=g.dx))
    ns["split_psi_hermite"]()
    save("march_ed8", meta_dx=g.dx, meta_dt=dt, meta_eps=eps, res=np.array(g.res),
         u_x=u[0], u_y=u[1], u_z=u[2], **{"in_" + k: v for k, v in inputs.items()},
         out_psi=ms["psi"], out_T_x=ms["T"][0], out_T_y=ms["T"][1], out_T_z=ms["T"][2],
         out_dT_x=ms["dT"][0], out_dT_y=ms["dT"][1], out_dT_z=ms["dT"][2],
         out_d2T_x=ms["d2T"][0], out_d2T_y=ms["d2T"][1], out_d2T_z=ms["d2T"][2],
         face_psi_x=Pf[0], face_psi_y=Pf[1], face_psi_z=Pf[2],
         face_T_x=Tf[0], face_T_y=Tf[1], face_T_z=Tf[2])


@fixture
def march_ge():
    """GE march advect_ps_garm (hermite.py:1398-1424, which ends in
    calc_fd_3_from_grad, hermite.py:1180-1256) followed by the face split of
    run_ge.py:185-217."""
    rng = np.random.default_rng(505)
    g = Grid(*G_SMALL)
    u = velocity(rng, g)
    ms = map_state(rng, g, with_dT=True, with_d2T=True)
    dt = dt_for(u, g)
    inputs = {"psi": ms["psi"].to_numpy(), **{f"T_{a}": ms["T"][i].to_numpy() for i, a in enumerate("xyz")},
              **{f"dT_{a}": ms["dT"][i].to_numpy() for i, a in enumerate("xyz")},
              **{f"d2T_{a}": ms["d2T"][i].to_numpy() for i, a in enumerate("xyz")}}
    tmp = [vfield(g.res) for _ in range(4)]
    H.advect_ps_garm(*tmp, ms["psi"], *ms["T"], *ms["dT"], *ms["d2T"], *u, g.X, g.dx, dt)
    fx, fy, fz = g.faces()
    Tf = [vfield(fx), vfield(fy), vfield(fz)]
    Pf = [vfield(fx), vfield(fy), vfield(fz)]
    ns = load_driver_kernels("run_ge.py", ["split_psi_hermite"], dict(
        T_x=Tf[0], T_y=Tf[1], T_z=Tf[2], psi_x=Pf[0], psi_y=Pf[1], psi_z=Pf[2],
        psi_garm=ms["psi"], T_x_garm=ms["T"][0], T_y_garm=ms["T"][1], T_z_garm=ms["T"][2],
        dT_x_garm=ms["dT"][0], dT_y_garm=ms["dT"][1], dT_z_garm=ms["dT"][2],
        d2T_x_garm=ms["d2T"][0], d2T_y_garm=ms["d2T"][1], d2T_z_garm=ms["d2T"][2],
        X_x=g.X_x, X_y=g.X_y, X_z=g.X_z, dx=g.dx))
    ns["split_psi_hermite"]()
    save("march_ge", meta_dx=g.dx, meta_dt=dt, res=np.array(g.res),
         u_x=u[0], u_y=u[1], u_z=u[2], **{"in_" + k: v for k, v in inputs.items()},
         out_psi=ms["psi"], out_T_x=ms["T"][0], out_T_y=ms["T"][1], out_T_z=ms["T"][2],
         out_dT_x=ms["dT"][0], out_dT_y=ms["dT"][1], out_dT_z=ms["dT"][2],
         out_d2T_x=ms["d2T"][0], out_d2T_y=ms["d2T"][1], out_d2T_z=ms["d2T"][2],
         face_psi_x=Pf[0], face_psi_y=Pf[1], face_psi_z=Pf[2],
         face_T_x=Tf[0], face_T_y=Tf[1], face_T_z=Tf[2])


@fixture
def efm_backtrack():
    """EFM backward map: backtrack_psi_grid (run_efm.py:179-186) through three
    cached velocity fields with their step sizes, from the identity."""
    rng = np.random.default_rng(606)
    g = Grid(*G_SMALL)
    nsteps = 3
    cache = [velocity(rng, g, amp=0.7) for _ in range(nsteps)]
    u_cur = [from_np(c.to_numpy()) for c in cache[-1]]  # the driver copies u into slot j before backtracking
    dts = sfield((nsteps,))
    dts.from_numpy(np.array([dt_for(c, g, 0.4) for c in cache], F32))
    fx, fy, fz = g.faces()
    psi = [vfield(fx), vfield(fy), vfield(fz)]
    T = [vfield(fx), vfield(fy), vfield(fz)]
    tmp = [sfield(s) for s in g.faces()]
    ns = load_driver_kernels("run_efm.py", ["reset_to_identity", "advance_map", "march_no_neural",
                                            "backtrack_psi_grid"], dict(
        psi_x=psi[0], psi_y=psi[1], psi_z=psi[2], T_x=T[0], T_y=T[1], T_z=T[2],
        u_x=u_cur[0], u_y=u_cur[1], u_z=u_cur[2], tmp_u_x=tmp[0], tmp_u_y=tmp[1], tmp_u_z=tmp[2],
        u_x_cache=[c[0] for c in cache], u_y_cache=[c[1] for c in cache], u_z_cache=[c[2] for c in cache],
        dts=dts, X_x=g.X_x, X_y=g.X_y, X_z=g.X_z, dx=g.dx))
    ns["backtrack_psi_grid"](nsteps - 1)
    out = dict(meta_dx=g.dx, res=np.array(g.res), dts=dts, out_psi_x=psi[0], out_psi_y=psi[1], out_psi_z=psi[2],
               out_T_x=T[0], out_T_y=T[1], out_T_z=T[2])
    for s, c in enumerate(cache):
        for a, f in zip("xyz", c):
            out[f"u{s}_{a}"] = f
    save("efm_backtrack", **out)


@fixture
def lp_init_positions():
    """Laden-particle initial positions of the ink cases (lp_init.py:6-20,
    69-86): the reference's seeded rejection sampling, 300 particles each."""
    import sim.lp_init as LPI
    out = {}
    for case, fn in ((0, LPI.ink_drop_particle_case0), (1, LPI.ink_drop_particle_case1)):
        pos = ti.Vector.field(3, float, shape=(300,))
        fn(pos, 300)
        out[f"pos_case{case}"] = pos
    save("lp_init_positions", **out)


@fixture
def advect_faces():
    """Semi-Lagrangian advect_u_semi_lagrangian (hermite.py:1578-1621), the
    forward-map march advance_map (run_edge.py:337-357), map_u
    (run_edge.py:361-373), clamp_u (run_edge.py:509-519) and calc_max_speed
    (run_edge.py:296-303)."""
    rng = np.random.default_rng(505)
    g = Grid(*G_SMALL)
    u = velocity(rng, g)
    dt = dt_for(u, g)
    out = [sfield(s) for s in g.faces()]
    H.advect_u_semi_lagrangian(*u, *out, g.dx, F32(0.5) * dt, g.X_x, g.X_y, g.X_z)
    # forward map: start from a perturbed state so F is not the identity
    fx, fy, fz = g.faces()
    phis, Fs = [], []
    for c, (shape, Xf) in enumerate(zip(g.faces(), [g.X_x, g.X_y, g.X_z])):
        phis.append(from_np(Xf.to_numpy() + 0.3 * float(g.dx) * np.stack(
            [smooth_noise(rng, shape, float(g.dx)) for _ in range(3)], -1), 3))
        Fs.append(from_np(np.eye(3, dtype=F32)[c] + 0.05 * np.stack(
            [smooth_noise(rng, shape, float(g.dx)) for _ in range(3)], -1), 3))
    phi_in = [p.to_numpy() for p in phis]
    F_in = [f.to_numpy() for f in Fs]
    max_speed = ti.field(float, shape=())
    nx, ny, nz = g.res
    ns = load_driver_kernels("run_edge.py", ["advance_map", "map_u", "clamp_u", "calc_max_speed"], dict(
        dx=g.dx, res_x=nx, res_y=ny, res_z=nz, max_speed=max_speed))
    for p, f in zip(phis, Fs):
        ns["advance_map"](p, f, *u, dt)
    mapped = [sfield(s) for s in g.faces()]
    ns["map_u"](*u, *mapped, *Fs, *phis, g.dx)
    other = [from_np(f.to_numpy() + 0.1 * smooth_noise(rng, f.shape, float(g.dx))) for f in u]
    clamped = [sfield(s) for s in g.faces()]
    for a, b, c in zip(other, u, clamped):
        ns["clamp_u"](a, b, c)
    ns["calc_max_speed"](*u)
    save("advect_faces", meta_dx=g.dx, meta_dt=dt, res=np.array(g.res),
         u_x=u[0], u_y=u[1], u_z=u[2], sl_x=out[0], sl_y=out[1], sl_z=out[2],
         phi_in_x=phi_in[0], phi_in_y=phi_in[1], phi_in_z=phi_in[2],
         F_in_x=F_in[0], F_in_y=F_in[1], F_in_z=F_in[2],
         phi_out_x=phis[0], phi_out_y=phis[1], phi_out_z=phis[2],
         F_out_x=Fs[0], F_out_y=Fs[1], F_out_z=Fs[2],
         mapu_x=mapped[0], mapu_y=mapped[1], mapu_z=mapped[2],
         clamp_in_x=other[0], clamp_in_y=other[1], clamp_in_z=other[2],
         clamp_x=clamped[0], clamp_y=clamped[1], clamp_z=clamped[2],
         meta_max_speed=max_speed[None])


def _pullback_fixture(name, variant, seed):
    rng = np.random.default_rng(seed)
    g = Grid(*G_SMALL)
    u0 = velocity(rng, g)
    ms = map_state(rng, g, with_dT=(variant == "edge"))
    smoke0 = smoke_field(rng, g)
    smoke_cur = smoke_field(rng, g)
    nx, ny, nz = g.res
    glb = dict(dx=g.dx, res_x=nx, res_y=ny, res_z=nz, X_x=g.X_x, X_y=g.X_y, X_z=g.X_z)
    if variant == "edge":
        glb.update(psi_garm=ms["psi"], T_x_garm=ms["T"][0], T_y_garm=ms["T"][1], T_z_garm=ms["T"][2],
                   dT_x_garm=ms["dT"][0], dT_y_garm=ms["dT"][1], dT_z_garm=ms["dT"][2])
        drv = "run_edge.py"
    else:
        glb.update(psi_ed=ms["psi"], T_x_ed=ms["T"][0], T_y_ed=ms["T"][1], T_z_ed=ms["T"][2])
        drv = "run_ed4.py"
    ns = load_driver_kernels(drv, ["map_u_psi", "split_to_mac", "map_smoke_psi", "clamp_smoke_psi",
                                   "map_smoke", "clamp_smoke"], glb)
    u1 = [sfield(s) for s in g.faces()]
    ns["map_u_psi"](*u0, *u1, g.dx)
    smoke1 = ti.Vector.field(4, float, shape=g.res)
    ns["map_smoke_psi"](smoke0, smoke1, g.dx)
    clamped = from_np(smoke_cur.to_numpy(), 4)
    ns["clamp_smoke_psi"](smoke0, clamped, g.dx)
    # forward-map dye pullback / clamp through face maps (run_edge.py:421-427, 470-477)
    phis = []
    for shape, Xf in zip(g.faces(), [g.X_x, g.X_y, g.X_z]):
        phis.append(from_np(Xf.to_numpy() + 0.3 * float(g.dx) * np.stack(
            [smooth_noise(rng, shape, float(g.dx)) for _ in range(3)], -1), 3))
    smoke2 = ti.Vector.field(4, float, shape=g.res)
    ns["map_smoke"](smoke0, smoke2, *phis, g.dx)
    clamped2 = from_np(smoke_cur.to_numpy(), 4)
    ns["clamp_smoke"](smoke0, clamped2, *phis, g.dx)
    arrs = dict(meta_dx=g.dx, res=np.array(g.res), u0_x=u0[0], u0_y=u0[1], u0_z=u0[2],
                psi=ms["psi"], T_x=ms["T"][0], T_y=ms["T"][1], T_z=ms["T"][2],
                smoke0=smoke0, smoke_cur=smoke_cur,
                u1_x=u1[0], u1_y=u1[1], u1_z=u1[2], smoke1=smoke1, smoke_clamped=clamped,
                phi_x=phis[0], phi_y=phis[1], phi_z=phis[2], smoke_fwd=smoke2, smoke_fwd_clamped=clamped2)
    if variant == "edge":
        arrs.update(dT_x=ms["dT"][0], dT_y=ms["dT"][1], dT_z=ms["dT"][2])
    save(name, **arrs)


@fixture
def pullback_edge():
    """EDGE map_u_psi / map_smoke_psi / clamp_smoke_psi (run_edge.py:377-505)
    plus map_smoke / clamp_smoke (run_edge.py:421-427, 470-477)."""
    _pullback_fixture("pullback_edge", "edge", 606)


@fixture
def pullback_ed4():
    """ED4 map_u_psi / map_smoke_psi / clamp_smoke_psi (run_ed4.py:219-336)."""
    _pullback_fixture("pullback_ed4", "ed4", 707)


def _capture_solve(fn):
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        fn()
    text = buf.getvalue()
    m = re.search(r"Converged at iter:\s+(\d+)", text)
    it = int(m.group(1)) if m else -1
    if it < 0:
        m = re.search(r"without converging at iter:\s+(\d+)", text)
        it = -int(m.group(1)) if m else -999
    return it, text


@fixture
def mgpcg_plain():
    """MGPCG_3.Poisson (mgpcg.py:364-445) on a 16x8x8 grid with 3 levels
    (base_level=1) and all-Neumann walls; also records one V-cycle
    application (apply_preconditioner, mgpcg.py:177-195) and one Ap."""
    rng = np.random.default_rng(808)
    res = (16, 8, 8)
    g = Grid(res, 1.0 / 8.0)
    u = velocity(rng, g)
    u_in = [f.to_numpy() for f in u]
    bt = ti.Matrix([[2, 2], [2, 2], [2, 2]], ti.i32)
    solver = MG.MGPCG_3(boundary_types=bt, N=list(res), base_level=1, real=ti.f32)
    it, text = _capture_solve(lambda: solver.Poisson(*u))
    div = solver.u_div.to_numpy()
    pres = solver.p.to_numpy()
    # one preconditioner application on a seeded right-hand side
    rhs = rng.normal(size=res).astype(F32)
    solver.r[0].from_numpy(rhs)
    solver.apply_preconditioner()
    z = solver.z[0].to_numpy()
    solver.p.from_numpy(rhs)
    solver.compute_Ap()
    Ap = solver.Ap.to_numpy()
    save("mgpcg_plain", res=np.array(res), meta_iters=it, meta_levels=solver.n_mg_levels,
         u_in_x=u_in[0], u_in_y=u_in[1], u_in_z=u_in[2], div=div, pressure=pres,
         u_out_x=u[0], u_out_y=u[1], u_out_z=u[2], vc_rhs=rhs, vc_z=z, ap_out=Ap)
    print("   ", text.strip().splitlines()[-1])


@fixture
def mgpcg_solid():
    """MGPCG_Solid_3.Poisson (mgpcg_solid.py:313-427) with a solid block and a
    solid outer shell carrying a prescribed velocity."""
    rng = np.random.default_rng(909)
    res = (16, 8, 8)
    g = Grid(res, 1.0 / 8.0)
    u = velocity(rng, g, amp=0.5)
    mask = np.zeros(res, np.int32)
    mask[0, :, :] = mask[-1, :, :] = 1
    mask[:, 0, :] = mask[:, -1, :] = 1
    mask[:, :, 0] = mask[:, :, -1] = 1
    mask[6:9, 3:5, 2:6] = 1
    bvel = np.zeros(res + (3,), F32)
    bvel[mask > 0] = np.array([0.6, 0.0, 0.2], F32)
    bvel[6:9, 3:5, 2:6] = 0.0
    u_in = [f.to_numpy() for f in u]
    bm = ti.field(ti.i32, shape=res)
    bm.from_numpy(mask)
    bv = from_np(bvel, 3)
    bt = ti.Matrix([[2, 2], [2, 2], [2, 2]], ti.i32)
    solver = MGS.MGPCG_Solid_3(boundary_types=bt, boundary_mask=bm, boundary_vel=bv, N=list(res),
                               base_level=1, real=ti.f32)
    it, text = _capture_solve(lambda: solver.Poisson(*u))
    m = re.findall(r"Sum of fluid div:\s+(\S+)", text)
    save("mgpcg_solid", res=np.array(res), meta_iters=it, meta_levels=solver.n_mg_levels,
         mask=mask, bvel=bvel, u_in_x=u_in[0], u_in_y=u_in[1], u_in_z=u_in[2],
         div=solver.u_div.to_numpy(), pressure=solver.p.to_numpy(),
         u_out_x=u[0], u_out_y=u[1], u_out_z=u[2],
         bm1=solver.bm[1].to_numpy(), bm2=solver.bm[2].to_numpy(),
         meta_div_sum=float(m[0]) if m else 0.0)
    print("   ", text.strip().splitlines()[-1])


@fixture
def particles():
    """Laden-particle kernels of sim/lp.py (G2P lp.py:7-29, 74-97; particle
    update 33-70, 159-181; P2G drag scatter 101-156; viscous force 184-219)."""
    rng = np.random.default_rng(1010)
    res = (12, 10, 8)
    dx = 1.0
    g = Grid(res, dx)
    u = velocity(rng, g)
    n = 64
    L = np.array(res, np.float64) * dx
    pos = rng.uniform(0.0, 1.0, size=(n, 3)) * L
    pos[:40] = rng.uniform(0.3, 0.7, size=(40, 3)) * L  # most inside the 3dx margin
    vel = rng.normal(size=(n, 3)) * 0.3
    rad = rng.uniform(0.005, 0.015, size=n)
    P = from_np(pos, 3)
    V = from_np(vel, 3)
    acc = vfield((n,))
    vdiff = vfield((n,))
    R = from_np(rad)
    drag = [sfield(s) for s in g.faces()]
    vis = [sfield(s) for s in g.faces()]
    num = n - 4  # the last four particles are beyond laden_particle_num
    dt, St, grav, dens, erad, Re, lrad = 0.05, 6.6e-2, 1.0, 2.0 / 3, 35.0, 5.5, 0.01
    LP.update_particles_acc(*u, V, P, acc, g.dx, dt, num, St, grav)
    acc0 = acc.to_numpy()
    LP.update_particles_velocity(acc, V, P, dt, g.dx, num, *[float(v) for v in L])
    vel1 = V.to_numpy()
    LP.calculate_velocity_diff(*u, V, vdiff, P, g.dx, num, St, dens, erad)
    LP.laden_particles_back_with_computing_particle(*drag, *u, V, vdiff, P, R, g.dx, num, lrad,
                                                    *[float(v) for v in L], *res)
    LP.update_particles_position(V, P, dt, num, *[float(v) for v in L])
    LP.calculate_viscous_force(*u, *vis, g.dx, Re)
    save("particles", res=np.array(res), meta_dx=g.dx, meta_num=num,
         meta_params=np.array([dt, St, grav, dens, erad, Re, lrad], np.float64),
         u_x=u[0], u_y=u[1], u_z=u[2], pos_in=pos.astype(F32), vel_in=vel.astype(F32),
         rad=rad.astype(F32), acc=acc0, vel1=vel1, vel_diff=vdiff,
         drag_x=drag[0], drag_y=drag[1], drag_z=drag[2], pos_out=P,
         vis_x=vis[0], vis_y=vis[1], vis_z=vis[2])


@fixture
def init_rings():
    """Vortex-ring initial velocity and dye add_vortex_ring_and_smoke
    (init_conditions.py:11-36) and the cell-to-face split
    split_central_vector (taichi_utils.py:104-116)."""
    res = (16, 8, 8)
    g = Grid(res, 1.0 / 8.0)
    u = vfield(res)
    smoke = ti.Vector.field(4, float, shape=res)
    IC.add_vortex_ring_and_smoke(w=0.1, rad=0.25, delta=0.06, c=ti.Vector([0.6, 0.5, 0.5]),
                                 unit_x=ti.Vector([0., 0., -1.]), unit_y=ti.Vector([0., 1., 0.]),
                                 pf=g.X, vf=u, smokef=smoke, color=ti.Vector([1., 0., 0.]), num_samples=64)
    faces = [sfield(s) for s in g.faces()]
    tu.split_central_vector(u, *faces)
    save("init_rings", res=np.array(res), meta_dx=g.dx, u_center=u, smoke=smoke,
         u_x=faces[0], u_y=faces[1], u_z=faces[2])


@fixture
def output_fields():
    """The output helpers get_central_vector (taichi_utils.py:95-100) and
    curl (taichi_utils.py:69-92) on a seeded velocity."""
    res = (12, 8, 10)
    g = Grid(res, 1.0 / 8.0)
    rng = np.random.default_rng(21)
    faces = [sfield(s) for s in g.faces()]
    for f, s in zip(faces, g.faces()):
        f.from_numpy(rng.standard_normal(s).astype(F32))
    vc = vfield(res)
    tu.get_central_vector(*faces, vc)
    w = vfield(res)
    tu.curl(vc, w, g.dx)
    save("output_fields", res=np.array(res), meta_dx=g.dx, u_x=faces[0], u_y=faces[1], u_z=faces[2],
         u_center=vc, curl=w)


@fixture
def edge_steps():
    """Two substeps of the EDGE driver loop (run_edge.py:588-712: reinit at
    j == 0, SL pre-advection, projection, EDGE and forward-map marches,
    BFECC pullback with clamps, projection) on a 8x8x8 grid, reinit_every=2,
    BFECC_clamp on.  The loop body is the reference's sequence of calls to its
    own kernels; dt follows run_edge.py:595-614 without frame output."""
    res = (8, 8, 8)
    nx, ny, nz = res
    dx = F32(1.0 / 8.0)
    g = Grid(res, dx)
    rng = np.random.default_rng(1111)
    u = velocity(rng, g, amp=0.8)
    smoke = smoke_field(rng, g)
    bt = ti.Matrix([[2, 2], [2, 2], [2, 2]], ti.i32)
    solver = MG.MGPCG_3(boundary_types=bt, N=list(res), base_level=1, real=ti.f32)
    _capture_solve(lambda: solver.Poisson(*u))
    u0 = [f.to_numpy() for f in u]
    smoke_in = smoke.to_numpy()
    faces = g.faces()
    fl = lambda: [sfield(s) for s in faces]  # noqa: E731
    init_u, err_u, tmp_u = fl(), fl(), fl()
    phi = [vfield(s) for s in faces]
    Fm = [vfield(s) for s in faces]
    init_smoke = ti.Vector.field(4, float, shape=res)
    err_smoke = ti.Vector.field(4, float, shape=res)
    tmp_smoke = ti.Vector.field(4, float, shape=res)
    psi = vfield(res)
    T = [vfield(res) for _ in range(3)]
    dT = [vfield(res) for _ in range(3)]
    tmpm = [vfield(res) for _ in range(7)]
    max_speed = ti.field(float, shape=())
    glb = dict(dx=dx, res_x=nx, res_y=ny, res_z=nz, X=g.X, X_x=g.X_x, X_y=g.X_y, X_z=g.X_z,
               psi_garm=psi, T_x_garm=T[0], T_y_garm=T[1], T_z_garm=T[2],
               dT_x_garm=dT[0], dT_y_garm=dT[1], dT_z_garm=dT[2], max_speed=max_speed)
    ns = load_driver_kernels("run_edge.py", ["calc_max_speed", "reset_to_identity", "advance_map", "map_u",
                                             "map_u_psi", "map_smoke", "split_to_mac", "map_smoke_psi",
                                             "clamp_smoke_psi", "clamp_u"], glb)
    CFL, reinit_every, ed_eps = 0.5, 2, 0.025 * float(dx)
    records = {}
    for i in range(2):
        j = i % reinit_every
        ns["calc_max_speed"](*u)
        curr_dt = CFL * float(dx) / float(max_speed[None])
        if j == 0:
            ns["reset_to_identity"](*phi, *Fm)
            H.reset_to_identity_2(psi, *T, *dT, g.X)
            for a, b in zip(init_u, u):
                a.copy_from(b)
            init_smoke.copy_from(smoke)
        H.advect_u_semi_lagrangian(*u, *tmp_u, dx, 0.5 * curr_dt, g.X_x, g.X_y, g.X_z)
        for a, b in zip(u, tmp_u):
            a.copy_from(b)
        it1, _ = _capture_solve(lambda: solver.Poisson(*u))
        H.advect_psi_garm_ed4_fusion_unroll(*tmpm, psi, *T, *dT, *u, g.X, dx, curr_dt, ed_eps)
        for p, f in zip(phi, Fm):
            ns["advance_map"](p, f, *u, curr_dt)
        ns["map_u_psi"](*init_u, *u, dx)
        ns["map_smoke_psi"](init_smoke, smoke, dx)
        ns["map_u"](*u, *err_u, *Fm, *phi, dx)
        ns["map_smoke"](smoke, err_smoke, *phi, dx)
        for e, a in zip(err_u, init_u):
            tu.add_fields(e, a, e, -1.)
        tu.add_fields(err_smoke, init_smoke, err_smoke, -1.)
        for e in err_u:
            tu.scale_field(e, 0.5, e)
        tu.scale_field(err_smoke, 0.5, err_smoke)
        ns["map_u_psi"](*err_u, *tmp_u, dx)
        ns["map_smoke_psi"](err_smoke, tmp_smoke, dx)
        for a, t, e in zip(u, tmp_u, err_u):
            tu.add_fields(a, t, e, -1.)
        tu.add_fields(smoke, tmp_smoke, smoke, -1.)
        ns["clamp_smoke_psi"](init_smoke, smoke, dx)
        for e, a, t in zip(err_u, u, tmp_u):
            ns["clamp_u"](e, a, t)
        for a, t in zip(u, tmp_u):
            a.copy_from(t)
        it2, _ = _capture_solve(lambda: solver.Poisson(*u))
        records[i] = dict(dt=curr_dt, it1=it1, it2=it2, u=[f.to_numpy() for f in u], smoke=smoke.to_numpy(),
                          psi=psi.to_numpy(), T=[t.to_numpy() for t in T], dT=[t.to_numpy() for t in dT],
                          phi=[p.to_numpy() for p in phi], F=[f.to_numpy() for f in Fm])
        print(f"    step {i}: dt={curr_dt:.5f} iters {it1} {it2}")
    out = dict(res=np.array(res), meta_dx=dx, meta_cfl=CFL, meta_reinit=reinit_every, meta_eps=F32(ed_eps),
               u_in_x=u0[0], u_in_y=u0[1], u_in_z=u0[2], smoke_in=smoke_in)
    for i, r in records.items():
        out[f"s{i}_meta_dt"] = r["dt"]
        out[f"s{i}_meta_iters"] = np.array([r["it1"], r["it2"]])
        for c, a in enumerate("xyz"):
            out[f"s{i}_u_{a}"] = r["u"][c]
            out[f"s{i}_T_{a}"] = r["T"][c]
            out[f"s{i}_dT_{a}"] = r["dT"][c]
            out[f"s{i}_phi_{a}"] = r["phi"][c]
            out[f"s{i}_F_{a}"] = r["F"][c]
        out[f"s{i}_smoke"] = r["smoke"]
        out[f"s{i}_psi"] = r["psi"]
    save("edge_steps", **out)


if __name__ == "__main__":
    for fn in FIXTURES:
        if args.only and fn.__name__ not in args.only.split(","):
            continue
        path = os.path.join(HERE, fn.__name__ + ".npz")
        if os.path.exists(path) and not args.force:
            print(f"skip {fn.__name__} (exists)")
            continue
        t0 = time.time()
        print(f"{fn.__name__} ...")
        fn()
        print(f"  {time.time() - t0:.1f}s")
