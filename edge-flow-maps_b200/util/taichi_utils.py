"""Drop-in for the host-callable kernels of the reference's
util/taichi_utils.py.  The ti.func samplers (sample, interp_2, interp_1, ...)
are device functions of libedgeb200.so (csrc/edge_common.cuh); point-wise
evaluation for testing is in edgeb200.ops (points_mac, points_dye)."""
import torch

from edgeb200 import ops

eps = 1.e-6  # taichi_utils.py:3


def scale_field(a, alpha, result):
    """taichi_utils.py:6-9."""
    ops.axpy(a, None, alpha, result)


def add_fields(f1, f2, dest, multiplier):
    """taichi_utils.py:12-15."""
    ops.axpy(f1, f2, multiplier, dest)


def _coords(pf, dx, off):
    idx = [torch.arange(n, device=pf.device, dtype=torch.float32) for n in pf.shape[:3]]
    g = torch.meshgrid(*idx, indexing="ij")
    pf.copy_(torch.stack([(g[c] + off[c]) * float(dx) for c in range(3)], -1))


def center_coords_func(pf, dx):
    """taichi_utils.py:22-26."""
    _coords(pf, dx, (0.5, 0.5, 0.5))


def x_coords_func(pf, dx):
    """taichi_utils.py:29-32."""
    _coords(pf, dx, (0.0, 0.5, 0.5))


def y_coords_func(pf, dx):
    """taichi_utils.py:35-38."""
    _coords(pf, dx, (0.5, 0.0, 0.5))


def z_coords_func(pf, dx):
    """taichi_utils.py:41-44."""
    _coords(pf, dx, (0.5, 0.5, 0.0))


def split_central_vector(vc, vx, vy, vz):
    """taichi_utils.py:103-116."""
    ops.split_central_vector(vc, (vx, vy, vz))


def get_central_vector(vx, vy, vz, vc):
    """taichi_utils.py:95-100 (output helper)."""
    vc[..., 0] = 0.5 * (vx[1:] + vx[:-1])
    vc[..., 1] = 0.5 * (vy[:, 1:] + vy[:, :-1])
    vc[..., 2] = 0.5 * (vz[:, :, 1:] + vz[:, :, :-1])


def curl(vf, cf, dx):
    """taichi_utils.py:70-92 (output helper; clamped central differences)."""
    p = torch.nn.functional.pad(vf.permute(3, 0, 1, 2)[None], (1, 1, 1, 1, 1, 1), mode="replicate")[0]
    inv = 1.0 / (2 * dx)
    d = lambda c, a: (p[c].narrow(a, 2, vf.shape[a]) - p[c].narrow(a, 0, vf.shape[a])).narrow(  # noqa: E731
        (a + 1) % 3, 1, vf.shape[(a + 1) % 3]).narrow((a + 2) % 3, 1, vf.shape[(a + 2) % 3]) * inv
    cf[..., 0] = d(2, 1) - d(1, 2)
    cf[..., 1] = d(0, 2) - d(2, 0)
    cf[..., 2] = d(1, 0) - d(0, 1)
