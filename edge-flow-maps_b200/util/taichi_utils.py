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
    ops.get_central_vector((vx, vy, vz), vc)


def curl(vf, cf, dx):
    """taichi_utils.py:69-92 (output helper; clamped central differences)."""
    ops.curl(vf, cf, dx)
