"""Tensor plumbing between torch and the C ABI.

Fields are torch float32 CUDA tensors with the reference's shapes (what
``ti.field(...).to_numpy()`` returns): scalar (nx, ny, nz), vec3
(nx, ny, nz, 3), vec4 (nx, ny, nz, 4); face grids (nx+1, ny, nz),
(nx, ny+1, nz), (nx, ny, nz+1).
"""
import ctypes

import torch

NULL = ctypes.c_void_p(0)


def require(t, name="field"):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor (got {type(t).__name__})")
    if not t.is_cuda:
        raise ValueError(f"{name} must live on a CUDA device")
    if t.dtype != torch.float32 and t.dtype != torch.int32:
        raise ValueError(f"{name} must be float32 (or int32 for masks), got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


def ptr(t, name="field"):
    if t is None:
        return NULL
    require(t, name)
    return ctypes.c_void_p(t.data_ptr())


def ptr_any(t, dtypes, name="tensor"):
    """Device pointer of a contiguous CUDA tensor of one of `dtypes` (the
    network's bf16 / int32 / float32 / float64 buffers)."""
    if t is None:
        return NULL
    if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous() or t.dtype not in dtypes:
        raise ValueError(f"{name} must be a contiguous CUDA tensor of {dtypes}")
    return ctypes.c_void_p(t.data_ptr())


def stream(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def cell_dims(t):
    return int(t.shape[0]), int(t.shape[1]), int(t.shape[2])


def dims_from_faces(u_x, u_y, u_z):
    nx, ny, nz = int(u_y.shape[0]), int(u_x.shape[1]), int(u_x.shape[2])
    if tuple(u_x.shape[:3]) != (nx + 1, ny, nz) or tuple(u_y.shape[:3]) != (nx, ny + 1, nz) or \
            tuple(u_z.shape[:3]) != (nx, ny, nz + 1):
        raise ValueError(f"inconsistent face grids {tuple(u_x.shape)}, {tuple(u_y.shape)}, {tuple(u_z.shape)}")
    return nx, ny, nz


def face_shapes(res):
    nx, ny, nz = res
    return [(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)]


def zeros_faces(res, comps=None, device="cuda"):
    extra = () if comps is None else (comps,)
    return [torch.zeros(s + extra, dtype=torch.float32, device=device) for s in face_shapes(res)]


def zeros_cells(res, comps=None, device="cuda"):
    extra = () if comps is None else (comps,)
    return torch.zeros(tuple(res) + extra, dtype=torch.float32, device=device)


def dx_of(dx):
    return ctypes.c_float(float(dx))
