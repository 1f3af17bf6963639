"""Drop-in for the reference's util/io_utils.py output writers
(io_utils.py:15-139).  The reference writes VTK XML files through the vtk and
pyevtk packages, which are not installed here; these functions write the same
files (ImageData .vti for the grid fields, UnstructuredGrid .vtu of vertex
cells for the particles: same array names, point layout and file names) with
a small XML writer of their own, raw little-endian appended data with UInt64
block headers.  read_vtk() reads such a file back (for tests and
post-processing without vtk).
"""
import os
import shutil
import struct
import xml.etree.ElementTree as ET

import numpy as np

_VTK_TYPES = {np.dtype(np.float32): "Float32", np.dtype(np.float64): "Float64", np.dtype(np.int32): "Int32",
              np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}
_NP_TYPES = {v: k for k, v in _VTK_TYPES.items()}
VTK_VERTEX = 1  # VTK cell type of a single point


def remove_everything_in(folder):
    """io_utils.py:15-26."""
    for name in os.listdir(folder):
        path = os.path.join(folder, name)
        try:
            if os.path.isfile(path) or os.path.islink(path):
                os.unlink(path)
            elif os.path.isdir(path):
                shutil.rmtree(path)
        except OSError as e:
            print(f"Failed to delete {path}. Reason: {e}")


class _Appended:
    """Collects arrays for the <AppendedData> block; each gets an offset."""

    def __init__(self):
        self.blocks, self.offset = [], 0

    def add(self, arr):
        raw = np.ascontiguousarray(arr).astype(np.asarray(arr).dtype.newbyteorder("<"), copy=False).tobytes()
        off = self.offset
        self.blocks.append(struct.pack("<Q", len(raw)) + raw)
        self.offset += 8 + len(raw)
        return off


def _data_array(parent, app, name, arr, ncomp):
    arr = np.asarray(arr)
    if arr.dtype not in _VTK_TYPES:
        arr = arr.astype(np.float32)
    ET.SubElement(parent, "DataArray", type=_VTK_TYPES[arr.dtype], Name=name, NumberOfComponents=str(ncomp),
                  format="appended", offset=str(app.add(arr)))


def _write(path, root, app):
    ET.SubElement(root, "AppendedData", encoding="raw").text = "_"
    head = ET.tostring(root, encoding="unicode")
    # the raw block follows the "_" marker directly
    pre, post = head.rsplit("_</AppendedData>", 1)
    with open(path, "wb") as f:
        f.write(b'<?xml version="1.0"?>\n')
        f.write(pre.encode() + b"_")
        for b in app.blocks:
            f.write(b)
        f.write(b"\n</AppendedData>" + post.encode() + b"\n")


def _vtkfile(kind):
    return ET.Element("VTKFile", type=kind, version="1.0", byte_order="LittleEndian", header_type="UInt64")


def _image(path, point_arrays, shape):
    """point_arrays: [(name, array in x-fastest order, ncomp)], the first is
    the active scalar."""
    root = _vtkfile("ImageData")
    ext = " ".join(f"0 {n - 1}" for n in shape)
    img = ET.SubElement(root, "ImageData", WholeExtent=ext, Origin="0 0 0", Spacing="1 1 1")
    piece = ET.SubElement(img, "Piece", Extent=ext)
    pd = ET.SubElement(piece, "PointData", Scalars=point_arrays[0][0])
    app = _Appended()
    for name, arr, nc in point_arrays:
        _data_array(pd, app, name, arr, nc)
    ET.SubElement(piece, "CellData")
    _write(path, root, app)


def _fortran_points(a, ncomp):
    """(nx, ny, nz[, c]) -> rows in x-fastest point order (numpy ravel(order="F")
    of the spatial axes), components kept together."""
    a = np.asarray(a)
    if ncomp == 1:
        return a.ravel(order="F")
    return a.reshape(-1, ncomp, order="F") if a.ndim == 2 else \
        np.stack([a[..., c].ravel(order="F") for c in range(ncomp)], 1)


def write_vtks(w_numpy, smoke_numpy, outdir, i):
    """io_utils.py:29-50: vorticity and smoke as point scalars of an image
    (one point per cell, unit spacing), field_{i:04d}.vti."""
    w = np.squeeze(w_numpy)
    s = np.squeeze(smoke_numpy)
    _image(os.path.join(outdir, "field_{:04d}.vti".format(i)),
           [("vorticity", _fortran_points(w, 1), 1), ("smoke", s.ravel(order="F"), 1)], w.shape)


def write_vtks_4channel_smoke(w_numpy, smoke_numpy, outdir, i):
    """io_utils.py:53-76: vorticity scalars and the 4-channel smoke as a
    4-component point array, field_{i:04d}.vti."""
    w = np.squeeze(w_numpy)
    # the reference reshapes the (nx, ny, nz, 4) array with order="F" into
    # (N, 4) rows, i.e. x-fastest points with their four channels
    s = np.asarray(smoke_numpy).reshape(-1, 4, order="F")
    _image(os.path.join(outdir, "field_{:04d}.vti".format(i)), [("vorticity", _fortran_points(w, 1), 1),
                                                                 ("smoke", s, 4)], w.shape)


def write_to_vtks_lp(pos, scalar_data, vector_data, file_path):
    """io_utils.py:83-139: particles as vertex cells of an unstructured grid
    with optional per-particle scalars and 3-vectors; writes file_path.vtu
    (the extension pyevtk appends)."""
    pos = np.asarray(pos)
    n = pos.shape[0]
    root = _vtkfile("UnstructuredGrid")
    grid = ET.SubElement(root, "UnstructuredGrid")
    piece = ET.SubElement(grid, "Piece", NumberOfPoints=str(n), NumberOfCells=str(n))
    app = _Appended()
    pts = ET.SubElement(piece, "Points")
    _data_array(pts, app, "points", pos.reshape(n, 3), 3)
    cells = ET.SubElement(piece, "Cells")
    _data_array(cells, app, "connectivity", np.arange(n, dtype=np.int32), 1)
    _data_array(cells, app, "offsets", np.arange(1, n + 1, dtype=np.int32), 1)
    _data_array(cells, app, "types", np.full(n, VTK_VERTEX, np.uint8), 1)
    sk, vk = sorted(scalar_data), sorted(vector_data)
    attrs = {}
    if sk:
        attrs["Scalars"] = sk[0]
    if vk:
        attrs["Vectors"] = vk[0]
    if not sk and not vk:
        attrs["Scalars"] = "scalar"
    pd = ET.SubElement(piece, "PointData", **attrs)
    for k in sk:
        _data_array(pd, app, k, np.asarray(scalar_data[k]).reshape(n), 1)
    for k in vk:
        _data_array(pd, app, k, np.asarray(vector_data[k]).reshape(n, 3), 3)
    _write(file_path + ".vtu", root, app)


def read_vtk(path):
    """Arrays of a file written above: {name: array} (points x-fastest, (N, C)
    for multi-component arrays) plus "_extent" / "_npoints"."""
    raw = open(path, "rb").read()
    start = raw.index(b'<AppendedData encoding="raw">') + len(b'<AppendedData encoding="raw">')
    mark = raw.index(b"_", start) + 1
    head = raw[:start].decode() + "</AppendedData></VTKFile>"
    root = ET.fromstring(head.split("?>", 1)[1])
    out = {}
    for da in root.iter("DataArray"):
        off = mark + int(da.get("offset"))
        nbytes = struct.unpack("<Q", raw[off:off + 8])[0]
        a = np.frombuffer(raw[off + 8:off + 8 + nbytes], dtype=_NP_TYPES[da.get("type")].newbyteorder("<"))
        nc = int(da.get("NumberOfComponents", "1"))
        out[da.get("Name")] = a.reshape(-1, nc) if nc > 1 else a
    img = root.find("ImageData")
    if img is not None:
        out["_extent"] = [int(v) for v in img.get("WholeExtent").split()]
    piece = root.find(".//Piece")
    if piece is not None and piece.get("NumberOfPoints"):
        out["_npoints"] = int(piece.get("NumberOfPoints"))
    return out
