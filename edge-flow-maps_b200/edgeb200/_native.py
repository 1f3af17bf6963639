"""ctypes binding of libedgeb200.so.

The argument types of every entry point are derived from the C header
(include/edge_b200.h), so the Python side cannot drift from the ABI.  The
library is required: there is no fallback implementation, and calls raise
``EdgeError`` on any non-zero status.
"""
import ctypes
import os
import re

_PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(_PKG))
HEADER = os.path.join(ROOT, "include", "edge_b200.h")
LIBPATH = os.path.join(_PKG, "libedgeb200.so")

EDGE_OK = 0
EDGE_EINVAL = -1
EDGE_EALIGN = -2
EDGE_ENOCONV = -3
EDGE_ENAN = -4
EDGE_ESTALL = -5
EDGE_ESTATE = -6

HERMITE_FD = 0
HERMITE_GARM = 1
HERMITE_FULL = 2


class EdgeError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed: {msg} (code {code})")
        self.code = code


_CTYPE = {
    "int": ctypes.c_int,
    "float": ctypes.c_float,
    "double": ctypes.c_double,
    "long long": ctypes.c_longlong,
}


def _param_type(decl):
    decl = decl.strip()
    if "*" in decl:
        return ctypes.c_void_p
    decl = re.sub(r"\bconst\b", "", decl).strip()
    base = " ".join(decl.split()[:-1])
    if base not in _CTYPE:
        raise ValueError(f"unsupported C parameter type in {decl!r}")
    return _CTYPE[base]


def parse_header(path=HEADER):
    """Return {name: (restype, [argtypes])} for every function the header
    declares."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"(const\s+char\s*\*|int)\s*(edge_\w+)\s*\(([^)]*)\)\s*;", text, flags=re.S):
        rtype, name, params = m.group(1), m.group(2), m.group(3)
        params = params.strip()
        args = [] if params in ("", "void") else [_param_type(p) for p in params.split(",")]
        res = ctypes.c_char_p if "char" in rtype else ctypes.c_int
        out[name] = (res, args)
    return out


_lib = None
SIGNATURES = None


def load():
    """Load the library (raises if it is missing: the CUDA path is the only
    path)."""
    global _lib, SIGNATURES
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(f"{LIBPATH} is missing; build it with "
                           f"'python edge-flow-maps_b200/csrc/build.py'")
    lib = ctypes.CDLL(LIBPATH)
    SIGNATURES = parse_header()
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def call(name, *args):
    """Call an entry point and raise EdgeError on a non-zero status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != EDGE_OK:
        msg = lib.edge_error_string(rc).decode()
        raise EdgeError(name, rc, msg)
    return rc


def raw(name, *args):
    """Call an entry point and return its status without raising."""
    return getattr(load(), name)(*args)
