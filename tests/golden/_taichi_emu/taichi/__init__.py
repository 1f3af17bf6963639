"""A small numpy emulation of the Taichi 1.7 subset that the EDGE reference
sources use, so that those sources can be executed unchanged on tiny grids to
produce golden vectors.  Test infrastructure only: nothing in the product
imports it, and it is put on ``sys.path`` by ``tests/golden/make_golden.py``
alone.

Semantics emulated (Taichi with ``default_fp=ti.f32``):

* ``ti.field`` / ``ti.Vector.field`` hold float32 (or int32) numpy arrays; a
  vector field element is returned as a writable view, so ``f[I][c] = v``
  writes through as in Taichi.
* Every float produced by vector arithmetic, by ``ti.*`` math functions and
  every ``float``-annotated kernel argument is float32; Python float constants
  meet float32 values as "weak" scalars (numpy NEP 50), which matches Taichi's
  conversion of Python constants to ``default_fp``.
* ``@ti.func`` parameters annotated ``ti.template()`` are pass-by-reference:
  the function source is rewritten so that it hands back the final values of
  those parameters, and every statement-level call site writes them back into
  the argument expressions (local names or field elements).
* ``ti.atomic_max(x, v)`` / ``ti.atomic_add(x, v)`` statements are rewritten to
  ``x = max(x, v)`` / ``x = x + v``; parallel-for loops run serially in index
  order (so atomic float sums are deterministic here, unlike on a GPU).
"""
import ast
import inspect
import itertools
import math as _pymath
import textwrap

import numpy as np

f32 = np.float32
f64 = np.float64
i32 = np.int32
i64 = np.int64
u8 = np.uint8
cpu = "cpu"
cuda = "cuda"
gpu = "gpu"

_default_fp = np.float32


def init(arch=None, debug=False, default_fp=None, **kwargs):
    global _default_fp
    if default_fp is not None:
        _default_fp = default_fp


def sync():
    pass


def _np_dtype(dtype):
    if dtype is float or dtype is None:
        return _default_fp
    if dtype is int:
        return np.int32
    return dtype


class _TemplateAnn:
    pass


def template():
    return _TemplateAnn()


class _types:
    @staticmethod
    def vector(n, dtype):
        return ("vector", n, dtype)

    @staticmethod
    def matrix(n, m, dtype):
        return ("matrix", n, m, dtype)


types = _types


# --------------------------------------------------------------------------
# vectors / matrices
# --------------------------------------------------------------------------
class Vec(np.ndarray):
    """ndarray subclass with the Taichi Vector/Matrix methods used by the
    reference; float64 results of arithmetic are narrowed to float32."""

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        args = [np.asarray(x) if isinstance(x, Vec) else x for x in inputs]
        out = kwargs.get("out")
        if out is not None:
            kwargs["out"] = tuple(np.asarray(o) if isinstance(o, Vec) else o for o in out)
        res = getattr(ufunc, method)(*args, **kwargs)
        if out is not None:
            return out[0] if len(out) == 1 else out
        if isinstance(res, np.ndarray):
            if res.dtype == np.float64:
                res = res.astype(np.float32)
            if res.ndim == 0:
                return res[()]
            return res.view(Vec)
        if isinstance(res, np.float64):
            return np.float32(res)
        return res

    def __matmul__(self, other):
        r = np.matmul(np.asarray(self), np.asarray(other))
        if r.dtype == np.float64:
            r = r.astype(np.float32)
        return r.view(Vec) if r.ndim else r[()]

    def norm(self):
        a = np.asarray(self, dtype=np.float32)
        return np.float32(np.sqrt(np.float32((a * a).sum(dtype=np.float32))))

    def normalized(self):
        return (self / self.norm()).view(Vec)

    def cross(self, other):
        a = np.asarray(self, dtype=np.float32)
        b = np.asarray(other, dtype=np.float32)
        return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                         a[0] * b[1] - a[1] * b[0]], dtype=np.float32).view(Vec)

    def dot(self, other):
        a = np.asarray(self)
        b = np.asarray(other)
        acc = (a[0] * b[0]).astype(np.result_type(a, b))
        for c in range(1, a.shape[0]):
            acc = acc + a[c] * b[c]
        if isinstance(acc, np.float64) or getattr(acc, "dtype", None) == np.float64:
            acc = np.float32(acc)
        return acc[()] if isinstance(acc, np.ndarray) else acc

    def _get(self, c):
        return np.asarray(self)[c]

    def _set(self, c, v):
        np.asarray(self)[c] = v

    x = property(lambda s: s._get(0), lambda s, v: s._set(0, v))
    y = property(lambda s: s._get(1), lambda s, v: s._set(1, v))
    z = property(lambda s: s._get(2), lambda s, v: s._set(2, v))
    w = property(lambda s: s._get(3), lambda s, v: s._set(3, v))

    @property
    def xyz(self):
        return np.asarray(self)[:3].copy().view(Vec)

    @xyz.setter
    def xyz(self, v):
        np.asarray(self)[:3] = np.asarray(v)


def _as_vec(data, dt=None):
    a = np.asarray(data)
    if dt is not None:
        a = a.astype(_np_dtype(dt))
    elif a.dtype == np.float64:
        a = a.astype(np.float32)
    elif a.dtype.kind in "iub" and a.dtype != np.int32:
        a = a.astype(np.int32)
    return np.array(a).view(Vec)


class _VectorMeta(type):
    def __call__(cls, data, dt=None):
        vals = [np.asarray(v)[()] if isinstance(v, np.ndarray) else v for v in data]
        return _as_vec(vals, dt)


class Vector(metaclass=_VectorMeta):
    @staticmethod
    def field(n, dtype=float, shape=(), **kw):
        return Field(dtype, shape, (n,))

    @staticmethod
    def unit(n, i, dt=None):
        a = np.zeros(n, dtype=_np_dtype(dt) if dt is not None else np.int32)
        a[i] = 1
        return a.view(Vec)

    @staticmethod
    def one(dt, n):
        return np.ones(n, dtype=_np_dtype(dt)).view(Vec)

    @staticmethod
    def zero(dt, n):
        return np.zeros(n, dtype=_np_dtype(dt)).view(Vec)


class _MatrixMeta(type):
    def __call__(cls, data, dt=None):
        return _as_vec(data, dt)


class Matrix(metaclass=_MatrixMeta):
    @staticmethod
    def rows(rows):
        return _as_vec([np.asarray(r) for r in rows])

    @staticmethod
    def cols(cols):
        return _as_vec([np.asarray(c) for c in cols]).T.copy().view(Vec)

    @staticmethod
    def field(n, m, dtype=float, shape=(), **kw):
        return Field(dtype, shape, (n, m))


# --------------------------------------------------------------------------
# fields
# --------------------------------------------------------------------------
def _index(I):
    if I is None:
        return ()
    if isinstance(I, tuple):
        return tuple(int(v) for v in I)
    if isinstance(I, np.ndarray):
        return tuple(int(v) for v in np.asarray(I).ravel())
    return (int(I),)


class Field:
    def __init__(self, dtype, shape, elem=()):
        if isinstance(shape, int):
            shape = (shape,)
        self.shape = tuple(int(s) for s in shape)
        self.elem = tuple(elem)
        self.dtype = _np_dtype(dtype)
        self.arr = np.zeros(self.shape + self.elem, dtype=self.dtype)

    def __getitem__(self, I):
        v = self.arr[_index(I)]
        if self.elem:
            return v.view(Vec)
        return v[()] if isinstance(v, np.ndarray) else v

    def __setitem__(self, I, val):
        self.arr[_index(I)] = np.asarray(val)

    def __iter__(self):
        return iter(itertools.product(*[range(s) for s in self.shape]))

    def fill(self, v):
        self.arr[...] = v

    def copy_from(self, other):
        self.arr[...] = other.arr

    def to_numpy(self):
        return self.arr.copy()

    def from_numpy(self, a):
        self.arr[...] = np.asarray(a).reshape(self.arr.shape)


def field(dtype=float, shape=(), **kw):
    return Field(dtype, shape)


# --------------------------------------------------------------------------
# loops
# --------------------------------------------------------------------------
class ndrange:
    def __init__(self, *dims):
        self.ranges = []
        for d in dims:
            if isinstance(d, (tuple, list)):
                self.ranges.append(range(int(d[0]), int(d[1])))
            else:
                self.ranges.append(range(int(d)))

    def __iter__(self):
        return iter(itertools.product(*self.ranges))


def grouped(x):
    if isinstance(x, Field):
        it = itertools.product(*[range(s) for s in x.shape])
    elif isinstance(x, ndrange):
        it = iter(x)
    else:
        it = iter(x)
    for idx in it:
        yield np.array(idx, dtype=np.int32).view(Vec)


def static(x):
    return x


def cast(x, dtype):
    return _np_dtype(dtype)(x)


# --------------------------------------------------------------------------
# math
# --------------------------------------------------------------------------
def _narrow(r):
    if isinstance(r, np.ndarray):
        if r.dtype == np.float64:
            r = r.astype(np.float32)
        return r.view(Vec) if r.ndim else r[()]
    if isinstance(r, (float, np.float64)):
        return np.float32(r)
    return r


def _align(a, b):
    """Python floats meeting float32 values become float32 (Taichi turns
    Python constants into default_fp)."""
    fa = isinstance(a, (np.floating, np.ndarray)) and np.asarray(a).dtype == np.float32
    fb = isinstance(b, (np.floating, np.ndarray)) and np.asarray(b).dtype == np.float32
    if fa and isinstance(b, float):
        b = np.float32(b)
    if fb and isinstance(a, float):
        a = np.float32(a)
    return a, b


def max(a, b):  # noqa: A001 - Taichi name
    a, b = _align(a, b)
    return _narrow(np.maximum(np.asarray(a), np.asarray(b)))


def min(a, b):  # noqa: A001 - Taichi name
    a, b = _align(a, b)
    return _narrow(np.minimum(np.asarray(a), np.asarray(b)))


def abs(x):  # noqa: A001
    return _narrow(np.abs(np.asarray(x)))


def floor(x):
    return _narrow(np.floor(np.asarray(x, dtype=np.float32)))


def sqrt(x):
    return _narrow(np.sqrt(np.asarray(x, dtype=np.float32)))


def exp(x):
    return _narrow(np.exp(np.asarray(x, dtype=np.float32)))


def cos(x):
    return _narrow(np.cos(np.asarray(x, dtype=np.float32)))


def sin(x):
    return _narrow(np.sin(np.asarray(x, dtype=np.float32)))


class _math:
    pi = _pymath.pi

    @staticmethod
    def clamp(x, lo, hi):
        x, lo = _align(x, lo)
        x, hi = _align(x, hi)
        return _narrow(np.minimum(np.maximum(np.asarray(x), np.asarray(lo)), np.asarray(hi)))

    @staticmethod
    def max(*args):
        r = np.asarray(args[0])
        for a in args[1:]:
            r = np.maximum(r, np.asarray(a))
        return _narrow(r)

    @staticmethod
    def min(*args):
        r = np.asarray(args[0])
        for a in args[1:]:
            r = np.minimum(r, np.asarray(a))
        return _narrow(r)

    @staticmethod
    def radians(d):
        return np.float32(d * _pymath.pi / 180.0)

    cos = staticmethod(cos)
    sin = staticmethod(sin)
    exp = staticmethod(exp)
    sqrt = staticmethod(sqrt)

    @staticmethod
    def inverse(m):
        return _narrow(np.linalg.inv(np.asarray(m, dtype=np.float64)))


math = _math


def _ti_int(x):
    """Taichi's int() cast: elementwise truncation for vectors."""
    a = np.asarray(x)
    if a.ndim and a.size > 1:
        return np.trunc(a).astype(np.int32).view(Vec)
    return int(a.reshape(()) if a.ndim else a)


def _atomic_max(x, v):
    return _math.max(x, v)


# --------------------------------------------------------------------------
# kernels / funcs (source rewriting for pass-by-reference template params)
# --------------------------------------------------------------------------
class _TR:
    """Return value of a ti.func that has ti.template() parameters: the
    original return value plus the final values of those parameters."""
    __slots__ = ("ret", "vals")

    def __init__(self, ret, vals):
        self.ret = ret
        self.vals = vals


def _is_template_ann(ann):
    return (isinstance(ann, ast.Call) and isinstance(ann.func, ast.Attribute)
            and ann.func.attr == "template")


def _assignable(expr):
    return isinstance(expr, (ast.Name, ast.Subscript, ast.Attribute))


class _Rewriter(ast.NodeTransformer):
    def __init__(self, tmpl_params):
        self.tmpl = tmpl_params  # list of (key_pos, name)
        self.counter = 0

    def _tr_tuple(self):
        keys = [ast.Constant(p) for p, _ in self.tmpl] + [ast.Constant(n) for _, n in self.tmpl]
        vals = [ast.Name(n, ast.Load()) for _, n in self.tmpl] * 2
        return ast.Dict(keys=keys, values=vals)

    def visit_FunctionDef(self, node):
        self.generic_visit(node)
        if self.tmpl:
            node.body.append(self.visit_Return(ast.Return(value=None)))
        return node

    def visit_Return(self, node):
        if not self.tmpl:
            return node
        val = node.value if node.value is not None else ast.Constant(None)
        return ast.Return(value=ast.Call(func=ast.Name("_ti_TR", ast.Load()),
                                         args=[val, self._tr_tuple()], keywords=[]))

    def visit_Call(self, node):
        self.generic_visit(node)
        if isinstance(node.func, ast.Name) and node.func.id == "int":
            node.func = ast.Name("_ti_int", ast.Load())
        return node

    def visit_Expr(self, node):
        call = node.value
        if not isinstance(call, ast.Call):
            return node
        f = call.func
        if isinstance(f, ast.Attribute) and f.attr in ("atomic_max", "atomic_add") and \
                isinstance(f.value, ast.Name) and f.value.id == "ti":
            target, value = call.args
            tgt_store = _to_store(target)
            if f.attr == "atomic_max":
                rhs = ast.Call(func=ast.Name("_ti_atomic_max", ast.Load()), args=[target, value], keywords=[])
            else:
                rhs = ast.BinOp(left=target, op=ast.Add(), right=value)
            return ast.Assign(targets=[tgt_store], value=rhs)
        self.counter += 1
        tmp = f"_ti_ret{self.counter}"
        out = [ast.Assign(targets=[ast.Name(tmp, ast.Store())], value=call)]
        body = []
        for i, a in enumerate(call.args):
            if _assignable(a):
                cond = ast.Compare(left=ast.Constant(i), ops=[ast.In()],
                                   comparators=[ast.Attribute(ast.Name(tmp, ast.Load()), "vals", ast.Load())])
                val = ast.Subscript(value=ast.Attribute(ast.Name(tmp, ast.Load()), "vals", ast.Load()),
                                    slice=ast.Constant(i), ctx=ast.Load())
                body.append(ast.If(test=cond, body=[ast.Assign(targets=[_to_store(a)], value=val)], orelse=[]))
        for kw in call.keywords:
            if kw.arg and _assignable(kw.value):
                cond = ast.Compare(left=ast.Constant(kw.arg), ops=[ast.In()],
                                   comparators=[ast.Attribute(ast.Name(tmp, ast.Load()), "vals", ast.Load())])
                val = ast.Subscript(value=ast.Attribute(ast.Name(tmp, ast.Load()), "vals", ast.Load()),
                                    slice=ast.Constant(kw.arg), ctx=ast.Load())
                body.append(ast.If(test=cond, body=[ast.Assign(targets=[_to_store(kw.value)], value=val)], orelse=[]))
        if body:
            test = ast.Call(func=ast.Name("isinstance", ast.Load()),
                            args=[ast.Name(tmp, ast.Load()), ast.Name("_ti_TR", ast.Load())], keywords=[])
            out.append(ast.If(test=test, body=body, orelse=[]))
        return out


def _to_store(expr):
    import copy
    e = copy.deepcopy(expr)
    e.ctx = ast.Store()
    return e


def _root_name(t):
    while isinstance(t, (ast.Subscript, ast.Attribute)):
        t = t.value
    return t.id if isinstance(t, ast.Name) else None


def _written_names(fdef):
    """Names that the function body rebinds or writes into."""
    out = set()

    def add(t):
        if isinstance(t, (ast.Tuple, ast.List)):
            for e in t.elts:
                add(e)
        else:
            n = _root_name(t)
            if n:
                out.add(n)

    for node in ast.walk(fdef):
        if isinstance(node, ast.Assign):
            for t in node.targets:
                add(t)
        elif isinstance(node, (ast.AugAssign, ast.AnnAssign)):
            add(node.target)
    return out


def _rewrite(fn, is_func):
    lines, first = inspect.getsourcelines(fn)
    src = textwrap.dedent("".join(lines))
    tree = ast.parse(src)
    ast.increment_lineno(tree, first - 1)
    fdef = tree.body[0]
    fdef.decorator_list = []
    params = [a for a in fdef.args.args]
    offset = 1 if params and params[0].arg == "self" else 0
    tmpl = []
    if is_func:
        written = _written_names(fdef)
        for pos, a in enumerate(params):
            if a.annotation is not None and _is_template_ann(a.annotation) and a.arg in written:
                tmpl.append((pos - offset, a.arg))
    for a in params:
        a.annotation = None
    _Rewriter(tmpl).visit(tree)
    ast.fix_missing_locations(tree)
    g = fn.__globals__
    g.setdefault("_ti_TR", _TR)
    g.setdefault("_ti_atomic_max", _atomic_max)
    g.setdefault("_ti_int", _ti_int)
    if fn.__closure__:
        # kernels defined inside a function: freeze the enclosing variables
        g = dict(g)
        for name, cell in zip(fn.__code__.co_freevars, fn.__closure__):
            g[name] = cell.cell_contents
    ns = {}
    code = compile(tree, inspect.getsourcefile(fn) or "<ti>", "exec")
    exec(code, g, ns)
    return ns[fdef.name]


def func(fn):
    return _rewrite(fn, True)


def kernel(fn):
    sig = inspect.signature(fn)
    anns = [p.annotation for p in sig.parameters.values()]
    names = list(sig.parameters)
    body = _rewrite(fn, False)

    def wrapper(*args, **kwargs):
        conv = []
        for i, a in enumerate(args):
            ann = anns[i] if i < len(anns) else None
            if ann is float:
                a = _default_fp(a)
            elif ann is int:
                a = int(a)
            conv.append(a)
        for k, v in list(kwargs.items()):
            ann = anns[names.index(k)] if k in names else None
            if ann is float:
                kwargs[k] = _default_fp(v)
            elif ann is int:
                kwargs[k] = int(v)
        return body(*conv, **kwargs)

    wrapper.__wrapped_kernel__ = body
    return wrapper


def data_oriented(cls):
    return cls
