"""A numpy stand-in for the small Taichi subset the reference solver uses.

Used ONLY by gen_golden.py, in the development container, to execute the
reference's own kernel source (LBM_3D_LES_air_over_waves_CODEX.py) on tiny
grids and record golden vectors for the CPU oracle.  Taichi itself is not
installable here.

How kernels run: a @ti.kernel / @ti.func body is re-compiled from its
source with three rewrites and then executed as plain Python, serially, in
row-major order of each struct-for:
  * `ti.atomic_add(F[idx], v)` -> `_atomic_add(F, idx, v)`;
  * builtin max/min/float inside kernels -> f32-typed versions (Taichi maps
    them to ti.max/ti.min/ti.cast);
  * the first assignment of a local name gives it Taichi's type (a Python
    float becomes f32, an int i32) and later assignments cast to that type.
With NumPy >= 2 (NEP 50), Python scalars combine with np.float32 as f32,
which matches Taichi's treatment of captured Python constants.

Transcendentals are evaluated in double and rounded to f32 once, the same
definition the oracle and the CUDA library use.  ti.random() is fed from
hooks so that the initial kick and the backscatter draws are the ones the
oracle uses.

For the kernels that race in parallel Taichi (redistribute_vof_mass_excess,
remove_orphan_vof_interface_cells) the stand-in gives the oracle's
semantics: reads of the mass/fill/type fields see the state at kernel entry
and atomic adds are applied at kernel exit, grouped by receiver in the
order the oracle uses.
"""
from __future__ import annotations

import ast
import inspect
import itertools
import textwrap

import numpy as np

f32 = "f32"
i32 = "i32"
cpu = "cpu"
gpu = "gpu"

_state = {
    "cell": None,          # linear index of the current struct-for cell
    "shape": None,
    "kernel": None,
    "random_hook": None,   # callable(kernel_name, cell) -> float in [0,1)
    "deferred": None,      # list of (field, idx, value, donor) when deferring
    "snapshot_fields": (),
    "calls": {},
}


def init(*args, **kwargs):
    return None


def _to_f32(x):
    return np.float32(x)


class Vec:
    """Local vector / view of one vector-field element."""

    def __init__(self, arr, is_int):
        self.arr = arr
        self.is_int = is_int

    def __getitem__(self, q):
        v = self.arr[q]
        return int(v) if self.is_int else np.float32(v)

    def __setitem__(self, q, v):
        self.arr[q] = v


class Field:
    def __init__(self, dtype, shape, n=None):
        if shape == ():
            shape = ()
        elif not isinstance(shape, tuple):
            shape = (shape,)
        self.shape = shape
        self.n = n
        self.is_int = dtype == i32
        npdt = np.int32 if self.is_int else np.float32
        self.arr = np.zeros(shape + ((n,) if n else ()), dtype=npdt)
        self.read_arr = None
        self.name = None

    def _idx(self, idx):
        if idx is None:
            return ()
        if not isinstance(idx, tuple):
            return (idx,)
        return idx

    def __iter__(self):
        ranges = [range(s) for s in self.shape]
        total_shape = self.shape
        for lin, idx in enumerate(itertools.product(*ranges)):
            _state["cell"] = lin
            _state["shape"] = total_shape
            yield idx if len(idx) > 1 else idx[0]
        _state["cell"] = None

    def __getitem__(self, idx):
        idx = self._idx(idx)
        src = self.read_arr if self.read_arr is not None else self.arr
        if self.n:
            return Vec(src[idx], self.is_int)
        v = src[idx]
        return int(v) if self.is_int else np.float32(v)

    def __setitem__(self, idx, val):
        idx = self._idx(idx)
        if isinstance(val, Vec):
            val = val.arr
        self.arr[idx] = val

    def to_numpy(self):
        return self.arr.copy()

    def from_numpy(self, a):
        self.arr[...] = a

    def fill(self, v):
        self.arr[...] = v


def field(dtype, shape):
    return Field(dtype, shape)


class Vector(Vec):
    def __init__(self, values):
        super().__init__(np.array([np.float32(v) for v in values], dtype=np.float32), False)

    @staticmethod
    def field(n, dtype, shape):
        return Field(dtype, shape, n)

    @staticmethod
    def zero(dtype, n):
        return Vec(np.zeros(n, dtype=np.int32 if dtype == i32 else np.float32), dtype == i32)


def static(x):
    return x


def ndrange(*dims):
    ranges = [range(d) for d in dims]
    shape = tuple(dims)
    for lin, idx in enumerate(itertools.product(*ranges)):
        _state["cell"] = lin
        _state["shape"] = shape
        yield idx
    _state["cell"] = None


def cast(x, dtype):
    if dtype == i32:
        return int(x)
    return np.float32(x)


def floor(x, dtype=None):
    v = np.floor(np.float32(x))
    return int(v) if dtype == i32 else np.float32(v)


def _round_d(fn, x):
    return np.float32(fn(np.float64(np.float32(x))))


def sqrt(x):
    return np.float32(np.sqrt(np.float32(x)))


def sin(x):
    return _round_d(np.sin, x)


def cos(x):
    return _round_d(np.cos, x)


def log(x):
    return _round_d(np.log, x)


def exp(x):
    return _round_d(np.exp, x)


def pow(x, n):
    if isinstance(n, int) and n == 2:
        x = np.float32(x)
        return x * x
    return np.float32(np.float32(x) ** n)


def abs(x):  # noqa: A001 - Taichi name
    if isinstance(x, (int, np.integer)):
        return int(x if x >= 0 else -x)
    return np.float32(x if x >= 0 else -x)


def _typed(a, b, pick):
    r = pick
    if isinstance(a, (float, np.floating)) or isinstance(b, (float, np.floating)):
        return np.float32(r)
    return r


def max(a, b):  # noqa: A001
    return _typed(a, b, a if a > b else b)


def min(a, b):  # noqa: A001
    return _typed(a, b, a if a < b else b)


def random(dtype=f32):
    hook = _state["random_hook"]
    if hook is None:
        raise RuntimeError("ti.random called without a hook")
    return hook(_state["kernel"], _state["cell"])


def _atomic_add(fld, idx, v):
    idx = fld._idx(idx)
    if _state["deferred"] is not None and fld.name in ("free_surface_mass",):
        _state["deferred"].append((fld, idx, v, _state["cell"]))
        return 0
    old = fld.arr[idx]
    fld.arr[idx] = old + v
    return old


def atomic_add(target, v):  # only reached if the rewrite missed a call
    raise RuntimeError("atomic_add on a value; the source rewrite should have caught this")


# ---------------------------------------------------------------------------
# source rewriting
# ---------------------------------------------------------------------------
class _Rewrite(ast.NodeTransformer):
    def visit_Call(self, node):
        self.generic_visit(node)
        f = node.func
        if (isinstance(f, ast.Attribute) and f.attr == "atomic_add" and isinstance(f.value, ast.Name)
                and f.value.id == "ti" and node.args and isinstance(node.args[0], ast.Subscript)):
            sub = node.args[0]
            idx = sub.slice
            return ast.copy_location(ast.Call(
                func=ast.Attribute(value=ast.Name(id="ti", ctx=ast.Load()), attr="_atomic_add", ctx=ast.Load()),
                args=[sub.value, idx, node.args[1]], keywords=[]), node)
        if isinstance(f, ast.Name) and f.id in ("max", "min"):
            node.func = ast.Attribute(value=ast.Name(id="ti", ctx=ast.Load()), attr=f.id, ctx=ast.Load())
        elif isinstance(f, ast.Name) and f.id == "float":
            return ast.copy_location(ast.Call(
                func=ast.Attribute(value=ast.Name(id="ti", ctx=ast.Load()), attr="_to_f32", ctx=ast.Load()),
                args=node.args, keywords=[]), node)
        return node

    def visit_Assign(self, node):
        self.generic_visit(node)
        if len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
            node.value = ast.Call(
                func=ast.Attribute(value=ast.Name(id="ti", ctx=ast.Load()), attr="_assign", ctx=ast.Load()),
                args=[ast.Call(func=ast.Name(id="locals", ctx=ast.Load()), args=[], keywords=[]),
                      ast.Constant(name), node.value], keywords=[])
        return node


def _assign(loc, name, v):
    if name in loc:
        old = loc[name]
        if isinstance(old, np.float32):
            return np.float32(v)
        if isinstance(old, bool):
            return v
        if isinstance(old, (int, np.integer)) and not isinstance(v, bool):
            return int(v)
        return v
    if isinstance(v, bool):
        return v
    if isinstance(v, (float, np.floating)):
        return np.float32(v)
    if isinstance(v, np.integer):
        return int(v)
    return v


_ANNOT = {}


def _compile(fn):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    fdef = _Rewrite().visit(fdef)
    mod = ast.Module(body=[fdef], type_ignores=[])
    ast.fix_missing_locations(mod)
    g = {}
    for key, val in fn.__globals__.items():
        if isinstance(val, np.floating):
            val = float(val)
        elif isinstance(val, np.integer) and not isinstance(val, np.bool_):
            val = int(val)
        g[key] = val
    import sys
    g["ti"] = sys.modules[__name__]
    code = compile(mod, filename=inspect.getsourcefile(fn) or "<kernel>", mode="exec")
    exec(code, g)
    return g[fn.__name__], g


class _Callable:
    def __init__(self, fn, is_kernel):
        self.fn = fn
        self.is_kernel = is_kernel
        self.compiled = None
        self.sig = inspect.signature(fn)
        self.__name__ = fn.__name__

    def __call__(self, *args):
        if self.compiled is None:
            self.compiled, self.globals = _compile(self.fn)
            for key, val in self.globals.items():
                if isinstance(val, Field):
                    val.name = key
        cast_args = []
        for a, (pname, prm) in zip(args, self.sig.parameters.items()):
            ann = prm.annotation
            if ann == "f32" or ann is f32:
                a = np.float32(a)
            elif ann == "i32" or ann is i32:
                a = int(a)
            cast_args.append(a)
        if not self.is_kernel:
            r = self.compiled(*cast_args)
            ret = self.sig.return_annotation
            if ret is f32 or ret == "f32":
                r = np.float32(r)
            return r
        name = self.fn.__name__
        _state["calls"][name] = _state["calls"].get(name, 0) + 1
        prev_kernel = _state["kernel"]
        _state["kernel"] = name
        racy = name in ("redistribute_vof_mass_excess", "remove_orphan_vof_interface_cells")
        snap_fields = []
        if racy:
            _state["deferred"] = []
            for key in ("free_surface_mass", "free_surface_fill", "free_surface_type"):
                fld = self.globals.get(key)
                if isinstance(fld, Field):
                    fld.read_arr = fld.arr.copy()
                    snap_fields.append(fld)
        try:
            return self.compiled(*cast_args)
        finally:
            _state["kernel"] = prev_kernel
            if racy:
                for fld in snap_fields:
                    fld.read_arr = None
                _apply_deferred(name)
                _state["deferred"] = None


def _apply_deferred(kernel_name):
    """Apply deferred atomic adds grouped by receiver, in the oracle's
    order: donors sorted by the (q, distance) of the donor->receiver link."""
    adds = _state["deferred"] or []
    if not adds:
        return
    fld = adds[0][0]
    nz, ny, nx = fld.shape
    cx = (0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0)
    cy = (0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1)
    cz = (0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1)

    def key(donor_lin, ridx):
        dk, rem = divmod(donor_lin, ny * nx)
        dj, di = divmod(rem, nx)
        rk, rj, ri = ridx
        if (dk, dj, di) == (rk, rj, ri):
            return (99, 99)  # self add goes last
        for q in range(1, 19):
            for dist in range(1, 5):
                if ((di + dist * cx[q]) % nx == ri and (dj + dist * cy[q]) % ny == rj
                        and dk + dist * cz[q] == rk):
                    return (q, dist)
        return (98, 98)

    by_recv = {}
    for (f, idx, v, donor) in adds:
        by_recv.setdefault(idx, []).append((key(donor, idx), v))
    for idx, lst in by_recv.items():
        lst.sort(key=lambda t: t[0])
        acc = fld.arr[idx]
        for _, v in lst:
            acc = np.float32(acc + v)
        fld.arr[idx] = acc


def kernel(fn):
    return _Callable(fn, True)


def func(fn):
    return _Callable(fn, False)


_to_f32 = _to_f32
_assign = _assign
