"""Serial numpy stand-in for the ``taichi`` package -- TEST INFRASTRUCTURE ONLY.

Taichi is not installable in this container, so the golden fixtures under
``tests/golden/`` are produced by executing the waam_twin reference's own,
unmodified ``kernels.py`` / ``cumulant_kernel.py`` / ``twin.py`` /
``solvers/coupled_step.py`` source on top of this module.  It implements only
the subset of the Taichi API that those files use:

* ``ti.field`` / ``ti.Vector.field`` backed by numpy arrays (``[None]`` -> 0-d),
* ``@ti.kernel`` / ``@ti.func``: the function source is re-compiled with its
  annotations stripped, ``ti.atomic_*(A[idx], v)`` rewritten to
  ``ti._atomic_*(A, idx, v)`` and integer powers ``x ** n`` expanded into
  repeated multiplication (what Taichi does for a constant integer exponent),
* scalar arguments annotated ``ti.f32`` / ``ti.i32`` are coerced to float32 /
  int on entry, and ``-> ti.f32`` function results are coerced on return, so
  arithmetic runs in float32 like a Taichi kernel with ``default_fp=f32``,
* struct-for loops run serially in lexicographic (i, j, k) order.

Racy in-place kernels.  Two reference kernels read neighbours of the field
they update in place (``advect_diffuse_temperature`` on ``H``,
``apply_contact_angle_phi_bc`` on ``phi``); real Taichi runs them in parallel
with an undefined result.  ``SNAPSHOT_SEMANTICS`` pins the deterministic
semantics the B200 build implements:

* ``"cell"``:   every read of another cell sees the value from before the
  kernel (Jacobi / snapshot semantics); a cell sees its own writes.
* ``"column"``: reads inside the cell's own (i, j) column see the live values
  (sequential in k, as the serial order gives), reads of other columns see the
  value from before the kernel.

Set ``SNAPSHOT_SEMANTICS = {}`` to get the plain serial semantics instead.
"""
from __future__ import annotations

import ast
import builtins
import inspect
import itertools
import math as _pymath
import textwrap
import types as _types

import numpy as np

f32 = np.float32
i32 = np.int32
f64 = np.float64
u8 = np.uint8
cpu = "cpu"
cuda = "cuda"
vulkan = "vulkan"
gpu = "gpu"
WARN = 0
INFO = 1


class _Cfg:
    arch = "shim"
    cpu_max_num_threads = 1


cfg = _Cfg()

# kernel name -> {argument name: "cell" | "column"}
SNAPSHOT_SEMANTICS = {
    "advect_diffuse_temperature": {"H": "cell"},
    "advect_diffuse_temperature_variable": {"H": "cell"},
    "apply_contact_angle_phi_bc": {"phi": "column"},
}


def init(arch=None, **kw):
    return None


def reset():
    return None


def template():
    return None


def static(x):
    return x


def ndrange(*dims):
    rs = []
    for d in dims:
        if isinstance(d, (int, np.integer)):
            rs.append(range(int(d)))
        else:
            rs.append(range(int(d[0]), int(d[1])))
    return itertools.product(*rs)


def grouped(fld):
    return (tuple(ix) for ix in np.ndindex(*fld.shape))


def cast(x, dt):
    if dt is i32 or dt is int:
        return int(x)
    return dt(x)


def select(c, a, b):
    return a if c else b


def min(*a):  # noqa: A001 - Taichi API name
    return builtins.min(*a)


def max(*a):  # noqa: A001 - Taichi API name
    return builtins.max(*a)


def abs(x):  # noqa: A001 - Taichi API name
    return builtins.abs(x)


def sqrt(x):
    return np.sqrt(f32(x))


def cos(x):
    return np.cos(f32(x))


def sin(x):
    return np.sin(f32(x))


_rng = np.random.default_rng(0)


def random(dtype=None):
    return f32(_rng.random())


class _Math:
    pi = f32(_pymath.pi)

    @staticmethod
    def exp(x):
        return np.exp(f32(x))


math = _Math()


class Field:
    """Dense field backed by a numpy array."""

    def __init__(self, dtype, shape):
        if shape == () or shape is None:
            shape = ()
        elif isinstance(shape, (int, np.integer)):
            shape = (int(shape),)
        else:
            shape = tuple(int(s) for s in shape)
        self.dtype = dtype
        self.arr = np.zeros(shape, dtype=dtype)
        self.shape = self.arr.shape

    @staticmethod
    def _k(key):
        return () if key is None else key

    def __getitem__(self, key):
        return self.arr[self._k(key)]

    def __setitem__(self, key, v):
        self.arr[self._k(key)] = v

    def __iter__(self):
        return iter(np.ndindex(*self.shape))

    def to_numpy(self):
        return self.arr.copy()

    def from_numpy(self, a):
        self.arr[...] = a

    def copy_from(self, o):
        self.arr[...] = o.arr

    def fill(self, v):
        self.arr[...] = v


class _SnapshotField:
    """Proxy giving a kernel snapshot semantics on one in-place field."""

    def __init__(self, fld, mode):
        self.fld = fld
        self.snap = fld.arr.copy()
        self.mode = mode
        self.shape = fld.shape
        self.dtype = fld.dtype
        self.cur = None

    def __iter__(self):
        for idx in np.ndindex(*self.shape):
            self.cur = idx
            yield idx
        self.cur = None

    def _live(self, key):
        if self.cur is None or not isinstance(key, tuple):
            return True
        if self.mode == "cell":
            return tuple(int(k) for k in key) == self.cur
        return int(key[0]) == self.cur[0] and int(key[1]) == self.cur[1]

    def __getitem__(self, key):
        if self._live(key):
            return self.fld.arr[key]
        return self.snap[key]

    def __setitem__(self, key, v):
        self.fld.arr[key] = v


def field(dtype, shape=()):
    return Field(dtype, shape)


class _Vec(np.ndarray):
    @property
    def x(self):
        return self[0]

    @property
    def y(self):
        return self[1]

    @property
    def z(self):
        return self[2]


class VectorField(Field):
    def __init__(self, n, dtype, shape):
        super().__init__(dtype, shape)
        self.arr = np.zeros(self.shape + (n,), dtype)

    def __getitem__(self, key):
        return self.arr[key].view(_Vec)

    def __iter__(self):
        return iter(np.ndindex(*self.shape))


class Vector:
    def __new__(cls, v):
        return np.asarray(v, dtype=f32).view(_Vec)

    @staticmethod
    def field(n, dtype, shape):
        return VectorField(n, dtype, shape)


class _Types:
    @staticmethod
    def vector(n, dt):
        return None


types = _Types()


class _Lang:
    class impl:
        @staticmethod
        def get_runtime():
            return _types.SimpleNamespace(prog=object())


lang = _Lang()
StructField = Field
Struct = dict


def _atomic(op):
    def f(fld, key, v):
        old = fld[key]
        fld[key] = op(old, v)
        return old

    return f


_atomic_add = _atomic(lambda a, b: a + b)
_atomic_sub = _atomic(lambda a, b: a - b)
_atomic_max = _atomic(lambda a, b: a if a >= b else b)
_atomic_min = _atomic(lambda a, b: a if a <= b else b)


def _ipow(x, n):
    out = x
    for _ in range(n - 1):
        out = out * x
    return out


class _Rewrite(ast.NodeTransformer):
    def visit_Call(self, node):
        self.generic_visit(node)
        fn = node.func
        if (
            isinstance(fn, ast.Attribute)
            and isinstance(fn.value, ast.Name)
            and fn.value.id == "ti"
            and fn.attr.startswith("atomic_")
            and isinstance(node.args[0], ast.Subscript)
        ):
            sub = node.args[0]
            return ast.copy_location(
                ast.Call(
                    func=ast.Attribute(value=ast.Name("ti", ast.Load()), attr="_" + fn.attr, ctx=ast.Load()),
                    args=[sub.value, sub.slice, node.args[1]],
                    keywords=[],
                ),
                node,
            )
        return node

    def visit_BinOp(self, node):
        self.generic_visit(node)
        if (
            isinstance(node.op, ast.Pow)
            and isinstance(node.right, ast.Constant)
            and isinstance(node.right.value, int)
            and 1 <= node.right.value <= 8
        ):
            return ast.copy_location(
                ast.Call(
                    func=ast.Attribute(value=ast.Name("ti", ast.Load()), attr="_ipow", ctx=ast.Load()),
                    args=[node.left, node.right],
                    keywords=[],
                ),
                node,
            )
        return node


def _scalar_kinds(fn):
    kinds = {}
    ret = None
    try:
        sig = inspect.signature(fn)
    except (TypeError, ValueError):
        return kinds, ret
    for name, p in sig.parameters.items():
        if p.annotation is f32:
            kinds[name] = f32
        elif p.annotation is i32:
            kinds[name] = i32
    if sig.return_annotation is f32:
        ret = f32
    return kinds, ret


def _compile(fn):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    for a in fdef.args.args:
        a.annotation = None
    fdef.returns = None
    tree = ast.fix_missing_locations(_Rewrite().visit(tree))
    ns = {}
    exec(compile(tree, inspect.getsourcefile(fn), "exec"), fn.__globals__, ns)
    return ns[fn.__name__]


def _wrap(fn, is_kernel):
    cache = {}
    kinds, ret = _scalar_kinds(fn)
    names = list(inspect.signature(fn).parameters)

    def wrapper(*a, **k):
        if "f" not in cache:
            cache["f"] = _compile(fn)
        args = list(a)
        for idx, name in enumerate(names[: len(args)]):
            kd = kinds.get(name)
            if kd is f32:
                args[idx] = f32(args[idx])
            elif kd is i32:
                args[idx] = int(args[idx])
        for name in list(k):
            kd = kinds.get(name)
            if kd is f32:
                k[name] = f32(k[name])
            elif kd is i32:
                k[name] = int(k[name])
        snaps = SNAPSHOT_SEMANTICS.get(fn.__name__, {}) if is_kernel else {}
        for idx, name in enumerate(names[: len(args)]):
            if name in snaps:
                args[idx] = _SnapshotField(args[idx], snaps[name])
        out = cache["f"](*args, **k)
        if ret is f32 and out is not None:
            out = f32(out)
        return out

    wrapper.__name__ = fn.__name__
    wrapper.__wrapped__ = fn
    return wrapper


def kernel(fn):
    return _wrap(fn, True)


def func(fn):
    return _wrap(fn, False)
