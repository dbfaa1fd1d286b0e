"""Minimal stand-in for the ``taichi`` package, used ONLY to execute the
reference's own, unmodified ``dem/`` kernels on the CPU so that golden
input/output vectors can be generated from the reference itself.

This is test infrastructure (it lives under ``tests/golden``).  Nothing in the
product imports it.

Execution model
---------------
* ``@ti.kernel`` / ``@ti.func`` bodies run as plain, serial Python.  The
  outermost loop of a Taichi kernel is parallel in real Taichi; here it runs in
  ascending order, which is the deterministic order the product reproduces
  (e.g. particles inside an octree leaf or a hash bucket appear in ascending
  index order).
* Fields are numpy arrays.  Scalar element reads return Python ``int``/``float``
  so arithmetic is IEEE binary64 (floats) or exact integers (ints).  Integer
  results that real Taichi would wrap at 32 bits are only ever used here after
  ``& mask`` (the spatial hash), where the low bits are identical.
* ``x ** k`` with an integer literal ``k`` inside kernels is rewritten to
  exponentiation by squaring (``r**7 == (r*(r*r))*((r*r)*(r*r))``), the way
  Taichi lowers integer powers.  Python-scope code keeps Python semantics.
* ``ti.atomic_add(F[idx], v)`` is rewritten to an in-place update that returns
  the old value.
* No fused multiply-add and no re-association: every operation rounds once, in
  source order.  Real Taichi's LLVM CPU backend may contract or re-associate
  (``fast_math``), so the last bits of a real Taichi run are not pinned by this
  shim.
"""

from __future__ import annotations

import ast
import inspect
import math as _m
import textwrap
import types as _pytypes

import numpy as np

__version__ = (1, 7, 4)


# ---------------------------------------------------------------------------
# dtypes
# ---------------------------------------------------------------------------
class _DType:
    def __init__(self, name: str, np_dtype, py):
        self.name = name
        self.np = np.dtype(np_dtype)
        self.py = py

    def __call__(self, x):
        return self.py(x)

    def __repr__(self) -> str:
        return f"ti.{self.name}"


f64 = _DType("f64", np.float64, float)
f32 = _DType("f32", np.float32, float)
i32 = _DType("i32", np.int32, int)
i64 = _DType("i64", np.int64, int)
u8 = _DType("u8", np.uint8, int)
u32 = _DType("u32", np.uint32, int)

cpu = "cpu"
gpu = "gpu"
cuda = "cuda"
vulkan = "vulkan"


def init(*args, **kwargs):
    return None


def sync():
    return None


def reset():
    return None


# ---------------------------------------------------------------------------
# fields
# ---------------------------------------------------------------------------
def _norm_shape(shape):
    if shape is None:
        return ()
    if isinstance(shape, (int, np.integer)):
        return (int(shape),)
    return tuple(int(s) for s in shape)


class Field:
    def __init__(self, dtype: _DType, shape, n: int | None = None):
        self.dtype = dtype
        self.shape = _norm_shape(shape)
        self.n = n
        full = self.shape + ((n,) if n else ())
        self.arr = np.zeros(full, dtype=dtype.np)

    @staticmethod
    def _key(key):
        return () if key is None else key

    def __getitem__(self, key):
        v = self.arr[self._key(key)]
        if self.n is None:
            return v.item()
        return np.array(v, dtype=self.arr.dtype)

    def __setitem__(self, key, value):
        self.arr[self._key(key)] = value

    def to_numpy(self):
        return self.arr.copy()

    def from_numpy(self, a):
        self.arr[...] = np.asarray(a, dtype=self.arr.dtype).reshape(self.arr.shape)

    def fill(self, value):
        self.arr.fill(value)


def field(dtype, shape=None, **kwargs):
    return Field(dtype, shape)


class _VectorType:
    """``ti.Vector``: value constructor and ``.field`` factory."""

    def __call__(self, values, dt=None):
        return np.array(values, dtype=np.float64 if dt in (None, f64, f32) else dt.np)

    def field(self, n, dtype, shape=None, **kwargs):
        return Field(dtype, shape, n=n)


Vector = _VectorType()


# ---------------------------------------------------------------------------
# builtins used by the reference kernels
# ---------------------------------------------------------------------------
def sqrt(x):
    return _m.sqrt(x)


def floor(x):
    return float(_m.floor(x))


def cast(x, dtype):
    return dtype.py(x)


def max(a, b):  # noqa: A001 - mirrors ti.max
    return a if a >= b else b


def min(a, b):  # noqa: A001 - mirrors ti.min
    return a if a <= b else b


def abs(x):  # noqa: A001 - mirrors ti.abs
    return -x if x < 0 else x


def static(x):
    return x


def loop_config(**kwargs):
    return None


def ndrange(*dims):
    """``for i, j in ti.ndrange(a, b)``: the index tuples in row-major order."""
    import itertools

    return itertools.product(*(range(d) if isinstance(d, int) else range(*d) for d in dims))


def random(dtype=None):
    return float(np.random.random())


def select(cond, a, b):
    return a if cond else b


class _Math:
    @staticmethod
    def sign(x):
        return 1.0 if x > 0 else (-1.0 if x < 0 else 0.0)

    sqrt = staticmethod(sqrt)
    floor = staticmethod(floor)


math = _Math()  # ``ti.math.sign``


def template():
    return None


class _Types:
    @staticmethod
    def ndarray(*args, **kwargs):
        return None

    @staticmethod
    def vector(n, dtype):
        return None

    @staticmethod
    def matrix(n, m, dtype):
        return None


types = _Types()


def data_oriented(cls):
    return cls


def _ipow(base, k: int):
    """Exponentiation by squaring, as Taichi lowers ``x ** <int>``."""
    if k < 0:
        return 1.0 / _ipow(base, -k)
    result = None
    b = base
    while k:
        if k & 1:
            result = b if result is None else result * b
        k >>= 1
        if k:
            b = b * b
    return 1 if result is None else result


def _atomic_add_sub(container, index, value):
    old = container[index]
    container[index] = old + value
    return old


def atomic_add(x, value):  # only reachable if the AST rewrite missed a form
    raise NotImplementedError("ti.atomic_add on a non-subscript target")


# ---------------------------------------------------------------------------
# kernel transformation
# ---------------------------------------------------------------------------
class _Rewrite(ast.NodeTransformer):
    def visit_BinOp(self, node):
        self.generic_visit(node)
        if (
            isinstance(node.op, ast.Pow)
            and isinstance(node.right, ast.Constant)
            and isinstance(node.right.value, int)
            and not isinstance(node.right.value, bool)
        ):
            return ast.Call(
                func=ast.Attribute(value=ast.Name(id="ti", ctx=ast.Load()), attr="_ipow", ctx=ast.Load()),
                args=[node.left, node.right],
                keywords=[],
            )
        return node

    def visit_AugAssign(self, node):
        self.generic_visit(node)
        if (
            isinstance(node.op, ast.Pow)
            and isinstance(node.value, ast.Constant)
            and isinstance(node.value.value, int)
        ):
            raise NotImplementedError("augmented integer power in kernel")
        return node

    def visit_Call(self, node):
        self.generic_visit(node)
        f = node.func
        if (
            isinstance(f, ast.Attribute)
            and f.attr == "atomic_add"
            and isinstance(f.value, ast.Name)
            and f.value.id == "ti"
            and node.args
            and isinstance(node.args[0], ast.Subscript)
        ):
            sub = node.args[0]
            idx = sub.slice
            return ast.Call(
                func=ast.Attribute(
                    value=ast.Name(id="ti", ctx=ast.Load()), attr="_atomic_add_sub", ctx=ast.Load()
                ),
                args=[sub.value, idx, node.args[1]],
                keywords=[],
            )
        return node


def _transform(fn):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    fdef.returns = None
    for a in fdef.args.args + fdef.args.kwonlyargs:
        a.annotation = None
    _Rewrite().visit(tree)
    ast.fix_missing_locations(tree)
    code = compile(tree, filename=inspect.getsourcefile(fn) or "<kernel>", mode="exec")
    ns: dict = {}
    exec(code, fn.__globals__, ns)  # noqa: S102 - executes the reference's own kernel source
    out = ns[fdef.name]
    out.__wrapped_taichi__ = True
    return out


def kernel(fn):
    return _transform(fn)


def func(fn):
    return _transform(fn)


real_func = func
pyfunc = func
