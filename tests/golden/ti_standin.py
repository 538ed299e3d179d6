"""A serial NumPy stand-in for the part of Taichi that nh-flood-2d's step
kernels use. It is test infrastructure: make_step_golden.py installs it as
the ``taichi`` module so that the reference's own kernel source
(core/solver_compact.py, core/clock.py, core/pressure.py,
core/device_budget.py) runs unchanged on the CPU, and it writes the
results as golden vectors for the step.

Taichi is a compiler. This module reproduces the semantics that the
reference's kernels rely on, not Taichi's implementation:

* Kernels run their top-level loops one after another, and each loop
  serially. The reference's passes have one writer per element and use
  atomics only for order-free min/max/count reductions and for the F32
  budget diagnostics. So a serial order is one valid schedule of the
  parallel one, and only the order of those F32 diagnostic additions is
  fixed here.
* Types follow Taichi's rules with default_fp = f32 and default_ip = i32.
  F32 values are NumPy float32 scalars. NumPy 2's weak Python scalars
  (NEP 50) round a Python float constant to F32 where it meets an F32
  value, which is what Taichi does with a constant in an F32 expression.
  Arithmetic on Python constants alone folds in F64, as Taichi's frontend
  folds it. I32 values are Python ints. U32 values are ``U32``, which wraps
  modulo 2**32 and wins over i32 in mixed operations (Taichi's "signed +
  unsigned -> unsigned"). Shifts keep the type of their left operand.
* Each F32 operation is rounded once, in the source's order. Taichi's CPU
  backend compiles with fast-math, which may contract a*b+c into an FMA.
  That contraction is not reproduced, and the tolerances of the comparison
  (1 mm of depth, 1e-4 m2/s of discharge) exist for it.
* ``x ** y`` with a float exponent calls the C library's powf, and
  ``ti.exp`` calls expf, which are the functions an LLVM CPU build calls.
  With an integer exponent, ``**`` multiplies (x ** 2 == x * x), as Taichi
  lowers a constant integer power. ``set_math('rounded')`` switches both
  to the exactly rounded F32 value, computed in F64 and rounded once.
* ``ti.atomic_*(field[i], v)`` takes the field element as its target. Python
  evaluates ``field[i]`` to a value, so ``transform`` rewrites these calls
  (and ``**``) before the source is compiled, as Taichi's own frontend
  rewrites the kernel's AST. Nothing else in the source is changed.
* A field read or write outside the field's shape raises IndexError; Taichi
  would not check it.
"""
from __future__ import annotations

import ast
import ctypes
import math
import sys
import types

import numpy as np

_MASK = 0xFFFFFFFF
_LIBM = ctypes.CDLL('libm.so.6')
_LIBM.powf.restype = ctypes.c_float
_LIBM.powf.argtypes = [ctypes.c_float, ctypes.c_float]
_LIBM.expf.restype = ctypes.c_float
_LIBM.expf.argtypes = [ctypes.c_float]
_MATH = {'mode': 'libm'}


def set_math(mode: str) -> None:
    """'libm': the C library's powf/expf; 'rounded': exactly rounded F32."""
    if mode not in ('libm', 'rounded'):
        raise ValueError(mode)
    _MATH['mode'] = mode


# ------------------------------------------------------------------ types

class DataType:
    def __init__(self, name, np_dtype):
        self.name, self.np = name, np.dtype(np_dtype)

    def __call__(self, value):
        return cast(value, self)

    def __repr__(self):
        return f'ti.{self.name}'


i32 = DataType('i32', np.int32)
u32 = DataType('u32', np.uint32)
f32 = DataType('f32', np.float32)
u8 = DataType('u8', np.uint8)
i64 = DataType('i64', np.int64)
f64 = DataType('f64', np.float64)


def _wrap_i32(v: int) -> int:
    return ((int(v) + (1 << 31)) & _MASK) - (1 << 31)


def _is_float(v) -> bool:
    return isinstance(v, (float, np.floating))


def _as_int(o):
    """The integer value of an i32/u32/bool operand, else None."""
    if isinstance(o, U32):
        return o.v
    if isinstance(o, (bool, int, np.integer, np.bool_)):
        return int(o)
    return None


class U32:
    """An unsigned 32-bit value with Taichi's wrap-around and promotion."""
    __slots__ = ('v',)

    def __init__(self, v):
        self.v = int(v) & _MASK

    def __index__(self):
        return self.v

    __int__ = __index__

    def __bool__(self):
        return self.v != 0

    def __float__(self):
        return float(self.v)

    def __hash__(self):
        return hash(self.v)

    def __repr__(self):
        return f'U32({self.v})'

    def _f32(self):
        return np.float32(self.v)

    def _bin(self, o, fn, reflected=False):
        x = _as_int(o)
        if x is None:
            if _is_float(o):  # integer with float: the float type (f32)
                a, b = self._f32(), np.float32(o)
                return fn(b, a) if reflected else fn(a, b)
            return NotImplemented
        return U32(fn(x, self.v) if reflected else fn(self.v, x))

    def __add__(self, o): return self._bin(o, lambda a, b: a + b)
    def __radd__(self, o): return self._bin(o, lambda a, b: a + b, True)
    def __sub__(self, o): return self._bin(o, lambda a, b: a - b)
    def __rsub__(self, o): return self._bin(o, lambda a, b: a - b, True)
    def __mul__(self, o): return self._bin(o, lambda a, b: a * b)
    def __rmul__(self, o): return self._bin(o, lambda a, b: a * b, True)

    def _bits(self, o, fn, reflected=False):
        x = _as_int(o)
        if x is None:
            return NotImplemented
        return U32(fn(x & _MASK, self.v) if reflected else fn(self.v, x & _MASK))

    def __and__(self, o): return self._bits(o, lambda a, b: a & b)
    def __rand__(self, o): return self._bits(o, lambda a, b: a & b, True)
    def __or__(self, o): return self._bits(o, lambda a, b: a | b)
    def __ror__(self, o): return self._bits(o, lambda a, b: a | b, True)
    def __xor__(self, o): return self._bits(o, lambda a, b: a ^ b)
    def __rxor__(self, o): return self._bits(o, lambda a, b: a ^ b, True)

    def __lshift__(self, o):
        s = _as_int(o)
        if s is None or not 0 <= s < 32:
            raise ValueError(f'u32 shift by {o}')
        return U32(self.v << s)

    def __rshift__(self, o):
        s = _as_int(o)
        if s is None or not 0 <= s < 32:
            raise ValueError(f'u32 shift by {o}')
        return U32(self.v >> s)

    def __floordiv__(self, o):
        x = _as_int(o)
        return U32(self.v // (x & _MASK))

    def __mod__(self, o):
        x = _as_int(o)
        return U32(self.v % (x & _MASK))

    def _cmp(self, o, fn):
        x = _as_int(o)
        if x is None:
            if _is_float(o):
                return bool(fn(self._f32(), np.float32(o)))
            return NotImplemented
        return bool(fn(self.v, x & _MASK))

    def __eq__(self, o): return self._cmp(o, lambda a, b: a == b)
    def __ne__(self, o): return self._cmp(o, lambda a, b: a != b)
    def __lt__(self, o): return self._cmp(o, lambda a, b: a < b)
    def __le__(self, o): return self._cmp(o, lambda a, b: a <= b)
    def __gt__(self, o): return self._cmp(o, lambda a, b: a > b)
    def __ge__(self, o): return self._cmp(o, lambda a, b: a >= b)


def cast(x, dtype):
    if dtype is f32:
        return np.float32(x.v if isinstance(x, U32) else x)
    if dtype is f64:
        return float(x.v if isinstance(x, U32) else x)
    if _is_float(x):
        x = math.trunc(float(x))  # float -> int truncates toward zero
    v = _as_int(x)
    if dtype is u32:
        return U32(v)
    if dtype is i32:
        return _wrap_i32(v)
    if dtype is u8:
        return v & 0xFF
    if dtype is i64:
        return v
    raise TypeError(dtype)


def bit_cast(x, dtype):
    if dtype is u32:
        return U32(int(np.float32(x).view(np.uint32)))
    if dtype is i32:
        return int(np.float32(x).view(np.int32))
    if dtype is f32:
        return np.uint32(_as_int(x) & _MASK).view(np.float32)
    raise TypeError(dtype)


# ----------------------------------------------------------------- fields

class Field:
    """A dense field: one NumPy array, read and written element by element."""

    def __init__(self, dtype, shape=()):
        if shape is None:
            shape = ()
        if isinstance(shape, (int, np.integer)):
            shape = (int(shape),)
        self.dtype = dtype
        self.arr = np.zeros(tuple(int(s) for s in shape), dtype=dtype.np)
        self._n0 = self.arr.shape[0] if self.arr.ndim == 1 else -1
        self._kind = {'f32': 0, 'u32': 1, 'f64': 2}.get(dtype.name, 3)

    @property
    def shape(self):
        return self.arr.shape

    def _key(self, key):
        if key.__class__ is int and 0 <= key < self._n0:  # the common case: a 1-D field
            return key
        if key.__class__ is tuple and len(key) == 2 and self.arr.ndim == 2:
            a, b = key
            if a.__class__ is int and b.__class__ is int and 0 <= a < self.arr.shape[0] and 0 <= b < self.arr.shape[1]:
                return key
        if key is None:
            if self.arr.ndim:
                raise IndexError('field[None] on a field with a shape')
            return ()
        key = key if isinstance(key, tuple) else (key,)
        if len(key) != self.arr.ndim:
            raise IndexError(f'{len(key)} indices for a {self.arr.ndim}-D field')
        out = []
        for k, n in zip(key, self.arr.shape):
            k = int(k)
            if not 0 <= k < n:
                raise IndexError(f'index {k} outside 0..{n - 1}')
            out.append(k)
        return tuple(out)

    def _convert(self, value):
        t = self.dtype
        if t is f32:
            return np.float32(value.v if isinstance(value, U32) else value)
        if t is f64:
            return float(value)
        return cast(value, t)

    def __getitem__(self, key):
        v = self.arr[self._key(key)]
        kind = self._kind
        if kind == 0:
            return v
        if kind == 1:
            return U32(int(v))
        if kind == 2:
            return float(v)
        return int(v)

    def __setitem__(self, key, value):
        self.arr[self._key(key)] = self._convert(value)

    def __iter__(self):
        if self.arr.ndim == 1:
            return iter(range(self.arr.shape[0]))
        return iter(np.ndindex(*self.arr.shape))

    def from_numpy(self, a):
        a = np.asarray(a)
        if a.size != self.arr.size:
            raise ValueError(f'from_numpy: {a.shape} into {self.arr.shape}')
        self.arr[...] = a.reshape(self.arr.shape).astype(self.arr.dtype)

    def to_numpy(self):
        return self.arr.copy()

    def fill(self, value):
        self.arr[...] = self._convert(value)


def field(dtype, shape=(), **_):
    return Field(dtype, shape)


# ------------------------------------------------------------- functions

_F32 = np.float32


def _result(r, args):
    kinds = {a.__class__ for a in args}
    if kinds == {_F32}:
        return r
    if U32 in kinds and not any(_is_float(a) for a in args):
        return U32(r)
    if any(_is_float(a) for a in args):
        return np.float32(r)
    return r


def max(*args):  # noqa: A001 - Taichi's name
    r = args[0]
    for a in args[1:]:
        if a > r:
            r = a
    return _result(r, args)


def min(*args):  # noqa: A001
    r = args[0]
    for a in args[1:]:
        if a < r:
            r = a
    return _result(r, args)


def select(cond, a, b):
    return _result(a if cond else b, (a, b))


def sqrt(x):
    return np.sqrt(np.float32(x))


def exp(x):
    x = np.float32(x)
    if _MATH['mode'] == 'libm':
        return np.float32(_LIBM.expf(float(x)))
    return np.float32(math.exp(float(x)))


def pow(x, y):  # noqa: A001
    if isinstance(y, (int, np.integer)) and not isinstance(y, bool) and y >= 0:
        if isinstance(x, (int, np.integer, U32)):
            return x ** int(y)
        x = np.float32(x)
        result, base, n = np.float32(1.0), x, int(y)
        first = True
        while n:  # exponentiation by squaring, as a constant integer power is lowered
            if n & 1:
                result = base if first else result * base
                first = False
            n >>= 1
            if n:
                base = base * base
        return result
    x, y = np.float32(x), np.float32(y)
    if _MATH['mode'] == 'libm':
        return np.float32(_LIBM.powf(float(x), float(y)))
    return np.float32(float(x) ** float(y))


def abs(x):  # noqa: A001
    return x if isinstance(x, U32) else (np.abs(x) if _is_float(x) else (x if x >= 0 else -x))


def static(x, *rest):
    return x if not rest else (x,) + rest


def template():
    return None


def func(fn):
    return fn


def kernel(fn):
    return fn


def data_oriented(cls):
    return cls


def _atomic(op, target, key, value):
    """ti.atomic_<op>(target[key], value): update the element, return the old value."""
    old = target[key]
    if op == 'add':
        new = old + value
    elif op == 'sub':
        new = old - value
    elif op == 'min':
        new = value if value < old else old
    elif op == 'max':
        new = value if value > old else old
    else:
        raise ValueError(op)
    target[key] = new
    return old


def atomic_add(*_):
    raise RuntimeError('ti.atomic_add needs a field element; compile the source with transform()')


atomic_min = atomic_max = atomic_sub = atomic_add


# -------------------------------------------------------------- frontend

class _Frontend(ast.NodeTransformer):
    """Rewrites ti.atomic_<op>(f[k], v) into __ti_atomic__('<op>', f, k, v)
    and a ** b into ti.pow(a, b)."""

    def visit_Call(self, node):
        self.generic_visit(node)
        f = node.func
        if (isinstance(f, ast.Attribute) and isinstance(f.value, ast.Name) and f.value.id == 'ti'
                and f.attr.startswith('atomic_') and node.args and isinstance(node.args[0], ast.Subscript)):
            target = node.args[0]
            key = target.slice
            call = ast.Call(func=ast.Name('__ti_atomic__', ast.Load()),
                            args=[ast.Constant(f.attr[len('atomic_'):]), target.value, key] + node.args[1:],
                            keywords=[])
            return ast.copy_location(call, node)
        return node

    def visit_BinOp(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Pow):
            call = ast.Call(func=ast.Attribute(ast.Name('ti', ast.Load()), 'pow', ast.Load()),
                            args=[node.left, node.right], keywords=[])
            return ast.copy_location(call, node)
        return node


def transform(tree):
    tree = _Frontend().visit(tree)
    return ast.fix_missing_locations(tree)


def namespace(**names) -> dict:
    ns = {'__ti_atomic__': _atomic, 'ti': sys.modules[__name__]}
    ns.update(names)
    return ns


def load_module(path, name, package):
    """Import one reference module from its unchanged source file, through
    ``transform``, with this stand-in installed as ``taichi``."""
    install()
    module = types.ModuleType(name)
    module.__file__ = str(path)
    module.__package__ = package
    sys.modules[name] = module
    tree = transform(ast.parse(open(path).read(), filename=str(path)))
    exec(compile(tree, str(path), 'exec'), module.__dict__)
    return module


def install() -> None:
    """Make ``import taichi`` resolve to this module."""
    sys.modules.setdefault('taichi', sys.modules[__name__])


# Taichi names the reference touches outside kernels (annotations, classes).
ScalarField = MatrixField = Field
cpu = gpu = 'cpu'
