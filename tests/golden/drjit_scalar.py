"""A scalar stand-in for the part of DrJit that gQuery's traversal code uses.

Used only to generate golden fixtures (tests/golden/make_golden.py): it lets the
reference's own Python traversal (bvh.py, bvh3d.py, snch.py, snch3d.py, math.py, the
primitive views) run one query at a time on the CPU, where DrJit cannot be installed.
`@dr.syntax` becomes the identity, so the reference's `while` / `if` statements run as
plain Python control flow on scalars.

Arithmetic is float32 with the rounding rules this project fixes for DrJit's library
calls (the same rules as gquery_b200/csrc/gq_fmath.h): Python operators are single
IEEE operations; dot = fma chain, norm = sqrt(dot), normalize = v * (1/sqrt(dot)),
lerp = fma(b, t, fma(-a, t, a)), cross = fma(a_j, b_k, -(a_k b_j)), clamp =
fmax(fmin(x, hi), lo), epsilon = 2^-24; acos/asin/atan2 are the shared implementation
exported by the oracle library.  fma is emulated exactly (exact rational rounding).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
import sys
import types
from fractions import Fraction

import numpy as np

F32 = np.float32

# ---------------------------------------------------------------------------
# exact fma in float32
# ---------------------------------------------------------------------------


def _round_f32(x: Fraction) -> np.float32:
    c = F32(float(x))
    if not np.isfinite(c):
        return c
    best, berr = c, abs(Fraction(float(c)) - x)
    for nb in (np.nextafter(c, F32(np.inf)), np.nextafter(c, F32(-np.inf))):
        if not np.isfinite(nb):
            continue
        e = abs(Fraction(float(nb)) - x)
        if e < berr or (e == berr and (int(nb.view(np.uint32)) & 1) == 0):
            best, berr = nb, e
    return F32(best)


def fma(a, b, c) -> np.float32:
    a, b, c = F32(a), F32(b), F32(c)
    if not (np.isfinite(a) and np.isfinite(b) and np.isfinite(c)):
        return F32(np.float64(a) * np.float64(b) + np.float64(c))
    p = np.float64(a) * np.float64(b)  # exact
    s = p + np.float64(c)
    # TwoSum error of the double addition: zero means s is exact
    bb = s - p
    err = (p - (s - bb)) + (np.float64(c) - bb)
    if err == 0:
        return F32(s)
    return _round_f32(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c)))


# ---------------------------------------------------------------------------
# scalar types
# ---------------------------------------------------------------------------


def _v(x):
    if isinstance(x, (Float, Int, Bool)):
        return x.v
    return x


class Bool:
    def __init__(self, v=False):
        self.v = v.v if isinstance(v, Bool) else (np.asarray(v, dtype=bool) if isinstance(v, np.ndarray) else bool(v))

    def __bool__(self):
        return bool(self.v)

    def __and__(self, o):
        return Bool(np.logical_and(self.v, _v(o)))

    __rand__ = __and__

    def __or__(self, o):
        return Bool(np.logical_or(self.v, _v(o)))

    __ror__ = __or__

    def __invert__(self):
        return Bool(np.logical_not(self.v))

    def __repr__(self):
        return f"Bool({self.v})"


class Float:
    def __init__(self, v=0.0):
        v = _v(v)
        self.v = np.asarray(v, dtype=F32) if isinstance(v, (np.ndarray, list)) else F32(v)

    def _b(self, o, op):
        return Float(op(self.v, F32(_v(o)) if not isinstance(_v(o), np.ndarray) else _v(o).astype(F32)))

    def __add__(self, o): return self._b(o, np.add)
    def __radd__(self, o): return Float(F32(_v(o)) + self.v)
    def __sub__(self, o): return self._b(o, np.subtract)
    def __rsub__(self, o): return Float(F32(_v(o)) - self.v)
    def __mul__(self, o):
        if isinstance(o, ArrayN):
            return o * self
        return self._b(o, np.multiply)
    def __rmul__(self, o): return Float(F32(_v(o)) * self.v)
    def __truediv__(self, o): return self._b(o, np.divide)
    def __rtruediv__(self, o): return Float(F32(_v(o)) / self.v)
    def __neg__(self): return Float(-self.v)
    def __lt__(self, o): return Bool(self.v < F32(_v(o)))
    def __le__(self, o): return Bool(self.v <= F32(_v(o)))
    def __gt__(self, o): return Bool(self.v > F32(_v(o)))
    def __ge__(self, o): return Bool(self.v >= F32(_v(o)))
    def __eq__(self, o): return Bool(self.v == F32(_v(o)))
    def __ne__(self, o): return Bool(self.v != F32(_v(o)))
    def __float__(self): return float(self.v)
    def __repr__(self): return f"Float({self.v})"
    def __hash__(self): return id(self)


class Int:
    def __init__(self, v=0):
        v = _v(v)
        if isinstance(v, np.ndarray):
            self.v = v.astype(np.int64) if v.dtype.kind != "f" else v.astype(np.float32).astype(np.int64)
        elif isinstance(v, (np.floating, float)):
            self.v = int(math.trunc(float(v)))  # DrJit Int(Float): truncation
        else:
            self.v = int(v)

    def _b(self, o, op):
        return Int(op(self.v, _v(o)))

    def __add__(self, o): return self._b(o, lambda a, b: a + b)
    __radd__ = __add__
    def __sub__(self, o): return self._b(o, lambda a, b: a - b)
    def __rsub__(self, o): return Int(_v(o) - self.v)
    def __mul__(self, o): return self._b(o, lambda a, b: a * b)
    __rmul__ = __mul__
    def __lt__(self, o): return Bool(self.v < _v(o))
    def __le__(self, o): return Bool(self.v <= _v(o))
    def __gt__(self, o): return Bool(self.v > _v(o))
    def __ge__(self, o): return Bool(self.v >= _v(o))
    def __eq__(self, o): return Bool(self.v == _v(o))
    def __ne__(self, o): return Bool(self.v != _v(o))
    def __index__(self): return int(self.v)
    def __int__(self): return int(self.v)
    def __repr__(self): return f"Int({self.v})"
    def __hash__(self): return id(self)


UInt = Int


class ArrayN:
    N = 0
    ELEM = Float

    def __init__(self, *args):
        if len(args) == 1 and isinstance(args[0], ArrayN):
            self.c = [self.ELEM(x) for x in args[0].c]
        elif len(args) == 1 and isinstance(args[0], np.ndarray):
            self.c = [self.ELEM(args[0][k]) for k in range(self.N)]
        elif len(args) == 0:
            self.c = [self.ELEM(0) for _ in range(self.N)]
        else:
            assert len(args) == self.N, (self.N, args)
            self.c = [a if isinstance(a, self.ELEM) else self.ELEM(a) for a in args]

    def numpy(self):
        return np.stack([np.asarray(x.v) for x in self.c])

    def __getitem__(self, k): return self.c[int(k)]
    def __setitem__(self, k, val): self.c[int(k)] = val if isinstance(val, self.ELEM) else self.ELEM(val)
    x = property(lambda s: s.c[0])
    y = property(lambda s: s.c[1])
    z = property(lambda s: s.c[2])

    def _zip(self, o, f):
        if isinstance(o, ArrayN):
            return type(self)(*[f(a, b) for a, b in zip(self.c, o.c)])
        return type(self)(*[f(a, o) for a in self.c])

    def __add__(self, o): return self._zip(o, lambda a, b: a + b)
    def __radd__(self, o): return self._zip(o, lambda a, b: b + a)
    def __sub__(self, o): return self._zip(o, lambda a, b: a - b)
    def __rsub__(self, o): return self._zip(o, lambda a, b: b - a)
    def __mul__(self, o): return self._zip(o, lambda a, b: a * b)
    def __rmul__(self, o): return self._zip(o, lambda a, b: b * a)
    def __truediv__(self, o): return self._zip(o, lambda a, b: a / b)
    def __neg__(self): return type(self)(*[-a for a in self.c])
    def __repr__(self): return f"{type(self).__name__}({[x.v for x in self.c]})"


class Array2(ArrayN): N = 2
class Array3(ArrayN): N = 3
class Array4(ArrayN): N = 4
class Array2i(ArrayN): N, ELEM = 2, Int
class Array3i(ArrayN): N, ELEM = 3, Int
class Array4i(ArrayN): N, ELEM = 4, Int


class _Unused:
    def __init__(self, *a, **k):
        raise NotImplementedError("not used by the traversal")


# ---------------------------------------------------------------------------
# drjit functions
# ---------------------------------------------------------------------------

inf = float("inf")
pi = math.pi
_fmath = None


def _fm(which, x, y=0.0):
    global _fmath
    if _fmath is None:
        import oracle
        _fmath = oracle.lib().orc_fmath
        _fmath.restype = None
    xa = np.array([F32(x)], F32)
    ya = np.array([F32(y)], F32)
    out = np.empty(1, F32)
    _fmath(C.c_int(which), C.c_void_p(xa.ctypes.data), C.c_void_p(ya.ctypes.data), C.c_void_p(out.ctypes.data),
           C.c_int64(1))
    return Float(out[0])


def syntax(f=None, **kw):
    return f if f is not None else (lambda g: g)


def width(x):
    if isinstance(x, ArrayN):
        return width(x.c[0])
    v = _v(x)
    return int(np.size(v)) if isinstance(v, np.ndarray) else 1


def arange(T, n):
    return T(np.arange(n))


def gather(T, data, idx):
    if isinstance(T, type) and issubclass(T, ArrayN):
        if isinstance(data, ArrayN):  # SoA source: one gather per component
            return T(*[gather(T.ELEM, c, idx) for c in data.c])
        # flat source: element k of item i sits at N * i + k
        i = np.asarray(_v(idx))
        flat = np.asarray(data.v)
        return T(*[T.ELEM(flat[T.N * i + k]) for k in range(T.N)])
    return T(np.asarray(data.v)[np.asarray(_v(idx))])


class _Local:
    def __init__(self, n):
        self.items = [None] * n

    def __getitem__(self, i): return self.items[int(i)]
    def __setitem__(self, i, v): self.items[int(i)] = v


def alloc_local(T, n):
    return _Local(n)


def zeros(T, shape=None):
    if T in (Int, UInt):
        return Int(0)
    if T is Float:
        return Float(0.0)
    if T is Bool:
        return Bool(False)
    if isinstance(T, type) and issubclass(T, ArrayN):
        return T()
    if dataclasses.is_dataclass(T):
        return T(**{f.name: zeros(f.type) for f in dataclasses.fields(T)})
    raise TypeError(f"zeros({T})")


def _f(x):
    return x if isinstance(x, Float) else Float(x)


def _map(f, *xs):
    for x in xs:
        if isinstance(x, ArrayN):
            n = x.N
            T = type(x)
            return T(*[f(*[(y.c[k] if isinstance(y, ArrayN) else y) for y in xs]) for k in range(n)])
    return f(*xs)


def maximum(a, b): return _map(lambda x, y: Float(np.fmax(_f(x).v, _f(y).v)), a, b)
def minimum(a, b): return _map(lambda x, y: Float(np.fmin(_f(x).v, _f(y).v)), a, b)
def abs(a): return _map(lambda x: Float(np.abs(_f(x).v)), a)  # noqa: A001
def sqrt(a): return _map(lambda x: Float(np.sqrt(_f(x).v)), a)
def clamp(x, lo, hi): return _map(lambda a, l, h: Float(np.fmax(np.fmin(_f(a).v, F32(_v(h))), F32(_v(l)))), x, lo, hi)
clip = clamp
def copysign(a, b): return Float(np.copysign(F32(_v(a)), _f(b).v))
def acos(x): return _fm(0, _f(x).v)
def asin(x): return _fm(1, _f(x).v)
def atan2(y, x): return _fm(2, _f(y).v, _f(x).v)
def epsilon(T): return F32(2.0 ** -24)


def select(c, a, b):
    return a if bool(c) else b


def max(v):  # noqa: A001 - horizontal maximum
    r = _f(v.c[0]).v
    for x in v.c[1:]:
        r = np.fmax(r, _f(x).v)
    return Float(r)


def min(v):  # noqa: A001
    r = _f(v.c[0]).v
    for x in v.c[1:]:
        r = np.fmin(r, _f(x).v)
    return Float(r)


def dot(a, b):
    r = F32(_f(a.c[0]).v * _f(b.c[0]).v)
    for x, y in zip(a.c[1:], b.c[1:]):
        r = fma(_f(x).v, _f(y).v, r)
    return Float(r)


def squared_norm(a): return dot(a, a)
def norm(a): return Float(np.sqrt(dot(a, a).v))


def normalize(a):
    inv = F32(1.0) / np.sqrt(dot(a, a).v)
    return type(a)(*[Float(x.v * inv) for x in a.c])


def lerp(a, b, t):
    return _map(lambda x, y, s: Float(fma(_f(y).v, _f(s).v, fma(-_f(x).v, _f(s).v, _f(x).v))), a, b, t)


def cross(a, b):
    ax, ay, az = (x.v for x in a.c)
    bx, by, bz = (x.v for x in b.c)
    return Array3(Float(fma(ay, bz, -(az * by))), Float(fma(az, bx, -(ax * bz))), Float(fma(ax, by, -(ay * bx))))


# ---------------------------------------------------------------------------
# module registration: drjit, drjit.auto, drjit.auto.ad
# ---------------------------------------------------------------------------


def install():
    dr = types.ModuleType("drjit")
    this = sys.modules[__name__]
    for name in ("syntax", "width", "arange", "gather", "alloc_local", "zeros", "maximum", "minimum", "abs",
                 "sqrt", "clamp", "clip", "copysign", "acos", "asin", "atan2", "epsilon", "select", "max", "min",
                 "dot", "squared_norm", "norm", "normalize", "lerp", "cross", "inf", "pi"):
        setattr(dr, name, getattr(this, name))
    ad = types.ModuleType("drjit.auto.ad")
    for name, val in dict(Float32=Float, Int32=Int, UInt32=UInt, Bool=Bool, Array2f=Array2, Array3f=Array3,
                          Array4f=Array4, Array2i=Array2i, Array3i=Array3i, Array4i=Array4i, TensorXf=_Unused,
                          TensorXi=_Unused, PCG32=_Unused, Quaternion4f=_Unused, Matrix2f=_Unused,
                          Matrix3f=_Unused).items():
        setattr(ad, name, val)
    auto = types.ModuleType("drjit.auto")
    auto.ad = ad
    dr.auto = auto
    sys.modules["drjit"] = dr
    sys.modules["drjit.auto"] = auto
    sys.modules["drjit.auto.ad"] = ad
    return dr
