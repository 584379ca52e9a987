"""A serial CPU stand-in for the part of NVIDIA Warp that FlatWorld's explicit
FEM step uses -- test infrastructure only.

It exists so that the reference's OWN Python source (its ``@wp.kernel`` /
``@wp.func`` definitions and the host classes that launch them) can be run in
a container where ``warp-lang`` is not installed, to produce golden fixtures.
Nothing in the product imports it; ``make_golden.py`` installs it as
``sys.modules["warp"]`` before importing the reference package.

Semantics, restated from Warp's public documentation (warp-lang 1.x, the
"Language reference" and "Built-ins" pages) -- every choice below is the
reading of Warp's CPU device that the fixtures then encode:

* A launch runs its threads one after another in ascending ``wp.tid()``
  order, each thread to completion, so ``atomic_add`` updates land in thread
  order, then program order (Warp's CPU backend runs a launch as a serial loop).
* ``float`` values are IEEE binary32; every + - * / and sqrt is rounded once
  (numpy float32 scalars; no fused multiply-add).  Python float literals and
  ``float(x)`` inside kernels become float32, ``int(x)`` truncates toward zero.
  Scalar kernel arguments are converted to their annotated type at launch (a
  Python float passed for ``dt: float`` is rounded to float32).
* ``wp.log``, ``sin``, ``cos``, ``atan2`` and ``pow`` call the C library's
  float functions (``logf`` ...), as Warp's CPU kernels do.
  ``floor``/``ceil`` are exact; ``round`` rounds half away from zero (C ``roundf``).
* vectors and matrices hold float32 (or int32) components; ``@`` and ``dot``
  sum products in ascending index order; ``inverse`` of a 2x2 is the adjugate
  times ``1/det`` when det is non-zero, else the zero matrix; ``normalize``
  divides by the length when it is positive, else gives zero;
  ``length`` is ``sqrt(dot(v, v))``.
* ``min``/``max`` pick ``a if a < b else b`` (resp. ``>``), component-wise for
  vectors; ``clamp(x, a, b)`` is ``min(max(x, a), b)``.
* Arrays are numpy-backed; ``.numpy()`` returns a copy (as for device arrays),
  ``.assign`` copies in.

Warp's generated code is never read: this module is written from the
documented behaviour above.
"""

from __future__ import annotations

import builtins
import copy as _copy
import ctypes
import itertools
import math
import types as _pytypes

import numpy as np

np.seterr(all="ignore")

_libm = ctypes.CDLL("libm.so.6")


def _cfun(name, nargs):
    f = getattr(_libm, name)
    f.restype = ctypes.c_float
    f.argtypes = [ctypes.c_float] * nargs
    return f


_logf = _cfun("logf", 1)
_sinf = _cfun("sinf", 1)
_cosf = _cfun("cosf", 1)
_atan2f = _cfun("atan2f", 2)
_powf = _cfun("powf", 2)
_expf = _cfun("expf", 1)
_F32 = np.float32

# ---------------------------------------------------------------------------
# scalar types
# ---------------------------------------------------------------------------


class _Scalar:
    def __init__(self, name, npt, is_float):
        self.__name__ = name
        self.np = np.dtype(npt)
        self.is_float = is_float
        self._t = npt

    def __call__(self, x=0):
        if self.is_float:
            return self._t(x)
        if self.np.kind == "u":
            return self._t(int(x) & ((1 << (8 * self.np.itemsize)) - 1))
        return self._t(int(x))

    def __repr__(self):
        return f"wp.{self.__name__}"


float32 = _Scalar("float32", np.float32, True)
float64 = _Scalar("float64", np.float64, True)
float16 = _Scalar("float16", np.float16, True)
int32 = _Scalar("int32", np.int32, False)
int64 = _Scalar("int64", np.int64, False)
int16 = _Scalar("int16", np.int16, False)
int8 = _Scalar("int8", np.int8, False)
uint32 = _Scalar("uint32", np.uint32, False)
uint64 = _Scalar("uint64", np.uint64, False)
uint16 = _Scalar("uint16", np.uint16, False)
uint8 = _Scalar("uint8", np.uint8, False)
bool_ = _Scalar("bool", np.bool_, False)


def _scalar_of(t):
    """Map a dtype spec (Python float/int, a _Scalar) to a _Scalar."""
    g = globals()
    if t is None or t is builtins.float or t is g.get("_kfloat"):  # inside kernels `float` is _kfloat
        return float32
    if t is builtins.int or t is g.get("_kint"):
        return int32
    if t is builtins.bool:
        return bool_
    if isinstance(t, _Scalar):
        return t
    return None


def _f32(x=0.0):
    return _F32(x)


def _conv(s, x):
    """Convert x to scalar type s."""
    return s(x)


# ---------------------------------------------------------------------------
# vectors
# ---------------------------------------------------------------------------


class _VecType:
    def __init__(self, length, dtype, name):
        self.length = length
        self.scalar = _scalar_of(dtype)
        self.__name__ = name
        self._shape = (length,)

    def __call__(self, *args):
        s = self.scalar
        n = self.length
        if len(args) == 0:
            return Vec(self, [s(0)] * n)
        if len(args) == 1:
            a = args[0]
            if isinstance(a, (Vec, list, tuple, np.ndarray)):
                return Vec(self, [s(c) for c in a])
            return Vec(self, [s(a)] * n)
        if len(args) != n:
            raise TypeError(f"{self.__name__} takes {n} components, got {len(args)}")
        return Vec(self, [s(c) for c in args])

    def __repr__(self):
        return f"wp.{self.__name__}"


def _is_scalar(x):
    return not isinstance(x, (Vec, Mat))


class Vec:
    __slots__ = ("t", "c")
    __array_ufunc__ = None  # numpy scalars defer to our operators

    def __init__(self, t, comps):
        self.t = t
        self.c = comps

    # element access
    def __getitem__(self, i):
        return self.c[i]

    def __setitem__(self, i, v):
        self.c[i] = self.t.scalar(v)

    def __len__(self):
        return len(self.c)

    def __iter__(self):
        return iter(self.c)

    @property
    def x(self):
        return self.c[0]

    @property
    def y(self):
        return self.c[1]

    @property
    def z(self):
        return self.c[2]

    @property
    def w(self):
        return self.c[3]

    def _s(self, v):
        return self.t.scalar(v)

    def __add__(self, o):
        return Vec(self.t, [a + b for a, b in zip(self.c, o.c)])

    def __sub__(self, o):
        return Vec(self.t, [a - b for a, b in zip(self.c, o.c)])

    def __neg__(self):
        return Vec(self.t, [-a for a in self.c])

    def __pos__(self):
        return self

    def __mul__(self, o):
        if isinstance(o, Vec):
            raise TypeError("vector * vector is not defined (use wp.cw_mul or wp.dot)")
        if isinstance(o, Mat):
            return _vec_mat(self, o)
        s = self._s(o)
        return Vec(self.t, [a * s for a in self.c])

    def __rmul__(self, o):
        s = self._s(o)
        return Vec(self.t, [s * a for a in self.c])

    def __truediv__(self, o):
        s = self._s(o)
        return Vec(self.t, [a / s for a in self.c])

    def __matmul__(self, o):
        return _vec_mat(self, o)

    def __eq__(self, o):
        return isinstance(o, Vec) and all(a == b for a, b in zip(self.c, o.c))

    def __ne__(self, o):
        return not self.__eq__(o)

    __hash__ = None

    def __repr__(self):
        return f"{self.t.__name__}({', '.join(repr(float(a)) for a in self.c)})"


def _vec_mat(v, m):
    # row vector times matrix: r[j] = sum_k v[k] m[k][j], ascending k
    out = []
    for j in range(m.t.cols):
        acc = v.c[0] * m.r[0][j]
        for k in range(1, m.t.rows):
            acc = acc + v.c[k] * m.r[k][j]
        out.append(acc)
    return Vec(_vec_type(m.t.cols, m.t.scalar), out)


_VEC_CACHE = {}


def _vec_type(n, scalar):
    key = (n, scalar.__name__)
    t = _VEC_CACHE.get(key)
    if t is None:
        t = _VecType(n, scalar, f"vec{n}{'' if scalar is float32 else scalar.__name__[0]}")
        _VEC_CACHE[key] = t
    return t


# ---------------------------------------------------------------------------
# matrices
# ---------------------------------------------------------------------------


class _MatType:
    def __init__(self, rows, cols, dtype, name):
        self.rows = rows
        self.cols = cols
        self.scalar = _scalar_of(dtype)
        self.__name__ = name
        self._shape = (rows, cols)

    def __call__(self, *args):
        s = self.scalar
        R, C = self.rows, self.cols
        if len(args) == 0:
            return Mat(self, [[s(0)] * C for _ in range(R)])
        if len(args) == 1:
            a = args[0]
            if isinstance(a, Mat):
                return Mat(self, [[s(x) for x in row] for row in a.r])
            if isinstance(a, np.ndarray) and a.ndim == 2:
                return Mat(self, [[s(a[i, j]) for j in range(C)] for i in range(R)])
            return Mat(self, [[s(a)] * C for _ in range(R)])
        if len(args) == R * C:
            return Mat(self, [[s(args[i * C + j]) for j in range(C)] for i in range(R)])
        if len(args) == R and all(isinstance(a, Vec) for a in args):
            # vectors given to a matrix constructor are its rows
            return Mat(self, [[s(x) for x in a.c] for a in args])
        raise TypeError(f"{self.__name__}: cannot build from {len(args)} arguments")

    def __repr__(self):
        return f"wp.{self.__name__}"


_MAT_CACHE = {}


def _mat_type(rows, cols, scalar):
    key = (rows, cols, scalar.__name__)
    t = _MAT_CACHE.get(key)
    if t is None:
        t = _MatType(rows, cols, scalar, f"mat{rows}{cols}")
        _MAT_CACHE[key] = t
    return t


class Mat:
    __slots__ = ("t", "r")
    __array_ufunc__ = None

    def __init__(self, t, rows):
        self.t = t
        self.r = rows

    def __getitem__(self, idx):
        if isinstance(idx, tuple):
            i, j = idx
            return self.r[i][j]
        return Vec(_vec_type(self.t.cols, self.t.scalar), list(self.r[idx]))

    def __setitem__(self, idx, v):
        s = self.t.scalar
        if isinstance(idx, tuple):
            i, j = idx
            self.r[i][j] = s(v)
        else:
            self.r[idx] = [s(x) for x in v.c]

    def _s(self, v):
        return self.t.scalar(v)

    def __add__(self, o):
        return Mat(self.t, [[a + b for a, b in zip(ra, rb)] for ra, rb in zip(self.r, o.r)])

    def __sub__(self, o):
        return Mat(self.t, [[a - b for a, b in zip(ra, rb)] for ra, rb in zip(self.r, o.r)])

    def __neg__(self):
        return Mat(self.t, [[-a for a in ra] for ra in self.r])

    def __mul__(self, o):
        if isinstance(o, Mat):
            return _mat_mat(self, o)
        if isinstance(o, Vec):
            return _mat_vec(self, o)
        s = self._s(o)
        return Mat(self.t, [[a * s for a in ra] for ra in self.r])

    def __rmul__(self, o):
        s = self._s(o)
        return Mat(self.t, [[s * a for a in ra] for ra in self.r])

    def __truediv__(self, o):
        s = self._s(o)
        return Mat(self.t, [[a / s for a in ra] for ra in self.r])

    def __matmul__(self, o):
        if isinstance(o, Mat):
            return _mat_mat(self, o)
        return _mat_vec(self, o)

    def __repr__(self):
        return f"{self.t.__name__}({[[float(a) for a in row] for row in self.r]})"


def _mat_mat(a, b):
    R, K, C = a.t.rows, a.t.cols, b.t.cols
    out = []
    for i in range(R):
        row = []
        ai = a.r[i]
        for j in range(C):
            acc = ai[0] * b.r[0][j]
            for k in range(1, K):
                acc = acc + ai[k] * b.r[k][j]
            row.append(acc)
        out.append(row)
    return Mat(_mat_type(R, C, a.t.scalar), out)


def _mat_vec(a, v):
    out = []
    for row in a.r:
        acc = row[0] * v.c[0]
        for k in range(1, len(row)):
            acc = acc + row[k] * v.c[k]
        out.append(acc)
    return Vec(_vec_type(a.t.rows, a.t.scalar), out)


# ---------------------------------------------------------------------------
# named types
# ---------------------------------------------------------------------------

vec2 = _vec_type(2, float32)
vec3 = _vec_type(3, float32)
vec4 = _vec_type(4, float32)
vec2f, vec3f, vec4f = vec2, vec3, vec4
vec2i = _vec_type(2, int32)
vec3i = _vec_type(3, int32)
vec4i = _vec_type(4, int32)
vec2d = _vec_type(2, float64)
vec3d = _vec_type(3, float64)
vec2ui = _vec_type(2, uint32)
for _r in (2, 3, 4, 6):
    for _c in (2, 3, 4, 6, 8, 12):
        globals()[f"mat{_r}{_c}"] = _mat_type(_r, _c, float32)
mat22f, mat33f, mat44f = mat22, mat33, mat44  # noqa: F821


class _TypesNS:
    float32 = float32
    float64 = float64
    int32 = int32
    uint32 = uint32
    int64 = int64
    uint8 = uint8
    int8 = int8
    vec2 = vec2
    vec3 = vec3

    @staticmethod
    def vector(length, dtype=float32):
        return _vec_type(length, _scalar_of(dtype))

    @staticmethod
    def matrix(shape, dtype=float32):
        return _mat_type(shape[0], shape[1], _scalar_of(dtype))


types = _TypesNS()


def vector(*args, length=None, dtype=float32):
    if length is None:
        return _vec_type(len(args), _scalar_of(dtype))(*args)
    return _vec_type(length, _scalar_of(dtype))(*args)


def matrix(*args, shape=None, dtype=float32):
    return _mat_type(shape[0], shape[1], _scalar_of(dtype))(*args)


# ---------------------------------------------------------------------------
# structs
# ---------------------------------------------------------------------------


def _zero_of(t):
    if isinstance(t, (_VecType, _MatType)):
        return t()
    s = _scalar_of(t)
    if s is not None:
        return s(0)
    if isinstance(t, type) and getattr(t, "_is_wp_struct", False):
        return t()
    return None


def struct(cls):
    fields = dict(getattr(cls, "__annotations__", {}))

    class S:
        _is_wp_struct = True
        _fields = fields

        def __init__(self):
            mod_globals = vars(__import__(cls.__module__)) if cls.__module__ in _sys_modules() else {}
            for k, t in fields.items():
                if isinstance(t, str):
                    try:
                        t = eval(t, dict(mod_globals), {"wp": _this_module()})
                    except Exception:
                        t = None
                setattr(self, k, _zero_of(t))

        def __repr__(self):
            return f"{cls.__name__}({', '.join(f'{k}={getattr(self, k)!r}' for k in fields)})"

    S.__name__ = cls.__name__
    S.__qualname__ = cls.__qualname__
    return S


def _sys_modules():
    import sys

    return sys.modules


def _this_module():
    import sys

    return sys.modules[__name__]


# ---------------------------------------------------------------------------
# arrays
# ---------------------------------------------------------------------------


def _dtype_info(dtype):
    """(inner shape, numpy dtype, kind) for an element type."""
    if isinstance(dtype, _VecType):
        return (dtype.length,), dtype.scalar.np, "vec"
    if isinstance(dtype, _MatType):
        return (dtype.rows, dtype.cols), dtype.scalar.np, "mat"
    s = _scalar_of(dtype)
    if s is not None:
        return (), s.np, "scalar"
    if isinstance(dtype, type) and getattr(dtype, "_is_wp_struct", False):
        return (), np.dtype(object), "struct"
    if isinstance(dtype, np.dtype) or (isinstance(dtype, type) and issubclass(dtype, np.generic)):
        return (), np.dtype(dtype), "scalar"
    raise TypeError(f"unsupported array dtype {dtype!r}")


class array:
    """numpy-backed array; kernel-side indexing returns Warp-style values."""

    def __init__(self, data=None, dtype=None, shape=None, device=None, ndim=None, copy=True,
                 requires_grad=False, _view=None, **_kw):
        if dtype is None:
            if isinstance(data, array):
                dtype = data.dtype
            elif data is not None and np.asarray(data).dtype.kind == "f":
                dtype = float32
            elif data is not None:
                dtype = int32
            else:
                dtype = float32
        self.dtype = dtype
        self.device = "cpu"
        self.requires_grad = requires_grad
        self.grad = None
        inner, npdt, kind = _dtype_info(dtype)
        self._inner = inner
        self._kind = kind
        self._vt = dtype if kind in ("vec", "mat") else None
        self._sc = dtype.scalar if kind in ("vec", "mat") else _scalar_of(dtype)
        if _view is not None:
            self.data = _view
        elif data is None:
            if shape is None:
                shape = (0,) * (ndim or 1)
            if isinstance(shape, int):
                shape = (shape,)
            full = tuple(shape) + inner
            if kind == "struct":
                self.data = np.empty(full, dtype=object)
                for idx in np.ndindex(*full):
                    self.data[idx] = dtype()
            else:
                self.data = np.zeros(full, dtype=npdt)
        else:
            if isinstance(data, array):
                src = data.data
            elif kind == "vec" and isinstance(data, (list, tuple)) and data and isinstance(data[0], Vec):
                src = np.array([v.c for v in data], dtype=npdt)
            else:
                src = data
            if kind == "struct":
                self.data = np.empty(len(src), dtype=object)
                for i, s in enumerate(src):
                    self.data[i] = s
            else:
                arr = np.array(src, dtype=npdt, copy=True)
                if shape is not None:
                    sh = (shape,) if isinstance(shape, int) else tuple(shape)
                    arr = arr.reshape(sh + inner)
                elif inner and arr.shape[-len(inner):] != inner:
                    arr = arr.reshape((-1,) + inner)
                self.data = arr
        self.shape = tuple(self.data.shape[: self.data.ndim - len(inner)])
        self.ndim = len(self.shape)
        self.size = int(np.prod(self.shape)) if self.shape else 1

    # host API
    def numpy(self):
        return self.data.copy()

    def list(self):
        return [self._get(i) for i in range(self.shape[0])]

    def assign(self, src):
        s = src.data if isinstance(src, array) else np.asarray(src)
        if self._kind == "struct":
            self.data[...] = s
        else:
            self.data[...] = np.asarray(s, dtype=self.data.dtype).reshape(self.data.shape)

    def fill_(self, value):
        if isinstance(value, Vec):
            self.data[...] = np.asarray(value.c, dtype=self.data.dtype)
        elif isinstance(value, Mat):
            self.data[...] = np.asarray(value.r, dtype=self.data.dtype)
        else:
            self.data[...] = value

    def zero_(self):
        if self._kind == "struct":
            for idx in np.ndindex(*self.shape):
                self.data[idx] = self.dtype()
        else:
            self.data[...] = 0

    def to(self, device):
        return self

    def contiguous(self):
        return self

    def flatten(self):
        return array(dtype=self.dtype, _view=self.data.reshape((-1,) + self._inner))

    def reshape(self, shape):
        if isinstance(shape, int):
            shape = (shape,)
        return array(dtype=self.dtype, _view=self.data.reshape(tuple(shape) + self._inner))

    @property
    def ptr(self):
        return self.data.ctypes.data if self._kind != "struct" else id(self.data)

    def __len__(self):
        return self.shape[0]

    def __array__(self, dtype=None, copy=None):
        return self.data if dtype is None else self.data.astype(dtype)

    # element access (kernel side); a slice gives a view array (host side)
    def _get(self, idx):
        k = self._kind
        if k == "scalar":
            return self.data[idx]
        if k == "vec":
            return Vec(self._vt, list(self.data[idx]))
        if k == "mat":
            m = self.data[idx]
            return Mat(self._vt, [list(row) for row in m])
        return _copy.deepcopy(self.data[idx])

    def __getitem__(self, idx):
        if isinstance(idx, slice) or (isinstance(idx, tuple) and any(isinstance(i, slice) for i in idx)):
            return array(dtype=self.dtype, _view=self.data[idx])
        if isinstance(idx, tuple) and len(idx) < self.ndim:
            return array(dtype=self.dtype, _view=self.data[idx])
        return self._get(idx)

    def __setitem__(self, idx, v):
        k = self._kind
        if k == "scalar":
            self.data[idx] = v
        elif k == "vec":
            self.data[idx] = v.c if isinstance(v, Vec) else v
        elif k == "mat":
            self.data[idx] = v.r if isinstance(v, Mat) else v
        else:
            self.data[idx] = _copy.deepcopy(v)

    def __repr__(self):
        return f"wp.array(shape={self.shape}, dtype={self.dtype!r})"


def _mk(shape, dtype, fill=None):
    if isinstance(shape, int):
        shape = (shape,)
    a = array(dtype=dtype if dtype is not None else float32, shape=shape)
    if fill is not None:
        a.fill_(fill)
    return a


def zeros(shape=0, dtype=float, device=None, requires_grad=False, **_kw):
    return _mk(shape, dtype)


def empty(shape=0, dtype=float, device=None, requires_grad=False, **_kw):
    return _mk(shape, dtype)


def ones(shape=0, dtype=float, device=None, requires_grad=False, **_kw):
    return _mk(shape, dtype, 1)


def full(shape=0, value=0, dtype=float, device=None, requires_grad=False, **_kw):
    return _mk(shape, dtype, value)


def zeros_like(a, **_kw):
    return _mk(a.shape, a.dtype)


def empty_like(a, **_kw):
    return _mk(a.shape, a.dtype)


def full_like(a, value, **_kw):
    return _mk(a.shape, a.dtype, value)


def clone(a, **_kw):
    return array(a.data.copy(), dtype=a.dtype, shape=a.shape)


def from_numpy(arr, dtype=None, shape=None, device=None, **_kw):
    return array(arr, dtype=dtype, shape=shape)


def copy(dest, src, dest_offset=0, src_offset=0, count=0, **_kw):
    d = dest.data.reshape((-1,) + dest._inner)
    s = src.data.reshape((-1,) + src._inner)
    n = count if count else min(len(d) - dest_offset, len(s) - src_offset)
    d[dest_offset : dest_offset + n] = s[src_offset : src_offset + n]


# ---------------------------------------------------------------------------
# builtins used inside kernels
# ---------------------------------------------------------------------------

_TID = [0]


def tid():
    return _TID[0]


def _s1(x):
    return x if isinstance(x, (np.floating, np.integer)) else (_F32(x) if isinstance(x, float) else x)


def abs(x):  # noqa: A001
    if isinstance(x, Vec):
        return Vec(x.t, [builtins.abs(a) for a in x.c])
    return builtins.abs(_s1(x))


def min(a, b):  # noqa: A001
    if isinstance(a, Vec):
        return Vec(a.t, [p if p < q else q for p, q in zip(a.c, b.c)])
    a, b = _s1(a), _s1(b)
    return a if a < b else b


def max(a, b):  # noqa: A001
    if isinstance(a, Vec):
        return Vec(a.t, [p if p > q else q for p, q in zip(a.c, b.c)])
    a, b = _s1(a), _s1(b)
    return a if a > b else b


def clamp(x, a, b):
    return min(max(x, a), b)


def sqrt(x):
    return np.sqrt(_F32(x))


def log(x):
    return _F32(_logf(_F32(x)))


def exp(x):
    return _F32(_expf(_F32(x)))


def sin(x):
    return _F32(_sinf(_F32(x)))


def cos(x):
    return _F32(_cosf(_F32(x)))


def atan2(y, x):
    return _F32(_atan2f(_F32(y), _F32(x)))


def pow(x, y):  # noqa: A001
    return _F32(_powf(_F32(x), _F32(y)))


def floor(x):
    return _F32(math.floor(_F32(x))) if np.isfinite(_F32(x)) else _F32(x)


def ceil(x):
    return _F32(math.ceil(_F32(x))) if np.isfinite(_F32(x)) else _F32(x)


def round(x):  # noqa: A001
    x = _F32(x)
    if not np.isfinite(x):
        return x
    r = math.floor(builtins.abs(float(x)) + 0.5)  # exact in double for any float32
    return _F32(math.copysign(r, float(x)))


def dot(a, b):
    acc = a.c[0] * b.c[0]
    for k in range(1, len(a.c)):
        acc = acc + a.c[k] * b.c[k]
    return acc


def length(v):
    return np.sqrt(dot(v, v))


def length_sq(v):
    return dot(v, v)


def normalize(v):
    n = length(v)
    if n > 0:
        return v / n
    return Vec(v.t, [v.t.scalar(0)] * len(v.c))


def cross(a, b):
    if len(a.c) == 3:
        return Vec(a.t, [a.c[1] * b.c[2] - a.c[2] * b.c[1],
                         a.c[2] * b.c[0] - a.c[0] * b.c[2],
                         a.c[0] * b.c[1] - a.c[1] * b.c[0]])
    raise TypeError("wp.cross is defined for vec3")


def transpose(m):
    t = _mat_type(m.t.cols, m.t.rows, m.t.scalar)
    return Mat(t, [[m.r[i][j] for i in range(m.t.rows)] for j in range(m.t.cols)])


def determinant(m):
    r = m.r
    if m.t.rows == 2:
        return r[0][0] * r[1][1] - r[0][1] * r[1][0]
    if m.t.rows == 3:
        return (r[0][0] * (r[1][1] * r[2][2] - r[2][1] * r[1][2])
                - r[0][1] * (r[1][0] * r[2][2] - r[2][0] * r[1][2])
                + r[0][2] * (r[1][0] * r[2][1] - r[2][0] * r[1][1]))
    raise TypeError("determinant: 2x2 or 3x3 only")


def inverse(m):
    r = m.r
    if m.t.rows == 2:
        det = r[0][0] * r[1][1] - r[0][1] * r[1][0]
        if det != 0:
            inv = _F32(1.0) / det
            return Mat(m.t, [[r[1][1] * inv, -r[0][1] * inv], [-r[1][0] * inv, r[0][0] * inv]])
        return m.t()
    raise TypeError("inverse: only the 2x2 form is on the FEM step")


def trace(m):
    acc = m.r[0][0]
    for i in range(1, m.t.rows):
        acc = acc + m.r[i][i]
    return acc


def identity(n=2, dtype=float32):
    t = _mat_type(n, n, _scalar_of(dtype))
    s = t.scalar
    return Mat(t, [[s(1) if i == j else s(0) for j in range(n)] for i in range(n)])


def select(cond, a, b):
    return b if cond else a


def where(cond, a, b):
    return a if cond else b


def _atomic(arr, args, op):
    *idx, val = args
    idx = idx[0] if len(idx) == 1 else tuple(idx)
    old = arr._get(idx)
    arr[idx] = op(old, val)
    return old


def atomic_add(arr, *args):
    return _atomic(arr, args, lambda o, v: o + v)


def atomic_sub(arr, *args):
    return _atomic(arr, args, lambda o, v: o - v)


def atomic_min(arr, *args):
    return _atomic(arr, args, min)


def atomic_max(arr, *args):
    return _atomic(arr, args, max)


def printf(fmt, *args):
    pass


# ---------------------------------------------------------------------------
# kernels, functions, launches
# ---------------------------------------------------------------------------


def _kfloat(x=0.0):
    return _F32(x)


def _kint(x=0):
    return builtins.int(x)


class _KernelGlobals(dict):
    """Globals of a kernel/function: the defining module's names, with the
    kernel-language meaning of float(), int(), min(), max() and abs()."""

    def __init__(self, module_dict):
        super().__init__(float=_kfloat, int=_kint, min=min, max=max, abs=abs, round=round)
        self._mod = module_dict

    def __missing__(self, key):
        try:
            return self._mod[key]
        except KeyError:
            return getattr(builtins, key)


_GLOBALS_CACHE = {}


def _rebind(fn):
    g = _GLOBALS_CACHE.get(id(fn.__globals__))
    if g is None:
        g = _KernelGlobals(fn.__globals__)
        _GLOBALS_CACHE[id(fn.__globals__)] = g
    f = _pytypes.FunctionType(fn.__code__, g, fn.__name__, fn.__defaults__, fn.__closure__)
    f.__annotations__ = fn.__annotations__
    f.__doc__ = fn.__doc__
    f.__wrapped__ = fn
    return f


def func(fn=None, **_kw):
    if fn is None:
        return lambda f: _rebind(f)
    return _rebind(fn)


def function(fn=None, **_kw):
    return func(fn)


class Kernel:
    def __init__(self, fn):
        self.fn = _rebind(fn)
        self.key = fn.__name__
        self.__name__ = fn.__name__
        self._conv = None

    def _converters(self):
        if self._conv is None:
            conv = []
            ann = self.fn.__annotations__
            glb = self.fn.__globals__
            for name in self.fn.__code__.co_varnames[: self.fn.__code__.co_argcount]:
                a = ann.get(name)
                t = None
                if isinstance(a, str):
                    try:
                        t = eval(a, {}, _AnnNS(glb))
                    except Exception:
                        t = None
                else:
                    t = a
                if isinstance(t, (_VecType, _MatType)):
                    conv.append(lambda v, t=t: v if isinstance(v, (Vec, Mat)) and v.t is t else t(*np.asarray(v).reshape(-1)) if not isinstance(v, (Vec, Mat)) else t(v))
                elif _scalar_of(t) is not None and not isinstance(t, array):
                    s = _scalar_of(t)
                    if s.is_float:
                        conv.append(lambda v, s=s: s(v))
                    else:
                        conv.append(lambda v: builtins.int(v))
                else:
                    conv.append(None)
            self._conv = conv
        return self._conv

    def __call__(self, *args):
        return self.fn(*args)


class _AnnNS(dict):
    def __init__(self, glb):
        super().__init__()
        self._g = glb

    def __missing__(self, key):
        if key == "float":
            return builtins.float
        if key == "int":
            return builtins.int
        try:
            return self._g[key]
        except KeyError:
            return getattr(builtins, key)


def kernel(fn=None, **_kw):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


LAUNCH_COUNT = [0]


def launch(kernel, dim, inputs=(), outputs=(), device=None, stream=None, adj_inputs=None,
           adj_outputs=None, adjoint=False, record_tape=True, record_cmd=False, max_blocks=0,
           block_dim=256, **_kw):
    args = list(inputs) + list(outputs)
    conv = kernel._converters()
    if len(conv) != len(args):
        raise TypeError(f"{kernel.key}: expected {len(conv)} arguments, got {len(args)}")
    args = [c(a) if c is not None else a for c, a in zip(conv, args)]
    fn = kernel.fn
    LAUNCH_COUNT[0] += 1
    if isinstance(dim, (tuple, list)):
        dims = [builtins.int(d) for d in dim]
        for t in itertools.product(*[range(d) for d in dims]):
            _TID[0] = t
            fn(*args)
    else:
        for t in range(builtins.int(dim)):
            _TID[0] = t
            fn(*args)


# ---------------------------------------------------------------------------
# runtime odds and ends
# ---------------------------------------------------------------------------


def constant(x):
    return x


def init():
    pass


def set_device(device=None):
    pass


def get_device(device=None):
    return "cpu"


def get_preferred_device():
    return "cpu"


def is_cuda_available():
    return False


def synchronize(*_a, **_k):
    pass


def synchronize_device(*_a, **_k):
    pass


class ScopedDevice:
    def __init__(self, *_a, **_k):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


ScopedTimer = ScopedDevice


class _Config:
    mode = "release"
    verify_fp = False
    verbose = False
    quiet = True


config = _Config()
Any = object
