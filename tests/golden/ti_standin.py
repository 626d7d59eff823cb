"""A small NumPy stand-in for the subset of the Taichi API that the reference's
``src/`` modules use, so that those modules can be executed unmodified on the
CPU to generate golden vectors.  Test infrastructure only.

Kernels run as plain Python loops (serial, so ``ti.atomic_add`` is an in-place
add); fields are NumPy arrays; ``ti.Vector``/``ti.Matrix`` values are NumPy
arrays of the default float type.  Float arithmetic stays in that type (float32
unless ``force_f64()`` was called before the reference is imported), which
mirrors Taichi's ``default_fp``.  Integer casts (``ti.cast(x, ti.i32)``)
truncate toward zero and return int16 so that mixing them with float32 values
stays float32, as Taichi's i32 -> f32 promotion does.

The 2x2 ``ti.svd`` follows Taichi's published ``svd2d`` algorithm (rotation
polar factor, one Jacobi rotation of the symmetric remainder, descending sort);
Taichi itself is a third-party dependency that the reference does not vendor
and whose version it does not pin.
"""
from __future__ import annotations

import itertools
import types

import numpy as np

f32 = np.float32
f64 = np.float64
i32 = np.int32
cuda = "cuda"
cpu = "cpu"
ijk = "ijk"
ij = "ij"
k = "k"
l = "l"  # noqa: E741

_REAL = [np.float32]


def force_f64():
    """Make ``ti.f32`` mean float64 (call before importing the reference)."""
    global f32
    f32 = np.float64
    _REAL[0] = np.float64


def init(arch=None, default_fp=None, **_kw):
    if default_fp is not None:
        _REAL[0] = default_fp


def reset():
    pass


# ---------------------------------------------------------------- values
class TiArr(np.ndarray):
    """Matrix/vector value with the Taichi methods the reference calls."""

    def _coerce(self, other):
        if isinstance(other, (list, tuple)):
            return np.asarray(other, dtype=self.dtype if self.dtype.kind == "f" else _REAL[0])
        return other

    def __add__(self, o):
        return np.ndarray.__add__(self, self._coerce(o))

    def __radd__(self, o):
        return np.ndarray.__radd__(self, self._coerce(o))

    def __sub__(self, o):
        return np.ndarray.__sub__(self, self._coerce(o))

    def __rsub__(self, o):
        return np.ndarray.__rsub__(self, self._coerce(o))

    def norm(self, eps=0):
        return np.sqrt(np.dot(self, self) + self.dtype.type(eps))

    def dot(self, o):
        return np.dot(np.asarray(self), np.asarray(o)).astype(self.dtype)[()]

    def outer_product(self, o):
        return np.outer(self, o).view(TiArr)

    def transpose(self):
        return np.ndarray.transpose(self).copy().view(TiArr)

    def inverse(self):
        return np.linalg.inv(np.asarray(self)).astype(self.dtype).view(TiArr)

    def determinant(self):
        return np.linalg.det(np.asarray(self)).astype(self.dtype)[()]


def _infer(vals):
    arr = np.asarray(vals)
    if arr.dtype.kind in "iub":
        return arr.astype(np.int32).view(TiArr)
    return arr.astype(_REAL[0]).view(TiArr)


def _vector_new(vals, dt=None):
    if dt is not None:
        return np.asarray(vals, dtype=dt).view(TiArr)
    return _infer([np.asarray(v)[()] for v in vals])


def _matrix_new(rows, dt=None):
    if dt is not None:
        return np.asarray(rows, dtype=dt).view(TiArr)
    return _infer([[np.asarray(v)[()] for v in r] for r in rows])


class _VectorNS:
    def __call__(self, vals, dt=None):
        return _vector_new(vals, dt)

    @staticmethod
    def zero(dt, n):
        return np.zeros(n, dtype=dt).view(TiArr)

    @staticmethod
    def field(n, dtype=None, shape=None):
        return Field(dtype or _REAL[0], (n,), shape)


class _MatrixNS:
    def __call__(self, rows, dt=None):
        return _matrix_new(rows, dt)

    @staticmethod
    def zero(dt, n, m):
        return np.zeros((n, m), dtype=dt).view(TiArr)

    @staticmethod
    def rows(vecs):
        return np.stack([np.asarray(v) for v in vecs], axis=0).view(TiArr)

    @staticmethod
    def cols(vecs):
        return np.stack([np.asarray(v) for v in vecs], axis=1).view(TiArr)

    @staticmethod
    def cross(a, b):
        return np.cross(a, b).view(TiArr)

    @staticmethod
    def field(n, m, dtype=None, shape=None):
        return Field(dtype or _REAL[0], (n, m), shape)


Vector = _VectorNS()
Matrix = _MatrixNS()


# ---------------------------------------------------------------- fields
class Field:
    def __init__(self, dtype, elem_shape=(), shape=None, is_grad=False):
        self.dtype = dtype
        self.elem_shape = tuple(elem_shape)
        self.arr = None
        self._grad = None
        self._is_grad = is_grad
        if shape is not None:
            self._allocate(shape if isinstance(shape, tuple) else (shape,))

    def _allocate(self, shape):
        self.shape = tuple(shape)
        self.arr = np.zeros(self.shape + self.elem_shape, dtype=self.dtype)

    @property
    def grad(self):
        if self._grad is None:
            self._grad = Field(self.dtype, self.elem_shape, self.shape, is_grad=True)
        return self._grad

    @staticmethod
    def _key(idx):
        if idx is None:
            return (Ellipsis,)
        if not isinstance(idx, tuple):
            idx = (idx,)
        flat = []
        for v in idx:
            a = np.asarray(v)
            if a.ndim == 0:
                flat.append(int(a))
            else:
                flat.extend(int(t) for t in a)
        return tuple(flat) + (Ellipsis,)

    def __getitem__(self, idx):
        view = self.arr[self._key(idx)]
        if idx is None and not view.ndim:
            # a 0-D field read as field[None] is a value, as Taichi returns a
            # Python number: a view would change when the field is written later
            return view[()]
        # element access stays a view: ti.atomic_add(field[i], v) adds through it
        return view.view(TiArr) if view.ndim else view

    def __setitem__(self, idx, value):
        self.arr[self._key(idx)] = np.asarray(value)

    def __iter__(self):
        return itertools.product(*[range(n) for n in self.shape])

    def from_numpy(self, a):
        a = np.asarray(a)
        if self.arr is None:
            self._allocate(a.shape[: a.ndim - len(self.elem_shape)])
        self.arr[...] = a.astype(self.dtype)

    def to_numpy(self):
        return self.arr.copy()


def field(dtype=None, shape=None):
    return Field(dtype or _REAL[0], (), shape)


class _SNode:
    def __init__(self, shape=()):
        self._shape = tuple(shape)

    def dense(self, axes, n):
        n_axes = len(axes) if axes in ("ijk", "ij") else 1
        return _SNode(self._shape + (n,) * n_axes)

    def place(self, *fields):
        for f in fields:
            f._allocate(self._shape)
        return self

    def lazy_grad(self):
        pass


root = _SNode()


# ---------------------------------------------------------------- language
def kernel(fn):
    return fn


def func(fn):
    return fn


def static(x):
    return x


def ndrange(*dims):
    return itertools.product(*[range(d) for d in dims])


def cast(x, dtype):
    a = np.asarray(x)
    if np.dtype(dtype).kind in "iu":
        out = (a if a.dtype.kind in "iu" else np.trunc(a)).astype(np.int16)
    else:
        out = a.astype(_REAL[0] if np.dtype(dtype).kind == "f" else dtype)
    return out.view(TiArr) if out.ndim else out[()]


def sqrt(x):
    return np.sqrt(x)


def atomic_add(ref, value):
    ref[...] += np.asarray(value, dtype=ref.dtype)
    return ref


def svd(A):
    """2x2 SVD in Taichi's convention (see module docstring)."""
    A = np.asarray(A)
    dt = A.dtype.type
    if A.shape != (2, 2):
        raise NotImplementedError("only the 2x2 ti.svd is used on the hot path")
    x = A[0, 0] + A[1, 1]
    y = A[1, 0] - A[0, 1]
    scale = dt(1.0) / np.sqrt(x * x + y * y)
    c0, s0 = x * scale, y * scale
    Rp = np.array([[c0, -s0], [s0, c0]], dtype=dt)
    S = Rp.T @ A
    if abs(S[0, 1]) < 1e-5:
        c, s = dt(1), dt(0)
        s1, s2 = S[0, 0], S[1, 1]
    else:
        tau = dt(0.5) * (S[0, 0] - S[1, 1])
        w = np.sqrt(tau * tau + S[0, 1] * S[0, 1])
        t = S[0, 1] / (tau + w) if tau > 0 else S[0, 1] / (tau - w)
        c = dt(1) / np.sqrt(t * t + dt(1))
        s = -t * c
        s1 = c * c * S[0, 0] - dt(2) * c * s * S[0, 1] + s * s * S[1, 1]
        s2 = s * s * S[0, 0] + dt(2) * c * s * S[0, 1] + c * c * S[1, 1]
    if s1 < s2:
        s1, s2 = s2, s1
        V = np.array([[-s, c], [-c, -s]], dtype=dt)
    else:
        V = np.array([[c, s], [-s, c]], dtype=dt)
    U = Rp @ V
    return U.view(TiArr), np.array([[s1, 0], [0, s2]], dtype=dt).view(TiArr), V.view(TiArr)


_FORWARD_TAPE = [False]


def allow_forward_tape():
    """Let ``ti.ad.Tape`` run its body as a plain forward pass (gradient fields
    stay zero).  The golden generator uses this to drive the reference's
    ``compute_grad`` for its losses and states; gradients come from finite
    differences instead."""
    _FORWARD_TAPE[0] = True


class _Tape:
    def __init__(self, loss=None):
        if not _FORWARD_TAPE[0]:
            raise NotImplementedError("Taichi's reverse-mode AD is not emulated by this stand-in")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


ad = types.SimpleNamespace(
    grad_replaced=lambda fn: fn,
    grad_for=lambda primal: (lambda fn: fn),
    Tape=_Tape,
)
