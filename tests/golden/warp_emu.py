"""Pure-Python emulation of the NVIDIA Warp builtins that the HOME-LBM kernels call.

Test infrastructure only: it exists so that the reference's own ``@wp.kernel`` source
(``envs/lbm/lbm_func.py``, ``envs/lbm3d/lbm_func_3d.py`` and their structs) can be executed
on the CPU of a machine without Warp, to produce golden fixtures for the oracle. Nothing in
the shipped library imports it.

Semantics reproduced (those of Warp's CPU backend):

* every launch runs its threads one after another in launch order, the last launch
  dimension fastest (``wp.tid()`` of a C-order linear index);
* ``float`` / ``wp.float32`` values are IEEE binary32: scalars are ``numpy.float32`` and
  Python float literals combine with them as weak scalars (NumPy >= 2 promotion rules), so
  ``1.0 / 9.0 * rho`` rounds ``1/9`` to binary32 exactly as a binary32 division would;
  no operation is fused (no FMA);
* struct fields annotated ``float`` are stored as binary32; arrays of structs hold the
  struct objects themselves (Warp copies a struct by value but its arrays are shared
  handles, which is the same thing for these kernels);
* ``wp.atomic_add`` adds in binary32 in thread order.

Builtins whose Warp implementation is third-party native code are restated here from
their mathematical definition, and say so: the quaternion rotation used by the
``transform_*`` functions and ``mesh_query_ray`` (a brute-force, double-sided
Moller-Trumbore ray/triangle test returning the closest hit with 0 <= t <= max_t).
Results on those paths are therefore pinned to this restatement, not to Warp's binary.
"""
from __future__ import annotations

import inspect
import itertools
import math
import sys
import types

import numpy as np

# --------------------------------------------------------------------------- scalars
float32 = np.float32
float64 = np.float64
int32 = np.int32
uint64 = np.uint64
int64 = np.int64
uint8 = np.uint8


def constant(x):
    return x


def _f32(v):
    return np.float32(v)


# --------------------------------------------------------------------------- vectors
class _VecBase:
    """Fixed-length vector backed by a NumPy array (owned, or a view into an array)."""

    _len = 0
    _dtype = np.float32
    __array_ufunc__ = None  # make NumPy scalars defer to the reflected vector operators

    __slots__ = ("a",)

    def __init__(self, *args):
        if len(args) == 0:
            self.a = np.zeros(self._len, self._dtype)
        elif len(args) == 1 and isinstance(args[0], (_VecBase,)):
            self.a = np.array(args[0].a, self._dtype)
        elif len(args) == 2 and all(isinstance(v, _VecBase) for v in args) \
                and args[0]._len + args[1]._len == self._len:
            self.a = np.concatenate([args[0].a, args[1].a]).astype(self._dtype)
        elif len(args) == 1 and hasattr(args[0], "__len__"):
            self.a = np.array([self._dtype(v) for v in args[0]], self._dtype)
        else:
            if len(args) != self._len:
                raise TypeError(f"{type(self).__name__} expects {self._len} values")
            self.a = np.array([self._dtype(v) for v in args], self._dtype)

    @classmethod
    def _view(cls, arr):
        obj = cls.__new__(cls)
        obj.a = arr
        return obj

    def __len__(self):
        return self._len

    def __getitem__(self, i):
        return self.a[int(i)]

    def __setitem__(self, i, v):
        self.a[int(i)] = v

    def _get(self, i):
        return self.a[i]

    def __call__(self, *args):
        # ``wp.types.vector(length=n, dtype=t)`` is a zero vector inside a kernel and a
        # constructor outside one; the zero instance doubles as that constructor.
        return type(self)(*args)

    x = property(lambda s: s.a[0], lambda s, v: s.a.__setitem__(0, v))
    y = property(lambda s: s.a[1], lambda s, v: s.a.__setitem__(1, v))
    z = property(lambda s: s.a[2], lambda s, v: s.a.__setitem__(2, v))
    w = property(lambda s: s.a[3], lambda s, v: s.a.__setitem__(3, v))

    def _new(self, arr):
        return type(self)._view(np.asarray(arr, self._dtype))

    def __add__(self, o):
        return self._new(self.a + o.a)

    def __sub__(self, o):
        return self._new(self.a - o.a)

    def __neg__(self):
        return self._new(-self.a)

    def __mul__(self, s):
        if isinstance(s, _VecBase):
            raise TypeError("vector * vector is not a Warp builtin")
        return self._new(self.a * self._dtype(s) if not isinstance(s, float) else self.a * s)

    __rmul__ = __mul__

    def __truediv__(self, s):
        return self._new(self.a / (self._dtype(s) if not isinstance(s, float) else s))

    def __eq__(self, o):
        return isinstance(o, _VecBase) and bool(np.array_equal(self.a, o.a))

    __hash__ = object.__hash__

    def __repr__(self):
        return f"{type(self).__name__}({', '.join(str(v) for v in self.a)})"


_vec_cache = {}


def _vector_type(length, dtype=np.float32, name=None):
    key = (length, np.dtype(dtype).name)
    if key not in _vec_cache:
        _vec_cache[key] = type(name or f"vec{length}_{np.dtype(dtype).name}", (_VecBase,),
                               {"_len": length, "_dtype": np.dtype(dtype).type, "__slots__": ()})
    return _vec_cache[key]


vec2 = _vector_type(2, np.float32, "vec2")
vec3 = _vector_type(3, np.float32, "vec3")
vec4 = _vector_type(4, np.float32, "vec4")
# quaternion: memory order x, y, z, w
quat = _vector_type(4, np.float32, "quat")
spatial_vector = _vector_type(6, np.float32, "spatial_vector")
spatial_vectorf = spatial_vector
mat33 = _vector_type(9, np.float32, "mat33")
# transform: p.x p.y p.z q.x q.y q.z q.w
transform = _vector_type(7, np.float32, "transform")


def _transform_ctor(p, q):
    t = transform()
    t.a[0:3] = p.a
    t.a[3:7] = q.a
    return t


class _TypesNS:
    @staticmethod
    def vector(length, dtype=np.float32):
        return _vector_type(length, dtype)()


types_ns = _TypesNS()


# --------------------------------------------------------------------------- arrays
class _ArrayAnnotation:
    def __init__(self, dtype=None, ndim=1):
        self.dtype = dtype
        self.ndim = ndim


class WArray:
    """N-d array of scalars, vectors or structs with Warp indexing semantics."""

    def __init__(self, data, dtype, shape=None):
        self.dtype = dtype
        if isinstance(dtype, type) and issubclass(dtype, _VecBase):
            n = dtype._len
            if isinstance(data, np.ndarray):
                arr = np.array(data, dtype=dtype._dtype)
            else:
                arr = np.array([v.a if isinstance(v, _VecBase) else v for v in data],
                               dtype=dtype._dtype)
            self.shape = tuple(arr.shape[:-1]) if shape is None else tuple(shape)
            self.np = arr.reshape(self.shape + (n,))
            self.kind = "vec"
        elif dtype in (np.float32, np.int32, np.uint64, np.float64, np.int64, np.uint8, int, float):
            dt = {int: np.int32, float: np.float32}.get(dtype, dtype)
            arr = np.array(data, dtype=dt)
            self.shape = tuple(arr.shape) if shape is None else tuple(shape)
            self.np = arr.reshape(self.shape)
            self.kind = "scalar"
        else:  # struct
            self.np = list(data)
            self.shape = (len(self.np),)
            self.kind = "struct"

    # indexing -------------------------------------------------------------
    def _key(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        return tuple(int(i) for i in idx)

    def __getitem__(self, idx):
        k = self._key(idx)
        if self.kind == "struct":
            return self.np[k[0]]
        if self.kind == "vec":
            return self.dtype._view(self.np[k])
        return self.np[k]

    def __setitem__(self, idx, v):
        k = self._key(idx)
        if self.kind == "struct":
            self.np[k[0]] = v
        elif self.kind == "vec":
            self.np[k] = v.a
        else:
            self.np[k] = v

    def numpy(self):
        return self.np

    def zero_(self):
        self.np[...] = 0

    def __len__(self):
        return self.shape[0]


class _ArrayMeta(type):
    """``wp.array`` is an annotation factory, a constructor and an ``isinstance`` target."""

    def __call__(cls, data=None, dtype=None, ndim=None, device=None, requires_grad=False,
                 shape=None):
        if data is None and shape is None:
            return _ArrayAnnotation(dtype, ndim or 1)
        if data is None:
            return zeros(shape, dtype=dtype)
        if isinstance(data, WArray):
            data = data.np
        return WArray(data, dtype)

    def __instancecheck__(cls, obj):
        return isinstance(obj, WArray)


class array(metaclass=_ArrayMeta):  # noqa: N801 - mirrors wp.array
    pass


def array2d(dtype=None):
    return _ArrayAnnotation(dtype, 2)


def array3d(dtype=None):
    return _ArrayAnnotation(dtype, 3)


def array1d(dtype=None):
    return _ArrayAnnotation(dtype, 1)


def _full(shape, dtype, value):
    if isinstance(shape, int):
        shape = (shape,)
    shape = tuple(shape)
    if isinstance(dtype, type) and issubclass(dtype, _VecBase):
        return WArray(np.full(shape + (dtype._len,), value, dtype._dtype), dtype, shape)
    dt = {int: np.int32, float: np.float32}.get(dtype, dtype)
    return WArray(np.full(shape, value, dt), dt, shape)


def zeros(shape, dtype=np.float32, device=None, requires_grad=False):
    return _full(shape, dtype, 0)


def ones(shape, dtype=np.float32, device=None, requires_grad=False):
    return _full(shape, dtype, 1)


# --------------------------------------------------------------------------- structs
def _convert_field(annotation, value):
    if (annotation is float or annotation is np.float32) and isinstance(value, (float, int, np.floating, np.integer)) \
            and not isinstance(value, bool):
        return np.float32(value)
    return value


def struct(cls):
    ann = dict(getattr(cls, "__annotations__", {}))

    def __setattr__(self, name, value):
        if name in ann:
            value = _convert_field(ann[name], value)
        object.__setattr__(self, name, value)

    cls.__setattr__ = __setattr__
    return cls


# --------------------------------------------------------------------------- kernels
_tid_stack = []


def tid():
    t = _tid_stack[-1]
    return t[0] if len(t) == 1 else t


class Kernel:
    def __init__(self, fn):
        self.fn = fn
        self.sig = inspect.signature(fn)
        self.__name__ = fn.__name__

    def _convert_inputs(self, inputs):
        out = []
        for (name, p), v in zip(self.sig.parameters.items(), inputs):
            out.append(_convert_field(p.annotation, v))
        return out

    def __call__(self, *args):
        return self.fn(*args)


def kernel(fn=None, **kw):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


def func(fn):
    return fn


def launch(kernel, dim, inputs=(), device=None, outputs=(), **kw):
    if isinstance(dim, int):
        dim = (dim,)
    args = kernel._convert_inputs(list(inputs) + list(outputs))
    for t in itertools.product(*[range(int(d)) for d in dim]):
        _tid_stack.append(t)
        try:
            kernel.fn(*args)
        finally:
            _tid_stack.pop()


def synchronize():
    pass


class _Device:
    def __init__(self, name="cpu"):
        self.name = name
        self.is_cuda = False

    def __repr__(self):
        return self.name


def get_device(d=None):
    return d if isinstance(d, _Device) else _Device(str(d or "cpu"))


def get_preferred_device():
    return _Device("cpu")


class ScopedDevice:
    def __init__(self, d):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class ScopedCapture:
    def __init__(self, *a, **k):
        raise RuntimeError("graph capture is CUDA-only; launch kernels directly")


def capture_launch(graph):
    raise RuntimeError("graph capture is CUDA-only")


# --------------------------------------------------------------------------- math
def length_sq(v):
    s = v.a[0] * v.a[0]
    for i in range(1, v._len):
        s = s + v.a[i] * v.a[i]
    return s


def length(v):
    return np.sqrt(length_sq(v))


def dot(a, b):
    s = a.a[0] * b.a[0]
    for i in range(1, a._len):
        s = s + a.a[i] * b.a[i]
    return s


def sqrt(x):
    return np.sqrt(np.float32(x))


def cos(x):
    return np.float32(math.cos(float(np.float32(x))))


def sin(x):
    return np.float32(math.sin(float(np.float32(x))))


def atan2(y, x):
    return np.float32(math.atan2(float(np.float32(y)), float(np.float32(x))))


def clamp(x, lo, hi):
    return min(max(x, lo), hi)


def max(a, b):  # noqa: A001 - mirrors wp.max
    return a if a > b else b


def min(a, b):  # noqa: A001
    return a if a < b else b


def abs(x):  # noqa: A001
    return -x if x < 0 else x


def log(x):
    return np.float32(np.log(np.float32(x)))


def atomic_add(arr, idx, value):
    k = arr._key(idx)
    if arr.kind == "vec":
        arr.np[k] = arr.np[k] + value.a
    else:
        arr.np[k] = arr.np[k] + value
    return None


# ---- quaternion / transform: restated from the mathematical definition -------------
def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _qrot(qx, qy, qz, qw, v):
    """Rotate v by unit quaternion q: v(2w^2-1) + 2w (q_v x v) + 2 (q_v . v) q_v, binary32."""
    two = np.float32(2.0)
    c = two * qw * qw - np.float32(1.0)
    d = two * (qx * v[0] + qy * v[1] + qz * v[2])
    cx, cy, cz = _cross((qx, qy, qz), v)
    e = two * qw
    return (v[0] * c + cx * e + qx * d,
            v[1] * c + cy * e + qy * d,
            v[2] * c + cz * e + qz * d)


def transform_identity():
    t = transform()
    t.a[6] = 1.0
    return t


def transform_get_translation(t):
    return vec3(t.a[0], t.a[1], t.a[2])


def transform_inverse(t):
    qx, qy, qz, qw = -t.a[3], -t.a[4], -t.a[5], t.a[6]
    p = _qrot(qx, qy, qz, qw, (t.a[0], t.a[1], t.a[2]))
    out = transform()
    out.a[:] = [-p[0], -p[1], -p[2], qx, qy, qz, qw]
    return out


def transform_point(t, p):
    r = _qrot(t.a[3], t.a[4], t.a[5], t.a[6], (p.a[0], p.a[1], p.a[2]))
    return vec3(r[0] + t.a[0], r[1] + t.a[1], r[2] + t.a[2])


def transform_vector(t, v):
    r = _qrot(t.a[3], t.a[4], t.a[5], t.a[6], (v.a[0], v.a[1], v.a[2]))
    return vec3(r[0], r[1], r[2])


def _transform_call(p, q=None):
    if q is None:
        return transform(p)
    return _transform_ctor(p, q)


# --------------------------------------------------------------------------- meshes
_meshes = {}


class Mesh:
    def __init__(self, points, indices, **kw):
        self.points = np.asarray(points.np if isinstance(points, WArray) else points, np.float32)
        self.indices = np.asarray(indices.np if isinstance(indices, WArray) else indices,
                                  np.int32).reshape(-1, 3)
        self.id = np.uint64(len(_meshes) + 1)
        _meshes[int(self.id)] = self


class _RayQuery:
    def __init__(self, result, t):
        self.result = result
        self.t = t


def ray_triangle(o, d, v0, v1, v2):
    """Double-sided Moller-Trumbore (1997) in binary32. Returns t or None."""
    e1 = (v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2])
    e2 = (v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2])
    p = _cross(d, e2)
    det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2]
    if det == 0.0:
        return None
    inv = np.float32(1.0) / det
    s = (o[0] - v0[0], o[1] - v0[1], o[2] - v0[2])
    u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv
    if u < 0.0 or u > 1.0:
        return None
    q = _cross(s, e1)
    v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv
    if v < 0.0 or u + v > 1.0:
        return None
    t = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv
    return t


def mesh_query_ray(mesh_id, origin, direction, max_t):
    m = _meshes[int(mesh_id)]
    o = tuple(origin.a)
    d = tuple(direction.a)
    best = None
    for tri in m.indices:
        t = ray_triangle(o, d, m.points[tri[0]], m.points[tri[1]], m.points[tri[2]])
        if t is None or t < 0.0 or t > max_t:
            continue
        if best is None or t < best:
            best = t
    if best is None:
        return _RayQuery(False, np.float32(0.0))
    return _RayQuery(True, np.float32(best))


# --------------------------------------------------------------------------- install
def install():
    """Register this module as ``warp`` in ``sys.modules`` and return it."""
    mod = sys.modules[__name__]
    shim = types.ModuleType("warp")
    for name in dir(mod):
        if not name.startswith("__"):
            setattr(shim, name, getattr(mod, name))
    shim.types = types_ns
    shim.transform = _TransformType
    shim.__emulated__ = True
    sys.modules["warp"] = shim
    return shim


class _TransformMeta(type):
    def __call__(cls, *args):
        if len(args) == 2:
            return _transform_ctor(args[0], args[1])
        return transform(*args)

    def __instancecheck__(cls, obj):
        return isinstance(obj, transform)


class _TransformType(metaclass=_TransformMeta):
    _len = 7
    _dtype = np.float32

    @classmethod
    def _view(cls, arr):
        return transform._view(arr)


# arrays created with dtype=wp.transform use the 7-float vector layout
def _is_vec(dtype):
    return isinstance(dtype, type) and (issubclass(dtype, _VecBase) or dtype is _TransformType)


_orig_full = _full


def _full(shape, dtype, value):  # noqa: F811 - transform-aware version
    if dtype is _TransformType:
        dtype = transform
    return _orig_full(shape, dtype, value)


_orig_warray_init = WArray.__init__


def _warray_init(self, data, dtype, shape=None):
    if dtype is _TransformType:
        dtype = transform
    _orig_warray_init(self, data, dtype, shape)


WArray.__init__ = _warray_init
