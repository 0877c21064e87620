"""A minimal NumPy emulation of the TensorFlow 2.5 / TFP 0.13 ops that FlowPM's
particle-mesh modules call, so that the reference's own Python source
(``flowpm/tfpm.py``, ``utils.py``, ``kernels.py``, ``tfbackground.py``,
``tfpower.py``, ``pk.py``, ``cosmology.py``) can be executed unmodified in a
container without TensorFlow.

Test infrastructure only: ``make_golden.py`` installs this module as
``tensorflow`` / ``tensorflow_probability`` in ``sys.modules``, imports the
reference modules from their source tree and records their outputs as the
golden fixtures under ``tests/golden/``.

Semantics emulated (TensorFlow 2.5.0, tensorflow-probability 0.13.0, the
versions pinned in the reference CI workflow ``.github/workflows/ci.yml:39``):

* Tensors are an ``ndarray`` subclass.  In a binary op, every operand that is
  not a Tensor (Python scalar or NumPy array) is converted to the dtype of the
  first Tensor operand, as ``tf.convert_to_tensor`` does inside TF ops; two
  Tensors of different dtypes raise, as TF does.  Arithmetic therefore stays in
  float32 / complex64 exactly where the reference's would.
* ``scatter_nd`` accumulates duplicate indices (sequential order),
  ``gather_nd(batch_dims=1)`` gathers per batch entry, ``math.mod`` is the
  floor modulo, ``cast`` from complex to real keeps the real part.
* ``signal.fft3d`` / ``ifft3d`` transform the three innermost axes in the
  input precision (NumPy 2 pocketfft keeps complex64).
* ``tfp.math.interp_regular_1d_grid`` is linear interpolation on a regular
  grid with constant extension outside the grid.
* ``random.normal`` draws from ``numpy.random.default_rng(seed)``: TF's Philox
  stream is not reproducible without TF, so white noise is an input recorded
  in the fixtures rather than something compared.
"""
import contextlib
import sys
import types
import warnings

import numpy as np

float16 = np.float16
float32 = np.float32
float64 = np.float64
complex64 = np.complex64
complex128 = np.complex128
int32 = np.int32
int64 = np.int64
bool_ = np.bool_


def _np_dtype(dt):
  if dt is None:
    return None
  return np.dtype(dt)


class TensorShape(object):

  def __init__(self, dims):
    self._dims = tuple(int(d) for d in dims)

  def __getitem__(self, key):
    if isinstance(key, slice):
      return TensorShape(self._dims[key])
    return self._dims[key]

  def __len__(self):
    return len(self._dims)

  def __iter__(self):
    return iter(self._dims)

  def as_list(self):
    return list(self._dims)

  def __repr__(self):
    return 'TensorShape(%r)' % (self._dims,)

  def __eq__(self, other):
    return tuple(self) == tuple(other)


class Tensor(np.ndarray):
  """ndarray subclass standing in for an eager ``tf.Tensor``."""

  def __array_finalize__(self, obj):
    pass

  def get_shape(self):
    return TensorShape(self.shape)

  def numpy(self):
    return np.asarray(self).copy()

  @property
  def dtype_tf(self):
    return self.dtype

  def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
    ref = None
    for x in inputs:
      if isinstance(x, Tensor):
        ref = x.dtype
        break
    conv = []
    for x in inputs:
      if isinstance(x, Tensor):
        if x.dtype != ref and ufunc.nin > 1 and ufunc not in _MIXED_OK:
          raise TypeError('tf op with mixed dtypes %s and %s' % (ref, x.dtype))
        conv.append(np.asarray(x))
      else:
        arr = np.asarray(x)
        if ufunc.nin > 1 and ufunc not in _MIXED_OK and arr.dtype != ref:
          with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            arr = arr.astype(ref)
        conv.append(arr)
    if 'out' in kwargs:
      kwargs['out'] = tuple(np.asarray(o) for o in kwargs['out'])
    res = getattr(ufunc, method)(*conv, **kwargs)
    if isinstance(res, tuple):
      return tuple(np.asarray(r).view(Tensor) for r in res)
    return np.asarray(res).view(Tensor)

  def __bool__(self):
    return bool(np.asarray(self))

  def __float__(self):
    return float(np.asarray(self))

  def __int__(self):
    return int(np.asarray(self))

  def __index__(self):
    return int(np.asarray(self))

  def __getitem__(self, key):
    res = np.ndarray.__getitem__(self, key)
    return np.asarray(res).view(Tensor)


# Ufuncs whose operands may legitimately differ in dtype (shifts, ldexp, ...).
_MIXED_OK = set([np.ldexp])


def _t(x, dtype=None):
  """Python / NumPy value -> Tensor, with TF's default dtype rules."""
  if isinstance(x, Tensor):
    if dtype is not None and x.dtype != _np_dtype(dtype):
      with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        return np.asarray(x).astype(_np_dtype(dtype)).view(Tensor)
    return x
  if isinstance(x, (list, tuple)) and len(x) and any(
      isinstance(e, Tensor) for e in _flatten(x)):
    ref = [e for e in _flatten(x) if isinstance(e, Tensor)][0].dtype
    x = np.asarray(_pack(x, ref), dtype=ref)
  if dtype is not None:
    with warnings.catch_warnings():
      warnings.simplefilter('ignore')
      return np.asarray(x).astype(_np_dtype(dtype)).view(Tensor)
  if isinstance(x, (np.ndarray, np.generic)):
    return np.asarray(x).view(Tensor)
  arr = np.asarray(x)
  if isinstance(x, bool):
    arr = arr.astype(np.bool_)
  elif isinstance(x, float) or (isinstance(x, (list, tuple)) and
                                arr.dtype == np.float64):
    arr = arr.astype(np.float32)
  elif isinstance(x, int) or (isinstance(x, (list, tuple)) and
                              arr.dtype == np.int64):
    arr = arr.astype(np.int32)
  elif isinstance(x, complex):
    arr = arr.astype(np.complex128)
  return arr.view(Tensor)


def _flatten(x):
  if isinstance(x, (list, tuple)):
    for e in x:
      for f in _flatten(e):
        yield f
  else:
    yield x


def _pack(x, ref):
  if isinstance(x, (list, tuple)):
    return [_pack(e, ref) for e in x]
  return np.asarray(x).astype(ref)


def convert_to_tensor(value, dtype=None, name=None, dtype_hint=None):
  return _t(value, dtype)


def constant(value, dtype=None, shape=None, name=None):
  out = _t(value, dtype)
  if shape is not None:
    out = np.broadcast_to(out, shape).copy().view(Tensor)
  return out


def cast(x, dtype, name=None):
  with warnings.catch_warnings():
    warnings.simplefilter('ignore')
    if np.iscomplexobj(x) and not np.issubdtype(_np_dtype(dtype),
                                                np.complexfloating):
      return np.asarray(np.real(np.asarray(x))).astype(
          _np_dtype(dtype)).view(Tensor)
    return np.asarray(_t(x)).astype(_np_dtype(dtype)).view(Tensor)


class _Dtypes(object):
  cast = staticmethod(cast)
  float32 = float32
  float64 = float64
  complex64 = complex64
  complex128 = complex128
  int32 = int32
  int64 = int64


dtypes = _Dtypes()
DType = np.dtype


@contextlib.contextmanager
def name_scope(name):
  yield name


def function(f=None, **kwargs):
  if f is None:
    return lambda g: g
  return f


def _binary(a, b, op):
  if isinstance(a, Tensor):
    return op(a, b)
  if isinstance(b, Tensor):
    return op(_t(a, b.dtype), b)
  ta = _t(a)
  return op(ta, _t(b, ta.dtype))


def multiply(x, y, name=None):
  return _binary(x, y, lambda u, v: u * v)


def add(x, y, name=None):
  return _binary(x, y, lambda u, v: u + v)


def subtract(x, y, name=None):
  return _binary(x, y, lambda u, v: u - v)


def zeros(shape, dtype=float32, name=None):
  return np.zeros([int(s) for s in shape], dtype=_np_dtype(dtype)).view(Tensor)


def ones(shape, dtype=float32, name=None):
  return np.ones([int(s) for s in shape], dtype=_np_dtype(dtype)).view(Tensor)


def zeros_like(x, dtype=None, name=None):
  x = _t(x)
  return np.zeros(x.shape, dtype=_np_dtype(dtype) or x.dtype).view(Tensor)


def ones_like(x, dtype=None, name=None):
  x = _t(x)
  return np.ones(x.shape, dtype=_np_dtype(dtype) or x.dtype).view(Tensor)


def stack(values, axis=0, name=None):
  vals = [np.asarray(_t(v)) for v in values]
  return np.stack(vals, axis=axis).view(Tensor)


def concat(values, axis, name=None):
  vals = [np.asarray(_t(v)) for v in values]
  return np.concatenate(vals, axis=axis).view(Tensor)


def reshape(x, shape, name=None):
  shp = [int(s) for s in np.asarray(shape).ravel()]
  return np.reshape(np.asarray(_t(x)), shp).view(Tensor)


def expand_dims(x, axis, name=None):
  return np.expand_dims(np.asarray(_t(x)), axis).view(Tensor)


def squeeze(x, axis=None, name=None):
  return np.squeeze(np.asarray(_t(x)), axis=axis).view(Tensor)


def tile(x, multiples, name=None):
  return np.tile(np.asarray(_t(x)), [int(m) for m in multiples]).view(Tensor)


def split(x, num_or_size_splits, axis=0, num=None, name=None):
  return [
      np.asarray(p).view(Tensor)
      for p in np.split(np.asarray(_t(x)), num_or_size_splits, axis=axis)
  ]


def range(start, limit=None, delta=1, dtype=None, name=None):  # noqa: A001
  if limit is None:
    start, limit = 0, start
  return np.arange(int(start), int(limit), int(delta),
                   dtype=_np_dtype(dtype) or np.int32).view(Tensor)


def shape(x, out_type=int32, name=None):
  return np.asarray(np.shape(x), dtype=np.int32).view(Tensor)


def reduce_sum(x, axis=None, keepdims=False, name=None):
  return np.asarray(np.sum(np.asarray(_t(x)), axis=axis,
                           keepdims=keepdims)).view(Tensor)


def reduce_prod(x, axis=None, keepdims=False, name=None):
  x = np.asarray(x)
  return np.asarray(np.prod(x, axis=axis, keepdims=keepdims)).view(Tensor)


def floor(x, name=None):
  return np.floor(_t(x))


def abs(x, name=None):  # noqa: A001
  return np.abs(_t(x))


def exp(x, name=None):
  return np.exp(_t(x))


def pow(x, y, name=None):  # noqa: A001
  return _binary(x, y, lambda u, v: np.power(u, v))


def sign(x, name=None):
  return np.sign(_t(x))


def where(condition, x=None, y=None, name=None):
  if x is None:
    return np.argwhere(np.asarray(condition)).astype(np.int64).view(Tensor)
  x = _t(x)
  return np.where(np.asarray(condition), np.asarray(x),
                  np.asarray(_t(y, x.dtype))).view(Tensor)


def einsum(equation, *inputs, **kwargs):
  ops = [np.asarray(_t(x)) for x in inputs]
  return np.einsum(equation, *ops).astype(ops[0].dtype).view(Tensor)


def gather(params, indices, axis=0, name=None):
  return np.take(np.asarray(_t(params)), np.asarray(indices),
                 axis=axis).view(Tensor)


def gather_nd(params, indices, batch_dims=0, name=None):
  params = np.asarray(_t(params))
  indices = np.asarray(indices)
  if batch_dims == 0:
    k = indices.shape[-1]
    return params[tuple(indices[..., i] for i in builtins_range(k))].view(
        Tensor)
  assert batch_dims == 1
  out = []
  for b in builtins_range(params.shape[0]):
    idx = indices[b]
    k = idx.shape[-1]
    out.append(params[b][tuple(idx[..., i] for i in builtins_range(k))])
  return np.stack(out).view(Tensor)


def scatter_nd(indices, updates, shape, name=None):
  indices = np.asarray(indices)
  updates = np.asarray(_t(updates))
  out = np.zeros([int(s) for s in shape], dtype=updates.dtype)
  k = indices.shape[-1]
  idx = tuple(indices[..., i].ravel() for i in builtins_range(k))
  upd = updates.reshape((-1,) + out.shape[k:])
  np.add.at(out, idx, upd)
  return out.view(Tensor)


def clip_by_value(t, clip_value_min, clip_value_max, name=None):
  t = _t(t)
  return np.clip(np.asarray(t), np.asarray(clip_value_min),
                 np.asarray(clip_value_max)).astype(t.dtype).view(Tensor)


def linspace(start, stop, num, name=None, axis=0):
  start = _t(start)
  return np.linspace(np.asarray(start), np.asarray(stop), int(num),
                     dtype=start.dtype).view(Tensor)


def less(x, y, name=None):
  return np.asarray(np.asarray(x) < np.asarray(y)).view(Tensor)


def while_loop(cond, body, loop_vars, swap_memory=False,
               maximum_iterations=None, **kwargs):
  loop_vars = list(loop_vars)
  it = 0
  while cond(*loop_vars):
    if maximum_iterations is not None and it >= maximum_iterations:
      break
    loop_vars = list(body(*loop_vars))
    it += 1
  return loop_vars


class TensorArray(object):

  def __init__(self, dtype, size=None, dynamic_size=False, **kwargs):
    self._dtype = _np_dtype(dtype)
    self._items = {}

  def write(self, index, value):
    self._items[int(index)] = np.asarray(_t(value, self._dtype))
    return self

  def stack(self):
    keys = sorted(self._items)
    return np.stack([self._items[k] for k in keys]).view(Tensor)


def map_fn(fn, elems, dtype=None, **kwargs):
  elems = _t(elems)
  return np.stack(
      [np.asarray(fn(elems[i])) for i in builtins_range(elems.shape[0])]).view(
          Tensor)


def _make_math():
  m = types.ModuleType('tensorflow.math')
  m.log = lambda x, name=None: np.log(_t(x))
  m.exp = lambda x, name=None: np.exp(_t(x))
  m.sqrt = lambda x, name=None: np.sqrt(_t(x))
  m.sin = lambda x, name=None: np.sin(_t(x))
  m.cos = lambda x, name=None: np.cos(_t(x))
  m.sinh = lambda x, name=None: np.sinh(_t(x))
  m.abs = lambda x, name=None: np.abs(_t(x))
  m.sign = lambda x, name=None: np.sign(_t(x))
  m.pow = pow
  m.real = lambda x, name=None: np.real(np.asarray(_t(x))).copy().view(Tensor)
  m.imag = lambda x, name=None: np.imag(np.asarray(_t(x))).copy().view(Tensor)
  m.conj = lambda x, name=None: np.conj(_t(x))
  m.mod = lambda x, y, name=None: _binary(x, y, lambda u, v: np.mod(u, v))
  m.argmin = lambda x, axis=None, name=None, output_type=int64: np.argmin(
      np.asarray(x), axis=axis).astype(np.int64).view(Tensor)

  def bincount(arr, weights=None, minlength=None, maxlength=None,
               dtype=int32, name=None):
    arr = np.asarray(arr).ravel()
    w = None if weights is None else np.asarray(weights).ravel()
    res = np.bincount(arr, weights=w, minlength=minlength or 0)
    if w is not None:
      res = res.astype(w.dtype)
    return res.view(Tensor)

  m.bincount = bincount
  return m


def _make_signal():
  s = types.ModuleType('tensorflow.signal')

  def fft3d(x, name=None):
    x = np.asarray(_t(x))
    return np.fft.fftn(x, axes=(-3, -2, -1)).astype(x.dtype).view(Tensor)

  def ifft3d(x, name=None):
    x = np.asarray(_t(x))
    return np.fft.ifftn(x, axes=(-3, -2, -1)).astype(x.dtype).view(Tensor)

  def fft2d(x, name=None):
    x = np.asarray(_t(x))
    return np.fft.fftn(x, axes=(-2, -1)).astype(x.dtype).view(Tensor)

  def ifft2d(x, name=None):
    x = np.asarray(_t(x))
    return np.fft.ifftn(x, axes=(-2, -1)).astype(x.dtype).view(Tensor)

  s.fft3d, s.ifft3d, s.fft2d, s.ifft2d = fft3d, ifft3d, fft2d, ifft2d
  return s


class _Random(object):
  """``tf.random.normal`` drawn from NumPy's PCG64 (see module docstring)."""

  @staticmethod
  def normal(shape, mean=0.0, stddev=1.0, dtype=float32, seed=None,
             name=None):
    rng = np.random.default_rng(seed)
    out = rng.standard_normal([int(s) for s in shape])
    return (out * float(stddev) + float(mean)).astype(
        _np_dtype(dtype)).view(Tensor)


builtins_range = __builtins__['range'] if isinstance(
    __builtins__, dict) else __builtins__.range

math = _make_math()
signal = _make_signal()
random = _Random()


def _make_tfp():
  tfp = types.ModuleType('tensorflow_probability')
  tfp_math = types.ModuleType('tensorflow_probability.math')

  def interp_regular_1d_grid(x, x_ref_min, x_ref_max, y_ref, axis=-1,
                             fill_value='constant_extension', name=None):
    """Linear interpolation on a regular grid, constant extension."""
    x = _t(x, float32)
    y_ref = np.asarray(_t(y_ref))
    dt = y_ref.dtype
    xmin = np.asarray(x_ref_min, dtype=dt)
    xmax = np.asarray(x_ref_max, dtype=dt)
    ny = y_ref.shape[-1]
    xa = np.asarray(x, dtype=dt)
    idx = (xa - xmin) / (xmax - xmin) * dt.type(ny - 1)
    idx = np.clip(idx, dt.type(0), dt.type(ny - 1))
    below = np.clip(np.floor(idx), 0, ny - 2).astype(np.int64)
    t = (idx - below.astype(dt)).astype(dt)
    y0 = y_ref[..., below]
    y1 = y_ref[..., below + 1]
    return (y0 + t * (y1 - y0)).astype(dt).view(Tensor)

  tfp_math.interp_regular_1d_grid = interp_regular_1d_grid
  tfp.math = tfp_math
  return tfp, tfp_math


def install():
  """Register this module as ``tensorflow`` and a TFP stand-in."""
  mod = sys.modules[__name__]
  sys.modules['tensorflow'] = mod
  sys.modules['tensorflow.math'] = math
  sys.modules['tensorflow.signal'] = signal
  tfp, tfp_math = _make_tfp()
  sys.modules['tensorflow_probability'] = tfp
  sys.modules['tensorflow_probability.math'] = tfp_math
  return mod
