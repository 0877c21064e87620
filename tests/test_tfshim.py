"""The NumPy emulation of TensorFlow that runs the reference's own source
for the golden fixtures (tests/golden/tfshim.py), checked op by op against
TensorFlow 2.5's documented semantics on hand-computed cases, for every op
whose semantics the fixtures depend on:

* tf.cast: float to int truncates toward zero; complex to real keeps the
  real part (the cell index and spectrum casts of flowpm/utils.py:78,
  :142, :204 and flowpm/pk.py:75-84);
* tf.math.mod: floor modulo, the sign of the divisor (the periodic wrap,
  flowpm/utils.py:79);
* tf.scatter_nd: duplicate indices are summed (the CIC paint,
  flowpm/utils.py:87-89);
* tf.gather_nd: the last index axis addresses the leading axes, per batch
  entry with batch_dims=1 (the readout, flowpm/utils.py:207-209);
* tf.signal.fft3d / ifft3d: unnormalised forward, 1/N inverse, over the
  three innermost axes, in the input precision (r2c3d / c2r3d,
  flowpm/utils.py:213-272);
* binary ops convert a Python or NumPy operand to the tensor's dtype
  (tf.convert_to_tensor inside the op), and refuse two tensors of
  different dtypes;
* tf.math.bincount with weights and minlength (flowpm/pk.py:77-82);
* tfp.math.interp_regular_1d_grid: linear on a regular grid, constant
  extension beyond it (the background tables, flowpm/tfbackground.py:678).
"""
import importlib.util
import os

import numpy as np
import pytest
from numpy.testing import assert_allclose, assert_array_equal

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def tf():
  spec = importlib.util.spec_from_file_location(
      'tfshim_under_test', os.path.join(HERE, 'golden', 'tfshim.py'))
  mod = importlib.util.module_from_spec(spec)
  spec.loader.exec_module(mod)
  return mod


def test_cast_truncates_and_keeps_real_part(tf):
  x = tf.constant([-1.7, -0.5, 0.0, 0.5, 1.7, 2.999], dtype=tf.float32)
  assert_array_equal(np.asarray(tf.cast(x, tf.int32)), [-1, 0, 0, 0, 1, 2])
  z = tf.constant([1.5 + 2j, -3 - 4j], dtype=tf.complex64)
  r = tf.cast(z, tf.float32)
  assert r.dtype == np.float32
  assert_array_equal(np.asarray(r), [1.5, -3.0])


def test_mod_is_floor_modulo(tf):
  x = tf.constant([-5, -1, 0, 3, 7, 8], dtype=tf.int32)
  assert_array_equal(np.asarray(tf.math.mod(x, 4)), [3, 3, 0, 3, 3, 0])


def test_scatter_nd_sums_duplicates(tf):
  out = tf.scatter_nd([[0], [2], [0], [3]],
                      tf.constant([1., 2., 3., 4.], dtype=tf.float32), [5])
  assert out.dtype == np.float32
  assert_array_equal(np.asarray(out), [4., 0., 2., 4., 0.])
  out2 = tf.scatter_nd([[0, 1], [0, 1], [1, 0]],
                       tf.constant([1., 1., 5.], dtype=tf.float32), [2, 2])
  assert_array_equal(np.asarray(out2), [[0., 2.], [5., 0.]])


def test_gather_nd(tf):
  p = tf.constant(np.arange(12, dtype=np.float32).reshape(3, 4))
  assert_array_equal(np.asarray(tf.gather_nd(p, [[1, 2], [0, 0], [2, 3]])),
                     [6., 0., 11.])
  pb = tf.constant(np.arange(24, dtype=np.float32).reshape(2, 3, 4))
  got = tf.gather_nd(pb, [[[0, 1], [2, 3]], [[1, 1], [0, 0]]], batch_dims=1)
  assert_array_equal(np.asarray(got), [[1., 11.], [17., 12.]])


def test_fft3d_normalisation_and_precision(tf):
  rng = np.random.default_rng(0)
  x = (rng.standard_normal((2, 4, 6, 8)) +
       1j * rng.standard_normal((2, 4, 6, 8))).astype(np.complex64)
  f = tf.signal.fft3d(tf.constant(x))
  assert f.dtype == np.complex64
  # unnormalised: the zero mode is the plain sum
  assert_allclose(np.asarray(f)[:, 0, 0, 0], x.sum(axis=(1, 2, 3)),
                  rtol=1e-5)
  # a single plane wave transforms to N at its own mode
  n = np.indices((4, 6, 8))
  wave = np.exp(2j * np.pi * (n[0] * 1 / 4 + n[1] * 2 / 6 + n[2] * 3 / 8))
  fw = np.asarray(tf.signal.fft3d(tf.constant(wave.astype(np.complex64))))
  assert_allclose(abs(fw[1, 2, 3]), 4 * 6 * 8, rtol=1e-5)
  assert np.abs(fw).sum() - abs(fw[1, 2, 3]) < 1e-2
  back = tf.signal.ifft3d(f)
  assert back.dtype == np.complex64
  assert_allclose(np.asarray(back), x, atol=1e-5)


def test_binary_ops_convert_to_the_tensor_dtype(tf):
  x = tf.constant([1.0, 2.0], dtype=tf.float32)
  assert (x * 0.1).dtype == np.float32
  assert (x * np.float64(0.1)).dtype == np.float32
  assert (np.array([0.5, 0.25]) + x).dtype == np.float32
  z = tf.constant([1 + 1j], dtype=tf.complex64)
  assert (z * 1j).dtype == np.complex64
  with pytest.raises(TypeError):
    _ = x + tf.constant([1.0, 2.0], dtype=tf.float64)


def test_bincount_weights_and_minlength(tf):
  out = tf.math.bincount(np.array([0, 2, 2, 5]),
                         weights=np.array([1., 2., 3., 4.], np.float32),
                         minlength=8)
  assert_allclose(np.asarray(out), [1., 0., 5., 0., 0., 4., 0., 0.])
  assert np.asarray(out).dtype == np.float32


def test_interp_regular_1d_grid(tf):
  tf_, tfp_math = tf._make_tfp()
  y = np.array([0., 10., 20., 40.], np.float32)
  got = tfp_math.interp_regular_1d_grid(
      np.array([-1., 0., 0.5, 1.5, 2.25, 3., 7.], np.float32), 0., 3., y)
  assert_allclose(np.asarray(got), [0., 0., 5., 15., 25., 40., 40.],
                  rtol=1e-6)
