"""Fourier-space operators of ``flowpm/kernels.py`` as host (NumPy) drop-ins.

These return the same arrays as the reference functions, including its
conventions (``laplace_kernel`` is 1 at k = 0, ``gradient_kernel`` order 1
is the 4-point finite difference).  The particle-mesh step itself never
materialises them: the CUDA Fourier kernels evaluate the same weights per
mode from per-axis tables, with k = 0 of the Green's function set to 0 (the
gradient factor is 0 there, so the force is unchanged).
"""
import numpy as np

__all__ = ['fftk', 'laplace_kernel', 'gradient_kernel', 'longrange_kernel',
           'PGD_kernel', 'cic_compensation']


def fftk(shape, symmetric=True, finite=False, dtype=np.float64):
  """k vectors 2*pi*fftfreq(n) per axis, broadcast shaped; with
  ``symmetric`` the last axis keeps its n//2 + 1 non-negative entries
  (flowpm/kernels.py:10-25)."""
  k = []
  nd = len(shape)
  for d in range(nd):
    kd = np.fft.fftfreq(shape[d])
    kd *= 2 * np.pi
    if symmetric and d == nd - 1:
      kd = kd[:shape[d] // 2 + 1]
    kshape = np.ones(nd, dtype='int')
    kshape[d] = len(kd)
    k.append(kd.reshape(kshape).astype(dtype))
  return k


def laplace_kernel(kvec):
  """1/k^2 (flowpm/kernels.py:28-48; 1 at k = 0 as in the reference)."""
  kk = sum(ki**2 for ki in kvec)
  kk = np.array(kk, copy=True)
  kk[kk == 0] = 1
  wts = 1. / kk
  imask = (~(kk == 0)).astype(int)
  return wts * imask


def gradient_kernel(kvec, direction, order=1):
  """i (8 sin k - sin 2k)/6 (order 1) or i k with the Nyquist entry zeroed
  (order 0), flowpm/kernels.py:51-78."""
  if order == 0:
    wts = 1j * kvec[direction]
    flat = np.squeeze(wts).copy()
    flat[len(flat) // 2] = 0
    return flat.reshape(kvec[direction].shape)
  wk = kvec[direction]
  return (1 / 6.0 * (8 * np.sin(wk) - np.sin(2 * wk))) * 1j


def longrange_kernel(kvec, r_split):
  """exp(-k^2 r_split^2), or 1 for r_split = 0 (flowpm/kernels.py:81-102)."""
  if r_split != 0:
    kk = sum(ki**2 for ki in kvec)
    return np.exp(-kk * r_split**2)
  return 1.


def PGD_kernel(kvec, kl, ks):
  """exp(-kl^2/k^2) exp(-k^4/ks^4) (flowpm/kernels.py:105-134)."""
  kk = sum(ki**2 for ki in kvec)
  kk = np.array(kk, copy=True)
  kk[kk == 0] = 1
  v = np.exp(-kl**2 / kk) * np.exp(-kk**2 / ks**4)
  imask = (~(kk == 0)).astype(int)
  return v * imask


def cic_compensation(kvec):
  """prod_d sinc(k_d / 2 pi)^-2 (flowpm/kernels.py:137-152)."""
  kwts = [np.sinc(kvec[i] / (2 * np.pi)) for i in range(3)]
  return (kwts[0] * kwts[1] * kwts[2])**(-2)
