"""Binned power spectrum mirroring ``flowpm/pk.py`` (``power_spectrum``),
computed on the device by the C library (fpm_power_spectrum)."""
import numpy as np
import torch

from . import _lib
from .utils import as_cuda

__all__ = ['power_spectrum', 'pk_edges']


def pk_edges(shape, boxsize, kmin, dk):
  """Bin edges of flowpm/pk.py:18-19: arange(kmin, pi min(N) / max(L) +
  dk / 2, dk)."""
  kmax = np.pi * np.min(shape) / np.max(boxsize) + dk / 2
  return np.arange(kmin, kmax, dk)


def power_spectrum(field, kmin=5, dk=0.5, boxsize=False):
  """Power spectrum of a real field (batch, nx, ny, nz) in a box of
  ``boxsize`` (3 lengths): returns (kbins, power) with kbins the bin
  centres (NumPy) and power a (batch, nbins) CUDA tensor, normalised as
  flowpm/pk.py:39-103."""
  field = as_cuda(field)
  if field.dim() != 4:
    raise ValueError('field must be (batch, nx, ny, nz)')
  B, nx, ny, nz = field.shape
  boxsize = np.asarray(boxsize, dtype=np.float64)
  if boxsize.size == 1:
    boxsize = np.repeat(boxsize.reshape(1), 3)
  kedges = pk_edges([nx, ny, nz], boxsize, kmin, dk)
  if len(kedges) < 2:
    raise ValueError('fewer than two bin edges')
  out = torch.empty((B, len(kedges) - 1), dtype=torch.float32,
                    device=field.device)
  _lib.call('fpm_power_spectrum', _lib.ptr(field), B, nx, ny, nz,
            _lib.dvec(boxsize), float(kmin), float(dk), len(kedges),
            _lib.ptr(out), _lib.stream_ptr())
  kbins = kedges[:-1] + (kedges[1:] - kedges[:-1]) / 2
  return kbins, out
