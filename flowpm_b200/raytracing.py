"""Lensing density planes from an N-body state (flowpm/raytracing.py:49-109).

``density_plane`` cuts one slab of the (optionally rotated and shifted)
particle distribution and projects it on a 2-D grid with CIC weights;
``density_planes`` does the same for many slabs in one pass over the
particles (fpm_density_planes).  Both are differentiable in the positions.
"""
import numpy as np
import torch

from . import _autograd
from . import _lib
from .utils import as_cuda

__all__ = ['density_plane', 'density_planes']

MAX_PLANES = 64  # slabs per library call


def _nc3(nc):
  return [nc] * 3 if isinstance(nc, int) else [int(n) for n in nc]


def _planes(X, nc, centers, widths, res, rotation, shift):
  B, npart = X.shape[0], X.shape[1]
  nx, ny, nz = nc
  rot = None if rotation is None else _lib.dvec(
      np.asarray(rotation, dtype=np.float64).reshape(9))
  sh = None if shift is None else _lib.dvec(
      np.asarray(shift, dtype=np.float64).reshape(3))
  args = {
      'shape': (B, len(centers), res, res),
      'c': (B, npart, nx, ny, nz, rot, sh, len(centers), _lib.dvec(centers),
            _lib.dvec(widths), res),
  }
  if _autograd.needs_grad(X):
    return _autograd.DensityPlanes.apply(X, args)
  out = torch.empty(args['shape'], dtype=torch.float32, device=X.device)
  _lib.call('fpm_density_planes', _lib.ptr(X), *args['c'], _lib.ptr(out),
            _lib.stream_ptr())
  return out


def density_planes(state, nc, centers, widths, plane_resolution,
                   rotation=None, shift=None):
  """Density planes (batch, len(centers), res, res) of the slabs
  center - width/2 < z <= center + width/2 (voxel units) of
  ``state[0]`` after ``rotation`` (3x3, applied as R x) and ``shift``
  (fractions of the box): the transform, the 2-D periodic wrap and the
  normalisation of flowpm/raytracing.py:49-109."""
  nc = _nc3(nc)
  X = as_cuda(state)[0]
  centers = [float(c) for c in np.atleast_1d(centers)]
  widths = np.broadcast_to(np.asarray(widths, dtype=np.float64),
                           (len(centers),)).tolist()
  res = int(plane_resolution)
  parts = []
  for i in range(0, len(centers), MAX_PLANES):
    parts.append(_planes(X, nc, centers[i:i + MAX_PLANES],
                         widths[i:i + MAX_PLANES], res, rotation, shift))
  return parts[0] if len(parts) == 1 else torch.cat(parts, dim=1)


def density_plane(state, nc, center, width, plane_resolution, rotation=None,
                  shift=None, name='density_plane'):
  """One density plane (batch, res, res) (flowpm/raytracing.py:49-109)."""
  return density_planes(state, nc, [center], [width], plane_resolution,
                        rotation=rotation, shift=shift)[:, 0]
