"""Mesh operators mirroring ``flowpm/utils.py``: CIC paint / readout, the
normalised 3-D FFT pair and white noise, on CUDA tensors through the C
library.  Inputs may be torch tensors or NumPy arrays (copied to the current
CUDA device); results are CUDA tensors.
"""
import os

import numpy as np
import torch

from . import _lib
from . import _autograd

__all__ = ['cic_paint', 'cic_paint_2d', 'cic_readout', 'cic_neighbours',
           'r2c3d', 'c2r3d', 'white_noise', 'compensate_cic']


def as_cuda(x, dtype=torch.float32):
  """Contiguous CUDA tensor of ``dtype`` (NumPy / lists are copied over)."""
  if not isinstance(x, torch.Tensor):
    x = torch.as_tensor(np.asarray(x))
  if not x.is_cuda:
    x = x.to('cuda')
  if x.dtype != dtype:
    x = x.to(dtype)
  return x.contiguous()


def _check_mesh(mesh):
  if mesh.dim() != 4:
    raise ValueError('mesh must be (batch, nx, ny, nz), got %s' %
                     (tuple(mesh.shape),))


def cic_paint(mesh, part, weight=None, name='CiCPaint'):
  """Paint particles on a 3D mesh (flowpm/utils.py:32-91).

  mesh: (batch, nx, ny, nz); part: (batch, npart, 3) (or any shape with a
  trailing 3 that flattens to it) in mesh units; weight: (batch, npart) or
  None.  Returns mesh + the CIC deposit; neighbours wrap periodically.
  Differentiable in mesh, part and weight (fpm_cic_paint_adjoint)."""
  mesh = as_cuda(mesh)
  _check_mesh(mesh)
  B, nx, ny, nz = mesh.shape
  part = as_cuda(part).reshape(B, -1, 3)
  npart = part.shape[1]
  w = None
  if weight is not None:
    w = as_cuda(weight).reshape(B, npart)
  if _autograd.needs_grad(mesh, part, w):
    return _autograd.CicPaint.apply(mesh, part, w)
  out = mesh.clone()
  _lib.call('fpm_cic_paint', _lib.ptr(out), B, nx, ny, nz, _lib.ptr(part),
            npart, _lib.ptr(w), _lib.stream_ptr())
  return out


def cic_paint_2d(mesh, part, weight=None, mask=None, name='CiCPaint2D'):
  """Paint particles on a 2-D mesh (flowpm/utils.py:94-160).

  mesh: (batch, nx, ny); part: (batch, npart, 2) in mesh units; weight:
  (batch, npart) or None; mask: (batch, npart) booleans or None (particles
  with False are left out).  Indices wrap modulo ny on both axes, as the
  reference's.  Differentiable in mesh, part and weight."""
  mesh = as_cuda(mesh)
  if mesh.dim() != 3 or mesh.dtype != torch.float32:
    raise ValueError('mesh must be a float32 (batch, nx, ny) tensor')
  mesh = mesh.contiguous()
  B, nx, ny = mesh.shape
  part = as_cuda(part).reshape(B, -1, 2).contiguous()
  npart = part.shape[1]
  w = None
  if weight is not None:
    w = as_cuda(weight).reshape(B, npart).contiguous()
  m = None
  if mask is not None:
    m = as_cuda(mask, dtype=torch.uint8).reshape(B, npart).contiguous()
  if _autograd.needs_grad(mesh, part, w):
    return _autograd.CicPaint2D.apply(mesh, part, w, m)
  out = mesh.clone()
  _lib.call('fpm_cic_paint_2d', _lib.ptr(out), B, nx, ny, _lib.ptr(part),
            npart, _lib.ptr(w), _lib.ptr(m), _lib.stream_ptr())
  return out


def cic_readout(mesh, part, name='CiCReadout'):
  """Read the mesh out at particle positions (flowpm/utils.py:163-210).
  Returns (batch, npart); differentiable in mesh and part
  (fpm_cic_readout_adjoint)."""
  mesh = as_cuda(mesh)
  _check_mesh(mesh)
  B, nx, ny, nz = mesh.shape
  part = as_cuda(part).reshape(B, -1, 3)
  npart = part.shape[1]
  if _autograd.needs_grad(mesh, part):
    return _autograd.CicReadout.apply(mesh, part)
  out = torch.empty((B, npart), dtype=torch.float32, device=mesh.device)
  _lib.call('fpm_cic_readout', _lib.ptr(mesh), B, nx, ny, nz, _lib.ptr(part),
            npart, _lib.ptr(out), _lib.stream_ptr())
  return out


def cic_neighbours(part, nc):
  """Flat neighbour cells (int32) and CIC weights, (npart, 8) each, in the
  reference's neighbour order, for positions ``part`` (npart, 3)."""
  nc = [nc] * 3 if isinstance(nc, int) else [int(n) for n in nc]
  part = as_cuda(part).reshape(-1, 3)
  n = part.shape[0]
  idx = torch.empty((n, 8), dtype=torch.int32, device=part.device)
  w = torch.empty((n, 8), dtype=torch.float32, device=part.device)
  _lib.call('fpm_cic_neighbours', nc[0], nc[1], nc[2], _lib.ptr(part), n,
            _lib.ptr(idx), _lib.ptr(w), _lib.stream_ptr())
  return idx, w


def r2c3d(rfield, norm=None, dtype=torch.complex64, name='R2C3D'):
  """Full complex FFT of a real (batch, nx, ny, nz) field times 1/norm
  (flowpm/utils.py:213-241).  float64 input / complex128 dtype use double
  precision."""
  dbl = dtype == torch.complex128
  rfield = as_cuda(rfield, torch.float64 if dbl else torch.float32)
  _check_mesh(rfield)
  B, nx, ny, nz = rfield.shape
  if norm is None:
    norm = nx * ny * nz
  out = torch.empty(rfield.shape, dtype=dtype, device=rfield.device)
  _lib.call('fpm_r2c3d', _lib.ptr(rfield), _lib.ptr(out), B, nx, ny, nz,
            1.0 / float(norm), int(dbl), _lib.stream_ptr())
  return out


def c2r3d(cfield, norm=None, dtype=torch.float32, name='C2R3D'):
  """Real part of the inverse FFT times norm (flowpm/utils.py:244-272)."""
  dbl = dtype == torch.float64
  cfield = as_cuda(cfield, torch.complex128 if dbl else torch.complex64)
  _check_mesh(cfield)
  B, nx, ny, nz = cfield.shape
  if norm is None:
    norm = nx * ny * nz
  out = torch.empty(cfield.shape, dtype=dtype, device=cfield.device)
  _lib.call('fpm_c2r3d', _lib.ptr(cfield), _lib.ptr(out), B, nx, ny, nz,
            float(norm) / float(nx * ny * nz), int(dbl), _lib.stream_ptr())
  return out


def _seed(seed):
  if seed is None:
    return int.from_bytes(os.urandom(8), 'little')
  return int(seed) & 0xFFFFFFFFFFFFFFFF


def white_noise(nc, batch_size=1, seed=None, type='complex',
                name='WhiteNoise'):
  """Gaussian white noise N(0, sqrt(N^3)) on a (batch, nx, ny, nz) cube
  (flowpm/utils.py:337-355), from the library's Philox4x32-10 counter
  generator (element e of the batch-major array uses counter e // 4)."""
  nc = [nc] * 3 if isinstance(nc, int) else [int(n) for n in nc]
  n = nc[0] * nc[1] * nc[2]
  white = torch.empty([batch_size] + nc, dtype=torch.float32, device='cuda')
  _lib.call('fpm_white_noise', _lib.ptr(white), batch_size * n, _seed(seed),
            float(n)**0.5, _lib.stream_ptr())
  if type == 'real':
    return white
  if type == 'complex':
    return r2c3d(white, norm=n)
  raise ValueError(type)


def compensate_cic(field, name='CompensateCiC'):
  """Divide a CIC-painted field by the CIC window
  (flowpm/utils.py:11-29); uses the full-spectrum FFT pair."""
  from . import kernels as fpk
  field = as_cuda(field)
  _check_mesh(field)
  nc = list(field.shape[1:])
  n = nc[0] * nc[1] * nc[2]
  kvec = fpk.fftk(nc, symmetric=False)
  w = torch.as_tensor(fpk.cic_compensation(kvec).astype(np.complex64),
                      device=field.device)
  dk = r2c3d(field, norm=n)
  return c2r3d(dk * w, norm=n)
