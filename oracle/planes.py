"""CPU restatement (test infrastructure only) of the reference's 2-D CIC paint
and lensing density planes: flowpm/utils.py:94-160 (cic_paint_2d) and
flowpm/raytracing.py:49-109 (density_plane).  Pinned to tests/golden/planes.npz,
produced by the reference's own source."""
import numpy as np
import torch

_CONN2 = ((0, 0), (1, 0), (0, 1), (1, 1))  # flowpm/utils.py:133


def cic_paint_2d(mesh, part, weight=None, mask=None):
  """flowpm/utils.py:94-160: 4 neighbours floor + {0,1}^2, weights
  (1 - |x - n|)(1 - |y - n|) (times weight), indices int-cast then taken
  modulo ny on both axes (the reference's nc = ny), masked particles
  dropped."""
  mesh = torch.as_tensor(mesh).clone()
  part = torch.as_tensor(part)
  B, nx, ny = mesh.shape
  part = part.reshape(B, -1, 2)
  fl = torch.floor(part)
  flat = mesh.reshape(-1)
  for cx, cy in _CONN2:
    n = fl + torch.tensor([cx, cy], dtype=part.dtype)
    k = 1. - torch.abs(part - n)
    w = k[..., 0] * k[..., 1]
    if weight is not None:
      w = torch.as_tensor(weight, dtype=part.dtype) * w
    idx = torch.remainder(n.to(torch.int32), ny).to(torch.int64)
    lin = (torch.arange(B).reshape(B, 1) * nx + idx[..., 0]) * ny + idx[..., 1]
    if mask is not None:
      keep = torch.as_tensor(mask).reshape(B, -1).to(torch.bool)
      lin, w = lin[keep], w[keep]
    flat.index_add_(0, lin.reshape(-1), w.reshape(-1).to(flat.dtype))
  return mesh


def density_plane(state, nc, center, width, plane_resolution, rotation=None,
                  shift=None):
  """flowpm/raytracing.py:49-109: optional rotation and shift of the
  positions, xy mod nx, rescaled to the plane grid, particles with
  center - width/2 < z <= center + width/2 painted in 2-D, normalised by
  (nx / res) (ny / res) width."""
  state = torch.as_tensor(state)
  if isinstance(nc, int):
    nc = [nc, nc, nc]
  nx, ny, nz = nc
  pos = state[0]
  B = pos.shape[0]
  if rotation is not None:
    pos = torch.einsum('ij,bkj->bki', torch.as_tensor(rotation, dtype=pos.dtype),
                       pos)
  if shift is not None:
    pos = pos + torch.tensor([nx, ny, nz], dtype=pos.dtype) * torch.as_tensor(
        shift, dtype=pos.dtype)
  xy = pos[..., :2]
  d = pos[..., 2]
  xy = torch.remainder(xy, nx)
  xy = xy / nx * plane_resolution
  mask = (d > (center - width / 2)) & (d <= (center + width / 2))
  plane = torch.zeros((B, plane_resolution, plane_resolution), dtype=pos.dtype)
  plane = cic_paint_2d(plane, xy, mask=mask)
  return plane / ((nx / plane_resolution) * (ny / plane_resolution) * width)
