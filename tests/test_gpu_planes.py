"""2-D CIC paint and lensing density planes (flowpm/utils.py:94-160,
flowpm/raytracing.py:49-109) through the C ABI: parity with the
reference's own output (golden) and with the oracle, the reference's wrap
of both axes by ny, and gradients against the oracle's autograd."""
import numpy as np
import pytest
import torch
from numpy.testing import assert_allclose

from conftest import golden
from oracle import planes as opl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def fpm(cuda):
  import flowpm_b200
  return flowpm_b200


def host(t):
  return t.detach().cpu().numpy()


def test_cic_paint_2d_golden(fpm):
  z = golden('planes')
  zz = np.zeros((2, 24, 24), np.float32)
  u = fpm.utils
  assert_allclose(host(u.cic_paint_2d(zz, z['pos'])), z['paint'], atol=2e-6)
  assert_allclose(host(u.cic_paint_2d(zz, z['pos'], weight=z['w'])),
                  z['paint_w'], atol=2e-6)
  assert_allclose(
      host(u.cic_paint_2d(zz, z['pos'], weight=z['w'], mask=z['mask'])),
      z['paint_wm'], atol=2e-6)
  assert_allclose(
      host(u.cic_paint_2d(np.zeros((1, 24, 16), np.float32), z['pos_rect'])),
      z['paint_rect'], atol=2e-6)


def test_cic_paint_2d_out_of_range(fpm):
  """nx < ny: the reference's x indices wrap by ny and can leave the mesh;
  those deposits are reported, not written out of bounds."""
  from flowpm_b200 import _lib
  part = np.array([[[10.25, 3.5], [2.5, 3.5]]], np.float32)
  with pytest.raises(_lib.FlowPMError) as e:
    fpm.utils.cic_paint_2d(np.zeros((1, 8, 16), np.float32), part)
  assert e.value.code == _lib.FPM_ERR_RANGE


def test_density_plane_golden(fpm):
  z, nb = golden('planes'), golden('nbody')
  st = nb['n32_final']
  out = fpm.raytracing.density_plane(st, 32, 16., 8., 48,
                                     shift=np.array([0.3, 0.7, 0.],
                                                    np.float32))
  assert_allclose(host(out), z['dp_plane'], rtol=1e-5, atol=1e-5)
  out = fpm.raytracing.density_plane(st, 32, 26., 4., 40, rotation=z['dp_rot'],
                                     shift=np.array([0.1, 0.2, 0.5],
                                                    np.float32))
  assert_allclose(host(out), z['dp_plane_rot'], rtol=1e-5, atol=1e-5)


def test_density_planes_many_slabs(fpm):
  """70 slabs (two library calls) in one call equal the single-slab calls
  and, summed over a partition of z, conserve the painted mass."""
  nb = golden('nbody')
  st = nb['n32_final']
  centers = np.linspace(0.25, 31.75, 70)
  w = 32. / 70.
  many = host(fpm.raytracing.density_planes(st, 32, centers, w, 32))
  assert many.shape == (1, 70, 32, 32)
  for i in (0, 33, 69):
    one = host(fpm.raytracing.density_plane(st, 32, centers[i], w, 32))
    assert_allclose(many[:, i], one, rtol=1e-6, atol=1e-6)
  # un-normalise and sum: every particle with 0 < z <= 32 (mod) counted once
  z = np.asarray(st[0][0, :, 2])
  inside = ((z > 0) & (z <= 32)).sum()
  assert abs((many * w).sum() - inside) < 1e-2 * inside


def test_planes_gradients(fpm):
  """Positions and weights: the adjoints against the oracle's autograd."""
  z, nb = golden('planes'), golden('nbody')
  g = np.random.default_rng(3).standard_normal((2, 24, 24)).astype(np.float32)
  p = torch.tensor(z['pos'], device='cuda', requires_grad=True)
  w = torch.tensor(z['w'], device='cuda', requires_grad=True)
  out = fpm.utils.cic_paint_2d(torch.zeros((2, 24, 24), device='cuda'), p,
                               weight=w, mask=z['mask'])
  gp, gw = torch.autograd.grad((out * torch.tensor(g, device='cuda')).sum(),
                               (p, w))
  pr = torch.tensor(z['pos'], dtype=torch.float64, requires_grad=True)
  wr = torch.tensor(z['w'], dtype=torch.float64, requires_grad=True)
  ref = opl.cic_paint_2d(torch.zeros((2, 24, 24), dtype=torch.float64), pr,
                         weight=wr, mask=z['mask'])
  rp, rw = torch.autograd.grad((ref * torch.tensor(g, dtype=torch.float64))
                               .sum(), (pr, wr))
  assert_allclose(host(gp), rp.numpy(), rtol=1e-4, atol=1e-5)
  assert_allclose(host(gw), rw.numpy(), rtol=1e-4, atol=1e-5)
  st = torch.tensor(nb['n32_final'], device='cuda')
  X = st[0].clone().requires_grad_(True)
  s = torch.stack((X, st[1], st[2]))
  rot, sh = z['dp_rot'], np.array([0.1, 0.2, 0.5], np.float32)
  gpl = np.random.default_rng(4).standard_normal((1, 40, 40)).astype(
      np.float32)
  out = fpm.raytracing.density_plane(s, 32, 26., 4., 40, rotation=rot,
                                     shift=sh)
  (gx,) = torch.autograd.grad((out * torch.tensor(gpl, device='cuda')).sum(),
                              X)
  # FP32 oracle on the same positions: the slab and cell decisions match
  Xr = torch.tensor(nb['n32_final'][0], requires_grad=True)
  sr = torch.stack((Xr, torch.tensor(nb['n32_final'][1]),
                    torch.tensor(nb['n32_final'][2])))
  ref = opl.density_plane(sr, 32, 26., 4., 40, rotation=rot, shift=sh)
  (rx,) = torch.autograd.grad((ref * torch.tensor(gpl)).sum(), Xr)
  bad = ~np.isclose(host(gx), rx.numpy(), rtol=1e-3, atol=1e-4)
  # a particle on a slab or cell edge may round to the other side
  assert bad.any(axis=-1).mean() < 1e-3, bad.any(axis=-1).sum()
