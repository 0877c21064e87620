"""The fused Fourier solve (power-of-two meshes of 16 to 128 cells per axis)
and the x-pass solve (256 or 512 cells along x: batched cuFFT plane
transforms around the x-pass kernel) against the three-dimensional cuFFT
path of the same library (plan flag FPM_PLAN_CUFFT): forces of random
particle sets through fpm_force, for single and batched plans whose runs
mix the paths.  (The oracle comparisons of the force, the leapfrog and the
density go through the fused solve wherever the mesh qualifies, e.g. every
16^3 / 32^3 golden case.)"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def fpm(cuda):
  import flowpm_b200
  return flowpm_b200


def host(t):
  return t.detach().cpu().numpy()


SHAPES = [
    [(16, 16, 16, 1)],
    [(32, 64, 16, 1)],
    [(64, 64, 64, 2)],
    [(128, 128, 128, 1)],
    # runs: fused 32^3 x2, cuFFT 24^3, fused 16x32x64 on a 2x finer mesh
    [(32, 32, 32, 1), (32, 32, 32, 1), (24, 24, 24, 1), (16, 32, 64, 2)],
    # x pass: 256^3; 512 along x; fused, x pass x2 (one on a 2x finer
    # mesh) and cuFFT runs in one plan
    [(256, 256, 256, 1)],
    [(512, 16, 16, 1)],
    # x pass on rectangular planes (512 x 256 and 256 x 512 cells)
    [(256, 512, 256, 1), (256, 256, 512, 1)],
    [(32, 32, 32, 1), (256, 16, 32, 1), (256, 16, 32, 1), (24, 24, 24, 1),
     (128, 24, 8, 2)],
    # three 128^3: the cuFFT plan takes the tiled gradient stencil (enough
    # tiles), the fused solve its own plane stencils
    [(128, 128, 128, 1)] * 3,
]


def _forces(dims, flags, r_split, disp, ffac):
  from flowpm_b200 import _lib
  from flowpm_b200._plans import Plan
  plan = Plan(dims, r_split=r_split, flags=flags)
  try:
    f = torch.empty_like(disp)
    _lib.call('fpm_force', plan.handle, _lib.ptr(disp), _lib.dvec(ffac),
              _lib.ptr(f), _lib.stream_ptr())
    torch.cuda.synchronize()
    return f
  finally:
    plan.close()


@pytest.mark.parametrize('dims', SHAPES, ids=lambda d: 'x'.join(
    '%d%d%d/%d' % t for t in d))
@pytest.mark.parametrize('opt', ['plain', 'deconv_split', 'order0'])
def test_fused_solve_matches_cufft(fpm, dims, opt):
  from flowpm_b200 import _lib
  flags, r_split = {
      'plain': (0, 0.0),
      'deconv_split': (_lib.FPM_PLAN_CIC_DECONV, 1.5),
      'order0': (_lib.FPM_PLAN_GRAD_ORDER0, 0.0),
  }[opt]
  g = torch.Generator(device='cpu').manual_seed(11)
  npart = sum(a * b * c for a, b, c, _ in dims)
  disp = ((torch.rand((npart, 3), generator=g) - 0.5) * 6).cuda()
  ffac = [0.47 + 0.01 * i for i in range(len(dims))]
  fused = _forces(dims, flags, r_split, disp, ffac)
  ref = _forces(dims, flags | _lib.FPM_PLAN_CUFFT, r_split, disp, ffac)
  off = 0
  for a, b, c, _ in dims:
    n = a * b * c
    x, y = host(fused[off:off + n]), host(ref[off:off + n])
    assert np.isfinite(x).all()
    print('fused vs cufft', (a, b, c), opt, rel_l2(x, y))
    assert rel_l2(x, y) < 1e-5, (a, b, c, rel_l2(x, y))
    off += n



def test_full_size_force_paths(fpm):
  """At the C5 mesh (512^3, 134M particles displaced by N(0, 2) cells): the
  x-pass solve (cuFFT plane transforms around the x-pass kernel, tiled
  stencil) and the three-dimensional cuFFT path agree, and the total force
  vanishes -- CIC paint and readout with the same weights, a symmetric
  transfer function and an antisymmetric stencil conserve momentum -- to
  FP32 rounding."""
  from flowpm_b200 import _lib
  n = 512
  g = torch.Generator(device='cuda').manual_seed(17)
  disp = torch.randn((n**3, 3), generator=g, device='cuda') * 2.0
  ffac = [0.45]
  fx = _forces([(n, n, n, 1)], 0, 0.0, disp, ffac)
  fc = _forces([(n, n, n, 1)], _lib.FPM_PLAN_CUFFT, 0.0, disp, ffac)
  del disp
  err = (torch.linalg.vector_norm(fx - fc) /
         torch.linalg.vector_norm(fc)).item()
  assert torch.isfinite(fx).all()
  print('512^3 x pass vs 3-D cuFFT: rel-L2 %.2e' % err)
  assert err < 1e-5, err
  for f in (fx, fc):
    tot = f.double().sum(dim=0).abs().max().item()
    scale = f.double().abs().sum(dim=0).max().item()
    assert tot < 1e-5 * scale, (tot, scale)
