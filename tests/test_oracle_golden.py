"""Pins the CPU oracle to the reference: golden fixtures produced by the
reference's own source (tests/golden/make_golden.py) and the reference's
FP64 background oracle flowpm/legacy_background.py, at the reference test
tolerances (tests/test_tfbackground.py, test_tfpower.py, test_utils.py)."""
import numpy as np
import pytest
import torch
from numpy.testing import assert_allclose

from conftest import golden, pk_table, rel_l2
from oracle import background, pm, power

ALT = dict(Omega_c=0.30, Omega_b=0.045, h=0.70, sigma8=0.75, n_s=0.96)
BG_FUNCS = ['E', 'dEa', 'Omega_m_a', 'Omega_de_a', 'D1', 'D2', 'D1f', 'D2f',
            'f1', 'f2', 'Gf', 'Gf2', 'gf', 'gf2']


@pytest.mark.parametrize('tag,kw', [('planck15', {}), ('alt', ALT)])
def test_background_matches_reference_fp32(tag, kw):
  z = golden('background')
  b = background.Background(kw, dtype=np.float32)
  for fn in BG_FUNCS:
    got = getattr(b, fn)(z['a_eval'])
    assert_allclose(got, z['%s_%s' % (tag, fn)], rtol=1e-6, err_msg=fn)
  ode = b.ode()
  for key in ['a', 'D1', 'D1f', 'F1p', 'D2', 'D2f', 'F2p']:
    assert_allclose(ode[key], z['%s_ode_%s' % (tag, key)], rtol=1e-6)


@pytest.mark.parametrize('dtype', [np.float32, np.float64])
def test_background_vs_legacy_fp64(dtype):
  """tests/test_tfbackground.py tolerances against MatterDominated(0.3075)."""
  z = golden('background')
  b = background.Background({}, dtype=dtype)
  a3 = z['legacy_a3']
  assert_allclose(b.E(a3), z['legacy_E'], rtol=1e-4)
  assert_allclose(b.dEa(a3), z['legacy_Eprime'], rtol=1e-4)
  assert_allclose(b.Omega_m_a(a3), z['legacy_Om'], rtol=1e-4)
  a = z['legacy_a']
  pairs = [('D1', 'D1'), ('D2', 'D2'), ('D1f', 'gp'), ('D2f', 'gp2'),
           ('f1', 'f1'), ('f2', 'f2'), ('Gf', 'Gf'), ('Gf2', 'Gf2'),
           ('gf', 'gf'), ('gf2', 'gf2')]
  for mine, ref in pairs:
    assert_allclose(getattr(b, mine)(a), z['legacy_' + ref], rtol=1e-2,
                    err_msg=mine)


def test_linear_power_matches_reference():
  z = golden('power')
  for tag, kw in [('planck15', {}), ('alt', ALT)]:
    b = background.Background(kw, dtype=np.float32)
    assert_allclose(power.linear_matter_power(b, z['k']), z[tag + '_pk'],
                    rtol=1e-5)
    assert_allclose(power.linear_matter_power(b, z['k'], a=0.5),
                    z[tag + '_pk_a0p5'], rtol=1e-5)
    assert_allclose(power.eisenstein_hu(b, z['k'], type='eisenhu'),
                    z[tag + '_T_eisenhu'], rtol=1e-5)


def test_linear_power_vs_nbodykit_table():
  """The data table is nbodykit's EH P(k) for astropy's Planck15 (not
  exactly the reference parameters): agreement within 3% on 1e-3..10."""
  z = golden('power')
  k = z['nbodykit_k']
  sel = (k >= 1e-3) & (k <= 10)
  b = background.Background({}, dtype=np.float64)
  assert_allclose(power.linear_matter_power(b, k[sel]), z['nbodykit_pk'][sel],
                  rtol=3e-2)


def test_kernels_match_reference():
  z = golden('kernels')
  for tag, shape in [('c8', [8, 8, 8]), ('r4610', [4, 6, 10])]:
    kv = pm.fftk(shape, symmetric=False)
    kvs = pm.fftk(shape, symmetric=True)
    for d in range(3):
      assert np.array_equal(kv[d], z['%s_fftk_%d' % (tag, d)])
      assert np.array_equal(kvs[d], z['%s_fftk_sym_%d' % (tag, d)])
      assert np.array_equal(pm.gradient_kernel(kv, d),
                            z['%s_grad1_%d' % (tag, d)])
      assert np.array_equal(pm.gradient_kernel(kv, d, order=0),
                            z['%s_grad0_%d' % (tag, d)])
    assert np.array_equal(pm.laplace_kernel(kv), z[tag + '_laplace'])
    assert np.array_equal(pm.longrange_kernel(kv, 1.3),
                          z[tag + '_longrange_r1p3'])
    assert pm.longrange_kernel(kv, 0) == 1.
    assert np.array_equal(pm.cic_compensation(kv), z[tag + '_ciccomp'])
    # reference quirk: the Green's function is 1 at k = 0
    assert pm.laplace_kernel(kv)[0, 0, 0] == 1.


def test_cic_matches_reference():
  z = golden('cic')
  pos, w = torch.tensor(z['pos']), torch.tensor(z['wts'])
  m = pm.cic_paint(torch.zeros(2, 16, 16, 16), pos, w)
  assert_allclose(m.numpy(), z['paint_w'], atol=1e-6)
  m = pm.cic_paint(torch.zeros(2, 16, 16, 16), pos)
  assert_allclose(m.numpy(), z['paint_1'], atol=1e-6)
  r = pm.cic_readout(torch.tensor(z['base']), pos)
  assert_allclose(r.numpy(), z['readout'], rtol=1e-6)
  m = pm.cic_paint(torch.zeros(1, 8, 6, 10), torch.tensor(z['pos_rect']))
  assert_allclose(m.numpy(), z['paint_rect'], atol=1e-6)
  r = pm.cic_readout(torch.tensor(z['base_rect']), torch.tensor(z['pos_rect']))
  assert_allclose(r.numpy(), z['readout_rect'], rtol=1e-5, atol=1e-6)


def test_fft_roundtrip_fp64():
  """tests/test_utils.py:51-61: r2c3d -> c2r3d is the identity, rtol 1e-9."""
  z = golden('cic')
  x = torch.tensor(z['rt_in'])
  c = pm.r2c3d(x)
  assert_allclose(c.numpy(), z['rt_k'], rtol=1e-9, atol=1e-9)
  assert_allclose(pm.c2r3d(c).numpy(), z['rt_in'], rtol=1e-9)


def test_lpt_matches_reference():
  z = golden('lpt')
  lin = torch.tensor(z['n16_linear'])
  lk = pm.r2c3d(lin)
  grid = pm.lattice([16] * 3, 1)
  assert_allclose(pm.lpt1(lk, grid).numpy(), z['n16_lpt1'], atol=1e-5)
  assert_allclose(pm.c2r3d(pm.lpt2_source(lk)).numpy(), z['n16_lpt2src'],
                  atol=1e-5)
  b = background.Background({}, dtype=np.float32)
  for order in (1, 2):
    s = pm.lpt_init(b, lin, 0.1, order=order)
    assert_allclose(s.numpy(), z['n16_init_o%d' % order], atol=1e-5)
  s = pm.lpt_init(b, torch.tensor(z['n32_linear']), 0.1, order=2)
  assert_allclose(s.numpy(), z['n32_init_o2'], atol=2e-5)


def test_linear_field_matches_reference():
  z = golden('lpt')
  for nc, bs in [(16, 50.), (32, 100.)]:
    lin = pm.linear_field_from_white(torch.tensor(z['n%d_white' % nc]), bs,
                                     pk_table())
    ref = z['n%d_linear' % nc]
    assert_allclose(lin.numpy(), ref, atol=1e-5 * np.abs(ref).max())


def test_force_kick_drift_match_reference():
  z, l = golden('nbody'), golden('lpt')
  b = background.Background({}, dtype=np.float32)
  s0 = torch.tensor(l['n16_init_o1'])
  assert_allclose(pm.force(b, s0, 16).numpy(), z['n16_force'], atol=2e-5)
  assert_allclose(pm.kick(b, s0, 0.1, 0.1, 0.12).numpy(), z['n16_kick'],
                  atol=1e-6)
  assert_allclose(pm.drift(b, s0, 0.1, 0.12, 0.15).numpy(), z['n16_drift'],
                  atol=1e-6)


def test_nbody_matches_reference():
  z, l = golden('nbody'), golden('lpt')
  b = background.Background({}, dtype=np.float32)
  stages = z['stages']
  st = pm.nbody(b, torch.tensor(l['n16_init_o1']), stages, 16)
  assert_allclose(st.numpy(), z['n16_b1_final'], atol=5e-5)
  st2 = pm.nbody(b, torch.tensor(l['n16_init_o1']), stages, 16,
                 pm_nc_factor=2)
  assert_allclose(st2.numpy(), z['n16_b2_final'], atol=5e-5)
  inter = pm.nbody(b, torch.tensor(l['n16_init_o1']), stages[:4], 16,
                   return_intermediate_states=True)
  assert [a for a, _ in inter] == list(z['n16_inter_a'])
  assert_allclose(np.stack([s.numpy() for _, s in inter]), z['n16_inter'],
                  atol=2e-5)
  ba = background.Background(ALT, dtype=np.float32)
  sr = pm.lpt_init(ba, torch.tensor(z['rect_linear']), 0.1, order=2)
  assert_allclose(sr.numpy(), z['rect_init'], atol=1e-5)
  assert_allclose(pm.nbody(ba, sr, stages, [8, 8, 24]).numpy(),
                  z['rect_final'], atol=5e-5)
  st = pm.nbody(b, torch.tensor(l['n32_init_o2']), stages, 32)
  assert_allclose(st.numpy(), z['n32_final'], atol=1e-4)
  rho = pm.cic_paint(torch.zeros(1, 32, 32, 32), st[0])
  assert rel_l2(rho.numpy(), z['n32_rho']) < 1e-5


def test_power_spectrum_matches_reference():
  z = golden('pk')
  for tag in ['rho32', 'lin16']:
    bs = float(z[tag + '_boxsize'])
    kb, p = pm.power_spectrum(torch.tensor(z[tag + '_field']), kmin=0.1,
                              dk=0.05, boxsize=np.array([bs] * 3))
    assert_allclose(kb, z[tag + '_k'], rtol=1e-12)
    assert_allclose(p.numpy(), z[tag + '_pk'], rtol=2e-5)


def test_known_answers():
  """Self-derived KATs: weights of a particle sum to its mass, an integer
  position paints a single cell, readout of a linear ramp is exact away
  from the wrap, periodic wrap at N - eps, D1 = a for Omega_m = 1."""
  part = torch.tensor([[[3.25, 7.5, 1.125]]])
  m = pm.cic_paint(torch.zeros(1, 8, 8, 8), part, torch.tensor([[2.5]]))
  assert abs(float(m.sum()) - 2.5) < 1e-6
  m = pm.cic_paint(torch.zeros(1, 8, 8, 8), torch.tensor([[[2., 3., 4.]]]))
  assert float(m[0, 2, 3, 4]) == 1.0 and float(m.sum()) == 1.0
  ramp = torch.arange(8, dtype=torch.float32).reshape(1, 8, 1, 1).expand(
      1, 8, 8, 8).contiguous()
  r = pm.cic_readout(ramp, torch.tensor([[[2.3, 5.5, 6.7]]]))
  assert abs(float(r) - 2.3) < 1e-6
  m = pm.cic_paint(torch.zeros(1, 8, 8, 8), torch.tensor([[[7.75, 0., 0.]]]))
  assert abs(float(m[0, 7, 0, 0]) - 0.25) < 1e-7
  assert abs(float(m[0, 0, 0, 0]) - 0.75) < 1e-7
  eds = background.Background(dict(Omega_c=1.0 - 0.0486), dtype=np.float64)
  a = np.linspace(0.1, 1.0, 7)
  assert_allclose(eds.D1(a), a, rtol=1e-4)


def test_single_plane_wave_lpt1():
  """1LPT of delta = A cos(k x) gives Psi_x = -A g(k) / k^2 sin(k x) with the
  4-point gradient g (flowpm/kernels.py:72-76)."""
  n, mode, A = 16, 2, 0.01
  x = np.arange(n)
  kx = 2 * np.pi * mode / n
  delta = np.broadcast_to(A * np.cos(kx * x)[:, None, None],
                          (n, n, n)).astype(np.float32)[None]
  lk = pm.r2c3d(torch.tensor(delta))
  psi = pm.lpt1(lk, pm.lattice([n] * 3, 1)).numpy()[0]
  g = (8 * np.sin(kx) - np.sin(2 * kx)) / 6
  expect = -A * g / kx**2 * np.sin(kx * x)
  got = psi[:, 0].reshape(n, n, n)[:, 0, 0]
  assert_allclose(got, expect, atol=1e-7)
  assert np.abs(psi[:, 1:]).max() < 1e-7


def test_oracle_pgd_golden():
  """PGD correction (flowpm/tfpm.py:222-270, :369-422, in nbody at
  :487-488): the oracle against the reference's own output, one call and
  a 9-step leapfrog at 16^3, pm_nc_factor 1 and 2."""
  z, l = golden('pgd'), golden('lpt')
  s0 = torch.tensor(l['n16_init_o1'])
  np.testing.assert_allclose(pm.pgd(s0, z['params'][0], 16).numpy(),
                             z['single'], atol=1e-5)
  np.testing.assert_allclose(
      pm.pgd(s0, z['params'][0], 16, pm_nc_factor=2).numpy(),
      z['single_b2'], atol=1e-5)
  b = background.Background({}, dtype=np.float32)
  out = pm.nbody(b, s0, z['stages'], 16, pgdparams=z['params']).numpy()
  np.testing.assert_allclose(out, z['final'], atol=2e-3)
  out = pm.nbody(b, s0, z['stages'], 16, pm_nc_factor=2,
                  pgdparams=z['params']).numpy()
  np.testing.assert_allclose(out, z['final_b2'], atol=5e-3)


def test_oracle_planes_golden():
  """2-D CIC paint (flowpm/utils.py:94-160) and density planes
  (flowpm/raytracing.py:49-109): the oracle against the reference's own
  output (weights, mask, the rectangular wrap by ny, shift, rotation)."""
  from oracle import planes
  z, nb = golden('planes'), golden('nbody')
  zz = np.zeros((2, 24, 24), np.float32)
  pos = torch.tensor(z['pos'])
  assert_allclose(planes.cic_paint_2d(zz, pos).numpy(), z['paint'],
                  atol=2e-6)
  assert_allclose(planes.cic_paint_2d(zz, pos, weight=z['w']).numpy(),
                  z['paint_w'], atol=2e-6)
  assert_allclose(
      planes.cic_paint_2d(zz, pos, weight=z['w'], mask=z['mask']).numpy(),
      z['paint_wm'], atol=2e-6)
  assert_allclose(
      planes.cic_paint_2d(np.zeros((1, 24, 16), np.float32),
                          torch.tensor(z['pos_rect'])).numpy(),
      z['paint_rect'], atol=2e-6)
  st = torch.tensor(nb['n32_final'])
  out = planes.density_plane(st, 32, 16., 8., 48,
                             shift=np.array([0.3, 0.7, 0.], np.float32))
  assert_allclose(out.numpy(), z['dp_plane'], rtol=1e-5, atol=1e-5)
  out = planes.density_plane(st, 32, 26., 4., 40, rotation=z['dp_rot'],
                             shift=np.array([0.1, 0.2, 0.5], np.float32))
  assert_allclose(out.numpy(), z['dp_plane_rot'], rtol=1e-5, atol=1e-5)


def test_nbody_checkpointed_same_as_nbody():
  """The step-checkpointed leapfrog used for FP64 tape gradients at full
  size computes what nbody computes, value and gradient."""
  rng = np.random.default_rng(3)
  b = background.Background({}, dtype=np.float64)
  lin = torch.tensor(rng.standard_normal((1, 8, 8, 8)) * 0.5,
                     requires_grad=True)
  stages = np.linspace(0.1, 1.0, 4)
  outs = []
  for fn in (pm.nbody, pm.nbody_checkpointed):
    s = fn(b, pm.lpt_init(b, lin, 0.1, order=2), stages, 8)
    (g,) = torch.autograd.grad((s[0]**2).sum() + s[1].sum(), lin)
    outs.append((s.detach().numpy(), g.numpy()))
  assert np.array_equal(outs[0][0], outs[1][0])
  assert_allclose(outs[0][1], outs[1][1], rtol=1e-12, atol=1e-12)
