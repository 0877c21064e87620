"""The binned forward step (fpm_plan_set_binning: particles kept sorted by
force-mesh cell, tiles painted through shared memory, re-sorted every few
steps) through the C ABI, against the reference's fixtures and against the
lattice walk on the same inputs.  The two orders sum the density's FP32
deposits differently, so the bar between them is FP32 rounding carried
through the run; against the reference it is the lattice walk's bar."""
import numpy as np
import pytest
import torch
from numpy.testing import assert_allclose

from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def fpm(cuda):
  import flowpm_b200
  return flowpm_b200


def host(t):
  return t.detach().cpu().numpy()


def _plan(dims, flags=0):
  from flowpm_b200._plans import get_plan
  return get_plan(dims, flags=flags)


@pytest.fixture
def binned(fpm):
  """Sets binning on cached plans; resets every plan it touched."""
  touched = []

  def set_(dims, tile, every, flags=0, mode=1, adj_every=0):
    p = _plan(dims, flags)
    p.set_binning(tile, every, mode)
    p.set_adjoint_binning(adj_every) if flags else None
    touched.append(p)
  yield set_
  for p in touched:
    if p.adjoint_binning:
      p.set_adjoint_binning(0)
    p.set_binning(0)


MODES = [(8, 1, 1), (16, 3, 1), (8, 4, 0), (16, 2, 0), (16, 1, 3), (8, 1, 3),
         (16, 1 << 20, 1)]


@pytest.mark.parametrize('tile,every,mode', MODES)
def test_binned_nbody_16_golden(fpm, binned, tile, every, mode):
  z, l = golden('nbody'), golden('lpt')
  c = fpm.cosmology.Planck15()
  stages = z['stages']
  ref = host(fpm.nbody(c, l['n16_init_o1'], stages, 16))
  binned([(16, 16, 16, 1)], tile, every, mode=mode)
  st = host(fpm.nbody(c, l['n16_init_o1'], stages, 16))
  assert_allclose(st, z['n16_b1_final'], atol=1e-4)
  assert_allclose(st, ref, atol=2e-5)
  # pm_nc_factor 2: 32^3 force mesh
  binned([(16, 16, 16, 2)], tile, every, mode=mode)
  st2 = host(fpm.nbody(c, l['n16_init_o1'], stages, 16, pm_nc_factor=2))
  assert_allclose(st2, z['n16_b2_final'], atol=1e-4)
  # intermediate states, written through the carried Lagrangian index
  inter = fpm.nbody(c, l['n16_init_o1'], stages[:4], 16,
                    return_intermediate_states=True)
  assert_allclose(np.stack([host(s) for _, s in inter]), z['n16_inter'],
                  atol=2e-5)


def test_binned_c1_density(fpm, binned, capsys):
  """C1 (32^3, box 100, 2LPT at 0.1, 10 stages): final density against the
  reference (bar 1e-4) and against the lattice walk."""
  z, l = golden('nbody'), golden('lpt')
  c = fpm.cosmology.Planck15()
  stages = z['stages']
  s0 = fpm.lpt_init(c, l['n32_linear'], 0.1, order=2)
  zeros = lambda: torch.zeros((1, 32, 32, 32))
  walk = host(fpm.cic_paint(zeros(), fpm.nbody(c, s0, stages, 32)[0]))
  errs = {}
  for tile, every, mode in ((8, 1, 1), (16, 2, 1), (8, 5, 0), (16, 2, 0),
                            (16, 1, 3)):
    binned([(32, 32, 32, 1)], tile, every, mode=mode)
    rho = host(fpm.cic_paint(zeros(), fpm.nbody(c, s0, stages, 32)[0]))
    e = errs[(tile, every, mode)] = (rel_l2(rho, z['n32_rho']),
                                     rel_l2(rho, walk))
    assert e[0] <= 1e-4
    assert e[1] <= 1e-5
  with capsys.disabled():
    print('\n  binned C1 density rel-L2 (vs reference, vs lattice walk): %s'
          % {k: '%.1e / %.1e' % v for k, v in errs.items()})


def test_binned_rectangular(fpm, binned):
  z = golden('nbody')
  c = fpm.cosmology.Planck15(Omega_c=0.30, Omega_b=0.045, h=0.70,
                             sigma8=0.75, n_s=0.96)
  s0 = fpm.lpt_init(c, z['rect_linear'], 0.1, order=2)
  # 8 x 8 x 24 lattice: force mesh 16 x 16 x 48 with pm_nc_factor 2
  ref = host(fpm.nbody(c, s0, z['stages'], [8, 8, 24], pm_nc_factor=2))
  for mode in (0, 1):
    binned([(8, 8, 24, 2)], 8, 2, mode=mode)
    st = host(fpm.nbody(c, s0, z['stages'], [8, 8, 24], pm_nc_factor=2))
    assert_allclose(st, ref, atol=2e-5)


def test_binned_batch_uneven(fpm):
  """Several runs of different shapes and step counts in one plan (the
  runs' chains on side streams), binned against the lattice walk."""
  rng = np.random.default_rng(3)
  specs, states = [], []
  for n, T in ((32, 6), (32, 4), (64, 5), (16, 7)):
    c = fpm.cosmology.Planck15(Omega_c=float(rng.uniform(0.2, 0.35)))
    lin = rng.standard_normal((1, n, n, n)).astype(np.float32) * 0.5
    specs.append(dict(nc=n, cosmo=c, stages=np.linspace(0.1, 1.0, T + 1)))
    states.append(fpm.lpt_init(c, lin, 0.1, order=2))
  r = fpm.BatchRunner(specs)
  try:
    r.load(states)
    r.run()
    ref = [host(s) for s in r.results()]
    # (16, 1, 3): the mix's runs take different step counts, so the flow
    # mode falls back to re-sorting every step
    for tile, every, mode in ((8, 1, 1), (16, 2, 1), (8, 2, 0), (16, 1, 3)):
      r.set_binning(tile, every, mode)
      r.load(states)
      r.run()
      got = [host(s) for s in r.results()]
      for a, b in zip(got, ref):
        assert_allclose(a, b, atol=3e-5)
      assert r.status() == 0
  finally:
    r.close()


@pytest.mark.parametrize('store', [False, True], ids=['rebuilt', 'potential'])
def test_binned_forward_gradient(fpm, binned, store):
  """The reverse sweep after a binned forward (checkpoints written through
  the carried index) gives the gradient of the lattice-walk forward."""
  rng = np.random.default_rng(21)
  nc = [16, 16, 16]
  lin = rng.standard_normal([1] + nc) * 0.6
  stages = np.linspace(0.1, 1.0, 6)
  target = rng.standard_normal([1] + nc) + 1.0
  c = fpm.cosmology.Planck15()

  def grad():
    x = torch.tensor(lin, dtype=torch.float32, device='cuda',
                     requires_grad=True)
    st = fpm.nbody(c, fpm.lpt_init(c, x, 0.1, order=2), stages, nc,
                   checkpoint_every=2, store_potential=store)
    rho = fpm.cic_paint(torch.zeros([1] + nc, device='cuda'), st[0])
    loss = ((rho - torch.tensor(target, dtype=torch.float32,
                                device='cuda'))**2).sum()
    (g,) = torch.autograd.grad(loss, x)
    return host(g)

  from flowpm_b200 import _lib
  g0 = grad()
  for mode in (0, 1, 3):
    binned([(16, 16, 16, 1)], 8, 2, flags=_lib.FPM_PLAN_ADJOINT, mode=mode)
    g1 = grad()
    assert rel_l2(g1, g0) < 1e-4


@pytest.mark.parametrize('nc,adj_every,mode', [(16, 1, 1), (16, 3, 2),
                                                (32, 2, 1), (32, 1, 2),
                                                (32, 2, 3)])
def test_binned_reverse_sweep(fpm, binned, nc, adj_every, mode):
  """The potential-tape reverse sweep over the binned particle order
  (fpm_plan_set_adjoint_binning: sorted state and cotangents, re-sorted
  every adj_every positions, results back in Lagrangian order) gives the
  lattice walk's gradient, with checkpoints and with the cotangent of the
  final force (the loss reads F); the forward binned too (mode 1) or on
  the lattice walk (mode 2, FPM_BIN_WALK)."""
  from flowpm_b200 import _lib
  rng = np.random.default_rng(nc + adj_every)
  dims = [nc] * 3
  lin = rng.standard_normal([1] + dims) * 0.6
  stages = np.linspace(0.1, 1.0, 8)
  target = rng.standard_normal([1] + dims) + 1.0
  c = fpm.cosmology.Planck15()

  def grad():
    x = torch.tensor(lin, dtype=torch.float32, device='cuda',
                     requires_grad=True)
    st = fpm.nbody(c, fpm.lpt_init(c, x, 0.1, order=2), stages, dims,
                   checkpoint_every=3, store_potential=True)
    rho = fpm.cic_paint(torch.zeros([1] + dims, device='cuda'), st[0])
    loss = ((rho - torch.tensor(target, dtype=torch.float32,
                                device='cuda'))**2).sum()
    loss = loss + 1e-3 * (st[2]**2).sum() + 1e-2 * (st[1]**2).sum()
    (g,) = torch.autograd.grad(loss, x)
    return host(g)

  g0 = grad()
  binned([tuple(dims) + (1,)], 8, 2, flags=_lib.FPM_PLAN_ADJOINT,
         mode=mode, adj_every=adj_every)
  g1 = grad()
  assert np.isfinite(g1).all()
  assert rel_l2(g1, g0) < 1e-4, rel_l2(g1, g0)


def test_adjoint_binning_needs_binning(fpm):
  from flowpm_b200 import _lib
  from flowpm_b200._plans import Plan
  p = Plan([(16, 16, 16, 1)], flags=_lib.FPM_PLAN_ADJOINT)
  q = Plan([(16, 16, 16, 1)])
  try:
    with pytest.raises(_lib.FlowPMError) as e:
      p.set_adjoint_binning(2)  # binning is off
    assert e.value.code == _lib.FPM_ERR_STATE
    q.set_binning(8, 1)
    with pytest.raises(_lib.FlowPMError) as e:
      q.set_adjoint_binning(2)  # not an adjoint plan
    assert e.value.code == _lib.FPM_ERR_STATE
    p.set_binning(8, 1)
    p.set_adjoint_binning(2)
    p.set_binning(16, 1)  # kept across a change of tile
    p.set_adjoint_binning(0)
  finally:
    p.close()
    q.close()


def test_binning_refused_when_tiles_do_not_fit(fpm):
  from flowpm_b200 import _lib
  from flowpm_b200._plans import Plan
  p = Plan([(12, 12, 12, 1)])
  try:
    with pytest.raises(_lib.FlowPMError) as e:
      p.set_binning(8, 1)
    assert e.value.code == _lib.FPM_ERR_UNSUPPORTED
    with pytest.raises(_lib.FlowPMError):
      p.set_binning(5, 1)
  finally:
    p.close()


def test_autotune_picks_and_caches(fpm):
  """fpm_plan_autotune times every configuration on scratch copies of the
  state, leaves the fastest on the plan (which then gives the lattice
  walk's state to rounding) and reuses the cached choice for an equal
  plan."""
  from flowpm_b200 import _lib, tfbackground
  from flowpm_b200._plans import Plan
  l = golden('lpt')
  c = fpm.cosmology.Planck15()
  stages = np.linspace(0.1, 1.0, 11)
  s0 = fpm.lpt_init(c, l['n32_linear'], 0.1, order=2)
  nc = [32, 32, 32]
  st = _lib.stream_ptr()
  coefs = tfbackground.nbody_coefficients(c, stages)

  def plan_with_steps():
    p = Plan([(32, 32, 32, 1)])
    _lib.call('fpm_nbody_set_steps', p.handle, 10, _lib.ivec([10]),
              _lib.dvec(coefs.ravel()), _lib.dvec([1.5 * c.Omega_m]), st)
    return p

  d0 = fpm.tfpm._to_disp(s0[0], nc).reshape(-1, 3).contiguous()
  p0 = s0[1].reshape(-1, 3).contiguous()
  keep = (d0.clone(), p0.clone())
  p = plan_with_steps()
  q = plan_with_steps()
  try:
    choice, ms = p.autotune(d0, p0, reps=2, retune=True)
    assert torch.equal(d0, keep[0]) and torch.equal(p0, keep[1])
    assert all(v is not None and v > 0 for v in ms.values()), ms
    best = min(ms, key=lambda k: ms[k])
    names = {'walk': (0, 1, 1), 'chunks16/4': (16, 4, 1),
             'chunks16/6': (16, 6, 1), 'chunks16/10': (16, 10, 1),
             'chunks16/16': (16, 16, 1), 'chunks16/once': (16, 1 << 20, 1),
             'flow16': (16, 1, 3), 'tiles16/4': (16, 4, 0)}
    assert choice == names[best]
    outs = {}
    for plan in (p, q):  # p tuned, q the lattice walk
      d, pm, f = d0.clone(), p0.clone(), torch.empty_like(d0)
      _lib.call('fpm_nbody_run', plan.handle, _lib.ptr(d), _lib.ptr(pm),
                _lib.ptr(f), None, 0, None, 0, st)
      outs[plan is p] = (host(d), host(pm), host(f))
    for a, b in zip(outs[True], outs[False]):
      assert_allclose(a, b, atol=3e-5)
    choice2, ms2 = q.autotune(d0, p0)
    assert choice2 == choice and all(v is None for v in ms2.values())
  finally:
    p.close()
    q.close()
