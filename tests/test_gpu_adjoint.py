"""Gradients of the CUDA path: the hand-written adjoints (CIC paint / readout,
LPT, reverse-time nbody) against the oracle's autograd -- the stand-in for
the reference's TensorFlow tape gradient -- and against central finite
differences of the FP64 oracle.  Bar: 1e-3 relative."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import background as obg
from oracle import pm as opm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def fpm(cuda):
  import flowpm_b200
  return flowpm_b200


def host(t):
  return t.detach().cpu().numpy()


def test_paint_readout_adjoint(fpm):
  rng = np.random.default_rng(5)
  B, n, N = 2, 3000, 16
  pos = rng.random((B, n, 3)) * N
  pos[0, :4] = [[3, 4, 5], [0, 0, 0], [15, 2.5, 7], [7.5, 8, 9.25]]
  w = rng.random((B, n))
  M = rng.standard_normal((B, N, N, N))
  mesh = rng.standard_normal((B, N, N, N))
  r = rng.standard_normal((B, n))

  def ours():
    x = torch.tensor(pos, dtype=torch.float32, device='cuda',
                     requires_grad=True)
    ww = torch.tensor(w, dtype=torch.float32, device='cuda',
                      requires_grad=True)
    m = torch.tensor(mesh, dtype=torch.float32, device='cuda',
                     requires_grad=True)
    l1 = (fpm.cic_paint(torch.zeros((B, N, N, N), device='cuda'), x, ww) *
          torch.tensor(M, dtype=torch.float32, device='cuda')).sum()
    l2 = (fpm.cic_readout(m, x) *
          torch.tensor(r, dtype=torch.float32, device='cuda')).sum()
    gx1, gw = torch.autograd.grad(l1, (x, ww))
    gm, gx2 = torch.autograd.grad(l2, (m, x))
    return [host(t) for t in (gx1, gw, gm, gx2)]

  def oracle():
    x = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    ww = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    m = torch.tensor(mesh, dtype=torch.float64, requires_grad=True)
    l1 = (opm.cic_paint(torch.zeros((B, N, N, N), dtype=torch.float64), x,
                        ww) * torch.tensor(M)).sum()
    l2 = (opm.cic_readout(m, x) * torch.tensor(r)).sum()
    gx1, gw = torch.autograd.grad(l1, (x, ww))
    gm, gx2 = torch.autograd.grad(l2, (m, x))
    return [t.numpy() for t in (gx1, gw, gm, gx2)]

  for a, b in zip(ours(), oracle()):
    assert rel_l2(a, b) < 1e-5


@pytest.mark.parametrize('order', [1, 2])
def test_lpt_adjoint(fpm, order):
  rng = np.random.default_rng(order)
  N = 16
  lin = (rng.standard_normal((2, N, N, N)) * 0.5)
  R = rng.standard_normal((3, 2, N**3, 3))
  c = fpm.cosmology.Planck15()
  x = torch.tensor(lin, dtype=torch.float32, device='cuda',
                   requires_grad=True)
  s = fpm.lpt_init(c, x, 0.1, order=order)
  (g,) = torch.autograd.grad(
      (s * torch.tensor(R, dtype=torch.float32, device='cuda')).sum(), x)
  b64 = obg.Background({}, dtype=np.float64)
  xo = torch.tensor(lin, requires_grad=True)
  so = opm.lpt_init(b64, xo, 0.1, order=order)
  (go,) = torch.autograd.grad((so * torch.tensor(R)).sum(), xo)
  assert rel_l2(host(g), go.numpy()) < 1e-4


def _chi2_ours(fpm, lin, target, stages, nc, pm_nc_factor=1, ckpt=None,
               store=None, pgdparams=None):
  c = fpm.cosmology.Planck15()
  x = torch.tensor(lin, dtype=torch.float32, device='cuda',
                   requires_grad=True)
  s0 = fpm.lpt_init(c, x, stages[0], order=2)
  st = fpm.nbody(c, s0, stages, nc, pm_nc_factor=pm_nc_factor,
                 checkpoint_every=ckpt, store_potential=store,
                 pgdparams=pgdparams)
  rho = fpm.cic_paint(torch.zeros((1,) + tuple(nc), device='cuda'), st[0])
  loss = ((rho - torch.tensor(target, dtype=torch.float32,
                              device='cuda'))**2).sum()
  (g,) = torch.autograd.grad(loss, x)
  return float(loss), host(g)


def _chi2_oracle(lin, target, stages, nc, pm_nc_factor=1, grad=True,
                 pgdparams=None):
  b64 = obg.Background({}, dtype=np.float64)
  x = torch.tensor(lin, dtype=torch.float64, requires_grad=grad)
  s0 = opm.lpt_init(b64, x, stages[0], order=2)
  st = opm.nbody(b64, s0, stages, nc, pm_nc_factor=pm_nc_factor,
                 pgdparams=pgdparams)
  rho = opm.cic_paint(torch.zeros((1,) + tuple(nc), dtype=torch.float64),
                      st[0])
  loss = ((rho - torch.tensor(target))**2).sum()
  if not grad:
    return float(loss), None
  (g,) = torch.autograd.grad(loss, x)
  return float(loss.detach()), g.numpy()


@pytest.mark.parametrize('store', [False, True], ids=['rebuilt', 'potential'])
@pytest.mark.parametrize('pm_nc_factor,ckpt', [(1, None), (2, None), (1, 2)])
def test_nbody_adjoint_vs_tape(fpm, capsys, pm_nc_factor, ckpt, store):
  """d chi^2 / d linear field through lpt_init -> nbody -> cic_paint, with
  the force meshes of the reverse sweep rebuilt (paint + Fourier solve at
  the reconstructed positions) or taken from the stored potential of the
  forward (fpm_nbody_set_tape)."""
  rng = np.random.default_rng(21)
  nc = [16, 16, 16]
  lin = rng.standard_normal([1] + nc) * 0.6
  stages = np.linspace(0.1, 1.0, 6)
  rho0 = _rho_oracle(lin, stages, nc, pm_nc_factor)
  target = rho0 + rng.standard_normal(rho0.shape)
  lo, go = _chi2_oracle(lin, target, stages, nc, pm_nc_factor)
  l, g = _chi2_ours(fpm, lin, target, stages, nc, pm_nc_factor, ckpt, store)
  err = rel_l2(g, go)
  with capsys.disabled():
    print('\n  adjoint vs FP64 tape gradient (B=%d, ckpt=%s, stored '
          'potential %s): rel-L2 %.2e, loss %.6g vs %.6g' %
          (pm_nc_factor, ckpt, store, err, l, lo))
  assert err < 1e-3


@pytest.mark.parametrize('pm_nc_factor,ckpt', [(1, None), (2, None), (1, 2)])
def test_nbody_pgd_adjoint_vs_tape(fpm, capsys, pm_nc_factor, ckpt):
  """d chi^2 / d linear field through lpt_init -> nbody with the PGD
  correction after every drift (flowpm/tfpm.py:487-488) -> cic_paint,
  against the FP64 oracle's autograd; the reverse sweep takes the
  positions before each PGD move and the PGD potentials from the tape."""
  rng = np.random.default_rng(23)
  nc = [16, 16, 16]
  lin = rng.standard_normal([1] + nc) * 0.6
  stages = np.linspace(0.1, 1.0, 6)
  T = len(stages) - 1
  par = np.stack([np.linspace(0.3, 0.5, T), np.full(T, 0.4),
                  np.full(T, 2.0)], axis=1)
  rho0 = _rho_oracle(lin, stages, nc, pm_nc_factor, par)
  target = rho0 + rng.standard_normal(rho0.shape)
  lo, go = _chi2_oracle(lin, target, stages, nc, pm_nc_factor,
                        pgdparams=par)
  l, g = _chi2_ours(fpm, lin, target, stages, nc, pm_nc_factor, ckpt,
                    pgdparams=par)
  _, g_plain = _chi2_oracle(lin, target, stages, nc, pm_nc_factor)
  err = rel_l2(g, go)
  with capsys.disabled():
    print('\n  PGD adjoint vs FP64 tape gradient (B=%d, ckpt=%s): rel-L2 '
          '%.2e (the PGD term moves the gradient by %.2e), loss %.6g vs %.6g'
          % (pm_nc_factor, ckpt, err, rel_l2(g_plain, go), l, lo))
  assert err < 1e-3


def _rho_oracle(lin, stages, nc, pm_nc_factor=1, pgdparams=None):
  b64 = obg.Background({}, dtype=np.float64)
  s0 = opm.lpt_init(b64, torch.tensor(lin), stages[0], order=2)
  st = opm.nbody(b64, s0, stages, nc, pm_nc_factor=pm_nc_factor,
                 pgdparams=pgdparams)
  return opm.cic_paint(torch.zeros((1,) + tuple(nc), dtype=torch.float64),
                       st[0]).numpy()


def test_nbody_adjoint_vs_finite_differences(fpm, capsys):
  """Directional derivatives of chi^2 along random directions: adjoint
  gradient vs central differences of the FP64 oracle."""
  rng = np.random.default_rng(8)
  nc = [16, 16, 16]
  lin = rng.standard_normal([1] + nc) * 0.6
  stages = np.linspace(0.1, 1.0, 6)
  target = _rho_oracle(lin, stages, nc) + rng.standard_normal([1] + nc)
  _, g = _chi2_ours(fpm, lin, target, stages, nc)
  errs = []
  for _ in range(4):
    u = rng.standard_normal(lin.shape)
    u /= np.linalg.norm(u)
    eps = 1e-4
    lp, _ = _chi2_oracle(lin + eps * u, target, stages, nc, grad=False)
    lm, _ = _chi2_oracle(lin - eps * u, target, stages, nc, grad=False)
    fd = (lp - lm) / (2 * eps)
    ad = float(np.sum(g * u))
    errs.append(abs(ad - fd) / abs(fd))
  with capsys.disabled():
    print('\n  adjoint vs FP64 central differences: max rel %.2e' %
          max(errs))
  assert max(errs) < 1e-3


def test_batched_adjoint_matches_single(fpm, capsys):
  """Three 128^3 simulations in one plan against one plan per simulation.
  The batched run has enough (y, z) tiles for the tiled divergence stencil
  of the reverse sweep, the single ones take the generic stencil.  A zero
  linear field keeps every particle on its lattice site with zero force,
  so each paint and scatter sum has a single non-zero term and the two
  gradients agree up to the batched versus single LPT transforms; the
  random target still drives a generic adjoint force field through the
  stencil.  (With a random field, reduction-order noise moves particles
  across cell faces, where the CIC weight derivative jumps, and the
  gradients differ by ~1e-3.)"""
  rng = np.random.default_rng(31)
  nc = [128, 128, 128]
  lin = np.zeros([3] + nc, dtype=np.float32)
  target = rng.standard_normal([3] + nc).astype(np.float32)
  stages = np.linspace(0.1, 1.0, 4)
  c = fpm.cosmology.Planck15()

  def grad(l, t):
    x = torch.tensor(l, device='cuda', requires_grad=True)
    st = fpm.nbody(c, fpm.lpt_init(c, x, stages[0], order=2), stages, nc)
    rho = fpm.cic_paint(torch.zeros(x.shape, device='cuda'), st[0])
    loss = ((rho - torch.tensor(t, device='cuda'))**2).sum()
    return host(torch.autograd.grad(loss, x)[0])

  gb = grad(lin, target)
  assert np.isfinite(gb).all() and np.abs(gb).max() > 0
  errs = [rel_l2(gb[b:b + 1], grad(lin[b:b + 1], target[b:b + 1]))
          for b in range(3)]
  with capsys.disabled():
    print('\n  batched vs single adjoint at 128^3: rel l2 %s' %
          ', '.join('%.2e' % e for e in errs))
  assert max(errs) < 1e-5


def test_potential_tape_arguments(fpm):
  """fpm_nbody_set_tape: order-0 plans have no potential; a tape shorter
  than (steps + 1) positions is refused by the forward and the adjoint."""
  from flowpm_b200 import _lib
  from flowpm_b200._plans import Plan
  p0 = Plan([(16, 16, 16, 1)],
            flags=_lib.FPM_PLAN_ADJOINT | _lib.FPM_PLAN_GRAD_ORDER0)
  buf = torch.empty(16**3 * 3, device='cuda')  # 3 of the 4 positions
  try:
    assert _lib.lib.fpm_nbody_set_tape(p0.handle, _lib.ptr(buf),
                                     buf.numel()) == _lib.FPM_ERR_UNSUPPORTED
  finally:
    p0.close()
  plan = Plan([(16, 16, 16, 1)], flags=_lib.FPM_PLAN_ADJOINT)
  try:
    st = _lib.stream_ptr()
    T = 3
    coefs = np.full((1, T, 3), 0.01)
    _lib.call('fpm_nbody_set_steps', plan.handle, T, _lib.ivec([T]),
              _lib.dvec(coefs.ravel()), _lib.dvec([0.45]), st)
    d = torch.zeros((16**3, 3), device='cuda')
    p, f = torch.zeros_like(d), torch.zeros_like(d)
    assert _lib.lib.fpm_nbody_set_tape(plan.handle, _lib.ptr(buf),
                                       buf.numel()) == _lib.FPM_OK
    assert _lib.lib.fpm_nbody_run(plan.handle, _lib.ptr(d), _lib.ptr(p),
                                  _lib.ptr(f), None, 0, None, 0,
                                  st) == _lib.FPM_ERR_ARG
    assert _lib.lib.fpm_nbody_adjoint(
        plan.handle, _lib.ptr(d), _lib.ptr(p), _lib.ptr(f), _lib.ptr(d),
        _lib.ptr(p), None, None, 0, st) == _lib.FPM_ERR_ARG
    assert _lib.lib.fpm_nbody_set_tape(plan.handle, None, 0) == _lib.FPM_OK
  finally:
    plan.close()


def _run_adjoint(sims, d0, p0, lx0, lp0, tape, nc=(16, 16, 16), flags=0):
  """Forward + reverse sweep through the C ABI for simulations
  [(T, stages)] of mesh nc in one plan: returns dL/dX_0, dL/dp_0 and the
  rebuilt initial displacement and momentum."""
  from flowpm_b200 import _lib, tfbackground
  from flowpm_b200._plans import Plan
  n = int(np.prod(nc))
  B = len(sims)
  maxT = max(T for T, _ in sims)
  c = __import__('flowpm_b200').cosmology.Planck15()
  co = np.zeros((B, maxT, 3))
  for s, (T, stages) in enumerate(sims):
    co[s, :T] = tfbackground.nbody_coefficients(c, stages)
  plan = Plan([tuple(nc) + (1,)] * B, flags=_lib.FPM_PLAN_ADJOINT | flags)
  try:
    st = _lib.stream_ptr()
    _lib.call('fpm_nbody_set_steps', plan.handle, maxT,
              _lib.ivec([T for T, _ in sims]), _lib.dvec(co.ravel()),
              _lib.dvec([1.5 * c.Omega_m] * B), st)
    buf = None
    if tape:
      buf = torch.empty((maxT + 1) * B * n, device='cuda')
      _lib.call('fpm_nbody_set_tape', plan.handle, _lib.ptr(buf), buf.numel())
    d, p = d0.clone(), p0.clone()
    f = torch.empty_like(d)
    _lib.call('fpm_nbody_run', plan.handle, _lib.ptr(d), _lib.ptr(p),
              _lib.ptr(f), None, 0, None, 0, st)
    lx, lp = lx0.clone(), lp0.clone()
    _lib.call('fpm_nbody_adjoint', plan.handle, _lib.ptr(d), _lib.ptr(p),
              _lib.ptr(f), _lib.ptr(lx), _lib.ptr(lp), None, None, 0, st)
    torch.cuda.synchronize()
    return host(lx), host(lp), host(d), host(p)
  finally:
    plan.close()


def test_potential_tape_uneven_batch(fpm):
  """A batch whose simulations take 5 and 3 steps, with the potential
  tape (the shorter one leaves its later positions unwritten and the
  reverse sweep must skip them), against one plan per simulation without
  a tape.  Cotangents of the initial state agree to FP32 rounding of the
  two routes to the force meshes, and so does the rebuilt initial state,
  which is close to the true one."""
  rng = np.random.default_rng(41)
  n = 16**3
  sims = [(5, np.linspace(0.1, 1.0, 6)), (3, np.linspace(0.2, 0.8, 4))]
  d0 = torch.tensor(rng.standard_normal((2 * n, 3)) * 0.3,
                    dtype=torch.float32, device='cuda')
  p0 = torch.tensor(rng.standard_normal((2 * n, 3)) * 0.1,
                    dtype=torch.float32, device='cuda')
  lx0 = torch.tensor(rng.standard_normal((2 * n, 3)), dtype=torch.float32,
                     device='cuda')
  lp0 = torch.tensor(rng.standard_normal((2 * n, 3)), dtype=torch.float32,
                     device='cuda')
  lx, lp, dd, pp = _run_adjoint(sims, d0, p0, lx0, lp0, tape=True)
  for s in range(2):
    sl = slice(s * n, (s + 1) * n)
    rx, rp, rd, rpp = _run_adjoint([sims[s]], d0[sl], p0[sl], lx0[sl],
                                   lp0[sl], tape=False)
    assert rel_l2(lx[sl], rx) < 1e-4, (s, rel_l2(lx[sl], rx))
    assert rel_l2(lp[sl], rp) < 1e-4, (s, rel_l2(lp[sl], rp))
    assert np.abs(dd[sl] - rd).max() < 1e-4, (s, np.abs(dd[sl] - rd).max())
    assert np.abs(pp[sl] - rpp).max() < 1e-4, (s, np.abs(pp[sl] - rpp).max())
    assert np.abs(dd[sl] - host(d0[sl])).max() < 1e-3
    assert np.abs(pp[sl] - host(p0[sl])).max() < 1e-3


@pytest.mark.parametrize('tape', [False, True], ids=['rebuilt', 'potential'])
def test_adjoint_xpass_vs_cufft(fpm, tape):
  """The reverse sweep on a 256 x 16 x 16 mesh, which takes the x-pass
  Fourier solve (cuFFT plane transforms around the x-pass kernel, whose x
  pass in the reverse sweep also clears the adjoint force mesh for the
  next position), against the same plan on the three-dimensional cuFFT
  path (FPM_PLAN_CUFFT, a memset per position).  Both are FP32 with the
  same CIC conventions, so they differ by transform rounding only, which
  the reverse integration amplifies where a particle sits next to a cell
  face (the weight derivative jumps there): usually below 1e-4.  The
  order of the FP32 reductions into the meshes also varies from run to
  run, and on some runs of either path that flips one particle across a
  face, which moves the cotangents by 1.6e-3 (measured on the B200 over
  repeated runs of the same path).  A missing clear of the adjoint force
  mesh would give O(1).  (On meshes this elongated the FP32 gradient sits
  ~5e-3 from the FP64 oracle's on either path, for the same reason.)"""
  from flowpm_b200 import _lib
  rng = np.random.default_rng(43)
  nc = (256, 16, 16)
  n = int(np.prod(nc))
  sims = [(4, np.linspace(0.1, 1.0, 5)), (3, np.linspace(0.2, 0.8, 4))]
  t = lambda a: torch.tensor(a, dtype=torch.float32, device='cuda')
  d0 = t(rng.standard_normal((2 * n, 3)) * 0.3)
  p0 = t(rng.standard_normal((2 * n, 3)) * 0.1)
  lx0 = t(rng.standard_normal((2 * n, 3)))
  lp0 = t(rng.standard_normal((2 * n, 3)))
  a = _run_adjoint(sims, d0, p0, lx0, lp0, tape, nc)
  b = _run_adjoint(sims, d0, p0, lx0, lp0, tape, nc, _lib.FPM_PLAN_CUFFT)
  tol = 5e-3 if tape else 1e-2
  for u, v in zip(a, b):
    assert np.isfinite(u).all()
    assert rel_l2(u, v) < tol, rel_l2(u, v)


@pytest.mark.parametrize('nc', [(256, 256, 256), (512, 256, 512)],
                         ids=['256^3', '512x256x512'])
def test_lattice_walk_sizes_agree(fpm, nc, capsys):
  """The particle kernels walk large lattices in long blocks (16x8x16
  particles from 2^23 particles, 64x8x16 from 2^26); FPM_PLAN_SMALL_BLOCKS
  keeps 8x8x16. Both walks must visit every particle once: the forward
  state of a random field (3 steps) and the adjoint of a zero field (each
  scatter and gather then has one non-zero term) agree to FP32 rounding."""
  from flowpm_b200 import _lib
  rng = np.random.default_rng(53)
  n = int(np.prod(nc))
  sims = [(3, np.linspace(0.1, 0.5, 4))]
  d0 = torch.tensor(rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32),
                    device='cuda')
  p0 = torch.tensor(rng.uniform(-0.1, 0.1, (n, 3)).astype(np.float32),
                    device='cuda')
  lx0 = torch.tensor(rng.standard_normal((n, 3)).astype(np.float32),
                     device='cuda')
  lp0 = torch.tensor(rng.standard_normal((n, 3)).astype(np.float32),
                     device='cuda')
  z = torch.zeros_like(d0)
  errs = []
  for dd, pp in ((d0, p0), (z, z)):
    a = _run_adjoint(sims, dd, pp, lx0, lp0, True, nc)
    b = _run_adjoint(sims, dd, pp, lx0, lp0, True, nc,
                     _lib.FPM_PLAN_SMALL_BLOCKS)
    for x, y in zip(a, b):
      assert np.isfinite(x).all()
    # relative L2 for the cotangents and the random-field state; the
    # zero-field state is rounding noise around 0: max absolute difference
    errs.append([rel_l2(a[0], b[0]), rel_l2(a[1], b[1])] +
                ([rel_l2(a[k], b[k]) for k in (2, 3)] if dd is d0 else
                 [float(np.abs(a[k] - b[k]).max()) for k in (2, 3)]))
  with capsys.disabled():
    print('\n  walk sizes at %s: random field (lx, lp, d, p) %s; zero field '
          '%s' % ('x'.join(map(str, nc)),
                  ' '.join('%.1e' % e for e in errs[0]),
                  ' '.join('%.1e' % e for e in errs[1])))
  assert max(errs[0][2:]) < 1e-5, errs[0]   # rebuilt state, random field
  assert max(errs[1][:2]) < 1e-5, errs[1]   # cotangents, zero field
  assert max(errs[1][2:]) < 1e-5, errs[1]   # rebuilt state, zero field


@pytest.mark.parametrize('store', [False, True], ids=['rebuilt', 'potential'])
def test_nbody_adjoint_64_20_steps_vs_tape(fpm, capsys, store):
  """The C4 problem at 64^3 (box 100 Mpc/h, the C4 spacing; seeded
  Eisenstein-Hu field, 2LPT at a0 = 0.1, 20 steps, checkpoints every 5):
  the reverse-time adjoint against the FP64 oracle's autograd over every
  component (rel-L2) and along 32 random directions."""
  from flowpm_b200 import tfpower
  n, box, steps = 64, 100.0, 20
  c = fpm.cosmology.Planck15()
  kk = np.logspace(-4, 2, 4096)
  pkv = tfpower.linear_matter_power(c, kk)
  pk = lambda k: np.interp(np.log(np.maximum(k, 1e-30)), np.log(kk), pkv,
                           left=0.0)
  lin = host(fpm.linear_field(n, box, pk, seed=6464)).astype(np.float64)
  stages = np.linspace(0.1, 1.0, steps + 1)
  nc = [n] * 3
  rng = np.random.default_rng(64)
  target = _rho_oracle(lin, stages, nc) + rng.standard_normal([1] + nc)
  def oracle_grad(dtype):
    b = obg.Background({}, dtype=np.float64 if dtype == torch.float64
                       else np.float32)
    x = torch.tensor(lin, dtype=dtype, requires_grad=True)
    st = opm.nbody_checkpointed(b, opm.lpt_init(b, x, 0.1, order=2), stages,
                                nc)
    rho = opm.cic_paint(torch.zeros([1] + nc, dtype=dtype), st[0])
    (go,) = torch.autograd.grad(
        ((rho - torch.tensor(target, dtype=dtype))**2).sum(), x)
    return go.double().numpy()

  go = oracle_grad(torch.float64)
  g32 = oracle_grad(torch.float32)  # the reference's own FP32 arithmetic
  _, g = _chi2_ours(fpm, lin, target, stages, nc, ckpt=5, store=store)
  err, floor = rel_l2(g, go), rel_l2(g32, go)
  dirs, dirs32 = [], []
  for _ in range(32):
    u = rng.standard_normal(lin.shape)
    t = float(np.sum(go * u))
    dirs.append(abs(float(np.sum(g * u)) - t) / abs(t))
    dirs32.append(abs(float(np.sum(g32 * u)) - t) / abs(t))
  with capsys.disabled():
    print('\n  adjoint 64^3 / 20 steps vs FP64 tape (stored potential %s): '
          'rel-L2 %.2e, 32 directions median %.2e max %.2e; the FP32 '
          'oracle tape: rel-L2 %.2e, median %.2e max %.2e' %
          (store, err, np.median(dirs), np.max(dirs), floor,
           np.median(dirs32), np.max(dirs32)))
  # an FP32 forward of this length is chaotic at the 1e-4 level: the bar is
  # the FP32 oracle's own distance from FP64 (and 1e-3 overall)
  assert err < 1e-3 and err < 2 * floor
  assert np.median(dirs) < 1e-3 and np.median(dirs) < 2 * np.median(dirs32)
