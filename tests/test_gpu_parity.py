"""Parity of the CUDA path (through the C ABI) with the reference: golden
fixtures from the reference's own source and the CPU oracle on the same
inputs.  Bars: cell indices / neighbour sets bit-exact; CIC values at
FP32 rounding; final density rel-L2 <= 1e-4; P(k) per bin <= 1e-4; the
error against the FP64 oracle is printed for every trajectory result."""
import numpy as np
import pytest
import torch
from numpy.testing import assert_allclose

from conftest import golden, pk_table, rel_l2
from oracle import background as obg
from oracle import pm as opm
from oracle import rng as orng

pytestmark = pytest.mark.gpu
ALT = dict(Omega_c=0.30, Omega_b=0.045, h=0.70, sigma8=0.75, n_s=0.96)


@pytest.fixture(scope='module')
def fpm(cuda):
  import flowpm_b200
  return flowpm_b200


def host(t):
  return t.detach().cpu().numpy()


# --------------------------------------------------------------------------
# CIC operators
# --------------------------------------------------------------------------
def test_cic_paint_readout_golden(fpm):
  z = golden('cic')
  m = fpm.cic_paint(np.zeros((2, 16, 16, 16), np.float32), z['pos'],
                    z['wts'])
  assert_allclose(host(m), z['paint_w'], atol=1e-6)
  m = fpm.cic_paint(np.zeros((2, 16, 16, 16), np.float32), z['pos'])
  assert_allclose(host(m), z['paint_1'], atol=1e-6)
  r = fpm.cic_readout(z['base'], z['pos'])
  assert_allclose(host(r), z['readout'], rtol=1e-6)
  m = fpm.cic_paint(np.zeros((1, 8, 6, 10), np.float32), z['pos_rect'])
  assert_allclose(host(m), z['paint_rect'], atol=1e-6)
  r = fpm.cic_readout(z['base_rect'], z['pos_rect'])
  assert_allclose(host(r), z['readout_rect'], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize('nc', [[16, 16, 16], [8, 6, 10], [128, 128, 128]])
def test_cic_neighbours_bit_exact(fpm, nc):
  rng = np.random.default_rng(7)
  n = 20000
  pos = (rng.random((n, 3)) * 3 - 1) * np.array(nc)
  # faces, integer points, the wrap at N - eps, huge and negative values
  pos[:6] = [[0, 0, 0], [nc[0] - 1e-5, 0.5, 1.0], [-1e-7, 3.0, 2.0],
             [nc[0], nc[1], nc[2]], [-nc[0] * 7.25, 1e4, -3e3],
             [0.999999, 1.0000001, 2.5]]
  # round-half ties, -0, and both sides of the 2^22 limit of the kernels'
  # exact small-magnitude floor
  pos[6:10] = [[3.5, -2.5, -0.0], [4194303.5, -4194303.5, 4194304.0],
               [-4194304.5, 8388607.0, -8388608.0],
               [-2 * nc[0] + 0.25, 2 * nc[1] - 0.25, -nc[2] - 0.5]]
  pos = pos.astype(np.float32)
  idx, w = fpm.utils.cic_neighbours(pos, nc)
  t = torch.tensor(pos).reshape(1, -1, 3)
  ref = opm._neighbours(t, nc)
  ref_idx = np.stack([f.numpy()[0] for _, f in ref], axis=1)
  ref_w = np.stack([k.numpy()[0] for k, _ in ref], axis=1)
  assert np.array_equal(host(idx).astype(np.int64), ref_idx)
  assert np.array_equal(host(w), ref_w)


def test_cic_empty_and_batched(fpm):
  mesh = torch.full((3, 8, 8, 8), 2.0, device='cuda')
  out = fpm.cic_paint(mesh, torch.zeros((3, 0, 3), device='cuda'))
  assert torch.equal(out, mesh)
  r = fpm.cic_readout(mesh, torch.zeros((3, 0, 3), device='cuda'))
  assert r.shape == (3, 0)


def test_cic_large_properties(fpm):
  """128^3 mesh, 2 x 2^21 particles: mass conservation, readout of a
  constant and of a linear ramp, and agreement with the oracle."""
  g = torch.Generator(device='cpu').manual_seed(3)
  B, n, N = 2, 1 << 21, 128
  pos = torch.rand((B, n, 3), generator=g) * N
  w = torch.rand((B, n), generator=g)
  m = fpm.cic_paint(torch.zeros((B, N, N, N)), pos, w)
  assert_allclose(host(m.double().sum(dim=(1, 2, 3))),
                  w.double().sum(dim=1).numpy(), rtol=1e-6)
  ref = opm.cic_paint(torch.zeros((B, N, N, N)), pos, w)
  assert_allclose(host(m), ref.numpy(), atol=2e-5)
  r = fpm.cic_readout(torch.full((B, N, N, N), 3.5), pos)
  assert_allclose(host(r), 3.5, rtol=1e-6)
  ramp = torch.arange(N, dtype=torch.float32).reshape(1, 1, 1, N).expand(
      B, N, N, N).contiguous()
  inner = pos.clone()
  inner[..., 2] = inner[..., 2].clamp(0, N - 1.01)
  r = fpm.cic_readout(ramp, inner)
  assert_allclose(host(r), inner[..., 2].numpy(), atol=2e-5)


def test_fft_pair(fpm):
  z = golden('cic')
  c = fpm.r2c3d(torch.tensor(z['rt_in']), dtype=torch.complex128)
  assert_allclose(host(c), z['rt_k'], rtol=1e-9, atol=1e-9)
  r = fpm.c2r3d(c, dtype=torch.float64)
  assert_allclose(host(r), z['rt_in'], rtol=1e-9)
  r32 = fpm.c2r3d(fpm.r2c3d(torch.tensor(z['rt_in'], dtype=torch.float32)))
  assert_allclose(host(r32), z['rt_in'], rtol=1e-4, atol=1e-3)


# --------------------------------------------------------------------------
# Initial conditions
# --------------------------------------------------------------------------
def test_white_noise_generator(fpm):
  w = fpm.white_noise([8, 8, 10], batch_size=3, seed=12345, type='real')
  ref = orng.white_noise(3 * 640, 12345, stddev=640**0.5)
  assert_allclose(host(w).ravel(), ref, rtol=1e-6, atol=1e-6)
  big = host(fpm.white_noise(64, batch_size=2, seed=1, type='real')).ravel()
  big /= 64**1.5
  assert abs(big.mean()) < 5e-3 and abs(big.std() - 1) < 5e-3


@pytest.mark.parametrize('nc,bs', [(16, 50.), (32, 100.)])
def test_linear_field_golden(fpm, nc, bs):
  z = golden('lpt')
  lin = fpm.linear_field(nc, bs, pk_table(), white=z['n%d_white' % nc])
  ref = z['n%d_linear' % nc]
  assert_allclose(host(lin), ref, atol=1e-5 * np.abs(ref).max())


def test_linear_field_seeded(fpm):
  a = fpm.linear_field(32, 100., pk_table(), batch_size=2, seed=9)
  b = fpm.linear_field(32, 100., pk_table(), batch_size=2, seed=9)
  assert torch.equal(a, b)
  white = orng.white_noise(2 * 32**3, 9, stddev=32**1.5).reshape(
      2, 32, 32, 32)
  ref = opm.linear_field_from_white(torch.tensor(white), 100., pk_table())
  assert_allclose(host(a), ref.numpy(), atol=1e-5 * float(ref.abs().max()))


def test_linear_field_caller_kvec(fpm):
  """linear_field on a caller's k grid (fftk's, doubled): |k| doubles, so
  the field equals the default grid's with P(2k), on the same noise."""
  pk = pk_table()
  kv = [2.0 * k for k in fpm.kernels.fftk([32] * 3, symmetric=False)]
  a = fpm.linear_field(32, 100., pk, kvec=kv, seed=4)
  b = fpm.linear_field(32, 100., lambda k: pk(2.0 * np.asarray(k)), seed=4)
  assert_allclose(host(a), host(b), atol=1e-5 * float(b.abs().max()))


@pytest.mark.parametrize('nc,order', [(16, 1), (16, 2), (32, 2)])
def test_lpt_init_golden(fpm, nc, order):
  z = golden('lpt')
  c = fpm.cosmology.Planck15()
  s = host(fpm.lpt_init(c, z['n%d_linear' % nc], 0.1, order=order))
  ref = z['n%d_init_o%d' % (nc, order)]
  assert_allclose(s, ref, atol=3e-5 * np.abs(ref).max(axis=(1, 2, 3),
                                                      keepdims=True).max())


def test_lpt1_lpt2_source_golden(fpm):
  """flowpm/tfpm.py:66-95 lpt1 and :98-145 lpt2_source as drop-ins, on the
  reference's own outputs (lpt1 at the lattice points, c2r3d of the 2LPT
  source spectrum)."""
  z = golden('lpt')
  lk = fpm.r2c3d(z['n16_linear'], norm=16**3)
  grid = np.indices([16] * 3).reshape(3, -1).T.astype(np.float32)[None]
  psi = host(fpm.tfpm.lpt1(lk, grid))
  ref = z['n16_lpt1']
  assert_allclose(psi, ref, atol=3e-5 * np.abs(ref).max())
  src = fpm.tfpm.lpt2_source(lk)
  assert src.shape == (1, 16, 16, 16) and src.dtype == torch.complex64
  ref = z['n16_lpt2src']
  assert_allclose(host(fpm.c2r3d(src, norm=16**3)), ref,
                  atol=3e-5 * np.abs(ref).max())


def test_lpt1_lpt2_source_oracle(fpm):
  """The drop-ins against the oracle on a batch of two rectangular meshes:
  lpt1 read out at displaced positions (faces and periodic wraps), and the
  full 2LPT source spectrum, including its Hermitian half l > nz/2."""
  rng = np.random.default_rng(11)
  nc = [16, 8, 12]
  lin = rng.standard_normal([2] + nc).astype(np.float32)
  lk = opm.r2c3d(torch.tensor(lin))
  grid = np.indices(nc).reshape(3, -1).T.astype(np.float32)
  pos = np.stack([grid + rng.uniform(-3, 3, grid.shape).astype(np.float32),
                  grid - 0.5]).astype(np.float32)
  pos[0, :4] = [[0, 0, 0], [15.999999, 7.5, -1e-6], [-16, 8, 12], [3, 4, 5]]
  ref = opm.lpt1(lk, torch.tensor(pos)).numpy()
  got = host(fpm.tfpm.lpt1(lk.numpy(), pos))
  assert_allclose(got, ref, atol=2e-5 * np.abs(ref).max())
  ref = opm.lpt2_source(lk).numpy()
  got = host(fpm.tfpm.lpt2_source(lk.numpy()))
  assert_allclose(got, ref, atol=2e-5 * np.abs(ref).max())


def test_lpt_init_rectangular_alt_cosmology(fpm):
  z = golden('nbody')
  c = fpm.cosmology.Planck15(**ALT)
  s = host(fpm.lpt_init(c, z['rect_linear'], 0.1, order=2))
  assert_allclose(s, z['rect_init'], atol=1e-5)


# --------------------------------------------------------------------------
# Force, kick, drift, nbody
# --------------------------------------------------------------------------
def test_force_kick_drift_golden(fpm):
  z, l = golden('nbody'), golden('lpt')
  c = fpm.cosmology.Planck15()
  s0 = l['n16_init_o1']
  f = host(fpm.tfpm.force(c, s0, 16))
  assert_allclose(f, z['n16_force'], atol=2e-5)
  assert_allclose(host(fpm.tfpm.kick(c, s0, 0.1, 0.1, 0.12)), z['n16_kick'],
                  atol=2e-6)
  assert_allclose(host(fpm.tfpm.drift(c, s0, 0.1, 0.12, 0.15)),
                  z['n16_drift'], atol=2e-6)


def _fp64_oracle_state(state0, stages, nc, cosmo_kw=None, pm_nc_factor=1):
  b64 = obg.Background(cosmo_kw or {}, dtype=np.float64)
  s = torch.tensor(state0, dtype=torch.float64)
  return opm.nbody(b64, s, stages, nc, pm_nc_factor=pm_nc_factor).numpy()


def test_nbody_16_golden(fpm, capsys):
  z, l = golden('nbody'), golden('lpt')
  c = fpm.cosmology.Planck15()
  stages = z['stages']
  st = host(fpm.nbody(c, l['n16_init_o1'], stages, 16))
  assert_allclose(st, z['n16_b1_final'], atol=1e-4)
  st2 = host(fpm.nbody(c, l['n16_init_o1'], stages, 16, pm_nc_factor=2))
  assert_allclose(st2, z['n16_b2_final'], atol=1e-4)
  inter = fpm.nbody(c, l['n16_init_o1'], stages[:4], 16,
                    return_intermediate_states=True)
  assert [a for a, _ in inter] == list(z['n16_inter_a'])
  assert_allclose(np.stack([host(s) for _, s in inter]), z['n16_inter'],
                  atol=2e-5)
  ref64 = _fp64_oracle_state(l['n16_init_o1'], stages, 16)
  with capsys.disabled():
    print('\n  nbody 16^3: max |X - X_fp64| = %.2e cells (reference FP32: '
          '%.2e)' % (np.abs(st[0] - ref64[0]).max(),
                     np.abs(z['n16_b1_final'][0] - ref64[0]).max()))


def test_nbody_rectangular_golden(fpm):
  z = golden('nbody')
  c = fpm.cosmology.Planck15(**ALT)
  s0 = fpm.lpt_init(c, z['rect_linear'], 0.1, order=2)
  st = host(fpm.nbody(c, s0, z['stages'], [8, 8, 24]))
  assert_allclose(st, z['rect_final'], atol=1e-4)


def _pk(field, bs):
  kb, p = opm.power_spectrum(torch.tensor(field, dtype=torch.float64),
                             kmin=0.1, dk=0.05, boxsize=np.array([bs] * 3))
  return p.numpy()


def test_nbody_32_density_and_pk(fpm, capsys):
  """C1 configuration (32^3, box 100, Planck15, 2LPT at a0=0.1, 10 stages):
  final density within 1e-4 relative L2 and P(k) within 1e-4 per bin of
  the reference."""
  z, l = golden('nbody'), golden('lpt')
  c = fpm.cosmology.Planck15()
  stages = z['stages']
  s0 = fpm.lpt_init(c, l['n32_linear'], 0.1, order=2)
  st = fpm.nbody(c, s0, stages, 32)
  rho = host(fpm.cic_paint(torch.zeros((1, 32, 32, 32)), st[0]))
  err = rel_l2(rho, z['n32_rho'])
  assert err <= 1e-4, err
  pk, pk_ref = _pk(rho, 100.), _pk(z['n32_rho'], 100.)
  pk_err = float(np.max(np.abs(pk - pk_ref) / np.abs(pk_ref)))
  assert pk_err <= 1e-4, pk_err
  ref64 = _fp64_oracle_state(l['n32_init_o2'], stages, 32)
  rho64 = opm.cic_paint(torch.zeros((1, 32, 32, 32), dtype=torch.float64),
                        torch.tensor(ref64[0])).numpy()
  with capsys.disabled():
    print('\n  nbody 32^3: density rel-L2 vs reference %.2e, vs FP64 %.2e '
          '(reference vs FP64 %.2e); P(k) max rel %.2e' %
          (err, rel_l2(rho, rho64), rel_l2(z['n32_rho'], rho64), pk_err))


def test_nbody_status_nonfinite(fpm):
  l = golden('lpt')
  c = fpm.cosmology.Planck15()
  s = l['n16_init_o1'].copy()
  s[0, 0, 5, 1] = np.nan
  with pytest.raises(fpm._lib.FlowPMError):
    fpm.nbody(c, s, [0.1, 0.2], 16)
  # the plan and the context stay usable
  st = fpm.nbody(c, l['n16_init_o1'], [0.1, 0.2], 16)
  assert torch.isfinite(st).all()


def test_plan_out_of_memory(fpm):
  """A plan far larger than the device (400 meshes of 512^3, 215 GB of
  density alone) fails in fpm_plan_create with a resource error
  (FPM_ERR_OOM, or FPM_ERR_CUFFT should cuFFT refuse the batch first),
  having freed what it allocated; the device and a normal plan work
  afterwards."""
  from flowpm_b200 import _lib
  from flowpm_b200._plans import Plan
  free0 = torch.cuda.mem_get_info()[0]
  with pytest.raises(_lib.FlowPMError) as e:
    Plan([(512, 512, 512, 1)] * 400)
  print('oversized plan:', e.value)
  assert e.value.code in (3, 5), e.value  # FPM_ERR_OOM, FPM_ERR_CUFFT
  torch.cuda.synchronize()
  assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)
  l = golden('lpt')
  st = fpm.nbody(fpm.cosmology.Planck15(), l['n16_init_o1'], [0.1, 0.2], 16)
  assert torch.isfinite(st).all()


def test_batched_uneven_plan(fpm):
  """Simulations of different sizes, cosmologies and step counts advanced
  by one plan match the same simulations run one at a time."""
  from flowpm_b200 import _lib, tfbackground
  from flowpm_b200._plans import Plan
  rng = np.random.default_rng(11)
  sims = [(16, dict(Omega_c=0.25, sigma8=0.8), 5),
          (16, dict(Omega_c=0.32, sigma8=0.72), 3),
          (8, dict(Omega_c=0.22, sigma8=0.88), 4),
          (32, {}, 6)]
  maxT = max(t for _, _, t in sims)
  dims, disp, mom, coefs, ffac, nsteps = [], [], [], [], [], []
  singles = []
  for n, kw, T in sims:
    c = fpm.cosmology.Planck15(**kw)
    lin = rng.standard_normal((1, n, n, n)).astype(np.float32) * 0.3
    s0 = fpm.lpt_init(c, lin, 0.1, order=2)
    stages = np.linspace(0.1, 1.0, T + 1)
    singles.append(host(fpm.nbody(c, s0, stages, n)))
    dims.append((n, n, n, 1))
    disp.append(fpm.tfpm._to_disp(s0[0], [n] * 3).reshape(-1, 3))
    mom.append(s0[1].reshape(-1, 3))
    co = np.zeros((maxT, 3))
    co[:T] = tfbackground.nbody_coefficients(c, stages)
    coefs.append(co)
    ffac.append(1.5 * c.Omega_m)
    nsteps.append(T)
  plan = Plan(dims)
  d = torch.cat(disp).contiguous()
  p = torch.cat(mom).contiguous()
  f = torch.empty_like(d)
  _lib.call('fpm_nbody', plan.handle, _lib.ptr(d), _lib.ptr(p), _lib.ptr(f),
            maxT, _lib.ivec(nsteps), _lib.dvec(np.concatenate(coefs).ravel()),
            _lib.dvec(ffac), None, 0, _lib.stream_ptr())
  off = 0
  for (n, _, _), ref in zip(sims, singles):
    npart = n**3
    X = d[off:off + npart] + torch.tensor(
        opm.lattice([n] * 3, 1)[0].numpy(), device='cuda')
    assert_allclose(host(X), ref[0, 0], atol=1e-4)
    assert_allclose(host(p[off:off + npart]), ref[1, 0], atol=1e-4)
    assert_allclose(host(f[off:off + npart]), ref[2, 0], atol=1e-4)
    off += npart
  assert plan.status() == 0


# --------------------------------------------------------------------------
# Power spectrum (flowpm/pk.py)
# --------------------------------------------------------------------------
def test_power_spectrum_golden(fpm):
  z = golden('pk')
  for tag in ['rho32', 'lin16']:
    bs = float(z[tag + '_boxsize'])
    kb, p = fpm.power_spectrum(z[tag + '_field'], kmin=0.1, dk=0.05,
                               boxsize=np.array([bs] * 3))
    assert_allclose(kb, z[tag + '_k'], rtol=1e-12)
    assert_allclose(host(p), z[tag + '_pk'], rtol=2e-5)


def test_power_spectrum_batched_rectangular(fpm):
  rng = np.random.default_rng(4)
  f = rng.standard_normal((3, 8, 12, 16)).astype(np.float32)
  box = np.array([40., 60., 80.])
  kb, p = fpm.power_spectrum(f, kmin=0.05, dk=0.02, boxsize=box)
  kb_o, p_o = opm.power_spectrum(torch.tensor(f, dtype=torch.float64),
                                 kmin=0.05, dk=0.02, boxsize=box)
  assert_allclose(kb, kb_o, rtol=1e-12)
  assert_allclose(host(p), p_o.numpy(), rtol=1e-5)


def test_nbody_many_matches_single_runs(fpm):
  """The batch API (one plan, one graph, finished simulations dropped from
  the transforms) equals nbody on each simulation, in the caller's order,
  whatever the input order of sizes and step counts."""
  rng = np.random.default_rng(12)
  spec = [(16, dict(Omega_c=0.22), 3), (8, {}, 5), (16, dict(sigma8=0.9), 6),
          (16, {}, 1), ([8, 8, 16], dict(Omega_c=0.3), 4), (8, {}, 0)]
  sims, states, singles = [], [], []
  for nc, kw, T in spec:
    c = fpm.cosmology.Planck15(**kw)
    n3 = [nc] * 3 if isinstance(nc, int) else nc
    lin = rng.standard_normal([1] + n3).astype(np.float32) * 0.3
    s0 = fpm.lpt_init(c, lin, 0.1, order=2)
    stages = np.linspace(0.1, 1.0, T + 1)
    sims.append(dict(nc=nc, cosmo=c, stages=stages))
    states.append(s0)
    singles.append(host(fpm.nbody(c, s0, stages, nc)))
  out = fpm.nbody_many(sims, states)
  for o, ref in zip(out, singles):
    assert_allclose(host(o), ref, atol=1e-4)
  # a second batch on the same shapes with other step counts reuses nothing
  # stale: run it twice through one runner
  r = fpm.BatchRunner(sims)
  r.load(states)
  r.run()
  r.load(states)
  r.run()
  for o, ref in zip(r.results(), singles):
    assert_allclose(host(o), ref, atol=1e-4)
  r.close()


def test_pgd_golden(fpm, capsys):
  """PGD correction (flowpm/tfpm.py:369-422; after every drift in nbody,
  :487-488) against the reference's own output: one call, and a 9-step
  leapfrog at pm_nc_factor 1 and 2 (also against the FP64 oracle).  The
  same cached plan then runs without PGD and gives the plain result."""
  z, l, nb = golden('pgd'), golden('lpt'), golden('nbody')
  c = fpm.cosmology.Planck15()
  s0 = l['n16_init_o1']
  out = host(fpm.tfpm.pgd(s0, z['params'][0], 16))
  assert_allclose(out, z['single'], atol=2e-5)
  out = host(fpm.tfpm.pgd(s0, z['params'][0], 16, pm_nc_factor=2))
  assert_allclose(out, z['single_b2'], atol=2e-5)
  for bf, key, tol in ((1, 'final', 2e-3), (2, 'final_b2', 5e-3)):
    out = host(fpm.nbody(c, s0, z['stages'], 16, pm_nc_factor=bf,
                         pgdparams=z['params']))
    b64 = obg.Background({}, dtype=np.float64)
    ref64 = opm.nbody(b64, torch.tensor(s0, dtype=torch.float64),
                      z['stages'], 16, pm_nc_factor=bf,
                      pgdparams=z['params']).numpy()
    with capsys.disabled():
      print('\npgd bf=%d: vs reference %.2e, vs FP64 %.2e, reference vs '
            'FP64 %.2e' % (bf, np.abs(out - z[key]).max(),
                           np.abs(out - ref64).max(),
                           np.abs(z[key] - ref64).max()))
    assert_allclose(out, z[key], atol=tol)
  # PGD off again on the same plan
  st = host(fpm.nbody(c, s0, z['stages'], 16))
  assert_allclose(st, nb['n16_b1_final'], atol=1e-4)
  # gradients through PGD need the stored potentials
  # (tests/test_gpu_adjoint.py checks them against the FP64 oracle)
  with pytest.raises(ValueError):
    x = torch.tensor(s0, device='cuda').requires_grad_(True)
    fpm.nbody(c, x, z['stages'], 16, pgdparams=z['params'],
              store_potential=False)


def test_nbody_stream_matches_nbody(fpm):
  """The host-streaming API (copies overlapped with the computation, double
  buffered, more simulations than buffers) returns, for every host state,
  what nbody returns for it on the device."""
  rng = np.random.default_rng(21)
  c = fpm.cosmology.Planck15()
  stages = np.linspace(0.1, 1.0, 5)
  for nc, B in ((16, 1), ([16, 8, 16], 2)):
    n3 = [nc] * 3 if isinstance(nc, int) else nc
    states, refs = [], []
    for _ in range(5):
      lin = rng.standard_normal([B] + n3).astype(np.float32) * 0.3
      s0 = fpm.lpt_init(c, lin, 0.1, order=2)
      refs.append(host(fpm.nbody(c, s0, stages, nc)))
      states.append(s0.cpu().pin_memory())
    out = fpm.nbody_stream(c, states, stages, nc)
    assert len(out) == len(states)
    for o, ref in zip(out, refs):
      assert o.shape == ref.shape
      assert_allclose(o.numpy(), ref, atol=1e-4)


def _oracle_force_variant(state, nc, omega_m, order=1, r_split=0.0,
                          deconv=False):
  """flowpm/tfpm.py:317-366 force with the Fourier operator options of
  flowpm/kernels.py: gradient order, Gaussian split, CIC compensation."""
  s = torch.tensor(state, dtype=torch.float64)
  B = s.shape[1]
  rho = opm.cic_paint(torch.zeros([B] + nc, dtype=torch.float64), s[0])
  dk = opm.r2c3d(rho, norm=nc[0] * nc[1] * nc[2])
  kvec = opm.fftk(nc, symmetric=False)
  w = opm.laplace_kernel(kvec) * opm.longrange_kernel(kvec, r_split)
  if deconv:
    w = w * opm.cic_compensation(kvec)
  f = []
  for d in range(3):
    kd = opm.gradient_kernel(kvec, d, order=order)
    forced = opm.c2r3d(dk * torch.as_tensor(w * kd),
                       norm=nc[0] * nc[1] * nc[2])
    f.append(opm.cic_readout(forced, s[0]))
  return (torch.stack(f, dim=2) * 1.5 * omega_m).numpy()


@pytest.mark.parametrize('flags,r_split,order,deconv', [
    (0, 0.0, 1, False), (0, 1.5, 1, False), (1, 0.0, 1, True),
    (4, 0.0, 0, False), (5, 1.2, 0, True)])
def test_force_operator_options(fpm, flags, r_split, order, deconv):
  """The fused Fourier force with the Green's function, the gradient of
  either order, the CIC deconvolution and the Gaussian long-range split
  (the plan options) against the oracle built from flowpm/kernels.py."""
  from flowpm_b200 import _lib
  from flowpm_b200._plans import Plan
  l = golden('lpt')
  c = fpm.cosmology.Planck15()
  s0 = l['n16_init_o2']
  plan = Plan([(16, 16, 16, 1)], r_split=r_split, flags=flags)
  x = torch.tensor(s0[0], device='cuda')
  d = fpm.tfpm._to_disp(x, [16] * 3)
  f = torch.empty_like(d)
  _lib.call('fpm_force', plan.handle, _lib.ptr(d),
            _lib.dvec([1.5 * c.Omega_m]), _lib.ptr(f), _lib.stream_ptr())
  ref = _oracle_force_variant(s0, [16] * 3, c.Omega_m, order, r_split, deconv)
  assert_allclose(host(f)[0], ref[0], atol=2e-5 * np.abs(ref).max())
  plan.close()
