"""Generate the golden fixtures under ``tests/golden/`` by executing the
reference FlowPM source itself.

Run with ``FLOWPM_REF`` set to a checkout of the reference (the directory
that holds ``flowpm/``; it is only read)::

    FLOWPM_REF=<reference checkout> python tests/golden/make_golden.py

TensorFlow is not installable here, so ``tfshim.py`` (a NumPy emulation of the
TF 2.5 / TFP 0.13 ops the reference calls) is registered as ``tensorflow``;
the reference modules ``flowpm/{tfpm,utils,kernels,tfbackground,tfpower,pk,
cosmology}.py`` are then imported from their source files and run unmodified.
``flowpm/legacy_background.py`` (NumPy + SciPy only, the reference's own
background test oracle) runs natively.

Every fixture records its inputs next to its outputs, so the tests need
neither the reference tree nor the shim at run time.
"""
import importlib
import os
import sys
import types

import numpy as np
from scipy.interpolate import InterpolatedUnivariateSpline as iuspline

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get('FLOWPM_REF')


def load_reference():
  if not REF or not os.path.isdir(os.path.join(REF, 'flowpm')):
    raise SystemExit('set FLOWPM_REF to a checkout of the reference (the '
                     'directory holding flowpm/)')
  sys.path.insert(0, HERE)
  import tfshim
  tfshim.install()
  pkg = types.ModuleType('flowpm')
  pkg.__path__ = [os.path.join(REF, 'flowpm')]
  sys.modules['flowpm'] = pkg
  mods = {}
  for name in ['tfpm', 'utils', 'kernels', 'tfbackground', 'tfpower', 'pk',
               'cosmology', 'legacy_background']:
    mods[name] = importlib.import_module('flowpm.' + name)
  return tfshim, mods


def planck_table():
  tab = np.loadtxt(os.path.join(REF, 'flowpm/data/Planck15_a1p00.txt'))
  return tab[:, 0].copy(), tab[:, 1].copy()


def save(name, **arrays):
  path = os.path.join(HERE, name)
  np.savez_compressed(path, **arrays)
  print('wrote', path, '%.1f KB' % (os.path.getsize(path) / 1024.))


def gen_kernels(m):
  k = m['kernels']
  out = {}
  for tag, shape in [('c8', [8, 8, 8]), ('r4610', [4, 6, 10])]:
    kv = k.fftk(shape, symmetric=False)
    kvs = k.fftk(shape, symmetric=True)
    for d in range(3):
      out['%s_fftk_%d' % (tag, d)] = kv[d]
      out['%s_fftk_sym_%d' % (tag, d)] = kvs[d]
      out['%s_grad1_%d' % (tag, d)] = k.gradient_kernel(kv, d, order=1)
      out['%s_grad0_%d' % (tag, d)] = k.gradient_kernel(kv, d, order=0)
    out['%s_laplace' % tag] = k.laplace_kernel(kv)
    out['%s_longrange_r1p3' % tag] = k.longrange_kernel(kv, 1.3)
    out['%s_longrange_r0' % tag] = np.asarray(k.longrange_kernel(kv, 0))
    out['%s_ciccomp' % tag] = k.cic_compensation(kv)
  save('kernels.npz', **out)


COSMOS = {
    'planck15': {},
    'alt': dict(Omega_c=0.30, Omega_b=0.045, h=0.70, sigma8=0.75, n_s=0.96),
}


def gen_background(m):
  bg, cosmology = m['tfbackground'], m['cosmology']
  out = {}
  a = np.logspace(-2, 0, 128)
  stages = np.linspace(0.1, 1.0, 10)
  ah = np.sqrt(stages[:-1] * stages[1:])
  a_eval = np.concatenate([a, stages, ah])
  out['a_eval'] = a_eval
  for tag, kw in COSMOS.items():
    c = cosmology.Planck15(**kw)
    out['%s_params' % tag] = np.array([
        float(c.Omega_c), float(c.Omega_b), float(c.h), float(c.n_s),
        float(c.sigma8), float(c.Omega_k), float(c.w0), float(c.wa)
    ])
    for fn in ['E', 'dEa', 'Omega_m_a', 'Omega_de_a', 'D1', 'D2', 'D1f',
               'D2f', 'f1', 'f2', 'Gf', 'Gf2', 'gf', 'gf2']:
      out['%s_%s' % (tag, fn)] = np.asarray(getattr(bg, fn)(c, a_eval))
    cache = bg.maybe_compute_ODE(c)
    for key in ['a', 'D1', 'D1f', 'F1p', 'D2', 'D2f', 'F2p']:
      out['%s_ode_%s' % (tag, key)] = np.asarray(cache[key])
  # The reference's own FP64 background oracle (tests/test_tfbackground.py).
  md = m['legacy_background'].MatterDominated(Omega0_m=0.3075)
  a3 = np.logspace(-3, 0)
  out['legacy_a3'] = a3
  out['legacy_E'] = md.E(a3)
  out['legacy_Eprime'] = md.efunc_prime(a3)
  out['legacy_Om'] = md.Om(a3)
  out['legacy_a'] = a
  for fn in ['D1', 'D2', 'gp', 'gp2', 'f1', 'f2', 'Gf', 'Gf2', 'gf', 'gf2']:
    out['legacy_%s' % fn] = getattr(md, fn)(a)
  save('background.npz', **out)


def gen_power(m):
  tfpower, cosmology = m['tfpower'], m['cosmology']
  out = {}
  k = np.logspace(-3, 1, 512)
  out['k'] = k
  for tag, kw in COSMOS.items():
    c = cosmology.Planck15(**kw)
    out['%s_pk' % tag] = np.asarray(tfpower.linear_matter_power(c, k, 1.))
    out['%s_pk_a0p5' % tag] = np.asarray(
        tfpower.linear_matter_power(c, k, 0.5))
    out['%s_T_eisenhu' % tag] = np.asarray(
        tfpower.Eisenstein_Hu(c, k, type='eisenhu'))
    out['%s_T_osc' % tag] = np.asarray(
        tfpower.Eisenstein_Hu(c, k, type='eisenhu_osc'))
  kt, pt = planck_table()
  out['nbodykit_k'] = kt
  out['nbodykit_pk'] = pt
  save('power.npz', **out)


def gen_cic(tf, m):
  u = m['utils']
  rng = np.random.default_rng(1234)
  nc, bs, n = 16, 50., 100
  out = {}
  pos = (bs * rng.random((2, n, 3)) * nc / bs).astype(np.float32)
  # Edge cases: integer positions, cell faces, the periodic wrap at N - eps
  # and positions outside [0, N) that the reference folds with mod.
  edge = np.array([[0, 0, 0], [15, 15, 15], [15.999999, 0.5, 3.25],
                   [7.0, 7.5, 8.0], [-0.25, 3.0, 15.75], [16.5, -1.5, 2.0],
                   [31.25, 0.0, -16.0], [0.5, 0.5, 0.5]], dtype=np.float32)
  pos[0, :len(edge)] = edge
  wts = rng.random((2, n)).astype(np.float32)
  base = (100 * rng.random((2, nc, nc, nc))).astype(np.float32)
  out['pos'] = pos
  out['wts'] = wts
  out['base'] = base
  out['paint_w'] = np.asarray(
      u.cic_paint(tf.zeros((2, nc, nc, nc)), pos, weight=wts))
  out['paint_1'] = np.asarray(u.cic_paint(tf.zeros((2, nc, nc, nc)), pos))
  out['readout'] = np.asarray(u.cic_readout(base, pos))
  # Rectangular mesh.
  posr = (rng.random((1, 64, 3)) * np.array([8, 6, 10])).astype(np.float32)
  baser = rng.standard_normal((1, 8, 6, 10)).astype(np.float32)
  out['pos_rect'] = posr
  out['base_rect'] = baser
  out['paint_rect'] = np.asarray(u.cic_paint(tf.zeros((1, 8, 6, 10)), posr))
  out['readout_rect'] = np.asarray(u.cic_readout(baser, posr))
  # FFT normalisation round trip (tests/test_utils.py:51-61 uses FP64).
  f64 = rng.standard_normal((3, nc, nc, nc)) * 100
  out['rt_in'] = f64
  c = u.r2c3d(tf.constant(f64, dtype=tf.float64), dtype=tf.complex128)
  out['rt_k'] = np.asarray(c)
  out['rt_out'] = np.asarray(u.c2r3d(c, dtype=tf.float64))
  save('cic.npz', **out)


def gen_lpt(tf, m):
  tfpm, u, cosmology = m['tfpm'], m['utils'], m['cosmology']
  kt, pt = planck_table()
  ipklin = iuspline(kt, pt)
  out = {}
  for nc, bs, seed in [(16, 50., 100), (32, 100., 7)]:
    tag = 'n%d' % nc
    white = tf.random.normal([1, nc, nc, nc], stddev=(nc**3)**0.5, seed=seed)
    out[tag + '_white'] = np.asarray(white)
    lin = tfpm.linear_field(nc, bs, ipklin, batch_size=1, seed=seed)
    out[tag + '_linear'] = np.asarray(lin)
    lk = u.r2c3d(lin, norm=nc**3)
    grid = np.indices([nc] * 3).reshape(3, -1).T.astype(np.float32)[None]
    c = cosmology.Planck15()
    if nc == 16:
      out[tag + '_lpt1'] = np.asarray(tfpm.lpt1(lk, grid))
      out[tag + '_lpt2src'] = np.asarray(u.c2r3d(tfpm.lpt2_source(lk),
                                                 norm=nc**3))
      out[tag + '_init_o1'] = np.asarray(tfpm.lpt_init(c, lin, 0.1, order=1))
    out[tag + '_init_o2'] = np.asarray(tfpm.lpt_init(c, lin, 0.1, order=2))
  save('lpt.npz', **out)


def gen_nbody(tf, m):
  tfpm, u, cosmology = m['tfpm'], m['utils'], m['cosmology']
  lpt = np.load(os.path.join(HERE, 'lpt.npz'))
  stages = np.linspace(0.1, 1.0, 10)
  out = {'stages': stages}
  c = cosmology.Planck15()
  # 16^3, box 50 (the reference's tests/test_tfpm.py:130-183 setup).
  s0 = lpt['n16_init_o1']
  st = tfpm.nbody(c, s0, stages, 16)
  out['n16_b1_final'] = np.asarray(st)
  out['n16_b1_rho'] = np.asarray(u.cic_paint(tf.zeros((1, 16, 16, 16)),
                                             st[0]))
  st2 = tfpm.nbody(c, s0, stages, 16, pm_nc_factor=2)
  out['n16_b2_final'] = np.asarray(st2)
  inter = tfpm.nbody(c, s0, stages[:4], 16, return_intermediate_states=True)
  out['n16_inter_a'] = np.array([x[0] for x in inter])
  out['n16_inter'] = np.stack([np.asarray(x[1]) for x in inter])
  # Single force / kick / drift calls on the initial state.
  out['n16_force'] = np.asarray(tfpm.force(c, s0, [16, 16, 16]))
  out['n16_kick'] = np.asarray(tfpm.kick(c, s0, 0.1, 0.1, 0.12))
  out['n16_drift'] = np.asarray(tfpm.drift(c, s0, 0.1, 0.12, 0.15))
  # Rectangular 8 x 8 x 24 mesh, 2LPT, alternate cosmology.
  rng = np.random.default_rng(55)
  ca = cosmology.Planck15(**COSMOS['alt'])
  linr = tf.constant(rng.standard_normal((1, 8, 8, 24)).astype(np.float32) *
                     0.5)
  out['rect_linear'] = np.asarray(linr)
  sr = tfpm.lpt_init(ca, linr, 0.1, order=2)
  out['rect_init'] = np.asarray(sr)
  out['rect_final'] = np.asarray(tfpm.nbody(ca, sr, stages, [8, 8, 24]))
  # 32^3, box 100, Planck15, 2LPT at a0 = 0.1, 10 stages to a = 1.
  s32 = lpt['n32_init_o2']
  f32 = tfpm.nbody(c, s32, stages, 32)
  out['n32_final'] = np.asarray(f32)
  out['n32_rho'] = np.asarray(u.cic_paint(tf.zeros((1, 32, 32, 32)), f32[0]))
  save('nbody.npz', **out)


def gen_pgd(tf, m):
  """PGD correction (flowpm/tfpm.py:222-270 apply_pgd, :369-422 pgd, applied
  after every drift by nbody at :487-488) at 16^3: one (alpha, kl, ks) per
  step; kl, ks in the mesh's own k units."""
  tfpm, cosmology = m['tfpm'], m['cosmology']
  lpt = np.load(os.path.join(HERE, 'lpt.npz'))
  stages = np.linspace(0.1, 1.0, 10)
  c = cosmology.Planck15()
  s0 = lpt['n16_init_o1']
  params = np.stack([np.linspace(0.2, 0.4, 9), np.full(9, 0.6),
                     np.full(9, 3.0)], axis=1).astype(np.float32)
  out = {'stages': stages, 'params': params}
  out['single'] = np.asarray(tfpm.pgd(s0, tf.constant(params[0]), [16, 16, 16]))
  out['single_b2'] = np.asarray(
      tfpm.pgd(s0, tf.constant(params[0]), [16, 16, 16], pm_nc_factor=2))
  out['final'] = np.asarray(
      tfpm.nbody(c, s0, stages, 16, pgdparams=tf.constant(params)))
  out['final_b2'] = np.asarray(
      tfpm.nbody(c, s0, stages, 16, pm_nc_factor=2,
                 pgdparams=tf.constant(params)))
  save('pgd.npz', **out)


def gen_planes(tf, m):
  """2-D CIC paint (flowpm/utils.py:94-160 cic_paint_2d) and lensing density
  planes (flowpm/raytracing.py:49-109 density_plane)."""
  u = m['utils']
  sys.modules.setdefault('tensorflow_addons',
                         types.ModuleType('tensorflow_addons'))
  rt = importlib.import_module('flowpm.raytracing')
  rng = np.random.default_rng(77)
  out = {}
  pos = (rng.random((2, 600, 2)) * 36 - 6).astype(np.float32)
  pos[0, :8] = [[0, 0], [23.999999, 0.5], [-0.0, 24.0], [48.5, -24.25],
                [3.0, 7.0], [11.5, 11.5], [-1e-6, 23.5], [5.25, -0.75]]
  w = rng.random((2, 600)).astype(np.float32)
  mask = rng.random((2, 600)) < 0.7
  out['pos'], out['w'], out['mask'] = pos, w, mask
  z = tf.zeros((2, 24, 24))
  out['paint'] = np.asarray(u.cic_paint_2d(z, pos))
  out['paint_w'] = np.asarray(u.cic_paint_2d(z, pos, weight=w))
  out['paint_wm'] = np.asarray(u.cic_paint_2d(z, pos, weight=w, mask=mask))
  # rectangular 24 x 16: the reference wraps both axes by ny
  posr = np.stack([rng.random(400) * 24, rng.random(400) * 28 - 6],
                  axis=-1)[None].astype(np.float32)
  out['pos_rect'] = posr
  out['paint_rect'] = np.asarray(u.cic_paint_2d(tf.zeros((1, 24, 16)), posr))
  # density planes of an evolved 32^3 state (the C1 fixture)
  nb = np.load(os.path.join(HERE, 'nbody.npz'))
  st = nb['n32_final']
  out['dp_plane'] = np.asarray(
      rt.density_plane(st, 32, 16., 8., 48,
                       shift=np.array([0.3, 0.7, 0.], np.float32)))
  ang = np.float32(0.5)
  rot = np.array([[np.cos(ang), -np.sin(ang), 0], [np.sin(ang), np.cos(ang), 0],
                  [0, 0, 1]], np.float32)
  out['dp_rot'] = rot
  out['dp_plane_rot'] = np.asarray(
      rt.density_plane(st, 32, 26., 4., 40, rotation=rot,
                       shift=np.array([0.1, 0.2, 0.5], np.float32)))
  save('planes.npz', **out)


def gen_pk(tf, m):
  pk = m['pk']
  nb = np.load(os.path.join(HERE, 'nbody.npz'))
  lpt = np.load(os.path.join(HERE, 'lpt.npz'))
  out = {}
  for tag, field, bs in [('rho32', nb['n32_rho'], 100.),
                         ('lin16', lpt['n16_linear'], 50.)]:
    field = tf.constant(field)
    kb, p = pk.power_spectrum(field, kmin=0.1, dk=0.05,
                              boxsize=np.array([bs] * 3))
    out[tag + '_field'] = np.asarray(field)
    out[tag + '_k'] = np.asarray(kb)
    out[tag + '_pk'] = np.asarray(p)
    out[tag + '_boxsize'] = np.array(bs)
  save('pk.npz', **out)


def main():
  tf, m = load_reference()
  gen_kernels(m)
  gen_background(m)
  gen_power(m)
  gen_cic(tf, m)
  gen_lpt(tf, m)
  gen_nbody(tf, m)
  gen_pk(tf, m)
  gen_pgd(tf, m)
  gen_planes(tf, m)


if __name__ == '__main__':
  if len(sys.argv) > 1:  # named generators only, e.g. `pgd`
    tf, m = load_reference()
    for name in sys.argv[1:]:
      globals()['gen_' + name](tf, m)
  else:
    main()
