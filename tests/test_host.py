"""Host-side logic of flowpm_b200 (no GPU): the FP64 background, P(k), the
kernels.py drop-ins, step prefactors, the linear-field amplitude table and
the C ABI (library loads, exports every declared symbol, rejects bad
arguments before touching the device)."""
import ctypes
import os
import re

import numpy as np
import pytest
from numpy.testing import assert_allclose

from conftest import ROOT, golden, pk_table
from oracle import background as obg
from oracle import pm as opm

ALT = dict(Omega_c=0.30, Omega_b=0.045, h=0.70, sigma8=0.75, n_s=0.96)


@pytest.fixture(scope='module')
def fpm():
  import flowpm_b200
  return flowpm_b200


def test_cosmology_mirror(fpm):
  c = fpm.cosmology.Planck15()
  assert c.Omega_m == pytest.approx(0.2589 + 0.0486)
  assert c.Omega_de == pytest.approx(1 - 0.2589 - 0.0486)
  assert c.k == 0 and c.sqrtk == 0.0
  c2 = fpm.cosmology.Planck15(Omega_c=0.3)
  assert c2.Omega_c == 0.3 and c2.to_dict()['sigma8'] == 0.8159


@pytest.mark.parametrize('tag,kw', [('planck15', {}), ('alt', ALT)])
def test_background_fp64_vs_reference(fpm, tag, kw):
  """FP64 background = the reference's method in double precision: within
  FP32 rounding of the reference's float32 numbers, and equal (1e-12) to
  the oracle run in float64."""
  z = golden('background')
  c = fpm.cosmology.Planck15(**kw)
  o64 = obg.Background(kw, dtype=np.float64)
  for fn in ['E', 'dEa', 'Omega_m_a', 'Omega_de_a', 'D1', 'D2', 'D1f', 'D2f',
             'f1', 'f2', 'Gf', 'Gf2', 'gf', 'gf2']:
    got = getattr(fpm.tfbackground, fn)(c, z['a_eval'])
    assert_allclose(got, z['%s_%s' % (tag, fn)], rtol=2e-5, err_msg=fn)
    assert_allclose(got, getattr(o64, fn)(z['a_eval']), rtol=1e-12,
                    err_msg=fn)


def test_background_vs_legacy(fpm):
  z = golden('background')
  c = fpm.cosmology.Planck15()
  bg = fpm.tfbackground
  assert_allclose(bg.E(c, z['legacy_a3']), z['legacy_E'], rtol=1e-4)
  assert_allclose(bg.dEa(c, z['legacy_a3']), z['legacy_Eprime'], rtol=1e-4)
  a = z['legacy_a']
  for mine, ref in [('D1', 'D1'), ('D2', 'D2'), ('D1f', 'gp'),
                    ('D2f', 'gp2'), ('f1', 'f1'), ('f2', 'f2'), ('Gf', 'Gf'),
                    ('Gf2', 'Gf2'), ('gf', 'gf'), ('gf2', 'gf2')]:
    assert_allclose(getattr(bg, mine)(c, a), z['legacy_' + ref], rtol=1e-2)


def test_step_coefficients(fpm):
  c = fpm.cosmology.Planck15()
  stages = np.linspace(0.1, 1.0, 10)
  co = fpm.tfbackground.nbody_coefficients(c, stages)
  o64 = obg.Background({}, dtype=np.float64)
  for i in range(9):
    a0, a1 = stages[i], stages[i + 1]
    ah = (a0 * a1)**0.5
    assert co[i, 0] == pytest.approx(float(o64.kick_factor(a0, a0, ah)),
                                     rel=1e-12)
    assert co[i, 1] == pytest.approx(float(o64.drift_factor(a0, ah, a1)),
                                     rel=1e-12)
    assert co[i, 2] == pytest.approx(float(o64.kick_factor(ah, a1, a1)),
                                     rel=1e-12)
  lc = fpm.tfbackground.lpt_coefficients(c, 0.1)
  assert lc[0] == pytest.approx(float(o64.D1(0.1)), rel=1e-12)
  assert lc[4] == pytest.approx(
      0.01 * float(o64.E(0.1) * o64.gf(0.1) / o64.D1(0.1)), rel=1e-12)


def test_power_fp64(fpm):
  z = golden('power')
  for tag, kw in [('planck15', {}), ('alt', ALT)]:
    c = fpm.cosmology.Planck15(**kw)
    assert_allclose(fpm.tfpower.linear_matter_power(c, z['k']),
                    z[tag + '_pk'], rtol=2e-4)
    assert_allclose(
        fpm.tfpower.Eisenstein_Hu(c, z['k'], type='eisenhu'),
        z[tag + '_T_eisenhu'], rtol=1e-5)


def test_kernels_dropin_exact(fpm):
  z = golden('kernels')
  k = fpm.kernels
  for tag, shape in [('c8', [8, 8, 8]), ('r4610', [4, 6, 10])]:
    kv = k.fftk(shape, symmetric=False)
    for d in range(3):
      assert np.array_equal(kv[d], z['%s_fftk_%d' % (tag, d)])
      assert np.array_equal(
          k.fftk(shape, symmetric=True)[d], z['%s_fftk_sym_%d' % (tag, d)])
      assert np.array_equal(k.gradient_kernel(kv, d),
                            z['%s_grad1_%d' % (tag, d)])
      assert np.array_equal(k.gradient_kernel(kv, d, order=0),
                            z['%s_grad0_%d' % (tag, d)])
    assert np.array_equal(k.laplace_kernel(kv), z[tag + '_laplace'])
    assert np.array_equal(k.longrange_kernel(kv, 1.3),
                          z[tag + '_longrange_r1p3'])
    assert np.array_equal(k.cic_compensation(kv), z[tag + '_ciccomp'])


@pytest.mark.parametrize('nc,box', [(16, 50.), ([8, 6, 10], [40., 30., 50.])])
def test_linear_amplitude(fpm, nc, box):
  pk = pk_table()
  amp = fpm.tfpm.linear_amplitude(nc, box, pk)
  n3 = [nc] * 3 if isinstance(nc, int) else nc
  b3 = [box] * 3 if isinstance(box, float) else box
  kv = opm.fftk(n3, symmetric=False)
  km = sum((kk / b3[i] * n3[i])**2 for i, kk in enumerate(kv))**0.5
  ref = (pk(km) / (b3[0] * b3[1] * b3[2]))**0.5
  assert_allclose(amp, ref[:, :, :n3[2] // 2 + 1], rtol=1e-6)


def test_linear_amplitude_caller_kvec(fpm):
  """A caller's per-axis k grid (here fftk's, rescaled per axis) gives the
  amplitude of the reference formula on that grid; grids whose |k| is not
  mirror-symmetric, or not per-axis, are refused."""
  pk = pk_table()
  n3, b3 = [8, 6, 10], [40., 30., 50.]
  kv = [k * s for k, s in zip(opm.fftk(n3, symmetric=False), (1.5, 0.7, 2.))]
  amp = fpm.tfpm.linear_amplitude(n3, b3, pk, kvec=kv)
  km = sum((kk / b3[i] * n3[i])**2 for i, kk in enumerate(kv))**0.5
  ref = (pk(km) / (b3[0] * b3[1] * b3[2]))**0.5
  assert_allclose(amp, ref[:, :, :n3[2] // 2 + 1], rtol=1e-6)
  default = fpm.tfpm.linear_amplitude(16, 50., pk)
  same = fpm.tfpm.linear_amplitude(16, 50., pk,
                                   kvec=opm.fftk([16] * 3, symmetric=False))
  assert_allclose(same, default, rtol=1e-6)
  skew = [k.copy() for k in kv]
  skew[1] = skew[1] + 0.1
  with pytest.raises(NotImplementedError):
    fpm.tfpm.linear_amplitude(n3, b3, pk, kvec=skew)
  with pytest.raises(NotImplementedError):
    fpm.tfpm.linear_amplitude(n3, b3, pk, kvec=[np.ravel(k) for k in kv])


# --------------------------------------------------------------------------
# C ABI
# --------------------------------------------------------------------------
def declared_symbols():
  with open(os.path.join(ROOT, 'include', 'flowpm_b200.h')) as f:
    src = f.read()
  src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
  return sorted(set(re.findall(r'\b(fpm_[a-z0-9_]+)\s*\(', src)))


def test_library_exports_declared_symbols(fpm):
  lib = ctypes.CDLL(fpm._lib.LIB_PATH)
  names = declared_symbols()
  assert len(names) >= 15
  for name in names:
    assert hasattr(lib, name), name
  assert set(names) == set(fpm._lib.SIGNATURES), (
      set(names) ^ set(fpm._lib.SIGNATURES))


def test_capi_rejects_bad_arguments(fpm):
  L = fpm._lib.lib
  assert L.fpm_version() >= 100
  assert L.fpm_error_string(1) == b'invalid argument'
  # null pointers / bad shapes are rejected on the host, before any CUDA call
  assert L.fpm_cic_paint(None, 1, 8, 8, 8, None, 10, None, None) == 1
  assert L.fpm_cic_paint(ctypes.c_void_p(8), 0, 8, 8, 8, None, 0, None,
                         None) == 1
  assert L.fpm_cic_readout(None, 1, 8, 8, 8, None, 1, None, None) == 1
  assert L.fpm_cic_neighbours(0, 8, 8, None, 1, None, None, None) == 1
  assert L.fpm_saxpy(None, None, ctypes.c_float(1.0), 5, None) == 1
  assert L.fpm_saxpy(None, None, ctypes.c_float(1.0), 0, None) == 0
  h = ctypes.c_void_p()
  dims = fpm._lib.ivec([16, 16, 16, 0])
  assert L.fpm_plan_create(ctypes.byref(h), 1, dims, 0.0, 0) == 1
  dims = fpm._lib.ivec([1, 16, 16, 1])
  assert L.fpm_plan_create(ctypes.byref(h), 1, dims, 0.0, 0) == 1
  assert L.fpm_plan_create(ctypes.byref(h), 0, dims, 0.0, 0) == 1
  assert L.fpm_plan_destroy(None) == 1
  assert L.fpm_nbody_run(None, None, None, None, None, 0, None, 0, None) == 1
  assert L.fpm_nbody_adjoint(None, None, None, None, None, None, None, None,
                             0, None) == 1


def test_c_host_builds_and_calls_the_library(fpm, tmp_path):
  """A C99 host (no C++) includes include/flowpm_b200.h, links
  libflowpm_b200.so and calls it the way a non-Python caller of the
  drop-in would: version, error text, and argument checks that return
  before any device work (so it runs without a GPU)."""
  import shutil
  import subprocess
  if shutil.which('gcc') is None:
    pytest.skip('no C compiler')
  src = tmp_path / 'host.c'
  src.write_text(r"""
#include <stdio.h>
#include <string.h>
#include "flowpm_b200.h"
int main(void) {
  fpm_plan* plan = NULL;
  int32_t dims[4] = {16, 16, 16, 0};   /* pm_nc_factor 0: rejected */
  if (fpm_version() < 100) return 2;
  if (strcmp(fpm_error_string(FPM_ERR_ARG), "invalid argument") != 0)
    return 3;
  if (fpm_plan_create(&plan, 1, dims, 0.0, 0) != FPM_ERR_ARG) return 4;
  if (fpm_cic_paint(NULL, 1, 8, 8, 8, NULL, 10, NULL, NULL) != FPM_ERR_ARG)
    return 5;
  if (fpm_plan_set_binning(NULL, 16, 4, FPM_BIN_CHUNKS) != FPM_ERR_ARG)
    return 6;
  if (fpm_pk_bin_noalloc(NULL, 1, 8, 8, 8, NULL, 0.0, 0.1, 4, NULL, NULL) !=
      FPM_ERR_ARG)
    return 7;
  printf("ok %d\n", fpm_version());
  return 0;
}
""")
  libdir = os.path.dirname(fpm._lib.LIB_PATH)
  exe = tmp_path / 'host'
  cmd = ['gcc', '-std=c99', '-Wall', '-Werror', '-o', str(exe), str(src),
         '-I', os.path.join(ROOT, 'include'), '-L', libdir, '-lflowpm_b200',
         '-Wl,-rpath,' + libdir]
  subprocess.run(cmd, check=True, capture_output=True)
  out = subprocess.run([str(exe)], capture_output=True, text=True)
  assert out.returncode == 0, (out.returncode, out.stderr)
  assert out.stdout.startswith('ok ')


def test_product_does_not_import_oracle():
  """The product package never references the oracle."""
  pkg = os.path.join(ROOT, 'flowpm_b200')
  for dirpath, _, files in os.walk(pkg):
    for f in files:
      if f.endswith(('.py', '.cu', '.cuh', '.h')):
        with open(os.path.join(dirpath, f)) as fh:
          src = fh.read()
        assert 'oracle' not in src, f
