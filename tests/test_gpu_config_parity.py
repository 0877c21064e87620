"""Parity at the size of the headline configuration (C2: 128^3 particles on a
128^3 mesh, box 200 Mpc/h, Planck15, seeded Eisenstein-Hu Gaussian initial
field, 2LPT at a0 = 0.1, 40 kick-drift-kick steps to a = 1).

The CUDA path (through the C ABI) and the oracle start from the same linear
field (the noise cannot be shared with the reference's TensorFlow stream,
so parity is defined from lpt_init downward).  Bars: final CIC density
within 1e-4 relative L2 and P(k) within 1e-4 per bin of the FP32 oracle,
the reference's own arithmetic; the error of both against the FP64 oracle
(the same method in double) is printed.  The two oracle runs take about a
minute on 16 host cores.
"""
import os

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import background as obg
from oracle import pm as opm

pytestmark = pytest.mark.gpu

N, BOX, A0, STEPS, SEED = 128, 200.0, 0.1, 40, 1000


@pytest.fixture(scope='module')
def fpm(cuda):
  import flowpm_b200
  return flowpm_b200


def eh_pk(fpm, cosmo):
  kk = np.logspace(-4, 2, 4096)
  pk = fpm.tfpower.linear_matter_power(cosmo, kk)
  return lambda k: np.interp(np.log(np.maximum(k, 1e-30)), np.log(kk), pk,
                             left=0.0)


def oracle_density(lin, stages, dtype):
  """Final CIC density of the oracle's 2LPT + nbody in float32 or float64."""
  torch.set_num_threads(os.cpu_count() or 1)
  b = obg.Background({}, dtype=np.float32 if dtype == torch.float32
                     else np.float64)
  s = opm.lpt_init(b, torch.tensor(lin, dtype=dtype), A0, order=2)
  s = opm.nbody(b, s, stages, N)
  return opm.cic_paint(torch.zeros((1, N, N, N), dtype=dtype), s[0]).numpy()


def pk_bins(rho):
  _, p = opm.power_spectrum(torch.tensor(rho, dtype=torch.float64),
                            kmin=0.02, dk=0.02, boxsize=np.array([BOX] * 3))
  return p.numpy()


def test_c2_density_and_pk_against_oracle(fpm, capsys):
  cosmo = fpm.cosmology.Planck15()
  stages = np.linspace(A0, 1.0, STEPS + 1)
  lin = fpm.linear_field(N, BOX, eh_pk(fpm, cosmo), seed=SEED)
  st = fpm.nbody(cosmo, fpm.lpt_init(cosmo, lin, A0, order=2), stages, N)
  rho = fpm.cic_paint(torch.zeros((1, N, N, N), device='cuda'), st[0])
  rho = rho.cpu().numpy()
  lin = lin.cpu().numpy()
  rho32 = oracle_density(lin, stages, torch.float32)
  rho64 = oracle_density(lin, stages, torch.float64)
  err32 = rel_l2(rho, rho32)
  pk, pk32, pk64 = pk_bins(rho), pk_bins(rho32), pk_bins(rho64)
  ok = np.isfinite(pk32) & (pk32 != 0)
  pk_err32 = float(np.max(np.abs(pk[ok] - pk32[ok]) / np.abs(pk32[ok])))
  pk_err64 = float(np.max(np.abs(pk[ok] - pk64[ok]) / np.abs(pk64[ok])))
  with capsys.disabled():
    print('\n  C2 128^3 / 40 steps: density rel-L2 vs FP32 oracle %.2e, vs '
          'FP64 oracle %.2e (FP32 oracle vs FP64 %.2e); P(k) max rel vs '
          'FP32 %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e)' %
          (err32, rel_l2(rho, rho64), rel_l2(rho32, rho64), pk_err32,
           pk_err64, float(np.max(np.abs(pk32[ok] - pk64[ok]) /
                                  np.abs(pk64[ok])))))
  assert err32 <= 1e-4, err32
  assert pk_err32 <= 1e-4, pk_err32
