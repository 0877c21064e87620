import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
  config.addinivalue_line(
      'markers', 'gpu: needs a CUDA device (B200) and the built library')


def golden(name):
  return np.load(os.path.join(GOLDEN, name + '.npz'))


@pytest.fixture(scope='session')
def cuda():
  import torch
  if not torch.cuda.is_available():
    pytest.fail('GPU test run without a CUDA device')
  import flowpm_b200  # noqa: F401  (loads the CUDA library, fails loudly)
  return torch.device('cuda:0')


def pk_table():
  """The nbodykit EH P(k) table of the reference (flowpm/data/
  Planck15_a1p00.txt), stored in the power fixture, as a spline."""
  from scipy.interpolate import InterpolatedUnivariateSpline as iuspline
  z = golden('power')
  return iuspline(z['nbodykit_k'], z['nbodykit_pk'])


def rel_l2(a, b):
  a = np.asarray(a, dtype=np.float64)
  b = np.asarray(b, dtype=np.float64)
  return float(np.linalg.norm(a - b) / np.linalg.norm(b))
