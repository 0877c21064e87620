"""The allocation-free power-spectrum binning entry point, fpm_pk_bin_noalloc,
called through the C ABI.

It exists for callers that cannot let a library allocate device memory
(their own memory pool owns the GPU, or allocation is forbidden after
start-up), so its bin sums live in a fixed device array inside the
library.  It must give the same P(k) as the allocating fpm_pk_bin, also on
a second call, which starts from whatever the first call left in that
array.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch
from numpy.testing import assert_allclose

pytestmark = pytest.mark.gpu

NEDGES_ARGS = dict(kmin=0.05, dk=0.02)


def _spectrum(seed, shape):
  g = torch.Generator(device='cpu').manual_seed(seed)
  field = torch.randn(shape, generator=g).to('cuda')
  return torch.fft.rfftn(field, dim=(-3, -2, -1)).to(torch.complex64)


def _call(lib, name, spec, box, nedges, out):
  B, nx, ny, _ = spec.shape
  nz = 2 * (spec.shape[3] - 1)
  boxd = (ctypes.c_double * 3)(*box)
  return getattr(lib, name)(
      ctypes.c_void_p(spec.data_ptr()), B, nx, ny, nz, boxd,
      ctypes.c_double(NEDGES_ARGS['kmin']), ctypes.c_double(NEDGES_ARGS['dk']),
      nedges, ctypes.c_void_p(out.data_ptr()),
      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_pk_bin_noalloc_matches_allocating_entry(cuda):
  from flowpm_b200 import _lib
  from flowpm_b200.pk import pk_edges
  lib = _lib.lib
  box = [40.0, 60.0, 80.0]
  shape = (2, 16, 24, 32)
  nedges = len(pk_edges(shape[1:], box, **NEDGES_ARGS))
  # Two calls in a row on different fields: the second must not see the
  # sums the first left in the shared array.
  for seed in (1, 2):
    spec = _spectrum(seed, shape)
    ref = torch.empty((shape[0], nedges - 1), device='cuda')
    got = torch.full_like(ref, float('nan'))
    assert _call(lib, 'fpm_pk_bin', spec, box, nedges, ref) == 0
    assert _call(lib, 'fpm_pk_bin_noalloc', spec, box, nedges, got) == 0
    torch.cuda.synchronize()
    assert_allclose(got.cpu().numpy(), ref.cpu().numpy(), rtol=1e-6)
  # Exactly at the limit (2 * 8 * 1024 = 16384 doubles, bins summed in
  # shared memory first), and at the limit with more bins than a
  # shared-memory histogram holds (2 * 2 * 4096), both twice in a row.
  for batch, nedges in ((8, 1023), (2, 4095), (1, 4000)):
    for seed in (4, 5):
      spec = _spectrum(seed, (batch, 8, 8, 8))
      ref = torch.empty((batch, nedges - 1), device='cuda')
      got = torch.full_like(ref, float('nan'))
      assert _call(lib, 'fpm_pk_bin', spec, box, nedges, ref) == 0
      assert _call(lib, 'fpm_pk_bin_noalloc', spec, box, nedges, got) == 0
      torch.cuda.synchronize()
      # bins that no mode reaches are 0/0 in both
      assert_allclose(got.cpu().numpy(), ref.cpu().numpy(), rtol=1e-6,
                      equal_nan=True)
  # Requests beyond the fixed array are refused before any work.
  assert _lib.FPM_ERR_LIMIT == 9
  big = torch.empty((64, 8200), device='cuda')
  spec = _spectrum(3, (64, 4, 4, 4))
  assert _call(lib, 'fpm_pk_bin_noalloc', spec, box, 8200, big) == 9
  # one double past the array: 2 * 1 * (8192 + 1) > 16384
  spec = _spectrum(3, (1, 4, 4, 4))
  assert _call(lib, 'fpm_pk_bin_noalloc', spec, box, 8192, big) == 9
  assert lib.fpm_error_string(9).startswith(b'request exceeds')
