"""Many simulations of uneven size advanced together.

``nbody_many`` (and the reusable ``BatchRunner`` behind it) runs a list of
independent simulations -- each with its own mesh, cosmology, stage list
and ``pm_nc_factor`` -- as ONE plan of the C library: every op is one
persistent launch over all simulations, equal-shaped simulations share
batched cuFFT plans, simulations that have finished their steps drop out of
the transforms, and the whole leapfrog is one CUDA graph replay.  Results
are those of calling ``nbody`` on each simulation separately.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from . import tfbackground as bg
from ._plans import Plan, tune
from .utils import as_cuda

__all__ = ['BatchRunner', 'nbody_many']


def _nc3(nc):
  return [nc] * 3 if isinstance(nc, int) else [int(n) for n in nc]


class BatchRunner(object):
  """One plan and one leapfrog graph for a fixed set of simulations.

  ``sims`` is a list of dicts with keys ``nc`` (int or 3 ints), ``cosmo``,
  ``stages`` and optionally ``pm_nc_factor``.  Simulations are reordered
  internally (by shape, then by decreasing step count) so that the finished
  ones form a suffix of each equal-shaped run."""

  def __init__(self, sims):
    self.specs = []
    for s in sims:
      nc = _nc3(s['nc'])
      stages = [float(a) for a in np.asarray(s['stages']).ravel()]
      if len(stages) < 1:
        raise ValueError('each simulation needs at least one stage')
      self.specs.append(dict(nc=nc, cosmo=s['cosmo'], stages=stages,
                             bf=int(s.get('pm_nc_factor', 1)),
                             T=len(stages) - 1))
    n = len(self.specs)
    self.order = sorted(range(n), key=lambda i: (
        tuple(self.specs[i]['nc']), self.specs[i]['bf'], -self.specs[i]['T']))
    dims = [tuple(self.specs[i]['nc']) + (self.specs[i]['bf'],)
            for i in self.order]
    self.plan = Plan(dims)
    self.max_steps = max(sp['T'] for sp in self.specs)
    coefs, nsteps, ffac, self.offsets = [], [], [], []
    off = 0
    for i in self.order:
      sp = self.specs[i]
      co = np.zeros((self.max_steps, 3))
      if sp['T'] > 0:
        co[:sp['T']] = bg.nbody_coefficients(sp['cosmo'], sp['stages'])
      coefs.append(co)
      nsteps.append(sp['T'])
      ffac.append(1.5 * sp['cosmo'].Omega_m)
      npart = int(np.prod(sp['nc']))
      self.offsets.append((off, npart))
      off += npart
    self._steps = (self.max_steps, nsteps, np.concatenate(coefs).ravel(),
                   ffac)
    self.d, self.p, self.f = self.plan.work()
    self._graph = None
    self._binning_set = False

  def _set_steps(self, st):
    T, nsteps, coefs, ffac = self._steps
    _lib.call('fpm_nbody_set_steps', self.plan.handle, T, _lib.ivec(nsteps),
              _lib.dvec(coefs), _lib.dvec(ffac), st)

  def load(self, states):
    """Copy the initial states (one (3, 1, Np, 3) or (3, Np, 3) tensor per
    simulation, in the caller's order) into the plan's buffers."""
    st = _lib.stream_ptr()
    for slot, i in enumerate(self.order):
      sp = self.specs[i]
      off, npart = self.offsets[slot]
      x = as_cuda(states[i]).reshape(3, npart, 3)
      nx, ny, nz = sp['nc']
      _lib.call('fpm_lattice_shift', _lib.ptr(x[0]),
                _lib.ptr(self.d[off:off + npart]), 1, nx, ny, nz, -1, st)
      self.p[off:off + npart].copy_(x[1])

  def run(self):
    """Advance every loaded simulation through its stages (graph replay)."""
    st = _lib.stream_ptr()
    if self._graph is None:
      self._set_steps(st)
      if not self._binning_set:
        tune(self.plan, self.d, self.p, (self.max_steps, False))
      g = ctypes.c_void_p()
      _lib.call('fpm_graph_capture_nbody', self.plan.handle,
                _lib.ptr(self.d), _lib.ptr(self.p), _lib.ptr(self.f), None, 0,
                None, 0, ctypes.byref(g))
      self._graph = g
    code = _lib.lib.fpm_graph_launch(self._graph, st)
    if code == _lib.FPM_ERR_STATE:  # tables moved: recapture once
      _lib.lib.fpm_graph_destroy(self._graph)
      self._graph = None
      self._set_steps(st)
      return self.run()
    _lib.check('fpm_graph_launch', code)

  def results(self):
    """Final states (3, 1, Np, 3), in the caller's order."""
    st = _lib.stream_ptr()
    out = [None] * len(self.specs)
    for slot, i in enumerate(self.order):
      sp = self.specs[i]
      off, npart = self.offsets[slot]
      nx, ny, nz = sp['nc']
      s = torch.empty((3, 1, npart, 3), dtype=torch.float32, device='cuda')
      _lib.call('fpm_lattice_shift', _lib.ptr(self.d[off:off + npart]),
                _lib.ptr(s[0]), 1, nx, ny, nz, 1, st)
      s[1, 0].copy_(self.p[off:off + npart])
      s[2, 0].copy_(self.f[off:off + npart])
      out[i] = s
    return out

  def set_binning(self, tile, sort_every=1, mode=_lib.FPM_BIN_CHUNKS):
    """Binned forward step for this batch (see ``Plan.set_binning``)."""
    if self._graph is not None:
      _lib.lib.fpm_graph_destroy(self._graph)
      self._graph = None
    self.plan.set_binning(tile, sort_every, mode)
    self._binning_set = True

  def status(self):
    return self.plan.status()

  def close(self):
    if self._graph is not None:
      _lib.lib.fpm_graph_destroy(self._graph)
      self._graph = None
    self.plan.close()


def nbody_many(sims, states, check_finite=True):
  """Run ``nbody`` on every simulation of ``sims`` (see ``BatchRunner``)
  from ``states`` (one per simulation) in one batched launch sequence;
  returns the final states in the same order."""
  r = BatchRunner(sims)
  try:
    r.load(states)
    r.run()
    out = r.results()
    if check_finite and r.status():
      raise _lib.FlowPMError('nbody_many', _lib.FPM_ERR_NONFINITE)
    return out
  finally:
    r.close()
