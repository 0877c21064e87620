"""Many simulations of one shape streamed through the GPU from host memory.

``nbody`` takes device tensors, so a caller that holds initial states on
the host pays a host-to-device copy before every simulation and a
device-to-host copy after it, each waiting for the other.  ``NBodyStream``
overlaps them with the computation: the upload of simulation i+1 and the
download of simulation i-1 run on two copy streams while simulation i
integrates on the compute stream (double-buffered device staging, ordered
by CUDA events).  Each simulation is the same leapfrog as ``nbody``
(flowpm/tfpm.py:425-503), replayed as one CUDA graph of the library.
"""
import numpy as np
import torch

from . import _lib
from . import tfbackground as bg
from ._plans import Plan

__all__ = ['NBodyStream', 'nbody_stream']


def _nc3(nc):
  return [nc] * 3 if isinstance(nc, int) else [int(n) for n in nc]


class NBodyStream(object):
  """Pipeline of forward simulations with fixed ``cosmo``, ``stages``,
  ``nc``, batch size and ``pm_nc_factor``.

  ``run(states)`` takes host states (3 or 2, batch, npart, 3) -- X and P are
  read, F is recomputed -- preferably in pinned memory, and writes each
  final state (3, batch, npart, 3) to pinned host memory.  ``depth``
  simulations are in flight at once (2: one uploading or downloading while
  one computes)."""

  def __init__(self, cosmo, stages, nc, batch_size=1, pm_nc_factor=1,
               depth=2):
    self.nc = _nc3(nc)
    self.B = int(batch_size)
    stages = [float(s) for s in np.asarray(stages).ravel()]
    if len(stages) < 2:
      raise ValueError('at least one leapfrog step (two stages) is needed')
    if depth < 1:
      raise ValueError('depth must be >= 1')
    self.T = len(stages) - 1
    self.depth = int(depth)
    self.npart = int(np.prod(self.nc))
    self.plan = Plan([tuple(self.nc) + (int(pm_nc_factor),)] * self.B)
    coefs = np.tile(bg.nbody_coefficients(cosmo, stages)[None], (self.B, 1, 1))
    _lib.call('fpm_nbody_set_steps', self.plan.handle, self.T,
              _lib.ivec([self.T] * self.B), _lib.dvec(coefs.ravel()),
              _lib.dvec([1.5 * cosmo.Omega_m] * self.B), _lib.stream_ptr())
    shape = (self.B, self.npart, 3)
    self.dev_in = [torch.empty((2,) + shape, device='cuda')
                   for _ in range(self.depth)]
    self.dev_out = [torch.empty((3,) + shape, device='cuda')
                    for _ in range(self.depth)]
    self.s_in = torch.cuda.Stream()
    self.s_out = torch.cuda.Stream()
    ev = lambda: [torch.cuda.Event() for _ in range(self.depth)]
    self.in_ready, self.in_free = ev(), ev()
    self.out_ready, self.out_free = ev(), ev()
    self.count = 0  # simulations issued
    # the autotuner's cached choice for this shape and step count, if a
    # tuned nbody call has made one (the stream has no state to time on)
    self.plan.apply_tuned()
    self.plan.nbody_graph(self.T)  # capture now, before any copy is in flight

  def host_buffers(self, n):
    """``n`` pinned host tensors for the outputs of ``run``."""
    return [torch.empty((3, self.B, self.npart, 3), dtype=torch.float32,
                        pin_memory=True) for _ in range(n)]

  def run(self, states, out=None, before_each=None):
    """Issue one simulation per host state; returns the output host
    tensors (``out`` if given, else freshly pinned ones).  Asynchronous:
    call ``synchronize`` before reading them.  ``before_each``, if given,
    is called on the compute stream before each simulation (benchmarks use
    it to evict L2)."""
    states = list(states)
    if out is None:
      out = self.host_buffers(len(states))
    if len(out) < len(states):
      raise ValueError('need one output buffer per state')
    comp = torch.cuda.current_stream()
    st = _lib.stream_ptr()
    d, p, f = self.plan.work()
    nx, ny, nz = self.nc
    for i, hs in enumerate(states):
      if tuple(hs.shape[1:]) != (self.B, self.npart, 3) or hs.shape[0] < 2:
        raise ValueError('state must be (3, %d, %d, 3)' % (self.B,
                                                          self.npart))
      k = self.count % self.depth
      reuse = self.count >= self.depth
      with torch.cuda.stream(self.s_in):
        if reuse:
          self.s_in.wait_event(self.in_free[k])
        self.dev_in[k].copy_(hs[:2], non_blocking=True)
        self.in_ready[k].record(self.s_in)
      comp.wait_event(self.in_ready[k])
      if before_each is not None:
        before_each()
      _lib.call('fpm_lattice_shift', _lib.ptr(self.dev_in[k][0]), _lib.ptr(d),
                self.B, nx, ny, nz, -1, st)
      p.copy_(self.dev_in[k][1].reshape(-1, 3))
      self.in_free[k].record(comp)
      self.plan.launch_nbody(self.T, st)
      if reuse:
        comp.wait_event(self.out_free[k])
      o = self.dev_out[k]
      _lib.call('fpm_lattice_shift', _lib.ptr(d), _lib.ptr(o[0]), self.B, nx,
                ny, nz, 1, st)
      o[1].copy_(p.reshape(o[1].shape))
      o[2].copy_(f.reshape(o[2].shape))
      self.out_ready[k].record(comp)
      with torch.cuda.stream(self.s_out):
        self.s_out.wait_event(self.out_ready[k])
        out[i].copy_(o, non_blocking=True)
        self.out_free[k].record(self.s_out)
      self.count += 1
    return out[:len(states)]

  def synchronize(self):
    """Wait for every issued copy and simulation."""
    self.s_out.synchronize()
    torch.cuda.current_stream().synchronize()

  def status(self):
    """Device status word (non-zero: a non-finite state was seen)."""
    return self.plan.status()

  def close(self):
    torch.cuda.synchronize()
    self.plan.close()


def nbody_stream(cosmo, states, stages, nc, pm_nc_factor=1,
                 check_finite=True):
  """``nbody`` on each host state of ``states`` (each (3, B, Np, 3) on the
  host), with the host copies overlapped; returns the final states as
  pinned host tensors in the same order."""
  states = list(states)
  if not states:
    return []
  s = NBodyStream(cosmo, stages, nc, batch_size=states[0].shape[1],
                  pm_nc_factor=pm_nc_factor)
  try:
    out = s.run(states)
    s.synchronize()
    if check_finite and s.status():
      raise _lib.FlowPMError('nbody_stream', _lib.FPM_ERR_NONFINITE)
    return out
  finally:
    s.close()
