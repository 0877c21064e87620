"""Plan objects of the C library (``fpm_plan_create``) and their cache.

A plan owns the cuFFT plans and mesh work buffers of one set of
simulations; creating it allocates device memory, so plans are cached per
(device, dims, options) and reused across calls.
"""
import ctypes

import torch

from . import _lib


class Plan(object):
  """One ``fpm_plan``: ``dims`` is a list of (nx, ny, nz, pm_nc_factor)."""

  def __init__(self, dims, r_split=0.0, flags=0):
    self.dims = [tuple(int(v) for v in d) for d in dims]
    self.flags = int(flags)
    self.r_split = float(r_split)
    flat = [v for d in self.dims for v in d]
    h = ctypes.c_void_p()
    _lib.call('fpm_plan_create', ctypes.byref(h), len(self.dims),
              _lib.ivec(flat), self.r_split, self.flags)
    self.handle = h
    np_tot, nbytes = ctypes.c_int64(), ctypes.c_int64()
    _lib.call('fpm_plan_info', h, ctypes.byref(np_tot), ctypes.byref(nbytes))
    self.total_particles = np_tot.value
    self.device_bytes = nbytes.value
    self._work = None
    self._graphs = {}

  @property
  def nsims(self):
    return len(self.dims)

  def status(self, stream=None):
    """Read and clear the device status word (synchronises the stream)."""
    v = ctypes.c_int32()
    _lib.call('fpm_plan_status', self.handle, ctypes.byref(v),
              stream or _lib.stream_ptr())
    return v.value

  def work(self):
    """Persistent (disp, mom, force) buffers of the plan, (total_np, 3)."""
    if self._work is None:
      shape = (self.total_particles, 3)
      self._work = tuple(
          torch.empty(shape, dtype=torch.float32, device='cuda')
          for _ in range(3))
    return self._work

  def nbody_graph(self, max_steps):
    """CUDA graph of one leapfrog run of ``max_steps`` on the work buffers
    (captured once per step count; the step tables are read at replay)."""
    g = self._graphs.get(('nbody', max_steps))
    if g is None:
      d, p, f = self.work()
      g = ctypes.c_void_p()
      _lib.call('fpm_graph_capture_nbody', self.handle, _lib.ptr(d),
                _lib.ptr(p), _lib.ptr(f), None, 0, None, 0, ctypes.byref(g))
      self._graphs[('nbody', max_steps)] = g
    return g

  def launch_nbody(self, max_steps, stream):
    """Replay the leapfrog graph (recaptured if the step tables moved)."""
    code = _lib.lib.fpm_graph_launch(self.nbody_graph(max_steps), stream)
    if code == _lib.FPM_ERR_STATE:
      _lib.lib.fpm_graph_destroy(self._graphs.pop(('nbody', max_steps)))
      code = _lib.lib.fpm_graph_launch(self.nbody_graph(max_steps), stream)
    _lib.check('fpm_graph_launch', code)

  def close(self):
    for g in getattr(self, '_graphs', {}).values():
      _lib.lib.fpm_graph_destroy(g)
    self._graphs = {}
    if getattr(self, 'handle', None) is not None and self.handle.value:
      _lib.lib.fpm_plan_destroy(self.handle)
      self.handle = None

  def __del__(self):
    try:
      self.close()
    except Exception:  # interpreter shutdown
      pass


_cache = {}


def get_plan(dims, r_split=0.0, flags=0):
  key = (torch.cuda.current_device(), tuple(tuple(d) for d in dims),
         float(r_split), int(flags))
  plan = _cache.get(key)
  if plan is None:
    plan = Plan(dims, r_split, flags)
    _cache[key] = plan
  return plan


def clear_plans():
  """Release every cached plan (their device buffers and cuFFT plans)."""
  torch.cuda.synchronize()
  for p in list(_cache.values()):
    p.close()
  _cache.clear()
