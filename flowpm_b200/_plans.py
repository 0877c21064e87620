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
    self.binning = (0, 1, _lib.FPM_BIN_CHUNKS)
    self.adjoint_binning = 0

  def set_binning(self, tile, sort_every=1, mode=_lib.FPM_BIN_CHUNKS):
    """Binned forward step (``fpm_plan_set_binning``): particles sorted by
    force-mesh cell, keys tile-major in tiles of ``tile``^3 cells (8 or 16;
    0: the lattice walk), re-sorted every ``sort_every`` steps; ``mode``
    FPM_BIN_CHUNKS (equal particle chunks), FPM_BIN_TILES (one block per
    tile, shared-memory paint) or FPM_BIN_WALK (the forward keeps the
    lattice walk; tiles and buffers for ``set_adjoint_binning`` only).
    Drops captured graphs."""
    _lib.call('fpm_plan_set_binning', self.handle, int(tile), int(sort_every),
              int(mode))
    self.binning = (int(tile), int(sort_every), int(mode)) if tile else (
        0, 1, _lib.FPM_BIN_CHUNKS)
    for g in self._graphs.values():
      _lib.lib.fpm_graph_destroy(g)
    self._graphs = {}

  def set_adjoint_binning(self, sort_every):
    """Reverse sweep of a potential-tape adjoint in the binned order
    (``fpm_plan_set_adjoint_binning``): re-sorted every ``sort_every``
    positions, 0 for the lattice walk.  Needs binning on.  Drops captured
    graphs."""
    _lib.call('fpm_plan_set_adjoint_binning', self.handle, int(sort_every))
    self.adjoint_binning = int(sort_every)
    for g in self._graphs.values():
      _lib.lib.fpm_graph_destroy(g)
    self._graphs = {}

  def autotune(self, disp, mom, reps=2, retune=False):
    """``fpm_plan_autotune`` on the plan's current step tables from the state
    (disp, mom) (each (total_particles, 3), left unchanged): the fastest of
    the lattice walk and the binned configurations is set on the plan.
    Returns ((tile, sort_every), {config: ms}); configurations the meshes do
    not support, or a cached choice, report no time."""
    choice = (ctypes.c_int32 * 3)()
    ms = (ctypes.c_float * _lib.FPM_TUNE_CONFIGS)()
    _lib.call('fpm_plan_autotune', self.handle, _lib.ptr(disp), _lib.ptr(mom),
              int(reps), int(bool(retune)), choice, ms, _lib.stream_ptr())
    self.binning = (choice[0], choice[1], choice[2])
    for g in self._graphs.values():
      _lib.lib.fpm_graph_destroy(g)
    self._graphs = {}
    names = ['walk', 'chunks16/4', 'chunks16/6', 'chunks16/10', 'chunks16/16',
             'chunks16/once', 'flow16', 'tiles16/4']
    return self.binning, {n: (float(t) if t >= 0 else None)
                          for n, t in zip(names, ms)}

  def apply_tuned(self):
    """Apply the autotuner's cached choice for this plan's key (device,
    flags, step tables' length, PGD, tape, shapes), if there is one;
    returns the (tile, sort_every) set, or None."""
    choice = (ctypes.c_int32 * 3)()
    code = _lib.lib.fpm_plan_autotune(self.handle, None, None, 1, 0, choice,
                                      None, _lib.stream_ptr())
    if code == _lib.FPM_ERR_STATE:
      return None
    _lib.check('fpm_plan_autotune', code)
    if (choice[0], choice[1], choice[2]) != self.binning:
      for g in self._graphs.values():
        _lib.lib.fpm_graph_destroy(g)
      self._graphs = {}
    self.binning = (choice[0], choice[1], choice[2])
    return self.binning

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

# Autotuning policy of the drop-in API (nbody, the batch runner, the stream):
# plans of at least min_particles particles time the lattice walk against
# the binned step configurations on their first run (fpm_plan_autotune) and
# keep the fastest; smaller plans, and every plan when disabled, apply a
# choice already cached for their key or keep the lattice walk.
TUNING = {'enabled': True, 'min_particles': 1 << 21, 'reps': 2}


def set_autotune(enabled=True, min_particles=1 << 21):
  """Switch the autotuning policy of nbody / BatchRunner / NBodyStream."""
  TUNING['enabled'] = bool(enabled)
  TUNING['min_particles'] = int(min_particles)


def tune(plan, disp, mom, key):
  """Apply the policy to ``plan`` (step tables set, ``disp``/``mom`` its
  initial state): once per plan and ``key`` (the step count, tape use)."""
  if getattr(plan, '_tuned_for', None) == key:
    return plan.binning
  plan._tuned_for = key
  if plan.apply_tuned() is not None:
    return plan.binning
  if TUNING['enabled'] and plan.total_particles >= TUNING['min_particles']:
    return plan.autotune(disp, mom, reps=TUNING['reps'])[0]
  return plan.binning


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
