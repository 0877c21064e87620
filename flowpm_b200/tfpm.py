"""Particle-mesh solver mirroring ``flowpm/tfpm.py``: Gaussian initial
conditions, 1LPT/2LPT initialisation and the FastPM kick-drift-kick
leapfrog, on CUDA tensors through the C library.

State layout is the reference's: ``(3, batch, npart, 3)`` = (X, P, F) with
X the absolute position in mesh units.  Inside ``nbody`` the library keeps
X as an FP32 displacement from the Lagrangian lattice, so position
resolution does not degrade with the mesh size; X is formed only at the
boundary.  Background prefactors are FP64 (``tfbackground``).
"""
import numpy as np
import torch

from . import _autograd
from . import _lib
from . import tfbackground as bg
from ._plans import get_plan, tune
from .kernels import fftk
from .utils import as_cuda, _seed

__all__ = ['linear_field', 'lpt1', 'lpt2_source', 'lpt_init', 'nbody',
           'force', 'kick', 'drift', 'pgd',
           'linear_amplitude']


def _nc3(nc):
  return [nc] * 3 if isinstance(nc, int) else [int(n) for n in nc]


def _box3(boxsize):
  if isinstance(boxsize, (int, float)):
    return [float(boxsize)] * 3
  return [float(b) for b in boxsize]


def _check_kvec(kvec, nc):
  if kvec is None:
    return
  ref = fftk(nc, symmetric=False)
  if len(kvec) != 3 or any(
      np.shape(k) != np.shape(r) or not np.allclose(k, r)
      for k, r in zip(kvec, ref)):
    raise NotImplementedError(
        'only the default k grid fftk(nc, symmetric=False) is supported')


def _axis_kvec(kvec, nc):
  """A caller's k grid as three per-axis vectors: each entry of ``kvec``
  must broadcast along one axis only (the shapes fftk returns, (nx, 1, 1),
  (1, ny, 1), (1, 1, nz)).  The field is built on the half spectrum, so
  the grid must give every mode and its mirror -k the same |k| (true of
  fftk's grid and of any rescaling of it)."""
  if len(kvec) != 3:
    raise ValueError('kvec must hold three arrays, one per axis')
  out = []
  for d, k in enumerate(kvec):
    k = np.asarray(k, dtype=np.float64)
    shape = [1, 1, 1]
    shape[d] = nc[d]
    if k.ndim != 3 or list(k.shape) != shape:
      raise NotImplementedError(
          'kvec[%d] must have shape %s (per-axis k vectors)' % (d, shape))
    k = k.ravel()
    if not np.array_equal(k * k, (k * k)[(-np.arange(nc[d])) % nc[d]]):
      raise NotImplementedError(
          'kvec[%d] must satisfy |k[i]| = |k[-i]| (half-spectrum field)' % d)
    out.append(k)
  return out


def linear_amplitude(nc, boxsize, pk, kvec=None):
  """Half-spectrum amplitude sqrt(P(|k|) / V), (nx, ny, nz//2 + 1) float32,
  with |k| = sqrt(sum_d (k_d / L_d * n_d)^2) as in flowpm/tfpm.py:55-56,
  k_d from ``kvec`` (per-axis vectors, default fftk(nc, symmetric=False)).

  For the default grid of a cubic mesh in a cubic box P is evaluated once
  per distinct i^2 + j^2 + l^2; otherwise on every mode."""
  nc, boxsize = _nc3(nc), _box3(boxsize)
  custom = kvec is not None
  kvec = _axis_kvec(kvec, nc) if custom else fftk(nc, symmetric=False)
  nzh = nc[2] // 2 + 1
  vol = boxsize[0] * boxsize[1] * boxsize[2]
  ax = [(np.ravel(kk) / boxsize[i] * nc[i])**2 for i, kk in enumerate(kvec)]
  ax[2] = ax[2][:nzh]
  if (not custom and nc[0] == nc[1] == nc[2] and
      boxsize[0] == boxsize[1] == boxsize[2]):
    f = np.rint(np.fft.fftfreq(nc[0]) * nc[0]).astype(np.int64)
    sq = f * f
    key = (sq[:, None, None] + sq[None, :, None] +
           sq[None, None, :nzh]).astype(np.int32)
    flat = key.ravel()
    first = np.full(int(flat.max()) + 1, -1, dtype=np.int64)
    first[flat[::-1]] = np.arange(flat.size - 1, -1, -1)
    present = first >= 0
    ii, jj, ll = np.unravel_index(first[present], key.shape)
    # |k| of one mode realising each i^2 + j^2 + l^2 (the reference's
    # per-mode sums differ from it at most in the last bit)
    kmesh = (ax[0][ii] + ax[1][jj] + ax[2][ll])**0.5
    table = np.zeros(first.size)
    table[present] = (np.asarray(pk(kmesh), dtype=np.float64) / vol)**0.5
    return table[key].astype(np.float32)
  kk = ax[0][:, None, None] + ax[1][None, :, None] + ax[2][None, None, :]
  pkm = np.asarray(pk(kk**0.5), dtype=np.float64)
  return ((pkm / vol)**0.5).astype(np.float32)


def linear_field(nc, boxsize, pk, kvec=None, batch_size=1, seed=None,
                 dtype=torch.float32, name='LinearField', white=None):
  """Gaussian linear field with power spectrum ``pk``
  (flowpm/tfpm.py:15-63): white noise N(0, sqrt(N^3)) -> r2c -> times
  sqrt(P(|k|)/V) -> c2r.  ``pk`` is called on a NumPy array of |k| in h/Mpc.
  ``white`` (batch, nx, ny, nz) replaces the generated noise when given.
  Returns (batch, nx, ny, nz) float32 on the current CUDA device."""
  nc = _nc3(nc)
  if dtype not in (torch.float32, np.float32):
    raise NotImplementedError('linear_field computes in float32')
  amp = as_cuda(linear_amplitude(nc, boxsize, pk, kvec))
  amp = amp.reshape(1, -1).expand(batch_size, -1).contiguous()
  plan = get_plan([tuple(nc) + (1,)] * batch_size, flags=_lib.FPM_PLAN_LPT)
  out = torch.empty([batch_size] + nc, dtype=torch.float32, device='cuda')
  if white is not None:
    white = as_cuda(white).reshape([batch_size] + nc)
    _lib.call('fpm_linear_field', plan.handle, _lib.ptr(amp), 0, 0,
              _lib.ptr(white), _lib.ptr(out), _lib.stream_ptr())
  else:
    _lib.call('fpm_linear_field', plan.handle, _lib.ptr(amp), _seed(seed), 1,
              None, _lib.ptr(out), _lib.stream_ptr())
  return out


def _spectrum(dlin_k):
  """Full complex spectra (batch, nx, ny, nz) as contiguous complex64 CUDA."""
  if not torch.is_tensor(dlin_k):
    dlin_k = torch.as_tensor(np.asarray(dlin_k))
  if not dlin_k.is_complex():
    raise ValueError('dlin_k must be a complex spectrum (batch, nx, ny, nz)')
  if dlin_k.dim() != 4:
    raise ValueError('dlin_k must be (batch, nx, ny, nz)')
  return dlin_k.to(device='cuda', dtype=torch.complex64).contiguous()


def lpt1(dlin_k, pos, kvec=None, name='LTP1'):
  """First-order LPT displacement read out at ``pos`` (flowpm/tfpm.py:66-95):
  psi_d = c2r3d(dlin_k * laplace_kernel * gradient_kernel_d), then
  cic_readout(psi_d, pos).  ``dlin_k`` is the full spectrum r2c3d(linear)
  (batch, nx, ny, nz) complex64; ``pos`` (batch, npart, 3) in mesh units.
  Returns (batch, npart, 3) float32."""
  dlin_k = _spectrum(dlin_k)
  B, nx, ny, nz = dlin_k.shape
  _check_kvec(kvec, [nx, ny, nz])
  pos = as_cuda(pos)
  if pos.dim() != 3 or pos.shape[0] != B or pos.shape[2] != 3:
    raise ValueError('pos must be (batch, npart, 3)')
  plan = get_plan([(nx, ny, nz, 1)] * B, flags=_lib.FPM_PLAN_LPT)
  out = torch.empty_like(pos)
  _lib.call('fpm_lpt1', plan.handle, _lib.ptr(dlin_k), _lib.ptr(pos),
            pos.shape[1], _lib.ptr(out), _lib.stream_ptr())
  return out


def lpt2_source(dlin_k, kvec=None, name='LPT2Source'):
  """Second-order LPT source term (flowpm/tfpm.py:98-145):
  3/7 sum_{i<j} (phi_ii phi_jj - phi_ij^2) with
  phi_ij = c2r3d(dlin_k * laplace_kernel * g_i g_j), returned as its full
  spectrum r2c3d(source), (batch, nx, ny, nz) complex64."""
  dlin_k = _spectrum(dlin_k)
  B, nx, ny, nz = dlin_k.shape
  _check_kvec(kvec, [nx, ny, nz])
  plan = get_plan([(nx, ny, nz, 1)] * B, flags=_lib.FPM_PLAN_LPT)
  out = torch.empty_like(dlin_k)
  _lib.call('fpm_lpt2_source', plan.handle, _lib.ptr(dlin_k), _lib.ptr(out),
            _lib.stream_ptr())
  return out


def lpt_init(cosmo, linear, a, order=2, kvec=None, name='LPTInit'):
  """1LPT / 2LPT initial state (3, batch, npart, 3) from a real linear field
  (batch, nx, ny, nz) at scale factor ``a`` (flowpm/tfpm.py:148-180).
  Differentiable in ``linear`` (fpm_lpt_adjoint)."""
  assert order in (1, 2)
  linear = as_cuda(linear)
  if linear.dim() != 4:
    raise ValueError('linear must be (batch, nx, ny, nz)')
  B, nx, ny, nz = linear.shape
  _check_kvec(kvec, [nx, ny, nz])
  if _autograd.needs_grad(linear):
    return _autograd.LptInit.apply(linear, cosmo, a, order)
  np_ = nx * ny * nz
  plan = get_plan([(nx, ny, nz, 1)] * B, flags=_lib.FPM_PLAN_LPT)
  coef = np.tile(bg.lpt_coefficients(cosmo, a), B)
  state = torch.empty((3, B, np_, 3), dtype=torch.float32, device=linear.device)
  st = _lib.stream_ptr()
  _lib.call('fpm_lpt_init', plan.handle, _lib.ptr(linear), _lib.dvec(coef),
            order, _lib.ptr(state[0]), _lib.ptr(state[1]), _lib.ptr(state[2]),
            st)
  _lib.call('fpm_lattice_shift', _lib.ptr(state[0]), _lib.ptr(state[0]), B,
            nx, ny, nz, 1, st)
  return state


def _state(state, nc):
  state = as_cuda(state)
  if state.dim() != 4 or state.shape[0] != 3 or state.shape[3] != 3:
    raise ValueError('state must be (3, batch, npart, 3)')
  if state.shape[2] != nc[0] * nc[1] * nc[2]:
    raise ValueError('npart %d does not match nc %s' % (state.shape[2], nc))
  return state


def _to_disp(X, nc):
  B = X.shape[0]
  d = torch.empty_like(X)
  _lib.call('fpm_lattice_shift', _lib.ptr(X), _lib.ptr(d), B, nc[0], nc[1],
            nc[2], -1, _lib.stream_ptr())
  return d


def _to_pos(d, nc, out):
  B = d.shape[0]
  _lib.call('fpm_lattice_shift', _lib.ptr(d), _lib.ptr(out), B, nc[0], nc[1],
            nc[2], 1, _lib.stream_ptr())
  return out


def force(cosmo, state, nc, pm_nc_factor=1, name='Force', **kwargs):
  """State with F replaced by the PM force at X (flowpm/tfpm.py:317-366)."""
  nc = _nc3(nc)
  state = _state(state, nc)
  B = state.shape[1]
  plan = get_plan([tuple(nc) + (int(pm_nc_factor),)] * B)
  d = _to_disp(state[0], nc)
  f = torch.empty_like(d)
  _lib.call('fpm_force', plan.handle, _lib.ptr(d),
            _lib.dvec([1.5 * cosmo.Omega_m] * B), _lib.ptr(f),
            _lib.stream_ptr())
  return torch.stack((state[0], state[1], f))


def _pgd_rows(pgdparams, rows):
  """(alpha, kl, ks) rows as a float64 array of shape (rows, 3)."""
  p = np.asarray(pgdparams, dtype=np.float64)
  if p.shape == (3,) and rows == 1:
    p = p.reshape(1, 3)
  if p.shape != (rows, 3):
    raise ValueError('pgdparams must hold %d rows of (alpha, kl, ks), got '
                     'shape %s' % (rows, p.shape))
  return p


def pgd(state, pgdparams, nc, pm_nc_factor=1, name='PGD', **kwargs):
  """State with X moved by the PGD correction (flowpm/tfpm.py:369-422):
  paint at X * pm_nc_factor, potential with the PGD kernel
  exp(-kl^2/k^2) exp(-k^4/ks^4) (kernels.py:105-134), 4-point gradient,
  readout, X += alpha * update / pm_nc_factor.  ``pgdparams`` =
  (alpha, kl, ks), kl and ks in the force mesh's k units."""
  nc = _nc3(nc)
  state = _state(state, nc)
  B = state.shape[1]
  par = _pgd_rows(pgdparams, 1)
  plan = get_plan([tuple(nc) + (int(pm_nc_factor),)] * B)
  d = _to_disp(state[0], nc)
  _lib.call('fpm_pgd', plan.handle, _lib.ptr(d),
            _lib.dvec(np.tile(par, (B, 1)).ravel()), _lib.stream_ptr())
  out = state.clone()
  _to_pos(d, nc, out[0])
  return out


def kick(cosmo, state, ai, ac, af, name='Kick', **kwargs):
  """P += fac F with the FP64 kick prefactor (flowpm/tfpm.py:273-292)."""
  state = as_cuda(state).clone()
  fac = bg.kick_factor(cosmo, ai, ac, af)
  _lib.call('fpm_saxpy', _lib.ptr(state[1]), _lib.ptr(state[2]), fac,
            state[1].numel(), _lib.stream_ptr())
  return state


def drift(cosmo, state, ai, ac, af, name='Drift', **kwargs):
  """X += fac P with the FP64 drift prefactor (flowpm/tfpm.py:295-314)."""
  state = as_cuda(state).clone()
  fac = bg.drift_factor(cosmo, ai, ac, af)
  _lib.call('fpm_saxpy', _lib.ptr(state[0]), _lib.ptr(state[1]), fac,
            state[0].numel(), _lib.stream_ptr())
  return state


def nbody(cosmo, state, stages, nc, pm_nc_factor=1,
          return_intermediate_states=False, pgdparams=None, name='NBody',
          check_finite=True, checkpoint_every=None, store_potential=None):
  """Integrate ``state`` across ``stages`` with the FastPM KDK leapfrog
  (flowpm/tfpm.py:425-503): one force at stages[0], then per step
  kick / drift / force / kick.  Returns the final state (3, B, Np, 3) or,
  with ``return_intermediate_states``, the list of (a_i, state_i).

  Differentiable in ``state``: the backward is the reverse-time adjoint
  (fpm_nbody_adjoint), which rebuilds the trajectory from the final state;
  ``checkpoint_every = k`` stores (d, p) every k steps in the forward and
  resets the rebuilt trajectory there, bounding its FP32 drift.
  ``store_potential`` keeps the potential of every force solve of the
  forward ((steps + 1) x B x (pm_nc_factor nc)^3 floats, fpm_nbody_set_tape),
  so the backward takes its force meshes from it instead of painting and
  solving again; None (default) stores it when that takes less than a
  quarter of the free device memory.

  With ``pgdparams`` (one row (alpha, kl, ks) per step) the PGD
  correction moves the particles after every drift (flowpm/tfpm.py:487-488,
  see ``pgd``); its gradient needs the stored potentials (the tape also
  keeps each step's PGD potential and pre-move displacement), so
  ``store_potential=False`` is refused there.

  With ``check_finite`` the device status word is read at the end and a
  non-finite particle state raises ``FlowPMError``."""
  nc = _nc3(nc)
  stages = [float(s) for s in np.asarray(stages).ravel()]
  state = _state(state, nc)
  if len(stages) == 0:
    return state
  B = state.shape[1]
  T = len(stages) - 1
  par = None
  if pgdparams is not None and T > 0:
    par = _pgd_rows(pgdparams, T)
  if _autograd.needs_grad(state):
    if return_intermediate_states:
      raise NotImplementedError(
          'gradients through intermediate states are not supported')
    out = _autograd.NBody.apply(state, cosmo, stages, nc, pm_nc_factor,
                                checkpoint_every, store_potential, par)
    if check_finite:
      plan = get_plan([tuple(nc) + (int(pm_nc_factor),)] * B,
                      flags=_lib.FPM_PLAN_ADJOINT)
      if plan.status():
        raise _lib.FlowPMError('nbody', _lib.FPM_ERR_NONFINITE)
    return out
  plan = get_plan([tuple(nc) + (int(pm_nc_factor),)] * B)
  coefs = np.tile(bg.nbody_coefficients(cosmo, stages)[None], (B, 1, 1))
  st = _lib.stream_ptr()
  _lib.call('fpm_nbody_set_steps', plan.handle, T, _lib.ivec([T] * B),
            _lib.dvec(coefs.ravel()), _lib.dvec([1.5 * cosmo.Omega_m] * B), st)
  # the plan is shared: PGD is switched on or off for this call
  _lib.call('fpm_nbody_set_pgd', plan.handle, 0 if par is None else 1,
            None if par is None else _lib.dvec(np.tile(par, (B, 1)).ravel()),
            st)
  d, p, f = plan.work()
  _lib.call('fpm_lattice_shift', _lib.ptr(state[0]), _lib.ptr(d), B, nc[0],
            nc[1], nc[2], -1, st)
  p.copy_(state[1].reshape(-1, 3))
  if par is None:
    tune(plan, d, p, (T, False))
  inter = None
  if return_intermediate_states and T > 0:
    inter = torch.empty((T, 3) + tuple(state.shape[1:]), dtype=torch.float32,
                        device=state.device)
    _lib.call('fpm_nbody_run', plan.handle, _lib.ptr(d), _lib.ptr(p),
              _lib.ptr(f), _lib.ptr(inter), _lib.FPM_NBODY_INTERMEDIATE, None,
              0, st)
  else:
    plan.launch_nbody(T, st)
  out = torch.empty_like(state)
  _to_pos(d.reshape(state[0].shape), nc, out[0])
  out[1].copy_(p.reshape(state[1].shape))
  out[2].copy_(f.reshape(state[2].shape))
  if check_finite:
    status = plan.status(st)
    if status:
      raise _lib.FlowPMError('nbody', _lib.FPM_ERR_NONFINITE)
  if return_intermediate_states:
    return [(stages[i + 1], inter[i]) for i in range(T)]
  return out
