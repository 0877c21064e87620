"""torch.autograd.Function wrappers around the library's adjoint kernels.

Gradients never come from recording the forward: each backward calls the
hand-written adjoint of the C library --
  cic_paint   -> fpm_cic_paint_adjoint   (gather with CIC weight derivatives)
  cic_readout -> fpm_cic_readout_adjoint (scatter + weight derivatives)
  lpt_init    -> fpm_lpt_adjoint         (transposed LPT transfer functions)
  nbody       -> fpm_nbody_adjoint       (reverse-time leapfrog adjoint that
                                          rebuilds the trajectory from the
                                          final state, with checkpoints)
"""
import numpy as np
import torch

from . import _lib
from . import tfbackground as bg
from ._plans import get_plan, tune


class CicPaint(torch.autograd.Function):

  @staticmethod
  def forward(ctx, mesh, part, weight):
    B, nx, ny, nz = mesh.shape
    out = mesh.detach().clone()
    w = None if weight is None else weight.detach()
    _lib.call('fpm_cic_paint', _lib.ptr(out), B, nx, ny, nz,
              _lib.ptr(part.detach()), part.shape[1], _lib.ptr(w),
              _lib.stream_ptr())
    ctx.save_for_backward(part, weight)
    ctx.dims = (B, nx, ny, nz)
    return out

  @staticmethod
  def backward(ctx, g):
    part, weight = ctx.saved_tensors
    B, nx, ny, nz = ctx.dims
    g = g.contiguous()
    lp = torch.empty_like(part) if ctx.needs_input_grad[1] else None
    lw = (torch.empty_like(weight) if weight is not None and
          ctx.needs_input_grad[2] else None)
    if lp is not None or lw is not None:
      _lib.call('fpm_cic_paint_adjoint', _lib.ptr(g), B, nx, ny, nz,
                _lib.ptr(part.detach()), part.shape[1],
                _lib.ptr(None if weight is None else weight.detach()),
                _lib.ptr(lp), _lib.ptr(lw), _lib.stream_ptr())
    return (g if ctx.needs_input_grad[0] else None), lp, lw


class CicPaint2D(torch.autograd.Function):

  @staticmethod
  def forward(ctx, mesh, part, weight, mask):
    B, nx, ny = mesh.shape
    out = mesh.detach().clone()
    w = None if weight is None else weight.detach()
    _lib.call('fpm_cic_paint_2d', _lib.ptr(out), B, nx, ny,
              _lib.ptr(part.detach()), part.shape[1], _lib.ptr(w),
              _lib.ptr(mask), _lib.stream_ptr())
    ctx.save_for_backward(part, weight, mask)
    ctx.dims = (B, nx, ny)
    return out

  @staticmethod
  def backward(ctx, g):
    part, weight, mask = ctx.saved_tensors
    B, nx, ny = ctx.dims
    g = g.contiguous()
    lp = torch.empty_like(part) if ctx.needs_input_grad[1] else None
    lw = (torch.empty_like(weight) if weight is not None and
          ctx.needs_input_grad[2] else None)
    if lp is not None or lw is not None:
      _lib.call('fpm_cic_paint_2d_adjoint', _lib.ptr(g), B, nx, ny,
                _lib.ptr(part.detach()), part.shape[1],
                _lib.ptr(None if weight is None else weight.detach()),
                _lib.ptr(mask), _lib.ptr(lp), _lib.ptr(lw), _lib.stream_ptr())
    return (g if ctx.needs_input_grad[0] else None), lp, lw, None


class DensityPlanes(torch.autograd.Function):
  """Planes of positions X (batch, npart, 3); ``args`` = the host
  parameters of fpm_density_planes after X."""

  @staticmethod
  def forward(ctx, X, args):
    out = torch.empty(args['shape'], dtype=torch.float32, device=X.device)
    _lib.call('fpm_density_planes', _lib.ptr(X.detach()), *args['c'],
              _lib.ptr(out), _lib.stream_ptr())
    ctx.save_for_backward(X)
    ctx.args = args
    return out

  @staticmethod
  def backward(ctx, g):
    (X,) = ctx.saved_tensors
    gX = torch.empty_like(X)
    _lib.call('fpm_density_planes_adjoint', _lib.ptr(X.detach()),
              *ctx.args['c'], _lib.ptr(g.contiguous()), _lib.ptr(gX),
              _lib.stream_ptr())
    return gX, None


class CicReadout(torch.autograd.Function):

  @staticmethod
  def forward(ctx, mesh, part):
    B, nx, ny, nz = mesh.shape
    out = torch.empty((B, part.shape[1]), dtype=torch.float32,
                      device=mesh.device)
    _lib.call('fpm_cic_readout', _lib.ptr(mesh.detach()), B, nx, ny, nz,
              _lib.ptr(part.detach()), part.shape[1], _lib.ptr(out),
              _lib.stream_ptr())
    ctx.save_for_backward(mesh, part)
    return out

  @staticmethod
  def backward(ctx, g):
    mesh, part = ctx.saved_tensors
    B, nx, ny, nz = mesh.shape
    g = g.contiguous()
    lm = torch.zeros_like(mesh) if ctx.needs_input_grad[0] else None
    lp = torch.empty_like(part) if ctx.needs_input_grad[1] else None
    if lm is not None or lp is not None:
      _lib.call('fpm_cic_readout_adjoint', _lib.ptr(mesh.detach()), B, nx, ny,
                nz, _lib.ptr(part.detach()), part.shape[1], _lib.ptr(g),
                _lib.ptr(lm), _lib.ptr(lp), _lib.stream_ptr())
    return lm, lp


class LptInit(torch.autograd.Function):

  @staticmethod
  def forward(ctx, linear, cosmo, a, order):
    B, nx, ny, nz = linear.shape
    plan = get_plan([(nx, ny, nz, 1)] * B, flags=_lib.FPM_PLAN_LPT)
    coef = np.tile(bg.lpt_coefficients(cosmo, a), B)
    state = torch.empty((3, B, nx * ny * nz, 3), dtype=torch.float32,
                        device=linear.device)
    st = _lib.stream_ptr()
    lin = linear.detach().contiguous()
    _lib.call('fpm_lpt_init', plan.handle, _lib.ptr(lin), _lib.dvec(coef),
              order, _lib.ptr(state[0]), _lib.ptr(state[1]),
              _lib.ptr(state[2]), st)
    _lib.call('fpm_lattice_shift', _lib.ptr(state[0]), _lib.ptr(state[0]), B,
              nx, ny, nz, 1, st)
    ctx.save_for_backward(lin)
    ctx.coef, ctx.order = coef, order
    return state

  @staticmethod
  def backward(ctx, g):
    (lin,) = ctx.saved_tensors
    B, nx, ny, nz = lin.shape
    plan = get_plan([(nx, ny, nz, 1)] * B, flags=_lib.FPM_PLAN_LPT)
    g = g.contiguous()
    out = torch.empty_like(lin)
    _lib.call('fpm_lpt_adjoint', plan.handle, _lib.ptr(lin),
              _lib.dvec(ctx.coef), ctx.order, _lib.ptr(g[0]), _lib.ptr(g[1]),
              _lib.ptr(g[2]), _lib.ptr(out), _lib.stream_ptr())
    return out, None, None, None


def _lattice_shift(x, nc, sign, out=None):
  B = x.shape[0]
  out = torch.empty_like(x) if out is None else out
  _lib.call('fpm_lattice_shift', _lib.ptr(x), _lib.ptr(out), B, nc[0], nc[1],
            nc[2], sign, _lib.stream_ptr())
  return out


class NBody(torch.autograd.Function):
  """nbody with the reverse-time adjoint as its backward."""

  @staticmethod
  def forward(ctx, state, cosmo, stages, nc, pm_nc_factor, checkpoint_every,
              store_potential=None, pgd_rows=None):
    B = state.shape[1]
    T = len(stages) - 1
    dims = [tuple(nc) + (int(pm_nc_factor),)] * B
    plan = get_plan(dims, flags=_lib.FPM_PLAN_ADJOINT)
    coefs = np.tile(bg.nbody_coefficients(cosmo, stages)[None], (B, 1, 1))
    ffac = [1.5 * cosmo.Omega_m] * B
    st = _lib.stream_ptr()
    _lib.call('fpm_nbody_set_steps', plan.handle, T, _lib.ivec([T] * B),
              _lib.dvec(coefs.ravel()), _lib.dvec(ffac), st)
    pgd = None if pgd_rows is None else np.tile(pgd_rows, (B, 1)).ravel()
    _set_pgd(plan, pgd, st)
    x = state.detach()
    d = _lattice_shift(x[0].contiguous(), nc, -1)
    p = x[1].clone().contiguous()
    f = torch.empty_like(p)
    ckpt = None
    k = int(checkpoint_every or 0)
    if k > 0:
      ckpt = torch.empty((T // k + 1, 2) + tuple(p.shape), dtype=torch.float32,
                         device=p.device)
    if pgd is not None and store_potential is False:
      raise ValueError('gradients through the PGD correction need '
                       'store_potential')
    tape = _potential_tape(dims, T, True if pgd is not None else
                           store_potential, p.device, pgd is not None)
    if tape is not None:
      _lib.call('fpm_nbody_set_tape', plan.handle, _lib.ptr(tape),
                tape.numel())
    try:
      if pgd is None:
        tune(plan, d, p, (T, tape is not None))
      _lib.call('fpm_nbody_run', plan.handle, _lib.ptr(d), _lib.ptr(p),
                _lib.ptr(f), None, 0, _lib.ptr(ckpt), k, st)
    finally:
      if tape is not None:  # the plan is shared: detach the buffer
        _lib.call('fpm_nbody_set_tape', plan.handle, None, 0)
    out = torch.empty_like(x)
    _lattice_shift(d, nc, 1, out=out[0])
    out[1].copy_(p)
    out[2].copy_(f)
    ctx.save_for_backward(d, p, f)
    ctx.ckpt = ckpt
    ctx.tape = tape
    ctx.args = (dims, T, coefs, ffac, k, list(nc), pgd)
    return out

  @staticmethod
  def backward(ctx, g):
    d, p, f = ctx.saved_tensors
    dims, T, coefs, ffac, k, nc, pgd = ctx.args
    B = len(dims)
    plan = get_plan(dims, flags=_lib.FPM_PLAN_ADJOINT)
    st = _lib.stream_ptr()
    _lib.call('fpm_nbody_set_steps', plan.handle, T, _lib.ivec([T] * B),
              _lib.dvec(coefs.ravel()), _lib.dvec(ffac), st)
    _set_pgd(plan, pgd, st)
    g = g.contiguous()
    lx = g[0].clone()
    lp = g[1].clone()
    lf = g[2].contiguous()
    dd, pp = d.clone(), p.clone()
    tape = ctx.tape
    if tape is not None:
      _lib.call('fpm_nbody_set_tape', plan.handle, _lib.ptr(tape),
                tape.numel())
    try:
      _lib.call('fpm_nbody_adjoint', plan.handle, _lib.ptr(dd), _lib.ptr(pp),
                _lib.ptr(f), _lib.ptr(lx), _lib.ptr(lp), _lib.ptr(lf),
                _lib.ptr(ctx.ckpt), k, st)
    finally:
      if tape is not None:
        _lib.call('fpm_nbody_set_tape', plan.handle, None, 0)
    ctx.tape = None
    grad = torch.stack((lx, lp, torch.zeros_like(lx)))
    return grad, None, None, None, None, None, None, None


def _set_pgd(plan, rows, st):
  """Switch PGD on (rows: nsims x steps x 3 doubles) or off on the shared
  plan for this call."""
  _lib.call('fpm_nbody_set_pgd', plan.handle, 0 if rows is None else 1,
            None if rows is None else _lib.dvec(rows), st)


def _potential_tape(dims, T, store, device, pgd=False):
  """The potential tape of a differentiable nbody call: (T + 1) x the
  plan's force-mesh cells (with PGD, also T PGD potentials and T particle
  displacements; the layout of fpm_nbody_set_tape), or None.  store: True,
  False, or None for automatic (when it takes under a quarter of the free
  device memory)."""
  if store is False:
    return None
  cells = sum((b * nx) * (b * ny) * (b * nz) for nx, ny, nz, b in dims)
  parts = sum(nx * ny * nz for nx, ny, nz, b in dims)
  n = (T + 1) * cells
  if pgd:
    n += T * (cells + 3 * parts)
  if store is None:
    if cells % 4:  # the tape's positions must stay 16-byte aligned
      return None
    free, _ = torch.cuda.mem_get_info(device)
    if 4 * n > free // 4:
      return None
  return torch.empty(n, dtype=torch.float32, device=device)


def needs_grad(*tensors):
  return torch.is_grad_enabled() and any(
      isinstance(t, torch.Tensor) and t.requires_grad for t in tensors)
