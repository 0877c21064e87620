"""Restatement of the reference particle-mesh path in torch on the CPU:
``flowpm/kernels.py``, ``flowpm/utils.py``, ``flowpm/tfpm.py`` and
``flowpm/pk.py``.  Test infrastructure only (see package docstring).

Arrays follow the reference layout: meshes ``(B, nx, ny, nz)``, particle
positions ``(B, Np, 3)`` in mesh units, state ``(3, B, Np, 3)`` = (X, P, F).
The float type follows the inputs (float32 reproduces the reference; float64
is the same method in double precision), and every op is differentiable with
torch autograd, which stands in for TensorFlow's tape gradient.

The background (growth factors, kick/drift prefactors) comes from an
``oracle.background.Background`` passed as ``bg``; its float type is chosen
independently of the particle state.
"""
import numpy as np
import torch

# CIC neighbour order, flowpm/utils.py:66-67 and :191-192.
CONNECTION = ((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0),
              (1, 0, 1), (0, 1, 1), (1, 1, 1))


def _cdtype(rdtype):
  return torch.complex128 if rdtype == torch.float64 else torch.complex64


# --------------------------------------------------------------------------
# flowpm/kernels.py (NumPy, float64, exactly as the reference)
# --------------------------------------------------------------------------
def fftk(shape, symmetric=True, dtype=np.float64):
  """flowpm/kernels.py:10-25: per-axis 2*pi*fftfreq vectors, broadcast
  shaped; the last axis is cut to n//2+1 when ``symmetric``."""
  k = []
  nd = len(shape)
  for d in range(nd):
    kd = np.fft.fftfreq(shape[d]) * 2 * np.pi
    if symmetric and d == nd - 1:
      kd = kd[:shape[d] // 2 + 1]
    kshape = [1] * nd
    kshape[d] = len(kd)
    k.append(kd.reshape(kshape).astype(dtype))
  return k


def laplace_kernel(kvec):
  """flowpm/kernels.py:28-48: 1/k^2 with the value 1 at k = 0 (the mask is
  applied after kk[k==0] was set to 1, so it never zeroes anything)."""
  kk = sum(ki**2 for ki in kvec)
  kk = np.array(kk, copy=True)
  kk[kk == 0] = 1
  return 1. / kk


def gradient_kernel(kvec, direction, order=1):
  """flowpm/kernels.py:51-78: order 1 is the 4-point finite difference
  i*(8 sin w - sin 2w)/6; order 0 is i*k with the Nyquist entry zeroed."""
  if order == 0:
    w = 1j * kvec[direction]
    flat = np.squeeze(w).copy()
    flat[len(flat) // 2] = 0
    return flat.reshape(kvec[direction].shape)
  w = kvec[direction]
  return 1j * (1 / 6.0 * (8 * np.sin(w) - np.sin(2 * w)))


def longrange_kernel(kvec, r_split):
  """flowpm/kernels.py:81-102: exp(-k^2 r_s^2), or the scalar 1 for r_s=0."""
  if r_split != 0:
    kk = sum(ki**2 for ki in kvec)
    return np.exp(-kk * r_split**2)
  return 1.


def PGD_kernel(kvec, kl, ks):
  """flowpm/kernels.py:105-134 (evaluated in float32, because the reference
  combines the float64 k^2 with float32 tensors kl, ks)."""
  kk = sum(ki**2 for ki in kvec)
  kk = np.array(kk, copy=True)
  kk[kk == 0] = 1
  kk = kk.astype(np.float32)
  kl2 = np.float32(kl)**2
  ks4 = np.float32(ks)**4
  return np.exp(-kl2 / kk) * np.exp(-kk**2 / ks4)


def cic_compensation(kvec):
  """flowpm/kernels.py:137-152: prod_d sinc(k_d / 2 pi)^-2."""
  kw = [np.sinc(kvec[i] / (2 * np.pi)) for i in range(3)]
  return (kw[0] * kw[1] * kw[2])**(-2)


def _cast_kernel(w, cdtype):
  return torch.as_tensor(np.asarray(w)).to(cdtype)


# --------------------------------------------------------------------------
# flowpm/utils.py
# --------------------------------------------------------------------------
def _neighbours(part, nc):
  """floor, neighbour coordinates, CIC weights and flat mesh indices of the
  8 neighbours (flowpm/utils.py:63-81 / :190-205)."""
  floor = torch.floor(part)
  out = []
  for c in CONNECTION:
    nb = floor + torch.tensor(c, dtype=part.dtype)
    kern = 1. - torch.abs(part - nb)
    kern = kern[..., 0] * kern[..., 1] * kern[..., 2]
    ic = nb.to(torch.int64)
    ix = torch.remainder(ic[..., 0], nc[0])
    iy = torch.remainder(ic[..., 1], nc[1])
    iz = torch.remainder(ic[..., 2], nc[2])
    out.append((kern, (ix * nc[1] + iy) * nc[2] + iz))
  return out


def cic_paint(mesh, part, weight=None):
  """flowpm/utils.py:32-91: 8-neighbour CIC deposit, duplicates
  accumulated (tf.scatter_nd), result added to ``mesh``."""
  B = mesh.shape[0]
  nc = list(mesh.shape[1:])
  ncell = nc[0] * nc[1] * nc[2]
  part = part.reshape(B, -1, 3)
  update = torch.zeros(B * ncell, dtype=mesh.dtype)
  boff = (torch.arange(B) * ncell).reshape(B, 1)
  for kern, flat in _neighbours(part, nc):
    if weight is not None:
      kern = weight.reshape(B, -1) * kern
    update = update.index_add(0, (flat + boff).reshape(-1), kern.reshape(-1))
  return mesh + update.reshape(mesh.shape)


def cic_readout(mesh, part):
  """flowpm/utils.py:163-210: sum over the 8 neighbours of
  mesh[neighbour] * weight."""
  B = mesh.shape[0]
  nc = list(mesh.shape[1:])
  part = part.reshape(B, -1, 3)
  flatmesh = mesh.reshape(B, -1)
  vals = []
  for kern, flat in _neighbours(part, nc):
    vals.append(torch.gather(flatmesh, 1, flat) * kern)
  return torch.stack(vals, dim=-1).sum(dim=-1)


def r2c3d(rfield, norm=None):
  """flowpm/utils.py:213-241: full complex FFT times 1/norm."""
  if norm is None:
    norm = int(np.prod(rfield.shape[1:]))
  cd = _cdtype(rfield.dtype)
  return torch.fft.fftn(rfield.to(cd), dim=(-3, -2, -1)) * (1 / norm)


def c2r3d(cfield, norm=None):
  """flowpm/utils.py:244-272: real part of the inverse FFT times norm."""
  if norm is None:
    norm = int(np.prod(cfield.shape[1:]))
  return torch.fft.ifftn(cfield, dim=(-3, -2, -1)).real * norm


# --------------------------------------------------------------------------
# flowpm/tfpm.py
# --------------------------------------------------------------------------
def _nc3(nc):
  return [nc] * 3 if isinstance(nc, int) else [int(n) for n in nc]


def linear_field_from_white(white, boxsize, pk):
  """flowpm/tfpm.py:15-63 given the real white noise that flowpm/utils.py
  :346-350 would draw (N(0, sqrt(N^3)) per cell)."""
  nc = list(white.shape[1:])
  if isinstance(boxsize, (int, float)):
    boxsize = [boxsize] * 3
  kvec = fftk(nc, symmetric=False)
  kmesh = sum((kk / boxsize[i] * nc[i])**2 for i, kk in enumerate(kvec))**0.5
  pkmesh = np.asarray(pk(kmesh))
  norm = nc[0] * nc[1] * nc[2]
  whitec = r2c3d(white, norm=norm)
  amp = (pkmesh / (boxsize[0] * boxsize[1] * boxsize[2]))**0.5
  lineark = whitec * _cast_kernel(amp, whitec.dtype)
  return c2r3d(lineark, norm=norm)


def lpt1(dlin_k, pos):
  """flowpm/tfpm.py:66-95: Psi_d = readout(c2r(delta_k * lap * i D_d))."""
  nc = list(dlin_k.shape[1:])
  kvec = fftk(nc, symmetric=False)
  cd = dlin_k.dtype
  lap = _cast_kernel(laplace_kernel(kvec), cd)
  disp = []
  for d in range(3):
    kweight = _cast_kernel(gradient_kernel(kvec, d), cd) * lap
    dispr = c2r3d(dlin_k * kweight, norm=nc[0] * nc[1] * nc[2])
    disp.append(cic_readout(dispr, pos))
  return torch.stack(disp, dim=2)


def lpt2_source(dlin_k):
  """flowpm/tfpm.py:98-145: 3/7 * sum (phi_ii phi_jj - phi_ij^2) -> r2c."""
  nc = list(dlin_k.shape[1:])
  norm = nc[0] * nc[1] * nc[2]
  kvec = fftk(nc, symmetric=False)
  cd = dlin_k.dtype
  rd = torch.float64 if cd == torch.complex128 else torch.float32
  lap = _cast_kernel(laplace_kernel(kvec), cd)
  D1, D2 = [1, 2, 0], [2, 0, 1]
  phi_ii = []
  for d in range(3):
    g = _cast_kernel(gradient_kernel(kvec, d), cd)
    phi_ii.append(c2r3d(dlin_k * (lap * g * g), norm=norm))
  source = torch.zeros(dlin_k.shape, dtype=rd)
  for d in range(3):
    source = source + phi_ii[D1[d]] * phi_ii[D2[d]]
  for d in range(3):
    gi = _cast_kernel(gradient_kernel(kvec, D1[d]), cd)
    gj = _cast_kernel(gradient_kernel(kvec, D2[d]), cd)
    phi = c2r3d(dlin_k * (lap * gi * gj), norm=norm)
    source = source - phi * phi
  source = source * (3.0 / 7.)
  return r2c3d(source, norm=norm)


def lattice(nc, B, dtype=torch.float32):
  """Lagrangian lattice Q (flowpm/tfpm.py:162-163), shape (B, Np, 3)."""
  q = np.indices(nc).reshape(3, -1).T.astype(np.float32)
  return torch.as_tensor(np.repeat(q[None], B, axis=0)).to(dtype)


def lpt_init(bg, linear, a, order=2):
  """flowpm/tfpm.py:148-180."""
  assert order in (1, 2)
  B = linear.shape[0]
  nc = list(linear.shape[1:])
  rd = linear.dtype
  t = bg.t
  Q = lattice(nc, B, rd)
  lineark = r2c3d(linear, norm=nc[0] * nc[1] * nc[2])

  def s(x):
    return torch.as_tensor(np.asarray(x, dtype=t)).to(rd)

  a2 = t(float(a)**2)
  DX = s(bg.D1(a)) * lpt1(lineark, Q)
  P = s(a2 * bg.f1(a) * bg.E(a)) * DX
  F = s(a2 * bg.E(a) * bg.gf(a) / bg.D1(a)) * DX
  if order == 2:
    DX2 = s(bg.D2(a)) * lpt1(lpt2_source(lineark), Q)
    P2 = s(a2 * bg.f2(a) * bg.E(a)) * DX2
    F2 = s(a2 * bg.E(a) * bg.gf2(a) / bg.D2(a)) * DX2
    DX = DX + DX2
    P = P + P2
    F = F + F2
  X = DX + Q
  return torch.stack((X, P, F), dim=0)


def apply_longrange(x, delta_k, split=0, factor=1):
  """flowpm/tfpm.py:183-219."""
  nc = list(delta_k.shape[1:])
  kvec = fftk(nc, symmetric=False)
  cd = delta_k.dtype
  norm = nc[0] * nc[1] * nc[2]
  lap = _cast_kernel(laplace_kernel(kvec), cd)
  kweight = lap * _cast_kernel(longrange_kernel(kvec, split), cd)
  pot_k = delta_k * kweight
  f = []
  for d in range(3):
    forced = c2r3d(pot_k * _cast_kernel(gradient_kernel(kvec, d), cd),
                   norm=norm)
    f.append(cic_readout(forced, x))
  return torch.stack(f, dim=2) * factor


def apply_pgd(x, delta_k, alpha, kl, ks):
  """flowpm/tfpm.py:222-270."""
  nc = list(delta_k.shape[1:])
  kvec = fftk(nc, symmetric=False)
  cd = delta_k.dtype
  norm = nc[0] * nc[1] * nc[2]
  lap = _cast_kernel(laplace_kernel(kvec), cd)
  pgdr = _cast_kernel(PGD_kernel(kvec, kl, ks), cd)
  pot_k = delta_k * (lap * pgdr)
  f = []
  for d in range(3):
    forced = c2r3d(pot_k * _cast_kernel(gradient_kernel(kvec, d), cd),
                   norm=norm)
    f.append(cic_readout(forced, x))
  return torch.stack(f, dim=2) * alpha


def kick(bg, state, ai, ac, af):
  """flowpm/tfpm.py:273-292: P += fac * F."""
  fac = torch.as_tensor(np.asarray(bg.kick_factor(ai, ac, af))).to(
      state.dtype)
  return torch.stack((state[0], state[1] + fac * state[2], state[2]))


def drift(bg, state, ai, ac, af):
  """flowpm/tfpm.py:295-314: X += fac * P."""
  fac = torch.as_tensor(np.asarray(bg.drift_factor(ai, ac, af))).to(
      state.dtype)
  return torch.stack((state[0] + fac * state[1], state[1], state[2]))


def _paint_density(state, nc, pm_nc_factor):
  B = state.shape[1]
  ncf = [n * pm_nc_factor for n in nc]
  rho = torch.zeros([B] + ncf, dtype=state.dtype)
  wts = torch.ones((B, nc[0] * nc[1] * nc[2]), dtype=state.dtype)
  nbar = nc[0] * nc[1] * nc[2] / (ncf[0] * ncf[1] * ncf[2])
  rho = cic_paint(rho, state[0] * pm_nc_factor, wts)
  rho = rho * (1. / nbar)
  return r2c3d(rho, norm=ncf[0] * ncf[1] * ncf[2])


def force(bg, state, nc, pm_nc_factor=1):
  """flowpm/tfpm.py:317-366: paint at X*B, /nbar, r2c, 1.5 Omega_m
  long-range force read out at X*B, /B, written to state[2]."""
  nc = _nc3(nc)
  delta_k = _paint_density(state, nc, pm_nc_factor)
  fac = torch.as_tensor(np.asarray(bg.t(1.5) * bg.c.Omega_m)).to(state.dtype)
  update = apply_longrange(state[0] * pm_nc_factor, delta_k, split=0,
                           factor=fac)
  update = update / pm_nc_factor
  return torch.stack((state[0], state[1], update))


def pgd(state, pgdparams, nc, pm_nc_factor=1):
  """flowpm/tfpm.py:369-422: X += alpha * PGD displacement."""
  nc = _nc3(nc)
  delta_k = _paint_density(state, nc, pm_nc_factor)
  alpha, kl, ks = [float(v) for v in pgdparams]
  update = apply_pgd(state[0] * pm_nc_factor, delta_k,
                     torch.tensor(alpha, dtype=state.dtype), kl, ks)
  update = update / pm_nc_factor
  return torch.stack((state[0] + update, state[1], state[2]))


def nbody(bg, state, stages, nc, pm_nc_factor=1,
          return_intermediate_states=False, pgdparams=None):
  """flowpm/tfpm.py:425-503: KDK leapfrog over ``stages`` (one force call
  to start, then kick / drift / [pgd] / force / kick per step)."""
  nc = _nc3(nc)
  if len(stages) == 0:
    return state
  ai = stages[0]
  state = force(bg, state, nc, pm_nc_factor=pm_nc_factor)
  x, p, f = ai, ai, ai
  inter = []
  for i in range(len(stages) - 1):
    a0, a1 = stages[i], stages[i + 1]
    ah = (a0 * a1)**0.5
    state = kick(bg, state, p, f, ah)
    p = ah
    state = drift(bg, state, x, p, a1)
    if pgdparams is not None:
      state = pgd(state, pgdparams[i], nc, pm_nc_factor=pm_nc_factor)
    x = a1
    state = force(bg, state, nc, pm_nc_factor=pm_nc_factor)
    f = a1
    state = kick(bg, state, p, f, a1)
    p = a1
    inter.append((a1, state))
  return inter if return_intermediate_states else state


def nbody_checkpointed(bg, state, stages, nc, pm_nc_factor=1):
  """``nbody`` (no PGD, final state only) with the same arithmetic, each
  force and leapfrog step wrapped in torch.utils.checkpoint: autograd keeps
  only the state between steps and recomputes a step's graph during the
  backward, so the FP64 tape gradient of a 128^3, 20-step run fits in host
  memory (the plain graph holds every step's neighbour indices)."""
  from torch.utils.checkpoint import checkpoint
  nc = _nc3(nc)
  if len(stages) == 0:
    return state

  def step(st, i):
    a0, a1 = stages[i], stages[i + 1]
    ah = (a0 * a1)**0.5
    st = kick(bg, st, a0, a0, ah)
    st = drift(bg, st, a0, ah, a1)
    st = force(bg, st, nc, pm_nc_factor=pm_nc_factor)
    return kick(bg, st, ah, a1, a1)

  state = checkpoint(lambda s: force(bg, s, nc, pm_nc_factor=pm_nc_factor),
                     state, use_reentrant=False)
  for i in range(len(stages) - 1):
    state = checkpoint(step, state, i, use_reentrant=False)
  return state


# --------------------------------------------------------------------------
# flowpm/pk.py
# --------------------------------------------------------------------------
def power_spectrum(field, kmin=5, dk=0.5, boxsize=None):
  """flowpm/pk.py:7-103: binned |delta_k|^2 with the reference's mode
  weights W (2 except on the first and last z planes), bin edges
  arange(kmin, kmax, dk), normalisation prod(boxsize) / N^6."""
  shape = list(field.shape[1:])
  boxsize = np.asarray(boxsize, dtype=np.float64)
  I = np.eye(3, dtype='int') * -2 + 1
  W = np.empty(shape, dtype='f4')
  W[...] = 2.0
  W[..., 0] = 1.0
  W[..., -1] = 1.0
  kmax = np.pi * np.min(shape) / np.max(boxsize) + dk / 2
  kedges = np.arange(kmin, kmax, dk)
  k = [
      np.fft.fftfreq(N, 1. / (N * 2 * np.pi / L))[:pks].reshape(ks)
      for N, L, ks, pks in zip(shape, boxsize, I, shape)
  ]
  kmag = sum(ki**2 for ki in k)**0.5
  nbins = len(kedges) + 1
  dig = np.digitize(kmag.flat, kedges)
  Nsum = np.bincount(dig, weights=W.flat, minlength=nbins)
  cd = _cdtype(field.dtype)
  fk = torch.fft.fftn(field.to(cd), dim=(-3, -2, -1))
  pk = (fk * torch.conj(fk)).real
  digt = torch.as_tensor(dig)
  Wt = torch.as_tensor(W.ravel()).to(field.dtype)
  out = []
  for b in range(field.shape[0]):
    psum = torch.zeros(nbins, dtype=field.dtype).index_add(
        0, digt, Wt * pk[b].reshape(-1))
    out.append(psum / torch.as_tensor(Nsum).to(field.dtype))
  power = torch.stack(out)[:, 1:-1] * float(boxsize.prod())
  norm = float(np.prod(shape))**2
  kbins = kedges[:-1] + (kedges[1:] - kedges[:-1]) / 2
  return kbins, power / norm
