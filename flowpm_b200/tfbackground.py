"""Background cosmology in FP64 on the host, mirroring ``flowpm/tfbackground.py``.

The method is the reference's -- the growth ODE (Leclercq thesis eq. 1.96,
flowpm/tfbackground.py:533-578) integrated by classic RK4 on 256 log-spaced
scale factors in [1e-2, 1] from a matter-dominated start
(flowpm/tfbackground.py:581-647), D and its derivatives read by linear
interpolation in ln a on that grid (tfp interp_regular_1d_grid,
flowpm/tfbackground.py:678) -- but evaluated in double precision instead of
float32.  These numbers only enter the particle-mesh step as per-step scalar
prefactors (kick, drift, LPT factors), which are rounded to float32 once.

The ODE tables are cached per cosmology in ``cosmo._workspace`` as the
reference does (flowpm/tfbackground.py:631-647).
"""
import numpy as np

__all__ = [
    'fde', 'w', 'E', 'H', 'dfde', 'dEa', 'Omega_m_a', 'Omega_de_a', 'D1', 'D2',
    'D1f', 'D2f', 'f1', 'f2', 'Gf', 'Gf2', 'gf', 'gf2', 'maybe_compute_ODE',
    'kick_factor', 'drift_factor', 'nbody_coefficients', 'lpt_coefficients'
]

_H0 = 100.0  # km/s/(Mpc/h), flowpm/constants.py:21


def _a(a):
  return np.asarray(a, dtype=np.float64)


def fde(cosmo, a, epsilon=1e-5):
  """Dark-energy density evolution exponent (flowpm/tfbackground.py:10-51)."""
  a = _a(a)
  return (-3.0 * (1.0 + cosmo.w0) + 3.0 * cosmo.wa *
          ((a - 1.0) / np.log(a - epsilon) - 1.0))


def w(cosmo, a):
  """Linder equation of state w0 + wa (1 - a) (:54-82)."""
  return cosmo.w0 + cosmo.wa * (1.0 - _a(a))


def E(cosmo, a):
  """E(a) = H(a)/H0 (:85-120)."""
  a = _a(a)
  return np.sqrt(cosmo.Omega_m / a**3 + cosmo.Omega_k / a**2 +
                 cosmo.Omega_de * np.power(a, fde(cosmo, a)))


def H(cosmo, a):
  """Hubble parameter in km/s/(Mpc/h) (:123-140)."""
  return _H0 * cosmo.h * E(cosmo, a)


def dfde(cosmo, a, epsilon=1e-5):
  """d fde / da (:143-176)."""
  a = _a(a)
  la = np.log(a - epsilon)
  return 3 * cosmo.wa * (la - (a - 1) / (a - epsilon)) / la**2


def dEa(cosmo, a):
  """dE/da (:179-212)."""
  a = _a(a)
  return 0.5 * (-3 * cosmo.Omega_m / a**4 - 2 * cosmo.Omega_k / a**3 +
                dfde(cosmo, a) * cosmo.Omega_de * np.power(a, fde(cosmo, a))
                ) / E(cosmo, a)


def Omega_m_a(cosmo, a):
  """Matter density parameter at a (:215-242)."""
  a = _a(a)
  return cosmo.Omega_m * a**-3 / E(cosmo, a)**2


def Omega_de_a(cosmo, a):
  """Dark-energy density parameter at a (:245-274)."""
  a = _a(a)
  return cosmo.Omega_de * np.power(a, fde(cosmo, a)) / E(cosmo, a)**2


def _growth_rhs(cosmo, a, y):
  """Right-hand side of the growth system for y = (D1, D1', D2, D2')."""
  om = Omega_m_a(cosmo, a)
  friction = Omega_de_a(cosmo, a) - 0.5 * om + 2.0
  d1, d1f, d2, d2f = y[..., 0], y[..., 1], y[..., 2], y[..., 3]
  dd1 = 1.5 * om * d1 / a**2 - (d1f / a) * friction
  dd2 = 1.5 * om * d2 / a**2 - (d2f / a) * friction - 1.5 * (
      om * d1**2) / a**2
  return np.stack([d1f, dd1, d2f, dd2], axis=-1)


def maybe_compute_ODE(cosmo, log10_amin=-2, steps=256):
  """Growth tables on a = logspace(log10_amin, 0, steps), normalised to 1 at
  a = 1, cached in ``cosmo._workspace`` (:631-647)."""
  key = ('cache_ODE_fp64', log10_amin, steps)
  if key in cosmo._workspace:
    return cosmo._workspace[key]
  a = np.logspace(log10_amin, 0.0, steps)
  y = np.array([a[0], 1.0, -3.0 / 7 * a[0]**2, -6.0 / 7 * a[0]])
  ys = [y]
  for i in range(steps - 1):
    t, dt = a[i], a[i + 1] - a[i]
    k1 = _growth_rhs(cosmo, t, y)
    k2 = _growth_rhs(cosmo, t + dt / 2.0, y + dt * k1 / 2.0)
    k3 = _growth_rhs(cosmo, t + dt / 2.0, y + dt * k2 / 2.0)
    k4 = _growth_rhs(cosmo, t + dt, y + dt * k3)
    y = y + dt * (k1 + 2.0 * k2 + 2.0 * k3 + k4) / 6.0
    ys.append(y)
  res = np.stack(ys)
  second = _growth_rhs(cosmo, a, res)
  cache = {
      'a': a,
      'D1': res[:, 0] / res[-1, 0],
      'D1f': res[:, 1] / res[-1, 0],
      'D2': res[:, 2] / res[-1, 2],
      'D2f': res[:, 3] / res[-1, 2],
      'F1p': second[:, 1] / res[-1, 0],
      'F2p': second[:, 3] / res[-1, 2],
  }
  cosmo._workspace[key] = cache
  return cache


def _interp(cosmo, a, name):
  """Linear interpolation in ln a on the regular ln-a grid of the ODE table,
  constant beyond its ends."""
  c = maybe_compute_ODE(cosmo)
  x = np.log(_a(a))
  xmin, xmax = np.log(c['a'][0]), np.log(c['a'][-1])
  y = c[name]
  n = len(y)
  idx = np.clip((x - xmin) / (xmax - xmin) * (n - 1), 0.0, n - 1.0)
  lo = np.clip(np.floor(idx), 0, n - 2).astype(np.int64)
  t = idx - lo
  return y[lo] + t * (y[lo + 1] - y[lo])


def D1(cosmo, a):
  """Normalised linear growth factor (:650-680)."""
  return _interp(cosmo, a, 'D1')


def D2(cosmo, a):
  """Normalised second-order growth factor (:683-714)."""
  return _interp(cosmo, a, 'D2')


def D1f(cosmo, a):
  """dD1/da (:717-749)."""
  return _interp(cosmo, a, 'D1f')


def D2f(cosmo, a):
  """dD2/da (:752-784)."""
  return _interp(cosmo, a, 'D2f')


def f1(cosmo, a):
  """Linear growth rate a D1'/D1 (:787-814)."""
  return D1f(cosmo, a) * _a(a) / D1(cosmo, a)


def f2(cosmo, a):
  """Second-order growth rate (:817-844)."""
  return D2f(cosmo, a) * _a(a) / D2(cosmo, a)


def Gf(cosmo, a):
  """FastPM growth factor function D1' a^3 E (:847-872)."""
  a = _a(a)
  return D1f(cosmo, a) * a**3 * E(cosmo, a)


def Gf2(cosmo, a):
  """Second-order Gf (:875-899)."""
  a = _a(a)
  return D2f(cosmo, a) * a**3 * E(cosmo, a)


def gf(cosmo, a):
  """dGf/da (:902-938)."""
  a = _a(a)
  d1f, f1p = _interp(cosmo, a, 'D1f'), _interp(cosmo, a, 'F1p')
  return (f1p * a**3 * E(cosmo, a) + d1f * a**3 * dEa(cosmo, a) +
          3 * a**2 * E(cosmo, a) * d1f)


def gf2(cosmo, a):
  """dGf2/da (:941-977)."""
  a = _a(a)
  d2f, f2p = _interp(cosmo, a, 'D2f'), _interp(cosmo, a, 'F2p')
  return (f2p * a**3 * E(cosmo, a) + d2f * a**3 * dEa(cosmo, a) +
          3 * a**2 * E(cosmo, a) * d2f)


def kick_factor(cosmo, ai, ac, af):
  """Kick prefactor of flowpm/tfpm.py:284-285."""
  return float(1 / (ac**2 * E(cosmo, ac)) * (Gf(cosmo, af) - Gf(cosmo, ai)) /
               gf(cosmo, ac))


def drift_factor(cosmo, ai, ac, af):
  """Drift prefactor of flowpm/tfpm.py:306-307."""
  return float(1. / (ac**3 * E(cosmo, ac)) * (D1(cosmo, af) - D1(cosmo, ai)) /
               D1f(cosmo, ac))


def nbody_coefficients(cosmo, stages):
  """Per-step {kick_start, drift, kick_end} of the KDK loop of
  flowpm/tfpm.py:475-498 for ``len(stages) - 1`` steps, shape (steps, 3)."""
  stages = [float(s) for s in stages]
  out = np.zeros((max(len(stages) - 1, 0), 3))
  for i in range(len(stages) - 1):
    a0, a1 = stages[i], stages[i + 1]
    ah = (a0 * a1)**0.5
    out[i, 0] = kick_factor(cosmo, a0, a0, ah)
    out[i, 1] = drift_factor(cosmo, a0, ah, a1)
    out[i, 2] = kick_factor(cosmo, ah, a1, a1)
  return out


def lpt_coefficients(cosmo, a):
  """{D1, D2, a^2 f1 E, a^2 f2 E, a^2 E gf / D1, a^2 E gf2 / D2} of
  flowpm/tfpm.py:168-177."""
  a = float(a)
  d1, d2, e = float(D1(cosmo, a)), float(D2(cosmo, a)), float(E(cosmo, a))
  return np.array([
      d1, d2, a**2 * float(f1(cosmo, a)) * e, a**2 * float(f2(cosmo, a)) * e,
      a**2 * e * float(gf(cosmo, a)) / d1, a**2 * e * float(gf2(cosmo, a)) / d2
  ])
