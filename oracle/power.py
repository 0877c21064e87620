"""Restatement of ``flowpm/tfpower.py`` (Eisenstein & Hu 1998 transfer
function, sigma8-normalised linear P(k)) and ``flowpm/scipy/integrate.py``
(Simpson's rule) in NumPy with a selectable float type.  Test infrastructure
only (see package docstring)."""
import numpy as np

from .background import Background

TCMB = 2.726  # flowpm/constants.py:13


def simps(f, a, b, N, t):
  """Composite Simpson's rule, flowpm/scipy/integrate.py:4-35."""
  dx = (b - a) / t(N)
  x = np.linspace(a, b, N + 1, dtype=t)
  y = f(x)
  return dx / t(3) * np.sum(y[0:-1:2] + t(4) * y[1::2] + y[2::2], axis=0)


def eisenstein_hu(bg, k, type='eisenhu_osc'):
  """flowpm/tfpower.py:28-159 (EH98 eqs. 2-7, 10-12, 14, 17-21, 29)."""
  t, c = bg.t, bg.c
  k = np.asarray(k, dtype=t)
  T27 = t((TCMB / 2.7)**2)
  h2 = c.h**2
  w_m = c.Omega_m * h2
  w_b = c.Omega_b * h2
  fb = c.Omega_b / c.Omega_m
  fc = (c.Omega_m - c.Omega_b) / c.Omega_m
  k_eq = t(7.46e-2) * w_m / T27 / c.h
  z_eq = t(2.50e4) * w_m / (T27)**2
  b1 = t(0.313) * np.power(w_m, t(-0.419)) * (
      t(1.0) + t(0.607) * np.power(w_m, t(0.674)))
  b2 = t(0.238) * np.power(w_m, t(0.223))
  z_d = (t(1291.0) * np.power(w_m, t(0.251)) /
         (t(1.0) + t(0.659) * np.power(w_m, t(0.828))) *
         (t(1.0) + b1 * np.power(w_b, b2)))
  R_d = t(31.5) * w_b / T27**2 * (t(1.0e3) / z_d)
  R_eq = t(31.5) * w_b / T27**2 * (t(1.0e3) / z_eq)
  sh_d = (t(2.0) / (t(3.0) * k_eq) * np.sqrt(t(6.0) / R_eq) * np.log(
      (np.sqrt(t(1.0) + R_d) + np.sqrt(R_eq + R_d)) /
      (t(1.0) + np.sqrt(R_eq))))
  k_silk = (t(1.6) * np.power(w_b, t(0.52)) * np.power(w_m, t(0.73)) *
            (t(1.0) + np.power(t(10.4) * w_m, t(-0.95))) / c.h)
  alpha_gamma = (t(1.0) - t(0.328) * np.log(t(431.0) * w_m) * w_b / w_m +
                 t(0.38) * np.log(t(22.3) * w_m) * (c.Omega_b / c.Omega_m)**2)
  gamma_eff = (c.Omega_m * c.h * (alpha_gamma + (t(1.0) - alpha_gamma) /
                                  (t(1.0) + (t(0.43) * k * sh_d)**4)))
  if type == 'eisenhu':
    q = k * np.power(t(TCMB / 2.7), t(2)) / gamma_eff
    L = np.log(t(2.0) * np.exp(t(1.0)) + t(1.8) * q)
    C = t(14.2) + t(731.0) / (t(1.0) + t(62.5) * q)
    return L / (L + C * q * q)
  if type != 'eisenhu_osc':
    raise NotImplementedError(type)
  a1 = np.power(t(46.9) * w_m, t(0.670)) * (
      t(1.0) + np.power(t(32.1) * w_m, t(-0.532)))
  a2 = np.power(t(12.0) * w_m, t(0.424)) * (
      t(1.0) + np.power(t(45.0) * w_m, t(-0.582)))
  alpha_c = np.power(a1, -fb) * np.power(a2, -(fb**3))
  bb1 = t(0.944) / (t(1.0) + np.power(t(458.0) * w_m, t(-0.708)))
  bb2 = np.power(t(0.395) * w_m, t(-0.0266))
  beta_c = t(1.0) / (t(1.0) + bb1 * (np.power(fc, bb2) - t(1.0)))

  def T_tilde(k1, alpha, beta):
    q = k1 / (t(13.41) * k_eq)
    L = np.log(np.exp(t(1.0)) + t(1.8) * beta * q)
    C = t(14.2) / alpha + t(386.0) / (t(1.0) + t(69.9) * np.power(q, t(1.08)))
    return L / (L + C * q * q)

  f = t(1.0) / (t(1.0) + (k * sh_d / t(5.4))**4)
  Tc = f * T_tilde(k, t(1.0), beta_c) + (t(1.0) - f) * T_tilde(
      k, alpha_c, beta_c)
  y = (t(1.0) + z_eq) / (t(1.0) + z_d)
  x = np.sqrt(t(1.0) + y)
  G = y * (t(-6.0) * x + (t(2.0) + t(3.0) * y) * np.log((x + t(1.0)) /
                                                         (x - t(1.0))))
  alpha_b = t(2.07) * k_eq * sh_d * np.power(t(1.0) + R_d, t(-0.75)) * G
  beta_node = t(8.41) * np.power(w_m, t(0.435))
  tilde_s = sh_d / np.power(t(1.0) + (beta_node / (k * sh_d))**3,
                            t(1.0 / 3.0))
  beta_b = t(0.5) + fb + (t(3.0) - t(2.0) * fb) * np.sqrt((t(17.2) * w_m)**2 +
                                                          t(1.0))
  Tb = (T_tilde(k, t(1.0), t(1.0)) / (t(1.0) + (k * sh_d / t(5.2))**2) +
        alpha_b / (t(1.0) + (beta_b / (k * sh_d))**3) *
        np.exp(-np.power(k / k_silk, t(1.4)))) * (
            np.sin(k * tilde_s) / (k * tilde_s + t(1e-9)))
  return fb * Tb + fc * Tc


def sigmasqr(bg, R, kmin=0.0001, kmax=1000.0, **kw):
  """flowpm/tfpower.py:193-218 (top-hat variance, 256 Simpson intervals in
  log10 k)."""
  t = bg.t

  def integrand(logk):
    k = np.exp(logk)
    x = k * t(R)
    w = t(3.0) * (np.sin(x) - x * np.cos(x)) / (x * x * x)
    pk = eisenstein_hu(bg, k, **kw)**2 * np.power(k, bg.c.n_s)
    return k * (k * w)**2 * pk

  lo = t(np.log(t(kmin))) / t(np.log(10))
  hi = t(np.log(t(kmax))) / t(np.log(10))
  y = simps(integrand, lo, hi, 256, t)
  return t(1.0 / (2.0 * np.pi**2.0)) * y


def linear_matter_power(bg, k, a=1.0, **kw):
  """flowpm/tfpower.py:162-190."""
  t = bg.t
  k = np.asarray(k, dtype=t)
  g = bg.D1(t(a))
  tr = eisenstein_hu(bg, k, **kw)
  pknorm = bg.c.sigma8**2 / sigmasqr(bg, 8.0, **kw)
  pk = np.power(k, bg.c.n_s) * tr**2 * g**2
  return np.squeeze(pk * pknorm)
