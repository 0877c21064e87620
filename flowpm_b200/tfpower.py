"""Linear matter power spectrum in FP64 on the host, mirroring
``flowpm/tfpower.py`` (Eisenstein & Hu 1998 transfer function with and
without BAO, sigma8 normalisation by Simpson's rule on 256 intervals of
log10 k in [-4, 3]).  Used to build the Gaussian initial conditions; it is
evaluated once per cosmology.
"""
import numpy as np

from . import tfbackground as bkgrd

TCMB = 2.726  # K, flowpm/constants.py:13

__all__ = ['primordial_matter_power', 'Eisenstein_Hu', 'linear_matter_power',
           'sigmasqr']


def primordial_matter_power(cosmo, k):
  """k^n_s (flowpm/tfpower.py:9-25)."""
  return np.asarray(k, dtype=np.float64)**cosmo.n_s


def Eisenstein_Hu(cosmo, k, type='eisenhu_osc'):
  """EH98 transfer function (flowpm/tfpower.py:28-159)."""
  k = np.asarray(k, dtype=np.float64)
  T27 = (TCMB / 2.7)**2
  h2 = cosmo.h**2
  w_m = cosmo.Omega_m * h2
  w_b = cosmo.Omega_b * h2
  fb = cosmo.Omega_b / cosmo.Omega_m
  fc = (cosmo.Omega_m - cosmo.Omega_b) / cosmo.Omega_m
  k_eq = 7.46e-2 * w_m / T27 / cosmo.h  # EH98 eq. 3, h/Mpc
  z_eq = 2.50e4 * w_m / T27**2  # eq. 2
  b1 = 0.313 * w_m**-0.419 * (1.0 + 0.607 * w_m**0.674)
  b2 = 0.238 * w_m**0.223
  z_d = (1291.0 * w_m**0.251 / (1.0 + 0.659 * w_m**0.828) *
         (1.0 + b1 * w_b**b2))  # eq. 4
  R_d = 31.5 * w_b / T27**2 * (1.0e3 / z_d)  # eq. 5
  R_eq = 31.5 * w_b / T27**2 * (1.0e3 / z_eq)
  sh_d = (2.0 / (3.0 * k_eq) * np.sqrt(6.0 / R_eq) * np.log(
      (np.sqrt(1.0 + R_d) + np.sqrt(R_eq + R_d)) / (1.0 + np.sqrt(R_eq))))
  k_silk = (1.6 * w_b**0.52 * w_m**0.73 * (1.0 + (10.4 * w_m)**-0.95) /
            cosmo.h)  # eq. 7
  alpha_gamma = (1.0 - 0.328 * np.log(431.0 * w_m) * w_b / w_m +
                 0.38 * np.log(22.3 * w_m) * (cosmo.Omega_b / cosmo.Omega_m)**2)
  gamma_eff = (cosmo.Omega_m * cosmo.h *
               (alpha_gamma + (1.0 - alpha_gamma) / (1.0 + (0.43 * k * sh_d)**4)))
  if type == 'eisenhu':
    q = k * (TCMB / 2.7)**2 / gamma_eff
    L = np.log(2.0 * np.exp(1.0) + 1.8 * q)  # eq. 29
    C = 14.2 + 731.0 / (1.0 + 62.5 * q)
    return L / (L + C * q * q)
  if type != 'eisenhu_osc':
    raise NotImplementedError(type)
  a1 = (46.9 * w_m)**0.670 * (1.0 + (32.1 * w_m)**-0.532)  # eq. 11
  a2 = (12.0 * w_m)**0.424 * (1.0 + (45.0 * w_m)**-0.582)
  alpha_c = a1**-fb * a2**-(fb**3)
  bb1 = 0.944 / (1.0 + (458.0 * w_m)**-0.708)  # eq. 12
  bb2 = (0.395 * w_m)**-0.0266
  beta_c = 1.0 / (1.0 + bb1 * (fc**bb2 - 1.0))

  def T_tilde(k1, alpha, beta):  # eq. 10, 19
    q = k1 / (13.41 * k_eq)
    L = np.log(np.exp(1.0) + 1.8 * beta * q)
    C = 14.2 / alpha + 386.0 / (1.0 + 69.9 * q**1.08)
    return L / (L + C * q * q)

  f = 1.0 / (1.0 + (k * sh_d / 5.4)**4)  # eq. 18
  Tc = f * T_tilde(k, 1.0, beta_c) + (1.0 - f) * T_tilde(k, alpha_c, beta_c)
  y = (1.0 + z_eq) / (1.0 + z_d)
  x = np.sqrt(1.0 + y)
  G = y * (-6.0 * x + (2.0 + 3.0 * y) * np.log((x + 1.0) / (x - 1.0)))
  alpha_b = 2.07 * k_eq * sh_d * (1.0 + R_d)**-0.75 * G  # eq. 14
  beta_node = 8.41 * w_m**0.435
  tilde_s = sh_d / (1.0 + (beta_node / (k * sh_d))**3)**(1.0 / 3.0)
  beta_b = 0.5 + fb + (3.0 - 2.0 * fb) * np.sqrt((17.2 * w_m)**2 + 1.0)
  Tb = (T_tilde(k, 1.0, 1.0) / (1.0 + (k * sh_d / 5.2)**2) + alpha_b /
        (1.0 + (beta_b / (k * sh_d))**3) * np.exp(-(k / k_silk)**1.4)) * (
            np.sin(k * tilde_s) / (k * tilde_s + 1e-9))  # eq. 21
  return fb * Tb + fc * Tc


def _simps(f, a, b, N):
  dx = (b - a) / N
  x = np.linspace(a, b, N + 1)
  y = f(x)
  return dx / 3 * np.sum(y[0:-1:2] + 4 * y[1::2] + y[2::2], axis=0)


def sigmasqr(cosmo, R, transfer_fn=Eisenstein_Hu, kmin=0.0001, kmax=1000.0,
             **kwargs):
  """Top-hat variance in a sphere of R Mpc/h (flowpm/tfpower.py:193-218)."""

  def integrand(logk):
    k = np.exp(logk)
    x = k * R
    wt = 3.0 * (np.sin(x) - x * np.cos(x)) / (x * x * x)
    pk = transfer_fn(cosmo, k, **kwargs)**2 * primordial_matter_power(cosmo, k)
    return k * (k * wt)**2 * pk

  y = _simps(integrand,
             np.log(kmin) / np.log(10),
             np.log(kmax) / np.log(10), 256)
  return 1.0 / (2.0 * np.pi**2.0) * y


def linear_matter_power(cosmo, k, a=1.0, transfer_fn=Eisenstein_Hu, **kwargs):
  """sigma8-normalised linear P(k) at scale factor a
  (flowpm/tfpower.py:162-190)."""
  k = np.asarray(k, dtype=np.float64)
  g = bkgrd.D1(cosmo, a)
  t = transfer_fn(cosmo, k, **kwargs)
  pknorm = cosmo.sigma8**2 / sigmasqr(cosmo, 8.0, transfer_fn, **kwargs)
  pk = primordial_matter_power(cosmo, k) * t**2 * g**2
  return np.squeeze(pk * pknorm)
