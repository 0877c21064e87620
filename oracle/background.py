"""Restatement of ``flowpm/tfbackground.py`` (growth ODE + FastPM factors) in
NumPy with a selectable float type.  Test infrastructure only (see package
docstring).

``Background(params, dtype=np.float32)`` reproduces the reference arithmetic
(float32, as TensorFlow computes it); ``dtype=np.float64`` is the same method
in double precision.
"""
import numpy as np

PLANCK15 = dict(Omega_c=0.2589, Omega_b=0.04860, Omega_k=0.0, h=0.6774,
                n_s=0.9667, sigma8=0.8159, w0=-1.0, wa=0.0)


class Params(object):
  """Cosmological parameters, ``flowpm/cosmology.py:5-129`` (derived
  Omega_m = Omega_b + Omega_c :82, Omega_de = 1 - Omega_k - Omega_m :66,86)."""

  def __init__(self, dtype=np.float32, **kw):
    p = dict(PLANCK15)
    p.update(kw)
    t = np.dtype(dtype).type
    for k, v in p.items():
      setattr(self, k, t(v))
    self.Omega_m = self.Omega_b + self.Omega_c
    self.Omega_de = (t(1.0) - self.Omega_k) - self.Omega_m


class Background(object):

  def __init__(self, params=None, dtype=np.float32, log10_amin=-2, steps=256,
               **kw):
    self.t = np.dtype(dtype).type
    self.c = Params(dtype, **(params or {})) if not isinstance(
        params, Params) else params
    for k, v in kw.items():
      setattr(self.c, k, self.t(v))
    self._ode = None
    self.log10_amin, self.steps = log10_amin, steps

  # -- flowpm/tfbackground.py:10-52
  def fde(self, a, epsilon=1e-5):
    t, c = self.t, self.c
    a = np.asarray(a, dtype=t)
    return (t(-3.0) * (t(1.0) + c.w0) + t(3.0) * c.wa *
            ((a - t(1.0)) / np.log(a - t(epsilon)) - t(1.0)))

  # -- flowpm/tfbackground.py:85-120
  def E(self, a):
    t, c = self.t, self.c
    a = np.asarray(a, dtype=t)
    return np.sqrt(c.Omega_m / np.power(a, t(3)) + c.Omega_k /
                   np.power(a, t(2)) + c.Omega_de * np.power(a, self.fde(a)))

  # -- flowpm/tfbackground.py:143-176
  def dfde(self, a, epsilon=1e-5):
    t, c = self.t, self.c
    a = np.asarray(a, dtype=t)
    e = t(epsilon)
    return (t(3) * c.wa * (np.log(a - e) - (a - t(1)) / (a - e)) /
            np.power(np.log(a - e), t(2)))

  # -- flowpm/tfbackground.py:179-212
  def dEa(self, a):
    t, c = self.t, self.c
    a = np.asarray(a, dtype=t)
    return t(0.5) * (t(-3) * c.Omega_m / np.power(a, t(4)) -
                     t(2) * c.Omega_k / np.power(a, t(3)) + self.dfde(a) *
                     c.Omega_de * np.power(a, self.fde(a))) / self.E(a)

  # -- flowpm/tfbackground.py:215-242
  def Omega_m_a(self, a):
    t, c = self.t, self.c
    a = np.asarray(a, dtype=t)
    return c.Omega_m * np.power(a, t(-3)) / self.E(a)**t(2)

  # -- flowpm/tfbackground.py:245-274
  def Omega_de_a(self, a):
    t, c = self.t, self.c
    a = np.asarray(a, dtype=t)
    return c.Omega_de * np.power(a, self.fde(a)) / self.E(a)**t(2)

  # -- flowpm/tfbackground.py:533-578 (Leclercq thesis eq. 1.96)
  def growth_ode(self, a, y):
    t = self.t
    a = np.asarray(a, dtype=t)
    d1, d1f, d2, d2f = [y[..., i:i + 1] for i in range(4)]
    om = self.Omega_m_a(a)
    ode = self.Omega_de_a(a)
    dd1 = t(1.5) * om * d1 / np.power(a, t(2)) - (d1f / a) * (
        ode - t(0.5) * om + t(2))
    dd2 = t(1.5) * om * d2 / np.power(a, t(2)) - (d2f / a) * (
        ode - t(0.5) * om + t(2)) - t(1.5) * (om * d1**2) / np.power(a, t(2))
    return np.concatenate([d1f, dd1, d2f, dd2], axis=-1)

  # -- flowpm/tfbackground.py:491-530 (classic RK4 on the given a grid)
  def rk4(self, a, y0):
    t = self.t
    da = a[1:] - a[:-1]
    ys = [y0]
    y = y0
    for i in range(len(da)):
      ti, dt = a[i], da[i]
      f1 = self.growth_ode(ti, y)
      f2 = self.growth_ode(ti + dt / t(2), y + dt * f1 / t(2))
      f3 = self.growth_ode(ti + dt / t(2), y + dt * f2 / t(2))
      f4 = self.growth_ode(ti + dt, y + dt * f3)
      y = y + dt * (f1 + t(2) * f2 + t(2) * f3 + f4) / t(6)
      ys.append(y)
    return np.stack(ys)

  # -- flowpm/tfbackground.py:581-647 (IC :601, normalisation :613-618,
  # 256 log steps on [1e-2, 1] :631-645)
  def ode(self):
    if self._ode is None:
      t = self.t
      a = np.logspace(self.log10_amin, 0., self.steps).astype(t)
      y0 = np.array([[a[0], 1.0, -3. / 7 * a[0]**2, -6. / 7 * a[0]]],
                    dtype=t)
      res = self.rk4(a, y0)[:, 0]
      second = self.growth_ode(a[:, None], res)
      self._ode = {
          'a': a,
          'D1': res[:, 0] / res[-1, 0],
          'D1f': res[:, 1] / res[-1, 0],
          'D2': res[:, 2] / res[-1, 2],
          'D2f': res[:, 3] / res[-1, 2],
          'F1p': second[:, 1] / res[-1, 0],
          'F2p': second[:, 3] / res[-1, 2],
      }
    return self._ode

  def _interp(self, a, key):
    """Linear interpolation in ln a on the regular ln-a grid, constant
    extension (tfp.math.interp_regular_1d_grid as called at
    flowpm/tfbackground.py:678)."""
    t = self.t
    c = self.ode()
    x = np.log(np.asarray(a, dtype=t))
    xmin, xmax = np.log(c['a'][0]), np.log(c['a'][-1])
    y = c[key]
    n = len(y)
    idx = np.clip((x - xmin) / (xmax - xmin) * t(n - 1), t(0), t(n - 1))
    lo = np.clip(np.floor(idx), 0, n - 2).astype(np.int64)
    w = (idx - lo.astype(t)).astype(t)
    return (y[lo] + w * (y[lo + 1] - y[lo])).astype(t)

  # -- flowpm/tfbackground.py:650-784
  def D1(self, a):
    return self._interp(a, 'D1')

  def D2(self, a):
    return self._interp(a, 'D2')

  def D1f(self, a):
    return self._interp(a, 'D1f')

  def D2f(self, a):
    return self._interp(a, 'D2f')

  # -- flowpm/tfbackground.py:787-844
  def f1(self, a):
    a = np.asarray(a, dtype=self.t)
    return self.D1f(a) * a / self.D1(a)

  def f2(self, a):
    a = np.asarray(a, dtype=self.t)
    return self.D2f(a) * a / self.D2(a)

  # -- flowpm/tfbackground.py:847-899
  def Gf(self, a):
    a = np.asarray(a, dtype=self.t)
    return self.D1f(a) * a**3 * self.E(a)

  def Gf2(self, a):
    a = np.asarray(a, dtype=self.t)
    return self.D2f(a) * a**3 * self.E(a)

  # -- flowpm/tfbackground.py:902-977
  def gf(self, a):
    t = self.t
    a = np.asarray(a, dtype=t)
    d1f, f1p = self._interp(a, 'D1f'), self._interp(a, 'F1p')
    return (f1p * a**3 * self.E(a) + d1f * a**3 * self.dEa(a) +
            t(3) * a**2 * self.E(a) * d1f)

  def gf2(self, a):
    t = self.t
    a = np.asarray(a, dtype=t)
    d2f, f2p = self._interp(a, 'D2f'), self._interp(a, 'F2p')
    return (f2p * a**3 * self.E(a) + d2f * a**3 * self.dEa(a) +
            t(3) * a**2 * self.E(a) * d2f)

  # -- prefactors of flowpm/tfpm.py:284-285 (kick) and :306-307 (drift)
  # (ac**2 / ac**3 are formed in double from the Python stage values and
  # rounded once, as in the reference).
  def kick_factor(self, ai, ac, af):
    t = self.t
    return (t(1) / (t(float(ac)**2) * self.E(ac)) *
            (self.Gf(af) - self.Gf(ai)) / self.gf(ac)).astype(t)

  def drift_factor(self, ai, ac, af):
    t = self.t
    return (t(1.) / (t(float(ac)**3) * self.E(ac)) *
            (self.D1(af) - self.D1(ai)) / self.D1f(ac)).astype(t)
