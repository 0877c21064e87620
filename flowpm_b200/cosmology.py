"""Cosmological parameters, mirroring ``flowpm/cosmology.py`` (``Cosmology``
:5-129 and ``Planck15`` :132-141).

Parameters are held as Python floats (FP64): the background quantities
derived from them are computed in double precision on the host.
"""
import math
from functools import partial


class Cosmology(object):
  """Cosmology object: primary and derived parameters plus a workspace where
  background functions cache their tables (flowpm/cosmology.py:39)."""

  def __init__(self, Omega_c, Omega_b, h, n_s, sigma8, Omega_k, w0, wa):
    self._Omega_c = float(Omega_c)
    self._Omega_b = float(Omega_b)
    self._h = float(h)
    self._n_s = float(n_s)
    self._sigma8 = float(sigma8)
    self._Omega_k = float(Omega_k)
    self._w0 = float(w0)
    self._wa = float(wa)
    self._flags = {}
    self._workspace = {}

  def to_dict(self):
    return {
        'Omega_c': self.Omega_c,
        'Omega_b': self.Omega_b,
        'h': self.h,
        'n_s': self.n_s,
        'sigma8': self.sigma8,
        'Omega_k': self.Omega_k,
        'w0': self.w0,
        'wa': self.wa
    }

  def key(self):
    """Hashable identity of the parameters (for caches)."""
    return tuple(sorted(self.to_dict().items()))

  def __str__(self):
    return ('Cosmological parameters: \n' + '    h:        ' + str(self.h) +
            ' \n' + '    Omega_b:  ' + str(self.Omega_b) + ' \n' +
            '    Omega_c:  ' + str(self.Omega_c) + ' \n' + '    Omega_k:  ' +
            str(self.Omega_k) + ' \n' + '    w0:       ' + str(self.w0) +
            ' \n' + '    wa:       ' + str(self.wa) + ' \n' +
            '    n:        ' + str(self.n_s) + ' \n' + '    sigma8:   ' +
            str(self.sigma8))

  __repr__ = __str__

  @property
  def Omega(self):
    return 1.0 - self._Omega_k

  @property
  def Omega_b(self):
    return self._Omega_b

  @property
  def Omega_c(self):
    return self._Omega_c

  @property
  def Omega_m(self):
    return self._Omega_b + self._Omega_c

  @property
  def Omega_de(self):
    return self.Omega - self.Omega_m

  @property
  def Omega_k(self):
    return self._Omega_k

  @property
  def k(self):
    if self.Omega > 1.0:
      return 1.0
    if self.Omega == 1.0:
      return 0
    return -1.0

  @property
  def sqrtk(self):
    return math.sqrt(abs(self._Omega_k))

  @property
  def h(self):
    return self._h

  @property
  def w0(self):
    return self._w0

  @property
  def wa(self):
    return self._wa

  @property
  def n_s(self):
    return self._n_s

  @property
  def sigma8(self):
    return self._sigma8


# Planck 2015 paper XII Table 4 final column (best fit).
Planck15 = partial(
    Cosmology,
    Omega_c=0.2589,
    Omega_b=0.04860,
    Omega_k=0.0,
    h=0.6774,
    n_s=0.9667,
    sigma8=0.8159,
    w0=-1.0,
    wa=0.0,
)
