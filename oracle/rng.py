"""NumPy restatement of the white-noise generator of the CUDA library
(Philox4x32-10 of Salmon, Moraes, Dror & Shaw, SC'11, with Box-Muller) --
test infrastructure only.

The reference draws its noise with TensorFlow's stateful Philox
(flowpm/utils.py:346-350 tf.random.normal), whose stream cannot be
reproduced without TensorFlow; this restatement only checks that the
library's generator is the documented one: element e of the output uses
counter (e // 4) and lane e % 4 of z = (r_a cos 2 pi u1, r_a sin 2 pi u1,
r_b cos 2 pi u3, r_b sin 2 pi u3), r = sqrt(-2 ln u), u = (x + 0.5) / 2^32.
"""
import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr, key):
  """ctr: (n, 4) uint32, key: (2,) uint32 -> (n, 4) uint32."""
  c = [ctr[:, i].astype(np.uint64) for i in range(4)]
  k0, k1 = np.uint64(key[0]), np.uint64(key[1])
  for _ in range(10):
    p0 = M0 * c[0]
    p1 = M1 * c[2]
    hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
    hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
    c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
    k0 = (k0 + np.uint64(W0)) & MASK
    k1 = (k1 + np.uint64(W1)) & MASK
  return np.stack(c, axis=1).astype(np.uint32)


def white_noise(n, seed, stddev=1.0):
  """First n values of the library's noise stream for ``seed``."""
  groups = (n + 3) // 4
  m = np.arange(groups, dtype=np.uint64)
  ctr = np.zeros((groups, 4), dtype=np.uint32)
  ctr[:, 0] = (m & MASK).astype(np.uint32)
  ctr[:, 1] = (m >> np.uint64(32)).astype(np.uint32)
  seed = int(seed) & 0xFFFFFFFFFFFFFFFF
  key = np.array([seed & 0xFFFFFFFF, seed >> 32], dtype=np.uint32)
  r = philox4x32_10(ctr, key).astype(np.float64)
  u = (r + 0.5) * (1.0 / 4294967296.0)
  ra = np.sqrt(-2.0 * np.log(u[:, 0]))
  rb = np.sqrt(-2.0 * np.log(u[:, 2]))
  z = np.stack([ra * np.cos(2 * np.pi * u[:, 1]), ra * np.sin(2 * np.pi * u[:, 1]),
                rb * np.cos(2 * np.pi * u[:, 3]), rb * np.sin(2 * np.pi * u[:, 3])],
               axis=1).ravel()[:n]
  return (stddev * z).astype(np.float32)
