"""Snapshot IO in the BigFile layout: ``save_state`` of flowpm/io.py:5-60,
and ``load_state`` to resume a run from such a snapshot.

A BigFile is a directory tree. Every block (``Header``, ``0/Position``, ...)
is a directory holding:

* ``header``, text: ``DTYPE: <f4`` / ``NMEMB: 3`` / ``NFILE: 1``, then one
  line per data file, ``%06X: <rows> : <byte sum> : <SysV checksum>``.
  The byte sum is the file's bytes added modulo 2^32; the checksum folds
  it to 16 bits twice (r = (s & 0xffff) + (s >> 16), then the same on r);
* ``attr-v2``, text: one attribute per line,
  ``<name> <dtype> <nmemb> <bytes as upper-case hex>``;
* the data files ``000000``, ... : rows of NMEMB items, little endian.

This is the on-disk layout that the ``bigfile`` library writes, restated
from its published description. The library is not installed here, so the
tests check the writer against this restatement and the reader, not
against the library itself.

IO is host work at the end of a run. It copies the state to host memory
and is not part of the device path.
"""
import os

import numpy as np

_DATA_FILE = '%06X'


def _le(dt):
  dt = np.dtype(dt)
  return dt if dt.byteorder in ('<', '|') else dt.newbyteorder('<')


def _dtype_name(dt):
  dt = np.dtype(dt)
  if dt.kind == 'S':
    return '|S1'
  return _le(dt).str


def _checksums(raw):
  s = int(np.frombuffer(raw, np.uint8).sum(dtype=np.uint64)) & 0xffffffff
  r = (s & 0xffff) + (s >> 16)
  return s, (r & 0xffff) + (r >> 16)


def _attr_array(value):
  if isinstance(value, (str, bytes)):
    b = value.encode() if isinstance(value, str) else value
    return np.frombuffer(b, dtype='S1')
  a = np.asarray(value)
  if a.dtype.kind in 'US':
    return np.frombuffer(str(a.item()).encode(), dtype='S1')
  if a.dtype.kind not in 'biuf':
    raise TypeError('attribute of unsupported type %s' % a.dtype)
  if a.dtype.kind == 'b':
    a = a.astype(np.uint8)
  return np.ascontiguousarray(a.reshape(-1), dtype=_le(a.dtype))


def write_block(root, name, data=None, attrs=None):
  """Write block ``name`` of the BigFile at ``root``: ``data`` (rows x NMEMB,
  or a vector) in one data file, and ``attrs`` (name -> number, array or
  string). ``data=None`` makes an attribute-only block."""
  path = os.path.join(root, *name.split('/'))
  os.makedirs(path, exist_ok=True)
  if data is None:
    lines = ['DTYPE: <i8', 'NMEMB: 1', 'NFILE: 0']
  else:
    data = np.asarray(data)
    nmemb = 1 if data.ndim == 1 else int(np.prod(data.shape[1:]))
    data = np.ascontiguousarray(data, dtype=_le(data.dtype))
    raw = data.tobytes()
    with open(os.path.join(path, _DATA_FILE % 0), 'wb') as f:
      f.write(raw)
    s, ck = _checksums(raw)
    lines = ['DTYPE: %s' % _dtype_name(data.dtype), 'NMEMB: %d' % nmemb,
             'NFILE: 1', '%06X: %d : %d : %d' % (0, data.shape[0], s, ck)]
  with open(os.path.join(path, 'header'), 'w') as f:
    f.write('\n'.join(lines) + '\n')
  with open(os.path.join(path, 'attr-v2'), 'w') as f:
    for key, value in (attrs or {}).items():
      a = _attr_array(value)
      f.write('%s %s %d %s\n' % (key, _dtype_name(a.dtype), a.size,
                                 a.tobytes().hex().upper()))


def read_attrs(root, name):
  """Attributes of block ``name`` (strings as str, the rest as arrays)."""
  out = {}
  path = os.path.join(root, *name.split('/'), 'attr-v2')
  if not os.path.exists(path):
    return out
  with open(path) as f:
    for line in f:
      line = line.rstrip('\n')
      if not line:
        continue
      key, dt, nmemb, hexdata = line.split(' ', 3)
      a = np.frombuffer(bytes.fromhex(hexdata), dtype=np.dtype(dt))
      if a.size != int(nmemb):
        raise ValueError('attribute %s of block %s: %d items, header says %s'
                         % (key, name, a.size, nmemb))
      out[key] = (a.tobytes().decode() if a.dtype.kind == 'S' else a.copy())
  return out


def read_block(root, name, verify=True):
  """Data of block ``name`` (rows x NMEMB, or a vector when NMEMB = 1),
  checking every data file's size and, with ``verify``, its checksums."""
  path = os.path.join(root, *name.split('/'))
  meta, files = {}, []
  with open(os.path.join(path, 'header')) as f:
    for line in f:
      line = line.strip()
      if not line:
        continue
      key, rest = line.split(':', 1)
      if key in ('DTYPE', 'NMEMB', 'NFILE'):
        meta[key] = rest.strip()
      else:
        rows, s, ck = (int(v) for v in rest.split(':'))
        files.append((int(key, 16), rows, s, ck))
  dt = np.dtype(meta['DTYPE'])
  nmemb = int(meta['NMEMB'])
  if len(files) != int(meta['NFILE']):
    raise ValueError('block %s: %d file lines, NFILE %s'
                     % (name, len(files), meta['NFILE']))
  parts = []
  for fid, rows, s, ck in sorted(files):
    with open(os.path.join(path, _DATA_FILE % fid), 'rb') as f:
      raw = f.read()
    if len(raw) != rows * nmemb * dt.itemsize:
      raise ValueError('block %s file %06X: %d bytes, expected %d'
                       % (name, fid, len(raw), rows * nmemb * dt.itemsize))
    if verify and _checksums(raw) != (s, ck):
      raise ValueError('block %s file %06X: checksum mismatch' % (name, fid))
    parts.append(np.frombuffer(raw, dtype=dt))
  data = (np.concatenate(parts) if parts else np.zeros(0, dt))
  return data.reshape(-1, nmemb) if nmemb > 1 else data


def _host(x):
  if hasattr(x, 'detach'):
    return x.detach().cpu().numpy()
  return np.asarray(x)


def _cell_size(nc, boxsize):
  # float32 as the reference: (1 / nc) * boxsize per axis (flowpm/io.py:52-56)
  return ((np.float32(1.0) / np.asarray(nc, dtype=np.float32)) *
          np.asarray(boxsize, dtype=np.float32)).astype(np.float32)


def save_state(cosmo, state, a, nc, boxsize, filename, attrs={}):
  """Write the snapshot of ``state`` (3, batch, npart, 3) at scale factor
  ``a`` to the BigFile ``filename`` (flowpm/io.py:5-60): a ``Header`` block
  with the attributes NC, BoxSize, OmegaCDM, OmegaB, OmegaK, h, Sigma8, w0,
  wa, Time and M0 (plus ``attrs``, best effort), and per batch entry i the
  blocks ``i/Position`` and ``i/Velocity``: X and P in Mpc/h (mesh units
  times boxsize / nc, in float32)."""
  state = _host(state)
  if state.ndim != 4 or state.shape[0] < 2 or state.shape[3] != 3:
    raise ValueError('state must be (3, batch, npart, 3), got %s'
                     % (state.shape,))
  f32 = np.float32
  header = {
      'NC': np.asarray(nc), 'BoxSize': np.asarray(boxsize),
      'OmegaCDM': f32(cosmo.Omega_c), 'OmegaB': f32(cosmo.Omega_b),
      'OmegaK': f32(cosmo.Omega_k), 'h': f32(cosmo.h),
      'Sigma8': f32(cosmo.sigma8), 'w0': f32(cosmo.w0), 'wa': f32(cosmo.wa),
      'Time': a, 'M0': [1.0],
  }
  for key in attrs:
    try:  # best effort, as the reference
      _attr_array(attrs[key])
      header[key] = attrs[key]
    except Exception:  # noqa: BLE001
      pass
  os.makedirs(filename, exist_ok=True)
  write_block(filename, 'Header', None, header)
  scale = _cell_size(nc, boxsize).reshape(1, 3)
  for i in range(state.shape[1]):
    write_block(filename, '%d/Position' % i,
                (state[0, i].astype(np.float32) * scale).astype(np.float32))
    write_block(filename, '%d/Velocity' % i,
                (state[1, i].astype(np.float32) * scale).astype(np.float32))


def load_state(filename, device='cuda'):
  """Read a snapshot written by ``save_state`` back into the state layout.

  Returns ``(state, a, header)``: ``state`` (3, batch, npart, 3) float32 in
  mesh units (X, P, and F = 0, which the next ``nbody`` call recomputes), on
  ``device``; ``a`` the snapshot's scale factor; ``header`` the Header
  attributes. X and P come back as (Mpc/h value) / (boxsize / nc) in
  float32, within one rounding of the saved state."""
  import torch
  header = read_attrs(filename, 'Header')
  nc = header['NC']
  scale = _cell_size(nc, header['BoxSize']).reshape(1, 3)
  batch = 0
  while os.path.isdir(os.path.join(filename, str(batch))):
    batch += 1
  if batch == 0:
    raise ValueError('%s holds no particle blocks' % filename)
  xs, ps = [], []
  for i in range(batch):
    xs.append(read_block(filename, '%d/Position' % i) / scale)
    ps.append(read_block(filename, '%d/Velocity' % i) / scale)
  x = np.stack(xs).astype(np.float32)
  p = np.stack(ps).astype(np.float32)
  state = np.stack([x, p, np.zeros_like(x)])
  return (torch.from_numpy(state).to(device), float(header['Time'][0]),
          header)
