"""Snapshot IO in the BigFile layout (flowpm_b200.io; flowpm/io.py:5-60 and
tests/test_io.py of the reference): the blocks and attributes that the
reference's test reads back, the exact text of the block headers and
attribute lines, corrupted and truncated data files, and the resume path
(load_state). The CPU tests use a host state; the GPU test follows the
reference's test (linear field, LPT at a = 0.1, batch of 2)."""
import os
import struct

import numpy as np
import pytest
from numpy.testing import assert_allclose, assert_array_equal

NC = [16, 16, 16]
BOX = [100., 100., 100.]


@pytest.fixture(scope='module')
def fio():
  from flowpm_b200 import io
  return io


@pytest.fixture(scope='module')
def cosmo():
  from flowpm_b200 import cosmology
  return cosmology.Planck15()


def _state(seed=0, batch=2, npart=16**3):
  rng = np.random.default_rng(seed)
  s = rng.standard_normal((3, batch, npart, 3)).astype(np.float32)
  s[0] = np.abs(s[0]) * 5.0  # positions in mesh units
  return s


def _cell():
  return ((np.float32(1) / np.asarray(NC, np.float32)) *
          np.asarray(BOX, np.float32)).astype(np.float32)


def test_save_state_blocks_and_header(fio, cosmo, tmp_path):
  """What the reference's test_save_state reads back through bigfile."""
  state = _state()
  fn = str(tmp_path / 'snap')
  fio.save_state(cosmo, state, 0.1, NC, BOX, fn)
  h = fio.read_attrs(fn, 'Header')
  assert_allclose(h['NC'], NC)
  assert_allclose(h['BoxSize'], BOX)
  assert_allclose(h['OmegaCDM'], np.float32(cosmo.Omega_c))
  assert_allclose(h['OmegaB'], np.float32(cosmo.Omega_b))
  assert_allclose(h['OmegaK'], np.float32(cosmo.Omega_k))
  assert_allclose(h['h'], np.float32(cosmo.h))
  assert_allclose(h['Sigma8'], np.float32(cosmo.sigma8))
  assert_allclose(h['w0'], np.float32(cosmo.w0))
  assert_allclose(h['wa'], np.float32(cosmo.wa))
  assert_allclose(h['Time'], 0.1)
  assert_allclose(h['M0'], [1.0])
  assert h['NC'].dtype == np.dtype('<i8') and h['h'].dtype == np.dtype('<f4')
  for i in range(2):
    pos = fio.read_block(fn, '%d/Position' % i)
    vel = fio.read_block(fn, '%d/Velocity' % i)
    assert pos.shape == (16**3, 3) and pos.dtype == np.dtype('<f4')
    # float32 products, as the reference's state * scaling_factor
    assert_array_equal(pos, state[0, i] * _cell())
    assert_array_equal(vel, state[1, i] * _cell())
    assert_allclose(pos, state[0, i] / NC[0] * BOX[0], rtol=1e-6)


def test_block_text_layout(fio, tmp_path):
  """Header and attr-v2 text, byte for byte, for a known block."""
  data = np.arange(12, dtype=np.float32).reshape(4, 3) - 2.5
  fn = str(tmp_path / 'f')
  fio.write_block(fn, '0/Position', data,
                  {'BoxSize': [100., 100., 100.], 'NC': [16, 16, 16],
                   'Name': 'pm'})
  raw = data.astype('<f4').tobytes()
  s = 0
  for b in raw:
    s = (s + b) % 2**32
  r = (s & 0xffff) + (s >> 16)
  ck = (r & 0xffff) + (r >> 16)
  with open(os.path.join(fn, '0', 'Position', 'header')) as f:
    assert f.read() == ('DTYPE: <f4\nNMEMB: 3\nNFILE: 1\n'
                        '000000: 4 : %d : %d\n' % (s, ck))
  with open(os.path.join(fn, '0', 'Position', '000000'), 'rb') as f:
    assert f.read() == raw
  with open(os.path.join(fn, '0', 'Position', 'attr-v2')) as f:
    lines = f.read().splitlines()
  assert lines[0] == 'BoxSize <f8 3 ' + struct.pack('<3d', 100., 100.,
                                                      100.).hex().upper()
  assert lines[1] == 'NC <i8 3 ' + struct.pack('<3q', 16, 16, 16).hex().upper()
  assert lines[2] == 'Name |S1 2 ' + b'pm'.hex().upper()
  a = fio.read_attrs(fn, '0/Position')
  assert a['Name'] == 'pm'
  assert_array_equal(fio.read_block(fn, '0/Position'), data)


def test_corrupt_and_truncated_files(fio, tmp_path):
  """A flipped byte fails the checksum; a truncated data file fails the
  size check; both raise instead of returning wrong particles."""
  data = np.linspace(0, 1, 30, dtype=np.float32).reshape(10, 3)
  fn = str(tmp_path / 'c')
  fio.write_block(fn, 'b', data)
  path = os.path.join(fn, 'b', '000000')
  raw = bytearray(open(path, 'rb').read())
  raw[7] ^= 0x10
  open(path, 'wb').write(bytes(raw))
  with pytest.raises(ValueError, match='checksum'):
    fio.read_block(fn, 'b')
  fio.read_block(fn, 'b', verify=False)  # sizes still agree
  open(path, 'wb').write(bytes(raw[:-4]))
  with pytest.raises(ValueError, match='bytes'):
    fio.read_block(fn, 'b')


def test_attrs_best_effort_and_vectors(fio, cosmo, tmp_path):
  state = _state(batch=1, npart=8)
  fn = str(tmp_path / 'a')
  fio.save_state(cosmo, state, 0.5, NC, BOX, fn,
                 attrs={'Seed': 7, 'Note': 'run', 'Bad': object(),
                        'Stages': np.linspace(0.1, 1.0, 4)})
  h = fio.read_attrs(fn, 'Header')
  assert 'Bad' not in h
  assert h['Note'] == 'run' and h['Seed'][0] == 7
  assert_allclose(h['Stages'], np.linspace(0.1, 1.0, 4))
  with pytest.raises(ValueError):
    fio.save_state(cosmo, state[0], 0.5, NC, BOX, str(tmp_path / 'bad'))


def test_load_state_resumes(fio, cosmo, tmp_path):
  """load_state returns X and P within one float32 rounding of the saved
  state, F = 0 and the snapshot's scale factor."""
  state = _state(seed=3)
  fn = str(tmp_path / 'r')
  fio.save_state(cosmo, state, 0.37, NC, BOX, fn)
  back, a, header = fio.load_state(fn, device='cpu')
  assert a == pytest.approx(0.37)
  assert tuple(back.shape) == state.shape
  b = back.numpy()
  assert_allclose(b[:2], state[:2], rtol=3e-7, atol=1e-6)
  assert not b[2].any()
  assert_allclose(header['BoxSize'], BOX)


@pytest.mark.gpu
def test_save_state_gpu_lpt(cuda, tmp_path):
  """The reference's test flow: a batch-2 linear field, LPT at a0 = 0.1,
  save_state, read back, on device tensors."""
  import flowpm_b200 as fpm
  from flowpm_b200 import io
  from conftest import pk_table
  c = fpm.cosmology.Planck15()
  lin = fpm.linear_field(NC, BOX, pk_table(), batch_size=2, seed=5)
  state = fpm.lpt_init(c, lin, 0.1)
  fn = str(tmp_path / 'testsave')
  io.save_state(c, state, 0.1, NC, BOX, fn)
  s = state.cpu().numpy()
  assert_array_equal(io.read_block(fn, '1/Position'), s[0, 1] * _cell())
  assert_allclose(io.read_block(fn, '1/Velocity'),
                  s[1, 1] / NC[0] * BOX[0], rtol=1e-6)
  back, a, _ = io.load_state(fn)
  assert back.is_cuda and a == pytest.approx(0.1)
  assert_allclose(back[:2].cpu().numpy(), s[:2], rtol=3e-7, atol=1e-5)


def test_read_block_of_several_files(fio, tmp_path):
  """A block split over two data files (NFILE 2, as a parallel writer
  makes them) reads back as one array in file order."""
  a = np.arange(12, dtype='<f8').reshape(4, 3)
  b = -np.arange(6, dtype='<f8').reshape(2, 3)
  path = tmp_path / 'm' / 'blk'
  os.makedirs(path)
  lines = ['DTYPE: <f8', 'NMEMB: 3', 'NFILE: 2']
  for i, part in enumerate((a, b)):
    raw = part.tobytes()
    (path / ('%06X' % i)).write_bytes(raw)
    s = int(np.frombuffer(raw, np.uint8).sum()) % 2**32
    r = (s & 0xffff) + (s >> 16)
    lines.append('%06X: %d : %d : %d' % (i, part.shape[0], s,
                                         (r & 0xffff) + (r >> 16)))
  (path / 'header').write_text('\n'.join(lines) + '\n')
  assert_array_equal(fio.read_block(str(tmp_path / 'm'), 'blk'),
                     np.concatenate([a, b]))
