"""Build of ``libflowpm_b200.so`` (the C-ABI CUDA library) for sm_100a.

``python flowpm_b200/_build.py`` compiles ``csrc/*.cu`` with nvcc into
``flowpm_b200/libflowpm_b200.so`` in the source tree, so the library travels
with the package.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libflowpm_b200.so')
SOURCES = ['fpm_cic.cu', 'fpm_kernels.cu', 'fpm_adjoint.cu', 'fpm_pk.cu',
           'fpm_fft.cu', 'fpm_planes.cu', 'fpm_bin.cu',
           'fpm_plan.cu']
CUDA_HOME = os.environ.get('CUDA_HOME', '/usr/local/cuda')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc_command(out=LIB, extra=()):
  nvcc = os.path.join(CUDA_HOME, 'bin', 'nvcc')
  cmd = [nvcc, '-O3', '-std=c++17', '-lineinfo'] + ARCH + [
      '-Xcompiler', '-fPIC', '-shared', '-o', out
  ] + [os.path.join(CSRC, s) for s in SOURCES] + [
      '-L' + os.path.join(CUDA_HOME, 'lib64'), '-lcufft', '-Xlinker',
      '-rpath,' + os.path.join(CUDA_HOME, 'lib64')
  ] + list(extra)
  return cmd


def needs_build():
  if not os.path.exists(LIB):
    return True
  t = os.path.getmtime(LIB)
  deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
  deps.append(os.path.join(HERE, '..', 'include', 'flowpm_b200.h'))
  return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
  if not force and not needs_build():
    return LIB
  cmd = nvcc_command()
  if verbose:
    print(' '.join(cmd))
  tmp = LIB + '.tmp'
  cmd[cmd.index(LIB)] = tmp
  subprocess.run(cmd, check=True)
  os.replace(tmp, LIB)
  return LIB


if __name__ == '__main__':
  build(force='--force' in sys.argv, verbose=True)
