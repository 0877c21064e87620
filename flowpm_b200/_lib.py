"""ctypes binding of ``libflowpm_b200.so`` (declared in include/flowpm_b200.h).

The library is the only compute path of this package: importing it fails
loudly when the shared object is missing, and every call checks its return
code.  There is no CPU or PyTorch fallback.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libflowpm_b200.so')

c_int, c_int64, c_uint64 = ctypes.c_int, ctypes.c_int64, ctypes.c_uint64
c_double, c_float, c_void_p = ctypes.c_double, ctypes.c_float, ctypes.c_void_p
c_uint, c_char_p = ctypes.c_uint, ctypes.c_char_p
P_int32 = ctypes.POINTER(ctypes.c_int32)
P_int64 = ctypes.POINTER(ctypes.c_int64)
P_double = ctypes.POINTER(ctypes.c_double)

# Exported symbols with their argument types (mirrors include/flowpm_b200.h).
SIGNATURES = {
    'fpm_version': (c_int, []),
    'fpm_error_string': (c_char_p, [c_int]),
    'fpm_launch_count': (c_int64, []),
    'fpm_plan_profile': (c_int, [c_void_p, c_int]),
    'fpm_plan_profile_read': (c_int, [c_void_p, c_int, P_double, P_int64]),
    'fpm_cic_paint': (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p,
                              c_int64, c_void_p, c_void_p]),
    'fpm_cic_readout': (c_int, [c_void_p, c_int, c_int, c_int, c_int,
                                c_void_p, c_int64, c_void_p, c_void_p]),
    'fpm_cic_neighbours': (c_int, [c_int, c_int, c_int, c_void_p, c_int64,
                                   c_void_p, c_void_p, c_void_p]),
    'fpm_r2c3d': (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                          c_double, c_int, c_void_p]),
    'fpm_c2r3d': (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                          c_double, c_int, c_void_p]),
    'fpm_plan_create': (c_int, [ctypes.POINTER(c_void_p), c_int, P_int32,
                                c_double, c_uint]),
    'fpm_plan_destroy': (c_int, [c_void_p]),
    'fpm_plan_info': (c_int, [c_void_p, P_int64, P_int64]),
    'fpm_plan_status': (c_int, [c_void_p, P_int32, c_void_p]),
    'fpm_force': (c_int, [c_void_p, c_void_p, P_double, c_void_p, c_void_p]),
    'fpm_nbody': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                          P_int32, P_double, P_double, c_void_p, c_uint,
                          c_void_p]),
    'fpm_nbody_set_steps': (c_int, [c_void_p, c_int, P_int32, P_double,
                                    P_double, c_void_p]),
    'fpm_nbody_set_pgd': (c_int, [c_void_p, c_int, P_double, c_void_p]),
    'fpm_plan_set_binning': (c_int, [c_void_p, c_int, c_int, c_int]),
    'fpm_plan_set_adjoint_binning': (c_int, [c_void_p, c_int]),
    'fpm_plan_autotune': (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int,
                                  P_int32, ctypes.POINTER(c_float),
                                  c_void_p]),
    'fpm_pgd': (c_int, [c_void_p, c_void_p, P_double, c_void_p]),
    'fpm_nbody_run': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p,
                              c_void_p, c_uint, c_void_p, c_int, c_void_p]),
    'fpm_nbody_adjoint': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_int, c_void_p]),
    'fpm_nbody_set_tape': (c_int, [c_void_p, c_void_p, c_int64]),
    'fpm_graph_capture_nbody': (c_int, [c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_uint, c_void_p,
                                        c_int, ctypes.POINTER(c_void_p)]),
    'fpm_graph_capture_adjoint': (c_int, [c_void_p, c_void_p, c_void_p,
                                          c_void_p, c_void_p, c_void_p,
                                          c_void_p, c_void_p, c_int,
                                          ctypes.POINTER(c_void_p)]),
    'fpm_graph_launch': (c_int, [c_void_p, c_void_p]),
    'fpm_graph_destroy': (c_int, [c_void_p]),
    'fpm_lpt_adjoint': (c_int, [c_void_p, c_void_p, P_double, c_int,
                                c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p]),
    'fpm_cic_paint_adjoint': (c_int, [c_void_p, c_int, c_int, c_int, c_int,
                                      c_void_p, c_int64, c_void_p, c_void_p,
                                      c_void_p, c_void_p]),
    'fpm_cic_readout_adjoint': (c_int, [c_void_p, c_int, c_int, c_int, c_int,
                                        c_void_p, c_int64, c_void_p, c_void_p,
                                        c_void_p, c_void_p]),
    'fpm_lpt_init': (c_int, [c_void_p, c_void_p, P_double, c_int, c_void_p,
                             c_void_p, c_void_p, c_void_p]),
    'fpm_lpt1': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p,
                         c_void_p]),
    'fpm_lpt2_source': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    'fpm_linear_field': (c_int, [c_void_p, c_void_p, c_uint64, c_int,
                                 c_void_p, c_void_p, c_void_p]),
    'fpm_lattice_shift': (c_int, [c_void_p, c_void_p, c_int, c_int, c_int,
                                  c_int, c_int, c_void_p]),
    'fpm_saxpy': (c_int, [c_void_p, c_void_p, c_float, c_int64, c_void_p]),
    'fpm_pk_bin': (c_int, [c_void_p, c_int, c_int, c_int, c_int, P_double,
                           c_double, c_double, c_int, c_void_p, c_void_p]),
    'fpm_pk_bin_noalloc': (c_int, [c_void_p, c_int, c_int, c_int, c_int,
                                   P_double, c_double, c_double, c_int,
                                   c_void_p, c_void_p]),
    'fpm_power_spectrum': (c_int, [c_void_p, c_int, c_int, c_int, c_int,
                                   P_double, c_double, c_double, c_int,
                                   c_void_p, c_void_p]),
    'fpm_white_noise': (c_int, [c_void_p, c_int64, c_uint64, c_double,
                                c_void_p]),
    'fpm_cic_paint_2d': (c_int, [c_void_p, c_int, c_int, c_int, c_void_p,
                                 c_int64, c_void_p, c_void_p, c_void_p]),
    'fpm_cic_paint_2d_adjoint': (c_int, [c_void_p, c_int, c_int, c_int,
                                         c_void_p, c_int64, c_void_p,
                                         c_void_p, c_void_p, c_void_p,
                                         c_void_p]),
    'fpm_density_planes': (c_int, [c_void_p, c_int, c_int64, c_int, c_int,
                                   c_int, P_double, P_double, c_int,
                                   P_double, P_double, c_int, c_void_p,
                                   c_void_p]),
    'fpm_density_planes_adjoint': (c_int, [c_void_p, c_int, c_int64, c_int,
                                           c_int, c_int, P_double, P_double,
                                           c_int, P_double, P_double, c_int,
                                           c_void_p, c_void_p, c_void_p]),
}

# Constants of include/flowpm_b200.h.
FPM_OK = 0
FPM_ERR_ARG = 1
FPM_ERR_UNSUPPORTED = 8
FPM_ERR_NONFINITE = 6
FPM_ERR_STATE = 7
FPM_ERR_LIMIT = 9
FPM_ERR_RANGE = 10
FPM_PLAN_CIC_DECONV = 1
FPM_PLAN_LPT = 2
FPM_PLAN_GRAD_ORDER0 = 4
FPM_PLAN_ADJOINT = 8
FPM_PLAN_CUFFT = 16
FPM_PLAN_SMALL_BLOCKS = 32
FPM_NBODY_INTERMEDIATE = 1
FPM_TUNE_CONFIGS = 8
FPM_BIN_TILES = 0
FPM_BIN_CHUNKS = 1
FPM_BIN_WALK = 2
FPM_BIN_FLOW = 3
FPM_STATUS_NONFINITE_POS = 1
FPM_STATUS_NONFINITE_MOM = 2


class FlowPMError(RuntimeError):
  """Error code returned by the CUDA library."""

  def __init__(self, fn, code):
    self.code = code
    msg = lib.fpm_error_string(code).decode() if lib is not None else '?'
    super(FlowPMError, self).__init__('%s failed: %s (code %d)' %
                                      (fn, msg, code))


def load(path=LIB_PATH):
  if not os.path.exists(path):
    raise ImportError(
        'flowpm_b200: the CUDA library %s is missing; build it with '
        '`python flowpm_b200/_build.py` (nvcc, sm_100a). There is no CPU '
        'fallback.' % path)
  handle = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
  for name, (res, args) in SIGNATURES.items():
    fn = getattr(handle, name)
    fn.restype = res
    fn.argtypes = args
  return handle


lib = load()


def check(fn, code):
  if code != FPM_OK:
    raise FlowPMError(fn, code)


def call(name, *args):
  check(name, getattr(lib, name)(*args))


def stream_ptr(device=None):
  return c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(t):
  return None if t is None else c_void_p(t.data_ptr())


def dvec(values):
  arr = (ctypes.c_double * len(values))(*[float(v) for v in values])
  return arr


def ivec(values):
  return (ctypes.c_int32 * len(values))(*[int(v) for v in values])
