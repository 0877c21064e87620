"""Throughput benchmark of the FlowPM particle-mesh step on B200.

Workload (one "step" = one full forward simulation through the library):
128^3 particles on a 128^3 mesh, box 200 Mpc/h, Planck15, 2LPT initial
conditions at a0 = 0.1 from a seeded Eisenstein-Hu Gaussian field, then 40
kick-drift-kick steps to a = 1 (41 force evaluations); FP32 displacement
state, FP64 background.  Metric: particle-updates/s = particles x leapfrog
steps / device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Beside the headline line's main figures, a single-GPU run also reports
C4 (128^3 forward + adjoint), C3 (a batch of uneven simulations against
one plan per simulation) and C5 (two 512^3 simulations, 30 steps, forward
+ reverse-time adjoint, with a per-kernel roofline table); --no-extras
skips them, --no-c5 skips C5.

Under torchrun every rank advances its own replica (different seed), the
timed region is bracketed by barriers and the max device time over ranks is
used.  ``--impl reference`` times the CPU restatement of the reference's
algorithm (torch on the host cores) on a bounded sample of the same
workload instead.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_MESH = 128
BOX = 200.0
A0 = 0.1
N_STEPS = 40
METRIC = 'particle-updates/s'
WORKLOAD = ('C2: forward PM, 128^3 particles / 128^3 mesh, box 200 Mpc/h, '
            'Planck15, 2LPT at a0=0.1, 40 KDK steps to a=1')
# Algorithmic HBM bytes (FP32, Np = Nc): per leapfrog step of the whole
# pass 60 Np + 64 Nc = 124 B per particle-update; per launch of the fused
# step kernel: read d, p (24 Np) + write d, p (24 Np) + gather the three
# force meshes (12 Nc) + paint the density (4 Nc) = 64 B per particle.
STEP_BYTES_PER_PART = 124
KERNEL_BYTES_PER_PART = 64
# DRAM bytes (read + write) of one step-kernel launch at 128^3, from one
# ncu capture each (dram__bytes_read.sum + dram__bytes_write.sum), by
# traversal: the lattice walk's k_step 84.1 + 8.3 MB; k_step_sorted (keys
# in tiles of 16 cells, equal chunks) 92.4 + 11.7 MB.
KSTEP_TRAFFIC_BYTES_128 = {'walk': 92.4e6, (16, 1): 104.1e6}
L2_FLUSH_BYTES = 256 << 20
# sort periods (in positions) of the reverse sweep over the binned particle
# order that C4 and C5 time beside the lattice walk's, and the cell tile of
# the keys when the forward keeps the lattice walk
ADJ_SORT_PERIODS = (4, 8, 1 << 20)  # 1 << 20: sorted once, at the start
ADJ_TILE = 16
# seed of replica r's linear field: replicas.replica_seed(1000, r)
REPLICA_SEED_BASE = 1000
# Accuracy of the C4 gradient at full size (128^3, 20 steps, checkpoints
# every 5), from the offline check against the FP64 oracle:
#   python tests/c4_gradient_check.py export C4.npz        (GPU)
#   python tests/c4_gradient_check.py check C4.npz R.json  (8 host cores,
#       32 random unit directions, FP64 central differences at three steps)
# Relative errors per direction, median and max over the 32; the largest
# comes from the direction whose projection is smallest (0.043 against a
# median of 1.30), where the oracle's FP32 tape (the reference's own
# arithmetic) is as far from FP64.
GRAD_CHECK_C4 = {
    'directions': 32,
    'fp64_tape_rel_l2': {'rebuilt': 8.52e-4, 'tape': 8.69e-4,
                         'oracle_fp32_tape': 1.30e-3},
    'vs_fp64_tape': {'rebuilt': {'median': 7.50e-4, 'max': 5.85e-2},
                     'tape': {'median': 6.42e-4, 'max': 5.35e-2},
                     'oracle_fp32_tape': {'median': 1.28e-3,
                                          'max': 5.18e-2}},
    'fd64_vs_fp64_tape': {'eps_1e-3': {'median': 5.94e-5, 'max': 2.21e-3},
                          'eps_1e-4': {'median': 4.24e-6, 'max': 2.79e-4},
                          'eps_1e-5': {'median': 3.19e-6, 'max': 8.54e-5}},
    'gpu_vs_fd64_eps_1e-4': {'rebuilt': {'median': 7.49e-4, 'max': 5.82e-2},
                             'tape': {'median': 6.40e-4, 'max': 5.33e-2}},
    'loss': {'gpu_fp32': 2097898.25, 'fp64': 2097898.2496},
    'eps': 'relative to the linear field standard deviation',
}
# Error of a simulation at the C5 spacing against the oracle, from
# python tests/c5_fp64_check.py (256^3, box 500 Mpc/h, Planck15, seed 5120,
# 30 steps; the oracle cannot run 512^3 in reasonable time on the host).
FP64_CHECK_C5 = {
    'workload': 'one C5 simulation at 256^3, box 500 Mpc/h (C5 spacing), '
                'Planck15, seed 5120, 2LPT at a0 = 0.1, 30 KDK steps',
    'how': 'python tests/c5_fp64_check.py (GPU run, oracle on 16 host '
           'cores: 219 s FP32, 326 s FP64)',
    'vs_oracle_fp32': {'density_rel_l2': 1.07e-05, 'pk_max_rel': 1.53e-06},
    'fp64_error': {'density_rel_l2': 5.62e-06, 'pk_max_rel': 1.69e-06,
                   'oracle_fp32_density_rel_l2': 1.11e-05,
                   'oracle_fp32_pk_max_rel': 1.06e-06},
}


def parse():
  ap = argparse.ArgumentParser()
  ap.add_argument('--gpus', type=int, default=1)
  ap.add_argument('--steps', type=int, default=10)
  ap.add_argument('--warmup', type=int, default=3)
  ap.add_argument('--impl', default='flowpm_b200',
                  choices=['flowpm_b200', 'reference'])
  ap.add_argument('--no-cpu-baseline', action='store_true')
  ap.add_argument('--no-autotune', action='store_true',
                  help='keep the lattice walk instead of the autotuned '
                  'traversal')
  ap.add_argument('--binning', default=None,
                  help='TILE,SORT_EVERY: this traversal instead of the '
                  'autotuned one (0,1: the lattice walk)')
  ap.add_argument('--c5', action='store_true',
                  help='measure the 2 x 512^3 forward + adjoint config even '
                  'with --no-extras (it runs by default otherwise)')
  ap.add_argument('--no-c5', action='store_true',
                  help='skip the 2 x 512^3 forward + adjoint config')
  ap.add_argument('--no-potential-tape', action='store_true',
                  help='C4 / C5: rebuild the force meshes of the reverse '
                  'sweep (paint + Fourier solve) instead of keeping the '
                  "forward's potentials (fpm_nbody_set_tape)")
  ap.add_argument('--c5-mesh', type=int, default=512,
                  help='mesh per side of the --c5 measurement, box scaled '
                  'to keep its spacing; for profiling other sizes (C5 is '
                  '512)')
  ap.add_argument('--no-extras', action='store_true',
                  help='skip the C4 (forward + adjoint) and C3 (batched) '
                  'measurements')
  ap.add_argument('--mesh', type=int, default=N_MESH,
                  help='mesh (= particle lattice) per side of the forward '
                  'workload, box scaled to keep the C2 spacing; for '
                  'profiling other sizes (C2 is 128)')
  return ap.parse_args()


def dist_env():
  rank = int(os.environ.get('RANK', 0))
  world = int(os.environ.get('WORLD_SIZE', 1))
  local = int(os.environ.get('LOCAL_RANK', 0))
  return rank, world, local


def pk_fn():
  from flowpm_b200 import cosmology, tfpower
  cosmo = cosmology.Planck15()
  kk = np.logspace(-4, 2, 4096)
  pk = tfpower.linear_matter_power(cosmo, kk)
  return lambda k: np.interp(np.log(np.maximum(k, 1e-30)), np.log(kk), pk,
                             left=0.0)


class ClockSampler(object):
  """nvidia-smi clock / throttle samples during the timed region."""
  Q = ('index,clocks.sm,clocks.max.sm,power.draw,'
       'clocks_event_reasons.hw_slowdown,'
       'clocks_event_reasons.hw_thermal_slowdown,'
       'clocks_event_reasons.sw_thermal_slowdown,'
       'clocks_event_reasons.sw_power_cap')

  def __init__(self, index):
    self.index = index
    self.proc = None

  def __enter__(self):
    try:
      self.proc = subprocess.Popen(
          ['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.Q,
           '--format=csv,noheader,nounits', '-lms', '200'],
          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
      self.proc = None
    time.sleep(0.3)
    return self

  def __exit__(self, *exc):
    self.lines = []
    if self.proc is not None:
      time.sleep(0.3)
      self.proc.terminate()
      out, _ = self.proc.communicate(timeout=10)
      self.lines = [l for l in out.splitlines() if l.strip()]
    return False

  def summary(self):
    sm, mx, reasons = [], None, set()
    names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
             'sw_power_cap']
    for l in self.lines:
      f = [x.strip() for x in l.split(',')]
      if len(f) < 8:
        continue
      try:
        sm.append(float(f[1]))
        mx = float(f[2])
      except ValueError:
        continue
      for n, v in zip(names, f[4:8]):
        if v.lower().startswith('active'):
          reasons.add(n)
    return {
        'sm_mhz': float(np.median(sm)) if sm else None,
        'sm_max_mhz': mx,
        'reasons': sorted(reasons),
        'samples': len(sm)
    }


def peaks():
  path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
  try:
    with open(path) as f:
      return float(json.load(f)['hbm_gbs']), 'measured'
  except (OSError, KeyError, ValueError):
    return 6650.0, 'fallback'


def workload_config(world=1):
  """The `config` of both arms' lines: the C2 workload."""
  return {
      'workload': WORKLOAD,
      'mesh': N_MESH,
      'particles': N_MESH**3,
      'box': BOX,
      'leapfrog_steps_per_step': N_STEPS,
      'background': 'f64',
      'initial_field': 'seeded Eisenstein-Hu Gaussian field (Philox noise, '
                       'seed %d)' % REPLICA_SEED_BASE,
      'parallelism': 'replicas x%d' % world,
      'l2': 'flushed (256 MB write) before every timed step',
  }


def oracle_linear_field(seed):
  """The GPU arm's seeded linear field, computed on the host by the oracle:
  the library's Philox noise restated (oracle/rng.py), the EH P(k) and
  flowpm/tfpm.py:15-63 linear_field."""
  from oracle import background as obg
  from oracle import pm as opm
  from oracle import power as opw
  from oracle import rng as orng
  n = N_MESH
  white = orng.white_noise(n**3, seed, stddev=float(n**3)**0.5)
  b = obg.Background({}, dtype=np.float64)
  kk = np.logspace(-4, 2, 4096)
  pk = opw.linear_matter_power(b, kk)
  pkf = lambda k: np.interp(np.log(np.maximum(k, 1e-30)), np.log(kk), pk,
                            left=0.0)
  return opm.linear_field_from_white(
      torch.tensor(white.reshape(1, n, n, n)), BOX, pkf)


def oracle_run(lin, dtype):
  """Oracle 2LPT + the 40-step leapfrog of the workload in float32 (the
  reference's arithmetic) or float64, on all host cores.  Returns the final
  density and the seconds the leapfrog took (initial force included)."""
  from oracle import background as obg
  from oracle import pm as opm
  torch.set_num_threads(os.cpu_count() or 1)
  b = obg.Background({}, dtype=np.float32 if dtype == torch.float32
                     else np.float64)
  s0 = opm.lpt_init(b, torch.as_tensor(lin).to(dtype), A0, order=2)
  stages = np.linspace(A0, 1.0, N_STEPS + 1)
  t0 = time.perf_counter()
  st = opm.nbody(b, s0, stages, N_MESH)
  dt = time.perf_counter() - t0
  n = N_MESH
  rho = opm.cic_paint(torch.zeros((1, n, n, n), dtype=dtype), st[0])
  return rho.numpy(), dt


def parity_and_cpu_baseline(lin, rho_gpu):
  """The GPU arm's final density against the oracle run from the same
  linear field, in float32 and float64, and the float32 oracle's leapfrog
  timed as the CPU baseline (the whole 40-step workload)."""
  from oracle import pm as opm
  rho32, dt32 = oracle_run(lin, torch.float32)
  rho64, _ = oracle_run(lin, torch.float64)

  def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))

  def pk(rho):
    _, p = opm.power_spectrum(torch.tensor(rho, dtype=torch.float64),
                              kmin=0.02, dk=0.02,
                              boxsize=np.array([BOX] * 3))
    return p.numpy().ravel()

  p, p32, p64 = pk(rho_gpu), pk(rho32), pk(rho64)
  ok = np.isfinite(p64) & (p64 != 0) & np.isfinite(p32) & (p32 != 0)
  prel = lambda a, b: float(np.max(np.abs(a[ok] - b[ok]) / np.abs(b[ok])))
  parity = {
      'workload': 'the timed simulation (rank 0), final CIC density',
      'vs_oracle_fp32': {'density_rel_l2': rel(rho_gpu, rho32),
                         'pk_max_rel': prel(p, p32),
                         'bar': 1e-4},
      'fp64_error': {'density_rel_l2': rel(rho_gpu, rho64),
                     'pk_max_rel': prel(p, p64),
                     'oracle_fp32_density_rel_l2': rel(rho32, rho64),
                     'oracle_fp32_pk_max_rel': prel(p32, p64)},
      'pk_bins': 'kmin 0.02, dk 0.02 h/Mpc',
  }
  cpu = {
      'value': N_MESH**3 * N_STEPS / dt32,
      'unit': METRIC,
      'cores': torch.get_num_threads(),
      'kind': 'port',
      'sample': 'the whole workload: the 40-step leapfrog (41 forces) of the '
                '128^3 simulation from the same seeded linear field, '
                'torch-CPU restatement of flowpm/tfpm.py, FP32, %.1f s' % dt32
  }
  return parity, cpu


def run_reference(args, rank, world):
  """CPU arm: the oracle port of the reference on the host cores.  One bench
  step = one leapfrog step (kick, drift, force, kick) of the workload,
  steps taken in order from the 2LPT state of the GPU arm's seeded linear
  field; the 40 steps of the workload repeat if K + W exceeds them."""
  if rank != 0:
    return
  from oracle import background as obg
  from oracle import pm as opm
  torch.set_num_threads(os.cpu_count() or 1)
  # replicas.replica_seed(REPLICA_SEED_BASE, 0), without loading the library
  lin = oracle_linear_field(REPLICA_SEED_BASE * 1000003)
  b = obg.Background({}, dtype=np.float32)
  s0 = opm.lpt_init(b, lin.to(torch.float32), A0, order=2)
  stages = np.linspace(A0, 1.0, N_STEPS + 1)
  # the initial force is computed once, untimed
  state = opm.force(b, s0, N_MESH)
  times = []
  for i in range(args.warmup + args.steps):
    if i % N_STEPS == 0 and i > 0:
      state = opm.force(b, s0, N_MESH)
    a0, a1 = stages[i % N_STEPS], stages[i % N_STEPS + 1]
    ah = (a0 * a1)**0.5
    t0 = time.perf_counter()
    st = opm.kick(b, state, a0, a0, ah)
    st = opm.drift(b, st, a0, ah, a1)
    st = opm.force(b, st, N_MESH)
    state = opm.kick(b, st, ah, a1, a1)
    dt = time.perf_counter() - t0
    if i >= args.warmup:
      times.append(dt)
  t = float(np.sum(times))
  v = N_MESH**3 * len(times) / t
  line = {
      'impl': 'reference',
      'metric': METRIC,
      'value': v,
      'unit': METRIC,
      'n_gpus': world,
      'steps': args.steps,
      'warmup': args.warmup,
      'ms_per_step': 1e3 * t / len(times),
      'higher_is_better': True,
      'scaling': 'weak',
      'vs_baseline': None,
      'dtype': 'f32',
      'data': 'synthetic',
      'config': workload_config(world),
      'cpu_baseline': {
          'value': v, 'unit': METRIC, 'cores': torch.get_num_threads(),
          'kind': 'port',
          'sample': 'leapfrog steps %d-%d of the 40 of the workload (one per '
                    'bench step, after %d warm-up steps), from the 2LPT state '
                    'of the same seeded linear field, torch-CPU restatement '
                    'of flowpm/tfpm.py (FP32)' % (
                        args.warmup % N_STEPS,
                        (args.warmup + len(times) - 1) % N_STEPS,
                        args.warmup)},
      'e2e': {'value': v, 'unit': METRIC, 'h2d_bytes_per_step': 0,
              'd2h_bytes_per_step': 0},
  }
  print(json.dumps(line))


def _pk_interp(cosmo):
  from flowpm_b200 import tfpower
  kk = np.logspace(-4, 2, 4096)
  pk = tfpower.linear_matter_power(cosmo, kk)
  return lambda k: np.interp(np.log(np.maximum(k, 1e-30)), np.log(kk), pk,
                             left=0.0)


def _timed(fn, reps, flush):
  """Device time (ms) of fn() per call, L2 flushed before every call."""
  ts = []
  for _ in range(reps):
    flush.fill_(1.0)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize()
    ts.append(e0.elapsed_time(e1))
  return float(np.median(ts))


def _sorted_name(k):
  """Method name of the reverse sweep in the binned order, re-sorted every
  k positions."""
  return 'potential_tape_sorted' + ('_once' if k >= 1 << 20 else str(k))


def measure_fwd_adjoint(fpm, flush, reps, n=128, steps=20, ckpt=5):
  """Config C4: 128^3, 20 steps, chi^2 of the final CIC density against
  (that density + N(0, 1) noise); gradient with respect to the initial
  linear field.  Timed step = forward leapfrog (graph, checkpoints every
  `ckpt`) + loss gradient + reverse-time adjoint (graph), for both methods
  of the reverse sweep: rebuilding the trajectory from the final state
  (paint + Fourier solve at every reconstructed position), and taking the
  force potentials the forward stored (the potential tape).  The gradient's
  accuracy at this size is measured offline against the FP64 oracle
  (tests/c4_gradient_check.py; GRAD_CHECK_C4 holds its result)."""
  from flowpm_b200 import _lib, tfbackground
  from flowpm_b200._plans import get_plan
  cosmo = fpm.cosmology.Planck15()
  nc = [n] * 3
  np_ = n**3
  st = _lib.stream_ptr()
  lin = fpm.linear_field(nc, BOX, _pk_interp(cosmo), seed=4242)
  stages = np.linspace(A0, 1.0, steps + 1)
  plan = get_plan([tuple(nc) + (1,)], flags=_lib.FPM_PLAN_ADJOINT)
  coefs = tfbackground.nbody_coefficients(cosmo, stages)
  _lib.call('fpm_nbody_set_steps', plan.handle, steps, _lib.ivec([steps]),
            _lib.dvec(coefs.ravel()), _lib.dvec([1.5 * cosmo.Omega_m]), st)
  s0 = fpm.lpt_init(cosmo, lin, A0, order=2)
  d0 = fpm.tfpm._to_disp(s0[0], nc).reshape(-1, 3).contiguous()
  p0 = s0[1].reshape(-1, 3).contiguous().clone()
  d, p, f = torch.empty_like(d0), torch.empty_like(p0), torch.empty_like(d0)
  lx, lp = torch.empty_like(d0), torch.empty_like(d0)
  X = torch.empty_like(d0)
  rho = torch.empty((1,) + tuple(nc), device='cuda')
  g = torch.empty_like(rho)
  nslot = steps // ckpt + 1
  ck = torch.empty((nslot, 2, np_, 3), device='cuda')
  # the forward's potential at every position, for the reverse sweep
  phi_tape = torch.empty((steps + 1) * np_, device='cuda')
  graphs = {}
  choice, _ = plan.autotune(d0, p0, reps=1, retune=True)

  def capture(method):
    if method == 'potential_tape':
      _lib.call('fpm_nbody_set_tape', plan.handle, _lib.ptr(phi_tape),
                phi_tape.numel())
    else:
      _lib.call('fpm_nbody_set_tape', plan.handle, None, 0)
    gf, ga = _lib.ctypes.c_void_p(), _lib.ctypes.c_void_p()
    _lib.call('fpm_graph_capture_nbody', plan.handle, _lib.ptr(d),
              _lib.ptr(p), _lib.ptr(f), None, 0, _lib.ptr(ck), ckpt,
              _lib.ctypes.byref(gf))
    _lib.call('fpm_graph_capture_adjoint', plan.handle, _lib.ptr(d),
              _lib.ptr(p), _lib.ptr(f), _lib.ptr(lx), _lib.ptr(lp), None,
              _lib.ptr(ck), ckpt, _lib.ctypes.byref(ga))
    graphs['f'], graphs['a'] = gf, ga

  def forward():
    d.copy_(d0)
    p.copy_(p0)
    _lib.call('fpm_graph_launch', graphs['f'], st)
    _lib.call('fpm_lattice_shift', _lib.ptr(d), _lib.ptr(X), 1, n, n, n, 1,
              st)
    rho.zero_()
    _lib.call('fpm_cic_paint', _lib.ptr(rho), 1, n, n, n, _lib.ptr(X), np_,
              None, st)

  def step():
    forward()
    # dL/drho = 2 (rho - target); dL/dX by the paint adjoint
    g.copy_(rho)
    _lib.call('fpm_saxpy', _lib.ptr(g), _lib.ptr(target), -1.0, g.numel(), st)
    _lib.call('fpm_cic_paint_adjoint', _lib.ptr(g), 1, n, n, n, _lib.ptr(X),
              np_, None, _lib.ptr(lx), None, st)
    _lib.call('fpm_saxpy', _lib.ptr(lx), _lib.ptr(lx), 1.0, lx.numel(), st)
    lp.zero_()
    _lib.call('fpm_graph_launch', graphs['a'], st)

  upd = float(np_) * steps
  out = {
      'workload': 'C4: 128^3, 20 KDK steps, chi^2(final CIC density, '
                  'density + N(0,1)), reverse-time adjoint, checkpoint every '
                  '%d' % ckpt,
      'unit': 'particle-updates/s (forward + adjoint)',
      'gradient_check': GRAD_CHECK_C4,
      'traversal': list(choice),
  }
  grads = {}
  # the reverse sweep over the binned particle order (re-sorted every k
  # positions) takes its cell tiles from the forward's binning, or, when
  # the forward keeps the lattice walk, from tiles set for it alone
  sorted_k = {_sorted_name(k): k for k in ADJ_SORT_PERIODS}
  methods = ['potential_tape', 'rebuilt'] + list(sorted_k)
  for method in methods:
    if method in sorted_k:
      if not plan.binning[0]:
        plan.set_binning(ADJ_TILE, 1, _lib.FPM_BIN_WALK)
      plan.set_adjoint_binning(sorted_k[method])
    capture('rebuilt' if method == 'rebuilt' else 'potential_tape')
    if method == 'potential_tape':
      forward()
      gen = torch.Generator(device='cuda').manual_seed(77)
      target = rho + torch.randn(rho.shape, generator=gen, device='cuda')
    for _ in range(3):
      step()
    ms = _timed(step, reps, flush)
    ms_fwd = _timed(forward, reps, flush)
    step()
    grads[method] = lx.clone()
    _lib.lib.fpm_graph_destroy(graphs['f'])
    _lib.lib.fpm_graph_destroy(graphs['a'])
    out[method] = {'value': upd / (ms * 1e-3), 'ms_per_step': ms,
                   'forward_ms': ms_fwd,
                   'adjoint_over_forward': (ms - ms_fwd) / ms_fwd}
  _lib.call('fpm_nbody_set_tape', plan.handle, None, 0)
  if sorted_k:
    plan.set_adjoint_binning(0)
  plan.set_binning(0)
  b = grads['rebuilt'].double()
  rel = lambda m: float((grads[m].double() - b).norm() / b.norm())
  tape = ['potential_tape'] + list(sorted_k)
  best = max(tape, key=lambda m: out[m]['value'])
  out['method'] = best
  out['value'] = out[best]['value']
  out['ms_per_step'] = out[best]['ms_per_step']
  out['potential_tape_gb'] = phi_tape.numel() * 4 / 1e9
  out['lam_x_rel_l2_tape_vs_rebuilt'] = rel('potential_tape')
  for name in sorted_k:
    out['lam_x_rel_l2_%s_vs_rebuilt' % name[len('potential_tape_'):]] = rel(
        name)
  return out


def measure_batched(fpm, flush, reps):
  """Config C3: 8 x 32^3 + 8 x 64^3 + 4 x 128^3 simulations, per-sim
  Omega_c ~ U[0.20, 0.35], sigma8 ~ U[0.70, 0.90], 10-20 steps each, in one
  plan and one CUDA graph, against the plain path (one simulation at a time,
  no graph)."""
  from flowpm_b200 import _lib, tfbackground
  from flowpm_b200._plans import Plan, get_plan
  rng = np.random.default_rng(2024)
  spec = [(32, 100.)] * 8 + [(64, 100.)] * 8 + [(128, 200.)] * 4
  sims = []
  for i, (n, box) in enumerate(spec):
    c = fpm.cosmology.Planck15(Omega_c=float(rng.uniform(0.20, 0.35)),
                               sigma8=float(rng.uniform(0.70, 0.90)))
    sims.append((n, box, c, int(rng.integers(10, 21)), 500 + i))
  maxT = max(s[3] for s in sims)
  st = _lib.stream_ptr()
  d0s, p0s, coefs, ffac, nsteps, dims = [], [], [], [], [], []
  for n, box, c, T, seed in sims:
    lin = fpm.linear_field(n, box, _pk_interp(c), seed=seed)
    s0 = fpm.lpt_init(c, lin, A0, order=2)
    d0s.append(fpm.tfpm._to_disp(s0[0], [n] * 3).reshape(-1, 3))
    p0s.append(s0[1].reshape(-1, 3).contiguous())
    co = np.zeros((maxT, 3))
    co[:T] = tfbackground.nbody_coefficients(c, np.linspace(A0, 1.0, T + 1))
    coefs.append(co)
    ffac.append(1.5 * c.Omega_m)
    nsteps.append(T)
    dims.append((n, n, n, 1))
  # batched: one plan, one graph (public batch API)
  runner = fpm.BatchRunner([dict(nc=n, cosmo=c, stages=np.linspace(
      A0, 1.0, T + 1)) for n, box, c, T, seed in sims])
  states = []
  for i, (n, box, c, T, seed) in enumerate(sims):
    s = torch.empty((3, 1, n**3, 3), device='cuda')
    _lib.call('fpm_lattice_shift', _lib.ptr(d0s[i]), _lib.ptr(s[0]), 1, n, n,
              n, 1, st)
    s[1, 0].copy_(p0s[i])
    states.append(s)

  def batched():
    runner.load(states)
    runner.run()

  batched()  # the first run applies the autotuning policy
  choice = runner.plan.binning

  # plain: one simulation at a time through fpm_nbody, no graph
  singles = []
  for i, (n, box, c, T, seed) in enumerate(sims):
    sp = get_plan([(n, n, n, 1)])
    # the batch's traversal, so that the two differ only by batching
    sp.set_binning(*choice)
    singles.append((sp, d0s[i], p0s[i], torch.empty_like(d0s[i]),
                    torch.empty_like(p0s[i]), torch.empty_like(d0s[i]),
                    coefs[i][:T].ravel(), T, ffac[i]))

  def plain(only=None):
    for sp, d0, p0, d, p, f, co, T, ff in singles:
      if only is not None and d0.shape[0] != only:
        continue
      d.copy_(d0)
      p.copy_(p0)
      _lib.call('fpm_nbody', sp.handle, _lib.ptr(d), _lib.ptr(p), _lib.ptr(f),
                T, _lib.ivec([T]), _lib.dvec(co), _lib.dvec([ff]), None, 0, st)

  batched()
  plain()
  torch.cuda.synchronize()
  # same answer both ways
  err = 0.0
  for res, (sp, d0, p0, d, p, f, co, T, ff) in zip(runner.results(),
                                                   singles):
    n = round(d.shape[0]**(1 / 3))
    x = torch.empty_like(d)
    _lib.call('fpm_lattice_shift', _lib.ptr(d), _lib.ptr(x), 1, n, n, n, 1,
              st)
    err = max(err, float((res[0, 0] - x).abs().max()))
  fp64 = c3_fp64_error(sims, d0s, p0s, runner.results())
  tb = _timed(batched, reps, flush)
  tp = _timed(plain, reps, flush)
  # Amdahl bound of the mix: the four 128^3 simulations hold 78 % of the
  # particles and already run at the single-simulation rate unbatched, so
  # even with the small simulations free the batched time is at least
  # their plain time.
  tp128 = _timed(lambda: plain(only=128**3), reps, flush)
  runner.close()
  for sp, *_ in singles:
    sp.set_binning(0)
  nsim = len(sims)
  return {
      'workload': 'C3: 8x32^3 + 8x64^3 + 4x128^3, per-sim cosmology, 10-20 '
                  'steps each',
      'value': nsim / (tb * 1e-3),
      'unit': 'sims/s',
      'plain_sims_per_s': nsim / (tp * 1e-3),
      'speedup_vs_plain': tp / tb,
      'speedup_bound': tp / tp128,
      'speedup_bound_how': 'plain_ms / plain_ms_128: the batched time '
                           'cannot fall below the plain time of the four '
                           '128^3 simulations',
      'batched_ms': tb,
      'plain_ms': tp,
      'plain_ms_128': tp128,
      'particles': int(sum(n**3 for n, *_ in sims)),
      'particle_updates_per_s': float(
          sum(n**3 * T for n, _, _, T, _ in sims)) / (tb * 1e-3),
      'max_abs_diff_batched_vs_plain': err,
      'fp64_error': fp64,
      'traversal': list(choice),
  }


def c3_fp64_error(sims, d0s, p0s, results):
  """Final-density error of the batched results against the oracle in
  float64 (and float32, the reference's arithmetic) run from the same
  initial states with each simulation's own cosmology and step count, for
  the first 32^3 and the first 64^3 simulation of the mix (the 128^3 size
  is C2's, whose error the headline line's `parity` states)."""
  from oracle import background as obg
  from oracle import pm as opm
  torch.set_num_threads(os.cpu_count() or 1)
  out = {}
  for size in (32, 64):
    i = next(k for k, s in enumerate(sims) if s[0] == size)
    n, box, c, T, seed = sims[i]
    q = torch.stack(torch.meshgrid(*[torch.arange(n, dtype=torch.float64)] *
                                   3, indexing='ij'), -1).reshape(-1, 3)
    d0, p0 = d0s[i].double().cpu(), p0s[i].double().cpu()
    x_gpu = results[i][0].double().cpu()  # (1, Np, 3) final positions
    params = dict(Omega_c=c.Omega_c, sigma8=c.sigma8)
    stages = np.linspace(A0, 1.0, T + 1)
    rhos = {}
    for name, dt, npdt in (('fp64', torch.float64, np.float64),
                           ('fp32', torch.float32, np.float32)):
      b = obg.Background(params, dtype=npdt)
      st = torch.stack([q + d0, p0, torch.zeros_like(d0)])[:, None].to(dt)
      st = opm.nbody(b, st, stages, n)
      rhos[name] = opm.cic_paint(torch.zeros((1, n, n, n), dtype=dt),
                                 st[0]).double()
    rg = opm.cic_paint(torch.zeros((1, n, n, n), dtype=torch.float64),
                       x_gpu)
    rel = lambda a, b: float((a - b).norm() / b.norm())
    out['%d^3' % n] = {'steps': T, 'density_rel_l2': rel(rg, rhos['fp64']),
                       'oracle_fp32_density_rel_l2': rel(rhos['fp32'],
                                                         rhos['fp64']),
                       'vs_oracle_fp32': rel(rg, rhos['fp32'])}
  return out


def measure_large(fpm, flush, reps=2, n=512, steps=30, ckpt=5, tape=True):
  """Config C5: two 512^3 simulations (different seeds and cosmologies),
  box 1000 Mpc/h, 30 steps, forward + reverse-time adjoint with a
  checkpoint every 5 steps, in one plan.  Reports forward and
  forward+adjoint particle-updates/s, the per-kernel device time of the
  forward (event pairs around every launch) and the HBM roofline fraction
  of the paint, step (readout + kick + drift + paint) and Fourier kernels."""
  from flowpm_b200 import _lib, tfbackground
  from flowpm_b200._plans import Plan, clear_plans
  box = 1000.0 * n / 512
  cosmos = [fpm.cosmology.Planck15(),
            fpm.cosmology.Planck15(Omega_c=0.27, sigma8=0.78)]
  seeds = [5120, 5121]
  nc = [n] * 3
  np_ = n**3
  st = _lib.stream_ptr()
  d0s, p0s = [], []
  for c, seed in zip(cosmos, seeds):
    lin = fpm.linear_field(nc, box, _pk_interp(c), seed=seed)
    s0 = fpm.lpt_init(c, lin, A0, order=2)
    d0s.append(fpm.tfpm._to_disp(s0[0], nc).reshape(-1, 3))
    p0s.append(s0[1].reshape(-1, 3).clone())
    del lin, s0
  clear_plans()
  torch.cuda.empty_cache()
  D0, P0 = torch.cat(d0s), torch.cat(p0s)
  del d0s, p0s
  stages = np.linspace(A0, 1.0, steps + 1)
  plan = Plan([tuple(nc) + (1,)] * 2, flags=_lib.FPM_PLAN_ADJOINT)
  coefs = np.concatenate(
      [tfbackground.nbody_coefficients(c, stages) for c in cosmos])
  ffac = [1.5 * c.Omega_m for c in cosmos]
  _lib.call('fpm_nbody_set_steps', plan.handle, steps, _lib.ivec([steps] * 2),
            _lib.dvec(coefs.ravel()), _lib.dvec(ffac), st)
  D, P, F = torch.empty_like(D0), torch.empty_like(P0), torch.empty_like(D0)
  LX, LP = torch.empty_like(D0), torch.empty_like(D0)
  X = torch.empty_like(D0)
  ck = torch.empty((steps // ckpt + 1, 2) + tuple(D0.shape), device='cuda')
  rho = torch.empty((2,) + tuple(nc), device='cuda')
  g = torch.empty_like(rho)
  # the forward's potential at every position, for the reverse sweep
  phi_tape = (torch.empty((steps + 1) * 2 * np_, device='cuda') if tape
              else None)
  if tape:
    _lib.call('fpm_nbody_set_tape', plan.handle, _lib.ptr(phi_tape),
              phi_tape.numel())
  choice, tune_ms = plan.autotune(D0, P0, reps=1, retune=True)
  gf, ga = _lib.ctypes.c_void_p(), _lib.ctypes.c_void_p()
  _lib.call('fpm_graph_capture_nbody', plan.handle, _lib.ptr(D), _lib.ptr(P),
            _lib.ptr(F), None, 0, _lib.ptr(ck), ckpt, _lib.ctypes.byref(gf))
  _lib.call('fpm_graph_capture_adjoint', plan.handle, _lib.ptr(D),
            _lib.ptr(P), _lib.ptr(F), _lib.ptr(LX), _lib.ptr(LP), None,
            _lib.ptr(ck), ckpt, _lib.ctypes.byref(ga))

  def forward():
    D.copy_(D0)
    P.copy_(P0)
    _lib.call('fpm_graph_launch', gf, st)

  def density():
    _lib.call('fpm_lattice_shift', _lib.ptr(D), _lib.ptr(X), 2, n, n, n, 1,
              st)
    rho.zero_()
    _lib.call('fpm_cic_paint', _lib.ptr(rho), 2, n, n, n, _lib.ptr(X), np_,
              None, st)

  forward()
  density()
  gen = torch.Generator(device='cuda').manual_seed(99)
  target = rho + torch.randn(rho.shape, generator=gen, device='cuda')
  status = plan.status(st)

  def fwd_seed():  # forward, chi^2 and its cotangents at the final state
    forward()
    density()
    g.copy_(rho)
    _lib.call('fpm_saxpy', _lib.ptr(g), _lib.ptr(target), -1.0, g.numel(), st)
    _lib.call('fpm_cic_paint_adjoint', _lib.ptr(g), 2, n, n, n, _lib.ptr(X),
              np_, None, _lib.ptr(LX), None, st)
    _lib.call('fpm_saxpy', _lib.ptr(LX), _lib.ptr(LX), 1.0, LX.numel(), st)
    LP.zero_()

  def fwd_adj():
    fwd_seed()
    _lib.call('fpm_graph_launch', ga, st)

  fwd_adj()
  t_fwd = _timed(forward, reps, flush)
  t_all = _timed(fwd_adj, reps, flush)
  status |= plan.status(st)
  # per-kernel device time of one forward run, GPU kept busy while enqueued
  _lib.call('fpm_plan_profile', plan.handle, 1)
  D.copy_(D0)
  P.copy_(P0)
  torch.cuda._sleep(100_000_000)
  _lib.call('fpm_nbody_run', plan.handle, _lib.ptr(D), _lib.ptr(P),
            _lib.ptr(F), None, 0, None, 0, st)
  torch.cuda.synchronize()
  kt = {}

  def read_kinds(kinds):
    for kind, name in kinds:
      tot, cnt = _lib.c_double(), _lib.c_int64()
      _lib.call('fpm_plan_profile_read', plan.handle, kind,
                _lib.ctypes.byref(tot), _lib.ctypes.byref(cnt))
      if cnt.value:
        kt[name] = (tot.value / cnt.value, cnt.value)

  read_kinds([(0, 'step'), (1, 'fourier'), (2, 'paint'), (3, 'green'),
              (4, 'stencil')])
  # and of one reverse sweep (from the checkpointed forward run)
  _lib.call('fpm_plan_profile', plan.handle, 0)
  fwd_seed()
  _lib.call('fpm_plan_profile', plan.handle, 1)
  torch.cuda._sleep(100_000_000)
  _lib.call('fpm_nbody_adjoint', plan.handle, _lib.ptr(D), _lib.ptr(P),
            _lib.ptr(F), _lib.ptr(LX), _lib.ptr(LP), None, _lib.ptr(ck), ckpt,
            st)
  torch.cuda.synchronize()
  read_kinds([(5, 'adj_drift_paint'),
              (6, 'adj_drift_vjp' if tape else 'adj_vjp'), (7, 'adj_div'),
              (8, 'adj_potential'), (9, 'adj_position'),
              (1, 'adj_force_solve')])
  _lib.call('fpm_plan_profile', plan.handle, 0)
  # the same reverse sweep over the binned particle order, re-sorted every
  # k positions (needs the forward's binning)
  sorted_adj = None
  if tape:
    sorted_adj = {}
    if not plan.binning[0]:  # tiles for the reverse sweep alone
      plan.set_binning(ADJ_TILE, 1, _lib.FPM_BIN_WALK)
    for k in ADJ_SORT_PERIODS[-1:]:  # the C4 sweep's longest period
      try:
        plan.set_adjoint_binning(k)
      except _lib.FlowPMError as e:  # e.g. its buffers do not fit
        sorted_adj['error'] = str(e)[:200]
        break
      # a changed schedule invalidates both graphs
      _lib.lib.fpm_graph_destroy(gf)
      _lib.lib.fpm_graph_destroy(ga)
      gf, ga = _lib.ctypes.c_void_p(), _lib.ctypes.c_void_p()
      _lib.call('fpm_graph_capture_nbody', plan.handle, _lib.ptr(D),
                _lib.ptr(P), _lib.ptr(F), None, 0, _lib.ptr(ck), ckpt,
                _lib.ctypes.byref(gf))
      _lib.call('fpm_graph_capture_adjoint', plan.handle, _lib.ptr(D),
                _lib.ptr(P), _lib.ptr(F), _lib.ptr(LX), _lib.ptr(LP), None,
                _lib.ptr(ck), ckpt, _lib.ctypes.byref(ga))
      fwd_adj()
      t_k = _timed(fwd_adj, reps, flush)
      status |= plan.status(st)
      fwd_seed()
      _lib.call('fpm_plan_profile', plan.handle, 1)
      torch.cuda._sleep(100_000_000)
      _lib.call('fpm_nbody_adjoint', plan.handle, _lib.ptr(D), _lib.ptr(P),
                _lib.ptr(F), _lib.ptr(LX), _lib.ptr(LP), None, _lib.ptr(ck),
                ckpt, st)
      torch.cuda.synchronize()
      kk = {}
      for kind, name in [(6, 'adj_drift_vjp'), (10, 'sort'),
                         (9, 'adj_position')]:
        tot, cnt = _lib.c_double(), _lib.c_int64()
        _lib.call('fpm_plan_profile_read', plan.handle, kind,
                  _lib.ctypes.byref(tot), _lib.ctypes.byref(cnt))
        if cnt.value:
          kk[name] = {'avg_launch_ms': tot.value / cnt.value,
                      'launches': cnt.value}
      _lib.call('fpm_plan_profile', plan.handle, 0)
      sorted_adj[k] = {'sort_every': k,
                       'value': 2.0 * np_ * steps / (t_k * 1e-3),
                       'forward_adjoint_ms': t_k, 'kernels': kk}
    plan.set_adjoint_binning(0)
  kb, pk = fpm.power_spectrum(rho, kmin=0.01, dk=0.01, boxsize=[box] * 3)
  peak, peak_kind = peaks()
  tot_np, nc_tot = 2 * np_, 2 * np_
  # algorithmic bytes per launch: step 64 B / particle (Np = Nc), paint
  # 12 Np + 4 Nc; the Fourier solve (density -> three force meshes, all of
  # its transforms and kernels) reads and zeroes the density and writes the
  # three force meshes, 20 Nc; its Green's-function kernel reads and writes
  # the half spectrum (8 B per mode each) and zeroes the density, its
  # stencil reads the potential and writes the three force meshes.
  # Reverse sweep, per particle (Np = Nc): the drift + paint kernel reads
  # d, F and reads and writes lam_x, p, lam_p (12 B each way), writes d,
  # gathers the adjoint density and paints (4 B per cell each), 116 B (112 B
  # with the potential tape, which drops the paint); the VJP reads d, lam_p,
  # the three force meshes (12 B per cell), reads and writes lam_x and p,
  # writes F and reduces into the adjoint force mesh (16 B per cell), 112 B;
  # the divergence stencil reads the adjoint force mesh and writes the
  # adjoint potential, 20 B per cell; the adjoint potential solve reads it
  # and writes the adjoint density, 8 B per cell.  With the potential tape,
  # the force meshes of a position are the stencil of the stored potential
  # (20 B per cell, as the forward stencil).
  half = 2 * n * n * (n // 2 + 1)
  kbytes = {
      'step': KERNEL_BYTES_PER_PART * tot_np,
      'paint': 12 * tot_np + 4 * nc_tot,
      'fourier': 20 * nc_tot,
      'green': 16 * half + 4 * nc_tot,
      'stencil': 16 * nc_tot,
      # with the potential tape the reverse drift does not paint
      'adj_drift_paint': (112 if tape else 116) * tot_np,
      'adj_vjp': 112 * tot_np,
      # one pass: read and write d, p, lam_x, lam_p (12 B each way; p
      # carries the next step's p_half, so no force buffer), gather the
      # adjoint density (4 B per cell) and the three force meshes (12 B
      # per cell), reduce into the adjoint force mesh (16 B per cell)
      'adj_drift_vjp': 128 * tot_np,
      'adj_div': 20 * nc_tot,
      # on x-pass meshes (256 or 512 along x) its x pass also clears the
      # adjoint force mesh for the next position, 16 B per cell
      'adj_potential': (24 if n in (256, 512) else 8) * nc_tot,
      # with the tape: the stencil of the stored potential, 16 B per cell
      'adj_force_solve': (16 if tape else 20) * nc_tot,
  }
  roof = {}
  for k, (ms, cnt) in kt.items():
    if k not in kbytes:
      roof[k] = {'avg_launch_ms': ms, 'launches': cnt}
      continue
    gbs = kbytes[k] / (ms * 1e-3) / 1e9
    roof[k] = {'avg_launch_ms': ms, 'launches': cnt,
               'algorithmic_bytes': kbytes[k], 'achieved_gbs': gbs,
               'frac': gbs / peak}
  # the same forward + adjoint with the reverse sweep rebuilding the force
  # meshes (paint + Fourier solve at each reconstructed position) instead
  # of reading the stored potentials
  rebuilt = None
  if tape:
    _lib.lib.fpm_graph_destroy(gf)
    _lib.lib.fpm_graph_destroy(ga)
    _lib.call('fpm_nbody_set_tape', plan.handle, None, 0)
    gf, ga = _lib.ctypes.c_void_p(), _lib.ctypes.c_void_p()
    _lib.call('fpm_graph_capture_nbody', plan.handle, _lib.ptr(D),
              _lib.ptr(P), _lib.ptr(F), None, 0, _lib.ptr(ck), ckpt,
              _lib.ctypes.byref(gf))
    _lib.call('fpm_graph_capture_adjoint', plan.handle, _lib.ptr(D),
              _lib.ptr(P), _lib.ptr(F), _lib.ptr(LX), _lib.ptr(LP), None,
              _lib.ptr(ck), ckpt, _lib.ctypes.byref(ga))
    fwd_adj()
    t_fwd_r = _timed(forward, reps, flush)
    t_all_r = _timed(fwd_adj, reps, flush)
    status |= plan.status(st)
    rebuilt = {'value': 2.0 * np_ * steps / (t_all_r * 1e-3),
               'forward_ms': t_fwd_r, 'forward_adjoint_ms': t_all_r,
               'device_gb_saved': phi_tape.numel() * 4 / 1e9}
  _lib.lib.fpm_graph_destroy(gf)
  _lib.lib.fpm_graph_destroy(ga)
  dev_gb = (plan.device_bytes + 7 * D0.numel() * 4 + ck.numel() * 4 +
            3 * rho.numel() * 4 +
            (phi_tape.numel() * 4 if tape else 0)) / 1e9
  _lib.call('fpm_nbody_set_tape', plan.handle, None, 0)
  plan.close()
  upd = 2.0 * np_ * steps
  method, t_best = 'potential_tape' if tape else 'rebuilt', t_all
  for k, v in (sorted_adj or {}).items():
    if k != 'error' and v['forward_adjoint_ms'] < t_best:
      method, t_best = _sorted_name(k), v['forward_adjoint_ms']
  if sorted_adj:
    for v in sorted_adj.values():
      a = v.get('kernels', {}).get('adj_drift_vjp') if isinstance(
          v, dict) else None
      if a:
        a['achieved_gbs'] = kbytes['adj_drift_vjp'] / (
            a['avg_launch_ms'] * 1e-3) / 1e9
        a['frac'] = a['achieved_gbs'] / peak
  return {
      'workload': ('C5: ' if n == 512 else '') +
                  '2 x %d^3, box %g Mpc/h, %d KDK steps, forward + '
                  'reverse-time adjoint, checkpoint every %d, different '
                  'seeds and cosmologies' % (n, box, steps, ckpt),
      'forward_value': upd / (t_fwd * 1e-3),
      'value': upd / (t_best * 1e-3),
      'unit': 'particle-updates/s (forward + adjoint)',
      'method': method,
      'lattice_walk_adjoint': {'value': upd / (t_all * 1e-3),
                               'forward_adjoint_ms': t_all},
      'sorted_adjoint': sorted_adj,
      'traversal': list(choice),
      'autotune_ms': tune_ms,
      'forward_ms': t_fwd,
      'forward_adjoint_ms': t_best,
      'sims_per_s_forward_adjoint': 2 / (t_best * 1e-3),
      'rebuilt': rebuilt,
      'fp64_check': FP64_CHECK_C5 if n == 512 else None,
      'kernel_roofline': roof,
      'peak_gbs': peak,
      'peak_kind': peak_kind,
      'status': status,
      'device_gb': dev_gb,
      'potential_tape_gb': phi_tape.numel() * 4 / 1e9 if tape else 0.0,
      'pk_final_first_bins': [float(v) for v in pk[0, :8].cpu()],
  }


def main():
  global N_MESH, BOX, WORKLOAD
  args = parse()
  rank, world, local = dist_env()
  if args.mesh != N_MESH:
    BOX = BOX * args.mesh / N_MESH
    N_MESH = args.mesh
    WORKLOAD = ('forward PM, %d^3 particles / %d^3 mesh, box %g Mpc/h, '
                'Planck15, 2LPT at a0=0.1, 40 KDK steps to a=1 (the C2 '
                'workload at another size)' % (N_MESH, N_MESH, BOX))
  if args.impl == 'reference':
    run_reference(args, rank, world)
    return
  import flowpm_b200 as fpm
  from flowpm_b200 import _lib, tfbackground
  from flowpm_b200._plans import get_plan
  torch.cuda.set_device(local)
  dist = None
  if world > 1:
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group('nccl', timeout=timedelta(seconds=300))

  def barrier():
    if dist is not None:
      dist.barrier()
    torch.cuda.synchronize()

  cosmo = fpm.cosmology.Planck15()
  nc = [N_MESH] * 3
  npart = N_MESH**3
  from flowpm_b200 import replicas
  lin = fpm.linear_field(nc, BOX, pk_fn(), batch_size=1,
                         seed=replicas.replica_seed(REPLICA_SEED_BASE, rank))
  s0 = fpm.lpt_init(cosmo, lin, A0, order=2)
  stages = np.linspace(A0, 1.0, N_STEPS + 1)
  plan = get_plan([tuple(nc) + (1,)])
  coefs = tfbackground.nbody_coefficients(cosmo, stages)
  st = _lib.stream_ptr()
  _lib.call('fpm_nbody_set_steps', plan.handle, N_STEPS, _lib.ivec([N_STEPS]),
            _lib.dvec(coefs.ravel()), _lib.dvec([1.5 * cosmo.Omega_m]), st)
  d0 = fpm.tfpm._to_disp(s0[0], nc).contiguous()
  p0 = s0[1].contiguous().clone()
  d, p = torch.empty_like(d0), torch.empty_like(p0)
  f = torch.empty_like(d0)
  flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device='cuda')
  # the library's autotuner: lattice walk or binned step (tile, sort period),
  # timed on this workload; the choice is cached for equal plans
  tuning = None
  if args.binning:
    plan.set_binning(*[int(v) for v in args.binning.split(',')])
  elif args.no_autotune:
    plan.set_binning(0)
  else:
    choice, tms = plan.autotune(d0, p0, reps=2, retune=True)
    tuning = {'choice': list(choice), 'ms_per_config': tms,
              'how': 'fpm_plan_autotune: one graph replay of the 40-step '
                     'run per configuration, best of 2 after a warm-up'}
  tile, every, mode = plan.binning

  # the whole 40-step leapfrog as one CUDA graph (kernels + cuFFT)
  graph = _lib.ctypes.c_void_p()
  _lib.call('fpm_graph_capture_nbody', plan.handle, _lib.ptr(d), _lib.ptr(p),
            _lib.ptr(f), None, 0, None, 0, _lib.ctypes.byref(graph))

  def one_step():
    _lib.call('fpm_graph_launch', graph, st)

  def one_step_profiled():
    _lib.call('fpm_nbody_run', plan.handle, _lib.ptr(d), _lib.ptr(p),
              _lib.ptr(f), None, 0, None, 0, st)

  def reset():
    d.copy_(d0)
    p.copy_(p0)
    flush.fill_(float(rank))  # evicts L2 (256 MB > 126 MB)

  for _ in range(args.warmup):
    reset()
    one_step()
  if plan.status(st):
    raise RuntimeError('non-finite state in warm-up')
  starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
  ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
  # kernels launched per graph replay = kernels of one non-graph run
  n_launch0 = _lib.lib.fpm_launch_count()
  reset()
  one_step_profiled()
  launches_per_step = _lib.lib.fpm_launch_count() - n_launch0
  barrier()
  with ClockSampler(local) as clk:
    for i in range(args.steps):
      reset()
      starts[i].record()
      one_step()
      ends[i].record()
    barrier()
  n_launch = launches_per_step * args.steps
  ms = float(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
  # per-kernel device time: event pairs around every launch of one extra,
  # non-graph pass of the same workload
  _lib.call('fpm_plan_profile', plan.handle, 1)
  reset()
  # keep the GPU busy (bounded spin, ~50 ms) while the host enqueues the
  # profiled pass, so that no event pair includes host launch latency
  torch.cuda._sleep(100_000_000)
  one_step_profiled()
  torch.cuda.synchronize()
  kt, kn = {}, {}
  for kind, name in [(0, 'step'), (1, 'fourier'), (2, 'paint'), (10, 'sort')]:
    tot, cnt = _lib.c_double(), _lib.c_int64()
    _lib.call('fpm_plan_profile_read', plan.handle, kind,
              _lib.ctypes.byref(tot), _lib.ctypes.byref(cnt))
    kt[name], kn[name] = tot.value, cnt.value
  _lib.call('fpm_plan_profile', plan.handle, 0)
  if plan.status(st):
    raise RuntimeError('non-finite state in the timed region')
  # final density of the timed simulation, for the parity leg at the end
  X = torch.empty_like(d)
  _lib.call('fpm_lattice_shift', _lib.ptr(d), _lib.ptr(X), 1, N_MESH, N_MESH,
            N_MESH, 1, st)
  rho_final = fpm.cic_paint(torch.zeros([1] + nc, device='cuda'),
                            X).cpu().numpy()
  del X
  ms_max = replicas.max_over_ranks(ms, device='cuda')
  updates = float(npart) * N_STEPS * args.steps * world
  value = updates / (ms_max * 1e-3)

  # End to end through the public API, host memory in and out every step:
  # X and P of each simulation come from pinned host memory (nbody
  # recomputes F) and the final (X, P, F) go back to pinned host memory.
  # (1) flowpm_b200.NBodyStream: the copies of neighbouring simulations
  #     overlap the computation -- the headline e2e;
  # (2) one fpm.nbody call per simulation, copies in line.
  # L2 is evicted before every simulation, as in the device timing.
  host_in = s0.cpu().pin_memory()
  ns = fpm.NBodyStream(cosmo, stages, nc)
  host_out = ns.host_buffers(2)
  evict = lambda: flush.fill_(1.0)
  ns.run([host_in] * args.warmup,
         out=[host_out[i % 2] for i in range(args.warmup)], before_each=evict)
  ns.synchronize()
  barrier()
  t0 = torch.cuda.Event(enable_timing=True)
  t1 = torch.cuda.Event(enable_timing=True)
  t0.record(ns.s_in)  # before the first upload
  ns.run([host_in] * args.steps,
         out=[host_out[i % 2] for i in range(args.steps)], before_each=evict)
  t1.record(ns.s_out)  # after the last download
  ns.synchronize()
  ms_stream = replicas.max_over_ranks(t0.elapsed_time(t1), device='cuda')
  if ns.status() or not np.isfinite(host_out[0].numpy()).all():
    raise RuntimeError('non-finite end-to-end result')
  ns.close()
  e2e_value = updates / (ms_stream * 1e-3)

  dev = torch.zeros_like(s0)
  single_out = torch.empty_like(host_in).pin_memory()
  e_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
  e_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
  for i in range(args.warmup + args.steps):
    if i >= args.warmup:
      flush.fill_(1.0)
      e_s[i - args.warmup].record()
    dev[:2].copy_(host_in[:2], non_blocking=True)
    out = fpm.nbody(cosmo, dev, stages, nc, check_finite=False)
    single_out.copy_(out, non_blocking=True)
    if i >= args.warmup:
      e_e[i - args.warmup].record()
  torch.cuda.synchronize()
  ms_single = replicas.max_over_ranks(
      float(sum(s.elapsed_time(e) for s, e in zip(e_s, e_e))), device='cuda')
  if not np.isfinite(single_out.numpy()).all():
    raise RuntimeError('non-finite end-to-end result')

  peak, peak_kind = peaks()
  step_ms = kt['step'] / max(kn['step'], 1)
  # the binned step also reads each particle's Lagrangian index (4 B)
  # the binned step also reads each particle's packed lattice site (4 B);
  # re-sorted as they move (mode 3) it also writes it to the new slot
  binned = tile and mode != 2
  kbytes = (KERNEL_BYTES_PER_PART + (4 if binned else 0) +
            (4 if binned and mode == 3 else 0)) * npart
  achieved = kbytes / (step_ms * 1e-3) / 1e9
  whole = STEP_BYTES_PER_PART * npart * N_STEPS * args.steps / (ms * 1e-3) / 1e9
  line = {
      'metric': METRIC,
      'value': value,
      'unit': METRIC,
      'n_gpus': world,
      'steps': args.steps,
      'warmup': args.warmup,
      'ms_per_step': ms_max / args.steps,
      'higher_is_better': True,
      'scaling': 'weak',
      'vs_baseline': None,
      'dtype': 'f32',
      'data': 'synthetic',
      'config': workload_config(world),
      'e2e': {
          'value': e2e_value,
          'unit': METRIC,
          'h2d_bytes_per_step': int(host_in[:2].numel() * 4),
          'd2h_bytes_per_step': int(host_out[0].numel() * 4),
          'api': 'flowpm_b200.NBodyStream (pinned host states in and out, '
                 'copies of neighbouring simulations overlapped)',
          'ms_per_step': ms_stream / args.steps,
          'single_call': {
              'api': 'flowpm_b200.nbody per simulation, copies in line',
              'value': updates / (ms_single * 1e-3),
              'ms_per_step': ms_single / args.steps,
          },
      },
      'gpu_launches': int(n_launch),
      'traversal': ('particles re-sorted by cell (keys in tiles of %d^3 '
                    'cells) as they move, at every step' % tile
                    if mode == 3 else
                    'particles sorted by cell (keys in tiles of %d^3 '
                    'cells) every %d steps, %s' % (
                        tile, every, 'equal chunks' if mode == 1 else
                        'one block per tile, shared-memory paint'))
                   if binned else 'lattice walk',
      'autotune': tuning,
      'roofline': {
          'kernel': (('k_step_binned' if mode == 0 else 'k_step_sorted')
                     if binned else 'k_step') +
                    ' (fused readout + kick + drift + CIC paint)',
          'bound': 'hbm',
          'achieved': achieved,
          'peak': peak,
          'peak_kind': peak_kind,
          'unit': 'GB/s',
          'frac': achieved / peak,
          'traffic': KSTEP_TRAFFIC_BYTES_128.get(
              (tile, mode) if binned else 'walk') if N_MESH == 128
                     else None,
          'algorithmic_bytes_per_launch': kbytes,
          'avg_launch_ms': step_ms,
      },
      'whole_step_roofline': {
          'bytes_per_particle_update': STEP_BYTES_PER_PART,
          'achieved_gbs': whole,
          'frac': whole / peak,
      },
      'kernel_ms_per_step': kt,
      'clocks': clk.summary(),
  }
  if world == 1 and not args.no_extras:
    line['fwd_adjoint'] = measure_fwd_adjoint(fpm, flush, max(args.steps, 3))
    torch.cuda.nvtx.range_push('c3')  # lets a profiler select this part
    line['batched'] = measure_batched(fpm, flush, max(args.steps, 3))
    torch.cuda.nvtx.range_pop()
  if world == 1 and (args.c5 or not (args.no_extras or args.no_c5)):
    torch.cuda.nvtx.range_push('c5')  # lets a profiler select this part
    try:
      line['large'] = measure_large(fpm, flush, n=args.c5_mesh,
                                    tape=not args.no_potential_tape)
    except (_lib.FlowPMError, RuntimeError) as e:  # e.g. out of memory
      line['large'] = {'error': str(e)[:300]}
      torch.cuda.empty_cache()
    finally:
      torch.cuda.nvtx.range_pop()
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    # final density of the timed simulation, against the oracle run from
    # the same linear field (FP32 and FP64); the FP32 run is also the CPU
    # baseline
    line['parity'], line['cpu_baseline'] = parity_and_cpu_baseline(
        lin.cpu(), rho_final)
  _lib.lib.fpm_graph_destroy(graph)
  if rank == 0:
    print(json.dumps(line))
  if dist is not None:
    dist.barrier()
    dist.destroy_process_group()


if __name__ == '__main__':
  main()
