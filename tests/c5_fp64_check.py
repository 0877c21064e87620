"""Error of a C5-spacing simulation against the oracle in float32 and float64.
Not collected by pytest (minutes of host CPU); run on a GPU machine:

  python tests/c5_fp64_check.py [--mesh 256] [--steps 30] [--out R.json]

C5 is two 512^3 simulations in a 1000 Mpc/h box, 30 KDK steps.  The oracle
(torch on the host cores) cannot run 512^3 in reasonable time, so by default
this takes one of C5's two simulations (Planck15, seed 5120) at 256^3 in a
500 Mpc/h box: the same spacing (1.95 Mpc/h), initial time, step count and
cosmology.  The CUDA path (seeded Eisenstein-Hu linear field, 2LPT at
a0 = 0.1, 30 steps) and the oracle start from the same linear field; the
script reports the relative L2 error of the final CIC density and the
largest per-bin P(k) error of the GPU result against the FP32 oracle (the
reference's arithmetic) and against the FP64 oracle (the same method in
double), and the FP32 oracle's own distance from FP64.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

A0, SEED = 0.1, 5120


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--mesh', type=int, default=256)
  ap.add_argument('--steps', type=int, default=30)
  ap.add_argument('--out', default=None)
  a = ap.parse_args()
  import torch
  import flowpm_b200 as fpm
  from flowpm_b200 import tfpower
  from oracle import background as obg
  from oracle import pm as opm
  n, box = a.mesh, 1000.0 * a.mesh / 512
  cosmo = fpm.cosmology.Planck15()
  kk = np.logspace(-4, 2, 4096)
  pkv = tfpower.linear_matter_power(cosmo, kk)
  pk = lambda k: np.interp(np.log(np.maximum(k, 1e-30)), np.log(kk), pkv,
                           left=0.0)
  stages = np.linspace(A0, 1.0, a.steps + 1)
  lin = fpm.linear_field(n, box, pk, seed=SEED)
  st = fpm.nbody(cosmo, fpm.lpt_init(cosmo, lin, A0, order=2), stages, n)
  rho = fpm.cic_paint(torch.zeros((1, n, n, n), device='cuda'), st[0])
  rho = rho.cpu().numpy()
  lin = lin.cpu()
  del st
  torch.cuda.empty_cache()
  torch.set_num_threads(os.cpu_count() or 1)

  def oracle(dtype):
    b = obg.Background({}, dtype=np.float32 if dtype == torch.float32
                       else np.float64)
    t0 = time.time()
    s = opm.lpt_init(b, lin.to(dtype), A0, order=2)
    s = opm.nbody(b, s, stages, n)
    r = opm.cic_paint(torch.zeros((1, n, n, n), dtype=dtype), s[0]).numpy()
    return r, time.time() - t0

  rho32, t32 = oracle(torch.float32)
  rho64, t64 = oracle(torch.float64)

  def rel(x, y):
    x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))

  def pks(r):
    _, p = opm.power_spectrum(torch.tensor(r, dtype=torch.float64),
                              kmin=0.01, dk=0.01, boxsize=np.array([box] * 3))
    return p.numpy().ravel()

  p, p32, p64 = pks(rho), pks(rho32), pks(rho64)
  ok = np.isfinite(p64) & (p64 != 0) & np.isfinite(p32) & (p32 != 0)
  prel = lambda x, y: float(np.max(np.abs(x[ok] - y[ok]) / np.abs(y[ok])))
  res = {
      'workload': 'one C5 simulation at %d^3, box %g Mpc/h (C5 spacing), '
                  'Planck15, seed %d, 2LPT at a0 = %g, %d KDK steps' %
                  (n, box, SEED, A0, a.steps),
      'vs_oracle_fp32': {'density_rel_l2': rel(rho, rho32),
                         'pk_max_rel': prel(p, p32)},
      'fp64_error': {'density_rel_l2': rel(rho, rho64),
                     'pk_max_rel': prel(p, p64),
                     'oracle_fp32_density_rel_l2': rel(rho32, rho64),
                     'oracle_fp32_pk_max_rel': prel(p32, p64)},
      'pk_bins': 'kmin 0.01, dk 0.01 h/Mpc',
      'oracle_seconds': {'fp32': t32, 'fp64': t64,
                         'threads': torch.get_num_threads()},
  }
  print(json.dumps(res))
  if a.out:
    with open(a.out, 'w') as f:
      json.dump(res, f, indent=1)


if __name__ == '__main__':
  main()
