"""Gradient check of configuration C4 at full size (128^3 particles and mesh,
box 200 Mpc/h, 20 KDK steps) against the FP64 oracle.  Not collected by
pytest: it runs in two halves, the first on a GPU, the second on the CPU
(about two hours on 8 cores for the default sweep).

  python tests/c4_gradient_check.py export OUT.npz             # GPU
  python tests/c4_gradient_check.py check OUT.npz RESULT.json  # CPU
      [--ndir 32] [--eps 1e-3,1e-4,1e-5] [--no-tape]

`export` builds the C4 problem on the GPU: seeded Eisenstein-Hu linear field,
2LPT at a0 = 0.1, 20 KDK steps, chi^2 of the final CIC density against a
target = that density + N(0, 1) noise (NumPy seed, so the CPU half draws the
same).  It computes d chi^2 / d linear with the reverse-time adjoint
(checkpoints every 5 steps) twice: rebuilding the trajectory from the final
state, and with the stored force potentials (the potential tape).

`check` runs the same problem through the oracle in float64 and compares:
* the FP64 tape gradient (autograd through the oracle, the stand-in for
  TensorFlow's tape; each step checkpointed so that it fits in about 20 GB
  of host memory) with both GPU gradients over all 2^21 components
  (relative L2) and along `ndir` random unit directions, beside the
  oracle's FP32 tape gradient (the reference's own arithmetic), whose
  distance from FP64 is the floor an FP32 gradient of this chaotic
  trajectory can reach;
* float64 central differences at each relative step eps (times the field's
  standard deviation) along the same directions, against the FP64 tape
  (this shows the finite differences converging, and where they stop) and
  against the GPU gradients.
Each direction's numbers are appended to RESULT.json as they come, so a
partial run still reports.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

N, BOX, A0, STEPS, CKPT = 128, 200.0, 0.1, 20, 5
LIN_SEED, NOISE_SEED, DIR_SEED = 4242, 77, 5


def export(path):
  import torch
  import flowpm_b200 as fpm
  from flowpm_b200 import tfpower
  cosmo = fpm.cosmology.Planck15()
  kk = np.logspace(-4, 2, 4096)
  pkv = tfpower.linear_matter_power(cosmo, kk)
  pk = lambda k: np.interp(np.log(np.maximum(k, 1e-30)), np.log(kk), pkv,
                           left=0.0)
  lin = fpm.linear_field(N, BOX, pk, seed=LIN_SEED)
  stages = np.linspace(A0, 1.0, STEPS + 1)
  zeros = lambda: torch.zeros((1, N, N, N), device='cuda')
  with torch.no_grad():
    st = fpm.nbody(cosmo, fpm.lpt_init(cosmo, lin, A0), stages, N)
    rho = fpm.cic_paint(zeros(), st[0])
  noise = np.random.default_rng(NOISE_SEED).standard_normal(
      (1, N, N, N)).astype(np.float32)
  target = rho + torch.tensor(noise, device='cuda')
  out = {'linear': lin.cpu().numpy(), 'target': target.cpu().numpy()}
  for name, tape in (('rebuilt', False), ('tape', True)):
    x = lin.clone().requires_grad_(True)
    st = fpm.nbody(cosmo, fpm.lpt_init(cosmo, x, A0), stages, N,
                   checkpoint_every=CKPT, store_potential=tape)
    rho = fpm.cic_paint(zeros(), st[0])
    loss = ((rho - target)**2).sum()
    (grad,) = torch.autograd.grad(loss, x)
    out['grad_' + name] = grad.cpu().numpy()
    out['loss_' + name] = float(loss.detach())
  np.savez(path, **out)
  print('exported', path, 'loss', out['loss_rebuilt'], out['loss_tape'])


def check(path, result, ndir, eps_list, tape):
  import torch
  from oracle import background as obg
  from oracle import pm as opm
  torch.set_num_threads(os.cpu_count() or 1)
  z = np.load(path)
  lin = z['linear'].astype(np.float64)
  target = torch.tensor(z['target'].astype(np.float64))
  g_gpu = {k: z['grad_' + k].astype(np.float64) for k in ('rebuilt', 'tape')}
  b = obg.Background({}, dtype=np.float64)
  stages = np.linspace(A0, 1.0, STEPS + 1)

  def loss(field, grad=False, dtype=torch.float64):
    bb = b if dtype == torch.float64 else obg.Background({}, dtype=np.float32)
    with torch.set_grad_enabled(grad):
      x = torch.tensor(field, dtype=dtype, requires_grad=grad)
      s = opm.lpt_init(bb, x, A0, order=2)
      st = (opm.nbody_checkpointed if grad else opm.nbody)(bb, s, stages, N)
      rho = opm.cic_paint(torch.zeros((1, N, N, N), dtype=dtype), st[0])
      l = ((rho - target.to(dtype))**2).sum()
      if grad:
        (g,) = torch.autograd.grad(l, x)
        return float(l), g.double().numpy()
      return float(l), None

  res = {'config': 'C4: 128^3, box %g, 20 KDK steps, 2LPT at a0 = %g, '
                   'chi^2(final CIC density, density + N(0,1))' % (BOX, A0),
         'loss_gpu_fp32': {k: float(z['loss_' + k]) for k in g_gpu},
         'cores': torch.get_num_threads()}

  def save():
    with open(result, 'w') as f:
      json.dump(res, f, indent=1)

  t0 = time.time()
  g_tape = None
  if tape:
    l0, g_tape = loss(lin, grad=True)
    # the reference's own arithmetic: the oracle's FP32 tape gradient
    _, g32 = loss(lin.astype(np.float32), grad=True, dtype=torch.float32)
    g_gpu_all = dict(g_gpu, oracle_fp32_tape=g32)
    res['grad_rel_l2_vs_fp64_tape'] = {
        k: float(np.linalg.norm(g - g_tape) / np.linalg.norm(g_tape))
        for k, g in g_gpu_all.items()}
  else:
    l0, _ = loss(lin)
  res['loss_fp64'] = l0
  res['tape_seconds'] = time.time() - t0
  save()
  print(json.dumps(res), flush=True)
  rng = np.random.default_rng(DIR_SEED)
  sd = float(np.std(lin))
  res['eps_rel_to_std'] = eps_list
  res['field_std'] = sd
  res['directions'] = []
  for i in range(ndir):
    u = rng.standard_normal(lin.shape)
    u /= np.linalg.norm(u)
    row = {k: float(np.sum(g * u)) for k, g in g_gpu.items()}
    if g_tape is not None:
      row['fp64_tape'] = float(np.sum(g_tape * u))
      row['oracle_fp32_tape'] = float(np.sum(g32 * u))
    row['fd'] = {}
    for e in eps_list:
      h = e * sd
      lp, _ = loss(lin + h * u)
      lm, _ = loss(lin - h * u)
      row['fd']['%g' % e] = (lp - lm) / (2 * h)
    res['directions'].append(row)
    save()
    print('direction', i, json.dumps(row), flush=True)
  res['summary'] = summarize(res)
  save()
  print(json.dumps(res['summary'], indent=1))


def summarize(res):
  """Median and max relative errors over the directions: GPU gradients and
  FD against the FP64 tape, GPU gradients against FD at each eps."""
  rows = res['directions']
  out = {'directions': len(rows)}

  def stats(vals):
    v = np.abs(np.asarray(vals))
    return {'median': float(np.median(v)), 'max': float(np.max(v))}

  if rows and 'fp64_tape' in rows[0]:
    t = np.array([r['fp64_tape'] for r in rows])
    scale = np.abs(t)
    for k in ('rebuilt', 'tape', 'oracle_fp32_tape'):
      out['%s_vs_fp64_tape' % (k if k.startswith('oracle') else
                               'gpu_' + k)] = stats(
          (np.array([r[k] for r in rows]) - t) / scale)
    for e in res['eps_rel_to_std']:
      fd = np.array([r['fd']['%g' % e] for r in rows])
      out['fd64_eps_%g_vs_fp64_tape' % e] = stats((fd - t) / scale)
  for e in res['eps_rel_to_std']:
    fd = np.array([r['fd']['%g' % e] for r in rows])
    for k in ('rebuilt', 'tape'):
      out['gpu_%s_vs_fd64_eps_%g' % (k, e)] = stats(
          (np.array([r[k] for r in rows]) - fd) / np.abs(fd))
  return out


if __name__ == '__main__':
  ap = argparse.ArgumentParser()
  ap.add_argument('phase', choices=['export', 'check', 'summary'])
  ap.add_argument('npz')
  ap.add_argument('result', nargs='?', default='c4_gradient_check.json')
  ap.add_argument('--ndir', type=int, default=32)
  ap.add_argument('--eps', default='1e-3,1e-4,1e-5')
  ap.add_argument('--no-tape', action='store_true')
  a = ap.parse_args()
  if a.phase == 'export':
    export(a.npz)
  elif a.phase == 'summary':
    with open(a.result) as f:
      r = json.load(f)
    print(json.dumps(summarize(r), indent=1))
  else:
    check(a.npz, a.result, a.ndir, [float(e) for e in a.eps.split(',')],
          not a.no_tape)
