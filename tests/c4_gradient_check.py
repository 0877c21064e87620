"""Gradient check of configuration C4 at full size (128^3, 20 steps) against
the FP64 oracle.  Not collected by pytest: it runs in two halves.

  python tests/c4_gradient_check.py export OUT.npz           # on a GPU
  python tests/c4_gradient_check.py check OUT.npz [N] [tape]  # on the CPU

`export` builds the C4 problem on the GPU (seeded Eisenstein-Hu linear field,
2LPT at a0 = 0.1, 20 KDK steps, chi^2 of the final CIC density against that
density + N(0, 1) noise), computes d chi^2 / d linear with the reverse-time
adjoint (checkpoints every 5 steps) and saves the linear field, the target
and the gradient.  `check` recomputes in float64 with the CPU oracle N
(default 32) central differences along random unit directions and prints
the relative errors of the GPU gradient against them; with `tape` it also
takes the oracle's autograd gradient (tens of GB of host memory at 128^3).
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

N, BOX, A0, STEPS, CKPT = 128, 200.0, 0.1, 20, 5


def export(path):
  import torch
  import flowpm_b200 as fpm
  from flowpm_b200 import tfpower
  cosmo = fpm.cosmology.Planck15()
  kk = np.logspace(-4, 2, 4096)
  pkv = tfpower.linear_matter_power(cosmo, kk)
  pk = lambda k: np.interp(np.log(np.maximum(k, 1e-30)), np.log(kk), pkv,
                           left=0.0)
  lin = fpm.linear_field(N, BOX, pk, seed=4242)
  stages = np.linspace(A0, 1.0, STEPS + 1)
  with torch.no_grad():
    st = fpm.nbody(cosmo, fpm.lpt_init(cosmo, lin, A0), stages, N)
    rho = fpm.cic_paint(torch.zeros((1, N, N, N), device='cuda'), st[0])
  g = torch.Generator(device='cuda').manual_seed(77)
  target = rho + torch.randn(rho.shape, generator=g, device='cuda')
  x = lin.clone().requires_grad_(True)
  st = fpm.nbody(cosmo, fpm.lpt_init(cosmo, x, A0), stages, N,
                 checkpoint_every=CKPT)
  rho = fpm.cic_paint(torch.zeros((1, N, N, N), device='cuda'), st[0])
  loss = ((rho - target)**2).sum()
  (grad,) = torch.autograd.grad(loss, x)
  np.savez(path, linear=lin.cpu().numpy(), target=target.cpu().numpy(),
           grad=grad.cpu().numpy(), loss=float(loss.detach()))
  print("exported", path, "loss", float(loss.detach()))


def check(path, ndir=32, tape=False):
  import torch
  from oracle import background as obg
  from oracle import pm as opm
  torch.set_num_threads(os.cpu_count() or 1)
  z = np.load(path)
  lin = z['linear'].astype(np.float64)
  target = torch.tensor(z['target'].astype(np.float64))
  g_gpu = z['grad'].astype(np.float64)
  b = obg.Background({}, dtype=np.float64)
  stages = np.linspace(A0, 1.0, STEPS + 1)

  def loss(field, grad=False):
    with torch.set_grad_enabled(grad):
      x = torch.tensor(field, requires_grad=grad)
      s = opm.lpt_init(b, x, A0, order=2)
      st = opm.nbody(b, s, stages, N)
      rho = opm.cic_paint(torch.zeros((1, N, N, N), dtype=torch.float64),
                          st[0])
      l = ((rho - target)**2).sum()
      if grad:
        (g,) = torch.autograd.grad(l, x)
        return float(l), g.numpy()
      return float(l), None

  res = {'loss_gpu_fp32': float(z['loss'])}
  g_tape = None
  if tape:
    l0, g_tape = loss(lin, grad=True)
    res['grad_rel_l2_vs_fp64_tape'] = float(
        np.linalg.norm(g_gpu - g_tape) / np.linalg.norm(g_tape))
  else:
    l0, _ = loss(lin)
  res['loss_fp64'] = l0
  rng = np.random.default_rng(5)
  eps = 1e-3 * float(np.std(lin))
  errs, errs_tape = [], []
  for _ in range(ndir):
    u = rng.standard_normal(lin.shape)
    u /= np.linalg.norm(u)
    lp, _ = loss(lin + eps * u)
    lm, _ = loss(lin - eps * u)
    fd = (lp - lm) / (2 * eps)
    errs.append(abs(float(np.sum(g_gpu * u)) - fd) / abs(fd))
    if g_tape is not None:
      errs_tape.append(abs(float(np.sum(g_tape * u)) - fd) / abs(fd))
    print('direction', len(errs), 'fd', fd, 'gpu', float(np.sum(g_gpu * u)),
          flush=True)
  res.update({
      'fd_directions': ndir, 'fd_eps': eps,
      'gpu_vs_fd_median_rel': float(np.median(errs)),
      'gpu_vs_fd_max_rel': float(np.max(errs)),
  })
  if errs_tape:
    res['fp64_tape_vs_fd_median_rel'] = float(np.median(errs_tape))
    res['fp64_tape_vs_fd_max_rel'] = float(np.max(errs_tape))
  print(json.dumps(res))


if __name__ == '__main__':
  if sys.argv[1] == 'export':
    export(sys.argv[2])
  else:
    check(sys.argv[2], int(sys.argv[3]) if len(sys.argv) > 3 else 32,
          len(sys.argv) > 4 and sys.argv[4] == 'tape')
