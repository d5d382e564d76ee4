"""Writes inlet_1m_oracle.npz: the FP64 oracle's flow steps of the benchmarked
workload -- the three-level telescoping tidal inlet of about 1.0M cells
(cms2d_b200.cases.tidal_inlet(1_000_000, seed=11), dt = 300 s) -- in the
reference's natural cell order, every solve (ILU(0)-BiCGStab) driven to a
1e-9 relative L2 residual or 600 iterations (FP64 BiCGStab stagnates near
3e-10 on the pressure-correction systems, so 1e-10 is not reachable; late in
a step, when a system's right-hand side is tiny, the reference's absolute
small = 1e-15 guards stall it earlier, and the cap ends those solves at their
attainable accuracy), the outer SIMPLEC loop ended by check_conv.

The full fields (3 x 8 MB per step) are too large to commit, so the file
holds, after each of STEPS steps: the water level and the velocities at
NSAMPLE seeded cells (and the 200 gauge cells of cms2d_b200.cases.gauges),
the outer iteration count, and statistics over all active cells (mean, min,
max and RMS of the water level, largest |u| and |v|, sum of the depths).

A run takes tens of minutes on the host cores (the reference's serial ILU(0)
factor and sweeps dominate).  From the repository root:

    python tests/golden/make_inlet_1m_oracle.py [threads]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cms2d_b200 import cases  # noqa: E402
from oracle import oracle as O  # noqa: E402

CELLS, SEED, STEPS, NSAMPLE, TOL, NSWP = 1_000_000, 11, 6, 8192, 1e-9, 600
OUT = os.path.join(HERE, "inlet_1m_oracle.npz")


def sample_cells(n: int) -> np.ndarray:
    return np.sort(np.random.default_rng(20261203).choice(n, size=NSAMPLE, replace=False))


def field_stats(eta, u, v, h):
    return np.array([eta.mean(), eta.min(), eta.max(), np.sqrt(np.mean(eta * eta)), np.abs(u).max(),
                     np.abs(v).max(), h.sum()])


STAT_NAMES = ["eta_mean", "eta_min", "eta_max", "eta_rms", "umax", "vmax", "h_sum"]


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    O.build()
    O.set_threads(threads)
    case = cases.tidal_inlet(CELLS, seed=SEED)
    n = case.grid.ncells
    idx = sample_cells(n)
    gauges = cases.gauges(case)
    f = O.FlowOracle(case)
    f.set_solver(nsolv=3, precond=O.PC_ILU0, tol=TOL, nswp_pp=NSWP, nswp_uv=NSWP, norm=2)
    f.init()
    eta_s, u_s, v_s, eta_g, stats, niter = [], [], [], [], [], []
    for s in range(STEPS):
        t0 = time.perf_counter()
        r = f.step()
        assert r["status"] == 0, r
        eta, u, v, h = (f.get(k)[:n] for k in ("eta", "u", "v", "h"))
        eta_s.append(eta[idx]); u_s.append(u[idx]); v_s.append(v[idx]); eta_g.append(eta[gauges])
        stats.append(field_stats(eta, u, v, h))
        niter.append(r["niter"])
        print(f"step {s + 1}: {r['niter']} outer iterations, {f.solve_iters} Krylov iterations so far, "
              f"{time.perf_counter() - t0:.0f} s", flush=True)
    np.savez_compressed(OUT, cells=np.int64(n), seed=np.int64(SEED), tol=TOL, nswp=NSWP, sample=idx, gauges=gauges,
                        eta=np.array(eta_s), u=np.array(u_s), v=np.array(v_s), eta_gauges=np.array(eta_g),
                        stats=np.array(stats), stat_names=np.array(STAT_NAMES), niter=np.array(niter))
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
