"""Generate tests/golden/balsara1024_ref.npz: Balsara-1 at its configured
size, 1024 x 16 x 16 cells (64 blocks of 16^3, periodic y and z, outflow
x), evolved to t = 0.4 with the adaptive CFL-0.4 step of evolve_impl
(find_stable_timestep after every step) by the reference's own per-cell
numerics (the pinning build oracle/_ref/libgrace_ref.so, GRACE's EOS, c2p,
WENO-Z, HLLE and UCT kernels compiled in place, driven by the restated
loops).  Run in a checkout where the pinning build exists:

    python tests/golden/make_balsara1024.py

The problem is one-dimensional and the transverse directions are periodic,
so the fixture keeps one x-line of the final density (the first interior
(y, z) cell of every block column), the largest difference between that
line and any other (y, z) line of the same run (the test compares the GPU's
whole field against the line, so this spread bounds what the line stands
for), the step count and the time steps taken.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from grace_b200 import abi, params, workloads  # noqa: E402
import _oracle  # noqa: E402

T_END, CFL = 0.4, 0.4


def density_line(aux, ngz, nb):
    """rho on the x-line of interior (y, z) cell (0, 0), blocks ordered by x."""
    g = ngz
    r = aux[:, abi.RHO, g:-g, g:-g, g:-g]      # (nq, nz, ny, nx)
    return np.concatenate([r[q, 0, 0] for q in range(nb)]), r


def main():
    assert _oracle.lib("ref") is not None, "build oracle/_ref first: make -C oracle ref"
    P = params.balsara1()
    su, f = workloads.balsara1(nb=(64, 1, 1), n=(16, 16, 16))
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, 16, 16, 16, su.ngz, su.nq, "ref")
    state = [st, bx, by, bz]
    _oracle.fill_ghosts("ref", su, state)
    S.compute_aux(su.idx().copy(), state, aux)
    sp = [x.copy() for x in state]
    spp = [x.copy() for x in state]
    dx = np.ascontiguousarray(1.0 / su.idx())
    dtn = S.find_stable_timestep(state, aux, dx, CFL)
    t, dts = 0.0, []
    t0 = time.time()
    while t < T_END - 1e-15:
        dt = min(dtn, T_END - t)
        _oracle.rk3_step(S, su, dt, state, sp, spp, aux, "ref")
        dtn = S.find_stable_timestep(state, aux, dx, CFL)
        t += dt
        dts.append(dt)
        if len(dts) % 100 == 0:
            print(f"step {len(dts)} t={t:.4f} ({time.time() - t0:.0f} s)", flush=True)
    line, r = density_line(aux, su.ngz, su.nq)
    spread = float(np.max(np.abs(r - r[:, :1, :1, :])))
    np.savez_compressed(os.path.join(HERE, "balsara1024_ref.npz"), rho_line=line, steps=len(dts),
                        dts=np.asarray(dts), t_end=t, transverse_spread=spread)
    print(f"{len(dts)} steps to t={t}, transverse spread {spread:.3e}, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
