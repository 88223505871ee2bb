"""Host-side helpers that need no GPU."""
import numpy as np

from grace_b200 import workloads


def test_outer_faces_of_a_brick():
    """Every block face on a non-periodic outer boundary, once; none on a
    periodic axis."""
    su = workloads.BrickSetup((3, 2, 1), (8, 8, 8), (0, 0, 0), (3, 2, 1), 4, (False, True, False))
    quad, face = su.outer_faces()
    pairs = set(zip(quad.tolist(), face.tolist()))
    assert len(pairs) == len(quad)
    # x: blocks at ix = 0 (low) and ix = 2 (high), 2 of each; y periodic;
    # z: one layer, every block has both z faces
    assert sorted(f for f in face.tolist() if f < 2) == [0, 0, 1, 1]
    assert not any(f in (2, 3) for f in face.tolist())
    assert sum(f == 4 for f in face.tolist()) == 6 and sum(f == 5 for f in face.tolist()) == 6
    for q, f in pairs:
        ix = q % 3
        if f == 0:
            assert ix == 0
        if f == 1:
            assert ix == 2


def test_brick_runs_cover_the_brick_and_name_every_neighbour():
    """brick_runs: consecutive runs of whole z-slabs covering every block
    once, and deps[r] holding the run of every face, edge and corner
    neighbour of each of run r's blocks (wrapping along periodic axes)."""
    from grace_b200.host import brick_runs
    for nb, per, nruns in (((4, 3, 7), (False, False, False), 3), ((2, 2, 6), (True, True, True), 4),
                           ((3, 1, 2), (False, True, False), 5), ((1, 1, 1), (True, True, True), 2)):
        runs, deps = brick_runs(nb, per, nruns)
        nq = nb[0] * nb[1] * nb[2]
        assert runs[0][0] == 0 and runs[-1][1] == nq
        assert all(a[1] == b[0] for a, b in zip(runs, runs[1:]))
        assert all((q1 - q0) % (nb[0] * nb[1]) == 0 and q1 > q0 for q0, q1 in runs)
        run_of = np.zeros(nq, dtype=int)
        for r, (q0, q1) in enumerate(runs):
            run_of[q0:q1] = r
        for q in range(nq):
            c = (q % nb[0], (q // nb[0]) % nb[1], q // (nb[0] * nb[1]))
            for o in np.ndindex(3, 3, 3):
                cc = []
                for a in range(3):
                    x = c[a] + o[a] - 1
                    if per[a]:
                        x %= nb[a]
                    x = min(max(x, 0), nb[a] - 1)
                    cc.append(x)
                src = cc[0] + nb[0] * (cc[1] + nb[1] * cc[2])
                assert run_of[src] in deps[run_of[q]], (nb, per, q, o)


def test_rk4_coefficients_are_fourth_order():
    """The rk4 branch's low-storage coefficients (as rk4_step applies them)
    integrate y' = -y with a local error shrinking as h^5: halving the step
    divides it by ~32."""
    from grace_b200.host import GRMHDEquationsSystem as G

    def step(y, h, lam=-1.0):
        (_, g11, g21, b1), (d2, g12, g22, b2), (d3, g13, g23, b3), (_, g14, g24, b4) = G.RK4_COEFFS
        s1 = s2 = y
        s3 = g11 * s1 + g21 * s2
        s3 = s3 + b1 * h * lam * s1
        s2 = s2 + d2 * s3
        s1 = g12 * s3 + g22 * s2
        s1 = s1 + b2 * h * lam * s3
        s2 = s2 + d3 * s1
        s3 = g13 * s1 + g23 * s2
        s3 = s3 + b3 * h * lam * s1
        s1 = g14 * s3 + g24 * s2
        return s1 + b4 * h * lam * s3

    e1 = abs(step(1.0, 0.1) - np.exp(-0.1))
    e2 = abs(step(1.0, 0.05) - np.exp(-0.05))
    assert 25.0 < e1 / e2 < 40.0, (e1, e2)
