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
