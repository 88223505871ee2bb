"""Checkpoint files in the layout of GRACE's checkpoint datasets (CPU):
names, lengths and element order of the datasets, the attributes, a save /
load round trip, and the reader's length check."""
import numpy as np
import pytest
import torch

from grace_b200 import abi
from grace_b200.checkpoint import (CELL, FACES, checkpoint_name, dataset_lengths, load_checkpoint,
                                   save_checkpoint)
from grace_b200.host import Blocks


def _fields(blocks, seed):
    rng = np.random.default_rng(seed)
    f = blocks.new_fields()
    for t in (f.state, f.bx, f.by, f.bz):
        t.copy_(torch.from_numpy(rng.standard_normal(tuple(t.shape))))
    return f


def test_file_name_follows_the_reference_pattern():
    assert checkpoint_name(42) == "checkpoint_data_000042.npz"
    assert checkpoint_name(1234567, ".h5") == "checkpoint_data_1234567.h5"


def test_datasets_are_layoutleft_spans_and_round_trip(tmp_path):
    b = Blocks(4, 3, 2, 4, 3, np.ones((3, 3)), device="cpu")
    f = _fields(b, 1)
    path = save_checkpoint(str(tmp_path), f, time=1.25, iteration=7, extents=((-1, 1), (-2, 2), (-3, 3)),
                           b_field_injection_fired=True)
    assert path.endswith("checkpoint_data_000007.npz")
    with np.load(path) as z:
        lens = dataset_lengths(b)
        for name in (CELL,) + FACES:
            assert z[name].ndim == 1 and z[name].dtype == np.float64 and z[name].size == lens[name]
        # element (i, j, k, v, q) of the LayoutLeft array sits at
        # i + NX (j + NY (k + NZ (v + nvars q)))
        i, j, k, v, q = 5, 2, 7, 11, 2
        NX, NY, NZ = b.NX, b.NY, b.NZ
        assert z[CELL][i + NX * (j + NY * (k + NZ * (v + abi.N_EVOL_VARS * q)))] == f.state[q, v, k, j, i].item()
        assert z[FACES[0]][(NX + 1) * (j + NY * (k + NZ * q)) + i] == f.bx[q, k, j, i].item()
        assert float(z["attrs/Time"]) == 1.25 and int(z["attrs/Iteration"]) == 7
        assert z["attrs/Iteration"].dtype == np.uint32
        np.testing.assert_array_equal(z["grid_extent_y"], [-2.0, 2.0])
        assert int(z["b_field_injection/has_fired"]) == 1
    g = b.new_fields()
    t, it, ext, fired = load_checkpoint(path, g)
    assert (t, it, ext, fired) == (1.25, 7, ((-1.0, 1.0), (-2.0, 2.0), (-3.0, 3.0)), True)
    for a, c in zip((f.state, f.bx, f.by, f.bz), (g.state, g.bx, g.by, g.bz)):
        assert torch.equal(a, c)


def test_reader_rejects_a_different_grid(tmp_path):
    b = Blocks(4, 4, 4, 4, 2, np.ones((2, 3)), device="cpu")
    path = save_checkpoint(str(tmp_path), _fields(b, 2), 0.0, 0, ((0, 1),) * 3)
    other = Blocks(4, 4, 4, 4, 3, np.ones((3, 3)), device="cpu")
    with pytest.raises(ValueError, match="dimensions do not match"):
        load_checkpoint(path, other.new_fields())
