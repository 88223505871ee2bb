"""Checkpoint and restart of the evolved state in the dataset layout of
GRACE's checkpoint files.

GRACE writes, per checkpoint, a forest file and a data file
(src/system/checkpoint_handler.cpp:415-620): the file attributes "Time"
(double) and "Iteration" (unsigned int), the datasets "grid_extent_x/y/z"
(the domain's [min, max]), the group "b_field_injection" with the integer
dataset "has_fired", and one 1-D double dataset per state array
(write_data_hdf5, :308-400): "CellCenteredData" for the cell-centred
var_array_t and "FaceCenteredDataX/Y/Z" for the face-staggered arrays, each
the array's contiguous LayoutLeft span — every cell of every block, ghost
zones included, i fastest, then j, k, variable and block — so that
dataset element i + NX (j + NY (k + NZ (v + nvars q))) is array element
(i, j, k, v, q).  Staggered arrays with no variables (corner and edge data
in this system) are not written (:334-335).  On restart the reader checks
each dataset's length against the array it fills (read_data_hdf5,
:160-230; load, :935-942).

The device arrays of this library are those LayoutLeft arrays, so a
checkpoint is one device-to-host copy per array.  The container is a NumPy
.npz archive with the same dataset names ("attrs/Time" and
"attrs/Iteration" hold the two file attributes, "b_field_injection/
has_fired" the group's dataset): this image has no HDF5 library.  File
names follow GRACE's checkpoint_data_<iteration, 6 digits> pattern.
"""
import os

import numpy as np
import torch

from . import abi

CELL = "CellCenteredData"
FACES = ("FaceCenteredDataX", "FaceCenteredDataY", "FaceCenteredDataZ")
EXTENTS = ("grid_extent_x", "grid_extent_y", "grid_extent_z")


def checkpoint_name(iteration, ext=".npz"):
    """checkpoint_data_<iteration, zero-padded to 6 digits><ext>, GRACE's
    get_filename (checkpoint_handler.cpp:89-98)."""
    return f"checkpoint_data_{int(iteration):06d}{ext}"


def _datasets(fields):
    """The state arrays by dataset name, in LayoutLeft order (C order of the
    (nq, nvars, NZ, NY, NX) tensors)."""
    return {CELL: fields.state, FACES[0]: fields.bx, FACES[1]: fields.by, FACES[2]: fields.bz}


def save_checkpoint(directory, fields, time, iteration, extents, b_field_injection_fired=False):
    """Write the checkpoint of `fields` (grace_b200.host.Fields on the
    device) for `iteration` into `directory`; extents: ((xmin, xmax),
    (ymin, ymax), (zmin, zmax)).  Returns the file's path."""
    os.makedirs(directory, exist_ok=True)
    out = {}
    for name, t in _datasets(fields).items():
        if not t.is_contiguous():
            raise ValueError(f"{name}: the device array must be contiguous")
        out[name] = t.detach().reshape(-1).to("cpu").numpy()
    for name, (lo, hi) in zip(EXTENTS, extents):
        out[name] = np.array([lo, hi], dtype=np.float64)
    out["b_field_injection/has_fired"] = np.array(int(bool(b_field_injection_fired)), dtype=np.int32)
    out["attrs/Time"] = np.array(float(time), dtype=np.float64)
    out["attrs/Iteration"] = np.array(int(iteration), dtype=np.uint32)
    path = os.path.join(directory, checkpoint_name(iteration))
    with open(path, "wb") as fh:
        np.savez(fh, **out)
    return path


def load_checkpoint(path, fields):
    """Fill `fields` (device Fields of the reserved geometry) from a
    checkpoint written by save_checkpoint; every dataset's length must match
    its array (ValueError otherwise, as GRACE's reader asserts).  Returns
    (time, iteration, extents, b_field_injection_fired).  The caller then
    refills the ghost zones and recomputes the primitives, as GRACE does
    after loading."""
    with np.load(path) as z:
        for name, t in _datasets(fields).items():
            if name not in z.files:
                raise ValueError(f"checkpoint {path} has no dataset {name}")
            d = z[name]
            if d.ndim != 1 or d.dtype != np.float64 or d.size != t.numel():
                raise ValueError(f"dataset {name} dimensions do not match: {d.size} != {t.numel()}")
        for name, t in _datasets(fields).items():
            t.copy_(torch.from_numpy(z[name]).reshape(t.shape))
        time = float(z["attrs/Time"])
        iteration = int(z["attrs/Iteration"])
        extents = tuple(tuple(float(x) for x in z[name]) for name in EXTENTS)
        fired = bool(int(z["b_field_injection/has_fired"])) if "b_field_injection/has_fired" in z.files else False
    return time, iteration, extents, fired


def dataset_lengths(blocks, n_state_vars=abi.N_EVOL_VARS):
    """Lengths of the four state datasets for a grid (grace_b200.host.Blocks):
    the cell array's NX NY NZ n_state_vars nq and each face array's one
    staggered variable over (NX + 1) NY NZ nq and the like."""
    NX, NY, NZ, nq = blocks.NX, blocks.NY, blocks.NZ, blocks.nq
    return {CELL: NX * NY * NZ * n_state_vars * nq, FACES[0]: (NX + 1) * NY * NZ * nq,
            FACES[1]: NX * (NY + 1) * NZ * nq, FACES[2]: NX * NY * (NZ + 1) * nq}
