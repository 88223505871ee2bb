"""FMR restriction into coarse buffers on the GPU (grb_restrict_to_coarse)
against the oracle (oracle/amr_oracle.hpp, itself pinned to the reference's
operators): bit for bit, both variable lists, every Morton child position,
the three face arrays; and div B of the restricted face field."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem

pytestmark = pytest.mark.gpu

N, G = 16, 4
NN = N + 2 * G


def test_restrict_to_coarse_matches_oracle_bitwise():
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(31)
    nq, ncb = 16, 16
    st = rng.standard_normal((nq, abi.N_EVOL_VARS, NN, NN, NN))
    fb = [rng.standard_normal((nq, NN, NN, NN + 1)), rng.standard_normal((nq, NN, NN + 1, NN)),
          rng.standard_normal((nq, NN + 1, NN, NN))]
    src_q = np.arange(nq, dtype=np.int64)
    dst_q = rng.permutation(ncb)[:nq].astype(np.int64)
    child = (np.arange(nq) % 8).astype(np.uint8)
    vlo, vhi = [0, 5, 6, 13], [1, 2, 3, 4]
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(N, N, N, G, nq, np.ones((nq, 3)), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    fine = Fields(T(st), T(fb[0]), T(fb[1]), T(fb[2]))
    cb = Fields(torch.zeros((ncb, abi.N_EVOL_VARS, NN, NN, NN), dtype=torch.float64, device=dev),
                *[torch.zeros((ncb,) + x.shape[1:], dtype=torch.float64, device=dev) for x in fb])
    g.restrict_to_coarse(fine, cb, T(src_q), T(dst_q), T(child), vlo, vhi)
    torch.cuda.synchronize()
    # oracle
    ost = np.zeros((ncb, abi.N_EVOL_VARS, NN, NN, NN))
    _oracle.restrict_cells("orc", N, G, abi.N_EVOL_VARS, st, ost, src_q, dst_q, child, vlo, vhi)
    np.testing.assert_array_equal(cb.state.cpu().numpy(), ost)
    for d in range(3):
        of = np.zeros((ncb,) + fb[d].shape[1:])
        _oracle.restrict_faces(d, N, G, np.ascontiguousarray(fb[d]), of, src_q, dst_q)
        np.testing.assert_array_equal((cb.bx, cb.by, cb.bz)[d].cpu().numpy(), of)
    assert g.status().device_flags == 0


def test_restricted_face_field_is_divergence_free():
    """A discretely divergence-free fine face field (curl of an edge vector
    potential) restricts to a divergence-free coarse one."""
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(8)
    Ax, Ay, Az = [rng.standard_normal((NN + 1, NN + 1, NN + 1)) for _ in range(3)]
    bx = (Az[:NN, 1:, :] - Az[:NN, :NN, :]) - (Ay[1:, :NN, :] - Ay[:NN, :NN, :])
    by = (Ax[1:, :, :NN] - Ax[:NN, :, :NN]) - (Az[:NN, :, 1:] - Az[:NN, :, :NN])
    bz = (Ay[:, :NN, 1:] - Ay[:, :NN, :NN]) - (Ax[:, 1:, :NN] - Ax[:, :NN, :NN])
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(N, N, N, G, 1, np.ones((1, 3)), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)[None]).to(dev)
    st = torch.zeros((1, abi.N_EVOL_VARS, NN, NN, NN), dtype=torch.float64, device=dev)
    fine = Fields(st, T(bx), T(by), T(bz))
    cb = Fields(st.clone(), *[torch.zeros_like(x) for x in (fine.bx, fine.by, fine.bz)])
    q = torch.zeros(1, dtype=torch.int64, device=dev)
    g.restrict_to_coarse(fine, cb, q, q)
    cx, cy, cz = (x[0].cpu().numpy() for x in (cb.bx, cb.by, cb.bz))
    h, s = N // 2, slice(G, G + N // 2)
    div = (cx[s, s, G + 1:G + h + 1] - cx[s, s, s]) + (cy[s, G + 1:G + h + 1, s] - cy[s, s, s]) + \
          (cz[G + 1:G + h + 1, s, s] - cz[s, s, s])
    assert np.max(np.abs(div)) < 1e-13
