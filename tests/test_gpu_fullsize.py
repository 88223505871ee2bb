"""The benchmark's full size, 256^3 cells in 4096 blocks of 16^3: one
SSP-RK3 step of the benchmark's own configuration cell by cell against the
oracle, and, through size-independent properties, two steps of the blast
wave with periodic boundaries so that nothing leaves the domain, in tuned
mode with the static-metric cache:

* div B stays at round-off: CT keeps the discrete divergence of the face
  field, so BDIV on the interior is ~1e-16 of |B| / dx;
* mass: the sum of D over the interior is conserved to round-off (fluxes
  telescope on a periodic grid, FOFC corrections included), up to the
  density resets of the c2p, bounded by the |C2P_DENS_ERR| they recorded;
* every value stays finite and no fatal condition is raised."""
import pytest
import torch

from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, GRMHDEquationsSystem

pytestmark = pytest.mark.gpu

NB, N, G = 16, 16, 4


def _device_blast(blocks, dev, chunk=256):
    st = blocks.new_fields()
    aux = blocks.new_aux()
    su = None
    for q0 in range(0, blocks.nq, chunk):
        q1 = min(blocks.nq, q0 + chunk)
        su, (s, bx, by, bz, a) = workloads.blast(nb=(NB,) * 3, n=(N,) * 3, qr=(q0, q1))
        st.state[q0:q1].copy_(torch.from_numpy(s))
        st.bx[q0:q1].copy_(torch.from_numpy(bx))
        st.by[q0:q1].copy_(torch.from_numpy(by))
        st.bz[q0:q1].copy_(torch.from_numpy(bz))
        aux[q0:q1].copy_(torch.from_numpy(a))
    return su, st, aux


def test_blast_256cubed_two_steps_properties():
    dev = torch.device("cuda:0")
    su0 = workloads.BrickSetup((NB,) * 3, (N,) * 3, (-6, -6, -6), (6, 6, 6), G, (True, True, True))
    blocks = Blocks(N, N, N, G, su0.nq, su0.idx(), device=dev)
    P = params.blast()
    P.ranges = abi.RANGES_NEXT_STAGE  # the benchmark's aux and linop ranges
    g = GRMHDEquationsSystem(P)
    g.reserve(blocks)
    _, state, aux = _device_blast(blocks, dev)
    bc = lambda fl: g.fill_ghosts_brick(fl, su0.nb, su0.periodic)
    bc(state)
    g.set_mode(abi.MODE_TUNED)
    g.set_static_metric(state)
    g.compute_auxiliary_quantities(state, aux)
    sp, spp = state.clone(), state.clone()
    g.set_tuning(1, 1, 1, 1)
    sl = (slice(None), slice(G, G + N), slice(G, G + N), slice(G, G + N))
    mass0 = state.state[:, abi.DENS][sl].sum().item()
    resets = 0.0
    dt = 0.25 / su0.idx()[0, 0]
    for _ in range(2):
        g.rk3_step(dt, state, sp, spp, aux, bc)
        # rk3_step resets the diagnostics at its start: collect each step's
        resets += aux[:, abi.C2P_DENS_ERR][sl].abs().sum().item()
    torch.cuda.synchronize()
    assert g.status().device_flags == 0
    for x in (state.state[:, :abi.N_HRSC], state.bx, state.by, state.bz, aux[:, :abi.BDIV]):
        assert torch.isfinite(x).all()
    bmax = max(x.abs().max().item() for x in (state.bx, state.by, state.bz))
    bdiv = aux[:, abi.BDIV][sl].abs().max().item()
    assert bdiv * su0.dx[0] < 1e-13 * bmax, (bdiv, bmax)
    mass1 = state.state[:, abi.DENS][sl].sum().item()
    assert abs(mass1 - mass0) <= 1e-12 * abs(mass0) + resets, (mass0, mass1, resets)


def test_blast_256cubed_step_matches_oracle():
    """The benchmark's own configuration at its full size — 4096 blocks of
    16^3 on [-6, 6]^3 with outflow boundaries, tuned mode, next-stage ranges,
    the static-metric cache and the autotuner's picks — one SSP-RK3 step
    against the oracle (OpenMP on the host cores, ~30 s), cell by cell: the
    interior state within the step tolerance (state-normalised), face B
    within it relative to its largest value, C2P_ERR on every interior cell
    and the last substep's FOFC face and edge counts as the oracle's (up to
    a few threshold cases that FMA contraction may move)."""
    import numpy as np
    import _oracle
    from grace_b200.host import Fields
    from parity import cons_rel_err

    dev = torch.device("cuda:0")
    su, f = workloads.blast(nb=(NB,) * 3, n=(N,) * 3)
    assert su.nq == 4096 and not any(su.periodic)
    P = params.blast()
    P.ranges = abi.RANGES_NEXT_STAGE
    blocks = Blocks(N, N, N, G, su.nq, su.idx(), device=dev)
    g = GRMHDEquationsSystem(P)
    g.reserve(blocks)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(*[T(x) for x in f[:4]])
    aux = T(f[4])
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)
    bc(state)
    g.set_mode(abi.MODE_TUNED)
    g.set_static_metric(state)
    g.compute_auxiliary_quantities(state, aux)
    sp, spp = state.clone(), state.clone()
    g.autotune(sp, state, aux)
    dt = 0.25 / su.idx()[0, 0]
    g.rk3_step(dt, state, sp, spp, aux, bc)
    torch.cuda.synchronize()
    st = g.status()
    assert st.device_flags == 0
    sl = (slice(None), slice(None), slice(G, G + N), slice(G, G + N), slice(G, G + N))
    gcons = state.state[:, :abi.N_HRSC][sl].cpu().numpy()
    gfaces = [x.cpu().numpy() for x in (state.bx, state.by, state.bz)]
    gerr = aux[:, abi.C2P_ERR][sl[:1] + sl[2:]].cpu().numpy()
    del state, sp, spp, aux
    torch.cuda.empty_cache()
    # the oracle on the same initial data
    ost = [np.ascontiguousarray(x) for x in f[:4]]
    oaux = np.ascontiguousarray(f[4])
    del f
    S = _oracle.Stage(P, N, N, N, G, su.nq)
    _oracle.fill_ghosts("orc", su, ost)
    S.compute_aux(su.idx().copy(), ost, oaux)
    osp = [x.copy() for x in ost]
    ospp = [x.copy() for x in ost]
    _oracle.rk3_step(S, su, dt, ost, osp, ospp, oaux)
    of, oe = S.fofc_counts()
    e = cons_rel_err(gcons, ost[0][:, :abi.N_HRSC][sl])
    assert e.max() < 1e-10, e
    for a, b in zip(gfaces, ost[1:]):
        assert np.max(np.abs(a - b)) < 1e-10 * np.max(np.abs(b))
    oerr = oaux[:, abi.C2P_ERR][sl[:1] + sl[2:]]
    mismatch = int(np.count_nonzero(gerr != oerr))
    assert mismatch <= 1e-6 * gerr.size, mismatch
    assert abs(st.fofc_faces - of) <= max(2, 1e-4 * of), (st.fofc_faces, of)
    assert abs(st.fofc_edges - oe) <= max(2, 1e-4 * oe), (st.fofc_edges, oe)
