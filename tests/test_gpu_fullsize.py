"""The benchmark's full size, 256^3 cells in 4096 blocks of 16^3, through
size-independent properties (the oracle's CPU step is out of reach here):
two SSP-RK3 steps of the blast wave, with periodic boundaries so that
nothing leaves the domain, in tuned mode with the static-metric cache.

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
