#!/usr/bin/env python
"""Benchmark: GRMHD zone-updates/s per RK stage on the 3-D blast wave.

Workload: 256^3 cells in 4096 blocks of 16^3 (4 ghost layers), ideal gas
Gamma=4/3, WENO-Z + HLLE + Gardiner-Stone CT + FOFC, SSP-RK3, flat Cowling
metric, seeded synthetic initial data.  One step = one full RK3 step (three
stages, each advance_substep + ghost fill + c2p/aux), so
value = interior cells x 3 x steps / time.  Inputs (the block arrays, ~60 GB
with scratch) are far larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N>1: one process per GPU (torchrun), each rank advances its own copy of the
workload (weak scaling, no collective in the data path); time = max over
ranks of the device-timed region.  `--impl reference` times the CPU
reference numerics (oracle/_ref: GRACE's own per-cell functions compiled in
place, driven by the restated loop drivers) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

# algorithmic FP64 bytes per item of each kernel kind (unique array
# footprint the kernel must touch; see the design notes for the accounting)
ALGO_BYTES = {
    # per face: 10 reconstructed aux vars + 10 metric comps + face B read
    # per cell crossed, 7 fluxes + 2 face EMFs written
    "flux": 8 * (10 + 10 + 1 + 9),
    # per cell incl. ghosts: 7 cons + 3 face B + 10 metric + C2P_ERR read;
    # 12 aux + C2P_ERR + 3 E_centre + ENTROPYSTAR written
    "aux": 8 * (7 + 3 + 10 + 1 + 12 + 1 + 3 + 1),
    # per interior cell: 21 face fluxes, 9 aux, 16 metric/curvature, 7 cons RMW
    "update": 8 * (21 + 9 + 16 + 14),
}
# Per-item counts of the tuned step measured by ncu on 64 blocks of the same
# workload (profiles/step_dram_fp64_blast64blocks.md: one RK3 step between
# cudaProfilerStart/Stop, every launch, cold L2 per kernel), scaled to a full
# launch by the items it computes:
#   the TMA-staged flux kernel (mean of the three directions), per face:
FLUX_DRAM_BYTES_PER_FACE = 312.1      # dram__bytes_read.sum + dram__bytes_write.sum
FLUX_FP64_FLOP_PER_FACE = 2234.7      # dadd + dmul + 2 dfma (thread instructions)
FLUX_FP64_INST_PER_FACE = 1684.0      # dadd + dmul + dfma
#   the whole RK3 step (54 launches), per zone-update:
STEP_DRAM_BYTES_PER_ZU = 4661.4
STEP_FP64_FLOP_PER_ZU = 15871.2
STEP_FP64_INST_PER_ZU = 11460.3
# algorithmic FP64 bytes per zone-update: 66 doubles on RK3 stage 1, 76 on
# stages 2 and 3 (they also read the u^n combination), 581 B averaged
ALGO_BYTES_PER_ZU = 581.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nb", type=int, default=16, help="blocks per axis")
    ap.add_argument("--n", type=int, default=16, help="cells per block per axis")
    ap.add_argument("--cfl", type=float, default=0.25)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--eager", action="store_true", help="launch the timed steps eagerly, not as a CUDA graph")
    ap.add_argument("--no-c2p", action="store_true")
    ap.add_argument("--no-restrict", action="store_true", help="skip the FMR restriction and prolongation measurements")
    ap.add_argument("--no-learned", action="store_true", help="c2p leg: plain bracket only")
    ap.add_argument("--c2p-only", action="store_true", help="run only the c2p micro-benchmark")
    ap.add_argument("--c2p-states", type=int, default=1 << 24, help="states of the c2p micro-benchmark")
    ap.add_argument("--mode", default="tuned", choices=["tuned", "plain"])
    ap.add_argument("--config", default="blast", choices=["blast", "tov", "torus"],
                    help="blast: the 256^3 blast wave (the headline); tov, torus: the magnetised TOV star and the "
                         "Fishbone-Moncrief torus on their FMR hierarchies (16^3 blocks, refluxing, gather-map "
                         "ghost fill)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form comparison run")
    ap.add_argument("--e2e-runs", type=int, default=8,
                    help="end-to-end leg: runs of blocks the host step pipelines over (1: no pipeline)")
    ap.add_argument("--ref-blocks", type=int, default=8,
                    help="reference arm: blocks per axis of the CPU sample (the central ones; --nb for the whole grid)")
    ap.add_argument("--profile-step", action="store_true",
                    help="after the warm-up, run one eager RK3 step between cudaProfilerStart/Stop and exit "
                         "(for ncu --profile-from-start off)")
    ap.add_argument("--tuning", default="", help="kernel variants flux,fofc_flag,update,aux (grb_set_tuning) "
                    "instead of the autotuner, e.g. 1,1,0,2")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.idx)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[0]) for r in self.rows if len(r) >= 8 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 8 for k in range(4)
                          if r[4 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(sm)}


# ---------------------------------------------------------------------------
def _workload_config(nb, n):
    """The bench line's config (both arms print the same one)."""
    return {"workload": f"blast wave {nb * n}^3 ({nb ** 3} blocks of {n}^3), Gamma=4/3, "
                        "WENO-Z+HLLE+GS CT+FOFC, SSP-RK3",
            "blocks": nb ** 3, "cells_per_block": n ** 3, "ngz": 4,
            "l2": "inputs larger than L2 (no flush)"}


class CpuReference:
    """RK3 steps of the blast wave on the CPU with the reference numerics
    (oracle/_ref: GRACE's own per-cell functions compiled in place, driven by
    the restated loops with OpenMP over blocks), or the oracle's port when
    the pinning build is absent.  Bounded sample of the workload: the central
    nb_side^3 blocks of the full grid (same cell size, same initial data),
    with zero-gradient ghosts at the sample's faces."""

    def __init__(self, nb_side, n, cfl):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import _oracle
        from grace_b200 import params, workloads
        self.o = _oracle
        self.which, self.kind = "ref", "reference"
        if _oracle.lib("ref") is None:
            self.which, self.kind = "orc", "port"
        half = 6.0 * nb_side / 16.0 * (n / 16.0) * 16.0 / n
        self.su, f = workloads.blast(nb=(nb_side,) * 3, n=(n, n, n), lo=(-half,) * 3, hi=(half,) * 3)
        P = params.blast()
        st, bx, by, bz, self.aux = [x.copy() for x in f]
        self.S = _oracle.Stage(P, n, n, n, self.su.ngz, self.su.nq, self.which)
        self.state = [st, bx, by, bz]
        _oracle.fill_ghosts(self.which, self.su, self.state)
        self.S.compute_aux(self.su.idx().copy(), self.state, self.aux)
        self.sp = [x.copy() for x in self.state]
        self.spp = [x.copy() for x in self.state]
        self.dt = cfl / self.su.idx()[0, 0]
        self.zones_per_step = self.su.nq * n ** 3 * 3
        self.cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        self.nb_side, self.n = nb_side, n

    def step(self):
        self.o.rk3_step(self.S, self.su, self.dt, self.state, self.sp, self.spp, self.aux, self.which)

    def sample(self):
        return (f"each step: one RK3 step of the blast wave on the central {self.nb_side}^3 blocks of "
                f"{self.n}^3 cells of the same grid (same cell size and initial data), {self.kind} numerics, "
                f"OpenMP over blocks on {self.cores} threads")


def cpu_reference_run(nb_side, n, cfl, min_s=10.0):
    """zone-updates/s of RK3 steps on the CPU sample (at least one step and
    min_s seconds); returns (rate, cores, kind, sample description)."""
    R = CpuReference(nb_side, n, cfl)
    done = 0
    t0 = time.perf_counter()
    while done < 1 or time.perf_counter() - t0 < min_s:
        R.step()
        done += 1
    el = time.perf_counter() - t0
    return R.zones_per_step * done / el, R.cores, R.kind, R.sample().replace("each step: one", f"{done}")


def reference_arm(args, rank):
    """The CPU reference on the host cores, rank 0 only: W warm-up and K
    timed steps, each one RK3 step of the bounded sample (by default the
    central 8^3 of the 16^3 blocks: an eighth of the workload, ~3 s per step
    on 16 threads, so that the whole run takes a couple of minutes;
    --ref-blocks 16 steps the whole grid)."""
    if rank != 0:
        return
    R = CpuReference(min(args.ref_blocks, args.nb), args.n, args.cfl)
    for _ in range(args.warmup):
        R.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        R.step()
    el = time.perf_counter() - t0
    value = R.zones_per_step * args.steps / el
    line = {
        "impl": "reference", "metric": "GRMHD zone-updates/s per RK stage", "value": value,
        "unit": "zone-updates/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded blast-wave initial data)",
        "config": _workload_config(args.nb, args.n),
        "cpu_baseline": {"value": value, "unit": "zone-updates/s", "cores": R.cores, "kind": R.kind,
                         "sample": R.sample()},
        "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def build_blast_on_device(blocks, su, nb, n, dev, torch, fields_cls, chunk=256):
    from grace_b200 import workloads
    st = blocks.new_fields()
    aux = blocks.new_aux()
    for q0 in range(0, su.nq, chunk):
        q1 = min(su.nq, q0 + chunk)
        _, (s, bx, by, bz, a) = workloads.blast(nb=(nb,) * 3, n=(n,) * 3, qr=(q0, q1))
        st.state[q0:q1].copy_(torch.from_numpy(s))
        st.bx[q0:q1].copy_(torch.from_numpy(bx))
        st.by[q0:q1].copy_(torch.from_numpy(by))
        st.bz[q0:q1].copy_(torch.from_numpy(bz))
        aux[q0:q1].copy_(torch.from_numpy(a))
    return st, aux


def _brick_pipeline(g, su, nruns):
    """(runs, fill_run, deps) of rk3_step_host for the brick: runs of whole
    z-slabs of blocks, each filled by the block-range brick fill."""
    from grace_b200.host import brick_runs
    runs, deps = brick_runs(su.nb, su.periodic, nruns)
    fill_run = lambda f, s, stream: g.fill_ghosts_brick(f, su.nb, su.periodic, stream=stream, blocks=runs[s])
    return runs, fill_run, deps, False


def _gather_pipeline(g, maps, blocks, nruns):
    """(runs, fill_run, deps, whole_grid_substeps) of rk3_step_host for an
    FMR hierarchy: runs of consecutive blocks, each filled by its part of the
    gather maps; the substeps stay on the whole grid (refluxing couples the
    runs)."""
    from grace_b200.host import gather_runs
    runs, run_maps, deps = gather_runs(maps, blocks, nruns)
    fill_run = lambda f, s, stream: g.fill_ghosts_gather(f, run_maps[s], stream=stream)
    return runs, fill_run, deps, True


def make_workload(args, dev):
    """The timed workload: blocks, parameters, a device-field builder, the
    ghost fill between stages, the bench line's config and data strings and
    the CPU-reference sample."""
    import torch
    from grace_b200 import abi, params, workloads
    from grace_b200.host import Blocks, Fields
    nb, n = args.nb, args.n
    if args.config == "blast":
        su = workloads.BrickSetup((nb,) * 3, (n,) * 3, (-6,) * 3, (6,) * 3, 4, (False,) * 3)
        blocks = Blocks(n, n, n, 4, su.nq, su.idx(), device=dev)
        return {"blocks": blocks, "params": params.blast(), "idx": su.idx(),
                "fields": lambda g: build_blast_on_device(blocks, su, nb, n, dev, torch, Fields),
                "bc": lambda g: (lambda f: g.fill_ghosts_brick(f, su.nb, su.periodic)),
                "runs": lambda g, nruns: _brick_pipeline(g, su, nruns),
                "config": _workload_config(nb, n), "data": "synthetic (seeded blast-wave initial data)",
                "cpu": lambda: cpu_reference_run(8 if nb >= 8 else nb, n, args.cfl, min_s=10.0)}
    if args.config == "tov":
        H = workloads.tov_hierarchy(n)
        (f, _), P = workloads.magnetised_tov(H), params.tov()
        desc = (f"magnetised TOV star (K=100, Gamma=2, rho_c=1.28e-3; hybrid EOS Gamma_th=1.8; poloidal field "
                f"max|B|=1e-4) in Cowling, +-48, {H.nq} blocks of {n}^3 on 5 FMR levels "
                f"({'/'.join(str(c) for c in H.level_counts())}), WENO-Z+HLLE+GS CT+FOFC, refluxing, SSP-RK3")
        data = "synthetic (TOV solution of the polytrope with seeded 1e-3 density noise)"
    else:
        H = workloads.torus_hierarchy(n)
        f, P = workloads.fm_torus(H), params.torus()
        desc = (f"Fishbone-Moncrief torus (a=0.9375, r_in=6, r_pmax=12, Gamma=4/3, beta=100) in fixed Kerr-Schild, "
                f"+-40, {H.nq} blocks of {n}^3 on 4 FMR levels ({'/'.join(str(c) for c in H.level_counts())}), "
                "WENO-Z+HLLE+GS CT+FOFC, refluxing, SSP-RK3")
        data = "synthetic (Fishbone-Moncrief equilibrium with seeded 2% pressure and 0.1% density noise)"
    st, bx, by, bz, aux = f
    H.fill_ghosts(st, bx, by, bz)
    maps, R = H.gather_maps(), H.reflux_lists()
    blocks = Blocks(n, n, n, H.ngz, H.nq, H.idx(), device=dev)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    def fields(g):
        g.set_reflux(R)
        return Fields(T(st), T(bx), T(by), T(bz)), T(aux)

    def cpu():
        # one RK3 step of the whole hierarchy with the reference numerics
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import _oracle
        which, kind = ("ref", "reference") if _oracle.lib("ref") is not None else ("orc", "port")
        S = _oracle.Stage(P, n, n, n, H.ngz, H.nq, which)
        S.set_reflux(R)
        idx = H.idx()
        state = [x.copy() for x in (st, bx, by, bz)]
        a = aux.copy()
        S.compute_aux(idx.copy(), state, a)
        sp, spp = [x.copy() for x in state], [x.copy() for x in state]
        dt = args.cfl / idx[:, 0].max()
        t0 = time.perf_counter()
        S.reset_diag(a)
        for st_out, st_in, fac, comb in ((sp, state, 1.0, None), (spp, sp, 0.25, (0.75, 0.25)),
                                         (state, spp, 2.0 / 3.0, (1.0 / 3.0, 2.0 / 3.0))):
            if comb is not None:
                S.linop(st_out, state, st_in, *comb)
            S.advance_substep(idx.copy(), dt, fac, st_out, st_in, a)
            H.fill_ghosts(*st_out)
            S.compute_aux(idx.copy(), st_out, a)
        el = time.perf_counter() - t0
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        return (H.nq * n ** 3 * 3 / el, cores, kind,
                f"one RK3 step of the whole hierarchy ({H.nq} blocks) with refluxing and the host ghost fill, "
                f"{kind} numerics, OpenMP over blocks on {cores} threads")

    return {"blocks": blocks, "params": P, "idx": H.idx(), "fields": fields,
            "bc": lambda g: (lambda fl: g.fill_ghosts_gather(fl, maps)),
            "runs": lambda g, nruns: _gather_pipeline(g, maps, blocks, nruns),
            "config": {"workload": desc, "blocks": H.nq, "cells_per_block": n ** 3, "ngz": H.ngz,
                       "l2": "inputs larger than L2 (no flush)"}, "data": data, "cpu": cpu}


def ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from grace_b200 import abi, params, workloads
    from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    nb, n = args.nb, args.n
    W = make_workload(args, dev)
    blocks, P, nq = W["blocks"], W["params"], W["blocks"].nq
    if args.mode == "tuned":
        # aux pass and linop on the cells the next stage reads (the stage's
        # own ghost exchange refills the rest every substep)
        P.ranges = abi.RANGES_NEXT_STAGE
    g = GRMHDEquationsSystem(P)
    g.reserve(blocks)
    state, aux = W["fields"](g)
    bc = W["bc"](g)
    bc(state)
    g.compute_auxiliary_quantities(state, aux)
    sp, spp = state.clone(), state.clone()
    idx_h = W["idx"]
    dt = args.cfl / idx_h[:, 0].max()
    tuning = None
    if args.mode == "tuned":
        g.set_mode(abi.MODE_TUNED)
        # Cowling: the metric is static, its derivatives are taken once
        g.set_static_metric(state)
        if args.tuning:
            g.set_tuning(*[int(x) for x in args.tuning.split(",")])
            tuning = g.tuning()
        else:
            tuning = g.autotune(sp, state, aux)

    def barrier():
        if world > 1:
            dist.barrier()

    # each step also reduces the next stable time step (find_stable_timestep,
    # fused into the last aux pass); the bench keeps dt fixed
    dx_d = torch.from_numpy(np.ascontiguousarray(1.0 / idx_h)).to(dev)
    dt_next = torch.zeros(1, dtype=torch.float64, device=dev)
    nd = (dx_d, args.cfl, dt_next)
    # warm-up: eager steps (one with the dt reduction fused into the last aux
    # pass, one with it as a separate pass: the faster form is kept), then the
    # step captured as one CUDA graph
    for _ in range(max(1, args.warmup - 3)):
        g.rk3_step(dt, state, sp, spp, aux, bc, next_dt=nd)

    def step_ms(fused):
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        g.rk3_step(dt, state, sp, spp, aux, bc, next_dt=nd, fused_dt=fused)
        a1.record()
        torch.cuda.synchronize()
        return a0.elapsed_time(a1)

    dt_pass = {"separate_step_ms": step_ms(False), "fused_step_ms": step_ms(True)}
    fused = dt_pass["fused_step_ms"] < dt_pass["separate_step_ms"]
    dt_pass["used"] = "fused" if fused else "separate"
    if args.profile_step:
        # one eager step between profiler start and stop (for ncu
        # --profile-from-start off): the launch list of exactly one step
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        g.rk3_step(dt, state, sp, spp, aux, bc, next_dt=nd, fused_dt=fused)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        if rank == 0:
            print(json.dumps({"profile_step": True, "blocks": nq, "cells_per_block": n ** 3,
                              "zone_updates": nq * n ** 3 * 3, "tuning": tuning}), flush=True)
        g.close()
        return
    graph, per_step = None, None
    if not args.eager:
        graph, per_step = g.capture_rk3_step(dt, state, sp, spp, aux, bc, next_dt=nd, fused_dt=fused)
        graph.replay()
    else:
        g.rk3_step(dt, state, sp, spp, aux, bc, next_dt=nd, fused_dt=fused)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    st0 = g.status()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        if graph is not None:
            graph.replay()
        else:
            g.rk3_step(dt, state, sp, spp, aux, bc, next_dt=nd, fused_dt=fused)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    st1 = g.status()
    launches = per_step * args.steps if graph is not None else st1.launches - st0.launches
    # per-kernel device times: one more eager step with event timing
    g.set_kernel_timing(True)
    g.rk3_step(dt, state, sp, spp, aux, bc, next_dt=nd, fused_dt=fused)
    torch.cuda.synchronize()
    kt = g.kernel_times()
    g.set_kernel_timing(False)
    kt = {k: (v[0] * args.steps, v[1] * args.steps) for k, v in kt.items()}
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    zu_rank = nq * n ** 3 * 3 * args.steps
    value = zu_rank * world / (ms * 1e-3)

    # --- the plain per-item form on the same state, for the speed-up ratio
    plain = None
    if args.mode == "tuned" and not args.no_plain:
        g.set_mode(abi.MODE_PLAIN)
        g.rk3_step(dt, state, sp, spp, aux, bc)
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        psteps = max(1, min(args.steps, 2))
        p0.record()
        for _ in range(psteps):
            g.rk3_step(dt, state, sp, spp, aux, bc)
        p1.record()
        torch.cuda.synchronize()
        pv = nq * n ** 3 * 3 * psteps / (p0.elapsed_time(p1) * 1e-3)
        plain = {"value": pv, "steps": psteps, "speedup_tuned_over_plain": (value / world) / pv}
        g.set_mode(abi.MODE_TUNED)

    # --- end to end: evolved variables from / to pinned host memory each step
    e2e = None
    if not args.no_e2e:
        host = g.packed_host_fields()
        g.copy_evolved_packed(host, state, to_device=False)
        ksteps = max(1, min(args.steps, 20))
        # the pipeline's runs and per-run fills set up (and their first-use
        # uploads made) before the timed region
        pipe = W["runs"](g, args.e2e_runs) if ("runs" in W and args.e2e_runs > 1) else None
        if pipe is not None:
            for r in range(len(pipe[0])):
                pipe[1](state, r, torch.cuda.current_stream())
        io = (torch.cuda.Stream(), torch.cuda.Stream())
        torch.cuda.synchronize()
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record()
        # face B is final after the last substep: its download runs on a
        # second stream while the boundary fill and the aux pass finish the
        # cell variables
        main = torch.cuda.current_stream()
        side = torch.cuda.Stream()
        faces_only, cells_only = (False, True, True, True), (True, False, False, False)

        def download_faces():
            side.wait_stream(main)
            g.copy_evolved_packed(host, state, to_device=False, stream=side, arrays=faces_only)

        prev = None
        for _ in range(ksteps):
            if pipe is not None:
                runs, fill_run, deps, whole = pipe
                prev = g.rk3_step_host(dt, host, state, sp, spp, aux, bc, runs, fill_run, deps, streams=io,
                                       after=prev, wait=False, whole_grid_substeps=whole)
                continue
            main.wait_stream(side)
            g.copy_evolved_packed(host, state, to_device=True)
            bc(state)
            g.compute_auxiliary_quantities(state, aux)
            g.linop_apply(sp, state, None, 1.0, 0.0)
            g.rk3_step(dt, state, sp, spp, aux, bc, after_update=download_faces)
            g.copy_evolved_packed(host, state, to_device=False, arrays=cells_only)
        main.wait_stream(side)
        main.wait_stream(io[1])
        f1.record()
        torch.cuda.synchronize()
        ems = f0.elapsed_time(f1)
        if world > 1:
            t = torch.tensor([ems], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        nx = ny = nz = n
        nbytes = 8 * nq * (abi.N_HRSC * nx * ny * nz + (nx + 1) * ny * nz + nx * (ny + 1) * nz +
                              nx * ny * (nz + 1))
        e2e = {"value": nq * n ** 3 * 3 * ksteps * world / (ems * 1e-3), "unit": "zone-updates/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": ksteps,
               "note": "interior of the evolved variables (7 HRSC + face B) copied between packed pinned host "
                       "arrays and the device every step (grb_copy_evolved_packed: one DMA copy per array "
                       "through a device staging buffer); each step refills the ghost zones and recomputes the "
                       "primitives of the uploaded state first"}
        if pipe is not None:
            e2e["pipeline"] = (f"GRMHDEquationsSystem.rk3_step_host over {len(pipe[0])} runs of blocks: "
                               + ("each run's upload overlaps the fill and primitives pass of the runs before it, its "
                                  "download the primitives pass of the runs after it, the substeps on the whole grid "
                                  "(refluxing couples the runs); " if pipe[3] else
                                  "each run's upload overlaps the first substep of the runs before it, its download "
                                  "the last substep of the runs after it; ") +
                               "upload, kernels, download on three streams; "
                               "a step's upload of a run waits only for the previous step's download of that run, so "
                               "it overlaps the previous step's tail; the timed region ends after the last "
                               "step's downloads")
        else:
            e2e["pipeline"] = ("none: upload, refill, primitives, rk3_step, download in sequence (face B downloaded "
                               "on a second stream once the last substep has made it final)")

    # --- FMR restriction into coarse buffers (a separate measurement, not
    # part of the step): every block restricted into a buffer, the 7 HRSC
    # variables by the 8-cell average, the 16 metric and curvature variables
    # by the 5-point Lagrange operator, and the three face-B arrays
    restrict = None
    if not args.no_restrict and args.mode == "tuned" and args.config == "blast":
        qs = torch.arange(nq, dtype=torch.int64, device=dev)
        ch = (qs % 8).to(torch.uint8)
        lo, hi = list(range(abi.N_HRSC)), list(range(abi.N_HRSC, abi.N_EVOL_VARS))
        run = lambda: g.restrict_to_coarse(state, spp, qs, qs, ch, lo, hi)
        for _ in range(2):
            run()
        torch.cuda.synchronize()
        r0 = torch.cuda.Event(enable_timing=True)
        r1 = torch.cuda.Event(enable_timing=True)
        reps = 5
        r0.record()
        for _ in range(reps):
            run()
        r1.record()
        torch.cuda.synchronize()
        rms = r0.elapsed_time(r1) / reps
        # algorithmic bytes: fine interior read once, coarse interior written
        cells, ccells = n ** 3, (n // 2) ** 3
        fcells = (n + 1) * n * n
        cfaces = (n // 2 + 1) * (n // 2) ** 2
        rbytes = 8 * nq * (abi.N_EVOL_VARS * (cells + ccells) + 3 * (fcells + cfaces))
        restrict = {"quads": nq, "ms": rms, "fine_cells_per_s": nq * cells / (rms * 1e-3),
                    "achieved_GBps": rbytes / (rms * 1e-3) / 1e9,
                    "note": "23 state variables (7 by the 8-cell average, 16 by the 5-point Lagrange "
                            "restriction) and the three face-B arrays of every block; bytes = the fine "
                            "interior read once plus the coarse image written"}

    # --- FMR prolongation into ghost zones (a separate measurement, not part
    # of the step): all 26 ghost elements (6 faces, 12 edges, 8 corners) of
    # every block filled from a coarse buffer, the 7 HRSC variables by the
    # minmod slope-limited operator, the 16 others by the 5-point Lagrange
    # one, face B by the divergence-preserving prolongation; the bench's
    # state serves as the coarse buffers and a scratch copy as the fine blocks
    prolong = None
    if not args.no_restrict and args.mode == "tuned" and args.config == "blast":
        lo, hi = list(range(abi.N_HRSC)), list(range(abi.N_HRSC, abi.N_EVOL_VARS))
        lists = []
        for kind, ne in ((0, 6), (1, 12), (2, 8)):
            fq = torch.arange(nq, dtype=torch.int64, device=dev).repeat_interleave(ne)
            el = torch.arange(ne, dtype=torch.uint8, device=dev).repeat(nq)
            hf = torch.zeros((nq * ne, 3, 2), dtype=torch.int8, device=dev)
            lists.append((kind, fq, el, hf))
        run = lambda: [g.prolong_to_ghosts(spp, state, k, fq, fq, el, hf, lo, hi) for k, fq, el, hf in lists]
        for _ in range(2):
            run()
        torch.cuda.synchronize()
        r0 = torch.cuda.Event(enable_timing=True)
        r1 = torch.cuda.Event(enable_timing=True)
        reps = 5
        r0.record()
        for _ in range(reps):
            run()
        r1.record()
        torch.cuda.synchronize()
        pms = r0.elapsed_time(r1) / reps
        # algorithmic bytes: the fine ghost cells (and one face per ghost cell
        # and array) written once, the coarse cells and faces covering them
        # read once (1/8 and 1/4 as many)
        NN = n + 2 * 4
        vg = NN ** 3 - n ** 3
        pbytes = 8 * nq * (abi.N_EVOL_VARS * (vg + vg / 8) + 3 * (vg + vg / 4))
        prolong = {"quads": nq, "ms": pms, "ghost_cells_per_s": nq * vg / (pms * 1e-3),
                   "achieved_GBps": pbytes / (pms * 1e-3) / 1e9, "launches": 12,
                   "note": "26 ghost elements of every block (3 calls, one per element kind): 23 state "
                           "variables (7 slope-limited, 16 by the 5-point Lagrange prolongation) and the "
                           "three face-B arrays; bytes = the fine ghost region written once plus the coarse "
                           "data covering it read once"}

    # --- FP64 throughput of this GPU (the FP64 roofline's denominator)
    import ctypes
    from grace_b200 import _lib
    fp64_tf, fp64_ms = ctypes.c_double(), ctypes.c_double()
    _lib.check(_lib.load().grb_measure_fp64_peak(ctypes.byref(fp64_tf), ctypes.byref(fp64_ms),
                                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
               "grb_measure_fp64_peak")
    fp64_peak = {"tflops": fp64_tf.value, "launch_ms": fp64_ms.value,
                 "how": "grb_measure_fp64_peak: 8 independent FMA chains per thread, 8 CTAs x 256 threads per "
                        "SM, best of 5, CUDA events"}

    # --- dominant kernel roofline (HBM), measured over the timed region
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    for leg in (restrict, prolong):
        if leg is not None:
            leg["hbm_frac"] = leg["achieved_GBps"] / hbm
            leg["peak_source"] = peak_src
    top = max(kt.items(), key=lambda kv: kv[1][0])
    name, (kms, kcnt) = top
    # faces one flux launch (one direction) computes: the reference's full
    # transverse ghost range in the plain form, only the faces the stage
    # reads in the tuned form (GS: n+2 transverse, UCT: n+6)
    tr = (n + 8) if args.mode != "tuned" else ((n + 2) if P.emf == abi.EMF_GS else (n + 6))
    items = {
        "flux": nq * (n + 3) * tr ** 2,
        "aux": nq * (n + 8) ** 3,
        "update": nq * n ** 3,
    }
    roof = None
    if name in ALGO_BYTES and kcnt:
        bytes_per_launch = ALGO_BYTES[name] * items[name]
        per_launch_ms = kms / kcnt
        ach = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
        traffic = FLUX_DRAM_BYTES_PER_FACE * items[name] if (name == "flux" and args.mode == "tuned") else None
        roof = {"bound": "hbm", "kernel": name, "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "peak_source": peak_src, "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_per_launch, "items_per_launch": items[name],
                "launch_ms": per_launch_ms}
        if name == "flux" and args.mode == "tuned":
            # the FP64 roofline of the same launches: flops and FP64
            # instructions per face from ncu, time from the events above,
            # against the FMA throughput measured on this GPU (2 flops or 1
            # instruction per lane per clock)
            fl = FLUX_FP64_FLOP_PER_FACE * items[name] / (per_launch_ms * 1e-3) / 1e12
            ins = FLUX_FP64_INST_PER_FACE * items[name] / (per_launch_ms * 1e-3) / 1e12
            roof["fp64"] = {"achieved": fl, "peak": fp64_peak["tflops"], "unit": "TFLOP/s",
                            "frac": fl / fp64_peak["tflops"],
                            "issue_frac": ins / (fp64_peak["tflops"] / 2.0),
                            "flop_per_face": FLUX_FP64_FLOP_PER_FACE, "inst_per_face": FLUX_FP64_INST_PER_FACE,
                            "peak_source": "measured (grb_measure_fp64_peak)"}
            roof["binding"] = (f"FP64 pipe: its FP64 instructions issue at {roof['fp64']['issue_frac']:.0%} of the "
                               f"measured FMA rate ({roof['fp64']['frac']:.0%} in flops: DADD/DMUL count one flop "
                               f"an issue), HBM at {ach / hbm:.0%}")
        # the whole step against both rooflines
        zu_s = value / world
        roof_step = {
            "algorithmic_bytes_per_zone_update": ALGO_BYTES_PER_ZU,
            "dram_bytes_per_zone_update": STEP_DRAM_BYTES_PER_ZU,
            "fp64_flop_per_zone_update": STEP_FP64_FLOP_PER_ZU,
            "hbm_frac_algorithmic": ALGO_BYTES_PER_ZU * zu_s / 1e9 / hbm,
            "hbm_frac_dram": STEP_DRAM_BYTES_PER_ZU * zu_s / 1e9 / hbm,
            "fp64_frac": STEP_FP64_FLOP_PER_ZU * zu_s / 1e12 / fp64_peak["tflops"],
            "fp64_issue_frac": STEP_FP64_INST_PER_ZU * zu_s / 1e12 / (fp64_peak["tflops"] / 2.0),
            "source": "per-zone-update counts of one tuned RK3 step on 64 blocks (ncu), rates of this run"}
        roof["step"] = roof_step

    # --- c2p micro-benchmark (2^24 states): plain, then with the learned
    # bracket trained on the GPU from 2^20 other seeded states
    c2p = None
    if not args.no_c2p and rank == 0:
        if args.config == "blast":
            c2p = c2p_bench(dev, learned=not args.no_learned)
        else:
            # the configuration's own cells after the timed steps: the c2p
            # with and without the learned bracket on the states it meets
            c2p = c2p_bench(dev, learned=not args.no_learned, states=_cell_states(torch, abi, state, blocks),
                            P=P)
            c2p["states_from"] = "every interior cell of the configuration after the timed steps"

    cpu = None
    if rank == 0 and not args.no_cpu and world == 1:
        v, cores, kind, sample = W["cpu"]()
        cpu = {"value": v, "unit": "zone-updates/s", "cores": cores, "kind": kind, "sample": sample}

    if rank == 0:
        line = {
            "metric": "GRMHD zone-updates/s per RK stage", "value": value, "unit": "zone-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": W["data"],
            "config": W["config"],
            "run": {"parallelism": f"replicas x{world}",
                       "launch": "cuda_graph" if graph is not None else "eager",
                       "step": "3 x (advance_substep + ghost fill + aux) + linops; the last aux pass "
                               "also reduces the next stable dt (dt itself held fixed)",
                       "next_dt": float(dt_next.item()), "dt_pass": dt_pass,
                       "static_metric": "metric derivatives cached once (Cowling)" if args.mode == "tuned"
                       else "metric differentiated every stage"},
            "clocks": clk, "gpu_launches": launches,
            "kernel_ms": {k: round(v[0], 3) for k, v in kt.items() if v[1]},
            "roofline": roof, "fp64_peak": fp64_peak, "e2e": e2e, "cpu_baseline": cpu, "c2p": c2p,
            "mode": args.mode, "plain_form": plain, "tuning": tuning, "restrict": restrict, "prolong": prolong,
        }
        print(json.dumps(line), flush=True)
    g.close()


def _cell_states(torch, abi, f, blocks):
    """(cons (10, n), metric (10, n)) of every interior cell of device
    Fields f: the 7 HRSC variables, the cell-centred B (means of the face
    pairs), the 3-metric, shift and lapse."""
    g, n = blocks.ngz, blocks.nx
    i = slice(g, g + n)
    st = f.state
    cons = torch.empty(10, blocks.nq, n, n, n, dtype=torch.float64, device=st.device)
    cons[:abi.N_HRSC] = st[:, :abi.N_HRSC, i, i, i].permute(1, 0, 2, 3, 4)
    cons[7] = 0.5 * (f.bx[:, i, i, g:g + n] + f.bx[:, i, i, g + 1:g + n + 1])
    cons[8] = 0.5 * (f.by[:, i, g:g + n, i] + f.by[:, i, g + 1:g + n + 1, i])
    cons[9] = 0.5 * (f.bz[:, g:g + n, i, i] + f.bz[:, g + 1:g + n + 1, i, i])
    met = torch.empty(10, blocks.nq, n, n, n, dtype=torch.float64, device=st.device)
    met[:6] = st[:, abi.GXX:abi.GXX + 6, i, i, i].permute(1, 0, 2, 3, 4)
    met[6:9] = st[:, abi.BETAX:abi.BETAX + 3, i, i, i].permute(1, 0, 2, 3, 4)
    met[9] = st[:, abi.ALP, i, i, i]
    return cons.reshape(10, -1).contiguous(), met.reshape(10, -1).contiguous()


def _c2p_agreement(torch, pr_a, pr_p):
    """State-normalised residual of primitives against the plain c2p's: the
    largest, its ratio to the bound 1e-12 max(1, W^2) (Brent's absolute
    window in mu amplified by W^2; the plain solver restarted from another
    bracket moves the same states as much), and the fraction within a
    flat 1e-12."""
    W = torch.sqrt(1.0 + (pr_p[2:5] ** 2).sum(0))
    scale = torch.maximum(torch.maximum(pr_p[0].abs(), pr_p[7].abs()),
                          torch.sqrt((pr_p[2:5] ** 2).sum(0)).clamp_min(1e-30))
    d = torch.stack([(pr_a[v] - pr_p[v]).abs() for v in (0, 7, 2, 3, 4)]).max(0).values / scale
    ok = torch.isfinite(d)
    return {"max_state_residual": float(d[ok].max()),
            "max_residual_over_W2_tol": float((d[ok] / (1e-12 * torch.clamp(W[ok] ** 2, min=1.0))).max()),
            "frac_within_1e-12": float((d[ok] <= 1e-12).double().mean())}


def c2p_bench(dev, learned=True, n=1 << 24, reps=5, states=None, P=None):
    """c2p solves/s, plain / tuned / learned bracket / learned + tuned, with
    the agreement of each with the plain solve.  Default: the 2^24 seeded
    states of the c2p workload (flat metric), the network trained on 2^20
    other seeded states.  states = (cons (10, n), metric (10, n)) device
    tensors and P their parameters: those states (a configuration's own
    cells), the network trained on 2^20 of them picked at random."""
    import torch
    from grace_b200 import abi, params, workloads
    from grace_b200.host import GRMHDEquationsSystem
    if states is None:
        cons, _ = workloads.c2p_states(n, seed=5)
        gc = GRMHDEquationsSystem(params.c2p_bench())
        c_d, m_d = torch.from_numpy(cons).to(dev), None
        del cons
    else:
        c_d, m_d = states
        n = c_d.shape[1]
        gc = GRMHDEquationsSystem(P)

    def timed(use_learned):
        for _ in range(2):
            gc.conservs_to_prims(c_d, m_d, use_learned=use_learned)
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(reps):
            gc.conservs_to_prims(c_d, m_d, use_learned=use_learned)
        a1.record()
        torch.cuda.synchronize()
        return n * reps / (a0.elapsed_time(a1) * 1e-3)

    def iters(use_learned):
        it = torch.zeros(n, dtype=torch.int32, device=dev)
        gu = torch.zeros(n, dtype=torch.int8, device=dev)
        pr = gc.conservs_to_prims(c_d, m_d, use_learned=use_learned, diag={"iters": it, "guess_used": gu})
        m = (n // 32) * 32
        st = {"mean_brent_iters": float(it.double().mean()), "max_brent_iters": int(it.max()),
              "warp_max_brent_iters": float(it[:m].view(-1, 32).max(1).values.double().mean())}
        if use_learned:
            st["guess_used"] = float(gu.double().mean())
        return pr, st

    out = {"states": n, "tolerance": 1e-12, "plain_solves_per_s": timed(False)}
    pr_p, out["plain"] = iters(False)
    # the tuned-mode c2p on the same states (plain bracket): the tuned
    # arithmetic, and the entropy backups deferred to a compacted second pass
    gc.set_mode(abi.MODE_TUNED)
    out["tuned_solves_per_s"] = timed(False)
    pr_t, _ = iters(False)
    out["tuned_vs_plain"] = _c2p_agreement(torch, pr_t, pr_p)
    gc.set_mode(abi.MODE_PLAIN)
    if learned:
        if states is None:
            tr, _ = workloads.c2p_states(1 << 20, seed=6)
            rep = gc.train_c2p_model(torch.from_numpy(tr).to(dev))
            del tr
        else:
            pick = torch.randperm(n, generator=torch.Generator().manual_seed(6))[:min(n, 1 << 20)].to(dev)
            rep = gc.train_c2p_model(c_d[:, pick].contiguous(), m_d[:, pick].contiguous())
        out["learned_solves_per_s"] = timed(True)
        pr_l, out["learned"] = iters(True)
        out["learned_vs_plain"] = _c2p_agreement(torch, pr_l, pr_p)
        gc.set_mode(abi.MODE_TUNED)
        out["learned_tuned_solves_per_s"] = timed(True)
        gc.set_mode(abi.MODE_PLAIN)
        out["training"] = {k: rep[k] for k in ("states", "labelled", "loss_first", "loss_last", "err_q50",
                                               "err_q90", "err_q99",
                                               "err_q999", "err_max", "delta", "delta_cand", "calib_ms", "calib_cost",
                                               "train_ms")}
        out["learned_speedup"] = out["learned_solves_per_s"] / out["plain_solves_per_s"]
        out["learned_tuned_speedup"] = out["learned_tuned_solves_per_s"] / out["plain_solves_per_s"]
    out["tuned_speedup"] = out["tuned_solves_per_s"] / out["plain_solves_per_s"]
    gc.close()
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if args.c2p_only:
        # the c2p micro-benchmark alone (for profiling; not the bench line)
        import torch
        if rank == 0:
            print(json.dumps(c2p_bench(torch.device("cuda:0"), learned=not args.no_learned, n=args.c2p_states)))
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
