"""Benchmark: Lagrangian hydro (subfvlagrange, scheme "classic") cell-updates/s.

Workload: the 2-D Sedov blast on [0,1.2]^2, 512x512 squares split into triangles with
alternating diagonals (524,288 prism cells, one layer thick, vertices jittered +-5% of
h, seed 1), rho = 1, u = 0, e = 1e-8/(gamma-1), energy 0.244816 deposited in the cells
touching the origin, CFL 0.5. A step is one time step of lagrange_main.F90:89-127
over the whole mesh (rhs, CFL reduction, mesh motion, geometry, update); one
cell-update = one cell advanced by one step (TEU, src/ns/ns_main.F90:114).

`value` times steps on the device with the state resident in HBM (CUDA events on the
library's stream, graph-replayed steps, max over ranks). `e2e` runs the same step
through the C-ABI with host buffers: every step uploads the state from host memory and
downloads the result. The working set of a step (about 1 GB) is larger than the 126 MB
L2, so no flush is needed between steps.

Multi-GPU: independent replicas of the problem, one per rank (weak scaling, no
data-path collective). `--impl reference` times the CPU restatement of the reference
(oracle/) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_SIDE = 512
SEED = 1
CFL = 0.5
E_SEDOV = 0.244816
WORKLOAD = "sedov2d_lagrange_prism_512x512"


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--n", type=int, default=N_SIDE)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _raw(n):
    from subfv_b200 import meshgen
    return meshgen.prism_slab(n, n, 0.0, 1.2, 0.0, 1.2, 0.0, 1.0, jitter=0.05, seed=SEED)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _mesh_sizes(topo):
    from subfv_b200.roofline import MeshSizes
    fr = topo.array("face_right")
    sff = topo.array("sub_face_face")
    vsf = topo.array("vert_sub_face")
    ncsf = int(vsf.size + np.count_nonzero(fr[sff[vsf - 1] - 1] > 0))
    return MeshSizes(topo.n_vert, topo.n_elems, topo.n_faces, topo.n_sub_faces, topo.n_sub_elems, ncsf)


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(kernel):
    """dram read+write bytes per launch from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "lagrange_step_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return d.get("per_launch_dram_bytes", {}).get(kernel)


def cpu_baseline(n_steps=4):
    """The oracle (serial CPU restatement) on the same 512x512 mesh, a bounded number of
    steps, on one host core."""
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    raw = _raw(N_SIDE)
    o = OracleMesh(raw)
    mask = meshgen.sedov_origin_mask(o.topo("elem_vert_off"), o.topo("elem_vert"), o.geom("vert_coord"))
    sol = o.sedov_init(e_total=E_SEDOV, mask=mask)
    mass = o.geom("elem_volume") / sol[:, 0]
    t0 = time.perf_counter()
    n, _, _, _ = o.lag_run(sol, mass, CFL, 1.0, n_steps)
    el = time.perf_counter() - t0
    return {"value": n * o.n_elems / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"{n} time steps of the same 512x512 Sedov mesh, serial C++ restatement (oracle/), "
                      f"{el:.1f} s"}


def run_reference(args, rank, world):
    """CPU restatement of the reference on all host threads: independent 128x128 Sedov
    replicas (one per thread, a 1/16 spatial sample of the 512x512 workload); each
    bench step advances every replica by one time step. ctypes releases the GIL, so the
    threads run the serial oracle concurrently."""
    if rank != 0:
        return
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    n_thr = max(1, min(os.cpu_count() or 1, 64))
    side = 128
    raw = _raw(side)
    reps = []

    def make(i):
        o = OracleMesh(raw)
        mask = meshgen.sedov_origin_mask(o.topo("elem_vert_off"), o.topo("elem_vert"), o.geom("vert_coord"))
        sol = o.sedov_init(e_total=E_SEDOV, mask=mask)
        reps.append((o, sol, o.geom("elem_volume") / sol[:, 0]))

    ths = [threading.Thread(target=make, args=(i,)) for i in range(n_thr)]
    [t.start() for t in ths]
    [t.join() for t in ths]

    def step_all():
        def one(r):
            r[0].lag_run(r[1], r[2], CFL, 1.0, 1)
        ts = [threading.Thread(target=one, args=(r,)) for r in reps]
        [t.start() for t in ts]
        [t.join() for t in ts]

    for _ in range(args.warmup):
        step_all()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_all()
    el = time.perf_counter() - t0
    cells = sum(r[0].n_elems for r in reps)
    v = cells * args.steps / el
    out = {"impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": {"workload": WORKLOAD, "cells_per_replica": cells // len(reps),
                                           "replicas": len(reps), "parallelism": f"{len(reps)} host threads"},
           "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": len(reps), "kind": "port",
                            "sample": f"{len(reps)} threads x one 128x128 Sedov prism replica each, one time "
                                      f"step per bench step"},
           "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = _args()
    rank, world, local = _dist()
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        backend = "nccl" if (args.impl == "ours" and torch.cuda.is_available()) else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            dist.destroy_process_group()
        return

    torch.cuda.set_device(local)
    from subfv_b200 import meshgen
    from subfv_b200.lagrange import MIXED, PLAIN_FP64, LagrangeState, init_sol_sedov
    from subfv_b200.mesh import Mesh
    from subfv_b200.roofline import lag_kernel_bytes

    prec = MIXED if args.precision == "mixed" else PLAIN_FP64
    raw = _raw(args.n)
    mesh = Mesh.from_raw(raw)
    topo = mesh.topo
    mask = meshgen.sedov_origin_mask(topo.array("elem_vert_off"), topo.array("elem_vert"), topo.coords())
    sol0 = init_sol_sedov(mesh, e_total=E_SEDOV, mask=mask)
    mass = mesh.geometry("elem_volume") / sol0[:, 0]
    coords0 = mesh.coords()
    state = LagrangeState(mesh, sol0, mass, cfl=CFL, t_max=1.0, precision=prec)
    stream = torch.cuda.ExternalStream(state.mesh_stream())

    state.advance(args.warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    state.advance_async(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    st, steps_done, t_now = state.sync()
    if world > 1:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    cells = mesh.n_elems
    value = world * cells * args.steps / (ms / 1e3)

    # per-kernel device times of eager steps (events between kernels, same stream)
    prof_steps = 10
    kms = state.profile_steps(prof_steps)
    names = ["node", "cell", "finalize", "move", "face_geom", "cell_geom"]
    per = {k: v / prof_steps for k, v in zip(names, kms)}
    dom = max(per, key=per.get)
    sizes = _mesh_sizes(topo)
    kb = lag_kernel_bytes(sizes)
    peak, peak_kind = _peaks()
    achieved = kb[dom] / (per[dom] / 1e3) / 1e9
    step_ms = sum(per.values())
    step_achieved = sum(kb.values()) / (step_ms / 1e3) / 1e9

    # e2e through the C-ABI with host buffers (a fresh state from the same initial data)
    mesh.set_coords(coords0)
    mesh.compute_geometry_mesh()
    st_e2e = LagrangeState(mesh, sol0, mass, cfl=CFL, t_max=1.0, precision=prec)
    host = np.ascontiguousarray(sol0.copy())
    for _ in range(3):
        st_e2e.step_host(host)
    k_e2e = max(10, min(args.steps, 100))
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        st_e2e.step_host(host)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        tt = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e = {"value": world * cells * k_e2e / e2e_s, "unit": "cell-updates/s",
           "h2d_bytes_per_step": 5 * 8 * cells, "d2h_bytes_per_step": 5 * 8 * cells,
           "steps": k_e2e, "api": "subfv_lag_step_host"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()

    if rank == 0:
        out = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == PLAIN_FP64 else "f64+f32",
            "data": "synthetic (seeded jittered mesh, Sedov initial state)",
            "config": {"workload": WORKLOAD, "cells": cells, "vertices": mesh.n_vert,
                       "sub_faces": mesh.n_sub_faces, "precision": args.precision, "cfl": CFL,
                       "l2": "working set ~1 GB per step > 126 MB L2 (no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "status_bits": st, "sim_time": t_now,
            "gpu_launches": 6 * args.steps,
            "clocks": clocks,
            "e2e": e2e,
            "roofline": {"bound": "hbm", "kernel": f"k_lag_{dom}", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": _traffic(dom), "algorithmic_bytes": kb[dom],
                         "kernel_ms": per[dom], "step_achieved_gbs": step_achieved},
            "kernel_ms": per,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
