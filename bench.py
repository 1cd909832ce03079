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

`parity`: the same 4 steps run by the oracle (the CPU restatement, also the
`cpu_baseline` sample) and by the GPU from the same initial state, compared bit for bit.

`batched_and_served` (one GPU, default run): the batched mixed-precision measurement
(`batched_mixed`: 256 shock tubes, N uniform in [200, 20000], about 10.6 M cells, K
steps at precision levels 0/1/2 against the plain FP64 path run one problem at a time,
and per-field L1 / Linf / drift of 16 problems run to their end time) and a serving
stream (`serve`: 32 Gresho or Sedov requests of up to 32,768 cells on a Poisson stream,
p50/p99 latency and aggregate cell-updates/s against the requests solved one by one).
`--workload shocktubes` / `serve` run those at their full sizes.

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
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--n", type=int, default=N_SIDE)
    p.add_argument("--renumber", default="bfs", choices=["bfs", "hilbert"],
                   help="vertex order of the Lagrangian mesh: the reference's breadth-first order or a Hilbert curve")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", default="lagrange",
                   choices=["lagrange", "gresho", "implicit", "shocktubes", "serve"])
    p.add_argument("--problems", type=int, default=1024)
    p.add_argument("--nmax", type=int, default=20000)
    p.add_argument("--solo-sample", type=int, default=64)
    p.add_argument("--requests", type=int, default=200)
    p.add_argument("--rate", type=float, default=20.0)
    p.add_argument("--max-cells", type=int, default=1 << 18)
    p.add_argument("--time-scale", type=float, default=0.05)
    p.add_argument("--no-batch-serve", action="store_true",
                   help="skip the batched-mixed and serving measurements of the default run")
    p.add_argument("--ns-problems", type=int, default=256, help="shock tubes in the default run's batch")
    p.add_argument("--ns-steps", type=int, default=10)
    p.add_argument("--serve-requests", type=int, default=32)
    p.add_argument("--serve-max-cells", type=int, default=1 << 15)
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


def _fp64_peak():
    """FP64 FMA issue rate of this GPU (subfv_probe_fp64_fma: eight independent FMA chains
    per thread at full occupancy), measured after the timed region; the denominator of
    the FP64 fractions in profiles/."""
    import ctypes as C
    from subfv_b200 import _lib
    tf, ms = C.c_double(), C.c_double()
    if _lib.load().subfv_probe_fp64_fma(4096, C.byref(tf), C.byref(ms)) != 0:
        return None
    return {"peak_tflops": tf.value, "probe_ms": ms.value, "how": "fma.rn.f64, 8 chains/thread, 8 blocks x 256 per SM"}


def _ns_roofline(sz, stages, ms_per_update):
    """HBM roofline of the explicit Euler update from the compulsory bytes of
    roofline.algorithmic_bytes("ns_update"); sz = dict(ne, nv, nsf, nse) summed over meshes."""
    from subfv_b200.roofline import algorithmic_bytes
    peak, kind = _peaks()
    b = algorithmic_bytes("ns_update", stages=stages, **sz)
    gbs = b / (ms_per_update * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "explicit update (all kernels)", "achieved": gbs, "peak": peak, "unit": "GB/s",
            "frac": gbs / peak, "peak_kind": kind, "traffic": None, "algorithmic_bytes": b,
            "note": "step-level compulsory bytes; the node kernel is FP64-latency-bound (profiles/)"}


def _traffic(kernel):
    """dram read+write bytes per launch from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "lagrange_step_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return d.get("per_launch_dram_bytes", {}).get(kernel)


def cpu_baseline(n_steps=4, renumber="bfs"):
    """The oracle (serial CPU restatement) on the same 512x512 mesh, in the same vertex
    order, a bounded number of steps, on one host core."""
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    raw = _raw(N_SIDE)
    o = OracleMesh(raw, renumber=renumber)
    mask = meshgen.sedov_origin_mask(o.topo("elem_vert_off"), o.topo("elem_vert"), o.geom("vert_coord"))
    sol = o.sedov_init(e_total=E_SEDOV, mask=mask)
    mass = o.geom("elem_volume") / sol[:, 0]
    t0 = time.perf_counter()
    n, _, _, _ = o.lag_run(sol, mass, CFL, 1.0, n_steps)
    el = time.perf_counter() - t0
    return {"value": n * o.n_elems / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "nproc": os.cpu_count(), "cpu_model": _cpu_model(),
            "sample": f"{n} time steps of the same 512x512 Sedov mesh, serial C++ restatement (oracle/), "
                      f"{el:.1f} s"}, sol


def _cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


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


KERNEL_NAMES = {"face": "k_lag_face<0>", "node": "k_lag_node<0>", "cell": "k_lag_cell<0>",
                "finalize": "k_lag_finalize", "move": "k_lag_move", "face_geom": "k_face_geom<0>",
                "cell_geom": "k_geom_step"}


def _time_device(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_gresho(args, rank, world, local):
    """2-D Gresho vortex, explicit Euler (subfvns): 64x64 hex slab on [-0.5,0.5]^2,
    interior vertices jittered +-10% of h (seed 1), slip walls, peak Mach 0.1, multi_point
    nodal solver, second order (method 4), two-stage scheme, CFL 0.4, 200 iterations
    (n_max_iter = 199). One cell-update = one cell advanced one iteration."""
    import torch
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsConfig, NsState, init_gresho
    n = 64 if args.n == N_SIDE else args.n
    raw = meshgen.hex_slab(n, n, jitter=0.1, seed=SEED)
    mesh = Mesh.from_raw(raw)
    mesh_sizes = dict(ne=mesh.n_elems, nv=mesh.n_vert, nsf=mesh.n_sub_faces, nse=mesh.n_sub_elems)
    sol0 = init_gresho(mesh, 0.1)
    out = {}
    # the last variant adds the Navier-Stokes diffusion terms (constant mu, the namelist's
    # default Neumann walls), point-implicit per cell
    for prec_name, prec in (("fp64", 0), ("mixed", 1), ("mixed_flux", 2), ("fp64_diffusion", 0)):
        cfg = NsConfig(cfl=0.4, precision=prec)
        if prec_name == "fp64_diffusion":
            cfg = NsConfig(cfl=0.4, activate_diffusion=True, mu_p=1e-3)
        s = NsState(mesh, cfg, sol0)
        s.advance(args.warmup)
        s.sync()
        s2 = NsState(mesh, cfg, sol0)
        s2.prepare()  # graph capture is set-up, outside the timed region
        stream = torch.cuda.ExternalStream(int(_libmod().load().subfv_mesh_stream(mesh._h)))
        torch.cuda.synchronize()
        ms = _time_device(stream, lambda: s2.advance_async(200))
        st, steps, t = s2.sync()
        out[prec_name] = {"ms": ms, "steps": steps, "status": st, "sol": s2.sol(), "t": t}
    a = out["fp64"]["sol"]
    l1 = {}
    for name in ("mixed", "mixed_flux"):
        e1, ei = field_errors(a, out[name]["sol"])
        l1[name] = {"l1_rel": dict(zip(FIELDS, e1)), "linf_rel": dict(zip(FIELDS, ei))}
    cells = mesh.n_elems
    cpu = None
    if not args.no_cpu_baseline:
        from oracle.oracle import OracleMesh
        o = OracleMesh(raw)
        so = o.ns_gresho(0.1)
        t0 = time.perf_counter()
        o.ns_run(NsConfig(cfl=0.4).oracle_dict(), so, 19)
        el = time.perf_counter() - t0
        cpu = {"value": 20 * cells / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
               "sample": f"20 of the 200 iterations on the same mesh, serial C++ restatement, {el:.1f} s"}
    res = {"metric": "cell-updates/s", "workload": "gresho2d_ns_multipoint_o2_64x64",
           "value": cells * 200 / (out["fp64"]["ms"] / 1e3), "unit": "cell-updates/s",
           "mixed_value": cells * 200 / (out["mixed"]["ms"] / 1e3),
           "mixed_flux_value": cells * 200 / (out["mixed_flux"]["ms"] / 1e3),
           "diffusion_value": cells * 200 / (out["fp64_diffusion"]["ms"] / 1e3),
           "ms_per_iteration": out["fp64"]["ms"] / 200, "cells": cells, "iterations": 200,
           "mixed_errors_vs_fp64": l1, "status": [out[k]["status"] for k in ("fp64", "mixed", "mixed_flux", "fp64_diffusion")],
           "sim_time_after_200": out["fp64"]["t"],
           "roofline": _ns_roofline(mesh_sizes, 2, out["fp64"]["ms"] / 200),
           "dtype": "f64", "cpu_baseline": cpu}
    print(json.dumps(res), flush=True)


def run_implicit(args, rank, world, local):
    """3-D periodic box [-0.5,0.5]^3 (the reference's stitching frame), 96^3 hexahedra
    (884,736 cells), interior vertices jittered +-5% of h (seed 1); uniform flow at Mach
    0.3 plus 8 seeded Fourier velocity modes (5%); Navier-Stokes at Re = 1000 (rho = 1,
    |u| = 1, L = 1: mu = 1e-3) and Pr = 0.72; one backward-Euler step: first-order
    two-wave residual with the viscous and heat terms, the exact frozen-speed Euler
    Jacobian (5x5 BCSR, 7-point face stencil) plus the point-implicit diffusion blocks,
    block-Jacobi GMRES(30) to 1e-8 relative, CFL 10. FP64 GMRES and FP32-matrix GMRES
    inside FP64 iterative refinement; FP64 GMRES with the coloured LU-SGS preconditioner
    and the inviscid step beside them."""
    import torch
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsConfig, NsState, init_fourier_flow
    n = 96 if args.n == N_SIDE else args.n
    t0 = time.perf_counter()
    raw = meshgen.hex_box(n, jitter=0.05, seed=SEED, periodic=True)
    mesh = Mesh.from_raw(raw, renumber=args.renumber)
    setup_s = time.perf_counter() - t0
    sol0 = init_fourier_flow(mesh, seed=SEED)
    inviscid = NsConfig(scheme=4, second_order=False, method=0, bc_style=2, boundary_2d=False, cfl=0.5)
    viscous = NsConfig(scheme=4, second_order=False, method=0, bc_style=2, boundary_2d=False, cfl=0.5,
                       activate_diffusion=True, mu_p=1e-3, prandtl=0.72)
    res = {"metric": "cell-updates/s", "workload": f"periodic_box_{n}^3_backward_euler_navier_stokes",
           "cells": mesh.n_elems, "mesh_setup_s": setup_s, "reynolds": 1000, "prandtl": 0.72,
           "vertex_order": args.renumber}
    # The first viscous state builds the diffusion stencil and, with this constant
    # viscosity, the mesh's cache of the state-independent diffusion arrays (one full
    # evaluation of the vertex systems); every later state and step reuses them.
    before = mesh.device_bytes
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    NsState(mesh, viscous, sol0).close()
    torch.cuda.synchronize()
    res["diffusion_invariants"] = {
        "build_s": time.perf_counter() - t0, "device_bytes": mesh.device_bytes - before,
        "note": "one-time per mesh and diffusion constants: the vertex systems' inverses and products, which "
                "depend on the mesh and the constant viscosity only; each step computes its diffusion terms "
                "from the current state with them"}
    for name, refine, pc, cfg in (("fp64", False, 1, viscous), ("fp32_refine", True, 1, viscous),
                                  ("fp64_lusgs", False, 2, viscous), ("fp64_inviscid", False, 1, inviscid)):
        s = NsState(mesh, cfg, sol0)
        s.implicit_step(cfl_implicit=10.0, refine_fp32=refine, precond=pc)  # warm-up (pattern, workspace)
        s2 = NsState(mesh, cfg, sol0)
        s2.implicit_step(cfl_implicit=10.0, refine_fp32=refine, precond=pc)
        s3 = NsState(mesh, cfg, sol0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st, stats = s3.implicit_step(cfl_implicit=10.0, refine_fp32=refine, precond=pc)
        el = time.perf_counter() - t0
        # a second step on the same state: no per-state uploads or workspace allocation
        t1 = time.perf_counter()
        st2, stats2 = s3.implicit_step(cfl_implicit=10.0, refine_fp32=refine, precond=pc)
        el2 = time.perf_counter() - t1
        dev_ms = stats["ms_assemble"] + stats["ms_solve"] + stats["ms_update"]
        stats["device_ms"] = dev_ms
        stats["wall_ms_first_step"] = el * 1e3
        stats["wall_ms_next_step"] = el2 * 1e3
        dev2 = stats2["ms_assemble"] + stats2["ms_solve"] + stats2["ms_update"]
        stats["next_step"] = {"status": st2, "restarts": stats2["restarts"], "conv": stats2["conv"],
                              "outer": stats2["outer"], "ms_assemble": stats2["ms_assemble"],
                              "ms_solve": stats2["ms_solve"], "device_ms": dev2}
        stats["status"] = st
        stats["cell_updates_per_s_first_step"] = mesh.n_elems / (dev_ms * 1e-3)
        stats["cell_updates_per_s"] = mesh.n_elems / (dev2 * 1e-3)
        res[name] = stats
    res["value"] = res["fp64"]["cell_updates_per_s"]
    res["diffusion_invariants"]["cell_updates_per_s_one_step_with_build"] = mesh.n_elems / (
        res["diffusion_invariants"]["build_s"] + res["fp64"]["next_step"]["device_ms"] * 1e-3)
    res["unit"] = "cell-updates/s"
    from subfv_b200.roofline import algorithmic_bytes
    peak, kind = _peaks()
    nx = res["fp64"]["next_step"]
    cyc = algorithmic_bytes("gmres_cycle", m=mesh.n_elems, bs=5, nnzb=res["fp64"]["nnz_blocks"], krylov=30)
    solve_b = nx["restarts"] * cyc
    gbs = solve_b / (nx["ms_solve"] * 1e-3) / 1e9
    res["roofline"] = {"bound": "hbm", "kernel": "GMRES(30) solve (SpMV, block Jacobi, MGS)", "achieved": gbs,
                       "peak": peak, "unit": "GB/s", "frac": gbs / peak, "peak_kind": kind, "traffic": None,
                       "algorithmic_bytes": solve_b}
    res["timing"] = ("device events around assemble, GMRES and update of the second step on a state "
                     "(the first step also captures the Arnoldi-cycle graph; both reported)")
    print(json.dumps(res), flush=True)


def _build_meshes(raws, local, threads=None):
    """Device meshes for a list of raw meshes, built on host threads (the topology build
    and the upload release the GIL); host topology is dropped once the mesh is on the
    device."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from subfv_b200.mesh import Mesh

    def one(raw):
        torch.cuda.set_device(local)
        m = Mesh.from_raw(raw() if callable(raw) else raw)
        m.topo.close()
        m.topo = None
        return m

    n_thr = threads or max(1, min(32, (os.cpu_count() or 2) - 1))
    with ThreadPoolExecutor(n_thr) as ex:
        return list(ex.map(one, raws))


FIELDS = ["rho", "rho_u", "rho_v", "rho_w", "E"]


def field_errors(a, b):
    """Per-field relative errors of b against a (n, 5): L1 = sum |b - a| / sum |a| and
    Linf = max |b - a| / max |a|. The three momentum components share one scale, that of
    the momentum vector (the largest component norm), so a transverse momentum that is
    zero up to round-off is measured against the flow's momentum, not against itself."""
    l1s, lis = np.abs(a).sum(0), np.abs(a).max(0)
    l1s[1:4], lis[1:4] = l1s[1:4].max(), lis[1:4].max()
    d = np.abs(b - a)
    return ([float(d[:, i].sum() / max(l1s[i], 1e-300)) for i in range(5)],
            [float(d[:, i].max() / max(lis[i], 1e-300)) for i in range(5)])


def shocktube_block(problems, nmax, K, warmup, solo_sample, local, acc_problems=16, tune=True, rank=0, world=1):
    """Batched shock tubes: `problems` independent Riemann problems on N x 4 quad strips,
    N uniform in [200, nmax] (seed 1), states as in subfv_b200.shocktube, first order
    multi_point nodal solver, CFL 0.4, walls all round. Timed: K steps of the whole batch
    in shared launches (graph-replayed) at three precision levels (0 plain FP64, 1 FP32
    wave-speed bounds, 2 also FP32 reconstruction and flux), autotuned and fixed launch
    shapes; the baseline is the plain FP64 path run one problem at a time (subfv_ns_state,
    graph-replayed) over a sample of the problems. Accuracy: `acc_problems` problems of
    N <= 2000 run to their end time at each level, against plain FP64 (per-field L1 and
    Linf, mass and energy drift).

    With several ranks (one per GPU) the problems are split by cell count
    (replicas.partition_by_cells, the same on every rank), each rank runs its share, and
    the figures are whole-job: all ranks' cell-updates over the slowest rank's time; no
    device collective."""
    import torch
    from subfv_b200 import autotune, replicas, shocktube
    from subfv_b200.ns import NsBatch, NsConfig, NsState
    all_tubes = shocktube.sample(problems, seed=SEED, n_max=nmax)
    mine = replicas.partition_by_cells([t.n_cells for t in all_tubes], world)[rank]
    rng_tubes = [all_tubes[i] for i in mine]
    t0 = time.perf_counter()
    meshes = _build_meshes([(lambda t=t: shocktube.raw_mesh(t)) for t in rng_tubes], local)
    setup_s = time.perf_counter() - t0
    sols = [shocktube.initial_state(m, t) for m, t in zip(meshes, rng_tubes)]
    cells = sum(m.n_elems for m in meshes)
    tube_sizes = dict(ne=cells, nv=sum(m.n_vert for m in meshes), nsf=sum(m.n_sub_faces for m in meshes),
                      nse=sum(m.n_sub_elems for m in meshes))
    base = dict(scheme=1, second_order=False, method=4, bc_style=2, boundary_2d=True, cfl=0.4)
    budget = int(150e9)
    res = {"workload": f"shocktubes_{problems}_strips_Nx4_N200-{nmax}", "problems": problems,
           "cells": int(sum(replicas.gather_lists([cells]))), "steps": K, "ranks": world,
           "mesh_setup_s": replicas.max_over_ranks(setup_s),
           "mesh_bytes_per_rank_max": int(replicas.max_over_ranks(sum(m.device_bytes for m in meshes)))}
    for name, prec in (("level1", 1), ("level2", 2), ("fp64", 0)):
        b = NsBatch(NsConfig(**base, precision=prec), capacity=max(1, len(meshes)), budget_bytes=budget)
        slots = [b.add(m, s, t.t_end) for m, s, t in zip(meshes, sols, rng_tubes)]
        assert None not in slots
        log = []
        best = autotune.DEFAULT
        if tune:
            best, _ = autotune.tune_ns_batch(b, log=log)
        for _ in range(warmup):
            b.time_steps(1)
        sampler = ClockSampler(local)
        sampler.start()
        ms_tuned = b.time_steps(K)
        clocks = sampler.stop()
        v_tuned, s_tuned = replicas.aggregate_throughput(cells * K, ms_tuned / 1e3)
        r = {"value": v_tuned, "ms_per_step": 1e3 * s_tuned / K,
             "roofline": _ns_roofline(tube_sizes, 1, ms_tuned / K),
             "tuned_shape": {"node_lanes": best[0], "block_v": best[1], "grid_v": best[2], "grid_c": best[3]},
             "autotune_trials": len(log), "clocks": clocks, "state_bytes": sum(b.state_bytes(m) for m in meshes)}
        if tune:
            autotune.apply(b, autotune.DEFAULT)
            b.time_steps(1)
            ms_fixed = b.time_steps(K)
            v_fixed, s_fixed = replicas.aggregate_throughput(cells * K, ms_fixed / 1e3)
            r.update(fixed_value=v_fixed, fixed_ms_per_step=1e3 * s_fixed / K)
        b.sync()
        r["status"] = int(replicas.max_over_ranks(max([b.info(k)[3] for k in slots], default=0)))
        res[name] = r
        b.close()
        torch.cuda.synchronize()
    # plain FP64, one problem at a time, over a sample of the problems
    idx = np.random.default_rng(SEED + 1 + rank).choice(len(meshes), size=min(solo_sample, len(meshes)),
                                                        replace=False)
    solo_ms, solo_cells = 0.0, 0
    for i in idx:
        m, s, t = meshes[i], sols[i], rng_tubes[i]
        st_ = NsState(m, NsConfig(**base, precision=0, tmax=t.t_end), s)
        st_.advance(8)
        st_.sync()
        stream = torch.cuda.ExternalStream(int(_libmod().load().subfv_mesh_stream(m._h)))
        solo_ms += _time_device(stream, lambda: st_.advance_async(K))
        solo_cells += m.n_elems * K
        st_.close()
    solo, _ = replicas.aggregate_throughput(solo_cells, solo_ms / 1e3)
    res["solo_fp64"] = {"value": solo, "problems": int(sum(replicas.gather_lists([len(idx)]))),
                        "note": "plain FP64 path, one problem at a time, K steps each"}
    for name in ("fp64", "level1", "level2"):
        res[name]["x_solo_fp64"] = res[name]["value"] / solo
    # accuracy: small problems run to their end time at each level
    acc_idx = [i for i in range(len(meshes)) if rng_tubes[i].n <= 2000][:max(1, acc_problems // world)]
    # every rank takes part in the gathers below, with or without small problems of its own
    if True:
        outs = {}
        for name, prec in (("fp64", 0), ("level1", 1), ("level2", 2)):
            if not acc_idx:
                outs[name] = []
                continue
            b = NsBatch(NsConfig(**base, precision=prec), capacity=len(acc_idx), budget_bytes=budget)
            sl = [b.add(meshes[i], sols[i], rng_tubes[i].t_end) for i in acc_idx]
            while True:
                b.advance(64)
                b.sync()
                if all(b.info(k)[2] for k in sl):
                    break
            outs[name] = [b.sol(k, meshes[i].n_elems) for k, i in zip(sl, acc_idx)]
            b.close()

        def drift(name):
            out = []
            for i, u in zip(acc_idx, outs[name]):
                vol = meshes[i].geometry("elem_volume")
                t0_, t1_ = (sols[i] * vol[:, None]).sum(0), (u * vol[:, None]).sum(0)
                out.append([float(abs(t1_[k] - t0_[k]) / abs(t0_[k])) for k in (0, 4)])
            return out

        def gmax(rows):  # the largest of every rank's rows, per column
            rows = replicas.gather_lists([list(map(float, r)) for r in rows])
            return np.array(rows).max(0).tolist() if rows else None

        acc = {"problems": int(sum(replicas.gather_lists([len(acc_idx)]))), "fields": FIELDS,
               "fp64_mass_energy_drift_max": gmax(drift("fp64")),
               "note": "each problem run to its end time; errors against the plain FP64 run (bit-identical to "
                       "the oracle); momentum components scaled by the momentum vector"}
        for name in ("level1", "level2"):
            e = [field_errors(a, c) for a, c in zip(outs["fp64"], outs[name])]
            l1 = gmax([x[0] for x in e])
            acc[name] = {"l1_rel_max": l1, "linf_rel_max": gmax([x[1] for x in e]),
                         "mass_energy_drift_max": gmax(drift(name)),
                         "meets_l1_1e-6": bool(l1 is not None and max(l1) <= 1e-6)}
        res["accuracy"] = acc
    return res


def run_shocktubes(args, rank, world, local):
    """The batched shock-tube workload at full size (`--problems`, `--nmax`), the
    problems split over the ranks."""
    res = shocktube_block(args.problems, args.nmax, args.steps, args.warmup, args.solo_sample, local,
                          rank=rank, world=world)
    res.update(metric="cell-updates/s", value=res["level1"]["value"], unit="cell-updates/s", n_gpus=world,
               scaling="strong")
    if rank == 0:
        print(json.dumps(res), flush=True)


def serve_block(n_requests, rate, max_cells, time_scale, solo_sample, local, rank=0, world=1):
    """Serving: solve requests (Gresho vortex or 2-D Sedov, triangles or quadrilaterals,
    cells log-uniform in [4096, max_cells], end time uniform in [0.1, 1] x nominal x
    time_scale) on a seeded Poisson stream of `rate` requests per second, served by
    subfv_b200.serve.Server under a 150 GB budget, in plain FP64 and at precision level
    1. Latency = arrival to result on the host. Baseline: a sample of the same requests
    solved one at a time on the plain FP64 solo path.

    With several ranks (one per GPU) the stream is split by cell count
    (replicas.partition_by_cells), each rank serves its requests at their arrival times,
    and the figures are whole-job: latencies of all requests, all ranks' cell-updates over
    the longest makespan; no device collective."""
    import torch
    from subfv_b200 import replicas, serve
    all_reqs = serve.make_requests(n_requests, rate=rate, seed=SEED, cells_max=max_cells, time_scale=time_scale)
    mine = replicas.partition_by_cells([r.n_cells for r in all_reqs], world)[rank]
    reqs = [all_reqs[i] for i in mine]
    res = {"workload": f"serve_{n_requests}_requests", "requests": n_requests, "rate_per_s": rate,
           "cells_max": max_cells, "time_scale": time_scale, "budget_bytes_per_gpu": int(150e9), "ranks": world}
    for name, prec in (("fp64", 0), ("level1", 1)):
        srv = serve.Server(budget_bytes=int(150e9), capacity=max(64, n_requests), precision=prec, chunk=8,
                           build_threads=max(1, min(16, (os.cpu_count() or 2) - 2)), keep_solutions=False)
        sampler = ClockSampler(local)
        sampler.start()
        results, makespan = srv.run(reqs) if reqs else ([], 1e-9)
        clocks = sampler.stop()
        srv.close()
        torch.cuda.synchronize()
        cu = sum(r.n_cells * r.steps for r in results)
        value, slowest = replicas.aggregate_throughput(cu, makespan)
        everything = replicas.gather_lists(results)
        res[name] = {"value": value, "makespan_s": slowest, "cell_updates": int(sum(r.n_cells * r.steps for r in everything)),
                     "completed": len(everything), "failed": sum(1 for r in everything if r.status),
                     "latency": serve.latency_stats(everything), "clocks": clocks,
                     "steps_mean": float(np.mean([r.steps for r in everything])) if everything else 0.0}
    # one request at a time on the plain FP64 path, over a sample of the stream
    idx = np.random.default_rng(SEED + 2 + rank).choice(len(reqs), size=min(solo_sample, len(reqs)), replace=False)
    t0 = time.perf_counter()
    cu = 0
    for i in idx:
        steps, t, st, _ = serve.solve_alone(reqs[i], precision=0)
        cu += reqs[i].n_cells * steps
    el = max(time.perf_counter() - t0, 1e-9)
    one, el = replicas.aggregate_throughput(cu, el)
    res["one_by_one_fp64"] = {"value": one, "requests": int(sum(replicas.gather_lists([len(idx)]))), "seconds": el,
                              "note": "each request built and solved alone on the solo path, sequentially"}
    for name in ("fp64", "level1"):
        res[name]["x_one_by_one_fp64"] = res[name]["value"] / res["one_by_one_fp64"]["value"]
    return res


def run_serve(args, rank, world, local):
    res = serve_block(args.requests, args.rate, args.max_cells, args.time_scale, args.solo_sample, local, rank, world)
    res.update(metric="cell-updates/s", value=res["level1"]["value"], unit="cell-updates/s", n_gpus=world,
               scaling="weak")
    if rank == 0:
        print(json.dumps(res), flush=True)


def _libmod():
    from subfv_b200 import _lib
    return _lib


def main():
    args = _args()
    rank, world, local = _dist()
    if args.workload != "lagrange":
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        sharded = world > 1 and args.workload in ("shocktubes", "serve")
        if sharded:  # independent problems split over the ranks; only host reductions
            dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        if sharded or rank == 0:  # the single-mesh workloads run once, on rank 0
            {"gresho": run_gresho, "implicit": run_implicit, "shocktubes": run_shocktubes,
             "serve": run_serve}[args.workload](args, rank, world, local)
        if sharded:
            dist.barrier()
            dist.destroy_process_group()
        return
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
    from subfv_b200 import meshgen, replicas
    from subfv_b200.lagrange import MIXED, PLAIN_FP64, LagrangeState, init_sol_sedov
    from subfv_b200.mesh import Mesh
    from subfv_b200.roofline import lag_kernel_bytes

    prec = MIXED if args.precision == "mixed" else PLAIN_FP64
    raw = _raw(args.n)
    mesh = Mesh.from_raw(raw, renumber=args.renumber)
    topo = mesh.topo
    mask = meshgen.sedov_origin_mask(topo.array("elem_vert_off"), topo.array("elem_vert"), topo.coords())
    sol0 = init_sol_sedov(mesh, e_total=E_SEDOV, mask=mask)
    mass = mesh.geometry("elem_volume") / sol0[:, 0]
    coords0 = mesh.coords()
    state = LagrangeState(mesh, sol0, mass, cfl=CFL, t_max=1.0, precision=prec)
    stream = torch.cuda.ExternalStream(state.mesh_stream())

    state.advance(args.warmup)
    state.prepare()  # the replayed step graph is captured before the timed region
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
    ms = replicas.max_over_ranks(ms)  # the slowest replica's device time
    cells = mesh.n_elems
    value = world * cells * args.steps / (ms / 1e3)

    # per-kernel device times of eager steps (events between kernels, same stream)
    prof_steps = 10
    kms = state.profile_steps(prof_steps)
    names = ["face", "node", "cell", "finalize", "move", "face_geom", "cell_geom"]
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
    # the step's input and result in page-locked host memory (copied directly by the C-ABI)
    host_t = torch.empty(sol0.shape, dtype=torch.float64, pin_memory=True)
    host = host_t.numpy()
    host[:] = sol0
    for _ in range(3):
        st_e2e.step_host(host)
    k_e2e = max(10, min(args.steps, 100))
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        st_e2e.step_host(host)
    e2e_s = replicas.max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * cells * k_e2e / e2e_s, "unit": "cell-updates/s",
           "h2d_bytes_per_step": 5 * 8 * cells, "d2h_bytes_per_step": 5 * 8 * cells,
           "steps": k_e2e, "api": "subfv_lag_step_host", "host_buffer": "page-locked"}

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, sol_oracle = cpu_baseline(renumber=args.renumber)
        # the same 4 steps on the GPU from the same initial state, compared bit for bit
        mesh.set_coords(coords0)
        mesh.compute_geometry_mesh()
        st_par = LagrangeState(mesh, sol0, mass, cfl=CFL, t_max=1.0, precision=prec)
        st_par.advance(4)
        got = st_par.sol()
        same = bool(np.array_equal(got, sol_oracle))
        parity = {"against": "oracle (serial C++ restatement of lagrange_module.F90)", "steps": 4,
                  "cells": cells, "bit_exact": same, "max_abs_diff": float(np.abs(got - sol_oracle).max())}
        if prec != PLAIN_FP64:
            e1, ei = field_errors(sol_oracle, got)
            parity.update(l1_rel=dict(zip(FIELDS, e1)), linf_rel=dict(zip(FIELDS, ei)))
        st_par.close()

    batch_serve = None
    if rank == 0 and world == 1 and not args.no_batch_serve:
        batch_serve = {"batched_mixed": shocktube_block(args.ns_problems, args.nmax, args.ns_steps, 3, 32, local),
                 "serve": serve_block(args.serve_requests, args.rate, args.serve_max_cells, args.time_scale, 8,
                                      local)}

    if rank == 0:
        out = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == PLAIN_FP64 else "f64+f32",
            "data": "synthetic (seeded jittered mesh, Sedov initial state)",
            "config": {"workload": WORKLOAD, "cells": cells, "vertices": mesh.n_vert,
                       "sub_faces": mesh.n_sub_faces, "precision": args.precision, "cfl": CFL,
                       "vertex_order": args.renumber,
                       "l2": "working set ~1 GB per step > 126 MB L2 (no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "status_bits": st, "sim_time": t_now,
            "gpu_launches": 6 * args.steps,
            "clocks": clocks,
            "e2e": e2e,
            "roofline": {"bound": "hbm", "kernel": KERNEL_NAMES[dom], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": _traffic(dom), "algorithmic_bytes": kb[dom],
                         "kernel_ms": per[dom], "step_achieved_gbs": step_achieved},
            "kernel_ms": per,
            "fp64": _fp64_peak(),
            "cpu_baseline": cpu,
            "parity": parity,
            "batched_and_served": batch_serve,
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
