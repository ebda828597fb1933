"""Benchmark of the explicit DG Euler path: DOF-stage updates/s of SSP-RK3 time stepping.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config tgv|dwave|vortex|dwave_p4] [--precision fp64|mixed]

Default workload: the 3D Taylor-Green vortex at Mach 0.1 on the periodic box [0, 2 pi]^3,
48^3 cubes x 6 = 663,552 tetrahedra, P3 (20 modes), volume rule Degree6Points23, face rule
Degree10Points24 (no degree-7 triangle rule exists in the reference), Roe flux, SSP-RK3 at CFL 0.3.
One step = one SSP-RK3 step (three residual evaluations + stage updates) over the whole mesh with
the state resident in HBM (531 MB in FP64, larger than the 126 MB L2, so no L2 flush is needed).

`--impl reference` times the reference's own CPU operator (ExplicitConvection::eval compiled from
source, oracle/_ref) with an SSP-RK3 loop written with its LongVector operators, on a bounded
sample of the same problem; under torchrun only rank 0 runs it.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (problem, n, lo/hi, jitter, P, qv, qf, flux, description)
    "tgv": dict(problem="taylor_green", n=48, L=2 * np.pi, jitter=0.0, P=3, qv=3, qf=3, flux="Roe",
                desc="Taylor-Green Ma 0.1, [0,2pi]^3 periodic, 48^3x6=663,552 tets, P3, "
                     "Degree6Points23/Degree10Points24, Roe, SSP-RK3 CFL 0.3"),
    "dwave": dict(problem="density_wave", n=32, L=1.0, jitter=0.1, P=2, qv=1, qf=2, flux="LF",
                  desc="density wave, [0,1]^3 periodic, 32^3x6=196,608 jittered tets, P2, "
                       "Degree4Points11/Degree4Points7, LF, SSP-RK3 CFL 0.3"),
    "vortex": dict(problem="vortex", n=8, L=10.0, jitter=0.0, P=1, qv=0, qf=1, flux="LF",
                   desc="isentropic vortex, [0,10]^3 periodic, 8^3x6=3,072 tets, P1, "
                        "Degree2Points4/Degree3Points6, LF, SSP-RK3 CFL 0.3"),
    "dwave_p4": dict(problem="density_wave", n=64, L=1.0, jitter=0.1, P=4, qv=5, qf=3, flux="LF",
                     desc="density wave, [0,1]^3 periodic, 64^3x6=1,572,864 jittered tets, P4, "
                          "Degree8Points44/Degree10Points24, LF, SSP-RK3 CFL 0.3"),
}
METRIC = "DOF-stage updates/s"
CFL = 0.3
SURVEY_BYTES_PER_DOF_STAGE = {1: 32.2, 2: 27.3, 3: 25.6, 4: 24.9}  # algorithmic minimum, DESIGN.md


def problem_fn(name, problems):
    if name == "taylor_green":
        return problems.taylor_green()
    if name == "density_wave":
        return problems.density_wave()
    return problems.isentropic_vortex()


def nb_of(P):
    return (P + 1) * (P + 2) * (P + 3) // 6


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
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
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def kernel_bytes(cls, P, ncell, nface, nqf, precision):
    """Algorithmic bytes one launch must move (each input read once, each output written once)."""
    nb = nb_of(P)
    state = ncell * 5 * nb * 8
    if precision == "fp64":
        fh = nface * nqf * 5 * 8
        if cls == 0:  # face_flux: state read, 48 B face record, Fh written
            return state + nface * 48 + fh
        # element: stage state + U^n read, new stage written, 80 B geometry + 32 B face list, Fh read
        return 3 * state + ncell * (80 + 32) + fh
    return None


def run_reference(args, cfg, rank):
    """The reference's own CPU path on a bounded sample of the workload (rank 0 only)."""
    if rank != 0:
        return
    from fve_dg_b200 import box_mesh, problems
    from oracle.pyoracle import RefLib, RefMesh, ref_available
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfvedg_ref.so was not built"}))
        return
    ref = RefLib()
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    n_s = max(4, min(cfg["n"], 12))
    m = box_mesh(n_s, hi=(cfg["L"],) * 3, jitter=cfg["jitter"])
    P, qv, qf = cfg["P"], cfg["qv"], cfg["qf"]
    U = problems.project(m, P, problem_fn(cfg["problem"], problems))
    rm = RefMesh.from_mesh(ref, m)
    b = rm.mass(P, qv)
    dt = 1e-4
    budget = 150.0
    t0 = time.perf_counter()
    for _ in range(args.warmup):
        U = rm.ssprk3(U, b, P, qv, qf, dt, 1)
    t_w = time.perf_counter() - t0
    per = t_w / max(args.warmup, 1)
    k = args.steps if per * args.steps <= budget else max(3, int(budget / max(per, 1e-9)))
    t0 = time.perf_counter()
    for _ in range(k):
        U = rm.ssprk3(U, b, P, qv, qf, dt, 1)
    el = time.perf_counter() - t0
    dofs = 5 * nb_of(P) * m.ncell * 3 * k
    val = dofs / el
    sample = (f"{cfg['problem']} P{P} on {n_s}^3x6={m.ncell} tets (same rules; LF flux, the reference has no Roe), "
              f"{k} SSP-RK3 steps of ExplicitConvection::eval + LongVector stage updates")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "DOF-stage/s", "n_gpus": args.gpus,
            "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * el / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.config, "desc": cfg["desc"], "precision": "fp64"},
            "cpu_baseline": {"value": val, "unit": "DOF-stage/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": val, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(cfg):
    """About 10-30 s of the reference's CPU operator on a sample of the workload (rank 0, N=1)."""
    from fve_dg_b200 import box_mesh, problems
    from oracle.pyoracle import RefLib, RefMesh, ref_available
    if not ref_available():
        return None
    ref = RefLib()
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    n_s = max(4, min(cfg["n"], 12))
    m = box_mesh(n_s, hi=(cfg["L"],) * 3, jitter=cfg["jitter"])
    P, qv, qf = cfg["P"], cfg["qv"], cfg["qf"]
    U = problems.project(m, P, problem_fn(cfg["problem"], problems))
    rm = RefMesh.from_mesh(ref, m)
    b = rm.mass(P, qv)
    U = rm.ssprk3(U, b, P, qv, qf, 1e-4, 1)  # warm-up step
    k, t0 = 0, time.perf_counter()
    while True:
        U = rm.ssprk3(U, b, P, qv, qf, 1e-4, 1)
        k += 1
        if time.perf_counter() - t0 > 10.0 or k >= 50:
            break
    el = time.perf_counter() - t0
    return {"value": 5 * nb_of(P) * m.ncell * 3 * k / el, "unit": "DOF-stage/s", "cores": threads,
            "kind": "reference",
            "sample": f"{cfg['problem']} P{P}, {n_s}^3x6={m.ncell} tets, {k} SSP-RK3 steps (LF flux), {el:.1f} s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="tgv", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=0, help="override the mesh size (cubes per side), for profiling")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    cfg = dict(CONFIGS[args.config])
    if args.n:
        cfg["n"] = args.n
        cfg["desc"] = cfg["desc"] + f" [mesh overridden: {args.n}^3x6 tets]"
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, cfg, rank)
        return

    import torch
    from fve_dg_b200 import ExplicitConvection, box_mesh, launch_count, problems
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    P, qv, qf = cfg["P"], cfg["qv"], cfg["qf"]
    m = box_mesh(cfg["n"], hi=(cfg["L"],) * 3, jitter=cfg["jitter"])
    U0 = problems.project(m, P, problem_fn(cfg["problem"], problems))
    conv = ExplicitConvection(m, order=P, flux=cfg["flux"], quad_vol=qv, quad_face=qf,
                              precision=args.precision, device=local)
    conv.set_state(U0)
    dt = problems.cfl_dt(CFL, cfg["L"] / cfg["n"], P, conv.max_wave_speed())
    nb = conv.num_basis
    dof_stage_per_step = 5 * nb * m.ncell * 3
    stream = torch.cuda.ExternalStream(conv.stream)

    sampler = ClockSampler(local)
    sampler.start()
    conv.ssprk3(dt, args.warmup, graph=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    l0 = launch_count()
    ev0.record(stream)
    conv.ssprk3(dt, args.steps, graph=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = launch_count() - l0
    ms = ev0.elapsed_time(ev1)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = dof_stage_per_step * args.steps * world / (ms / 1e3)

    # per-kernel durations with CUDA events on the context stream (same workload, separate pass)
    kt = conv.ssprk3_timed(dt, args.steps)
    peak, peak_kind = read_peaks()
    dom = max(kt, key=lambda k: kt[k][0])
    dom_ms = kt[dom][0] / kt[dom][1]
    names = {0: "face_flux_fp64", 1: "element_fp64"} if args.precision == "fp64" else {}
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            tj = json.load(f)
        traffic = tj.get(f"{args.config}:{args.precision}", {}).get(names.get(dom, str(dom)))
    except Exception:
        pass
    bytes_dom = kernel_bytes(dom, P, m.ncell, m.nface, conv.nq_face, args.precision)
    stage_ms = sum(v[0] for v in kt.values()) / (3 * args.steps)
    roofline = None
    if bytes_dom:
        ach = bytes_dom / (dom_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "kernel": names.get(dom, str(dom)), "achieved": ach, "peak": peak,
                    "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind, "traffic": traffic,
                    "algorithmic_bytes_per_launch": bytes_dom, "avg_launch_ms": dom_ms,
                    "stage": {"ms": stage_ms,
                              "bytes_per_dof_stage_min": SURVEY_BYTES_PER_DOF_STAGE[P],
                              "achieved_gbs_at_min_bytes": SURVEY_BYTES_PER_DOF_STAGE[P] * 5 * nb * m.ncell
                              / (stage_ms / 1e3) / 1e9},
                    "kernels_ms_per_launch": {names.get(k, str(k)): v[0] / v[1] for k, v in kt.items()}}

    # end to end through the public API: H2D of the state from pinned memory, one SSP-RK3 step,
    # D2H of the result, every step
    pinned = torch.empty(conv.shape, dtype=torch.float64, pin_memory=True)
    pinned.numpy()[:] = conv.get_state()
    host = pinned.numpy()
    k_e2e = max(3, min(args.steps, 20))
    from fve_dg_b200 import _lib as L
    lib = L.lib()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        L.check(lib.dg_set_state(conv._ctx, L.dptr(host), 0), "dg_set_state")
        L.check(lib.dg_ssprk3_graph(conv._ctx, float(dt), 1), "dg_ssprk3_graph")
        L.check(lib.dg_get_state(conv._ctx, L.dptr(host), 0), "dg_get_state")
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    state_bytes = int(np.prod(conv.shape)) * 8
    e2e = {"value": dof_stage_per_step * k_e2e * world / e2e_s, "unit": "DOF-stage/s",
           "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes, "steps": k_e2e}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(cfg)
        except Exception as e:  # reported, never silently substituted
            cpu = {"error": str(e)}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "bf16x3/f32/f64",
                "data": "synthetic",
                "config": {"workload": args.config, "desc": cfg["desc"], "precision": args.precision,
                           "tets": m.ncell, "order": P, "dof_per_stage": 5 * nb * m.ncell,
                           "l2": "state larger than L2 (no flush needed)",
                           "parallelism": f"independent instance per GPU x{world}"},
                "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    conv.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
