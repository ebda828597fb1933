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
                       "Degree4Points11/Degree4Points7 (the 7-point triangle rule is exact to degree 5), LF, "
                       "SSP-RK3 CFL 0.3"),
    "vortex": dict(problem="vortex", n=8, L=10.0, jitter=0.0, P=1, qv=0, qf=1, flux="LF",
                   desc="isentropic vortex, [0,10]^3 periodic, 8^3x6=3,072 tets, P1, "
                        "Degree2Points4/Degree3Points6, LF, SSP-RK3 CFL 0.3"),
    "ensemble": dict(problem="vortex", n=8, L=10.0, jitter=0.0, P=2, qv=1, qf=2, flux="LF",
                     desc="64 isentropic-vortex instances on meshes n^3x6, n in U{8..32}, P2 (reference CPU "
                          "sample: one 8^3x6 vortex)"),
    "dwave_p4": dict(problem="density_wave", n=64, L=1.0, jitter=0.1, P=4, qv=5, qf=3, flux="LF",
                     desc="density wave, [0,1]^3 periodic, 64^3x6=1,572,864 jittered tets, P4, "
                          "Degree8Points44/Degree10Points24, LF, SSP-RK3 CFL 0.3"),
}
METRIC = "DOF-stage updates/s"
CFL = 0.3
# Algorithmic minimum HBM bytes per DOF-stage of one SSP-RK3 stage: read U^(i) and U^n, write U^(i+1)
# (24 B per DOF) plus the per-element geometry and the per-face trace data, amortised over the DOFs.
MIN_BYTES_PER_DOF_STAGE = {1: 32.2, 2: 27.3, 3: 25.6, 4: 24.9}
# Algorithmic flops per DOF-stage of the same stage at the configs' rules: volume interpolation and
# projection, the flux at the volume and face points, the face traces and integrals, the update.
FLOP_PER_DOF_STAGE = {1: 219.0, 2: 262.0, 3: 651.0, 4: 801.0}
FP64_NOMINAL_TFLOPS = 40.0  # B200 FP64 (vector and tensor), the bound of the FP64 form


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


def kernel_bytes(name, P, ncell, nface, nqf):
    """Algorithmic bytes one launch must move: each input read once, each output written once."""
    nb = nb_of(P)
    state = ncell * 5 * nb * 8
    face_rec, elem_rec = 48, 80 + 32     # face record; element geometry + face list
    gp = (nqf + 7) // 8 * 8
    if name == "face_flux_tc":           # state read, face records + group records, FP64 face fluxes written
        return state + nface * face_rec + nface * 16 // 3 + nface * 5 * gp * 8
    if name == "element_tc":             # stage state + U^n read, new stage written, det J J^-T + 1/det J,
        return 3 * state + ncell * 80 + ncell * 96 // 3 + nface * 5 * gp * 8 * 2  # group records, Fh from both sides
    if name == "face_flux_fp64":         # state read, face records, FP64 face fluxes written
        return state + nface * face_rec + nface * nqf * 5 * 8
    if name == "element_fp64":           # stage state + U^n read, new stage written, face fluxes read
        return 3 * state + ncell * elem_rec + nface * nqf * 5 * 8
    if name == "limiter":                # bounds from the stage input, the output read and written
        return 3 * state + nface * (48 + 80) + ncell * 32
    if name == "viscous":                # state read by both launches, residual written, face blocks
        return 3 * state + 3 * nface * 8 * (5 * nqf + nb) + ncell * (80 + 8 + 32) + nface * 96
    kf = (nqf + 7) // 8 * 8
    fj = nface * (5 * kf * 4 + 2 * 5 * 8)  # face records: split flux deviations (A rows), FP64 reference, mode-0 sums
    grp = ncell * 96 // 3                  # element-group records
    if name == "face_flux_mixed":          # stage input rows (split in registers), face infos, face records written
        return state + nface * face_rec + fj
    if name == "element_mixed":            # geometry, face records, stage input + U^n read; new stage written
        return ncell * 88 + grp + fj + 3 * state
    if name == "stage_persistent_mixed":   # both phases, the face records written and read once
        return nface * face_rec + ncell * 88 + grp + 2 * fj + 3 * state
    raise ValueError(name)


def algorithmic_bytes(name, P, ncell, nface, nqf):
    """The algorithm's minimum HBM bytes for the work one launch does, independent of how this
    implementation stores its intermediates: the state rows the work must read and write (8 B per
    DOF each), the element geometry (80 B: J^-T and det J) and the face records (42 B: normal, 2A,
    two cell ids, two face maps). Face kernels: the stage input once plus the face records. Element
    kernels: the stage input, U^n and the new stage plus the geometry. A whole stage (the persistent
    kernel): both, with the stage input counted once. The limiter and the viscous operator have no
    such minimum of their own; their implementation bytes stand in."""
    state = ncell * 5 * nb_of(P) * 8
    if name.startswith("face_flux"):
        return state + 42 * nface
    if name.startswith("element"):
        return 3 * state + 80 * ncell
    if name == "stage_persistent_mixed":
        return 3 * state + 80 * ncell + 42 * nface
    return kernel_bytes(name, P, ncell, nface, nqf)


# Parameters of the problems for the oracle's own projection (ref_harness.cpp problem_state), equal
# to the defaults of fve_dg_b200.problems that the GPU arm uses.
ORACLE_PROBLEM = {
    "taylor_green": [0.1, 1.4],
    "density_wave": [0.2, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 1.0, 1.4],
    "vortex": [5.0, 5.0, 5.0, 0.0, 0.0, 1.0, 5.0, 1.4, 1.0, 1.0, 0.0, 0.0],
}


def oracle_setup(cfg, n=None):
    """The workload's mesh and initial state built by the oracle alone: the periodic box made inside
    the reference harness and the reference's func2coef projection (nothing of fve_dg_b200 is
    loaded). Returns (RefLib, RefMesh, U0, mass, seconds)."""
    from oracle.pyoracle import RefLib
    t0 = time.perf_counter()
    ref = RefLib()
    ref.set_threads(os.cpu_count() or 1)
    n = cfg["n"] if n is None else n
    rm = ref.box(n, hi=(cfg["L"],) * 3, jitter=cfg["jitter"])
    U = rm.project(cfg["P"], cfg["problem"], ORACLE_PROBLEM[cfg["problem"]])
    b = rm.mass(cfg["P"], cfg["qv"])
    return ref, rm, U, b, time.perf_counter() - t0


def time_reference_steps(rm, U, b, cfg, dt, budget_s, max_steps):
    """SSP-RK3 steps of the reference's own operator (ExplicitConvection::eval with LongVector stage
    updates, ref_harness.cpp run_ssprk3) on the whole mesh: one untimed residual evaluation first,
    then whole steps while the estimate stays within budget_s (at least one)."""
    P, qv, qf = cfg["P"], cfg["qv"], cfg["qf"]
    t0 = time.perf_counter()
    rm.eval(U, P, qv, qf)
    per_eval = time.perf_counter() - t0
    k = int(max(1, min(max_steps, budget_s // max(3.2 * per_eval, 1e-9))))
    t0 = time.perf_counter()
    U = rm.ssprk3(U, b, P, qv, qf, dt, k)
    return k, time.perf_counter() - t0, U


def run_reference(args, cfg, rank):
    """The reference's own CPU path on the whole workload mesh (rank 0 only): the oracle builds the
    mesh and the initial state itself, so the product's library is never loaded in this arm."""
    if rank != 0:
        return
    from oracle.pyoracle import ref_available
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfvedg_ref.so was not built"}))
        return
    threads = os.cpu_count() or 1
    ref, rm, U, b, setup_s = oracle_setup(cfg)
    P = cfg["P"]
    k, el, _ = time_reference_steps(rm, U, b, cfg, 1e-4, 90.0, args.steps)
    dofs = 5 * nb_of(P) * rm.ncell * 3 * k
    val = dofs / el
    flux_note = "LF flux (the reference has no Roe solver)" if cfg["flux"] == "Roe" else "LF flux"
    sample = (f"{cfg['problem']} P{P} on the whole {cfg['n']}^3x6={rm.ncell} tet mesh, same rules, {flux_note}; "
              f"{k} SSP-RK3 step(s) of ExplicitConvection::eval + LongVector stage updates, {el:.1f} s on {threads} "
              f"threads; mesh and func2coef projection made by the oracle ({setup_s:.1f} s, untimed)")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "DOF-stage/s", "n_gpus": args.gpus,
            "steps": k, "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / k,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.config, "desc": cfg["desc"], "precision": "fp64", "tets": rm.ncell,
                       "flux_timed": "LF", "same_mesh_and_rules": True},
            "cpu_baseline": {"value": val, "unit": "DOF-stage/s", "cores": threads, "kind": "reference",
                             "sample": sample, "cpu_model": cpu_model()},
            "e2e": {"value": val, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(cfg):
    """The reference's CPU operator timed on the GPU box's host cores (rank 0, N=1): one SSP-RK3 step
    of the whole workload mesh on all threads, and for context a one-thread figure on a 12^3x6 slice
    of the same problem. Mesh and state come from the oracle alone."""
    from oracle.pyoracle import ref_available
    if not ref_available():
        return None
    threads = os.cpu_count() or 1
    ref, rm, U, b, setup_s = oracle_setup(cfg)
    k, el, _ = time_reference_steps(rm, U, b, cfg, 1e-4, 40.0, 1)
    ncell = rm.ncell
    val = 5 * nb_of(cfg["P"]) * ncell * 3 * k / el
    del rm
    n1 = max(4, min(cfg["n"], 12))
    ref1, rm1, U1, b1, _ = oracle_setup(cfg, n=n1)
    ref1.set_threads(1)
    k1, el1, _ = time_reference_steps(rm1, U1, b1, cfg, 1e-4, 8.0, 20)
    ref1.set_threads(threads)
    val1 = 5 * nb_of(cfg["P"]) * rm1.ncell * 3 * k1 / el1
    flux_note = "LF flux (the reference has no Roe solver)" if cfg["flux"] == "Roe" else "LF flux"
    return {"value": val, "unit": "DOF-stage/s", "cores": threads, "kind": "reference",
            "sample": f"{cfg['problem']} P{cfg['P']}, whole {cfg['n']}^3x6={ncell} tet mesh, {k} SSP-RK3 step(s), "
                      f"{flux_note}, {el:.1f} s; mesh and func2coef projection made by the oracle",
            "value_1_thread": val1, "sample_1_thread": f"{n1}^3x6={rm1.ncell} tets, {k1} steps, {el1:.1f} s",
            "cpu_model": cpu_model()}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="tgv", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--schedule", default=None, choices=["two-launch", "persistent"])
    ap.add_argument("--no-compare", action="store_true", help="skip timing the FP64 form beside the mixed one")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--viscous", action="store_true",
                    help="time the explicit viscous operator (ExplicitDiffusion::eval) on the workload's mesh instead")
    ap.add_argument("--limiter", default=None, choices=["positive", "positive-avg"],
                    help="positivity-preserving limiter after every RK stage (timed as its own kernel class)")
    ap.add_argument("--mu", type=float, default=0.0,
                    help="viscosity: > 0 steps compressible Navier-Stokes (the viscous residual every stage, "
                         "timed as its own kernel class), e.g. 1/1600 for the Taylor-Green vortex at Re 1600")
    ap.add_argument("--prandtl", type=float, default=0.71)
    ap.add_argument("--n", type=int, default=0, help="override the mesh size (cubes per side), for profiling")
    ap.add_argument("--order-sweep", action="store_true",
                    help="P1..P4 on the workload's mesh: the mixed form (two-launch, and batched with the autotuner's "
                         "tiles) against the FP64 form per order, with the autotuner's record per order")
    ap.add_argument("--split", action="store_true",
                    help="one mesh split across the N ranks (element slabs with ghost elements), SSP-RK3 one "
                         "stage at a time with the NCCL halo exchange before every stage (strong scaling)")
    ap.add_argument("--part-of", type=int, default=0,
                    help="(one GPU) time part 1 of a K-way split alone, ghost rows held fixed, against the "
                         "whole mesh: the decomposition's compute overhead without the exchange")
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

    if args.order_sweep:
        run_order_sweep(args, cfg, rank, world, local, dist)
        if dist:
            dist.destroy_process_group()
        return
    if args.config == "ensemble":
        run_ensemble(args, rank, world, local, dist)
        if dist:
            dist.destroy_process_group()
        return
    if args.viscous:
        run_viscous(args, cfg, rank, world, local, dist)
        if dist:
            dist.destroy_process_group()
        return
    if args.split or args.part_of:
        run_split(args, cfg, rank, world, local, dist)
        if dist:
            dist.destroy_process_group()
        return

    P, qv, qf = cfg["P"], cfg["qv"], cfg["qf"]
    m = box_mesh(cfg["n"], hi=(cfg["L"],) * 3, jitter=cfg["jitter"])
    U0 = problems.project(m, P, problem_fn(cfg["problem"], problems))
    # one instance: two launches per stage (face fluxes, elements) is the faster schedule; the
    # persistent tile queue serves ensembles of uneven meshes (--config ensemble)
    schedule = args.schedule or "two-launch"
    conv = ExplicitConvection(m, order=P, flux=cfg["flux"], quad_vol=qv, quad_face=qf,
                              precision=args.precision, device=local, schedule=schedule, limiter=args.limiter,
                              mu=args.mu, prandtl=args.prandtl)
    conv.set_state(U0)
    dt = problems.cfl_dt(CFL, cfg["L"] / cfg["n"], P, conv.max_wave_speed())
    nb = conv.num_basis
    dof_stage_per_step = 5 * nb * m.ncell * 3
    # the autotuner's choice for this schedule (two-launch: the element kernel's shape; persistent:
    # the tile queue), made before timing and recorded in the line
    tune = {schedule: conv.autotune(dt)} if args.precision == "mixed" else None

    sampler = ClockSampler(local)
    sampler.start()
    ms, launches = time_steps(conv, dt, args.warmup, args.steps, dist, torch, launch_count)
    clocks = sampler.stop()
    value = dof_stage_per_step * args.steps * world / (ms / 1e3)
    U_head = conv.get_state()

    # per-kernel durations with CUDA events on the context stream (same workload, separate pass)
    kt = conv.ssprk3_timed(dt, args.steps)
    roofline = make_roofline(kt, args.precision, schedule, P, m.ncell, m.nface, conv.nq_face, nb, args.config)

    # the other form on the same problem, same dt and steps from the same initial state
    forms = {args.precision: {"value": value, "ms_per_step": ms / args.steps, "schedule": schedule}}
    accuracy = None
    if args.precision == "mixed" and not args.no_compare:
        f64 = ExplicitConvection(m, order=P, flux=cfg["flux"], quad_vol=qv, quad_face=qf, precision="fp64",
                                 device=local, limiter=args.limiter, mu=args.mu, prandtl=args.prandtl)
        f64.set_state(U0)
        ms64, _ = time_steps(f64, dt, args.warmup, args.steps, dist, torch, launch_count)
        U64 = f64.get_state()  # before the per-kernel timing pass below advances it
        kt64 = f64.ssprk3_timed(dt, 3)
        forms["fp64"] = {"value": dof_stage_per_step * args.steps * world / (ms64 / 1e3),
                         "ms_per_step": ms64 / args.steps, "schedule": "two-launch",
                         "kernels_ms_per_launch": {KNAMES[("fp64", "two-launch")].get(k, str(k)): v[0] / v[1]
                                                   for k, v in kt64.items()},
                         "roofline": make_roofline(kt64, "fp64", "two-launch", P, m.ncell, m.nface, conv.nq_face, nb,
                                                   args.config)}
        forms["mixed_over_fp64"] = forms["mixed"]["value"] / forms["fp64"]["value"]
        ctxs = {"mixed": conv, "fp64": f64}
        if schedule == "two-launch":
            # the batched form: one persistent launch per RK stage over the tile queue, the tiles chosen
            # by the autotuner on this mesh, one CUDA graph per step
            bat = ExplicitConvection(m, order=P, flux=cfg["flux"], quad_vol=qv, quad_face=qf, precision="mixed",
                                     device=local, schedule="persistent", limiter=args.limiter, mu=args.mu,
                                     prandtl=args.prandtl)
            bat.set_state(U0)
            tune["persistent"] = bat.autotune(dt)
            ms_b, _ = time_steps(bat, dt, args.warmup, args.steps, dist, torch, launch_count)
            ktb = bat.ssprk3_timed(dt, 3)
            vb = dof_stage_per_step * args.steps * world / (ms_b / 1e3)
            forms["mixed_batched"] = {"value": vb, "ms_per_step": ms_b / args.steps, "schedule": "persistent",
                                      "kernels_ms_per_launch": {KNAMES[("mixed", "persistent")].get(k, str(k)):
                                                                v[0] / v[1] for k, v in ktb.items()}}
            forms["mixed_batched_over_fp64"] = vb / forms["fp64"]["value"]
            ctxs["mixed_batched"] = bat
        # accuracy: every form stepped the configuration's number of steps from U0 with the same dt
        # (untimed, independent of --steps)
        accuracy = accuracy_report(ctxs, U0, dt, m, P, cfg, args.config, problems)
        for name in ctxs:
            if name != "fp64":
                forms[name]["l2_vs_fp64"] = accuracy.pop("l2_" + name + "_vs_fp64")
        for name, c in ctxs.items():
            if c is not conv:
                c.close()
    cons = conv.conservation()

    # end to end through the public API: H2D of the state from pinned memory, one SSP-RK3 step,
    # D2H of the result, every step
    e2e = time_e2e(conv, dt, args.steps, dof_stage_per_step, world, dist, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(cfg)
        except Exception as e:  # reported, never silently substituted
            cpu = {"error": str(e)}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "bf16x3 contractions, f32 flux, f64 state",
                "data": "synthetic",
                "config": {"workload": args.config + ("-ns" if args.mu > 0 else ""), "desc": cfg["desc"],
                           "precision": args.precision, "limiter": args.limiter,
                           "mu": args.mu, "prandtl": args.prandtl if args.mu > 0 else None,
                           "schedule": schedule, "tets": m.ncell, "order": P, "dof_per_stage": 5 * nb * m.ncell,
                           "dt": dt, "l2": "state larger than L2 (no flush needed)",
                           "parallelism": f"independent instance per GPU x{world}"},
                "gpu_launches": launches, "roofline": roofline, "forms": forms, "accuracy": accuracy,
                "autotune": tune,
                "conservation": {"mass": cons[0], "energy": cons[4], "kinetic": cons[5]},
                "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks}
        print(json.dumps(line), flush=True)
    conv.close()
    if dist:
        dist.destroy_process_group()


# SSP-RK3 steps of each configuration's run (the accuracy figures are taken after them)
RUN_STEPS = {"tgv": 100, "dwave": 200, "dwave_p4": 50, "vortex": 20, "ensemble": 20}


def accuracy_report(ctxs, U0, dt, m, P, cfg, config, problems):
    """Every form in ctxs ({name: context}, one named 'fp64') stepped RUN_STEPS[config] SSP-RK3 steps
    from U0 with the same dt: each other form's relative L2 error against the FP64 form per variable
    (momenta also against the norm of the whole momentum field), the drift of mass, energy and kinetic
    energy of each form over the run, and for the density wave the error of each form against the
    exact translated solution."""
    n = RUN_STEPS.get(config, 100)
    f64 = ctxs["fp64"]
    f64.set_state(U0)
    c0 = f64.conservation()
    out = {"after_steps": n, "t": n * dt}
    states, cons = {}, {}
    for name, c in ctxs.items():
        c.set_state(U0)
        c.ssprk3(dt, n, graph=True)
        states[name] = c.get_state()
        cons[name] = c.conservation()
    for name in states:
        if name == "fp64":
            continue
        err = problems.l2_errors(m, P, states[name], Uref=states["fp64"])
        errm = problems.l2_errors(m, P, states[name], Uref=states["fp64"], momentum_norm=True)
        out["l2_" + name + "_vs_fp64"] = {"rho": float(err[0]), "rhou": float(err[1]), "rhov": float(err[2]),
                                          "rhow": float(err[3]), "E": float(err[4]),
                                          "momenta_over_momentum_norm": [float(x) for x in errm[1:4]],
                                          "after_steps": n}
    for name in states:
        c = cons[name]
        out[name] = {"mass_drift": float((c[0] - c0[0]) / c0[0]), "energy_drift": float((c[4] - c0[4]) / c0[4]),
                     "kinetic_energy_change": float((c[5] - c0[5]) / c0[5]),
                     "momentum_drift": [float(c[i] - c0[i]) for i in (1, 2, 3)]}
    if cfg["problem"] == "density_wave":
        exact = problems.density_wave(t=n * dt)
        for name in states:
            e = problems.l2_errors(m, P, states[name], exact=exact)
            out[name]["l2_vs_exact"] = {"rho": float(e[0]), "E": float(e[4])}
    return out


KNAMES = {("fp64", "two-launch"): {0: "face_flux_tc", 1: "element_tc", 3: "viscous", 4: "limiter"},
          ("mixed", "two-launch"): {0: "face_flux_mixed", 1: "element_mixed", 3: "viscous", 4: "limiter"},
          ("mixed", "persistent"): {2: "stage_persistent_mixed", 3: "viscous", 4: "limiter"}}


def time_steps(conv, dt, warmup, steps, dist, torch, launch_count):
    """Device time of `steps` SSP-RK3 steps (one CUDA graph per step) on the context's stream,
    after `warmup` steps; barrier and synchronize on both sides, max over ranks."""
    stream = torch.cuda.ExternalStream(conv.stream)
    conv.ssprk3(dt, warmup, graph=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    l0 = launch_count()
    ev0.record(stream)
    conv.ssprk3(dt, steps, graph=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = launch_count() - l0
    ms = ev0.elapsed_time(ev1)
    if dist:
        dist.barrier()
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, launches


def time_e2e(conv, dt, steps, dof_stage_per_step, world, dist, torch):
    from fve_dg_b200 import _lib as L
    pinned = torch.empty(conv.shape, dtype=torch.float64, pin_memory=True)
    host = pinned.numpy()
    host[:] = conv.get_state()
    k = max(3, min(steps, 20))
    lib = L.lib()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(k):
        L.check(lib.dg_set_state(conv._ctx, L.dptr(host), 0), "dg_set_state")
        L.check(lib.dg_ssprk3_graph(conv._ctx, float(dt), 1), "dg_ssprk3_graph")
        L.check(lib.dg_get_state(conv._ctx, L.dptr(host), 0), "dg_get_state")
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    state_bytes = int(np.prod(conv.shape)) * 8
    return {"value": dof_stage_per_step * k * world / e2e_s, "unit": "DOF-stage/s",
            "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes, "steps": k}


def make_roofline(kt, precision, schedule, P, ncell, nface, nqf, nb, config):
    """Roofline object of the dominant kernel class of kt ({class: (total ms, launches)}): achieved GB/s
    on the algorithm's minimum bytes of one launch (algorithmic_bytes) over its average CUDA-event
    duration, against the measured HBM copy bandwidth. The bytes this implementation moves by design
    (its intermediates included) and the DRAM traffic ncu measured for the kernel are reported beside
    it, with their ratios to the algorithmic bytes. `stage` carries the stage-level figures on the
    algorithm's minimum bytes and flops per DOF-stage."""
    names = KNAMES[(precision, schedule)]
    peak, peak_kind = read_peaks()
    dom = max(kt, key=lambda k: kt[k][0])
    dom_ms = kt[dom][0] / kt[dom][1]
    name = names.get(dom, str(dom))
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            traffic = json.load(f).get(config, {}).get(name)
    except Exception:
        pass
    alg = algorithmic_bytes(name, P, ncell, nface, nqf)
    impl = kernel_bytes(name, P, ncell, nface, nqf)
    stage_ms = sum(v[0] for v in kt.values()) / kt[dom][1]  # every kernel class launches once per stage
    ach = alg / (dom_ms / 1e3) / 1e9
    dofs = 5 * nb * ncell
    stage_gbs = MIN_BYTES_PER_DOF_STAGE[P] * dofs / (stage_ms / 1e3) / 1e9
    stage_tf = FLOP_PER_DOF_STAGE[P] * dofs / (stage_ms / 1e3) / 1e12
    return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_kind": peak_kind, "traffic": traffic, "algorithmic_bytes_per_launch": alg,
            "implementation_bytes_per_launch": impl, "implementation_over_algorithmic": impl / alg,
            "traffic_over_algorithmic": (traffic / alg) if traffic else None,
            "frac_on_implementation_bytes": impl / (dom_ms / 1e3) / 1e9 / peak, "avg_launch_ms": dom_ms,
            "stage": {"ms": stage_ms, "bytes_per_dof_stage_min": MIN_BYTES_PER_DOF_STAGE[P],
                      "achieved_gbs_at_min_bytes": stage_gbs, "frac_of_hbm": stage_gbs / peak,
                      "flop_per_dof_stage": FLOP_PER_DOF_STAGE[P], "achieved_tflops": stage_tf,
                      "fp64_nominal_tflops": FP64_NOMINAL_TFLOPS,
                      "frac_of_fp64_nominal": stage_tf / FP64_NOMINAL_TFLOPS},
            "kernels_ms_per_launch": {names.get(k, str(k)): v[0] / v[1] for k, v in kt.items()}}


def run_viscous(args, cfg, rank, world, local, dist):
    """The explicit viscous operator (FP64, ExplicitDiffusion::eval) on the workload's mesh and state:
    residual evaluations per second on device buffers (CUDA events, max over ranks), end to end with
    host buffers through the C ABI, and the reference's own CPU operator on a bounded sample."""
    import torch
    from fve_dg_b200 import ExplicitConvection, box_mesh, launch_count, problems
    from fve_dg_b200 import _lib as L
    P, qv, qf = cfg["P"], cfg["qv"], cfg["qf"]
    m = box_mesh(cfg["n"], hi=(cfg["L"],) * 3, jitter=cfg["jitter"])
    U0 = problems.project(m, P, problem_fn(cfg["problem"], problems))
    conv = ExplicitConvection(m, order=P, flux=cfg["flux"], quad_vol=qv, quad_face=qf, device=local)
    nb = conv.num_basis
    dof = 5 * nb * m.ncell
    Ud = torch.from_numpy(U0).to(f"cuda:{local}")
    Rd = torch.empty_like(Ud)
    lib, s = L.lib(), conv.stream
    stream = torch.cuda.ExternalStream(s)

    def ev():
        L.check(lib.dg_viscous_residual_device(conv._ctx, Ud.data_ptr(), Rd.data_ptr(), 1.0, 1.0, s), "viscous")

    for _ in range(args.warmup):
        ev()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        ev()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = launch_count() - l0
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = dof * args.steps * world / (ms / 1e3)
    R = np.empty_like(U0)
    k = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(k):
        L.check(lib.dg_viscous_residual(conv._ctx, L.dptr(U0), L.dptr(R), 0, 1.0, 1.0), "viscous")
    e2e = dof * k * world / (time.perf_counter() - t0)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle.pyoracle import ref_available
        if ref_available():
            threads = os.cpu_count() or 1
            n_s = max(4, min(cfg["n"], 12))
            _, rm, Us, _, _ = oracle_setup(cfg, n=n_s)
            rm.diffusion(Us, P, qv, qf)
            kk, t0 = 0, time.perf_counter()
            while time.perf_counter() - t0 < 5.0 and kk < 50:
                rm.diffusion(Us, P, qv, qf)
                kk += 1
            el = time.perf_counter() - t0
            cpu = {"value": 5 * nb * rm.ncell * kk / el, "unit": "DOF-residual/s", "cores": threads,
                   "kind": "reference",
                   "sample": f"ExplicitDiffusion::eval, {cfg['problem']} P{P} on {n_s}^3x6={rm.ncell} tets, "
                             f"{kk} evaluations, {el:.1f} s", "cpu_model": cpu_model()}
    if rank == 0:
        ms_each = ms / args.steps
        # the state read by both launches, the residual written, the per-face buffer written once and
        # read from both sides, geometry and face records
        face_block = 8 * (5 * conv.nq_face + nb)
        bytes_each = 3 * dof * 8 + 3 * m.nface * face_block + m.ncell * (80 + 8 + 32) + m.nface * 48 * 2
        peak, peak_kind = read_peaks()
        traffic = None
        try:
            with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
                traffic = json.load(f).get(args.config, {}).get("viscous")
        except Exception:
            pass
        line = {"metric": "viscous residual DOF evaluations/s", "value": value, "unit": "DOF-residual/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_each,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": args.config + "-viscous", "desc": cfg["desc"] + "; ExplicitDiffusion, mu = Pr = 1",
                           "tets": m.ncell, "order": P, "parallelism": f"independent instance per GPU x{world}"},
                "gpu_launches": launches,
                "roofline": {"bound": "hbm", "kernel": "viscous_face + viscous_element",
                             "achieved": bytes_each / (ms_each / 1e3) / 1e9,
                             "peak": peak, "unit": "GB/s", "frac": bytes_each / (ms_each / 1e3) / 1e9 / peak,
                             "peak_kind": peak_kind, "traffic": traffic, "algorithmic_bytes_per_launch": bytes_each,
                             "note": "FP64 traces and contractions (on the FP64 tensor cores) per face and per "
                                     "element: bound by instruction issue and latency, not by HBM"},
                "cpu_baseline": cpu,
                "e2e": {"value": e2e, "unit": "DOF-residual/s", "h2d_bytes_per_step": dof * 8, "d2h_bytes_per_step": dof * 8,
                        "steps": k}}
        print(json.dumps(line), flush=True)
    conv.close()


def run_split(args, cfg, rank, world, local, dist):
    """One mesh across the ranks: rank r steps element slab r and its ghost elements, one SSP-RK3
    stage at a time, the ghost rows of every stage input filled by the NCCL halo exchange; all of
    it ordered on the context's stream (CUDA events there, max over ranks). With --part-of K on
    one GPU: part 1 of K alone (its ghost rows held fixed, no exchange) and the whole mesh, to
    measure the compute overhead of the decomposition."""
    import torch
    from fve_dg_b200 import ExplicitConvection, box_mesh, launch_count, problems
    from fve_dg_b200.partition import PartitionedConvection, partition_elements
    P, qv, qf = cfg["P"], cfg["qv"], cfg["qf"]
    m = box_mesh(cfg["n"], hi=(cfg["L"],) * 3, jitter=cfg["jitter"])
    U0 = problems.project(m, P, problem_fn(cfg["problem"], problems))
    schedule = args.schedule or "two-launch"
    kw = dict(order=P, flux=cfg["flux"], quad_vol=qv, quad_face=qf, precision=args.precision, schedule=schedule,
              limiter=args.limiter, device=local)
    nparts, me = (world, rank) if not args.part_of else (args.part_of, min(1, args.part_of - 1))
    if args.part_of and world > 1:
        raise SystemExit("--part-of runs on one GPU")
    part = partition_elements(m, nparts)
    if dist:
        pc = PartitionedConvection(m, part, me, dist=dist, **kw)
    else:
        pc = PartitionedConvection(m, part, me, exchange=lambda which: None, **kw)
    pc.set_state(U0)
    lam = torch.tensor([pc.conv.max_wave_speed()], dtype=torch.float64, device=f"cuda:{local}")
    if dist:
        dist.all_reduce(lam, op=dist.ReduceOp.MAX)
    dt = problems.cfl_dt(CFL, cfg["L"] / cfg["n"], P, float(lam.item()))
    nb = pc.conv.num_basis
    stream = torch.cuda.ExternalStream(pc.conv.stream)

    def timed(run, k):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = launch_count()
        e0.record(stream)
        run(k)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_, n_ = e0.elapsed_time(e1), launch_count() - l0
        if dist:
            t = torch.tensor([ms_], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_ = float(t.item())
        return ms_, n_

    def steps(k):
        for _ in range(k):
            for st in range(3):
                pc.overlapped_stage(dt, st)  # the exchange beside the faces between owned elements

    steps(args.warmup)
    ms, launches = timed(steps, args.steps)
    pc.wait()
    owned_dof = 5 * nb * pc.lm.n_owned * 3
    halo = {"parts": nparts, "owned": pc.lm.n_owned, "ghosts": int(len(pc.lm.ghosts)),
            "faces": pc.lm.mesh.nface, "recv_bytes_per_stage": int(len(pc.lm.ghosts)) * 5 * nb * 8,
            "neighbours": sorted(int(q) for q in pc.lm.recv)}
    if args.part_of:
        whole = ExplicitConvection(m, **kw)
        whole.set_state(U0)
        whole.ssprk3(dt, args.warmup, graph=True)
        wstream = torch.cuda.ExternalStream(whole.stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(wstream)
        whole.ssprk3(dt, args.steps, graph=True)
        e1.record(wstream)
        torch.cuda.synchronize()
        ms_whole = e0.elapsed_time(e1)
        whole.close()
        value = owned_dof * args.steps / (ms / 1e3)
        whole_value = 5 * nb * m.ncell * 3 * args.steps / (ms_whole / 1e3)
        halo.update({"whole_mesh_value": whole_value, "whole_ms_per_step": ms_whole / args.steps,
                     "part_times_parts_over_whole": value * nparts / whole_value,
                     "note": "part 1 alone on one GPU, ghost rows held fixed (no exchange), eager stages; the "
                             "whole mesh with one CUDA graph per step"})
        scaling, parallelism = "strong", f"part 1 of a {nparts}-way element split, alone on one GPU"
    else:
        value = 5 * nb * m.ncell * 3 * args.steps / (ms / 1e3)
        scaling, parallelism = "strong", (f"one mesh split into {world} element slabs, NCCL halo exchange per "
                                          "stage beside the fluxes of the faces between owned elements")
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": scaling, "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "bf16x3 contractions, f32 flux, f64 state",
                "data": "synthetic",
                "config": {"workload": args.config + "-split", "desc": cfg["desc"], "precision": args.precision,
                           "schedule": schedule, "limiter": args.limiter, "tets": m.ncell, "order": P, "dt": dt,
                           "l2": "state larger than L2 (no flush needed)", "parallelism": parallelism},
                "gpu_launches": launches, "halo": halo, "e2e": None}
        print(json.dumps(line), flush=True)
    pc.conv.close()


# the configurations' rules per order: (tet rule, triangle rule)
ORDER_RULES = {1: (0, 1), 2: (1, 2), 3: (3, 3), 4: (5, 3)}


def run_order_sweep(args, cfg, rank, world, local, dist):
    """P1..P4 on the workload's mesh and problem with each order's configuration rules: DOF-stage/s of
    the FP64 form, the mixed form with two launches per stage and the batched mixed form (one
    persistent launch per stage, tiles chosen by the autotuner, whose record is kept per order), and
    the density/energy error of the mixed form against FP64 after RUN_STEPS of the workload (at most
    50). One JSON line; rank 0 prints."""
    import torch
    from fve_dg_b200 import ExplicitConvection, box_mesh, launch_count, problems
    m = box_mesh(cfg["n"], hi=(cfg["L"],) * 3, jitter=cfg["jitter"])
    rows = []
    for P in (1, 2, 3, 4):
        qv, qf = ORDER_RULES[P]
        U0 = problems.project(m, P, problem_fn(cfg["problem"], problems))
        ctxs = {}
        for name, prec, sched in (("fp64", "fp64", "two-launch"), ("mixed", "mixed", "two-launch"),
                                  ("mixed_batched", "mixed", "persistent")):
            ctxs[name] = ExplicitConvection(m, order=P, flux=cfg["flux"], quad_vol=qv, quad_face=qf, precision=prec,
                                            device=local, schedule=sched)
            ctxs[name].set_state(U0)
        dt = problems.cfl_dt(CFL, cfg["L"] / cfg["n"], P, ctxs["fp64"].max_wave_speed())
        tune = {"two-launch": ctxs["mixed"].autotune(dt), "persistent": ctxs["mixed_batched"].autotune(dt)}
        dof = 5 * ctxs["fp64"].num_basis * m.ncell * 3
        row = {"order": P, "quad_vol": qv, "quad_face": qf, "dof_per_stage": dof // 3}
        for name, c in ctxs.items():
            ms, _ = time_steps(c, dt, args.warmup, args.steps, dist, torch, launch_count)
            row[name] = {"value": dof * args.steps * world / (ms / 1e3), "ms_per_step": ms / args.steps}
        row["mixed_over_fp64"] = row["mixed"]["value"] / row["fp64"]["value"]
        row["mixed_batched_over_fp64"] = row["mixed_batched"]["value"] / row["fp64"]["value"]
        n = min(50, RUN_STEPS.get(args.config, 50))
        states = {}
        for name, c in ctxs.items():
            c.set_state(U0)
            c.ssprk3(dt, n, graph=True)
            states[name] = c.get_state()
        for name in ("mixed", "mixed_batched"):
            e = problems.l2_errors(m, P, states[name], Uref=states["fp64"])
            row[name]["l2_vs_fp64"] = {"rho": float(e[0]), "E": float(e[4]), "after_steps": n}
        row["autotune"] = tune
        rows.append(row)
        for c in ctxs.values():
            c.close()
    if rank == 0:
        best = max(rows, key=lambda r: r["mixed_batched"]["value"])
        line = {"metric": METRIC, "value": rows[-1]["mixed_batched"]["value"], "unit": "DOF-stage/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": rows[-1]["mixed_batched"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16x3 contractions, f32 flux, f64 state", "data": "synthetic",
                "config": {"workload": args.config + "-order-sweep", "desc": cfg["desc"] + "; orders 1..4 with the "
                           "configurations' rules", "tets": m.ncell, "value_is": "P4 batched mixed form",
                           "fastest_batched_order": best["order"]},
                "orders": rows}
        print(json.dumps(line), flush=True)


def run_ensemble(args, rank, world, local, dist):
    """64 isentropic-vortex instances on meshes of 8^3..32^3 x 6 tets, P2: the batched mixed form
    (one persistent launch per RK stage over all instances, a CUDA graph per step, autotuned tiles)
    against 64 sequential plain FP64 solves. Instances are drawn from one seed per rank."""
    import torch
    from fve_dg_b200 import Ensemble, ExplicitConvection, box_mesh, launch_count, problems
    rng = np.random.default_rng(20261203 + rank)
    P, qv, qf, L = 2, 1, 2, 10.0
    meshes, states, lam = [], [], []
    for i in range(64):
        n = int(rng.integers(8, 33))
        beta = float(rng.uniform(1.0, 5.0))
        center = rng.uniform(0.0, L, 3)
        axis = rng.normal(size=3)
        m = box_mesh(n, hi=(L, L, L))
        U = problems.project(m, P, problems.isentropic_vortex(center=center, axis=axis, beta=beta, period=L))
        meshes.append(m)
        states.append(U)
    singles = []
    for m, U in zip(meshes, states):
        c = ExplicitConvection(m, order=P, quad_vol=qv, quad_face=qf, precision="fp64", device=local)
        c.set_state(U)
        lam.append(c.max_wave_speed())
        singles.append(c)
    dts = np.array([problems.cfl_dt(CFL, L / m.n, P, l) for m, l in zip(meshes, lam)])
    ens = Ensemble(meshes, order=P, quad_vol=qv, quad_face=qf, precision="mixed", schedule="persistent",
                   device=local)
    U0 = np.concatenate(states)
    ens.set_state(U0)
    tune = ens.autotune(float(dts.mean()))
    dofs = 5 * ens.num_basis * ens.ncell * 3
    stream = torch.cuda.ExternalStream(ens.stream)
    sampler = ClockSampler(local)
    sampler.start()
    ens.ssprk3(dts, args.warmup, graph=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = launch_count()
    e0.record(stream)
    ens.ssprk3(dts, args.steps, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = launch_count() - l0
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = dofs * args.steps * world / (ms / 1e3)
    U_batched = ens.get_state()  # after warmup + steps, before the timing pass below
    kt = ens.ssprk3_timed(float(dts.mean()), 3)
    # sequential plain FP64 solves of the same instances, same dt and steps
    torch.cuda.synchronize()
    ms_seq = 0.0
    for c, dt in zip(singles, dts):
        ms_c, _ = time_steps(c, float(dt), args.warmup, args.steps, None, torch, launch_count)
        ms_seq += ms_c
    seq_value = dofs * args.steps * world / (ms_seq / 1e3)
    got = ens.split(U_batched)
    errs = [problems.l2_errors(m, P, g, Uref=c.get_state()) for m, g, c in zip(meshes, got, singles)]
    e2e = None
    pinned = torch.empty(ens.shape, dtype=torch.float64, pin_memory=True)
    host = pinned.numpy()
    host[:] = ens.get_state()
    k = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(k):
        ens.set_state(host)
        ens.ssprk3(dts, 1, graph=True)
        host[:] = ens.get_state()
    e2e_s = time.perf_counter() - t0
    sb = int(np.prod(ens.shape)) * 8
    e2e = {"value": dofs * k * world / e2e_s, "unit": "DOF-stage/s", "h2d_bytes_per_step": sb,
           "d2h_bytes_per_step": sb, "steps": k,
           "note": "includes the host-side copies into and out of the numpy state arrays"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16x3 contractions, f32 flux, f64 state", "data": "synthetic",
                "config": {"workload": "ensemble", "desc": "64 isentropic vortices (strength U[1,5], centres and "
                           "axes seeded), meshes n^3x6 with n in U{8..32}, P2, Degree4Points11/Degree4Points7, "
                           "LF, SSP-RK3 CFL 0.3 per instance", "tets": int(ens.ncell), "instances": 64},
                "gpu_launches": launches,
                "forms": {"batched_mixed_persistent": {"value": value, "ms_per_step": ms / args.steps},
                          "sequential_fp64": {"value": seq_value, "ms_per_step": ms_seq / args.steps},
                          "batched_over_sequential": value / seq_value,
                          "l2_vs_fp64_max_over_instances": {"rho": float(max(e[0] for e in errs)),
                                                            "E": float(max(e[4] for e in errs))}},
                "kernels_ms_per_launch": {KNAMES[("mixed", "persistent")].get(kk, str(kk)): v[0] / v[1]
                                          for kk, v in kt.items()},
                "autotune": tune, "e2e": e2e, "clocks": clocks}
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
