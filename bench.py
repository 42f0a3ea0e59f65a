"""Benchmark: BSSN RK4 grid-point updates/s on B200 (libbssn_b200), with the reference's
CPU implementation timed beside it.

Workload (one "step" = one full RK4 step, MoL_step_forward_in_time): SinhSpherical
256x64x64 interior (+3 ghost zones), AMPL=10, SINHW=0.2, Brill-Lindquist masses
~U[0.3,0.7] and z = +/-U[0.3,0.8] from the seed, FP64 state, 4th-order FD, KO dissipation,
outgoing-radiation outer BCs, Hamiltonian-constraint L2 every 20 steps (inside the
timed region). Synthetic data: the Brill-Lindquist initial data computed in-process.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (under torchrun): independent replicas, one per GPU (a single evolution does not
shard without a halo exchange of 3 ghost layers x 24 gridfunctions per stage, and the inner
parity map crosses the axis), each with its own seed; value is the
whole-job rate = sum of all ranks' point updates / max over ranks of the device time.
"""

import argparse
import ctypes as C
import json
import os
import pathlib
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NXX = (256, 64, 64)
# Interior finite-difference order of this run (BSSN_B200_FD_ORDER: 4 by default, or 8 with
# libbssn_b200_fd8.so); the reference arm and baselines use the reference project of the same order.
FD_ORDER = int(os.environ.get("BSSN_B200_FD_ORDER", "4"))
NG = FD_ORDER // 2 + 1
SINH_VARIANT = "sinh3d" if FD_ORDER == 4 else f"sinh3d{FD_ORDER}"
AMPL, SINHW = 10.0, 0.2
H_EVERY = 20
B_ALG_PER_PT_STEP = 3072  # bytes: classic RK4 with an accumulator, each stage read once
STAGE_WORDS = (72, 120, 120, 72)  # per interior point, FP64 words, stages 1..4
# FP64 operations per interior point of one fused stage pass (both RHS output groups, 2 DFMA +
# DADD + DMUL), counted by ncu at 4th order: profiles/kernels_rhs_ricci_groups_sinh256x64x32.md.
RHS_FLOP_PER_PT_STAGE = {4: 3458 + 2920}
METRIC = "BSSN RK4 grid-point updates/s on 1 B200, FP64 vs mixed at equal H-error"
UNIT = "pt-updates/s"


def bl_params(seed: int):
    rng = np.random.default_rng(seed)
    m1, m2 = rng.uniform(0.3, 0.7, 2)
    z1, z2 = rng.uniform(0.3, 0.8), -rng.uniform(0.3, 0.8)
    return float(m1), float(z1), float(m2), float(z2)


def aggregate(pts_local: int, steps: int, ms_local: float, dist=None, device="cpu"):
    """Whole-job rate of N independent replicas: sum of the ranks' point updates divided by
    the slowest rank's device time (max over ranks). Returns (value, max_ms)."""
    if dist is None:
        return pts_local * steps / (ms_local * 1e-3), ms_local
    import torch

    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    n = torch.tensor([float(pts_local) * steps], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(n.item()) / (float(t.item()) * 1e-3), float(t.item())


def profiled_traffic():
    """DRAM bytes per fused stage pass at the bench size, from the committed ncu summary."""
    p = ROOT / "profiles" / "kernels_rhs_ricci_groups_sinh256x64x32.md"
    try:
        for line in p.read_text().splitlines():
            if line.startswith("traffic_bytes_per_launch_full_size:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


_HOST_CPU = None


def host_cpu():
    """The host CPU as lscpu reports it: model, physical cores (cores per socket x sockets,
    capped by this process's CPU affinity) and logical CPUs. Evaluated once, at the first
    call: an OpenMP runtime with OMP_PROC_BIND set later binds the main thread to one core,
    which would shrink the affinity seen afterwards."""
    global _HOST_CPU
    if _HOST_CPU is not None:
        return dict(_HOST_CPU)
    info = {"model": None, "physical_cores": None, "logical_cpus": os.cpu_count()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        kv = {}
        for line in out.splitlines():
            if ":" in line:
                k, v = line.split(":", 1)
                kv[k.strip()] = v.strip()
        info["model"] = kv.get("Model name")
        info["lscpu"] = {k: kv[k] for k in ("CPU(s)", "Thread(s) per core", "Core(s) per socket", "Socket(s)",
                                            "NUMA node(s)") if k in kv}
        cps, sock = int(kv.get("Core(s) per socket", "0")), int(kv.get("Socket(s)", "1") or 1)
        info["threads_per_core"] = int(kv.get("Thread(s) per core", "1") or 1)
        if cps > 0:
            info["physical_cores"] = cps * sock
    except (OSError, ValueError, subprocess.SubprocessError):
        pass
    if not info["physical_cores"]:
        try:
            import psutil

            info["physical_cores"] = psutil.cpu_count(logical=False)
        except Exception:  # noqa: BLE001
            info["physical_cores"] = os.cpu_count()
    try:
        aff = len(os.sched_getaffinity(0))
        info["affinity_cpus"] = aff
        tpc = info.get("threads_per_core", 1) or 1
        info["physical_cores"] = max(1, min(info["physical_cores"], aff // tpc if aff >= tpc else aff))
    except (AttributeError, OSError):
        pass
    _HOST_CPU = dict(info)
    return info


def set_reference_threads():
    """OpenMP settings of the reference's CPU runs: one thread per physical core, bound close.
    Set in the environment before the reference library is loaded, and through the OpenMP
    runtime the reference library links (libgomp.so.1) in case it is already initialised;
    `omp_max_threads` is what that runtime then reports."""
    cpu = host_cpu()
    n = int(cpu["physical_cores"])
    os.environ["OMP_NUM_THREADS"] = str(n)
    os.environ["OMP_PROC_BIND"] = "close"
    os.environ["OMP_PLACES"] = "cores"
    try:
        gomp = C.CDLL("libgomp.so.1")
        gomp.omp_set_num_threads(n)
        cpu["omp_max_threads"] = int(gomp.omp_get_max_threads())
    except OSError:
        cpu["omp_max_threads"] = None
    return cpu


def cpu_reference_rate(steps: int, warmup: int, runs: int, seed: int):
    """The reference's generated OpenMP C (oracle/_ref) on the same workload, on all physical
    host cores: `warmup` untimed RK4 steps, then `runs` timed runs of `steps` steps each
    (MoL_step_forward_in_time only); the median run is reported."""
    cpu = set_reference_threads()
    from oracle import ref

    if not ref.available(SINH_VARIANT):
        return None
    m1, z1, m2, z2 = bl_params(seed)
    rg = ref.RefGrid(SINH_VARIANT, NXX, AMPL, SINHW=SINHW, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2)
    if warmup > 0:
        rg.step(warmup)
    times = []
    for _ in range(runs):
        t0 = time.perf_counter()
        rg.step(steps)
        times.append(time.perf_counter() - t0)
    rg.close()
    dt = float(np.median(times))
    pts = NXX[0] * NXX[1] * NXX[2]
    return {"value": pts * steps / dt, "unit": UNIT, "cores": cpu.get("omp_max_threads") or int(os.environ["OMP_NUM_THREADS"]),
            "kind": "reference",
            "sample": f"median of {runs} runs of {steps} RK4 steps of the full {NXX[0]}x{NXX[1]}x{NXX[2]} "
                      f"SinhSpherical grid after {warmup} warm-up steps (reference generated OpenMP C, fd_order "
                      f"{FD_ORDER}, MoL_step_forward_in_time incl. BCs + detgammabar; OMP_NUM_THREADS = physical "
                      f"cores, OMP_PROC_BIND=close)",
            "s_per_step": dt / steps, "run_s": times, "cpu_model": cpu.get("model"),
            "physical_cores": cpu.get("physical_cores"), "logical_cpus": cpu.get("logical_cpus"),
            "lscpu": cpu.get("lscpu")}


def workload_name() -> str:
    """The workload both arms run (the same string in both JSON lines)."""
    return (f"BSSN RK4, SinhSpherical {NXX[0]}x{NXX[1]}x{NXX[2]} (+{NG} ghosts), AMPL=10, SINHW=0.2, FP64, "
            f"{FD_ORDER}th-order FD, KO, radiation BCs, H-constraint L2 every 20 steps")


def bench_config(seed: int, world: int):
    """The workload description both arms print (identical keys and values)."""
    return {"workload": workload_name(), "interior_points": NXX[0] * NXX[1] * NXX[2], "H_every": H_EVERY,
            "parallelism": f"replicas x{world}", "seed": seed, "bl": list(bl_params(seed))}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    res = cpu_reference_rate(args.steps, 5, 3, args.seed)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref/{SINH_VARIANT} not built (run oracle/gen_ref.py)"}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * res["s_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Brill-Lindquist initial data, seeded)",
        "config": bench_config(args.seed, args.gpus),
        "implementation": "reference generated OpenMP C on the host cores (rank 0 only)",
        "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample", "cpu_model",
                                             "physical_cores", "logical_cpus", "run_s")},
        "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", type=int, default=1, help="0: reference stage order; 1: fused stages")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--batch-tile", default=None,
                    help="batched tile shape bx,by (0,0: a shape per grid) instead of the autotuner's pick")
    ap.add_argument("--no-batch-sequential", action="store_true",
                    help="skip advancing the batched grids one at a time (profiling)")
    ap.add_argument("--no-diff", action="store_true", help="skip the adjoint-gradient section")
    ap.add_argument("--no-diag", action="store_true", help="skip the diagnostics-output section")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference's own CUDA build")
    ap.add_argument("--no-cyl", action="store_true", help="skip the SinhCylindrical (blackhole_spectroscopy grid) section")
    ap.add_argument("--diff-only", action="store_true",
                    help="run only the adjoint-gradient section (one GPU) and print it as JSON (profiling)")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the batched section (one GPU) and print it as JSON (profiling)")
    ap.add_argument("--nxx", default=None, help="override the grid, e.g. 256,64,32 (profiling only)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    global NXX
    if args.nxx:
        NXX = tuple(int(x) for x in args.nxx.split(","))
    # Every reference run in this process (reference arm, CPU baseline, reference diagnostics
    # and checkpoint timings) uses one OpenMP thread per physical core, bound close.
    set_reference_threads()
    if args.impl == "reference":
        return run_reference(args)
    if args.diff_only:
        print(json.dumps(run_differentiation(fd_check=False)))
        return None
    if args.batched_only:
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps(run_batched(args, 1, 0, None)))
        return None

    import torch

    from nrpy_b200 import lib as L
    from nrpy_b200.grid import BSSNGrid

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    lib = L.load()
    m1, z1, m2, z2 = bl_params(args.seed + rank)
    grid = BSSNGrid(coord="SinhSpherical", Nxx=NXX, grid_physical_size=AMPL, SINHW=SINHW, BH1_mass=m1, BH1_posn_z=z1,
                    BH2_mass=m2, BH2_posn_z=z2)
    pts = grid.n_interior
    y0 = grid.y_n.clone()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---------------- device-resident timed region: CUDA-graph RK4 steps + H every 20 steps
    stream = grid.make_stepper(mode=args.mode, mixed=False, steps_per_graph=1)
    h_hist = []
    with torch.cuda.stream(stream):
        grid.run_stepper(args.warmup)
        grid.constraint_norms()
    torch.cuda.synchronize()
    grid.y_n.copy_(y0)
    barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = lib.bssn_b200_kernel_launches()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            done = 0
            while done < args.steps:
                n = min(H_EVERY, args.steps - done)
                grid.run_stepper(n)
                done += n
                if done % H_EVERY == 0:
                    h_hist.append(grid.constraint_norms()["H_L2"])
            stop.record(stream)
        stop.synchronize()
    launches = lib.bssn_b200_kernel_launches() - launches0
    ms = start.elapsed_time(stop)
    value, ms = aggregate(pts, args.steps, ms, dist, device="cuda")
    clocks = clk.summary()

    y_fp64 = grid.y_n.clone()
    y0_host = y0.cpu().numpy() if rank == 0 else None
    mixed = None if args.no_mixed else run_mixed(grid, args, y0, y_fp64, h_hist, stream)

    # ---------------- dominant kernel alone: fused interior RHS + RK update, per stage
    kstats = time_fused_kernel(grid, lib, stream, reps=5)
    peak, peak_kind = peaks()
    bytes_launch = np.mean(STAGE_WORDS) * 8 * pts
    achieved = bytes_launch / (kstats["ms_per_launch"] * 1e-3) / 1e9
    fp64 = None
    if FD_ORDER in RHS_FLOP_PER_PT_STAGE:
        tf = C.c_double()
        L.check(lib.bssn_b200_fp64_fma_rate(5, C.byref(tf), C.c_void_p(stream.cuda_stream)))
        flop = RHS_FLOP_PER_PT_STAGE[FD_ORDER] * pts
        fp64_achieved = flop / (kstats["ms_per_launch"] * 1e-3) / 1e12
        fp64 = {"achieved": fp64_achieved, "peak": tf.value, "unit": "TFLOP/s", "frac": fp64_achieved / tf.value,
                "flop_per_point": RHS_FLOP_PER_PT_STAGE[FD_ORDER],
                "peak_source": "measured: independent FP64 FMA chains on every SM (bssn_b200_fp64_fma_rate)"}

    # ---------------- baseline leg: the reference's own CUDA build on this GPU, same state
    ref_gpu = None
    if rank == 0 and not args.no_ref_gpu:
        try:
            ref_gpu = run_reference_gpu(grid, args, y0, value / world)
        except Exception as e:  # noqa: BLE001
            ref_gpu = {"unavailable": str(e)}

    # ---------------- end-to-end through the public API with host buffers
    e2e = None if args.no_e2e else run_e2e(grid, args, y0)
    diag = None if (args.no_diag or rank != 0) else run_diagnostics(grid, args)
    ckpt = None if (args.no_diag or rank != 0) else run_checkpoint(grid, args)
    grid_dt = grid.dt
    grid.free_stepper()
    grid.close()
    del grid, y0, y_fp64
    torch.cuda.empty_cache()
    # The adjoint is built at 4th order only; the batched workload (grids down to Nxx2 = 2) is
    # measured at 4th order, its 8th-order test covering Nxx2 >= 4.
    batched = None if (args.no_batched or FD_ORDER != 4) else run_batched(args, world, rank, dist)
    differentiation = None if (args.no_diff or rank != 0 or FD_ORDER != 4) else run_differentiation()
    cylindrical = None if (args.no_cyl or rank != 0) else run_cylindrical(args)

    if rank == 0:
        cpu = None
        y_cmp = mixed.pop("_y_cmp", None) if mixed else None
        if not args.no_cpu_baseline:
            try:
                cpu = cpu_reference_rate(3, 5, 3, args.seed)
            except Exception as e:  # noqa: BLE001
                cpu = {"unavailable": str(e)}
            if mixed is not None and y_cmp is not None:
                try:
                    mixed.update(mixed_vs_reference(y0_host, y_cmp, mixed["compare_steps"], args.seed))
                except Exception as e:  # noqa: BLE001
                    mixed["oracle_unavailable"] = str(e)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (Brill-Lindquist initial data, seeded)",
            "config": bench_config(args.seed, world),
            "mode": "fused stages" if args.mode == 1 else "reference stage order",
            "l2": "inputs larger than L2 (5 state buffers x 246 MB), no flush",
            "dt": grid_dt, "H_L2_last": h_hist[-1] if h_hist else None,
            "roofline": {"bound": "hbm", "kernel": "rhs_fused_kernel, all output groups (one interior RK stage: RHS + RK4 update + projection)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind,
                         "traffic": profiled_traffic() if NXX == (256, 64, 64) and FD_ORDER == 4 else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the two rhs group "
                                           "launches of one stage at 256x64x32, scaled by point count",
                         "algorithmic_bytes_per_launch": bytes_launch, "ms_per_launch": kstats["ms_per_launch"],
                         "step_achieved": value / world * B_ALG_PER_PT_STEP / 1e9,
                         "step_frac": value / world * B_ALG_PER_PT_STEP / 1e9 / peak,
                         "fp64": fp64},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "mixed_value": mixed["value"] if mixed else None,
            "mixed_H_L2": mixed.get("H_L2_at_compare") if mixed else None,
            "mixed_H_L2_oracle": mixed.get("H_L2_oracle") if mixed else None,
            "mixed_H_L2_fp64": mixed.get("H_L2_fp64_at_compare") if mixed else None,
            "mixed_rel_l2_vs_oracle_max": mixed.get("rel_l2_vs_oracle_max") if mixed else None,
            "mixed_compare_steps": mixed.get("compare_steps") if mixed else None,
            "batched_value": batched["value"] if batched else None,
            "mixed": mixed,
            "batched": batched,
            "differentiation": differentiation,
            "diagnostics": diag,
            "checkpoint": ckpt,
            "cylindrical": cylindrical,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def mixed_vs_reference(y0_host, y_mixed, steps, seed):
    """The reference's generated C (host cores) advanced `steps` RK4 steps from the bench's
    initial state: its H-constraint L2 (its Ricci_eval + constraints_eval, volume measure of
    diagnostics_volume_integration) and the per-gridfunction relative L2 of the mixed run's
    state against it (gridfunctions that vanish analytically, the phi components for holes on
    the z axis, are measured against the largest gridfunction's norm)."""
    from oracle import ref

    m1, z1, m2, z2 = bl_params(seed)
    rg = ref.RefGrid(SINH_VARIANT, NXX, AMPL, SINHW=SINHW, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2)
    try:
        rg.set_y_n(y0_host)
        rg.step(steps)
        yr = rg.y_n()
        h = rg.h_l2(yr)
    finally:
        rg.close()
    r = yr.reshape(24, -1)
    m = y_mixed.reshape(24, -1)
    num = np.sqrt(((m - r) ** 2).sum(axis=1))
    den = np.sqrt((r**2).sum(axis=1))
    rel = num / np.where(den < 1e-8 * den.max(), den.max(), den)
    return {"H_L2_oracle": h, "rel_l2_vs_oracle_max": float(rel.max()),
            "rel_l2_vs_oracle_per_gf": [float(x) for x in rel]}


def run_reference_gpu(grid, args, y0, our_value):
    """Baseline leg: the reference's own GPU step (nrpy --cuda, its generated
    MoL_step_forward_in_time compiled for sm_100a; oracle/_ref/sinh3d_cuda) on the same grid
    and initial state, timed with CUDA events on its stream over the same number of RK4 steps
    after 3 warm-up steps; one step from the shared state is first compared with this
    library's step (per-gridfunction relative L2), so the timed code is known to compute the
    same evolution."""
    import torch

    from oracle import ref

    if not ref.cuda_available("sinh3d_cuda") or FD_ORDER != 4:
        return {"unavailable": "oracle/_ref/sinh3d_cuda not built (python oracle/gen_ref.py --variants sinh3d_cuda)"}
    m1, z1, m2, z2 = bl_params(args.seed)
    y_host = y0.cpu().numpy()
    rc = ref.RefCudaGrid(NXX, AMPL, SINHW=SINHW, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2)
    try:
        rc.set_y_n(y_host)
        rc.steps(1)
        y_ref = rc.y_n().reshape(24, -1)
        grid.y_n.copy_(y0)
        grid.MoL_step_forward_in_time(mode=args.mode)
        torch.cuda.synchronize()
        mine = grid.y_n.view(24, -1).cpu().numpy()
        num = np.sqrt(((mine - y_ref) ** 2).sum(axis=1))
        den = np.sqrt((y_ref**2).sum(axis=1))
        # each gridfunction's difference against the largest gridfunction's norm (several
        # components start at zero and hold rounding-size values after one step)
        rel = num / den.max()
        grid.y_n.copy_(y0)
        rc.set_y_n(y_host)
        rc.steps(3)  # warm-up
        rc.set_y_n(y_host)
        ms = rc.steps(args.steps)
    finally:
        rc.close()
    pts = NXX[0] * NXX[1] * NXX[2]
    v = pts * args.steps / (ms * 1e-3)
    return {"value": v, "unit": UNIT, "ms_per_step": ms / args.steps, "steps": args.steps,
            "speedup_of_this_library": our_value / v,
            "one_step_l2_diff_vs_this_library_max": float(rel.max()),
            "one_step_l2_diff_measure": "max over gridfunctions of ||reference GPU - this library|| / ||largest gridfunction||",
            "what": "the reference's generated CUDA (nrpy --cuda: Ricci_eval, rhs_eval, BCs, rk_substep_*, "
                    "enforce_detgammabar kernels) compiled with nvcc -O2 -arch=sm_100a -rdc=true, timed with "
                    "CUDA events around its MoL_step_forward_in_time calls"}


def oracle_steps(steps: int) -> int:
    """Steps at which the mixed run is compared with the reference on the host: the run's
    length capped at 40 (the reference takes about 0.2 s per step of this grid on 16 cores),
    a multiple of the H-constraint cadence."""
    return max(H_EVERY, (min(steps, 40) // H_EVERY) * H_EVERY)


def run_mixed(grid, args, y0, y_fp64, h_fp64, stream):
    """Same workload with the Ricci/RHS algebra in FP32 (stencils, state, RK accumulation,
    detgammabar projection and constraint reductions in FP64): rate, H-constraint L2 next
    to the FP64 run's, and the per-gridfunction relative L2 of the final state vs FP64. The
    state after oracle_steps() steps is kept (host copy) for the comparison with the
    reference."""
    import torch

    grid.free_stepper()
    grid.y_n.copy_(y0)
    st = grid.make_stepper(mode=args.mode, mixed=True, steps_per_graph=1)
    with torch.cuda.stream(st):
        grid.run_stepper(args.warmup)
    torch.cuda.synchronize()
    grid.y_n.copy_(y0)
    torch.cuda.synchronize()
    h = []
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        a.record(st)
        done = 0
        while done < args.steps:
            n = min(H_EVERY, args.steps - done)
            grid.run_stepper(n)
            done += n
            if done % H_EVERY == 0:
                h.append(grid.constraint_norms()["H_L2"])
        b.record(st)
    b.synchronize()
    ms = a.elapsed_time(b)
    # untimed: the mixed state at the step count compared with the reference
    ncmp = oracle_steps(args.steps)
    grid.y_n.copy_(y0)
    with torch.cuda.stream(st):
        grid.run_stepper(ncmp)
    torch.cuda.synchronize()
    y_cmp = grid.y_n.cpu().numpy()
    m = grid.y_n.view(24, -1)
    f = y_fp64.view(24, -1)
    num = torch.linalg.vector_norm(m - f, dim=1)
    den = torch.linalg.vector_norm(f, dim=1).clamp_min(1e-300)
    rel = (num / den).cpu().numpy()
    nz = (torch.linalg.vector_norm(f, dim=1) > 1e-12 * torch.linalg.vector_norm(f, dim=1).max()).cpu().numpy()
    grid.free_stepper()
    return {"value": grid.n_interior * args.steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / args.steps,
            "_y_cmp": y_cmp, "compare_steps": ncmp, "H_L2_at_compare": h[ncmp // H_EVERY - 1] if len(h) >= ncmp // H_EVERY else None,
            "H_L2_fp64_at_compare": h_fp64[ncmp // H_EVERY - 1] if len(h_fp64) >= ncmp // H_EVERY else None,
            "dtype": "f32 algebra / f64 state", "H_L2": h[-1] if h else None,
            "H_L2_fp64": h_fp64[-1] if h_fp64 else None,
            "H_L2_rel_diff": (abs(h[-1] - h_fp64[-1]) / h_fp64[-1]) if h and h_fp64 else None,
            "rel_l2_vs_fp64_max": float(rel[nz].max()) if nz.any() else None,
            "rel_l2_vs_fp64_per_gf": [float(x) for x in rel]}


def run_batched(args, world, rank, dist):
    """64 independent Brill-Lindquist evolutions (Spherical, Nxx ~ [48..128]x[8..32]x[2..16])
    advanced together: autotuned tile shape, one captured CUDA graph of 20 RK4 steps
    replayed; compared with the same evolutions advanced one grid at a time."""
    import torch

    from nrpy_b200.batch import BatchedEvolutions, batching_workload, partition_evolutions

    specs = batching_workload(seed=7, n=64)
    sizes = [s["Nxx"][0] * s["Nxx"][1] * s["Nxx"][2] for s in specs]
    mine = partition_evolutions(sizes, world)[rank]
    be = BatchedEvolutions([specs[i] for i in mine])
    if args.batch_tile:
        bx, by = (int(x) for x in args.batch_tile.split(","))
        tune = {"tile": (bx, by), "table": "not run (--batch-tile)"}
    else:
        tune = be.autotune(steps=2)
    spg = 20
    be.build(tile=tune["tile"], steps_per_graph=spg)
    be.run(1)
    torch.cuda.synchronize()
    steps = max(spg, (args.batch_steps // spg) * spg)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(be.stream)
    be.run(steps // spg)
    b.record(be.stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    pts = be.interior_points
    value, ms_max = aggregate(pts, steps, ms, dist, device="cuda")
    info = be.info()
    be.free()
    # the same evolutions one grid at a time (single-grid CUDA graphs), a few steps each
    seq_steps = 10
    seq_ms = 0.0
    for g in ([] if args.no_batch_sequential else be.grids):
        st = g.make_stepper(mode=1, steps_per_graph=seq_steps)
        with torch.cuda.stream(st):
            g.run_stepper(1)
        torch.cuda.synchronize()
        a2, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a2.record(st)
        with torch.cuda.stream(st):
            g.run_stepper(1)
        b2.record(st)
        b2.synchronize()
        seq_ms += a2.elapsed_time(b2)
        g.free_stepper()
    seq_value = aggregate(pts, seq_steps, seq_ms, dist, device="cuda")[0] if seq_ms > 0 else None
    be.close()
    return {"value": value, "unit": UNIT, "evolutions": len(specs), "steps": steps, "ms_per_step": ms_max / steps,
            "interior_points": pts if dist is None else None, "tile": list(tune["tile"]),
            "autotune": tune["table"], "graph_kernel_nodes_per_replay": info["kernel_nodes"],
            "tile_fill": info["tile_fill"],
            "sequential_single_grid_value": seq_value,
            "speedup_vs_sequential": value / seq_value if seq_value else None}


CYL_NXX = (400, 2, 1200)
CYL_L = 300.0


def run_cylindrical(args, steps: int = 20):
    """SinhCylindrical, axisymmetric about z, on blackhole_spectroscopy.py's grid (400x2x1200,
    AMPLRHO = AMPLZ = 300, SINHW 0.2) with this process's FD order and the bench's seeded
    Brill-Lindquist data: `steps` fused FP64 RK4 steps replayed from one CUDA graph, timed with
    CUDA events; beside it the reference's generated C of the same coordinates on the host
    cores (2 warm-up steps, median of 3 runs of 2 steps)."""
    import torch

    from nrpy_b200.grid import BSSNGrid

    m1, z1, m2, z2 = bl_params(args.seed)
    g = BSSNGrid(coord="SinhCylindrical", Nxx=CYL_NXX, grid_physical_size=CYL_L, SINHW=SINHW, BH1_mass=m1,
                 BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2, symmetry_axes="1")
    st = g.make_stepper(mode=1, steps_per_graph=steps)
    with torch.cuda.stream(st):
        g.run_stepper(1)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    with torch.cuda.stream(st):
        g.run_stepper(1)
    b.record(st)
    b.synchronize()
    ms = a.elapsed_time(b)
    pts = CYL_NXX[0] * CYL_NXX[1] * CYL_NXX[2]
    res = {"workload": f"SinhCylindrical {CYL_NXX[0]}x{CYL_NXX[1]}x{CYL_NXX[2]} (blackhole_spectroscopy's grid), "
                       f"AMPLRHO = AMPLZ = {CYL_L:g}, SINHW {SINHW}, symmetry_axes '1', {FD_ORDER}th-order FD, "
                       f"FP64 fused stages",
           "value": pts * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps}
    g.free_stepper()
    g.close()
    del g
    torch.cuda.empty_cache()
    if not args.no_cpu_baseline:
        try:
            from oracle import ref

            variant = "sinhcyl" if FD_ORDER == 4 else f"sinhcyl{FD_ORDER}"
            if ref.available(variant):
                rg = ref.RefGrid(variant, CYL_NXX, CYL_L, SINHW=SINHW, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2,
                                 BH2_posn_z=z2)
                rg.step(2)
                times = []
                for _ in range(3):
                    t0 = time.perf_counter()
                    rg.step(2)
                    times.append(time.perf_counter() - t0)
                rg.close()
                dt = float(np.median(times))
                res["reference_value"] = pts * 2 / dt
                res["reference_s_per_step"] = dt / 2
                res["reference_cores"] = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
                res["speedup_vs_reference"] = res["value"] / res["reference_value"]
        except Exception as e:  # noqa: BLE001
            res["reference_unavailable"] = str(e)
    return res


def run_diagnostics(grid, args, reps: int = 3):
    """One diagnostics() output step of the bench grid (Ricci + constraints on the device,
    nearest-point samples gathered on the device, volume integrals reduced on the device,
    the reference's ASCII files written), wall time per output step; beside it the
    reference's own diagnostics() on the host cores on the same grid and state."""
    import torch

    cwd = os.getcwd()
    res = {}
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        try:
            grid.diagnostics(1.0, nn=0, time=0.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k in range(reps):
                grid.diagnostics(1.0, nn=k + 1, time=0.0)
            torch.cuda.synchronize()
            res["ms_per_output"] = 1e3 * (time.perf_counter() - t0) / reps
            res["files"] = sorted(os.listdir(d))
        finally:
            os.chdir(cwd)
    n1, n2 = grid.N[1] - 6, grid.N[2] - 6
    n0 = grid.N[0] - 6
    samples = 1 + 4 * n0 + n0 * n2 + 2 * n0 * n1
    res["d2h_bytes_per_output"] = samples * 2 * 8 + 8 * 8
    # initial data (Brill-Lindquist -> BSSN on the device, lambda^i, BCs)
    t0 = time.perf_counter()
    grid.lib.initial_data(C.byref(grid.cd), grid.gd)
    torch.cuda.synchronize()
    res["initial_data_ms"] = 1e3 * (time.perf_counter() - t0)
    res["reference_cuda_path_d2h_bytes_per_output"] = grid.y_n.numel() * 8
    if not args.no_cpu_baseline:
        try:
            from oracle import ref

            if ref.available(SINH_VARIANT):
                m1, z1, m2, z2 = bl_params(args.seed)
                rg = ref.RefGrid(SINH_VARIANT, NXX, AMPL, SINHW=SINHW, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2,
                                 BH2_posn_z=z2)
                with tempfile.TemporaryDirectory() as d:
                    os.chdir(d)
                    try:
                        rg.diagnostics(0, 0.0, 1.0)
                        t0 = time.perf_counter()
                        rg.diagnostics(1, 0.0, 1.0)
                        res["reference_ms_per_output"] = 1e3 * (time.perf_counter() - t0)
                        t0 = time.perf_counter()
                        rg.initial_data()
                        res["reference_initial_data_ms"] = 1e3 * (time.perf_counter() - t0)
                    finally:
                        os.chdir(cwd)
                rg.close()
                res["reference_cores"] = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
        except Exception as e:  # noqa: BLE001
            res["reference_unavailable"] = str(e)
    return res


def run_checkpoint(grid, args, reps: int = 3):
    """write_checkpoint / read_checkpoint of the bench grid's state (the reference's file format,
    252 MB at 256x64x64): wall time per call, the restored state checked bit-for-bit; beside it
    the reference's own write_checkpoint / read_checkpoint (checkpoint-enabled project, same
    grid size) on the host cores. Each side writes `reps` times, each time to a new file, then
    reads `reps` times; best and median are reported, since the host's file system (page cache
    or disk) sets much of the time."""
    import torch

    cwd = os.getcwd()
    res = {}

    def timed(d, write, read):
        wt, rt = [], []
        for _ in range(reps):
            for f in os.listdir(d):
                os.remove(os.path.join(d, f))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            write()
            wt.append(1e3 * (time.perf_counter() - t0))
        size = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
        for _ in range(reps):
            t0 = time.perf_counter()
            read()
            torch.cuda.synchronize()
            rt.append(1e3 * (time.perf_counter() - t0))
        return wt, rt, size

    y_saved = grid.y_n.clone()
    clock = (grid.cd.nn, grid.cd.time, grid.cd.t_0, grid.cd.nn_0)
    every = grid.cd.time if grid.cd.time > 0 else 1.0
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        try:
            wt, rt, size = timed(d, lambda: grid.write_checkpoint(every), lambda: grid.read_checkpoint())
            res.update({"write_ms": float(np.median(wt)), "write_ms_best": min(wt), "read_ms": float(np.median(rt)),
                        "read_ms_best": min(rt), "file_bytes": size,
                        "restored_bitwise": bool(torch.equal(grid.y_n, y_saved))})
        finally:
            os.chdir(cwd)
    grid.cd.nn, grid.cd.time, grid.cd.t_0, grid.cd.nn_0 = clock
    grid.y_n.copy_(y_saved)
    del y_saved
    if not args.no_cpu_baseline:
        try:
            from oracle import ref

            if ref.available("sph3dck"):
                rg = ref.RefGrid("sph3dck", NXX, 7.5)
                rg.set_clock(1, rg.dt)
                with tempfile.TemporaryDirectory() as d:
                    os.chdir(d)
                    try:
                        wt, rt, _ = timed(d, lambda: rg.write_checkpoint(rg.dt), lambda: rg.read_checkpoint())
                        res.update({"reference_write_ms": float(np.median(wt)), "reference_write_ms_best": min(wt),
                                    "reference_read_ms": float(np.median(rt)), "reference_read_ms_best": min(rt)})
                    finally:
                        os.chdir(cwd)
                rg.close()
                res["reference_cores"] = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
        except Exception as e:  # noqa: BLE001
            res["reference_unavailable"] = str(e)
    return res


def run_differentiation(fd_check: bool = True):
    """Adjoint gradient dJ/d(m1, z1, m2, z2) of J = sum_interior H^2 + alpha(centre) after 200
    FP64 RK4 steps on Spherical 128x32x32 (checkpoints every 20), timed forward and backward
    (CUDA events on the grid's stream), checked against central differences (h = 1e-6) of
    the forward."""
    import torch

    from nrpy_b200.adjoint import BLGradient, differentiation_workload

    w = differentiation_workload(seed=2024)
    p = BLGradient(Nxx=w["Nxx"], grid_physical_size=w["grid_physical_size"], nsteps=w["nsteps"],
                   checkpoint_every=w["checkpoint_every"], theta=w["theta"])
    p.value_and_grad(w["theta"])  # warm-up
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    J = p.forward(w["theta"])
    ev[1].record(stream)
    grad = p.backward(1.0)
    ev[2].record(stream)
    ev[2].synchronize()
    ms_f, ms_b = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    res = {"workload": "Spherical 128x32x32 (+3 ghosts), grid_physical_size 7.5, 200 FP64 RK4 steps, radiation BCs, "
                       "checkpoints every 20; J = sum_interior H^2 + alpha(NGHOSTS, N1/2, N2/2)",
           "theta_names": ["BH1_mass", "BH1_posn_z", "BH2_mass", "BH2_posn_z"], "theta": list(w["theta"]),
           "seed": w["seed"], "J": J["J"], "grad": [float(x) for x in grad], "ms_forward": ms_f,
           "ms_backward": ms_b, "backward_over_forward": ms_b / ms_f,
           "pt_updates_per_s_forward": p.grid.n_interior * w["nsteps"] / (ms_f * 1e-3),
           "pt_updates_per_s_backward": p.grid.n_interior * w["nsteps"] / (ms_b * 1e-3)}
    if fd_check:
        h = 1e-6
        fd = []
        for k in range(4):
            tp, tm = list(w["theta"]), list(w["theta"])
            tp[k] += h
            tm[k] -= h
            fd.append((p.forward(tp)["J"] - p.forward(tm)["J"]) / (2 * h))
        res["central_fd_h"] = h
        res["central_fd"] = fd
        res["rel_err_vs_fd"] = [abs(a - b) / abs(b) for a, b in zip(grad, fd)]
    p.close()
    return res


def time_fused_kernel(grid, lib, stream, reps: int = 5):
    import torch

    from nrpy_b200 import lib as L

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(4 * reps)]
    k = 0
    for r in range(reps):
        for stage in (1, 2, 3, 4):
            a, b = ev[k]
            a.record(stream)
            L.check(lib.bssn_b200_rhs_fused_stage(C.byref(grid.cd), grid.gd, stage, 0, C.c_void_p(stream.cuda_stream)))
            b.record(stream)
            k += 1
    torch.cuda.synchronize()
    t = [a.elapsed_time(b) for a, b in ev[4:]]  # first round is warm-up
    return {"ms_per_launch": float(np.mean(t))}


def run_e2e(grid, args, y0):
    """End to end through the public API with host buffers: per step, the state is uploaded
    from pinned host memory, advanced one RK4 step by BSSNGrid.step_from_host and downloaded to
    pinned host memory; the H-constraint L2 is read back every 20 steps. step_from_host
    overlaps the uploads and downloads with the steps (two device state buffers, copy
    streams). The same loop with the copies in line with the steps is reported beside it."""
    import torch

    host_in = y0.cpu().pin_memory()
    host_out = [torch.empty_like(host_in).pin_memory() for _ in range(2)]
    steps = min(args.steps, 50)
    cur = torch.cuda.current_stream()

    def metric(i, y):
        if (i + 1) % H_EVERY == 0:
            grid.constraint_norms(y)

    grid.step_from_host([host_in] * 3, [host_out[k % 2] for k in range(3)], mode=args.mode)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(cur)
    grid.step_from_host([host_in] * steps, [host_out[k % 2] for k in range(steps)], mode=args.mode, on_step=metric)
    b.record(cur)
    b.synchronize()
    ms = a.elapsed_time(b)
    # in line: upload, step, download one after the other on one stream
    a.record(cur)
    for s in range(steps):
        grid.y_n.copy_(host_in, non_blocking=True)
        grid.MoL_step_forward_in_time(mode=args.mode)
        host_out[0].copy_(grid.y_n, non_blocking=True)
        metric(s, grid.y_n)
    b.record(cur)
    b.synchronize()
    ms_seq = a.elapsed_time(b)
    nbytes = grid.y_n.numel() * 8
    return {"value": grid.n_interior * steps / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "steps": steps, "copies": "overlapped with the steps (two device buffers)",
            "in_line_value": grid.n_interior * steps / (ms_seq * 1e-3)}


if __name__ == "__main__":
    main()
