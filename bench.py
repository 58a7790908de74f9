"""bench.py -- timestep throughput of the B200 DPD engine (one JSON line on rank 0).

Headline workload: the binary A5B5 diblock melt -- periodic 100^3 box at density 3,
N = 3.0M beads in 300k linear 10-bead chains, harmonic bonds k=4 r0=0, a_AA=a_BB=25,
a_AB=40, gamma=4.5, kT=1, dt=0.04 -- seeded synthetic input (chains grown as random walks
with step 0.9; no dataset), skin 0 (the tuner's choice: this system rebuilds its list
every step at any skin up to 0.3).  A step is one velocity-Verlet timestep of the whole
system (list build when due, pair+bond forces with the Saru random force, fused
integration).  Value: particle-steps/s.

Beside it (N=1 only): "batched" -- 256 uneven A/B mixtures in one packed engine against
the plain engine one replica at a time; "served" -- a Poisson stream of jobs through the
continuous-batching server (p50/p99 latency) against the plain engine one job at a time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent replica per GPU (replicas only: the single system is not
decomposed), launched by torch.distributed.run; value sums all ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s: batched/served vs plain at matched P,T error; p50/p99 latency"


def workload_name(args):
    if args.workload == "melt":
        return f"a5b5_diblock_melt_L100_N3M_skin{args.skin}"
    return f"{args.workload}_skin{args.skin}"


def build_launches(system, skin, pair_variant=8):
    """Kernels of one list build: counting pass, scan (one launch when the cells fit one
    4096-element block, else three), permutation (with the parity flip up to 1184 blocks
    of 256 slots, else a separate flip), list (none with the cell-tile schedule 11)."""
    cells = int(np.prod(np.floor(system.box / (1.0 + skin)))) + 1
    slots = system.n + 31
    return (2 if pair_variant == 11 else 3) + (1 if cells <= 4096 else 3) + \
        (0 if (slots + 255) // 256 <= 148 * 8 else 1)


def pair_kernel_name(system, pair_variant):
    """The pair kernel the engine launches for this system: on tiny grids (up to 148 blocks
    of 256 slots) one thread per list entry, on small grids (up to 1184) the flattened
    schedule as one launch, else the flattened schedule split by log steps."""
    gp = (system.n + 31 + 255) // 256
    if pair_variant == 11:
        return "k_tile + k_tile_logsteps (cell tiles staged in shared memory, no list)"
    if pair_variant == 8 and gp <= 148:
        return "k_pair_entry (thread per list entry, tiny grids)"
    if pair_variant == 8 and gp <= 148 * 8:
        return "k_pair_flat (flattened pair schedule, one launch on small grids)"
    return "k_pair_flat_split + k_pair_flat_logsteps (flattened pair schedule)"


def step_launches(system, pair_variant):
    """Kernels of one step after the list build: on small grids (up to 1184 blocks of 256
    slots) the pair pass and the integrate with the bookkeeping are one launch each; else
    the pair kernel(s), the integrate pair (non-log steps + log steps) and advance."""
    small = (system.n + 31 + 255) // 256 <= 148 * 8
    if small and pair_variant == 8:
        return 2
    if pair_variant == 11:
        return 2 + (1 if small else 3)
    return (2 if pair_variant in (7, 8, 9) else 1) + 3


def thermo_every(args):
    """Thermo cadence of the headline run, shared by both arms: the reference prints a
    thermo line every N steps and is timed between its lines at steps W and W+K, so N
    divides both W and K; logged steps cost both engines their virial/energy variants."""
    return math.gcd(args.warmup, args.steps)


def make_system(args, thermo=1000):
    from gpumdpd_b200 import inputs
    if args.workload == "melt":
        return inputs.diblock_melt(L=100.0, seed=7, nsteps=10 ** 6, thermo=thermo, skin=args.skin)
    if args.workload == "melt_mid":
        return inputs.diblock_melt(L=60.0, seed=7, nsteps=10 ** 6, thermo=thermo, skin=args.skin)
    if args.workload == "melt_small":
        return inputs.diblock_melt(L=30.0, seed=7, nsteps=10 ** 6, thermo=thermo, skin=args.skin)
    if args.workload == "plain":
        return inputs.plain_dpd(L=10.0, seed=2024, nsteps=10 ** 6, thermo=thermo, skin=args.skin)
    if args.workload == "slab":
        return inputs.mdpd_slab(nsteps=10 ** 6, thermo=thermo, skin=args.skin)
    raise SystemExit(f"unknown workload {args.workload}")


def block_stats(series, nblocks=10):
    """Mean and its standard error from block averages (consecutive blocks of equal
    length; rows that do not fill a block are left out of the error estimate)."""
    x = np.asarray(series, dtype=np.float64)
    nb = min(nblocks, len(x) // 2)
    if nb < 2:
        return float(x.mean()), float("nan")
    ln = len(x) // nb
    b = x[: nb * ln].reshape(nb, ln).mean(axis=1)
    return float(x.mean()), float(b.std(ddof=1) / math.sqrt(nb))


def compare(a, b, nblocks=10):
    """a (FP32 engine) against b (FP64 engine) for one observable's series over the same
    window: both means, their difference, its combined standard error and the ratio."""
    ma, sa = block_stats(a, nblocks)
    mb, sb = block_stats(b, nblocks)
    se = math.sqrt(sa * sa + sb * sb)
    return {"fp32": round(ma, 6), "fp64": round(mb, 6), "err": round(ma - mb, 6),
            "stderr": round(se, 6), "z": round((ma - mb) / se, 2) if se > 0 else None}


def compact(x, sig=4):
    """Floats of a nested summary rounded to `sig` significant digits (the printed line)."""
    if isinstance(x, float):
        return float(f"{x:.{sig}g}") if math.isfinite(x) else None
    if isinstance(x, dict):
        return {k: compact(v, sig) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [compact(v, sig) for v in x]
    return x


def with_thermo(run_in, every):
    import re
    return re.sub(r"(?m)^thermo \d+$", f"thermo {int(every)}", run_in)


def without_computes(run_in):
    """The run.in without its `compute` lines (the FP64 parity engine runs the force field
    and fix nve only; sampling computes do not change the trajectory)."""
    return "".join(ln + "\n" for ln in run_in.splitlines() if not ln.startswith("compute "))


def with_run(run_in, steps):
    import re
    return re.sub(r"(?m)^run \d+$", f"run {int(steps)}", run_in)


def state_system(s, x, v, run_in):
    """The system `s` at state (x, v) in tag order, with another run.in."""
    from gpumdpd_b200 import inputs
    return inputs.System(s.lo, s.hi, s.masses, s.types, x, v, bonds=s.bonds, n_bondtypes=s.n_bondtypes,
                         mol=s.mol, run_in=run_in, atom_style=s.atom_style, angles=s.angles,
                         n_angletypes=s.n_angletypes)


def fp32_fp64_window(s, x, v, steps, every, fields=("temp", "pressure"), extra=None, tuning=None):
    """Run the FP32 engine and the FP64 parity engine (the reference's -DDOUBLE
    arithmetic, pinned to the FP64 oracle by the test suite) from the same state (x, v)
    for `steps` steps with thermo every `every` steps; compare each field's mean over the
    rows after the first.  `extra` maps a name to a function of the thermo dict giving
    another series."""
    from gpumdpd_b200 import Engine
    run_in = with_run(with_thermo(without_computes(s.run_in), every), steps)
    rows = {}
    t = {}
    for prec in ("fp32", "fp64"):
        sysp = state_system(s, x, v, run_in)
        e = Engine(run_in, system=sysp.c_system(), precision=prec)
        if prec == "fp32" and tuning:
            e.set_tuning(**tuning)
        t0 = time.perf_counter()
        e.run(steps)
        t[prec] = time.perf_counter() - t0
        rows[prec] = e.thermo()
        e.close()
    out = {}
    for f in fields:
        out[f] = compare(rows["fp32"][f][1:], rows["fp64"][f][1:])
    for name, fn in (extra or {}).items():
        out[name] = compare(fn(rows["fp32"])[1:], fn(rows["fp64"])[1:])
    out["window"] = {"steps": steps, "thermo_every": every, "rows": int(len(rows["fp32"]["temp"]) - 1)}
    return out


class ClockSampler:
    """SM clocks and clock-event reasons read through NVML every 2 ms while the timed
    region runs (read-only queries: nothing about the GPU is changed).  A first sample is
    taken on entry, so a region of a few milliseconds still has samples; nvidia-smi's
    200 ms loop is the fallback when NVML cannot be loaded."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = int(gpu_index)
        self.rows = []  # (sm_mhz, max_mhz, {reason names})
        self.proc = None
        self.stop = threading.Event()
        self.thread = None

    def _nvml_loop(self, nv, h):
        while True:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.rows.append((float(sm), float(mx), {n for n, a in self.REASONS if bits & getattr(nv, a)}))
            if self.stop.wait(0.002):
                break

    def _smi_read(self):
        for line in self.proc.stdout:
            r = [c.strip() for c in line.split(",")]
            try:
                names = {n for k, (n, _) in enumerate(self.REASONS) if len(r) > 5 + k and r[5 + k].lower() == "active"}
                self.rows.append((float(r[1]), float(r[2]), names))
            except ValueError:
                pass

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = None
            try:  # the CUDA device itself (NVML numbers devices regardless of CUDA_VISIBLE_DEVICES)
                import torch
                u = str(torch.cuda.get_device_properties(self.gpu).uuid)
                h = nv.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
            while not self.rows:  # the first sample before the timed region starts
                time.sleep(0.0005)
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._smi_read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[0] for r in self.rows]
        reasons = sorted(set().union(*[r[2] for r in self.rows]))
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": reasons, "samples": len(self.rows),
                "source": "nvml" if self.proc is None else "nvidia-smi"}


def dist_setup(args, backend="nccl"):
    """One process per GPU (torch.distributed.run sets RANK/LOCAL_RANK/WORLD_SIZE).  The
    only collectives are the barriers around the timed region and the max-over-ranks of
    its time: replicas share nothing on the step path."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            os.environ["DPD_B200_DEVICE"] = str(local)  # the engine library's device
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(n_per_rank, steps, local_ms, world):
    """Whole-job particle-steps/s: every rank advances its own replica of n particles, and
    the job takes as long as the slowest rank."""
    total_ms = allreduce_max(local_ms, world)
    return world * n_per_rank * steps / (total_ms / 1000.0), total_ms


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def algorithmic_bytes_per_particle(mean_half_list, maxb, pair_variant=8):
    """Pair kernel, per particle-step: x,v of i (32 B) + force write (12 B) + list length
    (4 B) + list entries (4 B each); neighbour-j gathers are assumed cache-resident and not
    counted.  The fused bonds add their partner table (8 B per slot).  The cell-tile
    schedule (11) reads no list: 44 B + bonds."""
    if pair_variant == 11:
        return 44.0 + 8.0 * maxb
    return 48.0 + 4.0 * mean_half_list + 8.0 * maxb


def cpu_baseline(system, nthreads, nsteps=2, engine_state0=None):
    """FP64 oracle port of the reference algorithm (pair forces with the Saru random force
    on a half Verlet list, bonds, velocity Verlet) on the host cores: a bounded sample of
    the workload.  Given the engine's state after its zero step, the oracle also checks
    the engine's step-0 forces on that state (largest per-particle error over the RMS
    force)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    ff = oracle.ff_from_run_in(system.run_in, system.masses)
    tags = np.arange(1, system.n + 1)
    t0 = time.perf_counter()
    oracle.bench_steps(ff, tags, system.types, system.x, system.v, system.lo, system.box, 1, nsteps,
                       0.3, nthreads, bonds=system.bonds)
    dt = time.perf_counter() - t0
    out = {"value": system.n * nsteps / dt, "unit": "particle-steps/s", "cores": nthreads,
           "kind": "port",
           "sample": f"full {system.n}-particle system: step-0 forces + {nsteps} steps incl. one list "
                     f"build, FP64, pair + bond forces, {nthreads} threads; {dt:.1f} s"}
    if engine_state0 is not None:
        o = oracle.forces(ff, tags, system.types, engine_state0["x"], engine_state0["v"], system.lo,
                          system.box, 0, bonds=system.bonds)
        rms = float(np.sqrt((np.linalg.norm(o["f"], axis=1) ** 2).mean()))
        err = np.linalg.norm(engine_state0["f"] - o["f"], axis=1).max() / rms
        out["step0_force_max_err_over_rms"] = float(err)
    return out


def run_ours(args, world, rank, local):
    import torch
    from gpumdpd_b200 import Engine
    tuned = "defaults (skin and schedule chosen by gpumdpd_b200/tune.py on this workload)"
    if args.tune:
        from gpumdpd_b200 import tune
        best, table = tune.tune_system(make_system(args))
        args.skin = best["skin"]
        args.pair_variant = best["pair_variant"]
        tuned = {"best": best, "table": table}
    every = thermo_every(args)
    system = make_system(args, thermo=every)
    eng = Engine(system.run_in, system=system.c_system())
    pair_variant = 8 if args.pair_variant is None else args.pair_variant
    eng.set_tuning(pair_variant=pair_variant, tile=args.tile, pair_block=args.pair_block, **list_tuning(args))
    eng.run(0)
    st0 = eng.state(images=False) if rank == 0 and world == 1 and not args.no_cpu_baseline else None
    eng.run(args.warmup)
    ls = eng.list_stats()
    b0 = eng.info()["builds"]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        res = eng.time_steps(args.steps)
    torch.cuda.synchronize()
    barrier(world)
    builds_per_step = (eng.info()["builds"] - b0) / args.steps
    n = system.n
    value, total_ms = job_value(n, args.steps, res["total_ms"], world)
    pair_ms = res["pair_ms"]
    # end to end through the C ABI with host buffers: the state (x, v in FP64) goes host
    # -> device, K steps run (a zero-step force evaluation and list build first), the
    # final x, v come back device -> host with the thermo rows
    # (chunks of at least 1000 steps: a production call runs many steps per upload)
    chunk = max(args.steps, 1000)
    st = eng.state(forces=False, images=False)
    x = np.ascontiguousarray(st["x"])
    v = np.ascontiguousarray(st["v"])
    barrier(world)
    t0 = time.perf_counter()
    eng.set_state(x, v)
    eng.run(chunk)
    st2 = eng.state(forces=False, images=False)
    eng.thermo(max_rows=4)
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    e2e = world * n * chunk / e2e_s
    h2d = n * 6 * 8 / chunk
    d2h = (n * 6 * 8 + 4 * 8 * 16) / chunk
    maxb = 2 if system.bonds is not None else 0
    bpp = algorithmic_bytes_per_particle(ls["mean_half_list"], maxb, pair_variant)
    per_launch_ms = pair_ms / max(res["pair_launches"], 1)
    achieved = n * bpp / (per_launch_ms / 1000.0) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    # state (two parity buffers of position, velocity, image and bond partners) + half list
    foot = n * (2 * (48 + 8 * maxb) + 4 * 48 + 16)
    l2 = (f"inputs > L2 ({foot / 1e9:.2f} GB)" if foot > 126e6 else
          f"inputs < L2 ({foot / 1e6:.1f} MB), no flush: small latency-bound system")
    traffic, wipp = None, None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        t = prof.get(args.workload)
        if t and pair_variant == 8:
            traffic = t["dram_bytes_per_launch"]
            wipp = t.get("warp_instr_per_particle")
    except Exception:
        pass
    clk_summary = clk.summary()
    pairs_per_step = ls["pairs"]
    out = {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64-reductions",
        "data": "synthetic (seeded generator, gpumdpd_b200/inputs.py)",
        "config": {"workload": workload_name(args), "n_particles": n,
                   "n_bonds": 0 if system.bonds is None else len(system.bonds), "box": system.box.tolist(),
                   "dt": 0.04, "skin": args.skin, "thermo_every": every,
                   "mean_half_list": round(ls["mean_half_list"], 3),
                   "list_builds_per_step": builds_per_step, "pair_variant": pair_variant,
                   "tile": args.tile if pair_variant == 11 else None,
                   "tuned": "defaults (tune.py)" if isinstance(tuned, str) else "bench --tune",
                   "parallelism": f"replicas{world}", "l2": l2},
        "e2e": {"value": e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "chunk_steps": chunk, "path": "dpd_set_state+dpd_run+dpd_get_state"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": pair_kernel_name(system, pair_variant),
                     "bytes_per_particle": bpp, "pair_ms_per_launch": per_launch_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback",
                     # the kernel is issue-bound, not HBM-bound: the Saru chain's integer
                     # operations per pair inside rc set the compute-side ceiling
                     "binding": "issue (Saru integer chain), not HBM",
                     "pairs_per_step": pairs_per_step,
                     "saru_int_ops_per_pair": 130},
        "clocks": clk_summary,
        # per step: the list-build kernels (counting pass, 1 or 3 scan launches, permutation,
        # list; each returns at once unless a build is flagged), the pair kernel(s), the
        # integrate pair (non-log steps + log steps), advance; plus 2 before the graph
        "gpu_launches": int(args.steps * (build_launches(system, args.skin, pair_variant) +
                                          step_launches(system, pair_variant)) + 2),
        "impl": "ours",
    }
    if wipp and clk_summary.get("sm_mhz"):
        # the instruction-issue ceiling of the pair kernel: its warp instructions (ncu count per
        # particle) at one instruction per clock on each of the 4 schedulers of 148 SMs
        ceil_ms = n * wipp / (148 * 4 * clk_summary["sm_mhz"] * 1e6) * 1e3
        out["roofline"]["issue"] = {"warp_instr_per_particle": wipp, "ceiling_ms": ceil_ms,
                                    "frac": ceil_ms / per_launch_ms, "sm_mhz": clk_summary["sm_mhz"]}
    if world == 1 and not args.no_extras:
        # T and P of the headline system: the FP32 engine against the FP64 parity engine
        # from the same state over the same window, after the melt's bonds have relaxed
        # (2000 more steps of the FP32 engine)
        eng.run(args.acc_equil)
        st3 = eng.state(forces=False, images=False)
        out["accuracy"] = compact(fp32_fp64_window(system, st3["x"], st3["v"], args.acc_steps, 5,
                                                   tuning={"pair_variant": pair_variant, **list_tuning(args)}))
        out["accuracy"]["from_step"] = args.warmup + args.steps + chunk + args.acc_equil
        del st3
    eng.close()
    del st, st2
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(system, os.cpu_count() or 1, engine_state0=st0)
        del st0
    detail = {}
    if world == 1 and not args.no_extras:
        for name, fn in (("slab", run_slab), ("batched", run_batched), ("served", run_served),
                         ("fp64", run_fp64)):
            summary, det = fn(args)
            out[name] = compact(summary)
            detail[name] = det
    if rank == 0:
        if detail and args.detail:
            with open(args.detail, "w") as f:
                json.dump(detail, f)
            out["detail_file"] = os.path.basename(args.detail)
        print(json.dumps(out), flush=True)


def run_slab(args):
    """Many-body DPD liquid slab: box 40x40x120, density 6 in z in [40,80] (N = 384k), A=-40,
    B=25, rc=1, rd=0.75, gamma=4.5, kT=1, dt=0.01, two-pass density then force, 20k steps
    timed on the device; the z density profile (bins 0.5) of the final state and
    gamma_s = (Lz/2)<P_zz - (P_xx+P_yy)/2> over the second half of the run; then T, P and
    gamma_s of the FP32 engine against the FP64 parity engine from the final state."""
    from gpumdpd_b200 import Engine, inputs, observables, tune
    s = inputs.mdpd_slab(nsteps=args.slab_steps, thermo=100)
    s.run_in = tune.with_skin(s.run_in, args.batch_skin)
    eng = Engine(s.run_in, system=s.c_system())
    eng.set_tuning(pair_variant=8, **list_tuning(args))
    eng.run(0)
    total_ms, done = 0.0, 0
    while done < args.slab_steps:  # timed in graphs of at most 500 steps
        k = min(500, args.slab_steps - done)
        total_ms += eng.time_steps(k)["total_ms"]
        done += k
    th = eng.thermo()
    st = eng.state(forces=False, images=False)
    eng.close()
    c, rho = observables.density_profile(st["x"], s.lo, s.hi, axis=2, width=0.5)
    liq, vap = observables.slab_densities(c, rho, 40.0, 80.0, margin=5.0)
    half = len(th["step"]) // 2
    g, gerr = observables.surface_tension(th["p"], s.box[2], skip=half)
    lz = float(s.box[2])
    acc = fp32_fp64_window(s, st["x"], st["v"], args.slab_acc_steps, 10,
                           extra={"surface_tension": lambda t: 0.5 * lz * (t["p"][:, 5] - 0.5 * (t["p"][:, 0] + t["p"][:, 3]))})
    value = s.n * args.slab_steps / (total_ms / 1000.0)
    window = acc.pop("window")
    summary = {"workload": f"mdpd_slab_N{s.n}", "value": value, "ms_per_step": total_ms / args.slab_steps,
               "liquid_density": liq, "vapour_density": vap, "surface_tension": g,
               "surface_tension_stderr": gerr, "err_vs_fp64": acc}
    return summary, {"steps": args.slab_steps, "density_profile_z0.5": [round(float(x), 4) for x in rho],
                     "mean_temp_second_half": float(np.mean(th["temp"][half:])), "fp64_window": window}


def list_tuning(args):
    """Cell order and list build of every engine the bench creates."""
    return {"cell_order": args.cell_order, "build_variant": args.build_variant}


def plain_step_ms(system, steps):
    """The plain engine on one system alone: device ms per step over `steps` steps (after
    the zero step and a 3-step warm-up; creation is not timed)."""
    from gpumdpd_b200 import Engine
    eng = Engine(system.run_in, system=system.c_system())
    eng.run(0)
    eng.run(3)
    r = eng.time_steps(steps)
    eng.close()
    return r["total_ms"] / steps


def run_alone(system, precision="fp32"):
    """A system alone from its initial state for its run.in's `run N` (thermo rows)."""
    from gpumdpd_b200 import Engine
    run_in = system.run_in if precision == "fp32" else without_computes(system.run_in)
    import re
    steps = int(re.search(r"(?m)^run (\d+)$", run_in).group(1))
    e = Engine(run_in, system=system.c_system(), precision=precision)
    e.run(steps)
    th = e.thermo()
    e.close()
    return th


def run_batched(args):
    """Batched sweep: uneven A/B mixtures (a_AB over 25..45, L log-uniform over 8..24) in one
    packed engine, one launch per stage and the step captured in a CUDA graph, against the
    plain engine running the same replicas one at a time (device time per step summed).
    Accuracy: for 8 replicas (smallest, largest, a_AB extremes, 4 spread over the sweep)
    the packed run's mean T and P against the plain FP32 engine and the FP64 parity engine
    running the same replica alone from the same initial state over the same steps, each
    with its block-averaged standard error (rows after the first fifth)."""
    from gpumdpd_b200 import Batch, inputs, tune
    systems = inputs.replica_sweep(n_rep=args.replicas, nsteps=args.batch_steps, thermo=10)
    for s in systems:
        s.run_in = tune.with_skin(s.run_in, args.batch_skin)
    n_tot = sum(s.n for s in systems)
    b = Batch([s.run_in for s in systems], [s.c_system() for s in systems],
              tuning={"pair_variant": 8, **list_tuning(args)})
    b.run(0)
    K = args.batch_steps
    total_ms, done = 0.0, 0
    while done < K:  # the whole sweep, timed in graphs of at most 500 steps
        k = min(500, K - done)
        total_ms += b.time_steps(k)["total_ms"]
        done += k
    batched = n_tot * K / (total_ms / 1000.0)
    R = len(systems)
    ns = np.array([s.n for s in systems])
    sel = sorted({int(np.argmin(ns)), int(np.argmax(ns)), 0, R - 1} |
                 {int(k) for k in np.linspace(0, R - 1, 6)[1:-1]})
    rows_b = {k: b.thermo(k) for k in sel}
    per_rep = []
    for k, s in enumerate(systems):
        th = b.thermo(k)
        skip = max(1, len(th["pressure"]) // 5)
        g, nsamp = b.rdf(k, 150)
        rmax = min(3.0, 0.5 * float(s.box[0]))
        ipk = int(np.argmax(g))
        per_rep.append({"a_ab": round(25.0 + 20.0 * k / max(R - 1, 1), 3), "n": s.n,
                        "mean_p": round(float(th["pressure"][skip:].mean()), 4),
                        "rdf_peak": round(float(g[ipk]), 4), "rdf_peak_r": round((ipk + 0.5) * rmax / 150, 3),
                        "rdf_samples": nsamp})
    b.close()
    plain_ms = [plain_step_ms(s, args.plain_steps) for s in systems]
    plain = n_tot / (sum(plain_ms) / 1000.0)
    acc = []
    for k in sel:
        s = systems[k]
        tb = rows_b[k]
        tp = run_alone(s, "fp32")
        t64 = run_alone(s, "fp64")
        m = min(len(tb["temp"]), len(tp["temp"]), len(t64["temp"]))
        skip = max(1, m // 5)
        rec = {"replica": k, "n": s.n, "a_ab": round(25.0 + 20.0 * k / max(R - 1, 1), 3), "rows": m - skip}
        for f in ("temp", "pressure"):
            rec[f] = {"batched_vs_fp64": compare(tb[f][skip:m], t64[f][skip:m]),
                      "batched_vs_plain": compare(tb[f][skip:m], tp[f][skip:m])}
        acc.append(rec)

    def worst(f, key):
        r = max(acc, key=lambda a: abs(a[f][key]["z"] or 0.0))
        c = r[f][key]
        return {"rep": r["replica"], "err": c["err"], "stderr": c["stderr"], "z": c["z"],
                "rel": c["err"] / c["fp64"] if c["fp64"] else None}

    summary = {"workload": f"{R}_replica_AB_sweep_N{n_tot}", "value": batched,
               "plain_one_at_a_time": plain, "speedup_vs_plain": batched / plain,
               "err_vs_fp64": {"replicas": len(sel), "T": worst("temp", "batched_vs_fp64"),
                               "P": worst("pressure", "batched_vs_fp64")},
               "vs_plain": {"T": worst("temp", "batched_vs_plain"), "P": worst("pressure", "batched_vs_plain")}}
    return summary, {"steps": K, "thermo_every": 10, "plain_steps_per_replica": args.plain_steps,
                     "per_replica": per_rep, "accuracy": acc}


def served_run(jobs, args, rate_label):
    """One pass of a job stream through the server; returns (summary, results, ids)."""
    from gpumdpd_b200.server import Server, latency_percentiles
    srv = Server(120e9, chunk_steps=args.chunk, tuning={"pair_variant": 8, **list_tuning(args)})
    srv.set_policy(args.max_wait, args.min_jobs)
    pending = list(jobs)
    ids = []
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while pending and pending[0][0] <= now:
            _, s, _ = pending.pop(0)
            ids.append((srv.submit(s), s))
        a, q = srv.step()
        if a == 0 and q == 0:
            if not pending:
                break
            time.sleep(max(0.0, pending[0][0] - (time.perf_counter() - t0)))
    makespan = time.perf_counter() - t0
    res = [srv.result(j) for j, _ in ids]
    assert all(r["status"] == "done" for r in res), [r["status"] for r in res]
    work = sum(s.n * r["steps"] for (_, s), r in zip(ids, res))
    st = srv.stats()
    srv.close()
    pct = latency_percentiles(res)
    return {"rate_jobs_per_s": rate_label, "value": work / makespan, "makespan_s": round(makespan, 3),
            "busy_s": round(st["busy_s"], 3), "p50_latency_s": round(pct.get("p50"), 4),
            "p99_latency_s": round(pct.get("p99"), 4), "particle_steps": work}, res, ids


def run_served(args):
    """Served stream: Poisson arrivals of DPD jobs (1-3 species, a_ij ~ U[25,50], N
    log-uniform 1k-200k, A5B5 chains in 0-50% of beads, steps U[1k,20k], T/P/RDF
    requested) through the continuous-batching server under a 120 GB budget; aggregate
    particle-steps/s over the makespan and p50/p99 job latency, against the plain engine
    running the same jobs one at a time (device time per step x steps, per job).
    Accuracy: the 4 cheapest jobs' served mean T and P (with their block standard errors)
    against the FP64 parity engine running each job alone from its initial state."""
    from gpumdpd_b200 import inputs
    rates = [float(x) for x in args.rates.split(",")]
    sweep = []
    for rate in rates:
        jobs = inputs.job_stream(n_jobs=args.jobs, seed=11, rate=rate, skin=args.batch_skin)
        summary, res, ids = served_run(jobs, args, rate)
        sweep.append(summary)
    # the same jobs one at a time on the plain engine (job contents do not depend on the rate)
    plain_s = 0.0
    for (_, s), r in zip(ids, res):
        ms = plain_step_ms(s, min(args.plain_steps, r["steps"]))
        plain_s += ms / 1000.0 * r["steps"]
    plain = sweep[-1]["particle_steps"] / plain_s
    head = max(sweep, key=lambda x: x["value"])
    cheap = sorted(range(len(ids)), key=lambda k: ids[k][1].n * res[k]["steps"])[:4]
    acc = []
    for k in cheap:
        s = ids[k][1]
        r = res[k]
        t64 = run_alone(s, "fp64")
        rec = {"job": k, "n": s.n, "steps": r["steps"]}
        for f, fm, fs in (("temp", "mean_temp", "stderr_temp"), ("pressure", "mean_pressure", "stderr_pressure")):
            m64, s64 = block_stats(t64[f][1:])
            se = math.sqrt(r[fs] ** 2 + s64 ** 2)
            rec[f] = {"served": round(r[fm], 6), "fp64": round(m64, 6), "err": round(r[fm] - m64, 6),
                      "stderr": round(se, 6), "z": round((r[fm] - m64) / se, 2) if se > 0 else None}
        acc.append(rec)

    def worst(f):
        r = max(acc, key=lambda a: abs(a[f]["z"] or 0.0))
        c = r[f]
        return {"job": r["job"], "err": c["err"], "stderr": c["stderr"], "z": c["z"],
                "rel": c["err"] / c["fp64"] if c["fp64"] else None}

    summary = {"workload": f"{len(ids)}_job_poisson_stream", "value": head["value"],
               "plain_one_at_a_time": plain, "speedup_vs_plain": head["value"] / plain,
               "rates": [[x["rate_jobs_per_s"], x["value"], x["p50_latency_s"], x["p99_latency_s"]] for x in sweep],
               "rates_cols": "jobs/s, particle-steps/s, p50 s, p99 s",
               "err_vs_fp64": {"jobs": len(acc), "T": worst("temp"), "P": worst("pressure")}}
    return summary, {"rate_sweep": sweep, "accuracy": acc, "hbm_budget_bytes": 120e9, "chunk_steps": args.chunk,
                     "admission_window": {"max_wait_s": args.max_wait, "min_jobs": args.min_jobs}}


def time_reference_binary(binary, system, W, K, every):
    """Runs a reference executable on `system` for W+K steps with a thermo line every
    `every` steps (a divisor of W and K) and times steps W..W+K on the host clock between
    its thermo lines at W and W+K (setup and file I/O excluded; the reference flushes each
    line after the device work of its step).  Returns (seconds, None) or (None, the end
    of its output)."""
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        lines = [ln for ln in system.run_in.splitlines() if not ln.startswith(("run ", "thermo ", "read_data "))]
        lines += [f"run {W + K}", f"thermo {every}", "read_data system.data"]
        open(os.path.join(td, "run.in"), "w").write("\n".join(lines) + "\n")
        system.write_data(os.path.join(td, "system.data"))
        p = subprocess.Popen([binary], cwd=td, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, bufsize=1)
        stamps = {}
        log = []
        for line in p.stdout:
            log.append(line)
            if len(log) > 50:
                log.pop(0)
            tok = line.split()
            if tok and tok[0].isdigit() and len(tok) >= 5:
                stamps[int(tok[0])] = time.perf_counter()
        rc = p.wait()
    if rc != 0 or W not in stamps or W + K not in stamps:
        return None, f"rc={rc}: " + "".join(log[-3:]).strip().replace("\n", " | ")
    return stamps[W + K] - stamps[W], None


def run_fp64(args):
    """The FP64 parity mode against the reference's -DDOUBLE build on the same inputs: C1
    (plain DPD, 3000 particles, 2000 timed steps) and the 3M A5B5 melt (20 timed steps after
    10): the FP64 engine's device time per step (CUDA events) and the reference's host clock
    between its thermo lines (as the reference arm)."""
    from gpumdpd_b200 import Engine, inputs
    binary = os.path.join(ROOT, "oracle", "_ref", "gpudpd_double")
    out = {"dtype": "f64"}
    cases = [("c1", inputs.plain_dpd(L=10.0, seed=2024, nsteps=10 ** 6, thermo=1000, skin=0.0), 50, 2000, 1000)]
    if not args.no_fp64_melt:
        cases.append(("melt_3M", inputs.diblock_melt(L=100.0, seed=7, nsteps=10 ** 6, thermo=10, skin=0.0),
                      10, 20, 10))
    for name, s, W, K, every in cases:
        e = Engine(s.run_in, system=s.c_system(), precision="fp64")
        e.run(0)
        e.run(W)
        ms = e.time_steps(K)["total_ms"] / K
        e.close()
        rec = {"particles": s.n, "ms_per_step": ms, "value": s.n / (ms / 1000.0)}
        if os.path.exists(binary):
            dt, why = time_reference_binary(binary, s, max(W, every), K, every)
            if dt is not None:
                rec["reference_double_ms_per_step"] = dt * 1000 / K
                rec["speedup_vs_reference_double"] = rec["reference_double_ms_per_step"] / ms
            else:
                rec["reference_double"] = f"failed {why}"[:120]
        out[name] = rec
    return out, {}


def run_reference(args, world, rank):
    """The reference's own CUDA build (oracle/_ref/gpudpd_single, built from its sources by
    oracle/build_ref.sh) on the same system and thermo cadence: it reads run.in + a data
    file in its own format; after W warm-up steps, K steps are timed on the host clock
    between its thermo lines at steps W and W+K (setup and file I/O excluded)."""
    if rank != 0:
        return
    every = thermo_every(args)
    system = make_system(args, thermo=every)
    K, W = args.steps, args.warmup
    binary = os.path.join(ROOT, "oracle", "_ref", "gpudpd_single")
    if not os.path.exists(binary):
        # no reference build: time the FP64 port on the host cores instead
        cb = cpu_baseline(system, os.cpu_count() or 1)
        print(json.dumps({"metric": METRIC, "value": cb["value"], "unit": "particle-steps/s",
                          "n_gpus": world, "steps": 2, "warmup": 0, "higher_is_better": True, "impl": "reference",
                          "config": {"workload": workload_name(args)}, "cpu_baseline": cb,
                          "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    dt, why = time_reference_binary(binary, system, W, K, every)
    if dt is None:
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed {why}"}))
        return
    value = system.n * K / dt
    out = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
           "steps": K, "warmup": W, "ms_per_step": dt * 1000 / K, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator and seed)",
           "config": {"workload": workload_name(args), "n_particles": system.n, "skin": args.skin,
                      "thermo_every": every, "parallelism": "single GPU, rank 0 only"},
           "impl": "reference",
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
                            "sample": f"reference CUDA build (-DSINGLE, sm_100a) on one B200 driven by one host "
                                      f"thread; steps {W}..{W + K} timed between its thermo lines"},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="melt", choices=["melt", "melt_mid", "melt_small", "plain", "slab"])
    ap.add_argument("--skin", type=float, default=0.0,
                    help="neighbour skin (0.0: the tuner's choice for the 3M melt, which rebuilds every step)")
    ap.add_argument("--tune", action="store_true", help="run the autotuner first (skin and pair schedule)")
    ap.add_argument("--pair-variant", type=int, default=None,
                    help="pair-kernel schedule (default: the engine's choice)")
    ap.add_argument("--build-variant", type=int, default=5,
                    help="list-build kernel of every engine (0: cell ranges in registers; 1, 2: in shared memory; "
                         "4: cell tiles; 5: column ranges, contiguous under --cell-order 0 or 2)")
    ap.add_argument("--cell-order", type=int, default=0,
                    help="cell order of the slots of every engine (0: linear, 1: Morton, 2: x-y columns in "
                         "Morton order)")
    ap.add_argument("--pair-block", type=int, default=0,
                    help="pair schedule 11: 3 = the tile kernel at 3 CTAs per SM (default 4)")
    ap.add_argument("--tile", type=int, default=0,
                    help="pair schedule 11: home cells per tile edge (0: the engine's choice)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the slab, batched, served and fp64 objects")
    ap.add_argument("--detail", default="bench_detail.json",
                    help="file for the per-replica records, density profile and rate sweep ('' = none)")
    ap.add_argument("--acc-steps", type=int, default=300, help="FP32-vs-FP64 window of the headline system")
    ap.add_argument("--acc-equil", type=int, default=2000,
                    help="FP32 steps before the headline system's FP32-vs-FP64 window")
    ap.add_argument("--no-fp64-melt", action="store_true", help="skip the 3M melt in the fp64 object")
    ap.add_argument("--slab-steps", type=int, default=20000)
    ap.add_argument("--slab-acc-steps", type=int, default=1000)
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=5000)
    ap.add_argument("--batch-skin", type=float, default=0.0)
    ap.add_argument("--plain-steps", type=int, default=200)
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--rates", default="4,64", help="served arrival rates (jobs/s) to sweep")
    ap.add_argument("--max-wait", type=float, default=0.0, help="server admission window (s)")
    ap.add_argument("--min-jobs", type=int, default=1, help="server admission batch size")
    ap.add_argument("--chunk", type=int, default=200, help="server scheduling chunk (steps)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
