"""bench.py -- timestep throughput of the B200 DPD engine (one JSON line on rank 0).

Workload (default): the binary A5B5 diblock melt -- periodic 100^3 box at density 3,
N = 3.0M beads in 300k linear 10-bead chains, harmonic bonds k=4 r0=0, a_AA=a_BB=25,
a_AB=40, gamma=4.5, kT=1, dt=0.04, skin 0.3 -- seeded synthetic input (chains grown as
random walks with step 0.9; no dataset).  A step is one velocity-Verlet timestep of the
whole system (list build when due, pair+bond forces with the Saru random force, fused
integration).  Metric: particle-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent replica per GPU (replicas only: the single system is not
decomposed), launched by torch.distributed.run; value sums all ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "a5b5_diblock_melt_L100_N3M_skin0.3"


def make_system(args):
    from gpumdpd_b200 import inputs
    if args.workload == "melt":
        return inputs.diblock_melt(L=100.0, seed=7, nsteps=10 ** 6, thermo=1000, skin=args.skin)
    if args.workload == "melt_mid":
        return inputs.diblock_melt(L=60.0, seed=7, nsteps=10 ** 6, thermo=1000, skin=args.skin)
    if args.workload == "melt_small":
        return inputs.diblock_melt(L=30.0, seed=7, nsteps=10 ** 6, thermo=1000, skin=args.skin)
    if args.workload == "plain":
        return inputs.plain_dpd(L=10.0, seed=2024, nsteps=10 ** 6, thermo=1000, skin=args.skin)
    if args.workload == "slab":
        return inputs.mdpd_slab(nsteps=10 ** 6, thermo=1000, skin=args.skin)
    raise SystemExit(f"unknown workload {args.workload}")


class ClockSampler:
    """nvidia-smi clocks sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", self.gpu], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        os.environ.setdefault("CUDA_VISIBLE_DEVICES_ORIG", "")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def algorithmic_bytes_per_particle(mean_half_list, maxb):
    """Pair kernel, per particle-step: x,v of i (32 B) + force write (12 B) + list length
    (4 B) + list entries (4 B each); neighbour-j gathers are assumed cache-resident and not
    counted.  The fused bonds add their partner table (8 B per slot)."""
    return 48.0 + 4.0 * mean_half_list + 8.0 * maxb


def cpu_baseline(system, nthreads, nsteps=2):
    """FP64 oracle port of the reference algorithm on the host cores (bounded sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    ff = oracle.ff_from_run_in(system.run_in, system.masses)
    tags = np.arange(1, system.n + 1)
    t0 = time.perf_counter()
    oracle.bench_steps(ff, tags, system.types, system.x, system.v, system.lo, system.box, 1, nsteps,
                       0.3, nthreads)
    dt = time.perf_counter() - t0
    return {"value": system.n * nsteps / dt, "unit": "particle-steps/s", "cores": nthreads,
            "kind": "port",
            "sample": f"full {system.n}-particle system, step-0 force + {nsteps} steps incl. one list "
                      f"build, FP64, pair forces (bonds omitted), {nthreads} threads; {dt:.1f} s"}


def run_ours(args, world, rank, local):
    import torch
    from gpumdpd_b200 import Engine
    system = make_system(args)
    eng = Engine(system.run_in, system=system.c_system())
    if args.pair_variant is not None:
        eng.set_tuning(pair_variant=args.pair_variant, cell_order=1)
    eng.run(0)
    eng.run(args.warmup)
    ls = eng.list_stats()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        res = eng.time_steps(args.steps)
    torch.cuda.synchronize()
    barrier(world)
    total_ms = allreduce_max(res["total_ms"], world)
    pair_ms = res["pair_ms"]
    n = system.n
    value = world * n * args.steps / (total_ms / 1000.0)
    # end to end through the C ABI with host buffers: the state (x, v in FP64) goes host
    # -> device, K steps run (a zero-step force evaluation and list build first), the
    # final x, v come back device -> host with the thermo rows
    chunk = args.steps
    st = eng.state(forces=False, images=False)
    x = np.ascontiguousarray(st["x"])
    v = np.ascontiguousarray(st["v"])
    barrier(world)
    t0 = time.perf_counter()
    eng.set_state(x, v)
    eng.run(chunk)
    st2 = eng.state(forces=False, images=False)
    th = eng.thermo(max_rows=4)
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    e2e = world * n * chunk / e2e_s
    h2d = n * 6 * 8 / chunk
    d2h = (n * 6 * 8 + 4 * 8 * 16) / chunk
    maxb = 2 if system.bonds is not None else 0
    bpp = algorithmic_bytes_per_particle(ls["mean_half_list"], maxb)
    per_launch_ms = pair_ms / max(res["pair_launches"], 1)
    achieved = n * bpp / (per_launch_ms / 1000.0) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    traffic = None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        t = prof.get(args.workload)
        if t:
            traffic = t["dram_bytes_per_launch"]
    except Exception:
        pass
    out = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64-reductions",
        "data": "synthetic (seeded generator, gpumdpd_b200/inputs.py)",
        "config": {"workload": WORKLOAD if args.workload == "melt" else args.workload, "n_particles": n,
                   "n_bonds": 0 if system.bonds is None else len(system.bonds), "box": system.box.tolist(),
                   "dt": 0.04, "skin": args.skin, "mean_half_list": ls["mean_half_list"],
                   "list_builds": ls["builds"], "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (state+list > 1 GB)"},
        "e2e": {"value": e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "chunk_steps": chunk, "path": "dpd_set_state + dpd_run + dpd_get_state (C ABI, host buffers)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "k_pair (DPD + bonds)",
                     "bytes_per_particle": bpp, "pair_ms_per_launch": per_launch_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback"},
        "clocks": clk.summary(),
        "gpu_launches": int(res["pair_launches"] * 12 + 2),
        "impl": "ours",
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(system, os.cpu_count() or 1)
    if rank == 0:
        print(json.dumps(out))
    del th, st2
    eng.close()


def run_reference(args, world, rank):
    """The reference's own CUDA build (oracle/_ref/gpudpd_single, built from its sources by
    oracle/build_ref.sh) on the same system: it reads run.in + a data file in its own
    format; K steps are timed on the host clock between its thermo lines at steps K and 2K
    (thermo every K steps, so setup and file I/O are excluded)."""
    if rank != 0:
        return
    from gpumdpd_b200 import inputs  # noqa: F401
    binary = os.path.join(ROOT, "oracle", "_ref", "gpudpd_single")
    system = make_system(args)
    K = args.steps
    if not os.path.exists(binary):
        # no reference build: time the FP64 port on the host cores instead
        cb = cpu_baseline(system, os.cpu_count() or 1)
        print(json.dumps({"metric": "particle-steps/s", "value": cb["value"], "unit": "particle-steps/s",
                          "n_gpus": world, "steps": 2, "warmup": 0, "higher_is_better": True, "impl": "reference",
                          "config": {"workload": WORKLOAD}, "cpu_baseline": cb,
                          "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        lines = [ln for ln in system.run_in.splitlines() if not ln.startswith(("run ", "thermo ", "read_data "))]
        lines += [f"run {2 * K}", f"thermo {K}", "read_data system.data"]
        open(os.path.join(td, "run.in"), "w").write("\n".join(lines) + "\n")
        system.write_data(os.path.join(td, "system.data"))
        p = subprocess.Popen([binary], cwd=td, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, bufsize=1)
        stamps = {}
        log = []
        for line in p.stdout:
            log.append(line)
            tok = line.split()
            if tok and tok[0].isdigit() and len(tok) >= 5:
                stamps[int(tok[0])] = time.perf_counter()
        rc = p.wait()
    if rc != 0 or K not in stamps or 2 * K not in stamps:
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed rc={rc}: "
                          + "".join(log[-3:]).strip().replace("\n", " | ")}))
        return
    dt = stamps[2 * K] - stamps[K]
    value = system.n * K / dt
    out = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
           "steps": K, "warmup": K, "ms_per_step": dt * 1000 / K, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator and seed)",
           "config": {"workload": WORKLOAD, "n_particles": system.n, "skin": args.skin,
                      "parallelism": "single GPU, rank 0 only"},
           "impl": "reference",
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
                            "sample": f"reference CUDA build (-DSINGLE, sm_100a) on one B200 driven by one host "
                                      f"thread; steps {K}..{2 * K} timed between its thermo lines"},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="melt", choices=["melt", "melt_mid", "melt_small", "plain", "slab"])
    ap.add_argument("--skin", type=float, default=0.3)
    ap.add_argument("--pair-variant", type=int, default=None,
                    help="pair-kernel schedule (default: the engine's choice)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
