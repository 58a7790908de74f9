"""Generate golden fixtures from the reference's own CUDA build (run on a GPU host).

Runs the executables built by oracle/build_ref.sh (oracle/_ref/gpudpd_single,
gpudpd_double and the Saru known-answer harness ref_saru) on small seeded systems
written in the reference's own input formats, and stores what the reference
produced -- Saru outputs, dumped positions/velocities/forces (all.trj) and
thermo.txt rows -- as compressed .npz files.  The committed fixtures under
tests/golden/ were produced by:

    python tests/golden/gen_ref_fixtures.py --out tests/golden

Nothing here is used by the engine; tests/test_oracle.py pins the oracle against
these files, and the GPU tests compare the engine with the pinned oracle.
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from gpumdpd_b200 import inputs  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def saru_kat(out_dir, n=20000, seed=3):
    rng = np.random.default_rng(seed)
    t1 = rng.integers(1, 4_000_000, n).astype(np.uint32)
    t2 = t1 + rng.integers(1, 100000, n).astype(np.uint32)
    # include edge cases: small tags, huge tags, large seeds and steps
    t1[:8] = [1, 1, 2, 3, 1000, 2**27 - 2, 5, 7]
    t2[:8] = [2, 3, 3, 4, 1001, 2**27 - 1, 6, 8]
    seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    seeds[:4] = [0, 1, 123456, 2**32 - 1]
    steps = rng.integers(0, 2**31 - 1, n).astype(np.int32)
    steps[:6] = [0, 1, 2, 1000, 20000, 2**31 - 1]
    rec = np.stack([t1, t2, seeds, steps.view(np.uint32)], axis=1).astype(np.uint32)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            np.array([n], dtype=np.int32).tofile(f)
            rec.tofile(f)
        subprocess.run([os.path.join(REF, "ref_saru"), fin, fout], check=True)
        out = np.fromfile(fout, dtype=np.float32)
    np.savez_compressed(os.path.join(out_dir, "ref_saru_kat.npz"), t1=t1, t2=t2, seed=seeds,
                        step=steps, theta=out)


def parse_trj(path):
    frames = {}
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    while k < len(lines):
        if lines[k].startswith("ITEM: TIMESTEP"):
            step = int(lines[k + 1])
            n = int(lines[k + 3])
            cols = lines[k + 8].split()[2:]
            data = np.loadtxt(lines[k + 9: k + 9 + n])
            frames[step] = {c: data[:, q] for q, c in enumerate(cols)}
            k += 9 + n
        else:
            k += 1
    return frames


def parse_thermo(path):
    with open(path) as f:
        head = f.readline().split()
    data = np.loadtxt(path, skiprows=1, ndmin=2)
    return {h: data[:, q] for q, h in enumerate(head)}


KEEP_FRAMES = {"probe_fixes": (0, 1, 3, 4, 10)}  # steps after an rvcm (3) and a recenter (4)


def run_reference(name, system, out_dir, nsteps=10, binary="gpudpd_single"):
    run = system.run_in
    lines = [ln for ln in run.splitlines() if not ln.startswith(("run ", "thermo ", "read_data "))]
    lines += [f"run {nsteps}", "thermo 1", "read_data system.data",
              "dump 0 1 wrapped force_yes vel_yes"]
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(td, "run.in"), "w") as f:
            f.write("\n".join(lines) + "\n")
        system.write_data(os.path.join(td, "system.data"))
        r = subprocess.run([os.path.join(REF, binary)], cwd=td, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{name}: reference failed\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        frames = parse_trj(os.path.join(td, "all.trj"))
        thermo = parse_thermo(os.path.join(td, "thermo.txt"))
        spring = os.path.join(td, "spring.txt")  # fix spring's record file, when it has one
        spring = np.loadtxt(spring, skiprows=1, ndmin=2) if os.path.exists(spring) else None
        # files of computes (step + values per row)
        extra = {f[:-4]: np.loadtxt(os.path.join(td, f), skiprows=1, ndmin=2) for f in os.listdir(td)
                 if f.endswith(".txt") and f not in ("thermo.txt", "spring.txt")}
    save = {"run_in": np.array("\n".join(lines)), "masses": system.masses, "lo": system.lo,
            "hi": system.hi}
    if system.bonds is not None:
        save["bonds"] = system.bonds
    if system.angles is not None:
        save["angles"] = system.angles
    for step in sorted(frames):
        if step not in KEEP_FRAMES.get(name, (0, 1, nsteps)):
            continue
        fr = frames[step]
        order = np.argsort(fr["id"])
        for c in ("x", "y", "z", "fx", "fy", "fz", "vx", "vy", "vz"):
            save[f"s{step}_{c}"] = fr[c][order]
        save[f"s{step}_id"] = fr["id"][order].astype(np.int32)
        save[f"s{step}_type"] = fr["type"][order].astype(np.int32)
    for h, col in thermo.items():
        save[f"thermo_{h}"] = col
    if spring is not None:
        save["spring"] = spring
    for k, rows in extra.items():
        save[f"file_{k}"] = rows
    np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), **save)


def systems():
    out = {}
    out["dpd_c1"] = inputs.plain_dpd(L=10.0, seed=2024)
    s = inputs.plain_dpd(L=8.0, seed=77, a=0.0)  # random force only (A = 0, v = 0)
    s.v[:] = 0.0
    out["dpd_random_only"] = s
    out["mdpd_slab"] = inputs.mdpd_slab(Lx=8.0, Ly=8.0, Lz=24.0, z0=8.0, z1=16.0, seed=11, nsteps=10)
    out["diblock"] = inputs.diblock_melt(L=10.0, seed=5, nsteps=10)
    mix = inputs.binary_mixture(9.0, 40.0, seed=4)
    # per-pair cutoffs through the reference's 6-argument pair_coeff form
    mix.run_in = mix.run_in.replace("pair_coeff 1 2 40.0 4.5", "pair_coeff 1 2 40.0 4.5 0.8 0")
    mix.run_in = mix.run_in.replace("pair_coeff 2 2 25.0 4.5", "pair_coeff 2 2 30.0 3.0 0.9 0")
    out["mix_rc"] = mix
    # harmonic angles on every consecutive triple of A5B5 chains (atom_style angle)
    out["angle_chains"] = inputs.angle_chains(L=8.0, seed=19, nsteps=10, angle_k=3.0, theta0=120.0)
    # group fixes: spring on a probe cluster (record file every 2 steps), rvcm on all every
    # 3 steps (x and z), recenter of the probe every 4 steps
    out["probe_fixes"] = inputs.probe_fixes(L=9.0, seed=23, nsteps=10)
    # particle walls: a frozen bottom wall, a top wall moved by fix move, the liquid kept
    # between them by fix two_wall or fix wall_reflect; compute wall_contact on the bottom
    out["wall_channel"] = inputs.wall_channel(seed=71, nsteps=10)
    out["wall_reflect"] = inputs.wall_channel(seed=73, nsteps=10, walls="reflect")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--only", default=None, help="generate just this system's fixture")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.only:
        run_reference(a.only, systems()[a.only], a.out)
        print("fixture written to", a.out)
        return
    saru_kat(a.out)
    for name, s in systems().items():
        run_reference(name, s, a.out)
    run_reference("dpd_c1_double", systems()["dpd_c1"], a.out, binary="gpudpd_double")
    print("fixtures written to", a.out)


if __name__ == "__main__":
    main()
