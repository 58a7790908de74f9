"""Autotuner: picks the launch knobs of a system (or a packed batch of systems) by timing
whole steps of each candidate on the device.

The reference hard-codes the knobs this searches (src/force/neigh_list.cu:5-28 bin size
and list capacity, src/main/read_in.cu:93-118 rebuild check interval,
src/force/pair_dpd.cu:613-616 eight threads per particle):

- the skin, which sets the cell size (global_cut + skin) and the list length; the
  reference's rebuild rule (any particle moved more than skin/2) decides how often the
  list is rebuilt.  Large systems rebuild nearly every step at any practical skin (their
  fastest particle crosses skin/2 within a step or two), so a small skin wins; small
  systems rebuild rarely and a larger skin amortises the build;
- the rebuild check interval nl_f (the `neighbor` command's check frequency) for skins
  above 0.  Only intervals that cannot miss a rebuild are tried: nl_f times the largest
  per-step displacement seen over a few steps, times 1.5, must stay below skin/2;
- the pair schedule and its work split: a thread per particle (0), the warp pair queue
  (1), the flattened warp schedule (4, 8, 9), and the cell-tile kernel without a list
  (11) with 1, 2 or 4 home cells per tile edge (or the engine's choice);
- the launch mode (0: the fused small-grid launches where they apply; 1: never);
- the cell order of the slots and the list build that goes with it: linear cells with the
  build over column ranges (five contiguous slot ranges per particle), or Morton-ordered
  cells with the build cell by cell.

Candidates are timed with CUDA events over whole steps (list builds included) after a
short warm-up; the fastest is returned with the table of every candidate.
"""
import re

import numpy as np

from .engine import Batch, Engine

SKINS = (0.0, 0.1, 0.2, 0.3)
SCHEDULES = ({"pair_variant": 8}, {"pair_variant": 4}, {"pair_variant": 1}, {"pair_variant": 9},
             {"pair_variant": 11, "tile": 0}, {"pair_variant": 11, "tile": 2}, {"pair_variant": 11, "tile": 4})
LAUNCH_MODES = (0, 1)
INTERVALS = (1, 2, 5)
LISTS = ({"cell_order": 0, "build_variant": 5}, {"cell_order": 1, "build_variant": 0})
VARIANTS = tuple(sorted({s["pair_variant"] for s in SCHEDULES}))


def with_skin(run_in, skin, nl_f=None):
    """The run.in text with the skin (and, when given, the check interval) of its
    `neighbor` command replaced."""
    def sub(m):
        t = m.group(0).split()
        t[2] = repr(float(skin))
        if nl_f is not None:
            t[4] = str(int(nl_f))
        return " ".join(t)
    return re.sub(r"(?m)^neighbor\s+\S+\s+\S+\s+\S+\s+\S+", sub, run_in)


def _time(eng, steps, warmup):
    eng.run(0)
    eng.run(warmup)
    return eng.time_steps(steps)["total_ms"] / steps


def _max_step_displacement(eng, box, steps=3):
    """Largest displacement of any particle in one step, over a few steps."""
    eng.run(0)
    x0 = eng.state(forces=False, images=False)["x"]
    dmax = 0.0
    for _ in range(steps):
        eng.run(1)
        x1 = eng.state(forces=False, images=False)["x"]
        d = x1 - x0
        d -= box * np.round(d / box)
        dmax = max(dmax, float(np.sqrt((d * d).sum(axis=1)).max()))
        x0 = x1
    return dmax


def safe_intervals(skin, dmax, intervals=INTERVALS, margin=1.5):
    """Check intervals that keep every particle within skin/2 of its binned position
    between two checks, with a margin on the largest per-step displacement seen."""
    if skin <= 0.0:
        return (1,)
    return tuple(k for k in intervals if k == 1 or k * dmax * margin < 0.5 * skin)


def _candidates(schedules, launch_modes, lists):
    for sc in schedules:
        for lm in launch_modes:
            for li in lists:
                yield dict(sc, launch_mode=lm, **li)


def tune_system(system, skins=SKINS, schedules=SCHEDULES, launch_modes=LAUNCH_MODES, intervals=INTERVALS,
                steps=20, warmup=5, variants=None, lists=LISTS):
    """Best knobs for one system; returns (best, table of ms/step).  `variants` (pair
    schedules without tile options) narrows `schedules`."""
    if variants is not None:
        schedules = tuple({"pair_variant": v} for v in variants)
    table = []
    box = np.asarray(system.box, dtype=np.float64)
    for skin in skins:
        ivs = (1,)
        if skin > 0.0 and len(intervals) > 1:
            try:
                probe = Engine(with_skin(system.run_in, skin, 1), system=system.c_system())
                ivs = safe_intervals(skin, _max_step_displacement(probe, box), intervals)
                probe.close()
            except Exception as e:
                table.append({"skin": skin, "error": str(e)})
                continue
        for nl_f in ivs:
            try:
                eng = Engine(with_skin(system.run_in, skin, nl_f), system=system.c_system())
            except Exception as e:  # box too small for this skin's cells, for example
                table.append({"skin": skin, "nl_f": nl_f, "error": str(e)})
                continue
            for c in _candidates(schedules, launch_modes, lists):
                eng.set_tuning(**c)
                table.append(dict(c, skin=skin, nl_f=nl_f, ms_per_step=_time(eng, steps, warmup)))
            eng.close()
    ok = [t for t in table if "ms_per_step" in t]
    best = min(ok, key=lambda t: t["ms_per_step"])
    return best, table


def tune_batch(systems, skins=SKINS, schedules=SCHEDULES, launch_modes=LAUNCH_MODES, steps=10, warmup=3,
               variants=None, lists=LISTS):
    """Best knobs for a packed batch of systems (one skin for all; check interval 1)."""
    if variants is not None:
        schedules = tuple({"pair_variant": v} for v in variants)
    table = []
    for skin in skins:
        try:
            b = Batch([with_skin(s.run_in, skin) for s in systems], [s.c_system() for s in systems])
        except Exception as e:
            table.append({"skin": skin, "error": str(e)})
            continue
        for c in _candidates(schedules, launch_modes, lists):
            b.set_tuning(**c)
            table.append(dict(c, skin=skin, nl_f=1, ms_per_step=_time(b, steps, warmup)))
        b.close()
    ok = [t for t in table if "ms_per_step" in t]
    best = min(ok, key=lambda t: t["ms_per_step"])
    return best, table
