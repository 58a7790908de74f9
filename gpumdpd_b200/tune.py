"""Autotuner: picks the neighbour-list skin and the pair-kernel schedule of a system (or a
packed batch of systems) by timing a few steps of each candidate on the device.

The skin sets the cell size (global_cut + skin), the list length and how often the
reference's rebuild rule (any particle moved more than skin/2) fires; the rebuild
interval follows from it.  Large systems rebuild nearly every step at any practical skin
(their fastest particle crosses skin/2 within a step or two), so a small skin wins;
small systems rebuild rarely and a larger skin amortises the build.  Candidates are
timed with CUDA events over whole steps (list builds included) after a short warm-up.
"""
import re

from .engine import Batch, Engine

SKINS = (0.0, 0.1, 0.2, 0.3)
VARIANTS = (1, 4, 6, 8, 9)


def with_skin(run_in, skin):
    """The run.in text with the skin of its `neighbor` command replaced."""
    def sub(m):
        t = m.group(0).split()
        t[2] = repr(float(skin))
        return " ".join(t)
    return re.sub(r"(?m)^neighbor\s+\S+\s+\S+\s+\S+\s+\S+", sub, run_in)


def _time(eng, steps, warmup):
    eng.run(0)
    eng.run(warmup)
    return eng.time_steps(steps)["total_ms"] / steps


def tune_system(system, skins=SKINS, variants=VARIANTS, steps=20, warmup=5):
    """Best (skin, pair_variant) for one system; returns (best, table of ms/step)."""
    table = []
    for skin in skins:
        try:
            eng = Engine(with_skin(system.run_in, skin), system=system.c_system())
        except Exception as e:  # box too small for this skin's cells, for example
            table.append({"skin": skin, "error": str(e)})
            continue
        for v in variants:
            eng.set_tuning(pair_variant=v, cell_order=1)
            table.append({"skin": skin, "pair_variant": v, "ms_per_step": _time(eng, steps, warmup)})
        eng.close()
    ok = [t for t in table if "ms_per_step" in t]
    best = min(ok, key=lambda t: t["ms_per_step"])
    return best, table


def tune_batch(systems, skins=SKINS, variants=VARIANTS, steps=10, warmup=3):
    """Best (skin, pair_variant) for a packed batch of systems (one skin for all)."""
    table = []
    for skin in skins:
        try:
            b = Batch([with_skin(s.run_in, skin) for s in systems], [s.c_system() for s in systems],
                      tuning={"pair_variant": variants[0], "cell_order": 1})
        except Exception as e:
            table.append({"skin": skin, "error": str(e)})
            continue
        for v in variants:
            b.set_tuning(pair_variant=v, cell_order=1)
            table.append({"skin": skin, "pair_variant": v, "ms_per_step": _time(b, steps, warmup)})
        b.close()
    ok = [t for t in table if "ms_per_step" in t]
    best = min(ok, key=lambda t: t["ms_per_step"])
    return best, table
