"""Slab observables computed from the engine's outputs (new: the reference has no
density-profile or surface-tension compute; it writes positions and the pressure tensor
from which both follow, src/compute/thermo.cu:506-517).

- `density_profile`: number density along one axis in bins of a given width, from a
  state (positions wrapped into the box).
- `surface_tension`: gamma_s = (L_z / 2) <P_zz - (P_xx + P_yy) / 2> for a slab with two
  interfaces normal to z, from thermo rows (`Engine.thermo()["p"]`, columns
  pxx pxy pxz pyy pyz pzz).
"""
import numpy as np


def density_profile(x, lo, hi, axis=2, width=0.5):
    """Bin centres and number density along `axis` (particles per unit volume)."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    L = hi - lo
    nb = max(int(np.floor(L[axis] / width)), 1)
    w = L[axis] / nb
    z = np.mod(np.asarray(x)[:, axis] - lo[axis], L[axis])
    counts = np.bincount(np.minimum((z / w).astype(np.int64), nb - 1), minlength=nb)
    area = np.prod(np.delete(L, axis))
    centres = lo[axis] + (np.arange(nb) + 0.5) * w
    return centres, counts / (area * w)


def surface_tension(p_rows, Lz, skip=0):
    """(L_z / 2) times the mean of P_zz - (P_xx + P_yy) / 2 over the rows after `skip`;
    returns (gamma_s, its standard error from 8 blocks)."""
    p = np.asarray(p_rows, dtype=np.float64)[skip:]
    s = 0.5 * Lz * (p[:, 5] - 0.5 * (p[:, 0] + p[:, 3]))
    nb = min(8, len(s))
    if nb < 2:
        return float(s.mean()), float("nan")
    blocks = np.array([b.mean() for b in np.array_split(s, nb)])
    return float(s.mean()), float(blocks.std(ddof=1) / np.sqrt(nb))


def slab_densities(centres, rho, z0, z1, margin=5.0):
    """Mean density of the liquid (inside [z0+margin, z1-margin]) and of the vapour (at
    least `margin` outside the slab)."""
    c = np.asarray(centres)
    liq = (c > z0 + margin) & (c < z1 - margin)
    vap = (c < z0 - margin) | (c > z1 + margin)
    return float(np.mean(rho[liq])), float(np.mean(rho[vap])) if vap.any() else float("nan")
