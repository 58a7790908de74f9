"""Seeded synthetic inputs for the benchmark systems, and writers of the reference's
input formats (run.in command text and the data file layout of
src/system/read_data.cu:473-637), so the same system drives this engine, the
oracle and the reference executable.

Systems (no public dataset is involved; everything is generated from a seed):
  plain_dpd      single-species Groot-Warren DPD, L=10, rho=3 (N=3000)
  diblock_melt   A5B5 diblock chains, harmonic bonds k=4 r0=0, L=100 (N=3.0M)
  mdpd_slab      many-body DPD liquid slab rho=6 in z in [40,80], box 40x40x120
  replica_sweep  256 A/B mixtures, a_AB in [25,45], L log-uniform in [8,24]
  job_stream     served jobs: 1-3 species, a_ij ~ U[25,50], N log-uniform 1k-200k
"""
import math

import numpy as np

from . import capi


class System:
    """Arrays of one system (rows in tag order) plus its run.in text."""

    def __init__(self, lo, hi, masses, types, x, v, bonds=None, n_bondtypes=0, mol=None,
                 run_in="", atom_style="atomic", angles=None, n_angletypes=0):
        self.lo = np.asarray(lo, dtype=np.float64)
        self.hi = np.asarray(hi, dtype=np.float64)
        self.masses = np.asarray(masses, dtype=np.float64)
        self.types = np.asarray(types, dtype=np.int32)
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.v = np.ascontiguousarray(v, dtype=np.float64)
        self.bonds = None if bonds is None else np.ascontiguousarray(bonds, dtype=np.int32)
        self.n_bondtypes = n_bondtypes
        self.mol = None if mol is None else np.asarray(mol, dtype=np.int32)
        self.run_in = run_in
        self.atom_style = atom_style
        self.angles = None if angles is None else np.ascontiguousarray(angles, dtype=np.int32)  # type, i, j, k
        self.n_angletypes = n_angletypes

    @property
    def n(self):
        return len(self.types)

    @property
    def box(self):
        return self.hi - self.lo

    def c_system(self):
        return capi.make_system(self.lo, self.hi, self.masses, self.types, self.x, self.v,
                                self.bonds, self.n_bondtypes, self.mol, angles=self.angles,
                                n_angletypes=self.n_angletypes)

    def write_data(self, path):
        """Data file in the layout written by the reference's write_data."""
        with open(path, "w") as f:
            f.write("# Lammps format data file\n")
            f.write("                         \n")
            f.write(f"{self.n} atoms\n")
            if self.atom_style != "atomic":
                f.write(f"{0 if self.bonds is None else len(self.bonds)} bonds\n")
            if self.atom_style == "angle":
                f.write(f"{0 if self.angles is None else len(self.angles)} angles\n")
            f.write(f"{len(self.masses)} atom types\n")
            if self.atom_style != "atomic":
                f.write(f"{max(self.n_bondtypes, 1)} bond types\n")
            if self.atom_style == "angle":
                f.write(f"{max(self.n_angletypes, 1)} angle types\n")
            f.write("                           \n")
            for k, nm in enumerate(("x", "y", "z")):
                f.write(f"{self.lo[k]:.9f} {self.hi[k]:.9f} {nm}lo {nm}hi\n")
            f.write("                           \n")
            f.write("Masses\n")
            f.write("                           \n")
            for t, m in enumerate(self.masses):
                f.write(f"{t + 1} {m:.9f}\n")
            f.write("                           \n")
            f.write(f"Atoms  # {self.atom_style}\n")
            f.write("                           \n")
            ids = np.arange(1, self.n + 1)
            if self.atom_style == "atomic":
                cols = np.column_stack([ids, self.types, self.x])
                np.savetxt(f, cols, fmt=["%d", "%d", "%.9f", "%.9f", "%.9f"])
            else:
                mol = self.mol if self.mol is not None else np.zeros(self.n, dtype=np.int32)
                cols = np.column_stack([ids, mol, self.types, self.x])
                np.savetxt(f, cols, fmt=["%d", "%d", "%d", "%.9f", "%.9f", "%.9f"])
            f.write("                           \n")
            f.write("Velocities\n")
            f.write("                           \n")
            np.savetxt(f, np.column_stack([ids, self.v]), fmt=["%d", "%.9f", "%.9f", "%.9f"])
            f.write("                           \n")
            if self.atom_style != "atomic":
                f.write("Bonds\n")
                f.write("                           \n")
                nb = len(self.bonds)
                np.savetxt(f, np.column_stack([np.arange(1, nb + 1), self.bonds]), fmt="%d")
            if self.atom_style == "angle":
                f.write("                           \n")
                f.write("Angles\n")
                f.write("                           \n")
                na = len(self.angles)
                np.savetxt(f, np.column_stack([np.arange(1, na + 1), self.angles]), fmt="%d")


def _velocities(rng, n, kT, masses_of_atoms):
    v = rng.normal(0.0, 1.0, size=(n, 3)) * np.sqrt(kT / masses_of_atoms)[:, None]
    p = (v * masses_of_atoms[:, None]).sum(axis=0) / masses_of_atoms.sum()
    return v - p  # net momentum removed


def run_in_text(*, atom_style="atomic", global_cut=1.0, skin=0.3, max_rho=10.0, nl_f=1, dt=0.04,
                thermo=100, run=1000, data="system.data", pair="dpd", temp=1.0, rc=1.0, rd=0.75,
                seed=12345, coeffs=(), bond_style=None, bond_coeffs=(), groups=(("all", (1,)),),
                fixes=(("md", "all", "nve"),), computes=(), extra=(), angle_style=None, angle_coeffs=()):
    lines = [f"atom_style {atom_style}",
             f"neighbor {global_cut} {skin} {max_rho} {nl_f}",
             f"timestep {dt}",
             f"thermo {thermo}",
             f"run {run}",
             f"read_data {data}"]
    if pair == "dpd":
        lines.append(f"pair_style dpd {temp} {rc} {seed}")
    else:
        lines.append(f"pair_style mdpd {temp} {rc} {rd} {seed}")
    for c in coeffs:
        lines.append("pair_coeff " + " ".join(str(v) for v in c))
    if bond_style:
        lines.append(f"bond_style {bond_style}")
        for c in bond_coeffs:
            lines.append("bond_coeff " + " ".join(str(v) for v in c))
    if angle_style:
        lines.append(f"angle_style {angle_style}")
        for c in angle_coeffs:
            lines.append("angle_coeff " + " ".join(str(v) for v in c))
    for name, types in groups:
        lines.append(f"group {name} type " + " ".join(str(t) for t in types))
    for fid, grp, style in fixes:
        lines.append(f"fix {fid} {grp} {style}")
    for c in computes:
        lines.append("compute " + " ".join(str(v) for v in c))
    lines.extend(extra)
    return "\n".join(lines) + "\n"


def plain_dpd(L=10.0, rho=3.0, seed=2024, a=25.0, gamma=4.5, kT=1.0, dt=0.04, nsteps=1000,
              skin=0.3, thermo=100, data="system.data", max_rho=10.0):
    """Single-species Groot-Warren DPD in a cubic periodic box (N = rho L^3)."""
    rng = np.random.default_rng(seed)
    n = int(round(rho * L ** 3))
    x = rng.uniform(0.0, L, size=(n, 3))
    m = np.ones(n)
    v = _velocities(rng, n, kT, m)
    run = run_in_text(skin=skin, dt=dt, thermo=thermo, run=nsteps, data=data, temp=kT,
                      seed=seed % 1000003, coeffs=[(1, 1, a, gamma)], max_rho=max_rho)
    return System([0, 0, 0], [L, L, L], [1.0], np.ones(n, dtype=np.int32), x, v, run_in=run)


def diblock_melt(L=100.0, rho=3.0, chain=10, n_a=5, seed=7, bond_k=4.0, bond_step=0.9, kT=1.0,
                 dt=0.04, nsteps=10000, skin=0.3, thermo=1000, a_same=25.0, a_ab=40.0, gamma=4.5,
                 data="system.data", max_rho=10.0):
    """A5B5 diblock melt: chains grown as seeded random walks with step `bond_step`."""
    rng = np.random.default_rng(seed)
    n = int(round(rho * L ** 3))
    nchain = n // chain
    n = nchain * chain
    start = rng.uniform(0.0, L, size=(nchain, 3))
    d = rng.normal(size=(nchain, chain - 1, 3))
    d *= bond_step / np.linalg.norm(d, axis=2, keepdims=True)
    pos = np.concatenate([start[:, None, :], start[:, None, :] + np.cumsum(d, axis=1)], axis=1)
    x = np.mod(pos.reshape(-1, 3), L)
    types = np.tile(np.r_[np.ones(n_a, dtype=np.int32), 2 * np.ones(chain - n_a, dtype=np.int32)], nchain)
    mol = np.repeat(np.arange(1, nchain + 1, dtype=np.int32), chain)
    idx = np.arange(n, dtype=np.int64).reshape(nchain, chain)
    bi = idx[:, :-1].reshape(-1) + 1
    bj = idx[:, 1:].reshape(-1) + 1
    bonds = np.column_stack([np.ones(len(bi), dtype=np.int64), bi, bj]).astype(np.int32)
    m = np.ones(n)
    v = _velocities(rng, n, kT, m)
    run = run_in_text(atom_style="bond", skin=skin, dt=dt, thermo=thermo, run=nsteps, data=data,
                      temp=kT, seed=seed % 1000003, max_rho=max_rho,
                      coeffs=[(1, 1, a_same, gamma), (1, 2, a_ab, gamma), (2, 2, a_same, gamma)],
                      bond_style="harmonic", bond_coeffs=[(1, bond_k, 0.0)],
                      groups=(("all", (1, 2)),))
    return System([0, 0, 0], [L, L, L], [1.0, 1.0], types, x, v, bonds=bonds, n_bondtypes=1,
                  mol=mol, run_in=run, atom_style="bond")


def mdpd_slab(Lx=40.0, Ly=40.0, Lz=120.0, z0=40.0, z1=80.0, rho=6.0, rho_vapour=0.0, seed=11,
              A=-40.0, B=25.0, gamma=4.5, rd=0.75, kT=1.0, dt=0.01, nsteps=20000, skin=0.3,
              thermo=1000, data="system.data", max_rho=30.0):
    """Many-body DPD liquid slab of density rho between z0 and z1 (vapour at rho_vapour)."""
    rng = np.random.default_rng(seed)
    nl = int(round(rho * Lx * Ly * (z1 - z0)))
    xl = np.column_stack([rng.uniform(0, Lx, nl), rng.uniform(0, Ly, nl), rng.uniform(z0, z1, nl)])
    nv = int(round(rho_vapour * Lx * Ly * (Lz - (z1 - z0))))
    if nv:
        zv = rng.uniform(0, Lz - (z1 - z0), nv)
        zv = np.where(zv < z0, zv, zv + (z1 - z0))
        xv = np.column_stack([rng.uniform(0, Lx, nv), rng.uniform(0, Ly, nv), zv])
        x = np.vstack([xl, xv])
    else:
        x = xl
    n = len(x)
    v = _velocities(rng, n, kT, np.ones(n))
    run = run_in_text(skin=skin, dt=dt, thermo=thermo, run=nsteps, data=data, pair="mdpd",
                      temp=kT, rc=1.0, rd=rd, seed=seed % 1000003, coeffs=[(1, 1, A, B, gamma)],
                      max_rho=max_rho)
    return System([0, 0, 0], [Lx, Ly, Lz], [1.0], np.ones(n, dtype=np.int32), x, v, run_in=run)


def angle_chains(L=10.0, rho=3.0, chain=10, n_a=5, seed=17, bond_k=4.0, angle_k=2.0, theta0=180.0,
                 bond_step=0.9, kT=1.0, dt=0.04, nsteps=1000, skin=0.3, thermo=100, a_same=25.0,
                 a_ab=40.0, gamma=4.5, data="system.data", max_rho=10.0):
    """A5B5 chains with harmonic bonds and harmonic angles (E = k (theta - theta0)^2) on every
    consecutive bead triple (atom_style angle)."""
    s = diblock_melt(L=L, rho=rho, chain=chain, n_a=n_a, seed=seed, bond_k=bond_k, bond_step=bond_step,
                     kT=kT, dt=dt, nsteps=nsteps, skin=skin, thermo=thermo, a_same=a_same, a_ab=a_ab,
                     gamma=gamma, data=data, max_rho=max_rho)
    nchain = s.n // chain
    idx = np.arange(nchain * chain).reshape(nchain, chain) + 1
    ai, aj, ak = idx[:, :-2].reshape(-1), idx[:, 1:-1].reshape(-1), idx[:, 2:].reshape(-1)
    angles = np.column_stack([np.ones(len(ai), dtype=np.int64), ai, aj, ak]).astype(np.int32)
    run = run_in_text(atom_style="angle", skin=skin, dt=dt, thermo=thermo, run=nsteps, data=data,
                      temp=kT, seed=seed % 1000003, max_rho=max_rho,
                      coeffs=[(1, 1, a_same, gamma), (1, 2, a_ab, gamma), (2, 2, a_same, gamma)],
                      bond_style="harmonic", bond_coeffs=[(1, bond_k, 0.0)],
                      angle_style="harmonic", angle_coeffs=[(1, angle_k, theta0)],
                      groups=(("all", (1, 2)),))
    return System(s.lo, s.hi, s.masses, s.types, s.x, s.v, bonds=s.bonds, n_bondtypes=1, mol=s.mol,
                  run_in=run, atom_style="angle", angles=angles, n_angletypes=1)


def binary_mixture(L, a_ab, rho=3.0, seed=0, a_same=25.0, gamma=4.5, kT=1.0, dt=0.04, nsteps=5000,
                   skin=0.3, thermo=100, rdf=None, data="system.data", max_rho=10.0):
    """50/50 A/B monomer mixture; rdf=(rmax, nbins, every) adds an A-B RDF compute."""
    rng = np.random.default_rng(seed)
    n = int(round(rho * L ** 3))
    x = rng.uniform(0.0, L, size=(n, 3))
    types = np.ones(n, dtype=np.int32)
    types[rng.permutation(n)[: n // 2]] = 2
    v = _velocities(rng, n, kT, np.ones(n))
    computes = ()
    if rdf is not None:
        rmax, nbins, every = rdf
        computes = (("gab", "all", "rdf", 1, 2, rmax, nbins, every, "rdf.txt"),)
    run = run_in_text(skin=skin, dt=dt, thermo=thermo, run=nsteps, data=data, temp=kT,
                      seed=(seed * 7919 + 17) % 1000003, max_rho=max_rho,
                      coeffs=[(1, 1, a_same, gamma), (1, 2, a_ab, gamma), (2, 2, a_same, gamma)],
                      groups=(("all", (1, 2)),), computes=computes)
    return System([0, 0, 0], [L, L, L], [1.0, 1.0], types, x, v, run_in=run)


def probe_fixes(L=9.0, rho=3.0, seed=23, radius=1.5, probe_mass=2.0, spring_k=50.0, spring_r0=0.2,
                spring_file=("spring.txt", 2), rvcm=(3, 1, 0, 1), recenter_every=4, kT=1.0, dt=0.04,
                nsteps=1000, skin=0.3, thermo=100, a_same=25.0, a_ab=30.0, gamma=4.5,
                data="system.data", max_rho=10.0):
    """Solvent (type 1) around a spherical probe cluster (type 2, mass `probe_mass`) with the
    group fixes: a spring pulling the probe's centre of mass towards a point one unit
    from the box centre (to within spring_r0), rvcm on everything (every rvcm[0] steps,
    flags rvcm[1:]), and recenter of the probe to the box centre every `recenter_every`
    steps.  The probe starts one unit on the other side of the centre."""
    rng = np.random.default_rng(seed)
    n = int(round(rho * L ** 3))
    x = rng.uniform(0.0, L, size=(n, 3))
    centre = np.full(3, L / 2.0)
    probe_at = centre - np.array([1.0, 0.0, 0.0])
    types = np.where(np.linalg.norm(x - probe_at, axis=1) < radius, 2, 1).astype(np.int32)
    masses = [1.0, float(probe_mass)]
    v = _velocities(rng, n, kT, np.where(types == 2, probe_mass, 1.0))
    sx, sy, sz = centre + np.array([1.0, 0.0, 0.0])
    spring = f"spring {spring_k} {sx} {sy} {sz} {spring_r0}"
    if spring_file:
        spring += f" {spring_file[0]} {spring_file[1]}"
    fixes = (("md", "all", "nve"), ("spr", "probe", spring),
             ("rv", "all", "rvcm " + " ".join(str(q) for q in rvcm)),
             ("rc", "probe", f"recenter {recenter_every} {centre[0]} {centre[1]} {centre[2]}"))
    run = run_in_text(skin=skin, dt=dt, thermo=thermo, run=nsteps, data=data, temp=kT,
                      seed=(seed * 104729 + 3) % 1000003, max_rho=max_rho,
                      coeffs=[(1, 1, a_same, gamma), (1, 2, a_ab, gamma), (2, 2, a_same, gamma)],
                      groups=(("all", (1, 2)), ("probe", (2,))), fixes=fixes)
    return System([0, 0, 0], [L, L, L], masses, types, x, v, run_in=run)


def wall_channel(L=8.0, Lz=14.0, rho=3.0, wall=1.0, v_top=0.5, walls="two_wall", seed=71, kT=1.0, dt=0.04,
                 nsteps=1000, skin=0.3, thermo=100, a_ll=25.0, a_lw=30.0, gamma=4.5, contact=1.0,
                 data="system.data", max_rho=10.0):
    """Liquid (type 1) between two particle walls along z: a frozen lo wall (type 2) in
    [0, wall) and a hi wall (type 3) in [Lz - wall, Lz) moved along x at v_top by fix move
    (Couette).  The liquid is integrated by fix nve and kept between the walls by fix
    two_wall (walls="two_wall") or by fix wall_reflect at the wall faces ("reflect");
    compute wall_contact counts liquid atoms within `contact` of the lo wall."""
    rng = np.random.default_rng(seed)
    n = int(round(rho * L * L * Lz))
    x = np.column_stack([rng.uniform(0, L, n), rng.uniform(0, L, n), rng.uniform(0, Lz, n)])
    types = np.where(x[:, 2] < wall, 2, np.where(x[:, 2] >= Lz - wall, 3, 1)).astype(np.int32)
    v = _velocities(rng, n, kT, np.ones(n))
    v[types != 1] = 0.0
    fixes = [("md", "liquid", "nve"), ("mv", "top", f"move {v_top} 0.0 0.0")]
    if walls == "two_wall":
        fixes.append(("tw", "liquid", "two_wall bottom top z"))
    else:
        fixes.append(("wr", "liquid", f"wall_reflect {wall} {Lz - wall} z"))
    computes = (("cwc", "liquid", "wall_contact", 1, "bottom", "lo", "z", contact, "wall_contact.txt"),)
    c = [(1, 1, a_ll, gamma), (1, 2, a_lw, gamma), (1, 3, a_lw, gamma), (2, 2, a_ll, gamma), (2, 3, a_ll, gamma),
         (3, 3, a_ll, gamma)]
    run = run_in_text(skin=skin, dt=dt, thermo=thermo, run=nsteps, data=data, temp=kT,
                      seed=(seed * 7907 + 11) % 1000003, max_rho=max_rho, coeffs=c,
                      groups=(("liquid", (1,)), ("bottom", (2,)), ("top", (3,))), fixes=tuple(fixes),
                      computes=computes)
    return System([0, 0, 0], [L, L, Lz], [1.0, 1.0, 1.0], types, x, v, run_in=run)


def replica_sweep(n_rep=256,L_min=8.0, L_max=24.0, a_lo=25.0, a_hi=45.0, seed=99, nsteps=5000,
                  rdf=(3.0, 150, 100), skin=0.3, thermo=100):
    """Uneven replicas: a_AB uniformly spaced over [a_lo, a_hi]; L drawn log-uniform."""
    rng = np.random.default_rng(seed)
    Ls = np.exp(rng.uniform(math.log(L_min), math.log(L_max), n_rep))
    out = []
    for r in range(n_rep):
        a_ab = a_lo + (a_hi - a_lo) * r / max(n_rep - 1, 1)
        rr = min(rdf[0], 0.5 * Ls[r]) if rdf else None
        out.append(binary_mixture(float(Ls[r]), a_ab, seed=seed * 1000 + r, nsteps=nsteps, skin=skin,
                                  thermo=thermo, rdf=None if rdf is None else (rr, rdf[1], rdf[2])))
    return out


def job_stream(n_jobs=32, seed=5, n_min=1000, n_max=200000, steps_min=1000, steps_max=20000,
               rate=1.0, chain_frac_max=0.5, rdf=(3.0, 150, 100), skin=0.3, thermo=100):
    """Served jobs with Poisson arrival times: list of (arrival_s, System)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for j in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        nt = int(rng.integers(1, 4))
        n_target = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        L = (n_target / 3.0) ** (1.0 / 3.0)
        L = max(L, 4.0)
        n = int(round(3.0 * L ** 3))
        x = rng.uniform(0.0, L, size=(n, 3))
        types = rng.integers(1, nt + 1, size=n).astype(np.int32)
        a = rng.uniform(25.0, 50.0, size=(nt, nt))
        a = np.triu(a) + np.triu(a, 1).T
        coeffs = [(i + 1, k + 1, round(float(a[i, k]), 4), 4.5) for i in range(nt) for k in range(i, nt)]
        frac = rng.uniform(0.0, chain_frac_max)
        nchain = int(frac * n) // 10
        bonds = None
        atom_style = "atomic"
        if nchain > 0 and nt >= 2:
            atom_style = "bond"
            for c in range(nchain):
                types[c * 10: c * 10 + 5] = 1
                types[c * 10 + 5: c * 10 + 10] = 2
            idx = np.arange(nchain * 10).reshape(nchain, 10)
            bi = idx[:, :-1].reshape(-1) + 1
            bj = idx[:, 1:].reshape(-1) + 1
            bonds = np.column_stack([np.ones(len(bi), dtype=np.int64), bi, bj]).astype(np.int32)
            # place chain beads near each other
            start = x[idx[:, 0]]
            d = rng.normal(size=(nchain, 9, 3))
            d *= 0.9 / np.linalg.norm(d, axis=2, keepdims=True)
            pos = np.concatenate([start[:, None, :], start[:, None, :] + np.cumsum(d, axis=1)], axis=1)
            x[: nchain * 10] = np.mod(pos.reshape(-1, 3), L)
        steps = int(rng.integers(steps_min, steps_max + 1))
        v = _velocities(rng, n, 1.0, np.ones(n))
        computes = ()
        if rdf is not None and nt >= 2:
            computes = (("g12", "all", "rdf", 1, 2, min(rdf[0], 0.5 * L), rdf[1], rdf[2], "rdf.txt"),)
        run = run_in_text(atom_style=atom_style, skin=skin, thermo=thermo, run=steps,
                          seed=int(rng.integers(1, 1 << 30)), coeffs=coeffs,
                          bond_style="harmonic" if bonds is not None else None,
                          bond_coeffs=[(1, 4.0, 0.0)] if bonds is not None else (),
                          groups=(("all", tuple(range(1, nt + 1))),), computes=computes)
        sysj = System([0, 0, 0], [L, L, L], np.ones(nt), types, x, v, bonds=bonds,
                      n_bondtypes=1 if bonds is not None else 0, run_in=run, atom_style=atom_style)
        jobs.append((t, sysj, steps))
    return jobs
