"""dpd_pair_compute_aos: the drop-in for Pair::compute_force on the reference's own
device buffers (AoS float[3N] positions/velocities, int[N] ids/types, index = id-1),
checked against the FP64 oracle; per-atom PE and virial against the oracle's totals."""
import numpy as np
import pytest

from conftest import force_err

pytestmark = pytest.mark.gpu


def _aos_case(system_name):
    from gpumdpd_b200 import inputs
    if system_name == "dpd":
        return inputs.plain_dpd(L=8.0, seed=12, nsteps=10)
    return inputs.mdpd_slab(Lx=8.0, Ly=8.0, Lz=20.0, z0=6.0, z1=14.0, seed=13, nsteps=10)


@pytest.mark.parametrize("name", ["dpd", "mdpd"])
def test_pair_compute_aos_matches_oracle(oracle_mod, name):
    import torch
    from gpumdpd_b200 import Engine
    s = _aos_case(name)
    e = Engine(s.run_in, system=s.c_system())
    c = e.cells()
    L = c["nc"].astype(np.float64) * c["w"].astype(np.float64)
    ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
    rng = np.random.default_rng(3)
    x = s.x.astype(np.float32)
    v = s.v.astype(np.float32)
    dev = torch.device("cuda")
    ids = torch.arange(1, s.n + 1, dtype=torch.int32, device=dev)
    types = torch.tensor(s.types, dtype=torch.int32, device=dev)
    for call, step in enumerate((0, 1)):
        if call == 1:  # move the particles a little (list reuse) and a few across the box
            x = np.mod(x + rng.normal(0, 0.02, x.shape).astype(np.float32), L.astype(np.float32))
            x = np.where(x >= L.astype(np.float32), 0.0, x).astype(np.float32)
        xd = torch.tensor(x.reshape(-1), device=dev)
        vd = torch.tensor(v.reshape(-1), device=dev)
        fd = torch.zeros(3 * s.n, device=dev)
        pe = torch.zeros(s.n, device=dev)
        vir = torch.zeros(6 * s.n, device=dev)
        e.pair_compute_aos(xd.data_ptr(), vd.data_ptr(), ids.data_ptr(), types.data_ptr(), s.n, step,
                           fd.data_ptr(), pe.data_ptr(), vir.data_ptr())
        f = fd.cpu().numpy().reshape(-1, 3).astype(np.float64)
        o = oracle_mod.forces(ff, np.arange(1, s.n + 1), s.types, x.astype(np.float64), v.astype(np.float64),
                              s.lo, L, step)
        assert force_err(f, o["f"]) < 1e-5
        assert pe.sum().item() == pytest.approx(o["pair_pe"], rel=1e-5)
        vsum = vir.cpu().numpy().reshape(-1, 6).astype(np.float64).sum(axis=0)
        np.testing.assert_allclose(vsum, o["virial"], rtol=1e-4, atol=1e-3 * np.abs(o["virial"]).max())
        # forces only (no per-atom outputs) give the same forces
        fd2 = torch.zeros(3 * s.n, device=dev)
        e.pair_compute_aos(xd.data_ptr(), vd.data_ptr(), ids.data_ptr(), types.data_ptr(), s.n, step,
                           fd2.data_ptr(), None, None)
        assert force_err(fd2.cpu().numpy().reshape(-1, 3), o["f"]) < 1e-5


def test_pair_compute_aos_rejects_bad_input():
    import torch
    from gpumdpd_b200 import DpdError, Engine
    s = _aos_case("dpd")
    e = Engine(s.run_in, system=s.c_system())
    dev = torch.device("cuda")
    xd = torch.tensor(s.x.astype(np.float32).reshape(-1), device=dev)
    vd = torch.zeros(3 * s.n, device=dev)
    ids = torch.arange(1, s.n + 1, dtype=torch.int32, device=dev)
    types = torch.tensor(s.types, dtype=torch.int32, device=dev)
    fd = torch.zeros(3 * s.n, device=dev)
    with pytest.raises(DpdError):
        e.pair_compute_aos(xd.data_ptr(), vd.data_ptr(), ids.data_ptr(), types.data_ptr(), s.n - 1, 0,
                           fd.data_ptr())
    bad = ids.clone()
    bad[5] = s.n + 7
    with pytest.raises(DpdError) as ex:
        e.pair_compute_aos(xd.data_ptr(), vd.data_ptr(), bad.data_ptr(), types.data_ptr(), s.n, 0, fd.data_ptr())
    assert ex.value.code == -1


def test_bond_and_nve_aos_match_numpy():
    """dpd_bond_compute_aos and dpd_nve_aos on AoS device buffers against the same
    formulas in numpy (harmonic E = k (r - r0)^2 with the reference's minimum image; the
    velocity-Verlet half kick, drift and wrap): forces within FP32 rounding, per-bond
    energies and the virial, wrapped and unwrapped positions."""
    import torch
    from gpumdpd_b200 import Engine, inputs
    s = inputs.diblock_melt(L=8.0, seed=14, nsteps=10, bond_k=4.0)
    e = Engine(s.run_in, system=s.c_system())
    dev = torch.device("cuda")
    L = (s.hi - s.lo).astype(np.float32)
    x = s.x.astype(np.float32)
    bl = np.ascontiguousarray(s.bonds, dtype=np.int32)
    xd = torch.tensor(x.reshape(-1), device=dev)
    bd = torch.tensor(bl.reshape(-1), device=dev)
    fd = torch.zeros(3 * s.n, device=dev)
    pe = torch.zeros(len(bl), device=dev)
    vir = torch.zeros(6 * s.n, device=dev)
    e.bond_compute_aos(xd.data_ptr(), bd.data_ptr(), len(bl), fd.data_ptr(), pe.data_ptr(), vir.data_ptr())
    i, j = bl[:, 1] - 1, bl[:, 2] - 1
    d = x[i].astype(np.float64) - x[j]
    d -= L * ((d >= L / 2).astype(np.float64) - (d < -L / 2))
    r = np.linalg.norm(d, axis=1)
    fb = -2.0 * 4.0 * r / r  # bond_coeff 1 4.0 0.0: r0 = 0
    fvec = d * fb[:, None]
    f = np.zeros((s.n, 3))
    np.add.at(f, i, fvec)
    np.add.at(f, j, -fvec)
    assert np.abs(fd.cpu().numpy().reshape(-1, 3) - f).max() < 1e-4 * np.abs(f).max()
    np.testing.assert_allclose(pe.cpu().numpy(), 4.0 * r * r, rtol=1e-5)
    vsum = vir.cpu().numpy().reshape(-1, 6).astype(np.float64).sum(0)
    want = np.array([(d[:, a] * fvec[:, b]).sum() for a, b in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))])
    np.testing.assert_allclose(vsum, want, rtol=1e-4, atol=1e-4 * np.abs(want).max())
    # nve: the initial step on every atom, then the final half kick
    v = s.v.astype(np.float32)
    vd = torch.tensor(v.reshape(-1), device=dev)
    uw = torch.tensor(x.reshape(-1), device=dev)
    grp = torch.arange(s.n, dtype=torch.int32, device=dev)
    types = torch.tensor(s.types, dtype=torch.int32, device=dev)
    e.nve_aos(0, grp.data_ptr(), s.n, types.data_ptr(), xd.data_ptr(), uw.data_ptr(), vd.data_ptr(), fd.data_ptr())
    fa = fd.cpu().numpy().reshape(-1, 3).astype(np.float64)
    dt = 0.04
    v1 = v + 0.5 * dt * fa / s.masses[s.types - 1][:, None]
    xu = x + dt * v1
    np.testing.assert_allclose(vd.cpu().numpy().reshape(-1, 3), v1, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(uw.cpu().numpy().reshape(-1, 3), xu, rtol=1e-6, atol=1e-5)
    xw = xd.cpu().numpy().reshape(-1, 3)
    assert (xw >= 0).all() and (xw < L).all()
    dxw = xw - np.mod(xu, L)
    dxw -= L * np.round(dxw / L)
    assert np.abs(dxw).max() < 1e-5
    e.nve_aos(1, grp.data_ptr(), s.n, types.data_ptr(), xd.data_ptr(), uw.data_ptr(), vd.data_ptr(), fd.data_ptr())
    np.testing.assert_allclose(vd.cpu().numpy().reshape(-1, 3), v1 + 0.5 * dt * fa / s.masses[s.types - 1][:, None],
                               rtol=1e-5, atol=1e-5)
    # an index outside the system is reported, not used
    bad = torch.tensor([s.n + 5], dtype=torch.int32, device=dev)
    from gpumdpd_b200 import DpdError
    with pytest.raises(DpdError):
        e.nve_aos(1, bad.data_ptr(), 1, types.data_ptr(), xd.data_ptr(), uw.data_ptr(), vd.data_ptr(), fd.data_ptr())
