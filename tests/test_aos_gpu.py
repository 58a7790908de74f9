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
