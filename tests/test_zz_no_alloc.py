"""dpd_pair_forces_noalloc: the pair_style dpd force for callers that may not allocate
device memory (a plugin in a host code that owns every device buffer, or a
fixed-latency loop where cudaMalloc/cudaFree would synchronize the device).  It keeps
its cell binning in a fixed static device array instead of engine buffers.

Each test calls it through the C ABI on two calls in a row (different positions and
step, so the second call sees the first call's leftovers in the shared array) and
compares with dpd_pair_compute_aos, the engine-backed entry point, and with the FP64
oracle on the same inputs, within the force tolerance the other force tests use:
max |dF| / F_rms < 1e-5.  The device's free memory is the same before and after the
second call.  The file is named to run last, after every other GPU test has used the
device."""
import ctypes

import numpy as np
import pytest

from conftest import force_err

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _params(system):
    """dpd_pair_params of a pair_style dpd run.in and its box."""
    from gpumdpd_b200 import capi
    p = capi.dpd_pair_params()
    for k in range(3):
        p.lo[k], p.hi[k] = float(system.lo[k]), float(system.hi[k])
    p.ntypes = len(system.masses)
    rc = 1.0
    coeffs = {}
    for line in system.run_in.splitlines():
        t = line.split("#")[0].split()
        if t and t[0] == "timestep":
            p.dt = float(t[1])
        if t and t[0] == "pair_style":
            assert t[1] == "dpd"
            p.kT, rc, p.seed = float(t[2]), float(t[3]), int(t[4])
        if t and t[0] == "pair_coeff":
            coeffs[(int(t[1]), int(t[2]))] = [float(v) for v in t[3:]]
    for (a, b), c in coeffs.items():
        row = (c[0], c[1], c[2] if len(c) > 2 else rc)
        for (i, j) in ((a, b), (b, a)):
            for k in range(3):
                p.coeff[i - 1][j - 1][k] = row[k]
    return p


def _cases():
    from gpumdpd_b200 import inputs
    return {
        "one_type_L8": inputs.plain_dpd(L=8.0, seed=21, nsteps=10),
        "two_types_L10": inputs.binary_mixture(L=10.0, a_ab=40.0, seed=22, nsteps=10),
    }


@pytest.mark.parametrize("name", ["one_type_L8", "two_types_L10"])
def test_noalloc_matches_engine_entry_point(name, oracle_mod):
    import torch
    from gpumdpd_b200 import Engine, capi
    s = _cases()[name]
    lib = capi.load()
    e = Engine(s.run_in, system=s.c_system())
    c = e.cells()
    L = (c["nc"].astype(np.float64) * c["w"].astype(np.float64)).astype(np.float32)
    params = _params(s)
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    ids = torch.arange(1, s.n + 1, dtype=torch.int32, device=dev)
    types = torch.tensor(s.types, dtype=torch.int32, device=dev)
    rng = np.random.default_rng(5)
    x = s.x.astype(np.float32)
    v = s.v.astype(np.float32)
    for call, step in enumerate((3, 4)):
        if call == 1:  # move every particle a little, a few of them across the box
            x = np.mod(x + rng.normal(0, 0.05, x.shape).astype(np.float32), L)
            x = np.where(x >= L, 0.0, x).astype(np.float32)
            v = (v + rng.normal(0, 0.1, v.shape)).astype(np.float32)
        xd = torch.tensor(x.reshape(-1), device=dev)
        vd = torch.tensor(v.reshape(-1), device=dev)
        f_ref = torch.zeros(3 * s.n, device=dev)
        e.pair_compute_aos(xd.data_ptr(), vd.data_ptr(), ids.data_ptr(), types.data_ptr(), s.n, step,
                           f_ref.data_ptr())
        f_na = torch.full((3 * s.n,), float("nan"), device=dev)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        code = lib.dpd_pair_forces_noalloc(ctypes.byref(params), xd.data_ptr(), vd.data_ptr(), ids.data_ptr(),
                                           types.data_ptr(), s.n, step, f_na.data_ptr(), stream)
        assert code == 0
        if call == 1:  # after the first call has loaded the module: no device memory taken
            assert torch.cuda.mem_get_info()[0] == free0
        a = f_na.cpu().numpy().reshape(-1, 3).astype(np.float64)
        b = f_ref.cpu().numpy().reshape(-1, 3).astype(np.float64)
        assert np.isfinite(a).all()
        assert force_err(a, b) < TOL, (name, call)
        ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
        o = oracle_mod.forces(ff, np.arange(1, s.n + 1), s.types, x.astype(np.float64), v.astype(np.float64),
                              s.lo, L.astype(np.float64), step)
        assert force_err(a, o["f"]) < TOL, (name, call)
        np.testing.assert_allclose(a.sum(axis=0), 0.0, atol=1e-3 * np.sqrt(np.mean(b * b)) * np.sqrt(s.n))
    e.close()


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch
    from gpumdpd_b200 import capi, inputs
    lib = capi.load()
    s = inputs.plain_dpd(L=8.0, seed=23, nsteps=10)
    dev = torch.device("cuda")
    xd = torch.tensor(s.x.astype(np.float32).reshape(-1), device=dev)
    vd = torch.zeros(3 * s.n, device=dev)
    ids = torch.arange(1, s.n + 1, dtype=torch.int32, device=dev)
    types = torch.tensor(s.types, dtype=torch.int32, device=dev)
    fd = torch.zeros(3 * s.n, device=dev)
    args = (xd.data_ptr(), vd.data_ptr(), ids.data_ptr(), types.data_ptr())

    def call(p, n):
        return lib.dpd_pair_forces_noalloc(ctypes.byref(p), *args, n, 0, fd.data_ptr(), None)

    p = _params(s)
    assert call(p, capi.NOALLOC_MAX_ATOMS + 1) == -1   # too many atoms
    assert call(p, 0) == -1
    big = _params(s)
    for k in range(3):
        big.hi[k] = 70.0                                 # 70^3 cells > DPD_NOALLOC_MAX_CELLS
    assert call(big, s.n) == -1
    small = _params(s)
    small.hi[2] = 2.5                                    # fewer than 3 cells along z
    assert call(small, s.n) == -1
    many = _params(s)
    many.ntypes = capi.NOALLOC_MAX_TYPES + 1
    assert call(many, s.n) == -1
    bad = ids.clone()
    bad[7] = 0                                           # ids start at 1
    assert lib.dpd_pair_forces_noalloc(ctypes.byref(p), xd.data_ptr(), vd.data_ptr(), bad.data_ptr(),
                                       types.data_ptr(), s.n, 0, fd.data_ptr(), None) == -1
    far = xd.clone()
    far[3 * 11 + 1] = 9.5                                # a cell and a half beyond hi = 8
    assert lib.dpd_pair_forces_noalloc(ctypes.byref(p), far.data_ptr(), vd.data_ptr(), ids.data_ptr(),
                                       types.data_ptr(), s.n, 0, fd.data_ptr(), None) == -1
    # a valid call still works after the rejected ones
    assert call(p, s.n) == 0
    assert torch.isfinite(fd).all()
