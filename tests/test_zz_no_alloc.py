"""pmgpu_gb_forces_noalloc (GB forces from a static device scratch, no
device allocation) against the allocating path, pmgpu_force_evaluate on a
GBForce term, through the C ABI.  Kept in the last-collected file so it also
runs after every other GPU test has used the device."""
import ctypes as C

import numpy as np
import pytest

import fixtures as F
from protomol_b200 import ForceFactory, GpuSystem, ScalarStructure
from protomol_b200 import _lib as L

pytestmark = pytest.mark.gpu

SOLUTE, SOLVENT = 1.0, 78.3


def _noalloc(lib, topo, pos, precision, with_water=True):
    import torch
    dev = torch.device("cuda", 0)
    n = pos.shape[0]
    t = {k: torch.as_tensor(np.ascontiguousarray(v), device=dev)
         for k, v in (("pos", pos.reshape(-1)), ("charge", topo.charge),
                      ("vdwr", topo.gb_vdwr), ("scale", topo.gb_scale),
                      ("offset", topo.gb_offset))}
    water = torch.as_tensor(topo.water.astype(np.int32), device=dev) if with_water else None
    forces = torch.full((3 * n,), np.nan, dtype=torch.float64, device=dev)
    energy = torch.full((1,), np.nan, dtype=torch.float64, device=dev)
    obc = (C.c_double * 3)(*topo.gb_obc)
    stream = torch.cuda.current_stream(dev)
    rc = lib.pmgpu_gb_forces_noalloc(
        n, t["pos"].data_ptr(), t["charge"].data_ptr(), t["vdwr"].data_ptr(),
        t["scale"].data_ptr(), t["offset"].data_ptr(),
        water.data_ptr() if water is not None else None, obc,
        SOLUTE, SOLVENT, precision, forces.data_ptr(), energy.data_ptr(),
        stream.cuda_stream)
    L.check(rc)
    stream.synchronize()
    return forces.cpu().numpy().reshape(n, 3), float(energy.cpu()[0])


def _allocating(gb, pos):
    f = np.zeros_like(pos)
    e = ScalarStructure()
    gb.evaluate(pos, f, e)
    return f, e[0]


@pytest.mark.parametrize("precision,name", [("mixed", L.PREC_MIXED), ("double", L.PREC_DOUBLE)])
def test_noalloc_matches_allocating_path(ctx, precision, name):
    lib = L.load()
    z = F.load("fip35_gb")
    topo = F.topology(z)
    gs = GpuSystem(ctx, topo, precision)
    gb = ForceFactory(gs).make(
        f"GBForce -algorithm NonbondedSimpleFull -soluteDielec {SOLUTE} -solventDielec {SOLVENT}")
    rng = np.random.default_rng(7)
    # two calls in a row, the second at displaced positions: the shared
    # scratch keeps the first call's contents and must not leak into it
    for pos in (topo.pos, topo.pos + rng.normal(0.0, 0.05, topo.pos.shape)):
        f_ref, e_ref = _allocating(gb, pos)
        f, e = _noalloc(lib, topo, pos, name)
        assert np.all(np.isfinite(f))
        assert F.rms_rel(f, f_ref) <= 1e-12, F.rms_rel(f, f_ref)
        assert abs(e - e_ref) <= 1e-9 * max(1.0, abs(e_ref)), (e, e_ref)
    gs.close()


@pytest.mark.parametrize("precision,name", [("mixed", L.PREC_MIXED), ("double", L.PREC_DOUBLE)])
@pytest.mark.parametrize("n", [1, 33, 65, L.GB_STATIC_MAX_ATOMS])
def test_noalloc_small_ragged_and_limit_sizes(ctx, n, precision, name):
    """Heteropolymers below one 32-atom tile, with a ragged last tile, and
    at the static limit (where the carved scratch ends exactly at the end of
    the array), with no water array (every atom solute), twice in a row."""
    from protomol_b200 import systems
    lib = L.load()
    sm = systems.gb_polymer(n, seed=11)
    sm.water = np.zeros(n, np.int32)
    gs = GpuSystem(ctx, sm, precision)
    gb = ForceFactory(gs).make(
        f"GBForce -algorithm NonbondedSimpleFull -soluteDielec {SOLUTE} -solventDielec {SOLVENT}")
    rng = np.random.default_rng(n)
    for pos in (sm.pos, sm.pos + rng.normal(0.0, 0.05, sm.pos.shape)):
        f_ref, e_ref = _allocating(gb, pos)
        f, e = _noalloc(lib, sm, pos, name, with_water=False)
        assert np.all(np.isfinite(f))
        if np.abs(f_ref).max() > 0:
            assert F.rms_rel(f, f_ref) <= 1e-12, F.rms_rel(f, f_ref)
        else:
            assert np.abs(f).max() == 0.0
        assert abs(e - e_ref) <= 1e-9 * max(1.0, abs(e_ref)), (e, e_ref)
    gs.close()


def test_noalloc_rejects_oversize(ctx):
    lib = L.load()
    obc = (C.c_double * 3)(1.0, 0.8, 4.85)
    n = L.GB_STATIC_MAX_ATOMS + 1
    # rejected on the size alone, before any pointer is looked at
    rc = lib.pmgpu_gb_forces_noalloc(n, None, None, None, None, None, None, obc,
                                     1.0, 80.0, L.PREC_MIXED, None, None, None)
    assert rc == L.ERR_ARG
    assert b"static GB scratch limit" in lib.pmgpu_last_error()
