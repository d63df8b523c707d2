"""The allocation-free evolution entry point against the allocating one.

Some callers own every byte of device memory themselves -- a framework whose
memory pool holds the whole HBM budget, or a real-time loop that may not
allocate once it runs -- and so cannot let this library call cudaMalloc.
smd_evolve_fp64_noalloc serves them: its working memory is a static device
array.  These tests check, through the C ABI, that it computes what the
allocating smd_evolve computes, on two calls in a row (the array keeps the
previous call's contents between calls), in place and into a separate
buffer, on lattices with one and three sublattices, that the caller's status
word reports a clean run, and that oversized calls are refused.  The file is collected last so that a failure here leaves every
other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, samples as smp, smd
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings

pytestmark = pytest.mark.gpu

SPIN_TOL = 1e-10


def _model(s, lat, d_nbr):
    m = _lib.NoAllocModel()
    m.N = lat.N
    on = [True, s.j2_on, s.jx_on]
    J = [s.J1, s.J2, s.JX]
    lam = s.lambdas()
    for k in range(3):
        m.zn[k] = lat.zn[k] if on[k] else 0
        m.J[k] = J[k]
        for c in range(3):
            m.lambda_[3 * k + c] = lam[k][c]
    m.d_nbr = d_nbr
    m.h = s.h
    return m


def _ell(s, lat):
    on = [True, s.j2_on, s.jx_on]
    rows = [lat.nbrs[k].T for k in range(3) if on[k]]
    return np.ascontiguousarray(np.concatenate(rows, axis=0), np.int32)


CASES = {
    # square XXZ with field and three shells; triangular and kagome have more
    # neighbours per shell (kagome: three sublattices, a different table shape)
    "square_xxz_h": (SMDSettings(geom="square", L=16, J2=0.6, JX=0.1, zlamb1=0.9, zlamb2=0.9,
                                 h=0.2, dtm=0.01), "stripe"),
    "triang_j1j2": (SMDSettings(geom="triang", L=12, J2=0.12, dtm=0.02), "q120"),
    "kagome_j1j2": (SMDSettings(geom="kagome", L=6, J2=0.2, dtm=0.02), "ferro"),
}


@pytest.mark.parametrize("in_place", [False, True], ids=["separate", "in_place"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_noalloc_evolution_matches_smd_evolve_twice(ctx, name, in_place):
    """Two calls in a row through the C ABI equal smd_evolve within 1e-10 per
    spin, with the output in a separate buffer or written over the input,
    and the caller's status word reads 0 after each."""
    import torch
    s, state = CASES[name]
    lat = smd.build_lattice(s.geom, s.L)
    lid = ctx.lattice(s, lat)
    d_nbr = torch.from_numpy(_ell(s, lat)).cuda()
    model = _model(s, lat, d_nbr.data_ptr())
    lib = _lib.load()
    d_status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    for call in range(2):
        spins, _ = smp.make_samples(s, 4, state, 0.3, 100 + call)
        ref = ctx.evolve(lid, spins, s.dtm, 50)
        d_in = torch.from_numpy(spins).cuda()
        d_out = d_in if in_place else torch.empty_like(d_in)
        torch.cuda.synchronize()
        rc = lib.smd_evolve_fp64_noalloc(C.byref(model), 4, s.dtm, 50, d_in.data_ptr(),
                                         d_out.data_ptr(), d_status.data_ptr(), None)
        assert rc == _lib.SMD_OK
        torch.cuda.synchronize()
        assert int(d_status.item()) == 0
        out = d_out.cpu().numpy()
        assert np.max(np.abs(out - ref)) <= SPIN_TOL, (call, np.max(np.abs(out - ref)))


def test_noalloc_rejects_calls_beyond_its_static_scratch(ctx):
    import torch
    s = SMDSettings(geom="square", L=16, J2=0.6, dtm=0.01)
    lat = smd.build_lattice(s.geom, s.L)
    d_nbr = torch.from_numpy(_ell(s, lat)).cuda()
    model = _model(s, lat, d_nbr.data_ptr())
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    too_many = _lib.NOALLOC_SCRATCH_BYTES // (96 * lat.N) + 1
    rc = _lib.load().smd_evolve_fp64_noalloc(C.byref(model), too_many, s.dtm, 10,
                                             d.data_ptr(), d.data_ptr(), None, None)
    assert rc == _lib.SMD_ENOMEM_ADMIT
