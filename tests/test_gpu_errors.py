"""Error paths of the device pipeline (B200 only), made to happen on purpose
without faulting the GPU.

The time transform waits for the bulk copy of each sample's series with a
bounded poll.  SMD_TFFT_POLL_LIMIT=0 makes that wait give up at once: the
kernel must record the expiry in the job's status word, let the copy already
in flight land, and return; smd_run must then report SMD_ETIMEOUT, and the
context must stay usable for the next job.
"""
import numpy as np
import pytest

from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [_lib.SMD_FP64, _lib.SMD_FP32], ids=["fp64", "fp32"])
def test_time_transform_wait_expiry_is_reported(ctx, monkeypatch, precision):
    s = SMDSettings(geom="square", L=16, J2=0.6, dtm=0.01, ntm=64)
    lat = smd.build_lattice(s.geom, s.L)
    lid = ctx.lattice(s, lat)
    qid = ctx.qset(lid)
    spins, _ = smp.make_samples(s, 2, "stripe", 0.2, 3)
    kw = dict(stride=2, precision=precision, fix_every=1 if precision == _lib.SMD_FP64 else 16)
    good = ctx.run(lid, qid, spins, s.dtm, 64, **kw)
    monkeypatch.setenv("SMD_TFFT_POLL_LIMIT", "0")
    with pytest.raises(_lib.SMDError) as e:
        ctx.run(lid, qid, spins, s.dtm, 64, **kw)
    assert e.value.code == _lib.SMD_ETIMEOUT
    assert "time transform" in str(e.value)
    monkeypatch.delenv("SMD_TFFT_POLL_LIMIT")
    again = ctx.run(lid, qid, spins, s.dtm, 64, **kw)
    assert np.array_equal(again.spec, good.spec)
    assert np.array_equal(again.qss, good.qss)
