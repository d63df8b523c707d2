import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")


def load_golden(name):
    from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    s = SMDSettings(**{k: v for k, v in json.loads(str(d["settings"])).items()})
    return s, d


def golden_lattice(oracle_mod, s, d):
    """The oracle's lattice of a fixture: built from the geometry for a
    crystal, from the fixture's reference tables for a quasi-crystal."""
    if s.qcrystal:
        return oracle_mod.tables_lattice(d["rvec"], (d["nb1"], d["nb2"], d["nbx"]), s.G)
    return oracle_mod.make_lattice(s.geom, s.L)


def golden_names(prefix=""):
    """Fixture names with the prefix; without one, the trajectory and
    spectrum cases (the text_ output-stage and mc_ Monte Carlo fixtures have
    other layouts)."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))
    return names if prefix else [n for n in names if not n.startswith(("text_", "mc_"))]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ctx():
    """A device context; on a GPU box a missing library or device is an error."""
    from classical_mc_and_smd_for_2d_heisenberg_models_b200.smd import Context
    c = Context(0)
    yield c
    c.close()
