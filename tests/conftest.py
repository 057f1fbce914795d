"""Shared fixtures.  `gpu` marks tests that need a CUDA device (B200)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs with -m gpu)")


@pytest.fixture(scope="session")
def orc():
    """The CPU oracle (test infrastructure), built on first use."""
    import oracle
    if not os.path.exists(oracle.LIB_PATH):
        oracle.build()
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def atvb():
    """The product library; GPU tests fail loudly if it is not built."""
    import atomiverse_b200 as A
    A.load()
    return A


@pytest.fixture(scope="session")
def ctx(atvb):
    return atvb.Context(0)


def oracle_system(orc, desc: dict, frame: dict, **over):
    """An oracle system with the same description as a product system."""
    d = dict(desc)
    d.update(over)
    box = d["box"]
    kw = dict(nl_cutoff=d["nl_cutoff"], skin=d.get("nl_skin", 0.3),
              nl_every=d.get("nl_every", 1), nl_delay=d.get("nl_delay", 0),
              nl_check=d.get("nl_check", 1),
              has_lj=d.get("lj_enabled", 0), lj_eps=d.get("lj_epsilon", 1.0),
              lj_sigma=d.get("lj_sigma", 1.0), lj_rc=d.get("lj_cutoff", d["nl_cutoff"]),
              has_coul=d.get("coul_enabled", 0), coul_alpha=d.get("coul_alpha", 0.0),
              coul_rc=d.get("coul_cutoff", d["nl_cutoff"]),
              has_pme=d.get("pme_enabled", 0), pme_alpha=d.get("pme_alpha", 0.0),
              pme_K=d.get("pme_grid", (0, 0, 0)), pme_order=d.get("pme_order", 4),
              dt=d.get("dt", 1.0), thermostat=d.get("thermostat", 0),
              T=d.get("temperature", 0.0), tau=d.get("tau", 100.0),
              damp=d.get("damp", 100.0), seed=d.get("seed", 0),
              need_virial=d.get("stress_required", 1),
              T_stop=d.get("lang_T_stop", d.get("temperature", 0.0)),
              lang_nfirst=d.get("lang_nfirst", 0), lang_nlast=d.get("lang_nlast", 0),
              wall_axis=d.get("wall_axis", -1), wall_pos=d.get("wall_pos", 0.0),
              wall_k=d.get("wall_k", 0.0))
    s = orc.OracleSystem(orc.make_desc(d["n_atoms"], box, **kw))
    s.set_state(frame["x"], frame["y"], frame["z"], frame.get("vx"), frame.get("vy"),
                frame.get("vz"), frame.get("fx"), frame.get("fy"), frame.get("fz"),
                frame.get("mass"), frame.get("charge"), frame.get("tag"))
    return s


def rms_rel(f, fref):
    f = np.asarray(f)
    fref = np.asarray(fref)
    return float(np.sqrt(((f - fref) ** 2).sum()) / np.sqrt((fref ** 2).sum()))
