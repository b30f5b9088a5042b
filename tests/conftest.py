"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def mech_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("mechs"))


def _make(name, mech_dir):
    from openhurricane_b200 import synth, mechanism
    m = {"small": synth.small_mechanism, "large": synth.large_mechanism,
         "ext": synth.extended_mechanism, "fitted": synth.fitted_rates_mechanism}[name]()
    d = os.path.join(mech_dir, name)
    che, th, tr = synth.write_chemkin(m, d)
    tables = mechanism.compile_mechanism(che, th, tr)
    return {"mech": m, "tables": tables, "files": (che, th, tr), "dir": d}


@pytest.fixture(scope="session")
def small(mech_dir):
    return _make("small", mech_dir)


@pytest.fixture(scope="session")
def large(mech_dir):
    return _make("large", mech_dir)


@pytest.fixture(scope="session")
def ext(mech_dir):
    """The small mechanism's species with SRI, REV, FORD / RORD and unit keywords."""
    return _make("ext", mech_dir)


@pytest.fixture(scope="session")
def fitted(mech_dir):
    """The small mechanism with one Janev (JAN) and one power-series (FIT1) rate."""
    return _make("fitted", mech_dir)
