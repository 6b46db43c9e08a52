import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built extension")
    config.addinivalue_line("markers", "ref: needs the compiled reference library oracle/_ref")


_SYS_CACHE = {}


def get_system(name: str):
    """Build (once per session) the tomography tables of a preset."""
    if name not in _SYS_CACHE:
        from maos_b200 import config, geometry
        _SYS_CACHE[name] = geometry.build_tomo(config.PRESETS[name]())
    return _SYS_CACHE[name]


_FIT_CACHE = {}


def get_fit(name: str):
    """Build (once per session) the DM-fit tables of a preset."""
    if name not in _FIT_CACHE:
        from maos_b200 import fit_setup
        _FIT_CACHE[name] = fit_setup.build_fit(get_system(name))
    return _FIT_CACHE[name]


_AFIT_CACHE = {}


def get_fit_assembled(name: str):
    """Build (once per session) the assembled fit (reference defaults) of a preset."""
    if name not in _AFIT_CACHE:
        from maos_b200 import fit_assemble
        _AFIT_CACHE[name] = fit_assemble.build_fit_assembled(get_system(name))
    return _AFIT_CACHE[name]


@pytest.fixture(scope="session")
def ltao():
    return get_system("ltao_8m")


@pytest.fixture(scope="session")
def mcao():
    return get_system("mcao_30m")
