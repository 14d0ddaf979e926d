import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "ls-sph-benchmarks_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    import importlib.util
    lib = os.path.join(ROOT, "ls-sph-benchmarks_b200", "lib", "liblssph.so")
    if not os.path.exists(lib):
        spec = importlib.util.spec_from_file_location("lssph_build", os.path.join(ROOT, "ls-sph-benchmarks_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    orc = os.path.join(ROOT, "oracle", "_build", "liblssph_oracle.so")
    if not os.path.exists(orc):
        spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(ROOT, "oracle", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()


_ensure_built()


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="session")
def reference_root():
    """The reference checkout named by $LSSPH_REFERENCE_ROOT, only present where the
    fixtures are generated; tests that need it are skipped elsewhere."""
    path = os.environ.get("LSSPH_REFERENCE_ROOT", "")
    if not path or not os.path.isdir(os.path.join(path, "analysis")):
        pytest.skip("reference checkout not available on this machine")
    return path
