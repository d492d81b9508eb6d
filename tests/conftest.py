import importlib.util
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _load_package():
    """Import the t-blaeq_b200 package directory (not a valid identifier) as `tblaeq_b200`."""
    if "tblaeq_b200" in sys.modules:
        return sys.modules["tblaeq_b200"]
    pkg_dir = os.path.join(REPO, "t-blaeq_b200")
    spec = importlib.util.spec_from_file_location("tblaeq_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tblaeq_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def tb():
    return _load_package()


@pytest.fixture(scope="session")
def wl(tb):
    import importlib
    return importlib.import_module("tblaeq_b200.workloads")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.fail("this test needs a CUDA device")
    return True


def oracle_from_handler(oracle_mod, h, tmpdir):
    """Oracle view of a handler's index, read back from disk by the oracle's own loader."""
    path = os.path.join(str(tmpdir), "idx")
    h.save_index(path)
    return oracle_mod.load_index(path)


def ids_by_query(offsets, ids):
    offsets = np.asarray(offsets, dtype=np.int64)
    return [np.sort(ids[offsets[i]:offsets[i + 1]]) for i in range(len(offsets) - 1)]
