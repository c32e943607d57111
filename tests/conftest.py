import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
CLI_TOOLS = ("wgpu_solver_backend_cli", "wgpu_solver_backend_convert_cli")
BIN = os.path.join(ROOT, "wgpu_solver_backend_b200", "bin")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100a device")


@pytest.fixture(scope="session", autouse=True)
def _built():
    import oracle

    oracle.build()
    pkg = os.path.join(ROOT, "wgpu_solver_backend_b200")
    built = [os.path.join(pkg, "libwsb.so")] + [os.path.join(pkg, "bin", t) for t in CLI_TOOLS]
    if not all(os.path.exists(f) for f in built):
        import subprocess

        subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(ROOT, "wgpu_solver_backend_b200")])


@pytest.fixture(scope="session")
def ctx():
    import wgpu_solver_backend_b200 as wsb

    return wsb.GpuContext.create("auto", 0)


def load_case(k):
    from wgpu_solver_backend_b200 import io as wio

    case = wio.load_case_dir(os.path.join(GOLDEN, f"case_{k}"))
    x_ref = wio.load_vector_bin(os.path.join(GOLDEN, f"case_{k}", "x_ref.bin"))
    fx = np.load(os.path.join(GOLDEN, f"case_{k}", "oracle_ref_f32.npz"))
    return case, x_ref, fx


# compare-x gates of commands.txt:56-78 (rel_tol, abs_tol) per dataset.
COMPARE_X_GATES = {1: (1e-3, 1e-2), 2: (1e-3, 1e0), 3: (1e-3, 1e1)}
# Solver settings of commands.txt:26-54.
DATASET_SOLVE = dict(max_iter=2000, rel_tol=1e-4, abs_tol=1e-7)
