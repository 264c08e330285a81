import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def golden_names(prefix):
    return sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


@pytest.fixture(scope="session")
def oracle_port():
    from oracle import port

    if not port.available():
        import subprocess

        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       stdout=subprocess.DEVNULL)
    return port


def mesh_residual(fwd, density, n):
    """sum (A_f - e^2 rho_f)^2 / e^2 with A_f half the cross product of the diagonals of
    face f = j + i n (vertices v = j + i (n+1)), otsolver_2dgrid.cpp:425-465."""
    P = np.asarray(fwd).reshape(n + 1, n + 1, 2)  # [i, j]
    p00, p10, p01, p11 = P[:-1, :-1], P[1:, :-1], P[:-1, 1:], P[1:, 1:]
    a = p11 - p00
    b = p01 - p10
    area = 0.5 * (a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0])  # [i, j]
    e2 = 1.0 / (n * n)
    r = area.ravel() - e2 * np.asarray(density)
    return float((r * r).sum() / e2)
