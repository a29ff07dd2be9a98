"""Shared test setup.

Markers: tests that need a GPU are marked ``gpu``; everything else runs on
CPU (the CPU suite covers the oracle against the golden fixtures, the C-ABI
symbol table and the host-side argument checks).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "reference_small.npz"))


@pytest.fixture(scope="session")
def oracle():
    import oracle as O  # noqa: the restatement oracle (test infrastructure)
    O.lib()
    return O


def ref_available():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libflame_ref.so"))


@pytest.fixture(scope="session")
def flame():
    """The product binding; builds the library in-tree if it is missing."""
    lib_path = os.path.join(ROOT, "libflame_b200", "libflame_b200.so")
    if not os.path.exists(lib_path):
        subprocess.run([sys.executable, "-m", "libflame_b200.build"], cwd=ROOT, check=True)
    import libflame_b200 as F
    F.lib()
    return F


@pytest.fixture(scope="session")
def cuda(flame):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    flame.init()
    return torch


def seeded(seed):
    return np.random.default_rng(seed)


def spd(rng, n):
    G = rng.standard_normal((n, n))
    return G @ G.T / n + np.eye(n)


def to_dev(torch, a, dtype=None):
    """NumPy (any order) -> column-major CUDA tensor."""
    import torch as T
    t = T.from_numpy(np.asfortranarray(a))
    if dtype is not None:
        t = t.to(dtype)
    # column-major: allocate transposed storage
    d = T.empty((t.shape[1], t.shape[0]) if t.dim() == 2 else t.shape, dtype=t.dtype, device="cuda")
    if t.dim() == 2:
        d = d.t()
    d.copy_(t)
    return d


def to_host(t):
    return np.asfortranarray(t.cpu().numpy())


def rel_fro(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)
