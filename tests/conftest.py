import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "shallowwaters.jl_b200"), os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libswb200.so")


def seeded_inputs(S, seed=1, sigma=0.01, block=10):
    """Seeded η noise N(0, σ²) and a ±1 tracer checkerboard of block×block cells.

    Generated in Float64 with numpy's PCG64 and rounded once to Tprog by
    initial_conditions, so oracle and GPU receive identical bits.
    """
    G = S.grid
    rng = np.random.default_rng(seed)
    eta = rng.normal(0.0, sigma, (G.ny, G.nx))
    i = np.arange(G.nx)[None, :]
    j = np.arange(G.ny)[:, None]
    sst = np.where(((i // block) + (j // block)) % 2 == 0, 1.0, -1.0)
    return {"η0": eta, "sst0": sst}


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view({2: np.uint16, 4: np.uint32, 8: np.uint64}[a.dtype.itemsize])


def assert_bitwise(a, b, name=""):
    """Bit-identical arrays, except that any NaN equals any NaN."""
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, f"{name}: shape {a.shape} != {b.shape}"
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), f"{name}: NaN positions differ"
    diff = (bits(a) != bits(b)) & ~na
    if diff.any():
        idx = np.argwhere(diff)[:5]
        raise AssertionError(f"{name}: {int(diff.sum())} elements differ, first at {idx.tolist()}: "
                             f"{a[tuple(idx[0])]!r} vs {b[tuple(idx[0])]!r}")
