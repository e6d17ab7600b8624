"""sw_diagnostics_noalloc: the diagnostics for callers that cannot allocate.

A host that lets its own pool allocator own the GPU's memory (CUDA.jl, a
PyTorch caching allocator, a fixed arena), or that must not stall a running
time loop with the device-wide synchronisation of cudaMalloc/cudaFree, keeps
the fields in its own device buffers and asks for mass, energy, maximum speed
and NaN count without the library allocating anything.  The entry point
reduces into a fixed scratch array built into the library.  Here the test
itself places the fields in device memory (with torch) and checks the result
against sw_diagnostics on a context holding the same state, on two calls in a
row: the second on a smaller domain with planted NaNs, so partial sums left
in the shared scratch by the first call would show up if they were ever read.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import seeded_inputs
from swb200 import Model, Parameter, abi, initial_conditions, model_setup
from swb200.initial_conditions import PrognosticVars

pytestmark = pytest.mark.gpu

RTOL = 1e-12   # the tolerance of the FP64 diagnostics test in test_gpu_parity.py


def _noalloc(lib, S, state):
    """Copy the host-layout state and H to device buffers, then call the entry point."""
    import torch
    H = abi.StaticFields(S).arrays["H"]
    bufs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (*state, H)]
    torch.cuda.synchronize()
    cfg = abi.make_config(S)
    out = abi.SwDiag()
    rc = lib.sw_diagnostics_noalloc(C.byref(cfg), *[b.data_ptr() for b in bufs], None, C.byref(out))
    return rc, out


def _same(d, ref):
    np.testing.assert_allclose(d.mass, ref.mass, rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(d.energy, ref.energy, rtol=RTOL)
    assert d.max_speed == ref.max_speed
    assert d.nan_count == ref.nan_count


def _model(kw, seed, nsteps):
    P = Parameter(**kw)
    S = model_setup(P)
    m = Model(S)
    m.set_state(initial_conditions(P.Tprog, S, **seeded_inputs(S, seed)))
    m.run(nsteps)
    return S, m


TYPES = {"f32": dict(T=np.float32), "f64": dict(T=np.float64), "f32_f64": dict(T=np.float32, Tprog=np.float64)}


@pytest.mark.parametrize("types", list(TYPES))
def test_noalloc_diagnostics_match_sw_diagnostics_on_two_calls(types):
    """Each (T, Tprog) pair the entry point takes: 4- and 8-byte state and
    depth, and the mixed pair whose depth and state have different sizes."""
    lib = abi.load_library()
    tk = TYPES[types]

    # call 1: 200x100 periodic channel, three partial blocks of scratch
    S1, m1 = _model(dict(nx=200, Ndays=0.2, Uadv=1000, **tk), seed=11, nsteps=15)
    ref1 = m1.diagnostics()
    rc, d1 = _noalloc(lib, S1, m1.get_state())
    assert rc == abi.SW_OK
    _same(d1, ref1)
    assert np.isfinite(d1.energy) and d1.nan_count == 0
    m1.close()

    # call 2: 40x20 nonperiodic seamount (one block) with two NaNs planted in
    # the tracer, read back through the library so both paths see the same state
    S2, m2 = _model(dict(nx=40, Ndays=0.2, Uadv=1000, bc="nonperiodic", topography="seamount", **tk), seed=12,
                    nsteps=9)
    st = m2.get_state()
    sst = st.sst.copy()
    sst[5, 17] = np.nan
    sst[11, 20] = np.nan
    m2.set_state(PrognosticVars(st.u, st.v, st.η, sst))
    ref2 = m2.diagnostics()
    rc, d2 = _noalloc(lib, S2, m2.get_state())
    assert rc == abi.SW_OK
    _same(d2, ref2)
    assert d2.nan_count == 2
    m2.close()


def test_noalloc_rejects_domains_beyond_the_scratch_limit():
    lib = abi.load_library()
    S = model_setup(Parameter(nx=40))
    cfg = abi.make_config(S)
    cfg.nx, cfg.ny = 8192, 4096          # 33.5 M cells > 16,777,216
    out = abi.SwDiag()
    rc = lib.sw_diagnostics_noalloc(C.byref(cfg), None, None, None, None, None, None, C.byref(out))
    assert rc == abi.SW_ERR_ARG
