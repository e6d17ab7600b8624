"""The C ABI: header, ctypes mirror and exported symbols (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from conftest import REPO
from swb200 import abi

HEADER = os.path.join(REPO, "include", "swb200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\**\s*\**\s*(sw_[a-z_0-9]+)\s*\(",
                                 src, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("sw_time_integration", "sw_create", "sw_set_state", "sw_run", "sw_get_state", "sw_destroy"):
        assert n in names


def test_library_loads_and_exports_every_declared_symbol():
    lib = abi.load_library()
    for n in declared_functions():
        assert hasattr(lib, n), f"{n} declared in include/swb200.h but not exported"
    assert lib.sw_abi_version() == abi.ABI_VERSION
    assert lib.sw_strerror(3) == b"NaNs detected"


@pytest.mark.parametrize("build,kind", [("parity", abi.SW_BUILD_PARITY), ("fast", abi.SW_BUILD_FAST)])
def test_both_builds_load_and_export_every_declared_symbol(build, kind):
    """libswb200.so (no FMA contraction) and libswb200_fast.so export the same
    ABI and say which build they are."""
    lib = abi.load_library(build=build)
    for n in declared_functions():
        assert hasattr(lib, n), f"{n} missing from the {build} build"
    assert lib.sw_build_kind() == kind


def test_python_mirror_covers_exports():
    assert set(declared_functions()) <= set(abi.EXPORTS)


@pytest.mark.parametrize("struct,cname", [(abi.SwConfig, "sw_config"), (abi.SwStatic, "sw_static"),
                                          (abi.SwStatus, "sw_status"), (abi.SwDiag, "sw_diag"),
                                          (abi.SwProfile, "sw_profile"),
                                          (abi.SwAdjointStats, "sw_adjoint_stats")])
def test_ctypes_layout_matches_c(struct, cname):
    """sizeof and every field offset of the ctypes mirror equal the C compiler's."""
    fields = [f[0] for f in struct._fields_]
    prog = ['#include <stdio.h>', '#include <stddef.h>', '#include "swb200.h"', 'int main(void){',
            f'printf("%zu\\n", sizeof({cname}));']
    prog += [f'printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
    prog += ['return 0;}']
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "t.c"), os.path.join(d, "t")
        open(src, "w").write("\n".join(prog))
        subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), src, "-o", exe], check=True)
        out = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == C.sizeof(struct)
    for f, off in zip(fields, out[1:]):
        assert getattr(struct, f).offset == off, f


def test_create_without_gpu_fails_cleanly():
    """No CUDA device: sw_create returns an error code instead of aborting."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from conftest import seeded_inputs  # noqa: F401
    from swb200 import Parameter, model_setup
    S = model_setup(Parameter(nx=16))
    lib = abi.load_library()
    cfg, st = abi.make_config(S), abi.StaticFields(S)
    ctx = C.c_void_p()
    rc = lib.sw_create(C.byref(cfg), st.ptr(), C.byref(ctx))
    assert rc == abi.SW_ERR_NODEVICE and not ctx.value
