"""CPU checks of the boundary: the C-ABI library loads without a GPU and exports every entry point the
public header declares, the Python binding's struct layouts match the header's, and the package refuses to
run anywhere but CUDA."""

import ctypes
import re
from pathlib import Path

import pytest

from plume_b200 import _native as N

HEADER = Path(__file__).resolve().parents[1] / "include" / "plume_b200.h"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(plume_[a-z0-9_]+)\s*\(", text)))


def test_the_library_exports_every_declared_entry_point():
    lib = N.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [name for name in names if not hasattr(lib, name)]
    assert missing == []
    assert set(names) == set(N.EXPORTED)


def test_every_binding_has_a_signature():
    for name in declared_functions():
        if name not in ("plume_last_error", "plume_launch_count"):
            assert name in N.SIGNATURES, name


def test_struct_layouts_match_the_header():
    # sizes follow from the header's field lists (all 4-byte fields; pointers 8 bytes)
    assert ctypes.sizeof(N.PlumeGridInfo) == 4 * (3 + 1 + 3 + 3 + 3 + 3 + 1)
    assert ctypes.sizeof(N.PlumeEmitter) == 4 * (1 + 3 + 1 + 3 + 1 + 1 + 1 + 1 + 1 + 3 + 1 + 1 + 1 + 1)
    assert ctypes.sizeof(N.PlumeViewParams) == 4 * (3 + 3 + 3 + 1 + 1 + 1 + 1 + 3)
    assert ctypes.sizeof(N.PlumeLookParams) == 4 * 6
    assert ctypes.sizeof(N.PlumeField) == 3 * 8


def test_abi_version_and_error_message_need_no_gpu():
    lib = N.lib()
    assert lib.plume_abi_version() == 1
    status = lib.plume_buoyancy(None, None, None, None, 0.0, 0.0, 0.0, 1.0, 0.0, None)
    assert status == -1
    assert b"null" in lib.plume_last_error()


def test_the_cpu_device_is_refused():
    from plume_b200.sim.device import DeviceError, init_device

    with pytest.raises(DeviceError):
        init_device("cpu")


def test_kernels_refuse_host_tensors():
    import torch

    with pytest.raises(RuntimeError, match="CUDA"):
        N.ptr(torch.zeros(4))


def test_newer_entry_points_reject_bad_arguments_without_a_gpu():
    """Argument checks come before any device work: a null array, a missing scratch or an aliased output is
    refused with status -1 and a message."""
    lib = N.lib()
    info = N.PlumeGridInfo()
    info.dims = type(info.dims)(8, 8, 8)
    shape = N.c_int3(8, 8, 8)
    toward = N.f3((0.0, 1.0, 0.0))
    assert lib.plume_march_light_volume(shape, None, 0, toward, 0.1, 1.0, None, None, None) == -1
    assert b"march_light_volume" in lib.plume_last_error()
    fake = ctypes.c_void_p(0x1000)
    assert lib.plume_march_light_volume(shape, fake, 0, toward, 0.1, 1.0, fake, None, None) == -1  # no bricks
    assert lib.plume_residual_f64(ctypes.byref(info), None, None, None, None, None, None, None) == -1
    assert b"residual_f64" in lib.plume_last_error()
    assert lib.plume_norm_scratch_doubles(ctypes.byref(info)) > 0
    level = (N.PlumeLevel * 1)()
    level[0].info = info
    level[0].q = level[0].rhs = level[0].residual = 0x1000  # q aliases the residual array
    assert lib.plume_multigrid_correct(level, 1, 2, ctypes.c_void_p(0x2000), None, None) == -1
    assert b"multigrid_correct" in lib.plume_last_error()
    assert lib.plume_confinement_adjoint(ctypes.byref(info), None, None, None, None, None, None, 0.3, 0.1, None,
                                         None, None) == -1
    assert b"confinement_adjoint" in lib.plume_last_error()
    assert lib.plume_confinement_adjoint_scratch_floats(ctypes.byref(info)) == 10 * 8 * 8 * 8
