"""The C-ABI library loads and exports every symbol include/sfincs_bmi.h declares."""
import ctypes
import os
import re

import pytest

from sfincs_b200 import bmi as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "sfincs_bmi.h")).read()
    funcs = re.findall(r"^SFG_API\s+[\w\*\s]+?\b(\w+)\(", text, flags=re.M)
    consts = re.findall(r"^extern SFG_API int (\w+);", text, flags=re.M)
    return funcs, consts


def test_header_declares_the_reference_bmi_surface():
    funcs, consts = _declared()
    for name in B.BMI_FUNCTIONS:  # sfincs_bmi.f90:14-30 + set_logical, get_last_bmi_error
        assert name in funcs, name
    assert set(B.BMI_CONSTANTS) == set(consts)


def test_library_exports_every_declared_symbol():
    L = B.lib()
    funcs, consts = _declared()
    for name in funcs + consts:
        assert hasattr(L, name), f"libsfincs_gpu.so does not export {name}"


def test_bmi_constants():
    L = B.lib()
    want = {"BMI_LENVARADDRESS": 64, "BMI_LENVARTYPE": 64, "BMI_LENGRIDTYPE": 64, "BMI_LENCOMPONENTNAME": 64,
            "BMI_LENVERSION": 256, "BMI_LENERRMESSAGE": 1024}
    for k, v in want.items():
        assert ctypes.c_int.in_dll(L, k).value == v


def test_var_types_without_a_model():
    bmi = B.BMI()
    assert bmi.get_var_type("zs") == "double"
    for n in ("z_xz", "z_yz", "zb", "subgrid_z_zmin", "qext"):
        assert bmi.get_var_type(n) == "float"
    assert bmi.get_var_rank("zs") == 1
    with pytest.raises(RuntimeError):
        bmi.get_var_type("nonsense")


def test_calls_before_initialize_fail_cleanly():
    bmi = B.BMI()
    with pytest.raises(RuntimeError, match="not initialized"):
        bmi.update()
    with pytest.raises(RuntimeError, match="not initialized"):
        bmi.get_current_time()
    assert bmi.finalize() == 0  # nothing to release


def test_initialize_error_is_reported_not_fatal(tmp_path):
    """A bad model directory returns an error code and a message (the reference
    stops the process instead)."""
    bmi = B.BMI()
    with pytest.raises(RuntimeError, match="sfincs.inp"):
        bmi.initialize(str(tmp_path))
