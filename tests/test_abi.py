"""The C-ABI library loads here (no GPU needed) and exports every entry point
declared in include/pibm.h; the ctypes mirror matches the header's structs."""
import ctypes as C
import os
import re

import pytest

from pureibm_ps2d_fd1d_b200 import abi, build, LIB_PATH
import oracle_ctypes as oc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "pibm.h")).read()
    return sorted(set(re.findall(r"\b(pibm_[a-z0-9_]+)\s*\(", text)))


def test_header_lists_all_entry_points():
    names = header_functions()
    assert set(names) == set(abi.EXPORTED)


def test_library_exports_every_header_symbol():
    build.build()
    lib = C.CDLL(LIB_PATH)
    for name in header_functions():
        assert hasattr(lib, name), name


@pytest.mark.parametrize("which,cls", [(0, abi.pibm_params), (1, abi.pibm_particles), (2, abi.pibm_state_view),
                                       (3, abi.pibm_step_report), (4, abi.pibm_info)])
def test_struct_sizes_match_header(which, cls):
    assert oc.lib().orc_sizeof(which) == C.sizeof(cls)


def test_kernel_slot_names_match_header():
    lib = abi.bind(C.CDLL(LIB_PATH))
    names = [lib.pibm_kernel_name(k).decode() for k in range(abi.PIBM_NKERNEL)]
    assert names == abi.KERNEL_NAMES
    assert lib.pibm_kernel_name(abi.PIBM_NKERNEL) is None
    text = open(os.path.join(ROOT, "include", "pibm.h")).read()
    assert int(re.search(r"#define PIBM_NKERNEL\s+(\d+)", text).group(1)) == abi.PIBM_NKERNEL
