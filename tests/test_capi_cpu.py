"""CPU-only checks of the C-ABI library: it builds, loads without a GPU and exports every
entry point that include/hmc.h declares. No compute call is made here."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "hmc.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hmc_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    from hoomd_rs_b200 import build

    return build.build()


def test_header_declares_the_boundary():
    fns = declared_functions()
    for name in ("hmc_context_create", "hmc_system_create", "hmc_sweep", "hmc_tune", "hmc_overlap_check",
                 "hmc_eval_moves", "hmc_get_state", "hmc_set_state", "hmc_last_error_message"):
        assert name in fns


def test_library_exports_every_declared_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\b[TW]\s+(hmc_\w+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing


def test_library_loads_without_gpu_and_binds(lib_path):
    import hoomd_rs_b200 as h

    lib = h.load_library(lib_path)
    assert set(h.SIGNATURES) == set(declared_functions())
    assert lib.hmc_abi_version() == 3
    assert lib.hmc_status_string(h.RANGE_TOO_LARGE).decode().startswith("interaction range")


def test_library_targets_sm100a(lib_path):
    # the build log holds ptxas's report for every kernel it compiled: all of them for sm_100a
    log = open(lib_path + ".build.log").read()
    assert "arch=compute_100a,code=sm_100a" in log.splitlines()[0]
    targets = set(re.findall(r"ptxas info\s*: Compiling entry function '\w+' for '(\w+)'", log))
    assert targets == {"sm_100a"}, targets
