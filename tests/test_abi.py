"""The C-ABI library loads and exports every entry point include/rodgpu.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import rodgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "rodgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?\**\s*\b(rg_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_lists_entry_points():
    names = declared_symbols()
    assert "rg_create" in names and "rg_step" in names and "rg_detect" in names
    assert set(names) == set(rodgpu.ABI_SYMBOLS)


def test_library_exports_all_declared_symbols():
    L = ctypes.CDLL(rodgpu.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_config_layout_and_defaults():
    L = rodgpu.lib()
    assert L.rg_abi_version() == 2
    c = rodgpu.default_config()
    # NscContactCfg / SoftContactCfg defaults (include/config/config.hpp:6-88)
    assert c.nsc_velocity_iters == 40 and abs(c.nsc_beta - 0.2) < 1e-15
    assert abs(c.soft_delta - 0.005) < 1e-15 and abs(c.soft_k_scaler - 1000.0) < 1e-12
    assert c.nsc_position_iters == 5 and c.nsc_position_psor_iters == 50
    assert abs(c.hm_friction_static - 0.5) < 1e-15 and c.hm_enable_rolling == 1
    assert L.rg_status_string(3) == b"capacity exceeded"


def test_create_rejects_bad_arguments():
    L = rodgpu.lib()
    h = ctypes.c_void_p()
    c = rodgpu.default_config(n_bodies=0)
    assert L.rg_create(ctypes.byref(c), ctypes.byref(h)) == 1  # RG_ERR_ARG before any device use
    c = rodgpu.default_config(n_bodies=10, dt=-1.0)
    assert L.rg_create(ctypes.byref(c), ctypes.byref(h)) == 1
