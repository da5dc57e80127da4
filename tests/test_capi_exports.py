"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
LIBRARY = os.path.join(ROOT, "powder-play_b200", "libmpm_b200.so")


def declared_functions():
    names = set()
    for header in os.listdir(INCLUDE):
        if not header.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, header)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for match in re.finditer(r"^\s*(?:const\s+)?[\w]+\s*\*?\s*(mpm\w*)\s*\(", text, flags=re.M):
            names.add(match.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def library():
    if not os.path.exists(LIBRARY):
        import importlib.util
        spec = importlib.util.spec_from_file_location("mpm_build", os.path.join(ROOT, "powder-play_b200", "build.py"))
        module = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(module)
        module.build()
    return ctypes.CDLL(LIBRARY)


def test_header_declares_the_solver_interface():
    names = declared_functions()
    for required in ("mpm_create", "mpm_step_batch", "mpm_read_compact", "mpm_read_particles", "mpm_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol(library):
    for name in declared_functions():
        assert hasattr(library, name), f"{name} is declared in include/ but not exported"


def test_exports_are_plain_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", LIBRARY], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for name in declared_functions():
        assert name in exported


def test_host_binding_declares_the_same_symbols():
    from mpm_b200 import _lib
    assert set(_lib.EXPORTED_SYMBOLS) <= set(declared_functions())
