"""The C-ABI library loads without a GPU and exports every symbol include/*.h declares."""
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(cqg_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def _lib_path():
    from chronusq_public_b200 import _lib, build
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.LIB_PATH


def test_header_declares_entry_points():
    names = _declared()
    assert {"cqg_twoe_contract_direct", "cqg_form_pt", "cqg_set_basis", "cqg_create"} <= names


def test_library_exports_every_declared_symbol():
    path = _lib_path()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = _declared() - exported
    assert not missing, missing


def test_library_loads_and_answers_without_gpu():
    from chronusq_public_b200 import _lib
    _lib_path()
    L = _lib.load()
    assert L.cqg_version().startswith(b"cqgpu")
    assert L.cqg_status_string(7) == b"unsupported input"
    names = _lib.class_names()
    assert names[0] == "(ss|ss)" and names[-1] == "(ff|ff)" and len(names) == 55


def test_create_without_device_fails_cleanly():
    import ctypes
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from chronusq_public_b200 import _lib
    _lib_path()
    L = _lib.load()
    ctx = ctypes.c_void_p()
    assert L.cqg_create(ctypes.byref(ctx), 0) == 3
    assert not ctx.value
