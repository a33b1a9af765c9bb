"""The C-ABI library loads without a GPU and exports every entry point that
include/hit3d.h declares, with the signatures the host binding uses."""

import ctypes
import os
import re

from conftest import REPO


def _declared():
    src = open(os.path.join(REPO, "include", "hit3d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"\b(hit_[a-z0-9_]+)\s*\(", src))


def test_library_exports_every_declared_symbol(h3):
    from importlib import import_module
    nat = import_module("3dhit_b200._native")
    lib = nat.load()
    declared = _declared()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared but not exported"
    assert declared == set(nat.SIGNATURES), declared ^ set(nat.SIGNATURES)


def test_hit_params_layout_matches_header():
    from importlib import import_module
    nat = import_module("3dhit_b200._native")
    # double, int, unsigned, then six doubles: 8 + 4 + 4 + 6*8
    assert ctypes.sizeof(nat.HitParams) == 64
    assert nat.HitParams.A.offset == 16


def test_error_string_without_gpu():
    from importlib import import_module
    nat = import_module("3dhit_b200._native")
    lib = nat.load()
    h = ctypes.c_void_p()
    rc = lib.hit_plan_create(12, 16, 16, 6.28, 6.28, 6.28, 0, ctypes.byref(h))
    assert rc == nat.HIT_E_UNSUPPORTED
    assert b"powers of two" in lib.hit_last_error_string()
