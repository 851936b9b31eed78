"""The C-ABI library loads on a machine without a GPU and exports every
entry point that include/*.h declares; calls that need a device fail with a
status, never a crash (there is no CPU fallback)."""
import ctypes as C
import glob
import os
import re

import numpy as np

from cosims_b200 import abi, engine, host
from tests.common import load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(cosims_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_entry_point_is_exported():
    L = engine.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert declared_functions(), "no declarations found"
    assert not missing, missing


def test_abi_version_and_layouts():
    L = engine.lib()
    assert L.cosims_abi_version() == abi.ABI_VERSION
    assert C.sizeof(abi.TrajOut) == 24 and C.sizeof(abi.TrajIn) == 40
    assert C.sizeof(abi.CcsSums) == 15 * 8


def test_device_calls_fail_cleanly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        return
    assert engine.device_count() == 0
    mol, par, _ = load("c0_t5")
    try:
        engine.Context(mol, par, abi.PLAIN_F64)
    except engine.CosimsError as e:
        assert e.status == abi.ERR_UNSUPPORTED
    else:
        raise AssertionError("context creation must fail without a device")


def test_invalid_arguments_are_rejected():
    L = engine.lib()
    mol, par, _ = load("c0_t5")
    view = mol.view()
    bad = abi.Params.from_buffer_copy(bytes(par))
    bad.force_type = 9
    h = C.c_void_p()
    assert L.cosims_ctx_create(C.byref(view), C.byref(bad), 0, 0, C.byref(h)) == abi.ERR_INVALID
    assert b"force_type" in L.cosims_last_error()
    assert L.cosims_ctx_create(C.byref(view), C.byref(par), 7, 0, C.byref(h)) == abi.ERR_INVALID


def test_trace_and_structure_entry_points_reject_bad_arguments(tmp_path):
    L = host._bind()          # the library with host and device argument types bound
    assert L.cosims_trace_list(None, None, None, 1, 10, None, None, None, None) == abi.ERR_INVALID
    k = C.c_int32()
    assert L.cosims_molecule_file_structures(None, C.byref(k)) == abi.ERR_INVALID
    assert L.cosims_molecule_file_structures(str(tmp_path / "none.mfj").encode(),
                                             C.byref(k)) == abi.ERR_IO
    from cosims_b200 import synth
    mp = synth.config0_molecule().write_mfj(str(tmp_path / "one.mfj"))
    assert host.count_structures(mp) == 1
    try:
        host.setup_from_files(mp, seed=1, structure=1)
    except engine.CosimsError as e:
        assert e.status == abi.ERR_INVALID
    else:
        raise AssertionError("a structure index past the file's sets must be rejected")
