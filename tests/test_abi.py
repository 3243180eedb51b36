"""C-ABI library checks that need no GPU: it loads, exports every entry
point include/simox_gpu.h declares, and its host-only helpers agree with the
oracle."""
import os
import re

import numpy as np

from simox_b200 import _abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "simox_gpu.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(simox_[a-z0-9_]+)\s*\(", txt)))


def test_header_declarations_listed():
    assert declared_symbols() == sorted(_abi.EXPORTED)


def test_library_exports_every_symbol(simox_lib):
    for name in declared_symbols():
        assert hasattr(simox_lib, name), name


def test_status_strings_match(simox_lib):
    for code in range(0, -21, -1):
        assert simox_lib.simox_status_string(code).decode() == _abi.status_text(code)


def test_default_potential_equals_oracle(simox_lib):
    from simox_b200 import api
    from oracle import oracle as O
    assert _abi.potential_to_bytes(api.default_potential()) == _abi.potential_to_bytes(O.potential_setup())


def test_create_without_gpu_reports_status(simox_lib):
    """No GPU here: create must return a status, not crash or fall back."""
    import ctypes as C
    from simox_b200.api import _vp
    s = _abi.Setup()
    s.n_atoms = 2
    s.box[:] = [30.0, 30.0, 30.0]
    s.fft[:] = [16, 16, 16]
    s.pme_order = 4
    s.rcut = 10.0
    ctx = _vp()
    st = simox_lib.simox_create(C.byref(s), None, C.byref(ctx))
    try:
        import torch
        has = torch.cuda.is_available()
    except Exception:
        has = False
    if not has:
        assert st == _abi.SIMOX_E_NO_DEVICE
    else:
        assert st == 0
        simox_lib.simox_destroy(ctx)


def test_adjoint_eval_many_argument_checks(simox_lib):
    """Host-side checks of simox_adjoint_eval_many (no context is touched):
    nothing to do for m = 0, E_ARG for a NULL or repeated context."""
    import ctypes as C
    from simox_b200.api import _vp
    assert simox_lib.simox_adjoint_eval_many(None, 0, None, None, None, None, None, 0) == 0
    assert simox_lib.simox_adjoint_eval_many(None, 2, None, None, None, None, None, 0) == _abi.SIMOX_E_ARG
    fake = _vp(0x1000)   # never dereferenced: the duplicate check runs first
    arr = (_vp * 2)(fake, fake)
    assert simox_lib.simox_adjoint_eval_many(arr, 2, None, None, None, None, None, 0) == _abi.SIMOX_E_ARG
    arr = (_vp * 2)(fake, None)
    assert simox_lib.simox_adjoint_eval_many(arr, 2, None, None, None, None, None, 0) == _abi.SIMOX_E_ARG


def test_batch_entry_points_argument_checks(simox_lib):
    """Host-side checks of the batch entry points (no context or device is
    touched): E_ARG for no members, a NULL member, a NULL batch, an unknown
    mode."""
    import ctypes as C
    from simox_b200.api import Batch, _vp
    out = _vp()
    assert simox_lib.simox_batch_create(0, None, C.byref(out)) == _abi.SIMOX_E_ARG
    assert simox_lib.simox_batch_create(1, (_vp * 1)(None), C.byref(out)) == _abi.SIMOX_E_ARG
    assert simox_lib.simox_batch_destroy(None) == _abi.SIMOX_E_ARG
    assert simox_lib.simox_batch_md_run(None, None, 1, 1, None) == _abi.SIMOX_E_ARG
    assert simox_lib.simox_batch_set_mode(None, Batch.MODES["per_pass"]) == _abi.SIMOX_E_ARG
    m = C.c_int(-1)
    assert simox_lib.simox_batch_get_mode(None, C.byref(m)) == _abi.SIMOX_E_ARG
    n = C.c_longlong(0)
    assert simox_lib.simox_batch_launch_count(None, C.byref(n)) == _abi.SIMOX_E_ARG
    assert sorted(Batch.MODES.values()) == [0, 1]


def test_batch_mode_constants_match_header():
    from simox_b200.api import Batch
    txt = open(HEADER).read()
    vals = dict(re.findall(r"\b(SIMOX_BATCH_PER_\w+)\s*=\s*(\d+)", txt))
    assert {k: int(v) for k, v in vals.items()} == {"SIMOX_BATCH_PER_PASS": Batch.MODES["per_pass"],
                                                     "SIMOX_BATCH_PER_SYSTEM": Batch.MODES["per_system"]}
