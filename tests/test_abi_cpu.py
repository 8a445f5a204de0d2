"""CPU-side checks of the boundary: the C-ABI library loads and exports every
symbol include/kira_gpu.h declares; host packing and the dispatcher follow the
reference semantics without a device."""
import ctypes
import os
import re

import numpy as np
import pytest

import pyoracle as O
from refgen import BASES, XorShift

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "kira_gpu.h")).read()
    return sorted(set(re.findall(r"\b(kira_(?:gpu|server)_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from kira_ls_aligner_b200 import _abi
    lib = ctypes.CDLL(_abi.LIB_PATH)
    syms = declared_symbols()
    assert syms, "no declarations found"
    for s in syms:
        assert hasattr(lib, s), f"{s} not exported"
    assert sorted(_abi.EXPORTS) == syms


def test_no_device_errors_are_reported(monkeypatch):
    from kira_ls_aligner_b200 import _abi, runtime
    if _abi.lib().kira_gpu_is_available():
        pytest.skip("a device is present")
    h = ctypes.c_void_p()
    assert _abi.lib().kira_gpu_init(0, ctypes.byref(h)) == 4  # KIRA_ERR_NO_DEVICE
    with pytest.raises(runtime.NoDevice):
        runtime.GpuContext(0)


def test_dispatcher_without_device_answers_none():
    # dispatcher.rs:33-43: a worker whose init failed answers every request with an
    # error, which dispatch() turns into None (the caller keeps its CPU path).
    from kira_ls_aligner_b200 import _abi
    from kira_ls_aligner_b200.cuda import CudaJob, dispatcher
    if _abi.lib().kira_gpu_is_available():
        pytest.skip("a device is present")
    assert dispatcher.dispatch([CudaJob(b"\x1b", 4, [b"\x1b\x00"] * 4, 4, 0)]) is None
    dispatcher.start()
    assert dispatcher.is_active()
    assert dispatcher.dispatch([]) == []
    assert dispatcher.dispatch([CudaJob(b"\x1b", 4, [b"\x1b\x00"] * 4, 4, 0)]) is None
    dispatcher.stop()
    assert not dispatcher.is_active()


def test_read_too_long_is_raised_before_device_work():
    from kira_ls_aligner_b200.cuda import CudaBackend, CudaJob, ReadTooLong
    be = CudaBackend.__new__(CudaBackend)  # no context needed: validation comes first
    with pytest.raises(ReadTooLong) as ei:
        be.run_batch([CudaJob(bytes(65), 260, [bytes(70)] * 4, 280, 5)])
    assert ei.value.len == 65 and ei.value.max == 64


def test_host_packing_matches_oracle():
    from kira_ls_aligner_b200.bitpacked import PackedDna
    rng = XorShift(0x9ACC)
    for _ in range(200):
        n = rng.next() % 90
        alpha = b"ACGTacgtN"
        s = bytes(alpha[rng.next() % (9 if rng.next() % 4 == 0 else 4)] for _ in range(n))
        p = PackedDna.pack(s)
        bits, ln, valid = O.pack(s)
        assert (p.bits, p.len, p.valid) == (bits, ln, valid)
        assert p.pre_shifted_window() == O.pre_shift(bits)


def test_synthetic_workloads_are_seeded():
    from kira_ls_aligner_b200 import synth
    a = synth.make_workload("t", 200, 20_000, cands=4, seed=7)
    b = synth.make_workload("t", 200, 20_000, cands=4, seed=7)
    assert np.array_equal(a.reads, b.reads) and np.array_equal(a.win_off, b.win_off)
    assert a.n_pairs == 800 and a.is_true.sum() == 200
    arena, offs = a.windows_arena()
    p = 17
    w = arena[int(offs[p]):int(offs[p]) + 250]
    assert np.array_equal(w, a.reference[int(a.win_off[p]):int(a.win_off[p]) + 250])
