"""The C ABI library loads without a GPU, exports every symbol include/uqc.h
declares, and its host-side parts (configuration, footprint, admission
limits) work on the CPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

import uqcreator_b200._lib as L
from uqcreator_b200 import Solver, UqcError, workloads as W
from uqcreator_b200.serve import Server

HEADER = Path(__file__).resolve().parents[1] / "include" / "uqc.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(uqc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = L.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(L.EXPORTS) == names


def test_config_errors_are_reported_not_fatal():
    with pytest.raises(UqcError) as e:
        Solver(W.burgers1d().replace('closure = "BoundedBarrier"', 'closure = "NoSuchClosure"'))
    assert e.value.code == -2


def test_device_footprint_is_host_side_and_grows_with_cells():
    a = Solver(W.burgers1d(ncells=200)).device_bytes()
    b = Solver(W.burgers1d(ncells=2000)).device_bytes()
    assert 0 < a < b


def test_server_rejects_request_beyond_budget_without_gpu_work():
    toml = W.burgers1d(ncells=2000)
    need = Solver(toml).device_bytes()
    srv = Server(budget_bytes=need // 2, max_active=2, steps_per_slice=1)
    rid = srv.submit(toml)
    q, r, d = srv.progress()
    assert (q, r, d) == (0, 0, 1)
    info = srv.result(rid)
    assert info["state"] == "failed" and info["status"] == -7
    srv.release(rid)
    with pytest.raises(UqcError):
        srv.info(rid)
