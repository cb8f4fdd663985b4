"""Request serving: continuous batching of whole UQ solves on one GPU.

Thin binding of the library's request server (uqc_server_* in include/uqc.h).
Each request is a UQCreator TOML configuration run to its tEnd. Requests are
admitted, first fit in submission order, while their device memory fits the
budget; each admitted request keeps its moments and duals on the device, on
its own CUDA stream, and every progress() call advances each running request
by a slice of time steps, so the kernels of different requests overlap.

    srv = Server(budget_bytes=40 << 30, max_active=8, steps_per_slice=4)
    rid = srv.submit(toml_text)
    srv.drain()                          # or call srv.progress() from your loop
    res = srv.result(rid)                # dict with latency and mean/variance
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib as L
from ._lib import UqcError, RequestInfo, ptr

__all__ = ["Server", "latency_percentiles"]


class Server:
    def __init__(self, budget_bytes: int, max_active: int = 8, steps_per_slice: int = 4, policy: int | None = None,
                 max_stepping: int | None = None):
        self.lib = L.lib()
        h = C.c_void_p()
        rc = self.lib.uqc_server_create(int(budget_bytes), int(max_active), int(steps_per_slice), C.byref(h))
        if rc != 0:
            raise UqcError(rc, "server create")
        self.h = h
        if policy is not None:
            self.set_option("policy", policy)
        if max_stepping is not None:
            self.set_option("max_stepping", max_stepping)

    def set_option(self, key: str, value: float):
        """Scheduling options of uqc_server_set_option: "policy" (0 round robin,
        1 shortest remaining time first), "max_stepping" (0: no limit), "aging"."""
        self._check(self.lib.uqc_server_set_option(self.h, key.encode(), float(value)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.uqc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise UqcError(rc, self.lib.uqc_server_last_error(self.h).decode())

    def submit(self, toml_text: str, precision: int = L.FP64) -> int:
        rid = C.c_longlong()
        self._check(self.lib.uqc_server_submit(self.h, toml_text.encode(), int(precision), C.byref(rid)))
        return rid.value

    def progress(self):
        q, r, d = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.uqc_server_progress(self.h, C.byref(q), C.byref(r), C.byref(d)))
        return q.value, r.value, d.value

    def info(self, rid: int) -> dict:
        inf = RequestInfo()
        self._check(self.lib.uqc_server_request(self.h, int(rid), C.byref(inf), None))
        return inf.as_dict()

    def result(self, rid: int, mean_var: bool = True) -> dict:
        inf = RequestInfo()
        self._check(self.lib.uqc_server_request(self.h, int(rid), C.byref(inf), None))
        d = inf.as_dict()
        if mean_var and d["state"] == "done":
            mv = np.zeros((inf.n_cells, 2 * inf.n_states))
            self._check(self.lib.uqc_server_request(self.h, int(rid), C.byref(inf), ptr(mv)))
            d["mean_var"] = mv
        d["latency_ms"] = d["done_ms"] - d["submit_ms"] if d["state"] in ("done", "failed") else None
        d["queue_ms"] = d["admit_ms"] - d["submit_ms"] if d["state"] in ("running", "done", "failed") else None
        d["service_ms"] = d["done_ms"] - d["admit_ms"] if d["state"] in ("done", "failed") else None
        d["error"] = self.lib.uqc_server_request_error(self.h, int(rid)).decode()
        return d

    def release(self, rid: int):
        self._check(self.lib.uqc_server_release(self.h, int(rid)))

    def drain(self, poll_s: float = 0.0):
        """Runs scheduling passes until no request is queued or running."""
        while True:
            q, r, _ = self.progress()
            if q == 0 and r == 0:
                return
            if poll_s:
                time.sleep(poll_s)


def latency_percentiles(latencies_ms, qs=(50, 99)) -> dict:
    a = np.asarray(latencies_ms, dtype=float)
    return {f"p{q}_ms": float(np.percentile(a, q)) for q in qs} if a.size else {f"p{q}_ms": None for q in qs}
