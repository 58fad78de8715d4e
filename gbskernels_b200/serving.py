"""Continuous-batching server for chain-rule sampler queries (libgbs_b200 gbs_server_*).

    with Server(slots=2) as srv:
        st = srv.add_state(A, gamma)                      # resident on the device
        t = srv.submit_state("lhaf", st, idx, "auto", use_gamma=True)
        value, diag = srv.result(t)                       # blocks (bounded) until done

The scheduler runs in the library (a C++ thread): requests that arrive while
batches are on the GPU are admitted into the next free slot, up to a workspace
budget per batch, and up to `slots` batches overlap on the device.  A value is
independent of the batch it ran in.

Two slots by default: on the chain-rule stream (2000 requests, one B200) two, three,
four and six slots serve the same throughput below capacity, and two give the
lowest p99 there (104-117 ms at 0.75x the offline rate, against 128-141 ms with
four) and the highest saturated throughput (0.89 of offline against 0.88); eight
lose throughput.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from .workloads import serving_stream

_FN = {"perm": 0, "haf": 1, "lhaf": 2, "tor": 3}
_TIER = {"fp64": 0, "dd": 1, "auto": 2, "certified": 3}
_TIER_NAME = {0: "fp64", 1: "dd", 3: "certified-fp64"}

_vp = ctypes.c_void_p
_SIGS = {
    "gbs_server_open": ([ctypes.c_int, ctypes.c_longlong, ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
    "gbs_server_close": ([_vp], ctypes.c_int),
    "gbs_server_add_state": ([_vp, _lib._dp, _lib._dp, ctypes.c_int, _lib._ip], ctypes.c_int),
    "gbs_server_submit": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _lib._dp,
                           ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "gbs_server_submit_state": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _lib._ip,
                                 ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "gbs_server_poll": ([_vp, ctypes.c_longlong, _lib._ip, _lib._dp, _lib._dp, _lib._ip, _lib._ip, _lib._dp],
                        ctypes.c_int),
    "gbs_server_drain": ([_vp, ctypes.c_double], ctypes.c_int),
    "gbs_server_stats": ([_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                          ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
}
_lib.SIGNATURES.update(_SIGS)


def _l():
    lib = _lib.load()
    for name, (a, r) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = a, r
    return lib


class Server:
    """Serving session: `slots` concurrent batches, `budget_bytes` per batch."""

    def __init__(self, slots: int = 2, budget_bytes: int = 256 << 20, max_batch: int = 4096):
        self._lib = _l()
        h = _vp()
        _lib.check(self._lib.gbs_server_open(slots, budget_bytes, max_batch, ctypes.byref(h)), "gbs_server_open")
        self._h = h
        self._keep: list = []

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc) -> bool:
        self.close()
        return False

    def close(self) -> None:
        if self._h is not None:
            self._lib.gbs_server_close(self._h)
            self._h = None

    def add_state(self, A, gamma=None) -> int:
        A = np.ascontiguousarray(np.asarray(A, dtype=np.complex128))
        if A.ndim != 2 or A.shape[0] != A.shape[1]:
            raise ValueError("state must be a square matrix")
        g = None if gamma is None else np.ascontiguousarray(np.asarray(gamma, dtype=np.complex128))
        sid = np.zeros(1, dtype=np.int32)
        _lib.check(self._lib.gbs_server_add_state(self._h, _lib.dptr(A.view(np.float64)),
                                                  None if g is None else _lib.dptr(g.view(np.float64)),
                                                  A.shape[0], _lib.iptr(sid)), "gbs_server_add_state")
        return int(sid[0])

    def submit(self, func: str, mat, precision: str = "fp64") -> int:
        m = np.ascontiguousarray(np.asarray(mat, dtype=np.complex128))
        t = ctypes.c_longlong()
        _lib.check(self._lib.gbs_server_submit(self._h, _FN[func], _TIER[precision], m.shape[0],
                                               _lib.dptr(m.view(np.float64)), ctypes.byref(t)),
                   "gbs_server_submit")
        return t.value

    def submit_state(self, func: str, state: int, idx, precision: str = "fp64", use_gamma: bool = False) -> int:
        ix = np.ascontiguousarray(np.asarray(idx, dtype=np.int32))
        t = ctypes.c_longlong()
        _lib.check(self._lib.gbs_server_submit_state(self._h, _FN[func], _TIER[precision], state, ix.size,
                                                     _lib.iptr(ix), int(use_gamma), ctypes.byref(t)),
                   "gbs_server_submit_state")
        return t.value

    def poll(self, ticket: int):
        """(done, value, info) without blocking; info has tier, aux, status, latency_s."""
        done = np.zeros(1, dtype=np.int32)
        out = np.zeros(2)
        aux = np.zeros(1)
        st = np.zeros(1, dtype=np.int32)
        tier = np.zeros(1, dtype=np.int32)
        lat = np.zeros(1)
        _lib.check(self._lib.gbs_server_poll(self._h, ticket, _lib.iptr(done), _lib.dptr(out), _lib.dptr(aux),
                                             _lib.iptr(st), _lib.iptr(tier), _lib.dptr(lat)), "gbs_server_poll")
        if not done[0]:
            return False, None, None
        info = {"tier": _TIER_NAME.get(int(tier[0]), str(int(tier[0]))), "aux": float(aux[0]),
                "status": int(st[0]), "latency_s": float(lat[0])}
        return True, complex(out[0], out[1]), info

    def result(self, ticket: int, timeout_s: float = 120.0):
        t0 = time.perf_counter()
        while True:
            done, v, info = self.poll(ticket)
            if done:
                return v, info
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError(f"request {ticket} not done after {timeout_s} s")
            time.sleep(50e-6)

    def drain(self, timeout_s: float = 600.0) -> None:
        _lib.check(self._lib.gbs_server_drain(self._h, timeout_s), "gbs_server_drain")

    def stats(self) -> dict:
        c, b, p = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        _lib.check(self._lib.gbs_server_stats(self._h, ctypes.byref(c), ctypes.byref(b), ctypes.byref(p)),
                   "gbs_server_stats")
        return {"completed": c.value, "batches": b.value, "pending": p.value}


def _pct(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def offline_rate(n_req: int = 2000, seed: int = 5):
    """Requests/s of the serving stream's requests evaluated offline with the same
    tier semantics as the server, and their values: ONE persistent mixed launch of
    host-gathered matrices (auto as fp64 + indicator), then one double-double launch
    of the auto requests whose indicator reaches 1e8 -- the same work and the same
    results the server produces.  The rate is the median of three passes after a
    warm-up."""
    from . import Workspace, _AUTO_KAPPA_MAX

    reqs0 = serving_stream(n_req, 1.0, seed=seed)
    tier_of = {"fp64": "fp64", "auto": "kappa", "certified": "certified"}
    funcs = [r[1] for r in reqs0]
    mats = [r[3] for r in reqs0]
    tiers = [tier_of[r[2]] for r in reqs0]
    times = []
    with Workspace() as ws:
        ws.evaluate(funcs[:64], mats[:64], tiers[:64])  # warm-up
        # the median of three passes: one pass takes a fraction of a second, so a
        # single one is at the mercy of whatever ran just before (host or GPU)
        for _ in range(3):
            t0 = time.perf_counter()
            out, aux, st = ws.evaluate_full(funcs, mats, tiers)
            redo = [i for i, r in enumerate(reqs0)
                    if r[2] == "auto" and st[i] == 0 and not aux[i] / max(abs(out[i]), 1e-300) < _AUTO_KAPPA_MAX]
            if redo:
                out[redo] = ws.evaluate([funcs[i] for i in redo], [mats[i] for i in redo], ["dd"] * len(redo))
            times.append(time.perf_counter() - t0)
    return n_req / sorted(times)[1], out


def serve_stream(rate: float | None = None, n_req: int = 2000, seed: int = 5, rate_frac: float = 0.7,
                 slots: int = 2, budget_bytes: int = 64 << 20, offline=None, resident: bool = True):
    """Replay a Poisson stream of chain-rule sampler queries (haf / lhaf / tor,
    matrix side 6..30, growing prefixes per chain, fp64 70% / auto 20% / certified
    10%; workloads.serving_chains) against a Server.

    resident=True (default): the two states (the GBS kernel A with its loop weights,
    the threshold matrix O_x) are uploaded once with add_state and every query is
    submitted as (state, index list) -- its submatrix is gathered on the device.
    resident=False submits the host-gathered matrices instead.

    The offline rate of the same requests (one persistent mixed batch of host
    matrices) is measured first, unless `offline` passes the (rate, values) pair of
    `offline_rate` for the same n_req and seed; the stream is offered at `rate`
    requests/s, or at rate_frac x the offline rate when `rate` is None.  Returns
    throughput, p50/p99 latency, the offline rate, the ratio throughput / offline
    rate, whether every value (auto reruns included) equals the offline batch's bit
    for bit, and the rate at which the submitting thread actually handed the requests
    over (a Python submit costs tens of microseconds, so the highest offered rates
    are reached only in bursts)."""
    from .workloads import gather_query, serving_chains

    states, queries = serving_chains(n_req, 1.0, seed=seed)
    off_rate, ws_out = offline if offline is not None else offline_rate(n_req, seed)
    if rate is None:
        rate = rate_frac * off_rate
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, size=n_req)
    arrivals = np.cumsum(gaps)
    lat = []
    with Server(slots=slots, budget_bytes=budget_bytes) as srv:
        sid = {}
        if resident:
            sid["A"] = srv.add_state(states["A"], states["gamma"])
            sid["O"] = srv.add_state(states["O"])

        def submit(q):
            _, func, prec, key, idx, ug = q
            if resident:
                return srv.submit_state(func, sid[key], idx, prec, use_gamma=ug)
            return srv.submit(func, gather_query(states, key, idx, ug), prec)

        for q in queries[:8]:  # warm the slots
            srv.result(submit(q))
        tickets = []
        t_start = time.perf_counter()
        for i, q in enumerate(queries):
            while time.perf_counter() - t_start < arrivals[i]:
                pass
            tickets.append(submit(q))
        t_submitted = time.perf_counter()
        vals = []
        for t in tickets:
            v, info = srv.result(t)
            lat.append(info["latency_s"])
            vals.append(v)
        t_end = time.perf_counter()
        stats = srv.stats()
    thr = n_req / (t_end - t_start)
    same = bool(all(vals[i] == ws_out[i] or (np.isnan(vals[i]) and np.isnan(ws_out[i])) for i in range(n_req)))
    return {"offered_rate": rate, "submitted_rate": n_req / (t_submitted - t_start),
            "requests": n_req, "throughput": thr, "unit": "requests/s",
            "p50_ms": 1e3 * _pct(lat, 50), "p99_ms": 1e3 * _pct(lat, 99), "max_ms": 1e3 * max(lat),
            "offline_rate": off_rate, "throughput_vs_offline": thr / off_rate,
            "batches": stats["batches"], "slots": slots,
            "path": "resident states, device gather (submit_state)" if resident else "host matrices (submit)",
            "stream": "chain-rule queries: growing prefixes, 8 samplers side by side",
            "values_equal_to_offline_batch": same}
