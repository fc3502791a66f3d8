"""Serving front end: continuous batching of rod-assembly simulations
(``eb_server_*`` in include/elastica_b200.h).

    srv = Server(precision="mixed", hbm_budget_bytes=40e9)
    rid = srv.submit(rods, dt=1e-6, n_steps=10_000, gravity=(0, 0, -9.81), clamp=True, damper=(0.1, 0.1))
    while srv.tick():          # one launch per tick over every admitted request
        for done in srv.poll():
            tips = srv.result(done["request_id"], 0, "Position")[:, -1]
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Sequence

import numpy as np

from . import _lib as L
from .simulator import CosseratRodWithoutDamping, CosseratRod, StraightRod

_PRECISION = {"fp64": L.EB_PRECISION_FP64, "mixed": L.EB_PRECISION_MIXED}
_NAMES = {L.EB_PRECISION_FP64: "fp64", L.EB_PRECISION_MIXED: "mixed"}


class Server:
    def __init__(self, device: int = 0, precision: str = "mixed", steps_per_launch: int = 128,
                 hbm_budget_bytes: float = 40e9, energy_tolerance: float = 1e-3, force_fallback: bool = False):
        cfg = L.EbServerConfig(device, _PRECISION[precision], int(steps_per_launch),
                               L.EB_SERVER_FORCE_FALLBACK if force_fallback else 0, float(hbm_budget_bytes),
                               float(energy_tolerance))
        h = ctypes.c_void_p()
        L.call("eb_server_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        self._rods = {}

    def close(self) -> None:
        if self._h:
            L.load().eb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, rods: Sequence[StraightRod], dt: float, n_steps: int, gravity=None, clamp: bool = False,
               damper=None, velocities: Iterable[np.ndarray] | None = None, model=CosseratRodWithoutDamping) -> int:
        m = L.EB_ROD_DAMPED if model is CosseratRod else L.EB_ROD_UNDAMPED
        arr = (L.EbStraightRod * len(rods))(*[r.to_c(m) for r in rods])
        req = L.EbRequest()
        req.rods = ctypes.cast(arr, ctypes.POINTER(L.EbStraightRod))
        req.n_rods = len(rods)
        vel = None
        if velocities is not None:
            vel = np.ascontiguousarray(np.concatenate([np.asarray(v, dtype=np.float64).reshape(-1)
                                                      for v in velocities]))
            req.velocities = vel.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        req.dt = float(dt)
        req.n_steps = int(n_steps)
        opts = 0
        if gravity is not None:
            opts |= L.EB_REQUEST_GRAVITY
            for d in range(3):
                req.gravity[d] = float(gravity[d])
        if clamp:
            opts |= L.EB_REQUEST_CLAMP
        if damper is not None:
            opts |= L.EB_REQUEST_DAMPER
            req.damper_translational, req.damper_rotational = float(damper[0]), float(damper[1])
        req.options = opts
        rid = ctypes.c_int64()
        L.call("eb_server_submit", self._h, ctypes.byref(req), ctypes.byref(rid))
        self._rods[rid.value] = [int(r.n_elements) for r in rods]
        return rid.value

    def tick(self) -> int:
        """One tick; returns the number of requests still in flight."""
        n = ctypes.c_int64()
        L.call("eb_server_tick", self._h, ctypes.byref(n))
        return n.value

    def poll(self, capacity: int = 1024) -> list[dict]:
        buf = (L.EbCompletion * capacity)()
        n = ctypes.c_int32()
        L.call("eb_server_poll", self._h, buf, capacity, ctypes.byref(n))
        return [{"request_id": c.request_id, "precision": _NAMES[c.precision], "fell_back": bool(c.fell_back),
                 "latency_s": c.latency_s, "queued_s": c.queued_s, "energy_initial": c.energy_initial,
                 "energy_final": c.energy_final,
                 "elements": c.elements, "steps": c.steps} for c in buf[:n.value]]

    def result(self, request_id: int, rod: int, name: str) -> np.ndarray:
        place, nc = L.FIELD_SHAPE[name]
        n = self._rods[request_id][rod]
        count = n + 1 if place == 0 else n
        out = np.empty((nc, count), dtype=np.float64)
        L.call("eb_server_result", self._h, int(request_id), int(rod), L.FIELD_ID[name],
               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size)
        return out.reshape(3, 3, count) if name == "Director" else out

    def release(self, request_id: int) -> None:
        L.call("eb_server_release", self._h, int(request_id))
        self._rods.pop(request_id, None)

    _STATES = ("queued", "active", "finishing", "done")

    def request_status(self, request_id: int) -> dict:
        """Where a request is (queued, active, finishing, done), its age (its
        latency once done) and its queueing delay (a lower bound while it is
        still queued)."""
        st, age, q = ctypes.c_int32(), ctypes.c_double(), ctypes.c_double()
        L.call("eb_server_request_status", self._h, int(request_id), ctypes.byref(st), ctypes.byref(age),
               ctypes.byref(q))
        return {"state": self._STATES[st.value], "age_s": age.value, "queued_s": q.value}

    def stats(self) -> dict:
        st = L.EbServerStats()
        L.call("eb_server_get_stats", self._h, ctypes.byref(st))
        return {k: getattr(st, k) for k, _ in L.EbServerStats._fields_}

    def run_until_idle(self, max_ticks: int = 10_000_000) -> list[dict]:
        """Tick until nothing is in flight; returns every completion."""
        done = []
        for _ in range(max_ticks):
            left = self.tick()
            done += self.poll()
            if left == 0:
                break
        done += self.poll()
        return done
