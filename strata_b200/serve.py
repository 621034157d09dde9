"""Serving: window requests over a device-resident DEM mosaic, with
continuous batching (strata_server_*).

    srv = serve.Server(mosaic, budget_bytes=120 << 30)
    t = srv.submit(terrain.slope_stage(opts), x, y, w, h)
    res = srv.wait(t)        # the window's result (device memory) and its timings
    res.copy_to(dst)         # into a raster of the window's size
    srv.release(t)           # frees the outputs and their budget

Requests are admitted in arrival order while their outputs fit the memory
budget and run in batches as they arrive; batches on the server's streams
overlap on the device, so a request that arrives while others run joins
the next batch rather than waiting for the queue to drain. Each window is
a raster of its own (its border is its edge ring), so a request's result
is the one strata_process gives for the window view.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np

from . import _lib, engine
from .raster import Float32Raster


class Result:
    """A request's outputs (device rasters the server owns until release)
    and its submit / start / done times (steady clock, ns). The outputs of
    a result from wait_many are built on first use from the columns of the
    whole call's result table (cols, row)."""

    __slots__ = ("_outputs", "_cols", "t_submit_ns", "t_start_ns", "t_done_ns")

    def __init__(self, outputs: Optional[List[Float32Raster]], t_submit_ns: int, t_start_ns: int, t_done_ns: int,
                 cols=None):
        self._outputs = outputs
        self._cols = cols
        self.t_submit_ns, self.t_start_ns, self.t_done_ns = t_submit_ns, t_start_ns, t_done_ns

    @property
    def outputs(self) -> List[Float32Raster]:
        if self._outputs is None:
            (nout, data, width, height, stride, valid), i = self._cols
            self._outputs = [Float32Raster(data[i][k], width[i][k], height[i][k], stride[i][k], valid[i][k] or None, 0)
                             for k in range(nout[i])]
            self._cols = None
        return self._outputs

    @property
    def latency_ms(self) -> float:
        return (self.t_done_ns - self.t_submit_ns) / 1e6

    def copy(self, k: int = 0) -> Float32Raster:
        """Output k as a device raster of torch tensors the caller owns."""
        src = self.outputs[k]
        n = src.width * src.height
        data = _device_view(src.data, n, "<f4").clone()
        valid = _device_view(src.valid, (n + 63) // 64, "<i8").clone() if src.valid else None
        return Float32Raster(data, src.width, src.height, src.width, valid, 0)


def _device_view(ptr: int, n: int, typestr: str):
    """A torch tensor over n elements of device memory at ptr (no copy)."""
    import torch

    class _Buf:
        __cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Buf(), device="cuda")


class Server:
    def __init__(self, mosaic: Float32Raster, budget_bytes: int = 0, streams: int = 0, max_batch: int = 0,
                 device: int = 0, band: int = 0):
        self.mosaic = mosaic  # keeps the device buffers alive
        c = engine.device_context(device)
        o = _lib.ServerOpts(budget_bytes, streams, max_batch, band, 0)
        p = ctypes.c_void_p()
        _lib.check(_lib.lib().strata_server_create(c, ctypes.byref(engine.c_raster(mosaic)), ctypes.byref(o),
                                                   ctypes.byref(p)))
        self._h = p

    def submit(self, stages: engine.StageList, x: int, y: int, w: int, h: int) -> int:
        t = ctypes.c_uint64()
        _lib.check(_lib.lib().strata_server_submit(self._h, stages.c_array(), len(stages.stages), x, y, w, h,
                                                   ctypes.byref(t)))
        return t.value

    def submit_many(self, requests) -> List[int]:
        """Submits (stages, x, y, w, h) requests in one call; their tickets,
        in order. Checks every request first and submits none if one is
        invalid."""
        requests = list(requests)
        n = len(requests)
        req = np.zeros(n, _lib.SERVER_REQUEST_DTYPE)
        if n:
            req["stages"] = [r[0].c_address() for r in requests]
            req["nstages"] = [len(r[0].stages) for r in requests]
            xywh = np.array([r[1:5] for r in requests], dtype=np.int64)
            req["x"], req["y"], req["w"], req["h"] = xywh[:, 0], xywh[:, 1], xywh[:, 2], xywh[:, 3]
        t = np.zeros(n, np.uint64)
        _lib.check(_lib.lib().strata_server_submit_many(self._h, req.ctypes.data_as(ctypes.POINTER(_lib.ServerRequest)),
                                                        n, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return t.tolist()

    def wait_many(self, tickets: Sequence[int], timeout_ms: int = -1) -> List[Result]:
        """Waits for every ticket, in order; their results."""
        n = len(tickets)
        t = np.ascontiguousarray(tickets, dtype=np.uint64)
        res = np.zeros(n, _lib.SERVER_RESULT_DTYPE)
        _lib.check(_lib.lib().strata_server_wait_many(self._h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), n,
                                                      timeout_ms, res.ctypes.data_as(
                                                          ctypes.POINTER(_lib.ServerResult))))
        out = res["out"]
        cols = (res["nout"].tolist(), out["data"].tolist(), out["width"].tolist(), out["height"].tolist(),
                out["stride"].tolist(), out["valid"].tolist())
        ts, tb, td = res["t_submit_ns"].tolist(), res["t_start_ns"].tolist(), res["t_done_ns"].tolist()
        return [Result(None, ts[i], tb[i], td[i], (cols, i)) for i in range(n)]

    def release_many(self, tickets: Sequence[int]) -> None:
        n = len(tickets)
        t = np.ascontiguousarray(tickets, dtype=np.uint64)
        _lib.check(_lib.lib().strata_server_release_many(self._h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), n))

    @staticmethod
    def _result(r) -> Result:
        outs = [Float32Raster(r.out[k].data, r.out[k].width, r.out[k].height, r.out[k].stride,
                              r.out[k].valid if r.out[k].valid else None, 0) for k in range(r.nout)]
        return Result(outs, r.t_submit_ns, r.t_start_ns, r.t_done_ns)

    def wait(self, ticket: int, timeout_ms: int = -1) -> Result:
        r = _lib.ServerResult()
        _lib.check(_lib.lib().strata_server_wait(self._h, ticket, timeout_ms, ctypes.byref(r)))
        outs = []
        for k in range(r.nout):
            o = r.out[k]
            outs.append(Float32Raster(o.data, o.width, o.height, o.stride, o.valid if o.valid else None, 0))
        return Result(outs, r.t_submit_ns, r.t_start_ns, r.t_done_ns)

    def poll(self, ticket: int) -> Optional[Result]:
        """The request's result if it is done, else None (no waiting)."""
        r = _lib.ServerResult()
        rc = _lib.lib().strata_server_wait(self._h, ticket, 0, ctypes.byref(r))
        if rc == _lib.ETIMEDOUT:
            return None
        _lib.check(rc)
        outs = [Float32Raster(r.out[k].data, r.out[k].width, r.out[k].height, r.out[k].stride,
                              r.out[k].valid if r.out[k].valid else None, 0) for k in range(r.nout)]
        return Result(outs, r.t_submit_ns, r.t_start_ns, r.t_done_ns)

    def release(self, ticket: int) -> None:
        _lib.check(_lib.lib().strata_server_release(self._h, ticket))

    def stats(self):
        b, s, u = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.lib().strata_server_stats(self._h, ctypes.byref(b), ctypes.byref(s), ctypes.byref(u)))
        return {"batches": b.value, "served": s.value, "used_bytes": u.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().strata_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
