"""Python handle on an ``hdr_server`` (include/hdrestir.h): shared resident
scenes, FIFO admission by HBM budget, one frame of every admitted job per
step, RIS jobs of one scene traced in one batched launch."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .context import path_settings, ris_params
from .scene import Camera, Scene


class Server:
    def __init__(self, device: int = 0, hbm_budget: int = 0, max_batch: int = 0, serial: bool = False,
                 step_pixels: int = 0, age_weight: float = 0.0):
        self._lib = abi.lib()
        self._h = C.c_void_p()
        d = abi.ServerDesc(int(device), abi.SERVER_SERIAL if serial else 0, int(hbm_budget), int(max_batch),
                           int(step_pixels), float(age_weight))
        abi.check(self._lib.hdr_server_create(C.byref(self._h), C.byref(d)))
        self._sizes: dict[int, tuple[int, int]] = {}

    def close(self) -> None:
        if self._h:
            self._lib.hdr_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_scene(self, scene: Scene) -> int:
        sid = C.c_int32()
        abi.check(self._lib.hdr_server_add_scene(self._h, C.byref(scene.c_desc()), C.byref(sid)))
        return sid.value

    def submit(self, scene_id: int, cam: Camera, frames: int, pipeline: str = "ris", firefly: bool = True,
               **settings) -> int:
        """settings: RIS keywords of Context.ris_path_trace (candidate_count, use_reservoir, ...) and the
        path settings (max_depth, ...), which also configure the PathTracer pipeline."""
        j = abi.JobDesc()
        j.scene = int(scene_id)
        j.pipeline = abi.JOB_RIS if pipeline == "ris" else abi.JOB_PATH_TRACER
        j.frames = int(frames)
        j.firefly = int(firefly)
        j.camera = cam.c_desc()
        j.ris = ris_params(**settings) if pipeline == "ris" else abi.RisParams(path=path_settings(**settings))
        jid = C.c_int64()
        abi.check(self._lib.hdr_server_submit(self._h, C.byref(j), C.byref(jid)))
        self._sizes[jid.value] = (cam.width, cam.height)
        return jid.value

    def step(self) -> int:
        n = C.c_int32()
        abi.check(self._lib.hdr_server_step(self._h, C.byref(n)))
        return n.value

    def finished(self) -> list[int]:
        """Ids of the jobs that finished since the last call."""
        out: list[int] = []
        buf = (C.c_int64 * 256)()
        n = C.c_int32()
        while True:
            abi.check(self._lib.hdr_server_drain_finished(self._h, buf, 256, C.byref(n)))
            out.extend(buf[k] for k in range(n.value))
            if n.value < 256:
                return out

    def state(self, job_id: int) -> tuple[int, int]:
        st, fr = C.c_int32(), C.c_int32()
        abi.check(self._lib.hdr_server_job_state(self._h, C.c_int64(job_id), C.byref(st), C.byref(fr)))
        return st.value, fr.value

    def take(self, job_id: int, keep_image: bool = True) -> np.ndarray | None:
        w, h = self._sizes.pop(job_id)
        out = np.empty((w * h, 4), np.float32) if keep_image else None
        ptr = out.ctypes.data_as(C.c_void_p) if out is not None else None
        abi.check(self._lib.hdr_server_take_result(self._h, C.c_int64(job_id), ptr, out.nbytes if out is not None
                                                   else 0))
        return out

    def load(self) -> tuple[int, int, int]:
        q, r, b = C.c_int32(), C.c_int32(), C.c_size_t()
        abi.check(self._lib.hdr_server_load(self._h, C.byref(q), C.byref(r), C.byref(b)))
        return q.value, r.value, b.value
