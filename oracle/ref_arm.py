"""TEST INFRASTRUCTURE / CPU BASELINE: the reference's own CPU renderer on
the benchmark frame, with no product code loaded.

The closed room with the displaced 81,920-triangle icosphere, 1024 x 1024,
64 spp, depth 10, NEE on, is built through the reference's own classes by
oracle/_ref/libptref.so (ref_room_mesh_world: a restatement of the product's
generator, checked byte for byte against it by tests/test_ref_arm.py) and
rendered by the reference's render_row_linear on the host's cores with the
src/main.cpp row scheduler. This module imports only the standard library
and numpy; bench.py uses it for its reference arm and for the cpu_baseline
beside its own line, so the two are one measurement: the same fixed set of
rows (every 8th scanline of the frame), best of several runs.
"""
from __future__ import annotations

import ctypes as C
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libptref.so")

WIDTH, HEIGHT, SPP, DEPTH, SEED, SUBDIV = 1024, 1024, 64, 10, 1, 6
ROW_STRIDE = 8


def available() -> bool:
    return os.path.exists(REF_LIB)


def host_cpu() -> dict:
    """Threads this process may use and the CPU model (/proc/cpuinfo)."""
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"threads": cores, "cpu_count": os.cpu_count(), "model": model}


class RoomMeshFrame:
    """The benchmark frame in the reference's own geometry."""

    def __init__(self):
        if not available():
            raise RuntimeError("oracle/_ref/libptref.so is absent (built from the reference checkout)")
        L = C.CDLL(REF_LIB)
        L.ref_room_mesh_world.restype = C.c_void_p
        L.ref_room_mesh_world.argtypes = [C.c_uint64, C.c_int]
        L.ref_world_render_rows.restype = C.c_uint64
        L.ref_world_render_rows.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_void_p,
                                            C.c_int, C.c_void_p, C.c_int]
        L.ref_world_destroy.argtypes = [C.c_void_p]
        self.lib = L
        self.h = L.ref_room_mesh_world(SEED, SUBDIV)
        self.rows = [j for j in range(ROW_STRIDE // 2, HEIGHT, ROW_STRIDE)]
        self._rows = (C.c_int * len(self.rows))(*self.rows)

    def sample(self) -> str:
        return (f"every {ROW_STRIDE}th scanline ({len(self.rows)} rows x {WIDTH} px x {SPP} spp) of the "
                f"{WIDTH}x{HEIGHT} frame")

    def render_rows(self, threads: int) -> tuple[int, float]:
        """One pass over the row set: (rays, seconds)."""
        t0 = time.perf_counter()
        rays = self.lib.ref_world_render_rows(self.h, WIDTH, HEIGHT, SPP, DEPTH, SEED, self._rows, len(self.rows),
                                              None, threads)
        return int(rays), time.perf_counter() - t0

    def close(self):
        if self.h:
            self.lib.ref_world_destroy(self.h)
            self.h = None


def best_of(frame: RoomMeshFrame, runs: int, threads: int) -> tuple[float, list]:
    """Mrays/s of the fastest of `runs` passes over the row set, and every pass."""
    passes = [frame.render_rows(threads) for _ in range(runs)]
    rays, secs = min(passes, key=lambda p: p[1])
    return rays / secs / 1e6, passes
