"""Serving loop over the C ABI (mpm_server_*): jobs admitted by device-memory
budget into one batch, all resident scenes advanced together every substep,
per-job latency from arrival to completion on the device's timeline.

No counterpart in the reference (an interactive single-scene page)."""
import ctypes

import numpy as np

from . import abi
from .abi import BUF, JobResult, ServerDesc, ServerStats, check, load_library


class Server:
    def __init__(self, hbm_budget_bytes, scene_capacity=256, cells_per_particle=2.0, device=0, flags=0,
                 max_inflight=2, lib=None):
        self.lib = lib or load_library()
        d = ServerDesc(int(hbm_budget_bytes), float(cells_per_particle), int(scene_capacity), int(device),
                       int(flags), int(max_inflight))
        self.h = ctypes.c_void_p()
        check(self.lib.mpm_server_create(ctypes.byref(d), ctypes.byref(self.h)), "mpm_server_create")
        self.jobs = {}

    def submit(self, params, pos4, mass, substeps, arrival_s, vel4=None):
        j = ctypes.c_int64()
        check(self.lib.mpm_server_submit(self.h, ctypes.byref(params), abi.ptr(pos4), abi.ptr(vel4), abi.ptr(mass),
                                         len(mass), int(substeps), float(arrival_s), ctypes.byref(j)),
              "mpm_server_submit")
        self.jobs[j.value] = len(mass)
        return j.value

    def run(self):
        st = ServerStats()
        check(self.lib.mpm_server_run(self.h, ctypes.byref(st)), "mpm_server_run")
        return st

    def job(self, j):
        r = JobResult()
        check(self.lib.mpm_server_job(self.h, int(j), ctypes.byref(r)), "mpm_server_job")
        return r

    def download(self, j, name):
        n = self.jobs[j]
        shape = {"pos": (n, 4), "vel": (n, 4), "density": (n,)}[name]
        a = np.zeros(shape, np.float32)
        check(self.lib.mpm_server_download(self.h, int(j), BUF[name], abi.ptr(a), a.nbytes), "mpm_server_download")
        return a

    def close(self):
        if self.h:
            self.lib.mpm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
