"""Continuous-batching DPD job server over the C ABI (dpd_server_* in include/dpd_b200.h).

Jobs are a run.in text plus a system (:class:`gpumdpd_b200.inputs.System`).  Each call to
:meth:`Server.step` is one scheduling point: queued jobs that fit the device-memory
budget are admitted as a new cohort (one packed engine), every cohort advances by one
chunk of steps with all cohorts' kernels in flight together, and finished jobs are
retired with their thermo means, final state and RDF.  Latency of a job is its finish
time minus its submit time on the server's clock.
"""
import ctypes

import numpy as np

from . import capi
from .capi import DpdError


class Server:
    def __init__(self, hbm_budget_bytes, chunk_steps=200, tuning=None):
        self.lib = capi.load()
        self.h = ctypes.c_void_p()
        tune = None
        if tuning is not None:
            t = capi.tuning(**tuning)
            tune = ctypes.byref(t)
        code = self.lib.dpd_server_create(float(hbm_budget_bytes), int(chunk_steps), tune, ctypes.byref(self.h))
        if code:
            raise DpdError(code, "dpd_server_create failed")
        self.n_atoms = {}
        self.nbins = {}

    def _check(self, code):
        if code != 0:
            msg = self.lib.dpd_server_last_error(self.h)
            raise DpdError(code, msg.decode() if msg else "")

    def close(self):
        if self.h:
            self.lib.dpd_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_policy(self, max_wait_s=0.0, min_jobs=1):
        """Admission window: gather queued jobs into one batch until `min_jobs` wait or the
        oldest has waited `max_wait_s` (only while other jobs are running)."""
        self._check(self.lib.dpd_server_set_policy(self.h, float(max_wait_s), int(min_jobs)))

    def submit(self, system, run_in=None):
        """Queue a job; returns its id.  `run_in` defaults to the system's own text."""
        s, keep = system.c_system()
        jid = ctypes.c_int64()
        self._check(self.lib.dpd_server_submit(self.h, (run_in or system.run_in).encode(), ctypes.byref(s),
                                               ctypes.byref(jid)))
        del keep
        self.n_atoms[jid.value] = system.n
        return jid.value

    def step(self):
        """One scheduling point; returns (running jobs, queued jobs)."""
        a, q = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.dpd_server_step(self.h, ctypes.byref(a), ctypes.byref(q)))
        return a.value, q.value

    def result(self, job_id):
        r = capi.dpd_job_result()
        self._check(self.lib.dpd_server_result(self.h, int(job_id), ctypes.byref(r)))
        status = {0: "done", 1: "queued", 2: "running", -9: "cancelled"}.get(r.status, f"error {r.status}")
        return {"job_id": r.job_id, "status": status, "code": r.status, "steps": r.steps,
                "mean_temp": r.mean_temp, "mean_pressure": r.mean_pressure,
                "stderr_temp": r.stderr_temp, "stderr_pressure": r.stderr_pressure,
                "submit_s": r.submit_s, "start_s": r.start_s,
                "finish_s": r.finish_s, "latency_s": r.finish_s - r.submit_s if r.finish_s >= 0 else None,
                "last_temp": r.last.temp, "last_pressure": r.last.pressure, "last_step": r.last.step}

    def cancel(self, job_id):
        """Cancel a queued or running job (its status becomes "cancelled")."""
        self._check(self.lib.dpd_server_cancel(self.h, int(job_id)))

    def state(self, job_id):
        n = self.n_atoms[job_id]
        x, v = np.empty((n, 3)), np.empty((n, 3))
        self._check(self.lib.dpd_server_job_state(self.h, int(job_id), capi.ptr(x), capi.ptr(v)))
        return {"x": x, "v": v}

    def rdf(self, job_id, nbins):
        g = np.empty(nbins)
        ns = ctypes.c_int64()
        self._check(self.lib.dpd_server_job_rdf(self.h, int(job_id), capi.ptr(g), ctypes.byref(ns)))
        return g, ns.value

    def stats(self):
        ps, busy, db = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int64()
        self._check(self.lib.dpd_server_stats(self.h, ctypes.byref(ps), ctypes.byref(busy), ctypes.byref(db)))
        return {"particle_steps": ps.value, "busy_s": busy.value, "device_bytes": db.value}

    def drain(self, max_points=10 ** 7):
        """Step until no job is running or queued."""
        for _ in range(max_points):
            a, q = self.step()
            if a == 0 and q == 0:
                return
        raise RuntimeError("server did not drain")


def latency_percentiles(results, qs=(50, 99)):
    lat = np.array([r["latency_s"] for r in results if r["latency_s"] is not None])
    return {f"p{q}": float(np.percentile(lat, q)) for q in qs} if len(lat) else {}
