"""Served mode: continuous batching of simulation jobs (soil_server_* C ABI).

``Server`` wraps the native request loop: ``submit`` queues a job (one
periodic box with the harmonic consumer, optional shear, a step count), the
loop admits jobs against the HBM budget as memory and slots free up, advances
every resident job in one batched step, and retires finished ones.  Results
are bit-identical to running the same job alone with ``System.step``.

The server owns its ``Context`` for the GPU work of its loop thread; give it
a context that nothing else uses.
"""
import ctypes as C

import numpy as np

from . import abi


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Server:
    def __init__(self, ctx, hbm_budget_bytes=0, max_active=0, quantum_steps=0,
                 bytes_per_atom=0, bytes_per_job=0):
        self.ctx = ctx
        self.lib = ctx.lib
        cfg = abi.SoilServerCfg(hbm_budget_bytes, max_active, quantum_steps, bytes_per_atom,
                                bytes_per_job)
        h = C.c_void_p()
        ctx.check(self.lib.soil_server_create(ctx.h, C.byref(cfg), C.byref(h)),
                  "soil_server_create")
        self.h = h
        self.natoms = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.soil_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, st, where):
        if st != abi.SOIL_OK:
            raise abi.SoilError(st, where, "")

    def submit(self, w, steps=None):
        """Queue workload `w` (workloads.Workload) for `steps` (default w.steps)."""
        n = w.n
        keep = dict(
            tag=np.ascontiguousarray(w.tag, dtype=np.uint32),
            pos=np.ascontiguousarray(w.pos, dtype=np.float64).reshape(n, 3),
            vel=np.ascontiguousarray(w.vel, dtype=np.float64).reshape(n, 3),
            mass=np.ascontiguousarray(w.mass, dtype=np.float64),
            cut=np.ascontiguousarray(w.cutoff, dtype=np.float64),
            rad=np.ascontiguousarray(w.radius, dtype=np.float64))
        spec = abi.SoilJobSpec()
        spec.box = w.box
        spec.cfg = w.cfg
        spec.dt = w.dt
        spec.natoms = n
        spec.tag = _p(keep["tag"], C.c_uint32)
        spec.pos3 = _p(keep["pos"], C.c_double)
        spec.vel3 = _p(keep["vel"], C.c_double)
        spec.mass = _p(keep["mass"], C.c_double)
        spec.cutoff_radius = _p(keep["cut"], C.c_double)
        spec.radius = _p(keep["rad"], C.c_double)
        spec.harmonic_k = w.harmonic_k
        spec.shear_rate = w.shear_rate
        spec.steps = int(w.steps if steps is None else steps)
        jid = C.c_uint64()
        self._check(self.lib.soil_server_submit(self.h, C.byref(spec), C.byref(jid)),
                    "soil_server_submit")
        self.natoms[jid.value] = n
        return jid.value

    @staticmethod
    def _info(i):
        return dict(state=abi.JOB_STATES[i.state], natoms=i.natoms, steps=i.steps,
                    steps_done=i.steps_done, t_submit=i.t_submit, t_admit=i.t_admit,
                    t_done=i.t_done)

    def poll(self, jid):
        i = abi.SoilJobInfo()
        self._check(self.lib.soil_server_poll(self.h, jid, C.byref(i)), "soil_server_poll")
        return self._info(i)

    def wait(self, jid, timeout=None):
        """Block until the job ends; raises SoilError(SOIL_ERR_TIMEOUT) on timeout."""
        i = abi.SoilJobInfo()
        self._check(self.lib.soil_server_wait(self.h, jid, -1.0 if timeout is None else timeout,
                                              C.byref(i)), "soil_server_wait")
        return self._info(i)

    def cancel(self, jid):
        self._check(self.lib.soil_server_cancel(self.h, jid), "soil_server_cancel")

    def result(self, jid):
        n = self.natoms[jid]
        out = dict(tag=np.zeros(n, np.uint32), pos=np.zeros((n, 3)), vel=np.zeros((n, 3)),
                   image=np.zeros((n, 3), np.int32))
        self._check(self.lib.soil_server_result(self.h, jid, _p(out["tag"], C.c_uint32),
                                                _p(out["pos"], C.c_double),
                                                _p(out["vel"], C.c_double),
                                                _p(out["image"], C.c_int32)),
                    "soil_server_result")
        return out

    def error(self, jid):
        buf = C.create_string_buffer(512)
        self._check(self.lib.soil_server_job_error(self.h, jid, buf, 512), "job_error")
        return buf.value.decode(errors="replace")

    def release(self, jid):
        self._check(self.lib.soil_server_release(self.h, jid), "soil_server_release")
        self.natoms.pop(jid, None)

    def stats(self):
        s = abi.SoilServerStats()
        self._check(self.lib.soil_server_get_stats(self.h, C.byref(s)), "soil_server_get_stats")
        return {name: getattr(s, name) for name, _ in s._fields_}


def poisson_arrivals(rate_per_s, count, seed):
    """Arrival times (s) of a Poisson stream: exponential gaps from SplitMix64
    uniforms (inverse transform), first arrival at t = 0."""
    from . import workloads
    u = workloads.uniform(seed, 0, 92, count)
    gaps = -np.log1p(-u) / rate_per_s
    gaps[0] = 0.0
    return np.cumsum(gaps)


def fifo_latencies(arrivals, service):
    """Latency (completion - arrival) of each job on one FIFO server that
    runs jobs one at a time (Lindley recursion)."""
    t_free = 0.0
    lat = np.zeros(len(arrivals))
    for k, (a, s) in enumerate(zip(arrivals, service)):
        start = max(a, t_free)
        t_free = start + s
        lat[k] = t_free - a
    return lat
