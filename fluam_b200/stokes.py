"""Python mirror of the Stokes-limit scheme over the libfluamsl C ABI.

``StokesLimit`` owns one device instance (the state the reference keeps in
process globals between ``schemeStokesLimit`` and ``runSchemeStokesLimit``,
src/schemeStokesLimit.cu:27-98).  ``run_data_main`` is the drop-in driver of
``fluam data.main`` for the stokesLimit scheme.  Arrays are numpy: particle
arrays have shape (3, np) (x, y and z rows, as rxParticle/ryParticle/
rzParticle), fields have shape (3, mz, my, mx).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import (PAIR_NONE, PAIR_SOFT, PAIR_TABLE_LJ, RFD_PAPER, RFD_REFERENCE, SCHEME_FIRST_ORDER,
                   SCHEME_INCOMPRESSIBLE, SCHEME_MIDPOINT, SCHEME_QUASI2D, SCHEME_STOKES2D, check)

__all__ = ["StokesLimit", "Batch", "Server", "make_config", "run_data_main", "parse_data_main", "PAIR_NONE",
           "PAIR_SOFT", "PAIR_TABLE_LJ", "RFD_PAPER", "RFD_REFERENCE", "SCHEME_MIDPOINT",
           "SCHEME_FIRST_ORDER", "SCHEME_QUASI2D", "SCHEME_STOKES2D", "SCHEME_INCOMPRESSIBLE"]


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def make_config(cells, box, eta=1.0, kT=0.0, dt=0.01, cutoff=0.0, kernel=3, pair=PAIR_TABLE_LJ,
                soft_epsilon=1.0, rfd=RFD_REFERENCE, nonbonded=1, extra_mobility=0.0, seed=0,
                device=-1, scheme=0, precision=0, radius=1.0, ndrift=1, use_rfd=1,
                predictor_corrector=0, saffman_kc=0.0, saffman_width=0.0, shear_amp=0.0,
                density=1.0, observables=0):
    c = _lib.Config()
    _lib.load().fsl_config_defaults(ctypes.byref(c))
    c.mx, c.my, c.mz = (int(x) for x in cells)
    c.lx, c.ly, c.lz = (float(x) for x in box)
    c.shearviscosity, c.temperature, c.dt, c.cutoff = eta, kT, dt, cutoff
    c.kernel, c.pair, c.soft_epsilon, c.rfd = kernel, pair, soft_epsilon, rfd
    c.nonbonded, c.extra_mobility, c.seed, c.device = nonbonded, extra_mobility, seed, device
    c.scheme = scheme
    c.precision = precision
    # quasi-2D family (scheme SCHEME_QUASI2D / SCHEME_STOKES2D)
    c.radius, c.ndrift, c.use_rfd, c.predictor_corrector = radius, ndrift, use_rfd, predictor_corrector
    c.saffman_kc, c.saffman_width, c.shear_amp = saffman_kc, saffman_width, shear_amp
    c.density = density  # incompressible scheme
    c.observables = observables  # FP64 accumulators on the device (3-D Stokes schemes)
    return c


class StokesLimit:
    """One Stokes-limit instance on the GPU."""

    def __init__(self, config, q):
        self.L = _lib.load()
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(3, -1)
        self.np = q.shape[1]
        self.cfg = config
        self.shape = (config.mz, config.my, config.mx)
        self.nc = config.mx * config.my * config.mz
        h = ctypes.c_void_p()
        check(self.L.fsl_create(ctypes.byref(config), self.np, _dp(q), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.fsl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- scheme ------------------------------------------------------------
    def load_bonds(self, bi, bj, k, r0, fi=None, fk=None, fr0=None, fxyz=None, directed=False):
        """Bonds acting on both particles (fsl_load_bonds), or with
        directed=True entries acting on bi only (fsl_load_bonds_directed, the
        old bond-file format)."""
        bi = np.ascontiguousarray(bi, dtype=np.int32)
        bj = np.ascontiguousarray(bj, dtype=np.int32)
        k = np.ascontiguousarray(k, dtype=np.float64)
        r0 = np.ascontiguousarray(r0, dtype=np.float64)
        if fi is None:
            fi, fk, fr0, fxyz = np.zeros(0, np.int32), np.zeros(0), np.zeros(0), np.zeros((0, 3))
        fi = np.ascontiguousarray(fi, dtype=np.int32)
        fk = np.ascontiguousarray(fk, dtype=np.float64)
        fr0 = np.ascontiguousarray(fr0, dtype=np.float64)
        fxyz = np.ascontiguousarray(fxyz, dtype=np.float64).reshape(-1, 3)
        fn = self.L.fsl_load_bonds_directed if directed else self.L.fsl_load_bonds
        check(fn(self.h, len(bi), _ip(bi), _ip(bj), _dp(k), _dp(r0), len(fi),
                 _ip(fi), _dp(fk), _dp(fr0), _dp(fxyz)))

    def step(self, n=1):
        check(self.L.fsl_step(self.h, int(n)))

    def sync(self):
        check(self.L.fsl_sync(self.h))

    def set_graph(self, enable):
        check(self.L.fsl_set_graph(self.h, 1 if enable else 0))

    def positions(self):
        out = np.empty((3, self.np))
        check(self.L.fsl_get_positions(self.h, _dp(out)))
        return out

    def set_positions(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(3, self.np)
        check(self.L.fsl_set_positions(self.h, _dp(q)))

    def forces(self):
        out = np.empty((3, self.np))
        check(self.L.fsl_get_forces(self.h, _dp(out)))
        return out

    def set_velocity64(self, v):
        """Initial velocity of the incompressible scheme (projected)."""
        v = np.ascontiguousarray(v, dtype=np.float64).reshape((3,) + self.shape)
        check(self.L.fsl_set_velocity_f64(self.h, v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def velocity64(self):
        """The fluid velocity of the last solve as float64, in every precision form."""
        out = np.empty((3,) + self.shape, dtype=np.float64)
        check(self.L.fsl_get_velocity_f64(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def velocity(self):
        out = np.empty((3,) + self.shape, dtype=np.float32)
        check(self.L.fsl_get_velocity(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def observables(self):
        """FP64 device accumulators (config observables=1): msd, displacement,
        total force, fluid momentum and their sums over the steps."""
        o = _lib.Observables()
        check(self.L.fsl_get_observables(self.h, ctypes.byref(o)))
        return o.as_dict()

    def reset_observables(self):
        """q0 := the current positions, accumulators := 0."""
        check(self.L.fsl_reset_observables(self.h))

    def status(self):
        st = _lib.Status()
        check(self.L.fsl_get_status(self.h, ctypes.byref(st)))
        return {"step": st.step, "error_bits": st.error_bits, "np": st.np, "nc": st.nc,
                "graph": bool(st.graph), "launches_per_step": st.launches_per_step}

    def step_io(self, q_in, q_out):
        """One step with its positions in and out (fsl_step_io): q_in, q_out
        are host addresses of 3 x np doubles (page-locked for the in-graph
        copies), or (3, np) float64 arrays."""
        def addr(a):
            if isinstance(a, np.ndarray):
                assert a.dtype == np.float64 and a.size == 3 * self.np and a.flags.c_contiguous
                return a.ctypes.data
            return int(a)
        check(self.L.fsl_step_io(self.h, ctypes.c_void_p(addr(q_in)), ctypes.c_void_p(addr(q_out))))

    def tuning(self):
        """The autotuner's picks and timings (after the first step)."""
        t = _lib.ClassTuning()
        check(self.L.fsl_get_tuning(self.h, ctypes.byref(t)))
        return t.as_dict()

    def profile(self, enable=True):
        """Per-stage CUDA-event timing of every step (clears the totals)."""
        check(self.L.fsl_profile(self.h, 1 if enable else 0))

    def profile_read(self):
        n = ctypes.c_int32()
        check(self.L.fsl_profile_read(self.h, None, 0, ctypes.byref(n)))
        arr = (_lib.StageTime * max(n.value, 1))()
        check(self.L.fsl_profile_read(self.h, arr, n.value, ctypes.byref(n)))
        return {a.name.decode(): {"launches": a.launches, "total_ms": a.total_ms}
                for a in arr[:n.value]}

    def set_step(self, t):
        check(self.L.fsl_set_step(self.h, int(t)))

    def clear_errors(self):
        check(self.L.fsl_clear_errors(self.h))

    # -- components --------------------------------------------------------
    def neighbor_grid(self):
        d = np.zeros(3, np.int32)
        check(self.L.fsl_neighbor_grid(self.h, _ip(d)))
        return tuple(int(x) for x in d)

    def cell_list(self):
        m = int(np.prod(self.neighbor_grid()))
        cell_of = np.empty(self.np, np.int32)
        start = np.empty(m + 1, np.int32)
        srt = np.empty(self.np, np.int32)
        check(self.L.fsl_cell_list(self.h, _ip(cell_of), _ip(start), _ip(srt)))
        return cell_of, start, srt

    def compute_forces(self):
        F = np.empty((3, self.np))
        check(self.L.fsl_compute_forces(self.h, _dp(F)))
        return F

    def spread(self, F):
        F = np.ascontiguousarray(F, dtype=np.float64)
        f = np.empty((3,) + self.shape)
        check(self.L.fsl_spread(self.h, _dp(F), _dp(f)))
        return f

    def solve(self, W):
        W = np.ascontiguousarray(W, dtype=np.float64)
        v = np.empty((3,) + self.shape)
        check(self.L.fsl_solve(self.h, _dp(W), _dp(v)))
        return v

    def interpolate(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        u = np.empty((3, self.np))
        check(self.L.fsl_interpolate(self.h, _dp(v), _dp(u)))
        return u

    def noise(self, t, first, count):
        out = np.empty(count, np.float32)
        check(self.L.fsl_noise(self.h, int(t), int(first), int(count),
                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out


class Batch:
    """Independent Stokes-limit instances stepped together (fsl_batch_*).

    ``configs`` is a sequence of Config, ``positions`` a sequence of (3, np_i)
    arrays.  Instances of the same size class share every kernel launch; each
    instance's results equal those of the same instance run alone.
    """

    def __init__(self, configs, positions):
        self.L = _lib.load()
        n = len(configs)
        if len(positions) != n:
            raise ValueError("one position array per configuration")
        qs = [np.ascontiguousarray(q, dtype=np.float64).reshape(3, -1) for q in positions]
        self.nps = np.array([q.shape[1] for q in qs], dtype=np.int64)
        cfgs = (_lib.Config * max(n, 1))(*configs)
        qp = (ctypes.POINTER(ctypes.c_double) * max(n, 1))(*[_dp(q) for q in qs])
        h = ctypes.c_void_p()
        check(self.L.fsl_batch_create(n, cfgs, self.nps.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                      qp, ctypes.byref(h)))
        self.h = h
        self.n = n
        self.offsets = np.concatenate([[0], np.cumsum(3 * self.nps)]).astype(np.int64)

    def close(self):
        if getattr(self, "h", None):
            self.L.fsl_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def load_bonds(self, i, bi, bj, k, r0):
        bi = np.ascontiguousarray(bi, dtype=np.int32)
        bj = np.ascontiguousarray(bj, dtype=np.int32)
        k = np.ascontiguousarray(k, dtype=np.float64)
        r0 = np.ascontiguousarray(r0, dtype=np.float64)
        z, zi = np.zeros(1), np.zeros(1, np.int32)
        check(self.L.fsl_batch_load_bonds(self.h, int(i), len(bi), _ip(bi), _ip(bj), _dp(k), _dp(r0),
                                          0, _ip(zi), _dp(z), _dp(z), _dp(z)))

    def step(self, n=1):
        check(self.L.fsl_batch_step(self.h, int(n)))

    def sync(self):
        check(self.L.fsl_batch_sync(self.h))

    def set_graph(self, enable):
        check(self.L.fsl_batch_set_graph(self.h, 1 if enable else 0))

    def positions(self, i):
        out = np.empty((3, int(self.nps[i])))
        check(self.L.fsl_batch_get_positions(self.h, int(i), _dp(out)))
        return out

    def forces(self, i):
        out = np.empty((3, int(self.nps[i])))
        check(self.L.fsl_batch_get_forces(self.h, int(i), _dp(out)))
        return out

    def observables(self, i):
        o = _lib.Observables()
        check(self.L.fsl_batch_get_observables(self.h, int(i), ctypes.byref(o)))
        return o.as_dict()

    def reset_observables(self, i):
        check(self.L.fsl_batch_reset_observables(self.h, int(i)))

    def status(self, i):
        st = _lib.Status()
        check(self.L.fsl_batch_get_status(self.h, int(i), ctypes.byref(st)))
        return {"step": st.step, "error_bits": st.error_bits, "np": st.np, "nc": st.nc,
                "graph": bool(st.graph), "launches_per_step": st.launches_per_step}

    def positions_packed(self, out=None):
        if out is None:
            out = np.empty(int(self.offsets[-1]))
        check(self.L.fsl_batch_get_positions_packed(self.h, _dp(out)))
        return out

    def set_positions_packed(self, packed):
        packed = np.ascontiguousarray(packed, dtype=np.float64).reshape(-1)
        if packed.size != self.offsets[-1]:
            raise ValueError("packed array has the wrong size")
        check(self.L.fsl_batch_set_positions_packed(self.h, _dp(packed)))

    def positions_packed_async(self, host_ptr):
        """Queue the packed positions into host memory at host_ptr (an int)."""
        check(self.L.fsl_batch_get_positions_packed_async(self.h, ctypes.c_void_p(host_ptr)))

    def set_positions_packed_async(self, host_ptr):
        check(self.L.fsl_batch_set_positions_packed_async(self.h, ctypes.c_void_p(host_ptr)))

    def unpack(self, packed, i):
        return packed[self.offsets[i]:self.offsets[i + 1]].reshape(3, -1)

    def info(self):
        b = _lib.BatchInfo()
        check(self.L.fsl_batch_get_info(self.h, ctypes.byref(b)))
        return {f: getattr(b, f) for f, _ in _lib.BatchInfo._fields_}

    def step_io(self, q_in, q_out):
        """One step of every instance with the packed positions in and out
        (fsl_batch_step_io): host addresses of offsets[-1] doubles
        (page-locked for the in-graph copies), or float64 arrays."""
        def addr(a):
            if isinstance(a, np.ndarray):
                assert a.dtype == np.float64 and a.size == int(self.offsets[-1]) and a.flags.c_contiguous
                return a.ctypes.data
            return int(a)
        check(self.L.fsl_batch_step_io(self.h, ctypes.c_void_p(addr(q_in)), ctypes.c_void_p(addr(q_out))))

    def class_tuning(self):
        """Per size class: the autotuner's picks and timings (after the
        first step)."""
        out = []
        for k in range(self.info()["classes"]):
            t = _lib.ClassTuning()
            check(self.L.fsl_batch_get_class_tuning(self.h, k, ctypes.byref(t)))
            out.append(t.as_dict())
        return out

    def stream(self):
        return self.L.fsl_batch_stream(self.h)


class Server:
    """The serving loop (fsl_server_*): submit requests from any thread, wait
    for them, fetch their results.  The scheduler runs in the library."""

    def __init__(self, hbm_budget=None, device=-1, max_round_steps=8):
        self.L = _lib.load()
        c = _lib.ServerConfig()
        self.L.fsl_server_config_defaults(ctypes.byref(c))
        if hbm_budget is not None:
            c.hbm_budget = int(hbm_budget)
        c.device, c.max_round_steps = device, max_round_steps
        h = ctypes.c_void_p()
        check(self.L.fsl_server_create(ctypes.byref(c), ctypes.byref(h)))
        self.h = h
        self._np = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.fsl_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, config, q, nsteps):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(3, -1)
        rid = ctypes.c_int64()
        check(self.L.fsl_server_submit(self.h, ctypes.byref(config), q.shape[1], _dp(q), int(nsteps),
                                       ctypes.byref(rid)))
        self._np[rid.value] = q.shape[1]
        return rid.value

    @staticmethod
    def _info(i):
        return {f: getattr(i, f) for f, _ in _lib.RequestInfo._fields_}

    def poll(self, rid):
        i = _lib.RequestInfo()
        check(self.L.fsl_server_poll(self.h, int(rid), ctypes.byref(i)))
        return self._info(i)

    def wait(self, rid, timeout=-1.0):
        i = _lib.RequestInfo()
        check(self.L.fsl_server_wait(self.h, int(rid), float(timeout), ctypes.byref(i)))
        return self._info(i)

    def result(self, rid):
        n = self._np.pop(rid)
        q = np.empty((3, n))
        F = np.empty((3, n))
        check(self.L.fsl_server_result(self.h, int(rid), _dp(q), _dp(F)))
        return q, F

    def stats(self):
        st = _lib.ServerStats()
        check(self.L.fsl_server_get_stats(self.h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _lib.ServerStats._fields_}


def run_data_main(path):
    """Run `fluam data.main` for the stokesLimit scheme; raises on failure."""
    return check(_lib.load().fsl_run_data_main(str(path).encode()))


def parse_data_main(path):
    c = _lib.Config()
    ns, sf, rx, npart = (ctypes.c_int64() for _ in range(4))
    check(_lib.load().fsl_parse_data_main(str(path).encode(), ctypes.byref(c), ctypes.byref(ns),
                                          ctypes.byref(sf), ctypes.byref(rx), ctypes.byref(npart)))
    return c, {"numsteps": ns.value, "samplefreq": sf.value, "numstepsRelaxation": rx.value,
               "numberparticles": npart.value}
