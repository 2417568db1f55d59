"""ctypes binding of the FP64 CPU oracle (test infrastructure only).

Imported only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
leg, as the checker.  Arrays follow the oracle's layouts: particle arrays are
structure-of-arrays (3, np); fields are (3, mz, my, mx).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

PAIR_NONE, PAIR_TABLE_LJ, PAIR_SOFT = 0, 1, 2
RFD_REFERENCE, RFD_PAPER = 0, 1
SCHEME_MIDPOINT, SCHEME_FIRST_ORDER, SCHEME_QUASI2D, SCHEME_STOKES2D, SCHEME_INCOMPRESSIBLE = 0, 1, 2, 3, 4


def _config_struct(real_t):
    """orc_config with its floating-point fields of type real_t (c_double for
    the FP64 build, c_float for the FP32 one)."""
    class Cfg(ctypes.Structure):
        _fields_ = [
            ("mx", ctypes.c_int32), ("my", ctypes.c_int32), ("mz", ctypes.c_int32),
            ("kernel", ctypes.c_int32),
            ("lx", real_t), ("ly", real_t), ("lz", real_t),
            ("shearviscosity", real_t), ("temperature", real_t),
            ("dt", real_t), ("cutoff", real_t),
            ("extra_mobility", real_t), ("soft_epsilon", real_t),
            ("seed", ctypes.c_uint64),
            ("pair", ctypes.c_int32), ("rfd", ctypes.c_int32),
            ("nonbonded", ctypes.c_int32), ("scheme", ctypes.c_int32),
            ("ndrift", ctypes.c_int32), ("use_rfd", ctypes.c_int32),
            ("predictor_corrector", ctypes.c_int32), ("pad_", ctypes.c_int32),
            ("radius", real_t), ("saffman_kc", real_t),
            ("saffman_width", real_t), ("shear_amp", real_t),
            ("density", real_t),
        ]
    return Cfg


OrcConfig = _config_struct(ctypes.c_double)
_CONFIGS = {"f64": OrcConfig, "f32": _config_struct(ctypes.c_float)}
_REALS = {"f64": (ctypes.c_double, np.float64), "f32": (ctypes.c_float, np.float32)}

_lib = None
_libs = {}
_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int32)


def _build_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("_orc_build", os.path.join(HERE, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _load(real="f64", native=False):
    """The oracle library: FP64 (default) or the FP32 build of the same
    source, compiled portably or for this host (-march=native, built on first
    use)."""
    global _lib
    key = (real, bool(native))
    if key in _libs:
        return _libs[key]
    mod = None
    path = os.path.join(HERE, "liboracle_fsl" + ("_f32" if real == "f32" else "")
                        + ("_native" if native else "") + ".so")
    if native or not os.path.exists(path):
        mod = _build_module()
        path = mod.build_oracle(real=real, native=native)
    L = ctypes.CDLL(path)
    _D = ctypes.POINTER(_REALS[real][0])
    OrcConfig = _CONFIGS[real]
    vp = ctypes.c_void_p
    L.orc_create.restype = vp
    L.orc_create.argtypes = [ctypes.POINTER(OrcConfig), ctypes.c_int64, _D]
    L.orc_destroy.argtypes = [vp]
    L.orc_set_bonds.argtypes = [vp, ctypes.c_int64, _I, _I, _D, _D, ctypes.c_int64, _I, _D, _D, _D]
    L.orc_set_bonds_directed.argtypes = L.orc_set_bonds.argtypes
    L.orc_step.argtypes = [vp, ctypes.c_int64]
    L.orc_set_velocity.argtypes = [vp, _D]
    for name in ("orc_get_positions", "orc_set_positions", "orc_get_predictor",
                 "orc_get_forces", "orc_get_velocity"):
        getattr(L, name).argtypes = [vp, _D]
    L.orc_get_step.restype = ctypes.c_uint64
    L.orc_get_step.argtypes = [vp]
    L.orc_set_step.argtypes = [vp, ctypes.c_uint64]
    L.orc_noise.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int64, _D]
    L.orc_neighbor_grid.argtypes = [vp, _I]
    L.orc_cell_list.argtypes = [vp, _D, _I, _I, _I]
    L.orc_forces.argtypes = [vp, _D, _D]
    L.orc_spread.argtypes = [vp, _D, _D, _D]
    L.orc_solve.argtypes = [vp, _D, _D]
    L.orc_interp.argtypes = [vp, _D, _D, _D]
    L.orc_build_W.argtypes = [vp, _D, ctypes.c_int, _D]
    L.orc_fft3d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]
    L.orc_ljtable.argtypes = [vp, _F]
    L.orc_tex_linear.restype = ctypes.c_float
    L.orc_tex_linear.argtypes = [_F, ctypes.c_int, ctypes.c_float]
    L.orc_delta3.restype = _REALS[real][0]
    L.orc_delta3.argtypes = [_REALS[real][0]]
    L.orc_delta4.restype = _REALS[real][0]
    L.orc_delta4.argtypes = [_REALS[real][0]]
    L.orc_num_threads.restype = ctypes.c_int
    _libs[key] = L
    if key == ("f64", False):
        _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(_D)


def noise(seed, t, first, count):
    out = np.empty(count, dtype=np.float64)
    _load().orc_noise(seed, t, first, count, _dp(out))
    return out


def fft3d(a, sign):
    """Unnormalised 3-D DFT of a complex (mz, my, mx) array, sign -1 or +1."""
    z = np.ascontiguousarray(a, dtype=np.complex128).copy()
    mz, my, mx = z.shape
    _load().orc_fft3d(mx, my, mz, sign, z.ctypes.data_as(_D))
    return z


def delta3(x):
    return _load().orc_delta3(float(x))


def delta4(x):
    return _load().orc_delta4(float(x))


def tex_linear(table, x):
    t = np.ascontiguousarray(table, dtype=np.float32)
    return _load().orc_tex_linear(t.ctypes.data_as(_F), len(t), float(x))


def num_threads():
    return _load().orc_num_threads()


class Oracle:
    """One Stokes-limit instance on the CPU: FP64, or with real="f32" the FP32
    build of the same source (a timing baseline; the checker is FP64).
    native=True uses a build for this host's instruction set."""

    def __init__(self, mx, my, mz, lx, ly, lz, q, eta=1.0, kT=0.01, dt=0.01, cutoff=1.5,
                 kernel=3, pair=PAIR_SOFT, soft_epsilon=1.0, rfd=RFD_REFERENCE,
                 nonbonded=1, extra_mobility=0.0, seed=1, scheme=0, radius=1.0, ndrift=1,
                 use_rfd=1, predictor_corrector=0, saffman_kc=0.0, saffman_width=0.0,
                 shear_amp=0.0, density=1.0, real="f64", native=False):
        self.L = _load(real, native)
        self.real = np.dtype(_REALS[real][1])
        self._P = ctypes.POINTER(_REALS[real][0])
        OrcConfig = _CONFIGS[real]
        q = np.ascontiguousarray(q, dtype=self.real).reshape(3, -1)
        self.np = q.shape[1]
        self.shape = (mz, my, mx)
        self.nc = mx * my * mz
        c = OrcConfig(mx=mx, my=my, mz=mz, kernel=kernel, lx=lx, ly=ly, lz=lz,
                      shearviscosity=eta, temperature=kT, dt=dt, cutoff=cutoff,
                      extra_mobility=extra_mobility, soft_epsilon=soft_epsilon,
                      seed=seed, pair=pair, rfd=rfd, nonbonded=nonbonded, scheme=scheme,
                      ndrift=ndrift, use_rfd=use_rfd, predictor_corrector=predictor_corrector,
                      radius=radius, saffman_kc=saffman_kc, saffman_width=saffman_width,
                      shear_amp=shear_amp, density=density)
        self.cfg = c
        self.h = self.L.orc_create(ctypes.byref(c), self.np, self._p(q))
        if not self.h:
            raise ValueError("orc_create rejected the configuration")

    def _p(self, a):
        return a.ctypes.data_as(self._P)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.orc_destroy(h)
            self.h = None

    def set_bonds(self, bi, bj, k, r0, fi=None, fk=None, fr0=None, fxyz=None, directed=False):
        """Bonds (each acting on both particles), or with directed=True the
        entries of the old bond-file format (each acting on bi only)."""
        bi = np.ascontiguousarray(bi, dtype=np.int32)
        bj = np.ascontiguousarray(bj, dtype=np.int32)
        k = np.ascontiguousarray(k, dtype=self.real)
        r0 = np.ascontiguousarray(r0, dtype=self.real)
        if fi is None:
            fi = np.zeros(0, np.int32)
            fk = fr0 = np.zeros(0, self.real)
            fxyz = np.zeros((0, 3), self.real)
        fi = np.ascontiguousarray(fi, dtype=np.int32)
        fk = np.ascontiguousarray(fk, dtype=self.real)
        fr0 = np.ascontiguousarray(fr0, dtype=self.real)
        fxyz = np.ascontiguousarray(fxyz, dtype=self.real).reshape(-1, 3)
        fn = self.L.orc_set_bonds_directed if directed else self.L.orc_set_bonds
        rc = fn(self.h, len(bi), bi.ctypes.data_as(_I), bj.ctypes.data_as(_I),
                                  self._p(k), self._p(r0), len(fi), fi.ctypes.data_as(_I), self._p(fk),
                                  self._p(fr0), self._p(fxyz))
        if rc != 0:
            raise ValueError("bond index out of range")

    def step(self, n=1):
        self.L.orc_step(self.h, n)

    def positions(self):
        out = np.empty((3, self.np), self.real)
        self.L.orc_get_positions(self.h, self._p(out))
        return out

    def set_positions(self, q):
        q = np.ascontiguousarray(q, dtype=self.real).reshape(3, self.np)
        self.L.orc_set_positions(self.h, self._p(q))

    def predictor(self):
        out = np.empty((3, self.np), self.real)
        self.L.orc_get_predictor(self.h, self._p(out))
        return out

    def forces(self):
        out = np.empty((3, self.np), self.real)
        self.L.orc_get_forces(self.h, self._p(out))
        return out

    def set_velocity(self, v):
        """Initial velocity of the incompressible scheme, projected as the
        scheme does before its first step."""
        v = np.ascontiguousarray(v, dtype=self.real).reshape(3, self.nc)
        self.L.orc_set_velocity(self.h, self._p(v))

    def velocity(self):
        out = np.empty((3,) + self.shape, self.real)
        self.L.orc_get_velocity(self.h, self._p(out))
        return out

    @property
    def t(self):
        return int(self.L.orc_get_step(self.h))

    @t.setter
    def t(self, value):
        self.L.orc_set_step(self.h, int(value))

    def neighbor_grid(self):
        d = np.zeros(3, np.int32)
        m = self.L.orc_neighbor_grid(self.h, d.ctypes.data_as(_I))
        return tuple(int(x) for x in d), int(m)

    def cell_list(self, q):
        q = np.ascontiguousarray(q, dtype=self.real)
        (_, m) = self.neighbor_grid()
        cell_of = np.empty(self.np, np.int32)
        start = np.empty(m + 1, np.int32)
        srt = np.empty(self.np, np.int32)
        self.L.orc_cell_list(self.h, self._p(q), cell_of.ctypes.data_as(_I),
                             start.ctypes.data_as(_I), srt.ctypes.data_as(_I))
        return cell_of, start, srt

    def compute_forces(self, q):
        q = np.ascontiguousarray(q, dtype=self.real)
        F = np.empty((3, self.np), self.real)
        self.L.orc_forces(self.h, self._p(q), self._p(F))
        return F

    def spread(self, q, F):
        q = np.ascontiguousarray(q, dtype=self.real)
        F = np.ascontiguousarray(F, dtype=self.real)
        f = np.empty((3,) + self.shape, self.real)
        self.L.orc_spread(self.h, self._p(q), self._p(F), self._p(f))
        return f

    def solve(self, W):
        W = np.ascontiguousarray(W, dtype=self.real)
        v = np.empty((3,) + self.shape, self.real)
        self.L.orc_solve(self.h, self._p(W), self._p(v))
        return v

    def interp(self, q, v):
        q = np.ascontiguousarray(q, dtype=self.real)
        v = np.ascontiguousarray(v, dtype=self.real)
        u = np.empty((3, self.np), self.real)
        self.L.orc_interp(self.h, self._p(q), self._p(v), self._p(u))
        return u

    def build_W(self, f, second=False):
        f = np.ascontiguousarray(f, dtype=self.real)
        W = np.empty((3,) + self.shape, self.real)
        self.L.orc_build_W(self.h, self._p(f), 1 if second else 0, self._p(W))
        return W

    def ljtable(self):
        out = np.empty(4096, np.float32)
        self.L.orc_ljtable(self.h, out.ctypes.data_as(_F))
        return out
