"""clip_b200 -- B200-native (sm_100a) lattice update of CLIP (mshadkhah/CLIP).

The compute path is libclipb.so (clip_b200/csrc, C ABI in include/clipb.h), called here
through ctypes with plain pointers.  There is no CPU fallback: if the library is missing
or no CUDA device is present, every entry point raises.

Two layers:
  * ``Solver``: one case (config.txt) on one GPU -- create, init, solve, fields, monitors.
  * Reference-shaped mirror: ``InputData``, ``Domain``, ``Geometry``, ``Boundary``,
    ``DataArray`` and ``NSAllen`` keep the call sequence of the reference's main loop
    (src/main.cu:53-89): construct, ``initialCondition()``, ``DataArray.updateDevice()``,
    ``deviceInitializer()``, then ``solve()`` per step and ``DataArray.updateHost()``.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclipb.so")

FP64, FP32, FP16 = 0, 1, 2
PRECISIONS = {"fp64": FP64, "fp32": FP32, "fp16": FP16}
FIELDS = {"c": 0, "p": 1, "rho": 2, "vel": 3, "f": 4, "g": 5, "f_post": 6, "g_post": 7}
PARAM_NAMES = ["RhoL", "RhoH", "sigma", "muH", "muL", "tauH", "tauL", "kConstant", "betaConstant",
               "mobility", "interfaceWidth", "referenceLength", "gx", "gy", "gz", "caseType"]
WORKLOADS = os.path.join(HERE, "workloads")


class ClipError(RuntimeError):
    """A libclipb call returned an error status."""

    def __init__(self, code, message):
        super().__init__(f"libclipb error {code}: {message}")
        self.code = code


class _Info(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("q", ctypes.c_int), ("precision", ctypes.c_int),
                ("extent", ctypes.c_int * 3), ("interior", ctypes.c_int * 3), ("steps", ctypes.c_longlong),
                ("device_bytes", ctypes.c_size_t), ("pop_scale", ctypes.c_double)]


_LIB = None

EXPORTS = ["clipb_config_summary", "clipb_create", "clipb_destroy", "clipb_last_error", "clipb_set_stream", "clipb_get_info",
           "clipb_get_params", "clipb_initial_condition", "clipb_device_initializer", "clipb_init", "clipb_init_device",
           "clipb_solve", "clipb_get_field", "clipb_get_fields", "clipb_get_field_device", "clipb_monitors",
           "clipb_time_steps", "clipb_set_launch", "clipb_get_launch", "clipb_autotune", "clipb_set_graphs",
           "clipb_set_wait_limit",
           "clipb_field_sums_noalloc", "clipb_batch_create", "clipb_batch_destroy", "clipb_batch_size",
           "clipb_batch_case", "clipb_batch_init", "clipb_batch_solve", "clipb_batch_solve_sequential",
           "clipb_batch_set_launch", "clipb_batch_get_launch", "clipb_batch_autotune", "clipb_batch_set_graphs",
           "clipb_batch_time_steps", "clipb_batch_monitors", "clipb_seeded_case_config", "clipb_save", "clipb_load",
           "clipb_set_params", "clipb_objective", "clipb_tangent", "clipb_adjoint", "clipb_get_intervals",
           "clipb_get_checkpoint_copies", "clipb_get_upload_bytes", "clipb_solve_monitored",
           "clipb_write_vts_async", "clipb_vts_wait", "clipb_write_vts", "clipb_slab_create", "clipb_slab_info",
           "clipb_slab_pack", "clipb_slab_unpack", "clipb_slab_step_part"]
VTS_FORMATS = {"ascii": 0, "binary64": 1, "binary32": 2}


def load_library(path=LIB_PATH):
    """Load libclipb.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python clip_b200/build.py`")
    L = ctypes.CDLL(path)
    vp, ip, dp, sz = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t
    L.clipb_create.argtypes = [ctypes.c_char_p, ip, ctypes.POINTER(vp)]
    L.clipb_destroy.argtypes = [vp]
    L.clipb_destroy.restype = None
    L.clipb_last_error.restype = ctypes.c_char_p
    L.clipb_set_stream.argtypes = [vp, vp]
    L.clipb_get_info.argtypes = [vp, ctypes.POINTER(_Info)]
    L.clipb_get_params.argtypes = [vp, dp]
    L.clipb_initial_condition.argtypes = [vp, dp]
    L.clipb_device_initializer.argtypes = [vp, dp]
    L.clipb_init.argtypes = [vp]
    L.clipb_init_device.argtypes = [vp]
    L.clipb_solve.argtypes = [vp, ip]
    L.clipb_get_field.argtypes = [vp, ip, dp, sz]
    L.clipb_get_fields.argtypes = [vp, dp, dp, dp, dp]
    L.clipb_get_field_device.argtypes = [vp, ip, vp, sz]
    L.clipb_monitors.argtypes = [vp, dp, dp]
    L.clipb_time_steps.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_float)]
    L.clipb_config_summary.argtypes = [ctypes.c_char_p, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip), dp]
    pi = ctypes.POINTER(ip)
    L.clipb_set_launch.argtypes = [vp, ip, ip]
    L.clipb_get_launch.argtypes = [vp, pi, pi, pi]
    L.clipb_autotune.argtypes = [vp, ip, pi, pi, ctypes.POINTER(ctypes.c_float)]
    L.clipb_set_graphs.argtypes = [vp, ip]
    L.clipb_set_wait_limit.argtypes = [vp, ctypes.c_longlong, ctypes.c_uint]
    fp = ctypes.POINTER(ctypes.c_float)
    L.clipb_batch_create.argtypes = [ctypes.POINTER(ctypes.c_char_p), ip, ip, ip, ctypes.POINTER(vp)]
    L.clipb_batch_destroy.argtypes = [vp]
    L.clipb_batch_destroy.restype = None
    L.clipb_batch_size.argtypes = [vp]
    L.clipb_batch_case.argtypes = [vp, ip, ctypes.POINTER(vp)]
    L.clipb_batch_init.argtypes = [vp]
    L.clipb_batch_solve.argtypes = [vp, ip]
    L.clipb_batch_solve_sequential.argtypes = [vp, ip]
    L.clipb_batch_set_launch.argtypes = [vp, ip, ip, ip]
    L.clipb_batch_get_launch.argtypes = [vp, pi, pi, pi, pi]
    L.clipb_batch_autotune.argtypes = [vp, ip, pi, pi, pi, fp]
    L.clipb_batch_set_graphs.argtypes = [vp, ip]
    L.clipb_batch_time_steps.argtypes = [vp, ip, ip, fp]
    L.clipb_batch_monitors.argtypes = [vp, dp, dp]
    L.clipb_seeded_case_config.argtypes = [ctypes.c_ulonglong, ip, ctypes.c_char_p, sz]
    L.clipb_save.argtypes = [vp, ctypes.c_char_p]
    L.clipb_load.argtypes = [vp, ctypes.c_char_p]
    L.clipb_set_params.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.clipb_objective.argtypes = [vp, dp, ip, dp, dp]
    L.clipb_tangent.argtypes = [vp, dp, ip, dp, dp, dp, dp, dp]
    L.clipb_adjoint.argtypes = [vp, dp, ip, dp, ip, dp, dp, dp]
    L.clipb_get_intervals.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.clipb_get_checkpoint_copies.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.clipb_get_upload_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.clipb_solve_monitored.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double)]
    L.clipb_write_vts_async.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ip]
    L.clipb_vts_wait.argtypes = [vp]
    L.clipb_write_vts.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ip]
    L.clipb_slab_create.argtypes = [ctypes.c_char_p, ip, ip, ip, ip, ctypes.POINTER(vp)]
    L.clipb_slab_info.argtypes = [vp, pi, pi, pi, pi, ctypes.POINTER(ctypes.c_longlong)]
    L.clipb_slab_pack.argtypes = [vp, ip, vp, vp]
    L.clipb_slab_unpack.argtypes = [vp, ip, vp, vp]
    L.clipb_slab_step_part.argtypes = [vp, ip]
    _LIB = L
    return L


def _check(rc):
    if rc != 0:
        raise ClipError(rc, load_library().clipb_last_error().decode())


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def config_summary(config_path):
    """Parse a config.txt on the host only: dim, reference extent, side codes, parameters."""
    L = load_library()
    dim = ctypes.c_int()
    ext = (ctypes.c_int * 3)()
    sides = (ctypes.c_int * 6)()
    par = np.empty(16, dtype=np.float64)
    _check(L.clipb_config_summary(os.fsencode(config_path), ctypes.byref(dim), ext, sides, _dptr(par)))
    return dict(dim=dim.value, extent=tuple(ext), sides=list(sides), params=dict(zip(PARAM_NAMES, par.tolist())))


class Solver:
    """One CLIP case on the current CUDA device (owner of all its device memory)."""

    def __init__(self, config_path, precision="fp64"):
        L = load_library()
        self._h = ctypes.c_void_p()
        self._owned = True
        prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        _check(L.clipb_create(os.fsencode(config_path), prec, ctypes.byref(self._h)))
        self.config_path = config_path
        self._describe()

    @classmethod
    def _borrow(cls, handle, owner):
        """A case of a Batch (the batch keeps ownership)."""
        s = cls.__new__(cls)
        s._h = handle
        s._owned = False
        s._owner = owner
        s.config_path = None
        s._describe()
        return s

    def _describe(self):
        info = self.info()
        self.dim, self.Q = info.dim, info.q
        self.extent = tuple(info.extent)
        self.interior = tuple(info.interior)
        self.precision = info.precision

    # lifetime --------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            if getattr(self, "_owned", True):
                load_library().clipb_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # queries ---------------------------------------------------------------------
    def info(self):
        i = _Info()
        _check(load_library().clipb_get_info(self._h, ctypes.byref(i)))
        return i

    @property
    def steps(self):
        return self.info().steps

    def params(self):
        out = np.empty(16, dtype=np.float64)
        _check(load_library().clipb_get_params(self._h, _dptr(out)))
        return dict(zip(PARAM_NAMES, out.tolist()))

    def intervals(self):
        """finalStep, outputInterval, reportInterval, checkpointInterval of the config."""
        out = (ctypes.c_longlong * 4)()
        _check(load_library().clipb_get_intervals(self._h, out))
        return dict(zip(("finalStep", "outputInterval", "reportInterval", "checkpointInterval"), list(out)))

    def ncomp(self, name):
        return {"c": 1, "p": 1, "rho": 1, "vel": self.dim}.get(name, self.Q)

    # stepping --------------------------------------------------------------------
    def initial_condition(self):
        c = np.empty(self.extent, dtype=np.float64)
        _check(load_library().clipb_initial_condition(self._h, _dptr(c)))
        return c

    def device_initializer(self, c=None):
        if c is None:
            _check(load_library().clipb_device_initializer(self._h, None))
        else:
            a = np.ascontiguousarray(c, dtype=np.float64)
            if a.size != int(np.prod(self.extent)):
                raise ValueError("initial c must cover the ghosted extent %s" % (self.extent,))
            _check(load_library().clipb_device_initializer(self._h, _dptr(a)))

    def init(self, on_device=False):
        """Initial state; on_device evaluates the initial field on the GPU (clipb_init_device)."""
        _check(load_library().clipb_init_device(self._h) if on_device else load_library().clipb_init(self._h))

    def upload_bytes(self):
        """Host-to-device bytes of the last initial-field upload (clipb_get_upload_bytes)."""
        n = ctypes.c_longlong()
        _check(load_library().clipb_get_upload_bytes(self._h, ctypes.byref(n)))
        return n.value

    def solve(self, nsteps=1):
        _check(load_library().clipb_solve(self._h, int(nsteps)))

    def solve_monitored(self, nsteps=1):
        """nsteps steps, then (mass, kinetic energy) of the state they leave, the reduction
        folded into the last step where the launch variant allows (clipb_solve_monitored)."""
        m, k = ctypes.c_double(), ctypes.c_double()
        _check(load_library().clipb_solve_monitored(self._h, int(nsteps), ctypes.byref(m), ctypes.byref(k)))
        return m.value, k.value

    def time_steps(self, nsteps):
        ms = ctypes.c_float()
        _check(load_library().clipb_time_steps(self._h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def set_stream(self, stream_ptr):
        _check(load_library().clipb_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def set_launch(self, variant, seg=0):
        _check(load_library().clipb_set_launch(self._h, int(variant), int(seg)))

    def get_launch(self):
        v, s, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(load_library().clipb_get_launch(self._h, ctypes.byref(v), ctypes.byref(s), ctypes.byref(n)))
        return v.value, s.value, n.value

    def autotune(self, trial_steps=4):
        """Pick the fastest launch shape on the freshly initialised state (which is rebuilt)."""
        v, s, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        _check(load_library().clipb_autotune(self._h, int(trial_steps), ctypes.byref(v), ctypes.byref(s),
                                             ctypes.byref(ms)))
        return v.value, s.value, ms.value

    def set_graphs(self, enable):
        _check(load_library().clipb_set_graphs(self._h, 1 if enable else 0))

    def set_wait_limit(self, cycles=0, inject_bytes=0):
        """Wait limit (SM cycles, 0 = default) of the staged step's bounded waits; inject_bytes
        makes the first bulk load of every block expect more bytes than arrive (test hook)."""
        _check(load_library().clipb_set_wait_limit(self._h, int(cycles), int(inject_bytes)))

    # data ------------------------------------------------------------------------
    def field(self, name, out=None):
        """Field in the reference layout, shape (E_x, E_y, E_z, ncomp)."""
        shape = self.extent + (self.ncomp(name),)
        if out is None:
            out = np.empty(shape, dtype=np.float64)
        _check(load_library().clipb_get_field(self._h, FIELDS[name], _dptr(out), out.size))
        return out

    def interior_field(self, name):
        a = self.field(name)
        return a[1:-1, 1:-1, :, :] if self.dim == 2 else a[1:-1, 1:-1, 1:-1, :]

    def field_device(self, name, dev_ptr, count):
        """Interior field (x fastest, components as planes) into a device buffer."""
        _check(load_library().clipb_get_field_device(self._h, FIELDS[name], ctypes.c_void_p(dev_ptr), count))

    def write_vts(self, folder="results", base_name="results", fmt="ascii", wait=True):
        """<folder>/<base_name>_t<steps>.vts of the current state (Velocity, C, P, Rho over
        the interior).  fmt: "ascii" (the reference's text file), "binary64" or "binary32"
        (raw appended arrays).  wait=False returns once the fields are packed on the GPU; the
        copy and the file write then overlap the following steps (see vts_wait)."""
        L = load_library()
        call = L.clipb_write_vts if wait else L.clipb_write_vts_async
        _check(call(self._h, os.fsencode(str(folder)), os.fsencode(str(base_name)), VTS_FORMATS[fmt]))
        return os.path.join(str(folder), f"{base_name}_t{self.steps}.vts")

    def vts_wait(self):
        """Wait for the queued VTS writes; raises on the first one that failed."""
        _check(load_library().clipb_vts_wait(self._h))

    def save(self, folder):
        """Checkpoint folder (reference CheckPointer files + libclipb's exact state)."""
        _check(load_library().clipb_save(self._h, os.fsencode(str(folder))))

    def load(self, folder):
        """Resume from a checkpoint folder written by save() or by the reference."""
        _check(load_library().clipb_load(self._h, os.fsencode(str(folder))))

    # derivatives (2D, FP64) ------------------------------------------------------
    def set_params(self, gy, sigma, mobility):
        """Body-force g_y, surface tension and mobility (derived parameters follow)."""
        _check(load_library().clipb_set_params(self._h, float(gy), float(sigma), float(mobility)))

    @staticmethod
    def _opt(a):
        if a is None:
            return None, None
        a = np.ascontiguousarray(a, dtype=np.float64)
        return a, _dptr(a)

    def objective(self, nsteps, target, c0=None):
        c0a, c0p = self._opt(c0)
        t = np.ascontiguousarray(target, dtype=np.float64)
        J = ctypes.c_double()
        _check(load_library().clipb_objective(self._h, c0p, int(nsteps), _dptr(t), ctypes.byref(J)))
        return J.value

    def tangent(self, nsteps, target, c0=None, dc0=None, dparams=None):
        """(J, dJ) of the tangent-linear model along (dc0, dparams = (d g_y, d sigma, d M))."""
        c0a, c0p = self._opt(c0)
        da, dpp = self._opt(dc0)
        pa, pp = self._opt(dparams)
        t = np.ascontiguousarray(target, dtype=np.float64)
        J, dJ = ctypes.c_double(), ctypes.c_double()
        _check(load_library().clipb_tangent(self._h, c0p, int(nsteps), _dptr(t), dpp, pp, ctypes.byref(J),
                                            ctypes.byref(dJ)))
        return J.value, dJ.value

    def adjoint(self, nsteps, target, c0=None, checkpoint_every=100):
        """(J, dJ/dc0 over the ghosted extent, dJ/d(g_y, sigma, M)) by the adjoint.
        checkpoint_every: steps between the checkpoints the forward states are recomputed
        from; >= nsteps keeps every state in one tape; 0 picks one tape when it takes at
        most half of the free device memory, else 100."""
        c0a, c0p = self._opt(c0)
        t = np.ascontiguousarray(target, dtype=np.float64)
        J = ctypes.c_double()
        g0 = np.empty(self.extent, dtype=np.float64)
        gp = np.empty(3, dtype=np.float64)
        _check(load_library().clipb_adjoint(self._h, c0p, int(nsteps), _dptr(t), int(checkpoint_every),
                                            ctypes.byref(J), _dptr(g0), _dptr(gp)))
        return J.value, g0, gp

    def monitors(self):
        m, k = ctypes.c_double(), ctypes.c_double()
        _check(load_library().clipb_monitors(self._h, ctypes.byref(m), ctypes.byref(k)))
        return m.value, k.value


def seeded_case_config(seed, index):
    """Config text of case `index` of the seeded batch workload (host only)."""
    L = load_library()
    n = L.clipb_seeded_case_config(seed, index, None, 0)
    if n < 0:
        _check(n)
    buf = ctypes.create_string_buffer(n + 1)
    L.clipb_seeded_case_config(seed, index, buf, n + 1)
    return buf.value.decode()


class Batch:
    """Many independent 2D cases advanced together by one persistent launch per step."""

    def __init__(self, configs, precision="fp32", texts=False):
        L = load_library()
        self._h = ctypes.c_void_p()
        prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        arr = (ctypes.c_char_p * len(configs))(*[c.encode() if texts else os.fsencode(c) for c in configs])
        _check(L.clipb_batch_create(arr, len(configs), 1 if texts else 0, prec, ctypes.byref(self._h)))
        self.precision = prec
        self.size = L.clipb_batch_size(self._h)

    @classmethod
    def seeded(cls, seed, ncases, precision="fp32"):
        return cls([seeded_case_config(seed, i) for i in range(ncases)], precision, texts=True)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            load_library().clipb_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def case(self, i):
        """Borrowed Solver view of case i (fields, monitors); valid while the batch lives."""
        h = ctypes.c_void_p()
        _check(load_library().clipb_batch_case(self._h, int(i), ctypes.byref(h)))
        return Solver._borrow(h, self)

    def init(self):
        _check(load_library().clipb_batch_init(self._h))

    def solve(self, nsteps=1):
        _check(load_library().clipb_batch_solve(self._h, int(nsteps)))

    def solve_sequential(self, nsteps=1):
        _check(load_library().clipb_batch_solve_sequential(self._h, int(nsteps)))

    def set_launch(self, variant, rows_per_item, blocks_per_sm=0):
        _check(load_library().clipb_batch_set_launch(self._h, int(variant), int(rows_per_item), int(blocks_per_sm)))

    def get_launch(self):
        v, r, b, n = (ctypes.c_int() for _ in range(4))
        _check(load_library().clipb_batch_get_launch(self._h, ctypes.byref(v), ctypes.byref(r), ctypes.byref(b),
                                                     ctypes.byref(n)))
        return v.value, r.value, b.value, n.value

    def autotune(self, trial_steps=4):
        v, r, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = ctypes.c_float()
        _check(load_library().clipb_batch_autotune(self._h, int(trial_steps), ctypes.byref(v), ctypes.byref(r),
                                                   ctypes.byref(b), ctypes.byref(ms)))
        return v.value, r.value, b.value, ms.value

    def set_graphs(self, enable):
        _check(load_library().clipb_batch_set_graphs(self._h, 1 if enable else 0))

    def time_steps(self, nsteps, sequential=False):
        ms = ctypes.c_float()
        _check(load_library().clipb_batch_time_steps(self._h, int(nsteps), 1 if sequential else 0, ctypes.byref(ms)))
        return ms.value

    def monitors(self):
        m = np.empty(self.size)
        k = np.empty(self.size)
        _check(load_library().clipb_batch_monitors(self._h, _dptr(m), _dptr(k)))
        return m, k


# ---------------------------------------------------------------- reference-shaped mirror
class InputData:
    """config.txt reader (reference: include/input/InputData.cuh:38-149)."""

    def __init__(self, filename="config.txt", precision="fp64"):
        self.filename = filename
        self.precision = precision

    def getConfig(self):
        return self.filename


class Domain:
    """Extent bookkeeping (reference: include/domain/Domain.cuh:30-112); filled by NSAllen."""

    def __init__(self, idata):
        self.idata = idata
        self.info = None


class Geometry:
    """Geometry list (reference: include/geometry/Geometry.cuh:39-208); parsed inside libclipb."""

    def __init__(self, idata):
        self.idata = idata


class Boundary:
    """Boundary list (reference: include/boundary/Boundary.cuh:48-190); parsed inside libclipb."""

    def __init__(self, idata, domain=None):
        self.idata = idata
        self.domain = domain


class DataArray:
    """Host copies of the output fields (reference: include/data/DataArray.cuh:62-293)."""

    def __init__(self, idata, domain=None, boundary=None):
        self.idata = idata
        self.solver = None
        self.hostDA = {}

    def createVectors(self):
        pass

    def updateDevice(self):
        """Upload of the host c happens in NSAllen.deviceInitializer (one call)."""

    def updateHost(self):
        s = self.solver
        self.hostDA = {k: s.field(k) for k in ("c", "p", "rho", "vel")}
        return self.hostDA


class NSAllen:
    """The solver facade (reference: include/equation/NsAllen.cuh:38-126)."""

    def __init__(self, idata, domain=None, DA=None, boundary=None, geom=None):
        self.solver = Solver(idata.getConfig(), idata.precision)
        self.DA = DA
        if DA is not None:
            DA.solver = self.solver
        if domain is not None:
            domain.info = dict(extent=self.solver.extent, interior=self.solver.interior, dim=self.solver.dim)
        self._host_c = None

    def initialCondition(self):
        self._host_c = self.solver.initial_condition()
        if self.DA is not None:
            self.DA.hostDA["c"] = self._host_c
        return self._host_c

    def deviceInitializer(self):
        c = self.DA.hostDA.get("c", self._host_c) if self.DA is not None else self._host_c
        self.solver.device_initializer(c)

    def solve(self):
        self.solver.solve(1)


class TimeInfo:
    """Step counter (reference: include/utils/TimeInfo.cuh:31-95); the solver counts steps."""

    def __init__(self, idata, solver=None):
        self.idata = idata
        self.solver = solver
        self._final = None

    def getCurrentStep(self):
        return self.solver.steps

    def getFinalStep(self):
        if self._final is None:
            self._final = self.solver.intervals()["finalStep"]
        return self._final

    def increment(self):
        """The solver advances its own step count in solve()."""


class VTSwriter:
    """Field output (reference: src/io/VTSwriter.cu:39-140): writeToFile() writes
    <folder>/<baseName>_t<step>.vts when step % outputInterval == 0.  The reference copies
    every field to the host on every call; here nothing leaves the GPU between outputs, and
    with fmt "binary64"/"binary32" the write is queued (copy and file write off the step
    path; call wait() before reading the files)."""

    def __init__(self, DA, idata, domain, ti, folder="results", baseName="results", fmt="ascii"):
        self.solver = ti.solver if ti is not None and ti.solver is not None else DA.solver
        self.folder = folder
        self.baseName = baseName
        self.fmt = fmt
        self.interval = self.solver.intervals()["outputInterval"]

    def writeToFile(self):
        step = self.solver.steps
        if self.interval > 0 and step % self.interval == 0:
            return self.solver.write_vts(self.folder, self.baseName, self.fmt, wait=self.fmt == "ascii")
        return None

    def wait(self):
        self.solver.vts_wait()
