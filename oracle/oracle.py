"""ctypes binding of the CPU oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

The oracle is a C++ FP64 restatement of the reference CLIP step (see clip_oracle.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it; the
product (clip_b200) never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

CASE = {"bubble": 0, "drop": 1, "rti": 2, "jet": 3}
PARAM_NAMES = ["RhoL", "RhoH", "sigma", "muH", "muL", "tauH", "tauL", "kConstant", "betaConstant",
               "mobility", "interfaceWidth", "referenceLength", "gx", "gy", "gz", "caseType"]


def build():
    """Compile liboracle.so if it is missing or older than its source."""
    src = os.path.join(HERE, "clip_oracle.cpp")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "oracle"], check=True, stdout=subprocess.DEVNULL)


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, cp, dp = ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [cp]
        L.orc_last_error.restype = cp
        L.orc_destroy.argtypes = [vp]
        for n in ("orc_dim", "orc_q"):
            getattr(L, n).argtypes = [vp]
            getattr(L, n).restype = ctypes.c_int
        L.orc_extent.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.orc_steps.argtypes = [vp]
        L.orc_steps.restype = ctypes.c_long
        L.orc_params.argtypes = [vp, dp]
        L.orc_bc.argtypes = [vp, ctypes.POINTER(ctypes.c_int), dp]
        L.orc_sdf.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_sdf.restype = ctypes.c_double
        L.orc_field_size.argtypes = [vp, cp]
        L.orc_field_size.restype = ctypes.c_long
        L.orc_get.argtypes = [vp, cp, dp]
        L.orc_set.argtypes = [vp, cp, dp]
        L.orc_initial_condition.argtypes = [vp]
        L.orc_device_initializer.argtypes = [vp]
        L.orc_solve.argtypes = [vp, ctypes.c_long]
        L.orc_mass.argtypes = [vp]
        L.orc_mass.restype = ctypes.c_double
        L.orc_threads.restype = ctypes.c_int
        _lib = L
    return _lib


class Oracle:
    """One reference-semantics FP64 solver on the host (ghosted AoS layout, x slowest)."""

    def __init__(self, config_path):
        L = lib()
        h = L.orc_create(os.fsencode(config_path))
        if not h:
            raise ValueError(L.orc_last_error().decode())
        self._h = h
        self.dim = L.orc_dim(h)
        self.Q = L.orc_q(h)
        e = (ctypes.c_int * 3)()
        L.orc_extent(h, e)
        self.extent = tuple(e)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    @property
    def steps(self):
        return lib().orc_steps(self._h)

    def params(self):
        out = (ctypes.c_double * len(PARAM_NAMES))()
        lib().orc_params(self._h, out)
        return dict(zip(PARAM_NAMES, list(out)))

    def boundary(self):
        t = (ctypes.c_int * 6)()
        v = (ctypes.c_double * 18)()
        lib().orc_bc(self._h, t, v)
        return list(t), np.array(v).reshape(6, 3)

    def sdf(self, x, y, z=0.0):
        return lib().orc_sdf(self._h, x, y, z)

    def ncomp(self, name):
        return {"c": 1, "p": 1, "rho": 1, "mu": 1, "vel": self.dim, "dc": self.dim, "normal": self.dim,
                "f": self.Q, "g": self.Q, "f_post": self.Q, "g_post": self.Q}[name]

    def get(self, name):
        n = lib().orc_field_size(self._h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        lib().orc_get(self._h, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out.reshape(list(self.extent) + [self.ncomp(name)])

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        if a.size != lib().orc_field_size(self._h, name.encode()):
            raise ValueError("size mismatch for " + name)
        lib().orc_set(self._h, name.encode(), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def initial_condition(self):
        lib().orc_initial_condition(self._h)

    def device_initializer(self):
        lib().orc_device_initializer(self._h)

    def init(self):
        self.initial_condition()
        self.device_initializer()

    def solve(self, nsteps=1):
        lib().orc_solve(self._h, int(nsteps))

    def mass(self):
        return lib().orc_mass(self._h)

    def interior(self, name):
        a = self.get(name)
        if self.dim == 2:
            return a[1:-1, 1:-1, :, :]
        return a[1:-1, 1:-1, 1:-1, :]


def threads():
    return lib().orc_threads()


def vts_text(dim, c, p, rho, vel):
    """The .vts text that the reference's VTSwriter::writeVTSBinaryFile writes
    (src/io/VTSwriter.cu:84-205) for fields in the reference layout (ghosted extent,
    arrays shaped [X][Y][Z][components]), restated in numpy.

    Interior nodes only (Domain.cu:22-82: indices 1..N per axis, z = 0 in 2D); points in
    k, j, i order with x fastest; every number printed as the reference's
    default-formatted std::ofstream prints a double (printf "%g", 6 significant digits);
    the arrays Velocity (DIM components), C, P, Rho in that order."""
    ex, ey, ez = c.shape[:3]
    lo = (1, 1, 1) if dim == 3 else (1, 1, 0)
    hi = (ex - 2, ey - 2, ez - 2) if dim == 3 else (ex - 2, ey - 2, 0)
    sl = tuple(slice(a, b + 1) for a, b in zip(lo, hi))
    ext = f"{lo[0]} {hi[0]} {lo[1]} {hi[1]} {lo[2]} {hi[2]}"

    def order(a):  # [X][Y][Z][comp] interior -> points (z, y, x) flattened, comp last
        a = np.asarray(a, dtype=np.float64)[sl]
        return a.transpose(2, 1, 0, 3).reshape(-1, a.shape[3])

    def rows(a):
        return "".join(" ".join("%g" % v for v in r) + "\n" for r in a.tolist())

    zz, yy, xx = np.meshgrid(np.arange(lo[2], hi[2] + 1), np.arange(lo[1], hi[1] + 1),
                             np.arange(lo[0], hi[0] + 1), indexing="ij")
    pts = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1).astype(np.float64)
    out = ['<?xml version="1.0"?>\n',
           '<VTKFile type="StructuredGrid" version="0.1" byte_order="LittleEndian">\n',
           f'<StructuredGrid WholeExtent="{ext}">\n', f'<Piece Extent="{ext}">\n',
           '<Points>\n<DataArray type="Float64" NumberOfComponents="3" format="ascii">\n', rows(pts),
           '</DataArray>\n</Points>\n', '<PointData Scalars="scalars" Vectors="velocity">\n',
           f'<DataArray type="Float64" Name="Velocity" NumberOfComponents="{dim}" format="ascii">\n',
           rows(order(vel)), '</DataArray>\n']
    for name, a in (("C", c), ("P", p), ("Rho", rho)):
        out += [f'<DataArray type="Float64" Name="{name}" format="ascii">\n', rows(order(a)), '</DataArray>\n']
    out += ['</PointData>\n', '</Piece>\n</StructuredGrid>\n</VTKFile>\n']
    return "".join(out)
