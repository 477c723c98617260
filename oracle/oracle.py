"""ctypes bindings of the checker libraries (TEST INFRASTRUCTURE ONLY).

``Oracle``  -> liblt_oracle.so, the C restatement in lt_oracle.c.
``RefLib``  -> _ref/libltref.so, the reference's own code (built here from the reference
               sources by oracle/Makefile; the built .so travels with the repository).

A catalogue is any object with the Potential_SOA arrays as attributes: ``type`` (int32)
and position_x, position_y, anglecos, anglesin, ellipticity_potential, rcore, rcut, b0,
dlsds (float64), sorted into runs of equal type.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_SO = HERE / "liblt_oracle.so"
ORACLE_LD_SO = HERE / "liblt_oracle_ld.so"
REF_SO = HERE / "_ref" / "libltref.so"


def reference_tree() -> pathlib.Path:
    """The reference source tree the checker library is built from: $LT_REFERENCE_TREE,
    else the default of the build recipe (oracle/Makefile, variable REF)."""
    env = os.environ.get("LT_REFERENCE_TREE")
    if env:
        return pathlib.Path(env)
    r = subprocess.run(["make", "-s", "--no-print-directory", "print-ref"], cwd=HERE, capture_output=True, text=True)
    return pathlib.Path(r.stdout.strip() or ".")


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(with_reference: bool | None = None) -> None:
    """Compile the oracle, and the reference library when the reference tree exists."""
    subprocess.run(["make", "-s", "oracle"], cwd=HERE, check=True)
    tree = reference_tree()
    if with_reference is None:
        with_reference = (tree / "src" / "gradient.cpp").exists()
    if with_reference:
        subprocess.run(["make", "-s", "ref", f"REF={tree}"], cwd=HERE, check=True)


def _d(a):
    return a.ctypes.data_as(_dp)


class _Cat(C.Structure):
    _fields_ = [("n", C.c_int), ("type", _ip)] + [(f, _dp) for f in
                                                ("x", "y", "cs", "sn", "eps", "rc", "rcut", "b0", "dlsds")]


class _Grid(C.Structure):
    _fields_ = [("xmin", C.c_double), ("ymin", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
                ("nx", C.c_int), ("ny", C.c_int), ("istart", C.c_int), ("jstart", C.c_int)]


def _arrays(cat):
    t = np.ascontiguousarray(cat.type, dtype=np.int32)
    fl = [np.ascontiguousarray(getattr(cat, f), dtype=np.float64) for f in
          ("position_x", "position_y", "anglecos", "anglesin", "ellipticity_potential", "rcore", "rcut", "b0",
           "dlsds")]
    return t, fl


# map kinds of lto_map()
MAP_KINDS = {"ampli1": 1, "ampli2": 2, "ampli3": 3, "ampli4": 4, "ampli5": 5, "ampli6": 6,
             "shear1": 11, "shear2": 12, "shear3": 13, "shear4": 14,
             "kappa": 21, "gamma1": 22, "gamma2": 23, "mu": 24, "scale": 25}


class Oracle:
    """The C restatement.  All results are float64 numpy arrays."""

    def __init__(self, path=ORACLE_SO, threads: int = 0):
        if not pathlib.Path(path).exists():
            build(with_reference=False)
        self.lib = C.CDLL(str(path))
        self.threads = threads or os.cpu_count()
        L = self.lib
        L.lto_grad_grid.argtypes = [C.POINTER(_Cat), C.POINTER(_Grid), _dp, _dp, C.c_int]
        L.lto_hess_grid.argtypes = [C.POINTER(_Cat), C.POINTER(_Grid), C.c_int, _dp, _dp, _dp, _dp, C.c_int]
        L.lto_pot_grid.argtypes = [C.POINTER(_Cat), C.POINTER(_Grid), _dp, C.c_int]
        L.lto_grad_points.argtypes = [C.POINTER(_Cat), C.c_long, _dp, _dp, _dp, _dp, C.c_int]
        L.lto_hess_points.argtypes = [C.POINTER(_Cat), C.c_long, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp, C.c_int]
        L.lto_pot_points.argtypes = [C.POINTER(_Cat), C.c_long, _dp, _dp, _dp, C.c_int]
        L.lto_map.argtypes = [C.c_int, C.c_long, _dp, _dp, _dp, C.c_double, C.c_double, _dp]
        L.lto_source_barycenters.argtypes = [C.POINTER(_Cat), C.c_int, _ip, _dp, _dp, _dp, _dp, _dp]
        L.lto_delense.argtypes = [C.c_int] + [C.c_double] * 4 + [_dp, _dp, C.c_int, _dp, _dp, _dp, _ip, _dp, _dp]
        L.lto_chi2_images.argtypes = [C.c_int, _ip, _dp, _dp, _ip, _dp, _dp, _ip]
        L.lto_chi2_images.restype = C.c_double

    def _cat(self, cat):
        t, fl = _arrays(cat)
        s = _Cat(int(t.shape[0]), t.ctypes.data_as(_ip), *[_d(a) for a in fl])
        return s, (t, fl)

    @staticmethod
    def _grid(g):
        return _Grid(g.xmin, g.ymin, g.dx, g.dy, g.nx, g.ny, g.istart, g.jstart)

    @staticmethod
    def _check(rc):
        if rc != 0:
            raise ValueError(f"oracle error {rc} (unknown profile type or bad argument)")

    def grad_grid(self, cat, g):
        s, keep = self._cat(cat)
        ax = np.empty(g.nx * g.ny); ay = np.empty(g.nx * g.ny)
        self._check(self.lib.lto_grad_grid(C.byref(s), C.byref(self._grid(g)), _d(ax), _d(ay), self.threads))
        return ax.reshape(g.ny, g.nx), ay.reshape(g.ny, g.nx)

    def hess_grid(self, cat, g, kmap=False):
        s, keep = self._cat(cat)
        out = [np.empty(g.nx * g.ny) for _ in range(4)]
        self._check(self.lib.lto_hess_grid(C.byref(s), C.byref(self._grid(g)), int(kmap), *[_d(o) for o in out],
                                           self.threads))
        return tuple(o.reshape(g.ny, g.nx) for o in out)

    def pot_grid(self, cat, g):
        s, keep = self._cat(cat)
        psi = np.empty(g.nx * g.ny)
        self._check(self.lib.lto_pot_grid(C.byref(s), C.byref(self._grid(g)), _d(psi), self.threads))
        return psi.reshape(g.ny, g.nx)

    def grad_points(self, cat, px, py):
        s, keep = self._cat(cat)
        px = np.ascontiguousarray(px, np.float64); py = np.ascontiguousarray(py, np.float64)
        ax = np.empty_like(px); ay = np.empty_like(px)
        self._check(self.lib.lto_grad_points(C.byref(s), px.size, _d(px), _d(py), _d(ax), _d(ay), self.threads))
        return ax, ay

    def hess_points(self, cat, px, py, kmap=False):
        s, keep = self._cat(cat)
        px = np.ascontiguousarray(px, np.float64); py = np.ascontiguousarray(py, np.float64)
        out = [np.empty_like(px) for _ in range(4)]
        self._check(self.lib.lto_hess_points(C.byref(s), px.size, _d(px), _d(py), int(kmap), *[_d(o) for o in out],
                                             self.threads))
        return tuple(out)

    def pot_points(self, cat, px, py):
        s, keep = self._cat(cat)
        px = np.ascontiguousarray(px, np.float64); py = np.ascontiguousarray(py, np.float64)
        psi = np.empty_like(px)
        self._check(self.lib.lto_pot_points(C.byref(s), px.size, _d(px), _d(py), _d(psi), self.threads))
        return psi

    def map(self, kind, a, b, c, D=1., scale=1.):
        a = np.ascontiguousarray(a, np.float64).ravel()
        b = np.ascontiguousarray(b, np.float64).ravel()
        c = np.ascontiguousarray(c, np.float64).ravel()
        out = np.empty_like(a)
        self._check(self.lib.lto_map(MAP_KINDS[kind], a.size, _d(a), _d(b), _d(c), D, scale, _d(out)))
        return out


    # ---- strong-lensing chi2 (systems: nimg int array, ix/iy concatenated images, dr
    # per system; frame = (xmin, xmax, ymin, ymax) of an n x n grid) ----
    MAXIMG = 20

    def source_barycenters(self, cat, nimg, ix, iy, dr):
        s, keep = self._cat(cat)
        nimg = np.ascontiguousarray(nimg, np.int32)
        ix, iy, dr = (np.ascontiguousarray(a, np.float64) for a in (ix, iy, dr))
        bx = np.empty(nimg.size); by = np.empty(nimg.size)
        self._check(self.lib.lto_source_barycenters(C.byref(s), nimg.size, nimg.ctypes.data_as(_ip), _d(ix), _d(iy),
                                                    _d(dr), _d(bx), _d(by)))
        return bx, by

    def delense(self, n, frame, ax, ay, bx, by, dr):
        """Predicted images (delense_barycenter order): (nfound[nsys], fx, fy[nsys, 20])."""
        ax, ay, bx, by, dr = (np.ascontiguousarray(a, np.float64).ravel() for a in (ax, ay, bx, by, dr))
        ns = bx.size
        nf = np.zeros(ns, np.int32)
        fx = np.zeros(ns * self.MAXIMG); fy = np.zeros(ns * self.MAXIMG)
        self._check(self.lib.lto_delense(n, *frame, _d(ax), _d(ay), ns, _d(bx), _d(by), _d(dr),
                                         nf.ctypes.data_as(_ip), _d(fx), _d(fy)))
        return nf, fx.reshape(ns, self.MAXIMG), fy.reshape(ns, self.MAXIMG)

    def chi2_images(self, nimg, ix, iy, nfound, fx, fy):
        nimg = np.ascontiguousarray(nimg, np.int32)
        nfound = np.ascontiguousarray(nfound, np.int32)
        ix, iy, fx, fy = (np.ascontiguousarray(a, np.float64).ravel() for a in (ix, iy, fx, fy))
        found = C.c_int()
        chi = self.lib.lto_chi2_images(nimg.size, nimg.ctypes.data_as(_ip), _d(ix), _d(iy),
                                       nfound.ctypes.data_as(_ip), _d(fx), _d(fy), C.byref(found))
        return chi, found.value

    def chi2(self, cat, frame, n, nimg, ix, iy, dr):
        """chi2 of one model: deflection grid, source barycentres, delensing, image matching."""
        from types import SimpleNamespace
        g = SimpleNamespace(xmin=frame[0], ymin=frame[2], dx=(frame[1] - frame[0]) / (n - 1),
                            dy=(frame[3] - frame[2]) / (n - 1), nx=n, ny=n, istart=0, jstart=0)
        ax, ay = self.grad_grid(cat, g)
        bx, by = self.source_barycenters(cat, nimg, ix, iy, dr)
        nf, fx, fy = self.delense(n, frame, ax, ay, bx, by, dr)
        chi, found = self.chi2_images(nimg, ix, iy, nf, fx, fy)
        return {"chi2": chi, "images_found": found, "nfound": nf, "fx": fx, "fy": fy, "bx": bx, "by": by}


class RefLib:
    """The reference's own CPU code (and GPU kernels compiled for the host)."""

    def __init__(self, path=REF_SO):
        if not pathlib.Path(path).exists():
            raise FileNotFoundError(f"{path} not built (oracle/Makefile target 'ref')")
        self.lib = C.CDLL(str(path))
        soa = [C.c_int, _ip] + [_dp] * 9
        L = self.lib
        L.ltref_grad_grid.argtypes = soa + [C.c_double] * 4 + [C.c_int] * 4 + [_dp, _dp]
        L.ltref_hess_grid.argtypes = soa + [C.c_double] * 4 + [C.c_int] * 4 + [_dp] * 4
        L.ltref_amplif5_grid.argtypes = soa + [C.c_double] * 4 + [C.c_int, _dp]
        L.ltref_grad_points.argtypes = soa + [C.c_long, _dp, _dp, _dp, _dp]
        L.ltref_hess_points.argtypes = soa + [C.c_long, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ltref_pot81_points.argtypes = soa + [C.c_long, _dp, _dp, _dp]
        L.ltref_gpu_kernel_grid.argtypes = [C.c_int] + soa + [C.c_double] * 4 + [C.c_int] * 4 + [_dp] * 4
        L.ltref_chi2.argtypes = soa + [C.c_double] * 4 + [C.c_int, C.c_int, _ip, _dp, _dp, _dp, _dp, _ip, _ip,
                                                          _dp, _dp]

    @staticmethod
    def _soa(cat):
        t, fl = _arrays(cat)
        # argument order of ref_wrap.cpp: x, y, cs, sn, eps, rc, rcut, b0, dlsds
        return [int(t.shape[0]), t.ctypes.data_as(_ip)] + [_d(a) for a in fl], (t, fl)

    def grad_grid(self, cat, g):
        s, keep = self._soa(cat)
        ax = np.empty(g.nx * g.ny); ay = np.empty(g.nx * g.ny)
        self.lib.ltref_grad_grid(*s, g.xmin, g.ymin, g.dx, g.dy, g.nx, g.ny, g.istart, g.jstart, _d(ax), _d(ay))
        return ax.reshape(g.ny, g.nx), ay.reshape(g.ny, g.nx)

    def hess_grid(self, cat, g):
        s, keep = self._soa(cat)
        out = [np.empty(g.nx * g.ny) for _ in range(4)]
        self.lib.ltref_hess_grid(*s, g.xmin, g.ymin, g.dx, g.dy, g.nx, g.ny, g.istart, g.jstart,
                                 *[_d(o) for o in out])
        return tuple(o.reshape(g.ny, g.nx) for o in out)

    def amplif5_grid(self, cat, g):
        s, keep = self._soa(cat)
        out = np.empty(g.nx * g.nx)
        self.lib.ltref_amplif5_grid(*s, g.xmin, g.xmax, g.ymin, g.ymax, g.nx, _d(out))
        return out.reshape(g.nx, g.nx)

    def grad_points(self, cat, px, py):
        s, keep = self._soa(cat)
        px = np.ascontiguousarray(px, np.float64); py = np.ascontiguousarray(py, np.float64)
        ax = np.empty_like(px); ay = np.empty_like(px)
        self.lib.ltref_grad_points(*s, px.size, _d(px), _d(py), _d(ax), _d(ay))
        return ax, ay

    def hess_points(self, cat, px, py):
        s, keep = self._soa(cat)
        px = np.ascontiguousarray(px, np.float64); py = np.ascontiguousarray(py, np.float64)
        out = [np.empty_like(px) for _ in range(4)]
        self.lib.ltref_hess_points(*s, px.size, _d(px), _d(py), *[_d(o) for o in out])
        return tuple(out)

    def pot81_points(self, cat, px, py):
        s, keep = self._soa(cat)
        px = np.ascontiguousarray(px, np.float64); py = np.ascontiguousarray(py, np.float64)
        psi = np.empty_like(px)
        rc = self.lib.ltref_pot81_points(*s, px.size, _d(px), _d(py), _d(psi))
        if rc:
            raise ValueError("the reference potential exists for type 81 only")
        return psi

    def gpu_kernel_grid(self, which, cat, g):
        """Run a reference GPU grid kernel on the host: which = 'pot', 'hess' or 'kmap'."""
        s, keep = self._soa(cat)
        out = [np.zeros(g.nx * g.ny) for _ in range(4)]
        code = {"pot": 0, "hess": 1, "kmap": 2}[which]
        self.lib.ltref_gpu_kernel_grid(code, *s, g.xmin, g.ymin, g.dx, g.dy, g.nx, g.ny, g.istart, g.jstart,
                                       *[_d(o) for o in out])
        if which == "pot":
            return out[0].reshape(g.ny, g.nx)
        return tuple(o.reshape(g.ny, g.nx) for o in out)

    def chi2(self, cat, frame, n, nimg, ix, iy, dr):
        """The reference's chi2 of one model (delense_barycenter + chi_computation)."""
        s, keep = self._soa(cat)
        nimg = np.ascontiguousarray(nimg, np.int32)
        ix, iy, dr = (np.ascontiguousarray(a, np.float64) for a in (ix, iy, dr))
        ns = nimg.size
        chi = C.c_double()
        found = C.c_int()
        nf = np.zeros(ns, np.int32)
        fx = np.zeros(ns * 20); fy = np.zeros(ns * 20)
        self.lib.ltref_chi2(*s, *frame, n, ns, nimg.ctypes.data_as(_ip), _d(ix), _d(iy), _d(dr), C.byref(chi),
                            C.byref(found), nf.ctypes.data_as(_ip), _d(fx), _d(fy))
        return {"chi2": chi.value, "images_found": found.value, "nfound": nf, "fx": fx.reshape(ns, 20),
                "fy": fy.reshape(ns, 20)}

    def bayes_rows(self, model, nhalos, free_flags, n_z_param, potfiles, pot_free, rows):
        """The reference's module_readParameters_setbayesmapmodels over `rows` in turn:
        halos 0..nhalos-1 are parameter-file halos (free_flags nhalos x 9 in the order
        x, y, epot, emass, theta, rcore, vdisp, rcut, z), the rest potfile galaxies, potfile
        after potfile.  Returns {x, y, b0, epot, cos, sin, rcore, rcut}, each nrows x ntot."""
        L = self.lib
        L.ltref_bayes_rows.argtypes = [C.c_int, C.c_int, _ip] + [_dp] * 9 + [_ip, C.c_int, C.c_int, _dp, _ip,
                                                                              C.c_int, C.c_int, _dp, _dp]
        t, x, y, ep, em, th, rc, vd, rcut, mag = model.arrays()
        ntot = model.n
        if mag is None:
            mag = np.zeros(ntot)
        ff = np.ascontiguousarray(free_flags, np.int32).reshape(nhalos, 9)
        pp = np.ascontiguousarray([[p.count, p.mag0, p.sigma, p.cut, p.core, p.vdslope, p.slope] for p in potfiles],
                                  np.float64).reshape(-1, 7)
        pfree = np.ascontiguousarray(pot_free, np.int32).reshape(-1, 2)
        rows = np.ascontiguousarray(rows, np.float64)
        nrows, nparam = rows.shape
        out = np.zeros((nrows, 8, ntot))
        st = L.ltref_bayes_rows(nhalos, ntot, t.ctypes.data_as(_ip), *[_d(a) for a in (x, y, ep, em, th, rc, vd, rcut,
                                                                                       mag)],
                                ff.ctypes.data_as(_ip), n_z_param, len(potfiles), _d(pp), pfree.ctypes.data_as(_ip),
                                nparam, nrows, _d(rows), _d(out))
        if st:
            raise RuntimeError(f"ltref_bayes_rows: {st}")
        keys = ("x", "y", "b0", "epot", "cos", "sin", "rcore", "rcut")
        return {k: out[:, i, :] for i, k in enumerate(keys)}


REF_GPU_SO = {"fp64": HERE / "_ref" / "libltref_gpu.so", "fp32": HERE / "_ref" / "libltref_gpu32.so",
              "fp64_stock": HERE / "_ref" / "libltref_gpu_stock.so",
              "fp32_stock": HERE / "_ref" / "libltref_gpu32_stock.so"}


class RefGpuLib:
    """The reference's own GPU kernels (src/gradient2_GPU.cu, src/potential_GPU.cu) built
    for sm_100a: "fp64_stock" with the flags of its default build (-O3 -use_fast_math,
    type_t = double), "fp32_stock" the same with type_t = float, and "fp64" / "fp32"
    with -O3 alone."""

    def __init__(self, build="fp64"):
        path = REF_GPU_SO[build]
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (oracle/Makefile target 'ref')")
        self.build = build
        self.lib = C.CDLL(str(path))
        self.lib.ltrefgpu_grid.argtypes = [C.c_int, C.c_int, _ip] + [_dp] * 8 + [C.c_double] * 4 + [C.c_int] * 3 + [
            _dp, _dp]

    def grid(self, which, cat, g, reps=1, want=True):
        """which 'hessian' (planes a, b, c, d) or 'potential'; returns (ms per launch, planes)."""
        w = {"hessian": 0, "potential": 1}[which]
        t = np.ascontiguousarray(cat.type, np.int32)
        fl = [np.ascontiguousarray(getattr(cat, f), np.float64) for f in (
            "position_x", "position_y", "anglecos", "anglesin", "ellipticity_potential", "rcore", "rcut", "b0")]
        npl = 4 if w == 0 else 1
        out = np.empty((npl, g.ny, g.nx)) if want else None
        ms = C.c_double()
        st = self.lib.ltrefgpu_grid(w, int(t.size), t.ctypes.data_as(_ip), *[_d(a) for a in fl], g.xmin, g.ymin,
                                    g.dx, g.dy, g.nx, g.ny, reps, C.byref(ms), _d(out) if want else None)
        if st:
            raise RuntimeError(f"ltrefgpu_grid: status {st}")
        return ms.value, out
