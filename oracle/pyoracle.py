"""ORACLE -- test infrastructure only. ctypes access to

* ``oracle/lib/liboracle.so``: the plain-C restatement of the reference
  kernels and the uniform-mesh harness (oracle.c, harness.c), and
* ``oracle/_ref/libexaref{2d,3d}.so``: the reference's own generic kernels
  compiled from its sources (oracle/ref/Makefile), when present.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


def _pi(a):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_I)


class _Solver(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("order", ctypes.c_int), ("pde", ctypes.c_int), ("ps", ctypes.c_double * 6)]


# the point source of pde 4 (elastic waves with a Ricker-wavelet source on the
# normal stresses): position x0[3], delay t0, peak frequency f0, amplitude
DEFAULT_POINT_SOURCE = (0.5, 0.5, 0.5, 0.1, 8.0, 1.0)


def _ps6(point_source):
    ps = list(DEFAULT_POINT_SOURCE if point_source is None else point_source)
    assert len(ps) == 6
    return (ctypes.c_double * 6)(*[float(x) for x in ps])


def reference_root():
    """The reference checkout: $EXAHYPE_REFERENCE, else a directory named
    'reference' beside this repository; None when neither holds the
    reference's kernels."""
    for ref in (os.environ.get("EXAHYPE_REFERENCE"), os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")):
        if ref and os.path.isdir(os.path.join(ref, "ExaHyPE", "kernels")):
            return os.path.abspath(ref)
    return None


def build():
    """Builds liboracle.so (and oracle/_ref when the reference checkout exists)."""
    subprocess.check_call(["make", "-s", "-C", HERE])
    ref = reference_root()
    if ref:
        subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "ref"), "REF=" + ref])


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "lib", "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = ctypes.CDLL(path)
        _lib.orc_stable_dt.restype = ctypes.c_double
        _lib.orc_predictor.restype = ctypes.c_int
        _lib.orc_table.restype = _D
        if hasattr(_lib, "orc_mesh_time"):
            _lib.orc_mesh_time.restype = ctypes.c_double
            _lib.orc_mesh_dt.restype = ctypes.c_double
    return _lib


_ref = {}

# the timed builds of the reference kernels (oracle/ref/Makefile, target
# 'fast'): -O3 for the build host's CPU, for x86-64-v4 and for x86-64-v3, with
# the instruction-set flags each one needs from the CPU that runs it
_V3 = {"avx", "avx2", "fma", "bmi1", "bmi2", "movbe", "f16c", "abm", "xsave"}
_V4 = _V3 | {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}


def ref_available(dim=2):
    return os.path.exists(os.path.join(HERE, "_ref", "libexaref%dd.so" % dim))


def _cpu_flags(path="/proc/cpuinfo"):
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def fast_build(dim):
    """(path, name) of the fastest timed build of the reference kernels that
    this CPU can run, or (None, reason)."""
    d = os.path.join(HERE, "_ref", "fast")
    host = _cpu_flags()
    built_on = _cpu_flags(os.path.join(d, "build_host_cpuinfo.txt"))
    for name, need in (("native", built_on), ("x86-64-v4", _V4), ("x86-64-v3", _V3)):
        p = os.path.join(d, "libexaref%dd.%s.so" % (dim, name))
        if os.path.exists(p) and need and need <= host:
            return p, name
    return None, "no timed build of the reference kernels runs on this CPU (or none was built)"


def reflib(dim, fast=False):
    key = (dim, fast)
    if key not in _ref:
        path = fast_build(dim)[0] if fast else os.path.join(HERE, "_ref", "libexaref%dd.so" % dim)
        l = ctypes.CDLL(path)
        getattr(l, "ref%dd_stable_dt" % dim).restype = ctypes.c_double
        _ref[key] = l
    return _ref[key]


class Kernels:
    """Per-cell / per-face kernels of one (dim, order, pde), either the C
    restatement (impl='oracle') or the compiled reference (impl='ref')."""

    def __init__(self, dim, order, pde=0, impl="oracle", point_source=None):
        """point_source (pde 4): x0[3], t0, f0, amplitude"""
        self.dim, self.order, self.pde, self.impl = dim, order, pde, impl
        self.b = order + 1
        self.nvar = 9 if pde in (2, 4) else 5
        self.ndata = self.nvar + {1: 1, 2: 3, 3: 1, 4: 3}.get(pde, 0)
        self.P = self.b ** dim
        self.F = self.b ** (dim - 1)
        self.ps = _ps6(point_source)
        self._s = _Solver(dim, order, pde, self.ps)
        self._l = lib() if impl == "oracle" else reflib(dim, fast=impl == "ref_fast")
        self._pre = "orc_" if impl == "oracle" else "ref%dd_" % dim

    def _call(self, name, *args):
        f = getattr(self._l, self._pre + name)
        if self.impl == "oracle":
            return f(ctypes.byref(self._s), *args)
        return f(self.pde, self.order, *args)

    def predictor(self, luh, dx, dt, temps=False):
        b, P, F, d, nV, nD = self.b, self.P, self.F, self.dim, self.nvar, self.ndata
        luh = np.ascontiguousarray(luh, dtype=np.float64).reshape(-1)
        dx = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        qb = np.zeros(2 * d * F * nD)
        fb = np.zeros(2 * d * F * nV)
        du = np.zeros(P * nV)
        t = [np.zeros(P * b * nD), np.zeros(P * b * (d + 1) * nV), np.zeros(P * nD), np.zeros(P * (d + 1) * nV)]
        it = self._call("predictor", _p(luh), _p(dx), ctypes.c_double(dt), _p(qb), _p(fb), _p(du),
                        *[_p(x) for x in t])
        out = dict(lQhbnd=qb, lFhbnd=fb, lduh=du, iterations=it)
        if temps:
            out.update(lQi=t[0], lFi=t[1], lQhi=t[2], lFhi=t[3])
        return out

    def riemann(self, FL, FR, QL, QR, direction):
        FL = np.array(FL, dtype=np.float64).reshape(-1)
        FR = np.array(FR, dtype=np.float64).reshape(-1)
        QL = np.ascontiguousarray(QL, dtype=np.float64).reshape(-1)
        QR = np.ascontiguousarray(QR, dtype=np.float64).reshape(-1)
        if self.impl == "oracle":
            self._call("riemann", _p(FL), _p(FR), _p(QL), _p(QR), ctypes.c_int(direction))
        else:
            self._call("riemann", _p(FL), _p(FR), _p(QL), _p(QR), ctypes.c_double(0.0), ctypes.c_int(direction))
        return FL, FR

    def surface_integral(self, lduh, lFhbnd, dx):
        lduh = np.array(lduh, dtype=np.float64).reshape(-1)
        dx = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        self._call("surface_integral", _p(lduh), _p(np.ascontiguousarray(lFhbnd, dtype=np.float64).reshape(-1)),
                   _p(dx))
        return lduh

    def solution_update(self, luh, lduh, dt):
        luh = np.array(luh, dtype=np.float64).reshape(-1)
        self._call("solution_update", _p(luh), _p(np.ascontiguousarray(lduh, dtype=np.float64).reshape(-1)),
                   ctypes.c_double(dt))
        return luh

    def stable_dt(self, luh, dx):
        dx = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        return self._call("stable_dt", _p(np.ascontiguousarray(luh, dtype=np.float64).reshape(-1)), _p(dx))

    # linear kernels (oracle/linear.c; the reference's spaceTimePredictorLinear,
    # riemannSolverLinear, surfaceIntegralLinear, volumeIntegralLinear)
    def lin_predictor(self, luh, dx, dt):
        P, F, d, nV, nD = self.P, self.F, self.dim, self.nvar, self.ndata
        luh = np.ascontiguousarray(luh, dtype=np.float64).reshape(-1)
        dx = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        qb, fb = np.zeros(2 * d * F * nD), np.zeros(2 * d * F * nV)
        du, qh, fh = np.zeros(P * nV), np.zeros(P * nD), np.zeros(d * P * nV)
        self._call("lin_predictor", _p(luh), _p(dx), ctypes.c_double(dt), _p(qb), _p(fb), _p(du), _p(qh), _p(fh))
        return dict(lQhbnd=qb, lFhbnd=fb, lduh=du, lQhi=qh, lFhi=fh)

    def point_source(self, t, dt, centre, dx):
        """pointSource of the cell with the given centre and widths:
        PSi [b+1][b^d][nV]"""
        c = np.ascontiguousarray(np.resize(np.asarray(centre, dtype=np.float64), 3))
        dx = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        psi = np.zeros((self.b + 1) * self.P * self.nvar)
        if self.impl == "oracle":
            self._l.orc_point_source(ctypes.byref(self._s), ctypes.c_double(t), ctypes.c_double(dt), _p(c), _p(dx),
                                     _p(psi))
        else:
            getattr(self._l, self._pre + "point_source")(self.order, self.ps, ctypes.c_double(t), ctypes.c_double(dt),
                                                        _p(c), _p(dx), _p(psi))
        return psi.reshape(self.b + 1, self.P, self.nvar)

    def lin_predictor_at(self, luh, dx, dt, centre, t):
        """the linear predictor with point sources (usePointSource): the
        cell's pointSource at centre from t over [t, t + dt], then
        spaceTimePredictorLinear and volumeIntegralLinear"""
        P, F, d, nV, nD = self.P, self.F, self.dim, self.nvar, self.ndata
        luh = np.ascontiguousarray(luh, dtype=np.float64).reshape(-1)
        dx3 = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        c = np.ascontiguousarray(np.resize(np.asarray(centre, dtype=np.float64), 3))
        qb, fb = np.zeros(2 * d * F * nD), np.zeros(2 * d * F * nV)
        du, qh, fh = np.zeros(P * nV), np.zeros(P * nD), np.zeros(d * P * nV)
        if self.impl == "oracle":
            psi = np.ascontiguousarray(self.point_source(t, dt, centre, dx).reshape(-1))
            self._l.orc_lin_predictor_ps(ctypes.byref(self._s), _p(luh), _p(dx3), ctypes.c_double(dt), _p(psi),
                                         _p(qb), _p(fb), _p(du), _p(qh), _p(fh))
        else:
            getattr(self._l, self._pre + "lin_predictor_ps")(self.order, self.ps, _p(c), ctypes.c_double(t), _p(luh),
                                                            _p(dx3), ctypes.c_double(dt), _p(qb), _p(fb), _p(du),
                                                            _p(qh), _p(fh))
        return dict(lQhbnd=qb, lFhbnd=fb, lduh=du, lQhi=qh, lFhi=fh)

    def lin_riemann(self, QL, QR, direction):
        n = self.F * self.nvar
        FL, FR = np.zeros(n), np.zeros(n)
        QL = np.ascontiguousarray(QL, dtype=np.float64).reshape(-1)
        QR = np.ascontiguousarray(QR, dtype=np.float64).reshape(-1)
        if self.impl == "oracle":
            self._call("lin_riemann", _p(FL), _p(FR), _p(QL), _p(QR), ctypes.c_int(direction))
        else:
            self._call("lin_riemann", _p(FL), _p(FR), _p(QL), _p(QR), ctypes.c_double(0.0), ctypes.c_int(direction))
        return FL, FR

    def lin_boundary_face(self, FIn, QIn, face_index, kind=0):
        """boundary face of a linear solver (kind 0 outflow, 1 rigid wall):
        the cell's own fluctuation, returned as a new array"""
        FIn = np.array(FIn, dtype=np.float64).reshape(-1)
        QIn = np.ascontiguousarray(QIn, dtype=np.float64).reshape(-1)
        self._call("lin_boundary_face", _p(FIn), _p(QIn), ctypes.c_int(face_index), ctypes.c_int(kind))
        return FIn

    def lin_surface_integral(self, lduh, lFhbnd, dx):
        lduh = np.array(lduh, dtype=np.float64).reshape(-1)
        dx = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        self._call("lin_surface_integral", _p(lduh),
                   _p(np.ascontiguousarray(lFhbnd, dtype=np.float64).reshape(-1)), _p(dx))
        return lduh

    def lin_volume_integral(self, lFhi, dx):
        lduh = np.zeros(self.P * self.nvar)
        dx = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        self._call("lin_volume_integral", _p(lduh), _p(np.ascontiguousarray(lFhi, dtype=np.float64).reshape(-1)),
                   _p(dx))
        return lduh

    # limiter kernels of the C restatement (oracle/limiter.c); Euler only
    def fv_boundary(self, lim, face, kind=0):
        """FV ghost layers of a boundary face (boundaryLayerExtraction +
        boundaryConditions + ghostLayerFillingAtBoundary; kind 0 outflow, 1
        reflective); Euler, pde 0; returns the filled patch"""
        lim = np.array(lim, dtype=np.float64).reshape(-1)
        if self.impl == "oracle":
            self._l.orc_fv_boundary_fill_kind(ctypes.byref(self._s), _p(lim), ctypes.c_int(face), ctypes.c_int(kind))
        else:
            getattr(self._l, self._pre + "fv_boundary_kind")(self.order, _p(lim), ctypes.c_int(face),
                                                            ctypes.c_int(kind))
        return lim

    def fv_patch_size(self):
        E = 2 * self.order + 5
        return E ** self.dim * 5

    def project_fv(self, luh, lim=None):
        lim = np.zeros(self.fv_patch_size()) if lim is None else np.array(lim, dtype=np.float64).reshape(-1)
        self._l.orc_project_fv(ctypes.byref(self._s), _p(np.ascontiguousarray(luh, dtype=np.float64).reshape(-1)),
                               _p(lim))
        return lim

    def project_dg(self, lim):
        luh = np.zeros(self.P * 5)
        self._l.orc_project_dg(ctypes.byref(self._s), _p(np.ascontiguousarray(lim, dtype=np.float64).reshape(-1)),
                               _p(luh))
        return luh

    def musclhancock(self, lim_old, dx, dt):
        """MUSCL-Hancock update of one patch (ghost layers filled by the caller)"""
        old = np.ascontiguousarray(lim_old, dtype=np.float64).reshape(-1)
        new = old.copy()
        dx = np.ascontiguousarray(np.resize(np.asarray(dx, dtype=np.float64), 3))
        self._l.orc_musclhancock.restype = ctypes.c_double
        self._l.orc_musclhancock(ctypes.byref(self._s), _p(new), _p(old), _p(dx), ctypes.c_double(dt))
        return new

    def boundary_face(self, FIn, QIn, face_index, centre=(0.5, 0.5, 0.5), size=(0.1, 0.1, 0.1), t=0.0, dt=0.0,
                      kind=0):
        """kind 0: outflow values; 1: reflective walls (the demonstrator's
        boundaryValues; Euler, pde 0, for the reference's kernels)"""
        FIn = np.array(FIn, dtype=np.float64).reshape(-1)
        if kind == 1 and self.impl == "oracle":
            self._l.orc_boundary_face_reflective(ctypes.byref(self._s), _p(FIn),
                                                 _p(np.ascontiguousarray(QIn, dtype=np.float64).reshape(-1)),
                                                 ctypes.c_int(face_index))
            return FIn
        if kind == 1:
            assert self.pde == 0
            getattr(self._l, self._pre + "boundary_face_kind")(
                self.order, _p(FIn), _p(np.ascontiguousarray(QIn, dtype=np.float64).reshape(-1)),
                ctypes.c_int(face_index), ctypes.c_int(1))
            return FIn
        c = np.ascontiguousarray(np.resize(np.asarray(centre, dtype=np.float64), 3))
        s = np.ascontiguousarray(np.resize(np.asarray(size, dtype=np.float64), 3))
        self._call("boundary_face", _p(FIn), _p(np.ascontiguousarray(QIn, dtype=np.float64).reshape(-1)), _p(c),
                   _p(s), ctypes.c_double(t), ctypes.c_double(dt), ctypes.c_int(face_index))
        return FIn


def table(name, order):
    """Generated operator table (the same numbers the CUDA path uses)."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "exahype_b200", "csrc"))
    import gen_tables
    return np.array(gen_tables.build(order)[name])


class Mesh:
    """Uniform mesh run by the oracle harness (oracle/harness.c) over the C
    restatement (impl='oracle'), the compiled reference kernels (impl='ref',
    the parity build) or their timed -O3 build (impl='ref_fast')."""

    def __init__(self, dim, order, cells, size, bc, pde=0, impl="oracle", nthreads=1, point_source=None):
        """point_source (pde 4): x0[3], t0, f0, amplitude"""
        self.dim, self.order, self.pde, self.impl = dim, order, pde, impl
        ci = (ctypes.c_int * 3)(*(list(cells) + [1] * (3 - len(cells))))
        sz = (ctypes.c_double * 3)(*(list(size) + [1.0] * (3 - len(size))))
        if isinstance(bc, int):
            bc = [bc] * (2 * dim)
        b = (ctypes.c_int * 6)(*(list(bc) + [0] * (6 - len(bc))))
        if impl == "oracle":
            self._l = lib()
            self._pre = "orc_mesh_"
            create = self._l.orc_mesh_create
            create.restype = ctypes.c_void_p
            self._h = ctypes.c_void_p(create(dim, order, pde, ci, sz, b, nthreads))
        else:
            self._l = reflib(dim, fast=impl == "ref_fast")
            self._pre = "ref%dd_mesh_" % dim
            create = getattr(self._l, self._pre + "create")
            create.restype = ctypes.c_void_p
            self._h = ctypes.c_void_p(create(order, pde, ci, sz, b, nthreads))
        for nm, rt in (("time", ctypes.c_double), ("dt", ctypes.c_double), ("steps", ctypes.c_long),
                       ("sweeps", ctypes.c_long), ("run_until", ctypes.c_int)):
            getattr(self._l, self._pre + nm).restype = rt
        self.ncells = int(np.prod(cells))
        self.shape = (self.ncells, (order + 1) ** dim, {1: 6, 2: 12, 3: 6, 4: 12}.get(pde, 5))
        if pde == 4:
            self._f("set_point_source")(self._h, _ps6(point_source))

    def _f(self, nm):
        return getattr(self._l, self._pre + nm)

    def __del__(self):
        try:
            self._f("destroy")(self._h)
        except Exception:
            pass

    def set_solution(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.size == int(np.prod(self.shape))
        self._f("set_solution")(self._h, _p(u.reshape(-1)))

    def get_solution(self):
        u = np.empty(self.shape)
        self._f("get_solution")(self._h, _p(u.reshape(-1)))
        return u

    def init(self, t0=0.0):
        self._f("init")(self._h, ctypes.c_double(t0))

    def init_fused(self, t0=0.0, weight=0.99):
        """fused time stepping (the reference's fuse-algorithmic-steps) with
        the predictor-rerun weight"""
        self._f("init_fused")(self._h, ctypes.c_double(t0), ctypes.c_double(weight))

    def step(self, n=1):
        self._f("step")(self._h, int(n))

    def run_until(self, t_end, max_steps=10 ** 9):
        return self._f("run_until")(self._h, ctypes.c_double(t_end), int(max_steps))

    def state(self):
        return dict(t=self._f("time")(self._h), dt=self._f("dt")(self._h), steps=self._f("steps")(self._h),
                    picard_sweeps=self._f("sweeps")(self._h))

    def fused_state(self):
        f = self._f("predictor_dt")
        f.restype = ctypes.c_double
        g = self._f("reruns")
        g.restype = ctypes.c_long
        return dict(predictor_dt=f(self._h), reruns=g(self._h))


class RefinedMesh:
    """A periodic coarse grid with one box of coarse cells refined once (3^d
    fine cells each), stepped with global time steps by per-cell calls of the
    C restatement (impl='oracle') or of the compiled reference kernels
    (impl='ref'); small meshes only (a Python loop over cells and faces).

    Sequencing restated from the reference's traversals for such a mesh
    (exahype/solvers/ADERDGSolver.cpp): after the predictor of every cell,
    the refined coarse cells that face unrefined ones (ancestors) get their
    faces zeroed (prepareFaceDataOfAncestor :2300-2331) and the fine children's
    extrapolated states and fluxes restricted into them
    (restrictToTopMostParent :2465-2515, faceUnknownsRestriction); the
    virtual fine cells across the box's faces (descendants) get their coarse
    parent's face prolongated (prolongateFaceDataToDescendant :2334-2382,
    faceUnknownsProlongation). Riemann problems are solved for every pair of
    same-level neighbours of which one is a cell (solveRiemannProblemAtInterface
    :2789): coarse-coarse, coarse-ancestor, fine-fine and fine-descendant.
    Then surface integral, update and stable step of every cell with its own
    width; the step is the minimum over all cells.

    Cell order: the unrefined coarse cells (x fastest), then the box's fine
    cells (x fastest)."""

    def __init__(self, dim, order, cells, size, box_lo=None, box_hi=None, pde=0, impl="oracle", boxes=None, bc=-1,
                 level_boxes=None, point_source=None):
        """level_boxes: [(level, lo, hi)], the positions lo <= p < hi of that
        level refined once (several boxes per level refine their union);
        boxes: nested boxes, boxes[k] = (lo, hi) at level k; box_lo/box_hi:
        one box. bc: -1 periodic, 0 outflow or 1 reflective, one for all or
        per domain face (boundaryConditions on the level-0 cells' domain
        faces, ADERDGSolver.cpp:2893-2976)."""
        self.dim, self.order, self.pde = dim, order, pde
        self.linear = pde in (2, 4)
        self.K = Kernels(dim, order, pde, impl, point_source=point_source)
        self.impl = impl
        self._args = (dim, order, cells, size, pde, impl, bc)
        self._point_source = point_source
        d = dim
        cells = list(cells)[:d]
        if level_boxes is None:
            nest = boxes if boxes is not None else [(box_lo, box_hi)]
            level_boxes = [(k, lo, hi) for k, (lo, hi) in enumerate(nest)]
        level_boxes = [(int(l), list(lo)[:d], list(hi)[:d]) for l, lo, hi in level_boxes]
        L = max([b[0] + 2 for b in level_boxes] + [1])
        self.dxl = [[size[i] / cells[i] for i in range(d)]]  # a child's width: its parent's / 3
        for lev in range(1, L):
            self.dxl.append([x / 3.0 for x in self.dxl[-1]])
        bcs = [bc] * (2 * d) if isinstance(bc, int) else list(bc)
        box_pos = lambda lo, hi, s=1: [tuple(s * lo[i] + t[d - 1 - i] for i in range(d))  # noqa: E731
                                       for t in np.ndindex(*[s * (hi[i] - lo[i]) for i in reversed(range(d))])]
        # state per level: position -> 1 (cell) or 2 (refined)
        state = [dict() for _ in range(L)]
        for c in box_pos([0] * d, cells):
            state[0][c] = 1
        for lev, lo, hi in level_boxes:
            for c in box_pos(lo, hi, 3):
                state[lev + 1][c] = 1
        for lev, lo, hi in level_boxes:
            for c in box_pos(lo, hi):
                state[lev][c] = 2

        def nbr(lev, c, i, s):
            q = list(c)
            q[i] += 1 if s else -1
            if lev == 0 and bcs[2 * i] == -1:
                q[i] %= cells[i]
            return tuple(q)

        self.lstate = state
        order_key = lambda c: tuple(reversed(c))  # noqa: E731  x fastest
        self.cid = [dict() for _ in range(L)]
        self.level = []
        n = 0
        for lev in range(L):
            for c in sorted(state[lev], key=order_key):
                if state[lev][c] == 1:
                    self.cid[lev][c] = n
                    self.level.append(lev)
                    n += 1
        self.ncells = n
        # cell centres (point sources): position p at level l spans
        # [p dx_l, (p + 1) dx_l]
        self.centre = np.zeros((n, 3))
        for lev in range(L):
            for c, i in self.cid[lev].items():
                for e in range(d):
                    self.centre[i, e] = c[e] * self.dxl[lev][e] + 0.5 * self.dxl[lev][e]
        self.aid = [dict() for _ in range(L)]
        for lev in range(L - 1):
            for c in sorted(state[lev], key=order_key):
                if state[lev][c] == 2 and any(state[lev].get(nbr(lev, c, i, s)) == 1 for i in range(d) for s in (0, 1)):
                    self.aid[lev][c] = n
                    n += 1
        slot = lambda lev, c: self.cid[lev].get(c, self.aid[lev].get(c, -1))  # noqa: E731
        self.pairs, self.restr, self.prol, self.bnd = [], [], [], []
        for lev in range(L):
            for c in sorted(state[lev], key=order_key):
                sc = state[lev][c]
                me = slot(lev, c)
                for i in range(d):
                    q = nbr(lev, c, i, 1)
                    sq = state[lev].get(q, 0)
                    if sq and not (sc == 2 and sq == 2):
                        self.pairs.append((me, slot(lev, q), i))
                    if sc != 1:
                        continue
                    for side in (0, 1):
                        r = nbr(lev, c, i, side)
                        if state[lev].get(r, 0):
                            continue
                        face = 2 * i + side
                        if lev == 0:
                            self.bnd.append((me, face, bcs[face]))
                            continue
                        sub = [c[e] % 3 for e in range(d) if e != i]
                        desc = n
                        n += 1
                        self.pairs.append((desc, me, i) if side == 0 else (me, desc, i))
                        self.restr.append((me, face, self.aid[lev - 1][tuple(x // 3 for x in c)], face, sub))
                        dface = 2 * i + 1 - side
                        self.prol.append((self.cid[lev - 1][tuple(x // 3 for x in r)], dface, desc, dface, sub))
        nslot = n
        K = self.K
        self.nslot = nslot
        self.Q = np.zeros((nslot, 2 * d, K.F * K.ndata))
        self.Fb = np.zeros((nslot, 2 * d, K.F * K.nvar))
        self.u = np.zeros((self.ncells, K.P, K.ndata))
        self.du = np.zeros((self.ncells, K.P * K.nvar))
        self.t, self.dt, self.steps, self.sweeps = 0.0, 0.0, 0, 0

    def _dx(self, c):
        return self.dxl[self.level[c]]

    def regrid(self, level_boxes):
        """static AMR between steps, restating exa_mesh_regrid's data
        transfer with the reference's AMR operators: a cell that stays keeps
        its data, a new cell inside a coarser old cell gets that cell's
        volume prolongation, one covering finer old cells the sum of their
        volume restrictions (ADERDGSolver.cpp:1437-1470,1694-1735); t and the
        step count are kept, the step size recomputed, the predictor rerun"""
        dim, order, cells, size, pde, impl, bc = self._args
        new = RefinedMesh(dim, order, cells, size, pde=pde, impl=impl, bc=bc, level_boxes=level_boxes,
                          point_source=self._point_source)
        K, d = self.K, self.dim
        npar = K.ndata - K.nvar
        old_pos = [None] * self.ncells
        for lev, ids in enumerate(self.cid):
            for c, i in ids.items():
                old_pos[i] = (lev, c)
        oldL = len(self.lstate)
        for lev, ids in enumerate(new.cid):
            for p, i in ids.items():
                lv = min(lev, oldL - 1)
                a = tuple(x // 3 ** (lev - lv) for x in p)
                while lv > 0 and self.lstate[lv].get(a, 0) == 0:
                    lv -= 1
                    a = tuple(x // 3 for x in a)
                sa = self.lstate[lv][a]
                if sa == 1 and lv == lev:
                    new.u[i] = self.u[self.cid[lv][a]]
                elif sa == 1:
                    ld = lev - lv
                    sub = [p[e] - a[e] * 3 ** ld for e in range(d)]
                    new.u[i] = amr("volume_prolongation", d, order, K.nvar, npar, ld, sub,
                                   coarse=self.u[self.cid[lv][a]], impl=impl).reshape(new.u[i].shape)
                else:
                    acc = np.zeros(new.u[i].size)
                    for j, (l2, q) in enumerate(old_pos):
                        if l2 <= lev or any(q[e] // 3 ** (l2 - lev) != p[e] for e in range(d)):
                            continue
                        sub = [q[e] - p[e] * 3 ** (l2 - lev) for e in range(d)]
                        acc = amr("volume_restriction", d, order, K.nvar, npar, l2 - lev, sub, coarse=acc,
                                  fine=self.u[j], impl=impl)
                    new.u[i] = acc.reshape(new.u[i].shape)
        new.t, new.steps, new.sweeps = self.t, self.steps, self.sweeps
        new.fused = False
        new.dt = new._stable()
        new._predict()
        self.__dict__.update(new.__dict__)

    def set_solution(self, u):
        self.u = np.array(u, dtype=np.float64).reshape(self.u.shape)

    def get_solution(self):
        return self.u.copy()

    def _stable(self):
        return min(self.K.stable_dt(self.u[c], self._dx(c)) for c in range(self.ncells))

    def _predict(self, dt=None, t=None):
        """t: time stamp of the solution the predictor starts from (point
        sources)"""
        K, d = self.K, self.dim
        dt = self.dt if dt is None else dt
        t = self.t if t is None else t
        for c in range(self.ncells):
            if self.pde == 4:
                o = K.lin_predictor_at(self.u[c], self._dx(c), dt, self.centre[c], t)
            elif self.linear:
                o = K.lin_predictor(self.u[c], self._dx(c), dt)
            else:
                o = K.predictor(self.u[c], self._dx(c), dt)
                self.sweeps += int(o["iterations"])
            self.Q[c] = o["lQhbnd"].reshape(2 * d, -1)
            self.Fb[c] = o["lFhbnd"].reshape(2 * d, -1)
            self.du[c] = o["lduh"]
        for a in set(x[2] for x in self.restr):
            self.Q[a] = 0.0
            self.Fb[a] = 0.0
        for f, face, a, aface, sub in self.restr:
            q, fl = amr("face_restriction", d, self.order, K.nvar, K.ndata - K.nvar, 1, sub, coarse=self.Q[a, aface],
                        fine=self.Q[f, face], coarse_flux=self.Fb[a, aface], fine_flux=self.Fb[f, face],
                        impl=self.impl)
            self.Q[a, aface], self.Fb[a, aface] = q, fl
        for c, face, dsl, dface, sub in self.prol:
            q, fl = amr("face_prolongation", d, self.order, K.nvar, K.ndata - K.nvar, 1, sub,
                        coarse=self.Q[c, face], coarse_flux=self.Fb[c, face], impl=self.impl)
            self.Q[dsl, dface], self.Fb[dsl, dface] = q, fl

    def init(self, t0=0.0):
        self.t, self.steps, self.sweeps = t0, 0, 0
        self.fused = False
        self.dt = self._stable()
        self._predict()

    def init_fused(self, t0=0.0, weight=0.99):
        """fused time stepping, restating oracle/harness.c hrn_init_fused /
        hrn_step_fused (the reference's fuse-algorithmic-steps): the
        predictor runs right after the update with its own step estimate"""
        self.t, self.steps, self.sweeps, self.reruns = t0, 0, 0, 0
        self.fused, self.w = True, weight
        s0 = self._stable()
        self.dt = self.pdt = s0
        self.tp = t0 + s0
        self._predict(self.pdt)

    def fused_state(self):
        return dict(predictor_dt=self.pdt, reruns=self.reruns)

    def _update(self):
        K = self.K
        for l, r, i in self.pairs:
            if self.linear:
                fl, fr = K.lin_riemann(self.Q[l, 2 * i + 1], self.Q[r, 2 * i], i)
            else:
                fl, fr = K.riemann(self.Fb[l, 2 * i + 1], self.Fb[r, 2 * i], self.Q[l, 2 * i + 1],
                                   self.Q[r, 2 * i], i)
            self.Fb[l, 2 * i + 1], self.Fb[r, 2 * i] = fl, fr
        bf = K.lin_boundary_face if self.linear else K.boundary_face
        for c, face, kind in self.bnd:
            self.Fb[c, face] = bf(self.Fb[c, face], self.Q[c, face], face, kind=kind)
        for c in range(self.ncells):
            si = K.lin_surface_integral if self.linear else K.surface_integral
            du = si(self.du[c], self.Fb[c].reshape(-1), self._dx(c))
            self.u[c] = K.solution_update(self.u[c], du, self.dt).reshape(self.u[c].shape)

    def _step_fused(self):
        self._update()
        s = self._stable()
        self._predict(self.pdt, t=self.tp)
        nxt = s
        used = s if self.pdt == 0.0 else self.pdt
        unstable = used > s
        if unstable:
            ws = self.w * s
            nxt = min(nxt, ws)
            self.pdt = ws
        else:
            nxt = min(nxt, 0.5 * (used + self.w * s))
        self.t = self.tp
        self.dt = self.pdt
        self.tp = self.tp + self.pdt
        self.pdt = nxt
        self.steps += 1
        if unstable:
            self.reruns += 1
            self._predict(self.pdt)

    def step(self, n=1):
        for _ in range(n):
            if getattr(self, "fused", False):
                self._step_fused()
                continue
            self._update()
            self.t += self.dt
            self.steps += 1
            self.dt = self._stable()
            self._predict()

    def state(self):
        return dict(t=self.t, dt=self.dt, steps=self.steps, picard_sweeps=self.sweeps)


class LimitingMesh:
    """Uniform mesh with the a-posteriori subcell limiter, run by the oracle's
    limiting harness (oracle/limiting_harness.c) over the C restatement."""

    def __init__(self, dim, order, cells, size, bc, helper_layers=1, cure_steps=0, relax=1e-4, scale=1e-3,
                 nthreads=1):
        self.dim, self.order = dim, order
        l = lib()
        ci = (ctypes.c_int * 3)(*(list(cells) + [1] * (3 - len(cells))))
        sz = (ctypes.c_double * 3)(*(list(size) + [1.0] * (3 - len(size))))
        if isinstance(bc, int):
            bc = [bc] * (2 * dim)
        b = (ctypes.c_int * 6)(*(list(bc) + [0] * (6 - len(bc))))
        l.orc_lmesh_create.restype = ctypes.c_void_p
        for nm, rt in (("time", ctypes.c_double), ("dt", ctypes.c_double), ("steps", ctypes.c_long),
                       ("sweeps", ctypes.c_long), ("run_until", ctypes.c_int), ("irregular_steps", ctypes.c_long)):
            getattr(l, "orc_lmesh_" + nm).restype = rt
        self._l = l
        self._h = ctypes.c_void_p(l.orc_lmesh_create(dim, order, ci, sz, b, nthreads, helper_layers, cure_steps,
                                                     ctypes.c_double(relax), ctypes.c_double(scale)))
        self.ncells = int(np.prod(cells))
        self.shape = (self.ncells, (order + 1) ** dim, 5)

    def __del__(self):
        try:
            self._l.orc_lmesh_destroy(self._h)
        except Exception:
            pass

    def set_solution(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self._l.orc_lmesh_set_solution(self._h, _p(u.reshape(-1)))

    def get_solution(self):
        u = np.empty(self.shape)
        self._l.orc_lmesh_get_solution(self._h, _p(u.reshape(-1)))
        return u

    def set_fv_initial(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        self._l.orc_lmesh_set_fv_initial(self._h, _p(v.reshape(-1)))

    def init(self, t0=0.0):
        self._l.orc_lmesh_init(self._h, ctypes.c_double(t0))

    def step(self, n=1):
        self._l.orc_lmesh_step(self._h, int(n))

    def run_until(self, t_end, max_steps=10 ** 9):
        return self._l.orc_lmesh_run_until(self._h, ctypes.c_double(t_end), int(max_steps))

    def status(self):
        s = np.empty(self.ncells, dtype=np.int32)
        self._l.orc_lmesh_status(self._h, _pi(s))
        return s

    def limiter(self):
        """(FV patches (ncells, E^d, 5) incl. ghost layers, allocated flags)"""
        B = 2 * self.order + 1
        lim = np.empty((self.ncells, (B + 4) ** self.dim, 5))
        al = np.empty(self.ncells, dtype=np.int32)
        self._l.orc_lmesh_limiter(self._h, _p(lim.reshape(-1)), _pi(al))
        return lim, al

    def state(self):
        f = self._l
        return dict(t=f.orc_lmesh_time(self._h), dt=f.orc_lmesh_dt(self._h), steps=f.orc_lmesh_steps(self._h),
                    picard_sweeps=f.orc_lmesh_sweeps(self._h), irregular_steps=f.orc_lmesh_irregular_steps(self._h))


class RefLimitingMesh(LimitingMesh):
    """The limiting harness over the reference's own kernels (oracle/_ref; the
    timed -O3 build with fast=True)."""

    def __init__(self, dim, order, cells, size, bc, helper_layers=1, cure_steps=0, relax=1e-4, scale=1e-3,
                 nthreads=1, fast=False):
        self.dim, self.order = dim, order
        l = reflib(dim, fast=fast)
        pre = "ref%dd_lmesh_" % dim
        ci = (ctypes.c_int * 3)(*(list(cells) + [1] * (3 - len(cells))))
        sz = (ctypes.c_double * 3)(*(list(size) + [1.0] * (3 - len(size))))
        if isinstance(bc, int):
            bc = [bc] * (2 * dim)
        b = (ctypes.c_int * 6)(*(list(bc) + [0] * (6 - len(bc))))
        getattr(l, pre + "create").restype = ctypes.c_void_p
        for nm, rt in (("time", ctypes.c_double), ("dt", ctypes.c_double), ("steps", ctypes.c_long),
                       ("sweeps", ctypes.c_long), ("run_until", ctypes.c_int), ("irregular_steps", ctypes.c_long)):
            getattr(l, pre + nm).restype = rt
        self._l = _Prefixed(l, pre)
        self._h = ctypes.c_void_p(getattr(l, pre + "create")(order, ci, sz, b, nthreads, helper_layers, cure_steps,
                                                           ctypes.c_double(relax), ctypes.c_double(scale)))
        self.ncells = int(np.prod(cells))
        self.shape = (self.ncells, (order + 1) ** dim, 5)


class _Prefixed:
    """maps orc_lmesh_<name> to <prefix><name> of another library"""

    def __init__(self, lib, prefix):
        self._lib, self._pre = lib, prefix

    def __getattr__(self, name):
        return getattr(self._lib, self._pre + name.replace("orc_lmesh_", ""))


# ---- AMR transfer operators and the plotter's vertex projection ---------------
AMR_OPS = {"volume_prolongation": 0, "volume_restriction": 1, "face_prolongation": 2, "face_restriction": 3}


def amr(op, dim, N, nvar, npar, levelDelta, index, coarse=None, fine=None, coarse_flux=None, fine_flux=None,
        impl="oracle"):
    """One AMR transfer of the C restatement (impl='oracle') or of the
    reference's amrRoutines (impl='ref'). Volume data [b^d][nvar+npar], face
    states [b^(d-1)][nvar+npar] and fluxes [b^(d-1)][nvar]. Prolongations
    return the fine data (state, flux for faces); restrictions return the
    coarse data plus the restriction (the inputs `coarse`, `coarse_flux`
    are what is added to)."""
    b = N + 1
    nd = nvar + npar
    vol, face = b ** dim * nd, b ** (dim - 1) * nd
    ff = b ** (dim - 1) * nvar
    idx = (ctypes.c_int * 3)(*(list(index) + [0] * (3 - len(index))))
    arr = lambda a, n: np.ascontiguousarray(np.zeros(n) if a is None else np.array(a, dtype=np.float64).reshape(-1))
    k = AMR_OPS[op]
    if k == 0:
        out, src, o2, s2 = arr(None, vol), arr(coarse, vol), None, None
    elif k == 1:
        out, src, o2, s2 = arr(coarse, vol), arr(fine, vol), None, None
    elif k == 2:
        out, src, o2, s2 = arr(None, face), arr(coarse, face), arr(None, ff), arr(coarse_flux, ff)
    else:
        out, src, o2, s2 = arr(coarse, face), arr(fine, face), arr(coarse_flux, ff), arr(fine_flux, ff)
    if impl == "oracle":
        L = lib()
        if k == 0:
            L.orc_volume_prolongation(dim, N, nd, _p(out), _p(src), levelDelta, idx)
        elif k == 1:
            L.orc_volume_restriction(dim, N, nd, _p(out), _p(src), levelDelta, idx)
        elif k == 2:
            L.orc_face_prolongation(dim, N, nd, nvar, _p(out), _p(o2), _p(src), _p(s2), levelDelta, idx)
        else:
            L.orc_face_restriction(dim, N, nd, nvar, _p(out), _p(o2), _p(src), _p(s2), levelDelta, idx)
    else:
        f = getattr(reflib(dim), "ref%dd_amr" % dim)
        rc = f(k, nvar, npar, N, _p(out), _p(o2) if o2 is not None else None, _p(src),
               _p(s2) if s2 is not None else None, levelDelta, idx)
        assert rc == 0, "reference AMR routine not built for this shape"
    return (out, o2) if k >= 2 else out


def plot_vertices(dim, N, nvar, luh, impl="oracle"):
    """one cell's values at the (N+1)^d equidistant plot vertices, x fastest"""
    b = N + 1
    u = np.ascontiguousarray(luh, dtype=np.float64).reshape(-1)
    out = np.zeros(b ** dim * nvar)
    if impl == "oracle":
        lib().orc_equidistant_projection(dim, N, nvar, _p(u), _p(out))
    else:
        getattr(reflib(dim), "ref%dd_plot_vertices" % dim)(N, nvar, _p(u), _p(out))
    return out
