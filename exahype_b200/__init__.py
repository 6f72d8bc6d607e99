"""exahype_b200: B200 (sm_100a) ADER-DG hot path of ExaHyPE behind a C ABI.

This module is a thin ctypes binding of ``include/exahype_b200.h``; every call
runs the CUDA kernels of ``lib/libexahype_b200.so``. There is no CPU path: if
the library is missing or fails to load, :func:`load` raises.

Two levels, mirroring the reference:

* :class:`Solver` -- the kernel calls of the reference's generated solver glue
  (``spaceTimePredictor``, ``riemannSolver``, ``boundaryConditions``,
  ``surfaceIntegral`` + ``solutionUpdate`` + ``stableTimeStepSize``), batched
  over many cells/faces, on device buffers (torch CUDA tensors or raw device
  pointers).
* :class:`Mesh` -- a uniform Cartesian mesh with device-resident state driven
  by the reference's non-fused time step (Riemann, corrector + dt, predictor).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libexahype_b200.so")

PDE_EULER = 0
PDE_EULER_TEST = 1
PDE_ELASTIC = 2  # linear elastic waves: 9 variables + lambda, mu, rho; linear kernels
PDE_EULER_SOURCE_NCP = 3  # the kernel-test mock with an algebraic source and a non-conservative product
PDE_ELASTIC_POINT_SOURCE = 4  # PDE_ELASTIC with a Ricker-wavelet point source (Solver.set_point_source)
BC_PERIODIC, BC_OUTFLOW, BC_REFLECTIVE = -1, 0, 1
# predictor variants beyond the autotuned 0..3: the mixed-precision predictor
PREDICTOR_MIXED, PREDICTOR_MIXED_2 = 4, 5

_lib = None


class ExaError(RuntimeError):
    pass


def load():
    """Loads the CUDA library (building it first if this is a source tree
    without one). Raises if it cannot be loaded -- there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise ExaError("exahype_b200: cannot load %s: %s" % (LIB_PATH, e))
    lib.exa_last_error.restype = ctypes.c_char_p
    lib.exa_version.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _check(rc, what):
    if rc != 0:
        raise ExaError("%s failed (%d): %s" % (what, rc, load().exa_last_error().decode()))


def _ptr(x):
    """device pointer of a torch tensor / int / None"""
    if x is None:
        return None
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    return ctypes.c_void_p(x.data_ptr())


def _dbl3(v):
    a = (ctypes.c_double * 3)()
    for i, x in enumerate(v):
        a[i] = float(x)
    return a


def _stream(stream):
    if stream is None:
        try:
            import torch
            return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:
            return None
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


class Solver:
    """Kernel set for one (dim, order, pde) -- the ADERDGSolver of the reference."""

    def __init__(self, dim, order, pde=PDE_EULER):
        lib = load()
        h = ctypes.c_void_p()
        _check(lib.exa_solver_create(int(dim), int(order), int(pde), ctypes.byref(h)), "exa_solver_create")
        self._h = h
        self.dim, self.order, self.pde = dim, order, pde
        z = (ctypes.c_int * 4)()
        _check(lib.exa_solver_sizes(h, z), "exa_solver_sizes")
        self.unknowns_per_cell, self.data_per_cell, self.data_per_face, self.fluxes_per_face = list(z)
        self.nvar = self.unknowns_per_cell // (order + 1) ** dim
        self.ndata = self.data_per_cell // (order + 1) ** dim
        self.linear = pde in (PDE_ELASTIC, PDE_ELASTIC_POINT_SOURCE)

    def __del__(self):
        try:
            if self._h:
                load().exa_solver_destroy(self._h)
        except Exception:
            pass

    # -- reference kernel calls, batched over cells/faces (device buffers) --
    def space_time_predictor(self, luh, lQhbnd, lFhbnd, lduh, dt_dev, dx, ncells, cell_list=None, iterations=None,
                             stream=None):
        _check(load().exa_space_time_predictor_nonlinear(
            self._h, _ptr(luh), _ptr(lQhbnd), _ptr(lFhbnd), _ptr(lduh), _ptr(dt_dev), _dbl3(dx), int(ncells),
            _ptr(cell_list), _ptr(iterations), _stream(stream)), "exa_space_time_predictor_nonlinear")

    def space_time_predictor_temps(self, luh, lQhbnd, lFhbnd, lduh, dt_dev, dx, ncells, iterations, lQi, lFi, lQhi,
                                   lFhi, stream=None):
        _check(load().exa_space_time_predictor_nonlinear_temps(
            self._h, _ptr(luh), _ptr(lQhbnd), _ptr(lFhbnd), _ptr(lduh), _ptr(dt_dev), _dbl3(dx), int(ncells),
            _ptr(iterations), _ptr(lQi), _ptr(lFi), _ptr(lQhi), _ptr(lFhi), _stream(stream)),
            "exa_space_time_predictor_nonlinear_temps")

    def riemann_solver(self, lQhbnd, lFhbnd, face_left, face_right, face_dir, nfaces, stream=None):
        _check(load().exa_riemann_solver_nonlinear(self._h, _ptr(lQhbnd), _ptr(lFhbnd), _ptr(face_left),
                                                   _ptr(face_right), _ptr(face_dir), int(nfaces), _stream(stream)),
               "exa_riemann_solver_nonlinear")

    # -- linear kernels (solvers of a linear PDE, e.g. PDE_ELASTIC) --
    def space_time_predictor_linear(self, luh, lQhbnd, lFhbnd, lduh, dt_dev, dx, ncells, cell_list=None,
                                    stream=None):
        _check(load().exa_space_time_predictor_linear(
            self._h, _ptr(luh), _ptr(lQhbnd), _ptr(lFhbnd), _ptr(lduh), _ptr(dt_dev), _dbl3(dx), int(ncells),
            _ptr(cell_list), _stream(stream)), "exa_space_time_predictor_linear")

    def space_time_predictor_linear_temps(self, luh, lQhbnd, lFhbnd, lduh, dt_dev, dx, ncells, lQhi, lFhi,
                                          stream=None):
        _check(load().exa_space_time_predictor_linear_temps(
            self._h, _ptr(luh), _ptr(lQhbnd), _ptr(lFhbnd), _ptr(lduh), _ptr(dt_dev), _dbl3(dx), int(ncells),
            _ptr(lQhi), _ptr(lFhi), _stream(stream)), "exa_space_time_predictor_linear_temps")

    def set_point_source(self, x0, t0=0.1, f0=8.0, amplitude=1.0):
        """the point source of PDE_ELASTIC_POINT_SOURCE: a Ricker wavelet of
        peak frequency f0 and delay t0 on the normal stresses at x0"""
        x = (ctypes.c_double * 3)(*(list(x0) + [0.0] * (3 - len(x0))))
        _check(load().exa_solver_set_point_source(self._h, x, ctypes.c_double(t0), ctypes.c_double(f0),
                                                  ctypes.c_double(amplitude)), "exa_solver_set_point_source")

    def space_time_predictor_linear_point_source(self, luh, lQhbnd, lFhbnd, lduh, t_dev, dt_dev, dx, centres, ncells,
                                                 cell_list=None, lQhi=None, lFhi=None, stream=None):
        """the linear predictor with the point source evaluated per cell
        (centres: device [ncells][3]; t_dev: the solution's time stamp)"""
        _check(load().exa_space_time_predictor_linear_point_source(
            self._h, _ptr(luh), _ptr(lQhbnd), _ptr(lFhbnd), _ptr(lduh), _ptr(t_dev), _ptr(dt_dev), _dbl3(dx),
            _ptr(centres), int(ncells), _ptr(cell_list), _ptr(lQhi), _ptr(lFhi), _stream(stream)),
            "exa_space_time_predictor_linear_point_source")

    def riemann_solver_linear(self, lQhbnd, lFhbnd, face_left, face_right, face_dir, nfaces, stream=None):
        _check(load().exa_riemann_solver_linear(self._h, _ptr(lQhbnd), _ptr(lFhbnd), _ptr(face_left),
                                                _ptr(face_right), _ptr(face_dir), int(nfaces), _stream(stream)),
               "exa_riemann_solver_linear")

    def volume_integral_linear(self, lduh, lFhi, ncells, stream=None):
        _check(load().exa_volume_integral_linear(self._h, _ptr(lduh), _ptr(lFhi), int(ncells), _stream(stream)),
               "exa_volume_integral_linear")

    # -- AMR transfers and the plotter's vertex projection (device arrays) --
    def volume_unknowns_prolongation(self, luh_fine, luh_coarse, n, fine_cell, coarse_cell, level_delta,
                                     subcell_index, stream=None):
        _check(load().exa_volume_unknowns_prolongation(self._h, _ptr(luh_fine), _ptr(luh_coarse), int(n),
                                                       _ptr(fine_cell), _ptr(coarse_cell), _ptr(level_delta),
                                                       _ptr(subcell_index), _stream(stream)),
               "exa_volume_unknowns_prolongation")

    def volume_unknowns_restriction(self, luh_coarse, luh_fine, n, fine_cell, coarse_cell, level_delta,
                                    subcell_index, stream=None):
        _check(load().exa_volume_unknowns_restriction(self._h, _ptr(luh_coarse), _ptr(luh_fine), int(n),
                                                      _ptr(fine_cell), _ptr(coarse_cell), _ptr(level_delta),
                                                      _ptr(subcell_index), _stream(stream)),
               "exa_volume_unknowns_restriction")

    def face_unknowns_prolongation(self, q_fine, f_fine, q_coarse, f_coarse, n, fine_slot, coarse_slot, level_delta,
                                   subface_index, stream=None):
        _check(load().exa_face_unknowns_prolongation(self._h, _ptr(q_fine), _ptr(f_fine), _ptr(q_coarse),
                                                     _ptr(f_coarse), int(n), _ptr(fine_slot), _ptr(coarse_slot),
                                                     _ptr(level_delta), _ptr(subface_index), _stream(stream)),
               "exa_face_unknowns_prolongation")

    def face_unknowns_restriction(self, q_coarse, f_coarse, q_fine, f_fine, n, fine_slot, coarse_slot, level_delta,
                                  subface_index, stream=None):
        _check(load().exa_face_unknowns_restriction(self._h, _ptr(q_coarse), _ptr(f_coarse), _ptr(q_fine),
                                                    _ptr(f_fine), int(n), _ptr(fine_slot), _ptr(coarse_slot),
                                                    _ptr(level_delta), _ptr(subface_index), _stream(stream)),
               "exa_face_unknowns_restriction")

    def plot_vertices(self, luh, vertices, ncells, stream=None):
        _check(load().exa_plot_vertices(self._h, _ptr(luh), _ptr(vertices), int(ncells), _stream(stream)),
               "exa_plot_vertices")

    def boundary_conditions(self, lQhbnd, lFhbnd, bcell, bface, nb, kind=BC_OUTFLOW, stream=None):
        _check(load().exa_boundary_conditions(self._h, _ptr(lQhbnd), _ptr(lFhbnd), _ptr(bcell), _ptr(bface), int(nb),
                                              int(kind), _stream(stream)), "exa_boundary_conditions")

    def corrector(self, luh, lduh, lFhbnd, dt_dev, dt_min_dev, dx, ncells, cell_list=None, update=True, stream=None):
        _check(load().exa_corrector(self._h, _ptr(luh), _ptr(lduh), _ptr(lFhbnd), _ptr(dt_dev), _ptr(dt_min_dev),
                                    _dbl3(dx), int(ncells), _ptr(cell_list), int(bool(update)), _stream(stream)),
               "exa_corrector")

    # -- limiter kernels (Euler); FV patches lim[cell][(2N+5)^d][5] --
    def project_on_fv_limiter_space(self, luh, lim, ncells, cell_list=None, stream=None):
        _check(load().exa_project_on_fv_limiter_space(self._h, _ptr(luh), _ptr(lim), int(ncells), _ptr(cell_list),
                                                      _stream(stream)), "exa_project_on_fv_limiter_space")

    def project_on_dg_space(self, lim, luh, ncells, cell_list=None, stream=None):
        _check(load().exa_project_on_dg_space(self._h, _ptr(lim), _ptr(luh), int(ncells), _ptr(cell_list),
                                              _stream(stream)), "exa_project_on_dg_space")

    def fv_musclhancock_scratch_bytes(self, ncells):
        b = ctypes.c_size_t()
        _check(load().exa_fv_musclhancock_scratch_bytes(self._h, int(ncells), ctypes.byref(b)),
               "exa_fv_musclhancock_scratch_bytes")
        return b.value

    def fv_musclhancock_update(self, lim, lim_old, luh, dt_dev, dx, ncells, cell_list=None, scratch=None,
                               scratch_bytes=0, stream=None):
        _check(load().exa_fv_musclhancock_update(self._h, _ptr(lim), _ptr(lim_old), _ptr(luh), _ptr(dt_dev),
                                                 _dbl3(dx), int(ncells), _ptr(cell_list), _ptr(scratch),
                                                 ctypes.c_size_t(int(scratch_bytes)), _stream(stream)),
               "exa_fv_musclhancock_update")

    def fv_musclhancock_update_noalloc(self, lim, lim_old, luh, dt_dev, dx, ncells, cell_list=None, stream=None):
        """fv_musclhancock_update with the library's static scratch: no device
        allocation; overlapping calls race on the shared scratch."""
        _check(load().exa_fv_musclhancock_update_noalloc(self._h, _ptr(lim), _ptr(lim_old), _ptr(luh), _ptr(dt_dev),
                                                         _dbl3(dx), int(ncells), _ptr(cell_list), _stream(stream)),
               "exa_fv_musclhancock_update_noalloc")

    @property
    def variant(self):
        v = ctypes.c_int()
        _check(load().exa_solver_get_variant(self._h, ctypes.byref(v)), "exa_solver_get_variant")
        return v.value

    @variant.setter
    def variant(self, v):
        _check(load().exa_solver_set_variant(self._h, int(v)), "exa_solver_set_variant")

    def autotune(self, ncells=4096):
        """Times every predictor variant on `ncells` synthetic cells, keeps the
        fastest; returns (chosen, [ms per variant])."""
        n = 9  # EXA_PREDICTOR_VARIANTS; the mixed variants 4 and 5 report -1 (not timed)
        ms = (ctypes.c_double * n)()
        ch = ctypes.c_int()
        _check(load().exa_solver_autotune(self._h, int(ncells), ms, ctypes.byref(ch)), "exa_solver_autotune")
        return ch.value, list(ms)

    @staticmethod
    def reset_min(dev, stream=None):
        _check(load().exa_reset_min(_ptr(dev), _stream(stream)), "exa_reset_min")


class Mesh:
    """Uniform Cartesian mesh with device-resident ADER-DG state."""

    def __init__(self, solver, cells, offset, size, bc):
        lib = load()
        d = solver.dim
        c = (ctypes.c_int * 3)(*(list(cells) + [1] * (3 - len(cells))))
        o = _dbl3(list(offset) + [0.0] * (3 - len(offset)))
        s = _dbl3(list(size) + [1.0] * (3 - len(size)))
        if isinstance(bc, int):
            bc = [bc] * (2 * d)
        b = (ctypes.c_int * 6)(*(list(bc) + [0] * (6 - len(bc))))
        h = ctypes.c_void_p()
        _check(lib.exa_mesh_create(solver._h, c, o, s, b, ctypes.byref(h)), "exa_mesh_create")
        self._h = h
        self.solver = solver
        self.cells = tuple(cells)
        n = ctypes.c_int()
        _check(lib.exa_mesh_num_cells(h, ctypes.byref(n)), "exa_mesh_num_cells")
        self.ncells = n.value
        self.dx = [size[i] / cells[i] for i in range(d)]

    @classmethod
    def refined(cls, solver, cells, offset, size, box_lo, box_hi):
        """Periodic mesh of cells[d] coarse cells with the box of coarse cells
        box_lo[d] <= c[d] < box_hi[d] refined once (3^d fine cells each;
        exa_mesh_create_refined). Solution order: the unrefined coarse cells
        (x fastest, refined ones skipped), then the fine cells of the box."""
        return cls.nested(solver, cells, offset, size, [(box_lo, box_hi)])

    @classmethod
    def nested(cls, solver, cells, offset, size, boxes, bc=BC_PERIODIC):
        """Periodic mesh with nested refined boxes (exa_mesh_create_nested):
        boxes[k] = (lo, hi) in the cell coordinates of level k (level 0 the
        coarse grid; level k+1 box k refined once, coordinates over the whole
        domain at that level). bc: periodic, outflow or reflective, per domain face or
        one for all. Solution order: the unrefined cells of each level in
        turn, x fastest."""
        return cls.boxes(solver, cells, offset, size, [(k, lo, hi) for k, (lo, hi) in enumerate(boxes)], bc)

    @classmethod
    def boxes(cls, solver, cells, offset, size, boxes, bc=BC_PERIODIC):
        """Mesh refined by boxes (exa_mesh_create_boxes): boxes[k] = (level,
        lo, hi), the positions lo <= p < hi of that level refined once
        (several boxes per level refine their union)."""
        lib = load()
        d = solver.dim
        self = cls.__new__(cls)
        self._h = None
        c = (ctypes.c_int * 3)(*(list(cells) + [1] * (3 - len(cells))))
        o = _dbl3(list(offset) + [0.0] * (3 - len(offset)))
        s = _dbl3(list(size) + [1.0] * (3 - len(size)))
        nb = len(boxes)
        lev = (ctypes.c_int * nb)(*[int(b[0]) for b in boxes])
        lo = (ctypes.c_int * (3 * nb))(*sum((list(b[1]) + [0] * (3 - len(b[1])) for b in boxes), []))
        hi = (ctypes.c_int * (3 * nb))(*sum((list(b[2]) + [1] * (3 - len(b[2])) for b in boxes), []))
        if isinstance(bc, int):
            bc = [bc] * (2 * d)
        bcs = (ctypes.c_int * 6)(*(list(bc) + [BC_PERIODIC] * (6 - len(bc))))
        h = ctypes.c_void_p()
        _check(lib.exa_mesh_create_boxes(solver._h, c, o, s, bcs, nb, lev, lo, hi, ctypes.byref(h)),
               "exa_mesh_create_boxes")
        self._h = h
        self.solver = solver
        self.cells = tuple(cells)
        self.boxes = [(int(b[0]), tuple(b[1]), tuple(b[2])) for b in boxes]
        n = ctypes.c_int()
        _check(lib.exa_mesh_num_cells(h, ctypes.byref(n)), "exa_mesh_num_cells")
        self.ncells = n.value
        self.dx = [size[i] / cells[i] for i in range(d)]
        return self

    def regrid(self, boxes):
        """replace the refinement (exa_mesh_regrid): boxes = [(level, lo,
        hi)], may be empty; the data moves by copy, prolongation or
        restriction, t and the step count are kept"""
        lib = load()
        nb = len(boxes)
        lev = (ctypes.c_int * max(1, nb))(*[int(b[0]) for b in boxes])
        lo = (ctypes.c_int * max(3, 3 * nb))(*sum((list(b[1]) + [0] * (3 - len(b[1])) for b in boxes), []))
        hi = (ctypes.c_int * max(3, 3 * nb))(*sum((list(b[2]) + [1] * (3 - len(b[2])) for b in boxes), []))
        _check(lib.exa_mesh_regrid(self._h, nb, lev, lo, hi), "exa_mesh_regrid")
        self.boxes = [(int(b[0]), tuple(b[1]), tuple(b[2])) for b in boxes]
        n = ctypes.c_int()
        _check(lib.exa_mesh_num_cells(self._h, ctypes.byref(n)), "exa_mesh_num_cells")
        self.ncells = n.value

    def __del__(self):
        try:
            if self._h:
                load().exa_mesh_destroy(self._h)
        except Exception:
            pass

    @property
    def solution_shape(self):
        s = self.solver
        return (self.ncells, (s.order + 1) ** s.dim, s.ndata)

    def set_solution(self, luh):
        a = np.ascontiguousarray(luh, dtype=np.float64)
        assert a.size == int(np.prod(self.solution_shape))
        _check(load().exa_mesh_set_solution(self._h, a.ctypes.data_as(ctypes.c_void_p)), "exa_mesh_set_solution")

    def get_solution(self):
        a = np.empty(self.solution_shape, dtype=np.float64)
        _check(load().exa_mesh_get_solution(self._h, a.ctypes.data_as(ctypes.c_void_p)), "exa_mesh_get_solution")
        return a

    def init(self, t0=0.0):
        _check(load().exa_mesh_init(self._h, ctypes.c_double(t0)), "exa_mesh_init")

    def init_fused(self, t0=0.0, weight=0.99):
        """fused time stepping (predictor right after the update with an
        estimated step, rerun with weight * stable when the estimate was too
        large) instead of init()"""
        _check(load().exa_mesh_init_fused(self._h, ctypes.c_double(t0), ctypes.c_double(weight)),
               "exa_mesh_init_fused")

    def fused_state(self):
        p, r = ctypes.c_double(), ctypes.c_longlong()
        _check(load().exa_mesh_fused_state(self._h, ctypes.byref(p), ctypes.byref(r)), "exa_mesh_fused_state")
        return dict(predictor_dt=p.value, reruns=r.value)

    def step(self, nsteps=1):
        _check(load().exa_mesh_step(self._h, int(nsteps)), "exa_mesh_step")

    def run_until(self, t_end, max_steps=10 ** 9):
        n = ctypes.c_int()
        _check(load().exa_mesh_run_until(self._h, ctypes.c_double(t_end), int(max_steps), ctypes.byref(n)),
               "exa_mesh_run_until")
        return n.value

    def state(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        st, sw = ctypes.c_longlong(), ctypes.c_longlong()
        _check(load().exa_mesh_state(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st), ctypes.byref(sw)),
               "exa_mesh_state")
        return dict(t=t.value, dt=dt.value, steps=st.value, picard_sweeps=sw.value)

    def write_vtk(self, path, binary=False):
        """legacy VTK unstructured grid of the current solution (the layout of
        the reference's ADERDG2CartesianVTK vertex plotter)"""
        _check(load().exa_mesh_write_vtk(self._h, os.fsencode(path), int(bool(binary))), "exa_mesh_write_vtk")

    def validate(self):
        """number of cells with a non-finite value in their solution, update
        or face data (exa_mesh_validate)"""
        n = ctypes.c_longlong()
        _check(load().exa_mesh_validate(self._h, ctypes.byref(n)), "exa_mesh_validate")
        return n.value

    def write_vtk_legendre(self, path, binary=False):
        """legacy VTK unstructured grid of the nodal values at the
        Gauss-Legendre nodes (the reference's ADERDG2LegendreVTK vertex plotter)"""
        _check(load().exa_mesh_write_vtk_legendre(self._h, os.fsencode(path), int(bool(binary))),
               "exa_mesh_write_vtk_legendre")

    def synchronize(self):
        _check(load().exa_mesh_synchronize(self._h), "exa_mesh_synchronize")

    @property
    def stream_handle(self):
        """cudaStream_t of the mesh (for torch.cuda.ExternalStream / events)."""
        h = ctypes.c_void_p()
        _check(load().exa_mesh_stream(self._h, ctypes.byref(h)), "exa_mesh_stream")
        return h.value or 0

    def set_profiling(self, on=True):
        _check(load().exa_mesh_set_profiling(self._h, int(bool(on))), "exa_mesh_set_profiling")

    def set_priority(self, level):
        """stream priority level (0 default; higher levels run first when
        kernels of several streams wait for SMs); call between steps"""
        _check(load().exa_mesh_set_priority(self._h, int(level)), "exa_mesh_set_priority")

    PHASES = ("predictor", "riemann", "corrector", "bookkeeping")

    def phase_times(self, reset=False):
        """{phase: (milliseconds, launches)} accumulated while profiling was on."""
        ms = (ctypes.c_double * 4)()
        n = (ctypes.c_longlong * 4)()
        _check(load().exa_mesh_phase_times(self._h, ms, n, int(bool(reset))), "exa_mesh_phase_times")
        return {p: (ms[i], n[i]) for i, p in enumerate(self.PHASES)}

    def upload_solution_async(self, host_ptr, nbytes):
        """H2D copy of the solution from a (pinned) host pointer, ordered on the mesh stream."""
        _check(load().exa_mesh_copy_solution(self._h, ctypes.c_void_p(host_ptr), ctypes.c_size_t(nbytes), 1),
               "exa_mesh_copy_solution")

    def step_io(self, host_in_ptr, nin, host_out_ptr, nout, nbytes, nsteps):
        """nsteps steps, each taking its solution from the host and leaving its
        result on the host, the copies overlapping the compute of the
        neighbouring steps (pinned host memory; enqueued, see synchronize())."""
        _check(load().exa_mesh_step_io(self._h, ctypes.c_void_p(host_in_ptr), int(nin), ctypes.c_void_p(host_out_ptr),
                                       int(nout), ctypes.c_size_t(nbytes), int(nsteps)), "exa_mesh_step_io")

    def download_solution_async(self, host_ptr, nbytes):
        """D2H copy of the solution into a (pinned) host pointer, ordered on the mesh stream."""
        _check(load().exa_mesh_copy_solution(self._h, ctypes.c_void_p(host_ptr), ctypes.c_size_t(nbytes), 0),
               "exa_mesh_copy_solution")


class LimitingMesh:
    """Uniform Cartesian mesh with the a-posteriori subcell limiter
    (LimitingADERDGSolver): DG cells, FV-limited cells with MUSCL-Hancock
    patches of (2N+1)^d subcells, limiter status spreading and local
    recomputation, all device-resident. Euler PDE; periodic, outflow or reflective faces.

    helper_layers, cure_steps, relax and scale are the reference's
    helper-layers, steps-till-cured, DMP relaxation parameter (delta0) and
    DMP difference scaling (epsilon)."""

    def __init__(self, solver, cells, offset, size, bc, helper_layers=1, cure_steps=0, relax=1e-4, scale=1e-3):
        lib = load()
        d = solver.dim
        c = (ctypes.c_int * 3)(*(list(cells) + [1] * (3 - len(cells))))
        o = _dbl3(list(offset) + [0.0] * (3 - len(offset)))
        s = _dbl3(list(size) + [1.0] * (3 - len(size)))
        if isinstance(bc, int):
            bc = [bc] * (2 * d)
        b = (ctypes.c_int * 6)(*(list(bc) + [0] * (6 - len(bc))))
        h = ctypes.c_void_p()
        _check(lib.exa_lmesh_create(solver._h, c, o, s, b, int(helper_layers), int(cure_steps), ctypes.c_double(relax),
                                    ctypes.c_double(scale), ctypes.byref(h)), "exa_lmesh_create")
        self._h = h
        self.solver = solver
        self.cells = tuple(cells)
        self.ncells = int(np.prod(cells[:d]))
        self.dx = [size[i] / cells[i] for i in range(d)]
        B = 2 * solver.order + 1
        self.patch_shape = ((B + 4) ** d, 5)
        self.subcells = B ** d

    def __del__(self):
        try:
            if self._h:
                load().exa_lmesh_destroy(self._h)
        except Exception:
            pass

    @property
    def solution_shape(self):
        s = self.solver
        return (self.ncells, (s.order + 1) ** s.dim, s.ndata)

    def set_solution(self, luh):
        a = np.ascontiguousarray(luh, dtype=np.float64)
        assert a.size == int(np.prod(self.solution_shape))
        _check(load().exa_lmesh_set_solution(self._h, a.ctypes.data_as(ctypes.c_void_p)), "exa_lmesh_set_solution")

    def get_solution(self):
        a = np.empty(self.solution_shape, dtype=np.float64)
        _check(load().exa_lmesh_get_solution(self._h, a.ctypes.data_as(ctypes.c_void_p)), "exa_lmesh_get_solution")
        return a

    def set_fv_initial(self, fv):
        """FV initial condition at the subcell centres, (ncells, (2N+1)^d, 5)."""
        a = np.ascontiguousarray(fv, dtype=np.float64)
        assert a.size == self.ncells * self.subcells * 5
        _check(load().exa_lmesh_set_fv_initial(self._h, a.ctypes.data_as(ctypes.c_void_p)), "exa_lmesh_set_fv_initial")

    def init(self, t0=0.0):
        _check(load().exa_lmesh_init(self._h, ctypes.c_double(t0)), "exa_lmesh_init")

    def step(self, nsteps=1):
        _check(load().exa_lmesh_step(self._h, int(nsteps)), "exa_lmesh_step")

    def run_until(self, t_end, max_steps=10 ** 9):
        n = ctypes.c_int()
        _check(load().exa_lmesh_run_until(self._h, ctypes.c_double(t_end), int(max_steps), ctypes.byref(n)),
               "exa_lmesh_run_until")
        return n.value

    def state(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        st, sw, irr = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        _check(load().exa_lmesh_state(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st), ctypes.byref(sw),
                                      ctypes.byref(irr)), "exa_lmesh_state")
        return dict(t=t.value, dt=dt.value, steps=st.value, picard_sweeps=sw.value, irregular_steps=irr.value)

    def write_vtk(self, path, binary=False):
        """legacy VTK of the DG solution with the limiter status as vertex
        data (the reference's LimitingADERDG2CartesianVTK vertex plotter)"""
        _check(load().exa_lmesh_write_vtk(self._h, os.fsencode(path), int(bool(binary))), "exa_lmesh_write_vtk")

    def status(self):
        s = np.empty(self.ncells, dtype=np.int32)
        _check(load().exa_lmesh_get_status(self._h, s.ctypes.data_as(ctypes.c_void_p)), "exa_lmesh_get_status")
        return s

    def limiter(self):
        """(FV patches (ncells, E^d, 5) incl. ghost layers, allocated flags)"""
        lim = np.empty((self.ncells,) + self.patch_shape, dtype=np.float64)
        al = np.empty(self.ncells, dtype=np.int32)
        _check(load().exa_lmesh_get_limiter(self._h, lim.ctypes.data_as(ctypes.c_void_p),
                                            al.ctypes.data_as(ctypes.c_void_p)), "exa_lmesh_get_limiter")
        return lim, al

    def synchronize(self):
        _check(load().exa_lmesh_synchronize(self._h), "exa_lmesh_synchronize")

    def set_priority(self, level):
        _check(load().exa_lmesh_set_priority(self._h, int(level)), "exa_lmesh_set_priority")

    @property
    def stream_handle(self):
        h = ctypes.c_void_p()
        _check(load().exa_lmesh_stream(self._h, ctypes.byref(h)), "exa_lmesh_stream")
        return h.value or 0


class Batch:
    """Batched ragged ensemble of independent uniform-mesh solves (exa_batch_*):
    instances of one (dim, order) share device arrays, a step is one CUDA graph
    launch, and every instance computes what a Mesh of the same problem would."""

    def __init__(self):
        h = ctypes.c_void_p()
        _check(load().exa_batch_create(ctypes.byref(h)), "exa_batch_create")
        self._h = h
        self._shape = {}

    def __del__(self):
        try:
            if self._h:
                load().exa_batch_destroy(self._h)
        except Exception:
            pass

    def add(self, dim, order, cells, size, bc, luh, pde=PDE_EULER):
        c = (ctypes.c_int * 3)(*(list(cells) + [1] * (3 - len(cells))))
        s = _dbl3(list(size) + [1.0] * (3 - len(size)))
        if isinstance(bc, int):
            bc = [bc] * (2 * dim)
        b = (ctypes.c_int * 6)(*(list(bc) + [0] * (6 - len(bc))))
        a = np.ascontiguousarray(luh, dtype=np.float64)
        i = ctypes.c_int()
        _check(load().exa_batch_add(self._h, int(dim), int(order), int(pde), c, s, b,
                                    a.ctypes.data_as(ctypes.c_void_p), ctypes.byref(i)), "exa_batch_add")
        ndata = 5 + (1 if pde == PDE_EULER_TEST else 0)
        self._shape[i.value] = (int(np.prod(cells[:dim])), (order + 1) ** dim, ndata)
        return i.value

    def remove(self, iid):
        _check(load().exa_batch_remove(self._h, int(iid)), "exa_batch_remove")

    def commit(self):
        _check(load().exa_batch_commit(self._h), "exa_batch_commit")

    def step(self, nsteps=1):
        _check(load().exa_batch_step(self._h, int(nsteps)), "exa_batch_step")

    def set_graph(self, on=True):
        _check(load().exa_batch_set_graph(self._h, int(bool(on))), "exa_batch_set_graph")

    def variant(self, dim, order, pde=PDE_EULER):
        v = ctypes.c_int()
        _check(load().exa_batch_get_variant(self._h, int(dim), int(order), int(pde), ctypes.byref(v)),
               "exa_batch_get_variant")
        return v.value

    def set_variant(self, dim, order, variant, pde=PDE_EULER):
        _check(load().exa_batch_set_variant(self._h, int(dim), int(order), int(pde), int(variant)),
               "exa_batch_set_variant")

    def state(self, iid):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        _check(load().exa_batch_state(self._h, int(iid), ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st)),
               "exa_batch_state")
        return dict(t=t.value, dt=dt.value, steps=st.value)

    def get_solution(self, iid):
        a = np.empty(self._shape[iid], dtype=np.float64)
        _check(load().exa_batch_get_solution(self._h, int(iid), a.ctypes.data_as(ctypes.c_void_p)),
               "exa_batch_get_solution")
        return a

    @staticmethod
    def instance_bytes(dim, order, cells, pde=PDE_EULER):
        c = (ctypes.c_int * 3)(*(list(cells) + [1] * (3 - len(cells))))
        b = ctypes.c_size_t()
        _check(load().exa_batch_instance_bytes(int(dim), int(order), int(pde), c, ctypes.byref(b)),
               "exa_batch_instance_bytes")
        return b.value

    def device_bytes(self):
        b = ctypes.c_size_t()
        _check(load().exa_batch_device_bytes(self._h, ctypes.byref(b)), "exa_batch_device_bytes")
        return b.value

    def sweeps(self):
        v = ctypes.c_longlong()
        _check(load().exa_batch_sweeps(self._h, ctypes.byref(v)), "exa_batch_sweeps")
        return v.value

    def synchronize(self):
        _check(load().exa_batch_synchronize(self._h), "exa_batch_synchronize")

    @property
    def stream_handle(self):
        h = ctypes.c_void_p()
        _check(load().exa_batch_stream(self._h, ctypes.byref(h)), "exa_batch_stream")
        return h.value or 0


def cell_positions(mesh):
    """(level, position) of every cell of a mesh made by Mesh.boxes / nested /
    refined, in the solution's cell order (the same rule as
    exa_mesh_create_boxes: level by level, x fastest over each level's
    bounding rectangle)."""
    from . import problems
    d = mesh.solver.dim
    out = []
    boxes = getattr(mesh, "boxes", None)
    for lev, (r0, st) in enumerate(problems.box_levels(d, mesh.cells, boxes) if boxes else
                                   [[[0] * d, np.ones(tuple(reversed(mesh.cells[:d])), dtype=np.int8)]]):
        idx = np.argwhere(st == 1)  # (z, y, x) order, x fastest
        for t in idx:
            out.append((lev, tuple(int(r0[i] + t[d - 1 - i]) for i in range(d))))
    return out


# refinement controls a criterion returns per cell, with the reference's
# values (exahype::solvers::Solver::RefinementControl, Solver.h:446)
KEEP, REFINE, ERASE = 0, 1, 2


def adapt_boxes(mesh, controls, max_level):
    """The refinement of a mesh after a refinement criterion, as boxes for
    Mesh.regrid. controls[c] is the criterion's answer for cell c (in the
    solution's cell order): KEEP (0), REFINE (1) or ERASE (2); booleans read
    as REFINE / KEEP.

    Follows the reference's rules (ADERDGSolver::markForRefinement,
    ADERDGSolver.cpp:1078-1150): a cell below max_level that answers REFINE is
    refined; a refined position is erased only when every one of its 3^d
    children is an unrefined cell that answers ERASE (any child that answers
    KEEP or REFINE, or is refined itself, vetoes it), so KEEP leaves the
    refinement as it is. Coarser levels are then refined around every
    refined position so that each keeps one cell of margin inside its
    level's region (the reference's spacetree keeps the same 2:1-like
    balance with its helper cells); positions within one cell of the domain
    boundary are never refined. Returns [(level, lo, hi)] with one box per
    run of refined positions along x."""
    from . import problems
    d = mesh.solver.dim
    cells = list(mesh.cells[:d])
    pos = cell_positions(mesh)
    ctrl = {}
    for (lev, p), c in zip(pos, controls):
        ctrl[(lev, p)] = int(c)
    F = [set() for _ in range(max_level)]
    # the current refinement, minus the positions all of whose children erase
    boxes_now = getattr(mesh, "boxes", None) or []
    kids = [tuple(o) for o in np.ndindex(*([3] * d))]
    if boxes_now:
        for lev, (r0, st) in enumerate(problems.box_levels(d, mesh.cells, boxes_now)):
            if lev >= max_level:
                continue
            for t in np.argwhere(st == 2):
                p = tuple(int(r0[i] + t[d - 1 - i]) for i in range(d))
                erase = all(ctrl.get((lev + 1, tuple(3 * p[i] + k[i] for i in range(d)))) == ERASE for k in kids)
                if not erase:
                    F[lev].add(p)
    for (lev, p), c in ctrl.items():
        if c == REFINE and lev < max_level:
            F[lev].add(p)
    for lev in range(max_level - 1, 0, -1):  # ancestors of refined positions stay refined
        for p in list(F[lev]):
            F[lev - 1].add(tuple(x // 3 for x in p))
    # margins: every refined position at level l needs its neighbourhood
    # inside level l's region, i.e. the parents of that neighbourhood refined
    nbh = kids
    for lev in range(max_level - 1, 0, -1):
        for p in list(F[lev]):
            for o in nbh:
                F[lev - 1].add(tuple((p[i] + o[i] - 1) // 3 for i in range(d)))
    F[0] = {p for p in F[0] if all(1 <= p[i] <= cells[i] - 2 for i in range(d))}
    for lev in range(1, max_level):  # drop what lost its region
        region = F[lev - 1]
        F[lev] = {p for p in F[lev] if all(tuple((p[i] + o[i] - 1) // 3 for i in range(d)) in region for o in nbh)}
    boxes = []
    for lev in range(max_level):
        for p in sorted(F[lev], key=lambda c: tuple(reversed(c))):
            if boxes and boxes[-1][0] == lev and boxes[-1][2][0] == p[0] and list(boxes[-1][1][1:]) == list(p[1:]):
                boxes[-1][2][0] = p[0] + 1
            else:
                boxes.append((lev, list(p), [p[i] + 1 for i in range(d)]))
    return [(lev, tuple(lo), tuple(hi)) for lev, lo, hi in boxes]
