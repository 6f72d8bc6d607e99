"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares; no compute calls are made here."""
import ctypes
import glob
import os
import re

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?\w+\**\s+\**(exa_\w+)\s*\(", src, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_api():
    names = declared_functions()
    for required in ("exa_space_time_predictor_nonlinear", "exa_riemann_solver_nonlinear", "exa_boundary_conditions",
                     "exa_corrector", "exa_mesh_create", "exa_mesh_step", "exa_solver_create",
                     "exa_space_time_predictor_linear", "exa_riemann_solver_linear", "exa_volume_integral_linear",
                     "exa_volume_unknowns_prolongation", "exa_volume_unknowns_restriction",
                     "exa_face_unknowns_prolongation", "exa_face_unknowns_restriction", "exa_plot_vertices",
                     "exa_mesh_write_vtk", "exa_mesh_step_io", "exa_mesh_init_fused", "exa_mesh_fused_state",
                     "exa_mesh_create_refined", "exa_mesh_create_nested", "exa_mesh_write_vtk_legendre", "exa_lmesh_write_vtk", "exa_mesh_validate", "exa_mesh_create_boxes", "exa_mesh_regrid"):
        assert required in names


def test_library_exports_every_declared_symbol():
    import exahype_b200
    lib = exahype_b200.load()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_error_path_without_gpu_is_reported_not_raised():
    import exahype_b200
    lib = exahype_b200.load()
    h = ctypes.c_void_p()
    assert lib.exa_solver_create(4, 3, 0, ctypes.byref(h)) == -1  # bad dimension, no CUDA call made
    assert b"dim" in lib.exa_last_error()
    assert lib.exa_solver_create(2, 3, 0, None) == -1
