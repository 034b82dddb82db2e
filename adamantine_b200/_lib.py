"""ctypes binding of include/adamantine_b200.h (libadamantine_b200.so).

The library is the only compute path: if it is missing or fails to load, the
package raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

from .config import ConfigStruct, SourceStruct

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libadamantine_b200.so")

_VP = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_I64 = ctypes.POINTER(ctypes.c_int64)
_I32 = ctypes.POINTER(ctypes.c_int32)

# name -> argtypes (every function returns int)
SIGNATURES = {
    "adm_create": [ctypes.POINTER(ConfigStruct), ctypes.c_int, _VP, ctypes.POINTER(_VP)],
    "adm_destroy": [_VP],
    "adm_set_cells": [_VP, _U8, _U8, _U8, _D, _D],
    "adm_setup": [_VP],
    "adm_n_nodes": [_VP, _I64],
    "adm_n_cells": [_VP, _I64],
    "adm_get_active_cells": [_VP, _VP],
    "adm_node_layout": [_VP, _I64, _I64],
    "adm_set_time": [_VP, ctypes.c_double],
    "adm_vmult": [_VP, _VP, _VP],
    "adm_vmult_add": [_VP, _VP, _VP],
    "adm_vmult_host": [_VP, _D, _D],
    "adm_compute_inverse_mass_matrix": [_VP],
    "adm_get_inverse_mass_matrix": [_VP, _VP],
    "adm_evolve_one_time_step": [_VP, ctypes.c_double, ctypes.c_double, _VP, _D],
    "adm_evolve_one_time_step_host": [_VP, ctypes.c_double, ctypes.c_double, _D, _D],
    "adm_evolve_n_steps": [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32, _VP, _D],
    "adm_evaluate_material_properties": [_VP, _VP, _VP],
    "adm_set_state_to_material_properties": [_VP],
    "adm_get_state_from_material_properties": [_VP],
    "adm_get_cell_state": [_VP, _D],
    "adm_set_cell_state": [_VP, _D],
    "adm_get_qp_powder": [_VP, _D],
    "adm_mark_has_melted": [_VP, ctypes.c_double, _VP, _U8],
    "adm_activate_cells": [_VP, _I64, ctypes.c_int64, ctypes.c_double, _D, _D, _VP],
    "adm_update_beam": [_VP, ctypes.c_int32, ctypes.POINTER(SourceStruct)],
    "adm_vmult_host_static": [_VP, _D, _D],
    "adm_update_material": [_VP, ctypes.POINTER(ConfigStruct)],
    "adm_set_schedule": [_VP, ctypes.c_int32],
    "adm_get_schedule": [_VP, _I32],
    "adm_autotune": [_VP, _VP, _I32, _D],
    "adm_autotune_schedules": [_VP, _VP, _I32, _D, ctypes.c_int32],
    "adm_set_cells_per_thread": [_VP, ctypes.c_int32],
    "adm_set_cells_per_block": [_VP, ctypes.c_int32],
    "adm_get_cells_per_block": [_VP, _I32],
    "adm_get_cells_per_thread": [_VP, _I32],
    "adm_save_checkpoint": [_VP, ctypes.c_char_p, ctypes.c_double, _VP],
    "adm_load_checkpoint": [_VP, ctypes.c_char_p, ctypes.c_int32, _D, _VP],
    "adm_device_error": [_VP, _I32],
    "adm_synchronize": [_VP],
    # include/adamantine_b200_ensemble.h
    "adm_ensemble_create": [ctypes.POINTER(ConfigStruct), ctypes.c_int32, ctypes.c_int, _VP, ctypes.POINTER(_VP)],
    "adm_ensemble_destroy": [_VP],
    "adm_ensemble_set_cells": [_VP, ctypes.c_int32, _U8, _U8, _U8, _D, _D],
    "adm_ensemble_setup": [_VP],
    "adm_ensemble_stride": [_VP, _I64],
    "adm_ensemble_n_work_items": [_VP, _I64],
    "adm_ensemble_evolve_one_time_step": [_VP, ctypes.c_double, ctypes.c_double, _VP, _D],
    "adm_ensemble_evolve_looped": [_VP, ctypes.c_double, ctypes.c_double, _VP, _D],
    "adm_ensemble_evolve_n_steps": [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32, _VP, _D],
    "adm_ensemble_update_beam": [_VP, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(SourceStruct)],
    "adm_ensemble_update_material": [_VP, ctypes.c_int32, ctypes.POINTER(ConfigStruct)],
    "adm_ensemble_get_cell_state": [_VP, ctypes.c_int32, _D],
    "adm_ensemble_get_inverse_mass_matrix": [_VP, ctypes.c_int32, _VP],
    "adm_ensemble_set_schedule": [_VP, ctypes.c_int32],
    "adm_ensemble_autotune": [_VP, _VP, ctypes.c_double, _I32, _D],
    "adm_ensemble_autotune_schedules": [_VP, _VP, ctypes.c_double, _I32, _D, ctypes.c_int32],
    "adm_ensemble_set_cells_per_thread": [_VP, ctypes.c_int32],
    "adm_ensemble_get_cells_per_thread": [_VP, _I32],
    "adm_ensemble_device_error": [_VP, _I32],
    "adm_ensemble_synchronize": [_VP],
    "adm_enkf_create": [ctypes.c_int, _VP, ctypes.POINTER(_VP)],
    "adm_enkf_destroy": [_VP],
    # include/adamantine_b200_deposition.h
    "adm_deposition_boxes": [ctypes.POINTER(SourceStruct), ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, ctypes.c_double, ctypes.c_int64, _D, _D, _D, _D, _D, _I64],
    "adm_deposition_create": [_VP, ctypes.c_int64, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                              ctypes.POINTER(_VP)],
    "adm_deposition_destroy": [_VP],
    "adm_deposition_activate_range": [_VP, ctypes.c_int64, ctypes.c_int64, ctypes.c_double, _VP, _I64],
    "adm_deposition_step": [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_double, _VP, _I64],
    # include/adamantine_b200_adjoint.h
    "adm_adjoint_create": [_VP, ctypes.POINTER(_VP)],
    "adm_adjoint_destroy": [_VP],
    "adm_adjoint_set_observations": [_VP, ctypes.c_int32, _I32, ctypes.c_int32, _I64, _D],
    "adm_adjoint_objective": [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32, _VP, _D, _VP],
    "adm_adjoint_gradient": [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, _VP, _D, _D,
                             _VP],
    "adm_adjoint_vmult_transpose": [_VP, _VP, _VP, _VP, _D],
    "adm_adjoint_checkpoint_interval": [_VP, ctypes.POINTER(ctypes.c_int32)],
    "adm_adjoint_set_flush": [_VP, ctypes.c_double],
    "adm_enkf_observe": [_VP, ctypes.c_int32, _VP, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, _VP, _VP],
    "adm_enkf_gain": [_VP, ctypes.c_int32, ctypes.c_int32, _VP, _VP, _VP, _VP, _VP, _VP],
    "adm_enkf_local_sum": [_VP, ctypes.c_int32, _VP, ctypes.c_int64, ctypes.c_int64, _VP, ctypes.c_int32, _VP],
    "adm_enkf_partial_update": [_VP, ctypes.c_int32, ctypes.c_int32, _VP, ctypes.c_int64, ctypes.c_int64, _VP,
                                ctypes.c_int32, _VP, _VP, _VP],
    "adm_enkf_partial_update_localized": [_VP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _VP,
                                          ctypes.c_int64, ctypes.c_int64, _VP, ctypes.c_int32, _VP, _VP, _VP],
    "adm_enkf_set_localization": [_VP, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _VP, _VP, _VP, _VP,
                                  ctypes.c_int64],
    "adm_enkf_apply": [_VP, ctypes.c_int32, _VP, ctypes.c_int64, ctypes.c_int64, _VP, ctypes.c_int32, _VP, _VP],
    "adm_microstructure_create": [_VP, ctypes.POINTER(_VP)],
    "adm_microstructure_destroy": [_VP],
    "adm_microstructure_set_old_temperature": [_VP, _VP],
    "adm_microstructure_compute_G_and_R": [_VP, _VP, ctypes.c_double, ctypes.c_int64, _VP,
                                           ctypes.POINTER(ctypes.c_int64)],
    "adm_amr_mesh_create": [_VP, ctypes.c_int32, ctypes.POINTER(_VP)],
    "adm_amr_mesh_destroy": [_VP],
    "adm_amr_mesh_set_cells": [_VP, _VP, _VP, _VP],
    "adm_amr_mesh_refine_mesh": [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                                 ctypes.c_int32],
    "adm_amr_mesh_execute": [_VP, _VP, _VP],
    "adm_amr_mesh_build": [_VP],
    "adm_amr_mesh_n_leaves": [_VP, ctypes.POINTER(ctypes.c_int64)],
    "adm_amr_mesh_leaves": [_VP, _VP],
    "adm_amr_mesh_n_dofs": [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)],
    "adm_amr_mesh_dof_lattice": [_VP, _VP],
    "adm_amr_mesh_constraints": [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), _VP, _VP,
                                 _VP, _VP],
    "adm_amr_create": [_VP, ctypes.c_int32, ctypes.c_int32, _VP, ctypes.POINTER(_VP)],
    "adm_amr_destroy": [_VP],
    "adm_amr_set_cells": [_VP, _VP, _VP, _VP],
    "adm_amr_setup": [_VP, ctypes.c_double],
    "adm_amr_refine_mesh": [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32],
    "adm_amr_execute": [_VP, _VP, _VP],
    "adm_amr_n_dofs": [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)],
    "adm_amr_remesh_profile": [_VP, _VP],
    "adm_amr_n_leaves": [_VP, ctypes.POINTER(ctypes.c_int64)],
    "adm_amr_leaves": [_VP, _VP],
    "adm_amr_dof_lattice": [_VP, _VP],
    "adm_amr_solution": [_VP, ctypes.POINTER(_VP)],
    "adm_amr_get_solution": [_VP, _VP],
    "adm_amr_set_solution": [_VP, _VP],
    "adm_amr_set_time": [_VP, ctypes.c_double],
    "adm_amr_vmult": [_VP, _VP, _VP],
    "adm_amr_inverse_mass": [_VP, _VP],
    "adm_amr_evolve_one_time_step": [_VP, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)],
    "adm_amr_level_values": [_VP, ctypes.c_int32, _VP],
    "adm_amr_level_layout": [_VP, ctypes.c_int32, _VP, ctypes.POINTER(ctypes.c_int64)],
    "adm_amr_level_cell_state": [_VP, ctypes.c_int32, _VP],
    "adm_amr_set_schedule": [_VP, ctypes.c_int32],
    "adm_amr_mark_has_melted": [_VP, ctypes.c_double],
    "adm_amr_level_has_melted": [_VP, ctypes.c_int32, _VP],
    "adm_amr_synchronize": [_VP],
    "adm_mechanics_create": [_VP, _VP, ctypes.POINTER(_VP)],
    "adm_mechanics_destroy": [_VP],
    "adm_mechanics_setup": [_VP, _VP],
    "adm_mechanics_vmult": [_VP, _VP, _VP],
    "adm_mechanics_rhs": [_VP, _VP],
    "adm_mechanics_solve": [_VP, _VP, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)],
    "adm_mechanics_set_preconditioner": [_VP, ctypes.c_int32],
    "adm_mechanics_multigrid_levels": [_VP, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)],
    "adm_mechanics_n_dofs": [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)],
    "adm_mechanics_node_mask": [_VP, _VP],
    "adm_mechanics_stress_state": [_VP, _VP, _VP, _VP],
    "adm_enkf_analysis": [_VP, ctypes.c_int32, _VP, ctypes.c_int64, ctypes.c_int64, _VP, ctypes.c_int32,
                          ctypes.c_int32, _VP, _VP, _VP, _VP, _VP, _VP],
}

_lib = None


class AdmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"adamantine_b200 error {code}: {msg}")
        self.code = code


def load():
    """Load the CUDA library (building it first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build

        build.build()
    L = ctypes.CDLL(LIB_PATH)
    for name, argtypes in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = argtypes
        fn.restype = ctypes.c_int
    L.adm_last_error.restype = ctypes.c_char_p
    L.adm_last_error.argtypes = []
    _lib = L
    return L


def check(rc: int):
    if rc != 0:
        msg = load().adm_last_error().decode(errors="replace")
        raise AdmError(rc, msg)
