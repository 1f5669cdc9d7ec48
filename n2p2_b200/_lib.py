"""Loads libn2p2b200.so and declares the C ABI of include/n2p2_b200.h.

The product path has no fallback: if the library is missing or cannot be
loaded, importing the package's GPU entry points raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libn2p2b200.so")

OK = 0
ERR_RUNTIME = 1
ERR_RANGE = 2
ERR_OUT_OF_RANGE = 3
ERR_INVALID_ARGUMENT = 4
ERR_CUDA = 5
ERR_NULL = 6

PRECISION_FP64 = 0
PRECISION_MIXED = 1

EVAL_FORCES = 1
EVAL_STORE_DGDR = 2
EVAL_NO_GRAPH = 4
EVAL_SF_ONLY = 8

DERIVATIVES_NONE = 0
DERIVATIVES = 1
DERIVATIVES_STORED = 2

TRAINING_ENERGY = 0
TRAINING_FORCE = 1

# Every function the header declares, with (restype, argtypes).
_vp = ctypes.c_void_p
_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double
_cp = ctypes.c_char_p
_P = ctypes.POINTER

SIGNATURES = {
    "n2p2_last_error": (_cp, []),
    "n2p2_version": (_cp, []),
    "n2p2_mode_create": (_i, [_P(_vp), _i]),
    "n2p2_mode_get_network_topology": (_i, [_vp, _i, _i, _P(_i), _P(_i), _P(_i)]),
    "n2p2_shuffle_rng_create": (_i, [ctypes.c_uint64, _P(_vp)]),
    "n2p2_shuffle_rng_destroy": (_i, [_vp]),
    "n2p2_shuffle_rng_shuffle": (_i, [_vp, _P(_i64), _i64]),
    "n2p2_mode_destroy": (_i, [_vp]),
    "n2p2_mode_initialize": (_i, [_vp]),
    "n2p2_mode_load_settings_file": (_i, [_vp, _cp]),
    "n2p2_mode_setup_generic": (_i, [_vp]),
    "n2p2_mode_setup_symmetry_function_scaling": (_i, [_vp, _cp]),
    "n2p2_mode_setup_symmetry_function_scaling_none": (_i, [_vp]),
    "n2p2_mode_setup_neural_network_weights": (_i, [_vp, _cp]),
    "n2p2_mode_set_connections": (_i, [_vp, _i, _P(_d), _i64]),
    "n2p2_mode_setup_symmetry_function_statistics": (_i, [_vp, _i, _i, _i, _i]),
    "n2p2_mode_set_precision": (_i, [_vp, _i]),
    "n2p2_mode_get_max_cutoff_radius": (_i, [_vp, _P(_d)]),
    "n2p2_mode_get_num_elements": (_i, [_vp, _P(_i)]),
    "n2p2_mode_get_element_symbol": (_i, [_vp, _i, _cp, _i]),
    "n2p2_mode_get_element_index": (_i, [_vp, _cp, _P(_i)]),
    "n2p2_mode_get_num_symmetry_functions": (_i, [_vp, _i, _P(_i)]),
    "n2p2_mode_get_num_derivative_rows": (_i, [_vp, _i, _i, _P(_i)]),
    "n2p2_mode_get_symmetry_function": (_i, [_vp, _i, _i, _P(_i), _P(_i), _P(_i), _P(_d)]),
    "n2p2_batch_create": (_i, [_vp, _P(_vp)]),
    "n2p2_batch_destroy": (_i, [_vp]),
    "n2p2_batch_set_structures": (_i, [_vp, _i64, _P(_i64), _P(ctypes.c_int32), _P(_d), _P(ctypes.c_int32), _i]),
    "n2p2_batch_set_positions": (_i, [_vp, _vp, _i]),
    "n2p2_batch_evaluate": (_i, [_vp, _i]),
    "n2p2_batch_synchronize": (_i, [_vp]),
    "n2p2_batch_get_neighbor_capacity": (_i, [_vp, _P(_i64), _P(_i64)]),
    "n2p2_batch_calculate_neighbor_list": (_i, [_vp]),
    "n2p2_batch_calculate_symmetry_functions": (_i, [_vp, _i]),
    "n2p2_batch_calculate_symmetry_function_groups": (_i, [_vp, _i]),
    "n2p2_batch_calculate_atomic_neural_networks": (_i, [_vp, _i]),
    "n2p2_batch_calculate_energy": (_i, [_vp]),
    "n2p2_batch_calculate_forces": (_i, [_vp]),
    "n2p2_batch_get_energies": (_i, [_vp, _P(_d)]),
    "n2p2_batch_get_forces": (_i, [_vp, _P(_d)]),
    "n2p2_batch_evaluate_host": (_i, [_vp, _vp, _vp, _vp, _i]),
    "n2p2_batch_get_num_atoms": (_i, [_vp, _P(_i64)]),
    "n2p2_batch_get_num_neighbor_entries": (_i, [_vp, _P(_i64)]),
    "n2p2_batch_get_neighbors": (_i, [_vp, _P(_i64), _P(ctypes.c_int32), _P(ctypes.c_int32), _P(_d), _P(_d)]),
    "n2p2_batch_get_symmetry_functions": (_i, [_vp, _P(_d)]),
    "n2p2_batch_get_dEdG": (_i, [_vp, _P(_d)]),
    "n2p2_batch_get_atomic_energies": (_i, [_vp, _P(_d)]),
    "n2p2_batch_get_dGdr": (_i, [_vp, _P(_d), _P(_d)]),
    "n2p2_batch_get_internal_positions": (_i, [_vp, _P(_d)]),
    "n2p2_batch_get_extrapolation_warnings": (_i, [_vp, _P(_i64), _P(ctypes.c_int32)]),
    "n2p2_batch_get_launch_count": (_i, [_vp, _P(_i)]),
    "n2p2_neighbor_list_noalloc": (_i, [_vp, _i64, _P(_d), _d, _i64, _vp, _vp, _vp, _vp, _vp, _P(_i64), _vp]),
    "n2p2_neighbor_list_noalloc_status": (_i, [_i64, _vp, _i64, _P(_i64), _vp]),
    "n2p2_batch_get_stream": (_i, [_vp, _P(_vp)]),
    "n2p2_batch_profile_stages": (_i, [_vp, _i, _i, _cp, _P(_d), _P(_i)]),
    "n2p2_batch_count_work": (_i, [_vp, _P(_i64)]),
    "n2p2_device_fma_peak": (_i, [_i, _P(_d), _P(_d)]),
    "n2p2_cutoff_function": (_i, [_i, _i, _d, _d, _i, _P(_d), _i64, _P(_d), _P(_d)]),
    "n2p2_mode_set_autotune": (_i, [_vp, ctypes.c_int32]),
    "n2p2_batch_autotune": (_i, [_vp, ctypes.c_int32, _P(ctypes.c_int32), _P(_d), _P(ctypes.c_int32)]),
    "n2p2_batch_set_shapes": (_i, [_vp, ctypes.c_int32, ctypes.c_int32]),
    "n2p2_trainer_create": (_i, [_vp, _P(_vp)]),
    "n2p2_trainer_destroy": (_i, [_vp]),
    "n2p2_trainer_set_adam": (_i, [_vp, _d, _d, _d, _d]),
    "n2p2_trainer_set_learning_rate": (_i, [_vp, _d]),
    "n2p2_trainer_set_loss_weights": (_i, [_vp, _d, _d]),
    "n2p2_trainer_get_num_parameters": (_i, [_vp, _P(_i64)]),
    "n2p2_trainer_get_parameters": (_i, [_vp, _P(_d)]),
    "n2p2_trainer_set_parameters": (_i, [_vp, _P(_d)]),
    "n2p2_trainer_step": (_i, [_vp, _vp, _P(_d), _P(_d), ctypes.c_int32, _P(_d), _P(_d)]),
    "n2p2_training_create": (_i, [_vp, _P(_vp)]),
    "n2p2_training_destroy": (_i, [_vp]),
    "n2p2_training_set_references": (_i, [_vp, _P(_d), _P(_d)]),
    "n2p2_training_set_force_weight": (_i, [_vp, _d]),
    "n2p2_training_set_update_strategy": (_i, [_vp, ctypes.c_int32]),
    "n2p2_training_set_jacobian_mode": (_i, [_vp, ctypes.c_int32]),
    "n2p2_training_set_task_batch_size": (_i, [_vp, ctypes.c_int32, ctypes.c_int32]),
    "n2p2_training_set_kalman_standard": (_i, [_vp, _d, _d, _d, _d, _d, _d, _d]),
    "n2p2_training_set_kalman_fading_memory": (_i, [_vp, _d, _d, _d, _d, _d, _d]),
    "n2p2_training_set_gradient_fixed": (_i, [_vp, _d]),
    "n2p2_training_set_gradient_adam": (_i, [_vp, _d, _d, _d, _d]),
    "n2p2_training_update": (_i, [_vp, ctypes.c_int32, ctypes.c_int32, _P(ctypes.c_int32), _P(ctypes.c_int32),
                                  _P(ctypes.c_int32), _P(_d)]),
    "n2p2_training_observe": (_i, [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P(_d),
                                   _P(_d)]),
    "n2p2_training_update_threshold": (_i, [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            _P(ctypes.c_int32), _P(ctypes.c_int32), _P(ctypes.c_int32), _d,
                                            ctypes.c_int32, _d, _P(ctypes.c_int32), _P(_d)]),
    "n2p2_training_get_errors": (_i, [_vp, _P(_d)]),
    "n2p2_training_get_kalman_status": (_i, [_vp, _P(_d)]),
    "n2p2_training_get_num_weights": (_i, [_vp, _P(_i64)]),
    "n2p2_training_get_weights": (_i, [_vp, _P(_d)]),
    "n2p2_training_set_weights": (_i, [_vp, _P(_d)]),
    "n2p2_lammps_create": (_i, [_P(_vp), _i]),
    "n2p2_lammps_destroy": (_i, [_vp]),
    "n2p2_lammps_initialize": (_i, [_vp, _cp, _cp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    _d, _d, _d, ctypes.c_int32, ctypes.c_int32]),
    "n2p2_lammps_set_precision": (_i, [_vp, _i]),
    "n2p2_lammps_get_max_cutoff_radius": (_i, [_vp, _P(_d)]),
    "n2p2_lammps_set_local_atoms": (_i, [_vp, ctypes.c_int32, _vp]),
    "n2p2_lammps_add_neighbor": (_i, [_vp, ctypes.c_int32, ctypes.c_int32, _i64, ctypes.c_int32, _d, _d, _d, _d]),
    "n2p2_lammps_transfer_neighbor_list": (_i, [_vp, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp, _d]),
    "n2p2_lammps_process": (_i, [_vp]),
    "n2p2_lammps_get_energy": (_i, [_vp, _P(_d)]),
    "n2p2_lammps_get_atomic_energy": (_i, [_vp, ctypes.c_int32, _P(_d)]),
    "n2p2_lammps_get_forces": (_i, [_vp, _vp]),
    "n2p2_lammps_get_num_extrapolation_warnings": (_i, [_vp, _P(_i64)]),
    "n2p2_lammps_clear_extrapolation_warnings": (_i, [_vp]),
    "n2p2_batch_get_symmetry_function_statistics": (_i, [_vp, _P(_i64), _P(_d)]),
    "n2p2_structures_read_file": (_i, [_cp, _i64, _P(_vp)]),
    "n2p2_structures_read_text": (_i, [_cp, _i64, _i64, _P(_vp)]),
    "n2p2_structures_destroy": (_i, [_vp]),
    "n2p2_structures_get_count": (_i, [_vp, _P(_i64), _P(_i64)]),
    "n2p2_structures_get_structure_arrays": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "n2p2_structures_get_atom_arrays": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "n2p2_structures_get_comment": (_i, [_vp, _i64, _vp, ctypes.c_int32]),
    "n2p2_host_alloc": (_i, [_P(_vp), ctypes.c_size_t]),
    "n2p2_host_free": (_i, [_vp]),
}

_lib = None


class N2P2Error(RuntimeError):
    """Raised for a non-zero status; `code` is the C status (std::runtime_error)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class OutOfRangeError(N2P2Error):
    """std::out_of_range: evaluation stopped on an extrapolation warning."""


class RangeError(N2P2Error):
    """std::range_error."""


class InvalidArgumentError(N2P2Error, ValueError):
    """std::invalid_argument (e.g. cutoff parameters)."""


def load():
    """Load and declare the shared library (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m n2p2_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(status):
    if status != OK:
        msg = load().n2p2_last_error().decode(errors="replace")
        cls = {ERR_OUT_OF_RANGE: OutOfRangeError, ERR_RANGE: RangeError,
               ERR_INVALID_ARGUMENT: InvalidArgumentError}.get(status, N2P2Error)
        raise cls(status, msg)
    return status
