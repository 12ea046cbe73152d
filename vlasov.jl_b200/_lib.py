"""ctypes binding of the C ABI (include/vlasov_b200.h).

The shared library lives in-tree at ``vlasov.jl_b200/lib/libvlasov_b200.so``.
Loading fails loudly when it is missing: there is no CPU fallback for the
product path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libvlasov_b200.so"

VLB_OK = 0
VLB_ERR_ARG = -1
VLB_ERR_CUDA = -2
VLB_ERR_STATE = -3
VLB_ERR_TIMEOUT = -4
VLB_ERR_NOMEM = -5

VLB_DEPOSIT_FLOAT32 = 0
VLB_DEPOSIT_FIXED64 = 1

VLB_GRID_RHO_FINE = 0
VLB_GRID_RHO_COARSE = 1
VLB_GRID_PHI_FINE = 2
VLB_GRID_PHI_COARSE = 3
VLB_GRID_CSOL_FINE = 4
VLB_GRID_CSOL_COARSE = 5
VLB_GRID_CSOL_HARTREE_FINE = 6
VLB_GRID_CSOL_HARTREE_COARSE = 7

VLB_POISSON_FP32 = 0
VLB_POISSON_3XTF32 = 1
VLB_POISSON_BF16X3 = 2
VLB_ENERGY_TOTAL = 0
VLB_ENERGY_HARTREE = 1
VLB_SOFTENING_DEVICE = 0
VLB_SOFTENING_BALL = 1
VLB_STATUS_SCAN_TIMEOUT = 1
VLB_STATUS_BAD_CELL = 2
VLB_STATUS_OVERFLOW = 4
VLB_STATUS_MMA_TIMEOUT = 8

# every symbol include/vlasov_b200.h declares
EXPORTS = (
    "vlb_last_error", "vlb_version", "vlb_create", "vlb_destroy", "vlb_upload_particles",
    "vlb_download_particles", "vlb_sort", "vlb_get_sort", "vlb_get_sort_sizes", "vlb_deposit_fine", "vlb_deposit_coarse",
    "vlb_poisson", "vlb_set_precision", "vlb_coefficients", "vlb_mean_field", "vlb_forces", "vlb_projectile_forces",
    "vlb_push", "vlb_step", "vlb_interaction_energy", "vlb_film_reserve", "vlb_film_frames", "vlb_film_download",
    "vlb_film_clear", "vlb_dn_weight_count", "vlb_set_denoiser", "vlb_clear_denoiser", "vlb_dn_create",
    "vlb_dn_destroy", "vlb_dn_forward", "vlb_dn_gradient", "vlb_dn_adam", "vlb_dn_status", "vlb_dn_active_tiles", "vlb_set_tuning", "vlb_get_tuning", "vlb_batch_create", "vlb_batch_step",
    "vlb_batch_destroy", "vlb_exchange_buffers", "vlb_step_deposit", "vlb_step_fields", "vlb_step_advance",
    "vlb_get_grid", "vlb_set_grid", "vlb_get_forces", "vlb_set_forces",
    "vlb_enclosed_charge", "vlb_profile", "vlb_stage_count", "vlb_stage_name", "vlb_stage_times",
    "vlb_launch_count", "vlb_fp32_peak", "vlb_stream", "vlb_sample_thomas_fermi", "vlb_ran2", "vlb_pack_positions",
    "vlb_unpack_positions", "vlb_total_charge_noalloc", "vlb_upload_particles_range",
    "vlb_download_particles_range", "vlb_get_forces_range", "vlb_sampler_create", "vlb_sampler_draw",
    "vlb_sampler_destroy",
)

P_D = C.POINTER(C.c_double)
P_F = C.POINTER(C.c_float)
P_I = C.POINTER(C.c_int32)


class LevelDesc(C.Structure):
    _fields_ = [("nknots", C.c_int32), ("knots", P_D), ("colloc", P_D), ("sinv", P_D),
                ("laplacian", P_D), ("eigvec", P_D), ("eigvec_inv", P_D), ("eigval", P_D),
                ("dual_moments", P_D), ("dual_lengths", P_D), ("locate_x0", C.c_double),
                ("locate_invwidth", C.c_double), ("locate_ncells", C.c_int32), ("locate_cells", P_I)]


class SmoothingDesc(C.Structure):
    _fields_ = [("nbdt", C.c_int32), ("spacing", C.c_double), ("overlap", P_D), ("gradient", P_D),
                ("nodes", P_D)]


class Config(C.Structure):
    _fields_ = [("npart", C.c_int64), ("weight", C.c_double), ("fine", LevelDesc), ("coarse", LevelDesc),
                ("smoothing", SmoothingDesc), ("device", C.c_int32), ("flags", C.c_int32)]


class ProjectileDesc(C.Structure):
    _fields_ = [("position", C.c_double * 3), ("previous", C.c_double * 3), ("velocity", C.c_double * 3),
                ("charge", C.c_double), ("mass", C.c_double), ("sigma", C.c_double),
                ("ball_radius", C.c_double), ("active", C.c_int32), ("softening", C.c_int32)]


class StepParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("rcmax", C.c_double), ("jellium_nions", C.c_double),
                ("jellium_radius", C.c_double), ("capture_radius", C.c_double), ("deposit_mode", C.c_int32),
                ("advance_projectile", C.c_int32), ("push", C.c_int32), ("use_graph", C.c_int32),
                ("poisson_precision", C.c_int32), ("denoise", C.c_int32), ("energy", C.c_int32),
                ("film", C.c_int32)]


class StepResult(C.Structure):
    _fields_ = [("kinetic", C.c_double), ("escaped", C.c_double), ("angular", C.c_double * 3),
                ("projectile_force", C.c_double * 3), ("e_electrons", C.c_double), ("e_jellium", C.c_double),
                ("enclosed_charge", C.c_double), ("total_charge", C.c_double), ("nout", C.c_int32),
                ("outcount", C.c_int32), ("noccupied", C.c_int32), ("status", C.c_int32),
                ("denoised", C.c_int32), ("sort_path", C.c_int32), ("hartree", C.c_double),
                ("interaction", C.c_double)]


class Exchange(C.Structure):
    _fields_ = [("rho_fine", C.c_void_p), ("rho_fine_dtype", C.c_int32), ("pad0_", C.c_int32),
                ("rho_fine_count", C.c_int64), ("rho_coarse", C.c_void_p), ("rho_coarse_dtype", C.c_int32),
                ("pad3_", C.c_int32), ("rho_coarse_count", C.c_int64),
                ("scalars", C.c_void_p), ("scalars_count", C.c_int32), ("pad1_", C.c_int32),
                ("reaction", C.c_void_p), ("reaction_count", C.c_int32), ("pad2_", C.c_int32),
                ("stream", C.c_void_p)]


VLB_DTYPE_FLOAT32 = 0
VLB_DTYPE_INT64 = 1


class Tuning(C.Structure):
    _fields_ = [("chunk", C.c_int32), ("field_ctas_per_sm", C.c_int32), ("cic_ctas_per_sm", C.c_int32),
                ("push_ctas_per_sm", C.c_int32), ("move_ctas_per_sm", C.c_int32),
                ("field_tensor_cores", C.c_int32), ("scan_wait_polls", C.c_int32), ("reserved", C.c_int32 * 1)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "reserved"}


class VlbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"vlb error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with vlasov.jl_b200/build.py "
                               "(the device path has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        sig = {
            "vlb_last_error": (C.c_char_p, []),
            "vlb_version": (C.c_char_p, []),
            "vlb_create": (C.c_int, [C.POINTER(Config), C.POINTER(vp)]),
            "vlb_destroy": (C.c_int, [vp]),
            "vlb_upload_particles": (C.c_int, [vp, P_I, P_F, P_I, P_F]),
            "vlb_download_particles": (C.c_int, [vp, P_I, P_F, P_I, P_F]),
            "vlb_sort": (C.c_int, [vp, P_I, P_I]),
            "vlb_get_sort": (C.c_int, [vp, P_I, P_I, P_I, P_I]),
            "vlb_get_sort_sizes": (C.c_int, [vp, P_I, P_I]),
            "vlb_deposit_fine": (C.c_int, [vp, C.c_double, C.c_int32, P_I, P_D]),
            "vlb_deposit_coarse": (C.c_int, [vp, C.c_double]),
            "vlb_poisson": (C.c_int, [vp, C.c_int32]),
            "vlb_set_precision": (C.c_int, [vp, C.c_int32]),
            "vlb_coefficients": (C.c_int, [vp, C.c_int32]),
            "vlb_mean_field": (C.c_int, [vp, C.c_int32, C.c_double, C.c_double]),
            "vlb_forces": (C.c_int, [vp, C.POINTER(ProjectileDesc), P_D, P_I]),
            "vlb_projectile_forces": (C.c_int, [vp, C.POINTER(ProjectileDesc), C.c_double, C.c_double, P_D,
                                                P_D, P_D]),
            "vlb_push": (C.c_int, [vp, C.c_double, C.c_double, P_D]),
            "vlb_step": (C.c_int, [vp, C.POINTER(ProjectileDesc), C.POINTER(StepParams), C.POINTER(StepResult)]),
            "vlb_exchange_buffers": (C.c_int, [vp, C.c_int32, C.POINTER(Exchange)]),
            "vlb_interaction_energy": (C.c_int, [vp, C.c_int32, P_D]),
            "vlb_film_reserve": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, C.c_double]),
            "vlb_film_frames": (C.c_int, [vp, P_I, P_I]),
            "vlb_film_download": (C.c_int, [vp, C.c_int32, C.c_int32, P_F, P_D]),
            "vlb_film_clear": (C.c_int, [vp]),
            "vlb_dn_weight_count": (C.c_int, []),
            "vlb_set_denoiser": (C.c_int, [vp, P_F, C.c_int32, C.c_double, C.c_double]),
            "vlb_clear_denoiser": (C.c_int, [vp]),
            "vlb_dn_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(vp)]),
            "vlb_dn_destroy": (C.c_int, [vp]),
            "vlb_dn_forward": (C.c_int, [vp, vp, C.c_float, vp, vp, vp]),
            "vlb_dn_gradient": (C.c_int, [vp, vp, vp, C.c_float, vp, vp, C.POINTER(C.c_double), vp]),
            "vlb_dn_adam": (C.c_int, [vp, vp, vp, vp, vp, C.c_float, C.c_int32, vp]),
            "vlb_dn_status": (C.c_int, [vp, P_I]),
            "vlb_dn_active_tiles": (C.c_int, [vp, P_I]),
            "vlb_set_tuning": (C.c_int, [vp, C.POINTER(Tuning)]),
            "vlb_get_tuning": (C.c_int, [vp, C.POINTER(Tuning)]),
            "vlb_batch_create": (C.c_int, [C.POINTER(vp), C.c_int32, C.POINTER(vp)]),
            "vlb_batch_step": (C.c_int, [vp, C.POINTER(ProjectileDesc), C.POINTER(StepParams), C.POINTER(StepResult)]),
            "vlb_batch_destroy": (C.c_int, [vp]),
            "vlb_step_deposit": (C.c_int, [vp, C.POINTER(ProjectileDesc), C.POINTER(StepParams)]),
            "vlb_step_fields": (C.c_int, [vp, C.POINTER(StepParams), C.c_int64]),
            "vlb_step_advance": (C.c_int, [vp, C.POINTER(ProjectileDesc), C.POINTER(StepParams),
                                           C.POINTER(StepResult)]),
            "vlb_get_grid": (C.c_int, [vp, C.c_int32, P_F]),
            "vlb_set_grid": (C.c_int, [vp, C.c_int32, P_F]),
            "vlb_get_forces": (C.c_int, [vp, P_F]),
            "vlb_set_forces": (C.c_int, [vp, P_F]),
            "vlb_enclosed_charge": (C.c_int, [vp, P_D, C.c_double, P_D]),
            "vlb_profile": (C.c_int, [vp, C.c_int32]),
            "vlb_stage_count": (C.c_int, []),
            "vlb_stage_name": (C.c_char_p, [C.c_int32]),
            "vlb_stage_times": (C.c_int, [vp, P_D, C.c_int32]),
            "vlb_launch_count": (C.c_int, [vp, C.POINTER(C.c_int64)]),
            "vlb_stream": (C.c_int, [vp, C.POINTER(vp)]),
            "vlb_fp32_peak": (C.c_int, [C.c_int32, P_D]),
            "vlb_sample_thomas_fermi": (C.c_int, [P_D, C.c_int32, P_D, C.c_int32, C.c_double, C.c_int64,
                                                  C.c_double, C.c_int32, C.c_int32, P_D, P_D]),
            "vlb_ran2": (C.c_int, [C.c_int32, C.c_int32, C.c_int64, P_F]),
            "vlb_pack_positions": (C.c_int, [C.c_int64, P_D, C.c_double, C.c_double, P_I, P_F]),
            "vlb_unpack_positions": (C.c_int, [C.c_int64, P_I, P_F, C.c_double, C.c_double, P_D]),
            "vlb_total_charge_noalloc": (C.c_int, [vp, vp, C.c_int32, vp, vp]),
            "vlb_upload_particles_range": (C.c_int, [vp, C.c_int64, C.c_int64, P_I, P_F, P_I, P_F]),
            "vlb_download_particles_range": (C.c_int, [vp, C.c_int64, C.c_int64, P_I, P_F, P_I, P_F]),
            "vlb_get_forces_range": (C.c_int, [vp, C.c_int64, C.c_int64, P_F]),
            "vlb_sampler_create": (C.c_int, [P_D, C.c_int32, P_D, C.c_int32, C.c_double, C.c_double, C.c_int32,
                                             C.c_int32, C.POINTER(vp)]),
            "vlb_sampler_draw": (C.c_int, [vp, C.c_int64, P_D, P_D]),
            "vlb_sampler_destroy": (C.c_int, [vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int):
    if rc != VLB_OK:
        raise VlbError(rc, lib().vlb_last_error().decode())


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def pd(a):
    return ptr(a, C.c_double)


def pf(a):
    return ptr(a, C.c_float)


def pi(a):
    return ptr(a, C.c_int32)
