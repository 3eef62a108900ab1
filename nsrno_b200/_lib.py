"""ctypes binding of ``libnsrno_b200.so`` (the C ABI declared in include/nsrno_b200.h).

The reference binds its native kernels the same way (nsrno/native_time.py:25-41:
``ctypes.CDLL``, integer status codes raised as ``RuntimeError``).  There is no
fallback: if the library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "libnsrno_b200.so"

CONVERGED, ITERATION_BUDGET, BREAKDOWN, DIVERGED, NONFINITE, TIMEOUT, NOT_RUN = range(7)
REASONS = {CONVERGED: "converged", ITERATION_BUDGET: "iteration_budget", BREAKDOWN: "breakdown",
           DIVERGED: "diverged", NONFINITE: "nonfinite", TIMEOUT: "timeout", NOT_RUN: "not_run"}
ERR_TIMEOUT = 1006

EXPORTS = ("nsr_version", "nsr_error_string", "nsr_material_bytes", "nsr_setup_material", "nsr_apply",
           "nsr_precondition_workspace_size", "nsr_precondition", "nsr_precondition_noalloc", "nsr_plane_wave_rhs",
           "nsr_solve_workspace_size", "nsr_solve_batched", "nsr_solve_batched_sync", "nsr_solve_progress",
           "nsr_solve_progress_offset",
           "nsr_gmres_workspace_size", "nsr_gmres_batched",
           "nsr_grad_accum", "nsr_dense_coef_bytes", "nsr_dense_workspace_size", "nsr_dense_apply",
           "nsr_learned_state_bytes", "nsr_learned_setup", "nsr_learned_precondition",
           "nsr_learned_backward_workspace_size", "nsr_learned_map_backward", "nsr_learned_network_backward",
           "nsr_learned_spectral_workspace_size", "nsr_learned_spectral_backward", "nsr_learned_adam",
           "nsr_tangent_rhs", "nsr_dense_precondition_workspace_size", "nsr_dense_precondition", "nsr_band_rf",
           "nsr_true_residual_workspace_size", "nsr_true_residual", "nsr_dense_solve_workspace_size",
           "nsr_learned_setup_ex", "nsr_learned_map_backward_ex", "nsr_learned_network_backward_ex",
           "nsr_dense_grad",
           "nsr_dense_solve")

LEARNED_PARAMS = 3645
LEARNED_FP32, LEARNED_BF16 = 0, 1
PRECISIONS = {"fp32": LEARNED_FP32, "bf16": LEARNED_BF16}


class NsrGrid(ctypes.Structure):
    _fields_ = [("nz", ctypes.c_int32), ("nx", ctypes.c_int32), ("n_pml", ctypes.c_int32),
                ("face", ctypes.c_int32), ("h", ctypes.c_double), ("c0", ctypes.c_double),
                ("rho0", ctypes.c_double), ("pml_strength", ctypes.c_double),
                ("alpha_power", ctypes.c_double), ("aperture_half_width", ctypes.c_double)]


class NsrLearned(ctypes.Structure):
    _fields_ = [("params", ctypes.c_void_p), ("gains", ctypes.c_void_p), ("gain_index", ctypes.c_void_p),
                ("n_gain", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class NsrTiles(ctypes.Structure):
    _fields_ = [("stencil_width", ctypes.c_int32), ("stencil_depth", ctypes.c_int32),
                ("stencil_rows", ctypes.c_int32), ("stencil_ctas", ctypes.c_int32),
                ("cols_width", ctypes.c_int32), ("row_tile", ctypes.c_int32),
                ("slot_groups", ctypes.c_int32), ("stencil_cols", ctypes.c_int32), ("cols_staged", ctypes.c_int32),
                ("rows_staged", ctypes.c_int32), ("reserved", ctypes.c_int32 * 2)]

    FIELDS = ("stencil_width", "stencil_depth", "stencil_rows", "stencil_ctas", "cols_width", "row_tile",
              "slot_groups", "stencil_cols", "cols_staged", "rows_staged")

    def as_dict(self):
        return {k: int(getattr(self, k)) for k in self.FIELDS}


class NsrSolveParams(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("shift", ctypes.c_double), ("restart_factor", ctypes.c_double),
                ("warm_gate", ctypes.c_double), ("max_iterations", ctypes.c_int32), ("replace_every", ctypes.c_int32),
                ("n_slots", ctypes.c_int32), ("adjoint", ctypes.c_int32),
                ("graph_iterations", ctypes.c_int32), ("profile_iterations", ctypes.c_int32),
                ("fields_fp64", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("learned", ctypes.POINTER(NsrLearned)), ("time_limit_s", ctypes.c_double),
                ("tiles", ctypes.POINTER(NsrTiles))]


class NsrDenseGrid(ctypes.Structure):
    _fields_ = [("H", ctypes.c_int32), ("W", ctypes.c_int32), ("pz", ctypes.c_int32), ("px", ctypes.c_int32),
                ("h", ctypes.c_int32), ("w", ctypes.c_int32), ("dx", ctypes.c_double)]


class NsrGmresParams(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("shift", ctypes.c_double),
                ("max_iterations", ctypes.c_int32), ("restart", ctypes.c_int32),
                ("n_slots", ctypes.c_int32), ("adjoint", ctypes.c_int32),
                ("fields_fp64", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("learned", ctypes.POINTER(NsrLearned))]


class NsrDenseSolveParams(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("shift", ctypes.c_double), ("k0dx2", ctypes.c_double),
                ("scal_re", ctypes.c_double), ("scal_im", ctypes.c_double), ("restart", ctypes.c_int32),
                ("max_cycles", ctypes.c_int32), ("adjoint", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class NsrDenseSolveInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("steps", ctypes.c_int32), ("cycles", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("residual", ctypes.c_double)]


class NsrSolveStats(ctypes.Structure):
    _fields_ = [("loop_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double * 16),
                ("kernel_timed", ctypes.c_int32 * 16), ("launches", ctypes.c_int64),
                ("graph_launches", ctypes.c_int32), ("warm_accepted", ctypes.c_int32),
                ("warm_rejected", ctypes.c_int32), ("reserved", ctypes.c_int32)]

    KERNELS = ("fwd_h0", "cols_h0", "rinv_h0", "inv_h0", "fwd_h1", "cols_h1", "rinv_h1", "res_h1", "inv_h1")

    def as_dict(self):
        return dict(loop_ms=self.loop_ms, launches=int(self.launches), graph_launches=int(self.graph_launches),
                    warm_accepted=int(self.warm_accepted), warm_rejected=int(self.warm_rejected),
                    kernel_ms={k: self.kernel_ms[i] for i, k in enumerate(self.KERNELS)},
                    kernel_timed={k: int(self.kernel_timed[i]) for i, k in enumerate(self.KERNELS)})


_lib = None


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY.exists():
        raise RuntimeError(f"{LIBRARY} is missing: run `python -m nsrno_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(str(LIBRARY))
    P, I, D, S = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_size_t
    G = ctypes.POINTER(NsrGrid)
    lib.nsr_version.restype = ctypes.c_int
    lib.nsr_error_string.restype = ctypes.c_char_p
    lib.nsr_error_string.argtypes = [ctypes.c_int]
    lib.nsr_material_bytes.restype = S
    lib.nsr_material_bytes.argtypes = [G]
    lib.nsr_setup_material.argtypes = [G, P, P, P, P, P]
    lib.nsr_apply.argtypes = [G, P, P, I, I, I, P, P, P]
    lib.nsr_precondition_workspace_size.restype = S
    lib.nsr_precondition_workspace_size.argtypes = [G, I]
    lib.nsr_precondition.argtypes = [G, P, I, D, I, P, P, P, S, P]
    lib.nsr_precondition_noalloc.argtypes = [G, P, I, D, I, P, P, P]
    lib.nsr_plane_wave_rhs.argtypes = [G, P, P, I, P, P]
    lib.nsr_solve_workspace_size.restype = S
    lib.nsr_solve_workspace_size.argtypes = [G, I]
    lib.nsr_solve_batched.argtypes = [G, P, P, P, I, P, P, P, I, ctypes.POINTER(NsrSolveParams),
                                      P, S, P, P, P, P, P, ctypes.POINTER(NsrSolveStats), P]
    lib.nsr_solve_batched_sync.argtypes = lib.nsr_solve_batched.argtypes
    lib.nsr_solve_progress.argtypes = [G, I, P, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_int32), P]
    lib.nsr_solve_progress_offset.restype = S
    lib.nsr_solve_progress_offset.argtypes = [G, I]
    lib.nsr_grad_accum.argtypes = [G, P, P, I, I, P, P, P, P, P]
    lib.nsr_tangent_rhs.argtypes = [G, P, P, I, I, P, P, P, P, P]
    lib.nsr_band_rf.argtypes = [I, I, I, P, P, P, P]
    lib.nsr_true_residual_workspace_size.restype = S
    lib.nsr_true_residual_workspace_size.argtypes = [G, I]
    lib.nsr_true_residual.argtypes = [G, P, P, P, I, I, P, P, P, P, S, P]
    lib.nsr_gmres_workspace_size.restype = S
    lib.nsr_gmres_workspace_size.argtypes = [G, I, I]
    lib.nsr_gmres_batched.argtypes = [G, P, P, P, I, P, P, P, I, ctypes.POINTER(NsrGmresParams),
                                      P, S, P, P, P, P, P, P]
    DG = ctypes.POINTER(NsrDenseGrid)
    lib.nsr_dense_coef_bytes.restype = S
    lib.nsr_dense_coef_bytes.argtypes = [DG]
    lib.nsr_dense_workspace_size.restype = S
    lib.nsr_dense_workspace_size.argtypes = [DG, I, I]
    lib.nsr_dense_apply.argtypes = [DG, P, D, D, I, I, I, P, P, P, S, P]
    lib.nsr_dense_precondition_workspace_size.restype = S
    lib.nsr_dense_precondition_workspace_size.argtypes = [DG, I]
    lib.nsr_dense_precondition.argtypes = [DG, D, D, I, I, P, P, P, S, P]
    lib.nsr_dense_grad.argtypes = [DG, P, D, D, I, P, P, P, P, P, P]
    lib.nsr_dense_solve_workspace_size.restype = S
    lib.nsr_dense_solve_workspace_size.argtypes = [DG, I, I]
    lib.nsr_dense_solve.argtypes = [DG, P, ctypes.POINTER(NsrDenseSolveParams), I, P, P, P,
                                    ctypes.POINTER(NsrDenseSolveInfo), P, S, P]
    L = ctypes.POINTER(NsrLearned)
    lib.nsr_learned_state_bytes.restype = S
    lib.nsr_learned_state_bytes.argtypes = [G, I]
    lib.nsr_learned_setup.argtypes = [G, P, P, P, P, I, P, P, P, P]
    lib.nsr_learned_setup_ex.argtypes = [G, P, P, P, P, I, P, I, P, P, P]
    lib.nsr_learned_precondition.argtypes = [G, L, P, I, I, P, P, P, S, P]
    lib.nsr_learned_backward_workspace_size.restype = S
    lib.nsr_learned_backward_workspace_size.argtypes = [G, I]
    lib.nsr_learned_map_backward.argtypes = [G, P, I, P, P, P, P, S, P]
    lib.nsr_learned_network_backward.argtypes = [G, P, P, I, P, P, P, S, P]
    lib.nsr_learned_map_backward_ex.argtypes = [G, P, I, I, P, P, P, P, S, P]
    lib.nsr_learned_network_backward_ex.argtypes = [G, P, P, I, I, P, P, P, S, P]
    lib.nsr_learned_spectral_workspace_size.restype = S
    lib.nsr_learned_spectral_workspace_size.argtypes = [G, I]
    lib.nsr_learned_spectral_backward.argtypes = [G, P, P, I, P, P, P, P, S, P]
    lib.nsr_learned_adam.argtypes = [P, P, P, P, I, I, D, D, D, D, D, P, P]
    for name in EXPORTS:
        getattr(lib, name)
    _lib = lib
    return lib


def check(code):
    """Raise ``RuntimeError(nsr_error_string(code))`` for a non-zero return code."""
    if code:
        raise RuntimeError(load().nsr_error_string(int(code)).decode())
    return code
