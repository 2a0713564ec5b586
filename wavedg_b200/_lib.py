"""ctypes binding of libwdg_b200.so (declarations in include/wdg_b200.h).

The library is loaded from the package directory.  There is no fallback: if
it is missing, every entry point raises, naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# WDG_B200_LIB selects another build of the library (e.g. one compiled with different options)
PACKAGE_LIB = os.path.join(HERE, "libwdg_b200.so")
LIB_PATH = os.environ.get("WDG_B200_LIB") or PACKAGE_LIB
HEADER = os.path.join(ROOT, "include", "wdg_b200.h")

WDG_OK = 0
WDG_ERR_ARG = -1
WDG_ERR_CUDA = -2
WDG_ERR_ALLOC = -3
WDG_ERR_TIMEOUT = -4
WDG_ERR_UNSUPPORTED = -5
WDG_ERR_NOT_CONVERGED = -6
WDG_INTERIOR, WDG_BOUNDARY = 0, 1
WDG_FP64, WDG_FP32 = 0, 1


class WdgError(RuntimeError):
    """A C-ABI call returned a negative status (the reference's wdg_error throws std::runtime_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_v, _i, _d, _ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
_vp = C.POINTER(C.c_void_p)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

SIGNATURES = {
    "wdg_last_error": ([], C.c_char_p),
    "wdg_version": ([], _i),
    "wdg_supported_degrees": ([_ip, _i], _i),
    "wdg_mesh_from_vertices": ([_i, _v, _i, _v, _vp], _i),
    "wdg_mesh_uniform_rect": ([_i, _d, _d, _i, _d, _d, _vp], _i),
    "wdg_mesh_from_file": ([C.c_char_p, _vp], _i),
    "wdg_waveq_create": ([_v, _i, _v, _i, _vp], _i),
    "wdg_waveq_destroy": ([_v], None),
    "wdg_waveq_rules": ([_v, _v, _v, _v], _i),
    "wdg_waveq_wave": ([_v, _vp], _i),
    "wdg_waveq_div_action": ([_v, _v, _v], _i),
    "wdg_waveq_wave_action": ([_v, _v, _v], _i),
    "wdg_waveq_wavebc_action": ([_v, _v, _v], _i),
    "wdg_waveq_edge_flux": ([_v, _i, _v, _v], _i),
    "wdg_waveq_mass_action": ([_v, _i, _v, _v], _i),
    "wdg_waveq_mass_inv": ([_v, _i, _v], _i),
    "wdg_waveq_rhs": ([_v, _v, _v, _v, _d], _i),
    "wdg_waveq_rk4_steps": ([_v, _v, _d, _v, _i], _i),
    "wdg_waveholtz_create_exact": ([_v, _d, _vp], _i),
    "wdg_mesh_partner_table": ([_v, _i, _v, _v, _v], _i),
    "wdg_advect_create": ([_v, _i, _i, _v, _i, _vp], _i),
    "wdg_advect_destroy": ([_v], None),
    "wdg_advect_action": ([_v, _v, _v], _i),
    "wdg_advect_bc_action": ([_v, _v, _v], _i),
    "wdg_advect_rhs": ([_v, _v, _v], _i),
    "wdg_advect_rk4_steps": ([_v, _v, _d, _v, _i], _i),
    "wdg_massmatrix_create": ([_v, _i, _i, _i, _i, _vp], _i),
    "wdg_massmatrix_destroy": ([_v], None),
    "wdg_massmatrix_set_stream": ([_v, _v], _i),
    "wdg_massmatrix_action": ([_v, _i, _v, _v], _i),
    "wdg_massmatrix_inv": ([_v, _i, _v], _i),
    "wdg_massmatrix_points": ([_v, _v], _i),
    "wdg_massmatrix_load": ([_v, _i, _v, _v], _i),
    "wdg_vadvect_create": ([_v, _i, _i, _i, _v, _i, _i, _vp], _i),
    "wdg_vadvect_destroy": ([_v], None),
    "wdg_vadvect_set_stream": ([_v, _v], _i),
    "wdg_vadvect_sync": ([_v], _i),
    "wdg_vadvect_action": ([_v, _v, _v], _i),
    "wdg_vadvect_bc_action": ([_v, _v, _v], _i),
    "wdg_vadvect_rhs": ([_v, _v, _v], _i),
    "wdg_vadvect_steps": ([_v, _i, _v, _d, _dp, _i], _i),
    "wdg_euler_create": ([_v, _i, _i, _vp], _i),
    "wdg_euler_create_exact": ([_v, _i, _i, _vp], _i),
    "wdg_claw_destroy": ([_v], None),
    "wdg_claw_set_stream": ([_v, _v], _i),
    "wdg_claw_sync": ([_v], _i),
    "wdg_claw_div": ([_v, _v, _v], _i),
    "wdg_claw_flux": ([_v, _i, _v, _v], _i),
    "wdg_claw_rhs": ([_v, _v, _v], _i),
    "wdg_claw_steps": ([_v, _i, _v, _d, _dp, _i], _i),
    "wdg_wave_create_halo": ([_v, _i, _v, _i, _i, _i, _v, _v, _vp], _i),
    "wdg_halo_info": ([_v, _v, _v], _i),
    "wdg_halo_gather": ([_v, _i, _v, _i, _v], _i),
    "wdg_halo_put": ([_v, _i, _ll, _v, _ll], _i),
    "wdg_rk4_stage": ([_v, _i, _d], _i),
    "wdg_rk4_stage_forced": ([_v, _i, _d, _d, _v, _d, _v, _d], _i),
    "wdg_rk4_stage_elems": ([_v, _i, _d, _d, _v, _d, _v, _d, _i, _i], _i),
    "wdg_mesh_partition": ([_v, _i, _i, _v], _i),
    "wdg_write_raw": ([C.c_char_p, _ll, _v], _i),
    "wdg_read_raw": ([C.c_char_p, _ll, _v], _i),
    "wdg_mesh_from_tables": ([_i, _v, _i, _v, _i, _v, _vp], _i),
    "wdg_mesh_destroy": ([_v], None),
    "wdg_mesh_n_elem": ([_v], _i),
    "wdg_mesh_n_edges": ([_v, _i], _i),
    "wdg_mesh_edges": ([_v, _i, _v], _i),
    "wdg_mesh_min_h": ([_v, _dp], _i),
    "wdg_mesh_boundary_midpoints": ([_v, _v], _i),
    "wdg_gauss_lobatto": ([_i, _v, _v, _v], _i),
    "wdg_wave_create": ([_v, _i, _v, _i, _i, _vp], _i),
    "wdg_wave_destroy": ([_v], None),
    "wdg_wave_info": ([_v, _ip, _ip, C.POINTER(_ll), _ip], _i),
    "wdg_wave_set_stream": ([_v, _v], _i),
    "wdg_wave_sync": ([_v], _i),
    "wdg_wave_set_tile": ([_v, _i], _i),
    "wdg_wave_get_tile": ([_v, _ip], _i),
    "wdg_wave_set_max_ctas": ([_v, _i], _i),
    "wdg_wave_set_stages": ([_v, _i], _i),
    "wdg_wave_set_kernel": ([_v, _i], _i),
    "wdg_wave_get_launch": ([_v, _ip, _ip, _ip, _ip], _i),
    "wdg_wave_autotune": ([_v, _i, C.POINTER(C.c_float)], _i),
    "wdg_wave_node_coords": ([_v, _v], _i),
    "wdg_wave_set_wait_limit": ([_v, _d], _i),
    "wdg_test_skip_chunk": ([_v, _i], _i),
    "wdg_test_set_partner": ([_v, _i, _i, _i, _ip], _i),
    "wdg_div_action": ([_v, _v, _v], _i),
    "wdg_wave_action": ([_v, _v, _v], _i),
    "wdg_wavebc_action": ([_v, _v, _v], _i),
    "wdg_face_prolong": ([_v, _i, _v, _v], _i),
    "wdg_face_prolong_t": ([_v, _i, _v, _v], _i),
    "wdg_edge_flux": ([_v, _i, _v, _v], _i),
    "wdg_apply_bc": ([_v, _v], _i),
    "wdg_mass_action": ([_v, _i, _v, _v], _i),
    "wdg_mass_inv": ([_v, _i, _v], _i),
    "wdg_rhs": ([_v, _v, _v, _v, _d], _i),
    "wdg_rk4_steps": ([_v, _v, _d, _dp, _i], _i),
    "wdg_state_upload": ([_v, _v], _i),
    "wdg_state_download": ([_v, _v], _i),
    "wdg_state_device_ptr": ([_v, _vp], _i),
    "wdg_state_rk4_steps": ([_v, _d, _dp, _i], _i),
    "wdg_state_energy": ([_v, _dp], _i),
    "wdg_quad_points": ([_v, _v], _i),
    "wdg_linear_functional": ([_v, _i, _v, _v], _i),
    "wdg_load_gaussians": ([_v, _i, _v, _v, _v, _v, _d, _i, _i, _v], _i),
    "wdg_load_gaussians_noalloc": ([_v, _i, _v, _v, _v, _v, _d, _i, _i, _v], _i),
    "wdg_norm": ([_v, _v, _dp], _i),
    "wdg_error": ([_v, _v, _v, _dp], _i),
    "wdg_waveholtz_create": ([_v, _d, _vp], _i),
    "wdg_waveholtz_destroy": ([_v], None),
    "wdg_waveholtz_params": ([_v, _dp, _dp, _ip], _i),
    "wdg_waveholtz_pi0": ([_v, _v, _v], _i),
    "wdg_waveholtz_S": ([_v, _v], _i),
    "wdg_waveholtz_postprocess": ([_v, _v, _v], _i),
    "wdg_waveholtz_solve": ([_v, _v, _d, _i, _v, _ip, _dp], _i),
    "wdg_whbatch_create": ([_i, _v, _v, _vp], _i),
    "wdg_whbatch_destroy": ([_v], None),
    "wdg_whbatch_params": ([_v, _i, _dp, _dp, _ip], _i),
    "wdg_whbatch_set_launch": ([_v, _i, _i], _i),
    "wdg_whbatch_get_launch": ([_v, _ip, _ip, _ip], _i),
    "wdg_whbatch_autotune": ([_v, _i, C.POINTER(C.c_float)], _i),
    "wdg_whbatch_solve": ([_v, _v, _d, _i, _i, _v, _v, _v, _v, _v, _v], _i),
    # learned warm start (include/wdg_fno.h)
    "wdg_fno_gemm": ([_v, _v, _v, _i, _i, _i, _ll, _ll, _ll, _ll, _ll, _ll, _i, _i, _i, C.c_float, C.c_float, _i,
                      _v], _i),
    "wdg_fno_dft_y": ([_v, _v, _v, _v, _v, _i, _i, _i, _i, _i, C.c_float, _v], _i),
    "wdg_fno_mix": ([_v, _v, _v, _i, _i, _i, _i, _v], _i),
    "wdg_fno_mix_bwd": ([_v, _v, _v, _v, _v, _i, _i, _i, _i, _i, _v], _i),
    "wdg_fno_bias_act": ([_v, _v, _v, _v, _i, _i, _ll, _i, _v], _i),
    "wdg_fno_act_bwd": ([_v, _v, _v, _v, _ll, _i, _v], _i),
    "wdg_fno_bias_grad": ([_v, _v, _i, _i, _ll, _i, _v], _i),
    "wdg_fno_to_bf16": ([_v, _v, _ll, _v], _i),
    "wdg_fno_mse": ([_v, _v, _v, _v, _ll, C.c_float, _v], _i),
    "wdg_fno_adam": ([_v, _v, _v, _v, _ll, C.c_float, C.c_float, C.c_float, C.c_float, _i, C.c_float, _v], _i),
    "wdg_fno_inputs": ([_v, _i, _d, _d, _d, _d, _v], _i),
    "wdg_fno_nodes_to_grid": ([_v, _v, _i, _i, _v, _v, _i, C.c_float, _v], _i),
    "wdg_fno_grid_to_nodes": ([_v, _v, _i, _i, _v, _i, _d, _v], _i),
}

_lib = None


def header_symbols() -> list[str]:
    """Every function declared in include/*.h (used by the ABI tests)."""
    names = []
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(wdg_\w+)\s*\(", txt, flags=re.M)
    return names


def lib():
    """Load libwdg_b200.so once and attach the signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is not built; run `python -m wavedg_b200.build` "
                      "(or __graft_entry__.build()).  There is no CPU fallback.")
    L = C.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        if LIB_PATH != PACKAGE_LIB and not hasattr(L, name):
            continue  # another build without this entry point: calling it raises AttributeError
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(status: int, what: str = "") -> int:
    if status < 0:
        msg = lib().wdg_last_error().decode(errors="replace")
        raise WdgError(status, f"{what}: {msg}" if what else msg)
    return status
