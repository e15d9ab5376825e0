"""Loader of libwvlh.so and the ctypes signatures of its C ABI (include/wvlh.h)."""
import ctypes as C
import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libwvlh.so"
CSRC = PKG.parent / "csrc"

_lib = None


class WvlhError(RuntimeError):
    pass


ERRORS = {1: "CUDA runtime error", 2: "invalid argument", 3: "invalid segment keys",
          4: "device allocation failed", 5: "unsupported (k-points / spinors)", 6: "box too large for this path",
          7: "batch tables replaced by a newer orbital batch"}


def build(force=False):
    """Compile libwvlh.so for sm_100a (nvcc cross-compiles without a GPU)."""
    if force or not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-j4", "-C", str(CSRC)], check=True)


def check(rc, what=""):
    if rc != 0:
        raise WvlhError("%s failed: %s (code %d)" % (what, ERRORS.get(rc, "error"), rc))


vp = C.c_void_p
ip = C.POINTER(C.c_int)
u32p = C.POINTER(C.c_uint32)
dp = C.POINTER(C.c_double)


class LocregDesc(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("periodic", C.c_int * 3), ("hgrid", C.c_double * 3),
                ("nseg_c", C.c_int), ("nseg_f", C.c_int),
                ("keyg_c", C.POINTER(C.c_int32)), ("keyv_c", C.POINTER(C.c_int32)),
                ("keyg_f", C.POINTER(C.c_int32)), ("keyv_f", C.POINTER(C.c_int32))]


class OrbitalDesc(C.Structure):
    _fields_ = [("region", C.c_void_p), ("psi", C.c_void_p), ("hpsi", C.c_void_p), ("pot", C.c_void_p),
                ("rho", C.c_void_p)]


# every extern "C" symbol declared in include/wvlh.h
OCL_SYMBOLS = [
    "ocl_create_context_", "ocl_create_gpu_context_", "ocl_build_programs_", "ocl_create_command_queue_",
    "ocl_create_command_queue_id_", "ocl_create_read_buffer_", "ocl_create_write_buffer_",
    "ocl_create_read_write_buffer_", "ocl_create_read_buffer_and_copy_", "ocl_release_mem_object_",
    "ocl_enqueue_read_buffer_", "ocl_enqueue_write_buffer_", "ocl_enqueue_read_buffer_async_",
    "ocl_enqueue_write_buffer_async_", "ocl_finish_", "ocl_enqueue_barrier_", "ocl_clean_command_queue_",
    "ocl_clean_", "init_event_list_", "print_event_list_", "nanosec_",
    "ocl_create_read_buffer_host_", "ocl_create_write_buffer_host_", "ocl_create_read_write_buffer_host_",
    "ocl_map_read_buffer_", "ocl_map_write_buffer_", "ocl_map_read_write_buffer_", "ocl_map_read_buffer_async_",
    "ocl_map_write_buffer_async_", "ocl_map_read_write_buffer_async_", "ocl_unmap_mem_object_",
    "ocl_pin_read_write_buffer_", "ocl_pin_write_buffer_", "ocl_pin_read_buffer_",
    "ocl_pin_read_write_buffer_async_", "ocl_pin_write_buffer_async_", "ocl_pin_read_buffer_async_",
    "uncompress_d_", "compress_d_", "uncompress_scale_d_", "compress_scale_d_", "scale_psi_d_",
    "syn1d_d_", "syngrow1d_d_", "ana1d_d_", "anashrink1d_d_", "magicfilter1d_d_", "magicfiltergrow1d_d_",
    "magicfilter1d_t_d_", "magicfiltershrink1d_d_", "magicfilter1d_pot_d_", "kinetic1d_d_",
    "syn_self_d_", "ana_self_d_", "syn_self_d_generic_", "ana_self_d_generic_", "syn_d_generic_",
    "ana_d_generic_", "magic_filter_3d_generic_", "magic_filter_t_3d_generic_",
    "potential_application_d_generic_", "kinetic_d_generic_", "kinetic_d_", "magicfilter_den_d_generic_",
    "dot_d_", "dot_d_async_", "nrm2sq_d_", "axpy_d_", "axpy_self_d_", "scal_d_", "scal_self_d_", "copy_d_",
    "set_d_", "ocl_fulllocham_generic_", "ocl_fulllocham_generic_k_", "ocl_daub_to_isf_", "ocl_isf_to_daub_",
    "ocl_locden_generic_", "ocl_preconditioner_generic_", "ocl_preconditioner_generic_k_",
]
WVLH_SYMBOLS = [
    "wvlh_get_last_error", "wvlh_error_string", "wvlh_mem_ptr", "wvlh_ctx_create", "wvlh_ctx_destroy",
    "wvlh_ctx_set_stream", "wvlh_ctx_synchronize", "wvlh_batch_create", "wvlh_batch_destroy",
    "wvlh_batch_psi_size", "wvlh_batch_psi_offset", "wvlh_batch_scratch_bytes", "wvlh_locham_batched",
    "wvlh_locham_batched_host", "wvlh_locham_plain_batched", "wvlh_host_alloc", "wvlh_host_free",
    "wvlh_ctx_enable_timing", "wvlh_ctx_kernel_times", "wvlh_measure_fma_peak",
    "wvlh_locham_noalloc", "wvlh_noalloc_capacity", "wvlh_locden_batched", "wvlh_precond_batched",
    "wvlh_overlap", "wvlh_region_create", "wvlh_region_destroy", "wvlh_region_psi_size",
    "wvlh_region_grid_size", "wvlh_region_scratch_bytes", "wvlh_batch_create_orbitals", "wvlh_wpdot",
    "wvlh_locham_graph_create", "wvlh_graph_launch", "wvlh_graph_destroy",
    "wvlh_nlpsp_create", "wvlh_nlpsp_apply", "wvlh_nlpsp_destroy", "wvlh_subspace_matrix", "wvlh_panel_apply",
    "wvlh_batch_autotune",
    "wvlh_batch_autotune_precond",
    "wvlh_batch_block_sizes",
    "wvlh_psolver_periodic",
    "wvlh_xc_lda",
    "wvlh_ks_potential_periodic",
    "wvlh_psolver_free",
    "wvlh_ks_potential_free",
    "wvlh_psolver_free_tables",
    "wvlh_xc_lsda",
    "wvlh_psolver_surface",
    "wvlh_psolver_surface_table",
    "wvlh_psolver_wire",
    "wvlh_psolver_wire_table",
    "wvlh_ks_potential_bc",
    "wvlh_ks_potential_spin",
]


def lib():
    """The loaded library; raises loudly when it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise WvlhError("libwvlh.so not built (%s); run __graft_entry__.build()" % LIB_PATH)
    L = C.CDLL(str(LIB_PATH))
    L.wvlh_get_last_error.restype = C.c_int
    L.wvlh_error_string.restype = C.c_char_p
    L.wvlh_error_string.argtypes = [C.c_int]
    L.wvlh_mem_ptr.restype = vp
    L.wvlh_mem_ptr.argtypes = [vp]
    L.wvlh_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.wvlh_ctx_destroy.argtypes = [vp]
    L.wvlh_ctx_set_stream.argtypes = [vp, vp]
    L.wvlh_ctx_synchronize.argtypes = [vp]
    L.wvlh_batch_create.argtypes = [vp, C.c_int, C.POINTER(LocregDesc), C.c_int, C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int64), C.POINTER(vp)]
    L.wvlh_batch_destroy.argtypes = [vp]
    L.wvlh_batch_psi_size.restype = C.c_int64
    L.wvlh_batch_psi_size.argtypes = [vp]
    L.wvlh_batch_psi_offset.restype = C.c_int64
    L.wvlh_batch_psi_offset.argtypes = [vp, C.c_int]
    L.wvlh_batch_scratch_bytes.restype = C.c_int64
    L.wvlh_batch_scratch_bytes.argtypes = [vp, C.c_int]
    L.wvlh_locham_batched.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, C.c_int]
    L.wvlh_locham_batched_host.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp]
    L.wvlh_locham_plain_batched.argtypes = [vp, vp, vp, vp, vp, vp]
    L.wvlh_ctx_enable_timing.argtypes = [vp, C.c_int]
    L.wvlh_ctx_kernel_times.argtypes = [vp, dp, C.POINTER(C.c_longlong)]
    L.wvlh_measure_fma_peak.argtypes = [C.c_int, C.c_int, dp]
    i32p = C.POINTER(C.c_int32)
    L.wvlh_locham_noalloc.argtypes = [C.c_int, ip, ip, dp, C.c_int, i32p, i32p, C.c_int, i32p, i32p,
                                      vp, vp, vp, vp, vp, vp]
    L.wvlh_noalloc_capacity.restype = C.c_size_t
    L.wvlh_locden_batched.argtypes = [vp, C.c_int, vp, vp, vp]
    L.wvlh_precond_batched.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp]
    L.wvlh_overlap.argtypes = [vp, C.c_int, C.c_int, C.c_int64, C.c_int64, vp, vp]
    L.wvlh_region_create.argtypes = [vp, C.POINTER(LocregDesc), C.POINTER(vp)]
    L.wvlh_region_destroy.argtypes = [vp]
    for nm in ("wvlh_region_psi_size", "wvlh_region_grid_size"):
        getattr(L, nm).restype = C.c_int64
        getattr(L, nm).argtypes = [vp]
    L.wvlh_region_scratch_bytes.restype = C.c_int64
    L.wvlh_region_scratch_bytes.argtypes = [vp, C.c_int]
    L.wvlh_batch_create_orbitals.argtypes = [vp, C.c_int, C.POINTER(OrbitalDesc), C.POINTER(vp)]
    L.wvlh_wpdot.argtypes = [vp, C.c_int, vp, C.c_int, vp, C.c_int64, vp, C.c_int, vp, C.c_int64, vp]
    L.wvlh_locham_graph_create.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, C.c_int, C.POINTER(vp)]
    L.wvlh_graph_launch.argtypes = [vp]
    L.wvlh_graph_destroy.argtypes = [vp]
    L.wvlh_nlpsp_create.argtypes = [vp, vp, C.c_int, C.POINTER(vp), C.POINTER(C.c_int), vp,
                                    C.POINTER(C.c_double), C.POINTER(vp)]
    L.wvlh_nlpsp_apply.argtypes = [vp, C.c_int, vp, C.c_int64, vp, vp]
    L.wvlh_nlpsp_destroy.argtypes = [vp]
    L.wvlh_subspace_matrix.argtypes = [vp, C.c_int, C.c_int, C.c_int64, C.c_int64, vp, vp, vp]
    L.wvlh_batch_autotune.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.wvlh_batch_block_sizes.argtypes = [vp, C.POINTER(C.c_int)]
    L.wvlh_batch_autotune_precond.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, C.c_int, C.POINTER(C.c_int), vp,
                                              vp, C.POINTER(C.c_int)]
    L.wvlh_panel_apply.argtypes = [vp, C.c_int, C.c_int64, C.c_int64, vp, C.c_int, C.c_double, vp, C.c_double, vp]
    L.wvlh_psolver_periodic.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double), vp, vp, C.c_double, vp]
    L.wvlh_xc_lda.argtypes = [vp, C.c_int64, vp, vp, C.c_int, C.c_double, vp]
    L.wvlh_ks_potential_periodic.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double), vp, vp, vp, vp]
    L.wvlh_psolver_free.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double), vp, vp, vp]
    L.wvlh_ks_potential_free.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double), vp, vp, vp, vp]
    L.wvlh_psolver_free_tables.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int), vp,
                                           C.c_int64]
    L.wvlh_psolver_free_tables.restype = C.c_int64
    L.wvlh_psolver_surface.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double), vp, vp, vp]
    L.wvlh_psolver_surface_table.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int), vp,
                                             C.c_int64]
    L.wvlh_psolver_surface_table.restype = C.c_int64
    L.wvlh_psolver_wire.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double), vp, vp, vp]
    L.wvlh_psolver_wire_table.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int), vp,
                                          C.c_int64]
    L.wvlh_psolver_wire_table.restype = C.c_int64
    L.wvlh_ks_potential_bc.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), vp, vp, vp, vp, vp]
    L.wvlh_xc_lsda.argtypes = [vp, C.c_int64, vp, vp, vp, vp, C.c_int, C.c_double, vp]
    L.wvlh_ks_potential_spin.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), vp, vp, vp, vp,
                                         vp, vp, vp]
    L.wvlh_host_alloc.restype = vp
    L.wvlh_host_alloc.argtypes = [C.c_size_t]
    L.wvlh_host_free.argtypes = [vp]
    _lib = L
    return L


def exported_symbols():
    """Dynamic symbols the library exports (via nm -D)."""
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], check=True, capture_output=True, text=True)
    return {ln.split()[-1] for ln in out.stdout.splitlines() if ln.strip()}


def header_symbols():
    """Function names declared in include/wvlh.h."""
    import re
    hdr = (PKG.parent.parent / "include" / "wvlh.h").read_text()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", hdr)) - {"if", "sizeof", "defined"}


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise WvlhError("no CUDA device available: wvlh has no CPU path")
    return torch


def env_int(name, default):
    return int(os.environ.get(name, default))
