"""ctypes declarations of libclbool_b200.so (the C ABI in include/clbool_b200.h).

The library is the product: there is no CPU fallback.  If the shared object
is missing, importing this module raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclbool_b200.so")

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
vp = C.c_void_p


class clb_dcsr(C.Structure):
    _fields_ = [("nrows", C.c_uint64), ("ncols", C.c_uint64), ("nnz", C.c_uint64), ("nzr", C.c_uint64),
                ("rpt", vp), ("rows", vp), ("cols", vp)]


class clb_coo(C.Structure):
    _fields_ = [("nrows", C.c_uint64), ("ncols", C.c_uint64), ("nnz", C.c_uint64), ("rows", vp), ("cols", vp)]


class clb_csr(C.Structure):
    _fields_ = [("nrows", C.c_uint64), ("ncols", C.c_uint64), ("nnz", C.c_uint64), ("rpt", vp), ("cols", vp)]


class clb_profile_entry(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_uint32), ("reserved", C.c_uint32), ("ms", C.c_double)]


class clb_spgemm_stats(C.Structure):
    _fields_ = [("products", C.c_uint64), ("nnz", C.c_uint64), ("nzr", C.c_uint64),
                ("rows_per_bin", C.c_uint64 * 16), ("fallback_rows", C.c_uint64), ("capacity", C.c_uint64),
                ("kernel_launches", C.c_uint32), ("reserved", C.c_uint32), ("spilled_rows", C.c_uint64)]

    def as_dict(self) -> dict:
        return {"products": self.products, "nnz": self.nnz, "nzr": self.nzr,
                "rows_per_bin": list(self.rows_per_bin)[:14], "fallback_rows": self.fallback_rows,
                "capacity": self.capacity, "kernel_launches": self.kernel_launches,
                "spilled_rows": self.spilled_rows}


class clb_spgemm_tuning(C.Structure):
    _fields_ = [("form", C.c_uint32), ("warp_max", C.c_uint32), ("bitmap_min", C.c_uint32),
                ("bitmap_threads", C.c_uint32), ("small_lanes", C.c_uint32), ("wide_rows", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]

    def as_dict(self) -> dict:
        return {"form": {0: "two_pass", 1: "single_pass", 2: "two_pass_kept"}.get(self.form, self.form),
                "warp_max": self.warp_max,
                "bitmap_min": self.bitmap_min, "bitmap_threads": self.bitmap_threads,
                "small_lanes": self.small_lanes, "wide_rows": {1: "cluster", 2: "chunks"}.get(self.wide_rows, "chunks")}


P = C.POINTER

# name -> (restype, argtypes)
_SIGS = {
    "clb_status_string": (C.c_char_p, [C.c_int]),
    "clb_last_error": (C.c_char_p, []),
    "clb_version": (C.c_int, []),
    "clb_controls_create": (C.c_int, [C.c_int, P(vp)]),
    "clb_controls_destroy": (C.c_int, [vp]),
    "clb_controls_set_stream": (C.c_int, [vp, vp]),
    "clb_controls_get_stream": (vp, [vp]),
    "clb_controls_set_allocator": (C.c_int, [vp, vp, vp, vp]),
    "clb_controls_sync": (C.c_int, [vp]),
    "clb_controls_trim": (C.c_int, [vp]),
    "clb_controls_device": (C.c_int, [vp]),
    "clb_device_count": (C.c_int, [P(C.c_int)]),
    "clb_device_info": (C.c_int, [C.c_int, C.c_char_p, C.c_size_t, P(C.c_int), P(C.c_uint64)]),
    "clb_profile_enable": (C.c_int, [vp, C.c_int]),
    "clb_profile_read": (C.c_int, [vp, P(clb_profile_entry), C.c_int, P(C.c_int)]),
    "clb_coo_sort": (C.c_int, [vp, vp, vp, C.c_uint64]),
    "clb_coo_reduce_duplicates": (C.c_int, [vp, P(clb_coo), P(clb_coo)]),
    "clb_malloc": (C.c_int, [vp, C.c_size_t, P(vp)]),
    "clb_free": (C.c_int, [vp, vp]),
    "clb_memcpy_h2d": (C.c_int, [vp, vp, vp, C.c_size_t]),
    "clb_memcpy_d2h": (C.c_int, [vp, vp, vp, C.c_size_t]),
    "clb_memcpy_d2d": (C.c_int, [vp, vp, vp, C.c_size_t]),
    "clb_host_alloc": (C.c_int, [C.c_size_t, P(vp)]),
    "clb_host_free": (C.c_int, [vp]),
    "clb_dcsr_release": (C.c_int, [vp, P(clb_dcsr)]),
    "clb_coo_release": (C.c_int, [vp, P(clb_coo)]),
    "clb_csr_release": (C.c_int, [vp, P(clb_csr)]),
    "clb_prefix_sum_u32": (C.c_int, [vp, vp, C.c_uint64, P(C.c_uint64)]),
    "clb_prefix_sum_u64": (C.c_int, [vp, vp, C.c_uint64, P(C.c_uint64)]),
    "clb_fill_u32": (C.c_int, [vp, vp, C.c_uint64, C.c_uint32]),
    "clb_prefix_sum_u32_noalloc": (C.c_int, [vp, C.c_uint64, vp, vp]),
    "clb_coo_to_dcsr": (C.c_int, [vp, P(clb_coo), P(clb_dcsr), C.c_int]),
    "clb_dcsr_to_coo": (C.c_int, [vp, P(clb_dcsr), P(clb_coo), C.c_int]),
    "clb_dcsr_to_csr": (C.c_int, [vp, P(clb_dcsr), P(clb_csr)]),
    "clb_csr_to_dcsr": (C.c_int, [vp, P(clb_csr), P(clb_dcsr)]),
    "clb_dcsr_spgemm_hash": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), P(clb_dcsr), P(clb_spgemm_stats)]),
    "clb_dcsr_workload": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), vp, P(C.c_uint64)]),
    "clb_dcsr_spgemm_esc": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), P(clb_dcsr), P(clb_spgemm_stats)]),
    "clb_coo_add": (C.c_int, [vp, P(clb_coo), P(clb_coo), P(clb_coo)]),
    "clb_csr_add": (C.c_int, [vp, P(clb_csr), P(clb_csr), P(clb_csr)]),
    "clb_csr_add_batched": (C.c_int, [vp, C.c_uint32, P(clb_csr), P(clb_csr), P(clb_csr)]),
    "clb_dcsr_kronecker": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), P(clb_dcsr)]),
    "clb_dcsr_transpose": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr)]),
    "clb_dcsr_submatrix": (C.c_int, [vp, P(clb_dcsr), C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, P(clb_dcsr)]),
    "clb_dcsr_reduce": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr)]),
    # learned sizing
    "clb_sizer_num_params": (C.c_int, []),
    "clb_sizer_create": (C.c_int, [vp, C.c_uint64, P(vp)]),
    "clb_sizer_destroy": (C.c_int, [vp]),
    "clb_sizer_get_params": (C.c_int, [vp, vp, C.c_size_t]),
    "clb_sizer_set_params": (C.c_int, [vp, vp, C.c_size_t]),
    "clb_dcsr_row_features": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), vp, vp]),
    "clb_dcsr_row_nnz": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), vp]),
    "clb_sizer_predict": (C.c_int, [vp, vp, C.c_uint64, vp]),
    "clb_sizer_gradients": (C.c_int, [vp, vp, vp, C.c_uint64, vp, P(C.c_float)]),
    "clb_sizer_train": (C.c_int, [vp, vp, vp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_float, C.c_uint64,
                                  P(C.c_float)]),
    "clb_dcsr_spgemm_learned": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), vp, C.c_float, C.c_float,
                                          P(clb_spgemm_tuning), P(clb_dcsr), P(clb_spgemm_stats)]),
    # tuning and batching
    "clb_spgemm_tuning_default": (None, [P(clb_spgemm_tuning)]),
    "clb_dcsr_spgemm_tuned": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), P(clb_spgemm_tuning), P(clb_dcsr),
                                        P(clb_spgemm_stats)]),
    "clb_dcsr_spgemm_batched": (C.c_int, [vp, C.c_uint32, P(clb_dcsr), P(clb_dcsr), P(clb_dcsr),
                                          P(clb_spgemm_tuning), P(clb_spgemm_stats)]),
    "clb_dcsr_spgemm_batched_learned": (C.c_int, [vp, C.c_uint32, P(clb_dcsr), P(clb_dcsr), P(clb_dcsr), vp,
                                                  C.c_float, C.c_float, P(clb_spgemm_tuning),
                                                  P(clb_spgemm_stats)]),
    "clb_dcsr_union": (C.c_int, [vp, C.c_uint32, P(clb_dcsr), P(clb_spgemm_tuning), P(clb_dcsr),
                                 P(clb_spgemm_stats)]),
    "clb_spgemm_autotune": (C.c_int, [vp, C.c_uint32, P(clb_dcsr), P(clb_dcsr), P(clb_spgemm_tuning),
                                      P(clb_spgemm_tuning), P(C.c_double), C.c_uint32, P(C.c_uint32)]),
    # host-sync-free batched product and CUDA graphs
    "clb_spgemm_batched_plan": (C.c_int, [vp, C.c_uint32, P(clb_dcsr), P(clb_dcsr), P(C.c_uint64), P(C.c_uint64)]),
    "clb_dcsr_spgemm_batched_capture": (C.c_int, [vp, C.c_uint32, P(clb_dcsr), P(clb_dcsr), P(clb_spgemm_tuning),
                                                  C.c_uint64, vp, vp, vp, C.c_uint64, vp, vp]),
    "clb_spgemm_batched_plan_learned": (C.c_int, [vp, C.c_uint32, P(clb_dcsr), P(clb_dcsr), vp, C.c_float,
                                                  C.c_float, P(clb_spgemm_tuning), P(C.c_uint64), P(C.c_uint64)]),
    "clb_dcsr_spgemm_batched_capture_learned": (C.c_int, [vp, C.c_uint32, P(clb_dcsr), P(clb_dcsr), vp, C.c_float,
                                                          C.c_float, P(clb_spgemm_tuning), C.c_uint64, C.c_uint64,
                                                          vp, vp, vp, C.c_uint64, vp, vp]),
    "clb_dcsr_spgemm_to_host": (C.c_int, [vp, P(clb_dcsr), P(clb_dcsr), vp, C.c_float, C.c_float,
                                          P(clb_spgemm_tuning), C.c_uint32, vp, vp, vp, C.c_uint64, C.c_uint64,
                                          P(C.c_uint64), P(C.c_uint64), P(clb_spgemm_stats)]),
    "clb_dcsr_row_block": (C.c_int, [vp, P(clb_dcsr), C.c_uint64, C.c_uint64, P(clb_dcsr)]),
    "clb_graph_begin": (C.c_int, [vp]),
    "clb_graph_end": (C.c_int, [vp, P(vp)]),
    "clb_graph_launch": (C.c_int, [vp, vp]),
    "clb_graph_destroy": (C.c_int, [vp]),
}

def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libclbool_b200.so not built ({LIB_PATH}); run `python clbool_b200/build.py`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def declared_symbols() -> list[str]:
    return sorted(_SIGS)
