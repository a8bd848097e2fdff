"""ctypes binding of the drnum_b200 C ABI (include/drnum_b200.h).

The shared library is built in-tree by ``python -m drnum_b200.build``.  There
is no fallback: if the library is missing or cannot be loaded, every call
raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_uint8, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdrnum_b200.so")

DN_OK = 0
DN_ERR_ARG = -1
DN_ERR_CUDA = -2
DN_ERR_STATE = -3
DN_ERR_NOMEM = -4
DN_ERR_RANGE = -5
DN_ERR_DEVICE = -6

DN_FP64 = 0
DN_FP32 = 1

DN_FACE_PERIODIC = 0
DN_FACE_CLOSED = 1

DN_OPT_BATCHED = 0
DN_OPT_GRAPH = 1
DN_OPT_BATCH_WAVES = 2
DN_OPT_BATCH_MIN_PLANES = 3
DN_OPT_DONOR_TABLES = 4
DN_NUM_TILE_SHAPES = 3

DN_BC_ZERO_FLUX = 0
DN_BC_FARFIELD = 1
DN_BC_SLIP = 2
DN_BC_INFLOW = 3

DN_FLUX_AUSMPLUS = 0
DN_FLUX_AUSMPLUS_FUNCTOR = 1
DN_FLUX_VANLEER = 2
DN_FLUX_ROE = 3


class dn_stage_launch(ctypes.Structure):
    _fields_ = [
        ("patch", c_int),
        ("in_", c_void_p), ("un", c_void_p), ("out", c_void_p), ("active", c_void_p),
        ("ni", c_int), ("nj", c_int), ("nk", c_int),
        ("periodic", c_int * 3),
        ("dx", c_double), ("dy", c_double), ("dz", c_double),
        ("factor", c_double),
        ("stream", c_void_p),
        ("num_sms", c_int),
    ]


DN_STAGE_FN = ctypes.CFUNCTYPE(c_int, c_void_p, POINTER(dn_stage_launch))
DN_EXCHANGE_FN = ctypes.CFUNCTYPE(c_int, c_void_p)
DN_FIELD_DONOR_COPY = -1


class dn_patch_desc(ctypes.Structure):
    _fields_ = [
        ("ni", c_int32), ("nj", c_int32), ("nk", c_int32),
        ("face", c_int32 * 3),
        ("dx", c_double), ("dy", c_double), ("dz", c_double),
        ("origin", c_double * 3),
        ("length", c_double * 3),
        ("seek", c_int32 * 6),
        ("add_protect", c_int32),
    ]


# name -> (restype, argtypes); every declaration of include/drnum_b200.h
SIGNATURES = {
    "dn_ctx_create": (c_int, [c_int, c_int, POINTER(c_void_p)]),
    "dn_ctx_destroy": (c_int, [c_void_p]),
    "dn_last_error": (c_int, [c_void_p, ctypes.c_char_p, c_size_t]),
    "dn_set_stream": (c_int, [c_void_p, c_void_p]),
    "dn_patch_add": (c_int, [c_void_p, POINTER(dn_patch_desc), POINTER(c_int)]),
    "dn_patch_set_base": (c_int, [c_void_p, c_int, POINTER(c_double), POINTER(c_double)]),
    "dn_patch_upload": (c_int, [c_void_p, c_int, c_int, POINTER(c_double)]),
    "dn_patch_upload_f32": (c_int, [c_void_p, c_int, c_int, POINTER(c_float)]),
    "dn_patch_download": (c_int, [c_void_p, c_int, c_int, POINTER(c_double)]),
    "dn_patch_download_f32": (c_int, [c_void_p, c_int, c_int, POINTER(c_float)]),
    "dn_patch_set_active": (c_int, [c_void_p, c_int, POINTER(c_uint8)]),
    "dn_copy_field": (c_int, [c_void_p, c_int, c_int]),
    "dn_compute": (c_int, [c_void_p, c_double]),
    "dn_compute_patches": (c_int, [c_void_p, c_double, c_void_p, c_int]),
    "dn_patch_activate": (c_int, [c_void_p, c_int, c_int]),
    "dn_patch_set_levelset_gpu": (c_int, [c_void_p, c_int, c_void_p]),
    "dn_patch_levelset_gpu_counts": (c_int, [c_void_p, c_int, c_void_p]),
    "dn_patch_set_levelset_layers": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                             c_void_p]),
    "dn_rk_step": (c_int, [c_void_p, c_double, POINTER(c_double), c_int]),
    "dn_sync": (c_int, [c_void_p]),
    "dn_conservation_sums": (c_int, [c_void_p, POINTER(c_double)]),
    "dn_field_difference": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int,
                                    POINTER(c_double), POINTER(c_double)]),
    "dn_flow_stats": (c_int, [c_void_p, c_int, c_int, c_double, POINTER(c_double)]),
    "dn_launch_count": (c_int, [c_void_p, POINTER(c_int64)]),
    "dn_tma_patch_count": (c_int, [c_void_p, POINTER(c_int64)]),
    "dn_field_sums_noalloc": (c_int, [c_void_p, c_int64, c_double, POINTER(c_double), c_void_p]),
    "dn_grid_compute_dependencies": (c_int, [c_void_p, POINTER(c_int64)]),
    "dn_patch_donor_counts": (c_int, [c_void_p, c_int, POINTER(c_int64)]),
    "dn_patch_get_donors": (c_int, [c_void_p, c_int, POINTER(c_uint64), POINTER(c_int32), POINTER(c_int64),
                                    POINTER(c_int32), POINTER(c_uint64), POINTER(c_uint64), POINTER(c_double)]),
    "dn_patch_set_donors": (c_int, [c_void_p, c_int, POINTER(c_int64), POINTER(c_uint64), POINTER(c_int32),
                                    POINTER(c_int64), POINTER(c_int32), POINTER(c_uint64), POINTER(c_uint64),
                                    POINTER(c_double)]),
    "dn_overlap_build": (c_int, [POINTER(dn_patch_desc), c_int, POINTER(c_void_p), POINTER(c_int64)]),
    "dn_overlap_counts": (c_int, [c_void_p, c_int, POINTER(c_int64)]),
    "dn_overlap_get": (c_int, [c_void_p, c_int, POINTER(c_uint64), POINTER(c_int32), POINTER(c_int64),
                               POINTER(c_int32), POINTER(c_uint64), POINTER(c_uint64), POINTER(c_double)]),
    "dn_overlap_destroy": (c_int, [c_void_p]),
    "dn_copy_donor_data": (c_int, [c_void_p, c_int]),
    "dn_patch_set_bc": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_double), POINTER(c_double)]),
    "dn_patch_set_levelset": (c_int, [c_void_p, c_int, POINTER(c_double), c_int, c_int, c_double]),
    "dn_patch_levelset_count": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_int64)]),
    "dn_patch_levelset_get": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_uint64), POINTER(c_double),
                                      POINTER(c_double), POINTER(c_uint64), POINTER(c_double)]),
    "dn_apply_levelset_bc": (c_int, [c_void_p, c_int]),
    "dn_levelset_classify": (c_int, [POINTER(dn_patch_desc), POINTER(c_double), c_int, c_int, c_double,
                                     POINTER(c_void_p)]),
    "dn_lslayers_count": (c_int, [c_void_p, c_int, c_int, POINTER(c_int64)]),
    "dn_lslayers_get": (c_int, [c_void_p, c_int, c_int, POINTER(c_uint64), POINTER(c_double), POINTER(c_double),
                                POINTER(c_uint64), POINTER(c_double)]),
    "dn_lslayers_destroy": (c_int, [c_void_p]),
    "dn_set_option": (c_int, [c_void_p, c_int, c_int]),
    "dn_set_flux_scheme": (c_int, [c_void_p, c_int]),
    "dn_grid_read": (c_int, [ctypes.c_char_p, c_double, POINTER(c_void_p)]),
    "dn_gridfile_count": (c_int, [c_void_p, POINTER(c_int)]),
    "dn_gridfile_patch": (c_int, [c_void_p, c_int, POINTER(dn_patch_desc), ctypes.c_char_p, c_size_t]),
    "dn_gridfile_destroy": (c_int, [c_void_p]),
    "dn_grid_write": (c_int, [ctypes.c_char_p, c_int, POINTER(dn_patch_desc), POINTER(ctypes.c_char_p)]),
    "dn_write_data": (c_int, [c_void_p, c_int, ctypes.c_char_p, c_double, c_int]),
    "dn_patch_set_owned": (c_int, [c_void_p, c_int, c_int]),
    "dn_patch_add_shadow": (c_int, [c_void_p, POINTER(dn_patch_desc), POINTER(c_int)]),
    "dn_shadow_alloc": (c_int, [c_void_p, c_void_p]),
    "dn_set_exchange_hook": (c_int, [c_void_p, DN_EXCHANGE_FN, c_void_p]),
    "dn_patch_device_cells": (c_int, [c_void_p, c_int, POINTER(c_int64)]),
    "dn_patch_upload_async": (c_int, [c_void_p, c_int, c_int, POINTER(c_double)]),
    "dn_patch_upload_f32_async": (c_int, [c_void_p, c_int, c_int, POINTER(c_float)]),
    "dn_patch_download_async": (c_int, [c_void_p, c_int, c_int, POINTER(c_double)]),
    "dn_patch_download_f32_async": (c_int, [c_void_p, c_int, c_int, POINTER(c_float)]),
    "dn_exchange_build": (c_int, [c_void_p, POINTER(c_int32), c_int, c_int, POINTER(c_void_p)]),
    "dn_exchange_build_ctx": (c_int, [c_void_p, POINTER(c_int32), c_int, c_int, POINTER(c_void_p)]),
    "dn_exchange_counts": (c_int, [c_void_p, c_int, POINTER(c_int64), POINTER(c_int64)]),
    "dn_exchange_get": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "dn_exchange_pack": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p]),
    "dn_exchange_unpack": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p]),
    "dn_exchange_destroy": (c_int, [c_void_p]),
    "dn_read_data": (c_int, [c_void_p, c_int, ctypes.c_char_p, POINTER(c_double)]),
    "dn_set_stage_function": (c_int, [c_void_p, c_void_p, c_void_p]),
    "dn_patch_set_tile": (c_int, [c_void_p, c_int, c_int]),
    "dn_autotune": (c_int, [c_void_p, ctypes.c_char_p, POINTER(c_double)]),
}

_lib = None


def load(path: str | None = None) -> ctypes.CDLL:
    """Loads the library (once) and declares every C ABI signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"drnum_b200 native library not built: {p} "
                           "(run `python -m drnum_b200.build`)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class DnError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"drnum_b200 error {code}: {message}")
        self.code = code


def check(ctx, code: int) -> None:
    if code == DN_OK:
        return
    msg = ""
    if ctx:
        buf = ctypes.create_string_buffer(512)
        load().dn_last_error(ctx, buf, 512)
        msg = buf.value.decode(errors="replace")
    raise DnError(code, msg)


def dptr(a):
    return a.ctypes.data_as(POINTER(c_double))


def fptr(a):
    return a.ctypes.data_as(POINTER(c_float))


def u8ptr(a):
    return a.ctypes.data_as(POINTER(c_uint8))


def ptr(a, ctype):
    """ctypes pointer to the data of a contiguous numpy array (NULL for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(POINTER(ctype))


# donor-table arrays in the order of dn_patch_get_donors / dn_overlap_get:
# (name, numpy dtype, ctypes type, counts index)
DONOR_FIELDS = (
    ("rec_unique", "uint64", c_uint64, 0),
    ("donor_patch", "int32", c_int32, 1),
    ("num_receivers", "int64", c_int64, 1),
    ("stride", "int32", c_int32, 1),
    ("rec_concat", "uint64", c_uint64, 2),
    ("donor_idx", "uint64", c_uint64, 3),
    ("weight", "float64", c_double, 3),
)


def read_donor_tables(counts_fn, get_fn, handle, patch_id):
    """Reads one patch's donor tables through a counts/get function pair
    (dn_patch_donor_counts/dn_patch_get_donors or dn_overlap_counts/
    dn_overlap_get) into a dict of numpy arrays."""
    import numpy as np
    counts = np.zeros(4, dtype=np.int64)
    rc = counts_fn(handle, patch_id, ptr(counts, c_int64))
    if rc != DN_OK:
        raise DnError(rc, f"donor counts of patch {patch_id}")
    arrs = {name: np.zeros(int(counts[ci]), dtype=dt) for name, dt, _, ci in DONOR_FIELDS}
    rc = get_fn(handle, patch_id, *[ptr(arrs[name], ct) for name, _, ct, _ in DONOR_FIELDS])
    if rc != DN_OK:
        raise DnError(rc, f"donor tables of patch {patch_id}")
    arrs["counts"] = counts
    return arrs


def read_levelset_layers(count_fn, get_fn, handle, args, num_inner, num_outer):
    """Reads a level-set classification through a count/get pair
    (dn_patch_levelset_count/get with args = (patch_id,), or
    dn_lslayers_count/get with args = ()).  Returns
    {"inner": [layer dicts], "outer": [...]} with cells, g, grad, donors, weights."""
    import numpy as np
    out = {}
    for inner, num in ((1, num_inner), (0, num_outer)):
        layers = []
        for layer in range(num):
            n = c_int64()
            rc = count_fn(handle, *args, inner, layer, ctypes.byref(n))
            if rc != DN_OK:
                raise DnError(rc, "level-set layer count")
            m = n.value
            d = {"cells": np.zeros(m, np.uint64), "g": np.zeros(m), "grad": np.zeros((m, 3)),
                 "donors": np.zeros((m, 8), np.uint64), "weights": np.zeros((m, 8))}
            rc = get_fn(handle, *args, inner, layer, ptr(d["cells"], c_uint64), ptr(d["g"], c_double),
                        ptr(d["grad"], c_double), ptr(d["donors"], c_uint64), ptr(d["weights"], c_double))
            if rc != DN_OK:
                raise DnError(rc, "level-set layer")
            layers.append(d)
        out["inner" if inner else "outer"] = layers
    return out
