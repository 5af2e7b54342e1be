"""ctypes binding of the C ABI declared in include/afhe.h.

The library is the product: there is no Python or CPU fallback for any
operator. Loading fails loudly if libafhe.so is missing and cannot be built.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import threading

from . import build as _build

MAX_Q = 64
MAX_P = 16
MAX_PARTS = 16

OK, E_ARG, E_RANGE, E_NOKEY, E_LEVEL, E_BUDGET, E_TIMEOUT, E_CUDA, E_STATE = range(9)

OP_NTT, OP_INTT, OP_POLY_ADD, OP_POLY_SUB, OP_POLY_MUL_NTT = 1, 2, 3, 4, 5
OP_AUTOMORPHISM, OP_KEY_SWITCH, OP_RESCALE, OP_LOAD_CONTEXT = 6, 7, 8, 99
OPT_KS_FUSED, OPT_CHUNK, OPT_FUSED_MIN, OPT_KS_CAPACITY, OPT_KS_EPT, OPT_KS_SLICE = 1, 2, 3, 4, 5, 6

u32, u64, i32 = C.c_uint32, C.c_uint64, C.c_int32
P64 = C.POINTER(C.c_uint64)
P32 = C.POINTER(C.c_uint32)


class Params(C.Structure):
    _fields_ = [
        ("log_n", u32), ("num_q", u32), ("num_p", u32), ("alpha", u32),
        ("q", u64 * MAX_Q), ("p", u64 * MAX_P),
        ("poly_words", u64), ("key_words", u64), ("device", i32), ("max_batch", u32),
        ("psi_q", u64 * MAX_Q), ("psi_p", u64 * MAX_P),
    ]


class AccelArgs(C.Structure):
    _fields_ = [
        ("op_code", u32), ("active_limbs", u32),
        ("src_a_offset", u64), ("src_b_offset", u64), ("dst_offset", u64),
        ("evk_offset", u64),
        ("prime_idx", u32), ("galois_elt", u32),
        ("sizeQl", u32), ("sizeP", u32), ("numPartQ", u32), ("alpha", u32),
        ("rns_primes", u64 * MAX_Q), ("p_primes", u64 * MAX_P),
        ("barrett_m_q_lo", u64 * MAX_Q), ("barrett_m_q_hi", u64 * MAX_Q), ("barrett_k_q", u32 * MAX_Q),
        ("barrett_m_p_lo", u64 * MAX_P), ("barrett_m_p_hi", u64 * MAX_P), ("barrett_k_p", u32 * MAX_P),
        ("n_inv_q", u64 * MAX_Q), ("n_inv_p", u64 * MAX_P), ("n_inv_mod_q_last", u64),
        ("twiddles_q_offset", u64), ("inv_twiddles_q_offset", u64),
        ("twiddles_p_offset", u64), ("inv_twiddles_p_offset", u64),
        ("qhat_inv_offset", u64 * MAX_PARTS), ("qhat_modp_offset", u64 * MAX_PARTS),
        ("p_inv_mod_q_offset", u64), ("p_hat_inv_mod_p_offset", u64), ("p_hat_mod_q_offset", u64),
        ("qlql_offset", u64), ("qlinv_offset", u64),
    ]


class ContextLayout(C.Structure):
    _fields_ = [
        ("twiddles_q_offset", u64), ("inv_twiddles_q_offset", u64),
        ("twiddles_p_offset", u64), ("inv_twiddles_p_offset", u64),
        ("qhat_inv_offset", u64 * MAX_PARTS), ("qhat_modp_offset", u64 * MAX_PARTS),
        ("p_inv_mod_q_offset", u64), ("p_hat_inv_mod_p_offset", u64), ("p_hat_mod_q_offset", u64),
        ("qlql_offset", u64), ("qlinv_offset", u64),
        ("first_free_offset", u64), ("level", u32), ("num_parts", u32),
    ]


class CtRef(C.Structure):
    _fields_ = [("c0_offset", u64), ("c1_offset", u64)]


class MacTerm(C.Structure):
    _fields_ = [("pt", C.c_uint64), ("galois", C.c_uint32), ("reserved", C.c_uint32)]


class MacGroup(C.Structure):
    _fields_ = [("src", CtRef), ("first_term", C.c_uint32), ("n_terms", C.c_uint32)]


MAC_UNIT = (1 << 64) - 1


class PqIndex(C.Structure):
    _fields_ = [("n_list", u32), ("d", u32), ("M", u32), ("K", u32), ("n", u64),
                ("centroids", C.POINTER(C.c_float)), ("codebooks", C.POINTER(C.c_float)),
                ("codes", C.POINTER(C.c_uint8)), ("assignments", C.POINTER(u32))]


class KsOptions(C.Structure):
    _fields_ = [("fused", i32), ("chunk", u32), ("ept", u32), ("slice", u32), ("fused_min", u32)]


class IvfpqShape(C.Structure):
    _fields_ = [("D", u32), ("n_list", u32), ("slots", u32), ("lanes", u32), ("packed", u32), ("eval_level", u32)]


class IvfpqQuery(C.Structure):
    _fields_ = [("ct_query", CtRef), ("ct_dim", CtRef), ("compact", CtRef), ("norm", CtRef), ("results", C.POINTER(CtRef)),
                ("n_results", u32), ("level", u32), ("probes", C.POINTER(u32)), ("nprobe", u32),
                ("baby", C.POINTER(CtRef)), ("n_baby", u32)]


CTX = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "afhe_find_ntt_primes": (C.c_int, [u32, u32, u32, P64, u32, P64]),
    "afhe_min_primitive_root": (u64, [u32, u64]),
    "afhe_gen_twiddles": (C.c_int, [u32, u64, u64, P64, P64]),
    "afhe_barrett_constant": (None, [u64, P64, P64, P32]),
    "afhe_inv_mod": (u64, [u64, u64]),
    "afhe_galois_elt": (u32, [u32, i32]),
    "afhe_automorphism_map": (C.c_int, [u32, u32, P32]),
    "afhe_part_qhat_tables": (C.c_int, [P64, u32, u32, u32, P64, u32, P64, P64]),
    "afhe_moddown_tables": (C.c_int, [P64, u32, P64, u32, P64, P64, P64]),
    "afhe_rescale_tables": (C.c_int, [P64, u32, P64, P64]),
    "afhe_status_string": (C.c_char_p, [C.c_int]),
    "afhe_last_error": (C.c_char_p, []),
    "afhe_ctx_create": (C.c_int, [C.POINTER(Params), C.POINTER(CTX)]),
    "afhe_ctx_destroy": (C.c_int, [CTX]),
    "afhe_sync": (C.c_int, [CTX]),
    "afhe_stream": (C.c_void_p, [CTX]),
    "afhe_poly_gmem": (C.c_void_p, [CTX]),
    "afhe_key_gmem": (C.c_void_p, [CTX]),
    "afhe_scratch_words": (u64, [CTX]),
    "afhe_write_poly": (C.c_int, [CTX, u64, P64, u64]),
    "afhe_read_poly": (C.c_int, [CTX, u64, P64, u64]),
    "afhe_write_key": (C.c_int, [CTX, u64, P64, u64]),
    "afhe_read_key": (C.c_int, [CTX, u64, P64, u64]),
    "afhe_write_poly_async": (C.c_int, [CTX, u64, P64, u64]),
    "afhe_read_poly_async": (C.c_int, [CTX, u64, P64, u64]),
    "afhe_copy_poly": (C.c_int, [CTX, u64, u64, u64]),
    "afhe_read_poly_rows": (C.c_int, [CTX, u64, u64, u64, u64, P64]),
    "afhe_read_poly_rows_async": (C.c_int, [CTX, u64, u64, u64, u64, P64]),
    "afhe_fence": (C.c_int, [CTX, C.POINTER(C.c_uint64)]),
    "afhe_fence_wait": (C.c_int, [CTX, u64]),
    "afhe_host_alloc": (C.c_int, [u64, C.POINTER(C.c_void_p)]),
    "afhe_ctx_set_option": (C.c_int, [CTX, u32, C.c_int64]),
    "afhe_ctx_get_option": (C.c_int, [CTX, u32, C.POINTER(C.c_int64)]),
    "afhe_host_free": (C.c_int, [C.c_void_p]),
    "afhe_ctx_write_context_tables": (C.c_int, [CTX, u32, C.POINTER(ContextLayout)]),
    "afhe_dispatch": (C.c_int, [CTX, C.POINTER(AccelArgs)]),
    "afhe_set_relin_key": (C.c_int, [CTX, u64]),
    "afhe_add_rotation_key": (C.c_int, [CTX, i32, u64]),
    "afhe_has_rotation_key": (C.c_int, [CTX, i32]),
    "afhe_ntt": (C.c_int, [CTX, u64, u64, u32]),
    "afhe_intt": (C.c_int, [CTX, u64, u64, u32]),
    "afhe_poly_add": (C.c_int, [CTX, u64, u64, u64, u32]),
    "afhe_poly_sub": (C.c_int, [CTX, u64, u64, u64, u32]),
    "afhe_poly_mul_ntt": (C.c_int, [CTX, u64, u64, u64, u32]),
    "afhe_automorphism": (C.c_int, [CTX, u64, u32, u64, u32]),
    "afhe_rescale": (C.c_int, [CTX, u64, u64, u64, u64, u32]),
    "afhe_key_switch": (C.c_int, [CTX, u64, u64, u64, u64, u32]),
    "afhe_eval_add": (C.c_int, [CTX, u64, u64, u64, u64, u64, u64, u32]),
    "afhe_eval_sub_plain": (C.c_int, [CTX, u64, u64, u64, u64, u64, u32]),
    "afhe_eval_mult_relin_rescale": (C.c_int, [CTX, u64, u64, u64, u64, u64, u64, u32]),
    "afhe_eval_mult_plain_rescale": (C.c_int, [CTX, u64, u64, u64, u64, u64, u32]),
    "afhe_eval_rotate_single_step": (C.c_int, [CTX, u64, u64, u64, u64, i32, u32]),
    "afhe_eval_rotate": (C.c_int, [CTX, u64, u64, u64, u64, i32, u32]),
    "afhe_eval_mult_relin_rescale_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), C.POINTER(CtRef), u32, u32]),
    "afhe_eval_rotate_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), u32, i32, u32]),
    "afhe_ntt_batch": (C.c_int, [CTX, P64, u32, u32, C.c_int]),
    "afhe_kernel_launches": (u64, []),
    "afhe_decrypt_batch": (C.c_int, [CTX, C.POINTER(CtRef), u32, u64, u64, u32]),
    "afhe_key_switch_noalloc": (C.c_int, [CTX, C.c_void_p, u64, u32]),
    "afhe_eval_rotate_accumulate_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), u32, i32, u32]),
    "afhe_eval_rotate_accumulate_levels_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), P32, u32, i32]),
    "afhe_eval_add_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), C.POINTER(CtRef), u32, u32]),
    "afhe_eval_sub_plain_batch": (C.c_int, [CTX, C.POINTER(CtRef), P64, C.POINTER(CtRef), u32, u32]),
    "afhe_eval_mult_plain_rescale_batch": (C.c_int, [CTX, C.POINTER(CtRef), P64, C.POINTER(CtRef), u32, u32]),
    "afhe_rescale_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), u32, u32]),
    "afhe_eval_copy_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), u32, u32]),
    "afhe_eval_rotate_steps_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), C.POINTER(i32), u32, u32]),
    "afhe_ntt_plan_count": (C.c_int, [u32, P32]),
    "afhe_ntt_plan_describe": (C.c_int, [u32, u32, C.c_char_p, u32]),
    "afhe_ntt_set_plan": (C.c_int, [u32, u32]),
    "afhe_ntt_get_plan": (C.c_int, [u32, P32]),
    "afhe_automorphism_from_map": (C.c_int, [CTX, u64, u64, u64, u32, u32]),
    "afhe_automorphism_batch": (C.c_int, [CTX, P64, P32, P64, u32, u32]),
    "afhe_eval_sub_batch": (C.c_int, [CTX, C.POINTER(CtRef), C.POINTER(CtRef), C.POINTER(CtRef), u32, u32]),
    "afhe_eval_mac_plain_batch": (C.c_int, [CTX, C.POINTER(CtRef), P32, u32, C.POINTER(MacGroup), C.POINTER(MacTerm),
                                            u32, u32]),
    "afhe_ivfpq_set_units": (C.c_int, [C.c_void_p, P32, P32, u32]),
    "afhe_ivfpq_set_diagonals": (C.c_int, [C.c_void_p, u32, u64, u64, P64, P64, u32]),
    "afhe_ivfpq_set_scratch": (C.c_int, [C.c_void_p, C.POINTER(CtRef), u32]),
    "afhe_eval_diag_inner_batch": (C.c_int, [CTX, C.POINTER(CtRef), u32, C.POINTER(CtRef), u32, P64, P32, P32, u64,
                                             u32, u32]),
    "afhe_eval_add_plain_batch": (C.c_int, [CTX, C.POINTER(CtRef), P64, C.POINTER(CtRef), u32, u32]),
    "afhe_encode_batch": (C.c_int, [CTX, C.POINTER(C.c_double), u32, u32, C.c_double, u32, P64]),
    "afhe_pq_create": (C.c_int, [CTX, C.POINTER(PqIndex), C.POINTER(C.c_void_p)]),
    "afhe_pq_destroy": (C.c_int, [C.c_void_p]),
    "afhe_pq_encode_batches": (C.c_int, [C.c_void_p, P32, P32, P32, u32, C.c_double, u32, P64]),
    "afhe_pq_encode_norms": (C.c_int, [C.c_void_p, P32, P32, P32, u32, C.c_double, u32, P64]),
    "afhe_decode_batch": (C.c_int, [CTX, P64, C.POINTER(C.c_double), u32, u32, C.POINTER(C.c_double)]),
    "afhe_pq_encode_diagonals": (C.c_int, [C.c_void_p, P32, P32, P32, u32, u32, C.c_double, C.c_double, u32, P64]),
    "afhe_pq_encode_unit_norms": (C.c_int, [C.c_void_p, P32, P32, P32, u32, C.c_double, u32, P64]),
    "afhe_ivfpq_create": (C.c_int, [CTX, C.POINTER(IvfpqShape), C.POINTER(C.c_void_p)]),
    "afhe_ivfpq_destroy": (C.c_int, [C.c_void_p]),
    "afhe_ivfpq_set_centroids": (C.c_int, [C.c_void_p, P64, u32]),
    "afhe_ivfpq_set_level_masks": (C.c_int, [C.c_void_p, u32, P64, u32]),
    "afhe_ivfpq_set_prefix_mask": (C.c_int, [C.c_void_p, u32, u32, u64]),
    "afhe_ivfpq_set_list": (C.c_int, [C.c_void_p, u32, P64, P32, u32]),
    "afhe_ivfpq_set_lanes": (C.c_int, [C.c_void_p, C.POINTER(CtRef), u32, C.POINTER(CtRef)]),
    "afhe_ivfpq_set_norms": (C.c_int, [C.c_void_p, u32, P64, u32]),
    "afhe_ivfpq_set_tuning": (C.c_int, [C.c_void_p, u32, C.POINTER(KsOptions)]),
    "afhe_ivfpq_stage1": (C.c_int, [C.c_void_p, C.POINTER(IvfpqQuery), u32]),
    "afhe_ivfpq_stage3": (C.c_int, [C.c_void_p, C.POINTER(IvfpqQuery), u32]),
}

_lib = None
_lock = threading.Lock()


def header_symbols() -> list[str]:
    """Every function name declared in include/afhe.h."""
    path = os.path.join(_build.INCLUDE, "afhe.h")
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(afhe_[a-z0-9_]+)\s*\(", text)))


def load(build_if_needed: bool = True) -> C.CDLL:
    """Load libafhe.so (building it in-tree if it is missing or stale)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB
        if build_if_needed:
            path = _build.build()
        if not os.path.exists(path):
            raise RuntimeError(f"CUDA extension missing: {path}")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


class AfheError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = load()
        msg = lib.afhe_last_error().decode(errors="replace")
        name = lib.afhe_status_string(status).decode()
        super().__init__(f"{where}: status {status} ({name}): {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != OK:
        raise AfheError(status, where)
