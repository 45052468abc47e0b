"""Loader and ctypes prototypes for the in-tree CUDA libraries.

`gkr()` returns libnative_fp2_gpu.so with every entry point of
include/native_fp2.h and include/orion_gpu.h bound. It raises if the library is missing or no CUDA
device is usable: there is no CPU fallback anywhere in the product path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.realpath(__file__))
LIBDIR = os.path.join(HERE, "lib")

_U64 = ctypes.c_uint64
_I32 = ctypes.c_int
_SZ = ctypes.c_size_t
_VP = ctypes.c_void_p
_PU64 = ctypes.POINTER(_U64)
_PI32 = ctypes.POINTER(_I32)

GKR_SIGNATURES = {
    "native_fp2_init": (_I32, []),
    "native_fp2_cuda_available": (_I32, []),
    "native_fp2_fold": (None, [_PU64, _PU64, _SZ, _U64, _U64, _PU64, _PU64]),
    "native_fp2_expand": (None, [_PU64, _PU64, _SZ, _SZ, _PU64, _PU64]),
    "native_fp2_sumcheck_early": (None, [_I32, _PI32, _PI32, _PI32, _PU64, _PU64, _I32, _I32]
                                  + [_PU64] * 13),
    "native_fp2_compute_beta": (None, [_PU64, _PU64, _I32, _U64, _U64, _PU64, _PU64]),
    "native_fp2_mle_eval_base": (None, [_PU64, _PU64, _PU64, _I32, _PU64, _PU64]),
    "native_fp2_early_create": (_VP, [_I32, _PI32, _PI32, _PI32, _PU64, _PU64, _I32, _I32,
                                      _PU64, _PU64, _PU64, _PU64]),
    "native_fp2_early_claim": (_I32, [_VP, _PU64]),
    "native_fp2_early_fold": (_I32, [_VP, _U64, _U64]),
    "native_fp2_early_finish": (_I32, [_VP, _PU64, _PU64, _PU64, _PU64]),
    "native_fp2_early_n_copies": (_I32, [_VP]),
    "native_fp2_early_n_wires": (_I32, [_VP]),
    "native_fp2_early_destroy": (None, [_VP]),
    "tp_last_error_code": (_I32, []),
    "tp_last_error": (ctypes.c_char_p, []),
    "tp_clear_error": (None, []),
    "tp_last_launch_count": (_I32, []),
    "tp_gate_form": (_I32, [_I32, _PI32, _PI32, _PI32, _PU64, _PU64, _I32, _PU64, _PU64, _I32,
                            _PI32, _PU64]),
    "tp_early_create_dev": (_VP, [_I32, _VP, _VP, _VP, _VP, _VP, _I32, _I32, _VP, _VP, _I32, _VP]),
    "tp_early_claim_dev": (_I32, [_VP, _VP]),
    "tp_early_finish_dev": (_I32, [_VP, _VP, _VP]),
    "tp_early_launches": (_I32, [_VP]),
    "tp_fold_dev": (_I32, [_VP, _SZ, _U64, _U64, _VP, _VP]),
    "tp_compute_beta_dev": (_I32, [_VP, _I32, _U64, _U64, _VP, _VP]),
    "tp_mle_eval_base_dev": (_I32, [_VP, _VP, _I32, _VP, _VP]),
    "tp_table_from_pixels": (_I32, [_VP, _I32, _I32, _I32, _I32, _I32, _U64, _VP, _VP, _VP]),
    "tp_early_create_pixels": (_VP, [_I32, _VP, _VP, _VP, _VP, _VP, _VP, _I32, _I32, _I32, _I32,
                                     _I32, _U64, _VP, _VP]),
    "tp_mle_eval_pixels": (_I32, [_VP, _I32, _I32, _I32, _I32, _I32, _U64, _VP, _VP, _VP]),
    "tp_early_rounds_dev": (_I32, [_VP, _I32, _PU64, _VP]),
    "tp_batch_create": (_VP, [_I32, _VP]),
    "tp_batch_set_pixels": (_I32, [_VP, _I32, _I32, _VP, _VP, _VP, _VP, _VP, _VP, _I32, _I32, _I32,
                                   _I32, _I32, _U64, _VP]),
    "tp_batch_set_table": (_I32, [_VP, _I32, _I32, _VP, _VP, _VP, _VP, _VP, _I32, _I32, _VP, _VP,
                                  _I32]),
    "tp_batch_claim": (_I32, [_VP, _VP]),
    "tp_batch_fold": (_I32, [_VP, _PU64]),
    "tp_batch_n_copies": (_I32, [_VP, _I32]),
    "tp_batch_finish": (_I32, [_VP, _VP, _VP]),
    "tp_batch_launches": (_I32, [_VP]),
    "tp_batch_destroy": (None, [_VP]),
    "tp_batch_reset": (None, [_VP]),
    "tp_batch_finish_frame": (_I32, [_VP, _I32, _VP, _VP]),
    "tp_batch_release": (None, [_VP, _I32, _I32]),
    "tp_compute_beta_batch_dev": (_I32, [_VP, _I32, _I32, _VP, _VP]),
    "tp_mle_eval_pixels_batch": (_I32, [_I32, ctypes.POINTER(_VP), _PI32, _I32, _I32, _I32, _I32,
                                        _U64, _VP, _VP, _VP]),
    "tp_mle_eval_base_noalloc": (_I32, [_VP, _VP, _I32, _VP, _VP]),
    "tp_timer_enable": (_I32, [_I32]),
    "tp_timer_disable": (None, []),
    "tp_timer_reset": (None, []),
    "tp_timer_read": (_I32, [ctypes.POINTER(ctypes.c_float), _PI32, _I32]),
    # Orion commitment (include/orion_gpu.h)
    "tp_orion_codeword_len": (ctypes.c_longlong, [ctypes.c_longlong]),
    "tp_orion_tree_leaves": (ctypes.c_longlong, [ctypes.c_longlong]),
    "tp_orion_commit": (_I32, [_VP, ctypes.c_longlong, _VP, _VP]),
    "tp_orion_commit_dev": (_I32, [_VP, ctypes.c_longlong, _VP, _VP, _VP]),
    "tp_orion_commit_pixels_dev": (_I32, [_VP, _I32, _I32, _I32, _I32, _I32, _U64, _VP, _VP, _VP]),
    "tp_orion_commit_pair": (_I32, [_VP, _VP, ctypes.c_longlong, _VP, _VP]),
    "tp_orion_set_leaf_chunks": (_I32, [_I32]),
    "tp_orion_set_gather_lanes": (_I32, [_I32]),
    "tp_batch_fold_dev": (_I32, [_VP, _VP]),
    "tp_fs_state_bytes": (_I32, []),
    "tp_vole_state_bytes": (_I32, []),
    "tp_vole_state_init": (_I32, [_VP, _U64, _VP]),
    "tp_vole_round_dev": (_I32, [_VP, _VP, _I32, _VP, _VP, _VP, ctypes.c_longlong, ctypes.c_char_p, _VP, _VP,
                                 _VP]),
    "tp_fs_init": (_I32, [_VP, ctypes.c_char_p]),
    "tp_fs_absorb": (_I32, [_VP, _VP, ctypes.c_size_t]),
    "tp_fs_put_u64s": (_I32, [_VP, _VP, ctypes.c_size_t]),
    "tp_batch_vole_rounds_graph": (_I32, [_VP, _VP, _VP, _VP, _VP, _VP, ctypes.c_longlong, _I32, _VP, _VP, _VP, _VP]),
    "tp_batch_graph_replays": (_I32, [_VP]),
    "tp_vole_round_slots_dev": (_I32, [_VP, _VP, _I32, _VP, _VP, _VP, _VP, ctypes.c_longlong, _I32, _VP, _VP, _VP, _I32,
                                       _VP]),
    "tp_batch_autotune": (_I32, [_I32]),
    "tp_batch_tune_table": (_I32, [_VP, _VP, _VP, _I32]),
    "tp_batch_tune_set": (_I32, [_I32, _I32, _I32]),
    "tp_eq_table_host": (_I32, [_VP, _I32, _VP]),
    "tp_orion_opening_file_size": (ctypes.c_longlong, [ctypes.c_longlong, ctypes.c_longlong, _I32, _I32, _I32]),
    "tp_orion_opening_file": (ctypes.c_longlong, [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, _VP, _VP,
                                                  _VP, _VP, _I32, _VP, _VP, _VP, _VP, _I32, _VP, _VP, _I32, _I32,
                                                  _VP, ctypes.c_longlong]),
    "tp_orion_path_nodes": (_I32, [ctypes.c_longlong, _VP, _I32, _VP, _I32]),
    "tp_orion_gather_nodes_dev": (_I32, [_VP, ctypes.c_longlong, _VP, _I32, _VP, _VP]),
    "tp_fs_put_circuit_outputs_pixels": (_I32, [_VP, _VP, ctypes.c_longlong, _I32, _I32, _I32, _I32, _I32, _I32, _U64,
                                                _I32, _PI32, _PI32, _PI32]),
    "tp_host_sha_mb_available": (_I32, []),
    "tp_fs_put_fp2s": (_I32, [_VP, _VP, _VP, ctypes.c_size_t]),
    "tp_fs_put_str": (_I32, [_VP, ctypes.c_char_p]),
    "tp_fs_rand_scalar": (_I32, [_VP, _VP]),
    "tp_fs_rand_ext": (_I32, [_VP, ctypes.c_char_p, _VP, _VP]),
    "tp_fs_digest": (_I32, [_VP, _VP]),
    "tp_fs_put_fp2s_dev": (_I32, [_VP, _I32, _VP, _I32, _VP]),
    "tp_fs_rand_ext_dev": (_I32, [_VP, _I32, ctypes.c_char_p, _VP, _VP]),
    "tp_late_rounds_dev": (_I32, [_I32, _I32, _I32, _PI32, _PI32, _PI32, _VP, _VP, _VP, _I32, _VP, _VP, _VP, _VP,
                                  _VP, ctypes.c_longlong, _I32, _I32, _VP, _VP, _VP, _VP, _VP, _VP,
                                  ctypes.c_longlong, ctypes.c_longlong, _VP, _VP, _VP, _I32, _VP]),
    "tp_orion_open_queries": (_I32, [_VP, _U64, _I32, _VP, _I32, _VP, ctypes.c_longlong, ctypes.c_longlong, _I32,
                                     _I32, _VP]),
    "tp_orion_open_queries2": (_I32, [_VP, _U64, _I32, _VP, _I32, _VP, ctypes.c_longlong, ctypes.c_longlong, _I32,
                                      _I32, _VP, _VP]),
    "tp_orion_open_queries_multi": (_I32, [_I32, _VP, _U64, _VP, _VP, _I32, _VP, ctypes.c_longlong,
                                           ctypes.c_longlong, _VP, _I32, _VP, _VP]),
    "tp_orion_encode_dev": (_I32, [_VP, ctypes.c_longlong, _VP, _VP]),
    "tp_orion_verify_opening_dev": (_I32, [ctypes.c_longlong, ctypes.c_longlong, _VP, _VP, _VP, _I32, _VP, _VP, _VP,
                                           _VP, _VP, _I32, _VP, _VP, _I32, _VP, _VP, _VP, _VP]),
    "tp_fft_gkr": (_I32, [_I32, _VP, _VP, _VP, _VP, ctypes.c_char_p]),
    "tp_circuit_out_bits": (_I32, [_I32]),
    "tp_circuit_outputs_pixels_dev": (_I32, [_VP, _I32, _I32, _I32, _I32, _I32, _U64, _I32, _PI32, _PI32, _PI32,
                                            _VP, _VP]),
    "tp_virgo_layer_create": (_VP, [_I32, _I32, _VP, _VP, _VP, _VP, _VP, _VP]),
    "tp_virgo_layer_destroy": (None, [_VP]),
    "tp_virgo_phase1_init_dev": (_I32, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "tp_virgo_phase2_init_dev": (_I32, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "tp_orion_commit_zk_pixels_dev": (_I32, [_VP, _I32, _I32, _I32, _I32, _I32, _U64, _U64, _VP, _VP, _VP, _VP,
                                             _VP]),
    "tp_orion_pixel_vector_dev": (_I32, [_VP, _I32, _I32, _I32, _I32, _I32, _U64, _U64, _I32, _VP, _VP]),
    "tp_orion_rows_to_columns_dev": (_I32, [_VP, ctypes.c_longlong, _VP, _VP]),
    "tp_orion_last_launches": (_I32, []),
    "tp_orion_combine_dev": (_I32, [_VP, ctypes.c_longlong, _VP, _VP, _VP, _VP]),
    "tp_orion_query_columns_dev": (_I32, [_VP, ctypes.c_longlong, _VP, _I32, _VP, _VP]),
    "tp_orion_query_columns_async_dev": (_I32, [_VP, ctypes.c_longlong, _VP, _I32, _VP, _VP, _VP]),
    "tp_orion_answer_dev": (_I32, [_VP, ctypes.c_longlong, _VP, _VP, _VP]),
    "tp_sha256_peak_dev": (_I32, [_I32, _I32, _VP, _VP]),
    "tp_fft": (_I32, [_VP, _I32, _I32, _VP]),
    "tp_ifft": (_I32, [_VP, _I32, _I32, _VP]),
    "tp_fft_dev": (_I32, [_VP, ctypes.c_longlong, ctypes.c_longlong, _VP, _I32, ctypes.c_longlong,
                          ctypes.c_longlong, _VP]),
    "tp_ifft_dev": (_I32, [_VP, ctypes.c_longlong, ctypes.c_longlong, _VP, _I32, ctypes.c_longlong,
                           ctypes.c_longlong, _VP]),
    "tp_ntt_autotune": (_I32, [_I32, _I32, _PI32, ctypes.POINTER(ctypes.c_float)]),
    "tp_rs_commit": (_I32, [_VP, _I32, _VP, _VP]),
    "tp_fri_commit_step_dev": (_I32, [_VP, _I32, _U64, _U64, _VP, _VP, _VP]),
    "tp_rs_commit_dev": (_I32, [_VP, _I32, _VP, _VP, _VP]),
    "tp_virgo_sumcheck_update_dev": (_I32, [_VP, _VP, _VP, ctypes.c_longlong, _U64, _U64, _I32, _VP, _VP,
                                            _VP, _VP, _VP]),
}

_cache = {}


def _bind(path: str, sigs: dict, keep_lock: bool = False):
    lib = (ctypes.PyDLL if keep_lock else ctypes.CDLL)(path)
    for name, (res, args) in sigs.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    return lib


def lib_path(name: str) -> str:
    return os.path.join(LIBDIR, name)


def gkr(require_device: bool = True):
    """libnative_fp2_gpu.so, bound; raises when unusable."""
    if "gkr" not in _cache:
        path = os.environ.get("TRUEPIX_NATIVE_FP2_GPU_LIB", lib_path("libnative_fp2_gpu.so"))
        if not os.path.isfile(path):
            raise RuntimeError(f"CUDA library missing: {path} (run python -m truepix_b200.build)")
        _cache["gkr"] = _bind(path, GKR_SIGNATURES)
    lib = _cache["gkr"]
    if require_device:
        lib.native_fp2_init()
        if not lib.native_fp2_cuda_available():
            raise RuntimeError("no usable CUDA device: " + lib.tp_last_error().decode())
    return lib


def gkr_launcher():
    """The same library bound so that its calls keep the interpreter lock, for
    entry points that only queue device work (microseconds each): a launching
    thread that gives the lock up for each of hundreds of such calls per batch
    waits to take it back from the host threads every time."""
    if "gkr_launcher" not in _cache:
        gkr(require_device=False)
        path = os.environ.get("TRUEPIX_NATIVE_FP2_GPU_LIB", lib_path("libnative_fp2_gpu.so"))
        _cache["gkr_launcher"] = _bind(path, GKR_SIGNATURES, keep_lock=True)
    return _cache["gkr_launcher"]


def check(lib, rc=0, what="call"):
    """Raise with the library's message when rc is an error or an error is recorded."""
    if (rc is not None and rc != 0) or lib.tp_last_error_code() != 0:
        raise RuntimeError(f"{what} failed: {lib.tp_last_error().decode()}")
