"""ctypes binding of librotormap_b200.so (the C ABI declared in include/r2m.h).

The library is built in-tree (qpg-rotormap_b200/build.py).  There is no
fallback: if the shared object is missing or no sm_100 device is present,
every entry point raises R2MError.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

LIB_PATH = Path(os.environ.get(
    "R2M_LIB", Path(__file__).resolve().parent.parent / "lib" / "librotormap_b200.so"))

R2M_OK, R2M_EINVAL, R2M_ECUDA, R2M_ENOMEM, R2M_ETIMEOUT, R2M_ESTATE, R2M_EIO = 0, -1, -2, -3, -4, -5, -6
OUT_F32, OUT_F16, OUT_E4M3, OUT_E4M3_SCALED = 0, 1, 2, 3
SCORE_F16, SCORE_F32, SCORE_SCALED = 0, 1, 2

_CODES = {R2M_EINVAL: "EINVAL", R2M_ECUDA: "ECUDA", R2M_ENOMEM: "ENOMEM", R2M_ETIMEOUT: "ETIMEOUT",
          R2M_ESTATE: "ESTATE", R2M_EIO: "EIO"}


class R2MError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"r2m error {_CODES.get(code, code)}: {msg}")
        self.code = code


class Tuning(ctypes.Structure):
    _fields_ = [("splits", ctypes.c_int), ("ctas", ctypes.c_int), ("reserved", ctypes.c_int * 6)]


# (name, restype, argtypes) of every symbol in include/r2m.h
P = ctypes.c_void_p
I = ctypes.c_int
I64 = ctypes.c_int64
SZ = ctypes.c_size_t
SIGNATURES = [
    ("r2m_last_error", ctypes.c_char_p, []),
    ("r2m_version", I, []),
    ("r2m_device_check", I, []),
    ("r2m_check_device_error", I, [P]),
    ("r2m_selftest_bounded_wait", I, [I64, I, P]),
    ("r2m_encode_frag_real_batch", I, [P, I, P, P, P, I64, I, I, I, I, I, P]),
    ("r2m_revcomp_frag_words", I, [P, P, I, I64, P]),
    ("r2m_encode_ref_windows", I, [P, I, P, P, P, P, I64, I64, I, I, I, I, I, P]),
    ("r2m_f32_to_e4m3", I, [P, P, I64, P]),
    ("r2m_f16_to_e4m3", I, [P, P, I64, P]),
    ("r2m_engine_create", I, [P, P, I, I64, I, I, I, ctypes.POINTER(Tuning), ctypes.POINTER(P)]),
    ("r2m_engine_destroy", I, [P]),
    ("r2m_engine_set_tuning", I, [P, ctypes.POINTER(Tuning)]),
    ("r2m_engine_workspace_bytes", I64, [P]),
    ("r2m_engine_kernel_ms", I, [P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                 ctypes.POINTER(I)]),
    ("r2m_batch_gemm_topk", I, [P, P, P, I, P, P, P]),
    ("r2m_batch_gemm_topk_noalloc", I, [P, P, I, I64, P, P, I, I, I, P, P, P]),
    ("r2m_selftest_noalloc_timeout", I, [I64, I, I, P, P, P]),
    ("r2m_rescore_fp32", I, [P, I, P, I, P, P, P, I64, I, I, I, I, I, P, P, P, I, P]),
    ("r2m_check_fp64", I, [P, I, P, P, P, I64, I, I, I, I, P, I, P, P, P, P]),
    ("r2m_plain_engine_create", I, [P, I, I64, I, I, I, I, ctypes.POINTER(P)]),
    ("r2m_plain_engine_destroy", I, [P]),
    ("r2m_plain_batch_gemm_topk", I, [P, P, I, P, P, P]),
    ("r2m_fasta_reads", I, [ctypes.c_char_p, SZ, I, I, ctypes.POINTER(P)]),
    ("r2m_reads_count", I64, [P]),
    ("r2m_reads_words", P, [P]),
    ("r2m_reads_header", P, [P, I64, ctypes.POINTER(SZ)]),
    ("r2m_reads_header_blob", P, [P, ctypes.POINTER(SZ)]),
    ("r2m_reads_header_offsets", P, [P]),
    ("r2m_reads_free", None, [P]),
    ("r2m_format_table", I, [P, P, I64, I, ctypes.c_char_p, SZ, P, P, P, I64, ctypes.c_char_p, SZ, I,
                             ctypes.POINTER(P)]),
    ("r2m_text_data", P, [P, ctypes.POINTER(SZ)]),
    ("r2m_text_free", None, [P]),
    ("r2m_format_f32", I, [ctypes.c_float, ctypes.c_char_p, SZ]),
    ("r2m_compact_create", I, [P, P, I, I64, I, I, I, I64, I, I, I, P, ctypes.POINTER(P)]),
    ("r2m_compact_resident_chunks", I64, [P]),
    ("r2m_merge_topk_lists", I, [P, P, I, I, I, I, P, P, P]),
    ("r2m_compact_destroy", I, [P]),
    ("r2m_compact_chunks", I64, [P]),
    ("r2m_compact_is_pinned", I, [P]),
    ("r2m_compact_batch_gemm_topk", I, [P, P, P, I, P, P, P]),
    ("r2m_fasta_genome", I, [ctypes.c_void_p, SZ, I, ctypes.POINTER(P)]),
    ("r2m_genome_count", I64, [P]),
    ("r2m_genome_words", P, [P, ctypes.POINTER(SZ)]),
    ("r2m_genome_word_off", P, [P]),
    ("r2m_genome_nbases", P, [P]),
    ("r2m_genome_header_blob", P, [P, ctypes.POINTER(SZ)]),
    ("r2m_genome_free", None, [P]),
    ("r2m_fasta_reads_device", I, [P, SZ, I, P, ctypes.POINTER(P)]),
    ("r2m_dreads_count", I64, [P]),
    ("r2m_dreads_stopped", I, [P]),
    ("r2m_dreads_words", P, [P]),
    ("r2m_dreads_spans", P, [P]),
    ("r2m_dreads_header_blob", P, [P, ctypes.POINTER(SZ)]),
    ("r2m_dreads_free", None, [P]),
    ("r2m_engine_info", I, [P, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I),
                            ctypes.POINTER(I64)]),
    ("r2m_server_create", I, [P, I, I, I, I, I, I64, I64, I, ctypes.POINTER(P)]),
    ("r2m_server_submit", I, [P, P, I64, P, P, ctypes.c_double, ctypes.POINTER(I64)]),
    ("r2m_server_submit_fasta", I, [P, ctypes.c_char_p, SZ, I, ctypes.c_double, ctypes.POINTER(I64),
                                    ctypes.POINTER(I64)]),
    ("r2m_server_cancel", I, [P, I64]),
    ("r2m_server_wait", I, [P, I64, ctypes.c_double, ctypes.POINTER(I)]),
    ("r2m_server_request", I, [P, I64, ctypes.POINTER(I), ctypes.POINTER(I64), ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("r2m_server_request_error", ctypes.c_char_p, [P, I64]),
    ("r2m_server_copy_result", I, [P, I64, P, P]),
    ("r2m_server_reads", P, [P, I64]),
    ("r2m_server_release", I, [P, I64]),
    ("r2m_server_get_stats", I, [P, P]),
    ("r2m_server_request_bytes", I64, [P, I64]),
    ("r2m_server_destroy", I, [P, I]),
    ("r2m_jlbin_open", I, [ctypes.c_char_p, ctypes.POINTER(P)]),
    ("r2m_jlbin_parse", I, [P, SZ, ctypes.POINTER(P)]),
    ("r2m_jlbin_version", I, [P]),
    ("r2m_jlbin_nfields", I, [P]),
    ("r2m_jlbin_field", I, [P, I, P]),
    ("r2m_jlbin_close", None, [P]),
    ("r2m_jlbin_write", I, [ctypes.c_char_p, P, I]),
]

_lib = None
_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    """Load the library once; raises R2MError when it has not been built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not LIB_PATH.exists():
                    raise R2MError(R2M_ESTATE, f"{LIB_PATH} not found: build it with "
                                               "`python qpg-rotormap_b200/build.py`")
                L = ctypes.CDLL(str(LIB_PATH))
                for name, res, args in SIGNATURES:
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != R2M_OK:
        msg = lib().r2m_last_error()
        raise R2MError(rc, msg.decode() if msg else "")


def ptr(t) -> int | None:
    """Device/host address of a torch tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def stream_handle(stream=None) -> int | None:
    """cudaStream_t of a torch stream (default: torch's current stream)."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def require_device() -> None:
    """Fail loudly unless an sm_100 GPU is current (no CPU fallback exists)."""
    import torch
    if not torch.cuda.is_available():
        raise R2MError(R2M_ESTATE, "no CUDA device: librotormap_b200 runs on B200 (sm_100a) only")
    check(lib().r2m_device_check())
