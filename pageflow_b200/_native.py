"""ctypes binding of libpageflow_b200.so, the C ABI declared in
include/pageflow_b200.h.  Loading fails loudly when the library is missing:
there is no CPU fallback anywhere in the package."""
from __future__ import annotations

import ctypes
from pathlib import Path

import torch

import os

# The in-tree build; PAGEFLOW_B200_LIB names another build of the same
# sources (e.g. one compiled with different tuning macros).
LIB_PATH = Path(os.environ.get("PAGEFLOW_B200_LIB",
                               Path(__file__).resolve().parent / "libpageflow_b200.so"))

class JoinKnobs(ctypes.Structure):
    """pf_join_knobs: the run-time choices of a fused join + group-by."""
    _fields_ = [("path", ctypes.c_int), ("table", ctypes.c_int), ("sub_rows", ctypes.c_int),
                ("counted", ctypes.c_int)]


PF_OK = 0
PF_EINVAL = -1
PF_ECUDA = -2
PF_ETIMEOUT = -3
PF_ENOSPACE = -4
PF_EDEVICE = -5

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_sz = ctypes.c_size_t

# name -> (restype, argtypes)
_SIGS = {
    "pf_last_error": (ctypes.c_char_p, []),
    "pf_version": (ctypes.c_char_p, []),
    "pf_set_wait_timeout_ms": (None, [_i64]),
    "pf_launch_count": (_i64, []),
    "pf_profile_begin": (None, []),
    "pf_profile_end": (_int, [_int, ctypes.c_char_p, _int, ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(_i64)]),
    "pf_rows_per_unit": (_i64, [_i64]),
    "pf_partition_sort_workspace": (_sz, [_i64, _i64, _int, _int, _int]),
    "pf_partition_sort": (_int, [_vp, _vp, _vp, _vp, _int, _int, _vp, _i64, _i64,
                                 _i64, _int, _int, _vp, _vp, _vp, _sz, _vp]),
    "pf_join_unique_hash_workspace": (_sz, [_i64, _i64]),
    "pf_join_unique_hash": (_int, [_vp, _vp, _i64, _vp, _vp, _i64, _int, _vp, _vp,
                                   _vp, _vp, _sz, _vp]),
    "pf_join_unique_hash_static": (_int, [_vp, _vp, _i64, _vp, _vp, _i64, _int, _vp, _vp, _vp,
                                          _vp]),
    "pf_gather_segments_workspace": (_sz, [_int, _int]),
    "pf_gather_segments": (_int, [_vp, _vp, _int, _i64, _int, _vp, _vp, _vp, _vp, _vp, _i64,
                                  _int, _i64, _vp, _vp, _vp, _sz, _vp]),
    "pf_gather": (_int, [_vp, _vp, _vp, _vp, _vp, _int, _vp, _i64, _i64, _int, _i64, _vp, _vp]),
    "pf_join_semi_anti_workspace": (_sz, [_i64, _i64, _int]),
    "pf_join_semi_anti": (_int, [_vp, _i64, _vp, _i64, _vp, _vp, _int, _int, _vp,
                                 _vp, _vp, _sz, _vp]),
    "pf_join_expand_workspace": (_sz, [_i64]),
    "pf_join_expand_prepare": (_int, [_vp, _i64, _vp, _vp, _sz, _vp]),
    "pf_join_expand": (_int, [_vp, _vp, _vp, _i64, _i64, _vp, _vp, _vp, _sz, _vp]),
    "pf_slab_add": (_int, [_vp, _int, _i64, _i64, _i64, _vp, _int, _vp, _vp, _vp,
                           _vp, _vp, _vp, _vp]),
    "pf_slab_finish_workspace": (_sz, [_i64]),
    "pf_slab_finish": (_int, [_vp, _i64, _i64, _int, _vp, _vp, _vp, _vp, _vp, _vp,
                              _vp, _sz, _vp]),
    "pf_join_aggregate_workspace": (_sz, [_i64, _i64, _int, _i64]),
    "pf_join_aggregate": (_int, [_vp, _vp, _i64, _vp, _vp, _vp, _i64, _i64, _int,
                                 _i64, _i64, _vp, _vp, _vp, _vp, _sz, _vp]),
    "pf_join_aggregate_workspace_ex": (_sz, [_i64, _i64, _int, _i64, _vp]),
    "pf_join_aggregate_ex": (_int, [_vp, _vp, _i64, _vp, _vp, _vp, _i64, _i64, _int, _i64, _i64,
                                    _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "pf_join_partition_workspace": (_sz, [_i64, _i64, _int]),
    "pf_join_partition": (_int, [_vp, _vp, _i64, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp, _vp,
                                 _vp, _vp, _sz, _vp]),
    "pf_join_aggregate_buckets_workspace": (_sz, [_vp, _int, _i64, _vp]),
    "pf_join_aggregate_buckets": (_int, [_vp, _vp, _vp, _vp, _int, _int, _i64, _i64, _vp, _vp,
                                         _vp, _vp, _vp, _sz, _vp]),
    "pf_join_aggregate_pick_b": (_int, [_i64, _i64]),
    "pf_join_aggregate_counted_passes": (_int, []),
    "pf_groups_finish_workspace": (_sz, [_i64]),
    "pf_groups_finish": (_int, [_vp, _vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _sz,
                                _vp]),
    "pf_gen_build": (_int, [_int, ctypes.c_uint64, _i64, _i64, _i64, _i64, _vp, _vp,
                            _vp]),
    "pf_gen_probe": (_int, [_int, ctypes.c_uint64, _i64, _i64, _i64, _vp, _vp, _vp,
                            _vp]),
    "pf_gen_batch_probe": (_int, [ctypes.c_uint64, _i64, _i64, _i64, _int, _vp, _vp, _vp, _vp,
                                  _vp]),
    "pf_group_hash": (_int, [_vp, _vp, _vp, _int, _i64, _vp, _vp]),
    "pf_hash_buckets": (_int, [_vp, _i64, _int, _vp, _vp, _vp]),
    "pf_sort_pairs_workspace": (_sz, [_i64]),
    "pf_sort_pairs": (_int, [_vp, _vp, _i64, _vp, _vp, _vp, _sz, _vp]),
    "pf_unique_reduce_workspace": (_sz, [_i64]),
    "pf_unique_reduce": (_int, [_vp, _i64, _int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                ctypes.POINTER(_i64), _vp, _sz, _vp]),
    "pf_merge_sorted_runs_workspace": (_sz, [_i64]),
    "pf_merge_sorted_runs": (_int, [_vp, _vp, _i64, _vp, _vp, _i64, _int, _vp, _vp, _vp, _vp,
                                    _vp, _vp, ctypes.POINTER(_i64), _vp, _sz, _vp]),
    "pf_encode_pages_workspace": (_sz, [_int]),
    "pf_encode_pages": (_int, [_vp, _int, _vp, _int, _vp, _i64, _vp, _vp, _sz, _vp]),
    "pf_page_encode": (_i64, [_vp, _int, _i64, _vp, _i64]),
    "pf_paged_generate": (_int, [ctypes.c_uint64, _i64, _int, _i64, _vp, _vp, _int, _int,
                                 ctypes.POINTER(_vp), ctypes.POINTER(_i64)]),
    "pf_paged_fetch": (_int, [_vp, _vp, _vp, ctypes.POINTER(_i64)]),
    "pf_paged_scan_workspace": (_sz, [_vp, _i64, _int, _i64, _int, _int]),
    "pf_paged_scan": (_int, [_vp, _vp, _i64, _int, _vp, _i64, _i64, _int, _int, _i64, _i64,
                             _int, _int, _int, _vp, _i64, _vp, _vp, _vp, _sz, _vp]),
    "pf_dim_table_bytes": (_sz, [_i64]),
    "pf_dim_build": (_int, [_vp, _vp, _i64, _i64, _vp, _sz, _vp, _vp]),
    "pf_serve_workspace": (_sz, [_int]),
    "pf_serve_run": (_int, [_vp, _int, _vp, _sz, _vp, _vp]),
    "pf_gen_serve_dim": (_int, [ctypes.c_uint64, _i64, ctypes.c_uint64, _i64, _i64, _i64, _i64,
                                _vp, _vp, _vp]),
    "pf_gen_serve_fact": (_int, [ctypes.c_uint64, _i64, _int, _vp, _vp, _i64, _i64, _vp, _vp,
                                 _vp, _vp]),
    "pf_batch_workspace": (_sz, [_vp, _int]),
    "pf_batch_prepare": (_int, [_vp, _int, _vp, _sz, _vp]),
    "pf_batch_run": (_int, [_vp, _vp, _vp]),
    "pf_batch_slab": (_vp, [_vp, _int]),
}


class BatchInstance(ctypes.Structure):
    """pf_batch_instance (include/pageflow_b200.h)."""
    _fields_ = [("build_key", _vp), ("build_group", _vp), ("n_build", _i64),
                ("probe_fk", _vp), ("probe_value", _vp), ("n_probe", _i64),
                ("group_min", _i64), ("n_groups", _i64)]

class ServeRequest(ctypes.Structure):
    """pf_serve_request (include/pageflow_b200.h)."""
    _fields_ = [("table", _vp), ("n_keys", _i64), ("n_groups", _i64), ("fk", _vp),
                ("date", _vp), ("value", _vp), ("row_begin", _i64), ("row_end", _i64),
                ("date_lo", ctypes.c_int32), ("date_hi", ctypes.c_int32),
                ("finish", ctypes.c_int32), ("pad", ctypes.c_int32), ("slab", _vp),
                ("out_keys", _vp), ("out_sums", _vp), ("out_counts", _vp), ("out_n", _vp),
                ("done", _vp)]


_lib = None


class NativeLibraryMissing(ImportError):
    pass


def lib():
    """The loaded library (loaded once)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise NativeLibraryMissing(
                f"{LIB_PATH} is missing: build it with `python -m pageflow_b200.build` "
                f"(pageflow_b200 has no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def launch_count() -> int:
    """Kernels the library has launched in this process."""
    return int(lib().pf_launch_count())


def profile_begin() -> None:
    lib().pf_profile_begin()


def profile_end(max_kernels: int = 64) -> dict:
    """{kernel name: (total ms, launches)} of the calling thread's launches
    since profile_begin (waits for their events)."""
    name_len = 64
    names = ctypes.create_string_buffer(max_kernels * name_len)
    ms = (ctypes.c_double * max_kernels)()
    cnt = (_i64 * max_kernels)()
    n = lib().pf_profile_end(max_kernels, names, name_len, ms, cnt)
    if n < 0:
        check(n, "profile_end")
    out = {}
    raw = names.raw
    for i in range(min(n, max_kernels)):
        nm = raw[i * name_len:(i + 1) * name_len].split(b"\0", 1)[0].decode()
        out[nm] = (ms[i], int(cnt[i]))
    return out


def check(rc: int, what: str) -> None:
    """Raises RuntimeError (as the reference's TORCH_CHECK does) for a
    failed call, with the library's message."""
    if rc != PF_OK:
        msg = lib().pf_last_error().decode(errors="replace")
        raise RuntimeError(f"{what}: {msg} (status {rc})")


def ptr(t) -> int | None:
    """A tensor's data pointer (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_of(device) -> int:
    """The current torch stream of `device`, as the C ABI's stream handle."""
    return torch.cuda.current_stream(device).cuda_stream


def workspace(nbytes: int, device) -> torch.Tensor:
    """Scratch from torch's caching allocator (the pooled device arena)."""
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def arr(ctype, values):
    """A ctypes array of `values`."""
    values = list(values)
    return (ctype * max(len(values), 1))(*values)


def require_cuda(t: torch.Tensor, what: str) -> None:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RuntimeError(f"{what} must be a CUDA tensor")
