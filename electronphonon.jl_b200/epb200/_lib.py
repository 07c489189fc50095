"""ctypes binding of libepb200.so (the sm_100a C ABI declared in include/epb200.h).

The compute path is the shared library only: if it cannot be loaded, or no CUDA device is visible,
every call raises. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libepb200.so")

EPB_OK = 0
EPB_ERR_ARG = 1
EPB_ERR_OOM = 2
EPB_ERR_CUDA = 3
EPB_ERR_TIMEOUT = 4
EPB_ERR_UNSUPPORTED = 5
EPB_ERR_NOCONVERGE = 6
PREC_FP64 = 0
PREC_MIXED = 1

_STATUS = {1: "EPB_ERR_ARG", 2: "EPB_ERR_OOM", 3: "EPB_ERR_CUDA", 4: "EPB_ERR_TIMEOUT",
           5: "EPB_ERR_UNSUPPORTED", 6: "EPB_ERR_NOCONVERGE"}

P = C.c_void_p
I64 = C.c_int64
I32 = C.c_int
D = C.c_double

# name -> argtypes (restype is int unless listed in _RESTYPE)
SIGNATURES = {
    "epb_create": [C.POINTER(P), I32, P],
    "epb_destroy": [P],
    "epb_set_stream": [P, P],
    "epb_free_bytes": [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
    "epb_synchronize": [P],
    "epb_last_error": [],
    "epb_version": [],
    "epb_workspace_bytes": [P, C.POINTER(C.c_uint64)],
    "epb_debug_fail_alloc": [P, I32],
    "epb_launch_count": [P, C.POINTER(I64)],
    "epb_profile_enable": [P, I32],
    "epb_profile_read": [P, P, P, I32, I32],
    "epb_rset_create": [P, P, I64, C.POINTER(P)],
    "epb_rset_destroy": [P],
    "epb_fourier_phase": [P, P, P, I64, P],
    "epb_fourier_phase_mat": [P, P, I64, I64, P, I64, I64, P, I64],
    "epb_batched_zgemm": [P, C.c_char, C.c_char, I64, I64, I64, P, I64, I64, P, I64, I64, P, I64, I64, I64],
    "epb_fourier": [P, P, I64, I64, P, P, I64, P, I32],
    "epb_eigh_batched": [P, P, I64, I64, P, C.c_char, I32],
    "epb_eigh_varlen": [P, P, P, P, I64, P, P, C.c_char, I32],
    "epb_eigh_varlen_async": [P, P, P, P, I64, P, P, C.c_char, I32],
    "epb_eigh_status": [P],
    "epb_ph_eigen_batched": [P, P, P, I64, I64, P, I32],
    "epb_eph_RR_to_kR": [P, P, I64, I64, I64, P, P, I64, P, I64, P, P, I32],
    "epb_eph_apply_rotations": [P, P, I64, I64, I64, I64, I64, P, I64, P, P, P, P],
    "epb_eph_kR_to_kq": [P, P, I64, I64, I64, I64, I64, P, I64, P, I64, P, P, P, P, I32],
    "epb_window_filter": [P, P, I64, I64, D, D, P, P, P, P, P],
    "epb_window_filter_noalloc": [P, P, I64, I64, D, D, P, P, P, P, P],
    "epb_filtered_states": [P, P, P, I64, I64, P, P, P, I64, P],
    "epb_fill_iqs": [P, P, I64, P, I64, I64, I64, P, P],
    "epb_model_create": [P, P, I64, P, I64, P, P, I64, P, I64, P, P, I64, I32, C.POINTER(P)],
    "epb_model_destroy": [P],
    "epb_eph_pass": [P, P, P, I64, P, I64, I32, I64, I64, P, P, P, P, P],
    "epb_set_rotation_variant": [P, I32],
    "epb_tune_table_create": [C.POINTER(P)],
    "epb_tune_table_destroy": [P],
    "epb_tune_table_set": [P, C.c_char_p, I64],
    "epb_tune_table_get": [P, C.c_char_p, C.POINTER(I64), C.POINTER(I32)],
    "epb_tune_table_size": [P, C.POINTER(I64)],
    "epb_tune_table_serialize": [P, C.c_char_p, I64, C.POINTER(I64)],
    "epb_tune_table_parse": [P, C.c_char_p],
    "epb_tune_export": [P, P],
    "epb_tune_import": [P, P],
    "epb_bands_create": [P, P, I64, P, I64, C.POINTER(P)],
    "epb_bands_destroy": [P],
    "epb_bands_eigvals": [P, P, P, I64, P, I32],
    "epb_bands_band_energy": [P, P, P, I64, I64, P, I32],
    "epb_bands_window": [P, P, P, I64, D, D, I32, D, P, P, P, C.POINTER(I64), P],
    "epb_pair_window": [P, P, P, I64, P, I64, D, D, P, I32, D, P, P, P, I64, C.POINTER(I64), P],
    "epb_mlp_create": [P, P, I64, I64, I64, I64, C.c_uint64, C.POINTER(P)],
    "epb_mlp_destroy": [P],
    "epb_mlp_info": [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)],
    "epb_mlp_get_params": [P, P, P],
    "epb_mlp_set_params": [P, P, P],
    "epb_mlp_set_scaling": [P, P, P, P],
    "epb_mlp_get_scaling": [P, P, P, P],
    "epb_mlp_features": [P, P, P, I64, P],
    "epb_mlp_loss_grad": [P, P, P, P, I64, P, P],
    "epb_mlp_train": [P, P, P, P, I64, P, P],
    "epb_mlp_predict": [P, P, P, I64, P],
    "epb_mlp_calibrate": [P, P, P, P, I64, D, P],
    "epb_mlp_set_inference": [P, I32],
    "epb_bte_serta": [P, P, P, P, P, I64, P],
    "epb_set_graph_mode": [P, I32],
    "epb_epmat_el_to_ph": [P, P, I64, I64, I64, I64, P],
    "epb_eph_RR_to_Rq": [P, P, I64, I64, I64, P, P, I64, P, P, I32],
    "epb_eph_Rq_to_kq": [P, P, I64, I64, P, P, I64, P, I64, P, I64, P, P, P, I32],
    "epb_eph_outer_q": [P, P, P, P, I64, P, I64, P, P, I32, P, P],
    "epb_ind_range_for_k_range": [P, I64, I64, I64, I64, P, P],
    "epb_read_epmat": [P, C.c_char_p, I64, I64, I64, I64, P, P, P, I64, P, I64, I64, I32, I32, I32, P],
    "epb_tiled_plan": [P, I64, I64, I64, P],
    "epb_residency_use_block": [P, I64, D, P],
    "epb_tiled_create": [P, P, I32, I32, I32, I64, I32, D, P, I64, I64, I64, P],
    "epb_tiled_begin": [P, P, I64, I64],
    "epb_tiled_get_info": [P, P],
    "epb_tiled_device_array": [P, I32, P],
    "epb_tiled_download": [P, P, I32, P],
    "epb_tiled_free": [P],
    "epb_tiled_destroy": [P],
    "epb_eph_window_scatter": [P, P, P, P, P, P, I64, P, P, I64, I64, I64, I64, I64, I64],
    "epb_bte_window_accumulate": [P, P, I64, P, I64, I64, P, P, P, P, I64, P, P, P, P, P, P, P, I64, I32, D, I64, I64,
                                  I64, I64, I64],
    "epb_mlp_inference_path": [P, C.POINTER(I32)],
}


class WindowStats(C.Structure):
    """epb_window_stats."""
    _fields_ = [("tested", I64), ("culled", I64), ("evaluated", I64), ("rechecked", I64), ("kept", I64),
                ("audited", I64), ("violations", I64), ("fallback_chunks", I64), ("screened", I64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class BteParams(C.Structure):
    """epb_bte_params."""
    _fields_ = [("ngrid", I64), ("wmin", D), ("wmax", D), ("mu", D), ("temperature", D), ("smearing", D),
                ("omega_cutoff", D), ("spin_degeneracy", D), ("volume", D), ("lattice", D * 9), ("method", C.c_int32),
                ("prec", C.c_int32), ("k_batch", I64), ("pair_chunk", I64), ("shard_rank", I64),
                ("shard_count", I64)]


class TiledInfo(C.Structure):
    """epb_tiled_info."""
    _fields_ = [("allocated", C.c_int32), ("block", C.c_int32), ("ni_cap", I64), ("tile_offset", I64),
                ("tile_length", I64), ("tile_stride", I64)]


class OuterQParams(C.Structure):
    """epb_outer_q_params."""
    _fields_ = [("wmin_k", D), ("wmax_k", D), ("wmin_kq", D), ("wmax_kq", D), ("k_batch", I64), ("q_chunk", I64),
                ("prec", C.c_int32), ("phonon_basis", C.c_int32)]


class KBatchPayload(C.Structure):
    """epb_kbatch_payload (device pointers)."""
    _fields_ = [("iq", I64), ("k0", I64), ("nk", I64), ("nw", I64), ("nm", I64), ("eps", P), ("ek", P), ("ekq", P),
                ("uk", P), ("ukq", P), ("wtk", P), ("xk", P), ("ik", P), ("omega", P), ("stream", P)]


BEGIN_Q_FN = C.CFUNCTYPE(C.c_int, P, I64, P)
RUN_BATCH_FN = C.CFUNCTYPE(C.c_int, P, C.POINTER(KBatchPayload))
END_Q_FN = C.CFUNCTYPE(C.c_int, P, I64, P)


class OuterQCalc(C.Structure):
    """epb_outer_q_calc."""
    _fields_ = [("begin_q", BEGIN_Q_FN), ("run_batch", RUN_BATCH_FN), ("end_q", END_Q_FN), ("user", P)]


class MlpTrainOpts(C.Structure):
    """epb_mlp_train_opts."""
    _fields_ = [("epochs", I64), ("batch", I64), ("lr", D), ("lr_final", D), ("seed", C.c_uint64),
                ("use_graph", C.c_int32), ("reserved", C.c_int32)]
_RESTYPE = {"epb_last_error": C.c_char_p}

_lock = threading.Lock()
_lib = None


def lib():
    """Load (once) and return the library with every signature bound."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"libepb200.so not built ({LIB_PATH}); run electronphonon.jl_b200/build.py")
            L = C.CDLL(LIB_PATH)
            for name, argt in SIGNATURES.items():
                f = getattr(L, name)
                f.argtypes = argt
                f.restype = _RESTYPE.get(name, C.c_int)
            _lib = L
    return _lib


class EpbError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


def check(status):
    if status != EPB_OK:
        raise EpbError(status, lib().epb_last_error().decode(errors="replace"))
    return status


def ptr(t):
    """Device (or host) address of a torch tensor / numpy array, or None."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


class Context:
    """One epb_ctx bound to a device and a CUDA stream (torch's current stream by default)."""

    def __init__(self, device=0, stream=None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("epb200 needs a CUDA device (sm_100a); none is visible")
        L = lib()
        torch.cuda.set_device(device)
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self.stream = stream
        h = P()
        check(L.epb_create(C.byref(h), int(device), P(stream.cuda_stream)))
        self.h = h
        self.device = device

    def set_stream(self, stream):
        self.stream = stream
        check(lib().epb_set_stream(self.h, P(stream.cuda_stream)))

    def synchronize(self):
        check(lib().epb_synchronize(self.h))

    def set_rotation_variant(self, variant):
        """Rotation kernel of the mixed pass (nw = 16, nm = 12): 0 warp tensor cores, 1 FP32, -1 autotuned."""
        check(lib().epb_set_rotation_variant(self.h, int(variant)))

    def tune_text(self):
        """The context's tuning table as text (one "key value" per line)."""
        t = TuneTable()
        t.export_from(self)
        return t.text()

    def set_graph_mode(self, on=True):
        """Capture epb_eph_pass as a CUDA graph and replay it for repeated calls on the same buffers."""
        check(lib().epb_set_graph_mode(self.h, 1 if on else 0))

    def free_bytes(self):
        f, t = C.c_uint64(), C.c_uint64()
        check(lib().epb_free_bytes(self.h, C.byref(f), C.byref(t)))
        return f.value, t.value

    def workspace_bytes(self):
        b = C.c_uint64()
        check(lib().epb_workspace_bytes(self.h, C.byref(b)))
        return b.value

    def launch_count(self):
        c = I64()
        check(lib().epb_launch_count(self.h, C.byref(c)))
        return c.value

    PROF_NAMES = ["fourier_f64", "zgemm", "eigh", "rotation", "rr_rotation", "umma_h", "umma_kq", "umma_rr",
                  "split", "other", "eigh_refine", "tridiag", "mlp_train", "mlp_infer", "pairs"]

    def profile(self, on=True):
        check(lib().epb_profile_enable(self.h, 1 if on else 0))

    def profile_read(self, reset=True):
        import numpy as np

        n = len(self.PROF_NAMES)
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int64)
        check(lib().epb_profile_read(self.h, ms.ctypes.data, cnt.ctypes.data, n, 1 if reset else 0))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.PROF_NAMES)}

    def close(self):
        if getattr(self, "h", None):
            lib().epb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RSet:
    """Device copy of an R-vector list (epb_rset)."""

    def __init__(self, ctx: Context, irvec):
        import numpy as np

        self.ctx = ctx
        self.irvec = np.ascontiguousarray(np.asarray(irvec, dtype=np.int64).reshape(-1, 3))
        h = P()
        check(lib().epb_rset_create(ctx.h, self.irvec.ctypes.data, self.irvec.shape[0], C.byref(h)))
        self.h = h
        self.nr = self.irvec.shape[0]

    def close(self):
        if getattr(self, "h", None):
            lib().epb_rset_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = {}


class TuneTable:
    """The autotuner's choices as a host table (epb_tune_table_*): set / get / text round trip; export
    from and import into a context."""

    def __init__(self, text=None):
        h = C.c_void_p()
        check(lib().epb_tune_table_create(C.byref(h)))
        self.h = h
        if text is not None:
            self.parse(text)

    def __del__(self):
        if getattr(self, "h", None):
            lib().epb_tune_table_destroy(self.h)
            self.h = None

    def set(self, key, value):
        check(lib().epb_tune_table_set(self.h, key.encode(), int(value)))

    def get(self, key):
        v, f = I64(0), I32(0)
        check(lib().epb_tune_table_get(self.h, key.encode(), C.byref(v), C.byref(f)))
        return int(v.value) if f.value else None

    def __len__(self):
        n = I64(0)
        check(lib().epb_tune_table_size(self.h, C.byref(n)))
        return int(n.value)

    def text(self):
        n = I64(0)
        st = lib().epb_tune_table_serialize(self.h, None, 0, C.byref(n))
        if st not in (EPB_OK, EPB_ERR_ARG):
            check(st)
        buf = C.create_string_buffer(int(n.value) + 1)
        check(lib().epb_tune_table_serialize(self.h, buf, int(n.value) + 1, C.byref(n)))
        return buf.value.decode()

    def parse(self, text):
        check(lib().epb_tune_table_parse(self.h, text.encode()))

    def export_from(self, ctx):
        check(lib().epb_tune_export(ctx.h, self.h))

    def import_into(self, ctx):
        check(lib().epb_tune_import(ctx.h, self.h))


def default_context(device=None):
    import torch

    if device is None:
        device = torch.cuda.current_device()
    c = _default_ctx.get(device)
    stream = torch.cuda.current_stream(device)
    if c is None:
        c = Context(device, stream)
        _default_ctx[device] = c
    elif c.stream.cuda_stream != stream.cuda_stream:
        c.set_stream(stream)
    return c
