"""ctypes binding of the engine's C ABI (include/bw_engine.h).

The CUDA library ``libbw_b200.so`` is built in-tree by ``build.build()``.
There is no CPU fallback: every entry point here calls the CUDA library and
raises ``EngineError`` with the library's message on a nonzero status.

Device buffers are torch tensors (int32 storage of canonical residues; every
residue is below 2^15, so the int32 and uint32 bit patterns agree).  Host
buffers are numpy uint32 arrays.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libbw_b200.so"

FORM_PLAIN = 0
FORM_INT8 = 1
FORMS = {"plain": FORM_PLAIN, "int8": FORM_INT8}

_LIB = None


class EngineError(RuntimeError):
    """A nonzero status from the engine's C ABI."""

    def __init__(self, status, message):
        super().__init__(f"[status {status}] {message}")
        self.status = status


class KoszulDesc(ctypes.Structure):
    _fields_ = [
        ("r", ctypes.c_uint32), ("k", ctypes.c_uint32), ("dim_in", ctypes.c_uint32),
        ("dim_out", ctypes.c_uint32), ("prime", ctypes.c_uint32), ("block_width", ctypes.c_uint32),
        ("proj_width", ctypes.c_uint32), ("form", ctypes.c_uint32),
        ("maps", ctypes.c_void_p), ("diag", ctypes.c_void_p), ("diag_on_device", ctypes.c_uint32),
    ]


class KoszulInfo(ctypes.Structure):
    _fields_ = [
        ("n_src", ctypes.c_uint64), ("n_tgt", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64),
        ("scratch_bytes", ctypes.c_uint64), ("form", ctypes.c_uint32), ("sm_count", ctypes.c_uint32),
    ]


# Every symbol the header declares, with (restype, argtypes).
_VP, _U32, _U64, _INT = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
SIGNATURES = {
    "bw_last_error": (ctypes.c_char_p, []),
    "bw_abi_version": (_INT, []),
    "bw_seeded_fill": (_INT, [_VP, _U64, _U64, _U32, _U32, _U32, _INT, _VP]),
    "bw_seeded_fill_host": (_INT, [_VP, _U64, _U64, _U32, _U32, _U32]),
    "bw_koszul_create": (_INT, [ctypes.POINTER(KoszulDesc), _INT, ctypes.POINTER(_VP)]),
    "bw_koszul_info_get": (_INT, [_VP, ctypes.POINTER(KoszulInfo)]),
    "bw_koszul_destroy": (None, [_VP]),
    "bw_koszul_forward": (_INT, [_VP, _VP, _VP, _VP]),
    "bw_koszul_transpose": (_INT, [_VP, _VP, _VP, _INT, _VP]),
    "bw_koszul_apply": (_INT, [_VP, _VP, _VP, _VP]),
    "bw_koszul_seq_start": (_INT, [_VP, _VP, _VP, _VP, _U64, _VP]),
    "bw_koszul_seq_step": (_INT, [_VP, _U64, _VP]),
    "bw_koszul_seq_finish": (_INT, [_VP, _VP, ctypes.POINTER(_U64), _VP]),
    "bw_koszul_sequence_host": (_INT, [_VP, _VP, _VP, _U64, _VP, _VP]),
    "bw_koszul_seq_step_timed": (_INT, [_VP, _U64, ctypes.POINTER(ctypes.c_float), _VP]),
    "bw_koszul_launch_count": (_U64, [_VP]),
    "bw_koszul_plan": (_INT, [_VP, ctypes.c_char_p, ctypes.c_size_t]),
    "bw_koszul_batch_create": (_INT, [_VP, _U32, _INT, ctypes.POINTER(_VP)]),
    "bw_koszul_batch_destroy": (None, [_VP]),
    "bw_koszul_batch_sector": (_INT, [_VP, _U32, ctypes.POINTER(_VP)]),
    "bw_koszul_batch_seq_start": (_INT, [_VP, _VP, _VP, _VP, _U64, _VP]),
    "bw_koszul_batch_seq_step": (_INT, [_VP, _U64, _VP]),
    "bw_koszul_batch_seq_finish": (_INT, [_VP, _VP, ctypes.POINTER(_U64), _VP]),
    "bw_koszul_batch_launch_count": (_U64, [_VP]),
    "bw_cyclic_open": (_INT, [ctypes.c_char_p, ctypes.c_char_p, _U32, _U32, _U64, _U32, _U64, ctypes.c_char_p,
                              ctypes.c_char_p, _INT, ctypes.POINTER(_VP)]),
    "bw_cyclic_info_get": (_INT, [_VP, _VP]),
    "bw_cyclic_close": (None, [_VP]),
    "bw_cyclic_apply_host": (_INT, [_VP, _INT, _VP, _VP]),
    "bw_cyclic_generate": (_INT, [_VP, _U64]),
    "bw_cyclic_generate_timed": (_INT, [_VP, _U64, ctypes.POINTER(ctypes.c_float)]),
    "bw_cyclic_download": (_INT, [_VP, _VP, _U64, _VP]),
    "bw_cyclic_output_path": (_INT, [_VP, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]),
    "bw_cyclic_check_outputs_absent": (_INT, [ctypes.c_char_p]),
    "bw_cyclic_write_sidecar": (_INT, [_VP, ctypes.c_char_p]),
    "bw_cyclic_write_wdm": (_INT, [_VP, ctypes.c_char_p]),
    "bw_cyclic_validate": (_INT, [_VP, _U32]),
    "bw_cyclic_launch_count": (_U64, [_VP]),
    "bw_cyclic_gather_path": (_INT, [_VP, ctypes.c_char_p, ctypes.c_size_t]),
    "bw_file_read_text": (_INT, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "bw_project_noalloc": (_INT, [_VP, _VP, _U64, _U32, _U32, _U32, _VP, _INT, _VP]),
    "bw_cyclic_recover": (_INT, [ctypes.c_char_p, ctypes.c_char_p, _U32, ctypes.c_char_p, ctypes.c_char_p,
                                 ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                 ctypes.c_char_p, ctypes.c_int64, _U64, _INT, _INT, _INT, _INT]),
}


class CyclicInfo(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "rows", "cols", "x_cols", "z_cols", "t_rows", "y_rows", "dm_nnz", "d2_nnz", "default_nlen", "seq_len",
        "rowmix_realized_seed", "rowmix_hash", "device_bytes")] + [
        (name, ctypes.c_uint32) for name in ("genus", "prime", "order", "sector", "y_sector", "num_v")]


APPLY_SQUARE, APPLY_FORWARD, APPLY_TRANSPOSE, APPLY_SQUARE_UNFOLDED = 0, 1, 2, 3


def load():
    """Load libbw_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise EngineError(-1, f"{LIB_PATH} is missing: run prym_green_ancillary_b200.build.build()")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _check(status):
    if status != 0:
        msg = load().bw_last_error()
        raise EngineError(status, msg.decode() if msg else "")


def _host_ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"], "host buffers must be C-contiguous uint32"
    return ctypes.c_void_p(a.ctypes.data)


def _dev_ptr(t):
    import torch
    assert t.is_cuda and t.dtype in (torch.int32, torch.uint32) and t.is_contiguous()
    return ctypes.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        return None
    return ctypes.c_void_p(stream.cuda_stream)


def seeded_fill_host(count, seed, tag, p, lo=0):
    out = np.empty(count, dtype=np.uint32)
    _check(load().bw_seeded_fill_host(_host_ptr(out), count, seed, tag, p, lo))
    return out


def seeded_fill_device(out, seed, tag, p, lo=0, stream=None):
    """Fill a CUDA int32 tensor with the seeded stream (seed, tag) on [lo, p)."""
    _check(load().bw_seeded_fill(_dev_ptr(out), out.numel(), seed, tag, p, lo,
                                 out.device.index or 0, _stream_ptr(stream)))
    return out


def _koszul_desc(r, k, dim_in, dim_out, prime, block_width, proj_width, form, maps, diag):
    """bw_koszul_desc for the arguments, and the arrays it points into (keep them alive)."""
    maps = np.ascontiguousarray(maps, dtype=np.uint32).reshape(-1)
    desc = KoszulDesc(r, k, dim_in, dim_out, prime, block_width, proj_width, FORMS[form], maps.ctypes.data, 0, 0)
    if isinstance(diag, np.ndarray):
        diag = np.ascontiguousarray(diag, dtype=np.uint32)
        desc.diag = diag.ctypes.data
    else:
        desc.diag = diag.data_ptr()
        desc.diag_on_device = 1
    return desc, (maps, diag)


class KoszulEngine:
    """Synthetic Koszul operator S = D d^T d on one GPU (see include/bw_engine.h).

    ``maps`` is an (r, dim_out, dim_in) uint32 array; ``diag`` is either a
    host uint32 array or a CUDA int32 tensor of length n_src.
    """

    def __init__(self, r, k, dim_in, dim_out, prime, block_width, proj_width=None,
                 maps=None, diag=None, form="plain", device=0):
        lib = load()
        self.r, self.k, self.dim_in, self.dim_out, self.p = r, k, dim_in, dim_out, prime
        self.nb = block_width
        self.m = block_width if proj_width is None else proj_width
        self.form = form
        self.device = device
        desc, self._keep = _koszul_desc(r, k, dim_in, dim_out, prime, self.nb, self.m, form, maps, diag)
        handle = ctypes.c_void_p()
        _check(lib.bw_koszul_create(ctypes.byref(desc), device, ctypes.byref(handle)))
        self._h = handle
        self._read_info()

    @classmethod
    def _borrowed(cls, handle, r, k, dim_in, dim_out, prime, block_width, proj_width, form, device):
        """A view of a batch sector (the batch owns the context)."""
        eng = cls.__new__(cls)
        eng.r, eng.k, eng.dim_in, eng.dim_out, eng.p = r, k, dim_in, dim_out, prime
        eng.nb, eng.m, eng.form, eng.device = block_width, proj_width, form, device
        eng._h, eng._owned = handle, False
        eng._read_info()
        return eng

    def _read_info(self):
        info = KoszulInfo()
        _check(load().bw_koszul_info_get(self._h, ctypes.byref(info)))
        self.n_src, self.n_tgt = int(info.n_src), int(info.n_tgt)
        self.device_bytes, self.scratch_bytes = int(info.device_bytes), int(info.scratch_bytes)
        self.sm_count = int(info.sm_count)

    def close(self):
        if getattr(self, "_h", None) and getattr(self, "_owned", True):
            load().bw_koszul_destroy(self._h)
        self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- device-buffer API -------------------------------------------------
    def forward(self, y, z, stream=None):
        _check(load().bw_koszul_forward(self._h, _dev_ptr(y), _dev_ptr(z), _stream_ptr(stream)))

    def transpose(self, z, w, scale_by_diag=True, stream=None):
        _check(load().bw_koszul_transpose(self._h, _dev_ptr(z), _dev_ptr(w), int(scale_by_diag),
                                          _stream_ptr(stream)))

    def apply(self, y, out, stream=None):
        _check(load().bw_koszul_apply(self._h, _dev_ptr(y), _dev_ptr(out), _stream_ptr(stream)))

    def seq_start(self, x, y0, seq, stream=None):
        cap = seq.numel() // (self.m * self.nb)
        _check(load().bw_koszul_seq_start(self._h, _dev_ptr(x), _dev_ptr(y0), _dev_ptr(seq), cap,
                                          _stream_ptr(stream)))

    def seq_step(self, steps, stream=None):
        _check(load().bw_koszul_seq_step(self._h, steps, _stream_ptr(stream)))

    def seq_finish(self, y_out=None, stream=None):
        n = ctypes.c_uint64()
        _check(load().bw_koszul_seq_finish(self._h, _dev_ptr(y_out) if y_out is not None else None,
                                           ctypes.byref(n), _stream_ptr(stream)))
        return int(n.value)

    def seq_step_timed(self, steps, stream=None):
        """Steps with per-kernel CUDA events; returns average ms (forward, transpose, project)."""
        ms = (ctypes.c_float * 3)()
        _check(load().bw_koszul_seq_step_timed(self._h, steps, ms, _stream_ptr(stream)))
        return tuple(float(v) for v in ms)

    # -- host-buffer API ---------------------------------------------------
    def sequence_host(self, X, Y0, nlen, want_final=True, out=None):
        """Sequence of nlen entries through host buffers (bw_koszul_sequence_host).

        ``out`` = (seq, final) lets the caller supply the output arrays (for
        example views of pinned host memory, which the copies back reach
        directly); by default they are allocated here.
        """
        X = np.ascontiguousarray(X, dtype=np.uint32)
        Y0 = np.ascontiguousarray(Y0, dtype=np.uint32)
        if out is not None:
            seq, yf = out
            assert seq.dtype == np.uint32 and seq.shape == (nlen, self.m, self.nb) and seq.flags.c_contiguous
            if want_final:
                assert yf.dtype == np.uint32 and yf.shape == (self.n_src, self.nb) and yf.flags.c_contiguous
            else:
                yf = None
        else:
            seq = np.empty((nlen, self.m, self.nb), dtype=np.uint32)
            yf = np.empty((self.n_src, self.nb), dtype=np.uint32) if want_final else None
        _check(load().bw_koszul_sequence_host(self._h, _host_ptr(X), _host_ptr(Y0), nlen, _host_ptr(seq),
                                              _host_ptr(yf) if yf is not None else None))
        return seq, yf

    @property
    def launch_count(self):
        return int(load().bw_koszul_launch_count(self._h))

    @property
    def plan(self):
        """The kernel plan and the set-up autotuner's timings (bw_koszul_plan)."""
        buf = ctypes.create_string_buffer(4096)
        _check(load().bw_koszul_plan(self._h, buf, len(buf)))
        return buf.value.decode()


class KoszulBatch:
    """Sectors of uneven shapes advanced together (bw_koszul_batch_*).

    ``sectors`` is a list of dicts with the KoszulEngine arguments (r, k,
    dim_in, dim_out, prime, block_width, proj_width, maps, diag, form).
    """

    def __init__(self, sectors, device=0):
        lib = load()
        descs = (KoszulDesc * len(sectors))()
        self._keep = []
        for i, sec in enumerate(sectors):
            sec = dict(sec)
            sec.setdefault("proj_width", sec["block_width"])
            sec.setdefault("form", "int8")
            d, keep = _koszul_desc(sec["r"], sec["k"], sec["dim_in"], sec["dim_out"], sec["prime"],
                                   sec["block_width"], sec["proj_width"], sec["form"], sec["maps"], sec["diag"])
            descs[i] = d
            self._keep.append(keep)
        handle = ctypes.c_void_p()
        _check(lib.bw_koszul_batch_create(descs, len(sectors), device, ctypes.byref(handle)))
        self._h = handle
        self.engines = []
        for i, sec in enumerate(sectors):
            h = ctypes.c_void_p()
            _check(lib.bw_koszul_batch_sector(self._h, i, ctypes.byref(h)))
            self.engines.append(KoszulEngine._borrowed(
                h, sec["r"], sec["k"], sec["dim_in"], sec["dim_out"], sec["prime"], sec["block_width"],
                sec.get("proj_width", sec["block_width"]), sec.get("form", "int8"), device))

    def close(self):
        if getattr(self, "_h", None):
            for e in self.engines:
                e._h = None
            load().bw_koszul_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _ptrs(tensors):
        return (ctypes.c_void_p * len(tensors))(*[t.data_ptr() if t is not None else None for t in tensors])

    def seq_start(self, xs, ys, seqs, stream=None):
        cap = min(s.numel() // (e.m * e.nb) for s, e in zip(seqs, self.engines))
        self._arrays = (self._ptrs(xs), self._ptrs(ys), self._ptrs(seqs))
        _check(load().bw_koszul_batch_seq_start(self._h, *self._arrays, cap, _stream_ptr(stream)))

    def seq_step(self, steps, stream=None):
        _check(load().bw_koszul_batch_seq_step(self._h, steps, _stream_ptr(stream)))

    def seq_finish(self, y_outs=None, stream=None):
        n = ctypes.c_uint64()
        ptrs = self._ptrs(y_outs) if y_outs is not None else None
        _check(load().bw_koszul_batch_seq_finish(self._h, ptrs, ctypes.byref(n), _stream_ptr(stream)))
        return int(n.value)

    @property
    def launch_count(self):
        return int(load().bw_koszul_batch_launch_count(self._h))


def read_text(path):
    """A text file, decompressed when it carries the zstd magic (the WDM reader's framing)."""
    lib = load()
    n = ctypes.c_size_t()
    _check(lib.bw_file_read_text(str(path).encode(), None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(max(1, n.value))
    _check(lib.bw_file_read_text(str(path).encode(), buf, n.value, ctypes.byref(n)))
    return buf.raw[:n.value].decode()


class CyclicEngine:
    """Paper-mode operator of one sector (include/bw_engine.h): the eliminated
    cyclic operator, or with ``op="augmented"`` / ``"replacement"`` its
    deformation variants (``dense_file``, and ``drop_columns`` for replacement).

    ``device=-1`` opens a host-only context (assembly, seeded data, row-mixing
    plan and sidecar; no device calls).
    """

    def __init__(self, instance, sector, op="eliminated", num_v=4, seed=1, rowmix_rounds=2, rowmix_seed=10001,
                 device=0, dense_file=None, drop_columns=None):
        lib = load()
        handle = ctypes.c_void_p()
        _check(lib.bw_cyclic_open(str(instance).encode(), op.encode(), sector, num_v, seed, rowmix_rounds,
                                  rowmix_seed, str(dense_file).encode() if dense_file else None,
                                  str(drop_columns).encode() if drop_columns else None, device,
                                  ctypes.byref(handle)))
        self._h = handle
        self.refresh()

    def refresh(self):
        info = CyclicInfo()
        _check(load().bw_cyclic_info_get(self._h, ctypes.byref(info)))
        self.info = {name: getattr(info, name) for name, _ in CyclicInfo._fields_}
        return self.info

    def close(self):
        if getattr(self, "_h", None):
            load().bw_cyclic_close(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def apply(self, what, block):
        block = np.ascontiguousarray(block, dtype=np.uint32)
        rows = self.info["rows"] if what == APPLY_FORWARD else self.info["cols"]
        out = np.empty((rows, 4), dtype=np.uint32)
        _check(load().bw_cyclic_apply_host(self._h, what, _host_ptr(block), _host_ptr(out)))
        return out

    def generate(self, nlen=0):
        _check(load().bw_cyclic_generate(self._h, nlen))
        return self.refresh()["seq_len"]

    def generate_timed(self, nlen=0):
        """generate() plus the device time of its rounds in ms (CUDA events on the engine's stream)."""
        ms = ctypes.c_float()
        _check(load().bw_cyclic_generate_timed(self._h, nlen, ctypes.byref(ms)))
        self.refresh()
        return float(ms.value)

    def download(self):
        n = self.info["seq_len"]
        seq = np.empty((n, 10), dtype=np.uint32)
        cur = np.empty((self.info["cols"], 4), dtype=np.uint32)
        _check(load().bw_cyclic_download(self._h, _host_ptr(seq), n, _host_ptr(cur)))
        return seq, cur

    def output_path(self, out_dir):
        buf = ctypes.create_string_buffer(4096)
        _check(load().bw_cyclic_output_path(self._h, str(out_dir).encode(), buf, 4096))
        return buf.value.decode()

    def write_sidecar(self, wdm_path):
        _check(load().bw_cyclic_write_sidecar(self._h, str(wdm_path).encode()))

    def write_wdm(self, wdm_path):
        _check(load().bw_cyclic_write_wdm(self._h, str(wdm_path).encode()))

    def validate(self, columns=4):
        _check(load().bw_cyclic_validate(self._h, columns))

    @property
    def launch_count(self):
        return int(load().bw_cyclic_launch_count(self._h))

    @property
    def gather_path(self):
        """"subset: tables cached", "subset: tables evict-first" or "generic: <reason>"
        (bw_cyclic_gather_path)."""
        buf = ctypes.create_string_buffer(256)
        _check(load().bw_cyclic_gather_path(self._h, buf, len(buf)))
        return buf.value.decode()
