"""ctypes bindings of libsjcs.so (GPU, include/sjcs.h) and libsjcs_host.so (CPU, include/sjcs_host.h)."""
from __future__ import annotations

import ctypes
import os
import pathlib
import threading

import numpy as np

_PKG = pathlib.Path(__file__).resolve().parent
lib_path = _PKG / "lib" / "libsjcs.so"
host_lib_path = _PKG / "lib" / "libsjcs_host.so"

INDEX_GRID = 0
INDEX_LEARNED = 1
INDEX_MORTON = 2
INDEX_VERIFY = 0x1
QUERY_NONPERIODIC = 0
QUERY_PERIODIC = 1
SCHED_AUTO = 0
SCHED_STATIC = 1
SCHED_QUEUE = 2

# The reference's Halo struct (include/Gadget/BufHalo.h:26-30), 24 bytes.
HALO_DTYPE = np.dtype([("id", "<u8"), ("mass", "<f4"), ("point", "<f4", (3,))], align=False)
assert HALO_DTYPE.itemsize == 24

_c = ctypes
_vp = _c.c_void_p
_u64 = _c.c_uint64
_pp = _c.POINTER(_c.c_void_p)


class SjcsError(RuntimeError):
    """A libsjcs / libsjcs_host call failed (code, message)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code
        self.msg = msg


class sjcs_index_opts(_c.Structure):
    _fields_ = [("kind", _c.c_int), ("radius_hint", _c.c_float), ("grid", _c.c_uint32 * 3),
                ("flags", _c.c_uint32), ("reserved", _c.c_uint32 * 3)]


class sjcs_learned_info(_c.Structure):
    _fields_ = [("level", _c.c_uint32), ("leaves", _c.c_uint32), ("nonempty", _c.c_uint32),
                ("max_err", _c.c_uint32), ("mean_err", _c.c_double), ("checked", _c.c_uint64),
                ("mismatches", _c.c_uint64), ("sort_ms", _c.c_float), ("train_ms", _c.c_float)]


class sjcs_schedule(_c.Structure):
    _fields_ = [("mode", _c.c_int), ("piece", _c.c_uint32), ("max_pieces", _c.c_uint32), ("single", _c.c_uint32)]


class sjcs_server_opts(_c.Structure):
    _fields_ = [("slots", _c.c_uint32), ("pad_", _c.c_uint32), ("mem_budget", _c.c_uint64),
                ("reserved", _c.c_uint32 * 4)]


class sjcs_request_info(_c.Structure):
    _fields_ = [("queue_ms", _c.c_double), ("service_ms", _c.c_double), ("latency_ms", _c.c_double),
                ("status", _c.c_int)]


class sjcs_server_info(_c.Structure):
    _fields_ = [("submitted", _c.c_uint64), ("completed", _c.c_uint64), ("queued", _c.c_uint64),
                ("inflight", _c.c_uint32), ("max_inflight", _c.c_uint32), ("slots", _c.c_uint32),
                ("pad_", _c.c_uint32), ("budget_bytes", _c.c_uint64), ("in_use_bytes", _c.c_uint64),
                ("peak_bytes", _c.c_uint64)]


class sjcs_timing(_c.Structure):
    _fields_ = [("h2d_ms", _c.c_float), ("build_ms", _c.c_float), ("count_ms", _c.c_float),
                ("d2h_ms", _c.c_float), ("count_calls", _c.c_uint32)]


_lock = threading.Lock()
_lib = None
_host = None

# name -> (restype, argtypes); every function declared in include/sjcs.h
_SIGS = {
    "sjcs_last_error": (_c.c_char_p, []),
    "sjcs_version": (_c.c_char_p, []),
    "sjcs_ctx_create": (_c.c_int, [_c.c_int, _pp]),
    "sjcs_ctx_destroy": (_c.c_int, [_vp]),
    "sjcs_ctx_sync": (_c.c_int, [_vp]),
    "sjcs_ctx_num_sms": (_c.c_int, [_vp, _c.POINTER(_c.c_int)]),
    "sjcs_ctx_stream": (_c.c_int, [_vp, _c.c_int, _pp]),
    "sjcs_ctx_reserve": (_c.c_int, [_vp, _u64]),
    "sjcs_ctx_trim": (_c.c_int, [_vp]),
    "sjcs_ctx_memory": (_c.c_int, [_vp, _c.POINTER(_u64), _c.POINTER(_u64)]),
    "sjcs_launch_counter": (_c.c_uint64, []),
    "sjcs_ctx_set_overlap": (_c.c_int, [_vp, _c.c_int]),
    "sjcs_host_alloc": (_c.c_int, [_c.c_size_t, _pp]),
    "sjcs_host_free": (_c.c_int, [_vp]),
    "sjcs_index_build": (_c.c_int, [_vp, _vp, _u64, _c.POINTER(sjcs_index_opts), _pp]),
    "sjcs_index_build_device": (_c.c_int, [_vp, _vp, _u64, _c.POINTER(sjcs_index_opts), _pp]),
    "sjcs_index_wait": (_c.c_int, [_vp]),
    "sjcs_index_size": (_c.c_int, [_vp, _c.POINTER(_u64)]),
    "sjcs_index_grid": (_c.c_int, [_vp, _c.POINTER(_c.c_uint32)]),
    "sjcs_index_learned_info": (_c.c_int, [_vp, _c.POINTER(sjcs_learned_info)]),
    "sjcs_index_build_compressed": (_c.c_int, [_vp, _vp, _u64, _vp, _c.POINTER(sjcs_index_opts), _pp]),
    "sjcs_decode_compressed": (_c.c_int, [_vp, _vp, _u64, _vp, _vp]),
    "sjcs_step_create": (_c.c_int, [_vp, _vp, _vp, _u64, _c.POINTER(sjcs_index_opts), _pp]),
    "sjcs_step_launch": (_c.c_int, [_vp, _vp]),
    "sjcs_step_wait": (_c.c_int, [_vp]),
    "sjcs_step_time": (_c.c_int, [_vp, _c.POINTER(_c.c_float)]),
    "sjcs_step_destroy": (_c.c_int, [_vp]),
    "sjcs_server_create": (_c.c_int, [_vp, _c.POINTER(_vp), _c.c_int, _c.POINTER(sjcs_server_opts), _pp]),
    "sjcs_server_submit": (_c.c_int, [_vp, _vp, _c.c_size_t, _u64, _vp, _c.c_int, _c.c_int, _vp,
                                      _c.POINTER(_u64)]),
    "sjcs_server_wait": (_c.c_int, [_vp, _u64, _c.POINTER(sjcs_request_info)]),
    "sjcs_server_stats": (_c.c_int, [_vp, _c.POINTER(sjcs_server_info)]),
    "sjcs_server_destroy": (_c.c_int, [_vp]),
    "sjcs_query_set_schedule": (_c.c_int, [_vp, _vp, _c.POINTER(sjcs_schedule)]),
    "sjcs_query_get_schedule": (_c.c_int, [_vp, _c.POINTER(sjcs_schedule)]),
    "sjcs_autotune": (_c.c_int, [_vp, _vp, _vp, _c.POINTER(sjcs_schedule), _c.POINTER(_c.c_float), _c.c_int,
                                 _c.POINTER(_c.c_int)]),
    "sjcs_index_timing": (_c.c_int, [_vp, _c.POINTER(sjcs_timing)]),
    "sjcs_index_destroy": (_c.c_int, [_vp]),
    "sjcs_query_create": (_c.c_int, [_vp, _vp, _c.c_size_t, _u64, _vp, _c.c_int, _c.c_int, _pp]),
    "sjcs_query_create_device": (_c.c_int, [_vp, _vp, _c.c_size_t, _u64, _vp, _c.c_int, _c.c_int, _pp]),
    "sjcs_query_count": (_c.c_int, [_vp, _vp, _vp]),
    "sjcs_query_count_many": (_c.c_int, [_vp, _vp, _vp, _c.c_int]),
    "sjcs_query_wait": (_c.c_int, [_vp]),
    "sjcs_index_build_file": (_c.c_int, [_vp, _c.c_char_p, _c.POINTER(sjcs_index_opts), _pp]),
    "sjcs_ctx_prepare_files": (_c.c_int, [_vp, _u64]),
    "sjcs_query_read_counts": (_c.c_int, [_vp, _vp, _vp, _c.c_int]),
    "sjcs_query_read_counts_async": (_c.c_int, [_vp, _vp, _vp]),
    "sjcs_query_read_counts32_async": (_c.c_int, [_vp, _vp, _vp]),
    "sjcs_query_wait_read": (_c.c_int, [_vp]),
    "sjcs_query_device_counts": (_c.c_int, [_vp, _pp]),
    "sjcs_query_set_fold_limit": (_c.c_int, [_vp, _vp, _u64]),
    "sjcs_query_folds": (_c.c_int, [_vp, _c.POINTER(_c.c_uint32)]),
    "sjcs_query_reset": (_c.c_int, [_vp, _vp]),
    "sjcs_query_timing": (_c.c_int, [_vp, _c.POINTER(sjcs_timing)]),
    "sjcs_query_destroy": (_c.c_int, [_vp]),
    "sjcs_multi_range_count": (_c.c_int, [_vp, _vp, _vp, _c.c_size_t, _u64, _vp, _c.c_int, _c.c_int, _vp]),
    "sjcs_radius_table": (_c.c_int, [_c.c_double, _c.c_double, _c.c_int, _vp]),
    "sjcs_count_noalloc": (_c.c_int, [_vp, _u64, _vp, _c.c_size_t, _u64, _vp, _c.c_int, _c.c_int, _vp, _vp]),
}

_HOST_SIGS = {
    "sjcs_particle_file_count": (_c.c_int, [_c.c_char_p, _c.POINTER(_u64)]),
    "sjcs_read_particles": (_c.c_int, [_c.c_char_p, _vp, _u64, _c.POINTER(_u64)]),
    "sjcs_read_halos": (_c.c_int, [_c.c_char_p, _pp, _c.POINTER(_u64), _c.c_int]),
    "sjcs_read_and_filter_halos": (_c.c_int, [_c.c_char_p, _c.c_char_p, _pp, _c.POINTER(_u64)]),
    "sjcs_host_free_halos": (None, [_vp]),
    "sjcs_host_last_error": (_c.c_char_p, []),
    "sjcs_write_result": (_c.c_int, [_c.c_char_p, _vp, _u64, _vp, _c.c_int, _vp, _c.c_int]),
    "sjcs_host_radius_table": (_c.c_int, [_c.c_double, _c.c_double, _c.c_int, _vp]),
    "sjcs_mt_seed": (None, [_vp, _c.c_uint32]),
    "sjcs_mt_u32": (_c.c_uint32, [_vp]),
    "sjcs_mt_real1": (_c.c_double, [_vp]),
    "sjcs_gen_uniform_particles": (_c.c_int, [_c.c_uint32, _u64, _u64, _vp]),
    "sjcs_gen_uniform_halo_file": (_c.c_int, [_c.c_char_p, _c.c_uint32, _u64, _u64]),
    "sjcs_gen_uniform_halos": (_c.c_int, [_c.c_uint32, _u64, _u64, _vp, _c.c_int]),
    "sjcs_gen_face_halos": (_c.c_int, [_c.c_uint32, _u64, _u64, _c.c_float, _vp]),
    "sjcs_gen_clustered_particles": (_c.c_int, [_c.c_uint32, _u64, _c.c_uint32, _c.c_double, _c.c_double,
                                                 _c.c_double, _c.c_double, _c.c_uint32, _vp]),
    "sjcs_gen_clustered_halos": (_c.c_int, [_c.c_uint32, _u64, _u64, _c.c_uint32, _c.c_double, _c.c_double,
                                             _c.c_double, _c.c_double, _c.c_double, _c.c_uint32, _vp]),
    "sjcs_write_halo_file": (_c.c_int, [_c.c_char_p, _vp, _u64]),
    "sjcs_write_particle_file": (_c.c_int, [_c.c_char_p, _vp, _u64]),
    "sjcs_read_compressed_header": (_c.c_int, [_c.c_char_p, _vp]),
    "sjcs_read_compressed_particles": (_c.c_int, [_c.c_char_p, _vp, _vp, _u64, _c.POINTER(_u64)]),
    "sjcs_write_compressed_file": (_c.c_int, [_c.c_char_p, _vp, _vp, _u64]),
    "sjcs_gen_compressed": (_c.c_int, [_c.c_uint32, _c.c_int, _c.c_double, _c.c_float, _c.c_float, _c.c_int,
                                       _c.c_longlong, _u64, _vp, _vp]),
}


def _bind(handle, sigs):
    for name, (res, args) in sigs.items():
        f = getattr(handle, name)
        f.restype = res
        f.argtypes = args
    return handle


def lib():
    """libsjcs.so (GPU path).  Raises if it has not been built: there is no CPU fallback."""
    global _lib
    with _lock:
        if _lib is None:
            if not lib_path.exists():
                raise SjcsError(2, f"{lib_path} is missing; build it with "
                                   "`python -m spatialjoincountovershells_b200.build`")
            _lib = _bind(ctypes.CDLL(str(lib_path)), _SIGS)
        return _lib


def host_lib():
    global _host
    with _lock:
        if _host is None:
            if not host_lib_path.exists():
                raise SjcsError(2, f"{host_lib_path} is missing; build it with "
                                   "`python -m spatialjoincountovershells_b200.build`")
            _host = _bind(ctypes.CDLL(str(host_lib_path)), _HOST_SIGS)
        return _host


def _check(rc: int) -> None:
    if rc != 0:
        raise SjcsError(rc, lib().sjcs_last_error().decode(errors="replace"))


def _hcheck(rc: int) -> None:
    if rc != 0:
        raise SjcsError(rc, host_lib().sjcs_host_last_error().decode(errors="replace"))


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)


def _is_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _hand_over(ctx: "Context", which: int, t, call) -> None:
    """Run `call` (a library call that reads tensor t on the context's stream
    `which`: 0 build, 1 count) ordered after the work queued on torch's
    current stream (t's producer), and order torch's later work -- including
    the reuse of t's memory once it is freed -- after the library's reads."""
    import torch
    lib_s = torch.cuda.ExternalStream(ctx.stream(which), device=t.device)
    torch_s = torch.cuda.current_stream(t.device)
    lib_s.wait_stream(torch_s)
    call()
    torch_s.wait_stream(lib_s)


def _as_f32_xyz(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] != 3:
        a = a.reshape(-1, 3)
    return a


# ---------------------------------------------------------------------------
# GPU objects
# ---------------------------------------------------------------------------

class Context:
    """One GPU (sjcs_ctx): a build stream and a count stream."""

    def __init__(self, device: int = 0):
        h = _vp()
        _check(lib().sjcs_ctx_create(int(device), _c.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def num_sms(self) -> int:
        v = _c.c_int()
        _check(lib().sjcs_ctx_num_sms(self._h, _c.byref(v)))
        return v.value

    def sync(self) -> None:
        _check(lib().sjcs_ctx_sync(self._h))

    def reserve(self, nbytes: int) -> None:
        """Grow the device memory pool to hold at least nbytes (no new driver allocations later)."""
        _check(lib().sjcs_ctx_reserve(self._h, int(nbytes)))

    def trim(self) -> None:
        """Return the pool's unused memory to the driver."""
        _check(lib().sjcs_ctx_trim(self._h))

    def memory(self) -> dict:
        f, p = _u64(), _u64()
        _check(lib().sjcs_ctx_memory(self._h, _c.byref(f), _c.byref(p)))
        return {"free_bytes": f.value, "pool_bytes": p.value}

    def stream(self, which: int) -> int:
        """cudaStream_t of the build (0) or count (1) stream, as an integer."""
        p = _vp()
        _check(lib().sjcs_ctx_stream(self._h, int(which), _c.byref(p)))
        return p.value or 0

    def close(self) -> None:
        if self._h:
            _check(lib().sjcs_ctx_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def build_index(self, xyz, radius_hint: float = 0.0, grid=None, kind: int = INDEX_GRID,
                    level: int = 0, verify: bool = False) -> "Index":
        """Index over particles: host array (n,3) float32, or a CUDA tensor (device path).
        kind: INDEX_GRID (grid = cells per axis), INDEX_MORTON or INDEX_LEARNED (level =
        Morton cell level, 0 = automatic; verify = judge the model against the table)."""
        opts = _make_opts(radius_hint, grid, kind, level, verify)
        h = _vp()
        if _is_cuda(xyz):
            n = xyz.numel() // 3
            _hand_over(self, 0, xyz, lambda: _check(lib().sjcs_index_build_device(
                self._h, _vp(xyz.data_ptr()), n, _c.byref(opts), _c.byref(h))))
            keep = xyz
        else:
            arr = _as_f32_xyz(xyz)
            n = arr.shape[0]
            _check(lib().sjcs_index_build(self._h, _vp(arr.ctypes.data if n else 0), n, _c.byref(opts),
                                          _c.byref(h)))
            keep = arr
        return Index(self, h, keep)

    def build_index_file(self, path, radius_hint: float = 0.0, grid=None, kind: int = INDEX_GRID, level: int = 0,
                         verify: bool = False) -> "Index":
        """Index over a decoded particle file, read in chunks that are uploaded
        as they are read (no page-locked copy of the whole file)."""
        opts = _make_opts(radius_hint, grid, kind, level, verify)
        h = _vp()
        _check(lib().sjcs_index_build_file(self._h, os.fsencode(str(path)), _c.byref(opts), _c.byref(h)))
        return Index(self, h, None)

    def prepare_files(self, max_particles: int) -> None:
        """Page-lock the file staging slots and grow the device pool for files
        of up to max_particles (the first build_index_file then pays for neither)."""
        _check(lib().sjcs_ctx_prepare_files(self._h, int(max_particles)))

    def build_index_compressed(self, uv, header: bytes, radius_hint: float = 0.0, kind: int = INDEX_GRID,
                               level: int = 0) -> "Index":
        """Index over compressed particles: (n, 3) uint16 displacements and the
        file's 256-byte Gadget header; decoded on the device."""
        uv = np.ascontiguousarray(uv, dtype=np.uint16).reshape(-1, 3)
        hdr = _c.create_string_buffer(bytes(header), 256)
        opts = _make_opts(radius_hint, None, kind, level, False)
        h = _vp()
        _check(lib().sjcs_index_build_compressed(self._h, _vp(uv.ctypes.data if len(uv) else 0), len(uv), hdr,
                                                 _c.byref(opts), _c.byref(h)))
        return Index(self, h, (uv, hdr))

    def decode_compressed(self, uv, header: bytes) -> np.ndarray:
        """(n, 3) float32 positions decoded on the device."""
        uv = np.ascontiguousarray(uv, dtype=np.uint16).reshape(-1, 3)
        out = np.empty((len(uv), 3), np.float32)
        hdr = _c.create_string_buffer(bytes(header), 256)
        _check(lib().sjcs_decode_compressed(self._h, _vp(uv.ctypes.data if len(uv) else 0), len(uv), hdr,
                                            _vp(out.ctypes.data if len(uv) else 0)))
        return out

    def step(self, query: "Query", n: int, radius_hint: float = 0.0, kind: int = INDEX_GRID, level: int = 0,
             verify: bool = False) -> "Step":
        """A file step (copy, build, count) captured as a CUDA graph over a pinned
        host buffer of n particles (Step.buffer, an (n, 3) float32 array)."""
        return Step(self, query, n, _make_opts(radius_hint, None, kind, level, verify))

    def set_overlap(self, overlap: bool) -> None:
        """Let index builds' kernels run beside queued counts (default: they wait)."""
        _check(lib().sjcs_ctx_set_overlap(self._h, 1 if overlap else 0))

    def autotune(self, query: "Query", index: "Index") -> "dict":
        """Time the candidate count schedules on the full query; keep the fastest."""
        ch = sjcs_schedule()
        ms = (_c.c_float * 16)()
        nt = _c.c_int()
        _check(lib().sjcs_autotune(self._h, query._h, index._h, _c.byref(ch), ms, 16, _c.byref(nt)))
        return {"chosen": _sched_dict(ch), "trial_ms": [ms[i] for i in range(nt.value)]}

    def query(self, halos, r2, periodic: bool = True) -> "Query":
        """Halo set + squared-radius table.  halos: (n,3) float32, a HALO_DTYPE array
        (its .point field is read in place with stride 24), or a CUDA tensor."""
        r2 = np.ascontiguousarray(r2, dtype=np.float32)
        flags = QUERY_PERIODIC if periodic else QUERY_NONPERIODIC
        h = _vp()
        if _is_cuda(halos):
            stride = 4 * (halos.shape[-1] if halos.dim() == 2 else 3)
            n = halos.shape[0] if halos.dim() == 2 else halos.numel() // 3
            _hand_over(self, 1, halos, lambda: _check(lib().sjcs_query_create_device(
                self._h, _vp(halos.data_ptr()), stride, n, _vp(r2.ctypes.data), len(r2), flags, _c.byref(h))))
            keep = halos
        else:
            if isinstance(halos, np.ndarray) and halos.dtype == HALO_DTYPE:
                arr = np.ascontiguousarray(halos)
                base = arr.ctypes.data + HALO_DTYPE.fields["point"][1]
                stride = HALO_DTYPE.itemsize
            else:
                arr = _as_f32_xyz(halos)
                base = arr.ctypes.data
                stride = 12
            n = arr.shape[0]
            _check(lib().sjcs_query_create(self._h, _vp(base if n else 0), stride, n, _vp(r2.ctypes.data),
                                           len(r2), flags, _c.byref(h)))
            keep = arr
        return Query(self, h, n, len(r2), keep)


def _make_opts(radius_hint, grid, kind, level, verify) -> sjcs_index_opts:
    opts = sjcs_index_opts()
    opts.kind = kind
    opts.radius_hint = float(radius_hint)
    if grid is not None:
        for a in range(3):
            opts.grid[a] = int(grid[a])
    if kind != INDEX_GRID:
        opts.grid[0] = int(level)
    opts.flags = INDEX_VERIFY if verify else 0
    return opts


class PinnedBuffer:
    """Page-locked host memory (sjcs_host_alloc) viewed as a numpy array."""

    def __init__(self, shape, dtype=np.float32):
        self.nbytes = max(1, int(np.prod(shape)) * np.dtype(dtype).itemsize)
        self._p = _vp()
        _check(lib().sjcs_host_alloc(self.nbytes, _c.byref(self._p)))
        buf = (_c.c_char * self.nbytes).from_address(self._p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    @property
    def address(self) -> int:
        return self._p.value

    def free(self) -> None:
        if self._p:
            self.array = None
            lib().sjcs_host_free(self._p)
            self._p = _vp()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Step:
    """One particle file's copy + build + count captured as a CUDA graph."""

    def __init__(self, ctx: "Context", query: "Query", n: int, opts: sjcs_index_opts):
        self.ctx = ctx
        self.query = query
        self.pinned = PinnedBuffer((n, 3))
        self.buffer = self.pinned.array
        self._h = _vp()
        _check(lib().sjcs_step_create(ctx._h, query._h, _vp(self.pinned.address), n, _c.byref(opts),
                                      _c.byref(self._h)))

    def launch(self) -> "Step":
        _check(lib().sjcs_step_launch(self.ctx._h, self._h))
        return self

    def wait(self) -> "Step":
        _check(lib().sjcs_step_wait(self._h))
        return self

    def time_ms(self) -> float:
        ms = _c.c_float()
        _check(lib().sjcs_step_time(self._h, _c.byref(ms)))
        return ms.value

    def destroy(self) -> None:
        if self._h:
            _check(lib().sjcs_step_destroy(self._h))
            self._h = None
        self.buffer = None
        self.pinned.free()


class Index:
    def __init__(self, ctx: Context, h, keep):
        self.ctx = ctx
        self._h = h
        self._keep = keep  # host buffer must live until the build is done

    def wait(self) -> "Index":
        _check(lib().sjcs_index_wait(self._h))
        self._keep = None
        return self

    @property
    def size(self) -> int:
        v = _u64()
        _check(lib().sjcs_index_size(self._h, _c.byref(v)))
        return v.value

    @property
    def grid(self):
        g = (_c.c_uint32 * 3)()
        _check(lib().sjcs_index_grid(self._h, g))
        return tuple(g)

    def timing(self) -> dict:
        t = sjcs_timing()
        _check(lib().sjcs_index_timing(self._h, _c.byref(t)))
        return {"h2d_ms": t.h2d_ms, "build_ms": t.build_ms}

    def learned_info(self) -> dict:
        """Training record of a learned index (waits for the build)."""
        li = sjcs_learned_info()
        _check(lib().sjcs_index_learned_info(self._h, _c.byref(li)))
        return {f: getattr(li, f) for f, _ in sjcs_learned_info._fields_}

    def destroy(self) -> None:
        if self._h:
            _check(lib().sjcs_index_destroy(self._h))
            self._h = None
            self._keep = None

    def __del__(self):
        try:
            if self._h and self.ctx._h:
                lib().sjcs_index_destroy(self._h)
        except Exception:
            pass


class Query:
    def __init__(self, ctx: Context, h, nhalos: int, nrads: int, keep):
        self.ctx = ctx
        self._h = h
        self.nhalos = nhalos
        self.nrads = nrads
        self._keep = keep
        self._reading = None

    def count(self, index: Index) -> "Query":
        _check(lib().sjcs_query_count(self.ctx._h, self._h, index._h))
        return self

    def count_many(self, indexes) -> "Query":
        """The counts of count(i) for every index i, grid indexes of one cell
        grid counted in one pass (up to 4 at a time)."""
        indexes = list(indexes)
        arr = (_vp * max(1, len(indexes)))(*[i._h for i in indexes])
        _check(lib().sjcs_query_count_many(self.ctx._h, self._h, arr, len(indexes)))
        return self

    def wait(self) -> "Query":
        _check(lib().sjcs_query_wait(self._h))
        return self

    def read_counts(self, out: np.ndarray | None = None, accumulate: bool = False) -> np.ndarray:
        if out is None:
            out = np.zeros((self.nhalos, self.nrads), dtype=np.uint64)
        elif out.dtype != np.uint64 or not out.flags.c_contiguous or out.size != self.nhalos * self.nrads:
            raise ValueError("out must be a C-contiguous uint64 array of nhalos*nrads elements")
        _check(lib().sjcs_query_read_counts(self.ctx._h, self._h, _vp(_ptr(out)), 1 if accumulate else 0))
        return out

    def read_counts_async(self, out: np.ndarray) -> np.ndarray:
        """Queue a read of the counts into page-locked `out` (a PinnedBuffer's
        uint64 array of nhalos*nrads elements) and return at once; the counts
        are there after wait_read()."""
        if out.dtype != np.uint64 or not out.flags.c_contiguous or out.size != self.nhalos * self.nrads:
            raise ValueError("out must be a C-contiguous uint64 array of nhalos*nrads elements")
        _check(lib().sjcs_query_read_counts_async(self.ctx._h, self._h, _vp(_ptr(out))))
        self._reading = out  # keep the destination alive while the copy runs
        return out

    def read_counts32_async(self, out: np.ndarray) -> np.ndarray:
        """read_counts_async into a page-locked uint32 array: the 32-bit
        accumulators copied as they are, exact while the query has not folded
        (folds == 0); fails after a fold."""
        if out.dtype != np.uint32 or not out.flags.c_contiguous or out.size != self.nhalos * self.nrads:
            raise ValueError("out must be a C-contiguous uint32 array of nhalos*nrads elements")
        _check(lib().sjcs_query_read_counts32_async(self.ctx._h, self._h, _vp(_ptr(out))))
        self._reading = out
        return out

    def wait_read(self) -> None:
        _check(lib().sjcs_query_wait_read(self._h))
        self._reading = None

    def read_counts_into(self, ptr: int, accumulate: bool = False) -> None:
        """Read into caller memory given by address (e.g. a pinned torch tensor)."""
        _check(lib().sjcs_query_read_counts(self.ctx._h, self._h, _vp(ptr), 1 if accumulate else 0))

    @property
    def device_counts_ptr(self) -> int:
        p = _vp()
        _check(lib().sjcs_query_device_counts(self._h, _c.byref(p)))
        return p.value or 0

    def reset(self) -> None:
        _check(lib().sjcs_query_reset(self.ctx._h, self._h))

    def set_fold_limit(self, limit: int) -> "Query":
        """Fold the u32 device accumulators into the 64-bit totals once they could pass `limit`."""
        _check(lib().sjcs_query_set_fold_limit(self.ctx._h, self._h, int(limit)))
        return self

    @property
    def folds(self) -> int:
        v = _c.c_uint32()
        _check(lib().sjcs_query_folds(self._h, _c.byref(v)))
        return int(v.value)

    def set_schedule(self, mode: int = SCHED_AUTO, piece: int = 0, max_pieces: int = 0, single: int = 0) -> "Query":
        sc = sjcs_schedule(mode, piece, max_pieces, single)
        _check(lib().sjcs_query_set_schedule(self.ctx._h, self._h, _c.byref(sc)))
        return self

    def schedule(self) -> dict:
        sc = sjcs_schedule()
        _check(lib().sjcs_query_get_schedule(self._h, _c.byref(sc)))
        return _sched_dict(sc)

    def timing(self) -> dict:
        t = sjcs_timing()
        _check(lib().sjcs_query_timing(self._h, _c.byref(t)))
        return {"count_ms": t.count_ms, "count_calls": t.count_calls, "d2h_ms": t.d2h_ms}

    def destroy(self) -> None:
        if self._h:
            _check(lib().sjcs_query_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            if self._h and self.ctx._h:
                lib().sjcs_query_destroy(self._h)
        except Exception:
            pass


class Server:
    """Request loop over device-resident indexes (sjcs_server_*)."""

    def __init__(self, ctx: "Context", indexes, slots: int = 0, mem_budget: int = 0):
        self.ctx = ctx
        self._indexes = list(indexes)
        arr = (_vp * max(1, len(self._indexes)))(*[i._h for i in self._indexes])
        o = sjcs_server_opts()
        o.slots = slots
        o.mem_budget = mem_budget
        self._h = _vp()
        _check(lib().sjcs_server_create(ctx._h, arr, len(self._indexes), _c.byref(o), _c.byref(self._h)))
        self._live = {}

    def submit(self, halos, r2, periodic: bool = True, out: np.ndarray | None = None) -> int:
        """Queue a request; returns its ticket.  halos: (n,3) float32 or HALO_DTYPE array."""
        r2 = np.ascontiguousarray(r2, dtype=np.float32)
        if isinstance(halos, np.ndarray) and halos.dtype == HALO_DTYPE:
            arr = np.ascontiguousarray(halos)
            base, stride = arr.ctypes.data + HALO_DTYPE.fields["point"][1], 24
        else:
            arr = _as_f32_xyz(halos)
            base, stride = arr.ctypes.data, 12
        n = arr.shape[0]
        if out is None:
            out = np.empty((n, len(r2)), np.uint32)
        t = _u64()
        _check(lib().sjcs_server_submit(self._h, _vp(base if n else 0), stride, n, _vp(r2.ctypes.data), len(r2),
                                        QUERY_PERIODIC if periodic else QUERY_NONPERIODIC,
                                        _vp(out.ctypes.data if n else 0), _c.byref(t)))
        self._live[t.value] = (arr, r2, out)
        return t.value

    def wait(self, ticket: int):
        """(counts uint32 [n, nrads], info dict) of a submitted request."""
        info = sjcs_request_info()
        rc = lib().sjcs_server_wait(self._h, ticket, _c.byref(info))
        _, _, out = self._live.pop(ticket)
        _check(rc)
        return out, {f: getattr(info, f) for f, _ in sjcs_request_info._fields_}

    def stats(self) -> dict:
        st = sjcs_server_info()
        _check(lib().sjcs_server_stats(self._h, _c.byref(st)))
        return {f: getattr(st, f) for f, _ in sjcs_server_info._fields_ if f != "pad_"}

    def close(self) -> None:
        if self._h:
            _check(lib().sjcs_server_destroy(self._h))
            self._h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _sched_dict(sc) -> dict:
    return {f: getattr(sc, f) for f, _ in sjcs_schedule._fields_}


def launch_counter() -> int:
    """Kernels launched by libsjcs.so in this process so far."""
    return int(lib().sjcs_launch_counter())


def multi_range_count_with_periodic_bound(ctx: Context, index: Index, halos, r2, counts: np.ndarray,
                                          periodic: bool = True) -> np.ndarray:
    """counts (uint64 [nhalos, nrads]) += shell counts of `halos` against `index`
    (one file's pass of threadJoin: multiRangeCountWithPriodicBoundArraySTR per halo)."""
    r2 = np.ascontiguousarray(r2, dtype=np.float32)
    if isinstance(halos, np.ndarray) and halos.dtype == HALO_DTYPE:
        arr = np.ascontiguousarray(halos)
        base, stride = arr.ctypes.data + HALO_DTYPE.fields["point"][1], 24
    else:
        arr = _as_f32_xyz(halos)
        base, stride = arr.ctypes.data, 12
    n = arr.shape[0]
    if counts.dtype != np.uint64 or not counts.flags.c_contiguous or counts.size != n * len(r2):
        raise ValueError("counts must be a C-contiguous uint64 array of nhalos*nrads elements")
    _check(lib().sjcs_multi_range_count(ctx._h, index._h, _vp(base if n else 0), stride, n, _vp(r2.ctypes.data),
                                        len(r2), QUERY_PERIODIC if periodic else QUERY_NONPERIODIC,
                                        _vp(counts.ctypes.data)))
    return counts


# ---------------------------------------------------------------------------
# host formats and generators (CPU only)
# ---------------------------------------------------------------------------

def radius_table(minrad: float, maxrad: float, nrads: int) -> np.ndarray:
    """Squared radii as the reference driver builds them (Logspace then r*r in fp32)."""
    out = np.zeros(nrads, dtype=np.float32)
    _hcheck(host_lib().sjcs_host_radius_table(float(minrad), float(maxrad), int(nrads), _vp(out.ctypes.data)))
    return out


def read_particles(path) -> np.ndarray:
    n = _u64()
    _hcheck(host_lib().sjcs_particle_file_count(os.fsencode(path), _c.byref(n)))
    out = np.empty((n.value, 3), dtype=np.float32)
    got = _u64()
    _hcheck(host_lib().sjcs_read_particles(os.fsencode(path), _vp(out.ctypes.data), n.value, _c.byref(got)))
    return out[: got.value]


def _take_halos(p, n: int) -> np.ndarray:
    try:
        if n == 0:
            return np.zeros(0, dtype=HALO_DTYPE)
        buf = (_c.c_uint8 * (n * 24)).from_address(p.value)
        return np.frombuffer(buf, dtype=HALO_DTYPE).copy()
    finally:
        host_lib().sjcs_host_free_halos(p)


def read_halos(path, filter_path=None, nthreads: int = 0) -> np.ndarray:
    p = _vp()
    n = _u64()
    if filter_path is None:
        _hcheck(host_lib().sjcs_read_halos(os.fsencode(path), _c.byref(p), _c.byref(n), int(nthreads)))
    else:
        _hcheck(host_lib().sjcs_read_and_filter_halos(os.fsencode(path), os.fsencode(filter_path), _c.byref(p),
                                                      _c.byref(n)))
    return _take_halos(p, n.value)


def write_result(path, halos: np.ndarray, r2, counts: np.ndarray, nthreads: int = 0) -> None:
    r2 = np.ascontiguousarray(r2, dtype=np.float32)
    halos = np.ascontiguousarray(halos, dtype=HALO_DTYPE)
    counts = np.ascontiguousarray(counts, dtype=np.uint64)
    _hcheck(host_lib().sjcs_write_result(None if path is None else os.fsencode(path), _vp(halos.ctypes.data),
                                         len(halos), _vp(r2.ctypes.data), len(r2), _vp(counts.ctypes.data),
                                         int(nthreads)))


def gen_uniform_particles(seed: int, nfiles: int, n: int) -> np.ndarray:
    out = np.empty((nfiles * n, 3), dtype=np.float32)
    _hcheck(host_lib().sjcs_gen_uniform_particles(seed, nfiles, n, _vp(out.ctypes.data)))
    return out


def gen_uniform_halo_file(path, seed: int, n: int, id0: int = 0) -> None:
    _hcheck(host_lib().sjcs_gen_uniform_halo_file(os.fsencode(path), seed, n, id0))


def gen_uniform_halos(seed: int, n: int, id0: int = 0, nthreads: int = 0) -> np.ndarray:
    out = np.zeros(n, dtype=HALO_DTYPE)
    _hcheck(host_lib().sjcs_gen_uniform_halos(seed, n, id0, _vp(out.ctypes.data), nthreads))
    return out


def gen_face_halos(seed: int, n: int, id0: int = 0, margin: float = 5.0) -> np.ndarray:
    out = np.zeros(n, dtype=HALO_DTYPE)
    _hcheck(host_lib().sjcs_gen_face_halos(seed, n, id0, margin, _vp(out.ctypes.data)))
    return out


# Clustered workload: 1e4 clumps, sigma log-uniform [2, 20], weights lognormal(0, 1.5), 60% clumped.
CLUSTER_DEFAULTS = dict(nclumps=10000, sig_lo=2.0, sig_hi=20.0, wsig=1.5)


def gen_clustered_particles(seed: int, n: int, frac_clumped: float = 0.6, clump_seed: int = 31,
                            **kw) -> np.ndarray:
    p = {**CLUSTER_DEFAULTS, **kw}
    out = np.empty((n, 3), dtype=np.float32)
    _hcheck(host_lib().sjcs_gen_clustered_particles(seed, n, p["nclumps"], p["sig_lo"], p["sig_hi"], p["wsig"],
                                                    frac_clumped, clump_seed, _vp(out.ctypes.data)))
    return out


def gen_clustered_halos(seed: int, n: int, id0: int = 0, frac_at_clumps: float = 0.7, jitter: float = 1.0,
                        clump_seed: int = 31, **kw) -> np.ndarray:
    p = {**CLUSTER_DEFAULTS, **kw}
    out = np.zeros(n, dtype=HALO_DTYPE)
    _hcheck(host_lib().sjcs_gen_clustered_halos(seed, n, id0, p["nclumps"], p["sig_lo"], p["sig_hi"], p["wsig"],
                                                frac_at_clumps, jitter, clump_seed, _vp(out.ctypes.data)))
    return out


def gen_compressed(seed: int, n1d: int, box: float = 1000.0, disp_min: float = -4.0, disp_max: float = 4.0,
                   pos_bits: int = 16, id_start: int = 1, n: int | None = None):
    """Synthetic compressed particles: (256-byte header, (n, 3) uint16 displacements)."""
    n = n1d ** 3 if n is None else n
    hdr = _c.create_string_buffer(256)
    uv = np.empty((n, 3), np.uint16)
    _hcheck(host_lib().sjcs_gen_compressed(seed, n1d, box, disp_min, disp_max, pos_bits, id_start, n, hdr,
                                           _vp(uv.ctypes.data if n else 0)))
    return hdr.raw, uv


def write_compressed_file(path, header: bytes, uv) -> None:
    uv = np.ascontiguousarray(uv, dtype=np.uint16).reshape(-1, 3)
    hdr = _c.create_string_buffer(bytes(header), 256)
    _hcheck(host_lib().sjcs_write_compressed_file(os.fsencode(path), hdr, _vp(uv.ctypes.data if len(uv) else 0),
                                                  len(uv)))


def read_compressed(path):
    """(256-byte header, (n, 3) uint16 displacements) of a compressed particle file."""
    hdr = _c.create_string_buffer(256)
    n = _u64()
    _hcheck(host_lib().sjcs_read_compressed_particles(os.fsencode(path), hdr, None, 0, _c.byref(n)))
    uv = np.empty((n.value, 3), np.uint16)
    got = _u64()
    _hcheck(host_lib().sjcs_read_compressed_particles(os.fsencode(path), hdr, _vp(uv.ctypes.data if n.value else 0),
                                                      n.value, _c.byref(got)))
    return hdr.raw, uv[: got.value]


def write_halo_file(path, halos: np.ndarray) -> None:
    halos = np.ascontiguousarray(halos, dtype=HALO_DTYPE)
    _hcheck(host_lib().sjcs_write_halo_file(os.fsencode(path), _vp(halos.ctypes.data), len(halos)))


def write_particle_file(path, xyz) -> None:
    arr = _as_f32_xyz(xyz)
    _hcheck(host_lib().sjcs_write_particle_file(os.fsencode(path), _vp(arr.ctypes.data), arr.shape[0]))
