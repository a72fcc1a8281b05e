"""Event files of one camera with the interface of ``ballasim._export`` (src/export/export_module.cpp:331-387):
``RawWriter`` (Prophesee RAW: EVT 2.0, 2.1 or 3.0 words) and ``DatWriter`` (Prophesee DAT records), T1a times
u = floor(t_ns / 1000) - origin_us. The words of each appended batch are built on the device (bs_event_writer_*);
the header, the file and its SHA-256 on the host. Refusals raise ExportError (a ValueError), as the reference's.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _lib
from ._lib import ExportError

__all__ = ["RawWriter", "DatWriter", "ExportError"]


def _column(a, dtype, name: str) -> np.ndarray:
    """The exact-dtype 1-D C-contiguous column the reference's binding takes without conversion."""
    if not isinstance(a, np.ndarray) or a.dtype != dtype or a.ndim != 1 or not a.flags.c_contiguous:
        raise TypeError(f"append: {name} must be a 1-D C-contiguous {np.dtype(dtype).name} array")
    return a


class _EventWriter:
    def __init__(self, h: C.c_void_p, path: str):
        self._h = h
        self._path = path
        self._lock = threading.Lock()

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                _lib.lib().bs_event_writer_destroy(h)
            except Exception:  # interpreter shutdown
                pass

    def append(self, x, y, p, t_ns) -> None:
        """Events in output order: uint16 x, uint16 y, uint8 p (0/1) and int64 t_ns (t_reported on the camera's
        sensor clock), 1-D C-contiguous arrays of these exact dtypes; t_ns non-decreasing within and across calls
        and >= 1000 origin_us, x < width, y < height, t_ns mod 1000 in the declared t_ns_rem range. A batch that
        breaks any is refused whole (ExportError)."""
        x = _column(x, np.uint16, "x")
        y = _column(y, np.uint16, "y")
        p = _column(p, np.uint8, "p")
        t = _column(t_ns, np.int64, "t_ns")
        n = len(t)
        if len(x) != n or len(y) != n or len(p) != n:
            raise ExportError("append: x, y, p and t_ns must have one length")
        with self._lock:
            _lib.check(_lib.lib().bs_event_writer_append(self._h, x.ctypes.data, y.ctypes.data, p.ctypes.data,
                                                          t.ctypes.data, n))

    def append_device(self, x, y, p, t_ns, n: int, stream: int | None = None) -> None:
        """As append with device columns given as pointers (for example an output stage's buffers)."""
        with self._lock:
            _lib.check(_lib.lib().bs_event_writer_append_device(self._h, x, y, p, t_ns, int(n), stream))

    def close(self) -> dict:
        """Flushes, closes and hashes the file: {path, bytes, sha256, streams: [{camera, kind, id, count, t_first,
        t_last}]} with t_first and t_last in u (us after the origin, T1a); camera and id are the caller's to fill."""
        info = _lib.FileInfo()
        with self._lock:
            _lib.check(_lib.lib().bs_event_writer_close(self._h, C.byref(info)))
        return {"path": self._path, "bytes": int(info.bytes), "sha256": info.sha256.decode(),
                "streams": [{"camera": "", "kind": "events", "id": "", "count": int(info.count),
                             "t_first": int(info.t_first), "t_last": int(info.t_last)}]}

    def stats(self) -> dict:
        """This build's counters: kernel launches of the appends so far; the last append's kernel device time (ms),
        the bytes of its words, its wall time and its file writes' (ms); close's hash of the file (ms)."""
        n, ms, b = C.c_uint64(), C.c_double(), C.c_uint64()
        host = (C.c_double * 3)()
        _lib.check(_lib.lib().bs_event_writer_stats(self._h, C.byref(n), C.byref(ms), C.byref(b), host))
        return {"gpu_launches": n.value, "last_kernel_ms": ms.value, "last_words_bytes": b.value,
                "last_append_ms": host[0], "last_file_write_ms": host[1], "close_hash_ms": host[2]}


class RawWriter(_EventWriter):
    """A Prophesee RAW file of one camera's events (EVT 2.0, 2.1 or 3.0), T1a times: u = floor(t_ns / 1000) -
    origin_us. format: evt2, evt21 or evt3; width and height <= 2048; epoch_ns a multiple of 1000 (recorded in the
    header with the origin); evt2_time_high: openeb (a TIME_HIGH every 16 us, OpenEB's encoder) or change (EVT 2.0
    only; EVT 2.1 is always on change); [t_ns_rem_min, t_ns_rem_max]: the window's pre-scanned sub-us parts (-1, -1:
    no events); version: the header's 'plugin_version BallaSim <version>'."""

    def __init__(self, path: str, format: str, width: int, height: int, origin_us: int, epoch_ns: int,
                 evt2_time_high: str = "openeb", t_ns_rem_min: int = 0, t_ns_rem_max: int = 0, version: str = ""):
        h = C.c_void_p()
        _lib.check(_lib.lib().bs_raw_writer_create(str(path).encode(), str(format).encode(), int(width), int(height),
                                                   int(origin_us), int(epoch_ns), str(evt2_time_high).encode(),
                                                   int(t_ns_rem_min), int(t_ns_rem_max), str(version).encode(),
                                                   C.byref(h)))
        super().__init__(h, str(path))


class DatWriter(_EventWriter):
    """A Prophesee DAT file of one camera's events: u32 us under T1a, refused from u = 2^32 us on. As RawWriter,
    with width and height <= 16384; the version is not written (DAT has no plugin line)."""

    def __init__(self, path: str, width: int, height: int, origin_us: int, epoch_ns: int, t_ns_rem_min: int = 0,
                 t_ns_rem_max: int = 0, version: str = ""):
        h = C.c_void_p()
        _lib.check(_lib.lib().bs_dat_writer_create(str(path).encode(), int(width), int(height), int(origin_us),
                                                   int(epoch_ns), int(t_ns_rem_min), int(t_ns_rem_max),
                                                   str(version).encode(), C.byref(h)))
        super().__init__(h, str(path))


def sha256_hex(data: bytes) -> str:
    """SHA-256 of a byte string as lower-case hex (the library's own, which close() uses)."""
    out = C.create_string_buffer(65)
    b = bytes(data)
    _lib.check(_lib.lib().bs_sha256_hex(b, len(b), out))
    return out.value.decode()
