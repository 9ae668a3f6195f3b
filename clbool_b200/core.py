"""Host layer mirroring clBool's core types over the C ABI.

Reference types (clBool sources):
  Controls            src/core/controls.hpp:12-28
  Status / Exception  src/core/error.hpp:130-213
  matrix_dcsr         src/core/matrix_dcsr.hpp:11-84
  matrix_coo          src/core/matrix_coo.hpp:12-83, ctor src/core/matrix_coo.cpp:17-68
  matrix_csr          src/core/matrix_csr.hpp:7-42
  matrix_*_cpu        src/core/cpu_matrices.hpp:9-169

Device buffers are reference counted (Python references play the role of
cl::Buffer's refcount), so copies of a matrix are shallow and conversions
that the reference documents as "shallow for cols" share the column buffer.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._capi import clb_coo, clb_csr, clb_dcsr, lib

STATUS_NAMES = {
    0: "CLBOOL_SUCCESS", 1: "CLBOOL_NO_SUCH_PROGRAM", 2: "CLBOOL_CREATE_KERNEL_ERROR",
    3: "CLBOOL_BUILD_PROGRAM_ERROR", 4: "CLBOOL_INCOMPLETE_KERNEL", 5: "CLBOOL_RUN_KERNEL_FAILURE",
    6: "CLBOOL_EVENT_WAITING_ERROR", 7: "CLBOOL_CREATE_BUFFER_ERROR", 8: "CLBOOL_COPY_BUFFER_ERROR",
    9: "CLBOOL_READ_BUFFER_ERROR", 10: "CLBOOL_WRITE_BUFFER_ERROR", 11: "CLBOOL_CREATE_CONTROLS_ERROR",
    12: "CLBOOL_INVALID_ARGUMENT", 13: "CLBOOL_INVALID_VALUE", 14: "CLBOOL_INITIALIZATION_ERROR",
    64: "CLBOOL_DEVICE_STATUS_ERROR", 65: "CLBOOL_NOT_SUPPORTED",
}


class ClBoolException(Exception):
    """clbool::Exception: carries the Status name of the failing call."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"[{self.status_name}] {message}")


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = lib.clb_last_error().decode(errors="replace")
        raise ClBoolException(status, f"{what}: {msg}" if what else msg)


# ---------------------------------------------------------------- controls --
class Controls:
    """One CUDA device with a stream and a stream-ordered allocator."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.clb_controls_create(device, C.byref(h)), "create_controls")
        self._h = h
        self.device = device

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def sync(self) -> None:
        check(lib.clb_controls_sync(self._h), "sync")

    def trim(self) -> None:
        """Wait for the stream, then hand the memory pool's cached, unused
        device memory back to the driver (clb_controls_trim)."""
        check(lib.clb_controls_trim(self._h), "trim")

    def set_stream(self, stream_ptr: int) -> None:
        check(lib.clb_controls_set_stream(self._h, C.c_void_p(stream_ptr or None)), "set_stream")

    def profile(self, on: bool = True) -> None:
        """Enable (or disable) per-kernel CUDA-event timing; clears records."""
        check(lib.clb_profile_enable(self._h, 1 if on else 0), "profile_enable")

    def profile_read(self) -> dict:
        """{kernel name: (launches, total ms)} since the last read; clears."""
        from ._capi import clb_profile_entry
        buf = (clb_profile_entry * 64)()
        n = C.c_int()
        check(lib.clb_profile_read(self._h, buf, 64, C.byref(n)), "profile_read")
        return {buf[i].name.decode(): (int(buf[i].launches), float(buf[i].ms)) for i in range(n.value)}

    @property
    def stream(self) -> int:
        return lib.clb_controls_get_stream(self._h) or 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.clb_controls_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def create_controls(platform_id: int = 0, device_id: int = 0) -> Controls:
    """create_controls (src/common/env.cpp:7-36).  CUDA exposes one platform."""
    if platform_id != 0:
        raise ClBoolException(11, f"no platform with id {platform_id}")
    return Controls(device_id)


def device_count() -> int:
    n = C.c_int()
    check(lib.clb_device_count(C.byref(n)))
    return n.value


def show_devices() -> list[dict]:
    """show_devices (src/common/env.cpp:38-54): prints and returns the devices."""
    out = []
    for d in range(device_count()):
        name = C.create_string_buffer(256)
        sms = C.c_int()
        mem = C.c_uint64()
        check(lib.clb_device_info(d, name, 256, C.byref(sms), C.byref(mem)))
        info = {"device": d, "name": name.value.decode(), "sm_count": sms.value, "total_mem": mem.value}
        print(f"device id: {d}  {info['name']}  SMs={sms.value}  mem={mem.value // (1 << 20)} MiB")
        out.append(info)
    return out


# ------------------------------------------------------------ device memory --
class DeviceBuffer:
    """Owning handle of one device allocation (freed when the last reference goes)."""

    __slots__ = ("ctl", "ptr", "count", "dtype", "owned", "__weakref__")

    def __init__(self, ctl: Controls, ptr: int, count: int, dtype, owned: bool = True):
        self.ctl = ctl
        self.ptr = int(ptr or 0)
        self.count = int(count)
        self.dtype = np.dtype(dtype)
        self.owned = owned

    @classmethod
    def empty(cls, ctl: Controls, count: int, dtype) -> "DeviceBuffer":
        nbytes = int(count) * np.dtype(dtype).itemsize
        p = C.c_void_p()
        check(lib.clb_malloc(ctl.handle, nbytes, C.byref(p)), "create_buffer")
        return cls(ctl, p.value, count, dtype)

    @classmethod
    def from_host(cls, ctl: Controls, arr: np.ndarray, dtype) -> "DeviceBuffer":
        a = np.ascontiguousarray(arr, dtype=dtype)
        if a.size == 0:
            return cls(ctl, 0, 0, dtype)
        b = cls.empty(ctl, a.size, dtype)
        check(lib.clb_memcpy_h2d(ctl.handle, C.c_void_p(b.ptr), a.ctypes.data_as(C.c_void_p), a.nbytes),
              "write_buffer")
        return b

    @property
    def nbytes(self) -> int:
        return self.count * self.dtype.itemsize

    def to_host(self, count: Optional[int] = None) -> np.ndarray:
        n = self.count if count is None else int(count)
        out = np.empty(n, dtype=self.dtype)
        if n:
            check(lib.clb_memcpy_d2h(self.ctl.handle, out.ctypes.data_as(C.c_void_p), C.c_void_p(self.ptr),
                                     n * self.dtype.itemsize), "read_buffer")
        return out

    def __del__(self):
        try:
            if self.owned and self.ptr and self.ctl.handle:
                lib.clb_free(self.ctl.handle, C.c_void_p(self.ptr))
        except Exception:
            pass
        self.ptr = 0


def _buf(ctl, ptr, count, dtype, owned=True):
    if not ptr:
        return None
    return DeviceBuffer(ctl, ptr, count, dtype, owned)


def _p(b: Optional[DeviceBuffer]):
    return C.c_void_p(b.ptr if b is not None else None)


# ------------------------------------------------------------- host types --
class matrix_dcsr_cpu:
    """Host DCSR (cpu_matrices.hpp:9-52)."""

    def __init__(self, rpt=None, rows=None, cols=None):
        self.rpt = np.asarray(rpt if rpt is not None else [], dtype=np.uint64)
        self.rows = np.asarray(rows if rows is not None else [], dtype=np.uint32)
        self.cols = np.asarray(cols if cols is not None else [], dtype=np.uint32)


class matrix_coo_cpu:
    """Host COO (cpu_matrices.hpp:55-106)."""

    def __init__(self, rows=None, cols=None):
        self.rows = np.asarray(rows if rows is not None else [], dtype=np.uint32)
        self.cols = np.asarray(cols if cols is not None else [], dtype=np.uint32)


class matrix_csr_cpu:
    """Host CSR (cpu_matrices.hpp:108-169)."""

    def __init__(self, rpt=None, cols=None, nrows: int = 0, ncols: int = 0):
        self.rpt = np.asarray(rpt if rpt is not None else [], dtype=np.uint64)
        self.cols = np.asarray(cols if cols is not None else [], dtype=np.uint32)
        self.nrows = nrows
        self.ncols = ncols


# ----------------------------------------------------------- device types --
class _matrix_base:
    """details::matrix_base (src/core/matrix_base.hpp:10-56)."""

    def __init__(self, nrows=0, ncols=0, nnz=0):
        self._nrows, self._ncols, self._nnz = int(nrows), int(ncols), int(nnz)

    def nrows(self) -> int:
        return self._nrows

    def ncols(self) -> int:
        return self._ncols

    def nnz(self) -> int:
        return self._nnz

    def empty(self) -> bool:
        return self._nnz == 0


class matrix_dcsr(_matrix_base):
    def __init__(self, rpt: Optional[DeviceBuffer] = None, rows: Optional[DeviceBuffer] = None,
                 cols: Optional[DeviceBuffer] = None, nrows: int = 0, ncols: int = 0, nnz: int = 0, nzr: int = 0):
        super().__init__(nrows, ncols, nnz)
        self._rpt, self._rows, self._cols, self._nzr = rpt, rows, cols, int(nzr)

    @classmethod
    def zeros(cls, nrows: int, ncols: int) -> "matrix_dcsr":
        """matrix_dcsr(nrows, ncols): an empty matrix without buffers."""
        return cls(None, None, None, nrows, ncols, 0, 0)

    def nzr(self) -> int:
        return self._nzr

    def rpt_gpu(self):
        return self._rpt

    def rows_gpu(self):
        return self._rows

    def cols_gpu(self):
        return self._cols

    def _assign(self, other: "matrix_dcsr") -> "matrix_dcsr":
        self._nrows, self._ncols, self._nnz, self._nzr = other._nrows, other._ncols, other._nnz, other._nzr
        self._rpt, self._rows, self._cols = other._rpt, other._rows, other._cols
        return self

    def c_struct(self) -> clb_dcsr:
        s = clb_dcsr()
        s.nrows, s.ncols, s.nnz, s.nzr = self._nrows, self._ncols, self._nnz, self._nzr
        s.rpt, s.rows, s.cols = _p(self._rpt).value, _p(self._rows).value, _p(self._cols).value
        return s

    @classmethod
    def adopt(cls, ctl: Controls, s: clb_dcsr, cols_owner: Optional[DeviceBuffer] = None) -> "matrix_dcsr":
        """Wrap a clb_dcsr returned by the library (takes ownership of its arrays).
        `cols_owner`, when given, is the buffer a shallow conversion shares."""
        cols = cols_owner if (cols_owner is not None and s.cols == cols_owner.ptr) else _buf(ctl, s.cols, s.nnz,
                                                                                              np.uint32)
        return cls(_buf(ctl, s.rpt, s.nzr + 1, np.uint64), _buf(ctl, s.rows, s.nzr, np.uint32), cols,
                   s.nrows, s.ncols, s.nnz, s.nzr)


class matrix_coo(_matrix_base):
    """matrix_coo; construct from host arrays with `matrix_coo.from_host`."""

    def __init__(self, rows: Optional[DeviceBuffer] = None, cols: Optional[DeviceBuffer] = None, nrows: int = 0,
                 ncols: int = 0, nnz: int = 0):
        super().__init__(nrows, ncols, nnz)
        self._rows, self._cols = rows, cols

    @classmethod
    def zeros(cls, nrows: int, ncols: int) -> "matrix_coo":
        return cls(None, None, nrows, ncols, 0)

    @classmethod
    def from_host(cls, controls: Controls, rows, cols, nrows: int, ncols: int, nnz: Optional[int] = None,
                  sorted: bool = True, noDuplicates: bool = True) -> "matrix_coo":
        """matrix_coo(controls, rows, cols, nrows, ncols, nnz, sorted, noDuplicates)
        (src/core/matrix_coo.cpp:17-47): upload, sort if unsorted, drop
        duplicates if asked."""
        r = np.ascontiguousarray(rows, dtype=np.uint32)
        c = np.ascontiguousarray(cols, dtype=np.uint32)
        n = r.size if nnz is None else int(nnz)
        r, c = r[:n], c[:n]
        m = cls(DeviceBuffer.from_host(controls, r, np.uint32), DeviceBuffer.from_host(controls, c, np.uint32),
                nrows, ncols, n)
        return m._initialize(controls, sorted, noDuplicates)

    @classmethod
    def from_device(cls, controls: Controls, nrows: int, ncols: int, nnz: int, rows: DeviceBuffer,
                    cols: DeviceBuffer, sorted: bool = True, noDuplicates: bool = True) -> "matrix_coo":
        """matrix_coo(controls, nrows, ncols, nnz, rows, cols, sorted, noDuplicates)
        (src/core/matrix_coo.cpp:50-68)."""
        return cls(rows, cols, nrows, ncols, nnz)._initialize(controls, sorted, noDuplicates)

    def _initialize(self, controls, sorted, noDuplicates):
        from .ops import _coo_reduce_duplicates, _coo_sort
        if self._nnz == 0:
            return self
        if not sorted:
            _coo_sort(controls, self._rows, self._cols, self._nnz)
        if not noDuplicates:
            self._assign(_coo_reduce_duplicates(controls, self))
        return self

    def rows_gpu(self):
        return self._rows

    def cols_gpu(self):
        return self._cols

    def _assign(self, other: "matrix_coo") -> "matrix_coo":
        self._nrows, self._ncols, self._nnz = other._nrows, other._ncols, other._nnz
        self._rows, self._cols = other._rows, other._cols
        return self

    def c_struct(self) -> clb_coo:
        s = clb_coo()
        s.nrows, s.ncols, s.nnz = self._nrows, self._ncols, self._nnz
        s.rows, s.cols = _p(self._rows).value, _p(self._cols).value
        return s

    @classmethod
    def adopt(cls, ctl: Controls, s: clb_coo, rows_owner=None, cols_owner=None) -> "matrix_coo":
        rows = rows_owner if (rows_owner is not None and s.rows == rows_owner.ptr) else _buf(ctl, s.rows, s.nnz,
                                                                                              np.uint32)
        cols = cols_owner if (cols_owner is not None and s.cols == cols_owner.ptr) else _buf(ctl, s.cols, s.nnz,
                                                                                              np.uint32)
        return cls(rows, cols, s.nrows, s.ncols, s.nnz)


class matrix_csr(_matrix_base):
    def __init__(self, rpt: Optional[DeviceBuffer] = None, cols: Optional[DeviceBuffer] = None, nrows: int = 0,
                 ncols: int = 0, nnz: int = 0):
        super().__init__(nrows, ncols, nnz)
        self._rpt, self._cols = rpt, cols

    @classmethod
    def zeros(cls, nrows: int, ncols: int) -> "matrix_csr":
        return cls(None, None, nrows, ncols, 0)

    def rpt_gpu(self):
        return self._rpt

    def cols_gpu(self):
        return self._cols

    def _assign(self, other: "matrix_csr") -> "matrix_csr":
        self._nrows, self._ncols, self._nnz = other._nrows, other._ncols, other._nnz
        self._rpt, self._cols = other._rpt, other._cols
        return self

    def c_struct(self) -> clb_csr:
        s = clb_csr()
        s.nrows, s.ncols, s.nnz = self._nrows, self._ncols, self._nnz
        s.rpt, s.cols = _p(self._rpt).value, _p(self._cols).value
        return s

    @classmethod
    def adopt(cls, ctl: Controls, s: clb_csr, cols_owner=None) -> "matrix_csr":
        cols = cols_owner if (cols_owner is not None and s.cols == cols_owner.ptr) else _buf(ctl, s.cols, s.nnz,
                                                                                              np.uint32)
        return cls(_buf(ctl, s.rpt, s.nrows + 1, np.uint64), cols, s.nrows, s.ncols, s.nnz)
