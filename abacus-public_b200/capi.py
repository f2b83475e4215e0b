"""ctypes binding of libnfb200.so (include/nf_capi.h).

The library is the product; this module only marshals plain pointers and
sizes across the C ABI.  It never falls back to another implementation: if
the shared library is missing or exports are absent, loading fails loudly.
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
LIB_PATH = PKG / "lib" / "libnfb200.so"
HEADER = ROOT / "include" / "nf_capi.h"

NF_OK, NF_EINVAL, NF_ENOMEM, NF_EADMISSION, NF_ETIMEDOUT, NF_EDEVICE, NF_ENODEV, \
    NF_ENOTREADY, NF_ECANCELLED = range(9)
STATUS_NAMES = {0: "NF_OK", 1: "NF_EINVAL", 2: "NF_ENOMEM", 3: "NF_EADMISSION",
                4: "NF_ETIMEDOUT", 5: "NF_EDEVICE", 6: "NF_ENODEV", 7: "NF_ENOTREADY",
                8: "NF_ECANCELLED"}
SOFT_PLUMMER, SOFT_SINGLE_SPLINE, SOFT_CUBIC_SPLINE, SOFT_CUBIC_PLUMMER = range(4)
ACC_COMPENSATED, ACC_PLAIN = 0, 1
OUT_FLOAT3, OUT_FLOAT4 = 0, 1


class NfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("near_field_radius", ctypes.c_int),
                ("softening", ctypes.c_int), ("eps", ctypes.c_float), ("b2", ctypes.c_float),
                ("accumulation", ctypes.c_int), ("out_kind", ctypes.c_int),
                ("sinks_per_lane", ctypes.c_int), ("warps_per_cta", ctypes.c_int)]


class Timing(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_float), ("coadd_ms", ctypes.c_float),
                ("total_ms", ctypes.c_float), ("pairs", ctypes.c_uint64),
                ("padded_pairs", ctypes.c_uint64), ("launches", ctypes.c_int),
                ("items", ctypes.c_int)]


class GpuLimits(ctypes.Structure):
    _fields_ = [("max_sink_blocks", ctypes.c_int), ("max_source_blocks", ctypes.c_int),
                ("max_nsink", ctypes.c_int), ("max_nsource", ctypes.c_int),
                ("max_sink_size", ctypes.c_size_t), ("max_source_size", ctypes.c_size_t)]


class CellPlan(ctypes.Structure):
    _fields_ = [("start", ctypes.c_uint32), ("n", ctypes.c_int32)]


class SicDesc(ctypes.Structure):
    _fields_ = [("cpd", ctypes.c_int), ("nfradius", ctypes.c_int), ("nk", ctypes.c_int),
                ("nsinksets", ctypes.c_int), ("nsourcesets", ctypes.c_int),
                ("nsinkblocks", ctypes.c_int), ("nsourceblocks", ctypes.c_int),
                ("interaction_count", ctypes.c_int),
                ("sink_set_start", ctypes.c_void_p), ("sink_set_count", ctypes.c_void_p),
                ("sink_set_id_max", ctypes.c_void_p), ("sink_plan", ctypes.c_void_p),
                ("sink_wrapcell", ctypes.c_void_p), ("sink_block_parent", ctypes.c_void_p),
                ("source_set_start", ctypes.c_void_p), ("source_set_count", ctypes.c_void_p),
                ("source_plan", ctypes.c_void_p), ("interaction_list", ctypes.c_void_p),
                ("y_offset", ctypes.c_void_p), ("sink_pos_slab", ctypes.c_void_p),
                ("sink_nslab", ctypes.c_uint64), ("source_pos_slab", ctypes.c_void_p),
                ("source_nslab", ctypes.c_void_p), ("sink_acc_slab", ctypes.c_void_p),
                ("b2", ctypes.c_float), ("bytes_to_device", ctypes.c_void_p),
                ("bytes_from_device", ctypes.c_void_p)]


# Every symbol the header declares; the loader checks each one is exported.
EXPORTS = {
    "nf_config_default": (None, [ctypes.POINTER(Config)]),
    "nf_init": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    "nf_shutdown": (None, [ctypes.c_void_p]),
    "nf_last_error": (ctypes.c_char_p, []),
    "nf_abi_version": (ctypes.c_int, []),
    "nf_get_ngpu": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "nf_get_device_info": (ctypes.c_int, [ctypes.POINTER(ctypes.c_size_t), ctypes.c_char_p,
                                          ctypes.c_size_t]),
    "nf_gpu_setup": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.POINTER(GpuLimits)]),
    "nf_gpu_reset": (ctypes.c_int, [ctypes.c_void_p]),
    "nf_sic_execute": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SicDesc), ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "nf_sic_drain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "nf_box_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "nf_box_update": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p]),
    "nf_box_destroy": (None, [ctypes.c_void_p, ctypes.c_void_p]),
    "nf_box_device_bytes": (ctypes.c_size_t, [ctypes.c_void_p]),
    "nf_box_forces": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
    "nf_box_pair_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]),
    "nf_last_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Timing)]),
    "nf_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "nf_measure_fp32_peak": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double,
                                            ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double)]),
}

_lib = None


def declared_symbols() -> list[str]:
    """Function names declared in include/nf_capi.h."""
    import re
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(nf_[a-z0-9_]+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_t")))


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with abacus-public_b200/build.py "
                "(there is no fallback implementation)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in EXPORTS.items():
            fn = getattr(L, name)  # AttributeError if not exported
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return (lib().nf_last_error() or b"").decode()


def check(status: int, what: str = ""):
    if status != NF_OK:
        raise NfError(status, f"{what}: {last_error()}")


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def default_config(**kw) -> Config:
    c = Config()
    lib().nf_config_default(ctypes.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def ngpu() -> int:
    n = ctypes.c_int(0)
    st = lib().nf_get_ngpu(ctypes.byref(n))
    return n.value if st == NF_OK else 0


class Context:
    """nf_ctx: one device, one configuration."""

    def __init__(self, **cfg):
        self.cfg = default_config(**cfg)
        h = ctypes.c_void_p()
        check(lib().nf_init(ctypes.byref(self.cfg), ctypes.byref(h)), "nf_init")
        self.h = h

    def close(self):
        if self.h:
            lib().nf_shutdown(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def box(self, box) -> "DeviceBox":
        return DeviceBox(self, box)

    def set_stream(self, stream_handle: int | None):
        check(lib().nf_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)), "nf_set_stream")

    def fp32_peak(self, seconds_sustained: float = 1.0) -> tuple[float, float]:
        b, s = ctypes.c_double(), ctypes.c_double()
        check(lib().nf_measure_fp32_peak(self.h, seconds_sustained, ctypes.byref(b),
                                         ctypes.byref(s)), "nf_measure_fp32_peak")
        return b.value, s.value

    def last_timing(self) -> Timing:
        t = Timing()
        check(lib().nf_last_timing(self.h, ctypes.byref(t)), "nf_last_timing")
        return t


class DeviceBox:
    """nf_box: a synthetic/host box uploaded once and kept in HBM."""

    def __init__(self, ctx: Context, box):
        self.ctx = ctx
        self.src = box
        self.cpd = box.cpd
        self.np = box.n
        self._cs = np.ascontiguousarray(box.cell_start, dtype=np.int64)
        h = ctypes.c_void_p()
        check(lib().nf_box_create(ctx.h, box.cpd, box.n, _ptr(self._cs), _ptr(box.x), _ptr(box.y),
                                  _ptr(box.z), ctypes.byref(h)), "nf_box_create")
        self.h = h

    def close(self):
        if self.h:
            lib().nf_box_destroy(self.ctx.h, self.h)
            self.h = None

    def update(self, x, y, z):
        check(lib().nf_box_update(self.ctx.h, self.h, _ptr(x), _ptr(y), _ptr(z)), "nf_box_update")

    def slab_particles(self, lo: int, hi: int) -> tuple[int, int]:
        c2 = self.cpd * self.cpd
        return int(self._cs[lo * c2]), int(self._cs[hi * c2])

    def record_width(self) -> int:
        return 4 if self.ctx.cfg.out_kind == OUT_FLOAT4 else 3

    def forces(self, lo: int = 0, hi: int | None = None, out: np.ndarray | None = None):
        """Accelerations of slabs [lo, hi) into host memory (float32[n, 3|4])."""
        hi = self.cpd if hi is None else hi
        p0, p1 = self.slab_particles(lo, hi)
        if out is None:
            out = np.empty((p1 - p0, self.record_width()), dtype=np.float32)
        check(lib().nf_box_forces(self.ctx.h, self.h, lo, hi, _ptr(out), 0), "nf_box_forces")
        return out

    def forces_device(self, lo: int, hi: int, dev_ptr: int):
        """Accelerations of slabs [lo, hi) into device memory at dev_ptr."""
        check(lib().nf_box_forces(self.ctx.h, self.h, lo, hi, ctypes.c_void_p(dev_ptr), 1),
              "nf_box_forces")

    def pair_count(self, lo: int = 0, hi: int | None = None) -> int:
        hi = self.cpd if hi is None else hi
        v = ctypes.c_uint64(0)
        check(lib().nf_box_pair_count(self.ctx.h, self.h, lo, hi, ctypes.byref(v)),
              "nf_box_pair_count")
        return int(v.value)

    def device_bytes(self) -> int:
        return int(lib().nf_box_device_bytes(self.h))
