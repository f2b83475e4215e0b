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
ABI_VERSION = 2  # NF_ABI_VERSION of include/nf_capi.h


class NfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("near_field_radius", ctypes.c_int),
                ("softening", ctypes.c_int), ("eps", ctypes.c_float), ("b2", ctypes.c_float),
                ("accumulation", ctypes.c_int), ("out_kind", ctypes.c_int),
                ("sinks_per_lane", ctypes.c_int), ("kernel_variant", ctypes.c_int)]


class Timing(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_float), ("coadd_ms", ctypes.c_float),
                ("total_ms", ctypes.c_float), ("pairs", ctypes.c_uint64),
                ("padded_pairs", ctypes.c_uint64), ("launches", ctypes.c_int),
                ("items", ctypes.c_int), ("variant", ctypes.c_int)]


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
                ("bytes_from_device", ctypes.c_void_p), ("node_z_start", ctypes.c_int),
                ("node_z_size", ctypes.c_int)]


CELLINFO_DTYPE = np.dtype([("startindex", "<u8"), ("startindex_with_ghost", "<u8"),
                           ("count", "<i4"), ("active", "<i4"),
                           ("mean_square_velocity", "<f4"), ("max_component_velocity", "<f4"),
                           ("max_component_acceleration", "<f4")], align=True)


class SlabView(ctypes.Structure):
    _fields_ = [("posxyz", ctypes.c_void_p), ("nslab", ctypes.c_uint64),
                ("cellinfo", ctypes.c_void_p), ("acc", ctypes.c_void_p)]


class DriverParams(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("cpd", ctypes.c_int), ("np", ctypes.c_int64),
                ("near_field_radius", ctypes.c_int), ("softening", ctypes.c_int),
                ("softening_length", ctypes.c_double), ("density_kernel_rad2", ctypes.c_float),
                ("direct_bpd", ctypes.c_int), ("mem_per_gpu_buffer_gb", ctypes.c_double),
                ("max_ram_mb", ctypes.c_double), ("use_pinned_gpu_memory", ctypes.c_int),
                ("accumulation", ctypes.c_int), ("out_kind", ctypes.c_int),
                ("node_z_start", ctypes.c_int), ("node_z_size", ctypes.c_int)]


class DriverStats(ctypes.Structure):
    _fields_ = [("direct_interactions", ctypes.c_uint64),
                ("padded_direct_interactions", ctypes.c_uint64),
                ("gdi_gpu", ctypes.c_double), ("gdi_padded_gpu", ctypes.c_double),
                ("total_gb_to", ctypes.c_double), ("total_gb_from", ctypes.c_double),
                ("total_sinks", ctypes.c_double), ("total_sources", ctypes.c_double),
                ("total_padded_sinks", ctypes.c_double), ("total_padded_sources", ctypes.c_double),
                ("mean_splits_per_slab", ctypes.c_double), ("max_nsplits", ctypes.c_int),
                ("gpu_throughput_time", ctypes.c_double), ("calc_split_s", ctypes.c_double),
                ("sic_construction_s", ctypes.c_double), ("sic_execute_s", ctypes.c_double),
                ("finalize_s", ctypes.c_double), ("softening_length_internal", ctypes.c_double),
                ("eps", ctypes.c_float), ("ngpu", ctypes.c_int), ("nbuffers", ctypes.c_int),
                ("max_sink_blocks", ctypes.c_int), ("max_source_blocks", ctypes.c_int)]


class SicSummary(ctypes.Structure):
    _fields_ = [("nsinksets", ctypes.c_int), ("nsourcesets", ctypes.c_int),
                ("nsinkblocks", ctypes.c_int), ("nsourceblocks", ctypes.c_int),
                ("interaction_count", ctypes.c_int), ("direct_total", ctypes.c_uint64),
                ("padded_direct_total", ctypes.c_uint64), ("sink_total", ctypes.c_uint64),
                ("source_total", ctypes.c_uint64), ("padded_sink_total", ctypes.c_uint64),
                ("padded_source_total", ctypes.c_uint64)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_inflight", ctypes.c_int),
                ("max_queued", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("admitted", ctypes.c_uint64),
                ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("rejected", ctypes.c_uint64), ("cancelled", ctypes.c_uint64),
                ("pairs", ctypes.c_uint64), ("busy_s", ctypes.c_double),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("queue_p50_ms", ctypes.c_double), ("queue_p99_ms", ctypes.c_double),
                ("max_concurrent", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_size_t),
                ("hbm_peak_bytes", ctypes.c_size_t)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int), ("slab", ctypes.c_int),
                ("slot", ctypes.c_int), ("pairs", ctypes.c_uint64),
                ("submit_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("run_ms", ctypes.c_double), ("total_ms", ctypes.c_double)]


class KickParams(ctypes.Structure):
    _fields_ = [("near_scale", ctypes.c_float), ("rescale", ctypes.c_float),
                ("kick1", ctypes.c_float), ("kick2", ctypes.c_float), ("b2", ctypes.c_float)]


# Every symbol the header declares; the loader checks each one is exported.
EXPORTS = {
    "nf_box_update_aos": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "nf_box_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "nf_box_kick": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(KickParams), ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p]),
    "nf_server_request_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64,
                                              ctypes.POINTER(RequestInfo)]),
    "nf_server_start": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerConfig),
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "nf_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_uint64)]),
    "nf_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64,
                                      ctypes.POINTER(ctypes.c_int)]),
    "nf_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]),
    "nf_server_cancel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "nf_server_stats_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    "nf_server_stats_reset": (ctypes.c_int, [ctypes.c_void_p]),
    "nf_server_stop": (None, [ctypes.c_void_p]),
    "nf_driver_create": (ctypes.c_int, [ctypes.POINTER(DriverParams),
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "nf_driver_set_slab": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                          ctypes.POINTER(SlabView)]),
    "nf_driver_execute_slab": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "nf_driver_slab_done": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "nf_driver_finalize": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "nf_driver_aggregate_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(DriverStats)]),
    "nf_driver_context": (ctypes.c_void_p, [ctypes.c_void_p]),
    "nf_driver_destroy": (None, [ctypes.c_void_p]),
    "nf_driver_plan_sic": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.POINTER(SicSummary),
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
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
    "nf_sic_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]),
    "nf_box_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "nf_box_update": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p]),
    "nf_box_destroy": (None, [ctypes.c_void_p, ctypes.c_void_p]),
    "nf_box_device_bytes": (ctypes.c_size_t, [ctypes.c_void_p]),
    "nf_box_set_eps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float]),
    "nf_box_forces": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
    "nf_box_pair_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]),
    "nf_last_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Timing)]),
    "nf_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "nf_forces_noalloc": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    "nf_kernel_variant_count": (ctypes.c_int, []),
    "nf_kernel_variant_name": (ctypes.c_char_p, [ctypes.c_int]),
    "nf_box_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
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
        if L.nf_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI version {L.nf_abi_version()}, this binding "
                               f"expects {ABI_VERSION}: rebuild it with abacus-public_b200/build.py")
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
        # positions: numpy arrays (host) or torch tensors (host or device)
        p = (lambda a: ctypes.c_void_p(a.data_ptr()) if hasattr(a, "data_ptr") else _ptr(a))
        check(lib().nf_box_create(ctx.h, box.cpd, box.n, _ptr(self._cs), p(box.x), p(box.y),
                                  p(box.z), ctypes.byref(h)), "nf_box_create")
        self.h = h

    def close(self):
        if self.h:
            lib().nf_box_destroy(self.ctx.h, self.h)
            self.h = None

    def update(self, x, y, z):
        check(lib().nf_box_update(self.ctx.h, self.h, _ptr(x), _ptr(y), _ptr(z)), "nf_box_update")

    def step(self, x, y, z, out: np.ndarray, n_chunks: int = 0):
        """Upload + full sweep + download, pipelined over slab chunks (host arrays)."""
        check(lib().nf_box_step(self.ctx.h, self.h, _ptr(x), _ptr(y), _ptr(z), _ptr(out), n_chunks),
              "nf_box_step")
        return out

    def update_aos(self, xyz):
        """New positions as (N, 3) float32 records (host array or device pointer)."""
        ptr = ctypes.c_void_p(xyz) if isinstance(xyz, int) else _ptr(np.ascontiguousarray(xyz))
        check(lib().nf_box_update_aos(self.ctx.h, self.h, ptr), "nf_box_update_aos")

    def kick(self, lo: int, hi: int, vel_ptr: int, far_ptr: int = 0, acc_ptr: int = 0,
             stats_ptr: int = 0, near_scale: float = 1.0, rescale: float = 1.0,
             kick1: float = 0.0, kick2: float = 0.0, b2: float = 0.0):
        """Near field of slabs [lo, hi) fused with the rescale/co-add with the far
        field and the two half kicks (device pointers; see nf_box_kick)."""
        k = KickParams(near_scale, rescale, kick1, kick2, b2)
        check(lib().nf_box_kick(self.ctx.h, self.h, lo, hi, ctypes.byref(k),
                                ctypes.c_void_p(far_ptr or None), ctypes.c_void_p(vel_ptr),
                                ctypes.c_void_p(acc_ptr or None), ctypes.c_void_p(stats_ptr or None)),
              "nf_box_kick")

    def update_device(self, x_ptr: int, y_ptr: int, z_ptr: int):
        """New positions from device arrays (same cell counts)."""
        check(lib().nf_box_update(self.ctx.h, self.h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                  ctypes.c_void_p(z_ptr)), "nf_box_update")

    def slab_particles(self, lo: int, hi: int) -> tuple[int, int]:
        c2 = self.cpd * self.cpd
        return int(self._cs[lo * c2]), int(self._cs[hi * c2])

    def record_width(self) -> int:
        return 4 if self.ctx.cfg.out_kind == OUT_FLOAT4 else 3

    def forces(self, lo: int = 0, hi: int | None = None, out: np.ndarray | None = None):
        """Accelerations of slabs [lo, hi) into host memory (float32[n, 3|4])."""
        hi = self.cpd if hi is None else hi
        if not (0 <= lo < hi <= self.cpd):
            # let the library report the bad range with its own status code
            dummy = np.empty(1, dtype=np.float32)
            check(lib().nf_box_forces(self.ctx.h, self.h, lo, hi, _ptr(dummy), 0), "nf_box_forces")
        p0, p1 = self.slab_particles(lo, hi)
        if out is None:
            out = np.empty((p1 - p0, self.record_width()), dtype=np.float32)
        check(lib().nf_box_forces(self.ctx.h, self.h, lo, hi, _ptr(out), 0), "nf_box_forces")
        return out

    def forces_device(self, lo: int, hi: int, dev_ptr: int):
        """Accelerations of slabs [lo, hi) into device memory at dev_ptr."""
        check(lib().nf_box_forces(self.ctx.h, self.h, lo, hi, ctypes.c_void_p(dev_ptr), 1),
              "nf_box_forces")

    def set_eps(self, eps: float):
        """The box's own softening parameter (nf_config.eps convention; 0 = the context's)."""
        check(lib().nf_box_set_eps(self.ctx.h, self.h, float(eps)), "nf_box_set_eps")

    def pair_count(self, lo: int = 0, hi: int | None = None) -> int:
        hi = self.cpd if hi is None else hi
        v = ctypes.c_uint64(0)
        check(lib().nf_box_pair_count(self.ctx.h, self.h, lo, hi, ctypes.byref(v)),
              "nf_box_pair_count")
        return int(v.value)

    def tuning(self) -> tuple[int, list[float]]:
        v = ctypes.c_int(-1)
        n = lib().nf_kernel_variant_count()
        ms = (ctypes.c_float * n)()
        check(lib().nf_box_tuning(self.h, ctypes.byref(v), ms, n), "nf_box_tuning")
        return v.value, list(ms)

    def device_bytes(self) -> int:
        return int(lib().nf_box_device_bytes(self.h))


class AbacusSlabs:
    """A box laid out the way abacus holds it: one PosXYZ array
    (X[n] | Y[n] | Z[n]), one cellinfo array (cpd*cpd cells, y-major) and one
    AccSlab (accstruct per particle) per x-slab
    (singlestep/DataModel/cellparticles.cpp:62-266)."""

    def __init__(self, box, record_width: int = 4):
        self.cpd = box.cpd
        c2 = box.cpd * box.cpd
        self.posxyz, self.cellinfo, self.acc, self.ranges = [], [], [], []
        for s in range(box.cpd):
            p0, p1 = int(box.cell_start[s * c2]), int(box.cell_start[(s + 1) * c2])
            self.ranges.append((p0, p1))
            self.posxyz.append(np.ascontiguousarray(
                np.concatenate([box.x[p0:p1], box.y[p0:p1], box.z[p0:p1]]), dtype=np.float32))
            ci = np.zeros(c2, dtype=CELLINFO_DTYPE)
            starts = box.cell_start[s * c2:(s + 1) * c2] - p0
            ci["startindex"] = starts
            ci["startindex_with_ghost"] = starts
            ci["count"] = np.diff(box.cell_start[s * c2:(s + 1) * c2 + 1])
            ci["active"] = ci["count"]
            self.cellinfo.append(ci)
            self.acc.append(np.zeros((p1 - p0, record_width), dtype=np.float32))

    def view(self, s: int) -> SlabView:
        return SlabView(self.posxyz[s].ctypes.data, self.ranges[s][1] - self.ranges[s][0],
                        self.cellinfo[s].ctypes.data, self.acc[s].ctypes.data)

    def gather_acc(self, n: int) -> np.ndarray:
        out = np.zeros((n, self.acc[0].shape[1]), dtype=np.float32)
        for (p0, p1), a in zip(self.ranges, self.acc):
            out[p0:p1] = a
        return out


class AbacusNodeSlabs:
    """One node of a 2D (x, z) split as abacus holds it: the node owns z cells
    [zs, zs + zn) of every slab; PosXYZ holds, row by row, the R ghost cells
    below, the primary cells and the R ghost cells above
    (startindex_with_ghost), AccSlab the primary cells only (startindex);
    cells outside [zs - R, zs + zn + R) are empty.  `mask` marks the
    particles whose accelerations this node produces."""

    def __init__(self, box, zs: int, zn: int, R: int = 2, record_width: int = 4):
        cpd = self.cpd = box.cpd
        c2 = cpd * cpd
        zcells = (zs + np.arange(-R, zn + R)) % cpd          # row order: ghosts, primary, ghosts
        primary = np.zeros(len(zcells), bool)
        primary[R:R + zn] = True
        self.posxyz, self.cellinfo, self.acc, self.maps, self.nslab = [], [], [], [], []
        self.mask = np.zeros(box.n, bool)
        cs = np.asarray(box.cell_start, np.int64)
        for s in range(cpd):
            cid = (s * c2 + np.arange(cpd)[:, None] * cpd + zcells[None, :]).ravel()
            a, n = cs[cid], cs[cid + 1] - cs[cid]             # (y, z-in-row) order
            prim = np.tile(primary, cpd)
            start_g = np.concatenate([[0], np.cumsum(n)[:-1]])
            npri = np.where(prim, n, 0)
            start_p = np.concatenate([[0], np.cumsum(npri)[:-1]])
            ci = np.zeros(c2, dtype=CELLINFO_DTYPE)
            local = cid - s * c2
            ci["startindex_with_ghost"][local] = start_g
            ci["startindex"][local] = start_p
            ci["count"][local] = n
            ci["active"][local] = n
            idx = np.repeat(a, n) + (np.arange(int(n.sum())) - np.repeat(start_g, n))
            amap = idx[np.repeat(prim, n)]
            self.mask[amap] = True
            self.posxyz.append(np.ascontiguousarray(
                np.concatenate([box.x[idx], box.y[idx], box.z[idx]]), dtype=np.float32))
            self.nslab.append(len(idx))
            self.cellinfo.append(ci)
            self.maps.append(amap)
            self.acc.append(np.zeros((max(len(amap), 1), record_width), dtype=np.float32))

    def view(self, s: int) -> SlabView:
        return SlabView(self.posxyz[s].ctypes.data, self.nslab[s], self.cellinfo[s].ctypes.data,
                        self.acc[s].ctypes.data)

    def gather_acc(self, n: int) -> np.ndarray:
        out = np.zeros((n, self.acc[0].shape[1]), dtype=np.float32)
        for m, a in zip(self.maps, self.acc):
            out[m] = a[:len(m)]
        return out


class Driver:
    """nf_driver: the NearFieldDriver mirror (device < 0: planner only).
    node_z = (node_z_start, node_z_size) runs one node of a 2D z-split."""

    def __init__(self, box, softening: int, softening_length: float, device: int = 0,
                 near_field_radius: int = 2, direct_bpd: int = 3, mem_gb: float = 0.0,
                 b2: float = 0.0, accumulation: int = ACC_COMPENSATED,
                 out_kind: int = OUT_FLOAT4, use_pinned: int = -1,
                 node_z: tuple[int, int] | None = None):
        zs, zn = node_z if node_z else (0, 0)
        p = DriverParams(device=device, cpd=box.cpd, np=box.n,
                         near_field_radius=near_field_radius, softening=softening,
                         softening_length=softening_length, density_kernel_rad2=b2,
                         direct_bpd=direct_bpd, mem_per_gpu_buffer_gb=mem_gb, max_ram_mb=0.0,
                         use_pinned_gpu_memory=use_pinned, accumulation=accumulation,
                         out_kind=out_kind, node_z_start=zs, node_z_size=zn)
        h = ctypes.c_void_p()
        check(lib().nf_driver_create(ctypes.byref(p), ctypes.byref(h)), "nf_driver_create")
        self.h = h
        self.box = box
        rw = 4 if out_kind == OUT_FLOAT4 else 3
        self.slabs = (AbacusNodeSlabs(box, zs, zn, near_field_radius, rw) if zn
                      else AbacusSlabs(box, rw))
        for s in range(box.cpd):
            v = self.slabs.view(s)
            check(lib().nf_driver_set_slab(self.h, s, ctypes.byref(v)), "nf_driver_set_slab")

    def close(self):
        if self.h:
            lib().nf_driver_destroy(self.h)
            self.h = None

    def execute_slab(self, slab: int, blocking: int = 0):
        check(lib().nf_driver_execute_slab(self.h, slab, blocking), "ExecuteSlab")

    def slab_done(self, slab: int) -> int:
        return lib().nf_driver_slab_done(self.h, slab)

    def finalize(self, slab: int):
        check(lib().nf_driver_finalize(self.h, slab), "Finalize")

    def stats(self) -> DriverStats:
        s = DriverStats()
        check(lib().nf_driver_aggregate_stats(self.h, ctypes.byref(s)), "AggregateStats")
        return s

    def sic_timing(self, reset: bool = False) -> tuple[float, int, int]:
        """(summed pencil-kernel ms, SICs, unpadded pairs) of the SICs run since
        the last reset."""
        ms, n, p = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().nf_sic_timing(lib().nf_driver_context(self.h), ctypes.byref(ms),
                                  ctypes.byref(n), ctypes.byref(p), int(reset)), "nf_sic_timing")
        return ms.value, int(n.value), int(p.value)

    def plan_sic(self, slab: int, jlow: int, jhigh: int):
        s = SicSummary()
        check(lib().nf_driver_plan_sic(self.h, slab, jlow, jhigh, ctypes.byref(s), None, None,
                                       None), "plan")
        a = np.zeros(s.nsinksets, np.int32)
        b = np.zeros(s.nsinkblocks, np.int32)
        c = np.zeros(s.nsourcesets, np.int32)
        check(lib().nf_driver_plan_sic(self.h, slab, jlow, jhigh, ctypes.byref(s),
                                       a.ctypes.data, b.ctypes.data, c.ctypes.data), "plan")
        return s, a, b, c

    def run_all(self, timeout_s: float = 600.0, blocking: int = 0):
        """ExecuteSlab for every slab, then SlabDone polling and Finalize (the
        NearForce -> Kick order of singlestep/Timestep/pipeline.cpp)."""
        import time
        for s in range(self.box.cpd):
            self.execute_slab(s, blocking)
        t0 = time.time()
        pending = set(range(self.box.cpd))
        while pending:
            for s in list(pending):
                d = self.slab_done(s)
                if d < 0:
                    raise NfError(NF_EDEVICE, f"slab {s} failed: {last_error()}")
                if d == 1:
                    self.finalize(s)
                    pending.discard(s)
            if pending:
                if time.time() - t0 > timeout_s:
                    raise NfError(NF_ETIMEDOUT, "slabs still in flight")
                time.sleep(0.001)
        return self.slabs.gather_acc(self.box.n)


class Server:
    """nf_server: slab requests over resident boxes, continuous admission."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int = 0, max_inflight: int = 2,
                 max_queued: int = 65536):
        self.ctx = ctx
        cfg = ServerConfig(hbm_budget_bytes, max_inflight, max_queued)
        h = ctypes.c_void_p()
        check(lib().nf_server_start(ctx.h, ctypes.byref(cfg), ctypes.byref(h)), "nf_server_start")
        self.h = h
        self._held = {}  # ticket -> host output array, kept alive until the ticket is waited on

    def submit(self, box: DeviceBox, slab: int, out, out_on_device: bool = False) -> int:
        """Queue slab `slab` of `box`; `out` is a host numpy array or a device pointer."""
        t = ctypes.c_uint64()
        ptr = out if out_on_device else out.ctypes.data
        check(lib().nf_server_submit(self.h, box.h, slab, ctypes.c_void_p(ptr),
                                     int(out_on_device), ctypes.byref(t)), "nf_server_submit")
        if not out_on_device:
            self._held[t.value] = out  # the library writes into it until completion
        return t.value

    def poll(self, ticket: int) -> int:
        s = ctypes.c_int()
        check(lib().nf_server_poll(self.h, ticket, ctypes.byref(s)), "nf_server_poll")
        return s.value

    def wait(self, ticket: int, timeout_s: float = 120.0):
        st = lib().nf_server_wait(self.h, ticket, int(timeout_s * 1e9))
        if st != NF_ETIMEDOUT:
            self._held.pop(ticket, None)  # finished (done, failed or cancelled)
        check(st, "nf_server_wait")

    def cancel(self, ticket: int):
        check(lib().nf_server_cancel(self.h, ticket), "nf_server_cancel")

    def info(self, ticket: int) -> RequestInfo:
        """The request's record: state, slot, submit time and its latency split."""
        r = RequestInfo()
        check(lib().nf_server_request_info(self.h, ticket, ctypes.byref(r)),
              "nf_server_request_info")
        return r

    def stats(self) -> ServerStats:
        s = ServerStats()
        check(lib().nf_server_stats_get(self.h, ctypes.byref(s)), "nf_server_stats_get")
        return s

    def reset_stats(self):
        check(lib().nf_server_stats_reset(self.h), "nf_server_stats_reset")

    def close(self):
        if self.h:
            lib().nf_server_stop(self.h)  # waits for what runs: the held arrays are free after
            self.h = None
            self._held.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
