"""The C-ABI library loads and exports what include/nf_capi.h declares.
(No device calls: these run without a GPU.)"""
import ctypes


def test_library_exports_every_declared_symbol(capi):
    L = ctypes.CDLL(str(capi.LIB_PATH))
    declared = capi.declared_symbols()
    assert len(declared) >= 15
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert set(declared) == set(capi.EXPORTS), set(declared) ^ set(capi.EXPORTS)


def test_abi_version_and_defaults(capi):
    assert capi.lib().nf_abi_version() == capi.ABI_VERSION == 2
    c = capi.default_config()
    assert c.near_field_radius == 2
    assert c.softening == capi.SOFT_SINGLE_SPLINE
    assert c.accumulation == capi.ACC_COMPENSATED
    assert c.out_kind == capi.OUT_FLOAT4


def test_library_is_sm100a_only(capi):
    """The fatbin inside the library carries sm_100a code (checked through the
    build recipe's flags, not by reading the binary)."""
    from abacus_public_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_noalloc_rejects_boxes_beyond_32_bit_pencil_ids(capi):
    """cpd^3 must stay below 2^31 (pencil ids are 32-bit): the call refuses
    cpd = 1291 before it touches the device, so this runs without a GPU."""
    cfg = capi.default_config(softening=0, eps=1e-6)
    dummy = ctypes.c_void_p(16)
    rc = capi.lib().nf_forces_noalloc(ctypes.byref(cfg), 1291, dummy, dummy, 0, 1, dummy,
                                      ctypes.c_void_p(0))
    assert rc == capi.NF_EINVAL
    assert b"1290" in capi.lib().nf_last_error()
