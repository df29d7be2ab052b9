"""Host side of the flag contract (0 = keep, any other value = flagged): the
imager's host API passes bool and uint8 flag arrays as one byte per flag
(mtb_grid_params.flags_u8) with their values kept, and every other integer
type as the reference's int32 layout.  The kernels treat any non-zero flag as
flagged (tests/test_byte_flags.py checks that on the GPU)."""
import numpy as np
import torch

from mtb.imager import _dev, _is_byte_flags


def test_byte_layout_for_bool_and_uint8():
    assert _is_byte_flags(np.zeros((2, 4), bool))
    assert _is_byte_flags(np.zeros((2, 4), np.uint8))
    assert _is_byte_flags(torch.zeros((2, 4), dtype=torch.bool))
    assert not _is_byte_flags(np.zeros((2, 4), np.int32))
    assert not _is_byte_flags(np.zeros((2, 4), np.int64))


def test_flag_values_are_kept_on_the_way_to_the_device():
    b = np.array([[True, False, True, False]])
    assert _dev(b, torch.uint8, "cpu").tolist() == [[1, 0, 1, 0]]
    i = np.array([[0, 1, 2, 255]], np.int64)
    assert _dev(i, torch.int32, "cpu").tolist() == [[0, 1, 2, 255]]


def test_packed_flags_layout_and_mode():
    """pack_flags puts flag i = r*P + p in bit i % 8 of byte i / 8 (numpy and
    torch agree); a uint8 tensor of ceil(R*P/8) bytes selects flags_u8 = 2,
    [R][P] bytes 1, int32 0."""
    from mtb.imager import _flags_u8, pack_flags
    rng = np.random.default_rng(4)
    fl = (rng.random((13, 4)) < 0.3).astype(np.uint8)
    fl[2, 1] = 7                                    # any non-zero value is a set bit
    packed = pack_flags(fl)
    assert packed.dtype == np.uint8 and packed.size == (13 * 4 + 7) // 8
    bits = np.unpackbits(packed, bitorder="little")[: 13 * 4].reshape(13, 4)
    assert np.array_equal(bits, (fl != 0).astype(np.uint8))
    assert np.array_equal(pack_flags(torch.from_numpy(fl)).numpy(), packed)
    assert _flags_u8(torch.from_numpy(packed), 13, 4) == 2
    assert _flags_u8(torch.from_numpy(fl), 13, 4) == 1
    assert _flags_u8(torch.from_numpy(fl.astype(np.int32)), 13, 4) == 0


def test_other_flag_modes_are_refused():
    import ctypes
    from mtb import _lib as L
    lib = L.load()
    gp = L.GridParams()
    gp.nx = gp.ny = 64
    gp.npol, gp.sampling, gp.wplanes = 4, 4, 4
    gp.u_increment = gp.v_increment = 1.0
    gp.w_sq_increment = 1.0
    info = (ctypes.c_int * 8)(7, 0, 7, 49, 7, 98, 7, 147)
    n = ctypes.c_size_t(0)
    gp.flags_u8 = 3
    assert lib.mtb_grid_workspace_size(ctypes.byref(gp), ctypes.cast(info, ctypes.c_void_p), 1000,
                                       ctypes.byref(n)) == L.MTB_ERR_BAD_PARAM
