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
