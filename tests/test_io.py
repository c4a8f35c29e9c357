"""GHOST's field file names (ghost_io_filename, host only): dir/name.NNNN.out
with the index zero-padded to the fmtext width (pseudospec3D_mod.fpp:40),
and Fortran's asterisks for an index wider than the field."""
import pytest


def test_filename_default_width():
    from ghost_b200 import io_filename
    assert io_filename("out", "vx", 7) == "out/vx.0007.out"
    assert io_filename("/scratch/run", "th", 1234) == "/scratch/run/th.1234.out"


def test_filename_widths():
    from ghost_b200 import io_filename
    assert io_filename("d", "wz", 3, 6) == "d/wz.000003.out"
    assert io_filename("d", "vx", 12345, 4) == "d/vx.****.out"
    assert io_filename("d", "vx", 0, 1) == "d/vx.0.out"


def test_filename_errors():
    from ghost_b200 import GhostError, io_filename
    with pytest.raises(GhostError) as e:
        io_filename("d", "vx", -1)
    assert e.value.code == 1
    with pytest.raises(GhostError):
        io_filename("d", "vx", 1, 0)
