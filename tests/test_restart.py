"""triples.restart reader/writer (program.F90:42-49,195-223)."""
import numpy as np
import pytest

from libcc_b200 import restart as R
from libcc_b200 import synthetic as S


@pytest.mark.parametrize("no,nu,size", [
    (4, 36, 1_120_144),     # water aug-cc-pVDZ: w1-ccsdt-accd-gamess-reference.out:1410
    (4, 87, 12_645_736),    # water aug-cc-pVTZ: w1-acct.good.gamess:3126
    (4, 167, 82_202_856),   # water aug-cc-pVQZ: w1-accq.o21538:8882
])
def test_size_formula_matches_recorded_files(no, nu, size):
    """The scratch-file sizes GAMESS printed for the reference's three water runs
    pin the record layout: 8-byte integers, 4-byte record markers."""
    assert R.restart_file_size(no, nu, marker=4) == size


@pytest.mark.parametrize("marker", [4, 8])
def test_round_trip(tmp_path, marker):
    inp = S.generate(3, 7, 5)
    f = tmp_path / "triples.restart"
    n = R.write(f, inp, marker=marker)
    assert n == R.restart_file_size(3, 7, marker=marker)
    back = R.read(f)
    assert (back.no, back.nu) == (3, 7)
    for a, b in zip(inp.arrays(), back.arrays()):
        assert np.array_equal(a, b)


def test_truncated_file_is_rejected(tmp_path):
    inp = S.generate(3, 5, 1)
    f = tmp_path / "triples.restart"
    R.write(f, inp)
    data = f.read_bytes()
    f.write_bytes(data[:-20])
    with pytest.raises(R.RestartFormatError):
        R.read(f)


def test_wrong_first_record_is_rejected(tmp_path):
    f = tmp_path / "bad.restart"
    f.write_bytes(b"\x04\x00\x00\x00abcd\x04\x00\x00\x00")
    with pytest.raises(R.RestartFormatError):
        R.read(f)


def test_gfortran_subrecords_round_trip(tmp_path):
    """Records longer than the subrecord limit are split the way gfortran splits
    records over 2 GiB (negative leading marker while more follow, negative
    trailing marker after the first); the reader joins them.  A small limit
    stands in for the 2,147,483,639-byte one."""
    inp = S.generate(3, 6, 8)
    f = tmp_path / "triples.restart"
    n = R.write(f, inp, marker=4, max_sub=100)
    assert n == R.restart_file_size(3, 6, marker=4, max_sub=100) > R.restart_file_size(3, 6, marker=4)
    data = f.read_bytes()
    import struct
    # record 3 (eh, 24 bytes) is whole; record 6 (t2, 2592 bytes) starts with a continued subrecord
    assert struct.unpack_from("<i", data, 0)[0] == 8
    back = R.read(f)
    for a, b in zip(inp.arrays(), back.arrays()):
        assert np.array_equal(a, b)


def test_subrecord_with_bad_trailer_is_rejected(tmp_path):
    inp = S.generate(3, 6, 8)
    f = tmp_path / "triples.restart"
    R.write(f, inp, marker=4, max_sub=100)
    data = bytearray(f.read_bytes())
    # the first subrecord of the t1 record (3rd payload after no, nu, eh, ep): find the
    # first negative leading marker and flip the sign of its trailer
    import struct
    pos = 0
    while True:
        (h,) = struct.unpack_from("<i", data, pos)
        if h < 0:
            struct.pack_into("<i", data, pos + 4 + (-h), h)
            break
        pos += 8 + h
    f.write_bytes(bytes(data))
    with pytest.raises(R.RestartFormatError):
        R.read(f)
