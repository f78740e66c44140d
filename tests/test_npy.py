"""The .npy state format against the reference's own reader and writer
(LifeCore/IO/NpyWriter.cpp compiled for the CPU) and numpy: byte-identical
files, numpy round trips, and the same rejections of damaged files. No GPU."""
import numpy as np
import pytest

import life_simulation_b200 as lb
from oracle.lenia_oracle import RefLenia, ref_npy_read, ref_npy_write

pytestmark = pytest.mark.skipif(not RefLenia.available(), reason="oracle/_ref not built")

SHAPES = [(7, 5), (1080, 1920), (13,), (2, 3, 4), (1, 1), (0, 5)]


@pytest.mark.parametrize("shape", SHAPES)
def test_files_byte_identical_and_numpy_readable(tmp_path, shape):
    a = np.random.default_rng(0).random(shape).astype(np.float32)
    mine, ref = tmp_path / "mine.npy", tmp_path / "ref.npy"
    lb.npy_write(str(mine), a)
    ref_npy_write(str(ref), a)
    assert mine.read_bytes() == ref.read_bytes()
    assert np.array_equal(np.load(mine), a)
    assert np.array_equal(lb.npy_read(str(ref), shape), a)
    assert np.array_equal(ref_npy_read(str(mine), shape), a)


def test_numpy_written_files(tmp_path):
    a = np.random.default_rng(1).random((33, 17)).astype(np.float32)
    p = tmp_path / "np.npy"
    np.save(p, a)
    assert np.array_equal(lb.npy_read(str(p), a.shape), a)
    assert np.array_equal(ref_npy_read(str(p), a.shape), a)


def _both(path, shape):
    """(mine accepts, reference accepts)."""
    try:
        lb.npy_read(str(path), shape)
        m = True
    except lb.LeniaError:
        m = False
    try:
        ref_npy_read(str(path), shape)
        r = True
    except ValueError:
        r = False
    return m, r


def test_truncations_and_damage_rejected_like_the_reference(tmp_path):
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    good = tmp_path / "g.npy"
    lb.npy_write(str(good), a)
    raw = good.read_bytes()
    bad = tmp_path / "b.npy"
    for n in range(len(raw)):  # every truncation
        bad.write_bytes(raw[:n])
        assert _both(bad, (3, 4)) == (False, False), n
    damaged = [raw.replace(b"NUMPY", b"NUMPX"), raw[:6] + b"\x02" + raw[7:],
               raw.replace(b"'<f4'", b"'<f8'"), raw.replace(b"'<f4'", b"'>f4'"),
               raw.replace(b"(3, 4)", b"(4, 3)"), raw.replace(b"(3, 4)", b"(3, x)"),
               raw[:8] + b"\xff\xff" + raw[10:]]
    for d in damaged:
        bad.write_bytes(d)
        assert _both(bad, (3, 4)) == (False, False), d[:80]
    # Shape checked against the caller's.
    assert _both(good, (12,)) == (False, False) and _both(good, (3, 4)) == (True, True)
    # A Fortran-order array: the reference does not check the flag and would
    # read it transposed; this library rejects it.
    bad.write_bytes(raw.replace(b"'fortran_order': False", b"'fortran_order': True "))
    assert _both(bad, (3, 4)) == (False, True)
