"""Map.bin / nMap.bin format: 24-byte records, optional 64-byte header, round trips."""
import numpy as np

from conftest import GOLDEN
from midas_b200 import bin_io


def test_record_layout():
    assert bin_io.PXLIST_DTYPE.itemsize == 24
    assert [bin_io.PXLIST_DTYPE.fields[k][1] for k in ("y", "z", "frac", "deltaR", "areaWeight")] == [0, 4, 8, 16, 20]


def _sample():
    return bin_io.pack_records([(1.0, 2.0, 0.5, 0.1, 0.9), (3.0, 4.0, 0.25, -0.2, 0.7), (5.0, 6.0, 1.0, 0.0, 1.0)],
                               [[0, 1], [], [2]])


def test_roundtrip_without_header(tmp_path):
    pm = _sample()
    bin_io.write_map(tmp_path / "Map.bin", tmp_path / "nMap.bin", pxList=pm.pxList, counts=pm.counts,
                     offsets=pm.offsets)
    assert (tmp_path / "Map.bin").stat().st_size == 3 * 24
    back = bin_io.load_map(tmp_path / "Map.bin", tmp_path / "nMap.bin")
    assert back.map_header is None
    np.testing.assert_array_equal(back.pxList, pm.pxList)
    np.testing.assert_array_equal(back.counts, [2, 0, 1])
    np.testing.assert_array_equal(back.offsets, [0, 2, 2])


def test_roundtrip_with_header(tmp_path):
    pm = _sample()
    h = bin_io.MapHeader(param_hash=bytes(range(32)), q_mode=1, gradient_mode=1, wavelength=0.17)
    bin_io.write_map(tmp_path / "Map.bin", tmp_path / "nMap.bin", pxList=pm.pxList, counts=pm.counts,
                     offsets=pm.offsets, header=h)
    assert (tmp_path / "Map.bin").stat().st_size == 64 + 3 * 24
    back = bin_io.load_map(tmp_path / "Map.bin", tmp_path / "nMap.bin")
    assert back.map_header == h and back.nmap_header == h
    np.testing.assert_array_equal(back.pxList, pm.pxList)


def test_header_and_hash_match_reference_bytes():
    g = np.load(GOLDEN / "header.npz")
    params = eval(str(g["params"][0]))
    h = bin_io.compute_param_hash(**params)
    assert h == bytes(g["param_hash"])
    hdr = bin_io.MapHeader(param_hash=h, q_mode=0, gradient_mode=1, wavelength=0.172979)
    assert hdr.to_bytes() == bytes(g["header"])
    assert bin_io.MapHeader.from_bytes(bytes(g["header"])) == hdr


def test_truncated_map_is_rejected(tmp_path):
    (tmp_path / "Map.bin").write_bytes(b"\0" * 25)
    (tmp_path / "nMap.bin").write_bytes(b"\0" * 8)
    import pytest
    with pytest.raises(ValueError):
        bin_io.load_map(tmp_path / "Map.bin", tmp_path / "nMap.bin")
