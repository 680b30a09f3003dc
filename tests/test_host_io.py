"""Host text IO mirrored from app/io/header/io_views.hpp: load_view / write_part."""
import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg


def test_write_then_load_roundtrip(tmp_path):
    p = tmp_path / "part.txt"
    labels = np.array([4, 0, 2, 2, 1], np.int32)
    pg.write_part(labels, p)
    assert p.read_text() == "4\n0\n2\n2\n1\n"
    assert np.array_equal(pg.load_view(5, p, np.int32), labels)


def test_load_view_short_file_zero_fills_and_ignores_extra(tmp_path):
    p = tmp_path / "vw.txt"
    p.write_text("3 7\n 9\n")
    assert np.array_equal(pg.load_view(5, p), [3, 7, 9, 0, 0])
    assert np.array_equal(pg.load_view(2, p), [3, 7])
    assert np.array_equal(pg.load_view(2, p, np.float64), [3.0, 7.0])


def test_load_view_missing_file_raises(tmp_path):
    with pytest.raises(pg.InvalidArgument):
        pg.load_view(3, tmp_path / "absent.txt")
