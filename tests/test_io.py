"""The reference's file formats through the C ABI (host code, no GPU).

Fixtures (tests/golden/io_*, made by make_golden.py with the reference's own
Dataset::writeSources / writeTargets / readSources / readTargets and
tapas::util::RankCSV, built from its sources as oracle/_ref/io_ref):
* our writers produce the reference's files byte for byte;
* our readers return exactly what the reference's readers return from them,
  including across two successive calls that continue at the stream position;
* main.csv has the reference's fixed-width layout byte for byte.
"""
import pathlib

import numpy as np
import pytest

GDIR = pathlib.Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def fx():
    return np.load(GDIR / "io_formats.npz")


def test_writers_match_reference_bytes(tb, fx, tmp_path):
    v = fx["values"]
    tb.write_sources(tmp_path, 0, v[:, 0], v[:, 1], v[:, 2], v[:, 3])
    tb.write_targets(tmp_path, 0, v[:, 4:8])
    assert (tmp_path / "source0000.dat").read_bytes() == (GDIR / "io_source0000.dat").read_bytes()
    assert (tmp_path / "target0000.dat").read_bytes() == (GDIR / "io_target0000.dat").read_bytes()


def test_readers_match_reference(tb, fx, tmp_path):
    back = fx["readback"]
    n = len(back)
    for stem in ("source", "target"):
        (tmp_path / f"{stem}0003.dat").write_bytes((GDIR / f"io_{stem}0000.dat").read_bytes())
    h = n // 2
    x1, y1, z1, q1, pos = tb.read_sources(tmp_path, 3, h)
    x2, y2, z2, q2, pos2 = tb.read_sources(tmp_path, 3, n - h, position=pos)
    got = np.concatenate([np.stack([x1, y1, z1, q1], 1), np.stack([x2, y2, z2, q2], 1)])
    np.testing.assert_array_equal(got, back[:, :4])
    assert pos2 > pos > 0
    t1, p = tb.read_targets(tmp_path, 3, h)
    t2, _ = tb.read_targets(tmp_path, 3, n - h, position=p)
    np.testing.assert_array_equal(np.concatenate([t1, t2]), back[:, 4:8])


def test_round_trip_full_precision(tb, tmp_path):
    rng = np.random.default_rng(5)
    v = rng.standard_normal((100, 4)) * 10.0 ** rng.integers(-30, 30, (100, 4))
    tb.write_sources(tmp_path, 12, *v.T, digits=17)
    x, y, z, q, _ = tb.read_sources(tmp_path, 12, 100)
    np.testing.assert_array_equal(np.stack([x, y, z, q], 1), v)


def test_read_errors_are_statuses(tb, tmp_path):
    with pytest.raises(tb.TapasError) as e:
        tb.read_sources(tmp_path, 9, 10)
    assert e.value.code == -1 and "source0009.dat" in str(e.value)
    tb.write_sources(tmp_path, 9, [1.0], [2.0], [3.0], [4.0])
    with pytest.raises(tb.TapasError) as e:
        tb.read_sources(tmp_path, 9, 2)
    assert e.value.code == -1 and "fewer than 2" in str(e.value)


def test_main_csv_matches_reference_bytes(tb, fx, tmp_path):
    a = [str(s) for s in fx["csv_args"]]
    out = tmp_path / "main.csv"
    tb.write_main_csv(out, float(a[0]), float(a[1]), float(a[2]), float(a[3]), float(a[4]),
                      int(a[5]), int(a[6]))
    assert out.read_bytes() == (GDIR / "io_main.csv").read_bytes()
