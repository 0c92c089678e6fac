"""The MSv2 (casacore table) reader (rang.msv2), on the reference's own
fixtures (tests/golden/make_ms_fixtures.py):

* the two-window MS the reference's MSv4 fixture was converted from: every
  column the path needs read by rang.msv2 equals what rang.msv4 decodes from
  the converted store, bit for bit (the reference's own check of its two
  readers, its tests/test_msv4.py:1-13);
* the reference's MSv2 edge-case tables against its oracle.json: cells of
  four shapes in a TiledCellStMan, IncrementalStMan scalars and arrays,
  string scalars and arrays of every storage form;
* on the GPU, a data description's rows through Stokes I into the gridder:
  the same gridder inputs as the MSv4 path, bit for bit, and the same dirty
  image to float32 rounding.
"""

import json
import zipfile
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def tables(tmp_path_factory):
    root = tmp_path_factory.mktemp("ms")
    zipfile.ZipFile(GOLDEN / "msv4_m05.zip").extractall(root)
    zipfile.ZipFile(GOLDEN / "msv2_edge.zip").extractall(root / "edge")
    return root


def _sorted(r):
    k = np.lexsort((r["ANTENNA2"], r["ANTENNA1"], r["TIME"]))
    return {key: (v[k] if isinstance(v, np.ndarray) and v.ndim and len(v) == len(k) else v) for key, v in r.items()}


def test_main_table_description(tables):
    from rang import msv2

    t = msv2.Table(tables / "m05.ms")
    assert t.nrows == 36 and t.little
    assert t.columns["UVW"].direct and t.columns["UVW"].shape == [3]
    assert not t.columns["FLAG"].direct and t.columns["DATA"].is_array
    kinds = {type(m).__name__ if not isinstance(m, str) else m for m in t.managers.values()}
    assert kinds == {"_Ssm", "_Tsm"}
    assert sorted(set(t.read("DATA_DESC_ID").tolist())) == [0, 1]
    assert t.read("UVW", 5, 3).shape == (3, 3)


@pytest.mark.parametrize("ddid", [0, 1])
def test_msv2_equals_the_converted_msv4_store(tables, ddid):
    from rang import msv2, msv4

    ps = msv4.open_processing_set(GOLDEN / "msv4_m05.zip")
    part = ps.partition(ps.names()[ddid])
    a = _sorted(msv2.rows(tables / "m05.ms", ddid))
    b = _sorted(part.rows())
    for key in ("DATA", "FLAG", "WEIGHT_SPECTRUM", "UVW", "ANTENNA1", "ANTENNA2", "TIME", "FLAG_ROW"):
        assert a[key].dtype == b[key].dtype, key
        assert np.array_equal(a[key], b[key]), key
    assert np.array_equal(a["frequency"], part.frequency)
    assert a["polarization"] == part.polarization
    assert list(a["SCAN_NAME"]) == list(b["SCAN_NAME"])
    # xradio names a field by its MSv2 name and id ("F0" of FIELD row 0 -> "F0_0")
    fid = msv2.Table(tables / "m05.ms").read("FIELD_ID")
    assert all(f"{x}_{i}" == y for x, i, y in zip(a["FIELD_NAME"], fid, b["FIELD_NAME"]))


def test_row_counts_come_from_the_lock_record(tables):
    from rang import msv2

    field = msv2.Table(tables / "m05.ms" / "FIELD")
    assert field.nrows == 1 and list(field.read("NAME")) == ["F0"]


def test_edge_tables_against_the_reference_oracle(tables):
    from rang import msv2

    oracle = json.loads((tables / "edge" / "oracle.json").read_text())["tables"]
    cells = oracle["t05-tcellsm"]["columns"]["F32"]
    t = msv2.Table(tables / "edge" / "t05-tcellsm")
    assert t.nrows == oracle["t05-tcellsm"]["nrows"] == 4
    for row, want in enumerate(cells):
        got = t.read("F32", row, 1)[0]
        assert got.dtype == np.float32 and list(got.shape) == want["shape"]
        assert np.array_equal(got, np.asarray(want["values"], np.float32).reshape(want["shape"]))
    # IncrementalStMan: runs of rows sharing a value, scalars and an array.
    ism = oracle["t06-ism"]
    t = msv2.Table(tables / "edge" / "t06-ism")
    for name in ("I32", "F64", "B", "ARR"):
        whole = t.read(name)
        for row, want in enumerate(ism["columns"][name]):
            w = np.asarray(want["values"], want["dtype"]).reshape(want["shape"])
            assert np.array_equal(t.read(name, row, 1)[0], w) and np.array_equal(whole[row], w), (name, row)
    assert list(t.read("S")) == [c["values"][0] for c in ism["columns"]["S"]]
    # Strings: a variable-shape array (cells undefined in some rows), a
    # fixed-shape indirect array, a direct array (StandardStMan) and an
    # IncrementalStMan array.
    strings = oracle["t07-strings"]
    t = msv2.Table(tables / "edge" / "t07-strings")
    for name in ("VAR", "FIXED", "DIRECT", "ISM"):
        for row, want in enumerate(strings["columns"][name]):
            if want is None:
                with pytest.raises(ValueError, match="no array"):
                    t.read(name, row, 1)
                continue
            got = t.read(name, row, 1)[0]
            assert list(got.shape) == want["shape"] and list(got.reshape(-1)) == want["values"], (name, row)


def test_bad_tables_are_refused(tables, tmp_path):
    from rang import msv2

    bad = tmp_path / "bad.ms"
    bad.mkdir()
    (bad / "table.dat").write_bytes(b"\x00" * 64)
    with pytest.raises(ValueError, match="magic"):
        msv2.Table(bad)
    with pytest.raises(ValueError, match="no rows"):
        msv2.rows(tables / "m05.ms", 7)
    with pytest.raises(KeyError):
        msv2.Table(tables / "m05.ms").read("NO_SUCH_COLUMN")


@pytest.mark.gpu
def test_msv2_rows_feed_the_gridder_like_msv4(tables):
    from rang import gridder, msv2, msv4

    # The gridder's inputs are equal bit for bit; its float atomics make two
    # runs agree to rounding, not bit for bit.
    ps = msv4.open_processing_set(GOLDEN / "msv4_m05.zip")
    inputs, images = [], []
    for source in (msv2.DataDescription(tables / "m05.ms", 1), ps.partition(ps.names()[1])):
        r = _sorted(source.rows())
        g = msv4.gridder_inputs(source, r)
        inputs.append(g)
        images.append(gridder.vis2dirty(uvw=g["uvw"], freq=g["freq"], vis=g["vis"], wgt=g["wgt"],
                                              mask=g["mask"], npix_x=64, npix_y=64, pixsize_x=2e-4,
                                              pixsize_y=2e-4, epsilon=1e-5))
    for key in ("uvw", "freq", "vis", "wgt", "mask"):
        assert np.array_equal(inputs[0][key], inputs[1][key]), key
    assert np.abs(images[0]).max() > 0
    assert np.abs(images[0] - images[1]).max() <= 1e-6 * np.abs(images[1]).max()
