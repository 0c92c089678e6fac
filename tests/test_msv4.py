"""The MSv4 reader feeding the gridder (rang.msv4 over include/rang_msv4.h).

* The codec: LZ4 blocks against hand-built blocks of the published format
  and against an independent LZ4 (pyarrow's liblz4) both ways; Blosc-1
  chunks against hand-built chunks (stored, split streams with byte shuffle,
  a short last block) and encoder round trips; refusals.
* The reader on the reference's own fixture (tests/golden/msv4_m05.zip, an
  xradio store and the MSv2 it was converted from): the reference's row
  layout (python/rang/msv4.py:307-349), and every value decoded from the
  store found byte for byte in the MSv2 storage files of the same
  observation (DATA and WEIGHT_SPECTRUM tiles, UVW buckets), so the decode
  is pinned to the data the reference's own test compares against.
* A written store with pads, several time chunks and multi-block chunks
  read back exactly.
* On the GPU: a partition's rows through Stokes I into the gridder, against
  the oracle and the direct Fourier transform.
"""

import ctypes
import zipfile
from pathlib import Path

import numpy as np
import pytest

import oracle
from cases import rel_linf

FIXTURE = Path(__file__).resolve().parent / "golden" / "msv4_m05.zip"


def _lib():
    from rang import msv4

    return msv4._library()


def _lz4(src, cap):
    lib = _lib()
    src = np.frombuffer(bytes(src), np.uint8)
    out = np.zeros(max(cap, 1), np.uint8)
    w = ctypes.c_size_t()
    st = lib.rang_b200_lz4_decode(src.ctypes.data, src.size, out.ctypes.data, cap, ctypes.byref(w))
    return st, bytes(out[:w.value])


def test_library_exports_every_msv4_symbol():
    import re

    from rang import core

    text = (Path(__file__).resolve().parents[1] / "include" / "rang_msv4.h").read_text()
    names = sorted(set(re.findall(r"^\w+\s+(rang_b200_\w+)\s*\(", text, re.M)))
    assert len(names) == 6
    lib = ctypes.CDLL(core.library_path())
    for name in names:
        assert hasattr(lib, name), name


def test_lz4_known_blocks():
    # Literals then an overlapping match: offset 3, length 9.
    assert _lz4([0x35, *b"abc", 3, 0, 0x00], 12) == (0, b"abcabcabcabc")
    # 20 literals: the count continues in one byte (15 + 5).
    lit = bytes(range(65, 85))
    assert _lz4([0xF0, 5, *lit], 20) == (0, lit)
    # A run: one literal, a match of offset 1 and length 4 + 15 + 255 + 10,
    # then 5 literals.
    block = [0x1F, ord("z"), 1, 0, 255, 10, 0x50, *b"tail!"]
    st, out = _lz4(block, 1 + 284 + 5)
    assert st == 0 and out == b"z" * 285 + b"tail!"
    # Malformed: offset 0, offset before the output, truncated, too long.
    assert _lz4([0x10, ord("a"), 0, 0], 10)[0] == 1
    assert _lz4([0x10, ord("a"), 2, 0], 10)[0] == 1
    assert _lz4([0x35, *b"ab"], 12)[0] == 1
    assert _lz4([0x35, *b"abc", 3, 0], 6)[0] == 1


def test_lz4_agrees_with_an_independent_lz4():
    import pyarrow

    lib = _lib()
    codec = pyarrow.Codec("lz4_raw")
    for seed in range(12):
        rng = np.random.default_rng(seed)
        n = int(rng.integers(0, 150000))
        kind = seed % 4
        if kind == 0:
            data = rng.integers(0, 3, n)
        elif kind == 1:
            data = rng.integers(0, 256, n)
        elif kind == 2:
            data = np.repeat(rng.integers(0, 256, n // 40 + 1), 40)[:n]
        else:
            data = np.tile(rng.integers(0, 256, 300), n // 300 + 1)[:n]
        data = data.astype(np.uint8)
        theirs = codec.compress(data.tobytes()).to_pybytes()
        assert _lz4(theirs, n) == (0, data.tobytes())
        out = np.zeros(n + n // 255 + 32, np.uint8)
        w = ctypes.c_size_t()
        assert lib.rang_b200_lz4_encode(data.ctypes.data, n, out.ctypes.data, out.size, ctypes.byref(w)) == 0
        assert codec.decompress(out[:w.value].tobytes(), decompressed_size=n).to_pybytes() == data.tobytes()


def _header(flags, typesize, nbytes, blocksize, cbytes):
    return bytes([2, 1, flags, typesize]) + np.array([nbytes, blocksize, cbytes], "<u4").tobytes()


def test_blosc_known_chunks():
    from rang import msv4

    # Stored (memcpyed): the data follows the header.
    payload = bytes(range(40))
    assert msv4.blosc_decode(_header(0x02, 4, 40, 40, 56) + payload).tobytes() == payload
    # One block of 256 int32 (1024 bytes), byte-shuffled and split into 4
    # streams of 256 bytes: stream j holds byte j of every element. Stream
    # 0 raw; streams 1-3 zeros as LZ4 (a literal zero and a match of 255).
    vals = np.arange(256, dtype="<i4")
    # 256 zero bytes: one literal, a match of length 250 (4 + 15 + 231), 5 literals.
    lz_zero = bytes([0x1F, 0, 1, 0, 231, 0x50, 0, 0, 0, 0, 0])
    streams = [np.array([256], "<u4").tobytes() + vals.astype(np.uint8).tobytes()]
    streams += [np.array([len(lz_zero)], "<u4").tobytes() + lz_zero] * 3
    body = b"".join(streams)
    start = 16 + 4
    chunk = _header(0x21, 4, 1024, 1024, start + len(body)) + np.array([start], "<u4").tobytes() + body
    assert np.array_equal(msv4.blosc_decode(chunk).view("<i4"), vals)
    # Two blocks, the last one short (never split): 300 bytes in blocks of 256.
    data = np.random.default_rng(3).integers(0, 256, 300).astype(np.uint8).tobytes()
    blocks = [np.array([256], "<u4").tobytes() + data[:256], np.array([44], "<u4").tobytes() + data[256:]]
    offs = [24, 24 + len(blocks[0])]
    chunk = _header(0x20, 1, 300, 256, 24 + sum(map(len, blocks))) + np.array(offs, "<u4").tobytes() + b"".join(blocks)
    assert msv4.blosc_decode(chunk).tobytes() == data
    # Refusals: bit shuffle, a zstd chunk, a truncated chunk.
    with pytest.raises(ValueError, match="does not decode"):
        msv4.blosc_decode(_header(0x24, 1, 8, 8, 32) + bytes(16), 8)
    with pytest.raises(ValueError, match="does not decode"):
        msv4.blosc_decode(_header(0x80, 1, 8, 8, 32) + bytes(16), 8)
    with pytest.raises(ValueError, match="malformed"):
        msv4.blosc_decode(chunk[:-10], 300)


@pytest.mark.parametrize("shuffle,split,blocksize", [(True, True, 4096), (False, False, 0), (True, False, 1000),
                                                      (False, True, 512)])
def test_blosc_round_trips(shuffle, split, blocksize):
    from rang import msv4

    rng = np.random.default_rng(blocksize)
    for data in (np.repeat(rng.integers(0, 5, 5000), 3).astype(np.float32), rng.standard_normal(3000),
                 np.zeros(10000, np.uint8), np.arange(100000, dtype=np.int64),
                 (rng.standard_normal(4096) + 1j).astype(np.complex64)):
        chunk = msv4.blosc_encode(data.tobytes(), data.itemsize, shuffle, split, blocksize)
        assert msv4.blosc_nbytes(chunk) == data.nbytes
        assert msv4.blosc_decode(chunk).tobytes() == data.tobytes()
    many = msv4.blosc_decode_many([chunk] * 7, [data.nbytes] * 7, threads=3)
    assert all(m.tobytes() == data.tobytes() for m in many)


def test_reader_layout_on_the_reference_fixture():
    from rang import msv4

    ps = msv4.open_processing_set(FIXTURE)
    names = ps.names()
    assert names == ["m05-var-spw-tssm_0", "m05-var-spw-tssm_1"]
    for name, nchan in zip(names, (4, 8)):
        p = ps.partition(name)
        assert p.polarization == ("XX", "XY", "YX", "YY")
        assert p.antenna_names == ["A0", "A1", "A2", "A3"]
        assert p.antenna1.tolist() == [0, 0, 0, 1, 1, 2] and p.antenna2.tolist() == [1, 2, 3, 2, 3, 3]
        assert p.weight_variable == "WEIGHT"
        assert np.all(np.diff(p.frequency) > 0) and len(p.frequency) == nchan
        r = p.rows()
        n = 3 * 6
        assert r["PADS"] == 0 and r["DATA"].shape == (n, nchan, 4) and r["DATA"].dtype == np.complex64
        assert r["FLAG"].dtype == np.bool_ and r["WEIGHT_SPECTRUM"].dtype == np.float32
        assert r["UVW"].shape == (n, 3) and not r["FLAG_ROW"].any()
        assert np.array_equal(r["TIME"], np.repeat(p.time_unix, 6) + msv4.UNIX_TO_MJD_SECONDS)
        assert list(r["FIELD_NAME"]) == ["F0_0"] * n and list(r["SCAN_NAME"]) == ["1"] * n
        chunks = list(p.chunks(time_rows=2))
        assert len(chunks) == 2 and np.array_equal(np.concatenate([c["DATA"] for c in chunks]), r["DATA"])


def test_decoded_values_are_the_msv2_bytes():
    from rang import msv4

    z = zipfile.ZipFile(FIXTURE)
    ms = {n.split("/")[-1]: z.read(n) for n in z.namelist() if n.startswith("m05.ms/table.")}  # main table
    ps = msv4.open_processing_set(FIXTURE)
    for name, cube in zip(ps.names(), ("TSM1", "TSM2")):
        r = ps.partition(name).rows()
        data, weight = ms["table.f0_" + cube], ms["table.f1_" + cube]
        nchan = r["DATA"].shape[1]
        step = min(nchan, 4)  # the MSv2 tiles hold 4 channels of a cell
        for i in range(len(r["UVW"])):
            assert r["UVW"][i].astype("<f8").tobytes() in ms["table.f2"]
            for c in range(0, nchan, step):
                assert r["DATA"][i, c:c + step].astype("<c8").tobytes() in data
                assert r["WEIGHT_SPECTRUM"][i, c:c + step].astype("<f4").tobytes() in weight


def _synthetic(ntime=6, nant=5, nchan=7, seed=0):
    rng = np.random.default_rng(seed)
    a1, a2 = np.triu_indices(nant, 1)
    nbl = len(a1)
    shape = (ntime, nbl, nchan, 4)
    vis = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    uvw = rng.standard_normal((ntime, nbl, 3)) * 300.0
    flag = rng.random(shape) > 0.8
    weight = rng.random(shape).astype(np.float32)
    vis[2, 3] = np.nan
    uvw[2, 3] = np.nan
    vis[4, 0, 0, 0] = np.nan  # a NaN sample in a real row keeps the row
    return {"time": 1.6e9 + 8.0 * np.arange(ntime), "frequency": 1e9 + 1e6 * np.arange(nchan),
            "polarization": ["XX", "XY", "YX", "YY"], "antenna_name": [f"m{i:03d}" for i in range(nant)],
            "antenna1": a1, "antenna2": a2, "VISIBILITY": vis, "FLAG": flag, "WEIGHT": weight, "UVW": uvw}


def test_written_store_reads_back(tmp_path):
    from rang import msv4

    p = _synthetic()
    msv4.write_processing_set(tmp_path / "ps.zarr", {"obs_0": p}, time_chunk=4, blocksize=512)
    part = msv4.open_processing_set(tmp_path / "ps.zarr").partition("obs_0")
    r = part.rows()
    nt, nbl = p["VISIBILITY"].shape[:2]
    keep = np.ones((nt, nbl), bool)
    keep[2, 3] = False
    assert r["PADS"] == 1 and len(r["UVW"]) == keep.sum()
    assert np.array_equal(r["DATA"], p["VISIBILITY"][keep], equal_nan=True)
    assert np.array_equal(r["FLAG"], p["FLAG"][keep])
    assert np.array_equal(r["WEIGHT_SPECTRUM"], p["WEIGHT"][keep])
    assert np.array_equal(r["UVW"], p["UVW"][keep])
    assert np.array_equal(r["ANTENNA1"], np.tile(p["antenna1"], nt)[keep.ravel()])
    assert part.antenna_names == p["antenna_name"]


@pytest.mark.gpu
def test_fixture_rows_feed_the_gridder():
    from rang import gridder, msv4

    part = msv4.open_processing_set(FIXTURE).partition("m05-var-spw-tssm_1")
    g = msv4.gridder_inputs(part)
    ovis, owgt = oracle.stokes_i(part.rows()["DATA"], part.rows()["WEIGHT_SPECTRUM"], part.rows()["FLAG"])
    assert np.array_equal(g["vis"], ovis) and np.array_equal(g["wgt"], owgt)
    nx = ny = 64
    dx = 2.0e-4
    common = dict(uvw=g["uvw"], freq=g["freq"], npix_x=nx, npix_y=ny, pixsize_x=dx, pixsize_y=dx)
    got = gridder.vis2dirty(vis=g["vis"], wgt=g["wgt"], mask=g["mask"], epsilon=1e-5, **common)
    want = oracle.vis2dirty(vis=g["vis"], wgt=g["wgt"], mask=g["mask"], epsilon=1e-5, **common)
    assert rel_linf(got, want) < 2e-5
    dft = oracle.dft_dirty(g["uvw"], g["freq"], g["vis"].astype(np.complex128) * g["wgt"] * g["mask"], nx, ny, dx, dx)
    assert rel_linf(got, dft) < 1e-4
