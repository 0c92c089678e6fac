"""MSv4 processing sets into the gridder's layouts: the reference's
`rang.msv4` reader (python/rang/msv4.py) without xarray, zarr or numcodecs.

A processing set is a zarr v3 group (a directory or a .zip) of MSv4
partitions, each a group whose attributes name its data groups. Arrays are
read chunk by chunk: `bytes` (endianness) then `blosc` (this library's
Blosc-1/LZ4 codec, include/rang_msv4.h, threaded over chunks) or `zstd`
(pyarrow's codec); missing chunks take the fill value. A partition yields
row chunks in the reference's layout (msv4.py:1-43, `Partition.rows`
:307-349):

- `TIME`: MJD seconds, the MSv4 `time` (Unix seconds) plus 3506716800 s;
- `ANTENNA1`, `ANTENNA2`: int32 indices into the partition's
  `antenna_xds.antenna_name`;
- `FLAG_ROW`: false (MSv4 has no row flag);
- `DATA` complex64, `FLAG` bool, `WEIGHT_SPECTRUM` float32, each
  `(row, channel, corr)`, from the data group's correlated data and flag and
  the partition's weight W; `UVW` float64 `(row, 3)`. A uint8 `FLAG` is read
  as bool when every value is 0 or 1 and refused otherwise;
- `FIELD_NAME`, `SCAN_NAME`: the per-time names, per row; `PADS` the pad
  cells dropped.

Rows are time-major in `baseline_id` order; a (time, baseline) cell whose
`UVW` and `VISIBILITY` are all NaN is a pad and is dropped. W follows the
reference's rule (msv4.py:172-215): the one weight variable every data group
names, or for an xradio partition with a `corrected` group that group's.

`gridder_inputs` turns rows into what the gridder takes (uvw, frequencies,
Stokes I visibilities and weights on the GPU, the flag mask), and
`write_processing_set` writes a store in the same layout (blosc/LZ4 data,
zstd coordinates) for tests and benchmarks.
"""

import base64
import ctypes
import json
import os
import zipfile
from pathlib import Path

import numpy as np

from . import core

UNIX_TO_MJD_SECONDS = 3506716800.0
GRID = ("time", "baseline_id", "frequency", "polarization")
DTYPES = {
    "correlated_data": (np.dtype("complex64"),),
    "flag": (np.dtype("bool"), np.dtype("uint8")),
    "weight": (np.dtype("float32"),),
    "uvw": (np.dtype("float64"),),
}
_NUMERIC = {"bool": "?", "int8": "i1", "int16": "i2", "int32": "i4", "int64": "i8", "uint8": "u1", "uint16": "u2",
            "uint32": "u4", "uint64": "u8", "float32": "f4", "float64": "f8", "complex64": "c8", "complex128": "c16"}

# ------------------------------------------------------------------ codec

_lib = None


def _library():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(core.library_path())
        P, S, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32
        lib.rang_b200_blosc_header.argtypes = [P, S, ctypes.POINTER(S), ctypes.POINTER(S), ctypes.POINTER(S),
                                               ctypes.POINTER(I), ctypes.POINTER(I)]
        lib.rang_b200_blosc_decode.argtypes = [P, S, P, S]
        lib.rang_b200_blosc_encode.argtypes = [P, S, I, I, I, S, P, S, ctypes.POINTER(S)]
        lib.rang_b200_blosc_decode_many.argtypes = [S, P, P, P, P, I, P]
        lib.rang_b200_lz4_decode.argtypes = [P, S, P, S, ctypes.POINTER(S)]
        lib.rang_b200_lz4_encode.argtypes = [P, S, P, S, ctypes.POINTER(S)]
        for f in (lib.rang_b200_blosc_header, lib.rang_b200_blosc_decode, lib.rang_b200_blosc_encode,
                  lib.rang_b200_blosc_decode_many, lib.rang_b200_lz4_decode, lib.rang_b200_lz4_encode):
            f.restype = I
        _lib = lib
    return _lib


def _status(code, what):
    if code == 3:
        raise ValueError(f"{what}: a Blosc chunk this reader does not decode (bit shuffle or a codec other than LZ4)")
    if code != 0:
        raise ValueError(f"{what}: malformed Blosc chunk")


def blosc_nbytes(chunk):
    """The decoded size of a Blosc-1 chunk (bytes)."""
    src = np.frombuffer(chunk, np.uint8)
    n = ctypes.c_size_t()
    code = _library().rang_b200_blosc_header(src.ctypes.data, src.size, ctypes.byref(n), None, None, None, None)
    if code == 1:
        raise ValueError("malformed Blosc chunk")
    return n.value


def blosc_decode(chunk, nbytes=None):
    """A Blosc-1 chunk as bytes (a numpy uint8 array)."""
    src = np.frombuffer(chunk, np.uint8)
    n = blosc_nbytes(chunk) if nbytes is None else nbytes
    out = np.empty(n, np.uint8)
    _status(_library().rang_b200_blosc_decode(src.ctypes.data, src.size, out.ctypes.data, out.size), "decode")
    return out


def blosc_decode_many(chunks, sizes, threads=None, outs=None):
    """Chunks decoded on `threads` host threads (default: all cores), into
    new arrays or into `outs` (contiguous uint8 arrays of `sizes` bytes)."""
    n = len(chunks)
    if outs is None:
        outs = [np.empty(s, np.uint8) for s in sizes]
    if n == 0:
        return outs
    srcs = [np.frombuffer(c, np.uint8) for c in chunks]
    sp = (ctypes.c_void_p * n)(*[s.ctypes.data for s in srcs])
    sl = (ctypes.c_size_t * n)(*[s.size for s in srcs])
    dp = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
    dl = (ctypes.c_size_t * n)(*[o.size for o in outs])
    st = (ctypes.c_int32 * n)()
    worst = _library().rang_b200_blosc_decode_many(n, sp, sl, dp, dl, int(threads or os.cpu_count() or 1), st)
    _status(worst, "decode")
    return outs


def blosc_encode(data, typesize, shuffle=True, split=False, blocksize=0):
    """`data` (bytes-like) as a Blosc-1 chunk with LZ4 blocks."""
    src = np.frombuffer(memoryview(data).cast("B"), np.uint8)
    nb = 1 if not blocksize else -(-src.size // blocksize)
    out = np.empty(src.size + 16 + 4 * nb + 64, np.uint8)
    w = ctypes.c_size_t()
    code = _library().rang_b200_blosc_encode(src.ctypes.data, src.size, int(typesize), int(bool(shuffle)),
                                             int(bool(split)), int(blocksize), out.ctypes.data, out.size,
                                             ctypes.byref(w))
    if code:
        raise ValueError("Blosc encoding failed")
    return out[:w.value].tobytes()


def _zstd():
    import pyarrow

    return pyarrow.Codec("zstd")


# ------------------------------------------------------------------ zarr v3


class Store:
    """A zarr store: a directory, or a .zip holding one (its root is the
    first directory with a group `zarr.json`)."""

    def __init__(self, source):
        self.source = source
        p = Path(source)
        self._zip = None
        if p.is_file() and zipfile.is_zipfile(p):
            self._zip = zipfile.ZipFile(p)
            names = self._zip.namelist()
            roots = sorted((n[:-len("zarr.json")] for n in names if n.endswith("zarr.json")), key=len)
            self._names = set(names)
            self.root = roots[0] if roots else ""
        elif p.is_dir():
            self.root = str(p) + "/"
        else:
            raise FileNotFoundError(f"no zarr store at {source}")

    def get(self, key):
        """The bytes at `key` (relative to the root), or None."""
        full = self.root + key
        if self._zip is not None:
            return self._zip.read(full) if full in self._names else None
        try:
            with open(full, "rb") as f:
                return f.read()
        except FileNotFoundError:
            return None

    def json(self, key):
        raw = self.get(key)
        return None if raw is None else json.loads(raw)


def _dtype(spec):
    if isinstance(spec, str):
        if spec not in _NUMERIC:
            raise ValueError(f"zarr data type {spec!r} is not read")
        return np.dtype("<" + _NUMERIC[spec]) if spec != "bool" else np.dtype("?")
    if spec.get("name") == "fixed_length_utf32":
        return np.dtype(f"<U{spec['configuration']['length_bytes'] // 4}")
    raise ValueError(f"zarr data type {spec!r} is not read")


def _fill(value, dtype):
    if dtype.kind == "U":
        return value if isinstance(value, str) else ""
    if dtype.kind == "c":
        re, im = value if isinstance(value, (list, tuple)) else (value, 0.0)
        return complex(_fill(re, np.dtype("f8")), _fill(im, np.dtype("f8")))
    if isinstance(value, str):
        special = {"NaN": np.nan, "Infinity": np.inf, "-Infinity": -np.inf}
        if value in special:
            return special[value]
        if value.startswith("0x"):
            return np.frombuffer(int(value, 16).to_bytes(dtype.itemsize, "big")[::-1], dtype)[0]
        return np.frombuffer(base64.b64decode(value), dtype)[0]
    return value


class Array:
    """A zarr v3 array node: shape, dtype, regular chunks, codecs."""

    def __init__(self, store, path, meta):
        self.store, self.path, self.meta = store, path, meta
        self.shape = tuple(int(s) for s in meta["shape"])
        self.dtype = _dtype(meta["data_type"])
        grid = meta["chunk_grid"]
        if grid.get("name") != "regular":
            raise ValueError(f"{path}: chunk grid {grid.get('name')!r} is not read")
        self.chunks = tuple(int(c) for c in grid["configuration"]["chunk_shape"])
        enc = meta.get("chunk_key_encoding", {"name": "default"})
        self._v2 = enc.get("name") == "v2"
        self._sep = enc.get("configuration", {}).get("separator", "." if self._v2 else "/")
        self.fill_value = _fill(meta.get("fill_value"), self.dtype)
        self.dims = tuple(meta.get("dimension_names") or ())
        self.attrs = meta.get("attributes", {})
        self.codecs = meta.get("codecs", [])
        names = [c["name"] for c in self.codecs]
        if not names or names[0] != "bytes" or any(n not in ("bytes", "blosc", "zstd") for n in names) or len(names) > 2:
            raise ValueError(f"{path}: codecs {names} are not read")
        endian = (self.codecs[0].get("configuration") or {}).get("endian", "little")
        if endian == "big":
            self.dtype = self.dtype.newbyteorder(">")
        self.compressor = names[1] if len(names) == 2 else None

    def _key(self, idx):
        if self._v2:
            return self.path + "/" + self._sep.join(str(i) for i in idx)
        return self.path + "/c" + "".join(self._sep + str(i) for i in idx) if idx else self.path + "/c"

    def read(self, threads=None):
        """The whole array as a numpy array. Chunks that span every axis but
        the first are decoded straight into the result."""
        if 0 in self.shape:
            return np.full(self.shape, self.fill_value, dtype=self.dtype)
        grid = [-(-s // c) for s, c in zip(self.shape, self.chunks)]
        idxs = list(np.ndindex(*grid)) if self.shape else [()]
        raw, where = [], []
        for idx in idxs:
            data = self.store.get(self._key(idx))
            if data is not None:
                raw.append(data)
                where.append(idx)
        if len(raw) < len(idxs):
            out = np.full(self.shape, self.fill_value, dtype=self.dtype)
        else:
            out = np.empty(self.shape, dtype=self.dtype)
        nbytes = int(np.prod(self.chunks, dtype=np.int64)) * self.dtype.itemsize
        slab = len(self.shape) > 0 and tuple(self.chunks[1:]) == tuple(self.shape[1:])
        dsts, inplace = [], []
        for idx in where:
            lo = idx[0] * self.chunks[0] if self.shape else 0
            direct = self.compressor == "blosc" and slab and lo + self.chunks[0] <= self.shape[0]
            dsts.append(out[lo:lo + self.chunks[0]].reshape(-1).view(np.uint8) if direct else np.empty(nbytes, np.uint8))
            inplace.append(direct)
        if self.compressor == "blosc":
            decoded = blosc_decode_many(raw, [nbytes] * len(raw), threads, dsts)
        elif self.compressor == "zstd":
            z = _zstd()
            decoded = [np.frombuffer(z.decompress(r, decompressed_size=nbytes), np.uint8) for r in raw]
        else:
            decoded = [np.frombuffer(r, np.uint8) for r in raw]
        for idx, buf, direct in zip(where, decoded, inplace):
            if buf.size != nbytes:
                raise ValueError(f"{self.path}: chunk {idx} holds {buf.size} bytes, expected {nbytes}")
            if direct:
                continue
            block = buf.view(self.dtype).reshape(self.chunks)
            sl = tuple(slice(i * c, min((i + 1) * c, s)) for i, c, s in zip(idx, self.chunks, self.shape))
            out[sl] = block[tuple(slice(0, s.stop - s.start) for s in sl)]
        return out.astype(self.dtype.newbyteorder("="), copy=False)


class Group:
    """A zarr v3 group: attributes and members (from consolidated metadata
    where the store has it)."""

    def __init__(self, store, path, meta, members):
        self.store, self.path, self.meta = store, path, meta
        self.attrs = meta.get("attributes", {})
        self._members = members

    def __contains__(self, name):
        return name in self._members

    def __getitem__(self, name):
        meta, sub = self._members[name]
        path = (self.path + "/" if self.path else "") + name
        if meta.get("node_type") == "array":
            return Array(self.store, path, meta)
        return Group(self.store, path, meta, sub)

    def names(self):
        return list(self._members)


def _members(store, path, meta):
    """{name: (meta, members)} of a group, from its consolidated metadata or
    by reading each listed child's zarr.json."""
    cm = (meta.get("consolidated_metadata") or {}).get("metadata")
    if cm is None:
        raise ValueError(f"{path or 'the store'}: no consolidated metadata (write it with zarr's consolidate)")
    tree = {}
    for key in sorted(cm, key=lambda k: k.count("/")):
        parts = key.split("/")
        node = tree
        for p in parts[:-1]:
            node = node.setdefault(p, ({}, {}))[1]
        prev = node.get(parts[-1], (None, {}))[1]
        node[parts[-1]] = (cm[key], prev)
    return tree


def open_group(source):
    store = source if isinstance(source, Store) else Store(source)
    meta = store.json("zarr.json")
    if meta is None or meta.get("node_type") != "group" or meta.get("zarr_format") != 3:
        raise ValueError(f"{store.source}: not a zarr v3 group")
    return Group(store, "", meta, _members(store, "", meta))


# ------------------------------------------------------------------ processing sets


def open_processing_set(source):
    """The processing set at `source` (a directory or .zip)."""
    return ProcessingSet(open_group(source))


class ProcessingSet:
    def __init__(self, group):
        self.group = group

    def names(self):
        """The partitions (MSv4 visibility groups), in store order."""
        out = []
        for n in self.group.names():
            node = self.group[n]
            if isinstance(node, Group) and node.attrs.get("type") in ("visibility", "spectrum") and \
                    "data_groups" in node.attrs:
                out.append(n)
        return out

    def partition(self, name, data_group="base"):
        return Partition(self.group[name], name, data_group)


class Partition:
    """One MSv4 of a processing set: its grid and its rows (the reference's
    `Partition`, msv4.py:135-349)."""

    def __init__(self, node, name, data_group="base"):
        self.name, self.node = name, node
        groups = node.attrs["data_groups"]
        if data_group not in groups:
            raise ValueError(f"{name}: no data group {data_group!r} in {list(groups)}")
        group = groups[data_group]
        self.data_group = data_group
        self.variables = {}
        for role, dtypes in DTYPES.items():
            var = group.get(role)
            if var is None or var not in node:
                raise ValueError(f"{name}: data group {data_group!r} has no {role}")
            arr = node[var]
            want = GRID if role != "uvw" else ("time", "baseline_id", "uvw_label")
            if arr.dims != want:
                raise ValueError(f"{name}: {var} has dimensions {arr.dims}, not {want}")
            if arr.dtype.newbyteorder("=") not in dtypes:
                raise ValueError(f"{name}: {var} is {arr.dtype}, not {' or '.join(str(d) for d in dtypes)}")
            self.variables[role] = var
        self.time_unix = np.asarray(node["time"].read(), np.float64)
        self.time = self.time_unix + UNIX_TO_MJD_SECONDS
        self.frequency = np.asarray(node["frequency"].read(), np.float64)
        self.polarization = tuple(str(p) for p in node["polarization"].read())
        self.antenna_names = [str(a) for a in node["antenna_xds"]["antenna_name"].read()]
        index = {a: i for i, a in enumerate(self.antenna_names)}
        n1 = [str(a) for a in node["baseline_antenna1_name"].read()]
        n2 = [str(a) for a in node["baseline_antenna2_name"].read()]
        try:
            self.antenna1 = np.asarray([index[a] for a in n1], np.int32)
            self.antenna2 = np.asarray([index[a] for a in n2], np.int32)
        except KeyError as exc:
            raise ValueError(f"{name}: baseline antenna {exc} not in antenna_xds") from exc
        self.field_name = self._per_time("field_name")
        self.scan_name = self._per_time("scan_name")
        self._weights_rule(groups)
        self._cache = {}

    def _weights_rule(self, groups):
        names = {g: groups[g].get("weight") for g in groups}
        used = sorted({v for v in names.values() if v is not None})
        writer = (self.node.attrs.get("creator") or {}).get("software_name")
        self.weight_variable, self.weight_refusal = None, None
        if len(used) == 1:
            self.weight_variable = used[0]
        elif writer == "xradio" and names.get("corrected") in self.node:
            self.weight_variable = names["corrected"]
        else:
            self.weight_refusal = (f"{self.name}: data groups name weights {names} (writer {writer!r}); W is known "
                                   "only when they name one, or for an xradio partition with a 'corrected' group")
        if self.weight_variable is not None:
            arr = self.node[self.weight_variable]
            if arr.dims != GRID or arr.dtype.newbyteorder("=") != np.float32:
                self.weight_refusal = f"{self.name}: {self.weight_variable} is {arr.dtype} over {arr.dims}"
                self.weight_variable = None

    def _per_time(self, coord):
        if coord not in self.node:
            return np.full(len(self.time), "", dtype=object)
        return np.asarray([str(v) for v in self.node[coord].read()], dtype=object)

    def _read(self, var):
        if var not in self._cache:
            self._cache[var] = self.node[var].read()
        return self._cache[var]

    def _flag_as_bool(self, flag):
        if flag.dtype == np.bool_:
            return flag
        bad = flag > 1
        if bad.any():
            raise ValueError(f"{self.name}: {self.variables['flag']} is uint8 with values "
                             f"{np.unique(flag[bad])[:8].tolist()} other than 0 and 1")
        return flag != 0

    @property
    def nbaseline(self):
        return len(self.antenna1)

    def rows(self, start=0, stop=None):
        """The rows of times `start` to `stop` (exclusive), pads dropped."""
        stop = len(self.time) if stop is None else stop
        if self.weight_variable is None:
            raise ValueError(self.weight_refusal)
        sl = slice(start, stop)
        vis = self._read(self.variables["correlated_data"])[sl]
        flag = self._flag_as_bool(self._read(self.variables["flag"])[sl])
        weight = self._read(self.weight_variable)[sl]
        uvw = self._read(self.variables["uvw"])[sl]
        ntime, nbl, nchan, ncorr = vis.shape
        uvw = uvw.reshape(ntime * nbl, 3)
        vis = vis.reshape(ntime * nbl, nchan, ncorr)
        # A pad has all-NaN UVW; only those cells' visibilities are checked.
        pad = np.isnan(uvw).all(axis=1)
        if pad.any():
            cand = np.flatnonzero(pad)
            pad[cand] = np.isnan(vis[cand].reshape(len(cand), -1)).all(axis=1)
        npad = int(pad.sum())
        keep = slice(None) if npad == 0 else ~pad  # no pads: views, no copies
        return {
            "ANTENNA1": np.tile(self.antenna1, ntime)[keep],
            "ANTENNA2": np.tile(self.antenna2, ntime)[keep],
            "TIME": np.repeat(self.time[sl], nbl)[keep],
            "FLAG_ROW": np.zeros(ntime * nbl - npad, bool),
            "DATA": vis[keep],
            "FLAG": flag.reshape(ntime * nbl, nchan, ncorr)[keep],
            "WEIGHT_SPECTRUM": weight.reshape(ntime * nbl, nchan, ncorr)[keep],
            "UVW": uvw[keep],
            "FIELD_NAME": np.repeat(self.field_name[sl], nbl)[keep],
            "SCAN_NAME": np.repeat(self.scan_name[sl], nbl)[keep],
            "PADS": npad,
        }

    def chunks(self, time_rows=None):
        """Row chunks of `time_rows` times each (all times by default)."""
        ntime = len(self.time)
        step = ntime if not time_rows else int(time_rows)
        for start in range(0, ntime, max(step, 1)):
            yield self.rows(start, min(start + step, ntime))


# ------------------------------------------------------------------ into the gridder


def gridder_inputs(partition, rows=None):
    """The gridder's inputs from a partition's rows (linear XX, XY, YX, YY
    correlations): uvw (nrow, 3) float64, the channel frequencies, Stokes I
    visibilities complex64 and weights float32 (nrow, nchan), formed on the
    GPU (`weighting.stokes_i`), and the mask (nrow, nchan) uint8, 1 where
    the Stokes I sample is unflagged with a positive weight."""
    from . import weighting

    if partition.polarization != ("XX", "XY", "YX", "YY"):
        raise ValueError(f"{partition.name}: Stokes I needs XX, XY, YX, YY, not {partition.polarization}")
    r = partition.rows() if rows is None else rows
    vis, weight = weighting.stokes_i(r["DATA"], r["WEIGHT_SPECTRUM"], r["FLAG"])
    mask = (weight > 0).astype(np.uint8)
    return {"uvw": np.ascontiguousarray(r["UVW"], np.float64), "freq": partition.frequency.copy(), "vis": vis,
            "wgt": weight, "mask": mask}


# ------------------------------------------------------------------ writing


def _array_meta(shape, dtype, chunks, dims, compressor, fill, attrs=None):
    if dtype.kind == "U":
        dt = {"name": "fixed_length_utf32", "configuration": {"length_bytes": dtype.itemsize}}
    else:
        dt = dtype.name
        if dt not in _NUMERIC:
            raise ValueError(f"cannot write {dtype}")
    codecs = [{"name": "bytes", "configuration": {"endian": "little"}}]
    if compressor == "blosc":
        codecs.append({"name": "blosc", "configuration": {"typesize": int(dtype.itemsize), "cname": "lz4",
                                                          "clevel": 5, "shuffle": "shuffle", "blocksize": 0}})
    elif compressor == "zstd":
        codecs.append({"name": "zstd", "configuration": {"level": 0, "checksum": False}})
    return {"shape": list(shape), "data_type": dt,
            "chunk_grid": {"name": "regular", "configuration": {"chunk_shape": list(chunks)}},
            "chunk_key_encoding": {"name": "default", "configuration": {"separator": "/"}},
            "fill_value": fill, "codecs": codecs, "attributes": attrs or {}, "dimension_names": list(dims),
            "zarr_format": 3, "node_type": "array", "storage_transformers": []}


def write_processing_set(path, partitions, time_chunk=None, blocksize=0):
    """Write a processing set directory: `partitions` maps a name to a dict
    of `time` (Unix s), `frequency`, `polarization`, `antenna_name`,
    `antenna1`, `antenna2` (indices), `VISIBILITY` complex64, `FLAG` bool,
    `WEIGHT` float32 (time, baseline, frequency, polarization) and `UVW`
    float64 (time, baseline, 3). Data arrays are Blosc/LZ4 (byte shuffle)
    in chunks of `time_chunk` times; coordinates zstd. Consolidated metadata
    at the root, as xradio writes it."""
    import pyarrow

    z = pyarrow.Codec("zstd")
    root = Path(path)
    root.mkdir(parents=True, exist_ok=False)
    consolidated = {}

    def put(rel, arr, dims, compressor, fill, chunks=None, attrs=None):
        arr = np.ascontiguousarray(arr)
        chunks = tuple(chunks or arr.shape)
        meta = _array_meta(arr.shape, arr.dtype, chunks, dims, compressor, fill, attrs)
        d = root / rel
        d.mkdir(parents=True, exist_ok=True)
        (d / "zarr.json").write_text(json.dumps(meta))
        consolidated[rel] = meta
        for idx in np.ndindex(*[-(-s // c) for s, c in zip(arr.shape, chunks)]):
            sl = tuple(slice(i * c, (i + 1) * c) for i, c in zip(idx, chunks))
            block = np.zeros(chunks, arr.dtype)
            part = arr[sl]
            block[tuple(slice(0, s) for s in part.shape)] = part
            raw = block.tobytes()
            if compressor == "blosc":
                raw = blosc_encode(raw, arr.dtype.itemsize, shuffle=True, blocksize=blocksize)
            elif compressor == "zstd":
                raw = z.compress(raw).to_pybytes()
            f = d / "c" / "/".join(str(i) for i in idx)
            f.parent.mkdir(parents=True, exist_ok=True)
            f.write_bytes(raw)

    for name, p in partitions.items():
        nt = len(p["time"])
        tc = time_chunk or nt
        nbl = len(p["antenna1"])
        names = np.asarray(p["antenna_name"])
        grid_chunks = (tc, nbl, len(p["frequency"]), len(p["polarization"]))
        put(f"{name}/VISIBILITY", p["VISIBILITY"].astype(np.complex64), GRID, "blosc", [0.0, 0.0], grid_chunks)
        put(f"{name}/FLAG", p["FLAG"].astype(bool), GRID, "blosc", False, grid_chunks)
        put(f"{name}/WEIGHT", p["WEIGHT"].astype(np.float32), GRID, "blosc", "NaN", grid_chunks)
        put(f"{name}/UVW", p["UVW"].astype(np.float64), ("time", "baseline_id", "uvw_label"), "blosc", "NaN",
            (tc, nbl, 3))
        put(f"{name}/time", np.asarray(p["time"], np.float64), ("time",), "zstd", "NaN")
        put(f"{name}/frequency", np.asarray(p["frequency"], np.float64), ("frequency",), "zstd", "NaN")
        put(f"{name}/polarization", np.asarray(p["polarization"]), ("polarization",), "zstd", "")
        put(f"{name}/baseline_antenna1_name", names[np.asarray(p["antenna1"])], ("baseline_id",), "zstd", "")
        put(f"{name}/baseline_antenna2_name", names[np.asarray(p["antenna2"])], ("baseline_id",), "zstd", "")
        put(f"{name}/antenna_xds/antenna_name", names, ("antenna_name",), "zstd", "")
        groups = {"base": {"correlated_data": "VISIBILITY", "flag": "FLAG", "weight": "WEIGHT", "uvw": "UVW"}}
        for rel, attrs in ((f"{name}/antenna_xds", {"type": "antenna"}),
                           (name, {"schema_version": "4.0.1", "type": "visibility", "data_groups": groups,
                                   "creator": {"software_name": "rang-core_b200", "version": "1"}})):
            meta = {"attributes": attrs, "zarr_format": 3, "node_type": "group"}
            (root / rel / "zarr.json").write_text(json.dumps(meta))
            consolidated[rel] = meta
    top = {"attributes": {"type": "processing_set"}, "zarr_format": 3, "node_type": "group",
           "consolidated_metadata": {"kind": "inline", "must_understand": False, "metadata": consolidated}}
    (root / "zarr.json").write_text(json.dumps(top))
    return root
