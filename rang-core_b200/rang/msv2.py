"""MSv2 (casacore table) reader feeding the gridder: the columns the path
needs from a Measurement Set's main table and its DATA_DESCRIPTION,
SPECTRAL_WINDOW and POLARIZATION subtables, the reference's `ms.rs`
(core/src/ms.rs) for the storage managers a Measurement Set of the
reference's writer and casacore use for them.

* `table.dat` (AipsIO, core/src/ms.rs:1906-2087): the row count, the
  byte order, the column descriptions and the data managers with the
  columns bound to them.
* StandardStMan (ms.rs:438-846): scalars and booleans (bits), fixed-shape
  ("direct") arrays in the buckets, variable-shape ("indirect") arrays in
  `table.fNi` (ms.rs:965-1048).
* TiledShapeStMan, TiledColumnStMan and TiledCellStMan (ms.rs:1320-1860):
  hypercubes of tiles, each tile holding its columns' pixels in Fortran
  order, the columns in descending pixel size. A column is read here by
  mapping a hypercube's tiles into NumPy and reordering them with one
  reshape and transpose.
* IncrementalStMan (ms.rs:1049-1320): runs of rows sharing one value, for
  numeric and boolean scalars, fixed-shape arrays and indirect arrays.
* Strings (ms.rs:847-964, :1296-1318): fixed-length and indirect scalars in
  StandardStMan buckets, string arrays in its chained string buckets,
  IncrementalStMan strings and indirect string arrays in `table.fNi`; they
  come back as NumPy object arrays of `str`.
* The row count: that of `table.lock`'s sync record where it has one (rows
  added after `table.dat` was written), else `table.dat`'s.

Cells come back in NumPy order: a casacore array of shape (ncorr, nchan)
per row reads as (nrow, nchan, ncorr). `rows(path, data_desc_id)` gives the
rows of one data description in the layout of `rang.msv4.Partition.rows`,
so both readers feed `rang.msv4.gridder_inputs`.
"""

from pathlib import Path

import numpy as np

MAGIC = 0xBEBEBEBE
BUCKET_START = 512
NUMPY = {0: "bool", 1: "i1", 2: "u1", 3: "i2", 4: "u2", 5: "i4", 6: "u4", 7: "f4", 8: "f8", 9: "c8", 10: "c16",
         29: "i8"}
STRING = 11
CORR_NAMES = {5: "RR", 6: "RL", 7: "LR", 8: "LL", 9: "XX", 10: "XY", 11: "YX", 12: "YY"}


def _size(code):
    return 0 if code in (0, STRING) else np.dtype(NUMPY[code]).itemsize


def _dtype(code, big):
    return np.dtype(NUMPY[code]).newbyteorder(">" if big else "<")


def _bits(raw, first, count):
    """`count` booleans from bit `first` of `raw`, least significant bit first."""
    bits = np.unpackbits(np.frombuffer(raw, np.uint8), bitorder="little")
    if first + count > bits.size:
        raise ValueError("truncated boolean bits")
    return bits[first:first + count].astype(bool)


class Cursor:
    """AipsIO reading: objects are (length, type name, version), values
    big-endian (canonical) or little-endian."""

    def __init__(self, data, big):
        self.b, self.pos, self.big = data, 0, big

    def take(self, n):
        if self.pos + n > len(self.b):
            raise ValueError(f"truncated AipsIO data at byte {self.pos}")
        out = self.b[self.pos:self.pos + n]
        self.pos += n
        return out

    def _int(self, n, signed=False):
        return int.from_bytes(self.take(n), "big" if self.big else "little", signed=signed)

    def u8(self):
        return self.take(1)[0]

    def bool(self):
        return self.u8() != 0

    def u32(self):
        return self._int(4)

    def i32(self):
        return self._int(4, True)

    def u64(self):
        return self._int(8)

    def i64(self):
        return self._int(8, True)

    def string(self):
        return self.take(self.u32()).decode("utf-8", "replace")

    def magic(self):
        if self.u32() != MAGIC:
            raise ValueError("AipsIO magic value missing")

    def start(self, kind=None):
        at = self.pos
        length = self.u32()
        name = self.string()
        version = self.u32()
        if kind is not None and name != kind:
            raise ValueError(f"expected AipsIO object {kind}, found {name}")
        return at, length, version

    def end(self, obj):
        self.pos = obj[0] + obj[1]

    def skip(self):
        self.end(self.start())

    def iposition(self):
        obj = self.start("IPosition")
        n = self.u32()
        out = [self.i32() if obj[2] == 1 else self.i64() for _ in range(n)]
        self.end(obj)
        return out

    def block(self, wide=False):
        obj = self.start("Block")
        n = self.u32()
        out = [self.u64() if wide else self.u32() for _ in range(n)]
        self.end(obj)
        return out


def _lock_rows(path):
    """The row count of the sync record of `table.lock` (ms.rs:2254-2280):
    after the lock requests ((1 + 2 * 32) big-endian ints), the record's
    length and an AipsIO `sync` object whose first field is the row count;
    None when there is none."""
    lock = path / "table.lock"
    if not lock.is_file():
        return None
    raw = lock.read_bytes()
    at = (1 + 2 * 32) * 4
    if len(raw) < at + 4:
        return None
    n = int.from_bytes(raw[at:at + 4], "big")
    if n == 0:
        return None
    c = Cursor(raw[at + 4:at + 4 + n], True)
    c.magic()
    obj = c.start("sync")
    return c.u32() if obj[2] == 1 else c.u64()


class Column:
    def __init__(self, name, code, is_array, option, shape, max_length, manager):
        self.name, self.code, self.is_array, self.option = name, code, is_array, option
        self.shape, self.max_length, self.manager = list(shape), max_length, manager
        self.fixed_shape = bool(self.shape) and bool(option & 4)

    @property
    def direct(self):
        return self.is_array and bool(self.option & 1)


class Table:
    """One casacore table (a directory)."""

    def __init__(self, path):
        self.path = Path(path)
        raw = (self.path / "table.dat").read_bytes()
        c = Cursor(raw, True)
        c.magic()
        table = c.start("Table")
        if table[2] > 3:
            raise ValueError(f"table.dat version {table[2]} is not read")
        self.nrows = c.u64() if table[2] > 2 else c.u32()
        synced = _lock_rows(self.path)
        if synced:  # rows added after table.dat was written (ms.rs:1925-1933)
            self.nrows = synced
        self.little = c.u32() != 0
        kind = c.string()
        if kind != "PlainTable":
            raise ValueError(f"table type {kind} is not read")
        desc = c.start("TableDesc")
        c.string(), c.string(), c.string()
        c.skip()  # keywords
        if desc[2] != 1:
            c.skip()  # private keywords
        cols = []
        for _ in range(c.u32()):
            c.u32()
            cls = c.string()
            c.u32()
            name = c.string()
            c.string()
            c.string(), c.string()  # data manager type and group of the description
            code = c.i32()
            option = c.i32()
            c.i32()  # ndim
            is_array = cls.startswith("ArrayColumnDesc")
            if not is_array and not cls.startswith("ScalarColumnDesc"):
                raise ValueError(f"column class {cls} of {name} is not read")
            shape = c.iposition() if is_array else []
            max_length = c.u32()
            c.skip()  # keywords
            c.u32()
            if is_array:
                c.bool()
            elif code == STRING:
                c.string()  # default value
            elif code == 0:
                c.u8()
            else:
                c.take(_size(code))
            cols.append(Column(name, code, is_array, option, shape, max_length, None))
        c.end(desc)
        if table[2] == 1:
            c.skip()
        first = c.i32()
        version = 1
        if first < 0:
            version = -first
            c.u32() if version <= 2 else c.u64()
        if version >= 3:
            c.i32(), c.i32()  # storage option
        c.u32()
        kinds = [(c.string(), c.u32()) for _ in range(c.u32())]
        for col in cols:
            c.u32()
            c.string()
            c.u32()
            col.manager = c.u32()
            if col.is_array and c.bool():
                shape = c.iposition()
                if not col.shape:
                    col.shape = shape
                col.fixed_shape = bool(col.shape)
        blobs = [c.take(c.u32()) for _ in kinds]
        self.columns = {col.name: col for col in cols}
        self.managers = {}
        for (kind, seq), blob in zip(kinds, blobs):
            mine = [col for col in cols if col.manager == seq]
            if kind == "StandardStMan":
                self.managers[seq] = _Ssm(self, seq, blob, mine)
            elif kind in ("TiledShapeStMan", "TiledColumnStMan", "TiledCellStMan"):
                self.managers[seq] = _Tsm(self, seq, kind, mine)
            elif kind == "IncrementalStMan":
                self.managers[seq] = _Ism(self, seq, blob, mine)
            else:
                self.managers[seq] = kind

    def file(self, seq, suffix=""):
        return self.path / f"table.f{seq}{suffix}"

    def read(self, name, start=0, count=None):
        """Rows [start, start + count) of a column (all rows by default)."""
        if name not in self.columns:
            raise KeyError(f"{self.path.name}: no column {name}")
        col = self.columns[name]
        count = self.nrows - start if count is None else count
        mgr = self.managers[col.manager]
        if isinstance(mgr, str):
            raise ValueError(f"{name}: storage manager {mgr} is not read")
        return mgr.read(col, start, count)


class _Ssm:
    """StandardStMan: buckets after a 512-byte header; per column an offset
    in the bucket and an index mapping rows to buckets."""

    def __init__(self, table, seq, blob, cols):
        c = Cursor(blob, True)
        c.magic()
        obj = c.start("SSM")
        c.string()
        self.col_offset = c.block()
        self.col_index = c.block()
        c.end(obj)
        self.path = table.file(seq)
        head = self.path.read_bytes()[:BUCKET_START]
        h = Cursor(head, not table.little)
        h.magic()
        obj = h.start("StandardStMan")
        self.big = h.bool() if obj[2] >= 3 else True
        if self.big == table.little:
            raise ValueError("StandardStMan byte order differs from the table's")
        self.bucket_size = h.u32()
        self.nbuckets = h.u32()
        h.u32(), h.u32(), h.i32()
        n_idx_buckets = h.u32()
        bucket = h.i32()
        idx_offset = h.u32() if obj[2] >= 2 else 0
        h.i32()
        left = h.u32()
        n_indices = h.u32()
        with open(self.path, "rb") as f:
            data = bytearray()
            for _ in range(n_idx_buckets):
                if bucket < 0:
                    raise ValueError("StandardStMan index chain ends early")
                f.seek(BUCKET_START + bucket * self.bucket_size)
                b = f.read(self.bucket_size)
                nxt = int.from_bytes(b[4:8], "big", signed=True)
                if idx_offset:
                    data += b[idx_offset:idx_offset + left]
                else:
                    data += b[8:8 + min(left, self.bucket_size - 8)]
                left = max(0, left - (self.bucket_size - 8))
                bucket = nxt
        ic = Cursor(bytes(data), self.big)
        self.indices = []
        for _ in range(n_indices):
            ic.magic()
            obj = ic.start("SSMIndex")
            used = ic.u32()
            ic.u32(), ic.u32()
            ic.skip()
            last = ic.block(wide=obj[2] != 1)
            buckets = ic.block()
            self.indices.append((np.asarray(last[:used], np.int64), np.asarray(buckets[:used], np.int64)))
            ic.end(obj)
        self.slot = {col.name: i for i, col in enumerate(cols)}

    def _runs(self, col, start, count):
        """(bucket bytes, column offset, first row in bucket, rows) in row order."""
        i = self.slot[col.name]
        last, buckets = self.indices[self.col_index[i]]
        off = self.col_offset[i]
        row, end = start, start + count
        with open(self.path, "rb") as f:
            while row < end:
                k = int(np.searchsorted(last, row))
                if k >= len(last):
                    raise ValueError(f"row {row} beyond the StandardStMan index")
                first = 0 if k == 0 else int(last[k - 1]) + 1
                stop = min(int(last[k]) + 1, end)
                if buckets[k] >= self.nbuckets:
                    raise ValueError("StandardStMan bucket beyond the file")
                f.seek(BUCKET_START + int(buckets[k]) * self.bucket_size)
                yield f.read(self.bucket_size), off, row - first, stop - row
                row = stop

    def _bucket(self, f, n):
        if n < 0 or n >= self.nbuckets:
            raise ValueError("string bucket chain leaves the file")
        f.seek(BUCKET_START + n * self.bucket_size)
        return f.read(self.bucket_size)

    def _chars(self, f, bucket, offset, length, cursor=None):
        """`length` characters from (bucket, offset) of the string buckets
        (16 big-endian bookkeeping bytes: the bucket number, the bytes used,
        deleted bytes, the next bucket; then characters), following the chain;
        returns them and the position after them."""
        out = bytearray()
        b, at = bucket, offset
        data = self._bucket(f, b)
        guard = 0
        while len(out) < length:
            used = max(0, int.from_bytes(data[4:8], "big", signed=True))
            take = min(length - len(out), max(0, used - at))
            out += data[16 + at:16 + at + take]
            at += take
            if len(out) < length:
                guard += 1
                if guard > self.nbuckets:
                    raise ValueError("string bucket chain loops")
                b, at = int.from_bytes(data[12:16], "big", signed=True), 0
                data = self._bucket(f, b)
        return bytes(out), (b, at)

    def _strings_at(self, f, pos, n):
        """`n` strings from a position of the string buckets, each a
        big-endian length and its characters; returns them and the end."""
        out = []
        for _ in range(n):
            raw, pos = self._chars(f, pos[0], pos[1], 4)
            text, pos = self._chars(f, pos[0], pos[1], max(0, int.from_bytes(raw, "big", signed=True)))
            out.append(text.decode("utf-8", "replace"))
        return out, pos

    def _read_strings(self, col, start, count):
        fixed_scalar = not col.is_array and col.max_length > 0
        width = col.max_length if fixed_scalar else 12
        order = "big" if self.big else "little"
        slots = []
        for b, off, first, n in self._runs(col, start, count):
            for r in range(n):
                slots.append(b[off + (first + r) * width:off + (first + r + 1) * width])
        out = []
        with open(self.path, "rb") as f:
            for row, slot in enumerate(slots, start):
                if fixed_scalar:
                    out.append(slot.split(b"\0", 1)[0].decode("utf-8", "replace"))
                    continue
                bk, o, ln = (int.from_bytes(slot[4 * i:4 * i + 4], order, signed=True) for i in range(3))
                if not col.is_array:  # up to 8 characters sit in the slot itself
                    text = slot[:max(ln, 0)] if ln <= 8 else self._chars(f, bk, o, ln)[0]
                    out.append(text.decode("utf-8", "replace"))
                    continue
                if col.fixed_shape:
                    shape = list(col.shape)
                    n = int(np.prod(shape))
                    vals = self._strings_at(f, (bk, o), n)[0] if ln > 0 else [""] * n
                else:
                    if ln <= 0:
                        raise ValueError(f"row {row} of {col.name} has no array")
                    raw, pos = self._chars(f, bk, o, 4)
                    ndim = int.from_bytes(raw, "big", signed=True)
                    if not 0 <= ndim <= 64:
                        raise ValueError(f"row {row} of {col.name}: string array of {ndim} axes")
                    shape = []
                    for _ in range(ndim):
                        raw, pos = self._chars(f, pos[0], pos[1], 4)
                        shape.append(int.from_bytes(raw, "big", signed=True))
                    raw, pos = self._chars(f, pos[0], pos[1], 4)
                    n = int(np.prod(shape)) if shape else 1
                    vals = self._strings_at(f, pos, n)[0] if int.from_bytes(raw, "big") else [""] * n
                out.append(np.array(vals, dtype=object).reshape(tuple(reversed(shape))))
        if not col.is_array:
            return np.array(out, dtype=object)
        if any(a.shape != out[0].shape for a in out):
            raise ValueError(f"rows of {col.name} differ in shape; read fewer rows at once")
        return np.stack(out) if out else np.zeros(0, dtype=object)

    def read(self, col, start, count):
        if col.code == STRING:
            return self._read_strings(col, start, count)
        if not col.is_array:
            parts = []
            for b, off, first, n in self._runs(col, start, count):
                if col.code == 0:
                    parts.append(_bits(b[off:], first, n))
                else:
                    size = _size(col.code)
                    parts.append(np.frombuffer(b, _dtype(col.code, self.big), n, off + first * size))
            return np.concatenate(parts).astype(np.dtype(NUMPY[col.code])) if parts else \
                np.zeros(0, NUMPY[col.code])
        if col.direct:
            nelem = int(np.prod(col.shape))
            cell = tuple(reversed(col.shape))
            parts = []
            for b, off, first, n in self._runs(col, start, count):
                if col.code == 0:
                    parts.append(_bits(b[off:], first * nelem, n * nelem))
                else:
                    size = _size(col.code)
                    parts.append(np.frombuffer(b, _dtype(col.code, self.big), n * nelem, off + first * nelem * size))
            out = np.concatenate(parts) if parts else np.zeros(0)
            return out.astype(np.dtype(NUMPY[col.code])).reshape((count,) + cell)
        offsets = []
        for b, off, first, n in self._runs(col, start, count):
            offsets.append(np.frombuffer(b, np.dtype("u8").newbyteorder(">" if self.big else "<"), n, off + first * 8))
        offsets = np.concatenate(offsets) if offsets else np.zeros(0, np.uint64)
        return _indirect(Path(str(self.path) + "i"), self.big, col, offsets)


def _indirect(path, big, col, offsets):
    """Variable-shape arrays of a StandardStMan column from its `table.fNi`:
    at each row's offset, (a reference count in version > 0,) the number of
    axes, the shape (int32) and the values."""
    raw = path.read_bytes()
    version = int.from_bytes(raw[:4], "big" if big else "little")
    order = "big" if big else "little"
    out, shape0 = [], None
    for row, at in enumerate(int(o) for o in offsets):
        if at == 0:
            raise ValueError(f"row {row} of {col.name} has no array")
        p = at + (4 if version > 0 else 0)
        ndim = int.from_bytes(raw[p:p + 4], order)
        shape = [int.from_bytes(raw[p + 4 + 4 * i:p + 8 + 4 * i], order, signed=True) for i in range(ndim)]
        p += 4 + 4 * ndim
        n = int(np.prod(shape)) if shape else 1
        if shape0 is None:
            shape0 = shape
        elif shape != shape0:
            raise ValueError(f"rows of {col.name} differ in shape; read fewer rows at once")
        if col.code == 0:
            vals = _bits(raw[p:p + (n + 7) // 8], 0, n)
        elif col.code == STRING:  # per element an offset to (length, characters); 0 for ""
            vals = []
            for e in range(n):
                at_e = int.from_bytes(raw[p + 4 * e:p + 4 * e + 4], order)
                ln = int.from_bytes(raw[at_e:at_e + 4], order) if at_e else 0
                vals.append(raw[at_e + 4:at_e + 4 + ln].decode("utf-8", "replace") if at_e else "")
            vals = np.array(vals, dtype=object)
        else:
            vals = np.frombuffer(raw, _dtype(col.code, big), n, p).astype(np.dtype(NUMPY[col.code]))
        out.append(vals.reshape(tuple(reversed(shape))))
    if not out:
        return np.zeros((0,), NUMPY[col.code])
    return np.stack(out)


class _Ism:
    """IncrementalStMan (core/src/ms.rs:1049-1320): a value is stored once
    for a run of rows. Buckets follow the 512-byte header; each starts with
    the offset of its interval table (low 28 bits; a high bit marks 64-bit
    row numbers), which holds per column the first row of each run and the
    offset of its value; the index of buckets follows the initial buckets."""

    def __init__(self, table, seq, blob, cols):
        c = Cursor(blob, True)
        c.magic()
        obj = c.start("ISM")
        c.string()
        c.end(obj)
        self.path = table.file(seq)
        raw = self.path.read_bytes()
        h = Cursor(raw[:BUCKET_START], not table.little)
        h.magic()
        obj = h.start("IncrementalStMan")
        self.big = h.bool() if obj[2] >= 5 else True
        if self.big == table.little:
            raise ValueError("IncrementalStMan byte order differs from the table's")
        self.bucket_size = h.u32()
        ninit = h.u32()
        ic = Cursor(raw[BUCKET_START + ninit * self.bucket_size:], self.big)
        ic.magic()
        obj = ic.start("ISMIndex")
        used = ic.u32()
        self.starts = np.asarray(ic.block(wide=obj[2] > 1)[:used + 1], np.int64)
        self.buckets = ic.block()[:used]
        self.raw = raw
        self.slot = {col.name: i for i, col in enumerate(cols)}
        self.ncol = len(cols)

    def _intervals(self, bucket, k):
        order = "big" if self.big else "little"
        word = int.from_bytes(bucket[:4], order)
        wide = bool(word & 0xF0000000)
        at = word & 0x0FFFFFFF
        for col in range(self.ncol):
            n = int.from_bytes(bucket[at:at + 4], order)
            at += 4
            rsize = 8 if wide else 4
            rows = [int.from_bytes(bucket[at + rsize * i:at + rsize * (i + 1)], order) for i in range(n)]
            at += rsize * n
            offs = [int.from_bytes(bucket[at + 4 * i:at + 4 * (i + 1)], order) for i in range(n)]
            at += 4 * n
            if col == k:
                return rows, offs
        raise ValueError("IncrementalStMan bucket without the column")

    def _value(self, col, bucket, at):
        """One row's value at byte `at` of a bucket."""
        if col.is_array and not col.direct:
            off = int.from_bytes(bucket[at:at + 8], "big" if self.big else "little")
            if off == 0:
                raise ValueError(f"a row of {col.name} has no array")
            return _indirect(Path(str(self.path) + "i"), self.big, col, [off])[0]
        nelem = int(np.prod(col.shape)) if col.is_array else 1
        if col.is_array and not col.fixed_shape:
            raise ValueError(f"{col.name}: IncrementalStMan direct arrays without a fixed shape are not read")
        if col.code == STRING:
            # The total length (itself included), then one string's characters,
            # or for several strings each one's length and characters.
            order = "big" if self.big else "little"
            total = int.from_bytes(bucket[at:at + 4], order)
            body = bucket[at + 4:at + max(total, 4)]
            if nelem == 1 and not col.is_array:
                return body.decode("utf-8", "replace")
            vals, p = [], 0
            for _ in range(nelem):
                ln = int.from_bytes(body[p:p + 4], order)
                vals.append(body[p + 4:p + 4 + ln].decode("utf-8", "replace"))
                p += 4 + ln
            return np.array(vals, dtype=object).reshape(tuple(reversed(col.shape)))
        if col.code == 0:
            vals = _bits(bucket[at:at + (nelem + 7) // 8], 0, nelem)
        else:
            vals = np.frombuffer(bucket, _dtype(col.code, self.big), nelem, at).astype(np.dtype(NUMPY[col.code]))
        return vals.reshape(tuple(reversed(col.shape))) if col.is_array else vals[0]

    def read(self, col, start, count):
        k = self.slot[col.name]
        out = []
        row, end = start, start + count
        while row < end:
            i = int(np.searchsorted(self.starts, row, side="right")) - 1
            if i < 0 or i + 1 >= len(self.starts):
                raise ValueError(f"row {row} beyond the IncrementalStMan index")
            b0, b1 = int(self.starts[i]), int(self.starts[i + 1])
            at = BUCKET_START + self.buckets[i] * self.bucket_size
            bucket = self.raw[at:at + self.bucket_size]
            rows, offs = self._intervals(bucket, k)
            last = min(b1, end) - 1
            while row <= last:
                local = row - b0
                j = max(0, int(np.searchsorted(rows, local, side="right")) - 1)
                until = rows[j + 1] if j + 1 < len(rows) else b1 - b0
                n = min(until, last - b0 + 1) - local
                value = self._value(col, bucket, 4 + offs[j])
                out.extend([value] * n)
                row += n
        if col.code == STRING and not col.is_array:
            return np.array(out, dtype=object)
        if not out:
            return np.zeros(0, dtype=object if col.code == STRING else NUMPY[col.code])
        return np.stack([np.asarray(v) for v in out])


class _Tsm:
    """The tiled storage managers: hypercubes of tiles in `table.fN_TSMk`."""

    def __init__(self, table, seq, kind, cols):
        h = Cursor((table.file(seq)).read_bytes(), True)
        h.magic()
        outer = h.start(kind)
        fixed_tile = h.iposition() if kind in ("TiledColumnStMan", "TiledCellStMan") else None
        inner = h.start("TiledStMan")
        self.big = h.bool() if inner[2] >= 2 else True
        if self.big == table.little:
            raise ValueError("TiledStMan byte order differs from the table's")
        seqnr = h.u32()
        nrow = h.u64() if inner[2] >= 3 else h.u32()
        ncol = h.u32()
        if seqnr != seq or ncol != len(cols) or nrow != table.nrows:
            raise ValueError(f"TiledStMan header of {table.file(seq)} does not match the table")
        self.codes = []
        for col in cols:
            if h.i32() != col.code:
                raise ValueError("TiledStMan data type does not match the column")
            self.codes.append(col.code)
        h.string()
        h.u64() if inner[2] >= 3 else h.u32()
        self.per_row = kind == "TiledCellStMan"
        self.nrdim = h.u32() + int(self.per_row)
        files = []
        for _ in range(h.u64() if inner[2] >= 3 else h.u32()):
            if h.bool():
                v = h.u32()
                fseq = h.u32()
                h.u32() if v == 1 else h.u64()
                files.append(table.file(seq, f"_TSM{fseq}"))
            else:
                files.append(None)
        self.files = files
        self.cubes = []
        for _ in range(h.u64() if inner[2] >= 3 else h.u32()):
            v = h.u32()
            h.skip()
            h.bool()
            h.u32()
            shape, tile = h.iposition(), h.iposition()
            if self.per_row and shape:
                shape, tile = shape + [1], tile + [1]
            fseq = h.i32()
            foff = h.u32() if v == 1 else h.u64()
            self.cubes.append((shape, tile, fseq, foff))
        h.end(inner)
        self.by_row = fixed_tile is None and not self.per_row
        if self.by_row:
            h.iposition()
            n = h.u32()
            self.row_map = np.asarray(h.block()[:n], np.int64)
            self.cube_map = np.asarray(h.block()[:n], np.int64)
            self.pos_map = np.asarray(h.block()[:n], np.int64)
        h.end(outer)
        # Columns share a tile in descending order of pixel size (stable).
        order = sorted(range(len(cols)), key=lambda i: -self._pixel(self.codes[i]))
        self.rank = {cols[i].name: r for r, i in enumerate(order)}
        self.order = order
        self.index = {col.name: i for i, col in enumerate(cols)}

    @staticmethod
    def _pixel(code):
        return _size(code)

    @staticmethod
    def _tile_bytes(code, pixels):
        return (pixels + 7) // 8 if code == 0 else _size(code) * pixels

    def _locate(self, rows):
        """(cube, position along the last axis) of each row."""
        rows = np.asarray(rows, np.int64)
        if self.per_row:
            return rows, np.zeros_like(rows)
        if not self.by_row:
            return np.zeros_like(rows), rows
        if rows.size and (self.row_map.size == 0 or rows.max() > self.row_map[-1]):
            raise ValueError("a row has no tiled array")
        i = np.searchsorted(self.row_map, rows)
        cube = self.cube_map[i]
        if np.any(cube == 0):
            raise ValueError("a row has no tiled array")
        return cube, self.pos_map[i] - (self.row_map[i] - rows)

    def _cube_column(self, col, ci):
        """The whole of hypercube `ci` for column `col`, NumPy order (last
        casacore axis first)."""
        shape, tile, fseq, foff = self.cubes[ci]
        if fseq < 0 or self.files[fseq] is None:
            raise ValueError(f"hypercube {ci} of {col.name} has no file")
        k = self.index[col.name]
        tpix = int(np.prod(tile))
        sizes = [self._tile_bytes(self.codes[i], tpix) for i in range(len(self.codes))]
        bucket = sum(sizes)
        at = sum(sizes[i] for i in self.order[:self.rank[col.name]])
        ntile = [-(-s // t) for s, t in zip(shape, tile)]
        nt = int(np.prod(ntile))
        raw = np.fromfile(self.files[fseq], np.uint8, nt * bucket, offset=foff).reshape(nt, bucket)
        part = raw[:, at:at + sizes[k]]
        code = self.codes[k]
        if code == 0:
            vals = np.unpackbits(part, axis=1, bitorder="little")[:, :tpix].astype(bool)
        else:
            vals = np.ascontiguousarray(part).view(_dtype(code, self.big)).astype(np.dtype(NUMPY[code]))
        n = len(shape)
        a = vals.reshape(tuple(reversed(ntile)) + tuple(reversed(tile)))
        perm = [x for j in range(n) for x in (j, n + j)]
        a = a.transpose(perm).reshape(tuple(t * m for t, m in zip(reversed(tile), reversed(ntile))))
        return a[tuple(slice(0, s) for s in reversed(shape))]

    def read(self, col, start, count):
        rows = np.arange(start, start + count)
        cube, pos = self._locate(rows)
        out, cell = None, None
        for ci in np.unique(cube):
            sel = np.flatnonzero(cube == ci)
            data = self._cube_column(col, int(ci))
            if cell is None:
                cell = data.shape[1:]
                out = np.empty((count,) + cell, data.dtype)
            elif data.shape[1:] != cell:
                raise ValueError(f"rows of {col.name} differ in shape; read fewer rows at once")
            out[sel] = data[pos[sel]]
        if out is None:
            return np.zeros((0,), NUMPY[self.codes[self.index[col.name]]])
        return out


def rows(path, data_desc_id=0):
    """The main-table rows of one data description, in the layout of
    `rang.msv4.Partition.rows` (DATA, FLAG, WEIGHT_SPECTRUM (else WEIGHT per
    correlation), UVW, TIME (MJD s), ANTENNA1, ANTENNA2, FLAG_ROW,
    FIELD_NAME from the FIELD table, SCAN_NAME the scan number), plus the
    channel frequencies and the correlation names."""
    path = Path(path)
    main = Table(path)
    ddid = main.read("DATA_DESC_ID")
    sel = np.flatnonzero(ddid == data_desc_id)
    if sel.size == 0:
        raise ValueError(f"no rows with DATA_DESC_ID {data_desc_id}")
    lo, hi = int(sel[0]), int(sel[-1]) + 1

    def col(name):
        if sel.size == hi - lo:
            return main.read(name, lo, hi - lo)
        return np.concatenate([main.read(name, int(r), 1) for r in sel])

    dd = Table(path / "DATA_DESCRIPTION")
    spw = int(dd.read("SPECTRAL_WINDOW_ID", data_desc_id, 1)[0])
    pol = int(dd.read("POLARIZATION_ID", data_desc_id, 1)[0])
    freq = Table(path / "SPECTRAL_WINDOW").read("CHAN_FREQ", spw, 1)[0].astype(np.float64)
    corr = Table(path / "POLARIZATION").read("CORR_TYPE", pol, 1)[0]
    field = Table(path / "FIELD")
    names = field.read("NAME") if field.nrows else np.zeros(0, dtype=object)
    fid = col("FIELD_ID")
    field_name = np.array([str(names[i]) if 0 <= i < len(names) else "" for i in fid], dtype=object)
    scan_name = np.array([str(int(v)) for v in col("SCAN_NUMBER")], dtype=object)
    data = col("DATA")
    weight = col("WEIGHT_SPECTRUM") if "WEIGHT_SPECTRUM" in main.columns else \
        np.broadcast_to(col("WEIGHT")[:, None, :], data.shape).astype(np.float32)
    return {"ANTENNA1": col("ANTENNA1"), "ANTENNA2": col("ANTENNA2"), "TIME": col("TIME"),
            "FLAG_ROW": col("FLAG_ROW"), "DATA": data, "FLAG": col("FLAG"), "WEIGHT_SPECTRUM": weight,
            "UVW": col("UVW"), "FIELD_NAME": field_name, "SCAN_NAME": scan_name, "frequency": freq,
            "polarization": tuple(CORR_NAMES.get(int(c), str(c)) for c in corr)}


class DataDescription:
    """The rows of one data description of a Measurement Set, with the
    attributes `rang.msv4.gridder_inputs` reads (name, frequency,
    polarization), so that either reader feeds the gridder."""

    def __init__(self, path, data_desc_id=0):
        self.path, self.data_desc_id = Path(path), int(data_desc_id)
        self._rows = rows(self.path, self.data_desc_id)
        self.name = f"{self.path.name}:{self.data_desc_id}"
        self.frequency = self._rows["frequency"]
        self.polarization = self._rows["polarization"]

    def rows(self):
        return {k: v for k, v in self._rows.items() if k not in ("frequency", "polarization")}
