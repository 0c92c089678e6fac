"""Extract the MSv4 fixture of the reader tests from the reference.

`msv4_m05.zip` holds, from the reference's `tests/data/msv4/m05.zip` (an
xradio 1.3.1 processing set and the MSv2 it was converted from, the
reference's edge-case set's two-window MS, `tests/test_msv4.py:1-13`):

* the whole processing set `m05.ps.zarr/` (zarr v3, Blosc/LZ4 data arrays,
  zstd coordinates);
* the MSv2 main table's storage files that hold DATA and WEIGHT_SPECTRUM
  (TiledShapeStMan tiles `table.f0_TSM*`, `table.f1_TSM*`) and UVW
  (StandardStMan buckets `table.f2`), as raw bytes: the tests find every
  value the reader decodes from the store among them.

    python tests/golden/make_msv4_fixture.py /path/to/reference
"""

import sys
import zipfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
KEEP_MS = ("table.f0_TSM1", "table.f0_TSM2", "table.f1_TSM1", "table.f1_TSM2", "table.f2")


def main(reference):
    src = zipfile.ZipFile(Path(reference) / "tests" / "data" / "msv4" / "m05.zip")
    out = HERE / "msv4_m05.zip"
    with zipfile.ZipFile(out, "w", zipfile.ZIP_DEFLATED) as dst:
        for name in src.namelist():
            if name.startswith("m05.ps.zarr/") or name in {"m05.ms/" + f for f in KEEP_MS}:
                dst.writestr(name, src.read(name))
    print(out, out.stat().st_size)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
