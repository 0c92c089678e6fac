"""Extract the Measurement Set fixtures of the reader tests from the reference.

* `msv4_m05.zip`: the reference's `tests/data/msv4/m05.zip` (an xradio 1.3.1
  processing set `m05.ps.zarr/` and the MSv2 `m05.ms/` it was converted
  from, the reference's edge-case set's two-window MS,
  `tests/test_msv4.py:1-13`); the MSv2 lock files carry row counts.
* `msv2_edge.zip`: the reference's `tests/data/msv2-edge/` casacore tables
  (TiledCellStMan cells of four shapes, IncrementalStMan, string columns)
  with its `oracle.json` of their values.

    python tests/golden/make_ms_fixtures.py /path/to/reference
"""

import sys
import zipfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
def main(reference):
    ref = Path(reference) / "tests" / "data"
    src = zipfile.ZipFile(ref / "msv4" / "m05.zip")
    out = HERE / "msv4_m05.zip"
    with zipfile.ZipFile(out, "w", zipfile.ZIP_DEFLATED) as dst:
        for name in src.namelist():
            dst.writestr(name, src.read(name))
    print(out, out.stat().st_size)
    edge = ref / "msv2-edge"
    out = HERE / "msv2_edge.zip"
    with zipfile.ZipFile(out, "w", zipfile.ZIP_DEFLATED) as dst:
        for f in sorted(edge.rglob("*")):
            if f.is_file():
                dst.write(f, f.relative_to(edge).as_posix())
    print(out, out.stat().st_size)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {Path(__file__).name} REFERENCE_CHECKOUT")
    main(sys.argv[1])
