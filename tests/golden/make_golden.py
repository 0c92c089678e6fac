"""Generate the golden fixtures of the gridder tests from the reference itself.

    python tests/golden/make_golden.py REFERENCE_CHECKOUT

* `df1_cases.npz` — the four seeded synthetic cases of the reference's DF1
  protocol, made by importing the reference's own generator
  (`examples/oracle_ducc0.py`, which needs only NumPy): its `CASES` and
  `make_case` (`:216-286`: seeds 101-104, uv up to 0.45 of the Nyquist
  extent, w of both signs, point sources on pixel centres plus noise, weights
  in [0.5, 1.5)), whose `dft_dirty` / `dft_vis` (`:85-120`) give the FP64
  direct-Fourier-transform dirty image of the data and visibilities of a
  sparse 16-pixel image. Every array is the reference's output, stored as it
  returned it.
* `df1_reference_errors.json` — the reference gridder's own worst errors
  against that DFT per precision, epsilon and direction, as its DF1 run
  recorded them (`research/results/df1-wgridder.json`, "worst"), so the tests
  can hold this library's errors on the same cases against the reference's.
* `kernel_rows.json` — the 939 rows of the kernel table as parsed from the
  reference, after checking the SHA256 its own test pins
  (`tests/test_core_wgridder.py:16`), so the table can be checked where the
  reference checkout is absent.

The DFT is independent of every gridder (oracle and CUDA path alike).
"""

import importlib.util
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO / "rang-core_b200" / "csrc"))

# The case fields the tests read (the generator also returns "sources").
FIELDS = ("uvw", "freq", "vis", "wgt", "nx", "ny", "dx", "dy", "dft_dirty", "image", "dft_vis")


def reference_generator(reference: Path):
    """The reference's `examples/oracle_ducc0.py`, imported from its checkout."""
    path = reference / "examples" / "oracle_ducc0.py"
    spec = importlib.util.spec_from_file_location("reference_oracle_ducc0", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py REFERENCE_CHECKOUT")
    reference = Path(sys.argv[1])
    gen = reference_generator(reference)
    out = {}
    for case in gen.CASES:
        rec = gen.make_case(*case)
        for k in FIELDS:
            out[f"{case[0]}/{k}"] = np.asarray(rec[k])
    np.savez_compressed(HERE / "df1_cases.npz", **out)
    worst = json.loads((reference / "research" / "results" / "df1-wgridder.json").read_text())["worst"]
    vs_dft = {k: v for k, v in worst.items() if k.endswith("vs DFT")}
    (HERE / "df1_reference_errors.json").write_text(json.dumps(vs_dft, indent=1, sort_keys=True) + "\n")
    import gen_kernel_db

    rows, digest = gen_kernel_db.read_rows(reference)
    (HERE / "kernel_rows.json").write_text(json.dumps({"sha256": digest, "rows": rows}))
    print("wrote", HERE / "df1_cases.npz", HERE / "df1_reference_errors.json", HERE / "kernel_rows.json")


if __name__ == "__main__":
    main()
