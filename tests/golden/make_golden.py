"""Turn the reference's run records into committed golden fixtures.

Input: the JSON records written by ``oracle/ref_run.py`` on a GPU host (the
reference's own generated pipelines compiled for sm_100a by
``oracle/ref_harness.py``, run over this package's seeded tables).  Output:
``tests/golden/ref_<case>.json`` with the case spec, column names, row count,
canonical checksum, the sorted rows for small results, and the reference's own
``std::clock`` timing block (informational).

Usage: ``python tests/golden/make_golden.py <dir with ref_run records>``.
"""
import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(src):
    for path in sorted(glob.glob(os.path.join(src, "*.json"))):
        rec = json.load(open(path))
        if rec.get("returncode") != 0 or "checksum" not in rec:
            print("skipping", path, rec.get("error") or rec.get("returncode"))
            continue
        out = {k: rec[k] for k in ("case", "spec", "columns", "nrows", "checksum", "timing_ms") if k in rec}
        if "rows" in rec:
            out["rows"] = rec["rows"]
        dst = os.path.join(HERE, "ref_%s.json" % rec["case"])
        with open(dst, "w") as f:
            json.dump(out, f, indent=None, separators=(",", ":"))
            f.write("\n")
        print("wrote", dst, out["nrows"], out["checksum"][:12])


if __name__ == "__main__":
    main(sys.argv[1])
