"""Run the reference's generated pipelines on a GPU host and record their results.

Test infrastructure: needs only the binaries built by ``ref_harness.py``
(``oracle/_ref/bin/<case>``), this package's seeded generators and numpy; it does
not read the reference source tree.

For every case it writes the case's tables in the reference column-file format
into a scratch directory, runs the binary there, parses ``queryresult.csv`` and
stores ``<out>/<case>.json`` with the column names, the row count, a canonical
checksum of the sorted rows, the rows themselves when there are at most
``MAX_ROWS``, and the binary's own ``<timing>`` block (host ``std::clock``
around each synchronised launch, dogqc/code.py:4-26).

Usage: ``python oracle/ref_run.py OUTDIR [case ...]``.
"""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from canonical import canonical_checksum  # noqa: E402
from mmdb import parse_result, write_mmdb  # noqa: E402
from ref_cases import CASES  # noqa: E402
from dogqc_b200 import workloads  # noqa: E402

MAX_ROWS = 5000
BIN = os.path.join(HERE, "_ref", "bin")


def parse_timing(stdout):
    out = {}
    m = re.search(r"<timing>(.*?)</timing>", stdout, re.S)
    if not m:
        return out
    for line in m.group(1).splitlines():
        mm = re.match(r"\s*(.+?):\s+([0-9.]+) ms", line)
        if mm:
            out[mm.group(1).strip()] = float(mm.group(2))
    return out


def run_case(name, spec, outdir, scratch):
    exe = os.path.join(BIN, name)
    rec = {"case": name, "spec": spec}
    if not os.path.exists(exe):
        rec["error"] = "binary missing"
        return rec
    db = workloads.GENERATORS[spec["workload"]](spec["scale"], **spec.get("gen_kw", {}))
    work = os.path.join(scratch, name)
    os.makedirs(work, exist_ok=True)
    write_mmdb(db, os.path.join(work, "mmdb"))
    del db
    t0 = time.time()
    p = subprocess.run([exe], cwd=work, capture_output=True, timeout=900)
    rec["wall_s"] = time.time() - t0
    rec["returncode"] = p.returncode
    stdout = p.stdout.decode("latin-1")
    rec["stdout_tail"] = stdout[-3000:]
    rec["stderr_tail"] = p.stderr.decode("latin-1")[-2000:]
    rec["timing_ms"] = parse_timing(stdout)
    res = os.path.join(work, "queryresult.csv")
    if p.returncode == 0 and os.path.exists(res):
        names, rows = parse_result(res, spec.get("str_cols", ()))
        rec["columns"] = names
        rec["nrows"] = len(rows)
        rec["checksum"] = canonical_checksum(rows)
        if len(rows) <= MAX_ROWS:
            rec["rows"] = sorted(rows)
    shutil.rmtree(work, ignore_errors=True)
    return rec


def main(outdir, names):
    os.makedirs(outdir, exist_ok=True)
    scratch = tempfile.mkdtemp(prefix="dq_ref_")
    try:
        for name in names or list(CASES):
            rec = run_case(name, CASES[name], outdir, scratch)
            with open(os.path.join(outdir, name + ".json"), "w") as f:
                json.dump(rec, f, indent=1)
            print(name, rec.get("returncode"), rec.get("nrows"), rec.get("checksum"),
                  rec.get("timing_ms", {}).get("totalKernelTime"), flush=True)
    finally:
        shutil.rmtree(scratch, ignore_errors=True)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2:])
