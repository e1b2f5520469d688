"""Build the reference's own text importer for the lineitem benchmark sample
(test infrastructure: the timed CPU baseline of the text import).

The reference's importer is C++ that its Python writes per schema and table
size and compiles with ``g++ -std=c++11 -pthread`` (dogqc/dbio.py:140-149:
``loadDatabase`` -> ``CodeGenerator.compileCpu``, dogqc/codegen.py:195-207),
then runs once.  This script drives the same generator for the reference's
lineitem schema (query/schema/tpch.py:22-41) with relative paths -- it reads
``csv/lineitem.tbl`` and writes its column files into ``mmdb/`` of the working
directory -- and keeps the compiled program as
``oracle/_ref/tbl_import_lineitem_<rows>`` instead of running it.  The table
size is compiled in (the generated code allocates its column files from it),
so the program loads exactly ``rows`` lines: the first ``rows`` lines of the
benchmark's text.

Usage: ``python oracle/build_ref_importer.py [rows]`` (reads the reference at
$DOGQC_REFERENCE, default /root/reference; needs g++).
"""
import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("DOGQC_REFERENCE", "/root/reference")
OUT_DIR = os.path.join(HERE, "_ref")
ROWS = 2_000_000


def binary_path(rows=ROWS):
    return os.path.join(OUT_DIR, "tbl_import_lineitem_%d" % rows)


def build(rows=ROWS):
    sys.path.insert(0, REF)
    from dogqc import dbio
    from dogqc.codegen import CodeGenerator, CType
    from query.schema.tpch import tpchSchema
    work = tempfile.mkdtemp(prefix="dq_refimp_")
    cwd = os.getcwd()
    try:
        os.symlink(os.path.join(REF, "dogqc"), os.path.join(work, "dogqc"))
        src = os.path.join(work, "src")
        os.makedirs(os.path.join(src, "csv"))
        with open(os.path.join(src, "csv", "lineitem.tbl"), "w") as fh:
            fh.write("\n" * rows)            # the generator sizes the table with wc -l
        os.chdir(src)
        schema = {"dateformat": tpchSchema["dateformat"], "lineitem": dict(tpchSchema["lineitem"])}
        sized = dbio.Importer.retrieveTableSizes(schema, "csv")
        acc = dbio.Accessor("mmdb", sized)
        im = dbio.Importer(acc, "csv")
        # dbio.py:140-146 without the final execute
        codegen = CodeGenerator(CType.FP32)
        codegen.types.add(schema["dateformat"])
        im.codegen = codegen
        codegen.read.add(im.getCodeReadDatabase())
        codegen.compileCpu("loadDB")
        os.makedirs(OUT_DIR, exist_ok=True)
        shutil.copy2(os.path.join(src, "loadDB"), binary_path(rows))
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)
    return binary_path(rows)


if __name__ == "__main__":
    print(build(int(sys.argv[1]) if len(sys.argv) > 1 else ROWS))
