"""Build the reference's own generated pipelines for the oracle cases.

Test infrastructure.  Runs only where the reference source tree is present
(``DOGQC_REFERENCE``, default ``/root/reference``); writes generated ``.cu`` files
and sm_100a binaries into ``oracle/_ref/`` and nothing else.  No reference source
is copied: the generated code includes the reference's headers from where they lie
(through a symlink inside ``oracle/_ref``).

What it does per case (``oracle/ref_cases.py``), following the recipe in the
reference's drivers (query/tpch.py:40-69):

1. generate the seeded tables with ``dogqc_b200.workloads`` (only their sizes and
   string heap sizes enter the generated code);
2. build the plan with the reference's ``RelationalAlgebra`` and
   ``dogqc.scalarAlgebra`` and resolve it with the plan config;
3. translate with ``CudaCompiler(..., smArchitecture="sm_100a",
   decimalRepr=CType.ULL)`` so every decimal attribute and sum is an exact
   ``unsigned long long``;
4. compile with the reference's own ``compile`` (nvcc, dogqc/codegen.py:170-192).

Three settings are patched in the reference's modules at run time, without
editing its files:

* ``CType.zeroValue/minValue/maxValue[ULL]`` get ``ull`` literals; with plain
  ``0`` the emitted ``initArray<T>(T*, T, int)`` call cannot deduce ``T``;
* ``MaterializeTranslator.consumePrintResultSample`` also writes the full result
  to ``queryresult.csv`` (``printToFile`` is hard-wired off,
  dogqc/cudaTranslator.py:614);
* ``KernelCall.defaultGridSize`` is set to 8 blocks per SM of a 148-SM B200.

Usage: ``python oracle/ref_harness.py [case ...]``.
"""
import os
import sys
import types as pytypes

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from ref_cases import CASES  # noqa: E402
from dogqc_b200 import workloads  # noqa: E402

REF = os.environ.get("DOGQC_REFERENCE", "/root/reference")
OUT = os.path.join(HERE, "_ref")
GRID = 148 * 8
BLOCK = 128


def _reference_modules():
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import dogqc.cudaTranslator as ct
    import dogqc.scalarAlgebra as scal
    from dogqc.cudalang import CType
    from dogqc.hashJoins import EquiJoinTranslator
    from dogqc.kernel import KernelCall
    from dogqc.relationalAlgebra import RelationalAlgebra, Reduction
    from dogqc.types import Type

    CType.zeroValue[CType.ULL] = "0ull"
    CType.minValue[CType.ULL] = "0ull"
    CType.maxValue[CType.ULL] = "ULLONG_MAX"
    if not getattr(ct.MaterializeTranslator, "_dq_patched", False):
        sample = ct.MaterializeTranslator.consumePrintResultSample

        def both(self, ctxt, numOut):
            sample(self, ctxt, numOut)
            self.consumePrintToFile(ctxt, numOut)
        ct.MaterializeTranslator.consumePrintResultSample = both
        ct.MaterializeTranslator._dq_patched = True
    KernelCall.defaultGridSize = GRID
    KernelCall.defaultBlockSize = BLOCK
    return pytypes.SimpleNamespace(ct=ct, scal=scal, CType=CType, EquiJoinTranslator=EquiJoinTranslator,
                                   RelationalAlgebra=RelationalAlgebra, Reduction=Reduction, Type=Type)


def build_case(name, spec, ref):
    db = workloads.GENERATORS[spec["workload"]](spec["scale"], **spec.get("gen_kw", {}))
    schema = {}
    for tname, entry in db.schema.items():
        entry = dict(entry)
        entry["attributes"] = type(entry["attributes"])(
            (a, ref.Type[t.name]) for a, t in entry["attributes"].items())
        schema[tname] = entry
    alg = ref.RelationalAlgebra(pytypes.SimpleNamespace(schema=schema))
    plan, cfg = workloads.PLANS[spec["workload"]](alg, ref.scal, ref.Type, ref.Reduction,
                                                   **spec.get("plan_kw", {}))
    plan = alg.resolveAlgebraPlan(plan, cfg)
    compiler = ref.ct.CudaCompiler(algebraContext=alg, smArchitecture="sm_100a",
                                   decimalRepr=ref.CType.ULL, debug=False)
    ref.EquiJoinTranslator.usePushDownJoin = bool(spec.get("pushdown", False))
    if spec.get("buffers") == "selection":
        compiler.setBuffers([alg.selectionNodes[0].opId])
    cplan = alg.translateToCompilerPlan(plan, compiler)
    compiler.gencode(cplan)
    srcdir = os.path.join(OUT, "src")
    cwd = os.getcwd()
    os.chdir(srcdir)
    try:
        compiler.compile(name)
    finally:
        os.chdir(cwd)
    built = os.path.join(srcdir, name)
    if not os.path.exists(built):
        raise RuntimeError("reference compile failed for case %s" % name)
    exe = os.path.join(OUT, "bin", name)
    os.replace(built, exe)
    return exe


def main(names):
    """Generated sources stay in ``_ref/src`` (not shipped to GPU hosts); binaries
    go to ``_ref/bin``.  The header symlink exists only while compiling."""
    os.makedirs(os.path.join(OUT, "bin"), exist_ok=True)
    os.makedirs(os.path.join(OUT, "src"), exist_ok=True)
    link = os.path.join(OUT, "dogqc")
    if not os.path.islink(link):
        os.symlink(os.path.join(REF, "dogqc"), link)
    try:
        ref = _reference_modules()
        for name in names or list(CASES):
            exe = build_case(name, CASES[name], ref)
            print("built", exe)
    finally:
        os.unlink(link)


if __name__ == "__main__":
    main(sys.argv[1:])
