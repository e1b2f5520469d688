"""Drop-in replacement for the reference's ``CudaCompiler`` translator object.

The reference's drivers use the translator like this (query/tpch.py:61-69):

    compiler = CudaCompiler(algebraContext=alg, smArchitecture="sm_75", decimalRepr=CType.FP64)
    compilerPlan = alg.translateToCompilerPlan(plan, compiler)
    compiler.gencode(compilerPlan)
    compiler.compile("tpch1")
    compiler.execute()

``Backend`` accepts the same calls (dogqc/cudaTranslator.py:31-101): ``translate``
is invoked bottom-up by ``translateToCompilerPlan`` and returns light plan
nodes; ``gencode`` lowers the plan into the pipeline IR; ``compile`` prepares it
on the device through the C ABI (no nvcc at query time); ``execute`` runs it,
prints the reference's ``Result: N tuples`` summary and ``<timing>`` block, and
returns the ``Result``.  ``setBuffers`` places the lane refill after the given
selections and joins, as the reference places its ``LaneRefill`` (without it,
one refill per pipeline follows its first selective filter or probe);
``setProfilers`` adds lane-activity histograms where the given operators hand
their rows on, printed after the ``<timing>`` block.  The knobs the reference
reads from class attributes (``KernelCall.default*``,
``EquiJoinTranslator.usePushDownJoin``) do not apply: launch shapes come from
the device (or ``dq_tuning``), and multimatch probes always walk their match
ranges warp-cooperatively, the reference's push-down, with long ranges deferred
and grouped by range.

Tables are read from the database behind the plan context: a
``dogqc_b200.database.Database`` (host columns), or the reference's accessor
whose ``dbpath`` holds ``<table>_<attr>`` column files
(``dogqc_b200.importer.read_mmdb``).
"""
import sys

from dogqc_b200.engine import default_engine
from dogqc_b200.lowering import Lowering
from dogqc_b200.types import CType


class TranslatedNode(object):
    """What ``translate`` returns: the algebra node and its translated children."""

    def __init__(self, algExpr, children):
        self.algExpr = algExpr
        self.children = children

    def opId(self):
        return self.algExpr.opId


class Backend(object):
    def __init__(self, algebraContext, smArchitecture="sm_100a", decimalRepr=CType.ULL, debug=False,
                 engine=None, device=0):
        self.algebraContext = algebraContext
        self.smArchitecture = smArchitecture
        self.decimalRepr = decimalRepr
        self.debug = debug
        self.bufferPositions = []
        self._buffers_set = False
        self.profilerPositions = []
        self.engine = engine
        self.device = device
        self.lowering = None
        self.plan = None
        self.result = None
        self.filename = None

    # translator protocol (relationalAlgebra.py:243-282)
    def translate(self, algebraExpr, child1=None, child2=None):
        return TranslatedNode(algebraExpr, [c for c in (child1, child2) if c is not None])

    def setBuffers(self, positions):
        """Lane refill after these operators (selection or join ids) and
        nowhere else, where the reference places its LaneRefill
        (dogqc/cudaTranslator.py:59-63, 84-86); without a call the backend
        places one refill per pipeline after its first selective filter or
        probe."""
        self.bufferPositions = list(positions)
        self._buffers_set = True

    def setProfilers(self, positions):
        """Lane-activity histograms (warp steps by active lanes) where these
        operators hand their rows to their parents, as the reference's
        LaneActivityProfiler counts them (dogqc/cudaLaneActivityProfile.py);
        printed by execute() and returned by profiles()."""
        self.profilerPositions = list(positions)

    def gencode(self, translationPlan):
        roots = [t.algExpr if isinstance(t, TranslatedNode) else t for t in translationPlan]
        options = {}
        if self._buffers_set:
            options["buffers"] = list(self.bufferPositions)
        if self.profilerPositions:
            options["profilers"] = list(self.profilerPositions)
        self.lowering = Lowering(roots, options)
        return self.lowering

    def _database(self):
        ctxt = getattr(self.algebraContext, "ctxt", self.algebraContext)
        db = getattr(ctxt, "database", None)
        if db is not None and not hasattr(db, "tables") and hasattr(db, "dbpath"):
            from dogqc_b200.importer import read_mmdb
            db = read_mmdb(db.dbpath, schema=db.schema)
        return db

    def compile(self, filename=None):
        if self.lowering is None:
            raise RuntimeError("gencode() must run before compile()")
        self.filename = filename
        if self.engine is None:
            self.engine = default_engine(self.device)
        db = self._database()
        if db is not None:
            self.engine.register_database(db)
        self.plan = self.engine.prepare(self.lowering)
        return self.plan

    def execute(self, quiet=False):
        if self.plan is None:
            self.compile(self.filename)
        self.result = self.plan.execute()
        if not quiet:
            t = self.plan.timing()
            sys.stdout.write(self.result.format_sample())
            sys.stdout.write("<timing>\n")
            for i, ms in enumerate(t["pipeline_ms"]):
                sys.stdout.write("%32s: %6.3f ms\n" % ("pipeline%d" % i, ms))
            sys.stdout.write("%32s: %6.3f ms\n" % ("totalKernelTime", t["total_ms"]))
            sys.stdout.write("</timing>\n")
            for op_id, counts in self.profiles().items():
                sys.stdout.write("<p%d>\n" % op_id)
                sys.stdout.write("".join("%d, %d\n" % (i, c) for i, c in enumerate(counts)))
                sys.stdout.write("</p%d>\n\n" % op_id)
            sys.stdout.flush()
        return self.result

    def profiles(self):
        """Operator id -> lane-activity histogram of the last execute (33
        counts: warp steps with 0..32 active lanes as the operator handed its
        rows on), for the operators given to setProfilers."""
        if self.plan is None or self.lowering is None:
            return {}
        return {op_id: self.plan.profile(i) for i, op_id in enumerate(self.lowering.profile_points)}

    def showGraph(self, plan):
        raise NotImplementedError("plan graphs need graphviz, which this image does not ship")


CudaCompiler = Backend
