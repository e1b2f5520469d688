"""Relational-algebra plan front end.

Plan scripts and plan configs written for DogQC build their operator trees through
``RelationalAlgebra`` (the builder of dogqc/relationalAlgebra.py:57-144): the same
builder methods, operator classes, enums, per-operator hints and node fields that a
translator reads.  The backend (``dogqc_b200.backend.Backend``) reads only those
fields, so it takes trees built by DogQC's own classes as well.

What must agree with DogQC, because configs and results depend on it:

* operator ids count up in construction order (children before parents), and
  ``resolveAlgebraPlan`` wraps the last root in a result materialisation
  (relationalAlgebra.py:129-138, 151-152);
* attribute ids count up in creation order: aggregates when the aggregation is
  built, scanned and mapped attributes when the plan is bound
  (relationalAlgebra.py:48-52, 301-314, 518-531);
* an identifier is ``name``, ``table.name`` or ``alias.name``, and one that two
  input attributes share is ambiguous (relationalAlgebra.py:174-197);
* an operator's output keeps an attribute only if an operator above it uses it,
  except a materialisation, which keeps all its input (relationalAlgebra.py:199-204,
  640-642);
* the cardinality estimates and their hints ``selectivity``, ``multimatch`` (default
  True), ``htSizeFactor`` (default 2.0) and ``numgroups`` (default: the input's
  estimate) (relationalAlgebra.py:342-349, 441-458, 489-500, 564-574).

How it is organised here: each operator only declares what it contributes (the
attributes it creates, the identifiers it looks up, its output, its estimate).
The builder drives three passes over each plan root -- ``_bind`` (post-order: inputs
first, then the operator's own lookups, which stamp each used attribute with the
operator's id), ``_trim`` (outputs cut to what is used above) and ``_estimate``
(post-order cardinalities) -- so no operator class walks the tree itself.
"""
import itertools
from collections import Counter, OrderedDict
from collections.abc import Mapping
from enum import Enum

from dogqc_b200.types import Type


def _as_list(value):
    return value if isinstance(value, list) else [value]


def _hint(cfg, op_id, key, default):
    """Per-operator plan hint ``cfg[op_id][key]``, or ``default`` when the config
    has no entry for the operator or the key (DogQC's configs are dicts keyed by
    operator id; a missing config is ``None`` or ``{}``)."""
    if not isinstance(cfg, Mapping):
        return default
    entry = cfg.get(op_id)
    if isinstance(entry, Mapping) and key in entry:
        return entry[key]
    return default


class Join(Enum):
    CROSS = 1
    INNER = 2
    SEMI = 3
    ANTI = 4
    OUTER = 5


class Reduction(Enum):
    SUM = 1
    COUNT = 2
    AVG = 3
    MIN = 4
    MAX = 5


class MaterializationType(Enum):
    RESULT = 1
    TEMPTABLE = 2


class Attribute(object):
    """One column as it flows between operators.  The fields are the ones a
    translator reads: ``id``, ``name``, ``dataType``, ``identifiers`` (names it
    answers to), ``creation`` (operator counter when it was made), ``lastUse``
    (id of the highest operator that reads it) and ``numElements``."""

    def __init__(self, name, id, opId):
        self.id = id
        self.name = name
        self.identifiers = [name]
        self.creation = opId
        self.lastUse = 0
        self.dataType = None
        self.numElements = None


class Context(object):
    """Id counters and the catalogue a plan is built against (the database's
    schema plus the temp tables the plan creates)."""

    def __init__(self, database):
        self.database = database
        self.schema = dict(database.schema)
        self._ops = itertools.count(1)
        self._attrs = itertools.count(1)
        self.opIdNum = 0
        self.attributeIdNum = 0
        self.tableVersions = Counter()

    def opId(self):
        self.opIdNum = next(self._ops)
        return self.opIdNum

    def createTable(self, identifier):
        self.schema[identifier] = {"name": identifier, "attributes": OrderedDict()}
        return self.schema[identifier]

    def resolveTable(self, identifier):
        self.tableVersions[identifier] += 1
        return self.tableVersions[identifier], self.schema[identifier]

    def createAttribute(self, attributeName, tableName=None):
        self.attributeIdNum = next(self._attrs)
        return self.attributeIdNum, Attribute(attributeName, self.attributeIdNum, self.opIdNum)


class AlgExpr(object):
    """An operator.  ``inputs`` holds its input operators; ``inRelation`` and
    ``outRelation`` map attribute ids to attributes (insertion order is the
    column order of results)."""

    arity = 0

    def __init__(self, ctxt, *inputs):
        self.opId = ctxt.opId()
        self.inputs = inputs
        self.inRelation = dict()
        self.outRelation = dict()

    def children(self):
        return list(self.inputs)

    # -- what an operator contributes (overridden per class) --
    def bind(self, ctxt, bound_inputs):
        """Given its inputs' outputs (bound already), set ``inRelation``, look
        up identifiers and create attributes; return the output relation."""
        raise NotImplementedError

    def estimate(self, cfg, input_estimates):
        """Cardinality estimate from the inputs' estimates and the hints."""
        return input_estimates[0]

    trims_output = True

    # -- name lookup (called by scalar expressions while they bind) --
    def resolveAttribute(self, identifier):
        owners = {}
        for att in self.inRelation.values():
            for ident in att.identifiers:
                owners.setdefault(ident, []).append(att)
        found = owners.get(identifier)
        if not found:
            raise NameError("%s (operator %d) has no input attribute named '%s'"
                            % (type(self).__name__, self.opId, identifier))
        if len(found) > 1:
            raise SyntaxError("'%s' names %d input attributes of %s (operator %d)"
                              % (identifier, len(found), type(self).__name__, self.opId))
        att = found[0]
        att.lastUse = self.opId
        return att

    def touchAttribute(self, id):
        self.inRelation[id].lastUse = self.opId

    # -- DogQC's per-node entry points, driven by the passes below --
    def resolve(self, ctxt):
        return _bind(self, ctxt)

    def prune(self):
        _trim(self)

    def configure(self, cfg, ctxt):
        return _estimate(self, cfg)

    def translate(self, translator, ctxt):
        return translator.translate(self, *[i.translate(translator, ctxt) for i in self.inputs])


def _bind(node, ctxt):
    bound = [_bind(i, ctxt) for i in node.inputs]
    node.outRelation = node.bind(ctxt, bound)
    return node.outRelation


def _trim(node):
    for i in node.inputs:
        _trim(i)
    if node.trims_output:
        node.outRelation = {id: a for id, a in node.outRelation.items() if a.lastUse > node.opId}


def _estimate(node, cfg):
    node.tupleNum = node.estimate(cfg, [_estimate(i, cfg) for i in node.inputs])
    return node.tupleNum


# The arities, with the inputs under DogQC's names (translators tell unary and
# binary operators apart by these fields).
class LiteralAlgExpr(AlgExpr):
    arity = 0


class UnaryAlgExpr(AlgExpr):
    arity = 1

    @property
    def child(self):
        return self.inputs[0]


class BinaryAlgExpr(AlgExpr):
    arity = 2

    @property
    def leftChild(self):
        return self.inputs[0]

    @property
    def rightChild(self):
        return self.inputs[1]


class Scan(LiteralAlgExpr):
    def __init__(self, ctxt, tableName, alias=None):
        AlgExpr.__init__(self, ctxt)
        self.scanTableId, self.table = ctxt.resolveTable(tableName)
        self.tableAlias = alias
        self.isTempScan = "isTempTable" in self.table
        self.scanAttributes = dict()

    def bind(self, ctxt, bound_inputs):
        table = self.table
        prefixes = [table["name"]] + ([self.tableAlias] if self.tableAlias is not None else [])
        for column, ctype in table["attributes"].items():
            id, att = ctxt.createAttribute(column, table["name"])
            att.dataType = ctype
            att.numElements = table["size"]
            att.identifiers += ["%s.%s" % (p, column) for p in prefixes]
            if self.isTempScan:
                att.sourceId = table["sourceAttributes"][column]
            self.scanAttributes[id] = att
        return self.scanAttributes

    def estimate(self, cfg, input_estimates):
        return self.table["size"]


class Selection(UnaryAlgExpr):
    def __init__(self, ctxt, condition, child):
        AlgExpr.__init__(self, ctxt, child)
        self.condition = condition

    def bind(self, ctxt, bound_inputs):
        self.inRelation = bound_inputs[0]
        self.conditionAttributes = self.condition.resolve(self)
        return self.inRelation

    def estimate(self, cfg, input_estimates):
        self.selectivity = _hint(cfg, self.opId, "selectivity", 1.0)
        return int(input_estimates[0] * self.selectivity)


class Map(UnaryAlgExpr):
    def __init__(self, ctxt, attrName, expression, child):
        AlgExpr.__init__(self, ctxt, child)
        self.attrName = attrName
        self.expression = expression

    def bind(self, ctxt, bound_inputs):
        self.inRelation = bound_inputs[0]
        used = self.expression.resolve(self)
        self.mapStringAttributes = [a for a in used.values() if a.dataType == Type.STRING]
        _, self.mapAttr = ctxt.createAttribute(self.attrName)
        self.mapAttr.dataType = self.expression.type
        out = dict(self.inRelation)
        out[self.mapAttr.id] = self.mapAttr
        return out


class EquiJoin(BinaryAlgExpr):
    """Equality join of a build side (left) and a probe side (right), with
    optional further conditions; SEMI and ANTI output the probe side only."""

    def __init__(self, ctxt, joinType, equalityConditions, otherConditions, leftChild, rightChild):
        AlgExpr.__init__(self, ctxt, leftChild, rightChild)
        self.joinType = joinType
        self.equalities = _as_list(equalityConditions)
        self.conditions = otherConditions

    def bind(self, ctxt, bound_inputs):
        build, probe = bound_inputs
        self.inRelation = dict(build)
        self.inRelation.update(probe)
        cond = self.conditions.resolve(self) if self.conditions is not None else {}
        self.conditionProbeAttributes = {id: a for id, a in cond.items() if id in probe}
        self.buildKeyAttributes = OrderedDict()
        self.probeKeyAttributes = OrderedDict()
        for pair in self.equalities:
            a, b = (self.resolveAttribute(ident) for ident in pair)
            sides = (a.id in build, b.id in probe, b.id in build, a.id in probe)
            if sides[0] and sides[1]:
                bk, pk = a, b
            elif sides[2] and sides[3]:
                bk, pk = b, a
            else:
                raise NameError("join %d: %s and %s are not one build and one probe attribute"
                                % (self.opId, a.name, b.name))
            self.buildKeyAttributes[bk.id] = bk
            self.probeKeyAttributes[pk.id] = pk
        return self.inRelation if self.joinType in (Join.INNER, Join.OUTER) else dict(probe)

    def estimate(self, cfg, input_estimates):
        self.multimatch = _hint(cfg, self.opId, "multimatch", True)
        self.selectivity = _hint(cfg, self.opId, "selectivity", 1.0)
        self.htSizeFactor = _hint(cfg, self.opId, "htSizeFactor", 2.0)
        return int(max(input_estimates) * self.selectivity)


class CrossJoin(BinaryAlgExpr):
    """Every pair of left and right rows that satisfies ``condition``."""

    def __init__(self, ctxt, joinType, condition, leftChild, rightChild):
        AlgExpr.__init__(self, ctxt, leftChild, rightChild)
        self.joinType = joinType
        self.condition = condition

    def bind(self, ctxt, bound_inputs):
        self.inRelation = dict(bound_inputs[0])
        self.inRelation.update(bound_inputs[1])
        self.conditionAttributes = self.condition.resolve(self)
        return self.inRelation

    def estimate(self, cfg, input_estimates):
        self.multimatch = _hint(cfg, self.opId, "multimatch", True)
        self.selectivity = _hint(cfg, self.opId, "selectivity", 1.0)
        left, right = input_estimates
        return int(left * right * self.selectivity)


class Aggregation(UnaryAlgExpr):
    """Group by ``groupingIdentifiers`` with ``aggregates`` given as
    ``(Reduction, input identifier or "", alias)``.  An AVG gets a COUNT
    beside it when the list has none (its divisor).  The aggregate attributes
    are created here, when the operator is built."""

    def __init__(self, ctxt, groupingIdentifiers, aggregates, child):
        AlgExpr.__init__(self, ctxt, child)
        self.groupingIdentifiers = _as_list(groupingIdentifiers)
        specs = list(_as_list(aggregates))
        reductions = {spec[0] for spec in specs}
        if Reduction.AVG in reductions and Reduction.COUNT not in reductions:
            specs.append((Reduction.COUNT, "", "count_agg"))
        self.aggregates = specs
        self.aggregateAttributes = dict()
        self.avgAggregates = dict()
        self._specs = []
        for reduction, source, alias in specs:
            id, att = ctxt.createAttribute(alias)
            att.dataType = Type.INT if reduction == Reduction.COUNT else Type.DOUBLE
            if reduction == Reduction.COUNT:
                self.countAttr = att
            if reduction == Reduction.AVG:
                self.avgAggregates[id] = att
            self.aggregateAttributes[id] = att
            self._specs.append((att, source, reduction))

    def bind(self, ctxt, bound_inputs):
        self.inRelation = bound_inputs[0]
        self.groupAttributes = OrderedDict((a.id, a) for a in map(self.resolveAttribute, self.groupingIdentifiers))
        self.aggregateInAttributes = OrderedDict()
        self.aggregateTuples = dict()
        for att, source, reduction in self._specs:
            src = self.resolveAttribute(source) if source != "" else None
            if src is not None:
                self.aggregateInAttributes[src.id] = src
            self.aggregateTuples[att.id] = (src.id if src is not None else None, reduction)
        out = OrderedDict(self.groupAttributes)
        out.update(self.aggregateAttributes)
        return dict(out)

    def estimate(self, cfg, input_estimates):
        self.doGroup = bool(self.groupAttributes)
        self.numgroups = _hint(cfg, self.opId, "numgroups", input_estimates[0]) if self.doGroup else 1
        return self.numgroups


class Projection(UnaryAlgExpr):
    def __init__(self, ctxt, identifiers, child):
        AlgExpr.__init__(self, ctxt, child)
        self.identifiers = _as_list(identifiers)

    def bind(self, ctxt, bound_inputs):
        self.inRelation = bound_inputs[0]
        self.projectionAttributes = {a.id: a for a in map(self.resolveAttribute, self.identifiers)}
        return self.projectionAttributes


class Materialize(UnaryAlgExpr):
    """The plan's result, or a temp table that later plan roots scan."""

    trims_output = False

    def __init__(self, ctxt, child, matType=MaterializationType.RESULT, identifier=None):
        AlgExpr.__init__(self, ctxt, child)
        self.matType = matType
        if matType == MaterializationType.TEMPTABLE:
            self.table = ctxt.createTable(identifier)
            self.table["isTempTable"] = True

    @staticmethod
    def result(ctxt, child):
        return Materialize(ctxt, child)

    @staticmethod
    def temp(ctxt, identifier, child):
        return Materialize(ctxt, child, MaterializationType.TEMPTABLE, identifier)

    def bind(self, ctxt, bound_inputs):
        self.inRelation = bound_inputs[0]
        for att in self.inRelation.values():
            att.lastUse = self.opId
        if self.matType == MaterializationType.TEMPTABLE:
            self.table["sourceAttributes"] = {a.name: a.id for a in self.inRelation.values()}
            self.table["attributes"].update((a.name, a.dataType) for a in self.inRelation.values())
            self.table["numColumns"] = len(self.inRelation)
        return self.inRelation

    def estimate(self, cfg, input_estimates):
        if self.matType == MaterializationType.TEMPTABLE:
            self.table["size"] = input_estimates[0]
        return input_estimates[0]


class RelationalAlgebra(object):
    """DogQC's plan builder (relationalAlgebra.py:57-144): the same methods,
    keeping the selection and join nodes in the lists configs refer to."""

    def __init__(self, acc):
        self.ctxt = Context(acc)
        self.selectionNodes = []
        self.joinNodes = []
        self.semiJoinNodes = []
        self.antiJoinNodes = []

    def _kept(self, bucket, node):
        bucket.append(node)
        return node

    def scan(self, table, alias=None):
        return Scan(self.ctxt, table, alias)

    def selection(self, condition, child):
        return self._kept(self.selectionNodes, Selection(self.ctxt, condition, child))

    def projection(self, attributes, child):
        return Projection(self.ctxt, attributes, child)

    def map(self, attrName, expression, child):
        return Map(self.ctxt, attrName, expression, child)

    def createtemp(self, identifier, child):
        return Materialize.temp(self.ctxt, identifier, child)

    def result(self, child):
        return Materialize.result(self.ctxt, child)

    def join(self, condition, leftChild, rightChild):
        return self.innerjoin(condition, None, leftChild, rightChild)

    def crossjoin(self, condition, leftChild, rightChild):
        return CrossJoin(self.ctxt, Join.CROSS, condition, leftChild, rightChild)

    def innerjoin(self, equalityConditions, otherConditions, leftChild, rightChild):
        return self._kept(self.joinNodes, EquiJoin(self.ctxt, Join.INNER, equalityConditions, otherConditions,
                                                   leftChild, rightChild))

    def semijoin(self, equalityConditions, otherConditions, leftChild, rightChild):
        return self._kept(self.semiJoinNodes, EquiJoin(self.ctxt, Join.SEMI, equalityConditions, otherConditions,
                                                       leftChild, rightChild))

    def antijoin(self, equalityConditions, otherConditions, leftChild, rightChild):
        return self._kept(self.antiJoinNodes, EquiJoin(self.ctxt, Join.ANTI, equalityConditions, otherConditions,
                                                       leftChild, rightChild))

    def outerjoin(self, equalityConditions, otherConditions, leftChild, rightChild):
        return EquiJoin(self.ctxt, Join.OUTER, equalityConditions, otherConditions, leftChild, rightChild)

    def aggregation(self, groupAttributes, aggregates, child):
        return Aggregation(self.ctxt, groupAttributes, aggregates, child)

    def resolveAlgebraPlan(self, plan, cfg):
        """Wraps the last root in the result and runs the passes root by root
        (a temp table's size is known before a later root scans it)."""
        roots = _as_list(plan)
        roots[-1] = self.result(roots[-1])
        for root in roots:
            _bind(root, self.ctxt)
            _trim(root)
            _estimate(root, cfg)
        return roots

    def translateToCompilerPlan(self, plan, translator):
        return [root.translate(translator, self.ctxt) for root in plan]
