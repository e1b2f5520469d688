"""Relational-algebra plan front end.

This module restates the reference plan API (dogqc/relationalAlgebra.py:57-664) so
that plan scripts and plan configs written for DogQC build the same operator trees
here, with the same operator ids, attribute ids, attribute pruning and cardinality
estimates:

* operator ids are handed out bottom-up at construction time
  (relationalAlgebra.py:30-32, 151-152) and ``resolveAlgebraPlan`` appends a result
  materialisation as the root (:129-138);
* ``resolve`` creates attributes and resolves identifiers ("name", "table.name",
  "alias.name"; :301-314, 176-197);
* ``prune`` keeps an attribute in an operator's output only if a later operator
  uses it (:199-204);
* ``configure`` propagates ``tupleNum`` and reads the per-operator hints
  ``selectivity``, ``multimatch`` (default True), ``htSizeFactor`` (default 2.0)
  and ``numgroups`` (default: child cardinality) from the plan config
  (:342-349, 441-458, 564-574).

The backend (``dogqc_b200.backend.Backend``) reads only the attributes named above,
so it also accepts trees built with the reference's own classes.
"""
from collections import OrderedDict
from enum import Enum

from dogqc_b200.types import Type


def listWrap(elem):
    return elem if isinstance(elem, list) else [elem]


class Attribute(object):
    def __init__(self, name, id, opId):
        self.name = name
        self.id = id
        self.creation = opId
        self.numElements = None
        self.lastUse = 0
        self.dataType = None
        self.identifiers = [name]


class Context(object):
    def __init__(self, database):
        self.database = database
        self.schema = dict(database.schema)
        self.opIdNum = 0
        self.attributeIdNum = 0
        self.tableVersions = dict()

    def opId(self):
        self.opIdNum += 1
        return self.opIdNum

    def createTable(self, identifier):
        table = {"name": identifier, "attributes": OrderedDict()}
        self.schema[identifier] = table
        return table

    def resolveTable(self, identifier):
        table = self.schema[identifier]
        version = self.tableVersions.get(identifier, 0) + 1
        self.tableVersions[identifier] = version
        return version, table

    def createAttribute(self, attributeName, tableName=None):
        self.attributeIdNum += 1
        attr = Attribute(attributeName, self.attributeIdNum, self.opIdNum)
        return self.attributeIdNum, attr


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


class AlgExpr(object):
    def __init__(self, ctxt):
        self.opId = ctxt.opId()
        self.inRelation = dict()
        self.outRelation = dict()

    def resolve(self, ctxt):
        pass

    def prune(self):
        pass

    def configure(self, cfg, ctxt):
        pass

    def translate(self, translator, ctxt):
        pass

    def children(self):
        return []

    def touchAttribute(self, id):
        self.inRelation[id].lastUse = self.opId

    def resolveAttribute(self, identifier):
        known, ambiguous = {}, set()
        for id, att in self.inRelation.items():
            for ident in att.identifiers:
                if ident in known:
                    ambiguous.add(ident)
                else:
                    known[ident] = id
        if identifier in ambiguous:
            raise SyntaxError("Identifier %s is ambiguous in operator %s (%d)"
                              % (identifier, type(self).__name__, self.opId))
        if identifier not in known:
            raise NameError("Attribute %s not found in %s operator (%d)"
                            % (identifier, type(self).__name__, self.opId))
        id = known[identifier]
        self.touchAttribute(id)
        return self.inRelation[id]

    def pruneOutRelation(self):
        self.outRelation = {id: a for id, a in self.outRelation.items()
                            if a.lastUse > self.opId}

    @staticmethod
    def _cfg(cfg, opId, key, default):
        try:
            return cfg[opId][key]
        except (KeyError, TypeError, IndexError):
            return default


class LiteralAlgExpr(AlgExpr):
    def prune(self):
        self.pruneOutRelation()

    def translate(self, translator, ctxt):
        return translator.translate(self)


class UnaryAlgExpr(AlgExpr):
    def __init__(self, ctxt, child):
        AlgExpr.__init__(self, ctxt)
        self.child = child

    def children(self):
        return [self.child]

    def prune(self):
        self.child.prune()
        self.pruneOutRelation()

    def translate(self, translator, ctxt):
        return translator.translate(self, self.child.translate(translator, ctxt))


class BinaryAlgExpr(AlgExpr):
    def __init__(self, ctxt, leftChild, rightChild):
        AlgExpr.__init__(self, ctxt)
        self.leftChild = leftChild
        self.rightChild = rightChild

    def children(self):
        return [self.leftChild, self.rightChild]

    def prune(self):
        self.leftChild.prune()
        self.rightChild.prune()
        self.pruneOutRelation()

    def translate(self, translator, ctxt):
        left = self.leftChild.translate(translator, ctxt)
        right = self.rightChild.translate(translator, ctxt)
        return translator.translate(self, left, right)


class Scan(LiteralAlgExpr):
    def __init__(self, ctxt, tableName, alias=None):
        LiteralAlgExpr.__init__(self, ctxt)
        self.scanAttributes = dict()
        self.scanTableId, self.table = ctxt.resolveTable(tableName)
        self.isTempScan = "isTempTable" in self.table
        self.tableAlias = alias

    def resolve(self, ctxt):
        for attrName, typ in self.table["attributes"].items():
            id, attr = ctxt.createAttribute(attrName, self.table["name"])
            attr.dataType = typ
            attr.numElements = self.table["size"]
            attr.identifiers.append(self.table["name"] + "." + attrName)
            if self.tableAlias is not None:
                attr.identifiers.append(self.tableAlias + "." + attrName)
            if self.isTempScan:
                attr.sourceId = self.table["sourceAttributes"][attrName]
            self.scanAttributes[id] = attr
        self.outRelation = self.scanAttributes
        return self.outRelation

    def configure(self, cfg, ctxt):
        self.tupleNum = self.table["size"]
        return self.tupleNum


class Selection(UnaryAlgExpr):
    def __init__(self, ctxt, condition, child):
        UnaryAlgExpr.__init__(self, ctxt, child)
        self.condition = condition

    def resolve(self, ctxt):
        self.inRelation = self.child.resolve(ctxt)
        self.conditionAttributes = self.condition.resolve(self)
        self.outRelation = self.inRelation
        return self.outRelation

    def configure(self, cfg, ctxt):
        childNum = self.child.configure(cfg, ctxt)
        self.selectivity = self._cfg(cfg, self.opId, "selectivity", 1.0)
        self.tupleNum = int(childNum * self.selectivity)
        return self.tupleNum


class Map(UnaryAlgExpr):
    def __init__(self, ctxt, attrName, expression, child):
        UnaryAlgExpr.__init__(self, ctxt, child)
        self.expression = expression
        self.attrName = attrName

    def resolve(self, ctxt):
        self.inRelation = self.child.resolve(ctxt)
        used = self.expression.resolve(self)
        id, attr = ctxt.createAttribute(self.attrName)
        attr.dataType = self.expression.type
        self.mapAttr = attr
        self.mapStringAttributes = [a for a in used.values() if a.dataType == Type.STRING]
        out = dict(self.inRelation)
        out[attr.id] = attr
        self.outRelation = out
        return out

    def configure(self, cfg, ctxt):
        self.tupleNum = self.child.configure(cfg, ctxt)
        return self.tupleNum


class EquiJoin(BinaryAlgExpr):
    def __init__(self, ctxt, joinType, equalityConditions, otherConditions, leftChild, rightChild):
        BinaryAlgExpr.__init__(self, ctxt, leftChild, rightChild)
        self.equalities = listWrap(equalityConditions)
        self.conditions = otherConditions
        self.joinType = joinType

    def resolve(self, ctxt):
        inLeft = self.leftChild.resolve(ctxt)
        self.inRelation.update(inLeft)
        inRight = self.rightChild.resolve(ctxt)
        self.inRelation.update(inRight)
        condAtts = self.conditions.resolve(self) if self.conditions is not None else {}
        self.conditionProbeAttributes = {id: a for id, a in condAtts.items() if id in inRight}
        self.buildKeyAttributes = OrderedDict()
        self.probeKeyAttributes = OrderedDict()
        for ident1, ident2 in self.equalities:
            a1 = self.resolveAttribute(ident1)
            a2 = self.resolveAttribute(ident2)
            if a1.id in inLeft and a2.id in inRight:
                self.buildKeyAttributes[a1.id] = a1
                self.probeKeyAttributes[a2.id] = a2
            elif a1.id in inRight and a2.id in inLeft:
                self.buildKeyAttributes[a2.id] = a2
                self.probeKeyAttributes[a1.id] = a1
            else:
                raise NameError("Attributes %s and %s come from the same relation."
                                % (a1.name, a2.name))
        if self.joinType in (Join.INNER, Join.OUTER):
            self.outRelation = self.inRelation
        else:
            self.outRelation = inRight
        return self.outRelation

    def configure(self, cfg, ctxt):
        left = self.leftChild.configure(cfg, ctxt)
        right = self.rightChild.configure(cfg, ctxt)
        self.multimatch = self._cfg(cfg, self.opId, "multimatch", True)
        self.selectivity = self._cfg(cfg, self.opId, "selectivity", 1.0)
        self.htSizeFactor = self._cfg(cfg, self.opId, "htSizeFactor", 2.0)
        self.tupleNum = int(max(left, right) * self.selectivity)
        return self.tupleNum


class CrossJoin(BinaryAlgExpr):
    def __init__(self, ctxt, joinType, condition, leftChild, rightChild):
        BinaryAlgExpr.__init__(self, ctxt, leftChild, rightChild)
        self.condition = condition
        self.joinType = joinType

    def resolve(self, ctxt):
        self.inRelation.update(self.leftChild.resolve(ctxt))
        self.inRelation.update(self.rightChild.resolve(ctxt))
        self.conditionAttributes = self.condition.resolve(self)
        self.outRelation = self.inRelation
        return self.outRelation

    def configure(self, cfg, ctxt):
        left = self.leftChild.configure(cfg, ctxt)
        right = self.rightChild.configure(cfg, ctxt)
        self.multimatch = self._cfg(cfg, self.opId, "multimatch", True)
        self.selectivity = self._cfg(cfg, self.opId, "selectivity", 1.0)
        self.tupleNum = int(left * right * self.selectivity)
        return self.tupleNum


class Aggregation(UnaryAlgExpr):
    def __init__(self, ctxt, groupingIdentifiers, aggregates, child):
        UnaryAlgExpr.__init__(self, ctxt, child)
        self.groupingIdentifiers = listWrap(groupingIdentifiers)
        self.aggregates = listWrap(aggregates)
        self.aggregateTuplesCreated = OrderedDict()
        self.aggregateAttributes = dict()
        self.avgAggregates = dict()
        # AVG needs a COUNT next to it (relationalAlgebra.py:528-531)
        if any(a[0] == Reduction.AVG for a in self.aggregates):
            if not any(a[0] == Reduction.COUNT for a in self.aggregates):
                self.aggregates.append((Reduction.COUNT, "", "count_agg"))
        for reduction, inputIdentifier, alias in self.aggregates:
            id, attr = ctxt.createAttribute(alias)
            attr.dataType = Type.DOUBLE
            if reduction == Reduction.COUNT:
                attr.dataType = Type.INT
                self.countAttr = attr
            self.aggregateAttributes[id] = attr
            if reduction == Reduction.AVG:
                self.avgAggregates[id] = attr
            self.aggregateTuplesCreated[id] = (attr, inputIdentifier, reduction)

    def resolve(self, ctxt):
        self.inRelation = self.child.resolve(ctxt)
        self.groupAttributes = OrderedDict()
        for ident in self.groupingIdentifiers:
            a = self.resolveAttribute(ident)
            self.groupAttributes[a.id] = a
        self.aggregateInAttributes = OrderedDict()
        self.aggregateTuples = dict()
        for id, (attr, inputIdentifier, reduction) in self.aggregateTuplesCreated.items():
            inId = None
            if inputIdentifier != "":
                inAtt = self.resolveAttribute(inputIdentifier)
                self.aggregateInAttributes[inAtt.id] = inAtt
                inId = inAtt.id
            self.aggregateTuples[id] = (inId, reduction)
        self.outRelation.update(self.groupAttributes)
        self.outRelation.update(self.aggregateAttributes)
        return self.outRelation

    def configure(self, cfg, ctxt):
        childNum = self.child.configure(cfg, ctxt)
        self.doGroup = len(self.groupAttributes) > 0
        self.numgroups = self._cfg(cfg, self.opId, "numgroups", childNum)
        if not self.doGroup:
            self.numgroups = 1
        self.tupleNum = self.numgroups
        return self.tupleNum


class Projection(UnaryAlgExpr):
    def __init__(self, ctxt, identifiers, child):
        UnaryAlgExpr.__init__(self, ctxt, child)
        self.identifiers = listWrap(identifiers)

    def resolve(self, ctxt):
        self.inRelation = self.child.resolve(ctxt)
        self.projectionAttributes = dict()
        for ident in self.identifiers:
            a = self.resolveAttribute(ident)
            self.projectionAttributes[a.id] = a
        self.outRelation = self.projectionAttributes
        return self.outRelation

    def configure(self, cfg, ctxt):
        self.tupleNum = self.child.configure(cfg, ctxt)
        return self.tupleNum


class Materialize(UnaryAlgExpr):
    @staticmethod
    def result(ctxt, child):
        m = Materialize(ctxt, child)
        m.matType = MaterializationType.RESULT
        return m

    @staticmethod
    def temp(ctxt, identifier, child):
        m = Materialize(ctxt, child)
        m.table = ctxt.createTable(identifier)
        m.table["isTempTable"] = True
        m.matType = MaterializationType.TEMPTABLE
        return m

    def resolve(self, ctxt):
        self.inRelation = self.child.resolve(ctxt)
        for id in self.inRelation:
            self.touchAttribute(id)
        if self.matType == MaterializationType.TEMPTABLE:
            self.table["sourceAttributes"] = dict()
            for id, a in self.inRelation.items():
                self.table["attributes"][a.name] = a.dataType
                self.table["sourceAttributes"][a.name] = a.id
            self.table["numColumns"] = len(self.inRelation)
        self.outRelation = self.inRelation
        return self.outRelation

    def prune(self):
        # the materialisation keeps everything its child delivers (:640-642)
        self.child.prune()

    def configure(self, cfg, ctxt):
        self.tupleNum = self.child.configure(cfg, ctxt)
        if self.matType == MaterializationType.TEMPTABLE:
            self.table["size"] = self.tupleNum
        return self.tupleNum


class RelationalAlgebra(object):
    """Plan builder with the reference's method names (relationalAlgebra.py:57-144)."""

    def __init__(self, acc):
        self.ctxt = Context(acc)
        self.selectionNodes = []
        self.joinNodes = []
        self.semiJoinNodes = []
        self.antiJoinNodes = []

    def scan(self, table, alias=None):
        return Scan(self.ctxt, table, alias)

    def selection(self, condition, child):
        node = Selection(self.ctxt, condition, child)
        self.selectionNodes.append(node)
        return node

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
        node = EquiJoin(self.ctxt, Join.INNER, equalityConditions, otherConditions, leftChild, rightChild)
        self.joinNodes.append(node)
        return node

    def semijoin(self, equalityConditions, otherConditions, leftChild, rightChild):
        node = EquiJoin(self.ctxt, Join.SEMI, equalityConditions, otherConditions, leftChild, rightChild)
        self.semiJoinNodes.append(node)
        return node

    def antijoin(self, equalityConditions, otherConditions, leftChild, rightChild):
        node = EquiJoin(self.ctxt, Join.ANTI, equalityConditions, otherConditions, leftChild, rightChild)
        self.antiJoinNodes.append(node)
        return node

    def outerjoin(self, equalityConditions, otherConditions, leftChild, rightChild):
        return EquiJoin(self.ctxt, Join.OUTER, equalityConditions, otherConditions, leftChild, rightChild)

    def aggregation(self, groupAttributes, aggregates, child):
        return Aggregation(self.ctxt, groupAttributes, aggregates, child)

    def resolveAlgebraPlan(self, plan, cfg):
        plan = listWrap(plan)
        plan[-1] = self.result(plan[-1])
        for node in plan:
            node.resolve(self.ctxt)
            node.prune()
            node.configure(cfg, self.ctxt)
        return plan

    def translateToCompilerPlan(self, plan, translator):
        return [node.translate(translator, self.ctxt) for node in plan]
