"""Scalar expressions of the plan front end.

Same class names, constructor arguments and typing rules as the reference
(dogqc/scalarAlgebra.py:1-464), so plan scripts written against the reference
(``scal.MulExpr(scal.AttrExpr("x"), scal.ConstExpr("100", Type.INT))``) build the
same trees here.  Typing rules kept from the reference:

* a binary expression whose operands have equal types takes that type, otherwise
  DOUBLE (scalarAlgebra.py:84-87), including comparisons and logic operators;
* arithmetic nodes start as INT (scalarAlgebra.py:382), unary nodes take the type
  of their child (scalarAlgebra.py:54-57), CASE is FLOAT (scalarAlgebra.py:259),
  SUBSTRING is STRING;
* ``EqualsExpr`` rejects operands of different types unless one is FLOAT
  (scalarAlgebra.py:173-181) and ``LikeExpr`` needs two STRING operands
  (scalarAlgebra.py:196-203).

There is no code emission here: the backend lowers these trees into its own
expression program (``dogqc_b200.lowering``).
"""
from enum import Enum

from dogqc_b200.types import Type


class ScalarExpr(object):
    _next_id = 1000

    def __init__(self):
        self.type = None
        self.exprId = ScalarExpr._next_id
        ScalarExpr._next_id += 1

    def children(self):
        return []


class AttrExpr(ScalarExpr):
    def __init__(self, identifier):
        ScalarExpr.__init__(self)
        self.identifier = identifier

    def resolve(self, algExpr):
        self.attr = algExpr.resolveAttribute(self.identifier)
        self.type = self.attr.dataType
        return {self.attr.id: self.attr}


class ConstExpr(ScalarExpr):
    def __init__(self, token, type):
        ScalarExpr.__init__(self)
        self.token = token
        self.type = type

    def resolve(self, algExpr):
        return {}


class _Binary(ScalarExpr):
    def __init__(self, leftChild, rightChild):
        ScalarExpr.__init__(self)
        self.leftChild = leftChild
        self.rightChild = rightChild

    def children(self):
        return [self.leftChild, self.rightChild]

    def resolve(self, algExpr):
        found = dict(self.leftChild.resolve(algExpr))
        found.update(self.rightChild.resolve(algExpr))
        lt, rt = self.leftChild.type, self.rightChild.type
        self.type = lt if lt == rt else Type.DOUBLE
        self._check()
        return found

    def _check(self):
        pass


class _Unary(ScalarExpr):
    def __init__(self, child):
        ScalarExpr.__init__(self)
        self.child = child

    def children(self):
        return [self.child]

    def resolve(self, algExpr):
        found = self.child.resolve(algExpr)
        self.type = self.child.type
        return found


class EqualsExpr(_Binary):
    def _check(self):
        lt, rt = self.leftChild.type, self.rightChild.type
        if Type.FLOAT not in (lt, rt) and lt != rt:
            raise SyntaxError("Comparing unmatched types: %s and %s in scalar expr %d"
                              % (lt, rt, self.exprId))
        self.comparisonType = lt


class LikeExpr(_Binary):
    def _check(self):
        lt, rt = self.leftChild.type, self.rightChild.type
        if lt != rt:
            raise SyntaxError("Comparing unmatched types: %s and %s in scalar expr %d"
                              % (lt, rt, self.exprId))
        if lt != Type.STRING:
            raise SyntaxError("Prefix check only for strings.")
        self.comparisonType = lt


class SubstringExpr(ScalarExpr):
    def __init__(self, exprString, exprFrom, exprFor):
        ScalarExpr.__init__(self)
        self.exprString = exprString
        self.exprFrom = exprFrom
        self.exprFor = exprFor
        self.type = Type.STRING

    def children(self):
        return [self.exprString, self.exprFrom, self.exprFor]

    def resolve(self, algExpr):
        found = {}
        for e in self.children():
            found.update(e.resolve(algExpr))
        if self.exprString.type != Type.STRING:
            raise SyntaxError("Need STRING type, type is: " + str(self.exprString.type))
        for e in (self.exprFrom, self.exprFor):
            if e.type != Type.INT:
                raise SyntaxError("Need INT type, type is: " + str(e.type))
        return found


class CaseExpr(ScalarExpr):
    def __init__(self, exprListWhenThen, exprElse=None):
        ScalarExpr.__init__(self)
        if len(exprListWhenThen) == 0:
            raise SyntaxError("The case expression needs at least one when clause.")
        self.exprListWhenThen = exprListWhenThen
        self.exprElse = exprElse
        self.type = Type.FLOAT

    def children(self):
        out = []
        for w, t in self.exprListWhenThen:
            out += [w, t]
        if self.exprElse is not None:
            out.append(self.exprElse)
        return out

    def resolve(self, algExpr):
        found = {}
        for e in self.children():
            found.update(e.resolve(algExpr))
        return found


class AndExpr(_Binary):
    pass


class OrExpr(_Binary):
    pass


class NotExpr(_Unary):
    pass


def InExpr(v, exprList):
    """``v IN (e1, e2, ...)`` as a disjunction of equalities (scalarAlgebra.py:330-334)."""
    tree = EqualsExpr(v, exprList[0])
    for e in exprList[1:]:
        tree = OrExpr(EqualsExpr(v, e), tree)
    return tree


class SmallerExpr(_Binary):
    pass


class SmallerEqualExpr(_Binary):
    pass


class LargerExpr(_Binary):
    pass


class LargerEqualExpr(_Binary):
    pass


class MulExpr(_Binary):
    pass


class DivExpr(_Binary):
    pass


class AddExpr(_Binary):
    pass


class SubExpr(_Binary):
    pass


class AbsExpr(_Unary):
    pass


class ExtractType(Enum):
    DAY = 1
    MONTH = 2
    YEAR = 3


class ExtractExpr(_Unary):
    def __init__(self, child, extractType):
        _Unary.__init__(self, child)
        self.extract = extractType
