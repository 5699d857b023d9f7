"""Truncation policies (the ``TruncationPolicy`` built-ins) and their lowering.

``coeff(eps)`` keeps ``|c|^2 > eps^2`` (crates/paulistrings/src/truncation/builtin.rs:19-41),
``weight(k)`` keeps Pauli weight ``<= k`` (:43-59), ``topn(n)`` retains the ``n`` largest
magnitudes after every layer (:61-150), ``approx_topn(n)`` cuts at an octave of |c|^2 instead
(:240-468), ``collapse_sample(cache, samples, seed)`` resamples by |c| above a cache
(collapse_sample.rs), ``scored_topn(n, scorer)`` the ``n`` terms a learned
scorer ranks highest (``paulistrings_b200.learned``; a ``TruncationPolicy`` of this package,
crates/paulistrings/src/truncation/mod.rs:30-107).  ``a & b`` keeps a term iff both keep it and runs
a's layer passes then b's (:470-526); ``a | b`` combines per-term filters only (:574-625).
A policy lowers to a postfix keep program plus an ordered list of layer passes, the form
``ps_policy`` carries across the C ABI (KeepProgram, crates/paulistrings/src/engine/gpu/
truncation.rs:24-102).
"""

from __future__ import annotations

from . import _lib


class Truncation:
    """A truncation policy tree."""

    def __init__(self, kind: str, *args):
        self.kind = kind
        self.args = args

    def __and__(self, other: "Truncation") -> "Truncation":
        return Truncation("and", self, other)

    def __or__(self, other: "Truncation") -> "Truncation":
        for side, name in ((self, "first"), (other, "second")):
            if side.has_layer_pass():
                raise ValueError(
                    f"Or combines per-term filters only, but its {name} operand has a layer pass "
                    "(TopN); use & to add a filter to a layer pass"
                )
        return Truncation("or", self, other)

    def has_layer_pass(self) -> bool:
        if self.kind in ("topn", "scored_topn", "approx_topn", "collapse_sample"):
            return True
        if self.kind in ("and", "or"):
            return self.args[0].has_layer_pass() or self.args[1].has_layer_pass()
        return False

    def __repr__(self) -> str:
        if self.kind in ("and", "or"):
            op = " & " if self.kind == "and" else " | "
            return f"({self.args[0]!r}{op}{self.args[1]!r})"
        if self.kind == "scored_topn":
            return f"truncation.scored_topn({self.args[0]!r}, <scorer>, rescore_every={self.args[2]!r})"
        if self.kind == "collapse_sample":
            return f"truncation.collapse_sample({self.args[0]!r}, {self.args[1]!r}, {self.args[2]!r})"
        return f"truncation.{self.kind}({', '.join(repr(a) for a in self.args)})"

    # -- lowering ----------------------------------------------------------
    def _lower(self, nodes: list, passes: list) -> None:
        if self.kind == "coeff":
            nodes.append((_lib.PS_KEEP_COEFF, 0, float(self.args[0])))
        elif self.kind == "weight":
            nodes.append((_lib.PS_KEEP_WEIGHT, int(self.args[0]), 0.0))
        elif self.kind == "topn":
            nodes.append((_lib.PS_KEEP_TRUE, 0, 0.0))
            passes.append((_lib.PS_PASS_TOPN, int(self.args[0])))
        elif self.kind == "scored_topn":
            nodes.append((_lib.PS_KEEP_TRUE, 0, 0.0))
            passes.append((_lib.PS_PASS_SCORED_TOPN, int(self.args[0]), int(self.args[2]), 0, 0))
        elif self.kind == "approx_topn":
            nodes.append((_lib.PS_KEEP_TRUE, 0, 0.0))
            passes.append((_lib.PS_PASS_APPROX_TOPN, int(self.args[0])))
        elif self.kind == "collapse_sample":
            nodes.append((_lib.PS_KEEP_TRUE, 0, 0.0))
            state = self.args[3]
            passes.append((_lib.PS_PASS_COLLAPSE_SAMPLE, int(self.args[0]), int(self.args[1]), int(self.args[2]),
                           int(state["calls"])))
        elif self.kind in ("and", "or"):
            self.args[0]._lower(nodes, passes)
            self.args[1]._lower(nodes, passes)
            nodes.append((_lib.PS_KEEP_AND if self.kind == "and" else _lib.PS_KEEP_OR, 0, 0.0))
        else:
            raise ValueError(f"unknown truncation {self.kind}")

    def scorer(self):
        """The scorer of the tree's scored_topn pass, or None (at most one scorer per policy)."""
        if self.kind == "scored_topn":
            return self.args[1]
        if self.kind in ("and", "or"):
            a, b = self.args[0].scorer(), self.args[1].scorer()
            if a is not None and b is not None and a is not b:
                raise ValueError("a policy can carry one scorer")
            return a if a is not None else b
        return None

    def lowered(self):
        """(keep nodes, passes) with the keep program simplified of always-true nodes."""
        nodes: list = []
        passes: list = []
        self._lower(nodes, passes)
        nodes = _simplify(nodes)
        if len(nodes) > _lib.PS_MAX_KEEP_NODES:
            raise ValueError("truncation tree too deep for the device keep program (15 nodes)")
        if len(passes) > _lib.PS_MAX_PASSES:
            raise ValueError("at most 4 layer passes")
        return nodes, passes

    def to_c(self) -> _lib.Policy:
        nodes, passes = self.lowered()
        p = _lib.Policy()
        p.num_nodes = len(nodes)
        for i, (op, iarg, farg) in enumerate(nodes):
            p.nodes[i].op = op
            p.nodes[i].iarg = iarg
            p.nodes[i].farg = farg
        p.num_passes = len(passes)
        for i, ps_ in enumerate(passes):
            p.passes[i].kind = ps_[0]
            p.passes[i].n = ps_[1]
            if len(ps_) > 2:
                p.passes[i].samples, p.passes[i].seed, p.passes[i].call = ps_[2], ps_[3], ps_[4]
        return p

    def collapse_states(self):
        """The pass counters of the tree's CollapseSample passes (advanced after each run)."""
        if self.kind == "collapse_sample":
            return [self.args[3]]
        if self.kind in ("and", "or"):
            return self.args[0].collapse_states() + self.args[1].collapse_states()
        return []


def _simplify(nodes: list) -> list:
    """Fold ``true & x`` and ``x & true`` to ``x`` and ``true | x`` to ``true``."""
    stack: list = []
    for node in nodes:
        op = node[0]
        if op in (_lib.PS_KEEP_AND, _lib.PS_KEEP_OR):
            b = stack.pop()
            a = stack.pop()
            a_true = a == [(_lib.PS_KEEP_TRUE, 0, 0.0)]
            b_true = b == [(_lib.PS_KEEP_TRUE, 0, 0.0)]
            if op == _lib.PS_KEEP_AND:
                stack.append(b if a_true else a if b_true else a + b + [node])
            else:
                stack.append(a if a_true else b if b_true else a + b + [node])
        else:
            stack.append([node])
    out = stack[-1] if stack else []
    return [] if out == [(_lib.PS_KEEP_TRUE, 0, 0.0)] else out


def coeff(epsilon: float) -> Truncation:
    return Truncation("coeff", float(epsilon))


def weight(k: int) -> Truncation:
    if k < 0:
        raise ValueError("weight limit must be non-negative")
    return Truncation("weight", int(k))


def topn(n: int) -> Truncation:
    if n < 0:
        raise ValueError("topn needs n >= 0")
    return Truncation("topn", int(n))


def approx_topn(n: int) -> Truncation:
    """ApproxTopN (crates/paulistrings/src/truncation/builtin.rs:240-468): retain ``n`` terms,
    cutting at an octave of ``|c|^2`` — every octave that fits whole from the top, then the
    first terms of the boundary octave in key order; NaN never kept."""
    if n < 0:
        raise ValueError("approx_topn needs n >= 0")
    return Truncation("approx_topn", int(n))


class CollapseSample(Truncation):
    """CollapseSample (crates/paulistrings/src/truncation/collapse_sample.rs): whenever the sum holds
    more than ``cache`` terms after a layer, ``samples`` systematic draws in proportion to |c|
    replace it — an unbiased estimate.  One seed is one trajectory: the uniform of the k-th layer
    pass is a function of (seed, k), and the pass counter lives in the policy, so reusing a policy
    continues its sequence."""

    def __init__(self, cache: int, samples: int, seed: int):
        if samples < 1:
            raise ValueError("CollapseSample: samples must be at least 1")
        super().__init__("collapse_sample", int(cache), int(samples), int(seed) & 0xFFFFFFFFFFFFFFFF,
                         {"calls": 0, "collapses": 0})

    @property
    def calls(self) -> int:
        return self.args[3]["calls"]

    def collapses(self) -> int:
        return self.args[3]["collapses"]


def collapse_sample(cache: int, samples: int, seed: int) -> CollapseSample:
    return CollapseSample(cache, samples, seed)


def scored_topn(n: int, scorer, rescore_every: int = 1) -> Truncation:
    """Keep the ``n`` terms ``scorer`` (a ``paulistrings_b200.learned.Scorer``) ranks highest
    after every layer; ties first in key order, NaN scores never kept.

    ``rescore_every`` > 1 (a residual scorer, the policy's only pass): the network predicts for
    every term only every ``rescore_every`` layers; in the layers between, each term carries its
    prediction (a partner its parent's) and ranks by log|c| + that prediction, so a layer costs
    about what a plain TopN layer costs."""
    if n < 0:
        raise ValueError("scored_topn needs n >= 0")
    if rescore_every < 1:
        raise ValueError("scored_topn needs rescore_every >= 1")
    return Truncation("scored_topn", int(n), scorer, int(rescore_every))


def policy_to_c(policy):
    if policy is None:
        return None
    if not isinstance(policy, Truncation):
        raise TypeError("policy must be a paulistrings_b200.truncation policy or None")
    return policy.to_c()
