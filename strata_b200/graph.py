"""graph: the public way to build a pipeline (graph/graph.go, plan.go,
run.go), for the chains the device runs as one pass.

A Graph holds named inputs, nodes and named outputs. Plan lowers every
output whose value is one stencil op (terrain or focal) over an input,
followed by pointwise Lookup / Reclass / Rescale / RescaleRange / Clamp
nodes, to one device pass: strata_process with the stencil stage first and
the pointwise stages fused as its epilogue, as exec.Pipeline runs Slope -> Lookup -> Reclass
(graph/run.go:390-486, internal/exec/pipeline.go:187). A pointwise chain
straight over an input is a pass of its own. Anything else (two stencils
in a row, binary ops, reductions) raises NotSupported, the cue for a
caller to run the reference's CPU planner instead.

    g = graph.New()
    dem = g.Input("dem")
    cls = graph.Reclass(graph.Lookup(graph.Slope(dem, terrain.SlopeOptions(CellSize=10)), xs, ys), breaks, values)
    g.Output("class", cls)
    g.Plan().Run(ctx, {"dem": r}, {"class": out}, engine.Options())
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

from . import engine, focal, terrain, transfer
from ._lib import OP_MAX, OP_MEAN, OP_MIN
from .raster import NotSupported, StrataPanic


@dataclass
class _Node:
    kind: str  # "input", "stencil", "pointwise"
    label: str
    stage: Optional[Callable[[], engine.StageList]] = None
    src: Optional[int] = None
    name: Optional[str] = None


class Graph:
    def __init__(self):
        self.nodes: List[_Node] = []
        self.inputs: Dict[str, int] = {}
        self.outputs: Dict[str, int] = {}

    def _add(self, n: _Node) -> "Node":
        self.nodes.append(n)
        return Node(self, len(self.nodes) - 1)

    def Input(self, name: str) -> "Node":
        if name in self.inputs:
            raise StrataPanic(f"graph: input {name!r} declared twice")
        node = self._add(_Node("input", name, name=name))
        self.inputs[name] = node.v
        return node

    def Output(self, name: str, n: "Node") -> None:
        self._check("Output", n)
        if name in self.outputs or name in self.inputs:
            raise StrataPanic(f"graph: name {name!r} used twice")
        self.outputs[name] = n.v

    def _check(self, op: str, *ns: "Node") -> None:
        for n in ns:
            if n.g is not self:
                raise StrataPanic(f"graph: {op}: node from another graph")

    def Plan(self) -> "Plan":
        passes = {}
        for name, v in self.outputs.items():
            chain = []
            while self.nodes[v].kind == "pointwise":
                chain.append(v)
                v = self.nodes[v].src
            head = self.nodes[v]
            if head.kind == "stencil":
                if self.nodes[head.src].kind != "input":
                    raise NotSupported("graph: a stencil over a computed value is not one device pass")
                chain.append(v)
                src = self.nodes[head.src].name
            elif head.kind == "input":
                if not chain:
                    raise NotSupported("graph: an output that is an input needs no device pass")
                src = head.name
            else:
                raise NotSupported(f"graph: {head.label} is not on the device path")
            passes[name] = (src, list(reversed(chain)))
        return Plan(self, passes)


@dataclass
class Node:
    g: Graph
    v: int


def _stencil(op: str, n: Node, make) -> Node:
    n.g._check(op, n)
    return n.g._add(_Node("stencil", op, make, n.v))


def _pointwise(op: str, n: Node, make) -> Node:
    n.g._check(op, n)
    return n.g._add(_Node("pointwise", op, make, n.v))


def Slope(dem: Node, opts: terrain.SlopeOptions) -> Node:
    terrain.slope_stage(opts)  # the option checks run when the node is built, as in the reference
    return _stencil("terrain.Slope", dem, lambda: terrain.slope_stage(opts))


def Aspect(dem: Node, opts: terrain.AspectOptions) -> Node:
    terrain.aspect_stage(opts)
    return _stencil("terrain.Aspect", dem, lambda: terrain.aspect_stage(opts))


def Hillshade(dem: Node, opts: terrain.HillshadeOptions) -> Node:
    terrain.hillshade_stage(opts)
    return _stencil("terrain.Hillshade", dem, lambda: terrain.hillshade_stage(opts))


def Curvature(dem: Node, opts: terrain.CurvatureOptions) -> Node:
    terrain.curvature_stage(opts)
    return _stencil("terrain.Curvature", dem, lambda: terrain.curvature_stage(opts))


def Ruggedness(dem: Node, opts: terrain.RuggednessOptions) -> Node:
    terrain.ruggedness_stage(opts)
    return _stencil("terrain.Ruggedness", dem, lambda: terrain.ruggedness_stage(opts))


def FocalMean(src: Node, opts: focal.BoxOptions) -> Node:
    focal.box_stage(opts, OP_MEAN)
    return _stencil("focal.Mean", src, lambda: focal.box_stage(opts, OP_MEAN))


def FocalMin(src: Node, opts: focal.BoxOptions) -> Node:
    focal.box_stage(opts, OP_MIN)
    return _stencil("focal.Min", src, lambda: focal.box_stage(opts, OP_MIN))


def FocalMax(src: Node, opts: focal.BoxOptions) -> Node:
    focal.box_stage(opts, OP_MAX)
    return _stencil("focal.Max", src, lambda: focal.box_stage(opts, OP_MAX))


def Correlate(src: Node, opts: focal.WeightsOptions) -> Node:
    focal.weights_stage(opts, False)
    return _stencil("focal.Correlate", src, lambda: focal.weights_stage(opts, False))


def Convolve(src: Node, opts: focal.WeightsOptions) -> Node:
    focal.weights_stage(opts, True)
    return _stencil("focal.Convolve", src, lambda: focal.weights_stage(opts, True))


def CorrelateSeparable(src: Node, opts: focal.SeparableOptions) -> Node:
    focal.separable_stage(opts)
    return _stencil("focal.CorrelateSeparable", src, lambda: focal.separable_stage(opts))


def Lookup(src: Node, xs, ys) -> Node:
    transfer.lookup_stage(xs, ys)
    xs, ys = list(xs), list(ys)
    return _pointwise("transfer.Lookup", src, lambda: transfer.lookup_stage(xs, ys))


def Reclass(src: Node, breaks, values) -> Node:
    transfer.reclass_stage(breaks, values)
    breaks, values = list(breaks), list(values)
    return _pointwise("transfer.Reclass", src, lambda: transfer.reclass_stage(breaks, values))


def Rescale(src: Node, a: float, b: float) -> Node:
    """transfer.Rescale as a chain step (vec.OpAffine) of the pass."""
    return _pointwise("transfer.Rescale", src, lambda: transfer.rescale_stage(a, b))


def RescaleRange(src: Node, in_lo: float, in_hi: float, out_lo: float, out_hi: float) -> Node:
    transfer.rescale_range_stage(in_lo, in_hi, out_lo, out_hi)
    return _pointwise("transfer.RescaleRange", src,
                      lambda: transfer.rescale_range_stage(in_lo, in_hi, out_lo, out_hi))


def Clamp(src: Node, lo: float, hi: float) -> Node:
    """algebra.Clamp as a chain step (vec.OpClamp) of the pass."""
    from . import algebra

    return _pointwise("algebra.Clamp", src, lambda: algebra.clamp_stage(lo, hi))


class Plan:
    """The passes of a Graph: per output, its input and the stage chain run
    as one device pass."""

    def __init__(self, g: Graph, passes):
        self.g = g
        self.passes = passes

    def String(self) -> str:
        out = []
        for name, (src, chain) in self.passes.items():
            labels = " -> ".join(self.g.nodes[v].label for v in chain)
            out.append(f"pass {name}: {src} -> {labels}")
        return "\n".join(out)

    def _stages(self, chain) -> engine.StageList:
        sl = engine.StageList()
        for v in chain:
            sl.extend(self.g.nodes[v].stage())
        return sl

    def Run(self, ctx: engine.Context, inp: Dict, out: Dict, opts: Optional[engine.Options] = None):
        """Runs every pass over rasters in memory (graph/run.go:51).
        Returns None or the first error (a cancelled context)."""
        self._bind(inp, out)
        for name, (src, chain) in self.passes.items():
            err = engine.process(self._stages(chain), [out[name]], [inp[src]], opts, ctx)
            if err is not None:
                return err
        return None

    def RunChunked(self, ctx: engine.Context, inp: Dict, out: Dict, opts: Optional[engine.Options] = None):
        """Runs every pass over sources and sinks (graph/run.go:167)."""
        self._bind(inp, out)
        for name, (src, chain) in self.passes.items():
            err = engine.process_chunked(self._stages(chain), [out[name]], [inp[src]], opts, ctx)
            if err is not None:
                return err
        return None

    def _bind(self, inp, out):
        for name in self.g.inputs:
            if name not in inp:
                raise StrataPanic(f"graph: input {name!r} is not bound")
        for name in self.passes:
            if name not in out:
                raise StrataPanic(f"graph: output {name!r} is not bound")


def New() -> Graph:
    return Graph()
