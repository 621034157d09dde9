"""vec: the fused pointwise chain (internal/vec/chain.go) on the device.

A Chain is a left-deep sequence of pointwise operations run as one pass:
the running value starts as one input and is the first operand of every
step; a binary step (Add .. Max) takes a second input as its other
operand, the rest use the immediates K. NewChain applies the reference's
checks (chain.go:106-132) and Run computes dst from the inputs on the
device (strata_process with STRATA_OP_STEP stages: one kernel, the
running value in a register, and the output's validity the AND of the
masked inputs'). The same steps fuse after a stencil as the pointwise
tail of a pipeline (graph.Rescale, transfer.rescale_stage, algebra's
clamp_stage), where only the unary ops apply.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence, Tuple

from . import _lib
from .engine import Options, StageList, process
from .raster import Float32Raster, StrataPanic

# vec.Op (internal/vec/chain.go:24-38)
OpAdd, OpSub, OpMul, OpDiv, OpMin, OpMax = (_lib.VEC_ADD, _lib.VEC_SUB, _lib.VEC_MUL, _lib.VEC_DIV, _lib.VEC_MIN,
                                            _lib.VEC_MAX)
OpAddScalar, OpMulScalar, OpAffine, OpSubDiv = (_lib.VEC_ADD_SCALAR, _lib.VEC_MUL_SCALAR, _lib.VEC_AFFINE,
                                                _lib.VEC_SUB_DIV)
OpClamp, OpAbs, OpSqrt = _lib.VEC_CLAMP, _lib.VEC_ABS, _lib.VEC_SQRT
MaxSteps = _lib.MAX_STEPS

_NAMES = ["Add", "Sub", "Mul", "Div", "Min", "Max", "AddScalar", "MulScalar", "Affine", "SubDiv", "Clamp", "Abs",
          "Sqrt"]


def op_name(op: int) -> str:
    return _NAMES[op] if 0 <= op < len(_NAMES) else f"Op({op})"


def binary(op: int) -> bool:
    """Op.Binary: whether op reads a source slice."""
    return op <= OpMax


@dataclass
class Step:
    """vec.Step: the operation, the input a binary op reads (-1 for the
    others) and the immediates."""
    Op: int
    Src: int = -1
    K: Tuple[float, float] = (0.0, 0.0)


def step_stage(op: int, src: int = -1, k0: float = 0.0, k1: float = 0.0) -> StageList:
    """One chain step as a pipeline stage."""
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_step(op, src, k0, k1, ctypes.byref(st)))
    return StageList().add(st)


class Chain:
    """vec.Chain: inputs source rasters, the running value starting at
    srcs[first], then the steps."""

    def __init__(self, inputs: int, first: int, steps: Sequence[Step]):
        if inputs < 1:
            raise StrataPanic(f"vec: chain has {inputs} inputs; it needs at least one")
        if first < 0 or first >= inputs:
            raise StrataPanic(f"vec: chain starts from input {first}, which is not one of its {inputs}")
        if len(steps) == 0:
            raise StrataPanic("vec: chain has no steps")
        if len(steps) > MaxSteps:
            raise StrataPanic(f"vec: chain has {len(steps)} steps, at most {MaxSteps} fit")
        for i, s in enumerate(steps):
            if not 0 <= s.Op <= OpSqrt:
                raise StrataPanic(f"vec: chain step {i} has unknown operation {op_name(s.Op)}")
            if binary(s.Op) and not 0 <= s.Src < inputs:
                raise StrataPanic(f"vec: chain step {i} ({op_name(s.Op)}) reads input {s.Src}, which is not one "
                                  f"of its {inputs}")
            if not binary(s.Op) and s.Src != -1:
                raise StrataPanic(f"vec: chain step {i} ({op_name(s.Op)}) reads no input, so its Src must be -1, "
                                  f"not {s.Src}")
        if inputs > _lib.MAX_INPUTS:
            from .raster import NotSupported

            raise NotSupported(f"vec: the gpu backend takes at most {_lib.MAX_INPUTS} chain inputs, got {inputs}")
        self.inputs, self.first, self.steps = inputs, first, list(steps)

    def Inputs(self) -> int:
        return self.inputs

    def Steps(self) -> int:
        return len(self.steps)

    def _order(self):
        """The device chain starts at input 0: srcs[first] goes first, and
        input 0 takes first's place."""
        perm = list(range(self.inputs))
        perm[0], perm[self.first] = perm[self.first], perm[0]
        return perm

    def stages(self) -> StageList:
        perm = self._order()
        where = {orig: pos for pos, orig in enumerate(perm)}
        out = StageList()
        for s in self.steps:
            out.extend(step_stage(s.Op, where[s.Src] if binary(s.Op) else -1, s.K[0], s.K[1]))
        return out

    def Run(self, dst: Float32Raster, srcs: Sequence[Float32Raster], opts: Options = None):
        """Chain.Run over rasters: dst from srcs cell by cell, on the device."""
        if len(srcs) != self.inputs:
            raise StrataPanic(f"vec: chain takes {self.inputs} inputs, Run got {len(srcs)}")
        ordered = [srcs[i] for i in self._order()]
        return process(self.stages(), [dst], ordered, opts or Options(Workers=1))


def NewChain(inputs: int, first: int, steps: Sequence[Step]) -> Chain:
    return Chain(inputs, first, steps)
