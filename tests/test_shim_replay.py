"""The reference's own strokes.py driving the `_strokelib` shim.

The reference's Python layer imports ``_strokelib`` before it JIT-builds its own
(source/strokelib/strokes.py:7-10), so a module of that name on sys.path (the
``neural3dstrokes_b200/shim`` directory) replaces the backend with no edit. The
reference checkout is not available where the GPU tests run, so the proof has two
halves:

1. tests/golden/make_golden.py --strokespy imported the reference strokes.py with a
   recording backend and drove get_stroke / stroke_fn / compose_strokes and the
   backward for every shape type as models.py does (models.py:681-684, 709); the
   log (tests/golden/strokes_py_calls.*) holds exactly the calls strokes.py makes:
   argument order, shapes, dtypes, which outputs arrive zeroed, the scalars, and the
   values (the recording backend computed with the oracle's float32 port).
2. Here every recorded call is replayed, argument for argument, into the shim
   module (imported by name from the shim directory, as strokes.py imports it) and
   into the reference extension built from its sources (oracle/_ref), and the
   results are compared.

Tolerances (normwise): forward 1e-5; compat backward 1e-4 (the reference's
formulas). Curves: the shim's forward is within 1e-5 of float64 and never further
from the reference than the reference is from float64 (its float32 closed-form
Bezier solve); the quadratic Bezier's backward (whose reference adjoint is not
restated) is checked against float64 autograd.
"""
import importlib
import inspect
import json
import os
import sys

import numpy as np
import pytest
import torch

from helpers import FWD_TOL, GRAD_TOL, rel
from neural3dstrokes_b200 import scenes
from neural3dstrokes_b200 import strokelib as sl
from oracle import cpu_port
from oracle import strokefield as sf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
SHIM = os.path.join(ROOT, "neural3dstrokes_b200", "shim")


def log():
    with open(os.path.join(GOLDEN, "strokes_py_calls.json")) as f:
        meta = json.load(f)
    return meta, np.load(os.path.join(GOLDEN, "strokes_py_calls.npz"))


def import_shim():
    """``import _strokelib`` with the shim directory first on sys.path, as the
    reference strokes.py would resolve it."""
    sys.path.insert(0, SHIM)
    try:
        sys.modules.pop("_strokelib", None)
        return importlib.import_module("_strokelib")
    finally:
        sys.path.remove(SHIM)
        sys.modules.pop("_strokelib", None)


def test_recorded_calls_fit_the_shim_signatures():
    """Every call strokes.py made binds to the shim's function of that name with the
    same positional arguments; gradient outputs arrive zeroed and every tensor is a
    contiguous float32 (the reference's own contract, strokes.py:155-166, 206-216,
    332-336, 365-367)."""
    meta, _ = log()
    shim = import_shim()
    assert os.path.dirname(inspect.getsourcefile(shim)) == SHIM
    kinds = {g["kind"] for g in meta["groups"]}
    assert kinds == set(scenes.EVERY_KIND)
    for call in meta["calls"]:
        fn = getattr(shim, call["fn"])
        assert fn is getattr(sl, call["fn"])
        inspect.signature(fn).bind(*[None] * len(call["args"]))
        for a in call["args"]:
            if "tensor" in a:
                assert a["dtype"] == "float32" and a["contiguous"]
        if call["fn"].endswith("backward"):
            assert all(a["zero_before"] for a in call["args"] if a.get("output"))


def test_shim_raises_the_reference_errors_on_host_tensors():
    """CHECK_FLOAT_INPUT (common.h:10-23): a non-CUDA tensor raises RuntimeError."""
    meta, z = log()
    shim = import_shim()
    call = meta["calls"][0]
    args = [torch.from_numpy(z[a["tensor"]]) if ("tensor" in a and not a["output"])
            else torch.empty(a["shape"]) if "tensor" in a else a["value"] for a in call["args"]]
    with pytest.raises(RuntimeError, match="CUDA"):
        shim.stroke_forward(*args)


def build_args(call, z, dev):
    args = []
    for a in call["args"]:
        if "tensor" not in a:
            args.append(a["value"])
        elif a["output"]:
            shape = a["shape"]
            args.append(torch.zeros(shape, device=dev) if a["zero_before"]
                        else torch.full(shape, float("nan"), device=dev))  # unwritten elements would show
        else:
            args.append(torch.from_numpy(z[a["tensor"]].copy()).to(dev))
    return args


def outputs(call, args):
    return [args[i] for i, a in enumerate(call["args"]) if a.get("output") and a["shape"] and np.prod(a["shape"])]


def recorded(call, z):
    return [torch.from_numpy(z[a["tensor"]]) for a in call["args"]
            if a.get("output") and a["shape"] and np.prod(a["shape"])]


def float64_forward(call, z):
    v = [z[a["tensor"]] if "tensor" in a else a["value"] for a in call["args"]]
    x, r, vd, ps, cp = (torch.from_numpy(np.asarray(t)).double() for t in v[4:9])
    return sf.stroke_forward(x, r, ps, cp, v[9], v[11], v[12], v[13], color_id=v[10], viewdir=vd)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", scenes.EVERY_KIND)
def test_reference_strokes_py_calls_replayed_through_the_shim(cuda, kind):
    meta, z = log()
    shim = import_shim()
    ref = cpu_port.reference_extension()
    group = next(g for g in meta["groups"] if g["kind"] == kind)
    curve = kind in ("quadratic_bezier", "cubic_bezier", "catmull_rom")
    for k in group["calls"]:
        call = meta["calls"][k]
        fn = call["fn"]
        mine = build_args(call, z, cuda)
        sl.set_grad_mode("compat")
        try:
            getattr(shim, fn)(*mine)
            theirs = None
            if ref is not None:
                theirs = build_args(call, z, cuda)
                getattr(ref, fn)(*theirs)
        finally:
            sl.set_grad_mode("exact")
        torch.cuda.synchronize()
        got, port = outputs(call, mine), recorded(call, z)
        if fn == "stroke_forward":
            a64, c64 = float64_forward(call, z)
            assert rel(got[0], a64) < FWD_TOL and rel(got[1], c64) < FWD_TOL
            assert rel(got[0], port[0]) <= (rel(port[0], a64) if curve else 0.0) + FWD_TOL
            if theirs is not None:
                ref_a = outputs(call, theirs)[0]
                assert rel(got[0], ref_a) <= (rel(ref_a, a64) if curve else 0.0) + FWD_TOL
                assert rel(got[1], outputs(call, theirs)[1]) == 0.0
        elif fn == "stroke_backward" and kind == "quadratic_bezier":
            # the shim's compat adjoint of this type is the exact one: float64 autograd
            v = [z[a["tensor"]] if "tensor" in a and not a["output"] else a.get("value") for a in call["args"]]
            t64 = lambda i: torch.from_numpy(np.asarray(v[i])).double()
            x = t64(6).requires_grad_(True)
            ps = t64(10).requires_grad_(True)
            cp = t64(11).requires_grad_(True)
            a, c = sf.stroke_forward(x, t64(7), ps, cp, v[12], v[14], v[15], v[16])
            L = (a * t64(3)).sum() + (c * t64(4)).sum()
            gps, gcp, gx = torch.autograd.grad(L, [ps, cp, x])
            for o, e in zip(got, (gps, gcp, gx)):
                assert rel(o, e) < GRAD_TOL
        else:
            tol = FWD_TOL if fn == "compose_forward" else GRAD_TOL
            for o, p in zip(got, port):
                assert rel(o, p) < tol, (fn, rel(o, p))
            if theirs is not None:
                for o, t in zip(got, outputs(call, theirs)):
                    assert rel(o, t) < tol, (fn, rel(o, t))
