"""Batched, CUDA-graph-captured stroke-field steps.

``BatchedField`` owns static device buffers for a batch of uneven scenes (rays and
strokes concatenated), one workspace, and the ctypes argument blocks, so a forward +
backward over all scenes is a fixed sequence of kernel launches on one stream with
no host synchronisation and no allocation: it is captured once into a CUDA graph and
replayed.

``GraphedTrainer`` adds the training step of the reference loop
(train.py:132-143: forward, data loss, backward, nan_to_num of the gradients, Adam
with betas (0.9, 0.99) and eps 1e-15 from utils/training.py:119-136, parameter clamp
from models.py:576-584) on top, with an MSE loss against a fixed target image, all
inside the same graph.
"""
import ctypes
from typing import List, Optional

import torch

from . import _lib
from .field import FieldOptions
from .scenes import PARAM_STRIDE, SDF_ID, RaySet, Scene, param_ranges


class BatchedField:
    def __init__(self, scenes: List[Scene], rays: List[RaySet], sdf_delta=0.02, use_laplace=True,
                 inv_scale_radius=True, bg=1.0, opaque_background=False, options: Optional[FieldOptions] = None,
                 device="cuda", need_grad_x=True, cast: bool = False):
        """``cast``: keep only the rays (origins, directions, base radii ``RaySet.radii``,
        fence posts) on the device and let the kernels cast the samples
        (x = d t + o, radius = radii t, as cast_rays); no position gradient then."""
        dev = torch.device(device)
        self.device = dev
        self.n_scenes = len(scenes)
        self.n_samples = rays[0].n_samples
        if any(r.n_samples != self.n_samples for r in rays):
            raise ValueError("all scenes must use the same samples per ray")
        self.scene_rays = [r.n_rays for r in rays]
        self.scene_strokes = [s.n_strokes for s in scenes]
        cat = lambda ts: torch.cat(ts).to(dev).contiguous()
        self.cast = bool(cast)
        if self.cast:
            if any(r.radii is None for r in rays):
                raise ValueError("cast mode needs per-ray base radii (RaySet.radii)")
            self.origins = cat([r.origins for r in rays])
            self.radii = cat([r.radii for r in rays])
            self.x = self.radius = None
        else:
            self.origins = self.radii = None
            self.x = cat([r.x for r in rays])
            self.radius = cat([r.radius for r in rays])
        self.tdist = cat([r.tdist for r in rays])
        self.dirs = cat([r.dirs for r in rays])
        self.sdf_ids = cat([s.sdf_ids for s in scenes])
        self.shape = cat([s.shape_params for s in scenes])
        self.color = cat([s.color_params for s in scenes])
        self.density = cat([s.density for s in scenes])
        self.kinds = [k for s in scenes for k in s.kinds]
        S = self.shape.shape[0]
        R = self.tdist.shape[0]
        self.delta = torch.full((S,), float(sdf_delta), device=dev)
        self.rgb = torch.empty(R, 3, device=dev)
        self.acc = torch.empty(R, device=dev)
        self.depth = torch.empty(R, device=dev)
        self.g_rgb = torch.zeros(R, 3, device=dev)
        self.g_acc = torch.zeros(R, device=dev)
        self.g_depth = torch.zeros(R, device=dev)
        self.grad_x = torch.empty_like(self.x) if (need_grad_x and not self.cast) else None
        self.grad_shape = torch.empty_like(self.shape)
        self.grad_color = torch.empty_like(self.color)
        self.grad_density = torch.empty_like(self.density)
        self.grad_delta = torch.empty_like(self.delta)
        self.options = options or FieldOptions()
        self.bg_value = float(bg)
        self.opaque = bool(opaque_background)
        self.laplace = bool(use_laplace)
        self.inv_scale = bool(inv_scale_radius)
        self._bind()

    def _bind(self):
        n = self.n_scenes
        self._nr = (ctypes.c_int64 * n)(*self.scene_rays)
        self._ns = (ctypes.c_int32 * n)(*self.scene_strokes)
        self.c_batch = _lib.Batch(n, self._nr, self._ns, self.n_samples)
        self.c_rays = _lib.Rays(_lib.ptr(self.x), _lib.ptr(self.radius), _lib.ptr(self.tdist), _lib.ptr(self.dirs),
                                None, self.bg_value, int(self.opaque), _lib.ptr(self.origins), _lib.ptr(self.radii))
        # the bases present (from the host's kind list): a field of common primitives
        # only runs the forward build that carries just their code
        base_mask = 0
        for k in set(self.kinds):
            base_mask |= 1 << (SDF_ID[k] >> 4)
        self.c_strokes = _lib.Strokes(_lib.ptr(self.sdf_ids), _lib.ptr(self.shape), PARAM_STRIDE,
                                      _lib.ptr(self.color), _lib.ptr(self.density), _lib.ptr(self.delta),
                                      int(self.laplace), int(self.inv_scale), None, base_mask)
        self.c_opt = self.options.c()
        lib = _lib.load()
        self.ws_bytes = lib.n3ds_field_workspace_bytes(ctypes.byref(self.c_batch), ctypes.byref(self.c_opt))
        if self.ws_bytes == 0:
            raise RuntimeError("invalid batch")
        self.ws = _lib.workspace(self.ws_bytes, self.device)

    @property
    def nominal_pairs(self):
        return sum(s * r for s, r in zip(self.scene_strokes, self.scene_rays)) * self.n_samples

    def forward(self):
        _lib.check(_lib.load().n3ds_field_forward(
            ctypes.byref(self.c_batch), ctypes.byref(self.c_rays), ctypes.byref(self.c_strokes),
            ctypes.byref(self.c_opt), _lib.ptr(self.rgb), _lib.ptr(self.acc), _lib.ptr(self.depth),
            _lib.ptr(self.ws), self.ws_bytes, _lib.stream_ptr(self.device)))

    def backward(self):
        _lib.check(_lib.load().n3ds_field_backward(
            ctypes.byref(self.c_batch), ctypes.byref(self.c_rays), ctypes.byref(self.c_strokes),
            ctypes.byref(self.c_opt), _lib.ptr(self.g_rgb), _lib.ptr(self.g_acc), _lib.ptr(self.g_depth),
            _lib.ptr(self.grad_x), _lib.ptr(self.grad_shape), _lib.ptr(self.grad_color),
            _lib.ptr(self.grad_density), _lib.ptr(self.grad_delta), _lib.ptr(self.ws), self.ws_bytes,
            _lib.stream_ptr(self.device)))

    def step(self):
        self.forward()
        self.backward()

    def launch_count(self):
        """Kernel launches of one forward and one backward (host-side planning)."""
        f, b = ctypes.c_int32(0), ctypes.c_int32(0)
        _lib.check(_lib.load().n3ds_field_launch_count(ctypes.byref(self.c_batch), ctypes.byref(self.c_opt),
                                                       ctypes.byref(f), ctypes.byref(b)))
        return int(f.value), int(b.value)

    def pair_counts(self):
        """Evaluated (sample, stroke) pairs of the last forward, per base SDF type."""
        arr = (ctypes.c_uint64 * 16)()
        _lib.check(_lib.load().n3ds_field_read_pair_counts(_lib.ptr(self.ws), arr, _lib.stream_ptr(self.device)))
        return [int(v) for v in arr]

    def backward_pairs(self):
        """(sample, stroke) pairs the backwards since the last forward evaluated."""
        v = ctypes.c_uint64(0)
        _lib.check(_lib.load().n3ds_field_read_backward_pairs(_lib.ptr(self.ws), ctypes.byref(v),
                                                             _lib.stream_ptr(self.device)))
        return int(v.value)

    def status(self):
        st = ctypes.c_int32(0)
        pairs = ctypes.c_uint64(0)
        _lib.check(_lib.load().n3ds_field_read_status(_lib.ptr(self.ws), ctypes.byref(st), ctypes.byref(pairs),
                                                      _lib.stream_ptr(self.device)))
        return int(st.value), int(pairs.value)


def capture(fn, device="cuda", warmup=2):
    """Warm ``fn`` up on a side stream, then capture it into a CUDA graph."""
    s = torch.cuda.Stream(device)
    s.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(s):
        for _ in range(warmup):
            fn()
    torch.cuda.current_stream(device).wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    return g


class GraphedTrainer:
    """Forward + MSE + adjoint backward + Adam on all stroke parameters, one graph."""

    def __init__(self, field: BatchedField, target_rgb: torch.Tensor, lr=1e-3, betas=(0.9, 0.99), eps=1e-15):
        self.f = field
        dev = field.device
        self.target = target_rgb.to(dev).contiguous()
        self.lr, self.b1, self.b2, self.eps = float(lr), float(betas[0]), float(betas[1]), float(eps)
        self.loss = torch.zeros((), device=dev)
        self.step_count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.m = [torch.zeros_like(t) for t in (field.shape, field.color, field.density)]
        self.v = [torch.zeros_like(t) for t in (field.shape, field.color, field.density)]
        lo, hi = zip(*[param_ranges(k) for k in field.kinds])
        self.lo = [torch.tensor(lo, device=dev), torch.zeros_like(field.color), torch.zeros_like(field.density)]
        self.hi = [torch.tensor(hi, device=dev), torch.ones_like(field.color),
                   torch.full_like(field.density, float("inf"))]
        self.graph = None

    def _adam(self, p, g, m, v, lo, hi):
        _lib.check(_lib.load().n3ds_adam_step(_lib.ptr(p), _lib.ptr(g), _lib.ptr(m), _lib.ptr(v), _lib.ptr(lo),
                                              _lib.ptr(hi), p.numel(), self.lr, self.b1, self.b2, self.eps,
                                              _lib.ptr(self.step_count), _lib.stream_ptr(self.f.device)))

    def _step(self):
        f = self.f
        f.forward()
        diff = f.rgb - self.target
        n = float(diff.numel())
        self.loss.copy_((diff * diff).sum() / n)
        torch.mul(diff, 2.0 / n, out=f.g_rgb)
        f.backward()
        self.step_count.add_(1)
        for p, g, m, v, lo, hi in zip((f.shape, f.color, f.density), (f.grad_shape, f.grad_color, f.grad_density),
                                      self.m, self.v, self.lo, self.hi):
            self._adam(p, g, m, v, lo, hi)

    def capture(self):
        # warm-up steps would move the parameters: snapshot and restore them
        snap = [t.clone() for t in (self.f.shape, self.f.color, self.f.density)] + \
            [t.clone() for t in self.m + self.v] + [self.step_count.clone()]
        self.graph = capture(self._step, self.f.device)
        for dst, src in zip([self.f.shape, self.f.color, self.f.density] + self.m + self.v + [self.step_count], snap):
            dst.copy_(src)
        return self.graph

    def step(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()


class HostPipeline:
    """Run a captured step on batches that live in pinned host memory, overlapping the
    copies with the compute of the neighbouring steps.

    ``inputs`` / ``outputs``: the device tensors the captured step reads / writes
    (for a BatchedField: rays, upstream gradients, parameters / rgb, acc, depth,
    parameter and position gradients). An upload stream copies step i+1's host inputs
    into one of two device staging sets while step i computes; the compute stream
    copies the staged inputs into the step's own buffers (device to device), replays
    the step and copies the results into an output staging set, which a download
    stream copies to the host. Uploads and downloads run on separate streams, so the
    two directions of the host link (separate copy engines) overlap each other as well
    as the compute. Events order every hand-over. Usage::

        pipe.upload(0, host_in)
        for i in range(n):
            if i + 1 < n:
                pipe.upload(i + 1, host_in_next)
            pipe.run(i, host_out)
        pipe.synchronize()
    """

    def __init__(self, graph, inputs, outputs, device):
        self.graph = graph
        self.inputs = list(inputs)
        self.outputs = list(outputs)
        self.device = torch.device(device)
        self.compute = torch.cuda.current_stream(self.device)
        self.copy = torch.cuda.Stream(self.device)   # host -> device
        self.down = torch.cuda.Stream(self.device)   # device -> host
        self.stage_in = [[torch.empty_like(t) for t in self.inputs] for _ in range(2)]
        self.stage_out = [[torch.empty_like(t) for t in self.outputs] for _ in range(2)]
        self.loaded = [torch.cuda.Event() for _ in range(2)]   # upload into input stage k done
        self.taken = [torch.cuda.Event() for _ in range(2)]    # input stage k copied into the step buffers
        self.stored = [torch.cuda.Event() for _ in range(2)]   # results copied into output stage k
        self.fetched = [torch.cuda.Event() for _ in range(2)]  # output stage k downloaded
        self.taken_used = [False, False]
        self.fetched_used = [False, False]

    def upload(self, step, host_inputs):
        """Queue the upload of step ``step``'s inputs (before ``run(step)``, after
        ``run(step - 2)``)."""
        k = step % 2
        if self.taken_used[k]:
            self.copy.wait_event(self.taken[k])
        with torch.cuda.stream(self.copy):
            for d, h in zip(self.stage_in[k], host_inputs):
                d.copy_(h, non_blocking=True)
        self.loaded[k].record(self.copy)

    def run(self, step, host_outputs):
        """Queue step ``step`` on its uploaded inputs and the download of its results."""
        k = step % 2
        c = self.compute
        c.wait_event(self.loaded[k])
        for d, s in zip(self.inputs, self.stage_in[k]):
            d.copy_(s, non_blocking=True)
        self.taken[k].record(c)
        self.taken_used[k] = True
        self.graph.replay()
        if self.fetched_used[k]:
            c.wait_event(self.fetched[k])
        for s, d in zip(self.stage_out[k], self.outputs):
            s.copy_(d, non_blocking=True)
        self.stored[k].record(c)
        self.down.wait_event(self.stored[k])
        with torch.cuda.stream(self.down):
            for h, s in zip(host_outputs, self.stage_out[k]):
                h.copy_(s, non_blocking=True)
        self.fetched[k].record(self.down)
        self.fetched_used[k] = True

    def synchronize(self):
        self.copy.synchronize()
        self.down.synchronize()
        self.compute.synchronize()
