"""Seeded synthetic stroke scenes and rays with the benchmark workloads' shapes.

No dataset is needed: every scene is drawn from a ``torch.Generator`` with a fixed
seed. Stroke parameters use the reference layouts (strokes.py:40-82 via
_make_sdf_id strokes.py:95-106); rotations are uniform random unit quaternions
converted to the reference's ZYX Euler angles (R = Rz Ry Rx, strokes_sdf.h:28-39).

Rays: origins uniform on a sphere of radius 4, aimed at the origin with a random
direction jitter of up to 0.5 rad; fence posts stratified in [2, 6] (interior posts
jittered within +-0.4 of a bin), samples at the interval midpoints (render.py:20-25);
sample radius 1.
"""
import math
from dataclasses import dataclass, field
from typing import List, Optional

import torch

# reference sdf_ids (strokes.py:40-82, 95-106)
SDF_ID = {
    "sphere": 0x05, "ellipsoid": 0x0B, "aacube": 0x15, "cube": 0x17, "aabb": 0x19, "obb": 0x1B,
    "roundcube": 0x27, "roundbox": 0x2B, "cappedtorus": 0x37, "capsule": 0x47, "scapsule": 0x4B, "line": 0x57,
    "triprism": 0x67, "octahedron": 0x77, "tetrahedron": 0x87, "quadratic_bezier": 0x90, "cubic_bezier": 0xA0,
    "catmull_rom": 0xB0,
}
N_PARAMS = {"sphere": 4, "ellipsoid": 9, "aacube": 4, "cube": 7, "aabb": 6, "obb": 9, "roundcube": 8,
            "roundbox": 10, "cappedtorus": 9, "capsule": 8, "scapsule": 10, "line": 9, "triprism": 8,
            "octahedron": 7, "tetrahedron": 7, "quadratic_bezier": 11, "cubic_bezier": 14, "catmull_rom": 14}
PARAM_STRIDE = 16
MIXED_PRIMS = ["sphere", "cube", "roundcube", "tetrahedron", "octahedron", "capsule"]
ALL_KINDS = MIXED_PRIMS + ["quadratic_bezier", "cubic_bezier"]
# every shape type of the reference's get_stroke (strokes.py:40-82)
EVERY_KIND = list(SDF_ID)


@dataclass
class Scene:
    kinds: List[str]
    sdf_ids: torch.Tensor        # int32 [S]
    shape_params: torch.Tensor   # float32 [S, 16], zero padded
    color_params: torch.Tensor   # float32 [S, 3]
    density: torch.Tensor        # float32 [S]

    @property
    def n_strokes(self):
        return int(self.sdf_ids.numel())

    def to(self, device):
        return Scene(self.kinds, self.sdf_ids.to(device), self.shape_params.to(device),
                     self.color_params.to(device), self.density.to(device))


@dataclass
class RaySet:
    origins: torch.Tensor  # [R, 3]
    dirs: torch.Tensor     # [R, 3]
    tdist: torch.Tensor    # [R, N+1]
    x: torch.Tensor        # [R, N, 3]
    radius: torch.Tensor   # [R, N]
    radii: Optional[torch.Tensor] = None  # [R] base radii when radius = radii * t (cast_rays)

    @property
    def n_rays(self):
        return int(self.dirs.shape[0])

    @property
    def n_samples(self):
        return int(self.x.shape[1])

    def to(self, device):
        return RaySet(*(t.to(device) if t is not None else None
                        for t in (self.origins, self.dirs, self.tdist, self.x, self.radius, self.radii)))


def _unit(v):
    return v / v.norm(dim=-1, keepdim=True)


def random_quaternion_euler(n, g):
    """Uniform random rotations (Shoemake) -> Euler (ex, ey, ez) with R = Rz Ry Rx."""
    u1, u2, u3 = torch.rand(3, n, generator=g, dtype=torch.float64)
    qw = torch.sqrt(1 - u1) * torch.sin(2 * math.pi * u2)
    qx = torch.sqrt(1 - u1) * torch.cos(2 * math.pi * u2)
    qy = torch.sqrt(u1) * torch.sin(2 * math.pi * u3)
    qz = torch.sqrt(u1) * torch.cos(2 * math.pi * u3)
    r00 = 1 - 2 * (qy * qy + qz * qz)
    r10 = 2 * (qx * qy + qz * qw)
    r20 = 2 * (qx * qz - qy * qw)
    r21 = 2 * (qy * qz + qx * qw)
    r22 = 1 - 2 * (qx * qx + qy * qy)
    ey = torch.asin(torch.clamp(-r20, -1.0, 1.0))
    ex = torch.atan2(r21, r22)
    ez = torch.atan2(r10, r00)
    return torch.stack([ex, ey, ez], -1).float()


def _logu(n, lo, hi, g):
    return torch.exp(torch.rand(n, generator=g) * (math.log(hi) - math.log(lo)) + math.log(lo))


def make_strokes(kinds, g, density=10.0, ctrl_sigma=0.15):
    """Draw one stroke per entry of ``kinds`` (a list of kind names)."""
    S = len(kinds)
    params = torch.zeros(S, PARAM_STRIDE)
    centre = torch.rand(S, 3, generator=g) * 2 - 1
    euler = random_quaternion_euler(S, g)
    scale1 = _logu(S, 0.05, 0.3, g)
    scale3 = torch.stack([_logu(S, 0.05, 0.3, g) for _ in range(3)], -1)
    rround = torch.rand(S, generator=g) * 0.3
    cap_r = torch.rand(S, generator=g) * 0.08 + 0.02
    cap_half = _logu(S, 0.05, 0.3, g)
    ctrl = centre[:, None, :] + torch.randn(S, 4, 3, generator=g) * ctrl_sigma
    radii = torch.rand(S, 2, generator=g) * 0.05 + 0.01
    if any(k in ("cappedtorus", "line", "triprism") for k in kinds):
        extra = torch.rand(S, 2, generator=g)  # drawn only when needed: earlier scenes keep their streams
    for i, k in enumerate(kinds):
        if k == "sphere":
            row = [scale1[i:i + 1], centre[i]]
        elif k == "ellipsoid":
            row = [scale3[i], euler[i], centre[i]]
        elif k in ("cube", "octahedron", "tetrahedron"):
            row = [scale1[i:i + 1], euler[i], centre[i]]
        elif k == "roundcube":
            row = [rround[i:i + 1], scale1[i:i + 1], euler[i], centre[i]]
        elif k == "capsule":
            h = torch.clamp(cap_half[i] / cap_r[i], min=0.25)
            row = [h.reshape(1), cap_r[i:i + 1], euler[i], centre[i]]
        elif k == "aacube":
            row = [scale1[i:i + 1], centre[i]]
        elif k == "aabb":
            row = [scale3[i], centre[i]]
        elif k == "obb":
            row = [scale3[i], euler[i], centre[i]]
        elif k == "roundbox":
            row = [rround[i:i + 1], scale3[i], euler[i], centre[i]]
        elif k == "scapsule":
            row = [(cap_half[i] / scale3[i, 0]).clamp(min=0.25).reshape(1), scale3[i], euler[i], centre[i]]
        elif k == "cappedtorus":  # cap angle in [0.3, 2.8] rad, tube radius in [0.1, 0.5]
            row = [(0.3 + 2.5 * extra[i, 0]).reshape(1), (0.1 + 0.4 * extra[i, 1]).reshape(1), scale1[i:i + 1],
                   euler[i], centre[i]]
        elif k == "line":  # half-length in [0.25, 1.25], radius change in [-0.5, 0.5]
            row = [(0.25 + extra[i, 0]).reshape(1), (extra[i, 1] - 0.5).reshape(1), scale1[i:i + 1], euler[i],
                   centre[i]]
        elif k == "triprism":  # half-height in [0.2, 1.0]
            row = [(0.2 + 0.8 * extra[i, 0]).reshape(1), scale1[i:i + 1], euler[i], centre[i]]
        elif k == "quadratic_bezier":
            row = [ctrl[i, :3].reshape(-1), radii[i]]
        elif k in ("cubic_bezier", "catmull_rom"):
            row = [ctrl[i].reshape(-1), radii[i]]
        else:
            raise ValueError(k)
        v = torch.cat(row)
        params[i, :v.numel()] = v
    sdf_ids = torch.tensor([SDF_ID[k] for k in kinds], dtype=torch.int32)
    colors = torch.rand(S, 3, generator=g)
    dens = torch.full((S,), float(density))
    return Scene(list(kinds), sdf_ids, params, colors, dens)


def make_rays(n_rays, n_samples, g, near=2.0, far=6.0, jitter=0.5, base_radius=None):
    """Rays through the scene box. With ``base_radius`` (a float) the rays are cones as
    in cast_rays: per-ray base radii uniform in [0.5, 1.5] * base_radius and sample
    radius = radii * t; without it every sample radius is 1."""
    u = _unit(torch.randn(n_rays, 3, generator=g))
    origins = 4.0 * u
    d0 = -u
    w = torch.randn(n_rays, 3, generator=g)
    w = _unit(w - (w * d0).sum(-1, keepdim=True) * d0)
    theta = torch.rand(n_rays, 1, generator=g) * jitter
    dirs = torch.cos(theta) * d0 + torch.sin(theta) * w
    k = torch.arange(n_samples + 1, dtype=torch.float32)
    jit = (torch.rand(n_rays, n_samples + 1, generator=g) - 0.5) * 0.8
    jit[:, 0] = 0
    jit[:, -1] = 0
    tdist = near + (k[None, :] + jit) * ((far - near) / n_samples)
    t = 0.5 * (tdist[:, :-1] + tdist[:, 1:])
    x = origins[:, None, :] + dirs[:, None, :] * t[..., None]
    if base_radius is None:
        return RaySet(origins, dirs, tdist, x, torch.ones(n_rays, n_samples))
    radii = (torch.rand(n_rays, generator=g) + 0.5) * float(base_radius)
    return RaySet(origins, dirs, tdist, x, radii[:, None] * t, radii)


@dataclass
class Workload:
    name: str
    scenes: List[Scene]
    rays: List[RaySet]
    sdf_delta: float = 0.02
    use_laplace: bool = True
    inv_scale_radius: bool = True
    targets: List[torch.Tensor] = field(default_factory=list)

    @property
    def nominal_pairs(self):
        """Nominal (sample, stroke) pairs of one pass: sum over scenes of S * R * N."""
        return sum(s.n_strokes * r.n_rays * r.n_samples for s, r in zip(self.scenes, self.rays))


def config(idx, seed=0, scale=1.0, exclude=()):
    """Workload of benchmark configuration ``idx`` (0..4). ``scale`` < 1 shrinks the
    ray counts (tests); stroke counts and distributions are kept. ``exclude``: stroke
    kinds left out of config 4's draw (a diagnostic variant of that workload)."""
    g = torch.Generator().manual_seed(seed + 1000 * idx)
    gr = torch.Generator().manual_seed(seed + 1000 * idx + 1)  # rays: own stream, so scale keeps the strokes
    R = lambda n: max(32, int(n * scale))
    if idx == 0:
        sc = make_strokes(["ellipsoid"] * 64, g)
        return Workload("cfg0: 64 ellipsoids, 4096 rays x 64 samples, forward", [sc], [make_rays(R(4096), 64, gr)])
    if idx == 1:
        kinds = [MIXED_PRIMS[int(i)] for i in torch.randint(0, 6, (500,), generator=g)]
        sc = make_strokes(kinds, g)
        return Workload("cfg1: 500 mixed primitives, 65536 rays x 128 samples, fwd+bwd", [sc],
                        [make_rays(R(65536), 128, gr)])
    if idx == 2:
        kinds = ["quadratic_bezier"] * 1000 + ["cubic_bezier"] * 1000
        perm = torch.randperm(2000, generator=g)
        kinds = [kinds[int(i)] for i in perm]
        sc = make_strokes(kinds, g)
        return Workload("cfg2: 2000 Bezier tubes, 262144 rays x 64 samples, fwd+bwd", [sc],
                        [make_rays(R(262144), 64, gr)])
    if idx == 3:
        scenes, rays = [], []
        for _ in range(16):
            S = int(round(float(_logu(1, 50, 2000, g))))
            Rn = int(round(float(_logu(1, 4096, 65536, g))))
            kinds = [MIXED_PRIMS[int(i)] for i in torch.randint(0, 6, (S,), generator=g)]
            scenes.append(make_strokes(kinds, g))
            rays.append(make_rays(R(Rn), 64, gr))
        return Workload("cfg3: 16 uneven scenes (S~logU[50,2000], R~logU[4096,65536]) x 64 samples, "
                        "batched fwd+bwd", scenes, rays)
    if idx == 4:
        pool = [k for k in ALL_KINDS if k not in exclude]
        scenes, rays, targets = [], [], []
        for _ in range(4):
            kinds = [pool[int(i)] for i in torch.randint(0, len(pool), (2000,), generator=g)]
            scenes.append(make_strokes(kinds, g))
            rays.append(make_rays(R(131072), 96, gr))
            kt = [pool[int(i)] for i in torch.randint(0, len(pool), (2000,), generator=g)]
            targets.append(make_strokes(kt, g))
        w = Workload("cfg4: 4 scenes x 2000 mixed strokes, 131072 rays x 96 samples, graphed training step",
                     scenes, rays)
        w.target_scenes = targets
        return w
    raise ValueError(idx)


# clamp ranges of each parameter slot (strokes.py:40-82, 245-252), +-inf where unbounded
def param_ranges(kind):
    inf = float("inf")
    scale = (0.01, 0.5)
    rot = (-math.pi, math.pi)
    tr = (-1.0, 1.0)
    if kind in ("sphere", "aacube"):
        r = [scale] + [tr] * 3
    elif kind == "aabb":
        r = [scale] * 3 + [tr] * 3
    elif kind in ("ellipsoid", "obb"):
        r = [scale] * 3 + [rot] * 3 + [tr] * 3
    elif kind in ("cube", "octahedron", "tetrahedron"):
        r = [scale] + [rot] * 3 + [tr] * 3
    elif kind == "roundcube":
        r = [(0.0, 1.0), scale] + [rot] * 3 + [tr] * 3
    elif kind == "roundbox":
        r = [(0.0, 1.0)] + [scale] * 3 + [rot] * 3 + [tr] * 3
    elif kind == "capsule":
        r = [(0.25, inf), scale] + [rot] * 3 + [tr] * 3
    elif kind == "scapsule":
        r = [(0.25, inf)] + [scale] * 3 + [rot] * 3 + [tr] * 3
    elif kind == "cappedtorus":
        r = [(0.0, float(torch.acos(torch.tensor(0.0))) * 2), (0.0, inf), scale] + [rot] * 3 + [tr] * 3
    elif kind == "line":
        r = [(0.25, inf), (-0.8, 0.8), scale] + [rot] * 3 + [tr] * 3
    elif kind == "triprism":
        r = [(0.0, inf), scale] + [rot] * 3 + [tr] * 3
    elif kind == "quadratic_bezier":
        r = [(-1.0, 1.0)] * 9 + [(0.001, 0.2)] * 2
    elif kind in ("cubic_bezier", "catmull_rom"):
        r = [(-1.0, 1.0)] * 12 + [(0.001, 0.2)] * 2
    else:
        raise ValueError(kind)
    lo = [a for a, _ in r] + [-inf] * (PARAM_STRIDE - len(r))
    hi = [b for _, b in r] + [inf] * (PARAM_STRIDE - len(r))
    return lo, hi
