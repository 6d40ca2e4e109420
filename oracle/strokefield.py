"""Torch restatement of the reference strokelib kernels (oracle / CPU port).

TEST INFRASTRUCTURE ONLY: imported by tests, smoke() and the bench's CPU legs, never
by the product package.

Every function is dtype-generic and vectorised over [P samples, S strokes] for one
``sdf_id`` group, following the reference per-(sample, stroke) kernel line by line:

- ``stroke_forward``   <- strokes_forward.cu:17-109 (+ strokes_sdf.h, common.h)
- ``stroke_backward_compat`` <- strokes_backward.cu:17-157 (the reference's own
  hand-written adjoint formulas, including its known divergences)
- ``compose_forward``  <- compositing.cu:10-59
- ``compose_backward_compat`` <- compositing.cu:62-157

Run in float64 and differentiated with torch.autograd, ``stroke_forward`` +
``compose_forward`` is the exact-gradient oracle. Run in float32 it is the labelled
CPU port of the reference op.

Device float semantics are kept where they change results: ``clamp``/``min``/``max``
use fminf/fmaxf NaN handling (``torch.fmin``/``torch.fmax``), and sign tests use the
reference's ``v < 0 ? -1 : 1`` convention.
"""
import math

import torch

# strokes_sdf.h:8-23 / strokes.py:12-25
BASE_SDF = {
    "unit_sphere": 0, "unit_cube": 1, "unit_round_cube": 2, "unit_capped_torus": 3,
    "unit_capsule": 4, "unit_line": 5, "unit_triprism": 6, "unit_octahedron": 7,
    "unit_tetrahedron": 8, "quadratic_bezier": 9, "cubic_bezier": 10, "catmull_rom": 11,
}
# number of leading base parameters per base SDF (strokes.py:40-82)
N_BASE_PARAMS = {0: 0, 1: 0, 2: 1, 3: 2, 4: 1, 5: 2, 6: 1, 7: 0, 8: 0, 9: 11, 10: 14, 11: 14}
# the bases this build implements (the stroke-field hot path's primitive set)
SUPPORTED_BASES = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11)
INV_SQRT3 = 0.57735027  # strokes_sdf.h:587,612
# the linear soft step's upper clamp 0.9999f (strokes_forward.cu:88) as float32 rounds it
ALPHA_MAX = float(torch.tensor(0.9999, dtype=torch.float32))
SQRT3_BEZ = 1.732050808  # strokes_sdf.h:686


def decode_sdf_id(sdf_id):
    """Split a reference sdf_id (strokes.py:95-106) into (base, T, R, S1, S3)."""
    sdf_id = int(sdf_id)
    return (sdf_id >> 4, bool(sdf_id & 1), bool(sdf_id & 2), bool(sdf_id & 4), bool(sdf_id & 8))


def num_shape_params(sdf_id):
    base, t, r, s1, s3 = decode_sdf_id(sdf_id)
    return N_BASE_PARAMS[base] + (1 if s1 else 0) + (3 if (s3 and not s1) else 0) + \
        (3 if r else 0) + (3 if t else 0)


def cu_clamp(x, lo, hi):
    """helper_math clamp = fmaxf(lo, fminf(x, hi)); NaN maps to hi."""
    if not torch.is_tensor(lo):
        lo = torch.tensor(lo, dtype=x.dtype)
    if not torch.is_tensor(hi):
        hi = torch.tensor(hi, dtype=x.dtype)
    return torch.fmax(torch.fmin(x, hi), lo)


def _sgn(v):
    """The reference's ``v < 0 ? -1 : 1`` (never 0)."""
    return torch.where(v < 0, -torch.ones_like(v), torch.ones_like(v))


def split_params(shape_params, sdf_id):
    """Slice a [S, Ps] parameter block into its parts.

    Transform parameters are read backwards from the row end: translation (last 3),
    Euler angles (3 before), scale (1 or 3 before); base parameters lead
    (strokes_sdf.h:164-191).
    """
    base, t, r, s1, s3 = decode_sdf_id(sdf_id)
    off = num_shape_params(sdf_id)
    parts = {"base": shape_params[:, :N_BASE_PARAMS[base]]}
    if t:
        parts["trans"] = shape_params[:, off - 3:off]
        off -= 3
    if r:
        parts["euler"] = shape_params[:, off - 3:off]
        off -= 3
    if s1:
        parts["scale"] = shape_params[:, off - 1:off]
        off -= 1
    elif s3:
        parts["scale"] = shape_params[:, off - 3:off]
        off -= 3
    return parts


def euler_matrix(e):
    """R = Rz(e.z) Ry(e.y) Rx(e.x), entries as strokes_sdf.h:28-39. e [...,3] -> [...,3,3]."""
    sx, sy, sz = torch.sin(e).unbind(-1)
    cx, cy, cz = torch.cos(e).unbind(-1)
    r0 = torch.stack([cy * cz, sx * sy * cz - cx * sz, sx * sz + cx * sy * cz], -1)
    r1 = torch.stack([cy * sz, cx * cz + sx * sy * sz, cx * sy * sz - sx * cz], -1)
    r2 = torch.stack([-sy, sx * cy, cx * cy], -1)
    return torch.stack([r0, r1, r2], -2)


def euler_matrix_grads(e):
    """dR/d(e.x), dR/d(e.y), dR/d(e.z): [...,3,3,3] with the angle index first."""
    sx, sy, sz = torch.sin(e).unbind(-1)
    cx, cy, cz = torch.cos(e).unbind(-1)
    z = torch.zeros_like(sx)

    def m(rows):
        return torch.stack([torch.stack(r, -1) for r in rows], -2)
    dx = m([[z, cx * sy * cz + sx * sz, cx * sz - sx * sy * cz],
            [z, -sx * cz + cx * sy * sz, -sx * sy * sz - cx * cz],
            [z, cx * cy, -sx * cy]])
    dy = m([[-sy * cz, sx * cy * cz, cx * cy * cz],
            [-sy * sz, sx * cy * sz, cx * cy * sz],
            [-cy, -sx * sy, -cx * sy]])
    dz = m([[-cy * sz, -sx * sy * sz - cx * cz, sx * cz - cx * sy * sz],
            [cy * cz, -cx * sz + sx * sy * cz, cx * sy * cz + sx * sz],
            [z, z, z]])
    return torch.stack([dx, dy, dz], -3)


def to_local(x, parts, sdf_id):
    """inverse_transform (strokes_sdf.h:164-191): x [P,3] -> p [P,S,3]."""
    base, t, r, s1, s3 = decode_sdf_id(sdf_id)
    S = parts["base"].shape[0]
    p = x[:, None, :].expand(x.shape[0], S, 3)
    if t:
        p = p - parts["trans"][None]
    if r:
        R = euler_matrix(parts["euler"])  # [S,3,3]
        p = torch.einsum("sji,psj->psi", R, p)  # R^T p
    if s1:
        p = p / parts["scale"][None]
    elif s3:
        p = p / parts["scale"][None]
    return p


# --------------------------------------------------------------------------- SDFs

def _len_sq(v):
    return (v * v).sum(-1)


def sdf_sphere(p, bp):  # strokes_sdf.h:245-249
    return torch.sqrt(_len_sq(p) + 1e-8) - 1.0


def sdf_cube(p, bp):  # strokes_sdf.h:273-277
    q = p.abs() - 1.0
    qp = torch.fmax(q, torch.zeros_like(q))
    return torch.sqrt(_len_sq(qp)) + torch.fmin(torch.fmax(q[..., 0], torch.fmax(q[..., 1], q[..., 2])),
                                                torch.zeros_like(q[..., 0]))


def sdf_round_cube(p, bp):  # strokes_sdf.h:316-325
    q = p.abs() - 1.0
    qp = torch.fmax(q, torch.zeros_like(q))
    n = torch.sqrt(_len_sq(qp) + 1e-8)
    m = torch.fmin(torch.fmax(q[..., 0], torch.fmax(q[..., 1], q[..., 2])), torch.zeros_like(q[..., 0]))
    return n + m - bp[None, :, 0]


def _capsule_shift(p, h):
    y = p[..., 1]
    y2 = y - cu_clamp(y, -h, h)
    return torch.stack([p[..., 0], y2, p[..., 2]], -1)


def sdf_capsule(p, bp):  # strokes_sdf.h:434-440
    h = bp[None, :, 0]
    q = _capsule_shift(p, h)
    return torch.sqrt(_len_sq(q) + 1e-8) - 1.0


def sdf_octahedron(p, bp):  # strokes_sdf.h:584-588
    return (p.abs().sum(-1) - 1.0) * INV_SQRT3


def sdf_tetrahedron(p, bp):  # strokes_sdf.h:610-613
    x, y, z = p.unbind(-1)
    return (torch.fmax((x + y).abs() - z, (x - y).abs() + z) - 1.0) * INV_SQRT3


def sdf_capped_torus(p, bp):  # strokes_sdf.h:376-383
    ang, rb = bp[None, :, 0], bp[None, :, 1]
    px, py, pz = p[..., 0].abs(), p[..., 1], p[..., 2]
    s, c = torch.sin(ang), torch.cos(ang)
    cap = px * c - py * s > 0  # cross((px, py, 0), (s, c, 0)).z > 0
    k = torch.where(cap, px * s + py * c, torch.sqrt(px * px + py * py + 1e-8))
    return torch.sqrt(px * px + py * py + pz * pz + 1.0 - 2.0 * k + 1e-8) - rb


def sdf_line(p, bp):  # strokes_sdf.h:473-482
    h, rd = bp[None, :, 0], bp[None, :, 1]
    y = p[..., 1]
    t = cu_clamp((y + h) / (2.0 * h), 0.0, 1.0)
    r = (1.0 - rd) + t * ((1.0 + rd) - (1.0 - rd))  # helper_math lerp
    q = torch.stack([p[..., 0], y - cu_clamp(y, -h, h), p[..., 2]], -1)
    return torch.sqrt(_len_sq(q) + 1e-8) - r


def sdf_triprism(p, bp):  # strokes_sdf.h:527-531
    h = bp[None, :, 0]
    q = p.abs()
    return torch.fmax(q[..., 1] - h, torch.fmax(q[..., 0] * 0.866025 + p[..., 2] * 0.5, -p[..., 2]) - 0.5)


def _dot(a, b):
    return (a * b).sum(-1)


def quad_bezier_closest(pos, A, B, C):
    """Closed-form closest-parameter solve (strokes_sdf.h:649-701).

    Returns (squared distance res.x before the final sqrt, t).
    pos [P,S,3]; A,B,C [S,3].
    """
    A, B, C = A[None], B[None], C[None]
    a = B - A
    b = A - 2.0 * B + C
    c = a * 2.0
    d = A - pos
    kk = 1.0 / _dot(b, b)
    kx = kk * _dot(a, b)
    ky = kk * (2.0 * _dot(a, a) + _dot(d, b)) / 3.0
    kz = kk * _dot(d, a)
    p = ky - kx * kx
    p3 = p * p * p
    q = kx * (2.0 * kx * kx - 3.0 * ky) + kz
    h = q * q + 4.0 * p3
    pos_branch = h >= 0.0

    def dist2(t):
        e = d + (c + b * t[..., None]) * t[..., None]
        return _dot(e, e)

    # h >= 0 branch (one real root)
    hs = torch.sqrt(torch.where(pos_branch, h, torch.zeros_like(h)) + 1e-8)
    x0 = (hs - q) * 0.5
    x1 = -(hs + q) * 0.5
    # copysignf(powf(fabsf(x), 1/3), x); guard the autograd of |x|^(1/3) at 0
    def cbrt(v):
        av = v.abs()
        safe = torch.where(av > 0, av, torch.ones_like(av))
        return torch.where(av > 0, torch.sign(v) * safe ** (1.0 / 3.0), torch.zeros_like(v))
    t1 = cu_clamp(cbrt(x0) + cbrt(x1) - kx, 0.0, 1.0)
    r1 = dist2(t1)

    # h < 0 branch (three real roots; the middle one is never the closest)
    z = torch.sqrt(torch.where(pos_branch, torch.ones_like(p), -p) + 1e-8)
    arg = q / (p * z * 2.0 + 1e-8)
    arg_safe = torch.where(pos_branch, torch.zeros_like(arg), arg)
    v = torch.acos(arg_safe) / 3.0
    m = torch.cos(v)
    n = torch.sin(v) * SQRT3_BEZ
    ta = cu_clamp((m + n) * z - kx, 0.0, 1.0)
    tb = cu_clamp((-n - m) * z - kx, 0.0, 1.0)
    da = dist2(ta)
    db = dist2(tb)
    use_b = db < da
    r2 = torch.where(use_b, db, da)
    t2 = torch.where(use_b, tb, ta)

    resx = torch.where(pos_branch, r1, r2)
    rest = torch.where(pos_branch, t1, t2)
    return resx, rest


def sdf_quadratic_bezier(p, bp):  # strokes_sdf.h:649-715
    A, B, C = bp[:, 0:3], bp[:, 3:6], bp[:, 6:9]
    r1, r2 = bp[None, :, 9], bp[None, :, 10]
    resx, t = quad_bezier_closest(p, A, B, C)
    return torch.sqrt(resx + 1e-8) - (r1 + t * (r2 - r1))


def _cubic_point(t, A, B, C, D):
    u = 1.0 - t
    return (u * u * u)[..., None] * A + (3.0 * u * u * t)[..., None] * B + \
        (3.0 * u * t * t)[..., None] * C + (t * t * t)[..., None] * D


def cubic_bezier_closest(pos, A, B, C, D, num_segments=10):
    """10-segment polyline argmin (strokes_sdf.h:1241-1278). Returns t_min [P,S]."""
    A, B, C, D = A[None], B[None], C[None], D[None]
    dt = pos.dtype
    step = 1.0 / num_segments
    dist_min = torch.full(pos.shape[:-1], 1e9, dtype=dt)
    t_min = torch.zeros(pos.shape[:-1], dtype=dt)
    t_start = torch.zeros((), dtype=dt)
    seg_start = _cubic_point(t_start.expand(1, A.shape[1]), A, B, C, D)
    for i in range(1, num_segments + 1):
        t_end = torch.tensor(i * step, dtype=dt)
        seg_end = _cubic_point(t_end.expand(1, A.shape[1]), A, B, C, D)
        ab = seg_end - seg_start
        tt = _dot(pos - seg_start, ab) / _dot(ab, ab)
        tt = cu_clamp(tt, 0.0, 1.0)
        P = seg_start + tt[..., None] * ab
        dist = torch.sqrt(_dot(pos - P, pos - P))
        better = dist < dist_min
        dist_min = torch.where(better, dist, dist_min)
        t_min = torch.where(better, t_start * (1.0 - tt) + t_end * tt, t_min)
        t_start = t_end
        seg_start = seg_end
    return t_min


def catmull_rom_coeffs(p0, p1, p2, p3):
    """Power-basis coefficients (A, B, C, D) of the centripetal Catmull-Rom segment
    between p1 and p2 (strokes_sdf.h:1340-1349): tangents m1, m2 from the knot gaps
    t_ij = sqrt(|p_i - p_j| + 1e-8)."""
    t01 = torch.sqrt(torch.sqrt(_dot(p0 - p1, p0 - p1)) + 1e-8)[..., None]
    t12 = torch.sqrt(torch.sqrt(_dot(p1 - p2, p1 - p2)) + 1e-8)[..., None]
    t23 = torch.sqrt(torch.sqrt(_dot(p2 - p3, p2 - p3)) + 1e-8)[..., None]
    m1 = p2 - p1 + t12 * ((p1 - p0) / t01 - (p2 - p0) / (t01 + t12))
    m2 = p2 - p1 + t12 * ((p3 - p2) / t23 - (p3 - p1) / (t12 + t23))
    A = 2.0 * (p1 - p2) + m1 + m2
    B = 3.0 * (p2 - p1) - 2.0 * m1 - m2
    return A, B, m1, p1


def _catmull_point(t, A, B, C, D):  # strokes_sdf.h:1333-1338
    t2 = t * t
    return (t2 * t)[..., None] * A + t2[..., None] * B + t[..., None] * C + D


def _polyline_closest(pos, point_fn, num_segments=10):
    """argmin-t over a num_segments polyline of the curve point_fn(t) [1,S,3]
    (strokes_sdf.h:1255-1270 / 1352-1367). Returns t_min [P,S]."""
    dt = pos.dtype
    S = pos.shape[1]
    step = 1.0 / num_segments
    dist_min = torch.full(pos.shape[:-1], 1e9, dtype=dt)
    t_min = torch.zeros(pos.shape[:-1], dtype=dt)
    t_start = torch.zeros((), dtype=dt)
    seg_start = point_fn(t_start.expand(1, S))
    for i in range(1, num_segments + 1):
        t_end = torch.tensor(i * step, dtype=dt)
        seg_end = point_fn(t_end.expand(1, S))
        ab = seg_end - seg_start
        tt = cu_clamp(_dot(pos - seg_start, ab) / _dot(ab, ab), 0.0, 1.0)
        P = seg_start + tt[..., None] * ab
        dist = torch.sqrt(_dot(pos - P, pos - P))
        better = dist < dist_min
        dist_min = torch.where(better, dist, dist_min)
        t_min = torch.where(better, t_start * (1.0 - tt) + t_end * tt, t_min)
        t_start = t_end
        seg_start = seg_end
    return t_min


def sdf_catmull_rom(p, bp):  # strokes_sdf.h:1340-1385
    A, B, C, D = catmull_rom_coeffs(bp[:, 0:3], bp[:, 3:6], bp[:, 6:9], bp[:, 9:12])
    r1, r2 = bp[None, :, 12], bp[None, :, 13]
    t = _polyline_closest(p, lambda tt: _catmull_point(tt, A[None], B[None], C[None], D[None]))
    P = _catmull_point(t, A[None], B[None], C[None], D[None])
    dist = torch.sqrt(_dot(P - p, P - p))
    return dist - (r1 + t * (r2 - r1))


def sdf_cubic_bezier(p, bp):  # strokes_sdf.h:1241-1294
    A, B, C, D = bp[:, 0:3], bp[:, 3:6], bp[:, 6:9], bp[:, 9:12]
    r1, r2 = bp[None, :, 12], bp[None, :, 13]
    t = cubic_bezier_closest(p, A, B, C, D)
    P = _cubic_point(t, A[None], B[None], C[None], D[None])
    dist = torch.sqrt(_dot(P - p, P - p))
    return dist - (r1 + t * (r2 - r1))


SDF_FN = {0: sdf_sphere, 1: sdf_cube, 2: sdf_round_cube, 3: sdf_capped_torus, 4: sdf_capsule, 5: sdf_line,
          6: sdf_triprism, 7: sdf_octahedron, 8: sdf_tetrahedron, 9: sdf_quadratic_bezier, 10: sdf_cubic_bezier,
          11: sdf_catmull_rom}


# ------------------------------------------------- reference grad_sdf (compat formulas)

def grad_sdf_compat(base, p, bp, grad_sdf_upstream=None):
    """The reference's BaseSDF<...>::grad_sdf formulas (strokes_sdf.h).

    Returns (dSDF/dpos [P,S,3], dL/dbase-params [P,S,nb] or None). Base-parameter
    gradients are already multiplied by the upstream dL/dSDF, as the reference does.
    The quadratic Bezier is not restated here (its reference formulas are not
    reproduced; see ``stroke_backward_compat``).
    """
    one = torch.ones_like(p[..., 0])
    zero = torch.zeros_like(one)
    if base == 0:  # 252-257
        inv = torch.rsqrt(_len_sq(p) + 1e-8)
        return p * inv[..., None], None
    if base == 1:  # 279-301
        q = p.abs() - 1.0
        inside = torch.fmax(q[..., 0], torch.fmax(q[..., 1], q[..., 2])) <= 0
        qx, qy, qz = q.unbind(-1)
        sx, sy, sz = _sgn(p[..., 0]), _sgn(p[..., 1]), _sgn(p[..., 2])
        gi = torch.stack([torch.where((qx >= qy) & (qx >= qz), sx, zero),
                          torch.where((qx < qy) & (qy >= qz), sy, zero),
                          torch.where((qx < qz) & (qy < qz), sz, zero)], -1)
        gl = 2.0 * torch.fmax(q, torch.zeros_like(q))  # the reference's 2*max(q,0)
        gq = torch.where(q > 0, gl, torch.zeros_like(gl))
        go = torch.stack([sx, sy, sz], -1) * gq
        return torch.where(inside[..., None], gi, go), None
    if base == 2:  # 327-359
        q = p.abs() - 1.0
        qp = torch.fmax(q, torch.zeros_like(q))
        n = torch.sqrt(_len_sq(qp) + 1e-8)
        rinv = torch.rsqrt(_len_sq(qp) + 1e-8)
        gpos = torch.where((n > 0)[..., None], qp * rinv[..., None], torch.zeros_like(qp))
        sym = torch.stack([_sgn(p[..., 0]), _sgn(p[..., 1]), _sgn(p[..., 2])], -1)
        gpos = gpos * sym
        qx, qy, qz = q.unbind(-1)
        mn = torch.fmin(torch.fmax(qx, torch.fmax(qy, qz)), zero)
        gm = torch.where(mn < 0, one, zero)
        gmx = gm * torch.where((qx >= qy) & (qx >= qz), one, zero) * sym[..., 0]
        gmy = gm * torch.where((qx < qy) & (qy >= qz), one, zero) * sym[..., 1]
        gmz = gm * torch.where((qx < qz) & (qy < qz), one, zero) * sym[..., 2]
        g = gpos + torch.stack([gmx, gmy, gmz], -1)
        gb = None
        if grad_sdf_upstream is not None:
            gb = (-grad_sdf_upstream)[..., None]
        return g, gb
    if base == 4:  # 443-453
        h = bp[None, :, 0].expand_as(p[..., 1])
        y = p[..., 1]
        q = _capsule_shift(p, h)
        g = q * torch.rsqrt(_len_sq(q) + 1e-8)[..., None]
        inside = (-h <= y) & (y <= h)
        g = torch.stack([g[..., 0], torch.where(inside, zero, g[..., 1]), g[..., 2]], -1)
        gb = None
        if grad_sdf_upstream is not None:
            gb = torch.where(inside, zero, grad_sdf_upstream * g[..., 1] *
                             torch.where(y > 0, -one, one))[..., None]
        return g, gb
    if base == 3:  # 385-422: the branch follows k > 0, not the cap test of the forward
        ang, rb = bp[None, :, 0], bp[None, :, 1]
        x, y, z = p.unbind(-1)
        px = x.abs()
        s, c = torch.sin(ang), torch.cos(ang)
        cap = px * c - y * s > 0
        k = torch.where(cap, px * s + y * c, torch.sqrt(px * px + y * y))
        inv = torch.rsqrt(px * px + y * y + z * z + 1.0 - 2.0 * k + 1e-8)
        kpos = k > 0
        ga = torch.stack([x - _sgn(x) * s, y - c, z], -1) * inv[..., None]
        gb_ = torch.stack([2.0 * x, 2.0 * y, z], -1) * inv[..., None]
        g = torch.where(kpos[..., None], ga, gb_)
        gb = None
        if grad_sdf_upstream is not None:
            up = grad_sdf_upstream
            g0 = torch.where(kpos, -up * (px * c + y * s), zero)
            gb = torch.stack([g0, -up], -1)
        return g, gb
    if base == 5:  # 484-508
        h, rd = bp[None, :, 0], bp[None, :, 1]
        y = p[..., 1]
        t = cu_clamp((y + h) / (2.0 * h), 0.0, 1.0)
        q = torch.stack([p[..., 0], y - cu_clamp(y, -h, h), p[..., 2]], -1)
        gp = q * torch.rsqrt(_len_sq(q) + 1e-8)[..., None]
        inside = (-h <= y) & (y <= h)
        g = torch.stack([gp[..., 0], torch.where(inside, -rd / h * one, gp[..., 1]), gp[..., 2]], -1)
        gb = None
        if grad_sdf_upstream is not None:
            up = grad_sdf_upstream
            g0 = torch.where(inside, y * rd / (h * h), gp[..., 1] * torch.where(y > 0, -one, one))
            gb = torch.stack([up * g0, up * (1.0 - 2.0 * t)], -1)
        return g, gb
    if base == 6:  # 533-569
        h = bp[None, :, 0]
        q = p.abs()
        x, y, z = p.unbind(-1)
        a = q[..., 0] * 0.866025 + z * 0.5
        first = a > -z
        ytop = torch.where(first, q[..., 1] - h > a - 0.5, q[..., 1] - h > -z - 0.5)
        gy = torch.stack([zero, _sgn(y), zero], -1)
        gface = torch.where(first[..., None], torch.stack([0.866025 * _sgn(x), zero, 0.5 * one], -1),
                            torch.stack([zero, zero, -one], -1))
        g = torch.where(ytop[..., None], gy, gface)
        gb = None
        if grad_sdf_upstream is not None:
            gb = torch.where(ytop, -grad_sdf_upstream, zero)[..., None]
        return g, gb
    if base == 7:  # 590-596
        return torch.stack([_sgn(p[..., 0]), _sgn(p[..., 1]), _sgn(p[..., 2])], -1) * INV_SQRT3, None
    if base == 8:  # 615-632
        x, y, z = p.unbind(-1)
        a = x + y
        c = x - y
        first = a.abs() - z > c.abs() + z
        sa = torch.where(a < 0, -one, one) * INV_SQRT3
        sc = torch.where(c < 0, -one, one) * INV_SQRT3
        g = torch.where(first[..., None],
                        torch.stack([sa, sa, -INV_SQRT3 * one], -1),
                        torch.stack([sc, -sc, INV_SQRT3 * one], -1))
        return g, None
    if base == 10:  # 1296-1322 (returns -dL/dSDF*2v, scaled twice later)
        A, B, C, D = bp[:, 0:3], bp[:, 3:6], bp[:, 6:9], bp[:, 9:12]
        t = cubic_bezier_closest(p, A, B, C, D)
        u = 1.0 - t
        P = _cubic_point(t, A[None], B[None], C[None], D[None])
        v = P - p
        gs = grad_sdf_upstream if grad_sdf_upstream is not None else zero
        gv = gs[..., None] * 2.0 * v
        gb = None
        if grad_sdf_upstream is not None:
            gb = torch.cat([gv * (u * u * u)[..., None], gv * (3.0 * u * u * t)[..., None],
                            gv * (3.0 * u * t * t)[..., None], gv * (t * t * t)[..., None],
                            (-gs * u)[..., None], (-gs * t)[..., None]], -1)
        return -gv, gb
    if base == 11:  # 1387-1447: the knot-gap chain is taken element-wise, as written there
        p0, p1, p2, p3 = bp[:, 0:3], bp[:, 3:6], bp[:, 6:9], bp[:, 9:12]
        A, B, C, D = catmull_rom_coeffs(p0, p1, p2, p3)
        t = _polyline_closest(p, lambda tt: _catmull_point(tt, A[None], B[None], C[None], D[None]))
        P = _catmull_point(t, A[None], B[None], C[None], D[None])
        v = P - p
        gs = grad_sdf_upstream if grad_sdf_upstream is not None else zero
        gv = gs[..., None] * 2.0 * v
        gb = None
        if grad_sdf_upstream is not None:
            p0p1, p1p2, p2p3 = p0 - p1, p1 - p2, p2 - p3
            t01 = torch.sqrt(torch.sqrt(_dot(p0p1, p0p1)) + 1e-8)[:, None]
            t12 = torch.sqrt(torch.sqrt(_dot(p1p2, p1p2)) + 1e-8)[:, None]
            t23 = torch.sqrt(torch.sqrt(_dot(p2p3, p2p3)) + 1e-8)[:, None]
            tt = t[..., None]
            gA, gB, gC, gD = gv * tt ** 3, gv * tt * tt, gv * tt, gv
            gm1 = gA - gB * 2.0 + gC
            gm2 = gA - gB
            dm1_dp0 = t12 / (t01 + t12) - t12 / t01
            dm1_dp1 = -1.0 + t12 / t01
            dm1_dp2 = 1.0 - t12 / (t01 + t12)
            dm2_dp1 = -1.0 + t12 / (t12 + t23)
            dm2_dp2 = 1.0 - t12 / t23
            dm2_dp3 = t12 / t23 - t12 / (t12 + t23)
            dm1_dt01 = t12 * ((p2 - p0) / ((t01 + t12) * (t01 + t12)) - (p1 - p0) / (t01 * t01))
            dm1_dt12 = (p1 - p0) / t01 + t12 * (p2 - p0) / ((t01 + t12) * (t01 + t12)) - (p2 - p0) / (t01 + t12)
            dm2_dt12 = (p2 - p1) / t23 + t12 * (p3 - p1) / ((t12 + t23) * (t12 + t23)) - (p3 - p1) / (t12 + t23)
            dm2_dt23 = t12 * ((p2 - p3) / (t23 * t23) + (p3 - p1) / ((t12 + t23) * (t12 + t23)))
            dt01 = p0p1 / (2.0 * torch.pow(_dot(p0p1, p0p1) + 1e-8, 0.75))[:, None]
            dt12 = p1p2 / (2.0 * torch.pow(_dot(p1p2, p1p2) + 1e-8, 0.75))[:, None]
            dt23 = p2p3 / (2.0 * torch.pow(_dot(p2p3, p2p3) + 1e-8, 0.75))[:, None]
            g0 = gm1 * (dm1_dp0 + dm1_dt01 * dt01)
            g1 = gA * 2.0 + gB * -3.0 + gD + gm1 * (dm1_dp1 - dm1_dt01 * dt01 + dm1_dt12 * dt12) + \
                gm2 * (dm2_dp1 + dm2_dt12 * dt12)
            g2 = gA * -2.0 + gB * 3.0 + gm1 * (dm1_dp2 - dm1_dt12 * dt12) + \
                gm2 * (dm2_dp2 - dm2_dt12 * dt12 + dm2_dt23 * dt23)
            g3 = gm2 * (dm2_dp3 - dm2_dt23 * dt23)
            gb = torch.cat([g0, g1, g2, g3, (-gs * (1.0 - t))[..., None], (-gs * t)[..., None]], -1)
        return -gv, gb
    raise NotImplementedError(f"grad_sdf_compat: base {base}")


def _exact_sdf_grads(base, p, bp, upstream):
    """Exact dSDF/dpos [P,S,3] and the upstream-weighted base-parameter gradient
    summed over samples (returned as [1,S,nb] so callers can sum over dim 0)."""
    with torch.enable_grad():
        pp = p.detach().clone().requires_grad_(True)
        bb = bp.detach().clone().requires_grad_(True)
        sdf = SDF_FN[base](pp, bb)
        gp, = torch.autograd.grad(sdf.sum(), pp, retain_graph=True)
        gb, = torch.autograd.grad((sdf * upstream.detach()).sum(), bb)
    return gp, gb[None]


# --------------------------------------------------------------- stroke forward

def _radius_factor(base, p, bp, parts, sdf_id):
    """Radius rescale under inv_scale_radius (strokes_forward.cu:69-82).

    Returns the divisor f with radius' = radius / f."""
    _, _, _, s1, s3 = decode_sdf_id(sdf_id)
    if s1:
        return parts["scale"][None, :, 0]
    if s3:
        g, _ = grad_sdf_compat(base, p, bp)
        gs = g * parts["scale"][None]
        return torch.sqrt(_len_sq(gs)) / torch.sqrt(_len_sq(g))
    return None


def soft_step(sdf, radius_eff, sdf_delta, use_laplace):
    """SDF -> alpha (strokes_forward.cu:85-90, laplace_cdf common.h:48-51).

    sdf_delta is a float or a per-stroke tensor broadcasting over [P, S]; a
    non-positive value selects the hard step ``sdf <= 0``."""
    kappa = 2.0 if use_laplace else 0.5
    d = sdf_delta if torch.is_tensor(sdf_delta) else torch.tensor(float(sdf_delta), dtype=sdf.dtype)
    d = d.to(sdf.dtype)
    pos = d > 0
    d_safe = torch.where(pos, d, torch.ones_like(d))
    scale = kappa / (d_safe * radius_eff)
    s = -sdf * scale
    if use_laplace:
        e = torch.exp(-s.abs())
        soft = torch.where(s <= 0, 0.5 * e, 1.0 - 0.5 * e)
    else:
        soft = cu_clamp(s + 0.5, 0.0, ALPHA_MAX)
    hard = (sdf <= 0).to(sdf.dtype)
    return torch.where(pos, soft, hard)


# ------------------------------------------------------------- colour fields

def sh_weights(degree, d):
    """Real spherical-harmonic basis up to ``degree`` (2: 4 terms, 3: 9 terms) of the
    directions d [..., 3], the polynomial forms of sh.h:9-28 (tiny-cuda-nn's
    convention: Y_1 = -c1 y, c1 z, -c1 x; Y_2 terms with c2 = sqrt(15)/(2 sqrt(pi)))."""
    x, y, z = d.unbind(-1)
    pi = math.pi
    c0 = 1.0 / (2.0 * math.sqrt(pi))
    c1 = math.sqrt(3.0) / (2.0 * math.sqrt(pi))
    w = [torch.full_like(x, c0), -c1 * y, c1 * z, -c1 * x]
    if degree >= 3:
        c2 = math.sqrt(15.0) / (2.0 * math.sqrt(pi))
        c20 = math.sqrt(5.0) / (4.0 * math.sqrt(pi))
        c22 = math.sqrt(15.0) / (4.0 * math.sqrt(pi))
        w += [c2 * x * y, -c2 * y * z, c20 * (3.0 * z * z - 1.0), -c2 * x * z, c22 * (x * x - y * y)]
    return torch.stack(w, -1)


def color_field(color_id, p_local, x, viewdir_per_point, color_params):
    """Colour per (sample, stroke) [P,S,3] (strokes_color.h:34-171): constant rgb;
    gradient rgb between two points of the unit (local) frame; degree-2 / degree-3
    spherical harmonics of the world view direction through a sigmoid."""
    P, S = p_local.shape[0], p_local.shape[1]
    if color_id == 0:
        return color_params[None, :, :3].expand(P, -1, -1)
    if color_id == 1:
        pos0, pos1 = color_params[None, :, 0:3], color_params[None, :, 3:6]
        c0, c1 = color_params[None, :, 6:9], color_params[None, :, 9:12]
        v0 = p_local - pos0
        v1 = pos1 - pos0
        t = torch.sigmoid(_dot(v0, v1) / _dot(v1, v1) * 5.0 - 2.5)[..., None]
        return c0 * (1.0 - t) + c1 * t
    if color_id in (2, 3):
        n = 4 if color_id == 2 else 9
        w = sh_weights(color_id, viewdir_per_point)  # [P, n]
        coef = color_params[:, :3 * n].reshape(S, n, 3)
        return torch.sigmoid(torch.einsum("pn,snc->psc", w, coef))
    raise ValueError(color_id)


def color_param_grads(color_id, p_local, viewdir_per_point, color_params, grad_color):
    """dL/d(colour params) [S, Pc] from dL/dcolour [P,S,3], the reference's formulas
    (strokes_color.h:70-97, 115-131, 153-169): exact in the parameters, no position
    gradient."""
    S = color_params.shape[0]
    if color_id == 0:
        return grad_color.sum(0)
    if color_id == 1:
        pos0, pos1 = color_params[None, :, 0:3], color_params[None, :, 3:6]
        c0, c1 = color_params[None, :, 6:9], color_params[None, :, 9:12]
        v0 = p_local - pos0
        v1 = pos1 - pos0
        d0, d1 = _dot(v0, v1), _dot(v1, v1)
        t = torch.sigmoid(d0 / d1 * 5.0 - 2.5)
        gt = _dot(grad_color, c1 - c0)
        gtr = 5.0 * t * (1.0 - t) * gt
        gd0 = gtr / d1
        gd1 = -gtr * d0 / (d1 * d1)
        gv1 = gd0[..., None] * v0 + (gd1 * 2.0)[..., None] * v1
        gv0 = gd0[..., None] * v1
        return torch.cat([(-gv0 - gv1).sum(0), gv1.sum(0), (grad_color * (1.0 - t)[..., None]).sum(0),
                          (grad_color * t[..., None]).sum(0)], -1)
    n = 4 if color_id == 2 else 9
    w = sh_weights(color_id, viewdir_per_point)
    coef = color_params[:, :3 * n].reshape(S, n, 3)
    rgb = torch.sigmoid(torch.einsum("pn,snc->psc", w, coef))
    grgb = grad_color * rgb * (1.0 - rgb)
    return torch.einsum("psc,pn->snc", grgb, w).reshape(S, 3 * n)


# ---------------------------------------------------------- texture coordinates

def _permute_by_scale(d, sc):
    """permute_multiscale_axis (strokes_sdf.h:212-222): order the axes by the three
    values sc [S,3] (the per-axis scale, read at the base's offset)."""
    sx, sy, sz = (sc[None, :, k] for k in range(3))
    x, y, z = d.unbind(-1)
    c1 = sx > sy
    c2 = sy > sz
    c3 = sx > sz
    c4 = sz > sy
    out_x = torch.where(c1, torch.where(c2, x, torch.where(c3, x, z)), torch.where(c4, z, torch.where(c3, y, y)))
    out_y = torch.where(c1, torch.where(c2, y, torch.where(c3, z, x)), torch.where(c4, y, torch.where(c3, x, z)))
    out_z = torch.where(c1, torch.where(c2, z, torch.where(c3, y, y)), torch.where(c4, x, torch.where(c3, z, x)))
    return torch.stack([out_x, out_y, out_z], -1)


def texcoord(p, shape_params, sdf_id):
    """Surface texture coordinates (u, v) [P,S,2] of the local sample (BaseSDF::texcoord,
    strokes_sdf.h: sphere 259-267, cube / round cube 302-310 / 359-367, capsule 455-467,
    line 510-522; (0, 0) for the others). The per-axis permutation reads three values
    at the offset each base uses there (the round cube's reads its radius and two
    scales)."""
    base, t, r, s1, s3 = decode_sdf_id(sdf_id)
    P, S = p.shape[0], p.shape[1]
    zero = torch.zeros(P, S, dtype=p.dtype)
    pi = 3.14159265358979323846
    if base == 0:
        d = p * torch.rsqrt(_len_sq(p))[..., None]
        if s3:
            d = _permute_by_scale(d, shape_params[:, 0:3])
        u = torch.asin(cu_clamp(d[..., 0], -1.0, 1.0)) / pi + 0.5
        v = torch.atan2(d[..., 2], d[..., 1]) / (2.0 * pi) + 0.5
        return torch.stack([u, v], -1)
    if base in (1, 2):
        uvt = p * 0.5 + 0.5
        if s3:
            uvt = _permute_by_scale(uvt, shape_params[:, 0:3])
        return torch.stack([cu_clamp(uvt[..., 0], 0.0, 1.0), cu_clamp(uvt[..., 1], 0.0, 1.0)], -1)
    if base in (4, 5):
        h = shape_params[None, :, 0]
        y = p[..., 1]
        if base == 4:
            u = cu_clamp((y / (h + 1.0)) * 0.5 + 0.5, 0.0, 1.0)
        else:
            rd = shape_params[None, :, 1]
            u = cu_clamp((y + h + 1.0 - rd) / (2.0 * h + 2.0), 0.0, 1.0)
        px, pz = p[..., 0], p[..., 2]
        if s3:
            sc = shape_params[:, 1:4]
            swap = (sc[None, :, 2] > sc[None, :, 0])
            px, pz = torch.where(swap, p[..., 2], p[..., 0]), torch.where(swap, p[..., 0], p[..., 2])
        v = torch.atan2(pz, px) / (2.0 * pi) + 0.5
        return torch.stack([u, v], -1)
    return torch.stack([zero, zero], -1)


def viewdir_per_point(viewdir, n_points):
    """The view direction of each point: viewdir[p // (P / n_viewdirs)]
    (strokes_forward.cu:47-48, 195-197)."""
    if viewdir is None or viewdir.numel() == 0:
        return None
    spr = n_points // viewdir.shape[0]
    return viewdir.repeat_interleave(spr, dim=0)


def stroke_forward(x, radius, shape_params, color_params, sdf_id, sdf_delta,
                   use_laplace=False, inv_scale_radius=False, return_sdf=False, color_id=0, viewdir=None,
                   return_texcoord=False):
    """alpha [P,S], color [P,S,3] for one sdf_id group and colour type
    (strokes_forward.cu:17-109; ColorField strokes_color.h:34-171)."""
    base = decode_sdf_id(sdf_id)[0]
    if base not in SDF_FN:
        raise NotImplementedError(f"base sdf {base} is outside the implemented set")
    parts = split_params(shape_params, sdf_id)
    bp = parts["base"]
    p = to_local(x, parts, sdf_id)
    sdf = SDF_FN[base](p, bp)
    r = radius[:, None].expand_as(sdf)
    if inv_scale_radius:
        f = _radius_factor(base, p, bp, parts, sdf_id)
        if f is not None:
            r = r / f
    alpha = soft_step(sdf, r, sdf_delta, use_laplace)
    color = color_field(color_id, p, x, viewdir_per_point(viewdir, x.shape[0]), color_params)
    if return_texcoord:
        return alpha, color, sdf, texcoord(p, shape_params, sdf_id)
    if return_sdf:
        return alpha, color, sdf
    return alpha, color


def stroke_forward_mixed(x, radius, shape_params, sdf_ids, color_params, sdf_delta,
                         use_laplace=False, inv_scale_radius=False):
    """Mixed-type scene: evaluate each sdf_id group and scatter back into stroke
    order, as models.py would with one stroke_fn call per group (models.py:681-702).

    shape_params [S, Pmax] padded per stroke; sdf_ids list/tensor [S]."""
    ids = [int(v) for v in (sdf_ids.tolist() if torch.is_tensor(sdf_ids) else sdf_ids)]
    S = len(ids)
    P = x.shape[0]
    alpha = torch.zeros(P, S, dtype=x.dtype)
    cols = []
    for sid in sorted(set(ids)):
        idx = [i for i, v in enumerate(ids) if v == sid]
        it = torch.tensor(idx, dtype=torch.long)
        ps = shape_params[it][:, :num_shape_params(sid)]
        dl = sdf_delta[it] if torch.is_tensor(sdf_delta) and sdf_delta.dim() > 0 else sdf_delta
        a, _ = stroke_forward(x, radius, ps, color_params[it], sid, dl, use_laplace,
                              inv_scale_radius)
        alpha = alpha.index_copy(1, it, a)
    color = color_params[None, :, :3].expand(P, -1, -1)
    return alpha, color


# ------------------------------------------------------------------- compose

def _over_step(T, dens, col, a, d, c):
    """One stroke of 'over' compositing. The reference skips a zero alpha
    (compositing.cu:37); that changes the sums only where the stroke's colour or
    density is not finite, so only there is the term dropped (elsewhere the skip is
    the identity, and float64 autograd keeps the derivative at alpha = 0)."""
    w = a * T
    T = T * (1.0 - a)
    if torch.is_tensor(d):
        fin = torch.isfinite(c).all(dim=-1) & torch.isfinite(d)
    else:
        fin = torch.isfinite(c).all(dim=-1) & bool(torch.isfinite(torch.tensor(d)))
    keep = (a != 0) | fin
    dens = dens + torch.where(keep, d * w, torch.zeros_like(w))
    col = col + torch.where(keep[:, None], c * w[:, None], torch.zeros_like(c))
    return T, dens, col


def compose_forward(alphas, colors, density_params):
    """'over' compositing, last stroke on top (compositing.cu:10-59)."""
    P, S = alphas.shape
    T = torch.ones(P, dtype=alphas.dtype)
    dens = torch.zeros(P, dtype=alphas.dtype)
    col = torch.zeros(P, colors.shape[-1], dtype=alphas.dtype)
    for s in range(S - 1, -1, -1):
        T, dens, col = _over_step(T, dens, col, alphas[:, s], density_params[s], colors[:, s])
    col = cu_clamp(col * (1.0 / (1.0 + 1e-6 - T))[:, None], 0.0, 1.0)
    return dens, col


def compose_state(alphas, colors, density_params):
    """Raw per-sample composite state: (density, unnormalised colour sum, T_final)."""
    P, S = alphas.shape
    T = torch.ones(P, dtype=alphas.dtype)
    dens = torch.zeros(P, dtype=alphas.dtype)
    col = torch.zeros(P, colors.shape[-1], dtype=alphas.dtype)
    for s in range(S - 1, -1, -1):
        T, dens, col = _over_step(T, dens, col, alphas[:, s], density_params[s], colors[:, s])
    return dens, col, T


def compose_backward_compat(grad_density, grad_color, alphas, colors, density_params):
    """The reference compose adjoint (compositing.cu:62-157), suffix form with the
    clamp mask and 1/max(1-alpha, 1e-6). Returns (grad_alphas, grad_colors,
    grad_density_params)."""
    P, S = alphas.shape
    Cd = colors.shape[-1]
    dens, col, T = compose_state(alphas, colors, density_params)
    final_opacity = 1.0 + 1e-6 - T
    scale = 1.0 / final_opacity
    scaled = col * scale[:, None]
    in_range = (scaled >= 0) & (scaled <= 1)
    gc = torch.where(in_range, grad_color, torch.zeros_like(grad_color))
    gd = grad_density
    T = torch.ones(P, dtype=alphas.dtype)
    d2 = torch.zeros(P, dtype=alphas.dtype)
    c2 = torch.zeros(P, Cd, dtype=alphas.dtype)
    g_alpha = torch.zeros_like(alphas)
    g_colors = torch.zeros_like(colors)
    g_dp = torch.zeros_like(density_params)
    for s in range(S - 1, -1, -1):
        a = alphas[:, s]
        pos = a > 0
        w = torch.where(pos, a * T, torch.zeros_like(a))
        T = torch.where(pos, T * (1.0 - a), T)
        d2 = d2 + density_params[s] * w
        c2 = c2 + colors[:, s] * w[:, None]
        g_dp[s] = (gd * w).sum()
        g_colors[:, s] = gc * (scale * w)[:, None]
        sd = 1.0 / torch.clamp(1.0 - a, min=1e-6)
        ga = gd * (T * density_params[s] - (dens - d2)) * sd
        sd2 = sd * scale * scale
        ga = ga + (gc * (T[:, None] * colors[:, s] * (final_opacity - a)[:, None] - (col - c2))).sum(-1) * sd2
        g_alpha[:, s] = ga
    return g_alpha, g_colors, g_dp


def compose_mode(alphas, colors, density_params, composition_type):
    """The torch compositing modes of compose_strokes (strokes.py:390-417), restated."""
    d = torch.broadcast_to(density_params, alphas.shape)
    if composition_type in ("max", "max_density_weighted"):
        key = alphas if composition_type == "max" else alphas * d
        idx = torch.argmax(key, dim=-1, keepdim=True)
        a = torch.take_along_dim(alphas, idx, dim=-1).squeeze(-1)
        density = a * density_params[idx].squeeze(-1)
        color = torch.take_along_dim(colors, idx[..., None], dim=-2).squeeze(-2)
        return density, color
    if composition_type in ("softmax", "softmax_density_weighted"):
        key = alphas if composition_type == "softmax" else alphas * d
        w = torch.softmax(key * (1.0 / 0.05), dim=-1)
        density = torch.einsum("...s,...s->...", w, alphas * d)
        color = torch.einsum("...s,...sc->...c", w, colors)
        return density, color
    raise ValueError(composition_type)


# ------------------------------------------------------- stroke backward (compat)

def stroke_backward_compat(grad_alpha, grad_color, x, radius, alpha, shape_params,
                           color_params, sdf_id, sdf_delta, use_laplace=False,
                           inv_scale_radius=False, grad_sdf=None, need_grad_x=True, color_id=0, viewdir=None):
    """The reference stroke adjoint (strokes_backward.cu:17-157) for one sdf_id group.

    dAlpha/dSDF is taken from the saved alpha; the soft-step width is treated as a
    constant (no scale or position gradient through it); the reference grad_sdf
    formulas are used. Returns (grad_shape [S,Ps], grad_color [S,3], grad_x [P,3] or
    None)."""
    base, t_on, r_on, s1, s3 = decode_sdf_id(sdf_id)
    parts = split_params(shape_params, sdf_id)
    bp = parts["base"]
    p = to_local(x, parts, sdf_id)
    r = radius[:, None].expand(x.shape[0], shape_params.shape[0])
    if inv_scale_radius:
        f = _radius_factor(base, p, bp, parts, sdf_id)
        if f is not None:
            r = r / f
    kappa = 2.0 if use_laplace else 0.5
    sdf_scale = kappa / (sdf_delta * r)
    if float(sdf_delta) > 0:
        if use_laplace:
            dadsdf = torch.where(alpha < 0.5, alpha, 1.0 - alpha) * -sdf_scale
        else:
            dadsdf = torch.where((alpha > 0) & (alpha < ALPHA_MAX), -sdf_scale, torch.zeros_like(alpha))
    else:
        dadsdf = torch.zeros_like(alpha)
    dl_dsdf = grad_alpha * dadsdf
    if grad_sdf is not None:
        dl_dsdf = dl_dsdf + grad_sdf
    g_color = color_param_grads(color_id, p, viewdir_per_point(viewdir, x.shape[0]), color_params, grad_color)
    if base == 9:
        # The reference quadratic-Bezier adjoint (strokes_sdf.h:709-1172) is not
        # restated: its comma-operator and sign slips make it a different function.
        # Compat mode uses the exact SDF gradient for this primitive.
        dsdf_dpos, gbase = _exact_sdf_grads(base, p, bp, dl_dsdf)
    else:
        dsdf_dpos, gbase = grad_sdf_compat(base, p, bp, dl_dsdf)
    g = dl_dsdf[..., None] * dsdf_dpos  # dL/dpos (local)
    grads = []
    if gbase is not None:
        grads.append(gbase.sum(0))
    elif N_BASE_PARAMS[base] > 0:
        grads.append(torch.zeros(shape_params.shape[0], N_BASE_PARAMS[base], dtype=x.dtype))
    pos = p
    if s1:
        s = parts["scale"][None]
        g = g / s
        grads.append((-(g * pos).sum(-1, keepdim=True)).sum(0))
        pos = pos * s
    elif s3:
        s = parts["scale"][None]
        g = g / s
        grads.append((-(g * pos)).sum(0))
        pos = pos * s
    if r_on:
        e = parts["euler"]
        R = euler_matrix(e)
        pos = torch.einsum("sij,psj->psi", R, pos)  # forward rotation back to x - t
        dR = euler_matrix_grads(e)  # [S,3(angle),3,3]
        # d/da_k of p'_i = sum_j R_ji q_j  ->  sum_ij g_i q_j dR_ji
        grads.append(torch.einsum("psi,psj,skji->sk", g, pos, dR))
        g = torch.einsum("sij,psj->psi", R, g)
    if t_on:
        grads.append((-g).sum(0))
    grad_shape = torch.cat(grads, -1) if grads else torch.zeros_like(shape_params)
    grad_x = g.sum(1) if need_grad_x else None
    return grad_shape, g_color, grad_x


def image_texture(texcoords, colors, alphas, image, tint_ratio=1.0, modulate_alpha=False):
    """ImageTexture.forward (textures.py:58-83): tint = F.grid_sample of image [C,H,W]
    at texcoords [N,2] * 2 - 1 (bilinear, align_corners=True, zero padding);
    colours (colors * tint_ratio + 1 - tint_ratio) * tint; alphas * mean(tint) when
    modulate_alpha. Differentiable in colors and alphas (the texture is a buffer)."""
    import torch.nn.functional as F
    uvs = texcoords.reshape(1, 1, -1, 2) * 2 - 1
    tint = F.grid_sample(image.unsqueeze(0), uvs, align_corners=True)[0, :, 0, :].permute(1, 0)
    colors = (colors * tint_ratio + (1.0 - tint_ratio)) * tint
    if modulate_alpha:
        alphas = alphas * tint.mean(-1)
    return colors, alphas
