// Signed distance primitives of the stroke field: values and exact adjoints.
//
// Values follow the reference definitions (strokes_sdf.h, cited per function),
// including their 1e-8 regularisers, so outputs agree with the reference op.
// Adjoints are the exact derivatives of these computed functions (what float64
// autograd of the same definitions gives): the quadratic Bezier is differentiated
// in reverse mode through its closed-form closest-parameter solve, the cubic Bezier
// through its polyline projection, so both include the dependence of the closest
// parameter t on the sample and the control points.
#pragma once
#include "n3ds_record.cuh"

namespace n3ds {

constexpr float OCTA_K = 0.57735027f;  // strokes_sdf.h:587,612
constexpr float BEZ_SQRT3 = 1.732050808f;  // strokes_sdf.h:686

__device__ __forceinline__ V3 sub1(V3 a, float s) { return {a.x - s, a.y - s, a.z - s}; }

// Axis chosen by the reference's inside-cube argmax tie-breaking (strokes_sdf.h:283-286).
__device__ __forceinline__ V3 cube_inside_axis(V3 q, V3 sg) {
  return {(q.x >= q.y && q.x >= q.z) ? sg.x : 0.f,
          (q.x < q.y && q.y >= q.z) ? sg.y : 0.f,
          (q.x < q.z && q.y < q.z) ? sg.z : 0.f};
}

// ------------------------------------------------------------------ primitives
// p is the local-frame sample; base parameters are read from the record.

constexpr float PRISM_C = 0.866025f;  // strokes_sdf.h:530

// Capped torus term k (strokes_sdf.h:379-381): the cap test selects the projection on
// the cap direction (sin a, cos a) or the distance to the axis.
__device__ __forceinline__ bool torus_cap(float px, float py, float s, float c) { return px * c - py * s > 0.f; }

// |p|^2 + 1 - 2k of the capped torus (strokes_sdf.h:382) without its cancellation near
// the tube: (px - sin a)^2 + (py - cos a)^2 + pz^2 on the cap (sin^2 + cos^2 = 1), and
// (k - 1)^2 + pz^2 - 1e-8 off it (k^2 = px^2 + py^2 + 1e-8); the same function, evaluated
// to float32 accuracy where the reference's float32 form loses digits.
__device__ __forceinline__ float torus_q(float px, float py, float pz, float s, float c, float* k) {
  if (torus_cap(px, py, s, c)) {
    *k = px * s + py * c;
    const float dx = px - s, dy = py - c;
    return dx * dx + dy * dy + pz * pz;
  }
  *k = sqrtf(px * px + py * py + 1e-8f);
  const float d = *k - 1.f;
  return d * d + pz * pz - 1e-8f;
}

__device__ __forceinline__ float prim_sdf(int base, V3 p, const float* rec) {
  const float bp = rec[R_BP];
  switch (base) {
    case B_SPHERE:  // strokes_sdf.h:245-249
      return sqrtf(dot(p, p) + 1e-8f) - 1.f;
    case B_CUBE: {  // 273-277
      V3 q = sub1(vabs(p), 1.f);
      V3 qp = vmax0(q);
      return sqrtf(dot(qp, qp)) + fminf(max3(q), 0.f);
    }
    case B_ROUND_CUBE: {  // 316-325
      V3 q = sub1(vabs(p), 1.f);
      V3 qp = vmax0(q);
      return sqrtf(dot(qp, qp) + 1e-8f) + fminf(max3(q), 0.f) - bp;
    }
    case B_CAPPED_TORUS: {  // 376-383
      float k;
      const float q = torus_q(fabsf(p.x), p.y, p.z, rec[R_TSIN], rec[R_TCOS], &k);
      return sqrtf(q + 1e-8f) - rec[R_BP2];
    }
    case B_CAPSULE: {  // 434-440
      p.y -= clampf(p.y, -bp, bp);
      return sqrtf(dot(p, p) + 1e-8f) - 1.f;
    }
    case B_LINE: {  // 473-482
      const float rd = rec[R_BP2];
      const float t = clampf((p.y + bp) / (2.0f * bp), 0.f, 1.f);
      const float r = (1.f - rd) + t * ((1.f + rd) - (1.f - rd));
      p.y -= clampf(p.y, -bp, bp);
      return sqrtf(dot(p, p) + 1e-8f) - r;
    }
    case B_TRIPRISM: {  // 527-531
      const V3 q = vabs(p);
      return fmaxf(q.y - bp, fmaxf(q.x * PRISM_C + p.z * 0.5f, -p.z) - 0.5f);
    }
    case B_OCTAHEDRON:  // 584-588
      return (fabsf(p.x) + fabsf(p.y) + fabsf(p.z) - 1.f) * OCTA_K;
    case B_TETRAHEDRON:  // 610-613
      return (fmaxf(fabsf(p.x + p.y) - p.z, fabsf(p.x - p.y) + p.z) - 1.f) * OCTA_K;
    default:
      return __int_as_float(0x7fc00000);
  }
}

// Exact dSDF/dp of prim_sdf; gbp[0], gbp[1] receive dSDF/d(base parameters).
// compat != 0 reproduces the reference's own formulas where they differ: the cube
// exterior 2*max(q,0) (strokes_sdf.h:289) and the capped torus, whose branch follows
// k > 0 and whose distance-branch and angle terms are written differently there
// (strokes_sdf.h:385-422).
__device__ __forceinline__ V3 prim_grad(int base, V3 p, const float* rec, float* gbp, int compat) {
  const float bp = rec[R_BP];
  gbp[0] = 0.f;
  gbp[1] = 0.f;
  switch (base) {
    case B_SPHERE: {
      float inv = rsqrtf(dot(p, p) + 1e-8f);
      return p * inv;
    }
    case B_CUBE: {
      V3 q = sub1(vabs(p), 1.f);
      V3 sg = vsgn(p);
      if (max3(q) <= 0.f) return cube_inside_axis(q, sg);
      V3 qp = vmax0(q);
      if (compat) return sg * (qp * 2.f);
      return sg * (qp * rsqrtf(dot(qp, qp)));
    }
    case B_ROUND_CUBE: {
      V3 q = sub1(vabs(p), 1.f);
      V3 sg = vsgn(p);
      V3 qp = vmax0(q);
      V3 g = sg * (qp * rsqrtf(dot(qp, qp) + 1e-8f));
      if (max3(q) < 0.f) g += cube_inside_axis(q, sg);
      gbp[0] = -1.f;
      return g;
    }
    case B_CAPPED_TORUS: {
      const float px = fabsf(p.x), s = rec[R_TSIN], c = rec[R_TCOS];
      gbp[1] = -1.f;
      float k;
      const float inv = rsqrtf(torus_q(px, p.y, p.z, s, c, &k) + 1e-8f);
      if (compat) {
        if (k > 0.f) {
          gbp[0] = -(px * c + p.y * s);
          return V3{p.x - sgn(p.x) * s, p.y - c, p.z} * inv;
        }
        return V3{2.f * p.x, 2.f * p.y, p.z} * inv;
      }
      float kx, ky, ka;
      if (torus_cap(px, p.y, s, c)) {
        kx = s; ky = c; ka = px * c - p.y * s;
      } else {
        kx = px / k; ky = p.y / k; ka = 0.f;
      }
      gbp[0] = -ka * inv;
      return V3{p.x - sgn(p.x) * kx, p.y - ky, p.z} * inv;
    }
    case B_CAPSULE: {
      float y = p.y;
      p.y -= clampf(y, -bp, bp);
      float inv = rsqrtf(dot(p, p) + 1e-8f);
      gbp[0] = -sgn(y) * p.y * inv;  // p.y == 0 on the straight part
      return p * inv;
    }
    case B_LINE: {  // the reference formulas (strokes_sdf.h:484-508) are exact here
      const float rd = rec[R_BP2];
      const float y = p.y;
      const float t = clampf((y + bp) / (2.0f * bp), 0.f, 1.f);
      p.y -= clampf(y, -bp, bp);
      V3 g = p * rsqrtf(dot(p, p) + 1e-8f);
      if (-bp <= y && y <= bp) {
        g.y = -rd / bp;
        gbp[0] = y * rd / (bp * bp);
      } else {
        gbp[0] = g.y * (y > 0.f ? -1.f : 1.f);
      }
      gbp[1] = 1.f - 2.f * t;
      return g;
    }
    case B_TRIPRISM: {  // strokes_sdf.h:533-569
      const V3 q = vabs(p);
      const float a = q.x * PRISM_C + p.z * 0.5f;
      const bool first = a > -p.z;
      const bool ytop = first ? (q.y - bp > a - 0.5f) : (q.y - bp > -p.z - 0.5f);
      if (ytop) {
        gbp[0] = -1.f;
        return {0.f, sgn(p.y), 0.f};
      }
      return first ? V3{PRISM_C * sgn(p.x), 0.f, 0.5f} : V3{0.f, 0.f, -1.f};
    }
    case B_OCTAHEDRON:
      return vsgn(p) * OCTA_K;
    case B_TETRAHEDRON: {
      float a = p.x + p.y, c = p.x - p.y;
      if (fabsf(a) - p.z > fabsf(c) + p.z) {
        float sa = sgn(a) * OCTA_K;
        return {sa, sa, -OCTA_K};
      }
      float sc = sgn(c) * OCTA_K;
      return {sc, -sc, OCTA_K};
    }
    default:
      return {0.f, 0.f, 0.f};
  }
}

// Radius factor f of a multi-scale transform under inv_scale_radius
// (strokes_forward.cu:74-81): f = |g*s| / |g| with g the SDF gradient direction.
// For the sphere base g is parallel to p, so f = |s*p| / |p|.
__device__ __forceinline__ float s3_factor(int base, V3 p, V3 s, const float* rec) {
  V3 g;
  if (base == B_SPHERE) {
    g = p;
  } else {
    float unused[2];
    g = prim_grad(base, p, rec, unused, 1);  // the reference's own gradient formulas
  }
  V3 gs = g * s;
  return sqrtf(dot(gs, gs)) / sqrtf(dot(g, g));
}

// (dg/dp)^T w for the unnormalised reference gradient g of s3_factor (compat
// prim_grad), for the bases whose gradient direction varies with p; zero where g is
// piecewise constant (cube and round-cube interiors, octahedron, tetrahedron, prism).
// *gb0 receives w . dg/d(first base parameter) (the capsule half-length).
// The capped torus and the line, which the reference never combines with a per-axis
// scale, are treated as constant here.
__device__ __forceinline__ V3 s3_dir_adjoint(int base, V3 p, const float* rec, V3 w, float* gb0) {
  *gb0 = 0.f;
  switch (base) {
    case B_CUBE: {  // g = sgn(p) * 2 max(q, 0)
      const V3 q = sub1(vabs(p), 1.f);
      if (max3(q) <= 0.f) return {0.f, 0.f, 0.f};
      return {q.x > 0.f ? 2.f * w.x : 0.f, q.y > 0.f ? 2.f * w.y : 0.f, q.z > 0.f ? 2.f * w.z : 0.f};
    }
    case B_ROUND_CUBE: {  // g = sgn(p) * qp / n outside
      const V3 q = sub1(vabs(p), 1.f);
      if (max3(q) < 0.f) return {0.f, 0.f, 0.f};
      const V3 qp = vmax0(q), sg = vsgn(p);
      const float inv = rsqrtf(dot(qp, qp) + 1e-8f);
      const V3 u = qp * inv, sw = sg * w;
      const V3 r = (sw - u * dot(u, sw)) * inv;
      return {q.x > 0.f ? sg.x * r.x : 0.f, q.y > 0.f ? sg.y * r.y : 0.f, q.z > 0.f ? sg.z * r.z : 0.f};
    }
    case B_CAPSULE: {  // g = q / n with q = p - (0, clamp(y, -h, h), 0)
      const float h = rec[R_BP];
      const bool out = !(-h <= p.y && p.y <= h);
      V3 q = p;
      q.y -= clampf(p.y, -h, h);
      const float inv = rsqrtf(dot(q, q) + 1e-8f);
      const V3 u = q * inv;
      V3 r = (w - u * dot(u, w)) * inv;
      if (!out) {
        r.y = 0.f;
      } else {
        *gb0 = -sgn(p.y) * r.y;  // q_y = y - sgn(y) h
      }
      return r;
    }
    default:
      return {0.f, 0.f, 0.f};
  }
}

// ---------------------------------------------------------- quadratic Bezier
// strokes_sdf.h:649-715, with per-stroke constants from the record.

struct QuadFwd {
  float t, t_raw, dist;
  V3 d, e;
  float kx, ky, p, q;
  float sr, pt;  // refined depressed-cubic root s = t_raw + kx and the regularised p
  // h < 0 branch
  float z, den, arg, v, m, n, sigma;  // sigma = +1 for the (m+n) candidate, -1 for -(m+n)
  int pos_branch;
};

// Two Newton steps on the regularised depressed cubic s^3 + 3 pt s + q = 0 whose
// exact root the closed form represents (see quad_adjoint). The single-precision
// Cardano / trigonometric evaluation loses up to ~1e-3 in t to cancellation; the
// refinement restores the root to float32 accuracy.
__device__ __forceinline__ float quad_newton(float s, float pt, float q) {
#pragma unroll
  for (int it = 0; it < 2; it++) {
    const float g = (s * s + 3.f * pt) * s + q;
    const float gd = 3.f * (s * s + pt);
    if (fabsf(gd) > 1e-12f) s -= g / gd;
  }
  return s;
}

__device__ __forceinline__ float quad_eval(const float* rec, V3 pos, QuadFwd& s) {
  const float4 qA = rec4(rec)[R_QA / 4], qa = rec4(rec)[R_Qa / 4], qb = rec4(rec)[R_Qb / 4],
               qc = rec4(rec)[R_Qc / 4];
  V3 A = xyz(qA), a = xyz(qa), b = xyz(qb), c = xyz(qc);
  float kk = qA.w, kx = qa.w;
  V3 d = A - pos;
  float ky = kk * (qb.w + dot(d, b)) / 3.0f;
  float kz = kk * dot(d, a);
  float p = ky - kx * kx;
  float p3 = p * p * p;
  float q = kx * (2.0f * kx * kx - 3.0f * ky) + kz;
  float h = q * q + 4.0f * p3;
  s.d = d; s.kx = kx; s.ky = ky; s.p = p; s.q = q;
  const float pt = cbrtf(p3 + 2.5e-9f);
  s.pt = pt;
  float t, t_raw;
  if (h >= 0.0f) {
    s.pos_branch = 1;
    float H = sqrtf(h + 1e-8f);
    float x0 = (H - q) * 0.5f, x1 = -(H + q) * 0.5f;
    float u0 = copysignf(cbrtf(fabsf(x0)), x0), u1 = copysignf(cbrtf(fabsf(x1)), x1);
    const float sr = quad_newton(u0 + u1, pt, q);
    s.sr = sr;
    t_raw = sr - kx;
    t = clampf(t_raw, 0.f, 1.f);
  } else {
    s.pos_branch = 0;
    float z = sqrtf(-p + 1e-8f);
    float den = p * z * 2.0f + 1e-8f;
    float arg = q / den;
    float v = acosf(arg) / 3.0f;
    float sv, cv;
    sincosf(v, &sv, &cv);
    float m = cv, n = sv * BEZ_SQRT3;
    // (m + n) z is the reference's first candidate (not a root, kept as computed);
    // (-n - m) z is a true root and is refined
    const float sb = quad_newton((-n - m) * z, pt, q);
    float ra = (m + n) * z - kx, rb = sb - kx;
    float ta = clampf(ra, 0.f, 1.f), tb = clampf(rb, 0.f, 1.f);
    V3 ea = d + (c + b * ta) * ta, eb = d + (c + b * tb) * tb;
    float da = dot(ea, ea), db = dot(eb, eb);
    bool use_b = db < da;
    t = use_b ? tb : ta;
    t_raw = use_b ? rb : ra;
    s.sr = sb;
    s.z = z; s.den = den; s.arg = arg; s.v = v; s.m = m; s.n = n; s.sigma = use_b ? -1.f : 1.f;
  }
  V3 e = d + (c + b * t) * t;
  float dist = sqrtf(dot(e, e) + 1e-8f);
  s.t = t; s.t_raw = t_raw; s.e = e; s.dist = dist;
  float r1 = rec[R_QR1], r2 = rec[R_QR2];
  return dist - (r1 + t * (r2 - r1));
}

// Reverse mode of quad_eval for upstream w = dL/dSDF.
// Returns dL/dpos; g[0..8] += dL/d(A,B,C), g[9], g[10] += dL/d(r1, r2).
__device__ __forceinline__ V3 quad_adjoint(const float* rec, const QuadFwd& s, float w, float* g) {
  const float4 qA = rec4(rec)[R_QA / 4], qa = rec4(rec)[R_Qa / 4], qb = rec4(rec)[R_Qb / 4],
               qc = rec4(rec)[R_Qc / 4];
  V3 a = xyz(qa), b = xyz(qb), c = xyz(qc);
  float kk = qA.w;
  float r1 = rec[R_QR1], r2 = rec[R_QR2];
  float t = s.t;
  V3 ge = s.e * (w / s.dist);           // dL/de
  V3 gd = ge;                           // e = d + c t + b t^2
  V3 gc = ge * t;
  V3 gb = ge * (t * t);
  float gt = -w * (r2 - r1) + dot(ge, c + b * (2.f * t));
  g[9] += -w * (1.f - t);
  g[10] += -w * t;
  float gtr = (s.t_raw > 0.f && s.t_raw < 1.f) ? gt : 0.f;
  // One-real-root branch: t_raw + kx is a root of a depressed cubic (the stationarity
  // condition of |B(t) - pos|^2 divided by 2 |b|^2), differentiated by the implicit
  // function theorem. That stays well conditioned for a simple root, unlike
  // differentiating the cube roots of the closed form, whose 1/(3 u^2) factors blow up
  // when one Cardano term approaches zero.
  //
  // The three-real-root branch is differentiated through its trigonometric formula
  // instead: the reference's first candidate there is (m + n) z - kx
  // (strokes_sdf.h:687), which is not a root of G (the trigonometric root is 2 m z - kx),
  // so the implicit derivative does not apply when that candidate is the closest.
  //
  // With the reference's regulariser H = sqrt(h + 1e-8), the computed s = u0 + u1 is
  // exactly a root of the depressed cubic s^3 + 3 pt s + q = 0 with
  // pt^3 = p^3 + 2.5e-9 (Cardano: u0^3 + u1^3 = -q, u0 u1 = -pt), so differentiating
  // that cubic gives the exact derivative of the regularised closed form:
  //   ds = -(3 s dpt + dq) / (3 (s^2 + pt)),  dpt/dp = p^2 / pt^2.
  // dpt/dp has no bound where p^3 + 2.5e-9 crosses zero (the cube root's vertical
  // tangent; pt can round to exactly 0 there): it is capped at 1e3 so that one sample
  // in that thin shell cannot turn the stroke's gradient into inf / NaN. Likewise
  // 1 / sqrt(1 - arg^2) of the trigonometric branch is capped at 1e4 (the bound the
  // reference's own regulariser gives, strokes_sdf.h:1093-1095).
  float gkx = 0.f, gky = 0.f, gkz = 0.f;
  if (gtr != 0.f && (s.pos_branch || s.sigma < 0.f)) {
    // a (refined) true root: one-real-root branch, or the trig branch's -(m+n) root
    const float sr = s.sr;
    const float pt = s.pt;
    float den = 3.f * (sr * sr + pt);
    if (fabsf(den) < 1e-30f) den = copysignf(1e-30f, den);
    const float gq = -gtr / den;
    const float dpt = fminf((s.p * s.p) / (pt * pt), 1e3f);
    const float gp = -3.f * sr * dpt * gtr / den;
    gkx = -gtr - 2.f * s.kx * gp + gq * (6.f * s.kx * s.kx - 3.f * s.ky);
    gky = gp - 3.f * s.kx * gq;
    gkz = gq;
  } else if (gtr != 0.f) {
    // t_raw = sigma (m + n) z - kx, m = cos v, n = sqrt3 sin v, v = acos(q / (2 p z + 1e-8)) / 3,
    // z = sqrt(-p + 1e-8); p = ky - kx^2, q = kx (2 kx^2 - 3 ky) + kz
    float gz = gtr * s.sigma * (s.m + s.n);
    const float gm = gtr * s.sigma * s.z;
    const float gn = gm;
    float sv, cv;
    sincosf(s.v, &sv, &cv);
    const float gv = -sv * gm + BEZ_SQRT3 * cv * gn;
    const float garg = -(gv / 3.f) * rsqrtf(fmaxf(1.f - s.arg * s.arg, 1e-8f));
    const float gq = garg / s.den;
    const float gden = -garg * s.arg / s.den;
    float gp = 2.f * s.z * gden;
    gz += 2.f * s.p * gden;
    gp += gz * (-0.5f / s.z);
    gkx = -gtr - 2.f * s.kx * gp + gq * (6.f * s.kx * s.kx - 3.f * s.ky);
    gky = gp - 3.f * s.kx * gq;
    gkz = gq;
  }
  // ky = kk (aa2 + d.b) / 3 ; kz = kk (d.a)
  float db = dot(s.d, b), da = dot(s.d, a);
  float gkk = gky * (qb.w + db) / 3.f + gkz * da;
  float gaa2 = gky * kk / 3.f;
  float gdb = gky * kk / 3.f;
  float gda = gkz * kk;
  gd += b * gdb + a * gda;
  gb += s.d * gdb;
  V3 ga = s.d * gda;
  // stroke constants: kx = kk (a.b), kk = 1/(b.b), aa2 = 2 a.a, c = 2 a
  gkk += gkx * qc.w;
  ga += b * (gkx * kk);
  gb += a * (gkx * kk);
  gb += b * (-2.f * kk * kk * gkk);
  ga += a * (4.f * gaa2);
  ga += gc * 2.f;
  // a = B - A ; b = A - 2B + C ; d = A - pos
  V3 gA = gd - ga + gb, gB = ga - gb * 2.f, gC = gb;
  g[0] += gA.x; g[1] += gA.y; g[2] += gA.z;
  g[3] += gB.x; g[4] += gB.y; g[5] += gB.z;
  g[6] += gC.x; g[7] += gC.y; g[8] += gC.z;
  return -gd;
}

// -------------------------------------------------------------- cubic Bezier
// strokes_sdf.h:1238-1294: the closest parameter is taken from a 10-segment
// polyline (vertices precomputed per stroke), then the distance to the curve point.

__device__ __forceinline__ void cubic_weights(float t, float w[4]) {
  float u = 1.0f - t;
  w[0] = u * u * u;
  w[1] = 3.0f * u * u * t;
  w[2] = 3.0f * u * t * t;
  w[3] = t * t * t;
}

// Curve weights of the four stored vectors at t: Bernstein (cubic Bezier control
// points) or the power basis t^3, t^2, t, 1 (Catmull-Rom coefficients A, B, C, D,
// strokes_sdf.h:1333-1338).
__device__ __forceinline__ void curve_weights(float t, float w[4], bool power) {
  if (power) {
    const float t2 = t * t;
    w[0] = t2 * t;
    w[1] = t2;
    w[2] = t;
    w[3] = 1.f;
  } else {
    cubic_weights(t, w);
  }
}

struct CubicFwd {
  float t, tau, tau_raw, dist;
  int seg;  // winning segment 1..10, 0 when none
  V3 v;     // B(t) - pos
};

__device__ __forceinline__ float cubic_eval(const float* rec, V3 pos, CubicFwd& s, bool power) {
  constexpr float step = 1.0f / CUBIC_SEGMENTS;
  float best = 1e18f, tau_best = 0.f, tau_raw_best = 0.f;
  int seg = 0;
  float vtx[36];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const float4 q = rec4(rec)[R_CV / 4 + k];
    vtx[4 * k] = q.x; vtx[4 * k + 1] = q.y; vtx[4 * k + 2] = q.z; vtx[4 * k + 3] = q.w;
  }
  V3 s0 = v3(vtx[0], vtx[1], vtx[2]);
#pragma unroll
  for (int i = 1; i <= CUBIC_SEGMENTS; i++) {
    V3 s1 = v3(vtx[3 * i], vtx[3 * i + 1], vtx[3 * i + 2]);
    V3 ab = s1 - s0;
    float tr = dot(pos - s0, ab) / dot(ab, ab);
    float tt = clampf(tr, 0.f, 1.f);
    V3 dv = pos - (s0 + ab * tt);
    float d2 = dot(dv, dv);
    if (d2 < best) {
      best = d2;
      tau_best = tt;
      tau_raw_best = tr;
      seg = i;
    }
    s0 = s1;
  }
  // the winning segment's t, as the reference's t_start (1 - tau) + t_end tau with
  // t_start = (seg - 1) step, t_end = seg step (the same float values as in its loop)
  const float t_min = seg ? ((float)(seg - 1) * step) * (1.0f - tau_best) + ((float)seg * step) * tau_best : 0.f;
  float w[4];
  curve_weights(t_min, w, power);
  const float4 cA = rec4(rec)[R_CA / 4], cB = rec4(rec)[R_CB / 4], cC = rec4(rec)[R_CC / 4],
               cD = rec4(rec)[R_CD / 4];
  V3 P = xyz(cA) * w[0] + xyz(cB) * w[1] + xyz(cC) * w[2] + xyz(cD) * w[3];
  V3 v = P - pos;
  float dist = sqrtf(dot(v, v));
  s.t = t_min; s.tau = tau_best; s.tau_raw = tau_raw_best; s.seg = seg; s.v = v; s.dist = dist;
  float r1 = cA.w, r2 = cB.w;
  return dist - (r1 + t_min * (r2 - r1));
}

// Reverse mode of cubic_eval. compat != 0 reproduces the reference gradient
// (strokes_sdf.h:1296-1322): -w*2v for position, 2w v * weights for control points,
// no dependence of t on the inputs. Returns dL/dpos (before the reference's second
// multiplication by dL/dSDF, which the caller applies in compat mode).
// g[0..11] += dL/d(A,B,C,D); g[12], g[13] += dL/d(r1, r2). power: the stored
// vectors are Catmull-Rom power-basis coefficients (same adjoint, other weights).
__device__ __forceinline__ V3 cubic_adjoint(const float* rec, V3 pos, const CubicFwd& s, float w,
                                            float* g, int compat, bool power) {
  constexpr float step = 1.0f / CUBIC_SEGMENTS;
  const float4 cA = rec4(rec)[R_CA / 4], cB = rec4(rec)[R_CB / 4], cC = rec4(rec)[R_CC / 4],
               cD = rec4(rec)[R_CD / 4];
  float r1 = cA.w, r2 = cB.w;
  float t = s.t;
  float bw[4];
  curve_weights(t, bw, power);
  g[12] += -w * (1.f - t);
  g[13] += -w * t;
  if (compat) {
    V3 gv = s.v * (2.f * w);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      g[3 * k + 0] += gv.x * bw[k];
      g[3 * k + 1] += gv.y * bw[k];
      g[3 * k + 2] += gv.z * bw[k];
    }
    return -gv;
  }
  V3 A = xyz(cA), B = xyz(cB), C = xyz(cC), D = xyz(cD);
  V3 gv = s.v * (w / s.dist);
  float u = 1.f - t;
  V3 dB = power ? A * (3.f * t * t) + B * (2.f * t) + C
                : (B - A) * (3.f * u * u) + (C - B) * (6.f * u * t) + (D - C) * (3.f * t * t);
  float gt = -w * (r2 - r1) + dot(gv, dB);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    g[3 * k + 0] += gv.x * bw[k];
    g[3 * k + 1] += gv.y * bw[k];
    g[3 * k + 2] += gv.z * bw[k];
  }
  V3 gpos = -gv;
  if (s.seg > 0 && s.tau_raw > 0.f && s.tau_raw < 1.f) {
    float t0 = (s.seg - 1) * step, t1 = s.seg * step;
    float gtau = gt * (t1 - t0);
    V3 s0 = ld3(rec + R_CV + 3 * (s.seg - 1)), s1 = ld3(rec + R_CV + 3 * s.seg);
    V3 ab = s1 - s0;
    V3 wv = pos - s0;
    float inv = 1.f / dot(ab, ab);
    gpos += ab * (gtau * inv);
    V3 g0 = (ab * (2.f * s.tau - 1.f) - wv) * (gtau * inv);
    V3 g1 = (wv - ab * (2.f * s.tau)) * (gtau * inv);
    float w0[4], w1[4];
    curve_weights(t0, w0, power);
    curve_weights(t1, w1, power);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      g[3 * k + 0] += g0.x * w0[k] + g1.x * w1[k];
      g[3 * k + 1] += g0.y * w0[k] + g1.y * w1[k];
      g[3 * k + 2] += g0.z * w0[k] + g1.z * w1[k];
    }
  }
  return gpos;
}

}  // namespace n3ds
