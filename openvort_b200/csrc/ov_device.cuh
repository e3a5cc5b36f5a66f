// ov_device.cuh - device-side building blocks shared by the kernels of
// libov_gpu.so: the per-call parameter block, minimum-image wrapping, the
// straight-segment Biot-Savart formula (FP64, exactly as the reference, and
// an FP32 far-field form), and the 16 external flows.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define OV_MAX_IMAGES 32
#define OV_PI 3.14159265358979323846
#define OV_E 2.7182818284590452354

// node status (include/tangle.h:28-33 of the reference)
#define OV_EMPTY (-1)
#define OV_FREE 0
#define OV_PINNED 1
#define OV_PINNED_SLIP 2

// external flow kinds, in the order of the reference's v_confs[] table
// (src/external_velocity.c:85-170)
enum {
  OVF_NONE = 0, OVF_SPHERICAL, OVF_SIMPLE, OVF_SPHERICAL_SIMPLE, OVF_CYLINDRICAL,
  OVF_OSCILLATING, OVF_OSCILLATING_SLIT, OVF_COSCOS, OVF_COSCOS_DIVFREE,
  OVF_COS_DIVFREE, OVF_SIMPLE_SHEAR, OVF_ROTOSC, OVF_DG, OVF_ROTOSC_BOUNDARY,
  OVF_CONST_ACCEL, OVF_PARABOLIC, OVF_COUNT
};

struct OvFlow {
  int kind;
  double s[4];     // scalar parameters, in the order of the flow's parameter list
  double v[2][3];  // vector parameters
};

// Everything a kernel reads from the reference's globals and the tangle's
// box / image table, captured at the start of each call.  Passed by value.
struct OvParams {
  double kappa, core_a, f4pi;   // KAPPA, VORTEX_WIDTH, KAPPA/4/pi
  double lo[3], hi[3], L[3];    // domain box, L = hi - lo
  int periodic[3];              // wall[X_L], wall[Y_L], wall[Z_L] == WALL_PERIODIC
  int n_img;
  int img[OV_MAX_IMAGES][4];    // shift x,y,z, reflect face (-1 none)
  int lia_only, use_bh, quadtree, use_mf, hyperfriction, precision;
  double theta, grain, dl_max;
  double near2;                 // mixed form: squared radius of the FP64 near field
  double alpha, alpha_p, max_curv, hyperalpha;
  // colinearity cut-off of the FP64 direct sums and the adjoint: the
  // reference's 1e-8 (src/tangle.c:505), 0 switches it off
  double col_cut;
  OvFlow vn, vs, vb;
};

// ----------------------------------------------------------------------
// small FP64 vector helpers

struct d3 { double x, y, z; };

__host__ __device__ __forceinline__ d3 mk3(double a, double b, double c) { d3 r; r.x = a; r.y = b; r.z = c; return r; }
__host__ __device__ __forceinline__ d3 operator+(d3 a, d3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ d3 operator-(d3 a, d3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ d3 operator*(d3 a, double s) { return mk3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ d3 cross3(d3 u, d3 v) {
  return mk3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
}
__device__ __forceinline__ d3 ld3(const double* p, int k) { return mk3(p[3 * k], p[3 * k + 1], p[3 * k + 2]); }
__device__ __forceinline__ void st3(double* p, int k, d3 v) { p[3 * k] = v.x; p[3 * k + 1] = v.y; p[3 * k + 2] = v.z; }

// norm as the reference's vec3_d (src/vec3_maths.c:338-345): sequential sum
// of squares without fused multiply-adds, then IEEE sqrt
__device__ __forceinline__ double norm_ref(d3 a) {
  double s = __dmul_rn(a.x, a.x);
  s = __dadd_rn(s, __dmul_rn(a.y, a.y));
  s = __dadd_rn(s, __dmul_rn(a.z, a.z));
  return __dsqrt_rn(s);
}

__device__ __forceinline__ double axis_of(d3 a, int c) { return c == 0 ? a.x : (c == 1 ? a.y : a.z); }
__device__ __forceinline__ void set_axis(d3& a, int c, double v) { if (c == 0) a.x = v; else if (c == 1) a.y = v; else a.z = v; }

// Moves r2 by at most one box length per periodic axis (seg_pwrap,
// src/vec3_maths.c:105-138), exact FP64 operations.
__device__ __forceinline__ d3 pwrap(const OvParams& P, d3 r1, d3 r2) {
  if (P.periodic[0]) {
    double d = __dsub_rn(r2.x, r1.x);
    if (d > P.L[0] * 0.5) r2.x = __dsub_rn(r2.x, P.L[0]);
    else if (d < -P.L[0] * 0.5) r2.x = __dadd_rn(r2.x, P.L[0]);
  }
  if (P.periodic[1]) {
    double d = __dsub_rn(r2.y, r1.y);
    if (d > P.L[1] * 0.5) r2.y = __dsub_rn(r2.y, P.L[1]);
    else if (d < -P.L[1] * 0.5) r2.y = __dadd_rn(r2.y, P.L[1]);
  }
  if (P.periodic[2]) {
    double d = __dsub_rn(r2.z, r1.z);
    if (d > P.L[2] * 0.5) r2.z = __dsub_rn(r2.z, P.L[2]);
    else if (d < -P.L[2] * 0.5) r2.z = __dadd_rn(r2.z, P.L[2]);
  }
  return r2;
}

// image point of r for image j (shifted, src/tangle.c:39-79)
__device__ __forceinline__ d3 image_point(const OvParams& P, int j, d3 r) {
  const int* im = P.img[j];
  d3 rs = mk3(__dsub_rn(r.x, P.L[0] * im[0]), __dsub_rn(r.y, P.L[1] * im[1]),
              __dsub_rn(r.z, P.L[2] * im[2]));
  int face = im[3];
  if (face >= 0) {
    int c = face >> 1;
    double w = (face & 1) ? P.hi[c] : P.lo[c];
    set_axis(rs, c, __dsub_rn(2.0 * w, axis_of(r, c)));
  }
  return rs;
}

// inward face normal (src/vec3_maths.c:55-62)
__device__ __forceinline__ d3 face_normal(int face) {
  double s = (face & 1) ? -1.0 : 1.0;
  int c = face >> 1;
  return mk3(c == 0 ? s : 0.0, c == 1 ? s : 0.0, c == 2 ? s : 0.0);
}

// reflection of a direction in a wall (mirror_dir_reflect, src/vec3_maths.c:260-273)
__device__ __forceinline__ d3 mirror_dir(d3 v, int face) {
  d3 n = face_normal(face);
  double nc = dot3(v, n);
  return v + n * (-2.0 * nc);
}

// ----------------------------------------------------------------------
// straight-segment Biot-Savart (segment_field1, src/tangle.c:486-514)

// FP64, the reference's formula and cut-offs: zero when either endpoint is
// closer than 1e-8 or R, R' are colinear to 1e-8.
__device__ __forceinline__ d3 seg_vel64(double f4pi, d3 r1, d3 r2, d3 r, double col = 1e-8) {
  d3 R = r1 - r, Rp = r2 - r;
  double R2 = dot3(R, R), Rp2 = dot3(Rp, Rp);
  double lR = sqrt(R2), lRp = sqrt(Rp2);
  double RRp = dot3(R, Rp);
  if (lR < 1e-8 || lRp < 1e-8) return mk3(0, 0, 0);
  double p = lR * lRp;
  // colinearity test |R.R'/(|R||R'|) - 1| < 1e-8, evaluated exactly only
  // when the cheap estimate is within a factor 2 of the threshold
  double c = RRp / p;
  double e = fabs(c - 1.0);
  if (e < 2.0 * col) {
    double cref = __ddiv_rn(__ddiv_rn(RRp, lR), lRp);
    if (fabs(cref - 1.0) < col) return mk3(0, 0, 0);
  }
  double s = f4pi * (lR + lRp) / (p * (p + RRp));
  return cross3(R, Rp) * s;
}

// 1/sqrt(x) and 1/x in FP64 from the hardware approximations
// (rsqrt.approx.f64, rcp.approx.ftz.f64, relative error ~2^-22) refined by
// two Newton-Raphson steps each, which square the relative error per step:
//   1/sqrt(x):  y <- y + y (1 - x y^2) / 2
//   1/x:        y <- y + y (1 - x y)
// The results are within a few ulps of the correctly rounded values
// (ov_check_fast_math measures this on the device); positive normal x only.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.f64 %0, %1;" : "=d"(y) : "d"(x));
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double r = fma(-(x * y), y, 1.0);
    y = fma(0.5 * y, r, y);
  }
  return y;
}
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
  }
  return y;
}

// The reference's segment formula without IEEE square roots and divisions:
// with u = 1/(|R||R'|) from two refined reciprocal square roots,
//   f (|R| + |R'|) / (|R||R'| (|R||R'| + R.R')) = f (1/|R| + 1/|R'|) u / (1 + R.R' u).
// R' = R + d (d = r2 - r1, staged per segment) differs from r2 - r by an ulp
// of |R'|.  Where either cut-off could decide (|R| or |R'| within 1.5x of
// 1e-8, or cos within 2e-8 of 1) the reference's own operations decide
// (seg_vel64), so every cut-off decision is the reference's.
__device__ __forceinline__ d3 seg_vel64_nr(double f4pi, d3 r1, d3 r2, d3 d, d3 r, double col = 1e-8) {
  const d3 R = r1 - r;
  const d3 Rp = R + d;
  const double R2 = dot3(R, R), Rp2 = dot3(Rp, Rp), RRp = dot3(R, Rp);
  if (R2 < 2.25e-16 || Rp2 < 2.25e-16) return seg_vel64(f4pi, r1, r2, r, col);
  const double ia = rsqrt_nr(R2), ib = rsqrt_nr(Rp2);
  const double u = ia * ib;
  if (fabs(fma(RRp, u, -1.0)) < 2.0 * col) return seg_vel64(f4pi, r1, r2, r, col);
  const double s = f4pi * (ia + ib) * (u * rcp_nr(fma(RRp, u, 1.0)));
  return cross3(R, Rp) * s;
}

// FP32 far-field form: R and the segment vector ds are formed in FP64 by the
// caller and rounded once; R x R' = R x ds avoids the cancellation of the
// product of two nearly parallel long vectors.  Only used where |R| >= 4|ds|,
// where the reference's distance cut-off cannot trigger.  Its colinearity
// cut-off |cos - 1| < 1e-8 (src/tangle.c:505-506) zeroes far segments that
// point within ~1e-4 rad of the target, so it is applied here too, through
// 1 - cos = |R x ds|^2 / (|R||R'| (|R||R'| + R.R')), which has no
// cancellation.  Returns false when the test is within 2.5e-3 (relative) of
// the threshold: the caller then evaluates the segment in FP64.  That band
// bounds the FP32 error of |R x ds|^2: R and ds rounded once (2^-24 each)
// and the cross product's own rounding give |dC| <= ~5e-7 |R||ds|, while
// at the threshold |C| ~ 1.41e-4 |R|^2, so the relative error of C^2 is at
// most ~7e-3 |ds|/|R| <= 1.8e-3 for |R| >= 4|ds|.
__device__ __forceinline__ bool seg_vel32(float f4pi, float Rx, float Ry, float Rz,
                                          float dx, float dy, float dz,
                                          float& vx, float& vy, float& vz) {
  float Qx = Rx + dx, Qy = Ry + dy, Qz = Rz + dz;
  float R2 = fmaf(Rx, Rx, fmaf(Ry, Ry, Rz * Rz));
  float Q2 = fmaf(Qx, Qx, fmaf(Qy, Qy, Qz * Qz));
  float RQ = fmaf(Rx, Qx, fmaf(Ry, Qy, Rz * Qz));
  float ia = rsqrtf(R2), ib = rsqrtf(Q2);
  float a = R2 * ia, b = Q2 * ib;
  float ab = a * b;
  float cx = Ry * dz - Rz * dy, cy = Rz * dx - Rx * dz, cz = Rx * dy - Ry * dx;
  float C2 = fmaf(cx, cx, fmaf(cy, cy, cz * cz));
  float den = ab * (ab + RQ);
  vx = vy = vz = 0.f;
  if (C2 < (1e-8f * (1.0f - 2.5e-3f)) * den) return true;   // colinear: zero
  if (C2 <= (1e-8f * (1.0f + 2.5e-3f)) * den) return false; // too close to call
  // f (a+b) / (ab (ab + R.R'))
  float s = f4pi * (a + b) * ia * ib * __frcp_rn(ab + RQ);
  vx = cx * s; vy = cy * s; vz = cz * s;
  return true;
}

// ----------------------------------------------------------------------
// external flows (src/external_velocity.c:176-511); parameter slots follow
// each flow's parameter list in the reference's v_confs[] table

__device__ __forceinline__ d3 flow_eval(const OvFlow& f, d3 w, double t) {
  const double* s = f.s;
  d3 r = mk3(0, 0, 0);
  switch (f.kind) {
    case OVF_NONE: break;
    case OVF_SIMPLE: r = mk3(f.v[0][0], f.v[0][1], f.v[0][2]); break;
    case OVF_SPHERICAL:
    case OVF_SPHERICAL_SIMPLE: {
      double rr = norm_ref(w);
      double attn = (s[1] / rr) * (s[1] / rr);
      if (!(rr < 1e-8 || attn > 100)) {
        double fac = exp(-attn);
        r = w * (1.0 / norm_ref(w));
        r = r * (s[0] / (4 * OV_PI * rr * rr) * fac);
      }
      if (f.kind == OVF_SPHERICAL_SIMPLE) r = r + mk3(f.v[0][0], f.v[0][1], f.v[0][2]);
      break;
    }
    case OVF_CYLINDRICAL: {
      double rr = sqrt(w.x * w.x + w.y * w.y);
      double attn = (s[1] / rr) * (s[1] / rr);
      if (!(rr < 1e-8 || attn > 100)) {
        double fac = exp(-attn);
        r = mk3(w.x, w.y, 0);
        r = r * (1.0 / norm_ref(r));
        r = r * (s[0] / (2 * OV_PI * rr) * fac);
      }
      break;
    }
    case OVF_OSCILLATING: {
      double X = cos(2 * OV_PI * (f.v[0][0] * w.x + f.v[0][1] * w.y + f.v[0][2] * w.z));
      double T = sin(2 * OV_PI * s[1] * t);
      r = mk3(f.v[1][0], f.v[1][1], f.v[1][2]) * (s[0] * X * T);
      break;
    }
    case OVF_OSCILLATING_SLIT: {
      double rr = sqrt(w.x * w.x + w.z * w.z);
      d3 dir = mk3(w.x / rr, 0, w.z / rr);
      double attn = exp(-s[2] * s[2] / rr / rr);
      double osc = cos(2 * OV_PI * s[1] * t);
      r = dir * (osc * attn);
      break;
    }
    case OVF_COSCOS:
      r.z = s[1] * (1 + cos(s[0] * w.x) * cos(s[0] * w.y) * exp(-w.z / s[2]));
      break;
    case OVF_COSCOS_DIVFREE: {
      double k = s[0], v0 = s[1], l = s[2];
      r.x = v0 / 2 / l / k * sin(k * w.x) * cos(k * w.y) * exp(-w.z / l);
      r.y = v0 / 2 / l / k * cos(k * w.x) * sin(k * w.y) * exp(-w.z / l);
      r.z = v0 * (1 + cos(k * w.x) * cos(k * w.y) * exp(-w.z / l));
      break;
    }
    case OVF_COS_DIVFREE: {
      double k = s[0], v0 = s[1], l = s[2];
      r.x = v0 / l / k * sin(k * w.x) * exp(-w.z / l);
      r.z = v0 * (1 + cos(k * w.x) * exp(-w.z / l));
      break;
    }
    case OVF_SIMPLE_SHEAR: r.z = s[1] + s[0] * w.x; break;
    case OVF_ROTOSC:
    case OVF_ROTOSC_BOUNDARY:
      r = cross3(mk3(0, 0, 1), w) * (s[1] * cos(2 * OV_PI * s[0] * t));
      break;
    case OVF_DG:
      r = cross3(mk3(0, 0, 1), w) * s[0];
      r.z += s[1];
      break;
    case OVF_CONST_ACCEL: r = mk3(s[0] * t, 0, 0); break;
    case OVF_PARABOLIC: r = mk3(s[1] * w.z * (s[0] - w.z), 0, 0); break;
    default: break;
  }
  return r;
}

#define OV_CUDA_CHECK_LAUNCH() (cudaGetLastError())
