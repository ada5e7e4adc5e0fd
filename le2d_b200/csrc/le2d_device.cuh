// Device-side math of le2d's grid-characteristic step, shared by every kernel.
//
// One time step (le2d simple/le_core.c:605-620) is an x-sweep then a y-sweep.  A
// sweep along axis a maps the five fields of each node to four moving Riemann
// invariants (omega, simple/le_core.c:192-218), transports each with the
// second-order superbee-limited upwind scheme (tvd2, :48-69) and maps the change
// back to the fields (inc_x / inc_y, :221-249).
//
// Face form.  tvd2's slope ratio "r_1" at node i is the ratio "r" of node i-1, and
// its flux "f_12" at node i is the flux "f12" of node i-1 (same operands, same
// operations).  So the kernels compute one ratio and one limited flux per face and
// share it between the two nodes that touch the face:
//   right-moving invariant u (w1, w3):  D_i = u_{i+1} - u_i, P_i = D_i + eps,
//       F_i = u_i + psi_i D_i, psi_i = psi(P_{i-1} / P_i), new u_i = u_i - k (F_i - F_{i-1})
//   left-moving invariant u (w2, w4):   Q_i = eps - D_i,
//       G_i = u_i - psi'_i D_{i-1}, psi'_i = psi(Q_i / Q_{i-1}), new u_i = u_i - k (G_i - G_{i+1})
// with psi(r) = (1 - k)/2 * superbee(r).
//
// FP64 computes exactly these expressions in the reference's operation order, each
// operation rounded once as the reference double build rounds it (namespace ex), so its
// results are the reference's bit for bit: which faces see an exact tie P = 0 (D = -eps)
// depends on every rounding of the sweep before, and there the limiter jumps.
//
// FP32: difference form.  The flux differences need only the face differences D:
//   A_i = F_{i-1} - F_i = t_{i-1} - psi_i D_i,        t_i = (psi_i - 1) D_i
//   B_i = G_{i+1} - G_i = c_i - psi'_{i+1} D_i,       c_i = D_i + psi'_i D_{i-1}
// and D itself is formed from differences of the fields (face_differences), so the
// update never subtracts two large invariants: in FP32 this keeps the relative
// accuracy of small increments (e.g. residual velocities next to large static stresses)
// that differencing the invariants loses.  The field update uses the invariant changes
// directly, 0.5*(new u - u) = k/2 A_i (resp. k/2 B_i).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace le2d {

enum Field { VX = 0, VY = 1, SXX = 2, SXY = 3, SYY = 4, NF = 5 };

template <typename T>
struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };

// Constants of one directional sweep (built on the host by make_sweep()).
template <typename T>
struct Sweep {
  T irhoc1, irhoc2;          // omega: w = v -+ s * irhoc
  T kc1, kc2;                // (1 - k)/2 for the P (k1) and S (k2) Courant numbers
  T hk1, hk2;                // k/2
  T hk1rc1, hk1rc3, hk2rc2;  // k1/2 * rhoc1, k1/2 * rhoc3, k2/2 * rhoc2
  T k1, k2;                  // Courant numbers dt*c/h (plain per-node scheme)
  T rhoc1, rhoc2, rhoc3;     // the material's products (plain per-node scheme)
  // (irhoc1, irhoc2), (-irhoc1, -irhoc2), (kc1, kc2), (-kc1, -kc2): the operands of the
  // packed FP32 x-sweep, which works on the invariant pairs (w1, w3) and (w2, w4); as
  // aligned pairs in the kernel parameters a packed instruction takes each as one operand.
  typename Pair<T>::type irp, nirp, kcp, nkcp;
};

template <typename T>
struct StepConsts {
  Sweep<T> x, y;
};

// The y-sweep constants the packed FP32 pipeline multiplies by, each duplicated into an
// (x, y) pair, so a packed instruction can take it as one 8-byte operand from the kernel
// parameters instead of a pair assembled in registers every row.
struct YPairs {
  float2 ir1, nir1, ir2, nir2;  // +-irhoc1, +-irhoc2
  float2 k1, nk1, k2, nk2;      // +-kc1, +-kc2
  float2 hk1, hk2, hk1rc1, hk1rc3, hk2rc2;
};

__host__ __device__ inline YPairs make_ypairs(const Sweep<float>& c) {
  YPairs p;
  p.ir1 = make_float2(c.irhoc1, c.irhoc1);
  p.nir1 = make_float2(-c.irhoc1, -c.irhoc1);
  p.ir2 = make_float2(c.irhoc2, c.irhoc2);
  p.nir2 = make_float2(-c.irhoc2, -c.irhoc2);
  p.k1 = make_float2(c.kc1, c.kc1);
  p.nk1 = make_float2(-c.kc1, -c.kc1);
  p.k2 = make_float2(c.kc2, c.kc2);
  p.nk2 = make_float2(-c.kc2, -c.kc2);
  p.hk1 = make_float2(c.hk1, c.hk1);
  p.hk2 = make_float2(c.hk2, c.hk2);
  p.hk1rc1 = make_float2(c.hk1rc1, c.hk1rc1);
  p.hk1rc3 = make_float2(c.hk1rc3, c.hk1rc3);
  p.hk2rc2 = make_float2(c.hk2rc2, c.hk2rc2);
  return p;
}

template <typename T>
__device__ __forceinline__ T tvd_eps();
template <>
__device__ __forceinline__ float tvd_eps<float>() { return 1e-6f; }  // TVD2_EPS, simple/le_core.c:29
template <>
__device__ __forceinline__ double tvd_eps<double>() { return 1e-6; }

// Slope ratio a / b.  FP32: hardware reciprocal (rcp.approx, <= 1 ulp) times a;
// for b = +-0 it gives +-inf (a != 0) or NaN (a = 0) like the division does, and the
// limiter maps those exactly as the reference (superbee(+-inf) = 2 / 0, superbee(NaN) = 2).
__device__ __forceinline__ float ratio(float a, float b) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
  return a * r;
}
// FP64: Newton-Raphson division.  The hardware reciprocal estimate y0 (relative error
// around 2^-23) is refined by one Newton step y = y0 + y0 (1 - b y0) (error about its
// square, 2^-46), and the quotient q = a y by one correction with its FMA residual,
// r = q + (a - b q) y (Markstein's final step), whose error is of the order of the square
// of y's (2^-92) before the final rounding.  So r is the correctly rounded quotient unless
// a / b lies within about 2^-92 (relative) of a midpoint between two doubles -- on random
// operands about one division in 2^39; tests/test_division_gpu.py compares it with IEEE
// division.  The slope ratios have the form a = D' + eps, b = D + eps (or eps - D), so b is
// +0 exactly at a tie (D = -eps, never -0 under round-to-nearest) and otherwise at least
// 2^-73 in magnitude (the exact difference of two doubles near eps).  For b = 0 the
// division gives +inf (a > 0), -inf (a < 0) or NaN (a = 0), which the limiter maps to 2,
// 0 and 2: the select returns copysign(inf, a), which the limiter maps the same way (a is
// never -0 either).  Outside the supported range: magnitudes of 2^1022 and above (state
// values near overflow) and operands below about 2^-970, where the residual underflows.
// A select, not a branch: a branch per ratio costs more than the division.  The tie test
// reads b's high word with an integer compare (zero for +0 and for nothing else in range),
// which keeps it off the FP64 pipe the step is bound by.
__device__ __forceinline__ double quotient(double a, double b) {
  double y0;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(b));
  const double y = fma(y0, fma(-b, y0, 1.0), y0);
  const double q = a * y;
  return fma(fma(-b, q, a), y, q);
}
__device__ __forceinline__ double ratio(double a, double b) {
  const double inf = __hiloint2double((__double2hiint(a) & (int)0x80000000) | 0x7ff00000, 0);
  return __double2hiint(b) == 0 ? inf : quotient(a, b);
}

__device__ __forceinline__ float max3(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ double max3(double a, double b, double c) { return fmax(a, fmax(b, c)); }

// kc * superbee(r), superbee(r) = max(0, min(1, 2r), min(2, r))  (simple/le_core.c:38);
// the reference's le_min/le_max give superbee(NaN) = max(0, 1, 2) = 2.  FP32:
// max(sat(2r), min(2, r)), the same function with one min/max less -- sat clamps 2r to [0, 1] (so r <= 0 gives 0 from both
// terms) and flushes NaN to 0, while min(2, NaN) = 2, keeping superbee(NaN) = 2.
__device__ __forceinline__ float psi(float r, float kc) {
  return kc * fmaxf(__saturatef(r + r), fminf(2.0f, r));
}
__device__ __forceinline__ float psi_ratio(float a, float b, float kc) { return psi(ratio(a, b), kc); }
// FP64: kc * superbee(a / b), the limited slope ratio, without floating-point compares.
// superbee(r) is one of 0, 2r, 1, r and 2, and which one follows from r's high word h alone,
// because the breakpoints 0.5, 1 and 2 have zero low words (so, for r >= 0, r < 1 <=>
// h < h(1), and so on).  Below 1, t = h + 2^20 (one more in the exponent field: 2r, r being a
// normal number there -- the ratios' operands are at least 2^-73 or 0) capped at h(1) gives 2r
// below 0.5 and 1 from 0.5 on; from 1 on, t = h capped at h(2) gives r below 2 and 2 from 2
// on (with +inf); the low word stays only below the cap; r <= 0 (h <= 0 as a signed word,
// -0 included) gives 0.  Integer operations keep the FP64 pipe, which bounds the step, free.
// At a tie (b = +0) the division's limit, +-inf for a != 0 and NaN for 0 / 0 (superbee 2, 0
// and 2), enters as the high word of a with the exponent bits set: negative for a < 0 (0),
// at least h(2) otherwise (2) -- a is never -0.  The product kc * superbee(r), kc =
// (1 - k) / 2, rounds like the reference's `limiter(r) / 2.0 * (1.0 - c)`: halving is exact.
// The reference returns -0 for r = -0 where this gives +0 (the same number).
// le2d_selftest_limiter compares it with kc times the reference's superbee of IEEE a / b.
__device__ __forceinline__ double psi_ratio(double a, double b, double kc) {
  constexpr int kH1 = 0x3ff00000, kH2 = 0x40000000;  // high words of 1 and 2
  const double r = quotient(a, b);
  const int h = __double2hiint(b) == 0 ? (__double2hiint(a) | 0x7ff00000) : __double2hiint(r);
  const bool below1 = h < kH1, pos = h > 0;
  const int t = below1 ? h + 0x00100000 : h;
  const int cap = below1 ? kH1 : kH2;
  // written as selects: a branch here would diverge within the warp
  const int ho = pos ? min(t, cap) : 0;
  const int lo = pos && t < cap ? __double2loint(r) : 0;
  return kc * __hiloint2double(ho, lo);
}

// Uncontracted FP64 arithmetic: each operation rounds once, as the reference's double
// build computes (x86-64 baseline code, no fused multiply-add).  The compiler never fuses
// these intrinsics.
namespace ex {
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }

// omega_x / omega_y (simple/le_core.c:192-218) in the reference's operation order:
// n00 = sn * irhoc1, n01 = sxy * irhoc2, w = v -+ n.
__device__ __forceinline__ void invariants(double vn, double sn, double vt, double sxy,
                                           const Sweep<double>& c, double (&w)[4]) {
  const double n00 = mul(sn, c.irhoc1), n01 = mul(sxy, c.irhoc2);
  w[0] = sub(vn, n00);
  w[1] = add(vn, n00);
  w[2] = sub(vt, n01);
  w[3] = add(vt, n01);
}

// The tail of tvd2 (simple/le_core.c:66-68) and reconstruct (:251-257) for one invariant
// u: given the flux difference df = f12 - f_12, the change tvd2(...) - u.
__device__ __forceinline__ double change(double u, double k, double df) {
  return sub(sub(u, mul(k, df)), u);
}

// inc_x / inc_y (simple/le_core.c:221-249) from the four invariant changes, operation by
// operation: d = 0.5 * change, vn += d1 + d2, vt += d3 + d4, sn += (d2 - d1) * rhoc1,
// so += (d2 - d1) * rhoc3, sxy += rhoc2 * (d4 - d3).
template <int AXIS>
__device__ __forceinline__ void increment(double& vx, double& vy, double& sxx, double& sxy,
                                          double& syy, double c1, double c2, double c3, double c4,
                                          const Sweep<double>& c) {
  double& vn = AXIS == 0 ? vx : vy;
  double& vt = AXIS == 0 ? vy : vx;
  double& sn = AXIS == 0 ? sxx : syy;
  double& so = AXIS == 0 ? syy : sxx;
  const double d1 = mul(0.5, c1), d2 = mul(0.5, c2), d3 = mul(0.5, c3), d4 = mul(0.5, c4);
  const double p = sub(d2, d1);
  vn = add(vn, add(d1, d2));
  vt = add(vt, add(d3, d4));
  sn = add(sn, mul(p, c.rhoc1));
  so = add(so, mul(p, c.rhoc3));
  sxy = add(sxy, mul(c.rhoc2, sub(d4, d3)));
}
}  // namespace ex

// Differences of the four moving invariants across a face, formed from the differences
// of the fields that enter them (normal velocity vn, normal stress sn, tangential
// velocity vt, shear stress sxy) rather than by differencing the invariants.
template <typename T>
__device__ __forceinline__ void face_differences(T dvn, T dsn, T dvt, T dsxy, const Sweep<T>& c,
                                                 T& d1, T& d2, T& d3, T& d4) {
  d1 = fma(-dsn, c.irhoc1, dvn);
  d2 = fma(dsn, c.irhoc1, dvn);
  d3 = fma(-dsxy, c.irhoc2, dvt);
  d4 = fma(dsxy, c.irhoc2, dvt);
}

// Invariants of one node for a sweep along AXIS (0 = x, 1 = y).
template <int AXIS, typename T>
__device__ __forceinline__ void omega(T vx, T vy, T sxx, T sxy, T syy, const Sweep<T>& c, T& w1,
                                      T& w2, T& w3, T& w4) {
  const T vn = AXIS == 0 ? vx : vy;
  const T vt = AXIS == 0 ? vy : vx;
  const T sn = AXIS == 0 ? sxx : syy;
  const T n00 = sn * c.irhoc1;
  const T n01 = sxy * c.irhoc2;
  w1 = vn - n00;
  w2 = vn + n00;
  w3 = vt - n01;
  w4 = vt + n01;
}

// Field update of one node from the flux differences of its four invariants:
// a1 = F1_{i-1} - F1_i, b2 = G2_{i+1} - G2_i, a3, b4 likewise (inc_x / inc_y).
template <int AXIS, typename T>
__device__ __forceinline__ void apply_increment(T& vx, T& vy, T& sxx, T& sxy, T& syy, T a1, T b2,
                                                T a3, T b4, const Sweep<T>& c) {
  T& vn = AXIS == 0 ? vx : vy;
  T& vt = AXIS == 0 ? vy : vx;
  T& sn = AXIS == 0 ? sxx : syy;
  T& so = AXIS == 0 ? syy : sxx;
  const T p = b2 - a1;
  vn = fma(c.hk1, a1 + b2, vn);
  vt = fma(c.hk2, a3 + b4, vt);
  sn = fma(c.hk1rc1, p, sn);
  so = fma(c.hk1rc3, p, so);
  sxy = fma(c.hk2rc2, b4 - a3, sxy);
}

}  // namespace le2d
