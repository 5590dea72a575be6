// region_rule.cuh -- the per-region degree-9 rule on the device.
//
// Computes, for one box [L, L+H], the five embedded rule sums, the
// fourth-difference split axis and the null-rule error estimate, i.e. what
// the reference does in SampleRegionBlock / computePermutation
// (quad/GPUquad/GPUQuadSample.cu:35-220), re-designed for sm_100a:
//
//  * K lanes (1..32, a power of two, inside one warp) cooperate on a region.
//    K = 1 is thread-per-region: every lane of a warp runs the same point
//    sequence on a different region, so control flow is uniform and no
//    cross-lane reduction is needed.  Small region lists use K = 8 or 32.
//  * Points are enumerated by generator structure, not decoded from a
//    permutation table: axes/axis pairs/triples come from a shared-memory
//    item table, signs are compile-time inner loops, and the coordinates of
//    a point are built with register selects from the region centre.  No
//    divergent __constant__ indexing, no per-point table reads.
//  * f is accumulated into one sum per generator set (the weights are
//    constant within a set); the five rule sums are formed once per region
//    (sum_k w[k][r] * S_k).  The Jacobian is applied once per region.
//  * Rule-sum finishing, null rules and the error heuristic use explicit
//    round-to-nearest intrinsics so they match the CPU oracle bit for bit
//    when the set sums agree.
#pragma once

#include <cstdint>

#include "rule9.hpp"

namespace cubature {
namespace detail {

// Axis combinations of the pair/triple generator sets, in the enumeration
// order the oracle uses (lexicographic; ordered pairs skip d2 == d1).
template <int N>
struct ItemTable {
  static constexpr int kPairs = N * (N - 1) / 2;
  static constexpr int kOPairs = N * (N - 1);
  static constexpr int kTriples = N * (N - 1) * (N - 2) / 6;
  uint32_t pair[kPairs > 0 ? kPairs : 1];
  uint32_t opair[kOPairs > 0 ? kOPairs : 1];
  uint32_t triple[kTriples > 0 ? kTriples : 1];

  // Filled by thread 0 of a block; callers synchronise afterwards.
  __device__ void fill() {
    int p = 0, o = 0, t = 0;
    for (int d1 = 0; d1 < N; ++d1)
      for (int d2 = d1 + 1; d2 < N; ++d2) pair[p++] = d1 | (d2 << 8);
    for (int d1 = 0; d1 < N; ++d1)
      for (int d2 = 0; d2 < N; ++d2)
        if (d2 != d1) opair[o++] = d1 | (d2 << 8);
    for (int d1 = 0; d1 < N; ++d1)
      for (int d2 = d1 + 1; d2 < N; ++d2)
        for (int d3 = d2 + 1; d3 < N; ++d3) triple[t++] = d1 | (d2 << 8) | (d3 << 16);
  }
};

// v[d] for a runtime d, as a select chain (keeps v in registers).
template <int N>
__device__ __forceinline__ double pick(const double (&v)[N], int d) {
  double r = v[0];
#pragma unroll
  for (int i = 1; i < N; ++i) r = (d == i) ? v[i] : r;
  return r;
}

// Per-region sums produced by the point loop (before the K-lane reduction).
struct RegionSums {
  double S[kNumSets];  // sum of f over each generator set
  double best;         // largest fourth difference seen
  int axis;            // its axis (smallest axis on ties)
};

// Coefficient of the box width for a coordinate with generator value +g
// (minus = false) or -g (minus = true): x = L + (0.5 - g) H.
__host__ __device__ __forceinline__ constexpr double coef(double g, bool minus) {
  return minus ? (0.5 + g) : (0.5 - g);
}

// Evaluate the point sums of one region for lane `lane` of K.  L and H are
// the box's lower corner and widths (global coordinates).
template <int N, int K, class F>
__device__ __forceinline__ void region_point_sums(const F& f, const double (&L)[N],
                                                  const double (&H)[N], int lane,
                                                  const ItemTable<N>& tab, double ratio,
                                                  RegionSums& out) {
#pragma unroll
  for (int k = 0; k < kNumSets; ++k) out.S[k] = 0;
  out.best = 0;
  out.axis = -1;

  double C[N];
#pragma unroll
  for (int i = 0; i < N; ++i) C[i] = fma(0.5, H[i], L[i]);

  // Set 0: the centre.  Every lane evaluates it (the fourth difference of
  // each axis needs it); lane 0 adds it.
  const double f0 = f(C);
  if (lane == 0) out.S[0] = f0;
  const double base = __dmul_rn(__dmul_rn(f0, 2.0), __dadd_rn(1.0, -ratio));

  // Sets 1-4: +-g on one axis.  Sets 1 and 2 give the fourth difference.
  for (int d = lane; d < N; d += K) {
    const double Ld = pick(L, d), Hd = pick(H, d);
    double fv[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const double g = (s < 2) ? kGenA1 : (s < 4) ? kGenA2 : (s < 6) ? kGenA3 : kGenA4;
      const double v = fma(coef(g, s & 1), Hd, Ld);
      double x[N];
#pragma unroll
      for (int i = 0; i < N; ++i) x[i] = (i == d) ? v : C[i];
      fv[s] = f(x);
    }
    out.S[1] += fv[0];
    out.S[1] += fv[1];
    out.S[2] += fv[2];
    out.S[2] += fv[3];
    out.S[3] += fv[4];
    out.S[3] += fv[5];
    out.S[4] += fv[6];
    out.S[4] += fv[7];
    // |2(1-r) f0 + r (f1+ + f1-) - (f2+ + f2-)|  (GPUQuadSample.cu:155-162)
    const double fd = fabs(__dadd_rn(__dadd_rn(base, __dmul_rn(ratio, __dadd_rn(fv[0], fv[1]))),
                                     -__dadd_rn(fv[2], fv[3])));
    if (fd > out.best) {
      out.best = fd;
      out.axis = d;
    }
  }

  // Set 5: (+-a1, +-a1) on axis pairs d1 < d2.
  for (int t = lane; t < ItemTable<N>::kPairs; t += K) {
    const uint32_t it = tab.pair[t];
    const int d1 = it & 0xff, d2 = (it >> 8) & 0xff;
    const double L1 = pick(L, d1), H1 = pick(H, d1), L2 = pick(L, d2), H2 = pick(H, d2);
    const double v1p = fma(coef(kGenA1, false), H1, L1), v1m = fma(coef(kGenA1, true), H1, L1);
    const double v2p = fma(coef(kGenA1, false), H2, L2), v2m = fma(coef(kGenA1, true), H2, L2);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const double v1 = (s & 1) ? v1m : v1p, v2 = (s & 2) ? v2m : v2p;
      double x[N];
#pragma unroll
      for (int i = 0; i < N; ++i) x[i] = (i == d1) ? v1 : ((i == d2) ? v2 : C[i]);
      out.S[5] += f(x);
    }
  }

  // Set 6: (+-a1 on d1, +-a2 on d2), ordered pairs d1 != d2.
  for (int t = lane; t < ItemTable<N>::kOPairs; t += K) {
    const uint32_t it = tab.opair[t];
    const int d1 = it & 0xff, d2 = (it >> 8) & 0xff;
    const double L1 = pick(L, d1), H1 = pick(H, d1), L2 = pick(L, d2), H2 = pick(H, d2);
    const double v1p = fma(coef(kGenA1, false), H1, L1), v1m = fma(coef(kGenA1, true), H1, L1);
    const double v2p = fma(coef(kGenA2, false), H2, L2), v2m = fma(coef(kGenA2, true), H2, L2);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const double v1 = (s & 1) ? v1m : v1p, v2 = (s & 2) ? v2m : v2p;
      double x[N];
#pragma unroll
      for (int i = 0; i < N; ++i) x[i] = (i == d1) ? v1 : ((i == d2) ? v2 : C[i]);
      out.S[6] += f(x);
    }
  }

  // Set 7: (+-a1, +-a1, +-a1) on axis triples d1 < d2 < d3.
  for (int t = lane; t < ItemTable<N>::kTriples; t += K) {
    const uint32_t it = tab.triple[t];
    const int d1 = it & 0xff, d2 = (it >> 8) & 0xff, d3 = (it >> 16) & 0xff;
    const double L1 = pick(L, d1), H1 = pick(H, d1);
    const double L2 = pick(L, d2), H2 = pick(H, d2);
    const double L3 = pick(L, d3), H3 = pick(H, d3);
    const double v1p = fma(coef(kGenA1, false), H1, L1), v1m = fma(coef(kGenA1, true), H1, L1);
    const double v2p = fma(coef(kGenA1, false), H2, L2), v2m = fma(coef(kGenA1, true), H2, L2);
    const double v3p = fma(coef(kGenA1, false), H3, L3), v3m = fma(coef(kGenA1, true), H3, L3);
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const double v1 = (s & 1) ? v1m : v1p, v2 = (s & 2) ? v2m : v2p, v3 = (s & 4) ? v3m : v3p;
      double x[N];
#pragma unroll
      for (int i = 0; i < N; ++i)
        x[i] = (i == d1) ? v1 : ((i == d2) ? v2 : ((i == d3) ? v3 : C[i]));
      out.S[7] += f(x);
    }
  }

  // Set 8: (+-l, ..., +-l), all 2^N sign patterns; bit d of the pattern
  // makes coordinate d negative.  The low E bits run as a compile-time
  // inner loop, the high bits are one item.
  constexpr int E = N < 3 ? N : 3;
  constexpr int kItems8 = 1 << (N - E);
  double P[N], M[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    P[i] = fma(coef(kGenL, false), H[i], L[i]);
    M[i] = fma(coef(kGenL, true), H[i], L[i]);
  }
  for (int t = lane; t < kItems8; t += K) {
    double xh[N];
#pragma unroll
    for (int i = E; i < N; ++i) xh[i] = ((t >> (i - E)) & 1) ? M[i] : P[i];
#pragma unroll
    for (int s = 0; s < (1 << E); ++s) {
      double x[N];
#pragma unroll
      for (int i = 0; i < N; ++i) x[i] = (i < E) ? (((s >> i) & 1) ? M[i] : P[i]) : xh[i];
      out.S[8] += f(x);
    }
  }
}

// Combine the sums of the K lanes of a group (xor butterfly inside the
// aligned K-lane group).  Ties of the fourth difference keep the smaller
// axis, as the reference's strict '>' scan does.
template <int K>
__device__ __forceinline__ void reduce_lanes(RegionSums& r, unsigned mask) {
#pragma unroll
  for (int off = K / 2; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) r.S[k] += __shfl_xor_sync(mask, r.S[k], off);
    const double ob = __shfl_xor_sync(mask, r.best, off);
    const int oa = __shfl_xor_sync(mask, r.axis, off);
    const bool take = (ob > r.best) || (ob == r.best && oa >= 0 && (r.axis < 0 || oa < r.axis));
    if (take) {
      r.best = ob;
      r.axis = oa;
    }
  }
}

struct RegionResult {
  double avg, err;
  int axis;
};

// Rule sums -> value, null-rule error, split axis (GPUQuadSample.cu:195-216).
// jac is the box volume times 2^-div; fallback_axis is used when every
// fourth difference is zero.
template <int N>
__device__ __forceinline__ RegionResult finish_region(const RegionSums& r, const RuleTables& T,
                                                      double jac, int fallback_axis) {
  double sum[kNumRules];
#pragma unroll
  for (int q = 0; q < kNumRules; ++q) {
    double acc = 0;
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) acc = __dadd_rn(acc, __dmul_rn(T.wt[k][q], r.S[k]));
    sum[q] = __dmul_rn(acc, jac);
  }
  double nul[kNumRules];
#pragma unroll
  for (int q = 1; q < kNumRules - 1; ++q) {
    double m = 0;
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) {
      const double e =
          __dmul_rn(fabs(__dadd_rn(sum[q + 1], __dmul_rn(T.scale[k][q], sum[q]))), T.norm[k][q]);
      m = (m > e) ? m : e;
    }
    nul[q] = m;
  }
  RegionResult out;
  out.avg = sum[0];
  const double m12 = nul[1] > nul[2] ? nul[1] : nul[2];
  const double m123 = m12 > nul[3] ? m12 : nul[3];
  out.err = (__dmul_rn(5.0, nul[1]) <= nul[2] && __dmul_rn(5.0, nul[2]) <= nul[3])
                ? nul[1]
                : __dmul_rn(5.0, m123);
  out.axis = r.axis >= 0 ? r.axis : fallback_axis;
  return out;
}

}  // namespace detail
}  // namespace cubature
