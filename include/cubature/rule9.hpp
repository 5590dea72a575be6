// rule9.hpp -- host construction of the degree-9 fully symmetric cubature
// rule (9 generator sets, 5 embedded rules) and its null-rule tables.
//
// The rule is the one the reference engine hard-codes (RULE 9,
// quad/quad.h:73; tables built in quad/GPUquad/GPUQuadRule.cu:31-228).  The
// weights are polynomials in the dimension n; each polynomial is evaluated
// in the same order as the reference so the tables are bit-identical.
#pragma once

#include <cmath>
#include <cstring>

namespace cubature {

constexpr int kNumSets = 9;
constexpr int kNumRules = 5;
constexpr int kMaxDim = 16;

// Generator magnitudes (GPUQuadRule.cu:159-163).
constexpr double kGenA1 = .47795365790226950619;
constexpr double kGenA2 = .20302858736911986780;
constexpr double kGenA3 = .44762735462617812882;
constexpr double kGenA4 = .125;
constexpr double kGenL = .34303789878087814570;

// Points of the rule in n dimensions (quad/quad.h:83-85).
inline constexpr int rule9_points(int n) {
  return 1 + 8 * n + 6 * n * (n - 1) + 4 * n * (n - 1) * (n - 2) / 3 + (1 << n);
}

// Per-dimension rule tables, passed by value to the kernels.
struct RuleTables {
  double wt[kNumSets][kNumRules];     // weights of the 5 embedded rules
  double scale[kNumSets][kNumRules];  // null-rule combination factors
  double norm[kNumSets][kNumRules];   // 1-norm normalisation
  int count[kNumSets];                // points per generator set
  double ratio;                       // (a2/a1)^2 for the fourth difference
  int ndim;
  int npoints;
};

inline RuleTables make_rule9_tables(int ndim) {
  RuleTables T;
  std::memset(&T, 0, sizeof(T));
  const double n = static_cast<double>(ndim);
  const int ni = ndim;
  // Shared sub-polynomials of GPUQuadRule.cu:33-114.
  const double p0 = n * (n * (n * (-.0023611709677855117884) + .11415390023857325268) +
                         (-.63833920076702389094)) + .74849988504685208004;
  const double p1 = n * (n * (n * (-.0014324017033399125142) + .057471507864489725949) +
                         (-.14225104571434243234)) - (-.062875028738286979989);
  const double q0 = n * (n * .0035417564516782676826 + (-.072609367395893679605)) +
                    .10557491625218991012;
  const double q1 = n * (n * .0021486025550098687713 + (-.032268563892953949998)) +
                    .010636783990231217481;
  const double r0 = n * (-.04508628929435784076) + .21415883524352793401;
  const double r1 = n * (-.027351546526545644722) + .054941067048711234101;
  const double s0 = .015532417276607053264 - n * .0035417564516782676826;
  const double s1 = .0035328099607090870236 - n * .0021486025550098687713;
  const double t0 = .25150011495314791996 / static_cast<double>(1 << ni);
  const double t1 = -.062875028738286979989 / static_cast<double>(1 << ni);
  const double w[kNumSets][kNumRules] = {
      {p0, p1, n * (.254591133248959089) - p1,
       n * (n * (-1.207328566678236261) + .89567365764160676508) - 1 + p0,
       n * (-.36479356986049146661) + 1 - p0},
      {q0, q1, .014689102496143490175 - q1,
       n * .51134708346467591431 + .45976448120806344646 + q0, .18239678493024573331 - q0},
      {r0, r1, .11937596202570775297 - r1, n * .65089519391920250593 + .14744939829434460168,
       -r0},
      {.057693384490973483573, .034999626602143583822, -.057693384490973483573,
       -1.3868627719278281436, -.057693384490973483573},
      {0, 0, -.2386668732575008879, 0, 0},
      {s0, s1, -s1,
       .09231719987444221619 + .015532417276607053264 - n * .0035417564516782676826, -s0},
      {.02254314464717892038, .013675773263272822361, -.013675773263272822361,
       -.32544759695960125297, -.02254314464717892038},
      {.0017708782258391338413, .0010743012775049343856, -.0010743012775049343856,
       .0017708782258391338413, -.0017708782258391338413},
      {t0, t1, -t1, t0, -t0}};
  std::memcpy(T.wt, w, sizeof(w));
  const int cnt[kNumSets] = {1,
                             2 * ni,
                             2 * ni,
                             2 * ni,
                             2 * ni,
                             2 * ni * (ni - 1),
                             4 * ni * (ni - 1),
                             4 * ni * (ni - 1) * (ni - 2) / 3,
                             1 << ni};
  std::memcpy(T.count, cnt, sizeof(cnt));
  // Null rules (GPUQuadRule.cu:209-227): for each set k and rule q in 1..3
  // the combination of rules q and q+1 that vanishes on set k's weight.
  for (int k = 0; k < kNumSets; ++k) {
    for (int q = 1; q < kNumRules - 1; ++q) {
      const double scale = (T.wt[k][q] == 0) ? 100 : -T.wt[k][q + 1] / T.wt[k][q];
      double sum = 0;
      for (int x = 0; x < kNumSets; ++x)
        sum += T.count[x] * std::fabs(T.wt[x][q + 1] + scale * T.wt[x][q]);
      T.scale[k][q] = scale;
      T.norm[k][q] = 1 / sum;
    }
  }
  T.ratio = (kGenA2 / kGenA1) * (kGenA2 / kGenA1);
  T.ndim = ndim;
  T.npoints = rule9_points(ndim);
  return T;
}

}  // namespace cubature
