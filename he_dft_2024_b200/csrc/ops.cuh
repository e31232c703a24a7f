// ops.cuh -- consumers fused into the 13-point stencil pass, pointwise passes and the classical
// impurity integrator (binary64).
#pragma once
#include "stencil.cuh"

namespace he {

// ---- absorbing mask: timec = (Lambdah*(1+tx+1+ty+1+tz), 1)  (DFT4He3d.f90:592-601) -----------
struct Timec {
  const double* ax;  // tanh((|x_i|-txmean)/txsurf), host-evaluated per axis
  const double* ay;
  const double* az;
  double lambdah;
  HE_D void remap(const MemberMap& mm, int m) {
    ax = mm(ax, m);
    ay = mm(ay, m);
    az = mm(az, m);
  }
  // lambdah * (((1 + ax) + 1 + ay) + 1 + az), summed left to right; the stencil pass evaluates
  // the x-y part once per column (xy) and adds each plane's az (with_z)
  HE_D double xy(int ix, int iy) const { return (1.0 + ax[ix]) + 1.0 + ay[iy]; }
  HE_D double with_z(double sxy, double azv) const { return lambdah * (sxy + 1.0 + azv); }
  HE_D double re(int ix, int iy, int iz) const { return with_z(xy(ix, iy), az[iz]); }
};


// remap helpers for the Ops' operand arrays
template <class P, int K>
HE_D void remap_all(P* (&a)[K], const MemberMap& mm, int m) {
  for (int k = 0; k < K; ++k) a[k] = mm(a[k], m);
}

// H psi of the real-time classical path (steprk.f90:67, steppc.f90:51,118):
//   timec*((d2x+d2y+d2z)*h2o2m4 - pot4*psi) - i*uimp*psi,  timec = (tr, 1).
HE_D double2 hpsi_rt(double2 dx, double2 dy, double2 dz, double2 c, double pot, double u,
                     double tr, double h2o2m) {
  const double2 lap = cadd(cadd(dx, dy), dz);
  const double ax = lap.x * h2o2m - pot * c.x;
  const double ay = lap.y * h2o2m - pot * c.y;
  return make_double2(tr * ax - ay + u * c.y, tr * ay + ax - u * c.x);
}

// H psi of the quantum-impurity path (Dynamics_quantum_impurities/steprk.f90:68,94,
// steppc.f90:46,77): timec*((d2x+d2y+d2z)*h2o2m - v*psi), v = pot4 - mu4 for He and upotx_i
// for impurity i (no -i*uimp term: the impurities enter through the potentials).
HE_D double2 hpsi_q(double2 dx, double2 dy, double2 dz, double2 c, double v, double tr,
                    double h2o2m) {
  const double2 lap = cadd(cadd(dx, dy), dz);
  const double ax = lap.x * h2o2m - v * c.x;
  const double ay = lap.y * h2o2m - v * c.y;
  return make_double2(tr * ax - ay, tr * ay + ax);
}

// H psi of either path from the staged operands: QU = false reads {pot4, uimp}, QU = true reads
// {pot} and subtracts the constant mu.
template <bool QU>
HE_D double2 hpsi_any(double2 dx, double2 dy, double2 dz, double2 c, const double* v8, int vs,
                      double mu, double tr, double h2o2m) {
  if constexpr (QU) return hpsi_q(dx, dy, dz, c, v8[0] - mu, tr, h2o2m);
  else return hpsi_rt(dx, dy, dz, c, v8[0], v8[vs], tr, h2o2m);
}

// steppc predictor + modifier (steppc.f90:51-61; quantum path steppc.f90:46-56, :77-87).  po3 =
// psiold(ioldp(3)) is read and receives the new psi (the host then swaps it with the psi buffer,
// so psiold(ioldp(3)) holds the old psi).
template <bool QU>
struct OpPredictT {
  static const char* kname() { return QU ? "hpsi_pmc_predict_q" : "hpsi_pmc_predict"; }
  using T = double2;
  static constexpr int NV = 0, N8 = QU ? 1 : 2, N16 = 4;
  const double* s8[N8];      // pot4, uimp (QU: pot4 or upotx_i)
  const double2* s16[N16];   // psiold(ioldp(3)), hpsiold(ioldh(1)), hpsiold(ioldh(2)), pc
  double2* po3;
  double2* h2;
  double2* pc;
  double* den;
  Timec tm;
  double h2o2m, s43, c112, mu;
  HE_D void remap(const MemberMap& mm, int m) {
    remap_all(s8, mm, m); remap_all(s16, mm, m);
    po3 = mm(po3, m); h2 = mm(h2, m); pc = mm(pc, m); den = mm(den, m); tm.remap(mm, m);
  }
  HE_D void at_t(int ix, int iy, int iz, long i, double2 dx, double2 dy, double2 dz, double2 c,
               const double* v8, const double2* v16, int vs, double*, double tr) const {
    const double2 s4 = hpsi_any<QU>(dx, dy, dz, c, v8, vs, mu, tr, h2o2m);
    const double2 p3 = v16[0], hh1 = v16[vs], hh2 = v16[2 * vs], pcv = v16[3 * vs];
    const double2 t = make_double2(2.0 * s4.x - hh1.x + 2.0 * hh2.x, 2.0 * s4.y - hh1.y + 2.0 * hh2.y);
    const double2 sto1 = make_double2(p3.x + s43 * t.x, p3.y + s43 * t.y);
    const double2 pn = make_double2(sto1.x - c112 * pcv.x, sto1.y - c112 * pcv.y);
    pc[i] = sto1;
    h2[i] = s4;
    po3[i] = pn;
    den[i] = cnorm2(pn);
  }
};

// steppc corrector + final value (steppc.f90:118-127; quantum path steppc.f90:105-137);
// accumulates sum |pc|.
template <bool QU>
struct OpCorrectT {
  static const char* kname() { return QU ? "hpsi_pmc_correct_q" : "hpsi_pmc_correct"; }
  using T = double2;
  static constexpr int NV = 1, N8 = QU ? 1 : 2, N16 = 5;
  const double* s8[N8];      // pot4, uimp (QU: pot4 or upotx_i)
  const double2* s16[N16];   // psiold(ioldp(3)), psiold(ioldp(2)), hpsiold(ioldh(1)), (ioldh(2)), pc
  double2* pc;
  double2* out;
  double* den;
  Timec tm;
  double h2o2m, s3, c9, mu;
  HE_D void remap(const MemberMap& mm, int m) {
    remap_all(s8, mm, m); remap_all(s16, mm, m);
    pc = mm(pc, m); out = mm(out, m); den = mm(den, m); tm.remap(mm, m);
  }
  HE_D void at_t(int ix, int iy, int iz, long i, double2 dx, double2 dy, double2 dz, double2 c,
               const double* v8, const double2* v16, int vs, double* acc, double tr) const {
    const double2 s4 = hpsi_any<QU>(dx, dy, dz, c, v8, vs, mu, tr, h2o2m);
    const double2 a3 = v16[0], a2 = v16[vs], b1 = v16[2 * vs], b2 = v16[3 * vs], p = v16[4 * vs];
    const double2 inner = make_double2(s4.x + 2.0 * b1.x - b2.x, s4.y + 2.0 * b1.y - b2.y);
    const double2 s5 = make_double2(0.125 * (9.0 * a3.x - a2.x + s3 * inner.x),
                                    0.125 * (9.0 * a3.y - a2.y + s3 * inner.y));
    const double2 pn = make_double2(p.x - s5.x, p.y - s5.y);
    pc[i] = pn;
    const double2 o = make_double2(s5.x + c9 * pn.x, s5.y + c9 * pn.y);
    out[i] = o;
    den[i] = cnorm2(o);
    acc[0] += hypot(pn.x, pn.y);
  }
};

// One RK-Gill stage (steprk.f90:67-79; quantum path steprk.f90:68-80, :94-104).  hsave (stage 1
// only) receives H psi for hpsiold(1).
template <bool QU>
struct OpRKT {
  static const char* kname() { return QU ? "hpsi_rkgill_stage_q" : "hpsi_rkgill_stage"; }
  using T = double2;
  static constexpr int NV = 0, N8 = QU ? 1 : 2, N16 = 1;
  const double* s8[N8];      // pot4, uimp (QU: pot4 or upotx_i)
  const double2* s16[N16];   // q
  double2* q;
  double2* out;
  double2* hsave;
  double* den;
  Timec tm;
  double h2o2m, a, b, cc, dt, mu;
  HE_D void remap(const MemberMap& mm, int m) {
    remap_all(s8, mm, m); remap_all(s16, mm, m);
    q = mm(q, m); out = mm(out, m); hsave = mm(hsave, m); den = mm(den, m); tm.remap(mm, m);
  }
  HE_D void at_t(int ix, int iy, int iz, long i, double2 dx, double2 dy, double2 dz, double2 c,
               const double* v8, const double2* v16, int vs, double*, double tr) const {
    const double2 s4 = hpsi_any<QU>(dx, dy, dz, c, v8, vs, mu, tr, h2o2m);
    const double2 qq = v16[0];
    const double2 s1 = make_double2(a * (s4.x - b * qq.x), a * (s4.y - b * qq.y));
    q[i] = make_double2(qq.x + 3.0 * s1.x - cc * s4.x, qq.y + 3.0 * s1.y - cc * s4.y);
    if (hsave) hsave[i] = s4;
    const double2 pn = make_double2(c.x + dt * s1.x, c.y + dt * s1.y);
    out[i] = pn;
    den[i] = cnorm2(pn);
  }
};

using OpPredict = OpPredictT<false>;
using OpCorrect = OpCorrectT<false>;
using OpRK = OpRKT<false>;
using OpPredictQ = OpPredictT<true>;
using OpCorrectQ = OpCorrectT<true>;
using OpRKQ = OpRKT<true>;

// ---- the mixed path (HE_PREC_MIXED, classical dynamics) --------------------------------------
// psi and its history psiold are compensated binary32 pairs held as two float2 planes of one
// allocation (hi at [0, N), lo at [N, 2N)); the stencil differentiates the hi plane.  H psi, the
// history terms hpsiold, pc, q and the fields den, pot4, uimp are binary32.  The updates of psi
// (the RK-Gill stage, the Milne predictor, the Hamming corrector) are done on the pairs with
// error-free transformations, so psi keeps about 48 significant bits over the run while every
// stream but psi is half as wide as in binary64.
struct HL2 {
  HL x, y;
};
HE_D HL2 hl2(float2 hi, float2 lo) { return HL2{HL{hi.x, lo.x}, HL{hi.y, lo.y}}; }
HE_D HL2 hl2_add(HL2 a, float2 b) { return HL2{hl_add(a.x, b.x), hl_add(a.y, b.y)}; }
HE_D void hl2_store(float2* hi, float2* lo, long i, HL2 v) {
  hi[i] = make_float2(v.x.hi, v.y.hi);
  lo[i] = make_float2(v.x.lo, v.y.lo);
}
HE_D float den_of(HL2 v) {  // |psi|^2 of the pair, rounded once
  const double re = hl_value(v.x), im = hl_value(v.y);
  return (float)(re * re + im * im);
}

// H psi in binary32 (the binary64 hpsi_rt with float operands).
HE_D float2 hpsi_rt_f(float2 dx, float2 dy, float2 dz, float2 c, float pot, float u, float tr,
                      float h2o2m) {
  const float lx = dx.x + dy.x + dz.x, ly = dx.y + dy.y + dz.y;
  const float ax = lx * h2o2m - pot * c.x;
  const float ay = ly * h2o2m - pot * c.y;
  return make_float2(tr * ax - ay + u * c.y, tr * ay + ax - u * c.x);
}

// H psi of the quantum-impurity path in binary32: timec*(lap*h2o2m - v psi), v = pot - mu.
HE_D float2 hpsi_q_f(float2 dx, float2 dy, float2 dz, float2 c, float v, float tr, float h2o2m) {
  const float lx = dx.x + dy.x + dz.x, ly = dx.y + dy.y + dz.y;
  const float ax = lx * h2o2m - v * c.x;
  const float ay = ly * h2o2m - v * c.y;
  return make_float2(tr * ax - ay, tr * ay + ax);
}
// Either path from the staged operands: QU = false reads {pot4, uimp}, QU = true reads {pot}.
template <bool QU>
HE_D float2 hpsi_any_f(float2 dx, float2 dy, float2 dz, float2 c, const float* v8, int vs,
                       float mu, float tr, float h2o2m) {
  if constexpr (QU) return hpsi_q_f(dx, dy, dz, c, v8[0] - mu, tr, h2o2m);
  else return hpsi_rt_f(dx, dy, dz, c, v8[0], v8[vs], tr, h2o2m);
}

// One RK-Gill stage (steprk.f90:67-79; quantum path steprk.f90:68-104) on the pair planes.
template <bool QU>
struct OpRKMT {
  static const char* kname() { return QU ? "hpsi_rkgill_stage_q_f32" : "hpsi_rkgill_stage_f32"; }
  using T = float2;
  static constexpr int NV = 0, N8 = QU ? 1 : 2, N16 = 2;
  const float* s8[N8];       // pot4, uimp (QU: pot4 or upotx_i)
  const float2* s16[N16];    // q, psi lo plane
  float2* q;
  float2* out_hi;
  float2* out_lo;
  float2* hsave;
  float* den;
  Timec tm;
  float h2o2m, a, b, cc, dt, mu;
  HE_D void remap(const MemberMap& mm, int m) {
    remap_all(s8, mm, m); remap_all(s16, mm, m);
    q = mm(q, m); out_hi = mm(out_hi, m); out_lo = mm(out_lo, m); hsave = mm(hsave, m);
    den = mm(den, m); tm.remap(mm, m);
  }
  HE_D void at_t(int ix, int iy, int iz, long i, float2 dx, float2 dy, float2 dz, float2 c,
               const float* v8, const float2* v16, int vs, double*, double tr) const {
    const float2 s4 = hpsi_any_f<QU>(dx, dy, dz, c, v8, vs, mu, (float)tr, h2o2m);
    const float2 qq = v16[0];
    const float2 s1 = make_float2(a * (s4.x - b * qq.x), a * (s4.y - b * qq.y));
    q[i] = make_float2(qq.x + 3.0f * s1.x - cc * s4.x, qq.y + 3.0f * s1.y - cc * s4.y);
    if (hsave) hsave[i] = s4;
    const HL2 pn = hl2_add(hl2(c, v16[vs]), make_float2(dt * s1.x, dt * s1.y));
    hl2_store(out_hi, out_lo, i, pn);
    den[i] = den_of(pn);
  }
};

// steppc predictor + modifier (steppc.f90:51-61) on the pair planes: psi_pred = po3 +
// (s43 (2 H psi - hh1 + 2 hh2) - c112 pc), written over po3.  pc is not overwritten with the
// unmodified prediction sto1 (a full-size value the binary32 pc could not hold); the corrector
// rebuilds sto1 = psi_pred + c112 pc from the predicted pair instead.
template <bool QU>
struct OpPredictMT {
  static const char* kname() { return QU ? "hpsi_pmc_predict_q_f32" : "hpsi_pmc_predict_f32"; }
  using T = float2;
  static constexpr int NV = 0, N8 = QU ? 1 : 2, N16 = 5;
  const float* s8[N8];       // pot4, uimp (QU: pot4 or upotx_i)
  const float2* s16[N16];    // po3 hi, po3 lo, hpsiold(ioldh(1)), hpsiold(ioldh(2)), pc
  float2* po3_hi;
  float2* po3_lo;
  float2* h2;
  float* den;
  Timec tm;
  float h2o2m, s43, c112, mu;
  HE_D void remap(const MemberMap& mm, int m) {
    remap_all(s8, mm, m); remap_all(s16, mm, m);
    po3_hi = mm(po3_hi, m); po3_lo = mm(po3_lo, m); h2 = mm(h2, m); den = mm(den, m);
    tm.remap(mm, m);
  }
  HE_D void at_t(int ix, int iy, int iz, long i, float2 dx, float2 dy, float2 dz, float2 c,
               const float* v8, const float2* v16, int vs, double*, double tr) const {
    const float2 s4 = hpsi_any_f<QU>(dx, dy, dz, c, v8, vs, mu, (float)tr, h2o2m);
    const float2 hh1 = v16[2 * vs], hh2 = v16[3 * vs], pcv = v16[4 * vs];
    const float2 t = make_float2(2.0f * s4.x - hh1.x + 2.0f * hh2.x, 2.0f * s4.y - hh1.y + 2.0f * hh2.y);
    const float2 d = make_float2(s43 * t.x - c112 * pcv.x, s43 * t.y - c112 * pcv.y);
    const HL2 pn = hl2_add(hl2(v16[0], v16[vs]), d);
    h2[i] = s4;
    hl2_store(po3_hi, po3_lo, i, pn);
    den[i] = den_of(pn);
  }
};

// steppc corrector + final value (steppc.f90:118-127) on the pair planes; accumulates sum |pc|.
//   s5 = (9 a3 - a2 + s3 (H psi_pred + 2 b1 - b2)) / 8          (pairs)
//   pc = sto1 - s5 = (psi_pred - s5) + c112 pc_old              (a small difference, binary32)
//   psi = s5 + c9 pc                                            (pair)
template <bool QU>
struct OpCorrectMT {
  static const char* kname() { return QU ? "hpsi_pmc_correct_q_f32" : "hpsi_pmc_correct_f32"; }
  using T = float2;
  static constexpr int NV = 1, N8 = QU ? 1 : 2, N16 = 8;
  const float* s8[N8];       // pot4, uimp (QU: pot4 or upotx_i)
  const float2* s16[N16];    // psi_pred lo, a3 hi, a3 lo, a2 hi, a2 lo, hpsiold(ioldh(1)),
                             // hpsiold(ioldh(2)), pc
  float2* pc;
  float2* out_hi;
  float2* out_lo;
  float* den;
  Timec tm;
  float h2o2m, s3, c9, c112, mu;
  HE_D void remap(const MemberMap& mm, int m) {
    remap_all(s8, mm, m); remap_all(s16, mm, m);
    pc = mm(pc, m); out_hi = mm(out_hi, m); out_lo = mm(out_lo, m); den = mm(den, m);
    tm.remap(mm, m);
  }
  HE_D void at_t(int ix, int iy, int iz, long i, float2 dx, float2 dy, float2 dz, float2 c,
               const float* v8, const float2* v16, int vs, double* acc, double tr) const {
    const float2 s4 = hpsi_any_f<QU>(dx, dy, dz, c, v8, vs, mu, (float)tr, h2o2m);
    const HL2 pred = hl2(c, v16[0]);
    const HL2 a3 = hl2(v16[vs], v16[2 * vs]), a2 = hl2(v16[3 * vs], v16[4 * vs]);
    const float2 b1 = v16[5 * vs], b2 = v16[6 * vs], pco = v16[7 * vs];
    const float2 inner = make_float2(s3 * (s4.x + 2.0f * b1.x - b2.x), s3 * (s4.y + 2.0f * b1.y - b2.y));
    HL s5x = hl_add(hl_add(hl_mul(9.0f, a3.x), hl_neg(a2.x)), inner.x);
    HL s5y = hl_add(hl_add(hl_mul(9.0f, a3.y), hl_neg(a2.y)), inner.y);
    s5x = HL{0.125f * s5x.hi, 0.125f * s5x.lo};
    s5y = HL{0.125f * s5y.hi, 0.125f * s5y.lo};
    const HL dx_ = hl_add(pred.x, hl_neg(s5x)), dy_ = hl_add(pred.y, hl_neg(s5y));
    const float2 pn = make_float2((dx_.hi + dx_.lo) + c112 * pco.x, (dy_.hi + dy_.lo) + c112 * pco.y);
    pc[i] = pn;
    const HL2 o = HL2{hl_add(s5x, c9 * pn.x), hl_add(s5y, c9 * pn.y)};
    hl2_store(out_hi, out_lo, i, o);
    den[i] = den_of(o);
    acc[0] += hypot((double)pn.x, (double)pn.y);
  }
};

using OpRKM = OpRKMT<false>;
using OpPredictM = OpPredictMT<false>;
using OpCorrectM = OpCorrectMT<false>;
using OpRKMQ = OpRKMT<true>;
using OpPredictMQ = OpPredictMT<true>;
using OpCorrectMQ = OpCorrectMT<true>;

// energy(): Dynamics_TDDFT/energy.f90:107-165 sums (first derivatives of psi).
//   acc = {sum |grad psi|^2, sum delj4*den, sum den*dencg^2*(cp4/2+cpp4/3*dencg),
//          sum den*(1+tanh(beta*(den-den_m))), sum uimp*den}
// TT = float2 (the mixed path): gradients of the binary32 psi planes, the sums in binary64.
template <typename TT>
struct OpEnergy {
  static const char* kname() { return sizeof(TT) == 8 ? "energy_reduce_f32" : "energy_reduce"; }
  using T = TT;
  using R = typename RealOf<TT>::R;
  using Z = typename RealOf<TT>::Z;
  static constexpr int NV = 5, N8 = 4, N16 = 0;
  const R* s8[N8];           // den, dencg, delj4, uimp (den again when there is no uimp)
  const Z* s16[1];
  double aux1, aux2, beta, den_m;
  int lsolid, has_u;
  HE_D void remap(const MemberMap& mm, int m) {
    for (int k = 0; k < N8; ++k) s8[k] = mm(s8[k], m);
  }
  HE_D static double n2(double v) { return v * v; }
  HE_D static double n2(double2 v) { return v.x * v.x + v.y * v.y; }
  HE_D static double n2(float v) { return (double)v * (double)v; }
  HE_D static double n2(float2 v) { return (double)v.x * (double)v.x + (double)v.y * (double)v.y; }
  HE_D void at(int, int, int, long, T dx, T dy, T dz, T, const R* v8, const Z*, int vs,
               double* acc) const {
    const double a3 = v8[0], a4 = v8[vs];
    acc[0] += n2(dx) + n2(dy) + n2(dz);
    acc[1] += (double)v8[2 * vs] * a3;
    acc[2] += a3 * a4 * a4 * (aux1 + aux2 * a4);
    if (lsolid) acc[3] += a3 * (1.0 + tanh(beta * (a3 - den_m)));
    if (has_u) acc[4] += (double)v8[3 * vs] * a3;
  }
};

// Droplet observables of the dynamics driver (Dynamics_TDDFT/DFT4He3d.f90:720-838, r_cm.f90) in
// one pass over psi: with c_a = conj(psi) d_a psi, acc holds
//   [0..2]  Im sum c_x, c_y, c_z                   (<Vcom> = Im sum c_a dxyz / (N mhe))
//   [3..8]  Im sum y c_x, x c_y, x c_z, z c_x, z c_y, y c_z   (<L> about the origin; the
//           shift to the centre of mass uses [0..2] on the host)
//   [9..15] sum den, den x, den y, den z, den x^2, den y^2, den z^2     (N, r_cm, <r^2>)
// TT = float2: the mixed path's binary32 psi planes (products and sums in binary64).
template <typename TT>
struct OpObservablesT {
  static const char* kname() { return sizeof(TT) == 8 ? "observables_reduce_f32" : "observables_reduce"; }
  using T = TT;
  using R = typename RealOf<TT>::R;
  using Z = typename RealOf<TT>::Z;
  static constexpr int NV = 16, N8 = 1, N16 = 0;
  const R* s8[N8];           // den
  const Z* s16[1];
  double x0, y0, z0, hx, hy, hz;
  HE_D void at(int ix, int iy, int iz, long, T dx, T dy, T dz, T c, const R* v8, const Z*, int,
               double* acc) const {
    const double x = x0 + hx * ix, y = y0 + hy * iy, z = z0 + hz * iz;
    const double cr = c.x, ci = c.y;
    const double cx = cr * (double)dx.y - ci * (double)dx.x;  // Im conj(psi) d_x psi
    const double cy = cr * (double)dy.y - ci * (double)dy.x;
    const double cz = cr * (double)dz.y - ci * (double)dz.x;
    acc[0] += cx;
    acc[1] += cy;
    acc[2] += cz;
    acc[3] += y * cx;
    acc[4] += x * cy;
    acc[5] += x * cz;
    acc[6] += z * cx;
    acc[7] += z * cy;
    acc[8] += y * cz;
    const double d = v8[0];
    acc[9] += d;
    acc[10] += d * x;
    acc[11] += d * y;
    acc[12] += d * z;
    acc[13] += d * (x * x);
    acc[14] += d * (y * y);
    acc[15] += d * (z * z);
  }
};
using OpObservables = OpObservablesT<double2>;

// derden(): dxden, dyden, dzden (derden.f90:26-28).
struct OpDerden {
  static const char* kname() { return "derden"; }
  using T = double;
  static constexpr int NV = 0, N8 = 0, N16 = 0;
  const double* s8[1];
  const double2* s16[1];
  double* gx;
  double* gy;
  double* gz;
  HE_D void remap(const MemberMap& mm, int m) {
    gx = mm(gx, m);
    gy = mm(gy, m);
    gz = mm(gz, m);
  }
  HE_D void at(int, int, int, long i, double dx, double dy, double dz, double, const double*,
               const double2*, int, double*) const {
    gx[i] = dx;
    gy[i] = dy;
    gz[i] = dz;
  }
};

// ---- classical impurities ----------------------------------------------------------------------
constexpr int kMaxImp = 8;

// Device copy of the classicimp module (modules.f90:303-343).  Arrays use the Fortran layout
// with leading dimension n: (n,3) -> k + n*c, (n,3,slot) -> k + n*c + 3n*(slot-1).
struct ImpDev {
  int n;
  double m[kMaxImp];
  double rimp[3 * kMaxImp], vimp[3 * kMaxImp], aimp[3 * kMaxImp], F[3 * kMaxImp];
  double qr[3 * kMaxImp], qv[3 * kMaxImp], pcr[3 * kMaxImp], pcv[3 * kMaxImp];
  double rimpold[9 * kMaxImp], vimpold[9 * kMaxImp], aimpold[6 * kMaxImp];
  int ioldr[3], ioldv[3], iolda[2];
  double errimp, errvimp;
  int lstopimp, lgridnoout;
  int ii_kind;
  double ii_D, ii_re, ii_a, ii_rcut, ii_umax;
};

// updatepoten + the He part of forceimp (potenimp.f90:95-121, :49-52) in one stencil pass over
// den: uimp = sum_k V_k(|r-R_k|) by linear interpolation of the potenimpini table, and
// acc[3k+c] = sum d_c(den) * V_k.  Off-table radii set lstopimp (potenimp.f90:104-109); the
// radius is clamped to the table end and the index is taken after the clamp.
// The table index is int(r/DelInter) with the rounded IEEE quotient and the fraction is
// mod(r,DelInter)/DelInter with the exact remainder, as in the reference: when r/DelInter rounds
// up to an integer k although the exact quotient is below k, the reference takes bin k with a
// fraction of ~1 (it interpolates one bin further out), and so does this kernel.  The remainder
// r - i0*DelInter is one exact fma when i0 is the exact floor, else r - (i0-1)*DelInter.
// The index comes from q = r * (1/DelInter) instead of a division: with 1/DelInter rounded once
// and the product rounded once, q is within (r/DelInter) 2^-52 of r/DelInter and the IEEE
// quotient within (r/DelInter) 2^-53, so for q < 2^17 the two differ by less than 4.4e-11.
// Whenever q lies 1e-9 or more inside its unit interval both have the same integer part; closer
// to an integer (or for q >= 2^17) the IEEE division decides.
// The fraction is rm/DelInter as rm * (1/DelInter) refined by one residual step (a Newton
// correction, q1 = q0 + (rm - q0 DelInter)/DelInter, with the residual from an fma).
// kMinBlocks: 4 resident CTAs (64 registers); the pass is latency-bound and measured 54 -> 48 us
// per launch at 128^3 with the two changes.
// TT = float: the mixed path (binary32 den and uimp; positions, table and sums in binary64).
template <int NI, typename TT = double>
struct OpImpField {
  static const char* kname() { return sizeof(TT) == 4 ? "impurity_field_force_f32" : "impurity_field_force"; }
  using T = TT;
  static constexpr int NV = 3 * NI;
  const double* tab;  // (npot) per impurity, impurity-major
  ImpDev* imp;
  TT* uimp;
  int n, npot;
  double delinter, rmax, inv_delinter;
  double xmax, ymax, zmax, hx, hy, hz;
  static constexpr int N8 = 0, N16 = 0;
  static constexpr int kMinBlocks = 4;
  const TT* s8[1];
  const typename RealOf<TT>::Z* s16[1];
  HE_D void at(int ix, int iy, int iz, long i, TT dx, TT dy, TT dz, TT, const TT*,
               const typename RealOf<TT>::Z*, int, double* acc) const {
    const double x = -xmax + hx * ix, y = -ymax + hy * iy, z = -zmax + hz * iz;
    const double* __restrict__ rp = imp->rimp;
    double u = 0.0;
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      if (k < n) {
        const double rx = __ldg(rp + k), ry = __ldg(rp + k + n), rz = __ldg(rp + k + 2 * n);
        const double zt = (z - rz) * (z - rz);
        const double yt = (y - ry) * (y - ry) + zt;
        double r = sqrt((x - rx) * (x - rx) + yt);
        if (!(r <= rmax)) {  // also catches a NaN radius
          if (imp->lgridnoout) atomicExch(&imp->lstopimp, 1);
          r = rmax;
        }
        const double qf = r * inv_delinter;
        int i0 = (int)qf;
        {
          const double fr = qf - (double)i0;
          if (fr < 1e-9 || fr > 1.0 - 1e-9 || qf >= 131072.0) i0 = (int)(r / delinter);
        }
        double rm = fma(-(double)i0, delinter, r);
        if (rm < 0.0) rm = fma(-(double)(i0 - 1), delinter, r);
        else if (rm >= delinter) rm = fmod(r, delinter);
        if (i0 > npot - 2) i0 = npot - 2;
        const double rr = rm * inv_delinter;
        const double rmod = fma(fma(-rr, delinter, rm), inv_delinter, rr);
        const double* __restrict__ t = tab + (long)k * npot;
        const double uk = __ldg(t + i0) * (1.0 - rmod) + __ldg(t + i0 + 1) * rmod;
        u = u + uk;
        acc[3 * k + 0] += (double)dx * uk;
        acc[3 * k + 1] += (double)dy * uk;
        acc[3 * k + 2] += (double)dz * uk;
      }
    }
    uimp[i] = (TT)u;
  }
};

// The impurity kernels run on one CTA: the ImpDev struct is copied into shared memory by the
// whole CTA, updated by thread 0 (the integrator is a few dozen scalars), and copied back.
HE_D void imp_stage_in(ImpDev* dst, const ImpDev* src) {
  const unsigned* a = reinterpret_cast<const unsigned*>(src);
  unsigned* b = reinterpret_cast<unsigned*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(ImpDev) / 4); i += blockDim.x) b[i] = a[i];
  __syncthreads();
}
HE_D void imp_stage_out(ImpDev* dst, const ImpDev* src) {
  __syncthreads();
  const unsigned* a = reinterpret_cast<const unsigned*>(src);
  unsigned* b = reinterpret_cast<unsigned*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(ImpDev) / 4); i += blockDim.x) b[i] = a[i];
}

HE_D double pair_pot(const ImpDev& s, double r) {
  if (s.ii_kind == 0) return (r < s.ii_rcut) ? s.ii_umax : 0.0;
  if (r < s.ii_rcut) return s.ii_umax;
  const double e = 1.0 - exp(-s.ii_a * (r - s.ii_re));
  return s.ii_D * (e * e - 1.0);
}
HE_D double pair_dpot(const ImpDev& s, double r) {
  if (s.ii_kind == 0 || r < s.ii_rcut) return 0.0;
  const double ex = exp(-s.ii_a * (r - s.ii_re));
  return 2.0 * s.ii_D * s.ii_a * (1.0 - ex) * ex;
}

// forceimp: F(k,c) = -sum(d_c den * uimp_k)*dxyz + sum_m F_ij(k,m,c)  (potenimp.f90:40-58).
HE_D void imp_force_body(ImpDev* s, const double* sums, double dxyz) {
  const int n = s->n;
  for (int k = 0; k < n; ++k)
    for (int c = 0; c < 3; ++c) s->F[k + n * c] = -sums[3 * k + c] * dxyz;
  for (int k = 0; k < n; ++k)
    for (int m = 0; m < n; ++m) {
      if (m == k) continue;
      double d[3];
      for (int c = 0; c < 3; ++c) d[c] = s->rimp[k + n * c] - s->rimp[m + n * c];
      const double a1 = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      const double dv = pair_dpot(*s, a1);
      for (int c = 0; c < 3; ++c) s->F[k + n * c] = s->F[k + n * c] + (-dv * d[c] / a1);
    }
}
#ifndef HE_KERNEL_TU
static __global__ void k_imp_force(ImpDev* g, const double* sums, double dxyz) {
  __shared__ ImpDev st;
  imp_stage_in(&st, g);
  if (threadIdx.x == 0) imp_force_body(&st, sums, dxyz);
  imp_stage_out(g, &st);
}
#endif

// aimp = F / m_imp (DFT4He3d.f90:571-573).
HE_D void imp_accel_body(ImpDev* s) {
  const int n = s->n;
  for (int k = 0; k < n; ++k)
    for (int c = 0; c < 3; ++c) s->aimp[k + n * c] = s->F[k + n * c] / s->m[k];
}
#ifndef HE_KERNEL_TU
static __global__ void k_imp_accel(ImpDev* g) {
  __shared__ ImpDev st;
  imp_stage_in(&st, g);
  if (threadIdx.x == 0) imp_accel_body(&st);
  imp_stage_out(g, &st);
}
#endif

// Impurity part of one RK-Gill stage (steprk.f90:92-125).
HE_D void imp_rk_body(ImpDev* s, int jr, double a, double b, double cc, double dt) {
  const int n = s->n;
  double stor[3 * kMaxImp];
  for (int i = 0; i < 3 * n; ++i) {
    stor[i] = a * (s->vimp[i] - b * s->qr[i]);
    s->qr[i] = s->qr[i] + 3.0 * stor[i] - cc * s->vimp[i];
  }
  if (jr == 0)
    for (int i = 0; i < 3 * n; ++i) {
      s->rimpold[i + 6 * n] = s->rimpold[i + 3 * n];
      s->rimpold[i + 3 * n] = s->rimpold[i];
      s->rimpold[i] = s->rimp[i];
    }
  for (int i = 0; i < 3 * n; ++i) s->rimp[i] = s->rimp[i] + dt * stor[i];
  for (int i = 0; i < 3 * n; ++i) {
    stor[i] = a * (s->aimp[i] - b * s->qv[i]);
    s->qv[i] = s->qv[i] + 3.0 * stor[i] - cc * s->aimp[i];
  }
  if (jr == 0)
    for (int i = 0; i < 3 * n; ++i) {
      s->aimpold[i + 3 * n] = s->aimpold[i];
      s->aimpold[i] = s->aimp[i];
      s->vimpold[i + 6 * n] = s->vimpold[i + 3 * n];
      s->vimpold[i + 3 * n] = s->vimpold[i];
      s->vimpold[i] = s->vimp[i];
    }
  for (int i = 0; i < 3 * n; ++i) s->vimp[i] = s->vimp[i] + dt * stor[i];
  if (jr == 3) {
    for (int i = 0; i < 3; ++i) { s->ioldr[i] = i + 1; s->ioldv[i] = i + 1; }
    for (int i = 0; i < 2; ++i) s->iolda[i] = i + 1;
  }
}
#ifndef HE_KERNEL_TU
static __global__ void k_imp_rk(ImpDev* g, int jr, double a, double b, double cc, double dt) {
  __shared__ ImpDev st;
  imp_stage_in(&st, g);
  if (threadIdx.x == 0) imp_rk_body(&st, jr, a, b, cc, dt);
  imp_stage_out(g, &st);
}
#endif

// Impurity predictor + modifier (steppc.f90:80-99).  The velocity prediction is stored in
// vimpold(:,:,ioldv(3)) and vimp keeps v_n, as in the reference.
HE_D void imp_predict_body(ImpDev* s, double dt) {
  const int n = s->n;
  const double c112 = 112.0 / 121.0, c4o3 = 4.0 / 3.0;
  const double sd = c4o3 * dt;
  const int r3 = 3 * n * (s->ioldr[2] - 1);
  const int v1 = 3 * n * (s->ioldv[0] - 1), v2 = 3 * n * (s->ioldv[1] - 1),
            v3 = 3 * n * (s->ioldv[2] - 1);
  const int a1 = 3 * n * (s->iolda[0] - 1), a2 = 3 * n * (s->iolda[1] - 1);
  for (int i = 0; i < 3 * n; ++i) {
    const double st = s->rimpold[r3 + i] +
                      sd * (2.0 * s->vimp[i] - s->vimpold[v1 + i] + 2.0 * s->vimpold[v2 + i]);
    s->rimpold[r3 + i] = s->rimp[i];
    s->rimp[i] = st - c112 * s->pcr[i];
    s->pcr[i] = st;
  }
  for (int i = 0; i < 3 * n; ++i) {
    const double st = s->vimpold[v3 + i] +
                      sd * (2.0 * s->aimp[i] - s->aimpold[a1 + i] + 2.0 * s->aimpold[a2 + i]);
    s->vimpold[v3 + i] = st - c112 * s->pcv[i];
    s->pcv[i] = st;
  }
  for (int i = 0; i < 3 * n; ++i) s->aimpold[a2 + i] = s->aimp[i];
  const int t = s->iolda[1];
  s->iolda[1] = s->iolda[0];
  s->iolda[0] = t;
}
#ifndef HE_KERNEL_TU
static __global__ void k_imp_predict(ImpDev* g, double dt) {
  __shared__ ImpDev st;
  imp_stage_in(&st, g);
  if (threadIdx.x == 0) imp_predict_body(&st, dt);
  imp_stage_out(g, &st);
}
#endif

// Impurity corrector (steppc.f90:149-174).  aimp is the value set by the driver before the step
// (the forceimp inside steppc refreshes F but not aimp), as in the reference.
HE_D void imp_correct_body(ImpDev* s, double dt) {
  const int n = s->n;
  const double c9 = 9.0 / 121.0;
  const double s3 = 3.0 * dt;
  int r2 = 3 * n * (s->ioldr[1] - 1), r3 = 3 * n * (s->ioldr[2] - 1);
  int v1 = 3 * n * (s->ioldv[0] - 1), v2 = 3 * n * (s->ioldv[1] - 1),
      v3 = 3 * n * (s->ioldv[2] - 1);
  const int a1 = 3 * n * (s->iolda[0] - 1), a2 = 3 * n * (s->iolda[1] - 1);
  double er = 0.0;
  for (int i = 0; i < 3 * n; ++i) {
    const double st = 0.125 * (9.0 * s->rimpold[r3 + i] - s->rimpold[r2 + i] +
                               s3 * (s->vimpold[v3 + i] + 2.0 * s->vimp[i] - s->vimpold[v1 + i]));
    s->pcr[i] = s->pcr[i] - st;
    s->rimp[i] = st + c9 * s->pcr[i];
  }
  for (int i = 0; i < 3 * n; ++i) er += fabs(c9 * s->pcr[i]);
  s->errimp = er * 0.3333333333 / n;
  int t = s->ioldr[2];
  s->ioldr[2] = s->ioldr[1];
  s->ioldr[1] = s->ioldr[0];
  s->ioldr[0] = t;
  double ev = 0.0;
  for (int i = 0; i < 3 * n; ++i) {
    const double st = 0.125 * (9.0 * s->vimp[i] - s->vimpold[v2 + i] +
                               s3 * (s->aimp[i] + 2.0 * s->aimpold[a1 + i] - s->aimpold[a2 + i]));
    s->pcv[i] = s->pcv[i] - st;
    s->vimpold[v3 + i] = s->vimp[i];
    s->vimp[i] = st + c9 * s->pcv[i];
  }
  for (int i = 0; i < 3 * n; ++i) ev += fabs(c9 * s->pcv[i]);
  s->errvimp = ev * 0.3333333333 / n;
  t = s->ioldv[2];
  s->ioldv[2] = s->ioldv[1];
  s->ioldv[1] = s->ioldv[0];
  s->ioldv[0] = t;
}
#ifndef HE_KERNEL_TU
static __global__ void k_imp_correct(ImpDev* g, double dt) {
  __shared__ ImpDev st;
  imp_stage_in(&st, g);
  if (threadIdx.x == 0) imp_correct_body(&st, dt);
  imp_stage_out(g, &st);
}
#endif

// ---- statics (real psi) ------------------------------------------------------------------------
// hpsi = -(d2x+d2y+d2z)*h2o2m4 + pot4*psi; acc = sum psi*hpsi  (steppcr.f90:40-42).
// TT = float: the mixed path (binary32 hi plane of psi, binary32 pot4 and H psi; the sum in
// binary64).
template <typename TT>
struct OpHpsiRT {
  static const char* kname() { return sizeof(TT) == 4 ? "statics_hpsi_f32" : "statics_hpsi"; }
  using T = TT;
  static constexpr int NV = 1, N8 = 1, N16 = 0;
  const TT* s8[N8];          // pot4
  const typename RealOf<TT>::Z* s16[1];
  TT* out;
  TT h2o2m;
  HE_D void remap(const MemberMap& mm, int m) {
    s8[0] = mm(s8[0], m);
    out = mm(out, m);
  }
  HE_D void at(int, int, int, long i, TT dx, TT dy, TT dz, TT c, const TT* v8,
               const typename RealOf<TT>::Z*, int, double* acc) const {
    const TT h = -((dx + dy) + dz) * h2o2m + v8[0] * c;
    out[i] = h;
    acc[0] += (double)c * (double)h;
  }
};
using OpHpsiR = OpHpsiRT<double>;

}  // namespace he
