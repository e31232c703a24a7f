// setup.cuh -- device evaluation of the k-space kernels (run once per context).
//
// fvlj4: Fourier transform of the cored Lennard-Jones potential, Dynamics_TDDFT/fforma.f90:11-61
//        with sinx11 (:73-102), sinx5 (:108-137), sinint (:143-196), intcore (:221-245) and
//        bforce (:256-280) for p = 0.
// wcgk:  coarse-graining kernel 3(sin x - x cos x)/x^3, x = 2 pi p h (initcg.f90:32-49).
// kalfs: exp(-(pi l p)^2) (DFT4He3d.f90:527-531).
// The reference takes the sine integral from NAG's s13adf; here it is the Maclaurin series for
// |x| <= 4 and, above, Si(x) = pi/2 + Im E1(ix) with E1 from its continued fraction evaluated by
// the modified Lentz method (Abramowitz & Stegun 5.2.21-23, 5.1.22).
#pragma once
#include "common.cuh"

namespace he {

constexpr double kPi = 3.14159265358979323846;

HE_HD double freq_of(int i, int n, double h) {
  const double hp = 1.0 / (n * h), pmax = 1.0 / (2.0 * h);
  return (i <= n / 2) ? hp * i : -pmax + hp * (i + 1 - (n / 2 + 1));
}

HE_D double si_dev(double x) {
  const double ax = fabs(x);
  double res;
  if (ax <= 4.0) {
    const double x2 = ax * ax;
    double term = ax, sum = ax;
    for (int n = 1; n < 60; ++n) {
      term *= -x2 / ((2.0 * n) * (2.0 * n + 1.0));
      const double t = term / (2.0 * n + 1.0);
      sum += t;
      if (fabs(t) < 1e-18 * fabs(sum)) break;
    }
    res = sum;
  } else {
    const double tiny = 1e-300;
    double2 b = make_double2(1.0, ax);
    double2 c = make_double2(1.0 / tiny, 0.0);
    auto cdiv = [](double2 u, double2 v) {
      const double d = v.x * v.x + v.y * v.y;
      return make_double2((u.x * v.x + u.y * v.y) / d, (u.y * v.x - u.x * v.y) / d);
    };
    double2 d = cdiv(make_double2(1.0, 0.0), b);
    double2 h = d;
    for (int i = 2; i < 1000; ++i) {
      const double a = -(double)(i - 1) * (i - 1);
      b.x += 2.0;
      d = cdiv(make_double2(1.0, 0.0), make_double2(a * d.x + b.x, a * d.y + b.y));
      const double2 ac = cdiv(make_double2(a, 0.0), c);
      c = make_double2(b.x + ac.x, b.y + ac.y);
      const double2 del = cmul(c, d);
      h = cmul(h, del);
      if (fabs(del.x - 1.0) + fabs(del.y) < 1e-16) break;
    }
    h = cmul(h, make_double2(cos(ax), -sin(ax)));
    res = 0.5 * kPi + h.y;
  }
  return x < 0 ? -res : res;
}

HE_D double f_sinint(double a, double x) {
  const double r = si_dev(a * x);
  return (a > 0.0) ? 0.5 * kPi - r : 0.5 * kPi + r;
}
HE_D double f_sinx11(double a, double x) {
  const double y = a * x, y2 = y * y;
  const double d[5] = {1.0, y2, y2 * y2, y2 * y2 * y2, y2 * y2 * y2 * y2};
  const double b[5] = {40320.0, -720.0, 24.0, -2.0, 1.0};
  const double c[5] = {362880.0, -5040.0, 120.0, -6.0, 1.0};
  double bd = 0.0, cd = 0.0;
  for (int i = 0; i < 5; ++i) { bd += b[i] * d[i]; cd += c[i] * d[i]; }
  const double x9 = x * x * x * x * x * x * x * x * x;
  const double res1 = (a * bd * cos(y) + cd * sin(y) / x) / (3628800.0 * x9);
  const double a10 = a * a * a * a * a * a * a * a * a * a;
  return res1 - (a10 * f_sinint(a, x)) / 3628800.0;
}
HE_D double f_sinx5(double a, double x) {
  const double y = a * x, y2 = y * y;
  const double bd = -2.0 + y2, cd = -6.0 + y2;
  const double res1 = -(a * bd * cos(y) + cd * sin(y) / x) / (24.0 * x * x * x);
  return res1 + (a * a * a * a * f_sinint(a, x)) / 24.0;
}
HE_D double f_intcore(double a, double x) {
  const double y = a * x, y2 = y * y;
  const double d0 = x / (a * a * a * a * a), e0 = 1.0 / (a * a * a * a * a * a);
  const double bd = -120.0 * d0 + 20.0 * (d0 * y2) - (d0 * y2 * y2);
  const double ce = 120.0 * e0 - 60.0 * (e0 * y2) + 5.0 * (e0 * y2 * y2);
  return bd * cos(y) + ce * sin(y);
}
HE_HD double bforce_hd(int op_core, double eps, double sigma, double hc) {
  const double pi4 = 4.0 * kPi, eps4 = 4.0 * eps;
  const double sh = sigma / hc;
  const double xx = sh * sh * sh * sh * sh * sh;
  const double v0 = xx * (xx - 1.0) / (hc * hc * hc * hc);
  const double s6 = sigma * sigma * sigma * sigma * sigma * sigma, s12 = s6 * s6;
  const double hc3 = hc * hc * hc, hc9 = hc3 * hc3 * hc3;
  const double bb2 = pi4 * eps4 * s12 / (9.0 * hc9);
  const double bb3 = -pi4 * eps4 * s6 / (3.0 * hc3);
  if (op_core) return pi4 * eps4 * (v0 * hc3 * hc3 * hc) / 7.0 + bb2 + bb3;
  return bb2 + bb3;
}

struct KernArgs {
  int nx, ny, nz, nxh;
  double hx, hy, hz;
  int op_core, otc;
  double eps, sigma, hc, l;
  double* fvlj4;
  double* wcgk;
  double* kalfs;
};

#ifndef HE_KERNEL_TU
__global__ void k_kernels(const KernArgs a) {
  const long nk = (long)a.nxh * a.ny * a.nz;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nk;
       i += (long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % a.nxh);
    const long r = i / a.nxh;
    const int iy = (int)(r % a.ny), iz = (int)(r / a.ny);
    const double px = freq_of(ix, a.nx, a.hx), py = freq_of(iy, a.ny, a.hy),
                 pz = freq_of(iz, a.nz, a.hz);
    const double p = sqrt(px * px + py * py + pz * pz);
    const double twopi = 2.0 * kPi;
    // fforma
    double fv;
    if (fabs(p) < 1e-10) {
      fv = bforce_hd(a.op_core, a.eps, a.sigma, a.hc);
    } else {
      const double s3 = a.sigma * a.sigma * a.sigma, sigma6 = s3 * s3;
      const double hc3 = a.hc * a.hc * a.hc, hc6 = hc3 * hc3;
      const double aux1 = 8.0 * a.eps, aux3 = sigma6 / hc6;
      const double aux2 = twopi * p;
      const double t1 = f_sinx11(aux2, a.hc), t2 = f_sinx5(aux2, a.hc);
      if (a.op_core) {
        const double v0 = aux1 * aux3 * (aux3 - 1.0) / (a.hc * a.hc * a.hc * a.hc);
        fv = (aux1 * sigma6 * (sigma6 * t1 - t2) + v0 * f_intcore(aux2, a.hc)) / p;
      } else {
        fv = (aux1 * sigma6 * (sigma6 * t1 - t2)) / p;
      }
    }
    a.fvlj4[i] = fv;
    // initcg
    double w = 1.0;
    if (p > 0.0) {
      const double arg = twopi * p * a.hc;
      const double aux = sin(arg) - arg * cos(arg);
      w = (fabs(aux) < 1e-10) ? 1.0 : 3.0 * aux / (arg * arg * arg);
    }
    a.wcgk[i] = w;
    if (a.otc) {
      const double t = kPi * a.l * p;
      a.kalfs[i] = exp(-(t * t));
    }
  }
}
#endif

}  // namespace he
