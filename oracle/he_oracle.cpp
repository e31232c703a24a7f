// he_oracle.cpp -- CPU FP64 restatement of the BCN-4He-DFT mean-field and time-step path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU baseline.  Only
// tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and --impl reference) may load
// it.  The product path (he_dft_2024_b200/) never links, loads or calls it.
//
// Parity status: the reference is Fortran + FFTW/MKL and cannot be compiled in this image (no
// Fortran compiler, no FFTW).  This restatement is pinned to the reference's own known answers:
// the 13-point Bickley weights of Dynamics_TDDFT/blockds.f:615-708 (bit-exact), the
// b = bforce(OT, 10.22, 2.556, 2.190323) = -718.99 self-consistency of
// Dynamics_TDDFT/modules.f90:233 vs fforma.f90:256-280, and the bulk equation of state of
// He_statics/rhoasin0.f90 (mu(rho0)).  Full-step parity is otherwise UNPINNED by the reference
// (no reference run is possible here); the FFT and the field are cross-checked against an
// independent numpy restatement in tests/.
//
// Every function cites the reference file:line it restates.  Layout is Fortran column-major
// (x fastest), complex interleaved, half spectrum (nx/2+1, ny, nz).

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

typedef std::complex<double> cplx;

// ------------------------------------------------------------------------------------------------
// Parameters shared with the ctypes wrapper (oracle/oracle.py keeps the same field order).
// ------------------------------------------------------------------------------------------------
extern "C" {
typedef struct {
  int nx, ny, nz;
  double xmax, ymax, zmax;
  int npd, icon;             // 13 and 13 (zero padding), 8 (periodic) or 18 (antiperiodic)
  int core;                  // 0 'OT ', 1 'OP ', 2 'OTC'  (effective core after the Lsolid rule)
  double h4, eps4, sigma4;   // Lennard-Jones core radius, epsilon, sigma
  double cp4, cpp4, den4c, alphas, l, den0s, h2o2m4;
  int lsolid;
  double C, beta, den_m;     // solid penalty (He_statics/modules.f90:127-129)
  double lambdah, txmean, txsurf, tymean, tysurf, tzmean, tzsurf;  // absorbing mask
  int n_imp;                 // classical impurities (0 = none)
  int pot_kind;              // He-impurity pair potential: 0 null, 1 Morse
  double pot_D, pot_re, pot_a, pot_rcut, pot_umax;
  int ii_kind;               // impurity-impurity potential: 0 null, 1 Morse
  double ii_D, ii_re, ii_a, ii_rcut, ii_umax;
  double dtmin, sdmu, dmumax;  // statics local time step (He_statics/modules.f90:299)
  int nthreads;
} ho_params;
}

static const double kPi = 4.0 * std::atan(1.0);  // pi = 4*datan(1) as in the reference

// ------------------------------------------------------------------------------------------------
// 13-point Bickley weights, centred rows.  Restates newder.f:99-130 (ICON=1 fetch of the table
// in mates.f BLOCK DATA) for M=13, K=1,2; the values are the exact Lagrange-derivative rationals,
// each a single correctly-rounded division, and are checked bit-for-bit against the table text
// (blockds.f:615-708) by tests/test_oracle_golden.py.
// ------------------------------------------------------------------------------------------------
static void bickley13(double w1[13], double w2[13]) {
  const double f6sq = 518400.0;  // (6!)^2
  const double fact[13] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880, 3628800, 39916800,
                           479001600};
  for (int j = 0; j < 13; ++j) { w1[j] = 0.0; w2[j] = 0.0; }
  for (int j = 1; j <= 6; ++j) {
    double den1 = (double)j * fact[6 - j] * fact[6 + j];
    double den2 = (double)j * (double)j * fact[6 - j] * fact[6 + j];
    double s = (j % 2 == 1) ? 1.0 : -1.0;
    w1[6 + j] = s * (f6sq / den1);
    w1[6 - j] = -w1[6 + j];
    w2[6 + j] = s * ((2.0 * f6sq) / den2);
    w2[6 - j] = w2[6 + j];
  }
  w2[6] = -5369.0 / 1800.0;  // -2 * sum_{j=1..6} 1/j^2
}

// ------------------------------------------------------------------------------------------------
// Grid and k-grid: Dynamics_TDDFT/DFT4He3d.f90:265-278 (steps), :321-329 (x_i = -xmax + h(i-1)),
// :340-373 (FFTW-ordered frequencies and pmod over the half spectrum).
// ------------------------------------------------------------------------------------------------
struct Grid {
  int nx, ny, nz, nxh;
  double xmax, ymax, zmax, hx, hy, hz, dxyz;
  long nxyz, nk;
  std::vector<double> x, y, z, px, py, pz, pmod;
  void init(const ho_params& p) {
    nx = p.nx; ny = p.ny; nz = p.nz; nxh = nx / 2 + 1;
    xmax = p.xmax; ymax = p.ymax; zmax = p.zmax;
    hx = 2.0 * std::fabs(xmax) / nx;
    hy = 2.0 * std::fabs(ymax) / ny;
    hz = 2.0 * std::fabs(zmax) / nz;
    dxyz = hx * hy * hz;
    nxyz = (long)nx * ny * nz;
    nk = (long)nxh * ny * nz;
    x.resize(nx); y.resize(ny); z.resize(nz);
    for (int i = 0; i < nx; ++i) x[i] = -xmax + hx * i;
    for (int i = 0; i < ny; ++i) y[i] = -ymax + hy * i;
    for (int i = 0; i < nz; ++i) z[i] = -zmax + hz * i;
    auto freq = [](int n, double h, std::vector<double>& p) {
      double hp = 1.0 / (n * h), pmax = 1.0 / (2.0 * h);
      p.resize(n);
      for (int i = 1; i <= n / 2 + 1; ++i) p[i - 1] = hp * (i - 1);
      for (int i = n / 2 + 2; i <= n; ++i) p[i - 1] = -pmax + hp * (i - (n / 2 + 1));
    };
    freq(nx, hx, px); freq(ny, hy, py); freq(nz, hz, pz);
    pmod.resize(nk);
    for (int k = 0; k < nz; ++k) {
      double pz2 = pz[k] * pz[k];
      for (int j = 0; j < ny; ++j) {
        double py2 = py[j] * py[j];
        for (int i = 0; i < nxh; ++i) {
          double px2 = px[i] * px[i];
          pmod[i + (long)nxh * (j + (long)ny * k)] = std::sqrt(px2 + py2 + pz2);
        }
      }
    }
  }
};

// ------------------------------------------------------------------------------------------------
// FFT.  The reference calls threaded FFTW (fft.f90:50-75): unnormalised R2C forward, C2R backward
// scaled by renor = 1/(nx*ny*nz) (fft.f90:36,118-168).  This is an independent mixed-radix
// (2,3,4,5) Stockham restatement; twiddles from long-double sin/cos.
// ------------------------------------------------------------------------------------------------
struct FFT1 {
  int n = 0;
  std::vector<int> rad;
  std::vector<cplx> tw;  // exp(-2 pi i m / n)
  void init(int n_) {
    n = n_;
    rad.clear();
    int m = n;
    while (m % 4 == 0) { rad.push_back(4); m /= 4; }
    while (m % 2 == 0) { rad.push_back(2); m /= 2; }
    while (m % 3 == 0) { rad.push_back(3); m /= 3; }
    while (m % 5 == 0) { rad.push_back(5); m /= 5; }
    if (m != 1) { fprintf(stderr, "oracle FFT: unsupported length %d\n", n); rad.clear(); }
    tw.resize(n);
    for (int k = 0; k < n; ++k) {
      long double a = -2.0L * 3.14159265358979323846264338327950288L * k / n;
      tw[k] = cplx((double)cosl(a), (double)sinl(a));
    }
  }
  // sign = -1 forward, +1 backward; a and b are length-n work lines; result ends in a.
  void exec(cplx* a, cplx* b, int sign) const {
    int ns = 1;
    cplx* src = a; cplx* dst = b;
    for (size_t s = 0; s < rad.size(); ++s) {
      int R = rad[s];
      int nr = n / R;
      for (int j = 0; j < nr; ++j) {
        int k = j % ns;
        cplx v[5];
        for (int r = 0; r < R; ++r) {
          long m = ((long)r * k * (n / (ns * R))) % n;
          cplx w = tw[m];
          if (sign > 0) w = std::conj(w);
          v[r] = src[j + r * nr] * w;
        }
        cplx o[5];
        for (int q = 0; q < R; ++q) {
          cplx acc = 0.0;
          for (int r = 0; r < R; ++r) {
            long m = ((long)r * q * (n / R)) % n;
            cplx w = tw[m];
            if (sign > 0) w = std::conj(w);
            acc += v[r] * w;
          }
          o[q] = acc;
        }
        int base = (j / ns) * ns * R + k;
        for (int r = 0; r < R; ++r) dst[base + r * ns] = o[r];
      }
      ns *= R;
      std::swap(src, dst);
    }
    if (src != a) std::memcpy(a, src, sizeof(cplx) * n);
  }
};

struct FFT3 {
  const Grid* g = nullptr;
  FFT1 fx, fy, fz;
  void init(const Grid& gr) { g = &gr; fx.init(g->nx); fy.init(g->ny); fz.init(g->nz); }
  // Complex transforms along y and z of a half-spectrum array, batched over kx.
  void yz(cplx* c, int sign) const {
    const int nxh = g->nxh, ny = g->ny, nz = g->nz;
#pragma omp parallel
    {
      std::vector<cplx> a(std::max(ny, nz)), b(std::max(ny, nz));
#pragma omp for collapse(2) schedule(static)
      for (int k = 0; k < nz; ++k)
        for (int i = 0; i < nxh; ++i) {
          for (int j = 0; j < ny; ++j) a[j] = c[i + (long)nxh * (j + (long)ny * k)];
          fy.exec(a.data(), b.data(), sign);
          for (int j = 0; j < ny; ++j) c[i + (long)nxh * (j + (long)ny * k)] = a[j];
        }
#pragma omp for collapse(2) schedule(static)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nxh; ++i) {
          for (int k = 0; k < nz; ++k) a[k] = c[i + (long)nxh * (j + (long)ny * k)];
          fz.exec(a.data(), b.data(), sign);
          for (int k = 0; k < nz; ++k) c[i + (long)nxh * (j + (long)ny * k)] = a[k];
        }
    }
  }
  // out = R2C(in), unnormalised (FFTW dfftw_plan_dft_r2c_3d semantics).
  void r2c(const double* in, cplx* out) const {
    const int nx = g->nx, nxh = g->nxh, ny = g->ny, nz = g->nz;
#pragma omp parallel
    {
      std::vector<cplx> a(nx), b(nx);
#pragma omp for collapse(2) schedule(static)
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
          const double* row = in + (long)nx * (j + (long)ny * k);
          for (int i = 0; i < nx; ++i) a[i] = cplx(row[i], 0.0);
          fx.exec(a.data(), b.data(), -1);
          cplx* orow = out + (long)nxh * (j + (long)ny * k);
          for (int i = 0; i < nxh; ++i) orow[i] = a[i];
        }
    }
    yz(out, -1);
  }
  // out = C2R(in) * renor; 'in' is destroyed (FFTW c2r also destroys its input).
  void c2r(cplx* in, double* out, double renor) const {
    const int nx = g->nx, nxh = g->nxh, ny = g->ny, nz = g->nz;
    yz(in, +1);
#pragma omp parallel
    {
      std::vector<cplx> a(nx), b(nx);
#pragma omp for collapse(2) schedule(static)
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
          const cplx* irow = in + (long)nxh * (j + (long)ny * k);
          for (int i = 0; i < nxh; ++i) a[i] = irow[i];
          for (int i = nxh; i < nx; ++i) a[i] = std::conj(irow[nx - i]);
          fx.exec(a.data(), b.data(), +1);
          double* row = out + (long)nx * (j + (long)ny * k);
          for (int i = 0; i < nx; ++i) row[i] = a[i].real() * renor;
        }
    }
  }
};

// ------------------------------------------------------------------------------------------------
// Sine integral.  The reference calls NAG's s13adf (s13adf.f90); this is an independent
// evaluation: the Maclaurin series for |x| <= 4 and, above, the continued fraction for the
// exponential integral E1(ix) evaluated by the modified Lentz method, Si(x) = pi/2 + Im E1(ix)
// (Abramowitz & Stegun 5.2.21-23, 5.1.22).
// ------------------------------------------------------------------------------------------------
static double sine_integral(double x) {
  double ax = std::fabs(x);
  double res;
  if (ax <= 4.0) {
    double x2 = ax * ax, term = ax, sum = ax;
    for (int n = 1; n < 60; ++n) {
      term *= -x2 / ((2.0 * n) * (2.0 * n + 1.0));
      double t = term / (2.0 * n + 1.0);
      sum += t;
      if (std::fabs(t) < 1e-18 * std::fabs(sum)) break;
    }
    res = sum;
  } else {
    const double tiny = 1e-300;
    cplx b(1.0, ax), c(1.0 / tiny, 0.0), d = 1.0 / b, h = d;
    for (int i = 2; i < 1000; ++i) {
      double a = -(double)(i - 1) * (i - 1);
      b += 2.0;
      d = 1.0 / (a * d + b);
      c = b + a / c;
      cplx del = c * d;
      h *= del;
      if (std::fabs(del.real() - 1.0) + std::fabs(del.imag()) < 1e-16) break;
    }
    h *= cplx(std::cos(ax), -std::sin(ax));
    res = 0.5 * kPi + h.imag();
  }
  return x < 0 ? -res : res;
}

// Fourier transform of the cored Lennard-Jones kernel: Dynamics_TDDFT/fforma.f90:11-61 with the
// internal functions sinx11 (:73-102), sinx5 (:108-137), sinint (:143-196), intcore (:221-245)
// and bforce (:256-280).  'core' is the 2-character core passed by the driver ('OT'/'OP').
static double f_sinint(double a, double x) {
  double y = a * x;
  double res = sine_integral(y);
  return (a > 0.0) ? 0.5 * kPi - res : 0.5 * kPi + res;
}
static double f_sinx11(double a, double x) {
  double y = a * x, y2 = y * y;
  double b[5] = {40320.0, -720.0, 24.0, -2.0, 1.0};
  double c[5] = {362880.0, -5040.0, 120.0, -6.0, 1.0};
  double d[5] = {1.0, y2, y2 * y2, y2 * y2 * y2, y2 * y2 * y2 * y2};
  double bd = 0, cd = 0;
  for (int i = 0; i < 5; ++i) { bd += b[i] * d[i]; cd += c[i] * d[i]; }
  double x9 = x * x * x * x * x * x * x * x * x;
  double res1 = (a * bd * std::cos(y) + cd * std::sin(y) / x) / (3628800.0 * x9);
  double a10 = a * a * a * a * a * a * a * a * a * a;
  double res2 = -(a10 * f_sinint(a, x)) / 3628800.0;
  return res1 + res2;
}
static double f_sinx5(double a, double x) {
  double y = a * x, y2 = y * y;
  double bd = -2.0 * 1.0 + 1.0 * y2, cd = -6.0 * 1.0 + 1.0 * y2;
  double res1 = -(a * bd * std::cos(y) + cd * std::sin(y) / x) / (24.0 * x * x * x);
  double res2 = (a * a * a * a * f_sinint(a, x)) / 24.0;
  return res1 + res2;
}
static double f_intcore(double a, double x) {
  double y = a * x, y2 = y * y;
  double b[3] = {-120.0, 20.0, -1.0}, c[3] = {120.0, -60.0, 5.0};
  double d[3], e[3];
  d[0] = x / (a * a * a * a * a); e[0] = 1.0 / (a * a * a * a * a * a);
  d[1] = d[0] * y2; e[1] = e[0] * y2;
  d[2] = d[1] * y2; e[2] = e[1] * y2;
  double bd = 0, ce = 0;
  for (int i = 0; i < 3; ++i) { bd += b[i] * d[i]; ce += c[i] * e[i]; }
  return bd * std::cos(y) + ce * std::sin(y);
}
extern "C" double ho_bforce(int op_core, double eps, double sigma, double hc) {
  double pi4 = 4.0 * kPi, eps4 = 4.0 * eps;
  double xx = std::pow(sigma / hc, 6);
  double v0 = xx * (xx - 1.0) / (hc * hc * hc * hc);
  double s6 = std::pow(sigma, 6), s12 = s6 * s6;
  double bb2 = pi4 * eps4 * s12 / (9.0 * std::pow(hc, 9));
  double bb3 = -pi4 * eps4 * s6 / (3.0 * hc * hc * hc);
  if (op_core) {
    double bb1 = pi4 * eps4 * (v0 * std::pow(hc, 7)) / 7.0;
    return bb1 + bb2 + bb3;
  }
  return bb2 + bb3;
}
static void fforma(int op_core, double eps, double sigma, double hc, const Grid& g,
                   std::vector<double>& fvlj) {
  double sigma6 = std::pow(sigma, 6), aux1 = 8.0 * eps, aux3 = sigma6 / std::pow(hc, 6);
  double twopi = 2.0 * kPi;
  fvlj.resize(g.nk);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < g.nk; ++i) {
    double p = g.pmod[i];
    if (std::fabs(p) < 1e-10) {
      fvlj[i] = ho_bforce(op_core, eps, sigma, hc);
    } else {
      double aux2 = twopi * p;
      double t1 = f_sinx11(aux2, hc), t2 = f_sinx5(aux2, hc);
      if (op_core) {
        double v0 = aux1 * aux3 * (aux3 - 1.0) / (hc * hc * hc * hc);
        double t3 = f_intcore(aux2, hc);
        fvlj[i] = (aux1 * sigma6 * (sigma6 * t1 - t2) + v0 * t3) / p;
      } else {
        fvlj[i] = (aux1 * sigma6 * (sigma6 * t1 - t2)) / p;
      }
    }
  }
}
// Coarse-graining kernel: Dynamics_TDDFT/initcg.f90:32-49.
static void initcg(double h, const Grid& g, std::vector<double>& wcgk) {
  double twopi = 2.0 * kPi;
  wcgk.resize(g.nk);
  for (long i = 0; i < g.nk; ++i) {
    double p = g.pmod[i];
    if (p > 0.0) {
      double arg = twopi * p * h;
      double aux = std::sin(arg) - arg * std::cos(arg);
      wcgk[i] = (std::fabs(aux) < 1e-10) ? 1.0 : 3.0 * aux / (arg * arg * arg);
    } else {
      wcgk[i] = 1.0;
    }
  }
}

// Pair potentials behind the Select_Pot(selec,r,r_cutoff,umax) contract
// (Dynamics_TDDFT/V_impur.f90:90-2152: r < r_cutoff gives umax).  'null' and the Morse form
// V(r) = D[(1 - exp(-a(r-re)))^2 - 1] are restated; the Morse entry has no reference counterpart.
static double select_pot(int kind, double D, double re, double a, double rcut, double umax,
                         double r) {
  if (kind == 0) return (r < rcut) ? umax : 0.0;
  if (r < rcut) return umax;
  double e = 1.0 - std::exp(-a * (r - re));
  return D * (e * e - 1.0);
}
// dV/dr of the Morse form (the 'drselec' derivative entry used by forceimp).
static double select_dpot(int kind, double D, double re, double a, double rcut, double r) {
  if (kind == 0 || r < rcut) return 0.0;
  double ex = std::exp(-a * (r - re));
  return 2.0 * D * a * (1.0 - ex) * ex;
}

// ------------------------------------------------------------------------------------------------
// Finite differences: Deriv3D_p / Deriv3D_pc (init_deriv_parallel.f90:373-648, :933-1209) with
// the Redef boundary rows.  icon=13 (redef.f:151-170 then :133-150) makes every boundary row the
// centred row shifted with zero fill, i.e. a centred stencil with zero padding; icon=8/18 wrap
// periodically / antiperiodically (init_deriv_parallel.f90:1094-1206); icon=24 (redef.f:245-279,
// then ICON=4 at :18-56) folds the centred row into an even reflection about the end points.  Axes shorter than npd
// return zero (init_deriv_parallel.f90:949-953).  Weights are scaled by Sto = 1/h**id.
// ------------------------------------------------------------------------------------------------
template <typename T>
static void deriv3d(int id, const Grid& g, int axis, int icon, const double w1[13],
                    const double w2[13], const T* f, T* df) {
  const int n1 = g.nx, n2 = g.ny, n3 = g.nz;
  const int nn[3] = {n1, n2, n3};
  const double h = (axis == 0) ? g.hx : (axis == 1) ? g.hy : g.hz;
  const double sto = (id == 1) ? 1.0 / h : 1.0 / (h * h);
  double cd[13];
  for (int j = 0; j < 13; ++j) cd[j] = ((id == 1) ? w1[j] : w2[j]) * sto;
  const long N = g.nxyz;
  if (nn[axis] < 13) {
    for (long i = 0; i < N; ++i) df[i] = T(0);
    return;
  }
  const long stride = (axis == 0) ? 1 : (axis == 1) ? n1 : (long)n1 * n2;
  const int n = nn[axis];
  const double sgn = (icon == 18) ? -1.0 : 1.0;
  const bool wrap = (icon == 8 || icon == 18);
  const bool mirror = (icon == 24);  // redef.f:245-279 + ICON=4: even reflection about the ends
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < n3; ++k)
    for (int j = 0; j < n2; ++j)
      for (int i = 0; i < n1; ++i) {
        long p = i + (long)n1 * (j + (long)n2 * k);
        int c = (axis == 0) ? i : (axis == 1) ? j : k;
        long base = p - (long)c * stride;
        T acc = T(0);
        for (int m = 0; m < 13; ++m) {
          int q = c + m - 6;
          if (q >= 0 && q < n) {
            acc += cd[m] * f[base + q * stride];
          } else if (wrap) {
            int qq = (q < 0) ? q + n : q - n;
            acc += (sgn * cd[m]) * f[base + qq * stride];
          } else if (mirror) {
            int qq = (q < 0) ? -q : 2 * (n - 1) - q;
            acc += cd[m] * f[base + qq * stride];
          }
        }
        df[p] = acc;
      }
}

// ------------------------------------------------------------------------------------------------
// Common state (module variables of Dynamics_TDDFT/modules.f90:21-399 and He_statics/modules.f90).
// ------------------------------------------------------------------------------------------------
struct Common {
  ho_params p;
  Grid g;
  FFT3 fft;
  double w1[13], w2[13];
  double renor;
  std::vector<double> fvlj4, wcgk, kalfs;
  std::vector<double> den, dencg, delj4, pot4, sto1, penalty, dxden, dyden, dzden;
  std::vector<cplx> fden, wk1;
  // alpha_s term (core4 = 'OTC'; alphasterm module)
  std::vector<double> denalf, falfs, intxalf, intyalf, intzalf, ualphas, a1, a2, a3, a4, a5, a6;

  void init_common(const ho_params& pp) {
    p = pp;
    if (p.nthreads > 0) omp_set_num_threads(p.nthreads);
    g.init(p);
    fft.init(g);
    bickley13(w1, w2);
    renor = 1.0 / ((double)((long)g.nx * g.ny * g.nz));
    fforma(p.core == 1, p.eps4, p.sigma4, p.h4, g, fvlj4);
    initcg(p.h4, g, wcgk);
    if (p.core == 2) {
      kalfs.resize(g.nk);
      for (long i = 0; i < g.nk; ++i) {
        double t = kPi * p.l * g.pmod[i];
        kalfs[i] = std::exp(-(t * t));
      }
    }
    long N = g.nxyz;
    den.assign(N, 0); dencg.assign(N, 0); delj4.assign(N, 0); pot4.assign(N, 0);
    sto1.assign(N, 0); penalty.assign(N, 0);
    dxden.assign(N, 0); dyden.assign(N, 0); dzden.assign(N, 0);
    fden.assign(g.nk, 0); wk1.assign(g.nk, 0);
    if (p.core == 2)
      for (auto* v : {&denalf, &falfs, &intxalf, &intyalf, &intzalf, &ualphas, &a1, &a2, &a3, &a4,
                      &a5, &a6})
        v->assign(N, 0);
  }
  bool otc() const { return p.core == 2; }
  // g = C2R(R2C(f) * kalfs) * renor
  void conv_kalfs(const std::vector<double>& f, std::vector<double>& out) {
    fft.r2c(f.data(), wk1.data());
    for (long i = 0; i < g.nk; ++i) wk1[i] = kalfs[i] * wk1[i];
    fft.c2r(wk1.data(), out.data(), renor);
  }
  // denalf = C2R(fden*kalfs) (Dynamics_TDDFT/poten.f90:200-205; BCN4HeDFT.f90:1142-1148).
  void alfa_density() {
    for (long i = 0; i < g.nk; ++i) wk1[i] = fden[i] * kalfs[i];
    fft.c2r(wk1.data(), denalf.data(), renor);
  }
  // term_alfa: Dynamics_TDDFT/term_alfa.f90:5-117 (He_statics/term_alfa.f90 is the same
  // arithmetic).  Needs denalf and dxden/dyden/dzden.
  void term_alfa() {
    const long N = g.nxyz;
    const double d0 = p.den0s;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; ++i) {
      falfs[i] = 1.0 - denalf[i] / d0;
      a1[i] = falfs[i] * dxden[i];
      a2[i] = falfs[i] * dyden[i];
      a3[i] = falfs[i] * dzden[i];
    }
    conv_kalfs(a1, intxalf);
    conv_kalfs(a2, intyalf);
    conv_kalfs(a3, intzalf);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; ++i) a1[i] = dxden[i] * intxalf[i] + dyden[i] * intyalf[i] + dzden[i] * intzalf[i];
    conv_kalfs(a1, ualphas);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; ++i) {
      ualphas[i] = ualphas[i] / d0;
      a1[i] = falfs[i] * intxalf[i];
      a2[i] = falfs[i] * intyalf[i];
      a3[i] = falfs[i] * intzalf[i];
    }
    deriv3d<double>(1, g, 0, p.icon, w1, w2, a1.data(), a4.data());
    deriv3d<double>(1, g, 1, p.icon, w1, w2, a2.data(), a5.data());
    deriv3d<double>(1, g, 2, p.icon, w1, w2, a3.data(), a6.data());
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; ++i) ualphas[i] = (ualphas[i] + a4[i] + a5[i] + a6[i]) * p.h2o2m4 * p.alphas;
  }
  // ealphas of energy() (Dynamics_TDDFT/energy.f90:131-135, He_statics/energy.f90:110-114).
  double ealphas() const {
    if (!otc()) return 0.0;
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < g.nxyz; ++i)
      s += falfs[i] * (dxden[i] * intxalf[i] + dyden[i] * intyalf[i] + dzden[i] * intzalf[i]);
    return -p.h2o2m4 * 0.5 * p.alphas * s * g.dxyz;
  }
  // derden: Dynamics_TDDFT/derden.f90:26-28.
  void derden() {
    deriv3d<double>(1, g, 0, p.icon, w1, w2, den.data(), dxden.data());
    deriv3d<double>(1, g, 1, p.icon, w1, w2, den.data(), dyden.data());
    deriv3d<double>(1, g, 2, p.icon, w1, w2, den.data(), dzden.data());
  }
  // fftfw_den: fden = R2C(den) (fft.f90:96-100).
  void fftfw_den() { fft.r2c(den.data(), fden.data()); }
  // dencg = C2R(fden*wcgk)*renor (poten.f90:138-142).
  void coarse_grain() {
    for (long i = 0; i < g.nk; ++i) wk1[i] = fden[i] * wcgk[i];
    fft.c2r(wk1.data(), dencg.data(), renor);
  }
  // delj4 = C2R(fden*fvlj4)*renor (poten.f90:150-154).
  void lennard_jones() {
    for (long i = 0; i < g.nk; ++i) wk1[i] = fden[i] * fvlj4[i];
    fft.c2r(wk1.data(), delj4.data(), renor);
  }
  // Correlation convolution, penalty and pot4 assembly (poten.f90:160-198, :214-218).
  // extra (optional): potx4 of the quantum-impurity path, added after the correlation term
  // (Dynamics_quantum_impurities/poten.f90:116-121).
  // extra2 (optional): ualphas of the alpha_s term, added before the solid penalty
  // (poten.f90:200-210).
  void correlation_and_assembly(const double* extra = nullptr, const double* extra2 = nullptr) {
    const long N = g.nxyz;
    const double cp4 = p.cp4, cpp4 = p.cpp4;
    const double a0 = cp4 / 2.0, a1 = cpp4 / 3.0;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; ++i) sto1[i] = den[i] * dencg[i] * (cp4 + cpp4 * dencg[i]);
    fft.r2c(sto1.data(), wk1.data());
    for (long i = 0; i < g.nk; ++i) wk1[i] = wk1[i] * wcgk[i];
    fft.c2r(wk1.data(), sto1.data(), renor);
    if (p.lsolid) {
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) {
        double t = std::tanh(p.beta * (den[i] - p.den_m));
        penalty[i] = p.C * (1.0 + t + p.beta * den[i] * (1.0 - t * t));
      }
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; ++i) {
      double dc = dencg[i];
      pot4[i] = delj4[i] + dc * dc * (a0 + a1 * dc) + sto1[i];
      if (extra) pot4[i] = pot4[i] + extra[i];
      if (extra2) pot4[i] = pot4[i] + extra2[i];
    }
    if (p.lsolid) {
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) pot4[i] = pot4[i] + penalty[i];
    }
  }
  // Sum of the He energy densities shared by the three energy() variants
  // (Dynamics_TDDFT/energy.f90:111-155, He_statics/energy.f90:36-110).
  void he_energy_sums(double ekin_sum, double* ekin4, double* elj4, double* ecor4,
                      double* esolid) const {
    const long N = g.nxyz;
    double aux1 = 0.5 * p.cp4, aux2 = (1.0 / 3.0) * p.cpp4;
    double sl = 0, sc = 0, ss = 0;
#pragma omp parallel for reduction(+ : sl, sc, ss) schedule(static)
    for (long i = 0; i < N; ++i) {
      double a3 = den[i], a4 = dencg[i];
      sc += a3 * a4 * a4 * (aux1 + aux2 * a4);
      sl += delj4[i] * a3;
      if (p.lsolid) ss += a3 * (1.0 + std::tanh(p.beta * (a3 - p.den_m)));
    }
    *esolid = p.lsolid ? p.C * ss * g.dxyz : 0.0;
    *ekin4 = p.h2o2m4 * ekin_sum * g.dxyz;
    *elj4 = 0.5 * sl * g.dxyz;
    *ecor4 = sc * g.dxyz;
  }
};

// ------------------------------------------------------------------------------------------------
// Droplet observables printed every pener steps (Dynamics_TDDFT/DFT4He3d.f90:720-838, r_cm.f90),
// with the reference's loops: out = {N, xcm, ycm, zcm, Lx, Ly, Lz, Vcomx, Vcomy, Vcomz, <x^2>,
// <y^2>, <z^2>}.
// ------------------------------------------------------------------------------------------------
static void observables(const Grid& g, const ho_params& p, const double w1[13], const double w2[13],
                        const std::vector<cplx>& psi, const std::vector<double>& den, int npart,
                        double* out) {
  const long N = g.nxyz;
  std::vector<cplx> s1(N), s2(N), s3(N);
  double auxn4 = 0;
  for (long i = 0; i < N; ++i) auxn4 += den[i];
  auxn4 = auxn4 * g.dxyz;
  double xcm = 0, ycm = 0, zcm = 0;  // r_cm.f90:38-52
  for (int iz = 0; iz < g.nz; ++iz)
    for (int iy = 0; iy < g.ny; ++iy)
      for (int ix = 0; ix < g.nx; ++ix) {
        const double a = den[ix + (long)g.nx * (iy + (long)g.ny * iz)];
        xcm = xcm + a * g.x[ix];
        ycm = ycm + a * g.y[iy];
        zcm = zcm + a * g.z[iz];
      }
  xcm = xcm * g.dxyz / npart;
  ycm = ycm * g.dxyz / npart;
  zcm = zcm * g.dxyz / npart;
  deriv3d<cplx>(1, g, 0, p.icon, w1, w2, psi.data(), s1.data());
  deriv3d<cplx>(1, g, 1, p.icon, w1, w2, psi.data(), s2.data());
  deriv3d<cplx>(1, g, 2, p.icon, w1, w2, psi.data(), s3.data());
  const cplx ci(0.0, 1.0);
  cplx lx = 0, ly = 0, lz = 0, vx = 0, vy = 0, vz = 0;
  double r2x = 0, r2y = 0, r2z = 0;
  for (int iz = 0; iz < g.nz; ++iz)
    for (int iy = 0; iy < g.ny; ++iy)
      for (int ix = 0; ix < g.nx; ++ix) {
        const long i = ix + (long)g.nx * (iy + (long)g.ny * iz);
        const cplx c = std::conj(psi[i]);
        const double X = g.x[ix] - xcm, Y = g.y[iy] - ycm, Z = g.z[iz] - zcm;
        lz = lz + ci * c * (Y * s1[i] - X * s2[i]);
        ly = ly + ci * c * (X * s3[i] - Z * s1[i]);
        lx = lx + ci * c * (Z * s2[i] - Y * s3[i]);
        vx = vx - ci * c * s1[i];
        vy = vy - ci * c * s2[i];
        vz = vz - ci * c * s3[i];
        r2x = r2x + den[i] * (g.x[ix] * g.x[ix]);
        r2y = r2y + den[i] * (g.y[iy] * g.y[iy]);
        r2z = r2z + den[i] * (g.z[iz] * g.z[iz]);
      }
  const double mhe = 4.002572164 * 0.02061484;  // DFT4He3d.f90:103, :315
  const double v[13] = {auxn4, xcm, ycm, zcm, (lx * g.dxyz).real(), (ly * g.dxyz).real(),
                        (lz * g.dxyz).real(), (vx * g.dxyz).real() / (auxn4 * mhe),
                        (vy * g.dxyz).real() / (auxn4 * mhe), (vz * g.dxyz).real() / (auxn4 * mhe),
                        r2x * g.dxyz, r2y * g.dxyz, r2z * g.dxyz};
  std::memcpy(out, v, sizeof(v));
}

// ------------------------------------------------------------------------------------------------
// Real-time TDDFT with classical impurities (Dynamics_TDDFT).
// ------------------------------------------------------------------------------------------------
struct Dyn : Common {
  std::vector<cplx> psi, pc, q, timec, s1, s2, s3, s4, s5;
  std::vector<cplx> psiold[3], hpsiold[2];
  std::vector<double> uimp, uimp_k;  // uimp_k is (N_imp, nx, ny, nz), impurity fastest
  int ioldp[3] = {1, 2, 3}, ioldh[2] = {1, 2};
  // Impurity state, Fortran (N_imp,3) column-major and (N_imp,3,slot).
  int ni = 0;
  std::vector<double> rimp, vimp, aimp, F, m_imp, qr, qv, pcr, pcv, stor;
  std::vector<double> rimpold, vimpold, aimpold;  // (N_imp,3,3), (N_imp,3,3), (N_imp,3,2)
  int ioldr[3] = {1, 2, 3}, ioldv[3] = {1, 2, 3}, iolda[2] = {1, 2};
  // Interpolation table of potenimpini (potenimpini.f90:31-59).
  int npot = 0;
  double delinter = 0, rmaxinterpol = 0;
  std::vector<double> potion;  // (N_imp, npot)
  bool lstopimp = false, lgridnoout = true;

  void init(const ho_params& pp, const double* m_imp_u) {
    init_common(pp);
    long N = g.nxyz;
    psi.assign(N, 0); pc.assign(N, 0); q.assign(N, 0); timec.assign(N, 0);
    s1.assign(N, 0); s2.assign(N, 0); s3.assign(N, 0); s4.assign(N, 0); s5.assign(N, 0);
    for (auto& v : psiold) v.assign(N, 0);
    for (auto& v : hpsiold) v.assign(N, 0);
    uimp.assign(N, 0);
    ni = p.n_imp;
    rimp.assign(3 * ni, 0); vimp.assign(3 * ni, 0); aimp.assign(3 * ni, 0); F.assign(3 * ni, 0);
    qr.assign(3 * ni, 0); qv.assign(3 * ni, 0); pcr.assign(3 * ni, 0); pcv.assign(3 * ni, 0);
    stor.assign(3 * ni, 0);
    rimpold.assign(9 * ni, 0); vimpold.assign(9 * ni, 0); aimpold.assign(6 * ni, 0);
    m_imp.assign(ni, 0);
    for (int k = 0; k < ni; ++k) m_imp[k] = m_imp_u[k] * 0.02061484;  // mp_u, modules.f90:324
    uimp_k.assign((long)ni * N, 0);
    // timec: DFT4He3d.f90:592-601
    for (int k = 0; k < g.nz; ++k)
      for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i) {
          double s = 1.0 + std::tanh((std::fabs(g.x[i]) - p.txmean) / p.txsurf);
          s = s + 1.0 + std::tanh((std::fabs(g.y[j]) - p.tymean) / p.tysurf);
          s = s + 1.0 + std::tanh((std::fabs(g.z[k]) - p.tzmean) / p.tzsurf);
          timec[i + (long)g.nx * (j + (long)g.ny * k)] = cplx(p.lambdah * s, 1.0);
        }
    if (ni > 0) {
      int nmax = std::max(g.nx, std::max(g.ny, g.nz));
      npot = 100 * nmax + 1;
      double rmax = 4.0 * std::max(g.xmax, std::max(g.ymax, g.zmax));
      rmaxinterpol = rmax;
      delinter = rmax / (double)(npot - 1);
      potion.assign((long)ni * npot, 0);
      for (int k = 0; k < ni; ++k)
        for (int i = 0; i < npot; ++i) {
          double r = (double)i * delinter;
          potion[k + (long)ni * i] =
              select_pot(p.pot_kind, p.pot_D, p.pot_re, p.pot_a, p.pot_rcut, p.pot_umax, r);
        }
    }
  }
  double& R(std::vector<double>& a, int k, int d) { return a[k + ni * d]; }
  double& RS(std::vector<double>& a, int k, int d, int slot) {
    return a[k + ni * d + 3 * ni * (slot - 1)];
  }

  // updatepoten: potenimp.f90:83-123 (potenimp() at :1-19 only calls it).
  void potenimp() {
    const long N = g.nxyz;
    for (int k = 0; k < ni; ++k) {
      double rx = R(rimp, k, 0), ry = R(rimp, k, 1), rz = R(rimp, k, 2);
      for (int iz = 0; iz < g.nz; ++iz) {
        double zt = (g.z[iz] - rz) * (g.z[iz] - rz);
        for (int iy = 0; iy < g.ny; ++iy) {
          double yt = (g.y[iy] - ry) * (g.y[iy] - ry) + zt;
          for (int ix = 0; ix < g.nx; ++ix) {
            double r = std::sqrt((g.x[ix] - rx) * (g.x[ix] - rx) + yt);
            // Off-table radius: the reference flags lstopimp once and clamps r, but takes the
            // table index before the clamp and reads past the table; here r is clamped on every
            // point and the index is taken after it, so the interpolation stays in the table.
            if (!(r <= rmaxinterpol)) {  // also a NaN radius
              if (lgridnoout) { lstopimp = true; lgridnoout = false; }
              r = rmaxinterpol;
            }
            int ir = (int)(r / delinter) + 1;
            if (ir > npot - 1) ir = npot - 1;
            double rmod = std::fmod(r, delinter) / delinter;
            long pidx = ix + (long)g.nx * (iy + (long)g.ny * iz);
            uimp_k[k + (long)ni * pidx] = potion[k + (long)ni * (ir - 1)] * (1.0 - rmod) +
                                          potion[k + (long)ni * ir] * rmod;
          }
        }
      }
    }
    for (long i = 0; i < N; ++i) uimp[i] = 0.0;
    for (int k = 0; k < ni; ++k)
      for (long i = 0; i < N; ++i) uimp[i] = uimp[i] + uimp_k[k + (long)ni * i];
  }
  // poten (dynamics, ldroplet_frozen=.false.): poten.f90:131-218.
  void poten() {
    fftfw_den();
    coarse_grain();
    derden();
    lennard_jones();
    if (otc()) {
      alfa_density();
      term_alfa();
    }
    correlation_and_assembly(nullptr, otc() ? ualphas.data() : nullptr);
  }
  // forceimp: potenimp.f90:23-67.
  void forceimp() {
    const long N = g.nxyz;
    std::vector<double> Fij((long)ni * ni * 3, 0.0);
    for (int k = 0; k < ni; ++k)
      for (int m = k + 1; m < ni; ++m) {
        double d[3];
        for (int c = 0; c < 3; ++c) d[c] = R(rimp, k, c) - R(rimp, m, c);
        double a1 = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double dv = select_dpot(p.ii_kind, p.ii_D, p.ii_re, p.ii_a, p.ii_rcut, a1);
        for (int c = 0; c < 3; ++c) {
          Fij[k + ni * (m + ni * c)] = -dv * d[c] / a1;
          Fij[m + ni * (k + ni * c)] = -Fij[k + ni * (m + ni * c)];
        }
      }
    for (int k = 0; k < ni; ++k) {
      double sx = 0, sy = 0, sz = 0;
#pragma omp parallel for reduction(+ : sx, sy, sz) schedule(static)
      for (long i = 0; i < N; ++i) {
        double u = uimp_k[k + (long)ni * i];
        sx += dxden[i] * u; sy += dyden[i] * u; sz += dzden[i] * u;
      }
      R(F, k, 0) = -sx * g.dxyz; R(F, k, 1) = -sy * g.dxyz; R(F, k, 2) = -sz * g.dxyz;
      for (int m = 0; m < ni; ++m)
        for (int c = 0; c < 3; ++c) R(F, k, c) = R(F, k, c) + Fij[k + ni * (m + ni * c)];
    }
  }
  void set_accel() {  // aimp = F/m_imp (DFT4He3d.f90:571-573, :694-696)
    for (int k = 0; k < ni; ++k)
      for (int c = 0; c < 3; ++c) R(aimp, k, c) = R(F, k, c) / m_imp[k];
  }
  void field() { potenimp(); poten(); forceimp(); }

  // H psi for the classical-impurity path (steprk.f90:67, steppc.f90:51,118) into s4.
  void hpsi(const std::vector<cplx>& f) {
    deriv3d<cplx>(2, g, 0, p.icon, w1, w2, f.data(), s1.data());
    deriv3d<cplx>(2, g, 1, p.icon, w1, w2, f.data(), s2.data());
    deriv3d<cplx>(2, g, 2, p.icon, w1, w2, f.data(), s3.data());
    const cplx ci(0.0, 1.0);
    const double h2 = p.h2o2m4;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < g.nxyz; ++i) {
      cplx lap = s1[i] + s2[i] + s3[i];
      s4[i] = timec[i] * (lap * h2 - pot4[i] * f[i]) - ci * uimp[i] * f[i];
    }
  }
  void density() {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < g.nxyz; ++i) den[i] = std::norm(psi[i]);
  }

  // steprk: Dynamics_TDDFT/steprk.f90:1-144 (RK-Gill, Ralston & Wilf).
  void steprk(double deltat) {
    double arun[4] = {0.5, 1.0 - 1.0 / std::sqrt(2.0), 1.0 + 1.0 / std::sqrt(2.0), 1.0 / 6.0};
    double brun[4] = {2.0, 1.0, 1.0, 2.0};
    double crun[4] = {0.5, 1.0 - 1.0 / std::sqrt(2.0), 1.0 + 1.0 / std::sqrt(2.0), 0.5};
    const long N = g.nxyz;
    for (int jr = 0; jr < 4; ++jr) {
      hpsi(psi);
      if (jr == 0) {
        hpsiold[1] = hpsiold[0];
        psiold[2] = psiold[1];
        psiold[1] = psiold[0];
        psiold[0] = psi;
      }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) {
        cplx sto1c = arun[jr] * (s4[i] - brun[jr] * q[i]);
        q[i] = q[i] + 3.0 * sto1c - crun[jr] * s4[i];
        psi[i] = psi[i] + deltat * sto1c;
      }
      if (jr == 0) hpsiold[0] = s4;
      density();
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) {
          R(stor, k, c) = arun[jr] * (R(vimp, k, c) - brun[jr] * R(qr, k, c));
          R(qr, k, c) = R(qr, k, c) + 3.0 * R(stor, k, c) - crun[jr] * R(vimp, k, c);
        }
      if (jr == 0)
        for (int k = 0; k < ni; ++k)
          for (int c = 0; c < 3; ++c) {
            RS(rimpold, k, c, 3) = RS(rimpold, k, c, 2);
            RS(rimpold, k, c, 2) = RS(rimpold, k, c, 1);
            RS(rimpold, k, c, 1) = R(rimp, k, c);
          }
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) R(rimp, k, c) = R(rimp, k, c) + deltat * R(stor, k, c);
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) {
          R(stor, k, c) = arun[jr] * (R(aimp, k, c) - brun[jr] * R(qv, k, c));
          R(qv, k, c) = R(qv, k, c) + 3.0 * R(stor, k, c) - crun[jr] * R(aimp, k, c);
        }
      if (jr == 0)
        for (int k = 0; k < ni; ++k)
          for (int c = 0; c < 3; ++c) {
            aimpold[k + ni * c + 3 * ni * 1] = aimpold[k + ni * c];
            aimpold[k + ni * c] = R(aimp, k, c);
            RS(vimpold, k, c, 3) = RS(vimpold, k, c, 2);
            RS(vimpold, k, c, 2) = RS(vimpold, k, c, 1);
            RS(vimpold, k, c, 1) = R(vimp, k, c);
          }
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) R(vimp, k, c) = R(vimp, k, c) + deltat * R(stor, k, c);
      if (jr <= 2) field();
    }
    for (int i = 0; i < 3; ++i) { ioldp[i] = i + 1; ioldr[i] = i + 1; ioldv[i] = i + 1; }
    for (int i = 0; i < 2; ++i) { ioldh[i] = i + 1; iolda[i] = i + 1; }
  }

  // steppc: Dynamics_TDDFT/steppc.f90:1-180 (Hamming predictor-modifier-corrector).
  void steppc(double deltat, double* errHe, double* errimp, double* errvimp) {
    const double c112 = 112.0 / 121.0, c9 = 9.0 / 121.0, c4o3 = 4.0 / 3.0;
    const long N = g.nxyz;
    hpsi(psi);
    {
      std::vector<cplx>& po3 = psiold[ioldp[2] - 1];
      const std::vector<cplx>& h1 = hpsiold[ioldh[0] - 1];
      std::vector<cplx>& h2 = hpsiold[ioldh[1] - 1];
      const double s = c4o3 * deltat;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) {
        cplx sto1c = po3[i] + s * (2.0 * s4[i] - h1[i] + 2.0 * h2[i]);
        po3[i] = psi[i];
        psi[i] = sto1c - c112 * pc[i];
        pc[i] = sto1c;
        h2[i] = s4[i];
      }
      density();
      std::swap(ioldh[0], ioldh[1]);
    }
    if (ni > 0) {
      const double s = c4o3 * deltat;
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) {
          R(stor, k, c) = RS(rimpold, k, c, ioldr[2]) +
                          s * (2.0 * R(vimp, k, c) - RS(vimpold, k, c, ioldv[0]) +
                               2.0 * RS(vimpold, k, c, ioldv[1]));
          RS(rimpold, k, c, ioldr[2]) = R(rimp, k, c);
          R(rimp, k, c) = R(stor, k, c) - c112 * R(pcr, k, c);
          R(pcr, k, c) = R(stor, k, c);
        }
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) {
          R(stor, k, c) = RS(vimpold, k, c, ioldv[2]) +
                          s * (2.0 * R(aimp, k, c) - aimpold[k + ni * c + 3 * ni * (iolda[0] - 1)] +
                               2.0 * aimpold[k + ni * c + 3 * ni * (iolda[1] - 1)]);
          RS(vimpold, k, c, ioldv[2]) = R(stor, k, c) - c112 * R(pcv, k, c);
          R(pcv, k, c) = R(stor, k, c);
        }
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) aimpold[k + ni * c + 3 * ni * (iolda[1] - 1)] = R(aimp, k, c);
      std::swap(iolda[0], iolda[1]);
    }
    field();
    hpsi(psi);
    double sabs = 0.0;
    {
      const std::vector<cplx>& po3 = psiold[ioldp[2] - 1];
      const std::vector<cplx>& po2 = psiold[ioldp[1] - 1];
      const std::vector<cplx>& h1 = hpsiold[ioldh[0] - 1];
      const std::vector<cplx>& h2 = hpsiold[ioldh[1] - 1];
      const double s3 = 3.0 * deltat;
#pragma omp parallel for reduction(+ : sabs) schedule(static)
      for (long i = 0; i < N; ++i) {
        cplx sto5c = 0.125 * (9.0 * po3[i] - po2[i] + s3 * (s4[i] + 2.0 * h1[i] - h2[i]));
        pc[i] = pc[i] - sto5c;
        psi[i] = sto5c + c9 * pc[i];
        sabs += std::abs(pc[i]);
      }
      density();
      if (errHe) *errHe = c9 * sabs / (double)N;
      int a = ioldp[2];
      ioldp[2] = ioldp[1]; ioldp[1] = ioldp[0]; ioldp[0] = a;
    }
    double er = 0, ev = 0;
    if (ni > 0) {
      const double s3 = 3.0 * deltat;
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) {
          R(stor, k, c) = 0.125 * (9.0 * RS(rimpold, k, c, ioldr[2]) - RS(rimpold, k, c, ioldr[1]) +
                                   s3 * (RS(vimpold, k, c, ioldv[2]) + 2.0 * R(vimp, k, c) -
                                         RS(vimpold, k, c, ioldv[0])));
          R(pcr, k, c) = R(pcr, k, c) - R(stor, k, c);
          R(rimp, k, c) = R(stor, k, c) + c9 * R(pcr, k, c);
        }
      for (int i = 0; i < 3 * ni; ++i) er += std::fabs(c9 * pcr[i]);
      er = er * 0.3333333333 / ni;
      int a = ioldr[2];
      ioldr[2] = ioldr[1]; ioldr[1] = ioldr[0]; ioldr[0] = a;
      for (int k = 0; k < ni; ++k)
        for (int c = 0; c < 3; ++c) {
          R(stor, k, c) = 0.125 * (9.0 * R(vimp, k, c) - RS(vimpold, k, c, ioldv[1]) +
                                   s3 * (R(aimp, k, c) +
                                         2.0 * aimpold[k + ni * c + 3 * ni * (iolda[0] - 1)] -
                                         aimpold[k + ni * c + 3 * ni * (iolda[1] - 1)]));
          R(pcv, k, c) = R(pcv, k, c) - R(stor, k, c);
          RS(vimpold, k, c, ioldv[2]) = R(vimp, k, c);
          R(vimp, k, c) = R(stor, k, c) + c9 * R(pcv, k, c);
        }
      for (int i = 0; i < 3 * ni; ++i) ev += std::fabs(c9 * pcv[i]);
      ev = ev * 0.3333333333 / ni;
      a = ioldv[2];
      ioldv[2] = ioldv[1]; ioldv[1] = ioldv[0]; ioldv[0] = a;
    }
    if (errimp) *errimp = er;
    if (errvimp) *errvimp = ev;
  }

  // energy: Dynamics_TDDFT/energy.f90:107-178 (uext is never assigned in this program and is
  // taken as zero).  out = {etot4, ekin4, elj4, ecor4, esolid, ealphas, ekinx, eHeX, eimpu_impu,
  // eimpu, etot}.
  void energy(double* out) {
    deriv3d<cplx>(1, g, 0, p.icon, w1, w2, psi.data(), s1.data());
    deriv3d<cplx>(1, g, 1, p.icon, w1, w2, psi.data(), s2.data());
    deriv3d<cplx>(1, g, 2, p.icon, w1, w2, psi.data(), s3.data());
    double ek = 0;
#pragma omp parallel for reduction(+ : ek) schedule(static)
    for (long i = 0; i < g.nxyz; ++i) ek += std::norm(s1[i]) + std::norm(s2[i]) + std::norm(s3[i]);
    double ekin4, elj4, ecor4, esolid;
    he_energy_sums(ek, &ekin4, &elj4, &ecor4, &esolid);
    const double ea = ealphas();
    double etot4 = ekin4 + elj4 + ecor4 + esolid;
    if (otc()) etot4 = etot4 + ea;
    double ekinx = 0;
    for (int k = 0; k < ni; ++k) {
      double v2 = 0;
      for (int c = 0; c < 3; ++c) v2 += R(vimp, k, c) * R(vimp, k, c);
      ekinx = ekinx + 0.5 * m_imp[k] * v2;
    }
    double sh = 0;
#pragma omp parallel for reduction(+ : sh) schedule(static)
    for (long i = 0; i < g.nxyz; ++i) sh += uimp[i] * den[i];
    double eHeX = sh * g.dxyz;
    double eii = 0;
    for (int k = 0; k < ni; ++k)
      for (int m = k + 1; m < ni; ++m) {
        double s = 0;
        for (int c = 0; c < 3; ++c) {
          double d = R(rimp, k, c) - R(rimp, m, c);
          s += d * d;
        }
        eii += select_pot(p.ii_kind, p.ii_D, p.ii_re, p.ii_a, p.ii_rcut, p.ii_umax, std::sqrt(s));
      }
    double eimpu = ekinx + eHeX + eii;
    double v[11] = {etot4, ekin4, elj4, ecor4, esolid, ea, ekinx, eHeX, eii, eimpu, etot4 + eimpu};
    std::memcpy(out, v, sizeof(v));
  }
};

// ------------------------------------------------------------------------------------------------
// Cubic splines and interval search of the quantum-impurity path.
// findi: Dynamics_quantum_impurities/mates.f:4-33 -- bisection for the 1-based interval i with
//   x(i) < xc <= x(i+1); i = n-1 above the table, 1 below it.
// spline: mates.f:36-110 -- cubic spline with prescribed end second derivatives s1, sn
//   (Maron, Numerical Analysis, 1982), coefficients of p_i(x) = a + x(b + x(c + x d)) in the
//   absolute abscissa.  1-based helpers keep the restatement next to the reference's indexing.
// ------------------------------------------------------------------------------------------------
static int findi(const double* x, double xc, int n) {
  if (xc > x[n - 1]) return n - 1;
  if (xc < x[0]) return 1;
  int i = 1, i1 = n;
  do {
    const int it = (i + i1) / 2;
    if (xc > x[it - 1]) i = it;
    if (xc <= x[it - 1]) i1 = it;
  } while (i1 - i > 1);
  return i;
}

static void spline_maron(const double* xv, const double* yv, double* av, double* bv, double* cv,
                         double* dv, double s1, double sn, int n) {
  auto X = [&](int i) { return xv[i - 1]; };
  auto Y = [&](int i) { return yv[i - 1]; };
  auto A = [&](int i) -> double& { return av[i - 1]; };
  auto B = [&](int i) -> double& { return bv[i - 1]; };
  auto C = [&](int i) -> double& { return cv[i - 1]; };
  auto D = [&](int i) -> double& { return dv[i - 1]; };
  const int n1 = n - 1, n2 = n - 2;
  for (int i = 1; i <= n1; ++i) {
    A(i) = X(i + 1) - X(i);
    D(i) = (Y(i + 1) - Y(i)) / A(i);
  }
  for (int i = 1; i <= n2; ++i) {
    B(i) = 2.0 * (A(i) + A(i + 1));
    const int k = n1 - i + 1;
    D(k) = 6.0 * (D(k) - D(k - 1));
  }
  D(2) = D(2) - A(1) * s1;
  D(n1) = D(n1) - A(n1) * sn;
  for (int i = 2; i <= n2; ++i) {
    const double r = A(i) / B(i - 1);
    B(i) = B(i) - r * A(i);
    D(i + 1) = D(i + 1) - r * D(i);
  }
  D(n1) = D(n1) / B(n2);
  for (int i = 2; i <= n2; ++i) {
    const int k = n1 - i + 1;
    D(k) = (D(k) - A(k) * D(k + 1)) / B(k - 1);
  }
  D(n) = sn;
  double si1 = s1;
  for (int i = 1; i <= n1; ++i) {
    const double si = si1;
    si1 = D(i + 1);
    const double h = A(i), hi = 1.0 / h;
    const double x0 = X(i), x1 = X(i + 1);
    A(i) = (hi / 6.0) * (si * (x1 * x1 * x1) - si1 * (x0 * x0 * x0)) + hi * (Y(i) * x1 - Y(i + 1) * x0) +
           (h / 6.0) * (si1 * x0 - si * x1);
    B(i) = (hi / 2.0) * (si1 * (x0 * x0) - si * (x1 * x1)) + hi * (Y(i + 1) - Y(i)) + (h / 6.0) * (si - si1);
    C(i) = (hi / 2.0) * (si * x1 - si1 * x0);
    D(i) = (hi / 6.0) * (si1 - si);
  }
}

// A pair potential of the quantum path: {kind, D, re, a, r_cutoff, umax} (Select_Pot contract).
struct PairPot {
  int kind = 0;
  double D = 0, re = 0, a = 0, rcut = 0, umax = 0;
  double operator()(double r) const { return select_pot(kind, D, re, a, rcut, umax, r); }
  bool same(const PairPot& o) const {
    return kind == o.kind && D == o.D && re == o.re && a == o.a && rcut == o.rcut && umax == o.umax;
  }
};

// FT_V_spline (Dynamics_quantum_impurities/FT_V_spline.f90:14-276): the 3-D Fourier transform
// V(p) = 4 pi/q int r sin(q r) V(r) dr, q = 2 pi p, of a radial potential.  V is held at
// f_cutoff = umax below r_cutoff (integrated analytically, optionally by the inverted-parabola
// fit of :128-146), splined on [r_cutoff + 1e-8, 5000] with N_FT_V_spline nodes and second
// derivatives from 3-point differences at the ends (:92-120), and each cubic piece is
// integrated in closed form (:151-225).  The momentum table P_p = (i-1) H_p, i = 1..N_p with
// N_p = int(Pmax/H_p + 1.5), is redefined below small_q = 0.01 by a natural 4-point spline through
// p = 0 and the first three p > small_q (:229-258) and splined for evaluation (:262).
struct FTVSpline {
  std::vector<double> P, A, B, C, D, Vpp;
  int np = 0;
  static constexpr double kRmax = 5000.0, kEps = 1.0e-8, kSmallQ = 1.0e-2, kDr = 0.05;

  // Vpp(p) of one momentum, given the spline of V (x, a, b, c, d; n nodes).
  static double transform(double p, const PairPot& v, bool parabolic, const std::vector<double>& x,
                          const std::vector<double>& a, const std::vector<double>& b,
                          const std::vector<double>& c, const std::vector<double>& d, int n) {
    const double Qpi = 4.0 * kPi;
    const double r0 = v.rcut, f0 = v.umax;
    double aa = 0, cc = 0;
    if (parabolic) {
      const double r1 = r0 + kDr, f1 = v(r1);
      aa = (f0 - f1) / (r0 * r0 - r1 * r1);
      cc = (r0 * r0 * f1 - r1 * r1 * f0) / (r0 * r0 - r1 * r1);
    }
    if (p == 0.0) {
      double Vp = parabolic ? aa * (r0 * r0 * r0 * r0 * r0) * 0.2 + cc * (r0 * r0 * r0) / 3.0
                            : (r0 * r0 * r0) * f0 / 3.0;
      double Fi = 0.0;
      for (int j = 0; j < n - 1; ++j) {
        const double u = x[j], w = x[j + 1];
        const double u2 = u * u, w2 = w * w;
        Fi = Fi + a[j] / 3.0 * (w2 * w - u2 * u) + b[j] / 4.0 * (w2 * w2 - u2 * u2) +
             c[j] / 5.0 * (w2 * w2 * w - u2 * u2 * u) + d[j] / 6.0 * (w2 * w2 * w2 - u2 * u2 * u2);
      }
      return (Vp + Fi) * Qpi;
    }
    const double q = 2.0 * kPi * p;
    const double c1oq = 1.0 / q, c1oq2 = c1oq * c1oq, c1oq3 = c1oq2 * c1oq, c1oq4 = c1oq2 * c1oq2,
                 c1oq5 = c1oq4 * c1oq;
    double Vp;
    if (parabolic)
      Vp = c1oq * (std::cos(q * r0) * (6.0 * aa * r0 * c1oq2 - aa * (r0 * r0 * r0) - cc * r0) +
                   std::sin(q * r0) * ((3.0 * aa * (r0 * r0) + cc) * c1oq - 6.0 * aa * c1oq3));
    else
      Vp = f0 * c1oq * (std::sin(q * r0) * c1oq - r0 * std::cos(q * r0));
    double Fi = 0.0;
    for (int j = 0; j < n - 1; ++j) {
      const double rj = x[j], rj1 = x[j + 1];
      const double sqrj = std::sin(q * rj), cqrj = std::cos(q * rj);
      const double sqrj1 = std::sin(q * rj1), cqrj1 = std::cos(q * rj1);
      const double A_ = a[j], B_ = b[j], C_ = c[j], D_ = d[j];
      Fi = Fi + (A_ + (B_ + (C_ + D_ * rj) * rj) * rj) * rj * c1oq * cqrj -
           (A_ + (B_ + (C_ + D_ * rj1) * rj1) * rj1) * rj1 * c1oq * cqrj1 +
           (A_ + (2.0 * B_ + (3.0 * C_ + 4.0 * D_ * rj1) * rj1) * rj1) * c1oq2 * sqrj1 -
           (A_ + (2.0 * B_ + (3.0 * C_ + 4.0 * D_ * rj) * rj) * rj) * c1oq2 * sqrj +
           (2.0 * B_ + (6.0 * C_ + 12.0 * D_ * rj1) * rj1) * c1oq3 * cqrj1 -
           (2.0 * B_ + (6.0 * C_ + 12.0 * D_ * rj) * rj) * c1oq3 * cqrj +
           (6.0 * C_ + 24.0 * D_ * rj) * c1oq4 * sqrj - (6.0 * C_ + 24.0 * D_ * rj1) * c1oq4 * sqrj1 +
           24.0 * D_ * c1oq5 * (cqrj - cqrj1);
    }
    return (Vp + Fi) * c1oq * Qpi;
  }

  // The spline of V on [r_cutoff + eps, r_max] (FT_V_spline.f90:83-120).
  static void radial_spline(const PairPot& v, int n, std::vector<double>& x, std::vector<double>& a,
                            std::vector<double>& b, std::vector<double>& c, std::vector<double>& d) {
    const double X1 = v.rcut + kEps, XN = kRmax;
    double r0 = X1, r1 = r0 + kDr, r2 = r1 + kDr;
    const double S1 = (v(r0) - 2.0 * v(r1) + v(r2)) / (kDr * kDr);
    r0 = XN;
    const double Sn = (v(r0 - kDr) - 2.0 * v(r0) + v(r0 + kDr)) / (kDr * kDr);
    const double h = (XN - X1) / (n - 1);
    x.resize(n); a.resize(n); b.resize(n); c.resize(n); d.resize(n);
    std::vector<double> y(n);
    for (int i = 1; i <= n; ++i) {
      const double r = (i - 1) * h + X1;
      x[i - 1] = r;
      y[i - 1] = v(r);
    }
    spline_maron(x.data(), y.data(), a.data(), b.data(), c.data(), d.data(), S1, Sn, n);
  }

  // Table of Vpp at P_p (i-1)*hp after the small-q redefinition, and its spline.
  void build(const PairPot& v, double pmax, double hp, int n, bool parabolic) {
    std::vector<double> x, a, b, c, d;
    radial_spline(v, n, x, a, b, c, d);
    np = (int)(pmax / hp + 1.5);
    P.resize(np); Vpp.resize(np);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < np; ++i) {
      const double p = i * hp;
      P[i] = p;
      Vpp[i] = transform(p, v, parabolic, x, a, b, c, d, n);
    }
    redefine_small_q(P, Vpp);
    A.resize(np); B.resize(np); C.resize(np); D.resize(np);
    spline_maron(P.data(), Vpp.data(), A.data(), B.data(), C.data(), D.data(), 0.0, 0.0, np);
  }
  static void redefine_small_q(const std::vector<double>& P, std::vector<double>& V) {
    const int np = (int)P.size();
    double x[4] = {0.0, 0, 0, 0}, y[4] = {V[0], 0, 0, 0};
    int iaux = 1;
    for (int i = 2; i <= np; ++i) {
      const double p = P[i - 1];
      if (p > kSmallQ) {
        ++iaux;
        x[iaux - 1] = p;
        y[iaux - 1] = V[i - 1];
      }
      if (iaux == 4) break;
    }
    double a[4], b[4], c[4], d[4];
    spline_maron(x, y, a, b, c, d, 0.0, 0.0, 4);
    for (int i = 2; i <= np; ++i) {
      const double p = P[i - 1];
      if (p <= kSmallQ) V[i - 1] = a[0] + p * (b[0] + p * (c[0] + p * d[0]));
      else break;
    }
  }
  double eval(double p) const {
    const int k = findi(P.data(), p, np) - 1;
    return A[k] + p * (B[k] + p * (C[k] + p * D[k]));
  }
};

// ------------------------------------------------------------------------------------------------
// Real-time TDDFT with quantum impurities (Dynamics_quantum_impurities): the impurities are wave
// functions psix_i with masses m_imp_u(i) and He-X kernels uimp_k (FT_V_spline of the pair
// potential) and X-X kernels uimp_k_k.
// ------------------------------------------------------------------------------------------------
struct QDyn : Common {
  int ni = 0;
  double mu4 = 0.0;
  std::vector<double> h2o2mx;
  std::vector<cplx> psi, pc, q, timec, s1, s2, s3, s4, s5, wk2;
  std::vector<cplx> psiold[3], hpsiold[2];
  std::vector<std::vector<cplx>> psix, pcx, qx, psixold, hpsixold;  // [i], [3i+s], [2i+s]
  std::vector<std::vector<double>> upotx, uimpk, uimpkk;             // uimpkk[i + ni j]
  std::vector<double> potx4, sto2, sto1x;
  int ioldp[3] = {1, 2, 3}, ioldh[2] = {1, 2};
  std::vector<int> ioldpx, ioldhx;  // (3, N_imp), (2, N_imp) as in the rkpc module

  // potenimpini (Dynamics_quantum_impurities/potenimpini.f90:116-163): qmax = max(100,
  // |pmax|), Nq = max(10001, nq), Hq = qmax/(Nq-1), uimp_k = FT_V_spline(pmod), and uimp_k_k
  // for the non-'null' pairs i != j.
  void init(const ho_params& pp, int n, const double* m_imp_u, double mu, const double* hex,
            const double* xx, int nspline, int nq, int parabolic) {
    init_common(pp);
    ni = n;
    mu4 = mu;
    const long N = g.nxyz;
    for (auto* v : {&psi, &pc, &q, &timec, &s1, &s2, &s3, &s4, &s5}) v->assign(N, 0);
    for (auto& v : psiold) v.assign(N, 0);
    for (auto& v : hpsiold) v.assign(N, 0);
    wk2.assign(g.nk, 0);
    potx4.assign(N, 0); sto2.assign(N, 0); sto1x.assign(N, 0);
    psix.assign(ni, std::vector<cplx>(N)); pcx = psix; qx = psix;
    psixold.assign(3 * ni, std::vector<cplx>(N)); hpsixold.assign(2 * ni, std::vector<cplx>(N));
    upotx.assign(ni, std::vector<double>(N));
    h2o2mx.resize(ni);
    for (int i = 0; i < ni; ++i) h2o2mx[i] = p.h2o2m4 * 4.002603 / m_imp_u[i];
    ioldpx.resize(3 * ni); ioldhx.resize(2 * ni);
    for (int i = 0; i < ni; ++i) {
      for (int s = 0; s < 3; ++s) ioldpx[3 * i + s] = s + 1;
      for (int s = 0; s < 2; ++s) ioldhx[2 * i + s] = s + 1;
    }
    for (int k = 0; k < g.nz; ++k)  // timec: Dynamics_quantum_impurities/DFT4He3d.f90:581-591
      for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i) {
          double s = 1.0 + std::tanh((std::fabs(g.x[i]) - p.txmean) / p.txsurf);
          s = s + 1.0 + std::tanh((std::fabs(g.y[j]) - p.tymean) / p.tysurf);
          s = s + 1.0 + std::tanh((std::fabs(g.z[k]) - p.tzmean) / p.tzsurf);
          timec[i + (long)g.nx * (j + (long)g.ny * k)] = cplx(p.lambdah * s, 1.0);
        }
    const double pmx = 1.0 / (2.0 * g.hx), pmy = 1.0 / (2.0 * g.hy), pmz = 1.0 / (2.0 * g.hz);
    const double qmax = std::max(100.0, std::sqrt(pmx * pmx + pmy * pmy + pmz * pmz));
    const long Nq = std::max(10001L, (long)nq);
    const double Hq = qmax / (double)(Nq - 1);
    auto pot = [](const double* v) {
      PairPot pp_;
      pp_.kind = (int)v[0]; pp_.D = v[1]; pp_.re = v[2]; pp_.a = v[3]; pp_.rcut = v[4]; pp_.umax = v[5];
      return pp_;
    };
    std::vector<std::pair<PairPot, FTVSpline>> cache;
    auto table = [&](const PairPot& v) -> const FTVSpline& {
      for (auto& e : cache)
        if (e.first.same(v)) return e.second;
      cache.emplace_back(v, FTVSpline());
      cache.back().second.build(v, qmax, Hq, nspline, parabolic != 0);
      return cache.back().second;
    };
    uimpk.assign(ni, std::vector<double>());
    uimpkk.assign((size_t)ni * ni, std::vector<double>());
    for (int i = 0; i < ni; ++i) {
      const FTVSpline& t = table(pot(hex + 6 * i));
      uimpk[i].resize(g.nk);
#pragma omp parallel for schedule(static)
      for (long k = 0; k < g.nk; ++k) uimpk[i][k] = t.eval(g.pmod[k]);
      for (int j = 0; j < ni; ++j) {
        const double* v = xx + 6 * (i + (size_t)ni * j);
        if (i == j || (int)v[0] == 0) continue;
        const FTVSpline& tj = table(pot(v));
        auto& dst = uimpkk[i + (size_t)ni * j];
        dst.resize(g.nk);
#pragma omp parallel for schedule(static)
        for (long k = 0; k < g.nk; ++k) dst[k] = tj.eval(g.pmod[k]);
      }
    }
  }

  void density() {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < g.nxyz; ++i) den[i] = std::norm(psi[i]);
  }
  // Sto1 = psix*conjg(psix) (real part), R2C into wk1.
  void fft_denx(int i) {
    const cplx* f = psix[i].data();
#pragma omp parallel for schedule(static)
    for (long k = 0; k < g.nxyz; ++k) sto1x[k] = f[k].real() * f[k].real() + f[k].imag() * f[k].imag();
    fft.r2c(sto1x.data(), wk1.data());
  }
  // potenimp: Dynamics_quantum_impurities/potenimp.f90:1-43.
  void potenimp() {
    fftfw_den();
    const long N = g.nxyz;
    std::fill(potx4.begin(), potx4.end(), 0.0);
    for (int i = 0; i < ni; ++i) {
      fft_denx(i);
      for (long k = 0; k < g.nk; ++k) wk2[k] = wk1[k] * uimpk[i][k];
      fft.c2r(wk2.data(), sto2.data(), renor);
      for (long k = 0; k < N; ++k) potx4[k] = potx4[k] + sto2[k];
      for (long k = 0; k < g.nk; ++k) wk2[k] = fden[k] * uimpk[i][k];
      fft.c2r(wk2.data(), upotx[i].data(), renor);
      for (int j = 0; j < ni; ++j) {
        const auto& kk = uimpkk[i + (size_t)ni * j];
        if (j == i || kk.empty()) continue;
        fft_denx(j);
        for (long k = 0; k < g.nk; ++k) wk2[k] = wk1[k] * kk[k];
        fft.c2r(wk2.data(), sto2.data(), renor);
        for (long k = 0; k < N; ++k) upotx[i][k] = upotx[i][k] + sto2[k];
      }
    }
  }
  // poten: Dynamics_quantum_impurities/poten.f90:5-155 (fden comes from potenimp).
  void poten() {
    coarse_grain();
    if (otc()) derden();
    lennard_jones();
    if (otc()) {
      alfa_density();
      term_alfa();
    }
    correlation_and_assembly(potx4.data(), otc() ? ualphas.data() : nullptr);
  }
  // s4 = timec*((d2x+d2y+d2z)*h2o2m - (pot - shift)*f)  (steprk.f90:68,94; steppc.f90:46,77).
  void hpsi_q(const std::vector<cplx>& f, const std::vector<double>& pot, double shift, double h2) {
    deriv3d<cplx>(2, g, 0, p.icon, w1, w2, f.data(), s1.data());
    deriv3d<cplx>(2, g, 1, p.icon, w1, w2, f.data(), s2.data());
    deriv3d<cplx>(2, g, 2, p.icon, w1, w2, f.data(), s3.data());
#pragma omp parallel for schedule(static)
    for (long i = 0; i < g.nxyz; ++i) {
      const cplx lap = s1[i] + s2[i] + s3[i];
      s4[i] = timec[i] * (lap * h2 - (pot[i] - shift) * f[i]);
    }
  }

  // steprk: Dynamics_quantum_impurities/steprk.f90:1-124.
  void steprk(double deltat) {
    const double arun[4] = {0.5, 1.0 - 1.0 / std::sqrt(2.0), 1.0 + 1.0 / std::sqrt(2.0), 1.0 / 6.0};
    const double brun[4] = {2.0, 1.0, 1.0, 2.0};
    const double crun[4] = {0.5, 1.0 - 1.0 / std::sqrt(2.0), 1.0 + 1.0 / std::sqrt(2.0), 0.5};
    const long N = g.nxyz;
    auto stage = [&](int jr, std::vector<cplx>& f, std::vector<cplx>& qq, std::vector<cplx>* po,
                     std::vector<cplx>* ho) {
      if (jr == 0) {
        ho[1] = ho[0];
        ho[0] = s4;
        po[2] = po[1];
        po[1] = po[0];
        po[0] = f;
      }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) {
        const cplx sto1c = arun[jr] * (s4[i] - brun[jr] * qq[i]);
        qq[i] = qq[i] + 3.0 * sto1c - crun[jr] * s4[i];
        f[i] = f[i] + deltat * sto1c;
      }
    };
    for (int jr = 0; jr < 4; ++jr) {
      hpsi_q(psi, pot4, mu4, p.h2o2m4);
      stage(jr, psi, q, psiold, hpsiold);
      density();
      for (int i = 0; i < ni; ++i) {
        hpsi_q(psix[i], upotx[i], 0.0, h2o2mx[i]);
        stage(jr, psix[i], qx[i], &psixold[3 * i], &hpsixold[2 * i]);
      }
      if (jr <= 2) { potenimp(); poten(); }
    }
    for (int s = 0; s < 3; ++s) {
      ioldp[s] = s + 1;
      for (int i = 0; i < ni; ++i) ioldpx[3 * i + s] = s + 1;
    }
    for (int s = 0; s < 2; ++s) {
      ioldh[s] = s + 1;
      for (int i = 0; i < ni; ++i) ioldhx[2 * i + s] = s + 1;
    }
  }

  // steppc: Dynamics_quantum_impurities/steppc.f90:1-157.
  void steppc(double deltat, double* errHe, double* errpsix) {
    const double c112 = 112.0 / 121.0, c9 = 9.0 / 121.0, c4o3 = 4.0 / 3.0;
    const long N = g.nxyz;
    auto predict = [&](std::vector<cplx>& f, std::vector<cplx>& pcc, std::vector<cplx>* po,
                       std::vector<cplx>* ho, int* ip, int* ih) {
      std::vector<cplx>& po3 = po[ip[2] - 1];
      const std::vector<cplx>& h1 = ho[ih[0] - 1];
      std::vector<cplx>& h2 = ho[ih[1] - 1];
      const double s = c4o3 * deltat;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) {
        const cplx sto1c = po3[i] + s * (2.0 * s4[i] - h1[i] + 2.0 * h2[i]);
        po3[i] = f[i];
        f[i] = sto1c - c112 * pcc[i];
        pcc[i] = sto1c;
        h2[i] = s4[i];
      }
      std::swap(ih[0], ih[1]);
    };
    auto correct = [&](std::vector<cplx>& f, std::vector<cplx>& pcc, std::vector<cplx>* po,
                       std::vector<cplx>* ho, const int* ip, const int* ih) {
      const std::vector<cplx>& po3 = po[ip[2] - 1];
      const std::vector<cplx>& po2 = po[ip[1] - 1];
      const std::vector<cplx>& h1 = ho[ih[0] - 1];
      const std::vector<cplx>& h2 = ho[ih[1] - 1];
      const double s3 = 3.0 * deltat;
      double sabs = 0.0;
#pragma omp parallel for reduction(+ : sabs) schedule(static)
      for (long i = 0; i < N; ++i) {
        const cplx sto5c = 0.125 * (9.0 * po3[i] - po2[i] + s3 * (s4[i] + 2.0 * h1[i] - h2[i]));
        pcc[i] = pcc[i] - sto5c;
        f[i] = sto5c + c9 * pcc[i];
        sabs += std::abs(pcc[i]);
      }
      return c9 * sabs;
    };
    auto rotate = [](int* ip) {
      const int a = ip[2];
      ip[2] = ip[1]; ip[1] = ip[0]; ip[0] = a;
    };
    hpsi_q(psi, pot4, mu4, p.h2o2m4);
    predict(psi, pc, psiold, hpsiold, ioldp, ioldh);
    density();
    for (int i = 0; i < ni; ++i) {
      hpsi_q(psix[i], upotx[i], 0.0, h2o2mx[i]);
      predict(psix[i], pcx[i], &psixold[3 * i], &hpsixold[2 * i], &ioldpx[3 * i], &ioldhx[2 * i]);
    }
    potenimp();
    poten();
    hpsi_q(psi, pot4, mu4, p.h2o2m4);
    double eh = correct(psi, pc, psiold, hpsiold, ioldp, ioldh);
    density();
    double ex = 0.0;
    for (int i = 0; i < ni; ++i) {
      hpsi_q(psix[i], upotx[i], 0.0, h2o2mx[i]);
      ex = ex + correct(psix[i], pcx[i], &psixold[3 * i], &hpsixold[2 * i], &ioldpx[3 * i], &ioldhx[2 * i]);
    }
    if (errpsix) *errpsix = ex / (double)N;
    if (errHe) *errHe = eh / (double)N;
    rotate(ioldp);
    for (int i = 0; i < ni; ++i) rotate(&ioldpx[3 * i]);
  }

  // energy: Dynamics_quantum_impurities/energy.f90:12-139.  out = {etot4, ekin4, elj4, ecor4,
  // esolid, ealphas, ekinx, eHeX, eimpu_impu, eimpu, etot}.
  void energy(double* out) {
    const long N = g.nxyz;
    auto grad2 = [&](const std::vector<cplx>& f) {
      deriv3d<cplx>(1, g, 0, p.icon, w1, w2, f.data(), s1.data());
      deriv3d<cplx>(1, g, 1, p.icon, w1, w2, f.data(), s2.data());
      deriv3d<cplx>(1, g, 2, p.icon, w1, w2, f.data(), s3.data());
      double ek = 0;
#pragma omp parallel for reduction(+ : ek) schedule(static)
      for (long i = 0; i < N; ++i) ek += std::norm(s1[i]) + std::norm(s2[i]) + std::norm(s3[i]);
      return ek;
    };
    const double ek = grad2(psi);
    double ekin4, elj4, ecor4, esolid;
    he_energy_sums(ek, &ekin4, &elj4, &ecor4, &esolid);
    const double ea = ealphas();
    const double etot4 = ekin4 + elj4 + ecor4 + esolid + (otc() ? ea : 0.0);
    double ekinx = 0.0;
    std::fill(wk2.begin(), wk2.end(), cplx(0.0));
    for (int k = 0; k < ni; ++k) {
      ekinx = ekinx + h2o2mx[k] * grad2(psix[k]);
      fft_denx(k);
      for (long i = 0; i < g.nk; ++i) wk2[i] = wk2[i] + wk1[i] * uimpk[k][i];
    }
    ekinx = ekinx * g.dxyz;
    fft.c2r(wk2.data(), sto2.data(), renor);
    double sh = 0;
#pragma omp parallel for reduction(+ : sh) schedule(static)
    for (long i = 0; i < N; ++i) sh += sto2[i] * den[i];
    const double eHeX = sh * g.dxyz;
    double eii = 0.0;
    for (int k = 0; k < ni; ++k) {
      fft_denx(k);
      for (int m = k + 1; m < ni; ++m) {
        const auto& kk = uimpkk[k + (size_t)ni * m];
        for (long i = 0; i < g.nk; ++i) wk2[i] = kk.empty() ? cplx(0.0) : wk1[i] * kk[i];
        fft.c2r(wk2.data(), sto2.data(), renor);
        double s = 0;
        const cplx* f = psix[m].data();
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (long i = 0; i < N; ++i) s += sto2[i] * (f[i].real() * f[i].real() + f[i].imag() * f[i].imag());
        eii = eii + s;
      }
    }
    eii = eii * g.dxyz;
    const double eimpu = ekinx + eHeX + eii;
    const double v[11] = {etot4, ekin4, elj4, ecor4, esolid, ea, ekinx, eHeX, eii, eimpu, etot4 + eimpu};
    std::memcpy(out, v, sizeof(v));
  }

  // Norm and centre of |psix_k|^2 (Dynamics_quantum_impurities/DFT4He3d.f90:682-700):
  // out[4k..4k+3] = {sum |psix|^2 dxyz, <x>, <y>, <z>}.
  void moments(double* out) const {
    for (int k = 0; k < ni; ++k) {
      double a = 0, ax = 0, ay = 0, az = 0;
      const cplx* f = psix[k].data();
#pragma omp parallel for collapse(2) reduction(+ : a, ax, ay, az) schedule(static)
      for (int iz = 0; iz < g.nz; ++iz)
        for (int iy = 0; iy < g.ny; ++iy)
          for (int ix = 0; ix < g.nx; ++ix) {
            const cplx v = f[ix + (long)g.nx * (iy + (long)g.ny * iz)];
            const double s = v.real() * v.real() + v.imag() * v.imag();
            a += s; ax += s * g.x[ix]; ay += s * g.y[iy]; az += s * g.z[iz];
          }
      a = a * g.dxyz;
      out[4 * k] = a;
      out[4 * k + 1] = ax * g.dxyz / a;
      out[4 * k + 2] = ay * g.dxyz / a;
      out[4 * k + 3] = az * g.dxyz / a;
    }
  }
};

// ------------------------------------------------------------------------------------------------
// Imaginary-time statics (He_statics), pure droplet, real psi.
// ------------------------------------------------------------------------------------------------
struct Stat : Common {
  std::vector<double> psi, hpsi, q, pc, timec, t1, t2, t3, t4, t5;
  std::vector<double> psiold[3], hpsiold[2];
  int ioldp[3] = {1, 2, 3}, ioldh[2] = {1, 2};
  double errpc = 0.0;

  void init(const ho_params& pp) {
    init_common(pp);
    long N = g.nxyz;
    psi.assign(N, 0); hpsi.assign(N, 0); q.assign(N, 0); pc.assign(N, 0); timec.assign(N, 0);
    t1.assign(N, 0); t2.assign(N, 0); t3.assign(N, 0); t4.assign(N, 0); t5.assign(N, 0);
    for (auto& v : psiold) v.assign(N, 0);
    for (auto& v : hpsiold) v.assign(N, 0);
  }
  // poten (statics): He_statics/poten.f90:27-115.  fden and dencg are NOT refreshed here: the
  // driver refreshes them once per iteration (BCN4HeDFT.f90:1131-1155).
  void poten() {
    lennard_jones();
    if (otc()) term_alfa();
    correlation_and_assembly(nullptr, otc() ? ualphas.data() : nullptr);
  }
  // The driver's per-iteration refresh: derden, fftfw(den,fden), dencg (BCN4HeDFT.f90:1131-1155).
  void refresh() {
    derden();
    fftfw_den();
    coarse_grain();
    if (otc()) alfa_density();
  }
  void lap(const std::vector<double>& f) {
    deriv3d<double>(2, g, 0, p.icon, w1, w2, f.data(), t1.data());
    deriv3d<double>(2, g, 1, p.icon, w1, w2, f.data(), t2.data());
    deriv3d<double>(2, g, 2, p.icon, w1, w2, f.data(), t3.data());
  }
  double sum_psi2() const {
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < g.nxyz; ++i) s += psi[i] * psi[i];
    return s;
  }
  void renorm(int n4) {
    double cnorm = std::sqrt((double)n4 / (sum_psi2() * g.dxyz));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < g.nxyz; ++i) {
      psi[i] = std::fabs(psi[i]) * cnorm;
      den[i] = psi[i] * psi[i];
    }
  }
  // steprkr: He_statics/steprkr.f90:1-96.
  void steprkr(double deltat, double* mu4, double* mu4err, int n4) {
    double arun[4] = {0.5, 1.0 - 1.0 / std::sqrt(2.0), 1.0 + 1.0 / std::sqrt(2.0), 1.0 / 6.0};
    double brun[4] = {2.0, 1.0, 1.0, 2.0};
    double crun[4] = {0.5, 1.0 - 1.0 / std::sqrt(2.0), 1.0 + 1.0 / std::sqrt(2.0), 0.5};
    const long N = g.nxyz;
    double hmean = 0, err = 0;
    for (int jr = 0; jr < 4; ++jr) {
      lap(psi);
      double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
      for (long i = 0; i < N; ++i) {
        hpsi[i] = -(t1[i] + t2[i] + t3[i]) * p.h2o2m4 + pot4[i] * psi[i];
        s += psi[i] * hpsi[i];
      }
      err = s * g.dxyz / (double)n4;
      if (jr == 0) {
        hmean = err;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i)
          timec[i] = deltat / (1.0 + std::exp((std::fabs(hpsi[i] / psi[i]) - p.dmumax) / p.sdmu)) +
                     p.dtmin;
      }
      if (jr == 0) {
        hpsiold[1] = hpsiold[0];
        psiold[2] = psiold[1];
        psiold[1] = psiold[0];
        psiold[0] = psi;
      }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) {
        double sto4 = -(hpsi[i] - err * psi[i]);
        double sto1 = arun[jr] * (sto4 - brun[jr] * q[i]);
        q[i] = q[i] + 3.0 * sto1 - crun[jr] * sto4;
        if (jr == 0) hpsiold[0][i] = sto4;
        psi[i] = psi[i] + timec[i] * sto1;
      }
      renorm(n4);
      if (jr <= 2) poten();
    }
    for (int i = 0; i < 3; ++i) ioldp[i] = i + 1;
    for (int i = 0; i < 2; ++i) ioldh[i] = i + 1;
    *mu4err = std::fabs(1.0 - *mu4 / hmean);
    *mu4 = hmean;
  }
  // steppcr: He_statics/steppcr.f90:1-108.
  void steppcr(double deltat, double* mu4, double* mu4err, int n4) {
    const double c112 = 112.0 / 121.0, c9 = 9.0 / 121.0, c4o3 = 4.0 / 3.0;
    const long N = g.nxyz;
    lap(psi);
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < N; ++i) {
      hpsi[i] = -(t1[i] + t2[i] + t3[i]) * p.h2o2m4 + pot4[i] * psi[i];
      s += psi[i] * hpsi[i];
    }
    double hmean = s * g.dxyz / (double)n4;
    {
      std::vector<double>& po3 = psiold[ioldp[2] - 1];
      const std::vector<double>& h1 = hpsiold[ioldh[0] - 1];
      std::vector<double>& h2 = hpsiold[ioldh[1] - 1];
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) {
        timec[i] = deltat / (1.0 + std::exp((std::fabs(hpsi[i] / psi[i]) - p.dmumax) / p.sdmu)) +
                   p.dtmin;
        double sto4 = -(hpsi[i] - hmean * psi[i]);
        double sto1 = po3[i] + c4o3 * timec[i] * (2.0 * sto4 - h1[i] + 2.0 * h2[i]);
        po3[i] = psi[i];
        psi[i] = sto1 - c112 * pc[i];
        pc[i] = sto1;
        h2[i] = sto4;
      }
    }
    renorm(n4);
    std::swap(ioldh[0], ioldh[1]);
    poten();
    lap(psi);
    double s2 = 0;
#pragma omp parallel for reduction(+ : s2) schedule(static)
    for (long i = 0; i < N; ++i) {
      t4[i] = -(t1[i] + t2[i] + t3[i]) * p.h2o2m4 + pot4[i] * psi[i];
      s2 += psi[i] * t4[i];
    }
    double mu = s2 * g.dxyz / (double)n4;
    double sabs = 0;
    {
      const std::vector<double>& po3 = psiold[ioldp[2] - 1];
      const std::vector<double>& po2 = psiold[ioldp[1] - 1];
      const std::vector<double>& h1 = hpsiold[ioldh[0] - 1];
      const std::vector<double>& h2 = hpsiold[ioldh[1] - 1];
#pragma omp parallel for reduction(+ : sabs) schedule(static)
      for (long i = 0; i < N; ++i) {
        double sto4 = -(t4[i] - mu * psi[i]);
        double sto5 = 0.125 * (9.0 * po3[i] - po2[i] + 3.0 * timec[i] * (sto4 + 2.0 * h1[i] - h2[i]));
        pc[i] = pc[i] - sto5;
        psi[i] = sto5 + c9 * pc[i];
        sabs += std::fabs(pc[i]);
      }
    }
    errpc = c9 * sabs;
    renorm(n4);
    errpc = errpc / (double)N;
    int a = ioldp[2];
    ioldp[2] = ioldp[1]; ioldp[1] = ioldp[0]; ioldp[0] = a;
    *mu4err = std::fabs(1.0 - *mu4 / hmean);
    *mu4 = hmean;
  }
  // evolo(0.0, mu4, mu4err, n4) as called once before the loop (BCN4HeDFT.f90:1050,
  // evolo.f90:41-93 with deltat = 0): mu4 = <psi|H|psi>/N, then renormalisation.
  void evolo0(double* mu4, double* mu4err, int n4) {
    lap(psi);
    double s = 0;
    for (long i = 0; i < g.nxyz; ++i) {
      hpsi[i] = -(t1[i] + t2[i] + t3[i]) * p.h2o2m4 + pot4[i] * psi[i];
      s += psi[i] * hpsi[i];
    }
    double hmean = s * g.dxyz / (double)n4;
    *mu4err = std::fabs(1.0 - *mu4 / hmean);
    *mu4 = hmean;
    renorm(n4);
  }
  // energy (statics, pure): He_statics/energy.f90:36-150.  out as in Dyn::energy.
  void energy(double* out) {
    deriv3d<double>(1, g, 0, p.icon, w1, w2, psi.data(), t1.data());
    deriv3d<double>(1, g, 1, p.icon, w1, w2, psi.data(), t2.data());
    deriv3d<double>(1, g, 2, p.icon, w1, w2, psi.data(), t3.data());
    double ek = 0;
#pragma omp parallel for reduction(+ : ek) schedule(static)
    for (long i = 0; i < g.nxyz; ++i) ek += t1[i] * t1[i] + t2[i] * t2[i] + t3[i] * t3[i];
    double ekin4, elj4, ecor4, esolid;
    he_energy_sums(ek, &ekin4, &elj4, &ecor4, &esolid);
    const double ea = ealphas();
    double etot4 = ekin4 + elj4 + ecor4 + esolid;
    if (otc()) etot4 = etot4 + ea;
    double v[11] = {etot4, ekin4, elj4, ecor4, esolid, ea, 0.0, 0.0, 0.0, 0.0, etot4};
    std::memcpy(out, v, sizeof(v));
  }
  // varmu: He_statics/varmu.f90:31 (hpsi holds H psi of the last predictor).
  double varmu(int npart, double mu) const {
    double s = 0;
    for (long i = 0; i < g.nxyz; ++i) s += std::fabs(hpsi[i] - mu * psi[i]) * psi[i];
    return s * g.dxyz / (double)npart;
  }
};

// ------------------------------------------------------------------------------------------------
// C API used by oracle/oracle.py (ctypes).
// ------------------------------------------------------------------------------------------------
static double* dyn_field(Dyn* d, const char* name, long* n) {
  std::string s(name);
  long N = d->g.nxyz, K = d->g.nk;
  auto R = [&](std::vector<double>& v, long nn) { *n = nn; return v.data(); };
  auto C = [&](std::vector<cplx>& v, long nn) { *n = 2 * nn; return (double*)v.data(); };
  if (d->otc()) {
    if (s == "denalf") { *n = d->g.nxyz; return d->denalf.data(); }
    if (s == "falfs") { *n = d->g.nxyz; return d->falfs.data(); }
    if (s == "intxalf") { *n = d->g.nxyz; return d->intxalf.data(); }
    if (s == "intyalf") { *n = d->g.nxyz; return d->intyalf.data(); }
    if (s == "intzalf") { *n = d->g.nxyz; return d->intzalf.data(); }
    if (s == "ualphas") { *n = d->g.nxyz; return d->ualphas.data(); }
    if (s == "kalfs") { *n = d->g.nk; return d->kalfs.data(); }
  }
  if (s == "dxden") { *n = d->g.nxyz; return d->dxden.data(); }
  if (s == "den") return R(d->den, N);
  if (s == "dencg") return R(d->dencg, N);
  if (s == "delj4") return R(d->delj4, N);
  if (s == "pot4") return R(d->pot4, N);
  if (s == "uimp") return R(d->uimp, N);
  if (s == "dxden") return R(d->dxden, N);
  if (s == "dyden") return R(d->dyden, N);
  if (s == "dzden") return R(d->dzden, N);
  if (s == "fvlj4") return R(d->fvlj4, K);
  if (s == "wcgk") return R(d->wcgk, K);
  if (s == "psi") return C(d->psi, N);
  if (s == "pc") return C(d->pc, N);
  if (s == "q") return C(d->q, N);
  if (s == "fden") return C(d->fden, K);
  if (s == "psiold1") return C(d->psiold[0], N);
  if (s == "psiold2") return C(d->psiold[1], N);
  if (s == "psiold3") return C(d->psiold[2], N);
  if (s == "hpsiold1") return C(d->hpsiold[0], N);
  if (s == "hpsiold2") return C(d->hpsiold[1], N);
  if (s == "rimp") return R(d->rimp, 3 * d->ni);
  if (s == "vimp") return R(d->vimp, 3 * d->ni);
  if (s == "aimp") return R(d->aimp, 3 * d->ni);
  if (s == "F") return R(d->F, 3 * d->ni);
  if (s == "potion") return R(d->potion, (long)d->ni * d->npot);
  if (s == "rimpold") return R(d->rimpold, 9 * d->ni);
  if (s == "vimpold") return R(d->vimpold, 9 * d->ni);
  if (s == "aimpold") return R(d->aimpold, 6 * d->ni);
  if (s == "pcr") return R(d->pcr, 3 * d->ni);
  if (s == "pcv") return R(d->pcv, 3 * d->ni);
  if (s == "qr") return R(d->qr, 3 * d->ni);
  if (s == "qv") return R(d->qv, 3 * d->ni);
  return nullptr;
}
static double* stat_field(Stat* d, const char* name, long* n) {
  std::string s(name);
  long N = d->g.nxyz, K = d->g.nk;
  auto R = [&](std::vector<double>& v, long nn) { *n = nn; return v.data(); };
  if (d->otc()) {
    if (s == "denalf") { *n = d->g.nxyz; return d->denalf.data(); }
    if (s == "falfs") { *n = d->g.nxyz; return d->falfs.data(); }
    if (s == "intxalf") { *n = d->g.nxyz; return d->intxalf.data(); }
    if (s == "intyalf") { *n = d->g.nxyz; return d->intyalf.data(); }
    if (s == "intzalf") { *n = d->g.nxyz; return d->intzalf.data(); }
    if (s == "ualphas") { *n = d->g.nxyz; return d->ualphas.data(); }
    if (s == "kalfs") { *n = d->g.nk; return d->kalfs.data(); }
  }
  if (s == "dxden") { *n = d->g.nxyz; return d->dxden.data(); }
  if (s == "den") return R(d->den, N);
  if (s == "psi") return R(d->psi, N);
  if (s == "dencg") return R(d->dencg, N);
  if (s == "delj4") return R(d->delj4, N);
  if (s == "pot4") return R(d->pot4, N);
  if (s == "hpsi") return R(d->hpsi, N);
  if (s == "fvlj4") return R(d->fvlj4, K);
  if (s == "wcgk") return R(d->wcgk, K);
  if (s == "fden") { *n = 2 * K; return (double*)d->fden.data(); }
  return nullptr;
}

static double* qdyn_field(QDyn* d, const char* name, long* n) {
  std::string s(name);
  const long N = d->g.nxyz, K = d->g.nk;
  int idx = 0;
  const size_t colon = s.find(':');
  if (colon != std::string::npos) {
    idx = std::atoi(s.c_str() + colon + 1);
    s = s.substr(0, colon);
  }
  auto R = [&](std::vector<double>& v, long nn) { *n = nn; return v.data(); };
  auto C = [&](std::vector<cplx>& v, long nn) { *n = 2 * nn; return (double*)v.data(); };
  const bool ok = idx >= 0 && idx < d->ni;
  if (d->otc()) {
    if (s == "denalf") { *n = d->g.nxyz; return d->denalf.data(); }
    if (s == "falfs") { *n = d->g.nxyz; return d->falfs.data(); }
    if (s == "intxalf") { *n = d->g.nxyz; return d->intxalf.data(); }
    if (s == "intyalf") { *n = d->g.nxyz; return d->intyalf.data(); }
    if (s == "intzalf") { *n = d->g.nxyz; return d->intzalf.data(); }
    if (s == "ualphas") { *n = d->g.nxyz; return d->ualphas.data(); }
    if (s == "kalfs") { *n = d->g.nk; return d->kalfs.data(); }
  }
  if (s == "dxden") { *n = d->g.nxyz; return d->dxden.data(); }
  if (s == "den") return R(d->den, N);
  if (s == "dencg") return R(d->dencg, N);
  if (s == "delj4") return R(d->delj4, N);
  if (s == "pot4") return R(d->pot4, N);
  if (s == "potx4") return R(d->potx4, N);
  if (s == "fvlj4") return R(d->fvlj4, K);
  if (s == "wcgk") return R(d->wcgk, K);
  if (s == "psi") return C(d->psi, N);
  if (s == "pc") return C(d->pc, N);
  if (s == "q") return C(d->q, N);
  if (s == "fden") return C(d->fden, K);
  if (s == "psiold1") return C(d->psiold[0], N);
  if (s == "psiold2") return C(d->psiold[1], N);
  if (s == "psiold3") return C(d->psiold[2], N);
  if (s == "hpsiold1") return C(d->hpsiold[0], N);
  if (s == "hpsiold2") return C(d->hpsiold[1], N);
  if (!ok) return nullptr;
  if (s == "psix") return C(d->psix[idx], N);
  if (s == "pcx") return C(d->pcx[idx], N);
  if (s == "qx") return C(d->qx[idx], N);
  if (s == "upotx") return R(d->upotx[idx], N);
  if (s == "uimpk") return R(d->uimpk[idx], K);
  if (s == "psixold1" || s == "psixold2" || s == "psixold3")
    return C(d->psixold[3 * idx + (s[7] - '1')], N);
  if (s == "hpsixold1" || s == "hpsixold2") return C(d->hpsixold[2 * idx + (s[8] - '1')], N);
  if (s.rfind("uimpkk", 0) == 0) {  // "uimpkk:i" with j in name "uimpkk<j>:i"
    const int j = (s.size() > 6) ? std::atoi(s.c_str() + 6) : 0;
    if (j < 0 || j >= d->ni) return nullptr;
    auto& v = d->uimpkk[idx + (size_t)d->ni * j];
    if (v.empty()) return nullptr;
    return R(v, K);
  }
  return nullptr;
}

extern "C" {
// Generic helpers (tests).
double ho_sine_integral(double x) { return sine_integral(x); }
void ho_bickley13(double* w1, double* w2) { bickley13(w1, w2); }
void ho_fforma(const ho_params* p, double* out) {
  Grid g; g.init(*p);
  std::vector<double> f;
  fforma(p->core == 1, p->eps4, p->sigma4, p->h4, g, f);
  std::memcpy(out, f.data(), sizeof(double) * g.nk);
}
void ho_initcg(const ho_params* p, double h, double* out) {
  Grid g; g.init(*p);
  std::vector<double> f;
  initcg(h, g, f);
  std::memcpy(out, f.data(), sizeof(double) * g.nk);
}
void ho_r2c(const ho_params* p, const double* in, double* out) {
  Grid g; g.init(*p);
  FFT3 f; f.init(g);
  f.r2c(in, (cplx*)out);
}
void ho_c2r(const ho_params* p, const double* in, double* out) {
  Grid g; g.init(*p);
  FFT3 f; f.init(g);
  std::vector<cplx> tmp((cplx*)in, (cplx*)in + g.nk);
  f.c2r(tmp.data(), out, 1.0 / ((double)((long)g.nx * g.ny * g.nz)));
}
void ho_deriv(const ho_params* p, int id, int axis, int is_complex, const double* f, double* df) {
  Grid g; g.init(*p);
  double w1[13], w2[13];
  bickley13(w1, w2);
  if (is_complex)
    deriv3d<cplx>(id, g, axis, p->icon, w1, w2, (const cplx*)f, (cplx*)df);
  else
    deriv3d<double>(id, g, axis, p->icon, w1, w2, f, df);
}

void* ho_dyn_create(const ho_params* p, const double* m_imp_u) {
  Dyn* d = new Dyn();
  d->init(*p, m_imp_u);
  return d;
}
void ho_dyn_destroy(void* h) { delete (Dyn*)h; }
double* ho_dyn_field(void* h, const char* name, long* n) { return dyn_field((Dyn*)h, name, n); }
void ho_dyn_potenimp(void* h) { ((Dyn*)h)->potenimp(); }
void ho_dyn_poten(void* h) { ((Dyn*)h)->poten(); }
void ho_dyn_forceimp(void* h) { ((Dyn*)h)->forceimp(); }
void ho_dyn_set_accel(void* h) { ((Dyn*)h)->set_accel(); }
void ho_dyn_steprk(void* h, double dt) { ((Dyn*)h)->steprk(dt); }
void ho_dyn_steppc(void* h, double dt, double* err3) {
  ((Dyn*)h)->steppc(dt, &err3[0], &err3[1], &err3[2]);
}
void ho_dyn_energy(void* h, double* out) { ((Dyn*)h)->energy(out); }
int ho_dyn_lstopimp(void* h) { return ((Dyn*)h)->lstopimp ? 1 : 0; }
// Ring indices ioldp(3), ioldh(2), ioldr(3), ioldv(3), iolda(2): set != 0 writes them.
void ho_dyn_ring(void* h, int* r, int set) {
  Dyn* d = (Dyn*)h;
  int* dst[13] = {&d->ioldp[0], &d->ioldp[1], &d->ioldp[2], &d->ioldh[0], &d->ioldh[1],
                  &d->ioldr[0], &d->ioldr[1], &d->ioldr[2], &d->ioldv[0], &d->ioldv[1],
                  &d->ioldv[2], &d->iolda[0], &d->iolda[1]};
  for (int i = 0; i < 13; ++i) {
    if (set) *dst[i] = r[i];
    else r[i] = *dst[i];
  }
}

void* ho_stat_create(const ho_params* p) {
  Stat* d = new Stat();
  d->init(*p);
  return d;
}
void ho_stat_destroy(void* h) { delete (Stat*)h; }
double* ho_stat_field(void* h, const char* name, long* n) { return stat_field((Stat*)h, name, n); }
void ho_stat_refresh(void* h) { ((Stat*)h)->refresh(); }
void ho_stat_poten(void* h) { ((Stat*)h)->poten(); }
void ho_stat_evolo0(void* h, double* mu, double* muerr, int n4) {
  ((Stat*)h)->evolo0(mu, muerr, n4);
}
void ho_stat_steprkr(void* h, double dt, double* mu, double* muerr, int n4) {
  ((Stat*)h)->steprkr(dt, mu, muerr, n4);
}
void ho_stat_steppcr(void* h, double dt, double* mu, double* muerr, int n4) {
  ((Stat*)h)->steppcr(dt, mu, muerr, n4);
}
double ho_stat_errpc(void* h) { return ((Stat*)h)->errpc; }
void ho_stat_energy(void* h, double* out) { ((Stat*)h)->energy(out); }
double ho_stat_varmu(void* h, int npart, double mu) { return ((Stat*)h)->varmu(npart, mu); }

// Quantum impurities.  he_x: n_imp rows of {kind, D, re, a, r_cutoff, umax}; x_x: n_imp^2 rows
// (i + n_imp*j), kind 0 = 'null'.
void* ho_qdyn_create(const ho_params* p, int n_imp, const double* m_imp_u, double mu4,
                     const double* he_x, const double* x_x, int nspline, int nq, int parabolic) {
  QDyn* d = new QDyn();
  d->init(*p, n_imp, m_imp_u, mu4, he_x, x_x, nspline, nq, parabolic);
  return d;
}
void ho_qdyn_destroy(void* h) { delete (QDyn*)h; }
double* ho_qdyn_field(void* h, const char* name, long* n) { return qdyn_field((QDyn*)h, name, n); }
void ho_qdyn_potenimp(void* h) { ((QDyn*)h)->potenimp(); }
void ho_qdyn_poten(void* h) { ((QDyn*)h)->poten(); }
void ho_qdyn_steprk(void* h, double dt) { ((QDyn*)h)->steprk(dt); }
void ho_qdyn_steppc(void* h, double dt, double* err2) { ((QDyn*)h)->steppc(dt, &err2[0], &err2[1]); }
void ho_qdyn_energy(void* h, double* out) { ((QDyn*)h)->energy(out); }
void ho_qdyn_moments(void* h, double* out) { ((QDyn*)h)->moments(out); }
void ho_qdyn_ring(void* h, int* r, int set) {
  QDyn* d = (QDyn*)h;
  int* dst[5] = {&d->ioldp[0], &d->ioldp[1], &d->ioldp[2], &d->ioldh[0], &d->ioldh[1]};
  for (int i = 0; i < 5; ++i) {
    if (set) *dst[i] = r[i];
    else r[i] = *dst[i];
  }
  for (int k = 0; k < d->ni; ++k) {
    for (int s = 0; s < 3; ++s) {
      if (set) d->ioldpx[3 * k + s] = r[s];
    }
    for (int s = 0; s < 2; ++s) {
      if (set) d->ioldhx[2 * k + s] = r[3 + s];
    }
  }
}
// Vpp(P_p(i)), i < n_p, of FT_V_spline for one pair potential (after the small-q redefinition),
// and the spline evaluation at arbitrary momenta.
int ho_ft_vpp_table(const double* pot, double pmax, double hp, int nspline, int parabolic,
                    double* vpp, int n_p) {
  PairPot v;
  v.kind = (int)pot[0]; v.D = pot[1]; v.re = pot[2]; v.a = pot[3]; v.rcut = pot[4]; v.umax = pot[5];
  FTVSpline t;
  t.build(v, pmax, hp, nspline, parabolic != 0);
  if (n_p != t.np) return t.np;
  std::memcpy(vpp, t.Vpp.data(), sizeof(double) * n_p);
  return n_p;
}
// One raw transform value (no small-q redefinition) at momentum p.
double ho_ft_vpp_point(const double* pot, double p, int nspline, int parabolic) {
  PairPot v;
  v.kind = (int)pot[0]; v.D = pot[1]; v.re = pot[2]; v.a = pot[3]; v.rcut = pot[4]; v.umax = pot[5];
  std::vector<double> x, a, b, c, d;
  FTVSpline::radial_spline(v, nspline, x, a, b, c, d);
  return FTVSpline::transform(p, v, parabolic != 0, x, a, b, c, d, nspline);
}
// The spline of mates.f (for tests against an independent spline).
void ho_spline(const double* x, const double* y, double s1, double sn, int n, double* a, double* b,
               double* c, double* d) {
  spline_maron(x, y, a, b, c, d, s1, sn, n);
}
int ho_findi(const double* x, double xc, int n) { return findi(x, xc, n); }
void ho_dyn_observables(void* h, int npart, double* out) {
  Dyn* d = (Dyn*)h;
  observables(d->g, d->p, d->w1, d->w2, d->psi, d->den, npart, out);
}
void ho_qdyn_observables(void* h, int npart, double* out) {
  QDyn* d = (QDyn*)h;
  observables(d->g, d->p, d->w1, d->w2, d->psi, d->den, npart, out);
}
}
