// ch3d_oracle.cpp -- CPU oracle for the Channel3d RK3 channel-flow step.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++ (FP64,
// -ffp-contract=off), the reference's Fortran algorithm for the time step of
// the channel solvers.  Only tests/, the smoke check and the CPU-baseline leg
// of bench.py load it, and only as a checker or as the timed CPU baseline;
// the product library never links or calls it.
//
// Parity status: UNPINNED against reference runs.  The reference is Fortran
// 2003 + MPI and no Fortran compiler exists on any machine of this build, and
// the reference ships no tests, golden vectors or fixtures.  The restatement
// is pinned instead by known-answer tests (naive DFT, discrete-Laplacian
// residual of the Poisson solve, Taylor-Green and Poiseuille states,
// divergence after projection) that live in tests/.
//
// Every routine cites the reference routine it follows (paths relative to the
// reference project).  Array conventions follow the reference: Fortran order
// (i fastest), ghosted arrays with the bounds of `myallocate`
// (src/CFD_2nd/m_Decomp2d.f90:1517-1583) for a single rank (y1start=1,
// y1end=n).  Only periodic x and z are supported (the channel configuration);
// y may be no-slip, free-slip, or periodic (clcU*Hat_FIMP_000 or
// clcU*Hat_PIMP_0, clcPPE_z1_periodic).
//
// The FFT that the reference takes from FFTW 3.3.9 (r2r kinds R2HC/HC2R,
// src/CFD_2nd/m_Poisson.f90:267-307) is restated from its definition
// (unnormalised DFT, halfcomplex storage r0..r_{n/2}, i_{(n+1)/2-1}..i_1).

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

// ---------------------------------------------------------------------------
// Field with arbitrary Fortran lower/upper bounds (column-major).
// ---------------------------------------------------------------------------
struct F3 {
  int xl = 0, yl = 0, zl = 0, sx = 0, sy = 0, sz = 0;
  std::vector<double> a;
  void init(int xl_, int xh, int yl_, int yh, int zl_, int zh) {
    xl = xl_; yl = yl_; zl = zl_;
    sx = xh - xl_ + 1; sy = yh - yl_ + 1; sz = zh - zl_ + 1;
    a.assign((size_t)sx * sy * sz, 0.0);
  }
  inline double& operator()(int i, int j, int k) {
    return a[(size_t)(i - xl) + (size_t)sx * ((size_t)(j - yl) + (size_t)sy * (size_t)(k - zl))];
  }
  inline double operator()(int i, int j, int k) const {
    return a[(size_t)(i - xl) + (size_t)sx * ((size_t)(j - yl) + (size_t)sy * (size_t)(k - zl))];
  }
};

// 1-D array addressed with Fortran indices lo..hi.
struct V1 {
  int lo = 0;
  std::vector<double> a;
  void init(int lo_, int hi) { lo = lo_; a.assign((size_t)(hi - lo_ + 1), 0.0); }
  inline double& operator()(int j) { return a[(size_t)(j - lo)]; }
  inline double operator()(int j) const { return a[(size_t)(j - lo)]; }
};

const double zero = 0.0, quarter = 0.25, half = 0.5, one = 1.0, two = 2.0,
             three = 3.0, four = 4.0;
const double PI = 3.141592653589793238462643383279502884;

// ---------------------------------------------------------------------------
// FFT: unnormalised complex DFT by recursive mixed-radix decimation in time,
// with twiddles from an exact table.  Used to restate FFTW's R2HC/HC2R.
// ---------------------------------------------------------------------------
struct FFTPlan {
  int n = 0;
  std::vector<cplx> w;  // w[q] = exp(-2 pi i q / n)
  std::vector<int> factors;
  void init(int n_) {
    n = n_;
    w.resize(n);
    for (int q = 0; q < n; ++q) {
      long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)q / (long double)n;
      w[q] = cplx((double)cosl(ang), (double)sinl(ang));
    }
    factors.clear();
    int m = n;
    const int pref[] = {4, 2, 3, 5};
    for (int f : pref) while (m % f == 0) { factors.push_back(f); m /= f; }
    for (int f = 7; m > 1; f += 2) while (m % f == 0) { factors.push_back(f); m /= f; }
  }
  // out[k] = sum_j in[j*stride] * exp(sign * 2 pi i j k / len); len = n / step
  void rec(const cplx* in, cplx* out, int len, int stride, int step, size_t fi, bool inv) const {
    if (len == 1) { out[0] = in[0]; return; }
    int p = factors[fi];
    int m = len / p;
    for (int r = 0; r < p; ++r) rec(in + (size_t)r * stride, out + (size_t)r * m, m, stride * p, step * p, fi + 1, inv);
    cplx tmpa[16], resa[16];
    std::vector<cplx> tmpv, resv;
    cplx* tmp = tmpa; cplx* res = resa;
    if (p > 16) { tmpv.resize(p); resv.resize(p); tmp = tmpv.data(); res = resv.data(); }
    for (int k = 0; k < m; ++k) {
      for (int r = 0; r < p; ++r) {
        int q = (int)(((long long)r * k * step) % n);
        cplx tw = inv ? std::conj(w[q]) : w[q];
        tmp[r] = out[(size_t)r * m + k] * tw;
      }
      for (int s = 0; s < p; ++s) {
        cplx acc = 0.0;
        for (int r = 0; r < p; ++r) {
          int q = (int)(((long long)r * s * m * step) % n);
          acc += tmp[r] * (inv ? std::conj(w[q]) : w[q]);
        }
        res[s] = acc;
      }
      for (int s = 0; s < p; ++s) out[(size_t)s * m + k] = res[s];
    }
  }
  void exec(const cplx* in, cplx* out, bool inv) const { rec(in, out, n, 1, 1, 0, inv); }
};

// FFTW_R2HC on a contiguous line (in place).  Halfcomplex output layout:
// hc[k] = Re X_k (k = 0..n/2), hc[n-k] = Im X_k (k = 1..(n+1)/2-1).
void r2hc(const FFTPlan& pl, double* x, std::vector<cplx>& bufa, std::vector<cplx>& bufb) {
  int n = pl.n;
  bufa.resize(n); bufb.resize(n);
  for (int j = 0; j < n; ++j) bufa[j] = cplx(x[j], 0.0);
  pl.exec(bufa.data(), bufb.data(), false);
  for (int k = 0; k <= n / 2; ++k) x[k] = bufb[k].real();
  for (int k = 1; k < (n + 1) / 2; ++k) x[n - k] = bufb[k].imag();
}

// FFTW_HC2R on a contiguous line (in place), unnormalised:
// x_j = sum_{k=0}^{n-1} X_k exp(+2 pi i j k / n) with Hermitian X.
void hc2r(const FFTPlan& pl, double* x, std::vector<cplx>& bufa, std::vector<cplx>& bufb) {
  int n = pl.n;
  bufa.resize(n); bufb.resize(n);
  bufa[0] = cplx(x[0], 0.0);
  for (int k = 1; k < (n + 1) / 2; ++k) {
    bufa[k] = cplx(x[k], x[n - k]);
    bufa[n - k] = std::conj(bufa[k]);
  }
  if (n % 2 == 0) bufa[n / 2] = cplx(x[n / 2], 0.0);
  pl.exec(bufa.data(), bufb.data(), true);
  for (int j = 0; j < n; ++j) x[j] = bufb[j].real();
}

// cos(pi m / (2n)), m = 0..4n-1: the angles of both cosine transforms of length n
std::vector<double> dct_table(int n) {
  std::vector<double> t((size_t)4 * n);
  for (int m = 0; m < 4 * n; ++m)
    t[m] = (double)std::cos(3.141592653589793238462643383279502884L * (long double)m / (long double)(2 * n));
  return t;
}

// FFTW_REDFT10 (DCT-II) on a contiguous line (in place), unnormalised:
// Y_k = 2 sum_{j=0}^{n-1} X_j cos(pi (j + 1/2) k / n), the reference's forward
// transform in a direction between walls (src/CFD_2nd/m_Poisson.f90:267-307).
void redft10(int n, double* x, const std::vector<double>& tab, std::vector<double>& buf) {
  buf.assign(x, x + n);
  for (int k = 0; k < n; ++k) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += buf[j] * tab[(size_t)(((long long)(2 * j + 1) * k) % (4 * n))];
    x[k] = 2.0 * s;
  }
}

// FFTW_REDFT01 (DCT-III), the inverse of REDFT10 up to the factor 2n:
// Y_k = X_0 + 2 sum_{j=1}^{n-1} X_j cos(pi j (k + 1/2) / n).
void redft01(int n, double* x, const std::vector<double>& tab, std::vector<double>& buf) {
  buf.assign(x, x + n);
  for (int k = 0; k < n; ++k) {
    double s = 0.0;
    for (int j = 1; j < n; ++j) s += buf[j] * tab[(size_t)(((long long)j * (2 * k + 1)) % (4 * n))];
    x[k] = buf[0] + 2.0 * s;
  }
}

}  // namespace

// ===========================================================================
// Public C interface
// ===========================================================================
extern "C" {

typedef struct orc_params {
  int order;          // 2 = src/CFD_2nd, 4 = src/CFD_4th
  int nxc, nyc, nzc;
  double xlx, yly, zlz;
  double xnu;
  double dtMax;
  int iCFL;
  double CFLc;
  int ischeme;        // 1 AB2, 2 RK2, 3 RK3
  int IsImplicit;     // 0 FEXP, 1 PIMP, 2 FIMP
  int FlowType;       // 1 channel, 2 half channel
  int BcOption[6];
  double uxBcValue[6], uyBcValue[6], uzBcValue[6];
  double gravity[3];
  int IsUxConst;
  double ubulk, ybulk1, ybulk2;
  int LES_type;       // 0 none, 2 WALE, 3 MTS, 10 Smagorinsky + van Driest
  int FilterType;
  double Cs;          // Smagorinsky constant (LES_type 10)
  double vel_limit, div_limit;
  // mesh sections (&MeshSection / &MeshOptions), at most 8
  int nSection;
  double SectionLength[8];
  double SectioncStret[8];
  int nycSection[8];
  int StretType[8];
  int StretOption[8];
} orc_params;

typedef struct orc_info {
  double SimTime, dt, cflmp, divmax1, divmax2, vmax[3], uxm, PrGradAver;
  int itime;
  int status;         // 0 ok, 1 divergence limit, 2 velocity limit
} orc_info;

}  // extern "C"

namespace {

struct Oracle {
  orc_params P;
  int nxc, nyc, nzc, nxp, nyp, nzp;
  int iadvance = 3;
  double pmGammaConst[3], pmThetaConst[3], pmAlphaConst[3];
  double pmGamma = 0, pmTheta = 0, pmAlpha = 0, pmBeta = 0, pmAlphaC = 0, pmBetaT = 0;
  double dt = 0, SimTime = 0, PrGradAver = 0, PrGradNow = 0;
  int itime = 0;
  double ybulk1 = 0, ybulk2 = 0;

  // metrics (m_MeshAndMetries)
  double dx, dy, dz, dx2, dy2, dz2, rdx, rdy, rdz, rdx2, rdy2, rdz2;
  V1 yp, yc, dyp, dyc, rdyp, rdyc, YinterpCoe, VolCell, DeltaCell;
  V1 ap2Pr, ac2Pr, am2Pr, am1c, ac1c, ap1c, am2c, ac2c, ap2c, am2p, ac2p, ap2p, am3c, ac3c, ap3c;
  V1 am2cForCN, ap2cForCN, am1cForCN, ap1cForCN, am3cForCN, ap3cForCN;

  // 4th-order solver (src/CFD_4th): stencil constants and CN metrics
  bool o4 = false;
  double dxCoe1, dxCoe2, dxCoe3, dxCoe4, dzCoe1, dzCoe2, dzCoe3, dzCoe4;
  double dxxCoe1, dxxCoe2, dxxCoe3, dxxCoe4, dxxCoe5, dzzCoe1, dzzCoe2, dzzCoe3, dzzCoe4, dzzCoe5;
  double InterpCoe1, InterpCoe2, InterpCoe3, InterpCoe4;
  const double uCRF = 0.0;  // IsUseCRF = F (src/CFD_4th/m_Parameters.f90:152-156)
  V1 ac2cForCN;
  F3 uxhx, uyhx, uzhx, uxhz, uyhz, uzhz;

  // Poisson
  V1 WaveNumX, WaveNumZ;
  double normfft = 1.0;
  FFTPlan planx, planz;

  // state (m_Variables)
  F3 ux, uy, uz, pressure, RealHalo, nut;
  F3 HistX, HistY, HistZ, RealArr1, RealArr2;  // interior (1:nxc,1:nyc,1:nzc)
  std::vector<double> uy_ym, duy_ym;           // (nxc,nzc)

  // statistics (m_FlowType_Channel)
  std::vector<double> SumStat;  // (35, nyp)
  std::vector<double> SumGrad;  // (98, nyp), 4th order (src/CFD_4th/m_FlowCase.f90:24-26)
  int nfstime = 0;
  double PrGradsum = 0;

  double divmax1_last = 0;

  int nthreads() const {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
  }

  // ---- src/CFD_2nd/m_MeshAndMetries.f90:292-360 (clcCoord) ----
  void clcCoord(int id1, int id2, double c1, double c2, int StretType, double cStret, int StretOption) {
    int m = id2 - id1;
    double secLen = c2 - c1;
    yp(id1) = c1; yp(id2) = c2;
    switch (StretType) {
      case 0:
        for (int j = 0; j <= m; ++j) yp(id1 + j) = c1 + (double)j / (double)m * secLen;
        break;
      case 1: {
        double tstr = std::tanh(cStret);
        for (int j = 0; j <= m; ++j) {
          double xi = (double)j / (double)(float)m;
          double setCrd = std::tanh(cStret * (xi - one)) / tstr + one;
          if (StretOption == 0) yp(id1 + j) = c1 + setCrd * secLen;
          else yp(id2 - j) = c2 - setCrd * secLen;
        }
        break;
      }
      case 2: {
        double tstr = std::sin(half * cStret * PI);
        for (int j = 0; j <= m; ++j) {
          double xi = (double)j / (double)m - one;
          double setCrd = std::sin(cStret * xi * PI * half) / tstr + one;
          if (StretOption == 0) yp(id1 + j) = c1 + setCrd * secLen;
          else yp(id2 - j) = c2 - setCrd * secLen;
        }
        break;
      }
      case 3: {
        if (cStret == one) {
          for (int j = 0; j <= m; ++j) yp(j + id1) = c1 + (double)j / (double)m * secLen;
        } else {
          double tstr = (std::pow(cStret, m) - one) / (cStret - one);
          for (int j = 0; j <= m - 1; ++j) {
            double setCrd = std::pow(cStret, j) / tstr;
            if (StretOption == 0) yp(id1 + j + 1) = yp(id1 + j) + setCrd * secLen;
            else yp(id2 - j - 1) = yp(id2 - j) - setCrd * secLen;
          }
        }
        break;
      }
    }
    yp(id1) = c1; yp(id2) = c2;
  }

  // ---- src/CFD_2nd/m_MeshAndMetries.f90:64-287 (InitMeshAndMetries) ----
  void InitMeshAndMetries() {
    dx = P.xlx / (double)nxc; dy = P.yly / (double)nyc; dz = P.zlz / (double)nzc;
    rdx = (double)nxc / P.xlx; rdy = (double)nyc / P.yly; rdz = (double)nzc / P.zlz;
    dx2 = dx * dx; rdx2 = rdx * rdx; dy2 = dy * dy; rdy2 = rdy * rdy; dz2 = dz * dz; rdz2 = rdz * rdz;
    yp.init(0, nyp); yc.init(0, nyp); dyp.init(0, nyp); rdyp.init(0, nyp); dyc.init(0, nyp); rdyc.init(0, nyp);
    ap2Pr.init(1, nyc); ac2Pr.init(1, nyc); am2Pr.init(1, nyc);
    ap1c.init(1, nxc); ac1c.init(1, nxc); am1c.init(1, nxc);
    ap2c.init(1, nyc); ac2c.init(1, nyc); am2c.init(1, nyc);
    ap2p.init(1, nyc); ac2p.init(1, nyc); am2p.init(1, nyc);
    ap3c.init(1, nzc); ac3c.init(1, nzc); am3c.init(1, nzc);
    VolCell.init(0, nyp); DeltaCell.init(0, nyp); YinterpCoe.init(1, nyp);

    int ns = P.nSection;
    std::vector<int> nid(ns + 1, 1);
    std::vector<double> ysc(ns + 1, 0.0);
    double SumLength = 0;
    for (int j = 0; j < ns; ++j) SumLength += P.SectionLength[j];
    for (int j = 0; j < ns; ++j) {
      nid[j + 1] = nid[j] + P.nycSection[j];
      ysc[j + 1] = ysc[j] + P.SectionLength[j] / SumLength * P.yly;
    }
    ysc[ns] = P.yly;
    for (int j = 0; j < ns; ++j)
      clcCoord(nid[j], nid[j + 1], ysc[j], ysc[j + 1], P.StretType[j], P.SectioncStret[j], P.StretOption[j]);

    for (int j = 1; j <= nyc; ++j) yc(j) = half * (yp(j) + yp(j + 1));
    yc(0) = two * yp(1) - yc(1);
    yc(nyp) = two * yp(nyp) - yc(nyc);
    for (int j = 1; j <= nyc; ++j) dyp(j) = yp(j + 1) - yp(j);
    dyp(0) = dyp(1); dyp(nyp) = dyp(nyc);
    for (int j = 0; j <= nyp; ++j) VolCell(j) = dyp(j) * dx * dz;
    for (int j = 0; j <= nyp; ++j) DeltaCell(j) = std::pow(dyp(j) * dx * dz, one / three);
    for (int j = 2; j <= nyc; ++j) dyc(j) = yc(j) - yc(j - 1);
    dyc(1) = dyp(1); dyc(nyp) = dyp(nyc);
    for (int j = 0; j <= nyp; ++j) rdyp(j) = one / dyp(j);
    for (int j = 1; j <= nyp; ++j) rdyc(j) = one / dyc(j);
    for (int j = 1; j <= nyp; ++j) YinterpCoe(j) = dyp(j) / (dyp(j) + dyp(j - 1));

    const int* Bc = P.BcOption;
    for (int j = 1; j <= nyc; ++j) { am2Pr(j) = rdyp(j) * rdyc(j); ap2Pr(j) = rdyp(j) * rdyc(j + 1); }
    if (Bc[2] != 0) { am2Pr(1) = zero; ap2Pr(1) = rdyp(1) * rdyc(2); }
    if (Bc[3] != 0) { am2Pr(nyc) = rdyp(nyc) * rdyc(nyc); ap2Pr(nyc) = zero; }
    for (int j = 1; j <= nyc; ++j) ac2Pr(j) = -(am2Pr(j) + ap2Pr(j));

    for (int i = 1; i <= nxc; ++i) { am1c(i) = rdx2; ap1c(i) = rdx2; }
    if (Bc[0] == -1) { am1c(1) = four / three * rdx2; ap1c(1) = four / three * rdx2; }
    if (Bc[1] == -1) { am1c(nxc) = four / three * rdx2; ap1c(nxc) = four / three * rdx2; }
    for (int i = 1; i <= nxc; ++i) ac1c(i) = -(am1c(i) + ap1c(i));

    for (int j = 1; j <= nyc; ++j) { am2c(j) = rdyp(j) * rdyc(j); ap2c(j) = rdyp(j) * rdyc(j + 1); }
    if (Bc[2] == -1) {
      am2c(1) = four * rdyc(1) / (dyc(1) + two * dyc(2));
      ap2c(1) = four * rdyc(2) / (dyc(1) + two * dyc(2));
    }
    if (Bc[3] == -1) {
      am2c(nyc) = four * rdyc(nyc) / (dyc(nyp) + two * dyc(nyc));
      ap2c(nyc) = four * rdyc(nyp) / (dyc(nyp) + two * dyc(nyc));
    }
    for (int j = 1; j <= nyc; ++j) ac2c(j) = -(am2c(j) + ap2c(j));

    for (int k = 1; k <= nzc; ++k) { am3c(k) = rdz2; ap3c(k) = rdz2; }
    if (Bc[4] == -1) { am3c(1) = four / three * rdz2; ap3c(1) = four / three * rdz2; }
    if (Bc[5] == -1) { am3c(nzc) = four / three * rdz2; ap3c(nzc) = four / three * rdz2; }
    for (int k = 1; k <= nzc; ++k) ac3c(k) = -(am3c(k) + ap3c(k));

    for (int j = 1; j <= nyc; ++j) { am2p(j) = rdyc(j) * rdyp(j - 1); ap2p(j) = rdyc(j) * rdyp(j); }
    for (int j = 1; j <= nyc; ++j) ac2p(j) = -(am2p(j) + ap2p(j));
  }

  // ---- src/CFD_2nd/m_TScheme.f90:40-100 (CN metrics of InitTimeScheme) ----
  void InitTimeScheme() {
    ybulk1 = P.ybulk1; ybulk2 = P.ybulk2;
    const int* Bc = P.BcOption;
    am1cForCN.init(1, nxc); ap1cForCN.init(1, nxc);
    for (int i = 1; i <= nxc; ++i) { ap1cForCN(i) = ap1c(i); am1cForCN(i) = am1c(i); }
    if (Bc[0] == -1) am1cForCN(1) = two * am1c(1); else if (Bc[0] == -2) am1cForCN(1) = zero;
    if (Bc[1] == -1) ap1cForCN(nxc) = two * ap1c(nxc); else if (Bc[1] == -2) ap1cForCN(nxc) = zero;
    am2cForCN.init(1, nyc); ap2cForCN.init(1, nyc);
    for (int j = 1; j <= nyc; ++j) { ap2cForCN(j) = ap2c(j); am2cForCN(j) = am2c(j); }
    if (Bc[2] == -1) am2cForCN(1) = two * am2c(1); else if (Bc[2] == -2) am2cForCN(1) = zero;
    if (Bc[3] == -1) ap2cForCN(nyc) = two * ap2c(nyc); else if (Bc[3] == -2) ap2cForCN(nyc) = zero;
    am3cForCN.init(1, nzc); ap3cForCN.init(1, nzc);
    for (int k = 1; k <= nzc; ++k) { ap3cForCN(k) = ap3c(k); am3cForCN(k) = am3c(k); }
    if (Bc[4] == -1) am3cForCN(1) = two * am3c(1); else if (Bc[4] == -2) am3cForCN(1) = zero;
    if (Bc[5] == -1) ap3cForCN(nzc) = two * ap3c(nzc); else if (Bc[5] == -2) ap3cForCN(nzc) = zero;
  }

  // ---- src/CFD_2nd/m_Poisson.f90:28-66 (modified wavenumbers, normfft) ----
  std::vector<double> zcos, xcos;  // cosine tables of the z and x transforms between walls
  void InitPoissonSolver() {
    WaveNumX.init(1, nxc); WaveNumZ.init(1, nzc);
    normfft = one;
    // x or z between walls: cosine transform, WaveCoe = pi, norm = 2 (:39-64)
    const double wcx = xper() ? 2.0 * PI : PI, nrmx = xper() ? one : two;
    for (int i = 1; i <= nxc; ++i) {
      double wa1 = wcx * (double)(i - 1) / (double)nxc;
      WaveNumX(i) = two * rdx2 * (std::cos(wa1) - one);
    }
    normfft = normfft * nrmx * (double)nxc;
    const double wcz = zper() ? 2.0 * PI : PI, nrmz = zper() ? one : two;
    for (int k = 1; k <= nzc; ++k) {
      double wa3 = wcz * (double)(k - 1) / (double)nzc;
      WaveNumZ(k) = two * rdz2 * (std::cos(wa3) - one);
    }
    normfft = normfft * nrmz * (double)nzc;
    normfft = one / normfft;
    planx.init(nxc);
    planz.init(nzc);
    if (!zper()) zcos = dct_table(nzc);
    if (!xper()) xcos = dct_table(nxc);
  }

  // ---- src/CFD_4th/m_MeshAndMetries.f90:86-91 (4th-order FD constants) ----
  void Init4thCoefficients() {
    dxCoe1 = rdx / 24.0; dxCoe2 = -rdx * 1.125; dxCoe3 = rdx * 1.125; dxCoe4 = -rdx / 24.0;
    dzCoe1 = rdz / 24.0; dzCoe2 = -rdz * 1.125; dzCoe3 = rdz * 1.125; dzCoe4 = -rdz / 24.0;
    dxxCoe1 = -rdx2 / 12.0; dxxCoe2 = 4.0 / 3.0 * rdx2; dxxCoe3 = -2.5 * rdx2; dxxCoe4 = 4.0 / 3.0 * rdx2; dxxCoe5 = -rdx2 / 12.0;
    dzzCoe1 = -rdz2 / 12.0; dzzCoe2 = 4.0 / 3.0 * rdz2; dzzCoe3 = -2.5 * rdz2; dzzCoe4 = 4.0 / 3.0 * rdz2; dzzCoe5 = -rdz2 / 12.0;
    InterpCoe1 = -1.0 / 16.0; InterpCoe2 = 9.0 / 16.0; InterpCoe3 = 9.0 / 16.0; InterpCoe4 = -1.0 / 16.0;
  }

  // ---- src/CFD_4th/m_TScheme.f90:35-51 (InitTimeScheme, CN metrics) ----
  void InitTimeScheme4() {
    am2cForCN.init(1, nyc); ac2cForCN.init(1, nyc); ap2cForCN.init(1, nyc);
    for (int j = 1; j <= nyc; ++j) { ap2cForCN(j) = ap2c(j); ac2cForCN(j) = ac2c(j); am2cForCN(j) = am2c(j); }
    ap2cForCN(1) = ap2c(1);
    ac2cForCN(1) = ac2c(1) - am2c(1);
    am2cForCN(1) = two * am2c(1);
    if (P.FlowType == 1) {
      am2cForCN(nyc) = am2c(nyc);
      ac2cForCN(nyc) = ac2c(nyc) - ap2c(nyc);
      ap2cForCN(nyc) = two * ap2c(nyc);
    }
  }

  void init(const orc_params* p) {
    P = *p;
    o4 = (P.order == 4);
    nxc = P.nxc; nyc = P.nyc; nzc = P.nzc; nxp = nxc + 1; nyp = nyc + 1; nzp = nzc + 1;
    // src/CFD_2nd/m_Parameters.f90:135-150 (ReadAndInitParameters: the time-scheme constants)
    if (P.ischeme == 1) {
      iadvance = 1;
      pmGammaConst[0] = 1.5; pmGammaConst[1] = 0; pmGammaConst[2] = 0;
      pmThetaConst[0] = -0.5; pmThetaConst[1] = 0; pmThetaConst[2] = 0;
    } else if (P.ischeme == 2) {
      iadvance = 2;
      pmGammaConst[0] = 0.5; pmGammaConst[1] = 1.0; pmGammaConst[2] = 0;
      pmThetaConst[0] = 0; pmThetaConst[1] = -0.5; pmThetaConst[2] = 0;
    } else {
      iadvance = 3;
      pmGammaConst[0] = 8.0 / 15.0; pmGammaConst[1] = 5.0 / 12.0; pmGammaConst[2] = 3.0 / 4.0;
      pmThetaConst[0] = 0.0; pmThetaConst[1] = -17.0 / 60.0; pmThetaConst[2] = -5.0 / 12.0;
    }
    for (int s = 0; s < 3; ++s) pmAlphaConst[s] = pmGammaConst[s] + pmThetaConst[s];
    InitMeshAndMetries();
    InitTimeScheme();
    InitPoissonSolver();
    if (o4) {
      Init4thCoefficients();
      InitTimeScheme4();
      // src/CFD_4th/m_Poisson.f90:40-47 (4th-order modified wavenumbers)
      for (int i = 1; i <= nxc; ++i) {
        double wa1 = 2.0 * PI * (double)(i - 1) / (double)nxc;
        WaveNumX(i) = rdx2 / 288.0 * (std::cos(three * wa1) - 54.0 * std::cos(two * wa1) + 783.0 * std::cos(wa1) - 730.0);
      }
      for (int k = 1; k <= nzc; ++k) {
        double wa3 = 2.0 * PI * (double)(k - 1) / (double)nzc;
        WaveNumZ(k) = rdz2 / 288.0 * (std::cos(three * wa3) - 54.0 * std::cos(two * wa3) + 783.0 * std::cos(wa3) - 730.0);
      }
      normfft = one / ((double)nxc * (double)nzc);
    }
    // ghosts: src/CFD_2nd/m_Variables.f90:59-61 (xme=1,xpe=2,...) or
    // src/CFD_4th/m_Variables.f90:47-49 (xme=2,xpe=2,yme=1,ype=1,zme=2,zpe=2)
    const int gx0 = o4 ? -1 : 0, gx1 = nxc + 2, gy1 = o4 ? nyc + 1 : nyc + 2, gz0 = o4 ? -1 : 0, gz1 = nzc + 2;
    ux.init(gx0, gx1, 0, gy1, gz0, gz1);
    uy.init(gx0, gx1, 0, gy1, gz0, gz1);
    uz.init(gx0, gx1, 0, gy1, gz0, gz1);
    pressure.init(gx0, gx1, 0, gy1, gz0, gz1);
    RealHalo.init(gx0, gx1, 0, gy1, gz0, gz1);
    nut.init(gx0, gx1, 0, gy1, gz0, gz1);
    if (o4) {
      uxhx.init(gx0, gx1, 0, gy1, gz0, gz1); uyhx.init(gx0, gx1, 0, gy1, gz0, gz1); uzhx.init(gx0, gx1, 0, gy1, gz0, gz1);
      uxhz.init(gx0, gx1, 0, gy1, gz0, gz1); uyhz.init(gx0, gx1, 0, gy1, gz0, gz1); uzhz.init(gx0, gx1, 0, gy1, gz0, gz1);
    }
    HistX.init(1, nxc, 1, nyc, 1, nzc); HistY.init(1, nxc, 1, nyc, 1, nzc); HistZ.init(1, nxc, 1, nyc, 1, nzc);
    RealArr1.init(1, nxc, 1, nyc, 1, nzc); RealArr2.init(1, nxc, 1, nyc, 1, nzc);
    uy_ym.assign((size_t)nxc * nzc, 0.0); duy_ym.assign((size_t)nxc * nzc, 0.0);
    SumStat.assign((size_t)35 * nyp, 0.0);
    dt = P.dtMax; SimTime = 0;
  }

  // ---- src/CFD_2nd/m_Parameters.f90:329-342 (PMcoeUpdate) ----
  void PMcoeUpdate(int ns) {
    pmGamma = pmGammaConst[ns - 1] * dt;
    pmTheta = pmThetaConst[ns - 1] * dt;
    pmAlpha = pmAlphaConst[ns - 1] * dt;
    pmBeta = half * pmAlphaConst[ns - 1] * P.xnu * dt;
    SimTime = SimTime + dt * pmAlphaConst[ns - 1];
    pmAlphaC = pmAlphaConst[ns - 1];
    pmBetaT = half * pmAlphaConst[ns - 1] * dt;
    if (ns == 1) PrGradAver = zero;
  }

  // ---- src/CFD_2nd/m_FlowType_Channel.f90:157-168 (Update_uy_ym_CH) ----
  void Update_uy_ym() {
    for (size_t q = 0; q < uy_ym.size(); ++q) {
      double old = uy_ym[q];
      uy_ym[q] = P.uyBcValue[2];
      duy_ym[q] = uy_ym[q] - old;
    }
  }

  // ---- src/CFD_2nd/m_Decomp2d.f90:1588-1743 (myupdate_halo, y-pencil, one rank,
  //      periodic x and z: self copies over the full extent of the other dims) ----
  void halo(F3& m, int xmh, int xph, int ymh, int yph, int zmh, int zph) {
    int xmm = m.xl, xpm = m.xl + m.sx - 1, ymm = m.yl, ypm = m.yl + m.sy - 1, zmm = m.zl, zpm = m.zl + m.sz - 1;
    // step1/2: y (only when y periodic)
    if (ymh > 0)
      for (int k = 1; k <= nzc; ++k) for (int h = 1; h <= ymh; ++h) for (int i = 1; i <= nxc; ++i)
        m(i, 1 - h, k) = m(i, nyc - h + 1, k);
    if (yph > 0)
      for (int k = 1; k <= nzc; ++k) for (int h = 1; h <= yph; ++h) for (int i = 1; i <= nxc; ++i)
        m(i, nyc + h, k) = m(i, h, k);
    // step3: receive from xm (i = 1-xmh..0  <- nxc-xmh+1..nxc)
    if (xmh > 0)
      for (int k = zmm; k <= zpm; ++k) for (int j = ymm; j <= ypm; ++j) for (int h = 1; h <= xmh; ++h)
        m(1 - h, j, k) = m(nxc - h + 1, j, k);
    if (xph > 0)
      for (int k = zmm; k <= zpm; ++k) for (int j = ymm; j <= ypm; ++j) for (int h = 1; h <= xph; ++h)
        m(nxc + h, j, k) = m(h, j, k);
    if (zmh > 0)
      for (int h = 1; h <= zmh; ++h) for (int j = ymm; j <= ypm; ++j) for (int i = xmm; i <= xpm; ++i)
        m(i, j, 1 - h) = m(i, j, nzc - h + 1);
    if (zph > 0)
      for (int h = 1; h <= zph; ++h) for (int j = ymm; j <= ypm; ++j) for (int i = xmm; i <= xpm; ++i)
        m(i, j, nzc + h) = m(i, j, h);
  }
  bool yper() const { return P.BcOption[2] == 0; }
  bool zper() const { return P.BcOption[4] == 0; }
  bool xper() const { return P.BcOption[0] == 0; }

  // ---- src/CFD_2nd/m_BC_and_Halo.f90:232-344 (SetBC_and_UpdateHalo), x and z
  //      periodic or between walls ----
  void SetBC_and_UpdateHalo() {
    const int* Bc = P.BcOption;
    if (Bc[3] == -1) {
      for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) {
        ux(i, nyp, k) = P.uxBcValue[3] * two - ux(i, nyc, k);
        uy(i, nyp, k) = P.uyBcValue[3];
        uy(i, nyp + 1, k) = P.uyBcValue[3] * two - uy(i, nyc, k);
        uz(i, nyp, k) = P.uzBcValue[3] * two - uz(i, nyc, k);
      }
    } else if (Bc[3] == -2) {
      for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) {
        ux(i, nyp, k) = P.uxBcValue[3] * dyp(nyp) + ux(i, nyc, k);
        uy(i, nyp, k) = P.uyBcValue[3];
        uy(i, nyp + 1, k) = P.uyBcValue[3] * two - uy(i, nyc, k);
        uz(i, nyp, k) = P.uzBcValue[3] * dyp(nyp) + uz(i, nyc, k);
      }
    }
    if (Bc[2] == -1) {
      for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) {
        double w = uy_ym[(size_t)(i - 1) + (size_t)nxc * (k - 1)];
        ux(i, 0, k) = P.uxBcValue[2] * two - ux(i, 1, k);
        uy(i, 1, k) = w;
        uy(i, 0, k) = w * two - uy(i, 2, k);
        uz(i, 0, k) = P.uzBcValue[2] * two - uz(i, 1, k);
      }
    } else if (Bc[2] == -2) {
      for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) {
        double w = uy_ym[(size_t)(i - 1) + (size_t)nxc * (k - 1)];
        ux(i, 0, k) = ux(i, 1, k) - P.uxBcValue[2] * dyp(1);
        uy(i, 1, k) = w;
        uy(i, 0, k) = w * two - uy(i, 2, k);
        uz(i, 0, k) = uz(i, 1, k) - P.uzBcValue[2] * dyp(1);
      }
    }
    // x walls (:285-311): ghost planes i = 0 and nxp over j = 0..nyp, k = 1..nzc;
    // ux's wall faces i = 1 and nxp hold the wall values
    if (Bc[1] == -1 || Bc[1] == -2) {
      const bool ns = Bc[1] == -1;
      for (int k = 1; k <= nzc; ++k) for (int j = 0; j <= nyp; ++j) {
        ux(nxp, j, k) = P.uxBcValue[1];
        ux(nxp + 1, j, k) = P.uxBcValue[1] * two - ux(nxc, j, k);
        uy(nxp, j, k) = ns ? P.uyBcValue[1] * two - uy(nxc, j, k) : uy(nxc, j, k) + P.uyBcValue[1] * dx;
        uz(nxp, j, k) = ns ? P.uzBcValue[1] * two - uz(nxc, j, k) : uz(nxc, j, k) + P.uzBcValue[1] * dx;
      }
    }
    if (Bc[0] == -1 || Bc[0] == -2) {
      const bool ns = Bc[0] == -1;
      for (int k = 1; k <= nzc; ++k) for (int j = 0; j <= nyp; ++j) {
        ux(1, j, k) = P.uxBcValue[0];
        ux(0, j, k) = P.uxBcValue[0] * two - ux(2, j, k);
        uy(0, j, k) = ns ? P.uyBcValue[0] * two - uy(1, j, k) : uy(1, j, k) - P.uyBcValue[0] * dx;
        uz(0, j, k) = ns ? P.uzBcValue[0] * two - uz(1, j, k) : uz(1, j, k) - P.uzBcValue[0] * dx;
      }
    }
    // z walls (:313-338): ghost planes k = 0 and nzp over i = 1..nxc, j = 0..nyp;
    // uz's wall faces k = 1 and nzp hold the wall values
    if (Bc[5] == -1 || Bc[5] == -2) {
      const bool ns = Bc[5] == -1;
      for (int j = 0; j <= nyp; ++j) for (int i = 1; i <= nxc; ++i) {
        ux(i, j, nzp) = ns ? P.uxBcValue[5] * two - ux(i, j, nzc) : ux(i, j, nzc) + P.uxBcValue[5] * dz;
        uy(i, j, nzp) = ns ? P.uyBcValue[5] * two - uy(i, j, nzc) : uy(i, j, nzc) + P.uyBcValue[5] * dz;
        uz(i, j, nzp) = P.uzBcValue[5];
        uz(i, j, nzp + 1) = P.uzBcValue[5] * two - uz(i, j, nzc);
      }
    }
    if (Bc[4] == -1 || Bc[4] == -2) {
      const bool ns = Bc[4] == -1;
      for (int j = 0; j <= nyp; ++j) for (int i = 1; i <= nxc; ++i) {
        ux(i, j, 0) = ns ? P.uxBcValue[4] * two - ux(i, j, 1) : ux(i, j, 1) - P.uxBcValue[4] * dz;
        uy(i, j, 0) = ns ? P.uyBcValue[4] * two - uy(i, j, 1) : uy(i, j, 1) - P.uyBcValue[4] * dz;
        uz(i, j, 1) = P.uzBcValue[4];
        uz(i, j, 0) = P.uzBcValue[4] * two - uz(i, j, 2);
      }
    }
    int xh = xper() ? 1 : 0, yh = yper() ? 1 : 0, zh = zper() ? 1 : 0;  // no halo copies across walls
    halo(ux, xh, xh, yh, yh, zh, zh);
    halo(uy, xh, xh, yh, yh, zh, zh);
    halo(uz, xh, xh, yh, yh, zh, zh);
  }

  // ---- src/CFD_2nd/m_BC_and_Halo.f90:349-405 (SetBC_and_UpdateHaloForPrSrc) ----
  void SetBC_and_UpdateHaloForPrSrc() {
    const int* Bc = P.BcOption;
    if (Bc[3] == -1 || Bc[3] == -2)
      for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) uy(i, nyp, k) = P.uyBcValue[3];
    if (Bc[2] == -1 || Bc[2] == -2)
      for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i)
        uy(i, 1, k) = uy_ym[(size_t)(i - 1) + (size_t)nxc * (k - 1)];
    if (Bc[1] == -1 || Bc[1] == -2)
      for (int k = 1; k <= nzc; ++k) for (int j = 0; j <= nyp; ++j) ux(nxp, j, k) = P.uxBcValue[1];
    if (Bc[0] == -1 || Bc[0] == -2)
      for (int k = 1; k <= nzc; ++k) for (int j = 0; j <= nyp; ++j) ux(1, j, k) = P.uxBcValue[0];
    if (Bc[5] == -1 || Bc[5] == -2)
      for (int j = 0; j <= nyp; ++j) for (int i = 1; i <= nxc; ++i) uz(i, j, nzp) = P.uzBcValue[5];
    if (Bc[4] == -1 || Bc[4] == -2)
      for (int j = 0; j <= nyp; ++j) for (int i = 1; i <= nxc; ++i) uz(i, j, 1) = P.uzBcValue[4];
    halo(ux, 0, xper() ? 1 : 0, 0, 0, 0, 0);
    halo(uy, 0, 0, 0, yper() ? 1 : 0, 0, 0);
    halo(uz, 0, 0, 0, 0, 0, zper() ? 1 : 0);
  }

  // ---- src/CFD_2nd/m_BC_and_Halo.f90:410-456 (SetBC_and_UpdateHalo_pr) ----
  void SetBC_and_UpdateHalo_pr(F3& pr) {
    const int* Bc = P.BcOption;
    if (Bc[3] < 0) for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) pr(i, nyp, k) = pr(i, nyc, k);
    if (Bc[2] < 0) for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) pr(i, 0, k) = pr(i, 1, k);
    if (Bc[1] < 0) for (int k = 1; k <= nzc; ++k) for (int j = 0; j <= nyp; ++j) pr(nxp, j, k) = pr(nxc, j, k);
    if (Bc[0] < 0) for (int k = 1; k <= nzc; ++k) for (int j = 0; j <= nyp; ++j) pr(0, j, k) = pr(1, j, k);
    if (Bc[5] < 0) for (int j = 0; j <= nyp; ++j) for (int i = 1; i <= nxc; ++i) pr(i, j, nzp) = pr(i, j, nzc);
    if (Bc[4] < 0) for (int j = 0; j <= nyp; ++j) for (int i = 1; i <= nxc; ++i) pr(i, j, 0) = pr(i, j, 1);
    int xh = xper() ? 1 : 0, yh = yper() ? 1 : 0, zh = zper() ? 1 : 0;
    halo(pr, xh, xh, yh, yh, zh, zh);
  }

  // ---- src/CFD_2nd/m_Tools.f90:21-46 (CalcMaxCFL) ----
  double CalcMaxCFL() {
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      double m = 0;
      for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) {
        double vcf = std::fabs(ux(ic, jc, kc) + ux(ic + 1, jc, kc)) * rdx +
                     std::fabs(uy(ic, jc, kc) + uy(ic, jc + 1, kc)) * rdyp(jc) +
                     std::fabs(uz(ic, jc, kc) + uz(ic, jc, kc + 1)) * rdz;
        if (vcf > m) m = vcf;
      }
      part[kc] = m;
    }
    double m = 0;
    for (int kc = 1; kc <= nzc; ++kc) m = std::max(m, part[kc]);
    return m * half;
  }

  // ---- src/CFD_2nd/m_Tools.f90:51-75 (CheckDivergence) ----
  double CheckDivergence() {
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      double m = 0;
      for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) {
        double udiv = std::fabs((ux(ic + 1, jc, kc) - ux(ic, jc, kc)) * rdx + (uy(ic, jc + 1, kc) - uy(ic, jc, kc)) * rdyp(jc) +
                                (uz(ic, jc, kc + 1) - uz(ic, jc, kc)) * rdz);
        if (udiv > m) m = udiv;
      }
      part[kc] = m;
    }
    double m = 0;
    for (int kc = 1; kc <= nzc; ++kc) m = std::max(m, part[kc]);
    return m;
  }

  // ---- src/CFD_2nd/m_Tools.f90:80-104 (CalcVmax) ----
  void CalcVmax(double v[3]) {
    v[0] = v[1] = v[2] = 0;
    for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) {
      v[0] = std::max(v[0], std::fabs(ux(ic, jc, kc)));
      v[1] = std::max(v[1], std::fabs(uy(ic, jc, kc)));
      v[2] = std::max(v[2], std::fabs(uz(ic, jc, kc)));
    }
  }

  // ---- src/CFD_2nd/m_Tools.f90:250-270 (CalcUxAver) ----
  double CalcUxAver() {
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      double s = 0;
      for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) s += ux(ic, jc, kc) * dyp(jc);
      part[kc] = s;
    }
    double s = 0;
    for (int kc = 1; kc <= nzc; ++kc) s += part[kc];
    return s / ((double)nxc * (double)nzc) / P.yly;
  }

  // ---- src/CFD_2nd/m_Tools.f90:218-245 (InverseTridiagonal), one system ----
  static void InverseTridiagonal1(const double* aj, const double* bj, const double* cj, double* fj, int n, double* arr) {
    double vecm = bj[0];
    fj[0] = fj[0] / vecm;
    for (int j = 1; j < n; ++j) {
      arr[j] = cj[j - 1] / vecm;
      vecm = bj[j] - aj[j] * arr[j];
      fj[j] = (fj[j] - aj[j] * fj[j - 1]) / vecm;
    }
    for (int j = n - 2; j >= 0; --j) fj[j] = fj[j] - arr[j + 1] * fj[j + 1];
  }

  // ---- src/CFD_2nd/m_Tools.f90:109-162 (InversePeriodicTridiagonal), one cyclic
  //      system (aj: sub, bj: diagonal, cj: super; aj[0] and cj[n-1] wrap) ----
  static void InversePeriodicTridiagonal1(const double* aj, const double* bj, const double* cj, double* fj, int n,
                                          double* a1, double* a2, double* a3) {
    a1[0] = -cj[0] / bj[0];
    a2[0] = -aj[0] / bj[0];
    fj[0] = fj[0] / bj[0];
    for (int j = 1; j <= n - 2; ++j) {
      double ppj = one / (bj[j] + aj[j] * a1[j - 1]);
      a1[j] = -cj[j] * ppj;
      a2[j] = -aj[j] * a2[j - 1] * ppj;
      fj[j] = (fj[j] - aj[j] * fj[j - 1]) * ppj;
    }
    a2[n - 1] = one;
    a3[n - 1] = zero;
    for (int j = n - 2; j >= 0; --j) {
      a2[j] = a2[j] + a1[j] * a2[j + 1];
      a3[j] = fj[j] + a1[j] * a3[j + 1];
    }
    fj[n - 1] = (fj[n - 1] - cj[n - 1] * a3[0] - aj[n - 1] * a3[n - 2]) /
                (cj[n - 1] * a2[0] + aj[n - 1] * a2[n - 2] + bj[n - 1]);
    for (int j = n - 2; j >= 0; --j) fj[j] = fj[n - 1] * a2[j] + a3[j];
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:7-75 (clcRhsX_PIMP); scheme 2: the
  //      same loop is clcRhsX_FIMP (src/CFD_2nd/m_TSchemeFIMP_inc.f90:6-67): no
  //      explicit viscous term in convEd1, 2*pmBeta*(d11+d22+d33) instead;
  //      scheme 0: clcRhsX_FEXP (src/CFD_2nd/m_TSchemeFEXP_inc.f90:6-75), the
  //      whole viscous term in convEd1 and no pmBeta term ----
  void clcRhsX_PIMP(F3& RhsX, F3& Hist, int scheme = 1) {
    const bool fimp = scheme == 2, fexp = scheme == 0;
    double qdx1 = quarter * rdx, qdx3 = quarter * rdz;
    std::vector<double> part(nzc + 1, 0.0);
    const double g1 = P.gravity[0], xnu = P.xnu;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1;
      double s1tot = 0;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double s1totCoe = dyp(jc);
        double sucaj = half * rdyp(jc);
        if (yc(jc) < ybulk1 || yc(jc) >= ybulk2) s1totCoe = zero;
        double InterpY1 = YinterpCoe(jc), InterpY2 = one - InterpY1;
        double InterpY3 = YinterpCoe(jp), InterpY4 = one - InterpY3;
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1;
          double h11 = ((ux(ip, jc, kc) + ux(ic, jc, kc)) * (ux(ip, jc, kc) + ux(ic, jc, kc)) -
                        (ux(ic, jc, kc) + ux(im, jc, kc)) * (ux(ic, jc, kc) + ux(im, jc, kc))) * qdx1;
          double h12 = ((uy(ic, jp, kc) + uy(im, jp, kc)) * (InterpY3 * ux(ic, jc, kc) + InterpY4 * ux(ic, jp, kc)) -
                        (uy(ic, jc, kc) + uy(im, jc, kc)) * (InterpY1 * ux(ic, jm, kc) + InterpY2 * ux(ic, jc, kc))) * sucaj;
          double h13 = ((uz(ic, jc, kp) + uz(im, jc, kp)) * (ux(ic, jc, kp) + ux(ic, jc, kc)) -
                        (uz(ic, jc, kc) + uz(im, jc, kc)) * (ux(ic, jc, kc) + ux(ic, jc, km))) * qdx3;
          double d11q1 = (ux(ip, jc, kc) - two * ux(ic, jc, kc) + ux(im, jc, kc)) * rdx2;
          double d22q1 = ap2c(jc) * ux(ic, jp, kc) + ac2c(jc) * ux(ic, jc, kc) + am2c(jc) * ux(ic, jm, kc);
          double d33q1 = ap3c(kc) * ux(ic, jc, kp) + ac3c(kc) * ux(ic, jc, kc) + am3c(kc) * ux(ic, jc, km);
          double dcq13 = d11q1 + d33q1;
          double gradp1 = (pressure(ic, jc, kc) - pressure(im, jc, kc)) * rdx;
          s1tot = s1tot + ux(ic, jc, kc) * s1totCoe;
          double convEd1, dcn;
          if (fimp) { convEd1 = -h11 - h12 - h13 + g1; dcn = d11q1 + d22q1 + d33q1; }
          else { convEd1 = -h11 - h12 - h13 + xnu * dcq13 + g1; dcn = d22q1; }
          if (fexp) {  // clcRhsX_FEXP: the whole viscous term explicit
            convEd1 = -h11 - h12 - h13 + xnu * (d11q1 + d22q1 + d33q1) + g1;
            RhsX(ic, jc, kc) = pmGamma * convEd1 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp1;
          } else
          RhsX(ic, jc, kc) = pmGamma * convEd1 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp1 + two * pmBeta * dcn;
          Hist(ic, jc, kc) = convEd1;
        }
      }
      part[kc] = s1tot;
    }
    if (P.IsUxConst) {
      double s1tot1 = 0;
      for (int kc = 1; kc <= nzc; ++kc) s1tot1 += part[kc];
      s1tot1 = s1tot1 / ((double)nxc * (double)nzc) / (ybulk2 - ybulk1);
      double dpmdxns = pmAlphaC * (P.ubulk - s1tot1);
#pragma omp parallel for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) RhsX(ic, jc, kc) = RhsX(ic, jc, kc) + dpmdxns;
      PrGradNow = (P.ubulk - s1tot1) / dt;
      PrGradAver = PrGradAver + pmAlphaC * PrGradNow;
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:161-209 (clcRhsY_PIMP); fimp:
  //      clcRhsY_FIMP (src/CFD_2nd/m_TSchemeFIMP_inc.f90:72-119) ----
  void clcRhsY_PIMP(F3& RhsY, F3& Hist, int scheme = 1) {
    const bool fimp = scheme == 2, fexp = scheme == 0;
    double hdx1 = half * rdx, hdx3 = half * rdz;
    const double g2 = P.gravity[1], xnu = P.xnu;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double sucac = rdyc(jc), qsucac = quarter * sucac;
        double InterpY1 = YinterpCoe(jc), InterpY2 = one - InterpY1;
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1;
          double h21 = ((InterpY1 * ux(ip, jm, kc) + InterpY2 * ux(ip, jc, kc)) * (uy(ip, jc, kc) + uy(ic, jc, kc)) -
                        (InterpY1 * ux(ic, jm, kc) + InterpY2 * ux(ic, jc, kc)) * (uy(ic, jc, kc) + uy(im, jc, kc))) * hdx1;
          double h22 = ((uy(ic, jp, kc) + uy(ic, jc, kc)) * (uy(ic, jp, kc) + uy(ic, jc, kc)) -
                        (uy(ic, jc, kc) + uy(ic, jm, kc)) * (uy(ic, jc, kc) + uy(ic, jm, kc))) * qsucac;
          double h23 = ((InterpY1 * uz(ic, jm, kp) + InterpY2 * uz(ic, jc, kp)) * (uy(ic, jc, kp) + uy(ic, jc, kc)) -
                        (InterpY1 * uz(ic, jm, kc) + InterpY2 * uz(ic, jc, kc)) * (uy(ic, jc, kc) + uy(ic, jc, km))) * hdx3;
          double d11q2 = ap1c(ic) * uy(ip, jc, kc) + ac1c(ic) * uy(ic, jc, kc) + am1c(ic) * uy(im, jc, kc);
          double d22q2 = ap2p(jc) * uy(ic, jp, kc) + ac2p(jc) * uy(ic, jc, kc) + am2p(jc) * uy(ic, jm, kc);
          double d33q2 = ap3c(kc) * uy(ic, jc, kp) + ac3c(kc) * uy(ic, jc, kc) + am3c(kc) * uy(ic, jc, km);
          double dcq13 = d11q2 + d33q2;
          double gradp2 = (pressure(ic, jc, kc) - pressure(ic, jm, kc)) * sucac;
          double convEd2, dcn;
          if (fimp) { convEd2 = -h21 - h22 - h23 + g2; dcn = d11q2 + d22q2 + d33q2; }
          else { convEd2 = -h21 - h22 - h23 + xnu * dcq13 + g2; dcn = d22q2; }
          if (fexp) {  // clcRhsY_FEXP: the whole viscous term explicit
            convEd2 = -h21 - h22 - h23 + xnu * (d11q2 + d22q2 + d33q2) + g2;
            RhsY(ic, jc, kc) = pmGamma * convEd2 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp2;
          } else
          RhsY(ic, jc, kc) = pmGamma * convEd2 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp2 + two * pmBeta * dcn;
          Hist(ic, jc, kc) = convEd2;
        }
      }
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:277-325 (clcRhsZ_PIMP); RhsZ is the
  //      ghosted RealHalo in the reference, only its interior is written; fimp:
  //      clcRhsZ_FIMP (src/CFD_2nd/m_TSchemeFIMP_inc.f90:124-177) ----
  void clcRhsZ_PIMP(F3& RhsZ, F3& Hist, int scheme = 1) {
    const bool fimp = scheme == 2, fexp = scheme == 0;
    double qdx1 = quarter * rdx, qdx3 = quarter * rdz;
    const double g3 = P.gravity[2], xnu = P.xnu;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double sucaj = half * rdyp(jc);
        double InterpY1 = YinterpCoe(jc), InterpY2 = one - InterpY1;
        double InterpY3 = YinterpCoe(jp), InterpY4 = one - InterpY3;
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1;
          double h31 = ((ux(ip, jc, kc) + ux(ip, jc, km)) * (uz(ip, jc, kc) + uz(ic, jc, kc)) -
                        (ux(ic, jc, kc) + ux(ic, jc, km)) * (uz(ic, jc, kc) + uz(im, jc, kc))) * qdx1;
          double h32 = ((uy(ic, jp, kc) + uy(ic, jp, km)) * (InterpY3 * uz(ic, jc, kc) + InterpY4 * uz(ic, jp, kc)) -
                        (uy(ic, jc, kc) + uy(ic, jc, km)) * (InterpY1 * uz(ic, jm, kc) + InterpY2 * uz(ic, jc, kc))) * sucaj;
          double h33 = ((uz(ic, jc, kp) + uz(ic, jc, kc)) * (uz(ic, jc, kp) + uz(ic, jc, kc)) -
                        (uz(ic, jc, kc) + uz(ic, jc, km)) * (uz(ic, jc, kc) + uz(ic, jc, km))) * qdx3;
          double d11q3 = ap1c(ic) * uz(ip, jc, kc) + ac1c(ic) * uz(ic, jc, kc) + am1c(ic) * uz(im, jc, kc);
          double d22q3 = ap2c(jc) * uz(ic, jp, kc) + ac2c(jc) * uz(ic, jc, kc) + am2c(jc) * uz(ic, jm, kc);
          double d33q3 = (uz(ic, jc, kp) - two * uz(ic, jc, kc) + uz(ic, jc, km)) * rdz2;
          double dcq13 = d11q3 + d33q3;
          double gradp3 = (pressure(ic, jc, kc) - pressure(ic, jc, km)) * rdz;
          double convEd3, dcn;
          if (fimp) { convEd3 = -h31 - h32 - h33 + g3; dcn = d11q3 + d22q3 + d33q3; }
          else { convEd3 = -h31 - h32 - h33 + xnu * dcq13 + g3; dcn = d22q3; }
          if (fexp) {  // clcRhsZ_FEXP: the whole viscous term explicit
            convEd3 = -h31 - h32 - h33 + xnu * (d11q3 + d22q3 + d33q3) + g3;
            RhsZ(ic, jc, kc) = pmGamma * convEd3 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp3;
          } else
          RhsZ(ic, jc, kc) = pmGamma * convEd3 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp3 + two * pmBeta * dcn;
          Hist(ic, jc, kc) = convEd3;
        }
      }
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:392-430 (clcU1Hat_PIMP) and :702-740
  //      (clcU3Hat_PIMP): (I - pmBeta*L_y) du = Rhs, u += du, per k-slab ----
  void clcUHat_PIMP_c(F3& u, F3& Rhs) {
    std::vector<double> tp(nyc), tm(nyc), tc(nyc);
    for (int jc = 1; jc <= nyc; ++jc) {
      tp[jc - 1] = -pmBeta * ap2cForCN(jc);
      tm[jc - 1] = -pmBeta * am2cForCN(jc);
      tc[jc - 1] = -tp[jc - 1] - tm[jc - 1] + one;
    }
#pragma omp parallel
    {
      std::vector<double> f(nyc), arr(nyc);
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int jc = 1; jc <= nyc; ++jc) f[jc - 1] = Rhs(ic, jc, kc);
          InverseTridiagonal1(tm.data(), tc.data(), tp.data(), f.data(), nyc, arr.data());
          for (int jc = 1; jc <= nyc; ++jc) u(ic, jc, kc) = u(ic, jc, kc) + f[jc - 1];
        }
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:542-589 (clcU2Hat_PIMP) ----
  void clcU2Hat_PIMP(F3& Rhs) {
    std::vector<double> tp(nyc), tm(nyc), tc(nyc);
    tp[0] = zero; tc[0] = one; tm[0] = zero;
    for (int jc = 2; jc <= nyc; ++jc) {
      tp[jc - 1] = -pmBeta * ap2p(jc);
      tc[jc - 1] = -pmBeta * ac2p(jc) + one;
      tm[jc - 1] = -pmBeta * am2p(jc);
    }
#pragma omp parallel
    {
      std::vector<double> f(nyc), arr(nyc);
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int ic = 1; ic <= nxc; ++ic) {
          f[0] = duy_ym[(size_t)(ic - 1) + (size_t)nxc * (kc - 1)];
          for (int jc = 2; jc <= nyc; ++jc) f[jc - 1] = Rhs(ic, jc, kc);
          InverseTridiagonal1(tm.data(), tc.data(), tp.data(), f.data(), nyc, arr.data());
          for (int jc = 1; jc <= nyc; ++jc) uy(ic, jc, kc) = uy(ic, jc, kc) + f[jc - 1];
        }
    }
  }

  // ---- src/CFD_2nd/m_Tools.f90:167-219 (InversePTriFixedCoe), one periodic
  //      system with constant coefficients (a: sub, b: diagonal, c: super),
  //      values f[q*stride], q = 0..n-1 ----
  static void InversePTriFixedCoe1(double ajf, double bjf, double cjf, double* fj, int n, long long stride,
                                   std::vector<double>& ppj, std::vector<double>& vecn1, std::vector<double>& vecn2,
                                   std::vector<double>& arrmn) {
    // Fortran index j = 1..n maps to element j-1
    ppj.assign(n + 1, 0.0); vecn1.assign(n + 1, 0.0); vecn2.assign(n + 1, 0.0); arrmn.assign(n + 1, 0.0);
    auto F = [&](int j) -> double& { return fj[(long long)(j - 1) * stride]; };
    vecn1[1] = -cjf / bjf;
    vecn2[1] = -ajf / bjf;
    vecn2[n] = one;
    for (int j = 2; j <= n - 1; ++j) {
      ppj[j] = one / (bjf + ajf * vecn1[j - 1]);
      vecn1[j] = -cjf * ppj[j];
      vecn2[j] = -ajf * vecn2[j - 1] * ppj[j];
    }
    for (int j = n - 1; j >= 1; --j) vecn2[j] = vecn2[j] + vecn1[j] * vecn2[j + 1];
    F(1) = F(1) / bjf;
    for (int j = 2; j <= n - 1; ++j) F(j) = (F(j) - ajf * F(j - 1)) * ppj[j];
    arrmn[n] = zero;
    for (int j = n - 1; j >= 1; --j) arrmn[j] = F(j) + vecn1[j] * arrmn[j + 1];
    F(n) = (F(n) - cjf * arrmn[1] - ajf * arrmn[n - 1]) / (cjf * vecn2[1] + ajf * vecn2[n - 1] + bjf);
    for (int j = n - 1; j >= 1; --j) F(j) = F(n) * vecn2[j] + arrmn[j];
  }

  // ---- src/CFD_2nd/m_TSchemeFIMP_inc.f90:263-347 (clcU1Hat_FIMP_010), :636-729
  //      (clcU2Hat_FIMP_010), :1035-1128 (clcU3Hat_FIMP_010): periodic x sweep,
  //      periodic z sweep (constant coefficients), then the y sweep of the PIMP
  //      solvers.  The transposes of the reference only move data. ----
  void clcUHat_FIMP_xz(F3& Rhs) {
    const double mic = -pmBeta * rdx2, pic = -pmBeta * rdx2, cic = pmBeta * rdx2 * two + one;
    const double mkc = -pmBeta * rdz2, pkc = -pmBeta * rdz2, ckc = pmBeta * rdz2 * two + one;
#pragma omp parallel
    {
      std::vector<double> a, b, c, d, line(std::max(nxc, nzc));
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int jc = 1; jc <= nyc; ++jc) {
          for (int ic = 1; ic <= nxc; ++ic) line[ic - 1] = Rhs(ic, jc, kc);
          InversePTriFixedCoe1(mic, cic, pic, line.data(), nxc, 1, a, b, c, d);
          for (int ic = 1; ic <= nxc; ++ic) Rhs(ic, jc, kc) = line[ic - 1];
        }
    }
#pragma omp parallel
    {
      std::vector<double> a, b, c, d, line(std::max(nxc, nzc));
#pragma omp for schedule(static)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int kc = 1; kc <= nzc; ++kc) line[kc - 1] = Rhs(ic, jc, kc);
          InversePTriFixedCoe1(mkc, ckc, pkc, line.data(), nzc, 1, a, b, c, d);
          for (int kc = 1; kc <= nzc; ++kc) Rhs(ic, jc, kc) = line[kc - 1];
        }
    }
  }

  // ---- the periodic x sweep alone (src/CFD_2nd/m_TSchemeFIMP_inc.f90:375-393 of
  //      clcU1Hat_FIMP_011, :758-776 and :1165-1183 of the uy and uz routines) ----
  void clcUHat_FIMP_x(F3& Rhs) {
    const double mic = -pmBeta * rdx2, pic = -pmBeta * rdx2, cic = pmBeta * rdx2 * two + one;
#pragma omp parallel
    {
      std::vector<double> a, b, c, d, line(nxc);
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int jc = 1; jc <= nyc; ++jc) {
          for (int ic = 1; ic <= nxc; ++ic) line[ic - 1] = Rhs(ic, jc, kc);
          InversePTriFixedCoe1(mic, cic, pic, line.data(), nxc, 1, a, b, c, d);
          for (int ic = 1; ic <= nxc; ++ic) Rhs(ic, jc, kc) = line[ic - 1];
        }
    }
  }

  // ---- the x sweep between walls (clcU1/2/3Hat_FIMP_111, src/CFD_2nd/
  //      m_TSchemeFIMP_inc.f90:476-507, 868-890, 1286-1308): uy and uz with the
  //      Crank-Nicolson wall metrics am1cForCN / ap1cForCN, ux with constant
  //      coefficients and its wall face i = 1 held.  The reference accepts walls
  //      in x only together with walls in z (m_TScheme.f90:111-113). ----
  void clcUHat_FIMP_xwall(F3& Rhs, bool uxface) {
    std::vector<double> tm(nxc), tc(nxc), tp(nxc);
    for (int ic = 1; ic <= nxc; ++ic) {
      if (uxface) {
        tm[ic - 1] = -pmBeta * rdx2; tp[ic - 1] = -pmBeta * rdx2; tc[ic - 1] = pmBeta * rdx2 * two + one;
      } else {
        tp[ic - 1] = -pmBeta * ap1cForCN(ic);
        tm[ic - 1] = -pmBeta * am1cForCN(ic);
        tc[ic - 1] = -tp[ic - 1] - tm[ic - 1] + one;
      }
    }
    if (uxface) { tp[0] = zero; tc[0] = one; tm[0] = zero; }
#pragma omp parallel
    {
      std::vector<double> f(nxc), arr(nxc);
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int jc = 1; jc <= nyc; ++jc) {
          for (int ic = 1; ic <= nxc; ++ic) f[ic - 1] = Rhs(ic, jc, kc);
          if (uxface) f[0] = zero;
          InverseTridiagonal1(tm.data(), tc.data(), tp.data(), f.data(), nxc, arr.data());
          for (int ic = 1; ic <= nxc; ++ic) Rhs(ic, jc, kc) = f[ic - 1];
        }
    }
  }

  // ---- the z sweep between walls: ux and uy (src/CFD_2nd/m_TSchemeFIMP_inc.f90:
  //      395-417, and :778-800 of clcU2Hat_FIMP_011) with the Crank-Nicolson wall
  //      metrics am3cForCN / ap3cForCN; uz (:1185-1218 of clcU3Hat_FIMP_011) with
  //      constant coefficients and its wall face k = 1 held (row 1 = identity, zero
  //      right-hand side) ----
  void clcUHat_FIMP_zwall(F3& Rhs, bool uzface) {
    std::vector<double> tm(nzc), tc(nzc), tp(nzc);
    for (int kc = 1; kc <= nzc; ++kc) {
      if (uzface) {
        tm[kc - 1] = -pmBeta * rdz2; tp[kc - 1] = -pmBeta * rdz2; tc[kc - 1] = pmBeta * rdz2 * two + one;
      } else {
        tp[kc - 1] = -pmBeta * ap3cForCN(kc);
        tm[kc - 1] = -pmBeta * am3cForCN(kc);
        tc[kc - 1] = -tp[kc - 1] - tm[kc - 1] + one;
      }
    }
    if (uzface) { tp[0] = zero; tc[0] = one; tm[0] = zero; }
#pragma omp parallel
    {
      std::vector<double> f(nzc), arr(nzc);
#pragma omp for schedule(static)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int kc = 1; kc <= nzc; ++kc) f[kc - 1] = Rhs(ic, jc, kc);
          if (uzface) f[0] = zero;
          InverseTridiagonal1(tm.data(), tc.data(), tp.data(), f.data(), nzc, arr.data());
          for (int kc = 1; kc <= nzc; ++kc) Rhs(ic, jc, kc) = f[kc - 1];
        }
    }
  }

  // ---- src/CFD_2nd/m_TSchemeFIMP_inc.f90:241-257 (the y sweep of clcU1Hat_FIMP_000;
  //      :614-630 and :1013-1029 for uy and uz) and src/CFD_2nd/m_TSchemePIMP_inc.f90:
  //      435-461, 594-621, 745-771 (clcU1/2/3Hat_PIMP_0): periodic y, constant
  //      coefficients, u = u + the solution ----
  void clcUHat_y_periodic(F3& u, F3& Rhs) {
    const double mjc = -pmBeta * rdy2, pjc = -pmBeta * rdy2, cjc = pmBeta * rdy2 * two + one;
#pragma omp parallel
    {
      std::vector<double> a, b, c, d, line(nyc);
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int jc = 1; jc <= nyc; ++jc) line[jc - 1] = Rhs(ic, jc, kc);
          InversePTriFixedCoe1(mjc, cjc, pjc, line.data(), nyc, 1, a, b, c, d);
          for (int jc = 1; jc <= nyc; ++jc) u(ic, jc, kc) = u(ic, jc, kc) + line[jc - 1];
        }
    }
  }

  // ---- src/CFD_2nd/m_TScheme.f90:245-276 (clcPrSrc_FIMP): clcPrSrcOther plus
  //      pressure += -xnu/2 * div ----
  double clcPrSrc_FIMP(F3& prsrc) {
    double sudtal = one / pmAlpha, xnuhm = -half * P.xnu;
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int kp = kc + 1;
      double m = 0;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jp = jc + 1;
        double sucaj = rdyp(jc);
        for (int ic = 1; ic <= nxc; ++ic) {
          int ip = ic + 1;
          double rdiv = (ux(ip, jc, kc) - ux(ic, jc, kc)) * rdx + (uy(ic, jp, kc) - uy(ic, jc, kc)) * sucaj +
                        (uz(ic, jc, kp) - uz(ic, jc, kc)) * rdz;
          m = std::max(std::fabs(rdiv), m);
          prsrc(ic, jc, kc) = sudtal * rdiv;
          pressure(ic, jc, kc) = pressure(ic, jc, kc) + xnuhm * rdiv;
        }
      }
      part[kc] = m;
    }
    double m = 0;
    for (int kc = 1; kc <= nzc; ++kc) m = std::max(m, part[kc]);
    return m;
  }

  // ---- src/CFD_2nd/m_TSchemeFEXP_inc.f90:391-488 (clcU1/2/3Hat_FEXP): u = u + Rhs ----
  void clcUHat_FEXP(F3& u, F3& Rhs) {
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) u(ic, jc, kc) = u(ic, jc, kc) + Rhs(ic, jc, kc);
  }

  // ---- src/CFD_2nd/m_TSchemeFIMP_inc.f90:1371-1386 (PressureUpdate_FIMP), and
  //      src/CFD_2nd/m_TSchemeFEXP_inc.f90:513-528 (PressureUpdate_FEXP, the same) ----
  void PressureUpdate_FIMP(const F3& phi) {
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) pressure(ic, jc, kc) = pressure(ic, jc, kc) + phi(ic, jc, kc);
  }


  // =====================================================================
  // LES (src/CFD_2nd/m_LESModels.f90 and the *_PIMP_LES procedures of
  // src/CFD_2nd/m_TSchemePIMP_inc.f90); nut includes the molecular xnu
  // =====================================================================
  double utau_last = 0;

  // ---- src/CFD_2nd/m_LESModels.f90:72-135 (Clc_SGS_WALE) ----
  void Clc_SGS_WALE() {
    const double Cw_ = 0.325, xnu = P.xnu;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jp = jc + 1, jm = jc - 1;
        double caj = rdyp(jc), cac1 = rdyc(jc), cac2 = rdyc(jp), cac12 = cac1 - cac2;
        double CwDelta2 = Cw_ * DeltaCell(jc);
        CwDelta2 = CwDelta2 * CwDelta2;
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1;
          double dudx = (ux(ip, jc, kc) - ux(ic, jc, kc)) * rdx;
          double dudy = ((ux(ip, jp, kc) + ux(ic, jp, kc)) * cac2 + (ux(ip, jc, kc) + ux(ic, jc, kc)) * cac12 -
                         (ux(ip, jm, kc) + ux(ic, jm, kc)) * cac1) * 0.25;
          double dudz = (ux(ip, jc, kp) + ux(ic, jc, kp) - ux(ip, jc, km) - ux(ic, jc, km)) * rdz * 0.25;
          double dvdx = (uy(ip, jp, kc) - uy(im, jp, kc) + uy(ip, jc, kc) - uy(im, jc, kc)) * rdx * 0.25;
          double dvdy = (uy(ic, jp, kc) - uy(ic, jc, kc)) * caj;
          double dvdz = (uy(ic, jp, kp) + uy(ic, jc, kp) - uy(ic, jp, km) - uy(ic, jc, km)) * rdz * 0.25;
          double dwdx = (uz(ip, jc, kp) - uz(im, jc, kp) + uz(ip, jc, kc) - uz(im, jc, kc)) * rdx * 0.25;
          double dwdy = ((uz(ic, jp, kp) + uz(ic, jp, kc)) * cac2 + (uz(ic, jc, kp) + uz(ic, jc, kc)) * cac12 -
                         (uz(ic, jm, kp) + uz(ic, jm, kc)) * cac1) * 0.25;
          double dwdz = (uz(ic, jc, kp) - uz(ic, jc, kc)) * rdz;
          double S11 = dudx, S12 = (dudy + dvdx) * half, S13 = (dudz + dwdx) * half;
          double S22 = dvdy, S23 = (dvdz + dwdy) * half, S33 = dwdz;
          double SijSij = S11 * S11 + S22 * S22 + S33 * S33 + two * (S12 * S12 + S13 * S13 + S23 * S23);
          double Sd11 = dudx * dudx + dudy * dvdx + dudz * dwdx;
          double Sd12 = (dudx * dudy + dudy * dvdy + dudz * dwdy + dvdx * dudx + dvdy * dvdx + dvdz * dwdx) * half;
          double Sd13 = (dudx * dudz + dudy * dvdz + dudz * dwdz + dwdx * dudx + dwdy * dvdx + dwdz * dwdx) * half;
          double Sd22 = dvdx * dudy + dvdy * dvdy + dvdz * dwdy;
          double Sd23 = (dvdx * dudz + dvdy * dvdz + dvdz * dwdz + dwdx * dudy + dwdy * dvdy + dwdz * dwdy) * half;
          double Sd33 = dwdx * dudz + dwdy * dvdz + dwdz * dwdz;
          double SdTrace = (Sd11 + Sd22 + Sd33) / three;
          Sd11 = Sd11 - SdTrace; Sd22 = Sd22 - SdTrace; Sd33 = Sd33 - SdTrace;
          double SdijSdij = Sd11 * Sd11 + Sd22 * Sd22 + Sd33 * Sd33 + two * (Sd12 * Sd12 + Sd13 * Sd13 + Sd23 * Sd23);
          nut(ic, jc, kc) = CwDelta2 * std::pow(SdijSdij, 1.5) / (std::pow(SijSij, 2.5) + std::pow(SdijSdij, 1.25)) + xnu;
        }
      }
    }
  }

  // ---- src/CFD_2nd/m_LESModels.f90:328-370 (ClcVelStrainRate): |S| = sqrt(2 Sij Sij);
  // the same sum without the root is CalcDissipationRate (src/CFD_2nd/m_Tools.f90:497-540) ----
  double StrainRate(int ic, int jc, int kc) { return std::sqrt(StrainRate2(ic, jc, kc)); }
  double StrainRate2(int ic, int jc, int kc) {
    int ip = ic + 1, im = ic - 1, jp = jc + 1, jm = jc - 1, kp = kc + 1, km = kc - 1;
    double caj = rdyp(jc), cac1 = rdyc(jc), cac2 = rdyc(jp), cac12 = cac1 - cac2;
    const double oneEighth = 0.125;
    double st1 = (ux(ip, jc, kc) - ux(ic, jc, kc)) * rdx;
    double st2 = (uy(ic, jp, kc) - uy(ic, jc, kc)) * caj;
    double st3 = (uz(ic, jc, kp) - uz(ic, jc, kc)) * rdz;
    double st4 = oneEighth * ((uy(ip, jp, kc) - uy(im, jp, kc) + uy(ip, jc, kc) - uy(im, jc, kc)) * rdx +
                              (ux(ip, jp, kc) + ux(ic, jp, kc)) * cac2 + (ux(ip, jc, kc) + ux(ic, jc, kc)) * cac12 -
                              (ux(ip, jm, kc) + ux(ic, jm, kc)) * cac1);
    double st5 = oneEighth * ((ux(ip, jc, kp) + ux(ic, jc, kp) - ux(ip, jc, km) - ux(ic, jc, km)) * rdz +
                              (uz(ip, jc, kp) - uz(im, jc, kp) + uz(ip, jc, kc) - uz(im, jc, kc)) * rdx);
    double st6 = oneEighth * ((uy(ic, jp, kp) + uy(ic, jc, kp) - uy(ic, jp, km) - uy(ic, jc, km)) * rdz +
                              (uz(ic, jp, kp) + uz(ic, jp, kc)) * cac2 + (uz(ic, jc, kp) + uz(ic, jc, kc)) * cac12 -
                              (uz(ic, jm, kp) + uz(ic, jm, kc)) * cac1);
    return two * (st1 * st1 + st2 * st2 + st3 * st3) + four * (st4 * st4 + st5 * st5 + st6 * st6);
  }

  // ---- src/CFD_2nd/m_FlowType_TGVortex.f90:87-113 (clcStat_TG): xnu * sum(dissp) / (nxc nyc nzc) ----
  double TGDissipation() {
    SetBC_and_UpdateHalo();
    double sumr = 0.0;
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) sumr += StrainRate2(ic, jc, kc);
    return P.xnu * sumr / ((double)nxc * (double)nyc * (double)nzc);
  }

  // ---- src/CFD_2nd/m_LESModels.f90:145-258 (Clc_SGS_MTS), filter from InitFilterCoe :35-41 ----
  void Clc_SGS_MTS() {
    double Fc[9];
    if (P.FilterType == 1) { const double f[9] = {1, 4, 1, 4, 16, 4, 1, 4, 1}; for (int q = 0; q < 9; ++q) Fc[q] = f[q] / 36.0; }
    else { const double f[9] = {1, 2, 1, 2, 4, 2, 1, 2, 1}; for (int q = 0; q < 9; ++q) Fc[q] = f[q] / 16.0; }
    F3 Ktemp;
    Ktemp.init(ux.xl, ux.xl + ux.sx - 1, ux.yl, ux.yl + ux.sy - 1, ux.zl, ux.zl + ux.sz - 1);
    std::vector<double> Kes((size_t)nxc * nyc * nzc, 0.0);
    auto K = [&](int i, int j, int k) -> double& { return Kes[(size_t)(i - 1) + (size_t)nxc * ((size_t)(j - 1) + (size_t)nyc * (k - 1))]; };
    auto filt = [&](F3& u, int ic, int jc, int kc) {
      int im = ic - 1, ip = ic + 1, km = kc - 1, kp = kc + 1;
      return Fc[0] * u(im, jc, km) + Fc[1] * u(ic, jc, km) + Fc[2] * u(ip, jc, km) +
             Fc[3] * u(im, jc, kc) + (Fc[4] - one) * u(ic, jc, kc) + Fc[5] * u(ip, jc, kc) +
             Fc[6] * u(im, jc, kp) + Fc[7] * u(ic, jc, kp) + Fc[8] * u(ip, jc, kp);
    };
    for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) {
      double f = filt(ux, ic, jc, kc); Ktemp(ic, jc, kc) = f * f;
    }
    halo(Ktemp, 0, 1, 0, 0, 0, 0);
    for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic)
      K(ic, jc, kc) = half * (Ktemp(ic, jc, kc) + Ktemp(ic + 1, jc, kc));
    for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyp; ++jc) for (int ic = 1; ic <= nxc; ++ic) {
      double f = filt(uy, ic, jc, kc); Ktemp(ic, jc, kc) = f * f;
    }
    for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic)
      K(ic, jc, kc) = K(ic, jc, kc) + half * (Ktemp(ic, jc, kc) + Ktemp(ic, jc + 1, kc));
    for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) {
      double f = filt(uz, ic, jc, kc); Ktemp(ic, jc, kc) = f * f;
    }
    halo(Ktemp, 0, 0, 0, 0, 0, 1);
    for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic)
      K(ic, jc, kc) = K(ic, jc, kc) + half * (Ktemp(ic, jc, kc) + Ktemp(ic, jc, kc + 1));
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc) {
        double rdelta = one / DeltaCell(jc);
        for (int ic = 1; ic <= nxc; ++ic) {
          double Ksgs = K(ic, jc, kc);
          double Ts = std::sqrt(Ksgs) * rdelta + StrainRate(ic, jc, kc) / 10.0;
          if (Ts < 1.0e-10) Ts = zero; else Ts = one / Ts;
          nut(ic, jc, kc) = 0.05 * Ksgs * Ts + P.xnu;
        }
      }
  }

  // Smagorinsky with van Driest damping (LES_type 10; not in the reference,
  // whose LES_type 1 branch is empty): nut = xnu + (Cs D Delta)^2 |S|,
  // D = 1 - exp(-y+/26), y+ = d_wall u_tau / xnu, u_tau from the x-z mean
  // wall shear of the first cells of both walls, |S| from ClcVelStrainRate.
  double WallUtau() {
    double s1 = 0, sN = 0;
    for (int kc = 1; kc <= nzc; ++kc) for (int ic = 1; ic <= nxc; ++ic) { s1 += ux(ic, 1, kc); sN += ux(ic, nyc, kc); }
    const double inxz = one / ((double)nxc * (double)nzc);
    const double d1 = yc(1) - yp(1), dN = yp(nyp) - yc(nyc);
    const double tw = P.xnu * half * (std::fabs(s1 * inxz - P.uxBcValue[2]) / d1 + std::fabs(sN * inxz - P.uxBcValue[3]) / dN);
    return std::sqrt(tw);
  }
  void Clc_SGS_SmagVD() {
    const double utau = WallUtau();
    utau_last = utau;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc) {
        const double dw = std::min(yc(jc) - yp(1), yp(nyp) - yc(jc));
        const double D = one - std::exp(-(dw * utau / P.xnu) / 26.0);
        const double l = P.Cs * D * DeltaCell(jc);
        for (int ic = 1; ic <= nxc; ++ic) nut(ic, jc, kc) = l * l * StrainRate(ic, jc, kc) + P.xnu;
      }
  }

  // ---- src/CFD_2nd/m_LESModels.f90:375-428 (SetBC_and_UpdateHalo_SGS), channel ----
  void SetBC_and_UpdateHalo_SGS() {
    const double xnu = P.xnu;
    for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) {
      if (P.BcOption[3] == -1) nut(i, nyp, k) = two * xnu - nut(i, nyc, k);
      else if (P.BcOption[3] == -2) nut(i, nyp, k) = nut(i, nyc, k);
      if (P.BcOption[2] == -1) nut(i, 0, k) = two * xnu - nut(i, 1, k);
      else if (P.BcOption[2] == -2) nut(i, 0, k) = nut(i, 1, k);
    }
    halo(nut, 1, 1, 0, 0, 1, 1);
  }

  // ---- src/CFD_2nd/m_LESModels.f90:47-62 (Clc_SGS_Vis) ----
  void Clc_SGS_Vis() {
    if (P.LES_type == 2) Clc_SGS_WALE();
    else if (P.LES_type == 3) Clc_SGS_MTS();
    else if (P.LES_type == 10) Clc_SGS_SmagVD();
    else if (P.LES_type == 11) {  // learned closure: molecular viscosity, explicit stress force
      for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic)
        nut(ic, jc, kc) = P.xnu;
    }
    SetBC_and_UpdateHalo_SGS();
  }

  // Learned closure (no counterpart in the reference; the discretisation of
  // channel3d_b200/csrc/ch3d_les.cu k_sgs_force): the force -d tau_ij/dx_j of
  // cell-centred stresses set by the test (sgs_tau, 6 interior arrays) at the
  // staggered velocity points; off-diagonal stresses averaged onto the cell
  // edges from the four neighbouring cells, zero on the walls.
  std::vector<double> sgs_tau, sgs_f;
  void SgsForce() {
    const size_t N = (size_t)nxc * nyc * nzc;
    sgs_f.assign(3 * N, 0.0);
    if (sgs_tau.size() != 6 * N) return;
    auto T = [&](int q, int i, int j, int k) {  // periodic i, k; 1-based
      i = (i - 1 + nxc) % nxc; k = (k - 1 + nzc) % nzc;
      return sgs_tau[q * N + (size_t)i + (size_t)nxc * ((size_t)(j - 1) + (size_t)nyc * k)];
    };
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) {
          const int im = ic - 1, ip = ic + 1, km = kc - 1, kp = kc + 1, jm = jc - 1, jp = jc + 1;
          const size_t o = (size_t)(ic - 1) + (size_t)nxc * ((size_t)(jc - 1) + (size_t)nyc * (kc - 1));
          // x momentum at (i-1/2, j, k)
          double t12u = jc == nyc ? 0.0 : 0.25 * (T(1, im, jc, kc) + T(1, ic, jc, kc) + T(1, im, jp, kc) + T(1, ic, jp, kc));
          double t12d = jc == 1 ? 0.0 : 0.25 * (T(1, im, jm, kc) + T(1, ic, jm, kc) + T(1, im, jc, kc) + T(1, ic, jc, kc));
          double t13p = 0.25 * (T(2, im, jc, kc) + T(2, ic, jc, kc) + T(2, im, jc, kp) + T(2, ic, jc, kp));
          double t13m = 0.25 * (T(2, im, jc, km) + T(2, ic, jc, km) + T(2, im, jc, kc) + T(2, ic, jc, kc));
          sgs_f[o] = -((T(0, ic, jc, kc) - T(0, im, jc, kc)) * rdx + (t12u - t12d) * rdyp(jc) + (t13p - t13m) * rdz);
          // y momentum at (i, j-1/2, k); the wall row is fixed by the wall condition
          if (jc > 1) {
            double t12p = 0.25 * (T(1, ic, jm, kc) + T(1, ip, jm, kc) + T(1, ic, jc, kc) + T(1, ip, jc, kc));
            double t12m = 0.25 * (T(1, im, jm, kc) + T(1, ic, jm, kc) + T(1, im, jc, kc) + T(1, ic, jc, kc));
            double t23p = 0.25 * (T(4, ic, jm, kc) + T(4, ic, jm, kp) + T(4, ic, jc, kc) + T(4, ic, jc, kp));
            double t23m = 0.25 * (T(4, ic, jm, km) + T(4, ic, jm, kc) + T(4, ic, jc, km) + T(4, ic, jc, kc));
            sgs_f[N + o] = -((t12p - t12m) * rdx + (T(3, ic, jc, kc) - T(3, ic, jm, kc)) * rdyc(jc) + (t23p - t23m) * rdz);
          }
          // z momentum at (i, j, k-1/2)
          double t13p2 = 0.25 * (T(2, ic, jc, km) + T(2, ip, jc, km) + T(2, ic, jc, kc) + T(2, ip, jc, kc));
          double t13m2 = 0.25 * (T(2, im, jc, km) + T(2, ic, jc, km) + T(2, im, jc, kc) + T(2, ic, jc, kc));
          double t23u = jc == nyc ? 0.0 : 0.25 * (T(4, ic, jc, km) + T(4, ic, jc, kc) + T(4, ic, jp, km) + T(4, ic, jp, kc));
          double t23d = jc == 1 ? 0.0 : 0.25 * (T(4, ic, jm, km) + T(4, ic, jm, kc) + T(4, ic, jc, km) + T(4, ic, jc, kc));
          sgs_f[2 * N + o] = -((t13p2 - t13m2) * rdx + (t23u - t23d) * rdyp(jc) + (T(5, ic, jc, kc) - T(5, ic, jc, km)) * rdz);
        }
  }
  double sgsf(int q, int ic, int jc, int kc) const {
    if (sgs_f.empty()) return 0.0;
    const size_t N = (size_t)nxc * nyc * nzc;
    return sgs_f[q * N + (size_t)(ic - 1) + (size_t)nxc * ((size_t)(jc - 1) + (size_t)nyc * (kc - 1))];
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:80-156 (clcRhsX_PIMP_LES); fexp:
  //      src/CFD_2nd/m_TSchemeFEXP_inc.f90:80-155 (clcRhsX_FEXP_LES), the y
  //      viscous term inside convEd1 and no pmBetaT term ----
  void clcRhsX_PIMP_LES(F3& RhsX, F3& Hist, bool fexp = false) {
    double qdx1 = quarter * rdx, qdx3 = quarter * rdz;
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1;
      double s1tot = 0;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double s1totCoe = dyp(jc), sucaj = quarter * rdyp(jc);
        if (yc(jc) < ybulk1 || yc(jc) >= ybulk2) s1totCoe = zero;
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1;
          double h11 = ((ux(ip, jc, kc) + ux(ic, jc, kc)) * (ux(ip, jc, kc) + ux(ic, jc, kc)) -
                        (ux(ic, jc, kc) + ux(im, jc, kc)) * (ux(ic, jc, kc) + ux(im, jc, kc))) * qdx1;
          double h12 = ((uy(ic, jp, kc) + uy(im, jp, kc)) * (ux(ic, jp, kc) + ux(ic, jc, kc)) -
                        (uy(ic, jc, kc) + uy(im, jc, kc)) * (ux(ic, jc, kc) + ux(ic, jm, kc))) * sucaj;
          double h13 = ((uz(ic, jc, kp) + uz(im, jc, kp)) * (ux(ic, jc, kp) + ux(ic, jc, kc)) -
                        (uz(ic, jc, kc) + uz(im, jc, kc)) * (ux(ic, jc, kc) + ux(ic, jc, km))) * qdx3;
          double visa = quarter * (nut(ic, jc, kc) + nut(im, jc, kc) + nut(ic, jm, kc) + nut(im, jm, kc));
          double visb = quarter * (nut(ic, jc, kc) + nut(im, jc, kc) + nut(ic, jp, kc) + nut(im, jp, kc));
          double visc = quarter * (nut(ic, jc, kc) + nut(im, jc, kc) + nut(ic, jc, km) + nut(im, jc, km));
          double visd = quarter * (nut(ic, jc, kc) + nut(im, jc, kc) + nut(ic, jc, kp) + nut(im, jc, kp));
          double sgs1 = rdx2 * (nut(ic, jc, kc) * (ux(ip, jc, kc) - ux(ic, jc, kc)) - nut(im, jc, kc) * (ux(ic, jc, kc) - ux(im, jc, kc)));
          double sgs2 = rdx * rdyp(jc) * (visb * (uy(ic, jp, kc) - uy(im, jp, kc)) - visa * (uy(ic, jc, kc) - uy(im, jc, kc)));
          double sgs3 = rdx * rdz * (visd * (uz(ic, jc, kp) - uz(im, jc, kp)) - visc * (uz(ic, jc, kc) - uz(im, jc, kc)));
          double d11q1 = sgs1;
          double d22q1 = ap2c(jc) * visb * (ux(ic, jp, kc) - ux(ic, jc, kc)) - am2c(jc) * visa * (ux(ic, jc, kc) - ux(ic, jm, kc));
          double d33q1 = ap3c(kc) * visd * (ux(ic, jc, kp) - ux(ic, jc, kc)) - am3c(kc) * visc * (ux(ic, jc, kc) - ux(ic, jc, km));
          double dcq13 = fexp ? d11q1 + d22q1 + d33q1 : d11q1 + d33q1;
          double gradp1 = (pressure(ic, jc, kc) - pressure(im, jc, kc)) * rdx;
          s1tot = s1tot + ux(ic, jc, kc) * s1totCoe;
          double convEd1 = -h11 - h12 - h13 + sgs1 + sgs2 + sgs3 + dcq13 + P.gravity[0] + sgsf(0, ic, jc, kc);
          RhsX(ic, jc, kc) = pmGamma * convEd1 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp1;
          if (!fexp) RhsX(ic, jc, kc) = RhsX(ic, jc, kc) + two * pmBetaT * d22q1;
          Hist(ic, jc, kc) = convEd1;
        }
      }
      part[kc] = s1tot;
    }
    if (P.IsUxConst) {
      double s1tot1 = 0;
      for (int kc = 1; kc <= nzc; ++kc) s1tot1 += part[kc];
      s1tot1 = s1tot1 / ((double)nxc * (double)nzc) / (ybulk2 - ybulk1);
      double dpmdxns = pmAlphaC * (P.ubulk - s1tot1);
#pragma omp parallel for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) RhsX(ic, jc, kc) = RhsX(ic, jc, kc) + dpmdxns;
      PrGradNow = (P.ubulk - s1tot1) / dt;
      PrGradAver = PrGradAver + pmAlphaC * PrGradNow;
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:214-272 (clcRhsY_PIMP_LES) ----
  void clcRhsY_PIMP_LES(F3& RhsY, F3& Hist, bool fexp = false) {
    double qdx1 = quarter * rdx, qdx3 = quarter * rdz;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double sucac = rdyc(jc), qsucac = quarter * sucac;
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1;
          double h21 = ((ux(ip, jc, kc) + ux(ip, jm, kc)) * (uy(ip, jc, kc) + uy(ic, jc, kc)) -
                        (ux(ic, jc, kc) + ux(ic, jm, kc)) * (uy(ic, jc, kc) + uy(im, jc, kc))) * qdx1;
          double h22 = ((uy(ic, jp, kc) + uy(ic, jc, kc)) * (uy(ic, jp, kc) + uy(ic, jc, kc)) -
                        (uy(ic, jc, kc) + uy(ic, jm, kc)) * (uy(ic, jc, kc) + uy(ic, jm, kc))) * qsucac;
          double h23 = ((uz(ic, jc, kp) + uz(ic, jm, kp)) * (uy(ic, jc, kp) + uy(ic, jc, kc)) -
                        (uz(ic, jc, kc) + uz(ic, jm, kc)) * (uy(ic, jc, kc) + uy(ic, jc, km))) * qdx3;
          double visa = quarter * (nut(ic, jc, kc) + nut(im, jc, kc) + nut(ic, jm, kc) + nut(im, jm, kc));
          double visb = quarter * (nut(ic, jc, kc) + nut(ip, jc, kc) + nut(ic, jm, kc) + nut(ip, jm, kc));
          double visc = quarter * (nut(ic, jc, kc) + nut(ic, jm, kc) + nut(ic, jc, km) + nut(ic, jm, km));
          double visd = quarter * (nut(ic, jc, kc) + nut(ic, jm, kc) + nut(ic, jc, kp) + nut(ic, jm, kp));
          double sgs1 = rdx * sucac * (visb * (ux(ip, jc, kc) - ux(ip, jm, kc)) - visa * (ux(ic, jc, kc) - ux(ic, jm, kc)));
          double sgs2 = ap2p(jc) * nut(ic, jc, kc) * (uy(ic, jp, kc) - uy(ic, jc, kc)) - am2p(jc) * nut(ic, jm, kc) * (uy(ic, jc, kc) - uy(ic, jm, kc));
          double sgs3 = rdz * sucac * (visd * (uz(ic, jc, kp) - uz(ic, jm, kp)) - visc * (uz(ic, jc, kc) - uz(ic, jm, kc)));
          double d11q2 = ap1c(ic) * visb * (uy(ip, jc, kc) - uy(ic, jc, kc)) - am1c(ic) * visa * (uy(ic, jc, kc) - uy(im, jc, kc));
          double d22q2 = sgs2;
          double d33q2 = ap3c(kc) * visd * (uy(ic, jc, kp) - uy(ic, jc, kc)) - am3c(kc) * visc * (uy(ic, jc, kc) - uy(ic, jc, km));
          double dcq13 = fexp ? d11q2 + d22q2 + d33q2 : d11q2 + d33q2;
          double gradp2 = (pressure(ic, jc, kc) - pressure(ic, jm, kc)) * sucac;
          double convEd2 = -h21 - h22 - h23 + sgs1 + sgs2 + sgs3 + dcq13 + P.gravity[1] + sgsf(1, ic, jc, kc);
          RhsY(ic, jc, kc) = pmGamma * convEd2 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp2;
          if (!fexp) RhsY(ic, jc, kc) = RhsY(ic, jc, kc) + two * pmBetaT * d22q2;
          Hist(ic, jc, kc) = convEd2;
        }
      }
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:330-387 (clcRhsZ_PIMP_LES) ----
  void clcRhsZ_PIMP_LES(F3& RhsZ, F3& Hist, bool fexp = false) {
    double qdx1 = quarter * rdx, qdx3 = quarter * rdz;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double sucaj = quarter * rdyp(jc);
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1;
          double h31 = ((ux(ip, jc, kc) + ux(ip, jc, km)) * (uz(ip, jc, kc) + uz(ic, jc, kc)) -
                        (ux(ic, jc, kc) + ux(ic, jc, km)) * (uz(ic, jc, kc) + uz(im, jc, kc))) * qdx1;
          double h32 = ((uy(ic, jp, kc) + uy(ic, jp, km)) * (uz(ic, jp, kc) + uz(ic, jc, kc)) -
                        (uy(ic, jc, kc) + uy(ic, jc, km)) * (uz(ic, jc, kc) + uz(ic, jm, kc))) * sucaj;
          double h33 = ((uz(ic, jc, kp) + uz(ic, jc, kc)) * (uz(ic, jc, kp) + uz(ic, jc, kc)) -
                        (uz(ic, jc, kc) + uz(ic, jc, km)) * (uz(ic, jc, kc) + uz(ic, jc, km))) * qdx3;
          double visa = quarter * (nut(ic, jc, km) + nut(im, jc, km) + nut(ic, jc, kc) + nut(im, jc, kc));
          double visb = quarter * (nut(ic, jc, km) + nut(ip, jc, km) + nut(ic, jc, kc) + nut(ip, jc, kc));
          double visc = quarter * (nut(ic, jc, km) + nut(ic, jm, km) + nut(ic, jm, kc) + nut(ic, jc, kc));
          double visd = quarter * (nut(ic, jc, km) + nut(ic, jp, km) + nut(ic, jp, kc) + nut(ic, jc, kc));
          double sgs1 = rdx * rdz * (visb * (ux(ip, jc, kc) - ux(ip, jc, km)) - visa * (ux(ic, jc, kc) - ux(ic, jc, km)));
          double sgs2 = rdz * rdyp(jc) * (visd * (uy(ic, jp, kc) - uy(ic, jp, km)) - visc * (uy(ic, jc, kc) - uy(ic, jc, km)));
          double sgs3 = rdz2 * (nut(ic, jc, kc) * (uz(ic, jc, kp) - uz(ic, jc, kc)) - nut(ic, jc, km) * (uz(ic, jc, kc) - uz(ic, jc, km)));
          double d11q3 = ap1c(ic) * visb * (uz(ip, jc, kc) - uz(ic, jc, kc)) - am1c(ic) * visa * (uz(ic, jc, kc) - uz(im, jc, kc));
          double d22q3 = ap2c(jc) * visd * (uz(ic, jp, kc) - uz(ic, jc, kc)) - am2c(jc) * visc * (uz(ic, jc, kc) - uz(ic, jm, kc));
          double d33q3 = sgs3;
          double dcq13 = fexp ? d11q3 + d22q3 + d33q3 : d11q3 + d33q3;
          double gradp3 = (pressure(ic, jc, kc) - pressure(ic, jc, km)) * rdz;
          double convEd3 = -h31 - h32 - h33 + sgs1 + sgs2 + sgs3 + dcq13 + P.gravity[2] + sgsf(2, ic, jc, kc);
          RhsZ(ic, jc, kc) = pmGamma * convEd3 + pmTheta * Hist(ic, jc, kc) - pmAlpha * gradp3;
          if (!fexp) RhsZ(ic, jc, kc) = RhsZ(ic, jc, kc) + two * pmBetaT * d22q3;
          Hist(ic, jc, kc) = convEd3;
        }
      }
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:466-499, 626-662, 776-809
  //      (clcU1/2/3Hat_PIMP_LES): variable-coefficient y Crank-Nicolson ----
  void clcUHat_PIMP_LES(int comp, F3& u, F3& Rhs) {
#pragma omp parallel
    {
      std::vector<double> a(nyc), b(nyc), c(nyc), f(nyc), arr(nyc);
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int ic = 1; ic <= nxc; ++ic) {
          const int im = ic - 1, km = kc - 1;
          for (int jc = 1; jc <= nyc; ++jc) {
            const int jm = jc - 1, jp = jc + 1;
            double rt1, rt2;
            if (comp == 1) {
              if (jc == 1) { a[0] = zero; b[0] = one; c[0] = zero; f[0] = duy_ym[(size_t)(ic - 1) + (size_t)nxc * (kc - 1)]; continue; }
              rt1 = pmBetaT * nut(ic, jm, kc) * am2p(jc);
              rt2 = pmBetaT * nut(ic, jc, kc) * ap2p(jc);
            } else {
              double visc, visd;
              if (comp == 0) {
                visc = quarter * (nut(ic, jc, kc) + nut(im, jc, kc) + nut(ic, jm, kc) + nut(im, jm, kc));
                visd = quarter * (nut(ic, jc, kc) + nut(im, jc, kc) + nut(ic, jp, kc) + nut(im, jp, kc));
              } else {
                visc = quarter * (nut(ic, jc, km) + nut(ic, jm, km) + nut(ic, jc, kc) + nut(ic, jm, kc));
                visd = quarter * (nut(ic, jc, km) + nut(ic, jp, km) + nut(ic, jc, kc) + nut(ic, jp, kc));
              }
              rt1 = pmBetaT * visc * am2cForCN(jc);
              rt2 = pmBetaT * visd * ap2cForCN(jc);
            }
            a[jc - 1] = -rt1;
            b[jc - 1] = rt1 + rt2 + one;
            c[jc - 1] = -rt2;
            f[jc - 1] = Rhs(ic, jc, kc);
          }
          InverseTridiagonal1(a.data(), b.data(), c.data(), f.data(), nyc, arr.data());
          for (int jc = 1; jc <= nyc; ++jc) u(ic, jc, kc) = u(ic, jc, kc) + f[jc - 1];
        }
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:878-904 (PressureUpdate_PIMP_LES) ----
  void PressureUpdate_PIMP_LES(const F3& phi) {
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc) {
        int jp = jc + 1, jm = jc - 1;
        double metr1 = rdyp(jc) * rdyc(jc), metr2 = rdyp(jc) * rdyc(jp);
        for (int ic = 1; ic <= nxc; ++ic) {
          double visd = half * (nut(ic, jp, kc) + nut(ic, jc, kc));
          double visc = half * (nut(ic, jc, kc) + nut(ic, jm, kc));
          double pmBetap = -pmBetaT * metr2 * visd;
          double pmBetam = -pmBetaT * metr1 * visc;
          double pmBetac = -(pmBetap + pmBetam) + one;
          pressure(ic, jc, kc) = pressure(ic, jc, kc) + pmBetap * phi(ic, jp, kc) + pmBetac * phi(ic, jc, kc) + pmBetam * phi(ic, jm, kc);
        }
      }
  }

  // ---- src/CFD_2nd/m_TScheme.f90:213-241 (clcPrSrcOther) ----
  double clcPrSrcOther(F3& prsrc) {
    double sudtal = one / pmAlpha;
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int kp = kc + 1;
      double m = 0;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jp = jc + 1;
        double sucaj = rdyp(jc);
        for (int ic = 1; ic <= nxc; ++ic) {
          int ip = ic + 1;
          double rdiv = (ux(ip, jc, kc) - ux(ic, jc, kc)) * rdx + (uy(ic, jp, kc) - uy(ic, jc, kc)) * sucaj +
                        (uz(ic, jc, kp) - uz(ic, jc, kc)) * rdz;
          m = std::max(std::fabs(rdiv), m);
          prsrc(ic, jc, kc) = sudtal * rdiv;
        }
      }
      part[kc] = m;
    }
    double m = 0;
    for (int kc = 1; kc <= nzc; ++kc) m = std::max(m, part[kc]);
    return m;
  }

  // ---- src/CFD_2nd/m_Poisson.f90:1078-1201 (clcPPE_z1: z R2HC, x R2HC, per-slot
  //      y tridiagonal with the (1,1,1) pin, x HC2R, z HC2R, * normfft); with y
  //      periodic :954-1073 (clcPPE_z1_periodic: the same with cyclic y systems);
  //      with z between walls the z transforms are REDFT10 / REDFT01 (:267-307) ----
  void clcPPE(F3& prsrc, F3& prphiHalo) {
    // forward z transform of every (i,j) line
#pragma omp parallel
    {
      std::vector<double> line(nzc), db;
      std::vector<cplx> ba, bb;
#pragma omp for schedule(static)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int kc = 1; kc <= nzc; ++kc) line[kc - 1] = prsrc(ic, jc, kc);
          if (zper()) r2hc(planz, line.data(), ba, bb);
          else redft10(nzc, line.data(), zcos, db);  // z between walls: REDFT10
          for (int kc = 1; kc <= nzc; ++kc) prsrc(ic, jc, kc) = line[kc - 1];
        }
    }
    // forward x transform of every (j,k) line
#pragma omp parallel
    {
      std::vector<cplx> ba, bb;
      std::vector<double> db;
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int jc = 1; jc <= nyc; ++jc) {
          if (xper()) r2hc(planx, &prsrc(1, jc, kc), ba, bb);
          else redft10(nxc, &prsrc(1, jc, kc), xcos, db);  // x between walls: REDFT10
        }
    }
    // y tridiagonal per (ic,kc) slot
#pragma omp parallel
    {
      std::vector<double> a(nyc), b(nyc), c(nyc), f(nyc), arr(nyc), a2(nyc), a3(nyc);
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int jc = 1; jc <= nyc; ++jc) {
            a[jc - 1] = am2Pr(jc);
            c[jc - 1] = ap2Pr(jc);
            b[jc - 1] = ac2Pr(jc) + WaveNumX(ic) + WaveNumZ(kc);
            f[jc - 1] = prsrc(ic, jc, kc);
          }
          if (ic == 1 && kc == 1) { c[0] = zero; b[0] = one; a[0] = zero; f[0] = zero; }
          if (yper())  // clcPPE_z1_periodic (src/CFD_2nd/m_Poisson.f90:996-1052)
            InversePeriodicTridiagonal1(a.data(), b.data(), c.data(), f.data(), nyc, arr.data(), a2.data(), a3.data());
          else
            InverseTridiagonal1(a.data(), b.data(), c.data(), f.data(), nyc, arr.data());
          for (int jc = 1; jc <= nyc; ++jc) prsrc(ic, jc, kc) = f[jc - 1];
        }
    }
    // inverse x then inverse z
#pragma omp parallel
    {
      std::vector<cplx> ba, bb;
      std::vector<double> db;
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int jc = 1; jc <= nyc; ++jc) {
          if (xper()) hc2r(planx, &prsrc(1, jc, kc), ba, bb);
          else redft01(nxc, &prsrc(1, jc, kc), xcos, db);  // REDFT01
        }
    }
#pragma omp parallel
    {
      std::vector<double> line(nzc), db;
      std::vector<cplx> ba, bb;
#pragma omp for schedule(static)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int kc = 1; kc <= nzc; ++kc) line[kc - 1] = prsrc(ic, jc, kc);
          if (zper()) hc2r(planz, line.data(), ba, bb);
          else redft01(nzc, line.data(), zcos, db);  // REDFT01
          for (int kc = 1; kc <= nzc; ++kc) prsrc(ic, jc, kc) = line[kc - 1];
        }
    }
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) prphiHalo(ic, jc, kc) = prsrc(ic, jc, kc) * normfft;
  }

  // ---- src/CFD_2nd/m_TScheme.f90:281-306 (FluidVelUpdate) ----
  void FluidVelUpdate(const F3& phi) {
    double rdxEta2 = rdx * pmAlpha, rdzEta2 = rdz * pmAlpha;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1;
        double sucacEta2 = rdyc(jc) * pmAlpha;
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1;
          double locphi = phi(ic, jc, kc);
          ux(ic, jc, kc) = ux(ic, jc, kc) - (locphi - phi(im, jc, kc)) * rdxEta2;
          uy(ic, jc, kc) = uy(ic, jc, kc) - (locphi - phi(ic, jm, kc)) * sucacEta2;
          uz(ic, jc, kc) = uz(ic, jc, kc) - (locphi - phi(ic, jc, km)) * rdzEta2;
        }
      }
    }
  }

  // ---- src/CFD_2nd/m_TSchemePIMP_inc.f90:852-873 (PressureUpdate_PIMP) ----
  void PressureUpdate_PIMP(const F3& phi) {
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc) {
        int jp = jc + 1, jm = jc - 1;
        double pmBetap = -pmBeta * ap2Pr(jc);
        double pmBetac = -pmBeta * ac2Pr(jc) + one;
        double pmBetam = -pmBeta * am2Pr(jc);
        for (int ic = 1; ic <= nxc; ++ic)
          pressure(ic, jc, kc) = pressure(ic, jc, kc) + pmBetap * phi(ic, jp, kc) + pmBetac * phi(ic, jc, kc) + pmBetam * phi(ic, jm, kc);
      }
  }

  // =====================================================================
  // 4th-order solver (src/CFD_4th)
  // =====================================================================

  // ---- src/CFD_4th/m_BC_and_Halo.f90:51-96 (SetBC_and_UpdateHalo), channel ----
  void SetBC_and_UpdateHalo4() {
    for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) {
      if (P.FlowType == 1) {
        ux(i, nyp, k) = P.uxBcValue[3] * two - ux(i, nyc, k);
        uy(i, nyp, k) = P.uyBcValue[3];
        uz(i, nyp, k) = P.uzBcValue[3] * two - uz(i, nyc, k);
      } else {
        ux(i, nyp, k) = ux(i, nyc, k);
        uy(i, nyp, k) = zero;
        uz(i, nyp, k) = uz(i, nyc, k);
      }
      ux(i, 0, k) = P.uxBcValue[2] * two - ux(i, 1, k);
      uy(i, 1, k) = uy_ym[(size_t)(i - 1) + (size_t)nxc * (k - 1)];
      uz(i, 0, k) = P.uzBcValue[2] * two - uz(i, 1, k);
    }
    halo(ux, 2, 2, 0, 0, 2, 2);
    halo(uy, 2, 2, 0, 0, 2, 2);
    halo(uz, 2, 2, 0, 0, 2, 2);
  }

  // ---- src/CFD_4th/m_BC_and_Halo.f90:101-131 (SetBC_and_UpdateHaloForPrSrc) ----
  void SetBC_and_UpdateHaloForPrSrc4() {
    for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) {
      uy(i, nyp, k) = P.FlowType == 1 ? P.uyBcValue[3] : zero;
      uy(i, 1, k) = uy_ym[(size_t)(i - 1) + (size_t)nxc * (k - 1)];
    }
    halo(ux, 1, 2, 0, 0, 0, 0);
    halo(uz, 0, 0, 0, 0, 1, 2);
  }

  // ---- src/CFD_4th/m_BC_and_Halo.f90:136-150 (SetBC_and_UpdateHalo_pr) ----
  void SetBC_and_UpdateHalo_pr4(F3& pr) {
    for (int k = 1; k <= nzc; ++k) for (int i = 1; i <= nxc; ++i) {
      pr(i, 0, k) = pr(i, 1, k);
      pr(i, nyp, k) = pr(i, nyc, k);
    }
    halo(pr, 2, 1, 0, 0, 2, 1);
  }

  // ---- src/CFD_4th/m_TScheme.f90:189-377 (clcRhsXYZ without scalar/particles) ----
  void clcRhsXYZ4(F3& RhsX, F3& RhsY, F3& RhsZ) {
    const double xnu = P.xnu;
    // interpolated velocities (:209-227) and their halos (:228-233)
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) {
          int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
          uxhx(ic, jc, kc) = InterpCoe1 * ux(im, jc, kc) + InterpCoe2 * ux(ic, jc, kc) + InterpCoe3 * ux(ip, jc, kc) + InterpCoe4 * ux(iu, jc, kc);
          uyhx(ic, jc, kc) = InterpCoe1 * uy(is, jc, kc) + InterpCoe2 * uy(im, jc, kc) + InterpCoe3 * uy(ic, jc, kc) + InterpCoe4 * uy(ip, jc, kc);
          uzhx(ic, jc, kc) = InterpCoe1 * uz(is, jc, kc) + InterpCoe2 * uz(im, jc, kc) + InterpCoe3 * uz(ic, jc, kc) + InterpCoe4 * uz(ip, jc, kc);
          uxhz(ic, jc, kc) = InterpCoe1 * ux(ic, jc, ks) + InterpCoe2 * ux(ic, jc, km) + InterpCoe3 * ux(ic, jc, kc) + InterpCoe4 * ux(ic, jc, kp);
          uyhz(ic, jc, kc) = InterpCoe1 * uy(ic, jc, ks) + InterpCoe2 * uy(ic, jc, km) + InterpCoe3 * uy(ic, jc, kc) + InterpCoe4 * uy(ic, jc, kp);
          uzhz(ic, jc, kc) = InterpCoe1 * uz(ic, jc, km) + InterpCoe2 * uz(ic, jc, kc) + InterpCoe3 * uz(ic, jc, kp) + InterpCoe4 * uz(ic, jc, ku);
        }
      for (int ic = 1; ic <= nxc; ++ic) { uyhx(ic, nyp, kc) = zero; uyhz(ic, nyp, kc) = zero; }
    }
    halo(uxhx, 2, 1, 0, 0, 0, 0);
    halo(uyhx, 1, 2, 0, 0, 0, 0);
    halo(uzhx, 1, 2, 0, 0, 1, 2);
    halo(uxhz, 1, 2, 0, 0, 1, 2);
    halo(uyhz, 0, 0, 0, 0, 1, 2);
    halo(uzhz, 0, 0, 0, 0, 2, 1);

    // RhsX (:235-274)
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
      double s3tot = 0;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double sucaj = rdyp(jc);
        double InterpY1 = YinterpCoe(jc), InterpY2 = one - InterpY1;
        double InterpY3 = YinterpCoe(jp), InterpY4 = one - InterpY3;
        for (int ic = 1; ic <= nxc; ++ic) {
          int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
          double uxhyc = InterpY1 * ux(ic, jm, kc) + InterpY2 * ux(ic, jc, kc);
          double uxhyp = InterpY3 * ux(ic, jc, kc) + InterpY4 * ux(ic, jp, kc);
          double h11 = dxCoe1 * uxhx(is, jc, kc) * (uxhx(is, jc, kc) + uCRF) + dxCoe2 * uxhx(im, jc, kc) * (uxhx(im, jc, kc) + uCRF) +
                       dxCoe3 * uxhx(ic, jc, kc) * (uxhx(ic, jc, kc) + uCRF) + dxCoe4 * uxhx(ip, jc, kc) * (uxhx(ip, jc, kc) + uCRF);
          double h12 = (uyhx(ic, jp, kc) * uxhyp - uyhx(ic, jc, kc) * uxhyc) * sucaj;
          double h13 = dzCoe1 * uxhz(ic, jc, km) * uzhx(ic, jc, km) + dzCoe2 * uxhz(ic, jc, kc) * uzhx(ic, jc, kc) +
                       dzCoe3 * uxhz(ic, jc, kp) * uzhx(ic, jc, kp) + dzCoe4 * uxhz(ic, jc, ku) * uzhx(ic, jc, ku);
          double d11q1 = dxxCoe1 * ux(is, jc, kc) + dxxCoe2 * ux(im, jc, kc) + dxxCoe3 * ux(ic, jc, kc) + dxxCoe4 * ux(ip, jc, kc) + dxxCoe5 * ux(iu, jc, kc);
          double d22q1 = ap2c(jc) * ux(ic, jp, kc) + ac2c(jc) * ux(ic, jc, kc) + am2c(jc) * ux(ic, jm, kc);
          double d33q1 = dzzCoe1 * ux(ic, jc, ks) + dzzCoe2 * ux(ic, jc, km) + dzzCoe3 * ux(ic, jc, kc) + dzzCoe4 * ux(ic, jc, kp) + dzzCoe5 * ux(ic, jc, ku);
          double dcq13 = d11q1 + d33q1;
          s3tot = s3tot + (dcq13 + d22q1) * dyp(jc);
          double convEd1 = -h11 - h12 - h13 + xnu * dcq13 + P.gravity[0];
          double gradp1 = dxCoe1 * pressure(is, jc, kc) + dxCoe2 * pressure(im, jc, kc) + dxCoe3 * pressure(ic, jc, kc) + dxCoe4 * pressure(ip, jc, kc);
          RhsX(ic, jc, kc) = pmGamma * convEd1 + pmTheta * HistX(ic, jc, kc) - pmAlpha * gradp1 + two * pmBeta * d22q1;
          HistX(ic, jc, kc) = convEd1;
        }
      }
      part[kc] = s3tot;
    }
    // RhsY (:276-310)
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double sucac = rdyc(jc), qsucac = quarter * sucac;
        double InterpY1 = YinterpCoe(jc), InterpY2 = one - InterpY1;
        for (int ic = 1; ic <= nxc; ++ic) {
          int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
          double uxhym = InterpY1 * ux(im, jm, kc) + InterpY2 * ux(im, jc, kc) + uCRF, uzhym = InterpY1 * uz(ic, jm, km) + InterpY2 * uz(ic, jc, km);
          double uxhyc = InterpY1 * ux(ic, jm, kc) + InterpY2 * ux(ic, jc, kc) + uCRF, uzhyc = InterpY1 * uz(ic, jm, kc) + InterpY2 * uz(ic, jc, kc);
          double uxhyp = InterpY1 * ux(ip, jm, kc) + InterpY2 * ux(ip, jc, kc) + uCRF, uzhyp = InterpY1 * uz(ic, jm, kp) + InterpY2 * uz(ic, jc, kp);
          double uxhyu = InterpY1 * ux(iu, jm, kc) + InterpY2 * ux(iu, jc, kc) + uCRF, uzhyu = InterpY1 * uz(ic, jm, ku) + InterpY2 * uz(ic, jc, ku);
          double h21 = dxCoe1 * uyhx(im, jc, kc) * uxhym + dxCoe2 * uyhx(ic, jc, kc) * uxhyc + dxCoe3 * uyhx(ip, jc, kc) * uxhyp + dxCoe4 * uyhx(iu, jc, kc) * uxhyu;
          double h22 = ((uy(ic, jp, kc) + uy(ic, jc, kc)) * (uy(ic, jp, kc) + uy(ic, jc, kc)) -
                        (uy(ic, jc, kc) + uy(ic, jm, kc)) * (uy(ic, jc, kc) + uy(ic, jm, kc))) * qsucac;
          double h23 = dzCoe1 * uyhz(ic, jc, km) * uzhym + dzCoe2 * uyhz(ic, jc, kc) * uzhyc + dzCoe3 * uyhz(ic, jc, kp) * uzhyp + dzCoe4 * uyhz(ic, jc, ku) * uzhyu;
          double d11q2 = dxxCoe1 * uy(is, jc, kc) + dxxCoe2 * uy(im, jc, kc) + dxxCoe3 * uy(ic, jc, kc) + dxxCoe4 * uy(ip, jc, kc) + dxxCoe5 * uy(iu, jc, kc);
          double d22q2 = ap2p(jc) * uy(ic, jp, kc) + ac2p(jc) * uy(ic, jc, kc) + am2p(jc) * uy(ic, jm, kc);
          double d33q2 = dzzCoe1 * uy(ic, jc, ks) + dzzCoe2 * uy(ic, jc, km) + dzzCoe3 * uy(ic, jc, kc) + dzzCoe4 * uy(ic, jc, kp) + dzzCoe5 * uy(ic, jc, ku);
          double dcq13 = d11q2 + d33q2;
          double convEd2 = -h21 - h22 - h23 + xnu * dcq13 + P.gravity[1];
          double gradp2 = (pressure(ic, jc, kc) - pressure(ic, jm, kc)) * sucac;
          RhsY(ic, jc, kc) = pmGamma * convEd2 + pmTheta * HistY(ic, jc, kc) - pmAlpha * gradp2 + two * pmBeta * d22q2;
          HistY(ic, jc, kc) = convEd2;
        }
      }
    }
    // RhsZ (:312-343)
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1, jp = jc + 1;
        double sucaj = rdyp(jc);
        double InterpY1 = YinterpCoe(jc), InterpY2 = one - InterpY1;
        double InterpY3 = YinterpCoe(jp), InterpY4 = one - InterpY3;
        for (int ic = 1; ic <= nxc; ++ic) {
          int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
          double uzhyc = InterpY1 * uz(ic, jm, kc) + InterpY2 * uz(ic, jc, kc);
          double uzhyp = InterpY3 * uz(ic, jc, kc) + InterpY4 * uz(ic, jp, kc);
          double h31 = dxCoe1 * uzhx(im, jc, kc) * (uxhz(im, jc, kc) + uCRF) + dxCoe2 * uzhx(ic, jc, kc) * (uxhz(ic, jc, kc) + uCRF) +
                       dxCoe3 * uzhx(ip, jc, kc) * (uxhz(ip, jc, kc) + uCRF) + dxCoe4 * uzhx(iu, jc, kc) * (uxhz(iu, jc, kc) + uCRF);
          double h32 = (uyhz(ic, jp, kc) * uzhyp - uyhz(ic, jc, kc) * uzhyc) * sucaj;
          double h33 = dzCoe1 * uzhz(ic, jc, ks) * uzhz(ic, jc, ks) + dzCoe2 * uzhz(ic, jc, km) * uzhz(ic, jc, km) +
                       dzCoe3 * uzhz(ic, jc, kc) * uzhz(ic, jc, kc) + dzCoe4 * uzhz(ic, jc, kp) * uzhz(ic, jc, kp);
          double d11q3 = dxxCoe1 * uz(is, jc, kc) + dxxCoe2 * uz(im, jc, kc) + dxxCoe3 * uz(ic, jc, kc) + dxxCoe4 * uz(ip, jc, kc) + dxxCoe5 * uz(iu, jc, kc);
          double d22q3 = ap2c(jc) * uz(ic, jp, kc) + ac2c(jc) * uz(ic, jc, kc) + am2c(jc) * uz(ic, jm, kc);
          double d33q3 = dzzCoe1 * uz(ic, jc, ks) + dzzCoe2 * uz(ic, jc, km) + dzzCoe3 * uz(ic, jc, kc) + dzzCoe4 * uz(ic, jc, kp) + dzzCoe5 * uz(ic, jc, ku);
          double dcq13 = d11q3 + d33q3;
          double convEd3 = -h31 - h32 - h33 + xnu * dcq13 + P.gravity[2];
          double gradp3 = dzCoe1 * pressure(ic, jc, ks) + dzCoe2 * pressure(ic, jc, km) + dzCoe3 * pressure(ic, jc, kc) + dzCoe4 * pressure(ic, jc, kp);
          RhsZ(ic, jc, kc) = pmGamma * convEd3 + pmTheta * HistZ(ic, jc, kc) - pmAlpha * gradp3 + two * pmBeta * d22q3;
          HistZ(ic, jc, kc) = convEd3;
        }
      }
    }
    // constant flux from the mean viscous stress (:364-377)
    if (P.IsUxConst) {
      double s3tot1 = 0;
      for (int kc = 1; kc <= nzc; ++kc) s3tot1 += part[kc];
      double dpmdxns = xnu * s3tot1 / ((double)nxc * (double)nzc) / P.yly;
      double dp1ns = pmAlpha * dpmdxns;
#pragma omp parallel for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int jc = 1; jc <= nyc; ++jc) for (int ic = 1; ic <= nxc; ++ic) RhsX(ic, jc, kc) = RhsX(ic, jc, kc) - dp1ns;
      PrGradAver = PrGradAver + dpmdxns * pmAlphaC;
    }
  }

  // ---- src/CFD_4th/m_TScheme.f90:443-549 (clcU1Hat/clcU3Hat; clcU2Hat as PIMP) ----
  void clcUHat4_c(F3& u, F3& Rhs) {
    std::vector<double> tp(nyc), tm(nyc), tc(nyc);
    for (int jc = 1; jc <= nyc; ++jc) {
      tp[jc - 1] = -pmBeta * ap2cForCN(jc);
      tc[jc - 1] = -pmBeta * ac2cForCN(jc) + one;
      tm[jc - 1] = -pmBeta * am2cForCN(jc);
    }
#pragma omp parallel
    {
      std::vector<double> f(nyc), arr(nyc);
#pragma omp for schedule(static)
      for (int kc = 1; kc <= nzc; ++kc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int jc = 1; jc <= nyc; ++jc) f[jc - 1] = Rhs(ic, jc, kc);
          InverseTridiagonal1(tm.data(), tc.data(), tp.data(), f.data(), nyc, arr.data());
          for (int jc = 1; jc <= nyc; ++jc) u(ic, jc, kc) = u(ic, jc, kc) + f[jc - 1];
        }
    }
  }

  // ---- src/CFD_4th/m_TScheme.f90:114-143 (clcPrSrc) ----
  double clcPrSrc4(F3& prsrc) {
    double sudtal = one / pmAlpha;
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1, ku = kc + 2;
      double m = 0;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jp = jc + 1;
        double sucaj = rdyp(jc);
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1, iu = ic + 2;
          double dudx = dxCoe1 * ux(im, jc, kc) + dxCoe2 * ux(ic, jc, kc) + dxCoe3 * ux(ip, jc, kc) + dxCoe4 * ux(iu, jc, kc);
          double dvdy = (uy(ic, jp, kc) - uy(ic, jc, kc)) * sucaj;
          double dwdz = dzCoe1 * uz(ic, jc, km) + dzCoe2 * uz(ic, jc, kc) + dzCoe3 * uz(ic, jc, kp) + dzCoe4 * uz(ic, jc, ku);
          double rdiv = dudx + dvdy + dwdz;
          m = std::max(std::fabs(rdiv), m);
          prsrc(ic, jc, kc) = sudtal * rdiv;
        }
      }
      part[kc] = m;
    }
    double m = 0;
    for (int kc = 1; kc <= nzc; ++kc) m = std::max(m, part[kc]);
    return m;
  }

  // ---- src/CFD_4th/m_TScheme.f90:148-173 (FluidVelUpdate) ----
  void FluidVelUpdate4(const F3& phi) {
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int ks = kc - 2, km = kc - 1, kp = kc + 1;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jm = jc - 1;
        double sucac = rdyc(jc);
        for (int ic = 1; ic <= nxc; ++ic) {
          int is = ic - 2, im = ic - 1, ip = ic + 1;
          double dpdx = dxCoe1 * phi(is, jc, kc) + dxCoe2 * phi(im, jc, kc) + dxCoe3 * phi(ic, jc, kc) + dxCoe4 * phi(ip, jc, kc);
          double dpdy = (phi(ic, jc, kc) - phi(ic, jm, kc)) * sucac;
          double dpdz = dzCoe1 * phi(ic, jc, ks) + dzCoe2 * phi(ic, jc, km) + dzCoe3 * phi(ic, jc, kc) + dzCoe4 * phi(ic, jc, kp);
          ux(ic, jc, kc) = ux(ic, jc, kc) - pmAlpha * dpdx;
          uy(ic, jc, kc) = uy(ic, jc, kc) - pmAlpha * dpdy;
          uz(ic, jc, kc) = uz(ic, jc, kc) - pmAlpha * dpdz;
        }
      }
    }
  }

  // ---- src/CFD_4th/m_Tools.f90:54-81 (CheckDivergence) ----
  double CheckDivergence4() {
    std::vector<double> part(nzc + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; ++kc) {
      int km = kc - 1, kp = kc + 1, ku = kc + 2;
      double m = 0;
      for (int jc = 1; jc <= nyc; ++jc) {
        int jp = jc + 1;
        double sucaj = rdyp(jc);
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1, iu = ic + 2;
          double dudx = dxCoe1 * ux(im, jc, kc) + dxCoe2 * ux(ic, jc, kc) + dxCoe3 * ux(ip, jc, kc) + dxCoe4 * ux(iu, jc, kc);
          double dvdy = (uy(ic, jp, kc) - uy(ic, jc, kc)) * sucaj;
          double dwdz = dzCoe1 * uz(ic, jc, km) + dzCoe2 * uz(ic, jc, kc) + dzCoe3 * uz(ic, jc, kp) + dzCoe4 * uz(ic, jc, ku);
          double udiv = std::fabs(dudx + dvdy + dwdz);
          if (udiv > m) m = udiv;
        }
      }
      part[kc] = m;
    }
    double m = 0;
    for (int kc = 1; kc <= nzc; ++kc) m = std::max(m, part[kc]);
    return m;
  }

  // ---- src/CFD_4th/m_ChannelSystem.f90:106-141, one substep in stages ----
  void stage4(int st, int ns) {
    switch (st) {
      case 0: PMcoeUpdate(ns); Update_uy_ym(); break;
      case 1: clcRhsXYZ4(RealArr1, RealArr2, RealHalo); break;
      case 2:
        clcUHat4_c(ux, RealArr1);
        clcU2Hat_PIMP(RealArr2);
        clcUHat4_c(uz, RealHalo);
        break;
      case 3:
        SetBC_and_UpdateHaloForPrSrc4();
        divmax1_last = clcPrSrc4(RealArr1);
        break;
      case 4:
        clcPPE(RealArr1, RealHalo);
        SetBC_and_UpdateHalo_pr4(RealHalo);
        break;
      case 5: FluidVelUpdate4(RealHalo); break;
      case 6:
        PressureUpdate_PIMP(RealHalo);
        SetBC_and_UpdateHalo4();
        SetBC_and_UpdateHalo_pr4(pressure);
        break;
    }
  }

  // ---- src/CFD_2nd/m_ChannelSystem.f90:91-124, one substep split in stages ----
  // stage 0: PMcoeUpdate + Update_uy_ym; 1: clcRhsX/Y/Z; 2: clcU1/2/3Hat;
  // 3: SetBC_and_UpdateHaloForPrSrc + clcPrSrc; 4: clcPPE + SetBC_and_UpdateHalo_pr;
  // 5: FluidVelUpdate; 6: PressureUpdate + SetBC_and_UpdateHalo(u) + ..._pr(p)
  void stage(int st, int ns) {
    if (o4) { stage4(st, ns); return; }
    const bool fimp = P.IsImplicit == 2, fexp = P.IsImplicit == 0;
    const bool les = P.LES_type > 0;
    switch (st) {
      case 0: PMcoeUpdate(ns); Update_uy_ym(); break;
      case 1:
        if (les) {
          clcRhsX_PIMP_LES(RealArr1, HistX, fexp);
          clcRhsY_PIMP_LES(RealArr2, HistY, fexp);
          clcRhsZ_PIMP_LES(RealHalo, HistZ, fexp);
          break;
        }
        clcRhsX_PIMP(RealArr1, HistX, P.IsImplicit);
        clcRhsY_PIMP(RealArr2, HistY, P.IsImplicit);
        clcRhsZ_PIMP(RealHalo, HistZ, P.IsImplicit);
        break;
      case 2:
        if (fexp) { clcUHat_FEXP(ux, RealArr1); clcUHat_FEXP(uy, RealArr2); clcUHat_FEXP(uz, RealHalo); break; }
        if (les) {
          clcUHat_PIMP_LES(0, ux, RealArr1);
          clcUHat_PIMP_LES(1, uy, RealArr2);
          clcUHat_PIMP_LES(2, uz, RealHalo);
          break;
        }
        if (fimp && zper()) { clcUHat_FIMP_xz(RealArr1); clcUHat_FIMP_xz(RealArr2); clcUHat_FIMP_xz(RealHalo); }
        if (fimp && !zper()) {  // clcU1/2/3Hat_FIMP_011, or _111 with walls in x too
          if (xper()) { clcUHat_FIMP_x(RealArr1); clcUHat_FIMP_x(RealArr2); clcUHat_FIMP_x(RealHalo); }
          else { clcUHat_FIMP_xwall(RealArr1, true); clcUHat_FIMP_xwall(RealArr2, false); clcUHat_FIMP_xwall(RealHalo, false); }
          clcUHat_FIMP_zwall(RealArr1, false); clcUHat_FIMP_zwall(RealArr2, false); clcUHat_FIMP_zwall(RealHalo, true);
        }
        if (yper()) {  // clcU1/2/3Hat_FIMP_000 (after the x and z sweeps) or clcU1/2/3Hat_PIMP_0
          clcUHat_y_periodic(ux, RealArr1);
          clcUHat_y_periodic(uy, RealArr2);
          clcUHat_y_periodic(uz, RealHalo);
          break;
        }
        clcUHat_PIMP_c(ux, RealArr1);
        clcU2Hat_PIMP(RealArr2);
        clcUHat_PIMP_c(uz, RealHalo);
        break;
      case 3:
        SetBC_and_UpdateHaloForPrSrc();
        divmax1_last = fimp ? clcPrSrc_FIMP(RealArr1) : clcPrSrcOther(RealArr1);
        break;
      case 4:
        clcPPE(RealArr1, RealHalo);
        SetBC_and_UpdateHalo_pr(RealHalo);
        break;
      case 5: FluidVelUpdate(RealHalo); break;
      case 6:
        if (les && !fexp) PressureUpdate_PIMP_LES(RealHalo);
        else if (fimp || fexp) PressureUpdate_FIMP(RealHalo);  // PressureUpdate_FEXP is the same update
        else PressureUpdate_PIMP(RealHalo);
        SetBC_and_UpdateHalo();
        SetBC_and_UpdateHalo_pr(pressure);
        break;
    }
  }

  // ---- src/CFD_2nd/m_ChannelSystem.f90:73-154 (ChannelIterate) ----
  int ChannelIterate(orc_info* info) {
    itime += 1;
    double uddxmax = CalcMaxCFL();
    double cflmp = uddxmax * dt;
    if (P.iCFL == 1) { dt = P.CFLc / uddxmax; dt = std::min(dt, P.dtMax); }
    else dt = P.dtMax;
    if (P.LES_type > 0 && !o4) Clc_SGS_Vis();
    for (int ns = 1; ns <= iadvance; ++ns)
      for (int st = 0; st <= 6; ++st) stage(st, ns);
    double divmax2 = o4 ? CheckDivergence4() : CheckDivergence();
    double vmax[3];
    CalcVmax(vmax);
    int status = 0;
    if (divmax2 > P.div_limit) status = 1;
    else if (std::min(vmax[0], std::min(vmax[1], vmax[2])) > P.vel_limit) status = 2;
    if (info) {
      info->SimTime = SimTime; info->dt = dt; info->cflmp = cflmp; info->divmax1 = divmax1_last;
      info->divmax2 = divmax2; info->vmax[0] = vmax[0]; info->vmax[1] = vmax[1]; info->vmax[2] = vmax[2];
      info->uxm = CalcUxAver(); info->PrGradAver = PrGradAver; info->itime = itime; info->status = status;
    }
    return status;
  }

  // ---- src/CFD_2nd/m_FlowType_Channel.f90:175-330 (clcStat_CH moment sums) ----
  void clcStat_CH() {
    double rdxh = rdx * half;
    double inxz = one / ((double)nxc * (double)nzc);
    for (int jc = 1; jc <= nyc; ++jc) {
      int jp = jc + 1, jm = jc - 1;
      double InterpY1 = half * YinterpCoe(jc), InterpY2 = half - InterpY1;
      double cac = rdyc(jc), cacU = rdyc(jp), caj = rdyp(jc);
      double S[35] = {0};
      for (int kc = 1; kc <= nzc; ++kc) {
        int km = kc - 1, kp = kc + 1;
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1, ip = ic + 1;
          double uxloc = ux(ic, jc, kc), uyloc = uy(ic, jc, kc), uzloc = uz(ic, jc, kc), prloc = pressure(ic, jc, kc);
          double uxCell = half * (ux(ic, jc, kc) + ux(ip, jc, kc));
          double uyCell = half * (uy(ic, jc, kc) + uy(ic, jp, kc));
          double uzCell = half * (uz(ic, jc, kc) + uz(ic, jc, kp));
          double prloc2 = InterpY1 * (pressure(im, jm, kc) + pressure(ic, jm, kc)) + InterpY2 * (pressure(im, jc, kc) + pressure(ic, jc, kc));
          double dudx = (ux(ip, jc, kc) - ux(ic, jc, kc)) * rdx;
          double dudy = (ux(ic, jc, kc) - ux(ic, jm, kc)) * cac;
          double dudz = (ux(ic, jc, kc) - ux(ic, jc, km)) * rdz;
          double dvdx = (uy(ic, jc, kc) - uy(im, jc, kc)) * rdx;
          double dvdy = (uy(ic, jp, kc) - uy(ic, jc, kc)) * caj;
          double dvdz = (uy(ic, jc, kc) - uy(ic, jc, km)) * rdz;
          double dwdx = (uz(ic, jc, kc) - uz(im, jc, kc)) * rdx;
          double dwdy = (uz(ic, jc, kc) - uz(ic, jm, kc)) * cac;
          double dwdz = (uz(ic, jc, kp) - uz(ic, jc, kc)) * rdz;
          double dudxx = (ux(ip, jc, kc) - two * ux(ic, jc, kc) + ux(im, jc, kc)) * rdx2;
          double dudyy = ap2c(jc) * ux(ic, jp, kc) + ac2c(jc) * ux(ic, jc, kc) + am2c(jc) * ux(ic, jm, kc);
          double dudzz = (ux(ic, jc, kp) - two * ux(ic, jc, kc) + ux(ic, jc, km)) * rdz2;
          double dvdxx = (uy(ip, jc, kc) - two * uy(ic, jc, kc) + uy(im, jc, kc)) * rdx2;
          double dvdyy = ap2p(jc) * uy(ic, jp, kc) + ac2p(jc) * uy(ic, jc, kc) + am2p(jc) * uy(ic, jm, kc);
          double dvdzz = (uy(ic, jc, kp) - two * uy(ic, jc, kc) + uy(ic, jc, km)) * rdz2;
          double dwdxx = (uz(ip, jc, kc) - two * uz(ic, jc, kc) + uz(im, jc, kc)) * rdx2;
          double dwdyy = ap2c(jc) * uz(ic, jp, kc) + ac2c(jc) * uz(ic, jc, kc) + am2c(jc) * uz(ic, jm, kc);
          double dwdzz = (uz(ic, jc, kp) - two * uz(ic, jc, kc) + uz(ic, jc, km)) * rdz2;
          double vor_x = dwdy - dvdz, vor_y = dudz - dwdx, vor_z = dvdx - dudy;
          double dudxC = (ux(ip, jc, kc) - ux(im, jc, kc)) * rdxh;
          double dvdxU = (uy(ic, jp, kc) - uy(im, jp, kc)) * rdx;
          double dudyU = (ux(ic, jp, kc) - ux(ic, jc, kc)) * cacU;
          double dvdyM = (uy(im, jp, kc) - uy(im, jc, kc)) * caj;
          double dudzC = (InterpY1 * (ux(ic, jm, kp) - ux(ic, jm, km)) + InterpY2 * (ux(ic, jc, kp) - ux(ic, jc, km))) * rdz;
          double dvdzC = (uy(im, jc, kp) - uy(im, jc, km) + uy(ic, jc, kp) - uy(ic, jc, km)) * rdz * quarter;
          S[0] += uxloc; S[1] += uyloc; S[2] += uzloc; S[3] += prloc;
          S[4] += uxloc * uxloc; S[5] += uyloc * uyloc; S[6] += uzloc * uzloc; S[7] += prloc * prloc;
          S[8] += uxCell * uyCell; S[9] += uyCell * uzCell; S[10] += uxCell * uzCell;
          S[11] += uxCell * prloc; S[12] += uyCell * prloc; S[13] += uzCell * prloc;
          S[14] += uxCell * uxCell * uyCell; S[15] += uyloc * uyloc * uyloc; S[16] += uzCell * uzCell * uyCell;
          S[17] += uxCell * uyCell * uyCell; S[18] += uxloc * uxloc * uxloc; S[19] += uzloc * uzloc * uzloc;
          S[20] += uxloc * uxloc * uxloc * uxloc; S[21] += uyloc * uyloc * uyloc * uyloc; S[22] += uzloc * uzloc * uzloc * uzloc;
          S[23] += prloc * dudx; S[24] += prloc * dvdy; S[25] += prloc * dwdz;
          S[26] += prloc2 * (dudy + dvdx);
          S[27] += uxloc * (dudxx + dudyy + dudzz); S[28] += uyloc * (dvdxx + dvdyy + dvdzz); S[29] += uzloc * (dwdxx + dwdyy + dwdzz);
          S[30] += dudxC * (dvdxU + dvdx) * half + (dudyU + dudy) * (dvdyM + dvdy) * quarter;
          S[31] += dudzC * dvdzC;
          S[32] += vor_x * vor_x; S[33] += vor_y * vor_y; S[34] += vor_z * vor_z;
        }
      }
      for (int q = 0; q < 35; ++q) SumStat[(size_t)q + 35 * (size_t)(jc - 1)] += S[q] * inxz;
    }
    {
      int jc = nyp, jm = jc - 1;
      double cac = rdyc(jc);
      double InterpY1 = half * YinterpCoe(jc), InterpY2 = half - InterpY1;
      double S26 = 0, S32 = 0, S34 = 0;
      for (int kc = 1; kc <= nzc; ++kc)
        for (int ic = 1; ic <= nxc; ++ic) {
          int im = ic - 1;
          double prloc2 = InterpY1 * (pressure(im, jm, kc) + pressure(ic, jm, kc)) + InterpY2 * (pressure(im, jc, kc) + pressure(ic, jc, kc));
          double dudy = (ux(ic, jc, kc) - ux(ic, jm, kc)) * cac;
          double dwdy = (uz(ic, jc, kc) - uz(ic, jm, kc)) * cac;
          double vor_x = dwdy, vor_z = -dudy;
          S26 += prloc2 * (dudy + zero);
          S32 += vor_x * vor_x;
          S34 += vor_z * vor_z;
        }
      SumStat[26 + 35 * (size_t)(jc - 1)] += S26 * inxz;
      SumStat[32 + 35 * (size_t)(jc - 1)] += S32 * inxz;
      SumStat[34 + 35 * (size_t)(jc - 1)] += S34 * inxz;
    }
    PrGradsum = PrGradsum + PrGradAver;
    nfstime += 1;
  }

  // ---- src/CFD_4th/m_FlowCase.f90:330-640 (clcStat moments: SumStat(35,nyp) and, with
  //      HighOrderGradStat defined at :17, SumGrad(98,nyp)); the spectra branch
  //      (:642-) is separate.  pressure(nxc+2,:,:) and pressure(:,:,nzc+2) are never
  //      written by SetBC_and_UpdateHalo_pr (halo xph = zph = 1,
  //      src/CFD_4th/m_BC_and_Halo.f90:42-45), so dpdxx and dpdzz read the zero the
  //      array was allocated with (src/CFD_4th/m_Variables.f90:85) there. ----
  void clcStat4() {
    const double rdxt = rdx / 12.0, rdzt = rdz / 12.0;
    const double inxz = one / ((double)nxc * (double)nzc);
    if (SumGrad.empty()) SumGrad.assign((size_t)98 * nyp, 0.0);
    for (int jc = 1; jc <= nyc; ++jc) {
      const int jp = jc + 1, jm = jc - 1;
      const double InterpY1 = YinterpCoe(jc), InterpY2 = one - InterpY1;
      const double cac = rdyc(jc), cacU = rdyc(jp), caj = rdyp(jc);
      double S[35] = {0}, G[98] = {0};
      for (int kc = 1; kc <= nzc; ++kc) {
        const int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
        for (int ic = 1; ic <= nxc; ++ic) {
          const int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
          const F3 &U = ux, &V = uy, &W = uz, &pr = pressure;
          double uxloc = U(ic, jc, kc) + uCRF, uyloc = V(ic, jc, kc), uzloc = W(ic, jc, kc), prloc = pr(ic, jc, kc);
          double uxCell = InterpCoe1 * U(im, jc, kc) + InterpCoe2 * U(ic, jc, kc) + InterpCoe3 * U(ip, jc, kc) + InterpCoe4 * U(iu, jc, kc) + uCRF;
          double uyCell = (uyloc + V(ic, jp, kc)) * half;
          double uy_xc = InterpCoe1 * V(is, jc, kc) + InterpCoe2 * V(im, jc, kc) + InterpCoe3 * V(ic, jc, kc) + InterpCoe4 * V(ip, jc, kc);
          double uy_xp = InterpCoe1 * V(is, jp, kc) + InterpCoe2 * V(im, jp, kc) + InterpCoe3 * V(ic, jp, kc) + InterpCoe4 * V(ip, jp, kc);
          double uzCell = InterpCoe1 * W(ic, jc, km) + InterpCoe2 * W(ic, jc, kc) + InterpCoe3 * W(ic, jc, kp) + InterpCoe4 * W(ic, jc, ku);
          double prloc2 = InterpY1 * (InterpCoe1 * pr(is, jm, kc) + InterpCoe2 * pr(im, jm, kc) +
                                      InterpCoe3 * pr(ic, jm, kc) + InterpCoe4 * pr(ip, jm, kc)) +
                          InterpY2 * (InterpCoe1 * pr(is, jc, kc) + InterpCoe2 * pr(im, jc, kc) +
                                      InterpCoe3 * pr(ic, jc, kc) + InterpCoe4 * pr(ip, jc, kc));
          double dudx = dxCoe1 * U(im, jc, kc) + dxCoe2 * U(ic, jc, kc) + dxCoe3 * U(ip, jc, kc) + dxCoe4 * U(iu, jc, kc);
          double dudy = (U(ic, jc, kc) - U(ic, jm, kc)) * cac;
          double dudz = dzCoe1 * U(ic, jc, ks) + dzCoe2 * U(ic, jc, km) + dzCoe3 * U(ic, jc, kc) + dzCoe4 * U(ic, jc, kp);
          double dvdx = dxCoe1 * V(is, jc, kc) + dxCoe2 * V(im, jc, kc) + dxCoe3 * V(ic, jc, kc) + dxCoe4 * V(ip, jc, kc);
          double dvdy = (V(ic, jp, kc) - uyloc) * caj;
          double dvdz = dzCoe1 * V(ic, jc, ks) + dzCoe2 * V(ic, jc, km) + dzCoe3 * V(ic, jc, kc) + dzCoe4 * V(ic, jc, kp);
          double dwdx = dxCoe1 * W(is, jc, kc) + dxCoe2 * W(im, jc, kc) + dxCoe3 * W(ic, jc, kc) + dxCoe4 * W(ip, jc, kc);
          double dwdy = (uzloc - W(ic, jm, kc)) * cac;
          double dwdz = dzCoe1 * W(ic, jc, km) + dzCoe2 * W(ic, jc, kc) + dzCoe3 * W(ic, jc, kp) + dzCoe4 * W(ic, jc, ku);
          double dudxx = dxxCoe1 * U(is, jc, kc) + dxxCoe2 * U(im, jc, kc) + dxxCoe3 * U(ic, jc, kc) + dxxCoe4 * U(ip, jc, kc) + dxxCoe5 * U(iu, jc, kc);
          double dudyy = ap2c(jc) * U(ic, jp, kc) + ac2c(jc) * U(ic, jc, kc) + am2c(jc) * U(ic, jm, kc);
          double dudzz = dzzCoe1 * U(ic, jc, ks) + dzzCoe2 * U(ic, jc, km) + dzzCoe3 * U(ic, jc, kc) + dzzCoe4 * U(ic, jc, kp) + dzzCoe5 * U(ic, jc, ku);
          double dvdxx = dxxCoe1 * V(is, jc, kc) + dxxCoe2 * V(im, jc, kc) + dxxCoe3 * V(ic, jc, kc) + dxxCoe4 * V(ip, jc, kc) + dxxCoe5 * V(iu, jc, kc);
          double dvdyy = ap2p(jc) * V(ic, jp, kc) + ac2p(jc) * V(ic, jc, kc) + am2p(jc) * V(ic, jm, kc);
          double dvdzz = dzzCoe1 * V(ic, jc, ks) + dzzCoe2 * V(ic, jc, km) + dzzCoe3 * V(ic, jc, kc) + dzzCoe4 * V(ic, jc, kp) + dzzCoe5 * V(ic, jc, ku);
          double dwdxx = dxxCoe1 * W(is, jc, kc) + dxxCoe2 * W(im, jc, kc) + dxxCoe3 * W(ic, jc, kc) + dxxCoe4 * W(ip, jc, kc) + dxxCoe5 * W(iu, jc, kc);
          double dwdyy = ap2c(jc) * W(ic, jp, kc) + ac2c(jc) * W(ic, jc, kc) + am2c(jc) * W(ic, jm, kc);
          double dwdzz = dzzCoe1 * W(ic, jc, ks) + dzzCoe2 * W(ic, jc, km) + dzzCoe3 * W(ic, jc, kc) + dzzCoe4 * W(ic, jc, kp) + dzzCoe5 * W(ic, jc, ku);
          double vor_x = dwdy - dvdz, vor_y = dudz - dwdx, vor_z = dvdx - dudy;
          double dudxC = (-U(iu, jc, kc) + 8.0 * U(ip, jc, kc) - 8.0 * U(im, jc, kc) + U(is, jc, kc)) * rdxt;
          double dvdxU = dxCoe1 * V(is, jp, kc) + dxCoe2 * V(im, jp, kc) + dxCoe3 * V(ic, jp, kc) + dxCoe4 * V(ip, jp, kc);
          double dudyU = (U(ic, jp, kc) - U(ic, jc, kc)) * cacU;
          double dudzC = (InterpY1 * (-U(ic, jm, ku) + 8.0 * U(ic, jm, kp) - 8.0 * U(ic, jm, km) + U(ic, jm, ks)) +
                          InterpY2 * (-U(ic, jc, ku) + 8.0 * U(ic, jc, kp) - 8.0 * U(ic, jc, km) + U(ic, jc, ks))) * rdzt;
          double dvdzC = ((-V(is, jc, ku) + 8.0 * V(is, jc, kp) - 8.0 * V(is, jc, km) + V(is, jc, ks)) * InterpCoe1 +
                          (-V(im, jc, ku) + 8.0 * V(im, jc, kp) - 8.0 * V(im, jc, km) + V(im, jc, ks)) * InterpCoe2 +
                          (-V(ic, jc, ku) + 8.0 * V(ic, jc, kp) - 8.0 * V(ic, jc, km) + V(ic, jc, ks)) * InterpCoe3 +
                          (-V(ip, jc, ku) + 8.0 * V(ip, jc, kp) - 8.0 * V(ip, jc, km) + V(ip, jc, ks)) * InterpCoe4) * rdzt;
          S[0] += uxloc; S[1] += uyloc; S[2] += uzloc; S[3] += prloc;
          S[4] += uxloc * uxloc; S[5] += uyloc * uyloc; S[6] += uzloc * uzloc; S[7] += prloc * prloc;
          S[8] += uxCell * uyCell; S[9] += uyCell * uzCell; S[10] += uxCell * uzCell;
          S[11] += uxCell * prloc; S[12] += uyCell * prloc; S[13] += uzCell * prloc;
          S[14] += uxCell * uxCell * uyCell; S[15] += uyloc * uyloc * uyloc; S[16] += uzCell * uzCell * uyCell;
          S[17] += uxCell * uyCell * uyCell; S[18] += uxloc * uxloc * uxloc; S[19] += uzloc * uzloc * uzloc;
          S[20] += uxloc * uxloc * uxloc * uxloc; S[21] += uyloc * uyloc * uyloc * uyloc; S[22] += uzloc * uzloc * uzloc * uzloc;
          S[23] += prloc * dudx; S[24] += prloc * dvdy; S[25] += prloc * dwdz;
          S[26] += prloc2 * (dudy + dvdx);
          S[27] += uxloc * (dudxx + dudyy + dudzz); S[28] += uyloc * (dvdxx + dvdyy + dvdzz); S[29] += uzloc * (dwdxx + dwdyy + dwdzz);
          S[30] += (dudxC * (dvdxU + dvdx) + (dudyU + dudy) * (uy_xp - uy_xc) * caj) * half;
          S[31] += dudzC * dvdzC;
          S[32] += vor_x * vor_x; S[33] += vor_y * vor_y; S[34] += vor_z * vor_z;
          // pressure gradients (:485-490)
          double dpdx = dxCoe1 * pr(is, jc, kc) + dxCoe2 * pr(im, jc, kc) + dxCoe3 * pr(ic, jc, kc) + dxCoe4 * pr(ip, jc, kc);
          double dpdy = (pr(ic, jc, kc) - pr(ic, jm, kc)) * cac;
          double dpdz = dzCoe1 * pr(ic, jc, ks) + dzCoe2 * pr(ic, jc, km) + dzCoe3 * pr(ic, jc, kc) + dzCoe4 * pr(ic, jc, kp);
          double dpdxx = dxxCoe1 * pr(is, jc, kc) + dxxCoe2 * pr(im, jc, kc) + dxxCoe3 * pr(ic, jc, kc) + dxxCoe4 * pr(ip, jc, kc) + dxxCoe5 * pr(iu, jc, kc);
          double dpdyy = ap2c(jc) * pr(ic, jp, kc) + ac2c(jc) * pr(ic, jc, kc) + am2c(jc) * pr(ic, jm, kc);
          double dpdzz = dzzCoe1 * pr(ic, jc, ks) + dzzCoe2 * pr(ic, jc, km) + dzzCoe3 * pr(ic, jc, kc) + dzzCoe4 * pr(ic, jc, kp) + dzzCoe5 * pr(ic, jc, ku);
          G[0] += prloc * prloc * prloc;
          G[1] += prloc * prloc * prloc * prloc;
          // SumVec2(3..98): the first four powers of each gradient, in the order of :496-589
          const double q[24] = {dudx, dudy, dudz, dvdx, dvdy, dvdz, dwdx, dwdy, dwdz, dpdx, dpdy, dpdz,
                                dudxx, dudyy, dudzz, dvdxx, dvdyy, dvdzz, dwdxx, dwdyy, dwdzz, dpdxx, dpdyy, dpdzz};
          for (int t = 0; t < 24; ++t) {
            const double a = q[t];
            G[2 + 4 * t] += a;
            G[3 + 4 * t] += a * a;
            G[4 + 4 * t] += a * a * a;
            G[5 + 4 * t] += a * a * a * a;
          }
        }
      }
      for (int t = 0; t < 35; ++t) SumStat[(size_t)t + 35 * (size_t)(jc - 1)] += S[t] * inxz;
      for (int t = 0; t < 98; ++t) SumGrad[(size_t)t + 98 * (size_t)(jc - 1)] += G[t] * inxz;
    }
    {  // nyp only (:594-631)
      const int jc = nyp, jm = jc - 1;
      const double cac = rdyc(jc), InterpY1 = YinterpCoe(jc), InterpY2 = one - InterpY1;
      double S26 = 0, S32 = 0, S34 = 0, G[8] = {0};
      for (int kc = 1; kc <= nzc; ++kc)
        for (int ic = 1; ic <= nxc; ++ic) {
          const int is = ic - 2, im = ic - 1, ip = ic + 1;
          const F3& pr = pressure;
          double prloc2 = InterpY1 * (InterpCoe1 * pr(is, jm, kc) + InterpCoe2 * pr(im, jm, kc) + InterpCoe3 * pr(ic, jm, kc) + InterpCoe4 * pr(ip, jm, kc)) +
                          InterpY2 * (InterpCoe1 * pr(is, jc, kc) + InterpCoe2 * pr(im, jc, kc) + InterpCoe3 * pr(ic, jc, kc) + InterpCoe4 * pr(ip, jc, kc));
          double dudy = (ux(ic, jc, kc) - ux(ic, jm, kc)) * cac;
          double dwdy = (uz(ic, jc, kc) - uz(ic, jm, kc)) * cac;
          double vor_x = dwdy, vor_z = -dudy;
          S26 += prloc2 * (dudy + zero);
          S32 += vor_x * vor_x;
          S34 += vor_z * vor_z;
          G[0] += dudy; G[1] += dudy * dudy; G[2] += dudy * dudy * dudy; G[3] += dudy * dudy * dudy * dudy;
          G[4] += dwdy; G[5] += dwdy * dwdy; G[6] += dwdy * dwdy * dwdy; G[7] += dwdy * dwdy * dwdy * dwdy;
        }
      const size_t r = (size_t)(jc - 1);
      SumStat[26 + 35 * r] += S26 * inxz;
      SumStat[32 + 35 * r] += S32 * inxz;
      SumStat[34 + 35 * r] += S34 * inxz;
      for (int t = 0; t < 4; ++t) {
        SumGrad[6 + t + 98 * r] += G[t] * inxz;      // SumVec2(7..10): dudy
        SumGrad[30 + t + 98 * r] += G[4 + t] * inxz; // SumVec2(31..34): dwdy
      }
    }
    PrGradsum = PrGradsum + PrGradAver;
    nfstime += 1;
  }

  // ---- src/CFD_4th/m_FlowCase.f90:642-880 (clcStat, the 1-D spectra branch with
  //      clcSpectra1D: 18 x- and z-spectra per row: UU, VV, WW, PP energy spectra,
  //      UV and UV2 cospectra, and for UU, VV, WW, PP the linear coherence spectra
  //      R1, I1, R2 against the rows jForLCS(1:2)), with clcEnergySpectraX/Z and
  //      clcCospectraX/Z (:1152-1266), clcLTS_x/z (:1271-1632) and transform_uy
  //      (:2303-2332); R2HC transforms of every x and z line (FFTW_R2HC). ----
  std::vector<double> EnergySpecX, EnergySpecZ;  // (nxhp, nyc, 18), (nzhp, nyc, 18)
  std::vector<double> EnergySpec2D;              // (nxhp, nyc/2, nzhp, 9)
  int nSpectime = 0;
  void clcSpectra1D(int jFor1, int jFor2) {
    const int nxh = nxc / 2, nxhp = nxh + 1, nzh = nzc / 2, nzhp = nzh + 1;
    if (EnergySpecX.empty()) {
      EnergySpecX.assign((size_t)nxhp * nyc * 18, 0.0);
      EnergySpecZ.assign((size_t)nzhp * nyc * 18, 0.0);
      EnergySpec2D.assign((size_t)nxhp * (nyc / 2) * nzhp * 9, 0.0);
    }
    const size_t N3 = (size_t)nxc * nyc * nzc;
    auto I3 = [&](int ic, int jc, int kc) { return (size_t)(ic - 1) + (size_t)nxc * ((size_t)(jc - 1) + (size_t)nyc * (kc - 1)); };
    // the quantity arrays (interior, Fortran order)
    std::vector<double> qux(N3), quy(N3), quz(N3), qpr(N3), quxc(N3), quyc(N3);
    for (int kc = 1; kc <= nzc; ++kc)
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) {
          const size_t q = I3(ic, jc, kc);
          qux[q] = ux(ic, jc, kc) + uCRF;
          quxc[q] = InterpCoe1 * ux(ic - 1, jc, kc) + InterpCoe2 * ux(ic, jc, kc) + InterpCoe3 * ux(ic + 1, jc, kc) +
                    InterpCoe4 * ux(ic + 2, jc, kc) + uCRF;
          quyc[q] = half * (uy(ic, jc, kc) + uy(ic, jc + 1, kc));
          int jp = jc + 1;  // transform_uy, channel (FT_CH)
          if (jc > nyc / 2) jp = jc;
          quy[q] = uy(ic, jp, kc);
          quz[q] = uz(ic, jc, kc);
          qpr[q] = pressure(ic, jc, kc);
        }
    // R2HC of every x line and of every z line
    std::vector<cplx> ba, bb;
    auto hcx = [&](const std::vector<double>& a) {
      std::vector<double> h(a);
      for (int kc = 1; kc <= nzc; ++kc) for (int jc = 1; jc <= nyc; ++jc) r2hc(planx, &h[I3(1, jc, kc)], ba, bb);
      return h;
    };
    auto hcz = [&](const std::vector<double>& a) {
      std::vector<double> h(a), line(nzc);
      for (int jc = 1; jc <= nyc; ++jc)
        for (int ic = 1; ic <= nxc; ++ic) {
          for (int kc = 1; kc <= nzc; ++kc) line[kc - 1] = a[I3(ic, jc, kc)];
          r2hc(planz, line.data(), ba, bb);
          for (int kc = 1; kc <= nzc; ++kc) h[I3(ic, jc, kc)] = line[kc - 1];
        }
      return h;
    };
    const double normX = one / ((double)nxc * (double)nxc * (double)nzc);
    const double normZ = one / ((double)nxc * (double)nzc * (double)nzc);
    auto SX = [&](int ic, int jc, int m) -> double& { return EnergySpecX[(size_t)(ic - 1) + (size_t)nxhp * ((size_t)(jc - 1) + (size_t)nyc * m)]; };
    auto SZ = [&](int kc, int jc, int m) -> double& { return EnergySpecZ[(size_t)(kc - 1) + (size_t)nzhp * ((size_t)(jc - 1) + (size_t)nyc * m)]; };
    // clcEnergySpectraX / clcCospectraX (a == b for the energy spectra)
    auto cospX = [&](const std::vector<double>& a, const std::vector<double>& b, int m) {
      for (int jc = 1; jc <= nyc; ++jc) {
        std::vector<double> E(nxhp + 1, 0.0);
        for (int kc = 1; kc <= nzc; ++kc) {
          E[1] = E[1] + a[I3(1, jc, kc)] * b[I3(1, jc, kc)];
          E[nxhp] = E[nxhp] + a[I3(nxhp, jc, kc)] * b[I3(nxhp, jc, kc)];
          for (int ic = 2; ic <= nxh; ++ic) {
            const int icC = nxc + 2 - ic;
            E[ic] = E[ic] + (a[I3(ic, jc, kc)] * b[I3(ic, jc, kc)] + a[I3(icC, jc, kc)] * b[I3(icC, jc, kc)]) * two;
          }
        }
        for (int ic = 1; ic <= nxhp; ++ic) SX(ic, jc, m) = SX(ic, jc, m) + E[ic] * normX;
      }
    };
    auto cospZ = [&](const std::vector<double>& a, const std::vector<double>& b, int m) {
      for (int jc = 1; jc <= nyc; ++jc) {
        std::vector<double> E(nzhp + 1, 0.0);
        for (int ic = 1; ic <= nxc; ++ic) {
          E[1] = E[1] + a[I3(ic, jc, 1)] * b[I3(ic, jc, 1)];
          E[nzhp] = E[nzhp] + a[I3(ic, jc, nzhp)] * b[I3(ic, jc, nzhp)];
          for (int kc = 2; kc <= nzh; ++kc) {
            const int kcC = nzc + 2 - kc;
            E[kc] = E[kc] + (a[I3(ic, jc, kc)] * b[I3(ic, jc, kc)] + a[I3(ic, jc, kcC)] * b[I3(ic, jc, kcC)]) * two;
          }
        }
        for (int kc = 1; kc <= nzhp; ++kc) SZ(kc, jc, m) = SZ(kc, jc, m) + E[kc] * normZ;
      }
    };
    // clcLTS_x / clcLTS_z: products with the reference row (jForLCS, mirrored in the upper half)
    auto jref = [&](int jc, int jf) { return jc <= nyc / 2 ? jf : nyc + 1 - jf; };
    auto ltsX = [&](const std::vector<double>& h, int n1, int n2, int n3) {
      for (int jc = 1; jc <= nyc; ++jc) {
        std::vector<double> R1(nxhp + 1, 0.0), Im(nxhp + 1, 0.0), R2(nxhp + 1, 0.0);
        const int j1 = jref(jc, jFor1), j2 = jref(jc, jFor2);
        for (int kc = 1; kc <= nzc; ++kc) {
          R1[1] = R1[1] + h[I3(1, jc, kc)] * h[I3(1, j1, kc)];
          R1[nxhp] = R1[nxhp] + h[I3(nxhp, jc, kc)] * h[I3(nxhp, j1, kc)];
          R2[1] = R2[1] + h[I3(1, jc, kc)] * h[I3(1, j2, kc)];
          R2[nxhp] = R2[nxhp] + h[I3(nxhp, jc, kc)] * h[I3(nxhp, j2, kc)];
          for (int ic = 2; ic <= nxh; ++ic) {
            const int icC = nxc + 2 - ic;
            R1[ic] = R1[ic] + (h[I3(ic, jc, kc)] * h[I3(ic, j1, kc)] + h[I3(icC, jc, kc)] * h[I3(icC, j1, kc)]);
            Im[ic] = Im[ic] + (h[I3(icC, jc, kc)] * h[I3(ic, j1, kc)] - h[I3(ic, jc, kc)] * h[I3(icC, j1, kc)]);
            R2[ic] = R2[ic] + (h[I3(ic, jc, kc)] * h[I3(ic, j2, kc)] + h[I3(icC, jc, kc)] * h[I3(icC, j2, kc)]);
          }
        }
        for (int ic = 1; ic <= nxhp; ++ic) {
          SX(ic, jc, n1) = SX(ic, jc, n1) + R1[ic] * normX;
          SX(ic, jc, n2) = SX(ic, jc, n2) + Im[ic] * normX;
          SX(ic, jc, n3) = SX(ic, jc, n3) + R2[ic] * normX;
        }
      }
    };
    auto ltsZ = [&](const std::vector<double>& h, int n1, int n2, int n3) {
      for (int jc = 1; jc <= nyc; ++jc) {
        std::vector<double> R1(nzhp + 1, 0.0), Im(nzhp + 1, 0.0), R2(nzhp + 1, 0.0);
        const int j1 = jref(jc, jFor1), j2 = jref(jc, jFor2);
        for (int ic = 1; ic <= nxc; ++ic) {
          R1[1] = R1[1] + h[I3(ic, jc, 1)] * h[I3(ic, j1, 1)];
          R1[nzhp] = R1[nzhp] + h[I3(ic, jc, nzhp)] * h[I3(ic, j1, nzhp)];
          R2[1] = R2[1] + h[I3(ic, jc, 1)] * h[I3(ic, j2, 1)];
          R2[nzhp] = R2[nzhp] + h[I3(ic, jc, nzhp)] * h[I3(ic, j2, nzhp)];
          for (int kc = 2; kc <= nzh; ++kc) {
            const int kcC = nzc + 2 - kc;
            R1[kc] = R1[kc] + (h[I3(ic, jc, kc)] * h[I3(ic, j1, kc)] + h[I3(ic, jc, kcC)] * h[I3(ic, j1, kcC)]);
            Im[kc] = Im[kc] + (h[I3(ic, jc, kcC)] * h[I3(ic, j1, kc)] - h[I3(ic, jc, kc)] * h[I3(ic, j1, kcC)]);
            R2[kc] = R2[kc] + (h[I3(ic, jc, kc)] * h[I3(ic, j2, kc)] + h[I3(ic, jc, kcC)] * h[I3(ic, j2, kcC)]);
          }
        }
        for (int kc = 1; kc <= nzhp; ++kc) {
          SZ(kc, jc, n1) = SZ(kc, jc, n1) + R1[kc] * normZ;
          SZ(kc, jc, n2) = SZ(kc, jc, n2) + Im[kc] * normZ;
          SZ(kc, jc, n3) = SZ(kc, jc, n3) + R2[kc] * normZ;
        }
      }
    };
    // the order of :662-720 (x) and :786-849 (z); indices iSpec1D* - 1 (:43-60)
    {
      const std::vector<double> a = hcx(qux), b = hcx(quyc), f = hcx(quxc);
      cospX(a, a, 0); ltsX(a, 6, 7, 8); cospX(a, b, 5); cospX(f, b, 4);
      const std::vector<double> v = hcx(quy), w = hcx(quz), pp = hcx(qpr);
      cospX(v, v, 1); ltsX(v, 9, 10, 11);
      cospX(w, w, 2); ltsX(w, 12, 13, 14);
      cospX(pp, pp, 3); ltsX(pp, 15, 16, 17);
    }
    {
      const std::vector<double> a = hcz(qux), b = hcz(quyc), f = hcz(quxc);
      cospZ(a, a, 0); ltsZ(a, 6, 7, 8); cospZ(a, b, 5); cospZ(f, b, 4);
      const std::vector<double> v = hcz(quy), w = hcz(quz), pp = hcz(qpr);
      cospZ(v, v, 1); ltsZ(v, 9, 10, 11);
      cospZ(w, w, 2); ltsZ(w, 12, 13, 14);
      cospZ(pp, pp, 3); ltsZ(pp, 15, 16, 17);
    }
    // ---- 2-D spectra (clcSpecAndLCSR2DFrom1D :1896-2138, clcCosSpectra2D :2143-2298):
    //      the real part (ic = 1..nxhp) and the imaginary part (ic = 2..nxh, from
    //      nxc+2-ic) of every x spectrum transformed along z (R2HC); the two
    //      halves of the channel folded together (UV antisymmetric). ----
    {
      const int nyh = nyc / 2;
      const double norm2 = one / ((double)nxc * (double)nzc) / ((double)nxc * (double)nzc) * half;
      auto S2 = [&](int ic, int jc, int kc, int m) -> double& {
        return EnergySpec2D[(size_t)(ic - 1) + (size_t)nxhp * ((size_t)(jc - 1) + (size_t)nyh * ((size_t)(kc - 1) + (size_t)nzhp * m))];
      };
      // z transforms of the real and imaginary parts: (nxhp, nyc, nzc) each
      auto parts = [&](const std::vector<double>& h, std::vector<double>& R, std::vector<double>& I) {
        R.assign((size_t)nxhp * nyc * nzc, 0.0);
        I.assign((size_t)nxhp * nyc * nzc, 0.0);
        auto P3 = [&](int ic, int jc, int kc) { return (size_t)(ic - 1) + (size_t)nxhp * ((size_t)(jc - 1) + (size_t)nyc * (kc - 1)); };
        std::vector<double> lr(nzc), li(nzc);
        for (int jc = 1; jc <= nyc; ++jc)
          for (int ic = 1; ic <= nxhp; ++ic) {
            for (int kc = 1; kc <= nzc; ++kc) {
              lr[kc - 1] = h[I3(ic, jc, kc)];
              li[kc - 1] = (ic == 1 || ic == nxhp) ? zero : h[I3(nxc + 2 - ic, jc, kc)];
            }
            r2hc(planz, lr.data(), ba, bb);
            r2hc(planz, li.data(), ba, bb);
            for (int kc = 1; kc <= nzc; ++kc) { R[P3(ic, jc, kc)] = lr[kc - 1]; I[P3(ic, jc, kc)] = li[kc - 1]; }
          }
      };
      auto P3 = [&](int ic, int jc, int kc) { return (size_t)(ic - 1) + (size_t)nxhp * ((size_t)(jc - 1) + (size_t)nyc * (kc - 1)); };
      // sum over the real and imaginary parts of the z-spectrum products of rows j (A) and jb (B)
      auto prod = [&](const std::vector<double>& RA, const std::vector<double>& IA, const std::vector<double>& RB,
                      const std::vector<double>& IB, int ic, int j, int jb, int kc) {
        if (kc == 1 || kc == nzhp)
          return RA[P3(ic, j, kc)] * RB[P3(ic, jb, kc)] + IA[P3(ic, j, kc)] * IB[P3(ic, jb, kc)];
        const int kct = nzc + 2 - kc;
        return RA[P3(ic, j, kc)] * RB[P3(ic, jb, kc)] + RA[P3(ic, j, kct)] * RB[P3(ic, jb, kct)] +
               IA[P3(ic, j, kc)] * IB[P3(ic, jb, kc)] + IA[P3(ic, j, kct)] * IB[P3(ic, jb, kct)];
      };
      auto acc2 = [&](const std::vector<double>& RA, const std::vector<double>& IA, const std::vector<double>& RB,
                      const std::vector<double>& IB, int m, bool lcs, double rCoe) {
        for (int jc = 1; jc <= nyh; ++jc) {
          const int jcs = nyc + 1 - jc;
          const int ja = lcs ? jFor1 : jc, jb = lcs ? nyc + 1 - jFor1 : jcs;
          for (int kc = 1; kc <= nzhp; ++kc)
            for (int ic = 1; ic <= nxhp; ++ic)
              S2(ic, jc, kc, m) = S2(ic, jc, kc, m) +
                                  norm2 * (prod(RA, IA, RB, IB, ic, jc, ja, kc) + rCoe * prod(RA, IA, RB, IB, ic, jcs, jb, kc));
        }
      };
      std::vector<double> R1, I1, R2, I2;
      parts(hcx(qux), R1, I1);
      acc2(R1, I1, R1, I1, 0, false, one); acc2(R1, I1, R1, I1, 5, true, one);
      parts(hcx(quxc), R1, I1);
      parts(hcx(quyc), R2, I2);
      acc2(R1, I1, R2, I2, 4, false, -one);
      const std::vector<double>* qs[3] = {&quy, &quz, &qpr};
      for (int q = 0; q < 3; ++q) {
        parts(hcx(*qs[q]), R1, I1);
        acc2(R1, I1, R1, I1, 1 + q, false, one);
        acc2(R1, I1, R1, I1, 6 + q, true, one);
      }
    }
    nSpectime += 1;
  }

  F3* field(int id) {
    switch (id) {
      case 0: return &ux; case 1: return &uy; case 2: return &uz; case 3: return &pressure;
      case 4: return &HistX; case 5: return &HistY; case 6: return &HistZ;
      case 7: return &RealArr1; case 8: return &RealArr2; case 9: return &RealHalo; case 10: return &nut;
    }
    return nullptr;
  }
};

}  // namespace

extern "C" {

void* orc_create(const orc_params* p) {
  if (!p || p->nxc < 2 || p->nyc < 2 || p->nzc < 2) return nullptr;
  Oracle* o = new Oracle();
  o->init(p);
  return o;
}

void orc_destroy(void* h) { delete (Oracle*)h; }

// LES eddy viscosity of the current state (Clc_SGS_Vis); returns u_tau of the
// Smagorinsky / van Driest model (0 for the others)
double orc_sgs(void* h) {
  Oracle* o = (Oracle*)h;
  o->utau_last = 0;
  o->Clc_SGS_Vis();
  return o->utau_last;
}

// learned closure: cell-centred SGS stresses (6 interior arrays, or NULL to
// clear) whose divergence the LES right-hand sides add
void orc_set_sgs_tau(void* h, const double* tau) {
  Oracle* o = (Oracle*)h;
  const size_t N = (size_t)o->nxc * o->nyc * o->nzc;
  if (!tau) { o->sgs_tau.clear(); o->sgs_f.clear(); return; }
  o->sgs_tau.assign(tau, tau + 6 * N);
  o->SgsForce();
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// y grid yp(1..nyp) and the metric vectors, for cross-checking the product's own mesh code.
void orc_get_mesh(void* h, double* yp_out, double* yc_out, double* dyp_out, double* dyc_out) {
  Oracle* o = (Oracle*)h;
  for (int j = 1; j <= o->nyp; ++j) {
    if (yp_out) yp_out[j - 1] = o->yp(j);
    if (yc_out) yc_out[j - 1] = o->yc(j);
    if (dyp_out) dyp_out[j - 1] = o->dyp(j);
    if (dyc_out) dyc_out[j - 1] = o->dyc(j);
  }
}

// Interior (nxc,nyc,nzc) Fortran-order state, as in the restart file
// (src/CFD_2nd/m_IOAndVisu.f90:352-438).  hist may be NULL.  Afterwards the
// ghost cells are rebuilt like ChannelInitialize (m_ChannelSystem.f90:57-63).
void orc_set_state(void* h, const double* ux, const double* uy, const double* uz, const double* p, const double* hist) {
  Oracle* o = (Oracle*)h;
  size_t N = (size_t)o->nxc * o->nyc * o->nzc;
  size_t q = 0;
  for (int k = 1; k <= o->nzc; ++k) for (int j = 1; j <= o->nyc; ++j) for (int i = 1; i <= o->nxc; ++i, ++q) {
    o->ux(i, j, k) = ux[q]; o->uy(i, j, k) = uy[q]; o->uz(i, j, k) = uz[q]; o->pressure(i, j, k) = p[q];
    if (hist) { o->HistX(i, j, k) = hist[q]; o->HistY(i, j, k) = hist[N + q]; o->HistZ(i, j, k) = hist[2 * N + q]; }
    else { o->HistX(i, j, k) = 0; o->HistY(i, j, k) = 0; o->HistZ(i, j, k) = 0; }
  }
  o->Update_uy_ym();
  if (o->o4) {
    o->SetBC_and_UpdateHalo4();
    o->SetBC_and_UpdateHalo_pr4(o->pressure);
  } else {
    o->SetBC_and_UpdateHalo();
    o->SetBC_and_UpdateHalo_pr(o->pressure);
  }
  std::fill(o->RealArr1.a.begin(), o->RealArr1.a.end(), 0.0);
  std::fill(o->RealArr2.a.begin(), o->RealArr2.a.end(), 0.0);
  o->SimTime = 0; o->dt = o->P.dtMax; o->itime = 0;
}

void orc_get_state(void* h, double* ux, double* uy, double* uz, double* p, double* hist) {
  Oracle* o = (Oracle*)h;
  size_t N = (size_t)o->nxc * o->nyc * o->nzc;
  size_t q = 0;
  for (int k = 1; k <= o->nzc; ++k) for (int j = 1; j <= o->nyc; ++j) for (int i = 1; i <= o->nxc; ++i, ++q) {
    if (ux) ux[q] = o->ux(i, j, k);
    if (uy) uy[q] = o->uy(i, j, k);
    if (uz) uz[q] = o->uz(i, j, k);
    if (p) p[q] = o->pressure(i, j, k);
    if (hist) { hist[q] = o->HistX(i, j, k); hist[N + q] = o->HistY(i, j, k); hist[2 * N + q] = o->HistZ(i, j, k); }
  }
}

// Full array with its ghost cells (Fortran order over the allocated bounds).
// Returns the number of doubles written, or the needed size when out is NULL.
long long orc_get_array(void* h, int id, double* out) {
  Oracle* o = (Oracle*)h;
  F3* f = o->field(id);
  if (!f) return -1;
  if (out) std::memcpy(out, f->a.data(), f->a.size() * sizeof(double));
  return (long long)f->a.size();
}

long long orc_set_array(void* h, int id, const double* in) {
  Oracle* o = (Oracle*)h;
  F3* f = o->field(id);
  if (!f) return -1;
  std::memcpy(f->a.data(), in, f->a.size() * sizeof(double));
  return (long long)f->a.size();
}

void orc_set_dt(void* h, double dt) { ((Oracle*)h)->dt = dt; }

// ---- Tool/interpolateField/src/m_Interp.f90:20-179 (Interp_init, one rank) and
//      :184-361 (Interp_uvwp): trilinear resampling of the state of `src` onto the
//      grid of `dst` (same yly; x and z in coordinates normalised by the domain
//      length, Tool/interpolateField/src/m_MeshAndMetries.f90:40-59), with the
//      tool's ghost rules on the old grid (Tool/interpolateField/src/m_BC_and_Halo.f90:
//      21-340, periodic x and z), ux rescaled to ubulk when IsUxConst.  The result
//      becomes dst's state (as a restart read, orc_set_state; Hist zero). ----
void orc_interp(void* hdst, void* hsrc) {
  Oracle* N = (Oracle*)hdst;
  Oracle* O = (Oracle*)hsrc;
  const int nxo = O->nxc, nyo = O->nyc, nzo = O->nzc, nxn = N->nxc, nyn = N->nyc, nzn = N->nzc;
  const int nypo = nyo + 1;
  // normalised x/z point and centre coordinates
  auto pts = [](int n, std::vector<double>& xp, std::vector<double>& xc) {
    xp.assign(n + 2, 0.0); xc.assign(n + 2, 0.0);
    for (int j = 1; j <= n + 1; ++j) xp[j] = (double)(j - 1) / (double)n;
    xp[1] = 0.0; xp[n + 1] = 1.0;
    for (int j = 1; j <= n; ++j) xc[j] = 0.5 * (xp[j] + xp[j + 1]);
    xc[0] = 2.0 * xp[1] - xc[1];
    xc[n + 1] = 2.0 * xp[n + 1] - xc[n];
  };
  std::vector<double> xpO, xcO, xpN, xcN, zpO, zcO, zpN, zcN;
  pts(nxo, xpO, xcO); pts(nxn, xpN, xcN); pts(nzo, zpO, zcO); pts(nzn, zpN, zcN);
  std::vector<double> ypO(nypo + 1), ycO(nypo + 1), ypN(nyn + 2), ycN(nyn + 2);
  for (int j = 1; j <= nypo; ++j) ypO[j] = O->yp(j);
  for (int j = 1; j <= nyn + 1; ++j) ypN[j] = N->yp(j);
  for (int j = 1; j <= nyo; ++j) ycO[j] = 0.5 * (ypO[j] + ypO[j + 1]);
  ycO[0] = 2.0 * ypO[1] - ycO[1]; ycO[nypo] = 2.0 * ypO[nypo] - ycO[nyo];
  for (int j = 1; j <= nyn; ++j) ycN[j] = 0.5 * (ypN[j] + ypN[j + 1]);
  // index and ratio tables (Interp_init :130-179)
  auto xtab = [](int nn, int no, const std::vector<double>& pN, const std::vector<double>& pO, bool centred,
                 std::vector<int>& ind, std::vector<double>& rat) {
    ind.assign(nn + 1, 0); rat.assign(nn + 1, 0.0);
    const double rd = (double)no;
    for (int i = 1; i <= nn; ++i) {
      int ic = (int)std::floor(pN[i] * rd) + 1;
      ic = std::min(ic, no); ic = std::max(ic, 1);
      if (centred && pN[i] < pO[ic]) ic = ic - 1;
      ind[i] = ic; rat[i] = (pO[ic + 1] - pN[i]) * rd;
    }
  };
  std::vector<int> ixp, ixc, izp, izc, iyp(nyn + 1), iyc(nyn + 1);
  std::vector<double> rxp, rxc, rzp, rzc, ryp(nyn + 1), ryc(nyn + 1);
  xtab(nxn, nxo, xpN, xpO, false, ixp, rxp); xtab(nxn, nxo, xcN, xcO, true, ixc, rxc);
  xtab(nzn, nzo, zpN, zpO, false, izp, rzp); xtab(nzn, nzo, zcN, zcO, true, izc, rzc);
  auto ysearch = [&](double y) {  // largest jc in 0..nypo with ypO(jc) <= y (bisection of :148-156)
    int js = 0, je = nypo + 1, jc;
    for (;;) {
      jc = (js + je) / 2;
      if (je - js == 1) break;
      if (y < ypO[jc]) je = jc; else js = jc;
    }
    return jc;
  };
  for (int j = 1; j <= nyn; ++j) {
    int jc = ysearch(ypN[j]);
    iyp[j] = jc; ryp[j] = (ypO[jc + 1] - ypN[j]) / (ypO[jc + 1] - ypO[jc]);
    jc = ysearch(ycN[j]);
    if (ycN[j] < ycO[jc]) jc = jc - 1;
    iyc[j] = jc; ryc[j] = (ycO[jc + 1] - ycN[j]) / (ycO[jc + 1] - ycO[jc]);
  }
  // the old state with the tool's ghosts, bounds (0:nxc+1, 0:nyc+1, 0:nzc+1)
  const int* Bc = O->P.BcOption;
  auto ghosted = [&](const F3& a, int comp) {
    F3 g;
    g.init(0, nxo + 1, 0, nyo + 1, 0, nzo + 1);
    for (int k = 1; k <= nzo; ++k) for (int j = 1; j <= nyo; ++j) for (int i = 1; i <= nxo; ++i) g(i, j, k) = a(i, j, k);
    for (int k = 1; k <= nzo; ++k)
      for (int i = 1; i <= nxo; ++i) {
        if (comp == 3) { g(i, nypo, k) = g(i, nyo, k); g(i, 0, k) = g(i, 1, k); continue; }
        if (comp == 1) {
          g(i, nypo, k) = Bc[3] == -1 ? O->P.uyBcValue[3] : 0.0;
          g(i, 1, k) = Bc[2] == -1 ? O->P.uyBcValue[2] : 0.0;
          continue;
        }
        const double* w = comp == 0 ? O->P.uxBcValue : O->P.uzBcValue;
        g(i, nypo, k) = Bc[3] == -1 ? w[3] * 2.0 - g(i, nyo, k) : g(i, nyo, k);
        g(i, 0, k) = Bc[2] == -1 ? w[2] * 2.0 - g(i, 1, k) : g(i, 1, k);
      }
    for (int k = 1; k <= nzo; ++k) for (int j = 0; j <= nypo; ++j) { g(0, j, k) = g(nxo, j, k); g(nxo + 1, j, k) = g(1, j, k); }
    for (int j = 0; j <= nypo; ++j) for (int i = 0; i <= nxo + 1; ++i) { g(i, j, 0) = g(i, j, nzo); g(i, j, nzo + 1) = g(i, j, 1); }
    return g;
  };
  const size_t Nn = (size_t)nxn * nyn * nzn;
  std::vector<double> out[4];
  for (int comp = 0; comp < 4; ++comp) {
    const F3& src = comp == 0 ? O->ux : comp == 1 ? O->uy : comp == 2 ? O->uz : O->pressure;
    const F3 A = ghosted(src, comp);
    const std::vector<int>& IX = comp == 0 ? ixp : ixc;
    const std::vector<double>& RX = comp == 0 ? rxp : rxc;
    const std::vector<int>& IY = comp == 1 ? iyp : iyc;
    const std::vector<double>& RY = comp == 1 ? ryp : ryc;
    const std::vector<int>& IZ = comp == 2 ? izp : izc;
    const std::vector<double>& RZ = comp == 2 ? rzp : rzc;
    out[comp].assign(Nn, 0.0);
    for (int kc = 1; kc <= nzn; ++kc) {
      const int idz1 = IZ[kc], idz2 = idz1 + 1;
      const double prz1 = RZ[kc], prz2 = one - prz1;
      for (int jc = 1; jc <= nyn; ++jc) {
        const int idy1 = IY[jc], idy2 = idy1 + 1;
        const double pry1 = RY[jc], pry2 = one - pry1;
        for (int ic = 1; ic <= nxn; ++ic) {
          const int idx1 = IX[ic], idx2 = idx1 + 1;
          const double prx1 = RX[ic], prx2 = one - prx1;
          out[comp][(size_t)(ic - 1) + (size_t)nxn * ((size_t)(jc - 1) + (size_t)nyn * (kc - 1))] =
              A(idx1, idy1, idz1) * prx1 * pry1 * prz1 + A(idx2, idy1, idz1) * prx2 * pry1 * prz1 +
              A(idx1, idy2, idz1) * prx1 * pry2 * prz1 + A(idx2, idy2, idz1) * prx2 * pry2 * prz1 +
              A(idx1, idy1, idz2) * prx1 * pry1 * prz2 + A(idx2, idy1, idz2) * prx2 * pry1 * prz2 +
              A(idx1, idy2, idz2) * prx1 * pry2 * prz2 + A(idx2, idy2, idz2) * prx2 * pry2 * prz2;
        }
      }
    }
  }
  if (N->P.IsUxConst) {  // :225-236
    double MeanValue = zero;
    for (int kc = 1; kc <= nzn; ++kc)
      for (int jc = 1; jc <= nyn; ++jc)
        for (int ic = 1; ic <= nxn; ++ic)
          MeanValue = MeanValue + out[0][(size_t)(ic - 1) + (size_t)nxn * ((size_t)(jc - 1) + (size_t)nyn * (kc - 1))] *
                                      (ypN[jc + 1] - ypN[jc]);
    MeanValue = MeanValue / (double)nxn / (double)nzn / N->P.yly;
    const double s = N->P.ubulk / MeanValue;
    for (double& v : out[0]) v = s * v;
  }
  orc_set_state(hdst, out[0].data(), out[1].data(), out[2].data(), out[3].data(), nullptr);
}

void orc_stage(void* h, int st, int ns) { ((Oracle*)h)->stage(st, ns); }

int orc_step(void* h, int nsteps, orc_info* info) {
  Oracle* o = (Oracle*)h;
  int st = 0;
  for (int s = 0; s < nsteps; ++s) {
    st = o->ChannelIterate(info);
    if (st) break;
  }
  return st;
}

// Standalone Poisson solve: src and phi interior (nxc,nyc,nzc) arrays.
void orc_poisson(void* h, const double* src, double* phi) {
  Oracle* o = (Oracle*)h;
  size_t q = 0;
  for (int k = 1; k <= o->nzc; ++k) for (int j = 1; j <= o->nyc; ++j) for (int i = 1; i <= o->nxc; ++i, ++q)
    o->RealArr1(i, j, k) = src[q];
  o->clcPPE(o->RealArr1, o->RealHalo);
  q = 0;
  for (int k = 1; k <= o->nzc; ++k) for (int j = 1; j <= o->nyc; ++j) for (int i = 1; i <= o->nxc; ++i, ++q)
    phi[q] = o->RealHalo(i, j, k);
}

// FFTW-convention r2r transforms of one line, for known-answer tests.
void orc_r2hc(int n, double* x) {
  FFTPlan pl; pl.init(n);
  std::vector<cplx> a, b;
  r2hc(pl, x, a, b);
}
void orc_hc2r(int n, double* x) {
  FFTPlan pl; pl.init(n);
  std::vector<cplx> a, b;
  hc2r(pl, x, a, b);
}
// FFTW-convention cosine transforms (REDFT10, REDFT01) of one line, for known-answer tests.
void orc_redft10(int n, double* x) {
  std::vector<double> b;
  redft10(n, x, dct_table(n), b);
}
void orc_redft01(int n, double* x) {
  std::vector<double> b;
  redft01(n, x, dct_table(n), b);
}

double orc_dissipation(void* h) { return ((Oracle*)h)->TGDissipation(); }

void orc_stats_accumulate(void* h) {
  Oracle* o = (Oracle*)h;
  if (o->o4) o->clcStat4();
  else o->clcStat_CH();
}

// 1-D spectra of the 4th-order statistics (clcSpectra1D) at the current state.
void orc_spectra_accumulate(void* h, int jFor1, int jFor2) { ((Oracle*)h)->clcSpectra1D(jFor1, jFor2); }

// EnergySpecX(nxhp,nyc,18) and EnergySpecZ(nzhp,nyc,18) sums; returns nSpectime.
int orc_spectra_get(void* h, double* specx, double* specz) {
  Oracle* o = (Oracle*)h;
  const size_t nx = (size_t)(o->nxc / 2 + 1) * o->nyc * 18, nz = (size_t)(o->nzc / 2 + 1) * o->nyc * 18;
  for (size_t q = 0; q < nx; ++q) specx[q] = o->EnergySpecX.empty() ? 0.0 : o->EnergySpecX[q];
  for (size_t q = 0; q < nz; ++q) specz[q] = o->EnergySpecZ.empty() ? 0.0 : o->EnergySpecZ[q];
  return o->nSpectime;
}

// EnergySpec2D(nxhp, nyc/2, nzhp, 9) sums; returns nSpectime.
int orc_spectra_get2d(void* h, double* spec2d) {
  Oracle* o = (Oracle*)h;
  const size_t n = (size_t)(o->nxc / 2 + 1) * (o->nyc / 2) * (o->nzc / 2 + 1) * 9;
  for (size_t q = 0; q < n; ++q) spec2d[q] = o->EnergySpec2D.empty() ? 0.0 : o->EnergySpec2D[q];
  return o->nSpectime;
}

// SumGrad(98,nyp) of the 4th-order statistics (zeros before the first accumulation);
// returns nfstime.
int orc_stats_get_grad(void* h, double* sumgrad) {
  Oracle* o = (Oracle*)h;
  for (size_t q = 0; q < (size_t)98 * o->nyp; ++q) sumgrad[q] = o->SumGrad.empty() ? 0.0 : o->SumGrad[q];
  return o->nfstime;
}

// SumStat (35 x nyp, Fortran order), nfstime and PrGradsum.
int orc_stats_get(void* h, double* sumstat, double* prgradsum) {
  Oracle* o = (Oracle*)h;
  if (sumstat) std::memcpy(sumstat, o->SumStat.data(), o->SumStat.size() * sizeof(double));
  if (prgradsum) *prgradsum = o->PrGradsum;
  return o->nfstime;
}

}  // extern "C"
