// ch3d_api.cu -- host side of the C ABI declared in include/ch3d.h.
//
// Replaces, for one GPU, the start-up and time-step call sites of the
// reference (src/CFD_2nd/m_ChannelSystem.f90:28-154): metric vectors are built
// on the host exactly as InitMeshAndMetries does, uploaded once, and the whole
// RK3 step runs on the device as one captured CUDA graph.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/ch3d_mlp.h"
#include "ch3d_ctx.h"

using namespace ch3d;

namespace {

thread_local std::string g_err = "";

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CU(x)                                                                                  \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess) return fail(CH3D_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_));   \
  } while (0)

const double PI = 3.141592653589793238462643383279502884;

// src/CFD_2nd/m_MeshAndMetries.f90:292-360 (clcCoord), 1-based yp
void mesh_section(double* yp1, int id1, int id2, double c1, double c2, int StretType, double cStret, int StretOption) {
  double* yp = yp1 - 1;  // yp[j] with Fortran j
  int m = id2 - id1;
  double secLen = c2 - c1;
  yp[id1] = c1; yp[id2] = c2;
  switch (StretType) {
    case 0:
      for (int j = 0; j <= m; ++j) yp[id1 + j] = c1 + (double)j / (double)m * secLen;
      break;
    case 1: {
      double tstr = std::tanh(cStret);
      for (int j = 0; j <= m; ++j) {
        double xi = (double)j / (double)(float)m;  // real(m) is default (single) kind
        double setCrd = std::tanh(cStret * (xi - 1.0)) / tstr + 1.0;
        if (StretOption == 0) yp[id1 + j] = c1 + setCrd * secLen;
        else yp[id2 - j] = c2 - setCrd * secLen;
      }
      break;
    }
    case 2: {
      double tstr = std::sin(0.5 * cStret * PI);
      for (int j = 0; j <= m; ++j) {
        double xi = (double)j / (double)m - 1.0;
        double setCrd = std::sin(cStret * xi * PI * 0.5) / tstr + 1.0;
        if (StretOption == 0) yp[id1 + j] = c1 + setCrd * secLen;
        else yp[id2 - j] = c2 - setCrd * secLen;
      }
      break;
    }
    case 3: {
      if (cStret == 1.0) {
        for (int j = 0; j <= m; ++j) yp[j + id1] = c1 + (double)j / (double)m * secLen;
      } else {
        double tstr = (std::pow(cStret, m) - 1.0) / (cStret - 1.0);
        for (int j = 0; j <= m - 1; ++j) {
          double setCrd = std::pow(cStret, j) / tstr;
          if (StretOption == 0) yp[id1 + j + 1] = yp[id1 + j] + setCrd * secLen;
          else yp[id2 - j - 1] = yp[id2 - j] - setCrd * secLen;
        }
      }
      break;
    }
  }
  yp[id1] = c1; yp[id2] = c2;
}

bool factor23(int n, FFTPlanDev& pl) {
  pl.n = n; pl.npass = 0;
  int m = n;
  while (m % 4 == 0) { pl.radix[pl.npass++] = 4; m /= 4; }
  while (m % 2 == 0) { pl.radix[pl.npass++] = 2; m /= 2; }
  while (m % 3 == 0) { pl.radix[pl.npass++] = 3; m /= 3; }
  int Ns = 1;
  for (int p = 0; p < pl.npass; ++p) {
    pl.mNB[p] = fdiv_magic((unsigned)(n / pl.radix[p]));
    pl.mNs[p] = fdiv_magic((unsigned)Ns);
    Ns *= pl.radix[p];
  }
  return m == 1 && pl.npass <= CH3D_MAX_PASSES && n < (1 << 16);
}

template <class CT>
std::vector<CT> twiddles(int n, int count) {
  std::vector<CT> w(count);
  for (int q = 0; q < count; ++q) {
    long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)q / (long double)n;
    w[q].x = (decltype(w[q].x))cosl(ang);
    w[q].y = (decltype(w[q].y))sinl(ang);
  }
  return w;
}

enum { NMET = 17 };

// Host-side restatement of src/CFD_2nd/m_MeshAndMetries.f90:171-286 and the
// CN metrics of src/CFD_2nd/m_TScheme.f90:73-85.
void build_metrics(ch3d_ctx* c) {
  const ch3d_config& g = c->cfg;
  const int nyc = c->ny, nyp = nyc + 1, L = nyc + 3;
  auto vec = [&](std::vector<double>& v) { v.assign(L, 0.0); };
  vec(c->yc); vec(c->dyp); vec(c->dyc); vec(c->rdyp); vec(c->rdyc); vec(c->yinterp);
  vec(c->ap2c); vec(c->ac2c); vec(c->am2c); vec(c->ap2p); vec(c->ac2p); vec(c->am2p);
  vec(c->ap2Pr); vec(c->ac2Pr); vec(c->am2Pr); vec(c->am2cForCN); vec(c->ap2cForCN); vec(c->s1coe);
  std::vector<double>& yp = c->yp;
  for (int j = 1; j <= nyc; ++j) c->yc[j] = 0.5 * (yp[j] + yp[j + 1]);
  c->yc[0] = 2.0 * yp[1] - c->yc[1];
  c->yc[nyp] = 2.0 * yp[nyp] - c->yc[nyc];
  for (int j = 1; j <= nyc; ++j) c->dyp[j] = yp[j + 1] - yp[j];
  c->dyp[0] = c->dyp[1]; c->dyp[nyp] = c->dyp[nyc];
  for (int j = 2; j <= nyc; ++j) c->dyc[j] = c->yc[j] - c->yc[j - 1];
  c->dyc[1] = c->dyp[1]; c->dyc[nyp] = c->dyp[nyc];
  for (int j = 0; j <= nyp; ++j) c->rdyp[j] = 1.0 / c->dyp[j];
  for (int j = 1; j <= nyp; ++j) c->rdyc[j] = 1.0 / c->dyc[j];
  for (int j = 1; j <= nyp; ++j) c->yinterp[j] = c->dyp[j] / (c->dyp[j] + c->dyp[j - 1]);
  const int* Bc = g.BcOption;
  for (int j = 1; j <= nyc; ++j) { c->am2Pr[j] = c->rdyp[j] * c->rdyc[j]; c->ap2Pr[j] = c->rdyp[j] * c->rdyc[j + 1]; }
  if (Bc[2] != 0) { c->am2Pr[1] = 0.0; c->ap2Pr[1] = c->rdyp[1] * c->rdyc[2]; }
  if (Bc[3] != 0) { c->am2Pr[nyc] = c->rdyp[nyc] * c->rdyc[nyc]; c->ap2Pr[nyc] = 0.0; }
  for (int j = 1; j <= nyc; ++j) c->ac2Pr[j] = -(c->am2Pr[j] + c->ap2Pr[j]);
  for (int j = 1; j <= nyc; ++j) { c->am2c[j] = c->rdyp[j] * c->rdyc[j]; c->ap2c[j] = c->rdyp[j] * c->rdyc[j + 1]; }
  if (Bc[2] == -1) {
    c->am2c[1] = 4.0 * c->rdyc[1] / (c->dyc[1] + 2.0 * c->dyc[2]);
    c->ap2c[1] = 4.0 * c->rdyc[2] / (c->dyc[1] + 2.0 * c->dyc[2]);
  }
  if (Bc[3] == -1) {
    c->am2c[nyc] = 4.0 * c->rdyc[nyc] / (c->dyc[nyp] + 2.0 * c->dyc[nyc]);
    c->ap2c[nyc] = 4.0 * c->rdyc[nyp] / (c->dyc[nyp] + 2.0 * c->dyc[nyc]);
  }
  for (int j = 1; j <= nyc; ++j) c->ac2c[j] = -(c->am2c[j] + c->ap2c[j]);
  for (int j = 1; j <= nyc; ++j) { c->am2p[j] = c->rdyc[j] * c->rdyp[j - 1]; c->ap2p[j] = c->rdyc[j] * c->rdyp[j]; }
  for (int j = 1; j <= nyc; ++j) c->ac2p[j] = -(c->am2p[j] + c->ap2p[j]);
  for (int j = 1; j <= nyc; ++j) { c->ap2cForCN[j] = c->ap2c[j]; c->am2cForCN[j] = c->am2c[j]; }
  if (Bc[2] == -1) c->am2cForCN[1] = 2.0 * c->am2c[1]; else if (Bc[2] == -2) c->am2cForCN[1] = 0.0;
  if (Bc[3] == -1) c->ap2cForCN[nyc] = 2.0 * c->ap2c[nyc]; else if (Bc[3] == -2) c->ap2cForCN[nyc] = 0.0;
  // bulk-velocity weights (clcRhsX_PIMP, src/CFD_2nd/m_TSchemePIMP_inc.f90:25-27)
  for (int j = 1; j <= nyc; ++j) {
    double w = c->dyp[j];
    if (c->yc[j] < g.ybulk1 || c->yc[j] >= g.ybulk2) w = 0.0;
    c->s1coe[j] = w;
  }
  // x, z (uniform, periodic)
  c->dx = g.xlx / (double)c->nx; c->dz = g.zlz / (double)c->nz;
  c->rdx = (double)c->nx / g.xlx; c->rdz = (double)c->nz / g.zlz;
  c->rdx2 = c->rdx * c->rdx; c->rdz2 = c->rdz * c->rdz;
  double rdy = (double)nyc / g.yly;
  c->rdy2 = rdy * rdy;
  // modified wavenumbers, src/CFD_2nd/m_Poisson.f90:38-66
  c->WaveNumX.assign(c->nx, 0.0);
  c->WaveNumZ.assign(c->nz, 0.0);
  for (int i = 1; i <= c->nx; ++i) c->WaveNumX[i - 1] = 2.0 * c->rdx2 * (std::cos(2.0 * PI * (double)(i - 1) / (double)c->nx) - 1.0);
  for (int k = 1; k <= c->nz; ++k) c->WaveNumZ[k - 1] = 2.0 * c->rdz2 * (std::cos(2.0 * PI * (double)(k - 1) / (double)c->nz) - 1.0);
  if (g.order == 4) {
    // 4th-order modified wavenumbers, src/CFD_4th/m_Poisson.f90:40-47
    for (int i = 1; i <= c->nx; ++i) {
      const double wa = 2.0 * PI * (double)(i - 1) / (double)c->nx;
      c->WaveNumX[i - 1] = c->rdx2 / 288.0 * (std::cos(3.0 * wa) - 54.0 * std::cos(2.0 * wa) + 783.0 * std::cos(wa) - 730.0);
    }
    for (int k = 1; k <= c->nz; ++k) {
      const double wa = 2.0 * PI * (double)(k - 1) / (double)c->nz;
      c->WaveNumZ[k - 1] = c->rdz2 / 288.0 * (std::cos(3.0 * wa) - 54.0 * std::cos(2.0 * wa) + 783.0 * std::cos(wa) - 730.0);
    }
  }
  c->normfft = 1.0 / ((double)c->nx * (double)c->nz);
}

template <class T>
void pack_metrics(const ch3d_ctx* c, std::vector<T>& out) {
  const int L = c->ny + 3;
  out.assign((size_t)NMET * L, (T)0);
  const std::vector<double>* v[NMET] = {&c->dyp,   &c->rdyp,  &c->rdyc,  &c->yinterp,   &c->ap2c,      &c->ac2c,
                                        &c->am2c,  &c->ap2p,  &c->ac2p,  &c->am2p,      &c->ap2Pr,     &c->ac2Pr,
                                        &c->am2Pr, &c->s1coe, &c->ap2cForCN, &c->am2cForCN, &c->yc};
  for (int q = 0; q < NMET; ++q)
    for (int j = 0; j < L; ++j) out[(size_t)q * L + j] = (T)(*v[q])[j];
}

template <class T>
Metrics<T> metrics_ptrs(const T* base, int ny) {
  const int L = ny + 3;
  Metrics<T> m;
  m.dyp = base + 0 * L; m.rdyp = base + 1 * L; m.rdyc = base + 2 * L; m.yinterp = base + 3 * L;
  m.ap2c = base + 4 * L; m.ac2c = base + 5 * L; m.am2c = base + 6 * L;
  m.ap2p = base + 7 * L; m.ac2p = base + 8 * L; m.am2p = base + 9 * L;
  m.ap2Pr = base + 10 * L; m.ac2Pr = base + 11 * L; m.am2Pr = base + 12 * L;
  m.s1coe = base + 13 * L;
  return m;
}

int check_config(const ch3d_config* g) {
  if (!g) return fail(CH3D_ERR_INVALID, "config is NULL");
  if (g->order != 2 && g->order != 4) return fail(CH3D_ERR_INVALID, "order must be 2 or 4");
  if (g->order == 4 && (g->FlowType != 1 || g->BcOption[2] != -1 || g->BcOption[3] != -1))
    return fail(CH3D_ERR_UNSUPPORTED, "the 4th-order solver is built for the channel (FlowType=1, no-slip walls)");
  if (g->nxc < 4 || g->nyc < 4 || g->nzc < 2) return fail(CH3D_ERR_INVALID, "grid too small: %d %d %d", g->nxc, g->nyc, g->nzc);
  if (g->nxc % 2) return fail(CH3D_ERR_INVALID, "nxc must be even (real-to-complex x transform)");
  if (g->ischeme < 1 || g->ischeme > 3) return fail(CH3D_ERR_INVALID, "Time scheme WRONG!!! ischeme=%d", g->ischeme);
  if (g->IsImplicit != 1 && !(g->order == 2 && (g->IsImplicit == 2 || g->IsImplicit == 0)))
    return fail(CH3D_ERR_UNSUPPORTED, "IsImplicit=%d not built (PIMP=1; FIMP=2 and FEXP=0 for order 2)", g->IsImplicit);
  if (g->BcOption[0] != 0 || g->BcOption[1] != 0 || g->BcOption[4] != 0 || g->BcOption[5] != 0)
    return fail(CH3D_ERR_UNSUPPORTED, "x and z must be periodic (BcOption 1,2,5,6 = 0)");
  if ((g->BcOption[2] == 0) != (g->BcOption[3] == 0)) return fail(CH3D_ERR_INVALID, "Periodic Bc Wrong");
  for (int s = 2; s < 4; ++s)
    if (g->BcOption[s] != -1 && g->BcOption[s] != -2 && g->BcOption[s] != 0)
      return fail(CH3D_ERR_UNSUPPORTED, "y boundaries must be no-slip (-1), free-slip (-2) or periodic (0)");
  // periodic y: the triply periodic steps (clcU*Hat_FIMP_000, clcU*Hat_PIMP_0 or FEXP, clcPPE_z1_periodic)
  if (g->BcOption[2] == 0 && (g->order != 2 || g->LES_type != 0 || g->precision != CH3D_PREC_FP64))
    return fail(CH3D_ERR_UNSUPPORTED, "periodic y is built for the 2nd-order step (IsImplicit 0, 1 or 2), FP64, "
                "without LES");
  if (g->LES_type != 0) {
    if (g->LES_type != CH3D_LES_WALE && g->LES_type != CH3D_LES_MTS && g->LES_type != CH3D_LES_SMAG_VD &&
        g->LES_type != CH3D_LES_MLP)
      return fail(CH3D_ERR_UNSUPPORTED, "LES_type=%d not built", g->LES_type);
    if (g->order != 2 || g->IsImplicit == 2)
      return fail(CH3D_ERR_UNSUPPORTED, "LES is built for the 2nd-order partially implicit and explicit steps (the "
                  "reference has no FIMP+LES either)");
    if (g->LES_type == CH3D_LES_MTS && g->FilterType != 0 && g->FilterType != 1)
      return fail(CH3D_ERR_INVALID, "unrecognized FilterType");
  }
  if (g->precision != CH3D_PREC_FP64 && g->precision != CH3D_PREC_MIXED) return fail(CH3D_ERR_INVALID, "bad precision");
  if (g->device < 0 || g->device >= kMaxDevices)
    return fail(CH3D_ERR_INVALID, "device %d out of range (0..%d)", g->device, kMaxDevices - 1);
  if (g->IsUxConst && !(g->ybulk2 > g->ybulk1)) return fail(CH3D_ERR_INVALID, "ybulk1 OR ybulk2 wrong");
  if (!(g->dtMax > 0)) return fail(CH3D_ERR_INVALID, "dtMax must be positive");
  return CH3D_OK;
}

template <class T>
int alloc_fields(ch3d_ctx* c) {
  typedef typename CplxOf<T>::type CT;
  for (int q = 0; q < 15; ++q) {
    if (q == 11 && c->cfg.LES_type == 0) continue;  // nut: LES only
    CU(cudaMalloc(&c->f[q], (size_t)c->N * sizeof(T)));
    CU(cudaMemsetAsync(c->f[q], 0, (size_t)c->N * sizeof(T), c->stream));
    c->bytes += (long long)c->N * sizeof(T);
  }
  if (c->cfg.LES_type > 0) {
    // DeltaCell(jc) = (dyp dx dz)^(1/3) (src/CFD_2nd/m_MeshAndMetries.f90:204) and the
    // wall distance of the cell centres for the van Driest damping
    std::vector<double> h((size_t)2 * (c->ny + 2), 0.0);
    for (int j = 0; j <= c->ny + 1; ++j) h[j] = std::pow(c->dyp[j] * c->dx * c->dz, 1.0 / 3.0);
    for (int j = 1; j <= c->ny; ++j) h[c->ny + 2 + j] = std::min(c->yc[j] - c->yp[1], c->yp[c->ny + 1] - c->yc[j]);
    CU(cudaMalloc(&c->les_delta, h.size() * sizeof(double)));
    CU(cudaMemcpy(c->les_delta, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (c->cfg.LES_type == CH3D_LES_MLP) {
    CU(cudaMalloc(&c->mlp_params, CH3D_MLP_NPARAM * sizeof(float)));
    CU(cudaMalloc(&c->mlp_packed, 32 * 1024));  // the network's parameter image (21.3 KB)
    CU(cudaMalloc(&c->mlp_status, sizeof(int)));
    CU(cudaMemsetAsync(c->mlp_status, 0, sizeof(int), c->stream));
    CU(cudaMalloc(&c->sgs_tau, (size_t)c->N * 6 * sizeof(double)));
    CU(cudaMalloc(&c->sgs_f, (size_t)c->N * 3 * sizeof(double)));
    CU(cudaMemsetAsync(c->sgs_f, 0, (size_t)c->N * 3 * sizeof(double), c->stream));
    CU(launch_fill_nut(c));  // the closure's total viscosity stays xnu
    c->bytes += (long long)c->N * 9 * 8;
  }
  if ((c->cfg.order == 2 && c->cfg.IsImplicit == 2) || y_periodic(c)) {
    const size_t nb = ptri_factor_doubles(c->nx, c->ny, c->nz) * sizeof(double);
    CU(cudaMalloc(&c->pfac, nb));
    CU(cudaMemsetAsync(c->pfac, 0, nb, c->stream));
    c->bytes += (long long)nb;
  }
  if (c->cfg.order == 4)
    for (int q = 0; q < 6; ++q) {
      CU(cudaMalloc(&c->ih[q], (size_t)c->N * sizeof(T)));
      CU(cudaMemsetAsync(c->ih[q], 0, (size_t)c->N * sizeof(T), c->stream));
      c->bytes += (long long)c->N * sizeof(T);
    }
  CU(cudaMalloc(&c->spec, (size_t)c->NS * sizeof(CT)));
  c->bytes += (long long)c->NS * sizeof(CT);
  std::vector<T> met;
  pack_metrics<T>(c, met);
  CU(cudaMalloc(&c->met, met.size() * sizeof(T)));
  CU(cudaMemcpy(c->met, met.data(), met.size() * sizeof(T), cudaMemcpyHostToDevice));
  std::vector<CT> tx = twiddles<CT>(c->nx / 2, c->nx / 2), tr = twiddles<CT>(c->nx, c->nx / 2 + 1),
                  tz = twiddles<CT>(c->nz, c->nz);
  CU(cudaMalloc(&c->twx, tx.size() * sizeof(CT)));
  CU(cudaMalloc(&c->twr, tr.size() * sizeof(CT)));
  CU(cudaMalloc(&c->twz, tz.size() * sizeof(CT)));
  CU(cudaMemcpy(c->twx, tx.data(), tx.size() * sizeof(CT), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(c->twr, tr.data(), tr.size() * sizeof(CT), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(c->twz, tz.data(), tz.size() * sizeof(CT), cudaMemcpyHostToDevice));
  return CH3D_OK;
}

size_t gidx2(const ch3d_ctx* c, int i, int j, int k) {
  // (0:nxc+2, 0:nyc+2, 0:nzc+2)
  return (size_t)i + (size_t)(c->nx + 3) * ((size_t)j + (size_t)(c->ny + 3) * (size_t)k);
}
size_t gidx4(const ch3d_ctx* c, int i, int j, int k) {
  // (-1:nxc+2, 0:nyc+1, -1:nzc+2)
  return (size_t)(i + 1) + (size_t)(c->nx + 4) * ((size_t)j + (size_t)(c->ny + 2) * (size_t)(k + 1));
}

// interior (1-based Fortran i,j,k) value from a host array of the given layout
double host_get(const ch3d_ctx* c, int layout, const double* a, int i, int j, int k) {
  if (layout == CH3D_LAYOUT_INTERIOR) return a[(size_t)(i - 1) + (size_t)c->nx * ((size_t)(j - 1) + (size_t)c->ny * (k - 1))];
  if (layout == CH3D_LAYOUT_GHOST2) return a[gidx2(c, i, j, k)];
  return a[gidx4(c, i, j, k)];
}

// Host-side ghost fill of a downloaded field: the boundary rules and the
// periodic halo copies (myupdate_halo, src/CFD_2nd/m_Decomp2d.f90:1588-1743:
// x planes over the whole y and z extent first, then z planes over the whole
// x and y extent) of SetBC_and_UpdateHalo and SetBC_and_UpdateHalo_pr, with
// each tree's halo widths: 2nd order (src/CFD_2nd/m_BC_and_Halo.f90:20-29,
// 232-344, 410-456) one plane on each side in x and z; 4th order
// (src/CFD_4th/m_BC_and_Halo.f90:24-46, 51-96, 136-150) two on each side for
// the velocity, two below and one above for the pressure.  Cells those routines
// never write (x = nxc+2 and z = nzc+2 of the 2nd-order arrays, the y plane
// nyc+2 of ux, uz, p, uy(:,0,:) of the 4th-order tree) keep the host's values.
// Periodic x and z; y periodic (BcOption(3:4) = 0) copies the halo rows
// j = 0 and nyp first.  comp: 0 ux, 1 uy, 2 uz, 3 p.
void host_fill_ghosts(const ch3d_ctx* c, int layout, double* a, int comp) {
  const int nxc = c->nx, nyc = c->ny, nzc = c->nz, nyp = nyc + 1;
  const ch3d_config& g = c->cfg;
  const bool g2 = layout == CH3D_LAYOUT_GHOST2;
  auto at = [&](int i, int j, int k) -> double& { return g2 ? a[gidx2(c, i, j, k)] : a[gidx4(c, i, j, k)]; };
  for (int k = 1; k <= nzc; ++k)
    for (int i = 1; i <= nxc; ++i) {
      if (y_periodic(c)) {  // y halo rows (one each side, Init_Halo, m_BC_and_Halo.f90:25-29)
        at(i, 0, k) = at(i, nyc, k);
        at(i, nyp, k) = at(i, 1, k);
        continue;
      }
      if (comp == 3) { at(i, nyp, k) = at(i, nyc, k); at(i, 0, k) = at(i, 1, k); continue; }
      if (comp == 1) {
        at(i, nyp, k) = g.uyBcValue[3];
        if (g.order == 2) {
          at(i, nyp + 1, k) = g.uyBcValue[3] * 2.0 - at(i, nyc, k);
          at(i, 0, k) = g.uyBcValue[2] * 2.0 - at(i, 2, k);  // uy_ym = uyBcValue(ym_dir)
        }
        continue;
      }
      const double wl = comp == 0 ? g.uxBcValue[2] : g.uzBcValue[2];
      const double wh = comp == 0 ? g.uxBcValue[3] : g.uzBcValue[3];
      if (g.BcOption[3] == -1) at(i, nyp, k) = wh * 2.0 - at(i, nyc, k);
      else at(i, nyp, k) = wh * c->dyp[nyp] + at(i, nyc, k);
      if (g.BcOption[2] == -1) at(i, 0, k) = wl * 2.0 - at(i, 1, k);
      else at(i, 0, k) = at(i, 1, k) - wl * c->dyp[1];
    }
  // halo widths below / above in x and z, and the allocated bounds
  const int hm = g2 ? 1 : 2, hp = g2 ? 1 : (comp == 3 ? 1 : 2);
  const int xmm = g2 ? 0 : -1, xpm = nxc + 2, ypm = g2 ? nyc + 2 : nyc + 1, zmm = g2 ? 0 : -1, zpm = nzc + 2;
  for (int k = zmm; k <= zpm; ++k)
    for (int j = 0; j <= ypm; ++j) {
      for (int h = 1; h <= hm; ++h) at(1 - h, j, k) = at(nxc - h + 1, j, k);
      for (int h = 1; h <= hp; ++h) at(nxc + h, j, k) = at(h, j, k);
    }
  for (int h = 1; h <= hm; ++h)
    for (int j = 0; j <= ypm; ++j)
      for (int i = xmm; i <= xpm; ++i) at(i, j, 1 - h) = at(i, j, nzc - h + 1);
  for (int h = 1; h <= hp; ++h)
    for (int j = 0; j <= ypm; ++j)
      for (int i = xmm; i <= xpm; ++i) at(i, j, nzc + h) = at(i, j, h);
}

template <class T>
int upload_field(ch3d_ctx* c, int q, int layout, const double* a, int comp) {
  if (sizeof(T) == sizeof(double) && layout == CH3D_LAYOUT_INTERIOR) {
    // FP64 interior arrays are the device layout: one copy (DMA from pinned memory), then the uy wall row
    if (a) CU(cudaMemcpyAsync(c->f[q], a, (size_t)c->N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    else CU(cudaMemsetAsync(c->f[q], 0, (size_t)c->N * sizeof(double), c->stream));
    if (comp == 1 && !y_periodic(c)) CU(launch_fill_row0(c, q, c->cfg.uyBcValue[2]));  // uy(ic,1,kc) = uy_ym
    CU(cudaStreamSynchronize(c->stream));
    return CH3D_OK;
  }
  if (layout == CH3D_LAYOUT_INTERIOR) {
    // FP32 fields from FP64 interior arrays: FP64 chunks through the spectrum
    // buffer (free between steps), converted on the device
    if (!a) {
      CU(cudaMemsetAsync(c->f[q], 0, (size_t)c->N * sizeof(T), c->stream));
    } else {
      const long long cap = (long long)((size_t)c->NS * 2 * sizeof(T) / sizeof(double));
      for (long long off = 0; off < c->N; off += cap) {
        const long long n = c->N - off < cap ? c->N - off : cap;
        CU(cudaMemcpyAsync(c->spec, a + off, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CU(launch_convert(c, c->spec, (T*)c->f[q] + off, n, 1));
      }
    }
    if (comp == 1 && !y_periodic(c)) CU(launch_fill_row0(c, q, c->cfg.uyBcValue[2]));  // uy(ic,1,kc) = uy_ym
    CU(cudaStreamSynchronize(c->stream));
    return CH3D_OK;
  }
  std::vector<T> h((size_t)c->N);
  size_t n = 0;
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i, ++n) {
        double v = a ? host_get(c, layout, a, i, j, k) : 0.0;
        if (comp == 1 && j == 1 && !y_periodic(c)) v = c->cfg.uyBcValue[2];  // uy(ic,1,kc) = uy_ym
        h[n] = (T)v;
      }
  CU(cudaMemcpyAsync(c->f[q], h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return CH3D_OK;
}

template <class T>
int download_field(ch3d_ctx* c, int q, int layout, double* a, int comp) {
  if (sizeof(T) == sizeof(double) && layout == CH3D_LAYOUT_INTERIOR) {
    CU(cudaMemcpyAsync(a, c->f[q], (size_t)c->N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return CH3D_OK;
  }
  if (layout == CH3D_LAYOUT_INTERIOR) {  // FP32 fields: converted on the device, FP64 chunks to the host
    const long long cap = (long long)((size_t)c->NS * 2 * sizeof(T) / sizeof(double));
    for (long long off = 0; off < c->N; off += cap) {
      const long long n = c->N - off < cap ? c->N - off : cap;
      CU(launch_convert(c, (const T*)c->f[q] + off, c->spec, n, 0));
      CU(cudaMemcpyAsync(a + off, c->spec, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    CU(cudaStreamSynchronize(c->stream));
    return CH3D_OK;
  }
  std::vector<T> h((size_t)c->N);
  CU(cudaMemcpyAsync(h.data(), c->f[q], h.size() * sizeof(T), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  size_t n = 0;
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i, ++n) {
        size_t o = layout == CH3D_LAYOUT_INTERIOR ? n : (layout == CH3D_LAYOUT_GHOST2 ? gidx2(c, i, j, k) : gidx4(c, i, j, k));
        a[o] = (double)h[n];
      }
  if (layout != CH3D_LAYOUT_INTERIOR && comp >= 0) host_fill_ghosts(c, layout, a, comp);
  return CH3D_OK;
}

int init_scalars(ch3d_ctx* c) {
  DevScalars s;
  std::memset(&s, 0, sizeof(s));
  s.dt = c->cfg.dtMax;
  CU(cudaMemcpyAsync(c->sc, &s, sizeof(s), cudaMemcpyHostToDevice, c->stream));
  CU(launch_bulk_partials(c));
  CU(launch_diag(c));
  CU(cudaStreamSynchronize(c->stream));
  c->scalars_ready = true;
  return CH3D_OK;
}

// The 2nd-order partially implicit step without LES runs its right-hand
// sides and y solves as one column-march kernel (ch3d_march.cu).
static bool march_path(const ch3d_ctx* c) {
  return c->cfg.LES_type == 0 && c->cfg.order == 2 && c->cfg.IsImplicit == 1 && !y_periodic(c);
}

int record_step(ch3d_ctx* c) {
  CU(launch_step_begin(c));
  if (c->cfg.LES_type > 0) CU(launch_sgs_nut(c));  // once per step, after the CFL (m_ChannelSystem.f90:89)
  const bool o4 = c->cfg.order == 4, fimp = c->cfg.order == 2 && c->cfg.IsImplicit == 2;
  for (int ns = 1; ns <= c->iadvance; ++ns) {
    if (o4) CU(launch_visc4_partials(c));
    CU(launch_substep_setup(c, ns));
    if (march_path(c)) {  // RHS + y solves as one column march, its own Thomas factors
      CU(launch_rhs_march(c));
    } else if (c->cfg.LES_type > 0) {  // the LES y solves form their own coefficients (FEXP: none)
      CU(launch_rhs_les(c));
      CU(c->cfg.IsImplicit == 0 ? launch_uhat_fexp(c) : launch_uhat_les(c));
    } else if (fimp) {
      if (!y_periodic(c)) CU(launch_helm_factors(c));
      CU(launch_rhs_fimp(c));
      CU(launch_ptri_xz(c));
      CU(y_periodic(c) ? launch_ptri_y(c) : launch_uhat(c));  // FIMP_000 or FIMP_010
    } else if (c->cfg.IsImplicit == 0) {  // FEXP: explicit right-hand sides, u* = u + Rhs
      CU(launch_rhs_fimp(c));
      CU(launch_uhat_fexp(c));
    } else if (y_periodic(c)) {  // PIMP_0: the periodic y sweep alone
      CU(launch_rhs(c));
      CU(launch_ptri_y(c));
    } else {
      CU(launch_rhs_march(c));  // 4th order: the same column march with the 4th-order stencils
    }
    if (c->gsub) {
      CU(launch_div_bsub(c));
      CU(launch_prsrc_xfft(c, 3));
    } else {
      CU(launch_prsrc_xfft(c, 0));
    }
    CU(launch_poisson_spectral(c));
    CU(launch_xifft(c));
    if (ns == c->iadvance && march_diag_fusable(c)) {  // CheckDivergence etc. ride on the last projection
      CU(launch_diag_reset(c));
      CU(c->gsub ? launch_proj_bsub(c, true) : launch_proj_diag(c));
    } else {
      CU(c->gsub ? launch_proj_bsub(c, false) : launch_proj(c, 0));
    }
  }
  if (!march_diag_fusable(c)) CU(launch_diag(c));
  CU(launch_step_end(c));
  return CH3D_OK;
}

int build_graph(ch3d_ctx* c) {
  if (c->graph_exec) return CH3D_OK;
  // the first launch of each kernel sets its shared-memory attribute outside capture
  CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = record_step(c);
  cudaGraph_t gph = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->stream, &gph);
  if (rc != CH3D_OK) { if (gph) cudaGraphDestroy(gph); return rc; }
  if (e != cudaSuccess) return fail(CH3D_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  c->graph = gph;
  CU(cudaGraphInstantiate(&c->graph_exec, c->graph, 0));
  return CH3D_OK;
}

int fetch_info(ch3d_ctx* c, ch3d_step_info* info) {
  DevScalars s;
  CU(cudaMemcpyAsync(&s, c->sc, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  if (info) {
    info->SimTime = s.SimTime; info->dt = s.dt; info->cflmp = s.cflmp;
    info->divmax1 = __builtin_bit_cast(double, s.divmax1);
    info->divmax2 = __builtin_bit_cast(double, s.divmax2);
    for (int q = 0; q < 3; ++q) info->vmax[q] = __builtin_bit_cast(double, s.vmax[q]);
    info->uxm = s.uxm; info->PrGradAver = s.PrGradAver; info->itime = s.itime; info->status = s.status;
  }
  return s.status ? CH3D_ERR_DIVERGED : CH3D_OK;
}

}  // namespace

extern "C" {

const char* ch3d_version(void) { return "ch3d-b200 0.1 (sm_100a)"; }

const char* ch3d_last_error(void) { return g_err.c_str(); }

int ch3d_mesh_section(double* yp, int id1, int id2, double c1, double c2, int StretType, double cStret, int StretOption) {
  if (!yp || id2 <= id1 || id1 < 1) return fail(CH3D_ERR_INVALID, "bad mesh section");
  if (StretType < 0 || StretType > 3) return fail(CH3D_ERR_INVALID, "StretType Wrong !!!");
  mesh_section(yp, id1, id2, c1, c2, StretType, cStret, StretOption);
  return CH3D_OK;
}

// src/CFD_2nd/m_MeshAndMetries.f90:122-160
int ch3d_mesh_y(int nyc, double yly, int nSection, const double* SectionLength, const int* nycSection,
                const int* StretType, const int* StretOption, const double* SectioncStret, double* yp) {
  if (nSection < 1 || !yp) return fail(CH3D_ERR_INVALID, "nSection Wrong !!!");
  int tot = 0;
  for (int j = 0; j < nSection; ++j) {
    if (SectionLength[j] < 0) return fail(CH3D_ERR_INVALID, "SectionLength Wrong !!!");
    if (SectioncStret[j] < 0) return fail(CH3D_ERR_INVALID, "SectioncStret Wrong !!!");
    if (nycSection[j] < 1) return fail(CH3D_ERR_INVALID, "nycSection Wrong 1 !!!");
    if (StretType[j] < 0 || StretType[j] > 3) return fail(CH3D_ERR_INVALID, "StretType Wrong !!!");
    if (StretOption[j] < 0 || StretOption[j] > 1) return fail(CH3D_ERR_INVALID, "StretOption Wrong !!!");
    tot += nycSection[j];
  }
  if (tot != nyc) return fail(CH3D_ERR_INVALID, "nycSection Wrong 2 !!!");
  std::vector<int> nid(nSection + 1, 1);
  std::vector<double> ysc(nSection + 1, 0.0);
  double SumLength = 0;
  for (int j = 0; j < nSection; ++j) SumLength += SectionLength[j];
  for (int j = 0; j < nSection; ++j) {
    nid[j + 1] = nid[j] + nycSection[j];
    ysc[j + 1] = ysc[j] + SectionLength[j] / SumLength * yly;
  }
  ysc[nSection] = yly;
  for (int j = 0; j < nSection; ++j)
    mesh_section(yp, nid[j], nid[j + 1], ysc[j], ysc[j + 1], StretType[j], SectioncStret[j], StretOption[j]);
  return CH3D_OK;
}

int ch3d_create(const ch3d_config* cfg, const double* yp, ch3d_ctx** out) {
  if (!out) return fail(CH3D_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int rc = check_config(cfg);
  if (rc) return rc;
  if (!yp) return fail(CH3D_ERR_INVALID, "yp is NULL");
  for (int j = 1; j <= cfg->nyc; ++j)
    if (!(yp[j] > yp[j - 1])) return fail(CH3D_ERR_INVALID, "yp must increase (yp(%d) <= yp(%d))", j + 1, j);
  ch3d_ctx* c = new ch3d_ctx();
  c->cfg = *cfg;
  c->nx = cfg->nxc; c->ny = cfg->nyc; c->nz = cfg->nzc; c->nxh = cfg->nxc / 2 + 1;
  c->N = (long long)c->nx * c->ny * c->nz;
  c->NS = (long long)c->nxh * c->ny * c->nz;
  c->fp32 = cfg->precision == CH3D_PREC_MIXED;
  c->device = cfg->device;
  if (!factor23(c->nx / 2, c->planx) || !factor23(c->nz, c->planz)) {
    delete c;
    return fail(CH3D_ERR_UNSUPPORTED, "nxc/2 and nzc must be products of 2 and 3 (got %d, %d)", cfg->nxc / 2, cfg->nzc);
  }
  // time-scheme constants (src/CFD_2nd/m_Parameters.f90:135-150; the same in
  // src/CFD_4th/m_Parameters.f90:158-173): AB2 one substep, RK2 two, RK3 three
  if (cfg->ischeme == 1) {
    c->iadvance = 1;
    c->gam[0] = 1.5; c->the[0] = -0.5;
  } else if (cfg->ischeme == 2) {
    c->iadvance = 2;
    c->gam[0] = 0.5; c->gam[1] = 1.0;
    c->the[0] = 0.0; c->the[1] = -0.5;
  } else {
    c->iadvance = 3;
    c->gam[0] = 8.0 / 15.0; c->gam[1] = 5.0 / 12.0; c->gam[2] = 3.0 / 4.0;
    c->the[0] = 0.0; c->the[1] = -17.0 / 60.0; c->the[2] = -5.0 / 12.0;
  }
  for (int s = 0; s < 3; ++s) c->alp[s] = c->gam[s] + c->the[s];
  c->yp.assign(c->ny + 3, 0.0);
  for (int j = 1; j <= c->ny + 1; ++j) c->yp[j] = yp[j - 1];
  build_metrics(c);
  auto cleanup = [&](int code) { ch3d_destroy(c); return code; };
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) { int r = fail(CH3D_ERR_CUDA, "cudaSetDevice(%d): %s", c->device, cudaGetErrorString(e)); delete c; return r; }
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { int r = fail(CH3D_ERR_CUDA, "stream: %s", cudaGetErrorString(e)); delete c; return r; }
  if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess)
    return cleanup(fail(CH3D_ERR_CUDA, "event create failed"));
  if (c->fp32) {
    int lo = 0, hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess)
      return cleanup(fail(CH3D_ERR_CUDA, "side stream create failed"));
  }
  rc = c->fp32 ? alloc_fields<float>(c) : alloc_fields<double>(c);
  if (rc) return cleanup(rc);
  {
    std::vector<double> met;
    pack_metrics<double>(c, met);
    if (cudaMalloc(&c->met64, met.size() * sizeof(double)) != cudaSuccess) return cleanup(fail(CH3D_ERR_NOMEM, "metrics"));
    cudaMemcpy(c->met64, met.data(), met.size() * sizeof(double), cudaMemcpyHostToDevice);
    std::vector<double> w(c->nx + c->nz);
    for (int i = 0; i < c->nx; ++i) w[i] = c->WaveNumX[i];
    for (int k = 0; k < c->nz; ++k) w[c->nx + k] = c->WaveNumZ[k];
    if (cudaMalloc(&c->wave, w.size() * sizeof(double)) != cudaSuccess) return cleanup(fail(CH3D_ERR_NOMEM, "wave"));
    cudaMemcpy(c->wave, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice);
  }
  c->m64 = metrics_ptrs<double>(c->met64, c->ny);
  c->m64full = c->m64;
  if (c->fp32) c->m32 = metrics_ptrs<float>((const float*)c->met, c->ny);
  else c->m32 = Metrics<float>();
  if (!c->fp32) c->m64 = metrics_ptrs<double>((const double*)c->met, c->ny);
  c->TSy = 8;  // kx extent of the FP64 low modes of the mixed path
  // chunks of the partitioned Helmholtz solves: the power of two nearest below
  // sqrt(ny) (2..32), balancing the chunk sweeps (2 ny / P rows) against the
  // serial interface solve (P - 1 steps)
  c->Pv = 2;
  while (c->Pv < 32 && 4 * c->Pv * c->Pv <= c->ny) c->Pv <<= 1;
  while (c->Pv > 1 && c->ny < 2 * c->Pv) c->Pv >>= 1;
  {
    size_t nf = (size_t)2 * (5 * c->ny + 6 * (c->Pv > 1 ? c->Pv - 1 : 1));
    if (cudaMalloc(&c->hfac, nf * sizeof(double)) != cudaSuccess) return cleanup(fail(CH3D_ERR_NOMEM, "hfac"));
    if (cudaMalloc(&c->mtab, march_table_bytes(c->ny)) != cudaSuccess)
      return cleanup(fail(CH3D_ERR_NOMEM, "march table"));
    if (march_table_reset(c) != cudaSuccess) return cleanup(fail(CH3D_ERR_CUDA, "march table"));
  }
  {
    // mixed path: low modes kept in FP64: kx < TSy, |kz| <= KL (KL < nz/2 so the two kz ranges are disjoint)
    c->KL = 8;
    if (c->KL > c->nz / 2 - 1) c->KL = c->nz / 2 - 1;
    if (c->KL < 0) c->KL = 0;
    // Poisson y-solve (Thomas) factors per (kx, |kz|), computed once
    const size_t nrow = (size_t)(c->nz / 2 + 1) * c->ny * c->nxh;
    const size_t fw = c->fp32 ? sizeof(float) : sizeof(double);
    if (cudaMalloc(&c->yRM, nrow * fw) != cudaSuccess || cudaMalloc(&c->yCP, nrow * fw) != cudaSuccess)
      return cleanup(fail(CH3D_ERR_NOMEM, "Poisson factors"));
    c->bytes += (long long)(2 * nrow) * fw;
    if (c->fp32) {
      const size_t lr = (size_t)(c->KL + 1) * c->ny * c->TSy;
      const size_t ls = (size_t)(2 * c->KL + 1) * c->TSy * c->ny * 2;  // FP64 complex sweep scratch
      if (cudaMalloc(&c->yRM64, lr * sizeof(double)) != cudaSuccess ||
          cudaMalloc(&c->yCP64, lr * sizeof(double)) != cudaSuccess ||
          cudaMalloc(&c->ylow, ls * sizeof(double)) != cudaSuccess)
        return cleanup(fail(CH3D_ERR_NOMEM, "Poisson low-mode factors"));
    }
    if (y_periodic(c)) {
      if (cudaMalloc(&c->yA2, nrow * sizeof(double)) != cudaSuccess)
        return cleanup(fail(CH3D_ERR_NOMEM, "Poisson factors"));
      c->bytes += (long long)nrow * sizeof(double);
    }
    e = launch_ysolve_factors(c);
    if (e != cudaSuccess) return cleanup(fail(CH3D_ERR_CUDA, "Poisson factors: %s", cudaGetErrorString(e)));
  }
  {
    dim3 g((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz);
    c->npart = (int)(g.x * g.y * g.z);
    c->march = march_path(c);
    // large 2nd-order grids: the march stops at g, the divergence and projection substitute
    c->gsub = c->march && !march_twisted(c) && xplan_exists(c->nx / 2);
    c->npart_m = march_npart(c);
    if (c->npart_m > c->npart) c->npart = c->npart_m;
    if (diag_npart(c) > c->npart) c->npart = diag_npart(c);
    if (visc4_npart(c) > c->npart) c->npart = visc4_npart(c);
    if (cudaMalloc(&c->part, (size_t)c->npart * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->part2, (size_t)c->npart * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->red1, CH3D_NRED * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->red2, CH3D_NRED * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->sc, sizeof(DevScalars)) != cudaSuccess)
      return cleanup(fail(CH3D_ERR_NOMEM, "partials"));
    // SumStat(35, nyp) | PrGradsum [| SumGrad(98, nyp) of the 4th-order statistics]
    const size_t nstat = (size_t)35 * (c->ny + 1) + 1 + (cfg->order == 4 ? (size_t)98 * (c->ny + 1) : 0);
    const int kch = (c->nz + 7) / 8, nch = (c->nz + kch - 1) / kch;
    if (cudaMalloc(&c->stat, nstat * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->statpart, (size_t)35 * (c->ny + 1) * nch * sizeof(double)) != cudaSuccess)
      return cleanup(fail(CH3D_ERR_NOMEM, "statistics"));
    cudaMemsetAsync(c->stat, 0, nstat * sizeof(double), c->stream);
    cudaMemsetAsync(c->part, 0, (size_t)c->npart * sizeof(double), c->stream);
    cudaMemsetAsync(c->part2, 0, (size_t)c->npart * sizeof(double), c->stream);
    cudaMemsetAsync(c->sc, 0, sizeof(DevScalars), c->stream);
    c->bytes += 2LL * c->npart * sizeof(double);
  }
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cleanup(fail(CH3D_ERR_CUDA, "create: %s", cudaGetErrorString(e)));
  *out = c;
  return CH3D_OK;
}

int ch3d_destroy(ch3d_ctx* c) {
  if (!c) return CH3D_OK;
  cudaSetDevice(c->device);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  for (int q = 0; q < 15; ++q) if (c->f[q]) cudaFree(c->f[q]);
  for (int q = 0; q < 6; ++q) if (c->ih[q]) cudaFree(c->ih[q]);
  if (c->pfac) cudaFree(c->pfac);
  if (c->les_delta) cudaFree(c->les_delta);
  void* mbufs[] = {c->mlp_params, c->mlp_packed, c->mlp_status, c->sgs_tau, c->sgs_f, c->spec2,
                   c->specacc};
  for (void* b : mbufs) if (b) cudaFree(b);
  void* bufs[] = {c->hfac, c->mtab, c->yRM, c->yCP, c->ylow, c->yA2, c->yRM64, c->yCP64, c->spec, c->met, c->met64, c->wave, c->twx, c->twr, c->twz, c->sc, c->part, c->part2,
                  c->red1, c->red2, c->stat, c->statpart};
  for (void* b : bufs) if (b) cudaFree(b);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return CH3D_OK;
}

int ch3d_upload_state(ch3d_ctx* c, int layout, const double* ux, const double* uy, const double* uz, const double* p,
                      const double* hist) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  if (layout < 0 || layout > 2) return fail(CH3D_ERR_INVALID, "bad layout %d", layout);
  if (!ux || !uy || !uz || !p) return fail(CH3D_ERR_INVALID, "state arrays must not be NULL");
  CU(cudaSetDevice(c->device));
  int rc;
  const double* arrs[4] = {ux, uy, uz, p};
  for (int q = 0; q < 4; ++q) {
    rc = c->fp32 ? upload_field<float>(c, q, layout, arrs[q], q) : upload_field<double>(c, q, layout, arrs[q], q);
    if (rc) return rc;
  }
  for (int q = 0; q < 3; ++q) {
    const double* h = hist ? hist + (size_t)q * c->N : nullptr;
    rc = c->fp32 ? upload_field<float>(c, 4 + q, CH3D_LAYOUT_INTERIOR, h, -1)
                 : upload_field<double>(c, 4 + q, CH3D_LAYOUT_INTERIOR, h, -1);
    if (rc) return rc;
  }
  return init_scalars(c);
}

int ch3d_download_state(ch3d_ctx* c, int layout, double* ux, double* uy, double* uz, double* p, double* hist) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  if (layout < 0 || layout > 2) return fail(CH3D_ERR_INVALID, "bad layout %d", layout);
  CU(cudaSetDevice(c->device));
  double* arrs[4] = {ux, uy, uz, p};
  for (int q = 0; q < 4; ++q) {
    if (!arrs[q]) continue;
    int rc = c->fp32 ? download_field<float>(c, q, layout, arrs[q], q) : download_field<double>(c, q, layout, arrs[q], q);
    if (rc) return rc;
  }
  if (hist)
    for (int q = 0; q < 3; ++q) {
      int rc = c->fp32 ? download_field<float>(c, 4 + q, CH3D_LAYOUT_INTERIOR, hist + (size_t)q * c->N, -1)
                       : download_field<double>(c, 4 + q, CH3D_LAYOUT_INTERIOR, hist + (size_t)q * c->N, -1);
      if (rc) return rc;
    }
  return CH3D_OK;
}

static int mlp_check(ch3d_ctx* c) {
  if (c->cfg.LES_type != CH3D_LES_MLP) return CH3D_OK;
  if (!c->mlp_ready) return fail(CH3D_ERR_INVALID, "learned closure: call ch3d_sgs_mlp_set before stepping");
  int st = 0;
  CU(cudaMemcpy(&st, c->mlp_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) return fail(CH3D_ERR_CUDA, "learned closure: tensor-core kernel timed out waiting for its MMAs");
  return CH3D_OK;
}

int ch3d_step(ch3d_ctx* c, int nsteps, ch3d_step_info* info) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  if (nsteps < 0) return fail(CH3D_ERR_INVALID, "nsteps < 0");
  if (int rc = mlp_check(c)) return rc;
  CU(cudaSetDevice(c->device));
  if (!c->scalars_ready) {
    int rc = init_scalars(c);
    if (rc) return rc;
  }
  if (!c->graph_exec) {
    // run one uncaptured step first so that kernel attributes are set outside capture
    CU(cudaEventRecord(c->ev0, c->stream));
    int rc = record_step(c);
    if (rc) return rc;
    CU(cudaEventRecord(c->ev1, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    rc = build_graph(c);
    if (rc) return rc;
    nsteps -= 1;
    if (nsteps <= 0) {
      float ms = 0;
      cudaEventElapsedTime(&ms, c->ev0, c->ev1);
      c->last_ms = ms;
      return fetch_info(c, info);
    }
  }
  CU(cudaEventRecord(c->ev0, c->stream));
  for (int s = 0; s < nsteps; ++s) CU(cudaGraphLaunch(c->graph_exec, c->stream));
  CU(cudaEventRecord(c->ev1, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  float ms = 0;
  CU(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  if (int rc = mlp_check(c)) return rc;
  return fetch_info(c, info);
}

int ch3d_stage(ch3d_ctx* c, int stage, int ns) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  if (int rc = mlp_check(c)) return rc;
  if (ns < 1 || ns > c->iadvance) return fail(CH3D_ERR_INVALID, "ns out of range");
  CU(cudaSetDevice(c->device));
  if (!c->scalars_ready) {
    int rc = init_scalars(c);
    if (rc) return rc;
  }
  switch (stage) {
    case 0:
      if (c->cfg.order == 4) CU(launch_visc4_partials(c));  // forcing of clcRhsXYZ from the current ux
      CU(launch_substep_setup(c, ns));
      break;
    case 1:
      if (c->cfg.LES_type > 0) CU(launch_rhs_les(c));
      else CU(c->cfg.order == 4 ? launch_rhs4(c) : (c->cfg.IsImplicit != 1 ? launch_rhs_fimp(c) : launch_rhs(c)));
      break;
    case 2:
      if (c->cfg.IsImplicit == 0) { CU(launch_uhat_fexp(c)); break; }
      if (c->cfg.LES_type > 0) { CU(launch_uhat_les(c)); break; }
      if (c->cfg.order == 2 && c->cfg.IsImplicit == 2) CU(launch_ptri_xz(c));
      if (y_periodic(c)) { CU(launch_ptri_y(c)); break; }
      CU(launch_helm_factors(c));
      CU(launch_uhat(c));
      break;
    case 3: break;  // clcPrSrc is fused into the forward x transform of stage 4
    case 4:
      CU(launch_prsrc_xfft(c, 0));
      CU(launch_poisson_spectral(c));
      CU(launch_xifft(c));
      break;
    case 5: CU(launch_proj(c, 0)); break;  // FluidVelUpdate fused with PressureUpdate
    case 6: break;
    default: return fail(CH3D_ERR_INVALID, "bad stage %d", stage);
  }
  CU(cudaStreamSynchronize(c->stream));
  return CH3D_OK;
}

static int array_slot(int which) {
  // 0 ux, 1 uy, 2 uz, 3 p, 4..6 Hist, 7 RhsX, 8 RhsY, 9 RhsZ / prphi, 10 nut
  switch (which) {
    case 0: case 1: case 2: case 3: case 4: case 5: case 6: case 7: case 8: return which;
    case 9: return 10;   // prphi (the reference keeps RhsZ and prphiHalo in RealHalo)
    case 10: return 11;  // nut (LES), total viscosity
    case 11: return 9;   // RhsZ
    case 12: case 13: case 14: return which;  // u* (velocity after the Helmholtz solves)
    default: return -1;
  }
}

int ch3d_get_array(ch3d_ctx* c, int which, double* host) {
  if (!c || !host) return fail(CH3D_ERR_INVALID, "NULL argument");
  if (which >= 15 && which <= 20) {  // learned closure: SGS stress components at the cell centres
    if (!c->sgs_tau) return fail(CH3D_ERR_INVALID, "array %d exists for LES_type CH3D_LES_MLP only", which);
    CU(cudaSetDevice(c->device));
    CU(cudaMemcpy(host, c->sgs_tau + (size_t)(which - 15) * c->N, (size_t)c->N * sizeof(double),
                  cudaMemcpyDeviceToHost));
    return CH3D_OK;
  }
  int q = array_slot(which);
  if (q < 0) return fail(CH3D_ERR_INVALID, "bad array id %d", which);
  CU(cudaSetDevice(c->device));
  return c->fp32 ? download_field<float>(c, q, CH3D_LAYOUT_INTERIOR, host, -1)
                 : download_field<double>(c, q, CH3D_LAYOUT_INTERIOR, host, -1);
}

int ch3d_set_array(ch3d_ctx* c, int which, const double* host) {
  if (!c || !host) return fail(CH3D_ERR_INVALID, "NULL argument");
  int q = array_slot(which);
  if (q < 0) return fail(CH3D_ERR_INVALID, "bad array id %d", which);
  CU(cudaSetDevice(c->device));
  int rc = c->fp32 ? upload_field<float>(c, q, CH3D_LAYOUT_INTERIOR, host, q == 1 ? 1 : -1)
                   : upload_field<double>(c, q, CH3D_LAYOUT_INTERIOR, host, q == 1 ? 1 : -1);
  if (rc) return rc;
  c->scalars_ready = false;
  return CH3D_OK;
}

int ch3d_poisson(ch3d_ctx* c, const double* src, double* phi) {
  if (!c || !src || !phi) return fail(CH3D_ERR_INVALID, "NULL argument");
  CU(cudaSetDevice(c->device));
  if (!c->scalars_ready) { int rc = init_scalars(c); if (rc) return rc; }
  // src goes through slot 10 (phi) and mode 2 of the x transform
  int rc = c->fp32 ? upload_field<float>(c, 10, CH3D_LAYOUT_INTERIOR, src, -1)
                   : upload_field<double>(c, 10, CH3D_LAYOUT_INTERIOR, src, -1);
  if (rc) return rc;
  CU(launch_prsrc_xfft(c, 2));
  CU(launch_poisson_spectral(c));
  CU(launch_xifft(c));
  return c->fp32 ? download_field<float>(c, 10, CH3D_LAYOUT_INTERIOR, phi, -1)
                 : download_field<double>(c, 10, CH3D_LAYOUT_INTERIOR, phi, -1);
}

int ch3d_project(ch3d_ctx* c, double* divmax_before, double* divmax_after) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  CU(cudaSetDevice(c->device));
  if (!c->scalars_ready) { int rc = init_scalars(c); if (rc) return rc; }
  unsigned long long* slots = nullptr;
  CU(cudaMalloc(&slots, 2 * sizeof(unsigned long long)));
  CU(cudaMemsetAsync(slots, 0, 2 * sizeof(unsigned long long), c->stream));
  CU(launch_divmax(c, slots));
  CU(launch_prsrc_xfft(c, 1));
  CU(launch_poisson_spectral(c));
  CU(launch_xifft(c));
  CU(launch_proj(c, 1));
  CU(launch_divmax(c, slots + 1));
  unsigned long long h[2];
  CU(cudaMemcpyAsync(h, slots, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  cudaFree(slots);
  if (divmax_before) *divmax_before = __builtin_bit_cast(double, h[0]);
  if (divmax_after) *divmax_after = __builtin_bit_cast(double, h[1]);
  c->scalars_ready = false;
  return CH3D_OK;
}

int ch3d_set_dt(ch3d_ctx* c, double dt) {
  if (!c || !(dt > 0)) return fail(CH3D_ERR_INVALID, "bad dt");
  c->cfg.dtMax = dt;
  if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
  if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
  CU(cudaMemcpyAsync(&c->sc->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return CH3D_OK;
}

static size_t stat_doubles(const ch3d_ctx* c) {
  return (size_t)35 * (c->ny + 1) + 1 + (c->cfg.order == 4 ? (size_t)98 * (c->ny + 1) : 0);
}

int ch3d_stats_accumulate(ch3d_ctx* c) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  CU(cudaSetDevice(c->device));
  if (!c->scalars_ready) { int rc = init_scalars(c); if (rc) return rc; }
  CU(c->cfg.order == 4 ? launch_stats4(c) : launch_stats(c));
  CU(cudaStreamSynchronize(c->stream));
  c->nfstime += 1;
  return CH3D_OK;
}

int ch3d_stats_fetch(ch3d_ctx* c, double* sumstat, int* nfstime, double* prgradsum, int reset) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  CU(cudaSetDevice(c->device));
  const size_t n = (size_t)35 * (c->ny + 1);
  std::vector<double> h(n + 1);
  CU(cudaMemcpyAsync(h.data(), c->stat, (n + 1) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  if (sumstat) std::memcpy(sumstat, h.data(), n * sizeof(double));
  if (prgradsum) *prgradsum = h[n];
  if (nfstime) *nfstime = c->nfstime;
  if (reset) {
    CU(cudaMemsetAsync(c->stat, 0, stat_doubles(c) * sizeof(double), c->stream));
    CU(cudaStreamSynchronize(c->stream));
    c->nfstime = 0;
  }
  return CH3D_OK;
}

// EnergySpecX (nxh, ny, 18) | EnergySpecZ (nz/2+1, ny, 18) | EnergySpec2D (nxh, ny/2, nz/2+1, 9)
static size_t spectra_doubles(const ch3d_ctx* c) {
  return (size_t)18 * c->ny * (c->nxh + c->nz / 2 + 1) + (size_t)9 * c->nxh * (c->ny / 2) * (c->nz / 2 + 1);
}

int ch3d_spectra_accumulate(ch3d_ctx* c, int jfor1, int jfor2) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  if (c->cfg.order != 4)
    return fail(CH3D_ERR_UNSUPPORTED, "the spectra belong to the 4th-order statistics");
  if (jfor1 < 1 || jfor1 > c->ny / 2 || jfor2 < 1 || jfor2 > c->ny / 2)
    return fail(CH3D_ERR_INVALID, "jForLCS (%d, %d) must lie in 1..nyc/2", jfor1, jfor2);
  CU(cudaSetDevice(c->device));
  if (!c->specacc) {
    const size_t word = c->fp32 ? sizeof(float) : sizeof(double);
    if (cudaMalloc(&c->spec2, (size_t)c->NS * 2 * word) != cudaSuccess ||
        cudaMalloc(&c->specacc, spectra_doubles(c) * sizeof(double)) != cudaSuccess)
      return fail(CH3D_ERR_NOMEM, "spectra buffers");
    c->bytes += (long long)c->NS * 2 * word + (long long)spectra_doubles(c) * sizeof(double);
    CU(cudaMemsetAsync(c->specacc, 0, spectra_doubles(c) * sizeof(double), c->stream));
  }
  CU(launch_spectra(c, jfor1, jfor2));
  CU(cudaStreamSynchronize(c->stream));
  c->nspectime += 1;
  return CH3D_OK;
}

int ch3d_spectra_fetch(ch3d_ctx* c, double* specx, double* specz, double* spec2d, int* nspectime, int reset) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  if (c->cfg.order != 4)
    return fail(CH3D_ERR_UNSUPPORTED, "the spectra belong to the 4th-order statistics");
  CU(cudaSetDevice(c->device));
  const size_t nxs = (size_t)18 * c->ny * c->nxh, nzs = (size_t)18 * c->ny * (c->nz / 2 + 1);
  const size_t n2s = (size_t)9 * c->nxh * (c->ny / 2) * (c->nz / 2 + 1);
  if (!c->specacc) {
    if (specx) std::memset(specx, 0, nxs * sizeof(double));
    if (specz) std::memset(specz, 0, nzs * sizeof(double));
    if (spec2d) std::memset(spec2d, 0, n2s * sizeof(double));
  } else {
    if (specx) CU(cudaMemcpyAsync(specx, c->specacc, nxs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (specz) CU(cudaMemcpyAsync(specz, c->specacc + nxs, nzs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (spec2d)
      CU(cudaMemcpyAsync(spec2d, c->specacc + nxs + nzs, n2s * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (reset) CU(cudaMemsetAsync(c->specacc, 0, spectra_doubles(c) * sizeof(double), c->stream));
    CU(cudaStreamSynchronize(c->stream));
  }
  if (nspectime) *nspectime = c->nspectime;
  if (reset) c->nspectime = 0;
  return CH3D_OK;
}

int ch3d_stats_fetch_grad(ch3d_ctx* c, double* sumgrad) {
  if (!c || !sumgrad) return fail(CH3D_ERR_INVALID, "NULL argument");
  if (c->cfg.order != 4)
    return fail(CH3D_ERR_UNSUPPORTED, "the gradient moments belong to the 4th-order statistics");
  CU(cudaSetDevice(c->device));
  const size_t off = (size_t)35 * (c->ny + 1) + 1, n = (size_t)98 * (c->ny + 1);
  CU(cudaMemcpyAsync(sumgrad, c->stat + off, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return CH3D_OK;
}

int ch3d_dissipation(ch3d_ctx* c, double* eps) {
  if (!c || !eps) return fail(CH3D_ERR_INVALID, "NULL argument");
  if (c->cfg.order != 2) return fail(CH3D_ERR_UNSUPPORTED, "clcStat_TG belongs to the 2nd-order solver");
  CU(cudaSetDevice(c->device));
  int np = 0;
  CU(launch_dissipation(c, &np));
  CU(launch_reduce_partials(c, c->part2, np, c->red2));
  std::vector<double> r(CH3D_NRED);
  CU(cudaMemcpyAsync(r.data(), c->red2, CH3D_NRED * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  double s = 0.0;
  for (double v : r) s += v;
  *eps = c->cfg.xnu * s / ((double)c->nx * (double)c->ny * (double)c->nz);
  return CH3D_OK;
}

int ch3d_sgs_mlp_set(ch3d_ctx* c, const float* params, const float* norm) {
  if (!c || !params || !norm) return fail(CH3D_ERR_INVALID, "NULL argument");
  if (c->cfg.LES_type != CH3D_LES_MLP) return fail(CH3D_ERR_INVALID, "LES_type is not CH3D_LES_MLP");
  for (int q = 0; q < 10; ++q)
    if (!(norm[10 + q] > 0)) return fail(CH3D_ERR_INVALID, "input standard deviation %d not positive", q);
  for (int q = 0; q < 6; ++q)
    if (!(norm[46 + q] > 0)) return fail(CH3D_ERR_INVALID, "output standard deviation %d not positive", q);
  CU(cudaSetDevice(c->device));
  CU(cudaMemcpy(c->mlp_params, params, CH3D_MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  CU(launch_mlp_pack(c));
  CU(cudaStreamSynchronize(c->stream));
  std::memcpy(c->mlp_norm, norm, sizeof(c->mlp_norm));
  c->mlp_ready = true;
  if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }  // the norm is a kernel argument
  if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
  return CH3D_OK;
}

int ch3d_sgs_training_samples(ch3d_ctx* c, int fx, int fy, int fz, float* X, float* T, long long* nbox) {
  if (!c || !X || !T || !nbox) return fail(CH3D_ERR_INVALID, "NULL argument");
  if (c->fp32) return fail(CH3D_ERR_UNSUPPORTED, "training samples are taken from an FP64 field");
  if (fx < 1 || fy < 1 || fz < 1 || c->nx % fx || c->ny % fy || c->nz % fz)
    return fail(CH3D_ERR_INVALID, "box %d x %d x %d does not tile the grid", fx, fy, fz);
  CU(cudaSetDevice(c->device));
  if (!c->scalars_ready) { int rc = init_scalars(c); if (rc) return rc; }
  CU(launch_sgs_samples(c, fx, fy, fz, X, T));
  CU(cudaStreamSynchronize(c->stream));
  *nbox = (long long)(c->nx / fx) * (c->ny / fy) * (c->nz / fz);
  return CH3D_OK;
}

int ch3d_sgs_viscosity(ch3d_ctx* c) {
  if (!c) return fail(CH3D_ERR_INVALID, "ctx is NULL");
  if (c->cfg.LES_type == 0) return fail(CH3D_ERR_INVALID, "LES_type is 0");
  if (int rc = mlp_check(c)) return rc;
  CU(cudaSetDevice(c->device));
  if (!c->scalars_ready) { int rc = init_scalars(c); if (rc) return rc; }
  CU(launch_sgs_nut(c));
  CU(cudaStreamSynchronize(c->stream));
  return CH3D_OK;
}

int ch3d_memory_bytes(ch3d_ctx* c, long long* bytes) {
  if (!c || !bytes) return fail(CH3D_ERR_INVALID, "NULL argument");
  *bytes = c->bytes;
  return CH3D_OK;
}

// Runs `nsteps` steps kernel group by kernel group with CUDA events between
// the groups on the context's stream; out[q] = mean milliseconds per launch of
// group q: 0 rhs, 1 uhat, 2 prsrc+x FFT, 3 z FFT + y solve + z iFFT,
// 4 x iFFT, 5 projection, 6 scalar/reduction kernels.
int ch3d_kernel_times(ch3d_ctx* c, int nsteps, double* out, int nout) {
  if (!c || !out || nout < 7 || nsteps < 1) return fail(CH3D_ERR_INVALID, "bad argument");
  CU(cudaSetDevice(c->device));
  if (!c->scalars_ready) { int rc = init_scalars(c); if (rc) return rc; }
  const int G = 7;
  const int per_step = 1 + 7 * c->iadvance + 1;  // timed groups per step
  std::vector<cudaEvent_t> ev((size_t)2 * per_step * nsteps, nullptr);
  for (auto& e : ev) CU(cudaEventCreate(&e));
  std::vector<int> grp;
  size_t q = 0;
  auto mark = [&](int g) { grp.push_back(g); return cudaEventRecord(ev[q++], c->stream); };
  auto done = [&]() { return cudaEventRecord(ev[q++], c->stream); };
  for (int s = 0; s < nsteps; ++s) {
    CU(mark(6)); CU(launch_step_begin(c)); if (c->cfg.LES_type > 0) CU(launch_sgs_nut(c)); CU(done());
    for (int ns = 1; ns <= c->iadvance; ++ns) {
      CU(mark(6));
      if (c->cfg.order == 4) CU(launch_visc4_partials(c));
      CU(launch_substep_setup(c, ns));
      if (!march_path(c) && c->cfg.order != 4 && c->cfg.LES_type == 0 && !y_periodic(c) && c->cfg.IsImplicit != 0)
        CU(launch_helm_factors(c));
      CU(done());
      if (march_path(c)) {
        CU(mark(0)); CU(launch_rhs_march(c)); CU(done());
        CU(mark(1)); CU(done());
      } else if (c->cfg.LES_type > 0) {
        CU(mark(0)); CU(launch_rhs_les(c)); CU(done());
        CU(mark(1)); CU(c->cfg.IsImplicit == 0 ? launch_uhat_fexp(c) : launch_uhat_les(c)); CU(done());
      } else if (c->cfg.order == 2 && c->cfg.IsImplicit == 2) {
        CU(mark(0)); CU(launch_rhs_fimp(c)); CU(done());
        CU(mark(1)); CU(launch_ptri_xz(c)); CU(y_periodic(c) ? launch_ptri_y(c) : launch_uhat(c)); CU(done());
      } else if (c->cfg.IsImplicit == 0) {
        CU(mark(0)); CU(launch_rhs_fimp(c)); CU(done());
        CU(mark(1)); CU(launch_uhat_fexp(c)); CU(done());
      } else if (y_periodic(c)) {
        CU(mark(0)); CU(launch_rhs(c)); CU(done());
        CU(mark(1)); CU(launch_ptri_y(c)); CU(done());
      } else {
        CU(mark(0)); CU(launch_rhs_march(c)); CU(done());
        CU(mark(1)); CU(done());
      }
      if (c->gsub) {
        CU(mark(2)); CU(launch_div_bsub(c)); CU(launch_prsrc_xfft(c, 3)); CU(done());
      } else {
        CU(mark(2)); CU(launch_prsrc_xfft(c, 0)); CU(done());
      }
      CU(mark(3)); CU(launch_poisson_spectral(c)); CU(done());
      CU(mark(4)); CU(launch_xifft(c)); CU(done());
      if (ns == c->iadvance && march_diag_fusable(c)) {
        CU(mark(5)); CU(launch_diag_reset(c));
        CU(c->gsub ? launch_proj_bsub(c, true) : launch_proj_diag(c)); CU(done());
      } else {
        CU(mark(5)); CU(c->gsub ? launch_proj_bsub(c, false) : launch_proj(c, 0)); CU(done());
      }
    }
    CU(mark(6)); if (!march_diag_fusable(c)) CU(launch_diag(c)); CU(launch_step_end(c)); CU(done());
  }
  if (q != ev.size()) return fail(CH3D_ERR_INVALID, "kernel_times event count mismatch");
  CU(cudaStreamSynchronize(c->stream));
  std::vector<double> sum(G, 0.0);
  std::vector<int> cnt(G, 0);
  for (size_t m = 0; m < grp.size(); ++m) {
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, ev[2 * m], ev[2 * m + 1]));
    sum[grp[m]] += ms;
    cnt[grp[m]] += 1;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int g = 0; g < G - 1; ++g) out[g] = cnt[g] ? sum[g] / cnt[g] : 0.0;  // per substep
  out[G - 1] = sum[G - 1] / nsteps;                                          // per step
  return fetch_info(c, nullptr);
}

int ch3d_poisson_noalloc(int nxc, int nyc, int nzc, double xlx, double zlz, const double* yp, int bc_ym, int bc_yp,
                         const double* d_src, double* d_phi, void* stream) {
  if (!yp || !d_src || !d_phi) return fail(CH3D_ERR_INVALID, "NULL argument");
  if (nxc < 4 || nyc < 4 || nzc < 2 || (nxc % 2)) return fail(CH3D_ERR_INVALID, "bad grid %d %d %d", nxc, nyc, nzc);
  if (!(xlx > 0) || !(zlz > 0)) return fail(CH3D_ERR_INVALID, "bad domain lengths");
  if ((bc_ym != -1 && bc_ym != -2) || (bc_yp != -1 && bc_yp != -2))
    return fail(CH3D_ERR_UNSUPPORTED, "y boundaries must be no-slip (-1) or free-slip (-2)");
  for (int j = 1; j <= nyc; ++j)
    if (!(yp[j] > yp[j - 1])) return fail(CH3D_ERR_INVALID, "yp must increase");
  FFTPlanDev px, pz;
  if (!factor23(nxc / 2, px) || !factor23(nzc, pz))
    return fail(CH3D_ERR_UNSUPPORTED, "nxc/2 and nzc must be products of 2 and 3");
  const size_t need = noalloc_bytes(nxc, nyc, nzc);
  if (need > (size_t)CH3D_NOALLOC_SCRATCH_BYTES)
    return fail(CH3D_ERR_INVALID, "grid %d x %d x %d needs %zu bytes of scratch, more than the %u bytes of "
                "CH3D_NOALLOC_SCRATCH_BYTES", nxc, nyc, nzc, need, (unsigned)CH3D_NOALLOC_SCRATCH_BYTES);
  const size_t smem = noalloc_smem(nxc, nyc, nzc);
  if (smem > noalloc_smem_limit())
    return fail(CH3D_ERR_UNSUPPORTED, "grid %d x %d x %d: a transform or y-solve block of the allocation-free solve "
                "needs %zu bytes of shared memory, more than its %zu-byte limit", nxc, nyc, nzc, smem,
                noalloc_smem_limit());
  cudaError_t e = poisson_noalloc(nxc, nyc, nzc, xlx, zlz, yp, bc_ym, bc_yp, d_src, d_phi, (cudaStream_t)stream, px, pz);
  if (e != cudaSuccess) return fail(CH3D_ERR_CUDA, "ch3d_poisson_noalloc: %s", cudaGetErrorString(e));
  return CH3D_OK;
}

int ch3d_interp_state(ch3d_ctx* dst, const ch3d_ctx* src) {
  if (!dst || !src || dst == src) return fail(CH3D_ERR_INVALID, "need two distinct contexts");
  if (dst->device != src->device) return fail(CH3D_ERR_INVALID, "both contexts must be on one device");
  if (dst->fp32 != src->fp32) return fail(CH3D_ERR_INVALID, "both contexts must have the same precision");
  if (y_periodic(dst) || y_periodic(src))
    return fail(CH3D_ERR_UNSUPPORTED, "the resampling is built for walls in y (periodic x and z)");
  if (std::fabs(dst->cfg.yly - src->cfg.yly) > 1e-12 * std::fabs(src->cfg.yly))
    return fail(CH3D_ERR_INVALID, "yly differs (%g, %g): the resampling keeps the channel height", src->cfg.yly,
                dst->cfg.yly);
  CU(cudaSetDevice(dst->device));
  const cudaError_t e = launch_interp_state(dst, src);
  if (e == cudaErrorInvalidValue) return fail(CH3D_ERR_INVALID, "a new y point lies outside the old grid");
  if (e != cudaSuccess) return fail(CH3D_ERR_CUDA, "ch3d_interp_state: %s", cudaGetErrorString(e));
  // as a restart read of the resampled field: Hist zero, the wall row of uy, fresh scalars
  const size_t word = dst->fp32 ? sizeof(float) : sizeof(double);
  for (int q = 4; q < 7; ++q) CU(cudaMemsetAsync(dst->f[q], 0, (size_t)dst->N * word, dst->stream));
  CU(launch_fill_row0(dst, 1, dst->cfg.uyBcValue[2]));
  CU(cudaStreamSynchronize(dst->stream));
  return init_scalars(dst);
}

int ch3d_last_step_ms(ch3d_ctx* c, double* ms) {
  if (!c || !ms) return fail(CH3D_ERR_INVALID, "NULL argument");
  *ms = c->last_ms;
  return CH3D_OK;
}

int ch3d_path_flags(ch3d_ctx* c, int* flags) {
  if (!c || !flags) return fail(CH3D_ERR_INVALID, "NULL argument");
  CU(cudaSetDevice(c->device));
  const bool march = march_path(c) || c->cfg.order == 4;
  *flags = (march ? CH3D_PATH_MARCH : 0) | (march && march_twisted(c) ? CH3D_PATH_TWISTED : 0) |
           (c->gsub ? CH3D_PATH_GSUB : 0);
  return CH3D_OK;
}

}  // extern "C"
