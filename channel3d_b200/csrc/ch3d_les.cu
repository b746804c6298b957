// ch3d_les.cu -- sm_100a kernels of the LES step (2nd order, y Crank-Nicolson):
// the eddy viscosity of Clc_SGS_Vis (src/CFD_2nd/m_LESModels.f90:47-428)
// for the WALE and mixed-time-scale models and the Smagorinsky model with
// van Driest damping, the variable-viscosity right-hand sides
// clcRhsX/Y/Z_PIMP_LES and the variable-coefficient y solves
// clcU1/2/3Hat_PIMP_LES (src/CFD_2nd/m_TSchemePIMP_inc.f90:80-387, 466-809).
// FP64.  nut holds the total viscosity (xnu included), interior cells; its
// wall ghosts follow SetBC_and_UpdateHalo_SGS (2 xnu - nut for no-slip walls,
// nut for free-slip), x and z wrap.
#include <cstring>
#include "../../include/ch3d_mlp.h"
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"
#include "mlp_tc.cuh"

namespace ch3d {

// nut at a y row that may be the wall ghost (j = -1 or ny)
template <class T>
__device__ __forceinline__ double nut_at(const T* __restrict__ nut, const Geo<T>& g, const Nbr& n,
                                         long long o, int dj) {
  if (dj < 0 && n.jlo) {
    const double v = __ldg(nut + n.c + o);
    return g.bc.lo == -1 ? 2.0 * (double)g.xnu - v : v;
  }
  if (dj > 0 && n.jhi) {
    const double v = __ldg(nut + n.c + o);
    return g.bc.hi == -1 ? 2.0 * (double)g.xnu - v : v;
  }
  return __ldg(nut + n.c + o + (long long)dj * n.yp);
}

// |S| = sqrt(2 Sij Sij) of ClcVelStrainRate (src/CFD_2nd/m_LESModels.f90:328-370)
template <class T>
__device__ __forceinline__ double strain_rate(const Geo<T>& g, const Metrics<double>& m, const T* ux,
                                              const T* uy, const T* uz, const Nbr& n, int jc) {
  const double rdx = g.rdx, rdz = g.rdz;
  const double caj = m.rdyp[jc], cac1 = m.rdyc[jc], cac2 = m.rdyc[jc + 1], cac12 = cac1 - cac2;
  const double e = 0.125;
  const double st1 = (at(ux, n, n.xp) - at(ux, n, 0)) * rdx;
  const double st2 = (at_jp(uy, g, 1, n, 0) - at(uy, n, 0)) * caj;
  const double st3 = (at(uz, n, n.zp) - at(uz, n, 0)) * rdz;
  const double st4 = e * ((at_jp(uy, g, 1, n, n.xp) - at_jp(uy, g, 1, n, n.xm) + at(uy, n, n.xp) - at(uy, n, n.xm)) * rdx +
                          (at_jp(ux, g, 0, n, n.xp) + at_jp(ux, g, 0, n, 0)) * cac2 +
                          (at(ux, n, n.xp) + at(ux, n, 0)) * cac12 -
                          (at_jm(ux, g, 0, n, n.xp) + at_jm(ux, g, 0, n, 0)) * cac1);
  const double st5 = e * ((at(ux, n, n.xp + n.zp) + at(ux, n, n.zp) - at(ux, n, n.xp + n.zm) - at(ux, n, n.zm)) * rdz +
                          (at(uz, n, n.xp + n.zp) - at(uz, n, n.xm + n.zp) + at(uz, n, n.xp) - at(uz, n, n.xm)) * rdx);
  const double st6 = e * ((at_jp(uy, g, 1, n, n.zp) + at(uy, n, n.zp) - at_jp(uy, g, 1, n, n.zm) - at(uy, n, n.zm)) * rdz +
                          (at_jp(uz, g, 2, n, n.zp) + at_jp(uz, g, 2, n, 0)) * cac2 +
                          (at(uz, n, n.zp) + at(uz, n, 0)) * cac12 -
                          (at_jm(uz, g, 2, n, n.zp) + at_jm(uz, g, 2, n, 0)) * cac1);
  return sqrt(2.0 * (st1 * st1 + st2 * st2 + st3 * st3) + 4.0 * (st4 * st4 + st5 * st5 + st6 * st6));
}

struct LesPar {
  const double* delta;  // DeltaCell(jc), jc = 0..nyp
  const double* dwall;  // wall distance of the cell centre, jc = 1..nyc
  double Fc[9];         // MTS test filter (InitFilterCoe)
  double Cs;
  int model;            // CH3D_LES_*
};

// x-z mean wall shear -> u_tau (Smagorinsky / van Driest); one block
template <class T>
__global__ void __launch_bounds__(1024) k_wall_utau(Geo<T> g, const T* __restrict__ ux, double d1, double dN,
                                                    DevScalars* __restrict__ sc) {
  __shared__ double r1[1024], r2[1024];
  if (sc->status) return;
  const long long plane = (long long)g.nx * g.ny;
  double s1 = 0, s2 = 0;
  for (int q = threadIdx.x; q < g.nx * g.nz; q += blockDim.x) {
    const int i = q % g.nx, k = q / g.nx;
    s1 += ux[i + plane * k];
    s2 += ux[i + (long long)g.nx * (g.ny - 1) + plane * k];
  }
  r1[threadIdx.x] = s1; r2[threadIdx.x] = s2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { r1[threadIdx.x] += r1[threadIdx.x + w]; r2[threadIdx.x] += r2[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double inxz = 1.0 / ((double)g.nx * (double)g.nz);
    const double tw = (double)g.xnu * 0.5 * (fabs(r1[0] * inxz - g.bc.ux_lo) / d1 + fabs(r2[0] * inxz - g.bc.ux_hi) / dN);
    sc->utau = sqrt(tw);
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_sgs_nut(Geo<T> g, Metrics<double> m, LesPar lp,
                                                 const T* __restrict__ ux, const T* __restrict__ uy,
                                                 const T* __restrict__ uz, T* __restrict__ nut,
                                                 const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const Nbr n = make_nbr(g, i, j, k);
  const int jc = j + 1;
  const double xnu = g.xnu, rdx = g.rdx, rdz = g.rdz;
  double v;
  if (lp.model == CH3D_LES_WALE) {  // Clc_SGS_WALE (m_LESModels.f90:72-135)
    const double caj = m.rdyp[jc], cac1 = m.rdyc[jc], cac2 = m.rdyc[jc + 1], cac12 = cac1 - cac2;
    double CwDelta2 = 0.325 * lp.delta[jc];
    CwDelta2 = CwDelta2 * CwDelta2;
    const double dudx = (at(ux, n, n.xp) - at(ux, n, 0)) * rdx;
    const double dudy = ((at_jp(ux, g, 0, n, n.xp) + at_jp(ux, g, 0, n, 0)) * cac2 + (at(ux, n, n.xp) + at(ux, n, 0)) * cac12 -
                         (at_jm(ux, g, 0, n, n.xp) + at_jm(ux, g, 0, n, 0)) * cac1) * 0.25;
    const double dudz = (at(ux, n, n.xp + n.zp) + at(ux, n, n.zp) - at(ux, n, n.xp + n.zm) - at(ux, n, n.zm)) * rdz * 0.25;
    const double dvdx = (at_jp(uy, g, 1, n, n.xp) - at_jp(uy, g, 1, n, n.xm) + at(uy, n, n.xp) - at(uy, n, n.xm)) * rdx * 0.25;
    const double dvdy = (at_jp(uy, g, 1, n, 0) - at(uy, n, 0)) * caj;
    const double dvdz = (at_jp(uy, g, 1, n, n.zp) + at(uy, n, n.zp) - at_jp(uy, g, 1, n, n.zm) - at(uy, n, n.zm)) * rdz * 0.25;
    const double dwdx = (at(uz, n, n.xp + n.zp) - at(uz, n, n.xm + n.zp) + at(uz, n, n.xp) - at(uz, n, n.xm)) * rdx * 0.25;
    const double dwdy = ((at_jp(uz, g, 2, n, n.zp) + at_jp(uz, g, 2, n, 0)) * cac2 + (at(uz, n, n.zp) + at(uz, n, 0)) * cac12 -
                         (at_jm(uz, g, 2, n, n.zp) + at_jm(uz, g, 2, n, 0)) * cac1) * 0.25;
    const double dwdz = (at(uz, n, n.zp) - at(uz, n, 0)) * rdz;
    const double S11 = dudx, S12 = (dudy + dvdx) * 0.5, S13 = (dudz + dwdx) * 0.5;
    const double S22 = dvdy, S23 = (dvdz + dwdy) * 0.5, S33 = dwdz;
    const double SijSij = S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23);
    double Sd11 = dudx * dudx + dudy * dvdx + dudz * dwdx;
    const double Sd12 = (dudx * dudy + dudy * dvdy + dudz * dwdy + dvdx * dudx + dvdy * dvdx + dvdz * dwdx) * 0.5;
    const double Sd13 = (dudx * dudz + dudy * dvdz + dudz * dwdz + dwdx * dudx + dwdy * dvdx + dwdz * dwdx) * 0.5;
    double Sd22 = dvdx * dudy + dvdy * dvdy + dvdz * dwdy;
    const double Sd23 = (dvdx * dudz + dvdy * dvdz + dvdz * dwdz + dwdx * dudy + dwdy * dvdy + dwdz * dwdy) * 0.5;
    double Sd33 = dwdx * dudz + dwdy * dvdz + dwdz * dwdz;
    const double SdTrace = (Sd11 + Sd22 + Sd33) / 3.0;
    Sd11 -= SdTrace; Sd22 -= SdTrace; Sd33 -= SdTrace;
    const double Sd2 = Sd11 * Sd11 + Sd22 * Sd22 + Sd33 * Sd33 + 2.0 * (Sd12 * Sd12 + Sd13 * Sd13 + Sd23 * Sd23);
    v = CwDelta2 * pow(Sd2, 1.5) / (pow(SijSij, 2.5) + pow(Sd2, 1.25)) + xnu;
  } else if (lp.model == CH3D_LES_MTS) {  // Clc_SGS_MTS (m_LESModels.f90:145-258)
    const double* F = lp.Fc;
    // test-filtered fluctuation u - F(u) of a staggered component at offset o of row dj
    auto filt = [&](const T* u, int comp, long long o, int dj) {
      auto val = [&](long long oo) { return dj > 0 ? at_jp(u, g, comp, n, o + oo) : at(u, n, o + oo); };
      return F[0] * val(n.xm + n.zm) + F[1] * val(n.zm) + F[2] * val(n.xp + n.zm) +
             F[3] * val(n.xm) + (F[4] - 1.0) * val(0) + F[5] * val(n.xp) +
             F[6] * val(n.xm + n.zp) + F[7] * val(n.zp) + F[8] * val(n.xp + n.zp);
    };
    // ux at i and i+1 (the i+1 stencil wraps through the offsets of cell i+1)
    const Nbr nx1 = make_nbr(g, (i + 1 == g.nx) ? 0 : i + 1, j, k);
    const double fa = filt(ux, 0, 0, 0);
    double fb;
    {
      const Nbr& q = nx1;
      auto valb = [&](long long oo) { return at(ux, q, oo); };
      fb = F[0] * valb(q.xm + q.zm) + F[1] * valb(q.zm) + F[2] * valb(q.xp + q.zm) + F[3] * valb(q.xm) +
           (F[4] - 1.0) * valb(0) + F[5] * valb(q.xp) + F[6] * valb(q.xm + q.zp) + F[7] * valb(q.zp) +
           F[8] * valb(q.xp + q.zp);
    }
    double Kes = 0.5 * (fa * fa + fb * fb);
    const double ga = filt(uy, 1, 0, 0), gb = filt(uy, 1, 0, 1);  // uy at jc and jc+1 (jc+1 = nyp: wall value)
    Kes = Kes + 0.5 * (ga * ga + gb * gb);
    const Nbr nz1 = make_nbr(g, i, j, (k + 1 == g.nz) ? 0 : k + 1);
    const double ha = filt(uz, 2, 0, 0);
    double hb;
    {
      const Nbr& q = nz1;
      auto valb = [&](long long oo) { return at(uz, q, oo); };
      hb = F[0] * valb(q.xm + q.zm) + F[1] * valb(q.zm) + F[2] * valb(q.xp + q.zm) + F[3] * valb(q.xm) +
           (F[4] - 1.0) * valb(0) + F[5] * valb(q.xp) + F[6] * valb(q.xm + q.zp) + F[7] * valb(q.zp) +
           F[8] * valb(q.xp + q.zp);
    }
    Kes = Kes + 0.5 * (ha * ha + hb * hb);
    const double rdelta = 1.0 / lp.delta[jc];
    double Ts = sqrt(Kes) * rdelta + strain_rate(g, m, ux, uy, uz, n, jc) / 10.0;
    Ts = Ts < 1.0e-10 ? 0.0 : 1.0 / Ts;
    v = 0.05 * Kes * Ts + xnu;
  } else if (lp.model == CH3D_LES_MLP) {  // learned closure: explicit stress force, molecular viscosity
    v = xnu;
  } else {  // Smagorinsky + van Driest damping
    const double D = 1.0 - exp(-(lp.dwall[jc] * sc->utau / xnu) / 26.0);
    const double l = lp.Cs * D * lp.delta[jc];
    v = l * l * strain_rate(g, m, ux, uy, uz, n, jc) + xnu;
  }
  nut[n.c] = (T)v;
}

// clcRhsX/Y/Z_PIMP_LES at one cell; RhsX includes dpmdxns (:140-153).
template <class T>
__global__ void __launch_bounds__(256) k_rhs_les(Geo<T> g, Metrics<double> m, const T* __restrict__ ux,
                                                 const T* __restrict__ uy, const T* __restrict__ uz,
                                                 const T* __restrict__ pr, const T* __restrict__ nut,
                                                 T* __restrict__ hx, T* __restrict__ hy,
                                                 T* __restrict__ hz, T* __restrict__ rx,
                                                 T* __restrict__ ry, T* __restrict__ rz,
                                                 const double* __restrict__ fsgs, const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const Nbr n = make_nbr(g, i, j, k);
  const int jc = j + 1;
  // explicit SGS force of the learned closure (zero for the eddy-viscosity models)
  const double f1 = fsgs ? fsgs[n.c] : 0.0, f2 = fsgs ? fsgs[g.N + n.c] : 0.0, f3 = fsgs ? fsgs[2 * g.N + n.c] : 0.0;
  const double pmGamma = sc->pmGamma, pmTheta = sc->pmTheta, pmAlpha = sc->pmAlpha, pmBetaT = sc->pmBetaT;
  const double rdx = g.rdx, rdz = g.rdz, rdx2 = g.rdx2, rdz2 = g.rdz2;
  const double qdx1 = 0.25 * rdx, qdx3 = 0.25 * rdz;
  // the explicit scheme (clcRhsX/Y/Z_FEXP_LES, src/CFD_2nd/m_TSchemeFEXP_inc.f90:80-155,
  // 213-271, 329-386): the same terms, the y viscous term inside convEd, no pmBetaT term
  const bool fexp = g.implicit == 0;
  auto N = [&](long long o, int dj) { return nut_at(nut, g, n, o, dj); };
  {  // RhsX (m_TSchemePIMP_inc.f90:80-156)
    const double sucaj = 0.25 * m.rdyp[jc];
    const double u_c = at(ux, n, 0), u_ip = at(ux, n, n.xp), u_im = at(ux, n, n.xm);
    const double u_jp = at_jp(ux, g, 0, n, 0), u_jm = at_jm(ux, g, 0, n, 0);
    const double u_kp = at(ux, n, n.zp), u_km = at(ux, n, n.zm);
    const double h11 = ((u_ip + u_c) * (u_ip + u_c) - (u_c + u_im) * (u_c + u_im)) * qdx1;
    const double h12 = ((at_jp(uy, g, 1, n, 0) + at_jp(uy, g, 1, n, n.xm)) * (u_jp + u_c) -
                        (at(uy, n, 0) + at(uy, n, n.xm)) * (u_c + u_jm)) * sucaj;
    const double h13 = ((at(uz, n, n.zp) + at(uz, n, n.xm + n.zp)) * (u_kp + u_c) -
                        (at(uz, n, 0) + at(uz, n, n.xm)) * (u_c + u_km)) * qdx3;
    const double n_c = N(0, 0), n_im = N(n.xm, 0);
    const double visa = 0.25 * (n_c + n_im + N(0, -1) + N(n.xm, -1));
    const double visb = 0.25 * (n_c + n_im + N(0, 1) + N(n.xm, 1));
    const double visc = 0.25 * (n_c + n_im + N(n.zm, 0) + N(n.xm + n.zm, 0));
    const double visd = 0.25 * (n_c + n_im + N(n.zp, 0) + N(n.xm + n.zp, 0));
    const double sgs1 = rdx2 * (n_c * (u_ip - u_c) - n_im * (u_c - u_im));
    const double sgs2 = rdx * m.rdyp[jc] * (visb * (at_jp(uy, g, 1, n, 0) - at_jp(uy, g, 1, n, n.xm)) -
                                            visa * (at(uy, n, 0) - at(uy, n, n.xm)));
    const double sgs3 = rdx * rdz * (visd * (at(uz, n, n.zp) - at(uz, n, n.xm + n.zp)) - visc * (at(uz, n, 0) - at(uz, n, n.xm)));
    const double d22q1 = m.ap2c[jc] * visb * (u_jp - u_c) - m.am2c[jc] * visa * (u_c - u_jm);
    const double d33q1 = g.ap3c * visd * (u_kp - u_c) - g.am3c * visc * (u_c - u_km);
    const double dcq13 = fexp ? sgs1 + d22q1 + d33q1 : sgs1 + d33q1;  // FEXP: the y term explicit too
    const double gradp1 = (at(pr, n, 0) - at(pr, n, n.xm)) * rdx;
    const double conv = -h11 - h12 - h13 + sgs1 + sgs2 + sgs3 + dcq13 + g.g1 + f1;
    const double ho = hx[n.c];
    hx[n.c] = (T)conv;
    const double r = pmGamma * conv + pmTheta * ho - pmAlpha * gradp1;
    rx[n.c] = (T)((fexp ? r : r + 2.0 * pmBetaT * d22q1) + sc->dpmdxns);
  }
  {  // RhsY (:214-272)
    const double sucac = m.rdyc[jc], qsucac = 0.25 * sucac;
    const double v_c = at(uy, n, 0), v_ip = at(uy, n, n.xp), v_im = at(uy, n, n.xm);
    const double v_jp = at_jp(uy, g, 1, n, 0), v_jm = at_jm(uy, g, 1, n, 0);
    const double v_kp = at(uy, n, n.zp), v_km = at(uy, n, n.zm);
    const double h21 = ((at(ux, n, n.xp) + at_jm(ux, g, 0, n, n.xp)) * (v_ip + v_c) -
                        (at(ux, n, 0) + at_jm(ux, g, 0, n, 0)) * (v_c + v_im)) * qdx1;
    const double h22 = ((v_jp + v_c) * (v_jp + v_c) - (v_c + v_jm) * (v_c + v_jm)) * qsucac;
    const double h23 = ((at(uz, n, n.zp) + at_jm(uz, g, 2, n, n.zp)) * (v_kp + v_c) -
                        (at(uz, n, 0) + at_jm(uz, g, 2, n, 0)) * (v_c + v_km)) * qdx3;
    const double n_c = N(0, 0), n_jm = N(0, -1);
    const double visa = 0.25 * (n_c + N(n.xm, 0) + n_jm + N(n.xm, -1));
    const double visb = 0.25 * (n_c + N(n.xp, 0) + n_jm + N(n.xp, -1));
    const double visc = 0.25 * (n_c + n_jm + N(n.zm, 0) + N(n.zm, -1));
    const double visd = 0.25 * (n_c + n_jm + N(n.zp, 0) + N(n.zp, -1));
    const double sgs1 = rdx * sucac * (visb * (at(ux, n, n.xp) - at_jm(ux, g, 0, n, n.xp)) - visa * (at(ux, n, 0) - at_jm(ux, g, 0, n, 0)));
    const double sgs2 = m.ap2p[jc] * n_c * (v_jp - v_c) - m.am2p[jc] * n_jm * (v_c - v_jm);
    const double sgs3 = rdz * sucac * (visd * (at(uz, n, n.zp) - at_jm(uz, g, 2, n, n.zp)) - visc * (at(uz, n, 0) - at_jm(uz, g, 2, n, 0)));
    const double d11q2 = g.ap1c * visb * (v_ip - v_c) - g.am1c * visa * (v_c - v_im);
    const double d33q2 = g.ap3c * visd * (v_kp - v_c) - g.am3c * visc * (v_c - v_km);
    const double dcq13 = fexp ? d11q2 + sgs2 + d33q2 : d11q2 + d33q2;
    const double gradp2 = (at(pr, n, 0) - at_jm(pr, g, 3, n, 0)) * sucac;
    const double conv = -h21 - h22 - h23 + sgs1 + sgs2 + sgs3 + dcq13 + g.g2 + f2;
    const double ho = hy[n.c];
    hy[n.c] = (T)conv;
    const double r = pmGamma * conv + pmTheta * ho - pmAlpha * gradp2;
    ry[n.c] = (T)(fexp ? r : r + 2.0 * pmBetaT * sgs2);
  }
  {  // RhsZ (:330-387)
    const double sucaj = 0.25 * m.rdyp[jc];
    const double w_c = at(uz, n, 0), w_ip = at(uz, n, n.xp), w_im = at(uz, n, n.xm);
    const double w_jp = at_jp(uz, g, 2, n, 0), w_jm = at_jm(uz, g, 2, n, 0);
    const double w_kp = at(uz, n, n.zp), w_km = at(uz, n, n.zm);
    const double h31 = ((at(ux, n, n.xp) + at(ux, n, n.xp + n.zm)) * (w_ip + w_c) -
                        (at(ux, n, 0) + at(ux, n, n.zm)) * (w_c + w_im)) * qdx1;
    const double h32 = ((at_jp(uy, g, 1, n, 0) + at_jp(uy, g, 1, n, n.zm)) * (w_jp + w_c) -
                        (at(uy, n, 0) + at(uy, n, n.zm)) * (w_c + w_jm)) * sucaj;
    const double h33 = ((w_kp + w_c) * (w_kp + w_c) - (w_c + w_km) * (w_c + w_km)) * qdx3;
    const double n_c = N(0, 0), n_km = N(n.zm, 0);
    const double visa = 0.25 * (n_km + N(n.xm + n.zm, 0) + n_c + N(n.xm, 0));
    const double visb = 0.25 * (n_km + N(n.xp + n.zm, 0) + n_c + N(n.xp, 0));
    const double visc = 0.25 * (n_km + N(n.zm, -1) + N(0, -1) + n_c);
    const double visd = 0.25 * (n_km + N(n.zm, 1) + N(0, 1) + n_c);
    const double sgs1 = rdx * rdz * (visb * (at(ux, n, n.xp) - at(ux, n, n.xp + n.zm)) - visa * (at(ux, n, 0) - at(ux, n, n.zm)));
    const double sgs2 = rdz * m.rdyp[jc] * (visd * (at_jp(uy, g, 1, n, 0) - at_jp(uy, g, 1, n, n.zm)) -
                                            visc * (at(uy, n, 0) - at(uy, n, n.zm)));
    const double sgs3 = rdz2 * (n_c * (w_kp - w_c) - n_km * (w_c - w_km));
    const double d11q3 = g.ap1c * visb * (w_ip - w_c) - g.am1c * visa * (w_c - w_im);
    const double d22q3 = m.ap2c[jc] * visd * (w_jp - w_c) - m.am2c[jc] * visc * (w_c - w_jm);
    const double dcq13 = fexp ? d11q3 + d22q3 + sgs3 : d11q3 + sgs3;
    const double gradp3 = (at(pr, n, 0) - at(pr, n, n.zm)) * rdz;
    const double conv = -h31 - h32 - h33 + sgs1 + sgs2 + sgs3 + dcq13 + g.g3 + f3;
    const double ho = hz[n.c];
    hz[n.c] = (T)conv;
    const double r = pmGamma * conv + pmTheta * ho - pmAlpha * gradp3;
    rz[n.c] = (T)(fexp ? r : r + 2.0 * pmBetaT * d22q3);
  }
}

// clcU1/2/3Hat_PIMP_LES: one thread per (i, k) column, Thomas along y
// (InverseTridiagonal, src/CFD_2nd/m_Tools.f90:224-251) with the column's own
// coefficients; the u* buffer holds the elimination factors until the back
// substitution overwrites them.  blockIdx.y = component.
// coefficients (a, b, c) of row j of the variable-viscosity Crank-Nicolson
// system of component comp in column (i, k)
template <class T>
__device__ __forceinline__ void uhat_les_coef(const Geo<T>& g, const HelmCoef& hc, const T* __restrict__ nut,
                                              double pmBetaT, int comp, int i, int j, int k, double& a, double& b,
                                              double& c) {
  const Nbr n = make_nbr(g, i, j, k);
  const int jc = j + 1;
  double rt1, rt2;
  if (comp == 1) {
    if (j == 0) { a = 0.0; b = 1.0; c = 0.0; return; }
    rt1 = pmBetaT * nut_at(nut, g, n, 0, -1) * hc.am2p[jc];
    rt2 = pmBetaT * nut_at(nut, g, n, 0, 0) * hc.ap2p[jc];
  } else {
    const long long o = comp == 0 ? n.xm : n.zm;
    const double visc = comp == 0 ? 0.25 * (nut_at(nut, g, n, 0, 0) + nut_at(nut, g, n, o, 0) + nut_at(nut, g, n, 0, -1) + nut_at(nut, g, n, o, -1))
                                  : 0.25 * (nut_at(nut, g, n, o, 0) + nut_at(nut, g, n, o, -1) + nut_at(nut, g, n, 0, 0) + nut_at(nut, g, n, 0, -1));
    const double visd = comp == 0 ? 0.25 * (nut_at(nut, g, n, 0, 0) + nut_at(nut, g, n, o, 0) + nut_at(nut, g, n, 0, 1) + nut_at(nut, g, n, o, 1))
                                  : 0.25 * (nut_at(nut, g, n, o, 0) + nut_at(nut, g, n, o, 1) + nut_at(nut, g, n, 0, 0) + nut_at(nut, g, n, 0, 1));
    rt1 = pmBetaT * visc * hc.am2cForCN[jc];
    rt2 = pmBetaT * visd * hc.ap2cForCN[jc];
  }
  a = -rt1; b = rt1 + rt2 + 1.0; c = -rt2;
}

template <class T>
__global__ void __launch_bounds__(128) k_uhat_les(Geo<T> g, HelmCoef hc, const T* __restrict__ nut,
                                                  const T* __restrict__ ux, const T* __restrict__ uy,
                                                  const T* __restrict__ uz, T* __restrict__ rx,
                                                  T* __restrict__ ry, T* __restrict__ rz,
                                                  T* __restrict__ uxs, T* __restrict__ uys,
                                                  T* __restrict__ uzs, const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= g.nx * g.nz) return;
  const int comp = blockIdx.y;
  const int i = col % g.nx, k = col / g.nx;
  const T* u = comp == 0 ? ux : (comp == 1 ? uy : uz);
  T* r = comp == 0 ? rx : (comp == 1 ? ry : rz);  // the RHS column is consumed in place
  T* us = comp == 0 ? uxs : (comp == 1 ? uys : uzs);
  const double pmBetaT = sc->pmBetaT;
  const int ny = g.ny;
  const long long nxl = g.nx;
  auto coef = [&](int j, double& a, double& b, double& c) { uhat_les_coef(g, hc, nut, pmBetaT, comp, i, j, k, a, b, c); };
  const long long base = i + nxl * ny * k;
  double a, b, c;
  coef(0, a, b, c);
  double vecm = b;
  // row 1 of the uy system is the wall condition duy_ym = 0 (constant wall velocity)
  double f = (comp == 1 ? 0.0 : r[base]) / vecm;
  r[base] = f;
  double cprev = c;
  // forward sweep; arr(j) = c(j-1)/vecm(j-1) is parked in the u* column
  for (int j = 1; j < ny; ++j) {
    coef(j, a, b, c);
    const double arr = cprev / vecm;
    us[base + nxl * j] = arr;
    vecm = b - a * arr;
    f = (r[base + nxl * j] - a * f) / vecm;
    r[base + nxl * j] = f;
    cprev = c;
  }
  // back substitution f(j) -= arr(j+1) f(j+1), then u* = u + f
  double fn = f;
  for (int j = ny - 2; j >= 0; --j) {
    const double arr = us[base + nxl * (j + 1)];
    us[base + nxl * (j + 1)] = u[base + nxl * (j + 1)] + fn;
    fn = r[base + nxl * j] - arr * fn;
  }
  us[base] = u[base] + fn;
}

// The same solves for small grids, 16 columns per block of 128 threads (8
// row groups of 16): the threads form every row's coefficients and
// right-hand side in parallel (their loads independent of the recurrence)
// into shared memory, the first 16 threads run the forward elimination and
// the back substitution there, and all threads write u* = u + x and the
// forward-swept right-hand side (what the one-thread-per-column kernel
// leaves in the RHS array).  Shared memory: 4 x 16 x ny doubles; at 48^3 the
// 432 blocks are one wave on 148 SMs (32-column blocks: 1.5 waves, 21 us).
constexpr int kUhatTileCols = 16;
constexpr size_t kUhatTileSmemMax = 100 * 1024;  // ny <= 200
template <class T>
__global__ void __launch_bounds__(128) k_uhat_les_tile(Geo<T> g, HelmCoef hc, const T* __restrict__ nut,
                                                       const T* __restrict__ ux, const T* __restrict__ uy,
                                                       const T* __restrict__ uz, T* __restrict__ rx,
                                                       T* __restrict__ ry, T* __restrict__ rz,
                                                       T* __restrict__ uxs, T* __restrict__ uys,
                                                       T* __restrict__ uzs, const DevScalars* __restrict__ sc) {
  extern __shared__ double tl[];
  if (sc->status) return;  // uniform over the block
  const int ny = g.ny, ncol = g.nx * g.nz;
  double* A = tl;                                // a(j), then arr(j)
  double* B = A + kUhatTileCols * ny;            // b(j), then the solution x(j)
  double* C = B + kUhatTileCols * ny;            // c(j)
  double* F = C + kUhatTileCols * ny;            // right-hand side, then its forward-swept values
  const int lane = threadIdx.x % kUhatTileCols, wy = threadIdx.x / kUhatTileCols;  // wy: row group 0..7
  const int col = blockIdx.x * kUhatTileCols + lane;
  const bool valid = col < ncol;
  const int comp = blockIdx.y;
  const int i = valid ? col % g.nx : 0, k = valid ? col / g.nx : 0;
  const T* u = comp == 0 ? ux : (comp == 1 ? uy : uz);
  T* r = comp == 0 ? rx : (comp == 1 ? ry : rz);
  T* us = comp == 0 ? uxs : (comp == 1 ? uys : uzs);
  const double pmBetaT = sc->pmBetaT;
  const long long nxl = g.nx;
  const long long base = i + nxl * ny * k;
  if (valid) {
    for (int j = wy; j < ny; j += 8) {
      double a, b, c;
      uhat_les_coef(g, hc, nut, pmBetaT, comp, i, j, k, a, b, c);
      const int e = j * kUhatTileCols + lane;
      A[e] = a;
      B[e] = b;
      C[e] = c;
      // row 1 of the uy system is the wall condition duy_ym = 0 (constant wall velocity)
      F[e] = (comp == 1 && j == 0) ? 0.0 : r[base + nxl * j];
    }
  }
  __syncthreads();
  if (wy == 0 && valid) {
    double vecm = B[lane];
    double f = F[lane] / vecm;
    F[lane] = f;
    double cprev = C[lane];
    for (int j = 1; j < ny; ++j) {
      const int e = j * kUhatTileCols + lane;
      const double a = A[e];
      const double arr = cprev / vecm;
      A[e] = arr;
      vecm = B[e] - a * arr;
      f = (F[e] - a * f) / vecm;
      F[e] = f;
      cprev = C[e];
    }
    double fn = f;
    for (int j = ny - 2; j >= 0; --j) {
      const int e1 = (j + 1) * kUhatTileCols + lane;
      B[e1] = fn;
      fn = F[j * kUhatTileCols + lane] - A[e1] * fn;
    }
    B[lane] = fn;
  }
  __syncthreads();
  if (valid) {
    for (int j = wy; j < ny; j += 8) {
      const int e = j * kUhatTileCols + lane;
      const long long q = base + nxl * j;
      us[q] = u[q] + B[e];
      r[q] = F[e];
    }
  }
}

// ---------------------------------------------------------------------------
// Learned closure (LES_type = CH3D_LES_MLP; no counterpart in the reference).
// Per step: cell-centre velocity gradients g_ij = du_i/dx_j and y+ form the
// network input (standardised with the training statistics); the network
// predicts the six SGS stresses tau_ij / u_tau^2 (standardised); points whose
// input leaves the training range use the Smagorinsky / van Driest stress
// tau_ij = -2 nu_t S_ij instead.  The explicit force -d tau_ij / dx_j at the
// staggered velocity points enters the convective part of the RHS.
// ---------------------------------------------------------------------------
struct MlpNorm {
  float in_mean[10], in_std[10], in_lo[10], in_hi[10];  // lo/hi: training range of the standardised inputs
  float out_mean[6], out_std[6];
};
// the same on the device: input means and reciprocal standard deviations in FP64
struct MlpNormD {
  double in_mean[10], in_rstd[10];
  float in_lo[10], in_hi[10];
  float out_mean[6], out_std[6];
};

// cell-centre gradients (the WALE stencils, m_LESModels.f90:98-111)
template <class T>
__device__ __forceinline__ void cell_gradients(const Geo<T>& g, const Metrics<double>& m, const T* ux,
                                               const T* uy, const T* uz, const Nbr& n, int jc,
                                               double* G /* 9: dudx dudy dudz dvdx dvdy dvdz dwdx dwdy dwdz */) {
  const double rdx = g.rdx, rdz = g.rdz;
  const double caj = m.rdyp[jc], cac1 = m.rdyc[jc], cac2 = m.rdyc[jc + 1], cac12 = cac1 - cac2;
  G[0] = (at(ux, n, n.xp) - at(ux, n, 0)) * rdx;
  G[1] = ((at_jp(ux, g, 0, n, n.xp) + at_jp(ux, g, 0, n, 0)) * cac2 + (at(ux, n, n.xp) + at(ux, n, 0)) * cac12 -
          (at_jm(ux, g, 0, n, n.xp) + at_jm(ux, g, 0, n, 0)) * cac1) * 0.25;
  G[2] = (at(ux, n, n.xp + n.zp) + at(ux, n, n.zp) - at(ux, n, n.xp + n.zm) - at(ux, n, n.zm)) * rdz * 0.25;
  G[3] = (at_jp(uy, g, 1, n, n.xp) - at_jp(uy, g, 1, n, n.xm) + at(uy, n, n.xp) - at(uy, n, n.xm)) * rdx * 0.25;
  G[4] = (at_jp(uy, g, 1, n, 0) - at(uy, n, 0)) * caj;
  G[5] = (at_jp(uy, g, 1, n, n.zp) + at(uy, n, n.zp) - at_jp(uy, g, 1, n, n.zm) - at(uy, n, n.zm)) * rdz * 0.25;
  G[6] = (at(uz, n, n.xp + n.zp) - at(uz, n, n.xm + n.zp) + at(uz, n, n.xp) - at(uz, n, n.xm)) * rdx * 0.25;
  G[7] = ((at_jp(uz, g, 2, n, n.zp) + at_jp(uz, g, 2, n, 0)) * cac2 + (at(uz, n, n.zp) + at(uz, n, 0)) * cac12 -
          (at_jm(uz, g, 2, n, n.zp) + at_jm(uz, g, 2, n, 0)) * cac1) * 0.25;
  G[8] = (at(uz, n, n.zp) - at(uz, n, 0)) * rdz;
}

// The learned closure's stresses, one tile of 128 consecutive cells per CTA:
// each thread forms its cell's network inputs (the nine cell-centre velocity
// gradients in wall units g nu / u_tau^2, then y+; standardised in FP64 and
// rounded to FP32) and the Smagorinsky / van Driest fallback stress
// -2 nu_t S_ij, the CTA runs the network on the tensor cores (mlp_tc.cuh),
// and each thread writes tau [6][N]: the network's output de-standardised
// and scaled by u_tau^2, or the fallback where an input left the training
// range.  When a wait on the tensor cores expires the kernel records it in
// *mstatus and writes the fallback stresses.
template <class T>
__global__ void __launch_bounds__(ch3d_mlp::TILE, 6)
    k_sgs_mlp(Geo<T> g, Metrics<double> m, LesPar lp, MlpNormD nm, const T* __restrict__ ux,
              const T* __restrict__ uy, const T* __restrict__ uz, const unsigned char* __restrict__ img,
              double* __restrict__ tau, int* __restrict__ mstatus, const DevScalars* __restrict__ sc) {
  using namespace ch3d_mlp;
  extern __shared__ __align__(1024) unsigned char smem[];
  if (sc->status) return;  // uniform: every thread reads the same word
  fwd_prologue_packed(smem, img);  // the parameter image arrives while the inputs are formed
  const long long N = g.N;  // below 2^31 (checked by the launch)
  const int c = blockIdx.x * TILE + threadIdx.x;
  const bool valid = c < N;
  float x[NIN];
  double fb[6] = {0, 0, 0, 0, 0, 0};
  bool out = true;
  const double ut = sc->utau > 1e-30 ? sc->utau : 1e-30;
  if (valid) {
    const unsigned cu = (unsigned)c, row = cu / (unsigned)g.nx;
    const int i = (int)(cu - row * (unsigned)g.nx), k = (int)(row / (unsigned)g.ny), j = (int)(row - (unsigned)k * g.ny);
    const Nbr n = make_nbr(g, i, j, k);
    const int jc = j + 1;
    double G[9];
    cell_gradients(g, m, ux, uy, uz, n, jc, G);
    const double gs = (double)g.xnu / (ut * ut);
    const double yplus = lp.dwall[jc] * ut / (double)g.xnu;
    out = false;
#pragma unroll
    for (int q = 0; q < NIN; ++q) {
      const double v = q < 9 ? G[q] * gs : yplus;
      const float xs = (float)((v - nm.in_mean[q]) * nm.in_rstd[q]);
      x[q] = xs;
      out = out || !(xs >= nm.in_lo[q] && xs <= nm.in_hi[q]);
    }
    const double S11 = G[0], S22 = G[4], S33 = G[8];
    const double S12 = 0.5 * (G[1] + G[3]), S13 = 0.5 * (G[2] + G[6]), S23 = 0.5 * (G[5] + G[7]);
    const double Smag = sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23)));
    const double D = 1.0 - exp(-yplus / 26.0);
    const double l = lp.Cs * D * lp.delta[jc];
    const double nt = l * l * Smag;
    fb[0] = -2.0 * nt * S11;
    fb[1] = -2.0 * nt * S12;
    fb[2] = -2.0 * nt * S13;
    fb[3] = -2.0 * nt * S22;
    fb[4] = -2.0 * nt * S23;
    fb[5] = -2.0 * nt * S33;
  } else {
#pragma unroll
    for (int q = 0; q < NIN; ++q) x[q] = 0.f;
  }
  float y[NOUT];
  bool ok = false;
  if (fwd_inputs(smem, x)) ok = fwd_layers(smem, y, nullptr, nullptr, c, valid, N);
  else fwd_abort(smem);
  if (!ok && threadIdx.x == 0) atomicExch(mstatus, 1);
  if (!valid) return;
  const double u2 = sc->utau * sc->utau;
#pragma unroll
  for (int q = 0; q < NOUT; ++q)
    tau[(long long)q * N + c] = (out || !ok) ? fb[q] : ((double)y[q] * nm.out_std[q] + nm.out_mean[q]) * u2;
}

// f_i = -d tau_ij / dx_j at the staggered points of u_i.  Off-diagonal
// stresses are averaged from the four surrounding cell centres onto the cell
// edges; they vanish on the walls.
template <class T>
__global__ void __launch_bounds__(256) k_sgs_force(Geo<T> g, Metrics<double> m, const double* __restrict__ tau,
                                                   double* __restrict__ fx, double* __restrict__ fy,
                                                   double* __restrict__ fz, const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const Nbr n = make_nbr(g, i, j, k);
  const int jc = j + 1;
  const long long N = g.N;
  const double* t11 = tau;
  const double* t12 = tau + N;
  const double* t13 = tau + 2 * N;
  const double* t22 = tau + 3 * N;
  const double* t23 = tau + 4 * N;
  const double* t33 = tau + 5 * N;
  const double rdx = g.rdx, rdz = g.rdz;
  // edge averages of a cell-centred field over the cells at offsets {0, o1} x {0, o2}
  auto e4 = [&](const double* t, long long o1, long long o2) {
    return 0.25 * (at(t, n, 0) + at(t, n, o1) + at(t, n, o2) + at(t, n, o1 + o2));
  };
  // y-edge averages (j -/+ 1/2); zero on the walls
  auto ey = [&](const double* t, long long o1, int up) {
    if (up ? n.jhi : n.jlo) return 0.0;
    const long long oy = up ? (long long)n.yp : -(long long)n.yp;
    return 0.25 * (at(t, n, 0) + at(t, n, o1) + at(t, n, oy) + at(t, n, o1 + oy));
  };
  {  // x momentum at (i-1/2, j, k)
    const double d1 = (at(t11, n, 0) - at(t11, n, n.xm)) * rdx;
    const double d2 = (ey(t12, n.xm, 1) - ey(t12, n.xm, 0)) * m.rdyp[jc];
    const double d3 = (e4(t13, n.xm, n.zp) - e4(t13, n.xm, n.zm)) * rdz;
    fx[n.c] = -(d1 + d2 + d3);
  }
  {  // y momentum at (i, j-1/2, k); the wall row (j = 0) is fixed by the wall condition
    double v = 0.0;
    if (!n.jlo) {
      const long long ym = -(long long)n.yp;
      const double d1 = (e4(t12, n.xp, ym) - e4(t12, n.xm, ym)) * rdx;
      const double d2 = (at(t22, n, 0) - at(t22, n, ym)) * m.rdyc[jc];
      const double d3 = (e4(t23, n.zp, ym) - e4(t23, n.zm, ym)) * rdz;
      v = -(d1 + d2 + d3);
    }
    fy[n.c] = v;
  }
  {  // z momentum at (i, j, k-1/2)
    const double d1 = (e4(t13, n.xp, n.zm) - e4(t13, n.xm, n.zm)) * rdx;
    const double d2 = (ey(t23, n.zm, 1) - ey(t23, n.zm, 0)) * m.rdyp[jc];
    const double d3 = (at(t33, n, 0) - at(t33, n, n.zm)) * rdz;
    fz[n.c] = -(d1 + d2 + d3);
  }
}

// Training samples: one thread per box of fx x fy x fz cells (anchored at
// multiples of the box size), volume-weighted box averages in y.
__global__ void __launch_bounds__(128) k_sgs_train_samples(Geo<double> g, Metrics<double> m, const double* __restrict__ yc,
                                                           const double* __restrict__ ux, const double* __restrict__ uy,
                                                           const double* __restrict__ uz, int fx, int fy, int fz,
                                                           float* __restrict__ X, float* __restrict__ T, double ylo,
                                                           double yhi, const DevScalars* __restrict__ sc) {
  const int bx = g.nx / fx, by = g.ny / fy, bz = g.nz / fz;
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= (long long)bx * by * bz) return;
  const int ib = (int)(b % bx), jb = (int)((b / bx) % by), kb = (int)(b / ((long long)bx * by));
  double W = 0, Y = 0, U[3] = {0, 0, 0}, UU[6] = {0, 0, 0, 0, 0, 0}, GG[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int kk = 0; kk < fz; ++kk)
    for (int jj = 0; jj < fy; ++jj)
      for (int ii = 0; ii < fx; ++ii) {
        const int i = ib * fx + ii, j = jb * fy + jj, k = kb * fz + kk, jc = j + 1;
        const Nbr n = make_nbr(g, i, j, k);
        const double w = m.dyp[jc];
        const double u = 0.5 * (at(ux, n, 0) + at(ux, n, n.xp));
        const double v = 0.5 * (at(uy, n, 0) + at_jp(uy, g, 1, n, 0));
        const double z = 0.5 * (at(uz, n, 0) + at(uz, n, n.zp));
        double G[9];
        cell_gradients(g, m, ux, uy, uz, n, jc, G);
        W += w; Y += w * yc[jc];
        U[0] += w * u; U[1] += w * v; U[2] += w * z;
        UU[0] += w * u * u; UU[1] += w * u * v; UU[2] += w * u * z;
        UU[3] += w * v * v; UU[4] += w * v * z; UU[5] += w * z * z;
        for (int q = 0; q < 9; ++q) GG[q] += w * G[q];
      }
  const double iw = 1.0 / W;
  const double ut = sc->utau > 1e-30 ? sc->utau : 1e-30;
  const double gs = (double)g.xnu / (ut * ut), ts = 1.0 / (ut * ut);
  const double yb = Y * iw;
  const double dw = fmin(yb - ylo, yhi - yb);
  for (int q = 0; q < 9; ++q) X[b * 10 + q] = (float)(GG[q] * iw * gs);
  X[b * 10 + 9] = (float)(dw * ut / (double)g.xnu);
  const double u0 = U[0] * iw, u1 = U[1] * iw, u2 = U[2] * iw;
  T[b * 6 + 0] = (float)((UU[0] * iw - u0 * u0) * ts);
  T[b * 6 + 1] = (float)((UU[1] * iw - u0 * u1) * ts);
  T[b * 6 + 2] = (float)((UU[2] * iw - u0 * u2) * ts);
  T[b * 6 + 3] = (float)((UU[3] * iw - u1 * u1) * ts);
  T[b * 6 + 4] = (float)((UU[4] * iw - u1 * u2) * ts);
  T[b * 6 + 5] = (float)((UU[5] * iw - u2 * u2) * ts);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static LesPar les_par(const ch3d_ctx* c) {
  LesPar lp;
  lp.delta = c->les_delta;
  lp.dwall = c->les_delta + (c->ny + 2);
  const double tr[9] = {1, 2, 1, 2, 4, 2, 1, 2, 1}, si[9] = {1, 4, 1, 4, 16, 4, 1, 4, 1};
  for (int q = 0; q < 9; ++q) lp.Fc[q] = c->cfg.FilterType == 1 ? si[q] / 36.0 : tr[q] / 16.0;
  lp.Cs = c->cfg.Cs;
  lp.model = c->cfg.LES_type;
  return lp;
}

static dim3 les_grid(const ch3d_ctx* c) { return dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz); }

template <class T> static cudaError_t sgs_nut_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  const Geo<T> g = make_geo<T>(c);
  const LesPar lp = les_par(c);
  if (lp.model == CH3D_LES_SMAG_VD || lp.model == CH3D_LES_MLP) {
    const double d1 = c->yc[1] - c->yp[1], dN = c->yp[c->ny + 1] - c->yc[c->ny];
    k_wall_utau<T><<<1, 1024, 0, c->stream>>>(g, f[0], d1, dN, c->sc);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // the learned closure keeps nut = xnu (filled when the context was created)
  if (lp.model != CH3D_LES_MLP) {
    k_sgs_nut<T><<<les_grid(c), dim3(32, 8), 0, c->stream>>>(g, c->m64, lp, f[0], f[1], f[2], f[11], c->sc);
    return cudaGetLastError();
  }
  MlpNorm nh;
  static_assert(sizeof(MlpNorm) == CH3D_SGS_NORM_FLOATS * sizeof(float), "norm layout");
  memcpy(&nh, c->mlp_norm, sizeof(nh));
  MlpNormD nm;
  for (int q = 0; q < 10; ++q) {
    nm.in_mean[q] = nh.in_mean[q];
    nm.in_rstd[q] = 1.0 / (double)nh.in_std[q];
    nm.in_lo[q] = nh.in_lo[q];
    nm.in_hi[q] = nh.in_hi[q];
  }
  for (int q = 0; q < 6; ++q) { nm.out_mean[q] = nh.out_mean[q]; nm.out_std[q] = nh.out_std[q]; }
  if (c->N >= (1LL << 31)) return cudaErrorInvalidValue;  // 32-bit cell indices in k_sgs_mlp
  static PerDevice attr;  // per precision (template instance)
  cudaError_t e = once_per_device(attr, c->device, [] {
    cudaError_t r =
        cudaFuncSetAttribute(k_sgs_mlp<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ch3d_mlp::FwdSmem::BYTES);
    if (r == cudaSuccess)  // all of the SM's on-chip memory as shared memory: six CTAs per SM
      r = cudaFuncSetAttribute(k_sgs_mlp<T>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return r;
  });
  if (e != cudaSuccess) return e;
  k_sgs_mlp<T><<<(unsigned)((c->N + ch3d_mlp::TILE - 1) / ch3d_mlp::TILE), ch3d_mlp::TILE, ch3d_mlp::FwdSmem::BYTES,
                 c->stream>>>(g, c->m64, lp, nm, f[0], f[1], f[2], c->mlp_packed, c->sgs_tau, c->mlp_status, c->sc);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_sgs_force<T><<<les_grid(c), dim3(32, 8), 0, c->stream>>>(g, c->m64, c->sgs_tau, c->sgs_f, c->sgs_f + c->N,
                                                             c->sgs_f + 2 * c->N, c->sc);
  return cudaGetLastError();
}
cudaError_t launch_sgs_nut(ch3d_ctx* c) { return c->fp32 ? sgs_nut_t<float>(c) : sgs_nut_t<double>(c); }

// the network's parameter image (BF16 operands and FP32 biases as the
// forward pass holds them in shared memory), once per parameter set
__global__ void __launch_bounds__(128) k_mlp_pack(const float* __restrict__ P, unsigned char* __restrict__ img) {
  ch3d_mlp::pack_params(img, P);
}

cudaError_t launch_mlp_pack(ch3d_ctx* c) {
  k_mlp_pack<<<1, 128, 0, c->stream>>>(c->mlp_params, c->mlp_packed);
  return cudaGetLastError();
}

// nut = xnu everywhere (the learned closure's total viscosity)
template <class T> __global__ void k_fill_nut(T* __restrict__ nut, long long N, double xnu) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < N) nut[q] = (T)xnu;
}

cudaError_t launch_fill_nut(ch3d_ctx* c) {
  const unsigned grid = (unsigned)((c->N + 255) / 256);
  if (c->fp32) k_fill_nut<float><<<grid, 256, 0, c->stream>>>((float*)c->f[11], c->N, c->cfg.xnu);
  else k_fill_nut<double><<<grid, 256, 0, c->stream>>>((double*)c->f[11], c->N, c->cfg.xnu);
  return cudaGetLastError();
}

cudaError_t launch_sgs_samples(ch3d_ctx* c, int fx, int fy, int fz, float* X, float* T) {
  double** f = (double**)c->f;
  const Geo<double> g = make_geo<double>(c);
  const double d1 = c->yc[1] - c->yp[1], dN = c->yp[c->ny + 1] - c->yc[c->ny];
  k_wall_utau<<<1, 1024, 0, c->stream>>>(g, f[0], d1, dN, c->sc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long nb = (long long)(c->nx / fx) * (c->ny / fy) * (c->nz / fz);
  const double* yc = c->met64 + 16 * (c->ny + 3);  // packed yc (pack_metrics, vector 16)
  k_sgs_train_samples<<<(unsigned)((nb + 127) / 128), 128, 0, c->stream>>>(g, c->m64full, yc, f[0], f[1], f[2], fx, fy,
                                                                          fz, X, T, c->yp[1], c->yp[c->ny + 1], c->sc);
  return cudaGetLastError();
}

template <class T> static cudaError_t rhs_les_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  k_rhs_les<T><<<les_grid(c), dim3(32, 8), 0, c->stream>>>(make_geo<T>(c), c->m64, f[0], f[1], f[2], f[3], f[11], f[4],
                                                            f[5], f[6], f[7], f[8], f[9],
                                                            c->cfg.LES_type == CH3D_LES_MLP ? c->sgs_f : nullptr, c->sc);
  return cudaGetLastError();
}
cudaError_t launch_rhs_les(ch3d_ctx* c) { return c->fp32 ? rhs_les_t<float>(c) : rhs_les_t<double>(c); }

template <class T> static cudaError_t uhat_les_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  HelmCoef hc;
  const double* M = c->met64;
  const int L = c->ny + 3;
  hc.ap2p = M + 7 * L; hc.ac2p = M + 8 * L; hc.am2p = M + 9 * L;
  hc.ap2cForCN = M + 14 * L; hc.am2cForCN = M + 15 * L;
  const int ncol = c->nx * c->nz;
  // the tiled kernel while its shared memory (4 x 16 x ny doubles) fits
  const size_t tsm = (size_t)4 * kUhatTileCols * c->ny * sizeof(double);
  if (tsm <= kUhatTileSmemMax) {
    static PerDevice attr;  // per precision (template instance)
    cudaError_t e = once_per_device(attr, c->device, [] {
      return cudaFuncSetAttribute(k_uhat_les_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUhatTileSmemMax);
    });
    if (e != cudaSuccess) return e;
    k_uhat_les_tile<T><<<dim3((ncol + kUhatTileCols - 1) / kUhatTileCols, 3), 128, tsm, c->stream>>>(
        make_geo<T>(c), hc, f[11], f[0], f[1], f[2], f[7], f[8], f[9], f[12], f[13], f[14], c->sc);
    return cudaGetLastError();
  }
  k_uhat_les<T><<<dim3((ncol + 127) / 128, 3), 128, 0, c->stream>>>(make_geo<T>(c), hc, f[11], f[0], f[1], f[2], f[7],
                                                                    f[8], f[9], f[12], f[13], f[14], c->sc);
  return cudaGetLastError();
}
cudaError_t launch_uhat_les(ch3d_ctx* c) { return c->fp32 ? uhat_les_t<float>(c) : uhat_les_t<double>(c); }

}  // namespace ch3d
